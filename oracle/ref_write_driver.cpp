// ref_write_driver.cpp -- times the reference's own edge-list writer.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target `ref`) into
// oracle/_ref/write_ref.  The graph is the oracle's copy model with the
// reference's seed graph (pa_oracle.c, MT_REF draws, the same G[N][M] slot
// array the reference's generators fill); the timed part is the reference's
// PAHelper::writeGraphToDisk (src/PA/SPA/PAHelper.hpp:163-177), unmodified,
// which writes rows u = M..N-1 as "u v" lines through an ofstream.
//
// usage: write_ref <n> <m> <p> <output-file>
//   prints "Write Time : <s>" and "Edges : <count>"
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "PA/SPA/PAHelper.hpp"

extern "C" {
#include "pa_oracle.h"
}

int main(int argc, char **argv)
{
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s n m p output-file\n", argv[0]);
        return 2;
    }
    const uint64_t n = std::strtoull(argv[1], nullptr, 10);
    const uint32_t m = (uint32_t)std::strtoul(argv[2], nullptr, 10);
    const double p = std::atof(argv[3]);
    std::vector<int64_t> G64(n * m);
    if (orc_generate(n, m, p, 5489, ORC_SEED_STAR_REF, ORC_RNG_MT_REF, G64.data(), nullptr) != 0) {
        std::fprintf(stderr, "oracle rejected the parameters\n");
        return 2;
    }
    std::vector<NodeType> G(G64.begin(), G64.end());
    timeval t0, t1;
    gettimeofday(&t0, nullptr);
    PAHelper::writeGraphToDisk(G.data(), (NodeType)n, (EdgeIndexType)m, argv[4]);
    gettimeofday(&t1, nullptr);
    const double s = (t1.tv_sec - t0.tv_sec) + 1e-6 * (t1.tv_usec - t0.tv_usec);
    std::printf("Write Time : %f\nEdges : %llu\n", s, (unsigned long long)((n - m) * m));
    return 0;
}
