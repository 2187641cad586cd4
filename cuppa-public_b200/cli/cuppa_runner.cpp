// cuppa_runner -- command-line front end with the reference runner's options
// (src/main.cu:123-236, parseExperiments; dispatch at src/main.cu:91-121).
//
//   cuppa_runner -A cuppa -n 100000 -x 4 -a 0.5 [--seed 42] [--id-bits 32]
//                [--seed-mode clique|star] [-b blocks] [-t threads] [-s stages]
//                [--show-dd 1 --dd-filename dd.csv] [-o outdir]
//                [--out edges.txt --format text|binary] [--csr] [--layout pairs|slots]
//
// -A cuppa and -A cuppa-adaptive both run the copy model (-s is accepted and
// ignored: there are no stages); -A scm is the same model with the reference's
// star seed (src/PA/SPA/SerialCopyModel3.cpp); -A sba is the repeated-nodes
// Barabasi-Albert model (src/PA/SPA/SerialBA.cpp), star seed, -a ignored.
// Prints "Computation Time: <s>" like the reference (src/PA/cuPPA/cuPPA_1.cu:511)
// plus the device counters.
// --layout slots keeps only the targets on the device (half the bytes; --out and
// --show-dd work on it, --csr does not).  Errors are reported with their
// pa_strerror text and exit status 1.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "cuppa_pa.h"

namespace {

void usage()
{
    std::fprintf(stderr,
                 "usage: cuppa_runner -A cuppa|cuppa-adaptive|scm|sba -n N -x M -a P [--seed S]\n"
                 "       [--id-bits 32|64] [--seed-mode clique|star] [-b B] [-t T] [-s S]\n"
                 "       [--show-dd 0|1] [--dd-filename F] [-o DIR] [--out FILE]\n"
                 "       [--format text|binary] [--csr] [--layout pairs|slots]\n");
}

int fail(const char *what, int rc)
{
    std::fprintf(stderr, "%s: %s (status %d, cuda %d)\n", what, pa_strerror(rc), rc,
                 pa_last_cuda_error());
    return 1;
}

}  // namespace

int main(int argc, char **argv)
{
    pa_params prm;
    pa_params_init(&prm);
    std::string algo = "cuppa", outdir = "./", ddfile = "degreeDistribution.txt", out, format = "text";
    bool show_dd = false, csr = false, seed_given = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() -> const char * {
            if (i + 1 >= argc) {
                usage();
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "-A" || a == "--algorithm") algo = val();
        else if (a == "-n" || a == "--n1") prm.n = std::strtoull(val(), nullptr, 10);
        else if (a == "-x" || a == "--x1") prm.d = (uint32_t)std::strtoul(val(), nullptr, 10);
        else if (a == "-a" || a == "--alpha") prm.p = std::atof(val());
        else if (a == "-b" || a == "--blocks") prm.blocks = (uint32_t)std::strtoul(val(), nullptr, 10);
        else if (a == "-t" || a == "--threads") prm.threads = (uint32_t)std::strtoul(val(), nullptr, 10);
        else if (a == "-s" || a == "--stages" || a == "-w" || a == "--warps") (void)val();
        else if (a == "--seed") prm.seed = std::strtoull(val(), nullptr, 10);
        else if (a == "--id-bits") prm.id_bits = (uint32_t)std::strtoul(val(), nullptr, 10);
        else if (a == "--seed-mode") {
            prm.seed_mode = std::string(val()) == "star" ? PA_SEED_STAR_REF : PA_SEED_CLIQUE;
            seed_given = true;
        }
        else if (a == "--show-dd") show_dd = std::atoi(val()) != 0;
        else if (a == "--dd-filename") ddfile = val();
        else if (a == "-o" || a == "--output") outdir = val();
        else if (a == "--out") out = val();
        else if (a == "--format") format = val();
        else if (a == "--csr") csr = true;
        else if (a == "--layout") prm.layout = std::string(val()) == "slots" ? PA_LAYOUT_SLOTS : PA_LAYOUT_PAIRS;
        else if (a == "-h" || a == "--help") { usage(); return 0; }
        else { usage(); return 2; }
    }
    if (algo == "scm" || algo == "sba") {
        if (!seed_given) prm.seed_mode = PA_SEED_STAR_REF;
        if (algo == "sba") prm.model = PA_MODEL_BA;
    } else if (algo != "cuppa" && algo != "cuppa-adaptive") {
        std::fprintf(stderr, "only -A cuppa / cuppa-adaptive / scm / sba are provided here\n");
        return 2;
    }
    if (prm.threads != 0 && prm.threads != 256) prm.threads = 0;   // advisory, as -b

    std::printf("Method:\t%s\tN:\t%llu\tM:\t%u\ta:\t%f\tseed:\t%llu\tid bits:\t%u\n", algo.c_str(),
                (unsigned long long)prm.n, prm.d, prm.p, (unsigned long long)prm.seed, prm.id_bits);
    pa_graph g;
    int rc = pa_graph_create(&prm, &g);
    if (rc != PA_OK) return fail("pa_graph_create", rc);
    pa_stats st;
    const auto t0 = std::chrono::steady_clock::now();
    rc = pa_graph_generate(&g, nullptr, &st);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != PA_OK) return fail("generation", rc);
    std::printf("Computation Time: %f\n", secs);
    std::printf("Edges: %llu\tretries: %llu\twaits: %llu\tEdges/s: %.3e\n",
                (unsigned long long)g.n_edges, (unsigned long long)st.retries,
                (unsigned long long)st.waits, g.n_edges / secs);
    if (!out.empty()) {
        rc = pa_write_edges(&prm, g.edges, out.c_str(),
                            format == "binary" ? PA_FORMAT_BINARY : PA_FORMAT_TEXT, nullptr);
        if (rc != PA_OK) return fail("pa_write_edges", rc);
    }
    if (show_dd) {
        const std::string path = outdir + "/" + ddfile;
        rc = pa_write_degree_distribution(&prm, g.edges, path.c_str(), nullptr);
        if (rc != PA_OK) return fail("pa_write_degree_distribution", rc);
    }
    if (csr) {
        uint64_t rb, cb, sb;
        rc = pa_csr_bytes(&prm, &rb, &cb, &sb);
        if (rc != PA_OK) return fail("pa_csr_bytes", rc);
        void *rowptr = nullptr, *col = nullptr, *scratch = nullptr;
        if (cudaMalloc(&rowptr, rb) != cudaSuccess || cudaMalloc(&col, cb) != cudaSuccess ||
            cudaMalloc(&scratch, sb) != cudaSuccess)
            return fail("CSR buffers", PA_ERR_OOM);
        const auto c0 = std::chrono::steady_clock::now();
        rc = pa_build_csr(&prm, g.edges, (int64_t *)rowptr, col, scratch, sb, nullptr);
        const double cs = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
        if (rc != PA_OK) return fail("pa_build_csr", rc);
        std::printf("CSR Time: %f\n", cs);
        cudaFree(rowptr);
        cudaFree(col);
        cudaFree(scratch);
    }
    pa_graph_destroy(&g);
    return 0;
}
