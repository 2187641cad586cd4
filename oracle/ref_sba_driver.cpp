// ref_sba_driver.cpp -- runs the reference's own repeated-nodes BA generator.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target `ref`) together
// with the reference's unmodified sources, where they lie in the cuPPA-Public
// tree, into oracle/_ref/sba_ref.  It does what the reference runner does for
// `-A sba` (src/main.cu:99-104): SerialBA(n, m).generateGraph(conf), which
// prints "Computation Time : <s>" and, with the degree-distribution flag set,
// writes the "Degree,Count" CSV of src/PA/SPA/PAHelper.hpp:69-147.
//
// usage: sba_ref <n> <m> <output-dir> <dd-file-name|->
#include <cstdio>
#include <cstdlib>
#include <string>

#include "PA/SPA/SerialBA.h"
#include "Utility/ExperimentConfiguration.hpp"

int main(int argc, char **argv)
{
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s n m output-dir dd-file|-\n", argv[0]);
        return 2;
    }
    ExperimentConfiguration conf;
    conf._algorithm = "sba";
    conf._n1 = (NodeType)std::atoll(argv[1]);
    conf._x1 = (WeightType)std::atoi(argv[2]);
    conf._outputDir = std::string(argv[3]) + "/";
    const std::string dd = argv[4];
    conf._FLAG_SHOW_DEGREE_DISTRIBUTION = dd != "-";
    conf._distfile1 = dd == "-" ? "degreeDistribution.txt" : dd;

    SerialBA ba(conf._n1, conf._x1);
    ba.generateGraph(conf);
    return 0;
}
