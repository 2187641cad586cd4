// ref_scm_driver.cpp -- runs the reference's own sequential copy model.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target `ref`) together
// with the reference's unmodified sources, where they lie in the cuPPA-Public
// tree, into oracle/_ref/scm_ref.  It does exactly what the reference runner
// does for `-A scm` (src/main.cu:93-98): build an ExperimentConfiguration and
// call SerialCopyModel(n, m, p).generateGraph(conf).  The reference then prints
// "Computation Time : <s>" and, with the degree-distribution flag set, writes the
// "Degree,Count" CSV of src/PA/SPA/PAHelper.hpp:15-67.
//
// usage: scm_ref <n> <m> <p> <output-dir> <dd-file-name|->
#include <cstdio>
#include <cstdlib>
#include <string>

#include "PA/SPA/SerialCopyModel.h"
#include "Utility/ExperimentConfiguration.hpp"

int main(int argc, char **argv)
{
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s n m p output-dir dd-file|-\n", argv[0]);
        return 2;
    }
    ExperimentConfiguration conf;
    conf._algorithm = "scm";
    conf._n1 = (NodeType)std::atoll(argv[1]);
    conf._x1 = (WeightType)std::atoi(argv[2]);
    conf._alpha = std::atof(argv[3]);
    conf._outputDir = std::string(argv[4]) + "/";
    const std::string dd = argv[5];
    // The reference runner never default-initialises this flag (src/main.cu:216);
    // set it explicitly.
    conf._FLAG_SHOW_DEGREE_DISTRIBUTION = dd != "-";
    conf._distfile1 = dd == "-" ? "degreeDistribution.txt" : dd;

    SerialCopyModel scm(conf._n1, (EdgeIndexType)conf._x1, conf._alpha);
    scm.generateGraph(conf);
    return 0;
}
