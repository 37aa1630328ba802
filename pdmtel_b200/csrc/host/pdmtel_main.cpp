// pdmtel_run: non-interactive driver in place of the reference's console
// main (main.cpp:16-93).
//   pdmtel_run <working folder> [dynamic|static] [--fp32c]
#include <cstdio>
#include <cstring>
#include <string>

#include "pdDataManager.h"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <working folder> [dynamic|static] [--fp32c]\n", argv[0]);
        return 2;
    }
    std::string mode = argc > 2 ? argv[2] : "dynamic";
    int prec = PD_PREC_FP64;
    for (int k = 2; k < argc; ++k)
        if (!std::strcmp(argv[k], "--fp32c")) prec = PD_PREC_FP32C;
    pdh::pdDataManager dat;
    int rc = dat.SetWkDir(argv[1]);
    if (rc == PD_OK) rc = pdh::pdSolve::InitialProblem(dat);
    if (rc == PD_OK) rc = dat.SetPrecision(prec);
    if (rc == PD_OK) rc = mode == "static" ? pdh::pdSolve::SolveStatic(dat, prec) : pdh::pdSolve::SolveDynamic(dat);
    if (rc != PD_OK) {
        std::fprintf(stderr, "pdmtel_run: %s (status %d)\n", dat.LastError().c_str(), rc);
        return 1;
    }
    std::printf("nodes %d, bonds %lld, done\n", dat.GetNumNode(), (long long)dat.GetNumBond());
    return 0;
}
