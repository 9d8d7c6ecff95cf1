// ref_bench.cpp -- times the reference solver through its own public API
// (Solver::Solver, Solver::solve; include/Solver.h:46-52), compiled from the
// reference's unmodified sources with a case written into its config.h by
// build_ref.py.  TEST/BASELINE INFRASTRUCTURE ONLY.
//
//   ref_bench <warmup> <steps> [vtk-name]
// Each step is one Solver::solve() call of numOuterIter outer iterations (the
// generated config sets the tolerances so that no early stop happens unless a
// converged run is requested).  Prints one JSON line with per-step times.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

// The generated case first (see build_ref.py), then the reference's header.
#include "config.h"
#include "Solver.h"

int main(int argc, char **argv)
{
    const int warm = argc > 1 ? std::atoi(argv[1]) : 3;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 10;
    Solver s{0, 0, 0, 0, 0};
    for (int w = 0; w < warm; ++w) s.solve();
    std::vector<double> ms;
    for (int k = 0; k < steps; ++k) {
        auto t0 = std::chrono::steady_clock::now();
        s.solve();
        auto t1 = std::chrono::steady_clock::now();
        ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
    if (argc > 3) s.writeVTK(argv[3]);
    std::printf("{\"outer_per_step\": %d, \"nx\": %d, \"ny\": %d, \"nz\": %d, \"step_ms\": [", numOuterIter, nx, ny, nz);
    for (size_t k = 0; k < ms.size(); ++k) std::printf("%s%.6f", k ? ", " : "", ms[k]);
    std::printf("]}\n");
    return 0;
}
