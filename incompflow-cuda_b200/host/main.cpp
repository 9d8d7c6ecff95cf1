// main.cpp -- command-line driver with the reference's shape (main.cpp:5-17):
// construct the solver with all-zero initial fields, solve, write
// output/test1.vtk and print the elapsed wall time.
#include <chrono>
#include <iostream>

#include "Solver.h"

int main()
{
    const auto start = std::chrono::high_resolution_clock::now();
    Solver solver{0, 0, 0, 0, 0};
    solver.solve();
    solver.writeVTK("test1.vtk");
    const auto end = std::chrono::high_resolution_clock::now();
    const auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(end - start);
    std::cout << "Elapsed time: " << ms.count() << " ms\n";
    return solver.status() == IFC_OK || solver.status() == IFC_NOT_CONVERGED ? 0 : 1;
}
