// A compile-time case in the reference's config.h format: the 2D channel the
// reference's README documents as its default (512 x 128 cells, water,
// 0.001 m/s inlet on the west face, outlet on the east face, no-slip walls).
#ifndef CONFIG_H
#define CONFIG_H

#include "types.h"

constexpr int dim = 2;
constexpr int nx = 512, ny = 128, nz = 1;
constexpr scalar xmin = -0.0625, xmax = 0.0625;
constexpr scalar ymin = -0.0125, ymax = 0.0125;
constexpr scalar zmin = 0.0, zmax = 1.0;

constexpr scalar thermalConductivity = 0.598;
constexpr scalar specificHeatCapacity = 4186.0;
constexpr scalar density = 998.2;
constexpr scalar dynamicViscosity = 1.002e-3;
constexpr scalar thermalDiffusivity = thermalConductivity / specificHeatCapacity / density;

// face order: east, west, north, south, top, bottom; 0 wall, 1 inlet, 2 outlet
struct velBCs {
    static constexpr int type[6] = {2, 1, 0, 0, 0, 0};
    static constexpr scalar val[6][3] = {{0, 0, 0}, {0.001, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
};
// temperature BCs (0 given temperature, 1 zero gradient): used by the energy
// solve on the converged flow (ifc_solve_energy); Solver::solve() itself solves
// only the flow, as the reference does
struct TempBCs {
    static constexpr int type[6] = {1, 1, 0, 0, 1, 1};
    static constexpr scalar val[6] = {0.0, 0.0, 293.0, 373.0, 0.0, 0.0};
};

constexpr int numOuterIter = 100000;
constexpr int nIter_u = 10, nIter_v = 10, nIter_w = 10, nIter_p = 20;
constexpr scalar relax_u = 0.75, relax_v = 0.75, relax_w = 0.75, relax_p = 0.25;
constexpr scalar tol_u = 1e-4, tol_v = 1e-4, tol_w = 1e-4, tol_p = 1e-6, tol_mass = 1e-11;

#endif
