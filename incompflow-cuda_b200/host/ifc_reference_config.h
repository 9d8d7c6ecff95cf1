// ifc_reference_config.h -- builds an ifc_config from a reference-style
// compile-time case: the constexpr names of the reference's include/config.h
// (dim, nx, ny, nz, xmin..zmax, density, dynamicViscosity, velBCs::type/val,
// TempBCs, numOuterIter, nIter_*, relax_*, tol_*; include/config.h:6-81) and
// its `scalar` type (include/types.h:4).  Include it after that config.h.
#ifndef IFC_REFERENCE_CONFIG_H
#define IFC_REFERENCE_CONFIG_H

#include "ifc.h"

#ifndef IFC_SOLVER_CRITERION
// The drop-in Solver keeps the reference's stopping rule (src/Solver.cu:237-268)
// unless the including program selects IFC_CRIT_PER_FIELD.
#define IFC_SOLVER_CRITERION IFC_CRIT_REFERENCE
#endif

#ifndef IFC_SOLVER_CONVECTION
// First-order upwind, the reference's only convection scheme, unless the
// including program selects another IFC_CONV_* value.
#define IFC_SOLVER_CONVECTION IFC_CONV_UPWIND
#endif

inline ifc_config ifc_config_from_reference()
{
    ifc_config c;
    ifc_config_default(&c);
    c.dim = dim;
    c.nx = nx;
    c.ny = ny;
    c.nz = nz;
    c.xmin = xmin; c.xmax = xmax; c.ymin = ymin; c.ymax = ymax; c.zmin = zmin; c.zmax = zmax;
    c.thermal_conductivity = thermalConductivity;
    c.specific_heat_capacity = specificHeatCapacity;
    c.density = density;
    c.dynamic_viscosity = dynamicViscosity;
    for (int f = 0; f < 6; ++f) {
        c.vel_bc_type[f] = velBCs::type[f];
        for (int q = 0; q < 3; ++q) c.vel_bc_val[f][q] = velBCs::val[f][q];
        c.temp_bc_type[f] = TempBCs::type[f];
        c.temp_bc_val[f] = TempBCs::val[f];
    }
    c.num_outer_iter = numOuterIter;
    c.n_iter_u = nIter_u; c.n_iter_v = nIter_v; c.n_iter_w = nIter_w; c.n_iter_p = nIter_p;
    c.relax_u = relax_u; c.relax_v = relax_v; c.relax_w = relax_w; c.relax_p = relax_p;
    c.tol_u = tol_u; c.tol_v = tol_v; c.tol_w = tol_w; c.tol_p = tol_p; c.tol_mass = tol_mass;
    c.precision = sizeof(scalar) == sizeof(double) ? IFC_FP64 : IFC_FP32;
    c.criterion = IFC_SOLVER_CRITERION;
    c.convection_scheme = IFC_SOLVER_CONVECTION;
    c.log_level = 1;
    return c;
}

#endif
