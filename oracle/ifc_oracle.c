/*
 * ifc_oracle.c -- instantiates the CPU oracle (TEST INFRASTRUCTURE ONLY) in
 * float and double.  Build with -ffp-contract=off so that every operation is
 * rounded as written; see ifc_oracle.h for scope and deviations.
 */
#include "ifc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define T float
#define S f
#include "ifc_oracle_impl.h"
#undef T
#undef S

#define T double
#define S d
#include "ifc_oracle_impl.h"
#undef T
#undef S

/* Reverse pass of one outer iteration (FP64, 2D), see ifc_adjoint_impl.h. */
#include "ifc_adjoint_impl.h"

/* Continue a solve from loaded fields: outer iteration `it` > 0 skips the
 * face initialisation of the first iteration (include/kernels.cuh:10-45). */
void orc_set_iteration_count_f(orc_state_f *s, int it) { s->it = it; }
void orc_set_iteration_count_d(orc_state_d *s, int it) { s->it = it; }
