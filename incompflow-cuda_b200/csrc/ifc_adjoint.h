// ifc_adjoint.h -- host interface between a solver handle's engine and the
// discrete-adjoint driver (ifc_adjoint.cu).  The driver owns its FP64
// buffers and CUDA graphs; the engine passes its fields, stream and FP64
// parameters in.
#pragma once

#include <string>

#include "ifc.h"
#include "ifc_physics.cuh"

namespace ifc {

struct AdjointCtx;

struct AdjointReq {
    int mode;                 // 0: adjoint gradient, 1: one reverse pass
    int objective;            // IFC_OBJ_* (mode 0)
    const double *seed[5];    // mode 0: dJ/du, dJ/dv, dJ/dp (host, or null); mode 1: lambda u v p uf vf
    double *out[5];           // mode 1: G_x^T lambda (host)
    int max_iter;
    double tol;
    double *dtheta;           // host, ny
    double *dmu;              // mode 1
    int pin;                  // the forward iteration removes the mean of p'
};

template <typename T>
int adjoint_run(AdjointCtx *&ctx, const ifc_config &cfg, Params<double> Pd, const Fields<T> &f, const T *inlet,
                cudaStream_t stream, const AdjointReq &rq, ifc_adjoint_result *res, std::string &err);

void adjoint_free(AdjointCtx *ctx);

}  // namespace ifc
