// ifc_common.cuh -- shared device-side types of the B200 SIMPLE solver:
// geometry/parameter block, device field table, the control block that carries
// the SIMPLE loop's state between kernels, and the deterministic FP64 grid
// reduction used for every norm.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ifc {

// Slot order of the coefficient planes, include/constants.h:14-20.
enum { AC = 0, AE = 1, AW = 2, AN = 3, AS = 4, AT = 5, AB = 6 };
// Boundary faces and types, include/constants.h:7-12,32-34.
enum { EAST = 0, WEST = 1, NORTH = 2, SOUTH = 3, TOP = 4, BOTTOM = 5 };
enum { WALL = 0, INLET = 1, OUTLET = 2 };
enum { EQ_U = 0, EQ_V = 1, EQ_W = 2, EQ_P = 3 };

// Indices of the FP64 sums kept in Ctl::sq (one outer iteration).
enum { SQ_P = 0, SQ_U, SQ_V, SQ_W, SQ_UF, SQ_VF, SQ_WF, SQ_MASS, SQ_PCSUM, SQ_COUNT };

constexpr int kLogCap = 256;        // log records kept per solve call
constexpr int kMaxReduce = 16;      // values reduced per kernel

// Geometry and parameters, evaluated in the solver's scalar type exactly as the
// reference's constexpr values (include/constants.h:22-28).
template <typename T>
struct Geo {
    int dim, nx, ny, nz, N;
    T dx, dy, dz, Ax, Ay, Az, rho, mu;
    T relax[4];
    double tol[4];
    double tol_mass;
    int bc[6];
    int closed[6];                  // face pressure = cell pressure (wall or inlet)
    T bcv[6][3];
    const T *inlet;                 // west-face inlet profile (device, ny*nz) or nullptr
    int criterion;                  // 0 reference rule, 1 per-field rule, 2 per field on FP64 residuals
    int conv;                       // convection scheme (ifc_convection.cuh); 0 upwind
};

#ifdef IFC_BOUNDS_CHECK
// Bounds-checked build (make lib_bc): every field array is a view that knows
// its length.  An index outside [0, n) records the index in a device flag and
// is redirected to a scratch slot -- no trap, the context stays usable -- and
// the host returns IFC_BAD_ARGUMENT after the launch sequence.  Pointer
// copies taken from a view (T *x = f.u) are not checked.
static __device__ int g_ifc_bounds_err;
static __device__ unsigned long long g_ifc_bounds_idx;
static __device__ double g_ifc_bounds_sink[64];

template <typename T>
struct Checked {
    T *p;
    long long n;
    __host__ __device__ operator T *() const { return p; }
    // points the view at another buffer of the same length (ping-pong copies)
    __host__ __device__ Checked &operator=(T *q)
    {
        p = q;
        return *this;
    }
    __device__ __forceinline__ T &operator[](long long i) const
    {
        if (i < 0 || i >= n) {
            if (atomicCAS(&g_ifc_bounds_err, 0, 1) == 0) atomicExch(&g_ifc_bounds_idx, (unsigned long long)i);
            return reinterpret_cast<T *>(g_ifc_bounds_sink)[threadIdx.x & 31];
        }
        return p[i];
    }
};
template <typename T>
using FieldArr = Checked<T>;
#else
template <typename T>
using FieldArr = T *;
#endif

template <typename T>
struct Fields {
    FieldArr<T> u, v, w, p, temp, pc;
    FieldArr<T> uf, vf, wf;
    FieldArr<T> ac;                 // momentum diagonal after the boundary fold-in
    FieldArr<T> mc, pcoef;          // materialised coefficient planes (2*dim+1 each)
    FieldArr<T> su, sv, sw, sp;     // momentum sources and p' source (mass imbalance)
    FieldArr<T> tmp;                // scratch copy for Jacobi sweeps (3*N)
    FieldArr<T> rac;                // 1/aC (3D p' sweeps)
    FieldArr<T> sdc;                // deferred-correction sources of u, v, w (dim planes; conv != 0)
};

struct LogRec {
    int it;
    int converged;
    double rel[7];                  // p u v w uf vf wf
    double mass;
};

// Device-resident state of the SIMPLE loop.  Only kernels write it while a
// graph runs; the host reads it after synchronising.
struct Ctl {
    unsigned int counter;           // arrivals for the last-block reduction
    int it;                         // outer iterations done by this handle
    int it_begin;                   // value of `it` when the current call started
    int it_stop;                    // the loop ends when it reaches this value
    int act;                        // 1: stop at convergence, 0: fixed iteration count
    int converged;
    int status;                     // 0 ok, 2 diverged
    int stop[4];                    // inner early-exit flags of this outer iteration
    int sweeps[4];                  // sweeps done in this outer iteration
    int it_sweeps[4];               // sweeps done in the last finished outer iteration
    long long cell_updates;         // relaxed point updates since the last reset
    double inner_max[4];            // largest RMS sweep change of this outer iteration
    double half_sq[4];              // red-half sum of the sweep in progress
    double last_sweep_sq[4];        // sum (d phi)^2 of the last finished sweep
    double sq[SQ_COUNT];            // FP64 sums of this outer iteration
    double norm[8];                 // RMS norms p u v w uf vf wf mass
    double rel[7];
    double maxn[8];                 // running maxima (criterion)
    double res_sq[3];               // FP64 sums of squared momentum residuals (residual rule)
    double rmax[4];                 // running maxima of the u, v, w residual and mass RMS (residual rule)
    int log_n;                      // records written by this call
    int log_level;
    LogRec log[kLogCap];
};

// ---- row-segment work units ------------------------------------------------
// The cell-wise kernels below hand one warp a segment of kRowSeg consecutive
// cells of one x-row (row r = j + ny*k), lanes strided along x: the row and
// segment come from one division per unit instead of per cell, a warp's loads
// are contiguous, and small-ny grids still yield many units.
constexpr int kRowSeg = 128;

__host__ __device__ __forceinline__ int row_units(int nx, int rows) { return rows * ((nx + kRowSeg - 1) / kRowSeg); }

struct RowUnit {
    int r, j, k, i0, i1;  // row, its j and k, cells [i0, i1)
};

__device__ __forceinline__ RowUnit row_unit(int u, int nx, int ny)
{
    const int nseg = (nx + kRowSeg - 1) / kRowSeg;
    RowUnit w;
    w.r = u / nseg;
    w.i0 = (u - w.r * nseg) * kRowSeg;
    w.i1 = min(w.i0 + kRowSeg, nx);
    w.j = w.r % ny;
    w.k = w.r / ny;
    return w;
}

// ---- deterministic FP64 reduction over the whole grid --------------------
// Every block reduces its values, writes one partial per value, and the last
// block to arrive sums all partials in a fixed order.  The result therefore
// does not depend on block scheduling.  Kernels of one stream never overlap,
// so a single arrival counter in Ctl serves every kernel.

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Returns true in every thread of the last block; `out` (shared, NR entries)
// then holds the grid totals.  partials: NR * gridDim.x doubles.
template <int NR>
__device__ bool grid_reduce(double (&v)[NR], double *partials, Ctl *ctl, double *out)
{
    __shared__ double red[32][NR];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        double x = warp_sum(v[r]);
        if (lane == 0) red[warp][r] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            double x = lane < nwarps ? red[lane][r] : 0.0;
            x = warp_sum(x);
            if (lane == 0) partials[(size_t)r * gridDim.x + blockIdx.x] = x;
        }
        if (lane == 0) {
            __threadfence();
            unsigned int ticket = atomicAdd(&ctl->counter, 1u);
            last = (ticket == gridDim.x - 1);
        }
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // All loads first (one round trip to L2 for all values), then the sums.
    double x[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) x[r] = 0.0;
    for (int b0 = 0; b0 < (int)gridDim.x; b0 += blockDim.x) {
        const int b = b0 + threadIdx.x;
        double y[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) y[r] = b < (int)gridDim.x ? __ldcg(&partials[(size_t)r * gridDim.x + b]) : 0.0;
#pragma unroll
        for (int r = 0; r < NR; ++r) x[r] += y[r];
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const double t = warp_sum(x[r]);
        if (lane == 0) red[warp][r] = t;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            double x = lane < nwarps ? red[lane][r] : 0.0;
            x = warp_sum(x);
            if (lane == 0) out[r] = x;
        }
        if (lane == 0) ctl->counter = 0;
    }
    __syncthreads();
    return true;
}

}  // namespace ifc
