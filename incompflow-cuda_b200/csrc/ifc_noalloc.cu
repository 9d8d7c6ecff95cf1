// ifc_noalloc.cu -- red-black Gauss-Seidel sweeps that allocate no device memory.
//
// The solver handle (ifc_create) allocates its fields and a small scratch area
// (FP64 per-block partial sums and the control block of the deterministic norm
// reduction) with cudaMalloc.  Some callers cannot allocate: a host program that
// reserved the whole device for its own memory pool at start-up (as coupled
// simulation frameworks do) has no room for the handle's buffers, and a caller
// that runs the sweep inside a time-critical loop cannot afford cudaFree, which
// synchronises the whole device.  For them ifc_rb_sweeps_noalloc runs the same
// sweep kernel as ifc_sweep on buffers the caller owns, and takes its scratch
// from a fixed array compiled into this library.
#include <cstdio>

#include "ifc.h"
#include "ifc_kernels.cuh"

namespace {

using namespace ifc;

// Largest number of blocks one sweep launch uses; the grid-stride kernel covers
// any grid size with at most this many blocks.
constexpr int kNoAllocMaxBlocks = 1024;
// Largest grid the entry point accepts (cells); keeps every cell index, and
// cell + N*slot for the 7 coefficient planes, inside 32-bit arithmetic.
constexpr long long kNoAllocMaxCells = 1LL << 26;
constexpr size_t kCtlBytes = (sizeof(Ctl) + 255) / 256 * 256;
constexpr size_t kPartialBytes = (size_t)kNoAllocMaxBlocks * kMaxReduce * sizeof(double);
// 152 KB in every process that loads this library, on every GPU it touches,
// held until the process exits.
constexpr size_t kScratchBytes = kCtlBytes + kPartialBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch on the current device.  It is looked up
// on every call (a few microseconds next to two kernel launches and a stream
// synchronisation) rather than cached: after cudaDeviceReset, or when the
// primary context is torn down and recreated, the module is loaded again and
// the array may sit at another address.
int scratch_for_current_device(void **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return IFC_CUDA_ERROR;
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return IFC_CUDA_ERROR;
    *out = p;
    return IFC_OK;
}

template <typename T, int DIM>
int run(int nx, int ny, int nz, const void *coef, const void *src, void *phi, double relax, int n,
        double *sq_norms, cudaStream_t stream, unsigned char *scratch)
{
    Ctl *ctl = reinterpret_cast<Ctl *>(scratch);
    double *partials = reinterpret_cast<double *>(scratch + kCtlBytes);
    Params<T> P;
    memset(&P, 0, sizeof(P));
    P.g.dim = DIM;
    P.g.nx = nx;
    P.g.ny = ny;
    P.g.nz = DIM == 2 ? 1 : nz;
    P.g.N = nx * ny * P.g.nz;
    for (int q = 0; q < 4; ++q) {
        P.g.relax[q] = (T)relax;
        P.g.tol[q] = 0.0;  // no inner early exit: exactly n sweeps
    }
    // The control block must start from zero (arrival counter, stop flag).
    if (cudaMemsetAsync(ctl, 0, sizeof(Ctl), stream) != cudaSuccess) return IFC_CUDA_ERROR;
    SweepArgs<T, 1> A;
    A.coef = static_cast<const T *>(coef);
    A.phi[0] = static_cast<T *>(phi);
    A.old[0] = static_cast<T *>(phi);
    A.src[0] = static_cast<const T *>(src);
    A.eq[0] = EQ_U;
    A.active[0] = 1;
    const long long half = (long long)((nx + 1) / 2) * ny * P.g.nz;
    long long blocks = (half + 255) / 256;
    if (blocks < 1) blocks = 1;
    if (blocks > kNoAllocMaxBlocks) blocks = kNoAllocMaxBlocks;
    for (int s = 0; s < n; ++s) {
        A.color = 0;
        k_sweep<T, DIM, 1><<<(int)blocks, 256, 0, stream>>>(P, A, ctl, partials);
        A.color = 1;
        k_sweep<T, DIM, 1><<<(int)blocks, 256, 0, stream>>>(P, A, ctl, partials);
        if (cudaGetLastError() != cudaSuccess) return IFC_CUDA_ERROR;
        if (sq_norms) {
            if (cudaMemcpyAsync(&sq_norms[s], &ctl->last_sweep_sq[EQ_U], sizeof(double), cudaMemcpyDeviceToHost,
                                stream) != cudaSuccess)
                return IFC_CUDA_ERROR;
        }
    }
    return cudaStreamSynchronize(stream) == cudaSuccess ? IFC_OK : IFC_CUDA_ERROR;
}

}  // namespace

extern "C" int ifc_rb_sweeps_noalloc(int dim, int nx, int ny, int nz, int precision, const void *coef,
                                     const void *src, void *phi, double relax, int n_sweeps, double *sq_norms,
                                     void *stream)
{
    if (dim != 2 && dim != 3) return IFC_BAD_ARGUMENT;
    const int nzz = dim == 2 ? 1 : nz;
    if (nx < 1 || ny < 1 || nzz < 1 || n_sweeps < 0) return IFC_BAD_ARGUMENT;
    const long long cells = (long long)nx * ny * nzz;
    if (cells > kNoAllocMaxCells) {
        std::fprintf(stderr,
                     "ifc_rb_sweeps_noalloc: %lld cells exceed the maximum of %lld cells of this entry point; "
                     "use a solver handle (ifc_create) for larger grids\n",
                     cells, kNoAllocMaxCells);
        return IFC_BAD_ARGUMENT;
    }
    if (precision != IFC_FP32 && precision != IFC_FP64) return IFC_BAD_ARGUMENT;
    if (!coef || !src || !phi) return IFC_BAD_ARGUMENT;
    if (n_sweeps == 0) return IFC_OK;
    void *scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != IFC_OK) return rc;
    unsigned char *s = static_cast<unsigned char *>(scratch);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == IFC_FP64) {
        return dim == 2 ? run<double, 2>(nx, ny, nzz, coef, src, phi, relax, n_sweeps, sq_norms, st, s)
                        : run<double, 3>(nx, ny, nzz, coef, src, phi, relax, n_sweeps, sq_norms, st, s);
    }
    return dim == 2 ? run<float, 2>(nx, ny, nzz, coef, src, phi, relax, n_sweeps, sq_norms, st, s)
                    : run<float, 3>(nx, ny, nzz, coef, src, phi, relax, n_sweeps, sq_norms, st, s);
}
