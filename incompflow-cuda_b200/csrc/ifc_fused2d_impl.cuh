// ifc_fused2d_impl.cuh -- host-side launch sequences of the fused 2D kernels.
#pragma once

#include <cstdlib>

namespace ifc {

// Source and destination buffers of one fused pass (u, v or p').
template <typename T>
struct PassBufs {
    const T *in[2];
    T *out[2];
};


template <typename T, int KS>
static int launch_mom_pass(Engine<T> &e, const PassArgs &pa, const PassBufs<T> &b, bool prepare = false)
{
    using S = TileShape2D<T>;
    using R = Region<S::TX, S::TY, 2 * KS>;
    const size_t smem = (size_t)3 * R::NR * sizeof(T);
    auto kern = k_mom_pass2d<T, S::TX, S::TY, KS, S::NT>;
    if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
                               cudaSuccess ? IFC_OK : IFC_CUDA_ERROR;
    const int tiles = ((e.P.g.nx + S::TX - 1) / S::TX) * ((e.P.g.ny + S::TY - 1) / S::TY);
    kern<<<tiles, S::NT, smem, e.stream>>>(e.P, e.f, e.ctl, e.partials, pa, b.in[0], b.in[1], b.out[0], b.out[1]);
    ++e.launches;
    return IFC_OK;
}

template <typename T, int KS>
static int launch_pc_pass(Engine<T> &e, const PassArgs &pa, const PassBufs<T> &b, bool prepare = false)
{
    using S = TileShape2D<T>;
    using R = Region<S::TX, S::TY, 2 * KS>;
    const size_t smem = (size_t)2 * R::NR * sizeof(T);
    auto kern = k_pc_pass2d<T, S::TX, S::TY, KS, S::NT>;
    if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
                               cudaSuccess ? IFC_OK : IFC_CUDA_ERROR;
    const int tiles = ((e.P.g.nx + S::TX - 1) / S::TX) * ((e.P.g.ny + S::TY - 1) / S::TY);
    kern<<<tiles, S::NT, smem, e.stream>>>(e.P, e.f, e.ctl, e.partials, pa, b.in[0], b.out[0]);
    ++e.launches;
    return IFC_OK;
}

// Supported sweeps per pass; other values round down to the nearest one.
static inline int fused_ks(int want)
{
    if (want >= 8) return 8;
    if (want >= 5) return want >= 6 ? 6 : 5;
    if (want >= 4) return 4;
    if (want >= 3) return 3;
    if (want >= 2) return 2;
    return 1;
}

template <typename T>
static int dispatch_mom(Engine<T> &e, int ks, const PassArgs &pa, const PassBufs<T> &b, bool prepare = false)
{
    switch (ks) {
    case 1: return launch_mom_pass<T, 1>(e, pa, b, prepare);
    case 2: return launch_mom_pass<T, 2>(e, pa, b, prepare);
    case 3: return launch_mom_pass<T, 3>(e, pa, b, prepare);
    case 4: return launch_mom_pass<T, 4>(e, pa, b, prepare);
    case 5: return launch_mom_pass<T, 5>(e, pa, b, prepare);
    case 6: return launch_mom_pass<T, 6>(e, pa, b, prepare);
    default: return launch_mom_pass<T, 8>(e, pa, b, prepare);
    }
}

template <typename T>
static int dispatch_pc(Engine<T> &e, int ks, const PassArgs &pa, const PassBufs<T> &b, bool prepare = false)
{
    switch (ks) {
    case 1: return launch_pc_pass<T, 1>(e, pa, b, prepare);
    case 2: return launch_pc_pass<T, 2>(e, pa, b, prepare);
    case 3: return launch_pc_pass<T, 3>(e, pa, b, prepare);
    case 4: return launch_pc_pass<T, 4>(e, pa, b, prepare);
    case 5: return launch_pc_pass<T, 5>(e, pa, b, prepare);
    case 6: return launch_pc_pass<T, 6>(e, pa, b, prepare);
    default: return launch_pc_pass<T, 8>(e, pa, b, prepare);
    }
}


// Raise the dynamic shared-memory limit of the kernels this handle launches
// (done once at creation, outside any stream capture).
template <typename T>
int Engine<T>::prepare_fused()
{
    PassArgs pa = {};
    PassBufs<T> b = {};
    int rc = dispatch_mom<T>(*this, fused_ks(spp_mom), pa, b, true);
    if (rc == IFC_OK) rc = dispatch_pc<T>(*this, fused_ks(spp_p), pa, b, true);
    if (rc != IFC_OK) err = "cudaFuncSetAttribute(MaxDynamicSharedMemorySize) failed";
    return rc;
}

template <typename T>
void Engine<T>::enq_fused_mom()
{
    const int ks = fused_ks(spp_mom);
    const int nu = cfg.n_iter_u, nv = cfg.n_iter_v;
    const int nmax = nu > nv ? nu : nv;
    int npass = (nmax + ks - 1) / ks;
    if (npass < 1) npass = 1;  // the first pass also stores aC
    // A pass stages halos from one buffer and writes its tiles to the other,
    // so no tile reads a neighbour tile's values of the same pass.
    const size_t N = (size_t)P.g.N;
    T *bu[2] = {f.u, f.tmp}, *bv[2] = {f.v, f.tmp + N};
    for (int pass = 0; pass < npass; ++pass) {
        PassArgs pa;
        pa.ns[0] = clamp_sweeps(nu, pass, ks);
        pa.ns[1] = clamp_sweeps(nv, pass, ks);
        pa.ns[2] = 0;
        pa.first = pass == 0;
        PassBufs<T> b = {{bu[pass & 1], bv[pass & 1]}, {bu[(pass + 1) & 1], bv[(pass + 1) & 1]}};
        dispatch_mom<T>(*this, ks, pa, b);
    }
    if (npass & 1) {
        cudaMemcpyAsync(f.u, f.tmp, N * sizeof(T), cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(f.v, f.tmp + N, N * sizeof(T), cudaMemcpyDeviceToDevice, stream);
    }
}

template <typename T>
void Engine<T>::enq_fused_pcorr()
{
    const int ks = fused_ks(spp_p);
    const int np = cfg.n_iter_p;
    if (np == 0) {
        cudaMemsetAsync(f.pc, 0, (size_t)P.g.N * sizeof(T), stream);
        return;
    }
    const int npass = (np + ks - 1) / ks;
    // Ping-pong as for the momentum passes, ordered so that the last pass
    // writes f.pc (the first pass reads nothing: p' starts from 0).
    T *bp[2] = {f.pc, f.tmp + 2 * (size_t)P.g.N};
    for (int pass = 0; pass < npass; ++pass) {
        PassArgs pa;
        pa.ns[0] = clamp_sweeps(np, pass, ks);
        pa.ns[1] = pa.ns[2] = 0;
        pa.first = pass == 0;
        PassBufs<T> b = {{bp[(npass - pass) & 1], nullptr}, {bp[(npass - 1 - pass) & 1], nullptr}};
        dispatch_pc<T>(*this, ks, pa, b);
    }
}

template <typename T>
void Engine<T>::enq_fused_rc()
{
    k_rc_mass2d<T><<<grid(P.g.N), 256, 0, stream>>>(P, f, ctl, partials);
    ++launches;
}

}  // namespace ifc

namespace ifc {

// ---- the persistent single-launch 2D solve (ifc_persist2d.cuh) ----
// launch = false: set the kernel's shared-memory limit and return in *capacity
// the CTAs that can be co-resident.  launch = true: launch it on e.persist_grid
// CTAs (e.persist_mt: several tiles per CTA).
template <typename T, int KS, bool MT>
static int persist_kernel(Engine<T> &e, bool launch, int *capacity)
{
    using S = TileShape2D<T>;
    using R = Region<S::TX, S::TY, 2 * KS>;
    const size_t smem = (size_t)3 * R::NR * sizeof(T);
    auto kern = k_simple2d<T, S::TX, S::TY, KS, S::NT, MT>;
    if (!launch) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return IFC_CUDA_ERROR;
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, S::NT, smem) != cudaSuccess)
            return IFC_CUDA_ERROR;
        *capacity = per_sm * e.nsm;
        return IFC_OK;
    }
    PersistArgs pa;
    pa.n_iter[0] = e.cfg.n_iter_u;
    pa.n_iter[1] = e.cfg.n_iter_v;
    pa.n_iter[2] = 0;
    pa.n_iter[3] = e.cfg.n_iter_p;
    pa.pin = e.pin ? 1 : 0;
    const char *stall = std::getenv("IFC_TEST_STALL_BARRIER");
    pa.stall_test = (stall && stall[0] == '1') ? 1 : 0;
    void *args[] = {&e.P, &e.f, &e.ctl, &e.partials, &e.barrier, &pa};
    return cudaLaunchCooperativeKernel((const void *)kern, dim3(e.persist_grid), dim3(S::NT), args, smem, e.stream) ==
                   cudaSuccess
               ? IFC_OK
               : IFC_CUDA_ERROR;
}

template <typename T, bool MT>
static int persist_dispatch_t(Engine<T> &e, int ks, bool launch, int *capacity)
{
    switch (ks) {
    case 2: return persist_kernel<T, 2, MT>(e, launch, capacity);
    case 3: return persist_kernel<T, 3, MT>(e, launch, capacity);
    case 4: return persist_kernel<T, 4, MT>(e, launch, capacity);
    case 5: return persist_kernel<T, 5, MT>(e, launch, capacity);
    case 6: return persist_kernel<T, 6, MT>(e, launch, capacity);
    case 8: return persist_kernel<T, 8, MT>(e, launch, capacity);
    default: return persist_kernel<T, 10, MT>(e, launch, capacity);
    }
}

template <typename T>
static int persist_dispatch(Engine<T> &e, int ks, bool launch, int *capacity, bool mt)
{
    return mt ? persist_dispatch_t<T, true>(e, ks, launch, capacity)
              : persist_dispatch_t<T, false>(e, ks, launch, capacity);
}

static inline int persist_ks(int want)
{
    if (want >= 10) return 10;
    if (want >= 8) return 8;
    return want < 2 ? 2 : (want > 6 ? 6 : want);
}

// The whole 2D loop as one cooperative launch: one tile per CTA when all tiles'
// CTAs can be co-resident, otherwise (MT) every CTA visits ceil(tiles / CTAs)
// tiles in turn, on the fewest CTAs that give that count (so every CTA has the
// same number of tiles but the last ones).  IFC_PERSIST_OFF=1 keeps the multi-kernel graph; IFC_PERSIST_MAX_CTAS caps the CTAs
// (used by the tests to run the multi-tile form on small grids).
template <typename T>
int Engine<T>::prepare_persist()
{
    persist = false;
    persist_mt = false;
    if (dim != 2 || !fused || cfg.linear_solver != IFC_GAUSS_SEIDEL) return IFC_OK;
    // the residual rule needs the residual pass of the graph form
    if (P.g.criterion == 2) return IFC_OK;
    const char *off = std::getenv("IFC_PERSIST_OFF");  // the multi-kernel graph instead (A/B timing, tests)
    if (off && off[0] == '1') return IFC_OK;
    int coop = 0, dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return IFC_OK;
    const int ks = persist_ks(spp_persist);
    int capacity = 0, capacity_mt = 0;
    if (persist_dispatch<T>(*this, ks, false, &capacity, false) != IFC_OK ||
        persist_dispatch<T>(*this, ks, false, &capacity_mt, true) != IFC_OK) {
        cudaGetLastError();
        return IFC_OK;
    }
    if (const char *cap = std::getenv("IFC_PERSIST_MAX_CTAS")) {
        const int c = std::atoi(cap);
        if (c > 0) {
            capacity = capacity < c ? capacity : c;
            capacity_mt = capacity_mt < c ? capacity_mt : c;
        }
    }
    using S = TileShape2D<T>;
    const int tiles = ((P.g.nx + S::TX - 1) / S::TX) * ((P.g.ny + S::TY - 1) / S::TY);
    if (tiles <= capacity) {
        persist = true;
        persist_grid = tiles;
    } else if (capacity_mt > 0) {
        const int per = (tiles + capacity_mt - 1) / capacity_mt;
        persist = true;
        persist_mt = true;
        persist_grid = (tiles + per - 1) / per;
    }
    return IFC_OK;
}

template <typename T>
int Engine<T>::launch_persist()
{
    if (cudaMemsetAsync(barrier, 0, sizeof(GridBarrier), stream) != cudaSuccess) return IFC_CUDA_ERROR;
    ++launches;
    return persist_dispatch<T>(*this, persist_ks(spp_persist), true, nullptr, persist_mt);
}

}  // namespace ifc
