// ifc_fused2d_impl.cuh -- host-side launch sequences of the fused 2D kernels.
#pragma once

namespace ifc {

// Tile shapes: FP32 tiles are 32 x 16 cells, FP64 tiles 32 x 8 (the staged
// region of an FP64 tile needs twice the shared memory per cell).
template <typename T>
struct TileShape2D {
    static constexpr int TX = 32, TY = sizeof(T) == 4 ? 16 : 8, NT = sizeof(T) == 4 ? 1024 : 512;
};

template <typename T, int KS>
static int launch_mom_pass(Engine<T> &e, const PassArgs &pa, bool prepare = false)
{
    using S = TileShape2D<T>;
    using R = Region<S::TX, S::TY, 2 * KS>;
    const size_t smem = (size_t)3 * R::NR * sizeof(T);
    auto kern = k_mom_pass2d<T, S::TX, S::TY, KS, S::NT>;
    if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
                               cudaSuccess ? IFC_OK : IFC_CUDA_ERROR;
    const int tiles = ((e.P.g.nx + S::TX - 1) / S::TX) * ((e.P.g.ny + S::TY - 1) / S::TY);
    kern<<<tiles, S::NT, smem, e.stream>>>(e.P, e.f, e.ctl, e.partials, pa);
    ++e.launches;
    return IFC_OK;
}

template <typename T, int KS>
static int launch_pc_pass(Engine<T> &e, const PassArgs &pa, bool prepare = false)
{
    using S = TileShape2D<T>;
    using R = Region<S::TX, S::TY, 2 * KS>;
    const size_t smem = (size_t)2 * R::NR * sizeof(T);
    auto kern = k_pc_pass2d<T, S::TX, S::TY, KS, S::NT>;
    if (prepare) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) ==
                               cudaSuccess ? IFC_OK : IFC_CUDA_ERROR;
    const int tiles = ((e.P.g.nx + S::TX - 1) / S::TX) * ((e.P.g.ny + S::TY - 1) / S::TY);
    kern<<<tiles, S::NT, smem, e.stream>>>(e.P, e.f, e.ctl, e.partials, pa);
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
static int dispatch_mom(Engine<T> &e, int ks, const PassArgs &pa, bool prepare = false)
{
    switch (ks) {
    case 1: return launch_mom_pass<T, 1>(e, pa, prepare);
    case 2: return launch_mom_pass<T, 2>(e, pa, prepare);
    case 3: return launch_mom_pass<T, 3>(e, pa, prepare);
    case 4: return launch_mom_pass<T, 4>(e, pa, prepare);
    case 5: return launch_mom_pass<T, 5>(e, pa, prepare);
    case 6: return launch_mom_pass<T, 6>(e, pa, prepare);
    default: return launch_mom_pass<T, 8>(e, pa, prepare);
    }
}

template <typename T>
static int dispatch_pc(Engine<T> &e, int ks, const PassArgs &pa, bool prepare = false)
{
    switch (ks) {
    case 1: return launch_pc_pass<T, 1>(e, pa, prepare);
    case 2: return launch_pc_pass<T, 2>(e, pa, prepare);
    case 3: return launch_pc_pass<T, 3>(e, pa, prepare);
    case 4: return launch_pc_pass<T, 4>(e, pa, prepare);
    case 5: return launch_pc_pass<T, 5>(e, pa, prepare);
    case 6: return launch_pc_pass<T, 6>(e, pa, prepare);
    default: return launch_pc_pass<T, 8>(e, pa, prepare);
    }
}

static inline int clamp_sweeps(int n, int pass, int ks)
{
    int r = n - pass * ks;
    return r < 0 ? 0 : (r > ks ? ks : r);
}

// Raise the dynamic shared-memory limit of the kernels this handle launches
// (done once at creation, outside any stream capture).
template <typename T>
int Engine<T>::prepare_fused()
{
    PassArgs pa = {};
    int rc = dispatch_mom<T>(*this, fused_ks(spp_mom), pa, true);
    if (rc == IFC_OK) rc = dispatch_pc<T>(*this, fused_ks(spp_p), pa, true);
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
    for (int pass = 0; pass < npass; ++pass) {
        PassArgs pa;
        pa.ns[0] = clamp_sweeps(nu, pass, ks);
        pa.ns[1] = clamp_sweeps(nv, pass, ks);
        pa.ns[2] = 0;
        pa.first = pass == 0;
        dispatch_mom<T>(*this, ks, pa);
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
    for (int pass = 0; pass < npass; ++pass) {
        PassArgs pa;
        pa.ns[0] = clamp_sweeps(np, pass, ks);
        pa.ns[1] = pa.ns[2] = 0;
        pa.first = pass == 0;
        dispatch_pc<T>(*this, ks, pa);
    }
}

template <typename T>
void Engine<T>::enq_fused_rc()
{
    k_rc_mass2d<T><<<grid(P.g.N), 256, 0, stream>>>(P, f, ctl, partials);
    ++launches;
}

}  // namespace ifc
