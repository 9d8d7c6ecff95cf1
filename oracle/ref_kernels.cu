// ref_kernels.cu -- runs the reference's own kernels (include/kernels.cuh of
// WanZijun271/IncompFlow-CUDA, compiled with a generated config.h by
// build_ref.py) on seeded inputs and writes their outputs, to pin the CPU
// oracle against the reference.  TEST INFRASTRUCTURE ONLY; 2D cases only.
//
//   ref_kernels <in_dir> <out_dir>
// in_dir holds raw float32 arrays u v p uf vf coef pc (coef: 5 planes).  Each
// step starts again from those inputs and launches the reference kernels with
// the launch shapes of src/Solver.cu; boundary kernels run one after another
// (the reference's concurrent streams race on corner cells, defect D9).
#include <cstdio>
#include <string>
#include <vector>

// The generated case first: kernels.cuh includes "config.h" from its own
// directory, which the include guard then skips.
#include "config.h"
#include "kernels.cuh"

static_assert(dim == 2, "the kernel harness covers the 2D build");

namespace {

const int N = nx * ny * nz;
const int NUF = (nx + 1) * ny * nz, NVF = nx * (ny + 1) * nz, NC = N * (1 + 2 * dim);

std::vector<float> load(const std::string &dir, const char *name, size_t n)
{
    std::vector<float> v(n);
    FILE *f = std::fopen((dir + "/" + name + ".bin").c_str(), "rb");
    if (!f || std::fread(v.data(), sizeof(float), n, f) != n) {
        std::fprintf(stderr, "cannot read %s/%s.bin\n", dir.c_str(), name);
        std::exit(2);
    }
    std::fclose(f);
    return v;
}

void save(const std::string &dir, const std::string &name, const float *d, size_t n)
{
    std::vector<float> h(n);
    cudaMemcpy(h.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost);
    FILE *f = std::fopen((dir + "/" + name + ".bin").c_str(), "wb");
    std::fwrite(h.data(), sizeof(float), n, f);
    std::fclose(f);
}

struct Dev {
    float *u, *v, *w, *p, *pc, *uf, *vf, *wf, *coef, *vcoef, *wcoef, *pcoef, *su, *sv, *sw, *sp, *norm, *f0;
};

void upload(float *d, const std::vector<float> &h) { cudaMemcpy(d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice); }

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    const std::string in = argv[1], out = argv[2];
    const auto u = load(in, "u", N), v = load(in, "v", N), p = load(in, "p", N), pc = load(in, "pc", N);
    const auto uf = load(in, "uf", NUF), vf = load(in, "vf", NVF), coef = load(in, "coef", NC);
    Dev d;
    float **all[] = {&d.u, &d.v, &d.w, &d.p, &d.pc, &d.su, &d.sv, &d.sw, &d.sp, &d.f0};
    for (auto q : all) cudaMalloc(q, N * sizeof(float));
    cudaMalloc(&d.uf, NUF * sizeof(float));
    cudaMalloc(&d.vf, NVF * sizeof(float));
    cudaMalloc(&d.wf, N * 2 * sizeof(float));
    cudaMalloc(&d.coef, NC * sizeof(float));
    cudaMalloc(&d.vcoef, NC * sizeof(float));
    cudaMalloc(&d.wcoef, NC * sizeof(float));
    cudaMalloc(&d.pcoef, NC * sizeof(float));
    cudaMalloc(&d.norm, sizeof(float));
    auto reset = [&]() {
        upload(d.u, u); upload(d.v, v); upload(d.p, p); upload(d.pc, pc);
        upload(d.uf, uf); upload(d.vf, vf); upload(d.coef, coef); upload(d.vcoef, coef);
        cudaMemset(d.w, 0, N * sizeof(float));
        cudaMemset(d.wf, 0, N * 2 * sizeof(float));
        cudaMemset(d.su, 0, N * sizeof(float)); cudaMemset(d.sv, 0, N * sizeof(float));
        cudaMemset(d.sp, 0, N * sizeof(float)); cudaMemset(d.pcoef, 0, NC * sizeof(float));
        cudaMemset(d.norm, 0, sizeof(float));
    };
    const dim3 tb(32, 32, 1), tb1(1024, 1, 1);
    auto grid = [&](int x, int y) { return dim3((x + 31) / 32, (y + 31) / 32, 1); };
    const dim3 gW((ny + 1023) / 1024, 1, 1), gS((nx + 1023) / 1024, 1, 1);

    // kernels.cuh:10-95: face init (src/Solver.cu:384-392) then face BCs (:426-444)
    reset();
    initFaceVelKernel<xDir><<<grid(nx - 1, ny), tb>>>(d.u, d.uf);
    initFaceVelKernel<yDir><<<grid(nx, ny - 1), tb>>>(d.v, d.vf);
    applyBCsToFaceVelKernel<west, velBCs::type[west]><<<gW, tb1>>>(d.uf, d.u, velBCs::val[west][0]);
    applyBCsToFaceVelKernel<east, velBCs::type[east]><<<gW, tb1>>>(d.uf, d.u, velBCs::val[east][0]);
    applyBCsToFaceVelKernel<south, velBCs::type[south]><<<gS, tb1>>>(d.vf, d.v, velBCs::val[south][1]);
    applyBCsToFaceVelKernel<north, velBCs::type[north]><<<gS, tb1>>>(d.vf, d.v, velBCs::val[north][1]);
    cudaDeviceSynchronize();
    save(out, "faces_uf", d.uf, NUF);
    save(out, "faces_vf", d.vf, NVF);

    // kernels.cuh:97-334: coefficients, sources, boundary fold-in (src/Solver.cu:167-175)
    reset();
    calcMomLinkCoefKernel<<<grid(nx, ny), tb>>>(d.coef, d.uf, d.vf, d.wf);
    calcInteriorMomSrcTermKernel<xDir><<<grid(nx - 2, ny), tb>>>(d.su, d.p);
    calcInteriorMomSrcTermKernel<yDir><<<grid(nx, ny - 2), tb>>>(d.sv, d.p);
    calcBCMomSrcTermKernel<west, velBCs::type[west]><<<gW, tb1>>>(d.su, d.p);
    calcBCMomSrcTermKernel<east, velBCs::type[east]><<<gW, tb1>>>(d.su, d.p);
    calcBCMomSrcTermKernel<south, velBCs::type[south]><<<gS, tb1>>>(d.sv, d.p);
    calcBCMomSrcTermKernel<north, velBCs::type[north]><<<gS, tb1>>>(d.sv, d.p);
    cudaDeviceSynchronize();
    save(out, "mom_coef_raw", d.coef, NC);
    cudaMemcpy(d.vcoef, d.coef, NC * sizeof(float), cudaMemcpyDeviceToDevice);
    applyBCsToMomEqKernel<east, velBCs::type[east]><<<gW, tb1>>>(d.coef, d.vcoef, d.wcoef, d.su, d.sv, d.sw,
        velBCs::val[east][0], velBCs::val[east][1], velBCs::val[east][2]);
    cudaDeviceSynchronize();
    applyBCsToMomEqKernel<west, velBCs::type[west]><<<gW, tb1>>>(d.coef, d.vcoef, d.wcoef, d.su, d.sv, d.sw,
        velBCs::val[west][0], velBCs::val[west][1], velBCs::val[west][2]);
    cudaDeviceSynchronize();
    applyBCsToMomEqKernel<north, velBCs::type[north]><<<gS, tb1>>>(d.coef, d.vcoef, d.wcoef, d.su, d.sv, d.sw,
        velBCs::val[north][0], velBCs::val[north][1], velBCs::val[north][2]);
    cudaDeviceSynchronize();
    applyBCsToMomEqKernel<south, velBCs::type[south]><<<gS, tb1>>>(d.coef, d.vcoef, d.wcoef, d.su, d.sv, d.sw,
        velBCs::val[south][0], velBCs::val[south][1], velBCs::val[south][2]);
    cudaDeviceSynchronize();
    save(out, "mom_coef", d.coef, NC);
    save(out, "mom_vcoef", d.vcoef, NC);
    save(out, "mom_src_u", d.su, N);
    save(out, "mom_src_v", d.sv, N);

    // kernels.cuh:845-924: one Jacobi sweep of u on the folded coefficients
    // (deterministic, unlike the in-place Gauss-Seidel kernel); the field
    // ping-pong of src/Solver.cu:894-901 done explicitly.
    cudaMemcpy(d.f0, d.u, N * sizeof(float), cudaMemcpyDeviceToDevice);
    pointJacobiIterateKernel<<<grid(nx, ny), tb, sizeof(float) * 1024>>>(d.u, d.f0, d.coef, d.su, d.norm, relax_u);
    cudaDeviceSynchronize();
    save(out, "jacobi_u", d.u, N);

    // kernels.cuh:336-500: Rhie-Chow on the seeded u, v, p and coef (aC plane)
    reset();
    interiorRhieChowInterpolateKernel<xDir><<<grid(nx - 3, ny), tb>>>(d.uf, d.u, d.coef, d.p);
    interiorRhieChowInterpolateKernel<yDir><<<grid(nx, ny - 3), tb>>>(d.vf, d.v, d.coef, d.p);
    bcRhieChowInterpolateKernel<west, velBCs::type[west]><<<gW, tb1>>>(d.uf, d.u, d.coef, d.p);
    bcRhieChowInterpolateKernel<east, velBCs::type[east]><<<gW, tb1>>>(d.uf, d.u, d.coef, d.p);
    bcRhieChowInterpolateKernel<south, velBCs::type[south]><<<gS, tb1>>>(d.vf, d.v, d.coef, d.p);
    bcRhieChowInterpolateKernel<north, velBCs::type[north]><<<gS, tb1>>>(d.vf, d.v, d.coef, d.p);
    cudaDeviceSynchronize();
    save(out, "rc_uf", d.uf, NUF);
    save(out, "rc_vf", d.vf, NVF);

    // kernels.cuh:502-581: p' links from the seeded aC plane; p' source from the seeded faces
    reset();
    calcPresCorrLinkCoefKernel<<<grid(nx, ny), tb>>>(d.pcoef, d.coef, d.coef, d.coef);
    calcPresCorrSrcTermKernel<<<grid(nx, ny), tb, sizeof(float) * 1024>>>(d.sp, d.uf, d.vf, d.wf, d.norm);
    cudaDeviceSynchronize();
    save(out, "pcorr_coef", d.pcoef, NC);
    save(out, "pcorr_src", d.sp, N);

    // kernels.cuh:583-843: corrections from the seeded p' and aC plane
    reset();
    updatePresKernel<<<grid(nx, ny), tb, sizeof(float) * 1024>>>(d.p, d.pc, d.norm, relax_p);
    updateInteriorVelKernel<xDir><<<grid(nx - 2, ny), tb, sizeof(float) * 1024>>>(d.u, d.coef, d.pc, d.norm, relax_u);
    updateInteriorVelKernel<yDir><<<grid(nx, ny - 2), tb, sizeof(float) * 1024>>>(d.v, d.coef, d.pc, d.norm, relax_v);
    updateFaceVelKernel<xDir><<<grid(nx - 1, ny), tb, sizeof(float) * 1024>>>(d.uf, d.coef, d.pc, d.norm, relax_u);
    updateFaceVelKernel<yDir><<<grid(nx, ny - 1), tb, sizeof(float) * 1024>>>(d.vf, d.coef, d.pc, d.norm, relax_v);
    updateBCVelKernel<west, velBCs::type[west]><<<gW, tb1, sizeof(float) * 1024>>>(d.u, d.coef, d.pc, d.norm, relax_u);
    updateBCVelKernel<east, velBCs::type[east]><<<gW, tb1, sizeof(float) * 1024>>>(d.u, d.coef, d.pc, d.norm, relax_u);
    updateBCVelKernel<south, velBCs::type[south]><<<gS, tb1, sizeof(float) * 1024>>>(d.v, d.coef, d.pc, d.norm, relax_v);
    updateBCVelKernel<north, velBCs::type[north]><<<gS, tb1, sizeof(float) * 1024>>>(d.v, d.coef, d.pc, d.norm, relax_v);
    cudaDeviceSynchronize();
    save(out, "upd_p", d.p, N);
    save(out, "upd_u", d.u, N);
    save(out, "upd_v", d.v, N);
    save(out, "upd_uf", d.uf, NUF);
    save(out, "upd_vf", d.vf, NVF);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e));
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
