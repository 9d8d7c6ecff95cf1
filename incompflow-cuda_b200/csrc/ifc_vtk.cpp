// ifc_vtk.cpp -- VTK RECTILINEAR_GRID writer, byte-compatible with the
// reference's Solver::writeVTK (src/Solver.cu:301-367).
//
// The reference streams every value through std::ostream with the default
// format (6 significant digits, %g style) followed by a space.  This writer
// formats with snprintf("%g") into per-thread buffers and writes them in
// order, so the bytes are the same and large grids are formatted in parallel.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ifc.h"

namespace {

template <typename T>
void append_values(std::string &out, const T *a, const T *b, const T *c, size_t lo, size_t hi)
{
    char buf[64];
    out.reserve(out.size() + (hi - lo) * (c ? 36 : 12));
    for (size_t q = lo; q < hi; ++q) {
        int n = std::snprintf(buf, sizeof(buf), "%g ", (double)a[q]);
        out.append(buf, (size_t)n);
        if (b) {
            n = std::snprintf(buf, sizeof(buf), "%g ", (double)b[q]);
            out.append(buf, (size_t)n);
            n = std::snprintf(buf, sizeof(buf), "%g ", (double)c[q]);
            out.append(buf, (size_t)n);
        }
    }
}

// Formats [0, n) of one data block with several threads, in order.
template <typename T>
bool write_block(FILE *fp, const T *a, const T *b, const T *c, size_t n)
{
    unsigned hw = std::thread::hardware_concurrency();
    size_t nt = std::max<size_t>(1, std::min<size_t>(hw ? hw : 1, n / 65536 + 1));
    nt = std::min<size_t>(nt, 32);
    std::vector<std::string> parts(nt);
    std::vector<std::thread> th;
    for (size_t t = 0; t < nt; ++t) {
        size_t lo = n * t / nt, hi = n * (t + 1) / nt;
        if (nt == 1) append_values(parts[t], a, b, c, lo, hi);
        else th.emplace_back([&parts, t, a, b, c, lo, hi] { append_values(parts[t], a, b, c, lo, hi); });
    }
    for (auto &x : th) x.join();
    for (auto &s : parts)
        if (!s.empty() && std::fwrite(s.data(), 1, s.size(), fp) != s.size()) return false;
    return true;
}

template <typename T>
int write_vtk(const ifc_config *cfg, const T *u, const T *v, const T *w, const T *p, const T *temp,
              const char *path)
{
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->dim == 2 ? 1 : cfg->nz;
    // include/constants.h:22-24 and src/Solver.cu:325-337: coordinates are
    // min + (scalar)i * d evaluated in the scalar type.
    const T xmin = (T)cfg->xmin, ymin = (T)cfg->ymin, zmin = (T)cfg->zmin;
    const T dx = ((T)cfg->xmax - xmin) / (T)nx;
    const T dy = ((T)cfg->ymax - ymin) / (T)ny;
    const T dz = ((T)cfg->zmax - zmin) / (T)nz;
    FILE *fp = std::fopen(path, "wb");
    if (!fp) return IFC_IO_ERROR;
    std::vector<char> iobuf(1 << 20);
    std::setvbuf(fp, iobuf.data(), _IOFBF, iobuf.size());
    const long long ncell = (long long)nx * ny * nz;
    bool ok = true;
    ok = ok && std::fprintf(fp, "# vtk DataFile Version 3.0\nflash 3d grid and solution\nASCII\n"
                                "DATASET RECTILINEAR_GRID\n") > 0;
    ok = ok && std::fprintf(fp, "DIMENSIONS %d %d %d\n", nx + 1, ny + 1, nz + 1) > 0;
    const struct { const char *name; int n; T lo, d; } ax[3] = {
        {"X_COORDINATES", nx, xmin, dx}, {"Y_COORDINATES", ny, ymin, dy}, {"Z_COORDINATES", nz, zmin, dz}};
    for (const auto &A : ax) {
        ok = ok && std::fprintf(fp, "%s %d float\n", A.name, A.n + 1) > 0;
        for (int i = 0; i <= A.n && ok; ++i) {
            const T x = A.lo + (T)i * A.d;
            ok = std::fprintf(fp, "%g ", (double)x) > 0;
        }
        ok = ok && std::fputc('\n', fp) != EOF;
    }
    ok = ok && std::fprintf(fp, "CELL_DATA %lld\nFIELD FieldData 3\n", ncell) > 0;
    ok = ok && std::fprintf(fp, "temperature 1 %lld float\n", ncell) > 0;
    ok = ok && write_block<T>(fp, temp, nullptr, nullptr, (size_t)ncell);
    ok = ok && std::fputc('\n', fp) != EOF;
    ok = ok && std::fprintf(fp, "velocity 3 %lld float\n", ncell) > 0;
    ok = ok && write_block<T>(fp, u, v, w, (size_t)ncell);
    ok = ok && std::fputc('\n', fp) != EOF;
    ok = ok && std::fprintf(fp, "pressure 1 %lld float\n", ncell) > 0;
    ok = ok && write_block<T>(fp, p, nullptr, nullptr, (size_t)ncell);
    if (std::fclose(fp) != 0) ok = false;
    return ok ? IFC_OK : IFC_IO_ERROR;
}

}  // namespace

extern "C" int ifc_write_vtk_host(const ifc_config *cfg, const void *u, const void *v, const void *w,
                                  const void *p, const void *temp, const char *path)
{
    if (!cfg || !u || !v || !w || !p || !temp || !path) return IFC_BAD_ARGUMENT;
    if (ifc_config_check(cfg) != IFC_OK) return IFC_BAD_CONFIG;
    if (cfg->precision == IFC_FP64)
        return write_vtk<double>(cfg, (const double *)u, (const double *)v, (const double *)w,
                                 (const double *)p, (const double *)temp, path);
    return write_vtk<float>(cfg, (const float *)u, (const float *)v, (const float *)w, (const float *)p,
                            (const float *)temp, path);
}
