// ifc_vtk.cpp -- VTK RECTILINEAR_GRID writer, byte-compatible with the
// reference's Solver::writeVTK (src/Solver.cu:301-367).
//
// The reference streams every value through std::ostream with the default
// format (6 significant digits, %g style) followed by a space.  This writer
// produces the same bytes with its own formatter (fmt_g6, below; snprintf for
// the cases it cannot decide) into per-thread buffers written in order, so
// large grids are formatted in parallel.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ifc.h"

namespace {

// Exact powers of ten representable in double.
const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                           1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

// snprintf("%g", x) (precision 6, no flags) for finite x, in the C locale:
// 6 significant digits rounded to nearest, %e style when the decimal exponent
// X is < -4 or >= 6, else %f style, trailing zeros and a bare decimal point
// removed.  The 6 digits are x * 10^(5-X) rounded, computed with one double
// multiplication by an exact power of ten; when the product lies within 1e-7
// of a rounding tie (or the exponent needs an inexact power) the exact
// decimal value decides, so this defers to snprintf.  Returns the length.
int fmt_g6(double x, char *out)
{
    if (!std::isfinite(x)) return std::snprintf(out, 32, "%g", x);
    char *o = out;
    if (std::signbit(x)) {
        *o++ = '-';
        x = -x;
    }
    if (x == 0.0) {
        *o++ = '0';
        return (int)(o - out);
    }
    int e2;
    std::frexp(x, &e2);
    int X = (int)std::floor((e2 - 1) * 0.30102999566398120);  // floor(log10(x)), or one below
    if (X + 1 <= 308 && x >= (X + 1 >= 0 && X + 1 <= 22 ? kPow10[X + 1] : std::pow(10.0, X + 1))) ++X;
    const int k = 5 - X;
    if (k < -22 || k > 22) return (int)(o - out) + std::snprintf(o, 32, "%g", x);
    const double m = k >= 0 ? x * kPow10[k] : x / kPow10[-k];
    double fl = std::floor(m);
    const double fr = m - fl;
    if (std::fabs(fr - 0.5) < 1e-7) return (int)(o - out) + std::snprintf(o, 32, "%g", x);
    long long n = (long long)fl + (fr > 0.5 ? 1 : 0);
    if (n < 100000) {  // X was one too high (cannot happen after the check above; be safe)
        return (int)(o - out) + std::snprintf(o, 32, "%g", x);
    }
    if (n >= 1000000) {  // rounded up to the next power of ten
        n /= 10;
        ++X;
    }
    char d[6];
    for (int q = 5; q >= 0; --q) {
        d[q] = (char)('0' + n % 10);
        n /= 10;
    }
    int last = 5;  // last significant digit after removing trailing zeros
    while (last > 0 && d[last] == '0') --last;
    if (X < -4 || X >= 6) {
        *o++ = d[0];
        if (last > 0) {
            *o++ = '.';
            for (int q = 1; q <= last; ++q) *o++ = d[q];
        }
        *o++ = 'e';
        *o++ = X < 0 ? '-' : '+';
        const int ax = X < 0 ? -X : X;
        if (ax >= 100) *o++ = (char)('0' + ax / 100);
        *o++ = (char)('0' + (ax / 10) % 10);
        *o++ = (char)('0' + ax % 10);
    } else if (X >= 0) {
        for (int q = 0; q <= X; ++q) *o++ = d[q];
        if (last > X) {
            *o++ = '.';
            for (int q = X + 1; q <= last; ++q) *o++ = d[q];
        }
    } else {
        *o++ = '0';
        *o++ = '.';
        for (int q = 0; q < -X - 1; ++q) *o++ = '0';
        for (int q = 0; q <= last; ++q) *o++ = d[q];
    }
    return (int)(o - out);
}

template <typename T>
void append_values(std::string &out, const T *a, const T *b, const T *c, size_t lo, size_t hi)
{
    char buf[64];
    out.reserve(out.size() + (hi - lo) * (c ? 36 : 12));
    for (size_t q = lo; q < hi; ++q) {
        int n = fmt_g6((double)a[q], buf);
        buf[n++] = ' ';
        if (b) {
            n += fmt_g6((double)b[q], buf + n);
            buf[n++] = ' ';
            n += fmt_g6((double)c[q], buf + n);
            buf[n++] = ' ';
        }
        out.append(buf, (size_t)n);
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
            char buf[40];
            const int n = fmt_g6((double)x, buf);
            buf[n] = ' ';
            ok = std::fwrite(buf, 1, (size_t)n + 1, fp) == (size_t)n + 1;
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

// ---- legacy VTK BINARY ------------------------------------------------------
// The same file as above with the data blocks in the legacy format's binary
// encoding: big-endian values of the scalar type ("float" for FP32 handles,
// "double" for FP64 handles, so nothing is rounded), each block followed by a
// newline.  Header, coordinates (computed in the scalar type) and FIELD blocks
// are those of the ASCII file.

template <typename T>
void put_be(std::vector<unsigned char> &out, T x)
{
    unsigned char b[sizeof(T)];
    std::memcpy(b, &x, sizeof(T));
    for (int k = (int)sizeof(T) - 1; k >= 0; --k) out.push_back(b[k]);  // the hosts here are little-endian
}

template <typename T>
bool write_be_block(FILE *fp, const T *a, const T *b, const T *c, size_t n)
{
    std::vector<unsigned char> out;
    const size_t chunk = 1 << 16;
    for (size_t lo = 0; lo < n; lo += chunk) {
        const size_t hi = std::min(n, lo + chunk);
        out.clear();
        out.reserve((hi - lo) * sizeof(T) * (c ? 3 : 1));
        for (size_t q = lo; q < hi; ++q) {
            put_be(out, a[q]);
            if (c) {
                put_be(out, b[q]);
                put_be(out, c[q]);
            }
        }
        if (std::fwrite(out.data(), 1, out.size(), fp) != out.size()) return false;
    }
    return std::fputc('\n', fp) != EOF;
}

template <typename T>
int write_vtk_binary(const ifc_config *cfg, const T *u, const T *v, const T *w, const T *p, const T *temp,
                     const char *path)
{
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->dim == 2 ? 1 : cfg->nz;
    const T xmin = (T)cfg->xmin, ymin = (T)cfg->ymin, zmin = (T)cfg->zmin;
    const T dx = ((T)cfg->xmax - xmin) / (T)nx;
    const T dy = ((T)cfg->ymax - ymin) / (T)ny;
    const T dz = ((T)cfg->zmax - zmin) / (T)nz;
    const char *ty = sizeof(T) == 8 ? "double" : "float";
    FILE *fp = std::fopen(path, "wb");
    if (!fp) return IFC_IO_ERROR;
    const long long ncell = (long long)nx * ny * nz;
    bool ok = std::fprintf(fp, "# vtk DataFile Version 3.0\nflash 3d grid and solution\nBINARY\n"
                               "DATASET RECTILINEAR_GRID\n") > 0;
    ok = ok && std::fprintf(fp, "DIMENSIONS %d %d %d\n", nx + 1, ny + 1, nz + 1) > 0;
    const struct { const char *name; int n; T lo, d; } ax[3] = {
        {"X_COORDINATES", nx, xmin, dx}, {"Y_COORDINATES", ny, ymin, dy}, {"Z_COORDINATES", nz, zmin, dz}};
    for (const auto &A : ax) {
        ok = ok && std::fprintf(fp, "%s %d %s\n", A.name, A.n + 1, ty) > 0;
        std::vector<T> x((size_t)A.n + 1);
        for (int i = 0; i <= A.n; ++i) x[i] = A.lo + (T)i * A.d;
        ok = ok && write_be_block<T>(fp, x.data(), nullptr, nullptr, x.size());
    }
    ok = ok && std::fprintf(fp, "CELL_DATA %lld\nFIELD FieldData 3\n", ncell) > 0;
    ok = ok && std::fprintf(fp, "temperature 1 %lld %s\n", ncell, ty) > 0;
    ok = ok && write_be_block<T>(fp, temp, nullptr, nullptr, (size_t)ncell);
    ok = ok && std::fprintf(fp, "velocity 3 %lld %s\n", ncell, ty) > 0;
    ok = ok && write_be_block<T>(fp, u, v, w, (size_t)ncell);
    ok = ok && std::fprintf(fp, "pressure 1 %lld %s\n", ncell, ty) > 0;
    ok = ok && write_be_block<T>(fp, p, nullptr, nullptr, (size_t)ncell);
    if (std::fclose(fp) != 0) ok = false;
    return ok ? IFC_OK : IFC_IO_ERROR;
}

}  // namespace

extern "C" int ifc_write_vtk_binary_host(const ifc_config *cfg, const void *u, const void *v, const void *w,
                                         const void *p, const void *temp, const char *path)
{
    if (!cfg || !u || !v || !w || !p || !temp || !path) return IFC_BAD_ARGUMENT;
    if (ifc_config_check(cfg) != IFC_OK) return IFC_BAD_CONFIG;
    if (cfg->precision == IFC_FP64)
        return write_vtk_binary<double>(cfg, (const double *)u, (const double *)v, (const double *)w,
                                        (const double *)p, (const double *)temp, path);
    return write_vtk_binary<float>(cfg, (const float *)u, (const float *)v, (const float *)w, (const float *)p,
                                   (const float *)temp, path);
}

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
