// Solver.h -- drop-in replacement for the reference's Solver class
// (WanZijun271/IncompFlow-CUDA include/Solver.h:8-72), implemented over the C
// ABI of libifc.so (include/ifc.h).
//
// Same public surface: Solver(u, v, w, p, temp), ~Solver(), solve(),
// writeVTK(path).  Like the reference it is configured at compile time by the
// including program's "types.h" (scalar) and "config.h" (the case); the
// constructor turns those constants into an ifc_config.  Differences that a
// caller can see: errors are reported (stderr, and status()), copying is
// disabled (the reference's implicit copy would double-free), and the results
// are also readable through u()/v()/w()/p()/temperature() and stats().
#ifndef SOLVER_H
#define SOLVER_H

#include <cstdio>
#include <filesystem>
#include <string>
#include <vector>

#include "types.h"
#include "config.h"
#include "ifc.h"
#include "ifc_reference_config.h"

class Solver {
public:
    Solver(scalar u = 0.0, scalar v = 0.0, scalar w = 0.0, scalar p = 0.0, scalar temp = 273.0)
        : Solver(ifc_config_from_reference(), u, v, w, p, temp) {}

    explicit Solver(const ifc_config &cfg, scalar u = 0.0, scalar v = 0.0, scalar w = 0.0, scalar p = 0.0,
                    scalar temp = 273.0)
        : cfg_(cfg)
    {
        cfg_.precision = sizeof(scalar) == sizeof(double) ? IFC_FP64 : IFC_FP32;
        const size_t n = (size_t)cfg_.nx * cfg_.ny * (cfg_.dim == 2 ? 1 : cfg_.nz);
        _u.assign(n, u);
        _v.assign(n, v);
        _w.assign(n, w);
        _p.assign(n, p);
        _temp.assign(n, temp);
        status_ = ifc_create(&cfg_, &h_);
        if (status_ == IFC_OK) status_ = ifc_set_uniform(h_, u, v, w, p, temp);
        report("Solver::Solver");
    }

    ~Solver() { ifc_destroy(h_); }

    Solver(const Solver &) = delete;
    Solver &operator=(const Solver &) = delete;

    // src/Solver.cu:153-299: SIMPLE iterations until convergence or
    // numOuterIter, then the fields are copied to the host vectors.
    void solve()
    {
        if (!h_) return;
        status_ = ifc_solve(h_, &stats_);
        if (status_ != IFC_OK && status_ != IFC_NOT_CONVERGED) {
            report("Solver::solve");
            return;
        }
        const size_t bytes = _u.size() * sizeof(scalar);
        int rc = ifc_get_field(h_, IFC_FIELD_U, _u.data(), bytes);
        if (rc == IFC_OK) rc = ifc_get_field(h_, IFC_FIELD_V, _v.data(), bytes);
        if (rc == IFC_OK) rc = ifc_get_field(h_, IFC_FIELD_W, _w.data(), bytes);
        if (rc == IFC_OK) rc = ifc_get_field(h_, IFC_FIELD_P, _p.data(), bytes);
        if (rc == IFC_OK) rc = ifc_get_field(h_, IFC_FIELD_T, _temp.data(), bytes);
        if (rc != IFC_OK) {
            status_ = rc;
            report("Solver::solve (copy-back)");
        }
    }

    // src/Solver.cu:301-367: ASCII RECTILINEAR_GRID under output/.
    void writeVTK(const std::string &filepath) const
    {
        namespace fs = std::filesystem;
        const fs::path path = fs::path("output") / fs::path(filepath);
        std::error_code ec;
        if (!path.parent_path().empty()) fs::create_directories(path.parent_path(), ec);
        const int rc = ifc_write_vtk_host(&cfg_, _u.data(), _v.data(), _w.data(), _p.data(), _temp.data(),
                                          path.string().c_str());
        if (rc != IFC_OK) std::fprintf(stderr, "Failed to open the file: %s\n", path.string().c_str());
    }

    int status() const { return status_; }
    const ifc_stats &stats() const { return stats_; }
    const ifc_config &config() const { return cfg_; }
    const std::vector<scalar> &u() const { return _u; }
    const std::vector<scalar> &v() const { return _v; }
    const std::vector<scalar> &w() const { return _w; }
    const std::vector<scalar> &p() const { return _p; }
    const std::vector<scalar> &temperature() const { return _temp; }

private:
    void report(const char *where) const
    {
        if (status_ != IFC_OK)
            std::fprintf(stderr, "%s: %s (%s)\n", where, ifc_status_string(status_),
                         h_ ? ifc_last_error(h_) : "no handle");
    }

    ifc_config cfg_;
    ifc_solver *h_ = nullptr;
    int status_ = IFC_OK;
    ifc_stats stats_ = {};
    std::vector<scalar> _u, _v, _w, _p, _temp;
};

#endif
