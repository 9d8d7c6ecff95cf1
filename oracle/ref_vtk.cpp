// ref_vtk.cpp -- writes a VTK file with the reference's own Solver::writeVTK
// (src/Solver.cu:301-367) from seeded fields, so the library's writer can be
// compared with it byte for byte.  TEST INFRASTRUCTURE ONLY; built by
// build_ref.py with a generated config.h per case.
//
//   ref_vtk <in_dir> <vtk-name>
// in_dir holds raw float32 arrays u v w p T of nx*ny*nz cells.  The file goes
// to output/<vtk-name> under the working directory, as the reference writes it.
//
// writeVTK reads the Solver's private host vectors (include/Solver.h:10-14),
// which the reference fills only from the device after solve(); the harness
// opens the class's private section to fill them directly.  The standard
// headers are included first so that the redefinition touches Solver.h only.
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "config.h"
#define private public
#include "Solver.h"
#undef private

static std::vector<scalar> load(const std::string &dir, const char *name, size_t n)
{
    std::vector<float> v(n);
    FILE *f = std::fopen((dir + "/" + name + ".bin").c_str(), "rb");
    if (!f || std::fread(v.data(), sizeof(float), n, f) != n) {
        std::fprintf(stderr, "cannot read %s/%s.bin\n", dir.c_str(), name);
        std::exit(2);
    }
    std::fclose(f);
    return std::vector<scalar>(v.begin(), v.end());
}

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    const std::string in = argv[1];
    const size_t n = (size_t)nx * ny * nz;
    Solver s{0, 0, 0, 0, 0};
    s._u = load(in, "u", n);
    s._v = load(in, "v", n);
    s._w = load(in, "w", n);
    s._p = load(in, "p", n);
    s._temp = load(in, "T", n);
    s.writeVTK(argv[2]);
    return 0;
}
