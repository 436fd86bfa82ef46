// ref_integrand.cpp -- test infrastructure, NOT part of the library.
//
// Runs the REFERENCE's coefficient evaluator, femd::Integrand (include/femd/forms/integrand.hpp,
// read in place from the reference tree; nothing is copied), on one program given in a binary
// file, and writes the values it computes.  Used by tests/golden/make_golden.py to pin the C
// restatement (or_integrand_eval in femd_oracle.c).
//
// Usage: femd_ref_integrand <spec.bin> <out.bin>
//   spec.bin: int32 ninstr, nreg, nconst, ninput, npts, has_xy, has_normal; int32 code[4 ninstr];
//             float64 consts[nconst], then (has_xy) xs[npts], ys[npts], (has_normal) nx[npts],
//             ny[npts], then inputs[ninput][npts]
//   out.bin:  float64 out[npts]; on an error the exception text goes to stderr and the exit
//             status is 3
#include "femd/forms/integrand.hpp"

#include <cstdio>
#include <exception>
#include <fstream>
#include <vector>

int main(int argc, char **argv)
{
    if (argc != 3) { std::fprintf(stderr, "usage: femd_ref_integrand <spec.bin> <out.bin>\n"); return 2; }
    std::ifstream f(argv[1], std::ios::binary);
    if (!f) { std::fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
    int hdr[7];
    f.read(reinterpret_cast<char *>(hdr), sizeof hdr);
    const int ninstr = hdr[0], nreg = hdr[1], nconst = hdr[2], ninput = hdr[3], npts = hdr[4];
    const bool has_xy = hdr[5] != 0, has_normal = hdr[6] != 0;
    std::vector<int> code(4 * static_cast<std::size_t>(ninstr));
    f.read(reinterpret_cast<char *>(code.data()), static_cast<std::streamsize>(code.size() * sizeof(int)));
    auto doubles = [&](std::size_t n) {
        std::vector<double> v(n);
        f.read(reinterpret_cast<char *>(v.data()), static_cast<std::streamsize>(n * sizeof(double)));
        return v;
    };
    std::vector<double> consts = doubles(static_cast<std::size_t>(nconst));
    std::vector<double> xs, ys, nx, ny;
    if (has_xy) { xs = doubles(npts); ys = doubles(npts); }
    if (has_normal) { nx = doubles(npts); ny = doubles(npts); }
    std::vector<std::vector<double>> in(static_cast<std::size_t>(ninput));
    std::vector<const double *> ptrs;
    for (auto &v : in) { v = doubles(npts); ptrs.push_back(v.data()); }
    if (!f) { std::fprintf(stderr, "short read on %s\n", argv[1]); return 2; }
    std::vector<double> out(static_cast<std::size_t>(npts));
    try
    {
        femd::Integrand prog(code, nreg, nconst, ninput);
        prog.evaluate(static_cast<std::size_t>(npts), has_xy ? xs.data() : nullptr, has_xy ? ys.data() : nullptr,
                      has_normal ? nx.data() : nullptr, has_normal ? ny.data() : nullptr, ptrs, consts, out.data());
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "%s\n", e.what());
        return 3;
    }
    std::ofstream o(argv[2], std::ios::binary);
    o.write(reinterpret_cast<const char *>(out.data()), static_cast<std::streamsize>(out.size() * sizeof(double)));
    return 0;
}
