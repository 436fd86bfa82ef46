// ref_driver.cpp -- test infrastructure, NOT part of the library.
//
// A command-line driver that runs the REFERENCE implementation of FEMd's 2D P_k
// assembly + Jacobi-PCG path, compiled from the reference's own header-only C++
// (include/femd/**.hpp, read in place; nothing is copied).  It calls the same C++
// entry points that fd.form(...).assemble() and A.solver("cg", M="jacobi") reach:
//
//   rectangle_mesh              include/femd/mesh/structured.hpp:338
//   LagrangeSpace2D(m,k,{},true) include/femd/fe/lagrange_space_2d.hpp:32   (bc="dirichlet")
//   Cache2D(V, degree)          include/femd/fe/cache_2d.hpp:67
//   cell_pattern                include/femd/forms/assembly_2d.hpp:36
//   scatter_map_2d              include/femd/forms/assembly_2d.hpp:136
//   assemble_matrix_2d          include/femd/forms/assembly_2d.hpp:219
//   assemble_vector_2d          include/femd/forms/assembly_2d.hpp:173
//   Cache2D::eval_multi         include/femd/fe/cache_2d.hpp:245            (a field f at points)
//   JacobiPreconditioner        include/femd/sparse/precond.hpp:82
//   krylov::cg_jacobi           include/femd/krylov/cg.hpp:296
//   Cache2D(V, degree, {}, true)  include/femd/fe/cache_2d.hpp:126   (exterior facets, ds; --robin)
//   ILU0Preconditioner, SSORPreconditioner (natural ordering), krylov::cg with them
//                               include/femd/sparse/precond.hpp:105-200, krylov/cg.hpp:245   (--pc)
//   SparseCholesky              include/femd/sparse/cholesky.hpp:144        (the FP64 solution oracle)
//   asymmetry                   include/femd/sparse/csr.hpp:632
//
// The quadrature degree of each form is the one python/femd/forms.py:2487-2500 infers
// (restated in degree_* below).  Outputs go to a directory as raw little-endian arrays
// (<name>.bin) plus meta.txt (key value lines).  It is used (1) to generate the golden
// fixtures under tests/golden/ and (2) as the timed CPU baseline (OpenMP build).
//
// Usage:
//   femd_ref <form> <N> <k> <outdir|-> [options]
//     form: poisson_sin   a = c grad.grad,            L = 2 pi^2 sin(pi x) sin(pi y) v
//           helmholtz_sin a = grad.grad + u v,        L = (2 pi^2 sin sin + sin sin) v
//           varcoef_field a = k(x,y) grad.grad,       L = f v, f a P_k field read from --f
//                         k = 1 + 0.5 sin(2 pi x) sin(2 pi y)
//           poisson_vec   a = c grad.grad,            b read from --b (dim entries)
//           heat          M = u v and K = grad.grad (both written), no solve
//   options: --c <value> --tol <t> --f <file> --b <file> --nocg --chol --nodump --pc
//            --free (no Dirichlet elimination) --robin <alpha> (adds alpha u v ds to A and
//            g v ds to b, g = 1 + x y, over every exterior facet; ds degrees 2k and k + 2)
//            --time <reps> --cg-sample <iters> --full-first (the first timed step runs CG to convergence)
#include "femd/mesh/structured.hpp"
#include "femd/fe/lagrange_space_2d.hpp"
#include "femd/fe/cache_2d.hpp"
#include "femd/forms/assembly_2d.hpp"
#include "femd/sparse/csr.hpp"
#include "femd/sparse/precond.hpp"
#include "femd/sparse/cholesky.hpp"
#include "femd/krylov/cg.hpp"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace femd;

static const double PI = 3.141592653589793;

static double now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class T>
static void dump(const std::string &dir, const std::string &name, const std::vector<T> &v)
{
    if (dir == "-") return;
    std::ofstream f(dir + "/" + name + ".bin", std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

template <class T>
static std::vector<T> load(const std::string &path, std::size_t n)
{
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    if (!f) { std::fprintf(stderr, "cannot open %s\n", path.c_str()); std::exit(2); }
    f.read(reinterpret_cast<char *>(v.data()), static_cast<std::streamsize>(n * sizeof(T)));
    if (!f) { std::fprintf(stderr, "short read on %s\n", path.c_str()); std::exit(2); }
    return v;
}

// Quadrature degrees of forms.py:_init_2d (2487-2500): sum of argument degrees
// (k - derivative order) plus the coefficient degree; a non-polynomial coefficient of
// the data counts as kmax + 1 (quad_degree_estimate, forms.py:1481-1501).
static int deg_gradgrad(int k) { return std::max(2 * (k - 1), 1); }
static int deg_helmholtz(int k) { return std::max(std::max(2 * (k - 1), 2 * k), 1); }
static int deg_varcoef(int k) { return std::max(2 * (k - 1) + (k + 1), 1); }
static int deg_rhs_data(int k) { return std::max(k + (k + 1), 1); }
static int deg_rhs_field(int k) { return std::max(2 * k, 1); }
static int deg_mass(int k) { return std::max(2 * k, 1); }

struct Opts {
    std::string form, out;
    int N = 8, k = 1;
    double c = 1.0, tol = 1e-10;
    std::string fpath, bpath;
    bool cg = true, chol = false, dumpall = true;
    int time_reps = 0, cg_sample = 0;
    bool full_first = false;
    bool pc = false;                 // also ILU(0)- and SSOR-preconditioned CG
    bool free_bc = false;            // LagrangeSpace2D(m, k, {}, false)
    double robin = 0.0;              // alpha of alpha u v ds (0: no facet terms)
};

static std::vector<double> const_coeff(const Cache2D &Q, double v)
{
    return std::vector<double>(static_cast<std::size_t>(Q.nent()) * Q.nq(), v);
}

int main(int argc, char **argv)
{
    if (argc < 5) { std::fprintf(stderr, "usage: femd_ref <form> <N> <k> <outdir|-> [options]\n"); return 2; }
    Opts o;
    o.form = argv[1]; o.N = std::atoi(argv[2]); o.k = std::atoi(argv[3]); o.out = argv[4];
    for (int i = 5; i < argc; ++i)
    {
        std::string a = argv[i];
        auto next = [&]() { if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(2); } return std::string(argv[++i]); };
        if (a == "--c") o.c = std::atof(next().c_str());
        else if (a == "--tol") o.tol = std::atof(next().c_str());
        else if (a == "--f") o.fpath = next();
        else if (a == "--b") o.bpath = next();
        else if (a == "--nocg") o.cg = false;
        else if (a == "--chol") o.chol = true;
        else if (a == "--nodump") o.dumpall = false;
        else if (a == "--time") o.time_reps = std::atoi(next().c_str());
        else if (a == "--cg-sample") o.cg_sample = std::atoi(next().c_str());
        else if (a == "--full-first") o.full_first = true;
        else if (a == "--pc") o.pc = true;
        else if (a == "--free") o.free_bc = true;
        else if (a == "--robin") o.robin = std::atof(next().c_str());
        else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); return 2; }
    }
    const std::string &dir = o.out;
    const int N = o.N, k = o.k;
    std::FILE *meta = dir == "-" ? stdout : std::fopen((dir + "/meta.txt").c_str(), "w");
    if (!meta) { std::fprintf(stderr, "cannot write %s/meta.txt\n", dir.c_str()); return 2; }
#ifdef _OPENMP
    std::fprintf(meta, "threads %d\n", omp_get_max_threads());
#else
    std::fprintf(meta, "threads 1\n");
#endif

    // ---- setup: mesh, space (numbering), caches, pattern, scatter map ----------------------
    double t0 = now();
    Mesh2D mesh = rectangle_mesh(0.0, 0.0, 1.0, 1.0, N, N);
    LagrangeSpace2D V(mesh, k, {}, !o.free_bc);
    double t_space = now() - t0;
    int qa, qf = 0;
    bool rhs_data = false, rhs_field = false, rhs_vec = false;
    if (o.form == "poisson_sin") { qa = deg_gradgrad(k); qf = deg_rhs_data(k); rhs_data = true; }
    else if (o.form == "helmholtz_sin") { qa = deg_helmholtz(k); qf = deg_rhs_data(k); rhs_data = true; }
    else if (o.form == "varcoef_field") { qa = deg_varcoef(k); qf = deg_rhs_field(k); rhs_field = true; }
    else if (o.form == "poisson_vec") { qa = deg_gradgrad(k); rhs_vec = true; }
    else if (o.form == "heat") { qa = deg_mass(k); }
    else { std::fprintf(stderr, "unknown form %s\n", o.form.c_str()); return 2; }

    t0 = now();
    Cache2D Qa(V, qa);
    double t_cache = now() - t0;
    t0 = now();
    std::shared_ptr<SparsityPattern> P = cell_pattern(V, V);
    double t_pattern = now() - t0;
    t0 = now();
    std::vector<int> map = scatter_map_2d(Qa, Qa, *P, 0, 0);
    double t_map = now() - t0;
    const int n = V.dim();

    std::fprintf(meta, "N %d\nk %d\nne %d\nnv %d\nnloc %d\ndim %d\nraw_dim %d\nnnz %d\nnq_a %d\nqdeg_a %d\n", N, k,
                 V.ncells(), V.npoints(), V.nloc(), n, V.raw_dim(), P->nnz(), Qa.nq(), qa);
    std::fprintf(meta, "t_space %.6f\nt_cache %.6f\nt_pattern %.6f\nt_map %.6f\n", t_space, t_cache, t_pattern, t_map);

    if (o.dumpall)
    {
        std::vector<double> pts;
        for (int v = 0; v < mesh.npoints(); ++v) { pts.push_back(mesh.point(v).x); pts.push_back(mesh.point(v).y); }
        std::vector<int> tris;
        for (int c = 0; c < mesh.ntriangles(); ++c) for (int i = 0; i < 3; ++i) tris.push_back(mesh.triangle(c)[i]);
        dump(dir, "points", pts);
        dump(dir, "tris", tris);
        dump(dir, "cell_dofs", V.cell_dofs());
        dump(dir, "cell_raw_dofs", V.cell_raw_dofs());
        dump(dir, "indptr", P->indptr);
        dump(dir, "indices", P->indices);
        dump(dir, "scatter_map", map);
        // the reference tabulation and quadrature of Qa (point q: [phi, dphi/dxi, dphi/deta] x nloc)
        std::vector<double> ref;
        const int nl = V.nloc();
        for (int q = 0; q < Qa.nq(); ++q)
        {
            const double *R = Qa.ref(0, q);
            ref.insert(ref.end(), R, R + 3 * nl);
        }
        dump(dir, "ref_tab_a", ref);
        std::vector<double> qx, qy;
        TriangleQuadrature rule(qa);
        for (int q = 0; q < rule.size(); ++q) { qx.push_back(rule.xi(q)); qy.push_back(rule.eta(q)); }
        std::vector<double> qw;
        for (int q = 0; q < rule.size(); ++q) qw.push_back(rule.weight(q));
        dump(dir, "quad_xi_a", qx); dump(dir, "quad_eta_a", qy); dump(dir, "quad_w_a", qw);
        if (o.robin != 0.0)
        {
            // the exterior-facet cache of the ds matrix term: entries (cell, local edge, marker),
            // points, weights, outward normals, and the tabulation per local edge
            Cache2D Fa(V, 2 * k, {}, true);
            std::vector<int> fc, fv;
            for (int e = 0; e < Fa.nent(); ++e) { fc.push_back(Fa.cell(e)); fv.push_back(Fa.variant(e)); }
            dump(dir, "facet_cell", fc);
            dump(dir, "facet_local", fv);
            dump(dir, "facet_marker", Fa.markers());
            dump(dir, "facet_x", Fa.x()); dump(dir, "facet_y", Fa.y()); dump(dir, "facet_w", Fa.weights());
            dump(dir, "facet_nx", Fa.normal_x()); dump(dir, "facet_ny", Fa.normal_y());
            std::vector<double> fr;
            for (int v = 0; v < 3; ++v)
                for (int q = 0; q < Fa.nq(); ++q) { const double *R = Fa.ref(v, q); fr.insert(fr.end(), R, R + 3 * V.nloc()); }
            dump(dir, "facet_ref", fr);
            std::fprintf(meta, "facet_nq %d\nfacet_nent %d\nrobin %.17g\n", Fa.nq(), Fa.nent(), o.robin);
        }
    }

    // ---- numeric assembly ------------------------------------------------------------------
    auto assemble = [&](CSRMatrix &K, std::vector<double> &b, CSRMatrix *K2) {
        K.clear();
        if (o.form == "poisson_sin" || o.form == "poisson_vec")
        {
            auto c = const_coeff(Qa, o.c);
            assemble_matrix_2d(Qa, Qa, {1, 2}, {1, 2}, {c, c}, K, 0, 0, map.data());
        }
        else if (o.form == "helmholtz_sin")
        {
            auto one = const_coeff(Qa, 1.0);
            assemble_matrix_2d(Qa, Qa, {1, 2, 0}, {1, 2, 0}, {one, one, one}, K, 0, 0, map.data());
        }
        else if (o.form == "varcoef_field")
        {
            const std::size_t np = static_cast<std::size_t>(Qa.nent()) * Qa.nq();
            std::vector<double> kc(np);
            for (std::size_t p = 0; p < np; ++p)
                kc[p] = 1.0 + 0.5 * std::sin(2.0 * PI * Qa.x()[p]) * std::sin(2.0 * PI * Qa.y()[p]);
            assemble_matrix_2d(Qa, Qa, {1, 2}, {1, 2}, {kc, kc}, K, 0, 0, map.data());
        }
        else if (o.form == "heat")
        {
            auto one = const_coeff(Qa, 1.0);
            assemble_matrix_2d(Qa, Qa, {0}, {0}, {one}, K, 0, 0, map.data());
            K2->clear();
            assemble_matrix_2d(Qa, Qa, {1, 2}, {1, 2}, {one, one}, *K2, 0, 0, map.data());
        }
        if (rhs_data || rhs_field)
        {
            Cache2D Qf(V, qf);
            const std::size_t np = static_cast<std::size_t>(Qf.nent()) * Qf.nq();
            std::vector<double> fc(np);
            if (rhs_data)
                for (std::size_t p = 0; p < np; ++p)
                {
                    const double s = std::sin(PI * Qf.x()[p]) * std::sin(PI * Qf.y()[p]);
                    fc[p] = o.form == "poisson_sin" ? 2.0 * PI * PI * s : 2.0 * PI * PI * s + s;
                }
            else
            {
                std::vector<double> f = load<double>(o.fpath, static_cast<std::size_t>(n));
                const int code = 0;
                Qf.eval_multi(f.data(), false, &code, 1, fc.data());
            }
            b.assign(static_cast<std::size_t>(n), 0.0);
            assemble_vector_2d(Qf, {0}, {fc}, b);
        }
        else if (rhs_vec) b = load<double>(o.bpath, static_cast<std::size_t>(n));
        if (o.robin != 0.0)
        {
            // alpha u v ds and g v ds over every exterior facet (Cache2D on facets)
            Cache2D Fa(V, 2 * k, {}, true), Fb(V, k + 2, {}, true);
            std::vector<int> fmap = scatter_map_2d(Fa, Fa, *P, 0, 0);
            auto al = const_coeff(Fa, o.robin);
            assemble_matrix_2d(Fa, Fa, {0}, {0}, {al}, K, 0, 0, fmap.data());
            const std::size_t np = static_cast<std::size_t>(Fb.nent()) * Fb.nq();
            std::vector<double> g(np);
            for (std::size_t p = 0; p < np; ++p) g[p] = 1.0 + Fb.x()[p] * Fb.y()[p];
            if (b.size() != static_cast<std::size_t>(n)) b.assign(static_cast<std::size_t>(n), 0.0);
            assemble_vector_2d(Fb, {0}, {g}, b);
        }
    };

    CSRMatrix K(P), K2(P);
    std::vector<double> b;
    t0 = now();
    assemble(K, b, &K2);
    double t_asm = now() - t0;
    K.symmetric = asymmetry(K) <= 1e-13;
    std::fprintf(meta, "t_assemble %.6f\nsymmetric %d\nasymmetry %.17g\n", t_asm, K.symmetric ? 1 : 0, asymmetry(K));
    dump(dir, "data", K.data);
    if (o.form == "heat") { dump(dir, "data_K", K2.data); std::fprintf(meta, "done 1\n"); if (meta != stdout) std::fclose(meta); return 0; }
    dump(dir, "rhs", b);

    JacobiPreconditioner J(K);
    dump(dir, "inv_diag", J.inverse_diagonal());

    // one SpMV of a fixed vector (x_i = 1 + 0.5 sin(1 + 0.7 i)), for the SpMV parity test
    {
        std::vector<double> xs(static_cast<std::size_t>(n)), ys(static_cast<std::size_t>(n));
        for (int i = 0; i < n; ++i) xs[i] = 1.0 + 0.5 * std::sin(1.0 + 0.7 * i);
        double ts = now();
        const int reps = o.time_reps > 0 ? 3 : 1;
        for (int r = 0; r < reps; ++r) K.apply(xs.data(), ys.data());
        std::fprintf(meta, "t_spmv %.6f\n", (now() - ts) / reps);
        dump(dir, "spmv_y", ys);
    }

    const int maxiter = std::max(1000, 10 * n);      // python/femd/krylov.py:193
    if (o.cg)
    {
        auto op = [&K](const std::vector<double> &in, std::vector<double> &out) {
            out.resize(static_cast<std::size_t>(K.nrows()));
            K.apply(in.data(), out.data());
        };
        std::vector<double> x(static_cast<std::size_t>(n), 0.0);
        t0 = now();
        krylov::CGResult r = krylov::cg_jacobi(op, J.inverse_diagonal().data(), x, b, maxiter, o.tol);
        double t_cg = now() - t0;
        std::fprintf(meta, "t_cg %.6f\ncg_converged %d\ncg_iterations %d\ncg_residual %.17g\ncg_breakdown %d\n", t_cg,
                     r.converged ? 1 : 0, r.iterations, r.residual, r.breakdown ? 1 : 0);
        dump(dir, "x_cg", x);
    }
    if (o.pc)
    {
        // the ILU(0) and SSOR (omega 1) preconditioners on the natural ordering: one application
        // to the fixed vector of the SpMV test, and CG preconditioned by each
        auto op = [&K](const std::vector<double> &in, std::vector<double> &out) {
            out.resize(static_cast<std::size_t>(K.nrows()));
            K.apply(in.data(), out.data());
        };
        std::vector<double> xs(static_cast<std::size_t>(n));
        for (int i = 0; i < n; ++i) xs[i] = 1.0 + 0.5 * std::sin(1.0 + 0.7 * i);
        ILU0Preconditioner ilu(K);
        SSORPreconditioner ssor(K, 1.0);
        std::fprintf(meta, "ilu0_min_pivot %.17g\n", ilu.min_pivot());
        const SparsePreconditioner *pcs[2] = {&ilu, &ssor};
        const char *names[2] = {"ilu0", "ssor"};
        for (int m = 0; m < 2; ++m)
        {
            std::vector<double> z;
            (*pcs[m])(xs, z);
            dump(dir, std::string(names[m]) + "_apply_y", z);
            std::vector<double> x(static_cast<std::size_t>(n), 0.0);
            krylov::CGResult r = krylov::cg(op, *pcs[m], x, b, maxiter, o.tol);
            std::fprintf(meta, "%s_converged %d\n%s_iterations %d\n%s_residual %.17g\n%s_breakdown %d\n", names[m],
                         r.converged ? 1 : 0, names[m], r.iterations, names[m], r.residual, names[m], r.breakdown ? 1 : 0);
            dump(dir, std::string("x_") + names[m], x);
        }
    }
    if (o.chol)
    {
        t0 = now();
        SparseCholesky C(K, SparseCholesky::Ordering::AMD, true);
        double t_fac = now() - t0;
        std::vector<double> x(static_cast<std::size_t>(n));
        t0 = now();
        C.apply(b.data(), x.data());
        double t_sol = now() - t0;
        std::fprintf(meta, "t_chol_factor %.6f\nt_chol_solve %.6f\nnnz_L %lld\n", t_fac, t_sol, C.nnz_L());
        dump(dir, "x_chol", x);
    }
    // Timed steps for the CPU baseline: assembly of A and b plus cg_jacobi capped at
    // cg_sample iterations (0: to convergence).  One line per step: "step <t_asm> <t_cg> <its>".
    for (int rep = 0; rep < o.time_reps; ++rep)
    {
        std::vector<double> bb;
        double ta = now();
        assemble(K, bb, &K2);
        ta = now() - ta;
        auto op = [&K](const std::vector<double> &in, std::vector<double> &out) {
            out.resize(static_cast<std::size_t>(K.nrows()));
            K.apply(in.data(), out.data());
        };
        std::vector<double> x(static_cast<std::size_t>(n), 0.0);
        const int cap = (o.cg_sample > 0 && !(o.full_first && rep == 0)) ? o.cg_sample : maxiter;
        double tc = now();
        krylov::CGResult r = krylov::cg_jacobi(op, J.inverse_diagonal().data(), x, bb, cap, o.tol);
        tc = now() - tc;
        std::fprintf(meta, "step %.6f %.6f %d\n", ta, tc, r.iterations);
        std::fflush(meta);
    }
    std::fprintf(meta, "done 1\n");
    if (meta != stdout) std::fclose(meta);
    return 0;
}
