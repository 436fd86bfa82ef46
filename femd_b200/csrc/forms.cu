// forms.cu -- the coefficient side of a compiled form on the device: the Integrand register
// program evaluated at the quadrature points, and P_k fields (values and first derivatives) at
// the points of a cell rule.
//
// Integrand (include/femd/forms/integrand.hpp:33-45 instruction set, :47-66 checks, :300-342
// run).  A program is a list of 4-integer instructions (op, out register, a, b) over registers
// that hold one value per point; the coefficient is the last instruction's register.  Here one
// thread evaluates one point: the block stages the code and the constants in shared memory, and
// each thread keeps its registers in a shared-memory column (registers [r][thread], so a warp's
// accesses fall in distinct banks).  Every thread of a block runs the same instruction stream, so
// nothing diverges.  Sums and products are single IEEE operations with no contraction
// (__dadd_rn / __dmul_rn), squares, reciprocals and square roots are exact operations, as the
// reference's are; sin, cos, exp, log, tanh, sinh, cosh and pow are CUDA's double-precision
// functions (a few ulp from the host C library's), and sech z = 2 e / (1 + e^2) with
// e = exp(-|z|) (integrand.hpp:159-163).
//
// Points.  On cells the coordinates are formed from the mesh as the reference's cell cache does:
// x = P0.x + J0 xi + J1 eta, y = P0.y + J2 xi + J3 eta (lagrange_space_2d.hpp:86-87,
// cache_2d.hpp:108), in [e nq + q] order; other point sets (facets, or any given points) pass
// their coordinates and normals as arrays.
//
// Fields (Cache2D::eval_multi, cache_2d.hpp:245-288): per cell the nloc coefficients are gathered
// (constrained nodes read 0), then per point s0 = sum_l R_l c_l and, for derivatives,
// rx_l = Ji0 Rxi_l + Ji2 Reta_l, ry_l = Ji1 Rxi_l + Ji3 Reta_l, s1 = sum_l rx_l c_l,
// s2 = sum_l ry_l c_l, each sum in increasing l with no contraction.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace femd {

enum : int {
    IG_CONST = 0, IG_X, IG_Y, IG_NX, IG_NY, IG_INPUT, IG_ADD, IG_MUL, IG_POW, IG_SIN, IG_COS, IG_EXP, IG_LOG, IG_TANH,
    IG_SQRT, IG_SINH, IG_COSH, IG_SECH, IG_ABS, IG_SIGN
};

static constexpr int IG_BLOCK = 128;
static constexpr int IG_MAX_INPUTS = 16;
static constexpr int IG_MAX_INSTR = 2048;
static constexpr int IG_MAX_CONSTS = 1024;
static constexpr int IG_MAX_REGS = 160;       // 160 x 128 x 8 B = 160 KB of register columns

struct IgInputs {
    const double *p[IG_MAX_INPUTS];
};

// where the points are: arrays (xs, ys, nx, ny; any may be null when not read), or the cells of a
// mesh with the nq reference points (xi, eta) of a rule
struct IgPoints {
    const double *xs, *ys, *nx, *ny;
    const double *pts;
    const int *tris;
    const double *xi, *eta;
    int nq;
};

__device__ __forceinline__ double ig_sech(double z)
{
    const double e = exp(-fabs(z));
    return __ddiv_rn(__dmul_rn(2.0, e), __dadd_rn(1.0, __dmul_rn(e, e)));
}

__global__ void __launch_bounds__(IG_BLOCK) k_integrand(const int4 *__restrict__ code, int ninstr, int nreg,
                                                        const double *__restrict__ consts, int nconst, IgInputs in,
                                                        IgPoints P, long long npts, double *__restrict__ out)
{
    extern __shared__ int4 ig_smem[];
    int4 *scode = ig_smem;                                         // [ninstr], 16-byte aligned first
    double *regs = reinterpret_cast<double *>(scode + ninstr);     // [nreg][IG_BLOCK]
    double *sc = regs + (size_t)nreg * IG_BLOCK;                   // [nconst]
    for (int k = threadIdx.x; k < ninstr; k += IG_BLOCK) scode[k] = code[k];
    for (int k = threadIdx.x; k < nconst; k += IG_BLOCK) sc[k] = consts[k];
    __syncthreads();
    const int result = scode[ninstr - 1].y;
    double *R = regs + threadIdx.x;
    for (long long base = (long long)blockIdx.x * IG_BLOCK; base < npts; base += (long long)gridDim.x * IG_BLOCK) {
        const long long q = base + threadIdx.x;
        if (q >= npts) break;                                      // no barrier follows
        double x = 0.0, y = 0.0;
        if (P.xs) {
            x = P.xs[q];
            y = P.ys[q];
        } else if (P.pts) {
            const int e = (int)(q / P.nq), qq = (int)(q % P.nq);
            const int v0 = P.tris[3 * e], v1 = P.tris[3 * e + 1], v2 = P.tris[3 * e + 2];
            const double x0 = P.pts[2 * v0], y0 = P.pts[2 * v0 + 1];
            const double J0 = __dsub_rn(P.pts[2 * v1], x0), J1 = __dsub_rn(P.pts[2 * v2], x0);
            const double J2 = __dsub_rn(P.pts[2 * v1 + 1], y0), J3 = __dsub_rn(P.pts[2 * v2 + 1], y0);
            x = __dadd_rn(__dadd_rn(x0, __dmul_rn(J0, P.xi[qq])), __dmul_rn(J1, P.eta[qq]));
            y = __dadd_rn(__dadd_rn(y0, __dmul_rn(J2, P.xi[qq])), __dmul_rn(J3, P.eta[qq]));
        }
        for (int r = 0; r < nreg; ++r) R[(size_t)r * IG_BLOCK] = 0.0;   // a register read before it is written reads 0
        for (int k = 0; k < ninstr; ++k) {
            const int4 I = scode[k];
            const double ra = (I.x >= IG_ADD) ? R[(size_t)I.z * IG_BLOCK] : 0.0;
            double v = 0.0;
            switch (I.x) {
            case IG_CONST: v = sc[I.z]; break;
            case IG_X: v = x; break;
            case IG_Y: v = y; break;
            case IG_NX: v = (I.z < 0 ? -1.0 : 1.0) * P.nx[q]; break;
            case IG_NY: v = (I.z < 0 ? -1.0 : 1.0) * P.ny[q]; break;
            case IG_INPUT: v = in.p[I.z][q]; break;
            case IG_ADD: v = __dadd_rn(ra, R[(size_t)I.w * IG_BLOCK]); break;
            case IG_MUL: v = __dmul_rn(ra, R[(size_t)I.w * IG_BLOCK]); break;
            case IG_POW: {
                const double n = sc[I.w];
                if (n == 2.0) v = __dmul_rn(ra, ra);
                else if (n == -1.0) v = __ddiv_rn(1.0, ra);
                else if (n == 0.5) v = __dsqrt_rn(ra);
                else v = pow(ra, n);
                break;
            }
            case IG_SIN: v = sin(ra); break;
            case IG_COS: v = cos(ra); break;
            case IG_EXP: v = exp(ra); break;
            case IG_LOG: v = log(ra); break;
            case IG_TANH: v = tanh(ra); break;
            case IG_SQRT: v = __dsqrt_rn(ra); break;
            case IG_SINH: v = sinh(ra); break;
            case IG_COSH: v = cosh(ra); break;
            case IG_SECH: v = ig_sech(ra); break;
            case IG_ABS: v = fabs(ra); break;
            case IG_SIGN: v = ra > 0.0 ? 1.0 : (ra < 0.0 ? -1.0 : 0.0); break;
            default: break;
            }
            R[(size_t)I.y * IG_BLOCK] = v;
        }
        out[q] = R[(size_t)result * IG_BLOCK];
    }
}

// Field codes at the cell points: out[i np + e nq + q] for codes[i] (0 value, 1 d/dx, 2 d/dy).
// One thread per (cell, point); the cell's coefficients are read through the cell->dof map.
__global__ void __launch_bounds__(256) k_eval_field(const double *__restrict__ pts, const int *__restrict__ tris, int ne,
                                                    int nq, int nloc, const double *__restrict__ ref,
                                                    const int *__restrict__ dofs, const double *__restrict__ c, int c0,
                                                    int c1, int c2, int ncodes, int deriv, double *__restrict__ out)
{
    extern __shared__ double fs_ref[];                             // [nq][3][nloc]
    for (int k = threadIdx.x; k < nq * 3 * nloc; k += blockDim.x) fs_ref[k] = ref[k];
    __syncthreads();
    const long long np = (long long)ne * nq;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < np; t += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(t / nq), q = (int)(t % nq);
        const double *Rq = fs_ref + (size_t)q * 3 * nloc;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        if (!deriv) {
            for (int l = 0; l < nloc; ++l) {
                const int d = dofs[(size_t)e * nloc + l];
                s0 = __dadd_rn(s0, __dmul_rn(Rq[l], d >= 0 ? c[d] : 0.0));
            }
        } else {
            const int v0 = tris[3 * e], v1 = tris[3 * e + 1], v2 = tris[3 * e + 2];
            const double x0 = pts[2 * v0], y0 = pts[2 * v0 + 1];
            const double J0 = __dsub_rn(pts[2 * v1], x0), J1 = __dsub_rn(pts[2 * v2], x0);
            const double J2 = __dsub_rn(pts[2 * v1 + 1], y0), J3 = __dsub_rn(pts[2 * v2 + 1], y0);
            const double det = __dsub_rn(__dmul_rn(J0, J3), __dmul_rn(J1, J2));
            // J^{-1} = [J3, -J1; -J2, J0] / det (cache_2d.hpp:116-117)
            const double ax = __ddiv_rn(J3, det), ay = __ddiv_rn(-J1, det);
            const double bx = __ddiv_rn(-J2, det), by = __ddiv_rn(J0, det);
            for (int l = 0; l < nloc; ++l) {
                const int d = dofs[(size_t)e * nloc + l];
                const double cl = d >= 0 ? c[d] : 0.0;
                s0 = __dadd_rn(s0, __dmul_rn(Rq[l], cl));
                const double rx = __dadd_rn(__dmul_rn(ax, Rq[nloc + l]), __dmul_rn(bx, Rq[2 * nloc + l]));
                s1 = __dadd_rn(s1, __dmul_rn(rx, cl));
                const double ry = __dadd_rn(__dmul_rn(ay, Rq[nloc + l]), __dmul_rn(by, Rq[2 * nloc + l]));
                s2 = __dadd_rn(s2, __dmul_rn(ry, cl));
            }
        }
        const double s[3] = {s0, s1, s2};
        const int cd[3] = {c0, c1, c2};
        for (int i = 0; i < ncodes; ++i) out[(size_t)i * np + t] = s[cd[i]];
    }
}

// the reference's checks of a program (integrand.hpp:47-66), with its messages
static int check_program(const femd_integrand *g)
{
    FEMD_CHECK_ARG(g && (g->ncode == 0 || g->code_host), "Integrand: NULL program");
    FEMD_CHECK_ARG(g->ncode % 4 == 0, "Integrand: the code has 4 integers per instruction");
    FEMD_CHECK_ARG(g->nreg >= 1, "Integrand: at least one register");
    FEMD_CHECK_ARG(g->ncode > 0, "Integrand: empty program");
    const int *c = g->code_host;
    for (int k = 0; k < g->ncode; k += 4) {
        const int op = c[k], out = c[k + 1], a = c[k + 2], b = c[k + 3];
        FEMD_CHECK_ARG(out >= 0 && out < g->nreg, "Integrand: register out of range");
        FEMD_CHECK_ARG(!(op == IG_CONST && (a < 0 || a >= g->nconst)), "Integrand: constant out of range");
        FEMD_CHECK_ARG(!(op == IG_INPUT && (a < 0 || a >= g->ninput)), "Integrand: input out of range");
        FEMD_CHECK_ARG(!((op == IG_ADD || op == IG_MUL) && (a < 0 || a >= g->nreg || b < 0 || b >= g->nreg)),
                       "Integrand: register out of range");
        FEMD_CHECK_ARG(!(op == IG_POW && (a < 0 || a >= g->nreg || b < 0 || b >= g->nconst)),
                       "Integrand: pow operands out of range");
        FEMD_CHECK_ARG(!(op >= IG_SIN && op <= IG_SIGN && (a < 0 || a >= g->nreg)), "Integrand: register out of range");
        FEMD_CHECK_ARG(op >= 0 && op <= IG_SIGN, "Integrand: unknown instruction " + std::to_string(op));
    }
    // limits of this evaluator (no reference counterpart): the register columns and the code live
    // in shared memory
    FEMD_CHECK_ARG(g->nreg <= IG_MAX_REGS, "Integrand: more than " + std::to_string(IG_MAX_REGS) + " registers");
    FEMD_CHECK_ARG(g->ncode / 4 <= IG_MAX_INSTR, "Integrand: more than " + std::to_string(IG_MAX_INSTR) + " instructions");
    FEMD_CHECK_ARG(g->nconst <= IG_MAX_CONSTS, "Integrand: more than " + std::to_string(IG_MAX_CONSTS) + " constants");
    FEMD_CHECK_ARG(g->ninput >= 0 && g->ninput <= IG_MAX_INPUTS,
                   "Integrand: more than " + std::to_string(IG_MAX_INPUTS) + " inputs");
    return FEMD_OK;
}

static bool reads(const femd_integrand *g, int op0, int op1)
{
    for (int k = 0; k < g->ncode; k += 4)
        if (g->code_host[k] == op0 || g->code_host[k] == op1) return true;
    return false;
}

// Upload the code and constants (stream-ordered from pinned staging) and launch the program.
static int run_program(femd_ctx ctx, const femd_integrand *g, const double *consts_host, const double *const *inputs_dev,
                       const IgPoints &P, long long npts, double *out)
{
    cudaStream_t s = ctx->stream;
    const int ninstr = g->ncode / 4, nc = g->nconst;
    IgInputs in{};
    for (int i = 0; i < g->ninput; ++i) {
        FEMD_CHECK_ARG(inputs_dev && inputs_dev[i], "Integrand: wrong number of inputs");
        in.p[i] = inputs_dev[i];
    }
    FEMD_CHECK_ARG(nc == 0 || consts_host, "Integrand: wrong number of constants");
    if (npts == 0) return FEMD_OK;
    // code then constants in one device buffer (the program is a few KB)
    const size_t code_b = (size_t)ninstr * sizeof(int4), bytes = code_b + (size_t)nc * sizeof(double);
    DevBuf<char> buf;
    FEMD_TRY(buf.alloc(bytes));
    std::vector<char> h(bytes);
    memcpy(h.data(), g->code_host, code_b);
    if (nc) memcpy(h.data() + code_b, consts_host, (size_t)nc * sizeof(double));
    FEMD_TRY_CUDA(cudaMemcpyAsync(buf.p, h.data(), bytes, cudaMemcpyHostToDevice, s));
    const size_t shm = (size_t)g->nreg * IG_BLOCK * sizeof(double) + (size_t)nc * sizeof(double) + code_b;
    FEMD_TRY_CUDA(cudaFuncSetAttribute(k_integrand, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    const unsigned grid = grid_for((size_t)npts, IG_BLOCK, (unsigned)ctx->sm_count * 8);
    k_integrand<<<grid, IG_BLOCK, shm, counted(s)>>>(reinterpret_cast<const int4 *>(buf.p), ninstr, g->nreg,
                                                    reinterpret_cast<const double *>(buf.p + code_b), nc, in, P, npts, out);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));   // the code buffer is released on return
    return FEMD_OK;
}

}  // namespace femd

using namespace femd;

extern "C" {

int femd_cuda_integrand_eval(femd_ctx ctx, const femd_integrand *prog, const double *consts_host,
                             const double *const *inputs_dev, long long npts, const double *xs_dev, const double *ys_dev,
                             const double *nx_dev, const double *ny_dev, double *out_dev)
{
    clear_error();
    FEMD_CHECK_ARG(ctx, "Integrand: NULL context");
    FEMD_TRY(check_program(prog));
    FEMD_CHECK_ARG(npts >= 0 && (npts == 0 || out_dev), "Integrand: NULL output");
    FEMD_CHECK_ARG(!reads(prog, IG_X, IG_Y) || (xs_dev && ys_dev), "Integrand: the program reads x or y");
    FEMD_CHECK_ARG(!reads(prog, IG_NX, IG_NY) || (nx_dev && ny_dev), "Integrand: the program reads the normal");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    IgPoints P{};
    P.xs = xs_dev;
    P.ys = ys_dev;
    P.nx = nx_dev;
    P.ny = ny_dev;
    if (!P.xs || !P.ys) P.xs = P.ys = nullptr;
    return run_program(ctx, prog, consts_host, inputs_dev, P, npts, out_dev);
}

int femd_cuda_integrand_eval_cells(femd_ctx ctx, const femd_integrand *prog, const double *consts_host,
                                   const double *const *inputs_dev, const femd_mesh2d *mesh, const femd_rule *rule,
                                   double *out_dev)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && mesh && rule, "Integrand: NULL argument");
    FEMD_TRY(check_program(prog));
    FEMD_CHECK_ARG(!reads(prog, IG_NX, IG_NY), "FormAssembler2D::add_term: the coefficient reads the normal on a cell group");
    FEMD_CHECK_ARG(mesh->ncells >= 0 && (mesh->ncells == 0 || (mesh->points_dev && mesh->tris_dev)), "Integrand: bad mesh");
    FEMD_CHECK_ARG(rule->nq >= 1 && rule->nq <= 64 && rule->xi_host && rule->eta_host, "Integrand: bad rule");
    const long long npts = (long long)mesh->ncells * rule->nq;
    FEMD_CHECK_ARG(npts == 0 || out_dev, "Integrand: NULL output");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    DevBuf<double> xe;
    FEMD_TRY(xe.alloc(2 * (size_t)rule->nq));
    FEMD_TRY_CUDA(cudaMemcpyAsync(xe.p, rule->xi_host, rule->nq * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    FEMD_TRY_CUDA(cudaMemcpyAsync(xe.p + rule->nq, rule->eta_host, rule->nq * sizeof(double), cudaMemcpyHostToDevice,
                                  ctx->stream));
    IgPoints P{};
    P.pts = mesh->points_dev;
    P.tris = mesh->tris_dev;
    P.xi = xe.p;
    P.eta = xe.p + rule->nq;
    P.nq = rule->nq;
    return run_program(ctx, prog, consts_host, inputs_dev, P, npts, out_dev);
}

int femd_cuda_eval_field(femd_ctx ctx, const femd_mesh2d *mesh, const femd_rule *rule, const int *cell_dofs_dev,
                         const double *field_dev, int ncodes, const int *codes, double *out_dev)
{
    clear_error();
    FEMD_CHECK_ARG(ctx && mesh && rule && codes, "eval_multi: NULL argument");
    FEMD_CHECK_ARG(ncodes >= 1 && ncodes <= 3, "FormAssembler2D::add_field: no derivative codes");
    bool deriv = false;
    for (int i = 0; i < ncodes; ++i) {
        FEMD_CHECK_ARG(codes[i] >= 0 && codes[i] <= 2, "derivative code is 0 (value), 1 (d/dx) or 2 (d/dy)");
        deriv = deriv || codes[i] > 0;
    }
    FEMD_CHECK_ARG(rule->nq >= 1 && rule->nq <= 64 && rule->nloc >= 1 && rule->nloc <= 28 && rule->ref_host, "eval_multi: bad rule");
    const long long np = (long long)mesh->ncells * rule->nq;
    if (np == 0) return FEMD_OK;
    FEMD_CHECK_ARG(cell_dofs_dev && field_dev && out_dev && mesh->points_dev && mesh->tris_dev, "eval_multi: NULL array");
    FEMD_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const size_t nref = (size_t)rule->nq * 3 * rule->nloc;
    DevBuf<double> ref;
    FEMD_TRY(ref.alloc(nref));
    FEMD_TRY_CUDA(cudaMemcpyAsync(ref.p, rule->ref_host, nref * sizeof(double), cudaMemcpyHostToDevice, s));
    const size_t shm = nref * sizeof(double);
    FEMD_TRY_CUDA(cudaFuncSetAttribute(k_eval_field, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    k_eval_field<<<grid_for((size_t)np, 256, (unsigned)ctx->sm_count * 16), 256, shm, counted(s)>>>(
        mesh->points_dev, mesh->tris_dev, mesh->ncells, rule->nq, rule->nloc, ref.p, cell_dofs_dev, field_dev, codes[0],
        ncodes > 1 ? codes[1] : 0, ncodes > 2 ? codes[2] : 0, ncodes, deriv ? 1 : 0, out_dev);
    FEMD_TRY_CUDA(cudaGetLastError());
    FEMD_TRY_CUDA(cudaStreamSynchronize(s));   // the table is released on return
    return FEMD_OK;
}

}  // extern "C"
