"""Regenerate the golden fixtures in this directory from the REFERENCE itself.

Runs oracle/_ref/femd_ref (FEMd's own header-only C++ compiled from the reference tree by
oracle/Makefile; see oracle/ref_driver.cpp) on small cases and stores what it wrote as
compressed .npz files.  Needs the reference binary, so it runs where the reference tree is
(python tests/golden/make_golden.py); the fixtures are committed and the tests only read them.

Random inputs (a field f at the dofs, a load vector b) come from numpy's default_rng with the
seed named in the case, and are stored in the fixture beside the outputs.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "femd_ref")

# name: (form, N, k, extra args, random input kind, seed)
CASES = {
    "p1_poisson_n4": ("poisson_sin", 4, 1, [], None, None),
    "p2_helmholtz_n6": ("helmholtz_sin", 6, 2, [], None, None),
    "p3_poisson_n5": ("poisson_sin", 5, 3, [], None, None),
    "p2_varcoef_n6": ("varcoef_field", 6, 2, [], "f", 0),
    "p1_vec_n5": ("poisson_vec", 5, 1, ["--c", "2.5"], "b", 1),
    "p3_vec_n3": ("poisson_vec", 3, 3, ["--c", "0.4"], "b", 2),
    "p2_heat_n4": ("heat", 4, 2, [], None, None),
    "p2_varcoef_n16": ("varcoef_field", 16, 2, [], "f", 0),
    "c1_p3_poisson_n32": ("poisson_sin", 32, 3, [], None, None),
    # with the ILU(0)- and SSOR-preconditioned CG of the same system (--pc)
    "p2_poisson_pc_n16": ("poisson_sin", 16, 2, ["--pc"], None, None),
    "p3_varcoef_pc_n6": ("varcoef_field", 6, 3, ["--pc"], "f", 5),
    "p1_vec_pc_n20": ("poisson_vec", 20, 1, ["--c", "1.7", "--pc"], "b", 6),
    # no Dirichlet elimination, alpha u v ds and g v ds on every exterior facet (--free --robin)
    "p1_robin_ds_n6": ("poisson_sin", 6, 1, ["--free", "--robin", "2.5"], None, None),
    "p2_robin_ds_n5": ("poisson_sin", 5, 2, ["--free", "--robin", "0.7"], None, None),
    "p3_robin_ds_n4": ("poisson_sin", 4, 3, ["--free", "--robin", "4.0"], None, None),
}

INT_ARRAYS = ("tris", "cell_dofs", "cell_raw_dofs", "indptr", "indices", "scatter_map", "facet_cell", "facet_local",
              "facet_marker")

REF_INTEGRAND = os.path.join(ROOT, "oracle", "_ref", "femd_ref_integrand")
TWO_PI = 6.283185307179586


def _allops():
    """Every instruction once: u in [0.1, 2), v in [-1, 1); the sum of pow (2, -1, 0.5, 1.7,
    -2.5), sin ... sign of them, x, y and both normal components with both signs."""
    code = [[5, 0, 0, 0], [5, 1, 1, 0], [0, 2, 0, 0], [0, 3, 1, 0], [0, 4, 2, 0], [0, 5, 3, 0], [0, 6, 4, 0]]
    acc = [[8, 7, 0, 0], [8, 8, 0, 1], [8, 9, 0, 2], [8, 10, 0, 3], [8, 11, 0, 4]]
    acc += [[op, 11 + op - 8, 1 if op in (9, 10, 13, 15, 16, 17, 18, 19) else 0, 0] for op in range(9, 20)]
    code += acc
    nxt = 23
    code += [[1, nxt, 0, 0], [2, nxt + 1, 0, 0], [3, nxt + 2, 1, 0], [3, nxt + 3, -1, 0], [4, nxt + 4, 1, 0],
             [4, nxt + 5, -1, 0]]
    regs = list(range(7, 12)) + list(range(12, 23)) + list(range(nxt, nxt + 6))
    s = 29
    code.append([6, s, regs[0], regs[1]])
    for rg in regs[2:]:
        code.append([6, s + 1, s, rg])
        s += 1
    return code, s + 1, [2.0, -1.0, 0.5, 1.7, -2.5]


# name: (code, nreg, consts, input ranges, needs x/y, needs normal, seed)
INTEGRAND_CASES = {
    "integrand_convection": ([[5, 0, 0, 0], [5, 1, 2, 0], [7, 2, 0, 1], [5, 3, 1, 0], [5, 4, 3, 0], [7, 5, 3, 4],
                              [6, 6, 2, 5]], 7, [], [(-1, 1)] * 4, False, False, 11),
    "integrand_varcoef": ([[0, 0, 0, 0], [0, 1, 1, 0], [0, 2, 2, 0], [1, 3, 0, 0], [7, 4, 2, 3], [9, 5, 4, 0],
                           [2, 6, 0, 0], [7, 7, 2, 6], [9, 8, 7, 0], [7, 9, 5, 8], [7, 10, 1, 9], [6, 11, 0, 10]],
                          12, [1.0, 0.5, TWO_PI], [], True, False, 12),
    "integrand_allops": _allops() + ([(0.1, 2.0), (-1.0, 1.0)], True, True, 13),
}


def run_integrand(name):
    code, nreg, consts, ranges, xy, normal, seed = INTEGRAND_CASES[name]
    rng = np.random.default_rng(seed)
    npts = 1000                                     # four blocks of 256 and a partial one
    code = np.asarray(code, dtype=np.int32).reshape(-1, 4)
    consts = np.asarray(consts, dtype=np.float64)
    inputs = np.array([rng.uniform(lo, hi, npts) for lo, hi in ranges]).reshape(len(ranges), npts)
    xs, ys = rng.uniform(0, 1, npts), rng.uniform(0, 1, npts)
    th = rng.uniform(0, TWO_PI, npts)
    nx, ny = np.cos(th), np.sin(th)
    with tempfile.TemporaryDirectory() as d:
        spec = os.path.join(d, "spec.bin")
        with open(spec, "wb") as f:
            np.array([len(code), nreg, consts.size, len(ranges), npts, int(xy), int(normal)], dtype=np.int32).tofile(f)
            code.tofile(f)
            consts.tofile(f)
            if xy:
                xs.tofile(f)
                ys.tofile(f)
            if normal:
                nx.tofile(f)
                ny.tofile(f)
            inputs.tofile(f)
        outp = os.path.join(d, "out.bin")
        subprocess.run([REF_INTEGRAND, spec, outp], check=True)
        out = np.fromfile(outp, dtype=np.float64)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, code=code, nreg=np.int32(nreg), consts=consts, inputs=inputs, xs=xs, ys=ys, nx=nx, ny=ny,
                        has_xy=np.int32(xy), has_normal=np.int32(normal), out=out)
    return path


def dim_of(form, N, k):
    # the unknowns of P_k on an N x N rectangle mesh with every boundary node eliminated
    return (k * N - 1) ** 2


def run(name):
    form, N, k, extra, rnd, seed = CASES[name]
    with tempfile.TemporaryDirectory() as d:
        args = [REF, form, str(N), str(k), d] + extra
        arrays = {}
        if rnd is not None:
            v = np.random.default_rng(seed).standard_normal(dim_of(form, N, k))
            p = os.path.join(d, "input.bin")
            v.tofile(p)
            args += ["--" + rnd, p]
            arrays["input_" + rnd] = v
        if form != "heat":
            args += ["--chol"]
        subprocess.run(args, check=True)
        meta = {}
        steps = []
        for line in open(os.path.join(d, "meta.txt")):
            key, *vals = line.split()
            if key == "step":
                steps.append(vals)
            else:
                meta[key] = vals[0]
        for fn in sorted(os.listdir(d)):
            if not fn.endswith(".bin") or fn == "input.bin":
                continue
            key = fn[:-4]
            arrays[key] = np.fromfile(os.path.join(d, fn), dtype=np.int32 if key in INT_ARRAYS else np.float64)
    arrays["meta_keys"] = np.array(list(meta.keys()))
    arrays["meta_vals"] = np.array([str(v) for v in meta.values()])
    arrays["form"] = np.array(form)
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(out, **arrays)
    return out


if __name__ == "__main__":
    if not os.path.exists(REF):
        sys.exit(f"{REF} is missing: build it with `make -C oracle ref` where the reference tree is")
    for name in (sys.argv[1:] or list(CASES) + list(INTEGRAND_CASES)):
        path = run_integrand(name) if name in INTEGRAND_CASES else run(name)
        print(path, os.path.getsize(path))
