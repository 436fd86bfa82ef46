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
}

INT_ARRAYS = ("tris", "cell_dofs", "cell_raw_dofs", "indptr", "indices", "scatter_map")


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
    for name in (sys.argv[1:] or CASES):
        print(run(name), os.path.getsize(os.path.join(HERE, name + ".npz")))
