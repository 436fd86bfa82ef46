"""The bench's reference arm: the reference's own CPU build on the config-4 stream, driven by a
plain-numpy workload spec that never imports femd_b200 (whose import loads the CUDA library)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "femd_ref_omp")


def test_numpy_spec_is_the_package_spec():
    sys.path.insert(0, ROOT)
    import bench
    from femd_b200 import workloads as W
    sp = bench.c4_spec()
    assert sp == W.poisson_batch_spec(seed=0, nprob=256)
    idx = bench.c4_sample(sp)
    assert len(idx) == 8 and len(set(idx)) == 8
    work = [(sp[i]["k"] * sp[i]["N"]) ** 3 for i in idx]
    assert work == sorted(work)


@pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref is not built")
def test_reference_arm_runs_without_the_package():
    code = ("import sys, types, json; sys.path.insert(0, %r); import bench; "
            "a = types.SimpleNamespace(steps=1, warmup=0); line = bench.reference_c4(a, 0, 1); "
            "assert not any(m.startswith('femd_b200') for m in sys.modules), 'femd_b200 imported'; "
            "print(json.dumps(line))" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True, timeout=300).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 1
    assert line["cpu_baseline"]["kind"] == "reference" and line["e2e"]["h2d_bytes_per_step"] == 0
