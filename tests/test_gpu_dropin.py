"""The reference's own MAP2D and MAP3D drivers calling the library through
include/rome_gpu.h from C++ (oracle/_ref/map2d_dropin and map3d_dropin,
built from oracle/ref_harness/map{2,3}d_dropin.cpp against the reference's
objects and rome_b200/librome_b200.so): each fills the pool structure from
the optimizer's own state as a patched expectationSomeParticles() would,
calls the library, runs the reference's E-step functions on the same pool,
and compares (diff2 1e-5 relative, FP64 sums and back-projectors 1e-3
relative, poses identical but for near ties).  MAP3D in maximum-likelihood,
cross-correlation and scale-correction modes; MAP2D with one pass and with
adaptive oversampling; on the seeded datasets of the golden cases."""
import os
import re
import subprocess
import tempfile

import pytest

from rome_b200.synthetic import write_dataset_2d, write_dataset_3d
from tests.golden.make_golden import CASES, CASES3D

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "map3d_dropin")
BIN2D = os.path.join(ROOT, "oracle", "_ref", "map2d_dropin")
KEYS2D = ("K", "iter", "angpix", "tau2_fudge", "oversampling", "pool", "psi_step", "offset_range", "offset_step",
          "ctf")
KEYS = ("K", "iter", "angpix", "ini_high", "tau2_fudge", "oversampling", "healpix_order", "pool", "offset_range",
        "offset_step", "ctf", "uniform_directions", "always_cc", "scale")


@pytest.mark.parametrize("case", ["map3d_a", "map3d_cc", "map3d_scale"])
def test_reference_driver_calls_the_library(case):
    assert os.path.exists(BIN), "oracle/_ref/map3d_dropin is built by __graft_entry__.build()"
    spec, opt = CASES3D[case]
    with tempfile.TemporaryDirectory(prefix="rome_dropin_") as tmp:
        star, ref = write_dataset_3d(os.path.join(tmp, "data"), spec)
        cmd = [BIN, "-i", star, "-ref", ref]
        for k in KEYS:
            if k in opt:
                cmd += [f"-{k}", str(opt[k])]
        env = dict(os.environ, OMP_NUM_THREADS="8")
        r = subprocess.run(cmd, cwd=tmp, env=env, capture_output=True, text=True, timeout=900)
    line = [x for x in r.stdout.splitlines() if x.startswith("DROPIN")]
    assert line, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    print(case, line[-1])
    vals = dict(kv.split("=") for kv in line[-1].split()[1:])
    assert r.returncode == 0, line[-1]
    assert int(vals["cc"]) == int(opt.get("always_cc", 0)) and int(vals["scale"]) == int(opt.get("scale", 0))
    assert int(vals["same_pose"]) >= int(vals["particles"]) - 1
    assert float(vals["min_diff2"]) <= 1e-5
    for k in ("sum_weight", "wsum_sigma2_noise", "bp_data", "bp_weight"):
        assert float(vals[k]) <= 1e-3, k
    assert re.match(r"^\d+$", vals["same_nr_sign"])


@pytest.mark.parametrize("case", ["map2d_a", "map2d_b"])
def test_reference_2d_driver_calls_the_library(case):
    assert os.path.exists(BIN2D), "oracle/_ref/map2d_dropin is built by __graft_entry__.build()"
    spec, opt = CASES[case]
    with tempfile.TemporaryDirectory(prefix="rome_dropin2_") as tmp:
        star = write_dataset_2d(os.path.join(tmp, "data"), spec)
        cmd = [BIN2D, "-i", star]
        for k in KEYS2D:
            if k in opt:
                cmd += [f"-{k}", str(opt[k])]
        env = dict(os.environ, OMP_NUM_THREADS="8")
        r = subprocess.run(cmd, cwd=tmp, env=env, capture_output=True, text=True, timeout=900)
    line = [x for x in r.stdout.splitlines() if x.startswith("DROPIN")]
    assert line, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    print(case, line[-1])
    vals = dict(kv.split("=") for kv in line[-1].split()[1:])
    assert r.returncode == 0, line[-1]
    assert int(vals["passes"]) == (2 if opt["oversampling"] else 1)
    assert int(vals["same_pose"]) >= int(vals["particles"]) - 1
    assert float(vals["min_diff2"]) <= 1e-5
    for k in ("sum_weight", "wsum_sigma2_noise", "wsum_prior_offsetx", "bp_data", "bp_weight"):
        assert float(vals[k]) <= 1e-3, k
