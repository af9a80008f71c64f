"""Tile-shape autotuner of the tensor-core contractions.

Every candidate tile shape must give bit-identical outputs (each output
element accumulates the same K blocks in the same order whatever the tile
width), so the E-step's results cannot depend on the tuner's choice: the
exhaustive E-step in BF16 and BF16X3 is run with each candidate pinned
(ROME_TC_SHAPE) and with the tuner choosing, and diff2, weights and poses
must be identical.  The tuner's report must list the pool's contraction with
every candidate timed."""
import numpy as np
import pytest

from rome_b200 import abi
from rome_b200.map2d import GpuContext
from rome_b200.workload import Map2dWorkload, build_map2d

pytestmark = pytest.mark.gpu

WL = Map2dWorkload(n_particles=48, ori_size=128, n_classes=3, n_blobs=40, psi_step=5, offset_range=6, offset_step=2,
                   max_shift=6, pixel=1.5, snr=0.03, seed=41)


@pytest.mark.parametrize("prec", ["bf16", "bf16x3"])
def test_candidates_identical_and_tuner_reports(prec, monkeypatch):
    p, proj, r_max, _ = build_map2d(WL)
    outs = {}
    for mode in ["0", "1", "tuned"]:
        if mode == "tuned":
            monkeypatch.delenv("ROME_TC_SHAPE", raising=False)
        else:
            monkeypatch.setenv("ROME_TC_SHAPE", mode)
        with GpuContext(0, prec) as ctx:
            ctx.set_projectors(proj, p.ori_size, r_max)
            outs[mode] = ctx.map2d_estep_pool(p, checkpoints=True)
    for mode in ["1", "tuned"]:
        for k in ("diff2_0", "weight_0", "cls", "psi", "xoff", "yoff", "sum_weight", "significant_weight"):
            assert np.array_equal(outs[mode][k], outs["0"][k]), (mode, k)
    rep = [r for r in abi.tuning_report() if r["kind"] == "diff2" and r["planes"] == ("1" if prec == "bf16" else "2")]
    assert rep, abi.tuning_report()
    for r in rep:
        times = [float(v[:-2]) for k, v in r.items() if v.endswith("ms")]
        assert len(times) == 2 and min(times) > 0 and r["choice"] in r
        print(prec, r)
