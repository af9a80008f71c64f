"""A bounded device wait that runs out.

Every tensor-core kernel waits on mbarriers with a bound; on expiry it
records the timeout in the context's error flag, drains what it issued,
frees its tensor memory and returns, and the entry point reports
ROME_ERR_TIMEOUT.  rome_gpu_wait_selftest launches that same bounded wait on
a barrier nothing arrives on (no fault, no trap, no unbounded loop): the test
checks the status, that the wait lasted about its limit, and that the same
context then runs a normal E-step pool whose results match the oracle."""
import numpy as np
import pytest

from rome_b200 import abi
from rome_b200.map2d import GpuContext, RomeError
from rome_b200.workload import Map2dWorkload, build_map2d

pytestmark = pytest.mark.gpu


def small_pool():
    w = Map2dWorkload(n_particles=16, ori_size=32, n_classes=3, n_blobs=8, blob_sigma=(1.5, 3.0), psi_step=15,
                      offset_range=3, offset_step=1, max_shift=2, pixel=4.0, snr=0.1, seed=21)
    return build_map2d(w)


@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_wait_runs_out_and_context_stays_usable(prec):
    from oracle import oracle_py
    p, proj, r_max, _ = small_pool()
    with GpuContext(0, prec) as ctx:
        ctx.set_projectors(proj, p.ori_size, r_max)
        with pytest.raises(RomeError) as e:
            ctx.wait_selftest(0.05)
        assert e.value.code == abi.ROME_ERR_TIMEOUT
        assert "wait expired" in str(e.value)
        assert 0.05 <= ctx.last_wait_seconds < 1.0, ctx.last_wait_seconds
        # the error flag was cleared: the next pool runs and is right
        o = ctx.map2d_estep_pool(p, checkpoints=True)
    r, _, _ = oracle_py.map2d_estep_pool(p, proj, r_max, checkpoints=True)
    ok = r["diff2_0"] > -1e9
    rel = np.abs(o["diff2_0"][ok] - r["diff2_0"][ok]) / np.abs(r["diff2_0"][ok])
    assert rel.max() < (1e-5 if prec == "fp32" else 1e-3), rel.max()
    assert np.mean(o["cls"] == r["cls"]) >= 0.9


def test_wait_limit_is_checked():
    with GpuContext(0, "fp32") as ctx:
        with pytest.raises(RomeError) as e:
            ctx.wait_selftest(5.0)
        assert e.value.code == abi.ROME_ERR_ARG
