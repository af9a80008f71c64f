"""Reconstruction at known poses (rome_b200/reconstruct_poses.py) against the
reference's own rome_reconstruct.

tests/golden/recon3d_a.npz holds the volume the reference app wrote
(float32 MRC) for a seeded dataset of 300 particles of 32^2 with CTF and
their generating poses (tests/golden/make_golden.py, `CASESRECON`); the
dataset is regenerated here from the same spec.  Gates: FSC >= 0.999 at
every shell and <= 1e-5 relative RMS difference (the reference's volume is
rounded to float32; both sides accumulate in FP64, in different orders)."""
import os
import sys

import numpy as np
import pytest

from rome_b200 import synthetic
from rome_b200.reconstruct_poses import reconstruct_from_star

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import CASESRECON, recon_dataset  # noqa: E402


def test_pose_columns_required(tmp_path):
    synthetic.write_mrcs(str(tmp_path / "a.mrcs"), np.zeros((2, 8, 8), np.float32))
    with open(tmp_path / "p.star", "w") as f:
        f.write("data_\nloop_\n_rlnImageName #1\n_rlnMicrographName #2\n_rlnAngleRot #3\n")
        f.write("000001@a.mrcs mic000000 10.0\n000002@a.mrcs mic000000 20.0\n")
    with pytest.raises(ValueError, match="rlnAngleTilt"):
        reconstruct_from_star(str(tmp_path / "p.star"), 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASESRECON))
def test_matches_reference_rome_reconstruct(golden, tmp_path, case):
    from test_gpu_reconstruct import fsc
    _, opt = CASESRECON[case]
    star = recon_dataset(case, str(tmp_path))
    ref = golden[case]["vol"].astype(np.float64)
    for pool in (64, 1000):    # several pools, and one
        vol = reconstruct_from_star(star, opt["angpix"], iters=opt["iter"], do_ctf=bool(opt["ctf"]), pool=pool)
        rms = np.sqrt(np.mean((vol - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
        f = fsc(vol, ref)
        print(f"{case} pool {pool}: rel rms {rms:.2e}, min FSC {f.min():.7f}")
        assert f.min() >= 0.999
        assert rms <= 1e-5
