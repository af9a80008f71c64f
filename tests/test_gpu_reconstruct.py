"""GPU M-step (MyBackProjector::reconstruct) against the reference's own
maximization() outputs recorded in tests/golden (2D classes).

Gates: the reconstructed class has FSC >= 0.999 at every shell against the
reference reconstruction and <= 1e-6 relative RMS difference; sigma2 and
data_vs_prior spectra agree to 1e-9 relative (FP64 on both sides; only the
summation order of the radial sums differs)."""
import numpy as np
import pytest

from rome_b200.map2d import GpuContext
from tests.util import golden_pool

pytestmark = pytest.mark.gpu

CASES = ["map2d_a", "map2d_b", "map2d_c"]


def fsc(a, b):
    fa, fb = np.fft.fftn(a), np.fft.fftn(b)
    idx = np.indices(a.shape)
    c = [(n // 2) for n in a.shape]
    r = np.sqrt(sum(((np.fft.fftshift(idx[d]) - c[d]) ** 2) for d in range(a.ndim)))
    r = np.fft.ifftshift(r).astype(int)
    out = []
    for s in range(1, min(a.shape) // 2):
        m = r == s
        num = np.real(np.sum(fa[m] * np.conj(fb[m])))
        den = np.sqrt(np.sum(np.abs(fa[m]) ** 2) * np.sum(np.abs(fb[m]) ** 2))
        out.append(num / den if den > 0 else 1.0)
    return np.array(out)


@pytest.mark.parametrize("case", CASES)
def test_reconstruct_matches_reference(golden, case):
    g = golden[case]
    p, proj, r_max = golden_pool(g)
    K, ori = p.nr_classes, p.ori_size
    with GpuContext(0) as ctx:
        ctx.set_projectors(proj, ori, r_max)
        for k in range(K):
            if g["pdf_class"][k] <= 0:
                continue
            ctx.set_backprojector(k, g["iter_bp_data"][k], g["iter_bp_weight"][k])
            o = ctx.reconstruct(k, ori, 2, g["tau2_class_before"][k], float(g["tau2_fudge_factor"][0]),
                                float(g["iter_wsum_pdf_class"][k]), int(g["gridding_nr_iter"][0]),
                                bool(g["do_map"][0]), int(g["minres_map"][0]))
            ref = g["Irefs_after"][k]
            rms = np.sqrt(np.mean((o["vol"] - ref) ** 2)) / np.sqrt(np.mean(ref ** 2))
            f = fsc(o["vol"], ref)
            print(f"{case} class {k}: rel rms {rms:.2e}, min FSC {f.min():.6f}")
            assert f.min() >= 0.999
            assert rms <= 1e-6
            s_ref = g["sigma2_class_after"][k]
            d_ref = g["data_vs_prior_after"][k]
            assert np.max(np.abs(o["sigma2"] - s_ref)) <= 1e-9 * max(np.max(np.abs(s_ref)), 1e-300)
            assert np.max(np.abs(o["data_vs_prior"] - d_ref)) <= 1e-9 * max(np.max(np.abs(d_ref)), 1e-300)
