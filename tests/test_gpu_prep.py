"""GPU particle preparation (rome_gpu_prepare_particles) against the
reference's recorded setFourierTransforms outputs and the preparation oracle
(oracle/prep_oracle.py).  Tolerances: FP64 throughout; the transforms differ
from the reference's FFTW only by round-off (relative 1e-12 of the largest
coefficient), the seeded noise is drawn exactly like the reference's (a
wrong draw moves the masked transform by tens of percent)."""
import numpy as np
import pytest

from oracle import prep_oracle as po
from rome_b200.particles import ParticleImages, PrepOptions, prepare_particles

pytestmark = pytest.mark.gpu

CASES = ["map2d_a", "map2d_b", "map2d_c"]
TOL = 1e-12


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def opts_from(o: dict) -> PrepOptions:
    return PrepOptions(pixel_size=o["pixel_size"], particle_diameter=o["particle_diameter"],
                       width_mask_edge=o["width_mask_edge"], sigma2_fudge=o["sigma2_fudge"],
                       random_seed=o["random_seed"], avg_norm_correction=o["avg_norm_correction"],
                       do_norm_correction=o["do_norm_correction"], do_zero_mask=o["do_zero_mask"],
                       do_ctf_correction=o["do_ctf_correction"], ctf_phase_flipped=o.get("ctf_phase_flipped", False),
                       only_flip_phases=o.get("only_flip_phases", False),
                       intact_ctf_first_peak=o.get("intact_ctf_first_peak", False))


def images_from(raw, meta, group, first=0):
    return ParticleImages(images=raw, norm=meta[:, 0], xoff=meta[:, 1], yoff=meta[:, 2], ctf=meta[:, 3:10],
                          group=group, first_image=first)


@pytest.fixture(scope="module")
def ctx():
    from rome_b200.map2d import GpuContext
    with GpuContext(0, "fp32") as c:
        yield c


@pytest.mark.parametrize("case", CASES)
def test_matches_reference_outputs(ctx, golden, case):
    g = golden[case]
    o = po.options_from_golden(g)
    imgs = images_from(g["pool0_raw_images"], g["pool0_prep_metadata"], g["pool0_group"], int(g["pool0_first_image"][0]))
    out = prepare_particles(ctx, imgs, opts_from(o), g["sigma2_noise"], int(g["current_size"][0]))
    for name in ("Fimg_real", "Fimg_imag", "Fimg_nomask_real", "Fimg_nomask_imag", "Fctf"):
        assert rel(out[name], g["pool0_" + name]) < TOL, name
    assert rel(out["power_imgs"], g["pool0_power_imgs"]) < 1e-11
    assert rel(out["highres_Xi2"], g["pool0_highres_Xi2"]) < 1e-11
    assert np.array_equal(out["old_offsetx"], g["pool0_old_offsetx"])
    assert np.array_equal(out["old_offsety"], g["pool0_old_offsety"])


def synthetic(P, ori, G, seed, dtype=np.float32):
    rng = np.random.default_rng(seed)
    raw = rng.normal(size=(P, ori, ori)).astype(dtype)
    meta = np.zeros((P, 10))
    meta[:, 0] = rng.uniform(0.8, 1.2, P)
    meta[:, 1] = rng.uniform(-4.6, 4.6, P)
    meta[:, 2] = rng.uniform(-4.6, 4.6, P)
    meta[:3, 1] = [0.5, -0.5, 2.5][:P]  # C round(): halves away from zero
    meta[:, 3] = rng.uniform(8000, 30000, P)
    meta[:, 4] = meta[:, 3] - rng.uniform(0, 2000, P)
    meta[:, 5] = rng.uniform(0, 180, P)
    meta[:, 6:10] = [300., 2.7, 0.1, 40.]
    group = rng.integers(0, G, P).astype(np.int32)
    sig2 = rng.uniform(0.5, 2.0, (G, ori // 2 + 1)) / (ori * ori)
    sig2[0, 0] = 0.0  # a zero-sigma shell draws nothing
    sig2[-1, ori // 4] = 0.0
    return raw, meta, group, sig2


def oracle_opts(**kw):
    o = dict(avg_norm_correction=1.1, pixel_size=2.0, particle_diameter=90.0, width_mask_edge=4, sigma2_fudge=1.3,
             random_seed=7, do_norm_correction=True, do_zero_mask=False, do_ctf_correction=True)
    o.update(kw)
    return o


def compare(out, ref, tol=TOL):
    for name, key in (("Fimg_real", "Fimg"), ("Fimg_nomask_real", "Fimg_nomask")):
        r = ref[key]
        assert rel(out[name], r.real) < tol, name
        assert rel(out[name.replace("real", "imag")], r.imag) < tol, name
    assert rel(out["Fctf"], ref["Fctf"]) < tol
    assert np.array_equal(out["old_offsetx"], ref["old_offsetx"])
    assert np.array_equal(out["old_offsety"], ref["old_offsety"])
    if np.abs(ref["highres_Xi2"]).max() > 0:
        assert rel(out["highres_Xi2"], ref["highres_Xi2"]) < 1e-11
        assert rel(out["power_imgs"], ref["power_imgs"]) < 1e-11


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_norm_offsets_groups_against_oracle(ctx, dtype):
    P, ori, cur, G = 12, 48, 36, 3
    raw, meta, group, sig2 = synthetic(P, ori, G, 5, dtype)
    o = oracle_opts()
    ref = po.prepare_pool(raw, meta, group, sig2, cur, 100, o)
    out = prepare_particles(ctx, images_from(raw, meta, group, 100), opts_from(o), sig2, cur)
    compare(out, ref)
    assert out["old_offsetx"][0] == 1.0 and out["old_offsetx"][1] == -1.0 and out["old_offsetx"][2] == 3.0


def test_zero_mask_background_against_oracle(ctx):
    P, ori, cur, G = 6, 32, 32, 1
    raw, meta, group, sig2 = synthetic(P, ori, G, 6)
    o = oracle_opts(do_zero_mask=True, do_norm_correction=False)
    ref = po.prepare_pool(raw, meta, group, sig2, cur, 0, o)
    out = prepare_particles(ctx, images_from(raw, meta, group), opts_from(o), sig2, cur)
    compare(out, ref)
    assert np.all(out["highres_Xi2"] == 0) and np.all(out["power_imgs"] == 0)


@pytest.mark.parametrize("flags", [dict(ctf_phase_flipped=True), dict(only_flip_phases=True),
                                   dict(intact_ctf_first_peak=True), dict(do_ctf_correction=False)])
def test_ctf_options_against_oracle(ctx, flags):
    P, ori, cur, G = 4, 32, 24, 2
    raw, meta, group, sig2 = synthetic(P, ori, G, 8)
    o = oracle_opts(**flags)
    ref = po.prepare_pool(raw, meta, group, sig2, cur, 3, o)
    out = prepare_particles(ctx, images_from(raw, meta, group, 3), opts_from(o), sig2, cur)
    compare(out, ref)


def test_device_io_and_chunks():
    """Images on the device, outputs left on the device, and a workspace
    limit that splits the pool into chunks: rows at the chunk boundaries
    match the oracle run on those images alone (seed first_image + i)."""
    import torch
    from rome_b200.map2d import GpuContext
    P, ori, cur, G = 3000, 64, 56, 2
    limit = 64 << 20
    rng = np.random.default_rng(9)
    raw = rng.normal(size=(P, ori, ori)).astype(np.float32)
    meta = np.zeros((P, 10))
    meta[:, 0] = 1.0
    meta[:, 1:3] = rng.integers(-3, 4, (P, 2))
    meta[:, 3:10] = [15000., 14000., 30., 300., 2.7, 0.1, 0.]
    group = rng.integers(0, G, P).astype(np.int32)
    sig2 = np.full((G, ori // 2 + 1), 1.0 / (ori * ori))
    o = oracle_opts(do_norm_correction=False)
    with GpuContext(0, "fp32", workspace_limit=limit) as c:
        imgs = images_from(torch.from_numpy(raw).cuda(), meta, group, 11)
        dev = prepare_particles(c, imgs, opts_from(o), sig2, cur, on_device=True)
        host = prepare_particles(c, images_from(raw, meta, group, 11), opts_from(o), sig2, cur)
    for name in ("Fimg_real", "Fimg_nomask_imag", "Fctf"):
        assert np.array_equal(dev[name].cpu().numpy(), host[name]), name
    # the chunk size the library picks for host images (work buffers per image)
    n2, npix = ori * ori, ori * (ori // 2 + 1)
    per = n2 * 8 + npix * 16 + npix * 16 + n2 * 8 + n2 * 4
    cmax = max(1, min(P, limit // per))
    nchunk = -(-P // cmax)
    chunk = -(-P // nchunk)
    assert nchunk > 3
    rows = sorted({0, P - 1, chunk - 1, chunk, 2 * chunk - 1, 2 * chunk, (nchunk - 1) * chunk})
    for i in rows:
        ref = po.prepare_pool(raw[i:i + 1], meta[i:i + 1], group[i:i + 1], sig2, cur, 11 + i, o)
        one = {k: v[i:i + 1] for k, v in host.items()}
        compare(one, ref)


def test_bad_arguments_are_errors(ctx):
    from rome_b200.map2d import RomeError
    raw, meta, group, sig2 = synthetic(2, 32, 1, 1)
    o = oracle_opts()
    bad = meta.copy()
    bad[0, 8] = 1.5  # Q0 > 1: CTF::initialise refuses it
    with pytest.raises(RomeError):
        prepare_particles(ctx, images_from(raw, bad, group), opts_from(o), sig2, 32)
    with pytest.raises(RomeError):
        prepare_particles(ctx, images_from(raw, meta, group + 5), opts_from(o), sig2, 32)
    neg = opts_from(o)
    neg.random_seed = -10  # clock-seeded in the reference: not reproducible
    with pytest.raises(RomeError):
        prepare_particles(ctx, images_from(raw, meta, group), neg, sig2, 32)


@pytest.mark.parametrize("case", CASES)
def test_raw_images_to_estep_matches_reference(ctx, golden, case):
    """The pool prepared on the device from the raw images, handed to the
    E-step without leaving the device, reproduces the reference's E-step of
    that pool (diff2 of every pass, posterior sums, poses, model sums)."""
    from rome_b200.particles import prepared_pool
    from tests.test_gpu_map2d import DIFF2_TOL, SUM_TOL, check_diff2, check_poses
    from tests.util import golden_pool, relerr
    g = golden[case]
    p, proj, r_max = golden_pool(g)
    o = po.options_from_golden(g)
    ctx.set_projectors(proj, p.ori_size, r_max)
    imgs = images_from(g["pool0_raw_images"].astype(np.float64), g["pool0_prep_metadata"], g["pool0_group"],
                       int(g["pool0_first_image"][0]))
    sp = prepared_pool(ctx, p, imgs, opts_from(o))
    out = ctx.map2d_estep_pool(sp, checkpoints=True)
    for ip in range(p.npass()):
        check_diff2(out[f"diff2_{ip}"], g[f"pool0_pass{ip}_diff2"])
    last = f"pool0_pass{p.npass() - 1}_"
    assert relerr(out["min_diff2"], g[last + "min_diff2"]) < DIFF2_TOL
    assert relerr(out["sum_weight"], g[last + "sum_weight"]) < SUM_TOL
    frac = check_poses(out, g[last + "class"], g[last + "psi"], g[last + "xoff"], g[last + "yoff"], g[last + "weight"])
    assert frac >= 0.9
    for k in ["wsum_sigma2_noise", "wsum_pdf_class", "wsum_sigma2_offset", "wsum_sumw_group"]:
        assert relerr(out[k], g["pool0_after_update_" + k]) < SUM_TOL, k


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_size_128_against_oracle(ctx, dtype):
    """128^2 (the benchmark size, shared-memory transforms) with current_size
    < ori_size (power spectra, highres_Xi2), norm correction and offsets."""
    P, ori, cur, G = 3, 128, 100, 2
    raw, meta, group, sig2 = synthetic(P, ori, G, 12, dtype)
    o = oracle_opts(particle_diameter=150.0, pixel_size=1.5)
    ref = po.prepare_pool(raw, meta, group, sig2, cur, 40, o)
    out = prepare_particles(ctx, images_from(raw, meta, group, 40), opts_from(o), sig2, cur)
    compare(out, ref)
    assert np.abs(ref["highres_Xi2"]).max() > 0
