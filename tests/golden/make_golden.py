"""Generate the golden vectors of the MAP2D hot path from the reference itself.

Runs in a container that has the reference tree: builds oracle/_ref (the
reference's own sources, compiled by oracle/Makefile), writes seeded
synthetic datasets with rome_b200.synthetic, runs oracle/_ref/map2d_dump
(which drives the reference's Map2dOptimizer_old and records every E-step
stage of the first pool plus the M-step) and packs the arrays the tests
use into tests/golden/<case>.npz.

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py map2d_a    # one case

ROME_REFERENCE (or REF) names the reference tree oracle/Makefile compiles.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from rome_b200.map2d import load_dump  # noqa: E402
from rome_b200.synthetic import Map2dSpec, Map3dSpec, write_dataset_2d, write_dataset_3d  # noqa: E402

# (dataset spec, reference options)
CASES = {
    # small single-pass case, CTF on, iteration 2 (CTF-corrected references)
    "map2d_a": (Map2dSpec(n_particles=40, size=32, n_classes=2, n_blobs=8, blob_sigma=(1.5, 3.0), max_shift=2.0,
                          snr=0.2, pixel=4.0, seed=3),
                dict(K=2, iter=2, angpix=4.0, tau2_fudge=2, oversampling=0, pool=10, psi_step=30, offset_range=2,
                     offset_step=1, ctf=1)),
    # adaptive oversampling 1 (coarse + fine pass), 48^2, three classes, iteration 3
    "map2d_b": (Map2dSpec(n_particles=48, size=48, n_classes=3, n_blobs=10, blob_sigma=(1.5, 4.0), max_shift=3.0,
                          snr=0.1, pixel=3.0, seed=5),
                dict(K=3, iter=3, angpix=3.0, tau2_fudge=2, oversampling=1, pool=8, psi_step=20, offset_range=3,
                     offset_step=2, ctf=1)),
    # configuration-1 shapes at reduced count: 64^2, 10 deg psi, +-5 px step 1, no oversampling
    "map2d_c": (Map2dSpec(n_particles=36, size=64, n_classes=3, n_blobs=20, blob_sigma=(2.0, 6.0), max_shift=4.0,
                          snr=0.05, pixel=2.0, seed=1),
                dict(K=3, iter=2, angpix=2.0, tau2_fudge=2, oversampling=0, pool=6, psi_step=10, offset_range=5,
                     offset_step=1, ctf=1)),
    # norm correction (per-particle NORM and avg_norm_correction after iteration 1) and the zero mask
    # (zeros outside the particle instead of seeded noise), single pass
    "map2d_norm": (Map2dSpec(n_particles=40, size=32, n_classes=2, n_blobs=8, blob_sigma=(1.5, 3.0), max_shift=2.0,
                             snr=0.2, pixel=4.0, seed=4),
                   dict(K=2, iter=2, angpix=4.0, tau2_fudge=2, oversampling=0, pool=10, psi_step=30, offset_range=2,
                        offset_step=1, ctf=1, norm=1, zero_mask=1)),
}

# 3D cases: (dataset spec, reference options) for oracle/_ref/map3d_dump.  The reference fills a
# particle's power spectrum only when the current size is below the image size
# (setFourierTransforms, src/exp_model.h:568-571); at full size pool*_power_imgs holds whatever its
# buffer held, which nothing reads, so those bytes alone differ from one generation to the next.
CASES3D = {
    # HEALPix order 1 (48 directions, 12 psi), oversampling 1, +-2 px step 1, iteration 2
    "map3d_a": (Map3dSpec(n_particles=96, size=24, n_classes=2, n_blobs=10, blob_sigma=(1.2, 2.5), max_shift=2.0,
                          snr=2.0, pixel=4.0, seed=7),
                dict(K=2, iter=2, angpix=4.0, ini_high=16, tau2_fudge=2, oversampling=1, healpix_order=1, pool=4,
                     offset_range=2, offset_step=1, ctf=1, uniform_directions=1)),
    # the same shapes in cross-correlation mode (-always_cc: CC in the dumped iteration too)
    "map3d_cc": (Map3dSpec(n_particles=96, size=24, n_classes=2, n_blobs=10, blob_sigma=(1.2, 2.5), max_shift=2.0,
                           snr=2.0, pixel=4.0, seed=8),
                 dict(K=2, iter=2, angpix=4.0, ini_high=16, tau2_fudge=2, oversampling=1, healpix_order=1, pool=4,
                      offset_range=2, offset_step=1, ctf=1, uniform_directions=1, always_cc=1, dump_pools=6)),
    # intensity-scale correction (seven micrograph groups, per-group scales after iteration 1)
    "map3d_scale": (Map3dSpec(n_particles=96, size=24, n_classes=2, n_blobs=10, blob_sigma=(1.2, 2.5), max_shift=2.0,
                              snr=2.0, pixel=4.0, seed=9),
                    dict(K=2, iter=2, angpix=4.0, ini_high=16, tau2_fudge=2, oversampling=1, healpix_order=1,
                         pool=4, offset_range=2, offset_step=1, ctf=1, uniform_directions=1, scale=1)),
    # norm correction at 32^2 with the current size below the image size (30 of 32, coarse 12): the
    # windowing of the fine pass, the power-spectrum fill of storeWeightedSums and the new NORM
    "map3d_norm": (Map3dSpec(n_particles=96, size=32, n_classes=2, n_blobs=10, blob_sigma=(1.2, 2.5), max_shift=2.0,
                             snr=0.5, pixel=4.0, seed=13),
                   dict(K=2, iter=2, angpix=4.0, ini_high=24, tau2_fudge=2, oversampling=1, healpix_order=1,
                        pool=4, offset_range=2, offset_step=1, ctf=1, uniform_directions=1, norm=1)),
}
# 128^2 cases of the MAP3D configuration's shape (HEALPix order 2: 192 directions x 24 psi, 13
# translations, oversampling 1, fine pass at the full size, M-step into the pad-259 grid).  The
# whole dump (~1.2 GB: projectors and back-projectors at pad 259) is too large to commit: the
# fixture keeps every per-particle result, the model sums, checksums of the large arrays and the
# M-step outputs (class 0's map as float32), and the GPU tests regenerate the full dump from the
# same seeded dataset with oracle/_ref/map3d_dump (run_map3d_dump, M-step skipped) and check it
# against the fixture before comparing.
CASES3D_FULL = {
    # 24 particles in pools of 8 (every pool recorded), K=2, SNR 0.05, iteration 2 at full size
    "map3d_b": (Map3dSpec(n_particles=24, size=128, n_classes=2, n_blobs=60, blob_sigma=(2.0, 8.0), max_shift=4.0,
                          snr=0.05, pixel=1.5, seed=13),
                dict(K=2, iter=2, angpix=1.5, ini_high=30, tau2_fudge=2, oversampling=1, healpix_order=2, pool=8,
                     offset_range=4, offset_step=2, ctf=1, uniform_directions=1, full_size=1, light=1, dump_pools=3)),
}
# per-particle results and model sums copied whole from a CASES3D_FULL dump (name suffixes)
FULL_KEEP = ("min_diff2", "sum_weight", "significant_weight", "nr_sign", "pmax", "class", "rot", "tilt", "psi",
             "xoff", "yoff", "dLL", "norm_out", "wsum_norm_correction", "wsum_sigma2_noise", "wsum_pdf_class",
             "wsum_pdf_direction", "wsum_sigma2_offset", "wsum_sumw_group", "wsum_LL", "wsum_ave_Pmax",
             "current_size", "coarse_size", "nr_dir", "nr_psi", "nr_trans", "nr_images", "gridding_nr_iter",
             "minres_map", "do_map", "tau2_fudge_factor", "_count", "_after", "_before", "pdf_class",
             "projector_r_max", "projector_pad_size")
# large arrays represented by checksums (sum, sum of squares, element count)
FULL_CHECKSUM = ("projector_data", "iter_bp_data", "iter_bp_weight", "pass0_diff2_value", "pass1_diff2_value",
                 "pass0_weight_value", "pass1_weight_value", "Fimg_real", "Fimg_nomask_real", "Fctf",
                 "pass0_Mcoarse_significant")


def run_map3d_dump(name: str, out_dir: str, skip_mstep: bool = True, threads: int = 0) -> dict:
    """Write the seeded dataset of a CASES3D_FULL case under out_dir and run
    oracle/_ref/map3d_dump on it (the reference's own MAP3D path); returns
    the dump's arrays.  Used by make_case3d_full and by the GPU tests, which
    run it on the test machine (the binary is built from the reference here
    and travels with the repository; the reference tree itself is not read)."""
    from rome_b200.map2d import load_dump as _load
    spec, opt = CASES3D_FULL[name]
    os.makedirs(out_dir, exist_ok=True)
    star, ref = write_dataset_3d(os.path.join(out_dir, "data"), spec)
    dump = os.path.join(out_dir, "dump")
    cmd = [os.path.join(ROOT, "oracle", "_ref", "map3d_dump"), "-i", star, "-ref", ref, "-dump_dir", dump]
    for k, v in opt.items():
        cmd += [f"-{k}", str(v)]
    if skip_mstep:
        cmd += ["-skip_mstep", "1"]
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    subprocess.check_call(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env, cwd=out_dir)
    return _load(dump)


def checksum(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a, np.float64).ravel()
    return np.array([a.sum(), np.dot(a, a), a.size])


def make_case3d_full(name: str):
    tmp = tempfile.mkdtemp(prefix="rome_golden_")
    try:
        d = run_map3d_dump(name, tmp, skip_mstep=False)
        keep = {k: v for k, v in d.items() if k.endswith(FULL_KEEP) and v.nbytes <= (1 << 20)}
        for k, v in d.items():
            if k.endswith(FULL_CHECKSUM):
                keep["checksum_" + k] = checksum(v)
        keep["Irefs_after0_f32"] = d["Irefs_after"][0].astype(np.float32)
        keep["meta_options"] = np.array([str(CASES3D_FULL[name][1])])
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, **keep)
        print(f"{name}: {len(keep)} arrays, {os.path.getsize(out) / 1e6:.2f} MB")
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


# reconstruction at known poses: (dataset spec, rome_reconstruct options) for oracle/_ref/rome_reconstruct_ref
CASESRECON = {
    # 32^2 particles of one blob volume, CTF on, poses and origins from the generator, 10 gridding iterations
    "recon3d_a": (Map3dSpec(n_particles=300, size=32, n_classes=1, n_blobs=15, blob_sigma=(1.5, 3.0), max_shift=2.0,
                            snr=1.0, pixel=3.0, seed=11),
                  dict(angpix=3.0, ctf=1, iter=10)),
}

SKIP3D = ("Fimg_shifted_real", "Fimg_shifted_imag", "local_Fctf", "Minvsigma2", "local_sqrtXi2")
# cases whose fixture keeps the E-step records only: the whole-iteration back-projectors and the maps
# before and after the M-step are left out (no test of these cases reconstructs)
ESTEP_ONLY3D = ("map3d_norm",)
MSTEP3D = ("iter_bp_data", "iter_bp_weight", "Irefs_before", "Irefs_after")

# arrays copied from the dump into the fixture (the per-translation shifted
# images and per-orientation projections are large and are checked through
# the oracle instead)
SKIP_SUFFIXES = ("Fimg_shifted_real", "Fimg_shifted_imag", "Fref_real", "Fref_imag", "local_Fctf", "Minvsigma2")


def build_reference():
    ref = os.environ.get("ROME_REFERENCE") or os.environ.get("REF", "")
    subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", f"REF={ref}", "_ref/map2d_dump",
                           "_ref/map3d_dump",
                           "_ref/librome_oracle.so", "_ref/rome_reconstruct_ref"], stdout=subprocess.DEVNULL)


def make_case3d(name: str):
    spec, opt = CASES3D[name]
    tmp = tempfile.mkdtemp(prefix="rome_golden_")
    try:
        star, ref = write_dataset_3d(os.path.join(tmp, "data"), spec)
        dump = os.path.join(tmp, "dump")
        cmd = [os.path.join(ROOT, "oracle", "_ref", "map3d_dump"), "-i", star, "-ref", ref, "-dump_dir", dump]
        for k, v in opt.items():
            cmd += [f"-{k}", str(v)]
        env = dict(os.environ, OMP_NUM_THREADS="1")
        subprocess.check_call(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env, cwd=tmp)
        d = load_dump(dump)
        # the image norms of the CC denominator are kept where the dumped iteration runs in CC mode
        skip = tuple(x for x in SKIP3D if not (opt.get("always_cc") and x == "local_sqrtXi2"))
        if name in ESTEP_ONLY3D:
            skip += MSTEP3D
        keep = {k: v for k, v in d.items() if not k.endswith(skip)}
        keep["meta_options"] = np.array([str(opt)])
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, **keep)
        print(f"{name}: {len(keep)} arrays, {os.path.getsize(out) / 1e6:.2f} MB")
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def write_posed_star(path: str, mrcs: str, meta: dict, spec) -> None:
    """A particle STAR with the generating poses: rlnAngleRot/Tilt/Psi and
    rlnOriginX/Y = minus the generating shift (the offset that recentres the
    particle), plus the CTF columns."""
    labels = ["rlnImageName", "rlnMicrographName", "rlnDefocusU", "rlnDefocusV", "rlnDefocusAngle", "rlnVoltage",
              "rlnSphericalAberration", "rlnAmplitudeContrast", "rlnAngleRot", "rlnAngleTilt", "rlnAnglePsi",
              "rlnOriginX", "rlnOriginY"]
    with open(path, "w") as f:
        f.write("\ndata_\n\nloop_\n")
        for i, lab in enumerate(labels):
            f.write(f"_{lab} #{i + 1}\n")
        for p in range(len(meta["du"])):
            f.write(f"{p + 1:06d}@{mrcs} mic{p % 5:03d}.mrc {meta['du'][p]:.6f} {meta['dv'][p]:.6f} "
                    f"{meta['dang'][p]:.6f} {spec.voltage:.6f} {spec.cs:.6f} {spec.q0:.6f} {meta['rot'][p]:.6f} "
                    f"{meta['tilt'][p]:.6f} {meta['psi'][p]:.6f} {-meta['shx'][p]:.6f} {-meta['shy'][p]:.6f}\n")


def recon_dataset(name: str, out_dir: str) -> str:
    """Write the seeded dataset of a reconstruction case; returns the STAR path."""
    from rome_b200.synthetic import make_particles_3d, write_mrcs
    spec, _ = CASESRECON[name]
    os.makedirs(out_dir, exist_ok=True)
    imgs, meta, _ = make_particles_3d(spec)
    mrcs = os.path.abspath(os.path.join(out_dir, name + ".mrcs"))
    write_mrcs(mrcs, imgs, spec.pixel)
    star = os.path.join(out_dir, name + ".star")
    write_posed_star(star, mrcs, meta, spec)
    return star


def make_recon_case(name: str):
    """Run the reference's rome_reconstruct on the case's dataset and keep
    the reconstructed volume (float32, as the reference writes it)."""
    from rome_b200.star_mrcs import read_mrcs_header
    _, opt = CASESRECON[name]
    tmp = tempfile.mkdtemp(prefix="rome_golden_")
    try:
        star = recon_dataset(name, os.path.join(tmp, "data"))
        out = os.path.join(tmp, "recon")
        cmd = [os.path.join(ROOT, "oracle", "_ref", "rome_reconstruct_ref"), "-i", star, "-o", out]
        for k, v in opt.items():
            cmd += [f"-{k}", str(v)]
        env = dict(os.environ, OMP_NUM_THREADS="1")
        subprocess.check_call(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env, cwd=tmp)
        h = read_mrcs_header(out + ".mrc")
        vol = np.fromfile(out + ".mrc", "<f4", offset=1024).reshape(h.ns, h.nr, h.nc)
        dst = os.path.join(HERE, name + ".npz")
        np.savez_compressed(dst, vol=vol, meta_options=np.array([str(opt)]))
        print(f"{name}: volume {vol.shape}, {os.path.getsize(dst) / 1e6:.2f} MB")
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def make_case(name: str):
    spec, opt = CASES[name]
    tmp = tempfile.mkdtemp(prefix="rome_golden_")
    try:
        star = write_dataset_2d(os.path.join(tmp, "data"), spec)
        dump = os.path.join(tmp, "dump")
        cmd = [os.path.join(ROOT, "oracle", "_ref", "map2d_dump"), "-i", star, "-dump_dir", dump]
        for k, v in opt.items():
            cmd += [f"-{k}", str(v)]
        env = dict(os.environ, OMP_NUM_THREADS="1")
        subprocess.check_call(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, env=env, cwd=tmp)
        d = load_dump(dump)
        keep = {k: v for k, v in d.items() if not k.endswith(SKIP_SUFFIXES)}
        # a few shifted images / projections of pass 0 for the kernel-level checks
        keep["pass0_Fimg_shifted_real_t01"] = d["pass0_Fimg_shifted_real"][:, :2]
        keep["pass0_Fimg_shifted_imag_t01"] = d["pass0_Fimg_shifted_imag"][:, :2]
        keep["pool0_pass0_Fref_real_r01"] = d["pool0_pass0_Fref_real"][:, :2]
        keep["pool0_pass0_Fref_imag_r01"] = d["pool0_pass0_Fref_imag"][:, :2]
        keep["pass0_Minvsigma2"] = d["pass0_Minvsigma2"]
        keep["meta_options"] = np.array([str(opt)])
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, **keep)
        print(f"{name}: {len(keep)} arrays, {os.path.getsize(out) / 1e6:.2f} MB")
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    build_reference()
    names = sys.argv[1:] or list(CASES) + list(CASES3D) + list(CASESRECON) + list(CASES3D_FULL)
    for n in names:
        if n in CASES3D_FULL:
            make_case3d_full(n)
        elif n in CASESRECON:
            make_recon_case(n)
        elif n in CASES3D:
            make_case3d(n)
        else:
            make_case(n)
