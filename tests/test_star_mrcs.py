"""STAR/MRCS pool loader (rome_b200/star_mrcs.py).

Pinned against the reference's own reads: tests/golden/map2d_*.npz record
the raw images, the metadata fields (NORM, CTF) and the group index of the
first pool exactly as the reference's driver read them from a seeded
dataset (tests/golden/make_golden.py writes that dataset with
rome_b200.synthetic).  The dataset is regenerated here from the same spec
and every recorded image must be found among the loader's particles, with
identical metadata and group (bit-exact; the reference shuffles the records
before forming pools, so the match is by image)."""
import dataclasses
import os
import sys

import numpy as np
import pytest

from rome_b200 import synthetic
from rome_b200.star_mrcs import ParticleStack, read_mrcs_header, read_star

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import CASES  # noqa: E402


@pytest.fixture(scope="module")
def datasets(tmp_path_factory):
    out = {}
    for name, (spec, _) in CASES.items():
        d = tmp_path_factory.mktemp(name)
        out[name] = synthetic.write_dataset_2d(str(d), spec)
    return out


@pytest.mark.parametrize("case", list(CASES))
def test_matches_reference_reads(datasets, golden, case):
    g = golden[case]
    st = ParticleStack(datasets[case])
    assert st.ori_size == g["pool0_raw_images"].shape[-1]
    assert st.nr_groups == int(g["nr_groups"][0])
    imgs = st.read_images(np.arange(st.nr_images)).astype(np.float64)
    flat = imgs.reshape(st.nr_images, -1)
    meta = g["pool0_prep_metadata"]
    for p, ref in enumerate(g["pool0_raw_images"]):
        hit = np.nonzero((flat == ref.reshape(1, -1)).all(axis=1))[0]
        assert hit.size == 1, (p, hit)
        i = int(hit[0])
        # columns 1-2 (offsets), and column 0 (NORM) under norm correction, hold the previous
        # iteration's estimates, not the values read
        if not int(g["do_norm_correction"][0]):
            assert st.norm[i] == meta[p, 0], (p, st.norm[i], meta[p])
        assert np.array_equal(st.ctf[i], meta[p, 3:10]), (p, st.ctf[i], meta[p])
        assert st.group[i] == g["pool0_group"][p]


def test_pools_cover_order_and_seed_offsets(datasets):
    st = ParticleStack(datasets["map2d_b"])
    full = st.read_images(np.arange(st.nr_images))
    rng = np.random.default_rng(4)
    order = rng.permutation(st.nr_images)
    seen = []
    for pool in st.pools(7, first=3, last=40, order=order, nbuf=2):
        assert pool.first_image == 3 + 7 * len(seen)
        rows = order[pool.first_image:pool.first_image + pool.nr_images]
        assert np.array_equal(pool.images, full[rows])
        assert np.array_equal(pool.ctf, st.ctf[rows]) and np.array_equal(pool.group, st.group[rows])
        seen.append(pool.nr_images)
    assert seen == [7, 7, 7, 7, 7, 2]


def test_sorted_by_micrograph_and_groups(tmp_path):
    imgs = np.arange(5 * 8 * 8, dtype=np.float32).reshape(5, 8, 8)
    synthetic.write_mrcs(str(tmp_path / "a.mrcs"), imgs)
    mics = ["m2", "m1", "m2", "m0", "m1"]
    with open(tmp_path / "p.star", "w") as f:
        f.write("\ndata_\n\nloop_\n_rlnMicrographName #2\n_rlnImageName #1\n_rlnDefocusU #3\n")
        for i, m in enumerate(mics):
            f.write(f"{i + 1:06d}@a.mrcs {m} {1000.0 + i:.6f}\n")
    st = ParticleStack(str(tmp_path / "p.star"))
    assert st.micrograph == ["m0", "m1", "m1", "m2", "m2"]          # stable sort by micrograph
    assert list(st.index) == [4, 2, 5, 1, 3]
    assert list(st.group) == [0, 1, 1, 2, 2] and st.nr_groups == 3  # one group name -> one group per micrograph
    assert np.array_equal(st.ctf[:, 0], [1003.0, 1001.0, 1004.0, 1000.0, 1002.0])
    assert np.array_equal(st.norm, np.ones(5)) and np.array_equal(st.ctf[:, 6], np.zeros(5))
    assert np.array_equal(st.read_images(np.arange(5)), imgs[st.index - 1])


def test_group_names_take_precedence(tmp_path):
    synthetic.write_mrcs(str(tmp_path / "a.mrcs"), np.zeros((4, 8, 8), np.float32))
    with open(tmp_path / "p.star", "w") as f:
        f.write("data_\nloop_\n_rlnImageName #1\n_rlnMicrographName #2\n_rlnGroupName #3\n")
        for i, (m, gname) in enumerate([("m0", "g1"), ("m1", "g0"), ("m2", "g1"), ("m3", "g0")]):
            f.write(f"{i + 1:06d}@a.mrcs {m} {gname}\n")
    st = ParticleStack(str(tmp_path / "p.star"))
    assert list(st.group) == [0, 1, 0, 1] and st.nr_groups == 2


def test_two_stacks_and_header(tmp_path):
    a = np.random.default_rng(1).standard_normal((3, 16, 16)).astype(np.float32)
    b = np.random.default_rng(2).standard_normal((2, 16, 16)).astype(np.float32)
    synthetic.write_mrcs(str(tmp_path / "a.mrcs"), a)
    synthetic.write_mrcs(str(tmp_path / "b.mrcs"), b)
    h = read_mrcs_header(str(tmp_path / "b.mrcs"))
    assert (h.nc, h.nr, h.ns, h.mode) == (16, 16, 2, 2)
    with open(tmp_path / "p.star", "w") as f:
        f.write("data_\nloop_\n_rlnImageName\n_rlnMicrographName\n")
        for name in ["2@b.mrcs", "1@a.mrcs", "3@a.mrcs", "1@b.mrcs"]:
            f.write(f"{name} mic0000\n")
    cols = read_star(str(tmp_path / "p.star"))
    assert cols["rlnImageName"][0] == "2@b.mrcs"
    st = ParticleStack(str(tmp_path / "p.star"))
    got = st.read_images(np.arange(4))
    assert np.array_equal(got, np.stack([b[1], a[0], a[2], b[0]]))


def test_errors(tmp_path):
    synthetic.write_mrcs(str(tmp_path / "a.mrcs"), np.zeros((2, 8, 8), np.float32))
    with open(tmp_path / "p.star", "w") as f:
        f.write("data_\nloop_\n_rlnImageName #1\n_rlnMicrographName #2\n000003@a.mrcs mic000000\n")
    with pytest.raises(ValueError, match="outside its stack"):
        ParticleStack(str(tmp_path / "p.star"))
    raw = bytearray(open(tmp_path / "a.mrcs", "rb").read())
    raw[12:16] = (1).to_bytes(4, "little")                      # MODE 1 (int16)
    open(tmp_path / "b.mrcs", "wb").write(bytes(raw))
    with open(tmp_path / "q.star", "w") as f:
        f.write("data_\nloop_\n_rlnImageName #1\n_rlnMicrographName #2\n000001@b.mrcs mic000000\n")
    with pytest.raises(ValueError, match="mode 1"):
        ParticleStack(str(tmp_path / "q.star"))
    with open(tmp_path / "r.star", "w") as f:
        f.write("data_\nloop_\n_rlnImageName #1\n_rlnMicrographName #2\n000001@a.mrcs mic000000\n"
                "000002@a.mrcs\n")
    with pytest.raises(ValueError, match="fields"):
        ParticleStack(str(tmp_path / "r.star"))


@pytest.mark.gpu
def test_device_pools_feed_the_preparation(datasets, golden):
    """Pools streamed to the device (page-locked double buffer, side-stream
    copies) carry the same images as the host read, and the device image
    preparation gives the same spectra from them as from host images."""
    import torch

    from rome_b200.map2d import GpuContext
    from rome_b200.particles import prepare_particles
    from test_gpu_prep import opts_from
    from oracle import prep_oracle as po

    g = golden["map2d_c"]
    st = ParticleStack(datasets["map2d_c"])
    full = st.read_images(np.arange(st.nr_images))
    opts = opts_from(po.options_from_golden(g))
    cur = int(g["current_size"][0])
    n = 0
    with GpuContext(0, "fp32") as ctx:
        for pool in st.device_pools(0, 5):
            assert isinstance(pool.images, torch.Tensor) and pool.images.is_cuda
            host = full[pool.first_image:pool.first_image + pool.nr_images]
            assert np.array_equal(pool.images.cpu().numpy(), host)
            a = prepare_particles(ctx, pool, opts, g["sigma2_noise"], cur)
            b = prepare_particles(ctx, dataclasses.replace(pool, images=host), opts, g["sigma2_noise"], cur)
            for k in ("Fimg_real", "Fimg_nomask_imag", "Fctf"):
                assert np.array_equal(a[k], b[k]), k
            n += pool.nr_images
    assert n == st.nr_images


def test_early_stop_leaves_no_reader(datasets):
    import threading
    st = ParticleStack(datasets["map2d_a"])
    before = threading.active_count()
    for pool in st.pools(4):
        break
    gen = st.pools(4)
    next(gen)
    gen.close()
    assert threading.active_count() == before
