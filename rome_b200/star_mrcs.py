"""STAR metadata and MRCS particle stacks, read one pool at a time.

The reference reads every local image into host memory before the first
iteration (src/map3d_optimizer.cpp:267-327, the same in map2d_optimizer.cpp);
at 200,000 particles of 128^2 that is 13 GB per rank.  `ParticleStack`
instead keeps only the metadata resident and reads the images of one pool
at a time from memory-mapped stacks, into page-locked buffers that a
background thread fills for pool k + 1 while pool k is in use
(`ParticleStack.pools`); `ParticleStack.device_pools` also copies each pool
to the device on a side stream, so disk reads, host-to-device copies and the
caller's work on the previous pool overlap.  The pools are `ParticleImages`,
the input of the device image preparation (`rome_b200.particles`).

Reading rules restated from the reference:

* STAR (`MetaDataTable::readFromStar`, src/metadata.cpp:156-343): a header
  line containing ``_rln`` names a column, ``_rlnLabel #n`` with a 1-based
  column number, else the column is the header line's rank; the body starts
  at the first other line once at least two labels were seen and ends at the
  first line of 10 characters or fewer, or after as many lines as the file
  has lines containing ``.mrcs`` (`getImageNumber`, :519-526).  Unknown
  labels are skipped.
* Defaults of a record's fields when their column is absent
  (`METADATA_ELTS`, src/metadata.h:54-97): NormCorrection 1, OriginX/Y 0,
  the CTF fields 0, GroupNumber 1.
* ``rlnImageName`` is ``index@file``, split at the last ``@`` and the index
  read with `atoi` (`MetaName::set`, src/metadata.h:45-48).
* Records are stably sorted by micrograph name; groups are numbered 1, 2, ...
  in order of first appearance of rlnGroupName, and when every record has
  the same group name but there is more than one micrograph, each
  micrograph is its own group (metadata.cpp:290-334).  `group` holds
  GROUP_NO - 1, as the E-step's group index.
* MRCS (`Mrcs::readMrcsHead`, src/mrcs.cpp:28-38): the first 256 int32 of
  the header, NC (columns), NR (rows), NS (sections), MODE; only MODE 2
  (float32) is supported (src/mrcs.cpp:96).  Image ``index`` of a stack
  starts at byte (256 + (index - 1) * S^2) * 4
  (src/map3d_optimizer.cpp:305-313): the image data follow the 1024-byte
  header, and an extended header (NSYMBT) is not skipped, as in the
  reference.

The shuffle the reference's driver applies before dividing the particles
(`MetaDataTable::shuffle`) is the caller's: `pools` and `device_pools` read
records in the order given by `order` (default: the sorted STAR order).
"""
from __future__ import annotations

import dataclasses
import os
import threading
from typing import Dict, Iterator, List, Optional, Sequence

import numpy as np

from .particles import CTF_FIELDS, ParticleImages

__all__ = ["MrcsHeader", "read_mrcs_header", "read_star", "ParticleStack"]

#: STAR labels of ParticleImages.ctf, in CTF_FIELDS order (src/metadata.h:55-61)
CTF_LABELS = ("rlnDefocusU", "rlnDefocusV", "rlnDefocusAngle", "rlnVoltage", "rlnSphericalAberration",
              "rlnAmplitudeContrast", "rlnBfactor")
assert len(CTF_LABELS) == len(CTF_FIELDS)

MRC_HEADER_BYTES = 1024


@dataclasses.dataclass(frozen=True)
class MrcsHeader:
    nc: int      # columns (x)
    nr: int      # rows (y)
    ns: int      # sections (images in a stack)
    mode: int    # 2 = float32


def read_mrcs_header(path: str) -> MrcsHeader:
    """NC, NR, NS and MODE of an MRC/MRCS file (little-endian, as
    `Mrcs::readMrcsHead` reads it)."""
    with open(path, "rb") as f:
        raw = f.read(MRC_HEADER_BYTES)
    if len(raw) < MRC_HEADER_BYTES:
        raise ValueError(f"{path}: shorter than an MRC header ({len(raw)} bytes)")
    nc, nr, ns, mode = (int(v) for v in np.frombuffer(raw, "<i4", 4))
    return MrcsHeader(nc, nr, ns, mode)


def read_star(path: str) -> Dict[str, List[str]]:
    """The columns of a particle STAR file as lists of strings, keyed by
    label without the leading underscore (``rlnDefocusU`` ...), in file
    order."""
    with open(path, "r") as f:
        lines = f.read().split("\n")
    n_images = sum(1 for ln in lines if ".mrcs" in ln)
    columns: Dict[int, str] = {}
    n_columns = 0
    heads = 0
    pos = 0
    line = ""
    while pos < len(lines):
        line = lines[pos]
        pos += 1
        if "_rln" in line:
            label = line[line.find("_") + 1:].split(" ")[0].strip()
            if "#" in line:
                col = _atoi(line[line.find("#") + 1:]) - 1
            else:
                col = heads
            columns[col] = label
            n_columns = max(n_columns, col + 1)
            heads += 1
        elif heads > 1:
            break
    if heads == 0:
        raise ValueError(f"{path}: no _rln labels (star file format error)")
    out: Dict[str, List[str]] = {lab: [] for lab in columns.values()}
    body = 0
    while len(line) > 10 and body < n_images:
        fields = line.split()
        if len(fields) < n_columns:
            raise ValueError(f"{path}: body line {body + 1} has {len(fields)} fields, expected {n_columns}")
        for col, lab in columns.items():
            out[lab].append(fields[col])
        body += 1
        if pos >= len(lines):
            break
        line = lines[pos]
        pos += 1
    if body < n_images:
        raise ValueError(f"{path}: only {body} particle lines, expected {n_images}")
    return out


#: threads that copy one request's images out of the memory-mapped stacks
READ_THREADS = 4
_POOL = None
_POOL_LOCK = threading.Lock()


def _reader_pool():
    global _POOL
    with _POOL_LOCK:
        if _POOL is None:
            from concurrent.futures import ThreadPoolExecutor
            _POOL = ThreadPoolExecutor(max_workers=READ_THREADS, thread_name_prefix="mrcs-read")
        return _POOL


def _atoi(s: str) -> int:
    """C atoi: optional sign and leading digits, 0 if none."""
    s = s.strip()
    i = 1 if s[:1] in "+-" else 0
    j = i
    while j < len(s) and s[j].isdigit():
        j += 1
    return int(s[:j]) if j > i else 0


class ParticleStack:
    """A particle STAR file and the MRCS stacks it names, read pool by pool.

    Metadata arrays (one entry per particle, in the reference's sorted
    order): `index` (1-based image index in its stack), `stack` (index into
    `stack_paths`), `micrograph`, `norm`, `xoff`, `yoff`, `ctf` [N][7]
    (CTF_FIELDS order), `group` (GROUP_NO - 1), `nr_groups`.  Relative image
    paths are resolved against the STAR file's folder when they do not exist
    as given."""

    def __init__(self, star_path: str):
        cols = read_star(star_path)
        if "rlnImageName" not in cols:
            raise ValueError(f"{star_path}: no rlnImageName column")
        names = cols["rlnImageName"]
        n = len(names)
        mics = cols.get("rlnMicrographName", [""] * n)
        gnames = cols.get("rlnGroupName", [""] * n)
        order = sorted(range(n), key=lambda i: mics[i])      # stable: std::stable_sort on MICROGRAPH

        def col(label, default):
            v = cols.get(label)
            return np.full(n, default, np.float64) if v is None else np.asarray([float(x) for x in v])

        base = os.path.dirname(os.path.abspath(star_path))
        paths: List[str] = []
        path_id: Dict[str, int] = {}
        index = np.empty(n, np.int64)
        stack = np.empty(n, np.int32)
        for i, full in enumerate(names):
            at = full.rfind("@")
            index[i] = _atoi(full[:at]) if at >= 0 else 0
            fn = full[at + 1:]
            if fn not in path_id:
                path_id[fn] = len(paths)
                paths.append(fn if os.path.exists(fn) or os.path.isabs(fn) else os.path.join(base, fn))
            stack[i] = path_id[fn]
        o = np.asarray(order, np.int64)
        self.star_path = star_path
        self.stack_paths = paths
        self.index = index[o]
        self.stack = stack[o]
        self.micrograph = [mics[i] for i in order]
        self.norm = col("rlnNormCorrection", 1.0)[o]
        self.xoff = col("rlnOriginX", 0.0)[o]
        self.yoff = col("rlnOriginY", 0.0)[o]
        self.ctf = np.stack([col(lab, 0.0)[o] for lab in CTF_LABELS], axis=1) if n else np.zeros((0, 7))
        self.group, self.nr_groups = self._groups([gnames[i] for i in order], self.micrograph)
        self.columns = {k: [v[i] for i in order] for k, v in cols.items()}

        headers = [read_mrcs_header(p) for p in paths]
        if not headers:
            raise ValueError(f"{star_path}: no particles")
        h0 = headers[0]
        for p, h in zip(paths, headers):
            if h.mode != 2:
                raise ValueError(f"{p}: MRC mode {h.mode}; only mode 2 (float32) stacks are supported")
            if h.nc != h0.nc or h.nr != h0.nr or h.nc != h.nr:
                raise ValueError(f"{p}: images of {h.nc}x{h.nr}, expected square {h0.nc}x{h0.nc}")
        self.headers = headers
        self._size = h0.nc
        bad = np.nonzero((self.index < 1) | (self.index > np.asarray([headers[s].ns for s in self.stack])))[0]
        if bad.size:
            i = int(bad[0])
            raise ValueError(f"{star_path}: image {self.index[i]} of {paths[self.stack[i]]} is outside its stack "
                             f"of {headers[self.stack[i]].ns}")
        self._maps: Dict[int, np.memmap] = {}
        self._maps_lock = threading.Lock()

    @staticmethod
    def _groups(group_names: Sequence[str], mics: Sequence[str]):
        def number(keys):
            seen: Dict[str, int] = {}
            return np.asarray([seen.setdefault(k, len(seen)) for k in keys], np.int32), len(seen)

        g, ng = number(group_names)
        if ng == 1 and len(set(mics)) != 1:
            g, ng = number(mics)
        return g, ng

    @property
    def nr_images(self) -> int:
        return int(self.index.shape[0])

    @property
    def ori_size(self) -> int:
        return self._size

    def _map(self, s: int) -> np.memmap:
        # reader threads share the maps: one mapping per stack
        with self._maps_lock:
            m = self._maps.get(s)
            if m is None:
                S = self._size
                m = np.memmap(self.stack_paths[s], dtype="<f4", mode="r", offset=MRC_HEADER_BYTES,
                              shape=(self.headers[s].ns, S, S))
                self._maps[s] = m
            return m

    def read_images(self, rows: np.ndarray, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Images of the given particle rows, float32 [len(rows)][S][S];
        runs of consecutive images of one stack are read as one slice.  Large
        requests are split over `READ_THREADS` threads (the copies out of the
        memory-mapped stacks release the GIL), since one thread's copy from
        the page cache runs well below the host-to-device link."""
        rows = np.asarray(rows, np.int64)
        S = self._size
        if out is None:
            out = np.empty((rows.size, S, S), np.float32)
        nt = min(READ_THREADS, max(1, rows.size * S * S * 4 // (8 << 20)))
        if nt > 1:
            cuts = np.linspace(0, rows.size, nt + 1).astype(int)
            futs = [_reader_pool().submit(self._read_into, rows[a:b], out[a:b]) for a, b in zip(cuts[:-1], cuts[1:])]
            for f in futs:
                f.result()
            return out
        return self._read_into(rows, out)

    def _read_into(self, rows: np.ndarray, out: np.ndarray) -> np.ndarray:
        if rows.size and np.all(self.stack[rows] == self.stack[rows[0]]):
            # one stack (the usual case): one slice copy for consecutive images,
            # else a single gather in C, whatever the order
            mm, idx = self._map(int(self.stack[rows[0]])), self.index[rows] - 1
            if np.all(np.diff(idx) == 1):
                out[:] = mm[idx[0]:idx[0] + idx.size]
            else:
                # indices were range-checked when the STAR file was read; with
                # mode="clip" numpy gathers straight into `out` (the default
                # mode="raise" buffers the whole gather and copies it again)
                np.take(mm, idx, axis=0, out=out, mode="clip")
            return out
        i = 0
        while i < rows.size:
            s, first = int(self.stack[rows[i]]), int(self.index[rows[i]])
            j = i + 1
            while (j < rows.size and self.stack[rows[j]] == s and self.index[rows[j]] == first + (j - i)):
                j += 1
            out[i:j] = self._map(s)[first - 1:first - 1 + (j - i)]
            i = j
        return out

    def particles(self, rows: np.ndarray, images: np.ndarray, first_image: int) -> ParticleImages:
        rows = np.asarray(rows, np.int64)
        return ParticleImages(images=images, norm=self.norm[rows].copy(), xoff=self.xoff[rows].copy(),
                              yoff=self.yoff[rows].copy(), ctf=self.ctf[rows].copy(),
                              group=self.group[rows].copy(), first_image=first_image)

    def _ranges(self, pool: int, first: int, last: Optional[int]):
        last = self.nr_images if last is None else last
        if not (0 <= first <= last <= self.nr_images) or pool < 1:
            raise ValueError(f"bad range [{first}, {last}) or pool {pool} for {self.nr_images} particles")
        return [(lo, min(lo + pool, last)) for lo in range(first, last, pool)]

    def pools(self, pool: int, first: int = 0, last: Optional[int] = None, order: Optional[np.ndarray] = None,
              pinned: bool = False, nbuf: int = 2) -> Iterator[ParticleImages]:
        """ParticleImages of consecutive pools of `pool` particles over
        positions [first, last) of `order` (default: the STAR order).
        `first_image` is the pool's first position (the noise seed offset of
        the preparation).  A background thread reads the next pool while the
        caller holds the current one; the images live in a ring of `nbuf`
        buffers (page-locked when `pinned`), so a yielded pool's images are
        overwritten `nbuf - 1` pools later: copy them before then if they
        must outlive that."""
        if nbuf < 2:
            raise ValueError("nbuf must be at least 2")
        order = np.arange(self.nr_images) if order is None else np.asarray(order, np.int64)
        ranges = self._ranges(pool, first, last)
        if not ranges:
            return
        bufs = [self._buffer(min(pool, ranges[0][1] - ranges[0][0]), pinned) for _ in range(nbuf)]
        result: List[Optional[object]] = [None] * len(ranges)

        def load(q):
            lo, hi = ranges[q]
            try:
                result[q] = self.read_images(order[lo:hi], out=bufs[q % nbuf][:hi - lo])
            except BaseException as e:   # handed to the consumer
                result[q] = e

        th = threading.Thread(target=load, args=(0,))
        th.start()
        try:
            for q, (lo, hi) in enumerate(ranges):
                th.join()
                imgs = result[q]
                result[q] = None
                if isinstance(imgs, BaseException):
                    raise imgs
                if q + 1 < len(ranges):
                    th = threading.Thread(target=load, args=(q + 1,))
                    th.start()
                yield self.particles(order[lo:hi], imgs, lo)
        finally:
            th.join()   # a consumer that stops early leaves no reader behind

    def device_pools(self, device: int, pool: int, first: int = 0, last: Optional[int] = None,
                     order: Optional[np.ndarray] = None) -> Iterator[ParticleImages]:
        """As `pools`, with the images of each pool as a float32 CUDA tensor
        on `device`.  While the caller works on pool k, pool k + 1 is being
        copied from its page-locked buffer on a side stream and pool k + 2
        read from disk into the other buffer.  Each copy is complete before
        the caller receives its pool and before its buffer is refilled (two
        pools later), so two page-locked buffers suffice."""
        import torch
        dev = torch.device("cuda", device)
        side = torch.cuda.Stream(device=dev)
        consumer = torch.cuda.current_stream(dev)
        prev = None
        for host in self.pools(pool, first, last, order, pinned=True, nbuf=2):
            with torch.cuda.stream(side):
                t = torch.from_numpy(host.images).to(dev, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(side)
            # allocated on the side stream, used on the caller's: the allocator
            # must not hand the block back to the side stream before the
            # caller's work on it is done
            t.record_stream(consumer)
            if prev is not None:
                yield prev
            ev.synchronize()
            prev = dataclasses.replace(host, images=t)
        if prev is not None:
            yield prev

    def _buffer(self, n: int, pinned: bool) -> np.ndarray:
        S = self._size
        if pinned:
            import torch
            return torch.empty((n, S, S), dtype=torch.float32, pin_memory=True).numpy()
        return np.empty((n, S, S), np.float32)
