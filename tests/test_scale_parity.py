"""Parity at the benchmark configurations' own sizes, against the reference
programs (tests/golden/scale.json, made by tests/golden/make_scale_golden.py).

  rmat24_ef16    R-MAT scale 24, edge factor 16, degree-bucket colours: the
                 partition agreed by Valmari's exact minimiser, the reference rsc
                 and the rsc restatement; rounds in the GPU program's convention.
  wl_batch_100k  100,000 small graphs side by side, labels U{1..8}: Valmari and
                 the rsc restatement on the union; per-graph block counts.
  rmat28_ef32    R-MAT scale 28, edge factor 32, arcs in page-locked host memory
                 (streamed in batches of 25 % of the arcs): the rsc restatement
                 with 64-bit counters, run on the host cores.

Each test regenerates the input with the library's generator, checks its
checksum against the fixture's (the same input the oracles saw), refines it
on the GPU and compares the canonical labels (sha256), the block count and
the round count: zero tolerance."""
import hashlib
import json
import os

import numpy as np
import pytest

import rbsc_b200 as R
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

_P = os.path.join(GOLDEN, "scale.json")
FX = json.load(open(_P)) if os.path.exists(_P) else {}


def _sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        flat = np.ascontiguousarray(a).reshape(-1).view(np.uint8)
        for i in range(0, flat.size, 1 << 28):
            h.update(flat[i: i + (1 << 28)])
    return h.hexdigest()


class _Dev:
    """A numpy-less view of device memory for torch (raw address, count, type)."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False), "version": 3}


def _need(name):
    if name not in FX:
        pytest.skip(f"tests/golden/scale.json has no entry {name} (made by tests/golden/make_scale_golden.py)")
    return FX[name]


def test_rmat24_matches_the_reference_programs():
    import torch
    fx = _need("rmat24_ef16")
    with R.Context(0) as ctx:
        g = ctx.gen_rmat(24, 16, seed=1)
        n, m = g.n, g.m
        assert (n, m) == (fx["n"], fx["m"])
        d_off, d_idx = g.device_csr()
        off = torch.as_tensor(_Dev(d_off, n + 1, "<u8"), device="cuda").cpu().numpy()
        idx = torch.as_tensor(_Dev(d_idx, m, "<u4"), device="cuda").cpu().numpy()
        assert _sha(off, idx) == fx["graph_sha256"]
        d_init = torch.empty(n, dtype=torch.int32, device="cuda")
        d_out = torch.empty(n, dtype=torch.int32, device="cuda")
        g.degree_colors_device(d_init.data_ptr())
        r = g.refine_device(d_init.data_ptr(), d_out.data_ptr())
        labels = d_out.cpu().numpy().view(np.uint32)
        assert r.verified == 1 and r.done == 1
        assert r.blocks == fx["blocks"] and r.rounds == fx["rounds"]
        assert _sha(labels) == fx["labels_sha256"]
        init = d_init.cpu().numpy().view(np.uint32)
        g.free()
        # the one-shot call from host arrays (the bench's end-to-end path)
        r1 = ctx.refine(off, idx, init=init)
        assert r1.blocks == fx["blocks"] and r1.rounds == fx["rounds"] and _sha(r1.labels) == fx["labels_sha256"]


def test_wl_batch_100k_matches_valmari():
    fx = _need("wl_batch_100k")
    off, idx, gn, lab = R.gen_wl_batch(fx["graphs"], fx["nmin"], fx["nmax"], fx["num_labels"], seed=fx["seed"])
    assert _sha(off.astype(np.uint64), idx.astype(np.uint32), gn.astype(np.uint64), lab.astype(np.uint32)) == \
        fx["graph_sha256"]
    with R.Context(0) as ctx:
        b = ctx.batch_refine(off, idx, gn, lab)
    assert _sha(b.colors.astype(np.uint32)) == fx["labels_sha256"]
    assert _sha(b.blocks.astype(np.uint32)) == fx["per_graph_blocks_sha256"]
    assert b.stats.rounds == fx["rounds"]


def test_rmat28_streamed_matches_the_restatement():
    import torch
    fx = _need("rmat28_ef32")
    with R.Context(0) as ctx:
        pg = ctx.gen_rmat_pinned(28, 32, seed=1)
        try:
            assert (pg.n, pg.m) == (fx["n"], fx["m"])
            assert _sha(np.asarray(pg.off, dtype=np.uint64)) == fx["offsets_sha256"]
            g = ctx.upload_streamed(pg.off, pg.idx)
            d_init = torch.empty(pg.n, dtype=torch.int32, device="cuda")
            d_out = torch.empty(pg.n, dtype=torch.int32, device="cuda")
            g.degree_colors_device(d_init.data_ptr())
            r = g.refine_device(d_init.data_ptr(), d_out.data_ptr())
            assert r.streamed_passes >= 1
            labels = d_out.cpu().numpy().view(np.uint32)
            g.free()
        finally:
            pg.free()
            ctx.trim()
    assert r.verified == 1 and r.blocks == fx["blocks"] and r.rounds == fx["rounds"]
    assert _sha(labels) == fx["labels_sha256"]
