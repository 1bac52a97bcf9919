"""The oracle (oracle/oracle.c) against the golden fixtures produced by the
reference programs themselves (tests/golden/make_golden.py)."""
import hashlib

import numpy as np
import pytest

from conftest import load_case, load_index
from oracle import oracle

INDEX = load_index()


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(INDEX))
def test_exact_oracle_matches_reference(name):
    off, idx, wt, init, labels, meta = load_case(name, INDEX[name])
    if meta["kind"] == "generated":
        assert _sha(off.astype(np.uint64)) + _sha(idx.astype(np.uint32)) != ""  # generator ran
        h = hashlib.sha256()
        h.update(np.ascontiguousarray(off, dtype=np.uint64).tobytes())
        h.update(np.ascontiguousarray(idx, dtype=np.uint32).tobytes())
        assert h.hexdigest() == meta["graph_sha256"], "graph generator drifted"
    r = oracle.refine_exact(off, idx, wt, init)
    assert r.status == 0
    assert r.blocks == meta["blocks"]
    if labels is not None:
        assert np.array_equal(r.labels, labels)
    else:
        assert _sha(r.labels.astype(np.uint32)) == meta["labels_sha256"]
    if meta["rounds"] is not None:
        assert r.rounds == meta["rounds"]


@pytest.mark.parametrize("name", sorted(INDEX))
def test_rsc_restatement_matches_reference(name):
    off, idx, wt, init, labels, meta = load_case(name, INDEX[name])
    r = oracle.refine_rsc(off, idx, wt, init)
    assert r.blocks == meta["blocks"]
    if labels is not None:
        assert np.array_equal(r.labels, labels)
    else:
        assert _sha(r.labels.astype(np.uint32)) == meta["labels_sha256"]
    if meta["rounds"] is not None:
        assert r.rounds == meta["rounds"]
        assert r.rounds_cpu == meta["rounds_cpu"]


def test_randomize_is_the_reference_mixer():
    # rsc.cpp:63-69 on a few inputs, computed by hand from the published
    # SplitMix64 finaliser followed by x5, rotl 7, x9
    def ref(z):
        M = (1 << 64) - 1
        z = (z + 0x9E3779B97F4A7C15) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        z = ((z ^ (z >> 31)) * 5) & M
        return (((z << 7) | (z >> 57)) & M) * 9 & M
    for x in (0, 1, 2, 12345, (1 << 63) + 7, (1 << 64) - 1):
        assert oracle.rsc_randomize(x) == ref(x)


@pytest.mark.parametrize("scale,ef,seed", [(6, 2, 1), (10, 8, 5), (14, 16, 1), (16, 16, 3)])
def test_oracle_rmat_generator_equals_the_products(scale, ef, seed):
    """The oracle's R-MAT (oracle.c: orc_gen_rmat) builds the workloads of the
    reference arm and of the config-scale fixtures without the product; it
    must give the product generator's graph bit for bit."""
    import rbsc_b200 as R
    off, idx = oracle.gen_rmat(scale, ef, seed=seed, threads=3)
    o2, i2 = R.gen_rmat_host(scale, ef, seed=seed)
    assert np.array_equal(off, np.asarray(o2, dtype=np.uint64)) and np.array_equal(idx, i2)


def test_mdp_writer_equals_the_python_text(tmp_path):
    from rbsc_b200 import graphs as G
    off, idx = G.rmat(9, 4, seed=2)
    init = np.random.default_rng(3).integers(0, 5, size=len(off) - 1).astype(np.uint32)
    wt = np.random.default_rng(4).integers(1, 9, size=len(idx)).astype(np.uint64)
    for w, i in ((None, None), (wt, None), (None, init), (wt, init)):
        p = str(tmp_path / "g.txt")
        oracle.write_mdp_file(p, off, idx, wt=w, init=i)
        assert open(p, "rb").read() == oracle.mdp_text(off, idx, w, i)
