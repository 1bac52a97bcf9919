"""Lumping with double weights: the oracle (oracle.c: orc_refine_f64) against
the fixtures made by Valmari's minimiser built with double weights
(tests/golden/make_f64_golden.py), and the CUDA path (rbsc_refine_f64, through
the C ABI) against both.  The compared values are float bit patterns and
integer labels: results must be identical."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle

sys.path.insert(0, GOLDEN)
import f64_cases  # noqa: E402

with open(os.path.join(GOLDEN, "f64.json")) as f:
    FIXTURES = json.load(f)


def _id(e):
    return e["name"] if e["kind"] == "known" else f"{e['kind']}{e['seed']}"


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def _case(e):
    (off, idx, texts), init = f64_cases.make(e)
    assert len(off) - 1 == e["n"] and int(off[-1]) == e["m"], "case generator drifted"
    return off, idx, texts, oracle.reader_decimals(texts), init


# ---- the oracle (CPU) ------------------------------------------------------

@pytest.mark.parametrize("e", FIXTURES, ids=_id)
def test_oracle_matches_reference_fixture(e):
    off, idx, texts, w, init = _case(e)
    r = oracle.refine_f64(off, idx, w, init)
    assert r.status == 0
    assert r.blocks == e["blocks"] and r.rounds == e["rounds"]
    assert _sha(r.labels) == e["labels_sha256"]


def test_reader_decimal_restatement():
    # reader.cc:110-147 adds digit x scale with scale /= 10 per digit: "0.3"
    # is not the nearest double to 0.3, "0.1" and "0.5" are
    v = oracle.reader_decimals(["0.3", "0.1", "0.5", "-0.5", "+-2", "12.75", "7", "0.001"])
    assert v[0] == 0.1 * 3 and v[0] != 0.3
    assert v[1] == 0.1 and v[2] == 0.5 and v[3] == -0.5 and v[4] == -2.0 and v[5] == 12.75 and v[6] == 7.0
    with pytest.raises(ValueError):
        oracle.reader_decimals(["x"])


def test_oracle_rounds_to_float():
    # true doubles 0.1 + 0.2 != 0.3, but the sums rounded to float are equal
    off = np.array([0, 2, 3, 3, 3, 3], dtype=np.uint64)
    idx = np.array([2, 3, 4], dtype=np.uint32)
    r = oracle.refine_f64(off, idx, np.array([0.1, 0.2, 0.3]))
    assert r.labels.tolist() == [0, 0, 2, 2, 2]
    # a difference above float resolution splits
    r = oracle.refine_f64(off, idx, np.array([0.1, 0.2, 0.3001]))
    assert r.labels.tolist() == [0, 1, 2, 2, 2]


@pytest.mark.skipif(not os.path.exists(oracle.REF_VALMARI_F64),
                    reason="oracle/_ref/ref_valmari_f64 not built (make -C oracle with the reference checkout)")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_live_reference(seed):
    (off, idx, texts), init = f64_cases.random_graph(900 + seed, 60 + 10 * seed, 4, 1 + seed % 3, 1 + seed % 2)
    ref = oracle.run_ref_valmari_f64(off, idx, texts, init)
    r = oracle.refine_f64(off, idx, oracle.reader_decimals(texts), init)
    assert r.blocks == ref.blocks and np.array_equal(r.labels, ref.labels)


# ---- the CUDA path -----------------------------------------------------------

@pytest.fixture(scope="module")
def ctx():
    import rbsc_b200 as R
    c = R.Context(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("e", FIXTURES, ids=_id)
def test_cuda_matches_reference_fixture(ctx, e):
    off, idx, texts, w, init = _case(e)
    r = ctx.refine_f64(off, idx, w, init)
    assert r.done == 1 and r.verified == 1 and r.repairs == 0
    assert r.blocks == e["blocks"] and r.rounds == e["rounds"]
    assert _sha(r.labels) == e["labels_sha256"]
    assert r.kernel_launches > 0


@pytest.mark.gpu
@pytest.mark.parametrize("ob", [4, 8])
def test_cuda_offsets_and_edge_cases(ctx, ob):
    dt = np.uint32 if ob == 4 else np.uint64
    # empty graph, nodes without arcs, one node
    r = ctx.refine_f64(np.zeros(1, dt), np.zeros(0, np.uint32), np.zeros(0))
    assert r.blocks == 0 and r.labels.size == 0
    r = ctx.refine_f64(np.zeros(6, dt), np.zeros(0, np.uint32), np.zeros(0), init=np.array([3, 1, 3, 2, 1], np.uint32))
    assert r.labels.tolist() == [0, 1, 0, 3, 1] and r.rounds == 1
    # true doubles: float rounding merges 0.1 + 0.2 with 0.3, not with 0.3001
    off = np.array([0, 2, 3, 3, 3, 3], dtype=dt)
    idx = np.array([2, 3, 4], dtype=np.uint32)
    assert ctx.refine_f64(off, idx, np.array([0.1, 0.2, 0.3])).labels.tolist() == [0, 0, 2, 2, 2]
    assert ctx.refine_f64(off, idx, np.array([0.1, 0.2, 0.3001])).labels.tolist() == [0, 1, 2, 2, 2]
    # sums of either zero sign are no arc
    off2 = np.array([0, 2, 3, 3, 3], dtype=dt)
    r = ctx.refine_f64(off2, np.array([2, 3, 2], np.uint32), np.array([0.5, -0.5, -0.0]))
    assert r.labels.tolist() == [0, 0, 0, 0]


@pytest.mark.gpu
def test_cuda_rejects_bad_weights(ctx):
    import rbsc_b200 as R
    off = np.array([0, 1, 1], dtype=np.uint64)
    idx = np.array([1], dtype=np.uint32)
    for bad in (np.nan, np.inf, -np.inf, 2.0 ** 970):
        with pytest.raises(R.RbscError) as ei:
            ctx.refine_f64(off, idx, np.array([bad]))
        assert ei.value.status == -1
    with pytest.raises(R.RbscError):  # a head >= n
        ctx.refine_f64(off, np.array([2], np.uint32), np.array([1.0]))
    # the context stays usable
    assert ctx.refine_f64(off, idx, np.array([1.0])).blocks == 2


@pytest.mark.gpu
@pytest.mark.parametrize("bits", [3, -1])
def test_cuda_exact_check_repairs_collisions(bits):
    # truncated (or no) signatures: the hashed passes merge classes, the exact
    # check finds every merge and the result is still the exact partition
    import rbsc_b200 as R
    e = FIXTURES[-1]
    off, idx, texts, w, init = _case(e)
    with R.Context(0, test_hash_bits=bits) as c:
        r = c.refine_f64(off, idx, w, init)
    # with no signatures at all every split after the initial colours comes
    # from a repair; 3-bit signatures change with the pass salt, so a false
    # merge of one pass is usually split by the next before any check
    assert r.verified == 1 and (r.repairs > 0 or bits > 0)
    assert r.blocks == e["blocks"] and _sha(r.labels) == e["labels_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(4))
def test_cuda_matches_oracle_random_weights(ctx, seed):
    # weights with many digits: few sums are equal by accident, many by lifting
    rng = np.random.default_rng(seed)
    (off, idx, _), init = f64_cases.lifted(500 + seed, 300, 40, 3, 2)
    base = rng.random(int(off[-1]))
    w = np.round(base * 1000) / 1000.0 if seed % 2 else base
    r = ctx.refine_f64(off, idx, w, init)
    o = oracle.refine_f64(off, idx, w, init)
    assert r.blocks == o.blocks and r.rounds == o.rounds and np.array_equal(r.labels, o.labels)


def test_bench_weight_texts_parse_exactly():
    # the bench's double-weight workload writes k/2 as "0.0" .. "4.0"; the
    # minimiser's reader must make exactly k/2 of them, the doubles given to
    # the CUDA path
    texts = [f"{x / 2:.1f}" for x in range(9)]
    v = oracle.reader_decimals(texts)
    assert all(v[i] == i / 2 for i in range(9))
