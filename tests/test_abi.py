"""C ABI checks that need no GPU: librbsc.so loads, exports every function
include/rbsc.h declares, and its host-only entry points (arcs-cuda parser,
host R-MAT generator) behave; the CLI fails loudly without a device."""
import os
import re
import subprocess

import numpy as np
import pytest

from rbsc_b200 import _lib, graphs as G
import rbsc_b200 as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "rbsc.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rbsc_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.EXPORTED)
    assert lib.rbsc_abi_version() == 1


def test_exports_via_nm():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    syms = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    for name in _declared():
        assert name in syms, name


def test_no_device_gives_error_not_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(R.RbscError):
        R.Context(0)


def test_parse_arcs_roundtrip():
    off, idx = G.rmat(8, 4, seed=1)
    from oracle import oracle
    text = oracle.arcs_cuda_text(off, idx)
    o2, i2, w2 = R.parse_arcs(text)
    assert np.array_equal(off, o2) and np.array_equal(idx, i2) and w2 is None


def test_parse_weighted_and_unsorted_groups():
    text = b"4\n5\n2 3 0\n2 1 1\n0 7 3\n3 1 1\n1 1 2\n"
    off, idx, wt = R.parse_arcs(text)
    assert off.tolist() == [0, 1, 2, 4, 5]
    assert idx.tolist() == [3, 2, 0, 1, 1]
    assert wt.tolist() == [7, 1, 3, 1, 1]


@pytest.mark.parametrize("text,msg", [
    (b"3\n2\n0 1 1\n", "arcs"),                 # fewer arcs than announced
    (b"3\n1\n0 1 5\n", "range"),                # head out of range
    (b"3\n2\n0 1 1\n0 x 2\n", "malformed"),     # bad token
    (b"3\n3\n0 1 1\n1 1 2\n0 1 2\n", "grouped"),  # source 0 split in two runs
    (b"", "node count"),
])
def test_parse_rejects_malformed(text, msg):
    with pytest.raises(R.RbscError) as e:
        R.parse_arcs(text)
    assert msg in str(e.value)


def test_parse_no_trailing_newline():
    off, idx, wt = R.parse_arcs(b"2\n1\n0 1 1")
    assert off.tolist() == [0, 1, 1] and idx.tolist() == [1]


@pytest.mark.parametrize("scale,ef,seed", [(6, 4, 1), (10, 16, 3), (12, 8, 9)])
def test_host_rmat_matches_numpy(scale, ef, seed):
    o1, i1 = G.rmat(scale, ef, seed=seed)
    o2, i2 = R.gen_rmat_host(scale, ef, seed=seed)
    assert np.array_equal(o1, o2) and np.array_equal(i1, i2)


def test_cli_fails_loudly_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    r = subprocess.run([_lib.CLI_PATH], input=b"2\n1\n0 1 1\n", capture_output=True, timeout=60)
    assert r.returncode != 0
    assert b"CUDA" in r.stdout or b"failed" in r.stdout


def test_cli_parse_error_on_stdout():
    r = subprocess.run([_lib.CLI_PATH], input=b"2\n3\n0 1 1\n", capture_output=True, timeout=60)
    assert r.returncode != 0 and b"input error" in r.stdout


def test_csr_cache_roundtrip_and_checks(tmp_path):
    import rbsc_b200 as R
    from rbsc_b200 import graphs as G
    off, idx = G.rmat(10, 8, seed=2)
    wt = np.arange(len(idx), dtype=np.uint64) % 5 + 1
    for w in (None, wt):
        p = str(tmp_path / ("g_w.csr" if w is not None else "g.csr"))
        R.save_csr(p, off, idx, w)
        o2, i2, w2 = R.load_csr(p)
        assert np.array_equal(o2, off) and np.array_equal(i2, idx)
        assert (w2 is None) if w is None else np.array_equal(w2, w)
    # a flipped byte, a truncated file, a foreign file
    raw = bytearray(open(str(tmp_path / "g.csr"), "rb").read())
    raw[-1] ^= 0x40
    open(str(tmp_path / "bad.csr"), "wb").write(bytes(raw))
    open(str(tmp_path / "short.csr"), "wb").write(bytes(raw[:-3]))
    open(str(tmp_path / "text.csr"), "wb").write(b"3\n1\n0 1 2\n")
    for name in ("bad.csr", "short.csr", "text.csr"):
        with pytest.raises(R.RbscError):
            R.load_csr(str(tmp_path / name))


def _arcs_text(n, rows, weights=None):
    """arcs-cuda text with the rows given as (u, heads) in the listed order."""
    lines, m = [], 0
    for u, heads in rows:
        for j, v in enumerate(heads):
            w = 1 if weights is None else weights(u, j)
            lines.append(f"{u} {w} {v}")
            m += 1
    return (f"{n}\n{m}\n" + "\n".join(lines) + "\n").encode()


def _csr_of(n, rows, weights=None):
    deg = np.zeros(n + 1, dtype=np.uint64)
    for u, heads in rows:
        deg[u + 1] = len(heads)
    off = np.cumsum(deg, dtype=np.uint64)
    idx = np.zeros(int(off[-1]), dtype=np.uint32)
    wt = np.ones(int(off[-1]), dtype=np.uint64)
    for u, heads in rows:
        idx[off[u]:off[u + 1]] = heads
        if weights is not None:
            wt[off[u]:off[u + 1]] = [weights(u, j) for j in range(len(heads))]
    return off, idx, wt


def test_parse_large_unsorted_groups_across_threads():
    """More than 1 MB of text (parsed by several threads): rows in random
    order, one row long enough to cross chunk boundaries, weights other than 1
    only near the end."""
    rng = np.random.default_rng(5)
    n = 40000
    rows = [(u, rng.integers(0, n, size=int(rng.integers(1, 12)))) for u in range(0, n, 2)]
    rows.append((1, rng.integers(0, n, size=200000)))  # ~2 MB of one row
    order = rng.permutation(len(rows))
    rows = [rows[i] for i in order]
    late = {u for u, _ in rows[-50:]}
    wfun = lambda u, j: (j % 5) + 2 if u in late else 1
    text = _arcs_text(n, rows, wfun)
    assert len(text) > (1 << 21)
    off, idx, wt = R.parse_arcs(text)
    eo, ei, ew = _csr_of(n, rows, wfun)
    assert np.array_equal(off, eo) and np.array_equal(idx, ei) and np.array_equal(wt, ew)
    # unit weights: no weight array; sorted rows: the same CSR
    text = _arcs_text(n, sorted(rows, key=lambda r: r[0]))
    off, idx, wt = R.parse_arcs(text)
    assert wt is None and np.array_equal(off, eo) and np.array_equal(idx, ei)


def test_parse_rejects_a_group_split_across_threads():
    rng = np.random.default_rng(6)
    n = 30000
    rows = [(u, rng.integers(0, n, size=8)) for u in range(1, n)]
    rows = [(0, [1, 2])] + rows + [(0, [3])]
    with pytest.raises(R.RbscError) as e:
        R.parse_arcs(_arcs_text(n, rows))
    assert "grouped" in str(e.value)


def test_parse_long_numbers():
    big = (1 << 64) - 1
    off, idx, wt = R.parse_arcs(f"3\n2\n0 {big} 00000000000000000000002\n2 0000000000000000000000007 1\n".encode())
    assert idx.tolist() == [2, 1] and wt.tolist() == [big, 7]
    with pytest.raises(R.RbscError):
        R.parse_arcs(f"3\n1\n0 {big + 1} 2\n".encode())


def test_csr_cache_reads_version_1_files(tmp_path):
    """Files of the first format version (FNV-1a 64 over every byte) still
    load; a wrong checksum is still refused."""
    import struct
    off = np.array([0, 2, 3, 3], dtype=np.uint64)
    idx = np.array([1, 2, 0], dtype=np.uint32)
    payload = off.tobytes() + idx.tobytes()
    h = 0xcbf29ce484222325
    for b in payload:
        h = ((h ^ b) * 0x100000001b3) & 0xFFFFFFFFFFFFFFFF
    head = b"RBSCCSR1" + struct.pack("<IIQQQ", 1, 0, 3, 3, h) + bytes(24)
    p = str(tmp_path / "v1.csr")
    open(p, "wb").write(head + payload)
    o2, i2, w2 = R.load_csr(p)
    assert o2.tolist() == off.tolist() and i2.tolist() == idx.tolist() and w2 is None
    head = b"RBSCCSR1" + struct.pack("<IIQQQ", 1, 0, 3, 3, h ^ 1) + bytes(24)
    open(p, "wb").write(head + payload)
    with pytest.raises(R.RbscError):
        R.load_csr(p)


@pytest.mark.parametrize("weighted", [False, True], ids=["unit", "weighted"])
def test_parse_large_sorted_input_with_blank_lines(weighted):
    """More than 1 MB of text in source order, parsed by several threads
    straight into the heads array, with blank (and blank-looking) lines
    sprinkled through every chunk: the gaps they leave are closed and the CSR
    equals the one without them."""
    rng = np.random.default_rng(8)
    n = 60000
    rows = [(u, rng.integers(0, n, size=int(rng.integers(1, 9)))) for u in range(n)]
    wfun = (lambda u, j: (u + j) % 3 + 1) if weighted else None
    lines = _arcs_text(n, rows, wfun).decode().split("\n")
    body = []
    for k, ln in enumerate(lines[2:]):
        body.append(ln)
        if k % 97 == 0:
            body.append("" if k % 2 else "  \t")
    text = ("\n".join(lines[:2] + body)).encode()
    assert len(text) > (1 << 20)
    off, idx, wt = R.parse_arcs(text)
    eo, ei, ew = _csr_of(n, rows, wfun)
    assert np.array_equal(off, eo) and np.array_equal(idx, ei)
    if weighted:
        assert np.array_equal(wt, ew)
    else:
        assert wt is None
