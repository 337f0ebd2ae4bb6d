"""CPU: graph files of the reference's drivers.

DIMACS .gr -> RIPSCSR1 is pinned byte for byte to the reference's own
converter (gr_to_csr.cpp, compiled from its source into oracle/_ref by
oracle/Makefile), including its corner cases: repeated arcs, self-loops,
negative and fractional weights, CR line ends, unknown line kinds and a second
problem line.  The Lonestar / Galois binary .gr reader and writer are checked
against a numpy restatement of that layout (csr_graph.cpp:153-291: uint64
header {1, edge bytes, n, m}, uint64 row ends, uint32 destinations, padding to
8 bytes, edge data)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "gr_to_csr")

TRICKY = """c arcs with repeats, a self-loop, negative and fractional weights
p sp 7 12
a 1 2 3
a 1 2 1.5
a 2 2 4
a 3 1 -2
a 7 6 1e2\r
x a line of an unknown kind
a 4 5 0.1

a 5 4 7
a 4 5 0.05
a 6 7 2.25
c the end
"""


def _ref_convert(tmp_path, text, name="g"):
    if not os.path.exists(REF):
        pytest.skip("reference converter not built (needs the reference checkout)")
    gr = tmp_path / f"{name}.gr"
    gr.write_bytes(text.encode())
    out = tmp_path / f"{name}_ref.csrbin"
    r = subprocess.run([REF, str(gr), str(out)], capture_output=True, cwd=tmp_path)
    return gr, out, r.returncode


def _random_gr(seed, n=300, arcs=2500):
    rng = np.random.default_rng(seed)
    u = rng.integers(1, n + 1, arcs)
    v = rng.integers(1, n + 1, arcs)
    w = np.round(rng.uniform(-5, 50, arcs), 3)
    lines = [f"c random {seed}", f"p sp {n} {arcs + 7}"]
    lines += [f"a {a} {b} {float(c)!r}" for a, b, c in zip(u, v, w)]
    lines += [f"a {u[k]} {v[k]} {float(w[k]) - 1.0!r}" for k in range(0, arcs, 97)]   # repeats, smaller
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("case", ["tricky", "random", "restart"])
def test_dimacs_to_csrbin_matches_reference_converter(tmp_path, b2, case):
    text = {"tricky": TRICKY, "random": _random_gr(3),
            "restart": "p sp 3 2\na 1 2 1\np sp 4 1\na 2 3 5\na 4 1 2\n"}[case]
    gr, ref, rc = _ref_convert(tmp_path, text)
    assert rc == 0
    ours = tmp_path / "ours.csrbin"
    nnz = b2.dimacs_to_csrbin(str(gr), str(ours))
    assert ours.read_bytes() == ref.read_bytes()
    g, declared, loaded = b2.dimacs_read(str(gr))
    r = b2.csrbin_read(str(ref))
    assert g.orientation == "incoming" and g.m == nnz == r.m
    assert np.array_equal(g.rowptr, r.rowptr) and np.array_equal(g.colind, r.colind)
    assert np.array_equal(g.fweights.view(np.uint32), r.fweights.view(np.uint32))
    header = np.frombuffer(ref.read_bytes()[8:88], np.uint64)
    assert (declared, loaded) == (int(header[4]), int(header[5]))


def test_dimacs_reading_rules(tmp_path, b2):
    gr = tmp_path / "t.gr"
    gr.write_text(TRICKY)
    g, declared, loaded = b2.dimacs_read(str(gr))
    assert (g.n, declared, loaded) == (7, 12, 9)
    rows = {v: list(zip(g.colind[g.rowptr[v]:g.rowptr[v + 1]].tolist(),
                        g.fweights[g.rowptr[v]:g.rowptr[v + 1]].tolist())) for v in range(g.n)}
    assert rows[1] == [(0, 1.5), (1, 4.0)]          # repeated 1->2 keeps 1.5; self-loop 2->2 stays
    assert rows[0] == [(2, -2.0)] and rows[5] == [(6, 100.0)]
    assert rows[4] == [(3, np.float32(0.05))]        # repeated 4->5 keeps the smaller weight
    assert rows[6] == [(5, 2.25)] and rows[3] == [(4, 7.0)] and rows[2] == []


@pytest.mark.parametrize("text, status", [
    ("c no problem line\n", "INVALID_ARGUMENT"),
    ("a 1 2 3\np sp 3 1\n", "INVALID_ARGUMENT"),
    ("p sp 0 1\n", "INVALID_ARGUMENT"),
    ("p sp 3\n", "INVALID_ARGUMENT"),
    ("p sp 3 -1\n", "INVALID_ARGUMENT"),
    ("p sp 3 1\na 1 x 3\n", "INVALID_ARGUMENT"),
    ("p sp 3 1\na 0 2 3\n", "INVALID_INDEX"),
    ("p sp 3 1\na 1 4 3\n", "INVALID_INDEX"),
    ("p sp 3 1\na 1 2 inf\n", "INVALID_WEIGHT"),
    ("p sp 3 1\na 1 2 nan\n", "INVALID_WEIGHT"),
])
def test_dimacs_errors_match_reference(tmp_path, b2, text, status):
    from b200sssp import _lib
    gr, _, rc = _ref_convert(tmp_path, text)
    assert rc != 0                                    # the reference converter refuses it too
    with pytest.raises(_lib.B2Error) as e:
        b2.dimacs_read(str(gr))
    assert e.value.status == getattr(_lib, status)
    with pytest.raises(_lib.B2Error):
        b2.dimacs_to_csrbin(str(gr), str(tmp_path / "x.csrbin"))


def _lonestar_bytes(n, ends, dst, data=None, version=1, edge_bytes=None):
    """The Galois v1 layout, restated with numpy."""
    m = len(dst)
    eb = (4 if data is not None else 0) if edge_bytes is None else edge_bytes
    out = np.array([version, eb, n, m], np.uint64).tobytes()
    out += np.asarray(ends, np.uint64).tobytes() + np.asarray(dst, np.uint32).tobytes()
    if data is not None:
        if m % 2:
            out += b"\0\0\0\0"
        out += np.asarray(data).tobytes()
    return out


@pytest.mark.parametrize("m_odd", [False, True])
def test_lonestar_read_write_against_layout(tmp_path, b2, m_odd):
    g = b2.gen_er(200, 1501 if m_odd else 1500, 1, 100, seed=9)
    assert (g.m % 2 == 1) == m_odd
    ends = g.rowptr[1:]
    f = tmp_path / "f.gr"
    f.write_bytes(_lonestar_bytes(g.n, ends, g.colind, g.fweights.astype(np.float32)))
    r = b2.lonestar_read(str(f))
    assert r.orientation == "outgoing" and r.n == g.n
    assert np.array_equal(r.rowptr, g.rowptr) and np.array_equal(r.colind, g.colind)
    assert np.array_equal(r.fweights, g.fweights)
    ours = tmp_path / "ours.gr"
    b2.lonestar_write(str(ours), g)
    assert ours.read_bytes() == f.read_bytes()
    u = tmp_path / "u.gr"                              # uint32 edge data
    b2.lonestar_write(str(u), g, float_weights=False)
    assert u.read_bytes() == _lonestar_bytes(g.n, ends, g.colind, g.weights.astype(np.uint32))
    ru = b2.lonestar_read(str(u), float_weights=False)
    assert np.array_equal(ru.weights, g.weights) and np.array_equal(ru.fweights, g.weights.astype(np.float32))
    nw = tmp_path / "nw.gr"                            # no edge data: weight 1
    nw.write_bytes(_lonestar_bytes(g.n, ends, g.colind))
    r1 = b2.lonestar_read(str(nw))
    assert np.array_equal(r1.colind, g.colind) and np.all(r1.fweights == 1.0)


def test_lonestar_errors(tmp_path, b2):
    from b200sssp import _lib
    ends, dst, w = [2, 3, 3], [1, 2, 0], np.array([1.0, 2.0, 3.0], np.float32)
    cases = {
        "version": (_lonestar_bytes(3, ends, dst, w, version=2), _lib.INVALID_ARGUMENT),
        "edge bytes": (_lonestar_bytes(3, ends, dst, w, edge_bytes=8), _lib.INVALID_ARGUMENT),
        "truncated": (_lonestar_bytes(3, ends, dst, w)[:-4], _lib.INVALID_ARGUMENT),
        "destination": (_lonestar_bytes(3, ends, [1, 3, 0], w), _lib.INVALID_INDEX),
        "offsets": (_lonestar_bytes(3, [2, 1, 3], dst, w), _lib.INVALID_ROWPTR),
        "last offset": (_lonestar_bytes(3, [1, 2, 2], dst, w), _lib.INVALID_ROWPTR),
        "negative": (_lonestar_bytes(3, ends, dst, np.array([1, -1, 3], np.float32)), _lib.INVALID_WEIGHT),
        "nan": (_lonestar_bytes(3, ends, dst, np.array([1, np.nan, 3], np.float32)), _lib.INVALID_WEIGHT),
    }
    for name, (blob, status) in cases.items():
        f = tmp_path / "bad.gr"
        f.write_bytes(blob)
        with pytest.raises(_lib.B2Error) as e:
            b2.lonestar_read(str(f))
        assert e.value.status == status, name
    f = tmp_path / "ok.gr"
    f.write_bytes(_lonestar_bytes(3, ends, dst, w))
    assert b2.lonestar_read(str(f)).m == 3


def test_dimacs_to_lonestar_round_trip(tmp_path, b2):
    gr = tmp_path / "r.gr"
    gr.write_text(_random_gr(11).replace("-", ""))     # non-negative weights for the Lonestar reading
    g, _, _ = b2.dimacs_read(str(gr))
    out = g.transpose()
    out.fweights = out.fweights.astype(np.float32)
    f = tmp_path / "r_lonestar.gr"
    b2.lonestar_write(str(f), out)
    back = b2.lonestar_read(str(f)).transpose()
    assert np.array_equal(back.rowptr, g.rowptr) and np.array_equal(back.colind, g.colind)
    assert np.array_equal(back.fweights, g.fweights)


def test_reference_tiny_lonestar_file(b2, orc):
    """tests/golden/tiny.gr was written by the reference's own make_tiny_gr.py
    (tests/golden/make_golden.py): the reader gives its graph, the writer its
    bytes, and the oracle its expected distances (check_tiny_output.py:10)."""
    import json
    golden = os.path.join(ROOT, "tests", "golden")
    t = json.load(open(os.path.join(golden, "tiny_gr.json")))
    g = b2.lonestar_read(os.path.join(golden, "tiny.gr"))
    assert g.n == t["n"] and g.rowptr.tolist() == t["out_rowptr"] and g.colind.tolist() == t["out_colind"]
    assert g.fweights.tolist() == t["weights"]
    exp = np.array([np.inf if x is None else x for x in t["expected"]], np.float32)
    assert np.array_equal(orc.dijkstra(g.rowptr, g.colind, g.fweights, t["source"]), exp)
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "tiny.gr")
        b2.lonestar_write(out, g)
        assert open(out, "rb").read() == open(os.path.join(golden, "tiny.gr"), "rb").read()
