"""C ABI library: loads, exports every declared symbol, host-side logic (CPU only)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def _header_functions():
    src = open(os.path.join(ROOT, "include", "b200sssp.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(b2_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol(b2):
    from b200sssp import _lib
    L = _lib.lib()
    declared = _header_functions()
    assert len(declared) >= 25
    for name in declared:
        assert hasattr(L, name), name
    assert set(declared) == set(_lib.declared_symbols())
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (b2_[a-z0-9_]+)$", out, flags=re.M))
    assert set(declared) <= exported


def test_status_strings_and_defaults(b2):
    from b200sssp import _lib
    assert _lib.lib().b2_abi_version() == 1
    for s in range(12):
        assert _lib.status_string(s) and "unknown" not in _lib.status_string(s)
    import ctypes
    o = _lib.Opts()   # the library's own defaults (default_opts() also applies B2_TIMEOUT_MS)
    _lib.lib().b2_sssp_opts_default(ctypes.byref(o))
    assert o.max_iters == -1 and o.delta_scale == 16.0 and o.timeout_ms == 20000.0 and o.hub_degree == 256
    assert o.pull_fraction == 8.0 and o.dense_fraction == 0.0 and o.light_heavy == 1   # 0: by graph degree


def test_generators_deterministic_and_thread_independent(b2, monkeypatch):
    a = b2.gen_rmat(12, 8, seed=3)
    monkeypatch.setenv("B2_GEN_THREADS", "1")
    b = b2.gen_rmat(12, 8, seed=3)
    monkeypatch.setenv("B2_GEN_THREADS", "7")
    c = b2.gen_rmat(12, 8, seed=3)
    for x in (b, c):
        assert np.array_equal(a.rowptr, x.rowptr) and np.array_equal(a.colind, x.colind)
        assert np.array_equal(a.weights, x.weights)
    g1 = b2.gen_grid(40, 50, seed=2)
    monkeypatch.setenv("B2_GEN_THREADS", "3")
    g2 = b2.gen_grid(40, 50, seed=2)
    assert np.array_equal(g1.weights, g2.weights) and np.array_equal(g1.colind, g2.colind)


def _mix64(z):
    z = (z + np.uint64(0x9E3779B97F4A7C15))
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def test_er_generator_matches_numpy_restatement(b2):
    n, m, seed = 500, 3000, 9
    with np.errstate(over="ignore"):
        base = _mix64(np.uint64(seed) ^ (np.uint64(1) * np.uint64(0xD1B54A32D192ED03)))
        i = np.arange(4 * m, dtype=np.uint64)
        r = _mix64(base + i)
        u = ((r >> np.uint64(32)) * np.uint64(n)) >> np.uint64(32)
        v = ((r & np.uint64(0xFFFFFFFF)) * np.uint64(n)) >> np.uint64(32)
    keys = []
    seen = set()
    for a, b_ in zip(u.tolist(), v.tolist()):
        if a == b_ or (a, b_) in seen:
            continue
        seen.add((a, b_))
        keys.append((a, b_))
        if len(keys) == m:
            break
    keys.sort()
    g = b2.gen_er(n, m, 1, 100, seed)
    got = [(uu, int(g.colind[e])) for uu in range(n) for e in range(g.rowptr[uu], g.rowptr[uu + 1])]
    assert got == keys


def test_rmat_properties(b2):
    g = b2.gen_rmat(10, 16, seed=1)
    assert g.n == 1024
    src = np.repeat(np.arange(g.n), np.diff(g.rowptr))
    assert np.all(src != g.colind)                                   # no self-loops
    for u in range(g.n):
        row = g.colind[g.rowptr[u]:g.rowptr[u + 1]]
        assert np.all(np.diff(row) > 0)                             # sorted, no duplicates
    t = g.transpose()
    assert np.array_equal(t.rowptr, g.rowptr) and np.array_equal(t.colind, g.colind)   # symmetric
    assert np.array_equal(t.weights, g.weights)                     # one weight per undirected pair
    assert g.weights.min() >= 1 and g.weights.max() <= 255


def test_grid_properties(b2):
    g = b2.gen_grid(30, 20, shortcut_frac=0.02, seed=4)
    lattice = 2 * (30 * 19 + 29 * 20)
    assert lattice <= g.m <= lattice + 2 * round(0.02 * lattice)
    assert g.weights.min() >= 1
    assert np.all(g.fweights < 1.0) and np.all(g.fweights > 0.0)


def test_csrbin_roundtrip(tmp_path, b2):
    g = b2.gen_er(200, 900, 1, 50, 1).transpose()
    p = str(tmp_path / "g.csrbin")
    b2.csrbin_write(p, g)
    h = b2.csrbin_read(p)
    assert h.n == g.n and np.array_equal(h.rowptr, g.rowptr) and np.array_equal(h.colind, g.colind)
    assert np.array_equal(h.fweights, g.fweights)
    with open(p, "r+b") as f:
        f.write(b"XXXX")
    with pytest.raises(b2.B2Error):
        b2.csrbin_read(p)


def test_csrbin_matches_reference_converter(tmp_path, b2):
    """Byte-for-byte against the reference's gr_to_csr (compiled from its own
    source into oracle/_ref by oracle/Makefile)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "gr_to_csr")
    if not os.path.exists(exe):
        pytest.skip("reference converter not built (needs the reference checkout)")
    g = b2.gen_er(120, 700, 1, 30, 5)
    gr = tmp_path / "g.gr"
    with open(gr, "w") as f:
        f.write(f"c synthetic\np sp {g.n} {g.m}\n")
        for u in range(g.n):
            for e in range(g.rowptr[u], g.rowptr[u + 1]):
                f.write(f"a {u + 1} {int(g.colind[e]) + 1} {int(g.weights[e])}\n")
    out_ref = tmp_path / "ref.csrbin"
    subprocess.run([exe, str(gr), str(out_ref)], check=True, capture_output=True)
    gi = g.transpose()
    gi.fweights = gi.weights.astype(np.float32)
    ours = tmp_path / "ours.csrbin"
    b2.csrbin_write(str(ours), gi)
    assert open(out_ref, "rb").read() == open(ours, "rb").read()


def test_python_mirror_fails_loudly_without_library(monkeypatch):
    import b200sssp._lib as L
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", "/nonexistent/libb200sssp.so")
    with pytest.raises(L.LibraryMissing):
        L.lib()
