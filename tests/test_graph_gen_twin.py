"""CPU: the oracle's generator twins (oracle/oracle_gen.c) give the same bytes
as the library's b2_gen_rmat / b2_gen_grid.  The reference arm of bench.py
builds its RMAT-24 and 4096^2 grid inputs with the twins, so it never loads
libb200sssp.so; this pins that its graphs are the GPU arm's graphs."""
import numpy as np
import pytest


def _same(hg, tw):
    rp, ci, w, fw = tw
    assert np.array_equal(hg.rowptr, rp)
    assert np.array_equal(hg.colind, ci)
    assert np.array_equal(hg.weights, w)
    assert np.array_equal(hg.fweights.view(np.uint32), fw.view(np.uint32))


@pytest.mark.parametrize("scale,ef,seed,threads", [(10, 16, 1, 1), (14, 16, 1, 4), (16, 8, 7, 3), (12, 4, 0, 2)])
def test_rmat_twin_matches_library(b2, orc, scale, ef, seed, threads):
    hg = b2.gen_rmat(scale, ef, 0.57, 0.19, 0.19, 1, 255, seed)
    _same(hg, orc.gen_rmat(scale, ef, 0.57, 0.19, 0.19, 1, 255, seed, threads=threads))


def test_rmat_twin_other_quadrants_and_weights(b2, orc):
    hg = b2.gen_rmat(13, 12, 0.45, 0.25, 0.2, 5, 1000, 99)
    _same(hg, orc.gen_rmat(13, 12, 0.45, 0.25, 0.2, 5, 1000, 99, threads=5))


@pytest.mark.parametrize("rows,cols,frac,seed", [(64, 64, 0.02, 1), (100, 37, 0.05, 3), (256, 256, 0.02, 1),
                                                 (1, 50, 0.0, 2)])
def test_grid_twin_matches_library(b2, orc, rows, cols, frac, seed):
    hg = b2.gen_grid(rows, cols, frac, 5.0, 1.0, seed)
    _same(hg, orc.gen_grid(rows, cols, frac, 5.0, 1.0, seed, threads=4))


def test_grid_twin_lognormal_parameters(b2, orc):
    hg = b2.gen_grid(128, 96, 0.1, 3.0, 2.0, 11)
    _same(hg, orc.gen_grid(128, 96, 0.1, 3.0, 2.0, 11, threads=3))
