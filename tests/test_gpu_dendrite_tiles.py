"""FP32 3-D dendrite: the 32x8x8-cell tile kernel against the one-block kernel.

Both evaluate every cell through den_p_new / den_T_new (explicitly rounded), so
with the same DBA flags they must give the same bits for p, T and both
channels' flags -- with partial activity (p- and T-activity differ per block),
across periodic and zero-flux walls (the tile kernel clamps wall pieces cell by
cell), and in regular mode.
"""
import numpy as np
import pytest

import dba_b200
from cases import DENDRITE_REF, dendrite_cfg

pytestmark = pytest.mark.gpu


def _pair(bc, corner, shape=(96, 32, 40)):
    prm = dict(DENDRITE_REF, Delta=1.15, delta=0.2, metric_p=1e-3, metric_T=1e-5)
    sims = []
    for t in (1, 0):
        cfg = dendrite_cfg(prm, *shape, 8, precision=1, bc=bc, tiles=t, ic=1, ic_radius=6.0, ic_width=2.0,
                           ic_corner=corner)
        sims.append(dba_b200.Simulation(cfg).init())
    return sims


def _same(a, b):
    for f in ("p", "T"):
        u = a.field(f)
        assert np.all(np.isfinite(u)), f
        assert np.array_equal(u, b.field(f)), f
    for w in (0, 1, 2, 3):
        assert np.array_equal(a.flags(w), b.flags(w)), w


@pytest.mark.parametrize("bc,corner", [(0, 0), (1, 0), (1, 1)])
def test_dendrite3_tiles_bitexact_vs_block_kernel(bc, corner):
    t, k = _pair(bc, corner)
    act = []
    for n in (1, 1, 1, 5, 20, 48, 96, 96):
        t.step(n, 1)
        k.step(n, 1)
        _same(t, k)
        act.append(float(np.mean(t.flags(0))))
    assert 0.0 < min(act) < 0.9
    t.sync()
    k.sync()


def test_dendrite3_tiles_regular_then_dba():
    t, k = _pair(1, 1)
    for n, mode in ((10, 0), (60, 1), (10, 0), (50, 1)):
        t.step(n, mode)
        k.step(n, mode)
        _same(t, k)


def test_dendrite3_tiles_many_tiles_per_cta():
    """256x128x128 has 2048 tiles, several per CTA, so each CTA stages the next listed
    tile while it computes the current one; the results must still equal the block
    kernel's bit for bit, in regular steps and in DBA steps around a large seed."""
    prm = dict(DENDRITE_REF, Delta=1.15, delta=0.2, metric_p=1e-3, metric_T=1e-5)
    t, k = (dba_b200.Simulation(dendrite_cfg(prm, 256, 128, 128, 8, precision=1, bc=0, tiles=tl, ic=1,
                                             ic_radius=40.0, ic_width=2.0, ic_corner=0)).init()
            for tl in (1, 0))
    assert t.info.grid_ctas < (256 // 32) * (128 // 8) * (128 // 8)
    t.step(4, 0)
    k.step(4, 0)
    _same(t, k)
    act = []
    for n in (1, 3, 12, 48):
        t.step(n, 1)
        k.step(n, 1)
        _same(t, k)
        act.append(float(np.mean(t.flags(0))))
    assert 0.0 < min(act) < 0.9
