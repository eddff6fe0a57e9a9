"""The tile queue of the FP32 3-D dendrite and the KH tile kernels.

A scan kernel lists each step's tiles, the tile kernel's CTAs take them through
an atomic counter, and the last CTA to finish zeroes the counters for the next
step.  With wake-up thresholds no cell can pass, every DBA step after the first
lists nothing (every CTA finds the queue empty at once); the queue must still be
ready afterwards: regular steps (every tile listed) and DBA steps that follow
give the same bits as the one-block (dendrite) and stage (KH) kernels.
"""
import numpy as np
import pytest

import dba_b200
from cases import DENDRITE_REF, KH_REF, dendrite_cfg, kh_cfg

pytestmark = pytest.mark.gpu


def _same(a, b, fields):
    for f in fields:
        u = a.field(f)
        assert np.all(np.isfinite(u)), f
        assert np.array_equal(u, b.field(f)), f
    assert np.array_equal(a.flags(0), b.flags(0))


def _run(t, k, fields):
    for n, mode in ((1, 1), (1, 1), (7, 1), (48, 1)):
        c0 = t.cell_updates()
        t.step(n, mode)
        k.step(n, mode)
        _same(t, k, fields)
    assert t.cell_updates() == c0                 # the last DBA steps listed no tile
    for n, mode in ((5, 0), (1, 1), (6, 1), (3, 0)):
        t.step(n, mode)
        k.step(n, mode)
        _same(t, k, fields)
    t.sync()
    k.sync()


def test_dendrite3_queue_empty_steps_then_regular():
    # metric_p 0.6: metric_p <= p <= 1 - metric_p is empty; |dT| >= 1e30 never holds
    prm = dict(DENDRITE_REF, Delta=1.15, delta=0.2, metric_p=0.6, metric_T=1e30)
    t, k = (dba_b200.Simulation(dendrite_cfg(prm, 64, 32, 40, 8, precision=1, bc=1, tiles=tl, ic=1, ic_radius=6.0,
                                             ic_width=2.0, ic_corner=1)).init() for tl in (1, 0))
    assert t.info.grid_ctas > 1
    _run(t, k, ("p", "T"))


@pytest.mark.parametrize("B", [8, 16])
def test_kh_queue_empty_steps_then_regular(B):
    nx, ny = 96, 256
    prm = dict(KH_REF, metric_eps=1e30)
    rng = np.random.default_rng(3)
    Y, X = np.mgrid[0:ny, 0:nx]
    band = np.abs((Y + 0.5) / ny - 0.5) < 0.25
    ic = [np.where(band, 2.0, 1.0), np.full((ny, nx), 2.5), np.where(band, 0.5, -0.5),
          0.01 * np.sin(4 * np.pi * (X + 0.5) / nx) + 1e-4 * rng.standard_normal((ny, nx))]
    t, k = (dba_b200.Simulation(kh_cfg(prm, nx, ny, B, precision=1, conserved=0, tiles=tl)).init([a[None] for a in ic])
            for tl in (1, 0))
    _run(t, k, ("Mass", "Momx", "Momy", "Energy"))
