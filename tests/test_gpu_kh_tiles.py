"""KH one-kernel tile step against the four stage kernels and the CPU restatement.

Both GPU paths evaluate every KH formula through the same explicitly rounded
helpers, so with the same DBA flags they must give the same bits: conserved
fields, the primitives read back the reference's way, and the wake-up flags.
The initial state is the sharp-band shear layer (flat bands, a small sinusoidal
vy and white noise), so only blocks near the two interfaces are active: the
persisted (stale) primitives, gradients, half-step states and fluxes of
inactive neighbours are read across block and tile edges, and blocks wake up
and fall asleep as the layer develops.  In FP64 the tile path is also compared
with the CPU restatement step by step.
"""
import numpy as np
import pytest

import dba_b200
from cases import KH_REF, kh_cfg
from oracle_lib import OracleKH

pytestmark = pytest.mark.gpu

FIELDS = ("Mass", "Momx", "Momy", "Energy", "rho", "p", "vx", "vy")
NX, NY = 96, 256


def sharp_bands(nx, ny, seed=3):
    rng = np.random.default_rng(seed)
    Y, X = np.mgrid[0:ny, 0:nx]
    band = np.abs((Y + 0.5) / ny - 0.5) < 0.25
    rho = np.where(band, 2.0, 1.0)
    vx = np.where(band, 0.5, -0.5)
    p = np.full_like(rho, 2.5)
    vy = 0.01 * np.sin(4 * np.pi * (X + 0.5) / nx) + 1e-4 * rng.standard_normal((ny, nx))
    return rho, p, vx, vy


def _sim(prec, B, conserved, tiles):
    prm = dict(KH_REF, metric_eps=20.0)
    s = dba_b200.Simulation(kh_cfg(prm, NX, NY, B, precision=prec, conserved=conserved, tiles=tiles))
    return s.init([a[None] for a in sharp_bands(NX, NY)])


def _same(a, b):
    for f in FIELDS:
        u = a.field(f)
        assert np.all(np.isfinite(u)), f
        assert np.array_equal(u, b.field(f)), f
    assert np.array_equal(a.flags(0), b.flags(0))


@pytest.mark.parametrize("prec", [1, 0])
@pytest.mark.parametrize("B", [8, 16])
@pytest.mark.parametrize("conserved", [0, 1])
def test_kh_tiles_bitexact_vs_stage_kernels(prec, B, conserved):
    t, k = _sim(prec, B, conserved, 1), _sim(prec, B, conserved, 0)
    act = []
    for n in (1, 1, 1, 5, 20, 48, 48):
        t.step(n, 1)
        k.step(n, 1)
        _same(t, k)
        act.append(float(np.mean(t.flags(0))))
    assert 0.0 < min(act) < 0.8               # partial activity was exercised
    t.sync()
    k.sync()


@pytest.mark.parametrize("prec", [1, 0])
@pytest.mark.parametrize("B", [8, 16])
def test_kh_tiles_many_tiles_per_cta(prec, B):
    """A 1024x512 grid has 2048 tiles, several per CTA, so each CTA stages the next
    listed tile's inputs while it computes the current one; the results must still
    equal the stage kernels' bit for bit."""
    nx, ny = 1024, 512

    def sim(tiles):
        prm = dict(KH_REF, metric_eps=20.0)
        s = dba_b200.Simulation(kh_cfg(prm, nx, ny, B, precision=prec, conserved=0, tiles=tiles))
        return s.init([a[None] for a in sharp_bands(nx, ny, seed=5)])

    t, k = sim(1), sim(0)
    act = []
    for n in (1, 2, 7, 30, 60):
        t.step(n, 1)
        k.step(n, 1)
        _same(t, k)
        act.append(float(np.mean(t.flags(0))))
    assert 0.0 < min(act) < 0.8
    t.step(10, 0)
    k.step(10, 0)
    _same(t, k)


@pytest.mark.parametrize("prec", [1, 0])
def test_kh_tiles_regular_then_dba(prec):
    t, k = _sim(prec, 8, 0, 1), _sim(prec, 8, 0, 0)
    for n, mode in ((10, 0), (30, 1), (10, 0), (20, 1)):
        t.step(n, mode)
        k.step(n, mode)
        _same(t, k)


@pytest.mark.parametrize("B,conserved", [(8, 0), (8, 1), (16, 0)])
def test_kh_tiles_fp64_bitexact_vs_oracle(B, conserved):
    prm = dict(KH_REF, metric_eps=20.0)
    o = OracleKH(NX, NY, B, prm, conserved=conserved)
    o.set_primitive(*[a.ravel() for a in sharp_bands(NX, NY)])
    s = _sim(0, B, conserved, 1)
    for t in range(1, 41):
        o.step(1, 1)
        s.step(1, 1)
        if t % 5 == 0:
            for f in ("Mass", "Momx", "Momy", "Energy"):
                assert np.array_equal(s.field(f), o.field(f)), (f, t)
            w, nxt = o.flags()
            assert np.array_equal(s.flags(0).ravel() != 0, np.asarray(w).ravel() != 0), t
            assert np.array_equal(s.flags(1).ravel() != 0, np.asarray(nxt).ravel() != 0), t
