"""FP32 2-D Model B: the 32x32-cell tile kernel (both staging forms: `tiles = 1`
16-byte cp.async pieces, `tiles = 2` bulk copies) against the one-block-at-a-time kernel.

Both kernels evaluate every point formula with the same explicitly rounded
operations, so with the same DBA flags they must produce bit-identical fields,
wake-up flags and conserved totals.  The initial condition is noisy only inside
a disc, so most blocks go inactive after the first step: listed tiles then hold
inactive blocks whose persisted (stale) potentials are read, blocks wake up and
fall asleep across tile edges, and the periodic wrap is crossed by the disc.
"""
import numpy as np
import pytest

import dba_b200
from cases import MODELB_REF, modelb_cfg

pytestmark = pytest.mark.gpu


def patch_ic(nx, ny, cx, cy, radius, seed=7):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:ny, 0:nx]
    dx = np.minimum(np.abs(xx - cx), nx - np.abs(xx - cx))
    dy = np.minimum(np.abs(yy - cy), ny - np.abs(yy - cy))
    inside = (dx * dx + dy * dy) <= radius * radius
    x = np.where(inside, 0.2 + 0.05 * (rng.random((ny, nx)) - 0.5), 0.2)
    y = np.where(inside, 0.2 + 0.05 * (rng.random((ny, nx)) - 0.5), 0.2)
    z = np.where(inside, 0.1 + 0.001 * (rng.random((ny, nx)) - 0.5), 0.1)
    return [a[None] for a in (x, y, z)]


def _pair(B, conserved, nx=128, ny=96, form=1):
    prm = dict(MODELB_REF, metric_eps=3e-4, k_0=0.3)
    ic = patch_ic(nx, ny, cx=8, cy=40, radius=22)
    sims = []
    for tiles in (form, 0):
        cfg = modelb_cfg(prm, nx, ny, 1, B, precision=1, conserved=conserved, tiles=tiles)
        sims.append(dba_b200.Simulation(cfg).init(ic))
    return sims


def _same(a, b):
    for f in ("x", "y", "z"):
        u = a.field(f)
        assert np.all(np.isfinite(u)), f
        assert np.array_equal(u, b.field(f)), f
    assert np.array_equal(a.flags(0), b.flags(0))


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("B", [8, 16])
@pytest.mark.parametrize("conserved", [0, 1])
def test_tiles_bitexact_vs_block_kernel_dba(B, conserved, form):
    t, k = _pair(B, conserved, form=form)
    assert t.info.grid_ctas <= (128 // 32) * (96 // 32)      # tile grid: at most one CTA per tile
    seen = set()
    for _ in range(12):          # single steps through the first wake-up transients
        t.step(1, 1)
        k.step(1, 1)
        _same(t, k)
        seen.add(float(np.mean(t.flags(0))))
    for _ in range(6):           # longer chunks (captured graphs)
        t.step(48, 1)
        k.step(48, 1)
        _same(t, k)
        seen.add(float(np.mean(t.flags(0))))
    assert min(seen) < 0.7       # partial activity was exercised
    t.sync()
    k.sync()


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("B", [8, 16])
def test_tiles_bitexact_vs_block_kernel_regular_then_dba(B, form):
    t, k = _pair(B, 1, form=form)
    t.step(30, 0)
    k.step(30, 0)
    _same(t, k)
    t.step(60, 1)
    k.step(60, 1)
    _same(t, k)


def test_tiles_conserved_mass_exact():
    """Lazy conserved DBA on tiles: species totals stay at their initial values."""
    t, _ = _pair(16, 1)
    m0 = [t.field(f).sum() for f in ("x", "y", "z")]
    t.step(500, 1)
    m1 = [t.field(f).sum() for f in ("x", "y", "z")]
    for a, b in zip(m0, m1):
        assert abs(b - a) / abs(a) <= 1e-10, (a, b)


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("B", [8, 16])
def test_tiles_many_tiles_per_cta(B, form):
    """2048x1024 has 2048 tiles, several per CTA, so each CTA stages the next listed
    tile while it computes the current one (and loads the neighbour table of the one
    after); the results must still equal the block kernel's bit for bit, in regular
    steps (every tile listed) and in DBA steps with a large noisy disc."""
    nx, ny = 2048, 1024
    prm = dict(MODELB_REF, metric_eps=3e-4, k_0=0.3)
    ic = patch_ic(nx, ny, cx=700, cy=500, radius=380, seed=11)
    t, k = (dba_b200.Simulation(modelb_cfg(prm, nx, ny, 1, B, precision=1, conserved=1, tiles=tl)).init(ic)
            for tl in (form, 0))
    assert t.info.grid_ctas < (nx // 32) * (ny // 32)
    t.step(5, 0)
    k.step(5, 0)
    _same(t, k)
    act = []
    for n in (1, 3, 12, 48):
        t.step(n, 1)
        k.step(n, 1)
        _same(t, k)
        act.append(float(np.mean(t.flags(0))))
    assert 0.0 < min(act) < 0.9
