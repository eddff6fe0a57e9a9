"""Dendrite workloads at reduced size: DBA against the all-blocks regular mode.

The 2-D centre seed (undercooling 0.55 mapped as Delta = 1.15, anisotropy
eps4 = 0.05 as delta = 0.2, tanh seed radius 10, zero-flux walls) and the 3-D
corner seed (same parameters, octant symmetry) are advanced in DBA and in
regular mode from the same initial state.  DBA freezes blocks whose wake-up
tests are negative, so it is an approximation of the regular run: the tip
velocity must agree within 1 % while DBA updates a fraction of the blocks.
"""
import numpy as np
import pytest

import dba_b200

pytestmark = pytest.mark.gpu


def _cfg(nx, ny, nz, prec, corner):
    c = dba_b200.config("dendrite", nx=nx, ny=ny, nz=nz, block=8, precision=prec, bc=1, ic=1)
    c.Delta, c.delta, c.metric_p, c.metric_T = 1.15, 0.2, 1e-3, 1e-5
    c.ic_radius, c.ic_width, c.ic_corner = 10.0, 2.0, corner
    return c


def _run(cfg, mode, checkpoints):
    s = dba_b200.Simulation(cfg).init()
    tips, act, done = [], [], 0
    c0 = s.cell_updates()
    for t in checkpoints:
        s.step(t - done, mode)
        done = t
        tips.append(s.tip())
        act.append(float(np.mean(s.flags(0))))
    frac = (s.cell_updates() - c0) / (done * s.info.nb * s.info.cells_per_block)
    s.close()
    return np.array(tips), act, frac


def test_c0_centre_seed_dba_vs_regular_fp64():
    cps = [1000, 1500, 2000]              # the tip reaches the 256^2 wall near step 2600
    cfg = _cfg(256, 256, 1, 0, 0)
    td, ad, fd = _run(cfg, 1, cps)
    tr, ar, fr = _run(cfg, 0, cps)
    assert np.all(np.isfinite(td)) and np.all(np.isfinite(tr))
    vd = (td[-1] - td[0]) / (cps[-1] - cps[0])
    vr = (tr[-1] - tr[0]) / (cps[-1] - cps[0])
    assert vr > 0.02                                   # the dendrite grows (cells per step)
    assert abs(vd - vr) <= 0.01 * vr
    assert fr == pytest.approx(1.0) and fd < 0.5       # DBA updates well under half of the cells


def test_c3_corner_seed_dba_vs_regular_fp32():
    cps = [1000, 1200, 1400, 1600]        # the corner tip grows from about step 900 and meets the wall later
    cfg = _cfg(128, 128, 128, 1, 1)
    td, ad, fd = _run(cfg, 1, cps)
    tr, ar, fr = _run(cfg, 0, cps)
    ok = np.isfinite(td) & np.isfinite(tr)
    assert ok.sum() >= 2, (td, tr)
    i0, i1 = np.flatnonzero(ok)[0], np.flatnonzero(ok)[-1]
    vd = (td[i1] - td[i0]) / (cps[i1] - cps[i0])
    vr = (tr[i1] - tr[i0]) / (cps[i1] - cps[i0])
    assert vr > 0
    assert abs(vd - vr) <= 0.01 * vr, (td, tr)
    assert fd < 0.5 and max(ad) < 1.0
