"""KH with a CFL time step chosen on the device (cfl > 0, tile kernel).

Each step's dt must be cfl * min(dx, dy) / max over cells of (sound speed +
flow speed) of the state the previous step left, the device clock must be the
sum of the steps taken, and the run must stay finite through the growth of the
shear-layer instability.
"""
import numpy as np
import pytest

import dba_b200
from cases import KH_REF, kh_cfg
from test_gpu_kh_tiles import sharp_bands

pytestmark = pytest.mark.gpu


def _max_speed(s, gamma):
    M, X, Y, E = (s.field(f)[0] for f in ("Mass", "Momx", "Momy", "Energy"))
    vol = s.cfg.dx * s.cfg.dy
    rho = M / vol
    u = X / rho / vol
    v = Y / rho / vol
    p = (E / vol - 0.5 * rho * (u * u + v * v)) * (gamma - 1.0)
    return float(np.max(np.sqrt(gamma * p / rho) + np.sqrt(u * u + v * v)))


@pytest.mark.parametrize("prec,B,mode", [(1, 16, 1), (1, 8, 1), (0, 16, 1), (1, 16, 0)])
def test_kh_cfl_step_follows_the_state(prec, B, mode):
    nx, ny, gamma, cfl = 96, 256, 1.4, 0.4
    prm = dict(KH_REF, metric_eps=20.0, dx=1.0 / 96, dy=1.0 / 96, gamma=gamma)
    cfg = kh_cfg(prm, nx, ny, B, precision=prec, cfl=cfl)
    s = dba_b200.Simulation(cfg).init([a[None] for a in sharp_bands(nx, ny)])
    h = 1.0 / 96
    clock = 0.0
    # the device keeps speeds as float (FP64: rounded once; FP32: approximate divide/sqrt too)
    tol = 1e-5 if prec else 2e-7
    for k in range(30):
        o = s.observables()
        expect = cfl * h / _max_speed(s, gamma)
        assert abs(o["dt"] - expect) <= tol * expect, (k, o["dt"], expect)
        assert abs(o["time"] - clock) <= 1e-12 * max(clock, 1e-30)
        clock += o["dt"]
        s.step(1, mode)
    s.step(400, mode)
    for f in s.fields:
        assert np.all(np.isfinite(s.field(f))), f
    s.sync()


def test_kh_cfl_needs_the_tile_kernel():
    prm = dict(KH_REF, metric_eps=20.0)
    with pytest.raises(dba_b200.DBAError):
        dba_b200.Simulation(kh_cfg(prm, 64, 64, 4, precision=1, cfl=0.4))     # block 4: stage kernels
    with pytest.raises(dba_b200.DBAError):
        dba_b200.Simulation(kh_cfg(prm, 64, 64, 16, precision=1, cfl=0.4, tiles=0))
