"""Non-finite detection of the FP32 tile kernels: a NaN planted in an active block's
initial fields reaches the stored values, and dba_sync reports DBA_ERR_NONFINITE
(status 5) through the host-visible status word.  The kernels fold the check into
one fused multiply-add per stored value (x * 0 is 0 only for finite x)."""
import numpy as np
import pytest

import dba_b200
from cases import DENDRITE_REF, KH_REF, MODELB_REF, dendrite_cfg, kh_cfg, modelb_cfg

pytestmark = pytest.mark.gpu


def _expect_nonfinite(sim, steps=2):
    sim.step(steps, 1)
    with pytest.raises(dba_b200.DBAError) as e:
        sim.sync()
    assert e.value.code == 5


def test_dendrite3_tiles_nonfinite():
    cfg = dendrite_cfg(DENDRITE_REF, 64, 32, 32, 8, precision=1, tiles=1)
    s = dba_b200.Simulation(cfg).init()
    p, T = s.field("p"), s.field("T")
    T[16, 16, 20] = np.nan
    _expect_nonfinite(dba_b200.Simulation(cfg).init([p, T]))


@pytest.mark.parametrize("B", [8, 16])
def test_kh_tiles_nonfinite(B):
    nx, ny = 64, 64
    Y = np.mgrid[0:ny, 0:nx][0]
    band = np.abs((Y + 0.5) / ny - 0.5) < 0.25
    rho = np.where(band, 2.0, 1.0)
    rho[ny // 4, 10] = np.nan                      # on the interface: an active block
    ic = [rho, np.full((ny, nx), 2.5), np.where(band, 0.5, -0.5), np.full((ny, nx), 0.01)]
    cfg = kh_cfg(dict(KH_REF, metric_eps=0.0), nx, ny, B, precision=1, tiles=1)
    _expect_nonfinite(dba_b200.Simulation(cfg).init([a[None] for a in ic]))


def test_modelb_tiles_nonfinite():
    cfg = modelb_cfg(dict(MODELB_REF, metric_eps=1e-3), 64, 64, 1, 16, precision=1, tiles=1)
    x = np.full((1, 64, 64), 0.2)
    x[0, 20, 20] = np.nan
    _expect_nonfinite(dba_b200.Simulation(cfg).init([x, np.full_like(x, 0.2), np.full_like(x, 0.01)]))
