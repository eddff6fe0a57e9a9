"""One 2-D domain split into y-slabs, each slab an engine context, driven through
dba_b200.slabs' exchange protocol (dba_rows_pack / dba_rows_unpack / dba_flag_rows,
and for Model B dba_slab_rows / dba_lazy_change, on device buffers).  The ranks are
emulated in one process on one GPU with LocalComm (run one after another, buffers
handed between the contexts' streams after a synchronisation); the gathered slabs
must equal the single-domain engine run bit for bit: the fields and the next step's
wake flags."""
import numpy as np
import pytest

import dba_b200
from dba_b200 import slabs
from cases import DENDRITE_REF, MODELB_REF, dendrite_cfg, modelb_cfg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world,B,prec", [(2, 4, 0), (4, 8, 0), (2, 8, 1), (1, 8, 0)])
def test_engine_slabs_equal_single_domain(world, B, prec):
    nx = ny = 128
    cfg = dendrite_cfg(DENDRITE_REF, nx, ny, 1, B, precision=prec)
    single = dba_b200.Simulation(cfg).init()
    g = [single.field("p").ravel(), single.field("T").ravel()]
    L = slabs.SlabLayout(nx, ny, B, world)
    comm = slabs.LocalComm(world)
    runs, sims = [], []
    for r in range(world):
        s = dba_b200.Simulation(L.local_config(cfg)).init(slabs.local_initial_fields(g, L, r))
        run = slabs.SlabRun(slabs.EngineStepper(s, L), L, r, comm)
        run.start()
        runs.append(run)
        sims.append(s)
    nbx = nx // B
    for chunk in (1, 5, 20, 40, 60):
        slabs.SlabRun.step_all(runs, chunk)
        single.step(chunk, 1)
        for f in ("p", "T"):
            got = np.concatenate([slabs.owned(s.field(f), L) for s in sims])
            assert np.array_equal(got, single.field(f)[0]), (f, chunk)
        for which in (0, 2):
            got = np.concatenate([s.flags(which).reshape(-1, nbx)[1:1 + L.nbr] for s in sims])
            assert np.array_equal(got, single.flags(which).reshape(-1, nbx)), (which, chunk)
    assert single.flags(0).sum() > 0
    for s in sims:
        s.sync()


def _mb_ic(nx, ny, seed=9):
    """Noisy discs on a flat background across the slab boundaries of two and four
    ranks and across the periodic wrap."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:ny, 0:nx]
    inside = np.zeros((ny, nx), bool)
    for cx, cy, r in ((30, ny // 2, 12), (90, ny // 4, 10), (60, 3 * ny // 4 - 1, 9), (100, 2, 9)):
        dx = np.minimum(np.abs(xx - cx), nx - np.abs(xx - cx))
        dy = np.minimum(np.abs(yy - cy), ny - np.abs(yy - cy))
        inside |= dx * dx + dy * dy <= r * r
    x = np.where(inside, 0.2 + 0.05 * (rng.random((ny, nx)) - 0.5), 0.2)
    y = np.where(inside, 0.2 + 0.05 * (rng.random((ny, nx)) - 0.5), 0.2)
    z = np.where(inside, 0.1 + 0.001 * (rng.random((ny, nx)) - 0.5), 0.1)
    return x, y, z


@pytest.mark.parametrize("world,B,prec,cons,tiles", [
    (2, 8, 0, 0, 0),      # FP64, one-block kernel
    (4, 16, 1, 0, 1),     # FP32 tile kernel
    (2, 16, 1, 1, 1),     # FP32 tile kernel, conserved (fixed-point totals summed over the ranks)
    (4, 8, 1, 1, 1),      # FP32 conserved; slabs of 48 rows run the one-block FP32 kernel
    (1, 16, 1, 1, 1),
])
def test_engine_modelb_slabs_equal_single_domain(world, B, prec, cons, tiles):
    nx = ny = 128
    prm = dict(MODELB_REF, metric_eps=3e-4, k_0=0.3)
    ic = _mb_ic(nx, ny)
    cfg = modelb_cfg(prm, nx, ny, 1, B, precision=prec, conserved=cons, tiles=tiles)
    single = dba_b200.Simulation(cfg).init([a[None] for a in ic])
    L = slabs.SlabLayout(nx, ny, B, world)
    comm = slabs.LocalComm(world)
    runs, sims = {0: [], 1: []}, []
    for r in range(world):
        local = slabs.local_initial_fields([a.ravel() for a in ic], L, r)
        s = dba_b200.Simulation(L.local_config(cfg)).init([a.reshape(1, L.local_ny, nx) for a in local])
        st = slabs.EngineStepper(s, L)
        for mode in (0, 1):
            runs[mode].append(slabs.ModelBSlabRun(st, L, r, comm, mode=mode))
        runs[1][-1].start()
        sims.append(s)
    nbx = nx // B
    act = []
    for chunk, mode in ((1, 1), (5, 1), (14, 1), (10, 0), (20, 1), (50, 1)):
        slabs.ModelBSlabRun.step_all(runs[mode], chunk)
        single.step(chunk, mode)
        for f in ("x", "y", "z"):
            got = np.concatenate([slabs.owned(s.field(f), L) for s in sims])
            assert np.array_equal(got, single.field(f)[0]), (f, chunk, mode)
        got = np.concatenate([s.flags(0).reshape(-1, nbx)[1:1 + L.nbr] for s in sims])
        assert np.array_equal(got, single.flags(0).reshape(-1, nbx)), ("flags", chunk, mode)
        act.append(float(np.mean(single.flags(0))))
    assert 0.0 < min(act) < 0.8               # blocks asleep, and awake, at rank edges
    for s in sims:
        s.sync()                                # raises on a device error status
