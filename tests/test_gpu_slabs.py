"""One 2-D dendrite domain split into y-slabs, each slab an engine context, driven
through dba_b200.slabs' exchange protocol (dba_rows_pack / dba_rows_unpack /
dba_flag_rows on device buffers).  The ranks are emulated in one process on one
GPU with LocalComm (run one after another, buffers handed between the contexts'
streams after a synchronisation); the gathered slabs must equal the single-domain
engine run bit for bit: p, T and the next step's wake flags."""
import numpy as np
import pytest

import dba_b200
from dba_b200 import slabs
from cases import DENDRITE_REF, dendrite_cfg

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
