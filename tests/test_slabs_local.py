"""Model B y-slabs driven in one process (LocalComm, ranks stepped one after another,
ModelBSlabRun.step_all) with the CPU restatement as each slab's stepper: the gathered
slabs equal the single-domain restatement bit for bit every 10 steps, for 2 and 3
ranks, across DBA and regular steps."""
import numpy as np
import pytest

from dba_b200 import slabs
from oracle_lib import OracleModelB
from test_slabs_gloo import MB_B, MB_NX, MB_NY, MB_PRM, OracleModelBStepper, _mb_ic


@pytest.mark.parametrize("world", [2, 3])
def test_modelb_local_slabs_equal_single_domain(world):
    L = slabs.SlabLayout(MB_NX, MB_NY, MB_B, world)
    comm = slabs.LocalComm(world)
    ic = _mb_ic()
    runs, oracles = {0: [], 1: []}, []
    for r in range(world):
        lx, ly, lz = slabs.local_initial_fields([f.ravel() for f in ic], L, r)
        o = OracleModelB(MB_NX, L.local_ny, 1, MB_B, MB_PRM)
        o.set_fields(lx, ly, lz)
        st = OracleModelBStepper(o, L)
        for mode in (0, 1):
            runs[mode].append(slabs.ModelBSlabRun(st, L, r, comm, mode=mode))
        runs[1][-1].start()
        oracles.append(o)
    single = OracleModelB(MB_NX, MB_NY, 1, MB_B, MB_PRM)
    single.set_fields(*ic)
    nbx = MB_NX // MB_B
    act = []
    for k, mode in enumerate((1, 1, 0, 1, 1)):
        slabs.ModelBSlabRun.step_all(runs[mode], 10)
        single.step(10, mode)
        for n in ("x", "y", "z"):
            got = np.concatenate([slabs.owned(o.field(n), L) for o in oracles])
            assert np.array_equal(got, single.field(n)[0]), (n, k)
        got = np.concatenate([o.flags()[0].reshape(-1, nbx)[1:1 + L.nbr] for o in oracles])
        w = single.flags()[0].reshape(-1, nbx)
        assert np.array_equal(got, w), ("wake", k)
        act.append(w.mean())
    assert 0.0 < min(act) < 0.8
