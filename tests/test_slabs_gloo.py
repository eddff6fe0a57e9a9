"""One 2-D dendrite domain split into y-slabs across two gloo ranks (CPU), each rank
stepping its slab with the CPU restatement through dba_b200.slabs' exchange protocol
(halo block rows, ghost blocks kept inactive, wake-ups scattered into ghost rows
returned to their owners).  Every 10 steps the gathered slabs must equal the
single-domain restatement bit for bit: p, T and the next step's wake flags."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cases import DENDRITE_REF
from oracle_lib import OracleDendrite

NX, NY, B, STEPS = 64, 64, 4, 120


class OracleStepper:
    """The slab protocol's stepper interface on the CPU restatement (host arrays as CPU tensors)."""

    def __init__(self, o, layout):
        self.o, self.L = o, layout
        self.rows = lambda: torch.empty(2 * layout.B * layout.nx, dtype=torch.float64)
        self.flags = lambda: torch.empty(2 * (layout.nx // layout.B), dtype=torch.uint8)

    def _fields(self):
        d = self.o.get()
        return d["p"].reshape(self.L.local_ny, self.L.nx), d["T"].reshape(self.L.local_ny, self.L.nx), d

    def pack_rows(self, row0):
        p, T, _ = self._fields()
        return torch.from_numpy(np.concatenate([p[row0:row0 + self.L.B].ravel(), T[row0:row0 + self.L.B].ravel()]))

    def unpack_rows(self, row0, t):
        p, T, _ = self._fields()
        a = t.numpy()
        n = self.L.B * self.L.nx
        p[row0:row0 + self.L.B] = a[:n].reshape(self.L.B, self.L.nx)
        T[row0:row0 + self.L.B] = a[n:].reshape(self.L.B, self.L.nx)
        self.o.set_fields(p, T)

    def _flag_rows(self, d, brow):
        nbx = self.L.nx // self.L.B
        return d["wake_p"].reshape(-1, nbx), d["wake_T"].reshape(-1, nbx)

    def get_flags(self, brow):
        _, _, d = self._fields()
        wp, wT = self._flag_rows(d, brow)
        return torch.from_numpy(np.concatenate([wp[brow], wT[brow]]).astype(np.uint8))

    def or_flags(self, brow, t):
        _, _, d = self._fields()
        wp, wT = self._flag_rows(d, brow)
        a = t.numpy().astype(np.int32)
        nbx = self.L.nx // self.L.B
        wp[brow] |= a[:nbx]
        wT[brow] |= a[nbx:]
        self.o.set_flags(wp.ravel(), wT.ravel())

    def clear_flags(self, brow):
        _, _, d = self._fields()
        wp, wT = self._flag_rows(d, brow)
        wp[brow] = 0
        wT[brow] = 0
        self.o.set_flags(wp.ravel(), wT.ravel())

    def step(self, n=1, mode=1):
        self.o.step(n, mode)

    def ordered(self):
        import contextlib
        return contextlib.nullcontext()

    def barrier(self):
        pass


def _global():
    o = OracleDendrite(NX, NY, 1, B, DENDRITE_REF)
    o.init_cone()
    return o


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from dba_b200 import slabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        L = slabs.SlabLayout(NX, NY, B, world)
        g = _global().get()
        lp, lT = slabs.local_initial_fields([g["p"].ravel(), g["T"].ravel()], L, rank)
        o = OracleDendrite(NX, L.local_ny, 1, B, DENDRITE_REF)
        o.set_fields(lp, lT)
        run = slabs.SlabRun(OracleStepper(o, L), L, rank, slabs.DistComm(rank, world))
        run.start()
        snaps = []
        for _ in range(STEPS // 10):
            run.step(10)
            d = o.get()
            nbx = NX // B
            snaps.append((slabs.owned(d["p"], L).copy(), slabs.owned(d["T"], L).copy(),
                          d["wake_p"].reshape(-1, nbx)[1:1 + L.nbr].copy(), d["wake_T"].reshape(-1, nbx)[1:1 + L.nbr].copy()))
        out[rank] = snaps
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 4])
def test_slab_run_equals_single_domain(world):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    o = _global()
    nbx = NX // B
    for k in range(STEPS // 10):
        o.step(10, 1)
        d = o.get()
        p = np.concatenate([res[r][k][0] for r in range(world)])
        T = np.concatenate([res[r][k][1] for r in range(world)])
        wp = np.concatenate([res[r][k][2] for r in range(world)])
        wT = np.concatenate([res[r][k][3] for r in range(world)])
        assert np.array_equal(p, d["p"][0]), ("p", k)
        assert np.array_equal(T, d["T"][0]), ("T", k)
        assert np.array_equal(wp, d["wake_p"].reshape(-1, nbx)), ("wake_p", k)
        assert np.array_equal(wT, d["wake_T"].reshape(-1, nbx)), ("wake_T", k)
    assert d["wake_p"].sum() > 0
