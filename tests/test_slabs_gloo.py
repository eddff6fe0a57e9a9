"""One 2-D domain split into y-slabs across gloo ranks (CPU), each rank stepping its
slab with the CPU restatement through dba_b200.slabs' exchange protocol.  Dendrite:
halo block rows, ghost blocks kept inactive, wake-ups scattered into ghost rows
returned to their owners.  Model B: ghost blocks carry their owner's flags and the
persisted potentials travel with the halo; ghosts are never updated.  Every 10
steps the gathered slabs must equal the single-domain restatement bit for bit:
the fields and the next step's wake flags."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cases import DENDRITE_REF, MODELB_REF
from oracle_lib import OracleDendrite, OracleModelB

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


# ---- Model B ------------------------------------------------------------------------

MB_NX, MB_NY, MB_B, MB_STEPS = 64, 96, 8, 60
MB_PRM = dict(MODELB_REF, metric_eps=3e-4, k_0=0.3)


def _mb_ic():
    """Noisy discs on a flat background, across the slab boundaries at y = 48 (two ranks)
    and y = 24 (four ranks) and across the periodic wrap, so blocks wake and sleep on
    both sides of rank edges."""
    rng = np.random.default_rng(5)
    yy, xx = np.mgrid[0:MB_NY, 0:MB_NX]
    inside = np.zeros((MB_NY, MB_NX), bool)
    for cx, cy, r in ((20, 47, 6), (44, 24, 5), (36, 1, 5)):
        dx = np.minimum(np.abs(xx - cx), MB_NX - np.abs(xx - cx))
        dy = np.minimum(np.abs(yy - cy), MB_NY - np.abs(yy - cy))
        inside |= dx * dx + dy * dy <= r * r
    x = np.where(inside, 0.2 + 0.05 * (rng.random((MB_NY, MB_NX)) - 0.5), 0.2)
    y = np.where(inside, 0.2 + 0.05 * (rng.random((MB_NY, MB_NX)) - 0.5), 0.2)
    z = np.where(inside, 0.1 + 0.001 * (rng.random((MB_NY, MB_NX)) - 0.5), 0.1)
    return x, y, z


class OracleModelBStepper:
    """Model B's slab interface on the CPU restatement: x, y, z and the potentials
    (the restatement keeps full potential arrays, the reference's stale reads)."""

    FIELDS = ("x", "y", "z", "mu_x", "mu_y", "mu_z")

    def __init__(self, o, layout):
        self.o, self.L = o, layout
        self.nbx = layout.nx // layout.B
        self.rows = lambda: torch.empty(len(self.FIELDS) * layout.B * layout.nx, dtype=torch.float64)
        self.flags = lambda: torch.empty(self.nbx, dtype=torch.uint8)

    def _f(self, name):
        return self.o.field(name).reshape(self.L.local_ny, self.L.nx)

    def pack_rows(self, row0):
        return torch.from_numpy(np.concatenate([self._f(n)[row0:row0 + self.L.B].ravel() for n in self.FIELDS]))

    def unpack_rows(self, row0, t):
        a = t.numpy()
        k = self.L.B * self.L.nx
        for q, n in enumerate(self.FIELDS):
            f = self._f(n)
            f[row0:row0 + self.L.B] = a[q * k:(q + 1) * k].reshape(self.L.B, self.L.nx)
            self.o.set_field(n, f)

    def _wake(self):
        return self.o.flags()[0].reshape(-1, self.nbx)

    def get_flags(self, brow):
        return torch.from_numpy(self._wake()[brow].astype(np.uint8))

    def or_flags(self, brow, t):
        w = self._wake()
        w[brow] |= t.numpy().astype(np.int32)
        self.o.set_flags(w.ravel())

    def set_flags(self, brow, t):
        w = self._wake()
        w[brow] = t.numpy().astype(np.int32)
        self.o.set_flags(w.ravel())

    def own_rows(self, first, count, domain_cells):
        self.o.set_owned(first, first + count)

    def conserved_totals(self):
        return False

    def step(self, n=1, mode=1):
        self.o.step(n, mode)

    def ordered(self):
        import contextlib
        return contextlib.nullcontext()

    def barrier(self):
        pass


def _mb_worker(rank, world, port, out):
    import torch.distributed as dist
    from dba_b200 import slabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        L = slabs.SlabLayout(MB_NX, MB_NY, MB_B, world)
        lx, ly, lz = slabs.local_initial_fields([f.ravel() for f in _mb_ic()], L, rank)
        o = OracleModelB(MB_NX, L.local_ny, 1, MB_B, MB_PRM)
        o.set_fields(lx, ly, lz)
        comm = slabs.DistComm(rank, world)
        runs = {m: slabs.ModelBSlabRun(OracleModelBStepper(o, L), L, rank, comm, mode=m) for m in (0, 1)}
        runs[1].start()
        snaps = []
        for k in range(MB_STEPS // 10):
            runs[0 if k == 2 else 1].step(10)     # steps 20-29 regular, the rest DBA
            w = o.flags()[0].reshape(-1, MB_NX // MB_B)
            snaps.append(tuple(slabs.owned(o.field(n), L).copy() for n in ("x", "y", "z")) +
                         (w[1:1 + L.nbr].copy(),))
        out[rank] = snaps
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_modelb_slab_run_equals_single_domain(world):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_mb_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    o = OracleModelB(MB_NX, MB_NY, 1, MB_B, MB_PRM)
    o.set_fields(*_mb_ic())
    seen = []
    for k in range(MB_STEPS // 10):
        o.step(10, 0 if k == 2 else 1)
        for q, n in enumerate(("x", "y", "z")):
            got = np.concatenate([res[r][k][q] for r in range(world)])
            assert np.array_equal(got, o.field(n)[0]), (n, k)
        w = o.flags()[0].reshape(-1, MB_NX // MB_B)
        assert np.array_equal(np.concatenate([res[r][k][3] for r in range(world)]), w), ("wake", k)
        seen.append(w.mean())
    assert 0.0 < min(seen) < 0.8                  # partial activity, blocks asleep at rank edges
