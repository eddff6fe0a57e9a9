"""One 2-D domain split into y-slabs across ranks (one GPU each): dendrite and Model B.

The reference's CUDA-MPI programs decompose the domain across ranks and exchange,
every step, the halo layers of the fields and the wake-up flags of the boundary
blocks (example_Dendritic_growth/CUDA-MPI/dendrite.cpp:387-397, 459-644;
example_Reactive_ModelB/CUDA-MPI/reaction.cpp:416-438, 529-552).  Here:

* the global grid (nx, ny), DBA block edge B, is split into `world` slabs of
  H = ny / world rows (H a multiple of B); rank r owns global rows [r H, (r+1) H);
* rank r's engine context holds nx x (H + 2B) cells: local block rows 0 and
  H/B + 1 are ghost block rows, copies of the neighbouring slabs' boundary block
  rows; local rows [B, B + H) are its own.  The rank ring closes the periodic
  wrap in y;
* ghost blocks are kept inactive (their next-step wake flags are cleared before
  every step), so the local step never updates them and never scatters from them.

Per step, on every rank:
  1. halo: the first and last owned block rows (current p and T, B rows each) go
     to the neighbours, which write them into both buffers of their ghost rows;
  2. the step (the single-domain engine's kernels on the local grid);
  3. flags: the wake-ups the step scattered into the ghost block rows go to the
     ranks owning those blocks, which OR them into their next-step flags; the
     ghost rows' flags are cleared.

The dendrite's update reads p and T one cell around each cell and keeps no
stale intermediates, so with the flags exchanged the slab run advances exactly
the cells, with exactly the arithmetic, of the single-domain run: it equals it
bit for bit (tests/test_slabs_gloo.py, two gloo ranks on CPU with the CPU
restatement as the stepper; tests/test_gpu_slabs.py, engine contexts).

Model B (ModelBSlabRun) reads, across a block edge, the chemical potentials of
the neighbouring block -- recomputed where that block is active this step, its
persisted values where it is not (the reference's stale reads) -- so its ghost
blocks carry their owner's flags instead of being kept inactive:
  1. halo: the first and last owned block rows go to the neighbours -- x, y, z, the
     persisted potentials and the next step's flags of those blocks -- which write
     them into their ghost rows (the flags set, not OR-ed);
  2. the step; the context knows which block rows are its own (dba_slab_rows) and
     never updates, tests or wakes from a ghost block, whose flag only says whether
     its potentials are recomputed (from the ghost copy of x, y, z: the rows an own
     cell reads lie within the ghost row) or read persisted;
  3. wake-ups scattered into the ghost rows go to their owners and are OR-ed in;
  4. FP32 conserved contexts: the step's fixed-point change totals are summed over
     the ranks (exact integer sums), so every rank applies the whole domain's
     conservation offset.
The slab run again advances the cells of the single-domain run with the same
arithmetic and equals it bit for bit.

Communication: DistComm uses torch.distributed point-to-point operations (NCCL
between GPUs, gloo on CPU) on the buffers the stepper hands out (CUDA tensors
on the context's stream for the engine); LocalComm exchanges between slabs held
by one process (ranks emulated on one device, run one after another).
"""
import numpy as np

from . import engine


class SlabLayout:
    def __init__(self, nx, ny, block, world):
        if ny % world or (ny // world) % block:
            raise ValueError("ny / world must be a multiple of the block edge")
        self.nx, self.ny, self.B, self.world = nx, ny, block, world
        self.H = ny // world
        self.local_ny = self.H + 2 * block
        self.nbr = self.H // block          # owned block rows

    def global_rows(self, rank):
        """Global rows of local rows 0 .. local_ny - 1 (ghosts wrap around the ring)."""
        return [(rank * self.H - self.B + k) % self.ny for k in range(self.local_ny)]

    def local_config(self, cfg):
        """A copy of the global config for one slab (periodic in y: the ghost rows stand
        between the slab and its wrap)."""
        c = engine.Config()
        for k, _ in engine.Config._fields_:
            setattr(c, k, getattr(cfg, k))
        c.ny = self.local_ny
        return c


class EngineStepper:
    """One rank's slab on the engine: buffers are CUDA tensors, ordered on the context's stream."""

    def __init__(self, sim, layout):
        import torch
        self.sim, self.L = sim, layout
        self.torch = torch
        self.stream = torch.cuda.ExternalStream(sim.stream)
        dt = torch.float64 if sim.cfg.precision == 0 else torch.float32
        modelb = sim.cfg.model == engine.MODELS["modelb"]
        nf, nch = (6, 1) if modelb else (2, 2)     # exchanged fields (dba_rows_pack), flag channels
        self.rows = lambda: torch.empty(nf * layout.B * layout.nx, dtype=dt, device="cuda")
        self.flags = lambda: torch.empty(nch * (layout.nx // layout.B), dtype=torch.uint8, device="cuda")
        self.totals = lambda: torch.empty(3, dtype=torch.int64, device="cuda")

    def pack_rows(self, row0):
        t = self.rows()
        self.sim.rows_pack(row0, self.L.B, t.data_ptr())
        return t

    def unpack_rows(self, row0, t):
        self.sim.rows_unpack(row0, self.L.B, t.data_ptr())

    def get_flags(self, brow):
        t = self.flags()
        self.sim.flag_rows(0, brow, 1, t.data_ptr())
        return t

    def or_flags(self, brow, t):
        self.sim.flag_rows(1, brow, 1, t.data_ptr())

    def clear_flags(self, brow):
        self.sim.flag_rows(2, brow, 1)

    def set_flags(self, brow, t):
        self.sim.flag_rows(3, brow, 1, t.data_ptr())

    def own_rows(self, first, count, domain_cells):
        self.sim.slab_rows(first, count, domain_cells)

    def conserved_totals(self):
        """An FP32 conserved context keeps fixed-point totals that the ranks must share."""
        return bool(self.sim.cfg.conserved) and self.sim.cfg.precision == 1

    def get_totals(self):
        t = self.totals()
        self.sim.lazy_change(0, t.data_ptr())
        return t

    def put_totals(self, t):
        self.sim.lazy_change(1, t.data_ptr())

    def step(self, n=1, mode=1):
        self.sim.step(n, mode)

    def ordered(self):
        """Torch work (allocations, point-to-point transfers) on the context's stream."""
        return self.torch.cuda.stream(self.stream)

    def barrier(self):
        """Wait for this slab's queued work (ranks emulated in one process hand buffers
        from one context's stream to another's)."""
        self.stream.synchronize()


class LocalComm:
    """Exchange between the slabs of one process: exchange(rank, send_down, send_up) is
    called for every rank in turn, then collect(rank) returns (from_down, from_up)."""

    def __init__(self, world):
        self.world = world
        self.box = {}

    def post(self, rank, send_down, send_up):
        self.box[rank] = (send_down, send_up)

    def collect(self, rank):
        down, up = (rank - 1) % self.world, (rank + 1) % self.world
        return self.box[down][1], self.box[up][0]

    def sum_posted(self):
        """The sum over the ranks of what each posted as its first item."""
        total = None
        for r in range(self.world):
            t = self.box[r][0]
            total = t.clone() if total is None else total + t
        return total


class DistComm:
    """torch.distributed point-to-point exchange with the ring neighbours (NCCL or gloo).
    Every rank posts its two sends in the order (down, up) and its two receives in the
    order (from up, from down), which pairs them correctly for any world size >= 2."""

    def __init__(self, rank, world, group=None):
        import torch.distributed as dist
        self.dist, self.rank, self.world, self.group = dist, rank, world, group

    def sendrecv(self, send_down, send_up, recv_from_down, recv_from_up):
        d = self.dist
        down, up = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        ops = [d.P2POp(d.isend, send_down, down, self.group), d.P2POp(d.isend, send_up, up, self.group),
               d.P2POp(d.irecv, recv_from_up, up, self.group), d.P2POp(d.irecv, recv_from_down, down, self.group)]
        for r in d.batch_isend_irecv(ops):
            r.wait()

    def sum(self, t):
        """In place: the sum over the ranks (exact for integer tensors)."""
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)


class SlabRun:
    """Drives one rank's slab (stepper) through the exchange protocol above.

    `step(n)` advances n DBA steps.  With DistComm every rank calls it; with LocalComm,
    `SlabRun.step_all(runs, n)` advances all slabs of the process together."""

    def __init__(self, stepper, layout, rank, comm, mode=1):
        self.s, self.L, self.rank, self.comm = stepper, layout, rank, comm
        self.mode = mode                            # 1 DBA steps, 0 regular steps
        self.top_ghost = layout.H + layout.B        # first local row of the upper ghost block row
        self.top_gbrow = layout.nbr + 1

    def start(self):
        """After the context's init: ghost blocks are inactive from the first step on."""
        self.s.clear_flags(0)
        self.s.clear_flags(self.top_gbrow)

    # ---- one phase each, split so that LocalComm can interleave the ranks
    def _halo_send(self):
        return self.s.pack_rows(self.L.B), self.s.pack_rows(self.L.H)          # first, last owned block rows

    def _halo_recv(self, from_down, from_up):
        self.s.unpack_rows(0, from_down)
        self.s.unpack_rows(self.top_ghost, from_up)

    def _flags_send(self):
        return self.s.get_flags(0), self.s.get_flags(self.top_gbrow)

    def _flags_recv(self, from_down, from_up):
        # the lower neighbour's upper ghost row holds wake-ups for my first owned block row
        self.s.or_flags(1, from_down)
        self.s.or_flags(self.L.nbr, from_up)
        self.s.clear_flags(0)
        self.s.clear_flags(self.top_gbrow)

    def step(self, n=1):
        c = self.comm
        with self.s.ordered():
            for _ in range(n):
                down, up = self._halo_send()
                fd, fu = self.s.rows(), self.s.rows()
                c.sendrecv(down, up, fd, fu)
                self._halo_recv(fd, fu)
                self.s.step(1, 1)
                down, up = self._flags_send()
                fd, fu = self.s.flags(), self.s.flags()
                c.sendrecv(down, up, fd, fu)
                self._flags_recv(fd, fu)

    @staticmethod
    def step_all(runs, n=1):
        comm = runs[0].comm

        def phase(send, recv):
            for r in runs:
                with r.s.ordered():
                    comm.post(r.rank, *send(r))
            for r in runs:
                r.s.barrier()
            for r in runs:
                with r.s.ordered():
                    recv(r, *comm.collect(r.rank))

        for _ in range(n):
            phase(lambda r: r._halo_send(), lambda r, a, b: r._halo_recv(a, b))
            for r in runs:
                with r.s.ordered():
                    r.s.step(1, 1)
            phase(lambda r: r._flags_send(), lambda r, a, b: r._flags_recv(a, b))
        for r in runs:
            r.s.barrier()


class ModelBSlabRun(SlabRun):
    """Model B's slab protocol (module docstring): ghost blocks carry their owner's flags,
    persisted potentials travel with the halo, conserved totals are summed over the ranks."""

    def start(self):
        L = self.L
        self.s.own_rows(1, L.nbr, L.nx * L.ny)

    def _halo_send(self):
        L = self.L
        return (self.s.pack_rows(L.B), self.s.pack_rows(L.H), self.s.get_flags(1), self.s.get_flags(L.nbr))

    def _halo_recv(self, from_down, from_up, flags_from_down, flags_from_up):
        self.s.unpack_rows(0, from_down)
        self.s.unpack_rows(self.top_ghost, from_up)
        self.s.set_flags(0, flags_from_down)
        self.s.set_flags(self.top_gbrow, flags_from_up)

    def _flags_recv(self, from_down, from_up):
        # wake-ups the neighbours' steps scattered into their ghost rows, for my boundary rows
        self.s.or_flags(1, from_down)
        self.s.or_flags(self.L.nbr, from_up)

    def step(self, n=1):
        c = self.comm
        with self.s.ordered():
            for _ in range(n):
                down, up, f_down, f_up = self._halo_send()
                rd, ru, fd, fu = self.s.rows(), self.s.rows(), self.s.flags(), self.s.flags()
                c.sendrecv(down, up, rd, ru)
                c.sendrecv(f_down, f_up, fd, fu)
                self._halo_recv(rd, ru, fd, fu)
                self.s.step(1, 1 if self.mode else 0)
                down, up = self._flags_send()
                fd, fu = self.s.flags(), self.s.flags()
                c.sendrecv(down, up, fd, fu)
                self._flags_recv(fd, fu)
                if self.s.conserved_totals():
                    t = self.s.get_totals()
                    c.sum(t)
                    self.s.put_totals(t)

    @staticmethod
    def step_all(runs, n=1):
        comm = runs[0].comm

        def phase(send, recv):
            for r in runs:
                with r.s.ordered():
                    comm.post(r.rank, *send(r))
            for r in runs:
                r.s.barrier()
            for r in runs:
                with r.s.ordered():
                    recv(r, *comm.collect(r.rank))

        def halo_send(r):
            d, u, fd, fu = r._halo_send()
            return (d, fd), (u, fu)

        def halo_recv(r, from_down, from_up):
            r._halo_recv(from_down[0], from_up[0], from_down[1], from_up[1])

        for _ in range(n):
            phase(halo_send, halo_recv)
            for r in runs:
                with r.s.ordered():
                    r.s.step(1, 1 if r.mode else 0)
            phase(lambda r: r._flags_send(), lambda r, a, b: r._flags_recv(a, b))
            if runs[0].s.conserved_totals():
                for r in runs:
                    with r.s.ordered():
                        comm.post(r.rank, r.s.get_totals(), None)
                for r in runs:
                    r.s.barrier()
                total = comm.sum_posted()
                for r in runs:
                    with r.s.ordered():
                        r.s.put_totals(total)
        for r in runs:
            r.s.barrier()


def local_initial_fields(global_fields, layout, rank):
    """The slab's initial fields (p, T) with its ghost rows, from the global ones (ny, nx)."""
    rows = layout.global_rows(rank)
    return [np.ascontiguousarray(f.reshape(layout.ny, layout.nx)[rows]) for f in global_fields]


def owned(local_field, layout):
    """The owned rows of a local field (local_ny, nx)."""
    return local_field.reshape(layout.local_ny, layout.nx)[layout.B:layout.B + layout.H]
