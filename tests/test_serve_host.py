"""Host logic of the sweep server (dba_b200/serve.py) on the CPU: admission in
arrival order while the batch has room, retirement on the tip target or the step
limit, latency bookkeeping and the summary's percentiles.  The batch is a fake
with the engine.Batch methods: a fixed cell capacity and tips that grow by a
per-request rate each step, so every decision of the loop is known in advance."""
import numpy as np
import pytest

from dba_b200 import serve


class FakeBatch:
    def __init__(self, cell_capacity, max_slots=8, rate_of=None):
        self.capacity, self.max_slots = cell_capacity, max_slots
        self.used = 0
        self.slots = {}            # slot -> [cells, tip, steps, rate]
        self.rate_of = rate_of or (lambda cfg: 1.0)
        self.admitted, self.max_running, self.closed = [], 0, False

    def add(self, cfg, ic=None):
        cells = cfg.nx * cfg.ny
        free = [s for s in range(self.max_slots) if s not in self.slots]
        if not free or self.used + cells > self.capacity:
            return None
        s = free[0]
        self.slots[s] = [cells, 0.0, 0, self.rate_of(cfg)]
        self.used += cells
        self.admitted.append((cfg.nx, cfg.Delta))
        self.max_running = max(self.max_running, len(self.slots))
        return s

    def remove(self, slot):
        self.used -= self.slots.pop(slot)[0]

    def step(self, n):
        for v in self.slots.values():
            v[1] += v[3] * n
            v[2] += n

    def tips(self):
        t = np.full(self.max_slots, np.nan)
        st = np.zeros(self.max_slots, np.int64)
        for s, v in self.slots.items():
            t[s], st[s] = v[1], v[2]
        return t, st

    def field(self, slot, name):
        return np.zeros((1, 4, 4))

    def sync(self):
        pass

    def close(self):
        self.closed = True


def fake_clock(step=1e-3):
    t = [0.0]

    def clock():
        t[0] += step
        return t[0]
    return clock


def reqs(edges, t_arrive=0.0, u=0.5):
    return [dict(id=i, t_arrive=t_arrive + 1e-3 * i, edge=e, u=u + 0.01 * i, eps4=0.04, delta_offset=0.6)
            for i, e in enumerate(edges)]


def test_admission_in_arrival_order_within_capacity():
    fb = FakeBatch(cell_capacity=2 * 128 * 128)          # room for two 128^2 runs at a time
    srv = serve.SweepServer(chunk=10, target=0.8, batch=fb)
    rq = reqs([128] * 5)
    res = srv.run(rq, clock=fake_clock())
    assert fb.max_running == 2
    assert [d for _, d in fb.admitted] == [r["delta_offset"] + r["u"] for r in rq]   # first come, first served
    assert len(res) == 5 and all(r["completed"] for r in res)
    for r in res:
        # the tip grows 1 cell per step; the target is 80 % of the half-width (51.2 cells): 60 steps
        assert r["steps"] == 60 and r["tip"] >= 0.8 * 64
        assert r["latency"] == pytest.approx(r["t_done"] - r["t_arrive"]) and r["latency"] > 0
        assert r["t_admit"] >= r["t_arrive"]
    assert fb.used == 0 and not fb.slots


def test_large_request_waits_and_blocks_later_ones():
    # a 256^2 request needs the whole arena: it waits until both 128^2 runs retire,
    # and the 128^2 request behind it is not admitted ahead of it
    fb = FakeBatch(cell_capacity=256 * 256)
    srv = serve.SweepServer(chunk=10, target=0.8, batch=fb)
    rq = reqs([128, 128, 256, 128])
    res = srv.run(rq, clock=fake_clock())
    assert [e for e, _ in fb.admitted] == [128, 128, 256, 128]
    done = {r["id"]: r for r in res}
    assert done[2]["t_admit"] >= max(done[0]["t_done"], done[1]["t_done"])
    assert done[3]["t_admit"] >= done[2]["t_admit"]


def test_step_limit_retires_unfinished_runs():
    fb = FakeBatch(cell_capacity=1 << 20, rate_of=lambda cfg: 0.0 if cfg.nx == 512 else 1.0)
    srv = serve.SweepServer(chunk=16, target=0.8, max_steps=64, batch=fb)
    res = {r["edge"]: r for r in srv.run(reqs([128, 512]), clock=fake_clock())}
    assert res[128]["completed"] and res[128]["steps"] == 64       # 4 chunks of 16 reach 51.2 cells
    assert not res[512]["completed"] and res[512]["steps"] == 64    # never grows: retired at the limit
    srv.close()
    assert fb.closed


def test_summary_percentiles_and_rate():
    res = [dict(latency=float(k), t_arrive=0.0, t_done=float(k), completed=k % 2 == 0) for k in range(1, 101)]
    s = serve.summarize(res)
    assert s["runs"] == 100 and s["completed"] == 50
    assert s["makespan_s"] == 100.0 and s["runs_per_s"] == pytest.approx(1.0)
    assert s["p50_latency_s"] == pytest.approx(np.percentile(np.arange(1, 101), 50))
    assert s["p99_latency_s"] == pytest.approx(np.percentile(np.arange(1, 101), 99))


def test_sweep_requests_are_seeded_and_in_range():
    a, b = serve.sweep_requests(n=64, seed=3), serve.sweep_requests(n=64, seed=3)
    assert a == b
    assert all(r["edge"] in (128, 256, 512, 1024) for r in a)
    assert all(0.3 <= r["u"] <= 0.65 and 0.02 <= r["eps4"] <= 0.06 for r in a)
    t = [r["t_arrive"] for r in a]
    assert t == sorted(t) and t[0] > 0
    c = serve.request_config(a[0])
    assert c.Delta == pytest.approx(0.6 + a[0]["u"]) and c.delta == pytest.approx(4 * a[0]["eps4"])
    assert (c.nx, c.ny, c.nz, c.bc, c.ic) == (a[0]["edge"], a[0]["edge"], 1, 1, 1)


def test_request_larger_than_the_batch_is_rejected_not_waited_on():
    # the 512^2 request needs more cells than the whole arena holds: once nothing is
    # running it is returned as rejected, and the requests behind it are still served
    fb = FakeBatch(cell_capacity=2 * 128 * 128)
    srv = serve.SweepServer(chunk=10, target=0.8, batch=fb)
    res = {r["id"]: r for r in srv.run(reqs([128, 512, 128]), clock=fake_clock())}
    assert len(res) == 3
    assert not res[1]["completed"] and res[1]["steps"] == 0 and "rejected" in res[1]
    assert res[0]["completed"] and res[2]["completed"]
    assert [e for e, _ in fb.admitted] == [128, 128]


def test_batch_without_slots_rejects_every_request():
    fb = FakeBatch(cell_capacity=1 << 20, max_slots=0)
    srv = serve.SweepServer(chunk=10, target=0.8, batch=fb)
    res = srv.run(reqs([128, 256]), clock=fake_clock())
    assert len(res) == 2 and not any(r["completed"] for r in res) and all("rejected" in r for r in res)
