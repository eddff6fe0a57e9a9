"""Continuous-batching service for dendrite parameter sweeps.

Requests arrive over time (Poisson arrivals); each is one 2-D dendrite
simulation with its own grid edge, undercooling and anisotropy, run until its
tip (growth_front at x = Nx/2) reaches a fraction of the domain half-width.  The
server keeps one batch (dba_batch_*: one kernel launch per step over the active
blocks of every admitted simulation, fields resident on the GPU) and loops:

  * admit waiting requests, in arrival order, while the batch's device arena,
    block space and slot table have room (admission by device memory);
  * advance every admitted simulation `chunk` steps;
  * read all tips with one small kernel; retire the finished simulations,
    freeing their memory for the next admissions.

A request that does not fit even in an empty batch (more cells, blocks or slots
than the batch was created with) is returned at once with completed=False and
a `rejected` reason, so the requests behind it are still served.

Requests that arrive while others are on the GPU join at the next chunk
boundary, so their work overlaps on the device.  Latency is completion time
minus arrival time.

The sequential baseline runs the same requests one at a time, each in its own
single-simulation context (dba_create/dba_step), with the same chunking.
"""
import collections
import time

import numpy as np

from . import engine

# Kobayashi p/T parameters of the reference (example_Dendritic_growth/Input.txt)
REFERENCE = dict(dt=5e-5, dx=0.02, tau=0.0003, epsilon=0.01, alpha=0.9, gamma=40.0, metric_p=1e-3, metric_T=1e-5)


def sweep_requests(n=256, rate=200.0, seed=0, edges=(128, 256, 512, 1024), undercooling=(0.3, 0.65),
                   anisotropy=(0.02, 0.06), delta_offset=0.6):
    """Seeded sweep: grid edge uniform over `edges`, undercooling u and 4-fold
    anisotropy eps4 uniform over their ranges, Poisson arrivals at `rate` per
    second.  Mapped onto the Kobayashi p/T model: Delta = delta_offset + u (with
    unit latent heat a radius-8 seed keeps growing only near Delta >= 0.9; below
    it the interface warms and the tip remelts or splits) and anisotropy strength
    delta = 4 eps4 (sigma = 1 - delta (1 - |n|_4^4) varies by delta/4 around its
    mean, the amplitude eps4 describes)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    out = []
    for i in range(n):
        out.append(dict(id=i, t_arrive=float(t[i]), edge=int(rng.choice(edges)),
                        u=float(rng.uniform(*undercooling)), eps4=float(rng.uniform(*anisotropy)),
                        delta_offset=delta_offset))
    return out


def request_config(req, precision=1, block=8, radius=8.0):
    c = engine.config("dendrite", nx=req["edge"], ny=req["edge"], nz=1, block=block, precision=precision,
                      bc=1, ic=1, ic_radius=radius, ic_width=2.0)
    for k, v in REFERENCE.items():
        setattr(c, k, v)
    c.dy = c.dz = c.dx
    c.Delta = req["delta_offset"] + req["u"]
    c.delta = 4.0 * req["eps4"]
    return c


def _done(tip, edge, target):
    return np.isfinite(tip) and tip >= target * edge / 2


class SweepServer:
    def __init__(self, precision=1, block=8, max_slots=128, block_capacity=1 << 17, cell_capacity=0, chunk=96,
                 target=0.8, max_steps=200000, threads=256, batch=None, persistent=1):
        """`batch`: an object with the engine.Batch methods add / remove / step / tips /
        field / sync / close to serve from (default: a new engine.Batch on the current device,
        with persistent (1) or per-step (0) launches)."""
        if batch is None:
            batch = engine.Batch(precision=precision, block=block, max_slots=max_slots,
                                 block_capacity=block_capacity, cell_capacity=cell_capacity, threads=threads)
            batch.set_option(engine.BATCH_PERSISTENT, persistent)
        self.batch = batch
        self.precision, self.block, self.chunk = precision, block, chunk
        self.target, self.max_steps = target, max_steps

    def run(self, requests, keep_fields=False, clock=time.perf_counter):
        pending = collections.deque(sorted(requests, key=lambda r: r["t_arrive"]))
        waiting = collections.deque()
        running = {}
        results = []
        t0 = clock()
        while pending or waiting or running:
            now = clock() - t0
            while pending and pending[0]["t_arrive"] <= now:
                waiting.append(pending.popleft())
            while waiting:
                req = waiting[0]
                slot = self.batch.add(request_config(req, self.precision, self.block))
                if slot is None:
                    if running:
                        break                   # no room: wait for retirements
                    # nothing is running, so nothing will free room: this request can
                    # never be admitted (larger than the batch's arena, block space or
                    # slot table); reject it and serve the ones behind it
                    waiting.popleft()
                    now = clock() - t0
                    results.append(dict(req, t_done=now, latency=now - req["t_arrive"], tip=float("nan"), steps=0,
                                        completed=False, rejected="does not fit in an empty batch"))
                    continue
                waiting.popleft()
                running[slot] = dict(req, t_admit=clock() - t0)
            if not running:
                if pending:
                    time.sleep(max(0.0, pending[0]["t_arrive"] - (clock() - t0)))
                continue
            self.batch.step(self.chunk)
            tips, steps = self.batch.tips()     # synchronises
            now = clock() - t0
            for slot in list(running):
                req = running[slot]
                if _done(tips[slot], req["edge"], self.target) or steps[slot] >= self.max_steps:
                    r = dict(req, t_done=now, latency=now - req["t_arrive"], tip=float(tips[slot]),
                             steps=int(steps[slot]), completed=bool(_done(tips[slot], req["edge"], self.target)))
                    if keep_fields:
                        r["p"] = self.batch.field(slot, "p")
                        r["T"] = self.batch.field(slot, "T")
                    results.append(r)
                    self.batch.remove(slot)
                    del running[slot]
        self.batch.sync()
        return results

    def close(self):
        self.batch.close()


def run_sequential(requests, precision=1, block=8, chunk=96, target=0.8, max_steps=200000, keep_fields=False,
                   clock=time.perf_counter):
    """The same requests one at a time, each in its own single-simulation context."""
    results = []
    t0 = clock()
    for req in sorted(requests, key=lambda r: r["t_arrive"]):
        ts = clock() - t0
        sim = engine.Simulation(request_config(req, precision, block)).init()
        steps = 0
        tip = float("nan")
        while steps < max_steps:
            sim.step(chunk, 1)
            steps += chunk
            tip = sim.tip()
            if _done(tip, req["edge"], target):
                break
        r = dict(req, t_start=ts, t_done=clock() - t0, tip=tip, steps=steps, completed=_done(tip, req["edge"], target))
        if keep_fields:
            r["p"] = sim.field("p")
            r["T"] = sim.field("T")
        sim.close()
        results.append(r)
    return results


def summarize(results, makespan=None):
    lat = np.array([r["latency"] for r in results]) if results and "latency" in results[0] else None
    if makespan is None:
        makespan = max(r["t_done"] for r in results) - min(r["t_arrive"] for r in results)
    out = {"runs": len(results), "completed": int(sum(r["completed"] for r in results)),
           "makespan_s": makespan, "runs_per_s": len(results) / makespan if makespan > 0 else None}
    if lat is not None and len(lat):
        out["p50_latency_s"] = float(np.percentile(lat, 50))
        out["p99_latency_s"] = float(np.percentile(lat, 99))
    return out


def main(argv=None):
    """python -m dba_b200.serve: run one seeded sweep through the server and print its summary."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rate", type=float, default=200.0, help="Poisson arrivals per second (0: all at once)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", type=int, default=1, help="1 FP32, 0 FP64")
    ap.add_argument("--block", type=int, default=8)
    ap.add_argument("--threads", type=int, default=256)
    ap.add_argument("--chunk", type=int, default=96)
    ap.add_argument("--persistent", type=int, default=1, help="1 persistent batch launches, 0 one launch per step")
    a = ap.parse_args(argv)
    srv = SweepServer(precision=a.precision, block=a.block, threads=a.threads, chunk=a.chunk, persistent=a.persistent)
    res = srv.run(sweep_requests(n=a.requests, rate=a.rate, seed=a.seed))
    srv.close()
    print(json.dumps(summarize(res)))


if __name__ == "__main__":
    main()
