#!/usr/bin/env python
"""Benchmark of the DBA stencil hot path (active cell-updates/s, HBM roofline).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one time step of the DBA path over the whole grid.  Default workload
`modelb_2048_fp32_conserved`: reactive Model B on a 2048^2 periodic grid, FP32
stencils with FP64 conserved-change sums, 16x16 blocks, conserved DBA.  The
state is pre-rolled (untimed) to the middle of the 50 000-step run so the timed
steps see a representative active set, then W warm-up and K timed steps run on
the engine's own CUDA stream, bracketed by CUDA events (max over ranks).

Multi-GPU: the path does not shard in this build (one domain per GPU), so
`--gpus N` runs N independent replicas, one process per GPU, and `value` is the
sum of their active cell-updates divided by the slowest rank's time.

At N=1 the line also carries:
  * `workloads`: the other workloads measured the same way (value, roofline,
    vs_dense, e2e, cpu_baseline) -- the 512^2 FP64 dendrite, the 512^3 FP32
    dendrite and the 4096^2 FP32 KH flow, each pre-rolled to mid-run
    (`--no-side-workloads` skips them);
  * `full_runs_dba_vs_regular`: whole runs to the same end time in DBA and in
    regular mode with total wall times -- the dendrite workloads (512^2 FP64,
    10 000 steps; 512^3 FP32, 20 000 steps), the Model B workload (50 000 steps)
    and the KH flow to simulated time 2 (62 880 steps) at the wake-up thresholds
    of `--full-runs-kh` (default 1, the workload's) (`--no-full-runs` skips them);
  * `sweep`: the batched/served 2-D dendrite parameter sweep (256 seeded
    requests, Poisson arrivals, admission by device memory, autotuned block edge
    and threads) against the same requests run one at a time -- runs/s of both
    and p50/p99 time to completion (`--no-sweep` skips it).
For FP32 workloads, `fp32_error_vs_fp64` gives the relative L2 error and the
largest difference of each state field after `--error-steps` steps (default
1000) on the full grid, against the FP64 engine from the same initial state.

`--impl reference` times the reference's own serial CPU program for the same
model, built from the reference sources under oracle/_ref (Model B and KH: its
functions driven step by step by *_cpu_steps; dendrite: the program itself,
an n-step run minus a 0-step run) on this host; rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# bytes read + written per active cell-update by the algorithm (state fields only)
ALG_BYTES = {"dendrite": 4, "modelb": 6, "kh": 8}   # x element size

WORKLOADS = {
    # C1: reactive Model B, conserved DBA.  Symmetric quench inside the z-b
    # spinodal (x0=y0=0.05, z0=0.45, uniform noise +-0.01, chi_zb=3), mobility 1,
    # gradient coefficient 1, reaction rate 1e-4, dt=0.001 (0.005 diverges).
    "modelb_2048_fp32_conserved": dict(
        model="modelb", nx=2048, ny=2048, nz=1, block=16, precision=1, conserved=1, mode=1, t_total=50000,
        params=dict(dt=0.001, chi_zb=3.0, eps_x=1.0, eps_y=1.0, eps_z=1.0, k_0=1e-4, metric_eps=1e-3, x0=0.05,
                    y0=0.05, z0=0.45, noise_amp=0.02, noise_amp_z=0.02)),
    # C0: 2-D dendrite, FP64, 512^2, tanh seed r=10 at the centre, zero-flux walls, 8x8 blocks; undercooling
    # 0.55 and eps4 0.05 mapped onto the Kobayashi model as Delta = 0.6 + 0.55, delta = 4 eps4 (as the sweep)
    "dendrite_512_fp64": dict(
        model="dendrite", nx=512, ny=512, nz=1, block=8, precision=0, conserved=0, mode=1, t_total=10000,
        params=dict(Delta=1.15, delta=0.2, metric_p=1e-3, metric_T=1e-5, ic=1, ic_radius=10.0, ic_width=2.0, bc=1)),
    # C3: 3-D dendrite, FP32, 512^3, 8^3 blocks, tanh seed r=10 at the corner cell, zero-flux walls, C0's mapping
    "dendrite3d_512_fp32": dict(
        model="dendrite", nx=512, ny=512, nz=512, block=8, precision=1, conserved=0, mode=1, t_total=20000,
        params=dict(Delta=1.15, delta=0.2, metric_p=1e-3, metric_T=1e-5, ic=1, ic_radius=10.0, ic_width=2.0, bc=1,
                    ic_corner=1)),
    # C2: KH 4096^2 FP32, 16x16 blocks, gamma 1.4, sharp bands + seeded noise, CFL 0.4 chosen on the device;
    # simulated time 2 is reached after 62 880 steps (measured in both modes)
    "kh_4096_fp32": dict(
        model="kh", nx=4096, ny=4096, nz=1, block=16, precision=1, conserved=0, mode=1, t_total=62880,
        params=dict(dt=1.0 / 4096 * 0.4 / 3.0, dx=1.0 / 4096, dy=1.0 / 4096, kh_gamma=1.4, metric_eps=1.0, ic=2,
                    noise_amp=1e-4, cfl=0.4)),
    # the same flow on a 2048^2 grid (512 MB of state, above L2): the size kernel profiles are taken on
    "kh_2048_fp32": dict(
        model="kh", nx=2048, ny=2048, nz=1, block=16, precision=1, conserved=0, mode=1, t_total=24500,
        params=dict(dt=1.0 / 2048 * 0.4 / 3.0, dx=1.0 / 2048, dy=1.0 / 2048, kh_gamma=1.4, metric_eps=1.0, ic=2,
                    noise_amp=1e-4, cfl=0.4)),
}


def make_config(w):
    import dba_b200
    c = dba_b200.config(w["model"], nx=w["nx"], ny=w["ny"], nz=w["nz"], block=w["block"],
                        precision=w["precision"], conserved=w["conserved"])
    for k, v in w["params"].items():
        setattr(c, k, v)
    c.t_total = w["t_total"]
    return c


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        try:
            rows = [r.split(",") for r in open(self.out.name).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def aggregate(ms, cells, world, device="cuda"):
    """Replica aggregation: the slowest rank's time and the sum of all ranks' cell-updates.
    Every rank takes the same collective steps in the same order."""
    if world <= 1:
        return ms, cells
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(cells)], device=device, dtype=torch.float64)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measure(args, name, w, steps, warmup, preroll, world=1, rank=0, local=0, cpu_seconds=None,
            e2e_from="snapshot"):
    """One workload: `preroll` untimed steps, `warmup` more, then `steps` timed steps on the
    engine's stream (CUDA events; the max over ranks when world > 1), the dominant kernel's
    roofline, the same state in regular (dense) mode, and the end-to-end leg through the
    public API with host buffers.  Returns the JSON fields of the workload (rank 0)."""
    import numpy as np
    import torch

    import dba_b200

    cfg = make_config(w)
    sim = dba_b200.Simulation(cfg).init()
    stream = torch.cuda.ExternalStream(sim.stream)
    if preroll:
        sim.step(preroll, w["mode"])
    sim.step(warmup, w["mode"])
    sim.sync()
    # host copy of this state: the end-to-end run below starts from it
    blob = torch.empty(sim.state_size(), dtype=torch.uint8, pin_memory=True)
    sim.save_state(blob)
    sim.step_profiled(1, w["mode"])           # also a final warm-up of the direct-launch path
    sim.load_state(blob)
    # runs of 6 steps or more go through CUDA graphs (48- and 6-step, per start phase and mode),
    # captured on first use: capture the ones the timed steps use now, outside the timed region
    sim.step(steps, w["mode"])
    sim.load_state(blob)
    sim.sync()

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    st0 = sim.cell_updates()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        sim.step(steps, w["mode"])
        ev1.record(stream)
        torch.cuda.synchronize()
    status = sim._L.dba_sync(sim._h)
    ms = ev0.elapsed_time(ev1)
    cells = sim.cell_updates() - st0
    t_max, cells_all = aggregate(ms, cells, world)

    # dominant kernel: the fused stencil kernel, timed per launch with CUDA events on the same stream
    sim.load_state(blob)
    nprof = min(steps, 200)
    prof = sim.step_profiled(nprof, w["mode"])
    esz = 8 if w["precision"] == 0 else 4
    per_cell = ALG_BYTES[w["model"]] * esz
    if w["model"] == "dendrite":
        alg = esz * (2 * prof["active_blocks_ch"][0] + 2 * prof["active_blocks_ch"][1] + prof["ch0_only_blocks"]) \
            * prof["cells_per_block"]
    else:
        alg = per_cell * prof["active_blocks"] * prof["cells_per_block"]
    # average launch duration of the dominant kernel: when a step is that kernel (with its tile
    # scan, about 3 % of the step, where it has one), the timed region itself (K steps between
    # two events); otherwise its per-launch events
    if step_is_stencil(w):
        kernel_ms = ms / max(1, steps)
        alg_per_launch = cells * per_cell / max(1, steps) if w["model"] != "dendrite" else alg / nprof
    else:
        kernel_ms = prof["stencil_ms"] / nprof
        alg_per_launch = alg / nprof
    achieved = alg_per_launch / (kernel_ms * 1e-3) / 1e9 if kernel_ms > 0 else 0.0
    peak, peak_kind = hbm_peak()
    traffic = None
    tfile = os.path.join(ROOT, "profiles", f"{name}.traffic.json")
    if os.path.exists(tfile) and prof["active_blocks"]:
        try:
            tj = json.load(open(tfile))
            traffic = tj["dram_bytes_per_active_cell"] * prof["active_blocks"] * prof["cells_per_block"] / nprof
        except Exception:
            traffic = None

    # the same state advanced in regular (dense, every block) mode and in the workload's mode, both
    # through the captured-graph path and timed with CUDA events, for the DBA-vs-dense comparison
    def graph_ms(mode):
        sim.load_state(blob)
        sim.step(ncmp, mode)
        sim.load_state(blob)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        c0 = sim.cell_updates()
        e0.record(stream)
        sim.step(ncmp, mode)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / ncmp, (sim.cell_updates() - c0) / ncmp

    ncmp = min(max(steps, 48), 1000)
    dense_ms, dense_cells = graph_ms(0)
    dba_ms, _ = graph_ms(w["mode"])

    # end to end through the public API, host buffers in page-locked memory.  e2e_from ==
    # "initial fields": the workload's initial state fields go host -> device (dba_init_f32 for
    # FP32, dba_init for FP64), K steps, the state fields come back in the context's precision
    # (dba_read_field_f32 / dba_read_field) -- a whole run of K steps.  "snapshot": the mid-run
    # state is resumed from a host snapshot (dba_load_state), K steps, fields back.
    n = cfg.nx * cfg.ny * cfg.nz
    nf = {"dendrite": 2, "modelb": 3, "kh": 4}[w["model"]]
    f32 = w["precision"] == 1
    hdt = torch.float32 if f32 else torch.float64
    out_host = torch.empty((nf, n), dtype=hdt, pin_memory=True).numpy()   # page-locked result buffer
    read = (lambda q: sim.field_f32(q, out=out_host[q])) if f32 else (lambda q: sim.field(q, out=out_host[q]))
    ic_host = None
    if e2e_from == "initial fields":
        # the workload's own initial condition, as the caller would hold it
        sim.init()
        names = ["rho", "p", "vx", "vy"] if w["model"] == "kh" else list(range(nf))
        ic_host = torch.empty(nf * n, dtype=hdt, pin_memory=True).numpy()
        for q, nm in enumerate(names):
            ic_host[q * n:(q + 1) * n] = (sim.field_f32(nm) if f32 else sim.field(nm)).ravel()
        ic_list = None if f32 else [ic_host[q * n:(q + 1) * n] for q in range(nf)]

        def start():
            return sim.init_f32(ic_host) if f32 else sim.init(ic_list)
        start()
        sim.step(steps, w["mode"])   # graphs of this start phase, outside the timed region
        torch.cuda.synchronize()
    else:
        def start():
            sim.load_state(blob)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    start()
    st_e0 = sim.cell_updates()
    sim.step(steps, w["mode"])
    for q in range(nf):
        read(q)
    t_e2e = (time.perf_counter() - t0) * 1e3
    cells_e2e = sim.cell_updates() - st_e0
    h2d = ic_host.nbytes if ic_host is not None else blob.numel()
    d2h = out_host.nbytes
    t_e2e, cells_e2e = aggregate(t_e2e, cells_e2e, world)

    res = None
    if rank == 0:
        total_blocks = sim.info.nb
        res = {
            "value": cells_all / (t_max * 1e-3), "unit": "cell-updates/s", "steps": steps, "warmup": warmup,
            "ms_per_step": t_max / steps, "dtype": "f32" if w["precision"] else "f64",
            "config": {"workload": name, "model": w["model"], "grid": [cfg.nx, cfg.ny, cfg.nz],
                       "block": cfg.block, "conserved": bool(cfg.conserved), "mode": "DBA" if w["mode"] else "regular",
                       "metric_eps": w["params"].get("metric_eps"),
                       "preroll_steps": preroll,
                       "active_fraction": cells / max(1, steps) / (total_blocks * prof["cells_per_block"]),
                       "l2": ("state larger than L2 (%.0f MB resident), no flush" if sim.info.device_bytes > 126e6
                              else "state of %.0f MB fits in L2; no flush (the workload itself is L2-resident)")
                       % (sim.info.device_bytes / 1e6),
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": cells_e2e / (t_e2e * 1e-3), "unit": "cell-updates/s",
                    "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
                    "from": e2e_from, "ms": t_e2e, "host_dtype": "f32" if f32 else "f64"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "kernel": f"{w['model']}_step", "peak_kind": peak_kind,
                         "alg_bytes_per_active_cell": per_cell, "kernel_ms_avg": kernel_ms,
                         "kernel_timing": ("timed region, tile scan + tile kernel per step" if queue_path(w)
                                           else "timed region, one launch per step") if step_is_stencil(w)
                         else "per-launch CUDA events",
                         "frac_of_8tbs_spec": achieved / 8000.0},
            "step_breakdown_ms": {"stencil": prof["stencil_ms"] / nprof, "reduce": prof["reduce_ms"] / nprof,
                                  "correct": prof["correct_ms"] / nprof},
            "vs_dense": {"dba_ms_per_step": dba_ms, "dense_ms_per_step": dense_ms,
                         "dense_over_dba_time": dense_ms / dba_ms if dba_ms else None,
                         "dense_cell_updates_per_s": dense_cells / (dense_ms * 1e-3) if dense_ms else None,
                         "steps": ncmp, "timing": "captured graphs, CUDA events, same starting state"},
            "gpu_launches": steps * launches_per_step(w),
            "clocks": clk.summary(),
            "status": status,
        }
        if world == 1 and cpu_seconds:
            res["cpu_baseline"] = cpu_baseline(w, seconds=cpu_seconds)
    sim.close()
    return res


# the other workloads measured beside the headline (N = 1): untimed steps before the
# measurement, at least 48 timed steps
SIDE_WORKLOADS = {"dendrite_512_fp64": 5000, "dendrite3d_512_fp32": 10000, "kh_4096_fp32": 31440}


def run_ours(args, w):
    import datetime

    import torch
    import torch.distributed as dist

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    preroll = w["t_total"] // 2 if args.preroll < 0 else args.preroll
    # the headline's e2e is a whole run from host initial fields (every block of the Model B
    # workload is active from its first step to its last, so the active set is the timed one)
    m = measure(args, args.workload, w, args.steps, args.warmup, preroll, world, rank, local,
                cpu_seconds=None if args.no_cpu_baseline else args.cpu_seconds,
                e2e_from="initial fields" if w["model"] == "modelb" else "snapshot")
    result = None
    if rank == 0:
        result = {"metric": "active cell-updates/s", "value": m["value"], "unit": "cell-updates/s", "n_gpus": world,
                  "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
                  "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": m["dtype"],
                  "data": "synthetic (seeded initial condition)"}
        result.update({k: v for k, v in m.items() if k not in result and k not in ("steps", "warmup")})
        if world == 1 and not args.no_side_workloads:
            side = {}
            for name, pre in SIDE_WORKLOADS.items():
                if name == args.workload:
                    continue
                side[name] = measure(args, name, WORKLOADS[name], max(args.steps, 48), args.warmup, pre,
                                     cpu_seconds=None if args.no_cpu_baseline else args.side_cpu_seconds)
            result["workloads"] = side
        if world == 1 and not args.no_sweep:
            result["sweep"] = run_sweep(args)
        if world == 1 and not args.no_full_runs:
            result["full_runs_dba_vs_regular"] = run_full_runs(args)
        if world == 1 and w["precision"] == 1 and args.error_steps > 0:
            result["fp32_error_vs_fp64"] = run_fp32_error(w, args.error_steps)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


def queue_path(w):
    """Workloads whose step is a scan kernel listing the step's tiles and the tile kernel that
    takes them (KH tiles, FP32 3-D dendrite tiles)."""
    return w["model"] == "kh" or (w["model"] == "dendrite" and w["nz"] > 1 and w["precision"] == 1)


def launches_per_step(w):
    """This engine's kernel launches per step."""
    if w["model"] == "kh":   # tile scan + tile kernel (grids of 16-cell multiples, blocks 8 or 16)
        return 2 + (2 if w["conserved"] else 0)
    if queue_path(w):
        return 2
    if w["model"] == "modelb" and w["conserved"] and not (w["precision"] == 1 and w["nz"] == 1):
        return 3   # FP64 / 3-D conserved: step, reduce, correct
    return 1       # FP32 2-D conserved Model B: the reduction is inside the step kernel


def step_is_stencil(w):
    """The step is the stencil kernel alone (with its tile scan where it has one): no separate
    conserved reduction and correction launches."""
    return launches_per_step(w) == (2 if queue_path(w) else 1)


def _ref_input(w, nx, ny):
    p = w["params"]
    if w["model"] == "modelb":
        return (f"{nx} {ny} 1\n10 5 {p['dt']}\n1 1 1\n0 0 0 0 0 {p.get('chi_zb', 4)}\n1 1 2\n1 1 2\n1 1\n"
                f"{p['eps_x']} {p['eps_y']} {p['eps_z']} 0.01\n1 1 1 1\n{p['x0']} {p['y0']} {p['z0']}\n100 0.4 1\n"
                f"{p['k_0']}\n{p['metric_eps']}\n0\n")
    if w["model"] == "kh":
        return f"{nx} {ny} 1\n10 5 {p['dt']}\n{p['dx']} {p['dy']} {p['dx']}\n0\n0\n"
    raise ValueError(w["model"])


def time_reference_cpu(w, nsteps):
    """Wall time of nsteps steps of the reference's serial CPU program on the workload's grid."""
    binary = {"modelb": "modelb_cpu_steps", "kh": "kh_cpu_steps"}.get(w["model"])
    path = os.path.join(ROOT, "oracle", "_ref", binary) if binary else None
    d = tempfile.mkdtemp()
    if path and os.path.exists(path):
        with open(os.path.join(d, "Input.txt"), "w") as f:
            f.write(_ref_input(w, w["nx"], w["ny"]))
        out = subprocess.run([path, os.path.join(d, "Input.txt"), str(nsteps), "-"], capture_output=True, text=True,
                             check=True).stdout
        secs = float([ln for ln in out.splitlines() if ln.startswith("LOOP_SECONDS")][-1].split()[1])
        return secs, "reference", f"{binary} (reference CPU_version functions, regular mode, FP64)"
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from cases import DENDRITE_REF
    prm = dict(DENDRITE_REF, **{k: v for k, v in w["params"].items() if k in DENDRITE_REF})
    den = os.path.join(ROOT, "oracle", "_ref", "dendrite_cpu")
    if w["model"] == "dendrite" and os.path.exists(den):
        # the reference's own dendrite CPU program (CPU_version/Base.cpp, single precision, regular
        # mode): it reads ./Input.txt and writes no output while t_freq > t_total; the loop time is
        # the wall time of an nsteps run minus that of a 0-step run (setup, allocation, seed)
        def run(k):
            d = tempfile.mkdtemp()
            with open(os.path.join(d, "Input.txt"), "w") as f:
                f.write(f"{w['nx']} {w['ny']} {w['nz']}\n{k} {k + 1} {prm['dt']}\n{prm['dx']} {prm['dx']} {prm['dx']}\n"
                        f"{prm['delta']} {prm['tau']} {prm['epsilon']} {prm['alpha']} {prm['gamma']}\n{prm['Delta']}\n")
            t0 = time.perf_counter()
            subprocess.run([den], cwd=d, check=True, stdout=subprocess.DEVNULL)
            return time.perf_counter() - t0
        secs = max(run(nsteps) - run(0), 1e-9)
        return secs, "reference", "dendrite_cpu (reference CPU_version/Base.cpp, regular mode, float; n-step minus 0-step run)"
    # no reference program built: time the FP64 restatement
    from oracle_lib import OracleDendrite
    o = OracleDendrite(w["nx"], w["ny"], w["nz"], w["block"], prm, bc=w["params"].get("bc", 0))
    o.init_cone()
    t0 = time.perf_counter()
    o.step(nsteps, 0)
    return time.perf_counter() - t0, "port", "oracle restatement, regular mode, FP64"


def cpu_baseline(w, seconds=15.0):
    cells = w["nx"] * w["ny"] * w["nz"]
    # size the sample to about `seconds` of CPU time from a short probe
    t1, kind, what = time_reference_cpu(w, 1)
    n = max(1, min(200, int(seconds / max(t1, 1e-3))))
    t, kind, what = time_reference_cpu(w, n)
    return {"value": cells * n / t, "unit": "cell-updates/s", "cores": 1, "kind": kind,
            "sample": f"{what}: {w['nx']}x{w['ny']}x{w['nz']} grid, {n} steps (all cells updated), {t:.2f} s, 1 thread"}


def run_sweep(args):
    """Batched/served 2-D dendrite parameter sweep against sequential single-simulation runs.

    Seeded requests (grid edge from {128, 256, 512, 1024}, undercooling and
    anisotropy uniform, seed radius 8, FP32, each run until its tip reaches 80 %
    of the domain half-width) arrive as a Poisson stream.  The server admits
    them by device memory into one batch (one kernel launch per step over the
    merged active blocks of every admitted run, captured in CUDA graphs), with
    the block edge and threads per CTA picked by the autotuner.  The same
    requests are then run one at a time, each in its own context.  Reported:
    runs/s of both, p50/p99 time to completion of the served run, and how far
    each served result is from its sequential twin."""
    from dba_b200 import autotune, serve

    choice = autotune.tune(precision=1, use_cache=False)
    reqs = serve.sweep_requests(n=args.sweep_requests, rate=args.sweep_rate, seed=args.sweep_seed)
    srv = serve.SweepServer(precision=1, block=choice["block"], threads=choice["threads"], chunk=choice["chunk"],
                            persistent=choice.get("persistent", 1))
    t0 = time.perf_counter()
    res = srv.run(reqs)
    t_batched = time.perf_counter() - t0
    srv.close()
    summ = serve.summarize(res)
    t0 = time.perf_counter()
    seq = serve.run_sequential(reqs, precision=1, block=choice["block"], chunk=choice["chunk"])
    t_seq = time.perf_counter() - t0
    by_id = {r["id"]: r for r in seq}
    tip_rel = max(abs(r["tip"] - by_id[r["id"]]["tip"]) / max(abs(by_id[r["id"]]["tip"]), 1e-30) for r in res)
    same_steps = sum(r["steps"] == by_id[r["id"]]["steps"] for r in res)
    return {
        "requests": len(reqs), "arrival_rate_per_s": args.sweep_rate, "seed": args.sweep_seed,
        "autotune": {"block": choice["block"], "threads": choice["threads"], "chunk": choice["chunk"],
                     "launch": "persistent" if choice.get("persistent", 1) else "one per step",
                     "scores": choice.get("scores")},
        "batched_runs_per_s": summ["runs_per_s"], "sequential_runs_per_s": len(seq) / t_seq,
        "speedup": (summ["runs_per_s"] * t_seq / len(seq)) if summ["runs_per_s"] else None,
        "p50_latency_s": summ.get("p50_latency_s"), "p99_latency_s": summ.get("p99_latency_s"),
        "makespan_s": summ["makespan_s"], "sequential_wall_s": t_seq,
        "completed": summ["completed"], "completed_sequential": int(sum(r["completed"] for r in seq)),
        "max_tip_rel_diff_vs_sequential": tip_rel, "same_stop_step": same_steps,
        "note": "makespan from first arrival to last completion; sequential runs back to back, FP32 both",
    }


STATE_FIELDS = {"dendrite": ("p", "T"), "modelb": ("x", "y", "z"), "kh": ("Mass", "Momx", "Momy", "Energy")}


def run_fp32_error(w, nsteps):
    """Error of the FP32 engine on the workload's full grid against the FP64 engine (whose
    fields equal the CPU restatement bit for bit at every step, in the parity tests): both
    advanced nsteps in the workload's mode from the same initial state; per state field the
    relative L2 error and the largest absolute difference."""
    import numpy as np
    import dba_b200

    ref, act, status = {}, [], []
    out = {"steps": nsteps, "mode": "DBA" if w["mode"] else "regular",
           "against": "FP64 engine (bit-identical to the FP64 CPU restatement)", "fields": {}}
    for prec in (0, 1):
        sim = dba_b200.Simulation(make_config(dict(w, precision=prec))).init()
        sim.step(nsteps, w["mode"])
        status.append(sim._L.dba_sync(sim._h))
        act.append(float(np.mean(sim.flags(0) != 0)))
        for f in STATE_FIELDS[w["model"]]:
            a = sim.field(f)
            if prec == 0:
                ref[f] = a
            else:
                d = a - ref[f]
                nrm = float(np.linalg.norm(ref[f]))
                out["fields"][f] = {"rel_l2": float(np.linalg.norm(d)) / nrm if nrm else None,
                                    "max_abs": float(np.max(np.abs(d)))}
        sim.close()
    out["active_fraction_fp64_fp32"] = act
    out["status"] = status
    return out


def run_full_runs(args):
    """DBA against the all-blocks regular mode over whole runs of the dendrite workloads and
    the Model B workload (and of the KH flow with the wake-up thresholds of --full-runs-kh):
    each advanced from its initial state to its end in both modes (captured graphs, CUDA
    events on the engine's stream), with the active fraction and the tip or simulated time
    at the end (the KH step count is the one that reaches simulated time 2)."""
    import torch
    import dba_b200

    out = {}
    runs = [(n, WORKLOADS[n]) for n in ("dendrite_512_fp64", "dendrite3d_512_fp32", "modelb_2048_fp32_conserved")]
    for eps in (args.full_runs_kh.split(",") if args.full_runs_kh else []):
        w = WORKLOADS["kh_4096_fp32"]
        runs.append((f"kh_4096_fp32_eps{float(eps):g}", dict(w, params=dict(w["params"], metric_eps=float(eps)))))
    for name, w in runs:
        row = {"steps": w["t_total"], "grid": [w["nx"], w["ny"], w["nz"]], "dtype": "f32" if w["precision"] else "f64"}
        if w["model"] == "kh":
            row["metric_eps"] = w["params"]["metric_eps"]
        for mode, key in ((1, "dba"), (0, "regular")):
            sim = dba_b200.Simulation(make_config(w)).init()
            stream = torch.cuda.ExternalStream(sim.stream)
            sim.step(48, mode)        # captures the step graph (every 48-step launch from step 0 reuses it)
            sim.sync()
            sim.init()                # back to the initial state; the graph stays valid
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            c0 = sim.cell_updates()
            e0.record(stream)
            nsteps = w["t_total"]
            sim.step(nsteps, mode)
            e1.record(stream)
            torch.cuda.synchronize()
            row[key + "_s"] = e0.elapsed_time(e1) / 1e3
            row[key + "_mean_active_fraction"] = (sim.cell_updates() - c0) / (nsteps * sim.n)
            if w["model"] == "dendrite":
                row[key + "_tip"] = sim.tip()
            else:
                row[key + "_time"] = sim.observables()["time"]
            sim.close()
        row["dba_speedup"] = row["regular_s"] / row["dba_s"] if row["dba_s"] else None
        out[name] = row
    return out


def run_reference(args, w):
    world, rank, local = dist_setup()
    if rank != 0:
        return None
    # each bench step is one reference time step on the full grid; the warm-up
    # steps are timed in a separate run and subtracted
    secs, kind, what = time_reference_cpu(w, args.warmup + args.steps)
    if args.warmup:
        t_w, _, _ = time_reference_cpu(w, args.warmup)
        secs = max(secs - t_w, 1e-9)
    cells = w["nx"] * w["ny"] * w["nz"] * args.steps
    value = cells / secs
    return {
        "metric": "active cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded initial condition)",
        "impl": "reference",
        "config": {"workload": args.workload, "model": w["model"], "grid": [w["nx"], w["ny"], w["nz"]],
                   "mode": "regular (the reference CPU program has no DBA)"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": 1, "kind": kind,
                         "sample": f"{what}: {w['nx']}x{w['ny']}x{w['nz']}, {args.steps} timed steps"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def _finite(v):
    """The JSON line with non-finite numbers (a tip past the domain, say) as null."""
    import math
    if isinstance(v, dict):
        return {k: _finite(x) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [_finite(x) for x in v]
    if isinstance(v, float) and not math.isfinite(v):
        return None
    return v


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="modelb_2048_fp32_conserved", choices=sorted(WORKLOADS))
    ap.add_argument("--preroll", type=int, default=-1, help="untimed steps before warm-up (default: half the run)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--side-cpu-seconds", type=float, default=6.0,
                    help="CPU time of each side workload's reference CPU sample")
    ap.add_argument("--no-side-workloads", action="store_true",
                    help="skip the other workloads (512^2 dendrite, 512^3 dendrite, KH 4096^2) measured beside the headline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the batched dendrite sweep section")
    ap.add_argument("--no-full-runs", action="store_true",
                    help="skip the whole-run DBA-vs-regular comparison of the dendrite workloads")
    ap.add_argument("--full-runs-kh", default="1", metavar="EPS[,EPS..]",
                    help="KH flow (4096^2, to simulated time 2) whole runs with these wake-up thresholds "
                         "(default: the workload's, 1; empty: none)")
    ap.add_argument("--error-steps", type=int, default=1000,
                    help="steps of the FP32-against-FP64 error check on the full grid (0: skip)")
    ap.add_argument("--sweep-requests", type=int, default=256)
    ap.add_argument("--sweep-rate", type=float, default=200.0, help="Poisson arrival rate, requests per second")
    ap.add_argument("--sweep-seed", type=int, default=0)
    ap.add_argument("--metric-eps", type=float, default=None,
                    help="override the workload's wake-up threshold (Model B, KH), e.g. 0 to keep every block "
                         "active for a profile of the all-active DBA step")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    w = WORKLOADS[args.workload]
    if args.metric_eps is not None:
        if w["model"] == "dendrite":
            ap.error("--metric-eps applies to Model B and KH workloads")
        w = dict(w, params=dict(w["params"], metric_eps=args.metric_eps))
        WORKLOADS[args.workload] = w
    if args.impl == "reference":
        if args.steps > 40:
            args.steps = 40   # each reference step is a full dense CPU step; keep the run to minutes
        if args.warmup > 2:
            args.warmup = 2
        res = run_reference(args, w)
    else:
        res = run_ours(args, w)
    if res is not None:
        print(json.dumps(_finite(res)), flush=True)


if __name__ == "__main__":
    main()
