"""Batched simulations (dba_batch_*) and the continuous-batching server."""
import numpy as np
import pytest

import dba_b200
from dba_b200 import serve
from cases import DENDRITE_REF, dendrite_cfg
from oracle_lib import OracleDendrite

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("B,bc", [(4, 0), (8, 1)])
def test_batch_slot_fp64_bitexact_vs_oracle(B, bc):
    """A slot of an FP64 batch advances exactly as the CPU restatement does."""
    b = dba_b200.Batch(precision=0, block=B, max_slots=4, block_capacity=4096, cell_capacity=1 << 16)
    other = b.add(dendrite_cfg(dict(DENDRITE_REF, Delta=0.6), 32, 48, 1, B, precision=0, bc=1))
    s = b.add(dendrite_cfg(DENDRITE_REF, 64, 64, 1, B, precision=0, bc=bc))
    o = OracleDendrite(64, 64, 1, B, DENDRITE_REF, bc=bc)
    o.init_cone()
    for _ in range(3):
        b.step(20)
        o.step(20, 1)
        d = o.get()
        assert np.array_equal(b.field(s, "p"), d["p"])
        assert np.array_equal(b.field(s, "T"), d["T"])
    b.step(100)      # graph path
    o.step(100, 1)
    d = o.get()
    assert np.array_equal(b.field(s, "p"), d["p"])
    tips, steps = b.tips()
    assert tips[s] == o.tip() and steps[s] == 160 and steps[other] == 160
    b.sync()


@pytest.mark.parametrize("bc", [0, 1])
def test_batch_slot_fp32_equals_single_simulation(bc):
    """The FP32 batch kernel and the single-simulation FP32 kernel evaluate the same
    explicitly rounded point formulas (den_p_f32 / den_T_f32), so a slot of an FP32
    batch holds the same bits as the same simulation advanced on its own, step after
    step, periodic and zero-flux (several slots share the batch)."""
    b = dba_b200.Batch(precision=1, block=8, max_slots=4, block_capacity=4096, cell_capacity=1 << 16)
    b.add(dendrite_cfg(dict(DENDRITE_REF, Delta=0.6), 32, 48, 1, 8, precision=1, bc=1))
    s = b.add(dendrite_cfg(DENDRITE_REF, 64, 64, 1, 8, precision=1, bc=bc))
    sim = dba_b200.Simulation(dendrite_cfg(DENDRITE_REF, 64, 64, 1, 8, precision=1, bc=bc)).init()
    for n in (1, 19, 20, 120):
        b.step(n)
        sim.step(n, 1)
        assert np.array_equal(b.field(s, "p"), sim.field("p")), n
        assert np.array_equal(b.field(s, "T"), sim.field("T")), n
    b.sync()
    sim.sync()


def _req(edge, u, eps4, i=0):
    return dict(id=i, t_arrive=0.0, edge=edge, u=u, eps4=eps4, delta_offset=0.6)


def test_same_result_alone_and_in_the_mix():
    """Continuous batching: a simulation admitted while others are running gives
    bit-identical fields to the same simulation alone in a batch."""
    target = serve.request_config(_req(128, 0.4, 0.03))
    alone = dba_b200.Batch(precision=1, block=8, max_slots=8, block_capacity=1 << 14, cell_capacity=1 << 20)
    a = alone.add(target)
    alone.step(300)
    p_alone, T_alone = alone.field(a, "p"), alone.field(a, "T")
    mix = dba_b200.Batch(precision=1, block=8, max_slots=8, block_capacity=1 << 14, cell_capacity=1 << 20)
    s1 = mix.add(serve.request_config(_req(256, 0.6, 0.05, 1)))
    mix.step(97)
    s2 = mix.add(serve.request_config(_req(128, 0.3, 0.02, 2)))
    mix.step(50)
    t = mix.add(target)                     # joins while two others are on the GPU
    mix.step(150)
    mix.remove(s1)                          # a neighbour in block space retires mid-run
    s3 = mix.add(serve.request_config(_req(64 * 2, 0.5, 0.06, 3)))
    mix.step(150)
    _, steps = mix.tips()
    assert steps[t] == 300
    assert np.array_equal(mix.field(t, "p"), p_alone)
    assert np.array_equal(mix.field(t, "T"), T_alone)
    assert s2 != t and s3 >= 0
    mix.sync()


def test_admission_by_device_memory():
    b = dba_b200.Batch(precision=1, block=8, max_slots=16, block_capacity=1 << 12, cell_capacity=3 * 128 * 128)
    slots = [b.add(serve.request_config(_req(128, 0.4, 0.04, i))) for i in range(4)]
    assert slots[:3] == [0, 1, 2] and slots[3] is None          # the arena holds three 128^2 runs
    b.remove(1)
    assert b.add(serve.request_config(_req(128, 0.4, 0.04, 9))) == 1
    big = b.add(serve.request_config(_req(256, 0.4, 0.04, 10)))
    assert big is None
    assert b.info().live_slots == 3


def test_server_completes_sweep_and_matches_single_runs():
    reqs = serve.sweep_requests(n=6, rate=0.0, seed=3, edges=(128, 256))
    srv = serve.SweepServer(precision=1, block=8, max_slots=8, chunk=96)
    res = srv.run(reqs, keep_fields=False)
    srv.close()
    assert len(res) == 6 and all(r["completed"] for r in res)
    seq = serve.run_sequential(reqs, precision=1, block=8, chunk=96)
    by_id = {r["id"]: r for r in seq}
    for r in res:
        s = by_id[r["id"]]
        assert s["completed"] and s["steps"] == r["steps"]
        assert abs(s["tip"] - r["tip"]) <= 0.01 * abs(s["tip"])
    summ = serve.summarize(res)
    assert summ["p99_latency_s"] >= summ["p50_latency_s"] > 0


def test_sweep_fp32_error_vs_fp64():
    """A sweep run in FP32 against the same run in FP64 (FP64 slots are bit-exact with
    the CPU restatement): tip velocity within 1 %, relative L2 of p and T <= 1e-4."""
    req = _req(128, 0.45, 0.04)
    out = {}
    for prec in (1, 0):
        b = dba_b200.Batch(precision=prec, block=8, max_slots=2, block_capacity=1 << 12, cell_capacity=1 << 16)
        s = b.add(serve.request_config(req, precision=prec))
        b.step(480)
        t1, _ = b.tips()
        b.step(480)
        t2, steps = b.tips()
        out[prec] = dict(v=(t2[s] - t1[s]) / 480.0, tip=t2[s], p=b.field(s, "p"), T=b.field(s, "T"))
        b.close()
    f32, f64 = out[1], out[0]
    assert f64["tip"] >= 0.6 * 64                                     # the tip has crossed most of the half-width
    assert abs(f32["v"] - f64["v"]) <= 0.01 * abs(f64["v"])
    for k in ("p", "T"):
        assert np.linalg.norm(f32[k] - f64[k]) / np.linalg.norm(f64[k]) <= 1e-4, k


def _mixed_batch(persistent, precision=1):
    b = dba_b200.Batch(precision=precision, block=8, max_slots=8, block_capacity=1 << 14, cell_capacity=1 << 21)
    b.set_option(dba_b200.BATCH_PERSISTENT, persistent)
    slots = [b.add(serve.request_config(_req(e, u, k, i), precision=precision))
             for i, (e, u, k) in enumerate(((256, 0.6, 0.05), (128, 0.3, 0.02), (512, 0.45, 0.04)))]
    return b, slots


@pytest.mark.parametrize("precision", [0, 1])
def test_persistent_launch_equals_one_launch_per_step(precision):
    """The persistent form (one cooperative launch of up to 48 steps, grid barrier
    between steps) gives the same fields bit for bit as one launch per step, over
    graph-sized runs, direct remainders and an admission between launches."""
    a, sa = _mixed_batch(1, precision)
    b, sb = _mixed_batch(0, precision)
    for n in (5, 48, 96, 7):
        a.step(n)
        b.step(n)
        for x, y in zip(sa, sb):
            assert np.array_equal(a.field(x, "p"), b.field(y, "p")), n
            assert np.array_equal(a.field(x, "T"), b.field(y, "T")), n
    ta = a.add(serve.request_config(_req(128, 0.5, 0.03, 9), precision=precision))
    tb = b.add(serve.request_config(_req(128, 0.5, 0.03, 9), precision=precision))
    a.step(60)
    b.step(60)
    assert np.array_equal(a.field(ta, "p"), b.field(tb, "p"))
    assert np.array_equal(a.tips()[0], b.tips()[0], equal_nan=True)
    a.sync()
    b.sync()


def test_grid_barrier_wait_limit_reports_timeout():
    """With a wait limit of 0 polls, every CTA that reaches a grid barrier before the
    last one gives up at once: the launch ends early and dba_batch_sync reports
    DBA_ERR_TIMEOUT (a host-visible status; the context stays usable)."""
    b, _ = _mixed_batch(1)
    b.set_option(dba_b200.BATCH_WAIT_LIMIT, 0)
    b.step(10)
    with pytest.raises(dba_b200.DBAError) as e:
        b.sync()
    assert e.value.code == 6
    # the device is still fine: a new batch runs normally
    c, sc = _mixed_batch(1)
    c.step(10)
    c.sync()
    assert np.all(np.isfinite(c.field(sc[0], "p")))
