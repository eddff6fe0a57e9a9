"""Engine (CUDA, through the C ABI) against the CPU restatement on the same inputs.

FP64: every field value and every block flag must be bit-identical at every
step (the oracle runs in its shared-fpmath flavour, the engine's FP64 kernels
are built with -fmad=false).  FP32: tolerances stated per test.
"""
import numpy as np
import pytest

import dba_b200
from cases import DENDRITE_REF, KH_REF, MODELB_REF, dendrite_cfg, kh_cfg, modelb_cfg
from oracle_lib import OracleDendrite, OracleKH, OracleModelB

pytestmark = pytest.mark.gpu


def _flags_equal(sim, which, ref):
    got = sim.flags(which)
    assert np.array_equal(got, ref.astype(np.int32)), (which, np.flatnonzero(got != ref)[:10])


@pytest.mark.parametrize("nx,ny,nz,B,mode,bc", [
    (64, 64, 1, 4, 1, 0), (64, 64, 1, 4, 0, 0), (64, 48, 1, 8, 1, 0), (64, 64, 1, 16, 1, 0),
    (64, 64, 1, 4, 1, 1), (24, 24, 24, 4, 1, 0), (32, 32, 32, 8, 1, 0), (24, 24, 24, 4, 0, 1)])
def test_dendrite_fp64_bitexact_per_step(nx, ny, nz, B, mode, bc):
    steps = 40 if nz == 1 else 12
    o = OracleDendrite(nx, ny, nz, B, DENDRITE_REF, bc=bc)
    o.init_cone()
    s = dba_b200.Simulation(dendrite_cfg(DENDRITE_REF, nx, ny, nz, B, bc=bc)).init()
    for t in range(1, steps + 1):
        o.step(1, mode)
        s.step(1, mode)
        d = o.get()
        assert np.array_equal(s.field("p"), d["p"]), ("p", t)
        assert np.array_equal(s.field("T"), d["T"]), ("T", t)
        if mode:
            _flags_equal(s, 0, d["wake_p"])
            _flags_equal(s, 2, d["wake_T"])
            _flags_equal(s, 1, d["next_p"])
            _flags_equal(s, 3, d["next_T"])
    assert s.tip() == o.tip() or (np.isnan(s.tip()) and np.isnan(o.tip()))
    s.sync()


def test_dendrite_graph_path_matches_oracle():
    """dba_step(n >= 48) replays captured CUDA graphs; results stay bit-identical."""
    o = OracleDendrite(64, 64, 1, 4, DENDRITE_REF)
    o.init_cone()
    s = dba_b200.Simulation(dendrite_cfg(DENDRITE_REF, 64, 64, 1, 4)).init()
    s.step(3, 1)          # off the 6-step graph phase on purpose
    s.step(200, 1)
    o.step(203, 1)
    d = o.get()
    assert np.array_equal(s.field("p"), d["p"])
    assert np.array_equal(s.field("T"), d["T"])
    _flags_equal(s, 0, d["wake_p"])
    _flags_equal(s, 2, d["wake_T"])


@pytest.mark.parametrize("nx,ny,nz,B,mode,conserved,eps", [
    (64, 64, 1, 4, 1, 0, 1e-3), (64, 64, 1, 4, 1, 1, 1e-3), (64, 64, 1, 4, 0, 0, 1e-3),
    (64, 64, 1, 8, 1, 1, 1e-3), (64, 64, 1, 16, 1, 1, 1e-3), (16, 16, 16, 4, 1, 1, 1e-3), (16, 16, 16, 8, 1, 0, 1e-3)])
def test_modelb_fp64_bitexact_per_step(nx, ny, nz, B, mode, conserved, eps):
    prm = dict(MODELB_REF, metric_eps=eps)
    steps = 90 if nz == 1 else 25
    o = OracleModelB(nx, ny, nz, B, prm, conserved=conserved)
    o.init_mt()
    s = dba_b200.Simulation(modelb_cfg(prm, nx, ny, nz, B, conserved=conserved)).init()
    for t in range(1, steps + 1):
        o.step(1, mode)
        s.step(1, mode)
        if t % 3 == 0 or t == steps:
            for f in ("x", "y", "z"):
                assert np.array_equal(s.field(f), o.field(f)), (f, t)
        if mode:
            w, nxt = o.flags()
            _flags_equal(s, 0, w)
            _flags_equal(s, 1, nxt)
    s.sync()


@pytest.mark.parametrize("B,mode,conserved,eps", [(4, 1, 0, 10.0), (4, 1, 1, 10.0), (4, 0, 0, 10.0), (8, 1, 1, 50.0),
                                                  (16, 1, 0, 10.0)])
def test_kh_fp64_bitexact_per_step(B, mode, conserved, eps):
    nx = ny = 64
    prm = dict(KH_REF, metric_eps=eps)
    o = OracleKH(nx, ny, B, prm, conserved=conserved)
    o.init_smooth()
    s = dba_b200.Simulation(kh_cfg(prm, nx, ny, B, conserved=conserved)).init()
    for t in range(1, 61):
        o.step(1, mode)
        s.step(1, mode)
        if t % 4 == 0 or t == 60:
            for f in ("Mass", "Momx", "Momy", "Energy"):
                assert np.array_equal(s.field(f), o.field(f)), (f, t)
        if mode:
            w, nxt = o.flags()
            _flags_equal(s, 0, w)
            _flags_equal(s, 1, nxt)
    for f in ("rho", "p", "vx", "vy"):
        assert np.all(np.isfinite(s.field(f)))
    s.sync()


def test_dendrite_fp32_within_tolerance():
    """FP32 stencils against the FP64 oracle after 300 DBA steps: |dp|, |dT| <= 2e-5, tip within 1e-3 cells."""
    o = OracleDendrite(128, 128, 1, 8, DENDRITE_REF)
    o.init_cone()
    s = dba_b200.Simulation(dendrite_cfg(DENDRITE_REF, 128, 128, 1, 8, precision=1)).init()
    o.step(300, 1)
    s.step(300, 1)
    d = o.get()
    assert np.max(np.abs(s.field("p") - d["p"])) <= 2e-5
    assert np.max(np.abs(s.field("T") - d["T"])) <= 2e-5
    assert abs(s.tip() - o.tip()) <= 1e-3


def test_modelb_fp32_within_tolerance():
    """FP32 Model B (conserved DBA) against FP64: relative L2 <= 1e-4 per field after 200 steps."""
    prm = dict(MODELB_REF, metric_eps=1e-3)
    o = OracleModelB(64, 64, 1, 16, prm, conserved=1)
    o.init_mt()
    s = dba_b200.Simulation(modelb_cfg(prm, 64, 64, 1, 16, precision=1, conserved=1)).init()
    o.step(200, 1)
    s.step(200, 1)
    for f in ("x", "y", "z"):
        a, b = s.field(f), o.field(f)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-4, f


def test_kh_fp32_within_tolerance():
    prm = dict(KH_REF, metric_eps=10.0)
    o = OracleKH(64, 64, 8, prm, conserved=1)
    o.init_smooth()
    s = dba_b200.Simulation(kh_cfg(prm, 64, 64, 8, precision=1, conserved=1)).init()
    o.step(100, 1)
    s.step(100, 1)
    for f in ("Mass", "Momx", "Momy", "Energy"):
        a, b = s.field(f), o.field(f)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-4, f


@pytest.mark.parametrize("model", ["dendrite", "modelb", "kh"])
def test_checkpoint_restore_bitexact(tmp_path, model):
    if model == "dendrite":
        cfg = dendrite_cfg(DENDRITE_REF, 64, 64, 1, 4)
    elif model == "modelb":
        cfg = modelb_cfg(dict(MODELB_REF, metric_eps=1e-3), 64, 64, 1, 8, conserved=1)
    else:
        cfg = kh_cfg(dict(KH_REF, metric_eps=10.0), 64, 64, 8, conserved=1)
    a = dba_b200.Simulation(cfg).init()
    a.step(17, 1)
    a.checkpoint(tmp_path / "c.bin")
    a.step(60, 1)
    b = dba_b200.Simulation(cfg)
    b.restore(tmp_path / "c.bin")
    b.step(60, 1)
    for f in a.fields[:3]:
        assert np.array_equal(a.field(f), b.field(f)), f
    assert np.array_equal(a.flags(0), b.flags(0))


def test_nonfinite_status_reported():
    """A state that produces NaN is reported by dba_sync as DBA_ERR_NONFINITE (host-visible status)."""
    prm = dict(MODELB_REF, metric_eps=1e-3)
    cfg = modelb_cfg(prm, 32, 32, 1, 4)
    s = dba_b200.Simulation(cfg)
    x = np.full((1, 32, 32), 0.2)
    x[0, 5, 5] = -1.0          # log of a negative fraction -> NaN in the chemical potential
    s.init([x, np.full_like(x, 0.2), np.full_like(x, 0.01)])
    s.step(2, 1)
    with pytest.raises(dba_b200.DBAError) as e:
        s.sync()
    assert e.value.code == 5


def test_modelb_fp32_lazy_conserved_mass():
    """FP32 conserved DBA (lazy correction, exact fixed-point change totals, reduction
    fused in the step kernel): the total of each species stays at its initial value
    (relative drift <= 1e-10 after 1000 steps), and the fields track the FP64
    dense-correction oracle to relative L2 <= 1e-4."""
    prm = dict(MODELB_REF, metric_eps=1e-3, chi_zb=3.0, eps_x=1.0, eps_y=1.0, eps_z=1.0, k_0=1e-4,
               x0=0.05, y0=0.05, z0=0.45)
    cfg = modelb_cfg(prm, 64, 64, 1, 16, precision=1, conserved=1, noise_amp=0.02, noise_amp_z=0.02)
    s = dba_b200.Simulation(cfg).init()
    m0 = [s.field(f).sum() for f in ("x", "y", "z")]
    s.step(1000, 1)
    s.sync()
    m1 = [s.field(f).sum() for f in ("x", "y", "z")]
    for a, b in zip(m0, m1):
        assert abs(b - a) / abs(a) <= 1e-10, (a, b)
    o = OracleModelB(64, 64, 1, 16, prm, conserved=1)
    o.init_mt(amp=0.02, z_amp=0.02)
    o.step(1000, 1)
    for f in ("x", "y", "z"):
        a, b = s.field(f), o.field(f)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-4, f


@pytest.mark.parametrize("tiles", [1, 0])
def test_modelb_fp32_lazy_offset_across_mode_switches(tiles):
    """The lazy conserved offset of an FP32 context applies in every mode: conserved
    DBA steps, then regular steps (offset kept, not accumulated), then DBA again,
    track the FP64 oracle running the same sequence with its dense correction."""
    prm = dict(MODELB_REF, metric_eps=1e-3)
    o = OracleModelB(64, 64, 1, 16, prm, conserved=1)
    o.init_mt()
    s = dba_b200.Simulation(modelb_cfg(prm, 64, 64, 1, 16, precision=1, conserved=1, tiles=tiles)).init()
    # FP32 error grows with the step count (with k_0 = 1 the approximate exp/log of the
    # reaction bias the mean change slightly); the bound follows it
    for n, mode, tol in ((100, 1, 1e-4), (100, 0, 1e-4), (60, 1, 3e-4)):
        o.step(n, mode)
        s.step(n, mode)
        for f in ("x", "y", "z"):
            a, b = s.field(f), o.field(f)
            assert np.linalg.norm(a - b) / np.linalg.norm(b) <= tol, (f, n, mode)


@pytest.mark.parametrize("B", [4, 8, 32])
def test_modelb_fp32_fast_path_block_edges(B):
    prm = dict(MODELB_REF, metric_eps=1e-3)
    o = OracleModelB(64, 64, 1, B, prm, conserved=0)
    o.init_mt()
    s = dba_b200.Simulation(modelb_cfg(prm, 64, 64, 1, B, precision=1)).init()
    o.step(120, 1)
    s.step(120, 1)
    for f in ("x", "y", "z"):
        a, b = s.field(f), o.field(f)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-4, f
    agree = np.mean(s.flags(0) == o.flags()[0])
    assert agree >= 0.98


def test_field_into_caller_buffer():
    """field(name, out=...) fills a caller-provided (here page-locked) float64 array with
    the same values field(name) returns, and rejects a buffer of the wrong size or type."""
    import torch

    prm = dict(MODELB_REF, metric_eps=1e-3)
    s = dba_b200.Simulation(modelb_cfg(prm, 64, 64, 1, 16, precision=1, conserved=1)).init()
    s.step(20, 1)
    buf = torch.empty(64 * 64, dtype=torch.float64, pin_memory=True).numpy()
    for f in ("x", "y", "z", "b"):
        got = s.field(f, out=buf)
        assert np.array_equal(got, s.field(f)), f
    with pytest.raises(ValueError):
        s.field("x", out=np.empty(10))
    with pytest.raises(ValueError):
        s.field("x", out=np.empty(64 * 64, np.float32))


@pytest.mark.parametrize("model", ["dendrite", "modelb", "kh"])
def test_fp32_init_and_readback(model):
    """dba_init_f32 gives the same run as dba_init with the same values in FP64, and
    dba_read_field_f32 returns dba_read_field's values rounded to float."""
    if model == "dendrite":
        cfg = dendrite_cfg(DENDRITE_REF, 64, 64, 1, 8, precision=1)
    elif model == "modelb":
        cfg = modelb_cfg(dict(MODELB_REF, metric_eps=1e-3), 64, 64, 1, 16, precision=1, conserved=1)
    else:
        cfg = kh_cfg(dict(KH_REF, metric_eps=10.0), 64, 64, 8, precision=1)
    a = dba_b200.Simulation(cfg).init()
    nic = {"dendrite": 2, "modelb": 3, "kh": 4}[model]
    names = a.fields[:nic] if model != "kh" else ["rho", "p", "vx", "vy"]
    ic = np.concatenate([a.field_f32(f).ravel() for f in names]).astype(np.float32)
    b = dba_b200.Simulation(cfg).init_f32(ic)
    c = dba_b200.Simulation(cfg).init([ic[k * a.n:(k + 1) * a.n].astype(np.float64) for k in range(nic)])
    for s in (b, c):
        s.step(30, 1)
    for f in b.fields[:nic]:
        assert np.array_equal(b.field(f), c.field(f)), f
        assert np.array_equal(b.field_f32(f), c.field(f).astype(np.float32)), f
    b.sync()
