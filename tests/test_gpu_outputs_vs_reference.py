"""The drop-in's output files against the reference programs' own, and the
observables' values against restatements of the reference's formulas.

1. dba_run (the drop-in binary) runs the Input.txt stored in
   tests/golden/ref_out_{modelb,kh}.npz, on which the reference's serial CPU
   programs wrote the stored files (tests/golden/make_output_golden.py).  Both run
   regular mode in FP64 from the same initial condition; the engine's transcendentals
   differ from glibc's in the last bits, so values are compared with Compare_VTK's
   measure (example_Dendritic_growth/Compare_VTK.cpp:57-73) at 1e-5 of the values'
   L1 norm, and the .out tables (6 significant digits) to 1e-5 relative.  Headers and
   section names must be identical.
2. dba_observables: the integrals (Integral, example_Reactive_ModelB/kernel.cu:989-1010,
   example_Kelvin_Helmholtz/KH_DBA.cu:1273-1288) and the KH vy mode amplitude
   (Calc_Vy_mode, KH_DBA.cu:1291-1327) against numpy restatements evaluated on the
   CPU restatement's fields; the dendrite's RTValues.out velocity and active
   fractions (Calc_RealTime_Values, example_Dendritic_growth/kernel.cu:791-863)
   against the CPU restatement's tip and flags.
"""
import os
import subprocess

import numpy as np
import pytest

import dba_b200
from cases import DENDRITE_REF, KH_REF, MODELB_REF, kh_cfg, modelb_cfg
from oracle_lib import OracleDendrite, OracleKH, OracleModelB
from vtk_text import compare_vtk, read_table, read_vtk

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DBA_RUN = os.path.join(ROOT, "dba_b200", "bin", "dba_run")


def _run(model, text, d):
    with open(os.path.join(d, "Input.txt"), "w") as f:
        f.write(text)
    subprocess.run([DBA_RUN, model, "Input.txt", "--quiet"], cwd=d, check=True, stdout=subprocess.DEVNULL)


def _same_vtk(path, g, t):
    header, sec = read_vtk(path)
    assert "\n".join(header) == str(g[f"vtk{t}_header"])
    assert " ".join(sec) == str(g[f"vtk{t}_sections"])
    for name, v in sec.items():
        ref = g[f"vtk{t}_{name}"]
        assert v.shape == ref.shape, name
        m = compare_vtk(v, ref)
        assert m["relative"] <= 1e-5, (t, name, m)


def _same_table(path, ref):
    got = read_table(path)
    assert got.shape == ref.shape, (path, got.shape, ref.shape)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-12), (path, got, ref)


def test_modelb_files_match_reference_cpu_program(tmp_path):
    g = np.load(os.path.join(HERE, "golden", "ref_out_modelb.npz"))
    _run("modelb", str(g["input"]), tmp_path)
    for t in (0, 10, 20):
        _same_vtk(tmp_path / f"output_{t}.vtk", g, t)
    _same_table(tmp_path / "Integral.out", g["out_Integral_out"])


def test_kh_files_match_reference_cpu_program(tmp_path):
    g = np.load(os.path.join(HERE, "golden", "ref_out_kh.npz"))
    _run("kh", str(g["input"]), tmp_path)
    # the reference GPU program's names (output_<mode>_<t>.vtk); the CPU program writes output_<t>.vtk
    for t in (0, 10, 20):
        _same_vtk(tmp_path / f"output_0_{t}.vtk", g, t)
    _same_table(tmp_path / "Integral_mass.out", g["out_Integral_mass_out"])
    _same_table(tmp_path / "VY_mode.out", g["out_VY_mode_out"])


def vy_mode(vy):
    """Calc_Vy_mode restated (KH_DBA.cu:1291-1327); vy is (ny, nx)."""
    ny, nx = vy.shape
    xs = np.arange(nx) / nx
    ys = np.arange(ny) / ny
    c = np.where(ys < 0.5, 0.25, 0.75)
    w = np.exp(-4.0 * np.pi * np.abs(ys - c))[:, None]
    ss = np.sum(vy * np.sin(4.0 * np.pi * xs)[None, :] * w)
    sc = np.sum(vy * np.cos(4.0 * np.pi * xs)[None, :] * w)
    sd = np.sum(np.broadcast_to(w, vy.shape))
    return 2.0 * np.sqrt(ss * ss / (sd * sd) + sc * sc / (sd * sd))


def output_vy(o, prm, B):
    """vy as the reference's output path leaves it (KH_DBA.cu:1509-1537): getPrimitive_wakeup
    recomputes the primitives of the blocks flagged for the next step (vy = Momy / rho / vol,
    rho = Mass / vol, :403-404) before Calc_Vy_mode reads them; other blocks keep theirs."""
    vy = o.field("vy")[0].copy()
    vol = prm["dx"] * prm["dy"]
    rho = o.field("Mass")[0] / vol
    fresh = o.field("Momy")[0] / rho / vol
    wake = o.flags()[0].reshape(vy.shape[0] // B, vy.shape[1] // B)
    mask = np.kron(wake, np.ones((B, B), dtype=wake.dtype)).astype(bool)
    vy[mask] = fresh[mask]
    return vy


@pytest.mark.parametrize("conserved", [0, 1])
def test_kh_observables_values(conserved):
    prm = dict(KH_REF, metric_eps=10.0)
    o = OracleKH(64, 64, 8, prm, conserved=conserved)
    o.init_smooth()
    s = dba_b200.Simulation(kh_cfg(prm, 64, 64, 8, conserved=conserved)).init()
    for n in (0, 25, 25):
        o.step(n, 1)
        s.step(n, 1)
        ob = s.observables()
        assert ob["vy_mode"] == pytest.approx(vy_mode(output_vy(o, prm, 8)), rel=1e-12, abs=1e-15)
        want = [o.field(f).sum() for f in ("Mass", "Energy", "Momx", "Momy")] if conserved else [o.field("Mass").sum()]
        assert np.allclose(ob["integral"][:len(want)], want, rtol=1e-12, atol=1e-15), (ob["integral"], want)


def test_modelb_observables_values():
    prm = dict(MODELB_REF, metric_eps=1e-3)
    o = OracleModelB(64, 64, 1, 4, prm, conserved=1)
    o.init_mt()
    s = dba_b200.Simulation(modelb_cfg(prm, 64, 64, 1, 4, conserved=1)).init()
    for n in (0, 30, 30):
        o.step(n, 1)
        s.step(n, 1)
        ob = s.observables()
        want = [o.field(f).sum() for f in ("x", "y", "z", "b")]
        assert np.allclose(ob["integral"], want, rtol=1e-12), (ob["integral"], want)
        w = o.flags()[0]
        assert ob["active_blocks"][0] == int(w.sum())


def test_dendrite_rtvalues_velocity_and_fractions(tmp_path):
    """RTValues.out written by dba_run: at every t_freq, Vel = (tip - previous tip) / t_freq
    from growth_front at x = Nx/2 (the previous tip starts at 0, as in the reference),
    Act_portion_p / _T = active fractions of the next step's blocks."""
    nx, t_total, t_freq = 64, 400, 100
    p = DENDRITE_REF
    text = (f"{nx} {nx} 1\n{t_total} {t_freq} {p['dt']}\n{p['dx']} {p['dx']} {p['dx']}\n"
            f"{p['delta']} {p['tau']} {p['epsilon']} {p['alpha']} {p['gamma']}\n{p['Delta']}\n1\n{p['metric_p']}\n"
            f"{p['metric_T']}\n")
    with open(tmp_path / "Input.txt", "w") as f:
        f.write(text)
    subprocess.run([DBA_RUN, "dendrite", "Input.txt", "--quiet"], cwd=tmp_path, check=True, stdout=subprocess.DEVNULL)
    rt = read_table(tmp_path / "RTValues.out")
    assert rt.shape == (t_total // t_freq, 5)
    o = OracleDendrite(nx, nx, 1, 4, DENDRITE_REF)
    o.init_cone()
    prev = 0.0
    for k in range(t_total // t_freq):
        o.step(t_freq, 1)
        tip = o.tip()
        d = o.get()
        assert rt[k, 0] == (k + 1) * t_freq
        assert rt[k, 1] == pytest.approx((tip - prev) / t_freq, rel=1e-5, abs=1e-9)
        assert rt[k, 2] == pytest.approx(d["wake_p"].mean(), rel=1e-5)
        assert rt[k, 3] == pytest.approx(d["wake_T"].mean(), rel=1e-5)
        prev = tip
