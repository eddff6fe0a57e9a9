"""Pin the CPU restatement (oracle/) to the reference's own code.

1. Golden fixtures tests/golden/ref_cpu_*.npz were produced by the reference's
   serial CPU programs (example_Reactive_ModelB/CPU_version/base_CPU.cpp,
   example_Kelvin_Helmholtz/CPU_version/KH_CPU.cpp) driven step by step
   (tests/golden/make_cpu_golden.py).  The oracle's regular mode in its glibc
   flavour must reproduce every FP64 value bit for bit.
2. Golden fixtures tests/golden/ref_gpu_*.npz (when present) were produced by
   the reference's own GPU DBA kernels on a B200 (tests/golden/make_gpu_golden.py).
   The oracle's DBA mode must give the same per-step active-block sets and the
   same fields within FP64 library-rounding tolerance.
"""
import os

import numpy as np
import pytest

from cases import KH_REF, MODELB_REF, DENDRITE_REF
from oracle_lib import OracleDendrite, OracleKH, OracleModelB

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_modelb_regular_bitexact_vs_reference_cpu():
    g = np.load(os.path.join(GOLD, "ref_cpu_modelb.npz"))
    nx, ny = int(g["nx"]), int(g["ny"])
    prm = dict(MODELB_REF, dt=float(g["dt"]))
    o = OracleModelB(nx, ny, 1, 4, prm, libm=True)
    o.init_mt()
    o.step(int(g["steps"]), mode=0)
    for f in ("x", "y", "z", "b", "mu_x", "mu_y", "mu_z"):
        assert np.array_equal(o.field(f)[0], g[f]), f


def test_kh_regular_bitexact_vs_reference_cpu():
    g = np.load(os.path.join(GOLD, "ref_cpu_kh.npz"))
    nx, ny = int(g["nx"]), int(g["ny"])
    prm = dict(KH_REF, dt=float(g["dt"]), dx=float(g["dx"]), dy=float(g["dx"]))
    o = OracleKH(nx, ny, 8, prm)
    o.init_smooth()
    o.step(int(g["steps"]), mode=0)
    for f in ("Mass", "Momx", "Momy", "Energy", "rho", "p", "vx", "vy"):
        assert np.array_equal(o.field(f)[0], g[f]), f


def _gpu_fixture(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated yet (tests/golden/make_gpu_golden.py on a B200)")
    return np.load(path)


def _compare_run(g, oracle, field_names, flag_names, get_fields, get_flags, rtol):
    steps, every = int(g["steps"]), int(g["every"])
    flags = g["flags"]            # [steps][nflag][nb]
    fields = g["fields"]          # [1 + steps//every][nfield][...]
    mismatched = 0
    for t in range(1, steps + 1):
        oracle.step(1, mode=int(g["mode"]))
        of = get_flags()
        for k, nm in enumerate(flag_names):
            if not np.array_equal(of[k], flags[t - 1][k]):
                mismatched += 1
        if t % every == 0:
            ref = fields[t // every]
            for k, nm in enumerate(field_names):
                a = get_fields(nm)
                scale = max(1.0, float(np.max(np.abs(ref[k]))))
                assert np.max(np.abs(a - ref[k])) <= rtol * scale, (nm, t, np.max(np.abs(a - ref[k])))
    assert mismatched == 0, f"{mismatched} step/flag arrays differ from the reference GPU run"


def test_dendrite_dba_vs_reference_gpu():
    g = _gpu_fixture("ref_gpu_dendrite.npz")
    nx, ny = int(g["nx"]), int(g["ny"])
    o = OracleDendrite(nx, ny, 1, 4, DENDRITE_REF, libm=True)
    o.set_fields(g["fields"][0][0], g["fields"][0][1])
    def flags():
        d = o.get()
        return [d["wake_p"], d["wake_T"], d["next_p"], d["next_T"]]
    _compare_run(g, o, ["p", "T"], ["wake_p", "wake_T", "next_p", "next_T"],
                 lambda nm: o.get()[nm].reshape(ny, nx), flags, rtol=1e-9)


@pytest.mark.parametrize("name,conserved", [("ref_gpu_modelb.npz", 0), ("ref_gpu_modelb_cons.npz", 1)])
def test_modelb_dba_vs_reference_gpu(name, conserved):
    g = _gpu_fixture(name)
    nx, ny = int(g["nx"]), int(g["ny"])
    prm = dict(MODELB_REF, dt=float(g["dt"]), metric_eps=float(g["metric_eps"]))
    o = OracleModelB(nx, ny, 1, 4, prm, conserved=conserved, libm=True)
    f0 = g["fields"][0]
    o.set_fields(f0[0], f0[1], f0[2])
    _compare_run(g, o, ["x", "y", "z"], ["wake", "next"], lambda nm: o.field(nm)[0], lambda: list(o.flags()), rtol=1e-9)


@pytest.mark.parametrize("name,conserved", [("ref_gpu_kh.npz", 0), ("ref_gpu_kh_cons.npz", 1)])
def test_kh_dba_vs_reference_gpu(name, conserved):
    g = _gpu_fixture(name)
    nx, ny = int(g["nx"]), int(g["ny"])
    prm = dict(KH_REF, dt=float(g["dt"]), dx=float(g["dx"]), dy=float(g["dx"]), metric_eps=float(g["metric_eps"]))
    o = OracleKH(nx, ny, 4, prm, conserved=conserved)
    ic = g["ic"]
    o.set_primitive(ic[0], ic[1], ic[2], ic[3])
    _compare_run(g, o, ["Mass", "Momx", "Momy", "Energy"], ["wake", "next"], lambda nm: o.field(nm)[0],
                 lambda: list(o.flags()), rtol=1e-9)
