"""The C ABI without a GPU: the library loads, exports every function the
headers in include/ declare, its struct layouts match the Python binding, the
Input.txt parser reads the reference grammars, and context creation fails with
a status code (not a crash) when no CUDA device is present."""
import ctypes
import glob
import os
import re

import pytest

import dba_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(dba_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    L = dba_b200.load_library()
    names = declared_functions()
    assert len(names) >= 20, names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_sizes_match_binding():
    L = dba_b200.load_library()
    from dba_b200.engine import Info, Obs, Prof
    assert L.dba_struct_size(0) == ctypes.sizeof(dba_b200.Config)
    assert L.dba_struct_size(1) == ctypes.sizeof(Obs)
    assert L.dba_struct_size(2) == ctypes.sizeof(Info)
    assert L.dba_struct_size(3) == ctypes.sizeof(Prof)


def test_strerror_codes():
    L = dba_b200.load_library()
    assert L.dba_strerror(0) == b"ok"
    assert b"non-finite" in L.dba_strerror(5)
    assert L.dba_strerror(99) == b"unknown status"


DENDRITE_TXT = """128 96 1                  Nx, Ny, Nz

300 100 0.00005			 t_total, t_freq, dt

0.02 0.02 0.02				 dx, dy, dz

0.05 0.0003 0.01 0.9 40.      delta, tau, epsilon, alpha, gamma

0.55						 Delta

1							 Mode

0.001                        Metric_p

1e-5 Metric_T
block = 8
precision = fp32
bc = zeroflux
ic = tanh
"""

MODELB_TXT = """64 64 1
1000 100 0.001 # dt note
1 1 1
0 0 0 0 0 3
1 1 2
1 1 2
1 1
1 1 1 0.01
1 1 1 1
0.05 0.05 0.45
100 0.4 1
0.0001
1e-3 Metric_eps
1
conserved = 1
seed = 77
"""

KH_TXT = """256 128 1
500 100 0.0002
0.002 0.002 0.002
0
10 Metric_eps
"""


def test_parse_reference_grammars(tmp_path):
    p = tmp_path / "Input.txt"
    p.write_text(DENDRITE_TXT)
    c = dba_b200.parse_input(p, "dendrite")
    assert (c.nx, c.ny, c.nz, c.t_total, c.t_freq) == (128, 96, 1, 300, 100)
    assert (c.delta, c.tau, c.epsilon, c.alpha, c.gamma, c.Delta) == (0.05, 0.0003, 0.01, 0.9, 40.0, 0.55)
    assert (c.mode, c.metric_p, c.metric_T) == (1, 0.001, 1e-5)
    assert (c.block, c.precision, c.bc, c.ic) == (8, 1, 1, 1)
    p.write_text(MODELB_TXT)
    c = dba_b200.parse_input(p, "modelb")
    assert (c.nx, c.dt, c.chi_zb, c.vz, c.rz, c.eps_phi, c.x0, c.z0, c.K, c.k_0, c.metric_eps, c.mode) == \
        (64, 0.001, 3.0, 2, 2, 0.01, 0.05, 0.45, 100.0, 0.0001, 1e-3, 1)
    assert (c.conserved, c.seed) == (1, 77)
    p.write_text(KH_TXT)
    c = dba_b200.parse_input(p, "kh")
    assert (c.nx, c.ny, c.dt, c.dx, c.mode, c.metric_eps) == (256, 128, 0.0002, 0.002, 0, 10.0)
    assert abs(c.kh_gamma - 5.0 / 3.0) < 1e-15


def test_parse_missing_file_is_io_error(tmp_path):
    with pytest.raises(dba_b200.DBAError) as e:
        dba_b200.parse_input(tmp_path / "nope.txt", "kh")
    assert e.value.code == 4


def test_create_rejects_bad_config():
    L = dba_b200.load_library()
    c = dba_b200.config("modelb", nx=30, ny=32, nz=1, block=4)     # 30 not a multiple of 4
    h = ctypes.c_void_p()
    assert L.dba_create(ctypes.byref(c), ctypes.byref(h)) == 1
    c = dba_b200.config("kh", nx=64, ny=64, nz=8, block=8)         # KH is 2-D
    assert L.dba_create(ctypes.byref(c), ctypes.byref(h)) == 1


def test_create_without_gpu_returns_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = dba_b200.load_library()
    c = dba_b200.config("dendrite", nx=64, ny=64, nz=1, block=4)
    h = ctypes.c_void_p()
    assert L.dba_create(ctypes.byref(c), ctypes.byref(h)) == 2      # DBA_ERR_CUDA, no crash
