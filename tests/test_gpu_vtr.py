"""VTK XML RectilinearGrid output (dba_write_vtr): ASCII and appended-binary files,
y-slab pieces with a .pvtr index, and background writing -- parsed back here and
compared with the fields and flags read through the library."""
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import dba_b200
from cases import DENDRITE_REF, MODELB_REF, dendrite_cfg, modelb_cfg

pytestmark = pytest.mark.gpu


def read_vtr(path):
    """{name: array} of a .vtr written with format="ascii" or "appended" (raw, UInt64 headers)."""
    raw = open(path, "rb").read()
    cut = raw.find(b"<AppendedData")
    head = raw if cut < 0 else raw[:cut] + b"</VTKFile>"
    root = ET.fromstring(head.decode())
    piece = root.find("RectilinearGrid/Piece")
    ext = [int(v) for v in piece.get("Extent").split()]
    shape = (ext[5] - ext[4] + 1, ext[3] - ext[2] + 1, ext[1] - ext[0] + 1)
    data0 = None if cut < 0 else raw.index(b"_", cut) + 1
    out = {}
    for arr in piece.iter("DataArray"):
        dt = {"Float32": np.float32, "Int8": np.int8}[arr.get("type")]
        if arr.get("format") == "ascii":
            v = np.array(arr.text.split(), dtype=np.float64).astype(dt)
        else:
            o = data0 + int(arr.get("offset"))
            nbytes = int(np.frombuffer(raw[o:o + 8], np.uint64)[0])
            v = np.frombuffer(raw[o + 8:o + 8 + nbytes], dt)
        out[arr.get("Name")] = v
    return out, shape, ext


def _sim():
    prm = dict(DENDRITE_REF, Delta=1.15, delta=0.2, metric_p=1e-3, metric_T=1e-5)
    s = dba_b200.Simulation(dendrite_cfg(prm, 40, 24, 16, 8, precision=1, bc=1, ic=1, ic_radius=5.0,
                                         ic_width=2.0)).init()
    s.step(150, 1)
    return s


def _cell_flags(s, which):
    f = s.flags(which).reshape(s.info.nbz, s.info.nby, s.info.nbx)
    B = s.cfg.block
    return np.repeat(np.repeat(np.repeat(f, B, 0), B, 1), B, 2) != 0


@pytest.mark.parametrize("binary", [True, False])
def test_vtr_single_piece(tmp_path, binary):
    s = _sim()
    s.write_vtr(tmp_path / "out", binary=binary)
    d, shape, _ = read_vtr(tmp_path / "out.vtr")
    assert shape == (16, 24, 40)
    if binary:
        assert np.array_equal(d["phi"].reshape(shape), s.field("p").astype(np.float32))
        assert np.array_equal(d["T"].reshape(shape), s.field("T").astype(np.float32))
    else:   # ostream default precision 6, as the reference's ASCII writer
        assert np.allclose(d["phi"].reshape(shape), s.field("p"), rtol=1e-5, atol=1e-6)
    assert np.array_equal(d["active_phi"].reshape(shape) != 0, _cell_flags(s, 0))
    assert np.array_equal(d["active_T"].reshape(shape) != 0, _cell_flags(s, 2))
    assert np.array_equal(d["Array y"], np.arange(24, dtype=np.float32))


def test_vtr_pieces_and_index(tmp_path):
    s = _sim()
    s.write_vtr(tmp_path / "out", pieces=3, binary=True, background=True)
    s.step(10, 1)                       # the GPU keeps going while the files are written
    s.wait_io()
    idx = ET.parse(tmp_path / "out.pvtr").getroot()
    srcs = [p.get("Source") for p in idx.iter("Piece")]
    assert srcs == ["out_0.vtr", "out_1.vtr", "out_2.vtr"]
    whole = np.zeros((16, 24, 40), np.float32)
    rows = set()
    for src in srcs:
        d, shape, ext = read_vtr(tmp_path / src)
        whole[:, ext[2]:ext[3] + 1, :] = d["T"].reshape(shape)
        rows |= set(range(ext[2], ext[3] + 1))
    assert rows == set(range(24))
    s2 = _sim()                          # the same state as at the write
    assert np.array_equal(whole, s2.field("T").astype(np.float32))


def test_vtr_modelb_fields(tmp_path):
    s = dba_b200.Simulation(modelb_cfg(dict(MODELB_REF, metric_eps=1e-3), 32, 32, 1, 8, precision=0)).init()
    s.step(20, 1)
    s.write_vtr(tmp_path / "mb")
    d, shape, _ = read_vtr(tmp_path / "mb.vtr")
    for name, f in (("X", "x"), ("Y", "y"), ("Z", "z"), ("B", "b")):
        assert np.array_equal(d[name].reshape(shape), s.field(f).astype(np.float32)), name
