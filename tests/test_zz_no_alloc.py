"""dba_mean_change_noalloc: the allocation-free entry point.

Some callers cannot call cudaMalloc (work enqueued during CUDA-graph capture,
latency-critical loops that must not take an allocation's implicit device
synchronisation, hosts whose device memory belongs to another allocator).
This entry point computes the conserved-DBA mean change with its scratch in a
fixed array inside the library.  The test takes the per-block change sums and
the mean change that the existing entry point (dba_step, conserved FP64 Model B)
produced, feeds the same sums to the new entry point twice in a row, and checks
both results against the existing one (same fixed-order reduction, so the
tolerance used elsewhere for FP64 -- bit equality -- applies).  This file is
collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import dba_b200
from cases import MODELB_REF, modelb_cfg

pytestmark = pytest.mark.gpu


def _engine_sums_and_mean(sim, n, nb):
    """Per-block sums and mean change of the last conserved step, from the in-memory
    checkpoint.  Layout: step (8 B), time (8 B), then the context's device allocations
    in creation order, without the readback staging buffer.  For FP64 Model B:
    x,y,z x 2 buffers, 3 potentials, parity [2][nb], wake [3][nb], next [nb],
    block sums [3][nb] (FP64), run sums [3][ceil(nb/1024)], means [4] (FP64),
    ticket, status, striped activity counters [32 stripes x 16] (uint64)."""
    blob = np.empty(sim.state_size(), np.uint8)
    sim.save_state(blob)
    J = (nb + 1023) // 1024
    sizes = [8, 8] + [n * 8] * 6 + [n * 8] * 3 + [2 * nb, 3 * nb, nb, 3 * nb * 8, 3 * J * 8, 4 * 8, 4, 4, 32 * 16 * 8]
    assert sum(sizes) == blob.size, "checkpoint layout changed; update this test"
    off = np.cumsum([0] + sizes)
    bsum = blob[off[14]:off[15]].view(np.float64).copy()
    mean = blob[off[16]:off[17]].view(np.float64)[:3].copy()
    return bsum, mean


def test_mean_change_noalloc_matches_dba_step():
    import torch

    L = dba_b200.load_library()
    f = L.dba_mean_change_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]

    nx = ny = 64
    B = 4
    nb = (nx // B) * (ny // B)
    sim = dba_b200.Simulation(modelb_cfg(dict(MODELB_REF, metric_eps=1e-3), nx, ny, 1, B, conserved=1)).init()
    sim.step(7, 1)
    sim.sync()
    bsum, mean_ref = _engine_sums_and_mean(sim, nx * ny, nb)
    assert np.any(bsum != 0.0)

    dev_sums = torch.from_numpy(bsum).cuda()
    stream = torch.cuda.current_stream()
    for _ in range(2):                       # two calls in a row share the scratch
        out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
        st = f(dev_sums.data_ptr(), nb, 3, float(nx * ny), out.data_ptr(), stream.cuda_stream)
        assert st == 0, dba_b200.engine.DBA_ERR.get(st)
        stream.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got, mean_ref), (got, mean_ref)


def test_mean_change_noalloc_rejects_oversize():
    L = dba_b200.load_library()
    f = L.dba_mean_change_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    assert f(dummy, (1 << 20) + 1, 3, 1.0, dummy, None) == 8      # DBA_ERR_ARG: beyond the fixed scratch
    assert f(dummy, 16, 5, 1.0, dummy, None) == 8
