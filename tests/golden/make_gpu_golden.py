"""Generate tests/golden/ref_gpu_*.npz from the reference's own GPU DBA kernels.

Runs the checker harnesses oracle/_ref/*_gpu_steps (built here by
`make -C oracle ref` from the reference's unmodified .cu files; the binaries
travel to the B200 box) on small 2-D grids with 4x4 DBA blocks and stores, per
step, every block-flag array, plus FP64 field snapshots.  Harness launch shape
(one-warp 4x4x1 CTAs, grid sizes that keep every block index in bounds) is
described in oracle/refcheck/*.cu.

Usage (on a B200):  python tests/golden/make_gpu_golden.py <out_dir> [curand]
(`curand`: only the cuRAND initial-condition fixture, ref_gpu_modelb_curand.npz)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")

DEN_INPUT = "{nx} {ny} 1\n{steps} {steps} 0.00005\n0.02 0.02 0.02\n0.5 0.0003 0.01 0.9 40.\n0.25\n1\n0.01\n1e-5\n"
MB_INPUT = ("{nx} {ny} 1\n{steps} {steps} {dt}\n1 1 1\n0 0 0 0 0 4\n1 1 2\n1 1 2\n1 1\n4 4 4 0.01\n1 1 1 1\n"
            "0.2 0.2 0.01\n100 0.4 1\n1\n{eps}\n1\n")
KH_INPUT = "{nx} {ny} 1\n{steps} {steps} {dt}\n{dx} {dx} {dx}\n1\n{eps}\n"


def run(binary, text, steps, every, nflag, nb, nf, n, d, ic_fields=None, extra=()):
    open(f"{d}/Input.txt", "w").write(text)
    subprocess.check_call([f"{REF}/{binary}", f"{d}/Input.txt", str(steps), str(every), f"{d}/o", *extra],
                          stdout=subprocess.DEVNULL)
    flags = np.fromfile(f"{d}/o_flags.bin", dtype=np.int32).reshape(steps, nflag, nb).astype(np.uint8)
    raw = np.fromfile(f"{d}/o_fields.bin", dtype=np.float64)
    return flags, raw


def curand_fixture(out, d, nx=64, ny=64):
    """ref_gpu_modelb_curand.npz: the reference GPU program's own initial condition
    (cuRAND XORWOW, seed 1234, three uniform passes, Initialize) and 60 DBA steps
    from it, plain Model B, Metric_eps 1e-3."""
    n, nb = nx * ny, (nx // 4) * (ny // 4)
    steps, every = 60, 30
    flags, raw = run("modelb_gpu_steps", MB_INPUT.format(nx=nx, ny=ny, steps=steps, dt=0.001, eps=1e-3), steps, every,
                     2, nb, 3, n, d, extra=("curand",))
    fields = raw.reshape(-1, 3, ny, nx)
    np.savez_compressed(f"{out}/ref_gpu_modelb_curand.npz", nx=nx, ny=ny, steps=steps, every=every, mode=1,
                        dt=0.001, metric_eps=1e-3, flags=flags, fields=fields)


def main(out, only=None):
    os.makedirs(out, exist_ok=True)
    d = tempfile.mkdtemp()
    if only == "curand":
        curand_fixture(out, d)
        print("wrote ref_gpu_modelb_curand.npz")
        return
    nx = ny = 64
    n, nb = nx * ny, (nx // 4) * (ny // 4)
    # dendrite: 200 DBA steps, snapshots every 100
    steps, every = 200, 100
    flags, raw = run("dendrite_gpu_steps", DEN_INPUT.format(nx=nx, ny=ny, steps=steps), steps, every, 4, nb, 2, n, d)
    fields = raw.reshape(-1, 2, ny, nx)
    np.savez_compressed(f"{out}/ref_gpu_dendrite.npz", nx=nx, ny=ny, steps=steps, every=every, mode=1,
                        flags=flags, fields=fields)
    # Model B plain and conserved: 150 DBA steps, Metric_eps 1e-3
    steps, every = 150, 75
    for binary, name in (("modelb_gpu_steps", "ref_gpu_modelb.npz"), ("modelb_cons_gpu_steps", "ref_gpu_modelb_cons.npz")):
        flags, raw = run(binary, MB_INPUT.format(nx=nx, ny=ny, steps=steps, dt=0.001, eps=1e-3), steps, every, 2, nb, 3, n, d)
        fields = raw.reshape(-1, 3, ny, nx)
        np.savez_compressed(f"{out}/{name}", nx=nx, ny=ny, steps=steps, every=every, mode=1, dt=0.001,
                            metric_eps=1e-3, flags=flags, fields=fields)
    # KH plain and conserved: 150 DBA steps, Metric_eps 10
    steps, every = 150, 75
    for binary, name in (("kh_gpu_steps", "ref_gpu_kh.npz"), ("kh_cons_gpu_steps", "ref_gpu_kh_cons.npz")):
        flags, raw = run(binary, KH_INPUT.format(nx=nx, ny=ny, steps=steps, dt=0.0002, dx=0.002, eps=10.0),
                         steps, every, 2, nb, 4, n, d)
        ic = raw[:4 * n].reshape(4, ny, nx)
        dumps = raw[4 * n:].reshape(-1, 4, ny, nx)
        fields = np.concatenate([np.zeros((1, 4, ny, nx)), dumps])
        np.savez_compressed(f"{out}/{name}", nx=nx, ny=ny, steps=steps, every=every, mode=1, dt=0.0002, dx=0.002,
                            metric_eps=10.0, flags=flags, fields=fields, ic=ic)
    curand_fixture(out, d)
    print("wrote", sorted(os.listdir(out)))


if __name__ == "__main__":
    # python tests/golden/make_gpu_golden.py [out_dir] [curand]
    main(sys.argv[1] if len(sys.argv) > 1 else HERE, sys.argv[2] if len(sys.argv) > 2 else None)
