"""Generate tests/golden/ref_cpu_*.npz from the reference's own serial CPU code.

Runs the checker harnesses oracle/_ref/modelb_cpu_steps and oracle/_ref/kh_cpu_steps
(built by `make -C oracle ref` from the reference sources, which must be present)
on small grids and stores their FP64 fields.  The CPU restatement (oracle/) must
reproduce these bit for bit in its glibc-math flavour.

Usage: python tests/golden/make_cpu_golden.py
"""
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")

MODELB_INPUT = """{nx} {ny} 1
10 5 {dt}
1 1 1
0 0 0 0 0 4
1 1 2
1 1 2
1 1
4 4 4 0.01
1 1 1 1
0.2 0.2 0.01
100 0.4 1
1
1e-6
0
"""
KH_INPUT = """{nx} {ny} 1
10 5 {dt}
{dx} {dx} {dx}
0
0
"""


def main():
    d = tempfile.mkdtemp()
    cases = {}
    # Model B: 32x24, dt 0.001, 7 steps from mt19937_64(1234)
    open(f"{d}/Input.txt", "w").write(MODELB_INPUT.format(nx=32, ny=24, dt=0.001))
    subprocess.check_call([f"{REF}/modelb_cpu_steps", f"{d}/Input.txt", "7", f"{d}/mb.bin"], stdout=subprocess.DEVNULL)
    a = np.fromfile(f"{d}/mb.bin").reshape(7, 24, 32)
    np.savez_compressed(os.path.join(HERE, "ref_cpu_modelb.npz"), nx=32, ny=24, dt=0.001, steps=7,
                        x=a[0], y=a[1], z=a[2], b=a[3], mu_x=a[4], mu_y=a[5], mu_z=a[6])
    # KH: 64x48, dt 2e-4, dx 2e-3, 9 steps from the smooth interface
    open(f"{d}/Input.txt", "w").write(KH_INPUT.format(nx=64, ny=48, dt=0.0002, dx=0.002))
    subprocess.check_call([f"{REF}/kh_cpu_steps", f"{d}/Input.txt", "9", f"{d}/kh.bin"], stdout=subprocess.DEVNULL)
    a = np.fromfile(f"{d}/kh.bin").reshape(8, 48, 64)
    np.savez_compressed(os.path.join(HERE, "ref_cpu_kh.npz"), nx=64, ny=48, dt=0.0002, dx=0.002, steps=9,
                        Mass=a[0], Momx=a[1], Momy=a[2], Energy=a[3], rho=a[4], p=a[5], vx=a[6], vy=a[7])
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
