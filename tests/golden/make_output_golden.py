"""Generate tests/golden/ref_out_{modelb,kh}.npz: the output files of the reference's
own serial CPU programs (example_Reactive_ModelB/CPU_version/base_CPU.cpp and
example_Kelvin_Helmholtz/CPU_version/KH_CPU.cpp, unmodified, built by
`make -C oracle ref` into oracle/_ref/) on a small grid in regular mode.

Each program runs in a scratch directory on the Input.txt stored in the fixture
and writes output_<t>.vtk every t_freq steps, plus Integral.out (Model B: time,
sums of x, y, z, b) or Integral_mass.out and VY_mode.out (KH).  The fixture keeps
the Input.txt text, each VTK file's header lines and sections as parsed numbers,
and the .out tables.  RTValues.out (wall-clock steps per second) is not kept.

Usage (here, where the reference programs are built):  python tests/golden/make_output_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
from vtk_text import read_table, read_vtk  # noqa: E402

# regular mode (the CPU programs have no DBA); the reference's own parameters
MODELB_INPUT = ("64 64 1\n20 10 0.001\n1 1 1\n0 0 0 0 0 4\n1 1 2\n1 1 2\n1 1\n4 4 4 0.01\n1 1 1 1\n"
                "0.2 0.2 0.01\n100 0.4 1\n1\n1e-6\n0\n")
KH_INPUT = "64 64 1\n20 10 0.0002\n0.002 0.002 0.002\n0\n0\n"


def run(binary, text, outs):
    d = tempfile.mkdtemp()
    with open(os.path.join(d, "Input.txt"), "w") as f:
        f.write(text)
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", binary)], cwd=d, check=True, stdout=subprocess.DEVNULL)
    fix = {"input": np.array(text)}
    for t in (0, 10, 20):
        header, sec = read_vtk(os.path.join(d, f"output_{t}.vtk"))
        fix[f"vtk{t}_header"] = np.array("\n".join(header))
        fix[f"vtk{t}_sections"] = np.array(" ".join(sec))
        for name, v in sec.items():
            fix[f"vtk{t}_{name}"] = v
    for name in outs:
        fix["out_" + name.replace(".", "_")] = read_table(os.path.join(d, name))
    return fix


def main(out=HERE):
    np.savez_compressed(os.path.join(out, "ref_out_modelb.npz"), **run("modelb_cpu", MODELB_INPUT, ["Integral.out"]))
    np.savez_compressed(os.path.join(out, "ref_out_kh.npz"),
                        **run("kh_cpu", KH_INPUT, ["Integral_mass.out", "VY_mode.out"]))
    print("wrote ref_out_modelb.npz, ref_out_kh.npz")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
