"""Generate tests/golden/ref_post.npz: outputs of the reference's own analysis tools
(example_Dendritic_growth/Extract_Tip.cpp and example_Reactive_ModelB/coarsening_analysis.cpp,
unmodified, built by `make -C oracle ref` into oracle/_ref/) on fields whose values
are exact binary fractions, so the tools' threshold tests are unambiguous.

* Extract_Tip reads, after its fixed header skip (4 lines, the DIMENSIONS line, 6
  more lines), one value per cell in x-fastest order: the STRUCTURED_POINTS layout
  (DIMENSIONS, ORIGIN, SPACING, POINT_DATA, SCALARS, LOOKUP_TABLE).  (Given the
  reference's RECTILINEAR_GRID files it would read the z-coordinate row as data.)
  The field is 64^3: a solid region x < tip(y, z) with the profile varying in z,
  values 0.875 inside, 0.125 outside, 0.5 on a shell (not above the 0.5 threshold).
* coarsening_analysis has its grid hard-coded to 256^3 and reads the 21st line of
  output_0.vtk (the Z field of the reference's Model B writer, one line per field):
  the field is 0.875 inside seeded periodic spheres, 0.0625 elsewhere.  The
  spheres are stored; the tests rebuild the field from them.

Usage (here, where the tools are built):  python tests/golden/make_post_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")


def tip_field(n=64):
    """(nz, ny, nx) field with a z-dependent solid front along x."""
    z, y, x = np.mgrid[0:n, 0:n, 0:n]
    front = 20 + ((z * 7 + y * 3) % 13) - np.abs(z - n // 2) // 3
    f = np.where(x < front, 0.875, 0.125)
    f = np.where(x == front, 0.5, f)
    return f.astype(np.float64)


def spheres(seed=3, count=60, n=256):
    rng = np.random.default_rng(seed)
    c = rng.integers(0, n, size=(count, 3))
    r = rng.integers(2, 7, size=count)
    return np.concatenate([c, r[:, None]], axis=1).astype(np.int64)


def sphere_field(sph, n=256):
    """(nz, ny, nx) field: 0.875 inside the periodic spheres (cx, cy, cz, r), else 0.0625."""
    f = np.full((n, n, n), 0.0625)
    ax = np.arange(n)
    for cx, cy, cz, r in sph:
        dz = np.minimum(np.abs(ax - cz), n - np.abs(ax - cz))[:, None, None]
        dy = np.minimum(np.abs(ax - cy), n - np.abs(ax - cy))[None, :, None]
        dx = np.minimum(np.abs(ax - cx), n - np.abs(ax - cx))[None, None, :]
        f[dx * dx + dy * dy + dz * dz <= r * r] = 0.875
    return f


def write_structured_points(path, f):
    nz, ny, nx = f.shape
    with open(path, "w") as o:
        o.write("# vtk DataFile Version 2.0\nphi\nASCII\nDATASET STRUCTURED_POINTS\n")
        o.write(f"DIMENSIONS {nx} {ny} {nz}\nORIGIN 0 0 0\nSPACING 1 1 1\nPOINT_DATA {f.size}\n")
        o.write("SCALARS phi double\nLOOKUP_TABLE default\n")
        o.write(" ".join(repr(float(v)) for v in f.ravel()) + "\n")


def write_modelb_z(path, z):
    """The reference Model B writer's layout up to the Z field (its 21st line)."""
    nz, ny, nx = z.shape
    with open(path, "w") as o:
        o.write("# vtk DataFile Version 2.0\nOUTPUT\nASCII\nDATASET RECTILINEAR_GRID\n")
        o.write(f"DIMENSIONS {nx} {ny} {nz}\n")
        for nm, n in (("X", nx), ("Y", ny), ("Z", nz)):
            o.write(f"{nm}_COORDINATES {n} int\n" + "\t".join(str(i) for i in range(n)) + "\t\n")
        o.write(f"POINT_DATA {z.size}\nSCALARS X double\nLOOKUP_TABLE default\n0\n")
        o.write("SCALARS Y double\nLOOKUP_TABLE default\n0\nSCALARS Z double\nLOOKUP_TABLE default\n")
        vals = np.where(z.ravel() > 0.5, "0.875", "0.0625")
        o.write(" ".join(vals.tolist()) + " \n")


def main(out=HERE):
    d = tempfile.mkdtemp()
    tf = tip_field()
    write_structured_points(os.path.join(d, "tip.vtk"), tf)
    subprocess.run([os.path.join(REF, "extract_tip"), "tip.vtk"], cwd=d, check=True, stdout=subprocess.DEVNULL)
    rows = [ln.split() for ln in open(os.path.join(d, "Tip_Profile.dat")).read().splitlines()[1:]]
    tip_profile = np.array([[int(a) for a in r] for r in rows], dtype=np.int64)   # k, tip_x_max - tip_x[k]

    sph = spheres()
    write_modelb_z(os.path.join(d, "output_0.vtk"), sphere_field(sph))
    subprocess.run([os.path.join(REF, "coarsening_analysis")], cwd=d, check=True, stdout=subprocess.DEVNULL)
    sizes = np.array([int(a) for a in open(os.path.join(d, "size_dist.txt")).readline().split()], dtype=np.int64)
    radius = float(open(os.path.join(d, "avg_radius.txt")).readline().strip().split(",")[1])
    np.savez_compressed(os.path.join(out, "ref_post.npz"), tip_profile=tip_profile, spheres=sph, sizes=sizes,
                        avg_radius=radius)
    print("wrote ref_post.npz:", len(sizes), "islands, R_avg", radius)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
