"""Reader for the legacy ASCII VTK files the reference programs write (test helper).

The reference's writers (e.g. example_Reactive_ModelB/CPU_version/base_CPU.cpp:346-455,
example_Kelvin_Helmholtz/CPU_version/KH_CPU.cpp:560-630) print a RECTILINEAR_GRID
header, integer coordinates, then POINT_DATA sections `SCALARS <name> double` +
`LOOKUP_TABLE default` + one value per cell, or `VECTORS <name> double` + three
values per cell, with std::ostream's default 6 significant digits.
"""
import numpy as np


def read_vtk(path_or_text):
    """(header lines up to POINT_DATA, {section name: float64 array}) of one file."""
    text = path_or_text
    if "\n" not in str(path_or_text):
        with open(path_or_text) as f:
            text = f.read()
    lines = text.splitlines()
    header = []
    i = 0
    while i < len(lines) and not lines[i].startswith("POINT_DATA"):
        header.append(lines[i].rstrip())
        i += 1
    npts = int(lines[i].split()[1])
    toks = " ".join(lines[i + 1:]).split()
    out = {}
    j = 0
    while j < len(toks):
        kind, name = toks[j], toks[j + 1]
        j += 3                                   # kind, name, type
        if kind == "SCALARS":
            if toks[j] == "LOOKUP_TABLE":
                j += 2
            cnt = npts
        elif kind == "VECTORS":
            cnt = 3 * npts
        else:
            raise ValueError(f"unexpected token {kind!r}")
        out[name] = np.array([float(t) for t in toks[j:j + cnt]])
        j += cnt
    return header, out


def compare_vtk(a, b):
    """Compare_VTK's measures (example_Dendritic_growth/Compare_VTK.cpp:57-73): the
    total absolute difference of two value streams and its average per value; plus
    the total over the reference's L1 norm (the relative form the tests bound)."""
    d = float(np.sum(np.abs(a - b)))
    den = float(np.sum(np.abs(b)))
    return {"total": d, "average": d / max(1, a.size), "relative": d / (den if den > 0 else 1.0)}


def read_table(path):
    """Whitespace-separated numeric rows (the .out files); a text header row is skipped."""
    rows = []
    with open(path) as f:
        for ln in f:
            parts = ln.split()
            if not parts:
                continue
            try:
                rows.append([float(p) for p in parts])
            except ValueError:
                continue
    return np.array(rows)
