"""Text restart files of tri_hp (tri_hp::output text branch, tri_hp/output.cpp:147-181;
tri_hp::input text branch, output.cpp:1384-1474).

Layout: a header of 'p0 = P', 'npnt = N, nseg = S, ntri = T' and 'END OF HEADER', then
one line per vertex (NV values), per (side, side mode) and per (triangle, interior mode),
values in C++ scientific notation with 8 digits after the point, tab-terminated. Reading
a file written at another p keeps the modes both degrees share and zeroes the rest, as
the reference's input does: side modes 0 .. min(p, p_file) - 2; interior modes by their
(row m, column k) position, rows m = 1 .. p - 2 holding p - 1 - m modes each."""
import re

import numpy as np


def write_text(path, p, ugv, ugs, ugi):
    """Writes the state (vertices [npnt][NV], sides [nseg][p-1][NV], interiors
    [ntri][(p-1)(p-2)/2][NV]) in the reference's text restart layout."""
    ugv, ugs, ugi = (np.asarray(a, dtype=np.float64) for a in (ugv, ugs, ugi))
    npnt, NV = ugv.shape
    with open(path, "w") as f:
        f.write(f"p0 = {p}\n")
        f.write(f"npnt = {npnt}, nseg = {ugs.shape[0]}, ntri = {ugi.shape[0]}\n")
        f.write("END OF HEADER\n")
        for rows in (ugv, ugs.reshape(-1, NV), ugi.reshape(-1, NV)):
            for r in rows:
                f.write("".join(f"{x:.8e}\t" for x in r) + "\n")


def _interior_rows(p):
    """(m, k) of the interior modes of degree p in storage order."""
    return [(m, k) for m in range(1, p - 1) for k in range(0, p - 1 - m)]


def read_text(path, p, npnt, nseg, ntri, NV):
    """Reads a text restart written at any degree into arrays at degree p."""
    with open(path) as f:
        text = f.read()
    head, _, body = text.partition("END OF HEADER")
    pin = int(re.search(r"=\s*(\d+)", head).group(1))
    vals = np.array(body.split(), dtype=np.float64)
    smi, smo = pin - 1, p - 1
    imi, imo = (pin - 1) * (pin - 2) // 2, (p - 1) * (p - 2) // 2
    need = NV * (npnt + nseg * smi + ntri * imi)
    if vals.size < need:
        raise ValueError(f"{path}: {vals.size} values, {need} expected for p = {pin}")
    k = 0
    ugv = vals[k:k + npnt * NV].reshape(npnt, NV).copy()
    k += npnt * NV
    sides = vals[k:k + nseg * smi * NV].reshape(nseg, smi, NV)
    k += nseg * smi * NV
    ints = vals[k:k + ntri * imi * NV].reshape(ntri, imi, NV)
    ugs = np.zeros((nseg, smo, NV))
    keep = min(smi, smo)
    ugs[:, :keep] = sides[:, :keep]
    ugi = np.zeros((ntri, imo, NV))
    src = {mk: j for j, mk in enumerate(_interior_rows(pin))}
    for j, mk in enumerate(_interior_rows(p)):
        if mk in src:
            ugi[:, j] = ints[:, src[mk]]
    return ugv, ugs, ugi
