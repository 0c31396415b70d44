"""3D (tet_hp) path: tet_basis tables (hp_tet_basis_build) and their dense
operators (include/hp_tet.h)."""
import ctypes

import numpy as np

from . import _lib as L

MAXP, MAXG, MAXT, MAXQ, MAXM = 4, 5, 35, 125, 12
_D, _I = ctypes.c_double, ctypes.c_int


class TetTables(ctypes.Structure):
    _fields_ = ([(n, _I) for n in ("p", "G", "T", "em", "fm", "im", "bm", "nmodx", "nmody", "nmodz")] +
                [(n, _D * MAXM * MAXG) for n in ("gx", "dgx", "gy", "dgy", "gz", "dgz")] +
                [(n, _D * MAXG) for n in ("wtx", "wty", "wtz", "xp", "yp", "zp", "x0", "y0", "y1", "z0",
                                          "dltx", "dlty", "dltz")] +
                [(n, _D * MAXG * MAXG) for n in ("dltx2", "dltx3", "dlty2", "dlty3", "dltz2")] +
                [(n, _I * MAXT) for n in ("mx", "my", "mz")] + [("msg", _D * MAXT), ("w", _D * MAXQ)] +
                [(n, _D * MAXT * MAXQ) for n in ("F", "DX", "DY", "DZ")] +
                [(n, _D * MAXG * MAXG) for n in ("Ax", "Bx", "Ay", "By", "Az")])


def tables(p):
    """hp_tet_basis_build(p) as a TetTables structure."""
    lib = L.lib()
    lib.hp_tet_basis_build.argtypes = [_I, ctypes.POINTER(TetTables)]
    t = TetTables()
    rc = lib.hp_tet_basis_build(p, ctypes.byref(t))
    if rc != 0:
        raise ValueError(f"tet basis p={p} unsupported")
    return t


def arr(t, name):
    """A numpy copy of one table, cut to its used extent."""
    G, T = t.G, t.T
    a = np.ctypeslib.as_array(getattr(t, name)).copy()
    cols = {"gx": t.nmodx, "dgx": t.nmodx, "gy": t.nmody, "dgy": t.nmody, "gz": t.nmodz, "dgz": t.nmodz}
    if name in cols:
        return a[:G, :cols[name]]
    if name in ("F", "DX", "DY", "DZ"):
        return a[:G ** 3, :T]
    if name == "w":
        return a[:G ** 3]
    if name in ("mx", "my", "mz", "msg"):
        return a[:T]
    if a.ndim == 2:
        return a[:G, :G]
    return a[:G]


def deriv(t, direction, f):
    """derivr / derivs / derivt of point values f[G,G,G] (returned, not added)."""
    G = t.G
    f = np.asarray(f).reshape(G, G, G)
    y0 = arr(t, "y0")[None, :, None]
    z0 = arr(t, "z0")[None, None, :]
    ax = lambda A: np.einsum("in,njk->ijk", A, f)
    ay = lambda A: np.einsum("jn,ink->ijk", A, f)
    az = lambda A: np.einsum("kn,ijn->ijk", A, f)
    if direction == 0:
        return (y0 * z0 * ax(arr(t, "Ax"))).ravel()
    if direction == 1:
        return (y0 * z0 * ax(arr(t, "Bx")) + z0 * ay(arr(t, "Ay"))).ravel()
    return (y0 * z0 * ax(arr(t, "Bx")) + z0 * ay(arr(t, "By")) + az(arr(t, "Az"))).ravel()
