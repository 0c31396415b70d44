"""ctypes binding of the shipped C-ABI (include/hp_gpu.h, include/hp_host.h).

The library is lib/libhp_b200.so next to this package. Loading fails loudly when
it is missing: there is no CPU fallback for any call.
"""
import ctypes
import os

HP_MAXP = 8
HP_MXGP = HP_MAXP + 1
HP_MXX = HP_MAXP + 2
HP_MXTM = (HP_MAXP + 1) * (HP_MAXP + 2) // 2
HP_MXBM = 3 * HP_MAXP
HP_MXSM = HP_MAXP - 1
HP_MXIM = (HP_MAXP - 1) * (HP_MAXP - 2) // 2

HP_PHYS_CD = 0
HP_PHYS_INS = 1

HP_BC_FLUX_NONE = 0
HP_BC_FLUX_INS_GENERIC = 1 << 8

HP_FIELD_CONST = 0
HP_FIELD_KOVASZNAY = 1
HP_FIELD_SINSIN = 2
HP_FIELD_QUADX = 3
HP_FIELD_LID = 4
HP_FIELD_CYLINDER = 5

_D = ctypes.c_double
_I = ctypes.c_int


def _arr(*shape):
    t = _D
    for d in reversed(shape):
        t = t * d
    return t


class BasisTables(ctypes.Structure):
    """hp_basis_tables: the tables of tri_basis<p,0> (tri_basis/tri_basis.h:218-291)."""

    _fields_ = [(n, _I) for n in ("p", "sm", "im", "tm", "bm", "nmodx", "gpx", "gpn", "ibwth", "sbwth")] + [
        ("gx", _arr(HP_MXGP, HP_MXX)), ("dgx", _arr(HP_MXGP, HP_MXX)),
        ("wtx", _arr(HP_MXGP)), ("xp", _arr(HP_MXGP)), ("x0", _arr(HP_MXGP)),
        ("gxwtx", _arr(HP_MXX, HP_MXGP)), ("dgxwtx", _arr(HP_MXX, HP_MXGP)),
        ("dltx", _arr(HP_MXGP)), ("dltx1", _arr(HP_MXGP, HP_MXGP)),
        ("gn", _arr(HP_MXGP, HP_MXTM)), ("dgn", _arr(HP_MXGP, HP_MXTM)),
        ("wtn", _arr(HP_MXGP)), ("np", _arr(HP_MXGP)), ("n0", _arr(HP_MXGP)),
        ("gnwtn", _arr(HP_MXTM, HP_MXGP)), ("gnwtnn0", _arr(HP_MXTM, HP_MXGP)), ("dgnwtn", _arr(HP_MXTM, HP_MXGP)),
        ("dltn", _arr(HP_MXGP)), ("dltn1", _arr(HP_MXGP, HP_MXGP)), ("dltn2", _arr(HP_MXGP, HP_MXGP)),
        ("norm", _arr(HP_MXTM)),
        ("sfmv", _arr(2, HP_MXSM)), ("ifmb", _arr(HP_MXBM, HP_MXIM)), ("vdiag", _D), ("vfms", _arr(3, HP_MXSM)),
        ("sdiag", _arr(HP_MXSM)), ("sfms", _arr(HP_MXSM, HP_MXSM, 3)), ("bfmi", _arr(HP_MXBM, HP_MXIM)),
        ("idiag", _arr(HP_MXIM, 2)),
        ("sfmv1d", _arr(2, HP_MXSM)), ("vdiag1d", _D), ("vfms1d", _arr(2, HP_MXSM)), ("sdiag1d", _arr(HP_MXSM, 3)),
    ]


class MeshDesc(ctypes.Structure):
    _fields_ = [
        ("npnt", _I), ("nseg", _I), ("ntri", _I),
        ("pnts", ctypes.POINTER(_D)),
        ("seg_pnt", ctypes.POINTER(_I)), ("seg_tri", ctypes.POINTER(_I)),
        ("tri_pnt", ctypes.POINTER(_I)), ("tri_seg", ctypes.POINTER(_I)), ("tri_sgn", ctypes.POINTER(_I)),
        ("nbseg", _I), ("bseg", ctypes.POINTER(_I)), ("bseg_kind", ctypes.POINTER(_I)),
        ("bseg_pibc", ctypes.POINTER(_D)), ("bseg_crd", ctypes.POINTER(_D)),
    ]


class PhysParams(ctypes.Structure):
    _fields_ = [
        ("physics", _I), ("nstage", _I), ("alpha", _D * 8), ("beta", _D * 8),
        ("cfl", _D), ("bd0", _D), ("adis", _D), ("rho", _D), ("mu", _D),
        ("rhocv", _D), ("kcond", _D), ("ax", _D), ("ay", _D), ("src", _D),
    ]


class Field(ctypes.Structure):
    _fields_ = [("kind", _I), ("prm", _D * 4)]


_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libhp_b200.so")
_lib = None


def lib():
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C hp-multiphysics_b200` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.hp_basis_build.argtypes = [_I, ctypes.POINTER(BasisTables)]
        L.hp_gpu_create.argtypes = [ctypes.POINTER(MeshDesc), ctypes.POINTER(BasisTables), ctypes.POINTER(PhysParams),
                                    _I, P, ctypes.POINTER(P)]
        for name in ("hp_gpu_destroy", "hp_gpu_setup_preconditioner", "hp_gpu_minvrt", "hp_gpu_update", "hp_gpu_sync"):
            getattr(L, name).argtypes = [P]
        L.hp_gpu_rsdl.argtypes = [P, _I, _I]
        L.hp_gpu_l2error.argtypes = [P, P, P, P]
        L.hp_gpu_enqueue_rsdl.argtypes = [P, _I]
        L.hp_gpu_enqueue_update.argtypes = [P]
        L.hp_gpu_enqueue_element_rsdl.argtypes = [P, _I]
        L.hp_gpu_set_element_matrices.argtypes = [P, _I]
        L.hp_gpu_autotune.argtypes = [P, _I]
        L.hp_gpu_get_tuning.argtypes = [P, P, P]
        L.hp_gpu_sizes.argtypes = [P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]
        for name in ("hp_gpu_upload_state", "hp_gpu_enqueue_upload_state", "hp_gpu_enqueue_download_residual"):
            getattr(L, name).argtypes = [P, P, P, P]
        for name in ("hp_gpu_download_state", "hp_gpu_download_residual"):
            getattr(L, name).argtypes = [P, P, P, P]
        L.hp_gpu_download_prcn.argtypes = [P, P, P, P, P]
        L.hp_gpu_device_ptrs.argtypes = [P] + [ctypes.POINTER(P)] * 6
        L.hp_gpu_iterate.argtypes = [P, _I, _I, P]
        L.hp_gpu_maxres.argtypes = [P, P, P]
        L.hp_gpu_resnorm.argtypes = [P, P, P]
        L.hp_gpu_fp32_updates.argtypes = [P, _I]
        L.hp_gpu_solve.argtypes = [P, _I, _D, _I, _I, _I, _I, P, _I, ctypes.POINTER(_I), ctypes.POINTER(_D),
                                   ctypes.POINTER(_I)]
        L.hp_gpu_last_error.restype = ctypes.c_char_p
        L.hp_field_eval.argtypes = [ctypes.POINTER(Field), _I, _D, _D, P]
        L.hp_tobasis.argtypes = [ctypes.POINTER(BasisTables), ctypes.POINTER(MeshDesc), _I, ctypes.POINTER(Field),
                                 P, P, P]
        L.hp_curved_side_modes.argtypes = [ctypes.POINTER(BasisTables), _I, P, P, P]
        L.hp_setvalues.argtypes = [ctypes.POINTER(BasisTables), ctypes.POINTER(MeshDesc), _I, ctypes.POINTER(Field),
                                   P, P]
        L.hp_l2error.argtypes = [ctypes.POINTER(BasisTables), ctypes.POINTER(MeshDesc), _I, ctypes.POINTER(Field),
                                 P, P, P, P, P]
        _lib = L
    return _lib


def check(rc, what="call"):
    if rc < 0:
        msg = lib().hp_gpu_last_error().decode()
        raise RuntimeError(f"{what} failed with status {rc}: {msg}")
    return rc


def ptr(a):
    """Pointer to a contiguous numpy array (or NULL for None / empty)."""
    if a is None or a.size == 0:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(_I))


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(_D))
