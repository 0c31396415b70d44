"""ctypes access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module. It loads oracle/_build/libhp_oracle.so (the C++ restatement in
hp_oracle.cpp) and, when built, oracle/_ref/libtri_basis_ref.so (the
reference's own tri_basis compiled here).
"""
import ctypes
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libhp_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtri_basis_ref.so")
_o = None
_r = None


def build():
    import subprocess
    subprocess.check_call(["make", "-s", "-C", HERE, "_build/libhp_oracle.so"])


def lib():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            build()
        o = ctypes.CDLL(ORACLE_SO)
        P = ctypes.c_void_p
        o.or_create.restype = P
        o.or_create.argtypes = [P, P, P]
        o.or_destroy.argtypes = [P]
        for n in ("or_set_state", "or_get_state", "or_get_res"):
            getattr(o, n).argtypes = [P, P, P, P]
        o.or_get_prcn.argtypes = [P, P, P, P, P]
        o.or_set_prcn.argtypes = [P, P, P, P, P]
        o.or_rsdl.argtypes = [P, ctypes.c_int]
        o.or_setup_preconditioner.argtypes = [P]
        o.or_minvrt.argtypes = [P]
        o.or_update.argtypes = [P]
        o.or_maxres.argtypes = [P, P]
        o.or_maxres.restype = ctypes.c_double
        for n in ("or_basis_proj",):
            getattr(o, n).argtypes = [P, P, P, P, P, ctypes.c_int]
        o.or_basis_proj_val.argtypes = [P, P, P, ctypes.c_int]
        o.or_basis_derivr.argtypes = [P, P, P, ctypes.c_int]
        o.or_basis_derivs.argtypes = [P, P, P, ctypes.c_int]
        o.or_basis_intgrt.argtypes = [P, P, P, ctypes.c_int]
        o.or_basis_intgrtrs.argtypes = [P, P, P, P, ctypes.c_int]
        o.or_basis_proj1d.argtypes = [P, P, P, P]
        o.or_basis_intgrt1d.argtypes = [P, P, P]
        o.or_dpbtrsnu2.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_int]
        o.or_element_jacobian.argtypes = [P, P]
        I, D = ctypes.c_int, ctypes.c_double
        o.or_mg_attach_p.argtypes = [P, P, D]
        o.or_mg_attach_h.argtypes = [P, P, P, P, P, P, D]
        o.or_mg_restrict.argtypes = [P]
        o.or_mg_prolongate.argtypes = [P]
        o.or_cycle.argtypes = [P, I, I, I, I, I]
        o.or_resnorm_essential.argtypes = [P]
        o.or_resnorm_essential.restype = D
        o.or_solve_mg.argtypes = [P, I, D, I, I, I, I, I, P, I]
        I = ctypes.c_int
        o.ot_create.restype = P
        o.ot_create.argtypes = [P, P, I, I, I, I, P, P, P, P, P, P, P]
        o.ot_destroy.argtypes = [P]
        o.ot_set_state.argtypes = [P, P, P, P, P]
        o.ot_get.argtypes = [P, I, P, P, P, P]
        o.ot_get_prcn.argtypes = [P, P, P]
        o.ot_setup_preconditioner.argtypes = [P]
        o.ot_rsdl.argtypes = [P, I]
        o.ot_set_dirichlet.argtypes = [P, P, P, P]
        o.ot_jacobian_diagonal.argtypes = [P]
        o.ot_get_jacobian_diagonal.argtypes = [P, P, P, P, P]
        o.ot_update.argtypes = [P]
        o.ot_set_flux_faces.argtypes = [P, I, P, P, P, P, P, P]
        o.ot_set_smoother.argtypes = [P, I]
        o.ot_face_topology.argtypes = [P, P, P]
        _o = o
    return _o


def ref():
    """The reference's own tri_basis (oracle/_ref), or None when it was not built."""
    global _r
    if _r is None:
        if not os.path.exists(REF_SO):
            return None
        r = ctypes.CDLL(REF_SO)
        P = ctypes.c_void_p
        r.ref_tb_get.argtypes = [ctypes.c_int, ctypes.c_char_p, P]
        r.ref_tb_sizes.argtypes = [ctypes.c_int, P]
        r.ref_proj.argtypes = [ctypes.c_int, P, P, P, P, ctypes.c_int]
        r.ref_proj_val.argtypes = [ctypes.c_int, P, P, ctypes.c_int]
        r.ref_derivr.argtypes = [ctypes.c_int, P, P, ctypes.c_int]
        r.ref_derivs.argtypes = [ctypes.c_int, P, P, ctypes.c_int]
        r.ref_intgrt.argtypes = [ctypes.c_int, P, P, ctypes.c_int]
        r.ref_intgrtrs.argtypes = [ctypes.c_int, P, P, P, ctypes.c_int]
        r.ref_proj1d.argtypes = [ctypes.c_int, P, P, P]
        r.ref_intgrt1d.argtypes = [ctypes.c_int, P, P]
        r.ref_proj_bdry.argtypes = [ctypes.c_int, P, P, P, P, ctypes.c_int]
        _r = r
    return _r


_rt = None
REF_TET_SO = os.path.join(os.path.dirname(REF_SO), "libtet_basis_ref.so")


def ref_tet():
    """The reference's own tet_basis (oracle/_ref), or None when it was not built."""
    global _rt
    if _rt is None:
        if not os.path.exists(REF_TET_SO):
            return None
        r = ctypes.CDLL(REF_TET_SO)
        P, I = ctypes.c_void_p, ctypes.c_int
        r.ref_tet_sizes.argtypes = [I, P]
        r.ref_tet_get.argtypes = [I, ctypes.c_char_p, P]
        r.ref_tet_proj.argtypes = [I, P, P, P, P, P]
        r.ref_tet_intgrt.argtypes = [I, P, P]
        r.ref_tet_intgrtrst.argtypes = [I, P, P, P, P]
        r.ref_tet_deriv.argtypes = [I, I, P, P]
        r.ref_tet_proj2d.argtypes = [I, P, P, P, P]
        r.ref_tet_intgrt2d.argtypes = [I, P, P]
        _rt = r
    return _rt


def _p(a):
    return None if a is None or a.size == 0 else a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """CPU restatement of one tri_hp level (same inputs as the GPU context)."""

    def __init__(self, prob):
        self.prob = prob
        self.o = lib()
        self.h = self.o.or_create(ctypes.addressof(prob.desc), ctypes.addressof(prob.tab), ctypes.addressof(prob.phys))
        self.set_state(prob.ugv, prob.ugs, prob.ugi)

    def __del__(self):
        try:
            self.o.or_destroy(self.h)
        except Exception:
            pass

    def set_state(self, v, s, i):
        v, s, i = (np.ascontiguousarray(a, dtype=np.float64) for a in (v, s, i))
        self.o.or_set_state(self.h, _p(v), _p(s), _p(i))

    def state(self):
        p = self.prob
        v = np.zeros_like(p.ugv); s = np.zeros_like(p.ugs); i = np.zeros_like(p.ugi)
        self.o.or_get_state(self.h, _p(v), _p(s), _p(i))
        return v, s, i

    def residual(self):
        p = self.prob
        v = np.zeros_like(p.ugv); s = np.zeros_like(p.ugs); i = np.zeros_like(p.ugi)
        self.o.or_get_res(self.h, _p(v), _p(s), _p(i))
        return v, s, i

    def prcn(self):
        p = self.prob
        m = p.mesh
        vp = np.zeros((m.npnt, p.NV)); sp = np.zeros((m.nseg, p.NV))
        tp = np.zeros((m.ntri, p.NV)); tau = np.zeros((m.ntri, p.NV))
        self.o.or_get_prcn(self.h, _p(vp), _p(sp), _p(tp), _p(tau))
        return vp, sp, tp, tau

    def setup_preconditioner(self):
        return self.o.or_setup_preconditioner(self.h)

    def rsdl(self, stage):
        self.o.or_rsdl(self.h, stage)

    def minvrt(self):
        self.o.or_minvrt(self.h)

    def update(self):
        self.o.or_update(self.h)

    def maxres(self):
        out = np.zeros(self.prob.NV)
        return self.o.or_maxres(self.h, _p(out)), out


class OracleHierarchy:
    """The oracle's restatement of a multigrid hierarchy (tri_hp::mg_restrict /
    mg_prolongate / mg_source and block::cycle): one Oracle per level, levels[0] the
    finest, each next one a p-level ("p") or an h-level ("h") of the previous, with the
    same mgconnect transfer weights as hpb.multigrid.Hierarchy."""

    def __init__(self, probs, kinds, fadd=1.0):
        from hpb.multigrid import connect
        self.probs = probs
        self.levels = [Oracle(pr) for pr in probs]
        self._keep = []
        o = lib()
        for l in range(1, len(probs)):
            c, f = self.levels[l], self.levels[l - 1]
            if kinds[l] == "p":
                rc = o.or_mg_attach_p(c.h, f.h, fadd)
            else:
                f2c_t, f2c_w = connect(probs[l - 1].mesh, probs[l].mesh)
                c2f_t, c2f_w = connect(probs[l].mesh, probs[l - 1].mesh)
                arrs = [np.ascontiguousarray(a) for a in (f2c_t, f2c_w, c2f_t, c2f_w)]
                self._keep += arrs
                rc = o.or_mg_attach_h(c.h, f.h, *[_p(a) for a in arrs], fadd)
            if rc != 0:
                raise ValueError(f"level {l} cannot be attached as a {kinds[l]}-level")

    def _handles(self):
        return (ctypes.c_void_p * len(self.levels))(*[lv.h for lv in self.levels])

    def cycle(self, vw=1, itercrsn=2, iterrfne=2, eval_prcn=True):
        return lib().or_cycle(self._handles(), len(self.levels), vw, itercrsn, iterrfne, int(eval_prcn))

    def solve(self, drop=1e-10, max_cycles=500, vw=1, itercrsn=2, iterrfne=2, prcn_every=1):
        """Cycles until ||R64|| (essential rows excluded) has dropped by `drop`; returns
        (hist, cycles) as hpb.multigrid.Hierarchy.solve does (without the time)."""
        hist = np.zeros(max_cycles + 2)
        nc = lib().or_solve_mg(self._handles(), len(self.levels), drop, max_cycles, vw, itercrsn, iterrfne,
                               prcn_every, _p(hist), len(hist))
        if nc < 0:
            raise RuntimeError(f"preconditioner set-up met {-nc} bad elements")
        return hist[:nc + 1], nc


def element_jacobians(oracle):
    """tri_hp::element_jacobian of every element of an Oracle (K [ntri][tm*NV][tm*NV])."""
    pr = oracle.prob
    nj = pr.NV * (pr.p + 1) * (pr.p + 2) // 2
    K = np.zeros((pr.mesh.ntri, nj, nj))
    lib().or_element_jacobian(oracle.h, _p(K))
    return K


class OracleTet:
    """CPU restatement of the tet ins residual path (hp_oracle_tet.cpp) for a
    hpb.tet.TetProblem. Test infrastructure only."""

    def __init__(self, prob):
        o = lib()
        m = prob.mesh
        self.prob = prob
        self.h = o.ot_create(ctypes.byref(prob.tab), ctypes.byref(prob.phys), m.npnt, m.nseg, m.ntri, m.ntet,
                             _p(m.pnts), _p(m.tet_pnt), _p(m.tet_seg), _p(m.tet_sgn), _p(m.tet_tri), _p(m.tet_rot),
                             _p(m.vol))
        self.set_state(*prob.state)

    def __del__(self):
        if getattr(self, "h", None):
            lib().ot_destroy(self.h)
            self.h = None

    def set_state(self, v, e, f, i):
        lib().ot_set_state(self.h, _p(v), _p(e), _p(f), _p(i))

    def _get(self, which):
        out = [np.zeros_like(a) for a in self.prob.state]
        lib().ot_get(self.h, which, *[_p(a) for a in out])
        return out

    def residual(self):
        return self._get(0)

    def residual_r(self):
        return self._get(1)

    def state(self):
        return self._get(2)

    def setup_preconditioner(self):
        return lib().ot_setup_preconditioner(self.h)

    def prcn(self):
        m = self.prob.mesh
        tau = np.zeros((m.ntet, 2))
        ip = np.zeros((m.ntet, 4))
        lib().ot_get_prcn(self.h, _p(tau), _p(ip))
        return tau, ip

    def rsdl(self, stage):
        lib().ot_rsdl(self.h, stage)

    def set_dirichlet(self, masks):
        mv, me, mf = (np.ascontiguousarray(a, dtype=np.uint8) for a in masks)
        lib().ot_set_dirichlet(self.h, _p(mv), _p(me), _p(mf))

    def set_flux_faces(self, ff):
        a = {k: np.ascontiguousarray(v) for k, v in ff.items()}
        self._ff = a
        lib().ot_set_flux_faces(self.h, len(a["face_tri"]), _p(a["face_tri"]), _p(a["face_pnt"]),
                                _p(a["face_seg"]), _p(a["face_sgn"]), _p(a["kind"]), _p(a["pbc"]))

    def set_smoother(self, kind):
        if lib().ot_set_smoother(self.h, kind) != 0:
            raise ValueError("minvrt is restated for p = 1, 2 and 3 only")

    def face_topology(self):
        """(face vertices, face edges) [ntri][3] that minvrt's face steps use at p = 3."""
        m = self.prob.mesh
        fp = np.zeros((m.ntri, 3), np.int32)
        fs = np.zeros((m.ntri, 3), np.int32)
        lib().ot_face_topology(self.h, _p(fp), _p(fs))
        return fp, fs

    def jacobian_diagonal(self):
        lib().ot_jacobian_diagonal(self.h)
        out = [np.zeros_like(a) for a in self.prob.state]
        lib().ot_get_jacobian_diagonal(self.h, *[_p(a) for a in out])
        return out

    def update(self):
        lib().ot_update(self.h)
