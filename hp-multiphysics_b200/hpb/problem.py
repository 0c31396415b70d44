"""Problem set-up around the GPU path, mirroring the reference's tri_hp
initialisation (tri_hp/allocate.cpp, ins/allocate.cpp, cd/allocate.cpp,
tobasis.cpp, hp_boundary setvalues) for the workloads this library runs.

A Problem owns the numpy arrays behind an hp_mesh_desc, the basis tables of
its p, the physics constants and the initial state. ``Problem.gpu()`` opens a
device context (tri_hp_gpu in the reference's terms) through the C-ABI.
"""
import ctypes
import numpy as np

from . import _lib as L
from .mesh import square_mesh, channel_hole, splitmix64_uniform

# Multistage defaults (tri_mesh/blocks.cpp:1124-1148) and CFL per log2p (tri_hp/allocate.cpp:275)
ALPHA_DFLT = (0.25, 1.0 / 6.0, 0.375, 0.5, 1.0)
BETA_DFLT = (1.0, 0.0, 5.0 / 9.0, 0.0, 4.0 / 9.0)
CFL_DFLT = {0: 2.5, 1: 1.5, 2: 1.0, 3: 0.5}


def default_cfl(p):
    """hp_gbl->cfl(log2p) default; p that is not a power of two takes the next lower entry."""
    log2p = {1: 0, 2: 1, 3: 1, 4: 2, 5: 2, 6: 2, 7: 2, 8: 3}[p]
    return CFL_DFLT[log2p]


_TABLE_CACHE = {}


def basis_tables(p):
    """hp_basis_tables of tri_basis<p,0> built by the library (hp_basis_build)."""
    if p not in _TABLE_CACHE:
        t = L.BasisTables()
        rc = L.lib().hp_basis_build(p, ctypes.byref(t))
        if rc != 0:
            raise RuntimeError(f"hp_basis_build({p}) returned {rc}")
        _TABLE_CACHE[p] = t
    return _TABLE_CACHE[p]




class Problem:
    def __init__(self, mesh, p, physics, *, rho=1.0, mu=0.01, rhocv=1.0, kcond=1e-3, ax=1.0, ay=0.5, src=0.0,
                 adis=1.0, nstage=5, alpha=ALPHA_DFLT, beta=BETA_DFLT, cfl=None, field=None, bc=None):
        self.mesh = mesh
        self.p = p
        self.physics = physics
        self.NV = 3 if physics == L.HP_PHYS_INS else 1
        self.tab = basis_tables(p)
        self.sm = self.tab.sm
        self.im = self.tab.im
        self.field = field
        ph = L.PhysParams()
        ph.physics = physics
        ph.nstage = nstage
        for k in range(8):
            ph.alpha[k] = alpha[k] if k < nstage else 1.0
            ph.beta[k] = beta[k] if k < nstage else 1.0
        ph.cfl = default_cfl(p) if cfl is None else cfl
        ph.bd0 = 0.0
        ph.adis = adis
        ph.rho, ph.mu = rho, mu
        ph.rhocv, ph.kcond, ph.ax, ph.ay, ph.src = rhocv, kcond, ax, ay, src
        self.phys = ph
        self._set_bc(bc or [])
        self._build_desc()
        self.ugv = np.zeros((mesh.npnt, self.NV))
        self.ugs = np.zeros((mesh.nseg, self.sm, self.NV))
        self.ugi = np.zeros((mesh.ntri, self.im, self.NV))

    # --- boundary conditions -------------------------------------------------
    def _set_bc(self, bc):
        """bc: list of (segment-index array, kind[, curve]) with kind = essential mask |
        flux form; `curve(X, Y) -> (Xc, Yc)` maps points near the boundary onto it (the
        reference's mvpttobdry) and makes those sides curved (p > 1)."""
        bsegs, kinds, curved = [], [], []
        off = 0
        for entry in bc:
            segs, kind = entry[0], entry[1]
            curve = entry[2] if len(entry) > 2 else None
            segs = np.asarray(segs, dtype=np.int32)
            bsegs.append(segs)
            kinds.append(np.full(len(segs), kind, dtype=np.int32))
            curved.append((off, len(segs), curve))
            off += len(segs)
        self.bseg = np.ascontiguousarray(np.concatenate(bsegs) if bsegs else np.zeros(0, np.int32))
        self.bkind = np.ascontiguousarray(np.concatenate(kinds) if kinds else np.zeros(0, np.int32))
        G = self.tab.gpx
        gx = np.array([[self.tab.gx[k][n] for n in range(self.tab.nmodx)] for k in range(G)])
        v0 = self.mesh.seg_pnt[self.bseg, 0]
        v1 = self.mesh.seg_pnt[self.bseg, 1]
        # straight chord at the side Gauss points
        X = np.outer(self.mesh.pnts[v0, 0], gx[:, 1]) + np.outer(self.mesh.pnts[v1, 0], gx[:, 2])
        Y = np.outer(self.mesh.pnts[v0, 1], gx[:, 1]) + np.outer(self.mesh.pnts[v1, 1], gx[:, 2])
        self.bcrd = None
        if self.sm > 0 and any(c is not None for _, _, c in curved):
            # hp_edge_bdry::curv_init: side modes of (curve - chord)
            self.bcrd = np.zeros((len(self.bseg), self.sm, 2))
            for o, cnt, curve in curved:
                if curve is None or cnt == 0:
                    continue
                sl = slice(o, o + cnt)
                xc, yc = curve(X[sl], Y[sl])
                ends = np.ascontiguousarray(np.stack([self.mesh.pnts[v0[sl]], self.mesh.pnts[v1[sl]]], 1))
                cur = np.ascontiguousarray(np.stack([xc, yc], -1), dtype=np.float64)
                out = np.zeros((cnt, self.sm, 2))
                L.check(L.lib().hp_curved_side_modes(ctypes.byref(self.tab), cnt, L.ptr(ends), L.ptr(cur),
                                                     L.ptr(out)), "hp_curved_side_modes")
                self.bcrd[sl] = out
            self.bcrd = np.ascontiguousarray(self.bcrd)
            # positions on the curved sides (proj1d of the position modes)
            X = X + np.einsum("em,km->ek", self.bcrd[:, :, 0], gx[:, 3:3 + self.sm])
            Y = Y + np.einsum("em,km->ek", self.bcrd[:, :, 1], gx[:, 3:3 + self.sm])
        self.bpibc = np.zeros((max(len(self.bseg), 1), G))
        if self.physics == L.HP_PHYS_INS and self.field is not None and len(self.bseg):
            # ibc->f(NV-1, x) at the side Gauss points of each boundary edge
            self.bpibc[: len(self.bseg)] = self.eval_field(2, X, Y)
        self.bpibc = np.ascontiguousarray(self.bpibc)

    def eval_field(self, n, X, Y):
        f = self.field
        out = np.empty_like(X, dtype=np.float64)
        flat_x, flat_y, flat_o = X.ravel(), Y.ravel(), out.reshape(-1)
        v = ctypes.c_double()
        for k in range(flat_x.size):
            L.lib().hp_field_eval(ctypes.byref(f), n, float(flat_x[k]), float(flat_y[k]), ctypes.byref(v))
            flat_o[k] = v.value
        return out

    def _build_desc(self):
        m = self.mesh
        d = L.MeshDesc()
        d.npnt, d.nseg, d.ntri = m.npnt, m.nseg, m.ntri
        d.pnts = L.dptr(m.pnts)
        d.seg_pnt, d.seg_tri = L.iptr(m.seg_pnt), L.iptr(m.seg_tri)
        d.tri_pnt, d.tri_seg, d.tri_sgn = L.iptr(m.tri_pnt), L.iptr(m.tri_seg), L.iptr(m.tri_sgn)
        d.nbseg = len(self.bseg)
        d.bseg = L.iptr(self.bseg)
        d.bseg_kind = L.iptr(self.bkind)
        d.bseg_pibc = L.dptr(self.bpibc)
        d.bseg_crd = L.dptr(self.bcrd) if self.bcrd is not None else None
        self.desc = d

    # --- initial state -------------------------------------------------------
    def tobasis(self, noise=0.0, seed=0):
        """tri_hp::tobasis of self.field, optional seeded U[-1,1) noise of amplitude
        `noise` on every v/s/i coefficient, then the essential boundary values are
        set again (hp_edge_bdry::setvalues), as a time step's tadvance does."""
        lib = L.lib()
        rc = lib.hp_tobasis(ctypes.byref(self.tab), ctypes.byref(self.desc), self.NV, ctypes.byref(self.field),
                            L.ptr(self.ugv), L.ptr(self.ugs), L.ptr(self.ugi))
        L.check(rc, "hp_tobasis")
        if noise:
            nv, ns, ni = self.ugv.size, self.ugs.size, self.ugi.size
            r = splitmix64_uniform(seed, nv + ns + ni) * noise
            self.ugv += r[:nv].reshape(self.ugv.shape)
            self.ugs += r[nv:nv + ns].reshape(self.ugs.shape)
            self.ugi += r[nv + ns:].reshape(self.ugi.shape)
        L.check(lib.hp_setvalues(ctypes.byref(self.tab), ctypes.byref(self.desc), self.NV, ctypes.byref(self.field),
                                 L.ptr(self.ugv), L.ptr(self.ugs)), "hp_setvalues")
        return self

    def l2error(self, ugv=None, ugs=None, ugi=None):
        ugv = self.ugv if ugv is None else ugv
        ugs = self.ugs if ugs is None else ugs
        ugi = self.ugi if ugi is None else ugi
        l2 = np.zeros(self.NV)
        li = np.zeros(self.NV)
        L.check(L.lib().hp_l2error(ctypes.byref(self.tab), ctypes.byref(self.desc), self.NV, ctypes.byref(self.field),
                                   L.ptr(np.ascontiguousarray(ugv)), L.ptr(np.ascontiguousarray(ugs)),
                                   L.ptr(np.ascontiguousarray(ugi)), L.ptr(l2), L.ptr(li)), "hp_l2error")
        return l2, li

    @property
    def ndof(self):
        return self.NV * (self.mesh.npnt + self.mesh.nseg * self.sm + self.mesh.ntri * self.im)

    def gpu(self, device=0, stream=None):
        return GPULevel(self, device, stream)


class GPULevel:
    """One device context (hp_gpu_ctx) for a Problem: the reference's
    tri_hp::{rsdl, setup_preconditioner, minvrt, update, maxres} through the C-ABI."""

    def __init__(self, prob, device=0, stream=None):
        self.prob = prob
        self.lib = L.lib()
        h = ctypes.c_void_p()
        rc = self.lib.hp_gpu_create(ctypes.byref(prob.desc), ctypes.byref(prob.tab), ctypes.byref(prob.phys),
                                    device, stream, ctypes.byref(h))
        L.check(rc, "hp_gpu_create")
        self.h = h
        self.upload(prob.ugv, prob.ugs, prob.ugi)

    def close(self):
        if self.h:
            self.lib.hp_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, v, s, i):
        v, s, i = (np.ascontiguousarray(a, dtype=np.float64) for a in (v, s, i))
        L.check(self.lib.hp_gpu_upload_state(self.h, L.ptr(v), L.ptr(s), L.ptr(i)), "upload")

    def state(self):
        p = self.prob
        v = np.zeros_like(p.ugv); s = np.zeros_like(p.ugs); i = np.zeros_like(p.ugi)
        L.check(self.lib.hp_gpu_download_state(self.h, L.ptr(v), L.ptr(s), L.ptr(i)), "download_state")
        return v, s, i

    def residual(self):
        p = self.prob
        v = np.zeros_like(p.ugv); s = np.zeros_like(p.ugs); i = np.zeros_like(p.ugi)
        L.check(self.lib.hp_gpu_download_residual(self.h, L.ptr(v), L.ptr(s), L.ptr(i)), "download_residual")
        return v, s, i

    def prcn(self):
        p = self.prob
        m = p.mesh
        vp = np.zeros((m.npnt, p.NV)); sp = np.zeros((m.nseg, p.NV))
        tp = np.zeros((m.ntri, p.NV)); tau = np.zeros((m.ntri, p.NV))
        L.check(self.lib.hp_gpu_download_prcn(self.h, L.ptr(vp), L.ptr(sp), L.ptr(tp), L.ptr(tau)), "download_prcn")
        return vp, sp, tp, tau

    def setup_preconditioner(self):
        return L.check(self.lib.hp_gpu_setup_preconditioner(self.h), "setup_preconditioner")

    def rsdl(self, stage, precision=0):
        """tri_hp::rsdl(stage); precision 0 = FP64 kernels, 1 = FP32 kernels (result widened)."""
        L.check(self.lib.hp_gpu_rsdl(self.h, stage, precision), "rsdl")

    def l2error(self, field=None):
        """tri_hp::l2error on the device against `field` (default: the problem's field)."""
        f = self.prob.field if field is None else field
        l2 = np.zeros(self.prob.NV)
        li = np.zeros(self.prob.NV)
        L.check(self.lib.hp_gpu_l2error(self.h, ctypes.byref(f), L.ptr(l2), L.ptr(li)), "l2error")
        return l2, li

    def autotune(self, reps=5):
        """hp_gpu_autotune; returns the chosen shapes and tuned times of FP64 and FP32."""
        L.check(self.lib.hp_gpu_autotune(self.h, reps), "autotune")
        return self.tuning()

    def tuning(self):
        sh = np.zeros(8, dtype=np.int32)
        ms = np.zeros(4, dtype=np.float32)
        L.check(self.lib.hp_gpu_get_tuning(self.h, L.ptr(sh), L.ptr(ms)), "get_tuning")
        keys = ("elem_cap", "emat_tpp", "emat_ctas", "minv_threads")
        return {prec: dict({k: int(sh[4 * i + j]) for j, k in enumerate(keys)},
                           elem_ms=float(ms[2 * i]), minv_ms=float(ms[2 * i + 1]))
                for i, prec in enumerate(("fp64", "fp32"))}

    def element_jacobians(self):
        """tri_hp::element_jacobian of every element (hp_gpu_element_jacobian):
        K [ntri][tm*NV][tm*NV], row i*NV + n, column mode*NV + var."""
        tm = (self.prob.p + 1) * (self.prob.p + 2) // 2
        nj = tm * self.prob.NV
        K = np.zeros((self.prob.mesh.ntri, nj, nj))
        self.lib.hp_gpu_element_jacobian.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.check(self.lib.hp_gpu_element_jacobian(self.h, L.ptr(K)), "element_jacobian")
        return K

    def element_kernel(self, kind):
        """Element kernel (hp_gpu_set_element_kernel): "tensor" (ins default at p >= 3),
        "point" (ins default at p = 1) or "scalar"."""
        L.check(self.lib.hp_gpu_set_element_kernel(self.h, {"scalar": 0, "tensor": 1, "point": 2}[kind]),
                "set_element_kernel")

    def element_matrices(self, on=True):
        """cd only: rsdl from stored element operators (hp_gpu_set_element_matrices)."""
        L.check(self.lib.hp_gpu_set_element_matrices(self.h, 1 if on else 0), "set_element_matrices")

    def minvrt(self):
        L.check(self.lib.hp_gpu_minvrt(self.h), "minvrt")

    def update(self):
        L.check(self.lib.hp_gpu_update(self.h), "update")

    def iterate(self, iters, prcn_interval=0):
        hist = np.zeros(max(iters, 1))
        L.check(self.lib.hp_gpu_iterate(self.h, iters, prcn_interval, L.ptr(hist)), "iterate")
        return hist[:iters]

    def maxres(self):
        out = np.zeros(self.prob.NV)
        mx = ctypes.c_double()
        L.check(self.lib.hp_gpu_maxres(self.h, L.ptr(out), ctypes.byref(mx)), "maxres")
        return mx.value, out

    def solve(self, mixed=False, drop=1e-10, max_updates=20000, inner=20, check_every=10, prcn_every=0):
        """hp_gpu_solve: smooth until ||R64|| drops by `drop`. Returns (hist, seconds, updates)."""
        cap = max_updates // max(1, min(inner, check_every)) + 4
        hist = np.zeros(cap)
        nh = ctypes.c_int(); sec = ctypes.c_double(); nup = ctypes.c_int()
        L.check(self.lib.hp_gpu_solve(self.h, 1 if mixed else 0, drop, max_updates, inner, check_every, prcn_every,
                                      L.ptr(hist), cap, ctypes.byref(nh), ctypes.byref(sec), ctypes.byref(nup)),
                "solve")
        return hist[:nh.value], sec.value, nup.value

    def resnorm(self):
        l2 = ctypes.c_double(); li = ctypes.c_double()
        L.check(self.lib.hp_gpu_resnorm(self.h, ctypes.byref(l2), ctypes.byref(li)), "resnorm")
        return l2.value, li.value


# --- workloads ---------------------------------------------------------------

def _edges_where(mesh, pred):
    b = mesh.boundary_segments()
    mid = 0.5 * (mesh.pnts[mesh.seg_pnt[b, 0]] + mesh.pnts[mesh.seg_pnt[b, 1]])
    return b[pred(mid[:, 0], mid[:, 1])]


def kovasznay_ins(n=64, p=4, re=100.0, noise=1e-3, seed=20261204, mesh=None, **kw):
    """2D incompressible Navier-Stokes, Kovasznay flow at Re on an n x n split-square
    mesh of the unit square (or `mesh`, a mesh of the unit square); inflow (velocity
    essential) on left/top/bottom, outflow (generic flux with the analytic pressure) on the
    right; rho = 1, mu = 1/Re."""
    mesh = square_mesh(n) if mesh is None else mesh
    field = L.Field(L.HP_FIELD_KOVASZNAY, (ctypes.c_double * 4)(re, 0, 0, 0))
    eps = 1e-12
    inflow = _edges_where(mesh, lambda x, y: (x < eps) | (y < eps) | (y > 1 - eps))
    outflow = _edges_where(mesh, lambda x, y: (x > 1 - eps) & (y > eps) & (y < 1 - eps))
    bc = [(inflow, 0b011 | L.HP_BC_FLUX_INS_GENERIC), (outflow, L.HP_BC_FLUX_INS_GENERIC)]
    prob = Problem(mesh, p, L.HP_PHYS_INS, rho=1.0, mu=1.0 / re, field=field, bc=bc, **kw)
    return prob.tobasis(noise=noise, seed=seed)


def lid_cavity_ins(n=64, p=4, re=400.0, noise=1e-3, seed=20261206, mesh=None, **kw):
    """ins lid-driven cavity: u = 1 on the lid (y = 1), zero on the other walls, velocity
    essential everywhere; on the n x n split-square mesh of the unit square, or `mesh`."""
    mesh = square_mesh(n) if mesh is None else mesh
    field = L.Field(L.HP_FIELD_LID, (ctypes.c_double * 4)(0, 0, 0, 0))
    walls = mesh.boundary_segments()
    bc = [(walls, 0b011 | L.HP_BC_FLUX_INS_GENERIC)]
    prob = Problem(mesh, p, L.HP_PHYS_INS, rho=1.0, mu=1.0 / re, field=field, bc=bc, **kw)
    return prob.tobasis(noise=noise, seed=seed)


def cd_sinsin(mesh=None, n=64, p=4, ax=1.0, ay=0.5, kcond=1e-3, noise=1e-3, seed=20261205, field=None, **kw):
    """Scalar convection-diffusion, velocity (ax, ay), diffusivity kcond, Dirichlet data
    sin(pi x) sin(pi y) on every boundary edge (or `field`), initial state the same
    field plus noise."""
    mesh = mesh if mesh is not None else square_mesh(n)
    if field is None:
        field = L.Field(L.HP_FIELD_SINSIN, (ctypes.c_double * 4)(1.0, 0, 0, 0))
    bc = [(mesh.boundary_segments(), 0b1)]
    prob = Problem(mesh, p, L.HP_PHYS_CD, rhocv=1.0, kcond=kcond, ax=ax, ay=ay, field=field, bc=bc, **kw)
    return prob.tobasis(noise=noise, seed=seed)


def circle_curve(cx, cy, r):
    """mvpttobdry of a circular boundary: radial projection onto the circle."""
    def curve(X, Y):
        dx, dy = X - cx, Y - cy
        d = np.hypot(dx, dy)
        return cx + r * dx / d, cy + r * dy / d
    return curve


def channel_cylinder_ins(scale=1.0, p=4, re=100.0, noise=1e-3, seed=20261207, curved=True, mesh=None, **kw):
    """ins flow past a cylinder: channel [0,20] x [0,10] with a hole of radius 0.5 at
    (5, 5) (diameter 1, so Re = 1/mu at rho = 1 and free-stream speed 1), graded mesh
    channel_hole with edge lengths scaled by `scale` (1: ~150k triangles), or `mesh` (a
    channel_hole mesh). Free stream (velocity essential + generic flux) on the left, top
    and bottom walls, outflow (generic flux, p = 0) on the right, no-slip (velocity
    essential + generic flux) on the hole, whose sides are curved (isoparametric, p > 1)
    unless curved=False. Initial state: free stream u = 1 outside the cylinder plus
    seeded noise."""
    if mesh is None:
        mesh = channel_hole(hmin=0.02 * scale, hmax=0.2 * scale, grade=0.0085 * scale)
    cx, cy, r = mesh.hole
    field = L.Field(L.HP_FIELD_CYLINDER, (ctypes.c_double * 4)(cx, cy, r, 0))
    b = mesh.boundary_segments()
    mid = 0.5 * (mesh.pnts[mesh.seg_pnt[b, 0]] + mesh.pnts[mesh.seg_pnt[b, 1]])
    Lx, Hy = mesh.box
    eps = 1e-9
    hole = np.hypot(mid[:, 0] - cx, mid[:, 1] - cy) < r + eps
    outflow = (~hole) & (mid[:, 0] > Lx - eps)
    inflow = (~hole) & (~outflow)
    bc = [(b[inflow], 0b011 | L.HP_BC_FLUX_INS_GENERIC), (b[outflow], L.HP_BC_FLUX_INS_GENERIC),
          (b[hole], 0b011 | L.HP_BC_FLUX_INS_GENERIC, circle_curve(cx, cy, r) if curved else None)]
    prob = Problem(mesh, p, L.HP_PHYS_INS, rho=1.0, mu=1.0 / re, field=field, bc=bc, **kw)
    return prob.tobasis(noise=noise, seed=seed)


def cd_quadratic(n=4, p=2, noise=1e-2, seed=7, **kw):
    """Exactness case of Testing/tri_hp/conv-diff/Correctness: u = -(x-8)^2, nu = 1,
    no convection, source 2, Dirichlet everywhere; the p >= 2 discrete solution is exact."""
    mesh = square_mesh(n)
    field = L.Field(L.HP_FIELD_QUADX, (ctypes.c_double * 4)(-1.0, 8.0, 0, 0))
    bc = [(mesh.boundary_segments(), 0b1)]
    prob = Problem(mesh, p, L.HP_PHYS_CD, rhocv=1.0, kcond=1.0, ax=0.0, ay=0.0, src=2.0, field=field, bc=bc, **kw)
    return prob.tobasis(noise=noise, seed=seed)
