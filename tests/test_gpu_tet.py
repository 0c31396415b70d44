"""The tet_hp ins residual on the GPU (include/hp_tet.h) against the CPU oracle
(oracle/hp_oracle_tet.cpp): tau and the element diagonals of
tet_hp_ins::setup_preconditioner, and tet_hp::rsdl (res and res_r) at every kind of
stage, p = 1..4, on a cube of 3^3 x 6 tetrahedra with a Beltrami state plus noise.
The GPU sums points and modes in another order than the oracle: 1e-12 of max|oracle|."""
import numpy as np
import pytest

from hpb.tet import TetGPU, TetProblem
from hpb.tetmesh import cube_tets
from oracle.oracle import OracleTet

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a = np.concatenate([np.ravel(x) for x in a])
    b = np.concatenate([np.ravel(x) for x in b])
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_tet_rsdl_matches_oracle(p):
    pr = TetProblem(cube_tets(3), p, mu=0.01).set_beltrami()
    g, o = TetGPU(pr), OracleTet(pr)
    assert g.setup_preconditioner() == 0 and o.setup_preconditioner() == 0
    gt, gi = g.prcn()
    ot, oi = o.prcn()
    assert relerr([gt, gi], [ot, oi]) < 1e-13
    for stage in (pr.phys.nstage, 0, 1, 2):
        g.rsdl(stage)
        o.rsdl(stage)
        assert relerr(g.residual(), o.residual()) < 1e-12, f"res stage {stage}"
        assert relerr(g.residual(1), o.residual_r()) < 1e-12, f"res_r stage {stage}"
    g.close()


@pytest.mark.parametrize("outflow", [False, True])
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_tet_rsdl_with_face_fluxes_matches_oracle(p, outflow):
    """The boundary-face fluxes added by rsdl at every stage: bdry_ins::inflow on the six
    faces, or inflow on five and a neumann outflow with the Beltrami pressure at x = 1."""
    pr = TetProblem(cube_tets(3), p, mu=0.01).set_beltrami()
    masks, ff = pr.cube_boundary(outflow=outflow)
    g, o = TetGPU(pr), OracleTet(pr)
    g.set_flux_faces(ff)
    o.set_flux_faces(ff)
    assert g.setup_preconditioner() == 0 and o.setup_preconditioner() == 0
    for stage in (pr.phys.nstage, 0, 1):
        g.rsdl(stage)
        o.rsdl(stage)
        assert relerr(g.residual(), o.residual()) < 1e-12, f"res stage {stage}"
    # the fluxes changed the boundary rows
    bare = OracleTet(pr)
    bare.setup_preconditioner()
    bare.rsdl(1)
    assert relerr(o.residual(), bare.residual()) > 1e-3
    g.close()


def test_tet_set_flux_faces_rejects_bad_indices():
    pr = TetProblem(cube_tets(2), 2, mu=0.01).set_beltrami()
    _, ff = pr.cube_boundary(outflow=True)
    g = TetGPU(pr)
    bad = dict(ff)
    bad["face_seg"] = ff["face_seg"].copy()
    bad["face_seg"][1, 2] = pr.mesh.nseg
    with pytest.raises(RuntimeError, match="out of range"):
        g.set_flux_faces(bad)
    bad = dict(ff)
    bad["pbc"] = np.zeros((0, 9))
    with pytest.raises(RuntimeError, match="pbc"):
        g.set_flux_faces(bad)
    g.set_flux_faces(ff)
    g.close()


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_tet_jacobian_diagonal_matches_oracle(p):
    """tet_hp::jacobian_diagonal: finite differences divide rounding by dw ~ 1e-6 |u|, so
    the GPU and the oracle agree to ~1e-9 of max|diagonal|; checked at 1e-7."""
    pr = TetProblem(cube_tets(3), p, mu=0.01).set_beltrami()
    g, o = TetGPU(pr), OracleTet(pr)
    assert g.setup_preconditioner() == 0 and o.setup_preconditioner() == 0
    assert relerr(g.jacobian_diagonal(), o.jacobian_diagonal()) < 1e-7
    g.close()


@pytest.mark.parametrize("p", [2, 3])
def test_tet_jacobi_updates_match_oracle(p):
    """tet_hp::update of the JACOBI build with velocity fixed on every boundary face."""
    pr = TetProblem(cube_tets(3), p, mu=0.01).set_beltrami()
    masks = pr.dirichlet_masks()
    g, o = TetGPU(pr), OracleTet(pr)
    g.set_dirichlet(masks)
    o.set_dirichlet(masks)
    assert g.setup_preconditioner() == 0 and o.setup_preconditioner() == 0
    g.jacobian_diagonal()
    o.jacobian_diagonal()
    for _ in range(3):
        g.update()
        o.update()
    assert relerr(g.state(), o.state()) < 1e-9
    # fixed rows keep their values
    u0 = pr.ugv
    mv = masks[0].astype(bool)
    assert np.array_equal(g.state()[0][mv], u0[mv])
    g.close()


@pytest.mark.parametrize("p", [2, 3])
def test_tet_jacobi_updates_with_face_fluxes_match_oracle(p):
    pr = TetProblem(cube_tets(3), p, mu=0.01).set_beltrami()
    masks, ff = pr.cube_boundary(outflow=True)
    g, o = TetGPU(pr), OracleTet(pr)
    for x in (g, o):
        x.set_dirichlet(masks)
        x.set_flux_faces(ff)
        assert x.setup_preconditioner() == 0
        x.jacobian_diagonal()
    for _ in range(3):
        g.update()
        o.update()
    assert relerr(g.state(), o.state()) < 1e-9
    g.close()


def test_tet_multigrid_reduces_residual_and_keeps_essential_values():
    """p-levels 3, 2, 1 and two h-levels (tet_hp mg_restrict / mg_prolongate with the
    FAS source): the residual falls, and the velocity on the boundary faces (essential)
    is unchanged by smoothing and by every prolongation."""
    from hpb.tet import TetHierarchy
    H = TetHierarchy(8, 3, hlevels=2, mu=0.01, cfl={1: 0.5, 2: 0.5, 3: 0.5})
    u0 = [a.copy() for a in H.probs[0].state]
    hist, sec, cycles = H.solve(drop=1e-10, max_cycles=30, vw=1)
    assert np.all(np.isfinite(hist)) and hist[-1] < 0.2
    mv, me, mf = (m.astype(bool) for m in H.masks[0])
    u = H.levels[0].state()
    assert np.array_equal(u[0][mv], u0[0][mv])
    assert np.array_equal(u[1][np.broadcast_to(me[:, None, :], u[1].shape)],
                          u0[1][np.broadcast_to(me[:, None, :], u0[1].shape)])
    H.close()


@pytest.mark.parametrize("p,cfl", [(1, 2.2), (2, 1.5), (3, 1.0)])
def test_tet_minvrt_updates_match_oracle(p, cfl):
    """tet_hp::update with tet_hp::minvrt (p = 1: res.v *= vdiag / vprcn; p = 2: also the
    edge / vertex removals and the edge scaling; p = 3: also the face removals, the
    vertex-ball solves of the edges' first modes with the spoke factors, and the second edge
    modes and the faces), face fluxes and essential rows, at the reference's default cfl for
    that p."""
    pr = TetProblem(cube_tets(3), p, mu=0.01, cfl=cfl).set_beltrami()
    masks, ff = pr.cube_boundary()
    g, o = TetGPU(pr), OracleTet(pr)
    for x in (g, o):
        x.set_dirichlet(masks)
        x.set_flux_faces(ff)
        x.set_smoother(1)
        assert x.setup_preconditioner() == 0
    for _ in range(3):
        g.update()
        o.update()
    assert relerr(g.state(), o.state()) < 1e-12
    g.close()


def test_tet_set_smoother_minvrt_needs_p_at_most_3():
    pr = TetProblem(cube_tets(2), 4, mu=0.01).set_beltrami()
    g = TetGPU(pr)
    with pytest.raises(RuntimeError, match="p = 1, 2 and 3"):
        g.set_smoother(1)
    g.close()


def test_tet_minvrt_p3_fixed_rows_stay_and_the_spokes_factor():
    """minvrt at p = 3 keeps every row fixed by an essential condition at its value, and
    the preconditioner set-up reports no bad spoke factor."""
    pr = TetProblem(cube_tets(3), 3, mu=0.01, cfl=1.0).set_beltrami()
    masks, ff = pr.cube_boundary()
    g = TetGPU(pr)
    g.set_dirichlet(masks)
    g.set_flux_faces(ff)
    g.set_smoother(1)
    assert g.setup_preconditioner() == 0
    u0 = [a.copy() for a in g.state()]
    for _ in range(2):
        g.update()
    u = g.state()
    mv, me, mf = (np.asarray(a, dtype=bool) for a in masks)
    assert np.array_equal(u[0][mv], u0[0][mv])
    assert np.array_equal(u[1][np.broadcast_to(me[:, None, :], u[1].shape)],
                          u0[1][np.broadcast_to(me[:, None, :], u0[1].shape)])
    assert np.array_equal(u[2][np.broadcast_to(mf[:, None, :], u[2].shape)],
                          u0[2][np.broadcast_to(mf[:, None, :], u0[2].shape)])
    assert all(np.all(np.isfinite(a)) for a in u)
    g.close()


def test_tet_multigrid_with_minvrt_on_low_p_levels_reduces_residual():
    from hpb.tet import TetHierarchy
    H = TetHierarchy(8, 3, hlevels=2, mu=0.01, cfl={1: 2.2, 2: 1.5, 3: 0.5}, minvrt=True)
    hist, sec, cycles = H.solve(drop=1e-10, max_cycles=30, vw=2)
    assert np.all(np.isfinite(hist)) and hist[-1] < 1e-2
    H.close()


@pytest.mark.parametrize("p", [2, 3])
def test_tet_rsdl_and_minvrt_on_a_scrambled_mesh_match_oracle(p):
    """Residual with face fluxes and minvrt updates on a cube whose interior vertices are
    jittered and whose vertices are renumbered at random (every local orientation of the
    faces and edges that minvrt's face steps and vertex balls meet)."""
    from test_tet_face_flux import scrambled_cube
    pr = TetProblem(scrambled_cube(3, 11), p, mu=0.01, cfl=1.5 if p == 2 else 1.0).set_beltrami()
    masks, ff = pr.cube_boundary(outflow=True)
    g, o = TetGPU(pr), OracleTet(pr)
    for x in (g, o):
        x.set_dirichlet(masks)
        x.set_flux_faces(ff)
        assert x.setup_preconditioner() == 0
    for stage in (pr.phys.nstage, 0):
        g.rsdl(stage)
        o.rsdl(stage)
        assert relerr(g.residual(), o.residual()) < 1e-12
    if p in (2, 3):
        for x in (g, o):
            x.set_smoother(1)
            assert x.setup_preconditioner() == 0
        for _ in range(3):
            g.update()
            o.update()
        assert relerr(g.state(), o.state()) < 1e-11
    g.close()


@pytest.mark.parametrize("p,case,mesh", [(2, "shear", "scrambled"), (4, 1, "cube")])
def test_tet_exact_steady_solutions_have_zero_residual_on_gpu(p, case, mesh):
    """The known-answer test of tests/test_tet_face_flux.py on the GPU residual: the
    interpolant of an exact steady solution has a zero residual on every free row."""
    from test_tet_face_flux import modal_interpolant, poiseuille, scrambled_cube, shear
    msh = cube_tets(2) if mesh == "cube" else scrambled_cube(2, 5)
    pr = TetProblem(msh, p, mu=0.05).set_beltrami(noise=0.0)
    modal_interpolant(pr, shear if case == "shear" else poiseuille(case, 0.05))
    ff = pr.flux_faces(msh.boundary_faces())
    mk = pr.dirichlet_masks(msh.boundary_faces())

    def free_max(state):
        g = TetGPU(pr)
        g.upload(*state)
        g.set_flux_faces(ff)
        assert g.setup_preconditioner() == 0
        g.rsdl(pr.phys.nstage)
        r = g.residual()
        g.close()
        parts = [np.where(mk[0], 0.0, r[0]).ravel(), np.where(mk[1][:, None, :], 0.0, r[1]).ravel(), r[3].ravel()]
        if r[2].size:
            parts.append(np.where(mk[2][:, None, :], 0.0, r[2]).ravel())
        return np.max(np.abs(np.concatenate(parts)))
    rng = np.random.default_rng(3)
    pert = [a + 1e-3 * rng.uniform(-1, 1, a.shape) for a in pr.state]
    assert free_max(pr.state) < 1e-9 * free_max(pert)
