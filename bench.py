#!/usr/bin/env python
"""Benchmark of the tri_hp element-residual and multigrid-smoothing path on B200
(one process per GPU).

Default workload (N = 1): ins lid-driven cavity, Re 400 (rho 1, mu 1/400), p = 6,
512 x 512 split squares of the unit square (524,288 triangles, 28.3 M DOF), velocity
Dirichlet on every wall, u = 1 on the lid; state = the boundary field projected plus
U[-1,1) * 1e-3 seeded noise (splitmix64). Multigrid hierarchy: p-levels 6 -> 3 -> 1 on
the fine mesh, then h-levels of 131,072 / 32,768 / 8,192 triangles at p = 1.
A "step" is one full FP64 residual evaluation tri_hp::rsdl(nstage) of the fine level;
`value` is its rsdl GDoF/s (whole job, state resident in HBM, device time with CUDA
events, the 226 MB state exceeds L2 and L2 is flushed between steps as well); `e2e` is
the same metric through the C-ABI with host buffers (pinned state upload + rsdl +
residual download every step). `time_to_tol` runs W-cycles from the initial state to a
1e-10 drop of the FP64 residual: plain FP64, FP32 smoothing inside FP64 defect
correction, and that plus the learned preconditioner correction. `roofline` relates the
element kernel to the FP64 tensor-core (DMMA) throughput measured in the same run, with
the HBM fraction of the compulsory bytes beside it.

--gpus N > 1 runs N independent replicas (the path does not shard across GPUs in this
tier): value = sum over ranks.
--impl reference times the CPU oracle (the C++ restatement of the reference's rsdl) on
all host cores on bounded samples of the same workload.
--workload cd runs the earlier cd p = 4 line (stored element operators).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hp-multiphysics_b200"))
sys.path.insert(0, ROOT)

N_MESH = 317
P = 4
METRIC_CD = "rsdl GDoF/s (FP64 tri_hp::rsdl, cd p=4)"
METRIC = "time to 1e-10 residual drop: learned+FP32 vs plain FP64, 1xB200; rsdl GDoF/s"
C3_N, C3_P, C3_RE = 512, 6, 400.0
STRIP_ROWS = 8  # CPU samples: 512 x 8-square strips (8,192 triangles) of the C3 mesh


def c3_config():
    return {"workload": "C3: ins lid-driven cavity Re 400, p=6, 512x512 split squares (524,288 triangles, "
                        "28.3 M DOF); multigrid p-levels 6,3,1 then h-levels of 131,072 / 32,768 / 8,192 triangles",
            "physics": "ins", "p": C3_P, "ntri": 2 * C3_N * C3_N, "re": C3_RE, "nstage": 5,
            "step": "one FP64 tri_hp::rsdl(nstage) of the fine level",
            "l2": "state (226 MB) and residual exceed L2; L2 also flushed between timed steps (256 MiB write)",
            "parallelism": "replicas"}


def c3_factory(n, p, **kw):
    import hpb
    return hpb.lid_cavity_ins(n=n, p=p, re=C3_RE, **kw)


def strip_problem(k):
    """Strip k (from the lid down) of the C3 mesh: 512 x STRIP_ROWS squares with the C3
    spacing, the lid-cavity state on it (boundary field + 1e-3 noise), p = 6."""
    import hpb
    y1 = 1.0 - (k % (C3_N // STRIP_ROWS)) * STRIP_ROWS / C3_N
    m = hpb.square_mesh(C3_N, 0.0, 1.0, y1 - STRIP_ROWS / C3_N, y1, ny=STRIP_ROWS)
    return hpb.lid_cavity_ins(p=C3_P, re=C3_RE, mesh=m, seed=20261206 + k)


def cpu_strip_worker(args):
    """One host core: the oracle's rsdl(nstage) on strip k of the C3 mesh; `warmup`
    untimed then `steps` timed evaluations (steps = 0: until `secs` seconds passed)."""
    k, steps, warmup, secs = args
    sys.path.insert(0, os.path.join(ROOT, "hp-multiphysics_b200"))
    sys.path.insert(0, ROOT)
    from oracle.oracle import Oracle
    pr = strip_problem(k)
    o = Oracle(pr)
    o.setup_preconditioner()
    for _ in range(max(1, warmup)):
        o.rsdl(pr.phys.nstage)
    t0 = time.perf_counter()
    reps = 0
    while (reps < steps) if steps > 0 else (time.perf_counter() - t0 < secs):
        o.rsdl(pr.phys.nstage)
        reps += 1
    return pr.ndof * reps, time.perf_counter() - t0, reps


def run_cpu_strips(cores, steps, warmup, secs=0.0):
    """Oracle rsdl GDoF/s over `cores` processes (one strip each, run concurrently)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(cpu_strip_worker, [(k, steps, warmup, secs) for k in range(cores)])
    return sum(r[0] for r in res) / max(r[1] for r in res) / 1e9, min(r[2] for r in res)


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def ins_flops_per_element(p, beta_positive=True):
    """Algorithmic FP64 flops of one ins element residual (tri_hp_ins::element_rsdl with
    the sum-factorised tri_basis operators), from the table the oracle's op-counting
    build writes (profiles/flops_per_element.json); a loop-count estimate otherwise."""
    try:
        t = json.load(open(os.path.join(ROOT, "profiles", "flops_per_element.json")))
        return float(t["ins"][str(p)]["full" if beta_positive else "imaginary"]), "oracle op count"
    except Exception:
        G, X, T = p + 1, p + 2, (p + 1) * (p + 2) // 2
        projd = G * (4 * T + X) + 6 * G * G * X
        projv = 2 * G * T + 2 * G * G * X
        intrs = 2 * G * G + 4 * X * G * G + 4 * T * G
        der = 2 * G * G + 3 * G * G * (G - 1)
        return float(2 * projd + projv + 6 * intrs + 6 * der + 100 * G * G), "loop-count estimate"


def workload_config():
    return {
        "workload": f"tri_hp cd rsdl(nstage), p={P}, {N_MESH}x{N_MESH} split-square mesh "
                    f"({2 * N_MESH * N_MESH} triangles), velocity (1,0.5), kcond 1e-3",
        "mesh": "structured split squares standing in for the seeded 200k-triangle Delaunay mesh",
        "p": P, "physics": "cd", "ntri": 2 * N_MESH * N_MESH, "nstage": 5,
        "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas",
    }


def flops_per_element(p, nv_pairs=1, nv=1, ndv=1):
    """Loop-count FLOPs of one full-stage element residual of this library's
    kernel (cd: one variable, projected with derivatives)."""
    G, X, T = p + 1, p + 2, (p + 1) * (p + 2) // 2
    nqw = 2 * ndv + (nv - ndv)
    proj1 = 2 * nqw * G * T
    proj2 = G * G * (7 * X * ndv + 2 * X * (nv - ndv))
    intg = 2 * (6 * nv_pairs * X * G * G + 4 * nv * T * G)
    deriv = 9 * nv * G ** 3
    point = 40 * G * G
    return proj1 + proj2 + intg + deriv + point


def sample_clocks(stop_file, out):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "100"]
    try:
        return subprocess.Popen(cmd, stdout=open(out, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def parse_clocks(path, dev):
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        for line in open(path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or f[0] != str(dev):
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
    except FileNotFoundError:
        pass
    sm.sort()
    return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def cpu_worker(args):
    """One host core: oracle rsdl(nstage) on a bounded sample mesh for ~secs seconds."""
    n, p, secs = args
    sys.path.insert(0, os.path.join(ROOT, "hp-multiphysics_b200"))
    sys.path.insert(0, ROOT)
    import hpb
    from oracle.oracle import Oracle
    pr = hpb.cd_sinsin(n=n, p=p, ax=1.0, ay=0.5, kcond=1e-3, noise=1e-3, seed=20261205)
    o = Oracle(pr)
    o.setup_preconditioner()
    o.rsdl(pr.phys.nstage)
    t0 = time.perf_counter()
    reps = 0
    while True:
        o.rsdl(pr.phys.nstage)
        reps += 1
        el = time.perf_counter() - t0
        if el >= secs:
            break
    return pr.ndof * reps, el


def run_cpu(cores, secs, n=60):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(cpu_worker, [(n, P, secs)] * cores)
    dof = sum(r[0] for r in res)
    el = max(r[1] for r in res)
    return dof / el / 1e9, n


def replica_totals(dist, world, ndof, steps, t_ms, e2e_s, device):
    """Whole-job figures of N independent replicas: each rank processed `ndof` per step,
    and the slowest rank bounds the job (max over ranks of the timed region and of the
    e2e step time). Returns (value GDoF/s, e2e GDoF/s, t_ms, e2e_s)."""
    if dist is not None:
        import torch
        t = torch.tensor([t_ms, e2e_s], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms, e2e_s = float(t[0]), float(t[1])
    return world * ndof * steps / (t_ms * 1e-3) / 1e9, world * ndof / e2e_s / 1e9, t_ms, e2e_s


TOL_N = 64
MG_N = 320
CD_CFL = {8: 0.3, 6: 0.35, 4: 0.5, 3: 0.6, 2: 0.75, 1: 1.0}


def c3_sweep(hpb, dev, n, p, cycles, arms=None):
    """ins lid-driven cavity, Re 400 (rho 1, mu 1/400), p on an n x n split-square mesh
    (n = 512: 524,288 triangles, 28.3 M DOF at p = 6); u = 1 on the lid, velocity
    Dirichlet on every wall, initial state the boundary field projected plus 1e-3 noise.
    Hierarchy: p-levels p -> ... -> 1 on the fine mesh, then h-levels n/2, n/4, n/8 at
    p = 1 (the 524k/131k/32k/8k-triangle meshes). At most `cycles` W-cycles (vwcycle 2,
    the reference's ins Convergence test input; 2+2 updates per level, preconditioners
    every cycle) per arm, stopping at a 1e-10 drop of the FP64 residual; reports seconds,
    seconds per cycle and the drop reached. A V-cycle arm and the h-levels-only
    hierarchy of the reference's extra_finest_levels = 0 are run last."""
    import time as _t
    from hpb import multigrid as MG
    mk = lambda n, p, **kw: hpb.lid_cavity_ins(n=n, p=p, re=400.0, **kw)
    line = {"sweep": "c3", "workload": f"ins lid cavity Re 400, p={p}, {n}x{n} split squares", "cycles": cycles}
    for name, kw, plev in (("fp64_level_by_level", {"vw": 2}, True), ("fp64_graph", {"vw": 2, "graph": True}, True),
                           ("fp64_graph_autotuned", {"vw": 2, "graph": True, "tune": True}, True),
                           ("fp32_defect_correction", {"vw": 2, "mixed": True}, True),
                           ("fp32_defect_correction_autotuned", {"vw": 2, "mixed": True, "tune": True}, True),
                           ("fp64_v_cycle", {"vw": 1}, True), ("fp64_h_levels_only", {"vw": 2}, False)):
        if arms and name not in arms:
            continue
        t0 = _t.perf_counter()
        H = MG.build(mk, n=n, p=p, hlevels=3, plevels=plev)
        setup = _t.perf_counter() - t0
        kw = dict(kw)
        shapes = H.autotune(reps=3) if kw.pop("tune", False) else None
        hist, sec, cyc = H.solve(drop=1e-10, max_cycles=cycles, prcn_every=1, **kw)
        line[name] = {"seconds": sec, "cycles": cyc, "ms_per_cycle": 1e3 * sec / max(cyc, 1),
                      "drop": float(hist[-1]), "reached": bool(hist[-1] <= 1e-10),
                      "drop_history": [float(h) for h in hist[::max(1, cycles // 10)]],
                      "levels": [f"{len(lv.prob.mesh.tri_pnt)} tri p={lv.prob.p}" for lv in H.levels],
                      "setup_seconds_host": setup}
        if shapes:
            line[name]["shapes"] = shapes
        if name == "fp64_level_by_level":
            line["ndof"] = H.probs[0].ndof
        H.close()
        print(json.dumps({"arm": name, **line[name]}), flush=True)
    print(json.dumps(line), flush=True)


def c4_sweep(hpb, dev, scale, cycles):
    """ins past a cylinder: channel [0,20] x [0,10], hole of diameter 1 at (5, 5) with
    curved (isoparametric) sides, graded Delaunay mesh channel_hole scaled by `scale`
    (1: ~150k triangles), p = 4, free stream in, outflow p = 0 out, no-slip hole. The
    learned correction is trained on the GPU on solver-generated samples of 4 training
    instances with Re drawn from U[20, 200] (snapshot states after 0, 200, 1000 and 3000
    plain updates, every element of every snapshot one sample) and judged on 2 held-out
    Re by the time to a 1e-10 drop of the FP64 residual, at most `cycles` W-cycles
    (vwcycle 2, the cycle of the reference's ins Convergence test input; p 4 -> 2 -> 1,
    then channel meshes at 2x, 4x, 8x the edge lengths at p = 1; preconditioners every
    cycle): plain FP64, FP32 defect correction, and FP32 defect correction with the
    learned correction."""
    import time as _t
    import numpy as np
    from hpb import learned as LR
    from hpb import multigrid as MG
    meshes = {k: hpb.channel_hole(hmin=0.02 * scale * k, hmax=0.2 * scale * k, grade=0.0085 * scale * k)
              for k in (1, 2, 4, 8)}
    rng = np.random.default_rng(20261208)
    train_re = rng.uniform(20.0, 200.0, 4)
    test_re = rng.uniform(20.0, 200.0, 2)
    t0 = _t.perf_counter()
    F, T = [], []
    for k, re in enumerate(train_re):
        f, tg = LR.solver_samples(lambda: hpb.channel_cylinder_ins(mesh=meshes[1], p=4, re=float(re), seed=400 + k),
                                  snapshots=(0, 200, 1000, 3000))
        F.append(f)
        T.append(tg)
    F, T = np.concatenate(F), np.concatenate(T)
    net, hist = LR.train(F, T, steps=600)
    train_s = _t.perf_counter() - t0
    line = {"sweep": "c4", "workload": f"ins cylinder in a channel, p=4, curved hole, {meshes[1].ntri} triangles",
            "train_re": [float(x) for x in train_re], "test_re": [float(x) for x in test_re],
            "samples": int(len(T)), "snapshots": 16, "nonzero_targets": float(np.mean(T != 0)),
            "training_seconds": train_s, "loss_first_last": [float(hist[0]), float(hist[-1])], "cycles": cycles,
            "levels": [f"{meshes[k].ntri} tri" for k in (1, 2, 4, 8)]}

    def hierarchy(re):
        probs = [hpb.channel_cylinder_ins(mesh=meshes[1], p=4, re=re, seed=900)]
        kinds = ["fine"]
        for q in (2, 1):
            probs.append(hpb.channel_cylinder_ins(mesh=meshes[1], p=q, re=re, seed=900))
            kinds.append("p")
        for k in (2, 4, 8):
            probs.append(hpb.channel_cylinder_ins(mesh=meshes[k], p=1, re=re, seed=900))
            kinds.append("h")
        return MG.Hierarchy(probs, kinds)

    for re in test_re:
        res = {}
        for name, mixed, learned in (("fp64", False, False), ("fp32_defect_correction", True, False),
                                     ("learned_fp32", True, True)):
            H = hierarchy(float(re))
            if learned:
                LR.attach(H.levels[0], net, 1.0)
            h, sec, cyc = H.solve(drop=1e-10, max_cycles=cycles, vw=2, mixed=mixed, prcn_every=1)
            res[name] = {"seconds": sec, "cycles": cyc, "drop": float(h[-1]), "reached": bool(h[-1] <= 1e-10),
                         "min_drop": float(np.min(h)), "drop_history": [float(x) for x in h[::max(1, cycles // 10)]]}
            H.close()
        res["speedup_learned_fp32_vs_fp64"] = res["fp64"]["seconds"] / res["learned_fp32"]["seconds"]
        res["speedup_fp32_vs_fp64"] = res["fp64"]["seconds"] / res["fp32_defect_correction"]["seconds"]
        line[f"re_{re:.1f}"] = res
        print(json.dumps({"re": float(re), **{k: ((v["drop"], v["seconds"], v["cycles"]) if isinstance(v, dict) else v)
                                               for k, v in res.items()}}), flush=True)
    net.close()
    print(json.dumps(line), flush=True)


def tet_flops_per_element(p, beta_positive=True):
    """Multiply-adds of the dense basis operators per tetrahedron and residual,
    x 2 flops: projection of u, v, w with r, s, t derivatives and p by value
    (13 operator rows x Q x T when beta > 0, 4 otherwise) and intgrtrst of the four
    3-component fluxes (4 x 3Q x T) for the imaginary part and again for the real
    part. Pointwise flux, derivative and SUPG arithmetic is not counted."""
    G = p + 1
    Q, T = G ** 3, (p + 1) * (p + 2) * (p + 3) // 6
    proj = (13 if beta_positive else 4) * Q * T
    intg = (2 if beta_positive else 1) * 4 * 3 * Q * T
    return 2 * (proj + intg)


def c5_sweep(torch, dev, n, p, steps, warmup, timed, full_solve=False, hlevels=None, p1_minvrt=False, cfl3=None):
    """3D tet_hp ins: the unit cube split into n^3 hexahedra x 6 tetrahedra (n = 64:
    1,572,864 tetrahedra), p = 3, Re 100, the Ethier-Steinman Beltrami state at the
    vertices plus 1e-3 seeded noise on every coefficient. Times tet_hp::rsdl(nstage)
    (FP64, beta = 1: both parts of element_rsdl) on the GPU with CUDA events (the
    state, 230 MB at n = 64, exceeds L2; L2 flushed between steps anyway), the CPU
    oracle on a bounded 6^3 x 6 sample, and the FP64 tensor-core throughput of the
    GPU for the roofline."""
    import time as _t
    import numpy as np
    from hpb.tet import TetGPU, TetProblem
    from hpb.tetmesh import cube_tets
    from oracle.oracle import OracleTet
    t0 = _t.perf_counter()
    mesh = cube_tets(n)
    pr = TetProblem(mesh, p, mu=1.0 / 100.0).set_beltrami(re=100.0)
    import ctypes
    cur = torch.cuda.current_stream()
    masks, ff = pr.cube_boundary(re=100.0)
    g = TetGPU(pr, device=dev, stream=ctypes.c_void_p(cur.cuda_stream))  # events and kernels on one stream
    g.set_dirichlet(masks)
    g.set_flux_faces(ff)
    host_s = _t.perf_counter() - t0
    assert g.setup_preconditioner() == 0
    ns = pr.phys.nstage
    for _ in range(warmup):
        g.lib.hp_tet_enqueue_rsdl(g.h, ns)
    g.lib.hp_tet_sync(g.h)
    ms = timed(lambda: g.lib.hp_tet_enqueue_rsdl(g.h, ns), steps, cur)
    ms0 = timed(lambda: g.lib.hp_tet_enqueue_rsdl(g.h, 1), steps, cur)
    rsdl_ms = sum(ms) / len(ms)
    peak = ctypes.c_double()
    g.lib.hp_tet_fp64_mma_peak.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    g.lib.hp_tet_fp64_mma_peak(dev, 200.0, ctypes.byref(peak))
    fl = tet_flops_per_element(p) * mesh.ntet
    achieved = fl / (rsdl_ms * 1e-3) / 1e12
    line = {"sweep": "c5", "workload": f"tet ins p={p}, {n}^3 x 6 = {mesh.ntet} tetrahedra, Re 100 Beltrami + 1e-3 noise",
            "boundary": "bdry_ins::inflow (velocity essential, continuity flux) on the six faces, boundary flux "
                        f"balanced to zero; {len(ff['face_tri'])} flux faces",
            "ndof": pr.ndof, "ntet": mesh.ntet, "host_setup_seconds": host_s, "steps": steps, "warmup": warmup,
            "rsdl_ms": rsdl_ms, "rsdl_gdofs": pr.ndof / rsdl_ms / 1e6, "rsdl_beta0_ms": sum(ms0) / len(ms0),
            "operator_flops_per_tet": tet_flops_per_element(p), "l2_flushed": True,
            "roofline": {"bound": "fp64_tensor", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                         "frac": achieved / peak.value,
                         "peak_source": "hp_tet_fp64_mma_peak: mma.m8n8k4.f64 chains on every SM, measured in this run"}}
    g.close()
    # smoothing legs: the JACOBI build's update (finite-difference Jacobian diagonal,
    # omega 0.5) with the same boundary layout; cfl 0.5 on every level (the
    # reference's tet defaults 2.2 / 1.5 / 1.0 for p = 1 / 2 / 3 diverge with this smoother
    # at p >= 2)
    from hpb.tet import TetHierarchy
    cfl = {1: 0.5, 2: 0.5, 3: 0.5, 4: 0.5}
    small = 8
    ps = TetProblem(cube_tets(small), p, mu=1.0 / 100.0, cfl=cfl[p]).set_beltrami(re=100.0)
    masks, ff = ps.cube_boundary(re=100.0)
    gs = TetGPU(ps, device=dev, stream=ctypes.c_void_p(cur.cuda_stream))
    gs.set_dirichlet(masks)
    gs.set_flux_faces(ff)
    h, sec, nu = gs.solve(drop=1e-10, max_updates=20000, check_every=100)
    line["solve_single_grid_small"] = {"mesh": f"{small}^3 x 6", "ndof": ps.ndof, "seconds": sec, "updates": nu,
                                       "drop": float(h[-1]), "reached": bool(h[-1] <= 1e-10)}
    gs.close()
    H = TetHierarchy(small, p, hlevels=2, mu=1.0 / 100.0, cfl=cfl, stream=ctypes.c_void_p(cur.cuda_stream))
    h, sec, nc = H.solve(drop=1e-10, max_cycles=400, vw=1)
    line["solve_multigrid_small"] = {"mesh": f"{small}^3 x 6", "levels": f"p {p}..1, then {small // 2}^3, "
                                     f"{small // 4}^3 at p = 1", "seconds": sec, "cycles": nc,
                                     "drop": float(h[-1]), "reached": bool(h[-1] <= 1e-10)}
    H.close()
    H = TetHierarchy(n, p, hlevels=3, mu=1.0 / 100.0, cfl=cfl, stream=ctypes.c_void_p(cur.cuda_stream))
    ncyc = max(steps, 10)
    h, sec, nc = H.solve(drop=1e-10, max_cycles=ncyc, vw=1)
    line["multigrid_full"] = {"mesh": f"{n}^3 x 6", "levels": f"p {p}..1, then {n // 2}^3, {n // 4}^3, {n // 8}^3 "
                              "at p = 1", "seconds_incl_preconditioner_setup": sec, "cycles": nc,
                              "ms_per_cycle_incl_setup": 1e3 * sec / max(nc, 1), "drop": float(h[-1]),
                              "drop_history": [float(x) for x in h[::max(1, len(h) // 10)]]}
    if full_solve:
        # W-cycles (vwcycle 2) from the initial state on a hierarchy down to 2^3 x 6 for
        # n <= 32 and to 8^3 x 6 above (with more levels the W-cycle visits the coarsest
        # Jacobi-smoothed level 2^levels times per cycle, and at 64^3 down to 2^3 it diverged),
        # or `hlevels` h-levels
        H.close()
        ln = int(round(np.log2(n)))
        hl = hlevels or (max(1, ln - 1) if n <= 32 else max(1, ln - 3))
        # p1_minvrt: the p = 1 and 2 levels smoothed by the default build's tet_hp::minvrt at
        # the reference's cfl (2.2, 1.5) instead of the JACOBI build's relaxation; "all": every
        # level, the p = 3 level at its own cfl (1.0)
        cflw = {**cfl, **({1: 2.2, 2: 1.5} if p1_minvrt else {}), **({3: cfl3 or 1.0} if p1_minvrt == "all" else {})}
        arms = {}
        states = {}
        # the learned correction of the finest level's smoother, trained on the GPU on the
        # solver's own samples of 4 smaller instances (8^3 x 6, p, Beltrami at other Re)
        from hpb import learned as LR
        from hpb.tet import TetGPU
        t0 = _t.perf_counter()
        rng = np.random.default_rng(20261211)
        train_re = [float(x) for x in rng.uniform(40.0, 250.0, 4)]
        F, T = [], []
        for k, re in enumerate(train_re):
            def level(re=re, k=k):
                pr_ = TetProblem(cube_tets(8), p, mu=1.0 / re, cfl=cflw[p]).set_beltrami(re=re, seed=700 + k)
                mk_, ff_ = pr_.cube_boundary(re=re)
                g_ = TetGPU(pr_, stream=ctypes.c_void_p(cur.cuda_stream))
                g_.set_dirichlet(mk_)
                g_.set_flux_faces(ff_)
                if p1_minvrt == "all":
                    g_.set_smoother(1)
                return g_
            f, tg = LR.tet_solver_samples(level, snapshots=(0, 50, 200), jacobi=p1_minvrt != "all")
            F.append(f)
            T.append(tg)
        net, lh = LR.train(np.concatenate(F), np.concatenate(T), steps=400)
        arms["network"] = {"training_re": train_re, "samples": int(sum(len(t) for t in T)),
                           "nonzero_targets": float(np.mean(np.concatenate(T) != 0)),
                           "training_seconds": _t.perf_counter() - t0}
        for arm, mixed, learned in (("fp64", False, False), ("fp32_defect_correction", True, False),
                                    ("learned_fp32", True, True)):
            H = TetHierarchy(n, p, hlevels=hl, mu=1.0 / 100.0, cfl=cflw, stream=ctypes.c_void_p(cur.cuda_stream),
                             minvrt=p1_minvrt)
            if learned:
                H.levels[0].attach_net(net, 1.0)
            h, sec, nc = H.solve(drop=1e-10, max_cycles=400, vw=2, mixed=mixed)
            states[arm] = H.levels[0].state()
            arms[arm] = {"seconds": sec, "cycles": nc, "drop": float(h[-1]), "reached": bool(h[-1] <= 1e-10),
                         "ms_per_cycle": 1e3 * sec / max(nc, 1),
                         "drop_history": [float(x) for x in h[::max(1, len(h) // 10)]]}
            if arm != "fp64":
                a, b = states["fp64"], [x.copy() for x in states[arm]]
                b[0][:, 3] += np.mean(a[0][:, 3]) - np.mean(b[0][:, 3])  # free pressure level
                arms[arm]["rel_l2_state_diff_vs_fp64_modulo_pressure_level"] = float(
                    np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(a, b))) / np.sqrt(sum(np.sum(x * x) for x in a)))
            H.close()
            print(json.dumps({"c5_arm": arm, **arms[arm]}), flush=True)
        net.close()
        arms["speedup_fp32_vs_fp64"] = arms["fp64"]["seconds"] / arms["fp32_defect_correction"]["seconds"]
        arms["speedup_learned_fp32_vs_fp64"] = arms["fp64"]["seconds"] / arms["learned_fp32"]["seconds"]
        line["multigrid_full_w_to_1e-10"] = {"levels": f"p {p}..1, then h-levels down to {n >> hl}^3 at p = 1",
                                             "low_p_smoother": ("minvrt on every level (cfl 2.2, 1.5, 1.0)"
                                                                if p1_minvrt == "all" else
                                                                "minvrt (p = 1, 2; cfl 2.2, 1.5)" if p1_minvrt
                                                                else "jacobi, cfl 0.5"), **arms}
        H = TetHierarchy(n, p, hlevels=1, mu=1.0 / 100.0, cfl=cfl, stream=ctypes.c_void_p(cur.cuda_stream))
    H.close()
    # CPU oracle on a bounded sample
    ps = TetProblem(cube_tets(6), p, mu=1.0 / 100.0).set_beltrami(re=100.0)
    ff = ps.cube_boundary(re=100.0)[1]
    o = OracleTet(ps)
    o.set_flux_faces(ff)
    o.setup_preconditioner()
    reps, t2 = 0, _t.perf_counter()
    while _t.perf_counter() - t2 < 10.0:
        o.rsdl(ns)
        reps += 1
    cpu_s = (_t.perf_counter() - t2) / reps
    line["cpu_baseline"] = {"value": ps.ndof / cpu_s / 1e9, "unit": "GDoF/s", "cores": 1, "kind": "port",
                            "sample": f"oracle tet rsdl(nstage), 6^3 x 6 tetrahedra p={p}, {reps} repetitions"}
    print(json.dumps(line), flush=True)


def timed_factory(torch, flush):
    def timed(fn, n, stream):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]
    return timed


def c2_sweep(hpb, dev, n, ps, steps, timed):
    """cd, velocity (1, 0.5), kcond 1e-3, Dirichlet sin(pi x) sin(pi y) (so the converged
    state is 0; the initial state is that field projected plus 1e-3 noise) on the seeded
    Delaunay mesh delaunay_square(n) (n = 317: ~200k triangles, min angle >= 20 deg).
    Per p: FP64 rsdl GDoF/s matrix-free and from stored operators (with the operator
    kernel's HBM fraction), then time to a 1e-10 drop of the FP64 residual norm by V-cycles
    (p-levels p -> ... -> 1, then 4 Delaunay h-levels of n/2 .. n/16) for plain FP64
    (matrix-free), FP64 with stored operators and FP32 defect correction with stored
    operators, with the L2 difference of the converged states."""
    import ctypes as C
    import time as _t
    import numpy as np
    import torch
    from hpb import multigrid as MG
    from hpb._lib import check
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    meshes = {}

    def mesh(m):
        if m not in meshes:
            meshes[m] = hpb.delaunay_square(m, seed=20261205 + m)
        return meshes[m]

    def mk(n, p, **kw):
        return hpb.cd_sinsin(mesh=mesh(n), p=p, ax=1.0, ay=0.5, kcond=1e-3, noise=1e-3, seed=20261205, **kw)

    for p in ps:
        T = (p + 1) * (p + 2) // 2
        st = torch.cuda.Stream()
        pr = mk(n, p, cfl=CD_CFL[p])
        g = hpb.GPULevel(pr, device=dev, stream=C.c_void_p(st.cuda_stream))
        g.setup_preconditioner()
        ns = pr.phys.nstage
        rs = lambda: check(g.lib.hp_gpu_enqueue_rsdl(g.h, ns), "rsdl")
        el = lambda: check(g.lib.hp_gpu_enqueue_element_rsdl(g.h, ns), "element_rsdl")
        for _ in range(3):
            rs()
        mf = sum(timed(rs, steps, st)) / steps
        t0 = _t.perf_counter()
        g.element_matrices(True)
        build = _t.perf_counter() - t0
        for _ in range(3):
            rs()
        em = sum(timed(rs, steps, st)) / steps
        ek = sum(timed(el, steps, st)) / steps
        alg = pr.mesh.ntri * (2 * T * T + T) * 8 + 3 * pr.ndof * 8 + 36 * pr.mesh.ntri
        g.close()
        line = {"sweep": "c2", "p": p, "mesh": f"seeded Delaunay, {pr.mesh.ntri} triangles, min angle "
                                               f"{mesh(n).min_angle:.1f} deg", "ndof": pr.ndof,
                "rsdl_gdofs_matrix_free": pr.ndof / (mf * 1e-3) / 1e9, "rsdl_ms_matrix_free": mf,
                "rsdl_gdofs": pr.ndof / (em * 1e-3) / 1e9, "rsdl_ms": em, "operator_build_s": build,
                "k_rsdl_emat_ms": ek, "k_rsdl_emat_gbs": alg / (ek * 1e-3) / 1e9,
                "k_rsdl_emat_hbm_frac": alg / (ek * 1e-3) / 1e9 / hbm}
        states = {}
        for name, mixed, ops in (("fp64", False, False), ("fp64_elem_ops", False, True),
                                 ("fp32_defect_correction", True, True)):
            H = MG.build(mk, n=n, p=p, hlevels=4, cfl=CD_CFL)
            tb = 0.0
            if ops:
                t0 = _t.perf_counter()
                H.element_matrices(True)
                tb = _t.perf_counter() - t0
            hist, sec, cyc = H.solve(drop=1e-10, max_cycles=400, mixed=mixed, prcn_every=0)
            states[name] = H.levels[0].state()
            H.close()
            d = float(np.sqrt(sum(np.sum((a - b) ** 2) for a, b in zip(states["fp64"], states[name]))))
            line[name] = {"seconds": sec + tb, "solve_seconds": sec, "operator_build_seconds": tb, "cycles": cyc,
                          "final_drop": float(hist[-1]), "reached": bool(hist[-1] <= 1e-10),
                          "l2_coeff_diff_vs_fp64": d}
        line["state_l2_fp64"] = float(np.sqrt(sum(np.sum(a * a) for a in states["fp64"])))
        line["speedup_fp32_vs_fp64"] = line["fp64"]["seconds"] / line["fp32_defect_correction"]["seconds"]
        print(json.dumps(line), flush=True)


def _rel(a, b):
    import numpy as np
    return float(np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(a, b))) / np.sqrt(sum(np.sum(x * x) for x in a)))


def _rel_ins_modulo_pressure_level(a, b):
    """Relative L2 difference of two ins states (v, s, i arrays, variables u, v, p last) after
    removing the difference of their mean vertex pressure: with velocity given on every wall
    the pressure is fixed only up to a constant (a constant is the vertex modes alone)."""
    import numpy as np
    b = [x.copy() for x in b]
    b[0][:, 2] += np.mean(a[0][:, 2]) - np.mean(b[0][:, 2])
    return _rel(a, b)


def time_to_tolerance(hpb, dev):
    """Time to a 1e-10 drop of the FP64 residual norm (Dirichlet rows excluded) on cd p=4
    with Dirichlet data -(x-8)^2, velocity (1,0.5), kcond 1e-3, noise 1e-3. `seconds` is
    the device time of the whole solve (preconditioner set-up and residual checks
    included) plus, for the arms with stored element operators, the wall time of their
    one-time build (allocation included). Arms: plain FP64 (matrix-free element kernel, the reference's algorithm),
    FP64 with stored element operators, FP32 correction smoothing inside FP64 defect
    correction (stored operators), and that plus the learned preconditioner correction.
    Two drivers: single-grid smoothing on a 64x64 split-square mesh, and V-cycles
    (p 4 -> 2 -> 1, then 4 h-levels) on a 320x320 mesh (204,800 triangles)."""
    import ctypes as C
    import time as _t
    import numpy as np
    from hpb import _lib as L
    from hpb import learned as LR
    from hpb import multigrid as MG

    def field():
        return L.Field(L.HP_FIELD_QUADX, (C.c_double * 4)(-1.0, 8.0, 0, 0))

    # the network: trained on the GPU from the solver's own residual histories of 4
    # other instances of the same family (random velocity and diffusivity)
    t0 = _t.perf_counter()
    F, T = [], []
    for s in range(4):
        r = np.random.default_rng(300 + s)
        ax, ay = r.uniform(-1, 1, 2)
        kc = 10 ** r.uniform(-3, -1.5)
        fs, ts = LR.solver_samples(lambda: hpb.cd_sinsin(n=TOL_N, p=P, ax=ax, ay=ay, kcond=kc, cfl=0.5,
                                                         field=field(), noise=1e-3, seed=300 + s))
        F.append(fs)
        T.append(ts)
    net, _ = LR.train(np.concatenate(F), np.concatenate(T), steps=400)
    train_s = _t.perf_counter() - t0

    arms = (("fp64", False, False, False), ("fp64_elem_ops", False, True, False),
            ("fp32_defect_correction", True, True, False), ("learned_fp32", True, True, True))
    out = {"drop": 1e-10, "criterion": "||R64||_2 / ||R64(u0)||_2 over all non-Dirichlet v/s/i rows",
           "network": {"widths": "17-64-64-64-1", "dtype": "BF16 weights, FP32 accumulation",
                       "training": "400 Adam steps on the GPU, 4 solver-generated instances",
                       "training_seconds_offline": train_s}}
    sg = {"workload": f"single grid: cd p={P}, {TOL_N}x{TOL_N} split-square mesh ({2 * TOL_N * TOL_N} triangles), "
                      "cfl 0.5, 20 updates per defect-correction cycle"}
    states = {}
    for name, mixed, em, learned in arms:
        g = hpb.cd_sinsin(n=TOL_N, p=P, kcond=1e-3, cfl=0.5, field=field(), noise=1e-3, seed=20261205).gpu(device=dev)
        tb = 0.0
        if em:
            t0 = _t.perf_counter()
            g.element_matrices(True)
            tb = _t.perf_counter() - t0
        if learned:
            LR.attach(g, net, 1.0)
        hist, sec, upd = g.solve(mixed=mixed, drop=1e-10, max_updates=20000, inner=20, check_every=20)
        states[name] = g.state()
        sg[name] = {"seconds": sec + tb, "solve_seconds": sec, "operator_build_seconds": tb, "updates": upd,
                    "final_drop": float(hist[-1]), "reached": bool(hist[-1] <= 1e-10),
                    "rel_l2_state_diff_vs_fp64": _rel(states["fp64"], states[name])}
        g.close()
    sg["speedup_learned_fp32_vs_fp64"] = sg["fp64"]["seconds"] / sg["learned_fp32"]["seconds"]
    sg["speedup_learned_fp32_vs_fp64_elem_ops"] = sg["fp64_elem_ops"]["seconds"] / sg["learned_fp32"]["seconds"]
    out["single_grid"] = sg

    mg = {"workload": f"multigrid: cd p={P}, {MG_N}x{MG_N} split-square mesh ({2 * MG_N * MG_N} triangles), levels "
                      f"p=4,2,1 then h-levels {MG_N // 2},{MG_N // 4},{MG_N // 8},{MG_N // 16} at p=1, V-cycle with "
                      "2+2 updates per level, cfl 0.5/0.75/1.0 for p=4/2/1; learned correction on the finest level"}
    mk = lambda n, p, **kw: hpb.cd_sinsin(n=n, p=p, kcond=1e-3, field=field(), **kw)
    states = {}
    for name, mixed, em, learned in arms:
        H = MG.build(mk, n=MG_N, p=P, hlevels=4, cfl={4: 0.5, 2: 0.75, 1: 1.0})
        tb = 0.0
        if em:
            t0 = _t.perf_counter()
            H.element_matrices(True)
            tb = _t.perf_counter() - t0
        if learned:
            LR.attach(H.levels[0], net, 1.0)
        # cd preconditioners do not depend on the state: evaluated once (the learned
        # correction sees the initial state, as in its training data)
        hist, sec, cyc = H.solve(drop=1e-10, max_cycles=400, mixed=mixed, prcn_every=0)
        states[name] = H.levels[0].state()
        mg[name] = {"seconds": sec + tb, "solve_seconds": sec, "operator_build_seconds": tb, "cycles": cyc,
                    "final_drop": float(hist[-1]), "reached": bool(hist[-1] <= 1e-10),
                    "rel_l2_state_diff_vs_fp64": _rel(states["fp64"], states[name])}
        H.close()
    mg["speedup_learned_fp32_vs_fp64"] = mg["fp64"]["seconds"] / mg["learned_fp32"]["seconds"]
    mg["speedup_learned_fp32_vs_fp64_elem_ops"] = mg["fp64_elem_ops"]["seconds"] / mg["learned_fp32"]["seconds"]
    out["multigrid"] = mg
    net.close()
    return out


def kernel_sweep(hpb, dev, n, ps, steps, timed, stream):
    """FP64 element-kernel time per p on the lid cavity (n x n split squares): the tensor-core
    (DMMA) and the scalar warp kernel, with the algorithmic flop rate (oracle op count) and
    the FP64 tensor-core peak measured in the same run."""
    from hpb._lib import check
    peak = ctypes.c_double()
    lib = hpb._lib.lib()
    lib.hp_tet_fp64_mma_peak.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    check(lib.hp_tet_fp64_mma_peak(dev, 200.0, ctypes.byref(peak)), "fp64 mma peak")
    for p in ps:
        pr = hpb.lid_cavity_ins(n=n, p=p, re=C3_RE)
        g = hpb.GPULevel(pr, device=dev, stream=ctypes.c_void_p(stream.cuda_stream))
        g.setup_preconditioner()
        ns = pr.phys.nstage
        fl_el, src = ins_flops_per_element(p)
        line = {"sweep": "kernels", "p": p, "ntri": pr.mesh.ntri, "ndof": pr.ndof, "flops_per_element": fl_el,
                "fp64_tensor_peak_tflops": peak.value}
        for kind in ("tensor", "scalar") + (("point",) if p == 1 else ()):
            g.element_kernel(kind)
            el = lambda: check(lib.hp_gpu_enqueue_element_rsdl(g.h, ns), "element_rsdl")
            rs = lambda: check(lib.hp_gpu_enqueue_rsdl(g.h, ns), "rsdl")
            for _ in range(3):
                rs()
            k_ms = sum(timed(el, steps, stream)) / steps
            r_ms = sum(timed(rs, steps, stream)) / steps
            tf = fl_el * pr.mesh.ntri / (k_ms * 1e-3) / 1e12
            line[kind] = {"kernel_ms": k_ms, "rsdl_ms": r_ms, "rsdl_gdofs": pr.ndof / (r_ms * 1e-3) / 1e9,
                          "tflops": tf, "frac_of_fp64_tensor_peak": tf / peak.value}
        line["speedup_tensor_vs_scalar"] = line["scalar"]["kernel_ms"] / line["tensor"]["kernel_ms"]
        if "point" in line:
            line["speedup_point_vs_scalar"] = line["scalar"]["kernel_ms"] / line["point"]["kernel_ms"]
        g.close()
        print(json.dumps(line), flush=True)


def c3_time_to_tol(hpb, dev, stream, max_cycles=150, snapshots=(0,)):
    """C3 W-cycles (vwcycle 2, 2 + 2 updates per level, preconditioners every cycle) from
    the initial state to a 1e-10 drop of the FP64 residual: plain FP64, FP32 smoothing
    inside FP64 defect correction, and that plus the learned correction of the Jacobi
    blocks on the fine level. The network is trained on the GPU on solver-generated
    samples of 4 lid-cavity instances at other Reynolds numbers (64 x 64 squares, p = 6)."""
    import numpy as np
    from hpb import learned as LR
    from hpb import multigrid as MG
    t0 = time.perf_counter()
    rng = np.random.default_rng(20261210)
    train_re = [float(x) for x in rng.uniform(100.0, 1000.0, 4)]
    F, T = [], []
    for k, re in enumerate(train_re):
        f, tg = LR.solver_samples(lambda: hpb.lid_cavity_ins(n=64, p=C3_P, re=re, seed=500 + k), snapshots=snapshots)
        F.append(f)
        T.append(tg)
    net, lh = LR.train(np.concatenate(F), np.concatenate(T), steps=400)
    out = {"drop": 1e-10, "criterion": "||R64||_2 / ||R64(u0)||_2 over all non-Dirichlet v/s/i rows",
           "cycle": "W (vwcycle 2), 2+2 multistage updates per level, preconditioners every cycle",
           "network": {"widths": "17-64-64-64-1", "dtype": "BF16 weights, FP32 accumulation",
                       "training_re": train_re, "samples": int(sum(len(t) for t in T)), "snapshots": list(snapshots),
                       "nonzero_targets": float(np.mean(np.concatenate(T) != 0)),
                       "training_seconds": time.perf_counter() - t0}}
    states = {}
    for name, mixed, learned in (("fp64", False, False), ("fp32_defect_correction", True, False),
                                 ("learned_fp32", True, True)):
        H = MG.build(c3_factory, n=C3_N, p=C3_P, hlevels=3, stream=ctypes.c_void_p(stream.cuda_stream))
        if learned:
            LR.attach(H.levels[0], net, 1.0)
        hist, sec, cyc = H.solve(drop=1e-10, max_cycles=max_cycles, vw=2, mixed=mixed, prcn_every=1)
        states[name] = H.levels[0].state()
        out[name] = {"seconds": sec, "cycles": cyc, "ms_per_cycle": 1e3 * sec / max(cyc, 1),
                     "drop": float(hist[-1]), "reached": bool(hist[-1] <= 1e-10),
                     "rel_l2_state_diff_vs_fp64_modulo_pressure_level":
                         _rel_ins_modulo_pressure_level(states["fp64"], states[name])}
        H.close()
    net.close()
    out["speedup_learned_fp32_vs_fp64"] = out["fp64"]["seconds"] / out["learned_fp32"]["seconds"]
    out["speedup_fp32_vs_fp64"] = out["fp64"]["seconds"] / out["fp32_defect_correction"]["seconds"]
    return out


def c3_headline(args, torch, dist, rank, world, dev, stream):
    import numpy as np
    import hpb
    from hpb import multigrid as MG
    from hpb._lib import check
    t0 = time.perf_counter()
    H = MG.build(c3_factory, n=C3_N, p=C3_P, hlevels=3, stream=ctypes.c_void_p(stream.cuda_stream))
    setup_s = time.perf_counter() - t0
    fine, pr = H.levels[0], H.probs[0]
    lib = fine.lib
    ns = pr.phys.nstage
    if args.elem:
        fine.element_kernel(args.elem)
    check(lib.hp_gpu_setup_preconditioner(fine.h), "setup_preconditioner")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    timed = timed_factory(torch, flush)
    rsdl = lambda: check(lib.hp_gpu_enqueue_rsdl(fine.h, ns), "rsdl")
    elem = lambda: check(lib.hp_gpu_enqueue_element_rsdl(fine.h, ns), "element_rsdl")
    for _ in range(max(3, args.warmup)):
        rsdl()
    torch.cuda.synchronize()
    clk_file = os.path.join(ROOT, f"_clocks_{rank}.csv")
    clk = sample_clocks(None, clk_file)
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = timed(rsdl, args.steps, stream)
    if dist:
        dist.barrier()
    t_ms = sum(step_ms)
    k_ms = sum(timed(elem, args.steps, stream)) / args.steps
    if clk:
        clk.terminate()
        clk.wait()
    clocks = parse_clocks(clk_file, dev)
    try:
        os.remove(clk_file)
    except OSError:
        pass
    peak = ctypes.c_double()
    lib.hp_tet_fp64_mma_peak.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    check(lib.hp_tet_fp64_mma_peak(dev, 200.0, ctypes.byref(peak)), "fp64 mma peak")
    # e2e through the C-ABI with host buffers (pinned): every step uploads its state from the
    # host, evaluates rsdl(nstage) and downloads the residual to the host. Two contexts of the
    # fine level on two streams alternate, so that one step's copies (the two copy engines,
    # host to device and device to host) overlap the neighbouring steps' kernels; a step's
    # buffers are reused only after hp_gpu_sync of that context. The serial form (upload,
    # rsdl, download, wait) is reported beside it.
    P_ = hpb._lib.ptr
    bufs = []
    for _ in range(2):
        hv, hs, hi, rv, rs, ri = (torch.empty(a.shape, dtype=torch.float64, pin_memory=True).numpy()
                                  for a in (pr.ugv, pr.ugs, pr.ugi) * 2)
        hv[...] = pr.ugv; hs[...] = pr.ugs; hi[...] = pr.ugi
        bufs.append((hv, hs, hi, rv, rs, ri))
    stream2 = torch.cuda.Stream()
    fine2 = hpb.GPULevel(pr, device=dev, stream=ctypes.c_void_p(stream2.cuda_stream))
    assert fine2.setup_preconditioner() == 0
    ctxs = (fine, fine2)
    e2e_steps = max(4, min(args.steps, 12))

    def e2e_run(pipelined):
        for k in range(e2e_steps + 2):
            if k == 2:
                for c in ctxs:
                    check(lib.hp_gpu_sync(c.h), "sync")
                t0 = time.perf_counter()
            c = ctxs[k % 2] if pipelined else fine
            hv, hs, hi, rv, rs, ri = bufs[k % 2]
            if pipelined:
                check(lib.hp_gpu_sync(c.h), "sync")  # this context's previous step is done
            check(lib.hp_gpu_enqueue_upload_state(c.h, P_(hv), P_(hs), P_(hi)), "upload")
            check(lib.hp_gpu_enqueue_rsdl(c.h, ns), "rsdl")
            check(lib.hp_gpu_enqueue_download_residual(c.h, P_(rv), P_(rs), P_(ri)), "download")
            if not pipelined:
                check(lib.hp_gpu_sync(c.h), "sync")
        for c in ctxs:
            check(lib.hp_gpu_sync(c.h), "sync")
        return (time.perf_counter() - t0) / e2e_steps

    e2e_serial_s = e2e_run(False)
    e2e_s = e2e_run(True)
    fine2.close()
    io_bytes = hv.nbytes + hs.nbytes + hi.nbytes
    m = pr.mesh
    ndof = pr.ndof
    H.close()
    value, e2e, t_ms, e2e_s = replica_totals(dist, world, ndof, args.steps, t_ms, e2e_s, "cuda")
    tol = c3_time_to_tol(hpb, dev, stream, snapshots=tuple(args.c3_snapshots)) if (world == 1 and not args.no_tol) else None
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    fl_el, fl_src = ins_flops_per_element(C3_P)
    fl = fl_el * m.ntri
    achieved = fl / (k_ms * 1e-3) / 1e12
    comp_bytes = 16 * ndof + 36 * m.ntri + 16 * m.npnt
    peaks = load_peaks()
    hbm = peaks.get("hbm_gbs")
    hbm_src = "MEASURED_PEAKS.json hbm_gbs (measured)"
    if hbm is None:
        hbm, hbm_src = 6650.0, "fallback 6.65 TB/s (no measured peak file)"
    traffic = None
    try:  # DRAM bytes per triangle of the element kernel from an ncu capture, scaled to this launch
        tr = json.load(open(os.path.join(ROOT, "profiles", "k_rsdl_elem_ins_p6_traffic.json")))
        traffic = tr["dram_bytes_per_triangle"] * m.ntri
    except Exception:
        pass
    cpu = None
    if world == 1:
        cv, reps = run_cpu_strips(1, 0, 1, secs=10.0)
        cpu = {"value": cv, "unit": "GDoF/s", "cores": 1, "kind": "port",
               "sample": f"oracle rsdl(nstage) on a 512 x {STRIP_ROWS}-square strip of the C3 mesh "
                         f"({2 * C3_N * STRIP_ROWS} triangles, p={C3_P}, lid-cavity state), {reps} evaluations "
                         "in 10 s, 1 core"}
    # element kernel (k_rsdl_ins_mma or k_rsdl_elem), k_bdry_flux_ins, k_assemble, and the k_rsdl_fold
    # that hp_gpu_enqueue_rsdl adds (res += res_r for the caller, nstage.cpp:76-82)
    launches_per_step = 4
    line = {
        "metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": c3_config(),
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                     "frac": achieved / peak.value, "traffic": traffic, "kernel": "element residual (fine level)",
                     "kernel_ms": k_ms, "flops_per_element": fl_el, "flops_source": fl_src,
                     "peak_source": "FP64 tensor-core (DMMA) rate measured in this run by hp_tet_fp64_mma_peak "
                                    "(MEASURED_PEAKS.json has no FP64 figure)",
                     "hbm": {"compulsory_bytes": comp_bytes, "achieved_gbs": comp_bytes / (k_ms * 1e-3) / 1e9,
                             "peak_gbs": hbm, "frac": comp_bytes / (k_ms * 1e-3) / 1e9 / hbm,
                             "peak_source": hbm_src,
                             "bytes": "16 NDOF + 36 ntri + 16 npnt (state read, residual written, "
                                      "connectivity, coordinates)"}},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "GDoF/s", "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes,
                "steps": "pinned host state -> hp_gpu_enqueue_upload_state, hp_gpu_enqueue_rsdl(nstage), "
                         "hp_gpu_enqueue_download_residual -> pinned host residual; two contexts on two streams "
                         "alternate so that copies overlap the other step's kernels",
                "serial_value": world * ndof / e2e_serial_s / 1e9},
        "gpu_launches": launches_per_step * args.steps,
        "time_to_tol": tol, "ndof": ndof, "host_setup_seconds": setup_s, "clocks": clocks,
        "element_kernel": args.elem or "tensor",
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", choices=["c3", "cd"], default="c3",
                    help="c3 (default): the C3 ins p = 6 line; cd: the cd p = 4 line with stored element operators")
    ap.add_argument("--no-tol", action="store_true", help="skip the time-to-tolerance legs (profiling runs)")
    ap.add_argument("--elem", choices=["tensor", "scalar"], default=None,
                    help="FP64 ins element kernel of the timed fine level (default: the library's, tensor)")
    ap.add_argument("--mesh", type=int, default=N_MESH,
                    help="split-square mesh size n (2 n^2 triangles); smaller cases are for profiler runs")
    ap.add_argument("--quick", action="store_true",
                    help="device-timed rsdl steps only (no e2e, update or CPU legs); for profiler runs")
    ap.add_argument("--physics", choices=["cd", "ins"], default="cd",
                    help="with --quick / --profile: ins runs the Kovasznay workload (Re 100, p = 4) on the "
                         "--mesh split-square mesh with the matrix-free ins element kernel")
    ap.add_argument("--matrix-free", action="store_true",
                    help="with --quick / --profile: the matrix-free element kernel instead of stored operators")
    ap.add_argument("--profile", choices=["update64", "update32"], default=None,
                    help="run `steps` multistage updates of the workload in FP64 or FP32 (for profiler runs)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="with --sweep c4: edge-length scale of the channel mesh (1: ~150k triangles)")
    ap.add_argument("--sweep", choices=["c2", "c3", "c4", "c5", "kernels"], default=None,
                    help="c2: cd on the seeded 200k-triangle Delaunay mesh, p = 2, 4, 6, 8: rsdl GDoF/s and time "
                         "to a 1e-10 drop, plain FP64 vs FP32 defect correction (one JSON line per p); "
                         "c3: ins lid-driven cavity Re 400, p = 6, 512x512 split squares, V-cycles for --steps "
                         "cycles: level by level, one CUDA graph, autotuned graph, FP32 defect correction; "
                         "c4: ins past a cylinder in a channel (curved hole, graded ~150k triangles), learned "
                         "preconditioner trained on Re in [20, 200], judged on held-out Re by the FP64 residual")
    ap.add_argument("--p", type=int, nargs="*", default=None, help="with --sweep: the p values")
    ap.add_argument("--arms", nargs="*", default=None,
                    help="with --sweep c3: run only these arms (e.g. fp64_level_by_level fp32_defect_correction)")
    ap.add_argument("--tet-minvrt", action="store_true",
                    help="with --sweep c5 --tet-solve: smooth the p = 1, 2 levels with tet_hp::minvrt (cfl 2.2, 1.5)")
    ap.add_argument("--tet-minvrt-all", action="store_true",
                    help="with --sweep c5 --tet-solve: smooth every level with tet_hp::minvrt (cfl 2.2, 1.5, 1.0)")
    ap.add_argument("--c3-snapshots", type=int, nargs="*", default=[0],
                    help="plain-update counts of the states the C3 network's training samples come from")
    ap.add_argument("--tet-cfl3", type=float, default=None,
                    help="with --tet-minvrt-all: the cfl of the p = 3 level (default 1.0, the reference's)")
    ap.add_argument("--tet-hlevels", type=int, default=None,
                    help="with --sweep c5 --tet-solve: h-levels of the W-cycle hierarchy (default: down to 2^3 "
                         "for n <= 32, to 8^3 above)")
    ap.add_argument("--tet-solve", action="store_true",
                    help="with --sweep c5: also W-cycles on the full hierarchy to a 1e-10 drop (minutes)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        cores = os.cpu_count() or 1
        if args.workload == "cd":
            v, n = run_cpu(cores, 10.0)
            line = {"impl": "reference", "metric": METRIC_CD, "value": v, "unit": "GDoF/s", "n_gpus": args.gpus,
                    "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(),
                    "cpu_baseline": {"value": v, "unit": "GDoF/s", "cores": cores, "kind": "port",
                                     "sample": f"oracle rsdl(nstage) on a {n}x{n} split-square mesh, p={P}, "
                                               "10 s per core, one process per core"},
                    "e2e": {"value": v, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line))
            return
        v, reps = run_cpu_strips(cores, args.steps, args.warmup)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GDoF/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": c3_config(),
                "cpu_baseline": {"value": v, "unit": "GDoF/s", "cores": cores, "kind": "port",
                                 "sample": f"each step: the oracle's rsdl(nstage) on {cores} strips of the C3 mesh "
                                           f"at once (512 x {STRIP_ROWS} squares, {2 * C3_N * STRIP_ROWS} triangles, "
                                           f"p={C3_P}, lid-cavity state), one process per core"},
                "e2e": {"value": v, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import numpy as np
    import torch
    import hpb
    from hpb._lib import check

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()  # a non-default stream: the update graph is captured on it
    torch.cuda.set_stream(stream)

    if args.sweep is None and args.workload == "c3" and not (args.quick or args.profile):
        c3_headline(args, torch, dist, rank, world, dev, stream)
        return
    if args.sweep == "kernels":
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        kernel_sweep(hpb, dev, args.mesh if args.mesh != N_MESH else 256, args.p or list(range(1, 9)), args.steps,
                     timed_factory(torch, flush), stream)
        return
    if args.sweep == "c2":
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        c2_sweep(hpb, dev, args.mesh, args.p or [2, 4, 6, 8], args.steps, timed_factory(torch, flush))
        return
    if args.sweep == "c4":
        c4_sweep(hpb, dev, args.scale, args.steps)
        return
    if args.sweep == "c3":
        c3_sweep(hpb, dev, args.mesh if args.mesh != N_MESH else 512, (args.p or [6])[0], args.steps, arms=args.arms)
        return
    if args.sweep == "c5":
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        c5_sweep(torch, dev, args.mesh if args.mesh != N_MESH else 64, (args.p or [3])[0], args.steps, args.warmup,
                 timed_factory(torch, flush), full_solve=args.tet_solve, hlevels=args.tet_hlevels,
                 p1_minvrt="all" if args.tet_minvrt_all else args.tet_minvrt, cfl3=args.tet_cfl3)
        return

    if args.physics == "ins":
        if not (args.quick or args.profile):
            raise SystemExit("--physics ins is for --quick / --profile runs")
        pr = hpb.kovasznay_ins(n=args.mesh, p=P, re=100.0)
    else:
        pr = hpb.cd_sinsin(n=args.mesh, p=P, ax=1.0, ay=0.5, kcond=1e-3, noise=1e-3, seed=20261205)
    lvl = hpb.GPULevel(pr, device=dev, stream=ctypes.c_void_p(stream.cuda_stream))
    lib = lvl.lib
    rc = lvl.setup_preconditioner()
    assert rc == 0
    ns = pr.phys.nstage
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(fn, n):
        """Device ms of each of n calls of fn on the bench stream, L2 flushed before each."""
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    def rsdl():
        check(lib.hp_gpu_enqueue_rsdl(lvl.h, ns), "rsdl")

    def elem():
        check(lib.hp_gpu_enqueue_element_rsdl(lvl.h, ns), "element_rsdl")

    def update():
        check(lib.hp_gpu_enqueue_update(lvl.h), "update")

    if args.profile or args.quick:
        if not args.matrix_free and args.physics == "cd":
            lvl.element_matrices(True)
        if args.profile:
            for k in range(args.warmup + args.steps):
                if args.profile == "update64":
                    update()
                else:
                    check(lib.hp_gpu_fp32_updates(lvl.h, 1), "fp32 update")
            torch.cuda.synchronize()
            print(json.dumps({"profile": args.profile, "updates": args.warmup + args.steps}))
        else:
            for _ in range(max(3, args.warmup)):
                rsdl()
            ms = timed(rsdl, args.steps)
            print(json.dumps({"quick": True, "matrix_free": args.matrix_free or args.physics == "ins", "ntri": pr.mesh.ntri,
                              "ms_per_step": sum(ms) / args.steps,
                              "value": pr.ndof * args.steps / (sum(ms) * 1e-3) / 1e9}))
        lvl.close()
        return

    # matrix-free element kernel (the reference's per-call element_rsdl), for comparison
    for _ in range(3):
        rsdl()
    torch.cuda.synchronize()
    mf_ms = sum(timed(rsdl, args.steps)) / args.steps
    mf_k = sum(timed(elem, args.steps)) / args.steps
    mf_u = sum(timed(update, args.steps)) / args.steps

    # stored element operators: built once, then every rsdl is a streamed batched mat-vec
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lvl.element_matrices(True)
    build_ms = (time.perf_counter() - t0) * 1e3
    for _ in range(max(3, args.warmup)):
        rsdl()
    torch.cuda.synchronize()

    clk_file = os.path.join(ROOT, f"_clocks_{rank}.csv")
    clk = sample_clocks(None, clk_file)
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = timed(rsdl, args.steps)
    if dist:
        dist.barrier()
    t_ms = sum(step_ms)
    # the dominant kernel alone (k_rsdl_emat) for the roofline
    k_ms = sum(timed(elem, args.steps)) / args.steps
    # one multistage update (nstage x (rsdl + minvrt + ug update)), FP64 and FP32
    u_ms = sum(timed(update, args.steps)) / args.steps
    check(lib.hp_gpu_fp32_updates(lvl.h, 10), "fp32 updates")  # FP32 buffers and graph outside the timing
    u32_ms = sum(timed(lambda: check(lib.hp_gpu_fp32_updates(lvl.h, 10), "fp32 updates"), 3)) / 30
    if clk:
        clk.terminate()
        clk.wait()
    clocks = parse_clocks(clk_file, dev)
    try:
        os.remove(clk_file)
    except OSError:
        pass
    # e2e through the C-ABI with host buffers (pinned)
    hv = torch.empty(pr.ugv.shape, dtype=torch.float64, pin_memory=True).numpy()
    hs = torch.empty(pr.ugs.shape, dtype=torch.float64, pin_memory=True).numpy()
    hi = torch.empty(pr.ugi.shape, dtype=torch.float64, pin_memory=True).numpy()
    hv[...] = pr.ugv; hs[...] = pr.ugs; hi[...] = pr.ugi
    rv = torch.empty(pr.ugv.shape, dtype=torch.float64, pin_memory=True).numpy()
    rs = torch.empty(pr.ugs.shape, dtype=torch.float64, pin_memory=True).numpy()
    ri = torch.empty(pr.ugi.shape, dtype=torch.float64, pin_memory=True).numpy()
    P_ = hpb._lib.ptr
    for _ in range(2):
        lib.hp_gpu_upload_state(lvl.h, P_(hv), P_(hs), P_(hi))
        lib.hp_gpu_rsdl(lvl.h, ns, 0)
        lib.hp_gpu_download_residual(lvl.h, P_(rv), P_(rs), P_(ri))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        hpb._lib.check(lib.hp_gpu_upload_state(lvl.h, P_(hv), P_(hs), P_(hi)), "upload")
        hpb._lib.check(lib.hp_gpu_rsdl(lvl.h, ns, 0), "rsdl")
        hpb._lib.check(lib.hp_gpu_download_residual(lvl.h, P_(rv), P_(rs), P_(ri)), "download")
    e2e_s = (time.perf_counter() - t0) / args.steps
    io_bytes = hv.nbytes + hs.nbytes + hi.nbytes

    ndof = pr.ndof
    m = pr.mesh
    T = (P + 1) * (P + 2) // 2
    tol = time_to_tolerance(hpb, dev)
    value, e2e, t_ms, e2e_s = replica_totals(dist, world, ndof, args.steps, t_ms, e2e_s, "cuda")
    # algorithmic bytes of one k_rsdl_emat launch at beta = 1: both element operators and
    # b_re (ntri (2 T^2 + T) FP64), the state read once, res and res_r written once, and
    # the element connectivity (tri_pnt, tri_seg, tri_sgn: 9 int32 per triangle)
    op_bytes = m.ntri * (2 * T * T + T) * 8
    alg_bytes = op_bytes + 3 * ndof * 8 + 36 * m.ntri
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_source = "MEASURED_PEAKS.json hbm_gbs (measured)"
    if hbm is None:
        hbm, peak_source = 6650.0, "fallback 6.65 TB/s (no measured peak file)"
    achieved = alg_bytes / (k_ms * 1e-3) / 1e9
    traffic = None
    try:  # DRAM bytes per triangle of k_rsdl_emat from an ncu capture, scaled to this launch
        tr = json.load(open(os.path.join(ROOT, "profiles", "k_rsdl_emat_cd_p4_traffic.json")))
        traffic = tr["dram_bytes_per_triangle"] * m.ntri
    except Exception:
        pass
    fl = flops_per_element(P) * m.ntri
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    cpu = None
    if world == 1:
        cv, n = run_cpu(1, 10.0)
        cpu = {"value": cv, "unit": "GDoF/s", "cores": 1, "kind": "port",
               "sample": f"oracle rsdl(nstage) on a {n}x{n} split-square mesh, p={P}, 10 s, 1 core"}
    launches_per_step = 3  # k_rsdl_pre, k_rsdl_emat, k_rsdl_fold (cd has no boundary-flux kernel)
    cfg = workload_config()
    cfg["element_operators"] = ("stored: built once by the element kernel on unit vectors "
                                f"({build_ms:.1f} ms, {2 * op_bytes / 1e9:.2f} GB FP64 + FP32 copy), "
                                "outside the timed steps")
    line = {
        "metric": METRIC_CD, "value": value, "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "kernel": "k_rsdl_emat<double,4,beta>0>", "kernel_ms": k_ms,
                     "algorithmic_bytes": alg_bytes, "peak_source": peak_source},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "GDoF/s", "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
        "gpu_launches": launches_per_step * args.steps,
        "elem_operator_build_ms": build_ms,
        "update_ms": u_ms, "update_gdofs_per_stage": ndof * ns / (u_ms * 1e-3) / 1e9,
        "fp32_update_ms": u32_ms,
        "matrix_free": {"value": ndof / (mf_ms * 1e-3) / 1e9, "ms_per_step": mf_ms, "kernel": "k_rsdl_elem",
                        "kernel_ms": mf_k, "fp64_tflops": fl / (mf_k * 1e-3) / 1e12, "flops_per_launch": fl,
                        "update_ms": mf_u},
        "time_to_tol": tol,
        "ndof": ndof, "clocks": clocks,
    }
    print(json.dumps(line))
    lvl.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
