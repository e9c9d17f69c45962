#!/usr/bin/env python3
"""Benchmark of the B200 epsilon-div-div operator apply (TerraNeo hot path).

Workload (one "step"): one FP64 EpsilonDivDivKerngen apply, Dirichlet on both
radii, Replace mode with the additive inter-diamond halo, on the level-6 thick
shell r in [0.55, 1] (10 diamonds x 64 x 64 x 64 cells, 2,746,250 stored nodes,
7,987,590 velocity DoFs), viscosity k = exp(ln(1e4) (0.5 radial ramp + 0.5
Gaussian-blob field)) clamped to contrast 1e4, src ~ N(0,1) made consistent on
duplicated nodes.  GDoF/s = unique velocity DoFs / time per apply, the
reference's definition (apps/benchmarks/performance/benchmark_operators.cpp:208).

Inputs rotate over 4 (src, dst) buffer sets (4 x 132 MB > 126 MB L2) so no
step reads data cached by the previous one.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 (torchrun) every rank runs the same apply on its own GPU (replicas:
the ten diamonds of one level-6 shell fit one GPU, so the headline apply is
not sharded), timed with CUDA events, max over ranks; value is the aggregate
over ranks. The `sharded` object of the line (always with two or more ranks,
with --sharded on one) times the level-7 apply with the shell split over the
ranks by diamond and one all-reduce of the shared copies per apply.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "L6 Stokes time-to-1e-8 (FP32-MG+FP64 refine vs FP64); apply GDoF/s, %HBM"
LEVEL, RMIN, RMAX = 6, 0.55, 1.0
BYTES_PER_NODE_F64 = 56  # 3 src + 1 k + 3 dst doubles per stored node
BYTES_PER_NODE_F32 = 28
# DRAM bytes (read + write) of one level-6 kerngen_tile_kernel<double, 16> launch,
# from an ncu capture (profiles/kerngen_tile_kernel_f64_L6_dirichlet.md)
TILE_TRAFFIC_BYTES = 141426176 + 43898112


def _case_laplace6(shell, C, torch):
    m = shell.ShellMesh(6, RMIN, RMAX)
    s, d = shell.VectorQ1Scalar(m), shell.VectorQ1Scalar(m)
    s.data.uniform_(-1, 1)
    op = shell.Laplace(m, True)
    return {"Laplace apply, level 6, Dirichlet elimination": lambda: shell.apply(op, s, d)}


def _case_vlaplace6(shell, C, torch):
    m = shell.ShellMesh(6, RMIN, RMAX)
    u, v = shell.VectorQ1Vec(m), shell.VectorQ1Vec(m)
    u.data.uniform_(-1, 1)
    op = shell.VectorLaplace(m, C.BC_DIRICHLET, C.BC_DIRICHLET)
    return {"VectorLaplace apply, level 6, Dirichlet": lambda: shell.apply(op, u, v)}


def _case_divkgrad6(shell, C, torch):
    m = shell.ShellMesh(6, RMIN, RMAX)
    s, d, k = shell.VectorQ1Scalar(m), shell.VectorQ1Scalar(m), shell.VectorQ1Scalar(m)
    s.data.uniform_(-1, 1)
    k.data.uniform_(1, 10)
    op = shell.DivKGrad(m, k, True)
    return {"DivKGrad apply (3x2 rule), level 6, Dirichlet elimination": lambda: shell.apply(op, s, d)}


def _case_stokes_b6(shell, C, torch):
    mf, mc = shell.ShellMesh(6, RMIN, RMAX), shell.ShellMesh(5, RMIN, RMAX)
    u, v = shell.VectorQ1Vec(mf), shell.VectorQ1Vec(mf)
    p, q = shell.VectorQ1Scalar(mc), shell.VectorQ1Scalar(mc)
    u.data.uniform_(-1, 1)
    p.data.uniform_(-1, 1)
    B = shell.Divergence(mf, mc, C.BC_FREESLIP, C.BC_FREESLIP)
    BT = shell.Gradient(mf, mc, C.BC_FREESLIP, C.BC_FREESLIP)
    return {"Divergence (B), velocity level 6 -> pressure level 5, free-slip": lambda: shell.apply(B, u, q),
            "Gradient (B^T), pressure level 5 -> velocity level 6, free-slip": lambda: shell.apply(BT, p, v)}


def _case_stored5(shell, C, torch):
    m = shell.ShellMesh(5, RMIN, RMAX)
    coords, radii = m.geometry()
    k_np, _ = synthetic_inputs(coords, radii, None)
    k = shell.VectorQ1Scalar(m)
    k.set_numpy(k_np)
    m64 = shell.kerngen_local_matrices(m, k)
    m32 = m64.float()
    out = {}
    for tag, mats, dt in (("FP32", m32, torch.float32), ("FP64", m64, torch.float64)):
        u, v = shell.VectorQ1Vec(m, dt), shell.VectorQ1Vec(m, dt)
        u.data.uniform_(-1, 1)
        op = shell.StoredEpsilonDivDiv(m, mats, C.BC_FREESLIP, C.BC_FREESLIP)
        out[f"stored-matrix apply {tag}, level 5 (451 / 902 MB of matrices), free-slip"] = \
            (lambda op=op, u=u, v=v: shell.apply(op, u, v))
    return out


def _case_kerngen6_fs(shell, C, torch):
    m = shell.ShellMesh(6, RMIN, RMAX)
    coords, radii = m.geometry()
    k_np, _ = synthetic_inputs(coords, radii, None)
    out = {}
    for tag, dt in (("FP32", torch.float32), ("FP64", torch.float64)):
        k = shell.VectorQ1Scalar(m, dt)
        k.data.copy_(torch.as_tensor(k_np))
        u, v = shell.VectorQ1Vec(m, dt), shell.VectorQ1Vec(m, dt)
        u.data.uniform_(-1, 1)
        op = shell.EpsilonDivDivKerngen(m, k, C.BC_FREESLIP, C.BC_FREESLIP)
        out[f"EpsilonDivDivKerngen apply {tag}, level 6, free-slip both radii"] = \
            (lambda op=op, u=u, v=v: shell.apply(op, u, v))
    return out


def _case_stokes6(shell, C, torch):
    """30 FGMRES iterations of the level-6 free-slip Stokes solve (FP32 multigrid): the launch list
    of the C3 solve at a fixed iteration count"""
    pf, pc = shell.ShellMesh(6, RMIN, RMAX), shell.ShellMesh(5, RMIN, RMAX)
    coords, radii = pf.geometry()
    k_np, _ = synthetic_inputs(coords, radii, None)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k_np)
    fu, fp = stokes_rhs(shell, pf, coords, radii), shell.VectorQ1Scalar(pc)
    s = shell.StokesSolver(6, kv, mg_levels=4, bc_cmb=C.BC_FREESLIP, bc_surface=C.BC_FREESLIP, mg_fp32=True,
                           chebyshev_order=3, relative_tolerance=1e-30, max_iterations=30, restart=100,
                           r_min=RMIN, r_max=RMAX, gca=1)
    xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)

    def run():
        xu.data.zero_()
        xp.data.zero_()
        s.solve(fu, fp, xu, xp)
    return {"Stokes solve, level 6 free-slip, FP32 multigrid, 30 FGMRES(100) iterations": run}


def _case_stokes6_refine(shell, C, torch):
    """30 iterations of the level-6 free-slip Stokes solve in the mixed-precision refinement form (Krylov
    cycles in FP32, FGMRES(100), FP32 multigrid, coarse PCG FP64): the launch list of the C3 refinement
    solve at a fixed iteration count"""
    pf, pc = shell.ShellMesh(6, RMIN, RMAX), shell.ShellMesh(5, RMIN, RMAX)
    coords, radii = pf.geometry()
    k_np, _ = synthetic_inputs(coords, radii, None)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k_np)
    fu, fp = stokes_rhs(shell, pf, coords, radii), shell.VectorQ1Scalar(pc)
    s = shell.StokesSolver(6, kv, mg_levels=4, bc_cmb=C.BC_FREESLIP, bc_surface=C.BC_FREESLIP, mg_fp32=True,
                           chebyshev_order=3, relative_tolerance=1e-30, max_iterations=30, restart=100,
                           r_min=RMIN, r_max=RMAX, gca=1, outer=2)
    xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)

    def run():
        xu.data.zero_()
        xp.data.zero_()
        s.solve(fu, fp, xu, xp)
    return {"Stokes solve, level 6 free-slip, refinement form, 30 FGMRES(100) iterations": run}


def _case_stokes6_fp64(shell, C, torch):
    """30 FGMRES iterations of the level-6 free-slip Stokes solve in the plain FP64 form (FP64 multigrid)"""
    pf, pc = shell.ShellMesh(6, RMIN, RMAX), shell.ShellMesh(5, RMIN, RMAX)
    coords, radii = pf.geometry()
    k_np, _ = synthetic_inputs(coords, radii, None)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k_np)
    fu, fp = stokes_rhs(shell, pf, coords, radii), shell.VectorQ1Scalar(pc)
    s = shell.StokesSolver(6, kv, mg_levels=4, bc_cmb=C.BC_FREESLIP, bc_surface=C.BC_FREESLIP, mg_fp32=False,
                           chebyshev_order=3, relative_tolerance=1e-30, max_iterations=30, restart=100,
                           r_min=RMIN, r_max=RMAX, gca=1)
    xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)

    def run():
        xu.data.zero_()
        xp.data.zero_()
        s.solve(fu, fp, xu, xp)
    return {"Stokes solve, level 6 free-slip, FP64 multigrid, 30 FGMRES(100) iterations": run}


def _case_coarse_pcg3(shell, C, torch):
    """The coarsest-level solve of the C3 V-cycle: 50 iterations of the stored-matrix PCG at level 3,
    free-slip both radii, matrices coarsened (GCA, constant interpolation) from the level-4 kerngen matrices"""
    mf, m = shell.ShellMesh(4, RMIN, RMAX), shell.ShellMesh(3, RMIN, RMAX)
    coords, radii = mf.geometry()
    k_np, _ = synthetic_inputs(coords, radii, None)
    k = shell.VectorQ1Scalar(mf)
    k.set_numpy(k_np)
    mats = shell.gca_coarsen(mf, m, k_fine=k)
    op = shell.StoredEpsilonDivDiv(m, mats, C.BC_FREESLIP, C.BC_FREESLIP)
    b, x = shell.VectorQ1Vec(m), shell.VectorQ1Vec(m)
    b.data.normal_(generator=torch.Generator(device="cuda").manual_seed(3))
    b.halo_sum()
    shell.freeslip_project(b, True, True)

    def run():
        x.data.zero_()
        shell.stored_pcg(op, b, x, max_iterations=50, relative_tolerance=1e-30, check_every=0)
    return {"stored-matrix PCG, level 3, free-slip both radii, 50 iterations": run}


def _fct_case(shell, torch, level):
    m = shell.ShellMesh(level, RMIN, RMAX)
    fct = shell.FCTAdvectionDiffusion(m)
    v = shell.VectorQ1Vec(m)
    v.data.normal_(generator=torch.Generator(device="cuda").manual_seed(5))
    T = fct.field()
    T.uniform_(generator=torch.Generator(device="cuda").manual_seed(6))
    dt = 0.5 * fct.dt_stable(v)
    cells = 10 * (1 << level) ** 3
    return {f"FCT explicit step (predictor, limiter, correction), level {level}, {cells:,} cells":
            lambda: fct.step(T, v, dt),
            f"FCT stable time step, level {level}": lambda: fct.dt_stable(v)}


def _case_fct6(shell, C, torch):
    return _fct_case(shell, torch, 6)


def _case_fct7(shell, C, torch):
    return _fct_case(shell, torch, 7)


def _case_shard7(shell, C, torch):
    """The sharded apply on one GPU: rank 0's shard (the largest) of the level-7 shell split over P = 1, 2, 4, 8
    ranks, FP64 Dirichlet apply with the shard-local halo, then pack and unpack of the cross-rank exchange buffer
    (the all-reduce between the GPUs is not part of a one-GPU run)"""
    from terraneo_b200.distributed import ShellShard
    out = {}
    gen = torch.Generator(device="cuda").manual_seed(7)
    for P in (1, 2, 4, 8):
        sh = ShellShard(7, P, 0, RMIN, RMAX)
        k = torch.empty(sh.shape, dtype=torch.float64, device="cuda").uniform_(0.0, 9.2, generator=gen).exp_()
        u, v = sh.vector(3), sh.vector(3)
        u.uniform_(-1, 1, generator=gen)
        buf = sh.exchange_buffer(3)
        tag = (f"P={P}, rank 0: {sh.num_diamonds} diamonds, {3 * sh.stored_nodes:,} DoFs stored, exchange "
               f"{buf.numel() * 8:,} bytes")

        def apply_exchange(sh=sh, k=k, u=u, v=v, buf=buf):
            sh.epsdivdiv_apply(k, u, v, C.BC_DIRICHLET, C.BC_DIRICHLET)
            sh.pack(v, buf)
            sh.unpack(buf, v)

        def exchange_only(sh=sh, v=v, buf=buf):
            sh.pack(v, buf)
            sh.unpack(buf, v)
        out[f"shard apply + pack + unpack, level 7, {tag}"] = apply_exchange
        out[f"pack + unpack only, level 7, P={P}"] = exchange_only
    return out


# name -> builder returning {description: one launch sequence}
CASES = {"laplace6": _case_laplace6, "vlaplace6": _case_vlaplace6, "divkgrad6": _case_divkgrad6,
         "stokes_b6": _case_stokes_b6, "stored5": _case_stored5, "kerngen6_fs": _case_kerngen6_fs,
         "stokes6": _case_stokes6, "stokes6_refine": _case_stokes6_refine, "stokes6_fp64": _case_stokes6_fp64,
         "coarse_pcg3": _case_coarse_pcg3,
         "fct6": _case_fct6, "fct7": _case_fct7, "shard7": _case_shard7}


def kernel_breakdown(fn, torch, top=30):
    """One more call of fn under the CUDA activity trace (torch.profiler): per kernel name the device
    microseconds and launches of that call, largest first.  Kernels that run concurrently on two streams each
    count their whole duration, so the sum can exceed the call's elapsed time."""
    import re
    from torch.profiler import profile, ProfilerActivity
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    rows = {}
    for e in prof.key_averages():
        if e.device_time_total <= 0:
            continue
        k = re.sub(r"\(anonymous namespace\)::|tn::|void ", "", e.key)
        k = re.sub(r"\(.*", "", k)[:80]
        t, c = rows.get(k, (0.0, 0))
        rows[k] = (t + e.device_time_total, c + e.count)
    out = sorted(rows.items(), key=lambda kv: -kv[1][0])[:top]
    return [{"kernel": k, "us": round(t, 1), "launches": c} for k, (t, c) in out]


def run_case(args):
    """Times each workload of one case with CUDA events (after args.warmup calls) and prints one JSON line."""
    import torch
    sys.path.insert(0, ROOT)
    from terraneo_b200 import shell, _capi as C
    torch.cuda.set_device(0)
    work = CASES[args.case](shell, C, torch)
    res = {}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, fn in work.items():
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(args.steps):
            fn()
        ev1.record()
        torch.cuda.synchronize()
        res[name] = {"ms_per_call": round(ev0.elapsed_time(ev1) / args.steps, 5)}
        if args.kernel_breakdown:
            res[name]["kernels"] = kernel_breakdown(fn, torch)
    print(json.dumps({"case": args.case, "steps": args.steps, "warmup": args.warmup, "results": res}), flush=True)
    return 0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-laplace-cg", action="store_true", help="skip the level-5 Laplace CG leg")
    ap.add_argument("--no-stokes", action="store_true", help="skip the level-6 Stokes time-to-1e-8 leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the level-5 adjoint viscosity gradient leg")
    ap.add_argument("--no-timestep", action="store_true", help="skip the level-7 mantle-circulation time-step leg")
    ap.add_argument("--no-level8", action="store_true", help="skip the level-8 apply (the published configuration)")
    ap.add_argument("--case", choices=sorted(CASES), help="time one operator workload (see CASES) instead of the bench")
    ap.add_argument("--sharded", action="store_true",
                    help="also time the level-7 apply sharded over the ranks (always on with two or more ranks)")
    ap.add_argument("--kernel-breakdown", action="store_true",
                    help="with --case: also report one call's device time per kernel (CUDA activity trace)")
    return ap.parse_args()


def synthetic_inputs(coords, radii, omask_lat, seed=2024):
    """Seeded k and src fields in the reference layout (numpy, host)."""
    n1 = radii.shape[1]
    rng = np.random.default_rng(seed)
    rho = (radii - RMIN) / (RMAX - RMIN)
    x = coords[:, :, :, None, :] * radii[:, None, None, :, None]
    field = np.zeros((10, n1, n1, n1))
    for _ in range(6):
        c = rng.normal(size=3)
        c = c / np.linalg.norm(c) * rng.uniform(RMIN, RMAX)
        w = rng.uniform(0.1, 0.3)
        field += np.exp(-np.sum((x - c) ** 2, axis=-1) / (2 * w * w))
    field = (field - field.min()) / (field.max() - field.min())
    k = np.clip(np.exp(np.log(1e4) * (0.5 * rho[:, None, None, :] + 0.5 * field)), 1.0, 1e4)
    src = rng.normal(size=(3, 10, n1, n1, n1))
    return k, src


def stokes_rhs(shell, mesh, coords, radii, seed=2025):
    """Buoyancy RHS f = M (Ra T r_hat), Ra = 1e5, T = conductive profile
    (1/r - 1/r_max) / (1/r_min - 1/r_max) + 0.05 s(x), s a seeded smooth field
    of unit RMS (sum of Gaussian blobs); free-slip projected on both radii."""
    rng = np.random.default_rng(seed)
    r = radii[:, None, None, :]
    tc = (1 / r - 1 / RMAX) / (1 / RMIN - 1 / RMAX)
    x = coords[:, :, :, None, :] * radii[:, None, None, :, None]
    pert = np.zeros(x.shape[:-1])
    for _ in range(12):
        c = rng.normal(size=3)
        c = c / np.linalg.norm(c) * rng.uniform(RMIN, RMAX)
        pert += rng.normal() * np.exp(-np.sum((x - c) ** 2, axis=-1) / (2 * 0.15 ** 2))
    pert -= pert.mean()
    temp = tc + 0.05 * pert / np.sqrt(np.mean(pert ** 2))
    rhat = coords / np.linalg.norm(coords, axis=-1, keepdims=True)
    g = 1e5 * temp[..., None] * rhat[:, :, :, None, :]
    f = shell.VectorQ1Vec(mesh)
    tmp, out = shell.VectorQ1Scalar(mesh), shell.VectorQ1Scalar(mesh)
    mass = shell.KMass(mesh, None, 0)
    for c in range(3):
        tmp.set_numpy(g[..., c])
        shell.apply(mass, tmp, out)
        f.data[c].copy_(out.data[0])
    shell.freeslip_project(f, True, True)
    return f


def sh_rhs(coords, radii, seed, lmax=8):
    """f(x) = sum_{l<=lmax, |m|<=l} a_lm Y_lm(x/|x|) (r - r_min)(r_max - r), a_lm ~ N(0,1) seeded,
    Y_lm the orthonormal real spherical harmonics."""
    from scipy.special import sph_harm_y
    rng = np.random.default_rng(seed)
    u = coords / np.linalg.norm(coords, axis=-1, keepdims=True)
    theta, phi = np.arccos(np.clip(u[..., 2], -1, 1)), np.arctan2(u[..., 1], u[..., 0])
    ang = np.zeros(coords.shape[:-1])
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            y = sph_harm_y(l, abs(m), theta, phi)
            if m > 0:
                y = np.sqrt(2) * (-1) ** m * y.real
            elif m < 0:
                y = np.sqrt(2) * (-1) ** m * y.imag
            else:
                y = y.real
            ang += rng.normal() * y
    return ang[:, :, :, None] * ((radii - RMIN) * (RMAX - radii))[:, None, None, :]


def laplace_cg_leg(shell, torch, level=5, seed=2026, reference=True):
    """Plain FP64 CG on the scalar Laplace at level 5 (10 x 32^3 cells, 359,370 stored nodes),
    homogeneous Dirichlet on both radii, b = M f with f the seeded degree-8 spherical-harmonic
    field, from x = 0 to 1e-10 relative residual.  The reference's own Kokkos-OpenMP solver
    (compiled from its sources) solves the same system on the host cores beside it."""
    pm = shell.ShellMesh(level, RMIN, RMAX)
    coords, radii = pm.geometry()
    f = sh_rhs(coords, radii, seed)
    vf, vb, vx = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    vf.set_numpy(f)
    shell.apply(shell.KMass(pm, None, 0), vf, vb)
    shell.assign_boundary(vb, None, 0.0, True, True)
    shell.laplace_pcg(pm, vb, vx, 5000, 1e-10)  # warm-up
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    secs = []
    for _ in range(3):
        vx.data.zero_()
        torch.cuda.synchronize()
        ev0.record()
        it, rr = shell.laplace_pcg(pm, vb, vx, 5000, 1e-10)
        ev1.record()
        torch.cuda.synchronize()
        secs.append(ev0.elapsed_time(ev1) / 1e3)
    sec = min(secs)
    out = {"workload": f"FP64 CG, Laplace level {level} ({pm.unique_nodes:,} unique nodes), homogeneous Dirichlet "
                       "both radii, b = M f (degree-8 spherical harmonics x (r-0.55)(1-r)), x0 = 0, to 1e-10",
           "seconds": round(sec, 5), "iterations": it, "relres": float(f"{rr:.3e}"),
           "apply_gdofs": round(pm.unique_nodes * it / sec / 1e9, 3)}
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
    if reference and os.path.exists(ref):
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            vb.numpy()[0].tofile(os.path.join(d, "b.bin"))
            env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1), OMP_PROC_BIND="spread",
                       OMP_PLACES="cores")
            res = subprocess.run([ref, "laplace_cg", str(level), str(RMIN), str(RMAX), "5000", "1e-10", d], env=env,
                                 capture_output=True, text=True, timeout=900)
            line = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
            if res.returncode == 0 and line:
                info = json.loads(line[-1])
                xr = np.fromfile(os.path.join(d, "x.bin"))
                xg = vx.numpy()[0].reshape(-1)
                out["cpu_baseline"] = {"value": info["seconds"], "unit": "s", "cores": info["threads"],
                                       "kind": "reference", "iterations": info["iterations"],
                                       "sample": "the same solve with the reference's PCG<Laplace> (Kokkos-OpenMP)",
                                       "solution_rel_diff": float(f"{np.linalg.norm(xg - xr) / np.linalg.norm(xr):.3e}")}
                out["speedup_vs_cpu_reference"] = round(info["seconds"] / sec, 1)
    return out


def stokes_leg(shell, C, torch, k_np):
    """Level-6 free-slip Stokes solve to 1e-8 in three forms: FP64 FGMRES(100) with the FP32 V-cycle
    (fp32_mg) or the FP64 V-cycle (fp64_mg) inside the block-triangular preconditioner, and the
    mixed-precision refinement (fp32_refine: FP64 residual and update around FGMRES(100) cycles done
    entirely in FP32); 4-level V-cycle with Chebyshev order 3, coarse PCG in FP64 in every form.
    Each form: one warm-up solve, then two timed solves from x = 0; `seconds` is the faster one, and each
    sample carries the SM clocks and throttle reasons sampled during it."""
    pf, pc = shell.ShellMesh(LEVEL, RMIN, RMAX), shell.ShellMesh(LEVEL - 1, RMIN, RMAX)
    coords, radii = pf.geometry()
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k_np)
    fu, fp = stokes_rhs(shell, pf, coords, radii), shell.VectorQ1Scalar(pc)
    fnorm = np.sqrt(shell.dot(fu, fu))
    out = {"workload": "Stokes solve, velocity level 6 / pressure level 5, free-slip both radii, 1e4 viscosity "
                       "contrast, buoyancy RHS (Ra 1e5), FGMRES(100) + block-triangular preconditioner, V-cycle over "
                       "levels 3-6 (Chebyshev order 3, 2 smoothing steps, GCA coarse operators with constant "
                       "interpolation, coarse PCG FP64 50 its / 1e-6), "
                       "stop at 1e-8 relative FP64 residual; fp32_refine: the same preconditioner and cycle length "
                       "with the Krylov cycles in FP32 and the residual / update between cycles in FP64"}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for tag, mg32, outer in (("fp32_refine", True, 2), ("fp32_mg", True, 0), ("fp64_mg", False, 0)):
        s = shell.StokesSolver(LEVEL, kv, mg_levels=4, bc_cmb=C.BC_FREESLIP, bc_surface=C.BC_FREESLIP,
                               mg_fp32=mg32, chebyshev_order=3, relative_tolerance=1e-8, max_iterations=1000,
                               restart=100, r_min=RMIN, r_max=RMAX, gca=1, outer=outer)
        xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
        s.solve(fu, fp, xu, xp)  # warm-up: eigenvalue estimates, graph capture, first-touch
        samples, clocks = [], []
        for _ in range(2):
            xu.data.zero_()
            xp.data.zero_()
            with ClockSampler(0) as clk:
                torch.cuda.synchronize()
                ev0.record()
                it, rr = s.solve(fu, fp, xu, xp)
                ev1.record()
                torch.cuda.synchronize()
            samples.append(ev0.elapsed_time(ev1) / 1e3)
            clocks.append(clk.summary())
        ku, kp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
        s.apply(xu, xp, ku, kp)
        shell.lincomb(ku, [1.0, -1.0], [fu, ku])
        shell.lincomb(kp, [1.0, -1.0], [fp, kp])
        true_rr = np.sqrt(shell.dot(ku, ku) + shell.dot(kp, kp)) / fnorm
        out[tag] = {"seconds": round(min(samples), 4), "samples": [round(t, 4) for t in samples], "iterations": it,
                    "true_relres": float(f"{true_rr:.3e}"), "clocks": clocks}
        del s
    out["speedup_fp32_mg"] = round(out["fp64_mg"]["seconds"] / out["fp32_mg"]["seconds"], 3)
    out["speedup_fp32_refine"] = round(out["fp64_mg"]["seconds"] / out["fp32_refine"]["seconds"], 3)
    return out


def smooth_field(coords, radii, seed, blobs=4, width=0.2):
    """Seeded smooth nodal field (sum of Gaussian blobs), max |value| = 1."""
    rng = np.random.default_rng(seed)
    x = coords[:, :, :, None, :] * radii[:, None, None, :, None]
    f = np.zeros(x.shape[:-1])
    for _ in range(blobs):
        c = rng.normal(size=3)
        c = c / np.linalg.norm(c) * rng.uniform(RMIN + 0.05, RMAX - 0.05)
        f += rng.normal() * np.exp(-np.sum((x - c) ** 2, axis=-1) / (2 * width ** 2))
    return f / np.abs(f).max()


def adjoint_leg(shell, C, torch, level=5, directions=20, h=1e-6, exact_directions=20):
    """Adjoint viscosity gradient at level 5 (velocity L5 / pressure L4):
    J = 1/2 sum over owned velocity nodes |u - u_obs|^2, u_obs from a solve with
    a seeded perturbed viscosity; gradient = forward solve + adjoint solve +
    backward kernel (timed), checked against central differences (step h = 1e-6)
    in 20 seeded smooth directions, every solve to 1e-14 (the perturbed ones
    warm-started from the unperturbed solution), and against the exact
    directional derivatives -<lambda, A(k o delta) u> in 20 seeded smooth
    directions."""
    from terraneo_b200.adjoint import stokes_velocity
    pf, pc = shell.ShellMesh(level, RMIN, RMAX), shell.ShellMesh(level - 1, RMIN, RMAX)
    coords, radii = pf.geometry()
    _, omask = pf.masks()
    k0, _ = synthetic_inputs(coords, radii, None)
    m0 = torch.as_tensor(np.log(k0), device="cuda")
    fu, fp = stokes_rhs(shell, pf, coords, radii), shell.VectorQ1Scalar(pc)
    fu.data[:, :, :, :, 0] = 0.0  # Dirichlet rows of the right-hand side
    fu.data[:, :, :, :, -1] = 0.0
    # Dirichlet radii and a coarse-grid PCG run to 1e-12 (a nearly fixed preconditioner): the FP64 solves
    # reach 1e-14 (free-slip ones plateau near 1e-8, which would turn the central differences into noise)
    kw = dict(mg_levels=level - 2, bc_cmb=C.BC_DIRICHLET, bc_surface=C.BC_DIRICHLET, mg_fp32=False,
              relative_tolerance=1e-14, max_iterations=4000, restart=100, coarse_max_iterations=300,
              coarse_relative_tolerance=1e-12, r_min=RMIN, r_max=RMAX)
    owned = torch.as_tensor(omask.astype(np.float64), device="cuda")
    m_obs = m0 + 0.1 * torch.as_tensor(smooth_field(coords, radii, 31), device="cuda")
    u_obs = stokes_velocity(m_obs, level, fu, fp, **kw).detach()

    def J(m):
        u = stokes_velocity(m, level, fu, fp, **kw)
        return 0.5 * (owned * (u - u_obs) ** 2).sum()

    m = m0.clone().requires_grad_(True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    j = J(m)
    j.backward()
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    grad = m.grad.detach()
    # the unperturbed solution: the perturbed solves below start from it
    k0v = shell.VectorQ1Scalar(pf)
    k0v.data[0].copy_(torch.exp(m0))
    solver = shell.StokesSolver(level, k0v, **kw)
    xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    fwd_it, fwd_rr = solver.solve(fu, fp, xu, xp)
    kpert = shell.VectorQ1Scalar(pf)

    # warm-started solves: their initial residual is O(h) |f|, so 1e-10 of it is about 1e-16 |f|, below the
    # 1e-14 |f| of the cold solves; at most 150 iterations each
    kw_warm = dict(kw, relative_tolerance=1e-10, max_iterations=150)
    warm_stats = []

    def J_warm(mm):
        """J with the solve warm-started from the unperturbed solution, so the perturbed solutions carry an
        error of O(h) times the solver's tolerance instead of the tolerance itself"""
        kpert.data[0].copy_(torch.exp(mm))
        sp = shell.StokesSolver(level, kpert, **kw_warm)
        yu = shell.VectorQ1Vec(pf, data=xu.data.clone())
        yp = shell.VectorQ1Scalar(pc, data=xp.data.clone())
        warm_stats.append(sp.solve(fu, fp, yu, yp))
        return float(0.5 * (owned * (yu.data - u_obs) ** 2).sum())

    errs, errs_cold, fd_vals = [], [], []
    for s in range(directions):
        d = torch.as_tensor(smooth_field(coords, radii, 200 + s), device="cuda")
        ad = float((grad * d).sum())
        fd = (J_warm(m0 + h * d) - J_warm(m0 - h * d)) / (2 * h)
        errs.append(abs(fd - ad) / abs(ad))
        if s < 4:
            with torch.no_grad():
                fdc = (J(m0 + h * d) - J(m0 - h * d)).item() / (2 * h)
            errs_cold.append(abs(fdc - ad) / abs(ad))
    # exact directional derivatives: the viscous block is linear in k, so
    # dJ/dm . delta = -<lambda, A(k o delta) u> with the adjoint solution lambda
    # (the operator apply with the viscosity k o delta, Dirichlet both radii)
    gu = shell.VectorQ1Vec(pf, data=(owned * (xu.data - u_obs)).contiguous())
    lam_u, lam_p = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    grad2 = torch.empty(pf.shape, dtype=torch.float64, device="cuda")
    solver.viscosity_backward(xu, gu, grad2, C.COMM_SKIP, lam_u, lam_p)
    kd, out = shell.VectorQ1Scalar(pf), shell.VectorQ1Vec(pf)
    dir_errs = []
    for s in range(exact_directions):
        d = torch.as_tensor(smooth_field(coords, radii, 300 + s, blobs=6), device="cuda")
        kd.data[0].copy_(k0v.data[0] * d)
        shell.apply(shell.EpsilonDivDivKerngen(pf, kd, C.BC_DIRICHLET, C.BC_DIRICHLET), xu, out)
        ref = -shell.dot(lam_u, out)
        dir_errs.append(abs(float((grad2 * d).sum()) - ref) / abs(ref))
    return {"workload": f"adjoint viscosity gradient, velocity level {level} / pressure level {level - 1}, Dirichlet "
                        "both radii, J = 1/2 sum_owned |u - u_obs|^2, FP64 solves to 1e-14 (FGMRES(100), FP64 "
                        f"multigrid over {level - 2} levels, coarse PCG to 1e-12)",
            "forward_iterations": fwd_it, "forward_relres": float(f"{fwd_rr:.3e}"),
            "seconds_forward_adjoint_backward": round(sec, 4),
            "J": float(j.item()), "fd_directions": directions, "fd_step": h,
            "fd_max_rel_error": float(f"{max(errs):.3e}"),
            "fd_median_rel_error": float(f"{float(np.median(errs)):.3e}"),
            "fd_form": "each perturbed solve warm-started from the unperturbed solution, to 1e-10 of its O(h) initial "
                       "residual (at most 150 FGMRES iterations)",
            "fd_warm_iterations_max": max(it for it, _ in warm_stats),
            "fd_warm_relres_max": float(f"{max(rr for _, rr in warm_stats):.3e}"),
            "fd_cold_start_max_rel_error_4_directions": float(f"{max(errs_cold):.3e}"),
            "exact_directions": exact_directions,
            "exact_directional_max_rel_error": float(f"{max(dir_errs):.3e}")}


def level8_leg(shell, C, torch, steps=5, warmup=3):
    """The reference's only published measurement is the epsilon-div-div apply at level 8 (505,284,102 velocity
    DoFs) on an H100 SXM: 7.841 GDoF/s (doc/epsdivdiv_benchmarks/throughput_data.csv:13; GDoF/s = owned vector
    DoFs / time per apply, dst zero-fill and halo included, benchmark_operators.cpp:143-166,208,469).  The same
    apply here on one B200: FP64, Dirichlet/Dirichlet, Replace + halo, the bench's viscosity law (1e4 contrast,
    radial ramp + 6 seeded Gaussian blobs, built on the device) and a seeded N(0,1) src made consistent on
    duplicated nodes.  Another GPU and another input than the published number: context, not a ratio."""
    level = 8
    mesh = shell.ShellMesh(level, RMIN, RMAX)
    coords, radii = mesh.geometry()
    c = torch.as_tensor(coords, device="cuda")
    rd = torch.as_tensor(radii, device="cuda")
    x = c[:, :, :, None, :] * rd[:, None, None, :, None]
    rng = np.random.default_rng(2024)
    field = torch.zeros(x.shape[:-1], dtype=torch.float64, device="cuda")
    for _ in range(6):
        ctr = rng.normal(size=3)
        ctr = ctr / np.linalg.norm(ctr) * rng.uniform(RMIN, RMAX)
        w = rng.uniform(0.1, 0.3)
        field += torch.exp(-((x - torch.as_tensor(ctr, device="cuda")) ** 2).sum(-1) / (2 * w * w))
    del x
    field = (field - field.min()) / (field.max() - field.min())
    rho = ((rd - RMIN) / (RMAX - RMIN))[:, None, None, :]
    k = shell.VectorQ1Scalar(mesh)
    k.data[0].copy_(torch.exp(np.log(1e4) * (0.5 * rho + 0.5 * field)).clamp(1.0, 1e4))
    del field
    src, dst = shell.VectorQ1Vec(mesh), shell.VectorQ1Vec(mesh)
    src.data.normal_(generator=torch.Generator(device="cuda").manual_seed(8))
    _, omask = mesh.masks()
    src.data.mul_(torch.as_tensor(omask, device="cuda", dtype=torch.float64))
    src.halo_sum()
    op = shell.EpsilonDivDivKerngen(mesh, k, C.BC_DIRICHLET, C.BC_DIRICHLET)
    for _ in range(warmup):
        shell.apply(op, src, dst)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        shell.apply(op, src, dst)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    dofs = 3 * mesh.unique_nodes
    out = {"workload": f"EpsilonDivDivKerngen FP64 apply, level-8 shell ({dofs:,} velocity DoFs), Dirichlet/Dirichlet, "
                       "Replace + halo",
           "value": round(dofs / (ms * 1e-3) / 1e9, 3), "unit": "GDoF/s", "ms_per_apply": round(ms, 4),
           "steps": steps, "published_h100": {"value": 7.841, "unit": "GDoF/s",
                                              "source": "doc/epsdivdiv_benchmarks/throughput_data.csv:13"}}
    del op, src, dst, k
    torch.cuda.empty_cache()
    return out


def checkpoint_leg(shell, torch, ts):
    """The app's XDMF checkpoint of the level-7 step (T, u_u, eta as FP32, mantlecirculation.cpp:789-799) into a
    temporary directory: the first write (with geometry.bin and topology.bin), then one steady-state write
    timed three ways (the device time of its conversion kernels on the caller's stream, the host time until
    write() returns, the time until the files are complete), then the recovery of step 1 (velocity, FE
    temperature, FV temperature by l2_project_fe_to_fv).  The directory is removed afterwards."""
    import shutil
    import tempfile
    d = tempfile.mkdtemp(prefix="tn_checkpoint_")
    try:
        ns = ts.mesh_u.stored_nodes
        out = ts.checkpoint_output(d)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out.write()
        out.wait()
        first = time.perf_counter() - t0
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev[0].record()
        out.write()
        ev[1].record()
        t_ret = time.perf_counter() - t0
        out.wait()
        t_all = time.perf_counter() - t0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ts.restore_checkpoint(d, 1)
        torch.cuda.synchronize()
        t_restore = time.perf_counter() - t0
        per_write = ns * 5 * 4
        files = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
        return {"grids": "T, u_u, eta as FP32 (the app's XDMFOutput defaults)", "bytes_per_write": per_write,
                "first_write_seconds": round(first, 3), "write_stream_ms": round(ev[0].elapsed_time(ev[1]), 3),
                "write_returns_ms": round(t_ret * 1e3, 3), "write_complete_seconds": round(t_all, 3),
                "write_complete_gbs": round(per_write / t_all / 1e9, 2), "restore_seconds": round(t_restore, 3),
                "directory_bytes": files}
    except Exception as e:  # a full or read-only scratch disk: report it, keep the bench line
        return {"error": str(e)[:300]}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def timestep_leg(shell, C, torch, level=7, warm_steps=2, spinup_solves=20):
    """One mantle-circulation time step at level 7 (velocity 63,406,854 DoFs, pressure level 6, 20,971,520 FV
    cells) as the app takes it, with the app's solver settings (shell.MantleTimestep; mantlecirculation.cpp:
    870-1045, parameters.hpp): the buoyancy right-hand side from the FE temperature (Ra = 1e5), the Stokes solve
    warm-started from the previous step (FGMRES(10), at most 10 iterations, 1e-6 relative / 1e-12 absolute, the
    FP32 GCA V-cycle with Chebyshev order 2, 2 pre/post smoothing steps, 10 power iterations), the pressure
    normalisation, dt = 0.5 dt_stable, one FP64 FCT step with the Dirichlet temperatures, the FV -> FE L2
    projection (Q1 mass + PCG to 1e-12, warm-started) and the NaN guard.  Before the steps, the first Stokes
    system is solved by repeated warm-started calls of the same solver (untimed, at most `spinup_solves`) so
    that the timed step starts from a converged flow; timed is the step after `warm_steps` steps."""
    free0, total = torch.cuda.mem_get_info()
    pf = shell.ShellMesh(level, RMIN, RMAX)
    coords, radii = pf.geometry()
    k_np, _ = synthetic_inputs(coords, radii, None)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k_np)
    del k_np
    fct0 = shell.FCTAdvectionDiffusion(pf)
    c = fct0.centers
    rr = torch.sqrt(c[0] ** 2 + c[1] ** 2 + c[2] ** 2).clamp_min(1e-30)
    T = ((1 / rr - 1 / RMAX) / (1 / RMIN - 1 / RMAX)).clamp(0, 1) + 0.05 * torch.sin(4 * c[0]) * torch.cos(3 * c[1])
    del fct0, c, rr
    t0 = time.perf_counter()
    ts = shell.MantleTimestep(level, kv, T, rayleigh=1e5, dt_scaling=0.5, bc_cmb=C.BC_FREESLIP,
                              bc_surface=C.BC_FREESLIP, r_min=RMIN, r_max=RMAX, mg_levels=4, mg_fp32=True,
                              chebyshev_order=2, smoothing_steps=2, power_iterations=10, relative_tolerance=1e-6,
                              absolute_tolerance=1e-12, max_iterations=10, restart=10, gca=1)
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    pc = ts.mesh_p
    ku, kp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)

    def true_relres():
        ts.solver.apply(ts.u, ts.p, ku, kp)
        shell.lincomb(ku, [1.0, -1.0], [ts.f_u, ku])
        shell.lincomb(kp, [1.0, -1.0], [ts.f_p, kp])
        return float(np.sqrt(shell.dot(ku, ku) + shell.dot(kp, kp)) / np.sqrt(shell.dot(ts.f_u, ts.f_u)))

    shell.stokes_buoyancy_rhs(pf, ts.T, ts.rayleigh, *ts.bcs, ts.f_u)
    spin, t0 = [], time.perf_counter()
    for _ in range(spinup_solves):
        ts.solver.solve(ts.f_u, ts.f_p, ts.u, ts.p)
        spin.append(true_relres())
        if spin[-1] <= 1e-6:
            break
    spin_s = time.perf_counter() - t0
    warm = []
    for _ in range(warm_steps):
        ts.step()
        warm.append({"stokes_iterations": ts.last["stokes_iterations"], "true_relres": float(f"{true_relres():.3e}")})
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        ev[0].record()
        ok = ts.step()
        ev[1].record()
        torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    n = pf.N
    Ti = ts.T_fv[:, 1:n + 1, 1:n + 1, 1:n + 1]
    last = ts.last
    out = {"workload": f"one time step at level {level} with the mantle-circulation app's settings "
                       f"(shell.MantleTimestep: buoyancy RHS, Stokes velocity level {level} / pressure level {level - 1}, "
                       "free-slip, warm-started FGMRES(10) <= 10 iterations to 1e-6 with the FP32 GCA V-cycle, "
                       "Chebyshev order 2, pressure normalisation, FP64 FCT step of 20,971,520 FV cells at "
                       "0.5 dt_stable, FV -> FE L2 projection, NaN guard), from a spun-up flow",
           "seconds_per_step": round(ev[0].elapsed_time(ev[1]) / 1e3, 4),
           "stokes_iterations": last["stokes_iterations"],
           "stokes_relres_vs_initial": float(f"{last['stokes_relres']:.3e}"),
           "stokes_true_relres": float(f"{true_relres():.3e}"),
           "projection_iterations": last["projection_iterations"], "dt": last["dt"], "finite": ok,
           "spinup": {"solves": len(spin), "seconds": round(spin_s, 2),
                      "true_relres": [float(f"{x:.2e}") for x in spin]},
           "warm_up_steps": warm, "setup_seconds": round(setup, 2),
           "device_memory_gb": round((total - free1) / 1e9, 2),
           "T_range": [float(Ti.min()), float(Ti.max())], "clocks": clk.summary()}
    # last: the recovery overwrites the step's state (the pressure restarts from zero, as in the app)
    out["checkpoint"] = checkpoint_leg(shell, torch, ts)
    del ts, T, kv, ku, kp
    torch.cuda.empty_cache()
    return out


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx, self.rows, self.proc = str(gpu_index), [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_min_mhz": min(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons), "samples": len(sm)}


def reference_inputs(directory):
    """The bench's own level-6 inputs (synthetic_inputs, seed 2024; src consistent on duplicated nodes) written
    as k.bin / src.bin for the compiled reference; the mesh geometry from the oracle (bit-equal to the library's
    and to the reference's)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Mesh
    m = Mesh(LEVEL, RMIN, RMAX)
    k, src = synthetic_inputs(m.coords, m.radii, None)
    k.tofile(os.path.join(directory, "k.bin"))
    m.make_consistent(src).tofile(os.path.join(directory, "src.bin"))
    return m


def apply_errors_vs_reference(ref, env, d, m):
    """The reference's FP64 apply (ref_dump kerngen, Dirichlet both radii) of the inputs in d against the B200's
    FP64 and FP32 applies of the same inputs: relative 2-norm differences over all stored nodes"""
    import torch
    from terraneo_b200 import shell, _capi as C
    out = subprocess.run([ref, "kerngen", str(LEVEL), str(RMIN), str(RMAX), "1", "1", "0", d], env=env,
                         capture_output=True, text=True, timeout=600)
    if out.returncode != 0:
        return None
    want = np.fromfile(os.path.join(d, "dst.bin")).reshape((3,) + m.shape)
    k = np.fromfile(os.path.join(d, "k.bin")).reshape(m.shape)
    u = np.fromfile(os.path.join(d, "src.bin")).reshape((3,) + m.shape)
    pm = shell.ShellMesh(LEVEL, RMIN, RMAX)
    res = {}
    for tag, dt in (("fp64", torch.float64), ("fp32", torch.float32)):
        kv, s, o = shell.VectorQ1Scalar(pm, dt), shell.VectorQ1Vec(pm, dt), shell.VectorQ1Vec(pm, dt)
        kv.set_numpy(k)
        s.set_numpy(u)
        shell.apply(shell.EpsilonDivDivKerngen(pm, kv, C.BC_DIRICHLET, C.BC_DIRICHLET), s, o)
        torch.cuda.synchronize()
        res[tag] = float(f"{np.linalg.norm(o.numpy().astype(np.float64) - want) / np.linalg.norm(want):.3e}")
    return res


def cpu_baseline(steps, shell_mods=True):
    """The reference's own Kokkos-OpenMP apply (oracle/_ref) on the bench's seeded inputs, else the C oracle,
    on this host; with shell_mods, also the B200 FP64 / FP32 applies' relative errors against the reference's
    output on the same inputs."""
    import tempfile
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
    cores = os.cpu_count() or 1
    dofs = 3 * (10 * (1 << LEVEL) ** 2 + 2) * ((1 << LEVEL) + 1)
    with tempfile.TemporaryDirectory() as d:
        m = reference_inputs(d)
        if os.path.exists(ref):
            env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="spread", OMP_PLACES="cores")
            out = subprocess.run([ref, "time_kerngen", str(LEVEL), str(RMIN), str(RMAX), "1", "1", str(steps), d],
                                 env=env, capture_output=True, text=True, timeout=1800)
            line = [l for l in out.stdout.splitlines() if l.startswith("{")]
            if out.returncode == 0 and line:
                info = json.loads(line[-1])
                sec = info["seconds_per_apply"]
                errors = apply_errors_vs_reference(ref, env, d, m) if shell_mods else None
                return {"value": dofs / sec / 1e9, "unit": "GDoF/s", "cores": info["threads"], "kind": "reference",
                        "rel_error_vs_reference": errors,
                        "sample": f"{steps} EpsilonDivDivKerngen<double> applies (Dirichlet/Dirichlet, level {LEVEL}, "
                                  f"the bench's seeded 1e4-contrast k and N(0,1) src) after 1 warm-up, "
                                  f"Kokkos-OpenMP, {info['threads']} threads",
                        "seconds_per_apply": sec}
        # C restatement (single thread) as fallback
        k = np.fromfile(os.path.join(d, "k.bin")).reshape(m.shape)
        u = np.fromfile(os.path.join(d, "src.bin")).reshape((3,) + m.shape)
        t0 = time.perf_counter()
        m.kerngen(k, u, 1, 1, False)
        sec = time.perf_counter() - t0
    return {"value": dofs / sec / 1e9, "unit": "GDoF/s", "cores": 1, "kind": "port",
            "sample": f"1 oracle apply (Dirichlet/Dirichlet, level {LEVEL}, the bench's seeded inputs), single thread",
            "seconds_per_apply": sec}


def stokes_reference_solution(shell, C, torch):
    """Each solver form against the reference's own FP64 solution of a level-4 free-slip Stokes problem
    (tests/golden/ref_stokes_mg_L4.npz: ref_dump stokes_mg, FGMRES(30) to 1e-7 with the app's preconditioner
    stack over 3 levels; inputs in tests/golden/stokes_mg_L4_inputs.npz), the same settings and the smoothers'
    eigenvalue estimates the reference drew."""
    gdir = os.path.join(ROOT, "tests", "golden")
    ref = np.load(os.path.join(gdir, "ref_stokes_mg_L4.npz"))
    inp = np.load(os.path.join(gdir, "stokes_mg_L4_inputs.npz"))
    pf, pc = shell.ShellMesh(4, RMIN, RMAX), shell.ShellMesh(3, RMIN, RMAX)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(inp["k"])
    fu, fp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    fu.set_numpy(inp["f_u"])
    fp.set_numpy(inp["f_p"])
    u_ref, p_ref = ref["x_u_22"].astype(np.float64), ref["x_p_22"].astype(np.float64)
    out = {"workload": "level-4 velocity / level-3 pressure, free-slip both radii, 1e3-contrast viscosity, FGMRES(30) "
                       "to 1e-7 + block-triangular preconditioner + V-cycle over 3 levels (Chebyshev order 3, GCA, "
                       "coarse PCG 50 / 1e-6)",
           "reference_iterations": int(ref["iterations_22"])}
    for tag, mg32, outer in (("fp64_mg", False, 0), ("fp32_mg", True, 0), ("fp32_refine", True, 2)):
        s = shell.StokesSolver(4, kv, mg_levels=3, bc_cmb=C.BC_FREESLIP, bc_surface=C.BC_FREESLIP, mg_fp32=mg32,
                               chebyshev_order=3, smoothing_steps=2, power_iterations=10, vcycles=1,
                               coarse_max_iterations=50, coarse_relative_tolerance=1e-6, restart=30, max_iterations=300,
                               relative_tolerance=1e-7, r_min=RMIN, r_max=RMAX, gca=1, outer=outer,
                               chebyshev_estimates=list(ref["eigenvalues_22"]))
        xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
        it, rr = s.solve(fu, fp, xu, xp)
        du = np.linalg.norm(xu.numpy() - u_ref) / np.linalg.norm(u_ref)
        dp = np.linalg.norm(xp.numpy()[0] - p_ref) / np.linalg.norm(p_ref)
        out[tag] = {"iterations": it, "relres": float(f"{rr:.3e}"), "u_rel_diff": float(f"{du:.3e}"),
                    "p_rel_diff": float(f"{dp:.3e}")}
        del s
    return out


def stokes_cpu_baseline(shell, C, torch, level=5, cores=None):
    """The reference's own FP64 Stokes stack (oracle/_ref/ref_dump stokes_mg: FGMRES(100) + block-triangular
    preconditioner + V-cycle with Chebyshev order 3, 2 smoothing steps, GCA coarse operators, coarse PCG 50 /
    1e-6, mantlecirculation.cpp:486-735) on this host's cores, on the C3 problem at level 5 (velocity level 5,
    pressure level 4, 4 multigrid levels; the level-6 solve takes about 20-40 s per FGMRES iteration on a host,
    hours to 1e-8): the time per FGMRES iteration from a 1- and a 3-iteration solve (their difference leaves
    out the smoothers' first-use power iterations), beside the B200's FP64 and refinement forms on the same
    inputs and settings."""
    import tempfile
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_dump")
    if not os.path.exists(ref):
        return {"unavailable": "oracle/_ref/ref_dump is not built"}
    cores = cores or os.cpu_count() or 1
    pf, pc = shell.ShellMesh(level, RMIN, RMAX), shell.ShellMesh(level - 1, RMIN, RMAX)
    coords, radii = pf.geometry()
    k_np, _ = synthetic_inputs(coords, radii, None)
    fu, fp = stokes_rhs(shell, pf, coords, radii), shell.VectorQ1Scalar(pc)
    secs = {}
    with tempfile.TemporaryDirectory() as d:
        k_np.tofile(os.path.join(d, "k.bin"))
        np.ascontiguousarray(k_np[:, ::2, ::2, ::2]).tofile(os.path.join(d, "kp.bin"))
        fu.numpy().tofile(os.path.join(d, "f_u.bin"))
        fp.numpy().tofile(os.path.join(d, "f_p.bin"))
        env = dict(os.environ, OMP_NUM_THREADS=str(cores), OMP_PROC_BIND="spread", OMP_PLACES="cores")
        for its in (1, 3):
            out = subprocess.run([ref, "stokes_mg", str(level), "4", str(RMIN), str(RMAX), "2", "2", "100", str(its),
                                  "1e-30", "3", "2", "10", "1", "1", "50", d], env=env, capture_output=True, text=True,
                                 timeout=1200)
            line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
            if out.returncode != 0 or not line:
                return {"unavailable": f"ref_dump stokes_mg failed (rc {out.returncode})"}
            secs[its] = json.loads(line[-1])["seconds"]
    per_it_ref = (secs[3] - secs[1]) / 2
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k_np)
    gpu = {}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for tag, mg32, outer in (("fp64_mg", False, 0), ("fp32_refine", True, 2)):
        s = shell.StokesSolver(level, kv, mg_levels=4, bc_cmb=C.BC_FREESLIP, bc_surface=C.BC_FREESLIP, mg_fp32=mg32,
                               chebyshev_order=3, relative_tolerance=1e-30, max_iterations=20, restart=100,
                               r_min=RMIN, r_max=RMAX, gca=1, outer=outer)
        xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
        s.solve(fu, fp, xu, xp)  # warm-up: eigenvalue estimates, graph capture
        best = None
        for _ in range(3):  # best of three (the FP32 forms show sporadic slow solves on some boxes)
            xu.data.zero_()
            xp.data.zero_()
            torch.cuda.synchronize()
            ev0.record()
            it, _ = s.solve(fu, fp, xu, xp)
            ev1.record()
            torch.cuda.synchronize()
            t = ev0.elapsed_time(ev1) / 1e3 / it
            best = t if best is None else min(best, t)
        gpu[tag] = round(best, 6)
        del s
    return {"kind": "reference", "cores": cores, "level": level,
            "seconds_per_iteration": round(per_it_ref, 4), "unit": "s per FGMRES iteration",
            "sample": f"ref_dump stokes_mg at level {level} (free-slip both radii, the bench's 1e4-contrast viscosity "
                      f"and buoyancy RHS), 1 and 3 FGMRES(100) iterations ({secs[1]:.1f} s, {secs[3]:.1f} s), "
                      f"Kokkos-OpenMP, {cores} threads",
            "b200_seconds_per_iteration": gpu}


def max_over_ranks(value, world, device):
    """The largest of the ranks' values (every rank calls this, in the same order); the value itself at N = 1."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gdofs(world, dofs, ms):
    """Whole-job throughput: each of `world` ranks applies the operator to its own replica of `dofs` DoFs per
    step, and a step takes `ms` milliseconds on the slowest rank."""
    return world * dofs / (ms * 1e-3) / 1e9


def run_reference(args, rank):
    if rank != 0:
        return 0
    steps = max(1, args.steps)  # the same number of timed applies as the library's arm
    cb = cpu_baseline(steps, shell_mods=False)  # the reference alone: none of this library's kernels
    line = {"metric": METRIC, "impl": "reference", "value": cb["value"], "unit": "GDoF/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": 1, "ms_per_step": cb["seconds_per_apply"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"EpsilonDivDivKerngen apply, level {LEVEL} shell (7,987,590 velocity DoFs), "
                                   "Dirichlet/Dirichlet, FP64, the bench's seeded 1e4-contrast k and N(0,1) src"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def sharded_leg(C, torch, world, rank, steps, warmup, level=7):
    """The level-7 EpsilonDivDivKerngen FP64 apply with the shell sharded over the ranks (one process per GPU):
    every rank applies the operator on the diamonds the reference's rank map gives it, then the copies shared
    between ranks are summed by one all-reduce of the exchange buffer (NCCL).  Timed with CUDA events on the
    launching stream, max over ranks; the value is the whole shell's DoFs per second (strong scaling)."""
    import torch.distributed as dist
    from terraneo_b200.distributed import DistributedShell, partition
    ds = DistributedShell(level, RMIN, RMAX)
    sh = ds.shard
    gen = torch.Generator(device="cuda").manual_seed(17 + rank)
    k = torch.empty(sh.shape, dtype=torch.float64, device="cuda").uniform_(0.0, 9.2, generator=gen).exp_()
    u, v = sh.vector(3), sh.vector(3)
    u.uniform_(-1, 1, generator=gen)

    def step():
        ds.epsdivdiv_apply(k, u, v, C.BC_DIRICHLET, C.BC_DIRICHLET)
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / steps, world, "cuda")
    n1 = (1 << level) + 1
    dofs = 3 * (10 * (n1 - 1) ** 2 + 2) * n1
    return {"workload": f"EpsilonDivDivKerngen FP64 apply, level-{level} shell ({dofs:,} velocity DoFs), "
                        f"Dirichlet/Dirichlet, sharded over {world} rank(s) by diamond, one all-reduce of the "
                        "cross-rank copies per apply",
            "value": round(dofs / (ms * 1e-3) / 1e9, 3), "unit": "GDoF/s", "ms_per_apply": round(ms, 5),
            "scaling": "strong", "ranks": world,
            "diamonds_per_rank": [partition(world, q)[1] for q in range(world)],
            "exchange_bytes_per_apply": 3 * sh.exchange_values * 8}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.case:
        return run_case(args)

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from terraneo_b200 import shell, _capi as C

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    assert args.warmup >= 3, "at least 3 warm-up steps"

    mesh = shell.ShellMesh(LEVEL, RMIN, RMAX)
    coords, radii = mesh.geometry()
    _, omask = mesh.masks()
    k_np, src_np = synthetic_inputs(coords, radii, omask)
    k = shell.VectorQ1Scalar(mesh)
    k.set_numpy(k_np)
    nsets = 4
    srcs, dsts = [], []
    for i in range(nsets):
        s = shell.VectorQ1Vec(mesh)
        s.set_numpy(np.roll(src_np, i, axis=-1))
        # consistent on duplicated nodes: keep owner values, then sum copies
        s.data.mul_(torch.as_tensor(omask, device="cuda", dtype=torch.float64))
        s.halo_sum()
        srcs.append(s)
        dsts.append(shell.VectorQ1Vec(mesh))
    op = shell.EpsilonDivDivKerngen(mesh, k, C.BC_DIRICHLET, C.BC_DIRICHLET)
    stream = torch.cuda.current_stream()

    def step(i):
        shell.apply(op, srcs[i % nsets], dsts[i % nsets])

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(args.steps):
            step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world, "cuda")
    dofs = 3 * mesh.unique_nodes
    value = whole_job_gdofs(world, dofs, ms)

    # dominant kernel: Neumann/Neumann without communication is one launch of the
    # tiled apply kernel (same per-cell work as the headline step) after the small
    # kernel that zeros its tile-seam columns (1/16 of the nodes); both are timed
    op_k = shell.EpsilonDivDivKerngen(mesh, k, C.BC_NEUMANN, C.BC_NEUMANN, comm_mode=C.COMM_SKIP)
    for i in range(3):
        shell.apply(op_k, srcs[i % nsets], dsts[i % nsets])
    torch.cuda.synchronize()
    ev0.record(stream)
    for i in range(args.steps):
        shell.apply(op_k, srcs[i % nsets], dsts[i % nsets])
    ev1.record(stream)
    torch.cuda.synchronize()
    kms = ev0.elapsed_time(ev1) / args.steps
    alg_bytes = BYTES_PER_NODE_F64 * mesh.stored_nodes
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg_bytes / (kms * 1e-3) / 1e9

    # FP32 apply (same workload, FP32 storage and arithmetic)
    k32 = shell.VectorQ1Scalar(mesh, torch.float32)
    k32.data.copy_(k.data)
    s32 = [shell.VectorQ1Vec(mesh, torch.float32) for _ in range(nsets)]
    d32 = [shell.VectorQ1Vec(mesh, torch.float32) for _ in range(nsets)]
    for a, b in zip(s32, srcs):
        a.data.copy_(b.data)
    op32 = shell.EpsilonDivDivKerngen(mesh, k32, C.BC_DIRICHLET, C.BC_DIRICHLET)
    for i in range(3):
        shell.apply(op32, s32[i % nsets], d32[i % nsets])
    torch.cuda.synchronize()
    ev0.record(stream)
    for i in range(args.steps):
        shell.apply(op32, s32[i % nsets], d32[i % nsets])
    ev1.record(stream)
    torch.cuda.synchronize()
    ms32 = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world, "cuda")

    # end to end through the public API with host buffers: pinned H2D of src,
    # apply, D2H of dst, every step
    h_src = torch.empty((3,) + mesh.shape, dtype=torch.float64).pin_memory()
    h_src.copy_(srcs[0].data.cpu())
    h_dst = torch.empty_like(h_src).pin_memory()
    e_src, e_dst = shell.VectorQ1Vec(mesh), shell.VectorQ1Vec(mesh)
    e2e_steps = max(3, args.steps // 5)
    for i in range(2):
        e_src.data.copy_(h_src, non_blocking=True)
        shell.apply(op, e_src, e_dst)
        h_dst.copy_(e_dst.data, non_blocking=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for i in range(e2e_steps):
        e_src.data.copy_(h_src, non_blocking=True)
        shell.apply(op, e_src, e_dst)
        h_dst.copy_(e_dst.data, non_blocking=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_serial_ms = max_over_ranks(ev0.elapsed_time(ev1) / e2e_steps, world, "cuda")
    vec_bytes = 3 * mesh.stored_nodes * 8

    # the same end-to-end steps pipelined as a serving loop runs them: step i's host->device copy on an input
    # stream and its device->host copy on an output stream overlap the neighbouring steps' applies (two
    # device buffer pairs, two pinned result buffers; events order each buffer's reuse)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    p_src = [shell.VectorQ1Vec(mesh) for _ in range(2)]
    p_dst = [shell.VectorQ1Vec(mesh) for _ in range(2)]
    h_out = [torch.empty_like(h_src).pin_memory() for _ in range(2)]

    def pipelined(nsteps, start):
        ev_in = [torch.cuda.Event() for _ in range(2)]
        ev_comp = [torch.cuda.Event() for _ in range(2)]
        ev_out = [torch.cuda.Event() for _ in range(2)]
        s_in.wait_event(start)
        s_out.wait_event(start)
        for i in range(nsteps):
            b = i % 2
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_comp[b])          # the apply of step i-2 has read p_src[b]
                p_src[b].data.copy_(h_src, non_blocking=True)
                ev_in[b].record(s_in)
            stream.wait_event(ev_in[b])
            if i >= 2:
                stream.wait_event(ev_out[b])             # step i-2's result has left p_dst[b]
            shell.apply(op, p_src[b], p_dst[b])
            ev_comp[b].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_comp[b])
                h_out[b].copy_(p_dst[b].data, non_blocking=True)
                ev_out[b].record(s_out)
        for b in range(min(2, nsteps)):
            stream.wait_event(ev_out[b])

    st0 = torch.cuda.Event()
    st0.record(stream)
    pipelined(3, st0)
    torch.cuda.synchronize()
    ev0.record(stream)
    pipelined(e2e_steps, ev0)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1) / e2e_steps, world, "cuda")
    # the last results arrived: compare with the serial loop's
    e2e_check = float((h_out[(e2e_steps - 1) % 2] - h_dst).abs().max())

    # every rank takes part in the sharded leg (collectives), before the rank-0-only legs
    sharded = sharded_leg(C, torch, world, rank, args.steps, args.warmup) if (world > 1 or args.sharded) else None

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 5), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "EpsilonDivDivKerngen FP64 apply, level-6 shell (10x64x64x64 cells, "
                                   "7,987,590 velocity DoFs), Dirichlet/Dirichlet, Replace + halo",
                       "l2": "inputs rotate over 4 buffer sets (528 MB > 126 MB L2)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": TILE_TRAFFIC_BYTES,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                           "kerngen_tile_kernel<double, 16> launch at level 6 (Dirichlet apply; "
                                           "profiles/kerngen_tile_kernel_f64_L6_dirichlet.md)",
                         "kernel": "kerngen_tile_kernel<double, 16>", "kernel_ms": round(kms, 5),
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
            "fp32_apply": {"value": round(whole_job_gdofs(world, dofs, ms32), 3), "unit": "GDoF/s",
                           "ms_per_step": round(ms32, 5)},
            "e2e": {"value": round(whole_job_gdofs(world, dofs, e2e_ms), 3), "unit": "GDoF/s",
                    "h2d_bytes_per_step": vec_bytes, "d2h_bytes_per_step": vec_bytes,
                    "form": "pinned host src -> device, apply, device -> pinned host dst every step; copies on "
                            "their own streams overlap the neighbouring steps' applies",
                    "serial": {"value": round(whole_job_gdofs(world, dofs, e2e_serial_ms), 3),
                               "form": "copy in, apply, copy out one after another on one stream"},
                    "max_abs_diff_vs_serial": e2e_check},
            "gpu_launches": 4 * args.steps,  # seam zeros, tile, boundary cells, halo sum
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_laplace_cg:
            line["laplace_cg"] = laplace_cg_leg(shell, torch, reference=not args.no_cpu_baseline)
        if world == 1 and not args.no_stokes:
            line["stokes"] = stokes_leg(shell, C, torch, k_np)
            line["stokes"]["vs_reference_solution"] = stokes_reference_solution(shell, C, torch)
            if not args.no_cpu_baseline:
                line["stokes"]["cpu_baseline"] = stokes_cpu_baseline(shell, C, torch)
        if world == 1 and not args.no_adjoint:
            line["adjoint"] = adjoint_leg(shell, C, torch)
        if world == 1 and not args.no_level8:
            line["level8"] = level8_leg(shell, C, torch)
        if sharded is not None:
            line["sharded"] = sharded
        if world == 1 and not args.no_timestep:
            line["timestep"] = timestep_leg(shell, C, torch)
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(steps=3)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            # the C2 comparison: the B200's FP64 and FP32 applies against the reference's own FP64 apply
            line["apply_rel_error_vs_reference"] = cb.get("rel_error_vs_reference")
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
