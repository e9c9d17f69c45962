"""Generate the golden fixtures in this folder from the reference itself.

Runs the reference's own operators, compiled from its sources into
oracle/_ref/ref_dump (recipe: oracle/ref_build/Makefile), on small seeded
meshes and writes their outputs to ref_L2.npz.  Inputs are not stored: they
are regenerated from numpy's frozen legacy generator (RandomState) with the
seeds below, and the fixture keeps their checksums so a drift in generation
shows up as a failing check instead of a silent mismatch.

Usage (in a container that has the reference sources and a built ref_dump):
    python tests/golden/make_golden.py               # ref_L2.npz
    python tests/golden/make_golden.py --stokes-mg   # ref_stokes_mg_L4.npz (a few minutes on one thread)
    python tests/golden/make_golden.py --xdmf        # xdmf_L2/: a checkpoint written by io::XDMFOutput
    python tests/golden/make_golden.py --supg        # adds the SUPG operator cases to ref_L2.npz
    python tests/golden/make_golden.py --agca        # adds the adaptive-GCA cases (level 3) to ref_L2.npz
    python tests/golden/make_golden.py --stokes-mg-inputs  # stokes_mg_L4_inputs.npz: the free-slip inputs of
                                                           # ref_stokes_mg_L4.npz for a reader without the oracle
    python tests/golden/make_golden.py --shard       # shard_L2.npz: the reference run as rank q of P
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle_lib import Mesh, run_ref  # noqa: E402

L = 2
R_MIN, R_MAX = 0.55, 1.0
KERNGEN_CASES = [(1, 1, 0), (2, 2, 0), (2, 1, 0), (1, 2, 0), (0, 0, 0), (0, 1, 0), (1, 1, 1), (2, 2, 1)]
LAPLACE_CASES = [(1, 0), (0, 0), (1, 1)]
STOKES_BCS = [(1, 1), (2, 2), (0, 0)]
STOKES_OP_BCS = [(1, 1), (2, 2), (2, 1)]
KMASS_MODES = [0, 1, 2]
MASS_MODES = [0, 1, 2]
VMASS_MODES = [0, 1]
DIVKGRAD_CASES = [(1, 0, 0), (0, 0, 0), (1, 1, 0), (1, 0, 1)]
EPSDIVDIV_CASES = [(1, 0), (0, 0), (1, 1)]
VLAPLACE_CASES = [(1, 1, 0), (0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 1)]
# FV -> FE transfer (consistent mass + PCG, lumped) of a seeded FV field, and the app's Stokes buoyancy
# right-hand side (Ra = 1e5) of a seeded FE temperature for these boundary conditions
L2PROJ_MODES = [0, 1]
STOKES_RHS_BCS = [(2, 2), (1, 1), (2, 1), (1, 2), (0, 0)]
STOKES_RHS_RA = 1e5


def timestep_inputs(fine):
    """seeded FV field (with ghosts) and FE temperature in [0, 1] consistent on duplicated nodes"""
    rs = np.random.RandomState(55)
    fv = rs.normal(size=fine.fv_shape)
    T = fine.make_consistent(rs.uniform(size=fine.shape)).reshape(fine.shape)
    return fv, T


# kerngen slow path (the reference's own assembled wedge matrices stored in Full mode): (bcc, bcs, diag)
KSLOW_CASES = [(1, 1, 0), (2, 2, 0), (2, 1, 0), (0, 0, 0), (2, 2, 1)]
# wedge matrices kept in the fixture: these cells (flat index (d, x, y, r)), both wedges
KSLOW_CELLS = [0, 37, 311, 639]
# TwoGridGCA of the Neumann kerngen operator (level L -> L-1), then the stored-matrix apply of the coarse
# operator to the coarse vector uc: (interpolation mode 0 constant / 1 linear, bcc, bcs, diag)
GCA_CASES = [(0, 1, 1, 0), (0, 2, 2, 0), (0, 2, 1, 0), (0, 0, 0, 0), (0, 2, 2, 1),
             (1, 1, 1, 0), (1, 2, 2, 0), (1, 1, 2, 0), (1, 1, 1, 1)]


def inputs(fine, coarse):
    """Seeded inputs (numpy RandomState is stream-stable across versions)."""
    rs = np.random.RandomState(20240601)
    k = fine.make_consistent(np.exp(rs.normal(size=fine.shape)))
    u = fine.make_consistent(rs.normal(size=(3,) + fine.shape))
    s = fine.make_consistent(rs.normal(size=fine.shape))
    p = coarse.make_consistent(rs.normal(size=coarse.shape))
    uc = coarse.make_consistent(rs.normal(size=(3,) + coarse.shape))
    pc = coarse.make_consistent(rs.normal(size=coarse.shape))
    return dict(k=k, u=u, s=s, p=p, uc=uc, pc=pc)


FCT_CASES = [(0.0, 0), (0.01, 1)]


def fct_inputs(fine):
    """rigid rotation plus a smooth perturbation; temperature from the oracle's cell centres (seeded)"""
    rs = np.random.RandomState(77)
    x = fine.coords[:, :, :, None, :] * fine.radii[:, None, None, :, None]
    w = rs.normal(size=3)
    vel = np.cross(np.broadcast_to(w, x.shape), x)
    vel += 0.2 * np.stack([np.sin(3 * x[..., 1]), np.cos(2 * x[..., 2]), np.sin(4 * x[..., 0])], axis=-1)
    vel = fine.make_consistent(np.ascontiguousarray(np.moveaxis(vel, -1, 0)))
    c = fine.fv_cell_centers()
    N = fine.N
    inner = (slice(None), slice(1, N + 1), slice(1, N + 1), slice(1, N + 1))
    T = np.zeros(fine.fv_shape)
    cc = c[(slice(None),) + inner]
    T[inner] = 0.5 + 0.3 * np.sin(4 * cc[0]) * np.cos(3 * cc[1]) + 0.2 * (cc[2] > 0)
    src = np.zeros(fine.fv_shape)
    src[inner] = 0.1 * np.cos(cc[0])
    return vel, T, src


CG_MAXIT, CG_TOL = 500, 1e-13


def cg_rhs(s):
    """the seeded scalar field with its radial boundary layers zeroed (homogeneous Dirichlet rows)"""
    b = s.copy()
    b[..., 0] = 0.0
    b[..., -1] = 0.0
    return b


# Chebyshev smoother on the Laplace (the CG right-hand side): order 3, 2 sweeps, 50 power iterations; run on
# one thread, where the reference's randomised eigenvalue start is reproducible
CHEBYSHEV_CASE = dict(order=3, iters=2, pits=50)

# PBiCGStab(2) on the Laplace (the CG right-hand side), at most 40 iterations, 1e-10; the fixture keeps the
# shadow residual the reference drew
BICGSTAB_CASE = dict(l=2, maxit=40, tol=1e-10)

# PMINRES on the Laplace (the CG right-hand side), at most 60 iterations, 1e-10
MINRES_CASE = dict(maxit=60, tol=1e-10)

# FGMRES(10) on the Laplace (the CG right-hand side), at most 60 iterations, 1e-10
FGMRES_CASE = dict(restart=10, maxit=60, tol=1e-10)

# FGMRES(10) on the Stokes block operator with the block-triangular preconditioner (2 Jacobi sweeps,
# damping 0.5; Schur block from the pressure-level viscosity exp(0.3 pc)), 30 iterations
STOKES_FGMRES = dict(restart=10, maxit=30, tol=1e-8, sweeps=2, omega=0.5, bcs=[(2, 2), (1, 1)])


# PMINRES on the Stokes block operator with the block-diagonal preconditioner (1 Jacobi sweep, damping 0.5:
# a symmetric positive diagonal velocity block), 40 iterations
STOKES_MINRES = dict(maxit=40, tol=1e-8, sweeps=1, omega=0.5, bcs=[(1, 1), (2, 2)])


def pressure_viscosity(x):
    return np.exp(0.3 * x["pc"])


# Laplace V-cycles over levels 1-3 (Jacobi omega 0.6, 2 sweeps, 2 cycles, coarse PCG <= 50 iterations)
VCYCLE = dict(lmin=1, lmax=3, omega=0.6, smooth=2, cycles=2, cmaxit=50)


# epsilon-div-div V-cycles over levels 1-3, free-slip both radii (the Stokes velocity block's boundaries):
# Jacobi omega 0.5, 2 sweeps, 2 cycles, coarse PCG <= 50 iterations; viscosity injected from level 3
KVCYCLE = dict(lmin=1, lmax=3, bcs=(2, 2), omega=0.5, smooth=2, cycles=2, cmaxit=50)


def kvcycle_inputs():
    """seeded viscosity per level (the finest field injected to the coarser levels) and right-hand side"""
    m = Mesh(KVCYCLE["lmax"])
    rs = np.random.RandomState(47)
    kf = m.make_consistent(np.exp(rs.normal(size=m.shape))).reshape(m.shape)
    b = m.make_consistent(rs.normal(size=(3,) + m.shape)).reshape((3,) + m.shape)
    ks = [np.ascontiguousarray(kf[:, ::s, ::s, ::s]) for s in (4, 2, 1)]
    return ks, b


def vcycle_rhs():
    """seeded right-hand side on the finest V-cycle level"""
    m = Mesh(VCYCLE["lmax"])
    return m.make_consistent(np.random.RandomState(31).normal(size=m.shape)).reshape(m.shape)


# The app's Stokes solver stack (ref_dump stokes_mg): velocity level 4 / pressure level 3, 3 multigrid levels
# (GCA coarse operators with constant interpolation at levels 3 and 2), Chebyshev order 3 with 2 sweeps and 10
# power iterations, 1 V-cycle, coarse PCG(50, 1e-6), FGMRES(30) to 1e-8 (Dirichlet) / 1e-7 (free-slip: the
# pressure's constant mode makes the system singular and the residual stalls near 9e-8); run on one thread,
# where the smoothers' randomised eigenvalue estimates are reproducible (the fixture keeps them)
STOKES_MG = dict(level=4, mg_levels=3, restart=30, maxit=300, order=3, steps=2, pits=10, vcycles=1, gca=1,
                 cmaxit=50, bcs=[(1, 1), (2, 2)], tol={(1, 1): 1e-8, (2, 2): 1e-7})


def stokes_mg_inputs(bcc, bcs):
    """seeded 1e3-contrast viscosity (level 4), its injection to level 3, and a velocity right-hand side with
    the boundary rows enforced (zero on Dirichlet layers, tangential on free-slip layers); zero pressure RHS"""
    f = Mesh(STOKES_MG["level"])
    rs = np.random.RandomState(4242)
    x = f.coords[:, :, :, None, :] * f.radii[:, None, None, :, None]
    ramp = np.broadcast_to(((f.radii - R_MIN) / (R_MAX - R_MIN))[:, None, None, :], f.shape)
    blobs = np.zeros(f.shape)
    for _ in range(6):
        c = rs.normal(size=3)
        c *= rs.uniform(R_MIN, R_MAX) / np.linalg.norm(c)
        blobs += np.exp(-np.sum((x - c) ** 2, axis=-1) / (2 * 0.2 ** 2))
    blobs /= blobs.max()
    k = np.exp(np.log(1e3) * (0.5 * ramp + 0.5 * blobs))
    kp = np.ascontiguousarray(k[:, ::2, ::2, ::2])
    fu = f.make_consistent(rs.normal(size=(3,) + f.shape)).reshape((3,) + f.shape)
    n = f.coords / np.linalg.norm(f.coords, axis=-1, keepdims=True)
    for bc, r in ((bcc, 0), (bcs, -1)):
        if bc == 1:
            fu[..., r] = 0.0
        elif bc == 2:
            nn = np.moveaxis(n, -1, 0)
            fu[..., r] -= np.sum(fu[..., r] * nn, axis=0) * nn
    fp = np.zeros((10,) + (f.N // 2 + 1,) * 3)
    return k, kp, fu, fp


def make_stokes_mg():
    """ref_stokes_mg_L4.npz: the reference's solution, residual history, iteration count and the eigenvalue
    estimates its smoothers drew, for both boundary cases of STOKES_MG."""
    S = STOKES_MG
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for bcc, bcs in S["bcs"]:
            k, kp, fu, fp = stokes_mg_inputs(bcc, bcs)
            out[f"checksum_fu_{bcc}{bcs}"] = checksum(fu)
            out["checksum_k"] = checksum(k)
            k.tofile(f"{d}/k.bin")
            kp.tofile(f"{d}/kp.bin")
            fu.tofile(f"{d}/f_u.bin")
            fp.tofile(f"{d}/f_p.bin")
            info = run_ref(["stokes_mg", S["level"], S["mg_levels"], R_MIN, R_MAX, bcc, bcs, S["restart"], S["maxit"],
                            S["tol"][(bcc, bcs)], S["order"], S["steps"], S["pits"], S["vcycles"], S["gca"], S["cmaxit"], d], d,
                           threads=1, json_out=True)
            # solutions kept in FP32 (the fixture's size; 6e-8 rounding, far below the comparison's tolerance)
            out[f"x_u_{bcc}{bcs}"] = np.fromfile(f"{d}/x_u.bin").reshape(fu.shape).astype(np.float32)
            out[f"x_p_{bcc}{bcs}"] = np.fromfile(f"{d}/x_p.bin").reshape(fp.shape).astype(np.float32)
            out[f"hist_{bcc}{bcs}"] = np.fromfile(f"{d}/hist.bin")
            out[f"iterations_{bcc}{bcs}"] = np.array(info["iterations"])
            out[f"eigenvalues_{bcc}{bcs}"] = np.array(info["eigenvalues"])
            print("stokes_mg", bcc, bcs, info)
    path = os.path.join(HERE, "ref_stokes_mg_L4.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


def make_stokes_mg_inputs():
    """stokes_mg_L4_inputs.npz: the free-slip (2, 2) inputs of ref_stokes_mg_L4.npz as arrays (the bench compares
    its solver forms with the reference's solution there and does not load the oracle)"""
    k, kp, fu, fp = stokes_mg_inputs(2, 2)
    path = os.path.join(HERE, "stokes_mg_L4_inputs.npz")
    np.savez_compressed(path, k=k, kp=kp, f_u=fu, f_p=fp)
    print("wrote", path, os.path.getsize(path), "bytes")


def checksum(a):
    a = np.asarray(a, dtype=np.float64)
    return np.array([a.sum(), (a * a).sum(), np.abs(a).max()])


def main():
    fine, coarse = Mesh(L), Mesh(L - 1)
    x = inputs(fine, coarse)
    out = {"level": np.array(L), "r_range": np.array([R_MIN, R_MAX])}
    for name, a in x.items():
        out["checksum_" + name] = checksum(a)
    with tempfile.TemporaryDirectory() as d:
        run_ref(["mesh", L, R_MIN, R_MAX, d], d)
        out["coords"] = np.fromfile(f"{d}/coords.bin").reshape(fine.coords.shape)
        out["radii"] = np.fromfile(f"{d}/radii.bin").reshape(fine.radii.shape)
        out["bmask"] = np.fromfile(f"{d}/bmask.bin", np.uint8).reshape(fine.shape)
        out["omask"] = np.fromfile(f"{d}/omask.bin", np.uint8).reshape(fine.shape)

        x["k"].tofile(f"{d}/k.bin")
        x["u"].tofile(f"{d}/src.bin")
        for bcc, bcs, diag in KERNGEN_CASES:
            run_ref(["kerngen", L, R_MIN, R_MAX, bcc, bcs, diag, d], d)
            out[f"kerngen_{bcc}{bcs}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)

        for bcc, bcs, diag in KSLOW_CASES:
            run_ref(["kerngen_slow", L, R_MIN, R_MAX, bcc, bcs, diag, d], d)
            out[f"kslow_{bcc}{bcs}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)
        out["kslow_mats"] = np.fromfile(f"{d}/mats.bin").reshape(-1, 2, 18, 18)[KSLOW_CELLS]

        x["uc"].tofile(f"{d}/src.bin")
        for mode, bcc, bcs, diag in GCA_CASES:
            run_ref(["gca", L, R_MIN, R_MAX, bcc, bcs, diag, mode, d], d)
            out[f"gca_{mode}_{bcc}{bcs}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + coarse.shape)

        fv, Tfe = timestep_inputs(fine)
        out["checksum_ts_fv"], out["checksum_ts_T"] = checksum(fv), checksum(Tfe)
        fv.tofile(f"{d}/fv.bin")
        for lumped in L2PROJ_MODES:
            run_ref(["l2proj", L, R_MIN, R_MAX, lumped, d], d)
            out[f"l2proj_{lumped}"] = np.fromfile(f"{d}/x.bin").reshape(fine.shape)
        Tfe.tofile(f"{d}/T.bin")
        for bcc, bcs in STOKES_RHS_BCS:
            run_ref(["stokes_rhs", L, R_MIN, R_MAX, STOKES_RHS_RA, bcc, bcs, d], d)
            out[f"stokes_rhs_{bcc}{bcs}"] = np.fromfile(f"{d}/f_u.bin").reshape((3,) + fine.shape)
        run_ref(["fe2fv", L, R_MIN, R_MAX, d], d)
        out["fe2fv"] = np.fromfile(f"{d}/fv.bin").reshape(fine.fv_shape)

        x["s"].tofile(f"{d}/src.bin")
        for treat, diag in LAPLACE_CASES:
            run_ref(["laplace", L, R_MIN, R_MAX, treat, diag, d], d)
            out[f"laplace_{treat}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)

        for bcc, bcs in STOKES_BCS:
            x["u"].tofile(f"{d}/src.bin")
            run_ref(["divergence", L, R_MIN, R_MAX, bcc, bcs, d], d)
            out[f"divergence_{bcc}{bcs}"] = np.fromfile(f"{d}/dst.bin").reshape(coarse.shape)
            x["p"].tofile(f"{d}/src.bin")
            run_ref(["gradient", L, R_MIN, R_MAX, bcc, bcs, d], d)
            out[f"gradient_{bcc}{bcs}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)

        x["k"].tofile(f"{d}/k.bin")
        x["u"].tofile(f"{d}/src_u.bin")
        x["p"].tofile(f"{d}/src_p.bin")
        for bcc, bcs in STOKES_OP_BCS:
            run_ref(["stokes", L, R_MIN, R_MAX, bcc, bcs, d], d)
            out[f"stokes_u_{bcc}{bcs}"] = np.fromfile(f"{d}/dst_u.bin").reshape((3,) + fine.shape)
            out[f"stokes_p_{bcc}{bcs}"] = np.fromfile(f"{d}/dst_p.bin").reshape(coarse.shape)

        cg_rhs(x["s"]).tofile(f"{d}/b.bin")
        C = CHEBYSHEV_CASE
        info = run_ref(["laplace_chebyshev", L, R_MIN, R_MAX, C["order"], C["iters"], C["pits"], d], d, threads=1,
                       json_out=True)
        out["chebyshev_x"] = np.fromfile(f"{d}/x.bin").reshape(fine.shape)
        out["chebyshev_lambda"] = np.array(info["lambda"])
        out["power_start"] = np.fromfile(f"{d}/start.bin").reshape(fine.shape)
        B = BICGSTAB_CASE
        run_ref(["laplace_bicgstab", L, R_MIN, R_MAX, B["l"], B["maxit"], B["tol"], d], d)
        out["bicgstab_x"] = np.fromfile(f"{d}/x.bin").reshape(fine.shape)
        out["bicgstab_hist"] = np.fromfile(f"{d}/hist.bin")
        out["bicgstab_rshadow"] = np.fromfile(f"{d}/rshadow.bin").reshape(fine.shape)
        run_ref(["laplace_minres", L, R_MIN, R_MAX, MINRES_CASE["maxit"], MINRES_CASE["tol"], d], d)
        out["minres_x"] = np.fromfile(f"{d}/x.bin").reshape(fine.shape)
        out["minres_hist"] = np.fromfile(f"{d}/hist.bin")
        F = FGMRES_CASE
        run_ref(["laplace_fgmres", L, R_MIN, R_MAX, F["restart"], F["maxit"], F["tol"], d], d)
        out["fgmres_x"] = np.fromfile(f"{d}/x.bin").reshape(fine.shape)
        out["fgmres_hist"] = np.fromfile(f"{d}/hist.bin")

        S = STOKES_FGMRES
        x["k"].tofile(f"{d}/k.bin")
        pressure_viscosity(x).tofile(f"{d}/kp.bin")
        x["u"].tofile(f"{d}/src_u.bin")
        x["p"].tofile(f"{d}/src_p.bin")
        for bcc, bcs in S["bcs"]:
            run_ref(["stokes_fgmres", L, R_MIN, R_MAX, bcc, bcs, S["restart"], S["maxit"], S["tol"], S["sweeps"],
                     S["omega"], d], d)
            out[f"stokes_fgmres_u_{bcc}{bcs}"] = np.fromfile(f"{d}/x_u.bin").reshape((3,) + fine.shape)
            out[f"stokes_fgmres_p_{bcc}{bcs}"] = np.fromfile(f"{d}/x_p.bin").reshape(coarse.shape)
            out[f"stokes_fgmres_hist_{bcc}{bcs}"] = np.fromfile(f"{d}/hist.bin")

        S = STOKES_MINRES
        for bcc, bcs in S["bcs"]:
            run_ref(["stokes_minres", L, R_MIN, R_MAX, bcc, bcs, S["maxit"], S["tol"], S["sweeps"], S["omega"], d], d)
            out[f"stokes_minres_u_{bcc}{bcs}"] = np.fromfile(f"{d}/x_u.bin").reshape((3,) + fine.shape)
            out[f"stokes_minres_p_{bcc}{bcs}"] = np.fromfile(f"{d}/x_p.bin").reshape(coarse.shape)
            out[f"stokes_minres_hist_{bcc}{bcs}"] = np.fromfile(f"{d}/hist.bin")

        ks, kb = kvcycle_inputs()
        out["checksum_kvcycle_b"] = checksum(kb)
        K = KVCYCLE
        for level, k in zip(range(K["lmin"], K["lmax"] + 1), ks):
            k.tofile(f"{d}/k{level}.bin")
        kb.tofile(f"{d}/b.bin")
        run_ref(["kerngen_vcycle", K["lmin"], K["lmax"], R_MIN, R_MAX, *K["bcs"], K["omega"], K["smooth"],
                 K["cycles"], K["cmaxit"], d], d)
        out["kvcycle_x"] = np.fromfile(f"{d}/x.bin").reshape(kb.shape)

        vb = vcycle_rhs()
        out["checksum_vcycle_b"] = checksum(vb)
        vb.tofile(f"{d}/b.bin")
        V = VCYCLE
        run_ref(["vcycle", V["lmin"], V["lmax"], R_MIN, R_MAX, V["omega"], V["smooth"], V["cycles"], V["cmaxit"], d], d)
        out["vcycle_x"] = np.fromfile(f"{d}/x.bin").reshape(vb.shape)

        x["uc"].tofile(f"{d}/src.bin")
        run_ref(["prolong", L, R_MIN, R_MAX, d], d)
        out["prolong"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)
        x["u"].tofile(f"{d}/src.bin")
        run_ref(["restrict", L, R_MIN, R_MAX, d], d)
        out["restrict"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + coarse.shape)

        x["pc"].tofile(f"{d}/src.bin")
        run_ref(["prolong_linear", L, R_MIN, R_MAX, d], d)
        out["prolong_linear"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
        x["s"].tofile(f"{d}/src.bin")
        run_ref(["restrict_linear", L, R_MIN, R_MAX, d], d)
        out["restrict_linear"] = np.fromfile(f"{d}/dst.bin").reshape(coarse.shape)

        x["k"].tofile(f"{d}/k.bin")
        x["s"].tofile(f"{d}/src.bin")
        for mode in KMASS_MODES:
            run_ref(["kmass", L, R_MIN, R_MAX, mode, d], d)
            out[f"kmass_{mode}"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
        for mode in MASS_MODES:
            run_ref(["mass", L, R_MIN, R_MAX, mode, d], d)
            out[f"mass_{mode}"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
        x["u"].tofile(f"{d}/src.bin")
        for mode in VMASS_MODES:
            run_ref(["vmass", L, R_MIN, R_MAX, mode, d], d)
            out[f"vmass_{mode}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)
        x["u"].tofile(f"{d}/src.bin")
        for treat, diag in EPSDIVDIV_CASES:
            run_ref(["epsdivdiv", L, R_MIN, R_MAX, treat, diag, d], d)
            out[f"epsdivdiv_{treat}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)
        x["s"].tofile(f"{d}/src.bin")
        for treat, diag, single in DIVKGRAD_CASES:
            run_ref(["divkgrad", L, R_MIN, R_MAX, treat, diag, single, d], d)
            out[f"divkgrad_{treat}{diag}{single}"] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
        x["u"].tofile(f"{d}/src.bin")
        for bcc, bcs, diag in VLAPLACE_CASES:
            run_ref(["vlaplace", L, R_MIN, R_MAX, bcc, bcs, diag, d], d)
            out[f"vlaplace_{bcc}{bcs}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + fine.shape)
        # unpreconditioned PCG on the Laplace, homogeneous Dirichlet right-hand side
        cg_rhs(x["s"]).tofile(f"{d}/b.bin")
        info = run_ref(["laplace_cg", L, R_MIN, R_MAX, CG_MAXIT, CG_TOL, d], d, json_out=True)
        out["laplace_cg_x"] = np.fromfile(f"{d}/x.bin").reshape(fine.shape)
        out["laplace_cg_iterations"] = np.array(info["iterations"])
        # FCT: one fct_explicit_step on a rotation-dominated velocity
        vel, T, src = fct_inputs(fine)
        vel.tofile(f"{d}/vel.bin")
        for kappa, bc in FCT_CASES:
            T.tofile(f"{d}/T.bin")
            src.tofile(f"{d}/src.bin")
            run_ref(["fct", L, R_MIN, R_MAX, -1, kappa, bc, d], d)
            tag = f"fct_{kappa:g}_{bc}"
            out[tag + "_dt"] = np.fromfile(f"{d}/dt.bin")
            out[tag + "_T"] = np.fromfile(f"{d}/T.bin").reshape(fine.fv_shape)
            out[tag + "_TL"] = np.fromfile(f"{d}/TL.bin").reshape(fine.fv_shape)
        out["fct_centers"] = np.fromfile(f"{d}/centers.bin").reshape((3,) + fine.fv_shape)
    path = os.path.join(HERE, f"ref_L{L}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


# UnsteadyAdvectionDiffusionSUPG: (kappa, dt, mass_scaling, lumped, treat_boundary, diagonal)
SUPG_CASES = [(1e-3, 1e-2, 1.0, 0, 0, 0), (1e-2, 5e-2, 1.5, 1, 1, 0), (0.0, 1e-2, 1.0, 0, 1, 1), (1e-3, 1e-2, 1.0, 0, 1, 0),
              (1e-4, 2e-2, 1.0, 1, 0, 1)]


def supg_inputs(fine):
    """seeded velocity [3][nodes] (magnitude about 0.5) and source, both consistent on duplicated nodes"""
    rs = np.random.RandomState(66)
    vel = np.stack([fine.make_consistent(rs.normal(size=fine.shape)).reshape(fine.shape) for _ in range(3)]) * 0.5
    src = fine.make_consistent(rs.normal(size=fine.shape)).reshape(fine.shape)
    return vel, src


def make_supg():
    """adds supg_* (and the inputs' checksums) to ref_L2.npz, keeping the other entries as they are"""
    fine = Mesh(L)
    path = os.path.join(HERE, "ref_L2.npz")
    out = dict(np.load(path))
    vel, src = supg_inputs(fine)
    out["checksum_supg_vel"], out["checksum_supg_src"] = checksum(vel), checksum(src)
    with tempfile.TemporaryDirectory() as d:
        vel.tofile(f"{d}/vel.bin")
        src.tofile(f"{d}/src.bin")
        for case in SUPG_CASES:
            run_ref(["supg", L, R_MIN, R_MAX, *case, d], d)
            out["supg_" + "_".join(str(c) for c in case)] = np.fromfile(f"{d}/dst.bin").reshape(fine.shape)
    np.savez_compressed(path, **out)
    print("wrote", path)


# Adaptive GCA over levels 3 (fine), 2 (coarse) and 1 (coarsest, the marks): (bcc, bcs, diag) of the coarse apply
AGCA_L = 3
AGCA_CASES = [(1, 1, 0), (2, 2, 0), (0, 0, 0), (2, 1, 1)]


def blob_viscosity(mesh, centre=(0.6, 0.3, 0.4), amp=400.0, width=0.01):
    """1 + amp exp(-|x - centre|^2 / width) at the nodes: a sharp blob the GCA element collector marks only
    around"""
    x = mesh.coords[:, :, :, None, :] * mesh.radii[:, None, None, :, None]
    return 1.0 + amp * np.exp(-np.sum((x - np.array(centre)) ** 2, axis=-1) / width)


def agca_inputs():
    fine, coarse = Mesh(AGCA_L), Mesh(AGCA_L - 1)
    src = np.random.RandomState(91).normal(size=(3,) + coarse.shape)
    return fine, coarse, blob_viscosity(fine), blob_viscosity(coarse), src


def make_agca():
    """adds agca_marks and agca_<bcc><bcs><diag> (and the source's checksum) to ref_L2.npz"""
    path = os.path.join(HERE, "ref_L2.npz")
    out = dict(np.load(path))
    fine, coarse, k, kc, src = agca_inputs()
    out["checksum_agca_src"] = checksum(src)
    z = Mesh(AGCA_L - 2)
    with tempfile.TemporaryDirectory() as d:
        k.tofile(f"{d}/k.bin")
        kc.tofile(f"{d}/kc.bin")
        src.tofile(f"{d}/src.bin")
        for bcc, bcs, diag in AGCA_CASES:
            run_ref(["agca", AGCA_L, R_MIN, R_MAX, bcc, bcs, diag, d], d)
            out[f"agca_{bcc}{bcs}{diag}"] = np.fromfile(f"{d}/dst.bin").reshape((3,) + coarse.shape)
        g = np.fromfile(f"{d}/gcae.bin").reshape(z.shape)
        out["agca_marks"] = (g[:, :-1, :-1, :-1] != 0).astype(np.uint8)
    np.savez_compressed(path, **out)
    print("wrote", path)


# The checkpoint fixture: io::XDMFOutput<double> on the L2 mesh with FP32 points and int64 connectivity, the
# grids of XDMF_GRIDS (label, input bytes, output bytes, vec_dim) filled from the FE temperature of
# timestep_inputs and the velocity u of inputs(); two writes, the second with T + 1 and 2 u.
XDMF_DIR = os.path.join(HERE, "xdmf_L2")
XDMF_GRIDS = [("T", 8, 4, 1), ("T64", 8, 8, 1), ("s32", 4, 4, 1), ("u", 8, 4, 3), ("u64", 8, 8, 3), ("v32", 4, 8, 3)]
XDMF_PTS, XDMF_CONN = 4, 8


def xdmf_fields(fine, coarse, step):
    """the grids written at `step`: [(label, in_bytes, out_bytes, vec, data)] with data as the writer holds it"""
    _, T = timestep_inputs(fine)
    u = inputs(fine, coarse)["u"]
    t, w = T + step, u * (1 + step)
    data = {"T": t, "T64": t, "s32": t.astype(np.float32), "u": w, "u64": w, "v32": w.astype(np.float32)}
    return [(lab, ib, ob, v, data[lab]) for lab, ib, ob, v in XDMF_GRIDS]


def make_xdmf():
    import shutil
    fine, coarse = Mesh(L), Mesh(L - 1)
    _, T = timestep_inputs(fine)
    u = inputs(fine, coarse)["u"]
    with tempfile.TemporaryDirectory() as d:
        T.tofile(f"{d}/T.bin")
        u.tofile(f"{d}/u.bin")
        run_ref(["xdmf_write", L, R_MIN, R_MAX, XDMF_PTS, XDMF_CONN, d], d)
        os.makedirs(XDMF_DIR, exist_ok=True)
        for f in sorted(os.listdir(f"{d}/xdmf")):
            shutil.copyfile(f"{d}/xdmf/{f}", os.path.join(XDMF_DIR, f))


# The distributed domain as rank q of P (subdomain refinement level 0, the reference's default rank map): the
# diamonds of every rank for P = 1..10, and the copy-wise (SkipCommunication) kerngen apply of the ranks of
# SHARD_APPLY_P with the boundary conditions SHARD_BCS on the seeded inputs of shard_inputs.
SHARD_L = 2
SHARD_APPLY_P = (3, 8)
SHARD_BCS = [(1, 2), (2, 0)]


def shard_inputs(fine):
    """seeded positive k and a source, both consistent on duplicated nodes"""
    rs = np.random.RandomState(123)
    k = fine.make_consistent(np.exp(rs.normal(size=fine.shape))).reshape(fine.shape)
    src = np.stack([fine.make_consistent(rs.normal(size=fine.shape)).reshape(fine.shape) for _ in range(3)])
    return k, src


def make_shard():
    """shard_L2.npz: diamonds_P<P>_q<q> (the reference's local subdomains, in local order) and
    dst_<bcc><bcs>_P<P>_q<q> (the rank's copy-wise apply), plus the inputs' checksums"""
    fine = Mesh(SHARD_L)
    k, src = shard_inputs(fine)
    out = {"checksum_k": checksum(k), "checksum_src": checksum(src)}
    with tempfile.TemporaryDirectory() as d:
        for P in range(1, 11):
            first = 0
            for q in range(P):
                # the rank's diamonds are not known before the run: a first run reads the leading entries of the
                # whole shell's fields and reports them; the apply runs again on the rank's own slices
                k.tofile(f"{d}/k.bin")
                src.tofile(f"{d}/src.bin")
                info = run_ref(["kerngen_rank", SHARD_L, R_MIN, R_MAX, 1, 2, P, q, d], d, json_out=True)
                dia = np.array(info["diamonds"], np.int32)
                out[f"diamonds_P{P}_q{q}"] = dia
                assert dia[0] == first and np.all(np.diff(dia) == 1), dia
                first = dia[-1] + 1
                if P not in SHARD_APPLY_P:
                    continue
                sl = slice(int(dia[0]), int(dia[-1]) + 1)
                k[sl].tofile(f"{d}/k.bin")
                np.ascontiguousarray(src[:, sl]).tofile(f"{d}/src.bin")
                for bcc, bcs in SHARD_BCS:
                    run_ref(["kerngen_rank", SHARD_L, R_MIN, R_MAX, bcc, bcs, P, q, d], d)
                    out[f"dst_{bcc}{bcs}_P{P}_q{q}"] = np.fromfile(f"{d}/dst.bin").reshape((3, len(dia)) + fine.shape[1:])
            assert first == 10
    path = os.path.join(HERE, "shard_L2.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    if "--stokes-mg" in sys.argv and "--stokes-mg-inputs" not in sys.argv:
        make_stokes_mg()
    elif "--xdmf" in sys.argv:
        make_xdmf()
    elif "--supg" in sys.argv:
        make_supg()
    elif "--agca" in sys.argv:
        make_agca()
    elif "--stokes-mg-inputs" in sys.argv:
        make_stokes_mg_inputs()
    elif "--shard" in sys.argv:
        make_shard()
    else:
        main()
