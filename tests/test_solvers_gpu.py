"""Solver drivers through the C ABI: PCG on the Laplace and the Stokes solve
(FP64 and FP32 multigrid), checked against oracle operators."""
import numpy as np
import pytest
import torch

from helpers import random_vector, rel, viscosity_field
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


def oracle_pcg(om, b, tol, maxit=2000):
    """Unpreconditioned CG with the oracle Laplace (pcg.hpp:78-160)."""
    x = np.zeros_like(b)
    r = b - om.laplace(x)
    p = r.copy()
    r0 = np.sqrt(om.dot(r, r))
    for it in range(1, maxit + 1):
        an = om.dot(r, r)
        ap = om.laplace(p)
        alpha = an / om.dot(ap, p)
        x += alpha * p
        r -= alpha * ap
        rr = np.sqrt(om.dot(r, r)) / r0
        if rr <= tol:
            return x, it, rr
        p = r + (om.dot(r, r) / an) * p
    return x, maxit, rr


def test_laplace_pcg_matches_oracle_cg():
    from terraneo_b200 import shell
    L = 3
    om, pm = Mesh(L), shell.ShellMesh(L)
    b = random_vector(om, seed=11, ncomp=1)
    b[om.bmask != 1] = 0.0  # homogeneous Dirichlet rows
    xo, ito, rro = oracle_pcg(om, b, 1e-10)
    vb, vx = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    vb.set_numpy(b)
    it, rr = shell.laplace_pcg(pm, vb, vx, relative_tolerance=1e-10)
    assert rr <= 1e-10
    assert abs(it - ito) <= 2
    assert rel(vx.numpy()[0], xo) <= 1e-7


@pytest.fixture(scope="module")
def stokes_case():
    L = 4
    of, oc = Mesh(L), Mesh(L - 1)
    k = viscosity_field(of, seed=5, contrast=1e2)
    f = random_vector(of, seed=21)
    return L, of, oc, k, f


@pytest.mark.parametrize("mg_fp32", [False, True])
def test_stokes_solve_true_residual(stokes_case, mg_fp32):
    from terraneo_b200 import shell
    L, of, oc, k, f = stokes_case
    pf, pc = shell.ShellMesh(L), shell.ShellMesh(L - 1)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k)
    fu, fp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    fu.set_numpy(f)
    shell.freeslip_project(fu)
    xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    solver = shell.StokesSolver(L, kv, mg_levels=2, mg_fp32=mg_fp32, relative_tolerance=1e-8, max_iterations=300)
    it, rr = solver.solve(fu, fp, xu, xp)
    torch.cuda.synchronize()
    assert rr <= 1e-8, (it, rr)
    # true FP64 residual with the oracle operators
    u, p, b = xu.numpy(), xp.numpy()[0], fu.numpy()
    ru = of.kerngen(k, u, 2, 2) + of.gradient(oc, p, 2, 2) - b
    rp = of.divergence(oc, u, 2, 2)
    res = np.sqrt(of.dot(ru, ru) + oc.dot(rp, rp)) / np.sqrt(of.dot(b, b))
    assert res <= 2e-8, res
    hist, skips = solver.history()
    assert hist[0] == 1.0 and skips == 0


def test_stokes_fp32_mg_matches_fp64_mg(stokes_case):
    from terraneo_b200 import shell
    L, of, oc, k, f = stokes_case
    pf, pc = shell.ShellMesh(L), shell.ShellMesh(L - 1)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k)
    fu, fp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    fu.set_numpy(f)
    shell.freeslip_project(fu)
    sols = []
    for mg32 in (False, True):
        xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
        s = shell.StokesSolver(L, kv, mg_levels=2, mg_fp32=mg32, relative_tolerance=1e-10, max_iterations=400)
        s.solve(fu, fp, xu, xp)
        sols.append(xu.numpy())
    assert rel(sols[1], sols[0]) <= 1e-7
