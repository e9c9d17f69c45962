"""Adjoint viscosity gradient: the backward kernel against the oracle operator
(exact identity) and the whole gradient against central finite differences."""
import numpy as np
import pytest
import torch

from helpers import random_vector, rel, viscosity_field
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bc", [(1, 1), (2, 2), (2, 1), (1, 2), (0, 0), (0, 1)])
def test_kgrad_is_the_k_derivative_of_the_form(bc):
    """sum_n grad_n delta_n = lambda^T A(delta) u - lambda^T A(0) u for any u, lambda, delta
    (A linear in k; A(0) is the k-independent rigid-rotation penalty)."""
    from terraneo_b200 import _capi as C, shell
    L = 3
    om, pm = Mesh(L), shell.ShellMesh(L)
    u, lam = random_vector(om, seed=1), random_vector(om, seed=2)
    delta = random_vector(om, seed=3, ncomp=1)
    vu, vl = shell.VectorQ1Vec(pm), shell.VectorQ1Vec(pm)
    vu.set_numpy(u)
    vl.set_numpy(lam)
    g_add, g_skip = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    shell.epsdivdiv_kgrad(pm, bc[0], bc[1], vu, vl, g_add, C.COMM_ADDITIVE)
    shell.epsdivdiv_kgrad(pm, bc[0], bc[1], vu, vl, g_skip, C.COMM_SKIP)
    torch.cuda.synchronize()
    rhs = om.dot(lam, om.kerngen(delta, u, bc[0], bc[1])) - om.dot(lam, om.kerngen(0 * delta, u, bc[0], bc[1]))
    lhs_add = om.dot(g_add.numpy()[0], delta)
    lhs_skip = float((g_skip.numpy()[0] * delta).sum())
    assert abs(lhs_add - rhs) <= 1e-12 * abs(rhs)
    assert abs(lhs_skip - rhs) <= 1e-12 * abs(rhs)
    # copies summed: the additive result is the halo sum of the copy-wise one
    assert rel(g_add.numpy()[0], om.halo_sum(g_skip.numpy()[0])) <= 1e-13


def _smooth_direction(om, seed):
    rng = np.random.default_rng(seed)
    x = om.coords[:, :, :, None, :] * om.radii[:, None, None, :, None]
    f = np.zeros(om.shape)
    for _ in range(4):
        c = rng.normal(size=3)
        c = c / np.linalg.norm(c) * rng.uniform(0.6, 0.95)
        f += rng.normal() * np.exp(-np.sum((x - c) ** 2, axis=-1) / (2 * 0.2 ** 2))
    return f / np.abs(f).max()


@pytest.mark.parametrize("bc", [(1, 1), (2, 2)])
def test_viscosity_gradient_matches_central_differences(bc):
    from terraneo_b200 import shell
    from terraneo_b200.adjoint import stokes_velocity
    L = 3
    om, pf, pc = Mesh(L), shell.ShellMesh(L), shell.ShellMesh(L - 1)
    k0 = viscosity_field(om, seed=7, contrast=1e2)
    m0 = np.log(k0)
    kw = dict(mg_levels=2, bc_cmb=bc[0], bc_surface=bc[1], mg_fp32=False, relative_tolerance=1e-14,
              max_iterations=600, restart=100, coarse_max_iterations=200, coarse_relative_tolerance=1e-12)
    f = random_vector(om, seed=8)
    if bc[0] == 1:
        f[:, :, :, :, 0] = 0
    if bc[1] == 1:
        f[:, :, :, :, -1] = 0
    fu, fp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    fu.set_numpy(f)
    fu.halo_sum()
    if 2 in bc:
        shell.freeslip_project(fu, bc[0] == 2, bc[1] == 2)
    owned = torch.as_tensor(om.omask.astype(np.float64), device="cuda")
    # observations from a perturbed viscosity
    m_obs = torch.as_tensor(m0 + 0.3 * _smooth_direction(om, 11), device="cuda")
    u_obs = stokes_velocity(m_obs, L, fu, fp, **kw).detach()

    def J(m):
        u = stokes_velocity(m, L, fu, fp, **kw)
        return 0.5 * (owned * (u - u_obs) ** 2).sum()

    m = torch.as_tensor(m0, device="cuda").requires_grad_(True)
    j = J(m)
    j.backward()
    grad = m.grad.detach()
    h = 1e-5
    errs = []
    for s in range(3):
        d = torch.as_tensor(_smooth_direction(om, 100 + s), device="cuda")
        with torch.no_grad():
            fd = (J(m.detach() + h * d) - J(m.detach() - h * d)).item() / (2 * h)
        ad = float((grad * d).sum())
        errs.append(abs(fd - ad) / abs(ad))
    assert max(errs) <= 1e-6, errs
