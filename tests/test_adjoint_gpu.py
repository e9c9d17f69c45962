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


@pytest.fixture(scope="module")
def level5_adjoint():
    """The adjoint configuration at level 5 (velocity L5 / pressure L4, Dirichlet both radii, 1e4-contrast
    viscosity): forward solution u, adjoint solution lambda and the copy-wise gradient dJ/dlog k of
    J = 1/2 sum_owned |u - u_obs|^2, every solve to 1e-14."""
    from terraneo_b200 import _capi as C, shell
    L = 5
    om, pf, pc = Mesh(L), shell.ShellMesh(L), shell.ShellMesh(L - 1)
    k0 = viscosity_field(om, seed=17, contrast=1e4)
    f = random_vector(om, seed=18)
    f[:, :, :, :, 0] = 0
    f[:, :, :, :, -1] = 0
    fu, fp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    fu.set_numpy(f)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k0)
    kw = dict(mg_levels=3, bc_cmb=1, bc_surface=1, mg_fp32=False, relative_tolerance=1e-14, max_iterations=1500,
              restart=100, coarse_max_iterations=300, coarse_relative_tolerance=1e-12)
    owned = torch.as_tensor(om.omask.astype(np.float64), device="cuda")
    u_obs = torch.as_tensor(random_vector(om, seed=19), device="cuda") * 1e-3
    solver = shell.StokesSolver(L, kv, **kw)
    xu, xp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    it, rr = solver.solve(fu, fp, xu, xp)
    assert rr <= 1e-14, (it, rr)
    gu = shell.VectorQ1Vec(pf, data=(owned * (xu.data - u_obs)).contiguous())
    lam_u, lam_p = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    grad = torch.empty(pf.shape, dtype=torch.float64, device="cuda")
    solver.viscosity_backward(xu, gu, grad, C.COMM_SKIP, lam_u, lam_p)
    return dict(om=om, pf=pf, pc=pc, k0=k0, fu=fu, fp=fp, kw=kw, owned=owned, u_obs=u_obs, u=xu.numpy(),
                p=xp.numpy(), lam=lam_u.numpy(), grad=grad.cpu().numpy(), L=L)


def test_gradient_matches_reference_directional_derivative_level5(level5_adjoint):
    """<dJ/dlog k, delta> = -lambda^T A(k o delta) u (the viscous block is linear in k), with A the reference's
    own EpsilonDivDivKerngen<double> (oracle/_ref/ref_dump, Dirichlet, Replace + halo) given k o delta as its
    coefficient field, in 8 seeded smooth directions; the oracle's kerngen when the compiled reference is
    absent (the oracle is pinned to it)."""
    import tempfile
    from oracle_lib import ref_available, run_ref
    a = level5_adjoint
    om, u, lam, grad, k0 = a["om"], a["u"], a["lam"], a["grad"], a["k0"]
    errs = []
    with tempfile.TemporaryDirectory() as d:
        u.tofile(f"{d}/src.bin")
        for s in range(8):
            delta = _smooth_direction(om, 300 + s)
            kd = np.ascontiguousarray(k0 * delta)
            if ref_available():
                kd.tofile(f"{d}/k.bin")
                run_ref(["kerngen", a["L"], 0.55, 1.0, 1, 1, 0, d], d, threads=8)
                au = np.fromfile(f"{d}/dst.bin").reshape(u.shape)
            else:
                au = om.kerngen(kd, u, 1, 1, False)
            ref = -om.dot(lam, au)
            got = float((grad * delta).sum())
            errs.append(abs(got - ref) / abs(ref))
    assert max(errs) <= 1e-12, errs


def test_gradient_matches_central_differences_level5(level5_adjoint):
    """Central differences with step 1e-6 in 4 seeded smooth directions at the level-5 configuration: the
    perturbed solves start from the unperturbed solution (FGMRES to 1e-10 of their O(h) initial residual, at
    most 150 iterations), so the difference of the two solutions is not swamped by the solver tolerance;
    agreement to 1e-7 relative (cold starts to 1e-14 agree to about 1e-5)."""
    from terraneo_b200 import shell
    a = level5_adjoint
    om, pf, pc, fu, fp, kw, owned, u_obs = (a["om"], a["pf"], a["pc"], a["fu"], a["fp"], a["kw"], a["owned"],
                                            a["u_obs"])
    m0 = torch.as_tensor(np.log(a["k0"]), device="cuda")
    grad = torch.as_tensor(a["grad"], device="cuda")
    u0, p0 = torch.as_tensor(a["u"], device="cuda"), torch.as_tensor(a["p"], device="cuda")
    kw_warm = dict(kw, relative_tolerance=1e-10, max_iterations=150)
    kv = shell.VectorQ1Scalar(pf)

    def J(m):
        kv.data[0].copy_(torch.exp(m))
        s = shell.StokesSolver(a["L"], kv, **kw_warm)
        yu = shell.VectorQ1Vec(pf, data=u0.clone())
        yp = shell.VectorQ1Scalar(pc, data=p0.clone())
        s.solve(fu, fp, yu, yp)
        return float(0.5 * (owned * (yu.data - u_obs) ** 2).sum())

    h = 1e-6
    errs = []
    for s in range(4):
        d = torch.as_tensor(_smooth_direction(om, 400 + s), device="cuda")
        fd = (J(m0 + h * d) - J(m0 - h * d)) / (2 * h)
        ad = float((grad * d).sum())
        errs.append(abs(fd - ad) / abs(ad))
    assert max(errs) <= 1e-7, errs
