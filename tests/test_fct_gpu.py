"""Finite-volume FCT advection-diffusion against the oracle (pinned to the
reference's fct_explicit_step, compute_dt_stable and ghost-layer exchange)."""
import numpy as np
import pytest
import torch

from helpers import rel
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


def _case(om, seed=0):
    """rotation-dominated Q1 velocity, smooth FV temperature with a jump, small source"""
    rng = np.random.default_rng(seed)
    x = om.coords[:, :, :, None, :] * om.radii[:, None, None, :, None]
    w = rng.normal(size=3)
    vel = np.cross(np.broadcast_to(w, x.shape), x)
    vel += 0.2 * np.stack([np.sin(3 * x[..., 1]), np.cos(2 * x[..., 2]), np.sin(4 * x[..., 0])], axis=-1)
    vel = om.make_consistent(np.ascontiguousarray(np.moveaxis(vel, -1, 0)))
    c = om.fv_cell_centers()
    N = om.N
    inner = (slice(None), slice(1, N + 1), slice(1, N + 1), slice(1, N + 1))
    T = np.zeros(om.fv_shape)
    cc = c[(slice(None),) + inner]
    T[inner] = 0.5 + 0.3 * np.sin(4 * cc[0]) * np.cos(3 * cc[1]) + 0.2 * (cc[2] > 0)
    src = np.zeros(om.fv_shape)
    src[inner] = 0.1 * np.cos(cc[0])
    return vel, c, T, src, inner


@pytest.fixture(scope="module", params=[2, 4])
def level(request):
    from terraneo_b200 import shell
    L = request.param
    om, pm = Mesh(L), shell.ShellMesh(L)
    return om, pm, shell.FCTAdvectionDiffusion(pm)


def test_cell_centers_and_ghosts(level):
    om, pm, fct = level
    assert rel(fct.centers.cpu().numpy(), om.fv_cell_centers()) <= 1e-14
    f = np.random.default_rng(1).normal(size=om.fv_shape)
    g = torch.as_tensor(f, device="cuda")
    fct.ghost_update(g)
    assert np.array_equal(g.cpu().numpy(), om.fv_ghost_update(f))


@pytest.mark.parametrize("kappa", [0.0, 1e-2])
def test_dt_stable(level, kappa):
    from terraneo_b200 import shell
    om, pm, fct = level
    vel, c, T, src, inner = _case(om)
    v = shell.VectorQ1Vec(pm)
    v.set_numpy(vel)
    assert fct.dt_stable(v, kappa) == pytest.approx(om.fct_dt_stable(c, vel, kappa), rel=1e-13)


@pytest.mark.parametrize("kappa,bc,with_src", [(0.0, False, False), (0.0, True, True), (1e-2, True, True),
                                               (1e-2, False, True)])
def test_fct_step_matches_oracle(level, kappa, bc, with_src):
    from terraneo_b200 import shell
    om, pm, fct = level
    vel, c, T, src, inner = _case(om, seed=3)
    v = shell.VectorQ1Vec(pm)
    v.set_numpy(vel)
    bcs = fct.dirichlet(1.0, 0.0) if bc else None
    T0 = om.fct_dirichlet(T) if bc else T.copy()
    dt = 0.5 * om.fct_dt_stable(c, vel, kappa)
    ref, ref_TL = om.fct_step(c, vel, om.fv_ghost_update(T0), dt, kappa, src if with_src else None, True,
                              (1.0, 0.0, 1, 1) if bc else None)
    Tg = torch.as_tensor(T0, device="cuda")
    sg = torch.as_tensor(src, device="cuda") if with_src else None
    fct.step(Tg, v, dt, kappa, sg, True, bcs)
    out = Tg.cpu().numpy()
    assert rel(out[inner], ref[inner]) <= 1e-13
    assert rel(fct.T_L.cpu().numpy()[inner], ref_TL[inner]) <= 1e-13


def test_fct_is_bounded_for_pure_advection():
    """The limiter keeps a divergence-free advected field within its initial bounds."""
    from terraneo_b200 import shell
    L = 4
    om, pm = Mesh(L), shell.ShellMesh(L)
    fct = shell.FCTAdvectionDiffusion(pm)
    x = om.coords[:, :, :, None, :] * om.radii[:, None, None, :, None]
    vel = np.cross(np.broadcast_to(np.array([0.0, 0.0, 1.0]), x.shape), x)  # rigid rotation
    vel = om.make_consistent(np.ascontiguousarray(np.moveaxis(vel, -1, 0)))
    v = shell.VectorQ1Vec(pm)
    v.set_numpy(vel)
    c = fct.centers.cpu().numpy()
    N = om.N
    inner = (slice(1, None), slice(1, N + 1), slice(1, N + 1), slice(1, N + 1))
    T = np.zeros(om.fv_shape)
    T[:, 1:N + 1, 1:N + 1, 1:N + 1] = (c[0][:, 1:N + 1, 1:N + 1, 1:N + 1] > 0.2).astype(float)
    Tg = torch.as_tensor(T, device="cuda")
    dt = 0.5 * fct.dt_stable(v)
    for _ in range(10):
        fct.step(Tg, v, dt)
    out = Tg.cpu().numpy()[:, 1:N + 1, 1:N + 1, 1:N + 1]
    assert out.min() >= -1e-12 and out.max() <= 1 + 1e-12
