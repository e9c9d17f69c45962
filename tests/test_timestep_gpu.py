"""The pieces of the mantle-circulation time step around the Stokes solve and the FCT step, through the C ABI,
against the oracle (pinned to the reference by tests/test_oracle_pinning.py) and the golden fixture: the FV ->
FE L2 projection (consistent and lumped), the Stokes buoyancy right-hand side, the pressure normalisation, and
one whole step of shell.MantleTimestep checked piece by piece."""
import os
import sys

import numpy as np
import pytest
import torch

from helpers import rel, viscosity_field
from oracle_lib import Mesh

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_L2.npz")


def _fields(L, seed):
    om = Mesh(L)
    rs = np.random.RandomState(seed)
    fv = rs.normal(size=om.fv_shape)
    T = om.make_consistent(rs.uniform(size=om.shape)).reshape(om.shape)
    return om, fv, T


@pytest.mark.parametrize("lumped", [False, True])
@pytest.mark.parametrize("L", [2, 3])
def test_l2_projection_matches_oracle_and_reference(L, lumped):
    from terraneo_b200 import shell
    if L == 2:
        om = Mesh(L)
        fv, _ = G.timestep_inputs(om)
        ref = np.load(GOLDEN)[f"l2proj_{int(lumped)}"]
    else:
        om, fv, _ = _fields(L, 3)
        ref = om.l2_project_fv_to_fe(fv, lumped=lumped)
    pm = shell.ShellMesh(L)
    x = shell.VectorQ1Scalar(pm)
    its = shell.l2_project_fv_to_fe(pm, torch.as_tensor(fv, device="cuda"), x, lumped=lumped)
    assert rel(x.numpy()[0], ref) <= (1e-12 if lumped else 1e-10), its
    if not lumped:
        assert its > 0


@pytest.mark.parametrize("bc", G.STOKES_RHS_BCS)
def test_buoyancy_rhs_matches_reference(bc):
    from terraneo_b200 import shell
    om = Mesh(G.L)
    _, T = G.timestep_inputs(om)
    pm = shell.ShellMesh(G.L)
    Tv, f = shell.VectorQ1Scalar(pm), shell.VectorQ1Vec(pm)
    Tv.set_numpy(T)
    shell.stokes_buoyancy_rhs(pm, Tv, G.STOKES_RHS_RA, bc[0], bc[1], f)
    g = np.load(GOLDEN)
    assert rel(f.numpy(), g[f"stokes_rhs_{bc[0]}{bc[1]}"]) <= 1e-12
    om3 = Mesh(3)
    _, _, T3 = _fields(3, 4)
    pm3 = shell.ShellMesh(3)
    Tv3, f3 = shell.VectorQ1Scalar(pm3), shell.VectorQ1Vec(pm3)
    Tv3.set_numpy(T3)
    shell.stokes_buoyancy_rhs(pm3, Tv3, 3e4, bc[0], bc[1], f3)
    assert rel(f3.numpy(), om3.stokes_buoyancy_rhs(T3, 3e4, *bc)) <= 1e-12


def test_pressure_mean_removal():
    from terraneo_b200 import shell
    L = 3
    om = Mesh(L)
    p = om.make_consistent(np.random.default_rng(5).normal(size=om.shape) + 2.0).reshape(om.shape)
    pm = shell.ShellMesh(L)
    pv = shell.VectorQ1Scalar(pm)
    pv.set_numpy(p)
    mean = shell.pressure_remove_mean(pv)
    expect = om.dot(p, np.ones(om.shape)) / pm.unique_nodes
    assert abs(mean - expect) <= 1e-14 * abs(expect)
    assert rel(pv.numpy()[0], p - expect) <= 1e-15
    assert abs(om.dot(pv.numpy()[0], np.ones(om.shape))) <= 1e-10 * pm.unique_nodes


def test_mantle_timestep_pieces_match_oracle():
    """One time step of shell.MantleTimestep at level 3 (free-slip both radii), each piece against the oracle
    on the step's own intermediates: the right-hand side from the projected temperature, the true residual of
    the Stokes solution, the zero pressure mean, the FCT step with the computed velocity, and the projection of
    the advected temperature; a second (warm-started) step stays finite."""
    from terraneo_b200 import shell
    L = 3
    om, oc = Mesh(L), Mesh(L - 1)
    c = om.fv_cell_centers()
    rr = np.sqrt((c ** 2).sum(0)).clip(1e-30)
    T0 = ((1 / rr - 1.0) / (1 / 0.55 - 1.0)).clip(0, 1) + 0.05 * np.sin(4 * c[0]) * np.cos(3 * c[1])
    k = viscosity_field(om, seed=9, contrast=1e2)
    pm = shell.ShellMesh(L)
    kv = shell.VectorQ1Scalar(pm)
    kv.set_numpy(k)
    Tg = torch.as_tensor(T0, device="cuda")
    ts = shell.MantleTimestep(L, kv, Tg, rayleigh=1e4, mg_levels=2, mg_fp32=False, relative_tolerance=1e-10,
                              max_iterations=600, restart=50, gca=1)
    # the initial projection (Dirichlet temperatures applied first)
    T_fv0 = om.fct_dirichlet(T0)
    assert rel(ts.T.numpy()[0], om.l2_project_fv_to_fe(T_fv0)) <= 1e-10
    T_fe0 = ts.T.numpy()[0].copy()
    assert ts.step()
    info = ts.last
    # right-hand side of the step
    f = om.stokes_buoyancy_rhs(T_fe0, 1e4, 2, 2)
    assert rel(ts.f_u.numpy(), f) <= 1e-12
    # the Stokes solution: true residual with the oracle operators, with the pressure the solve returned (the
    # normalisation shifts p after the solve; with free-slip radii B^T 1 is not zero at the boundary nodes, whose
    # normal is projected out with the node's radial direction, not the discrete faces' normals)
    u, p = ts.u.numpy(), ts.p.numpy()[0]
    ru = om.kerngen(k, u, 2, 2) + om.gradient(oc, p + info["pressure_mean_removed"], 2, 2) - f
    rp = om.divergence(oc, u, 2, 2)
    assert np.sqrt(om.dot(ru, ru) + oc.dot(rp, rp)) / np.sqrt(om.dot(f, f)) <= 1e-8, info
    assert abs(oc.dot(p, np.ones(oc.shape))) <= 1e-12 * np.abs(p).max() * oc.ns
    # the FCT step with that velocity, then the projection
    dt = 0.5 * om.fct_dt_stable(c, u, 0.0)
    assert info["dt"] == pytest.approx(dt, rel=1e-12)
    T1, _ = om.fct_step(c, u, om.fv_ghost_update(T_fv0), info["dt"], 0.0, None, True, (1.0, 0.0, 1, 1))
    T1 = om.fct_dirichlet(T1)
    N = om.N
    inner = (slice(None), slice(1, N + 1), slice(1, N + 1), slice(1, N + 1))
    assert rel(ts.T_fv.cpu().numpy()[inner], T1[inner]) <= 1e-12
    # the step's projection is warm-started from the previous FE temperature, the oracle's from zero: both
    # PCG runs stop at 1e-12 of their own initial residual, so the iterates agree to the mass matrix's
    # condition number times that
    assert rel(ts.T.numpy()[0], om.l2_project_fv_to_fe(ts.T_fv.cpu().numpy())) <= 1e-9
    assert ts.step() and ts.last["finite"]
