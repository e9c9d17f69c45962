"""The SUPG energy operator (tn_supg_apply_*, UnsteadyAdvectionDiffusionSUPG) against the reference's outputs
(tests/golden/ref_L2.npz) and the oracle (pinned to the reference by tests/test_oracle_pinning.py), and the
implicit BDF step solved with PBiCGStab(l) (tn_supg_solve_f64) as the reference's SUPG tests take it."""
import os
import sys

import numpy as np
import pytest
import torch

from helpers import rel
from oracle_lib import Mesh

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_L2.npz")


def _op(shell, pm, vel, dtype, c, **kw):
    v = shell.VectorQ1Vec(pm, dtype)
    v.set_numpy(vel)
    kappa, dt, ms, lumped, treat, diag = c
    return shell.UnsteadyAdvectionDiffusionSUPG(pm, v, kappa, dt, bool(treat), bool(diag), ms, bool(lumped), **kw)


@pytest.mark.parametrize("c", G.SUPG_CASES)
def test_supg_apply_matches_reference(c):
    from terraneo_b200 import shell
    om = Mesh(G.L)
    vel, src = G.supg_inputs(om)
    ref = np.load(GOLDEN)["supg_" + "_".join(str(v) for v in c)]
    pm = shell.ShellMesh(G.L)
    for dtype, tol in ((torch.float64, 1e-12), (torch.float32, 2e-5)):
        op = _op(shell, pm, vel, dtype, c)
        s, d = shell.VectorQ1Scalar(pm, dtype), shell.VectorQ1Scalar(pm, dtype)
        s.set_numpy(src)
        shell.apply(op, s, d)
        assert rel(d.numpy()[0], ref) <= tol, dtype


@pytest.mark.parametrize("c", [(1e-3, 1e-2, 1.0, 0, 1, 0), (0.02, 0.05, 1.5, 1, 0, 0), (0.0, 0.03, 1.0, 0, 1, 1),
                               (1e-6, 0.1, 1.0, 0, 0, 0)])
def test_supg_apply_matches_oracle_level3(c):
    """level 3, a velocity of magnitude about 1 (so tau takes both its clamped and its coth branch) and a
    nearly vanishing diffusivity"""
    from terraneo_b200 import _capi as C, shell
    om, pm = Mesh(3), shell.ShellMesh(3)
    rs = np.random.RandomState(12)
    vel = np.stack([om.make_consistent(rs.normal(size=om.shape)).reshape(om.shape) for _ in range(3)])
    src = om.make_consistent(rs.normal(size=om.shape)).reshape(om.shape)
    kappa, dt, ms, lumped, treat, diag = c
    want = om.supg(vel, src, kappa, dt, ms, bool(lumped), bool(treat), bool(diag))
    op = _op(shell, pm, vel, torch.float64, c)
    s, d = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    s.set_numpy(src)
    shell.apply(op, s, d)
    assert rel(d.numpy()[0], want) <= 1e-12
    # the copy-wise form (no halo sum) sums to the additive one; Add mode adds the copy-wise contributions to a
    # prefilled destination (with the additive communication the halo sum would also sum the prefilled copies)
    d3 = shell.VectorQ1Scalar(pm)
    op.set_operator_apply_and_communication_modes(C.APPLY_REPLACE, C.COMM_SKIP)
    shell.apply(op, s, d3)
    copywise = d3.numpy()[0].copy()
    d3.halo_sum()
    assert rel(d3.numpy()[0], want) <= 1e-12
    d2 = shell.VectorQ1Scalar(pm)
    d2.data.fill_(1.0)
    op.set_operator_apply_and_communication_modes(C.APPLY_ADD, C.COMM_SKIP)
    shell.apply(op, s, d2)
    assert rel(d2.numpy()[0] - 1.0, copywise) <= 1e-12


def test_supg_bdf_steps():
    """BDF1 steps of the reference's SUPG test at level 3 (kappa 1e-3, dt 1e-2, PBiCGStab(2), 1e-12): every step
    solves to its tolerance and the solution satisfies the oracle's operator (true relative residual), a
    transported field stays bounded"""
    from terraneo_b200 import shell
    L = 3
    om, pm = Mesh(L), shell.ShellMesh(L)
    x = om.coords[:, :, :, None, :] * om.radii[:, None, None, :, None]
    # rigid rotation about the z axis, a Gaussian temperature blob
    vel = np.stack([-x[..., 1], x[..., 0], 0.0 * x[..., 2]])
    T0 = np.exp(-np.sum((x - np.array([0.75, 0.0, 0.2])) ** 2, axis=-1) / 0.02)
    c = (1e-3, 1e-2, 1.0, 0, 0, 0)
    op = _op(shell, pm, vel, torch.float64, c)
    M = shell.KMass(pm)
    T, f = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    T.set_numpy(T0)
    Tn = T0
    for _ in range(3):
        shell.apply(M, T, f)
        fn = f.numpy()[0]
        its, rr = op.solve(f, T, l=2, max_iterations=50, relative_tolerance=1e-12, absolute_tolerance=1e-14)
        assert rr <= 1e-12 or its < 50, (its, rr)
        Tn = T.numpy()[0]
        res = om.supg(vel, Tn, *c[:3]) - fn
        assert np.sqrt(om.dot(res, res)) <= 1e-10 * np.sqrt(om.dot(fn, fn)), (its, rr)
    assert np.abs(Tn).max() <= 1.5 and np.isfinite(Tn).all()
