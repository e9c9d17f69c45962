"""Parity of the CUDA Laplace apply with the oracle."""
import numpy as np
import pytest
import torch

from helpers import random_vector, rel
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [1, 2, 3, 4])
@pytest.mark.parametrize("treat,diag", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_laplace_f64(L, treat, diag):
    from terraneo_b200 import shell
    om = Mesh(L)
    pm = shell.ShellMesh(L)
    u = random_vector(om, seed=L, ncomp=1)
    src, dst = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    src.set_numpy(u)
    shell.apply(shell.Laplace(pm, treat, diag), src, dst)
    torch.cuda.synchronize()
    assert rel(dst.numpy()[0], om.laplace(u, treat, diag)) <= 1e-12


@pytest.mark.parametrize("L", [1, 2, 3, 4])
@pytest.mark.parametrize("treat,diag,single", [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)])
def test_divkgrad_f64(L, treat, diag, single):
    from terraneo_b200 import shell
    from helpers import viscosity_field
    om, pm = Mesh(L), shell.ShellMesh(L)
    k = viscosity_field(om, seed=L)
    u = random_vector(om, seed=10 + L, ncomp=1)
    kv, src, dst = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    kv.set_numpy(k)
    src.set_numpy(u)
    shell.apply(shell.DivKGrad(pm, kv, treat, diag, single_quadpoint=single), src, dst)
    torch.cuda.synchronize()
    assert rel(dst.numpy()[0], om.divkgrad(k, u, treat, diag, single)) <= 1e-12


def test_divkgrad_f32_and_add_mode():
    from terraneo_b200 import shell, _capi as C
    from helpers import viscosity_field
    L = 3
    om, pm = Mesh(L), shell.ShellMesh(L)
    k = viscosity_field(om, seed=5)
    u = random_vector(om, seed=6, ncomp=1)
    ref = om.divkgrad(k, u, 1, 0, 0)
    kv, src, dst = (shell.VectorQ1Scalar(pm, torch.float32) for _ in range(3))
    kv.set_numpy(k)
    src.set_numpy(u)
    shell.apply(shell.DivKGrad(pm, kv, 1), src, dst)
    assert rel(dst.numpy()[0].astype(float), ref) <= 1e-5
    k64, s64, d64 = (shell.VectorQ1Scalar(pm) for _ in range(3))
    k64.set_numpy(k)
    s64.set_numpy(u)
    d64.data.fill_(1.0)
    shell.apply(shell.DivKGrad(pm, k64, 1, apply_mode=C.APPLY_ADD), s64, d64)
    # Add mode with additive communication sums the old dst over duplicated nodes too
    assert rel(d64.numpy()[0], om.halo_sum(np.ones(om.shape)) + ref) <= 1e-12


@pytest.mark.parametrize("L", [1, 2, 3, 4])
@pytest.mark.parametrize("bcc,bcs,diag", [(0, 0, 0), (1, 1, 0), (1, 0, 0), (0, 1, 0), (1, 1, 1), (0, 0, 1)])
def test_vector_laplace_f64(L, bcc, bcs, diag):
    from terraneo_b200 import shell
    om, pm = Mesh(L), shell.ShellMesh(L)
    u = random_vector(om, seed=20 + L)
    src, dst = shell.VectorQ1Vec(pm), shell.VectorQ1Vec(pm)
    src.set_numpy(u)
    shell.apply(shell.VectorLaplace(pm, bcc, bcs, diag), src, dst)
    torch.cuda.synchronize()
    assert rel(dst.numpy(), om.vector_laplace(u, bcc, bcs, diag)) <= 1e-12


def test_vector_laplace_f32_and_rejects_freeslip():
    from terraneo_b200 import shell, _capi as C
    L = 3
    om, pm = Mesh(L), shell.ShellMesh(L)
    u = random_vector(om, seed=31)
    src, dst = shell.VectorQ1Vec(pm, torch.float32), shell.VectorQ1Vec(pm, torch.float32)
    src.set_numpy(u)
    shell.apply(shell.VectorLaplace(pm, 1, 1), src, dst)
    assert rel(dst.numpy().astype(float), om.vector_laplace(u, 1, 1)) <= 1e-5
    with pytest.raises(RuntimeError):
        shell.apply(shell.VectorLaplace(pm, C.BC_FREESLIP, 1), src, dst)


def test_strong_dirichlet_enforcement_matches_oracle_composition():
    """b - A_N g with diag(A_N) g on the boundary layers (Laplace, inhomogeneous g)."""
    from terraneo_b200 import shell
    L = 3
    om, pm = Mesh(L), shell.ShellMesh(L)
    b = random_vector(om, seed=70, ncomp=1)
    g = random_vector(om, seed=71, ncomp=1)
    vb, vg, tmp = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    vb.set_numpy(b)
    vg.set_numpy(g)
    shell.strong_algebraic_dirichlet_enforcement(shell.Laplace(pm, False), shell.Laplace(pm, False, True), vg, tmp, vb)
    ref = b - om.laplace(g, 0, 0)
    dg = om.laplace(g, 0, 1)
    ref[om.bmask != 1] = dg[om.bmask != 1]
    assert rel(vb.numpy()[0], ref) <= 1e-13
    # homogeneous, surface only
    vb.set_numpy(b)
    shell.assign_boundary(vb, None, 0.0, cmb=False, surface=True)
    ref = b.copy()
    ref[:, :, :, -1] = 0.0
    assert np.array_equal(vb.numpy()[0], ref)
