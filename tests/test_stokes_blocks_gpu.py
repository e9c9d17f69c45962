"""Parity of the CUDA Divergence / Gradient (Stokes B, B^T) with the oracle."""
import numpy as np
import pytest
import torch

from helpers import random_vector, rel
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[2, 3, 4])
def meshes(request):
    from terraneo_b200 import shell
    L = request.param
    return L, Mesh(L), Mesh(L - 1), shell.ShellMesh(L), shell.ShellMesh(L - 1)


@pytest.mark.parametrize("bc", [(1, 1), (2, 2), (2, 1), (0, 0)])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_divergence_and_gradient(meshes, bc, dtype, tol):
    from terraneo_b200 import shell
    L, of, oc, pf, pc = meshes
    u = random_vector(of, seed=L)
    p = random_vector(oc, seed=L + 1, ncomp=1)
    vu, vp = shell.VectorQ1Vec(pf, dtype), shell.VectorQ1Scalar(pc, dtype)
    vu.set_numpy(u)
    out_p = shell.VectorQ1Scalar(pc, dtype)
    shell.apply(shell.Divergence(pf, pc, *bc), vu, out_p)
    vp.set_numpy(p)
    out_u = shell.VectorQ1Vec(pf, dtype)
    shell.apply(shell.Gradient(pf, pc, *bc), vp, out_u)
    torch.cuda.synchronize()
    assert rel(out_p.numpy()[0], of.divergence(oc, u, *bc)) <= tol
    assert rel(out_u.numpy(), of.gradient(oc, p, *bc)) <= tol


def test_gradient_is_divergence_transpose(meshes):
    """<B u, p> == <u, B^T p> on owned nodes (FP64)."""
    from terraneo_b200 import shell
    L, of, oc, pf, pc = meshes
    u = random_vector(of, seed=3)
    p = random_vector(oc, seed=4, ncomp=1)
    vu, vp = shell.VectorQ1Vec(pf), shell.VectorQ1Scalar(pc)
    vu.set_numpy(u)
    vp.set_numpy(p)
    bu, btp = shell.VectorQ1Scalar(pc), shell.VectorQ1Vec(pf)
    shell.apply(shell.Divergence(pf, pc, 2, 1), vu, bu)
    shell.apply(shell.Gradient(pf, pc, 2, 1), vp, btp)
    a, b = shell.dot(bu, vp), shell.dot(vu, btp)
    assert abs(a - b) <= 1e-12 * (abs(a) + abs(b))
