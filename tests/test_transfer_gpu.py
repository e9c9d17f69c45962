"""Parity of the CUDA constant grid transfers with the oracle."""
import numpy as np
import pytest
import torch

from helpers import random_vector, rel
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [2, 3, 4])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-14), (torch.float32, 1e-6)])
def test_prolongation_restriction(L, dtype, tol):
    from terraneo_b200 import shell
    of, oc = Mesh(L), Mesh(L - 1)
    pf, pc = shell.ShellMesh(L), shell.ShellMesh(L - 1)
    uc = random_vector(oc, seed=L)
    uf = random_vector(of, seed=L + 7)
    vc, vf = shell.VectorQ1Vec(pc, dtype), shell.VectorQ1Vec(pf, dtype)
    vc.set_numpy(uc)
    outf = shell.VectorQ1Vec(pf, dtype)
    shell.apply(shell.ProlongationVecConstant(pf, pc), vc, outf)
    vf.set_numpy(uf)
    outc = shell.VectorQ1Vec(pc, dtype)
    shell.apply(shell.RestrictionVecConstant(pf, pc), vf, outc)
    torch.cuda.synchronize()
    assert rel(outf.numpy(), of.prolong(oc, uc)) <= tol
    assert rel(outc.numpy(), of.restrict(oc, uf)) <= tol


def test_restriction_is_prolongation_transpose():
    """<R u_f, v_c> == <u_f, P v_c> on owned nodes (the reference's test_restriction check)."""
    from terraneo_b200 import shell
    L = 3
    of, oc = Mesh(L), Mesh(L - 1)
    pf, pc = shell.ShellMesh(L), shell.ShellMesh(L - 1)
    uf, vc = random_vector(of, seed=1), random_vector(oc, seed=2)
    a, b = shell.VectorQ1Vec(pf), shell.VectorQ1Vec(pc)
    a.set_numpy(uf)
    b.set_numpy(vc)
    ra, pb = shell.VectorQ1Vec(pc), shell.VectorQ1Vec(pf)
    shell.apply(shell.RestrictionVecConstant(pf, pc), a, ra)
    shell.apply(shell.ProlongationVecConstant(pf, pc), b, pb)
    x, y = shell.dot(ra, b), shell.dot(a, pb)
    assert abs(x - y) <= 1e-13 * (abs(x) + abs(y))


@pytest.mark.parametrize("L", [2, 3, 4])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_linear_transfers_match_oracle(L, dtype):
    from terraneo_b200 import shell
    of, oc = Mesh(L), Mesh(L - 1)
    pf, pc = shell.ShellMesh(L), shell.ShellMesh(L - 1)
    uc = random_vector(oc, seed=40 + L, ncomp=1)
    uf = random_vector(of, seed=50 + L, ncomp=1)
    tol = 1e-13 if dtype == torch.float64 else 1e-6
    vc, vf = shell.VectorQ1Scalar(pc, dtype), shell.VectorQ1Scalar(pf, dtype)
    vc.set_numpy(uc)
    shell.apply(shell.ProlongationLinear(pf, pc), vc, vf)
    assert rel(vf.numpy()[0].astype(float), of.prolong_linear(oc, uc)) <= tol
    vf.set_numpy(uf)
    shell.apply(shell.RestrictionLinear(pf, pc), vf, vc)
    assert rel(vc.numpy()[0].astype(float), of.restrict_linear(oc, uf)) <= tol


def test_linear_transfer_vector_components_and_affine_exactness():
    """Every component uses the scalar weights; affine functions prolongate exactly."""
    from terraneo_b200 import shell
    L = 3
    of, oc = Mesh(L), Mesh(L - 1)
    pf, pc = shell.ShellMesh(L), shell.ShellMesh(L - 1)
    xc = oc.coords[:, :, :, None, :] * oc.radii[:, None, None, :, None]
    xf = of.coords[:, :, :, None, :] * of.radii[:, None, None, :, None]
    aff = lambda x, a: a[0] * x[..., 0] + a[1] * x[..., 1] + a[2] * x[..., 2] + a[3]
    coefs = [(1.0, -2.0, 0.5, 0.3), (0.0, 1.0, 1.0, -1.0), (2.0, 0.0, -1.0, 0.0)]
    vc, vf = shell.VectorQ1Vec(pc), shell.VectorQ1Vec(pf)
    vc.set_numpy(np.stack([aff(xc, a) for a in coefs]))
    shell.apply(shell.ProlongationLinear(pf, pc), vc, vf)
    ref = np.stack([aff(xf, a) for a in coefs])
    assert rel(vf.numpy(), ref) <= 1e-12
    assert rel(vf.numpy()[1], of.prolong_linear(oc, vc.numpy()[1])) <= 1e-13
