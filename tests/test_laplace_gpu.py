"""Parity of the CUDA Laplace apply with the oracle."""
import pytest
import torch

from helpers import random_vector, rel
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [2, 3, 4])
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
