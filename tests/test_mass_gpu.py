"""Parity of the CUDA KMass / Mass apply with the oracle."""
import numpy as np
import pytest
import torch

from helpers import random_vector, rel
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [1, 2, 3])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_kmass(L, mode):
    from terraneo_b200 import shell
    om, pm = Mesh(L), shell.ShellMesh(L)
    k = om.make_consistent(np.exp(np.random.default_rng(L).normal(size=om.shape)))
    u = random_vector(om, seed=L + 3, ncomp=1)
    kv, src, dst = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    kv.set_numpy(k)
    src.set_numpy(u)
    shell.apply(shell.KMass(pm, kv, mode), src, dst)
    torch.cuda.synchronize()
    assert rel(dst.numpy()[0], om.kmass(k, u, mode)) <= 1e-13
    dst2 = shell.VectorQ1Scalar(pm)
    shell.apply(shell.KMass(pm, None, mode), src, dst2)
    torch.cuda.synchronize()
    assert rel(dst2.numpy()[0], om.kmass(np.ones(om.shape), u, mode)) <= 1e-13


@pytest.mark.parametrize("diag", [False, True])
def test_vector_mass_matches_reference_golden(diag):
    """VectorMass against the reference's own VectorMass outputs (golden level-2 fixture)."""
    import os
    import sys
    from terraneo_b200 import shell
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden as G
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_L2.npz"))
    fine, coarse = Mesh(G.L), Mesh(G.L - 1)
    u = G.inputs(fine, coarse)["u"]
    pm = shell.ShellMesh(G.L)
    src, dst = shell.VectorQ1Vec(pm), shell.VectorQ1Vec(pm)
    src.set_numpy(u)
    shell.apply(shell.VectorMass(pm, diag), src, dst)
    assert rel(dst.numpy(), g[f"vmass_{int(diag)}"]) <= 1e-13
