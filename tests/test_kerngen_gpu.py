"""Parity of the CUDA epsilon-div-div apply (C ABI) with the oracle."""
import numpy as np
import pytest
import torch

from helpers import random_vector, rel, viscosity_field
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu

BCS = [(1, 1), (2, 2), (2, 1), (1, 2), (0, 0), (0, 1), (0, 2)]


# level 1 (the smallest shell, the cell kernel), levels 2-3 (the cell kernel and 8-column tiles), 4 (16-column
# tiles, half the lanes of the radial chunk idle) and 5 (one full radial chunk, the top level written by its last
# lane)
@pytest.fixture(scope="module", params=[1, 2, 3, 4, 5])
def setup(request):
    from terraneo_b200 import shell
    L = request.param
    om = Mesh(L)
    pm = shell.ShellMesh(L)
    k = viscosity_field(om, seed=L)
    u = random_vector(om, seed=10 + L)
    return L, om, pm, k, u


def test_mesh_matches_oracle(setup):
    L, om, pm, k, u = setup
    coords, radii = pm.geometry()
    assert np.array_equal(coords, om.coords)
    assert np.array_equal(radii, om.radii)
    b, o = pm.masks()
    assert np.array_equal(b, om.bmask)
    assert np.array_equal(o, om.omask)


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("diag", [False, True])
def test_epsdivdiv_f64_matches_oracle(setup, bc, diag):
    from terraneo_b200 import shell
    L, om, pm, k, u = setup
    kv = shell.VectorQ1Scalar(pm)
    kv.set_numpy(k)
    src = shell.VectorQ1Vec(pm)
    src.set_numpy(u)
    dst = shell.VectorQ1Vec(pm)
    dst.data.fill_(123.0)  # Replace mode must overwrite
    op = shell.EpsilonDivDivKerngen(pm, kv, bc[0], bc[1], diagonal=diag)
    shell.apply(op, src, dst)
    torch.cuda.synchronize()
    ref = om.kerngen(k, u, bc[0], bc[1], diag)
    assert rel(dst.numpy(), ref) <= 1e-12


@pytest.mark.parametrize("bc", [(1, 1), (2, 2), (2, 1)])
def test_epsdivdiv_f32_matches_oracle(setup, bc):
    from terraneo_b200 import shell
    L, om, pm, k, u = setup
    kv = shell.VectorQ1Scalar(pm, torch.float32)
    kv.set_numpy(k)
    src = shell.VectorQ1Vec(pm, torch.float32)
    src.set_numpy(u)
    dst = shell.VectorQ1Vec(pm, torch.float32)
    op = shell.EpsilonDivDivKerngen(pm, kv, bc[0], bc[1])
    shell.apply(op, src, dst)
    torch.cuda.synchronize()
    ref = om.kerngen(k, u, bc[0], bc[1], False)
    # FP32 with FP32 accumulation: stated bound 1e-5 relative (k contrast 1e4)
    assert rel(dst.numpy(), ref) <= 1e-5


def test_epsdivdiv_add_mode_and_skip_comm(setup):
    from terraneo_b200 import shell, _capi as C
    L, om, pm, k, u = setup
    kv = shell.VectorQ1Scalar(pm)
    kv.set_numpy(k)
    src = shell.VectorQ1Vec(pm)
    src.set_numpy(u)
    base = random_vector(om, seed=99)
    dst = shell.VectorQ1Vec(pm)
    dst.set_numpy(base)
    op = shell.EpsilonDivDivKerngen(pm, kv, 1, 1, apply_mode=C.APPLY_ADD, comm_mode=C.COMM_SKIP)
    shell.apply(op, src, dst)
    dst.halo_sum()
    torch.cuda.synchronize()
    # (base + A_local u) summed over copies = halo(base) + A u
    ref = om.halo_sum(base) + om.kerngen(k, u, 1, 1, False)
    assert rel(dst.numpy(), ref) <= 1e-12


@pytest.mark.parametrize("L", [2, 3, 4])
@pytest.mark.parametrize("treat,diag", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_epsdivdiv3x2_f64(L, treat, diag):
    """EpsilonDivDiv with the 3x2 rule against the oracle (pinned to the reference)."""
    from terraneo_b200 import shell
    from helpers import random_vector, rel, viscosity_field
    om, pm = Mesh(L), shell.ShellMesh(L)
    k = viscosity_field(om, seed=L, contrast=1e3)
    u = random_vector(om, seed=60 + L)
    kv, src, dst = shell.VectorQ1Scalar(pm), shell.VectorQ1Vec(pm), shell.VectorQ1Vec(pm)
    kv.set_numpy(k)
    src.set_numpy(u)
    shell.apply(shell.EpsilonDivDiv(pm, kv, treat, diag), src, dst)
    assert rel(dst.numpy(), om.epsdivdiv3x2(k, u, treat, diag)) <= 1e-12


def test_epsdivdiv3x2_f32():
    from terraneo_b200 import shell
    from helpers import random_vector, rel, viscosity_field
    L = 3
    om, pm = Mesh(L), shell.ShellMesh(L)
    k = viscosity_field(om, seed=1, contrast=1e3)
    u = random_vector(om, seed=61)
    kv, src, dst = (shell.VectorQ1Scalar(pm, torch.float32), shell.VectorQ1Vec(pm, torch.float32),
                    shell.VectorQ1Vec(pm, torch.float32))
    kv.set_numpy(k)
    src.set_numpy(u)
    shell.apply(shell.EpsilonDivDiv(pm, kv, 1), src, dst)
    assert rel(dst.numpy().astype(float), om.epsdivdiv3x2(k, u, 1, 0)) <= 1e-5
