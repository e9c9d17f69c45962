"""Stored wedge matrices, GCA coarsening and the stored-matrix apply against the oracle
(which is pinned to the reference's TwoGridGCA and slow path)."""
import numpy as np
import pytest
import torch

from helpers import random_vector, rel, viscosity_field
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu

BCS = [(0, 0), (1, 1), (2, 2), (1, 2), (2, 1)]


_IU = np.triu_indices(18)


def _colmajor(m):
    """oracle layout [cells][2][18][18] -> the library's layout: packed upper triangles (171 per
    wedge plus one zero, wedge w = 2 cell + wedge) with 32 consecutive wedges interleaved in chunks
    of 4 entries"""
    p = m[..., _IU[0], _IU[1]].reshape(-1, 171)
    p = np.concatenate([p, np.zeros((p.shape[0], 1))], axis=1)
    nw = p.shape[0]
    pad = (-nw) % 32
    p = np.concatenate([p, np.zeros((pad, 172))])
    return np.ascontiguousarray(p.reshape(-1, 32, 43, 4).transpose(0, 2, 1, 3)).reshape(-1)


@pytest.fixture(scope="module")
def level3():
    from terraneo_b200 import shell
    L = 3
    of, oc = Mesh(L), Mesh(L - 1)
    pf, pc = shell.ShellMesh(L), shell.ShellMesh(L - 1)
    k = viscosity_field(of, seed=9, contrast=1e3)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k)
    return of, oc, pf, pc, k, kv


def test_local_matrices_match_oracle(level3):
    from terraneo_b200 import shell
    of, oc, pf, pc, k, kv = level3
    m = shell.kerngen_local_matrices(pf, kv).cpu().numpy().reshape(-1)
    assert rel(m, _colmajor(of.local_matrices(k))) <= 1e-13


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("diag", [False, True])
def test_stored_apply_with_kerngen_matrices_equals_kerngen_apply(level3, bc, diag):
    from terraneo_b200 import shell
    of, oc, pf, pc, k, kv = level3
    m = shell.kerngen_local_matrices(pf, kv)
    u = random_vector(of, seed=3)
    src, d1, d2 = shell.VectorQ1Vec(pf), shell.VectorQ1Vec(pf), shell.VectorQ1Vec(pf)
    src.set_numpy(u)
    shell.apply(shell.StoredEpsilonDivDiv(pf, m, bc[0], bc[1], diag), src, d1)
    shell.apply(shell.EpsilonDivDivKerngen(pf, kv, bc[0], bc[1], diagonal=diag), src, d2)
    assert rel(d1.numpy(), d2.numpy()) <= 1e-12
    assert rel(d1.numpy(), of.kerngen(k, u, bc[0], bc[1], diag)) <= 1e-12


@pytest.mark.parametrize("mode", [0, 1])
def test_gca_coarsening_matches_oracle(level3, mode):
    from terraneo_b200 import shell
    of, oc, pf, pc, k, kv = level3
    mk = shell.gca_coarsen(pf, pc, k_fine=kv, mode=mode).cpu().numpy().reshape(-1)
    ref = _colmajor(of.gca_coarsen(oc, k=k, mode=mode))
    assert rel(mk, ref) <= 1e-13
    # from stored fine matrices gives the same
    mf = shell.kerngen_local_matrices(pf, kv)
    ms = shell.gca_coarsen(pf, pc, mats_fine=mf.reshape(-1), mode=mode).cpu().numpy().reshape(-1)
    assert rel(ms, mk) <= 1e-14


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("diag", [False, True])
def test_gca_operator_apply_matches_oracle(level3, bc, diag):
    from terraneo_b200 import shell
    of, oc, pf, pc, k, kv = level3
    mats = shell.gca_coarsen(pf, pc, k_fine=kv)
    ref_m = of.gca_coarsen(oc, k=k)
    u = random_vector(oc, seed=4)
    src, dst = shell.VectorQ1Vec(pc), shell.VectorQ1Vec(pc)
    src.set_numpy(u)
    shell.apply(shell.StoredEpsilonDivDiv(pc, mats, bc[0], bc[1], diag), src, dst)
    assert rel(dst.numpy(), oc.stored_apply(ref_m, u, bc[0], bc[1], diag)) <= 1e-12


def test_gca_two_levels_and_fp32(level3):
    """Level 4 -> 3 -> 2 (second step from stored matrices) and the FP32 apply."""
    from terraneo_b200 import shell, _capi as C
    L = 4
    o4, o3, o2 = Mesh(L), Mesh(L - 1), Mesh(L - 2)
    p4, p3, p2 = shell.ShellMesh(L), shell.ShellMesh(L - 1), shell.ShellMesh(L - 2)
    k = viscosity_field(o4, seed=2, contrast=1e2)
    kv = shell.VectorQ1Scalar(p4)
    kv.set_numpy(k)
    m3 = shell.gca_coarsen(p4, p3, k_fine=kv)
    m2 = shell.gca_coarsen(p3, p2, mats_fine=m3.reshape(-1))
    ref2 = o3.gca_coarsen(o2, mats_fine=o4.gca_coarsen(o3, k=k))
    assert rel(m2.cpu().numpy().reshape(-1), _colmajor(ref2)) <= 1e-13
    m2f = torch.empty(m2.numel(), dtype=torch.float32, device="cuda")
    C.check(C.lib().tn_array_cast_f64_to_f32(m2.numel(), m2.data_ptr(), m2f.data_ptr(), None), "cast")
    u = random_vector(o2, seed=5)
    src, dst = shell.VectorQ1Vec(p2, torch.float32), shell.VectorQ1Vec(p2, torch.float32)
    src.set_numpy(u)
    shell.apply(shell.StoredEpsilonDivDiv(p2, m2f, 2, 2), src, dst)
    assert rel(dst.numpy().astype(float), o2.stored_apply(ref2, u, 2, 2)) <= 1e-5


def _oracle_pcg(apply, dot, b, maxit, rtol):
    """pcg.hpp:78-102 with z = r, from x = 0; returns (x, relative residual history)"""
    x = np.zeros_like(b)
    r = b - apply(x)
    p = r.copy()
    an = dot(r, r)
    r0 = np.sqrt(an)
    hist = [1.0]
    for it in range(1, maxit + 1):
        ap = apply(p)
        alpha = an / dot(ap, p)
        x += alpha * p
        r -= alpha * ap
        rr = dot(r, r)
        hist.append(np.sqrt(rr) / r0)
        if hist[-1] <= rtol:
            break
        p = r + (rr / an) * p
        an = rr
    return x, hist


def _check_stored_pcg(of, pf, bc, contrast, check_every, n):
    from terraneo_b200 import shell
    k = viscosity_field(of, seed=9, contrast=contrast) if contrast > 1 else np.ones(of.shape)
    kv = shell.VectorQ1Scalar(pf)
    kv.set_numpy(k)
    m = shell.kerngen_local_matrices(pf, kv)
    f = random_vector(of, seed=17)
    if bc[0] == 1:
        f[:, :, :, :, 0] = 0.0
    if bc[1] == 1:
        f[:, :, :, :, -1] = 0.0
    fb = shell.VectorQ1Vec(pf)
    fb.set_numpy(f)
    if 2 in bc:
        shell.freeslip_project(fb, bc[0] == 2, bc[1] == 2)
    b = fb.numpy()
    op = shell.StoredEpsilonDivDiv(pf, m, bc[0], bc[1])
    x = shell.VectorQ1Vec(pf)
    its, hist = shell.stored_pcg(op, fb, x, max_iterations=n, relative_tolerance=1e-30, check_every=check_every)
    assert its == n
    xo, ho = _oracle_pcg(lambda v: of.kerngen(k, v, bc[0], bc[1]), of.dot, b, n, 1e-30)
    np.testing.assert_allclose(hist, ho, rtol=1e-6)
    assert rel(x.numpy(), xo) <= 1e-7
    # the stopping rule (gated launches after convergence), and an initial guess (continue from x)
    x2 = shell.VectorQ1Vec(pf)
    tol = ho[n // 2] * (1 + 1e-6)
    its2, _ = shell.stored_pcg(op, fb, x2, max_iterations=n, relative_tolerance=tol, check_every=check_every)
    assert abs(its2 - next(i for i in range(1, n + 1) if ho[i] <= tol)) <= 1
    its3, hist3 = shell.stored_pcg(op, fb, x2, max_iterations=n - its2, relative_tolerance=1e-30,
                                   check_every=check_every)
    assert its3 == n - its2 and hist3[0] == 1.0


@pytest.mark.parametrize("bc", [(1, 1), (2, 2), (2, 1)])
@pytest.mark.parametrize("contrast", [1.0, 1e3])
@pytest.mark.parametrize("check_every", [8, 0])
def test_fused_stored_pcg_matches_oracle_cg(level3, bc, contrast, check_every):
    """The stored-matrix PCG follows the oracle CG on the oracle operator step by step.  At level 3 the vector
    steps of each iteration run as one thread-block-cluster launch.  Unpreconditioned CG amplifies rounding (the
    atomics order on the GPU), so with the 1e3 viscosity contrast only the first iterations are compared tightly."""
    of, oc, pf, pc, _, _ = level3
    _check_stored_pcg(of, pf, bc, contrast, check_every, 60 if contrast == 1.0 else 15)


@pytest.mark.parametrize("bc", [(1, 1), (2, 2)])
@pytest.mark.parametrize("check_every", [8, 0])
def test_fused_stored_pcg_multi_launch_matches_oracle_cg(bc, check_every):
    """Level 4: the multi-launch form (4 gated launches per iteration, device-side stopping flag)."""
    from terraneo_b200 import shell
    _check_stored_pcg(Mesh(4), shell.ShellMesh(4), bc, 1.0, check_every, 30)
