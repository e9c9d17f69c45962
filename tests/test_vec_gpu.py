"""Krylov vector kernels through the C ABI against numpy / the oracle."""
import numpy as np
import pytest
import torch

from helpers import rel
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def meshes():
    from terraneo_b200 import shell
    return Mesh(3), shell.ShellMesh(3)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("nx", [0, 1, 2, 3])
def test_lincomb(meshes, dtype, nx):
    from terraneo_b200 import shell
    om, pm = meshes
    rng = np.random.default_rng(nx)
    xs = [rng.normal(size=(3,) + om.shape) for _ in range(nx)]
    c = list(rng.normal(size=nx))
    vx = []
    for x in xs:
        v = shell.VectorQ1Vec(pm, dtype)
        v.set_numpy(x)
        vx.append(v)
    y = shell.VectorQ1Vec(pm, dtype)
    shell.lincomb(y, c, vx, 0.25)
    ref = 0.25 + sum(ci * xi for ci, xi in zip(c, xs)) if nx else np.full((3,) + om.shape, 0.25)
    tol = 1e-15 if dtype == torch.float64 else 1e-6
    assert rel(y.numpy(), ref) <= tol


def test_lincomb_rejects_four_inputs(meshes):
    from terraneo_b200 import shell
    om, pm = meshes
    y = shell.VectorQ1Scalar(pm)
    with pytest.raises(RuntimeError):
        shell.lincomb(y, [1, 1, 1, 1], [y, y, y, y])


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_dot_owned_mask(meshes, dtype):
    from terraneo_b200 import shell
    om, pm = meshes
    rng = np.random.default_rng(5)
    a, b = rng.normal(size=(3,) + om.shape), rng.normal(size=(3,) + om.shape)
    va, vb = shell.VectorQ1Vec(pm, dtype), shell.VectorQ1Vec(pm, dtype)
    va.set_numpy(a)
    vb.set_numpy(b)
    if dtype == torch.float32:
        a, b = a.astype(np.float32).astype(np.float64), b.astype(np.float32).astype(np.float64)
    ref = om.dot(a, b)
    assert abs(shell.dot(va, vb) - ref) <= 1e-12 * abs(ref) + 1e-12


def test_elementwise_and_reductions(meshes):
    from terraneo_b200 import shell
    om, pm = meshes
    rng = np.random.default_rng(7)
    a = rng.uniform(0.5, 2.0, size=om.shape)
    b = rng.normal(size=om.shape)
    va, vb = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    va.set_numpy(a)
    vb.set_numpy(b)
    va.invert_entries_impl()
    assert rel(va.numpy()[0], 1 / a) <= 1e-15
    va.scale_with_vector_impl(vb)
    assert rel(va.numpy()[0], b / a) <= 1e-15
    assert va.max_abs_entry_impl() == pytest.approx(np.abs(b / a).max(), rel=1e-15)
    assert not va.has_nan_or_inf_impl()
    va.data[0, 3, 2, 1, 0] = float("nan")
    assert va.has_nan_or_inf_impl()


def test_halo_sum_matches_oracle(meshes):
    from terraneo_b200 import shell
    om, pm = meshes
    f = np.random.default_rng(3).normal(size=(3,) + om.shape)
    v = shell.VectorQ1Vec(pm)
    v.set_numpy(f)
    v.halo_sum()
    assert rel(v.numpy(), om.halo_sum(f)) <= 1e-15


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("beta", [0.0, -0.37])
@pytest.mark.parametrize("layout", ["blocked", "shifted"])
def test_chebyshev_step(meshes, dtype, beta, layout):
    """tn_vec_chebyshev_step: d = alpha D^-1 (b - Ax) + beta d, x += d (chebyshev.hpp:127-160).  'blocked': the
    three components of each field are rows of one tensor (component 1 starts 8 bytes past a 16-byte boundary in
    FP32, so the vector path starts with a scalar head); 'shifted': x starts one entry later in its buffer than
    the other fields, so the offsets modulo 16 bytes differ and the scalar path runs."""
    import ctypes
    from terraneo_b200 import shell, _capi as C
    om, pm = meshes
    ns = pm.stored_nodes
    rng = np.random.default_rng(11)
    ref = {k: rng.normal(size=(3, ns)) for k in ("x", "d", "b", "ax", "inv")}
    dev = {k: torch.as_tensor(v, dtype=dtype, device="cuda").contiguous() for k, v in ref.items()}
    if layout == "shifted":
        buf = torch.zeros(3 * ns + 1, dtype=dtype, device="cuda")
        xs = buf[1:].view(3, ns)
        xs.copy_(dev["x"])
        dev["x"] = xs
    alpha = 0.81
    P = lambda t: C.ptrs(*[t[c].data_ptr() for c in range(3)])
    f = C.lib().tn_vec_chebyshev_step_f64 if dtype == torch.float64 else C.lib().tn_vec_chebyshev_step_f32
    C.check(f(pm.handle, 3, P(dev["x"]), P(dev["d"]), P(dev["b"]), P(dev["ax"]), P(dev["inv"]), alpha, beta,
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "chebyshev_step")
    torch.cuda.synchronize()
    dn = alpha * ref["inv"] * (ref["b"] - ref["ax"]) + beta * ref["d"]
    tol = 1e-14 if dtype == torch.float64 else 2e-6
    assert rel(dev["d"].cpu().numpy(), dn) <= tol
    assert rel(dev["x"].cpu().numpy(), ref["x"] + dn) <= tol


@pytest.mark.parametrize("L", [1, 3])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_masked_sum_over_owned_nodes(L, dtype):
    """tn_vec_sum (masked_sum with the ownership mask, grid_operations.hpp:569) against the oracle's owned mask"""
    from terraneo_b200 import shell
    om, pm = Mesh(L), shell.ShellMesh(L)
    rs = np.random.RandomState(3 + L)
    a = rs.normal(size=(3,) + om.shape)
    v = shell.VectorQ1Vec(pm, dtype)
    v.set_numpy(a)
    want = float((a.astype(np.float32 if dtype == torch.float32 else np.float64).astype(np.float64)
                  * om.omask[None]).sum())
    got = v.masked_sum_impl()
    assert abs(got - want) <= 1e-12 * np.abs(a).sum(), (got, want)
