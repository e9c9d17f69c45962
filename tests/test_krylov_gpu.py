"""Device-resident Krylov steps (tn_krylov_axpy_dot_*, tn_pcg_*) through the C ABI.

axpy_dot is checked against numpy on segmented vectors (velocity on a fine
mesh plus pressure on the next coarser one, as in the Stokes block vector);
the PCG steps are driven by hand over the Laplace operator and checked against
the oracle's CG, including that steps issued after convergence change nothing.
"""
import ctypes

import numpy as np
import pytest
import torch

from helpers import random_vector, rel
from oracle_lib import Mesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def meshes():
    from terraneo_b200 import shell
    return Mesh(3), Mesh(2), shell.ShellMesh(3), shell.ShellMesh(2)


def _seg(vs):
    """(nseg, mesh handles, field pointers) of a list of shell vectors."""
    from terraneo_b200 import _capi as C
    ms, fs = [], []
    for v in vs:
        for c in range(v.ncomp):
            ms.append(v.mesh.handle)
            fs.append(v.data[c].data_ptr())
    return len(fs), C.ptrs(*ms), C.ptrs(*fs)


def _block(shell, pf, pc, uf, pcv, dtype):
    u, p = shell.VectorQ1Vec(pf, dtype), shell.VectorQ1Scalar(pc, dtype)
    u.set_numpy(uf)
    p.set_numpy(pcv)
    return u, p


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("mode", ["update_project", "update_norm", "project_only"])
def test_axpy_dot_block_vector(meshes, dtype, mode):
    from terraneo_b200 import _capi as C, shell
    of, oc, pf, pc = meshes
    rng = np.random.default_rng({"update_project": 1, "update_norm": 2, "project_only": 3}[mode])
    w_u, w_p = rng.normal(size=(3,) + of.shape), rng.normal(size=oc.shape)
    x_u, x_p = rng.normal(size=(3,) + of.shape), rng.normal(size=oc.shape)
    v_u, v_p = rng.normal(size=(3,) + of.shape), rng.normal(size=oc.shape)
    if dtype == torch.float32:
        w_u, w_p, x_u, x_p, v_u, v_p = (a.astype(np.float32).astype(np.float64)
                                        for a in (w_u, w_p, x_u, x_p, v_u, v_p))
    W = _block(shell, pf, pc, w_u, w_p, dtype)
    X = _block(shell, pf, pc, x_u, x_p, dtype)
    V = _block(shell, pf, pc, v_u, v_p, dtype)
    coeff = torch.tensor([0.37], dtype=torch.float64, device="cuda")
    result = torch.full((1,), -7.0, dtype=torch.float64, device="cuda")
    n, ms, wf = _seg(W)
    _, _, xf = _seg(X)
    _, _, vf = _seg(V)
    upd = mode != "project_only"
    proj = mode != "update_norm"
    f = getattr(C.lib(), "tn_krylov_axpy_dot_" + ("f64" if dtype == torch.float64 else "f32"))
    C.check(f(n, ms, wf, xf if upd else None, coeff.data_ptr() if upd else None, vf if proj else None, None,
              result.data_ptr(), None), "axpy_dot")
    torch.cuda.synchronize()
    eu = w_u - 0.37 * x_u if upd else w_u
    ep = w_p - 0.37 * x_p if upd else w_p
    tol = 1e-15 if dtype == torch.float64 else 1e-6
    assert rel(W[0].numpy(), eu) <= tol
    assert rel(W[1].numpy()[0], ep) <= tol
    if dtype == torch.float32:
        eu, ep = W[0].numpy().astype(np.float64), W[1].numpy()[0].astype(np.float64)
    ref = of.dot(eu, v_u if proj else eu) + oc.dot(ep, v_p if proj else ep)
    assert abs(result.item() - ref) <= 1e-12 * max(1.0, abs(ref))


def test_axpy_dot_gate_leaves_everything(meshes):
    from terraneo_b200 import _capi as C, shell
    of, oc, pf, pc = meshes
    rng = np.random.default_rng(1)
    w = shell.VectorQ1Vec(pf)
    w.set_numpy(rng.normal(size=(3,) + of.shape))
    x = shell.VectorQ1Vec(pf)
    x.set_numpy(rng.normal(size=(3,) + of.shape))
    before = w.numpy().copy()
    coeff = torch.tensor([2.0], dtype=torch.float64, device="cuda")
    gate = torch.tensor([1.0], dtype=torch.float64, device="cuda")
    result = torch.full((1,), -7.0, dtype=torch.float64, device="cuda")
    n, ms, wf = _seg([w])
    _, _, xf = _seg([x])
    C.check(C.lib().tn_krylov_axpy_dot_f64(n, ms, wf, xf, coeff.data_ptr(), None, gate.data_ptr(), result.data_ptr(),
                                          None), "axpy_dot")
    torch.cuda.synchronize()
    assert np.array_equal(w.numpy(), before)
    assert result.item() == -7.0


def test_axpy_dot_rejects_bad_segments(meshes):
    from terraneo_b200 import _capi as C, shell
    of, oc, pf, pc = meshes
    w = shell.VectorQ1Vec(pf)
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    n, ms, wf = _seg([w])
    assert C.lib().tn_krylov_axpy_dot_f64(0, ms, wf, None, None, None, None, res.data_ptr(), None) != 0
    assert C.lib().tn_krylov_axpy_dot_f64(5, ms, wf, None, None, None, None, res.data_ptr(), None) != 0
    assert C.lib().tn_krylov_axpy_dot_f64(n, ms, wf, None, None, None, None, None, None) != 0


def _oracle_cg(om, b, rtol, maxit):
    x = np.zeros_like(b)
    r = b - om.laplace(x)
    p = r.copy()
    r0 = np.sqrt(om.dot(r, r))
    hist = [1.0]
    for it in range(1, maxit + 1):
        an = om.dot(r, r)
        ap = om.laplace(p)
        alpha = an / om.dot(ap, p)
        x += alpha * p
        r -= alpha * ap
        rr = np.sqrt(om.dot(r, r)) / r0
        hist.append(rr)
        if rr <= rtol:
            return x, it, hist
        p = r + (om.dot(r, r) / an) * p
    return x, maxit, hist


@pytest.mark.parametrize("extra", [0, 7])
def test_pcg_steps_match_oracle_and_stop(meshes, extra):
    """All steps issued without reading the flag: the iterate equals the
    host-stopped CG's, and steps after convergence leave it unchanged."""
    from terraneo_b200 import _capi as C, shell
    om, _, pm, _ = meshes
    b = random_vector(om, seed=4, ncomp=1)
    b[om.bmask != 1] = 0.0
    rtol = 1e-8
    xo, ito, histo = _oracle_cg(om, b, rtol, 500)
    A = shell.Laplace(pm, True)
    vb, x, r, p, ap = (shell.VectorQ1Scalar(pm) for _ in range(5))
    vb.set_numpy(b)
    shell.apply(A, x, r)
    shell.lincomb(r, [1.0, -1.0], [vb, r])
    maxit = ito + 1 + extra
    state = torch.zeros(8 + maxit + 1, dtype=torch.float64, device="cuda")
    n, ms, xf = _seg([x])
    _, _, rf = _seg([r])
    _, _, pf_ = _seg([p])
    _, _, af = _seg([ap])
    L = C.lib()
    C.check(L.tn_pcg_begin_f64(n, ms, rf, pf_, state.data_ptr(), 1e-30, None), "begin")
    for it in range(1, maxit + 1):
        shell.apply(A, p, ap)
        C.check(L.tn_pcg_pap_f64(n, ms, af, pf_, state.data_ptr(), None), "pap")
        C.check(L.tn_pcg_update_f64(n, ms, xf, rf, pf_, af, state.data_ptr(), it, rtol, 1e-30, None), "update")
        C.check(L.tn_pcg_direction_f64(n, ms, pf_, rf, state.data_ptr(), None), "direction")
    st = state.cpu().numpy()
    assert st[4] == 1.0
    its = int(st[5])
    assert abs(its - ito) <= 1
    assert st[6] <= rtol
    assert rel(x.numpy()[0], xo) <= 1e-8
    h = st[8:8 + its + 1]
    k = min(its, ito) + 1
    assert np.allclose(h[:k], histo[:k], rtol=1e-6, atol=1e-14)


def test_pcg_begin_zero_rhs_is_done(meshes):
    from terraneo_b200 import _capi as C, shell
    om, _, pm, _ = meshes
    r, p = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    state = torch.full((12,), 5.0, dtype=torch.float64, device="cuda")
    n, ms, rf = _seg([r])
    _, _, pf_ = _seg([p])
    C.check(C.lib().tn_pcg_begin_f64(n, ms, rf, pf_, state.data_ptr(), 1e-30, None), "begin")
    st = state.cpu().numpy()
    assert st[4] == 1.0 and st[5] == 0.0 and st[8] == 1.0
