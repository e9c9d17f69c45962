"""tn_vec_dot_noalloc_f64 (static device scratch, no mesh handle) against tn_vec_dot_f64.

Named to be collected last, so it also runs after every other test has used
the library on the same device.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_ENTRIES = 16384 * 256 * 8


def _noalloc_dot(n, a, b, owned):
    from terraneo_b200 import _capi as C
    r = ctypes.c_double()
    rc = C.lib().tn_vec_dot_noalloc_f64(n, a.ncomp, a.comp_ptrs(), b.comp_ptrs(),
                                        owned.data_ptr() if owned is not None else None, ctypes.byref(r), None)
    C.check(rc, "dot_noalloc")
    return r.value


@pytest.mark.parametrize("level", [3, 6])
def test_noalloc_dot_matches_mesh_dot_two_calls_in_a_row(level):
    from terraneo_b200 import shell
    pm = shell.ShellMesh(level)
    _, omask = pm.masks()
    owned = torch.as_tensor(np.ascontiguousarray(omask).reshape(-1), device="cuda")
    rng = np.random.default_rng(level)
    for call in range(2):
        a, b = shell.VectorQ1Vec(pm), shell.VectorQ1Vec(pm)
        a.set_numpy(rng.normal(size=(3,) + pm.shape))
        b.set_numpy(rng.normal(size=(3,) + pm.shape) + call)
        ref = shell.dot(a, b)
        got = _noalloc_dot(pm.stored_nodes, a, b, owned)
        assert abs(got - ref) <= 1e-13 * max(1.0, abs(ref)), (call, got, ref)


def test_noalloc_dot_without_mask_is_plain_sum():
    from terraneo_b200 import shell
    pm = shell.ShellMesh(2)
    a, b = shell.VectorQ1Scalar(pm), shell.VectorQ1Scalar(pm)
    a.data.fill_(2.0)
    b.data.fill_(0.5)
    assert _noalloc_dot(pm.stored_nodes, a, b, None) == float(pm.stored_nodes)


def test_noalloc_dot_rejects_sizes_beyond_the_static_scratch():
    from terraneo_b200 import _capi as C, shell
    pm = shell.ShellMesh(2)
    a = shell.VectorQ1Vec(pm)
    r = ctypes.c_double(-1.0)
    L = C.lib()
    assert L.tn_vec_dot_noalloc_f64(MAX_ENTRIES + 1, 3, a.comp_ptrs(), a.comp_ptrs(), None, ctypes.byref(r), None) != 0
    assert L.tn_vec_dot_noalloc_f64(pm.stored_nodes, 4, a.comp_ptrs(), a.comp_ptrs(), None, ctypes.byref(r), None) != 0
    assert L.tn_vec_dot_noalloc_f64(pm.stored_nodes, 3, a.comp_ptrs(), a.comp_ptrs(), None, None, None) != 0
    assert r.value == -1.0
