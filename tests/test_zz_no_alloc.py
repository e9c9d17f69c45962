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


_FIRST_CALL = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from oracle_lib import Mesh
from terraneo_b200 import _capi as C
torch.cuda.set_device(0)
out = []
for level in (3, 6):
    m = Mesh(level)
    rng = np.random.default_rng(level)
    a = rng.normal(size=(3, m.ns))
    b = rng.normal(size=(3, m.ns))
    own = np.ascontiguousarray(m.omask.reshape(-1)).astype(np.uint8)
    ta, tb = torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda")
    to = torch.as_tensor(own, device="cuda")
    pa = (ctypes.c_void_p * 3)(*[ta[c].data_ptr() for c in range(3)])
    pb = (ctypes.c_void_p * 3)(*[tb[c].data_ptr() for c in range(3)])
    r = ctypes.c_double()
    rc = C.lib().tn_vec_dot_noalloc_f64(m.ns, 3, pa, pb, to.data_ptr(), ctypes.byref(r), None)
    assert rc == 0, C.lib().tn_last_error()
    ref = float(np.sum(a * b * own[None, :]))
    assert abs(r.value - ref) <= 1e-12 * max(1.0, np.sum(np.abs(a * b))), (level, r.value, ref)
    out.append(r.value)
print("first-call ok", out)
"""


def test_noalloc_dot_as_first_library_call_of_a_fresh_process():
    """The case the entry point exists for: a process whose first library call is tn_vec_dot_noalloc_f64 (its
    set-up looks the static array up and, under lazy module loading, loads the module), at levels 3 and 6,
    against the numpy dot of the same fields."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", _FIRST_CALL, root], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "first-call ok" in out.stdout
