"""The checkpoint metadata reader of the C ABI (tn_read_xdmf_checkpoint_metadata, host code only) on the
checkpoint the reference's io::XDMFOutput wrote (tests/golden/xdmf_L2) and on damaged copies of it, against
read_xdmf_checkpoint_metadata's fields and error texts (io/xdmf.hpp:1162-1268).  No GPU needed."""
import os
import shutil
import struct
import sys

import numpy as np
import pytest

from oracle_lib import Mesh

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as G  # noqa: E402


def test_metadata_of_the_reference_checkpoint():
    from terraneo_b200 import shell
    md = shell.read_xdmf_checkpoint_metadata(G.XDMF_DIR)
    n1 = (1 << G.L) + 1
    assert (md["version"], md["subdomains_lateral"], md["subdomains_radial"]) == (1, 1, 1)
    assert (md["size_x"], md["size_y"], md["size_r"]) == (n1, n1, n1)
    assert md["grid_scalar_bytes"] == G.XDMF_PTS and md["ordering"] == 0
    assert np.array_equal(md["radii"], Mesh(G.L).radii[0])
    assert md["subdomain_ids"] == [d << 57 for d in range(10)]
    # the reference's write order: FP32 scalars, FP64 scalars, FP32 vectors, FP64 vectors
    want = [("s32", 4, 1), ("T", 4, 1), ("T64", 8, 1), ("v32", 8, 3), ("u", 4, 3), ("u64", 8, 3)]
    got = [(f["label"], f["scalar_bytes"], f["vec_dim"]) for f in md["grid_data_files"]]
    assert got == want
    assert all(f["scalar_data_type"] == 2 for f in md["grid_data_files"])


def _copy(tmp_path):
    d = tmp_path / "ck"
    shutil.copytree(G.XDMF_DIR, d)
    return d


def _expect_error(d, text):
    from terraneo_b200 import _capi as C, shell
    with pytest.raises(C.TNError) as e:
        shell.read_xdmf_checkpoint_metadata(d)
    assert text in str(e.value), str(e.value)


def test_metadata_errors(tmp_path):
    missing = tmp_path / "none"
    _expect_error(missing, f"Could not find file: {missing}/checkpoint_metadata.bin")
    d = _copy(tmp_path)
    p = d / "checkpoint_metadata.bin"
    raw = p.read_bytes()
    p.write_bytes(raw[:30])
    _expect_error(d, "Failed to read from input stream.")
    # radii out of order
    n1 = (1 << G.L) + 1
    bad = bytearray(raw)
    bad[24 + 8:24 + 16] = struct.pack("<d", 0.1)
    p.write_bytes(bytes(bad))
    _expect_error(d, "Radii are not sorted correctly in checkpoint.")
    # the id list cut short
    p.write_bytes(raw[:-12])
    _expect_error(d, "Failed to read from input stream. (global_subdomain_id reading error)")
    assert n1 == 5
