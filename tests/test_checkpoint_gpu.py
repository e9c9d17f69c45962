"""XDMF output and checkpoint reading on the GPU (tn_xdmf_output_*, tn_read_xdmf_checkpoint_grid) against the
checkpoint the reference's io::XDMFOutput wrote (tests/golden/xdmf_L2, byte for byte) and the oracle's
restatement of the format (pinned to it by tests/test_oracle_pinning.py); the FE -> FV transfer of the
checkpoint recovery against the oracle and the reference's fixture; a checkpoint round trip of the
mantle-circulation step."""
import os
import sys

import numpy as np
import pytest
import torch

from helpers import rel, viscosity_field
from oracle_lib import (Mesh, xdmf_geometry, xdmf_grid_bytes, xdmf_metadata, xdmf_read_grid, xdmf_step_xml,
                        xdmf_topology, xdmf_write_dir)

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_L2.npz")


def _vec(shell, mesh, data, dtype):
    t = torch.as_tensor(np.asarray(data), device="cuda").to(dtype)
    if t.dim() == 4:
        return shell.VectorQ1Scalar(mesh, dtype, data=t[None].contiguous())
    return shell.VectorQ1Vec(mesh, dtype, data=t.contiguous())


def _fixture_writer(shell, directory, pts, conn, level=G.L):
    """the fixture's six grids as device vectors added to a writer; returns (writer, {label: vector})"""
    om, oc = Mesh(level), Mesh(level - 1)
    pm = shell.ShellMesh(level)
    w = shell.XDMFOutput(directory, pm, pts, conn)
    vecs = {}
    for lab, ib, ob, v, data in G.xdmf_fields(om, oc, 0):
        vecs[lab] = _vec(shell, pm, data, torch.float32 if ib == 4 else torch.float64)
        w.add(vecs[lab], lab, ob)
    return w, vecs, om, oc


def _set_step(vecs, om, oc, step):
    for lab, ib, ob, v, data in G.xdmf_fields(om, oc, step):
        t = torch.as_tensor(np.asarray(data), device="cuda").to(vecs[lab].dtype)
        vecs[lab].data.copy_(t if t.dim() == 5 else t[None])


def test_writer_reproduces_the_reference_checkpoint(tmp_path):
    """the fixture's two writes through the GPU writer: every file equal to the reference's, byte for byte"""
    from terraneo_b200 import shell
    d = tmp_path / "out"
    w, vecs, om, oc = _fixture_writer(shell, d, G.XDMF_PTS, G.XDMF_CONN)
    w.write()
    _set_step(vecs, om, oc, 1)   # changed right after write() returned: the files hold step 0
    w.write()
    w.wait()
    names = sorted(os.listdir(G.XDMF_DIR))
    assert sorted(os.listdir(d)) == names
    for n in names:
        with open(os.path.join(G.XDMF_DIR, n), "rb") as a, open(d / n, "rb") as b:
            assert a.read() == b.read(), n


def test_writer_fp64_points_int32_connectivity_level3(tmp_path):
    """points FP64, connectivity int32, level 3, a set write counter: against the restatement"""
    from terraneo_b200 import shell
    d = tmp_path / "out"
    w, vecs, om, oc = _fixture_writer(shell, d, 8, 4, level=3)
    w.set_write_counter(7)
    w.write()
    w.wait()
    grids = [dict(label=lab, in_bytes=ib, out_bytes=ob, vec=v, data=a) for lab, ib, ob, v, a in G.xdmf_fields(om, oc, 0)]
    geo = np.fromfile(d / "geometry.bin")
    assert np.array_equal(geo, np.frombuffer(xdmf_geometry(om, 8), dtype=np.float64))
    assert (d / "topology.bin").read_bytes() == xdmf_topology(om, 4)
    assert (d / "checkpoint_metadata.bin").read_bytes() == xdmf_metadata(om, grids, 8)
    for g in grids:
        assert (d / f'{g["label"]}_7.bin').read_bytes() == xdmf_grid_bytes(g["data"], g["vec"], g["out_bytes"])
    assert (d / "step_7.xmf").read_text() == xdmf_step_xml(om, grids, 7, 8, 4)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_reader_on_the_reference_checkpoint(dtype):
    """every grid of both steps of the reference's checkpoint read into FP64 and FP32 device vectors"""
    from terraneo_b200 import shell
    om = Mesh(G.L)
    pm = shell.ShellMesh(G.L)
    for step in (0, 1):
        for lab, ib, ob, v, _ in G.xdmf_fields(om, Mesh(G.L - 1), step):
            x = shell.VectorQ1Scalar(pm, dtype) if v == 1 else shell.VectorQ1Vec(pm, dtype)
            shell.read_xdmf_checkpoint_grid(G.XDMF_DIR, lab, step, x)
            want = xdmf_read_grid(G.XDMF_DIR, lab, step, om, v == 3)
            got = x.data.double().cpu().numpy()
            got = got[0] if v == 1 else got
            assert np.array_equal(got, want.astype(np.float32).astype(np.float64) if dtype == torch.float32
                                  else want), (lab, step)


def test_reader_follows_the_subdomain_ids(tmp_path):
    """a checkpoint with the diamonds' chunks in a shuffled order (as a multi-process writer may leave it)"""
    from terraneo_b200 import shell
    L = 3
    om = Mesh(L)
    rs = np.random.RandomState(5)
    T, u = rs.normal(size=om.shape), rs.normal(size=(3,) + om.shape)
    grids = [dict(label="T", in_bytes=8, out_bytes=8, vec=1, data=T),
             dict(label="u_u", in_bytes=8, out_bytes=4, vec=3, data=u)]
    xdmf_write_dir(tmp_path, om, [grids], order=[9, 2, 4, 0, 7, 1, 8, 3, 5, 6])
    pm = shell.ShellMesh(L)
    x, y = shell.VectorQ1Scalar(pm), shell.VectorQ1Vec(pm)
    shell.read_xdmf_checkpoint_grid(tmp_path, "T", 0, x)
    shell.read_xdmf_checkpoint_grid(tmp_path, "u_u", 0, y)
    assert np.array_equal(x.numpy()[0], T)
    assert np.array_equal(y.numpy(), u.astype(np.float32).astype(np.float64))


def test_reader_errors_are_the_references(tmp_path):
    from terraneo_b200 import _capi as C, shell
    pm, p3 = shell.ShellMesh(G.L), shell.ShellMesh(3)
    s, v = shell.VectorQ1Scalar(pm), shell.VectorQ1Vec(pm)
    cases = [
        (lambda: shell.read_xdmf_checkpoint_grid(tmp_path, "T", 0, s),
         "Could not read checkpoint metadata: Could not find file: "),
        (lambda: shell.read_xdmf_checkpoint_grid(G.XDMF_DIR, "nope", 0, s),
         "Could not find requested data (nope) in checkpoint"),
        (lambda: shell.read_xdmf_checkpoint_grid(G.XDMF_DIR, "T", 5, s),
         "Could not find checkpoint data file for requested label and step."),
        (lambda: shell.read_xdmf_checkpoint_grid(G.XDMF_DIR, "T", 0, shell.VectorQ1Scalar(p3)),
         "Grid data extents do not match metadata."),
        (lambda: shell.read_xdmf_checkpoint_grid(G.XDMF_DIR, "u", 0, s),
         "Checkpoint is scalar, passed grid data view dims do not match."),
        (lambda: shell.read_xdmf_checkpoint_grid(G.XDMF_DIR, "T", 0, v),
         "Checkpoint is vector-valued, passed grid data view dims do not match."),
    ]
    for call, text in cases:
        with pytest.raises(C.TNError) as e:
            call()
        assert text in str(e.value), str(e.value)


def test_writer_argument_errors(tmp_path):
    from terraneo_b200 import _capi as C, shell
    pm = shell.ShellMesh(2)
    w = shell.XDMFOutput(tmp_path / "w", pm)
    a = shell.VectorQ1Scalar(pm)
    w.add(a, "a")
    with pytest.raises(C.TNError, match="identical label"):
        w.add(shell.VectorQ1Scalar(pm), "a")
    w.write()
    with pytest.raises(C.TNError, match="Cannot add data after write"):
        w.add(shell.VectorQ1Scalar(pm), "b")
    w.wait()


def test_round_trip_level6(tmp_path):
    """level 6 (2.7 M stored nodes): FP64 output reads back bit-exact, FP32 output as the FP32 cast"""
    from terraneo_b200 import shell
    pm = shell.ShellMesh(6)
    u = shell.VectorQ1Vec(pm)
    u.data.normal_(generator=torch.Generator(device="cuda").manual_seed(2))
    w = shell.XDMFOutput(tmp_path, pm)
    w.add(u, "u64", 8)
    w.add(shell.VectorQ1Vec(pm, data=u.data), "u32", 4)
    w.write()
    w.wait()
    x = shell.VectorQ1Vec(pm)
    shell.read_xdmf_checkpoint_grid(tmp_path, "u64", 0, x)
    assert torch.equal(x.data, u.data)
    shell.read_xdmf_checkpoint_grid(tmp_path, "u32", 0, x)
    assert torch.equal(x.data, u.data.float().double())


def test_fe_to_fv_matches_oracle_and_reference():
    from terraneo_b200 import shell
    om = Mesh(G.L)
    _, T = G.timestep_inputs(om)
    pm = shell.ShellMesh(G.L)
    fe = shell.VectorQ1Scalar(pm)
    fe.set_numpy(T)
    fv = torch.zeros(om.fv_shape, dtype=torch.float64, device="cuda")
    shell.l2_project_fe_to_fv(pm, fe, fv)
    ref = np.load(GOLDEN)["fe2fv"]
    assert np.abs(fv.cpu().numpy() - ref).max() <= 1e-15 * np.abs(ref).max()
    om3, p3 = Mesh(3), shell.ShellMesh(3)
    T3 = om3.make_consistent(np.random.RandomState(8).uniform(size=om3.shape)).reshape(om3.shape)
    fe3 = shell.VectorQ1Scalar(p3)
    fe3.set_numpy(T3)
    fv3 = torch.full(om3.fv_shape, 7.0, dtype=torch.float64, device="cuda")
    shell.l2_project_fe_to_fv(p3, fe3, fv3)
    want = om3.l2_project_fe_to_fv(T3, np.full(om3.fv_shape, 7.0))
    assert np.abs(fv3.cpu().numpy() - want).max() <= 1e-15 * np.abs(want).max()


def test_mantle_timestep_checkpoint_restart(tmp_path):
    """The app's checkpoint cycle at level 3: write T, u_u and eta after a step, restore them into a fresh
    time step (the FV temperature from the FE one), and the restored state equals the written one (FP64
    output)."""
    from terraneo_b200 import shell
    L = 3
    om = Mesh(L)
    c = om.fv_cell_centers()
    rr = np.sqrt((c ** 2).sum(0)).clip(1e-30)
    T0 = ((1 / rr - 1.0) / (1 / 0.55 - 1.0)).clip(0, 1)
    k = viscosity_field(om, seed=9, contrast=1e2)
    pm = shell.ShellMesh(L)
    kv = shell.VectorQ1Scalar(pm)
    kv.set_numpy(k)
    kw = dict(mg_levels=2, mg_fp32=False, relative_tolerance=1e-8, max_iterations=200, restart=50, gca=1)
    ts = shell.MantleTimestep(L, kv, torch.as_tensor(T0, device="cuda"), rayleigh=1e4, **kw)
    out = ts.checkpoint_output(tmp_path, output=8)
    out.write()
    assert ts.step()
    out.write()
    out.wait()
    ts2 = shell.MantleTimestep(L, kv, torch.zeros(om.fv_shape, dtype=torch.float64, device="cuda"), rayleigh=1e4, **kw)
    ts2.restore_checkpoint(tmp_path, 1)
    assert torch.equal(ts2.u.data, ts.u.data) and torch.equal(ts2.T.data, ts.T.data)
    want = om.l2_project_fe_to_fv(ts.T.numpy()[0], ts2.T_fv.cpu().numpy())
    assert rel(ts2.T_fv.cpu().numpy(), want) <= 1e-15
    assert ts2.step() and ts2.last["finite"]
