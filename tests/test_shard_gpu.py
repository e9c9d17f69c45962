"""The sharded shell on the GPU: tn_shard_* through terraneo_b200.distributed.

Several ranks are emulated in one process on one GPU, one after another, never waiting on one another: every
rank's shard applies the operator and packs its exchange buffer, the buffers are summed (what the all-reduce over
the ranks' GPUs does), every shard unpacks.  The result is compared with the oracle's whole-shell apply (pinned to
the reference), with the whole-shell GPU apply at the benchmark size, and, copy-wise, with the reference's own
applies as rank q of P (tests/golden/shard_L2.npz).  The torch.distributed path is run as a one-rank NCCL group.
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from helpers import rel
from oracle_lib import Mesh

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "shard_L2.npz")


def _dev(a, dtype):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _emulated_apply(level, P, k, src, bcc, bcs, diag=False, dtype=torch.float64):
    from terraneo_b200.distributed import ShellShard
    shards = [ShellShard(level, P, q) for q in range(P)]
    outs, bufs = [], []
    for sh in shards:
        f, n = sh.first_diamond, sh.num_diamonds
        d = sh.vector(3, dtype)
        sh.epsdivdiv_apply(_dev(k[f:f + n], dtype), _dev(src[:, f:f + n], dtype), d, bcc, bcs, diag)
        b = sh.exchange_buffer(3, dtype)
        sh.pack(d, b)
        outs.append(d), bufs.append(b)
    total = torch.stack(bufs).sum(dim=0)  # the all-reduce over the ranks
    for sh, d in zip(shards, outs):
        sh.unpack(total, d)
    torch.cuda.synchronize()
    return shards, [d.double().cpu().numpy() for d in outs]


def _inputs(om):
    k, src = G.shard_inputs(om)
    return k, src


@pytest.mark.parametrize("P", [1, 2, 3, 4, 8, 10])
def test_shard_geometry_masks_and_ownership(P):
    from terraneo_b200.distributed import ShellShard
    om = Mesh(3)
    owned = 0
    for q in range(P):
        sh = ShellShard(3, P, q)
        f, n = sh.first_diamond, sh.num_diamonds
        coords, radii = sh.geometry()
        assert np.array_equal(coords, om.coords[f:f + n]) and np.array_equal(radii, om.radii[f:f + n])
        b, o = sh.masks()
        assert np.array_equal(b, om.bmask[f:f + n]) and np.array_equal(o, om.omask[f:f + n])
        assert sh.owned_nodes == int(o.sum())
        owned += sh.owned_nodes
    assert owned == (10 * om.N ** 2 + 2) * om.n1


@pytest.mark.parametrize("level", [2, 3, 4])
@pytest.mark.parametrize("P", [1, 2, 3, 4, 8, 10])
def test_sharded_apply_matches_oracle(level, P):
    om = Mesh(level)
    k, src = _inputs(om)
    for bcc, bcs, diag in ((1, 1, 0), (1, 2, 0), (2, 0, 0), (0, 0, 0), (2, 1, 0), (1, 1, 1), (2, 2, 1)):
        want = om.kerngen(k, src, bcc, bcs, bool(diag))
        _, outs = _emulated_apply(level, P, k, src, bcc, bcs, bool(diag))
        for q, d in enumerate(outs):
            from terraneo_b200.distributed import partition
            f, n = partition(P, q)
            assert rel(d, want[:, f:f + n]) <= 1e-12, (bcc, bcs, diag, q)


@pytest.mark.parametrize("P", [2, 5])
def test_sharded_apply_fp32(P):
    from terraneo_b200.distributed import partition
    om = Mesh(4)
    k, src = _inputs(om)
    want = om.kerngen(k, src, 1, 2)
    _, outs = _emulated_apply(4, P, k, src, 1, 2, dtype=torch.float32)
    for q, d in enumerate(outs):
        f, n = partition(P, q)
        assert rel(d, want[:, f:f + n]) <= 2e-5, q


def test_copywise_shard_apply_matches_reference_rank_applies():
    from terraneo_b200 import _capi as C
    from terraneo_b200.distributed import ShellShard
    g = np.load(GOLDEN)
    om = Mesh(G.SHARD_L)
    k, src = G.shard_inputs(om)
    for bcc, bcs in G.SHARD_BCS:
        for P in G.SHARD_APPLY_P:
            for q in range(P):
                sh = ShellShard(G.SHARD_L, P, q)
                f, n = sh.first_diamond, sh.num_diamonds
                d = sh.vector(3)
                sh.epsdivdiv_apply(_dev(k[f:f + n], torch.float64), _dev(src[:, f:f + n], torch.float64), d, bcc,
                                   bcs, comm_mode=C.COMM_SKIP)
                assert rel(d.cpu().numpy(), g[f"dst_{bcc}{bcs}_P{P}_q{q}"]) <= 1e-12, (bcc, bcs, P, q)


@pytest.mark.parametrize("P", [2, 8])
def test_sharded_apply_at_level6_matches_whole_shell_gpu_apply(P):
    """the benchmark size: the emulated ranks against the whole-shell apply of the same kernels (only the order in
    which the copies of a shared node are summed differs)"""
    from terraneo_b200 import shell
    from terraneo_b200.distributed import partition
    L = 6
    pm = shell.ShellMesh(L)
    rs = np.random.RandomState(5)
    k = np.exp(rs.uniform(0, np.log(1e4), size=pm.shape))  # a 1e4 viscosity contrast
    src = rs.normal(size=(3,) + pm.shape)
    kv = shell.VectorQ1Scalar(pm)
    kv.set_numpy(k)
    u, v = shell.VectorQ1Vec(pm), shell.VectorQ1Vec(pm)
    u.set_numpy(src)
    for bcc, bcs in ((1, 1), (2, 1)):
        op = shell.EpsilonDivDivKerngen(pm, kv, bcc, bcs)
        shell.apply(op, u, v)
        want = v.numpy()
        _, outs = _emulated_apply(L, P, k, src, bcc, bcs)
        for q, d in enumerate(outs):
            f, n = partition(P, q)
            assert rel(d, want[:, f:f + n]) <= 1e-13, (bcc, bcs, q)


def test_freeslip_both_radii_refused_on_two_ranks():
    from terraneo_b200 import _capi as C
    from terraneo_b200.distributed import ShellShard
    sh = ShellShard(3, 2, 0)
    d = sh.vector(3)
    with pytest.raises(C.TNError):
        sh.epsdivdiv_apply(torch.ones(sh.shape, dtype=torch.float64, device="cuda"), sh.vector(3), d, 2, 2)


def test_distributed_shell_single_rank_dot_and_cg():
    """without a process group the shell is one rank: the dot is the owned-node dot and CG on the Dirichlet
    operator reaches its tolerance with the oracle's true residual"""
    from terraneo_b200.distributed import DistributedShell
    L = 3
    om = Mesh(L)
    k, src = _inputs(om)
    ds = DistributedShell(L)
    assert ds.world == 1 and ds.shard.num_diamonds == 10
    a, b = _dev(src, torch.float64), _dev(src[::-1].copy(), torch.float64)
    assert abs(ds.dot(a, b) - om.dot(src, src[::-1])) <= 1e-12 * abs(om.dot(src, src[::-1]))
    kd = _dev(k, torch.float64)
    x = ds.shard.vector(3)
    its, rr = ds.cg(kd, a, x, max_iterations=400, relative_tolerance=1e-10)
    xs = x.cpu().numpy()
    res = om.kerngen(k, xs, 1, 1) - src
    assert np.sqrt(om.dot(res, res)) <= 1e-9 * np.sqrt(om.dot(src, src)), (its, rr)


_NCCL_ONE_RANK = r"""
import os, socket, sys, datetime
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
sys.path.insert(0, os.path.join(sys.argv[1], "tests", "golden"))
import numpy as np, torch, torch.distributed as dist
with socket.socket() as s:
    s.bind(("127.0.0.1", 0)); port = s.getsockname()[1]
os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
torch.cuda.set_device(0)
dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
try:
    import make_golden as G
    from oracle_lib import Mesh
    from terraneo_b200.distributed import DistributedShell
    om = Mesh(3)
    k, src = G.shard_inputs(om)
    ds = DistributedShell(3)
    assert ds.world == 1 and ds.backend == "nccl"
    kd = torch.tensor(k, device="cuda"); s = torch.tensor(src, device="cuda"); d = ds.shard.vector(3)
    ds.epsdivdiv_apply(kd, s, d, 1, 2)
    want = om.kerngen(k, src, 1, 2)
    err = np.abs(d.cpu().numpy() - want).max() / np.abs(want).max()
    dd = ds.dot(s, s)
    print("RESULT", err, abs(dd - om.dot(src, src)) / om.dot(src, src))
finally:
    dist.destroy_process_group()
"""


def test_distributed_shell_in_a_one_rank_nccl_group():
    out = subprocess.run([sys.executable, "-c", _NCCL_ONE_RANK, ROOT], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("RESULT")][-1].split()
    assert float(line[1]) <= 1e-12 and float(line[2]) <= 1e-12, line


def test_bench_sharded_leg_on_one_rank():
    """bench.py --sharded on one GPU: the leg the bench runs on every rank of a multi-GPU job"""
    import json
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "3", "--warmup", "3", "--no-stokes",
           "--no-cpu-baseline", "--no-laplace-cg", "--no-adjoint", "--no-timestep", "--no-level8", "--sharded"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1])
    sh = line["sharded"]
    assert sh["ranks"] == 1 and sh["diamonds_per_rank"] == [10] and sh["exchange_bytes_per_apply"] == 0
    assert sh["value"] > 1.0 and sh["scaling"] == "strong"


@pytest.mark.parametrize("bc", [(1, 1), (1, 2), (2, 1), (2, 2)])
def test_emulated_ranks_cg_matches_one_rank(bc):
    """CG over P = 2, 3, 5, 8 emulated ranks (distributed.EmulatedShell: the ranks one after another on one GPU,
    the exchange a sum of their buffers) against the one-rank solve: the same iteration count within 2, the
    solutions within the tolerance, and the oracle's true residual"""
    from terraneo_b200.distributed import EmulatedShell
    L = 3
    om = Mesh(L)
    k, _ = _inputs(om)
    rs = np.random.RandomState(40)
    b = np.stack([om.make_consistent(rs.normal(size=om.shape)).reshape(om.shape) for _ in range(3)])
    sols, its = {}, {}
    for P in (1, 2, 3, 5, 8):
        D = EmulatedShell(L, P)
        kk, bb, x = D.scatter(k), D.scatter(b), D.vector(3)
        its[P], rr = D.cg(kk, bb, x, *bc, max_iterations=1000, relative_tolerance=1e-10)
        assert rr <= 1e-10, (P, its[P], rr)
        sols[P] = D.gather(x)
        res = om.kerngen(k, sols[P], *bc) - b
        assert np.sqrt(om.dot(res, res)) <= 2e-10 * np.sqrt(om.dot(b, b)), P
    for P in (2, 3, 5, 8):
        assert abs(its[P] - its[1]) <= 2, its
        assert rel(sols[P], sols[1]) <= 1e-8, P


@pytest.mark.parametrize("bc", [(1, 1), (1, 2), (2, 2)])
def test_emulated_ranks_multigrid_pcg(bc):
    """the sharded multigrid (distributed.ShardedMultigrid: Chebyshev order 3, 2 sweeps, constant transfers, CG on
    the coarsest level; levels 4, 3, 2) as the preconditioner of CG, over P = 1, 2, 3, 5 emulated ranks: the oracle's
    true residual, the one-rank iteration count within 1, the solutions within the tolerance, and far fewer
    iterations than plain CG"""
    from terraneo_b200.distributed import EmulatedShell, ShardedMultigrid, mg_pcg
    L = 4
    om = Mesh(L)
    k, _ = _inputs(om)
    rs = np.random.RandomState(41)
    b = np.stack([om.make_consistent(rs.normal(size=om.shape)).reshape(om.shape) for _ in range(3)])
    its, sols, evs = {}, {}, {}
    for P in (1, 2, 3, 5):
        levels = [EmulatedShell(lv, P) for lv in (L, L - 1, L - 2)]
        kk = levels[0].scatter(k)
        mg = ShardedMultigrid(levels, kk, *bc, order=3, smoothing_steps=2, power_iterations=10,
                              coarse_max_iterations=50, coarse_relative_tolerance=1e-6)
        evs[P] = mg.ev
        x = levels[0].vector(3)
        its[P], rr = mg_pcg(levels[0], mg, kk, levels[0].scatter(b), x, *bc, max_iterations=100,
                            relative_tolerance=1e-8)
        assert rr <= 1e-8, (P, its[P], rr)
        sols[P] = levels[0].gather(x)
        res = om.kerngen(k, sols[P], *bc) - b
        assert np.sqrt(om.dot(res, res)) <= 2e-8 * np.sqrt(om.dot(b, b)), P
    # free-slip on both radii converges more slowly (the smoother's diagonal leaves out the rotation penalty)
    assert its[1] <= (40 if bc != (2, 2) else 90), its
    for P in (2, 3, 5):
        assert np.allclose(evs[P], evs[1], rtol=1e-10), (evs[P], evs[1])
        assert abs(its[P] - its[1]) <= 1, its
        assert rel(sols[P], sols[1]) <= 1e-6, P


@pytest.mark.parametrize("level", [3, 4])
def test_emulated_ranks_freeslip_both_radii(level):
    """free-slip on both radii over 2-10 emulated ranks: every rank's part of the rotation dots
    (tn_shard_penalty_dots), their sum, the apply with the sums (tn_shard_epsdivdiv_apply_fsfs) and the exchange
    give the oracle's whole-shell apply with the rigid-rotation penalty"""
    from terraneo_b200.distributed import EmulatedShell
    om = Mesh(level)
    k, src = _inputs(om)
    want = om.kerngen(k, src, 2, 2)
    for P in (2, 3, 5, 8, 10):
        D = EmulatedShell(level, P)
        for dtype, tol in ((torch.float64, 1e-12), (torch.float32, 2e-5)):
            kk = [t.to(dtype) for t in D.scatter(k)]
            ss = [t.to(dtype) for t in D.scatter(src)]
            dd = D.vector(3, dtype)
            D.epsdivdiv_apply(kk, ss, dd, 2, 2)
            assert rel(D.gather(dd), want) <= tol, (P, dtype)


def test_shard_calls_refuse_mismatched_tensors():
    """wrong dtypes, shapes, component counts and host tensors are refused before a kernel sees their pointers"""
    from terraneo_b200.distributed import ShellShard
    sh = ShellShard(3, 2, 0)
    good = sh.vector(3)
    k = torch.ones(sh.shape, dtype=torch.float64, device="cuda")
    bad = [sh.vector(3, torch.float32), torch.zeros((3, 1) + sh.shape[1:], dtype=torch.float64, device="cuda"),
           good.cpu(), good[:, :1], good.transpose(3, 4)]
    for b in bad:
        with pytest.raises(TypeError):
            sh.local_dot(good, b)
        with pytest.raises(TypeError):
            sh.lincomb(good, 0.0, [1.0], [b])
        with pytest.raises(TypeError):
            sh.epsdivdiv_apply(k, b, good, 1, 1)
    with pytest.raises(TypeError):
        sh.epsdivdiv_apply(k[:1], good, sh.vector(3), 1, 1)
    with pytest.raises(TypeError):
        sh.pack(good, torch.zeros(1, dtype=torch.float64, device="cuda"))
    coarse = ShellShard(2, 2, 0)
    with pytest.raises(TypeError):
        sh.restrict(coarse, good, sh.vector(3))  # the destination lives on the coarse shard
