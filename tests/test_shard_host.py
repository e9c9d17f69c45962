"""The sharded shell's host side on CPU (no GPU needed).

* The rank map (tn_shell_partition) against the reference's own DistributedDomain built as rank q of P
  (tests/golden/shard_L2.npz, made by `ref_dump kerngen_rank`).
* The oracle's copy-wise kerngen apply against the reference's applies of single ranks.
* The halo exchange plan (tn_shard_halo_plan): every rank's copy-wise apply, the shard-local halo sum, pack, a sum
  over the ranks (an all-reduce) and unpack give the whole shell's additive apply, in process for P = 2..10 and over
  two gloo ranks.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

from oracle_lib import Mesh

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as G  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "shard_L2.npz")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _D():
    from terraneo_b200 import distributed
    return distributed


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_partition_matches_the_reference_rank_map():
    D = _D()
    g = np.load(GOLDEN)
    for P in range(1, 11):
        covered = []
        for q in range(P):
            f, n = D.partition(P, q)
            assert np.array_equal(np.arange(f, f + n), g[f"diamonds_P{P}_q{q}"]), (P, q)
            covered += list(range(f, f + n))
        assert covered == list(range(10))


def test_partition_refuses_bad_ranks():
    from terraneo_b200 import _capi as C
    D = _D()
    for P, q in ((11, 0), (0, 0), (2, 2), (3, -1)):
        with pytest.raises(C.TNError):
            D.partition(P, q)


def test_oracle_copywise_apply_matches_the_reference_rank_applies():
    D = _D()
    g = np.load(GOLDEN)
    om = Mesh(G.SHARD_L)
    k, src = G.shard_inputs(om)
    assert np.allclose(G.checksum(k), g["checksum_k"], rtol=1e-13, atol=0)
    assert np.allclose(G.checksum(src), g["checksum_src"], rtol=1e-13, atol=0)
    for bcc, bcs in G.SHARD_BCS:
        cw = om.kerngen(k, src, bcc, bcs, halo=False)
        for P in G.SHARD_APPLY_P:
            for q in range(P):
                f, n = D.partition(P, q)
                assert _rel(cw[:, f:f + n], g[f"dst_{bcc}{bcs}_P{P}_q{q}"]) <= 1e-14, (bcc, bcs, P, q)


def _sum_groups(field, off, mem, n1):
    """field (3, nd, n1, n1, n1): per group the sum of its copies, (3, groups, n1)"""
    f = field.reshape(3, -1, n1)
    return np.stack([np.stack([f[c, mem[off[i]:off[i + 1]]].sum(axis=0) for i in range(len(off) - 1)])
                     if len(off) > 1 else np.zeros((0, n1)) for c in range(3)])


def _assign_groups(field, off, mem, vals, n1):
    f = field.reshape(3, -1, n1)
    for i in range(len(off) - 1):
        for c in range(3):
            f[c, mem[off[i]:off[i + 1]]] = vals[c, i]


def _rank_pack(level, P, q, part):
    """the rank's copy-wise field after the shard-local halo sum, and its exchange buffer"""
    D = _D()
    n1 = (1 << level) + 1
    off, mem = D.halo_plan(level, P, q, cross=False)
    _assign_groups(part, off, mem, _sum_groups(part, off, mem, n1), n1)
    xoff, xmem = D.halo_plan(level, P, q, cross=True)
    return part, _sum_groups(part, xoff, xmem, n1), (xoff, xmem)


@pytest.mark.parametrize("level", [2, 3])
def test_exchange_plan_gives_the_whole_shell_apply(level):
    D = _D()
    om = Mesh(level)
    k, src = G.shard_inputs(om)
    n1 = om.n1
    for bcc, bcs in ((1, 2), (2, 0), (1, 1)):
        full = om.kerngen(k, src, bcc, bcs)
        cw = om.kerngen(k, src, bcc, bcs, halo=False)
        for P in (1, 2, 3, 4, 5, 8, 10):
            parts, bufs, plans = [], [], []
            for q in range(P):
                f, n = D.partition(P, q)
                part, buf, plan = _rank_pack(level, P, q, cw[:, f:f + n].copy())
                parts.append(part), bufs.append(buf), plans.append(plan)
            assert len({b.shape for b in bufs}) == 1  # one buffer layout on every rank
            total = sum(bufs)  # the all-reduce
            for q in range(P):
                f, n = D.partition(P, q)
                _assign_groups(parts[q], *plans[q], total, n1)
                assert _rel(parts[q], full[:, f:f + n]) <= 1e-13, (bcc, bcs, P, q)


def test_plan_covers_every_copy_once():
    """over the ranks, the local groups and the rank's copies of the cross groups hold every copy of the whole
    shell's duplicate groups exactly once; a single rank has no cross group"""
    D = _D()
    level = 3
    n1 = (1 << level) + 1
    off1, mem1 = D.halo_plan(level, 1, 0, cross=False)
    xoff1, _ = D.halo_plan(level, 1, 0, cross=True)
    assert len(xoff1) == 1
    whole = sorted(mem1.tolist())
    for P in (2, 3, 4, 5, 8, 10):
        seen, n_cross = [], set()
        for q in range(P):
            f, _ = D.partition(P, q)
            for cross in (False, True):
                off, mem = D.halo_plan(level, P, q, cross)
                seen += (mem + f * n1 * n1).tolist()
                if cross:
                    n_cross.add(len(off) - 1)
        assert sorted(seen) == whole, P
        assert len(n_cross) == 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import torch
    import torch.distributed as dist
    import make_golden as Gm
    from oracle_lib import Mesh as OM
    from terraneo_b200 import distributed as Dm
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        level = 3
        om = OM(level)
        k, src = Gm.shard_inputs(om)
        full = om.kerngen(k, src, 1, 2)
        cw = om.kerngen(k, src, 1, 2, halo=False)
        f, n = Dm.partition(world, rank)
        part, buf, plan = _rank_pack(level, world, rank, cw[:, f:f + n].copy())
        t = torch.from_numpy(np.ascontiguousarray(buf))
        dist.all_reduce(t)
        _assign_groups(part, *plan, t.numpy(), om.n1)
        q.put((rank, float(_rel(part, full[:, f:f + n]))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_exchange_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] <= 1e-13 for r in res), res
