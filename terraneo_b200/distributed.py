"""The shell sharded over the ranks of a torch.distributed process group: one process per GPU, each holding the
diamonds the reference's rank map gives it (DistributedDomain::create_uniform with subdomain refinement level 0 and
subdomain_to_rank_iterate_diamond_subdomains, grid/shell/spherical_shell.hpp:717-745,2566-2590).

The operator kernels run on the shard's diamonds unchanged; the additive halo of an apply
(communication/shell/communication.hpp:242-747) is the shard-local halo kernel plus, for the nodes with copies on
two or more ranks, tn_shard_pack -> an all-reduce (SUM) of the exchange buffer over the process group (NCCL over
NVLink / NVSwitch on GPUs) -> tn_shard_unpack.  Dot products are the owned-node parts of every rank, all-reduced.

Vectors are CUDA tensors of shape (ncomp, diamonds, N+1, N+1, N+1), the component-major layout of the library.
"""
import ctypes

import numpy as np
import torch
import torch.distributed as dist

from . import _capi as C


def partition(num_ranks, rank):
    """(first diamond, number of diamonds) of `rank` among `num_ranks` (host only)."""
    f, n = ctypes.c_int(), ctypes.c_int()
    C.check(C.lib().tn_shell_partition(num_ranks, rank, ctypes.byref(f), ctypes.byref(n)), "tn_shell_partition")
    return f.value, n.value


def halo_plan(level, num_ranks, rank, cross):
    """The rank's local (cross False) or cross-rank (cross True) duplicate groups as CSR arrays over local lateral
    indices (host only): (offsets int32[groups + 1], members int32[copies])."""
    L = C.lib()
    g, m = ctypes.c_int(), ctypes.c_int()
    C.check(L.tn_shard_halo_plan(level, num_ranks, rank, int(cross), ctypes.byref(g), ctypes.byref(m), None, None),
            "tn_shard_halo_plan")
    off = np.zeros(g.value + 1, np.int32)
    mem = np.zeros(max(m.value, 1), np.int32)
    C.check(L.tn_shard_halo_plan(level, num_ranks, rank, int(cross), ctypes.byref(g), ctypes.byref(m),
                                 off.ctypes.data_as(ctypes.c_void_p), mem.ctypes.data_as(ctypes.c_void_p)),
            "tn_shard_halo_plan")
    return off, mem[:m.value]


def _comp_ptrs(t):
    return C.ptrs(*[t[c].data_ptr() for c in range(t.shape[0])])


def _f64(what, *ts):
    """the FP64-only shard calls: refuse other dtypes and non-contiguous or host tensors before any kernel sees
    their pointers"""
    for t in ts:
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
            raise TypeError(f"{what}: needs contiguous float64 CUDA tensors, got {t.dtype} on {t.device}")


def _fields(what, shard, dtype, *ts):
    """every tensor a field of `shard`, shaped (1 to 3 components, diamonds, N+1, N+1, N+1), contiguous, on the GPU,
    of dtype: checked before a kernel gets the component pointers, so no launch reads or writes past a tensor"""
    for t in ts:
        if (t.dtype != dtype or not t.is_cuda or not t.is_contiguous() or t.dim() != 5
                or tuple(t.shape[1:]) != shard.shape or not 1 <= t.shape[0] <= 3):
            raise TypeError(f"{what}: needs contiguous {dtype} CUDA fields of shape (ncomp,) + {shard.shape}, got "
                            f"{tuple(t.shape)} {t.dtype} on {t.device}")


def _scalar(what, shard, dtype, k):
    """a coefficient field passed by its data pointer: the shard's stored nodes, contiguous, on the GPU"""
    if k.dtype != dtype or not k.is_cuda or not k.is_contiguous() or k.numel() != shard.stored_nodes:
        raise TypeError(f"{what}: the coefficient field needs {shard.stored_nodes} contiguous {dtype} CUDA values, "
                        f"got {tuple(k.shape)} {k.dtype} on {k.device}")


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class ShellShard:
    """One rank's diamonds of the level-`level` shell on the current CUDA device (tn_shard)."""

    def __init__(self, level, num_ranks, rank, r_min=0.55, r_max=1.0):
        L = C.lib()
        self.level, self.num_ranks, self.rank = level, num_ranks, rank
        self.N, self.n1 = 1 << level, (1 << level) + 1
        self.r_min, self.r_max = r_min, r_max
        h = ctypes.c_void_p()
        C.check(L.tn_shard_create(level, r_min, r_max, num_ranks, rank, ctypes.byref(h)), "tn_shard_create")
        self.handle = h
        f, n = ctypes.c_int(), ctypes.c_int()
        st, ow, ex = c_size(), c_size(), c_size()
        C.check(L.tn_shard_dims(h, ctypes.byref(f), ctypes.byref(n), ctypes.byref(st), ctypes.byref(ow),
                                ctypes.byref(ex)), "tn_shard_dims")
        self.first_diamond, self.num_diamonds = f.value, n.value
        self.stored_nodes, self.owned_nodes, self.exchange_values = st.value, ow.value, ex.value
        self.shape = (self.num_diamonds, self.n1, self.n1, self.n1)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and C is not None and C._lib is not None:
            C.lib().tn_shard_destroy(h)
            self.handle = None

    def geometry(self):
        coords = np.zeros((self.num_diamonds, self.n1, self.n1, 3))
        radii = np.zeros((self.num_diamonds, self.n1))
        C.check(C.lib().tn_shard_geometry(self.handle, coords.ctypes.data_as(ctypes.c_void_p),
                                          radii.ctypes.data_as(ctypes.c_void_p)), "tn_shard_geometry")
        return coords, radii

    def masks(self):
        b = np.zeros(self.shape, np.uint8)
        o = np.zeros(self.shape, np.uint8)
        C.check(C.lib().tn_shard_masks(self.handle, b.ctypes.data_as(ctypes.c_void_p),
                                       o.ctypes.data_as(ctypes.c_void_p)), "tn_shard_masks")
        return b, o

    def vector(self, ncomp=3, dtype=torch.float64):
        return torch.zeros((ncomp,) + self.shape, dtype=dtype, device="cuda")

    def exchange_buffer(self, ncomp, dtype=torch.float64):
        return torch.zeros(ncomp * self.exchange_values, dtype=dtype, device="cuda")

    def epsdivdiv_apply(self, k, src, dst, bc_cmb, bc_surface, diagonal=False, apply_mode=C.APPLY_REPLACE,
                        comm_mode=C.COMM_ADDITIVE, penalty_eps=1.0):
        """The kerngen apply on this rank's cells; with COMM_ADDITIVE the copies on this rank are summed (the
        cross-rank copies by pack / all-reduce / unpack)."""
        f64 = src.dtype == torch.float64
        _fields("epsdivdiv_apply", self, src.dtype, src, dst)
        _scalar("epsdivdiv_apply", self, src.dtype, k)
        if src.shape[0] != 3 or dst.shape[0] != 3:
            raise TypeError("epsdivdiv_apply: src and dst need 3 components")
        p = C.EpsDivDivParams(bc_cmb, bc_surface, int(diagonal), apply_mode, comm_mode, penalty_eps)
        fn = C.lib().tn_shard_epsdivdiv_apply_f64 if f64 else C.lib().tn_shard_epsdivdiv_apply_f32
        C.check(fn(self.handle, ctypes.byref(p), ctypes.c_void_p(k.data_ptr()), _comp_ptrs(src), _comp_ptrs(dst),
                   _stream()), "tn_shard_epsdivdiv_apply")

    def penalty_dots(self, src, dots):
        """this rank's part of the three rigid-rotation dots of src into the device tensor dots (3 doubles)"""
        _fields("penalty_dots", self, src.dtype, src)
        _f64("penalty_dots", dots)
        if src.shape[0] != 3 or dots.numel() < 3:
            raise TypeError("penalty_dots: src needs 3 components, dots 3 doubles")
        fn = C.lib().tn_shard_penalty_dots_f64 if src.dtype == torch.float64 else C.lib().tn_shard_penalty_dots_f32
        C.check(fn(self.handle, _comp_ptrs(src), ctypes.c_void_p(dots.data_ptr()), _stream()), "tn_shard_penalty_dots")

    def epsdivdiv_apply_fsfs(self, k, src, dst, dots, apply_mode=C.APPLY_REPLACE, comm_mode=C.COMM_ADDITIVE,
                             penalty_eps=1.0):
        """the free-slip (both radii) apply with the whole shell's rotation dots given (device tensor, 3 doubles)"""
        _fields("epsdivdiv_apply_fsfs", self, src.dtype, src, dst)
        _scalar("epsdivdiv_apply_fsfs", self, src.dtype, k)
        _f64("epsdivdiv_apply_fsfs", dots)
        if src.shape[0] != 3 or dst.shape[0] != 3 or dots.numel() < 3:
            raise TypeError("epsdivdiv_apply_fsfs: src and dst need 3 components, dots 3 doubles")
        p = C.EpsDivDivParams(C.BC_FREESLIP, C.BC_FREESLIP, 0, apply_mode, comm_mode, penalty_eps)
        fn = C.lib().tn_shard_epsdivdiv_apply_fsfs_f64 if src.dtype == torch.float64 else \
            C.lib().tn_shard_epsdivdiv_apply_fsfs_f32
        C.check(fn(self.handle, ctypes.byref(p), ctypes.c_void_p(k.data_ptr()), _comp_ptrs(src), _comp_ptrs(dst),
                   ctypes.c_void_p(dots.data_ptr()), _stream()), "tn_shard_epsdivdiv_apply_fsfs")

    def pack(self, fields, buf):
        _fields("pack", self, fields.dtype, fields)
        if buf.dtype != fields.dtype or not buf.is_cuda or buf.numel() < fields.shape[0] * self.exchange_values:
            raise TypeError("pack: the exchange buffer needs ncomp x exchange_values entries of the fields' dtype")
        fn = C.lib().tn_shard_pack_f64 if fields.dtype == torch.float64 else C.lib().tn_shard_pack_f32
        C.check(fn(self.handle, _comp_ptrs(fields), fields.shape[0], ctypes.c_void_p(buf.data_ptr()), _stream()),
                "tn_shard_pack")

    def unpack(self, buf, fields):
        _fields("unpack", self, fields.dtype, fields)
        if buf.dtype != fields.dtype or not buf.is_cuda or buf.numel() < fields.shape[0] * self.exchange_values:
            raise TypeError("unpack: the exchange buffer needs ncomp x exchange_values entries of the fields' dtype")
        fn = C.lib().tn_shard_unpack_f64 if fields.dtype == torch.float64 else C.lib().tn_shard_unpack_f32
        C.check(fn(self.handle, ctypes.c_void_p(buf.data_ptr()), _comp_ptrs(fields), fields.shape[0], _stream()),
                "tn_shard_unpack")

    def local_dot(self, a, b):
        _fields("local_dot", self, torch.float64, a, b)
        if a.shape[0] != b.shape[0]:
            raise TypeError("local_dot: the fields need the same number of components")
        r = ctypes.c_double()
        C.check(C.lib().tn_shard_vec_dot_f64(self.handle, a.shape[0], _comp_ptrs(a), _comp_ptrs(b), ctypes.byref(r),
                                             _stream()), "tn_shard_vec_dot_f64")
        return r.value

    def lincomb(self, y, c0, coeffs, xs):
        """y = c0 + sum_i coeffs[i] xs[i] (up to three inputs, FP64)."""
        _fields("lincomb", self, torch.float64, y, *xs)
        if any(x.shape[0] != y.shape[0] for x in xs) or len(xs) > 3:
            raise TypeError("lincomb: up to three inputs with the output's number of components")
        c = (ctypes.c_double * 3)(*list(coeffs) + [0.0] * (3 - len(coeffs)))
        x = (ctypes.c_void_p * 9)()  # three pointer slots per input vector
        for i, v in enumerate(xs):
            for cpt in range(v.shape[0]):
                x[3 * i + cpt] = v[cpt].data_ptr()
        C.check(C.lib().tn_shard_vec_lincomb_f64(self.handle, y.shape[0], _comp_ptrs(y), c0, len(xs), c, x,
                                                 _stream()), "tn_shard_vec_lincomb_f64")

    # multigrid pieces: this shard and the same rank's shard one level coarser
    def prolong_add(self, coarse, src_c, dst_f):
        """dst_f += P src_c (constant prolongation)"""
        _fields("prolong_add", coarse, torch.float64, src_c)
        _fields("prolong_add", self, torch.float64, dst_f)
        if src_c.shape[0] != dst_f.shape[0]:
            raise TypeError("prolong_add: the fields need the same number of components")
        C.check(C.lib().tn_shard_prolongation_constant_f64(self.handle, coarse.handle, src_c.shape[0], C.APPLY_ADD,
                                                           _comp_ptrs(src_c), _comp_ptrs(dst_f), _stream()),
                "tn_shard_prolongation_constant_f64")

    def restrict(self, coarse, src_f, dst_c):
        """dst_c = R src_f (constant restriction, coarse copies on this rank summed)"""
        _fields("restrict", self, torch.float64, src_f)
        _fields("restrict", coarse, torch.float64, dst_c)
        if src_f.shape[0] != dst_c.shape[0]:
            raise TypeError("restrict: the fields need the same number of components")
        C.check(C.lib().tn_shard_restriction_constant_f64(self.handle, coarse.handle, src_f.shape[0], _comp_ptrs(src_f),
                                                          _comp_ptrs(dst_c), _stream()),
                "tn_shard_restriction_constant_f64")

    def inject(self, coarse, src_f, dst_c):
        """dst_c = src_f at the coarse nodes; a scalar field may come without its component axis"""
        src_f = src_f.unsqueeze(0) if src_f.dim() == 4 else src_f
        dst_c = dst_c.unsqueeze(0) if dst_c.dim() == 4 else dst_c
        _fields("inject", self, torch.float64, src_f)
        _fields("inject", coarse, torch.float64, dst_c)
        if src_f.shape[0] != dst_c.shape[0]:
            raise TypeError("inject: the fields need the same number of components")
        C.check(C.lib().tn_shard_injection_f64(self.handle, coarse.handle, src_f.shape[0], _comp_ptrs(src_f),
                                               _comp_ptrs(dst_c), _stream()), "tn_shard_injection_f64")

    def invert(self, y):
        _fields("invert", self, torch.float64, y)
        C.check(C.lib().tn_shard_vec_invert_f64(self.handle, y.shape[0], _comp_ptrs(y), _stream()),
                "tn_shard_vec_invert_f64")

    def mult(self, y, x):
        """y *= x elementwise"""
        _fields("mult", self, torch.float64, y, x)
        if x.shape[0] != y.shape[0]:
            raise TypeError("mult: the fields need the same number of components")
        C.check(C.lib().tn_shard_vec_mult_f64(self.handle, y.shape[0], _comp_ptrs(y), _comp_ptrs(x), _stream()),
                "tn_shard_vec_mult_f64")

    def chebyshev_step(self, x, d, b, ax, inv_diag, alpha, beta):
        """d = alpha D^-1 (b - ax) + beta d;  x += d"""
        _fields("chebyshev_step", self, torch.float64, x, d, b, ax, inv_diag)
        if len({t.shape[0] for t in (x, d, b, ax, inv_diag)}) != 1:
            raise TypeError("chebyshev_step: the fields need the same number of components")
        C.check(C.lib().tn_shard_vec_chebyshev_step_f64(self.handle, x.shape[0], _comp_ptrs(x), _comp_ptrs(d),
                                                        _comp_ptrs(b), _comp_ptrs(ax), _comp_ptrs(inv_diag), alpha,
                                                        beta, _stream()), "tn_shard_vec_chebyshev_step_f64")

    def random(self, ncomp, seed):
        """a start vector in [-0.5, 0.5) that depends on the node's global index only (every partition draws the
        same values): frac(sin(12.9898 g + 78.233 (seed + c)) 43758.5453) - 0.5"""
        ns = self.stored_nodes
        g = torch.arange(ns, dtype=torch.float64, device="cuda") + float(self.first_diamond * self.n1 ** 3)
        out = torch.empty((ncomp,) + self.shape, dtype=torch.float64, device="cuda")
        for c in range(ncomp):
            v = torch.sin(g * 12.9898 + 78.233 * (seed + c)) * 43758.5453
            out[c] = (v - torch.floor(v) - 0.5).reshape(self.shape)
        return out


def c_size():
    return ctypes.c_size_t()


class DistributedShell:
    """The level-`level` shell over the ranks of a process group (the default group when None): this process's
    shard, the exchange and the global dot.  Without an initialised process group it is the whole shell on one
    rank.  With the NCCL backend the all-reduces run on the GPUs over NVLink; with gloo they stage through the
    host.  Vectors are the shard's tensors; the solvers below (`cg`) take this object as their domain."""

    def __init__(self, level, r_min=0.55, r_max=1.0, group=None):
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.world, self.rank = dist.get_world_size(group), dist.get_rank(group)
            self.backend = dist.get_backend(group)
        else:
            self.world, self.rank, self.backend = 1, 0, None
        self.shard = ShellShard(level, self.world, self.rank, r_min, r_max)
        self._bufs = {}

    def _all_reduce(self, t):
        if self.world == 1:
            return t
        if self.backend == "nccl" or t.device.type == "cpu":
            dist.all_reduce(t, group=self.group)
            return t
        h = t.cpu()  # gloo on CUDA tensors: through the host
        dist.all_reduce(h, group=self.group)
        t.copy_(h)
        return t

    def vector(self, ncomp=3, dtype=torch.float64):
        return self.shard.vector(ncomp, dtype)

    def exchange(self, fields):
        """Sum the copies of the nodes shared with other ranks (the cross-rank part of the additive halo)."""
        key = (fields.shape[0], fields.dtype)
        buf = self._bufs.get(key)
        if buf is None:
            buf = self._bufs[key] = self.shard.exchange_buffer(fields.shape[0], fields.dtype)
        if buf.numel() == 0 and self.world == 1:
            return
        self.shard.pack(fields, buf)
        self._all_reduce(buf)
        self.shard.unpack(buf, fields)

    def epsdivdiv_apply(self, k, src, dst, bc_cmb, bc_surface, diagonal=False, apply_mode=C.APPLY_REPLACE):
        """EpsilonDivDivKerngen apply with the additive halo over all ranks (every copy of a node holds the sum);
        with free-slip on both radii the rotation dots are all-reduced first."""
        if self.world > 1 and not diagonal and bc_cmb == C.BC_FREESLIP and bc_surface == C.BC_FREESLIP:
            dots = torch.zeros(3, dtype=torch.float64, device="cuda")
            self.shard.penalty_dots(src, dots)
            self._all_reduce(dots)
            self.shard.epsdivdiv_apply_fsfs(k, src, dst, dots, apply_mode)
        else:
            self.shard.epsdivdiv_apply(k, src, dst, bc_cmb, bc_surface, diagonal, apply_mode, C.COMM_ADDITIVE)
        self.exchange(dst)

    def dot(self, a, b):
        """Global owned-node dot product (every rank returns the same value)."""
        part = self.shard.local_dot(a, b)
        if self.world == 1:
            return part
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([part], dtype=torch.float64, device=dev)
        self._all_reduce(t)
        return float(t.item())

    def lincomb(self, y, c0, coeffs, xs):
        self.shard.lincomb(y, c0, coeffs, xs)

    def copy(self, dst, src):
        self.shard.lincomb(dst, 0.0, [1.0], [src])

    def restrict_to(self, coarse, src_f, dst_c):
        self.shard.restrict(coarse.shard, src_f, dst_c)
        coarse.exchange(dst_c)

    def prolong_add_from(self, coarse, src_c, dst_f):
        self.shard.prolong_add(coarse.shard, src_c, dst_f)

    def inject_to(self, coarse, src_f, dst_c):
        self.shard.inject(coarse.shard, src_f, dst_c)

    def invert(self, y):
        self.shard.invert(y)

    def mult(self, y, x):
        self.shard.mult(y, x)

    def chebyshev_step(self, x, d, b, ax, inv_diag, alpha, beta):
        self.shard.chebyshev_step(x, d, b, ax, inv_diag, alpha, beta)

    def random(self, ncomp, seed):
        return self.shard.random(ncomp, seed)

    def cg(self, k, b, x, bc_cmb=C.BC_DIRICHLET, bc_surface=C.BC_DIRICHLET, max_iterations=500,
           relative_tolerance=1e-10, absolute_tolerance=0.0):
        return cg(self, k, b, x, bc_cmb, bc_surface, max_iterations, relative_tolerance, absolute_tolerance)


class EmulatedShell:
    """All P ranks of a sharded shell in one process, on the current GPU: the same domain interface as
    `DistributedShell`, with vectors as lists of the ranks' tensors.  Each operation runs rank after rank, the
    exchange sums the ranks' buffers (what the all-reduce does across GPUs) and the dot sums their owned parts,
    so no kernel ever waits on another.  For checking a decomposition (and the solvers over it) on one GPU."""

    def __init__(self, level, num_ranks, r_min=0.55, r_max=1.0):
        self.world = num_ranks
        self.shards = [ShellShard(level, num_ranks, q, r_min, r_max) for q in range(num_ranks)]
        self._bufs = {}

    def vector(self, ncomp=3, dtype=torch.float64):
        return [sh.vector(ncomp, dtype) for sh in self.shards]

    def scatter(self, whole):
        """the ranks' parts of a whole-shell array [ncomp][10][...] (numpy or tensor) as a vector"""
        out = []
        for sh in self.shards:
            f, n = sh.first_diamond, sh.num_diamonds
            part = whole[..., f:f + n, :, :, :]
            out.append(torch.as_tensor(np.ascontiguousarray(part) if isinstance(part, np.ndarray) else part,
                                       device="cuda").contiguous())
        return out

    def gather(self, v):
        """a vector as one whole-shell numpy array"""
        return np.concatenate([t.detach().cpu().numpy() for t in v], axis=-4)

    def exchange(self, fields):
        key = (fields[0].shape[0], fields[0].dtype)
        bufs = self._bufs.get(key)
        if bufs is None:
            bufs = self._bufs[key] = [sh.exchange_buffer(*key) for sh in self.shards]
        if bufs[0].numel() == 0:
            return
        for sh, f, b in zip(self.shards, fields, bufs):
            sh.pack(f, b)
        total = bufs[0].clone()
        for b in bufs[1:]:
            total += b
        for sh, f in zip(self.shards, fields):
            sh.unpack(total, f)

    def epsdivdiv_apply(self, k, src, dst, bc_cmb, bc_surface, diagonal=False, apply_mode=C.APPLY_REPLACE):
        if self.world > 1 and not diagonal and bc_cmb == C.BC_FREESLIP and bc_surface == C.BC_FREESLIP:
            parts = []
            for sh, s in zip(self.shards, src):
                parts.append(torch.zeros(3, dtype=torch.float64, device="cuda"))
                sh.penalty_dots(s, parts[-1])
            dots = torch.stack(parts).sum(dim=0)  # the all-reduce over the ranks
            for sh, kk, s, d in zip(self.shards, k, src, dst):
                sh.epsdivdiv_apply_fsfs(kk, s, d, dots, apply_mode)
        else:
            for sh, kk, s, d in zip(self.shards, k, src, dst):
                sh.epsdivdiv_apply(kk, s, d, bc_cmb, bc_surface, diagonal, apply_mode, C.COMM_ADDITIVE)
        self.exchange(dst)

    def dot(self, a, b):
        return sum(sh.local_dot(x, y) for sh, x, y in zip(self.shards, a, b))

    def lincomb(self, y, c0, coeffs, xs):
        for q, sh in enumerate(self.shards):
            sh.lincomb(y[q], c0, coeffs, [x[q] for x in xs])

    def copy(self, dst, src):
        self.lincomb(dst, 0.0, [1.0], [src])

    def restrict_to(self, coarse, src_f, dst_c):
        for f, c, x, y in zip(self.shards, coarse.shards, src_f, dst_c):
            f.restrict(c, x, y)
        coarse.exchange(dst_c)

    def prolong_add_from(self, coarse, src_c, dst_f):
        for f, c, x, y in zip(self.shards, coarse.shards, src_c, dst_f):
            f.prolong_add(c, x, y)

    def inject_to(self, coarse, src_f, dst_c):
        for f, c, x, y in zip(self.shards, coarse.shards, src_f, dst_c):
            f.inject(c, x, y)

    def invert(self, y):
        for sh, v in zip(self.shards, y):
            sh.invert(v)

    def mult(self, y, x):
        for sh, a, b in zip(self.shards, y, x):
            sh.mult(a, b)

    def chebyshev_step(self, x, d, b, ax, inv_diag, alpha, beta):
        for q, sh in enumerate(self.shards):
            sh.chebyshev_step(x[q], d[q], b[q], ax[q], inv_diag[q], alpha, beta)

    def random(self, ncomp, seed):
        return [sh.random(ncomp, seed) for sh in self.shards]

    def cg(self, k, b, x, bc_cmb=C.BC_DIRICHLET, bc_surface=C.BC_DIRICHLET, max_iterations=500,
           relative_tolerance=1e-10, absolute_tolerance=0.0):
        return cg(self, k, b, x, bc_cmb, bc_surface, max_iterations, relative_tolerance, absolute_tolerance)


def cg(D, k, b, x, bc_cmb=C.BC_DIRICHLET, bc_surface=C.BC_DIRICHLET, max_iterations=500, relative_tolerance=1e-10,
       absolute_tolerance=0.0):
    """Unpreconditioned CG on the kerngen operator over a sharded domain D (`DistributedShell` or `EmulatedShell`):
    the reference's PCG (linalg/solvers/pcg.hpp:78-160) with the identity preconditioner.  b and x are consistent
    vectors (every copy of a node equal), k the shard-local viscosity.  Returns (iterations, relative residual)."""
    r, p, ap = D.vector(3), D.vector(3), D.vector(3)
    D.epsdivdiv_apply(k, x, ap, bc_cmb, bc_surface)
    D.lincomb(r, 0.0, [1.0, -1.0], [b, ap])
    rr = D.dot(r, r)
    r0 = rr ** 0.5
    if r0 <= absolute_tolerance or r0 == 0.0:
        return 0, 0.0
    D.copy(p, r)
    res = r0
    for it in range(1, max_iterations + 1):
        D.epsdivdiv_apply(k, p, ap, bc_cmb, bc_surface)
        alpha = rr / D.dot(p, ap)
        D.lincomb(x, 0.0, [1.0, alpha], [x, p])
        D.lincomb(r, 0.0, [1.0, -alpha], [r, ap])
        rr_new = D.dot(r, r)
        res = rr_new ** 0.5
        if res / r0 <= relative_tolerance or res <= absolute_tolerance:
            return it, res / r0
        D.lincomb(p, 0.0, [1.0, rr_new / rr], [r, p])
        rr = rr_new
    return max_iterations, res / r0


class ShardedMultigrid:
    """Geometric multigrid V-cycle for the kerngen (epsilon-div-div) operator over a hierarchy of sharded domains
    `levels` (finest first, one level apart, the same partition): the operator re-discretised on every level with
    the viscosity injected from the finest, the Chebyshev smoother (linalg/solvers/chebyshev.hpp:50-175: order,
    `smoothing_steps` sweeps before and after, lambda_max = 1.5 x the power-iteration estimate of D^-1 A,
    lambda_min = 0.1 x it), constant vector transfers and CG on the coarsest level, as the reference's Multigrid
    (linalg/solvers/multigrid.hpp:184-211) composes them.  Every operation is sharded: applies and restrictions
    finish with the exchange, dots are global."""

    def __init__(self, levels, k_fine, bc_cmb, bc_surface, order=3, smoothing_steps=2, power_iterations=10,
                 coarse_max_iterations=50, coarse_relative_tolerance=1e-6, seed=7):
        self.D, self.bc = levels, (bc_cmb, bc_surface)
        self.order, self.steps = order, smoothing_steps
        self.coarse_maxit, self.coarse_rtol = coarse_max_iterations, coarse_relative_tolerance
        self.k = [k_fine]
        for lf, lc in zip(levels[:-1], levels[1:]):
            kc = lc.vector(1)
            lf.inject_to(lc, self.k[-1], kc)
            self.k.append(kc)
        # per level: residual, correction, smoother direction, operator result
        self.tmp = [tuple(D.vector(3) for _ in range(4)) for D in levels]
        self.inv_diag, self.ev = [], []
        for lev, (D, k) in enumerate(zip(levels[:-1], self.k[:-1])):
            dg = D.vector(3)
            D.lincomb(self.tmp[lev][0], 1.0, [], [])
            D.epsdivdiv_apply(k, self.tmp[lev][0], dg, bc_cmb, bc_surface, diagonal=True)
            D.invert(dg)
            self.inv_diag.append(dg)
            self.ev.append(self._power_iteration(lev, power_iterations, seed + lev))

    def _power_iteration(self, lev, iterations, seed):
        """power_iteration (linalg/solvers/power_iteration.hpp:13-48) on D^-1 A, from a start vector that depends
        on the global node index only"""
        D, k, dinv = self.D[lev], self.k[lev], self.inv_diag[lev]
        it, aux = D.random(3, seed), self.tmp[lev][3]

        def op(src, dst):
            D.epsdivdiv_apply(k, src, dst, *self.bc)
            D.mult(dst, dinv)
        n = D.dot(it, it) ** 0.5
        D.lincomb(it, 0.0, [1.0 / n], [it])
        op(it, aux)
        radius = 0.0
        for _ in range(iterations):
            n = D.dot(aux, aux) ** 0.5
            D.lincomb(it, 0.0, [1.0 / n], [aux])
            op(it, aux)
            radius = D.dot(it, aux)
        return radius

    def _smooth(self, lev, x, b):
        D, k, dinv, ev = self.D[lev], self.k[lev], self.inv_diag[lev], self.ev[lev]
        d, z = self.tmp[lev][2], self.tmp[lev][3]
        lmax, lmin = 1.5 * ev, 0.1 * ev
        theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
        sigma = theta / delta
        rho = 1.0 / sigma  # carried across sweeps as in the reference (chebyshev.hpp:119)
        for _ in range(self.steps):
            D.epsdivdiv_apply(k, x, z, *self.bc)
            D.chebyshev_step(x, d, b, z, dinv, 1.0 / theta, 0.0)
            for _ in range(2, self.order + 1):
                rho_new = 1.0 / (2.0 * sigma - rho)
                D.epsdivdiv_apply(k, x, z, *self.bc)
                D.chebyshev_step(x, d, b, z, dinv, 2.0 * rho_new / delta, rho_new * rho)
                rho = rho_new

    def _recurse(self, lev, x, b):
        D, k = self.D[lev], self.k[lev]
        if lev == len(self.D) - 1:
            cg(D, k, b, x, *self.bc, max_iterations=self.coarse_maxit, relative_tolerance=self.coarse_rtol)
            return
        self._smooth(lev, x, b)
        r = self.tmp[lev][0]
        D.epsdivdiv_apply(k, x, r, *self.bc)
        D.lincomb(r, 0.0, [1.0, -1.0], [b, r])
        rc, ec = self.tmp[lev + 1][0], self.tmp[lev + 1][1]
        D.restrict_to(self.D[lev + 1], r, rc)
        self.D[lev + 1].lincomb(ec, 0.0, [], [])
        self._recurse(lev + 1, ec, rc)
        D.prolong_add_from(self.D[lev + 1], ec, x)
        self._smooth(lev, x, b)

    def solve(self, x, b):
        """one V-cycle on A x = b from the given x"""
        self._recurse(0, x, b)


def mg_pcg(D, mg, k, b, x, bc_cmb, bc_surface, max_iterations=200, relative_tolerance=1e-8,
           absolute_tolerance=0.0):
    """The reference's PCG (linalg/solvers/pcg.hpp:78-160) over a sharded domain with the V-cycle `mg`
    (ShardedMultigrid, z = V(r) from z = 0) as the preconditioner.  Returns (iterations, relative residual)."""
    r, z, p, ap = D.vector(3), D.vector(3), D.vector(3), D.vector(3)
    D.epsdivdiv_apply(k, x, r, bc_cmb, bc_surface)
    D.lincomb(r, 0.0, [1.0, -1.0], [b, r])
    D.lincomb(z, 0.0, [], [])
    mg.solve(z, r)
    D.copy(p, z)
    r0 = D.dot(r, r) ** 0.5
    if r0 <= absolute_tolerance or r0 == 0.0:
        return 0, 0.0
    res = r0
    for it in range(1, max_iterations + 1):
        an = D.dot(z, r)
        D.epsdivdiv_apply(k, p, ap, bc_cmb, bc_surface)
        alpha = an / D.dot(ap, p)
        D.lincomb(x, 0.0, [1.0, alpha], [x, p])
        D.lincomb(r, 0.0, [1.0, -alpha], [r, ap])
        res = D.dot(r, r) ** 0.5
        if res / r0 <= relative_tolerance or res < absolute_tolerance:
            return it, res / r0
        D.lincomb(z, 0.0, [], [])
        mg.solve(z, r)
        beta = D.dot(z, r) / an
        D.lincomb(p, 0.0, [1.0, beta], [z, p])
    return max_iterations, res / r0
