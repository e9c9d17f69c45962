"""ctypes binding of the C oracle (oracle/liboracle.so) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product never imports it.
"""
import ctypes
import json
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_DUMP = os.path.join(ORACLE_DIR, "_ref", "ref_dump")

_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_uint8)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(ORACLE_DIR, "liboracle.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
        L = ctypes.CDLL(path)
        L.or_unit_sphere_coords.argtypes = [ctypes.c_int, _D]
        L.or_shell_radii.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _D]
        L.or_boundary_mask.argtypes = [ctypes.c_int, _U8]
        L.or_ownership_mask.argtypes = [ctypes.c_int, _D, _U8]
        L.or_halo_sum.argtypes = [ctypes.c_int, _D, _D, ctypes.c_int]
        L.or_kerngen_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_kerngen_apply_copywise.argtypes = L.or_kerngen_apply.argtypes
        L.or_laplace_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int]
        L.or_divergence_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int]
        L.or_gradient_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int]
        L.or_epsdivdiv3x2_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int]
        L.or_divkgrad_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_vector_laplace_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_vector_laplace_apply.restype = ctypes.c_int
        L.or_prolongation_linear.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D]
        L.or_restriction_linear.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _U8, _D, _D]
        L.or_kerngen_local_matrices.argtypes = [ctypes.c_int, _D, _D, _D, _D]
        L.or_gca_coarsen.argtypes = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_int, _D]
        L.or_stored_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_fv_ghost_update.argtypes = [ctypes.c_int, _D, _D]
        L.or_fv_cell_centers.argtypes = [ctypes.c_int, _D, _D, _D]
        L.or_fct_dt_stable.argtypes = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_double]
        L.or_fct_dt_stable.restype = ctypes.c_double
        L.or_fct_dirichlet.argtypes = [ctypes.c_int, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.or_fct_step.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double, _D,
                                  ctypes.c_int, _D, _D]
        L.or_prolongation_constant.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D]
        L.or_restriction_constant.argtypes = [ctypes.c_int, ctypes.c_int, _D, _U8, _D, _D]
        L.or_kmass_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int]
        L.or_fv_to_fe_rhs.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D]
        L.or_fe_to_fv.argtypes = [ctypes.c_int, _D, _D, _D, _D]
        L.or_gca_elements.argtypes = [ctypes.c_int, _D, ctypes.c_int, _U8]
        L.or_supg_apply.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_masked_dot.restype = ctypes.c_double
        L.or_masked_dot.argtypes = [ctypes.c_size_t, _D, _D, _U8]
        _lib = L
    return _lib


def _p(a):
    assert a.flags.c_contiguous
    if a.dtype == np.float64:
        return a.ctypes.data_as(_D)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(_U8)
    raise TypeError(a.dtype)


class Mesh:
    """Oracle mesh of the 10-diamond shell at level L (one subdomain per diamond)."""

    def __init__(self, L, rmin=0.55, rmax=1.0):
        self.L, self.N, self.n1 = L, 1 << L, (1 << L) + 1
        n1 = self.n1
        self.shape = (10, n1, n1, n1)
        self.ns = 10 * n1 ** 3
        self.coords = np.zeros((10, n1, n1, 3))
        lib().or_unit_sphere_coords(L, _p(self.coords))
        self.radii = np.zeros((10, n1))
        lib().or_shell_radii(L, rmin, rmax, _p(self.radii))
        self.bmask = np.zeros(self.shape, np.uint8)
        lib().or_boundary_mask(L, _p(self.bmask))
        self.omask = np.zeros(self.shape, np.uint8)
        lib().or_ownership_mask(L, _p(self.coords), _p(self.omask))

    def halo_sum(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        ncomp = f.size // self.ns
        lib().or_halo_sum(self.L, _p(self.coords), _p(f), ncomp)
        return f

    def make_consistent(self, f):
        """Copy the owner's value to every duplicate of a node."""
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        ncomp = f.size // self.ns
        om = np.tile(self.omask.reshape(-1), ncomp).reshape(f.shape)
        return self.halo_sum(np.where(om == 1, f, 0.0))

    def kerngen(self, k, src, bc_cmb, bc_surf, diag=False, halo=True):
        """halo=False: the copy-wise result (no additive halo), every diamond's copy holding its own cells' sum"""
        dst = np.zeros((3,) + self.shape)
        k = np.ascontiguousarray(k, dtype=np.float64)
        src = np.ascontiguousarray(src, dtype=np.float64)
        fn = lib().or_kerngen_apply if halo else lib().or_kerngen_apply_copywise
        fn(self.L, _p(self.coords), _p(self.radii), _p(k), _p(src), _p(dst), bc_cmb, bc_surf, int(diag))
        return dst

    def laplace(self, src, treat_boundary=True, diag=False):
        dst = np.zeros(self.shape)
        src = np.ascontiguousarray(src, dtype=np.float64)
        lib().or_laplace_apply(self.L, _p(self.coords), _p(self.radii), _p(src), _p(dst),
                               int(treat_boundary), int(diag))
        return dst

    def epsdivdiv3x2(self, k, src, treat_boundary=True, diag=False):
        dst = np.zeros((3,) + self.shape)
        lib().or_epsdivdiv3x2_apply(self.L, _p(self.coords), _p(self.radii), _p(np.ascontiguousarray(k, dtype=np.float64)),
                                    _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst), int(treat_boundary),
                                    int(diag))
        return dst

    def divkgrad(self, k, src, treat_boundary=True, diag=False, single=False):
        dst = np.zeros(self.shape)
        lib().or_divkgrad_apply(self.L, _p(self.coords), _p(self.radii), _p(np.ascontiguousarray(k, dtype=np.float64)),
                                _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst), int(treat_boundary),
                                int(diag), int(single))
        return dst

    def vector_laplace(self, src, bc_cmb, bc_surf, diag=False):
        dst = np.zeros((3,) + self.shape)
        rc = lib().or_vector_laplace_apply(self.L, _p(self.coords), _p(self.radii),
                                           _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst), bc_cmb, bc_surf,
                                           int(diag))
        if rc != 0:
            raise ValueError("VectorLaplace: Neumann or Dirichlet only")
        return dst

    def divergence(self, coarse, u, bc_cmb, bc_surf):
        dst = np.zeros(coarse.shape)
        u = np.ascontiguousarray(u, dtype=np.float64)
        lib().or_divergence_apply(self.L, _p(self.coords), _p(self.radii), _p(coarse.coords), _p(u), _p(dst),
                                  bc_cmb, bc_surf)
        return dst

    def gradient(self, coarse, p, bc_cmb, bc_surf):
        dst = np.zeros((3,) + self.shape)
        p = np.ascontiguousarray(p, dtype=np.float64)
        lib().or_gradient_apply(self.L, _p(self.coords), _p(self.radii), _p(p), _p(dst), bc_cmb, bc_surf)
        return dst

    def prolong(self, coarse, src, ncomp=3):
        """constant prolongation from `coarse` (level L-1) to this mesh"""
        dst = np.zeros((ncomp,) + self.shape)
        lib().or_prolongation_constant(coarse.L, ncomp, _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst))
        return dst

    def restrict(self, coarse, src, ncomp=3):
        """constant restriction from this mesh to `coarse` (level L-1)"""
        dst = np.zeros((ncomp,) + coarse.shape)
        lib().or_restriction_constant(self.L, ncomp, _p(coarse.coords), _p(np.ascontiguousarray(self.omask)),
                                      _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst))
        return dst

    def prolong_linear(self, coarse, src, ncomp=1):
        """linear prolongation from `coarse` (level L-1) to this mesh"""
        dst = np.zeros((ncomp,) + self.shape)
        lib().or_prolongation_linear(coarse.L, ncomp, _p(self.coords), _p(self.radii),
                                     _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst))
        return dst[0] if ncomp == 1 else dst

    def restrict_linear(self, coarse, src, ncomp=1):
        """linear restriction from this mesh to `coarse` (level L-1)"""
        dst = np.zeros((ncomp,) + coarse.shape)
        lib().or_restriction_linear(self.L, ncomp, _p(self.coords), _p(self.radii), _p(coarse.coords),
                                    _p(np.ascontiguousarray(self.omask)),
                                    _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst))
        return dst[0] if ncomp == 1 else dst

    @property
    def cells(self):
        return 10 * self.N ** 3

    def local_matrices(self, k):
        """kerngen 18x18 wedge matrices [cells][2][18][18] (DIMENSIONWISE, row-major)"""
        mats = np.zeros((self.cells, 2, 18, 18))
        lib().or_kerngen_local_matrices(self.L, _p(self.coords), _p(self.radii),
                                        _p(np.ascontiguousarray(k, dtype=np.float64)), _p(mats))
        return mats

    def gca_coarsen(self, coarse, mats_fine=None, k=None, mode=0):
        """GCA matrices of `coarse` (level L-1) from this level's stored matrices or kerngen matrices of k"""
        out = np.zeros((coarse.cells, 2, 18, 18))
        mf = None if mats_fine is None else _p(np.ascontiguousarray(mats_fine))
        kf = None if k is None else _p(np.ascontiguousarray(k, dtype=np.float64))
        lib().or_gca_coarsen(self.L, _p(self.coords), _p(self.radii), kf, mf, mode, _p(out))
        return out

    def gca_elements(self, k, level_range):
        """GCAElementsCollector: marks [10, N0, N0, N0] (uint8) of the coarsest cells, N0 = N >> level_range"""
        N0 = self.N >> level_range
        marks = np.zeros((10, N0, N0, N0), np.uint8)
        lib().or_gca_elements(self.L, _p(np.ascontiguousarray(k, dtype=np.float64)), level_range, _p(marks))
        return marks

    def agca_coarsen(self, coarse, marks, level_range_coarse, k_coarse, mats_fine=None, k=None):
        """Adaptive GCA matrices of `coarse` (TwoGridGCA with LocalMatrixStorage::Selective, gca.hpp:155-163,
        local_matrix_storage.hpp:185-216): the GCA matrix of every coarse cell whose coarsest ancestor (cell >>
        level_range_coarse) is marked, the kerngen matrix of k_coarse (assembled on the fly by the reference)
        elsewhere"""
        mats = self.gca_coarsen(coarse, mats_fine=mats_fine, k=k)
        asm = coarse.local_matrices(k_coarse)
        N, lr = coarse.N, level_range_coarse
        d, x, y, r = np.meshgrid(np.arange(10), np.arange(N), np.arange(N), np.arange(N), indexing="ij")
        keep = marks[d, x >> lr, y >> lr, r >> lr].reshape(-1) != 0
        mats[~keep] = asm[~keep]
        return mats

    def stored_apply(self, mats, src, bc_cmb, bc_surf, diag=False):
        dst = np.zeros((3,) + self.shape)
        lib().or_stored_apply(self.L, _p(self.coords), _p(self.radii), _p(np.ascontiguousarray(mats)),
                              _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst), bc_cmb, bc_surf, int(diag))
        return dst

    @property
    def fv_shape(self):
        return (10, self.N + 2, self.N + 2, self.N + 2)

    def fv_cell_centers(self):
        c = np.zeros((3,) + self.fv_shape)
        lib().or_fv_cell_centers(self.L, _p(self.coords), _p(self.radii), _p(c))
        return c

    def fv_ghost_update(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        lib().or_fv_ghost_update(self.L, _p(self.coords), _p(f))
        return f

    def fct_dt_stable(self, centers, vel, diffusivity=0.0):
        return lib().or_fct_dt_stable(self.L, _p(self.coords), _p(self.radii), _p(np.ascontiguousarray(centers)),
                                      _p(np.ascontiguousarray(vel, dtype=np.float64)), diffusivity)

    def fct_dirichlet(self, T, T_cmb=1.0, T_surf=0.0, cmb=True, surf=True):
        T = np.ascontiguousarray(T, dtype=np.float64).copy()
        lib().or_fct_dirichlet(self.L, _p(T), T_cmb, T_surf, int(cmb), int(surf))
        return T

    def fct_step(self, centers, vel, T, dt, diffusivity=0.0, source=None, subtract_divergence=True, bcs=None):
        """one FCT step; returns (T_new, T_L); bcs = (T_cmb, T_surface, apply_cmb, apply_surface) or None"""
        T = np.ascontiguousarray(T, dtype=np.float64).copy()
        TL = np.zeros(self.fv_shape)
        b = None if bcs is None else _p(np.array(bcs, dtype=np.float64))
        sp = None if source is None else _p(np.ascontiguousarray(source, dtype=np.float64))
        lib().or_fct_step(self.L, _p(self.coords), _p(self.radii), _p(np.ascontiguousarray(centers)),
                          _p(np.ascontiguousarray(vel, dtype=np.float64)), _p(T), dt, diffusivity, sp,
                          int(subtract_divergence), b, _p(TL))
        return T, TL

    def fv_to_fe_rhs(self, fv=None, lumped_diagonal=False):
        """b = sum_K fv_K int_K phi_i (and / or the lumped diagonal), node copies summed (conversion.hpp:146-190)"""
        b = np.zeros(self.shape) if fv is not None else None
        D = np.zeros(self.shape) if lumped_diagonal else None
        f = None if fv is None else _p(np.ascontiguousarray(fv, dtype=np.float64))
        lib().or_fv_to_fe_rhs(self.L, _p(self.coords), _p(self.radii), f, None if b is None else _p(b),
                              None if D is None else _p(D))
        return b, D

    def l2_project_fv_to_fe(self, fv, lumped=False, max_iterations=1000, rtol=1e-12, atol=1e-12):
        """l2_project_fv_to_fe (PCG on the Q1 mass matrix from x = 0) or its lumped form (conversion.hpp:131-300)"""
        b, D = self.fv_to_fe_rhs(fv, lumped_diagonal=lumped)
        if lumped:
            return b / D
        ones = np.ones(self.shape)
        return pcg(lambda v: self.kmass(ones, v, 0), self.dot, b, max_iterations, rtol, atol)[0]

    def supg(self, vel, src, kappa, dt, mass_scaling=1.0, lumped=False, treat_boundary=False, diag=False):
        """UnsteadyAdvectionDiffusionSUPG apply, halo summed (unsteady_advection_diffusion_supg.hpp:199-420)"""
        dst = np.zeros(self.shape)
        lib().or_supg_apply(self.L, _p(self.coords), _p(self.radii), _p(np.ascontiguousarray(vel, dtype=np.float64)),
                            _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst), kappa, dt, mass_scaling,
                            int(lumped), int(treat_boundary), int(diag))
        return dst

    def l2_project_fe_to_fv(self, fe, fv=None):
        """FV cell averages of the FE scalar fe with the 3x2 rule, lateral ghosts updated (conversion.hpp:349-416);
        the radial ghost cells keep the values of fv (zeros when fv is None)"""
        out = np.zeros(self.fv_shape) if fv is None else np.array(fv, dtype=np.float64)
        lib().or_fe_to_fv(self.L, _p(self.coords), _p(self.radii), _p(np.ascontiguousarray(fe, dtype=np.float64)),
                          _p(out))
        return out

    def stokes_buoyancy_rhs(self, T, rayleigh, bc_cmb, bc_surf):
        """f = VectorMass (Ra T n), n the unit radial direction, Dirichlet rows zeroed, the normal component of
        free-slip rows removed (mantlecirculation.cpp:117-150, 883-899).  As the app calls the enforcement, each
        condition acts on the boundary get_shell_boundary_flag names, the first with that condition (CMB before
        SURFACE; grid/shell/bit_masks.hpp:68-76): with the same condition on both radii only the CMB rows."""
        n = self.coords / np.linalg.norm(self.coords, axis=-1, keepdims=True)
        ones = np.ones(self.shape)
        f = np.stack([self.kmass(ones, rayleigh * T * n[:, :, :, None, c], 0) for c in range(3)])
        nn = np.moveaxis(n, -1, 0)
        for cond in (1, 2):
            r = 0 if bc_cmb == cond else (-1 if bc_surf == cond else None)
            if r is None:
                continue
            if cond == 1:
                f[..., r] = 0.0
            else:
                f[..., r] -= np.sum(f[..., r] * nn, axis=0) * nn
        return f

    def kmass(self, k, src, mode=0):
        dst = np.zeros(self.shape)
        lib().or_kmass_apply(self.L, _p(self.coords), _p(self.radii), _p(np.ascontiguousarray(k, dtype=np.float64)),
                             _p(np.ascontiguousarray(src, dtype=np.float64)), _p(dst), mode)
        return dst

    def laplace_pcg(self, b, max_iterations=1000, relative_tolerance=1e-10, absolute_tolerance=1e-30):
        """Unpreconditioned PCG from x = 0 (linalg/solvers/pcg.hpp:78-160, z = r) on
        Laplace(treat_boundary=True).  Returns (x, iterations)."""
        x = np.zeros(self.shape)
        r = np.array(b, dtype=np.float64)
        p = r.copy()
        r0 = np.sqrt(self.dot(r, r))
        if r0 < absolute_tolerance:
            return x, 0
        for it in range(1, max_iterations + 1):
            rz = self.dot(r, r)
            ap = self.laplace(p, True, False)
            alpha = rz / self.dot(ap, p)
            x += alpha * p
            r -= alpha * ap
            res = np.sqrt(self.dot(r, r))
            if res / r0 <= relative_tolerance or res < absolute_tolerance:
                return x, it
            p = r + (self.dot(r, r) / rz) * p
        return x, max_iterations

    def dot(self, a, b):
        """Owned-masked dot product summed over components."""
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1, self.ns)
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, self.ns)
        om = np.ascontiguousarray(self.omask.reshape(-1))
        return sum(lib().or_masked_dot(self.ns, _p(np.ascontiguousarray(a[i])), _p(np.ascontiguousarray(b[i])), _p(om))
                   for i in range(a.shape[0]))


def fgmres(apply, dot, b, restart, max_iterations, relative_tolerance, absolute_tolerance=1e-30, prec=None):
    """FGMRES from x = 0 (linalg/solvers/fgmres.hpp:100-330): z_j = prec(v_j) (identity when None), modified
    Gram-Schmidt Arnoldi, Givens rotations, the breakdown and stagnation exits, restarts from the true
    residual.  Returns (x, relative residual history: 1 at the start, then one entry per iteration)."""
    eps = np.finfo(np.float64).eps
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    r = b - apply(x)
    beta0 = np.sqrt(dot(r, r))
    r0 = beta0
    hist = [1.0]
    if beta0 <= absolute_tolerance:
        return x, hist
    m, total = restart, 0
    while total < max_iterations:
        V, Z = [r * (1.0 / beta0)], []
        H = np.zeros((m + 1, m))
        g = np.zeros(m + 1)
        cs, sn = np.zeros(m + 1), np.zeros(m + 1)
        g[0] = beta0
        inner, j = 0, 0
        while j < m and total < max_iterations:
            Z.append(V[j].copy() if prec is None else prec(V[j]))
            w = apply(Z[j])
            for i in range(j + 1):
                H[i, j] = dot(w, V[i])
                w = w + (-H[i, j]) * V[i]
            h = np.sqrt(dot(w, w))
            if h < eps * r0:
                H[j + 1, j] = 0.0
                inner = j + 1
                break
            H[j + 1, j] = h
            if h > 0:
                V.append(w * (1.0 / h))
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            a, bb = H[j, j], H[j + 1, j]
            rab = np.hypot(a, bb)
            cs[j] = 1.0 if rab == 0 else a / rab
            sn[j] = 0.0 if rab == 0 else bb / rab
            H[j, j], H[j + 1, j] = rab, 0.0
            if abs(H[j, j]) < eps:
                inner = j
                break
            g[j], g[j + 1] = cs[j] * g[j] + sn[j] * g[j + 1], -sn[j] * g[j] + cs[j] * g[j + 1]
            hist.append(abs(g[j + 1]) / r0)
            inner = j + 1
            if hist[-1] <= relative_tolerance or abs(g[j + 1]) < absolute_tolerance:
                break
            j += 1
            total += 1
        y = np.zeros(inner)
        for row in range(inner - 1, -1, -1):
            y[row] = (g[row] - sum(H[row, col] * y[col] for col in range(row + 1, inner))) / H[row, row]
        acc = np.zeros_like(b)
        for i in range(inner):
            acc = acc + y[i] * Z[i]
        x = x + acc
        r = b - apply(x)
        beta0 = np.sqrt(dot(r, r))
        if beta0 <= absolute_tolerance or beta0 / r0 <= relative_tolerance:
            break
    return x, hist


def pminres(apply, dot, b, max_iterations, relative_tolerance, absolute_tolerance=1e-30, prec=None):
    """Preconditioned MINRES from x = 0 (linalg/solvers/pminres.hpp:30-175; prec None = identity), with the
    reference's three-term updates of v and w and its stopping on |eta|.  Returns (x, relative residual
    history: 1 at the start, then one entry per iteration)."""
    P = (lambda v: v.copy()) if prec is None else prec
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    v_prev, w, w_prev = np.zeros_like(b), np.zeros_like(b), np.zeros_like(b)
    v = b - apply(x)
    z = P(v)
    g_prev, g = 1.0, np.sqrt(dot(z, v))
    eta = g
    s_prev = s = 0.0
    c_prev = c = 1.0
    r0 = g
    hist = [1.0]
    if r0 < absolute_tolerance:
        return x, hist
    for _ in range(max_iterations):
        z = z * (1.0 / g)
        az = apply(z)
        delta = dot(az, z)
        v_prev, v = v, 1.0 * az + (-delta / g) * v + (-g / g_prev) * v_prev
        z_next = P(v)
        g_next = np.sqrt(dot(z_next, v))
        a0 = c * delta - c_prev * s * g
        a1 = np.sqrt(a0 * a0 + g_next * g_next)
        a2 = s * delta + c_prev * c * g
        a3 = s_prev * g
        c_next, s_next = a0 / a1, g_next / a1
        w_prev, w = w, (1.0 / a1) * z + (-a3 / a1) * w_prev + (-a2 / a1) * w
        x = x + (c_next * eta) * w
        eta = -s_next * eta
        hist.append(abs(eta) / r0)
        if hist[-1] <= relative_tolerance or abs(eta) < absolute_tolerance:
            break
        z = z_next
        g_prev, g = g, g_next
        c_prev, c = c, c_next
        s_prev, s = s, s_next
    return x, hist


def pbicgstab(apply, dot, b, l, max_iterations, relative_tolerance, r_shadow, absolute_tolerance=1e-30):
    """PBiCGStab(l) with the identity preconditioner from x = 0 (linalg/solvers/pbicgstab.hpp:98-260): l BiCG
    steps, then the minimal-residual correction with gamma = M^-1 M0 (M_ij = <r_i+1, r_j+1>, M0_j = <r_0, r_j+1>),
    the reference's updates u_0 -= sum gamma_j-1 u_j, x += sum gamma_j r_j, r_0 -= sum gamma_j-1 r_j and
    omega = gamma_l-1; the shadow residual is given (the reference draws it with randomize).  Returns
    (x, history: the relative residual of every statistics row, the final row repeated)."""
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    us = [np.zeros_like(b) for _ in range(l + 1)]
    rs = [b - apply(x)] + [np.zeros_like(b) for _ in range(l)]
    r0 = np.sqrt(dot(rs[0], rs[0]))
    absolute, relative = r0, 1.0
    hist = [1.0]
    if r0 < absolute_tolerance:
        return x, hist + [1.0]
    omega = sigma = 1.0
    for _ in range(1, max_iterations):
        sigma = -omega * sigma
        for j in range(l):
            rho = dot(r_shadow, rs[j])
            beta = rho / sigma
            for i in range(j + 1):
                us[i] = 1.0 * rs[i] + (-beta) * us[i]
            us[j + 1] = apply(us[j])
            sigma = dot(r_shadow, us[j + 1])
            alpha = rho / sigma
            for i in range(j + 1):
                rs[i] = rs[i] + (-alpha) * us[i + 1]
            rs[j + 1] = apply(rs[j])
            x = x + alpha * us[0]
        M0 = np.array([dot(rs[0], rs[j]) for j in range(1, l + 1)])
        M = np.array([[dot(rs[i + 1], rs[j + 1]) for j in range(l)] for i in range(l)])
        gamma = np.linalg.solve(M, M0)
        for j in range(1, l + 1):
            us[0] = us[0] + (-gamma[j - 1]) * us[j]
        for j in range(l):
            x = x + gamma[j] * rs[j]
        for j in range(1, l + 1):
            rs[0] = rs[0] + (-gamma[j - 1]) * rs[j]
        omega = gamma[l - 1]
        absolute = np.sqrt(dot(rs[0], rs[0]))
        relative = absolute / r0
        hist.append(relative)
        if relative <= relative_tolerance or absolute < absolute_tolerance:
            break
    hist.append(relative)
    return x, hist


def power_iteration(apply, dot, start, iterations):
    """Largest-eigenvalue estimate (linalg/solvers/power_iteration.hpp:13-48) from the given start vector (the
    reference draws it with randomize): normalise, apply, then `iterations` times normalise the image, apply
    and take the Rayleigh quotient <v, A v>.  Norms are the owned-masked 2-norms."""
    v = np.asarray(start, dtype=np.float64)
    v = (1.0 / np.sqrt(dot(v, v))) * v
    av = apply(v)
    radius = 0.0
    for _ in range(iterations):
        v = (1.0 / np.sqrt(dot(av, av))) * av
        av = apply(v)
        radius = dot(v, av)
    return radius


def chebyshev_smoother(apply, inv_diag, b, x, order, iterations, lambda_estimate):
    """Chebyshev smoothing (linalg/solvers/chebyshev.hpp:100-160) of A x = b with the inverse diagonal, given the
    power-iteration estimate of the largest eigenvalue of D^-1 A: bounds [0.1, 1.5] x estimate; rho is set once
    and carried across the sweeps, as in the reference.  Returns the updated x."""
    lmax, lmin = 1.5 * lambda_estimate, 0.1 * lambda_estimate
    theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
    sigma = theta / delta
    rho = 1.0 / sigma
    x = np.array(x, dtype=np.float64)
    for _ in range(iterations):
        z = (b - apply(x)) * inv_diag
        d = (1.0 / theta) * z
        x = x + d
        for _ in range(2, order + 1):
            rho_new = 1.0 / (2.0 * sigma - rho)
            beta, alpha = rho_new * rho, 2.0 * rho_new / delta
            z = (b - apply(x)) * inv_diag
            d = alpha * z + beta * d
            x = x + d
            rho = rho_new
    return x


class _StokesParts:
    """The Stokes block operator [A B^T; B 0] (epsilon_divdiv_stokes.hpp:55-90) on flattened (u, p) vectors, its
    owned-masked dot, and the app's preconditioner blocks (mantlecirculation.cpp:684-717): the inverse lumped
    KMass(1 / kp) on the pressure mesh and `sweeps` damped Jacobi sweeps from zero with the kerngen diagonal."""

    def __init__(self, fine, coarse, k, kp, bc_cmb, bc_surf, sweeps, omega):
        self.fine, self.coarse, self.k, self.bc = fine, coarse, k, (bc_cmb, bc_surf)
        self.nu, self.sweeps, self.omega = 3 * fine.ns, sweeps, omega
        self.inv_d = 1.0 / fine.kerngen(k, np.ones((3,) + fine.shape), bc_cmb, bc_surf, diag=True)
        self.inv_m = 1.0 / coarse.kmass(1.0 / np.asarray(kp, dtype=np.float64), np.ones(coarse.shape), mode=2)

    def split(self, v):
        return v[:self.nu].reshape((3,) + self.fine.shape), v[self.nu:].reshape(self.coarse.shape)

    @staticmethod
    def join(u, p):
        return np.concatenate([np.ravel(u), np.ravel(p)])

    def apply(self, v):
        u, p = self.split(v)
        f, c = self.fine, self.coarse
        return self.join(f.kerngen(self.k, u, *self.bc) + f.gradient(c, p, *self.bc), f.divergence(c, u, *self.bc))

    def dot(self, a, b):
        (ua, pa), (ub, pb) = self.split(a), self.split(b)
        return self.fine.dot(ua, ub) + self.coarse.dot(pa, pb)

    def jacobi(self, rhs):
        x1 = np.zeros_like(rhs)
        for _ in range(self.sweeps):
            x1 = x1 + self.omega * (self.inv_d * (rhs - self.fine.kerngen(self.k, x1, *self.bc)))
        return x1

    def triangular(self, v):
        """block_preconditioner_2x2.hpp:205-217: x_2 = P22 b_2, x_1 = P11 (b_1 + B^T x_2), x_2 = -x_2"""
        b1, b2 = self.split(v)
        x2 = b2 * self.inv_m
        t1 = self.fine.gradient(self.coarse, x2, *self.bc) + b1
        return self.join(self.jacobi(t1), -x2)

    def diagonal(self, v):
        """block_preconditioner_2x2.hpp:38-100: x_1 = P11 b_1, x_2 = P22 b_2"""
        b1, b2 = self.split(v)
        return self.join(self.jacobi(b1), b2 * self.inv_m)


def stokes_block_fgmres(fine, coarse, k, kp, b_u, b_p, bc_cmb, bc_surf, restart, max_iterations, tolerance,
                        sweeps, omega):
    """FGMRES on the Stokes block operator with the app's block-triangular preconditioner (Jacobi velocity
    block, see _StokesParts), from x = 0; returns (u, p, relative residual history)."""
    S = _StokesParts(fine, coarse, k, kp, bc_cmb, bc_surf, sweeps, omega)
    x, hist = fgmres(S.apply, S.dot, S.join(b_u, b_p), restart, max_iterations, tolerance, prec=S.triangular)
    u, p = S.split(x)
    return u, p, hist


def stokes_block_minres(fine, coarse, k, kp, b_u, b_p, bc_cmb, bc_surf, max_iterations, tolerance, sweeps, omega):
    """PMINRES on the Stokes block operator with the block-diagonal preconditioner (same blocks), from x = 0;
    returns (u, p, relative residual history)."""
    S = _StokesParts(fine, coarse, k, kp, bc_cmb, bc_surf, sweeps, omega)
    x, hist = pminres(S.apply, S.dot, S.join(b_u, b_p), max_iterations, tolerance, prec=S.diagonal)
    u, p = S.split(x)
    return u, p, hist


def pcg(apply, dot, b, max_iterations, relative_tolerance, absolute_tolerance=1e-30):
    """Unpreconditioned PCG from x = 0 (linalg/solvers/pcg.hpp:78-160 with z = r), the arithmetic of
    Mesh.laplace_pcg for any operator.  Returns (x, iterations)."""
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    r0 = np.sqrt(dot(r, r))
    if r0 < absolute_tolerance:
        return x, 0
    for it in range(1, max_iterations + 1):
        rz = dot(r, r)
        ap = apply(p)
        alpha = rz / dot(ap, p)
        x += alpha * p
        r -= alpha * ap
        res = np.sqrt(dot(r, r))
        if res / r0 <= relative_tolerance or res < absolute_tolerance:
            return x, it
        p = r + (dot(r, r) / rz) * p
    return x, max_iterations


def _vcycles(applies, inv_diags, restricts, prolongs, coarse_solve, b, omega, smooth, cycles):
    """V-cycles from x = 0 (linalg/solvers/multigrid.hpp:108-211) over levels 0 (coarsest) .. n-1: Jacobi pre /
    post smoothing (jacobi.hpp:51-62: x += omega D^-1 (b - A x), `smooth` sweeps), restriction of the residual,
    recursion from a zero correction, additive prolongation; coarse_solve(rhs) on level 0."""
    def jacobi(l, x, rhs):
        for _ in range(smooth):
            x += omega * (inv_diags[l] * (rhs - applies[l](x)))

    def cycle(l, x, rhs):
        if l == 0:
            x[...] = coarse_solve(rhs)
            return
        jacobi(l, x, rhs)
        rc = restricts[l](rhs - applies[l](x))
        ec = np.zeros_like(rc)
        cycle(l - 1, ec, rc)
        x += prolongs[l](ec)
        jacobi(l, x, rhs)

    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    for _ in range(cycles):
        cycle(len(applies) - 1, x, b)
    return x


def laplace_vcycles(meshes, b, omega, smooth, cycles, coarse_max_iterations):
    """Multigrid V-cycles from x = 0 (multigrid.hpp:108-211) on Laplace with Dirichlet rows over `meshes`
    (coarsest first): Jacobi smoothing with the diagonal of the Dirichlet operator, constant scalar restriction
    and additive prolongation, and on the coarsest mesh the unpreconditioned PCG from zero (pcg.hpp; relative
    1e-8, absolute 1e-30)."""
    n = len(meshes)
    applies = [lambda v, m=m: m.laplace(v, True, False) for m in meshes]
    inv = [1.0 / m.laplace(np.ones(m.shape), True, True) for m in meshes]
    restricts = [None] + [lambda r, f=meshes[l], c=meshes[l - 1]: f.restrict(c, r, ncomp=1)[0] for l in range(1, n)]
    prolongs = [None] + [lambda e, f=meshes[l], c=meshes[l - 1]: f.prolong(c, e, ncomp=1)[0] for l in range(1, n)]
    coarse = lambda rhs: meshes[0].laplace_pcg(rhs, coarse_max_iterations, 1e-8, 1e-30)[0]
    return _vcycles(applies, inv, restricts, prolongs, coarse, b, omega, smooth, cycles)


def kerngen_vcycles(meshes, ks, b, bc_cmb, bc_surf, omega, smooth, cycles, coarse_max_iterations):
    """The same V-cycles on the epsilon-div-div (kerngen) operator with boundary conditions (bc_cmb, bc_surf),
    the viscosity ks[l] on meshes[l], Jacobi with the kerngen diagonal, constant vector transfers, and the PCG
    on the coarsest kerngen operator."""
    n = len(meshes)
    applies = [lambda v, m=m, k=k: m.kerngen(k, v, bc_cmb, bc_surf) for m, k in zip(meshes, ks)]
    inv = [1.0 / m.kerngen(k, np.ones((3,) + m.shape), bc_cmb, bc_surf, diag=True) for m, k in zip(meshes, ks)]
    restricts = [None] + [lambda r, f=meshes[l], c=meshes[l - 1]: f.restrict(c, r) for l in range(1, n)]
    prolongs = [None] + [lambda e, f=meshes[l], c=meshes[l - 1]: f.prolong(c, e) for l in range(1, n)]
    coarse = lambda rhs: pcg(applies[0], meshes[0].dot, rhs, coarse_max_iterations, 1e-8)[0]
    return _vcycles(applies, inv, restricts, prolongs, coarse, b, omega, smooth, cycles)

def ref_available():
    return os.path.exists(REF_DUMP)


def run_ref(args, workdir, threads=4, json_out=False):
    """Run the compiled reference (ref_dump); with json_out, parse its last JSON output line."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="false")
    out = subprocess.run([REF_DUMP] + [str(a) for a in args], cwd=workdir, env=env, check=True,
                         stdout=subprocess.PIPE if json_out else subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                         text=True)
    if json_out:
        return json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1])


# ---------------------------------------------------------------------------
# XDMF output / checkpoint format (io/xdmf.hpp:80-145, 283-1115), restated with numpy for one subdomain per
# diamond.  grids: list of dicts {label, in_bytes, out_bytes, vec, data} with data [10, n1, n1, n1] (scalar) or
# [3, 10, n1, n1, n1] (vector) in the node layout (r fastest).

def xdmf_order(grids):
    """the reference's write order: FP32 scalars, FP64 scalars, FP32 vectors, FP64 vectors (io/xdmf.hpp:490-512)"""
    return [g for vec in (1, 3) for ib in (4, 8) for g in grids if g["vec"] == vec and g["in_bytes"] == ib]


def xdmf_geometry(om, pts):
    """node coordinates, subdomain by subdomain in (r, y, x) order, x fastest (io/xdmf.hpp:615-645)"""
    X = om.coords.transpose(0, 2, 1, 3)[:, None] * om.radii[:, :, None, None, None]
    return np.ascontiguousarray(X.astype(np.float32 if pts == 4 else np.float64)).tobytes()


def xdmf_topology(om, conn):
    """six node ids per wedge, two wedges per hex cell in (diamond, r, y, x) order (io/xdmf.hpp:647-690)"""
    n1, N = om.N + 1, om.N
    d, r, y, x = np.meshgrid(np.arange(10), np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    v0 = d * n1 ** 3 + r * n1 ** 2 + y * n1 + x
    v4 = v0 + n1 ** 2
    w = np.stack([v0, v0 + 1, v0 + n1, v4, v4 + 1, v4 + n1,
                  v0 + n1 + 1, v0 + n1, v0 + 1, v4 + n1 + 1, v4 + n1, v4 + 1], axis=-1)
    return np.ascontiguousarray(w.astype(np.int32 if conn == 4 else np.int64)).tobytes()


def xdmf_grid_bytes(data, vec, out_bytes):
    """one grid's file: [10][r][y][x] (x fastest), vector components interleaved (io/xdmf.hpp:692-880)"""
    a = np.transpose(data, (0, 3, 2, 1)) if vec == 1 else np.transpose(data, (1, 4, 3, 2, 0))
    return np.ascontiguousarray(a.astype(np.float32 if out_bytes == 4 else np.float64)).tobytes()


def xdmf_metadata(om, grids, pts):
    """checkpoint_metadata.bin (io/xdmf.hpp:882-1063): version 1, one subdomain per diamond"""
    import struct
    n1 = om.N + 1
    b = struct.pack("<6i", 1, 1, 1, n1, n1, n1) + struct.pack(f"<{n1}d", *om.radii[0])
    order = xdmf_order(grids)
    b += struct.pack("<2i", pts, len(order))
    for g in order:
        lab = g["label"].encode()
        b += struct.pack("<i", len(lab)) + lab + struct.pack("<3i", 2, g["out_bytes"], g["vec"])
    return b + struct.pack("<i", 0) + struct.pack("<10q", *[d << 57 for d in range(10)])


def _xml_escape(s):
    return (s.replace("&", "&amp;").replace('"', "&quot;").replace("'", "&apos;").replace("<", "&lt;")
            .replace(">", "&gt;"))


def xdmf_step_xml(om, grids, step, pts, conn):
    """step_<step>.xmf (io/xdmf.hpp:455-520 with util/xml.hpp: attributes sorted by name, two-space indent)"""
    n1 = om.N + 1
    nodes, elems = 10 * n1 ** 3, 10 * om.N ** 3 * 2

    def item(dtype, dims, prec, content):
        return (f'<DataItem DataType="{dtype}" Dimensions="{dims}" Endian="Little" Format="Binary" '
                f'Precision="{prec}">{_xml_escape(content)}</DataItem>\n')
    s = '<?xml version="1.0" ?>\n<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>\n<Xdmf Version="2.0">\n  <Domain>\n'
    s += '    <Grid GridType="Uniform" Name="Grid">\n      <Geometry Type="XYZ">\n'
    s += "        " + item("Float", f"{nodes} 3", pts, "geometry.bin") + "      </Geometry>\n"
    s += f'      <Topology NumberOfElements="{elems}" Type="Wedge">\n'
    s += "        " + item("Int", f"{6 * elems}", conn, "topology.bin") + "      </Topology>\n"
    for g in xdmf_order(grids):
        kind = "Scalar" if g["vec"] == 1 else "Vector"
        dims = f"{nodes}" if g["vec"] == 1 else f"{nodes} 3"
        s += f'      <Attribute AttributeType="{kind}" Center="Node" Name="{_xml_escape(g["label"])}">\n'
        s += "        " + item("Float", dims, g["out_bytes"], f'{g["label"]}_{step}.bin') + "      </Attribute>\n"
    return s + "    </Grid>\n  </Domain>\n</Xdmf>\n"


def xdmf_read_grid(directory, label, step, om, vec):
    """read_xdmf_checkpoint_grid (io/xdmf.hpp:1270-1500) for one subdomain per diamond: the grid as FP64 in the
    node layout ([10, n1, n1, n1] or [3, 10, n1, n1, n1])"""
    import struct
    with open(os.path.join(directory, "checkpoint_metadata.bin"), "rb") as f:
        md = f.read()
    n1 = om.N + 1
    _, sl, sr, sx, sy, sz = struct.unpack_from("<6i", md, 0)
    pos = 24 + 8 * (sr * (sz - 1) + 1) + 4
    nf, = struct.unpack_from("<i", md, pos)
    pos += 4
    rec = None
    for _ in range(nf):
        ln, = struct.unpack_from("<i", md, pos)
        lab = md[pos + 4:pos + 4 + ln].decode()
        t, nb, vd = struct.unpack_from("<3i", md, pos + 4 + ln)
        pos += 16 + ln
        if lab == label and rec is None:
            rec = (nb, vd)
    pos += 4
    ids = struct.unpack_from(f"<{10 * sl * sl * sr}q", md, pos)
    nb, vd = rec
    assert vd == (1 if not vec else 3) and (sx, sy, sz) == (n1, n1, n1)
    raw = np.fromfile(os.path.join(directory, f"{label}_{step}.bin"), dtype=np.float32 if nb == 4 else np.float64)
    chunk = n1 ** 3 * vd
    parts = [raw[ids.index(d << 57) * chunk:(ids.index(d << 57) + 1) * chunk] for d in range(10)]
    a = np.stack(parts).astype(np.float64)
    if vd == 1:
        return np.transpose(a.reshape(10, n1, n1, n1), (0, 3, 2, 1)).copy()
    return np.transpose(a.reshape(10, n1, n1, n1, 3), (4, 0, 3, 2, 1)).copy()


def xdmf_write_dir(directory, om, steps, pts=4, conn=8, order=None):
    """A whole checkpoint directory from the restatement: steps = [grids of write 0, grids of write 1, ...];
    order: the diamonds' order in the data files (a permutation of 0..9; io/xdmf.hpp allows any, the metadata's
    id list says where each subdomain is)."""
    import struct
    order = list(range(10)) if order is None else list(order)
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "geometry.bin"), "wb") as f:
        f.write(_permute_chunks(xdmf_geometry(om, pts), order))
    with open(os.path.join(directory, "topology.bin"), "wb") as f:
        f.write(xdmf_topology(om, conn))
    md = xdmf_metadata(om, steps[0], pts)
    md = md[:-80] + struct.pack("<10q", *[d << 57 for d in order])
    with open(os.path.join(directory, "checkpoint_metadata.bin"), "wb") as f:
        f.write(md)
    for step, grids in enumerate(steps):
        for g in grids:
            with open(os.path.join(directory, f'{g["label"]}_{step}.bin'), "wb") as f:
                f.write(_permute_chunks(xdmf_grid_bytes(g["data"], g["vec"], g["out_bytes"]), order))
        with open(os.path.join(directory, f"step_{step}.xmf"), "w") as f:
            f.write(xdmf_step_xml(om, grids, step, pts, conn))


def _permute_chunks(b, order):
    n = len(b) // 10
    return b"".join(b[d * n:(d + 1) * n] for d in order)
