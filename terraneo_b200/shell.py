"""Python mirror of the reference's shell/vector/operator interface over the C ABI.

Names follow the reference (src/terra): a mesh replaces DistributedDomain with
one subdomain per diamond (grid/shell/spherical_shell.hpp:2520), VectorQ1Scalar /
VectorQ1Vec hold device fields in the reference layout (linalg/vector_q1.hpp),
and operator classes expose apply_impl(src, dst) (linalg/operator.hpp:57-71).
Device memory is allocated through torch (plumbing only); every computation is
a call into libterraneo_b200.so.
"""
import ctypes

import numpy as np
import torch

from . import _capi as C

_DT = {torch.float64: "f64", torch.float32: "f32"}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class ShellMesh:
    """Thick spherical shell, 10 diamonds x N x N lateral x N radial cells, N = 2**level."""

    def __init__(self, level, r_min=0.55, r_max=1.0):
        h = ctypes.c_void_p()
        C.check(C.lib().tn_mesh_create(level, r_min, r_max, ctypes.byref(h)), "tn_mesh_create")
        self._h = h
        self.level, self.N, self.n1 = level, 1 << level, (1 << level) + 1
        ns, nu, lv = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int()
        C.check(C.lib().tn_mesh_dims(h, ctypes.byref(lv), ctypes.byref(ns), ctypes.byref(nu)), "tn_mesh_dims")
        self.stored_nodes, self.unique_nodes = ns.value, nu.value
        self.shape = (10, self.n1, self.n1, self.n1)
        self.r_min, self.r_max = r_min, r_max

    @property
    def handle(self):
        return self._h

    def geometry(self):
        coords = np.zeros((10, self.n1, self.n1, 3))
        radii = np.zeros((10, self.n1))
        C.check(C.lib().tn_mesh_geometry(self._h, coords.ctypes.data, radii.ctypes.data), "tn_mesh_geometry")
        return coords, radii

    def masks(self):
        b = np.zeros(self.shape, np.uint8)
        o = np.zeros(self.shape, np.uint8)
        C.check(C.lib().tn_mesh_masks(self._h, b.ctypes.data, o.ctypes.data), "tn_mesh_masks")
        return b, o

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and C is not None and C._lib is not None:
            C.lib().tn_mesh_destroy(h)
            self._h = None


class _VectorBase:
    ncomp = 1

    def __init__(self, mesh, dtype=torch.float64, data=None):
        self.mesh = mesh
        self.dtype = dtype
        if data is None:
            data = torch.zeros((self.ncomp,) + mesh.shape, dtype=dtype, device="cuda")
        self.data = data  # shallow handle semantics: copies share this tensor

    @property
    def tag(self):
        return _DT[self.dtype]

    def comp_ptrs(self):
        return C.ptrs(*[self.data[c].data_ptr() for c in range(self.ncomp)])

    # VectorLike (linalg/vector.hpp:8-37)
    def lincomb_impl(self, c, xs, c0=0.0):
        if len(c) != len(xs):
            raise RuntimeError("lincomb: c and x must have the same size")
        if len(xs) > 3:
            raise RuntimeError("lincomb: not implemented")
        xarr = (ctypes.c_void_p * 9)()
        for i, x in enumerate(xs):
            for k in range(self.ncomp):
                xarr[3 * i + k] = x.data[k].data_ptr()
        carr = (ctypes.c_double * 3)(*([float(v) for v in c] + [0.0] * (3 - len(c))))
        f = getattr(C.lib(), f"tn_vec_lincomb_{self.tag}")
        C.check(f(self.mesh.handle, self.ncomp, self.comp_ptrs(), float(c0), len(xs), carr, xarr, _stream()), "lincomb")

    def dot_impl(self, other):
        r = ctypes.c_double()
        f = getattr(C.lib(), f"tn_vec_dot_{self.tag}")
        C.check(f(self.mesh.handle, self.ncomp, self.comp_ptrs(), other.comp_ptrs(), ctypes.byref(r), _stream()), "dot")
        return r.value

    def masked_sum_impl(self):
        """the sum over owned nodes (masked_sum with the ownership mask), components summed"""
        r = ctypes.c_double()
        f = getattr(C.lib(), f"tn_vec_sum_{self.tag}")
        C.check(f(self.mesh.handle, self.ncomp, self.comp_ptrs(), ctypes.byref(r), _stream()), "sum")
        return r.value

    def invert_entries_impl(self):
        C.check(getattr(C.lib(), f"tn_vec_invert_{self.tag}")(self.mesh.handle, self.ncomp, self.comp_ptrs(),
                                                              _stream()), "invert")

    def scale_with_vector_impl(self, x):
        C.check(getattr(C.lib(), f"tn_vec_mult_{self.tag}")(self.mesh.handle, self.ncomp, self.comp_ptrs(),
                                                            x.comp_ptrs(), _stream()), "mult")

    def has_nan_or_inf_impl(self):
        r = ctypes.c_int()
        C.check(getattr(C.lib(), f"tn_vec_has_nan_or_inf_{self.tag}")(self.mesh.handle, self.ncomp, self.comp_ptrs(),
                                                                      ctypes.byref(r), _stream()), "has_nan")
        return bool(r.value)

    def max_abs_entry_impl(self):
        if self.dtype != torch.float64:
            raise NotImplementedError
        r = ctypes.c_double()
        C.check(C.lib().tn_vec_max_abs_f64(self.mesh.handle, self.ncomp, self.comp_ptrs(), ctypes.byref(r),
                                           _stream()), "max_abs")
        return r.value

    def swap_impl(self, other):
        self.data, other.data = other.data, self.data

    def halo_sum(self):
        f = getattr(C.lib(), f"tn_halo_sum_{self.tag}")
        C.check(f(self.mesh.handle, self.comp_ptrs(), self.ncomp, _stream()), "halo_sum")

    def numpy(self):
        return self.data.detach().cpu().numpy()

    def set_numpy(self, arr):
        self.data.copy_(torch.as_tensor(np.asarray(arr).reshape(self.data.shape), dtype=self.dtype))


class VectorQ1Scalar(_VectorBase):
    ncomp = 1


class VectorQ1Vec(_VectorBase):
    ncomp = 3


class EpsilonDivDivKerngen:
    """EpsilonDivDivKerngen (fe/wedge/operators/shell/epsilon_divdiv_kerngen.hpp:62)."""

    def __init__(self, mesh, k, bc_cmb, bc_surface, diagonal=False, apply_mode=C.APPLY_REPLACE,
                 comm_mode=C.COMM_ADDITIVE, penalty_eps=1.0):
        self.mesh, self.k = mesh, k
        self.p = C.EpsDivDivParams(bc_cmb, bc_surface, int(diagonal), apply_mode, comm_mode, penalty_eps)

    def set_diagonal(self, v):
        self.p.diagonal = int(v)

    def set_operator_apply_and_communication_modes(self, apply_mode, comm_mode):
        self.p.apply_mode, self.p.comm_mode = apply_mode, comm_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_epsdivdiv_apply_{src.tag}")
        C.check(f(self.mesh.handle, ctypes.byref(self.p), ctypes.c_void_p(self.k.data.data_ptr()), src.comp_ptrs(),
                  dst.comp_ptrs(), _stream()), "epsdivdiv_apply")


def local_matrix_count(mesh):
    n = ctypes.c_size_t()
    C.check(C.lib().tn_local_matrix_count(mesh.handle, ctypes.byref(n)), "local_matrix_count")
    return n.value


def kerngen_local_matrices(mesh, k=None):
    """kerngen 18x18 wedge matrices in the library's stored layout (packed upper triangles, 32 wedges
    interleaved; torch FP64 vector of tn_local_matrix_count entries)."""
    out = torch.empty(local_matrix_count(mesh), dtype=torch.float64, device="cuda")
    kp = ctypes.c_void_p(k.data.data_ptr()) if k is not None else None
    C.check(C.lib().tn_kerngen_local_matrices_f64(mesh.handle, kp, ctypes.c_void_p(out.data_ptr()), _stream()),
            "kerngen_local_matrices")
    return out


def gca_coarsen(fine, coarse, k_fine=None, mats_fine=None, mode=0):
    """TwoGridGCA matrices of `coarse` from kerngen (k_fine) or stored (mats_fine) fine matrices."""
    out = torch.empty(local_matrix_count(coarse), dtype=torch.float64, device="cuda")
    kp = ctypes.c_void_p(k_fine.data.data_ptr()) if k_fine is not None else None
    mp = ctypes.c_void_p(mats_fine.data_ptr()) if mats_fine is not None else None
    C.check(C.lib().tn_gca_coarsen_f64(fine.handle, coarse.handle, kp, mp, mode, ctypes.c_void_p(out.data_ptr()),
                                       _stream()), "gca_coarsen")
    return out


def gca_elements(fine, k_fine, level_range):
    """GCAElementsCollector (linalg/solvers/gca/gca_elements_collector.hpp:19-96): uint8 marks [10, N0, N0, N0]
    of the coarsest cells (N0 = N >> level_range) below which the adaptive GCA builds Galerkin matrices."""
    N0 = fine.N >> level_range
    marks = torch.empty((10, N0, N0, N0), dtype=torch.uint8, device="cuda")
    C.check(C.lib().tn_gca_elements_f64(fine.handle, ctypes.c_void_p(k_fine.data.data_ptr()), level_range,
                                        ctypes.c_void_p(marks.data_ptr()), _stream()), "gca_elements")
    return marks


def agca_coarsen(fine, coarse, marks, level_range_coarse, k_coarse=None, k_fine=None, mats_fine=None):
    """Adaptive GCA matrices of `coarse` (TwoGridGCA with Selective storage, gca.hpp:155-163): the GCA matrices of
    the cells below a marked coarsest cell (cell >> level_range_coarse), the kerngen matrices of k_coarse (None:
    k = 1) elsewhere, in the stored layout."""
    out = gca_coarsen(fine, coarse, k_fine=k_fine, mats_fine=mats_fine)
    kp = ctypes.c_void_p(k_coarse.data.data_ptr()) if k_coarse is not None else None
    C.check(C.lib().tn_agca_unmarked_local_matrices_f64(coarse.handle, kp, ctypes.c_void_p(marks.data_ptr()),
                                                        level_range_coarse, ctypes.c_void_p(out.data_ptr()),
                                                        _stream()), "agca_unmarked_local_matrices")
    return out


def stored_pcg(op, b, x, max_iterations=50, relative_tolerance=1e-6, absolute_tolerance=1e-30, check_every=8):
    """Unpreconditioned PCG (linalg/solvers/pcg.hpp:78) on a StoredEpsilonDivDiv (FP64) with the operator's steps
    fused into the PCG steps (tn_stored_pcg_f64); x is updated in place.
    Returns (iterations, relative residual history)."""
    m = op.mesh
    work = [VectorQ1Vec(m) for _ in range(4)]
    ptrs = (ctypes.c_void_p * 12)(*[w.data[c].data_ptr() for w in work for c in range(3)])
    state = torch.zeros(9 + max_iterations, dtype=torch.float64, device="cuda")
    C.check(C.lib().tn_stored_pcg_f64(m.handle, ctypes.c_void_p(op.mats.data_ptr()), ctypes.byref(op.prm),
                                      b.comp_ptrs(), x.comp_ptrs(), ptrs, ctypes.c_void_p(state.data_ptr()),
                                      max_iterations, relative_tolerance, absolute_tolerance, check_every,
                                      _stream()), "stored_pcg")
    st = state.cpu().numpy()
    its = int(st[5])
    return its, list(st[8:9 + its])


class StoredEpsilonDivDiv:
    """EpsilonDivDivKerngen with OperatorStoredMatrixMode::Full: stored wedge matrices + boundary treatment."""

    def __init__(self, mesh, mats, bc_cmb, bc_surface, diagonal=False, apply_mode=C.APPLY_REPLACE,
                 comm_mode=C.COMM_ADDITIVE, penalty_eps=1.0):
        self.mesh, self.mats = mesh, mats
        self.prm = C.EpsDivDivParams(bc_cmb, bc_surface, int(diagonal), apply_mode, comm_mode, penalty_eps)

    def set_diagonal(self, v):
        self.prm.diagonal = int(v)

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_stored_epsdivdiv_apply_{src.tag}")
        C.check(f(self.mesh.handle, ctypes.c_void_p(self.mats.data_ptr()), ctypes.byref(self.prm), src.comp_ptrs(),
                  dst.comp_ptrs(), _stream()), "stored_apply")


class Laplace:
    """Laplace (fe/wedge/operators/shell/laplace.hpp:18)."""

    def __init__(self, mesh, treat_boundary, diagonal=False, apply_mode=C.APPLY_REPLACE, comm_mode=C.COMM_ADDITIVE):
        self.mesh = mesh
        self.treat, self.diag, self.am, self.cm = int(treat_boundary), int(diagonal), apply_mode, comm_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_laplace_apply_{src.tag}")
        C.check(f(self.mesh.handle, self.treat, self.diag, self.am, self.cm, ctypes.c_void_p(src.data.data_ptr()),
                  ctypes.c_void_p(dst.data.data_ptr()), _stream()), "laplace_apply")


class EpsilonDivDiv:
    """EpsilonDivDiv (fe/wedge/operators/shell/epsilon_divdiv.hpp:18): 3x2 rule, k interpolated, Dirichlet radii."""

    def __init__(self, mesh, k, treat_boundary, diagonal=False, apply_mode=C.APPLY_REPLACE, comm_mode=C.COMM_ADDITIVE):
        self.mesh, self.k = mesh, k
        self.treat, self.diag, self.am, self.cm = int(treat_boundary), int(diagonal), apply_mode, comm_mode

    def set_diagonal(self, v):
        self.diag = int(v)

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_epsdivdiv3x2_apply_{src.tag}")
        C.check(f(self.mesh.handle, ctypes.c_void_p(self.k.data.data_ptr()), self.treat, self.diag, self.am, self.cm,
                  src.comp_ptrs(), dst.comp_ptrs(), _stream()), "epsdivdiv3x2_apply")


class DivKGrad:
    """DivKGrad (fe/wedge/operators/shell/div_k_grad.hpp:18): int k grad u . grad v."""

    def __init__(self, mesh, k, treat_boundary, diagonal=False, apply_mode=C.APPLY_REPLACE,
                 comm_mode=C.COMM_ADDITIVE, single_quadpoint=False):
        self.mesh, self.k = mesh, k
        self.treat, self.diag, self.am, self.cm = int(treat_boundary), int(diagonal), apply_mode, comm_mode
        self.single = int(single_quadpoint)

    def set_diagonal(self, v):
        self.diag = int(v)

    def set_single_quadpoint(self, v):
        self.single = int(v)

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_divkgrad_apply_{src.tag}")
        C.check(f(self.mesh.handle, ctypes.c_void_p(self.k.data.data_ptr()), self.treat, self.diag, self.single,
                  self.am, self.cm, ctypes.c_void_p(src.data.data_ptr()), ctypes.c_void_p(dst.data.data_ptr()),
                  _stream()), "divkgrad_apply")


class VectorLaplace:
    """VectorLaplace (fe/wedge/operators/shell/vector_laplace.hpp:32); Neumann / Dirichlet only."""

    def __init__(self, mesh, bc_cmb, bc_surface, diagonal=False, apply_mode=C.APPLY_REPLACE,
                 comm_mode=C.COMM_ADDITIVE):
        self.mesh, self.bc = mesh, (bc_cmb, bc_surface)
        self.diag, self.am, self.cm = int(diagonal), apply_mode, comm_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_vector_laplace_apply_{src.tag}")
        C.check(f(self.mesh.handle, self.bc[0], self.bc[1], self.diag, self.am, self.cm, src.comp_ptrs(),
                  dst.comp_ptrs(), _stream()), "vector_laplace_apply")


class KMass:
    """KMass (fe/wedge/operators/shell/kmass.hpp:17); k=None gives Mass. mode: 0 full, 1 diagonal, 2 lumped."""

    def __init__(self, mesh, k=None, mode=0, apply_mode=C.APPLY_REPLACE, comm_mode=C.COMM_ADDITIVE):
        self.mesh, self.k, self.mode, self.am, self.cm = mesh, k, mode, apply_mode, comm_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_kmass_apply_{src.tag}")
        kp = ctypes.c_void_p(self.k.data.data_ptr()) if self.k is not None else ctypes.c_void_p(0)
        C.check(f(self.mesh.handle, kp, self.mode, self.am, self.cm, ctypes.c_void_p(src.data.data_ptr()),
                  ctypes.c_void_p(dst.data.data_ptr()), _stream()), "kmass_apply")


class VectorMass:
    """VectorMass (fe/wedge/operators/shell/vector_mass.hpp:17): Mass (k = 1) on each component; full or diagonal."""

    def __init__(self, mesh, diagonal=False, apply_mode=C.APPLY_REPLACE, comm_mode=C.COMM_ADDITIVE):
        self.mesh, self.mode, self.am, self.cm = mesh, int(bool(diagonal)), apply_mode, comm_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_kmass_apply_{src.tag}")
        for c in range(src.ncomp):
            C.check(f(self.mesh.handle, ctypes.c_void_p(0), self.mode, self.am, self.cm,
                      ctypes.c_void_p(src.data[c].data_ptr()), ctypes.c_void_p(dst.data[c].data_ptr()), _stream()),
                    "vector_mass_apply")


class Divergence:
    """Divergence (fe/wedge/operators/shell/divergence.hpp:30): fine velocity -> coarse pressure."""

    def __init__(self, mesh_u, mesh_p, bc_cmb, bc_surface, apply_mode=C.APPLY_REPLACE, comm_mode=C.COMM_ADDITIVE):
        self.mu, self.mp, self.bc = mesh_u, mesh_p, (bc_cmb, bc_surface)
        self.am, self.cm = apply_mode, comm_mode

    def set_operator_apply_and_communication_modes(self, apply_mode, comm_mode):
        self.am, self.cm = apply_mode, comm_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_divergence_apply_{src.tag}")
        C.check(f(self.mu.handle, self.mp.handle, self.bc[0], self.bc[1], self.am, self.cm, src.comp_ptrs(),
                  ctypes.c_void_p(dst.data.data_ptr()), _stream()), "divergence_apply")


class Gradient:
    """Gradient (fe/wedge/operators/shell/gradient.hpp:28): coarse pressure -> fine velocity."""

    def __init__(self, mesh_u, mesh_p, bc_cmb, bc_surface, apply_mode=C.APPLY_REPLACE, comm_mode=C.COMM_ADDITIVE):
        self.mu, self.mp, self.bc = mesh_u, mesh_p, (bc_cmb, bc_surface)
        self.am, self.cm = apply_mode, comm_mode

    def set_operator_apply_and_communication_modes(self, apply_mode, comm_mode):
        self.am, self.cm = apply_mode, comm_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_gradient_apply_{src.tag}")
        C.check(f(self.mu.handle, self.mp.handle, self.bc[0], self.bc[1], self.am, self.cm,
                  ctypes.c_void_p(src.data.data_ptr()), dst.comp_ptrs(), _stream()), "gradient_apply")


class ProlongationVecConstant:
    """ProlongationVecConstant (fe/wedge/operators/shell/prolongation_constant.hpp:103): coarse -> fine."""

    def __init__(self, mesh_fine, mesh_coarse, apply_mode=C.APPLY_REPLACE):
        self.mf, self.mc, self.am = mesh_fine, mesh_coarse, apply_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_prolongation_constant_{src.tag}")
        C.check(f(self.mf.handle, self.mc.handle, src.ncomp, self.am, src.comp_ptrs(), dst.comp_ptrs(), _stream()),
                "prolongation")


class RestrictionVecConstant:
    """RestrictionVecConstant (fe/wedge/operators/shell/restriction_constant.hpp:134): fine -> coarse."""

    def __init__(self, mesh_fine, mesh_coarse):
        self.mf, self.mc = mesh_fine, mesh_coarse

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_restriction_constant_{src.tag}")
        C.check(f(self.mf.handle, self.mc.handle, src.ncomp, src.comp_ptrs(), dst.comp_ptrs(), _stream()),
                "restriction")


class ProlongationLinear:
    """ProlongationLinear (fe/wedge/operators/shell/prolongation_linear.hpp:15): coarse -> fine, per component."""

    def __init__(self, mesh_fine, mesh_coarse, apply_mode=C.APPLY_REPLACE):
        self.mf, self.mc, self.am = mesh_fine, mesh_coarse, apply_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_prolongation_linear_{src.tag}")
        C.check(f(self.mf.handle, self.mc.handle, src.ncomp, self.am, src.comp_ptrs(), dst.comp_ptrs(), _stream()),
                "prolongation_linear")


class RestrictionLinear:
    """RestrictionLinear (fe/wedge/operators/shell/restriction_linear.hpp:15): fine -> coarse, per component."""

    def __init__(self, mesh_fine, mesh_coarse):
        self.mf, self.mc = mesh_fine, mesh_coarse

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_restriction_linear_{src.tag}")
        C.check(f(self.mf.handle, self.mc.handle, src.ncomp, src.comp_ptrs(), dst.comp_ptrs(), _stream()),
                "restriction_linear")


def laplace_pcg(mesh, b, x, max_iterations=1000, relative_tolerance=1e-10, absolute_tolerance=1e-30):
    """Unpreconditioned PCG (linalg/solvers/pcg.hpp:78) on Laplace(treat_boundary=True); x is updated in place.
    Returns (iterations, relative residual)."""
    it, rr = ctypes.c_int(), ctypes.c_double()
    C.check(C.lib().tn_laplace_pcg_solve_f64(mesh.handle, ctypes.c_void_p(b.data.data_ptr()),
                                             ctypes.c_void_p(x.data.data_ptr()), max_iterations, relative_tolerance,
                                             absolute_tolerance, ctypes.byref(it), ctypes.byref(rr)), "laplace_pcg")
    return it.value, rr.value


def divkgrad_mg_pcg(level, b, x, k=None, mg_levels=3, smoother=1, smoothing_steps=2, chebyshev_order=2,
                    power_iterations=10, jacobi_omega=0.6, vcycles=1, coarse_max_iterations=100,
                    coarse_relative_tolerance=1e-8, max_iterations=200, relative_tolerance=1e-10,
                    absolute_tolerance=1e-30, r_min=0.55, r_max=1.0, krylov=0):
    """Multigrid-preconditioned Krylov solve on DivKGrad (k None: Laplace), Dirichlet radii; x updated in place.
    smoother: 0 Chebyshev, 1 Jacobi; krylov: 0 PCG, 1 PBiCGStab(2), 2 PMINRES.  Returns (iterations, relres)."""
    prm = C.ScalarMGParams(level, mg_levels, smoother, smoothing_steps, chebyshev_order, power_iterations,
                           jacobi_omega, vcycles, coarse_max_iterations, coarse_relative_tolerance, max_iterations,
                           relative_tolerance, absolute_tolerance, krylov)
    it, rr = ctypes.c_int(), ctypes.c_double()
    kp = ctypes.c_void_p(k.data.data_ptr()) if k is not None else None
    C.check(C.lib().tn_divkgrad_mg_pcg_solve_f64(ctypes.byref(prm), r_min, r_max, kp,
                                                 ctypes.c_void_p(b.data.data_ptr()),
                                                 ctypes.c_void_p(x.data.data_ptr()), ctypes.byref(it),
                                                 ctypes.byref(rr)), "divkgrad_mg_pcg")
    return it.value, rr.value


class StokesSolver:
    """FGMRES + block-triangular preconditioner + multigrid on the viscous block
    (apps/mantlecirculation/mantlecirculation.cpp:486-735); mg_fp32 selects the FP32 V-cycle.
    outer: 0 FGMRES(restart) in FP64; 1 PMINRES + block-diagonal preconditioner; 2 mixed-precision
    iterative refinement (needs mg_fp32): FP64 residual and update around FGMRES cycles done entirely in
    FP32, the coarsest-level PCG in FP64 (no counterpart in the reference)."""

    def __init__(self, level, viscosity, mg_levels=4, bc_cmb=C.BC_FREESLIP, bc_surface=C.BC_FREESLIP, mg_fp32=True,
                 chebyshev_order=3, smoothing_steps=2, power_iterations=10, vcycles=1, coarse_max_iterations=50,
                 coarse_relative_tolerance=1e-6, restart=30, max_iterations=200, relative_tolerance=1e-8,
                 absolute_tolerance=1e-30, r_min=0.55, r_max=1.0, gca=0, outer=0, eager=False,
                 chebyshev_estimates=None):
        """chebyshev_estimates: None (power iterations, as the reference) or one largest-eigenvalue estimate of
        D^-1 A per multigrid level, coarsest first, used as given."""
        est = None
        if chebyshev_estimates is not None:
            assert len(chebyshev_estimates) == mg_levels
            self._est = (ctypes.c_double * mg_levels)(*[float(e) for e in chebyshev_estimates])
            est = ctypes.cast(self._est, ctypes.POINTER(ctypes.c_double))
        self.prm = C.StokesParams(level, mg_levels, bc_cmb, bc_surface, int(mg_fp32), chebyshev_order, smoothing_steps,
                                  power_iterations, vcycles, coarse_max_iterations, coarse_relative_tolerance, restart,
                                  max_iterations, relative_tolerance, absolute_tolerance, int(gca), int(outer),
                                  int(eager), est)
        h = ctypes.c_void_p()
        C.check(C.lib().tn_stokes_solver_create(ctypes.byref(self.prm), r_min, r_max,
                                                ctypes.c_void_p(viscosity.data.data_ptr()), ctypes.byref(h)),
                "stokes_solver_create")
        self._h = h

    def solve(self, f_u, f_p, x_u, x_p):
        it, rr = ctypes.c_int(), ctypes.c_double()
        C.check(C.lib().tn_stokes_solve(self._h, f_u.comp_ptrs(), ctypes.c_void_p(f_p.data.data_ptr()),
                                        x_u.comp_ptrs(), ctypes.c_void_p(x_p.data.data_ptr()), ctypes.byref(it),
                                        ctypes.byref(rr)), "stokes_solve")
        return it.value, rr.value

    def history(self):
        n, skips = ctypes.c_int(), ctypes.c_int()
        C.check(C.lib().tn_stokes_history(self._h, None, 0, ctypes.byref(n), ctypes.byref(skips)), "history")
        out = (ctypes.c_double * max(1, n.value))()
        C.check(C.lib().tn_stokes_history(self._h, out, n.value, ctypes.byref(n), ctypes.byref(skips)), "history")
        return list(out[:n.value]), skips.value

    def viscosity_backward(self, u, grad_u, grad_log_k, comm_mode=C.COMM_SKIP, lambda_u=None, lambda_p=None):
        """dJ/dlog k from the copy-wise dJ/du (adjoint solve + backward kernel); returns adjoint iterations."""
        it = ctypes.c_int()
        C.check(C.lib().tn_stokes_viscosity_backward(
            self._h, u.comp_ptrs(), grad_u.comp_ptrs(), comm_mode, ctypes.c_void_p(grad_log_k.data_ptr()),
            lambda_u.comp_ptrs() if lambda_u is not None else None,
            ctypes.c_void_p(lambda_p.data.data_ptr()) if lambda_p is not None else None, ctypes.byref(it)),
            "viscosity_backward")
        return it.value

    def apply(self, u, p, out_u, out_p):
        C.check(C.lib().tn_stokes_apply(self._h, u.comp_ptrs(), ctypes.c_void_p(p.data.data_ptr()), out_u.comp_ptrs(),
                                        ctypes.c_void_p(out_p.data.data_ptr())), "stokes_apply")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and C is not None and C._lib is not None:
            C.lib().tn_stokes_solver_destroy(h)
            self._h = None


def epsdivdiv_kgrad(mesh, bc_cmb, bc_surface, u, lam, out, comm_mode=C.COMM_ADDITIVE):
    """out = d(lam^T A(k) u)/dk (tn_epsdivdiv_kgrad_*); out is a VectorQ1Scalar."""
    f = getattr(C.lib(), f"tn_epsdivdiv_kgrad_{u.tag}")
    C.check(f(mesh.handle, bc_cmb, bc_surface, comm_mode, u.comp_ptrs(), lam.comp_ptrs(),
              ctypes.c_void_p(out.data.data_ptr()), _stream()), "epsdivdiv_kgrad")


class FCTAdvectionDiffusion:
    """FV FCT advection-diffusion (fv/hex/operators/fct_advection_diffusion.hpp) on the cells of `mesh`:
    cell centres computed once, workspace kept; fields are torch [10, N+2, N+2, N+2] FP64 tensors."""

    def __init__(self, mesh):
        self.mesh = mesh
        n2 = mesh.N + 2
        self.fv_shape = (10, n2, n2, n2)
        self.centers = torch.zeros((3,) + self.fv_shape, dtype=torch.float64, device="cuda")
        C.check(C.lib().tn_fv_cell_centers_f64(mesh.handle, C.ptrs(*[self.centers[a].data_ptr() for a in range(3)]),
                                               _stream()), "fv_cell_centers")
        n = ctypes.c_size_t()
        C.check(C.lib().tn_fct_workspace_size(mesh.handle, ctypes.byref(n)), "fct_workspace_size")
        self.work = torch.zeros(n.value, dtype=torch.float64, device="cuda")

    def field(self):
        return torch.zeros(self.fv_shape, dtype=torch.float64, device="cuda")

    def _c(self):
        return C.ptrs(*[self.centers[a].data_ptr() for a in range(3)])

    def dt_stable(self, vel, diffusivity=0.0):
        dt = ctypes.c_double()
        C.check(C.lib().tn_fct_dt_stable_f64(self.mesh.handle, vel.comp_ptrs(), self._c(), diffusivity,
                                             ctypes.byref(dt), _stream()), "fct_dt_stable")
        return dt.value

    @staticmethod
    def dirichlet(T_cmb, T_surface, cmb=True, surface=True):
        return C.FCTDirichlet(T_cmb, T_surface, int(cmb), int(surface))

    def apply_dirichlet(self, T, bcs):
        C.check(C.lib().tn_fct_apply_dirichlet_f64(self.mesh.handle, ctypes.c_void_p(T.data_ptr()), ctypes.byref(bcs),
                                                   _stream()), "fct_apply_dirichlet")

    def ghost_update(self, f):
        C.check(C.lib().tn_fv_ghost_update_f64(self.mesh.handle, ctypes.c_void_p(f.data_ptr()), _stream()),
                "fv_ghost_update")

    def step(self, T, vel, dt, diffusivity=0.0, source=None, subtract_divergence=True, bcs=None):
        sp = ctypes.c_void_p(source.data_ptr()) if source is not None else None
        bp = ctypes.byref(bcs) if bcs is not None else None
        C.check(C.lib().tn_fct_step_f64(self.mesh.handle, ctypes.c_void_p(T.data_ptr()), vel.comp_ptrs(), self._c(),
                                        dt, diffusivity, sp, int(subtract_divergence), bp,
                                        ctypes.c_void_p(self.work.data_ptr()), _stream()), "fct_step")

    @property
    def T_L(self):
        return self.work[:self.centers[0].numel()].view(self.fv_shape)


def assign_boundary(y, x=None, c=0.0, cmb=True, surface=True):
    """y = x (or c) on the CMB / SURFACE layers (assign_masked_else_keep_old with the boundary flags)."""
    f = getattr(C.lib(), f"tn_vec_assign_boundary_{y.tag}")
    C.check(f(y.mesh.handle, y.ncomp, y.comp_ptrs(), x.comp_ptrs() if x is not None else None, float(c), int(cmb),
              int(surface), _stream()), "assign_boundary")


def strong_algebraic_dirichlet_enforcement(A_neumann, A_neumann_diag, g, tmp, b, cmb=True, surface=True):
    """b <- b - A_N g; b <- diag(A_N) g on the Dirichlet layers
    (fe/strong_algebraic_dirichlet_enforcement.hpp:10-45)."""
    apply(A_neumann, g, tmp)
    lincomb(b, [1.0, -1.0], [b, tmp])
    apply(A_neumann_diag, g, tmp)
    assign_boundary(b, tmp, 0.0, cmb, surface)


def freeslip_project(u, cmb=True, surface=True):
    C.check(C.lib().tn_freeslip_project_f64(u.mesh.handle, u.comp_ptrs(), int(cmb), int(surface), _stream()),
            "freeslip_project")


def apply(op, src, dst):
    """linalg::apply (linalg/operator.hpp:156)."""
    op.apply_impl(src, dst)


def lincomb(y, c, xs, c0=0.0):
    y.lincomb_impl(c, xs, c0)


def assign(y, c0):
    y.lincomb_impl([], [], c0)


def dot(a, b):
    return a.dot_impl(b)


# --- the mantle-circulation time step (apps/mantlecirculation/mantlecirculation.cpp:870-1045) ---------------

def fv_to_fe_rhs(mesh, fv, lumped_diagonal=False):
    """b = sum_K fv_K int_K phi_i (fv/hex/conversion.hpp:146-190), and the lumped diagonal if asked; FE scalars."""
    b = VectorQ1Scalar(mesh)
    D = VectorQ1Scalar(mesh) if lumped_diagonal else None
    C.check(C.lib().tn_fv_to_fe_rhs_f64(mesh.handle, ctypes.c_void_p(fv.data_ptr()),
                                        ctypes.c_void_p(b.data.data_ptr()),
                                        ctypes.c_void_p(D.data.data_ptr()) if D is not None else None, _stream()),
            "fv_to_fe_rhs")
    return b, D


def l2_project_fv_to_fe(mesh, fv, dst, lumped=False, max_iterations=1000, relative_tolerance=1e-12,
                        absolute_tolerance=1e-12, work=None):
    """l2_project_fv_to_fe / l2_project_fv_to_fe_lumped (fv/hex/conversion.hpp:131-300): dst (VectorQ1Scalar,
    its values the PCG's start) from the FV tensor fv [10, N+2, N+2, N+2]; returns the PCG iterations."""
    if work is None:
        work = torch.empty(5 * mesh.stored_nodes, dtype=torch.float64, device="cuda")
    its = ctypes.c_int()
    C.check(C.lib().tn_l2_project_fv_to_fe_f64(mesh.handle, ctypes.c_void_p(fv.data_ptr()),
                                               ctypes.c_void_p(dst.data.data_ptr()), int(lumped), max_iterations,
                                               relative_tolerance, absolute_tolerance,
                                               ctypes.c_void_p(work.data_ptr()), ctypes.byref(its), _stream()),
            "l2_project_fv_to_fe")
    return its.value


def stokes_buoyancy_rhs(mesh, T, rayleigh, bc_cmb, bc_surface, f_u, work=None):
    """f_u = VectorMass (Ra T n) with the app's strong Dirichlet / free-slip enforcement
    (mantlecirculation.cpp:117-150, 876-899); T a VectorQ1Scalar on the velocity mesh."""
    if work is None:
        work = torch.empty(3 * mesh.stored_nodes, dtype=torch.float64, device="cuda")
    C.check(C.lib().tn_stokes_buoyancy_rhs_f64(mesh.handle, ctypes.c_void_p(T.data.data_ptr()), float(rayleigh),
                                               bc_cmb, bc_surface, f_u.comp_ptrs(), ctypes.c_void_p(work.data_ptr()),
                                               _stream()), "stokes_buoyancy_rhs")


def pressure_remove_mean(p, work=None):
    """p -= sum_owned p / unique nodes (mantlecirculation.cpp:930-936); returns the subtracted mean."""
    if work is None:
        work = torch.empty(p.mesh.stored_nodes, dtype=torch.float64, device="cuda")
    mean = ctypes.c_double()
    C.check(C.lib().tn_pressure_remove_mean_f64(p.mesh.handle, ctypes.c_void_p(p.data.data_ptr()),
                                                ctypes.c_void_p(work.data_ptr()), ctypes.byref(mean), _stream()),
            "pressure_remove_mean")
    return mean.value


class UnsteadyAdvectionDiffusionSUPG:
    """UnsteadyAdvectionDiffusionSUPG (fe/wedge/operators/shell/unsteady_advection_diffusion_supg.hpp:134): the
    BDF left-hand side mass_scaling M + dt (K + C + G) for the velocity (a VectorQ1Vec of the same precision)."""

    def __init__(self, mesh, velocity, diffusivity, dt, treat_boundary, diagonal=False, mass_scaling=1.0,
                 lumped_mass=False, apply_mode=C.APPLY_REPLACE, comm_mode=C.COMM_ADDITIVE):
        self.mesh, self.velocity = mesh, velocity
        self.diffusivity, self.dt, self.treat, self.diagonal = float(diffusivity), float(dt), treat_boundary, diagonal
        self.mass_scaling, self.lumped = float(mass_scaling), lumped_mass
        self.apply_mode, self.comm_mode = apply_mode, comm_mode

    def set_operator_apply_and_communication_modes(self, apply_mode, comm_mode):
        self.apply_mode, self.comm_mode = apply_mode, comm_mode

    def apply_impl(self, src, dst):
        f = getattr(C.lib(), f"tn_supg_apply_{src.tag}")
        C.check(f(self.mesh.handle, self.velocity.comp_ptrs(), self.diffusivity, self.dt, self.mass_scaling,
                  int(self.lumped), int(self.treat), int(self.diagonal), self.apply_mode, self.comm_mode,
                  ctypes.c_void_p(src.data.data_ptr()), ctypes.c_void_p(dst.data.data_ptr()), _stream()), "supg apply")

    def solve(self, rhs, x, l=2, max_iterations=10, relative_tolerance=1e-12, absolute_tolerance=1e-12, work=None):
        """x <- the solution of this operator x = rhs by PBiCGStab(l) from x (the reference tests' time step,
        tests/test_unsteady_advection_diffusion_supg.cpp:158-172); FP64; returns (iterations, relative residual)"""
        assert self.velocity.data.is_contiguous() and x.dtype == torch.float64
        if work is None:
            work = torch.empty((2 * (l + 1) + 2) * self.mesh.stored_nodes, dtype=torch.float64, device="cuda")
        its, rr = ctypes.c_int(), ctypes.c_double()
        C.check(C.lib().tn_supg_solve_f64(self.mesh.handle, self.velocity.comp_ptrs(), self.diffusivity, self.dt,
                                          self.mass_scaling, int(self.lumped), int(self.treat),
                                          ctypes.c_void_p(rhs.data.data_ptr()), ctypes.c_void_p(x.data.data_ptr()),
                                          l, max_iterations, relative_tolerance, absolute_tolerance,
                                          ctypes.c_void_p(work.data_ptr()), ctypes.byref(its), ctypes.byref(rr),
                                          _stream()), "supg solve")
        return its.value, rr.value


def l2_project_fe_to_fv(mesh, fe, fv):
    """FV cell averages of the FE scalar fe (VectorQ1Scalar) into fv [10, N+2, N+2, N+2], lateral ghost layers
    updated (l2_project_fe_to_fv, fv/hex/conversion.hpp:349-416)."""
    C.check(C.lib().tn_l2_project_fe_to_fv_f64(mesh.handle, ctypes.c_void_p(fe.data.data_ptr()),
                                               ctypes.c_void_p(fv.data_ptr()), _stream()), "l2_project_fe_to_fv")


class XDMFOutput:
    """io::XDMFOutput (io/xdmf.hpp:147-1115): visualisation output and checkpoint in the reference's directory
    format.  add() device grids (VectorQ1Scalar / VectorQ1Vec, FP32 or FP64) before the first write(); write()
    converts them on the current stream and returns while the files are written in the background; wait()
    blocks until they are complete.  points / connectivity: 4 or 8 bytes."""

    FLOAT32, FLOAT64 = 4, 8
    INT32, INT64 = 4, 8

    def __init__(self, directory, mesh, points=4, connectivity=8):
        h = ctypes.c_void_p()
        C.check(C.lib().tn_xdmf_output_create(mesh.handle, str(directory).encode(), points, connectivity,
                                              ctypes.byref(h)), "xdmf_output_create")
        self._h, self.mesh, self.directory, self._keep = h, mesh, str(directory), []

    def set_write_counter(self, counter):
        C.check(C.lib().tn_xdmf_output_set_write_counter(self._h, counter), "set_write_counter")

    def add(self, vec, label, output=4):
        """vec: VectorQ1Scalar or VectorQ1Vec (kept alive by the writer); label: the grid's name in the files"""
        self._keep.append(vec)
        C.check(C.lib().tn_xdmf_output_add(self._h, label.encode(), vec.data.element_size(), vec.ncomp,
                                           vec.comp_ptrs(), output), "xdmf_output_add")

    def write(self):
        C.check(C.lib().tn_xdmf_output_write(self._h, _stream()), "xdmf_output_write")

    def wait(self):
        C.check(C.lib().tn_xdmf_output_wait(self._h), "xdmf_output_wait")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and C is not None and C._lib is not None:
            C.lib().tn_xdmf_output_destroy(h)
            self._h = None


def read_xdmf_checkpoint_metadata(directory):
    """read_xdmf_checkpoint_metadata (io/xdmf.hpp:1162-1268) as a dict; raises C.TNError with the reference's
    error text.  Host only."""
    info = C.CheckpointInfo()
    d = str(directory).encode()
    C.check(C.lib().tn_read_xdmf_checkpoint_metadata(d, ctypes.byref(info), None, 0, None, 0), "checkpoint metadata")
    radii = (ctypes.c_double * max(1, info.num_radii))()
    ids = (ctypes.c_longlong * max(1, info.num_subdomain_ids))()
    C.check(C.lib().tn_read_xdmf_checkpoint_metadata(d, ctypes.byref(info), radii, info.num_radii, ids,
                                                     info.num_subdomain_ids), "checkpoint metadata")
    out = {k: getattr(info, k) for k, _ in C.CheckpointInfo._fields_}
    out["radii"] = list(radii[:info.num_radii])
    out["subdomain_ids"] = list(ids[:info.num_subdomain_ids])
    files = []
    for i in range(info.num_grid_data_files):
        label = ctypes.create_string_buffer(4096)
        t, b, v = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        C.check(C.lib().tn_xdmf_checkpoint_grid_data_file(d, i, label, 4096, ctypes.byref(t), ctypes.byref(b),
                                                          ctypes.byref(v)), "checkpoint grid record")
        files.append({"label": label.value.decode(), "scalar_data_type": t.value, "scalar_bytes": b.value,
                      "vec_dim": v.value})
    out["grid_data_files"] = files
    return out


def read_xdmf_checkpoint_grid(directory, label, step, vec):
    """read_xdmf_checkpoint_grid (io/xdmf.hpp:1270-1500) into vec (VectorQ1Scalar / VectorQ1Vec on the mesh the
    checkpoint was written on); raises C.TNError with the reference's error text."""
    C.check(C.lib().tn_read_xdmf_checkpoint_grid(vec.mesh.handle, str(directory).encode(), label.encode(), step,
                                                 vec.data.element_size(), vec.ncomp, vec.comp_ptrs(), _stream()),
            "read_xdmf_checkpoint_grid")


class MantleTimestep:
    """One time step of the mantle-circulation app on the GPU (mantlecirculation.cpp:870-1045), in its order:
    the Stokes right-hand side from the FE temperature (buoyancy Ra T n, VectorMass, strong enforcement), the
    Stokes solve warm-started from the previous velocity and pressure, the pressure normalisation, dt =
    dt_scaling x compute_dt_stable, `energy_substeps` FCT explicit steps with the Dirichlet temperatures
    applied after each, the FV -> FE L2 projection of the temperature (warm-started from the previous FE
    temperature), and the NaN / Inf guard on it (the app stops its run there; step() returns False).

    T_fv: FV temperature [10, N+2, N+2, N+2] (with ghosts); the FE temperature is projected from it at set-up.
    solver_kwargs: shell.StokesSolver arguments (the app's: FGMRES(restart), block-triangular preconditioner,
    V-cycle).  Every array stays on the device."""

    def __init__(self, level, viscosity, T_fv, rayleigh=1e5, dt_scaling=0.5, diffusivity=0.0, energy_substeps=1,
                 T_cmb=1.0, T_surface=0.0, bc_cmb=C.BC_FREESLIP, bc_surface=C.BC_FREESLIP, lumped_projection=False,
                 r_min=0.55, r_max=1.0, **solver_kwargs):
        self.mesh_u = ShellMesh(level, r_min, r_max)
        self.mesh_p = ShellMesh(level - 1, r_min, r_max)
        self.rayleigh, self.dt_scaling, self.kappa = rayleigh, dt_scaling, diffusivity
        self.substeps, self.bcs = energy_substeps, (bc_cmb, bc_surface)
        self.lumped = lumped_projection
        self.viscosity = viscosity
        self.solver = StokesSolver(level, viscosity, bc_cmb=bc_cmb, bc_surface=bc_surface, r_min=r_min, r_max=r_max,
                                   **solver_kwargs)
        self.fct = FCTAdvectionDiffusion(self.mesh_u)
        self.fct_bcs = self.fct.dirichlet(T_cmb, T_surface)
        self.T_fv = T_fv
        self.T = VectorQ1Scalar(self.mesh_u)
        self.u, self.p = VectorQ1Vec(self.mesh_u), VectorQ1Scalar(self.mesh_p)
        self.f_u, self.f_p = VectorQ1Vec(self.mesh_u), VectorQ1Scalar(self.mesh_p)
        ns = self.mesh_u.stored_nodes
        self._work = torch.empty(5 * ns, dtype=torch.float64, device="cuda")
        self._pwork = torch.empty(self.mesh_p.stored_nodes, dtype=torch.float64, device="cuda")
        self.fct.apply_dirichlet(self.T_fv, self.fct_bcs)
        self.project_temperature()
        self.last = {}

    def project_temperature(self):
        return l2_project_fv_to_fe(self.mesh_u, self.T_fv, self.T, self.lumped, work=self._work)

    def step(self):
        """One time step; False when the temperature holds NaN or Inf afterwards (the app's guard, :1041)."""
        stokes_buoyancy_rhs(self.mesh_u, self.T, self.rayleigh, *self.bcs, self.f_u, work=self._work)
        its, rr = self.solver.solve(self.f_u, self.f_p, self.u, self.p)
        mean = pressure_remove_mean(self.p, work=self._pwork)
        dt = self.dt_scaling * self.fct.dt_stable(self.u, self.kappa)
        for _ in range(self.substeps):
            self.fct.step(self.T_fv, self.u, dt, self.kappa, None, True, self.fct_bcs)
            self.fct.apply_dirichlet(self.T_fv, self.fct_bcs)
        pits = self.project_temperature()
        ok = not self.T.has_nan_or_inf_impl()
        self.last = {"stokes_iterations": its, "stokes_relres": rr, "pressure_mean_removed": mean, "dt": dt,
                     "projection_iterations": pits, "finite": ok}
        return ok

    def checkpoint_output(self, directory, points=4, connectivity=8, output=4):
        """The app's XDMF output (mantlecirculation.cpp:789-799): T, the velocity as "u_u" and the viscosity
        "eta", written as `output`-byte floats; call write() on it after set-up and after each output step."""
        x = XDMFOutput(directory, self.mesh_u, points, connectivity)
        x.add(self.T, "T", output)
        x.add(self.u, "u_u", output)
        x.add(self.viscosity, "eta", output)
        return x

    def restore_checkpoint(self, directory, step):
        """The app's checkpoint recovery (mantlecirculation.cpp:803-846): the velocity and the FE temperature
        of `step`, the FV temperature recovered from the FE one (l2_project_fe_to_fv); the pressure restarts
        from zero, as in the app."""
        read_xdmf_checkpoint_grid(directory, "u_u", step, self.u)
        read_xdmf_checkpoint_grid(directory, "T", step, self.T)
        l2_project_fe_to_fv(self.mesh_u, self.T, self.T_fv)
        self.p.data.zero_()
