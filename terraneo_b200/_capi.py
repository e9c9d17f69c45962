"""ctypes binding of libterraneo_b200.so, the C ABI declared in include/terraneo_b200.h.

The library is the product: every operator, vector kernel and solver call below
runs CUDA code from it.  There is no CPU fallback; importing this module without
the built library raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libterraneo_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "terraneo_b200.h")

TN_OK = 0
BC_NEUMANN, BC_DIRICHLET, BC_FREESLIP = 0, 1, 2
APPLY_REPLACE, APPLY_ADD = 0, 1
COMM_SKIP, COMM_ADDITIVE = 0, 1

c_int, c_double, c_size_t, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p
P = ctypes.POINTER


class EpsDivDivParams(ctypes.Structure):
    _fields_ = [("bc_cmb", c_int), ("bc_surface", c_int), ("diagonal", c_int), ("apply_mode", c_int),
                ("comm_mode", c_int), ("penalty_eps", c_double)]


class StokesParams(ctypes.Structure):
    _fields_ = [("level", c_int), ("mg_levels", c_int), ("bc_cmb", c_int), ("bc_surface", c_int), ("mg_fp32", c_int),
                ("chebyshev_order", c_int), ("smoothing_steps", c_int), ("power_iterations", c_int),
                ("vcycles", c_int), ("coarse_max_iterations", c_int), ("coarse_relative_tolerance", c_double),
                ("restart", c_int), ("max_iterations", c_int), ("relative_tolerance", c_double),
                ("absolute_tolerance", c_double), ("gca", c_int), ("outer", c_int), ("eager", c_int),
                ("chebyshev_estimates", P(c_double))]


class ScalarMGParams(ctypes.Structure):
    _fields_ = [("level", c_int), ("mg_levels", c_int), ("smoother", c_int), ("smoothing_steps", c_int),
                ("chebyshev_order", c_int), ("power_iterations", c_int), ("jacobi_omega", c_double),
                ("vcycles", c_int), ("coarse_max_iterations", c_int), ("coarse_relative_tolerance", c_double),
                ("max_iterations", c_int), ("relative_tolerance", c_double), ("absolute_tolerance", c_double),
                ("krylov", c_int)]


class FCTDirichlet(ctypes.Structure):
    _fields_ = [("T_cmb", c_double), ("T_surface", c_double), ("apply_cmb", c_int), ("apply_surface", c_int)]


class CheckpointInfo(ctypes.Structure):
    _fields_ = [(n, c_int) for n in ("version", "subdomains_lateral", "subdomains_radial", "size_x", "size_y", "size_r",
                                     "grid_scalar_bytes", "num_grid_data_files", "ordering", "num_radii",
                                     "num_subdomain_ids")]


class TNError(RuntimeError):
    pass


_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "tn_last_error": (ctypes.c_char_p, []),
    "tn_mesh_create": (c_int, [c_int, c_double, c_double, P(c_void_p)]),
    "tn_mesh_destroy": (c_int, [c_void_p]),
    "tn_mesh_dims": (c_int, [c_void_p, P(c_int), P(c_size_t), P(c_size_t)]),
    "tn_mesh_geometry": (c_int, [c_void_p, c_void_p, c_void_p]),
    "tn_mesh_masks": (c_int, [c_void_p, c_void_p, c_void_p]),
    "tn_halo_sum_f64": (c_int, [c_void_p, P(c_void_p), c_int, c_void_p]),
    "tn_halo_sum_f32": (c_int, [c_void_p, P(c_void_p), c_int, c_void_p]),
    "tn_epsdivdiv_apply_f64": (c_int, [c_void_p, P(EpsDivDivParams), c_void_p, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_epsdivdiv_apply_f32": (c_int, [c_void_p, P(EpsDivDivParams), c_void_p, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_laplace_apply_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "tn_laplace_apply_f32": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "tn_divergence_apply_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, P(c_void_p), c_void_p, c_void_p]),
    "tn_divergence_apply_f32": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, P(c_void_p), c_void_p, c_void_p]),
    "tn_gradient_apply_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p, P(c_void_p), c_void_p]),
    "tn_gradient_apply_f32": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p, P(c_void_p), c_void_p]),
    "tn_prolongation_constant_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_prolongation_constant_f32": (c_int, [c_void_p, c_void_p, c_int, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_restriction_constant_f64": (c_int, [c_void_p, c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_restriction_constant_f32": (c_int, [c_void_p, c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_kmass_apply_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "tn_kmass_apply_f32": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "tn_injection_f64": (c_int, [c_void_p, c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_freeslip_project_f64": (c_int, [c_void_p, P(c_void_p), c_int, c_int, c_void_p]),
    "tn_krylov_axpy_dot_f64": (c_int, [c_int, P(c_void_p), P(c_void_p), P(c_void_p), c_void_p, P(c_void_p), c_void_p,
                                       c_void_p, c_void_p]),
    "tn_krylov_axpy_dot_f32": (c_int, [c_int, P(c_void_p), P(c_void_p), P(c_void_p), c_void_p, P(c_void_p), c_void_p,
                                       c_void_p, c_void_p]),
    "tn_pcg_begin_f64": (c_int, [c_int, P(c_void_p), P(c_void_p), P(c_void_p), c_void_p, c_double, c_void_p]),
    "tn_pcg_pap_f64": (c_int, [c_int, P(c_void_p), P(c_void_p), P(c_void_p), c_void_p, c_void_p]),
    "tn_pcg_update_f64": (c_int, [c_int, P(c_void_p), P(c_void_p), P(c_void_p), P(c_void_p), P(c_void_p), c_void_p,
                                  c_int, c_double, c_double, c_void_p]),
    "tn_pcg_direction_f64": (c_int, [c_int, P(c_void_p), P(c_void_p), P(c_void_p), c_void_p, c_void_p]),
    "tn_divkgrad_apply_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                      c_void_p]),
    "tn_divkgrad_apply_f32": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                      c_void_p]),
    "tn_vector_laplace_apply_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, P(c_void_p), P(c_void_p),
                                            c_void_p]),
    "tn_vector_laplace_apply_f32": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, P(c_void_p), P(c_void_p),
                                            c_void_p]),
    "tn_epsdivdiv_kgrad_f64": (c_int, [c_void_p, c_int, c_int, c_int, P(c_void_p), P(c_void_p), c_void_p, c_void_p]),
    "tn_epsdivdiv_kgrad_f32": (c_int, [c_void_p, c_int, c_int, c_int, P(c_void_p), P(c_void_p), c_void_p, c_void_p]),
    "tn_stokes_viscosity_backward": (c_int, [c_void_p, P(c_void_p), P(c_void_p), c_int, c_void_p, P(c_void_p),
                                             c_void_p, P(c_int)]),
    "tn_prolongation_linear_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_prolongation_linear_f32": (c_int, [c_void_p, c_void_p, c_int, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_restriction_linear_f64": (c_int, [c_void_p, c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_restriction_linear_f32": (c_int, [c_void_p, c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_divkgrad_mg_pcg_solve_f64": (c_int, [P(ScalarMGParams), c_double, c_double, c_void_p, c_void_p, c_void_p,
                                             P(c_int), P(c_double)]),
    "tn_local_matrix_count": (c_int, [c_void_p, P(c_size_t)]),
    "tn_kerngen_local_matrices_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "tn_gca_coarsen_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "tn_gca_elements_f64": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "tn_agca_unmarked_local_matrices_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "tn_stored_epsdivdiv_apply_f64": (c_int, [c_void_p, c_void_p, P(EpsDivDivParams), P(c_void_p), P(c_void_p),
                                              c_void_p]),
    "tn_stored_epsdivdiv_apply_f32": (c_int, [c_void_p, c_void_p, P(EpsDivDivParams), P(c_void_p), P(c_void_p),
                                              c_void_p]),
    "tn_array_cast_f64_to_f32": (c_int, [c_size_t, c_void_p, c_void_p, c_void_p]),
    "tn_fv_field_size": (c_int, [c_void_p, P(c_size_t)]),
    "tn_fct_workspace_size": (c_int, [c_void_p, P(c_size_t)]),
    "tn_fv_ghost_update_f64": (c_int, [c_void_p, c_void_p, c_void_p]),
    "tn_fv_cell_centers_f64": (c_int, [c_void_p, P(c_void_p), c_void_p]),
    "tn_fct_dt_stable_f64": (c_int, [c_void_p, P(c_void_p), P(c_void_p), c_double, P(c_double), c_void_p]),
    "tn_fct_apply_dirichlet_f64": (c_int, [c_void_p, c_void_p, P(FCTDirichlet), c_void_p]),
    "tn_fct_step_f64": (c_int, [c_void_p, c_void_p, P(c_void_p), P(c_void_p), c_double, c_double, c_void_p, c_int,
                                P(FCTDirichlet), c_void_p, c_void_p]),
    "tn_epsdivdiv3x2_apply_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, P(c_void_p), P(c_void_p),
                                          c_void_p]),
    "tn_epsdivdiv3x2_apply_f32": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, P(c_void_p), P(c_void_p),
                                          c_void_p]),
    "tn_laplace_krylov_solve_f64": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_double,
                                             c_double, P(c_int), c_void_p, c_int, P(c_int)]),
    "tn_laplace_pcg_solve_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_double, c_double, P(c_int),
                                         P(c_double)]),
    "tn_stokes_solver_create": (c_int, [P(StokesParams), c_double, c_double, c_void_p, P(c_void_p)]),
    "tn_stokes_solve": (c_int, [c_void_p, P(c_void_p), c_void_p, P(c_void_p), c_void_p, P(c_int), P(c_double)]),
    "tn_stokes_history": (c_int, [c_void_p, P(c_double), c_int, P(c_int), P(c_int)]),
    "tn_stokes_apply": (c_int, [c_void_p, P(c_void_p), c_void_p, P(c_void_p), c_void_p]),
    "tn_stokes_solver_destroy": (c_int, [c_void_p]),
    "tn_fv_to_fe_rhs_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "tn_l2_project_fv_to_fe_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_double, c_double, c_void_p,
                                           P(c_int), c_void_p]),
    "tn_stokes_buoyancy_rhs_f64": (c_int, [c_void_p, c_void_p, c_double, c_int, c_int, P(c_void_p), c_void_p,
                                           c_void_p]),
    "tn_pressure_remove_mean_f64": (c_int, [c_void_p, c_void_p, c_void_p, P(c_double), c_void_p]),
    "tn_l2_project_fe_to_fv_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "tn_supg_apply_f64": (c_int, [c_void_p, P(c_void_p), c_double, c_double, c_double, c_int, c_int, c_int, c_int,
                                  c_int, c_void_p, c_void_p, c_void_p]),
    "tn_supg_apply_f32": (c_int, [c_void_p, P(c_void_p), c_double, c_double, c_double, c_int, c_int, c_int, c_int,
                                  c_int, c_void_p, c_void_p, c_void_p]),
    "tn_supg_solve_f64": (c_int, [c_void_p, P(c_void_p), c_double, c_double, c_double, c_int, c_int, c_void_p, c_void_p,
                                  c_int, c_int, c_double, c_double, c_void_p, P(c_int), P(c_double), c_void_p]),
    "tn_xdmf_output_create": (c_int, [c_void_p, ctypes.c_char_p, c_int, c_int, P(c_void_p)]),
    "tn_xdmf_output_set_write_counter": (c_int, [c_void_p, c_int]),
    "tn_xdmf_output_add": (c_int, [c_void_p, ctypes.c_char_p, c_int, c_int, P(c_void_p), c_int]),
    "tn_xdmf_output_write": (c_int, [c_void_p, c_void_p]),
    "tn_xdmf_output_wait": (c_int, [c_void_p]),
    "tn_xdmf_output_destroy": (c_int, [c_void_p]),
    "tn_read_xdmf_checkpoint_metadata": (c_int, [ctypes.c_char_p, P(CheckpointInfo), P(c_double), c_int,
                                                 P(ctypes.c_longlong), c_int]),
    "tn_xdmf_checkpoint_grid_data_file": (c_int, [ctypes.c_char_p, c_int, ctypes.c_char_p, c_int, P(c_int), P(c_int),
                                                  P(c_int)]),
    "tn_read_xdmf_checkpoint_grid": (c_int, [c_void_p, ctypes.c_char_p, ctypes.c_char_p, c_int, c_int, c_int,
                                             P(c_void_p), c_void_p]),
    "tn_vec_lincomb_f64": (c_int, [c_void_p, c_int, P(c_void_p), c_double, c_int, P(c_double), P(c_void_p), c_void_p]),
    "tn_vec_lincomb_f32": (c_int, [c_void_p, c_int, P(c_void_p), c_double, c_int, P(c_double), P(c_void_p), c_void_p]),
    "tn_vec_sum_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_double), c_void_p]),
    "tn_vec_sum_f32": (c_int, [c_void_p, c_int, P(c_void_p), P(c_double), c_void_p]),
    "tn_vec_dot_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), P(c_double), c_void_p]),
    "tn_vec_dot_f32": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), P(c_double), c_void_p]),
    "tn_vec_invert_f64": (c_int, [c_void_p, c_int, P(c_void_p), c_void_p]),
    "tn_vec_invert_f32": (c_int, [c_void_p, c_int, P(c_void_p), c_void_p]),
    "tn_vec_mult_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_vec_mult_f32": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_vec_max_abs_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_double), c_void_p]),
    "tn_vec_max_abs_f32": (c_int, [c_void_p, c_int, P(c_void_p), P(c_double), c_void_p]),
    "tn_vec_has_nan_or_inf_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_int), c_void_p]),
    "tn_vec_has_nan_or_inf_f32": (c_int, [c_void_p, c_int, P(c_void_p), P(c_int), c_void_p]),
    "tn_vec_dot_noalloc_f64": (c_int, [c_size_t, c_int, P(c_void_p), P(c_void_p), c_void_p, P(c_double), c_void_p]),
    "tn_stored_pcg_f64": (c_int, [c_void_p, c_void_p, c_void_p, P(c_void_p), P(c_void_p), P(c_void_p), c_void_p,
                                  c_int, c_double, c_double, c_int, c_void_p]),
    "tn_vec_assign_boundary_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), c_double, c_int, c_int,
                                           c_void_p]),
    "tn_vec_assign_boundary_f32": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), c_double, c_int, c_int,
                                           c_void_p]),
    "tn_vec_chebyshev_step_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), P(c_void_p), P(c_void_p),
                                          P(c_void_p), c_double, c_double, c_void_p]),
    "tn_vec_chebyshev_step_f32": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), P(c_void_p), P(c_void_p),
                                          P(c_void_p), c_double, c_double, c_void_p]),
    "tn_vec_randomize_f64": (c_int, [c_void_p, c_int, P(c_void_p), ctypes.c_ulonglong, c_void_p]),
    "tn_vec_randomize_f32": (c_int, [c_void_p, c_int, P(c_void_p), ctypes.c_ulonglong, c_void_p]),
    "tn_vec_cast_f64_to_f32": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_vec_cast_f32_to_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_shell_partition": (c_int, [c_int, c_int, P(c_int), P(c_int)]),
    "tn_shard_halo_plan": (c_int, [c_int, c_int, c_int, c_int, P(c_int), P(c_int), c_void_p, c_void_p]),
    "tn_shard_create": (c_int, [c_int, c_double, c_double, c_int, c_int, P(c_void_p)]),
    "tn_shard_destroy": (c_int, [c_void_p]),
    "tn_shard_dims": (c_int, [c_void_p, P(c_int), P(c_int), P(c_size_t), P(c_size_t), P(c_size_t)]),
    "tn_shard_geometry": (c_int, [c_void_p, c_void_p, c_void_p]),
    "tn_shard_masks": (c_int, [c_void_p, c_void_p, c_void_p]),
    "tn_shard_epsdivdiv_apply_f64": (c_int, [c_void_p, P(EpsDivDivParams), c_void_p, P(c_void_p), P(c_void_p),
                                             c_void_p]),
    "tn_shard_epsdivdiv_apply_f32": (c_int, [c_void_p, P(EpsDivDivParams), c_void_p, P(c_void_p), P(c_void_p),
                                             c_void_p]),
    "tn_shard_penalty_dots_f64": (c_int, [c_void_p, P(c_void_p), c_void_p, c_void_p]),
    "tn_shard_penalty_dots_f32": (c_int, [c_void_p, P(c_void_p), c_void_p, c_void_p]),
    "tn_shard_epsdivdiv_apply_fsfs_f64": (c_int, [c_void_p, P(EpsDivDivParams), c_void_p, P(c_void_p), P(c_void_p),
                                                  c_void_p, c_void_p]),
    "tn_shard_epsdivdiv_apply_fsfs_f32": (c_int, [c_void_p, P(EpsDivDivParams), c_void_p, P(c_void_p), P(c_void_p),
                                                  c_void_p, c_void_p]),
    "tn_shard_pack_f64": (c_int, [c_void_p, P(c_void_p), c_int, c_void_p, c_void_p]),
    "tn_shard_pack_f32": (c_int, [c_void_p, P(c_void_p), c_int, c_void_p, c_void_p]),
    "tn_shard_unpack_f64": (c_int, [c_void_p, c_void_p, P(c_void_p), c_int, c_void_p]),
    "tn_shard_unpack_f32": (c_int, [c_void_p, c_void_p, P(c_void_p), c_int, c_void_p]),
    "tn_shard_vec_dot_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), P(c_double), c_void_p]),
    "tn_shard_vec_lincomb_f64": (c_int, [c_void_p, c_int, P(c_void_p), c_double, c_int, P(c_double), P(c_void_p),
                                         c_void_p]),
    "tn_shard_prolongation_constant_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, P(c_void_p), P(c_void_p),
                                                   c_void_p]),
    "tn_shard_restriction_constant_f64": (c_int, [c_void_p, c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_shard_injection_f64": (c_int, [c_void_p, c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_shard_vec_invert_f64": (c_int, [c_void_p, c_int, P(c_void_p), c_void_p]),
    "tn_shard_vec_mult_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), c_void_p]),
    "tn_shard_vec_chebyshev_step_f64": (c_int, [c_void_p, c_int, P(c_void_p), P(c_void_p), P(c_void_p), P(c_void_p),
                                                P(c_void_p), c_double, c_double, c_void_p]),
}


def lib():
    """Load the CUDA library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"terraneo_b200: {LIB_PATH} is missing; build it with "
                              "`make -C terraneo_b200/csrc` or __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def check(rc, what=""):
    if rc != TN_OK:
        msg = lib().tn_last_error().decode()
        raise TNError(f"{what}: status {rc}: {msg}")


def ptrs(*addrs):
    """A C array of device pointers (void*[n])."""
    arr = (c_void_p * max(3, len(addrs)))()
    for i, a in enumerate(addrs):
        arr[i] = a
    return arr
