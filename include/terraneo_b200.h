/* terraneo_b200: C ABI of the B200 (sm_100a) matrix-free hot path of TerraNeo.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns
 * an int status (0 = success, negative = error, see TN_ERR_*) and never throws.
 * Device pointers are CUDA global-memory pointers of the current device;
 * `stream` is a cudaStream_t (NULL = legacy default stream).  Apply and vector
 * kernels are asynchronous on `stream`; functions that return a host scalar
 * (dot products, norms) synchronise that stream before returning, which keeps
 * the reference's synchronous semantics at every apply_impl / dot_impl.
 *
 * Data layout is the reference's own (src/terra/grid/grid_types.hpp:12-57):
 * a scalar field is [10][N+1][N+1][N+1] (diamond, x, y, r), r fastest; a vector
 * field is three such scalar fields passed as three pointers (the reference's
 * Grid4DDataVec holds three separate scalar views).  N = 2^level, one
 * subdomain per diamond, all ten diamonds on one GPU.
 *
 * Boundary-condition codes follow grid/shell/bit_masks.hpp:24:
 * 0 = NEUMANN, 1 = DIRICHLET, 2 = FREESLIP. */
#ifndef TERRANEO_B200_H
#define TERRANEO_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined( __GNUC__ )
#define TN_API __attribute__( ( visibility( "default" ) ) )
#else
#define TN_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define TN_OK 0
#define TN_ERR_ARG -1      /* invalid argument (sizes, codes, null pointers) */
#define TN_ERR_CUDA -2     /* a CUDA runtime call failed */
#define TN_ERR_NOMEM -3    /* device or host allocation failed */
#define TN_ERR_STATE -4    /* object not set up for this call */
#define TN_ERR_IO -5       /* a file could not be read or written, or its content is not as expected */

#define TN_BC_NEUMANN 0
#define TN_BC_DIRICHLET 1
#define TN_BC_FREESLIP 2

/* OperatorApplyMode / OperatorCommunicationMode (linalg/operator.hpp:29-44) */
#define TN_APPLY_REPLACE 0
#define TN_APPLY_ADD 1
#define TN_COMM_SKIP 0
#define TN_COMM_ADDITIVE 1

typedef struct tn_mesh tn_mesh;

/* Last error message of the calling thread (never NULL). */
TN_API const char* tn_last_error( void );

/* ---------------------------------------------------------------------------
 * Shell mesh: geometry, masks and the duplicated-node (halo) map.
 * Replaces DistributedDomain::create_uniform_single_subdomain_per_diamond
 * (grid/shell/spherical_shell.hpp:2520), subdomain_unit_sphere_single_shell_coords
 * (:2724), subdomain_shell_radii (:2759), setup_node_ownership_mask_data
 * (grid/bit_masks.hpp:29) and setup_boundary_mask_data (grid/shell/bit_masks.hpp:82).
 * `level` refines laterally and radially alike (N = 2^level cells per side). */
TN_API int tn_mesh_create( int level, double r_min, double r_max, tn_mesh** out );
TN_API int tn_mesh_destroy( tn_mesh* mesh );
/* stored nodes = 10 (N+1)^3, unique nodes = (10 N^2 + 2)(N+1) */
TN_API int tn_mesh_dims( const tn_mesh* mesh, int* level, size_t* stored_nodes, size_t* unique_nodes );
/* host copies: coords [10][N+1][N+1][3], radii [10][N+1] (either may be NULL) */
TN_API int tn_mesh_geometry( const tn_mesh* mesh, double* coords, double* radii );
/* host copies of the boundary flags (1 INNER, 6 CMB, 10 SURFACE) and the
 * ownership flags (1 OWNED), both [10][N+1][N+1][N+1] (either may be NULL) */
TN_API int tn_mesh_masks( const tn_mesh* mesh, uint8_t* boundary_mask, uint8_t* ownership_mask );

/* Additive inter-diamond halo: every copy of a duplicated node becomes the sum
 * of all copies.  Replaces send_recv_with_plan / pack_send_and_recv +
 * unpack_and_reduce_local_subdomain_boundaries (communication/shell/
 * communication.hpp:242-747, communication_plan.hpp:48-68) for one GPU. */
TN_API int tn_halo_sum_f64( const tn_mesh* mesh, double* const* fields, int nfields, void* stream );
TN_API int tn_halo_sum_f32( const tn_mesh* mesh, float* const* fields, int nfields, void* stream );

/* ---------------------------------------------------------------------------
 * EpsilonDivDivKerngen::apply_impl (fe/wedge/operators/shell/epsilon_divdiv_kerngen.hpp:513)
 * a(u,v) = int k (2 eps(u):eps(v) - 2/3 div u div v), one-point quadrature;
 * Dirichlet / Neumann / free-slip at CMB and SURFACE; `diagonal` != 0 gives the
 * diagonal-only action; with free-slip on both boundaries the rigid-rotation
 * penalty dst += eps_p sum_i (m_i^T src) m_i is added (eps_p = penalty_eps,
 * the reference default is 1, :138).  `k` is the nodal coefficient field. */
typedef struct
{
    int    bc_cmb;
    int    bc_surface;
    int    diagonal;
    int    apply_mode; /* TN_APPLY_* */
    int    comm_mode;  /* TN_COMM_* */
    double penalty_eps;
} tn_epsdivdiv_params;

TN_API int tn_epsdivdiv_apply_f64( const tn_mesh* mesh, const tn_epsdivdiv_params* p, const double* k,
                            const double* const* src, double* const* dst, void* stream );
TN_API int tn_epsdivdiv_apply_f32( const tn_mesh* mesh, const tn_epsdivdiv_params* p, const float* k,
                            const float* const* src, float* const* dst, void* stream );

/* ---------------------------------------------------------------------------
 * Stored local matrices and GCA coarse operators of the epsilon-div-div
 * operator (OperatorStoredMatrixMode::Full, linalg/operator.hpp:46; the
 * kerngen slow path epsilon_divdiv_kerngen.hpp:823-1052; TwoGridGCA
 * linalg/solvers/gca/gca.hpp:42-528; LocalMatrixStorage
 * linalg/solvers/gca/local_matrix_storage.hpp:29-243).
 *
 * Storage: DIMENSIONWISE local order (local node + 6 * dimension).  The
 * matrices are symmetric and only the upper triangle is stored, row by row:
 * entry (I, J), I <= J, is entry e = 18 I - I (I - 1) / 2 + J - I of 171,
 * followed by one zero padding entry (172 per wedge).  Wedges are numbered
 * w = 2 cell + wedge with cells (diamond, x, y, r), r fastest, and 32
 * consecutive wedges are interleaved in chunks of 4 entries: entry e of
 * wedge w lives at (((w / 32) * 43 + e / 4) * 32 + w % 32) * 4 + e % 4.
 * tn_local_matrix_count gives the number of entries (2 * 10 N^3 wedges padded
 * to a multiple of 32, times 172; FP64 about 2,752 bytes per cell, the
 * reference stores the full 5,184). */
TN_API int tn_local_matrix_count( const tn_mesh* mesh, size_t* entries );
/* Unpreconditioned PCG (linalg/solvers/pcg.hpp:78-102, z = r) on the
 * stored-matrix operator of tn_stored_epsdivdiv_apply_f64 (non-diagonal,
 * Replace, additive halo; the Dirichlet / free-slip treatment and the fs/fs
 * penalty as there) with the operator's steps fused into the PCG steps: four
 * launches per iteration (direction + clearing + penalty dots, wedge
 * products, halo sum + penalty + <p, Ap>, tn_pcg_update_f64).  The same
 * recurrences, owned-node dot products, stopping rule (|r| / |r0| <=
 * relative_tolerance or |r| < absolute_tolerance, at most max_iterations)
 * and state layout as the tn_pcg_* steps; every launch after the first
 * three is gated by the stopping flag.  x: initial guess in, solution out.
 * work: 12 fields (r, p, two operator results; 3 components each).  state:
 * >= 9 + max_iterations doubles.  check_every > 0: outside stream capture the
 * host reads the stopping flag every check_every iterations and stops
 * launching (synchronises); 0: never (fully asynchronous). */
TN_API int tn_stored_pcg_f64( const tn_mesh* mesh, const double* mats, const tn_epsdivdiv_params* p,
                              const double* const* b, double* const* x, double* const* work, double* state,
                              int max_iterations, double relative_tolerance, double absolute_tolerance,
                              int check_every, void* stream );
/* kerngen assemble_local_matrix (:2051-2110) of every wedge: one-point rule,
 * nodal coefficient k (NULL: k = 1), no boundary treatment. */
TN_API int tn_kerngen_local_matrices_f64( const tn_mesh* mesh, const double* k, double* mats, void* stream );
/* TwoGridGCA: mats_coarse = per coarse cell sum of P^T A_fine P over its
 * 8 fine hexes x 2 wedges; A_fine from the kerngen matrices of k_fine (the
 * finest level, Neumann operator) or from stored matrices mats_fine (exactly
 * one of the two non-NULL); mode 0 constant (the reference default),
 * 1 linear interpolation weights. */
TN_API int tn_gca_coarsen_f64( const tn_mesh* fine, const tn_mesh* coarse, const double* k_fine,
                               const double* mats_fine, int mode, double* mats_coarse, void* stream );
/* GCAElementsCollector (linalg/solvers/gca/gca_elements_collector.hpp:19-96): marks (one byte per cell of the
 * coarsest grid, [10][N0][N0][N0], N0 = N >> level_range, zeroed here) the coarsest cell (x, y, r) >> level_range
 * of every cell of `fine` with a wedge whose nodal k has a reference-coordinate gradient of norm > 10 at the
 * centroid.  The adaptive GCA (mantlecirculation.cpp:379-387 with gca == 2) builds Galerkin coarse matrices
 * only below marked cells. */
TN_API int tn_gca_elements_f64( const tn_mesh* fine, const double* k_fine, int level_range, uint8_t* marks,
                                void* stream );
/* The elements the adaptive GCA leaves unmarked (LocalMatrixStorage::Selective, local_matrix_storage.hpp:185-216:
 * assembled on the fly from the level's own coefficient): overwrites, in the stored-matrix table `mats` of
 * `mesh`, the matrices of the cells whose coarsest ancestor (>> level_range) is not marked with the kerngen
 * matrices of k (NULL: k = 1); marked cells keep their (GCA) matrices. */
TN_API int tn_agca_unmarked_local_matrices_f64( const tn_mesh* mesh, const double* k, const uint8_t* marks,
                                                int level_range, double* mats, void* stream );
/* Apply with stored matrices: the slow path's boundary treatment (Dirichlet
 * masks, free-slip rotation with the normal component decoupled), diagonal
 * mode, the fs/fs rotation penalty (p->penalty_eps) and apply / communication
 * modes as tn_epsdivdiv_apply_*. */
TN_API int tn_stored_epsdivdiv_apply_f64( const tn_mesh* mesh, const double* mats, const tn_epsdivdiv_params* p,
                                          const double* const* src, double* const* dst, void* stream );
TN_API int tn_stored_epsdivdiv_apply_f32( const tn_mesh* mesh, const float* mats, const tn_epsdivdiv_params* p,
                                          const float* const* src, float* const* dst, void* stream );
/* dst[i] = (float) src[i], i < n (FP32 copies of stored matrices) */
TN_API int tn_array_cast_f64_to_f32( size_t n, const double* src, float* dst, void* stream );

/* EpsilonDivDiv::apply_impl (fe/wedge/operators/shell/epsilon_divdiv.hpp:218-600):
 * the same form as the kerngen operator with the 3x2 Felippa rule and k
 * interpolated by the shape functions at each quadrature point;
 * treat_boundary eliminates the CMB nodes of layer 0 (else the SURFACE nodes
 * of layer N-1) keeping their diagonal; diagonal != 0 keeps the diagonal only. */
TN_API int tn_epsdivdiv3x2_apply_f64( const tn_mesh* mesh, const double* k, int treat_boundary, int diagonal,
                                      int apply_mode, int comm_mode, const double* const* src, double* const* dst,
                                      void* stream );
TN_API int tn_epsdivdiv3x2_apply_f32( const tn_mesh* mesh, const float* k, int treat_boundary, int diagonal,
                                      int apply_mode, int comm_mode, const float* const* src, float* const* dst,
                                      void* stream );

/* ---------------------------------------------------------------------------
 * Laplace::apply_impl (fe/wedge/operators/shell/laplace.hpp:68): int grad u . grad v,
 * 3x2 Felippa quadrature; treat_boundary != 0 eliminates the CMB/SURFACE
 * Dirichlet rows and columns keeping the diagonal; diagonal != 0 gives the
 * diagonal-only action. */
TN_API int tn_laplace_apply_f64( const tn_mesh* mesh, int treat_boundary, int diagonal, int apply_mode, int comm_mode,
                          const double* src, double* dst, void* stream );
TN_API int tn_laplace_apply_f32( const tn_mesh* mesh, int treat_boundary, int diagonal, int apply_mode, int comm_mode,
                          const float* src, float* dst, void* stream );

/* DivKGrad::apply_impl (fe/wedge/operators/shell/div_k_grad.hpp:219-345):
 * int k grad u . grad v with k (nodal field) interpolated by the wedge shape
 * functions at each quadrature point; treat_boundary / diagonal as for the
 * Laplace; single_quadpoint != 0 uses the 1-point rule (set_single_quadpoint). */
TN_API int tn_divkgrad_apply_f64( const tn_mesh* mesh, const double* k, int treat_boundary, int diagonal,
                                  int single_quadpoint, int apply_mode, int comm_mode, const double* src, double* dst,
                                  void* stream );
TN_API int tn_divkgrad_apply_f32( const tn_mesh* mesh, const float* k, int treat_boundary, int diagonal,
                                  int single_quadpoint, int apply_mode, int comm_mode, const float* src, float* dst,
                                  void* stream );

/* VectorLaplace::apply_impl (fe/wedge/operators/shell/vector_laplace.hpp:131-255):
 * the Laplace on each of three components, 3x2 rule.  Boundary handling as
 * the reference selects it per cell from the flag of the cell's (x, y, r)
 * node: layer 0 follows bc_cmb, every other layer bc_surface (Dirichlet
 * decouples that side's nodes keeping their diagonal).  Only TN_BC_NEUMANN
 * and TN_BC_DIRICHLET are accepted (the reference aborts otherwise). */
TN_API int tn_vector_laplace_apply_f64( const tn_mesh* mesh, int bc_cmb, int bc_surface, int diagonal, int apply_mode,
                                        int comm_mode, const double* const* src, double* const* dst, void* stream );
TN_API int tn_vector_laplace_apply_f32( const tn_mesh* mesh, int bc_cmb, int bc_surface, int diagonal, int apply_mode,
                                        int comm_mode, const float* const* src, float* const* dst, void* stream );

/* Viscosity derivative of the epsilon-div-div form (backward kernel of the
 * adjoint viscosity gradient; no reference counterpart).  The one-point
 * operator A(k) of tn_epsdivdiv_apply_* is linear in k, so
 *     grad_k[n] = d (lambda^T A(k) u) / d k_n
 * does not depend on k: the sum over the wedges w holding n of
 * lambda_w^T A_w(1) u_w / 6, with the same Dirichlet / free-slip treatment as
 * the apply and without the k-independent fs/fs rotation penalty.
 * comm_mode TN_COMM_SKIP: derivative with respect to each stored copy of k;
 * TN_COMM_ADDITIVE: with respect to each unique node, on all its copies. */
TN_API int tn_epsdivdiv_kgrad_f64( const tn_mesh* mesh, int bc_cmb, int bc_surface, int comm_mode,
                                   const double* const* u, const double* const* lambda, double* grad_k, void* stream );
TN_API int tn_epsdivdiv_kgrad_f32( const tn_mesh* mesh, int bc_cmb, int bc_surface, int comm_mode,
                                   const float* const* u, const float* const* lambda, float* grad_k, void* stream );

/* ---------------------------------------------------------------------------
 * Stokes coupling blocks of the Q1-iso-Q2 / Q1 pair: `mesh` carries the P1
 * velocity (level L), `mesh_p` the P1 pressure (level L-1, same radii range).
 * Divergence::apply_impl (fe/wedge/operators/shell/divergence.hpp:90): p = B u;
 * Gradient::apply_impl (gradient.hpp:87): u = B^T p.  3x2 Felippa quadrature;
 * Dirichlet velocity nodes are eliminated, free-slip ones projected tangentially. */
TN_API int tn_divergence_apply_f64( const tn_mesh* mesh, const tn_mesh* mesh_p, int bc_cmb, int bc_surface,
                                    int apply_mode, int comm_mode, const double* const* u, double* p, void* stream );
TN_API int tn_divergence_apply_f32( const tn_mesh* mesh, const tn_mesh* mesh_p, int bc_cmb, int bc_surface,
                                    int apply_mode, int comm_mode, const float* const* u, float* p, void* stream );
TN_API int tn_gradient_apply_f64( const tn_mesh* mesh, const tn_mesh* mesh_p, int bc_cmb, int bc_surface,
                                  int apply_mode, int comm_mode, const double* p, double* const* u, void* stream );
TN_API int tn_gradient_apply_f32( const tn_mesh* mesh, const tn_mesh* mesh_p, int bc_cmb, int bc_surface,
                                  int apply_mode, int comm_mode, const float* p, float* const* u, void* stream );

/* ---------------------------------------------------------------------------
 * KMass::apply_impl (fe/wedge/operators/shell/kmass.hpp:66): int k u v, 3x2
 * Felippa rule, k interpolated at the quadrature points (k == NULL means
 * k = 1, i.e. Mass, mass.hpp).  mode 0 consistent, 1 diagonal, 2 lumped
 * diagonal (set_lumped_diagonal, :64). */
TN_API int tn_kmass_apply_f64( const tn_mesh* mesh, const double* k, int mode, int apply_mode, int comm_mode,
                               const double* src, double* dst, void* stream );
TN_API int tn_kmass_apply_f32( const tn_mesh* mesh, const float* k, int mode, int apply_mode, int comm_mode,
                               const float* src, float* dst, void* stream );

/* ---------------------------------------------------------------------------
 * Constant grid transfer of `ncomp` fields between `coarse` (level L-1) and
 * `fine` (level L): ProlongationVecConstant::apply_impl
 * (fe/wedge/operators/shell/prolongation_constant.hpp:121) and
 * RestrictionVecConstant::apply_impl (restriction_constant.hpp:161; owned fine
 * nodes only, followed by the additive coarse halo, Replace mode). */
TN_API int tn_prolongation_constant_f64( const tn_mesh* fine, const tn_mesh* coarse, int ncomp, int apply_mode,
                                         const double* const* src, double* const* dst, void* stream );
TN_API int tn_prolongation_constant_f32( const tn_mesh* fine, const tn_mesh* coarse, int ncomp, int apply_mode,
                                         const float* const* src, float* const* dst, void* stream );
TN_API int tn_restriction_constant_f64( const tn_mesh* fine, const tn_mesh* coarse, int ncomp,
                                        const double* const* src, double* const* dst, void* stream );
TN_API int tn_restriction_constant_f32( const tn_mesh* fine, const tn_mesh* coarse, int ncomp,
                                        const float* const* src, float* const* dst, void* stream );

/* ProlongationLinear / RestrictionLinear (fe/wedge/operators/shell/
 * prolongation_linear.hpp:14-190, restriction_linear.hpp:14-223, weights
 * fe/wedge/shell/grid_transfer_linear.hpp): a fine node on a coarse node
 * copies it, one between radially aligned coarse nodes interpolates by
 * radius, any other interpolates radially between the chord midpoints of two
 * lateral coarse pairs (exact for affine functions).  Restriction is the
 * transpose over OWNED fine nodes followed by the coarse halo sum (Replace).
 * ncomp fields are transferred with the same weights (the reference's vector
 * variants are unused; see the design notes). */
TN_API int tn_prolongation_linear_f64( const tn_mesh* fine, const tn_mesh* coarse, int ncomp, int apply_mode,
                                       const double* const* src, double* const* dst, void* stream );
TN_API int tn_prolongation_linear_f32( const tn_mesh* fine, const tn_mesh* coarse, int ncomp, int apply_mode,
                                       const float* const* src, float* const* dst, void* stream );
TN_API int tn_restriction_linear_f64( const tn_mesh* fine, const tn_mesh* coarse, int ncomp, const double* const* src,
                                      double* const* dst, void* stream );
TN_API int tn_restriction_linear_f32( const tn_mesh* fine, const tn_mesh* coarse, int ncomp, const float* const* src,
                                      float* const* dst, void* stream );

/* Injection coarse(X,Y,R) = fine(2X,2Y,2R) of `ncomp` fields (coefficient
 * fields on coarser multigrid levels). */
TN_API int tn_injection_f64( const tn_mesh* fine, const tn_mesh* coarse, int ncomp, const double* const* src,
                             double* const* dst, void* stream );
/* In-place tangential projection of a 3-vector field at the CMB (cmb != 0)
 * and SURFACE (surface != 0) nodes: strong_algebraic_freeslip_enforcement_in_place
 * (fe/strong_algebraic_freeslip_enforcement.hpp:23). */
TN_API int tn_freeslip_project_f64( const tn_mesh* mesh, double* const* y, int cmb, int surface, void* stream );

/* ---------------------------------------------------------------------------
 * Krylov vector kernels (kernels/common/grid_operations.hpp).  A vector is
 * `ncomp` scalar fields (1 or 3) of stored-node length.
 *
 * lincomb: y = c0 + sum_i c[i] x_i, nx = 0..3 (grid_operations.hpp:12,154;
 *          VectorQ1Vec::lincomb_impl, linalg/vector_q1.hpp:52-87)
 * dot:     owned-node dot product summed over components, compensated FP64
 *          accumulation in both precisions (masked_dot_product, :644)
 * others:  invert_inplace (:253), mult_elementwise_inplace (:273),
 *          max_abs_entry (:337), has_nan_or_inf (:714), cast (:746). */
TN_API int tn_vec_lincomb_f64( const tn_mesh* mesh, int ncomp, double* const* y, double c0, int nx, const double* c,
                        const double* const* x, void* stream );
TN_API int tn_vec_lincomb_f32( const tn_mesh* mesh, int ncomp, float* const* y, double c0, int nx, const double* c,
                        const float* const* x, void* stream );
TN_API int tn_vec_dot_f64( const tn_mesh* mesh, int ncomp, const double* const* a, const double* const* b, double* result,
                    void* stream );
TN_API int tn_vec_dot_f32( const tn_mesh* mesh, int ncomp, const float* const* a, const float* const* b, double* result,
                    void* stream );
/* Allocation-free variant of tn_vec_dot_f64 (no counterpart in the
 * reference): for callers that cannot let a library allocate device memory.
 * It needs no mesh handle and calls no cudaMalloc / cudaFree / allocating
 * library routine: its reduction scratch is a static device array of
 * 262,656 bytes inside the library.  result = sum over c < ncomp and
 * i < n of a[c][i] b[c][i] where owned[i] != 0 (owned NULL: every entry),
 * compensated FP64; returns after the value is on the host.  Limits:
 * n <= 33,554,432 entries per component (a larger n is rejected with
 * TN_ERR_ARG), ncomp 1..3.  No call may be made while the stream is being
 * captured into a CUDA graph: every call copies its result to host memory
 * and synchronises the stream (a capturing stream is rejected with
 * TN_ERR_ARG).  The stream must belong to the calling thread's current
 * device, whose scratch address the first call on that device looks up and
 * caches (a stream of another device is rejected).  All calls on one device
 * share the scratch: calls that can overlap (several streams or host
 * threads) race and must be serialised by the caller. */
TN_API int tn_vec_dot_noalloc_f64( size_t n, int ncomp, const double* const* a, const double* const* b,
                                   const uint8_t* owned, double* result, void* stream );
TN_API int tn_vec_invert_f64( const tn_mesh* mesh, int ncomp, double* const* y, void* stream );
TN_API int tn_vec_invert_f32( const tn_mesh* mesh, int ncomp, float* const* y, void* stream );
TN_API int tn_vec_mult_f64( const tn_mesh* mesh, int ncomp, double* const* y, const double* const* x, void* stream );
TN_API int tn_vec_mult_f32( const tn_mesh* mesh, int ncomp, float* const* y, const float* const* x, void* stream );
/* masked_sum (grid_operations.hpp:569-590) with the ownership mask: the sum over owned nodes, components summed,
 * compensated FP64 accumulation; the number of owned nodes (count_masked, :544) is tn_mesh_dims' unique_nodes */
TN_API int tn_vec_sum_f64( const tn_mesh* mesh, int ncomp, const double* const* x, double* result, void* stream );
TN_API int tn_vec_sum_f32( const tn_mesh* mesh, int ncomp, const float* const* x, double* result, void* stream );
TN_API int tn_vec_max_abs_f64( const tn_mesh* mesh, int ncomp, const double* const* x, double* result, void* stream );
TN_API int tn_vec_max_abs_f32( const tn_mesh* mesh, int ncomp, const float* const* x, double* result, void* stream );
TN_API int tn_vec_has_nan_or_inf_f64( const tn_mesh* mesh, int ncomp, const double* const* x, int* result, void* stream );
TN_API int tn_vec_has_nan_or_inf_f32( const tn_mesh* mesh, int ncomp, const float* const* x, int* result, void* stream );
/* assign_masked_else_keep_old (kernels/common/grid_operations.hpp) with the
 * CMB / SURFACE boundary flags: on the radial boundary layers selected by cmb
 * (r = 0) and surface (r = N), y = x, or the constant c when x is NULL; other
 * nodes keep their values.  The strong Dirichlet enforcement of
 * fe/strong_algebraic_dirichlet_enforcement.hpp is b -= A_neumann g followed by
 * this assign with x = diag(A_neumann) g (or c = 0, homogeneous). */
TN_API int tn_vec_assign_boundary_f64( const tn_mesh* mesh, int ncomp, double* const* y, const double* const* x,
                                       double c, int cmb, int surface, void* stream );
TN_API int tn_vec_assign_boundary_f32( const tn_mesh* mesh, int ncomp, float* const* y, const float* const* x,
                                       double c, int cmb, int surface, void* stream );
/* One fused Chebyshev step (linalg/solvers/chebyshev.hpp:127-160):
 * d = alpha D^{-1} (b - ax) + beta d;  x = x + d.  beta = 0 does not read d. */
TN_API int tn_vec_chebyshev_step_f64( const tn_mesh* mesh, int ncomp, double* const* x, double* const* d,
                                      const double* const* b, const double* const* ax, const double* const* inv_diag,
                                      double alpha, double beta, void* stream );
TN_API int tn_vec_chebyshev_step_f32( const tn_mesh* mesh, int ncomp, float* const* x, float* const* d,
                                      const float* const* b, const float* const* ax, const float* const* inv_diag,
                                      double alpha, double beta, void* stream );
/* randomize (grid_operations.hpp:759) made deterministic: uniform [-1, 1)
 * from a counter-based hash of (seed, component, index). */
TN_API int tn_vec_randomize_f64( const tn_mesh* mesh, int ncomp, double* const* y, unsigned long long seed,
                                 void* stream );
TN_API int tn_vec_randomize_f32( const tn_mesh* mesh, int ncomp, float* const* y, unsigned long long seed, void* stream );
TN_API int tn_vec_cast_f64_to_f32( const tn_mesh* mesh, int ncomp, float* const* y, const double* const* x, void* stream );
TN_API int tn_vec_cast_f32_to_f64( const tn_mesh* mesh, int ncomp, double* const* y, const float* const* x, void* stream );

/* ---------------------------------------------------------------------------
 * Finite-volume FCT advection-diffusion of a cell-centred scalar
 * (fv/hex/operators/fct_advection_diffusion.hpp).  FV fields are
 * [10][N+2][N+2][N+2] with one ghost layer, r fastest (linalg/vector_fv.hpp);
 * cell (x, y, r), 1 <= x, y, r <= N, is FE cell (x-1, y-1, r-1) of `mesh`;
 * vector FV fields (cell centres) are three such arrays.  `vel` is the Q1
 * velocity on the mesh's stored nodes (3 fields). */
typedef struct
{
    double T_cmb;
    double T_surface;
    int    apply_cmb;
    int    apply_surface;
} tn_fct_dirichlet; /* fv/hex/helpers.hpp DirichletBCs */

/* entries of one FV field: 10 (N+2)^3 */
TN_API int tn_fv_field_size( const tn_mesh* mesh, size_t* entries );
/* doubles of the tn_fct_step_f64 workspace: 9 FV fields (T^L, 6 antidiffusive
 * fluxes per cell, R+, R-) */
TN_API int tn_fct_workspace_size( const tn_mesh* mesh, size_t* entries );
/* update_fv_ghost_layers (communication/shell/fv_communication.hpp): lateral
 * ghost cells := the real cells across each diamond face */
TN_API int tn_fv_ghost_update_f64( const tn_mesh* mesh, double* field, void* stream );
/* initialize_cell_centers (fv/hex/helpers.hpp:101-169): volume centroids of
 * the cells, lateral ghosts filled, radial ghosts 0 */
TN_API int tn_fv_cell_centers_f64( const tn_mesh* mesh, double* const* centers, void* stream );
/* compute_dt_stable (fct_advection_diffusion.hpp:193-254): min over cells of
 * volume / (inflow + two-point diffusion); synchronises */
TN_API int tn_fct_dt_stable_f64( const tn_mesh* mesh, const double* const* vel, const double* const* centers,
                                 double diffusivity, double* dt_stable, void* stream );
/* apply_dirichlet_bcs (fv/hex/helpers.hpp:26-64): first / last real layer
 * and its radial ghost */
TN_API int tn_fct_apply_dirichlet_f64( const tn_mesh* mesh, double* T, const tn_fct_dirichlet* bcs, void* stream );
/* fct_explicit_step (fct_advection_diffusion.hpp:720-750): T^{n+1} in place
 * (T's lateral ghosts are refreshed first).  source (FV field) may be NULL;
 * bcs NULL skips the Dirichlet treatment of T^L.  workspace holds
 * tn_fct_workspace_size doubles; its first FV field is T^L on return. */
TN_API int tn_fct_step_f64( const tn_mesh* mesh, double* T, const double* const* vel, const double* const* centers,
                            double dt, double diffusivity, const double* source, int subtract_divergence,
                            const tn_fct_dirichlet* bcs, double* workspace, void* stream );

/* ---------------------------------------------------------------------------
 * Device-resident Krylov steps (no host synchronisation).
 *
 * A Krylov vector is passed as `nseg` (1..4) scalar fields, field k living on
 * mesh[k] (stored-node length, reduced over mesh[k]'s owned nodes): a
 * velocity field is 3 segments, the Stokes block vector (velocity on the fine
 * mesh, pressure on the coarse one; linalg/vector_q1isoq2_q1.hpp:19) is 4.
 * Scalars (`coeff`, `gate`, `result`, `state`) are DEVICE pointers.  These
 * restate the host loops of linalg/solvers/fgmres.hpp:197-229 and
 * linalg/solvers/pcg.hpp:78-102 with their scalars kept on the device; the
 * reference has no C entry point of this shape.
 *
 * axpy_dot: if gate != NULL and *gate != 0 does nothing; otherwise
 *   w = w - coeff[0] * x  (skipped when x == NULL), then
 *   result[0] = <w, v>    (v == NULL: <w, w>), compensated FP64.
 * Chaining these gives one pass per modified Gram-Schmidt step. */
TN_API int tn_krylov_axpy_dot_f64( int nseg, const tn_mesh* const* mesh, double* const* w, const double* const* x,
                                   const double* coeff, const double* const* v, const double* gate, double* result,
                                   void* stream );
TN_API int tn_krylov_axpy_dot_f32( int nseg, const tn_mesh* const* mesh, float* const* w, const float* const* x,
                                   const double* coeff, const float* const* v, const double* gate, double* result,
                                   void* stream );

/* Unpreconditioned PCG (pcg.hpp:78-102; z = r) with its state in device
 * memory.  state is a device array of at least 8 + max_iterations + 1
 * doubles: [0] <r,r>, [1] <Ap,p>, [2] |r0|, [3] beta, [4] done flag (0/1),
 * [5] iterations, [6] last relative residual, [8 + k] relative residual after
 * iteration k ([8] = 1).  One iteration k (1-based) is
 *     ap = A p                (any operator apply; runs regardless of done)
 *     tn_pcg_pap_f64          <ap, p>
 *     tn_pcg_update_f64(k)    x += alpha p, r -= alpha ap, stopping rule, beta
 *     tn_pcg_direction_f64    p = r + beta p
 * after tn_pcg_begin_f64 on r = b - A x.  Once the stopping rule fires
 * (relres <= rtol or |r| < atol; begin: |r0| < atol) every later step leaves
 * x, r, p and state untouched, so a caller may read the flag only now and
 * then, or issue all iterations.  iteration <= 0 takes the step number from the state (the count of the
 * steps done so far + 1), so a captured graph of steps can be replayed; the caller issues at most max_iterations
 * steps in all (the history has room for that many). */
TN_API int tn_pcg_begin_f64( int nseg, const tn_mesh* const* mesh, const double* const* r, double* const* p,
                             double* state, double atol, void* stream );
TN_API int tn_pcg_pap_f64( int nseg, const tn_mesh* const* mesh, const double* const* ap, const double* const* p,
                           double* state, void* stream );
TN_API int tn_pcg_update_f64( int nseg, const tn_mesh* const* mesh, double* const* x, double* const* r,
                              const double* const* p, const double* const* ap, double* state, int iteration,
                              double rtol, double atol, void* stream );
TN_API int tn_pcg_direction_f64( int nseg, const tn_mesh* const* mesh, double* const* p, const double* const* r,
                                 const double* state, void* stream );

/* ---------------------------------------------------------------------------
 * Solver drivers.
 *
 * PCG (linalg/solvers/pcg.hpp:78) without preconditioner on the scalar
 * Laplace with homogeneous Dirichlet elimination on both radii
 * (tests/test_laplace_cg.cpp:115-200 composition): solves A x = b from the
 * initial guess in x; stops at ||r|| / ||r0|| <= relative_tolerance or
 * ||r|| < absolute_tolerance. */
TN_API int tn_laplace_pcg_solve_f64( const tn_mesh* mesh, const double* b, double* x, int max_iterations,
                                     double relative_tolerance, double absolute_tolerance, int* iterations,
                                     double* relative_residual );

/* The library's Krylov solver templates without a preconditioner on the
 * scalar Laplace with Dirichlet elimination (fe/wedge/operators/shell/laplace.hpp:106,
 * treat_boundary = true), from the given x (the compositions of the
 * reference's tests/test_laplace_fgmres.cpp, test_laplace_minres.cpp and
 * test_laplace_bicgstab.cpp): solver 0 = FGMRES(param) (linalg/solvers/fgmres.hpp:108-330),
 * 1 = PMINRES (linalg/solvers/pminres.hpp:30-175, param unused),
 * 2 = PBiCGStab(param) (linalg/solvers/pbicgstab.hpp:29-290) with the shadow
 * residual `shadow` (device, stored nodes) or, when NULL, this library's
 * seeded random field. history (host, optional): the relative residual
 * estimates the solver records (entry 0 = 1), at most history_capacity of
 * them; *history_count = how many it recorded. */
TN_API int tn_laplace_krylov_solve_f64( const tn_mesh* mesh, int solver, int param, const double* b, double* x,
                                        const double* shadow, int max_iterations, double relative_tolerance,
                                        double absolute_tolerance, int* iterations, double* history,
                                        int history_capacity, int* history_count );

/* Multigrid-preconditioned Krylov solve (CG, BiCGStab(2) or MINRES) on
 * DivKGrad (k NULL: k = 1, the Laplace) with
 * homogeneous Dirichlet elimination on both radii: one V-cycle per CG
 * iteration over levels [level - mg_levels + 1, level], linear transfers
 * (prolongation_linear.hpp / restriction_linear.hpp), Jacobi (smoother 1,
 * jacobi.hpp: smoothing_steps sweeps with jacobi_omega) or Chebyshev
 * (smoother 0, chebyshev.hpp: chebyshev_order, smoothing_steps sweeps,
 * power_iterations), unpreconditioned PCG on the coarsest level; coarser
 * levels use k injected from the finest (the composition of the reference's
 * tests/test_div_k_grad_multigrid*.cpp).  b, x, k are device fields of the
 * finest mesh; x holds the initial guess and receives the solution. */
typedef struct
{
    int    level;
    int    mg_levels;
    int    smoother;        /* 0 Chebyshev, 1 Jacobi */
    int    smoothing_steps; /* sweeps before and after the coarse correction */
    int    chebyshev_order;
    int    power_iterations;
    double jacobi_omega;
    int    vcycles;
    int    coarse_max_iterations;
    double coarse_relative_tolerance;
    int    max_iterations;
    double relative_tolerance;
    double absolute_tolerance;
    int    krylov; /* outer solver: 0 PCG (pcg.hpp), 1 PBiCGStab(2) (pbicgstab.hpp), 2 PMINRES (pminres.hpp) */
} tn_scalar_mg_params;

TN_API int tn_divkgrad_mg_pcg_solve_f64( const tn_scalar_mg_params* params, double r_min, double r_max,
                                         const double* k, const double* b, double* x, int* iterations,
                                         double* relative_residual );

/* Stokes solver composed as apps/mantlecirculation/mantlecirculation.cpp:486-735:
 * FGMRES(restart) (fgmres.hpp:108) on EpsDivDivStokes [A B^T; B 0]
 * (epsilon_divdiv_stokes.hpp:55), BlockTriangularPreconditioner2x2
 * (block_preconditioner_2x2.hpp:205) with a multigrid V-cycle (multigrid.hpp:119,
 * Chebyshev smoothing chebyshev.hpp:100, constant transfers, PCG coarse solve)
 * on A and the inverse lumped KMass(1/eta) (kmass.hpp) on the Schur block.
 * Velocity on `level`, pressure on level-1; the multigrid spans mg_levels
 * levels ending at `level`, coarser viscous operators re-discretised with the
 * viscosity injected from `level`.  mg_fp32 != 0 runs the V-cycle in FP32
 * (FP32 operators, smoothers, transfers) inside the FP64 FGMRES; the outer
 * residual, dots, Schur diagonal and coarsest PCG are FP64. */
typedef struct
{
    int    level;
    int    mg_levels;
    int    bc_cmb;
    int    bc_surface;
    int    mg_fp32;
    int    chebyshev_order;
    int    smoothing_steps;
    int    power_iterations;
    int    vcycles;
    int    coarse_max_iterations;
    double coarse_relative_tolerance;
    int    restart;
    int    max_iterations;
    double relative_tolerance;
    double absolute_tolerance;
    int    gca; /* coarse viscous operators: 0 re-discretised with injected viscosity, 1 GCA with
                   constant interpolation (TwoGridGCA default), 2 GCA with linear interpolation, 3 adaptive GCA
                   (the app's gca == 2, mantlecirculation.cpp:379-387, 565-592): Galerkin matrices with constant
                   interpolation below the coarsest cells GCAElementsCollector marks on the finest viscosity,
                   the re-discretised matrices of the injected viscosity elsewhere */
    int    outer; /* 0 FGMRES(restart) + block-triangular preconditioner, 1 PMINRES + block-diagonal
                     preconditioner (pminres.hpp, block_preconditioner_2x2.hpp:38-100), 2 mixed-precision
                     iterative refinement (needs mg_fp32 = 1): FP64 residual and update around an FGMRES(restart)
                     + block-triangular solve done entirely in FP32 (coarsest PCG in FP64); no counterpart in
                     the reference.  `iterations` counts the inner FGMRES iterations of all cycles. */
    int    eager; /* 0: after its first application the preconditioner is captured once per vector pair as a
                     CUDA graph and replayed; 1: always launched kernel by kernel */
    const double* chebyshev_estimates; /* NULL: each level's Chebyshev smoother estimates the largest eigenvalue of
                     D^-1 A by power iteration on its first use (chebyshev.hpp:159-163); otherwise mg_levels
                     estimates, coarsest level first, used as given (the reference draws the power iteration's
                     start vector at random, so reproducing one of its runs needs the estimates it drew) */
} tn_stokes_params;

typedef struct tn_stokes_solver tn_stokes_solver;

/* `viscosity`: device FP64 field on `level` (copied) */
TN_API int tn_stokes_solver_create( const tn_stokes_params* params, double r_min, double r_max,
                                    const double* viscosity, tn_stokes_solver** out );
/* f_u (3 fields, level) / f_p (level-1): right-hand side; x_u / x_p: initial
 * guess on entry, solution on return (device pointers). */
TN_API int tn_stokes_solve( tn_stokes_solver* solver, const double* const* f_u, const double* f_p,
                            double* const* x_u, double* x_p, int* iterations, double* relative_residual );
/* relative residual history of the last solve (FGMRES estimates, entry 0 = 1) */
TN_API int tn_stokes_history( const tn_stokes_solver* solver, double* out, int capacity, int* count,
                              int* preconditioner_skips );
/* out = K in (the FP64 Stokes operator of the solver) */
TN_API int tn_stokes_apply( tn_stokes_solver* solver, const double* const* u, const double* p, double* const* out_u,
                            double* out_p );
/* Backward of the Stokes solve with respect to the log-viscosity (adjoint
 * viscosity gradient; no reference counterpart).  u is the forward velocity
 * solution of this solver, grad_u the derivative of an objective J with
 * respect to the stored velocity entries (copy-wise: for J = 1/2 sum over
 * owned nodes |u - u_obs|^2 it is (u - u_obs) on owned copies, 0 elsewhere).
 * Sums grad_u over node copies, applies the velocity boundary treatment,
 * solves the adjoint system K lambda = (grad_u, 0) with the solver's FGMRES
 * (K is symmetric) and returns grad_log_k = dJ/d log k = -k * d(lambda^T K x)/dk
 * (tn_epsdivdiv_kgrad_f64 with comm_mode: per stored copy, or per unique node
 * on all copies).  lambda_u / lambda_p receive the adjoint solution when not
 * NULL; iterations the adjoint FGMRES iterations.  Synchronises. */
TN_API int tn_stokes_viscosity_backward( tn_stokes_solver* solver, const double* const* u, const double* const* grad_u,
                                         int comm_mode, double* grad_log_k, double* const* lambda_u, double* lambda_p,
                                         int* iterations );
TN_API int tn_stokes_solver_destroy( tn_stokes_solver* solver );

/* Pieces of the mantle-circulation time step (apps/mantlecirculation/mantlecirculation.cpp:870-1045).
 * tn_fv_to_fe_rhs_f64: b_i = sum_K fv_K int_K phi_i (fv: FV field [10][N+2]^3 with ghosts) and / or the lumped
 * diagonal D_i = sum_K int_K phi_i over the FV cells K (3x2 rule), both summed over node copies
 * (fv/hex/conversion.hpp:146-190); either output may be NULL (b needs fv). */
TN_API int tn_fv_to_fe_rhs_f64( const tn_mesh* mesh, const double* fv, double* b, double* lumped_diagonal, void* stream );
/* FV -> FE transfer (l2_project_fv_to_fe, conversion.hpp:131-205, and l2_project_fv_to_fe_lumped, :243-300):
 * lumped = 0 solves M dst = b with the unpreconditioned PCG on the Q1 mass matrix starting from dst's values
 * (the reference uses max_iterations 1000, tolerances 1e-12 / 1e-12); lumped != 0 sets dst = b / D.  work: 5
 * stored-node fields (2 for the lumped form).  iterations (optional): PCG iterations. */
TN_API int tn_l2_project_fv_to_fe_f64( const tn_mesh* mesh, const double* fv, double* dst, int lumped, int max_iterations,
                                       double relative_tolerance, double absolute_tolerance, double* work,
                                       int* iterations, void* stream );
/* Stokes buoyancy right-hand side (RHSVelocityInterpolator, mantlecirculation.cpp:117-150, and :883-899):
 * f_u = VectorMass (rayleigh T n), n the unit radial direction, then zero velocity rows on Dirichlet boundaries
 * (strong_algebraic_homogeneous_velocity_dirichlet_enforcement_stokes_like) and the normal component removed on
 * free-slip ones (strong_algebraic_freeslip_enforcement_in_place), each on the boundary the app passes: the first
 * with that condition (CMB before SURFACE), so the same condition on both radii treats only the CMB rows.
 * T: FE scalar; work: 3 stored-node fields. */
TN_API int tn_stokes_buoyancy_rhs_f64( const tn_mesh* mesh, const double* T, double rayleigh, int bc_cmb,
                                       int bc_surface, double* const* f_u, double* work, void* stream );
/* Pressure normalisation (mantlecirculation.cpp:930-936): p -= sum over owned nodes of p / unique nodes.
 * work: one stored-node field; mean (optional) receives the subtracted value.  Synchronises. */
TN_API int tn_pressure_remove_mean_f64( const tn_mesh* mesh, double* p, double* work, double* mean, void* stream );

/* ---- FE -> FV transfer -------------------------------------------------- */
/* Cell averages of the FE scalar fe on the FV cells of the mesh (fv/hex/conversion.hpp:349-416,
 * l2_project_fe_to_fv): fv[d][x][y][r] = int_K fe / |K| for the cells x, y, r in 1..N (the two wedges of the
 * hex cell, integrals in closed form, exact as the reference's 3x2 rule), then the lateral FV ghost layers
 * (tn_fv_ghost_update_f64).  Radial ghost cells are left as they are.  fv: [10][N+2]^3. */
TN_API int tn_l2_project_fe_to_fv_f64( const tn_mesh* mesh, const double* fe, double* fv, void* stream );

/* ---- SUPG energy operator ----------------------------------------------- */
/* UnsteadyAdvectionDiffusionSUPG::apply_impl (fe/wedge/operators/shell/unsteady_advection_diffusion_supg.hpp:
 * 199-420): dst = (mass_scaling M + dt (K + C + G)) src, the BDF left-hand side of the temperature equation with
 * SUPG stabilisation for the velocity vel (three SoA components), constant diffusivity kappa, mass lumping,
 * the reference's boundary mask (treat_boundary: off-diagonal entries of CMB / surface rows and columns
 * dropped) and diagonal mode; apply / communication modes as the other operators. */
TN_API int tn_supg_apply_f64( const tn_mesh* mesh, const double* const* vel, double kappa, double dt, double mass_scaling,
                              int lumped_mass, int treat_boundary, int diagonal, int apply_mode, int comm_mode,
                              const double* src, double* dst, void* stream );
TN_API int tn_supg_apply_f32( const tn_mesh* mesh, const float* const* vel, double kappa, double dt, double mass_scaling,
                              int lumped_mass, int treat_boundary, int diagonal, int apply_mode, int comm_mode,
                              const float* src, float* dst, void* stream );
/* One implicit BDF step of the SUPG temperature equation as the reference's tests solve it
 * (tests/test_unsteady_advection_diffusion_supg.cpp:124-172): x <- solution of
 * (mass_scaling M + dt (K + C + G)) x = rhs with PBiCGStab(l) (pbicgstab.hpp:29-290, no preconditioner) from the
 * given x, at most max_iterations iterations, stopping at relative_tolerance (of the initial residual) or
 * absolute_tolerance.  vel: one contiguous [3][nodes] array (vel[1] = vel[0] + nodes, vel[2] = vel[0] + 2 nodes).
 * work: (2 (l + 1) + 2) stored-node FP64 fields.  iterations / relative_residual: optional outputs.  Synchronises. */
TN_API int tn_supg_solve_f64( const tn_mesh* mesh, const double* const* vel, double kappa, double dt, double mass_scaling,
                              int lumped_mass, int treat_boundary, const double* rhs, double* x, int l, int max_iterations,
                              double relative_tolerance, double absolute_tolerance, double* work, int* iterations,
                              double* relative_residual, void* stream );

/* ---- XDMF output and checkpoints (io/xdmf.hpp) -------------------------- */
/* io::XDMFOutput (io/xdmf.hpp:147-1115): a time series of node fields in the reference's directory format,
 * which is both the visualisation output and the checkpoint: geometry.bin, topology.bin and
 * checkpoint_metadata.bin at the first write, <label>_<step>.bin per grid and step_<step>.xmf (written last)
 * per write.  One subdomain per diamond (global ids diamond << 57), one process.
 * points_bytes: 4 or 8 (OutputTypeFloat of the coordinates); connectivity_bytes: 4 or 8 (OutputTypeInt). */
typedef struct tn_xdmf_output tn_xdmf_output;
TN_API int tn_xdmf_output_create( const tn_mesh* mesh, const char* directory, int points_bytes, int connectivity_bytes,
                                  tn_xdmf_output** out );
/* XDMFOutput::set_write_counter (:204): the step number of the next write */
TN_API int tn_xdmf_output_set_write_counter( tn_xdmf_output* w, int counter );
/* XDMFOutput::add (:210-280): a device grid of vec_dim 1 or 3 components (SoA pointers, input_bytes 4 = FP32
 * or 8 = FP64 entries) written as output_bytes 4 or 8 floats under `label`.  The pointers must stay valid for
 * the writer's lifetime.  Errors (TN_ERR_ARG) after the first write and for a label already added. */
TN_API int tn_xdmf_output_add( tn_xdmf_output* w, const char* label, int input_bytes, int vec_dim,
                               const void* const* components, int output_bytes );
/* XDMFOutput::write (:283-520): converts every grid to the file order and type on `stream` (the grids may
 * change as soon as the stream has passed this point), copies them to pinned host memory on the writer's own
 * stream and writes the files from a host thread; returns before the files are complete.  The first call also
 * writes the mesh and metadata files (synchronously).  A file error of the previous write is returned by the
 * next write or wait (TN_ERR_IO). */
TN_API int tn_xdmf_output_write( tn_xdmf_output* w, void* stream );
/* blocks until the files of the last write are complete; TN_ERR_IO if one could not be written */
TN_API int tn_xdmf_output_wait( tn_xdmf_output* w );
TN_API int tn_xdmf_output_destroy( tn_xdmf_output* w );

/* CheckpointMetadata (io/xdmf.hpp:1117-1153) without its lists */
typedef struct
{
    int version, subdomains_lateral, subdomains_radial, size_x, size_y, size_r;
    int grid_scalar_bytes, num_grid_data_files, ordering, num_radii, num_subdomain_ids;
} tn_checkpoint_info;
/* read_xdmf_checkpoint_metadata (:1162-1268), host only: the fixed fields, the radii (up to radii_capacity)
 * and the global subdomain ids in file order (up to ids_capacity; either array may be null).
 * TN_ERR_IO with the reference's error text in tn_last_error(). */
TN_API int tn_read_xdmf_checkpoint_metadata( const char* directory, tn_checkpoint_info* info, double* radii,
                                             int radii_capacity, long long* subdomain_ids, int ids_capacity );
/* the index-th grid record of the metadata: label (NUL-terminated), scalar_data_type (2 = float),
 * scalar_bytes, vec_dim; host only */
TN_API int tn_xdmf_checkpoint_grid_data_file( const char* directory, int index, char* label, int label_capacity,
                                              int* scalar_data_type, int* scalar_bytes, int* vec_dim );
/* read_xdmf_checkpoint_grid (:1270-1500): grid `label` of write `step` into the device field dst (vec_dim 1
 * or 3 SoA pointers of dst_bytes 4 or 8 entries), converted from the file's type; the diamonds' chunks are
 * found through the metadata's subdomain ids.  Synchronises the stream.  TN_ERR_IO with the reference's error
 * text (missing metadata, label or step file, extents, ordering, data type, scalar / vector mismatch). */
TN_API int tn_read_xdmf_checkpoint_grid( const tn_mesh* mesh, const char* directory, const char* label, int step,
                                         int dst_bytes, int vec_dim, void* const* dst, void* stream );

/* ---------------------------------------------------------------------------
 * Sharded shell: one rank's diamonds, one process per GPU.
 *
 * The reference's DistributedDomain::create_uniform (grid/shell/spherical_shell.hpp:2566-2590) with lateral and
 * radial subdomain refinement level 0 and its default map subdomain_to_rank_iterate_diamond_subdomains (:717-745)
 * gives rank q of P a contiguous block of diamonds: 10 / P of them, one more on the first 10 % P ranks.  A shard
 * holds that block compactly (local diamond index = global id - first diamond; the node layout of the mesh for each
 * diamond).  Finer subdomains are not supported: the operator kernels sweep whole diamonds.
 *
 * The additive halo of the reference's apply (send_recv: pack_send_and_recv_local_subdomain_boundaries +
 * unpack_and_reduce_local_subdomain_boundaries with SUM, communication/shell/communication.hpp:242-747) is split:
 * an apply with TN_COMM_ADDITIVE sums the copies of the duplicated nodes that all lie on this rank; the nodes with
 * copies on two or more ranks ("cross groups", in one order on every rank) are summed by
 *     tn_shard_pack   (buf = per cross group and radius the sum of this rank's copies, layout [field][group][r]),
 *     an all-reduce (SUM) of buf over the ranks by the caller's communicator (NCCL, MPI),
 *     tn_shard_unpack (every local copy = buf).
 * An exchange buffer holds nfields * exchange_values entries (tn_shard_dims); it is the same size on every rank. */
typedef struct tn_shard tn_shard;

/* Host only: the first diamond and the number of diamonds of `rank` (num_ranks in [1, 10]). */
TN_API int tn_shell_partition( int num_ranks, int rank, int* first_diamond, int* num_diamonds );
/* Host only: the rank's duplicate groups at `level`, CSR over local lateral indices
 * (local diamond * (N+1)^2 + x (N+1) + y), copies ascending: cross = 0 the groups whose copies all lie on this rank,
 * cross = 1 the cross groups (a group without a copy here is empty).  offsets has n_groups + 1 entries, members
 * n_members; pass NULL arrays to query the counts. */
TN_API int tn_shard_halo_plan( int level, int num_ranks, int rank, int cross, int* n_groups, int* n_members,
                               int* offsets, int* members );
TN_API int tn_shard_create( int level, double r_min, double r_max, int num_ranks, int rank, tn_shard** out );
TN_API int tn_shard_destroy( tn_shard* shard );
/* stored nodes = diamonds (N+1)^3; owned = the nodes this rank owns (ownership as on the whole shell: the copy in
 * the lowest diamond), summing to (10 N^2 + 2)(N+1) over the ranks; exchange_values = cross groups x (N+1) */
TN_API int tn_shard_dims( const tn_shard* shard, int* first_diamond, int* num_diamonds, size_t* stored_nodes,
                          size_t* owned_nodes, size_t* exchange_values );
/* host copies: coords [diamonds][N+1][N+1][3], radii [diamonds][N+1]; masks [diamonds][N+1][N+1][N+1] */
TN_API int tn_shard_geometry( const tn_shard* shard, double* coords, double* radii );
TN_API int tn_shard_masks( const tn_shard* shard, uint8_t* boundary_mask, uint8_t* ownership_mask );
/* EpsilonDivDivKerngen apply on the shard's cells (tn_epsdivdiv_apply_*); free-slip on both radii (the global
 * rigid-rotation penalty) only with num_ranks = 1 here, with more ranks through the two calls below */
TN_API int tn_shard_epsdivdiv_apply_f64( const tn_shard* shard, const tn_epsdivdiv_params* p, const double* k,
                                         const double* const* src, double* const* dst, void* stream );
TN_API int tn_shard_epsdivdiv_apply_f32( const tn_shard* shard, const tn_epsdivdiv_params* p, const float* k,
                                         const float* const* src, float* const* dst, void* stream );
/* Free-slip on both radii with two or more ranks: the rigid-rotation penalty needs the whole shell's three rotation
 * dots b_j = sum over owned nodes of (e_j x x) . src.  tn_shard_penalty_dots_* writes this rank's part to `dots`
 * (3 doubles, device); the caller sums them over the ranks (an all-reduce) and passes the sums to
 * tn_shard_epsdivdiv_apply_fsfs_*, which forms the penalty vector eps G^-1 b from them (kerngen :287-408, :585-606). */
TN_API int tn_shard_penalty_dots_f64( const tn_shard* shard, const double* const* src, double* dots, void* stream );
TN_API int tn_shard_penalty_dots_f32( const tn_shard* shard, const float* const* src, double* dots, void* stream );
TN_API int tn_shard_epsdivdiv_apply_fsfs_f64( const tn_shard* shard, const tn_epsdivdiv_params* p, const double* k,
                                              const double* const* src, double* const* dst, const double* dots,
                                              void* stream );
TN_API int tn_shard_epsdivdiv_apply_fsfs_f32( const tn_shard* shard, const tn_epsdivdiv_params* p, const float* k,
                                              const float* const* src, float* const* dst, const double* dots,
                                              void* stream );
TN_API int tn_shard_pack_f64( const tn_shard* shard, const double* const* fields, int nfields, double* buf,
                              void* stream );
TN_API int tn_shard_pack_f32( const tn_shard* shard, const float* const* fields, int nfields, float* buf, void* stream );
TN_API int tn_shard_unpack_f64( const tn_shard* shard, const double* buf, double* const* fields, int nfields,
                                void* stream );
TN_API int tn_shard_unpack_f32( const tn_shard* shard, const float* buf, float* const* fields, int nfields,
                                void* stream );
/* this rank's owned-node part of a dot product (tn_vec_dot_f64); the global dot is its sum over the ranks */
TN_API int tn_shard_vec_dot_f64( const tn_shard* shard, int ncomp, const double* const* a, const double* const* b,
                                 double* result, void* stream );
TN_API int tn_shard_vec_lincomb_f64( const tn_shard* shard, int ncomp, double* const* y, double c0, int nx,
                                     const double* c, const double* const* x, void* stream );
/* Multigrid on shards (a rank's shards at two levels, the same rank of the same partition):
 * tn_prolongation_constant_f64, tn_restriction_constant_f64 (its coarse halo sums the copies on this rank; the
 * cross-rank copies follow with pack / all-reduce / unpack on the coarse shard), tn_injection_f64,
 * tn_vec_invert_f64, tn_vec_mult_f64 and tn_vec_chebyshev_step_f64 on the shard's nodes. */
TN_API int tn_shard_prolongation_constant_f64( const tn_shard* fine, const tn_shard* coarse, int ncomp, int apply_mode,
                                               const double* const* src, double* const* dst, void* stream );
TN_API int tn_shard_restriction_constant_f64( const tn_shard* fine, const tn_shard* coarse, int ncomp,
                                              const double* const* src, double* const* dst, void* stream );
TN_API int tn_shard_injection_f64( const tn_shard* fine, const tn_shard* coarse, int ncomp, const double* const* src,
                                   double* const* dst, void* stream );
TN_API int tn_shard_vec_invert_f64( const tn_shard* shard, int ncomp, double* const* y, void* stream );
TN_API int tn_shard_vec_mult_f64( const tn_shard* shard, int ncomp, double* const* y, const double* const* x,
                                  void* stream );
TN_API int tn_shard_vec_chebyshev_step_f64( const tn_shard* shard, int ncomp, double* const* x, double* const* d,
                                            const double* const* b, const double* const* ax,
                                            const double* const* inv_diag, double alpha, double beta, void* stream );

#ifdef __cplusplus
}
#endif
#endif
