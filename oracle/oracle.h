/* CPU restatement of the reference's hot-path algorithms (TEST INFRASTRUCTURE).
 *
 * This library is the oracle: tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py use it to check the CUDA product.  The product
 * never links, loads or calls it.  Each function cites the reference file
 * (path inside the reference project) whose behaviour it restates.
 *
 * Parity pinning: tests/test_oracle_pinning.py compares these functions with
 * the reference itself (compiled by oracle/ref_build into oracle/_ref) and
 * with the committed fixtures in tests/golden/ generated from it.
 *
 * Layout conventions (identical to the reference, grid/grid_types.hpp:12-57):
 *   lateral coords  [10][N+1][N+1][3]   unit-sphere points of each diamond
 *   radii           [10][N+1]
 *   scalar field    [10][N+1][N+1][N+1] (diamond, x, y, r), r fastest
 *   vector field    3 scalar fields one after another (SoA)
 * with N = 2^L cells per diamond side and one subdomain per diamond.
 * Boundary-condition codes: 0 Neumann, 1 Dirichlet, 2 free-slip. */
#ifndef TN_ORACLE_H
#define TN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* mesh + masks */
void or_unit_sphere_coords( int L, double* coords );
void or_shell_radii( int L, double rmin, double rmax, double* radii );
void or_boundary_mask( int L, uint8_t* bmask );
void or_ownership_mask( int L, const double* coords, uint8_t* omask );
/* duplicated-node additive reduction (halo SUM) of ncomp scalar fields */
void or_halo_sum( int L, const double* coords, double* field, int ncomp );
void or_fv_to_fe_rhs( int L, const double* coords, const double* radii, const double* fv, double* b, double* D );
void or_fe_to_fv( int L, const double* coords, const double* radii, const double* fe, double* fv );
void or_gca_elements( int L, const double* k, int level_range, uint8_t* marks );
void or_supg_apply( int L, const double* coords, const double* radii, const double* vel, const double* src, double* dst,
                    double kappa, double dt, double mass_scaling, int lumped, int treat_boundary, int diag );

/* operators (Replace mode, additive communication) */
void or_kerngen_apply( int L, const double* coords, const double* radii, const double* k, const double* src,
                       double* dst, int bc_cmb, int bc_surf, int diag );
void or_kerngen_apply_copywise( int L, const double* coords, const double* radii, const double* k, const double* src,
                                double* dst, int bc_cmb, int bc_surf, int diag );
void or_laplace_apply( int L, const double* coords, const double* radii, const double* src, double* dst,
                       int treat_boundary, int diag );

/* EpsilonDivDiv, 3x2 rule, k interpolated; Dirichlet elimination on both radii */
void or_epsdivdiv3x2_apply( int L, const double* coords, const double* radii, const double* k, const double* src,
                            double* dst, int treat_boundary, int diag );
/* DivKGrad: int k grad u . grad v, k interpolated at the quadrature points;
 * single_quadpoint selects the 1-point rule */
void or_divkgrad_apply( int L, const double* coords, const double* radii, const double* k, const double* src,
                        double* dst, int treat_boundary, int diag, int single_quadpoint );
/* VectorLaplace on three components; bc codes 0 Neumann, 1 Dirichlet only
 * (returns -1 otherwise) */
int or_vector_laplace_apply( int L, const double* coords, const double* radii, const double* src, double* dst,
                             int bc_cmb, int bc_surf, int diag );

/* Stokes coupling blocks (fine velocity at level L, coarse pressure at L-1) */
void or_divergence_apply( int L, const double* coords, const double* radii, const double* coords_coarse,
                          const double* src_u, double* dst_p, int bc_cmb, int bc_surf );
void or_gradient_apply( int L, const double* coords, const double* radii, const double* src_p, double* dst_u,
                        int bc_cmb, int bc_surf );

/* KMass: mode 0 consistent, 1 diagonal, 2 lumped diagonal */
void or_kmass_apply( int L, const double* coords, const double* radii, const double* k, const double* src, double* dst,
                     int mode );

/* constant grid transfer of ncomp fields between levels Lc and Lc+1 */
void or_prolongation_constant( int Lc, int ncomp, const double* src_coarse, double* dst_fine );
void or_restriction_constant( int Lf, int ncomp, const double* coords_coarse, const uint8_t* omask_fine,
                              const double* src_fine, double* dst_coarse );

/* linear grid transfer of ncomp fields (coords / radii of the FINE mesh) */
void or_prolongation_linear( int Lc, int ncomp, const double* coords_fine, const double* radii_fine,
                             const double* src_coarse, double* dst_fine );
void or_restriction_linear( int Lf, int ncomp, const double* coords_fine, const double* radii_fine,
                            const double* coords_coarse, const uint8_t* omask_fine, const double* src_fine,
                            double* dst_coarse );

/* stored local matrices: [cell (d, x, y, r), r fastest][wedge][18][18],
 * DIMENSIONWISE (node + 6 dim), row-major */
void or_kerngen_local_matrices( int L, const double* coords, const double* radii, const double* k, double* mats );
/* GCA coarsening Lf -> Lf-1 from fine stored matrices (mats_fine) or, when
 * mats_fine is NULL, from the kerngen matrices of k_fine; mode 0 constant,
 * 1 linear interpolation */
void or_gca_coarsen( int Lf, const double* coords_f, const double* radii_f, const double* k_fine,
                     const double* mats_fine, int mode, double* mats_coarse );
/* apply with stored matrices and boundary treatment (+ fs/fs penalty) */
void or_stored_apply( int L, const double* coords, const double* radii, const double* mats, const double* src,
                      double* dst, int bc_cmb, int bc_surf, int diag );

/* finite-volume FCT on the hex cells: fields [10][N+2][N+2][N+2] with ghosts */
void   or_fv_ghost_update( int L, const double* coords, double* field );
void   or_fv_cell_centers( int L, const double* coords, const double* radii, double* centers );
double or_fct_dt_stable( int L, const double* coords, const double* radii, const double* centers, const double* vel,
                         double diffusivity );
void   or_fct_dirichlet( int L, double* T, double T_cmb, double T_surf, int apply_cmb, int apply_surf );
/* bcs: NULL or {T_cmb, T_surface, apply_cmb, apply_surface} */
void   or_fct_step( int L, const double* coords, const double* radii, const double* centers, const double* vel,
                    double* T, double dt, double diffusivity, const double* source, int subtract_divergence,
                    const double* bcs, double* T_L_out );

/* Krylov vector kernels */
double or_masked_dot( size_t n, const double* a, const double* b, const uint8_t* omask );

#ifdef __cplusplus
}
#endif
#endif
