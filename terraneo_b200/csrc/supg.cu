// SUPG-stabilised unsteady advection-diffusion operator (B200 design of
// UnsteadyAdvectionDiffusionSUPG, fe/wedge/operators/shell/
// unsteady_advection_diffusion_supg.hpp): the left-hand side
// mass_scaling M + dt (K + C + G) of an implicit BDF step for the temperature,
//   M_ij = int phi_i phi_j,  K_ij = int kappa grad phi_i . grad phi_j,
//   C_ij = int phi_i (u . grad phi_j),
//   G_ij = sum_E tau_E int_E (u . grad phi_i) (u . grad phi_j),
// on the 3x2 Felippa rule with the velocity interpolated at the quadrature
// points and tau_E the weight-averaged pointwise supg_tau of the wedge
// (h = r2 - r1; :16-50, :286-312).
//
// Matrix-free: instead of forming the 6 x 6 wedge matrices (:314-341) each
// quadrature point forms the source value s_q, its physical gradient gs and
// u . gs once, and every node's row follows as
//   ms phi_i s_q + dt (kappa grad phi_i . gs + phi_i u . gs + tau (u . grad phi_i)(u . gs)),
// O(6) per point instead of O(36).  The matrix modifications of the reference
// are expressed on that form: the lumped mass is ms phi_i per point times the
// node's own value; the boundary mask (off-diagonal entries of the rows and
// columns of CMB / surface nodes zeroed, :350-386) is the action on the source
// with those nodes zeroed for the other rows and the diagonal entry times the
// node's value for the boundary rows; the diagonal mode (:388-394) is the
// diagonal entries alone.
//
// One thread per fine wedge (the first half of the grid takes wedge 0 of every
// cell, the second half wedge 1: the wedge is uniform within a warp and the
// node offsets compile-time), lanes along r, node contributions added with
// atomics, then the additive halo sum.
#include <cmath>

#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

template < typename T >
struct SupgParams
{
    int             N, n1;
    const double*   coords;
    const T*        radii;
    Ptr3< const T > vel;
    const T*        src;
    T*              dst;
    T               kappa, dt, ms;
    int             lumped, treat, diag;
};

// 3x2 Felippa points (xi, eta, zeta); every weight 1/6
__device__ __forceinline__ double qp_xi( int q ) { return ( q % 3 ) == 0 ? 0.6666666666666666 : 0.1666666666666667; }
__device__ __forceinline__ double qp_eta( int q ) { return ( q % 3 ) == 1 ? 0.6666666666666666 : 0.1666666666666667; }
__device__ __forceinline__ double qp_zeta( int q ) { return q < 3 ? -0.5773502691896257 : 0.5773502691896257; }
constexpr double kSupgW = 0.1666666666666667;

template < typename T >
__device__ __forceinline__ T shape_at( int n, T xi, T eta, T zeta )
{
    const int m   = n % 3;
    const T   lat = m == 0 ? T( 1 ) - xi - eta : ( m == 1 ? xi : eta );
    return lat * ( n < 3 ? T( 0.5 ) * ( T( 1 ) - zeta ) : T( 0.5 ) * ( T( 1 ) + zeta ) );
}

// supg_tau (:16-50)
template < typename T >
__device__ __forceinline__ T supg_tau( T vel_norm, T kappa, T h )
{
    const T kv = kappa > T( 1e-8 ) ? kappa : T( 1e-8 );
    if ( vel_norm <= T( 1e-12 ) )
        return T( 0 );
    const T pe = vel_norm * h / ( T( 2 ) * kv );
    if ( pe <= T( 1e-8 ) )
        return T( 0 );
    const T tau_max = T( 10 ) * h / ( vel_norm > T( 1e-12 ) ? vel_norm : T( 1e-12 ) );
    const T coth    = T( 1 ) / tanh( pe ) - T( 1 ) / pe;
    const T tau     = ( h / ( T( 2 ) * vel_norm ) ) * coth;
    return tau > tau_max ? tau_max : tau;
}

template < typename T, int W >
__device__ __forceinline__ void supg_wedge( const SupgParams< T >& P, int d, int x, int y, int r )
{
    const int n1 = P.n1;
    T         p[3][3], s[6], v[6][3];
    size_t    id[6];
#pragma unroll
    for ( int n = 0; n < 6; ++n )
    {
        const size_t lat = lat_index( n1, d, x + wedge_node( W, n, 0 ), y + wedge_node( W, n, 1 ) );
        if ( n < 3 )
        {
#pragma unroll
            for ( int a = 0; a < 3; ++a )
                p[n][a] = T( P.coords[lat * 3 + a] );
        }
        id[n] = lat * n1 + r + wedge_node( W, n, 2 );
        s[n]  = P.src[id[n]];
#pragma unroll
        for ( int c = 0; c < 3; ++c )
            v[n][c] = P.vel.at( c )[id[n]];
    }
    const T r1 = P.radii[d * n1 + r], r2 = P.radii[d * n1 + r + 1];
    const T h  = r2 - r1;
    // tau: the weight-averaged pointwise value (:298-312)
    T tau_acc = 0, w_acc = 0;
#pragma unroll
    for ( int q = 0; q < 6; ++q )
    {
        const T xi = T( qp_xi( q ) ), eta = T( qp_eta( q ) ), zeta = T( qp_zeta( q ) );
        T       u[3] = { 0, 0, 0 };
#pragma unroll
        for ( int i = 0; i < 6; ++i )
        {
            const T sh = shape_at( i, xi, eta, zeta );
#pragma unroll
            for ( int c = 0; c < 3; ++c )
                u[c] += v[i][c] * sh;
        }
        tau_acc += supg_tau( sqrt( u[0] * u[0] + u[1] * u[1] + u[2] * u[2] ), P.kappa, h ) * T( kSupgW );
        w_acc += T( kSupgW );
    }
    const T tau = w_acc > T( 0 ) ? tau_acc / w_acc : T( 0 );

    const bool cmb = P.treat && r == 0, surf = P.treat && r == P.N - 1;
    const bool diag = P.diag != 0, lumped = P.lumped != 0;
    T          sm[6], out[6], dg[6];
#pragma unroll
    for ( int i = 0; i < 6; ++i )
    {
        const bool inB = ( cmb && i < 3 ) || ( surf && i >= 3 );
        sm[i]          = inB ? T( 0 ) : s[i];
        out[i] = dg[i] = T( 0 );
    }
    const bool need_dg = diag || cmb || surf;
#pragma unroll
    for ( int q = 0; q < 6; ++q )
    {
        const T xi = T( qp_xi( q ) ), eta = T( qp_eta( q ) ), zeta = T( qp_zeta( q ) );
        T       IT[3][3];
        const T ad = fabs( wedge_jacobian_it( p[0], p[1], p[2], r1, r2, xi, eta, zeta, IT ) ) * T( kSupgW );
        T       u[3] = { 0, 0, 0 }, g[6][3], sh[6];
#pragma unroll
        for ( int i = 0; i < 6; ++i )
        {
            sh[i] = shape_at( i, xi, eta, zeta );
            T gr[3];
            grad_shape_ref( i, xi, eta, zeta, gr );
#pragma unroll
            for ( int a = 0; a < 3; ++a )
                g[i][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
#pragma unroll
            for ( int c = 0; c < 3; ++c )
                u[c] += v[i][c] * sh[i];
        }
        if ( !diag )
        {
            T sq = 0, gs[3] = { 0, 0, 0 };
#pragma unroll
            for ( int j = 0; j < 6; ++j )
            {
                sq += sh[j] * sm[j];
#pragma unroll
                for ( int a = 0; a < 3; ++a )
                    gs[a] += g[j][a] * sm[j];
            }
            const T ugs = u[0] * gs[0] + u[1] * gs[1] + u[2] * gs[2];
#pragma unroll
            for ( int i = 0; i < 6; ++i )
            {
                const T ugi  = u[0] * g[i][0] + u[1] * g[i][1] + u[2] * g[i][2];
                const T gigs = g[i][0] * gs[0] + g[i][1] * gs[1] + g[i][2] * gs[2];
                const T mass = lumped ? P.ms * sh[i] * sm[i] : P.ms * sh[i] * sq;
                out[i] += ad * ( mass + P.dt * ( P.kappa * gigs + sh[i] * ugs + tau * ugi * ugs ) );
            }
        }
        if ( need_dg )
        {
#pragma unroll
            for ( int i = 0; i < 6; ++i )
            {
                const T ugi = u[0] * g[i][0] + u[1] * g[i][1] + u[2] * g[i][2];
                const T gg  = g[i][0] * g[i][0] + g[i][1] * g[i][1] + g[i][2] * g[i][2];
                const T mii = lumped ? P.ms * sh[i] : P.ms * sh[i] * sh[i];
                dg[i] += ad * ( mii + P.dt * ( P.kappa * gg + sh[i] * ugi + tau * ugi * ugi ) );
            }
        }
    }
#pragma unroll
    for ( int i = 0; i < 6; ++i )
    {
        const bool inB = ( cmb && i < 3 ) || ( surf && i >= 3 );
        atomicAdd( P.dst + id[i], ( diag || inB ) ? dg[i] * s[i] : out[i] );
    }
}

template < typename T >
__global__ void __launch_bounds__( 128 ) supg_kernel( SupgParams< T > P )
{
    const long long N = P.N, cells = 10LL * N * N * N;
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= 2 * cells )
        return;
    const long long c = t < cells ? t : t - cells;
    const int       r = int( c % N ), y = int( ( c / N ) % N ), x = int( ( c / ( N * N ) ) % N ), d = int( c / ( N * N * N ) );
    if ( t < cells )
        supg_wedge< T, 0 >( P, d, x, y, r );
    else
        supg_wedge< T, 1 >( P, d, x, y, r );
}

template < typename T >
int supg_apply( const tn_mesh* m, const T* const* vel, double kappa, double dt, double mass_scaling, int lumped,
                int treat_boundary, int diagonal, int apply_mode, int comm_mode, const T* src, T* dst, void* s )
{
    TN_CHECK_ARG( m && vel && vel[0] && vel[1] && vel[2] && src && dst, "supg apply: null argument" );
    TN_CHECK_ARG( apply_mode == TN_APPLY_REPLACE || apply_mode == TN_APPLY_ADD, "supg apply: bad apply mode" );
    TN_CHECK_ARG( comm_mode == TN_COMM_SKIP || comm_mode == TN_COMM_ADDITIVE, "supg apply: bad communication mode" );
    cudaStream_t st = as_stream( s );
    if ( apply_mode == TN_APPLY_REPLACE )
        TN_CUDA_TRY( cudaMemsetAsync( dst, 0, m->ns * sizeof( T ), st ) );
    SupgParams< T > P;
    P.N = m->N, P.n1 = m->n1, P.coords = m->d_coords;
    P.radii = sizeof( T ) == 8 ? reinterpret_cast< const T* >( m->d_radii ) : reinterpret_cast< const T* >( m->d_radii32 );
    P.vel   = Ptr3< const T >{ { vel[0], vel[1], vel[2] } };
    P.src = src, P.dst = dst;
    P.kappa = T( kappa ), P.dt = T( dt ), P.ms = T( mass_scaling );
    P.lumped = lumped != 0, P.treat = treat_boundary != 0, P.diag = diagonal != 0;
    const long long cells = 10LL * m->N * m->N * m->N;
    supg_kernel< T ><<< unsigned( ( 2 * cells + 127 ) / 128 ), 128, 0, st >>>( P );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( m, &dst, 1, st );
    return TN_OK;
}

}  // namespace
}  // namespace tn

using namespace tn;

extern "C" int tn_supg_apply_f64( const tn_mesh* m, const double* const* vel, double kappa, double dt,
                                  double mass_scaling, int lumped_mass, int treat_boundary, int diagonal, int apply_mode,
                                  int comm_mode, const double* src, double* dst, void* stream )
{
    return supg_apply< double >( m, vel, kappa, dt, mass_scaling, lumped_mass, treat_boundary, diagonal, apply_mode,
                                 comm_mode, src, dst, stream );
}

extern "C" int tn_supg_apply_f32( const tn_mesh* m, const float* const* vel, double kappa, double dt, double mass_scaling,
                                  int lumped_mass, int treat_boundary, int diagonal, int apply_mode, int comm_mode,
                                  const float* src, float* dst, void* stream )
{
    return supg_apply< float >( m, vel, kappa, dt, mass_scaling, lumped_mass, treat_boundary, diagonal, apply_mode,
                                comm_mode, src, dst, stream );
}

#include "../cpp/tn/operators.hpp"
#include "../cpp/tn/solvers.hpp"

extern "C" int tn_supg_solve_f64( const tn_mesh* m, const double* const* vel, double kappa, double dt,
                                  double mass_scaling, int lumped_mass, int treat_boundary, const double* rhs, double* x,
                                  int l, int max_iterations, double relative_tolerance, double absolute_tolerance,
                                  double* work, int* iterations, double* relative_residual, void* s )
{
    TN_CHECK_ARG( m && vel && vel[0] && vel[1] && vel[2] && rhs && x && work, "tn_supg_solve_f64: null argument" );
    TN_CHECK_ARG( l >= 1 && l <= 8 && max_iterations >= 1, "tn_supg_solve_f64: bad solver parameters" );
    cudaStream_t st = as_stream( s );
    const size_t ns = m->ns;
    try
    {
        struct StreamScope // the C++ layer issues on tn::stream(): this call's stream for its duration
        {
            cudaStream_t prev;
            explicit StreamScope( cudaStream_t s ) : prev( stream_ref() ) { stream_ref() = s; }
            ~StreamScope() { stream_ref() = prev; }
        } scope( st );
        Mesh                     mesh = Mesh::wrap( m );
        VectorQ1Scalar< double > b( mesh, const_cast< double* >( rhs ) ), xx( mesh, x );
        // the velocity as a non-owning view of its three contiguous components
        TN_CHECK_ARG( vel[1] == vel[0] + ns && vel[2] == vel[0] + 2 * ns,
                      "tn_supg_solve_f64: the velocity components must be one contiguous [3][nodes] array" );
        VectorQ1Vec< double > u( mesh, const_cast< double* >( vel[0] ) );
        std::vector< VectorQ1Scalar< double > > tmps;
        for ( int i = 0; i < 2 * ( l + 1 ) + 2; ++i )
            tmps.emplace_back( mesh, work + size_t( i ) * ns );
        UnsteadyAdvectionDiffusionSUPG< double > A( mesh, u, kappa, dt, treat_boundary != 0, false, mass_scaling,
                                                    lumped_mass != 0 );
        PBiCGStab< UnsteadyAdvectionDiffusionSUPG< double > > solver(
            l, IterativeSolverParameters{ max_iterations, relative_tolerance, absolute_tolerance }, tmps );
        solve( solver, A, xx, b );
        if ( iterations )
            *iterations = solver.stats.iterations;
        if ( relative_residual )
            *relative_residual = solver.stats.relative_residuals.empty() ? 0.0 : solver.stats.relative_residuals.back();
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_supg_solve_f64: " ) + e.what() );
        return TN_ERR_CUDA;
    }
    return TN_OK;
}
