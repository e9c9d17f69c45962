// Pieces of the mantle-circulation time step around the Stokes solve and the
// FCT step (apps/mantlecirculation/mantlecirculation.cpp:870-1045):
//  * the FV -> FE transfers (fv/hex/conversion.hpp:131-260): the right-hand
//    side b_i = sum_K T_K int_K phi_i of the L2 projection, solved with the
//    unpreconditioned PCG on the Q1 mass matrix (consistent form) or divided by
//    the lumped diagonal D_i = sum_K int_K phi_i (lumped form);
//  * the Stokes buoyancy right-hand side f = M (Ra T n) (RHSVelocityInterpolator,
//    mantlecirculation.cpp:117-150, then VectorMass and the strong Dirichlet /
//    free-slip enforcement, :883-899);
//  * the pressure normalisation p -= sum_owned p / (unique pressure nodes)
//    (:930-936).
#include <cmath>

#include "../cpp/tn/operators.hpp"
#include "../cpp/tn/solvers.hpp"
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

constexpr int kTsThreads = 128;

__device__ __forceinline__ size_t fv_idx( int n2, int d, int x, int y, int r )
{
    return ( ( size_t( d ) * n2 + x ) * n2 + y ) * n2 + r;
}

// One thread per FV cell (x, y, r in 1..N, the FE cell (x-1, y-1, r-1)).  The
// reference integrates shape_i |det J| with the 3x2 Felippa rule (6 points,
// weights 1/6; conversion.hpp:150-188).  On the wedge map |det J| =
// r(zeta)^2 h |(a x b) . p0| (h = (r2 - r1) / 2, a = p1 - p0, b = p2 - p0) and
// each lateral shape function sums to 1 over the rule's three lateral points,
// so the integral of a bottom (top) node function is
// h |D| / 6 (r(-g)^2 (1 + g) / 2 + r(g)^2 (1 - g) / 2)   (g and -g swapped
// for top), g = 0.5773502691896257: the same sums in closed form.
__global__ void __launch_bounds__( kTsThreads ) fv_to_fe_rhs_kernel( int N, const double* __restrict__ coords,
                                                                     const double* __restrict__ radii,
                                                                     const double* __restrict__ fv, double* b,
                                                                     double* D )
{
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int    r = int( t % N ) + 1, y = int( ( t / N ) % N ) + 1, x = int( ( t / ( (long long) N * N ) ) % N ) + 1;
    const int    d  = int( t / ( (long long) N * N * N ) );
    const int    n1 = N + 1, n2 = N + 2;
    const double g  = 0.5773502691896257;
    const double r1 = radii[d * n1 + r - 1], r2 = radii[d * n1 + r];
    const double h  = 0.5 * ( r2 - r1 );
    const double rm = r1 + h * ( 1.0 - g ), rp = r1 + h * ( 1.0 + g );
    const double Ib = ( rm * rm * 0.5 * ( 1.0 + g ) + rp * rp * 0.5 * ( 1.0 - g ) ) * 0.1666666666666667;
    const double It = ( rm * rm * 0.5 * ( 1.0 - g ) + rp * rp * 0.5 * ( 1.0 + g ) ) * 0.1666666666666667;
    const double v  = fv ? fv[fv_idx( n2, d, x, y, r )] : 0.0;
    for ( int w = 0; w < 2; ++w )
    {
        double p[3][3];
        for ( int i = 0; i < 3; ++i )
        {
            const size_t lat = lat_index( n1, d, x - 1 + kWedgeNode[w][i][0], y - 1 + kWedgeNode[w][i][1] );
            for ( int a = 0; a < 3; ++a )
                p[i][a] = coords[lat * 3 + a];
        }
        const double a0 = p[1][0] - p[0][0], a1 = p[1][1] - p[0][1], a2 = p[1][2] - p[0][2];
        const double b0 = p[2][0] - p[0][0], b1 = p[2][1] - p[0][1], b2 = p[2][2] - p[0][2];
        const double Dw = ( a1 * b2 - a2 * b1 ) * p[0][0] + ( a2 * b0 - a0 * b2 ) * p[0][1] + ( a0 * b1 - a1 * b0 ) * p[0][2];
        const double hd = h * fabs( Dw );
        for ( int i = 0; i < 6; ++i )
        {
            const size_t id = lat_index( n1, d, x - 1 + kWedgeNode[w][i][0], y - 1 + kWedgeNode[w][i][1] ) * n1 + r - 1 +
                              kWedgeNode[w][i][2];
            const double I = hd * ( i < 3 ? Ib : It );
            if ( b )
                atomicAdd( b + id, I * v );
            if ( D )
                atomicAdd( D + id, I );
        }
    }
}

__global__ void divide_kernel( size_t n, const double* __restrict__ num, const double* __restrict__ den, double* out )
{
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < n; i += size_t( gridDim.x ) * blockDim.x )
        out[i] = num[i] / den[i];
}

// g = Ra T n at every stored node, n the unit radial direction of the node
// (RHSVelocityInterpolator, mantlecirculation.cpp:136-149)
__global__ void buoyancy_kernel( size_t ns, int n1, const double* __restrict__ coords, const double* __restrict__ T,
                                 double ra, Ptr3< double > g )
{
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        const size_t  lat = i / size_t( n1 );
        const double* u   = coords + lat * 3;
        const double  nn  = sqrt( u[0] * u[0] + u[1] * u[1] + u[2] * u[2] );
        const double  s   = ra * T[i] / nn;
        g.p[0][i]         = s * u[0];
        g.p[1][i]         = s * u[1];
        g.p[2][i]         = s * u[2];
    }
}

// One thread per FV cell: the cell average of the FE field over the hex cell's two wedges,
// sum_w sum_i u_i int phi_i |det J| / sum_w int |det J| with the closed-form node integrals of
// fv_to_fe_rhs_kernel (the reference evaluates the same integrals with the 3x2 rule, conversion.hpp:371-411)
__global__ void __launch_bounds__( kTsThreads ) fe_to_fv_kernel( int N, const double* __restrict__ coords,
                                                                 const double* __restrict__ radii,
                                                                 const double* __restrict__ fe, double* fv )
{
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int    r = int( t % N ) + 1, y = int( ( t / N ) % N ) + 1, x = int( ( t / ( (long long) N * N ) ) % N ) + 1;
    const int    d  = int( t / ( (long long) N * N * N ) );
    const int    n1 = N + 1, n2 = N + 2;
    const double g  = 0.5773502691896257;
    const double r1 = radii[d * n1 + r - 1], r2 = radii[d * n1 + r];
    const double h  = 0.5 * ( r2 - r1 );
    const double rm = r1 + h * ( 1.0 - g ), rp = r1 + h * ( 1.0 + g );
    const double Ib = ( rm * rm * 0.5 * ( 1.0 + g ) + rp * rp * 0.5 * ( 1.0 - g ) ) * 0.1666666666666667;
    const double It = ( rm * rm * 0.5 * ( 1.0 - g ) + rp * rp * 0.5 * ( 1.0 + g ) ) * 0.1666666666666667;
    double       integral = 0.0, volume = 0.0;
    for ( int w = 0; w < 2; ++w )
    {
        double p[3][3];
        size_t lat[3];
        for ( int i = 0; i < 3; ++i )
        {
            lat[i] = lat_index( n1, d, x - 1 + kWedgeNode[w][i][0], y - 1 + kWedgeNode[w][i][1] );
            for ( int a = 0; a < 3; ++a )
                p[i][a] = coords[lat[i] * 3 + a];
        }
        const double a0 = p[1][0] - p[0][0], a1 = p[1][1] - p[0][1], a2 = p[1][2] - p[0][2];
        const double b0 = p[2][0] - p[0][0], b1 = p[2][1] - p[0][1], b2 = p[2][2] - p[0][2];
        const double Dw = ( a1 * b2 - a2 * b1 ) * p[0][0] + ( a2 * b0 - a0 * b2 ) * p[0][1] + ( a0 * b1 - a1 * b0 ) * p[0][2];
        const double hd = h * fabs( Dw );
        double       sb = 0.0, st = 0.0;
        for ( int i = 0; i < 3; ++i )
        {
            sb += fe[lat[i] * n1 + r - 1];
            st += fe[lat[i] * n1 + r];
        }
        integral += hd * ( Ib * sb + It * st );
        volume += hd * 3.0 * ( Ib + It );
    }
    fv[fv_idx( n2, d, x, y, r )] = integral / volume;
}

unsigned blocks_for( size_t n ) { return unsigned( std::min< size_t >( ( n + 255 ) / 256, 148 * 8 ) ); }

}  // namespace
}  // namespace tn

using namespace tn;

extern "C" int tn_fv_to_fe_rhs_f64( const tn_mesh* m, const double* fv, double* b, double* lumped_diagonal, void* s )
{
    TN_CHECK_ARG( m && ( b || lumped_diagonal ) && ( fv || !b ), "tn_fv_to_fe_rhs_f64: bad arguments" );
    cudaStream_t    st    = as_stream( s );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    if ( b )
        TN_CUDA_TRY( cudaMemsetAsync( b, 0, sizeof( double ) * m->ns, st ) );
    if ( lumped_diagonal )
        TN_CUDA_TRY( cudaMemsetAsync( lumped_diagonal, 0, sizeof( double ) * m->ns, st ) );
    fv_to_fe_rhs_kernel<<< unsigned( ( cells + kTsThreads - 1 ) / kTsThreads ), kTsThreads, 0, st >>>(
        m->N, m->d_coords, m->d_radii, fv, b, lumped_diagonal );
    TN_LAUNCH_CHECK();
    // contributions of the other diamonds' copies (communication::shell::send_recv)
    double* f[2] = { b, lumped_diagonal };
    for ( int i = 0; i < 2; ++i )
        if ( f[i] )
        {
            int rc = halo_sum< double >( m, &f[i], 1, st );
            if ( rc )
                return rc;
        }
    return TN_OK;
}

// dst (FE scalar) from the FV field src (with ghost layers):
// lumped != 0: l2_project_fv_to_fe_lumped (conversion.hpp:243-300), dst = b / D;
// lumped == 0: l2_project_fv_to_fe (conversion.hpp:131-205), the Q1 mass system M dst = b solved by the
// unpreconditioned PCG from dst's entry values (the reference passes 1000, 1e-12, 1e-12).
// work: 5 stored-node fields (consistent) or 2 (lumped).
extern "C" int tn_l2_project_fv_to_fe_f64( const tn_mesh* m, const double* src, double* dst, int lumped,
                                           int max_iterations, double relative_tolerance, double absolute_tolerance,
                                           double* work, int* iterations, void* s )
{
    TN_CHECK_ARG( m && src && dst && work, "tn_l2_project_fv_to_fe_f64: null argument" );
    cudaStream_t st = as_stream( s );
    const size_t ns = m->ns;
    if ( lumped )
    {
        int rc = tn_fv_to_fe_rhs_f64( m, src, work, work + ns, s );
        if ( rc )
            return rc;
        divide_kernel<<< blocks_for( ns ), 256, 0, st >>>( ns, work, work + ns, dst );
        TN_LAUNCH_CHECK();
        if ( iterations )
            *iterations = 0;
        return TN_OK;
    }
    int rc = tn_fv_to_fe_rhs_f64( m, src, work, nullptr, s );
    if ( rc )
        return rc;
    try
    {
        struct StreamScope // the C++ layer issues on tn::stream(): this call's stream for its duration
        {
            cudaStream_t prev;
            explicit StreamScope( cudaStream_t s ) : prev( stream_ref() ) { stream_ref() = s; }
            ~StreamScope() { stream_ref() = prev; }
        } scope( st );
        Mesh                              mesh = Mesh::wrap( m );
        VectorQ1Scalar< double >          b( mesh, work ), x( mesh, dst ), none;
        std::vector< VectorQ1Scalar< double > > tmps;
        for ( int i = 1; i <= 4; ++i )
            tmps.emplace_back( mesh, work + i * ns );
        KMass< double > M( mesh, none, 0 );
        PCG< KMass< double > > pcg( IterativeSolverParameters{ max_iterations, relative_tolerance, absolute_tolerance },
                                    tmps );
        solve( pcg, M, x, b );
        if ( iterations )
            *iterations = pcg.stats.iterations;
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_l2_project_fv_to_fe_f64: " ) + e.what() );
        return TN_ERR_CUDA;
    }
    return TN_OK;
}

// f = VectorMass (Ra T n) with n the unit radial direction (mantlecirculation.cpp:117-150, 883-886), then the
// velocity rows of Dirichlet boundaries zeroed (strong_algebraic_homogeneous_velocity_dirichlet_enforcement_
// stokes_like, strong_algebraic_dirichlet_enforcement.hpp:115-124) and the normal component removed on
// free-slip boundaries (strong_algebraic_freeslip_enforcement_in_place, strong_algebraic_freeslip_enforcement.hpp:23).
// T: FE scalar on the velocity mesh; work: 3 stored-node fields.
extern "C" int tn_stokes_buoyancy_rhs_f64( const tn_mesh* m, const double* T, double rayleigh, int bc_cmb,
                                           int bc_surface, double* const* f_u, double* work, void* s )
{
    TN_CHECK_ARG( m && T && f_u && f_u[0] && f_u[1] && f_u[2] && work, "tn_stokes_buoyancy_rhs_f64: null argument" );
    TN_CHECK_ARG( bc_cmb >= 0 && bc_cmb <= 2 && bc_surface >= 0 && bc_surface <= 2,
                  "tn_stokes_buoyancy_rhs_f64: boundary condition codes must be 0, 1 or 2" );
    cudaStream_t   st = as_stream( s );
    const size_t   ns = m->ns;
    Ptr3< double > g{ { work, work + ns, work + 2 * ns } };
    buoyancy_kernel<<< blocks_for( ns ), 256, 0, st >>>( ns, m->n1, m->d_coords, T, rayleigh, g );
    TN_LAUNCH_CHECK();
    for ( int c = 0; c < 3; ++c )
    {
        int rc = tn_kmass_apply_f64( m, nullptr, 0, TN_APPLY_REPLACE, TN_COMM_ADDITIVE, g.p[c], f_u[c], s );
        if ( rc )
            return rc;
    }
    // as the app calls the enforcement: each condition on the boundary get_shell_boundary_flag names, the first
    // with that condition (CMB before SURFACE, grid/shell/bit_masks.hpp:68-76), so with the same condition on
    // both radii only the CMB rows are treated
    const int dir_cmb = bc_cmb == TN_BC_DIRICHLET, dir_surf = !dir_cmb && bc_surface == TN_BC_DIRICHLET;
    if ( dir_cmb || dir_surf )
    {
        int rc = tn_vec_assign_boundary_f64( m, 3, f_u, nullptr, 0.0, dir_cmb, dir_surf, s );
        if ( rc )
            return rc;
    }
    const int fs_cmb = bc_cmb == TN_BC_FREESLIP, fs_surf = !fs_cmb && bc_surface == TN_BC_FREESLIP;
    if ( fs_cmb || fs_surf )
        return tn_freeslip_project_f64( m, f_u, fs_cmb, fs_surf, s );
    return TN_OK;
}

// p -= (sum over owned nodes of p) / (unique nodes of the mesh) (mantlecirculation.cpp:930-936); work: one
// stored-node field; mean (optional) receives the subtracted value.  Synchronises (the sum is read back).
extern "C" int tn_pressure_remove_mean_f64( const tn_mesh* m, double* p, double* work, double* mean, void* s )
{
    TN_CHECK_ARG( m && p && work, "tn_pressure_remove_mean_f64: null argument" );
    double* one[1] = { work };
    int     rc     = tn_vec_lincomb_f64( m, 1, one, 1.0, 0, nullptr, nullptr, s );
    if ( rc )
        return rc;
    const double* a[1] = { p };
    const double* b[1] = { work };
    double        sum  = 0.0;
    if ( ( rc = tn_vec_dot_f64( m, 1, a, b, &sum, s ) ) )
        return rc;
    const double avg   = sum / double( m->nu );
    double*      y[1]  = { p };
    const double c1[1] = { 1.0 };
    const double* x[1] = { p };
    if ( ( rc = tn_vec_lincomb_f64( m, 1, y, -avg, 1, c1, x, s ) ) )
        return rc;
    if ( mean )
        *mean = avg;
    return TN_OK;
}

// FV cell averages of an FE scalar (l2_project_fe_to_fv, fv/hex/conversion.hpp:349-416), then the lateral
// FV ghost layers
extern "C" int tn_l2_project_fe_to_fv_f64( const tn_mesh* m, const double* fe, double* fv, void* s )
{
    TN_CHECK_ARG( m && fe && fv, "tn_l2_project_fe_to_fv_f64: null argument" );
    cudaStream_t    st    = as_stream( s );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    fe_to_fv_kernel<<< unsigned( ( cells + kTsThreads - 1 ) / kTsThreads ), kTsThreads, 0, st >>>(
        m->N, m->d_coords, m->d_radii, fe, fv );
    TN_LAUNCH_CHECK();
    return tn_fv_ghost_update_f64( m, fv, s );
}
