// Stokes coupling blocks: Divergence B (fine P1 velocity -> coarse P1
// pressure, fe/wedge/operators/shell/divergence.hpp) and Gradient B^T
// (gradient.hpp), Q1-iso-Q2 / Q1 with the 3x2 Felippa rule.
//
// B_{i,(d,j)} = -int (J^{-T} grad N_j)_d N^c_i |det J| over each fine wedge,
// N^c_i the coarse shape functions of the coarse wedge containing it
// (shape_coarse, integrands.hpp:266-400).  The coarse node each wedge-local
// coarse slot is added to follows the reference's wedge map
// (atomically_add_local_wedge_scalar_coefficients, kernel_helpers.hpp:407):
// fine wedge w always scatters to coarse wedge w's node positions, also for
// the two middle fine triangles whose shape functions belong to the other
// coarse wedge.  Kept as is for parity; Gradient uses the same map, so B^T is
// the exact transpose.
//
// Boundary conditions act on the velocity side: Dirichlet nodes are dropped,
// free-slip nodes are projected onto the tangent plane (the reference's
// rotate / eliminate-normal / rotate-back sequence, :226-290).
//
// One thread per fine cell (r fastest), both wedges, contributions summed per
// node in registers and added with atomics.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

__device__ __constant__ const double kQP[6][3] = { { 0.6666666666666666, 0.1666666666666667, -0.5773502691896257 },
                                                   { 0.1666666666666667, 0.6666666666666666, -0.5773502691896257 },
                                                   { 0.1666666666666667, 0.1666666666666667, -0.5773502691896257 },
                                                   { 0.6666666666666666, 0.1666666666666667, 0.5773502691896257 },
                                                   { 0.1666666666666667, 0.6666666666666666, 0.5773502691896257 },
                                                   { 0.1666666666666667, 0.1666666666666667, 0.5773502691896257 } };
constexpr double kQW = 0.1666666666666667;

// coarse lateral shape coefficients (a, b xi, c eta) per [node % 3][fine lateral wedge index]
__device__ __constant__ const double kCoarseLat[3][4][3] = {
    { { 1.0, -0.5, -0.5 }, { 0.5, -0.5, -0.5 }, { 0.5, -0.5, -0.5 }, { 0.0, 0.5, 0.5 } },
    { { 0.0, 0.5, 0.0 }, { 0.5, 0.5, 0.0 }, { 0.0, 0.5, 0.0 }, { 0.5, -0.5, 0.0 } },
    { { 0.0, 0.0, 0.5 }, { 0.0, 0.0, 0.5 }, { 0.5, 0.0, 0.5 }, { 0.5, 0.0, -0.5 } } };

template < typename T >
__device__ __forceinline__ T shape_coarse( int i, int frad, int flat, T xi, T eta, T zeta )
{
    const T lat = T( kCoarseLat[i % 3][flat][0] ) + T( kCoarseLat[i % 3][flat][1] ) * xi +
                  T( kCoarseLat[i % 3][flat][2] ) * eta;
    T rad;
    if ( i < 3 )
        rad = frad == 0 ? T( 0.25 ) * ( T( 3 ) - zeta ) : T( 0.25 ) * ( T( 1 ) - zeta );
    else
        rad = frad == 0 ? T( 0.25 ) * ( T( 1 ) + zeta ) : T( 0.25 ) * ( T( 3 ) + zeta );
    return lat * rad;
}

__device__ __forceinline__ int fine_lateral_wedge( int x, int y, int w )
{
    // fine_lateral_wedge_idx (kernel_helpers.hpp:601)
    const int xm = x & 1, ym = y & 1;
    return w == 0 ? ( ym * 2 + xm ) : ( 3 - ( ym * 2 + xm ) );
}

template < typename T >
struct StokesParams
{
    int           N, n1, nc1;
    const double* coords; // fine lateral coords
    const T*      radii;  // fine radii
    int           bc_cmb, bc_surf;
};

// 0: interior, 1: Dirichlet (drop), 2: free-slip (project)
__device__ __forceinline__ int velocity_bc( int N, int r, int n, int bc_cmb, int bc_surf )
{
    if ( r == 0 && n < 3 )
        return bc_cmb;
    if ( r == N - 1 && n >= 3 )
        return bc_surf;
    return 0;
}

template < typename T >
__device__ __forceinline__ void unit_normal( const double* c, T n[3] )
{
    double m = sqrt( c[0] * c[0] + c[1] * c[1] + c[2] * c[2] );
    n[0] = T( c[0] / m ), n[1] = T( c[1] / m ), n[2] = T( c[2] / m );
}

// Quadrature data of one fine wedge: for lateral point ql and radial point
// qz, J = M(ql) diag(r(qz), r(qz), dr/2) with M = [p1-p0, p2-p0, p(xi,eta)], so
// J^{-T} = M^{-T} diag(1/r, 1/r, 2/dr) and |det J| = |det M| r^2 dr/2: one 3x3
// inverse per lateral point serves both radial points.  Calls f(q, wdet, g, xi,
// eta, zeta) with g the 6 physical shape gradients.
template < typename T, typename F >
__device__ __forceinline__ void for_each_qp( const T p[3][3], T r1, T r2, F&& f )
{
    const T dr = T( 0.5 ) * ( r2 - r1 );
#pragma unroll 1
    for ( int ql = 0; ql < 3; ++ql )
    {
        const T xi = T( kQP[ql][0] ), eta = T( kQP[ql][1] );
        T       M[3][3];
#pragma unroll
        for ( int a = 0; a < 3; ++a )
        {
            M[a][0] = p[1][a] - p[0][a];
            M[a][1] = p[2][a] - p[0][a];
            M[a][2] = ( T( 1 ) - xi - eta ) * p[0][a] + xi * p[1][a] + eta * p[2][a];
        }
        const T c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1], c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2],
                c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
        const T det = M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02;
        const T id  = T( 1 ) / det;
        // Q = M^{-T}
        T Q[3][3];
        Q[0][0] = c00 * id, Q[0][1] = c01 * id, Q[0][2] = c02 * id;
        Q[1][0] = ( M[0][2] * M[2][1] - M[0][1] * M[2][2] ) * id;
        Q[1][1] = ( M[0][0] * M[2][2] - M[0][2] * M[2][0] ) * id;
        Q[1][2] = ( M[0][1] * M[2][0] - M[0][0] * M[2][1] ) * id;
        Q[2][0] = ( M[0][1] * M[1][2] - M[0][2] * M[1][1] ) * id;
        Q[2][1] = ( M[0][2] * M[1][0] - M[0][0] * M[1][2] ) * id;
        Q[2][2] = ( M[0][0] * M[1][1] - M[0][1] * M[1][0] ) * id;
#pragma unroll
        for ( int qz = 0; qz < 2; ++qz )
        {
            const int q    = ql + 3 * qz;
            const T   zeta = T( kQP[q][2] );
            const T   rq   = r1 + dr * ( T( 1 ) + zeta );
            const T   s0 = T( 1 ) / rq, s2 = T( 1 ) / dr;
            const T   wdet = T( kQW ) * fabs( det ) * rq * rq * dr;
            T         g[6][3];
#pragma unroll
            for ( int n = 0; n < 6; ++n )
            {
                T gr[3];
                grad_shape_ref( n, xi, eta, zeta, gr );
                gr[0] *= s0, gr[1] *= s0, gr[2] *= s2;
#pragma unroll
                for ( int a = 0; a < 3; ++a )
                    g[n][a] = Q[a][0] * gr[0] + Q[a][1] * gr[1] + Q[a][2] * gr[2];
            }
            f( q, wdet, g, xi, eta, zeta );
        }
    }
}

template < typename T >
__device__ __forceinline__ void wedge_points( const StokesParams< T >& P, int dm, int x, int y, int w, T p[3][3] )
{
#pragma unroll
    for ( int n = 0; n < 3; ++n )
    {
        const double* c = P.coords + lat_index( P.n1, dm, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * 3;
        p[n][0] = T( c[0] ), p[n][1] = T( c[1] ), p[n][2] = T( c[2] );
    }
}

// p_coarse += B u: per quadrature point -w |det J| N^c_i div u
template < typename T >
__global__ void __launch_bounds__( 128 ) divergence_kernel( StokesParams< T > P, Ptr3< const T > u, T* __restrict__ p )
{
    const int       N = P.N, n1 = P.n1, nc1 = P.nc1;
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int r  = int( t % N );
    const int y  = int( ( t / N ) % N );
    const int x  = int( ( t / ( (long long) N * N ) ) % N );
    const int dm = int( t / ( (long long) N * N * N ) );
    T         out[2][2][2];
#pragma unroll
    for ( int i = 0; i < 8; ++i )
        out[i >> 2][( i >> 1 ) & 1][i & 1] = T( 0 );
    const T   r1 = P.radii[dm * n1 + r], r2 = P.radii[dm * n1 + r + 1];
    const int frad = r & 1;
#pragma unroll
    for ( int w = 0; w < 2; ++w )
    {
        T p3[3][3];
        wedge_points( P, dm, x, y, w, p3 );
        const int flat = fine_lateral_wedge( x, y, w );
        T         uu[6][3];
#pragma unroll
        for ( int n = 0; n < 6; ++n )
        {
            const int    X = x + kWedgeNode[w][n][0], Y = y + kWedgeNode[w][n][1];
            const size_t i = lat_index( n1, dm, X, Y ) * n1 + r + kWedgeNode[w][n][2];
            uu[n][0] = u.p[0][i], uu[n][1] = u.p[1][i], uu[n][2] = u.p[2][i];
            const int bc = velocity_bc( N, r, n, P.bc_cmb, P.bc_surf );
            if ( bc == TN_BC_DIRICHLET )
                uu[n][0] = uu[n][1] = uu[n][2] = T( 0 );
            else if ( bc == TN_BC_FREESLIP )
            {
                T nn[3];
                unit_normal( P.coords + lat_index( n1, dm, X, Y ) * 3, nn );
                const T dt = nn[0] * uu[n][0] + nn[1] * uu[n][1] + nn[2] * uu[n][2];
                uu[n][0] -= dt * nn[0], uu[n][1] -= dt * nn[1], uu[n][2] -= dt * nn[2];
            }
        }
        T acc[6] = { 0, 0, 0, 0, 0, 0 };
        for_each_qp( p3, r1, r2, [&]( int, T wdet, const T ( &g )[6][3], T xi, T eta, T zeta ) {
            T div = 0;
#pragma unroll
            for ( int n = 0; n < 6; ++n )
                div += g[n][0] * uu[n][0] + g[n][1] * uu[n][1] + g[n][2] * uu[n][2];
            const T s = -wdet * div;
#pragma unroll
            for ( int i = 0; i < 6; ++i )
                acc[i] += s * shape_coarse( i, frad, flat, xi, eta, zeta );
        } );
#pragma unroll
        for ( int i = 0; i < 6; ++i )
            out[kWedgeNode[w][i][0]][kWedgeNode[w][i][1]][kWedgeNode[w][i][2]] += acc[i];
    }
    const int xc = x >> 1, yc = y >> 1, rc = r >> 1;
#pragma unroll
    for ( int a = 0; a < 8; ++a )
    {
        const int dx = a >> 2, dy = ( a >> 1 ) & 1, dr = a & 1;
        atomicAdd( p + lat_index( nc1, dm, xc + dx, yc + dy ) * nc1 + rc + dr, out[dx][dy][dr] );
    }
}

// u_fine += B^T p: per quadrature point -w |det J| p^c(q) grad N_j
template < typename T >
__global__ void __launch_bounds__( 128 ) gradient_kernel( StokesParams< T > P, const T* __restrict__ p, Ptr3< T > u )
{
    const int       N = P.N, n1 = P.n1, nc1 = P.nc1;
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int r  = int( t % N );
    const int y  = int( ( t / N ) % N );
    const int x  = int( ( t / ( (long long) N * N ) ) % N );
    const int dm = int( t / ( (long long) N * N * N ) );
    T         out[2][2][2][3];
#pragma unroll
    for ( int i = 0; i < 8; ++i )
#pragma unroll
        for ( int c = 0; c < 3; ++c )
            out[i >> 2][( i >> 1 ) & 1][i & 1][c] = T( 0 );
    const int xc = x >> 1, yc = y >> 1, rc = r >> 1;
    const T   r1 = P.radii[dm * n1 + r], r2 = P.radii[dm * n1 + r + 1];
    const int frad = r & 1;
#pragma unroll
    for ( int w = 0; w < 2; ++w )
    {
        T p3[3][3];
        wedge_points( P, dm, x, y, w, p3 );
        const int flat = fine_lateral_wedge( x, y, w );
        T         pc[6];
#pragma unroll
        for ( int i = 0; i < 6; ++i )
            pc[i] = p[lat_index( nc1, dm, xc + kWedgeNode[w][i][0], yc + kWedgeNode[w][i][1] ) * nc1 + rc +
                      kWedgeNode[w][i][2]];
        T acc[6][3];
#pragma unroll
        for ( int n = 0; n < 6; ++n )
            acc[n][0] = acc[n][1] = acc[n][2] = T( 0 );
        for_each_qp( p3, r1, r2, [&]( int, T wdet, const T ( &g )[6][3], T xi, T eta, T zeta ) {
            T pq = 0;
#pragma unroll
            for ( int i = 0; i < 6; ++i )
                pq += shape_coarse( i, frad, flat, xi, eta, zeta ) * pc[i];
            const T s = -wdet * pq;
#pragma unroll
            for ( int n = 0; n < 6; ++n )
                acc[n][0] += s * g[n][0], acc[n][1] += s * g[n][1], acc[n][2] += s * g[n][2];
        } );
#pragma unroll
        for ( int j = 0; j < 6; ++j )
        {
            T         v[3] = { acc[j][0], acc[j][1], acc[j][2] };
            const int bc   = velocity_bc( N, r, j, P.bc_cmb, P.bc_surf );
            if ( bc == TN_BC_DIRICHLET )
                continue;
            if ( bc == TN_BC_FREESLIP )
            {
                T nn[3];
                unit_normal( P.coords + lat_index( n1, dm, x + kWedgeNode[w][j][0], y + kWedgeNode[w][j][1] ) * 3, nn );
                const T dt = nn[0] * v[0] + nn[1] * v[1] + nn[2] * v[2];
                v[0] -= dt * nn[0], v[1] -= dt * nn[1], v[2] -= dt * nn[2];
            }
            T* o = out[kWedgeNode[w][j][0]][kWedgeNode[w][j][1]][kWedgeNode[w][j][2]];
            o[0] += v[0], o[1] += v[1], o[2] += v[2];
        }
    }
#pragma unroll
    for ( int a = 0; a < 8; ++a )
    {
        const int    dx = a >> 2, dy = ( a >> 1 ) & 1, dr = a & 1;
        const size_t i  = lat_index( n1, dm, x + dx, y + dy ) * n1 + r + dr;
        atomicAdd( u.p[0] + i, out[dx][dy][dr][0] );
        atomicAdd( u.p[1] + i, out[dx][dy][dr][1] );
        atomicAdd( u.p[2] + i, out[dx][dy][dr][2] );
    }
}

template < typename T >
const T* radii_of( const tn_mesh* m )
{
    return sizeof( T ) == 8 ? reinterpret_cast< const T* >( m->d_radii ) : reinterpret_cast< const T* >( m->d_radii32 );
}

int check_pair( const tn_mesh* f, const tn_mesh* c )
{
    TN_CHECK_ARG( f && c, "stokes block: null mesh" );
    TN_CHECK_ARG( c->level == f->level - 1 && c->r_min == f->r_min && c->r_max == f->r_max,
                  "stokes block: the pressure mesh must be the velocity mesh coarsened once" );
    return TN_OK;
}

}  // namespace

template < typename T >
int divergence_apply( const tn_mesh* f, const tn_mesh* c, int bc_cmb, int bc_surf, int apply_mode, int comm_mode,
                      const T* const* u, T* p, cudaStream_t st )
{
    int rc;
    if ( ( rc = check_pair( f, c ) ) )
        return rc;
    TN_CHECK_ARG( u && u[0] && u[1] && u[2] && p, "divergence: null vector" );
    if ( apply_mode == TN_APPLY_REPLACE )
        TN_CUDA_TRY( cudaMemsetAsync( p, 0, c->ns * sizeof( T ), st ) );
    StokesParams< T > P{ f->N, f->n1, c->n1, f->d_coords, radii_of< T >( f ), bc_cmb, bc_surf };
    const long long   cells = (long long) kDiamonds * f->N * f->N * f->N;
    divergence_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( P, Ptr3< const T >{ { u[0], u[1], u[2] } },
                                                                                p );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
    {
        T* fl[1] = { p };
        return halo_sum< T >( c, fl, 1, st );
    }
    return TN_OK;
}

template < typename T >
int gradient_apply( const tn_mesh* f, const tn_mesh* c, int bc_cmb, int bc_surf, int apply_mode, int comm_mode,
                    const T* p, T* const* u, cudaStream_t st )
{
    int rc;
    if ( ( rc = check_pair( f, c ) ) )
        return rc;
    TN_CHECK_ARG( u && u[0] && u[1] && u[2] && p, "gradient: null vector" );
    if ( apply_mode == TN_APPLY_REPLACE )
        for ( int i = 0; i < 3; ++i )
            TN_CUDA_TRY( cudaMemsetAsync( u[i], 0, f->ns * sizeof( T ), st ) );
    StokesParams< T > P{ f->N, f->n1, c->n1, f->d_coords, radii_of< T >( f ), bc_cmb, bc_surf };
    const long long   cells = (long long) kDiamonds * f->N * f->N * f->N;
    gradient_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( P, p, Ptr3< T >{ { u[0], u[1], u[2] } } );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( f, u, 3, st );
    return TN_OK;
}

template int divergence_apply< double >( const tn_mesh*, const tn_mesh*, int, int, int, int, const double* const*,
                                         double*, cudaStream_t );
template int divergence_apply< float >( const tn_mesh*, const tn_mesh*, int, int, int, int, const float* const*,
                                        float*, cudaStream_t );
template int gradient_apply< double >( const tn_mesh*, const tn_mesh*, int, int, int, int, const double*,
                                       double* const*, cudaStream_t );
template int gradient_apply< float >( const tn_mesh*, const tn_mesh*, int, int, int, int, const float*, float* const*,
                                      cudaStream_t );

}  // namespace tn

using namespace tn;

extern "C" int tn_divergence_apply_f64( const tn_mesh* f, const tn_mesh* c, int bcc, int bcs, int am, int cm,
                                        const double* const* u, double* p, void* s )
{
    return divergence_apply< double >( f, c, bcc, bcs, am, cm, u, p, as_stream( s ) );
}
extern "C" int tn_divergence_apply_f32( const tn_mesh* f, const tn_mesh* c, int bcc, int bcs, int am, int cm,
                                        const float* const* u, float* p, void* s )
{
    return divergence_apply< float >( f, c, bcc, bcs, am, cm, u, p, as_stream( s ) );
}
extern "C" int tn_gradient_apply_f64( const tn_mesh* f, const tn_mesh* c, int bcc, int bcs, int am, int cm,
                                      const double* p, double* const* u, void* s )
{
    return gradient_apply< double >( f, c, bcc, bcs, am, cm, p, u, as_stream( s ) );
}
extern "C" int tn_gradient_apply_f32( const tn_mesh* f, const tn_mesh* c, int bcc, int bcs, int am, int cm,
                                      const float* p, float* const* u, void* s )
{
    return gradient_apply< float >( f, c, bcc, bcs, am, cm, p, u, as_stream( s ) );
}
