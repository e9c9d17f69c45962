// Scalar Laplace apply (B200 design of fe/wedge/operators/shell/laplace.hpp).
//
// int grad u . grad v with the 3x2 Felippa rule and the curved radial map.
// With treat_boundary, cells touching the CMB (SURFACE) eliminate the coupling
// of the boundary nodes and keep their diagonal (laplace.hpp:200-305).
//
// One thread per cell (r fastest, so neighbouring threads share lateral data
// and touch consecutive addresses); the Jacobian is evaluated at each of the
// six quadrature points.  Contributions are summed over the cell's 8 nodes in
// registers and added with one atomic per node.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

__device__ __constant__ const double kQP32[3][2] = { { 0.6666666666666666, 0.1666666666666667 },
                                                     { 0.1666666666666667, 0.6666666666666666 },
                                                     { 0.1666666666666667, 0.1666666666666667 } };
constexpr double kZeta32 = 0.5773502691896257;
constexpr double kW32    = 0.1666666666666667;

template < typename T >
__global__ void __launch_bounds__( 128 ) laplace_cell_kernel( int N, int n1, const double* __restrict__ coords,
                                                             const T* __restrict__ radii, const T* __restrict__ src,
                                                             T* __restrict__ dst, int treat, int diag )
{
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    // r fastest: consecutive threads share lateral data and touch consecutive addresses
    const int r = int( t % N );
    const int y = int( ( t / N ) % N );
    const int x = int( ( t / ( (long long) N * N ) ) % N );
    const int d = int( t / ( (long long) N * N * N ) );

    const bool bot = treat && r == 0;
    const bool top = treat && !bot && r == N - 1;
    const T    r1 = radii[d * n1 + r], r2 = radii[d * n1 + r + 1];
    const T    dr = T( 0.5 ) * ( r2 - r1 );

    T out[2][2][2] = { { { 0 } } };
    for ( int w = 0; w < 2; ++w )
    {
        T p[3][3], s[6];
        for ( int n = 0; n < 3; ++n )
        {
            const double* u = coords + lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * 3;
            p[n][0] = T( u[0] ), p[n][1] = T( u[1] ), p[n][2] = T( u[2] );
        }
        for ( int n = 0; n < 6; ++n )
            s[n] = src[lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * n1 + r + kWedgeNode[w][n][2]];
        T o[6] = { 0, 0, 0, 0, 0, 0 };
        for ( int ql = 0; ql < 3; ++ql )
        {
            const T xi = T( kQP32[ql][0] ), eta = T( kQP32[ql][1] );
            for ( int qz = 0; qz < 2; ++qz )
            {
                const T zeta = qz == 0 ? T( -kZeta32 ) : T( kZeta32 );
                T       IT[3][3];
                const T det  = wedge_jacobian_it( p[0], p[1], p[2], r1, r2, xi, eta, zeta, IT );
                const T wdet = T( kW32 ) * fabs( det );
                T       g[6][3];
                for ( int n = 0; n < 6; ++n )
                {
                    T gr[3];
                    grad_shape_ref( n, xi, eta, zeta, gr );
                    for ( int a = 0; a < 3; ++a )
                        g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
                }
                int lo = 0, hi = 6;
                if ( bot )
                    lo = 3;
                if ( top )
                    hi = 3;
                if ( diag )
                    lo = hi = 6;
                T gu[3] = { 0, 0, 0 };
                for ( int n = lo; n < hi; ++n )
                    for ( int a = 0; a < 3; ++a )
                        gu[a] += s[n] * g[n][a];
                for ( int n = lo; n < hi; ++n )
                    o[n] += wdet * ( g[n][0] * gu[0] + g[n][1] * gu[1] + g[n][2] * gu[2] );
                for ( int n = 0; n < 6; ++n )
                    if ( diag || ( bot && n < 3 ) || ( top && n >= 3 ) )
                        o[n] += wdet * s[n] * ( g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2] );
            }
        }
        for ( int n = 0; n < 6; ++n )
            out[kWedgeNode[w][n][0]][kWedgeNode[w][n][1]][kWedgeNode[w][n][2]] += o[n];
    }
    (void) dr;
    for ( int dx = 0; dx < 2; ++dx )
        for ( int dy = 0; dy < 2; ++dy )
            for ( int dz = 0; dz < 2; ++dz )
                atomicAdd( dst + lat_index( n1, d, x + dx, y + dy ) * n1 + r + dz, out[dx][dy][dz] );
}

}  // namespace

template < typename T >
int laplace_apply( const tn_mesh* m, int treat, int diag, int apply_mode, int comm_mode, const T* src, T* dst,
                   cudaStream_t st )
{
    TN_CHECK_ARG( m && src && dst, "laplace_apply: null argument" );
    TN_CHECK_ARG( apply_mode == TN_APPLY_REPLACE || apply_mode == TN_APPLY_ADD, "laplace_apply: bad apply mode" );
    if ( apply_mode == TN_APPLY_REPLACE )
        TN_CUDA_TRY( cudaMemsetAsync( dst, 0, m->ns * sizeof( T ), st ) );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    const T*        radii = sizeof( T ) == 8 ? reinterpret_cast< const T* >( m->d_radii )
                                             : reinterpret_cast< const T* >( m->d_radii32 );
    laplace_cell_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( m->N, m->n1, m->d_coords, radii, src,
                                                                                 dst, treat, diag );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
    {
        T* f[1] = { dst };
        return halo_sum< T >( m, f, 1, st );
    }
    return TN_OK;
}

}  // namespace tn

using namespace tn;

extern "C" int tn_laplace_apply_f64( const tn_mesh* m, int treat, int diag, int am, int cm, const double* src,
                                     double* dst, void* s )
{
    return laplace_apply< double >( m, treat, diag, am, cm, src, dst, as_stream( s ) );
}
extern "C" int tn_laplace_apply_f32( const tn_mesh* m, int treat, int diag, int am, int cm, const float* src,
                                     float* dst, void* s )
{
    return laplace_apply< float >( m, treat, diag, am, cm, src, dst, as_stream( s ) );
}
