// EpsilonDivDiv with the 3x2 Felippa rule (fe/wedge/operators/shell/
// epsilon_divdiv.hpp:218-600): int k (2 eps(u):eps(v) - 2/3 div u div v) with
// k interpolated by the wedge shape functions at each of the six quadrature
// points.  treat_boundary eliminates the CMB nodes of layer 0 (otherwise the
// SURFACE nodes of layer N-1) keeping their diagonal; diagonal mode keeps only
// the diagonal.  The reference runs nine (dim_i, dim_j) passes per cell; here
// one pass per quadrature point forms grad u over the coupled nodes and tests
// it with every node at once.
//
// One thread per cell (r fastest), the 8 x 3 node sums in registers, one
// atomic per node and component, then the additive halo.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

__device__ __constant__ const double kEQP[3][2] = { { 0.6666666666666666, 0.1666666666666667 },
                                                    { 0.1666666666666667, 0.6666666666666666 },
                                                    { 0.1666666666666667, 0.1666666666666667 } };

template < typename T >
struct E32Params
{
    int             N, n1;
    const double*   coords;
    const T*        radii;
    const T*        k;
    Ptr3< const T > src;
    Ptr3< T >       dst;
    int             treat, diag;
};

template < typename T >
__global__ void __launch_bounds__( 128 ) epsdivdiv3x2_kernel( E32Params< T > P )
{
    const int       N = P.N, n1 = P.n1;
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int r = int( t % N );
    const int y = int( ( t / N ) % N );
    const int x = int( ( t / ( (long long) N * N ) ) % N );
    const int d = int( t / ( (long long) N * N * N ) );

    const bool bot = P.treat && r == 0;
    const bool top = P.treat && !bot && r == N - 1;
    const T    r1 = P.radii[d * n1 + r], r2 = P.radii[d * n1 + r + 1];
    T          acc[2][2][2][3];
    for ( int i = 0; i < 24; ++i )
        ( &acc[0][0][0][0] )[i] = T( 0 );
    for ( int w = 0; w < 2; ++w )
    {
        T    p[3][3], s[6][3], kv[6], out[6][3];
        bool coupled[6];
        for ( int n = 0; n < 6; ++n )
        {
            const size_t lat = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] );
            if ( n < 3 )
                for ( int a = 0; a < 3; ++a )
                    p[n][a] = T( P.coords[lat * 3 + a] );
            const size_t i = lat * n1 + r + kWedgeNode[w][n][2];
            kv[n]          = P.k[i];
            for ( int c = 0; c < 3; ++c )
            {
                s[n][c]   = P.src.p[c][i];
                out[n][c] = T( 0 );
            }
            coupled[n] = !P.diag && !( bot && n < 3 ) && !( top && n >= 3 );
        }
        for ( int q = 0; q < 6; ++q )
        {
            const T xi = T( kEQP[q % 3][0] ), eta = T( kEQP[q % 3][1] );
            const T zeta = q < 3 ? T( -0.5773502691896257 ) : T( 0.5773502691896257 );
            T       IT[3][3];
            const T det = wedge_jacobian_it( p[0], p[1], p[2], r1, r2, xi, eta, zeta, IT );
            const T lat[3] = { T( 1 ) - xi - eta, xi, eta };
            T       ke = T( 0 ), g[6][3];
            for ( int n = 0; n < 6; ++n )
            {
                T gr[3];
                grad_shape_ref( n, xi, eta, zeta, gr );
                for ( int a = 0; a < 3; ++a )
                    g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
                ke += lat[n % 3] * ( n < 3 ? T( 0.5 ) * ( T( 1 ) - zeta ) : T( 0.5 ) * ( T( 1 ) + zeta ) ) * kv[n];
            }
            const T wk = T( 0.1666666666666667 ) * ke * fabs( det );
            T       G[3][3] = { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } };
            for ( int n = 0; n < 6; ++n )
                if ( coupled[n] )
                    for ( int a = 0; a < 3; ++a )
                        for ( int b = 0; b < 3; ++b )
                            G[a][b] += g[n][a] * s[n][b];
            const T div = G[0][0] + G[1][1] + G[2][2];
            for ( int n = 0; n < 6; ++n )
            {
                if ( coupled[n] )
                {
                    for ( int c = 0; c < 3; ++c )
                    {
                        const T e = g[n][0] * ( G[0][c] + G[c][0] ) + g[n][1] * ( G[1][c] + G[c][1] ) +
                                    g[n][2] * ( G[2][c] + G[c][2] );
                        out[n][c] += wk * ( e - T( 2.0 / 3.0 ) * g[n][c] * div );
                    }
                }
                else
                {
                    const T gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
                    for ( int c = 0; c < 3; ++c )
                        out[n][c] += wk * s[n][c] * ( gg + g[n][c] * g[n][c] * T( 1.0 / 3.0 ) );
                }
            }
        }
        for ( int n = 0; n < 6; ++n )
            for ( int c = 0; c < 3; ++c )
                acc[kWedgeNode[w][n][0]][kWedgeNode[w][n][1]][kWedgeNode[w][n][2]][c] += out[n][c];
    }
    for ( int dx = 0; dx < 2; ++dx )
        for ( int dy = 0; dy < 2; ++dy )
            for ( int dr = 0; dr < 2; ++dr )
            {
                const size_t i = lat_index( n1, d, x + dx, y + dy ) * n1 + r + dr;
                for ( int c = 0; c < 3; ++c )
                    atomicAdd( P.dst.p[c] + i, acc[dx][dy][dr][c] );
            }
}

}  // namespace

template < typename T >
int epsdivdiv3x2_apply( const tn_mesh* m, const T* k, int treat, int diag, int apply_mode, int comm_mode,
                        const T* const* src, T* const* dst, cudaStream_t st )
{
    TN_CHECK_ARG( m && k && src && dst, "epsdivdiv3x2_apply: null argument" );
    TN_CHECK_ARG( apply_mode == TN_APPLY_REPLACE || apply_mode == TN_APPLY_ADD, "epsdivdiv3x2_apply: bad apply mode" );
    E32Params< T > P{};
    for ( int c = 0; c < 3; ++c )
    {
        TN_CHECK_ARG( src[c] && dst[c], "epsdivdiv3x2_apply: null vector component" );
        P.src.p[c] = src[c];
        P.dst.p[c] = dst[c];
        if ( apply_mode == TN_APPLY_REPLACE )
            TN_CUDA_TRY( cudaMemsetAsync( dst[c], 0, m->ns * sizeof( T ), st ) );
    }
    P.N = m->N, P.n1 = m->n1, P.coords = m->d_coords, P.k = k, P.treat = treat != 0, P.diag = diag != 0;
    P.radii = sizeof( T ) == 8 ? reinterpret_cast< const T* >( m->d_radii ) : reinterpret_cast< const T* >( m->d_radii32 );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    epsdivdiv3x2_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( P );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( m, dst, 3, st );
    return TN_OK;
}

}  // namespace tn

using namespace tn;

extern "C" int tn_epsdivdiv3x2_apply_f64( const tn_mesh* m, const double* k, int treat_boundary, int diagonal,
                                          int apply_mode, int comm_mode, const double* const* src, double* const* dst,
                                          void* s )
{
    return epsdivdiv3x2_apply< double >( m, k, treat_boundary, diagonal, apply_mode, comm_mode, src, dst,
                                         as_stream( s ) );
}
extern "C" int tn_epsdivdiv3x2_apply_f32( const tn_mesh* m, const float* k, int treat_boundary, int diagonal,
                                          int apply_mode, int comm_mode, const float* const* src, float* const* dst,
                                          void* s )
{
    return epsdivdiv3x2_apply< float >( m, k, treat_boundary, diagonal, apply_mode, comm_mode, src, dst,
                                        as_stream( s ) );
}
