// KMass apply (fe/wedge/operators/shell/kmass.hpp): int k u v with the 3x2
// Felippa rule, k interpolated at the quadrature points; consistent,
// diagonal or lumped-diagonal action.  With k = 1 it is the plain Mass
// (mass.hpp); applied per component it is the VectorMass used for right-hand
// sides (vector_mass.hpp).  One thread per cell, atomic accumulation, then the
// additive halo.  Setup / right-hand-side work, not on the iteration path.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

__device__ __constant__ const double kMQP[6][3] = { { 0.6666666666666666, 0.1666666666666667, -0.5773502691896257 },
                                                    { 0.1666666666666667, 0.6666666666666666, -0.5773502691896257 },
                                                    { 0.1666666666666667, 0.1666666666666667, -0.5773502691896257 },
                                                    { 0.6666666666666666, 0.1666666666666667, 0.5773502691896257 },
                                                    { 0.1666666666666667, 0.6666666666666666, 0.5773502691896257 },
                                                    { 0.1666666666666667, 0.1666666666666667, 0.5773502691896257 } };

template < typename T >
__global__ void __launch_bounds__( 128 ) kmass_kernel( int N, int n1, const double* __restrict__ coords,
                                                      const T* __restrict__ radii, const T* __restrict__ k,
                                                      const T* __restrict__ src, T* __restrict__ dst, int mode )
{
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int r = int( t % N ), y = int( ( t / N ) % N ), x = int( ( t / ( (long long) N * N ) ) % N );
    const int d = int( t / ( (long long) N * N * N ) );
    const T   r1 = radii[d * n1 + r], r2 = radii[d * n1 + r + 1];
    for ( int w = 0; w < 2; ++w )
    {
        T      p[3][3], kn[6], s[6], o[6] = { 0, 0, 0, 0, 0, 0 };
        size_t idx[6];
        for ( int n = 0; n < 6; ++n )
        {
            const size_t lat = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] );
            if ( n < 3 )
            {
                const double* c = coords + lat * 3;
                p[n][0] = T( c[0] ), p[n][1] = T( c[1] ), p[n][2] = T( c[2] );
            }
            idx[n] = lat * n1 + r + kWedgeNode[w][n][2];
            kn[n]  = k ? k[idx[n]] : T( 1 );
            s[n]   = src[idx[n]];
        }
        for ( int q = 0; q < 6; ++q )
        {
            const T xi = T( kMQP[q][0] ), eta = T( kMQP[q][1] ), zeta = T( kMQP[q][2] );
            T       M[3][3];
            for ( int a = 0; a < 3; ++a )
            {
                M[a][0] = p[1][a] - p[0][a];
                M[a][1] = p[2][a] - p[0][a];
                M[a][2] = ( T( 1 ) - xi - eta ) * p[0][a] + xi * p[1][a] + eta * p[2][a];
            }
            const T det = M[0][0] * ( M[1][1] * M[2][2] - M[1][2] * M[2][1] ) -
                          M[0][1] * ( M[1][0] * M[2][2] - M[1][2] * M[2][0] ) +
                          M[0][2] * ( M[1][0] * M[2][1] - M[1][1] * M[2][0] );
            const T rq = r1 + T( 0.5 ) * ( r2 - r1 ) * ( T( 1 ) + zeta ), gr = T( 0.5 ) * ( r2 - r1 );
            const T lat[3] = { T( 1 ) - xi - eta, xi, eta };
            T       Nn[6], kq = 0, us = 0;
            for ( int n = 0; n < 6; ++n )
            {
                Nn[n] = lat[n % 3] * ( n < 3 ? T( 0.5 ) * ( T( 1 ) - zeta ) : T( 0.5 ) * ( T( 1 ) + zeta ) );
                kq += Nn[n] * kn[n];
                us += Nn[n] * s[n];
            }
            const T f = T( 0.1666666666666667 ) * kq * rq * rq * gr * fabs( det );
            for ( int i = 0; i < 6; ++i )
            {
                if ( mode == 0 )
                    o[i] += f * Nn[i] * us; // consistent: sum_j N_i N_j s_j
                else if ( mode == 1 )
                    o[i] += f * Nn[i] * Nn[i] * s[i];
                else
                    o[i] += f * Nn[i] * s[i]; // lumped: sum_j N_i N_j = N_i
            }
        }
        for ( int n = 0; n < 6; ++n )
            atomicAdd( dst + idx[n], o[n] );
    }
}

}  // namespace

template < typename T >
int kmass_apply( const tn_mesh* m, const T* k, int mode, int apply_mode, int comm_mode, const T* src, T* dst,
                 cudaStream_t st )
{
    TN_CHECK_ARG( m && src && dst, "kmass: null argument" );
    TN_CHECK_ARG( mode >= 0 && mode <= 2, "kmass: mode must be 0 (full), 1 (diagonal) or 2 (lumped)" );
    if ( apply_mode == TN_APPLY_REPLACE )
        TN_CUDA_TRY( cudaMemsetAsync( dst, 0, m->ns * sizeof( T ), st ) );
    const T* radii = sizeof( T ) == 8 ? reinterpret_cast< const T* >( m->d_radii )
                                      : reinterpret_cast< const T* >( m->d_radii32 );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    kmass_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( m->N, m->n1, m->d_coords, radii, k, src, dst,
                                                                          mode );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
    {
        T* f[1] = { dst };
        return halo_sum< T >( m, f, 1, st );
    }
    return TN_OK;
}

template int kmass_apply< double >( const tn_mesh*, const double*, int, int, int, const double*, double*, cudaStream_t );
template int kmass_apply< float >( const tn_mesh*, const float*, int, int, int, const float*, float*, cudaStream_t );

}  // namespace tn

using namespace tn;

extern "C" int tn_kmass_apply_f64( const tn_mesh* m, const double* k, int mode, int am, int cm, const double* src,
                                   double* dst, void* s )
{
    return kmass_apply< double >( m, k, mode, am, cm, src, dst, as_stream( s ) );
}
extern "C" int tn_kmass_apply_f32( const tn_mesh* m, const float* k, int mode, int am, int cm, const float* src,
                                   float* dst, void* s )
{
    return kmass_apply< float >( m, k, mode, am, cm, src, dst, as_stream( s ) );
}
