// Deterministic block reductions with Neumaier-compensated FP64 sums.
//
// Each block reduces its threads' (sum, compensation) pairs with warp
// shuffles, writes one partial per block, and the last block to finish
// (ticket from an atomic counter) combines all partials in block order and
// resets the counter.  The order of every addition is fixed by the launch
// shape, so results are reproducible run to run.
#pragma once

#include "common.cuh"

namespace tn {

struct Neumaier
{
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add( double v )
    {
        const double t = s + v;
        c += fabs( s ) >= fabs( v ) ? ( s - t ) + v : ( v - t ) + s;
        s = t;
    }
    __device__ __forceinline__ void merge( const Neumaier& o )
    {
        add( o.s );
        c += o.c;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

__device__ __forceinline__ Neumaier warp_reduce( Neumaier a )
{
#pragma unroll
    for ( int off = 16; off > 0; off >>= 1 )
    {
        Neumaier o;
        o.s = __shfl_down_sync( 0xffffffffu, a.s, off );
        o.c = __shfl_down_sync( 0xffffffffu, a.c, off );
        a.merge( o );
    }
    return a;
}

// Reduces K compensated sums over the whole grid; result[k] = total k.
// Requires blockDim.x to be a multiple of 32 and <= 1024.  Returns true in
// the last block (where thread 0 has just written `result`), false elsewhere.
template < int K >
__device__ bool block_sum_finish( Neumaier* acc, double* partials, unsigned int* counter, double* result )
{
    __shared__ double   sh_s[32][K], sh_c[32][K];
    __shared__ bool     is_last;
    const int           lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
#pragma unroll
    for ( int k = 0; k < K; ++k )
    {
        Neumaier w = warp_reduce( acc[k] );
        if ( lane == 0 )
            sh_s[warp][k] = w.s, sh_c[warp][k] = w.c;
    }
    __syncthreads();
    if ( threadIdx.x == 0 )
    {
        for ( int k = 0; k < K; ++k )
        {
            Neumaier b;
            for ( int w = 0; w < nwarps; ++w )
                b.merge( Neumaier{ sh_s[w][k], sh_c[w][k] } );
            partials[( size_t( blockIdx.x ) * K + k ) * 2]     = b.s;
            partials[( size_t( blockIdx.x ) * K + k ) * 2 + 1] = b.c;
        }
        __threadfence();
        const unsigned ticket = atomicAdd( counter, 1u );
        is_last               = ( ticket == gridDim.x - 1 );
    }
    __syncthreads();
    if ( !is_last )
        return false;
    __threadfence();
    // each thread merges the partials of blocks tid, tid + blockDim, ... in that order; the loads of J of them
    // (all K sums) are issued before their merges, so the L2 round trips overlap (a merge of the zero padding past
    // the last block leaves a sum unchanged)
    constexpr int J = K == 1 ? 4 : 2;
    Neumaier      t[K];
    for ( unsigned b0 = threadIdx.x; b0 < gridDim.x; b0 += J * blockDim.x )
    {
        double vs[J][K], vc[J][K];
#pragma unroll
        for ( int j = 0; j < J; ++j )
        {
            const unsigned b  = b0 + j * blockDim.x;
            const bool     in = b < gridDim.x;
#pragma unroll
            for ( int k = 0; k < K; ++k )
            {
                vs[j][k] = in ? __ldcg( &partials[( size_t( b ) * K + k ) * 2] ) : 0.0;
                vc[j][k] = in ? __ldcg( &partials[( size_t( b ) * K + k ) * 2 + 1] ) : 0.0;
            }
        }
#pragma unroll
        for ( int j = 0; j < J; ++j )
#pragma unroll
            for ( int k = 0; k < K; ++k )
                t[k].merge( Neumaier{ vs[j][k], vc[j][k] } );
    }
#pragma unroll
    for ( int k = 0; k < K; ++k )
    {
        const Neumaier w = warp_reduce( t[k] );
        if ( lane == 0 )
            sh_s[warp][k] = w.s, sh_c[warp][k] = w.c;
    }
    __syncthreads();
    if ( threadIdx.x == 0 )
    {
        for ( int k = 0; k < K; ++k )
        {
            Neumaier b;
            for ( int w = 0; w < nwarps; ++w )
                b.merge( Neumaier{ sh_s[w][k], sh_c[w][k] } );
            result[k] = b.value();
        }
        *counter = 0u;
    }
    return true;
}

// Grid-wide maximum of non-negative values (same last-block scheme).
__device__ inline void block_max_finish( double v, double* partials, unsigned int* counter, double* result )
{
    __shared__ double sh[32];
    __shared__ bool   is_last;
    const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
#pragma unroll
    for ( int off = 16; off > 0; off >>= 1 )
        v = fmax( v, __shfl_down_sync( 0xffffffffu, v, off ) );
    if ( lane == 0 )
        sh[warp] = v;
    __syncthreads();
    if ( threadIdx.x == 0 )
    {
        double b = 0.0;
        for ( int w = 0; w < nwarps; ++w )
            b = fmax( b, sh[w] );
        partials[blockIdx.x] = b;
        __threadfence();
        is_last = ( atomicAdd( counter, 1u ) == gridDim.x - 1 );
    }
    __syncthreads();
    if ( !is_last )
        return;
    __threadfence();
    double t = 0.0;
    for ( unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x )
        t = fmax( t, __ldcg( &partials[b] ) );
#pragma unroll
    for ( int off = 16; off > 0; off >>= 1 )
        t = fmax( t, __shfl_down_sync( 0xffffffffu, t, off ) );
    if ( lane == 0 )
        sh[warp] = t;
    __syncthreads();
    if ( threadIdx.x == 0 )
    {
        double b = 0.0;
        for ( int w = 0; w < nwarps; ++w )
            b = fmax( b, sh[w] );
        result[0] = b;
        *counter  = 0u;
    }
}

}  // namespace tn
