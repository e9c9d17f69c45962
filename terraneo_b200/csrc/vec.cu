// Krylov vector kernels (restating kernels/common/grid_operations.hpp).
//
// Elementwise kernels run over all components of a vector in one launch (the
// reference launches one kernel per component and fences after each).  The
// dot product accumulates in FP64 with Neumaier compensation, reduces with
// warp shuffles inside a block and finishes deterministically in the last
// block (fixed order over block partials), so results do not depend on timing.
#include <algorithm>

#include "common.cuh"
#include "reduce.cuh"

#include <mutex>
#include <string>

namespace tn {

namespace {

constexpr int kThreads = 256;

unsigned grid_for( size_t n, int per_thread = 4 )
{
    size_t b = ( n + size_t( kThreads ) * per_thread - 1 ) / ( size_t( kThreads ) * per_thread );
    if ( b < 1 )
        b = 1;
    if ( b > 148 * 32 )
        b = 148 * 32;
    return unsigned( b );
}

// component c of a pointer triple with compile-time indices only (indexing
// the kernel-parameter array with a run-time c copies it to the stack)
template < typename T >
__device__ __forceinline__ T* comp_ptr( const Ptr3< T >& p, int c )
{
    return p.at( c );
}

template < typename T >
__global__ void lincomb_kernel( size_t ns, int ncomp, Ptr3< T > y, T c0, int nx, T c1, Ptr3< const T > x1, T c2,
                                Ptr3< const T > x2, T c3, Ptr3< const T > x3 )
{
    const int c  = blockIdx.y;
    T*        py = comp_ptr( y, c );
    const T * p1 = comp_ptr( x1, c ), *p2 = comp_ptr( x2, c ), *p3 = comp_ptr( x3, c );
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        T v = c0;
        if ( nx >= 1 )
            v = v + c1 * p1[i];
        if ( nx >= 2 )
            v = v + c2 * p2[i];
        if ( nx >= 3 )
            v = v + c3 * p3[i];
        py[i] = v;
    }
}

template < typename T, int OP >
__global__ void elementwise_kernel( size_t ns, int ncomp, Ptr3< T > y, Ptr3< const T > x )
{
    const int c = blockIdx.y;
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        if ( OP == 0 )
            y.at( c )[i] = T( 1 ) / y.at( c )[i]; // invert_inplace (grid_operations.hpp:253)
        else
            y.at( c )[i] = y.at( c )[i] * x.at( c )[i]; // mult_elementwise_inplace (:273)
    }
}

// Deterministic replacement of the reference's randomize (grid_operations.hpp:759),
// whose XorShift pool assignment depends on thread scheduling: uniform values
// in [-1, 1) from a splitmix64 hash of (seed, component, index).
template < typename T >
__global__ void randomize_kernel( size_t ns, Ptr3< T > y, unsigned long long seed )
{
    const int c = blockIdx.y;
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * ( ( unsigned long long ) c * ns + i + 1 );
        z                    = ( z ^ ( z >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
        z                    = ( z ^ ( z >> 27 ) ) * 0x94D049BB133111EBull;
        z                    = z ^ ( z >> 31 );
        y.at( c )[i]         = T( double( z >> 11 ) * ( 2.0 / 9007199254740992.0 ) - 1.0 );
    }
}

template < typename TO, typename TI >
__global__ void cast_kernel( size_t ns, int ncomp, Ptr3< TO > y, Ptr3< const TI > x )
{
    const int c = blockIdx.y;
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
        y.at( c )[i] = TO( x.at( c )[i] );
}

// Owned-node dot product over a flat per-stored-node ownership mask; each
// thread keeps a Neumaier-compensated FP64 partial over a grid-stride range.
template < typename T >
__global__ void dot_kernel( size_t ns, int ncomp, Ptr3< const T > a, Ptr3< const T > b,
                            const uint8_t* __restrict__ owned, double* partials, unsigned int* counter,
                            double* result )
{
    Neumaier acc;
    for ( int c = 0; c < ncomp; ++c )
    {
        const T* __restrict__ pa = a.at( c );
        const T* __restrict__ pb = b.at( c );
        for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
        {
            const double v = double( pa[i] ) * double( pb[i] );
            acc.add( owned[i] ? v : 0.0 );
        }
    }
    block_sum_finish< 1 >( &acc, partials, counter, result );
}

// Owned-node sum of a field's components (masked_sum, grid_operations.hpp:569-590), compensated FP64.
template < typename T >
__global__ void sum_kernel( size_t ns, int ncomp, Ptr3< const T > a, const uint8_t* __restrict__ owned,
                            double* partials, unsigned int* counter, double* result )
{
    Neumaier acc;
    for ( int c = 0; c < ncomp; ++c )
    {
        const T* __restrict__ pa = a.at( c );
        for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
            acc.add( owned[i] ? double( pa[i] ) : 0.0 );
    }
    block_sum_finish< 1 >( &acc, partials, counter, result );
}

// One Chebyshev step (linalg/solvers/chebyshev.hpp:127-160) fused into a
// single pass: z = D^{-1} (b - Ax), d = alpha z + beta d, x = x + d.
template < typename T >
__device__ __forceinline__ void chebyshev_entry( size_t i, T* __restrict__ px, T* __restrict__ pd,
                                                 const T* __restrict__ pb, const T* __restrict__ pa,
                                                 const T* __restrict__ pi, T alpha, T beta, bool use_d )
{
    const T z  = pi[i] * ( pb[i] - pa[i] );
    const T dn = use_d ? alpha * z + beta * pd[i] : alpha * z;
    pd[i]      = dn;
    px[i]      = px[i] + dn;
}

template < typename T >
__device__ __forceinline__ void chebyshev_lane( T b, T a, T inv, T d, T& x, T& dn, T alpha, T beta, bool use_d )
{
    const T z = inv * ( b - a );
    dn        = use_d ? alpha * z + beta * d : alpha * z;
    x         = x + dn;
}

template < typename T >
struct Vec16;
template <>
struct Vec16< float >
{
    using type = float4;
    static __device__ __forceinline__ void step( const float4& b, const float4& a, const float4& i, const float4& d,
                                                 float4& x, float4& dn, float al, float be, bool u )
    {
        chebyshev_lane( b.x, a.x, i.x, d.x, x.x, dn.x, al, be, u );
        chebyshev_lane( b.y, a.y, i.y, d.y, x.y, dn.y, al, be, u );
        chebyshev_lane( b.z, a.z, i.z, d.z, x.z, dn.z, al, be, u );
        chebyshev_lane( b.w, a.w, i.w, d.w, x.w, dn.w, al, be, u );
    }
};
template <>
struct Vec16< double >
{
    using type = double2;
    static __device__ __forceinline__ void step( const double2& b, const double2& a, const double2& i,
                                                 const double2& d, double2& x, double2& dn, double al, double be,
                                                 bool u )
    {
        chebyshev_lane( b.x, a.x, i.x, d.x, x.x, dn.x, al, be, u );
        chebyshev_lane( b.y, a.y, i.y, d.y, x.y, dn.y, al, be, u );
    }
};

// When the five fields share their offset modulo 16 bytes (always for the
// library's own vectors), the entries up to the first 16-byte boundary are
// done one by one and the rest with 16-byte vector loads and stores, two
// vectors per thread in flight: one load instruction moves 4 FP32 / 2 FP64
// entries, so the load queue stops throttling the stream.  Otherwise each
// thread loads kU entries a grid stride apart before it stores any.
template < typename T >
__global__ void chebyshev_kernel( size_t ns, Ptr3< T > x, Ptr3< T > d, Ptr3< const T > b, Ptr3< const T > ax,
                                  Ptr3< const T > inv_diag, T alpha, T beta )
{
    const int c = blockIdx.y;
    T* __restrict__ px       = comp_ptr( x, c );
    T* __restrict__ pd       = comp_ptr( d, c );
    const T* __restrict__ pb = comp_ptr( b, c );
    const T* __restrict__ pa = comp_ptr( ax, c );
    const T* __restrict__ pi = comp_ptr( inv_diag, c );
    const size_t stride      = size_t( gridDim.x ) * blockDim.x;
    const size_t tid         = blockIdx.x * size_t( blockDim.x ) + threadIdx.x;
    const bool   use_d       = beta != T( 0 );
    const size_t mis         = reinterpret_cast< size_t >( px ) & 15;
    const bool   vec = mis % sizeof( T ) == 0 && ( reinterpret_cast< size_t >( pd ) & 15 ) == mis &&
                     ( reinterpret_cast< size_t >( pb ) & 15 ) == mis &&
                     ( reinterpret_cast< size_t >( pa ) & 15 ) == mis &&
                     ( reinterpret_cast< size_t >( pi ) & 15 ) == mis;
    if ( vec )
    {
        using V                 = typename Vec16< T >::type;
        constexpr int kV        = 16 / sizeof( T );
        constexpr int kU        = 2;
        const size_t  head      = std::min( ns, ( ( 16 - mis ) & 15 ) / sizeof( T ) );
        const size_t  nv        = ( ns - head ) / kV;
        const size_t  tail      = head + nv * kV;
        V* __restrict__ vx       = reinterpret_cast< V* >( px + head );
        V* __restrict__ vd       = reinterpret_cast< V* >( pd + head );
        const V* __restrict__ vb = reinterpret_cast< const V* >( pb + head );
        const V* __restrict__ va = reinterpret_cast< const V* >( pa + head );
        const V* __restrict__ vi = reinterpret_cast< const V* >( pi + head );
        if ( tid < head )
            chebyshev_entry( tid, px, pd, pb, pa, pi, alpha, beta, use_d );
        if ( tid < ns - tail )
            chebyshev_entry( tail + tid, px, pd, pb, pa, pi, alpha, beta, use_d );
        for ( size_t j0 = tid; j0 < nv; j0 += kU * stride )
        {
            V bv[kU], av[kU], iv[kU], dv[kU], xv[kU];
#pragma unroll
            for ( int u = 0; u < kU; ++u )
            {
                const size_t j = j0 + u * stride;
                if ( j < nv )
                {
                    bv[u] = vb[j], av[u] = va[j], iv[u] = vi[j], xv[u] = vx[j];
                    dv[u] = use_d ? vd[j] : V{};
                }
            }
#pragma unroll
            for ( int u = 0; u < kU; ++u )
            {
                const size_t j = j0 + u * stride;
                if ( j < nv )
                {
                    V dn;
                    Vec16< T >::step( bv[u], av[u], iv[u], dv[u], xv[u], dn, alpha, beta, use_d );
                    vd[j] = dn;
                    vx[j] = xv[u];
                }
            }
        }
        return;
    }
    constexpr int kU = 4;
    for ( size_t i0 = tid; i0 < ns; i0 += kU * stride )
    {
        T z[kU], dv[kU], xv[kU];
#pragma unroll
        for ( int u = 0; u < kU; ++u )
        {
            const size_t i = i0 + u * stride;
            if ( i < ns )
            {
                z[u]  = pi[i] * ( pb[i] - pa[i] );
                dv[u] = use_d ? pd[i] : T( 0 );
                xv[u] = px[i];
            }
        }
#pragma unroll
        for ( int u = 0; u < kU; ++u )
        {
            const size_t i = i0 + u * stride;
            if ( i < ns )
            {
                const T dn = use_d ? alpha * z[u] + beta * dv[u] : alpha * z[u];
                pd[i]      = dn;
                px[i]      = xv[u] + dn;
            }
        }
    }
}

template < typename T >
__global__ void max_abs_kernel( size_t ns, int ncomp, Ptr3< const T > x, double* partials, unsigned int* counter,
                                double* result )
{
    double m = 0.0;
    for ( int c = 0; c < ncomp; ++c )
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        const double v = fabs( double( x.at( c )[i] ) );
        // NaN propagates as in Kokkos::max reductions only through comparisons;
        // keep the reference's max-of-abs semantics for finite input.
        m = v > m ? v : m;
    }
    block_max_finish( m, partials, counter, result );
}

template < typename T >
__global__ void nan_kernel( size_t ns, int ncomp, Ptr3< const T > x, double* partials, unsigned int* counter,
                            double* result )
{
    double flag = 0.0;
    for ( int c = 0; c < ncomp; ++c )
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        if ( !isfinite( double( x.at( c )[i] ) ) )
            flag = 1.0;
    }
    block_max_finish( flag, partials, counter, result );
}

template < typename T >
int ptr3( int ncomp, T* const* in, Ptr3< T >& out, const char* what )
{
    TN_CHECK_ARG( ncomp >= 1 && ncomp <= 3, std::string( what ) + ": ncomp must be 1..3" );
    TN_CHECK_ARG( in, std::string( what ) + ": null vector" );
    out = {};
    for ( int c = 0; c < ncomp; ++c )
    {
        TN_CHECK_ARG( in[c], std::string( what ) + ": null component" );
        out.p[c] = in[c];
    }
    return TN_OK;
}

template < typename T >
int ptr3c( int ncomp, const T* const* in, Ptr3< const T >& out, const char* what )
{
    TN_CHECK_ARG( ncomp >= 1 && ncomp <= 3, std::string( what ) + ": ncomp must be 1..3" );
    TN_CHECK_ARG( in, std::string( what ) + ": null vector" );
    out = {};
    for ( int c = 0; c < ncomp; ++c )
    {
        TN_CHECK_ARG( in[c], std::string( what ) + ": null component" );
        out.p[c] = in[c];
    }
    return TN_OK;
}

int fetch_result( const tn_mesh* m, int n, cudaStream_t st, double* out )
{
    TN_CUDA_TRY( cudaMemcpyAsync( m->h_red_result, m->d_red_result, sizeof( double ) * n, cudaMemcpyDeviceToHost, st ) );
    TN_CUDA_TRY( cudaStreamSynchronize( st ) );
    for ( int i = 0; i < n; ++i )
        out[i] = m->h_red_result[i];
    return TN_OK;
}

}  // namespace

template < typename T >
int vec_lincomb( const tn_mesh* m, int ncomp, T* const* y, double c0, int nx, const double* c, const T* const* x,
                 cudaStream_t st )
{
    TN_CHECK_ARG( m, "lincomb: mesh is NULL" );
    TN_CHECK_ARG( nx >= 0 && nx <= 3, "lincomb: only 0 to 3 input vectors are supported" );
    TN_CHECK_ARG( nx == 0 || ( c && x ), "lincomb: coefficients/vectors missing" );
    Ptr3< T >       py;
    Ptr3< const T > px[3] = {};
    int             rc;
    if ( ( rc = ptr3( ncomp, y, py, "lincomb" ) ) )
        return rc;
    for ( int i = 0; i < nx; ++i )
        if ( ( rc = ptr3c( ncomp, reinterpret_cast< const T* const* >( x + 3 * i ), px[i], "lincomb" ) ) )
            return rc;
    const T k1 = nx > 0 ? T( c[0] ) : T( 0 ), k2 = nx > 1 ? T( c[1] ) : T( 0 ), k3 = nx > 2 ? T( c[2] ) : T( 0 );
    lincomb_kernel< T ><<< dim3( grid_for( m->ns ), ncomp ), kThreads, 0, st >>>( m->ns, ncomp, py, T( c0 ), nx, k1, px[0], k2,
                                                                          px[1], k3, px[2] );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template < typename T >
int vec_sum( const tn_mesh* m, int ncomp, const T* const* a, double* result, cudaStream_t st )
{
    TN_CHECK_ARG( m && result, "sum: bad arguments" );
    Ptr3< const T > pa;
    if ( const int rc = ptr3c( ncomp, a, pa, "sum" ) )
        return rc;
    const unsigned blocks = std::min< unsigned >( grid_for( m->ns, 8 ), kRedMaxBlocks );
    sum_kernel< T ><<< blocks, kThreads, 0, st >>>( m->ns, ncomp, pa, m->d_node_owned, m->d_red_partials,
                                                   m->d_red_counter, m->d_red_result );
    TN_LAUNCH_CHECK();
    return fetch_result( m, 1, st, result );
}

template < typename T >
int vec_dot( const tn_mesh* m, int ncomp, const T* const* a, const T* const* b, double* result, cudaStream_t st )
{
    TN_CHECK_ARG( m && result, "dot: bad arguments" );
    Ptr3< const T > pa, pb;
    int             rc;
    if ( ( rc = ptr3c( ncomp, a, pa, "dot" ) ) || ( rc = ptr3c( ncomp, b, pb, "dot" ) ) )
        return rc;
    const unsigned blocks = std::min< unsigned >( grid_for( m->ns, 8 ), kRedMaxBlocks );
    dot_kernel< T ><<< blocks, kThreads, 0, st >>>( m->ns, ncomp, pa, pb, m->d_node_owned, m->d_red_partials,
                                                   m->d_red_counter, m->d_red_result );
    TN_LAUNCH_CHECK();
    return fetch_result( m, 1, st, result );
}

template < typename T, int OP >
int vec_elementwise( const tn_mesh* m, int ncomp, T* const* y, const T* const* x, cudaStream_t st )
{
    TN_CHECK_ARG( m, "elementwise: mesh is NULL" );
    Ptr3< T >       py;
    Ptr3< const T > px{};
    int             rc;
    if ( ( rc = ptr3( ncomp, y, py, "elementwise" ) ) )
        return rc;
    if ( OP == 1 && ( rc = ptr3c( ncomp, x, px, "elementwise" ) ) )
        return rc;
    elementwise_kernel< T, OP ><<< dim3( grid_for( m->ns ), ncomp ), kThreads, 0, st >>>( m->ns, ncomp, py, px );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template < typename TO, typename TI >
int vec_cast( const tn_mesh* m, int ncomp, TO* const* y, const TI* const* x, cudaStream_t st )
{
    TN_CHECK_ARG( m, "cast: mesh is NULL" );
    Ptr3< TO >       py;
    Ptr3< const TI > px;
    int              rc;
    if ( ( rc = ptr3( ncomp, y, py, "cast" ) ) || ( rc = ptr3c( ncomp, x, px, "cast" ) ) )
        return rc;
    cast_kernel< TO, TI ><<< dim3( grid_for( m->ns ), ncomp ), kThreads, 0, st >>>( m->ns, ncomp, py, px );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template int vec_lincomb< double >( const tn_mesh*, int, double* const*, double, int, const double*,
                                    const double* const*, cudaStream_t );
template int vec_lincomb< float >( const tn_mesh*, int, float* const*, double, int, const double*, const float* const*,
                                   cudaStream_t );
template int vec_dot< double >( const tn_mesh*, int, const double* const*, const double* const*, double*, cudaStream_t );
template int vec_dot< float >( const tn_mesh*, int, const float* const*, const float* const*, double*, cudaStream_t );

}  // namespace tn

using namespace tn;

// `x` holds nx vectors of 3 pointer slots each (only ncomp slots are read).
extern "C" int tn_vec_lincomb_f64( const tn_mesh* m, int ncomp, double* const* y, double c0, int nx, const double* c,
                                   const double* const* x, void* s )
{
    return vec_lincomb< double >( m, ncomp, y, c0, nx, c, x, as_stream( s ) );
}
extern "C" int tn_vec_lincomb_f32( const tn_mesh* m, int ncomp, float* const* y, double c0, int nx, const double* c,
                                   const float* const* x, void* s )
{
    return vec_lincomb< float >( m, ncomp, y, c0, nx, c, x, as_stream( s ) );
}
extern "C" int tn_vec_sum_f64( const tn_mesh* m, int ncomp, const double* const* a, double* r, void* s )
{
    return vec_sum< double >( m, ncomp, a, r, as_stream( s ) );
}
extern "C" int tn_vec_sum_f32( const tn_mesh* m, int ncomp, const float* const* a, double* r, void* s )
{
    return vec_sum< float >( m, ncomp, a, r, as_stream( s ) );
}
extern "C" int tn_vec_dot_f64( const tn_mesh* m, int ncomp, const double* const* a, const double* const* b, double* r,
                               void* s )
{
    return vec_dot< double >( m, ncomp, a, b, r, as_stream( s ) );
}
extern "C" int tn_vec_dot_f32( const tn_mesh* m, int ncomp, const float* const* a, const float* const* b, double* r,
                               void* s )
{
    return vec_dot< float >( m, ncomp, a, b, r, as_stream( s ) );
}
extern "C" int tn_vec_invert_f64( const tn_mesh* m, int ncomp, double* const* y, void* s )
{
    return vec_elementwise< double, 0 >( m, ncomp, y, nullptr, as_stream( s ) );
}
extern "C" int tn_vec_invert_f32( const tn_mesh* m, int ncomp, float* const* y, void* s )
{
    return vec_elementwise< float, 0 >( m, ncomp, y, nullptr, as_stream( s ) );
}
extern "C" int tn_vec_mult_f64( const tn_mesh* m, int ncomp, double* const* y, const double* const* x, void* s )
{
    return vec_elementwise< double, 1 >( m, ncomp, y, x, as_stream( s ) );
}
extern "C" int tn_vec_mult_f32( const tn_mesh* m, int ncomp, float* const* y, const float* const* x, void* s )
{
    return vec_elementwise< float, 1 >( m, ncomp, y, x, as_stream( s ) );
}
template < typename T >
static int max_abs( const tn_mesh* m, int ncomp, const T* const* x, double* result, void* s )
{
    TN_CHECK_ARG( m && result, "max_abs: bad arguments" );
    Ptr3< const T > px;
    int             rc;
    if ( ( rc = ptr3c( ncomp, x, px, "max_abs" ) ) )
        return rc;
    const unsigned blocks = std::min< unsigned >( grid_for( m->ns * ncomp, 8 ), kRedMaxBlocks );
    max_abs_kernel< T ><<< blocks, kThreads, 0, as_stream( s ) >>>( m->ns, ncomp, px, m->d_red_partials,
                                                                   m->d_red_counter, m->d_red_result );
    TN_LAUNCH_CHECK();
    return fetch_result( m, 1, as_stream( s ), result );
}
extern "C" int tn_vec_max_abs_f64( const tn_mesh* m, int ncomp, const double* const* x, double* result, void* s )
{
    return max_abs< double >( m, ncomp, x, result, s );
}
extern "C" int tn_vec_max_abs_f32( const tn_mesh* m, int ncomp, const float* const* x, double* result, void* s )
{
    return max_abs< float >( m, ncomp, x, result, s );
}
template < typename T >
static int has_nan( const tn_mesh* m, int ncomp, const T* const* x, int* result, void* s )
{
    TN_CHECK_ARG( m && result, "has_nan_or_inf: bad arguments" );
    Ptr3< const T > px;
    int             rc;
    if ( ( rc = ptr3c( ncomp, x, px, "has_nan_or_inf" ) ) )
        return rc;
    const unsigned blocks = std::min< unsigned >( grid_for( m->ns * ncomp, 8 ), kRedMaxBlocks );
    nan_kernel< T ><<< blocks, kThreads, 0, as_stream( s ) >>>( m->ns, ncomp, px, m->d_red_partials, m->d_red_counter,
                                                               m->d_red_result );
    TN_LAUNCH_CHECK();
    double f = 0;
    if ( ( rc = fetch_result( m, 1, as_stream( s ), &f ) ) )
        return rc;
    *result = f != 0.0;
    return TN_OK;
}
extern "C" int tn_vec_has_nan_or_inf_f64( const tn_mesh* m, int ncomp, const double* const* x, int* r, void* s )
{
    return has_nan< double >( m, ncomp, x, r, s );
}
extern "C" int tn_vec_has_nan_or_inf_f32( const tn_mesh* m, int ncomp, const float* const* x, int* r, void* s )
{
    return has_nan< float >( m, ncomp, x, r, s );
}
// assign_masked_else_keep_old (grid_operations.hpp) on the radial boundary
// layers: y = x (or the constant c when x is NULL) at r = 0 (cmb) and r = N
// (surface), unchanged elsewhere; thread per (lateral node, side), blockIdx.y
// = component.
template < typename T >
__global__ void assign_boundary_kernel( size_t nlat, int n1, Ptr3< T > y, Ptr3< const T > x, T c, int cmb, int surf )
{
    const size_t t = blockIdx.x * size_t( blockDim.x ) + threadIdx.x;
    if ( t >= 2 * nlat )
        return;
    const int side = int( t / nlat );
    if ( ( side == 0 && !cmb ) || ( side == 1 && !surf ) )
        return;
    const size_t i = ( t % nlat ) * n1 + ( side == 0 ? 0 : n1 - 1 );
    const int    k  = blockIdx.y;
    const T*     xs = x.at( k );
    y.at( k )[i]    = xs ? xs[i] : c;
}

template < typename T >
static int assign_boundary( const tn_mesh* m, int ncomp, T* const* y, const T* const* x, double c, int cmb, int surf,
                            void* s )
{
    TN_CHECK_ARG( m, "assign_boundary: mesh is NULL" );
    Ptr3< T >       py;
    Ptr3< const T > px{};
    int             rc;
    if ( ( rc = ptr3( ncomp, y, py, "assign_boundary" ) ) )
        return rc;
    if ( x && ( rc = ptr3c( ncomp, x, px, "assign_boundary" ) ) )
        return rc;
    const size_t n = 2 * m->nlat;
    assign_boundary_kernel< T ><<< dim3( unsigned( ( n + 255 ) / 256 ), ncomp ), 256, 0, as_stream( s ) >>>(
        m->nlat, m->n1, py, px, T( c ), cmb, surf );
    TN_LAUNCH_CHECK();
    return TN_OK;
}
extern "C" int tn_vec_assign_boundary_f64( const tn_mesh* m, int ncomp, double* const* y, const double* const* x,
                                           double c, int cmb, int surface, void* s )
{
    return assign_boundary< double >( m, ncomp, y, x, c, cmb, surface, s );
}
extern "C" int tn_vec_assign_boundary_f32( const tn_mesh* m, int ncomp, float* const* y, const float* const* x,
                                           double c, int cmb, int surface, void* s )
{
    return assign_boundary< float >( m, ncomp, y, x, c, cmb, surface, s );
}

template < typename T >
static int chebyshev_step( const tn_mesh* m, int ncomp, T* const* x, T* const* d, const T* const* b, const T* const* ax,
                           const T* const* inv_diag, double alpha, double beta, void* s )
{
    TN_CHECK_ARG( m, "chebyshev_step: mesh is NULL" );
    Ptr3< T >       px, pd;
    Ptr3< const T > pb, pa, pi;
    int             rc;
    if ( ( rc = ptr3( ncomp, x, px, "chebyshev_step" ) ) || ( rc = ptr3( ncomp, d, pd, "chebyshev_step" ) ) ||
         ( rc = ptr3c( ncomp, b, pb, "chebyshev_step" ) ) || ( rc = ptr3c( ncomp, ax, pa, "chebyshev_step" ) ) ||
         ( rc = ptr3c( ncomp, inv_diag, pi, "chebyshev_step" ) ) )
        return rc;
    chebyshev_kernel< T ><<< dim3( grid_for( m->ns, 8 ), ncomp ), kThreads, 0, as_stream( s ) >>>(
        m->ns, px, pd, pb, pa, pi, T( alpha ), T( beta ) );
    TN_LAUNCH_CHECK();
    return TN_OK;
}
extern "C" int tn_vec_chebyshev_step_f64( const tn_mesh* m, int ncomp, double* const* x, double* const* d,
                                          const double* const* b, const double* const* ax,
                                          const double* const* inv_diag, double alpha, double beta, void* s )
{
    return chebyshev_step< double >( m, ncomp, x, d, b, ax, inv_diag, alpha, beta, s );
}
extern "C" int tn_vec_chebyshev_step_f32( const tn_mesh* m, int ncomp, float* const* x, float* const* d,
                                          const float* const* b, const float* const* ax, const float* const* inv_diag,
                                          double alpha, double beta, void* s )
{
    return chebyshev_step< float >( m, ncomp, x, d, b, ax, inv_diag, alpha, beta, s );
}
template < typename T >
static int randomize( const tn_mesh* m, int ncomp, T* const* y, unsigned long long seed, void* s )
{
    TN_CHECK_ARG( m, "randomize: mesh is NULL" );
    Ptr3< T > py;
    int       rc;
    if ( ( rc = ptr3( ncomp, y, py, "randomize" ) ) )
        return rc;
    randomize_kernel< T ><<< dim3( grid_for( m->ns ), ncomp ), kThreads, 0, as_stream( s ) >>>( m->ns, py, seed );
    TN_LAUNCH_CHECK();
    return TN_OK;
}
extern "C" int tn_vec_randomize_f64( const tn_mesh* m, int ncomp, double* const* y, unsigned long long seed, void* s )
{
    return randomize< double >( m, ncomp, y, seed, s );
}
extern "C" int tn_vec_randomize_f32( const tn_mesh* m, int ncomp, float* const* y, unsigned long long seed, void* s )
{
    return randomize< float >( m, ncomp, y, seed, s );
}
extern "C" int tn_vec_cast_f64_to_f32( const tn_mesh* m, int ncomp, float* const* y, const double* const* x, void* s )
{
    return vec_cast< float, double >( m, ncomp, y, x, as_stream( s ) );
}
extern "C" int tn_vec_cast_f32_to_f64( const tn_mesh* m, int ncomp, double* const* y, const float* const* x, void* s )
{
    return vec_cast< double, float >( m, ncomp, y, x, as_stream( s ) );
}

// ---------------------------------------------------------------------------
// Allocation-free owned-node dot product (tn_vec_dot_noalloc_f64).
//
// For callers that cannot let a library allocate device memory: no mesh
// handle, no cudaMalloc / cudaFree / allocating library call.  The reduction
// scratch is one file-scope device array loaded with the module:
//   [0, 262144)        2 doubles (sum, compensation) per block, 16384 blocks
//   [262144, +8)       result
//   [262400, +4)       block ticket (cleared by every call before its launch)
// One block per 2048 entries, so at most 16384 x 2048 = 33,554,432 entries
// per component; longer fields are rejected.  All calls on a device share the
// array: calls that can overlap (several streams or host threads) race on it
// and must be serialised by the caller.  The first call on each device looks
// the array's address up (cudaGetSymbolAddress) and caches it; the array
// itself is made resident on a device when the library's module is loaded
// there (with lazy loading, by the first launch or symbol lookup), never by
// an allocation.  No call may be made while its stream is being captured:
// every call copies its result to the host and synchronises the stream.
namespace tn {
namespace {

constexpr unsigned kNoAllocMaxBlocks     = 16384;
constexpr unsigned kNoAllocPerThread     = 8;
constexpr size_t   kNoAllocMaxEntries    = size_t( kNoAllocMaxBlocks ) * kThreads * kNoAllocPerThread;
constexpr size_t   kNoAllocPartialsBytes = sizeof( double ) * 2 * kNoAllocMaxBlocks;
constexpr size_t   kNoAllocResultOffset  = kNoAllocPartialsBytes;
constexpr size_t   kNoAllocCounterOffset = kNoAllocPartialsBytes + 256;
constexpr size_t   kNoAllocBytes         = kNoAllocPartialsBytes + 512;
constexpr int      kNoAllocMaxDevices    = 64;

static __device__ __align__( 256 ) unsigned char g_dot_scratch[kNoAllocBytes];

std::mutex     g_dot_scratch_mutex;
unsigned char* g_dot_scratch_addr[kNoAllocMaxDevices] = {};

int dot_scratch_address( unsigned char** out )
{
    int dev = 0;
    TN_CUDA_TRY( cudaGetDevice( &dev ) );
    TN_CHECK_ARG( dev >= 0 && dev < kNoAllocMaxDevices, "tn_vec_dot_noalloc_f64: device index out of range" );
    std::lock_guard< std::mutex > lock( g_dot_scratch_mutex );
    if ( !g_dot_scratch_addr[dev] )
    {
        void* p = nullptr;
        TN_CUDA_TRY( cudaGetSymbolAddress( &p, g_dot_scratch ) );
        g_dot_scratch_addr[dev] = static_cast< unsigned char* >( p );
    }
    *out = g_dot_scratch_addr[dev];
    return TN_OK;
}

// Neumaier-compensated FP64 sum of a[i] b[i] over entries with owned[i] != 0
// (owned == NULL: all entries), grid-stride, deterministic last-block finish.
__global__ void dot_noalloc_kernel( size_t n, int ncomp, Ptr3< const double > a, Ptr3< const double > b,
                                    const uint8_t* __restrict__ owned, double* partials, unsigned int* counter,
                                    double* result )
{
    Neumaier acc;
    for ( int c = 0; c < ncomp; ++c )
    {
        const double* __restrict__ pa = a.at( c );
        const double* __restrict__ pb = b.at( c );
        for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < n; i += size_t( gridDim.x ) * blockDim.x )
        {
            const double v = pa[i] * pb[i];
            acc.add( ( owned && !owned[i] ) ? 0.0 : v );
        }
    }
    block_sum_finish< 1 >( &acc, partials, counter, result );
}

}  // namespace
}  // namespace tn

extern "C" int tn_vec_dot_noalloc_f64( size_t n, int ncomp, const double* const* a, const double* const* b,
                                       const uint8_t* owned, double* result, void* s )
{
    using namespace tn;
    TN_CHECK_ARG( a && b && result, "tn_vec_dot_noalloc_f64: NULL argument" );
    TN_CHECK_ARG( ncomp >= 1 && ncomp <= 3, "tn_vec_dot_noalloc_f64: ncomp must be 1, 2 or 3" );
    if ( n > kNoAllocMaxEntries )
    {
        set_error( "tn_vec_dot_noalloc_f64: " + std::to_string( n ) + " entries per component exceed the static scratch "
                   "(at most " + std::to_string( kNoAllocMaxEntries ) + ")" );
        return TN_ERR_ARG;
    }
    Ptr3< const double > pa{}, pb{};
    for ( int c = 0; c < ncomp; ++c )
    {
        TN_CHECK_ARG( a[c] && b[c], "tn_vec_dot_noalloc_f64: NULL field pointer" );
        pa.p[c] = a[c];
        pb.p[c] = b[c];
    }
    if ( n == 0 )
    {
        *result = 0.0;
        return TN_OK;
    }
    cudaStream_t st = as_stream( s );
    // the set-up, the counter clear, the result copy to pageable host memory
    // and the synchronisation are all illegal while the stream is captured
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    TN_CUDA_TRY( cudaStreamIsCapturing( st, &cap ) );
    TN_CHECK_ARG( cap == cudaStreamCaptureStatusNone,
                  "tn_vec_dot_noalloc_f64: the stream is being captured (the call reads its result back and synchronises)" );
    // the cached scratch address is the current device's: the stream must belong to it
    int cur = 0, sdev = 0;
    TN_CUDA_TRY( cudaGetDevice( &cur ) );
    TN_CUDA_TRY( cudaStreamGetDevice( st, &sdev ) );
    TN_CHECK_ARG( sdev == cur, "tn_vec_dot_noalloc_f64: the stream belongs to another device than the current one" );
    unsigned char* base = nullptr;
    int            rc   = dot_scratch_address( &base );
    if ( rc )
        return rc;
    double*       partials = reinterpret_cast< double* >( base );
    double*       dres     = reinterpret_cast< double* >( base + kNoAllocResultOffset );
    unsigned int* counter  = reinterpret_cast< unsigned int* >( base + kNoAllocCounterOffset );
    const size_t  per_block = size_t( kThreads ) * kNoAllocPerThread;
    const unsigned blocks   = unsigned( ( n + per_block - 1 ) / per_block );
    TN_CUDA_TRY( cudaMemsetAsync( counter, 0, sizeof( unsigned int ), st ) );
    dot_noalloc_kernel<<< blocks, kThreads, 0, st >>>( n, ncomp, pa, pb, owned, partials, counter, dres );
    TN_LAUNCH_CHECK();
    TN_CUDA_TRY( cudaMemcpyAsync( result, dres, sizeof( double ), cudaMemcpyDeviceToHost, st ) );
    TN_CUDA_TRY( cudaStreamSynchronize( st ) );
    return TN_OK;
}
