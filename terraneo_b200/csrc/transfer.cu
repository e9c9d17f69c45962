// Grid transfer between levels L-1 (coarse) and L (fine): constant
// (fe/wedge/shell/grid_transfer_constant.hpp, prolongation_constant.hpp,
// restriction_constant.hpp) and linear (grid_transfer_linear.hpp,
// prolongation_linear.hpp, restriction_linear.hpp).
//
// The reference scatters from each coarse node into its 21-point fine
// stencil with atomics.  Here both directions are gathers without atomics:
//  * prolongation: each fine node reads its (at most 2 x 2) coarse parents —
//    1 / 1/2 laterally (edge and anti-diagonal midpoints), 1 / 1/2 radially;
//  * restriction: each coarse node sums its 21-point stencil of OWNED fine
//    values with the same weights, then the coarse halo adds duplicates.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

template < typename T >
__global__ void prolong_constant_kernel( int nd, int nf1, int nc1, Ptr3< const T > src, Ptr3< T > dst, int ncomp,
                                         int add )
{
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) nd * nf1 * nf1 * nf1;
    if ( t >= total )
        return;
    const int rf = int( t % nf1 ), yf = int( ( t / nf1 ) % nf1 ), xf = int( ( t / ( (long long) nf1 * nf1 ) ) % nf1 );
    const int d  = int( t / ( (long long) nf1 * nf1 * nf1 ) );
    // lateral parents
    int lx[2], ly[2], nl;
    if ( !( xf & 1 ) && !( yf & 1 ) )
        lx[0] = xf / 2, ly[0] = yf / 2, nl = 1;
    else if ( ( xf & 1 ) && !( yf & 1 ) )
        lx[0] = ( xf - 1 ) / 2, ly[0] = yf / 2, lx[1] = ( xf + 1 ) / 2, ly[1] = yf / 2, nl = 2;
    else if ( !( xf & 1 ) && ( yf & 1 ) )
        lx[0] = xf / 2, ly[0] = ( yf - 1 ) / 2, lx[1] = xf / 2, ly[1] = ( yf + 1 ) / 2, nl = 2;
    else
        lx[0] = ( xf + 1 ) / 2, ly[0] = ( yf - 1 ) / 2, lx[1] = ( xf - 1 ) / 2, ly[1] = ( yf + 1 ) / 2, nl = 2;
    const int r0 = rf / 2, r1 = ( rf + 1 ) / 2;
    const T   wl = nl == 1 ? T( 1 ) : T( 0.5 );
    const T   wr = r0 == r1 ? T( 1 ) : T( 0.5 );
    for ( int c = 0; c < ncomp; ++c )
    {
        T v = 0;
        for ( int a = 0; a < nl; ++a )
        {
            const T* col = src.at( c ) + ( ( size_t( d ) * nc1 + lx[a] ) * nc1 + ly[a] ) * nc1;
            v += wl * ( r0 == r1 ? wr * col[r0] : wr * col[r0] + wr * col[r1] );
        }
        T* o = dst.at( c ) + t;
        *o   = add ? *o + v : v;
    }
}

template < typename T >
__global__ void restrict_constant_kernel( int nd, int nf1, int nc1, const uint8_t* __restrict__ owned_f,
                                          Ptr3< const T > src, Ptr3< T > dst, int ncomp, int add )
{
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) nd * nc1 * nc1 * nc1;
    if ( t >= total )
        return;
    const int rc = int( t % nc1 ), yc = int( ( t / nc1 ) % nc1 ), xc = int( ( t / ( (long long) nc1 * nc1 ) ) % nc1 );
    const int d  = int( t / ( (long long) nc1 * nc1 * nc1 ) );
    constexpr int off[7][2] = { { -1, 0 }, { -1, 1 }, { 0, 1 }, { 1, 0 }, { 1, -1 }, { 0, -1 }, { 0, 0 } };
    T             v[3]      = { 0, 0, 0 };
    // unrolled with guards: compile-time table and component indices (no stack), same summation order
#pragma unroll
    for ( int s = 0; s < 7; ++s )
    {
        const int xf = 2 * xc + off[s][0], yf = 2 * yc + off[s][1];
        if ( xf < 0 || xf >= nf1 || yf < 0 || yf >= nf1 )
            continue;
        const size_t lat = ( size_t( d ) * nf1 + xf ) * nf1 + yf;
        if ( !owned_f[lat] )
            continue;
        const T wl = s == 6 ? T( 1 ) : T( 0.5 );
#pragma unroll
        for ( int dr = -1; dr <= 1; ++dr )
        {
            const int rf = 2 * rc + dr;
            if ( rf < 0 || rf >= nf1 )
                continue;
            const T w = dr == 0 ? wl : T( 0.5 ) * wl;
#pragma unroll
            for ( int c = 0; c < 3; ++c )
                if ( c < ncomp )
                    v[c] += w * src.at( c )[lat * nf1 + rf];
        }
    }
#pragma unroll
    for ( int c = 0; c < 3; ++c )
        if ( c < ncomp )
        {
            T* o = dst.at( c ) + t;
            *o   = add ? *o + v[c] : v[c];
        }
}

// coarse(X, Y, R) = fine(2X, 2Y, 2R): coefficient fields on coarser levels
template < typename T >
__global__ void inject_kernel( int nd, int nf1, int nc1, Ptr3< const T > src, Ptr3< T > dst, int ncomp )
{
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) nd * nc1 * nc1 * nc1;
    if ( t >= total )
        return;
    const int rc = int( t % nc1 ), yc = int( ( t / nc1 ) % nc1 ), xc = int( ( t / ( (long long) nc1 * nc1 ) ) % nc1 );
    const int d  = int( t / ( (long long) nc1 * nc1 * nc1 ) );
    for ( int c = 0; c < ncomp; ++c )
        dst.at( c )[t] = src.at( c )[( ( size_t( d ) * nf1 + 2 * xc ) * nf1 + 2 * yc ) * nf1 + 2 * rc];
}

// tangential projection of 3-vectors at CMB / SURFACE nodes
// (strong_algebraic_freeslip_enforcement_in_place, fe/strong_algebraic_freeslip_enforcement.hpp:23)
template < typename T >
__global__ void freeslip_project_kernel( int nd, int n1, const double* __restrict__ coords, Ptr3< T > y, int cmb,
                                         int surf )
{
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) nd * n1 * n1 * 2;
    if ( t >= total )
        return;
    const int    side = int( t & 1 );
    const size_t lat  = size_t( t >> 1 );
    if ( ( side == 0 && !cmb ) || ( side == 1 && !surf ) )
        return;
    const double* c = coords + lat * 3;
    const double  m = sqrt( c[0] * c[0] + c[1] * c[1] + c[2] * c[2] );
    const double  n[3] = { c[0] / m, c[1] / m, c[2] / m };
    const size_t  i    = lat * n1 + ( side == 0 ? 0 : n1 - 1 );
    const double  v[3] = { double( y.p[0][i] ), double( y.p[1][i] ), double( y.p[2][i] ) };
    const double  dt   = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
    y.p[0][i] = T( v[0] - dt * n[0] ), y.p[1][i] = T( v[1] - dt * n[1] ), y.p[2][i] = T( v[2] - dt * n[2] );
}

// Prolongation: each fine node gathers its coarse parents (blockIdx.y = component).
template < typename T >
__global__ void prolong_linear_kernel( int nd, int Nf, int nc1, const double* __restrict__ coords,
                                       const double* __restrict__ radii, Ptr3< const T > src, Ptr3< T > dst, int add )
{
    const int       nf1   = Nf + 1;
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) nd * nf1 * nf1 * nf1;
    if ( t >= total )
        return;
    const int r = int( t % nf1 ), y = int( ( t / nf1 ) % nf1 ), x = int( ( t / ( (long long) nf1 * nf1 ) ) % nf1 );
    const int d = int( t / ( (long long) nf1 * nf1 * nf1 ) );
    int       cx[4], cy[4], cr[4];
    double    w[4];
    const int k = linear_stencil( Nf, coords, radii, d, x, y, r, cx, cy, cr, w );
    const T*  s = src.at( blockIdx.y );
    T         v = T( 0 );
    for ( int i = 0; i < k; ++i )
        v += T( w[i] ) * s[( ( size_t( d ) * nc1 + cx[i] ) * nc1 + cy[i] ) * nc1 + cr[i]];
    T* o = dst.at( blockIdx.y ) + t;
    *o   = add ? *o + v : v;
}

// Restriction = transpose over owned fine nodes: each pushes its weighted
// value to its coarse parents (restriction_linear.hpp:106-222); the coarse
// halo then sums duplicated coarse nodes.
template < typename T >
__global__ void restrict_linear_kernel( int nd, int Nf, int nc1, const double* __restrict__ coords,
                                        const double* __restrict__ radii, const uint8_t* __restrict__ owned,
                                        Ptr3< const T > src, Ptr3< T > dst )
{
    const int       nf1   = Nf + 1;
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) nd * nf1 * nf1 * nf1;
    if ( t >= total || !owned[t] )
        return;
    const int r = int( t % nf1 ), y = int( ( t / nf1 ) % nf1 ), x = int( ( t / ( (long long) nf1 * nf1 ) ) % nf1 );
    const int d = int( t / ( (long long) nf1 * nf1 * nf1 ) );
    int       cx[4], cy[4], cr[4];
    double    w[4];
    const int k = linear_stencil( Nf, coords, radii, d, x, y, r, cx, cy, cr, w );
    const T   v = src.at( blockIdx.y )[t];
    for ( int i = 0; i < k; ++i )
        atomicAdd( dst.at( blockIdx.y ) + ( ( size_t( d ) * nc1 + cx[i] ) * nc1 + cy[i] ) * nc1 + cr[i], T( w[i] ) * v );
}

int check_levels( const tn_mesh* f, const tn_mesh* c, int ncomp )
{
    TN_CHECK_ARG( f && c, "transfer: null mesh" );
    TN_CHECK_ARG( c->level == f->level - 1, "transfer: coarse mesh must be one level below the fine mesh" );
    TN_CHECK_ARG( c->d0 == f->d0 && c->nd == f->nd, "transfer: the meshes must hold the same diamonds" );
    TN_CHECK_ARG( ncomp >= 1 && ncomp <= 3, "transfer: ncomp must be 1..3" );
    return TN_OK;
}

}  // namespace

template < typename T >
int prolong_constant( const tn_mesh* f, const tn_mesh* c, int ncomp, int apply_mode, const T* const* src, T* const* dst,
                      cudaStream_t st )
{
    int rc;
    if ( ( rc = check_levels( f, c, ncomp ) ) )
        return rc;
    Ptr3< const T > s{};
    Ptr3< T >       o{};
    for ( int i = 0; i < ncomp; ++i )
    {
        TN_CHECK_ARG( src[i] && dst[i], "prolongation: null component" );
        s.p[i] = src[i], o.p[i] = dst[i];
    }
    const long long n = (long long) f->ns;
    prolong_constant_kernel< T ><<< unsigned( ( n + 255 ) / 256 ), 256, 0, st >>>( f->nd, f->n1, c->n1, s, o, ncomp,
                                                                                 apply_mode == TN_APPLY_ADD );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template < typename T >
int restrict_constant( const tn_mesh* f, const tn_mesh* c, int ncomp, int apply_mode, const T* const* src,
                       T* const* dst, cudaStream_t st )
{
    int rc;
    if ( ( rc = check_levels( f, c, ncomp ) ) )
        return rc;
    TN_CHECK_ARG( apply_mode == TN_APPLY_REPLACE, "restriction: only Replace mode (the halo sums the whole field)" );
    Ptr3< const T > s{};
    Ptr3< T >       o{};
    for ( int i = 0; i < ncomp; ++i )
    {
        TN_CHECK_ARG( src[i] && dst[i], "restriction: null component" );
        s.p[i] = src[i], o.p[i] = dst[i];
    }
    const long long n = (long long) c->ns;
    restrict_constant_kernel< T ><<< unsigned( ( n + 255 ) / 256 ), 256, 0, st >>>( f->nd, f->n1, c->n1, f->d_lat_owned, s, o,
                                                                                  ncomp, 0 );
    TN_LAUNCH_CHECK();
    return halo_sum< T >( c, dst, ncomp, st );
}

template < typename T >
int prolong_linear( const tn_mesh* f, const tn_mesh* c, int ncomp, int apply_mode, const T* const* src, T* const* dst,
                    cudaStream_t st )
{
    int rc;
    if ( ( rc = check_levels( f, c, ncomp ) ) )
        return rc;
    TN_CHECK_ARG( src && dst, "prolongation: null argument" );
    Ptr3< const T > s{};
    Ptr3< T >       o{};
    for ( int i = 0; i < ncomp; ++i )
    {
        TN_CHECK_ARG( src[i] && dst[i], "prolongation: null component" );
        s.p[i] = src[i], o.p[i] = dst[i];
    }
    const long long n = (long long) f->ns;
    prolong_linear_kernel< T ><<< dim3( unsigned( ( n + 255 ) / 256 ), ncomp ), 256, 0, st >>>(
        f->nd, f->N, c->n1, f->d_coords, f->d_radii, s, o, apply_mode == TN_APPLY_ADD );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template < typename T >
int restrict_linear( const tn_mesh* f, const tn_mesh* c, int ncomp, const T* const* src, T* const* dst,
                     cudaStream_t st )
{
    int rc;
    if ( ( rc = check_levels( f, c, ncomp ) ) )
        return rc;
    TN_CHECK_ARG( src && dst, "restriction: null argument" );
    Ptr3< const T > s{};
    Ptr3< T >       o{};
    for ( int i = 0; i < ncomp; ++i )
    {
        TN_CHECK_ARG( src[i] && dst[i], "restriction: null component" );
        s.p[i] = src[i], o.p[i] = dst[i];
        TN_CUDA_TRY( cudaMemsetAsync( dst[i], 0, sizeof( T ) * c->ns, st ) );
    }
    const long long n = (long long) f->ns;
    restrict_linear_kernel< T ><<< dim3( unsigned( ( n + 255 ) / 256 ), ncomp ), 256, 0, st >>>(
        f->nd, f->N, c->n1, f->d_coords, f->d_radii, f->d_node_owned, s, o );
    TN_LAUNCH_CHECK();
    return halo_sum< T >( c, dst, ncomp, st );
}

template < typename T >
int inject( const tn_mesh* f, const tn_mesh* c, int ncomp, const T* const* src, T* const* dst, cudaStream_t st )
{
    int rc;
    if ( ( rc = check_levels( f, c, ncomp ) ) )
        return rc;
    Ptr3< const T > s{};
    Ptr3< T >       o{};
    for ( int i = 0; i < ncomp; ++i )
    {
        TN_CHECK_ARG( src[i] && dst[i], "injection: null component" );
        s.p[i] = src[i], o.p[i] = dst[i];
    }
    const long long n = (long long) c->ns;
    inject_kernel< T ><<< unsigned( ( n + 255 ) / 256 ), 256, 0, st >>>( f->nd, f->n1, c->n1, s, o, ncomp );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template < typename T >
int freeslip_project( const tn_mesh* m, T* const* y, int cmb, int surf, cudaStream_t st )
{
    TN_CHECK_ARG( m && y && y[0] && y[1] && y[2], "freeslip_project: null argument" );
    const long long n = (long long) m->nlat * 2;
    freeslip_project_kernel< T ><<< unsigned( ( n + 255 ) / 256 ), 256, 0, st >>>(
        m->nd, m->n1, m->d_coords, Ptr3< T >{ { y[0], y[1], y[2] } }, cmb, surf );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template int prolong_constant< double >( const tn_mesh*, const tn_mesh*, int, int, const double* const*,
                                         double* const*, cudaStream_t );
template int prolong_constant< float >( const tn_mesh*, const tn_mesh*, int, int, const float* const*, float* const*,
                                        cudaStream_t );
template int restrict_constant< double >( const tn_mesh*, const tn_mesh*, int, int, const double* const*,
                                          double* const*, cudaStream_t );
template int restrict_constant< float >( const tn_mesh*, const tn_mesh*, int, int, const float* const*, float* const*,
                                         cudaStream_t );

}  // namespace tn

using namespace tn;

extern "C" int tn_prolongation_constant_f64( const tn_mesh* f, const tn_mesh* c, int ncomp, int am,
                                             const double* const* src, double* const* dst, void* s )
{
    return prolong_constant< double >( f, c, ncomp, am, src, dst, as_stream( s ) );
}
extern "C" int tn_prolongation_constant_f32( const tn_mesh* f, const tn_mesh* c, int ncomp, int am,
                                             const float* const* src, float* const* dst, void* s )
{
    return prolong_constant< float >( f, c, ncomp, am, src, dst, as_stream( s ) );
}
extern "C" int tn_prolongation_linear_f64( const tn_mesh* f, const tn_mesh* c, int ncomp, int am,
                                           const double* const* src, double* const* dst, void* s )
{
    return prolong_linear< double >( f, c, ncomp, am, src, dst, as_stream( s ) );
}
extern "C" int tn_prolongation_linear_f32( const tn_mesh* f, const tn_mesh* c, int ncomp, int am,
                                           const float* const* src, float* const* dst, void* s )
{
    return prolong_linear< float >( f, c, ncomp, am, src, dst, as_stream( s ) );
}
extern "C" int tn_restriction_linear_f64( const tn_mesh* f, const tn_mesh* c, int ncomp, const double* const* src,
                                          double* const* dst, void* s )
{
    return restrict_linear< double >( f, c, ncomp, src, dst, as_stream( s ) );
}
extern "C" int tn_restriction_linear_f32( const tn_mesh* f, const tn_mesh* c, int ncomp, const float* const* src,
                                          float* const* dst, void* s )
{
    return restrict_linear< float >( f, c, ncomp, src, dst, as_stream( s ) );
}
extern "C" int tn_injection_f64( const tn_mesh* f, const tn_mesh* c, int ncomp, const double* const* src,
                                 double* const* dst, void* s )
{
    return inject< double >( f, c, ncomp, src, dst, as_stream( s ) );
}
extern "C" int tn_freeslip_project_f64( const tn_mesh* m, double* const* y, int cmb, int surface, void* s )
{
    return freeslip_project< double >( m, y, cmb, surface, as_stream( s ) );
}
extern "C" int tn_restriction_constant_f64( const tn_mesh* f, const tn_mesh* c, int ncomp, const double* const* src,
                                            double* const* dst, void* s )
{
    return restrict_constant< double >( f, c, ncomp, TN_APPLY_REPLACE, src, dst, as_stream( s ) );
}
extern "C" int tn_restriction_constant_f32( const tn_mesh* f, const tn_mesh* c, int ncomp, const float* const* src,
                                            float* const* dst, void* s )
{
    return restrict_constant< float >( f, c, ncomp, TN_APPLY_REPLACE, src, dst, as_stream( s ) );
}
