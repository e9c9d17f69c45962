// Device-resident Krylov steps: the scalars of PCG and of FGMRES's
// modified Gram-Schmidt stay in device memory, so a solver issues its
// iterations without a host round trip per dot product.
//
// A Krylov vector is a list of up to four scalar-field segments, each one
// stored-node field of some mesh reduced over that mesh's owned nodes: a
// velocity field is three segments on the fine mesh, the Stokes block vector
// (u fine, p coarse; linalg/vector_q1isoq2_q1.hpp:19) four.  Reductions are
// Neumaier-compensated FP64 with the same deterministic last-block finish as
// tn_vec_dot_*.
//
// PCG (linalg/solvers/pcg.hpp:60-140, identity preconditioner as in the
// coarse solve of apps/mantlecirculation/mantlecirculation.cpp:657) keeps its
// state in a device array; every step reads a `done` flag first and returns
// without touching memory once the stopping rule has fired, so a host may
// issue all max_iterations steps (or capture them) and still obtain the
// iterate the host-checked loop stops at.
#include "common.cuh"
#include "reduce.cuh"

namespace tn {

namespace {

constexpr int kThreads  = 256;
constexpr int kMaxSegs  = 4;

struct Segs
{
    int            n;
    size_t         len[kMaxSegs];
    const uint8_t* owned[kMaxSegs];
};

template < typename T >
struct SegPtr
{
    T* p[kMaxSegs];
};

int make_segs( int nseg, const tn_mesh* const* mesh, Segs& s, const char* what )
{
    if ( nseg < 1 || nseg > kMaxSegs || !mesh )
    {
        set_error( std::string( what ) + ": need 1 to 4 segments" );
        return TN_ERR_ARG;
    }
    s.n = nseg;
    for ( int k = 0; k < kMaxSegs; ++k )
    {
        s.len[k]   = 0;
        s.owned[k] = nullptr;
        if ( k < nseg )
        {
            if ( !mesh[k] )
            {
                set_error( std::string( what ) + ": segment mesh is NULL" );
                return TN_ERR_ARG;
            }
            s.len[k]   = mesh[k]->ns;
            s.owned[k] = mesh[k]->d_node_owned;
        }
    }
    return TN_OK;
}

template < typename T, typename P >
int make_ptr( int nseg, P in, SegPtr< T >& out, bool optional, const char* what )
{
    for ( int k = 0; k < kMaxSegs; ++k )
        out.p[k] = nullptr;
    if ( !in )
    {
        if ( optional )
            return TN_OK;
        set_error( std::string( what ) + ": field list is NULL" );
        return TN_ERR_ARG;
    }
    for ( int k = 0; k < nseg; ++k )
    {
        if ( !in[k] )
        {
            set_error( std::string( what ) + ": field pointer is NULL" );
            return TN_ERR_ARG;
        }
        out.p[k] = const_cast< T* >( in[k] );
    }
    return TN_OK;
}

unsigned red_blocks( const Segs& s )
{
    size_t n = 0;
    for ( int k = 0; k < s.n; ++k )
        n += s.len[k];
    // 8 entries per thread on large fields; small (coarse-level) fields get one
    // entry per thread up to two blocks per SM, since there the latency of a
    // thread's dependent loads, not bandwidth, sets the time
    size_t b = ( n + size_t( kThreads ) * 8 - 1 ) / ( size_t( kThreads ) * 8 );
    b        = std::max( b, std::min< size_t >( ( n + kThreads - 1 ) / kThreads, 296 ) );
    return unsigned( std::max< size_t >( 1, std::min< size_t >( b, kRedMaxBlocks ) ) );
}

// w = w - coeff[0] * x (x non-NULL), then result[0] = <w, v> (v NULL: <w, w>).
// One MGS step of linalg/solvers/fgmres.hpp:203-209 with the update of basis
// vector i fused to the projection on basis vector i + 1.
template < typename T >
__global__ void axpy_dot_kernel( Segs s, SegPtr< T > w, SegPtr< const T > x, const double* coeff,
                                 SegPtr< const T > v, const double* gate, double* partials, unsigned int* counter,
                                 double* result )
{
    if ( gate && gate[0] != 0.0 )
        return;
    const bool upd = x.p[0] != nullptr;
    const T    a   = upd ? T( -coeff[0] ) : T( 0 );
    // kU entries per thread and step, all loads issued before the arithmetic;
    // plain FP64 sums per thread (two chains), compensated across threads
    constexpr int kU     = 4;
    double        sum[2] = { 0.0, 0.0 };
    const size_t  stride = size_t( gridDim.x ) * blockDim.x;
#pragma unroll
    for ( int k = 0; k < kMaxSegs; ++k ) // compile-time segment indices (no stack copy)
        if ( k < s.n )
    {
        T* __restrict__ pw             = w.p[k];
        const T* __restrict__ px       = x.p[k];
        const T* __restrict__ pv       = v.p[k];
        const uint8_t* __restrict__ ow = s.owned[k];
        const size_t n                 = s.len[k];
        for ( size_t i0 = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i0 < n; i0 += kU * stride )
        {
            T       wi[kU], xi[kU], vi[kU];
            uint8_t oi[kU];
#pragma unroll
            for ( int u = 0; u < kU; ++u )
            {
                const size_t i = i0 + u * stride;
                const bool   in = i < n;
                wi[u]           = in ? pw[i] : T( 0 );
                xi[u]           = in && upd ? px[i] : T( 0 );
                vi[u]           = in && pv ? pv[i] : T( 0 );
                oi[u]           = in ? ow[i] : uint8_t( 0 );
            }
#pragma unroll
            for ( int u = 0; u < kU; ++u )
            {
                const size_t i = i0 + u * stride;
                if ( upd )
                {
                    wi[u] = wi[u] + a * xi[u];
                    if ( i < n )
                        pw[i] = wi[u];
                }
                const double prod = double( wi[u] ) * double( pv ? vi[u] : wi[u] );
                sum[u & 1] += oi[u] ? prod : 0.0;
            }
        }
    }
    Neumaier acc;
    acc.add( sum[0] );
    acc.add( sum[1] );
    block_sum_finish< 1 >( &acc, partials, counter, result );
}

// PCG state layout (doubles): see tn_pcg_* in the public header.
enum : int
{
    kAn = 0,
    kPap,
    kR0,
    kBeta,
    kDone,
    kIts,
    kRelres,
    kHist = 8
};

// p = r; r0 = |r|; an = <r, r>  (pcg.hpp:79-86 with z = r)
template < typename T >
__global__ void pcg_begin_kernel( Segs s, SegPtr< const T > r, SegPtr< T > p, double* state, double atol,
                                  double* partials, unsigned int* counter )
{
    Neumaier acc;
#pragma unroll
    for ( int k = 0; k < kMaxSegs; ++k ) // compile-time segment indices (no stack copy)
        if ( k < s.n )
        for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < s.len[k];
              i += size_t( gridDim.x ) * blockDim.x )
        {
            const T ri = r.p[k][i];
            p.p[k][i]  = ri;
            acc.add( s.owned[k][i] ? double( ri ) * double( ri ) : 0.0 );
        }
    if ( block_sum_finish< 1 >( &acc, partials, counter, state + kAn ) && threadIdx.x == 0 )
    {
        const double r0      = sqrt( state[kAn] );
        state[kR0]           = r0;
        state[kBeta]         = 0.0;
        state[kDone]         = r0 < atol ? 1.0 : 0.0;
        state[kIts]          = 0.0;
        state[kRelres]       = 1.0;
        state[kHist]         = 1.0;
    }
}

// alpha = an / pap; x += alpha p; r -= alpha ap; stopping rule; beta
// (pcg.hpp:91-100 with z = r)
template < typename T >
__global__ void pcg_update_kernel( Segs s, SegPtr< T > x, SegPtr< T > r, SegPtr< const T > p, SegPtr< const T > ap,
                                   double* state, int it, double rtol, double atol, double* partials,
                                   unsigned int* counter, double* scratch )
{
    if ( state[kDone] != 0.0 )
        return;
    const double alpha = state[kAn] / state[kPap];
    const T      ta = T( alpha ), tm = T( -alpha );
    Neumaier     acc;
#pragma unroll
    for ( int k = 0; k < kMaxSegs; ++k ) // compile-time segment indices (no stack copy)
        if ( k < s.n )
        for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < s.len[k];
              i += size_t( gridDim.x ) * blockDim.x )
        {
            x.p[k][i]    = x.p[k][i] + ta * p.p[k][i];
            const T ri   = r.p[k][i] + tm * ap.p[k][i];
            r.p[k][i]    = ri;
            acc.add( s.owned[k][i] ? double( ri ) * double( ri ) : 0.0 );
        }
    if ( block_sum_finish< 1 >( &acc, partials, counter, scratch ) && threadIdx.x == 0 )
    {
        // it <= 0: the step number follows the device's count (a replayed graph of steps)
        const int    k  = it > 0 ? it : int( state[kIts] ) + 1;
        const double rr = scratch[0], ar = sqrt( rr ), rel = ar / state[kR0];
        state[kHist + k] = rel;
        state[kRelres]   = rel;
        state[kIts]      = double( k );
        if ( rel <= rtol || ar < atol )
            state[kDone] = 1.0;
        else
        {
            state[kBeta] = rr / state[kAn];
            state[kAn]   = rr;
        }
    }
}

// p = r + beta p  (pcg.hpp:101)
template < typename T >
__global__ void pcg_direction_kernel( Segs s, SegPtr< T > p, SegPtr< const T > r, const double* state )
{
    if ( state[kDone] != 0.0 )
        return;
    const T beta = T( state[kBeta] );
#pragma unroll
    for ( int k = 0; k < kMaxSegs; ++k ) // compile-time segment indices (no stack copy)
        if ( k < s.n )
        for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < s.len[k];
              i += size_t( gridDim.x ) * blockDim.x )
            p.p[k][i] = r.p[k][i] + beta * p.p[k][i];
}

}  // namespace

template < typename T >
static int axpy_dot( int nseg, const tn_mesh* const* mesh, T* const* w, const T* const* x, const double* coeff,
                     const T* const* v, const double* gate, double* result, void* st )
{
    Segs              s;
    SegPtr< T >       pw;
    SegPtr< const T > px, pv;
    int               rc;
    if ( ( rc = make_segs( nseg, mesh, s, "axpy_dot" ) ) || ( rc = make_ptr( nseg, w, pw, false, "axpy_dot" ) ) ||
         ( rc = make_ptr( nseg, x, px, true, "axpy_dot" ) ) || ( rc = make_ptr( nseg, v, pv, true, "axpy_dot" ) ) )
        return rc;
    TN_CHECK_ARG( result, "axpy_dot: result is NULL" );
    TN_CHECK_ARG( !x || coeff, "axpy_dot: coefficient is NULL" );
    const tn_mesh* m0 = mesh[0];
    axpy_dot_kernel< T ><<< red_blocks( s ), kThreads, 0, as_stream( st ) >>>( s, pw, px, coeff, pv, gate,
                                                                              m0->d_red_partials, m0->d_red_counter,
                                                                              result );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

}  // namespace tn

using namespace tn;

extern "C" int tn_krylov_axpy_dot_f64( int nseg, const tn_mesh* const* mesh, double* const* w,
                                       const double* const* x, const double* coeff, const double* const* v,
                                       const double* gate, double* result, void* stream )
{
    return axpy_dot< double >( nseg, mesh, w, x, coeff, v, gate, result, stream );
}
extern "C" int tn_krylov_axpy_dot_f32( int nseg, const tn_mesh* const* mesh, float* const* w, const float* const* x,
                                       const double* coeff, const float* const* v, const double* gate,
                                       double* result, void* stream )
{
    return axpy_dot< float >( nseg, mesh, w, x, coeff, v, gate, result, stream );
}

extern "C" int tn_pcg_begin_f64( int nseg, const tn_mesh* const* mesh, const double* const* r, double* const* p,
                                 double* state, double atol, void* stream )
{
    Segs                   s;
    SegPtr< const double > pr;
    SegPtr< double >       pp;
    int                    rc;
    if ( ( rc = make_segs( nseg, mesh, s, "pcg_begin" ) ) || ( rc = make_ptr( nseg, r, pr, false, "pcg_begin" ) ) ||
         ( rc = make_ptr( nseg, p, pp, false, "pcg_begin" ) ) )
        return rc;
    TN_CHECK_ARG( state, "pcg_begin: state is NULL" );
    pcg_begin_kernel< double ><<< red_blocks( s ), kThreads, 0, as_stream( stream ) >>>(
        s, pr, pp, state, atol, mesh[0]->d_red_partials, mesh[0]->d_red_counter );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

extern "C" int tn_pcg_pap_f64( int nseg, const tn_mesh* const* mesh, const double* const* ap,
                               const double* const* p, double* state, void* stream )
{
    return axpy_dot< double >( nseg, mesh, const_cast< double* const* >( ap ), nullptr, nullptr, p, state + kDone,
                               state + kPap, stream );
}

extern "C" int tn_pcg_update_f64( int nseg, const tn_mesh* const* mesh, double* const* x, double* const* r,
                                  const double* const* p, const double* const* ap, double* state, int iteration,
                                  double rtol, double atol, void* stream )
{
    Segs                   s;
    SegPtr< double >       px, pr;
    SegPtr< const double > pp, pa;
    int                    rc;
    if ( ( rc = make_segs( nseg, mesh, s, "pcg_update" ) ) || ( rc = make_ptr( nseg, x, px, false, "pcg_update" ) ) ||
         ( rc = make_ptr( nseg, r, pr, false, "pcg_update" ) ) || ( rc = make_ptr( nseg, p, pp, false, "pcg_update" ) ) ||
         ( rc = make_ptr( nseg, ap, pa, false, "pcg_update" ) ) )
        return rc;
    TN_CHECK_ARG( state, "pcg_update: state is NULL" );
    const tn_mesh* m0 = mesh[0];
    pcg_update_kernel< double ><<< red_blocks( s ), kThreads, 0, as_stream( stream ) >>>(
        s, px, pr, pp, pa, state, iteration, rtol, atol, m0->d_red_partials, m0->d_red_counter, m0->d_red_result + 8 );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

extern "C" int tn_pcg_direction_f64( int nseg, const tn_mesh* const* mesh, double* const* p, const double* const* r,
                                     const double* state, void* stream )
{
    Segs                   s;
    SegPtr< double >       pp;
    SegPtr< const double > pr;
    int                    rc;
    if ( ( rc = make_segs( nseg, mesh, s, "pcg_direction" ) ) ||
         ( rc = make_ptr( nseg, p, pp, false, "pcg_direction" ) ) ||
         ( rc = make_ptr( nseg, r, pr, false, "pcg_direction" ) ) )
        return rc;
    TN_CHECK_ARG( state, "pcg_direction: state is NULL" );
    size_t n = 0;
    for ( int k = 0; k < nseg; ++k )
        n = std::max( n, s.len[k] );
    const unsigned blocks = unsigned( std::max< size_t >( 1, std::min< size_t >( ( n + 1023 ) / 1024, 148 * 32 ) ) );
    pcg_direction_kernel< double ><<< blocks, kThreads, 0, as_stream( stream ) >>>( s, pp, pr, state );
    TN_LAUNCH_CHECK();
    return TN_OK;
}
