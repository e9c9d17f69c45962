// C++ mirror of the reference's vector concept over the terraneo_b200 C ABI.
//
// VectorQ1Scalar / VectorQ1Vec / VectorQ1IsoQ2Q1 follow linalg/vector_q1.hpp
// and linalg/vector_q1isoq2_q1.hpp: device fields in the reference layout,
// shallow-copy handle semantics (copies share device memory, like Kokkos
// views), and the *_impl members the VectorLike concept needs
// (linalg/vector.hpp:8-37).  Free functions lincomb / dot / assign / apply /
// solve mirror linalg/vector.hpp:72-250 and linalg/operator.hpp:156.
//
// Every call is asynchronous on tn::stream() except those that return a host
// value (dot, max_abs_entry, has_nan_or_inf), which synchronise, keeping the
// reference's synchronous semantics.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../../include/terraneo_b200.h"

namespace tn {

inline void check( int rc, const char* what )
{
    if ( rc != TN_OK )
        throw std::runtime_error( std::string( what ) + ": " + tn_last_error() );
}

// The stream every call of this layer is issued on (default: the legacy
// default stream).  A solver may switch it for the duration of a solve, e.g.
// to capture a preconditioner into a CUDA graph.
inline cudaStream_t& stream_ref()
{
    static thread_local cudaStream_t s = nullptr;
    return s;
}
inline cudaStream_t stream() { return stream_ref(); }

// shared device allocation
template < typename T >
std::shared_ptr< T > device_alloc( size_t n )
{
    T* p = nullptr;
    if ( cudaMalloc( &p, sizeof( T ) * ( n ? n : 1 ) ) != cudaSuccess )
        throw std::runtime_error( "terraneo_b200: cudaMalloc failed" );
    return std::shared_ptr< T >( p, []( T* q ) { cudaFree( q ); } );
}

// one shell mesh (level, radii range) owning its tn_mesh handle
class Mesh
{
  public:
    Mesh() = default;
    Mesh( int level, double r_min, double r_max )
    {
        tn_mesh* m = nullptr;
        check( tn_mesh_create( level, r_min, r_max, &m ), "tn_mesh_create" );
        h_ = std::shared_ptr< tn_mesh >( m, []( tn_mesh* q ) { tn_mesh_destroy( q ); } );
        check( tn_mesh_dims( m, &level_, &ns_, &nu_ ), "tn_mesh_dims" );
        r_min_ = r_min, r_max_ = r_max;
    }
    // non-owning view of a mesh created through the C ABI
    static Mesh wrap( const tn_mesh* m )
    {
        Mesh out;
        out.h_ = std::shared_ptr< tn_mesh >( const_cast< tn_mesh* >( m ), []( tn_mesh* ) {} );
        check( tn_mesh_dims( m, &out.level_, &out.ns_, &out.nu_ ), "tn_mesh_dims" );
        return out;
    }
    const tn_mesh* get() const { return h_.get(); }
    size_t         stored_nodes() const { return ns_; }
    size_t         unique_nodes() const { return nu_; }
    int            level() const { return level_; }
    double         r_min() const { return r_min_; }
    double         r_max() const { return r_max_; }

  private:
    std::shared_ptr< tn_mesh > h_;
    int                        level_ = 0;
    size_t                     ns_ = 0, nu_ = 0;
    double                     r_min_ = 0, r_max_ = 0;
};

namespace detail {
// dispatch helpers on the scalar type
template < typename T >
struct abi;
template <>
struct abi< double >
{
    static constexpr auto lincomb  = tn_vec_lincomb_f64;
    static constexpr auto dot      = tn_vec_dot_f64;
    static constexpr auto invert   = tn_vec_invert_f64;
    static constexpr auto mult     = tn_vec_mult_f64;
    static constexpr auto has_nan  = tn_vec_has_nan_or_inf_f64;
    static constexpr auto max_abs  = tn_vec_max_abs_f64;
    static constexpr auto rand     = tn_vec_randomize_f64;
    static constexpr auto cheb     = tn_vec_chebyshev_step_f64;
    static constexpr auto halo     = tn_halo_sum_f64;
};
template <>
struct abi< float >
{
    static constexpr auto lincomb  = tn_vec_lincomb_f32;
    static constexpr auto dot      = tn_vec_dot_f32;
    static constexpr auto invert   = tn_vec_invert_f32;
    static constexpr auto mult     = tn_vec_mult_f32;
    static constexpr auto has_nan  = tn_vec_has_nan_or_inf_f32;
    static constexpr auto max_abs  = tn_vec_max_abs_f32;
    static constexpr auto rand     = tn_vec_randomize_f32;
    static constexpr auto cheb     = tn_vec_chebyshev_step_f32;
    static constexpr auto halo     = tn_halo_sum_f32;
};
inline unsigned long long& rand_counter()
{
    static unsigned long long c = 0x5eed;
    return c;
}
}  // namespace detail

// `NC` scalar fields of stored-node length on one mesh
template < typename T, int NC >
class VectorQ1Base
{
  public:
    using ScalarType = T;
    VectorQ1Base() = default;
    VectorQ1Base( const Mesh& mesh )
    : mesh_( mesh )
    , buf_( device_alloc< T >( mesh.stored_nodes() * NC ) )
    {
        cudaMemset( buf_.get(), 0, sizeof( T ) * mesh.stored_nodes() * NC );
    }
    // non-owning view of NC contiguous fields at `external` (device memory)
    VectorQ1Base( const Mesh& mesh, T* external )
    : mesh_( mesh )
    , buf_( external, []( T* ) {} )
    {}
    const Mesh& mesh() const { return mesh_; }
    T*          comp( int c ) const { return buf_.get() + size_t( c ) * mesh_.stored_nodes(); }
    T*          data() const { return buf_.get(); }
    size_t      size() const { return mesh_.stored_nodes() * NC; }
    static constexpr int ncomp = NC;

    void ptrs( T* p[3] ) const
    {
        for ( int c = 0; c < 3; ++c )
            p[c] = c < NC ? comp( c ) : nullptr;
    }

    // VectorLike members (linalg/vector.hpp:8-37)
    template < typename V >
    void lincomb_impl( const std::vector< T >& c, const std::vector< V >& x, const T c0 )
    {
        if ( c.size() != x.size() )
            throw std::runtime_error( "lincomb: c and x must have the same size" );
        if ( x.size() > 3 )
            throw std::runtime_error( "lincomb: not implemented" );
        T*          y[3];
        const T*    xs[9] = {};
        double      cc[3] = { 0, 0, 0 };
        ptrs( y );
        for ( size_t i = 0; i < x.size(); ++i )
        {
            cc[i] = double( c[i] );
            for ( int k = 0; k < NC; ++k )
                xs[3 * i + k] = x[i].comp( k );
        }
        check( detail::abi< T >::lincomb( mesh_.get(), NC, y, double( c0 ), int( x.size() ), cc, xs, stream() ),
               "lincomb" );
    }
    T dot_impl( const VectorQ1Base& x ) const
    {
        const T* a[3] = { comp( 0 ), NC > 1 ? comp( 1 ) : nullptr, NC > 2 ? comp( 2 ) : nullptr };
        const T* b[3] = { x.comp( 0 ), NC > 1 ? x.comp( 1 ) : nullptr, NC > 2 ? x.comp( 2 ) : nullptr };
        double   r    = 0;
        check( detail::abi< T >::dot( mesh_.get(), NC, a, b, &r, stream() ), "dot" );
        return T( r );
    }
    void invert_entries_impl()
    {
        T* y[3];
        ptrs( y );
        check( detail::abi< T >::invert( mesh_.get(), NC, y, stream() ), "invert" );
    }
    void scale_with_vector_impl( const VectorQ1Base& x )
    {
        T*       y[3];
        const T* xs[3] = { x.comp( 0 ), NC > 1 ? x.comp( 1 ) : nullptr, NC > 2 ? x.comp( 2 ) : nullptr };
        ptrs( y );
        check( detail::abi< T >::mult( mesh_.get(), NC, y, xs, stream() ), "scale_with_vector" );
    }
    void randomize_impl()
    {
        T* y[3];
        ptrs( y );
        check( detail::abi< T >::rand( mesh_.get(), NC, y, detail::rand_counter()++, stream() ), "randomize" );
    }
    bool has_nan_or_inf_impl() const
    {
        const T* a[3] = { comp( 0 ), NC > 1 ? comp( 1 ) : nullptr, NC > 2 ? comp( 2 ) : nullptr };
        int      r    = 0;
        check( detail::abi< T >::has_nan( mesh_.get(), NC, a, &r, stream() ), "has_nan_or_inf" );
        return r != 0;
    }
    T max_abs_entry_impl() const
    {
        const T* a[3] = { comp( 0 ), NC > 1 ? comp( 1 ) : nullptr, NC > 2 ? comp( 2 ) : nullptr };
        double   r    = 0;
        check( detail::abi< T >::max_abs( mesh_.get(), NC, a, &r, stream() ), "max_abs_entry" );
        return T( r );
    }
    void swap_impl( VectorQ1Base& o ) { std::swap( buf_, o.buf_ ); }
    void halo_sum()
    {
        T* y[3];
        ptrs( y );
        check( detail::abi< T >::halo( mesh_.get(), y, NC, stream() ), "halo_sum" );
    }
    void copy_from( const VectorQ1Base& o )
    {
        if ( cudaMemcpyAsync( data(), o.data(), sizeof( T ) * size(), cudaMemcpyDeviceToDevice, stream() ) != cudaSuccess )
            throw std::runtime_error( "copy_from: cudaMemcpyAsync failed" );
    }

  protected:
    Mesh                 mesh_;
    std::shared_ptr< T > buf_;
};

template < typename T >
class VectorQ1Scalar : public VectorQ1Base< T, 1 >
{
  public:
    using VectorQ1Base< T, 1 >::VectorQ1Base;
};

template < typename T >
class VectorQ1Vec : public VectorQ1Base< T, 3 >
{
  public:
    using VectorQ1Base< T, 3 >::VectorQ1Base;
};

// Q1-iso-Q2 velocity (level L) + Q1 pressure (level L-1) block vector
// (linalg/vector_q1isoq2_q1.hpp:19); dot = dot(u) + dot(p) (:74-76).
template < typename T >
class VectorQ1IsoQ2Q1
{
  public:
    using ScalarType = T;
    using Block1Type = VectorQ1Vec< T >;
    using Block2Type = VectorQ1Scalar< T >;
    VectorQ1IsoQ2Q1() = default;
    VectorQ1IsoQ2Q1( const Mesh& mu, const Mesh& mp )
    : u_( mu )
    , p_( mp )
    {}
    Block1Type&       block_1() { return u_; }
    Block2Type&       block_2() { return p_; }
    const Block1Type& block_1() const { return u_; }
    const Block2Type& block_2() const { return p_; }

    void lincomb_impl( const std::vector< T >& c, const std::vector< VectorQ1IsoQ2Q1 >& x, const T c0 )
    {
        std::vector< Block1Type > xu;
        std::vector< Block2Type > xp;
        for ( auto& v : x )
            xu.push_back( v.u_ ), xp.push_back( v.p_ );
        u_.lincomb_impl( c, xu, c0 );
        p_.lincomb_impl( c, xp, c0 );
    }
    T    dot_impl( const VectorQ1IsoQ2Q1& x ) const { return u_.dot_impl( x.u_ ) + p_.dot_impl( x.p_ ); }
    void invert_entries_impl() { u_.invert_entries_impl(), p_.invert_entries_impl(); }
    void scale_with_vector_impl( const VectorQ1IsoQ2Q1& x )
    {
        u_.scale_with_vector_impl( x.u_ ), p_.scale_with_vector_impl( x.p_ );
    }
    void randomize_impl() { u_.randomize_impl(), p_.randomize_impl(); }
    bool has_nan_or_inf_impl() const { return u_.has_nan_or_inf_impl() || p_.has_nan_or_inf_impl(); }
    T    max_abs_entry_impl() const { return std::max( u_.max_abs_entry_impl(), p_.max_abs_entry_impl() ); }
    void swap_impl( VectorQ1IsoQ2Q1& o ) { u_.swap_impl( o.u_ ), p_.swap_impl( o.p_ ); }

  private:
    Block1Type u_;
    Block2Type p_;
};

// A vector as a list of scalar-field segments (one per component and block)
// for the device-resident Krylov steps tn_krylov_axpy_dot_* / tn_pcg_*.
template < typename T >
struct Segments
{
    int            n = 0;
    const tn_mesh* mesh[4]{};
    T*             f[4]{};
};
template < typename T, int NC >
void add_segments( const VectorQ1Base< T, NC >& v, Segments< T >& s )
{
    for ( int c = 0; c < NC; ++c )
    {
        if ( s.n >= 4 )
            throw std::runtime_error( "segments: more than 4 fields" );
        s.mesh[s.n] = v.mesh().get();
        s.f[s.n++]  = v.comp( c );
    }
}
template < typename T >
void add_segments( const VectorQ1IsoQ2Q1< T >& v, Segments< T >& s )
{
    add_segments( v.block_1(), s );
    add_segments( v.block_2(), s );
}
template < typename V >
Segments< typename V::ScalarType > segments( const V& v )
{
    Segments< typename V::ScalarType > s;
    add_segments( v, s );
    return s;
}

// w = w - coeff[0] x (x != NULL); result[0] = <w, v> (v == NULL: <w, w>).
// coeff, gate and result are device pointers; no synchronisation.
template < typename T >
void axpy_dot( const Segments< T >& w, const Segments< T >* x, const double* coeff, const Segments< T >* v,
               const double* gate, double* result )
{
    const T* const* px = x ? x->f : nullptr;
    const T* const* pv = v ? v->f : nullptr;
    if constexpr ( std::is_same_v< T, double > )
        check( tn_krylov_axpy_dot_f64( w.n, w.mesh, w.f, const_cast< const T* const* >( px ), coeff, pv, gate, result,
                                       stream() ),
               "axpy_dot" );
    else
        check( tn_krylov_axpy_dot_f32( w.n, w.mesh, w.f, px, coeff, pv, gate, result, stream() ), "axpy_dot" );
}

// free functions (linalg/vector.hpp:72-250, linalg/operator.hpp:156).  They live in
// tn::fn, made visible inside tn by a using-directive: argument-dependent
// lookup ignores using-directives, so the reference's own solver templates,
// which call these names unqualified on tn vectors, find only the reference's
// linalg:: overloads and run over this library's vectors and operators
// unchanged.
namespace fn {
template < typename V >
void lincomb( V& y, const std::vector< typename V::ScalarType >& c, const std::vector< V >& x,
              typename V::ScalarType c0 = 0 )
{
    y.lincomb_impl( c, x, c0 );
}
template < typename V >
void assign( V& y, typename V::ScalarType c0 )
{
    y.lincomb_impl( {}, std::vector< V >{}, c0 );
}
template < typename V >
void assign( V& y, const V& x )
{
    y.lincomb_impl( { typename V::ScalarType( 1 ) }, std::vector< V >{ x }, typename V::ScalarType( 0 ) );
}
template < typename V >
typename V::ScalarType dot( const V& a, const V& b )
{
    return a.dot_impl( b );
}
template < typename V >
typename V::ScalarType norm_2( const V& a )
{
    return std::sqrt( a.dot_impl( a ) );
}
template < typename V >
void scale_in_place( V& y, const V& x )
{
    y.scale_with_vector_impl( x );
}
template < typename V >
void invert_entries( V& y )
{
    y.invert_entries_impl();
}
template < typename V >
void randomize( V& y )
{
    y.randomize_impl();
}
template < typename V >
bool has_nan_or_inf( const V& y )
{
    return y.has_nan_or_inf_impl();
}

// linalg::apply (linalg/operator.hpp:156) and linalg::solvers::solve
template < typename Op, typename Src, typename Dst >
void apply( Op& op, const Src& src, Dst& dst )
{
    op.apply_impl( src, dst );
}
template < typename Solver, typename Op, typename X, typename B >
void solve( Solver& s, Op& A, X& x, const B& b )
{
    s.solve_impl( A, x, b );
}
}  // namespace fn
using namespace fn;

// One fused Chebyshev step: d = alpha D^{-1} (b - ax) + beta d, x += d
template < typename T, int NC >
void chebyshev_step( VectorQ1Base< T, NC >& x, VectorQ1Base< T, NC >& d, const VectorQ1Base< T, NC >& b,
                     const VectorQ1Base< T, NC >& ax, const VectorQ1Base< T, NC >& inv_diag, double alpha,
                     double beta )
{
    T *      px[3], *pd[3];
    const T *pb[3], *pa[3], *pi[3];
    x.ptrs( px );
    d.ptrs( pd );
    for ( int c = 0; c < 3; ++c )
    {
        pb[c] = c < NC ? b.comp( c ) : nullptr;
        pa[c] = c < NC ? ax.comp( c ) : nullptr;
        pi[c] = c < NC ? inv_diag.comp( c ) : nullptr;
    }
    check( detail::abi< T >::cheb( x.mesh().get(), NC, px, pd, pb, pa, pi, alpha, beta, stream() ), "chebyshev_step" );
}

// FP64 <-> FP32 copies for the mixed-precision preconditioner
inline void cast( VectorQ1Vec< float >& y, const VectorQ1Vec< double >& x )
{
    float*        yp[3];
    const double* xp[3] = { x.comp( 0 ), x.comp( 1 ), x.comp( 2 ) };
    y.ptrs( yp );
    check( tn_vec_cast_f64_to_f32( y.mesh().get(), 3, yp, xp, stream() ), "cast" );
}
inline void cast( VectorQ1Vec< double >& y, const VectorQ1Vec< float >& x )
{
    double*      yp[3];
    const float* xp[3] = { x.comp( 0 ), x.comp( 1 ), x.comp( 2 ) };
    y.ptrs( yp );
    check( tn_vec_cast_f32_to_f64( y.mesh().get(), 3, yp, xp, stream() ), "cast" );
}
inline void cast( VectorQ1Scalar< float >& y, const VectorQ1Scalar< double >& x )
{
    float*        yp[1] = { y.data() };
    const double* xp[1] = { x.data() };
    check( tn_vec_cast_f64_to_f32( y.mesh().get(), 1, yp, xp, stream() ), "cast" );
}
inline void cast( VectorQ1Scalar< double >& y, const VectorQ1Scalar< float >& x )
{
    double*      yp[1] = { y.data() };
    const float* xp[1] = { x.data() };
    check( tn_vec_cast_f32_to_f64( y.mesh().get(), 1, yp, xp, stream() ), "cast" );
}
template < typename TO, typename TI >
void cast( VectorQ1IsoQ2Q1< TO >& y, const VectorQ1IsoQ2Q1< TI >& x )
{
    cast( y.block_1(), x.block_1() );
    cast( y.block_2(), x.block_2() );
}

}  // namespace tn
