// C++ restatement of the reference's solver drivers (linalg/solvers/*.hpp)
// over the terraneo_b200 C ABI.  Same concepts (SolverLike: solve_impl(A, x,
// b)), same recurrences and stopping rules; the per-iteration vector work runs
// in the CUDA library.  Iteration histories replace util::Table rows.
#pragma once

#include <cmath>
#include <cstdio>
#include <limits>
#include <map>
#include <vector>

#include "operators.hpp"

namespace tn {

// IterativeSolverParameters (linalg/solvers/iterative_solver_info.hpp:6)
struct IterativeSolverParameters
{
    int    max_iterations              = 100;
    double relative_residual_tolerance = 1e-12;
    double absolute_residual_tolerance = 1e-12;
};

struct SolverStatistics
{
    std::vector< double > relative_residuals;
    int                   iterations = 0;
};

// IdentitySolver (identity_solver.hpp): x = b
template < typename Op >
class IdentitySolver
{
  public:
    template < typename X, typename B >
    void solve_impl( Op&, X& x, const B& b )
    {
        assign( x, b );
    }
};

// DiagonalSolver (diagonal_solver.hpp:20): x = D^{-1} b, D inverted at construction
template < typename Op, typename V >
class DiagonalSolver
{
  public:
    explicit DiagonalSolver( const V& diagonal ) : inv_( diagonal ) { invert_entries( inv_ ); }
    template < typename A >
    void solve_impl( A&, V& x, const V& b )
    {
        assign( x, b );
        scale_in_place( x, inv_ );
    }

  private:
    V inv_;
};

// PCG (pcg.hpp:78-160)
template < typename Op, typename Prec = IdentitySolver< Op > >
class PCG
{
  public:
    using V = typename Op::SrcVectorType;
    PCG( IterativeSolverParameters prm, std::vector< V > tmps, Prec prec = Prec() )
    : prm_( prm ), tmps_( std::move( tmps ) ), prec_( prec )
    {
        if ( tmps_.size() < 4 )
            throw std::runtime_error( "PCG: needs 4 temporary vectors" );
    }
    SolverStatistics stats;
    void             solve_impl( Op& A, V& x, const V& b )
    {
        auto& r = tmps_[0];
        auto& p = tmps_[1];
        auto& ap = tmps_[2];
        auto& z = tmps_[3];
        stats   = {};
        apply( A, x, r );
        lincomb( r, { 1.0, -1.0 }, { b, r } );
        solve( prec_, A, z, r );
        assign( p, z );
        const double r0 = std::sqrt( double( dot( r, r ) ) );
        stats.relative_residuals.push_back( 1.0 );
        if ( r0 < prm_.absolute_residual_tolerance )
            return;
        for ( int it = 1; it <= prm_.max_iterations; ++it )
        {
            const auto an = dot( z, r );
            apply( A, p, ap );
            const auto alpha = an / dot( ap, p );
            lincomb( x, { 1.0, alpha }, { x, p } );
            lincomb( r, { 1.0, -alpha }, { r, ap } );
            const double ar = std::sqrt( double( dot( r, r ) ) );
            stats.relative_residuals.push_back( ar / r0 );
            stats.iterations = it;
            if ( ar / r0 <= prm_.relative_residual_tolerance || ar < prm_.absolute_residual_tolerance )
                return;
            solve( prec_, A, z, r );
            const auto beta = dot( z, r ) / an;
            lincomb( p, { 1.0, beta }, { z, p } );
        }
    }

  private:
    IterativeSolverParameters prm_;
    std::vector< V >          tmps_;
    Prec                      prec_;
};

// PCG with an identity preconditioner whose scalars live in device memory
// (tn_pcg_* in the C ABI): the same iteration and stopping rule as PCG above
// (pcg.hpp:78-102 with z = r), issued without a host round trip per
// iteration.  The done flag is read every `check_every` iterations unless the
// stream is being captured, in which case all max_iterations are issued and
// the gated steps leave the converged iterate untouched.
template < typename Op >
class DevicePCG
{
  public:
    using V = typename Op::SrcVectorType;
    DevicePCG( IterativeSolverParameters prm, std::vector< V > tmps, int check_every = 8 )
    : prm_( prm ), tmps_( std::move( tmps ) ), check_every_( check_every ),
      state_( device_alloc< double >( 8 + size_t( std::max( prm.max_iterations, 0 ) ) + 1 ) )
    {
        if ( tmps_.size() < 3 )
            throw std::runtime_error( "DevicePCG: needs 3 temporary vectors" );
    }
    // with the stored-matrix FP64 viscous operator and a 4th temporary the
    // operator's steps are fused into the PCG steps (tn_stored_pcg_f64)
    bool fused = true;
    void solve_impl( Op& A, V& x, const V& b )
    {
        if constexpr ( std::is_same_v< Op, ViscousOp< double > > )
        {
            const StoredEpsilonDivDiv< double >* so = A.stored();
            if ( fused && so && tmps_.size() >= 4 && !so->params().diagonal &&
                 so->params().apply_mode == TN_APPLY_REPLACE && so->params().comm_mode == TN_COMM_ADDITIVE )
            {
                const double* bb[3] = { b.comp( 0 ), b.comp( 1 ), b.comp( 2 ) };
                double*       xx[3];
                x.ptrs( xx );
                double* w[12];
                for ( int k = 0; k < 4; ++k )
                    tmps_[k].ptrs( w + 3 * k );
                check( tn_stored_pcg_f64( so->mesh().get(), so->matrices(), &so->params(), bb, xx, w, state_.get(),
                                          prm_.max_iterations, prm_.relative_residual_tolerance,
                                          prm_.absolute_residual_tolerance, check_every_, stream() ),
                       "stored_pcg" );
                return;
            }
        }
        auto& r  = tmps_[0];
        auto& p  = tmps_[1];
        auto& ap = tmps_[2];
        apply( A, x, r );
        lincomb( r, { 1.0, -1.0 }, { b, r } );
        const auto sx = segments( x ), sr = segments( r ), sp = segments( p ), sap = segments( ap );
        double*    st = state_.get();
        check( tn_pcg_begin_f64( sr.n, sr.mesh, sr.f, sp.f, st, prm_.absolute_residual_tolerance, stream() ),
               "pcg_begin" );
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing( stream(), &cs );
        const bool capturing = cs != cudaStreamCaptureStatusNone;
        // one step; it <= 0: the step number follows the device's count (replayable in a graph)
        auto step = [&]( int it ) {
            apply( A, p, ap );
            check( tn_pcg_pap_f64( sp.n, sp.mesh, sap.f, sp.f, st, stream() ), "pcg_pap" );
            check( tn_pcg_update_f64( sx.n, sx.mesh, sx.f, sr.f, sp.f, sap.f, st, it, prm_.relative_residual_tolerance,
                                      prm_.absolute_residual_tolerance, stream() ),
                   "pcg_update" );
            check( tn_pcg_direction_f64( sp.n, sp.mesh, sp.f, sr.f, st, stream() ), "pcg_direction" );
        };
        if ( capturing || !graphs || check_every_ < 2 )
        {
            for ( int it = 1; it <= prm_.max_iterations; ++it )
            {
                if ( !capturing && ( it == 1 || ( it - 1 ) % check_every_ == 0 ) && done() )
                    break;
                step( it );
            }
            return;
        }
        // Outside a capture: the first step runs eagerly (tables an operator builds on first use), then a graph of
        // check_every steps, captured once per operator and storage, is replayed with the stopping flag read
        // between replays; the steps after convergence are no-ops on the device.  At most max_iterations steps
        // are issued.
        int issued = 0;
        if ( prm_.max_iterations >= 1 && !done() )
            step( ++issued );
        const std::vector< const void* > key{ &A, sx.f[0], sr.f[0], sp.f[0], sap.f[0] };
        while ( issued < prm_.max_iterations && !done() )
        {
            if ( issued + check_every_ > prm_.max_iterations )
            {
                while ( issued < prm_.max_iterations )
                {
                    step( 0 );
                    ++issued;
                }
                break;
            }
            if ( !chunk_ || chunk_key_ != key )
                capture_chunk( step, key );
            if ( cudaGraphLaunch( static_cast< cudaGraphExec_t >( chunk_.get() ), stream() ) != cudaSuccess )
                throw std::runtime_error( "DevicePCG: cudaGraphLaunch failed" );
            issued += check_every_;
        }
    }
    // replay the iterations from a captured graph outside stream capture (on by default)
    bool graphs = true;
    // statistics of the last solve (synchronises)
    SolverStatistics statistics() const
    {
        const size_t          n = 8 + size_t( std::max( prm_.max_iterations, 0 ) ) + 1;
        std::vector< double > h( n );
        if ( cudaMemcpyAsync( h.data(), state_.get(), n * sizeof( double ), cudaMemcpyDeviceToHost, stream() ) !=
                 cudaSuccess ||
             cudaStreamSynchronize( stream() ) != cudaSuccess )
            throw std::runtime_error( "DevicePCG: reading the state failed" );
        SolverStatistics out;
        out.iterations = int( h[5] );
        out.relative_residuals.assign( h.begin() + 8, h.begin() + 8 + out.iterations + 1 );
        return out;
    }

  private:
    bool done() const
    {
        double f = 0;
        if ( cudaMemcpyAsync( &f, state_.get() + 4, sizeof( double ), cudaMemcpyDeviceToHost, stream() ) !=
                 cudaSuccess ||
             cudaStreamSynchronize( stream() ) != cudaSuccess )
            throw std::runtime_error( "DevicePCG: reading the done flag failed" );
        return f != 0.0;
    }
    // capture check_every steps (device-counted) on a private stream into chunk_
    template < typename Step >
    void capture_chunk( Step& step, const std::vector< const void* >& key )
    {
        if ( !cap_ )
        {
            cudaStream_t c = nullptr;
            if ( cudaStreamCreateWithFlags( &c, cudaStreamNonBlocking ) != cudaSuccess )
                throw std::runtime_error( "DevicePCG: creating the capture stream failed" );
            cap_ = std::shared_ptr< void >( c, []( void* q ) { cudaStreamDestroy( static_cast< cudaStream_t >( q ) ); } );
        }
        cudaStream_t cap   = static_cast< cudaStream_t >( cap_.get() );
        cudaStream_t saved = stream_ref();
        // the capture stream starts after the work already queued on the solve's stream
        cudaEvent_t ev = nullptr;
        if ( cudaEventCreateWithFlags( &ev, cudaEventDisableTiming ) != cudaSuccess ||
             cudaEventRecord( ev, saved ) != cudaSuccess || cudaStreamWaitEvent( cap, ev, 0 ) != cudaSuccess )
        {
            if ( ev )
                cudaEventDestroy( ev );
            throw std::runtime_error( "DevicePCG: ordering the capture stream failed" );
        }
        cudaEventDestroy( ev );
        stream_ref()  = cap;
        cudaGraph_t g = nullptr;
        if ( cudaStreamBeginCapture( cap, cudaStreamCaptureModeThreadLocal ) != cudaSuccess )
        {
            stream_ref() = saved;
            throw std::runtime_error( "DevicePCG: cudaStreamBeginCapture failed" );
        }
        try
        {
            for ( int i = 0; i < check_every_; ++i )
                step( 0 );
        }
        catch ( ... )
        {
            cudaStreamEndCapture( cap, &g );
            if ( g )
                cudaGraphDestroy( g );
            stream_ref() = saved;
            throw;
        }
        const cudaError_t ec = cudaStreamEndCapture( cap, &g );
        stream_ref()         = saved;
        cudaGraphExec_t e    = nullptr;
        if ( ec != cudaSuccess || cudaGraphInstantiate( &e, g, 0 ) != cudaSuccess )
        {
            if ( g )
                cudaGraphDestroy( g );
            throw std::runtime_error( "DevicePCG: capturing the iteration failed" );
        }
        cudaGraphDestroy( g );
        chunk_     = std::shared_ptr< void >( e, []( void* q ) { cudaGraphExecDestroy( static_cast< cudaGraphExec_t >( q ) ); } );
        chunk_key_ = key;
    }
    IterativeSolverParameters  prm_;
    std::vector< V >           tmps_;
    int                        check_every_;
    std::shared_ptr< double >  state_;
    std::shared_ptr< void >    cap_, chunk_;
    std::vector< const void* > chunk_key_;
};

// power_iteration (power_iteration.hpp:13-48) from a deterministic random start
template < typename Op, typename V >
double power_iteration( Op& op, V& it, V& aux, int iterations )
{
    using S = typename V::ScalarType;
    randomize( it );
    auto n = norm_2( it );
    lincomb( it, { S( 1.0 / n ) }, { it }, S( 0 ) );
    apply( op, it, aux );
    double radius = 0;
    for ( int k = 0; k < iterations; ++k )
    {
        n = norm_2( aux );
        lincomb( it, { S( 1.0 / n ) }, { aux }, S( 0 ) );
        apply( op, it, aux );
        radius = double( dot( it, aux ) );
    }
    return radius;
}

// Chebyshev smoother (chebyshev.hpp:50-175): lambda_max = 1.5 * power-iteration
// estimate of D^{-1} A, lambda_min = 0.1 * estimate.
template < typename Op >
class Chebyshev
{
  public:
    using V = typename Op::SrcVectorType;
    Chebyshev( int order, const V& inverse_diagonal, std::vector< V > tmps, int iterations, int power_iterations )
    : order_( order ), inv_diag_( inverse_diagonal ), tmps_( std::move( tmps ) ), iterations_( iterations ),
      power_iterations_( power_iterations )
    {
        // the reference aborts on both (chebyshev.hpp:83-91)
        if ( order_ < 1 )
            throw std::runtime_error( "Chebyshev: order must be at least 1" );
        if ( tmps_.size() < 2 )
            throw std::runtime_error( "Chebyshev: needs 2 temporary vectors" );
    }
    void refresh_max_eigenvalue_estimate_in_next_solve() { need_ev_ = true; }
    // use a given estimate of the largest eigenvalue of D^{-1} A instead of the
    // power iteration (the reference's smoother draws its start vector at
    // random; a caller that reproduces a reference run passes its estimate)
    void set_max_eigenvalue_estimate( double ev )
    {
        ev_      = ev;
        need_ev_ = false;
    }
    double max_eigenvalue_estimate() const { return ev_; }
    void   solve_impl( Op& A, V& x, const V& b )
    {
        if ( need_ev_ )
        {
            DiagonallyScaledOperator< Op > dA( A, inv_diag_ );
            ev_      = power_iteration( dA, tmps_[0], tmps_[1], power_iterations_ );
            need_ev_ = false;
        }
        auto&        d     = tmps_[0];
        auto&        z     = tmps_[1];
        const double lmax  = 1.5 * ev_, lmin = 0.1 * ev_;
        const double theta = 0.5 * ( lmax + lmin ), delta = 0.5 * ( lmax - lmin );
        const double sigma = theta / delta;
        double rho         = 1.0 / sigma; // carried across sweeps as in the reference (chebyshev.hpp:119)
        for ( int it = 0; it < iterations_; ++it )
        {
            // z = A x;  d = D^{-1}(b - z) / theta;  x += d   (one fused vector pass)
            apply( A, x, z );
            chebyshev_step( x, d, b, z, inv_diag_, 1.0 / theta, 0.0 );
            for ( int i = 2; i <= order_; ++i )
            {
                const double rho_new = 1.0 / ( 2.0 * sigma - rho );
                const double beta = rho_new * rho, alpha = 2.0 * rho_new / delta;
                // z = A x;  d = alpha D^{-1}(b - z) + beta d;  x += d
                apply( A, x, z );
                chebyshev_step( x, d, b, z, inv_diag_, alpha, beta );
                rho = rho_new;
            }
        }
    }

  private:
    int              order_;
    V                inv_diag_;
    std::vector< V > tmps_;
    int              iterations_, power_iterations_;
    bool             need_ev_ = true;
    double           ev_      = 0;
};

// Jacobi (jacobi.hpp:14-62): x += omega D^{-1} (b - A x), `iterations`
// times; the update is one fused pass (tn_vec_chebyshev_step with beta = 0).
template < typename Op >
class Jacobi
{
  public:
    using V = typename Op::SrcVectorType;
    Jacobi( const V& inverse_diagonal, int iterations, std::vector< V > tmps, double omega = 1.0 )
    : inv_diag_( inverse_diagonal ), iterations_( iterations ), tmps_( std::move( tmps ) ), omega_( omega )
    {
        if ( tmps_.size() < 2 )
            throw std::runtime_error( "Jacobi: needs 2 temporary vectors" );
    }
    void solve_impl( Op& A, V& x, const V& b )
    {
        for ( int it = 0; it < iterations_; ++it )
        {
            apply( A, x, tmps_[0] );
            chebyshev_step( x, tmps_[1], b, tmps_[0], inv_diag_, omega_, 0.0 );
        }
    }

  private:
    V                inv_diag_;
    int              iterations_;
    std::vector< V > tmps_;
    double           omega_;
};

// Multigrid V-cycle (multigrid.hpp:24-211).  Level 0 is the coarsest.
template < typename Op, typename P, typename R, typename Smoother, typename Coarse >
class Multigrid
{
  public:
    using V = typename Op::SrcVectorType;
    Multigrid( std::vector< P > prolong_additive, std::vector< R > restrict_, std::vector< Op > coarse_ops,
               std::vector< V > tmp_r, std::vector< V > tmp_e, std::vector< V > tmp, std::vector< Smoother > smoothers,
               Coarse coarse, int cycles )
    : P_( std::move( prolong_additive ) ), R_( std::move( restrict_ ) ), A_c_( std::move( coarse_ops ) ),
      tmp_r_( std::move( tmp_r ) ), tmp_e_( std::move( tmp_e ) ), tmp_( std::move( tmp ) ),
      smoothers_( std::move( smoothers ) ), coarse_( std::move( coarse ) ), cycles_( cycles )
    {
        if ( A_c_.empty() )
            throw std::runtime_error( "Multigrid: needs at least one coarse level" );
        if ( P_.size() != A_c_.size() || R_.size() != A_c_.size() || tmp_r_.size() != A_c_.size() ||
             tmp_e_.size() != A_c_.size() || tmp_.size() != A_c_.size() + 1 || smoothers_.size() != A_c_.size() + 1 )
            throw std::runtime_error( "Multigrid: inconsistent level sizes" );
    }
    Coarse& coarse_solver() { return coarse_; }
    void    solve_impl( Op& A, V& x, const V& b )
    {
        for ( int c = 0; c < cycles_; ++c )
            recurse( A, x, b, int( P_.size() ) );
    }

  private:
    void recurse( Op& A, V& x, const V& b, int level )
    {
        using S = typename V::ScalarType;
        if ( level == 0 )
        {
            solve( coarse_, A, tmp_e_[0], tmp_r_[0] );
            return;
        }
        solve( smoothers_[level], A, x, b );
        apply( A, x, tmp_[level] );
        lincomb( tmp_[level], { S( 1 ), S( -1 ) }, { b, tmp_[level] } );
        apply( R_[level - 1], tmp_[level], tmp_r_[level - 1] );
        assign( tmp_e_[level - 1], S( 0 ) );
        recurse( A_c_[level - 1], tmp_e_[level - 1], tmp_r_[level - 1], level - 1 );
        apply( P_[level - 1], tmp_e_[level - 1], x );
        solve( smoothers_[level], A, x, b );
    }

    std::vector< P >        P_;
    std::vector< R >        R_;
    std::vector< Op >       A_c_;
    std::vector< V >        tmp_r_, tmp_e_, tmp_;
    std::vector< Smoother > smoothers_;
    Coarse                  coarse_;
    int                     cycles_;
};

// Replays one captured CUDA graph of a solver's launch sequence per (x, b)
// storage.  The first solve runs eagerly (one-off host work such as the
// Chebyshev eigenvalue estimates and lazily built tables happens there);
// every later solve with storage not seen before is captured on a private
// stream and instantiated, then launched on tn::stream().  The inner solver
// must issue a fixed, data-independent launch sequence after its first solve
// (the device-gated PCG coarse solver does so while capturing) and must not
// change the values baked into its launches (e.g. smoother coefficients)
// afterwards.
template < typename Inner >
class GraphReplay
{
  public:
    GraphReplay( Inner& inner, bool enabled = true ) : inner_( inner ), enabled_( enabled ) {}
    GraphReplay( const GraphReplay& )            = delete;
    GraphReplay& operator=( const GraphReplay& ) = delete;
    ~GraphReplay()
    {
        for ( auto& e : execs_ )
            cudaGraphExecDestroy( e.second );
        if ( cap_ )
            cudaStreamDestroy( cap_ );
    }
    template < typename Op, typename V >
    void solve_impl( Op& A, V& x, const V& b )
    {
        if ( !warm_ || !enabled_ )
        {
            solve( inner_, A, x, b );
            warm_ = true;
            return;
        }
        const auto         sx = segments( x ), sb = segments( b );
        std::vector< const void* > key;
        for ( int i = 0; i < sx.n; ++i )
            key.push_back( sx.f[i] );
        for ( int i = 0; i < sb.n; ++i )
            key.push_back( sb.f[i] );
        auto it = execs_.find( key );
        if ( it == execs_.end() )
        {
            if ( !cap_ && cudaStreamCreateWithFlags( &cap_, cudaStreamNonBlocking ) != cudaSuccess )
                throw std::runtime_error( "GraphReplay: creating the capture stream failed" );
            cudaStream_t saved = stream_ref();
            stream_ref()       = cap_;
            cudaGraph_t g      = nullptr;
            if ( cudaStreamBeginCapture( cap_, cudaStreamCaptureModeThreadLocal ) != cudaSuccess )
            {
                stream_ref() = saved;
                throw std::runtime_error( "GraphReplay: cudaStreamBeginCapture failed" );
            }
            try
            {
                solve( inner_, A, x, b );
            }
            catch ( ... )
            {
                cudaStreamEndCapture( cap_, &g );
                if ( g )
                    cudaGraphDestroy( g );
                stream_ref() = saved;
                throw;
            }
            const cudaError_t ec = cudaStreamEndCapture( cap_, &g );
            stream_ref()         = saved;
            cudaGraphExec_t e    = nullptr;
            if ( ec != cudaSuccess || cudaGraphInstantiate( &e, g, 0 ) != cudaSuccess )
            {
                if ( g )
                    cudaGraphDestroy( g );
                throw std::runtime_error( "GraphReplay: capturing the solver failed" );
            }
            cudaGraphDestroy( g );
            it = execs_.emplace( std::move( key ), e ).first;
        }
        if ( cudaGraphLaunch( it->second, stream() ) != cudaSuccess )
            throw std::runtime_error( "GraphReplay: cudaGraphLaunch failed" );
    }
    size_t graphs() const { return execs_.size(); }

  private:
    Inner&                                                     inner_;
    bool                                                       enabled_;
    bool                                                       warm_ = false;
    cudaStream_t                                               cap_  = nullptr;
    std::map< std::vector< const void* >, cudaGraphExec_t > execs_;
};

// BlockTriangularPreconditioner2x2 (block_preconditioner_2x2.hpp:145-217)
template < typename Block11, typename Block12, typename Prec11, typename Prec22, typename BV >
class BlockTriangularPreconditioner2x2
{
  public:
    BlockTriangularPreconditioner2x2( Block11& a11, Block12& a12, BV tmp, Prec11& p11, Prec22& p22 )
    : a11_( a11 ), a12_( a12 ), tmp_( tmp ), p11_( p11 ), p22_( p22 )
    {}
    template < typename Op >
    void solve_impl( Op&, BV& x, const BV& b )
    {
        using S = typename BV::ScalarType;
        solve( p22_, a11_, x.block_2(), b.block_2() );
        apply( a12_, x.block_2(), tmp_.block_1() );
        lincomb( tmp_.block_1(), { S( 1 ), S( 1 ) }, { tmp_.block_1(), b.block_1() } );
        lincomb( x.block_2(), { S( -1 ) }, { x.block_2() } );
        solve( p11_, a11_, x.block_1(), tmp_.block_1() );
    }

  private:
    Block11& a11_;
    Block12& a12_;
    BV       tmp_;
    Prec11&  p11_;
    Prec22&  p22_;
};

// BlockDiagonalPreconditioner2x2 (block_preconditioner_2x2.hpp:38-100):
// x_1 = P11(b_1), x_2 = P22(b_2)
template < typename Block11, typename Prec11, typename Prec22, typename BV >
class BlockDiagonalPreconditioner2x2
{
  public:
    BlockDiagonalPreconditioner2x2( Block11& a11, Prec11& p11, Prec22& p22 ) : a11_( a11 ), p11_( p11 ), p22_( p22 ) {}
    template < typename Op >
    void solve_impl( Op&, BV& x, const BV& b )
    {
        solve( p11_, a11_, x.block_1(), b.block_1() );
        solve( p22_, a11_, x.block_2(), b.block_2() );
    }

  private:
    Block11& a11_;
    Prec11&  p11_;
    Prec22&  p22_;
};

// swap of two vector handles (the VectorLike swap_impl)
template < typename V >
void swap_vectors( V& a, V& b )
{
    a.swap_impl( b );
}

// Preconditioned MINRES (pminres.hpp:30-175): Lanczos with the
// preconditioner's inner product, Givens QR, short recurrences; stops on the
// preconditioned residual estimate |eta|.
template < typename Op, typename Prec = IdentitySolver< Op > >
class PMINRES
{
  public:
    using V = typename Op::SrcVectorType;
    PMINRES( IterativeSolverParameters prm, std::vector< V > tmps, Prec prec = Prec() )
    : prm_( prm ), tmp_( std::move( tmps ) ), prec_( prec )
    {
        if ( tmp_.size() < 7 )
            throw std::runtime_error( "PMINRES: needs 7 temporary vectors" );
    }
    SolverStatistics stats;
    void             solve_impl( Op& A, V& x, const V& b )
    {
        using S     = typename V::ScalarType;
        auto& az    = tmp_[0];
        auto& vjm1  = tmp_[1];
        auto& vj    = tmp_[2];
        auto& wjm1  = tmp_[3];
        auto& wj    = tmp_[4];
        auto& zjp1  = tmp_[5];
        auto& z     = tmp_[6];
        stats       = {};
        assign( vjm1, S( 0 ) );
        assign( wj, S( 0 ) );
        assign( wjm1, S( 0 ) );
        apply( A, x, vj );
        lincomb( vj, { S( 1 ), S( -1 ) }, { b, vj } );
        assign( z, S( 0 ) );
        solve( prec_, A, z, vj );
        double gjm1 = 1.0, gj = std::sqrt( double( dot( z, vj ) ) ), eta = gj;
        double sjm1 = 0.0, sj = 0.0, cjm1 = 1.0, cj = 1.0;
        const double r0 = gj;
        stats.relative_residuals.push_back( 1.0 );
        if ( r0 < prm_.absolute_residual_tolerance )
            return;
        for ( int it = 1; it <= prm_.max_iterations; ++it )
        {
            lincomb( z, { S( 1.0 / gj ) }, { z } );
            apply( A, z, az );
            const double delta = double( dot( az, z ) );
            lincomb( vjm1, { S( 1 ), S( -delta / gj ), S( -gj / gjm1 ) }, { az, vj, vjm1 } );
            swap_vectors( vjm1, vj );
            assign( zjp1, S( 0 ) );
            solve( prec_, A, zjp1, vj );
            const double gjp1 = std::sqrt( double( dot( zjp1, vj ) ) );
            const double a0 = cj * delta - cjm1 * sj * gj;
            const double a1 = std::sqrt( a0 * a0 + gjp1 * gjp1 );
            const double a2 = sj * delta + cjm1 * cj * gj;
            const double a3 = sjm1 * gj;
            const double cjp1 = a0 / a1, sjp1 = gjp1 / a1;
            lincomb( wjm1, { S( 1.0 / a1 ), S( -a3 / a1 ), S( -a2 / a1 ) }, { z, wjm1, wj } );
            swap_vectors( wjm1, wj );
            lincomb( x, { S( 1 ), S( cjp1 * eta ) }, { x, wj } );
            eta = -sjp1 * eta;
            const double ar = std::abs( eta ), rr = ar / r0;
            stats.relative_residuals.push_back( rr );
            stats.iterations = it;
            if ( rr <= prm_.relative_residual_tolerance || ar < prm_.absolute_residual_tolerance )
                return;
            swap_vectors( z, zjp1 );
            gjm1 = gj, gj = gjp1;
            cjm1 = cj, cj = cjp1;
            sjm1 = sj, sj = sjp1;
        }
    }

  private:
    IterativeSolverParameters prm_;
    std::vector< V >          tmp_;
    Prec                      prec_;
};

// small dense solve with full pivoting (the reference uses Eigen's
// fullPivLu for BiCGStab(l)'s l x l minimal-residual system)
inline std::vector< double > dense_solve_full_pivot( std::vector< double > M, std::vector< double > rhs, int n )
{
    std::vector< int > colp( n );
    for ( int i = 0; i < n; ++i )
        colp[i] = i;
    for ( int k = 0; k < n; ++k )
    {
        int    pi = k, pj = k;
        double best = -1.0;
        for ( int i = k; i < n; ++i )
            for ( int j = k; j < n; ++j )
                if ( std::abs( M[i * n + j] ) > best )
                    best = std::abs( M[i * n + j] ), pi = i, pj = j;
        if ( pi != k )
        {
            for ( int j = 0; j < n; ++j )
                std::swap( M[k * n + j], M[pi * n + j] );
            std::swap( rhs[k], rhs[pi] );
        }
        if ( pj != k )
        {
            for ( int i = 0; i < n; ++i )
                std::swap( M[i * n + k], M[i * n + pj] );
            std::swap( colp[k], colp[pj] );
        }
        if ( M[k * n + k] == 0.0 )
            continue;
        for ( int i = k + 1; i < n; ++i )
        {
            const double f = M[i * n + k] / M[k * n + k];
            for ( int j = k; j < n; ++j )
                M[i * n + j] -= f * M[k * n + j];
            rhs[i] -= f * rhs[k];
        }
    }
    std::vector< double > y( n, 0.0 ), out( n, 0.0 );
    for ( int i = n - 1; i >= 0; --i )
    {
        double v = rhs[i];
        for ( int j = i + 1; j < n; ++j )
            v -= M[i * n + j] * y[j];
        y[i] = M[i * n + i] != 0.0 ? v / M[i * n + i] : 0.0;
    }
    for ( int i = 0; i < n; ++i )
        out[colp[i]] = y[i];
    return out;
}

// Preconditioned BiCGStab(l) (pbicgstab.hpp:29-290): l BiCG steps and an
// l-dimensional minimal-residual update per iteration, left preconditioning;
// the shadow residual is the deterministic randomize of this library, or a
// given field (set_shadow: the reference draws its own, pbicgstab.hpp:98).
template < typename Op, typename Prec = IdentitySolver< Op > >
class PBiCGStab
{
  public:
    using V = typename Op::SrcVectorType;
    PBiCGStab( int l, IterativeSolverParameters prm, std::vector< V > tmps, Prec prec = Prec() )
    : l_( l ), prm_( prm ), tmp_( std::move( tmps ) ), prec_( prec )
    {
        if ( int( tmp_.size() ) < 2 * ( l + 1 ) + 2 )
            throw std::runtime_error( "PBiCGStab: needs 2 (l + 1) + 2 temporary vectors" );
    }
    SolverStatistics stats;
    // use `shadow` as the shadow residual of every later solve instead of a random field
    void set_shadow( const V& shadow )
    {
        assign( rshadow(), shadow );
        shadow_given_ = true;
    }
    void solve_impl( Op& A, V& x, const V& b )
    {
        using S = typename V::ScalarType;
        stats   = {};
        if ( !shadow_given_ )
            randomize( rshadow() );
        for ( int j = 0; j < l_ + 1; ++j )
            assign( us( j ), S( 0 ) );
        apply( A, x, rs( 0 ) );
        lincomb( rs( 0 ), { S( 1 ), S( -1 ) }, { b, rs( 0 ) } );
        precondition( A, rs( 0 ) );
        const double r0 = std::sqrt( double( dot( rs( 0 ), rs( 0 ) ) ) );
        double       ar = r0;
        stats.relative_residuals.push_back( 1.0 );
        if ( r0 < prm_.absolute_residual_tolerance )
            return;
        double omega = 1.0, sigma = 1.0;
        int    it    = 1;
        for ( ; it < prm_.max_iterations; ++it )
        {
            sigma = -omega * sigma;
            for ( int j = 0; j < l_; ++j )
            {
                const double rho  = double( dot( rshadow(), rs( j ) ) );
                const double beta = rho / sigma;
                for ( int i = 0; i <= j; ++i )
                    lincomb( us( i ), { S( 1 ), S( -beta ) }, { rs( i ), us( i ) } );
                apply( A, us( j ), us( j + 1 ) );
                precondition( A, us( j + 1 ) );
                sigma             = double( dot( rshadow(), us( j + 1 ) ) );
                const double alpha = rho / sigma;
                for ( int i = 0; i <= j; ++i )
                    lincomb( rs( i ), { S( 1 ), S( -alpha ) }, { rs( i ), us( i + 1 ) } );
                apply( A, rs( j ), rs( j + 1 ) );
                precondition( A, rs( j + 1 ) );
                lincomb( x, { S( 1 ), S( alpha ) }, { x, us( 0 ) } );
            }
            std::vector< double > M( l_ * l_ ), m0( l_ );
            for ( int j = 1; j <= l_; ++j )
                m0[j - 1] = double( dot( rs( 0 ), rs( j ) ) );
            for ( int i = 0; i < l_; ++i )
                for ( int j = 0; j < l_; ++j )
                    M[i * l_ + j] = double( dot( rs( i + 1 ), rs( j + 1 ) ) );
            const auto g = dense_solve_full_pivot( M, m0, l_ );
            for ( int j = 1; j <= l_; ++j )
                lincomb( us( 0 ), { S( 1 ), S( -g[j - 1] ) }, { us( 0 ), us( j ) } );
            for ( int j = 0; j < l_; ++j )
                lincomb( x, { S( 1 ), S( g[j] ) }, { x, rs( j ) } );
            for ( int j = 1; j <= l_; ++j )
                lincomb( rs( 0 ), { S( 1 ), S( -g[j - 1] ) }, { rs( 0 ), rs( j ) } );
            omega            = g[l_ - 1];
            ar               = std::sqrt( double( dot( rs( 0 ), rs( 0 ) ) ) );
            stats.iterations = it;
            stats.relative_residuals.push_back( ar / r0 );
            if ( ar / r0 <= prm_.relative_residual_tolerance || ar < prm_.absolute_residual_tolerance )
                return;
        }
    }

  private:
    V&   rshadow() { return tmp_[0]; }
    V&   rs( int i ) { return tmp_[1 + i]; }
    V&   us( int i ) { return tmp_[1 + l_ + 1 + i]; }
    V&   tmp_prec() { return tmp_[1 + 2 * ( l_ + 1 )]; }
    void precondition( Op& A, V& v )
    {
        if constexpr ( !std::is_same_v< Prec, IdentitySolver< Op > > )
        {
            assign( tmp_prec(), v );
            solve( prec_, A, tmp_prec(), v );
            assign( v, tmp_prec() );
        }
    }
    int                       l_;
    IterativeSolverParameters prm_;
    std::vector< V >          tmp_;
    Prec                      prec_;
    bool                      shadow_given_ = false;
};

// FGMRES(m) with modified Gram-Schmidt Arnoldi and Givens rotations
// (fgmres.hpp:108-330), including the reference's fall-back of skipping the
// preconditioner when it returns NaN / Inf.
template < typename Op, typename Prec >
class FGMRES
{
  public:
    using V = typename Op::SrcVectorType;
    FGMRES( std::vector< V > tmps, int restart, IterativeSolverParameters prm, Prec& prec )
    : tmp_( std::move( tmps ) ), m_( restart ), prm_( prm ), prec_( prec )
    {
        if ( int( tmp_.size() ) < 2 * m_ + 4 )
            throw std::runtime_error( "FGMRES: needs 2 * restart + 4 temporary vectors" );
        hdev_ = device_alloc< double >( size_t( m_ ) + 2 );
        hhost_.assign( size_t( m_ ) + 2, 0.0 );
    }
    SolverStatistics stats;
    int              preconditioner_skips = 0;
    void             set_parameters( const IterativeSolverParameters& prm ) { prm_ = prm; }

    void solve_impl( Op& A, V& x, const V& b )
    {
        using S = typename V::ScalarType;
        stats   = {};
        auto& r = tmp_[0];
        apply( A, x, r );
        lincomb( r, { S( 1 ), S( -1 ) }, { b, r } );
        double       beta0 = std::sqrt( double( dot( r, r ) ) );
        const double r0    = beta0;
        stats.relative_residuals.push_back( 1.0 );
        if ( beta0 <= prm_.absolute_residual_tolerance )
            return;
        const int offV = 1, offZ = offV + m_ + 1, idxW = offZ + m_, idxAcc = idxW + 1;
        std::vector< double > H( ( m_ + 1 ) * m_ ), g( m_ + 1 ), cs( m_ + 1 ), sn( m_ + 1 );
        auto h = [&]( int i, int j ) -> double& { return H[i * m_ + j]; };
        int  total = 0;
        while ( total < prm_.max_iterations )
        {
            lincomb( tmp_[offV], { S( 1.0 / beta0 ) }, { r } );
            std::fill( H.begin(), H.end(), 0.0 );
            std::fill( g.begin(), g.end(), 0.0 );
            std::fill( cs.begin(), cs.end(), 0.0 );
            std::fill( sn.begin(), sn.end(), 0.0 );
            g[0]      = beta0;
            int inner = 0;
            for ( int j = 0; j < m_ && total < prm_.max_iterations; ++j, ++total )
            {
                auto& vj = tmp_[offV + j];
                auto& zj = tmp_[offZ + j];
                assign( zj, S( 0 ) );
                solve( prec_, A, zj, vj );
                auto&   w  = tmp_[idxW];
                double* hd = hdev_.get();
                // w = A z, then modified Gram-Schmidt (fgmres.hpp:197-209):
                // h_ij = <w, v_i>, w -= h_ij v_i for i = 0..j, then |w|; each
                // pass fuses the update by v_{i-1} with the projection on v_i
                // and the coefficients stay on the device until one read at
                // the end.  A NaN / Inf in z (the reference replaces z by v,
                // fgmres.hpp:180-186) reaches every h_ij through A z, so the
                // column read doubles as the check and the step is redone
                // with z = v.
                auto arnoldi = [&]() {
                    apply( A, zj, w );
                    const auto sw = segments( w );
                    for ( int i = 0; i <= j + 1; ++i )
                    {
                        const auto sv = segments( tmp_[offV + std::min( i, j )] );
                        const auto su = segments( tmp_[offV + std::max( i - 1, 0 )] );
                        axpy_dot( sw, i > 0 ? &su : nullptr, i > 0 ? hd + i - 1 : nullptr, i <= j ? &sv : nullptr,
                                  nullptr, hd + i );
                    }
                    if ( cudaMemcpyAsync( hhost_.data(), hd, sizeof( double ) * ( j + 2 ), cudaMemcpyDeviceToHost,
                                          stream() ) != cudaSuccess ||
                         cudaStreamSynchronize( stream() ) != cudaSuccess )
                        throw std::runtime_error( "FGMRES: reading the Hessenberg column failed" );
                    for ( int i = 0; i <= j + 1; ++i )
                        if ( !std::isfinite( hhost_[i] ) )
                            return false;
                    return true;
                };
                if ( !arnoldi() )
                {
                    assign( zj, vj );
                    ++preconditioner_skips;
                    arnoldi();
                }
                for ( int i = 0; i <= j; ++i )
                    h( i, j ) = hhost_[i];
                const double hj1 = std::sqrt( hhost_[j + 1] );
                if ( hj1 < std::numeric_limits< double >::epsilon() * r0 )
                {
                    h( j + 1, j ) = 0;
                    inner         = j + 1;
                    break;
                }
                h( j + 1, j ) = hj1;
                lincomb( tmp_[offV + j + 1], { S( 1.0 / hj1 ) }, { w } );
                for ( int i = 0; i < j; ++i )
                {
                    const double t = cs[i] * h( i, j ) + sn[i] * h( i + 1, j );
                    h( i + 1, j )  = -sn[i] * h( i, j ) + cs[i] * h( i + 1, j );
                    h( i, j )      = t;
                }
                const double a = h( j, j ), bb = h( j + 1, j ), rab = std::hypot( a, bb );
                cs[j]          = rab == 0 ? 1.0 : a / rab;
                sn[j]          = rab == 0 ? 0.0 : bb / rab;
                h( j, j )      = rab;
                h( j + 1, j )  = 0;
                if ( std::abs( rab ) < std::numeric_limits< double >::epsilon() )
                {
                    inner = j;
                    break;
                }
                const double gj = g[j], gj1 = g[j + 1];
                g[j]     = cs[j] * gj + sn[j] * gj1;
                g[j + 1] = -sn[j] * gj + cs[j] * gj1;
                stats.relative_residuals.push_back( std::abs( g[j + 1] ) / r0 );
                stats.iterations = total + 1;
                inner            = j + 1;
                if ( std::abs( g[j + 1] ) / r0 <= prm_.relative_residual_tolerance ||
                     std::abs( g[j + 1] ) < prm_.absolute_residual_tolerance )
                {
                    ++total;
                    break;
                }
            }
            std::vector< double > y( inner, 0.0 );
            for ( int row = inner - 1; row >= 0; --row )
            {
                double s = g[row];
                for ( int col = row + 1; col < inner; ++col )
                    s -= h( row, col ) * y[col];
                y[row] = s / h( row, row );
            }
            auto& acc = tmp_[idxAcc];
            assign( acc, S( 0 ) );
            for ( int i = 0; i < inner; ++i )
                lincomb( acc, { S( 1 ), S( y[i] ) }, { acc, tmp_[offZ + i] } );
            lincomb( x, { S( 1 ), S( 1 ) }, { x, acc } );
            apply( A, x, r );
            lincomb( r, { S( 1 ), S( -1 ) }, { b, r } );
            beta0 = std::sqrt( double( dot( r, r ) ) );
            true_relative_residual = beta0 / r0;
            if ( beta0 <= prm_.absolute_residual_tolerance || beta0 / r0 <= prm_.relative_residual_tolerance )
                return;
        }
    }
    double true_relative_residual = 1.0;

  private:
    std::shared_ptr< double > hdev_;
    std::vector< double >     hhost_;
    std::vector< V >          tmp_;
    int                       m_;
    IterativeSolverParameters prm_;
    Prec&                     prec_;
};

}  // namespace tn
