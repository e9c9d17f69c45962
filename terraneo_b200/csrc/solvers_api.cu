// C ABI of the solver drivers: PCG on the scalar Laplace (the CG benchmark
// configuration) and the Stokes solver (FGMRES + block-triangular
// preconditioner, geometric multigrid on the viscous block with Chebyshev
// smoothing and a PCG coarse solve, lumped inverse KMass(1/eta) Schur
// approximation), composed as in the reference's mantle-circulation app
// (apps/mantlecirculation/mantlecirculation.cpp:486-735).
//
// The multigrid preconditioner runs in FP32 (operators, smoothers, transfers,
// FP32 viscosity) inside the FP64 outer FGMRES when mg_fp32 != 0; the outer
// residual, dot products (compensated), Schur diagonal and the coarsest-level
// PCG stay FP64.  Coarser-level viscous operators are re-discretised with the
// viscosity injected from the finest level.
#include <functional>
#include <memory>

#include "../cpp/tn/enforcement.hpp"
#include "../cpp/tn/solvers.hpp"
#include "common.cuh"

using namespace tn;

namespace {

using A64 = EpsilonDivDivKerngen< double >;
using A32 = EpsilonDivDivKerngen< float >;
using V64 = ViscousOp< double >;
using V32 = ViscousOp< float >;

// FP32 V-cycle's coarsest solve done in FP64: cast, PCG, cast back
struct CoarseFp64
{
    std::shared_ptr< DevicePCG< V64 > > pcg;
    std::shared_ptr< V64 >              A;
    VectorQ1Vec< double >               x, b;
    void                                solve_impl( V32&, VectorQ1Vec< float >& xo, const VectorQ1Vec< float >& bi )
    {
        cast( b, bi );
        assign( x, 0.0 );
        solve( *pcg, *A, x, b );
        cast( xo, x );
    }
};

template < typename T, typename Coarse >
using MG = Multigrid< ViscousOp< T >, ProlongationVecConstant< T >, RestrictionVecConstant< T >,
                      Chebyshev< ViscousOp< T > >, Coarse >;

// FP32 multigrid as a preconditioner of the FP64 viscous block
template < typename Inner >
struct Fp32Preconditioner
{
    std::shared_ptr< Inner > mg;
    std::shared_ptr< V32 >   A;
    VectorQ1Vec< float >     x, b;
    void                     solve_impl( A64&, VectorQ1Vec< double >& xo, const VectorQ1Vec< double >& bi )
    {
        cast( b, bi );
        assign( x, 0.0f );
        solve( *mg, *A, x, b );
        cast( xo, x );
    }
};

// FP32 multigrid on FP32 vectors (the inner system of the refinement form)
template < typename Inner >
struct Fp32Direct
{
    std::shared_ptr< Inner > mg;
    std::shared_ptr< V32 >   A;
    void solve_impl( A32&, VectorQ1Vec< float >& x, const VectorQ1Vec< float >& b ) { solve( *mg, *A, x, b ); }
};

template < typename Inner >
struct Fp64Preconditioner
{
    std::shared_ptr< Inner > mg;
    std::shared_ptr< V64 >   A;
    void solve_impl( A64&, VectorQ1Vec< double >& x, const VectorQ1Vec< double >& b ) { solve( *mg, *A, x, b ); }
};

}  // namespace

struct tn_stokes_solver
{
    tn_stokes_params                                         prm{};
    std::vector< Mesh >                                      mesh; // index = level
    std::vector< VectorQ1Scalar< double > >                  k64;
    std::vector< VectorQ1Scalar< float > >                   k32;
    std::vector< std::shared_ptr< double > >                 mats64; // GCA matrices per coarse level
    std::vector< std::shared_ptr< float > >                  mats32;
    std::shared_ptr< uint8_t >                               gca_marks; // adaptive GCA: marked coarsest cells
    std::shared_ptr< A64 >                                   A64fine;
    std::unique_ptr< EpsDivDivStokes< double > >             K;
    std::unique_ptr< Gradient< double > >                    BT;
    std::function< void( VectorQ1IsoQ2Q1< double >&, const VectorQ1IsoQ2Q1< double >& ) > run;
    std::vector< double >                                    history;
    std::vector< double >                                    chebyshev_estimates;
    int                                                      iterations = 0;
    double                                                   relres     = 1.0;
    int                                                      skips      = 0;
};

namespace {

template < typename Op >
VectorQ1Vec< typename Op::ScalarType > inverse_diagonal_vec( Op& A, const Mesh& m )
{
    using T = typename Op::ScalarType;
    VectorQ1Vec< T > ones( m ), d( m );
    assign( ones, T( 1 ) );
    A.set_diagonal( true );
    apply( A, ones, d );
    A.set_diagonal( false );
    invert_entries( d );
    return d;
}

// viscous operator of level l: stored GCA matrices on coarse levels when
// enabled, matrix-free kerngen otherwise
template < typename T >
ViscousOp< T > level_op( tn_stokes_solver& s, int l )
{
    BoundaryConditions bcs{ s.prm.bc_cmb, s.prm.bc_surface };
    if ( s.prm.gca && l < s.prm.level )
    {
        if constexpr ( std::is_same_v< T, double > )
            return ViscousOp< T >( std::make_shared< StoredEpsilonDivDiv< T > >( s.mesh[l], s.mats64[l], bcs ) );
        else
            return ViscousOp< T >( std::make_shared< StoredEpsilonDivDiv< T > >( s.mesh[l], s.mats32[l], bcs ) );
    }
    if constexpr ( std::is_same_v< T, double > )
        return ViscousOp< T >( std::make_shared< EpsilonDivDivKerngen< T > >( s.mesh[l], s.k64[l], bcs, false ) );
    else
        return ViscousOp< T >( std::make_shared< EpsilonDivDivKerngen< T > >( s.mesh[l], s.k32[l], bcs, false ) );
}

// GCA matrices of levels [Lmin, L-1] (mantlecirculation.cpp:580-592): the
// finest from the Neumann kerngen matrices of the finest viscosity, each
// coarser one from the stored matrices above it
// With gca == 3 (adaptive) the coarsest cells are marked once from the finest viscosity
// (GCAElementsCollector with level range L - Lmin) and each level keeps the GCA matrices of the cells below a
// marked cell, the kerngen matrices of its injected viscosity elsewhere (the reference's Selective storage
// assembles those on the fly; here every cell's matrix is stored, the apply is the same stored-matrix kernel).
void build_gca( tn_stokes_solver& s )
{
    const int L = s.prm.level, Lmin = L - s.prm.mg_levels + 1, mode = s.prm.gca == 2 ? 1 : 0;
    const bool adaptive = s.prm.gca == 3;
    s.mats64.assign( L + 1, nullptr );
    s.mats32.assign( L + 1, nullptr );
    if ( adaptive )
    {
        const size_t N0 = size_t( 1 ) << Lmin;
        s.gca_marks     = device_alloc< uint8_t >( 10 * N0 * N0 * N0 );
        check( tn_gca_elements_f64( s.mesh[L].get(), s.k64[L].data(), L - Lmin, s.gca_marks.get(), stream() ),
               "gca_elements" );
    }
    for ( int l = L - 1; l >= Lmin; --l )
    {
        size_t n = 0;
        check( tn_local_matrix_count( s.mesh[l].get(), &n ), "local_matrix_count" );
        s.mats64[l] = device_alloc< double >( n );
        check( tn_gca_coarsen_f64( s.mesh[l + 1].get(), s.mesh[l].get(), l == L - 1 ? s.k64[L].data() : nullptr,
                                   l == L - 1 ? nullptr : s.mats64[l + 1].get(), mode, s.mats64[l].get(), stream() ),
               "gca_coarsen" );
        if ( adaptive )
            check( tn_agca_unmarked_local_matrices_f64( s.mesh[l].get(), s.k64[l].data(), s.gca_marks.get(), l - Lmin,
                                                        s.mats64[l].get(), stream() ),
                   "agca unmarked matrices" );
        if ( s.prm.mg_fp32 )
        {
            s.mats32[l] = device_alloc< float >( n );
            check( tn_array_cast_f64_to_f32( n, s.mats64[l].get(), s.mats32[l].get(), stream() ), "cast matrices" );
        }
    }
}

// builds the multigrid hierarchy in precision T over levels [Lmin, L]
template < typename T, typename Coarse >
std::shared_ptr< MG< T, Coarse > > build_mg( tn_stokes_solver& s, std::vector< std::shared_ptr< ViscousOp< T > > >& ops,
                                             Coarse coarse )
{
    const auto&                                 prm = s.prm;
    const int                                   L = prm.level, Lmin = prm.level - prm.mg_levels + 1;
    std::vector< ProlongationVecConstant< T > > P;
    std::vector< RestrictionVecConstant< T > >  R;
    std::vector< ViscousOp< T > >               Ac;
    std::vector< VectorQ1Vec< T > >             tr, te, tmp;
    std::vector< Chebyshev< ViscousOp< T > > >  sm;
    for ( int l = Lmin; l <= L; ++l )
    {
        const Mesh& m = s.mesh[l];
        ops.push_back( std::make_shared< ViscousOp< T > >( level_op< T >( s, l ) ) );
        auto inv = inverse_diagonal_vec( *ops.back(), m );
        sm.emplace_back( prm.chebyshev_order, inv, std::vector< VectorQ1Vec< T > >{ VectorQ1Vec< T >( m ), VectorQ1Vec< T >( m ) },
                         prm.smoothing_steps, prm.power_iterations );
        if ( prm.chebyshev_estimates )
            sm.back().set_max_eigenvalue_estimate( prm.chebyshev_estimates[l - Lmin] );
        tmp.emplace_back( m );
        if ( l < L )
        {
            Ac.push_back( *ops.back() );
            tr.emplace_back( m );
            te.emplace_back( m );
            P.emplace_back( s.mesh[l + 1], m, OperatorApplyMode::Add );
            R.emplace_back( s.mesh[l + 1], m );
        }
    }
    return std::make_shared< MG< T, Coarse > >( P, R, Ac, tr, te, tmp, sm, coarse, prm.vcycles );
}

template < typename Prec11 >
void finish( tn_stokes_solver& s, std::shared_ptr< Prec11 > p11 )
{
    const auto& prm = s.prm;
    const int   L   = prm.level;
    BoundaryConditions bcs{ prm.bc_cmb, prm.bc_surface };
    s.K  = std::make_unique< EpsDivDivStokes< double > >( s.mesh[L], s.mesh[L - 1], s.k64[L], bcs );
    s.BT = std::make_unique< Gradient< double > >( s.mesh[L], s.mesh[L - 1], bcs );
    // Schur: lumped KMass with k = 1 / eta on the pressure level (mantlecirculation.cpp:684-699)
    VectorQ1Scalar< double > kp( s.mesh[L - 1] ), ones( s.mesh[L - 1] ), dp( s.mesh[L - 1] );
    assign( kp, s.k64[L - 1] );
    invert_entries( kp );
    assign( ones, 1.0 );
    KMass< double > pm( s.mesh[L - 1], kp, 2 );
    apply( pm, ones, dp );
    auto p22 = std::make_shared< DiagonalSolver< KMass< double >, VectorQ1Scalar< double > > >( dp );
    auto a11 = s.A64fine;
    IterativeSolverParameters ip{ prm.max_iterations, prm.relative_tolerance, prm.absolute_tolerance };
    tn_stokes_solver*         sp = &s;
    if ( prm.outer == 1 )
    {
        // PMINRES with the block-diagonal preconditioner (pminres.hpp, block_preconditioner_2x2.hpp:38-100)
        using BD  = BlockDiagonalPreconditioner2x2< A64, Prec11, DiagonalSolver< KMass< double >, VectorQ1Scalar< double > >,
                                                    VectorQ1IsoQ2Q1< double > >;
        auto prec  = std::make_shared< BD >( *a11, *p11, *p22 );
        auto graph = std::make_shared< GraphReplay< BD > >( *prec, prm.eager == 0 );
        std::vector< VectorQ1IsoQ2Q1< double > > tmps;
        for ( int i = 0; i < 7; ++i )
            tmps.emplace_back( s.mesh[L], s.mesh[L - 1] );
        auto mr = std::make_shared< PMINRES< EpsDivDivStokes< double >, GraphReplay< BD >& > >( ip, tmps, *graph );
        s.run = [sp, mr, prec, graph, p11, p22, a11]( VectorQ1IsoQ2Q1< double >& x,
                                                      const VectorQ1IsoQ2Q1< double >& b ) {
            solve( *mr, *sp->K, x, b );
            sp->history    = mr->stats.relative_residuals;
            sp->iterations = mr->stats.iterations;
            sp->relres     = mr->stats.relative_residuals.back();
            sp->skips      = 0;
        };
        return;
    }
    using BT = BlockTriangularPreconditioner2x2< A64, Gradient< double >, Prec11,
                                                 DiagonalSolver< KMass< double >, VectorQ1Scalar< double > >,
                                                 VectorQ1IsoQ2Q1< double > >;
    auto prec  = std::make_shared< BT >( *a11, *s.BT, VectorQ1IsoQ2Q1< double >( s.mesh[L], s.mesh[L - 1] ), *p11, *p22 );
    auto graph = std::make_shared< GraphReplay< BT > >( *prec, prm.eager == 0 );
    std::vector< VectorQ1IsoQ2Q1< double > > tmps;
    for ( int i = 0; i < 2 * prm.restart + 4; ++i )
        tmps.emplace_back( s.mesh[L], s.mesh[L - 1] );
    auto fg = std::make_shared< FGMRES< EpsDivDivStokes< double >, GraphReplay< BT > > >( tmps, prm.restart, ip, *graph );
    s.run = [sp, fg, prec, graph, p11, p22, a11]( VectorQ1IsoQ2Q1< double >& x, const VectorQ1IsoQ2Q1< double >& b ) {
        solve( *fg, *sp->K, x, b );
        sp->history    = fg->stats.relative_residuals;
        sp->iterations = fg->stats.iterations;
        sp->relres     = fg->true_relative_residual;
        sp->skips      = fg->preconditioner_skips;
    };
}

// Mixed-precision iterative refinement (outer = 2): the FP64 residual
// r = b - K x of the full Stokes system, one FGMRES cycle (at most `restart`
// iterations) on K32 d = r / |r| entirely in FP32 (Krylov vectors,
// Gram-Schmidt, operator, B, B^T, the block-triangular preconditioner with the
// FP32 V-cycle; the coarsest-level PCG stays FP64), and the FP64 update
// x += |r| d, until the FP64 residual meets the tolerance.  A cycle is the
// counterpart of one restart of the FP64 FGMRES(restart): the Krylov space is
// built in FP32 and the residual it restarts from is the true FP64 one.  A
// cycle stops early when its residual estimate reaches rtol / (the current
// relative residual); more inner cycles on the same FP32 system would only
// chase the FP32 rounding level.

template < typename MGT >
void finish_refine( tn_stokes_solver& s, std::shared_ptr< MGT > mg, std::shared_ptr< V32 > a32ml )
{
    const auto&        prm = s.prm;
    const int          L   = prm.level;
    const Mesh &       mu = s.mesh[L], &mp = s.mesh[L - 1];
    BoundaryConditions bcs{ prm.bc_cmb, prm.bc_surface };
    s.K  = std::make_unique< EpsDivDivStokes< double > >( mu, mp, s.k64[L], bcs );
    s.BT = std::make_unique< Gradient< double > >( mu, mp, bcs );
    auto K32  = std::make_shared< EpsDivDivStokes< float > >( mu, mp, s.k32[L], bcs );
    auto a11  = std::make_shared< A32 >( mu, s.k32[L], bcs, false );
    auto bt32 = std::make_shared< Gradient< float > >( mu, mp, bcs );
    // Schur: lumped KMass with k = 1 / eta on the pressure level (mantlecirculation.cpp:684-699), in FP32
    VectorQ1Scalar< double > kp( mp ), ones( mp ), dp( mp );
    VectorQ1Scalar< float >  dp32( mp );
    assign( kp, s.k64[L - 1] );
    invert_entries( kp );
    assign( ones, 1.0 );
    KMass< double > pm( mp, kp, 2 );
    apply( pm, ones, dp );
    cast( dp32, dp );
    using P22  = DiagonalSolver< KMass< float >, VectorQ1Scalar< float > >;
    using P11  = Fp32Direct< MGT >;
    using BTP  = BlockTriangularPreconditioner2x2< A32, Gradient< float >, P11, P22, VectorQ1IsoQ2Q1< float > >;
    auto p22   = std::make_shared< P22 >( dp32 );
    auto p11   = std::make_shared< P11 >( P11{ mg, a32ml } );
    auto prec  = std::make_shared< BTP >( *a11, *bt32, VectorQ1IsoQ2Q1< float >( mu, mp ), *p11, *p22 );
    auto graph = std::make_shared< GraphReplay< BTP > >( *prec, prm.eager == 0 );
    std::vector< VectorQ1IsoQ2Q1< float > > tmps;
    for ( int i = 0; i < 2 * prm.restart + 4; ++i )
        tmps.emplace_back( mu, mp );
    auto fg = std::make_shared< FGMRES< EpsDivDivStokes< float >, GraphReplay< BTP > > >(
        tmps, prm.restart, IterativeSolverParameters{ prm.restart, prm.relative_tolerance, 0.0 }, *graph );
    auto r64 = std::make_shared< VectorQ1IsoQ2Q1< double > >( mu, mp );
    auto d64 = std::make_shared< VectorQ1IsoQ2Q1< double > >( mu, mp );
    auto r32 = std::make_shared< VectorQ1IsoQ2Q1< float > >( mu, mp );
    auto d32 = std::make_shared< VectorQ1IsoQ2Q1< float > >( mu, mp );
    tn_stokes_solver* sp = &s;
    s.run = [sp, fg, prec, graph, p11, p22, a11, bt32, K32, r64, d64, r32, d32](
                VectorQ1IsoQ2Q1< double >& x, const VectorQ1IsoQ2Q1< double >& b ) {
        const auto& prm = sp->prm;
        auto        residual = [&]() {
            apply( *sp->K, x, *r64 );
            lincomb( *r64, { 1.0, -1.0 }, { b, *r64 } );
            return std::sqrt( dot( *r64, *r64 ) );
        };
        double       rn = residual();
        const double r0 = rn;
        sp->history     = { 1.0 };
        sp->skips       = 0;
        int total       = 0;
        while ( rn > prm.absolute_tolerance && rn / r0 > prm.relative_tolerance && total < prm.max_iterations )
        {
            const double rel = rn / r0;
            lincomb( *r64, { 1.0 / rn }, { *r64 } );
            cast( *r32, *r64 );
            assign( *d32, 0.0f );
            fg->set_parameters( IterativeSolverParameters{ std::min( prm.restart, prm.max_iterations - total ),
                                                           prm.relative_tolerance / rel, 0.0 } );
            solve( *fg, *K32, *d32, *r32 );
            const int its = fg->stats.iterations;
            total += its;
            sp->skips += fg->preconditioner_skips;
            fg->preconditioner_skips = 0;
            // inner estimates relative to the outer start: (inner relative residual) x (outer relative residual)
            for ( size_t i = 1; i < fg->stats.relative_residuals.size(); ++i )
                sp->history.push_back( fg->stats.relative_residuals[i] * rel );
            cast( *d64, *d32 );
            lincomb( x, { 1.0, rn }, { x, *d64 } );
            rn = residual();
            if ( !sp->history.empty() && its > 0 )
                sp->history.back() = rn / r0; // the cycle ends at the true FP64 residual
            if ( its == 0 )
                break;
        }
        sp->iterations = total;
        sp->relres     = rn / r0;
    };
}

}  // namespace

extern "C" int tn_stokes_solver_create( const tn_stokes_params* p, double r_min, double r_max, const double* k,
                                        tn_stokes_solver** out )
{
    TN_CHECK_ARG( p && k && out, "tn_stokes_solver_create: null argument" );
    *out = nullptr;
    TN_CHECK_ARG( p->mg_levels >= 2 && p->level - p->mg_levels + 1 >= 2 && p->level <= 8,
                  "tn_stokes_solver_create: need mg_levels >= 2, level - mg_levels + 1 >= 2 and level <= 8" );
    TN_CHECK_ARG( p->restart >= 1 && p->max_iterations >= 1, "tn_stokes_solver_create: bad Krylov parameters" );
    TN_CHECK_ARG( p->gca >= 0 && p->gca <= 3, "tn_stokes_solver_create: gca must be 0, 1, 2 or 3" );
    TN_CHECK_ARG( p->outer >= 0 && p->outer <= 2, "tn_stokes_solver_create: outer must be 0, 1 or 2" );
    TN_CHECK_ARG( p->outer != 2 || p->mg_fp32, "tn_stokes_solver_create: outer = 2 (refinement) needs mg_fp32 = 1" );
    try
    {
        auto s = std::make_unique< tn_stokes_solver >();
        s->prm = *p;
        if ( p->chebyshev_estimates )
        {
            // kept with the solver: the caller's array need not outlive this call
            s->chebyshev_estimates.assign( p->chebyshev_estimates, p->chebyshev_estimates + p->mg_levels );
            s->prm.chebyshev_estimates = s->chebyshev_estimates.data();
        }
        const int L = p->level, Lmin = L - p->mg_levels + 1;
        const int Llo = std::min( Lmin, L - 1 );
        s->mesh.resize( L + 1 );
        s->k64.resize( L + 1 );
        s->k32.resize( L + 1 );
        for ( int l = Llo; l <= L; ++l )
        {
            s->mesh[l] = Mesh( l, r_min, r_max );
            s->k64[l]  = VectorQ1Scalar< double >( s->mesh[l] );
            s->k32[l]  = VectorQ1Scalar< float >( s->mesh[l] );
        }
        check( cudaMemcpy( s->k64[L].data(), k, sizeof( double ) * s->mesh[L].stored_nodes(), cudaMemcpyDeviceToDevice ) ==
                       cudaSuccess
                   ? TN_OK
                   : TN_ERR_CUDA,
               "copy viscosity" );
        for ( int l = L - 1; l >= Llo; --l )
        {
            const double* src[1] = { s->k64[l + 1].data() };
            double*       dst[1] = { s->k64[l].data() };
            check( tn_injection_f64( s->mesh[l + 1].get(), s->mesh[l].get(), 1, src, dst, nullptr ), "injection" );
        }
        for ( int l = Llo; l <= L; ++l )
        {
            const double* src[1] = { s->k64[l].data() };
            float*        dst[1] = { s->k32[l].data() };
            check( tn_vec_cast_f64_to_f32( s->mesh[l].get(), 1, dst, src, nullptr ), "cast viscosity" );
        }
        // GCA coarse operators (optional), the FP64 fine operator of the outer system
        BoundaryConditions bcs{ p->bc_cmb, p->bc_surface };
        if ( p->gca )
            build_gca( *s );
        s->A64fine = std::make_shared< A64 >( s->mesh[L], s->k64[L], bcs, false );
        // FP64 coarsest solve (both precisions): device-resident PCG; the 4th
        // temporary lets the stored-matrix (GCA) operator use the fused steps
        auto Ac64 = std::make_shared< V64 >( level_op< double >( *s, Lmin ) );
        std::vector< VectorQ1Vec< double > > ct;
        for ( int i = 0; i < 4; ++i )
            ct.emplace_back( s->mesh[Lmin] );
        auto pcg = std::make_shared< DevicePCG< V64 > >(
            IterativeSolverParameters{ p->coarse_max_iterations, p->coarse_relative_tolerance, 1e-16 }, ct );
        if ( p->mg_fp32 )
        {
            std::vector< std::shared_ptr< V32 > > ops32;
            CoarseFp64 cs{ pcg, Ac64, VectorQ1Vec< double >( s->mesh[Lmin] ), VectorQ1Vec< double >( s->mesh[Lmin] ) };
            auto       mg  = build_mg< float, CoarseFp64 >( *s, ops32, cs );
            if ( p->outer == 2 )
            {
                finish_refine( *s, mg, ops32.back() );
                *out = s.release();
                return TN_OK;
            }
            auto       p11 = std::make_shared< Fp32Preconditioner< MG< float, CoarseFp64 > > >(
                Fp32Preconditioner< MG< float, CoarseFp64 > >{ mg, ops32.back(), VectorQ1Vec< float >( s->mesh[L] ),
                                                                VectorQ1Vec< float >( s->mesh[L] ) } );
            finish( *s, p11 );
        }
        else
        {
            std::vector< std::shared_ptr< V64 > > ops64;
            auto mg  = build_mg< double, DevicePCG< V64 > >( *s, ops64, *pcg );
            auto p11 = std::make_shared< Fp64Preconditioner< MG< double, DevicePCG< V64 > > > >(
                Fp64Preconditioner< MG< double, DevicePCG< V64 > > >{ mg, ops64.back() } );
            finish( *s, p11 );
        }
        *out = s.release();
        return TN_OK;
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_stokes_solver_create: " ) + e.what() );
        return TN_ERR_STATE;
    }
}

extern "C" int tn_stokes_solve( tn_stokes_solver* s, const double* const* f_u, const double* f_p, double* const* x_u,
                                double* x_p, int* iterations, double* relative_residual )
{
    TN_CHECK_ARG( s && f_u && f_p && x_u && x_p, "tn_stokes_solve: null argument" );
    try
    {
        const int                 L = s->prm.level;
        const size_t              nu = s->mesh[L].stored_nodes();
        VectorQ1IsoQ2Q1< double > b( s->mesh[L], s->mesh[L - 1] ), x( s->mesh[L], s->mesh[L - 1] );
        for ( int c = 0; c < 3; ++c )
        {
            TN_CUDA_TRY( cudaMemcpyAsync( b.block_1().comp( c ), f_u[c], sizeof( double ) * nu, cudaMemcpyDeviceToDevice ) );
            TN_CUDA_TRY( cudaMemcpyAsync( x.block_1().comp( c ), x_u[c], sizeof( double ) * nu, cudaMemcpyDeviceToDevice ) );
        }
        const size_t np = s->mesh[L - 1].stored_nodes();
        TN_CUDA_TRY( cudaMemcpyAsync( b.block_2().data(), f_p, sizeof( double ) * np, cudaMemcpyDeviceToDevice ) );
        TN_CUDA_TRY( cudaMemcpyAsync( x.block_2().data(), x_p, sizeof( double ) * np, cudaMemcpyDeviceToDevice ) );
        s->run( x, b );
        for ( int c = 0; c < 3; ++c )
            TN_CUDA_TRY( cudaMemcpyAsync( x_u[c], x.block_1().comp( c ), sizeof( double ) * nu, cudaMemcpyDeviceToDevice ) );
        TN_CUDA_TRY( cudaMemcpyAsync( x_p, x.block_2().data(), sizeof( double ) * np, cudaMemcpyDeviceToDevice ) );
        TN_CUDA_TRY( cudaDeviceSynchronize() );
        if ( iterations )
            *iterations = s->iterations;
        if ( relative_residual )
            *relative_residual = s->relres;
        return TN_OK;
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_stokes_solve: " ) + e.what() );
        return TN_ERR_STATE;
    }
}

extern "C" int tn_stokes_history( const tn_stokes_solver* s, double* out, int cap, int* n, int* preconditioner_skips )
{
    TN_CHECK_ARG( s, "tn_stokes_history: null solver" );
    const int m = int( s->history.size() );
    if ( n )
        *n = m;
    if ( out )
        for ( int i = 0; i < m && i < cap; ++i )
            out[i] = s->history[i];
    if ( preconditioner_skips )
        *preconditioner_skips = s->skips;
    return TN_OK;
}

extern "C" int tn_stokes_apply( tn_stokes_solver* s, const double* const* u, const double* p, double* const* ou,
                                double* op )
{
    TN_CHECK_ARG( s && u && p && ou && op, "tn_stokes_apply: null argument" );
    try
    {
        const int                 L = s->prm.level;
        VectorQ1IsoQ2Q1< double > src( s->mesh[L], s->mesh[L - 1] ), dst( s->mesh[L], s->mesh[L - 1] );
        const size_t              nu = s->mesh[L].stored_nodes(), np = s->mesh[L - 1].stored_nodes();
        for ( int c = 0; c < 3; ++c )
            TN_CUDA_TRY( cudaMemcpyAsync( src.block_1().comp( c ), u[c], sizeof( double ) * nu, cudaMemcpyDeviceToDevice ) );
        TN_CUDA_TRY( cudaMemcpyAsync( src.block_2().data(), p, sizeof( double ) * np, cudaMemcpyDeviceToDevice ) );
        apply( *s->K, src, dst );
        for ( int c = 0; c < 3; ++c )
            TN_CUDA_TRY( cudaMemcpyAsync( ou[c], dst.block_1().comp( c ), sizeof( double ) * nu, cudaMemcpyDeviceToDevice ) );
        TN_CUDA_TRY( cudaMemcpyAsync( op, dst.block_2().data(), sizeof( double ) * np, cudaMemcpyDeviceToDevice ) );
        return TN_OK;
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_stokes_apply: " ) + e.what() );
        return TN_ERR_STATE;
    }
}

extern "C" int tn_stokes_viscosity_backward( tn_stokes_solver* s, const double* const* u, const double* const* grad_u,
                                             int comm_mode, double* grad_log_k, double* const* lambda_u,
                                             double* lambda_p, int* iterations )
{
    TN_CHECK_ARG( s && u && grad_u && grad_log_k, "tn_stokes_viscosity_backward: null argument" );
    try
    {
        const int                 L  = s->prm.level;
        const Mesh&               mu = s->mesh[L];
        const tn_mesh*            m  = mu.get();
        const size_t              nu = mu.stored_nodes(), np = s->mesh[L - 1].stored_nodes();
        VectorQ1IsoQ2Q1< double > b( mu, s->mesh[L - 1] ), lam( mu, s->mesh[L - 1] );
        // adjoint right-hand side: the copy-wise derivative summed over the
        // copies of every node (the derivative with respect to the unique
        // node), with the velocity boundary treatment of the forward RHS
        for ( int c = 0; c < 3; ++c )
            TN_CUDA_TRY( cudaMemcpyAsync( b.block_1().comp( c ), grad_u[c], sizeof( double ) * nu,
                                          cudaMemcpyDeviceToDevice, stream() ) );
        b.block_1().halo_sum();
        const int bcc = s->prm.bc_cmb, bcs = s->prm.bc_surface;
        for ( int c = 0; c < 3; ++c )
        {
            if ( bcc == TN_BC_DIRICHLET )
                TN_CUDA_TRY( cudaMemset2DAsync( b.block_1().comp( c ), sizeof( double ) * m->n1, 0, sizeof( double ),
                                                m->nlat, stream() ) );
            if ( bcs == TN_BC_DIRICHLET )
                TN_CUDA_TRY( cudaMemset2DAsync( b.block_1().comp( c ) + m->N, sizeof( double ) * m->n1, 0,
                                                sizeof( double ), m->nlat, stream() ) );
        }
        if ( bcc == TN_BC_FREESLIP || bcs == TN_BC_FREESLIP )
        {
            double* f[3];
            b.block_1().ptrs( f );
            check( tn_freeslip_project_f64( m, f, bcc == TN_BC_FREESLIP, bcs == TN_BC_FREESLIP, stream() ),
                   "freeslip_project" );
        }
        // adjoint solve (the Stokes operator is symmetric)
        s->run( lam, b );
        if ( iterations )
            *iterations = s->iterations;
        // dJ/dlog k = -k (d (lambda^T K(k) x) / dk)
        const double* pu[3] = { u[0], u[1], u[2] };
        const double* pl[3] = { lam.block_1().comp( 0 ), lam.block_1().comp( 1 ), lam.block_1().comp( 2 ) };
        check( tn_epsdivdiv_kgrad_f64( m, bcc, bcs, comm_mode, pu, pl, grad_log_k, stream() ), "kgrad" );
        VectorQ1Scalar< double > g( mu, grad_log_k );
        scale_in_place( g, s->k64[L] );
        lincomb( g, { -1.0 }, { g } );
        if ( lambda_u )
            for ( int c = 0; c < 3; ++c )
                TN_CUDA_TRY( cudaMemcpyAsync( lambda_u[c], lam.block_1().comp( c ), sizeof( double ) * nu,
                                              cudaMemcpyDeviceToDevice, stream() ) );
        if ( lambda_p )
            TN_CUDA_TRY( cudaMemcpyAsync( lambda_p, lam.block_2().data(), sizeof( double ) * np,
                                          cudaMemcpyDeviceToDevice, stream() ) );
        TN_CUDA_TRY( cudaStreamSynchronize( stream() ) );
        return TN_OK;
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_stokes_viscosity_backward: " ) + e.what() );
        return TN_ERR_STATE;
    }
}

extern "C" int tn_stokes_solver_destroy( tn_stokes_solver* s )
{
    delete s;
    return TN_OK;
}

// ---------------------------------------------------------------------------
// Multigrid-preconditioned CG on DivKGrad with homogeneous Dirichlet radii:
// linear transfers, Jacobi or Chebyshev smoothing, coarse PCG, coarser
// operators re-discretised with injected k (the composition of the
// reference's tests/test_div_k_grad_multigrid*.cpp and
// tests/test_laplace_multigrid*.cpp).
namespace {

using DKG = DivKGrad< double >;

// runtime choice of the two smoothers of the reference
struct ScalarSmoother
{
    std::shared_ptr< Jacobi< DKG > >    jacobi;
    std::shared_ptr< Chebyshev< DKG > > cheb;
    void solve_impl( DKG& A, VectorQ1Scalar< double >& x, const VectorQ1Scalar< double >& b )
    {
        if ( jacobi )
            solve( *jacobi, A, x, b );
        else
            solve( *cheb, A, x, b );
    }
};

using ScalarMG = Multigrid< DKG, ProlongationLinear< double >, RestrictionLinear< double >, ScalarSmoother,
                            DevicePCG< DKG > >;

struct MGPreconditioner
{
    std::shared_ptr< ScalarMG > mg;
    void solve_impl( DKG& A, VectorQ1Scalar< double >& z, const VectorQ1Scalar< double >& r )
    {
        assign( z, 0.0 );
        solve( *mg, A, z, r );
    }
};

}  // namespace

extern "C" int tn_divkgrad_mg_pcg_solve_f64( const tn_scalar_mg_params* p, double r_min, double r_max, const double* k,
                                             const double* b, double* x, int* iterations, double* relative_residual )
{
    TN_CHECK_ARG( p && b && x, "tn_divkgrad_mg_pcg_solve_f64: null argument" );
    TN_CHECK_ARG( p->mg_levels >= 2 && p->level - p->mg_levels + 1 >= 0, "tn_divkgrad_mg_pcg_solve_f64: bad levels" );
    TN_CHECK_ARG( p->smoother == 0 || p->smoother == 1, "tn_divkgrad_mg_pcg_solve_f64: smoother must be 0 or 1" );
    TN_CHECK_ARG( p->krylov >= 0 && p->krylov <= 2, "tn_divkgrad_mg_pcg_solve_f64: krylov must be 0, 1 or 2" );
    try
    {
        const int                                L = p->level, Lmin = L - p->mg_levels + 1;
        std::vector< Mesh >                      mesh( L + 1 );
        std::vector< VectorQ1Scalar< double > >  kl( L + 1 );
        for ( int l = Lmin; l <= L; ++l )
        {
            mesh[l] = Mesh( l, r_min, r_max );
            kl[l]   = VectorQ1Scalar< double >( mesh[l] );
        }
        if ( k )
            TN_CUDA_TRY( cudaMemcpy( kl[L].data(), k, sizeof( double ) * mesh[L].stored_nodes(), cudaMemcpyDeviceToDevice ) );
        else
            assign( kl[L], 1.0 );
        for ( int l = L - 1; l >= Lmin; --l )
        {
            const double* src[1] = { kl[l + 1].data() };
            double*       dst[1] = { kl[l].data() };
            check( tn_injection_f64( mesh[l + 1].get(), mesh[l].get(), 1, src, dst, stream() ), "injection" );
        }
        std::vector< ProlongationLinear< double > > P;
        std::vector< RestrictionLinear< double > >  R;
        std::vector< DKG >                          A;
        std::vector< VectorQ1Scalar< double > >     tr, te, tmp;
        std::vector< ScalarSmoother >               sm;
        for ( int l = Lmin; l <= L; ++l )
        {
            DKG op( mesh[l], kl[l], true );
            VectorQ1Scalar< double > ones( mesh[l] ), inv( mesh[l] );
            assign( ones, 1.0 );
            op.set_diagonal( true );
            apply( op, ones, inv );
            op.set_diagonal( false );
            invert_entries( inv );
            std::vector< VectorQ1Scalar< double > > t2{ VectorQ1Scalar< double >( mesh[l] ),
                                                        VectorQ1Scalar< double >( mesh[l] ) };
            ScalarSmoother s;
            if ( p->smoother == 1 )
                s.jacobi = std::make_shared< Jacobi< DKG > >( inv, p->smoothing_steps, t2, p->jacobi_omega );
            else
                s.cheb = std::make_shared< Chebyshev< DKG > >( p->chebyshev_order, inv, t2, p->smoothing_steps,
                                                               p->power_iterations );
            sm.push_back( s );
            tmp.emplace_back( mesh[l] );
            A.push_back( op );
            if ( l < L )
            {
                tr.emplace_back( mesh[l] );
                te.emplace_back( mesh[l] );
                P.emplace_back( mesh[l + 1], mesh[l], OperatorApplyMode::Add );
                R.emplace_back( mesh[l + 1], mesh[l] );
            }
        }
        DKG                                     Afine = A.back();
        std::vector< DKG >                      Ac( A.begin(), A.end() - 1 );
        std::vector< VectorQ1Scalar< double > > ct{ VectorQ1Scalar< double >( mesh[Lmin] ),
                                                    VectorQ1Scalar< double >( mesh[Lmin] ),
                                                    VectorQ1Scalar< double >( mesh[Lmin] ) };
        DevicePCG< DKG > coarse( IterativeSolverParameters{ p->coarse_max_iterations, p->coarse_relative_tolerance, 1e-30 },
                                 ct );
        MGPreconditioner prec{ std::make_shared< ScalarMG >( P, R, Ac, tr, te, tmp, sm, coarse, p->vcycles ) };
        std::vector< VectorQ1Scalar< double > > t4;
        for ( int i = 0; i < 4; ++i )
            t4.emplace_back( mesh[L] );
        const IterativeSolverParameters ip{ p->max_iterations, p->relative_tolerance, p->absolute_tolerance };
        VectorQ1Scalar< double >        vb( mesh[L], const_cast< double* >( b ) ), vx( mesh[L], x );
        SolverStatistics                st;
        if ( p->krylov == 1 )
        {
            // PBiCGStab(2), left-preconditioned (tests/test_laplace_pbicgstab_multigrid.cpp composition)
            std::vector< VectorQ1Scalar< double > > t8;
            for ( int i = 0; i < 2 * 3 + 2; ++i )
                t8.emplace_back( mesh[L] );
            PBiCGStab< DKG, MGPreconditioner > bicg( 2, ip, t8, prec );
            solve( bicg, Afine, vx, vb );
            st = bicg.stats;
        }
        else if ( p->krylov == 2 )
        {
            std::vector< VectorQ1Scalar< double > > t7;
            for ( int i = 0; i < 7; ++i )
                t7.emplace_back( mesh[L] );
            PMINRES< DKG, MGPreconditioner > mr( ip, t7, prec );
            solve( mr, Afine, vx, vb );
            st = mr.stats;
        }
        else
        {
            PCG< DKG, MGPreconditioner > pcg( ip, t4, prec );
            solve( pcg, Afine, vx, vb );
            st = pcg.stats;
        }
        TN_CUDA_TRY( cudaDeviceSynchronize() );
        if ( iterations )
            *iterations = st.iterations;
        if ( relative_residual )
            *relative_residual = st.relative_residuals.back();
        return TN_OK;
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_divkgrad_mg_pcg_solve_f64: " ) + e.what() );
        return TN_ERR_STATE;
    }
}

extern "C" int tn_laplace_pcg_solve_f64( const tn_mesh* mesh, const double* b, double* x, int max_iterations,
                                         double relative_tolerance, double absolute_tolerance, int* iterations,
                                         double* relative_residual )
{
    TN_CHECK_ARG( mesh && b && x, "tn_laplace_pcg_solve_f64: null argument" );
    try
    {
        Mesh                     m = Mesh::wrap( mesh );
        Laplace< double >        A( m, true, false );
        VectorQ1Scalar< double > vb( m, const_cast< double* >( b ) ), vx( m, x );
        std::vector< VectorQ1Scalar< double > > t;
        for ( int i = 0; i < 3; ++i )
            t.emplace_back( m );
        DevicePCG< Laplace< double > > pcg(
            IterativeSolverParameters{ max_iterations, relative_tolerance, absolute_tolerance }, t );
        solve( pcg, A, vx, vb );
        const SolverStatistics st = pcg.statistics();
        TN_CUDA_TRY( cudaDeviceSynchronize() );
        if ( iterations )
            *iterations = st.iterations;
        if ( relative_residual )
            *relative_residual = st.relative_residuals.back();
        return TN_OK;
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_laplace_pcg_solve_f64: " ) + e.what() );
        return TN_ERR_STATE;
    }
}

// The library's Krylov solver templates without a preconditioner on the scalar
// Laplace with Dirichlet elimination (the compositions of the reference's
// tests/test_laplace_fgmres.cpp, test_laplace_minres.cpp, test_laplace_bicgstab.cpp).
extern "C" int tn_laplace_krylov_solve_f64( const tn_mesh* mesh, int solver, int param, const double* b, double* x,
                                            const double* shadow, int max_iterations, double relative_tolerance,
                                            double absolute_tolerance, int* iterations, double* history,
                                            int history_capacity, int* history_count )
{
    TN_CHECK_ARG( mesh && b && x, "tn_laplace_krylov_solve_f64: null argument" );
    TN_CHECK_ARG( solver >= 0 && solver <= 2, "tn_laplace_krylov_solve_f64: solver must be 0, 1 or 2" );
    TN_CHECK_ARG( solver == 1 || param >= 1, "tn_laplace_krylov_solve_f64: restart / l must be at least 1" );
    TN_CHECK_ARG( history_capacity >= 0 && ( history_capacity == 0 || history ),
                  "tn_laplace_krylov_solve_f64: history buffer missing" );
    try
    {
        using Lap = Laplace< double >;
        Mesh                     m = Mesh::wrap( mesh );
        Lap                      A( m, true, false );
        VectorQ1Scalar< double > vb( m, const_cast< double* >( b ) ), vx( m, x );
        auto                     tmps = [&m]( int n ) {
            std::vector< VectorQ1Scalar< double > > t;
            for ( int i = 0; i < n; ++i )
                t.emplace_back( m );
            return t;
        };
        const IterativeSolverParameters ip{ max_iterations, relative_tolerance, absolute_tolerance };
        SolverStatistics                st;
        if ( solver == 0 )
        {
            IdentitySolver< Lap >                id;
            FGMRES< Lap, IdentitySolver< Lap > > s( tmps( 2 * param + 4 ), param, ip, id );
            solve( s, A, vx, vb );
            st = s.stats;
        }
        else if ( solver == 1 )
        {
            PMINRES< Lap > s( ip, tmps( 7 ) );
            solve( s, A, vx, vb );
            st = s.stats;
        }
        else
        {
            PBiCGStab< Lap > s( param, ip, tmps( 2 * ( param + 1 ) + 2 ) );
            if ( shadow )
                s.set_shadow( VectorQ1Scalar< double >( m, const_cast< double* >( shadow ) ) );
            solve( s, A, vx, vb );
            st = s.stats;
        }
        TN_CUDA_TRY( cudaDeviceSynchronize() );
        if ( iterations )
            *iterations = st.iterations;
        const int n = int( st.relative_residuals.size() );
        for ( int i = 0; i < std::min( n, history_capacity ); ++i )
            history[i] = st.relative_residuals[size_t( i )];
        if ( history_count )
            *history_count = n;
        return TN_OK;
    }
    catch ( const std::exception& e )
    {
        set_error( std::string( "tn_laplace_krylov_solve_f64: " ) + e.what() );
        return TN_ERR_STATE;
    }
}

// compile the header-only operators that no driver above instantiates
template class tn::VectorMass< double, 3 >;
template class tn::VectorMass< float, 3 >;
