// Reference dump/timing driver (test infrastructure, never shipped).
//
// Compiles the reference's own header-only implementation of the hot path on
// Kokkos-OpenMP and exposes it as a command-line tool that reads seeded inputs
// from raw little-endian files and writes the reference's outputs, so the C
// restatement in oracle/ and the CUDA product can be compared with the
// reference itself.  Inputs are always generated outside (never with the
// reference's non-deterministic `randomize`).
//
// File layout of every field: the reference's own (subdomain, x, y, r) order,
// r fastest; vector fields are three such scalar blocks one after another
// (Grid4DDataVec is SoA, grid/grid_types.hpp:57).
//
// Commands (bc codes: 0 = Neumann, 1 = Dirichlet, 2 = free-slip):
//   mesh    L rmin rmax OUT               coords/radii/boundary+ownership masks
//   kerngen L rmin rmax bcc bcs diag DIR  EpsilonDivDivKerngen<double> apply
//   laplace L rmin rmax treat diag DIR    Laplace<double> apply
//   divergence L rmin rmax bcc bcs DIR    Divergence<double>: fine velocity -> coarse pressure
//   gradient   L rmin rmax bcc bcs DIR    Gradient<double>: coarse pressure -> fine velocity
//   stokes     L rmin rmax bcc bcs DIR    EpsDivDivStokes<double>: (src_u, src_p) -> (dst_u, dst_p), k.bin
//   laplace_minres L rmin rmax maxit reltol DIR  PMINRES on Laplace from x = 0 on b.bin: x.bin, hist.bin
//   laplace_bicgstab L rmin rmax l maxit reltol DIR  PBiCGStab(l) on Laplace from x = 0 on b.bin: x.bin,
//                                          hist.bin, rshadow.bin (its random shadow residual)
//   laplace_chebyshev L rmin rmax order iters pits DIR  Chebyshev smoother from x = 0 on b.bin (run on one
//                                          thread): x.bin, prints the eigenvalue estimate it used
//   laplace_fgmres L rmin rmax restart maxit reltol DIR  FGMRES on Laplace from x = 0 on b.bin: x.bin, hist.bin
//   stokes_fgmres L rmin rmax bcc bcs restart maxit tol sweeps omega DIR  FGMRES on EpsDivDivStokes with the
//                                          block-triangular preconditioner (Jacobi velocity block, lumped
//                                          KMass(1/kp) Schur block): x_u.bin, x_p.bin, hist.bin
//   stokes_minres L rmin rmax bcc bcs maxit tol sweeps omega DIR  PMINRES on EpsDivDivStokes with the
//                                          block-diagonal preconditioner (same blocks): x_u, x_p, hist
//   kerngen_vcycle Lmin Lmax rmin rmax bcc bcs omega smooth cycles cmaxit DIR  epsilon-div-div multigrid
//                                          (k<l>.bin per level, Jacobi, constant vector transfers, coarse PCG)
//   vcycle Lmin Lmax rmin rmax omega smooth cycles cmaxit DIR  Laplace multigrid (Jacobi, constant
//                                          transfers, coarse PCG) from x = 0 on b.bin, writes x.bin
//   prolong / restrict Lf rmin rmax DIR    constant vector transfer between Lf-1 and Lf
//   kmass   L rmin rmax mode DIR          KMass<double> (0 full, 1 diagonal, 2 lumped)
//   divkgrad L rmin rmax treat diag single DIR   DivKGrad<double> (k.bin, src.bin)
//   epsdivdiv L rmin rmax treat diag DIR   EpsilonDivDiv<double> (3x2 rule; k.bin, src.bin)
//   prolong_linear / restrict_linear Lf rmin rmax DIR  scalar linear transfer between Lf-1 and Lf
//   fct L rmin rmax dt kappa bc DIR  one fct_explicit_step on vel.bin (FE vector), T.bin and src.bin (FV
//                                    fields with ghosts); bc 1: Dirichlet T_cmb = 1, T_surface = 0 on T before
//                                    and in the step; writes centers.bin, dt.bin (dt_stable, dt), TL.bin, T.bin
//   gca L rmin rmax bcc bcs diag mode DIR  TwoGridGCA (mode 0 constant, 1 linear) of the Neumann kerngen
//                                          operator at level L (k.bin) into level L-1 with bcs, then the
//                                          stored-matrix apply of the coarse operator to src.bin
//   stokes_mg L mglevels rmin rmax bcc bcs restart maxit tol order steps pits vcycles gca cmaxit DIR
//                                          the app's Stokes solver stack (FGMRES, block-triangular preconditioner,
//                                          Chebyshev multigrid with GCA coarse operators, coarse PCG) on
//                                          k.bin / kp.bin / f_u.bin / f_p.bin: x_u, x_p, hist, JSON (iterations,
//                                          seconds, per-level Chebyshev eigenvalue estimates)
//   l2proj L rmin rmax lumped DIR  FV -> FE transfer of fv.bin (consistent mass + PCG, or lumped): x.bin
//   stokes_rhs L rmin rmax Ra bcc bcs DIR  buoyancy right-hand side of T.bin (FE): f_u.bin
//   kerngen_slow L rmin rmax bcc bcs diag DIR  the kerngen slow path on the reference's own assembled
//                                          wedge matrices (written to mats.bin) stored in Full mode
//   vlaplace L rmin rmax bcc bcs diag DIR  VectorLaplace<double>
//   xdmf_write L rmin rmax pts conn DIR    io::XDMFOutput of T.bin / u.bin (FE, FP64) under DIR/xdmf: the six
//                                          grids T (FP32 out), T64 (FP64), u (FP32), u64 (FP64), s32 (FP32 input,
//                                          FP32 out), v32 (FP32 input, FP64 out); two write() steps, the second
//                                          with T + 1 and 2 u; pts / conn = 4|8 bytes of points / connectivity
//   xdmf_read L rmin rmax label step vec CKDIR DIR  read_xdmf_checkpoint_grid of `label` at `step` from CKDIR
//                                          into a FP64 grid (vec 0: scalar, 1: 3-vector): out.bin; the metadata
//                                          as text in meta.txt; on a read error its message in error.txt, exit 3
//   fe2fv L rmin rmax DIR                  l2_project_fe_to_fv of T.bin (FE): fv.bin ([10][N+2]^3, ghosts set)
//   agca L rmin rmax bcc bcs diag DIR      adaptive GCA over three levels: GCAElementsCollector of k.bin (level L,
//                                          level range 2) on level L-2 (gcae.bin: the marks as a node field), the
//                                          level-(L-1) kerngen operator with kc.bin in Selective storage, TwoGridGCA
//                                          from the level-L Neumann kerngen operator, then its apply to src.bin
//                                          (level L-1): dst.bin
//   supg L rmin rmax kappa dt ms lumped treat diag DIR  UnsteadyAdvectionDiffusionSUPG<double> with the velocity
//                                          vel.bin (3 x nodes) applied to src.bin: dst.bin
//   kerngen_rank L rmin rmax bcc bcs P q DIR  the distributed domain as rank q of P (subdomain refinement
//                                          level 0, the default rank map): prints the rank's diamonds in local
//                                          order as JSON, then the EpsilonDivDivKerngen<double> apply on them with
//                                          SkipCommunication (the copy-wise result) of k.bin / src.bin (the rank's
//                                          nodes): dst.bin
//   time_kerngen L rmin rmax bcc bcs reps [DIR]  prints seconds per apply (CPU baseline); with DIR the
//                                          inputs are k.bin / src.bin there, else k = 1, src = 1
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "communication/shell/communication.hpp"
#include "fe/wedge/operators/shell/epsilon_divdiv.hpp"
#include "fe/wedge/operators/shell/epsilon_divdiv_kerngen.hpp"
#include "fe/wedge/operators/shell/epsilon_divdiv_stokes.hpp"
#include "fe/wedge/operators/shell/div_k_grad.hpp"
#include "fe/wedge/operators/shell/divergence.hpp"
#include "fe/wedge/operators/shell/gradient.hpp"
#include "fe/wedge/operators/shell/kmass.hpp"
#include "fe/wedge/operators/shell/mass.hpp"
#include "fe/wedge/operators/shell/vector_mass.hpp"
#include "fe/wedge/operators/shell/laplace.hpp"
#include "fe/wedge/operators/shell/prolongation_constant.hpp"
#include "fe/wedge/operators/shell/prolongation_linear.hpp"
#include "fe/wedge/operators/shell/restriction_constant.hpp"
#include "fe/wedge/operators/shell/restriction_linear.hpp"
#include "fe/wedge/operators/shell/vector_laplace.hpp"
#include "fe/wedge/operators/shell/unsteady_advection_diffusion_supg.hpp"
#include "fe/strong_algebraic_dirichlet_enforcement.hpp"
#include "fe/strong_algebraic_freeslip_enforcement.hpp"
#include "fv/hex/conversion.hpp"
#include "io/xdmf.hpp"
#include "fv/hex/helpers.hpp"
#include "fv/hex/operators/fct_advection_diffusion.hpp"
#include "grid/bit_masks.hpp"
#include "linalg/solvers/gca/gca.hpp"
#include "linalg/solvers/gca/gca_elements_collector.hpp"
#include "linalg/solvers/block_preconditioner_2x2.hpp"
#include "linalg/solvers/chebyshev.hpp"
#include "linalg/solvers/power_iteration.hpp"
#include "linalg/solvers/diagonal_solver.hpp"
#include "linalg/solvers/fgmres.hpp"
#include "linalg/solvers/jacobi.hpp"
#include "linalg/solvers/multigrid.hpp"
#include "linalg/solvers/pbicgstab.hpp"
#include "linalg/solvers/pcg.hpp"
#include "linalg/solvers/pminres.hpp"
#include "util/table.hpp"
#include "grid/shell/bit_masks.hpp"
#include "grid/shell/spherical_shell.hpp"
#include "linalg/vector_fv.hpp"
#include "linalg/vector_q1.hpp"
#include "util/init.hpp"

using namespace terra;
using grid::shell::BoundaryConditionFlag;
using grid::shell::BoundaryConditions;
using grid::shell::DistributedDomain;
using grid::shell::ShellBoundaryFlag;

namespace {

template < typename T >
std::vector< T > read_file( const std::string& path, size_t n )
{
    std::vector< T > v( n );
    std::ifstream    f( path, std::ios::binary );
    if ( !f )
        throw std::runtime_error( "cannot open " + path );
    f.read( reinterpret_cast< char* >( v.data() ), n * sizeof( T ) );
    if ( size_t( f.gcount() ) != n * sizeof( T ) )
        throw std::runtime_error( "short read " + path );
    return v;
}

template < typename T >
void write_file( const std::string& path, const T* p, size_t n )
{
    std::ofstream f( path, std::ios::binary );
    f.write( reinterpret_cast< const char* >( p ), n * sizeof( T ) );
}

template < typename View >
void view_from_host( View& v, const typename View::value_type* src )
{
    auto h = Kokkos::create_mirror_view( v );
    std::copy( src, src + h.size(), h.data() );
    Kokkos::deep_copy( v, h );
}

template < typename View >
std::vector< typename View::non_const_value_type > view_to_host( const View& v )
{
    auto h = Kokkos::create_mirror_view( v );
    Kokkos::deep_copy( h, v );
    return std::vector< typename View::non_const_value_type >( h.data(), h.data() + h.size() );
}

BoundaryConditionFlag bc_of( int c )
{
    return c == 1 ? BoundaryConditionFlag::DIRICHLET : ( c == 2 ? BoundaryConditionFlag::FREESLIP :
                                                                  BoundaryConditionFlag::NEUMANN );
}

struct Setup
{
    DistributedDomain                                        domain;
    grid::Grid4DDataScalar< grid::NodeOwnershipFlag >        omask;
    grid::Grid4DDataScalar< grid::shell::ShellBoundaryFlag > bmask;
    grid::Grid3DDataVec< double, 3 >                         coords;
    grid::Grid2DDataScalar< double >                         radii;
    size_t                                                   nodes;

    Setup( int L, double rmin, double rmax )
    {
        domain = DistributedDomain::create_uniform_single_subdomain_per_diamond( L, L, rmin, rmax );
        omask  = grid::setup_node_ownership_mask_data( domain );
        bmask  = grid::shell::setup_boundary_mask_data( domain );
        coords = grid::shell::subdomain_unit_sphere_single_shell_coords< double >( domain );
        radii  = grid::shell::subdomain_shell_radii< double >( domain );
        nodes  = omask.size();
    }
};

void load_vec( linalg::VectorQ1Vec< double >& v, const std::string& path, size_t n )
{
    auto h = read_file< double >( path, 3 * n );
    for ( int d = 0; d < 3; ++d )
        view_from_host( v.grid_data().comp_[d], h.data() + d * n );
}

void save_vec( const linalg::VectorQ1Vec< double >& v, const std::string& path, size_t n )
{
    std::vector< double > out( 3 * n );
    for ( int d = 0; d < 3; ++d )
    {
        auto c = view_to_host( v.grid_data().comp_[d] );
        std::copy( c.begin(), c.end(), out.begin() + d * n );
    }
    write_file( path, out.data(), out.size() );
}

int cmd_mesh( int L, double rmin, double rmax, const std::string& out )
{
    Setup s( L, rmin, rmax );
    auto  c  = view_to_host( s.coords );
    auto  r  = view_to_host( s.radii );
    auto  bm = view_to_host( s.bmask );
    auto  om = view_to_host( s.omask );
    write_file( out + "/coords.bin", c.data(), c.size() );
    write_file( out + "/radii.bin", r.data(), r.size() );
    write_file( out + "/bmask.bin", reinterpret_cast< const uint8_t* >( bm.data() ), bm.size() );
    write_file( out + "/omask.bin", reinterpret_cast< const uint8_t* >( om.data() ), om.size() );
    return 0;
}

using Kerngen = fe::wedge::operators::shell::EpsilonDivDivKerngen< double >;

Kerngen make_kerngen( Setup& s, linalg::VectorQ1Scalar< double >& k, int bcc, int bcs, bool diag )
{
    BoundaryConditions bcs_ = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    return Kerngen( s.domain, s.coords, s.radii, s.bmask, k.grid_data(), bcs_, diag );
}

int cmd_kerngen( int L, double rmin, double rmax, int bcc, int bcs, int diag, const std::string& dir )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Scalar< double > k( "k", s.domain, s.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", s.nodes ).data() );
    linalg::VectorQ1Vec< double > src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
    load_vec( src, dir + "/src.bin", s.nodes );
    auto op = make_kerngen( s, k, bcc, bcs, diag != 0 );
    linalg::apply( op, src, dst );
    save_vec( dst, dir + "/dst.bin", s.nodes );
    return 0;
}

// The apply of one rank of a distributed run: the stub poses as rank q of P while the domain is built
// (DistributedDomain::create_uniform_single_subdomain_per_diamond -> subdomain_to_rank_iterate_diamond_subdomains,
// grid/shell/spherical_shell.hpp:717-745,2520-2590); the apply skips the halo exchange, whose messages the stub
// cannot deliver.  The ownership mask is left unset (only dot products read it).
int cmd_kerngen_rank( int L, double rmin, double rmax, int bcc, int bcs, int P, int q, const std::string& dir )
{
    tn_mpi_stub_world_size = P, tn_mpi_stub_rank = q;
    DistributedDomain domain = DistributedDomain::create_uniform_single_subdomain_per_diamond( L, L, rmin, rmax );
    auto              omask  = grid::shell::allocate_scalar_grid< grid::NodeOwnershipFlag >( "omask", domain );
    auto              bmask  = grid::shell::setup_boundary_mask_data( domain );
    auto              coords = grid::shell::subdomain_unit_sphere_single_shell_coords< double >( domain );
    auto              radii  = grid::shell::subdomain_shell_radii< double >( domain );
    const size_t      nodes  = omask.size();
    std::printf( "{\"diamonds\": [" );
    for ( int i = 0; i < int( domain.subdomains().size() ); ++i )
        std::printf( "%s%d", i ? ", " : "", domain.subdomain_info_from_local_idx( i ).diamond_id() );
    std::printf( "], \"nodes\": %zu}\n", nodes );
    linalg::VectorQ1Scalar< double > k( "k", domain, omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", nodes ).data() );
    linalg::VectorQ1Vec< double > src( "src", domain, omask ), dst( "dst", domain, omask );
    load_vec( src, dir + "/src.bin", nodes );
    BoundaryConditions bcs_ = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    Kerngen            op( domain, coords, radii, bmask, k.grid_data(), bcs_, false );
    op.set_operator_apply_and_communication_modes(
        linalg::OperatorApplyMode::Replace, linalg::OperatorCommunicationMode::SkipCommunication );
    linalg::apply( op, src, dst );
    save_vec( dst, dir + "/dst.bin", nodes );
    tn_mpi_stub_world_size = 1, tn_mpi_stub_rank = 0;
    return 0;
}

int cmd_time_kerngen( int L, double rmin, double rmax, int bcc, int bcs, int reps, const std::string& dir = "" )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Scalar< double > k( "k", s.domain, s.omask );
    linalg::VectorQ1Vec< double >    src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
    if ( dir.empty() )
    {
        linalg::assign( k, 1.0 );
        linalg::assign( src, 1.0 );
    }
    else
    {
        view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", s.nodes ).data() );
        load_vec( src, dir + "/src.bin", s.nodes );
    }
    auto op = make_kerngen( s, k, bcc, bcs, false );
    linalg::apply( op, src, dst ); // warm-up, as measure_run_time does
    Kokkos::fence();
    auto t0 = std::chrono::steady_clock::now();
    for ( int i = 0; i < reps; ++i )
        linalg::apply( op, src, dst );
    Kokkos::fence();
    auto   t1 = std::chrono::steady_clock::now();
    double dt = std::chrono::duration< double >( t1 - t0 ).count() / reps;
    std::printf( "{\"seconds_per_apply\": %.9g, \"threads\": %d, \"stored_nodes\": %zu}\n",
                 dt,
                 Kokkos::DefaultExecutionSpace().concurrency(),
                 s.nodes );
    return 0;
}

int cmd_laplace( int L, double rmin, double rmax, int treat, int diag, const std::string& dir )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Scalar< double > src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
    view_from_host( src.grid_data(), read_file< double >( dir + "/src.bin", s.nodes ).data() );
    fe::wedge::operators::shell::Laplace< double > op( s.domain, s.coords, s.radii, s.bmask, treat != 0, diag != 0 );
    linalg::apply( op, src, dst );
    auto out = view_to_host( dst.grid_data() );
    write_file( dir + "/dst.bin", out.data(), out.size() );
    return 0;
}

// Unpreconditioned PCG (linalg/solvers/pcg.hpp) on Laplace(treat_boundary =
// true) from x = 0 for the right-hand side in b.bin; writes x.bin and prints
// iterations, final relative residual ||b - A x|| / ||b||, solve seconds and
// threads as one JSON line.
int cmd_laplace_cg( int L, double rmin, double rmax, int maxit, double reltol, const std::string& dir )
{
    using V = linalg::VectorQ1Scalar< double >;
    Setup s( L, rmin, rmax );
    V     b( "b", s.domain, s.omask ), x( "x", s.domain, s.omask ), r( "r", s.domain, s.omask );
    std::vector< V > tmps;
    for ( int i = 0; i < 4; ++i )
        tmps.emplace_back( "tmp" + std::to_string( i ), s.domain, s.omask );
    view_from_host( b.grid_data(), read_file< double >( dir + "/b.bin", s.nodes ).data() );
    linalg::assign( x, 0.0 );
    using Lap = fe::wedge::operators::shell::Laplace< double >;
    Lap  A( s.domain, s.coords, s.radii, s.bmask, true, false );
    auto table = std::make_shared< util::Table >();
    linalg::solvers::PCG< Lap > pcg( linalg::solvers::IterativeSolverParameters{ maxit, reltol, 1e-30 }, table, tmps );
    Kokkos::fence();
    auto t0 = std::chrono::steady_clock::now();
    linalg::solvers::solve( pcg, A, x, b );
    Kokkos::fence();
    const double sec = std::chrono::duration< double >( std::chrono::steady_clock::now() - t0 ).count();
    linalg::apply( A, x, r );
    linalg::lincomb( r, { 1.0, -1.0 }, { b, r } );
    const double rel = std::sqrt( linalg::dot( r, r ) / linalg::dot( b, b ) );
    auto         out = view_to_host( x.grid_data() );
    write_file( dir + "/x.bin", out.data(), out.size() );
    std::printf( "{\"iterations\": %zu, \"relres\": %.6e, \"seconds\": %.9g, \"threads\": %d}\n",
                 table->rows().size() - 1,
                 rel,
                 sec,
                 Kokkos::DefaultExecutionSpace().concurrency() );
    return 0;
}

int cmd_stokes_block( bool div, int L, double rmin, double rmax, int bcc, int bcs, const std::string& dir )
{
    Setup              f( L, rmin, rmax ), c( L - 1, rmin, rmax );
    BoundaryConditions b = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    linalg::VectorQ1Vec< double >    u( "u", f.domain, f.omask );
    linalg::VectorQ1Scalar< double > p( "p", c.domain, c.omask );
    if ( div )
    {
        load_vec( u, dir + "/src.bin", f.nodes );
        fe::wedge::operators::shell::Divergence< double > op( f.domain, c.domain, f.coords, f.radii, f.bmask, b );
        linalg::apply( op, u, p );
        auto out = view_to_host( p.grid_data() );
        write_file( dir + "/dst.bin", out.data(), out.size() );
    }
    else
    {
        view_from_host( p.grid_data(), read_file< double >( dir + "/src.bin", c.nodes ).data() );
        fe::wedge::operators::shell::Gradient< double > op( f.domain, c.domain, f.coords, f.radii, f.bmask, b );
        linalg::apply( op, p, u );
        save_vec( u, dir + "/dst.bin", f.nodes );
    }
    return 0;
}

// `cycles` multigrid V-cycles (multigrid.hpp:108-211) on Laplace<double> (Dirichlet rows) over levels
// Lmin..Lmax from x = 0: Jacobi pre / post smoothing (jacobi.hpp:51-62, inverse diagonal of the
// Dirichlet operator, `smooth` sweeps, damping omega), constant scalar transfers, coarsest-level PCG
// (pcg.hpp, max `cmaxit` iterations, relative 1e-8, absolute 1e-30); b.bin on Lmax, writes x.bin
int cmd_vcycle( int Lmin, int Lmax, double rmin, double rmax, double omega, int smooth, int cycles, int cmaxit,
                const std::string& dir )
{
    using V   = linalg::VectorQ1Scalar< double >;
    using Lap = fe::wedge::operators::shell::Laplace< double >;
    using P   = fe::wedge::operators::shell::ProlongationConstant< double >;
    using R   = fe::wedge::operators::shell::RestrictionConstant< double >;
    std::vector< Setup > lv;
    for ( int l = Lmin; l <= Lmax; ++l )
        lv.emplace_back( l, rmin, rmax );
    std::vector< P >                            Ps;
    std::vector< R >                            Rs;
    std::vector< Lap >                          Ac;
    std::vector< V >                            tr, te, tmp, ctmps;
    std::vector< linalg::solvers::Jacobi< Lap > > sm;
    for ( size_t i = 0; i < lv.size(); ++i )
    {
        Setup& s = lv[i];
        tmp.emplace_back( "tmp" + std::to_string( i ), s.domain, s.omask );
        V ts( "ts" + std::to_string( i ), s.domain, s.omask ), inv( "inv" + std::to_string( i ), s.domain, s.omask );
        Lap Ad( s.domain, s.coords, s.radii, s.bmask, true, true );
        linalg::assign( ts, 1.0 );
        linalg::apply( Ad, ts, inv );
        linalg::invert_entries( inv );
        sm.emplace_back( inv, smooth, ts, omega );
        if ( i == 0 )
            for ( int k = 0; k < 4; ++k )
                ctmps.emplace_back( "ct" + std::to_string( k ), s.domain, s.omask );
        if ( i + 1 < lv.size() )
        {
            tr.emplace_back( "tr" + std::to_string( i ), s.domain, s.omask );
            te.emplace_back( "te" + std::to_string( i ), s.domain, s.omask );
            Ac.emplace_back( s.domain, s.coords, s.radii, s.bmask, true, false );
            Ps.emplace_back( linalg::OperatorApplyMode::Add );
            Rs.emplace_back( s.domain );
        }
    }
    Setup& f = lv.back();
    V      b( "b", f.domain, f.omask ), x( "x", f.domain, f.omask );
    view_from_host( b.grid_data(), read_file< double >( dir + "/b.bin", f.nodes ).data() );
    linalg::assign( x, 0.0 );
    Lap  A( f.domain, f.coords, f.radii, f.bmask, true, false );
    auto table = std::make_shared< util::Table >();
    linalg::solvers::PCG< Lap > coarse( linalg::solvers::IterativeSolverParameters{ cmaxit, 1e-8, 1e-30 }, table,
                                        ctmps );
    linalg::solvers::Multigrid< Lap, P, R, linalg::solvers::Jacobi< Lap >, linalg::solvers::PCG< Lap > > mg(
        Ps, Rs, Ac, tr, te, tmp, sm, sm, coarse, cycles, 0.0 );
    linalg::solvers::solve( mg, A, x, b );
    auto out = view_to_host( x.grid_data() );
    write_file( dir + "/x.bin", out.data(), out.size() );
    return 0;
}

// Chebyshev<Laplace<double>> smoother (chebyshev.hpp:100-175, Dirichlet rows, inverse diagonal) applied
// from x = 0 to b.bin: `iters` sweeps of order `order`, the eigenvalue estimate from `pits` power
// iterations.  The estimate starts from randomize(), a generator pool with a fixed seed created per call:
// deterministic on one thread (run with OMP_NUM_THREADS=1).  The same estimate is computed here once more
// (same operator, same start) and printed, so the smoother after it can be checked, and the start vector is
// written out (start.bin) so the power iteration itself can be checked.  Writes x.bin; prints {"lambda": ...}
int cmd_laplace_chebyshev( int L, double rmin, double rmax, int order, int iters, int pits, const std::string& dir )
{
    using V   = linalg::VectorQ1Scalar< double >;
    using Lap = fe::wedge::operators::shell::Laplace< double >;
    Setup s( L, rmin, rmax );
    V     b( "b", s.domain, s.omask ), x( "x", s.domain, s.omask ), inv( "inv", s.domain, s.omask ),
        ones( "ones", s.domain, s.omask ), t0( "t0", s.domain, s.omask ), t1( "t1", s.domain, s.omask );
    view_from_host( b.grid_data(), read_file< double >( dir + "/b.bin", s.nodes ).data() );
    Lap A( s.domain, s.coords, s.radii, s.bmask, true, false ), Ad( s.domain, s.coords, s.radii, s.bmask, true, true );
    linalg::assign( ones, 1.0 );
    linalg::apply( Ad, ones, inv );
    linalg::invert_entries( inv );
    linalg::DiagonallyScaledOperator< Lap > scaled( A, inv );
    // the start vector power_iteration draws (randomize re-seeds its pool on every call)
    linalg::randomize( t0 );
    auto start = view_to_host( t0.grid_data() );
    write_file( dir + "/start.bin", start.data(), start.size() );
    const double lambda = linalg::solvers::power_iteration( scaled, t0, t1, pits );
    std::vector< V > tmps;
    for ( int i = 0; i < 2; ++i )
        tmps.emplace_back( "tmp" + std::to_string( i ), s.domain, s.omask );
    linalg::solvers::Chebyshev< Lap > cheb( order, inv, tmps, iters, pits );
    linalg::assign( x, 0.0 );
    linalg::solvers::solve( cheb, A, x, b );
    auto out = view_to_host( x.grid_data() );
    write_file( dir + "/x.bin", out.data(), out.size() );
    std::printf( "{\"lambda\": %.17g}\n", lambda );
    return 0;
}

// PBiCGStab(l)<Laplace<double>> (pbicgstab.hpp:29-290, identity preconditioner, Dirichlet rows) from x = 0 on
// b.bin; writes x.bin, hist.bin (the relative residual of every statistics row) and rshadow.bin, the shadow
// residual the solver drew with randomize() (it keeps it in its first workspace vector, unchanged)
int cmd_laplace_bicgstab( int L, double rmin, double rmax, int l, int maxit, double reltol, const std::string& dir )
{
    using V   = linalg::VectorQ1Scalar< double >;
    using Lap = fe::wedge::operators::shell::Laplace< double >;
    Setup s( L, rmin, rmax );
    V     b( "b", s.domain, s.omask ), x( "x", s.domain, s.omask );
    std::vector< V > tmps;
    for ( int i = 0; i < 2 * ( l + 1 ) + 2; ++i )
        tmps.emplace_back( "tmp" + std::to_string( i ), s.domain, s.omask );
    view_from_host( b.grid_data(), read_file< double >( dir + "/b.bin", s.nodes ).data() );
    linalg::assign( x, 0.0 );
    Lap  A( s.domain, s.coords, s.radii, s.bmask, true, false );
    auto table = std::make_shared< util::Table >();
    linalg::solvers::PBiCGStab< Lap > bi( l, linalg::solvers::IterativeSolverParameters{ maxit, reltol, 1e-30 },
                                          table, tmps );
    linalg::solvers::solve( bi, A, x, b );
    std::vector< double > hist;
    for ( const auto& row : table->rows() )
        hist.push_back( std::get< double >( row.at( "relative_residual" ) ) );
    write_file( dir + "/hist.bin", hist.data(), hist.size() );
    auto out = view_to_host( x.grid_data() );
    write_file( dir + "/x.bin", out.data(), out.size() );
    auto rsh = view_to_host( tmps[0].grid_data() );
    write_file( dir + "/rshadow.bin", rsh.data(), rsh.size() );
    return 0;
}

// PMINRES<Laplace<double>> (pminres.hpp:30-175, identity preconditioner, Dirichlet rows) from x = 0 on b.bin;
// writes x.bin and hist.bin (the relative residual of every statistics row)
int cmd_laplace_minres( int L, double rmin, double rmax, int maxit, double reltol, const std::string& dir )
{
    using V   = linalg::VectorQ1Scalar< double >;
    using Lap = fe::wedge::operators::shell::Laplace< double >;
    Setup s( L, rmin, rmax );
    V     b( "b", s.domain, s.omask ), x( "x", s.domain, s.omask );
    std::vector< V > tmps;
    for ( int i = 0; i < 7; ++i )
        tmps.emplace_back( "tmp" + std::to_string( i ), s.domain, s.omask );
    view_from_host( b.grid_data(), read_file< double >( dir + "/b.bin", s.nodes ).data() );
    linalg::assign( x, 0.0 );
    Lap  A( s.domain, s.coords, s.radii, s.bmask, true, false );
    auto table = std::make_shared< util::Table >();
    linalg::solvers::PMINRES< Lap > mr( linalg::solvers::IterativeSolverParameters{ maxit, reltol, 1e-30 }, table,
                                        tmps );
    linalg::solvers::solve( mr, A, x, b );
    std::vector< double > hist;
    for ( const auto& row : table->rows() )
        hist.push_back( std::get< double >( row.at( "relative_residual" ) ) );
    write_file( dir + "/hist.bin", hist.data(), hist.size() );
    auto out = view_to_host( x.grid_data() );
    write_file( dir + "/x.bin", out.data(), out.size() );
    return 0;
}

// FGMRES<Laplace<double>> (fgmres.hpp:100-330, identity preconditioner, Dirichlet rows) from x = 0 on b.bin;
// writes x.bin and hist.bin (the relative residual of every row of the solver's statistics table)
int cmd_laplace_fgmres( int L, double rmin, double rmax, int restart, int maxit, double reltol, const std::string& dir )
{
    using V   = linalg::VectorQ1Scalar< double >;
    using Lap = fe::wedge::operators::shell::Laplace< double >;
    Setup s( L, rmin, rmax );
    V     b( "b", s.domain, s.omask ), x( "x", s.domain, s.omask );
    std::vector< V > tmps;
    for ( int i = 0; i < 2 * restart + 4; ++i )
        tmps.emplace_back( "tmp" + std::to_string( i ), s.domain, s.omask );
    view_from_host( b.grid_data(), read_file< double >( dir + "/b.bin", s.nodes ).data() );
    linalg::assign( x, 0.0 );
    Lap  A( s.domain, s.coords, s.radii, s.bmask, true, false );
    auto table = std::make_shared< util::Table >();
    linalg::solvers::FGMRESOptions< double > opt;
    opt.restart = restart, opt.relative_residual_tolerance = reltol, opt.absolute_residual_tolerance = 1e-30;
    opt.max_iterations = maxit;
    linalg::solvers::FGMRES< Lap > fg( tmps, opt, table );
    linalg::solvers::solve( fg, A, x, b );
    std::vector< double > hist;
    for ( const auto& row : table->rows() )
        hist.push_back( std::get< double >( row.at( "relative_residual" ) ) );
    write_file( dir + "/hist.bin", hist.data(), hist.size() );
    auto out = view_to_host( x.grid_data() );
    write_file( dir + "/x.bin", out.data(), out.size() );
    return 0;
}

// FGMRES on EpsDivDivStokes with the app's block-triangular preconditioner (mantlecirculation.cpp:684-717):
// Schur block the inverse lumped KMass(1 / eta_p) (kp.bin = eta on the pressure level), velocity block
// `sweeps` damped Jacobi sweeps with the kerngen diagonal (deterministic, unlike the Chebyshev smoother's
// randomised power iteration); b = (src_u, src_p), x = 0; writes x_u.bin, x_p.bin, hist.bin
int cmd_stokes_fgmres( int L, double rmin, double rmax, int bcc, int bcs, int restart, int maxit, double tol,
                       int sweeps, double omega, const std::string& dir )
{
    using Stokes  = fe::wedge::operators::shell::EpsDivDivStokes< double >;
    using Viscous = Stokes::Block11Type;
    using Grad    = Stokes::Block12Type;
    using PMass   = fe::wedge::operators::shell::KMass< double >;
    using BV      = linalg::VectorQ1IsoQ2Q1< double >;
    using PrecV   = linalg::solvers::Jacobi< Viscous >;
    using PrecS   = linalg::solvers::DiagonalSolver< PMass >;
    using Prec    = linalg::solvers::BlockTriangularPreconditioner2x2< Stokes, Viscous, PMass, Grad, PrecV, PrecS >;
    Setup f( L, rmin, rmax ), c( L - 1, rmin, rmax );
    BoundaryConditions b = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    linalg::VectorQ1Scalar< double > k( "k", f.domain, f.omask ), kp( "kp", c.domain, c.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", f.nodes ).data() );
    view_from_host( kp.grid_data(), read_file< double >( dir + "/kp.bin", c.nodes ).data() );
    linalg::invert_entries( kp );
    Stokes K( f.domain, c.domain, f.coords, f.radii, f.bmask, k.grid_data(), b, false );
    // velocity block: inverse of the kerngen diagonal (diagonal mode of the same operator)
    linalg::VectorQ1Vec< double > ones( "ones", f.domain, f.omask ), inv( "inv", f.domain, f.omask ),
        jt( "jt", f.domain, f.omask );
    Viscous Kd( f.domain, f.coords, f.radii, f.bmask, k.grid_data(), b, true );
    linalg::assign( ones, 1.0 );
    linalg::apply( Kd, ones, inv );
    linalg::invert_entries( inv );
    PrecV pv( inv, sweeps, jt, omega );
    PMass pmass( c.domain, c.coords, c.radii, kp.grid_data(), false );
    pmass.set_lumped_diagonal( true );
    linalg::VectorQ1Scalar< double > lumped( "lumped", c.domain, c.omask ), t1( "t1", c.domain, c.omask );
    linalg::assign( t1, 1.0 );
    linalg::apply( pmass, t1, lumped );
    PrecS ps( lumped );
    BV    ptmp( "ptmp", f.domain, c.domain, f.omask, c.omask );
    Prec  prec( K.block_11(), pmass, K.block_12(), ptmp, pv, ps );
    std::vector< BV > tmps;
    for ( int i = 0; i < 2 * restart + 4; ++i )
        tmps.emplace_back( "tmp" + std::to_string( i ), f.domain, c.domain, f.omask, c.omask );
    BV rhs( "rhs", f.domain, c.domain, f.omask, c.omask ), x( "x", f.domain, c.domain, f.omask, c.omask );
    load_vec( rhs.block_1(), dir + "/src_u.bin", f.nodes );
    view_from_host( rhs.block_2().grid_data(), read_file< double >( dir + "/src_p.bin", c.nodes ).data() );
    linalg::assign( x, 0.0 );
    auto table = std::make_shared< util::Table >();
    linalg::solvers::FGMRESOptions< double > opt;
    opt.restart = restart, opt.relative_residual_tolerance = tol, opt.absolute_residual_tolerance = 1e-30;
    opt.max_iterations = maxit;
    linalg::solvers::FGMRES< Stokes, Prec > fg( tmps, opt, table, prec );
    linalg::solvers::solve( fg, K, x, rhs );
    std::vector< double > hist;
    for ( const auto& row : table->rows() )
        hist.push_back( std::get< double >( row.at( "relative_residual" ) ) );
    write_file( dir + "/hist.bin", hist.data(), hist.size() );
    save_vec( x.block_1(), dir + "/x_u.bin", f.nodes );
    auto xp = view_to_host( x.block_2().grid_data() );
    write_file( dir + "/x_p.bin", xp.data(), xp.size() );
    return 0;
}

// PMINRES on EpsDivDivStokes with the block-diagonal preconditioner (block_preconditioner_2x2.hpp:38-100):
// velocity block `sweeps` damped Jacobi sweeps with the kerngen diagonal, pressure block the inverse lumped
// KMass(1 / kp); b = (src_u, src_p), x = 0; writes x_u.bin, x_p.bin, hist.bin
int cmd_stokes_minres( int L, double rmin, double rmax, int bcc, int bcs, int maxit, double tol, int sweeps,
                       double omega, const std::string& dir )
{
    using Stokes  = fe::wedge::operators::shell::EpsDivDivStokes< double >;
    using Viscous = Stokes::Block11Type;
    using PMass   = fe::wedge::operators::shell::KMass< double >;
    using BV      = linalg::VectorQ1IsoQ2Q1< double >;
    using PrecV   = linalg::solvers::Jacobi< Viscous >;
    using PrecS   = linalg::solvers::DiagonalSolver< PMass >;
    using Prec    = linalg::solvers::BlockDiagonalPreconditioner2x2< Stokes, Viscous, PMass, PrecV, PrecS >;
    Setup f( L, rmin, rmax ), c( L - 1, rmin, rmax );
    BoundaryConditions b = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    linalg::VectorQ1Scalar< double > k( "k", f.domain, f.omask ), kp( "kp", c.domain, c.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", f.nodes ).data() );
    view_from_host( kp.grid_data(), read_file< double >( dir + "/kp.bin", c.nodes ).data() );
    linalg::invert_entries( kp );
    Stokes K( f.domain, c.domain, f.coords, f.radii, f.bmask, k.grid_data(), b, false );
    linalg::VectorQ1Vec< double > ones( "ones", f.domain, f.omask ), inv( "inv", f.domain, f.omask ),
        jt( "jt", f.domain, f.omask );
    Viscous Kd( f.domain, f.coords, f.radii, f.bmask, k.grid_data(), b, true );
    linalg::assign( ones, 1.0 );
    linalg::apply( Kd, ones, inv );
    linalg::invert_entries( inv );
    PrecV pv( inv, sweeps, jt, omega );
    PMass pmass( c.domain, c.coords, c.radii, kp.grid_data(), false );
    pmass.set_lumped_diagonal( true );
    linalg::VectorQ1Scalar< double > lumped( "lumped", c.domain, c.omask ), t1( "t1", c.domain, c.omask );
    linalg::assign( t1, 1.0 );
    linalg::apply( pmass, t1, lumped );
    PrecS ps( lumped );
    Prec  prec( K.block_11(), pmass, pv, ps );
    std::vector< BV > tmps;
    for ( int i = 0; i < 7; ++i )
        tmps.emplace_back( "tmp" + std::to_string( i ), f.domain, c.domain, f.omask, c.omask );
    BV rhs( "rhs", f.domain, c.domain, f.omask, c.omask ), x( "x", f.domain, c.domain, f.omask, c.omask );
    load_vec( rhs.block_1(), dir + "/src_u.bin", f.nodes );
    view_from_host( rhs.block_2().grid_data(), read_file< double >( dir + "/src_p.bin", c.nodes ).data() );
    linalg::assign( x, 0.0 );
    auto table = std::make_shared< util::Table >();
    linalg::solvers::PMINRES< Stokes, Prec > mr( linalg::solvers::IterativeSolverParameters{ maxit, tol, 1e-30 },
                                                 table, tmps, prec );
    linalg::solvers::solve( mr, K, x, rhs );
    std::vector< double > hist;
    for ( const auto& row : table->rows() )
        hist.push_back( std::get< double >( row.at( "relative_residual" ) ) );
    write_file( dir + "/hist.bin", hist.data(), hist.size() );
    save_vec( x.block_1(), dir + "/x_u.bin", f.nodes );
    auto xp = view_to_host( x.block_2().grid_data() );
    write_file( dir + "/x_p.bin", xp.data(), xp.size() );
    return 0;
}

// `cycles` V-cycles on EpsilonDivDivKerngen<double> (bcc, bcs) over levels Lmin..Lmax from x = 0: the
// viscosity of level l from k<l>.bin, Jacobi pre / post smoothing with the kerngen diagonal (`smooth` sweeps,
// damping omega), constant vector transfers, coarsest-level PCG (max `cmaxit`, relative 1e-8, absolute
// 1e-30); b.bin (vector) on Lmax, writes x.bin
int cmd_kerngen_vcycle( int Lmin, int Lmax, double rmin, double rmax, int bcc, int bcs, double omega, int smooth,
                        int cycles, int cmaxit, const std::string& dir )
{
    using V  = linalg::VectorQ1Vec< double >;
    using Op = Kerngen;
    using P  = fe::wedge::operators::shell::ProlongationVecConstant< double >;
    using R  = fe::wedge::operators::shell::RestrictionVecConstant< double >;
    std::vector< Setup >                           lv;
    std::vector< linalg::VectorQ1Scalar< double > > ks;
    for ( int l = Lmin; l <= Lmax; ++l )
    {
        lv.emplace_back( l, rmin, rmax );
        ks.emplace_back( "k" + std::to_string( l ), lv.back().domain, lv.back().omask );
        view_from_host( ks.back().grid_data(),
                        read_file< double >( dir + "/k" + std::to_string( l ) + ".bin", lv.back().nodes ).data() );
    }
    std::vector< P >                            Ps;
    std::vector< R >                            Rs;
    std::vector< Op >                           Ac;
    std::vector< V >                            tr, te, tmp, ctmps;
    std::vector< linalg::solvers::Jacobi< Op > > sm;
    for ( size_t i = 0; i < lv.size(); ++i )
    {
        Setup& s = lv[i];
        tmp.emplace_back( "tmp" + std::to_string( i ), s.domain, s.omask );
        V  ts( "ts" + std::to_string( i ), s.domain, s.omask ), inv( "inv" + std::to_string( i ), s.domain, s.omask );
        Op Ad = make_kerngen( s, ks[i], bcc, bcs, true );
        linalg::assign( ts, 1.0 );
        linalg::apply( Ad, ts, inv );
        linalg::invert_entries( inv );
        sm.emplace_back( inv, smooth, ts, omega );
        if ( i == 0 )
            for ( int k = 0; k < 4; ++k )
                ctmps.emplace_back( "ct" + std::to_string( k ), s.domain, s.omask );
        if ( i + 1 < lv.size() )
        {
            tr.emplace_back( "tr" + std::to_string( i ), s.domain, s.omask );
            te.emplace_back( "te" + std::to_string( i ), s.domain, s.omask );
            Ac.push_back( make_kerngen( s, ks[i], bcc, bcs, false ) );
            Ps.emplace_back( linalg::OperatorApplyMode::Add );
            Rs.emplace_back( s.domain );
        }
    }
    Setup& f = lv.back();
    V      b( "b", f.domain, f.omask ), x( "x", f.domain, f.omask );
    load_vec( b, dir + "/b.bin", f.nodes );
    linalg::assign( x, 0.0 );
    Op   A     = make_kerngen( f, ks.back(), bcc, bcs, false );
    auto table = std::make_shared< util::Table >();
    linalg::solvers::PCG< Op > coarse( linalg::solvers::IterativeSolverParameters{ cmaxit, 1e-8, 1e-30 }, table,
                                       ctmps );
    linalg::solvers::Multigrid< Op, P, R, linalg::solvers::Jacobi< Op >, linalg::solvers::PCG< Op > > mg(
        Ps, Rs, Ac, tr, te, tmp, sm, sm, coarse, cycles, 0.0 );
    linalg::solvers::solve( mg, A, x, b );
    save_vec( x, dir + "/x.bin", f.nodes );
    return 0;
}

// The mantle-circulation app's Stokes solver stack (apps/mantlecirculation/mantlecirculation.cpp:486-735):
// FGMRES(restart) on EpsDivDivStokes with the block-triangular preconditioner, velocity block one
// Multigrid V-cycle per application (`vcycles`) over levels L-mglevels+1..L with Chebyshev(order, `steps`
// sweeps, `pits` power iterations) smoothing, constant vector transfers, GCA coarse operators (gca 1:
// constant interpolation, Full storage; 2: linear) built from the Neumann block of the finest operator, and
// the coarse PCG(cmaxit, 1e-6, 1e-16); Schur block the inverse lumped KMass(1 / kp).  Inputs k.bin (level L),
// kp.bin (level L-1), f_u.bin, f_p.bin; x = 0.  Writes x_u.bin, x_p.bin, hist.bin and prints a JSON line with
// the iteration count, the solve's seconds and, per level (coarsest first), the largest-eigenvalue estimate
// each Chebyshev smoother draws (the same power iteration from the same random start, which is reproducible
// only on one thread).
int cmd_stokes_mg( int L, int mglevels, double rmin, double rmax, int bcc, int bcs, int restart, int maxit, double tol,
                   int order, int steps, int pits, int vcycles, int gca, int cmaxit, const std::string& dir )
{
    using Stokes   = fe::wedge::operators::shell::EpsDivDivStokes< double >;
    using Viscous  = Stokes::Block11Type;
    using Grad     = Stokes::Block12Type;
    using PMass    = fe::wedge::operators::shell::KMass< double >;
    using BV       = linalg::VectorQ1IsoQ2Q1< double >;
    using V        = linalg::VectorQ1Vec< double >;
    using P        = fe::wedge::operators::shell::ProlongationVecConstant< double >;
    using R        = fe::wedge::operators::shell::RestrictionVecConstant< double >;
    using Smoother = linalg::solvers::Chebyshev< Viscous >;
    using Coarse   = linalg::solvers::PCG< Viscous >;
    using PrecV    = linalg::solvers::Multigrid< Viscous, P, R, Smoother, Coarse >;
    using PrecS    = linalg::solvers::DiagonalSolver< PMass >;
    using Prec     = linalg::solvers::BlockTriangularPreconditioner2x2< Stokes, Viscous, PMass, Grad, PrecV, PrecS >;
    const int          Lmin = L - mglevels + 1;
    std::vector< Setup > lv;
    for ( int l = Lmin; l <= L; ++l )
        lv.emplace_back( l, rmin, rmax );
    Setup&             f = lv.back();
    Setup              c( L - 1, rmin, rmax );
    BoundaryConditions b  = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    BoundaryConditions bn = { { ShellBoundaryFlag::CMB, BoundaryConditionFlag::NEUMANN },
                              { ShellBoundaryFlag::SURFACE, BoundaryConditionFlag::NEUMANN } };
    linalg::VectorQ1Scalar< double > k( "k", f.domain, f.omask ), kp( "kp", c.domain, c.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", f.nodes ).data() );
    view_from_host( kp.grid_data(), read_file< double >( dir + "/kp.bin", c.nodes ).data() );
    linalg::invert_entries( kp );
    Stokes K( f.domain, c.domain, f.coords, f.radii, f.bmask, k.grid_data(), b, false );
    Stokes Kn( f.domain, c.domain, f.coords, f.radii, f.bmask, k.grid_data(), bn, false );

    std::vector< linalg::VectorQ1Scalar< double > > kc, gcae;
    std::vector< Viscous >                          Ac;
    std::vector< P >                                Ps;
    std::vector< R >                                Rs;
    std::vector< V >                                tr, te, tmp, tmp2;
    for ( int i = 0; i < mglevels; ++i )
    {
        Setup& s = lv[i];
        tmp.emplace_back( "tmp" + std::to_string( i ), s.domain, s.omask );
        tmp2.emplace_back( "tmp2" + std::to_string( i ), s.domain, s.omask );
        if ( i + 1 < mglevels )
        {
            kc.emplace_back( "kc" + std::to_string( i ), s.domain, s.omask );
            gcae.emplace_back( "gcae" + std::to_string( i ), s.domain, s.omask );
            linalg::assign( kc.back(), 1.0 ); // replaced by the stored GCA matrices
            linalg::assign( gcae.back(), 1.0 );
            Ac.emplace_back( s.domain, s.coords, s.radii, s.bmask, kc.back().grid_data(), b, false );
            if ( gca )
                Ac.back().set_stored_matrix_mode( linalg::OperatorStoredMatrixMode::Full, i, gcae.back().grid_data() );
            tr.emplace_back( "tr" + std::to_string( i ), s.domain, s.omask );
            te.emplace_back( "te" + std::to_string( i ), s.domain, s.omask );
            Ps.emplace_back( linalg::OperatorApplyMode::Add );
            Rs.emplace_back( s.domain );
        }
    }
    if ( gca )
        for ( int i = mglevels - 2; i >= 0; --i )
            linalg::solvers::TwoGridGCA< double, Viscous >(
                i == mglevels - 2 ? Kn.block_11() : Ac[i + 1], Ac[i], i, gcae[i].grid_data(), true,
                gca == 2 ? linalg::solvers::InterpolationMode::Linear : linalg::solvers::InterpolationMode::Constant );

    std::vector< V >        invd;
    std::vector< Smoother > sm;
    std::vector< double >   ev;
    for ( int i = 0; i < mglevels; ++i )
    {
        Setup&   s = lv[i];
        Viscous& A = i + 1 == mglevels ? K.block_11() : Ac[i];
        invd.emplace_back( "invd" + std::to_string( i ), s.domain, s.omask );
        V ones( "ones", s.domain, s.omask );
        linalg::assign( ones, 1.0 );
        A.set_diagonal( true );
        linalg::apply( A, ones, invd.back() );
        A.set_diagonal( false );
        linalg::invert_entries( invd.back() );
        {
            V                                         t0( "t0", s.domain, s.omask ), t1( "t1", s.domain, s.omask );
            linalg::DiagonallyScaledOperator< Viscous > dA( A, invd.back() );
            ev.push_back( linalg::solvers::power_iteration( dA, t0, t1, pits ) );
        }
        sm.emplace_back( order, invd.back(), std::vector< V >{ tmp[i], tmp2[i] }, steps, pits );
    }
    std::vector< V > ct;
    for ( int i = 0; i < 4; ++i )
        ct.emplace_back( "ct" + std::to_string( i ), lv[0].domain, lv[0].omask );
    auto   table = std::make_shared< util::Table >();
    Coarse coarse( linalg::solvers::IterativeSolverParameters{ cmaxit, 1e-6, 1e-16 }, table, ct );
    PrecV  pv( Ps, Rs, Ac, tr, te, tmp, sm, sm, coarse, vcycles, 1e-6 );

    PMass pmass( c.domain, c.coords, c.radii, kp.grid_data(), false );
    pmass.set_lumped_diagonal( true );
    linalg::VectorQ1Scalar< double > lumped( "lumped", c.domain, c.omask ), t1( "t1", c.domain, c.omask );
    linalg::assign( t1, 1.0 );
    linalg::apply( pmass, t1, lumped );
    PrecS ps( lumped );
    BV    ptmp( "ptmp", f.domain, c.domain, f.omask, c.omask );
    Prec  prec( K.block_11(), pmass, K.block_12(), ptmp, pv, ps );
    std::vector< BV > tmps;
    for ( int i = 0; i < 2 * restart + 4; ++i )
        tmps.emplace_back( "tmp" + std::to_string( i ), f.domain, c.domain, f.omask, c.omask );
    BV rhs( "rhs", f.domain, c.domain, f.omask, c.omask ), x( "x", f.domain, c.domain, f.omask, c.omask );
    load_vec( rhs.block_1(), dir + "/f_u.bin", f.nodes );
    view_from_host( rhs.block_2().grid_data(), read_file< double >( dir + "/f_p.bin", c.nodes ).data() );
    linalg::assign( x, 0.0 );
    auto ftable = std::make_shared< util::Table >();
    linalg::solvers::FGMRESOptions< double > opt;
    opt.restart = restart, opt.relative_residual_tolerance = tol, opt.absolute_residual_tolerance = 1e-30;
    opt.max_iterations = maxit;
    linalg::solvers::FGMRES< Stokes, Prec > fg( tmps, opt, ftable, prec );
    Kokkos::fence();
    auto t0 = std::chrono::steady_clock::now();
    linalg::solvers::solve( fg, K, x, rhs );
    Kokkos::fence();
    const double sec = std::chrono::duration< double >( std::chrono::steady_clock::now() - t0 ).count();
    std::vector< double > hist;
    for ( const auto& row : ftable->rows() )
        hist.push_back( std::get< double >( row.at( "relative_residual" ) ) );
    write_file( dir + "/hist.bin", hist.data(), hist.size() );
    save_vec( x.block_1(), dir + "/x_u.bin", f.nodes );
    auto xp = view_to_host( x.block_2().grid_data() );
    write_file( dir + "/x_p.bin", xp.data(), xp.size() );
    std::printf( "{\"iterations\": %d, \"seconds\": %.9g, \"threads\": %d, \"eigenvalues\": [",
                 int( hist.size() ) - 1,
                 sec,
                 Kokkos::DefaultExecutionSpace().concurrency() );
    for ( size_t i = 0; i < ev.size(); ++i )
        std::printf( "%s%.17g", i ? ", " : "", ev[i] );
    std::printf( "]}\n" );
    return 0;
}

// EpsDivDivStokes<double> (epsilon_divdiv_stokes.hpp:55-90): [A B^T; B 0] applied to (u, p), A the
// kerngen operator with k.bin on level L, p on level L-1
int cmd_stokes_op( int L, double rmin, double rmax, int bcc, int bcs, const std::string& dir )
{
    Setup                            f( L, rmin, rmax ), c( L - 1, rmin, rmax );
    BoundaryConditions b = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    linalg::VectorQ1Scalar< double > k( "k", f.domain, f.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", f.nodes ).data() );
    linalg::VectorQ1IsoQ2Q1< double > src( "src", f.domain, c.domain, f.omask, c.omask ),
        dst( "dst", f.domain, c.domain, f.omask, c.omask );
    load_vec( src.block_1(), dir + "/src_u.bin", f.nodes );
    view_from_host( src.block_2().grid_data(), read_file< double >( dir + "/src_p.bin", c.nodes ).data() );
    fe::wedge::operators::shell::EpsDivDivStokes< double > op( f.domain, c.domain, f.coords, f.radii, f.bmask,
                                                               k.grid_data(), b, false );
    linalg::apply( op, src, dst );
    save_vec( dst.block_1(), dir + "/dst_u.bin", f.nodes );
    auto out = view_to_host( dst.block_2().grid_data() );
    write_file( dir + "/dst_p.bin", out.data(), out.size() );
    return 0;
}

int cmd_transfer( bool prolong, int Lf, double rmin, double rmax, const std::string& dir )
{
    Setup                         f( Lf, rmin, rmax ), c( Lf - 1, rmin, rmax );
    linalg::VectorQ1Vec< double > uf( "uf", f.domain, f.omask ), uc( "uc", c.domain, c.omask );
    if ( prolong )
    {
        load_vec( uc, dir + "/src.bin", c.nodes );
        fe::wedge::operators::shell::ProlongationVecConstant< double > P;
        linalg::apply( P, uc, uf );
        save_vec( uf, dir + "/dst.bin", f.nodes );
    }
    else
    {
        load_vec( uf, dir + "/src.bin", f.nodes );
        fe::wedge::operators::shell::RestrictionVecConstant< double > R( c.domain );
        linalg::apply( R, uf, uc );
        save_vec( uc, dir + "/dst.bin", c.nodes );
    }
    return 0;
}

int cmd_kmass( int L, double rmin, double rmax, int mode, const std::string& dir )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Scalar< double > k( "k", s.domain, s.omask ), src( "src", s.domain, s.omask ),
        dst( "dst", s.domain, s.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", s.nodes ).data() );
    view_from_host( src.grid_data(), read_file< double >( dir + "/src.bin", s.nodes ).data() );
    fe::wedge::operators::shell::KMass< double > op( s.domain, s.coords, s.radii, k.grid_data(), mode == 1 );
    op.set_lumped_diagonal( mode == 2 );
    linalg::apply( op, src, dst );
    auto out = view_to_host( dst.grid_data() );
    write_file( dir + "/dst.bin", out.data(), out.size() );
    return 0;
}

// Mass (mass.hpp) on the scalar src (mode 0 full, 1 diagonal, 2 lumped) and
// VectorMass< double, 3 > (vector_mass.hpp) on the vector src (mode 0 full,
// 1 diagonal)
int cmd_mass( bool vec, int L, double rmin, double rmax, int mode, const std::string& dir )
{
    Setup s( L, rmin, rmax );
    if ( !vec )
    {
        linalg::VectorQ1Scalar< double > src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
        view_from_host( src.grid_data(), read_file< double >( dir + "/src.bin", s.nodes ).data() );
        fe::wedge::operators::shell::Mass< double > op( s.domain, s.coords, s.radii, mode == 1, mode == 2 );
        linalg::apply( op, src, dst );
        auto out = view_to_host( dst.grid_data() );
        write_file( dir + "/dst.bin", out.data(), out.size() );
        return 0;
    }
    linalg::VectorQ1Vec< double > src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
    load_vec( src, dir + "/src.bin", s.nodes );
    fe::wedge::operators::shell::VectorMass< double, 3 > op( s.domain, s.coords, s.radii, mode == 1 );
    linalg::apply( op, src, dst );
    save_vec( dst, dir + "/dst.bin", s.nodes );
    return 0;
}

int cmd_transfer_linear( bool prolong, int Lf, double rmin, double rmax, const std::string& dir )
{
    Setup                            f( Lf, rmin, rmax ), c( Lf - 1, rmin, rmax );
    linalg::VectorQ1Scalar< double > uf( "uf", f.domain, f.omask ), uc( "uc", c.domain, c.omask );
    if ( prolong )
    {
        view_from_host( uc.grid_data(), read_file< double >( dir + "/src.bin", c.nodes ).data() );
        fe::wedge::operators::shell::ProlongationLinear< double > P( f.coords, f.radii );
        linalg::apply( P, uc, uf );
        auto out = view_to_host( uf.grid_data() );
        write_file( dir + "/dst.bin", out.data(), out.size() );
    }
    else
    {
        view_from_host( uf.grid_data(), read_file< double >( dir + "/src.bin", f.nodes ).data() );
        fe::wedge::operators::shell::RestrictionLinear< double > R( c.domain, f.coords, f.radii );
        linalg::apply( R, uf, uc );
        auto out = view_to_host( uc.grid_data() );
        write_file( dir + "/dst.bin", out.data(), out.size() );
    }
    return 0;
}

// FV -> FE transfer on the FV field fv.bin ([10][N+2]^3 with ghosts): l2_project_fv_to_fe (consistent mass,
// PCG 1000 / 1e-12 / 1e-12 from x = 0; conversion.hpp:131-205) or l2_project_fv_to_fe_lumped (:243-300);
// writes x.bin
int cmd_l2proj( int L, double rmin, double rmax, int lumped, const std::string& dir )
{
    Setup                                             s( L, rmin, rmax );
    linalg::VectorFVScalar< double >                  fv( "fv", s.domain );
    linalg::VectorQ1Scalar< double >                  x( "x", s.domain, s.omask );
    std::vector< linalg::VectorQ1Scalar< double > >   tmps;
    for ( int i = 0; i < 5; ++i )
        tmps.emplace_back( "t" + std::to_string( i ), s.domain, s.omask );
    view_from_host( fv.grid_data(), read_file< double >( dir + "/fv.bin", fv.grid_data().size() ).data() );
    linalg::assign( x, 0.0 );
    if ( lumped )
        fv::hex::l2_project_fv_to_fe_lumped( x, fv, s.domain, s.coords, s.radii, tmps );
    else
        fv::hex::l2_project_fv_to_fe( x, fv, s.domain, s.coords, s.radii, tmps );
    auto h = view_to_host( x.grid_data() );
    write_file( dir + "/x.bin", h.data(), h.size() );
    return 0;
}

// The app's Stokes buoyancy right-hand side (mantlecirculation.cpp:876-899): g = Ra T n at every node with n the
// unit radial direction (RHSVelocityInterpolator, :117-150, restated: it is app code), f = VectorMass g, then the
// library's strong Dirichlet and free-slip enforcement for the boundary conditions (bcc, bcs); T.bin (FE scalar)
// -> f_u.bin
int cmd_stokes_rhs( int L, double rmin, double rmax, double ra, int bcc, int bcs, const std::string& dir )
{
    Setup                            f( L, rmin, rmax ), c( L - 1, rmin, rmax );
    BoundaryConditions b = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    auto                             T = read_file< double >( dir + "/T.bin", f.nodes );
    linalg::VectorQ1Vec< double >    g( "g", f.domain, f.omask );
    linalg::VectorQ1IsoQ2Q1< double > rhs( "rhs", f.domain, c.domain, f.omask, c.omask );
    {
        auto coords = view_to_host( f.coords );
        auto radii  = view_to_host( f.radii );
        (void) radii;
        const int n1 = ( 1 << L ) + 1;
        std::vector< double > h( 3 * f.nodes );
        for ( size_t i = 0; i < f.nodes; ++i )
        {
            const size_t lat = i / n1;
            const double u0 = coords[lat * 3], u1 = coords[lat * 3 + 1], u2 = coords[lat * 3 + 2];
            const double nn = std::sqrt( u0 * u0 + u1 * u1 + u2 * u2 );
            h[i]                = ra * ( u0 / nn ) * T[i];
            h[f.nodes + i]      = ra * ( u1 / nn ) * T[i];
            h[2 * f.nodes + i]  = ra * ( u2 / nn ) * T[i];
        }
        for ( int dd = 0; dd < 3; ++dd )
            view_from_host( g.grid_data().comp_[dd], h.data() + dd * f.nodes );
    }
    fe::wedge::operators::shell::VectorMass< double > M( f.domain, f.coords, f.radii, false );
    linalg::apply( M, g, rhs.block_1() );
    linalg::assign( rhs.block_2(), 0.0 );
    fe::strong_algebraic_homogeneous_velocity_dirichlet_enforcement_stokes_like(
        rhs, f.bmask, grid::shell::get_shell_boundary_flag( b, BoundaryConditionFlag::DIRICHLET ) );
    fe::strong_algebraic_freeslip_enforcement_in_place(
        rhs, f.coords, f.bmask, grid::shell::get_shell_boundary_flag( b, BoundaryConditionFlag::FREESLIP ) );
    save_vec( rhs.block_1(), dir + "/f_u.bin", f.nodes );
    return 0;
}

int cmd_fct( int L, double rmin, double rmax, double dt, double kappa, int bc, const std::string& dir )
{
    Setup                               s( L, rmin, rmax );
    linalg::VectorQ1Vec< double >       vel( "vel", s.domain, s.omask );
    linalg::VectorFVScalar< double >    T( "T", s.domain ), src( "src", s.domain );
    linalg::VectorFVVec< double, 3 >    centers( "centers", s.domain );
    load_vec( vel, dir + "/vel.bin", s.nodes );
    const size_t nf = T.grid_data().size();
    view_from_host( T.grid_data(), read_file< double >( dir + "/T.bin", nf ).data() );
    view_from_host( src.grid_data(), read_file< double >( dir + "/src.bin", nf ).data() );
    fv::hex::initialize_cell_centers( centers, s.domain, s.coords, s.radii );
    fv::hex::operators::FVFCTBuffers< double > bufs( s.domain );
    const fv::hex::DirichletBCs< double > bcs{ .T_cmb = 1.0, .T_surface = 0.0, .apply_cmb = true, .apply_surface = true };
    if ( bc )
        fv::hex::apply_dirichlet_bcs( T, s.bmask, bcs, s.domain );
    communication::shell::update_fv_ghost_layers( s.domain, T.grid_data() );
    const double dt_stable =
        fv::hex::operators::compute_dt_stable( s.domain, vel, centers.grid_data(), s.coords, s.radii, kappa );
    const double step = dt > 0 ? dt : 0.5 * dt_stable;
    if ( bc )
        fv::hex::operators::fct_explicit_step( s.domain, T, vel, centers.grid_data(), s.coords, s.radii, step, bufs,
                                               kappa, src.grid_data(), true, s.bmask, bcs );
    else
        fv::hex::operators::fct_explicit_step( s.domain, T, vel, centers.grid_data(), s.coords, s.radii, step, bufs,
                                               kappa, src.grid_data(), true );
    std::vector< double > c( 3 * nf );
    for ( int a = 0; a < 3; ++a )
    {
        auto v = view_to_host( centers.grid_data().comp_[a] );
        std::copy( v.begin(), v.end(), c.begin() + a * nf );
    }
    write_file( dir + "/centers.bin", c.data(), c.size() );
    const double dts[2] = { dt_stable, step };
    write_file( dir + "/dt.bin", dts, 2 );
    auto tl = view_to_host( bufs.T_L );
    write_file( dir + "/TL.bin", tl.data(), tl.size() );
    auto tn = view_to_host( T.grid_data() );
    write_file( dir + "/T.bin", tn.data(), tn.size() );
    return 0;
}

int cmd_gca( int L, double rmin, double rmax, int bcc, int bcs, int diag, int mode, const std::string& dir )
{
    using Op = fe::wedge::operators::shell::EpsilonDivDivKerngen< double >;
    Setup                            f( L, rmin, rmax ), c( L - 1, rmin, rmax );
    linalg::VectorQ1Scalar< double > k( "k", f.domain, f.omask ), kc( "kc", c.domain, c.omask ),
        gcae( "gcae", c.domain, c.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", f.nodes ).data() );
    linalg::assign( kc, 1.0 );
    linalg::assign( gcae, 1.0 );
    BoundaryConditions bn = { { ShellBoundaryFlag::CMB, BoundaryConditionFlag::NEUMANN },
                              { ShellBoundaryFlag::SURFACE, BoundaryConditionFlag::NEUMANN } };
    BoundaryConditions b  = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    Op Af( f.domain, f.coords, f.radii, f.bmask, k.grid_data(), bn, false );
    Op Ac( c.domain, c.coords, c.radii, c.bmask, kc.grid_data(), b, false );
    Ac.set_stored_matrix_mode( linalg::OperatorStoredMatrixMode::Full, 0, gcae.grid_data() );
    linalg::solvers::TwoGridGCA< double, Op >( Af, Ac, 0, gcae.grid_data(), true,
                                               mode == 1 ? linalg::solvers::InterpolationMode::Linear :
                                                           linalg::solvers::InterpolationMode::Constant );
    Ac.set_diagonal( diag != 0 );
    linalg::VectorQ1Vec< double > src( "src", c.domain, c.omask ), dst( "dst", c.domain, c.omask );
    load_vec( src, dir + "/src.bin", c.nodes );
    linalg::apply( Ac, src, dst );
    save_vec( dst, dir + "/dst.bin", c.nodes );
    return 0;
}

// The kerngen slow path on the reference's own assembled wedge matrices: the
// matrices come from get_local_matrix with storage off (assemble_local_matrix,
// epsilon_divdiv_kerngen.hpp:482-498,2051-2110), are written to mats.bin
// ([sd][x][y][r][wedge][18][18], row-major), then stored with
// set_local_matrix under OperatorStoredMatrixMode::Full, which selects the
// slow path (:151-172, :823-1052) for the apply of src.bin -> dst.bin.
int cmd_kerngen_slow( int L, double rmin, double rmax, int bcc, int bcs, int diag, const std::string& dir )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Scalar< double > k( "k", s.domain, s.omask ), gcae( "gcae", s.domain, s.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", s.nodes ).data() );
    linalg::assign( gcae, 1.0 );
    linalg::VectorQ1Vec< double > src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
    load_vec( src, dir + "/src.bin", s.nodes );
    auto      op = make_kerngen( s, k, bcc, bcs, false );
    const int N  = 1 << L;
    using Mat    = dense::Mat< double, 18, 18 >;
    std::vector< Mat > mats( size_t( 10 ) * N * N * N * 2 );
    auto cell = [N]( int sd, int x, int y, int r ) { return ( ( size_t( sd ) * N + x ) * N + y ) * N + r; };
    for ( int sd = 0; sd < 10; ++sd )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                    for ( int w = 0; w < 2; ++w )
                        mats[cell( sd, x, y, r ) * 2 + w] = op.get_local_matrix( sd, x, y, r, w );
    std::vector< double > flat( mats.size() * 18 * 18 );
    for ( size_t i = 0; i < mats.size(); ++i )
        for ( int a = 0; a < 18; ++a )
            for ( int b = 0; b < 18; ++b )
                flat[( i * 18 + a ) * 18 + b] = mats[i]( a, b );
    write_file( dir + "/mats.bin", flat.data(), flat.size() );
    op.set_stored_matrix_mode( linalg::OperatorStoredMatrixMode::Full, 0, gcae.grid_data() );
    for ( int sd = 0; sd < 10; ++sd )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                    for ( int w = 0; w < 2; ++w )
                        op.set_local_matrix( sd, x, y, r, w, mats[cell( sd, x, y, r ) * 2 + w] );
    op.set_diagonal( diag != 0 );
    linalg::apply( op, src, dst );
    save_vec( dst, dir + "/dst.bin", s.nodes );
    return 0;
}

int cmd_epsdivdiv( int L, double rmin, double rmax, int treat, int diag, const std::string& dir )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Scalar< double > k( "k", s.domain, s.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", s.nodes ).data() );
    linalg::VectorQ1Vec< double > src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
    load_vec( src, dir + "/src.bin", s.nodes );
    fe::wedge::operators::shell::EpsilonDivDiv< double > op( s.domain, s.coords, s.radii, s.bmask, k.grid_data(),
                                                             treat != 0, diag != 0 );
    linalg::apply( op, src, dst );
    save_vec( dst, dir + "/dst.bin", s.nodes );
    return 0;
}

int cmd_divkgrad( int L, double rmin, double rmax, int treat, int diag, int single, const std::string& dir )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Scalar< double > k( "k", s.domain, s.omask ), src( "src", s.domain, s.omask ),
        dst( "dst", s.domain, s.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", s.nodes ).data() );
    view_from_host( src.grid_data(), read_file< double >( dir + "/src.bin", s.nodes ).data() );
    fe::wedge::operators::shell::DivKGrad< double > op( s.domain, s.coords, s.radii, s.bmask, k.grid_data(),
                                                        treat != 0, diag != 0 );
    op.set_single_quadpoint( single != 0 );
    linalg::apply( op, src, dst );
    auto out = view_to_host( dst.grid_data() );
    write_file( dir + "/dst.bin", out.data(), out.size() );
    return 0;
}

int cmd_vlaplace( int L, double rmin, double rmax, int bcc, int bcs, int diag, const std::string& dir )
{
    Setup              s( L, rmin, rmax );
    BoundaryConditions b = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    linalg::VectorQ1Vec< double > src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
    load_vec( src, dir + "/src.bin", s.nodes );
    fe::wedge::operators::shell::VectorLaplace< double > op( s.domain, s.coords, s.radii, s.bmask, b, diag != 0 );
    linalg::apply( op, src, dst );
    save_vec( dst, dir + "/dst.bin", s.nodes );
    return 0;
}

// io::XDMFOutput (io/xdmf.hpp:147-1115) of the FE fields T.bin (scalar) and u.bin (3 x nodes, SoA) under DIR/xdmf
int cmd_xdmf_write( int L, double rmin, double rmax, int pts, int conn, const std::string& dir )
{
    Setup     s( L, rmin, rmax );
    const int n1 = ( 1 << L ) + 1;
    auto      T  = read_file< double >( dir + "/T.bin", s.nodes );
    auto      u  = read_file< double >( dir + "/u.bin", 3 * s.nodes );
    grid::Grid4DDataScalar< double > gT( "T", 10, n1, n1, n1 ), gT64( "T64", 10, n1, n1, n1 );
    grid::Grid4DDataScalar< float >  gs( "s32", 10, n1, n1, n1 );
    grid::Grid4DDataVec< double, 3 > gu( "u", 10, n1, n1, n1 ), gu64( "u64", 10, n1, n1, n1 );
    grid::Grid4DDataVec< float, 3 >  gv( "v32", 10, n1, n1, n1 );
    using X = io::XDMFOutput< double >;
    X out( dir + "/xdmf", s.domain, s.coords, s.radii,
           pts == 8 ? X::OutputTypeFloat::Float64 : X::OutputTypeFloat::Float32,
           conn == 4 ? X::OutputTypeInt::Int32 : X::OutputTypeInt::Int64 );
    out.add( gT );
    out.add( gT64, X::OutputTypeFloat::Float64 );
    out.add( gs );
    out.add( gu );
    out.add( gu64, X::OutputTypeFloat::Float64 );
    out.add( gv, X::OutputTypeFloat::Float64 );
    for ( int step = 0; step < 2; ++step )
    {
        std::vector< double > t( T ), w( u );
        std::vector< float >  t32( s.nodes ), w32( 3 * s.nodes );
        for ( size_t i = 0; i < s.nodes; ++i )
            t[i] += step;
        for ( auto& x : w )
            x *= ( 1 + step );
        for ( size_t i = 0; i < s.nodes; ++i )
            t32[i] = float( t[i] );
        for ( size_t i = 0; i < 3 * s.nodes; ++i )
            w32[i] = float( w[i] );
        view_from_host( gT, t.data() );
        view_from_host( gT64, t.data() );
        view_from_host( gs, t32.data() );
        for ( int d = 0; d < 3; ++d )
        {
            view_from_host( gu.comp_[d], w.data() + d * s.nodes );
            view_from_host( gu64.comp_[d], w.data() + d * s.nodes );
            view_from_host( gv.comp_[d], w32.data() + d * s.nodes );
        }
        Kokkos::fence();
        out.write();
    }
    return 0;
}

// io::read_xdmf_checkpoint_metadata / read_xdmf_checkpoint_grid (io/xdmf.hpp:1162-1500) into a FP64 grid
int cmd_xdmf_read( int L, double rmin, double rmax, const std::string& label, int step, int vec,
                   const std::string& ck, const std::string& dir )
{
    Setup     s( L, rmin, rmax );
    const int n1 = ( 1 << L ) + 1;
    {
        auto          m = io::read_xdmf_checkpoint_metadata( ck );
        std::ofstream f( dir + "/meta.txt" );
        if ( m.is_err() )
            f << "error " << m.error() << "\n";
        else
        {
            const auto& md = m.unwrap();
            f << "version " << md.version << "\nsubdomains " << md.num_subdomains_per_diamond_lateral_direction << " "
              << md.num_subdomains_per_diamond_radial_direction << "\nsize " << md.size_x << " " << md.size_y << " "
              << md.size_r << "\ngrid_scalar_bytes " << md.grid_scalar_bytes << "\nordering "
              << md.checkpoint_subdomain_ordering << "\nradii " << md.radii.size() << "\n";
            for ( const auto& g : md.grid_data_files )
                f << "file " << g.grid_name_string << " " << g.scalar_data_type << " " << g.scalar_bytes << " "
                  << g.vec_dim << "\n";
            for ( auto id : md.checkpoint_ordering_0_global_subdomain_ids )
                f << "id " << id << "\n";
        }
    }
    auto fail = [&]( const std::string& msg ) {
        std::ofstream( dir + "/error.txt" ) << msg;
        return 3;
    };
    if ( vec )
    {
        grid::Grid4DDataVec< double, 3 > g( label, 10, n1, n1, n1 );
        auto                             r = io::read_xdmf_checkpoint_grid( ck, label, step, s.domain, g );
        if ( r.is_err() )
            return fail( r.error() );
        std::vector< double > out( 3 * s.nodes );
        for ( int d = 0; d < 3; ++d )
        {
            auto c = view_to_host( g.comp_[d] );
            std::copy( c.begin(), c.end(), out.begin() + d * s.nodes );
        }
        write_file( dir + "/out.bin", out.data(), out.size() );
    }
    else
    {
        grid::Grid4DDataScalar< double > g( label, 10, n1, n1, n1 );
        auto                             r = io::read_xdmf_checkpoint_grid( ck, label, step, s.domain, g );
        if ( r.is_err() )
            return fail( r.error() );
        auto h = view_to_host( g );
        write_file( dir + "/out.bin", h.data(), h.size() );
    }
    return 0;
}

// FE -> FV cell averages (fv/hex/conversion.hpp:349-416) of T.bin, ghost layers updated: fv.bin
int cmd_fe2fv( int L, double rmin, double rmax, const std::string& dir )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Scalar< double > T( "T", s.domain, s.omask );
    linalg::VectorFVScalar< double > fv( "fv", s.domain );
    view_from_host( T.grid_data(), read_file< double >( dir + "/T.bin", s.nodes ).data() );
    linalg::assign( fv, 0.0 );
    fv::hex::l2_project_fe_to_fv( fv, T, s.domain, s.coords, s.radii );
    auto h = view_to_host( fv.grid_data() );
    write_file( dir + "/fv.bin", h.data(), h.size() );
    return 0;
}

// UnsteadyAdvectionDiffusionSUPG (fe/wedge/operators/shell/unsteady_advection_diffusion_supg.hpp:134-420):
// diffusivity kappa, time step dt, mass scaling ms, lumped mass, boundary treatment, diagonal mode; velocity vel.bin
int cmd_supg( int L, double rmin, double rmax, double kappa, double dt, double ms, int lumped, int treat, int diag,
              const std::string& dir )
{
    Setup                            s( L, rmin, rmax );
    linalg::VectorQ1Vec< double >    u( "u", s.domain, s.omask );
    linalg::VectorQ1Scalar< double > src( "src", s.domain, s.omask ), dst( "dst", s.domain, s.omask );
    load_vec( u, dir + "/vel.bin", s.nodes );
    view_from_host( src.grid_data(), read_file< double >( dir + "/src.bin", s.nodes ).data() );
    fe::wedge::operators::shell::UnsteadyAdvectionDiffusionSUPG< double > A(
        s.domain, s.coords, s.radii, s.bmask, u, kappa, dt, treat != 0, diag != 0, ms, lumped != 0 );
    linalg::apply( A, src, dst );
    auto h = view_to_host( dst.grid_data() );
    write_file( dir + "/dst.bin", h.data(), h.size() );
    return 0;
}

// Adaptive GCA (mantlecirculation.cpp:379-387, 565-592 with gca == 2): GCAElementsCollector
// (gca_elements_collector.hpp:19-96) on the fine viscosity, Selective local-matrix storage on the coarse operator
// (local_matrix_storage.hpp:60-216), TwoGridGCA on the marked elements (gca.hpp:155-163) and the coarse apply,
// which assembles the unmarked elements' matrices from kc on the fly (epsilon_divdiv_kerngen.hpp:856-869)
int cmd_agca( int L, double rmin, double rmax, int bcc, int bcs, int diag, const std::string& dir )
{
    using Op = fe::wedge::operators::shell::EpsilonDivDivKerngen< double >;
    Setup                            f( L, rmin, rmax ), c( L - 1, rmin, rmax ), z( L - 2, rmin, rmax );
    linalg::VectorQ1Scalar< double > k( "k", f.domain, f.omask ), kc( "kc", c.domain, c.omask ),
        gcae( "gcae", z.domain, z.omask );
    view_from_host( k.grid_data(), read_file< double >( dir + "/k.bin", f.nodes ).data() );
    view_from_host( kc.grid_data(), read_file< double >( dir + "/kc.bin", c.nodes ).data() );
    linalg::assign( gcae, 0.0 );
    linalg::solvers::GCAElementsCollector< double >( f.domain, k.grid_data(), 2, gcae.grid_data() );
    Kokkos::fence();
    {
        auto h = view_to_host( gcae.grid_data() );
        write_file( dir + "/gcae.bin", h.data(), h.size() );
    }
    BoundaryConditions bn = { { ShellBoundaryFlag::CMB, BoundaryConditionFlag::NEUMANN },
                              { ShellBoundaryFlag::SURFACE, BoundaryConditionFlag::NEUMANN } };
    BoundaryConditions b  = { { ShellBoundaryFlag::CMB, bc_of( bcc ) }, { ShellBoundaryFlag::SURFACE, bc_of( bcs ) } };
    Op Af( f.domain, f.coords, f.radii, f.bmask, k.grid_data(), bn, false );
    Op Ac( c.domain, c.coords, c.radii, c.bmask, kc.grid_data(), b, false );
    Ac.set_stored_matrix_mode( linalg::OperatorStoredMatrixMode::Selective, 1, gcae.grid_data() );
    linalg::solvers::TwoGridGCA< double, Op >( Af, Ac, 1, gcae.grid_data() );
    Ac.set_diagonal( diag != 0 );
    linalg::VectorQ1Vec< double > src( "src", c.domain, c.omask ), dst( "dst", c.domain, c.omask );
    load_vec( src, dir + "/src.bin", c.nodes );
    linalg::apply( Ac, src, dst );
    save_vec( dst, dir + "/dst.bin", c.nodes );
    return 0;
}

} // namespace

int main( int argc, char** argv )
{
    util::terra_initialize( &argc, &argv );
    if ( argc < 2 )
    {
        std::fprintf( stderr, "usage: ref_dump <command> ...\n" );
        return 2;
    }
    const std::string cmd = argv[1];
    auto              I   = [&]( int i ) { return std::atoi( argv[i] ); };
    auto              D   = [&]( int i ) { return std::atof( argv[i] ); };
    if ( cmd == "mesh" && argc == 6 )
        return cmd_mesh( I( 2 ), D( 3 ), D( 4 ), argv[5] );
    if ( cmd == "kerngen" && argc == 9 )
        return cmd_kerngen( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), argv[8] );
    if ( cmd == "time_kerngen" && argc == 8 )
        return cmd_time_kerngen( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ) );
    if ( cmd == "time_kerngen" && argc == 9 )
        return cmd_time_kerngen( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), argv[8] );
    if ( ( cmd == "divergence" || cmd == "gradient" ) && argc == 8 )
        return cmd_stokes_block( cmd == "divergence", I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), argv[7] );
    if ( ( cmd == "prolong" || cmd == "restrict" ) && argc == 6 )
        return cmd_transfer( cmd == "prolong", I( 2 ), D( 3 ), D( 4 ), argv[5] );
    if ( cmd == "stokes_minres" && argc == 12 )
        return cmd_stokes_minres( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), D( 8 ), I( 9 ), D( 10 ), argv[11] );
    if ( cmd == "stokes_fgmres" && argc == 13 )
        return cmd_stokes_fgmres( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), I( 8 ), D( 9 ), I( 10 ), D( 11 ),
                                  argv[12] );
    if ( cmd == "laplace_chebyshev" && argc == 9 )
        return cmd_laplace_chebyshev( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), argv[8] );
    if ( cmd == "laplace_bicgstab" && argc == 9 )
        return cmd_laplace_bicgstab( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), D( 7 ), argv[8] );
    if ( cmd == "laplace_minres" && argc == 8 )
        return cmd_laplace_minres( I( 2 ), D( 3 ), D( 4 ), I( 5 ), D( 6 ), argv[7] );
    if ( cmd == "laplace_fgmres" && argc == 9 )
        return cmd_laplace_fgmres( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), D( 7 ), argv[8] );
    if ( cmd == "kerngen_vcycle" && argc == 13 )
        return cmd_kerngen_vcycle( I( 2 ), I( 3 ), D( 4 ), D( 5 ), I( 6 ), I( 7 ), D( 8 ), I( 9 ), I( 10 ), I( 11 ),
                                   argv[12] );
    if ( cmd == "vcycle" && argc == 11 )
        return cmd_vcycle( I( 2 ), I( 3 ), D( 4 ), D( 5 ), D( 6 ), I( 7 ), I( 8 ), I( 9 ), argv[10] );
    if ( cmd == "stokes" && argc == 8 )
        return cmd_stokes_op( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), argv[7] );
    if ( cmd == "kmass" && argc == 7 )
        return cmd_kmass( I( 2 ), D( 3 ), D( 4 ), I( 5 ), argv[6] );
    if ( ( cmd == "prolong_linear" || cmd == "restrict_linear" ) && argc == 6 )
        return cmd_transfer_linear( cmd == "prolong_linear", I( 2 ), D( 3 ), D( 4 ), argv[5] );
    if ( cmd == "fct" && argc == 9 )
        return cmd_fct( I( 2 ), D( 3 ), D( 4 ), D( 5 ), D( 6 ), I( 7 ), argv[8] );
    if ( cmd == "gca" && argc == 10 )
        return cmd_gca( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), I( 8 ), argv[9] );
    if ( cmd == "l2proj" && argc == 7 )
        return cmd_l2proj( I( 2 ), D( 3 ), D( 4 ), I( 5 ), argv[6] );
    if ( cmd == "stokes_rhs" && argc == 9 )
        return cmd_stokes_rhs( I( 2 ), D( 3 ), D( 4 ), D( 5 ), I( 6 ), I( 7 ), argv[8] );
    if ( cmd == "stokes_mg" && argc == 18 )
        return cmd_stokes_mg( I( 2 ), I( 3 ), D( 4 ), D( 5 ), I( 6 ), I( 7 ), I( 8 ), I( 9 ), D( 10 ), I( 11 ), I( 12 ),
                              I( 13 ), I( 14 ), I( 15 ), I( 16 ), argv[17] );
    if ( cmd == "kerngen_slow" && argc == 9 )
        return cmd_kerngen_slow( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), argv[8] );
    if ( cmd == "epsdivdiv" && argc == 8 )
        return cmd_epsdivdiv( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), argv[7] );
    if ( cmd == "divkgrad" && argc == 9 )
        return cmd_divkgrad( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), argv[8] );
    if ( cmd == "vlaplace" && argc == 9 )
        return cmd_vlaplace( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), argv[8] );
    if ( ( cmd == "mass" || cmd == "vmass" ) && argc == 7 )
        return cmd_mass( cmd == "vmass", I( 2 ), D( 3 ), D( 4 ), I( 5 ), argv[6] );
    if ( cmd == "laplace_cg" && argc == 8 )
        return cmd_laplace_cg( I( 2 ), D( 3 ), D( 4 ), I( 5 ), D( 6 ), argv[7] );
    if ( cmd == "laplace" && argc == 8 )
        return cmd_laplace( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), argv[7] );
    if ( cmd == "xdmf_write" && argc == 8 )
        return cmd_xdmf_write( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), argv[7] );
    if ( cmd == "xdmf_read" && argc == 10 )
        return cmd_xdmf_read( I( 2 ), D( 3 ), D( 4 ), argv[5], I( 6 ), I( 7 ), argv[8], argv[9] );
    if ( cmd == "fe2fv" && argc == 6 )
        return cmd_fe2fv( I( 2 ), D( 3 ), D( 4 ), argv[5] );
    if ( cmd == "supg" && argc == 12 )
        return cmd_supg( I( 2 ), D( 3 ), D( 4 ), D( 5 ), D( 6 ), D( 7 ), I( 8 ), I( 9 ), I( 10 ), argv[11] );
    if ( cmd == "kerngen_rank" && argc == 10 )
        return cmd_kerngen_rank( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), I( 8 ), argv[9] );
    if ( cmd == "agca" && argc == 9 )
        return cmd_agca( I( 2 ), D( 3 ), D( 4 ), I( 5 ), I( 6 ), I( 7 ), argv[8] );
    std::fprintf( stderr, "ref_dump: bad command line\n" );
    return 2;
}
