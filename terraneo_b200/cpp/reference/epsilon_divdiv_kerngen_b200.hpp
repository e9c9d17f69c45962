// Reference-side binding: the class a maintainer adds to the reference's tree
// (e.g. as fe/wedge/operators/shell/epsilon_divdiv_kerngen_b200.hpp) so the
// reference's own drivers (linalg::apply, PCG, FGMRES, Chebyshev, Multigrid)
// run the B200 epsilon-div-div apply on the reference's vectors.
//
// It satisfies linalg::OperatorLike (linalg/operator.hpp:57-71) on
// linalg::VectorQ1Vec (linalg/vector_q1.hpp) and mirrors the members of
// EpsilonDivDivKerngen it replaces (epsilon_divdiv_kerngen.hpp:175-432):
// the constructor's boundary conditions and diagonal flag, set_diagonal,
// set_operator_apply_and_communication_modes and apply_impl.  apply_impl
// forwards the views' data pointers to tn_epsdivdiv_apply_f64 / _f32; on a
// Kokkos CUDA build the views live in device memory, as the C ABI expects.
// Errors of the C ABI surface as std::runtime_error, the reference's host
// error convention (vector_q1.hpp:61).
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "grid/grid_types.hpp"
#include "grid/shell/bit_masks.hpp"
#include "linalg/operator.hpp"
#include "linalg/vector_q1.hpp"
#include "terraneo_b200.h"

namespace terra::fe::wedge::operators::shell {

template < typename ScalarT >
class EpsilonDivDivKerngenB200
{
  public:
    using SrcVectorType = linalg::VectorQ1Vec< ScalarT >;
    using DstVectorType = linalg::VectorQ1Vec< ScalarT >;
    using ScalarType    = ScalarT;

    // level / radii of the subdomain-per-diamond shell (DistributedDomain::create_uniform(level, level, r_min,
    // r_max, 0, 0)), the nodal viscosity field and the boundary conditions of EpsilonDivDivKerngen
    EpsilonDivDivKerngenB200( int                                         level,
                              double                                      r_min,
                              double                                      r_max,
                              const grid::Grid4DDataScalar< ScalarT >&    k,
                              const grid::shell::BoundaryConditions       bcs,
                              bool                                        diagonal = false )
    : k_( k )
    {
        tn_mesh* m = nullptr;
        check( tn_mesh_create( level, r_min, r_max, &m ) );
        mesh_ = std::shared_ptr< tn_mesh >( m, []( tn_mesh* q ) { tn_mesh_destroy( q ); } );
        prm_  = { code( grid::shell::get_boundary_condition_flag( bcs, grid::shell::ShellBoundaryFlag::CMB ) ),
                  code( grid::shell::get_boundary_condition_flag( bcs, grid::shell::ShellBoundaryFlag::SURFACE ) ),
                  diagonal ? 1 : 0,
                  TN_APPLY_REPLACE,
                  TN_COMM_ADDITIVE,
                  1.0 };
    }

    void set_diagonal( bool d ) { prm_.diagonal = d ? 1 : 0; }

    void set_operator_apply_and_communication_modes( linalg::OperatorApplyMode         a,
                                                     linalg::OperatorCommunicationMode c )
    {
        prm_.apply_mode = a == linalg::OperatorApplyMode::Add ? TN_APPLY_ADD : TN_APPLY_REPLACE;
        prm_.comm_mode  = c == linalg::OperatorCommunicationMode::SkipCommunication ? TN_COMM_SKIP : TN_COMM_ADDITIVE;
    }

    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const ScalarT* s[3] = { src.grid_data().comp_[0].data(), src.grid_data().comp_[1].data(),
                                src.grid_data().comp_[2].data() };
        ScalarT*       d[3] = { dst.grid_data().comp_[0].data(), dst.grid_data().comp_[1].data(),
                                dst.grid_data().comp_[2].data() };
        if constexpr ( std::is_same_v< ScalarT, double > )
            check( tn_epsdivdiv_apply_f64( mesh_.get(), &prm_, k_.data(), s, d, nullptr ) );
        else
            check( tn_epsdivdiv_apply_f32( mesh_.get(), &prm_, k_.data(), s, d, nullptr ) );
    }

  private:
    static int code( grid::shell::BoundaryConditionFlag f )
    {
        switch ( f )
        {
        case grid::shell::BoundaryConditionFlag::DIRICHLET:
            return TN_BC_DIRICHLET;
        case grid::shell::BoundaryConditionFlag::FREESLIP:
            return TN_BC_FREESLIP;
        default:
            return TN_BC_NEUMANN;
        }
    }
    static void check( int rc )
    {
        if ( rc != TN_OK )
            throw std::runtime_error( std::string( "EpsilonDivDivKerngenB200: " ) + tn_last_error() );
    }

    std::shared_ptr< tn_mesh >        mesh_; // shared: the reference's drivers copy operators
    tn_epsdivdiv_params               prm_{};
    grid::Grid4DDataScalar< ScalarT > k_;
};

}  // namespace terra::fe::wedge::operators::shell
