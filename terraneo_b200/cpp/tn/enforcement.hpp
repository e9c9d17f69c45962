// Strong algebraic boundary-condition enforcement on right-hand sides
// (fe/strong_algebraic_dirichlet_enforcement.hpp,
// fe/strong_algebraic_freeslip_enforcement.hpp) over the C ABI.
//
// Dirichlet: b <- b - A_neumann g everywhere, then b <- diag(A_neumann) g on
// the Dirichlet boundary layers (tn_vec_assign_boundary_*); homogeneous
// variants set the boundary entries to 0.  Free-slip: the normal component of
// the velocity right-hand side is removed on the free-slip layers (the
// reference rotates to the (n, t1, t2) basis, zeroes n and rotates back).
#pragma once

#include "operators.hpp"

namespace tn {

// y = x (or c when x is null) on the selected radial boundary layers
template < typename T, int NC >
void assign_boundary( VectorQ1Base< T, NC >& y, const VectorQ1Base< T, NC >* x, double c, bool cmb, bool surface )
{
    T*       py[3];
    const T* px[3] = { nullptr, nullptr, nullptr };
    y.ptrs( py );
    if ( x )
        for ( int k = 0; k < NC; ++k )
            px[k] = x->comp( k );
    if constexpr ( std::is_same_v< T, double > )
        check( tn_vec_assign_boundary_f64( y.mesh().get(), NC, py, x ? px : nullptr, c, cmb, surface, stream() ),
               "assign_boundary" );
    else
        check( tn_vec_assign_boundary_f32( y.mesh().get(), NC, py, x ? px : nullptr, c, cmb, surface, stream() ),
               "assign_boundary" );
}

// strong_algebraic_dirichlet_enforcement_poisson_like / _vectorlaplace_like
// (strong_algebraic_dirichlet_enforcement.hpp:10-45): A_neumann and
// A_neumann_diag are the operator without boundary treatment and its
// diagonal-only version
template < typename Op, typename V >
void strong_algebraic_dirichlet_enforcement( Op& A_neumann, Op& A_neumann_diag, const V& g, V& tmp, V& b, bool cmb,
                                             bool surface )
{
    using S = typename V::ScalarType;
    apply( A_neumann, g, tmp );
    lincomb( b, { S( 1 ), S( -1 ) }, { b, tmp } );
    apply( A_neumann_diag, g, tmp );
    assign_boundary( b, &tmp, 0.0, cmb, surface );
}

// strong_algebraic_homogeneous_dirichlet_enforcement_* (:47-95)
template < typename V >
void strong_algebraic_homogeneous_dirichlet_enforcement( V& b, bool cmb, bool surface )
{
    assign_boundary( b, static_cast< const V* >( nullptr ), 0.0, cmb, surface );
}

// strong_algebraic_freeslip_enforcement_in_place (strong_algebraic_freeslip_enforcement.hpp:9-24)
inline void strong_algebraic_freeslip_enforcement_in_place( VectorQ1Vec< double >& b, bool cmb, bool surface )
{
    double* p[3];
    b.ptrs( p );
    check( tn_freeslip_project_f64( b.mesh().get(), p, cmb, surface, stream() ), "freeslip_project" );
}

}  // namespace tn
