// Wedge-element helpers shared by the operator kernels.
//
// Cell (x, y, r) of a diamond is split into two wedges whose lateral
// vertices are (0,0),(1,0),(0,1) and (1,1),(0,1),(1,0)
// (fe/wedge/kernel_helpers.hpp:26-60); nodes 0-2 lie on shell r, 3-5 on r+1.
#pragma once

#include "common.cuh"

namespace tn {

static __device__ __constant__ const int kWedgeNode[2][6][3] = {
    { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 }, { 1, 0, 1 }, { 0, 1, 1 } },
    { { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } } };

__host__ __device__ inline size_t lat_index( int n1, int d, int x, int y ) { return ( size_t( d ) * n1 + x ) * n1 + y; }
// kWedgeNode as a constant expression: offset k (0: x, 1: y, 2: r) of node n of wedge w.  In fully
// unrolled loops the indices it yields are compile-time, so per-node arrays indexed with them stay in
// registers (indexing through the __constant__ table puts them in local memory).
__host__ __device__ constexpr int wedge_node( int w, int n, int k )
{
    return k == 2 ? int( n >= 3 ) : ( w == 0 ? int( n % 3 == ( k == 0 ? 1 : 2 ) ) : int( n % 3 != ( k == 0 ? 1 : 2 ) ) );
}


// Lateral triangle matrix M = [p1-p0, p2-p0, (p0+p1+p2)/3] of a wedge.  For
// the one-point rule J = M diag(r_mid, r_mid, dr/2); Q = M^{-T}.  Writes Q's
// columns q0, q1, q2 (9 values) and |det M|.
__device__ inline void lateral_geometry( const double* p0, const double* p1, const double* p2, double* q, double* adet )
{
    double M[3][3];
    for ( int a = 0; a < 3; ++a )
    {
        M[a][0] = p1[a] - p0[a];
        M[a][1] = p2[a] - p0[a];
        M[a][2] = ( p0[a] + p1[a] + p2[a] ) * ( 1.0 / 3.0 );
    }
    const double det = M[0][0] * ( M[1][1] * M[2][2] - M[1][2] * M[2][1] ) -
                       M[0][1] * ( M[1][0] * M[2][2] - M[1][2] * M[2][0] ) +
                       M[0][2] * ( M[1][0] * M[2][1] - M[1][1] * M[2][0] );
    const double id = 1.0 / det;
    // Q[a][b] = (M^{-1})[b][a]; column b of Q stored at q[3 b + a]
    double Q[3][3];
    Q[0][0] = ( M[1][1] * M[2][2] - M[1][2] * M[2][1] ) * id;
    Q[0][1] = ( M[1][2] * M[2][0] - M[1][0] * M[2][2] ) * id;
    Q[0][2] = ( M[1][0] * M[2][1] - M[1][1] * M[2][0] ) * id;
    Q[1][0] = ( M[0][2] * M[2][1] - M[0][1] * M[2][2] ) * id;
    Q[1][1] = ( M[0][0] * M[2][2] - M[0][2] * M[2][0] ) * id;
    Q[1][2] = ( M[0][1] * M[2][0] - M[0][0] * M[2][1] ) * id;
    Q[2][0] = ( M[0][1] * M[1][2] - M[0][2] * M[1][1] ) * id;
    Q[2][1] = ( M[0][2] * M[1][0] - M[0][0] * M[1][2] ) * id;
    Q[2][2] = ( M[0][0] * M[1][1] - M[0][1] * M[1][0] ) * id;
    for ( int b = 0; b < 3; ++b )
        for ( int a = 0; a < 3; ++a )
            q[3 * b + a] = Q[a][b];
    *adet = fabs( det );
}

// Jacobian of x = r(zeta) ((1-xi-eta) p0 + xi p1 + eta p2) at (xi, eta, zeta)
// (fe/wedge/integrands.hpp:579-681), its determinant and inverse transpose.
template < typename T >
__device__ inline T wedge_jacobian_it( const T* p0, const T* p1, const T* p2, T r1, T r2, T xi, T eta, T zeta,
                                       T IT[3][3] )
{
    const T r  = r1 + T( 0.5 ) * ( r2 - r1 ) * ( T( 1 ) + zeta );
    const T dr = T( 0.5 ) * ( r2 - r1 );
    T       J[3][3];
    for ( int a = 0; a < 3; ++a )
    {
        J[a][0] = ( p1[a] - p0[a] ) * r;
        J[a][1] = ( p2[a] - p0[a] ) * r;
        J[a][2] = ( ( T( 1 ) - xi - eta ) * p0[a] + xi * p1[a] + eta * p2[a] ) * dr;
    }
    const T det = J[0][0] * ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) - J[0][1] * ( J[1][0] * J[2][2] - J[1][2] * J[2][0] ) +
                  J[0][2] * ( J[1][0] * J[2][1] - J[1][1] * J[2][0] );
    const T id = T( 1 ) / det;
    IT[0][0]   = ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) * id;
    IT[0][1]   = ( J[1][2] * J[2][0] - J[1][0] * J[2][2] ) * id;
    IT[0][2]   = ( J[1][0] * J[2][1] - J[1][1] * J[2][0] ) * id;
    IT[1][0]   = ( J[0][2] * J[2][1] - J[0][1] * J[2][2] ) * id;
    IT[1][1]   = ( J[0][0] * J[2][2] - J[0][2] * J[2][0] ) * id;
    IT[1][2]   = ( J[0][1] * J[2][0] - J[0][0] * J[2][1] ) * id;
    IT[2][0]   = ( J[0][1] * J[1][2] - J[0][2] * J[1][1] ) * id;
    IT[2][1]   = ( J[0][2] * J[1][0] - J[0][0] * J[1][2] ) * id;
    IT[2][2]   = ( J[0][0] * J[1][1] - J[0][1] * J[1][0] ) * id;
    return det;
}

// Reference-element gradient of wedge shape function n (integrands.hpp:160-227).
template < typename T >
__device__ inline void grad_shape_ref( int n, T xi, T eta, T zeta, T g[3] )
{
    const T nrad = n < 3 ? T( 0.5 ) * ( T( 1 ) - zeta ) : T( 0.5 ) * ( T( 1 ) + zeta );
    const T grad = n < 3 ? T( -0.5 ) : T( 0.5 );
    const int m  = n % 3;
    g[0]         = ( m == 0 ? T( -1 ) : ( m == 1 ? T( 1 ) : T( 0 ) ) ) * nrad;
    g[1]         = ( m == 0 ? T( -1 ) : ( m == 2 ? T( 1 ) : T( 0 ) ) ) * nrad;
    g[2]         = ( m == 0 ? T( 1 ) - xi - eta : ( m == 1 ? xi : eta ) ) * grad;
}

// Normal / tangential basis (rows n, t1, t2) of
// trafo_mat_cartesian_to_normal_tangential (linalg/trafo/local_basis_trafo_normal_tangential.hpp:36-73).
template < typename T >
__device__ inline void trafo_normal_tangential( const T nin[3], T R[3][3] )
{
    T       n[3] = { nin[0], nin[1], nin[2] };
    T       s    = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    T       m    = sqrt( s );
    const T tiny = sizeof( T ) == 8 ? T( 1e-15 ) : T( 1e-6 );
    if ( m > T( 1e-15 ) )
        n[0] /= m, n[1] /= m, n[2] /= m;
    const T ax = fabs( n[0] ), ay = fabs( n[1] ), az = fabs( n[2] );
    T       ref[3] = { 0, 0, 0 };
    if ( ax <= ay && ax <= az )
        ref[0] = 1;
    else if ( ay <= ax && ay <= az )
        ref[1] = 1;
    else
        ref[2] = 1;
    T t1[3] = { ref[1] * n[2] - ref[2] * n[1], ref[2] * n[0] - ref[0] * n[2], ref[0] * n[1] - ref[1] * n[0] };
    m       = sqrt( t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2] );
    if ( m > T( 1e-15 ) )
        t1[0] /= m, t1[1] /= m, t1[2] /= m;
    if ( sqrt( t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2] ) < tiny )
    {
        t1[0] = n[1], t1[1] = -n[0], t1[2] = 0;
        m     = sqrt( t1[0] * t1[0] + t1[1] * t1[1] );
        if ( m > T( 1e-15 ) )
            t1[0] /= m, t1[1] /= m;
    }
    T t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
    m       = sqrt( t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2] );
    if ( m > T( 1e-15 ) )
        t2[0] /= m, t2[1] /= m, t2[2] /= m;
    for ( int k = 0; k < 3; ++k )
        R[0][k] = n[k], R[1][k] = t1[k], R[2][k] = t2[k];
}

// Linear transfer stencil of fine node (d, x, y, r) on a fine mesh of Nf
// cells (grid_transfer_linear.hpp:14-158, prolongation_linear.hpp:104-189):
// on a coarse node: weight 1; between two radially aligned coarse nodes:
// interpolation by radius; otherwise on the wedge facet of two lateral coarse
// pairs: radial interpolation between the pairs' chord midpoints, each pair
// member weighted half.  Returns the number of (coarse x, y, r, weight).
__device__ __forceinline__ int linear_stencil( int Nf, const double* __restrict__ coords, const double* __restrict__ radii, int d,
                               int x, int y, int r, int cx[4], int cy[4], int cr[4], double w[4] )
{
    const int n1 = Nf + 1;
    if ( !( x & 1 ) && !( y & 1 ) && !( r & 1 ) )
    {
        cx[0] = x / 2, cy[0] = y / 2, cr[0] = r / 2, w[0] = 1.0;
        return 1;
    }
    const int     rb = r < Nf ? r / 2 : r / 2 - 1, rt = rb + 1;
    const double* c  = coords + lat_index( n1, d, x, y ) * 3;
    const double  Rf = radii[d * n1 + r], Rb = radii[d * n1 + 2 * rb], Rt = radii[d * n1 + 2 * rt];
    const double  nf = sqrt( ( c[0] * Rf ) * ( c[0] * Rf ) + ( c[1] * Rf ) * ( c[1] * Rf ) + ( c[2] * Rf ) * ( c[2] * Rf ) );
    if ( !( x & 1 ) && !( y & 1 ) )
    {
        const double nb = sqrt( ( c[0] * Rb ) * ( c[0] * Rb ) + ( c[1] * Rb ) * ( c[1] * Rb ) + ( c[2] * Rb ) * ( c[2] * Rb ) );
        const double nt = sqrt( ( c[0] * Rt ) * ( c[0] * Rt ) + ( c[1] * Rt ) * ( c[1] * Rt ) + ( c[2] * Rt ) * ( c[2] * Rt ) );
        const double nu = ( nf - nb ) / ( nt - nb );
        cx[0] = cx[1] = x / 2, cy[0] = cy[1] = y / 2, cr[0] = rb, cr[1] = rt;
        w[0] = 1.0 - nu, w[1] = nu;
        return 2;
    }
    int x0, x1, y0, y1;
    if ( !( x & 1 ) )
        x0 = x1 = x / 2, y0 = y / 2, y1 = y / 2 + 1;
    else if ( !( y & 1 ) )
        x0 = x / 2, x1 = x / 2 + 1, y0 = y1 = y / 2;
    else
        x0 = x / 2 + 1, x1 = x / 2, y0 = y / 2, y1 = y / 2 + 1;
    const double* c0 = coords + lat_index( n1, d, 2 * x0, 2 * y0 ) * 3;
    const double* c1 = coords + lat_index( n1, d, 2 * x1, 2 * y1 ) * 3;
    double        sb = 0.0, st = 0.0;
    for ( int a = 0; a < 3; ++a )
    {
        const double b = 0.5 * ( c0[a] * Rb + c1[a] * Rb ), t = 0.5 * ( c0[a] * Rt + c1[a] * Rt );
        sb += b * b, st += t * t;
    }
    const double nb = sqrt( sb ), nt = sqrt( st );
    const double nu = ( nf - nb ) / ( nt - nb );
    const double wb = 0.5 * ( 1.0 - nu ), wt = 0.5 * nu;
    cx[0] = x0, cy[0] = y0, cr[0] = rb, w[0] = wb;
    cx[1] = x1, cy[1] = y1, cr[1] = rb, w[1] = wb;
    cx[2] = x0, cy[2] = y0, cr[2] = rt, w[2] = wt;
    cx[3] = x1, cy[3] = y1, cr[3] = rt, w[3] = wt;
    return 4;
}

}  // namespace tn
