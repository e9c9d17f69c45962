/* CPU restatement of the reference's hot path (TEST INFRASTRUCTURE, not the
 * product).  See oracle.h for layout conventions.  Plain scalar C; every
 * function names the reference code it restates. */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NDIAMOND 10

static inline size_t lat_idx( int n1, int d, int x, int y ) { return ( (size_t) d * n1 + x ) * n1 + y; }
static inline size_t node_idx( int n1, int d, int x, int y, int r )
{
    return ( ( (size_t) d * n1 + x ) * n1 + y ) * n1 + r;
}

/* ------------------------------------------------------------------------ */
/* Mesh: grid/shell/spherical_shell.hpp                                      */
/* ------------------------------------------------------------------------ */

static void normalize3( double v[3] )
{
    /* dense/vec.hpp:76-98: norm = sqrt(sum of squares), divide if > 1e-15 */
    double s = 0.0;
    for ( int i = 0; i < 3; ++i )
        s += v[i] * v[i];
    double m = sqrt( s );
    if ( m > 1e-15 )
        for ( int i = 0; i < 3; ++i )
            v[i] /= m;
}

/* Icosahedral base points and diamond table: spherical_shell.hpp:420-559.
 * Diamond corners p00 = pole, pN0 = "left", pNN = opposite, p0N = "right". */
static void diamond_corners( int diamond, double p00[3], double pN0[3], double pNN[3], double p0N[3] )
{
    double node[12][3];
    double fifthpi = 0.4 * asin( 1.0 );
    double w       = 2.0 * acos( 1.0 / ( 2.0 * sin( fifthpi ) ) );
    double cosw = cos( w ), sinw = sin( w );
    node[0][0] = 0.0, node[0][1] = 0.0, node[0][2] = 1.0;
    node[11][0] = 0.0, node[11][1] = 0.0, node[11][2] = -1.0;
    for ( int k = 1; k <= 5; ++k )
    {
        double phi = 2.0 * ( (double) k - 0.5 ) * fifthpi;
        node[k][0] = sinw * cos( phi ), node[k][1] = sinw * sin( phi ), node[k][2] = cosw;
    }
    for ( int k = 1; k <= 5; ++k )
    {
        double phi     = 2.0 * ( (double) k - 1 ) * fifthpi;
        node[k + 5][0] = sinw * cos( phi ), node[k + 5][1] = sinw * sin( phi ), node[k + 5][2] = -cosw;
    }
    static const int dn[10][4] = { { 0, 5, 6, 1 },   { 0, 1, 7, 2 },  { 0, 2, 8, 3 },  { 0, 3, 9, 4 },
                                   { 0, 4, 10, 5 },  { 11, 7, 1, 6 }, { 11, 8, 2, 7 }, { 11, 9, 3, 8 },
                                   { 11, 10, 4, 9 }, { 11, 6, 5, 10 } };
    int L = diamond < 5 ? 1 : 3, R = diamond < 5 ? 3 : 1;
    for ( int i = 0; i < 3; ++i )
    {
        p00[i] = node[dn[diamond][0]][i];
        pN0[i] = node[dn[diamond][L]][i];
        pNN[i] = node[dn[diamond][2]][i];
        p0N[i] = node[dn[diamond][R]][i];
    }
}

/* compute_node_recursive (spherical_shell.hpp:231-346): each new point is
 * normalize(p1 + p2) of its two parents on the next-coarser grid; rows
 * (i%l==0, j%l==l/2), columns (i%l==l/2, j%l==0), diagonals (both l/2, parents
 * (i-l/2, j+l/2) and (i+l/2, j-l/2)).  Restated level by level, coarse to fine. */
void or_unit_sphere_coords( int L, double* coords )
{
    const int N = 1 << L, n1 = N + 1;
    for ( int d = 0; d < NDIAMOND; ++d )
    {
        double* c = coords + (size_t) d * n1 * n1 * 3;
#define P( i, j ) ( c + ( (size_t) ( i ) * n1 + ( j ) ) * 3 )
        diamond_corners( d, P( 0, 0 ), P( N, 0 ), P( N, N ), P( 0, N ) );
        for ( int l = N; l >= 2; l /= 2 )
        {
            const int h = l / 2;
            for ( int i = 0; i <= N; i += h )
                for ( int j = 0; j <= N; j += h )
                {
                    const int ri = i % l, rj = j % l;
                    const double *a, *b;
                    if ( ri == 0 && rj == h )
                        a = P( i, j - h ), b = P( i, j + h );
                    else if ( ri == h && rj == 0 )
                        a = P( i - h, j ), b = P( i + h, j );
                    else if ( ri == h && rj == h )
                        a = P( i - h, j + h ), b = P( i + h, j - h );
                    else
                        continue;
                    double* o = P( i, j );
                    for ( int k = 0; k < 3; ++k )
                        o[k] = a[k] + b[k];
                    normalize3( o );
                }
        }
#undef P
    }
}

/* uniform_shell_radii (spherical_shell.hpp:28-50) + subdomain_shell_radii (:2759) */
void or_shell_radii( int L, double rmin, double rmax, double* radii )
{
    const int    N    = 1 << L;
    const double step = ( rmax - rmin ) / N;
    for ( int d = 0; d < NDIAMOND; ++d )
    {
        for ( int i = 0; i <= N; ++i )
            radii[d * ( N + 1 ) + i] = rmin + i * step;
        radii[d * ( N + 1 ) + N] = rmax;
    }
}

/* setup_boundary_mask_data (grid/shell/bit_masks.hpp:82-137):
 * INNER = 1 everywhere, CMB = 6 at r = 0, SURFACE = 10 at r = N. */
void or_boundary_mask( int L, uint8_t* bmask )
{
    const int n1 = ( 1 << L ) + 1;
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < n1; ++x )
            for ( int y = 0; y < n1; ++y )
                for ( int r = 0; r < n1; ++r )
                    bmask[node_idx( n1, d, x, y, r )] = r == 0 ? 6 : ( r == n1 - 1 ? 10 : 1 );
}

/* Duplicated lateral positions: nodes of different diamonds that are the
 * same point on the sphere (shared diamond edges and icosahedral vertices).
 * They are found by exact comparison of the unit-sphere coordinates, which
 * the bisection produces bit-identically on both sides of a shared edge. */
typedef struct
{
    double c[3];
    int    d, x, y;
} LatNode;

static int cmp_latnode( const void* pa, const void* pb )
{
    const LatNode* a = (const LatNode*) pa;
    const LatNode* b = (const LatNode*) pb;
    for ( int k = 0; k < 3; ++k )
    {
        if ( a->c[k] < b->c[k] )
            return -1;
        if ( a->c[k] > b->c[k] )
            return 1;
    }
    return a->d - b->d;
}

/* Returns sorted lateral nodes; *ngroups groups given by start offsets. */
static LatNode* build_groups( int L, const double* coords, int** gstart, int* ngroups )
{
    const int n1 = ( 1 << L ) + 1;
    const int nl = NDIAMOND * n1 * n1;
    LatNode*  v  = (LatNode*) malloc( sizeof( LatNode ) * nl );
    int       t  = 0;
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < n1; ++x )
            for ( int y = 0; y < n1; ++y, ++t )
            {
                memcpy( v[t].c, coords + lat_idx( n1, d, x, y ) * 3, sizeof( double ) * 3 );
                v[t].d = d, v[t].x = x, v[t].y = y;
            }
    qsort( v, nl, sizeof( LatNode ), cmp_latnode );
    int* gs = (int*) malloc( sizeof( int ) * ( nl + 1 ) );
    int  g  = 0;
    for ( int i = 0; i < nl; ++i )
        if ( i == 0 || memcmp( v[i].c, v[i - 1].c, sizeof( double ) * 3 ) != 0 )
            gs[g++] = i;
    gs[g]    = nl;
    *gstart  = gs;
    *ngroups = g;
    return v;
}

/* setup_node_ownership_mask_data (grid/bit_masks.hpp:29-80): a node is OWNED
 * (1) on the copy whose global subdomain id is the minimum among all copies;
 * with one subdomain per diamond that is the lowest diamond id. */
void or_ownership_mask( int L, const double* coords, uint8_t* omask )
{
    const int n1 = ( 1 << L ) + 1;
    int *     gs, ng;
    LatNode*  v = build_groups( L, coords, &gs, &ng );
    memset( omask, 0, (size_t) NDIAMOND * n1 * n1 * n1 );
    for ( int g = 0; g < ng; ++g )
    {
        const LatNode* o = &v[gs[g]]; /* sorted by diamond inside a group */
        for ( int r = 0; r < n1; ++r )
            omask[node_idx( n1, o->d, o->x, o->y, r )] = 1;
    }
    free( gs );
    free( v );
}

/* Additive halo exchange (communication/shell/communication.hpp:242-747 and
 * communication_plan.hpp:48-68): every copy of a duplicated node receives the
 * sum of all copies. */
void or_halo_sum( int L, const double* coords, double* field, int ncomp )
{
    const int    n1 = ( 1 << L ) + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    int *        gs, ng;
    LatNode*     v = build_groups( L, coords, &gs, &ng );
    for ( int c = 0; c < ncomp; ++c )
    {
        double* f = field + c * ns;
        for ( int g = 0; g < ng; ++g )
        {
            if ( gs[g + 1] - gs[g] < 2 )
                continue;
            for ( int r = 0; r < n1; ++r )
            {
                double s = 0.0;
                for ( int i = gs[g]; i < gs[g + 1]; ++i )
                    s += f[node_idx( n1, v[i].d, v[i].x, v[i].y, r )];
                for ( int i = gs[g]; i < gs[g + 1]; ++i )
                    f[node_idx( n1, v[i].d, v[i].x, v[i].y, r )] = s;
            }
        }
    }
    free( gs );
    free( v );
}

double or_masked_dot( size_t n, const double* a, const double* b, const uint8_t* omask )
{
    /* kernels/common/grid_operations.hpp:644 masked_dot_product */
    double s = 0.0;
    for ( size_t i = 0; i < n; ++i )
        if ( omask[i] & 1 )
            s += a[i] * b[i];
    return s;
}

/* ------------------------------------------------------------------------ */
/* Wedge geometry: fe/wedge/integrands.hpp, kernel_helpers.hpp               */
/* ------------------------------------------------------------------------ */

/* wedge node -> (dx, dy, dr) inside the hex cell (kernel_helpers.hpp:26-60,
 * epsilon_divdiv_kerngen.hpp:1160-1162) */
static const int WNODE[2][6][3] = { { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 }, { 1, 0, 1 }, { 0, 1, 1 } },
                                    { { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } } };

/* Jacobian of x = r(zeta) ((1-xi-eta) p0 + xi p1 + eta p2) (integrands.hpp:634-681) */
static void wedge_jac( const double* p[3], double r1, double r2, double xi, double eta, double zeta, double J[3][3] )
{
    const double r  = r1 + 0.5 * ( r2 - r1 ) * ( 1 + zeta );
    const double dr = 0.5 * ( r2 - r1 );
    for ( int a = 0; a < 3; ++a )
    {
        J[a][0] = ( p[1][a] - p[0][a] ) * r;
        J[a][1] = ( p[2][a] - p[0][a] ) * r;
        J[a][2] = ( ( 1 - xi - eta ) * p[0][a] + xi * p[1][a] + eta * p[2][a] ) * dr;
    }
}

static double det3( double J[3][3] )
{
    return J[0][0] * ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) - J[0][1] * ( J[1][0] * J[2][2] - J[1][2] * J[2][0] ) +
           J[0][2] * ( J[1][0] * J[2][1] - J[1][1] * J[2][0] );
}

/* inverse transposed: IT[a][b] = (J^{-1})[b][a] */
static void inv_transposed3( double J[3][3], double det, double IT[3][3] )
{
    const double id = 1.0 / det;
    IT[0][0]        = ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) * id;
    IT[0][1]        = ( J[1][2] * J[2][0] - J[1][0] * J[2][2] ) * id;
    IT[0][2]        = ( J[1][0] * J[2][1] - J[1][1] * J[2][0] ) * id;
    IT[1][0]        = ( J[0][2] * J[2][1] - J[0][1] * J[2][2] ) * id;
    IT[1][1]        = ( J[0][0] * J[2][2] - J[0][2] * J[2][0] ) * id;
    IT[1][2]        = ( J[0][1] * J[2][0] - J[0][0] * J[2][1] ) * id;
    IT[2][0]        = ( J[0][1] * J[1][2] - J[0][2] * J[1][1] ) * id;
    IT[2][1]        = ( J[0][2] * J[1][0] - J[0][0] * J[1][2] ) * id;
    IT[2][2]        = ( J[0][0] * J[1][1] - J[0][1] * J[1][0] ) * id;
}

/* reference-element gradient of wedge shape function n (integrands.hpp:160-227) */
static void grad_shape_ref( int n, double xi, double eta, double zeta, double g[3] )
{
    static const double gxi[3] = { -1.0, 1.0, 0.0 }, geta[3] = { -1.0, 0.0, 1.0 };
    const double        nrad   = n < 3 ? 0.5 * ( 1 - zeta ) : 0.5 * ( 1 + zeta );
    const double        grad   = n < 3 ? -0.5 : 0.5;
    const double        lat[3] = { 1.0 - xi - eta, xi, eta };
    g[0]                       = gxi[n % 3] * nrad;
    g[1]                       = geta[n % 3] * nrad;
    g[2]                       = lat[n % 3] * grad;
}

static void wedge_lateral_points( int n1, const double* coords, int d, int x, int y, int w, const double* p[3] )
{
    for ( int i = 0; i < 3; ++i )
        p[i] = coords + lat_idx( n1, d, x + WNODE[w][i][0], y + WNODE[w][i][1] ) * 3;
}

/* trafo_mat_cartesian_to_normal_tangential
 * (linalg/trafo/local_basis_trafo_normal_tangential.hpp:36-73): rows n, t1, t2 */
static void trafo_nt( const double nin[3], double R[3][3] )
{
    double n[3] = { nin[0], nin[1], nin[2] };
    normalize3( n );
    const double ax = fabs( n[0] ), ay = fabs( n[1] ), az = fabs( n[2] );
    double       ref[3] = { 0, 0, 0 };
    if ( ax <= ay && ax <= az )
        ref[0] = 1;
    else if ( ay <= ax && ay <= az )
        ref[1] = 1;
    else
        ref[2] = 1;
    double t1[3] = { ref[1] * n[2] - ref[2] * n[1], ref[2] * n[0] - ref[0] * n[2], ref[0] * n[1] - ref[1] * n[0] };
    normalize3( t1 );
    if ( sqrt( t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2] ) < 1e-15 )
    {
        t1[0] = n[1], t1[1] = -n[0], t1[2] = 0;
        normalize3( t1 );
    }
    double t2[3] = { n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0] };
    normalize3( t2 );
    for ( int k = 0; k < 3; ++k )
        R[0][k] = n[k], R[1][k] = t1[k], R[2][k] = t2[k];
}

/* ------------------------------------------------------------------------ */
/* EpsilonDivDivKerngen (fe/wedge/operators/shell/epsilon_divdiv_kerngen.hpp) */
/* ------------------------------------------------------------------------ */

/* One-point (centroid) quadrature of the wedge: physical gradients g[6][3]
 * and kwJ = mean nodal k * |det J| (kerngen :1189-1259). */
static void kerngen_wedge_geometry( const double* p[3], double r0, double r1, const double kn[6], double g[6][3],
                                    double* kwJ )
{
    double J[3][3], IT[3][3];
    wedge_jac( p, r0, r1, 1.0 / 3.0, 1.0 / 3.0, 0.0, J );
    const double det = det3( J );
    inv_transposed3( J, det, IT );
    double ks = 0.0;
    for ( int n = 0; n < 6; ++n )
        ks += kn[n];
    *kwJ = ( ks / 6.0 ) * fabs( det );
    for ( int n = 0; n < 6; ++n )
    {
        double gr[3];
        grad_shape_ref( n, 1.0 / 3.0, 1.0 / 3.0, 0.0, gr );
        for ( int a = 0; a < 3; ++a )
            g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
    }
}

static void fs_project( const double n[3], double v[3] )
{
    const double dt = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
    for ( int k = 0; k < 3; ++k )
        v[k] -= dt * n[k];
}

/* Penalty null modes for free-slip on both boundaries (kerngen :287-408):
 * m_i = tangential part of (e_i x x) on boundary nodes, Gram-Schmidt
 * orthonormalised with owned-masked dot products. modes: [3][3*ns]. */
static void kerngen_null_modes( int L, const double* coords, const double* radii, const uint8_t* omask, double* modes )
{
    const int    n1 = ( 1 << L ) + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    for ( int ax = 0; ax < 3; ++ax )
    {
        double* m = modes + (size_t) ax * 3 * ns;
        for ( int d = 0; d < NDIAMOND; ++d )
            for ( int x = 0; x < n1; ++x )
                for ( int y = 0; y < n1; ++y )
                    for ( int r = 0; r < n1; ++r )
                    {
                        const size_t  i  = node_idx( n1, d, x, y, r );
                        const double* u  = coords + lat_idx( n1, d, x, y ) * 3;
                        const double  rr = radii[d * n1 + r];
                        double        c[3] = { u[0] * rr, u[1] * rr, u[2] * rr };
                        double        v[3] = { 0, 0, 0 };
                        const int     a1 = ( ax + 1 ) % 3, a2 = ( ax + 2 ) % 3;
                        v[a1]              = c[a2];
                        v[a2]              = -c[a1];
                        if ( r == 0 || r == n1 - 1 )
                        {
                            double n[3] = { u[0], u[1], u[2] };
                            normalize3( n );
                            fs_project( n, v );
                        }
                        for ( int k = 0; k < 3; ++k )
                            m[k * ns + i] = v[k];
                    }
    }
    for ( int i = 0; i < 3; ++i )
    {
        double* mi = modes + (size_t) i * 3 * ns;
        for ( int j = 0; j < i; ++j )
        {
            double* mj = modes + (size_t) j * 3 * ns;
            double  dt = 0.0;
            for ( int k = 0; k < 3; ++k )
                dt += or_masked_dot( ns, mi + k * ns, mj + k * ns, omask );
            for ( size_t t = 0; t < 3 * ns; ++t )
                mi[t] -= dt * mj[t];
        }
        double nn = 0.0;
        for ( int k = 0; k < 3; ++k )
            nn += or_masked_dot( ns, mi + k * ns, mi + k * ns, omask );
        const double inv = 1.0 / sqrt( nn );
        for ( size_t t = 0; t < 3 * ns; ++t )
            mi[t] *= inv;
    }
}

/* Matrix-free apply of the production viscous operator
 *   a(u, v) = int k (2 eps(u):eps(v) - 2/3 div u div v)
 * with one-point quadrature, restating the fast Dirichlet/Neumann path
 * (kerngen :1055-1389), the fast free-slip path (:1421-1940) and the fs/fs
 * penalty (:585-606) followed by the additive halo (:611-616).  Replace mode. */
static void kerngen_apply( int L, const double* coords, const double* radii, const double* k, const double* src,
                           double* dst, int bc_cmb, int bc_surf, int diag, int halo );
void or_kerngen_apply( int L, const double* coords, const double* radii, const double* k, const double* src,
                       double* dst, int bc_cmb, int bc_surf, int diag )
{
    kerngen_apply( L, coords, radii, k, src, dst, bc_cmb, bc_surf, diag, 1 );
}
/* the same without the closing halo sum: every diamond's copy of a node holds that diamond's cells' contributions
 * (the copy-wise result of the reference's apply with OperatorCommunicationMode::SkipCommunication) */
void or_kerngen_apply_copywise( int L, const double* coords, const double* radii, const double* k, const double* src,
                                double* dst, int bc_cmb, int bc_surf, int diag )
{
    kerngen_apply( L, coords, radii, k, src, dst, bc_cmb, bc_surf, diag, 0 );
}
static void kerngen_apply( int L, const double* coords, const double* radii, const double* k, const double* src,
                           double* dst, int bc_cmb, int bc_surf, int diag, int halo )
{
    const int    N = 1 << L, n1 = N + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    memset( dst, 0, sizeof( double ) * 3 * ns );

    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                {
                    const int at_cmb = r == 0, at_surf = r == N - 1;
                    const int cmb_dir = at_cmb && bc_cmb == 1, surf_dir = at_surf && bc_surf == 1;
                    const int cmb_fs = at_cmb && bc_cmb == 2, surf_fs = at_surf && bc_surf == 2;
                    /* node of cell-corner (dx,dy,dr) -> 8-slot accumulator */
                    double acc[2][2][2][3];
                    double ann[2][2][2];
                    memset( acc, 0, sizeof( acc ) );
                    memset( ann, 0, sizeof( ann ) );
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        double kn[6], s[6][3], sp[6][3], nrm[6][3];
                        for ( int n = 0; n < 6; ++n )
                        {
                            const int    X = x + WNODE[w][n][0], Y = y + WNODE[w][n][1], Rr = r + WNODE[w][n][2];
                            const size_t i = node_idx( n1, d, X, Y, Rr );
                            kn[n]          = k[i];
                            for ( int c = 0; c < 3; ++c )
                                s[n][c] = sp[n][c] = src[c * ns + i];
                            const double* u = coords + lat_idx( n1, d, X, Y ) * 3;
                            nrm[n][0] = u[0], nrm[n][1] = u[1], nrm[n][2] = u[2];
                            normalize3( nrm[n] );
                            if ( ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 ) )
                                fs_project( nrm[n], sp[n] );
                        }
                        double g[6][3], kwJ;
                        kerngen_wedge_geometry( p, radii[d * n1 + r], radii[d * n1 + r + 1], kn, g, &kwJ );
                        /* Dirichlet boundary nodes drop out of gather and scatter (matvec only) */
                        int active[6];
                        for ( int n = 0; n < 6; ++n )
                            active[n] = diag ? 1 : !( ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 ) );
                        if ( !diag )
                        {
                            double G[3][3] = { { 0 } }, div = 0.0;
                            for ( int n = 0; n < 6; ++n )
                                if ( active[n] )
                                    for ( int a = 0; a < 3; ++a )
                                        for ( int b = 0; b < 3; ++b )
                                            G[a][b] += g[n][a] * sp[n][b]; /* G[a][b] = sum g_a u_b */
                            div = G[0][0] + G[1][1] + G[2][2];
                            double E[3][3];
                            for ( int a = 0; a < 3; ++a )
                                for ( int b = 0; b < 3; ++b )
                                    E[a][b] = 0.5 * ( G[a][b] + G[b][a] );
                            for ( int n = 0; n < 6; ++n )
                            {
                                if ( !active[n] )
                                    continue;
                                double* o = acc[WNODE[w][n][0]][WNODE[w][n][1]][WNODE[w][n][2]];
                                for ( int c = 0; c < 3; ++c )
                                    o[c] += kwJ * ( 2.0 * ( g[n][0] * E[0][c] + g[n][1] * E[1][c] + g[n][2] * E[2][c] ) -
                                                    ( 2.0 / 3.0 ) * g[n][c] * div );
                                if ( ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 ) )
                                {
                                    const double gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
                                    const double ng = nrm[n][0] * g[n][0] + nrm[n][1] * g[n][1] + nrm[n][2] * g[n][2];
                                    ann[WNODE[w][n][0]][WNODE[w][n][1]][WNODE[w][n][2]] += kwJ * ( gg + ng * ng / 3.0 );
                                }
                            }
                        }
                        /* diagonal blocks: all nodes in diagonal mode, Dirichlet nodes in matvec mode */
                        for ( int n = 0; n < 6; ++n )
                        {
                            const int is_dir = ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 );
                            const int is_fs  = ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 );
                            if ( !( diag || is_dir ) )
                                continue;
                            double*      o  = acc[WNODE[w][n][0]][WNODE[w][n][1]][WNODE[w][n][2]];
                            const double gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
                            if ( diag && is_fs )
                            {
                                /* R^T diag(R A_nn R^T) R s, A_nn = kwJ (|g|^2 I + g g^T / 3) */
                                double R[3][3], Rg[3], Rs[3], v[3];
                                trafo_nt( nrm[n], R );
                                for ( int a = 0; a < 3; ++a )
                                {
                                    Rg[a] = R[a][0] * g[n][0] + R[a][1] * g[n][1] + R[a][2] * g[n][2];
                                    Rs[a] = R[a][0] * s[n][0] + R[a][1] * s[n][1] + R[a][2] * s[n][2];
                                    v[a]  = kwJ * ( gg + Rg[a] * Rg[a] / 3.0 ) * Rs[a];
                                }
                                for ( int c = 0; c < 3; ++c )
                                    o[c] += R[0][c] * v[0] + R[1][c] * v[1] + R[2][c] * v[2];
                            }
                            else
                            {
                                for ( int c = 0; c < 3; ++c )
                                    o[c] += kwJ * s[n][c] * ( gg + g[n][c] * g[n][c] / 3.0 );
                            }
                        }
                    }
                    /* free-slip: test-side projection + normal-normal add back (:1880-1935) */
                    if ( !diag && ( cmb_fs || surf_fs ) )
                    {
                        const int dr = cmb_fs ? 0 : 1;
                        for ( int dx = 0; dx < 2; ++dx )
                            for ( int dy = 0; dy < 2; ++dy )
                            {
                                const size_t  i   = node_idx( n1, d, x + dx, y + dy, r + dr );
                                const double* u   = coords + lat_idx( n1, d, x + dx, y + dy ) * 3;
                                double        n[3] = { u[0], u[1], u[2] };
                                normalize3( n );
                                double* o = acc[dx][dy][dr];
                                fs_project( n, o );
                                const double un = n[0] * src[i] + n[1] * src[ns + i] + n[2] * src[2 * ns + i];
                                for ( int c = 0; c < 3; ++c )
                                    o[c] += ann[dx][dy][dr] * un * n[c];
                            }
                    }
                    for ( int dx = 0; dx < 2; ++dx )
                        for ( int dy = 0; dy < 2; ++dy )
                            for ( int dr = 0; dr < 2; ++dr )
                            {
                                const size_t i = node_idx( n1, d, x + dx, y + dy, r + dr );
                                for ( int c = 0; c < 3; ++c )
                                    dst[c * ns + i] += acc[dx][dy][dr][c];
                            }
                }

    if ( !diag && bc_cmb == 2 && bc_surf == 2 )
    {
        /* dst += eps * sum_i (m_i^T src)_owned m_i on every stored node, eps = 1 */
        uint8_t* om    = (uint8_t*) malloc( ns );
        double*  modes = (double*) malloc( sizeof( double ) * 9 * ns );
        or_ownership_mask( L, coords, om );
        kerngen_null_modes( L, coords, radii, om, modes );
        for ( int i = 0; i < 3; ++i )
        {
            const double* m  = modes + (size_t) i * 3 * ns;
            double        al = 0.0;
            for ( int c = 0; c < 3; ++c )
                al += or_masked_dot( ns, m + c * ns, src + c * ns, om );
            for ( size_t t = 0; t < 3 * ns; ++t )
                dst[t] += al * m[t];
        }
        free( modes );
        free( om );
    }
    if ( halo )
        or_halo_sum( L, coords, dst, 3 );
}

/* ------------------------------------------------------------------------ */
/* Stored local matrices and GCA coarse operators                            */
/* ------------------------------------------------------------------------ */

static int    linear_stencil( int Nf, const double* coords_f, const double* radii_f, int d, int x, int y, int r,
                              int cx[4], int cy[4], int cr[4], double w[4] );
static double prolong_weight( int xf, int yf, int rf, int xc, int yc, int rc );

/* kerngen assemble_local_matrix (epsilon_divdiv_kerngen.hpp:2051-2110): the
 * wedge's 18x18 matrix in DIMENSIONWISE order (node + 6 dim), one-point rule,
 * no boundary treatment:
 * A[i+6a][j+6b] = kwJ (2 sym(g_j e_b):sym(g_i e_a) - 2/3 g_{j,b} g_{i,a}) */
static void kerngen_local_matrix( const double* p[3], double r0, double r1, const double kn[6], double A[18][18] )
{
    double g[6][3], kwJ;
    kerngen_wedge_geometry( p, r0, r1, kn, g, &kwJ );
    for ( int a = 0; a < 3; ++a )
        for ( int b = 0; b < 3; ++b )
            for ( int i = 0; i < 6; ++i )
                for ( int j = 0; j < 6; ++j )
                {
                    const double gg = a == b ? g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2] : 0.0;
                    A[i + 6 * a][j + 6 * b] = kwJ * ( gg + g[i][b] * g[j][a] - 2.0 / 3.0 * g[j][b] * g[i][a] );
                }
}

void or_kerngen_local_matrices( int L, const double* coords, const double* radii, const double* k, double* mats )
{
    const int N = 1 << L, n1 = N + 1;
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        double kn[6];
                        for ( int n = 0; n < 6; ++n )
                            kn[n] = k[node_idx( n1, d, x + WNODE[w][n][0], y + WNODE[w][n][1], r + WNODE[w][n][2] )];
                        double A[18][18];
                        kerngen_local_matrix( p, radii[d * n1 + r], radii[d * n1 + r + 1], kn, A );
                        const size_t cell = ( ( (size_t) d * N + x ) * N + y ) * N + r;
                        memcpy( mats + ( cell * 2 + w ) * 324, A, sizeof( A ) );
                    }
}

/* TwoGridGCA (linalg/solvers/gca/gca.hpp:154-528): per coarse cell, sum over
 * its 8 fine hexes x 2 wedges of P^T A_fine P with the 6x6 local interpolation
 * P (columns = local nodes of the coarse wedge the fine wedge lies in),
 * constant (mode 0, the default) or linear (mode 1) weights. */
static void gca_local_P( int Nf, const double* coords_f, const double* radii_f, int d, int xh, int yh, int rh, int w,
                         int mode, double P[6][6] )
{
    const int n1 = Nf + 1;
    memset( P, 0, sizeof( double ) * 36 );
    for ( int i = 0; i < 6; ++i )
    {
        const int x = xh + WNODE[w][i][0], y = yh + WNODE[w][i][1], r = rh + WNODE[w][i][2];
        if ( x % 2 == 0 && y % 2 == 0 && r % 2 == 0 )
        {
            P[i][i] = 1.0;
            continue;
        }
        const int rb = r < n1 - 1 ? r / 2 : r / 2 - 1, rt = rb + 1;
        int       cx[4], cy[4], cr[4];
        double    wl[4];
        if ( x % 2 == 0 && y % 2 == 0 )
        {
            double w0 = 0.5, w1 = 0.5;
            if ( mode == 1 )
            {
                linear_stencil( Nf, coords_f, radii_f, d, x, y, r, cx, cy, cr, wl );
                w0 = wl[0], w1 = wl[1];
            }
            const int col = i % 3;
            P[i][col]     = w0;
            P[i][col + 3] = w1;
            continue;
        }
        int x0, x1, y0, y1, li[4];
        if ( x % 2 == 0 )
        {
            x0 = x1 = x / 2, y0 = y / 2, y1 = y / 2 + 1;
            li[0] = 0, li[1] = 2, li[2] = 3, li[3] = 5;
        }
        else if ( y % 2 == 0 )
        {
            x0 = x / 2, x1 = x / 2 + 1, y0 = y1 = y / 2;
            li[0] = 0, li[1] = 1, li[2] = 3, li[3] = 4;
        }
        else
        {
            x0 = x / 2 + 1, x1 = x / 2, y0 = y / 2, y1 = y / 2 + 1;
            li[0] = 1, li[1] = 2, li[2] = 4, li[3] = 5;
        }
        if ( mode == 1 )
        {
            linear_stencil( Nf, coords_f, radii_f, d, x, y, r, cx, cy, cr, wl );
            P[i][li[0]] = wl[0], P[i][li[1]] = wl[0], P[i][li[2]] = wl[2], P[i][li[3]] = wl[2];
        }
        else
        {
            P[i][li[0]] = prolong_weight( x, y, r, x0, y0, rb );
            P[i][li[1]] = prolong_weight( x, y, r, x1, y1, rb );
            P[i][li[2]] = prolong_weight( x, y, r, x0, y0, rt );
            P[i][li[3]] = prolong_weight( x, y, r, x1, y1, rt );
        }
    }
}

/* coarse wedge (0 or 1) holding fine wedge w of fine hex h (gca.hpp:434-452) */
static int gca_coarse_wedge( int h, int w )
{
    if ( ( w == 0 && ( h == 0 || h == 1 || h == 2 || h == 4 || h == 5 || h == 6 ) ) || ( w == 1 && ( h == 0 || h == 4 ) ) )
        return 0;
    return 1;
}

void or_gca_coarsen( int Lf, const double* coords_f, const double* radii_f, const double* k_fine,
                     const double* mats_fine, int mode, double* mats_coarse )
{
    const int Nf = 1 << Lf, Nc = Nf / 2, n1 = Nf + 1;
    static const int HS[8][3] = { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 1, 1, 0 },
                                  { 0, 0, 1 }, { 1, 0, 1 }, { 0, 1, 1 }, { 1, 1, 1 } };
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int xc = 0; xc < Nc; ++xc )
            for ( int yc = 0; yc < Nc; ++yc )
                for ( int rc = 0; rc < Nc; ++rc )
                {
                    double Ac[2][18][18];
                    memset( Ac, 0, sizeof( Ac ) );
                    for ( int h = 0; h < 8; ++h )
                        for ( int w = 0; w < 2; ++w )
                        {
                            const int xh = 2 * xc + HS[h][0], yh = 2 * yc + HS[h][1], rh = 2 * rc + HS[h][2];
                            double    P[6][6], A[18][18];
                            gca_local_P( Nf, coords_f, radii_f, d, xh, yh, rh, w, mode, P );
                            if ( mats_fine )
                            {
                                const size_t cell = ( ( (size_t) d * Nf + xh ) * Nf + yh ) * Nf + rh;
                                memcpy( A, mats_fine + ( cell * 2 + w ) * 324, sizeof( A ) );
                            }
                            else
                            {
                                const double* p[3];
                                wedge_lateral_points( n1, coords_f, d, xh, yh, w, p );
                                double kn[6];
                                for ( int n = 0; n < 6; ++n )
                                    kn[n] = k_fine[node_idx( n1, d, xh + WNODE[w][n][0], yh + WNODE[w][n][1],
                                                             rh + WNODE[w][n][2] )];
                                kerngen_local_matrix( p, radii_f[d * n1 + rh], radii_f[d * n1 + rh + 1], kn, A );
                            }
                            const int cw = gca_coarse_wedge( h, w );
                            /* P_vec = blockdiag(P, P, P) in DIMENSIONWISE order */
                            for ( int a = 0; a < 3; ++a )
                                for ( int b = 0; b < 3; ++b )
                                    for ( int i = 0; i < 6; ++i )
                                        for ( int j = 0; j < 6; ++j )
                                        {
                                            double v = 0.0;
                                            for ( int m = 0; m < 6; ++m )
                                                for ( int n = 0; n < 6; ++n )
                                                    v += P[m][i] * A[m + 6 * a][n + 6 * b] * P[n][j];
                                            Ac[cw][i + 6 * a][j + 6 * b] += v;
                                        }
                        }
                    const size_t cell = ( ( (size_t) d * Nc + xc ) * Nc + yc ) * Nc + rc;
                    memcpy( mats_coarse + cell * 2 * 324, Ac, sizeof( Ac ) );
                }
}

/* kerngen slow path with stored matrices (epsilon_divdiv_kerngen.hpp:823-1052):
 * Dirichlet cells mask the boundary nodes' couplings (keeping the node's own
 * same-dimension diagonal); free-slip cells rotate the boundary nodes to the
 * (n, t1, t2) basis, decouple the normal component keeping its diagonal and
 * rotate back; diag keeps the diagonal of the treated matrix; fs/fs adds the
 * rigid-rotation penalty; additive halo. */
void or_stored_apply( int L, const double* coords, const double* radii, const double* mats, const double* src,
                      double* dst, int bc_cmb, int bc_surf, int diag )
{
    const int    N = 1 << L, n1 = N + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    memset( dst, 0, sizeof( double ) * 3 * ns );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                {
                    const int at_cmb = r == 0, at_surf = r == N - 1;
                    int       bcf = 0;
                    if ( at_cmb || at_surf )
                        bcf = at_cmb ? bc_cmb : bc_surf;
                    for ( int w = 0; w < 2; ++w )
                    {
                        const size_t cell = ( ( (size_t) d * N + x ) * N + y ) * N + r;
                        double       A[18][18], M[18][18], s[18], out[18];
                        memcpy( A, mats + ( cell * 2 + w ) * 324, sizeof( A ) );
                        size_t idx[6];
                        for ( int n = 0; n < 6; ++n )
                        {
                            idx[n] = node_idx( n1, d, x + WNODE[w][n][0], y + WNODE[w][n][1], r + WNODE[w][n][2] );
                            for ( int a = 0; a < 3; ++a )
                                s[n + 6 * a] = src[a * ns + idx[n]];
                        }
                        if ( bcf == 2 )
                        {
                            /* NODEWISE order (3 node + dim), rotate the 3 boundary nodes */
                            double R[18][18], An[18][18], sn[18], T[18][18];
                            memset( R, 0, sizeof( R ) );
                            for ( int i = 0; i < 18; ++i )
                                R[i][i] = 1.0;
                            for ( int i = 0; i < 6; ++i )
                                for ( int a = 0; a < 3; ++a )
                                {
                                    sn[3 * i + a] = s[i + 6 * a];
                                    for ( int j = 0; j < 6; ++j )
                                        for ( int b = 0; b < 3; ++b )
                                            An[3 * i + a][3 * j + b] = A[i + 6 * a][j + 6 * b];
                                }
                            const int off = at_cmb ? 0 : 3;
                            for ( int bn = 0; bn < 3; ++bn )
                            {
                                const int     node = off + bn;
                                const double* c    = coords + lat_idx( n1, d, x + WNODE[w][node][0], y + WNODE[w][node][1] ) * 3;
                                const double  rad  = radii[d * n1 + r + ( at_cmb ? 0 : 1 )];
                                double        nv[3] = { c[0] * rad, c[1] * rad, c[2] * rad }, Ri[3][3];
                                trafo_nt( nv, Ri );
                                for ( int a = 0; a < 3; ++a )
                                    for ( int b = 0; b < 3; ++b )
                                        R[3 * node + a][3 * node + b] = Ri[a][b];
                            }
                            /* An <- R An R^T, sn <- R sn */
                            for ( int i = 0; i < 18; ++i )
                                for ( int j = 0; j < 18; ++j )
                                {
                                    double v = 0.0;
                                    for ( int m = 0; m < 18; ++m )
                                        v += An[i][m] * R[j][m];
                                    T[i][j] = v;
                                }
                            for ( int i = 0; i < 18; ++i )
                                for ( int j = 0; j < 18; ++j )
                                {
                                    double v = 0.0;
                                    for ( int m = 0; m < 18; ++m )
                                        v += R[i][m] * T[m][j];
                                    An[i][j] = v;
                                }
                            double sr[18];
                            for ( int i = 0; i < 18; ++i )
                            {
                                double v = 0.0;
                                for ( int m = 0; m < 18; ++m )
                                    v += R[i][m] * sn[m];
                                sr[i] = v;
                            }
                            /* decouple the normal components (row/col 3 node), keep the diagonal */
                            for ( int bn = 0; bn < 3; ++bn )
                            {
                                const int q = 3 * ( off + bn );
                                for ( int k = 0; k < 18; ++k )
                                    if ( k != q )
                                        An[q][k] = An[k][q] = 0.0;
                            }
                            double yr[18];
                            for ( int i = 0; i < 18; ++i )
                            {
                                double v = 0.0;
                                if ( diag )
                                    v = An[i][i] * sr[i];
                                else
                                    for ( int m = 0; m < 18; ++m )
                                        v += An[i][m] * sr[m];
                                yr[i] = v;
                            }
                            for ( int i = 0; i < 18; ++i )
                            {
                                double v = 0.0;
                                for ( int m = 0; m < 18; ++m )
                                    v += R[m][i] * yr[m];
                                out[( i / 3 ) + 6 * ( i % 3 )] = v;
                            }
                        }
                        else
                        {
                            for ( int a = 0; a < 3; ++a )
                                for ( int b = 0; b < 3; ++b )
                                    for ( int i = 0; i < 6; ++i )
                                        for ( int j = 0; j < 6; ++j )
                                        {
                                            int keep = 1;
                                            if ( bcf == 1 )
                                            {
                                                const int bi = at_cmb ? i < 3 : i >= 3, bj = at_cmb ? j < 3 : j >= 3;
                                                if ( a == b ? ( i != j && ( bi || bj ) ) : ( bi || bj ) )
                                                    keep = 0;
                                            }
                                            M[i + 6 * a][j + 6 * b] = keep ? A[i + 6 * a][j + 6 * b] : 0.0;
                                        }
                            for ( int i = 0; i < 18; ++i )
                            {
                                double v = 0.0;
                                if ( diag )
                                    v = M[i][i] * s[i];
                                else
                                    for ( int m = 0; m < 18; ++m )
                                        v += M[i][m] * s[m];
                                out[i] = v;
                            }
                        }
                        for ( int n = 0; n < 6; ++n )
                            for ( int a = 0; a < 3; ++a )
                                dst[a * ns + idx[n]] += out[n + 6 * a];
                    }
                }
    if ( !diag && bc_cmb == 2 && bc_surf == 2 )
    {
        uint8_t* om    = (uint8_t*) malloc( ns );
        double*  modes = (double*) malloc( sizeof( double ) * 9 * ns );
        or_ownership_mask( L, coords, om );
        kerngen_null_modes( L, coords, radii, om, modes );
        for ( int i = 0; i < 3; ++i )
        {
            const double* m  = modes + (size_t) i * 3 * ns;
            double        al = 0.0;
            for ( int c = 0; c < 3; ++c )
                al += or_masked_dot( ns, m + c * ns, src + c * ns, om );
            for ( size_t t = 0; t < 3 * ns; ++t )
                dst[t] += al * m[t];
        }
        free( modes );
        free( om );
    }
    or_halo_sum( L, coords, dst, 3 );
}

/* ------------------------------------------------------------------------ */
/* Laplace (fe/wedge/operators/shell/laplace.hpp:106-330), 3x2 Felippa rule  */
/* ------------------------------------------------------------------------ */

static const double QP32[6][3] = { { 0.6666666666666666, 0.1666666666666667, -0.5773502691896257 },
                                   { 0.1666666666666667, 0.6666666666666666, -0.5773502691896257 },
                                   { 0.1666666666666667, 0.1666666666666667, -0.5773502691896257 },
                                   { 0.6666666666666666, 0.1666666666666667, 0.5773502691896257 },
                                   { 0.1666666666666667, 0.6666666666666666, 0.5773502691896257 },
                                   { 0.1666666666666667, 0.1666666666666667, 0.5773502691896257 } };
static const double QW32       = 0.1666666666666667;

void or_laplace_apply( int L, const double* coords, const double* radii, const double* src, double* dst,
                       int treat_boundary, int diag )
{
    const int    N = 1 << L, n1 = N + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    memset( dst, 0, sizeof( double ) * ns );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                {
                    /* bottom check wins when a cell touches both (laplace.hpp:140-168) */
                    const int bot = treat_boundary && r == 0;
                    const int top = treat_boundary && !bot && r == N - 1;
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        size_t idx[6];
                        double s[6], out[6] = { 0 };
                        for ( int n = 0; n < 6; ++n )
                        {
                            idx[n] = node_idx( n1, d, x + WNODE[w][n][0], y + WNODE[w][n][1], r + WNODE[w][n][2] );
                            s[n]   = src[idx[n]];
                        }
                        for ( int q = 0; q < 6; ++q )
                        {
                            double J[3][3], IT[3][3], g[6][3];
                            wedge_jac( p, radii[d * n1 + r], radii[d * n1 + r + 1], QP32[q][0], QP32[q][1], QP32[q][2], J );
                            const double det = det3( J );
                            inv_transposed3( J, det, IT );
                            for ( int n = 0; n < 6; ++n )
                            {
                                double gr[3];
                                grad_shape_ref( n, QP32[q][0], QP32[q][1], QP32[q][2], gr );
                                for ( int a = 0; a < 3; ++a )
                                    g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
                            }
                            const double wdet = QW32 * fabs( det );
                            /* coupled node set: all, or the side away from the Dirichlet boundary */
                            int lo = 0, hi = 6;
                            if ( bot )
                                lo = 3;
                            if ( top )
                                hi = 3;
                            if ( diag )
                                lo = 6, hi = 6;
                            double gu[3] = { 0, 0, 0 };
                            for ( int n = lo; n < hi; ++n )
                                for ( int a = 0; a < 3; ++a )
                                    gu[a] += s[n] * g[n][a];
                            for ( int n = lo; n < hi; ++n )
                                out[n] += wdet * ( g[n][0] * gu[0] + g[n][1] * gu[1] + g[n][2] * gu[2] );
                            for ( int n = 0; n < 6; ++n )
                            {
                                const int dg = diag || ( bot && n < 3 ) || ( top && n >= 3 );
                                if ( dg )
                                    out[n] += wdet * s[n] * ( g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2] );
                            }
                        }
                        for ( int n = 0; n < 6; ++n )
                            dst[idx[n]] += out[n];
                    }
                }
    or_halo_sum( L, coords, dst, 1 );
}

/* ------------------------------------------------------------------------ */
/* DivKGrad (div_k_grad.hpp:219-572) and VectorLaplace                       */
/* (vector_laplace.hpp:131-420): the Laplace form, with k interpolated by    */
/* the wedge shape functions at every quadrature point (DivKGrad) or applied */
/* to each of three components (VectorLaplace).  Per cell one of four       */
/* couplings: all nodes (NEU), boundary nodes of the CMB side (BOT) or of the */
/* SURFACE side (TOP) decoupled keeping their diagonal, or diagonal only.    */
/* ------------------------------------------------------------------------ */

enum { GM_NEU = 0, GM_BOT = 1, GM_TOP = 2, GM_DIAG = 3 };

static double shape_ref( int n, double xi, double eta, double zeta )
{
    /* integrands.hpp:86-159: lateral P1 times radial linear */
    const double lat = n % 3 == 0 ? 1 - xi - eta : ( n % 3 == 1 ? xi : eta );
    return lat * ( n < 3 ? 0.5 * ( 1 - zeta ) : 0.5 * ( 1 + zeta ) );
}

static void grad_family_apply( int L, const double* coords, const double* radii, const double* k, int ncomp,
                               const double* src, double* dst, const int* cell_mode_of_r, int single )
{
    const int    N = 1 << L, n1 = N + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    memset( dst, 0, sizeof( double ) * ns * ncomp );
    const int nq = single ? 1 : 6;
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                {
                    const int mode = cell_mode_of_r[r];
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        size_t idx[6];
                        double s[3][6], kv[6], out[3][6];
                        memset( out, 0, sizeof( out ) );
                        for ( int n = 0; n < 6; ++n )
                        {
                            idx[n] = node_idx( n1, d, x + WNODE[w][n][0], y + WNODE[w][n][1], r + WNODE[w][n][2] );
                            for ( int c = 0; c < ncomp; ++c )
                                s[c][n] = src[c * ns + idx[n]];
                            kv[n] = k ? k[idx[n]] : 1.0;
                        }
                        for ( int q = 0; q < nq; ++q )
                        {
                            /* quad_felippa_1x1: (1/3, 1/3, 0), weight 1 (quadrature.hpp:32-46) */
                            const double xi   = single ? 1.0 / 3.0 : QP32[q][0];
                            const double eta  = single ? 1.0 / 3.0 : QP32[q][1];
                            const double zeta = single ? 0.0 : QP32[q][2];
                            const double wq   = single ? 1.0 : QW32;
                            double       J[3][3], IT[3][3], g[6][3];
                            wedge_jac( p, radii[d * n1 + r], radii[d * n1 + r + 1], xi, eta, zeta, J );
                            const double det = det3( J );
                            inv_transposed3( J, det, IT );
                            for ( int n = 0; n < 6; ++n )
                            {
                                double gr[3];
                                grad_shape_ref( n, xi, eta, zeta, gr );
                                for ( int a = 0; a < 3; ++a )
                                    g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
                            }
                            double wdet = wq * fabs( det );
                            if ( k )
                            {
                                double ke = 0.0;
                                for ( int n = 0; n < 6; ++n )
                                    ke += shape_ref( n, xi, eta, zeta ) * kv[n];
                                wdet *= ke;
                            }
                            int lo = 0, hi = 6;
                            if ( mode == GM_BOT )
                                lo = 3;
                            if ( mode == GM_TOP )
                                hi = 3;
                            if ( mode == GM_DIAG )
                                lo = hi = 6;
                            for ( int c = 0; c < ncomp; ++c )
                            {
                                double gu[3] = { 0, 0, 0 };
                                for ( int n = lo; n < hi; ++n )
                                    for ( int a = 0; a < 3; ++a )
                                        gu[a] += s[c][n] * g[n][a];
                                for ( int n = lo; n < hi; ++n )
                                    out[c][n] += wdet * ( g[n][0] * gu[0] + g[n][1] * gu[1] + g[n][2] * gu[2] );
                                for ( int n = 0; n < 6; ++n )
                                {
                                    const int dg = mode == GM_DIAG || ( mode == GM_BOT && n < 3 ) ||
                                                   ( mode == GM_TOP && n >= 3 );
                                    if ( dg )
                                        out[c][n] += wdet * s[c][n] *
                                                     ( g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2] );
                                }
                            }
                        }
                        for ( int c = 0; c < ncomp; ++c )
                            for ( int n = 0; n < 6; ++n )
                                dst[c * ns + idx[n]] += out[c][n];
                    }
                }
    or_halo_sum( L, coords, dst, ncomp );
}

void or_divkgrad_apply( int L, const double* coords, const double* radii, const double* k, const double* src,
                        double* dst, int treat_boundary, int diag, int single_quadpoint )
{
    /* coupling per cell: div_k_grad.hpp:455-512 (the CMB check wins; diagonal
     * mode couples nothing and keeps every node's diagonal) */
    const int N = 1 << L;
    int*      mode = (int*) malloc( sizeof( int ) * N );
    for ( int r = 0; r < N; ++r )
    {
        const int bot = treat_boundary && r == 0;
        const int top = treat_boundary && !bot && r == N - 1;
        mode[r]       = diag ? GM_DIAG : ( bot ? GM_BOT : ( top ? GM_TOP : GM_NEU ) );
    }
    grad_family_apply( L, coords, radii, k, 1, src, dst, mode, single_quadpoint );
    free( mode );
}

int or_vector_laplace_apply( int L, const double* coords, const double* radii, const double* src, double* dst,
                             int bc_cmb, int bc_surf, int diag )
{
    /* vector_laplace.hpp:181-210: the branch follows the boundary flag of the
     * cell's own (x, y, r) node: CMB for r = 0, otherwise SURFACE, so a
     * Dirichlet surface selects the top-boundary coupling for every cell
     * above the first layer.  Only Neumann and Dirichlet are accepted. */
    const int N = 1 << L;
    if ( ( bc_cmb != 0 && bc_cmb != 1 ) || ( bc_surf != 0 && bc_surf != 1 ) )
        return -1;
    int* mode = (int*) malloc( sizeof( int ) * N );
    for ( int r = 0; r < N; ++r )
    {
        const int bc = r == 0 ? bc_cmb : bc_surf;
        mode[r]      = diag ? GM_DIAG : ( bc == 1 ? ( r == 0 ? GM_BOT : GM_TOP ) : GM_NEU );
    }
    grad_family_apply( L, coords, radii, NULL, 3, src, dst, mode, 0 );
    free( mode );
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Stokes coupling blocks: Divergence (divergence.hpp:118-322) and Gradient  */
/* (gradient.hpp:115-325).  Fine (level L) P1 velocity against coarse        */
/* (level L-1) P1 pressure shape functions evaluated on the fine wedges      */
/* (shape_coarse, integrands.hpp:266-400), 3x2 Felippa rule.                 */
/* ------------------------------------------------------------------------ */

/* coarse lateral shape value: coefficient table [node%3][fine lateral idx] = (a, b_xi, c_eta) */
static const double COARSE_LAT[3][4][3] = {
    { { 1.0, -0.5, -0.5 }, { 0.5, -0.5, -0.5 }, { 0.5, -0.5, -0.5 }, { 0.0, 0.5, 0.5 } },
    { { 0.0, 0.5, 0.0 }, { 0.5, 0.5, 0.0 }, { 0.0, 0.5, 0.0 }, { 0.5, -0.5, 0.0 } },
    { { 0.0, 0.0, 0.5 }, { 0.0, 0.0, 0.5 }, { 0.5, 0.0, 0.5 }, { 0.5, 0.0, -0.5 } } };

static double shape_coarse( int i, int frad, int flat, double xi, double eta, double zeta )
{
    const double* c   = COARSE_LAT[i % 3][flat];
    const double  lat = c[0] + c[1] * xi + c[2] * eta;
    double        rad;
    if ( i / 3 == 0 )
        rad = frad == 0 ? 0.25 * ( 3 - zeta ) : 0.25 * ( 1 - zeta );
    else
        rad = frad == 0 ? 0.25 * ( 1 + zeta ) : 0.25 * ( 3 + zeta );
    return lat * rad;
}

/* fine_lateral_wedge_idx (kernel_helpers.hpp:601) */
static int fine_lat_idx( int x, int y, int w )
{
    static const int idx[2][2][2] = { { { 0, 1 }, { 2, 3 } }, { { 3, 2 }, { 1, 0 } } };
    return idx[w][y % 2][x % 2];
}

/* per fine wedge: B_w[i][d][j] = sum_q w_q (-(J^-T grad N_j)_d N^c_i |det J|) */
static void stokes_wedge_matrix( const double* p[3], double r1, double r2, int x, int y, int r, int w,
                                 double B[6][3][6] )
{
    memset( B, 0, sizeof( double ) * 6 * 3 * 6 );
    const int frad = r % 2, flat = fine_lat_idx( x, y, w );
    for ( int q = 0; q < 6; ++q )
    {
        double J[3][3], IT[3][3];
        wedge_jac( p, r1, r2, QP32[q][0], QP32[q][1], QP32[q][2], J );
        const double det = det3( J );
        inv_transposed3( J, det, IT );
        double g[6][3];
        for ( int n = 0; n < 6; ++n )
        {
            double gr[3];
            grad_shape_ref( n, QP32[q][0], QP32[q][1], QP32[q][2], gr );
            for ( int a = 0; a < 3; ++a )
                g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
        }
        for ( int i = 0; i < 6; ++i )
        {
            const double Ni = shape_coarse( i, frad, flat, QP32[q][0], QP32[q][1], QP32[q][2] );
            for ( int d = 0; d < 3; ++d )
                for ( int j = 0; j < 6; ++j )
                    B[i][d][j] += QW32 * ( -g[j][d] * Ni * fabs( det ) );
        }
    }
}

/* velocity node of fine wedge w is on the Dirichlet / free-slip boundary of this cell */
static int stokes_bc_node( int N, int r, int n, int bc_cmb, int bc_surf, int* kind )
{
    *kind = 0;
    if ( r == 0 && n < 3 )
        *kind = bc_cmb;
    else if ( r == N - 1 && n >= 3 )
        *kind = bc_surf;
    return *kind;
}

void or_divergence_apply( int L, const double* coords, const double* radii, const double* coords_c, const double* src,
                          double* dst, int bc_cmb, int bc_surf )
{
    const int    N = 1 << L, n1 = N + 1, nc1 = N / 2 + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1, nsc = (size_t) NDIAMOND * nc1 * nc1 * nc1;
    memset( dst, 0, sizeof( double ) * nsc );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        double B[6][3][6];
                        stokes_wedge_matrix( p, radii[d * n1 + r], radii[d * n1 + r + 1], x, y, r, w, B );
                        double u[6][3];
                        for ( int n = 0; n < 6; ++n )
                        {
                            const int    X = x + WNODE[w][n][0], Y = y + WNODE[w][n][1];
                            const size_t i = node_idx( n1, d, X, Y, r + WNODE[w][n][2] );
                            for ( int c = 0; c < 3; ++c )
                                u[n][c] = src[c * ns + i];
                            int kind;
                            if ( stokes_bc_node( N, r, n, bc_cmb, bc_surf, &kind ) == 1 )
                                u[n][0] = u[n][1] = u[n][2] = 0.0;
                            else if ( kind == 2 )
                            {
                                double nn[3];
                                memcpy( nn, coords + lat_idx( n1, d, X, Y ) * 3, sizeof( nn ) );
                                normalize3( nn );
                                fs_project( nn, u[n] );
                            }
                        }
                        for ( int i = 0; i < 6; ++i )
                        {
                            double v = 0.0;
                            for ( int dd = 0; dd < 3; ++dd )
                                for ( int j = 0; j < 6; ++j )
                                    v += B[i][dd][j] * u[j][dd];
                            /* scatter with the coarse wedge-w node map (kernel_helpers.hpp:407-435) */
                            const int X = x / 2 + WNODE[w][i][0], Y = y / 2 + WNODE[w][i][1], R = r / 2 + WNODE[w][i][2];
                            dst[node_idx( nc1, d, X, Y, R )] += v;
                        }
                    }
    or_halo_sum( L - 1, coords_c, dst, 1 );
}

void or_gradient_apply( int L, const double* coords, const double* radii, const double* src, double* dst, int bc_cmb,
                        int bc_surf )
{
    const int    N = 1 << L, n1 = N + 1, nc1 = N / 2 + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    memset( dst, 0, sizeof( double ) * 3 * ns );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        double B[6][3][6];
                        stokes_wedge_matrix( p, radii[d * n1 + r], radii[d * n1 + r + 1], x, y, r, w, B );
                        double pc[6];
                        for ( int i = 0; i < 6; ++i )
                            pc[i] = src[node_idx( nc1, d, x / 2 + WNODE[w][i][0], y / 2 + WNODE[w][i][1],
                                                  r / 2 + WNODE[w][i][2] )];
                        for ( int j = 0; j < 6; ++j )
                        {
                            double v[3] = { 0, 0, 0 };
                            for ( int dd = 0; dd < 3; ++dd )
                                for ( int i = 0; i < 6; ++i )
                                    v[dd] += B[i][dd][j] * pc[i];
                            const int X = x + WNODE[w][j][0], Y = y + WNODE[w][j][1];
                            int       kind;
                            if ( stokes_bc_node( N, r, j, bc_cmb, bc_surf, &kind ) == 1 )
                                continue;
                            if ( kind == 2 )
                            {
                                double nn[3];
                                memcpy( nn, coords + lat_idx( n1, d, X, Y ) * 3, sizeof( nn ) );
                                normalize3( nn );
                                fs_project( nn, v );
                            }
                            const size_t i = node_idx( n1, d, X, Y, r + WNODE[w][j][2] );
                            for ( int c = 0; c < 3; ++c )
                                dst[c * ns + i] += v[c];
                        }
                    }
    or_halo_sum( L, coords, dst, 3 );
}

/* ------------------------------------------------------------------------ */
/* Constant grid transfer (fe/wedge/shell/grid_transfer_constant.hpp:6-82,  */
/* prolongation_constant.hpp:103-190, restriction_constant.hpp:134-248).    */
/* ------------------------------------------------------------------------ */

/* prolongation_constant_weight: 1 / 1/2 on the coarse shell, 1/2 / 1/4 one fine shell off */
static double prolong_weight( int xf, int yf, int rf, int xc, int yc, int rc )
{
    const int dx = xf - 2 * xc, dy = yf - 2 * yc, dr = rf - 2 * rc;
    double    lat = 0.0;
    if ( dx == 0 && dy == 0 )
        lat = 1.0;
    else if ( ( dy == 0 && ( dx == 1 || dx == -1 ) ) || ( dx == 0 && ( dy == 1 || dy == -1 ) ) ||
              ( dx == -1 && dy == 1 ) || ( dx == 1 && dy == -1 ) )
        lat = 0.5;
    if ( dr == 0 )
        return lat;
    if ( dr == 1 || dr == -1 )
        return 0.5 * lat;
    return 0.0;
}

static const int STENCIL7[7][2] = { { -1, 0 }, { -1, 1 }, { 0, 1 }, { 1, 0 }, { 1, -1 }, { 0, -1 }, { 0, 0 } };

/* coarse level Lc -> fine level Lc+1, ncomp fields, Replace mode, no communication */
void or_prolongation_constant( int Lc, int ncomp, const double* src, double* dst )
{
    const int    nc1 = ( 1 << Lc ) + 1, nf1 = ( 1 << ( Lc + 1 ) ) + 1;
    const size_t nsc = (size_t) NDIAMOND * nc1 * nc1 * nc1, nsf = (size_t) NDIAMOND * nf1 * nf1 * nf1;
    memset( dst, 0, sizeof( double ) * nsf * ncomp );
    for ( int c = 0; c < ncomp; ++c )
        for ( int d = 0; d < NDIAMOND; ++d )
            for ( int x = 0; x < nc1; ++x )
                for ( int y = 0; y < nc1; ++y )
                    for ( int r = 0; r < nc1; ++r )
                        for ( int dr = -1; dr <= 1; ++dr )
                            for ( int s = 0; s < 7; ++s )
                            {
                                const int xf = 2 * x + STENCIL7[s][0], yf = 2 * y + STENCIL7[s][1], rf = 2 * r + dr;
                                if ( xf < 0 || xf >= nf1 || yf < 0 || yf >= nf1 || rf < 0 || rf >= nf1 )
                                    continue;
                                dst[c * nsf + node_idx( nf1, d, xf, yf, rf )] +=
                                    prolong_weight( xf, yf, rf, x, y, r ) * src[c * nsc + node_idx( nc1, d, x, y, r )];
                            }
}

/* fine level Lf -> coarse Lf-1: sum of weighted OWNED fine values, then coarse halo */
void or_restriction_constant( int Lf, int ncomp, const double* coords_c, const uint8_t* omask_f, const double* src,
                              double* dst )
{
    const int    nf1 = ( 1 << Lf ) + 1, nc1 = ( 1 << ( Lf - 1 ) ) + 1;
    const size_t nsc = (size_t) NDIAMOND * nc1 * nc1 * nc1, nsf = (size_t) NDIAMOND * nf1 * nf1 * nf1;
    memset( dst, 0, sizeof( double ) * nsc * ncomp );
    for ( int c = 0; c < ncomp; ++c )
        for ( int d = 0; d < NDIAMOND; ++d )
            for ( int x = 0; x < nc1; ++x )
                for ( int y = 0; y < nc1; ++y )
                    for ( int r = 0; r < nc1; ++r )
                    {
                        double v = 0.0;
                        for ( int dr = -1; dr <= 1; ++dr )
                            for ( int s = 0; s < 7; ++s )
                            {
                                const int xf = 2 * x + STENCIL7[s][0], yf = 2 * y + STENCIL7[s][1], rf = 2 * r + dr;
                                if ( xf < 0 || xf >= nf1 || yf < 0 || yf >= nf1 || rf < 0 || rf >= nf1 )
                                    continue;
                                const size_t i = node_idx( nf1, d, xf, yf, rf );
                                v += prolong_weight( xf, yf, rf, x, y, r ) * ( omask_f[i] ? 1.0 : 0.0 ) * src[c * nsf + i];
                            }
                        dst[c * nsc + node_idx( nc1, d, x, y, r )] = v;
                    }
    or_halo_sum( Lf - 1, coords_c, dst, ncomp );
}

/* ------------------------------------------------------------------------ */
/* KMass (fe/wedge/operators/shell/kmass.hpp): int k u v, 3x2 rule, k        */
/* interpolated at the quadrature points; mode 0 full, 1 diagonal, 2 lumped. */
/* ------------------------------------------------------------------------ */
/* ------------------------------------------------------------------------ */
/* Linear grid transfer (prolongation_linear.hpp:104-189,                    */
/* restriction_linear.hpp:106-222, weights grid_transfer_linear.hpp:14-158): */
/* a fine node on a coarse node takes its value; one between two radially    */
/* aligned coarse nodes interpolates by radius; any other lies on a wedge    */
/* facet spanned by two lateral coarse pairs and interpolates radially       */
/* between the chord midpoints of the pairs (weights halved per pair).       */
/* ------------------------------------------------------------------------ */

static double norm3v( const double v[3] ) { return sqrt( v[0] * v[0] + v[1] * v[1] + v[2] * v[2] ); }

/* contributions (coarse x, y, r, weight) of the coarse nodes to fine node (x, y, r) */
static int linear_stencil( int Nf, const double* coords_f, const double* radii_f, int d, int x, int y, int r,
                           int cx[4], int cy[4], int cr[4], double w[4] )
{
    const int n1 = Nf + 1;
    if ( x % 2 == 0 && y % 2 == 0 && r % 2 == 0 )
    {
        cx[0] = x / 2, cy[0] = y / 2, cr[0] = r / 2, w[0] = 1.0;
        return 1;
    }
    const int rb = r < Nf ? r / 2 : r / 2 - 1, rt = rb + 1;
    const double* c  = coords_f + lat_idx( n1, d, x, y ) * 3;
    const double  Rf = radii_f[d * n1 + r], Rb = radii_f[d * n1 + 2 * rb], Rt = radii_f[d * n1 + 2 * rt];
    double        fine[3];
    for ( int a = 0; a < 3; ++a )
        fine[a] = c[a] * Rf;
    if ( x % 2 == 0 && y % 2 == 0 )
    {
        double pb[3], pt[3];
        for ( int a = 0; a < 3; ++a )
            pb[a] = c[a] * Rb, pt[a] = c[a] * Rt;
        const double nu = ( norm3v( fine ) - norm3v( pb ) ) / ( norm3v( pt ) - norm3v( pb ) );
        cx[0] = cx[1] = x / 2, cy[0] = cy[1] = y / 2, cr[0] = rb, cr[1] = rt;
        w[0] = 1.0 - nu, w[1] = nu;
        return 2;
    }
    int x0, x1, y0, y1;
    if ( x % 2 == 0 )
        x0 = x1 = x / 2, y0 = y / 2, y1 = y / 2 + 1; /* "vertical" edge */
    else if ( y % 2 == 0 )
        x0 = x / 2, x1 = x / 2 + 1, y0 = y1 = y / 2; /* "horizontal" edge */
    else
        x0 = x / 2 + 1, x1 = x / 2, y0 = y / 2, y1 = y / 2 + 1; /* "diagonal" edge */
    const double* c0 = coords_f + lat_idx( n1, d, 2 * x0, 2 * y0 ) * 3;
    const double* c1 = coords_f + lat_idx( n1, d, 2 * x1, 2 * y1 ) * 3;
    double        bot[3], top[3];
    for ( int a = 0; a < 3; ++a )
    {
        bot[a] = 0.5 * ( c0[a] * Rb + c1[a] * Rb );
        top[a] = 0.5 * ( c0[a] * Rt + c1[a] * Rt );
    }
    const double nu = ( norm3v( fine ) - norm3v( bot ) ) / ( norm3v( top ) - norm3v( bot ) );
    const double wb = 0.5 * ( 1.0 - nu ), wt = 0.5 * nu;
    cx[0] = x0, cy[0] = y0, cr[0] = rb, w[0] = wb;
    cx[1] = x1, cy[1] = y1, cr[1] = rb, w[1] = wb;
    cx[2] = x0, cy[2] = y0, cr[2] = rt, w[2] = wt;
    cx[3] = x1, cy[3] = y1, cr[3] = rt, w[3] = wt;
    return 4;
}

void or_prolongation_linear( int Lc, int ncomp, const double* coords_f, const double* radii_f, const double* src,
                             double* dst )
{
    const int    Nf = 2 << Lc, n1f = Nf + 1, n1c = ( 1 << Lc ) + 1;
    const size_t nsf = (size_t) NDIAMOND * n1f * n1f * n1f, nsc = (size_t) NDIAMOND * n1c * n1c * n1c;
    for ( int c = 0; c < ncomp; ++c )
        for ( int d = 0; d < NDIAMOND; ++d )
            for ( int x = 0; x <= Nf; ++x )
                for ( int y = 0; y <= Nf; ++y )
                    for ( int r = 0; r <= Nf; ++r )
                    {
                        int    cx[4], cy[4], cr[4];
                        double w[4], v = 0.0;
                        const int k = linear_stencil( Nf, coords_f, radii_f, d, x, y, r, cx, cy, cr, w );
                        for ( int i = 0; i < k; ++i )
                            v += w[i] * src[c * nsc + node_idx( n1c, d, cx[i], cy[i], cr[i] )];
                        dst[c * nsf + node_idx( n1f, d, x, y, r )] = v;
                    }
}

void or_restriction_linear( int Lf, int ncomp, const double* coords_f, const double* radii_f, const double* coords_c,
                            const uint8_t* omask_f, const double* src, double* dst )
{
    const int    Nf = 1 << Lf, n1f = Nf + 1, n1c = Nf / 2 + 1;
    const size_t nsf = (size_t) NDIAMOND * n1f * n1f * n1f, nsc = (size_t) NDIAMOND * n1c * n1c * n1c;
    memset( dst, 0, sizeof( double ) * nsc * ncomp );
    for ( int c = 0; c < ncomp; ++c )
        for ( int d = 0; d < NDIAMOND; ++d )
            for ( int x = 0; x <= Nf; ++x )
                for ( int y = 0; y <= Nf; ++y )
                    for ( int r = 0; r <= Nf; ++r )
                    {
                        const size_t f = node_idx( n1f, d, x, y, r );
                        if ( !omask_f[f] )
                            continue;
                        int       cx[4], cy[4], cr[4];
                        double    w[4];
                        const int k = linear_stencil( Nf, coords_f, radii_f, d, x, y, r, cx, cy, cr, w );
                        for ( int i = 0; i < k; ++i )
                            dst[c * nsc + node_idx( n1c, d, cx[i], cy[i], cr[i] )] += w[i] * src[c * nsf + f];
                    }
    or_halo_sum( Lf - 1, coords_c, dst, ncomp );
}

void or_kmass_apply( int L, const double* coords, const double* radii, const double* k, const double* src, double* dst,
                     int mode )
{
    const int    N = 1 << L, n1 = N + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    memset( dst, 0, sizeof( double ) * ns );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        size_t idx[6];
                        for ( int n = 0; n < 6; ++n )
                            idx[n] = node_idx( n1, d, x + WNODE[w][n][0], y + WNODE[w][n][1], r + WNODE[w][n][2] );
                        const double r1 = radii[d * n1 + r], r2 = radii[d * n1 + r + 1];
                        double       A[6][6] = { { 0 } };
                        for ( int q = 0; q < 6; ++q )
                        {
                            const double xi = QP32[q][0], eta = QP32[q][1], zeta = QP32[q][2];
                            double       M[3][3];
                            for ( int a = 0; a < 3; ++a )
                            {
                                M[a][0] = p[1][a] - p[0][a];
                                M[a][1] = p[2][a] - p[0][a];
                                M[a][2] = ( 1 - xi - eta ) * p[0][a] + xi * p[1][a] + eta * p[2][a];
                            }
                            const double rq = r1 + 0.5 * ( r2 - r1 ) * ( 1 + zeta ), gr = 0.5 * ( r2 - r1 );
                            double       N6[6];
                            const double lat[3] = { 1 - xi - eta, xi, eta };
                            double       kq     = 0.0;
                            for ( int n = 0; n < 6; ++n )
                            {
                                N6[n] = lat[n % 3] * ( n < 3 ? 0.5 * ( 1 - zeta ) : 0.5 * ( 1 + zeta ) );
                                kq += N6[n] * k[idx[n]];
                            }
                            const double f = QW32 * kq * rq * rq * gr * fabs( det3( M ) );
                            for ( int i = 0; i < 6; ++i )
                                for ( int j = 0; j < 6; ++j )
                                    A[i][j] += f * N6[i] * N6[j];
                        }
                        for ( int i = 0; i < 6; ++i )
                        {
                            double v = 0.0;
                            for ( int j = 0; j < 6; ++j )
                            {
                                if ( mode == 0 )
                                    v += A[i][j] * src[idx[j]];
                                else if ( mode == 1 && i == j )
                                    v += A[i][j] * src[idx[j]];
                                else if ( mode == 2 )
                                    v += A[i][j] * src[idx[i]];
                            }
                            dst[idx[i]] += v;
                        }
                    }
    or_halo_sum( L, coords, dst, 1 );
}

/* ------------------------------------------------------------------------ */
/* Finite-volume FCT advection-diffusion on the hex cells of the shell       */
/* (fv/hex/operators/fct_advection_diffusion.hpp, geometry_helper.hpp,       */
/* fv/hex/helpers.hpp, communication/shell/fv_communication.hpp).            */
/* FV fields: [10][N+2][N+2][N+2] with one ghost layer, r fastest; the cell  */
/* (x, y, r), 1 <= x, y, r <= N, is the FE cell (x-1, y-1, r-1).             */
/* ------------------------------------------------------------------------ */

static inline size_t fv_idx( int n2, int d, int x, int y, int r ) { return ( ( (size_t) d * n2 + x ) * n2 + y ) * n2 + r; }

static const int FV_OFF[6][3] = { { -1, 0, 0 }, { 1, 0, 0 }, { 0, -1, 0 }, { 0, 1, 0 }, { 0, 0, -1 }, { 0, 0, 1 } };

/* wedge shape value (integrands.hpp:146) */
static double shape_val( int n, double xi, double eta, double zeta )
{
    const double lat = n % 3 == 0 ? 1 - xi - eta : ( n % 3 == 1 ? xi : eta );
    return lat * ( n < 3 ? 0.5 * ( 1 - zeta ) : 0.5 * ( 1 + zeta ) );
}

static void cross3( const double a[3], const double b[3], double c[3] )
{
    c[0] = a[1] * b[2] - a[2] * b[1], c[1] = a[2] * b[0] - a[0] * b[2], c[2] = a[0] * b[1] - a[1] * b[0];
}

/* lateral ghost map: for every ghost cell on the four lateral sides of a
 * diamond, the real cell across the shared face in the neighbouring diamond
 * (the two diamonds share the face's two edge nodes).  map[(d*4+side)*N + i]
 * = (d', x', y') in FV indices; sides: x = 0, x = N+1, y = 0, y = N+1. */
static void fv_ghost_map( int L, const double* coords, int* map )
{
    const int N = 1 << L, n1 = N + 1;
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int side = 0; side < 4; ++side )
            for ( int i = 0; i < N; ++i )
            {
                int px, py, qx, qy; /* edge nodes (lateral FE indices) */
                if ( side < 2 )
                    px = qx = side == 0 ? 0 : N, py = i, qy = i + 1;
                else
                    py = qy = side == 2 ? 0 : N, px = i, qx = i + 1;
                const double* P = coords + lat_idx( n1, d, px, py ) * 3;
                const double* Q = coords + lat_idx( n1, d, qx, qy ) * 3;
                int* out = map + ( (size_t) ( d * 4 + side ) * N + i ) * 3;
                out[0] = out[1] = out[2] = -1;
                for ( int e = 0; e < NDIAMOND && out[0] < 0; ++e )
                {
                    if ( e == d )
                        continue;
                    /* boundary lines of diamond e: (X fixed 0 / N) or (Y fixed 0 / N) */
                    for ( int line = 0; line < 4 && out[0] < 0; ++line )
                        for ( int j = 0; j < N; ++j )
                        {
                            int ax, ay, bx, by;
                            if ( line < 2 )
                                ax = bx = line == 0 ? 0 : N, ay = j, by = j + 1;
                            else
                                ay = by = line == 2 ? 0 : N, ax = j, bx = j + 1;
                            const double* A = coords + lat_idx( n1, e, ax, ay ) * 3;
                            const double* B = coords + lat_idx( n1, e, bx, by ) * 3;
                            const int same = ( !memcmp( A, P, 24 ) && !memcmp( B, Q, 24 ) ) ||
                                             ( !memcmp( A, Q, 24 ) && !memcmp( B, P, 24 ) );
                            if ( !same )
                                continue;
                            out[0] = e;
                            if ( line == 0 )
                                out[1] = 1, out[2] = j + 1;
                            else if ( line == 1 )
                                out[1] = N, out[2] = j + 1;
                            else if ( line == 2 )
                                out[1] = j + 1, out[2] = 1;
                            else
                                out[1] = j + 1, out[2] = N;
                            break;
                        }
                }
            }
}

void or_fv_ghost_update( int L, const double* coords, double* field )
{
    const int N = 1 << L, n2 = N + 2;
    int*      map = (int*) malloc( sizeof( int ) * 3 * NDIAMOND * 4 * N );
    fv_ghost_map( L, coords, map );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int side = 0; side < 4; ++side )
            for ( int i = 0; i < N; ++i )
            {
                const int* m  = map + ( (size_t) ( d * 4 + side ) * N + i ) * 3;
                const int  gx = side == 0 ? 0 : ( side == 1 ? N + 1 : i + 1 );
                const int  gy = side == 2 ? 0 : ( side == 3 ? N + 1 : i + 1 );
                for ( int r = 1; r <= N; ++r )
                    field[fv_idx( n2, d, gx, gy, r )] = field[fv_idx( n2, m[0], m[1], m[2], r )];
            }
    free( map );
}

/* compute_cell_centers (fv/hex/helpers.hpp:101-150): volume-weighted
 * centroid over both wedges with the 3x2 rule, then the lateral ghosts */
void or_fv_cell_centers( int L, const double* coords, const double* radii, double* centers )
{
    const int    N = 1 << L, n1 = N + 1, n2 = N + 2;
    const size_t nf = (size_t) NDIAMOND * n2 * n2 * n2;
    memset( centers, 0, sizeof( double ) * 3 * nf );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 1; x <= N; ++x )
            for ( int y = 1; y <= N; ++y )
                for ( int r = 1; r <= N; ++r )
                {
                    double vol = 0.0, c[3] = { 0, 0, 0 };
                    const double r1 = radii[d * n1 + r - 1], r2 = radii[d * n1 + r];
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x - 1, y - 1, w, p );
                        for ( int q = 0; q < 6; ++q )
                        {
                            double J[3][3];
                            wedge_jac( p, r1, r2, QP32[q][0], QP32[q][1], QP32[q][2], J );
                            const double Jw = fabs( det3( J ) ) * QW32;
                            const double rq = r1 + 0.5 * ( r2 - r1 ) * ( 1 + QP32[q][2] );
                            vol += Jw;
                            for ( int a = 0; a < 3; ++a )
                                c[a] += ( ( 1 - QP32[q][0] - QP32[q][1] ) * p[0][a] + QP32[q][0] * p[1][a] +
                                          QP32[q][1] * p[2][a] ) *
                                        rq * Jw;
                        }
                    }
                    for ( int a = 0; a < 3; ++a )
                        centers[a * nf + fv_idx( n2, d, x, y, r )] = c[a] / vol;
                }
    for ( int a = 0; a < 3; ++a )
        or_fv_ghost_update( L, coords, centers + a * nf );
}

/* GeometryHelper::compute_geometry (geometry_helper.hpp:180-363): face fluxes
 * beta_n = int u . dS, face vectors S_n (oriented from the cell towards the
 * neighbour's centre) and the cell volume M_ii */
static void fv_geometry( int L, const double* coords, const double* radii, const double* centers, const double* vel,
                         int d, int x, int y, int r, double beta[6], double* Mii, double S[6][3] )
{
    const int    N = 1 << L, n1 = N + 1, n2 = N + 2;
    const size_t nf = (size_t) NDIAMOND * n2 * n2 * n2, ns = (size_t) NDIAMOND * n1 * n1 * n1;
    const double r1 = radii[d * n1 + r - 1], r2 = radii[d * n1 + r];
    static const double TQ[3][2] = { { 0.6666666666666666, 0.1666666666666667 },
                                     { 0.1666666666666667, 0.6666666666666666 },
                                     { 0.1666666666666667, 0.1666666666666667 } };
    const double        g1      = -1.0 / sqrt( 3.0 ), g2 = 1.0 / sqrt( 3.0 );
    const double        GL[2]   = { g1, g2 };
    for ( int n = 0; n < 6; ++n )
    {
        beta[n] = 0.0;
        S[n][0] = S[n][1] = S[n][2] = 0.0;
    }
    *Mii = 0.0;
    const double* p[2][3];
    double        u[2][6][3];
    for ( int w = 0; w < 2; ++w )
    {
        wedge_lateral_points( n1, coords, d, x - 1, y - 1, w, p[w] );
        for ( int i = 0; i < 6; ++i )
        {
            const size_t id = node_idx( n1, d, x - 1 + WNODE[w][i][0], y - 1 + WNODE[w][i][1], r - 1 + WNODE[w][i][2] );
            for ( int a = 0; a < 3; ++a )
                u[w][i][a] = vel[a * ns + id];
        }
    }
    for ( int nb = 0; nb < 6; ++nb )
    {
        for ( int w = 0; w < 2; ++w )
        {
            /* contribution(): wedge 0 owns faces 0, 2 (quad), wedge 1 faces 1, 3; both the radial triangles */
            int quad;
            if ( nb >= 4 )
                quad = 0;
            else if ( ( w == 0 && ( nb == 0 || nb == 2 ) ) || ( w == 1 && ( nb == 1 || nb == 3 ) ) )
                quad = 1;
            else
                continue;
            const int nq = quad ? 4 : 3;
            for ( int q = 0; q < nq; ++q )
            {
                double s, t, wq;
                if ( quad )
                    s = 0.5 * ( GL[q / 2] + 1.0 ), t = GL[q % 2], wq = 0.5;
                else
                    s = TQ[q][0], t = TQ[q][1], wq = 0.1666666666666667;
                double xi, eta, zeta;
                int    cpt; /* 0 xi-eta, 1 xi-zeta, 2 eta-zeta */
                if ( nb == 0 || nb == 1 )
                    xi = 0, eta = s, zeta = t, cpt = 2;
                else if ( nb == 2 || nb == 3 )
                    xi = s, eta = 0, zeta = t, cpt = 1;
                else
                    xi = s, eta = t, zeta = nb == 4 ? -1.0 : 1.0, cpt = 0;
                double dxi[3] = { 0, 0, 0 }, deta[3] = { 0, 0, 0 }, dzeta[3] = { 0, 0, 0 }, uq[3] = { 0, 0, 0 };
                for ( int i = 0; i < 6; ++i )
                {
                    double gr[3];
                    grad_shape_ref( i, xi, eta, zeta, gr );
                    const double sh = shape_val( i, xi, eta, zeta );
                    const double rr = i < 3 ? r1 : r2;
                    for ( int a = 0; a < 3; ++a )
                    {
                        const double xa = p[w][i % 3][a] * rr;
                        dxi[a] += gr[0] * xa;
                        deta[a] += gr[1] * xa;
                        dzeta[a] += gr[2] * xa;
                        uq[a] += sh * u[w][i][a];
                    }
                }
                double nv[3];
                if ( cpt == 0 )
                    cross3( dxi, deta, nv );
                else if ( cpt == 1 )
                    cross3( dxi, dzeta, nv );
                else
                    cross3( deta, dzeta, nv );
                beta[nb] += wq * ( uq[0] * nv[0] + uq[1] * nv[1] + uq[2] * nv[2] );
                for ( int a = 0; a < 3; ++a )
                    S[nb][a] += wq * nv[a];
            }
        }
        double dc = 0.0;
        for ( int a = 0; a < 3; ++a )
            dc += S[nb][a] * ( centers[a * nf + fv_idx( n2, d, x + FV_OFF[nb][0], y + FV_OFF[nb][1], r + FV_OFF[nb][2] )] -
                               centers[a * nf + fv_idx( n2, d, x, y, r )] );
        if ( dc < 0 )
        {
            for ( int a = 0; a < 3; ++a )
                S[nb][a] = -S[nb][a];
            beta[nb] = -beta[nb];
        }
    }
    for ( int w = 0; w < 2; ++w )
        for ( int q = 0; q < 6; ++q )
        {
            double J[3][3];
            wedge_jac( p[w], r1, r2, QP32[q][0], QP32[q][1], QP32[q][2], J );
            *Mii += fabs( det3( J ) ) * QW32;
        }
}

/* compute_dt_stable (fct_advection_diffusion.hpp:193-254) */
double or_fct_dt_stable( int L, const double* coords, const double* radii, const double* centers, const double* vel,
                         double diffusivity )
{
    const int    N = 1 << L, n2 = N + 2;
    const size_t nf = (size_t) NDIAMOND * n2 * n2 * n2;
    double       dtmin = 1e300;
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 1; x <= N; ++x )
            for ( int y = 1; y <= N; ++y )
                for ( int r = 1; r <= N; ++r )
                {
                    double beta[6], Mii, S[6][3], lambda = 0.0;
                    fv_geometry( L, coords, radii, centers, vel, d, x, y, r, beta, &Mii, S );
                    for ( int n = 0; n < 6; ++n )
                    {
                        if ( beta[n] < 0 )
                            lambda -= beta[n];
                        if ( diffusivity > 0 )
                        {
                            double dx[3], den = 0.0, ss = 0.0;
                            for ( int a = 0; a < 3; ++a )
                            {
                                dx[a] = centers[a * nf + fv_idx( n2, d, x + FV_OFF[n][0], y + FV_OFF[n][1], r + FV_OFF[n][2] )] -
                                        centers[a * nf + fv_idx( n2, d, x, y, r )];
                                den += dx[a] * S[n][a];
                                ss += S[n][a] * S[n][a];
                            }
                            if ( den > 0 )
                                lambda += diffusivity * ss / den;
                        }
                    }
                    const double dtc = lambda > 0 ? Mii / lambda : 1e30;
                    if ( dtc < dtmin )
                        dtmin = dtc;
                }
    return dtmin;
}

/* apply_dirichlet_bcs (fv/hex/helpers.hpp:26-64): first / last real layer and its ghost */
void or_fct_dirichlet( int L, double* T, double T_cmb, double T_surf, int apply_cmb, int apply_surf )
{
    const int N = 1 << L, n2 = N + 2;
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 1; x <= N; ++x )
            for ( int y = 1; y <= N; ++y )
            {
                if ( apply_cmb )
                    T[fv_idx( n2, d, x, y, 1 )] = T[fv_idx( n2, d, x, y, 0 )] = T_cmb;
                if ( apply_surf )
                    T[fv_idx( n2, d, x, y, N )] = T[fv_idx( n2, d, x, y, N + 1 )] = T_surf;
            }
}

/* fct_explicit_step (fct_advection_diffusion.hpp:720-750): predictor (low
 * order upwind + two-point diffusion, pre-scaled antidiffusive fluxes),
 * Dirichlet on T^L, limiter (Zalesak R+-), correction.  T is updated in
 * place (its lateral ghosts are refreshed first); source may be NULL;
 * bcs NULL skips the Dirichlet step; T_L_out (optional) receives T^L. */
void or_fct_step( int L, const double* coords, const double* radii, const double* centers, const double* vel,
                  double* T, double dt, double diffusivity, const double* source, int subtract_divergence,
                  const double* bcs, double* T_L_out )
{
    const int    N = 1 << L, n2 = N + 2;
    const size_t nf = (size_t) NDIAMOND * n2 * n2 * n2;
    double*      TL = (double*) calloc( nf, sizeof( double ) );
    double*      F  = (double*) calloc( nf * 6, sizeof( double ) );
    double*      Rp = (double*) calloc( nf, sizeof( double ) );
    double*      Rm = (double*) calloc( nf, sizeof( double ) );
    or_fv_ghost_update( L, coords, T );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 1; x <= N; ++x )
            for ( int y = 1; y <= N; ++y )
                for ( int r = 1; r <= N; ++r )
                {
                    double       beta[6], Mii, S[6][3];
                    const size_t i = fv_idx( n2, d, x, y, r );
                    fv_geometry( L, coords, radii, centers, vel, d, x, y, r, beta, &Mii, S );
                    const double Ti = T[i];
                    double       lo_diag = 0.0, lo_update = 0.0, bsum = 0.0;
                    for ( int n = 0; n < 6; ++n )
                    {
                        const size_t j  = fv_idx( n2, d, x + FV_OFF[n][0], y + FV_OFF[n][1], r + FV_OFF[n][2] );
                        const double Tj = T[j];
                        if ( beta[n] >= 0 )
                            lo_diag += beta[n];
                        else
                            lo_update += beta[n] * Tj;
                        bsum += beta[n];
                        double den = 0.0, ss = 0.0;
                        for ( int a = 0; a < 3; ++a )
                        {
                            den += ( centers[a * nf + j] - centers[a * nf + i] ) * S[n][a];
                            ss += S[n][a] * S[n][a];
                        }
                        const double dc = diffusivity * ( ss / den );
                        lo_diag += dc;
                        lo_update -= dc * Tj;
                        F[i * 6 + n] = ( dt / Mii ) * ( fabs( beta[n] ) / 2.0 ) * ( Ti - Tj );
                    }
                    if ( subtract_divergence )
                        lo_diag -= bsum;
                    double tl = Ti - ( dt / Mii ) * ( lo_diag * Ti + lo_update );
                    if ( source )
                        tl += dt * source[i];
                    TL[i] = tl;
                }
    if ( bcs )
        or_fct_dirichlet( L, TL, bcs[0], bcs[1], bcs[2] != 0, bcs[3] != 0 );
    or_fv_ghost_update( L, coords, TL );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 1; x <= N; ++x )
            for ( int y = 1; y <= N; ++y )
                for ( int r = 1; r <= N; ++r )
                {
                    const size_t i = fv_idx( n2, d, x, y, r );
                    double       Pp = 0.0, Pm = 0.0, tmax = TL[i], tmin = TL[i];
                    for ( int n = 0; n < 6; ++n )
                    {
                        const double f = F[i * 6 + n];
                        if ( f > 0 )
                            Pp += f;
                        else
                            Pm += f;
                        const double tj = TL[fv_idx( n2, d, x + FV_OFF[n][0], y + FV_OFF[n][1], r + FV_OFF[n][2] )];
                        tmax = tj > tmax ? tj : tmax;
                        tmin = tj < tmin ? tj : tmin;
                    }
                    const double Qp = tmax - TL[i], Qm = tmin - TL[i];
                    Rp[i] = Pp > 0 ? ( Qp / Pp < 1.0 ? Qp / Pp : 1.0 ) : 1.0;
                    Rm[i] = Pm < 0 ? ( Qm / Pm < 1.0 ? Qm / Pm : 1.0 ) : 1.0;
                }
    or_fv_ghost_update( L, coords, Rp );
    or_fv_ghost_update( L, coords, Rm );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 1; x <= N; ++x )
            for ( int y = 1; y <= N; ++y )
                for ( int r = 1; r <= N; ++r )
                {
                    const size_t i = fv_idx( n2, d, x, y, r );
                    double       corr = 0.0;
                    for ( int n = 0; n < 6; ++n )
                    {
                        const size_t j = fv_idx( n2, d, x + FV_OFF[n][0], y + FV_OFF[n][1], r + FV_OFF[n][2] );
                        const double f = F[i * 6 + n];
                        double       al;
                        if ( f > 0 )
                            al = Rp[i] < Rm[j] ? Rp[i] : Rm[j];
                        else
                            al = Rm[i] < Rp[j] ? Rm[i] : Rp[j];
                        corr += al * f;
                    }
                    T[i] = TL[i] + corr;
                }
    if ( T_L_out )
        memcpy( T_L_out, TL, sizeof( double ) * nf );
    free( TL );
    free( F );
    free( Rp );
    free( Rm );
}

/* ------------------------------------------------------------------------ */
/* EpsilonDivDiv with the 3x2 Felippa rule (epsilon_divdiv.hpp:218-600):     */
/* int k (2 eps(u):eps(v) - 2/3 div u div v), k interpolated by the wedge    */
/* shape functions at every quadrature point; treat_boundary eliminates the  */
/* CMB nodes of layer 0 (else the SURFACE nodes of layer N-1) keeping their  */
/* diagonal; diagonal mode keeps only the diagonal.                          */
/* ------------------------------------------------------------------------ */

void or_epsdivdiv3x2_apply( int L, const double* coords, const double* radii, const double* k, const double* src,
                            double* dst, int treat_boundary, int diag )
{
    const int    N = 1 << L, n1 = N + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    memset( dst, 0, sizeof( double ) * 3 * ns );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                {
                    const int bot = treat_boundary && r == 0;
                    const int top = treat_boundary && !bot && r == N - 1;
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        size_t idx[6];
                        double s[6][3], kv[6], out[6][3];
                        memset( out, 0, sizeof( out ) );
                        for ( int n = 0; n < 6; ++n )
                        {
                            idx[n] = node_idx( n1, d, x + WNODE[w][n][0], y + WNODE[w][n][1], r + WNODE[w][n][2] );
                            kv[n]  = k[idx[n]];
                            for ( int c = 0; c < 3; ++c )
                                s[n][c] = src[c * ns + idx[n]];
                        }
                        int coupled[6];
                        for ( int n = 0; n < 6; ++n )
                            coupled[n] = !diag && !( bot && n < 3 ) && !( top && n >= 3 );
                        for ( int q = 0; q < 6; ++q )
                        {
                            double J[3][3], IT[3][3], g[6][3];
                            wedge_jac( p, radii[d * n1 + r], radii[d * n1 + r + 1], QP32[q][0], QP32[q][1], QP32[q][2], J );
                            const double det = det3( J );
                            inv_transposed3( J, det, IT );
                            double ke = 0.0;
                            for ( int n = 0; n < 6; ++n )
                            {
                                double gr[3];
                                grad_shape_ref( n, QP32[q][0], QP32[q][1], QP32[q][2], gr );
                                for ( int a = 0; a < 3; ++a )
                                    g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
                                ke += shape_ref( n, QP32[q][0], QP32[q][1], QP32[q][2] ) * kv[n];
                            }
                            const double wk = QW32 * ke * fabs( det );
                            /* coupled part: grad u over coupled nodes, tested by coupled nodes */
                            double G[3][3] = { { 0 } };
                            for ( int n = 0; n < 6; ++n )
                                if ( coupled[n] )
                                    for ( int a = 0; a < 3; ++a )
                                        for ( int b = 0; b < 3; ++b )
                                            G[a][b] += g[n][a] * s[n][b];
                            const double div = G[0][0] + G[1][1] + G[2][2];
                            for ( int n = 0; n < 6; ++n )
                            {
                                if ( coupled[n] )
                                    for ( int c = 0; c < 3; ++c )
                                    {
                                        double e = 0.0;
                                        for ( int a = 0; a < 3; ++a )
                                            e += g[n][a] * ( G[a][c] + G[c][a] );
                                        out[n][c] += wk * ( e - 2.0 / 3.0 * g[n][c] * div );
                                    }
                                else
                                {
                                    /* uncoupled (boundary or diagonal mode): the node's own diagonal */
                                    const double gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
                                    for ( int c = 0; c < 3; ++c )
                                        out[n][c] += wk * s[n][c] * ( gg + g[n][c] * g[n][c] / 3.0 );
                                }
                            }
                        }
                        for ( int n = 0; n < 6; ++n )
                            for ( int c = 0; c < 3; ++c )
                                dst[c * ns + idx[n]] += out[n][c];
                    }
                }
    or_halo_sum( L, coords, dst, 3 );
}


/* l2_project_fv_to_fe right-hand side (fv/hex/conversion.hpp:146-190): for every FV cell K (ghosts excluded),
   b_i += fv_K sum_q shape_i(q) |det J(q)| w_q over the 3x2 Felippa rule on each of the cell's two wedges, and
   the lumped diagonal D_i += sum_q shape_i(q) |det J(q)| w_q (l2_project_fv_to_fe_lumped, :243-300); then the
   node copies summed (communication::shell::send_recv).  fv [10][N+2]^3; b, D stored-node fields (either NULL). */
void or_fv_to_fe_rhs( int L, const double* coords, const double* radii, const double* fv, double* b, double* D )
{
    const int    N = 1 << L, n1 = N + 1, n2 = N + 2;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    if ( b )
        memset( b, 0, ns * sizeof( double ) );
    if ( D )
        memset( D, 0, ns * sizeof( double ) );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 1; x <= N; ++x )
            for ( int y = 1; y <= N; ++y )
                for ( int r = 1; r <= N; ++r )
                {
                    const double v  = fv ? fv[fv_idx( n2, d, x, y, r )] : 0.0;
                    const double r1 = radii[d * n1 + r - 1], r2 = radii[d * n1 + r];
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x - 1, y - 1, w, p );
                        for ( int i = 0; i < 6; ++i )
                        {
                            double acc = 0.0;
                            for ( int q = 0; q < 6; ++q )
                            {
                                double J[3][3];
                                wedge_jac( p, r1, r2, QP32[q][0], QP32[q][1], QP32[q][2], J );
                                acc += shape_val( i, QP32[q][0], QP32[q][1], QP32[q][2] ) * fabs( det3( J ) ) * QW32;
                            }
                            const size_t id = node_idx( n1, d, x - 1 + WNODE[w][i][0], y - 1 + WNODE[w][i][1],
                                                        r - 1 + WNODE[w][i][2] );
                            if ( b )
                                b[id] += acc * v;
                            if ( D )
                                D[id] += acc;
                        }
                    }
                }
    if ( b )
        or_halo_sum( L, coords, b, 1 );
    if ( D )
        or_halo_sum( L, coords, D, 1 );
}

/* FE -> FV cell averages (fv/hex/conversion.hpp:349-416): the integral of the FE field over the hex cell's two
 * wedges with the 3x2 rule divided by the cell volume from the same rule, for the cells x, y, r in 1..N of
 * fv ([10][N+2]^3); then the lateral FV ghost layers. */
void or_fe_to_fv( int L, const double* coords, const double* radii, const double* fe, double* fv )
{
    const int N = 1 << L, n1 = N + 1, n2 = N + 2;
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 1; x <= N; ++x )
            for ( int y = 1; y <= N; ++y )
                for ( int r = 1; r <= N; ++r )
                {
                    const double r1 = radii[d * n1 + r - 1], r2 = radii[d * n1 + r];
                    double       volume = 0.0, integral = 0.0;
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x - 1, y - 1, w, p );
                        double u[6];
                        for ( int i = 0; i < 6; ++i )
                            u[i] = fe[node_idx( n1, d, x - 1 + WNODE[w][i][0], y - 1 + WNODE[w][i][1],
                                                r - 1 + WNODE[w][i][2] )];
                        for ( int q = 0; q < 6; ++q )
                        {
                            double J[3][3];
                            wedge_jac( p, r1, r2, QP32[q][0], QP32[q][1], QP32[q][2], J );
                            const double jw = fabs( det3( J ) ) * QW32;
                            double       uq = 0.0;
                            for ( int i = 0; i < 6; ++i )
                                uq += u[i] * shape_val( i, QP32[q][0], QP32[q][1], QP32[q][2] );
                            volume += jw;
                            integral += uq * jw;
                        }
                    }
                    fv[fv_idx( n2, d, x, y, r )] = integral / volume;
                }
    or_fv_ghost_update( L, coords, fv );
}

/* ------------------------------------------------------------------------ */
/* UnsteadyAdvectionDiffusionSUPG (fe/wedge/operators/shell/                 */
/* unsteady_advection_diffusion_supg.hpp:16-50, 243-420)                     */
/* ------------------------------------------------------------------------ */

/* supg_tau (:16-50): h / (2 |u|) (coth(Pe) - 1 / Pe), Pe = |u| h / (2 max(kappa, 1e-8)), zero for |u| <= 1e-12
 * or Pe <= Pe_tol, clamped to 10 h / |u| */
static double supg_tau( double vel_norm, double kappa, double h, double pe_tol )
{
    const double kv = kappa > 1e-8 ? kappa : 1e-8;
    if ( vel_norm <= 1e-12 )
        return 0.0;
    const double pe = vel_norm * h / ( 2.0 * kv );
    if ( pe <= pe_tol )
        return 0.0;
    const double tau_max = 10.0 * h / ( vel_norm > 1e-12 ? vel_norm : 1e-12 );
    const double coth    = 1.0 / tanh( pe ) - 1.0 / pe;
    const double tau     = ( h / ( 2.0 * vel_norm ) ) * coth;
    return tau > tau_max ? tau_max : tau;
}

/* dst = (mass_scaling M + dt (K + C + G)) src per hex cell, the 6 x 6 wedge matrices built on the 3x2 rule with
 * the velocity interpolated at the quadrature points and one tau per wedge (the weight-averaged pointwise tau,
 * h = r2 - r1), then lumping (row sums of M), the boundary mask (off-diagonal entries of rows and columns of
 * CMB / surface nodes zeroed), the diagonal mode, and the additive halo sum (:243-420). vel: [3][nodes]. */
void or_supg_apply( int L, const double* coords, const double* radii, const double* vel, const double* src, double* dst,
                    double kappa, double dt, double mass_scaling, int lumped, int treat_boundary, int diag )
{
    const int    N = 1 << L, n1 = N + 1;
    const size_t ns = (size_t) NDIAMOND * n1 * n1 * n1;
    memset( dst, 0, ns * sizeof( double ) );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                {
                    const double r1 = radii[d * n1 + r], r2 = radii[d * n1 + r + 1];
                    const double h  = r2 - r1;
                    for ( int w = 0; w < 2; ++w )
                    {
                        const double* p[3];
                        wedge_lateral_points( n1, coords, d, x, y, w, p );
                        size_t id[6];
                        for ( int i = 0; i < 6; ++i )
                            id[i] = node_idx( n1, d, x + WNODE[w][i][0], y + WNODE[w][i][1], r + WNODE[w][i][2] );
                        double uq[6][3];
                        for ( int q = 0; q < 6; ++q )
                            for ( int c = 0; c < 3; ++c )
                            {
                                uq[q][c] = 0.0;
                                for ( int i = 0; i < 6; ++i )
                                    uq[q][c] += vel[(size_t) c * ns + id[i]] * shape_val( i, QP32[q][0], QP32[q][1], QP32[q][2] );
                            }
                        double tau_acc = 0.0, w_acc = 0.0;
                        for ( int q = 0; q < 6; ++q )
                        {
                            const double vn = sqrt( uq[q][0] * uq[q][0] + uq[q][1] * uq[q][1] + uq[q][2] * uq[q][2] );
                            tau_acc += supg_tau( vn, kappa, h, 1e-8 ) * QW32;
                            w_acc += QW32;
                        }
                        const double tau = w_acc > 0.0 ? tau_acc / w_acc : 0.0;
                        double       M[6][6] = { { 0 } }, A[6][6] = { { 0 } };
                        for ( int q = 0; q < 6; ++q )
                        {
                            double J[3][3], IT[3][3], g[6][3], sh[6];
                            wedge_jac( p, r1, r2, QP32[q][0], QP32[q][1], QP32[q][2], J );
                            const double det = det3( J );
                            inv_transposed3( J, det, IT );
                            for ( int i = 0; i < 6; ++i )
                            {
                                double gr[3];
                                grad_shape_ref( i, QP32[q][0], QP32[q][1], QP32[q][2], gr );
                                for ( int a = 0; a < 3; ++a )
                                    g[i][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
                                sh[i] = shape_val( i, QP32[q][0], QP32[q][1], QP32[q][2] );
                            }
                            const double ad = fabs( det );
                            for ( int i = 0; i < 6; ++i )
                                for ( int j = 0; j < 6; ++j )
                                {
                                    const double mass = sh[i] * sh[j];
                                    const double diff = kappa * ( g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2] );
                                    const double ugj  = uq[q][0] * g[j][0] + uq[q][1] * g[j][1] + uq[q][2] * g[j][2];
                                    const double ugi  = uq[q][0] * g[i][0] + uq[q][1] * g[i][1] + uq[q][2] * g[i][2];
                                    M[i][j] += QW32 * mass_scaling * mass * ad;
                                    A[i][j] += QW32 * dt * ( diff + ugj * sh[i] + tau * ugj * ugi ) * ad;
                                }
                        }
                        if ( lumped )
                            for ( int i = 0; i < 6; ++i )
                            {
                                double s = 0.0;
                                for ( int j = 0; j < 6; ++j )
                                    s += M[i][j];
                                for ( int j = 0; j < 6; ++j )
                                    M[i][j] = i == j ? s : 0.0;
                            }
                        if ( treat_boundary )
                        {
                            const int cmb = r == 0, surf = r + 1 == N;
                            for ( int i = 0; i < 6; ++i )
                                for ( int j = 0; j < 6; ++j )
                                    if ( i != j && ( ( cmb && ( i < 3 || j < 3 ) ) || ( surf && ( i >= 3 || j >= 3 ) ) ) )
                                        M[i][j] = A[i][j] = 0.0;
                        }
                        if ( diag )
                            for ( int i = 0; i < 6; ++i )
                                for ( int j = 0; j < 6; ++j )
                                    if ( i != j )
                                        M[i][j] = A[i][j] = 0.0;
                        for ( int i = 0; i < 6; ++i )
                        {
                            double s = 0.0;
                            for ( int j = 0; j < 6; ++j )
                                s += ( M[i][j] + A[i][j] ) * src[id[j]];
                            dst[id[i]] += s;
                        }
                    }
                }
    or_halo_sum( L, coords, dst, 1 );
}

/* ------------------------------------------------------------------------ */
/* Adaptive GCA: GCAElementsCollector (linalg/solvers/gca/                   */
/* gca_elements_collector.hpp:19-96)                                          */
/* ------------------------------------------------------------------------ */

/* Marks the coarsest-grid cell (x >> level_range, y >> level_range, r >> level_range) of every fine cell one of
 * whose wedges has |sum_j grad_ref phi_j(1/3, 1/3, 0) k_j| > 10 (the gradient in reference coordinates at the
 * one-point rule's centroid).  marks: [10][N0][N0][N0] with N0 = N >> level_range, zeroed here. */
void or_gca_elements( int L, const double* k, int level_range, uint8_t* marks )
{
    const int N = 1 << L, n1 = N + 1, N0 = N >> level_range;
    memset( marks, 0, (size_t) NDIAMOND * N0 * N0 * N0 );
    for ( int d = 0; d < NDIAMOND; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int r = 0; r < N; ++r )
                    for ( int w = 0; w < 2; ++w )
                    {
                        double kg[3] = { 0, 0, 0 };
                        for ( int j = 0; j < 6; ++j )
                        {
                            double g[3];
                            grad_shape_ref( j, 1.0 / 3.0, 1.0 / 3.0, 0.0, g );
                            const double kj = k[node_idx( n1, d, x + WNODE[w][j][0], y + WNODE[w][j][1], r + WNODE[w][j][2] )];
                            for ( int a = 0; a < 3; ++a )
                                kg[a] = kg[a] + g[a] * kj;
                        }
                        if ( sqrt( kg[0] * kg[0] + kg[1] * kg[1] + kg[2] * kg[2] ) > 10.0 )
                            marks[( ( (size_t) d * N0 + ( x >> level_range ) ) * N0 + ( y >> level_range ) ) * N0 +
                                  ( r >> level_range )] = 1;
                    }
}
