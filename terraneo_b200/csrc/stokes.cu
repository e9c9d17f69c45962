// Stokes coupling blocks: Divergence B (fine P1 velocity -> coarse P1
// pressure, fe/wedge/operators/shell/divergence.hpp) and Gradient B^T
// (gradient.hpp), Q1-iso-Q2 / Q1 with the 3x2 Felippa rule.
//
// B_{i,(d,j)} = -int (J^{-T} grad N_j)_d N^c_i |det J| over each fine wedge,
// N^c_i the coarse shape functions of the coarse wedge containing it
// (shape_coarse, integrands.hpp:266-400).  The coarse node each wedge-local
// coarse slot is added to follows the reference's wedge map
// (atomically_add_local_wedge_scalar_coefficients, kernel_helpers.hpp:407):
// fine wedge w always scatters to coarse wedge w's node positions, also for
// the two middle fine triangles whose shape functions belong to the other
// coarse wedge.  Kept as is for parity; Gradient uses the same map, so B^T is
// the exact transpose.
//
// Boundary conditions act on the velocity side: Dirichlet nodes are dropped,
// free-slip nodes are projected onto the tangent plane (the reference's
// rotate / eliminate-normal / rotate-back sequence, :226-290).
//
// Factored form.  With the fine wedge's a = p1 - p0, b = p2 - p0, v = a x b,
// D = v . p0, c = p0 + xi a + eta b, u_1 = b x c, u_2 = c x a,
// u_0 = -(u_1 + u_2) and h = (r2 - r1) / 2, every quadrature point has
//     |det J| grad N_n = sign(D) ( r h nr_n(zeta) u_m + r^2 s_n lat_m v )
// (m the lateral vertex of node n, s_n = -+1/2, nr_n = (1 -+ zeta)/2), and the
// coarse shape function is a lateral factor times a radial one.  On the
// tensor-product 3x2 rule the block therefore separates into
//     B_{i,(n,:)} = Ra[i/3][n/3] Uc[i%3][n%3] + s_n Rb[i/3] Lc[i%3][n%3] vt
// with per-triangle lateral tables (Uc = -w sign(D) sum_q latc_i(q) u_m(q),
// vt = -w sign(D) v, Lc = sum_q latc_i(q) lat_m(q)) built once per mesh and
// the radial sums Ra = sum_zeta radc_i r h nr_n, Rb = sum_zeta radc_i r^2
// formed per cell: the same integrals as the per-point Jacobian of
// fe/wedge/integrands.hpp at a fraction of the arithmetic.
//
// One thread per fine wedge (the wedge uniform within a warp), contributions
// added with atomics.  In B the lanes of a warp are consecutive radial cells:
// a lane takes its bottom nodes from the lane below by shuffle, and the two
// fine cells of one coarse cell add their coarse contributions together.
#include <cmath>

#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

constexpr double kQPHost[3][2] = { { 0.6666666666666666, 0.1666666666666667 },
                                   { 0.1666666666666667, 0.6666666666666666 },
                                   { 0.1666666666666667, 0.1666666666666667 } };
constexpr double kZeta = 0.5773502691896257;
constexpr double kQW   = 0.1666666666666667;

// coarse lateral shape coefficients (a, b xi, c eta) per [node % 3][fine lateral wedge index]
// (shape_coarse, integrands.hpp:266-400)
constexpr double kCoarseLat[3][4][3] = {
    { { 1.0, -0.5, -0.5 }, { 0.5, -0.5, -0.5 }, { 0.5, -0.5, -0.5 }, { 0.0, 0.5, 0.5 } },
    { { 0.0, 0.5, 0.0 }, { 0.5, 0.5, 0.0 }, { 0.0, 0.5, 0.0 }, { 0.5, -0.5, 0.0 } },
    { { 0.0, 0.0, 0.5 }, { 0.0, 0.0, 0.5 }, { 0.5, 0.0, 0.5 }, { 0.5, 0.0, -0.5 } } };

__host__ __device__ __forceinline__ int fine_lateral_wedge( int x, int y, int w )
{
    // fine_lateral_wedge_idx (kernel_helpers.hpp:601)
    const int xm = x & 1, ym = y & 1;
    return w == 0 ? ( ym * 2 + xm ) : ( 3 - ( ym * 2 + xm ) );
}

// per fine wedge: Uc[3][3][3] (27), vt (3), Lc[3][3] (9)
constexpr int kStokesStride = 39;

template < typename T >
struct StokesParams
{
    int           N, n1, nc1;
    const double* coords; // fine lateral coords
    const double* geom;   // kStokesStride doubles per fine wedge
    const T*      radii;  // fine radii
    int           bc_cmb, bc_surf;
};

// 0: interior, 1: Dirichlet (drop), 2: free-slip (project)
__device__ __forceinline__ int velocity_bc( int N, int r, int n, int bc_cmb, int bc_surf )
{
    if ( r == 0 && n < 3 )
        return bc_cmb;
    if ( r == N - 1 && n >= 3 )
        return bc_surf;
    return 0;
}

// outward unit normal x / |x| (one reciprocal square root)
template < typename T >
__device__ __forceinline__ void unit_normal( const double* c, T n[3] )
{
    const double im = rsqrt( c[0] * c[0] + c[1] * c[1] + c[2] * c[2] );
    n[0] = T( c[0] * im ), n[1] = T( c[1] * im ), n[2] = T( c[2] * im );
}

// radial sums of one fine cell: Ra[ib][nb] = h sum_zeta radc_ib r nr_nb, Rb[ib] = sum_zeta radc_ib r^2
template < typename T >
__device__ __forceinline__ void radial_sums( T r1, T r2, int frad, T Ra[2][2], T Rb[2] )
{
    const T h = T( 0.5 ) * ( r2 - r1 );
    Ra[0][0] = Ra[0][1] = Ra[1][0] = Ra[1][1] = Rb[0] = Rb[1] = T( 0 );
#pragma unroll
    for ( int zq = 0; zq < 2; ++zq )
    {
        const T zeta = zq ? T( kZeta ) : T( -kZeta );
        const T rr   = r1 + h * ( T( 1 ) + zeta );
        const T nr[2] = { T( 0.5 ) * ( T( 1 ) - zeta ), T( 0.5 ) * ( T( 1 ) + zeta ) };
        const T rc[2] = { frad == 0 ? T( 0.25 ) * ( T( 3 ) - zeta ) : T( 0.25 ) * ( T( 1 ) - zeta ),
                          frad == 0 ? T( 0.25 ) * ( T( 1 ) + zeta ) : T( 0.25 ) * ( T( 3 ) + zeta ) };
#pragma unroll
        for ( int ib = 0; ib < 2; ++ib )
        {
            Rb[ib] += rc[ib] * rr * rr;
#pragma unroll
            for ( int nb = 0; nb < 2; ++nb )
                Ra[ib][nb] += rc[ib] * rr * h * nr[nb];
        }
    }
}

__device__ __forceinline__ size_t stokes_tri( int N, int dm, int x, int y, int w )
{
    return ( ( size_t( dm ) * N + x ) * N + y ) * 2 + w;
}

// One thread per fine wedge: the first half of the grid takes wedge 0 of
// every fine cell, the second half wedge 1, so the wedge is uniform within a
// warp and a compile-time constant in the body; each wedge adds its six node
// contributions with atomics (half the registers of a two-wedge thread, twice
// the threads).
__device__ __forceinline__ void fine_cell( int N, long long c, int& dm, int& x, int& y, int& r )
{
    r  = int( c % N );
    y  = int( ( c / N ) % N );
    x  = int( ( c / ( (long long) N * N ) ) % N );
    dm = int( c / ( (long long) N * N * N ) );
}

// p_coarse += B u, wedge W of fine cell (dm, x, y, r)
template < typename T, int W >
__device__ __forceinline__ void divergence_wedge( const StokesParams< T >& P, const Ptr3< const T >& u, T* p, int dm,
                                                  int x, int y, int r )
{
    const int N = P.N, n1 = P.n1, nc1 = P.nc1;
    T         Ra[2][2], Rb[2];
    radial_sums( P.radii[dm * n1 + r], P.radii[dm * n1 + r + 1], r & 1, Ra, Rb );
    const double* G = P.geom + stokes_tri( N, dm, x, y, W ) * kStokesStride;
    // lanes are consecutive radial cells of one column: the bottom nodes of a
    // lane are the top nodes of the lane below (raw values, shuffled before
    // any boundary treatment); the first lane of a column loads its own
    const int  lane = threadIdx.x & 31;
    const bool own_bottom = lane == 0 || r == 0;
    T          uu[6][3];
#pragma unroll
    for ( int n = 3; n < 6; ++n )
    {
        const size_t i = lat_index( n1, dm, x + kWedgeNode[W][n][0], y + kWedgeNode[W][n][1] ) * n1 + r + 1;
        uu[n][0] = u.p[0][i], uu[n][1] = u.p[1][i], uu[n][2] = u.p[2][i];
    }
#pragma unroll
    for ( int n = 0; n < 3; ++n )
    {
        // node n lies below node n + 3 (kWedgeNode rows 0-2 and 3-5 share their lateral positions)
#pragma unroll
        for ( int a = 0; a < 3; ++a )
            uu[n][a] = __shfl_up_sync( 0xffffffffu, uu[n + 3][a], 1 );
        if ( own_bottom )
        {
            const size_t i = lat_index( n1, dm, x + kWedgeNode[W][n][0], y + kWedgeNode[W][n][1] ) * n1 + r;
            uu[n][0] = u.p[0][i], uu[n][1] = u.p[1][i], uu[n][2] = u.p[2][i];
        }
    }
#pragma unroll
    for ( int n = 0; n < 6; ++n )
    {
        const int X = x + kWedgeNode[W][n][0], Y = y + kWedgeNode[W][n][1];
        const int bc = velocity_bc( N, r, n, P.bc_cmb, P.bc_surf );
        if ( bc == TN_BC_DIRICHLET )
            uu[n][0] = uu[n][1] = uu[n][2] = T( 0 );
        else if ( bc == TN_BC_FREESLIP )
        {
            T nn[3];
            unit_normal( P.coords + lat_index( n1, dm, X, Y ) * 3, nn );
            const T dt = nn[0] * uu[n][0] + nn[1] * uu[n][1] + nn[2] * uu[n][2];
            uu[n][0] -= dt * nn[0], uu[n][1] -= dt * nn[1], uu[n][2] -= dt * nn[2];
        }
    }
    const T vt[3] = { T( G[27] ), T( G[28] ), T( G[29] ) };
    T       vu[6];
#pragma unroll
    for ( int n = 0; n < 6; ++n )
        vu[n] = ( n < 3 ? T( -0.5 ) : T( 0.5 ) ) * ( vt[0] * uu[n][0] + vt[1] * uu[n][1] + vt[2] * uu[n][2] );
    T acc[6] = { 0, 0, 0, 0, 0, 0 };
#pragma unroll
    for ( int ic = 0; ic < 3; ++ic )
#pragma unroll
        for ( int m = 0; m < 3; ++m )
        {
            const double* U  = G + ( ic * 3 + m ) * 3;
            const T       U0 = T( U[0] ), U1 = T( U[1] ), U2 = T( U[2] ), lc = T( G[30 + ic * 3 + m] );
#pragma unroll
            for ( int nb = 0; nb < 2; ++nb )
            {
                const int n  = nb * 3 + m;
                const T   cu = U0 * uu[n][0] + U1 * uu[n][1] + U2 * uu[n][2];
                const T   lv = lc * vu[n];
#pragma unroll
                for ( int ib = 0; ib < 2; ++ib )
                    acc[ib * 3 + ic] += Ra[ib][nb] * cu + Rb[ib] * lv;
            }
        }
    // the two fine cells r = 2 rc, 2 rc + 1 (lanes 2k, 2k + 1) add to the same
    // six coarse nodes: the even lane adds both
    const int xc = x >> 1, yc = y >> 1, rc = r >> 1;
#pragma unroll
    for ( int i = 0; i < 6; ++i )
        acc[i] += __shfl_down_sync( 0xffffffffu, acc[i], 1 );
    if ( lane & 1 )
        return;
#pragma unroll
    for ( int i = 0; i < 6; ++i )
        atomicAdd( p + lat_index( nc1, dm, xc + kWedgeNode[W][i][0], yc + kWedgeNode[W][i][1] ) * nc1 + rc +
                       kWedgeNode[W][i][2],
                   acc[i] );
}

template < typename T >
__global__ void __launch_bounds__( 128 ) divergence_kernel( StokesParams< T > P, Ptr3< const T > u, T* __restrict__ p )
{
    const long long cells = (long long) kDiamonds * P.N * P.N * P.N;
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= 2 * cells )
        return;
    int dm, x, y, r;
    fine_cell( P.N, t < cells ? t : t - cells, dm, x, y, r );
    if ( t < cells )
        divergence_wedge< T, 0 >( P, u, p, dm, x, y, r );
    else
        divergence_wedge< T, 1 >( P, u, p, dm, x, y, r );
}

// u_fine += B^T p, wedge W of fine cell (dm, x, y, r).  Lanes are consecutive radial cells of one column
// (whole columns per warp): the top-node contributions of a lane go to the lane above by shuffle, where they
// meet the same nodes as that lane's bottom nodes, so each lane adds its bottom nodes and only the column's
// last cell in the warp also adds its top nodes (about half the reductions).  Boundary treatment acts on
// bottom nodes at r = 0 and top nodes at r = N - 1, never on a handed-over value.
template < typename T, int W >
__device__ __forceinline__ void gradient_wedge( const StokesParams< T >& P, const T* p, const Ptr3< T >& u, int dm,
                                                int x, int y, int r )
{
    const int N = P.N, n1 = P.n1, nc1 = P.nc1;
    const int xc = x >> 1, yc = y >> 1, rc = r >> 1;
    const int lane = threadIdx.x & 31;
    T         Ra[2][2], Rb[2];
    radial_sums( P.radii[dm * n1 + r], P.radii[dm * n1 + r + 1], r & 1, Ra, Rb );
    const double* G = P.geom + stokes_tri( N, dm, x, y, W ) * kStokesStride;
    T             pc[6];
#pragma unroll
    for ( int i = 0; i < 6; ++i )
        pc[i] = p[lat_index( nc1, dm, xc + kWedgeNode[W][i][0], yc + kWedgeNode[W][i][1] ) * nc1 + rc +
                  kWedgeNode[W][i][2]];
    const T vt[3] = { T( G[27] ), T( G[28] ), T( G[29] ) };
    // pr[nb][ic] = sum_ib Ra[ib][nb] pc[ib][ic]; pl[ic] = sum_ib Rb[ib] pc[ib][ic]
    T pr[2][3], pl[3];
#pragma unroll
    for ( int ic = 0; ic < 3; ++ic )
    {
        pl[ic] = Rb[0] * pc[ic] + Rb[1] * pc[3 + ic];
#pragma unroll
        for ( int nb = 0; nb < 2; ++nb )
            pr[nb][ic] = Ra[0][nb] * pc[ic] + Ra[1][nb] * pc[3 + ic];
    }
    const bool from_below = lane > 0 && r > 0;        // the lane below is cell r - 1 of this column
    const bool adds_top   = lane == 31 || r == N - 1; // no lane above takes this cell's top nodes
#pragma unroll
    for ( int m = 0; m < 3; ++m )
    {
        T sv = T( 0 );
#pragma unroll
        for ( int ic = 0; ic < 3; ++ic )
            sv += T( G[30 + ic * 3 + m] ) * pl[ic];
        T v[2][3];
#pragma unroll
        for ( int nb = 0; nb < 2; ++nb )
        {
            const T s = ( nb ? T( 0.5 ) : T( -0.5 ) ) * sv;
            v[nb][0] = s * vt[0], v[nb][1] = s * vt[1], v[nb][2] = s * vt[2];
#pragma unroll
            for ( int ic = 0; ic < 3; ++ic )
            {
                const double* U = G + ( ic * 3 + m ) * 3;
                v[nb][0] += pr[nb][ic] * T( U[0] ), v[nb][1] += pr[nb][ic] * T( U[1] ),
                    v[nb][2] += pr[nb][ic] * T( U[2] );
            }
        }
        const int X = x + kWedgeNode[W][m][0], Y = y + kWedgeNode[W][m][1];
#pragma unroll
        for ( int c = 0; c < 3; ++c )
        {
            const T below = __shfl_up_sync( 0xffffffffu, v[1][c], 1 );
            if ( from_below )
                v[0][c] += below;
        }
#pragma unroll
        for ( int nb = 0; nb < 2; ++nb )
        {
            if ( nb == 1 && !adds_top )
                continue;
            const int bc = velocity_bc( N, r, nb * 3 + m, P.bc_cmb, P.bc_surf );
            if ( bc == TN_BC_DIRICHLET )
                continue;
            if ( bc == TN_BC_FREESLIP )
            {
                T nn[3];
                unit_normal( P.coords + lat_index( n1, dm, X, Y ) * 3, nn );
                const T dt = nn[0] * v[nb][0] + nn[1] * v[nb][1] + nn[2] * v[nb][2];
                v[nb][0] -= dt * nn[0], v[nb][1] -= dt * nn[1], v[nb][2] -= dt * nn[2];
            }
            const size_t i = lat_index( n1, dm, X, Y ) * n1 + r + nb;
            atomicAdd( u.p[0] + i, v[nb][0] );
            atomicAdd( u.p[1] + i, v[nb][1] );
            atomicAdd( u.p[2] + i, v[nb][2] );
        }
    }
}

template < typename T >
__global__ void __launch_bounds__( 128 ) gradient_kernel( StokesParams< T > P, const T* __restrict__ p, Ptr3< T > u )
{
    const long long cells = (long long) kDiamonds * P.N * P.N * P.N;
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= 2 * cells )
        return;
    int dm, x, y, r;
    fine_cell( P.N, t < cells ? t : t - cells, dm, x, y, r );
    if ( t < cells )
        gradient_wedge< T, 0 >( P, p, u, dm, x, y, r );
    else
        gradient_wedge< T, 1 >( P, p, u, dm, x, y, r );
}

// Host tabulation of the lateral factors of every fine wedge (double).
void build_stokes_geometry( const tn_mesh* m, std::vector< double >& G )
{
    const int N = m->N, n1 = m->n1;
    const int wn[2][3][2] = { { { 0, 0 }, { 1, 0 }, { 0, 1 } }, { { 1, 1 }, { 0, 1 }, { 1, 0 } } };
    auto      cross = []( const double* a, const double* b, double* o ) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    G.assign( size_t( kDiamonds ) * N * N * 2 * kStokesStride, 0.0 );
    for ( int d = 0; d < kDiamonds; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int w = 0; w < 2; ++w )
                {
                    double*       g = G.data() + ( ( ( size_t( d ) * N + x ) * N + y ) * 2 + w ) * kStokesStride;
                    const int     flat = fine_lateral_wedge( x, y, w );
                    const double* p[3];
                    for ( int k = 0; k < 3; ++k )
                        p[k] = m->h_coords.data() + lat_index( n1, d, x + wn[w][k][0], y + wn[w][k][1] ) * 3;
                    double a[3], b[3], v[3];
                    for ( int k = 0; k < 3; ++k )
                        a[k] = p[1][k] - p[0][k], b[k] = p[2][k] - p[0][k];
                    cross( a, b, v );
                    const double D   = v[0] * p[0][0] + v[1] * p[0][1] + v[2] * p[0][2];
                    const double sig = -kQW * ( D < 0 ? -1.0 : 1.0 );
                    for ( int q = 0; q < 3; ++q )
                    {
                        const double xi = kQPHost[q][0], eta = kQPHost[q][1];
                        const double lat[3] = { 1.0 - xi - eta, xi, eta };
                        double       c[3], u[3][3];
                        for ( int k = 0; k < 3; ++k )
                            c[k] = p[0][k] + xi * a[k] + eta * b[k];
                        cross( b, c, u[1] );
                        cross( c, a, u[2] );
                        for ( int k = 0; k < 3; ++k )
                            u[0][k] = -( u[1][k] + u[2][k] );
                        for ( int ic = 0; ic < 3; ++ic )
                        {
                            const double lc = kCoarseLat[ic][flat][0] + kCoarseLat[ic][flat][1] * xi +
                                              kCoarseLat[ic][flat][2] * eta;
                            for ( int mm = 0; mm < 3; ++mm )
                            {
                                for ( int k = 0; k < 3; ++k )
                                    g[( ic * 3 + mm ) * 3 + k] += sig * lc * u[mm][k];
                                g[30 + ic * 3 + mm] += lc * lat[mm];
                            }
                        }
                    }
                    for ( int k = 0; k < 3; ++k )
                        g[27 + k] = sig * v[k];
                }
}

const double* stokes_geometry( const tn_mesh* m )
{
    tn_mesh*                      mm = const_cast< tn_mesh* >( m );
    std::lock_guard< std::mutex > lock( mm->geom_mutex );
    if ( !mm->d_stokes_geom )
    {
        std::vector< double > G;
        build_stokes_geometry( m, G );
        double* ptr = nullptr;
        if ( cudaMalloc( &ptr, G.size() * sizeof( double ) ) != cudaSuccess )
            return nullptr;
        if ( cudaMemcpy( ptr, G.data(), G.size() * sizeof( double ), cudaMemcpyHostToDevice ) != cudaSuccess )
        {
            cudaFree( ptr );
            return nullptr;
        }
        mm->d_stokes_geom = ptr;
    }
    return mm->d_stokes_geom;
}

template < typename T >
const T* radii_of( const tn_mesh* m )
{
    return sizeof( T ) == 8 ? reinterpret_cast< const T* >( m->d_radii ) : reinterpret_cast< const T* >( m->d_radii32 );
}

int check_pair( const tn_mesh* f, const tn_mesh* c )
{
    TN_CHECK_ARG( f && c, "stokes block: null mesh" );
    TN_CHECK_ARG( c->level == f->level - 1 && c->r_min == f->r_min && c->r_max == f->r_max,
                  "stokes block: the pressure mesh must be the velocity mesh coarsened once" );
    // the B / B^T kernels run one fine wedge per thread with full-mask warp
    // shuffles between even and odd lanes: every warp must hold one wedge type
    // and whole radial columns, i.e. 10 N^3 a multiple of 32 and N even (N >= 4)
    const long long N = f->N;
    TN_CHECK_ARG( N >= 4 && N % 2 == 0 && ( 10LL * N * N * N ) % 32 == 0,
                  "stokes block: the velocity mesh needs level >= 2 (whole radial columns per warp)" );
    return TN_OK;
}

}  // namespace

template < typename T >
int divergence_apply( const tn_mesh* f, const tn_mesh* c, int bc_cmb, int bc_surf, int apply_mode, int comm_mode,
                      const T* const* u, T* p, cudaStream_t st )
{
    int rc;
    if ( ( rc = check_pair( f, c ) ) )
        return rc;
    TN_CHECK_ARG( u && u[0] && u[1] && u[2] && p, "divergence: null vector" );
    if ( apply_mode == TN_APPLY_REPLACE )
        TN_CUDA_TRY( cudaMemsetAsync( p, 0, c->ns * sizeof( T ), st ) );
    StokesParams< T > P{ f->N, f->n1, c->n1, f->d_coords, stokes_geometry( f ), radii_of< T >( f ), bc_cmb, bc_surf };
    if ( !P.geom )
    {
        set_error( "stokes block: allocating the lateral quadrature table failed" );
        return TN_ERR_NOMEM;
    }
    const long long   cells = (long long) kDiamonds * f->N * f->N * f->N;
    divergence_kernel< T ><<< unsigned( ( 2 * cells + 127 ) / 128 ), 128, 0, st >>>( P, Ptr3< const T >{ { u[0], u[1], u[2] } },
                                                                                p );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
    {
        T* fl[1] = { p };
        return halo_sum< T >( c, fl, 1, st );
    }
    return TN_OK;
}

template < typename T >
int gradient_apply( const tn_mesh* f, const tn_mesh* c, int bc_cmb, int bc_surf, int apply_mode, int comm_mode,
                    const T* p, T* const* u, cudaStream_t st )
{
    int rc;
    if ( ( rc = check_pair( f, c ) ) )
        return rc;
    TN_CHECK_ARG( u && u[0] && u[1] && u[2] && p, "gradient: null vector" );
    if ( apply_mode == TN_APPLY_REPLACE )
        for ( int i = 0; i < 3; ++i )
            TN_CUDA_TRY( cudaMemsetAsync( u[i], 0, f->ns * sizeof( T ), st ) );
    StokesParams< T > P{ f->N, f->n1, c->n1, f->d_coords, stokes_geometry( f ), radii_of< T >( f ), bc_cmb, bc_surf };
    if ( !P.geom )
    {
        set_error( "stokes block: allocating the lateral quadrature table failed" );
        return TN_ERR_NOMEM;
    }
    const long long   cells = (long long) kDiamonds * f->N * f->N * f->N;
    gradient_kernel< T ><<< unsigned( ( 2 * cells + 127 ) / 128 ), 128, 0, st >>>( P, p, Ptr3< T >{ { u[0], u[1], u[2] } } );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( f, u, 3, st );
    return TN_OK;
}

template int divergence_apply< double >( const tn_mesh*, const tn_mesh*, int, int, int, int, const double* const*,
                                         double*, cudaStream_t );
template int divergence_apply< float >( const tn_mesh*, const tn_mesh*, int, int, int, int, const float* const*,
                                        float*, cudaStream_t );
template int gradient_apply< double >( const tn_mesh*, const tn_mesh*, int, int, int, int, const double*,
                                       double* const*, cudaStream_t );
template int gradient_apply< float >( const tn_mesh*, const tn_mesh*, int, int, int, int, const float*, float* const*,
                                      cudaStream_t );

}  // namespace tn

using namespace tn;

extern "C" int tn_divergence_apply_f64( const tn_mesh* f, const tn_mesh* c, int bcc, int bcs, int am, int cm,
                                        const double* const* u, double* p, void* s )
{
    return divergence_apply< double >( f, c, bcc, bcs, am, cm, u, p, as_stream( s ) );
}
extern "C" int tn_divergence_apply_f32( const tn_mesh* f, const tn_mesh* c, int bcc, int bcs, int am, int cm,
                                        const float* const* u, float* p, void* s )
{
    return divergence_apply< float >( f, c, bcc, bcs, am, cm, u, p, as_stream( s ) );
}
extern "C" int tn_gradient_apply_f64( const tn_mesh* f, const tn_mesh* c, int bcc, int bcs, int am, int cm,
                                      const double* p, double* const* u, void* s )
{
    return gradient_apply< double >( f, c, bcc, bcs, am, cm, p, u, as_stream( s ) );
}
extern "C" int tn_gradient_apply_f32( const tn_mesh* f, const tn_mesh* c, int bcc, int bcs, int am, int cm,
                                      const float* p, float* const* u, void* s )
{
    return gradient_apply< float >( f, c, bcc, bcs, am, cm, p, u, as_stream( s ) );
}
