// Epsilon-div-div operator apply (B200 design of EpsilonDivDivKerngen,
// fe/wedge/operators/shell/epsilon_divdiv_kerngen.hpp).
//
// a(u, v) = int k (2 eps(u):eps(v) - 2/3 div u div v) with the one-point
// (centroid) wedge rule and k averaged over the six wedge nodes (:1189-1196).
//
// Kernels
//  * kerngen_tile_kernel: the hot path.  One CTA owns a tile of 8 x 8 lateral
//    node columns of one diamond over the full radial extent and computes every
//    cell touching them (owner computes: no global atomics, no zero-fill pass,
//    every stored node written exactly once with coalesced stores).  Lanes of
//    a warp are 32 consecutive radial cells of one cell column, so loads are
//    coalesced along r and the radial node sharing is a warp shuffle; lateral
//    node sharing goes through a shared-memory accumulator in four colour
//    phases (cells of one colour share no node).  Per-wedge geometry is
//    factorised as J = M diag(r_mid, r_mid, dr/2) with M the lateral triangle
//    matrix, so M^{-T} is computed once per tile and each cell only rescales.
//    Boundary-layer cells of a non-Neumann boundary are left out and added by
//  * kerngen_cell_kernel: one thread per cell with the full boundary logic
//    (Dirichlet elimination with kept diagonal, free-slip projection with the
//    normal-normal add-back, rotated diagonal), accumulating with atomics.  It
//    also provides the diagonal mode and levels too small for tiling.
//  * penalty kernels for free-slip on both boundaries.
#include <algorithm>

#include "common.cuh"
#include "reduce.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

constexpr int kTile    = 8;  // owned lateral node columns per tile side
constexpr int kWarps   = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kRC      = 32; // radial cells per chunk (one per lane)
constexpr int kCols    = ( kTile + 1 ) * ( kTile + 1 );
constexpr int kAccCol  = kRC + 1;

template < typename T >
struct TileParams
{
    int           N, n1, tiles;
    const double* coords;
    const T*      radii;
    const T*      k;
    Ptr3< const T > src;
    Ptr3< T >     dst;
    int           add_mode;
    int           skip_cmb, skip_surface; // leave that boundary layer of cells to the cell kernel
    const double* beta;                   // fs/fs penalty vector (3) or nullptr
};

template < typename T >
size_t tile_smem_bytes( int n1 )
{
    return sizeof( T ) * ( size_t( ( n1 + 1 ) & ~1 ) + size_t( kCols ) * 20 + size_t( 3 ) * kCols * kAccCol );
}

// Per-wedge flux vectors S1 = sigma q0, S2 = sigma q1, S3 = kappa sigma q2 with
// sigma = omega (2 sym(G) - 2/3 tr(G) I), G = q0 (x) v1 + q1 (x) v2 + q2 (x) kappa v3.
template < typename T >
__device__ __forceinline__ void wedge_flux( const T* __restrict__ g, const T v1[3], const T v2[3], const T v3[3],
                                            T kappa, T omega, T S1[3], T S2[3], T S3[3] )
{
    T q0[3], q1[3], q2[3];
#pragma unroll
    for ( int a = 0; a < 3; ++a )
        q0[a] = g[a], q1[a] = g[3 + a], q2[a] = g[6 + a];
    const T w3[3] = { kappa * v3[0], kappa * v3[1], kappa * v3[2] };
    const T G00   = q0[0] * v1[0] + q1[0] * v2[0] + q2[0] * w3[0];
    const T G11   = q0[1] * v1[1] + q1[1] * v2[1] + q2[1] * w3[1];
    const T G22   = q0[2] * v1[2] + q1[2] * v2[2] + q2[2] * w3[2];
    const T H01   = q0[0] * v1[1] + q1[0] * v2[1] + q2[0] * w3[1] + q0[1] * v1[0] + q1[1] * v2[0] + q2[1] * w3[0];
    const T H02   = q0[0] * v1[2] + q1[0] * v2[2] + q2[0] * w3[2] + q0[2] * v1[0] + q1[2] * v2[0] + q2[2] * w3[0];
    const T H12   = q0[1] * v1[2] + q1[1] * v2[2] + q2[1] * w3[2] + q0[2] * v1[1] + q1[2] * v2[1] + q2[2] * w3[1];
    const T div   = G00 + G11 + G22;
    const T tdiv  = T( 2.0 / 3.0 ) * div;
    const T s00 = omega * ( T( 2 ) * G00 - tdiv ), s11 = omega * ( T( 2 ) * G11 - tdiv ),
            s22 = omega * ( T( 2 ) * G22 - tdiv );
    const T s01 = omega * H01, s02 = omega * H02, s12 = omega * H12;
    S1[0] = s00 * q0[0] + s01 * q0[1] + s02 * q0[2];
    S1[1] = s01 * q0[0] + s11 * q0[1] + s12 * q0[2];
    S1[2] = s02 * q0[0] + s12 * q0[1] + s22 * q0[2];
    S2[0] = s00 * q1[0] + s01 * q1[1] + s02 * q1[2];
    S2[1] = s01 * q1[0] + s11 * q1[1] + s12 * q1[2];
    S2[2] = s02 * q1[0] + s12 * q1[1] + s22 * q1[2];
    S3[0] = kappa * ( s00 * q2[0] + s01 * q2[1] + s02 * q2[2] );
    S3[1] = kappa * ( s01 * q2[0] + s11 * q2[1] + s12 * q2[2] );
    S3[2] = kappa * ( s02 * q2[0] + s12 * q2[1] + s22 * q2[2] );
}

template < typename T >
__global__ void __launch_bounds__( kThreads ) kerngen_tile_kernel( TileParams< T > P )
{
    extern __shared__ __align__( 16 ) unsigned char smem_raw[];
    const int N = P.N, n1 = P.n1;
    int       b  = blockIdx.x;
    const int tx = b % P.tiles;
    b /= P.tiles;
    const int ty = b % P.tiles;
    const int d  = b / P.tiles;

    // owned node columns [xlo, xhi] x [ylo, yhi]; cells touching them
    const int xlo = tx == 0 ? 0 : tx * kTile + 1, xhi = tx * kTile + kTile;
    const int ylo = ty == 0 ? 0 : ty * kTile + 1, yhi = ty * kTile + kTile;
    const int nyo = yhi - ylo + 1;
    const int nxo = xhi - xlo + 1;
    const int cxlo = tx * kTile, cxhi = min( xhi, N - 1 );
    const int cylo = ty * kTile, cyhi = min( yhi, N - 1 );
    const int ncx = cxhi - cxlo + 1, ncy = cyhi - cylo + 1;

    T* s_radii = reinterpret_cast< T* >( smem_raw );
    T* s_geo   = s_radii + ( ( n1 + 1 ) & ~1 );
    T* s_acc   = s_geo + kCols * 20;
    constexpr int kAccComp = kCols * kAccCol;

    for ( int i = threadIdx.x; i < n1; i += blockDim.x )
        s_radii[i] = P.radii[d * n1 + i];
    for ( int i = threadIdx.x; i < ncx * ncy * 2; i += blockDim.x )
    {
        const int     w = i & 1, col = i >> 1;
        const int     X = cxlo + col / ncy, Y = cylo + col % ncy;
        const double* c00 = P.coords + lat_index( n1, d, X, Y ) * 3;
        const double* c10 = P.coords + lat_index( n1, d, X + 1, Y ) * 3;
        const double* c01 = P.coords + lat_index( n1, d, X, Y + 1 ) * 3;
        const double* c11 = P.coords + lat_index( n1, d, X + 1, Y + 1 ) * 3;
        double        q[9], adet;
        if ( w == 0 )
            lateral_geometry( c00, c10, c01, q, &adet );
        else
            lateral_geometry( c11, c01, c10, q, &adet );
        T* g = s_geo + i * 10;
        for ( int j = 0; j < 9; ++j )
            g[j] = T( q[j] );
        g[9] = T( adet );
    }
    for ( int i = threadIdx.x; i < 3 * kAccComp; i += blockDim.x )
        s_acc[i] = T( 0 );
    double beta[3] = { 0, 0, 0 };
    if ( P.beta )
        beta[0] = P.beta[0], beta[1] = P.beta[1], beta[2] = P.beta[2];
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int RC   = min( kRC, N );
    constexpr unsigned FULL = 0xffffffffu;

    for ( int r0 = 0; r0 < N; r0 += RC )
    {
        const bool last_chunk = ( r0 + RC == N );
        const int  r          = r0 + lane;
        const int  rl         = min( r, N - 1 );
        bool       valid      = lane < RC;
        if ( ( P.skip_cmb && r == 0 ) || ( P.skip_surface && r == N - 1 ) )
            valid = false;
        const T r_lo = s_radii[rl], r_hi = s_radii[rl + 1];
        const T h     = T( 0.5 ) * ( r_hi - r_lo );
        const T kappa = T( 0.5 ) * ( r_hi + r_lo ) / ( T( 3 ) * h );
        const T wbase = h * T( 0.25 ) * T( 1.0 / 6.0 ); // omega = k_sum/6 * |det M| * h/4

        for ( int phase = 0; phase < 4; ++phase )
        {
            const int ox = ( phase & 1 ) ^ ( cxlo & 1 ), oy = ( ( phase >> 1 ) & 1 ) ^ ( cylo & 1 );
            const int nxp = ncx > ox ? ( ncx - ox + 1 ) / 2 : 0, nyp = ncy > oy ? ( ncy - oy + 1 ) / 2 : 0;
            for ( int task = warp; task < nxp * nyp; task += kWarps )
            {
                const int lx = ox + 2 * ( task / nyp ), ly = oy + 2 * ( task % nyp );
                const int X = cxlo + lx, Y = cylo + ly;

                // corner order: 0 = (0,0), 1 = (1,0), 2 = (0,1), 3 = (1,1)
                T      ub[4][3], ut[4][3], kb[4], kt[4];
                size_t base[4];
#pragma unroll
                for ( int q = 0; q < 4; ++q )
                {
                    base[q] = lat_index( n1, d, X + ( q & 1 ), Y + ( q >> 1 ) ) * n1;
                    kb[q]   = __ldg( P.k + base[q] + rl );
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        ub[q][c] = __ldg( P.src.p[c] + base[q] + rl );
                }
#pragma unroll
                for ( int q = 0; q < 4; ++q )
                {
                    kt[q] = __shfl_down_sync( FULL, kb[q], 1 );
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        ut[q][c] = __shfl_down_sync( FULL, ub[q][c], 1 );
                }
                if ( lane == RC - 1 )
                {
#pragma unroll
                    for ( int q = 0; q < 4; ++q )
                    {
                        kt[q] = __ldg( P.k + base[q] + rl + 1 );
#pragma unroll
                        for ( int c = 0; c < 3; ++c )
                            ut[q][c] = __ldg( P.src.p[c] + base[q] + rl + 1 );
                    }
                }

                T bot[4][3], top[4][3];
                {
                    T S[4][3], D[4][3];
#pragma unroll
                    for ( int q = 0; q < 4; ++q )
#pragma unroll
                        for ( int c = 0; c < 3; ++c )
                            S[q][c] = ub[q][c] + ut[q][c], D[q][c] = ut[q][c] - ub[q][c];
                    const T* g0 = s_geo + ( ( lx * ncy + ly ) * 2 ) * 10;
                    const T* g1 = g0 + 10;
                    T        v1[3], v2[3], v3[3], A1[3], A2[3], A3[3], B1[3], B2[3], B3[3];
                    // wedge 0: nodes (0,0),(1,0),(0,1)
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        v1[c] = S[1][c] - S[0][c], v2[c] = S[2][c] - S[0][c], v3[c] = D[0][c] + D[1][c] + D[2][c];
                    const T k0 = ( kb[0] + kb[1] + kb[2] ) + ( kt[0] + kt[1] + kt[2] );
                    wedge_flux( g0, v1, v2, v3, kappa, wbase * k0 * g0[9], A1, A2, A3 );
                    // wedge 1: nodes (1,1),(0,1),(1,0)
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        v1[c] = S[2][c] - S[3][c], v2[c] = S[1][c] - S[3][c], v3[c] = D[3][c] + D[2][c] + D[1][c];
                    const T k1 = ( kb[3] + kb[2] + kb[1] ) + ( kt[3] + kt[2] + kt[1] );
                    wedge_flux( g1, v1, v2, v3, kappa, wbase * k1 * g1[9], B1, B2, B3 );
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                    {
                        const T xa = A1[c] + A2[c], xb = B1[c] + B2[c];
                        const T s33 = A3[c] + B3[c];
                        const T e10 = A1[c] + B2[c], e01 = A2[c] + B1[c];
                        bot[0][c] = -xa - A3[c], top[0][c] = -xa + A3[c];
                        bot[1][c] = e10 - s33, top[1][c] = e10 + s33;
                        bot[2][c] = e01 - s33, top[2][c] = e01 + s33;
                        bot[3][c] = -xb - B3[c], top[3][c] = -xb + B3[c];
                        if ( !valid )
                            bot[0][c] = top[0][c] = bot[1][c] = top[1][c] = bot[2][c] = top[2][c] = bot[3][c] =
                                top[3][c] = T( 0 );
                    }
                }

#pragma unroll
                for ( int q = 0; q < 4; ++q )
                {
                    const int  Xn = X + ( q & 1 ), Yn = Y + ( q >> 1 );
                    const bool owned = Xn >= xlo && Xn <= xhi && Yn >= ylo && Yn <= yhi; // warp uniform
                    T*         acc   = s_acc + ( ( Xn - xlo ) * ( kTile + 1 ) + ( Yn - ylo ) ) * kAccCol;
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                    {
                        const T below = __shfl_up_sync( FULL, top[q][c], 1 );
                        if ( owned )
                        {
                            if ( lane < RC )
                                acc[c * kAccComp + lane] += bot[q][c] + ( lane > 0 ? below : T( 0 ) );
                            if ( lane == RC - 1 )
                                acc[c * kAccComp + RC] += top[q][c];
                        }
                    }
                }
            }
            __syncthreads();
        }

        // write out completed node levels of all owned columns
        const int nlev = last_chunk ? RC + 1 : RC;
        for ( int t = warp; t < nxo * nyo * 3; t += kWarps )
        {
            const int    c = t % 3, col = t / 3;
            const int    lx = col / nyo, ly = col % nyo;
            const int    X = xlo + lx, Y = ylo + ly;
            const size_t lat = lat_index( n1, d, X, Y );
            const T*     acc = s_acc + c * kAccComp + ( lx * ( kTile + 1 ) + ly ) * kAccCol;
            T*           out = P.dst.p[c] + lat * n1 + r0;
            for ( int l = lane; l < nlev; l += 32 )
            {
                T v = acc[l];
                if ( P.beta )
                {
                    const double  rr = double( s_radii[r0 + l] );
                    const double* u  = P.coords + lat * 3;
                    const double  x[3] = { u[0] * rr, u[1] * rr, u[2] * rr };
                    const double  bx   = c == 0 ? beta[1] * x[2] - beta[2] * x[1]
                                                : ( c == 1 ? beta[2] * x[0] - beta[0] * x[2] : beta[0] * x[1] - beta[1] * x[0] );
                    v += T( bx );
                }
                out[l] = P.add_mode ? out[l] + v : v;
            }
        }
        __syncthreads();
        for ( int i = threadIdx.x; i < 3 * kCols; i += blockDim.x )
        {
            T* a = s_acc + size_t( i ) * kAccCol;
            a[0] = a[RC];
            for ( int l = 1; l <= RC; ++l )
                a[l] = T( 0 );
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Per-cell kernel with full boundary handling (restates the reference's fast
// Dirichlet/Neumann path :1055-1389 and fast free-slip path :1421-1940).
template < typename T >
struct CellParams
{
    int           N, n1;
    const double* coords;
    const T*      radii;
    const T*      k;
    Ptr3< const T > src;
    Ptr3< T >     dst;
    int           bc_cmb, bc_surf, diag;
    int           layers; // 0: all cells; 1: r = 0 only; 2: r = N-1 only; 3: both boundary layers
};

template < typename T >
__device__ __forceinline__ void project_out( const T n[3], T v[3] )
{
    const T dt = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
    v[0] -= dt * n[0], v[1] -= dt * n[1], v[2] -= dt * n[2];
}

template < typename T >
__global__ void __launch_bounds__( 128 ) kerngen_cell_kernel( CellParams< T > P )
{
    const int       N = P.N, n1 = P.n1;
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const int       nr = P.layers == 0 ? N : ( P.layers == 3 ? 2 : 1 );
    if ( t >= (long long) kDiamonds * N * N * nr )
        return;
    const int ri = int( t % nr );
    const int y  = int( ( t / nr ) % N );
    const int x  = int( ( t / ( (long long) nr * N ) ) % N );
    const int d  = int( t / ( (long long) nr * N * N ) );
    const int r  = P.layers == 0 ? ri : ( P.layers == 1 ? 0 : ( P.layers == 2 ? N - 1 : ( ri == 0 ? 0 : N - 1 ) ) );

    const bool at_cmb = r == 0, at_surf = r == N - 1;
    const bool cmb_dir = at_cmb && P.bc_cmb == TN_BC_DIRICHLET, surf_dir = at_surf && P.bc_surf == TN_BC_DIRICHLET;
    const bool cmb_fs = at_cmb && P.bc_cmb == TN_BC_FREESLIP, surf_fs = at_surf && P.bc_surf == TN_BC_FREESLIP;
    const bool diag = P.diag != 0;

    T acc[2][2][2][3];
    T ann[2][2][2];
#pragma unroll
    for ( int i = 0; i < 8; ++i )
    {
        ann[i >> 2][( i >> 1 ) & 1][i & 1] = T( 0 );
        for ( int c = 0; c < 3; ++c )
            acc[i >> 2][( i >> 1 ) & 1][i & 1][c] = T( 0 );
    }
    const T r0 = P.radii[d * n1 + r], r1 = P.radii[d * n1 + r + 1];

    for ( int w = 0; w < 2; ++w )
    {
        T      p[3][3];
        T      kn[6], s[6][3], sp[6][3], nrm[6][3];
        size_t idx[6];
        for ( int n = 0; n < 6; ++n )
        {
            const int X = x + kWedgeNode[w][n][0], Y = y + kWedgeNode[w][n][1], R = r + kWedgeNode[w][n][2];
            const size_t  lat = lat_index( n1, d, X, Y );
            const double* u   = P.coords + lat * 3;
            if ( n < 3 )
                for ( int a = 0; a < 3; ++a )
                    p[n][a] = T( u[a] );
            idx[n] = lat * n1 + R;
            kn[n]  = P.k[idx[n]];
            T nn[3] = { T( u[0] ), T( u[1] ), T( u[2] ) };
            const T mm = sqrt( nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2] );
            for ( int c = 0; c < 3; ++c )
            {
                nrm[n][c] = nn[c] / mm;
                s[n][c] = sp[n][c] = P.src.p[c][idx[n]];
            }
            if ( ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 ) )
                project_out( nrm[n], sp[n] );
        }
        T       IT[3][3];
        const T third = T( 1.0 / 3.0 );
        const T det   = wedge_jacobian_it( p[0], p[1], p[2], r0, r1, third, third, T( 0 ), IT );
        T       ksum  = 0;
        for ( int n = 0; n < 6; ++n )
            ksum += kn[n];
        const T kwJ = ( ksum / T( 6 ) ) * fabs( det );
        T       g[6][3];
        for ( int n = 0; n < 6; ++n )
        {
            T gr[3];
            grad_shape_ref( n, third, third, T( 0 ), gr );
            for ( int a = 0; a < 3; ++a )
                g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
        }
        if ( !diag )
        {
            T G[3][3] = { { 0 } };
            for ( int n = 0; n < 6; ++n )
            {
                if ( ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 ) )
                    continue;
                for ( int a = 0; a < 3; ++a )
                    for ( int bb = 0; bb < 3; ++bb )
                        G[a][bb] += g[n][a] * sp[n][bb];
            }
            const T div = G[0][0] + G[1][1] + G[2][2];
            T       E[3][3];
            for ( int a = 0; a < 3; ++a )
                for ( int bb = 0; bb < 3; ++bb )
                    E[a][bb] = T( 0.5 ) * ( G[a][bb] + G[bb][a] );
            for ( int n = 0; n < 6; ++n )
            {
                if ( ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 ) )
                    continue;
                T* o = acc[kWedgeNode[w][n][0]][kWedgeNode[w][n][1]][kWedgeNode[w][n][2]];
                for ( int c = 0; c < 3; ++c )
                    o[c] += kwJ * ( T( 2 ) * ( g[n][0] * E[0][c] + g[n][1] * E[1][c] + g[n][2] * E[2][c] ) -
                                    T( 2.0 / 3.0 ) * g[n][c] * div );
                if ( ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 ) )
                {
                    const T gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
                    const T ng = nrm[n][0] * g[n][0] + nrm[n][1] * g[n][1] + nrm[n][2] * g[n][2];
                    ann[kWedgeNode[w][n][0]][kWedgeNode[w][n][1]][kWedgeNode[w][n][2]] += kwJ * ( gg + ng * ng * third );
                }
            }
        }
        for ( int n = 0; n < 6; ++n )
        {
            const bool is_dir = ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 );
            const bool is_fs  = ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 );
            if ( !( diag || is_dir ) )
                continue;
            T*      o  = acc[kWedgeNode[w][n][0]][kWedgeNode[w][n][1]][kWedgeNode[w][n][2]];
            const T gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
            if ( diag && is_fs )
            {
                T R[3][3], v[3];
                trafo_normal_tangential( nrm[n], R );
                for ( int a = 0; a < 3; ++a )
                {
                    const T Rg = R[a][0] * g[n][0] + R[a][1] * g[n][1] + R[a][2] * g[n][2];
                    const T Rs = R[a][0] * s[n][0] + R[a][1] * s[n][1] + R[a][2] * s[n][2];
                    v[a]       = kwJ * ( gg + Rg * Rg * third ) * Rs;
                }
                for ( int c = 0; c < 3; ++c )
                    o[c] += R[0][c] * v[0] + R[1][c] * v[1] + R[2][c] * v[2];
            }
            else
            {
                for ( int c = 0; c < 3; ++c )
                    o[c] += kwJ * s[n][c] * ( gg + g[n][c] * g[n][c] * third );
            }
        }
    }
    if ( !diag && ( cmb_fs || surf_fs ) )
    {
        const int dr = cmb_fs ? 0 : 1;
        for ( int dx = 0; dx < 2; ++dx )
            for ( int dy = 0; dy < 2; ++dy )
            {
                const size_t  lat = lat_index( n1, d, x + dx, y + dy );
                const double* u   = P.coords + lat * 3;
                T             n[3] = { T( u[0] ), T( u[1] ), T( u[2] ) };
                const T       mm   = sqrt( n[0] * n[0] + n[1] * n[1] + n[2] * n[2] );
                n[0] /= mm, n[1] /= mm, n[2] /= mm;
                T* o = acc[dx][dy][dr];
                project_out( n, o );
                const size_t i  = lat * n1 + r + dr;
                const T      un = n[0] * P.src.p[0][i] + n[1] * P.src.p[1][i] + n[2] * P.src.p[2][i];
                for ( int c = 0; c < 3; ++c )
                    o[c] += ann[dx][dy][dr] * un * n[c];
            }
    }
    for ( int dx = 0; dx < 2; ++dx )
        for ( int dy = 0; dy < 2; ++dy )
            for ( int dr = 0; dr < 2; ++dr )
            {
                const size_t i = lat_index( n1, d, x + dx, y + dy ) * n1 + r + dr;
                for ( int c = 0; c < 3; ++c )
                    atomicAdd( P.dst.p[c] + i, acc[dx][dy][dr][c] );
            }
}

// ---------------------------------------------------------------------------
// fs/fs rigid-rotation penalty (kerngen :287-408, :585-606).  The reference
// orthonormalises m_i = tangential part of (x x e_i) with owned-masked dot
// products and adds eps sum_i (m_i . src) m_i.  Rotation fields are tangential
// to every shell, so the projection is the identity, and with m = C raw,
// C^T C = Gram^{-1}: the update is beta x x with beta = eps Gram^{-1} b,
// b = sum_owned x x src.
struct Mat3
{
    double a[9];
};

template < typename T >
__global__ void penalty_dots_kernel( size_t ns, int n1, const double* __restrict__ coords, const T* __restrict__ radii,
                                     Ptr3< const T > src, const uint8_t* __restrict__ lat_owned, double* partials, unsigned int* counter, double* result )
{
    Neumaier acc[3];
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        const size_t lat = i / n1;
        if ( !lat_owned[lat] )
            continue;
        const int     r  = int( i - lat * n1 );
        const int     d  = int( lat / ( size_t( n1 ) * n1 ) );
        const double  rr = double( radii[d * n1 + r] );
        const double* u  = coords + lat * 3;
        const double  x[3] = { u[0] * rr, u[1] * rr, u[2] * rr };
        const double  v[3] = { double( src.p[0][i] ), double( src.p[1][i] ), double( src.p[2][i] ) };
        acc[0].add( x[1] * v[2] - x[2] * v[1] );
        acc[1].add( x[2] * v[0] - x[0] * v[2] );
        acc[2].add( x[0] * v[1] - x[1] * v[0] );
    }
    block_sum_finish< 3 >( acc, partials, counter, result );
}

__global__ void penalty_beta_kernel( double eps, Mat3 ginv, double* result )
{
    const double b0 = result[0], b1 = result[1], b2 = result[2];
    result[3]       = eps * ( ginv.a[0] * b0 + ginv.a[1] * b1 + ginv.a[2] * b2 );
    result[4]       = eps * ( ginv.a[3] * b0 + ginv.a[4] * b1 + ginv.a[5] * b2 );
    result[5]       = eps * ( ginv.a[6] * b0 + ginv.a[7] * b1 + ginv.a[8] * b2 );
}

template < typename T >
__global__ void penalty_axpy_kernel( size_t ns, int n1, const double* __restrict__ coords, const T* __restrict__ radii,
                                     const double* beta, Ptr3< T > dst )
{
    const double b[3] = { beta[0], beta[1], beta[2] };
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        const size_t  lat = i / n1;
        const int     r   = int( i - lat * n1 );
        const int     d   = int( lat / ( size_t( n1 ) * n1 ) );
        const double  rr  = double( radii[d * n1 + r] );
        const double* u   = coords + lat * 3;
        const double  x[3] = { u[0] * rr, u[1] * rr, u[2] * rr };
        dst.p[0][i] += T( b[1] * x[2] - b[2] * x[1] );
        dst.p[1][i] += T( b[2] * x[0] - b[0] * x[2] );
        dst.p[2][i] += T( b[0] * x[1] - b[1] * x[0] );
    }
}

template < typename T >
const T* mesh_radii( const tn_mesh* m );
template <>
const double* mesh_radii< double >( const tn_mesh* m )
{
    return m->d_radii;
}
template <>
const float* mesh_radii< float >( const tn_mesh* m )
{
    return m->d_radii32;
}

template < typename T >
int launch_cells( const tn_mesh* m, const tn_epsdivdiv_params* p, const T* k, Ptr3< const T > src, Ptr3< T > dst,
                  int layers, cudaStream_t st )
{
    CellParams< T > C{ m->N, m->n1, m->d_coords, mesh_radii< T >( m ), k, src, dst, p->bc_cmb, p->bc_surface,
                       p->diagonal, layers };
    const int       nr    = layers == 0 ? m->N : ( layers == 3 ? 2 : 1 );
    const long long cells = (long long) kDiamonds * m->N * m->N * nr;
    kerngen_cell_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( C );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

}  // namespace

template < typename T >
int epsdivdiv_apply( const tn_mesh* m, const tn_epsdivdiv_params* p, const T* k, const T* const* src, T* const* dst,
                     cudaStream_t st )
{
    TN_CHECK_ARG( m && p && k && src && dst, "epsdivdiv_apply: null argument" );
    for ( int c = 0; c < 3; ++c )
        TN_CHECK_ARG( src[c] && dst[c], "epsdivdiv_apply: null vector component" );
    TN_CHECK_ARG( p->bc_cmb >= 0 && p->bc_cmb <= 2 && p->bc_surface >= 0 && p->bc_surface <= 2,
                  "epsdivdiv_apply: boundary condition codes must be 0, 1 or 2" );
    TN_CHECK_ARG( p->apply_mode == TN_APPLY_REPLACE || p->apply_mode == TN_APPLY_ADD, "epsdivdiv_apply: bad apply mode" );
    TN_CHECK_ARG( p->comm_mode == TN_COMM_SKIP || p->comm_mode == TN_COMM_ADDITIVE, "epsdivdiv_apply: bad comm mode" );
    Ptr3< const T > s{ { src[0], src[1], src[2] } };
    Ptr3< T >       o{ { dst[0], dst[1], dst[2] } };
    const bool      fsfs = !p->diagonal && p->bc_cmb == TN_BC_FREESLIP && p->bc_surface == TN_BC_FREESLIP;
    const int       N    = m->N;

    if ( fsfs )
    {
        Mat3 gi;
        for ( int i = 0; i < 9; ++i )
            gi.a[i] = m->penalty_gram_inv[i];
        const unsigned blocks = unsigned( std::min< size_t >( ( m->ns + 1023 ) / 1024, kRedMaxBlocks ) );
        penalty_dots_kernel< T ><<< blocks, 256, 0, st >>>( m->ns, m->n1, m->d_coords, mesh_radii< T >( m ), s,
                                                           m->d_lat_owned, m->d_red_partials,
                                                           m->d_red_counter, m->d_red_result );
        TN_LAUNCH_CHECK();
        penalty_beta_kernel<<< 1, 1, 0, st >>>( p->penalty_eps, gi, m->d_red_result );
        TN_LAUNCH_CHECK();
    }

    if ( p->diagonal || N < kTile )
    {
        if ( p->apply_mode == TN_APPLY_REPLACE )
            for ( int c = 0; c < 3; ++c )
                TN_CUDA_TRY( cudaMemsetAsync( dst[c], 0, m->ns * sizeof( T ), st ) );
        int rc = launch_cells< T >( m, p, k, s, o, 0, st );
        if ( rc )
            return rc;
        if ( fsfs )
        {
            penalty_axpy_kernel< T ><<< 148 * 8, 256, 0, st >>>( m->ns, m->n1, m->d_coords, mesh_radii< T >( m ),
                                                                m->d_red_result + 3, o );
            TN_LAUNCH_CHECK();
        }
    }
    else
    {
        const bool      skip_cmb = p->bc_cmb != TN_BC_NEUMANN, skip_surf = p->bc_surface != TN_BC_NEUMANN;
        TileParams< T > P{ N,
                           m->n1,
                           N / kTile,
                           m->d_coords,
                           mesh_radii< T >( m ),
                           k,
                           s,
                           o,
                           p->apply_mode == TN_APPLY_ADD,
                           skip_cmb,
                           skip_surf,
                           fsfs ? m->d_red_result + 3 : nullptr };
        const size_t smem = tile_smem_bytes< T >( m->n1 );
        static bool  attr_set[2] = { false, false };
        if ( !attr_set[sizeof( T ) == 8] )
        {
            TN_CUDA_TRY( cudaFuncSetAttribute( kerngen_tile_kernel< T >, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int( smem ) + 8192 ) );
            attr_set[sizeof( T ) == 8] = true;
        }
        const unsigned blocks = unsigned( kDiamonds * ( N / kTile ) * ( N / kTile ) );
        kerngen_tile_kernel< T ><<< blocks, kThreads, smem, st >>>( P );
        TN_LAUNCH_CHECK();
        if ( skip_cmb || skip_surf )
        {
            int rc = launch_cells< T >( m, p, k, s, o, skip_cmb && skip_surf ? 3 : ( skip_cmb ? 1 : 2 ), st );
            if ( rc )
                return rc;
        }
    }
    if ( p->comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( m, dst, 3, st );
    return TN_OK;
}

}  // namespace tn

using namespace tn;

extern "C" int tn_epsdivdiv_apply_f64( const tn_mesh* m, const tn_epsdivdiv_params* p, const double* k,
                                       const double* const* src, double* const* dst, void* s )
{
    return epsdivdiv_apply< double >( m, p, k, src, dst, as_stream( s ) );
}
extern "C" int tn_epsdivdiv_apply_f32( const tn_mesh* m, const tn_epsdivdiv_params* p, const float* k,
                                       const float* const* src, float* const* dst, void* s )
{
    return epsdivdiv_apply< float >( m, p, k, src, dst, as_stream( s ) );
}
