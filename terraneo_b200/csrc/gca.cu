// Stored wedge matrices and Galerkin coarse-grid approximation (GCA) of the
// epsilon-div-div operator.
//
//  * local matrices: the one-point kerngen 18x18 wedge matrix
//    (fe/wedge/operators/shell/epsilon_divdiv_kerngen.hpp:2051-2110), no
//    boundary treatment, DIMENSIONWISE order (node + 6 dim);
//  * coarsening: TwoGridGCA (linalg/solvers/gca/gca.hpp:154-528): per coarse
//    cell the sum over its 8 fine hexes x 2 wedges of P^T A_fine P, P the 6x6
//    local interpolation (constant or linear weights) applied per dimension;
//  * apply with stored matrices and the boundary treatment of the reference's
//    slow path (epsilon_divdiv_kerngen.hpp:823-1052), the fs/fs penalty and
//    the additive halo.
//
// Storage: the wedge matrices are symmetric (the kerngen form and every
// P^T A P of it) and only the upper triangle is kept, row by row (entry
// (I, J), I <= J, is entry e = 18 I - I (I - 1) / 2 + J - I of 171, plus
// one zero padding entry).  Wedges are numbered w = 2 cell + wedge (cells
// (d, x, y, r), r fastest) and 32 consecutive wedges are interleaved in
// chunks of 4 entries: entry e of wedge w at
// (((w / 32) 43 + e / 4) 32 + w % 32) 4 + e % 4.  FP64 2,752 B per cell.
//
// Coarsening: one 324-thread block per coarse cell, thread t owning entry
// (t / 18, t % 18) of both coarse wedges; the interpolation matrices (and, at
// the finest level, the fine wedges' geometry) of all 16 fine wedges are staged
// in shared memory once, then per fine wedge T = A_f P and C += P^T T are two
// 6-term passes.  Apply: one thread per wedge streams its 43 chunks with
// vector loads (each warp load is 32 x 4 consecutive values) and uses the
// symmetry.
#include <algorithm>

#include <cooperative_groups.h>

#include "common.cuh"
#include "reduce.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );
template < typename T >
int fsfs_penalty_fork( const tn_mesh* m, double eps, const T* const* src, cudaStream_t st );
template < typename T >
int fsfs_penalty_join( const tn_mesh* m, T* const* dst, cudaStream_t st );

namespace {

constexpr int kM          = 324; // entries of an 18 x 18 matrix
constexpr int kP          = 171; // stored entries of a symmetric 18 x 18 matrix

constexpr int kChunks     = 43;  // 4-entry chunks of a wedge (172 entries, the last one padding)

// Position of entry e of wedge w (w = 2 cell + wedge) in a stored array: 32
// consecutive wedges are interleaved in chunks of 4 entries, so a warp with
// one thread per wedge reads one 4-entry chunk per thread and 32 x 4
// consecutive values per vector load.
__host__ __device__ __forceinline__ size_t stored_pos( long long w, int e )
{
    return ( ( size_t( w >> 5 ) * kChunks + size_t( e >> 2 ) ) * 32 + size_t( w & 31 ) ) * 4 + size_t( e & 3 );
}

// position of entry (I, J) in the packed upper triangle
__device__ __forceinline__ int packed( int I, int J )
{
    const int i = I < J ? I : J, j = I < J ? J : I;
    return 18 * i - ( i * ( i - 1 ) ) / 2 + ( j - i );
}
constexpr int kGcaThreads = 352; // 11 warps, threads >= 324 only stage data

// one-point kerngen geometry of wedge w of cell (d, x, y, r): physical
// gradients g and k_eval |det J| (k == NULL: k = 1)
__device__ void kerngen_geometry( const double* __restrict__ coords, const double* __restrict__ radii,
                                  const double* __restrict__ k, int n1, int d, int x, int y, int r, int w,
                                  double g[6][3], double& kwJ )
{
    double p[3][3], ks = 0.0;
    for ( int n = 0; n < 6; ++n )
    {
        const size_t lat = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] );
        if ( n < 3 )
            for ( int a = 0; a < 3; ++a )
                p[n][a] = coords[lat * 3 + a];
        ks += k ? k[lat * n1 + r + kWedgeNode[w][n][2]] : 1.0;
    }
    double       IT[3][3];
    const double third = 1.0 / 3.0;
    const double det   = wedge_jacobian_it( p[0], p[1], p[2], radii[d * n1 + r], radii[d * n1 + r + 1], third, third,
                                            0.0, IT );
    kwJ                = ( ks / 6.0 ) * fabs( det );
    for ( int n = 0; n < 6; ++n )
    {
        double gr[3];
        grad_shape_ref( n, third, third, 0.0, gr );
        for ( int a = 0; a < 3; ++a )
            g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
    }
}

// entry (I, J) of the kerngen wedge matrix:
// kwJ (delta_ab g_i.g_j + g_{i,b} g_{j,a} - 2/3 g_{j,b} g_{i,a}), I = i + 6a, J = j + 6b
__device__ __forceinline__ double kerngen_entry( const double ( *g )[3], double kwJ, int I, int J )
{
    const int    i = I % 6, a = I / 6, j = J % 6, b = J / 6;
    const double gg = a == b ? g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2] : 0.0;
    return kwJ * ( gg + g[i][b] * g[j][a] - ( 2.0 / 3.0 ) * g[j][b] * g[i][a] );
}

// constant prolongation weight (grid_transfer_constant.hpp:25-82)
__device__ __forceinline__ double constant_weight( int xf, int yf, int rf, int xc, int yc, int rc )
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

// row i of the 6x6 local interpolation of fine wedge w of fine hex
// (xh, yh, rh): columns are the local nodes of the coarse wedge holding it
// (gca.hpp:186-366, with its choice of coarse columns per edge type)
__device__ void gca_P_row( int Nf, const double* coords, const double* radii, int d, int xh, int yh, int rh, int w,
                           int i, int mode, double row[6] )
{
    for ( int c = 0; c < 6; ++c )
        row[c] = 0.0;
    const int x = xh + kWedgeNode[w][i][0], y = yh + kWedgeNode[w][i][1], r = rh + kWedgeNode[w][i][2];
    if ( !( x & 1 ) && !( y & 1 ) && !( r & 1 ) )
    {
        row[i] = 1.0;
        return;
    }
    const int rb = r < Nf ? r / 2 : r / 2 - 1, rt = rb + 1;
    int       cx[4], cy[4], cr[4];
    double    wl[4];
    if ( !( x & 1 ) && !( y & 1 ) )
    {
        double w0 = 0.5, w1 = 0.5;
        if ( mode == 1 )
        {
            linear_stencil( Nf, coords, radii, d, x, y, r, cx, cy, cr, wl );
            w0 = wl[0], w1 = wl[1];
        }
        row[i % 3]     = w0;
        row[i % 3 + 3] = w1;
        return;
    }
    int x0, x1, y0, y1, l0, l1, l2, l3;
    if ( !( x & 1 ) )
        x0 = x1 = x / 2, y0 = y / 2, y1 = y / 2 + 1, l0 = 0, l1 = 2, l2 = 3, l3 = 5;
    else if ( !( y & 1 ) )
        x0 = x / 2, x1 = x / 2 + 1, y0 = y1 = y / 2, l0 = 0, l1 = 1, l2 = 3, l3 = 4;
    else
        x0 = x / 2 + 1, x1 = x / 2, y0 = y / 2, y1 = y / 2 + 1, l0 = 1, l1 = 2, l2 = 4, l3 = 5;
    if ( mode == 1 )
    {
        linear_stencil( Nf, coords, radii, d, x, y, r, cx, cy, cr, wl );
        row[l0] = wl[0], row[l1] = wl[0], row[l2] = wl[2], row[l3] = wl[2];
    }
    else
    {
        row[l0] = constant_weight( x, y, r, x0, y0, rb );
        row[l1] = constant_weight( x, y, r, x1, y1, rb );
        row[l2] = constant_weight( x, y, r, x0, y0, rt );
        row[l3] = constant_weight( x, y, r, x1, y1, rt );
    }
}

// coarse wedge holding fine wedge w of fine hex h (hex order x, y, r bits)
__device__ __forceinline__ int gca_coarse_wedge( int h, int w )
{
    if ( w == 0 )
        return ( h == 3 || h == 7 ) ? 1 : 0;
    return ( h == 0 || h == 4 ) ? 0 : 1;
}

// the coarsest-grid ancestor (x, y, r) >> lr of a cell is marked (GCAElements, gca.hpp:155-163)
__device__ __forceinline__ bool agca_marked( const uint8_t* marks, int N, int lr, int d, int x, int y, int r )
{
    const int N0 = N >> lr;
    return marks[( ( size_t( d ) * N0 + ( x >> lr ) ) * N0 + ( y >> lr ) ) * N0 + ( r >> lr )] != 0;
}

// marks: nullptr for every cell, else only the cells whose coarsest ancestor is not marked (the elements the
// adaptive GCA leaves to the re-discretised operator)
__global__ void __launch_bounds__( 64 ) local_matrices_kernel( int N, const double* __restrict__ coords,
                                                               const double* __restrict__ radii,
                                                               const double* __restrict__ k, double* __restrict__ mats,
                                                               const uint8_t* __restrict__ marks, int lr )
{
    __shared__ double sg[2][6][3], skw[2];
    const long long   cell = blockIdx.x;
    const int         n1   = N + 1;
    const int         r = int( cell % N ), y = int( ( cell / N ) % N ), x = int( ( cell / ( (long long) N * N ) ) % N );
    const int         d = int( cell / ( (long long) N * N * N ) );
    if ( marks && agca_marked( marks, N, lr, d, x, y, r ) )
        return; // uniform over the block: one cell per block
    if ( threadIdx.x < 2 )
        kerngen_geometry( coords, radii, k, n1, d, x, y, r, threadIdx.x, sg[threadIdx.x], skw[threadIdx.x] );
    __syncthreads();
    for ( int e = threadIdx.x; e < 2 * kM; e += blockDim.x )
    {
        const int w = e / kM, I = ( e % kM ) / 18, J = ( e % kM ) % 18;
        if ( I <= J )
            mats[stored_pos( cell * 2 + w, packed( I, J ) )] = kerngen_entry( sg[w], skw[w], I, J );
        if ( I == 17 && J == 17 )
            mats[stored_pos( cell * 2 + w, kP )] = 0.0; // padding entry
    }
}

// GCAElementsCollector (gca_elements_collector.hpp:59-94): one thread per fine cell; a wedge whose nodal
// viscosity has a reference-coordinate gradient of norm > 10 at the centroid (1/3, 1/3, 0) marks the coarsest
// cell (x, y, r) >> lr.  Concurrent writers store the same value.
__global__ void gca_elements_kernel( int N, int lr, const double* __restrict__ k, uint8_t* marks )
{
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int n1 = N + 1;
    const int r = int( t % N ), y = int( ( t / N ) % N ), x = int( ( t / ( (long long) N * N ) ) % N );
    const int d = int( t / ( (long long) N * N * N ) );
#pragma unroll
    for ( int w = 0; w < 2; ++w )
    {
        double kg[3] = { 0, 0, 0 };
#pragma unroll
        for ( int j = 0; j < 6; ++j )
        {
            double g[3];
            grad_shape_ref( j, 1.0 / 3.0, 1.0 / 3.0, 0.0, g );
            const double kj = k[lat_index( n1, d, x + wedge_node( w, j, 0 ), y + wedge_node( w, j, 1 ) ) * n1 + r +
                                wedge_node( w, j, 2 )];
#pragma unroll
            for ( int a = 0; a < 3; ++a )
                kg[a] = kg[a] + g[a] * kj;
        }
        if ( sqrt( kg[0] * kg[0] + kg[1] * kg[1] + kg[2] * kg[2] ) > 10.0 )
        {
            const int N0 = N >> lr;
            marks[( ( size_t( d ) * N0 + ( x >> lr ) ) * N0 + ( y >> lr ) ) * N0 + ( r >> lr )] = 1;
        }
    }
}

template < bool FROM_K >
__global__ void __launch_bounds__( kGcaThreads ) gca_coarsen_kernel( int Nf, const double* __restrict__ coords,
                                                                   const double* __restrict__ radii,
                                                                   const double* __restrict__ k,
                                                                   const double* __restrict__ mats_f, int mode,
                                                                   double* __restrict__ mats_c )
{
    __shared__ double sP[16][6][6];
    __shared__ double sG[16][6][3];
    __shared__ double sK[16];
    __shared__ double sA[kM];
    __shared__ double sT[kM];
    __shared__ int    sCW[16];
    const int         Nc = Nf / 2, n1 = Nf + 1;
    const long long   cell = blockIdx.x;
    const int rc = int( cell % Nc ), yc = int( ( cell / Nc ) % Nc ), xc = int( ( cell / ( (long long) Nc * Nc ) ) % Nc );
    const int d  = int( cell / ( (long long) Nc * Nc * Nc ) );
    const int t  = threadIdx.x;
    if ( t < 96 )
    {
        const int fw = t / 6, i = t % 6, h = fw >> 1, w = fw & 1;
        gca_P_row( Nf, coords, radii, d, 2 * xc + ( h & 1 ), 2 * yc + ( ( h >> 1 ) & 1 ), 2 * rc + ( h >> 2 ), w, i,
                   mode, sP[fw][i] );
    }
    else if ( t < 112 )
    {
        const int fw = t - 96, h = fw >> 1, w = fw & 1;
        sCW[fw] = gca_coarse_wedge( h, w );
        if ( FROM_K )
            kerngen_geometry( coords, radii, k, n1, d, 2 * xc + ( h & 1 ), 2 * yc + ( ( h >> 1 ) & 1 ),
                              2 * rc + ( h >> 2 ), w, sG[fw], sK[fw] );
    }
    __syncthreads();
    const bool live = t < kM;
    const int  I = live ? t / 18 : 0, J = live ? t % 18 : 0;
    const int  i = I % 6, a = I / 6, j = J % 6, b = J / 6;
    double     acc0 = 0.0, acc1 = 0.0;
    for ( int fw = 0; fw < 16; ++fw )
    {
        if ( !FROM_K )
        {
            const int       h = fw >> 1, w = fw & 1;
            const int       xh = 2 * xc + ( h & 1 ), yh = 2 * yc + ( ( h >> 1 ) & 1 ), rh = 2 * rc + ( h >> 2 );
            const long long cf = ( ( (long long) d * Nf + xh ) * Nf + yh ) * Nf + rh;
            if ( live )
                sA[I * 18 + J] = mats_f[stored_pos( cf * 2 + w, packed( I, J ) )];
            __syncthreads();
        }
        // T(I, J) = sum_n A(I, n + 6b) P(n, j)
        if ( live )
        {
            double v = 0.0;
            for ( int n = 0; n < 6; ++n )
            {
                const double A = FROM_K ? kerngen_entry( sG[fw], sK[fw], I, n + 6 * b ) : sA[I * 18 + n + 6 * b];
                v += A * sP[fw][n][j];
            }
            sT[I * 18 + J] = v;
        }
        __syncthreads();
        // C(I, J) += sum_m P(m, i) T(m + 6a, J)
        if ( live )
        {
            double v = 0.0;
            for ( int m = 0; m < 6; ++m )
                v += sP[fw][m][i] * sT[( m + 6 * a ) * 18 + J];
            if ( sCW[fw] == 0 )
                acc0 += v;
            else
                acc1 += v;
        }
        __syncthreads();
    }
    if ( live && I <= J )
    {
        mats_c[stored_pos( cell * 2 + 0, packed( I, J ) )] = acc0;
        mats_c[stored_pos( cell * 2 + 1, packed( I, J ) )] = acc1;
        if ( I == 17 && J == 17 )
            mats_c[stored_pos( cell * 2 + 0, kP )] = mats_c[stored_pos( cell * 2 + 1, kP )] = 0.0;
    }
}

__device__ __forceinline__ void load4( const float* p, float v[4] )
{
    const float4 q = __ldg( reinterpret_cast< const float4* >( p ) );
    v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
}
__device__ __forceinline__ void load4( const double* p, double v[4] )
{
    const double2 a = __ldg( reinterpret_cast< const double2* >( p ) );
    const double2 b = __ldg( reinterpret_cast< const double2* >( p ) + 1 );
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
}

// outward unit normal at a lateral node (x / |x|, in the precision of the
// apply; one reciprocal square root instead of a root and three divisions)
__device__ __forceinline__ void unit_normal_of( const double* __restrict__ coords, int n1, int d, int X, int Y,
                                                double n[3] )
{
    const double* c  = coords + lat_index( n1, d, X, Y ) * 3;
    const double  im = rsqrt( c[0] * c[0] + c[1] * c[1] + c[2] * c[2] );
    n[0] = c[0] * im, n[1] = c[1] * im, n[2] = c[2] * im;
}
__device__ __forceinline__ void unit_normal_of( const double* __restrict__ coords, int n1, int d, int X, int Y,
                                                float n[3] )
{
    const double* c  = coords + lat_index( n1, d, X, Y ) * 3;
    const float   c0 = float( c[0] ), c1 = float( c[1] ), c2 = float( c[2] );
    const float   im = rsqrtf( c0 * c0 + c1 * c1 + c2 * c2 );
    n[0] = c0 * im, n[1] = c1 * im, n[2] = c2 * im;
}

template < typename T >
struct StoredParams
{
    int             N, n1;
    const double*   coords;
    const T*        mats;
    Ptr3< const T > src;
    Ptr3< T >       dst;
    int             bc_cmb, bc_surf, diag;
    const double*   gate; // skip the launch when *gate != 0 (the PCG stopping flag), or NULL
};

// One thread per wedge (w = 2 cell + wedge).  The 171 stored values stream
// in with compile-time offsets (fully unrolled), each contributing to rows I
// and J by symmetry; the boundary treatment follows the slow path.
template < typename T, bool DIAG >
__device__ __forceinline__ void stored_wedge( const StoredParams< T >& P, long long gw )
{
    const int       N = P.N, n1 = P.n1;
    const long long cell = gw >> 1;
    const int       w    = int( gw & 1 );
    const int r = int( cell % N ), y = int( ( cell / N ) % N ), x = int( ( cell / ( (long long) N * N ) ) % N );
    const int d = int( cell / ( (long long) N * N * N ) );
    const bool at_cmb = r == 0, at_surf = r == N - 1;
    const int  bcf    = at_cmb ? P.bc_cmb : ( at_surf ? P.bc_surf : TN_BC_NEUMANN );
    const int  boff   = at_cmb ? 0 : 3; // boundary-side local nodes boff..boff+2
    const bool dir = bcf == TN_BC_DIRICHLET, fs = bcf == TN_BC_FREESLIP;

    size_t idx[6];
    T      s[18], nrm[3][3], sn[3] = { 0, 0, 0 };
    bool   bn[6];
#pragma unroll
    for ( int n = 0; n < 6; ++n )
    {
        const size_t lat = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] );
        idx[n]           = lat * n1 + r + kWedgeNode[w][n][2];
        bn[n]            = bcf != TN_BC_NEUMANN && n >= boff && n < boff + 3;
#pragma unroll
        for ( int a = 0; a < 3; ++a )
            s[n + 6 * a] = P.src.p[a][idx[n]];
    }
    if ( fs )
    {
#pragma unroll
        for ( int q = 0; q < 3; ++q )
        {
            const int     n  = boff + q;
            const double* c  = P.coords + lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * 3;
            const double  mm = sqrt( c[0] * c[0] + c[1] * c[1] + c[2] * c[2] );
            for ( int a = 0; a < 3; ++a )
                nrm[q][a] = T( c[a] / mm );
            sn[q] = nrm[q][0] * s[n] + nrm[q][1] * s[n + 6] + nrm[q][2] * s[n + 12];
        }
    }
    const T* gm = P.mats + stored_pos( gw, 0 ); // chunk c at gm + 128 c
    T        yv[18];
#pragma unroll
    for ( int I = 0; I < 18; ++I )
        yv[I] = T( 0 );

    if ( !DIAG )
    {
        // free-slip: boundary nodes enter with their tangential part
        T sv[18];
#pragma unroll
        for ( int I = 0; I < 18; ++I )
            sv[I] = s[I];
        if ( fs )
        {
#pragma unroll
            for ( int q = 0; q < 3; ++q )
#pragma unroll
                for ( int a = 0; a < 3; ++a )
                {
                    // boff is 0 or 3: select the node without dynamic indexing
                    const T t0 = sv[q + 6 * a] - sn[q] * nrm[q][a], t3 = sv[q + 3 + 6 * a] - sn[q] * nrm[q][a];
                    if ( boff == 0 )
                        sv[q + 6 * a] = t0;
                    else
                        sv[q + 3 + 6 * a] = t3;
                }
        }
        T ann[3] = { 0, 0, 0 };
        constexpr int kRing = 8; // vector-register ring, each chunk loaded kRing chunks ahead
        T             ring[kRing][4];
#pragma unroll
        for ( int c = 0; c < kRing; ++c )
            load4( gm + 128 * c, ring[c] );
#pragma unroll
        for ( int I = 0; I < 18; ++I )
#pragma unroll
            for ( int J = I; J < 18; ++J )
            {
                const int e = 18 * I - ( I * ( I - 1 ) ) / 2 + J - I;
                const T   v = ring[( e >> 2 ) % kRing][e & 3];
                if ( ( e & 3 ) == 3 && ( e >> 2 ) + kRing < kChunks )
                    load4( gm + 128 * ( ( e >> 2 ) + kRing ), ring[( e >> 2 ) % kRing] );
                const int ni = I % 6, nj = J % 6, a = I / 6, b = J / 6;
                bool      keep = true;
                if ( dir )
                    keep = ( a == b ) ? !( ni != nj && ( bn[ni] || bn[nj] ) ) : !( bn[ni] || bn[nj] );
                if ( keep )
                {
                    yv[I] += v * sv[J];
                    if ( I != J )
                        yv[J] += v * sv[I];
                }
                if ( fs && ni == nj && bn[ni] )
                {
                    // (n^T A_nn n) of boundary node ni, both triangles
                    const int q   = ni - boff;
                    const T   f   = ( I == J ? T( 1 ) : T( 2 ) ) * v;
                    const T   nab = q == 0 ? nrm[0][a] * nrm[0][b] : ( q == 1 ? nrm[1][a] * nrm[1][b] : nrm[2][a] * nrm[2][b] );
                    if ( q == 0 )
                        ann[0] += f * nab;
                    else if ( q == 1 )
                        ann[1] += f * nab;
                    else
                        ann[2] += f * nab;
                }
            }
        if ( fs )
        {
#pragma unroll
            for ( int q = 0; q < 3; ++q )
            {
                const int n0 = q, n3 = q + 3; // candidates for boff = 0 / 3
                T         y3[3];
                for ( int a = 0; a < 3; ++a )
                    y3[a] = boff == 0 ? yv[n0 + 6 * a] : yv[n3 + 6 * a];
                const T yn = nrm[q][0] * y3[0] + nrm[q][1] * y3[1] + nrm[q][2] * y3[2];
                for ( int a = 0; a < 3; ++a )
                {
                    const T v = y3[a] - yn * nrm[q][a] + ann[q] * sn[q] * nrm[q][a];
                    if ( boff == 0 )
                        yv[n0 + 6 * a] = v;
                    else
                        yv[n3 + 6 * a] = v;
                }
            }
        }
    }
    else
    {
        // diagonal; free-slip boundary nodes: diagonal of R A R^T rotated back
        T blk[3][3][3];
#pragma unroll
        for ( int I = 0; I < 18; ++I )
#pragma unroll
            for ( int J = I; J < 18; ++J )
            {
                const int ni = I % 6, nj = J % 6;
                if ( ni != nj )
                    continue;
                const int e = 18 * I - ( I * ( I - 1 ) ) / 2 + J - I;
                const T   v = gm[128 * ( e >> 2 ) + ( e & 3 )];
                const int a = I / 6, b = J / 6;
                if ( I == J )
                    yv[I] = v * s[I];
                if ( fs )
                {
                    const int q = ni < 3 ? ni : ni - 3;
                    if ( ( ni < 3 ) == ( boff == 0 ) )
                    {
                        blk[q][a][b] = v;
                        blk[q][b][a] = v;
                    }
                }
            }
        if ( fs )
        {
#pragma unroll
            for ( int q = 0; q < 3; ++q )
            {
                T R[3][3];
                trafo_normal_tangential( nrm[q], R );
                T s3[3], o3[3] = { 0, 0, 0 };
                for ( int a = 0; a < 3; ++a )
                    s3[a] = boff == 0 ? s[q + 6 * a] : s[q + 3 + 6 * a];
                for ( int k = 0; k < 3; ++k )
                {
                    T rar = T( 0 );
                    for ( int b = 0; b < 3; ++b )
                        for ( int c = 0; c < 3; ++c )
                            rar += R[k][b] * blk[q][b][c] * R[k][c];
                    const T rs = R[k][0] * s3[0] + R[k][1] * s3[1] + R[k][2] * s3[2];
                    for ( int a = 0; a < 3; ++a )
                        o3[a] += R[k][a] * rar * rs;
                }
                for ( int a = 0; a < 3; ++a )
                {
                    if ( boff == 0 )
                        yv[q + 6 * a] = o3[a];
                    else
                        yv[q + 3 + 6 * a] = o3[a];
                }
            }
        }
    }
#pragma unroll
    for ( int n = 0; n < 6; ++n )
#pragma unroll
        for ( int a = 0; a < 3; ++a )
            atomicAdd( P.dst.p[a] + idx[n], yv[n + 6 * a] );
}

// Diagonal mode, every wedge.
template < typename T >
__global__ void __launch_bounds__( 128 ) stored_diag_kernel( StoredParams< T > P )
{
    const long long gw = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( gw < 2LL * kDiamonds * P.N * P.N * P.N )
        stored_wedge< T, true >( P, gw );
}

// Non-diagonal apply, one thread per wedge.  The 43 chunks stream through a
// ring of kRing vector registers, each loaded kRing chunks ahead of its use,
// so every warp keeps kRing x 512 (FP32) or 1024 (FP64) bytes in flight.
// The boundary treatment of the slow path is expressed around the plain
// symmetric product, so every lane runs the same instruction stream:
//  * Dirichlet: the boundary-node inputs are zeroed, so interior rows see
//    only interior couplings, and afterwards the boundary rows are replaced
//    by their diagonal entry times the input;
//  * free-slip: the boundary-node inputs enter with their tangential part,
//    the boundary rows are projected on the tangent plane afterwards and
//    get n (n^T A_nn n)(n . s) back, A_nn the node's 3x3 block.
// The diagonal blocks of the three boundary-side nodes are picked up from
// the stream as it passes (compile-time positions, runtime side select).
template < typename T >
__global__ void __launch_bounds__( 128, sizeof( T ) == 4 ? 5 : 2 ) stored_apply_kernel( StoredParams< T > P )
{
    const long long gw = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const int       N = P.N, n1 = P.n1;
    if ( gw >= 2LL * kDiamonds * N * N * N || ( P.gate && *P.gate != 0.0 ) )
        return;
    const long long cell = gw >> 1;
    const int       w    = int( gw & 1 );
    const int r = int( cell % N ), y = int( ( cell / N ) % N ), x = int( ( cell / ( (long long) N * N ) ) % N );
    const int d = int( cell / ( (long long) N * N * N ) );
    const int bcf = r == 0 ? P.bc_cmb : ( r == N - 1 ? P.bc_surf : TN_BC_NEUMANN );
    const bool top = r != 0; // boundary-side nodes 3..5 (SURFACE) rather than 0..2 (CMB)
    const bool dir = bcf == TN_BC_DIRICHLET, fs = bcf == TN_BC_FREESLIP;

    T sv[18], yv[18], sn[3] = { 0, 0, 0 };
#pragma unroll
    for ( int n = 0; n < 6; ++n )
    {
        const size_t i = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * n1 + r +
                         kWedgeNode[w][n][2];
#pragma unroll
        for ( int a = 0; a < 3; ++a )
            sv[n + 6 * a] = P.src.p[a][i];
    }
    // boundary-side node q of the wedge is node q + 3 top (nodes q and q + 3
    // share the lateral position); selects keep every index compile-time
    if ( dir || fs )
    {
#pragma unroll
        for ( int q = 0; q < 3; ++q )
        {
            T nn[3] = { 0, 0, 0 };
            if ( fs )
                unit_normal_of( P.coords, n1, d, x + kWedgeNode[w][q][0], y + kWedgeNode[w][q][1], nn );
            T b3[3];
#pragma unroll
            for ( int a = 0; a < 3; ++a )
                b3[a] = top ? sv[q + 3 + 6 * a] : sv[q + 6 * a];
            sn[q] = nn[0] * b3[0] + nn[1] * b3[1] + nn[2] * b3[2];
#pragma unroll
            for ( int a = 0; a < 3; ++a )
            {
                const T t = dir ? T( 0 ) : b3[a] - sn[q] * nn[a];
                if ( top )
                    sv[q + 3 + 6 * a] = t;
                else
                    sv[q + 6 * a] = t;
            }
        }
    }
#pragma unroll
    for ( int I = 0; I < 18; ++I )
        yv[I] = T( 0 );
    T blk[3][6]; // boundary-side node q: (a, b) = 00 01 02 11 12 22
#pragma unroll
    for ( int q = 0; q < 3; ++q )
#pragma unroll
        for ( int i = 0; i < 6; ++i )
            blk[q][i] = T( 0 );
    const T*      gm    = P.mats + stored_pos( gw, 0 ); // chunk c at gm + 128 c
    constexpr int kRing = 8;
    T             ring[kRing][4];
#pragma unroll
    for ( int c = 0; c < kRing; ++c )
        load4( gm + 128 * c, ring[c] );
#pragma unroll
    for ( int I = 0; I < 18; ++I )
#pragma unroll
        for ( int J = I; J < 18; ++J )
        {
            const int e = 18 * I - ( I * ( I - 1 ) ) / 2 + J - I;
            const T   v = ring[( e >> 2 ) % kRing][e & 3];
            if ( ( e & 3 ) == 3 && ( e >> 2 ) + kRing < kChunks )
                load4( gm + 128 * ( ( e >> 2 ) + kRing ), ring[( e >> 2 ) % kRing] );
            yv[I] += v * sv[J];
            if ( I != J )
                yv[J] += v * sv[I];
            if ( I % 6 == J % 6 )
            {
                const int n = I % 6, a = I / 6, b = J / 6;
                const int ab = a == 0 ? b : ( a == 1 ? 2 + b : 5 );
                if ( ( n >= 3 ) == top )
                    blk[n % 3][ab] = v;
            }
        }
    if ( dir || fs )
    {
#pragma unroll
        for ( int q = 0; q < 3; ++q )
        {
            const T* B = blk[q];
            T        y3[3];
#pragma unroll
            for ( int a = 0; a < 3; ++a )
                y3[a] = top ? yv[q + 3 + 6 * a] : yv[q + 6 * a];
            if ( dir )
            {
                const int    X = x + kWedgeNode[w][q][0], Y = y + kWedgeNode[w][q][1];
                const size_t i = lat_index( n1, d, X, Y ) * n1 + r + ( top ? 1 : 0 );
                y3[0]          = B[0] * P.src.p[0][i];
                y3[1]          = B[3] * P.src.p[1][i];
                y3[2]          = B[5] * P.src.p[2][i];
            }
            else
            {
                T nn[3];
                unit_normal_of( P.coords, n1, d, x + kWedgeNode[w][q][0], y + kWedgeNode[w][q][1], nn );
                const T ann = nn[0] * nn[0] * B[0] + nn[1] * nn[1] * B[3] + nn[2] * nn[2] * B[5] +
                              T( 2 ) * ( nn[0] * nn[1] * B[1] + nn[0] * nn[2] * B[2] + nn[1] * nn[2] * B[4] );
                const T yn = nn[0] * y3[0] + nn[1] * y3[1] + nn[2] * y3[2];
#pragma unroll
                for ( int a = 0; a < 3; ++a )
                    y3[a] += ( ann * sn[q] - yn ) * nn[a];
            }
#pragma unroll
            for ( int a = 0; a < 3; ++a )
            {
                if ( top )
                    yv[q + 3 + 6 * a] = y3[a];
                else
                    yv[q + 6 * a] = y3[a];
            }
        }
    }
#pragma unroll
    for ( int n = 0; n < 6; ++n )
    {
        const size_t i = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * n1 + r +
                         kWedgeNode[w][n][2];
#pragma unroll
        for ( int a = 0; a < 3; ++a )
            atomicAdd( P.dst.p[a] + i, yv[n + 6 * a] );
    }
}

__global__ void cast_array_kernel( size_t n, const double* __restrict__ src, float* __restrict__ dst )
{
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < n; i += size_t( gridDim.x ) * blockDim.x )
        dst[i] = float( src[i] );
}

// ---------------------------------------------------------------------------
// PCG on the stored-matrix operator with the operator's pieces fused into the
// PCG steps (pcg.hpp:78-102, z = r; the state layout and the x / r update of
// the tn_pcg_* kernels).  Per iteration four launches instead of the ~11 of
// the generic composition (memsets, apply, penalty dots / vector / axpy,
// halo sum, <p, Ap>, update, direction):
//   prepare: p = r + beta p (from the second iteration), ap = 0 and the fs/fs
//            penalty dots sum_owned x_node x p, whose last block turns them
//            into the penalty vector g = eps G^-1 d;
//   stored_apply_kernel: ap += wedge products of p (atomics);
//   gather:  aq = sum over the node's copies of (ap + g x x_node) -- the
//            penalty added on every copy before the halo sum, in the order
//            the operator uses -- and <p, aq> over owned nodes;
//   tn_pcg_update_f64: x += alpha p, r -= alpha aq, <r, r>, stopping rule.
// Every launch is gated by the stopping flag, so a fixed sequence (CUDA
// graph capture) gives the iterate the host-checked loop stops at.
enum : int
{
    kSpAn = 0, // tn_pcg_* state layout
    kSpPap,
    kSpR0,
    kSpBeta,
    kSpDone,
    kSpIts,
    kSpRelres,
    kSpHist = 8
};

struct SpcgParams
{
    size_t         ns;
    int            n1, fsfs;
    double         eps, ginv[9];
    const double * coords, *radii;
    const int *    lat_group, *offsets, *members;
    const uint8_t* owned;
    double*        state;
    double*        scratch; // [0..2] penalty dots, [3..5] penalty vector g
    double*        partials;
    unsigned*      counter;
};

__device__ __forceinline__ void spcg_position( const SpcgParams& S, unsigned i, double xp[3] )
{
    const unsigned n1  = unsigned( S.n1 );
    const unsigned lat = i / n1; // ns < 2^32 at every level tn_mesh_create accepts (<= 9)
    const unsigned r   = i - lat * n1;
    const unsigned d   = lat / ( n1 * n1 );
    const double   rr  = S.radii[d * n1 + r];
    const double*  c   = S.coords + size_t( lat ) * 3;
    xp[0] = c[0] * rr, xp[1] = c[1] * rr, xp[2] = c[2] * rr;
}

// v = p (after p = r + beta p when update_p) or the given field; ap = 0;
// penalty dots of v and, in the last block, g = eps G^-1 d
__global__ void __launch_bounds__( 256 ) spcg_prepare_kernel( SpcgParams S, Ptr3< double > p, Ptr3< const double > r,
                                                               Ptr3< const double > v, Ptr3< double > ap, int update_p,
                                                               int gated )
{
    if ( gated && S.state[kSpDone] != 0.0 )
        return;
    const double beta   = update_p ? S.state[kSpBeta] : 0.0;
    const size_t stride = size_t( gridDim.x ) * blockDim.x;
    double       sum[3] = { 0.0, 0.0, 0.0 };
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < S.ns; i += stride )
    {
        double w[3];
#pragma unroll
        for ( int c = 0; c < 3; ++c )
        {
            if ( update_p )
            {
                w[c]      = r.p[c][i] + beta * p.p[c][i];
                p.p[c][i] = w[c];
            }
            else
                w[c] = v.p[c][i];
            ap.p[c][i] = 0.0;
        }
        if ( S.fsfs && S.owned[i] )
        {
            double xp[3];
            spcg_position( S, unsigned( i ), xp );
            sum[0] += xp[1] * w[2] - xp[2] * w[1];
            sum[1] += xp[2] * w[0] - xp[0] * w[2];
            sum[2] += xp[0] * w[1] - xp[1] * w[0];
        }
    }
    if ( !S.fsfs )
        return;
    Neumaier acc[3];
    for ( int k = 0; k < 3; ++k )
        acc[k].add( sum[k] );
    if ( block_sum_finish< 3 >( acc, S.partials, S.counter, S.scratch ) && threadIdx.x == 0 )
    {
        const double d0 = S.scratch[0], d1 = S.scratch[1], d2 = S.scratch[2];
        for ( int k = 0; k < 3; ++k )
            S.scratch[3 + k] = S.eps * ( S.ginv[3 * k] * d0 + S.ginv[3 * k + 1] * d1 + S.ginv[3 * k + 2] * d2 );
    }
}

// a = halo sum over the node's copies of (ap + g x x).  mode 0 (initial
// residual): r = b - a, p = r, state from <r, r> (pcg.hpp:79-86); mode 1:
// aq = a, state[kSpPap] = <p, aq>
__global__ void __launch_bounds__( 256 ) spcg_gather_kernel( SpcgParams S, Ptr3< const double > ap, int mode,
                                                              Ptr3< const double > b, Ptr3< double > r,
                                                              Ptr3< double > p, Ptr3< double > aq, double atol )
{
    if ( mode == 1 && S.state[kSpDone] != 0.0 )
        return;
    const double g[3]   = { S.fsfs ? S.scratch[3] : 0.0, S.fsfs ? S.scratch[4] : 0.0, S.fsfs ? S.scratch[5] : 0.0 };
    const size_t stride = size_t( gridDim.x ) * blockDim.x;
    const unsigned n1   = unsigned( S.n1 );
    Neumaier      acc;
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < S.ns; i += stride )
    {
        double pen[3] = { 0.0, 0.0, 0.0 };
        if ( S.fsfs )
        {
            double xp[3];
            spcg_position( S, unsigned( i ), xp );
            pen[0] = g[1] * xp[2] - g[2] * xp[1];
            pen[1] = g[2] * xp[0] - g[0] * xp[2];
            pen[2] = g[0] * xp[1] - g[1] * xp[0];
        }
        const unsigned lat = unsigned( i ) / n1, rr = unsigned( i ) - lat * n1;
        const int      grp = S.lat_group[lat];
        double         dot = 0.0;
#pragma unroll
        for ( int c = 0; c < 3; ++c )
        {
            double a;
            if ( grp < 0 )
                a = ap.p[c][i] + pen[c];
            else
            {
                a = 0.0;
                for ( int k = S.offsets[grp]; k < S.offsets[grp + 1]; ++k )
                    a += ap.p[c][size_t( S.members[k] ) * n1 + rr] + pen[c];
            }
            if ( mode == 0 )
            {
                const double ri = b.p[c][i] - a;
                r.p[c][i]       = ri;
                p.p[c][i]       = ri;
                dot += ri * ri;
            }
            else
            {
                aq.p[c][i] = a;
                dot += p.p[c][i] * a;
            }
        }
        acc.add( S.owned[i] ? dot : 0.0 );
    }
    double* st = S.state;
    if ( block_sum_finish< 1 >( &acc, S.partials, S.counter, mode == 0 ? st + kSpAn : st + kSpPap ) &&
         threadIdx.x == 0 && mode == 0 )
    {
        const double r0 = sqrt( st[kSpAn] );
        st[kSpR0]       = r0;
        st[kSpBeta]     = 0.0;
        st[kSpDone]     = r0 < atol ? 1.0 : 0.0;
        st[kSpIts]      = 0.0;
        st[kSpRelres]   = 1.0;
        st[kSpHist]     = 1.0;
    }
}

// ---------------------------------------------------------------------------
// The vector steps of one coarse-grid PCG iteration in one launch of one
// thread-block cluster.
//
// On the coarsest level (level 3: 7,290 stored nodes) the vector steps of the
// multi-launch form are latency-bound: each launch costs its ramp and a
// last-block reduction through global memory.  Here the steps between two
// wedge-product launches (stored_apply_kernel over the whole GPU) run in one
// cluster of 16 CTAs (8 where the GPU cannot schedule 16): halo gather +
// <p, Ap>, the x / r update + <r, r> + stopping test, and the next direction
// p = r + beta p with ap cleared and the penalty dots of p, separated by the
// hardware cluster barrier (release / acquire at cluster scope).  Each
// reduction is combined through distributed shared memory: every CTA writes
// its compensated partial to its own shared memory and, after the barrier,
// reads all partials in rank order, so all CTAs hold bit-identical sums and
// take the same stopping decision.  Vectors are read with ld.global.cg (L2).
// The arithmetic per node is that of the multi-launch form (pcg.hpp:79-110).
//
// Every thread runs the same sequence of cluster barriers: the stopping flag
// is read by every thread before the first barrier (nothing writes it before
// then), so an early return is uniform over the cluster.
namespace cg = cooperative_groups;

constexpr int kCpThreads      = 512; // 16 x 512 threads: one level-3 node per thread
constexpr int kClusterMax     = 16;
constexpr int kClusterPcgMaxN = 8; // levels <= 3

struct ClusterPcgParams
{
    SpcgParams           S;
    Ptr3< const double > b;
    Ptr3< double >       x, r, p, ap, aq;
    int                  it; // 0: initial residual (r = b - a, p = r); >= 1: PCG iteration it
    double               rtol, atol;
};

// sum over the cluster of K compensated per-thread partials; the result is
// the same in every thread of every CTA.  part: this CTA's partials in the
// given slot (each slot is used once per launch).
template < int K >
__device__ void cluster_sum( cg::cluster_group& cl, Neumaier* acc, double ( *part )[K][2], int slot, double* out )
{
    __shared__ double sh[32][K][2];
    __shared__ double res[K];
    const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for ( int k = 0; k < K; ++k )
    {
        const Neumaier w = warp_reduce( acc[k] );
        if ( lane == 0 )
            sh[warp][k][0] = w.s, sh[warp][k][1] = w.c;
    }
    __syncthreads();
    if ( threadIdx.x == 0 )
        for ( int k = 0; k < K; ++k )
        {
            Neumaier b;
            for ( int w = 0; w < int( blockDim.x >> 5 ); ++w )
                b.merge( Neumaier{ sh[w][k][0], sh[w][k][1] } );
            part[slot][k][0] = b.s, part[slot][k][1] = b.c;
        }
    cl.sync();
    if ( warp == 0 )
    {
        // lane j fetches rank j's partials (one round of remote loads), then
        // every lane merges them in rank order from shuffles
        const unsigned nb = cl.num_blocks();
        double         qs[K], qc[K];
#pragma unroll
        for ( int k = 0; k < K; ++k )
            qs[k] = qc[k] = 0.0;
        if ( unsigned( lane ) < nb )
        {
            const double* q = cl.map_shared_rank( &part[slot][0][0], unsigned( lane ) );
#pragma unroll
            for ( int k = 0; k < K; ++k )
                qs[k] = q[2 * k], qc[k] = q[2 * k + 1];
        }
#pragma unroll
        for ( int k = 0; k < K; ++k )
        {
            Neumaier t;
            for ( unsigned j = 0; j < nb; ++j )
                t.merge( Neumaier{ __shfl_sync( 0xffffffffu, qs[k], int( j ) ),
                                   __shfl_sync( 0xffffffffu, qc[k], int( j ) ) } );
            if ( lane == 0 )
                res[k] = t.value();
        }
    }
    __syncthreads();
#pragma unroll
    for ( int k = 0; k < K; ++k )
        out[k] = res[k];
}

__global__ void __launch_bounds__( kCpThreads ) spcg_step_cluster_kernel( ClusterPcgParams P )
{
    __shared__ double part3[1][3][2];
    __shared__ double part1[2][1][2];
    cg::cluster_group cl = cg::this_cluster();
    const SpcgParams& S  = P.S;
    double*           st = S.state;
    if ( P.it > 0 && st[kSpDone] != 0.0 ) // uniform: read by every thread before any barrier
        return;
    const size_t   ns   = S.ns;
    const size_t   t0   = size_t( cl.block_rank() ) * blockDim.x + threadIdx.x;
    const size_t   nt   = size_t( cl.num_blocks() ) * blockDim.x;
    const unsigned n1   = unsigned( S.n1 );
    const bool     lead = cl.block_rank() == 0 && threadIdx.x == 0;
    const double   g[3] = { S.fsfs ? S.scratch[3] : 0.0, S.fsfs ? S.scratch[4] : 0.0, S.fsfs ? S.scratch[5] : 0.0 };
    double         an = st[kSpAn], r0 = st[kSpR0];

    // a = halo sum over the node's copies of (ap + g x x); it 0: r = b - a,
    // p = r and <r, r>; else aq = a and <p, aq>
    double red;
    {
        Neumaier acc;
        for ( size_t i = t0; i < ns; i += nt )
        {
            double pen[3] = { 0.0, 0.0, 0.0 };
            if ( S.fsfs )
            {
                double xp[3];
                spcg_position( S, unsigned( i ), xp );
                pen[0] = g[1] * xp[2] - g[2] * xp[1];
                pen[1] = g[2] * xp[0] - g[0] * xp[2];
                pen[2] = g[0] * xp[1] - g[1] * xp[0];
            }
            const unsigned lat = unsigned( i ) / n1, rr = unsigned( i ) - lat * n1;
            const int      grp = S.lat_group[lat];
            // every load of the node before any store (the fields may alias as far as the compiler knows)
            double a[3], q[3];
#pragma unroll
            for ( int c = 0; c < 3; ++c )
                q[c] = __ldcg( ( P.it == 0 ? P.b.p[c] : P.p.p[c] ) + i );
            if ( grp < 0 )
            {
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                    a[c] = __ldcg( P.ap.p[c] + i ) + pen[c];
            }
            else
            {
                a[0] = a[1] = a[2] = 0.0;
                for ( int k = S.offsets[grp]; k < S.offsets[grp + 1]; ++k )
                {
                    const size_t j = size_t( S.members[k] ) * n1 + rr;
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        a[c] += __ldcg( P.ap.p[c] + j ) + pen[c];
                }
            }
            double dot = 0.0;
#pragma unroll
            for ( int c = 0; c < 3; ++c )
            {
                if ( P.it == 0 )
                {
                    const double ri = q[c] - a[c];
                    __stcg( P.r.p[c] + i, ri );
                    __stcg( P.p.p[c] + i, ri );
                    dot += ri * ri;
                }
                else
                {
                    __stcg( P.aq.p[c] + i, a[c] );
                    dot += q[c] * a[c];
                }
            }
            acc.add( S.owned[i] ? dot : 0.0 );
        }
        cluster_sum< 1 >( cl, &acc, part1, 0, &red );
    }
    bool   done;
    double beta = 0.0;
    if ( P.it == 0 )
    {
        an   = red;
        r0   = sqrt( an );
        done = r0 < P.atol;
        if ( lead )
        {
            st[kSpAn] = an, st[kSpR0] = r0, st[kSpBeta] = 0.0, st[kSpDone] = done ? 1.0 : 0.0;
            st[kSpIts] = 0.0, st[kSpRelres] = 1.0, st[kSpHist] = 1.0;
        }
    }
    else
    {
        // x += alpha p, r -= alpha aq, <r, r>, stopping test  (pcg.hpp:88-110)
        const double pap = red, alpha = an / pap;
        double       rr;
        {
            Neumaier acc;
            for ( size_t i = t0; i < ns; i += nt )
            {
                double xv[3], pv[3], rv[3], qv[3], dot = 0.0;
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                {
                    xv[c] = __ldcg( P.x.p[c] + i ), pv[c] = __ldcg( P.p.p[c] + i );
                    rv[c] = __ldcg( P.r.p[c] + i ), qv[c] = __ldcg( P.aq.p[c] + i );
                }
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                {
                    __stcg( P.x.p[c] + i, xv[c] + alpha * pv[c] );
                    const double ri = rv[c] + ( -alpha ) * qv[c];
                    __stcg( P.r.p[c] + i, ri );
                    dot += ri * ri;
                }
                acc.add( S.owned[i] ? dot : 0.0 );
            }
            cluster_sum< 1 >( cl, &acc, part1, 1, &rr );
        }
        const double ar = sqrt( rr ), rel = ar / r0;
        done            = rel <= P.rtol || ar < P.atol;
        if ( !done )
            beta = rr / an;
        if ( lead )
        {
            st[kSpPap] = pap, st[kSpHist + P.it] = rel, st[kSpRelres] = rel, st[kSpIts] = double( P.it );
            if ( done )
                st[kSpDone] = 1.0;
            else
                st[kSpBeta] = beta, st[kSpAn] = rr;
        }
    }
    if ( !done )
    {
        // next direction p = r + beta p (p = r after the initial residual),
        // ap = 0, penalty dots of p and g = eps G^-1 d for the next apply
        double sum[3] = { 0.0, 0.0, 0.0 };
        for ( size_t i = t0; i < ns; i += nt )
        {
            double w[3], rv[3];
#pragma unroll
            for ( int c = 0; c < 3; ++c )
            {
                w[c]  = __ldcg( P.p.p[c] + i );
                rv[c] = P.it > 0 ? __ldcg( P.r.p[c] + i ) : 0.0;
            }
#pragma unroll
            for ( int c = 0; c < 3; ++c )
            {
                if ( P.it > 0 )
                {
                    w[c] = rv[c] + beta * w[c];
                    __stcg( P.p.p[c] + i, w[c] );
                }
                __stcg( P.ap.p[c] + i, 0.0 );
            }
            if ( S.fsfs && S.owned[i] )
            {
                double xp[3];
                spcg_position( S, unsigned( i ), xp );
                sum[0] += xp[1] * w[2] - xp[2] * w[1];
                sum[1] += xp[2] * w[0] - xp[0] * w[2];
                sum[2] += xp[0] * w[1] - xp[1] * w[0];
            }
        }
        if ( S.fsfs )
        {
            Neumaier acc[3];
            for ( int k = 0; k < 3; ++k )
                acc[k].add( sum[k] );
            double d[3];
            cluster_sum< 3 >( cl, acc, part3, 0, d );
            if ( lead )
                for ( int k = 0; k < 3; ++k )
                    S.scratch[3 + k] =
                        S.eps * ( S.ginv[3 * k] * d[0] + S.ginv[3 * k + 1] * d[1] + S.ginv[3 * k + 2] * d[2] );
        }
    }
    cl.sync(); // no CTA leaves while another may still read its shared memory
}

// Cluster size for the coarse-grid PCG step on this device: 16 where the GPU
// can schedule a 16-CTA cluster of the kernel, else 8, else 0 (the
// multi-launch form is used).
int spcg_cluster_size()
{
    static int size_of[kMaxDevices];
    static bool known[kMaxDevices] = {};
    const int   dev  = current_device();
    int&        size = size_of[dev];
    if ( known[dev] )
        return size;
    known[dev] = true;
    size       = 0;
    if ( cudaFuncSetAttribute( spcg_step_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1 ) !=
         cudaSuccess )
    {
        cudaGetLastError();
        return size;
    }
    for ( int c : { kClusterMax, 8 } )
    {
        cudaLaunchConfig_t  cfg{};
        cudaLaunchAttribute attr{};
        attr.id               = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = unsigned( c ), attr.val.clusterDim.y = 1, attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3( unsigned( c ) ), cfg.blockDim = dim3( kCpThreads ), cfg.attrs = &attr, cfg.numAttrs = 1;
        int n = 0;
        if ( cudaOccupancyMaxActiveClusters( &n, spcg_step_cluster_kernel, &cfg ) == cudaSuccess && n >= 1 )
        {
            size = c;
            break;
        }
        cudaGetLastError();
    }
    return size;
}

}  // namespace

template < typename T >
int stored_apply( const tn_mesh* m, const T* mats, const tn_epsdivdiv_params* p, const T* const* src, T* const* dst,
                  cudaStream_t st )
{
    TN_CHECK_ARG( m && mats && p && src && dst, "stored_apply: null argument" );
    TN_CHECK_ARG( p->bc_cmb >= 0 && p->bc_cmb <= 2 && p->bc_surface >= 0 && p->bc_surface <= 2,
                  "stored_apply: boundary condition codes must be 0, 1 or 2" );
    TN_CHECK_ARG( p->apply_mode == TN_APPLY_REPLACE || p->apply_mode == TN_APPLY_ADD, "stored_apply: bad apply mode" );
    StoredParams< T > P{};
    for ( int c = 0; c < 3; ++c )
    {
        TN_CHECK_ARG( src[c] && dst[c], "stored_apply: null vector component" );
        P.src.p[c] = src[c];
        P.dst.p[c] = dst[c];
        if ( p->apply_mode == TN_APPLY_REPLACE )
            TN_CUDA_TRY( cudaMemsetAsync( dst[c], 0, m->ns * sizeof( T ), st ) );
    }
    P.N = m->N, P.n1 = m->n1, P.coords = m->d_coords, P.mats = mats;
    P.bc_cmb = p->bc_cmb, P.bc_surf = p->bc_surface, P.diag = p->diagonal != 0;
    const long long wedges = 2LL * kDiamonds * m->N * m->N * m->N;
    const bool      fsfs   = !p->diagonal && p->bc_cmb == TN_BC_FREESLIP && p->bc_surface == TN_BC_FREESLIP;
    if ( fsfs )
    {
        // the penalty dots of src overlap the wedge kernel on the mesh's side stream
        int rc = fsfs_penalty_fork< T >( m, p->penalty_eps, src, st );
        if ( rc )
            return rc;
    }
    if ( p->diagonal )
        stored_diag_kernel< T ><<< unsigned( ( wedges + 127 ) / 128 ), 128, 0, st >>>( P );
    else
    {
        stored_apply_kernel< T ><<< unsigned( ( wedges + 127 ) / 128 ), 128, 0, st >>>( P );
    }
    TN_LAUNCH_CHECK();
    if ( fsfs )
    {
        int rc = fsfs_penalty_join< T >( m, dst, st );
        if ( rc )
            return rc;
    }
    if ( p->comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( m, dst, 3, st );
    return TN_OK;
}

// Host driver of the fused stored-matrix PCG (see spcg_prepare_kernel).
static int stored_pcg( const tn_mesh* m, const double* mats, const tn_epsdivdiv_params* p, const double* const* b,
                       double* const* x, double* const* work, double* state, int max_it, double rtol, double atol,
                       int check_every, cudaStream_t st )
{
    TN_CHECK_ARG( m && mats && p && b && x && work && state, "stored_pcg: null argument" );
    TN_CHECK_ARG( !p->diagonal && p->apply_mode == TN_APPLY_REPLACE && p->comm_mode == TN_COMM_ADDITIVE,
                  "stored_pcg: needs the non-diagonal operator in Replace mode with the additive halo" );
    TN_CHECK_ARG( p->bc_cmb >= 0 && p->bc_cmb <= 2 && p->bc_surface >= 0 && p->bc_surface <= 2,
                  "stored_pcg: boundary condition codes must be 0, 1 or 2" );
    TN_CHECK_ARG( max_it >= 0, "stored_pcg: max_iterations must be >= 0" );
    Ptr3< const double > pb{}, cx{};
    Ptr3< double >       px{}, pr{}, pp{}, pap{}, paq{};
    for ( int c = 0; c < 3; ++c )
    {
        TN_CHECK_ARG( b[c] && x[c], "stored_pcg: null vector component" );
        for ( int k = 0; k < 4; ++k )
            TN_CHECK_ARG( work[3 * k + c], "stored_pcg: null work field" );
        pb.p[c] = b[c], px.p[c] = x[c], cx.p[c] = x[c];
        pr.p[c] = work[c], pp.p[c] = work[3 + c], pap.p[c] = work[6 + c], paq.p[c] = work[9 + c];
    }
    SpcgParams S{};
    S.ns = m->ns, S.n1 = m->n1, S.fsfs = p->bc_cmb == TN_BC_FREESLIP && p->bc_surface == TN_BC_FREESLIP;
    S.eps = p->penalty_eps;
    for ( int i = 0; i < 9; ++i )
        S.ginv[i] = m->penalty_gram_inv[i];
    S.coords = m->d_coords, S.radii = m->d_radii;
    S.lat_group = m->d_lat_group, S.offsets = m->d_halo_offsets, S.members = m->d_halo_members;
    S.owned = m->d_node_owned, S.state = state, S.scratch = m->d_red_result;
    S.partials = m->d_red_partials, S.counter = m->d_red_counter;

    StoredParams< double > A{};
    A.N = m->N, A.n1 = m->n1, A.coords = m->d_coords, A.mats = mats;
    A.bc_cmb = p->bc_cmb, A.bc_surf = p->bc_surface, A.diag = 0;
    for ( int c = 0; c < 3; ++c )
        A.dst.p[c] = pap.p[c];
    const long long wedges   = 2LL * kDiamonds * m->N * m->N * m->N;
    const unsigned  ablocks  = unsigned( ( wedges + 127 ) / 128 );
    // one node per thread: at coarse levels the dependent loads of a node, not bandwidth, set the time
    const unsigned  nblocks  = unsigned( std::max< size_t >( 1, std::min< size_t >( ( m->ns + 255 ) / 256, kRedMaxBlocks ) ) );
    const tn_mesh*  seg[3]   = { m, m, m };
    double*         xs[3]    = { x[0], x[1], x[2] };
    double*         rs[3]    = { work[0], work[1], work[2] };
    const double*   ps[3]    = { work[3], work[4], work[5] };
    const double*   aqs[3]   = { work[9], work[10], work[11] };
    Ptr3< const double > cap{ { pap.p[0], pap.p[1], pap.p[2] } }, cr{ { pr.p[0], pr.p[1], pr.p[2] } };

    // coarse meshes: the vector steps of an iteration as one cluster launch
    const int           csize = m->N <= kClusterPcgMaxN ? spcg_cluster_size() : 0;
    ClusterPcgParams    CP{};
    cudaLaunchConfig_t  cfg{};
    cudaLaunchAttribute attr{};
    if ( csize > 0 )
    {
        CP.S = S, CP.b = pb, CP.x = px, CP.r = pr, CP.p = pp, CP.ap = pap, CP.aq = paq;
        CP.rtol = rtol, CP.atol = atol;
        attr.id               = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = unsigned( csize ), attr.val.clusterDim.y = 1, attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3( unsigned( csize ) ), cfg.blockDim = dim3( kCpThreads ), cfg.dynamicSmemBytes = 0;
        cfg.stream = st, cfg.attrs = &attr, cfg.numAttrs = 1;
    }

    // r = b - A x, p = r
    spcg_prepare_kernel<<< nblocks, 256, 0, st >>>( S, pp, cr, cx, pap, 0, 0 );
    TN_LAUNCH_CHECK();
    A.src = cx, A.gate = nullptr;
    stored_apply_kernel< double ><<< ablocks, 128, 0, st >>>( A );
    TN_LAUNCH_CHECK();
    if ( csize > 0 )
    {
        // also clears ap and forms the penalty vector of p for the first iteration
        CP.it = 0;
        TN_CUDA_TRY( cudaLaunchKernelEx( &cfg, spcg_step_cluster_kernel, CP ) );
    }
    else
        spcg_gather_kernel<<< nblocks, 256, 0, st >>>( S, cap, 0, pb, pr, pp, paq, atol );
    TN_LAUNCH_CHECK();
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    TN_CUDA_TRY( cudaStreamIsCapturing( st, &cs ) );
    const bool capturing = cs != cudaStreamCaptureStatusNone;
    A.src  = Ptr3< const double >{ { pp.p[0], pp.p[1], pp.p[2] } };
    A.gate = state + kSpDone;
    for ( int it = 1; it <= max_it; ++it )
    {
        if ( !capturing && check_every > 0 && ( it == 1 || ( it - 1 ) % check_every == 0 ) )
        {
            double done = 0.0;
            TN_CUDA_TRY( cudaMemcpyAsync( &done, state + kSpDone, sizeof( double ), cudaMemcpyDeviceToHost, st ) );
            TN_CUDA_TRY( cudaStreamSynchronize( st ) );
            if ( done != 0.0 )
                break;
        }
        if ( csize > 0 )
        {
            // wedge products over the whole GPU, then gather + update + next direction in one cluster
            stored_apply_kernel< double ><<< ablocks, 128, 0, st >>>( A );
            TN_LAUNCH_CHECK();
            CP.it = it;
            TN_CUDA_TRY( cudaLaunchKernelEx( &cfg, spcg_step_cluster_kernel, CP ) );
            TN_LAUNCH_CHECK();
            continue;
        }
        spcg_prepare_kernel<<< nblocks, 256, 0, st >>>( S, pp, cr, A.src, pap, it > 1, 1 );
        TN_LAUNCH_CHECK();
        stored_apply_kernel< double ><<< ablocks, 128, 0, st >>>( A );
        TN_LAUNCH_CHECK();
        spcg_gather_kernel<<< nblocks, 256, 0, st >>>( S, cap, 1, pb, pr, pp, paq, atol );
        TN_LAUNCH_CHECK();
        int rc = tn_pcg_update_f64( 3, seg, xs, rs, ps, aqs, state, it, rtol, atol, st );
        if ( rc )
            return rc;
    }
    return TN_OK;
}

}  // namespace tn

using namespace tn;

extern "C" int tn_local_matrix_count( const tn_mesh* m, size_t* entries )
{
    TN_CHECK_ARG( m && entries, "tn_local_matrix_count: null argument" );
    const size_t wedges = size_t( kDiamonds ) * m->N * m->N * m->N * 2;
    *entries            = ( ( wedges + 31 ) / 32 ) * 32 * kChunks * 4; // whole groups of 32 wedges, 172 entries each
    return TN_OK;
}

extern "C" int tn_kerngen_local_matrices_f64( const tn_mesh* m, const double* k, double* mats, void* s )
{
    TN_CHECK_ARG( m && mats, "tn_kerngen_local_matrices_f64: null argument" );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    local_matrices_kernel<<< unsigned( cells ), 64, 0, as_stream( s ) >>>( m->N, m->d_coords, m->d_radii, k, mats,
                                                                          nullptr, 0 );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

extern "C" int tn_gca_elements_f64( const tn_mesh* fine, const double* k_fine, int level_range, uint8_t* marks, void* s )
{
    TN_CHECK_ARG( fine && k_fine && marks, "tn_gca_elements_f64: null argument" );
    TN_CHECK_ARG( level_range >= 0 && level_range <= fine->level, "tn_gca_elements_f64: bad level range" );
    const int       N0    = fine->N >> level_range;
    const long long cells = (long long) kDiamonds * fine->N * fine->N * fine->N;
    TN_CUDA_TRY( cudaMemsetAsync( marks, 0, size_t( kDiamonds ) * N0 * N0 * N0, as_stream( s ) ) );
    gca_elements_kernel<<< unsigned( ( cells + 127 ) / 128 ), 128, 0, as_stream( s ) >>>( fine->N, level_range, k_fine,
                                                                                         marks );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

extern "C" int tn_agca_unmarked_local_matrices_f64( const tn_mesh* m, const double* k, const uint8_t* marks,
                                                    int level_range, double* mats, void* s )
{
    TN_CHECK_ARG( m && mats && marks, "tn_agca_unmarked_local_matrices_f64: null argument" );
    TN_CHECK_ARG( level_range >= 0 && level_range <= m->level, "tn_agca_unmarked_local_matrices_f64: bad level range" );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    local_matrices_kernel<<< unsigned( cells ), 64, 0, as_stream( s ) >>>( m->N, m->d_coords, m->d_radii, k, mats,
                                                                          marks, level_range );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

extern "C" int tn_gca_coarsen_f64( const tn_mesh* fine, const tn_mesh* coarse, const double* k_fine,
                                   const double* mats_fine, int mode, double* mats_coarse, void* s )
{
    TN_CHECK_ARG( fine && coarse && mats_coarse, "tn_gca_coarsen_f64: null argument" );
    TN_CHECK_ARG( coarse->level == fine->level - 1, "tn_gca_coarsen_f64: coarse mesh must be one level below" );
    TN_CHECK_ARG( ( k_fine != nullptr ) != ( mats_fine != nullptr ),
                  "tn_gca_coarsen_f64: give exactly one of k_fine and mats_fine" );
    TN_CHECK_ARG( mode == 0 || mode == 1, "tn_gca_coarsen_f64: mode must be 0 (constant) or 1 (linear)" );
    const long long cells = (long long) kDiamonds * coarse->N * coarse->N * coarse->N;
    if ( k_fine )
        gca_coarsen_kernel< true ><<< unsigned( cells ), kGcaThreads, 0, as_stream( s ) >>>(
            fine->N, fine->d_coords, fine->d_radii, k_fine, nullptr, mode, mats_coarse );
    else
        gca_coarsen_kernel< false ><<< unsigned( cells ), kGcaThreads, 0, as_stream( s ) >>>(
            fine->N, fine->d_coords, fine->d_radii, nullptr, mats_fine, mode, mats_coarse );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

extern "C" int tn_stored_epsdivdiv_apply_f64( const tn_mesh* m, const double* mats, const tn_epsdivdiv_params* p,
                                              const double* const* src, double* const* dst, void* s )
{
    return stored_apply< double >( m, mats, p, src, dst, as_stream( s ) );
}
extern "C" int tn_stored_epsdivdiv_apply_f32( const tn_mesh* m, const float* mats, const tn_epsdivdiv_params* p,
                                              const float* const* src, float* const* dst, void* s )
{
    return stored_apply< float >( m, mats, p, src, dst, as_stream( s ) );
}

extern "C" int tn_array_cast_f64_to_f32( size_t n, const double* src, float* dst, void* s )
{
    TN_CHECK_ARG( src && dst, "tn_array_cast_f64_to_f32: null argument" );
    if ( n == 0 )
        return TN_OK;
    const unsigned blocks = unsigned( std::min< size_t >( ( n + 1023 ) / 1024, 148 * 32 ) );
    cast_array_kernel<<< blocks, 256, 0, as_stream( s ) >>>( n, src, dst );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

extern "C" int tn_stored_pcg_f64( const tn_mesh* m, const double* mats, const tn_epsdivdiv_params* p,
                                  const double* const* b, double* const* x, double* const* work, double* state,
                                  int max_iterations, double relative_tolerance, double absolute_tolerance,
                                  int check_every, void* s )
{
    return stored_pcg( m, mats, p, b, x, work, state, max_iterations, relative_tolerance, absolute_tolerance,
                       check_every, as_stream( s ) );
}
