// Epsilon-div-div operator apply (B200 design of EpsilonDivDivKerngen,
// fe/wedge/operators/shell/epsilon_divdiv_kerngen.hpp).
//
// a(u, v) = int k (2 eps(u):eps(v) - 2/3 div u div v) with the one-point
// (centroid) wedge rule and k averaged over the six wedge nodes (:1189-1196).
//
// Kernels
//  * kerngen_tile_kernel: the hot path.  One CTA of TS warps owns TS cell
//    strips (x) of one diamond over a run of y rows and the full radial
//    extent; each warp marches its strip along y, lanes = 32 consecutive
//    radial cells, so loads are coalesced along r and the radial node sharing
//    is a warp shuffle.  Node rows stream through a shared-memory ring; the
//    node column shared by two strips of the CTA is summed in shared memory,
//    the one shared with the previous tile (seam column) by two atomic halves
//    onto the zeros seam_zero_kernel writes first; every other node is written
//    once with coalesced stores.  Per-wedge geometry is factorised as
//    J = M diag(r_mid, r_mid, dr/2) with M the lateral triangle matrix, so
//    M^{-T} is computed once per wedge column and each cell only rescales.
//    Boundary-layer cells of a non-Neumann boundary are left out and added by
//  * kerngen_bcell_kernel: one thread per boundary-layer cell with the full
//    boundary logic of cell_full (Dirichlet elimination with kept diagonal,
//    free-slip projection with the normal-normal add-back), atomics onto the
//    tile kernel's output;
//  * kerngen_cell_kernel: the same per-cell logic for every cell (and the
//    rotated diagonal), for the diagonal mode and levels too small for tiling.
//  * penalty kernels for free-slip on both boundaries.
#include <cuda_pipeline.h>

#include <algorithm>

#include "common.cuh"
#include "reduce.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

constexpr int kRC     = 32; // radial cells per chunk (one per lane)
constexpr int kSegMax = 24; // longest run of node rows a CTA finalises in one y march
constexpr int kLev    = kRC + 1; // node levels per chunk
constexpr int kSlots  = 4;       // row ring depth (prefetch distance 3)

// The shape of the tiled kernel for x tiles of TS cell strips: TS warps per
// CTA, one strip each; 16 strips where N allows it (one 512-thread CTA per SM),
// 8 at N = 8 (two 256-thread CTAs per SM).  Sixteen warps per SM leave 128
// registers per thread (each SM sub-partition holds 16,384 registers for its
// four warps; a seventeenth warp would cap every thread at 96).
template < int TS >
struct Tile
{
    static constexpr int W         = TS;            // warps = cell strips per CTA
    static constexpr int Threads   = W * 32;
    static constexpr int MinBlocks = TS == 8 ? 2 : 1; // resident CTAs per SM the kernel is compiled for
    static constexpr int Group     = Threads / 4;   // fill threads per field
    static constexpr int FieldEl   = ( W + 1 ) * kLev;
    static constexpr int FillPer   = ( FieldEl + Group - 1 ) / Group;
};

template < typename T >
struct TileParams
{
    int           N, n1, xtiles, seg_max; // seg_max: longest run of node rows one segment finalises
    int           nd;                     // stored diamonds
    const double* coords;
    const T*      radii;
    const T*      k;
    Ptr3< const T > src;
    Ptr3< T >     dst;
    int           add_mode;
    int           skip_cmb, skip_surface; // leave that boundary layer of cells to the boundary kernel
    const double* beta;                   // fs/fs penalty vector (3) or nullptr
};

// Per-wedge flux vectors S1 = sigma q0, S2 = sigma q1, S3 = sigma kq2 with
// sigma = omega (2 sym(G) - 2/3 tr(G) I), G = q0 (x) v1 + q1 (x) v2 + kq2 (x) v3
// and kq2 = kappa q2 (the radial factor folded into the third row once per wedge).
// A lane whose cell does not contribute (ok false) gets sigma = 0: the six stress
// components are selected, so its fluxes are exact zeros whatever its (possibly
// unloaded) corner values hold.
template < typename T >
__device__ __forceinline__ void wedge_flux( const T* __restrict__ g, const T v1[3], const T v2[3], const T v3[3],
                                            T kappa, T omega, bool ok, T S1[3], T S2[3], T S3[3] )
{
    T q0[3], q1[3], q2[3];
#pragma unroll
    for ( int a = 0; a < 3; ++a )
        q0[a] = g[a], q1[a] = g[3 + a], q2[a] = kappa * g[6 + a];
    const T G00  = q0[0] * v1[0] + q1[0] * v2[0] + q2[0] * v3[0];
    const T G11  = q0[1] * v1[1] + q1[1] * v2[1] + q2[1] * v3[1];
    const T G22  = q0[2] * v1[2] + q1[2] * v2[2] + q2[2] * v3[2];
    const T H01  = q0[0] * v1[1] + q1[0] * v2[1] + q2[0] * v3[1] + q0[1] * v1[0] + q1[1] * v2[0] + q2[1] * v3[0];
    const T H02  = q0[0] * v1[2] + q1[0] * v2[2] + q2[0] * v3[2] + q0[2] * v1[0] + q1[2] * v2[0] + q2[2] * v3[0];
    const T H12  = q0[1] * v1[2] + q1[1] * v2[2] + q2[1] * v3[2] + q0[2] * v1[1] + q1[2] * v2[1] + q2[2] * v3[1];
    const T div  = G00 + G11 + G22;
    const T tdiv = T( 2.0 / 3.0 ) * div;
    T       s00 = omega * ( T( 2 ) * G00 - tdiv ), s11 = omega * ( T( 2 ) * G11 - tdiv ),
      s22 = omega * ( T( 2 ) * G22 - tdiv );
    T s01 = omega * H01, s02 = omega * H02, s12 = omega * H12;
    if ( !ok )
        s00 = s11 = s22 = s01 = s02 = s12 = T( 0 );
    S1[0] = s00 * q0[0] + s01 * q0[1] + s02 * q0[2];
    S1[1] = s01 * q0[0] + s11 * q0[1] + s12 * q0[2];
    S1[2] = s02 * q0[0] + s12 * q0[1] + s22 * q0[2];
    S2[0] = s00 * q1[0] + s01 * q1[1] + s02 * q1[2];
    S2[1] = s01 * q1[0] + s11 * q1[1] + s12 * q1[2];
    S2[2] = s02 * q1[0] + s12 * q1[1] + s22 * q1[2];
    S3[0] = s00 * q2[0] + s01 * q2[1] + s02 * q2[2];
    S3[1] = s01 * q2[0] + s11 * q2[1] + s12 * q2[2];
    S3[2] = s02 * q2[0] + s12 * q2[1] + s22 * q2[2];
}

// Tiled owner-computes apply.  CTA = kW warps; warp w handles the cell strip
// X = sx0 + w of one y segment, lanes = 32 consecutive radial cells.  The
// warp marches along y: at step s it computes cell (X, cy) and finalises node
// row cy, carrying its contributions to row cy+1 in registers.  A node column
// X gets its two halves from strips X (left side) and X-1 (right side); right
// halves are exchanged through shared memory, one barrier per step.  The tile's
// first column sx0 (sx0 > 0) has its right half in the previous tile's last
// strip: both tiles add their halves to it atomically (two addends onto the
// zeros seam_zero_kernel left, so the sum does not depend on their order), and
// every other node is written once with plain stores.  Node rows
// (the CTA's kW+1 columns x 3 src components + k x 33 levels) are streamed
// into a 4-slot shared-memory ring with cp.async three rows ahead (fill_row),
// so global latency overlaps the arithmetic of the previous steps.  The radial chunk
// boundary level r0 + 32 is carried to the next chunk in shared memory.
template < typename T, int TS >
size_t tile_smem_bytes( int n1, int SY )
{
    constexpr int kW = Tile< TS >::W, kThreads = Tile< TS >::Threads;
    const size_t radii = size_t( 10 ) * ( ( n1 + 1 ) & ~1 );
    const size_t geo   = size_t( kW ) * ( SY + 2 ) * 20;
    const size_t rows  = size_t( kSlots ) * ( kW + 1 ) * 4 * kLev;
    const size_t xbuf  = size_t( 2 ) * kW * 3 * kLev;
    const size_t carry = size_t( kW + 1 ) * ( SY + 2 ) * 3;
    const size_t top   = size_t( kW ) * 6;
    return sizeof( T ) * ( radii + geo + rows + xbuf + carry + top ) + 16 + 32 * kThreads; // + fill descriptors
}

// Row fill.  A ring slot holds one node row of the CTA's kW+1 columns, stored
// [field][column][level] (fields: 3 src components, k).  The threads form 4
// groups of kThreads / 4, one per field; a thread copies elements t, t + group,
// ... of its field's (kW+1) x kLev block, each a fixed (column, level) whose
// 32-bit element offset advances by one node row (n1) per step, so a fill costs
// one offset add and one 8-byte cp.async per element.  The offsets of the
// chunk's first row live in shared memory (2 x 16 bytes per thread) and hold
// no registers across the wedge arithmetic.  Columns outside the diamond and
// levels past the chunk are not copied; rows outside the diamond not at all
// (no contributing cell reads them).
template < int TS >
__device__ __forceinline__ void fill_setup( uint4* desc, int N, int n1, int d, int X0, int Y0, int r0, int RC )
{
    constexpr int kGroup = Tile< TS >::Group, kFieldEl = Tile< TS >::FieldEl, kFillPer = Tile< TS >::FillPer;
    static_assert( kFillPer == 5, "descriptor layout" );
    const int t = threadIdx.x % kGroup;
    unsigned  off[kFillPer], valid = 0;
#pragma unroll
    for ( int i = 0; i < kFillPer; ++i )
    {
        const int  j   = t + i * kGroup;
        const int  col = j / kLev, lev = j - col * kLev;
        const int  X   = X0 + col;
        const bool ok  = j < kFieldEl && X >= 0 && X <= N && lev <= RC;
        off[i]         = ok ? unsigned( ( ( d * n1 + X ) * n1 + Y0 ) * n1 + r0 + lev ) : 0u;
        valid |= ok ? ( 1u << i ) : 0u;
    }
    desc[2 * threadIdx.x]     = make_uint4( off[0], off[1], off[2], off[3] );
    desc[2 * threadIdx.x + 1] = make_uint4( off[4], valid, 0u, 0u );
}

// node row Y = Y0 + step into `slot`
template < int TS, typename T >
__device__ __forceinline__ void fill_row( const uint4* desc, const T* f0, const T* f1, const T* f2, const T* f3, T* slot,
                                          int step, int Y, int N, int n1 )
{
    constexpr int kGroup = Tile< TS >::Group, kFieldEl = Tile< TS >::FieldEl, kFillPer = Tile< TS >::FillPer;
    const int      f = threadIdx.x / kGroup, t = threadIdx.x - f * kGroup;
    const T*       fb = f == 0 ? f0 : ( f == 1 ? f1 : ( f == 2 ? f2 : f3 ) );
    const uint4    a = desc[2 * threadIdx.x], b = desc[2 * threadIdx.x + 1];
    const unsigned off[kFillPer] = { a.x, a.y, a.z, a.w, b.x };
    const unsigned valid         = b.y;
    if ( Y < 0 || Y > N )
        return;
    const unsigned adv = unsigned( step * n1 );
    T*             dst = slot + f * kFieldEl + t;
#pragma unroll
    for ( int i = 0; i < kFillPer; ++i )
        if ( t + i * kGroup < kFieldEl && ( valid >> i & 1u ) )
            __pipeline_memcpy_async( dst + i * kGroup, fb + ( off[i] + adv ), sizeof( T ) );
}

template < typename T, int TS >
__global__ void __launch_bounds__( Tile< TS >::Threads, Tile< TS >::MinBlocks ) kerngen_tile_kernel( TileParams< T > P )
{
    constexpr int kTS = TS, kW = Tile< TS >::W, kFieldEl = Tile< TS >::FieldEl;
    extern __shared__ __align__( 16 ) unsigned char smem_raw[];
    constexpr unsigned FULL = 0xffffffffu;
    const int          N = P.N, n1 = P.n1, SM = P.seg_max;
    const T *          f0 = P.src.p[0], *f1 = P.src.p[1], *f2 = P.src.p[2], *f3 = P.k;
    T *                o0 = P.dst.p[0], *o1 = P.dst.p[1], *o2 = P.dst.p[2];
    const bool         add_mode = P.add_mode != 0;
    const double*      beta     = P.beta;

    T* s_radii = reinterpret_cast< T* >( smem_raw );
    T* s_geo   = s_radii + 10 * ( ( n1 + 1 ) & ~1 );
    T* s_rows  = s_geo + kW * ( SM + 2 ) * 20;
    T* s_xbuf  = s_rows + kSlots * ( kW + 1 ) * 4 * kLev;
    T* s_carry = s_xbuf + 2 * kW * 3 * kLev;
    T* s_top   = s_carry + ( kW + 1 ) * ( SM + 2 ) * 3; // [w][column][c]: top sums of lane RC-1 (level r0 + RC)
    uint4* s_fill = reinterpret_cast< uint4* >( ( reinterpret_cast< uintptr_t >( s_top + kW * 6 ) + 15 ) &
                                                ~uintptr_t( 15 ) ); // fill descriptors, 16-byte aligned
    auto slot  = [s_rows]( int y ) { return s_rows + ( ( y + kSlots ) % kSlots ) * ( ( kW + 1 ) * 4 * kLev ); };

    for ( int i = threadIdx.x; i < P.nd * n1; i += blockDim.x )
        s_radii[( i / n1 ) * ( ( n1 + 1 ) & ~1 ) + i % n1] = P.radii[i];

    const int  lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int  RC   = min( kRC, N );

    // Even split of all (diamond, x tile, node row) items over the grid: this
    // CTA finalises rows [g_begin, g_end) of the flattened list, in runs
    // (segments) of at most seg_max consecutive rows of one x tile.
    const long long rows_per_tile = N + 1;
    const long long total         = (long long) P.nd * P.xtiles * rows_per_tile;
    const long long g_begin       = total * blockIdx.x / gridDim.x;
    const long long g_end         = total * ( blockIdx.x + 1 ) / gridDim.x;

    for ( long long g = g_begin; g < g_end; )
    {
        const long long tile   = g / rows_per_tile;
        const int       row_lo = int( g - tile * rows_per_tile );
        const int       row_hi = int( min( (long long) N, row_lo + min( (long long) SM, g_end - g ) - 1 ) );
        g += row_hi - row_lo + 1;
        const int  tx        = int( tile % P.xtiles );
        const int  d         = int( tile / P.xtiles );
        const int  sx0       = tx * kTS; // strip of warp 0
        const int  nsteps    = row_hi - row_lo + 2; // step s computes cell cy = row_lo - 1 + s
        const int  X         = sx0 + w;
        const bool strip_ok  = X >= 0 && X <= N - 1;
        const bool seam_lo   = w == 0 && tx > 0;                   // column X: its right half is the last tile's
        const bool last_tile = tx == P.xtiles - 1;
        const bool seam_hi   = w == kW - 1 && !last_tile;           // column X + 1: the next tile's column sx0
        const bool owns_last = w == kW - 1 && last_tile;            // column N = X + 1, whole
        const int  s0        = row_lo == 0 ? 1 : 0;
        const T*   radii     = s_radii + d * ( ( n1 + 1 ) & ~1 );

        __syncthreads(); // previous segment done with the geometry buffer
        for ( int i = threadIdx.x; i < kW * nsteps * 2; i += blockDim.x )
        {
            const int wdg = i & 1, cs = i >> 1;
            const int ww = cs / nsteps, s = cs % nsteps;
            const int Xg = sx0 + ww, Y = row_lo - 1 + s;
            T*        gg = s_geo + ( ( ww * ( SM + 2 ) + s ) * 2 + wdg ) * 10;
            if ( Xg < 0 || Xg > N - 1 || Y < 0 || Y > N - 1 )
            {
                // no cell: zero geometry, so the masked flux of the step is exactly zero
                for ( int j = 0; j < 10; ++j )
                    gg[j] = T( 0 );
                continue;
            }
            const double* c00 = P.coords + lat_index( n1, d, Xg, Y ) * 3;
            const double* c10 = P.coords + lat_index( n1, d, Xg + 1, Y ) * 3;
            const double* c01 = P.coords + lat_index( n1, d, Xg, Y + 1 ) * 3;
            const double* c11 = P.coords + lat_index( n1, d, Xg + 1, Y + 1 ) * 3;
            double        q[9], adet;
            if ( wdg == 0 )
                lateral_geometry( c00, c10, c01, q, &adet );
            else
                lateral_geometry( c11, c01, c10, q, &adet );
            for ( int j = 0; j < 9; ++j )
                gg[j] = T( q[j] );
            gg[9] = T( adet );
        }

        for ( int r0 = 0; r0 < N; r0 += RC )
        {
            const bool last_chunk = r0 + RC == N;
            const int  r          = r0 + lane;
            const int  rl         = min( r, N - 1 );
            bool       lane_ok    = lane < RC;
            if ( ( P.skip_cmb && r == 0 ) || ( P.skip_surface && r == N - 1 ) )
                lane_ok = false;

            const int cyb = row_lo - 1 + s0;
            fill_setup< TS >( s_fill, N, n1, d, sx0, cyb, r0, RC );
            for ( int j = 0; j < kSlots - 1; ++j )
            {
                fill_row< TS >( s_fill, f0, f1, f2, f3, slot( cyb + j ), j, cyb + j, N, n1 );
                __pipeline_commit();
            }
            __pipeline_wait_prior( kSlots - 3 );
            __syncthreads();

            const T   r_lo = radii[rl], r_hi = radii[rl + 1];
            const T   h     = T( 0.5 ) * ( r_hi - r_lo );
            const T   kappa = T( 0.5 ) * ( r_hi + r_lo ) / ( T( 3 ) * h );
            const T   wbase = h * T( 0.25 / 6.0 ); // omega = (k_sum / 6) |det M| h / 4
            const int lb    = min( lane, kRC - 1 );

            // y-carry of the cell row below: its contributions to the node row it shares with this one, per
            // column (L: X, R: X + 1), bottom (level r) and top (level r + 1, still to be handed to the lane
            // above) parts kept apart so one shuffle per column and component moves both rows' tops
            T  cLb[3] = { 0, 0, 0 }, cLt[3] = { 0, 0, 0 }, cRb[3] = { 0, 0, 0 }, cRt[3] = { 0, 0, 0 };
            T* tw = s_top + w * 6; // lane RC - 1: its top sums (level r0 + RC) of columns X and X + 1
            for ( int s = s0; s < nsteps; ++s )
            {
                const int  cy      = row_lo - 1 + s;
                const bool cell_ok = strip_ok && cy <= N - 1;
                // row cy + 3 into the slot of row cy - 1, which every warp finished reading before the last
                // barrier; issued here, where few registers are live
                fill_row< TS >( s_fill, f0, f1, f2, f3, slot( cy + kSlots - 1 ), cy + kSlots - 1 - cyb, cy + kSlots - 1, N,
                                n1 );
                T          L[3], R[3];
                {
                    // corners: 0 = (X, cy), 1 = (X+1, cy), 2 = (X, cy+1), 3 = (X+1, cy+1)
                    const T* rp = slot( cy ) + w * kLev;
                    const T* rn = slot( cy + 1 ) + w * kLev;
                    T        S[4][3], D[4][3], K[4];
#pragma unroll
                    for ( int q = 0; q < 4; ++q )
                    {
                        const T* base = ( q < 2 ? rp : rn ) + ( q & 1 ) * kLev;
#pragma unroll
                        for ( int c = 0; c < 3; ++c )
                        {
                            const T bv = base[c * kFieldEl + lb], tv = base[c * kFieldEl + lb + 1];
                            S[q][c] = bv + tv, D[q][c] = tv - bv;
                        }
                        K[q] = base[3 * kFieldEl + lb] + base[3 * kFieldEl + lb + 1];
                    }
                    const T* g0 = s_geo + ( ( w * ( SM + 2 ) + s ) * 2 ) * 10;
                    const T* g1 = g0 + 10;
                    const bool ok = cell_ok && lane_ok;
                    T        v1[3], v2[3], v3[3], A1[3], A2[3], A3[3], B1[3], B2[3], B3[3];
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        v1[c] = S[1][c] - S[0][c], v2[c] = S[2][c] - S[0][c], v3[c] = D[0][c] + D[1][c] + D[2][c];
                    wedge_flux( g0, v1, v2, v3, kappa, wbase * ( K[0] + K[1] + K[2] ) * g0[9], ok, A1, A2, A3 );
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        v1[c] = S[2][c] - S[3][c], v2[c] = S[1][c] - S[3][c], v3[c] = D[3][c] + D[2][c] + D[1][c];
                    wedge_flux( g1, v1, v2, v3, kappa, wbase * ( K[3] + K[2] + K[1] ) * g1[9], ok, B1, B2, B3 );
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                    {
                        const T xa = A1[c] + A2[c], xb = B1[c] + B2[c];
                        const T s33 = A3[c] + B3[c];
                        const T e10 = A1[c] + B2[c], e01 = A2[c] + B1[c];
                        // the cell's bottom (level r) and top (level r + 1) parts at its four corner columns
                        const T bo0 = -xa - A3[c], tp0 = -xa + A3[c];
                        const T bo1 = e10 - s33, tp1 = e10 + s33;
                        const T bo2 = e01 - s33, tp2 = e01 + s33;
                        const T bo3 = -xb - B3[c], tp3 = -xb + B3[c];
                        // node row cy: this cell's near corners plus the carried far corners of the cell below
                        const T tL = tp0 + cLt[c], tR = tp1 + cRt[c];
                        const T bL = __shfl_up_sync( FULL, tL, 1 ), bR = __shfl_up_sync( FULL, tR, 1 );
                        L[c]   = bo0 + cLb[c] + ( lane > 0 ? bL : T( 0 ) );
                        R[c]   = bo1 + cRb[c] + ( lane > 0 ? bR : T( 0 ) );
                        cLb[c] = bo2, cLt[c] = tp2, cRb[c] = bo3, cRt[c] = tp3;
                        if ( lane == RC - 1 ) // level r0 + RC: only the top cell of the chunk contributes
                            tw[c] = tL, tw[3 + c] = tR;
                    }
                }

                T* xb = s_xbuf + ( ( s & 1 ) * kW + w ) * 3 * kLev;
                if ( lane < RC )
                {
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        xb[c * kLev + lane] = R[c];
                }
                if ( lane == RC - 1 )
                {
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                        xb[c * kLev + RC] = tw[3 + c];
                }
                __pipeline_commit();
                __pipeline_wait_prior( kSlots - 3 );
                __syncthreads();

                if ( s == 0 )
                    continue; // row row_lo - 1 belongs to another segment
#pragma unroll
                for ( int side = 0; side < 2; ++side )
                {
                    if ( side == 1 && !owns_last && !seam_hi )
                        continue;
                    const bool seam = side == 0 ? seam_lo : seam_hi; // half of the column: atomic add
                    const int  Xn   = X + side;
                    const int  slt  = side == 0 ? w : kW;
                    T          F[3], F32[3];
                    const T*   xl = s_xbuf + ( ( s & 1 ) * kW + max( w - 1, 0 ) ) * 3 * kLev;
#pragma unroll
                    for ( int c = 0; c < 3; ++c )
                    {
                        if ( side == 0 )
                        {
                            F[c]   = L[c] + ( w > 0 && lane < RC ? xl[c * kLev + lane] : T( 0 ) );
                            F32[c] = tw[c] + ( w > 0 ? xl[c * kLev + RC] : T( 0 ) );
                        }
                        else
                        {
                            F[c]   = R[c];
                            F32[c] = tw[3 + c];
                        }
                    }
                    T* carry = s_carry + ( slt * ( SM + 2 ) + s ) * 3;
                    if ( r0 > 0 && lane == 0 )
                    {
#pragma unroll
                        for ( int c = 0; c < 3; ++c )
                            F[c] += carry[c];
                    }
                    __syncwarp();
                    const size_t nb  = lat_index( n1, d, Xn, cy ) * n1;
                    const int    lev = lane < RC ? r : N; // lanes < RC: level r; lane RC-1 also level N
                    if ( beta && !( side == 1 && seam ) ) // the penalty once per node: with the left half
                    {
                        const double* u   = P.coords + lat_index( n1, d, Xn, cy ) * 3;
                        const double  rr  = double( radii[lane < RC ? r : 0] ), rN = double( radii[N] );
                        const double  x0  = u[0] * rr, x1 = u[1] * rr, x2 = u[2] * rr;
                        const double  y0  = u[0] * rN, y1 = u[1] * rN, y2 = u[2] * rN;
                        F[0] += T( beta[1] * x2 - beta[2] * x1 );
                        F[1] += T( beta[2] * x0 - beta[0] * x2 );
                        F[2] += T( beta[0] * x1 - beta[1] * x0 );
                        // the top level is level N only in the last radial chunk; otherwise it is the
                        // next chunk's level r0 + RC, whose lane 0 adds that level's penalty itself
                        if ( last_chunk )
                        {
                            F32[0] += T( beta[1] * y2 - beta[2] * y1 );
                            F32[1] += T( beta[2] * y0 - beta[0] * y2 );
                            F32[2] += T( beta[0] * y1 - beta[1] * y0 );
                        }
                    }
                    (void) lev;
                    if ( lane < RC )
                    {
                        T* p0 = o0 + nb + r;
                        T* p1 = o1 + nb + r;
                        T* p2 = o2 + nb + r;
                        if ( seam )
                            atomicAdd( p0, F[0] ), atomicAdd( p1, F[1] ), atomicAdd( p2, F[2] );
                        else
                        {
                            *p0 = add_mode ? *p0 + F[0] : F[0];
                            *p1 = add_mode ? *p1 + F[1] : F[1];
                            *p2 = add_mode ? *p2 + F[2] : F[2];
                        }
                    }
                    if ( lane == RC - 1 )
                    {
                        if ( last_chunk )
                        {
                            T* p0 = o0 + nb + N;
                            T* p1 = o1 + nb + N;
                            T* p2 = o2 + nb + N;
                            if ( seam )
                                atomicAdd( p0, F32[0] ), atomicAdd( p1, F32[1] ), atomicAdd( p2, F32[2] );
                            else
                            {
                                *p0 = add_mode ? *p0 + F32[0] : F32[0];
                                *p1 = add_mode ? *p1 + F32[1] : F32[1];
                                *p2 = add_mode ? *p2 + F32[2] : F32[2];
                            }
                        }
                        else
                        {
                            carry[0] = F32[0], carry[1] = F32[1], carry[2] = F32[2];
                        }
                    }
                }
            }
            __pipeline_wait_prior( 0 );
            __syncthreads();
        }
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
    int           nd; // stored diamonds
};

template < typename T >
__device__ __forceinline__ void project_out( const T n[3], T v[3] )
{
    const T dt = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
    v[0] -= dt * n[0], v[1] -= dt * n[1], v[2] -= dt * n[2];
}

// Free-slip rows of the cell's nodes on layer r + DR: the tangential projection of the accumulated rows plus
// the normal-normal term ann (n . src) n.  DR is a template argument so every acc / ann index is compile-time
// (a run-time choice of the layer puts both arrays in local memory).
template < int DR, typename T >
__device__ __forceinline__ void freeslip_rows( const CellParams< T >& P, int d, int x, int y, int r, T acc[2][2][2][3],
                                               const T ann[2][2][2] )
{
    const int n1 = P.n1;
#pragma unroll
    for ( int dx = 0; dx < 2; ++dx )
#pragma unroll
        for ( int dy = 0; dy < 2; ++dy )
        {
            const size_t  lat = lat_index( n1, d, x + dx, y + dy );
            const double* u   = P.coords + lat * 3;
            T             n[3] = { T( u[0] ), T( u[1] ), T( u[2] ) };
            const T       im   = rsqrt( n[0] * n[0] + n[1] * n[1] + n[2] * n[2] );
            n[0] *= im, n[1] *= im, n[2] *= im;
            T* o = acc[dx][dy][DR];
            project_out( n, o );
            const size_t i  = lat * n1 + r + DR;
            const T      un = n[0] * P.src.p[0][i] + n[1] * P.src.p[1][i] + n[2] * P.src.p[2][i];
#pragma unroll
            for ( int c = 0; c < 3; ++c )
                o[c] += ann[dx][dy][DR] * un * n[c];
        }
}

// Full contribution of cell (d, x, y, r) to its 8 nodes, acc[dx][dy][dr][c].  DIAG: the diagonal-mode apply
// (kerngen :540-575).  Every per-node array is indexed with compile-time indices (loops fully unrolled,
// wedge_node), so none of them goes to local memory; the unit normals are kept per lateral vertex (the top
// and bottom nodes of a wedge share them), and one source array holds the source (DIAG) or the source with
// the normal part of free-slip nodes removed (the only form the full apply reads).
template < bool DIAG, typename T >
__device__ __forceinline__ void cell_full( const CellParams< T >& P, int d, int x, int y, int r, T acc[2][2][2][3] )
{
    const int  N = P.N, n1 = P.n1;
    const bool at_cmb = r == 0, at_surf = r == N - 1;
    const bool cmb_dir = at_cmb && P.bc_cmb == TN_BC_DIRICHLET, surf_dir = at_surf && P.bc_surf == TN_BC_DIRICHLET;
    const bool cmb_fs = at_cmb && P.bc_cmb == TN_BC_FREESLIP, surf_fs = at_surf && P.bc_surf == TN_BC_FREESLIP;

    T ann[2][2][2];
#pragma unroll
    for ( int i = 0; i < 8; ++i )
    {
        ann[i >> 2][( i >> 1 ) & 1][i & 1] = T( 0 );
#pragma unroll
        for ( int c = 0; c < 3; ++c )
            acc[i >> 2][( i >> 1 ) & 1][i & 1][c] = T( 0 );
    }
    const T r0 = P.radii[d * n1 + r], r1 = P.radii[d * n1 + r + 1];

#pragma unroll
    for ( int w = 0; w < 2; ++w )
    {
        T p[3][3], nrm[3][3], kn[6], v[6][3];
#pragma unroll
        for ( int n = 0; n < 6; ++n )
        {
            const int X = x + wedge_node( w, n, 0 ), Y = y + wedge_node( w, n, 1 ), R = r + wedge_node( w, n, 2 );
            const size_t  lat = lat_index( n1, d, X, Y );
            const double* u   = P.coords + lat * 3;
            if ( n < 3 )
            {
#pragma unroll
                for ( int a = 0; a < 3; ++a )
                    p[n][a] = T( u[a] );
                // outward unit normals, needed by free-slip layers only (one reciprocal square root)
                T       nn[3] = { T( u[0] ), T( u[1] ), T( u[2] ) };
                const T im    = ( cmb_fs || surf_fs ) ? rsqrt( nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2] ) : T( 0 );
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                    nrm[n][c] = nn[c] * im;
            }
            const size_t id = lat * n1 + R;
            kn[n]           = P.k[id];
#pragma unroll
            for ( int c = 0; c < 3; ++c )
                v[n][c] = P.src.at( c )[id];
            if constexpr ( !DIAG )
                if ( ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 ) )
                    project_out( nrm[n % 3], v[n] );
        }
        T       IT[3][3];
        const T third = T( 1.0 / 3.0 );
        const T det   = wedge_jacobian_it( p[0], p[1], p[2], r0, r1, third, third, T( 0 ), IT );
        T       ksum  = 0;
#pragma unroll
        for ( int n = 0; n < 6; ++n )
            ksum += kn[n];
        const T kwJ = ( ksum / T( 6 ) ) * fabs( det );
        T       g[6][3];
#pragma unroll
        for ( int n = 0; n < 6; ++n )
        {
            T gr[3];
            grad_shape_ref( n, third, third, T( 0 ), gr );
#pragma unroll
            for ( int a = 0; a < 3; ++a )
                g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
        }
        if constexpr ( !DIAG )
        {
            T G[3][3] = { { 0 } };
#pragma unroll
            for ( int n = 0; n < 6; ++n )
            {
                if ( ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 ) )
                    continue;
#pragma unroll
                for ( int a = 0; a < 3; ++a )
#pragma unroll
                    for ( int bb = 0; bb < 3; ++bb )
                        G[a][bb] += g[n][a] * v[n][bb];
            }
            const T div = G[0][0] + G[1][1] + G[2][2];
            T       E[3][3];
#pragma unroll
            for ( int a = 0; a < 3; ++a )
#pragma unroll
                for ( int bb = 0; bb < 3; ++bb )
                    E[a][bb] = T( 0.5 ) * ( G[a][bb] + G[bb][a] );
#pragma unroll
            for ( int n = 0; n < 6; ++n )
            {
                if ( ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 ) )
                    continue;
                T* o = acc[wedge_node( w, n, 0 )][wedge_node( w, n, 1 )][wedge_node( w, n, 2 )];
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                    o[c] += kwJ * ( T( 2 ) * ( g[n][0] * E[0][c] + g[n][1] * E[1][c] + g[n][2] * E[2][c] ) -
                                    T( 2.0 / 3.0 ) * g[n][c] * div );
                if ( ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 ) )
                {
                    const T* nv = nrm[n % 3];
                    const T  gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
                    const T  ng = nv[0] * g[n][0] + nv[1] * g[n][1] + nv[2] * g[n][2];
                    ann[wedge_node( w, n, 0 )][wedge_node( w, n, 1 )][wedge_node( w, n, 2 )] += kwJ * ( gg + ng * ng * third );
                }
            }
        }
        // kept diagonal of Dirichlet nodes (there v is the unprojected source), or the diagonal mode
#pragma unroll
        for ( int n = 0; n < 6; ++n )
        {
            const bool is_dir = ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 );
            const bool is_fs  = ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 );
            if ( !( DIAG || is_dir ) )
                continue;
            T*      o  = acc[wedge_node( w, n, 0 )][wedge_node( w, n, 1 )][wedge_node( w, n, 2 )];
            const T gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
            if ( DIAG && is_fs )
            {
                T R[3][3], q[3];
                trafo_normal_tangential( nrm[n % 3], R );
#pragma unroll
                for ( int a = 0; a < 3; ++a )
                {
                    const T Rg = R[a][0] * g[n][0] + R[a][1] * g[n][1] + R[a][2] * g[n][2];
                    const T Rs = R[a][0] * v[n][0] + R[a][1] * v[n][1] + R[a][2] * v[n][2];
                    q[a]       = kwJ * ( gg + Rg * Rg * third ) * Rs;
                }
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                    o[c] += R[0][c] * q[0] + R[1][c] * q[1] + R[2][c] * q[2];
            }
            else
            {
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                    o[c] += kwJ * v[n][c] * ( gg + g[n][c] * g[n][c] * third );
            }
        }
    }
    if constexpr ( !DIAG )
    {
        if ( cmb_fs )
            freeslip_rows< 0 >( P, d, x, y, r, acc, ann );
        else if ( surf_fs )
            freeslip_rows< 1 >( P, d, x, y, r, acc, ann );
    }
}

// One thread per cell, atomics (diagonal mode and levels below the tile size).
template < typename T >
__global__ void __launch_bounds__( 128 ) kerngen_cell_kernel( CellParams< T > P )
{
    const int       N = P.N, n1 = P.n1;
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) P.nd * N * N * N )
        return;
    const int r = int( t % N );
    const int y = int( ( t / N ) % N );
    const int x = int( ( t / ( (long long) N * N ) ) % N );
    const int d = int( t / ( (long long) N * N * N ) );
    T         acc[2][2][2][3];
    if ( P.diag )
        cell_full< true >( P, d, x, y, r, acc );
    else
        cell_full< false >( P, d, x, y, r, acc );
#pragma unroll
    for ( int dx = 0; dx < 2; ++dx )
#pragma unroll
        for ( int dy = 0; dy < 2; ++dy )
#pragma unroll
            for ( int dr = 0; dr < 2; ++dr )
            {
                const size_t i = lat_index( n1, d, x + dx, y + dy ) * n1 + r + dr;
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                    atomicAdd( P.dst.at( c ) + i, acc[dx][dy][dr][c] );
            }
}

// Boundary cell layers, cell-centric: one thread per cell of the CMB layer
// (r = 0) and / or the SURFACE layer (r = N - 1), both wedges with the full
// boundary treatment of cell_full, atomics onto the values the tile kernel
// wrote (it leaves these cells out).  Neighbouring threads are neighbouring
// cells in y of one layer.
#ifndef TN_BCELL_MINBLOCKS
#define TN_BCELL_MINBLOCKS 1 // resident 128-thread blocks per SM the boundary-cell kernel is compiled for
#endif
template < typename T >
__global__ void __launch_bounds__( 128, TN_BCELL_MINBLOCKS ) kerngen_bcell_kernel( CellParams< T > P, int sides )
{
    const int       N = P.N, n1 = P.n1;
    const long long per = (long long) P.nd * N * N;
    const long long t   = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= per * ( sides == 3 ? 2 : 1 ) )
        return;
    const int side = sides == 3 ? int( t / per ) : ( sides == 1 ? 0 : 1 );
    const int r    = side == 0 ? 0 : N - 1;
    const int y    = int( t % N );
    const int x    = int( ( t / N ) % N );
    const int d    = int( ( t % per ) / ( (long long) N * N ) );
    T         acc[2][2][2][3];
    cell_full< false >( P, d, x, y, r, acc );
#pragma unroll
    for ( int dx = 0; dx < 2; ++dx )
#pragma unroll
        for ( int dy = 0; dy < 2; ++dy )
#pragma unroll
            for ( int dr = 0; dr < 2; ++dr )
            {
                const size_t i = lat_index( n1, d, x + dx, y + dy ) * n1 + r + dr;
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                    atomicAdd( P.dst.at( c ) + i, acc[dx][dy][dr][c] );
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

// <m_j, u> over owned nodes for the three rotation modes m_j = e_j x x:
// sum over owned lateral columns of c_lat x (sum_r rad_r u(lat, r)), c the
// unit lateral position.  One warp per column (lanes along r, coalesced);
// the cross product is linear, so every lane crosses its own part of the
// column's radial sum and keeps accumulating across columns in FP64, and the
// lanes are combined once, in the compensated block / grid reduction.  Indices
// are 32-bit (nlat < 2^32 at every level).
template < typename T >
__global__ void __launch_bounds__( 256 ) penalty_dots_kernel( size_t nlat, int n1, const double* __restrict__ coords,
                                                              const T* __restrict__ radii, Ptr3< const T > src,
                                                              const uint8_t* __restrict__ lat_owned, double* partials,
                                                              unsigned int* counter, double* result, double eps,
                                                              Mat3 ginv )
{
    const int      lane  = threadIdx.x & 31;
    const unsigned warp  = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
    const unsigned warps = ( gridDim.x * blockDim.x ) >> 5;
    const unsigned per   = unsigned( n1 ) * unsigned( n1 ), nl = unsigned( nlat );
    const T *      s0 = src.at( 0 ), *s1 = src.at( 1 ), *s2 = src.at( 2 );
    double         sum[3] = { 0.0, 0.0, 0.0 };
    for ( unsigned lat = warp; lat < nl; lat += warps )
    {
        if ( !lat_owned[lat] )
            continue;
        const T*       rd   = radii + ( lat / per ) * unsigned( n1 );
        const unsigned base = lat * unsigned( n1 );
        double         v0 = 0.0, v1 = 0.0, v2 = 0.0;
        for ( int r = lane; r < n1; r += 32 )
        {
            const double rad = double( rd[r] );
            v0 += rad * double( s0[base + r] );
            v1 += rad * double( s1[base + r] );
            v2 += rad * double( s2[base + r] );
        }
        const double* c = coords + size_t( lat ) * 3;
        const double  c0 = c[0], c1 = c[1], c2 = c[2];
        sum[0] += c1 * v2 - c2 * v1;
        sum[1] += c2 * v0 - c0 * v2;
        sum[2] += c0 * v1 - c1 * v0;
    }
    Neumaier acc[3];
    for ( int k = 0; k < 3; ++k )
        acc[k].add( sum[k] );
    // the last block also forms the penalty vector beta = eps G^-1 d in result[3..5]
    if ( block_sum_finish< 3 >( acc, partials, counter, result ) && threadIdx.x == 0 )
    {
        const double b0 = result[0], b1 = result[1], b2 = result[2];
        result[3]       = eps * ( ginv.a[0] * b0 + ginv.a[1] * b1 + ginv.a[2] * b2 );
        result[4]       = eps * ( ginv.a[3] * b0 + ginv.a[4] * b1 + ginv.a[5] * b2 );
        result[5]       = eps * ( ginv.a[6] * b0 + ginv.a[7] * b1 + ginv.a[8] * b2 );
    }
}


// blocks of the penalty-dot reduction (8 warps, one lateral column per warp
// and step): about 4 columns per warp on large meshes, one column per warp
// up to two blocks per SM on coarse ones (latency-bound there)
inline unsigned penalty_blocks( size_t nlat )
{
    size_t b = ( nlat + 31 ) / 32;
    b        = std::max( b, std::min< size_t >( ( nlat + 7 ) / 8, 296 ) );
    return unsigned( std::min< size_t >( b, kRedMaxBlocks ) );
}

template < typename T >
__global__ void penalty_axpy_kernel( size_t ns, int n1, const double* __restrict__ coords, const T* __restrict__ radii,
                                     const double* beta, Ptr3< T > dst )
{
    const double b[3] = { beta[0], beta[1], beta[2] };
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < ns; i += size_t( gridDim.x ) * blockDim.x )
    {
        const unsigned lat = unsigned( i ) / unsigned( n1 ); // ns < 2^32 at every level tn_mesh_create accepts (<= 9)
        const int      r   = int( unsigned( i ) - lat * unsigned( n1 ) );
        const int      d   = int( lat / unsigned( n1 * n1 ) );
        const double  rr  = double( radii[d * n1 + r] );
        const double* u   = coords + size_t( lat ) * 3;
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
CellParams< T > cell_params( const tn_mesh* m, const tn_epsdivdiv_params* p, const T* k, Ptr3< const T > src,
                             Ptr3< T > dst )
{
    return CellParams< T >{
        m->N, m->n1, m->d_coords, mesh_radii< T >( m ), k, src, dst, p->bc_cmb, p->bc_surface, p->diagonal, m->nd };
}

// Zeros the tile-seam node columns X = j TS (0 < j < xtiles) of dst, which the
// tile kernel then fills with two atomic halves: one block per (component,
// diamond, seam), each column a contiguous run of n1 x n1 values.
template < typename T >
__global__ void __launch_bounds__( 256 ) seam_zero_kernel( Ptr3< T > o, int n1, int ts, int seams )
{
    const int    b = blockIdx.x, j = b % seams + 1, dc = b / seams;
    const int    d = dc / 3, c = dc - 3 * d;
    T*           col = o.at( c ) + lat_index( n1, d, j * ts, 0 ) * n1;
    const int    n   = n1 * n1;
    for ( int i = threadIdx.x; i < n; i += blockDim.x )
        col[i] = T( 0 );
}

}  // namespace

// The tiled kernel over the interior layers (all layers the boundary-cell kernel does not take).
template < typename T, int TS >
int tile_launch( const tn_mesh* m, const tn_epsdivdiv_params* p, const T* k, Ptr3< const T > s, Ptr3< T > o, bool fsfs,
                 bool skip_cmb, bool skip_surf, cudaStream_t st )
{
    const int  N   = m->N;
    const int  dev = current_device();
    static int sms_of[kMaxDevices] = {};
    if ( sms_of[dev] == 0 )
        TN_CUDA_TRY( cudaDeviceGetAttribute( &sms_of[dev], cudaDevAttrMultiProcessorCount, dev ) );
    const int num_sms = sms_of[dev];
    const int       xtiles = N / TS;
    const long long items  = (long long) m->nd * xtiles * ( N + 1 );
    const int       grid   = int( std::min< long long >( (long long) num_sms * Tile< TS >::MinBlocks, items ) );
    const int       seg    = int( std::min< long long >( kSegMax, ( items + grid - 1 ) / grid ) );
    TileParams< T > P{ N,
                       m->n1,
                       xtiles,
                       seg,
                       m->nd,
                       m->d_coords,
                       mesh_radii< T >( m ),
                       k,
                       s,
                       o,
                       p->apply_mode == TN_APPLY_ADD,
                       skip_cmb,
                       skip_surf,
                       fsfs ? m->d_red_result + 3 : nullptr };
    if ( xtiles > 1 && p->apply_mode != TN_APPLY_ADD )
    {
        seam_zero_kernel< T ><<< unsigned( m->nd * 3 * ( xtiles - 1 ) ), 256, 0, st >>>( o, m->n1, TS, xtiles - 1 );
        TN_LAUNCH_CHECK();
    }
    const size_t smem      = tile_smem_bytes< T, TS >( m->n1, seg );
    static int   smem_attr[kMaxDevices] = {}; // largest dynamic shared memory set so far for this instantiation
    if ( int( smem ) > smem_attr[dev] )
    {
        TN_CUDA_TRY( cudaFuncSetAttribute( kerngen_tile_kernel< T, TS >, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int( smem ) ) );
        smem_attr[dev] = int( smem );
    }
    kerngen_tile_kernel< T, TS ><<< grid, Tile< TS >::Threads, smem, st >>>( P );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

// beta = eps G^-1 b from the three rotation dots b of the whole shell (a sharded apply: the ranks' parts summed)
__global__ void penalty_beta_kernel( const double* __restrict__ dots, double eps, Mat3 ginv, double* beta )
{
    if ( threadIdx.x == 0 && blockIdx.x == 0 )
    {
        const double b0 = dots[0], b1 = dots[1], b2 = dots[2];
        beta[0]         = eps * ( ginv.a[0] * b0 + ginv.a[1] * b1 + ginv.a[2] * b2 );
        beta[1]         = eps * ( ginv.a[3] * b0 + ginv.a[4] * b1 + ginv.a[5] * b2 );
        beta[2]         = eps * ( ginv.a[6] * b0 + ginv.a[7] * b1 + ginv.a[8] * b2 );
    }
}

// The rotation dots of src over this mesh's owned nodes into dots[0..2] (device); a whole shell's penalty needs
// the sum of these over the meshes that partition it.
template < typename T >
int penalty_dots( const tn_mesh* m, const T* const* src, double* dots, cudaStream_t st )
{
    TN_CHECK_ARG( m && src && src[0] && src[1] && src[2] && dots, "penalty_dots: null argument" );
    Ptr3< const T > s{ { src[0], src[1], src[2] } };
    Mat3            gi;
    for ( int i = 0; i < 9; ++i )
        gi.a[i] = m->penalty_gram_inv[i];
    penalty_dots_kernel< T ><<< penalty_blocks( m->nlat ), 256, 0, st >>>( m->nlat, m->n1, m->d_coords,
                                                                            mesh_radii< T >( m ), s, m->d_lat_owned,
                                                                            m->d_red_partials, m->d_red_counter,
                                                                            m->d_red_result, 1.0, gi );
    TN_LAUNCH_CHECK();
    TN_CUDA_TRY( cudaMemcpyAsync( dots, m->d_red_result, 3 * sizeof( double ), cudaMemcpyDeviceToDevice, st ) );
    return TN_OK;
}
template int penalty_dots< double >( const tn_mesh*, const double* const*, double*, cudaStream_t );
template int penalty_dots< float >( const tn_mesh*, const float* const*, double*, cudaStream_t );

// global_dots != nullptr (free-slip on both radii only): the rotation dots of the whole shell are given, so the
// penalty vector is formed from them instead of from this mesh's own dots
template < typename T >
int epsdivdiv_apply( const tn_mesh* m, const tn_epsdivdiv_params* p, const T* k, const T* const* src, T* const* dst,
                     cudaStream_t st, const double* global_dots )
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
        if ( global_dots )
            penalty_beta_kernel<<< 1, 32, 0, st >>>( global_dots, p->penalty_eps, gi, m->d_red_result + 3 );
        else
            penalty_dots_kernel< T ><<< penalty_blocks( m->nlat ), 256, 0, st >>>(
                m->nlat, m->n1, m->d_coords, mesh_radii< T >( m ), s, m->d_lat_owned, m->d_red_partials,
                m->d_red_counter, m->d_red_result, p->penalty_eps, gi );
        TN_LAUNCH_CHECK();
    }

    if ( p->diagonal || N < 8 )
    {
        if ( p->apply_mode == TN_APPLY_REPLACE )
            for ( int c = 0; c < 3; ++c )
                TN_CUDA_TRY( cudaMemsetAsync( dst[c], 0, m->ns * sizeof( T ), st ) );
        const long long cells = (long long) m->nd * N * N * N;
        kerngen_cell_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( cell_params( m, p, k, s, o ) );
        TN_LAUNCH_CHECK();
        if ( fsfs )
        {
            penalty_axpy_kernel< T ><<< 148 * 8, 256, 0, st >>>( m->ns, m->n1, m->d_coords, mesh_radii< T >( m ),
                                                                m->d_red_result + 3, o );
            TN_LAUNCH_CHECK();
        }
    }
    else
    {
        const bool skip_cmb = p->bc_cmb != TN_BC_NEUMANN, skip_surf = p->bc_surface != TN_BC_NEUMANN;
        const int  rc       = N >= 16 ? tile_launch< T, 16 >( m, p, k, s, o, fsfs, skip_cmb, skip_surf, st )
                                      : tile_launch< T, 8 >( m, p, k, s, o, fsfs, skip_cmb, skip_surf, st );
        if ( rc )
            return rc;
        if ( skip_cmb || skip_surf )
        {
            const int       sides   = skip_cmb && skip_surf ? 3 : ( skip_cmb ? 1 : 2 );
            const long long cells = (long long) m->nd * N * N * ( sides == 3 ? 2 : 1 );
            kerngen_bcell_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( cell_params( m, p, k, s, o ),
                                                                                            sides );
            TN_LAUNCH_CHECK();
        }
    }
    if ( p->comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( m, dst, 3, st );
    return TN_OK;
}

template int epsdivdiv_apply< double >( const tn_mesh*, const tn_epsdivdiv_params*, const double*, const double* const*,
                                        double* const*, cudaStream_t, const double* );
template int epsdivdiv_apply< float >( const tn_mesh*, const tn_epsdivdiv_params*, const float*, const float* const*,
                                       float* const*, cudaStream_t, const double* );

// dst += eps sum_i (m_i^T src) m_i, the fs/fs rigid-rotation penalty on every
// stored node (no halo), in two parts for the stored-matrix apply: the dots
// of src run on the mesh's side stream, forked from st, so they overlap the
// wedge kernel the caller launches on st in between; the join makes st wait
// for them before the update.  The dots use the mesh's reduction scratch:
// the caller launches no other reduction over the mesh in between.
template < typename T >
int fsfs_penalty_fork( const tn_mesh* m, double eps, const T* const* src, cudaStream_t st )
{
    Ptr3< const T > s{ { src[0], src[1], src[2] } };
    Mat3            gi;
    for ( int i = 0; i < 9; ++i )
        gi.a[i] = m->penalty_gram_inv[i];
    TN_CUDA_TRY( cudaEventRecord( m->ev_fork, st ) );
    TN_CUDA_TRY( cudaStreamWaitEvent( m->side_stream, m->ev_fork, 0 ) );
    penalty_dots_kernel< T ><<< penalty_blocks( m->nlat ), 256, 0, m->side_stream >>>(
        m->nlat, m->n1, m->d_coords, mesh_radii< T >( m ), s, m->d_lat_owned, m->d_red_partials, m->d_red_counter,
        m->d_red_result, eps, gi );
    TN_LAUNCH_CHECK();
    TN_CUDA_TRY( cudaEventRecord( m->ev_join, m->side_stream ) );
    return TN_OK;
}
template < typename T >
int fsfs_penalty_join( const tn_mesh* m, T* const* dst, cudaStream_t st )
{
    Ptr3< T > o{ { dst[0], dst[1], dst[2] } };
    TN_CUDA_TRY( cudaStreamWaitEvent( st, m->ev_join, 0 ) );
    penalty_axpy_kernel< T ><<< 148 * 8, 256, 0, st >>>( m->ns, m->n1, m->d_coords, mesh_radii< T >( m ),
                                                        m->d_red_result + 3, o );
    TN_LAUNCH_CHECK();
    return TN_OK;
}
template int fsfs_penalty_fork< double >( const tn_mesh*, double, const double* const*, cudaStream_t );
template int fsfs_penalty_fork< float >( const tn_mesh*, double, const float* const*, cudaStream_t );
template int fsfs_penalty_join< double >( const tn_mesh*, double* const*, cudaStream_t );
template int fsfs_penalty_join< float >( const tn_mesh*, float* const*, cudaStream_t );

}  // namespace tn

using namespace tn;

extern "C" int tn_epsdivdiv_apply_f64( const tn_mesh* m, const tn_epsdivdiv_params* p, const double* k,
                                       const double* const* src, double* const* dst, void* s )
{
    return epsdivdiv_apply< double >( m, p, k, src, dst, as_stream( s ), nullptr );
}
extern "C" int tn_epsdivdiv_apply_f32( const tn_mesh* m, const tn_epsdivdiv_params* p, const float* k,
                                       const float* const* src, float* const* dst, void* s )
{
    return epsdivdiv_apply< float >( m, p, k, src, dst, as_stream( s ), nullptr );
}
