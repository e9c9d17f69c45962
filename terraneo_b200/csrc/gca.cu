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
// Storage: [cell][wedge][18 x 18] with cells (d, x, y, r), r fastest, and each
// matrix COLUMN-major (entry (I, J) at J * 18 + I) so that lane I of a warp
// reading column J touches consecutive addresses.  FP64 5,184 B per cell.
//
// Coarsening: one 324-thread block per coarse cell, thread t owning entry
// (t / 18, t % 18) of both coarse wedges; the interpolation matrices (and, at
// the finest level, the fine wedges' geometry) of all 16 fine wedges are staged
// in shared memory once, then per fine wedge T = A_f P and C += P^T T are two
// 6-term passes.  Apply: one warp per wedge, lanes 0..17 own the rows.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );
template < typename T >
int fsfs_penalty_add( const tn_mesh* m, double eps, const T* const* src, T* const* dst, cudaStream_t st );

namespace {

constexpr int kM          = 324; // entries of an 18 x 18 matrix
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

__global__ void __launch_bounds__( 64 ) local_matrices_kernel( int N, const double* __restrict__ coords,
                                                               const double* __restrict__ radii,
                                                               const double* __restrict__ k, double* __restrict__ mats )
{
    __shared__ double sg[2][6][3], skw[2];
    const long long   cell = blockIdx.x;
    const int         n1   = N + 1;
    const int         r = int( cell % N ), y = int( ( cell / N ) % N ), x = int( ( cell / ( (long long) N * N ) ) % N );
    const int         d = int( cell / ( (long long) N * N * N ) );
    if ( threadIdx.x < 2 )
        kerngen_geometry( coords, radii, k, n1, d, x, y, r, threadIdx.x, sg[threadIdx.x], skw[threadIdx.x] );
    __syncthreads();
    for ( int e = threadIdx.x; e < 2 * kM; e += blockDim.x )
    {
        const int w = e / kM, J = ( e % kM ) / 18, I = ( e % kM ) % 18;
        mats[cell * 2 * kM + e] = kerngen_entry( sg[w], skw[w], I, J );
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
                sA[t] = mats_f[( cf * 2 + w ) * kM + t]; // column-major: sA[J * 18 + I] = A(I, J)
            __syncthreads();
        }
        // T(I, J) = sum_n A(I, n + 6b) P(n, j)
        if ( live )
        {
            double v = 0.0;
            for ( int n = 0; n < 6; ++n )
            {
                const double A = FROM_K ? kerngen_entry( sG[fw], sK[fw], I, n + 6 * b ) : sA[( n + 6 * b ) * 18 + I];
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
    if ( live )
    {
        mats_c[( cell * 2 + 0 ) * kM + J * 18 + I] = acc0;
        mats_c[( cell * 2 + 1 ) * kM + J * 18 + I] = acc1;
    }
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
};

// One warp per wedge, lanes 0..17 own the rows (node = lane % 6, dim = lane / 6).
template < typename T >
__global__ void __launch_bounds__( 128 ) stored_apply_kernel( StoredParams< T > P )
{
    __shared__ T    s_src[4][18], s_sp[4][18], s_y[4][18];
    __shared__ T    s_n[4][3][3];
    const int       lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
    const long long gw   = ( blockIdx.x * (long long) blockDim.x + threadIdx.x ) >> 5;
    const int       N = P.N, n1 = P.n1;
    const long long cells = (long long) kDiamonds * N * N * N;
    if ( gw >= 2 * cells )
        return; // whole warp
    const long long cell = gw >> 1;
    const int       w    = int( gw & 1 );
    const int r = int( cell % N ), y = int( ( cell / N ) % N ), x = int( ( cell / ( (long long) N * N ) ) % N );
    const int d = int( cell / ( (long long) N * N * N ) );
    const bool at_cmb = r == 0, at_surf = r == N - 1;
    const int  bcf    = at_cmb ? P.bc_cmb : ( at_surf ? P.bc_surf : TN_BC_NEUMANN );
    const int  boff   = at_cmb ? 0 : 3; // boundary-side local nodes boff..boff+2
    const T*   M      = P.mats + ( cell * 2 + w ) * kM;

    const int    node = lane % 6, a = lane / 6;
    const bool   row  = lane < 18;
    const bool   bnd_node = bcf != TN_BC_NEUMANN && node >= boff && node < boff + 3;
    size_t       idx  = 0;
    if ( row )
    {
        idx              = lat_index( n1, d, x + kWedgeNode[w][node][0], y + kWedgeNode[w][node][1] ) * n1 + r +
              kWedgeNode[w][node][2];
        s_src[wl][lane] = P.src.p[a][idx];
    }
    if ( bcf == TN_BC_FREESLIP && lane < 3 )
    {
        const int     bn = boff + lane;
        const double* c  = P.coords + lat_index( n1, d, x + kWedgeNode[w][bn][0], y + kWedgeNode[w][bn][1] ) * 3;
        const double  mm = sqrt( c[0] * c[0] + c[1] * c[1] + c[2] * c[2] );
        for ( int q = 0; q < 3; ++q )
            s_n[wl][lane][q] = T( c[q] / mm );
    }
    __syncwarp();
    // free-slip: boundary nodes enter with their tangential part
    if ( row )
    {
        T v = s_src[wl][lane];
        if ( bcf == TN_BC_FREESLIP && bnd_node )
        {
            const T* n  = s_n[wl][node - boff];
            const T  dt = n[0] * s_src[wl][node] + n[1] * s_src[wl][node + 6] + n[2] * s_src[wl][node + 12];
            v -= dt * n[a];
        }
        s_sp[wl][lane] = v;
    }
    __syncwarp();
    T yv = T( 0 );
    if ( row )
    {
        if ( P.diag )
        {
            if ( bcf == TN_BC_FREESLIP && bnd_node )
            {
                // diagonal of R A R^T in the (n, t1, t2) basis, rotated back
                T R[3][3];
                trafo_normal_tangential( s_n[wl][node - boff], R );
                T s3[3] = { s_src[wl][node], s_src[wl][node + 6], s_src[wl][node + 12] };
                for ( int q = 0; q < 3; ++q )
                {
                    T rar = T( 0 );
                    for ( int b = 0; b < 3; ++b )
                        for ( int c = 0; c < 3; ++c )
                            rar += R[q][b] * M[( node + 6 * c ) * 18 + node + 6 * b] * R[q][c];
                    const T rs = R[q][0] * s3[0] + R[q][1] * s3[1] + R[q][2] * s3[2];
                    yv += R[q][a] * rar * rs;
                }
            }
            else
                yv = M[lane * 18 + lane] * s_src[wl][lane];
        }
        else if ( bcf == TN_BC_DIRICHLET )
        {
            const bool bi = node >= boff && node < boff + 3;
            for ( int J = 0; J < 18; ++J )
            {
                const int  nj = J % 6, b = J / 6;
                const bool bj = nj >= boff && nj < boff + 3;
                const bool masked = ( a == b ) ? ( node != nj && ( bi || bj ) ) : ( bi || bj );
                if ( !masked )
                    yv += M[J * 18 + lane] * s_src[wl][J];
            }
        }
        else
        {
            const T* sv = bcf == TN_BC_FREESLIP ? s_sp[wl] : s_src[wl];
            for ( int J = 0; J < 18; ++J )
                yv += M[J * 18 + lane] * sv[J];
        }
    }
    if ( bcf == TN_BC_FREESLIP && !P.diag )
    {
        // boundary rows: tangential part of (A P s) plus (n^T A_nn n)(n . s) n
        if ( row )
            s_y[wl][lane] = yv;
        __syncwarp();
        if ( row && bnd_node )
        {
            const T* n   = s_n[wl][node - boff];
            const T  yn  = n[0] * s_y[wl][node] + n[1] * s_y[wl][node + 6] + n[2] * s_y[wl][node + 12];
            const T  sn  = n[0] * s_src[wl][node] + n[1] * s_src[wl][node + 6] + n[2] * s_src[wl][node + 12];
            T        ann = T( 0 );
            for ( int b = 0; b < 3; ++b )
                for ( int c = 0; c < 3; ++c )
                    ann += n[b] * M[( node + 6 * c ) * 18 + node + 6 * b] * n[c];
            yv = yv - yn * n[a] + ann * sn * n[a];
        }
    }
    if ( row )
        atomicAdd( P.dst.p[a] + idx, yv );
}

__global__ void cast_array_kernel( size_t n, const double* __restrict__ src, float* __restrict__ dst )
{
    for ( size_t i = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; i < n; i += size_t( gridDim.x ) * blockDim.x )
        dst[i] = float( src[i] );
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
    const long long warps = 2LL * kDiamonds * m->N * m->N * m->N;
    stored_apply_kernel< T ><<< unsigned( ( warps * 32 + 127 ) / 128 ), 128, 0, st >>>( P );
    TN_LAUNCH_CHECK();
    if ( !p->diagonal && p->bc_cmb == TN_BC_FREESLIP && p->bc_surface == TN_BC_FREESLIP )
    {
        int rc = fsfs_penalty_add< T >( m, p->penalty_eps, src, dst, st );
        if ( rc )
            return rc;
    }
    if ( p->comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( m, dst, 3, st );
    return TN_OK;
}

}  // namespace tn

using namespace tn;

extern "C" int tn_local_matrix_count( const tn_mesh* m, size_t* entries )
{
    TN_CHECK_ARG( m && entries, "tn_local_matrix_count: null argument" );
    *entries = size_t( kDiamonds ) * m->N * m->N * m->N * 2 * kM;
    return TN_OK;
}

extern "C" int tn_kerngen_local_matrices_f64( const tn_mesh* m, const double* k, double* mats, void* s )
{
    TN_CHECK_ARG( m && mats, "tn_kerngen_local_matrices_f64: null argument" );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    local_matrices_kernel<<< unsigned( cells ), 64, 0, as_stream( s ) >>>( m->N, m->d_coords, m->d_radii, k, mats );
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
