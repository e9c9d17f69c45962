// The gradient-form operators: Laplace (fe/wedge/operators/shell/laplace.hpp),
// DivKGrad (div_k_grad.hpp) and VectorLaplace (vector_laplace.hpp).
//
// int k grad u . grad v with the 3x2 Felippa rule (or the 1-point rule for
// DivKGrad's single-quadpoint mode) and the curved radial map; k = 1 for
// Laplace and VectorLaplace, k interpolated by the wedge shape functions at
// each quadrature point for DivKGrad; three independent components for
// VectorLaplace.  Boundary layers decouple their boundary nodes and keep the
// diagonal, as selected per operator below.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

__device__ __constant__ const double kQP32[3][2] = { { 0.6666666666666666, 0.1666666666666667 },
                                                     { 0.1666666666666667, 0.6666666666666666 },
                                                     { 0.1666666666666667, 0.1666666666666667 } };
constexpr double kZeta32 = 0.5773502691896257;
constexpr double kW32    = 0.1666666666666667;

// Coupling of a cell's wedge nodes: all (kNeu), CMB-side nodes decoupled
// keeping their diagonal (kBot), SURFACE-side ones likewise (kTop), or the
// diagonal alone (kDiag).  It depends on the cell's radial layer only.
enum : int
{
    kNeu  = 0,
    kBot  = 1,
    kTop  = 2,
    kDiag = 3
};

template < typename T >
struct GradParams
{
    int             N, n1;
    const double*   coords;
    const T*        radii;
    const T*        k; // nodal coefficient (DivKGrad) or NULL
    Ptr3< const T > src;
    Ptr3< T >       dst;
    int             mode_first, mode_inner, mode_last; // coupling of layer 0, 1..N-2, N-1
    int             single;                            // 1-point rule instead of 3x2
};

__device__ __forceinline__ int layer_mode( int r, int N, int first, int inner, int last )
{
    return r == 0 ? first : ( r == N - 1 ? last : inner );
}

// One thread per cell (r fastest: neighbouring threads share lateral data
// and touch consecutive addresses).  Per wedge and quadrature point the
// physical gradients of the six shape functions are formed once and used
// for all NC components; the 8 node sums of the cell are kept in registers
// and added with one atomic per node and component.
template < typename T, int NC, bool HAS_K >
__global__ void __launch_bounds__( 128 ) grad_cell_kernel( GradParams< T > P )
{
    const int       N = P.N, n1 = P.n1;
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int r = int( t % N );
    const int y = int( ( t / N ) % N );
    const int x = int( ( t / ( (long long) N * N ) ) % N );
    const int d = int( t / ( (long long) N * N * N ) );

    const int mode = layer_mode( r, N, P.mode_first, P.mode_inner, P.mode_last );
    const T   r1 = P.radii[d * n1 + r], r2 = P.radii[d * n1 + r + 1];
    int       lo = 0, hi = 6;
    if ( mode == kBot )
        lo = 3;
    if ( mode == kTop )
        hi = 3;
    if ( mode == kDiag )
        lo = hi = 6;
    const int nq = P.single ? 1 : 6;

    T out[NC][2][2][2];
#pragma unroll
    for ( int c = 0; c < NC; ++c )
        for ( int i = 0; i < 8; ++i )
            ( &out[c][0][0][0] )[i] = T( 0 );
    for ( int w = 0; w < 2; ++w )
    {
        T p[3][3], s[NC][6], kv[6];
        for ( int n = 0; n < 3; ++n )
        {
            const double* u = P.coords + lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * 3;
            p[n][0] = T( u[0] ), p[n][1] = T( u[1] ), p[n][2] = T( u[2] );
        }
        for ( int n = 0; n < 6; ++n )
        {
            const size_t i = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * n1 + r +
                             kWedgeNode[w][n][2];
#pragma unroll
            for ( int c = 0; c < NC; ++c )
                s[c][n] = P.src.p[c][i];
            kv[n] = HAS_K ? P.k[i] : T( 1 );
        }
        T o[NC][6];
#pragma unroll
        for ( int c = 0; c < NC; ++c )
            for ( int n = 0; n < 6; ++n )
                o[c][n] = T( 0 );
        for ( int q = 0; q < nq; ++q )
        {
            // quad_felippa_1x1: (1/3, 1/3, 0), weight 1; 3x2: kQP32 x (-+ 1/sqrt 3), weight 1/6
            const T xi   = P.single ? T( 1.0 / 3.0 ) : T( kQP32[q >> 1][0] );
            const T eta  = P.single ? T( 1.0 / 3.0 ) : T( kQP32[q >> 1][1] );
            const T zeta = P.single ? T( 0 ) : ( ( q & 1 ) ? T( kZeta32 ) : T( -kZeta32 ) );
            const T wq   = P.single ? T( 1 ) : T( kW32 );
            T       IT[3][3];
            const T det  = wedge_jacobian_it( p[0], p[1], p[2], r1, r2, xi, eta, zeta, IT );
            T       wdet = wq * fabs( det );
            if ( HAS_K )
            {
                const T lat[3] = { T( 1 ) - xi - eta, xi, eta };
                const T rb = T( 0.5 ) * ( T( 1 ) - zeta ), rt = T( 0.5 ) * ( T( 1 ) + zeta );
                T       ke = T( 0 );
                for ( int n = 0; n < 6; ++n )
                    ke += lat[n % 3] * ( n < 3 ? rb : rt ) * kv[n];
                wdet *= ke;
            }
            T g[6][3];
            for ( int n = 0; n < 6; ++n )
            {
                T gr[3];
                grad_shape_ref( n, xi, eta, zeta, gr );
                for ( int a = 0; a < 3; ++a )
                    g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
            }
#pragma unroll
            for ( int c = 0; c < NC; ++c )
            {
                T gu[3] = { 0, 0, 0 };
                for ( int n = lo; n < hi; ++n )
                    for ( int a = 0; a < 3; ++a )
                        gu[a] += s[c][n] * g[n][a];
                for ( int n = lo; n < hi; ++n )
                    o[c][n] += wdet * ( g[n][0] * gu[0] + g[n][1] * gu[1] + g[n][2] * gu[2] );
                for ( int n = 0; n < 6; ++n )
                    if ( mode == kDiag || ( mode == kBot && n < 3 ) || ( mode == kTop && n >= 3 ) )
                        o[c][n] += wdet * s[c][n] * ( g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2] );
            }
        }
#pragma unroll
        for ( int c = 0; c < NC; ++c )
            for ( int n = 0; n < 6; ++n )
                out[c][kWedgeNode[w][n][0]][kWedgeNode[w][n][1]][kWedgeNode[w][n][2]] += o[c][n];
    }
#pragma unroll
    for ( int c = 0; c < NC; ++c )
        for ( int dx = 0; dx < 2; ++dx )
            for ( int dy = 0; dy < 2; ++dy )
                for ( int dz = 0; dz < 2; ++dz )
                    atomicAdd( P.dst.p[c] + lat_index( n1, d, x + dx, y + dy ) * n1 + r + dz, out[c][dx][dy][dz] );
}

}  // namespace

// Shared driver: Replace zeroes dst, the cell kernel accumulates, and the
// additive communication mode sums duplicated nodes.
template < typename T, int NC >
int grad_family_apply( const tn_mesh* m, const T* k, const T* const* src, T* const* dst, int mode_first,
                       int mode_inner, int mode_last, int single, int apply_mode, int comm_mode, cudaStream_t st,
                       const char* what )
{
    TN_CHECK_ARG( m && src && dst, std::string( what ) + ": null argument" );
    TN_CHECK_ARG( apply_mode == TN_APPLY_REPLACE || apply_mode == TN_APPLY_ADD, std::string( what ) + ": bad apply mode" );
    GradParams< T > P{};
    for ( int c = 0; c < 3; ++c )
    {
        P.src.p[c] = nullptr;
        P.dst.p[c] = nullptr;
    }
    for ( int c = 0; c < NC; ++c )
    {
        TN_CHECK_ARG( src[c] && dst[c], std::string( what ) + ": null field pointer" );
        P.src.p[c] = src[c];
        P.dst.p[c] = dst[c];
        if ( apply_mode == TN_APPLY_REPLACE )
            TN_CUDA_TRY( cudaMemsetAsync( dst[c], 0, m->ns * sizeof( T ), st ) );
    }
    P.N = m->N, P.n1 = m->n1, P.coords = m->d_coords;
    P.radii = sizeof( T ) == 8 ? reinterpret_cast< const T* >( m->d_radii ) : reinterpret_cast< const T* >( m->d_radii32 );
    P.k = k, P.mode_first = mode_first, P.mode_inner = mode_inner, P.mode_last = mode_last, P.single = single;
    const long long cells  = (long long) kDiamonds * m->N * m->N * m->N;
    const unsigned  blocks = unsigned( ( cells + 127 ) / 128 );
    if ( k )
        grad_cell_kernel< T, NC, true ><<< blocks, 128, 0, st >>>( P );
    else
        grad_cell_kernel< T, NC, false ><<< blocks, 128, 0, st >>>( P );
    TN_LAUNCH_CHECK();
    if ( comm_mode == TN_COMM_ADDITIVE )
        return halo_sum< T >( m, dst, NC, st );
    return TN_OK;
}

// Laplace / DivKGrad coupling (laplace.hpp:140-168, div_k_grad.hpp:455-512):
// with treat_boundary the first layer decouples its CMB nodes, the last one
// (unless it is also the first) its SURFACE nodes; diagonal mode keeps only
// the diagonal everywhere.
static void scalar_modes( int N, int treat, int diag, int& first, int& inner, int& last )
{
    inner = diag ? kDiag : kNeu;
    first = diag ? kDiag : ( treat ? kBot : kNeu );
    last  = diag ? kDiag : ( treat ? ( N == 1 ? kBot : kTop ) : kNeu );
}

template < typename T >
int laplace_apply( const tn_mesh* m, int treat, int diag, int apply_mode, int comm_mode, const T* src, T* dst,
                   cudaStream_t st )
{
    TN_CHECK_ARG( m && src && dst, "laplace_apply: null argument" );
    int f, i, l;
    scalar_modes( m->N, treat, diag, f, i, l );
    const T* s[1] = { src };
    T*       d[1] = { dst };
    return grad_family_apply< T, 1 >( m, nullptr, s, d, f, i, l, 0, apply_mode, comm_mode, st, "laplace_apply" );
}

template < typename T >
int divkgrad_apply( const tn_mesh* m, const T* k, int treat, int diag, int single, int apply_mode, int comm_mode,
                    const T* src, T* dst, cudaStream_t st )
{
    TN_CHECK_ARG( m && k && src && dst, "divkgrad_apply: null argument" );
    int f, i, l;
    scalar_modes( m->N, treat, diag, f, i, l );
    const T* s[1] = { src };
    T*       d[1] = { dst };
    return grad_family_apply< T, 1 >( m, k, s, d, f, i, l, single != 0, apply_mode, comm_mode, st, "divkgrad_apply" );
}

// VectorLaplace coupling (vector_laplace.hpp:181-210): the branch follows the
// boundary flag of the cell's own (x, y, r) node, CMB for layer 0 and
// SURFACE for every other layer, so a Dirichlet surface decouples the
// SURFACE-side nodes of every cell above layer 0.  Neumann and Dirichlet
// only (the reference aborts on free-slip).
template < typename T >
int vector_laplace_apply( const tn_mesh* m, int bc_cmb, int bc_surface, int diag, int apply_mode, int comm_mode,
                          const T* const* src, T* const* dst, cudaStream_t st )
{
    TN_CHECK_ARG( m, "vector_laplace_apply: mesh is NULL" );
    TN_CHECK_ARG( ( bc_cmb == TN_BC_NEUMANN || bc_cmb == TN_BC_DIRICHLET ) &&
                      ( bc_surface == TN_BC_NEUMANN || bc_surface == TN_BC_DIRICHLET ),
                  "vector_laplace_apply: boundary conditions must be Neumann or Dirichlet" );
    const int first = diag ? kDiag : ( bc_cmb == TN_BC_DIRICHLET ? kBot : kNeu );
    const int inner = diag ? kDiag : ( bc_surface == TN_BC_DIRICHLET ? kTop : kNeu );
    return grad_family_apply< T, 3 >( m, nullptr, src, dst, first, inner, inner, 0, apply_mode, comm_mode, st,
                                      "vector_laplace_apply" );
}

}  // namespace tn

using namespace tn;

extern "C" int tn_laplace_apply_f64( const tn_mesh* m, int treat, int diag, int am, int cm, const double* src,
                                     double* dst, void* s )
{
    return laplace_apply< double >( m, treat, diag, am, cm, src, dst, as_stream( s ) );
}
extern "C" int tn_laplace_apply_f32( const tn_mesh* m, int treat, int diag, int am, int cm, const float* src,
                                     float* dst, void* s )
{
    return laplace_apply< float >( m, treat, diag, am, cm, src, dst, as_stream( s ) );
}
extern "C" int tn_divkgrad_apply_f64( const tn_mesh* m, const double* k, int treat, int diag, int single, int am,
                                      int cm, const double* src, double* dst, void* s )
{
    return divkgrad_apply< double >( m, k, treat, diag, single, am, cm, src, dst, as_stream( s ) );
}
extern "C" int tn_divkgrad_apply_f32( const tn_mesh* m, const float* k, int treat, int diag, int single, int am,
                                      int cm, const float* src, float* dst, void* s )
{
    return divkgrad_apply< float >( m, k, treat, diag, single, am, cm, src, dst, as_stream( s ) );
}
extern "C" int tn_vector_laplace_apply_f64( const tn_mesh* m, int bcc, int bcs, int diag, int am, int cm,
                                            const double* const* src, double* const* dst, void* s )
{
    return vector_laplace_apply< double >( m, bcc, bcs, diag, am, cm, src, dst, as_stream( s ) );
}
extern "C" int tn_vector_laplace_apply_f32( const tn_mesh* m, int bcc, int bcs, int diag, int am, int cm,
                                            const float* const* src, float* const* dst, void* s )
{
    return vector_laplace_apply< float >( m, bcc, bcs, diag, am, cm, src, dst, as_stream( s ) );
}
