// The gradient-form operators: Laplace (fe/wedge/operators/shell/laplace.hpp),
// DivKGrad (div_k_grad.hpp) and VectorLaplace (vector_laplace.hpp).
//
// int k grad u . grad v with the 3x2 Felippa rule (or the 1-point rule for
// DivKGrad's single-quadpoint mode) and the curved radial map; k = 1 for
// Laplace and VectorLaplace, k interpolated by the wedge shape functions at
// each quadrature point for DivKGrad; three independent components for
// VectorLaplace.  Boundary layers decouple their boundary nodes and keep the
// diagonal, as selected per operator below.
#include <cmath>

#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

__device__ __constant__ const double kQP32[3][2] = { { 0.6666666666666666, 0.1666666666666667 },
                                                     { 0.1666666666666667, 0.6666666666666666 },
                                                     { 0.1666666666666667, 0.1666666666666667 } };
constexpr double kQP32Host[3][2] = { { 0.6666666666666666, 0.1666666666666667 },
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
    const double*   geom; // lateral quadrature table, kGeomStride doubles per wedge
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

// Factored wedge stiffness.  For x = r(zeta) ((1-xi-eta) p0 + xi p1 + eta p2)
// with a = p1 - p0, b = p2 - p0, v = a x b, c = p0 + xi a + eta b and
// h = (r2 - r1) / 2, the Jacobian columns are r a, r b, h c, so
// |det J| = r^2 h |D| with D = v . p0 (constant on the wedge) and the
// physical gradient of the shape function of node n (lateral vertex m, side
// sign s_n = -+1/2, radial factor nr_n(zeta) = (1 -+ zeta)/2) is
//     g_n = ( nr_n / r u_m + s_n lat_m / h v ) / D,
//     u_1 = b x c, u_2 = c x a, u_0 = -(u_1 + u_2).
// A quadrature point's contribution w |det J| g_i . g_j therefore splits into
// lateral factors (u_m . u_m', lat_m lat_m' |v|^2, (u_m . v) lat_m', all
// / |D|) times radial ones (h nr_i nr_j, r^2 / h, r nr), and on the
// tensor-product 3x2 rule the lateral and radial sums separate.  The lateral
// factors depend only on the triangle, so they are tabulated once per mesh:
// set 0 is the sum over the three lateral points of the 3x2 rule with weight
// 1/6, sets 1-3 the points one by one and set 4 the centroid (weights
// applied in the kernel).  Each set is U (6, symmetric), Lam (6, symmetric),
// W (9, row-major).  Mathematically the same stiffness as the per-point
// Jacobian of fe/wedge/integrands.hpp, evaluated with far fewer operations.
constexpr int kGeomSet    = 21;
constexpr int kGeomStride = 5 * kGeomSet;

// radial factors of one set: R[li + lj] (bottom/top node pairs), S2, P[l]
template < typename T >
struct Radial
{
    T R[3], S2, P[2];
};

template < typename T >
__device__ __forceinline__ void add_set( T A[21], const double* __restrict__ G, const Radial< T >& f )
{
    T U[3][3], Lm[3][3], W[3][3];
    U[0][0] = T( G[0] ), U[0][1] = U[1][0] = T( G[1] ), U[0][2] = U[2][0] = T( G[2] );
    U[1][1] = T( G[3] ), U[1][2] = U[2][1] = T( G[4] ), U[2][2] = T( G[5] );
    Lm[0][0] = T( G[6] ), Lm[0][1] = Lm[1][0] = T( G[7] ), Lm[0][2] = Lm[2][0] = T( G[8] );
    Lm[1][1] = T( G[9] ), Lm[1][2] = Lm[2][1] = T( G[10] ), Lm[2][2] = T( G[11] );
#pragma unroll
    for ( int i = 0; i < 9; ++i )
        ( &W[0][0] )[i] = T( G[12 + i] );
    int e = 0;
#pragma unroll
    for ( int i = 0; i < 6; ++i )
#pragma unroll
        for ( int j = i; j < 6; ++j )
        {
            const int li = i / 3, lj = j / 3, mi = i % 3, mj = j % 3;
            const T   si = li ? T( 0.5 ) : T( -0.5 ), sj = lj ? T( 0.5 ) : T( -0.5 );
            A[e++] += f.R[li + lj] * U[mi][mj] + ( si * sj ) * f.S2 * Lm[mi][mj] + sj * f.P[li] * W[mi][mj] +
                      si * f.P[lj] * W[mj][mi];
        }
}

__host__ __device__ constexpr int sym6( int i, int j )
{
    return i <= j ? 6 * i - i * ( i - 1 ) / 2 + j - i : 6 * j - j * ( j - 1 ) / 2 + i - j;
}

// One thread per cell (r fastest: neighbouring threads share the lateral
// table entry and touch consecutive addresses).  Each wedge's symmetric 6x6
// matrix is formed from its table entry and the layer's radial factors and
// applied to all NC components; the 8 node sums of the cell are kept in
// registers and added with one atomic per node and component.
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
    const T   h = T( 0.5 ) * ( r2 - r1 );
    bool      cpl[6];
#pragma unroll
    for ( int n = 0; n < 6; ++n )
        cpl[n] = mode == kNeu || ( mode == kBot && n >= 3 ) || ( mode == kTop && n < 3 );

    T out[NC][2][2][2];
#pragma unroll
    for ( int c = 0; c < NC; ++c )
        for ( int i = 0; i < 8; ++i )
            ( &out[c][0][0][0] )[i] = T( 0 );
#pragma unroll
    for ( int w = 0; w < 2; ++w )
    {
        const double* G = P.geom + ( ( ( size_t( d ) * N + x ) * N + y ) * 2 + w ) * kGeomStride;
        T             s[NC][6], kv[6];
#pragma unroll
        for ( int n = 0; n < 6; ++n )
        {
            const size_t i = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] ) * n1 + r +
                             kWedgeNode[w][n][2];
#pragma unroll
            for ( int c = 0; c < NC; ++c )
                s[c][n] = P.src.p[c][i];
            kv[n] = HAS_K ? P.k[i] : T( 1 );
        }
        T A[21];
#pragma unroll
        for ( int e = 0; e < 21; ++e )
            A[e] = T( 0 );
        if ( P.single )
        {
            // quad_felippa_1x1: (1/3, 1/3, 0), weight 1; k at the centroid is the mean of the six
            T ke = T( 1 );
            if ( HAS_K )
                ke = ( kv[0] + kv[1] + kv[2] + kv[3] + kv[4] + kv[5] ) * T( 1.0 / 6.0 );
            const T    rm = r1 + h;
            Radial< T > f;
            f.R[0] = f.R[1] = f.R[2] = ke * h * T( 0.25 );
            f.S2                     = ke * rm * rm / h;
            f.P[0] = f.P[1] = ke * rm * T( 0.5 );
            add_set( A, G + 4 * kGeomSet, f );
        }
        else if ( !HAS_K )
        {
            Radial< T > f{};
#pragma unroll
            for ( int zq = 0; zq < 2; ++zq )
            {
                const T zeta = zq ? T( kZeta32 ) : T( -kZeta32 );
                const T nb = T( 0.5 ) * ( T( 1 ) - zeta ), nt = T( 0.5 ) * ( T( 1 ) + zeta );
                const T rr = r1 + h * ( T( 1 ) + zeta );
                f.R[0] += h * nb * nb, f.R[1] += h * nb * nt, f.R[2] += h * nt * nt;
                f.S2 += rr * rr / h;
                f.P[0] += rr * nb, f.P[1] += rr * nt;
            }
            add_set( A, G, f );
        }
        else
        {
#pragma unroll
            for ( int q = 0; q < 3; ++q )
            {
                const T lat[3] = { T( 1.0 - kQP32[q][0] - kQP32[q][1] ), T( kQP32[q][0] ), T( kQP32[q][1] ) };
                const T kb = lat[0] * kv[0] + lat[1] * kv[1] + lat[2] * kv[2];
                const T kt = lat[0] * kv[3] + lat[1] * kv[4] + lat[2] * kv[5];
                Radial< T > f{};
#pragma unroll
                for ( int zq = 0; zq < 2; ++zq )
                {
                    const T zeta = zq ? T( kZeta32 ) : T( -kZeta32 );
                    const T nb = T( 0.5 ) * ( T( 1 ) - zeta ), nt = T( 0.5 ) * ( T( 1 ) + zeta );
                    const T rr = r1 + h * ( T( 1 ) + zeta );
                    const T wk = T( kW32 ) * ( nb * kb + nt * kt );
                    f.R[0] += wk * h * nb * nb, f.R[1] += wk * h * nb * nt, f.R[2] += wk * h * nt * nt;
                    f.S2 += wk * rr * rr / h;
                    f.P[0] += wk * rr * nb, f.P[1] += wk * rr * nt;
                }
                add_set( A, G + ( 1 + q ) * kGeomSet, f );
            }
        }
#pragma unroll
        for ( int c = 0; c < NC; ++c )
        {
            T sc[6];
#pragma unroll
            for ( int n = 0; n < 6; ++n )
                sc[n] = cpl[n] ? s[c][n] : T( 0 );
#pragma unroll
            for ( int i = 0; i < 6; ++i )
            {
                T acc = T( 0 );
#pragma unroll
                for ( int j = 0; j < 6; ++j )
                    acc += A[sym6( i, j )] * sc[j];
                if ( !cpl[i] )
                    acc = A[sym6( i, i )] * s[c][i];
                out[c][kWedgeNode[w][i][0]][kWedgeNode[w][i][1]][kWedgeNode[w][i][2]] += acc;
            }
        }
    }
#pragma unroll
    for ( int c = 0; c < NC; ++c )
        for ( int dx = 0; dx < 2; ++dx )
            for ( int dy = 0; dy < 2; ++dy )
                for ( int dz = 0; dz < 2; ++dz )
                    atomicAdd( P.dst.p[c] + lat_index( n1, d, x + dx, y + dy ) * n1 + r + dz, out[c][dx][dy][dz] );
}

// Host tabulation of the lateral factors (double), one entry per wedge.
void build_grad_geometry( const tn_mesh* m, std::vector< double >& G )
{
    const int    N = m->N, n1 = m->n1;
    const int    wn[2][3][2] = { { { 0, 0 }, { 1, 0 }, { 0, 1 } }, { { 1, 1 }, { 0, 1 }, { 1, 0 } } };
    const double pts[4][2]   = { { kQP32Host[0][0], kQP32Host[0][1] },
                                 { kQP32Host[1][0], kQP32Host[1][1] },
                                 { kQP32Host[2][0], kQP32Host[2][1] },
                                 { 1.0 / 3.0, 1.0 / 3.0 } };
    auto cross = []( const double* a, const double* b, double* o ) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto dotp = []( const double* a, const double* b ) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    G.assign( size_t( kDiamonds ) * N * N * 2 * kGeomStride, 0.0 );
    for ( int d = 0; d < kDiamonds; ++d )
        for ( int x = 0; x < N; ++x )
            for ( int y = 0; y < N; ++y )
                for ( int w = 0; w < 2; ++w )
                {
                    double* g = G.data() + ( ( ( size_t( d ) * N + x ) * N + y ) * 2 + w ) * kGeomStride;
                    const double* p[3];
                    for ( int k = 0; k < 3; ++k )
                        p[k] = m->h_coords.data() + lat_index( n1, d, x + wn[w][k][0], y + wn[w][k][1] ) * 3;
                    double a[3], b[3], v[3];
                    for ( int k = 0; k < 3; ++k )
                        a[k] = p[1][k] - p[0][k], b[k] = p[2][k] - p[0][k];
                    cross( a, b, v );
                    const double sig = 1.0 / std::fabs( dotp( v, p[0] ) ), vv = dotp( v, v );
                    for ( int q = 0; q < 4; ++q )
                    {
                        const double xi = pts[q][0], eta = pts[q][1];
                        const double lat[3] = { 1.0 - xi - eta, xi, eta };
                        double       c[3], u[3][3];
                        for ( int k = 0; k < 3; ++k )
                            c[k] = p[0][k] + xi * a[k] + eta * b[k];
                        cross( b, c, u[1] );
                        cross( c, a, u[2] );
                        for ( int k = 0; k < 3; ++k )
                            u[0][k] = -( u[1][k] + u[2][k] );
                        double set[kGeomSet];
                        int    e = 0;
                        for ( int i = 0; i < 3; ++i )
                            for ( int j = i; j < 3; ++j )
                                set[e++] = sig * dotp( u[i], u[j] );
                        for ( int i = 0; i < 3; ++i )
                            for ( int j = i; j < 3; ++j )
                                set[e++] = sig * lat[i] * lat[j] * vv;
                        for ( int i = 0; i < 3; ++i )
                            for ( int j = 0; j < 3; ++j )
                                set[e++] = sig * dotp( u[i], v ) * lat[j];
                        for ( int k = 0; k < kGeomSet; ++k )
                        {
                            g[( 1 + q ) * kGeomSet + k] = set[k];
                            if ( q < 3 )
                                g[k] += kW32 * set[k];
                        }
                    }
                }
}

const double* grad_geometry( const tn_mesh* m )
{
    tn_mesh*                     mm = const_cast< tn_mesh* >( m );
    std::lock_guard< std::mutex > lock( mm->geom_mutex );
    if ( !mm->d_grad_geom )
    {
        std::vector< double > G;
        build_grad_geometry( m, G );
        double* p = nullptr;
        if ( cudaMalloc( &p, G.size() * sizeof( double ) ) != cudaSuccess )
            return nullptr;
        if ( cudaMemcpy( p, G.data(), G.size() * sizeof( double ), cudaMemcpyHostToDevice ) != cudaSuccess )
        {
            cudaFree( p );
            return nullptr;
        }
        mm->d_grad_geom = p;
    }
    return mm->d_grad_geom;
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
    P.N = m->N, P.n1 = m->n1, P.geom = grad_geometry( m );
    if ( !P.geom )
    {
        set_error( std::string( what ) + ": allocating the lateral quadrature table failed" );
        return TN_ERR_NOMEM;
    }
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
