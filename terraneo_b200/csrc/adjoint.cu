// Viscosity derivative of the epsilon-div-div form (the backward kernel of
// the adjoint viscosity gradient; no reference counterpart).
//
// The one-point kerngen operator (fe/wedge/operators/shell/
// epsilon_divdiv_kerngen.hpp:1055-1940) is linear in the nodal coefficient:
// every wedge uses k_eval = (1/6) sum of its six nodal k, so
//     d(lambda^T A(k) u) / d k_n = sum over wedges w containing n of c_w / 6,
//     c_w = lambda_w^T A_w(k = 1) u_w,
// with A_w the wedge's 18x18 action including the boundary treatment:
// Dirichlet nodes leave the coupling and keep their diagonal
// |det J| (|g_n|^2 + g_{n,c}^2 / 3); free-slip nodes enter projected on the
// tangent plane on both sides and add |det J| (|g_n|^2 + (n.g_n)^2 / 3)
// (n.u)(n.lambda).  The rigid-rotation penalty does not depend on k and
// does not enter.  In the interior c_w = |det J| (2 E(u):E(lambda) -
// 2/3 div u div lambda) at the single quadrature point.
//
// One thread per cell, the two wedges in registers, one atomic per cell node.
// Without communication the result is the derivative with respect to each
// stored copy of k (each diamond's wedges use their own copy); with the
// additive halo it is the derivative with respect to the unique node's value,
// stored on all of its copies.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st );

namespace {

template < typename T >
struct KGradParams
{
    int             N, n1;
    const double*   coords;
    const T*        radii;
    Ptr3< const T > u, lam;
    T*              out;
    int             bc_cmb, bc_surf;
};

template < typename T >
__device__ __forceinline__ void tangential( const T n[3], T v[3] )
{
    const T dt = n[0] * v[0] + n[1] * v[1] + n[2] * v[2];
    v[0] -= dt * n[0], v[1] -= dt * n[1], v[2] -= dt * n[2];
}

template < typename T >
__global__ void __launch_bounds__( 128 ) kgrad_cell_kernel( KGradParams< T > P )
{
    const int       N = P.N, n1 = P.n1;
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return;
    const int r = int( t % N );
    const int y = int( ( t / N ) % N );
    const int x = int( ( t / ( (long long) N * N ) ) % N );
    const int d = int( t / ( (long long) N * N * N ) );

    const bool at_cmb = r == 0, at_surf = r == N - 1;
    const bool cmb_dir = at_cmb && P.bc_cmb == TN_BC_DIRICHLET, surf_dir = at_surf && P.bc_surf == TN_BC_DIRICHLET;
    const bool cmb_fs = at_cmb && P.bc_cmb == TN_BC_FREESLIP, surf_fs = at_surf && P.bc_surf == TN_BC_FREESLIP;
    const T    r0 = P.radii[d * n1 + r], r1 = P.radii[d * n1 + r + 1];
    const T    third = T( 1.0 / 3.0 );

    T acc[2][2][2];
    for ( int i = 0; i < 8; ++i )
        ( &acc[0][0][0] )[i] = T( 0 );

    for ( int w = 0; w < 2; ++w )
    {
        T p[3][3], up[6][3], lp[6][3], nrm[6][3];
        T bnd = T( 0 ); // boundary diagonal terms of the wedge (before |det J|)
        bool dir[6], fs[6];
        for ( int n = 0; n < 6; ++n )
        {
            const size_t  lat = lat_index( n1, d, x + kWedgeNode[w][n][0], y + kWedgeNode[w][n][1] );
            const double* c   = P.coords + lat * 3;
            if ( n < 3 )
                for ( int a = 0; a < 3; ++a )
                    p[n][a] = T( c[a] );
            const T cc[3] = { T( c[0] ), T( c[1] ), T( c[2] ) };
            const T mm    = sqrt( cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2] );
            for ( int a = 0; a < 3; ++a )
                nrm[n][a] = cc[a] / mm;
            const size_t i = lat * n1 + r + kWedgeNode[w][n][2];
            for ( int a = 0; a < 3; ++a )
            {
                up[n][a] = P.u.p[a][i];
                lp[n][a] = P.lam.p[a][i];
            }
            dir[n] = ( cmb_dir && n < 3 ) || ( surf_dir && n >= 3 );
            fs[n]  = ( cmb_fs && n < 3 ) || ( surf_fs && n >= 3 );
        }
        T       IT[3][3];
        const T det = wedge_jacobian_it( p[0], p[1], p[2], r0, r1, third, third, T( 0 ), IT );
        T       g[6][3];
        for ( int n = 0; n < 6; ++n )
        {
            T gr[3];
            grad_shape_ref( n, third, third, T( 0 ), gr );
            for ( int a = 0; a < 3; ++a )
                g[n][a] = IT[a][0] * gr[0] + IT[a][1] * gr[1] + IT[a][2] * gr[2];
        }
        for ( int n = 0; n < 6; ++n )
        {
            const T gg = g[n][0] * g[n][0] + g[n][1] * g[n][1] + g[n][2] * g[n][2];
            if ( dir[n] )
            {
                for ( int a = 0; a < 3; ++a )
                    bnd += lp[n][a] * up[n][a] * ( gg + g[n][a] * g[n][a] * third );
            }
            else if ( fs[n] )
            {
                const T ng = nrm[n][0] * g[n][0] + nrm[n][1] * g[n][1] + nrm[n][2] * g[n][2];
                const T un = nrm[n][0] * up[n][0] + nrm[n][1] * up[n][1] + nrm[n][2] * up[n][2];
                const T ln = nrm[n][0] * lp[n][0] + nrm[n][1] * lp[n][1] + nrm[n][2] * lp[n][2];
                bnd += ( gg + ng * ng * third ) * un * ln;
                tangential( nrm[n], up[n] );
                tangential( nrm[n], lp[n] );
            }
        }
        // interior form on the coupled (non-Dirichlet) nodes
        T Gu[3][3] = { { 0 } }, Gl[3][3] = { { 0 } };
        for ( int n = 0; n < 6; ++n )
        {
            if ( dir[n] )
                continue;
            for ( int a = 0; a < 3; ++a )
                for ( int b = 0; b < 3; ++b )
                {
                    Gu[a][b] += g[n][a] * up[n][b];
                    Gl[a][b] += g[n][a] * lp[n][b];
                }
        }
        T ee = T( 0 );
        for ( int a = 0; a < 3; ++a )
            for ( int b = 0; b < 3; ++b )
                ee += ( Gu[a][b] + Gu[b][a] ) * ( Gl[a][b] + Gl[b][a] );
        const T divu = Gu[0][0] + Gu[1][1] + Gu[2][2], divl = Gl[0][0] + Gl[1][1] + Gl[2][2];
        // 2 E(u):E(l) = (1/2) sum (Gu + Gu^T)(Gl + Gl^T)
        const T cw = fabs( det ) * ( T( 0.5 ) * ee - T( 2.0 / 3.0 ) * divu * divl + bnd ) / T( 6 );
        for ( int n = 0; n < 6; ++n )
            acc[kWedgeNode[w][n][0]][kWedgeNode[w][n][1]][kWedgeNode[w][n][2]] += cw;
    }
    for ( int dx = 0; dx < 2; ++dx )
        for ( int dy = 0; dy < 2; ++dy )
            for ( int dr = 0; dr < 2; ++dr )
                atomicAdd( P.out + lat_index( n1, d, x + dx, y + dy ) * n1 + r + dr, acc[dx][dy][dr] );
}

}  // namespace

template < typename T >
int epsdivdiv_kgrad( const tn_mesh* m, int bc_cmb, int bc_surf, int comm_mode, const T* const* u, const T* const* lam,
                     T* out, cudaStream_t st )
{
    TN_CHECK_ARG( m && u && lam && out, "epsdivdiv_kgrad: null argument" );
    TN_CHECK_ARG( bc_cmb >= 0 && bc_cmb <= 2 && bc_surf >= 0 && bc_surf <= 2, "epsdivdiv_kgrad: bad boundary code" );
    KGradParams< T > P{};
    for ( int c = 0; c < 3; ++c )
    {
        TN_CHECK_ARG( u[c] && lam[c], "epsdivdiv_kgrad: null field pointer" );
        P.u.p[c]   = u[c];
        P.lam.p[c] = lam[c];
    }
    P.N = m->N, P.n1 = m->n1, P.coords = m->d_coords, P.out = out, P.bc_cmb = bc_cmb, P.bc_surf = bc_surf;
    P.radii = sizeof( T ) == 8 ? reinterpret_cast< const T* >( m->d_radii ) : reinterpret_cast< const T* >( m->d_radii32 );
    TN_CUDA_TRY( cudaMemsetAsync( out, 0, m->ns * sizeof( T ), st ) );
    const long long cells = (long long) kDiamonds * m->N * m->N * m->N;
    kgrad_cell_kernel< T ><<< unsigned( ( cells + 127 ) / 128 ), 128, 0, st >>>( P );
    TN_LAUNCH_CHECK();
    if ( comm_mode != TN_COMM_ADDITIVE )
        return TN_OK;
    T* f[1] = { out };
    return halo_sum< T >( m, f, 1, st );
}

template int epsdivdiv_kgrad< double >( const tn_mesh*, int, int, int, const double* const*, const double* const*,
                                        double*, cudaStream_t );

}  // namespace tn

using namespace tn;

extern "C" int tn_epsdivdiv_kgrad_f64( const tn_mesh* m, int bc_cmb, int bc_surface, int comm_mode,
                                       const double* const* u, const double* const* lambda, double* grad_k, void* s )
{
    return epsdivdiv_kgrad< double >( m, bc_cmb, bc_surface, comm_mode, u, lambda, grad_k, as_stream( s ) );
}
extern "C" int tn_epsdivdiv_kgrad_f32( const tn_mesh* m, int bc_cmb, int bc_surface, int comm_mode,
                                       const float* const* u, const float* const* lambda, float* grad_k, void* s )
{
    return epsdivdiv_kgrad< float >( m, bc_cmb, bc_surface, comm_mode, u, lambda, grad_k, as_stream( s ) );
}
