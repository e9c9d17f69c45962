// Finite-volume FCT advection-diffusion on the hex cells of the shell
// (fv/hex/operators/fct_advection_diffusion.hpp, geometry_helper.hpp,
// fv/hex/helpers.hpp, communication/shell/fv_communication.hpp).
//
// FV fields are [10][N+2][N+2][N+2] with one ghost layer (r fastest); cell
// (x, y, r), 1 <= x, y, r <= N, is the FE cell (x-1, y-1, r-1).  Lateral
// ghosts are copies of the real cells across each diamond face (the mesh's
// FV ghost map); radial ghosts hold what the boundary treatment writes.
//
// Every kernel runs one thread per interior cell, r fastest.  The cell
// geometry (face fluxes beta, face vectors S, volume M) is recomputed from the
// wedge map and the Q1 velocity in FP64 in the dt and predictor kernels, with
// the reference's face and volume quadrature sums evaluated in closed form
// (fv_geometry).  The antidiffusive fluxes are stored as six planes (SoA),
// F[n * nf + i] for neighbour n of cell i.
#include "common.cuh"
#include "wedge.cuh"

namespace tn {

namespace {

constexpr int kFvThreads = 128;

__device__ __constant__ const int kFvOff[6][3] = { { -1, 0, 0 }, { 1, 0, 0 }, { 0, -1, 0 },
                                                   { 0, 1, 0 },  { 0, 0, -1 }, { 0, 0, 1 } };

__device__ __forceinline__ size_t fv_index( int n2, int d, int x, int y, int r )
{
    return ( ( size_t( d ) * n2 + x ) * n2 + y ) * n2 + r;
}

struct FvGeom
{
    int                  N;
    const double*        coords;
    const double*        radii;
    Ptr3< const double > cen; // FV cell centres with ghosts
    Ptr3< const double > vel; // Q1 velocity (stored nodes)
    const uint8_t*       orient; // face orientation bits per cell (nullptr: the centre test)
};

__device__ __forceinline__ void cross3( const double a[3], const double b[3], double c[3] )
{
    c[0] = a[1] * b[2] - a[2] * b[1], c[1] = a[2] * b[0] - a[0] * b[2], c[2] = a[0] * b[1] - a[1] * b[0];
}

// GeometryHelper::compute_geometry (geometry_helper.hpp:180-363) in closed form.
//
// The reference integrates each face of the two wedges of the cell with a
// quadrature rule over the wedge map x = r(zeta) (p0 + xi a + eta b),
// a = p1 - p0, b = p2 - p0, r(zeta) = r1 + h (1 + zeta), h = (r2 - r1) / 2, and
// the Q1 velocity u(q) = sum_i N_i(q) u_i: beta = sum_q w_q u(q) . n(q),
// S = sum_q w_q n(q), and M = sum over the 3x2 volume rule of |det J| / 6.  On
// this map every such sum has a closed form:
//   * the radial triangles zeta = -+1 (neighbours 4, 5; 3-point rule, 1/6
//     weights): n = r^2 (a x b) is constant, each lateral shape function sums
//     to 1 over the points, so beta = r^2 / 6 (a x b) . (u_0 + u_1 + u_2) of
//     the face's nodes and S = r^2 / 2 (a x b);
//   * the quad xi = 0 (2x2 Gauss, weights 1/2 on [0,1] x [-1,1]): n = r(zeta)
//     h (b x p0), so beta = h (b x p0) . (R_b (u_0 + u_2) + R_t (u_3 + u_5)),
//     S = (r(-g) + r(g)) h (b x p0), with g = 1/sqrt(3),
//     R_b = (r(-g) (1 + g) + r(g) (1 - g)) / 4 and R_t = (r(-g) (1 - g) +
//     r(g) (1 + g)) / 4 the Gauss sums of r(zeta) times the bottom / top
//     radial shape functions; the quad eta = 0 alike with a in place of b and
//     nodes 1, 4 in place of 2, 5;
//   * det J = r(zeta)^2 h (a x b) . p0, so M = sum_w h |(a x b) . p0|
//     (r(-g)^2 + r(g)^2) / 2.
// These are the same sums (exact algebra, different rounding: ~1e-16
// relative), about 150 FP64 operations per cell instead of ~3,000.  Every face
// is then oriented from this cell towards the neighbour's centre.
// WITH_VELOCITY: the face fluxes beta (false: geometry only); WITH_S: the face vectors S, needed by the
// orientation test and the diffusion term only (with the orientation bits and no diffusivity they are dead).
template < bool WITH_VELOCITY = true, bool WITH_S = true >
__device__ void fv_geometry( const FvGeom& G, int d, int x, int y, int r, double beta[6], double& Mii, double S[6][3],
                             uint8_t* flips = nullptr )
{
    const int    N = G.N, n1 = N + 1, n2 = N + 2;
    const double r1 = G.radii[d * n1 + r - 1], r2 = G.radii[d * n1 + r];
    const double g  = 0.5773502691896258; // 1 / sqrt(3)
    const double h  = 0.5 * ( r2 - r1 );
    const double rm = r1 + h * ( 1.0 - g ), rp = r1 + h * ( 1.0 + g ); // r(-g), r(+g)
    const double Rb = 0.25 * ( rm * ( 1.0 + g ) + rp * ( 1.0 - g ) ), Rt = 0.25 * ( rm * ( 1.0 - g ) + rp * ( 1.0 + g ) );
    const double rs = rm + rp, r1s = r1 * r1, r2s = r2 * r2;
#pragma unroll
    for ( int n = 0; n < 6; ++n )
    {
        beta[n] = 0.0;
        S[n][0] = S[n][1] = S[n][2] = 0.0;
    }
    Mii = 0.0;
#pragma unroll
    for ( int w = 0; w < 2; ++w )
    {
        double p[3][3], u[6][3];
#pragma unroll
        for ( int i = 0; i < 6; ++i )
        {
            const size_t lat = lat_index( n1, d, x - 1 + kWedgeNode[w][i][0], y - 1 + kWedgeNode[w][i][1] );
            if ( i < 3 )
#pragma unroll
                for ( int c = 0; c < 3; ++c )
                    p[i][c] = G.coords[lat * 3 + c];
            const size_t id = lat * n1 + r - 1 + kWedgeNode[w][i][2];
#pragma unroll
            for ( int c = 0; c < 3; ++c )
                u[i][c] = WITH_VELOCITY ? G.vel.p[c][id] : 0.0;
        }
        double va[3], vb[3], ab[3], bp[3], ap[3];
#pragma unroll
        for ( int c = 0; c < 3; ++c )
            va[c] = p[1][c] - p[0][c], vb[c] = p[2][c] - p[0][c];
        cross3( va, vb, ab );
        cross3( vb, p[0], bp );
        cross3( va, p[0], ap );
        const int nx = w == 0 ? 0 : 1, ny = w == 0 ? 2 : 3; // the wedge's xi = 0 and eta = 0 faces
        double    bx = 0.0, by = 0.0, bl = 0.0, bt = 0.0;
#pragma unroll
        for ( int c = 0; c < 3; ++c )
        {
            bx += bp[c] * ( Rb * ( u[0][c] + u[2][c] ) + Rt * ( u[3][c] + u[5][c] ) );
            by += ap[c] * ( Rb * ( u[0][c] + u[1][c] ) + Rt * ( u[3][c] + u[4][c] ) );
            bl += ab[c] * ( u[0][c] + u[1][c] + u[2][c] );
            bt += ab[c] * ( u[3][c] + u[4][c] + u[5][c] );
            if ( WITH_S )
            {
                S[nx][c] += rs * h * bp[c];
                S[ny][c] += rs * h * ap[c];
                S[4][c] += 0.5 * r1s * ab[c];
                S[5][c] += 0.5 * r2s * ab[c];
            }
        }
        beta[nx] += h * bx;
        beta[ny] += h * by;
        beta[4] += r1s / 6.0 * bl;
        beta[5] += r2s / 6.0 * bt;
        const double D = ab[0] * p[0][0] + ab[1] * p[0][1] + ab[2] * p[0][2];
        Mii += 0.5 * h * fabs( D ) * ( rm * rm + rp * rp );
    }
    // orient every face from this cell towards the neighbour's centre: from the mesh's orientation bits (the
    // same test, made once per mesh), else the test itself
    const size_t ci   = fv_index( n2, d, x, y, r );
    unsigned     bits = 0;
    if ( G.orient )
        bits = G.orient[ci];
    else if ( WITH_S )
    {
#pragma unroll
        for ( int nb = 0; nb < 6; ++nb )
        {
            const size_t cj = fv_index( n2, d, x + kFvOff[nb][0], y + kFvOff[nb][1], r + kFvOff[nb][2] );
            double       dc = 0.0;
#pragma unroll
            for ( int a = 0; a < 3; ++a )
                dc += S[nb][a] * ( G.cen.p[a][cj] - G.cen.p[a][ci] );
            if ( dc < 0 )
                bits |= 1u << nb;
        }
    }
    if ( flips )
        *flips = uint8_t( bits );
#pragma unroll
    for ( int nb = 0; nb < 6; ++nb )
        if ( bits >> nb & 1u )
        {
            if ( WITH_S )
#pragma unroll
                for ( int a = 0; a < 3; ++a )
                    S[nb][a] = -S[nb][a];
            beta[nb] = -beta[nb];
        }
}

__device__ __forceinline__ bool cell_of_thread( int N, int& d, int& x, int& y, int& r )
{
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N * N )
        return false;
    r = int( t % N ) + 1;
    y = int( ( t / N ) % N ) + 1;
    x = int( ( t / ( (long long) N * N ) ) % N ) + 1;
    d = int( t / ( (long long) N * N * N ) );
    return true;
}

// compute_cell_centers (fv/hex/helpers.hpp:101-150)
__global__ void __launch_bounds__( kFvThreads ) cell_centers_kernel( int N, const double* __restrict__ coords,
                                                                     const double* __restrict__ radii, Ptr3< double > c )
{
    int d, x, y, r;
    if ( !cell_of_thread( N, d, x, y, r ) )
        return;
    const int    n1 = N + 1, n2 = N + 2;
    const double r1 = radii[d * n1 + r - 1], r2 = radii[d * n1 + r];
    double       vol = 0.0, acc[3] = { 0, 0, 0 };
    for ( int w = 0; w < 2; ++w )
    {
        double p[3][3];
        for ( int i = 0; i < 3; ++i )
        {
            const size_t lat = lat_index( n1, d, x - 1 + kWedgeNode[w][i][0], y - 1 + kWedgeNode[w][i][1] );
            for ( int a = 0; a < 3; ++a )
                p[i][a] = coords[lat * 3 + a];
        }
        for ( int q = 0; q < 6; ++q )
        {
            const double xi = q % 3 == 0 ? 0.6666666666666666 : 0.1666666666666667;
            const double et = q % 3 == 1 ? 0.6666666666666666 : 0.1666666666666667;
            const double ze = q < 3 ? -0.5773502691896257 : 0.5773502691896257;
            double       IT[3][3];
            const double Jw = fabs( wedge_jacobian_it( p[0], p[1], p[2], r1, r2, xi, et, ze, IT ) ) * 0.1666666666666667;
            const double rq = r1 + 0.5 * ( r2 - r1 ) * ( 1.0 + ze );
            vol += Jw;
            for ( int a = 0; a < 3; ++a )
                acc[a] += ( ( 1.0 - xi - et ) * p[0][a] + xi * p[1][a] + et * p[2][a] ) * rq * Jw;
        }
    }
    const size_t i = fv_index( n2, d, x, y, r );
    for ( int a = 0; a < 3; ++a )
        c.p[a][i] = acc[a] / vol;
}

// lateral ghost layer: thread per (ghost cell, r)
__global__ void fv_ghost_kernel( int N, const int* __restrict__ map, double* __restrict__ f )
{
    const long long t     = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) kDiamonds * 4 * N * N;
    if ( t >= total )
        return;
    const int  r     = int( t % N ) + 1;
    const long long e = t / N; // (d * 4 + side) * N + i
    const int  i     = int( e % N );
    const int  side  = int( ( e / N ) % 4 );
    const int  d     = int( e / ( 4LL * N ) );
    const int* m     = map + e * 3;
    const int  n2    = N + 2;
    const int  gx    = side == 0 ? 0 : ( side == 1 ? N + 1 : i + 1 );
    const int  gy    = side == 2 ? 0 : ( side == 3 ? N + 1 : i + 1 );
    f[fv_index( n2, d, gx, gy, r )] = f[fv_index( n2, m[0], m[1], m[2], r )];
}

// compute_dt_stable (fct_advection_diffusion.hpp:193-254): min over cells of
// M / (inflow + diffusion); positive doubles order like their bit patterns
// the face orientation bits of every interior cell (fv_geometry's centre test, no velocity)
__global__ void __launch_bounds__( kFvThreads ) orient_kernel( FvGeom G, uint8_t* bits )
{
    int d, x, y, r;
    if ( !cell_of_thread( G.N, d, x, y, r ) )
        return;
    double beta[6], Mii, S[6][3];
    fv_geometry< false >( G, d, x, y, r, beta, Mii, S, bits + fv_index( G.N + 2, d, x, y, r ) );
}

template < bool DIFFUSION >
__global__ void __launch_bounds__( kFvThreads ) dt_kernel( FvGeom G, double kappa, unsigned long long* out )
{
    int    d, x, y, r;
    double dtc = 1e300;
    if ( cell_of_thread( G.N, d, x, y, r ) )
    {
        const int n2 = G.N + 2;
        double    beta[6], Mii, S[6][3], lambda = 0.0;
        fv_geometry< true, DIFFUSION >( G, d, x, y, r, beta, Mii, S );
        const size_t ci = fv_index( n2, d, x, y, r );
        for ( int n = 0; n < 6; ++n )
        {
            if ( beta[n] < 0 )
                lambda -= beta[n];
            if ( DIFFUSION && kappa > 0 )
            {
                const size_t cj  = fv_index( n2, d, x + kFvOff[n][0], y + kFvOff[n][1], r + kFvOff[n][2] );
                double       den = 0.0, ss = 0.0;
                for ( int a = 0; a < 3; ++a )
                {
                    den += ( G.cen.p[a][cj] - G.cen.p[a][ci] ) * S[n][a];
                    ss += S[n][a] * S[n][a];
                }
                if ( den > 0 )
                    lambda += kappa * ss / den;
            }
        }
        dtc = lambda > 0 ? Mii / lambda : 1e30;
    }
    for ( int off = 16; off > 0; off >>= 1 )
        dtc = fmin( dtc, __shfl_down_sync( 0xffffffffu, dtc, off ) );
    if ( ( threadIdx.x & 31 ) == 0 )
        atomicMin( out, (unsigned long long) __double_as_longlong( dtc ) );
}

// FCTPredictorKernel (fct_advection_diffusion.hpp:262-376); DIFFUSION: kappa != 0
template < bool DIFFUSION >
__global__ void __launch_bounds__( kFvThreads )
    predictor_kernel( FvGeom G, const double* __restrict__ T, double* __restrict__ TL, double* __restrict__ F, double dt,
                      double kappa, const double* __restrict__ src, int subtract_divergence )
{
    int d, x, y, r;
    if ( !cell_of_thread( G.N, d, x, y, r ) )
        return;
    const int n2 = G.N + 2;
    double    beta[6], Mii, S[6][3];
    fv_geometry< true, DIFFUSION >( G, d, x, y, r, beta, Mii, S );
    const size_t i  = fv_index( n2, d, x, y, r );
    const size_t nf = size_t( kDiamonds ) * n2 * n2 * n2; // F holds 6 planes of nf (SoA)
    const double Ti = T[i];
    double       lo_diag = 0.0, lo_update = 0.0, bsum = 0.0;
    for ( int n = 0; n < 6; ++n )
    {
        const size_t j  = fv_index( n2, d, x + kFvOff[n][0], y + kFvOff[n][1], r + kFvOff[n][2] );
        const double Tj = T[j];
        if ( beta[n] >= 0 )
            lo_diag += beta[n];
        else
            lo_update += beta[n] * Tj;
        bsum += beta[n];
        if ( DIFFUSION ) // the diffusion term; zero without diffusivity (no centre loads)
        {
            double den = 0.0, ss = 0.0;
            for ( int a = 0; a < 3; ++a )
            {
                den += ( G.cen.p[a][j] - G.cen.p[a][i] ) * S[n][a];
                ss += S[n][a] * S[n][a];
            }
            const double dc = kappa * ( ss / den );
            lo_diag += dc;
            lo_update -= dc * Tj;
        }
        F[n * nf + i] = ( dt / Mii ) * ( fabs( beta[n] ) / 2.0 ) * ( Ti - Tj );
    }
    if ( subtract_divergence )
        lo_diag -= bsum;
    double tl = Ti - ( dt / Mii ) * ( lo_diag * Ti + lo_update );
    if ( src )
        tl += dt * src[i];
    TL[i] = tl;
}

// apply_dirichlet_bcs (fv/hex/helpers.hpp:26-64): thread per lateral column
__global__ void dirichlet_kernel( int N, double* __restrict__ T, double t_cmb, double t_surf, int cmb, int surf )
{
    const long long t = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if ( t >= (long long) kDiamonds * N * N )
        return;
    const int y = int( t % N ) + 1, x = int( ( t / N ) % N ) + 1, d = int( t / ( (long long) N * N ) );
    const int n2 = N + 2;
    if ( cmb )
        T[fv_index( n2, d, x, y, 1 )] = T[fv_index( n2, d, x, y, 0 )] = t_cmb;
    if ( surf )
        T[fv_index( n2, d, x, y, N )] = T[fv_index( n2, d, x, y, N + 1 )] = t_surf;
}

// FCTLimiterKernel (fct_advection_diffusion.hpp:486-531)
__global__ void __launch_bounds__( kFvThreads ) limiter_kernel( int N, const double* __restrict__ TL,
                                                                const double* __restrict__ F, double* __restrict__ Rp,
                                                                double* __restrict__ Rm )
{
    int d, x, y, r;
    if ( !cell_of_thread( N, d, x, y, r ) )
        return;
    const int    n2 = N + 2;
    const size_t i  = fv_index( n2, d, x, y, r );
    const size_t nf = size_t( kDiamonds ) * n2 * n2 * n2;
    const double ti = TL[i];
    double       Pp = 0.0, Pm = 0.0, tmax = ti, tmin = ti;
    for ( int n = 0; n < 6; ++n )
    {
        const double f = F[n * nf + i];
        if ( f > 0 )
            Pp += f;
        else
            Pm += f;
        const double tj = TL[fv_index( n2, d, x + kFvOff[n][0], y + kFvOff[n][1], r + kFvOff[n][2] )];
        tmax            = fmax( tmax, tj );
        tmin            = fmin( tmin, tj );
    }
    Rp[i] = Pp > 0 ? fmin( 1.0, ( tmax - ti ) / Pp ) : 1.0;
    Rm[i] = Pm < 0 ? fmin( 1.0, ( tmin - ti ) / Pm ) : 1.0;
}

// FCTCorrectionKernel (fct_advection_diffusion.hpp:605-650)
__global__ void __launch_bounds__( kFvThreads )
    correction_kernel( int N, const double* __restrict__ TL, const double* __restrict__ F,
                       const double* __restrict__ Rp, const double* __restrict__ Rm, double* __restrict__ T )
{
    int d, x, y, r;
    if ( !cell_of_thread( N, d, x, y, r ) )
        return;
    const int    n2 = N + 2;
    const size_t i  = fv_index( n2, d, x, y, r );
    const size_t nf = size_t( kDiamonds ) * n2 * n2 * n2;
    double       corr = 0.0;
    for ( int n = 0; n < 6; ++n )
    {
        const size_t j  = fv_index( n2, d, x + kFvOff[n][0], y + kFvOff[n][1], r + kFvOff[n][2] );
        const double f  = F[n * nf + i];
        const double al = f > 0 ? fmin( Rp[i], Rm[j] ) : fmin( Rm[i], Rp[j] );
        corr += al * f;
    }
    T[i] = TL[i] + corr;
}

size_t fv_size( const tn_mesh* m )
{
    const size_t n2 = size_t( m->N ) + 2;
    return size_t( kDiamonds ) * n2 * n2 * n2;
}

unsigned cell_blocks( const tn_mesh* m )
{
    return unsigned( ( (long long) kDiamonds * m->N * m->N * m->N + kFvThreads - 1 ) / kFvThreads );
}

int ghost_update( const tn_mesh* m, double* f, cudaStream_t st )
{
    const long long n = (long long) kDiamonds * 4 * m->N * m->N;
    fv_ghost_kernel<<< unsigned( ( n + 255 ) / 256 ), 256, 0, st >>>( m->N, m->d_fv_ghost, f );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

// The face orientation bits of the mesh, from its own cell centres (compute_cell_centers, the centres
// tn_fv_cell_centers_f64 gives), built on the first FCT call of the mesh: the orientation is geometry, so the
// per-step kernels read one byte per cell instead of the six neighbours' centres.
const uint8_t* fv_orientation( const tn_mesh* m, cudaStream_t st )
{
    tn_mesh*                      mm = const_cast< tn_mesh* >( m );
    std::lock_guard< std::mutex > lock( mm->geom_mutex );
    if ( !mm->d_fv_orient )
    {
        const size_t nf = fv_size( m );
        double*      c  = nullptr;
        uint8_t*     b  = nullptr;
        if ( cudaMalloc( &c, 3 * nf * sizeof( double ) ) != cudaSuccess )
            return nullptr;
        if ( cudaMalloc( &b, nf ) != cudaSuccess )
        {
            cudaFree( c );
            return nullptr;
        }
        bool ok = cudaMemsetAsync( c, 0, 3 * nf * sizeof( double ), st ) == cudaSuccess &&
                  cudaMemsetAsync( b, 0, nf, st ) == cudaSuccess;
        Ptr3< double > cp{ { c, c + nf, c + 2 * nf } };
        if ( ok )
        {
            cell_centers_kernel<<< cell_blocks( m ), kFvThreads, 0, st >>>( m->N, m->d_coords, m->d_radii, cp );
            ok = cudaGetLastError() == cudaSuccess;
        }
        for ( int a = 0; a < 3 && ok; ++a )
            ok = ghost_update( m, c + a * nf, st ) == TN_OK;
        if ( ok )
        {
            FvGeom G{};
            G.N = m->N, G.coords = m->d_coords, G.radii = m->d_radii;
            G.cen    = Ptr3< const double >{ { c, c + nf, c + 2 * nf } };
            G.orient = nullptr;
            orient_kernel<<< cell_blocks( m ), kFvThreads, 0, st >>>( G, b );
            ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize( st ) == cudaSuccess;
        }
        cudaFree( c );
        if ( !ok )
        {
            cudaFree( b );
            return nullptr;
        }
        mm->d_fv_orient = b;
    }
    return mm->d_fv_orient;
}

int make_geom( const tn_mesh* m, const double* const* vel, const double* const* cen, FvGeom& G, cudaStream_t st )
{
    TN_CHECK_ARG( vel && cen, "fct: null field list" );
    for ( int a = 0; a < 3; ++a )
    {
        TN_CHECK_ARG( vel[a] && cen[a], "fct: null field pointer" );
        G.vel.p[a] = vel[a];
        G.cen.p[a] = cen[a];
    }
    G.N = m->N, G.coords = m->d_coords, G.radii = m->d_radii;
    G.orient = fv_orientation( m, st );
    if ( !G.orient )
    {
        set_error( "fct: building the face orientation of the mesh failed" );
        return TN_ERR_CUDA;
    }
    return TN_OK;
}

}  // namespace

}  // namespace tn

using namespace tn;

extern "C" int tn_fv_field_size( const tn_mesh* m, size_t* n )
{
    TN_CHECK_ARG( m && n, "tn_fv_field_size: null argument" );
    *n = fv_size( m );
    return TN_OK;
}

extern "C" int tn_fct_workspace_size( const tn_mesh* m, size_t* n )
{
    TN_CHECK_ARG( m && n, "tn_fct_workspace_size: null argument" );
    *n = 9 * fv_size( m );
    return TN_OK;
}

extern "C" int tn_fv_ghost_update_f64( const tn_mesh* m, double* field, void* s )
{
    TN_CHECK_ARG( m && field, "tn_fv_ghost_update_f64: null argument" );
    return ghost_update( m, field, as_stream( s ) );
}

extern "C" int tn_fv_cell_centers_f64( const tn_mesh* m, double* const* centers, void* s )
{
    TN_CHECK_ARG( m && centers && centers[0] && centers[1] && centers[2], "tn_fv_cell_centers_f64: null argument" );
    cudaStream_t st = as_stream( s );
    Ptr3< double > c{ { centers[0], centers[1], centers[2] } };
    for ( int a = 0; a < 3; ++a )
        TN_CUDA_TRY( cudaMemsetAsync( centers[a], 0, sizeof( double ) * fv_size( m ), st ) );
    cell_centers_kernel<<< cell_blocks( m ), kFvThreads, 0, st >>>( m->N, m->d_coords, m->d_radii, c );
    TN_LAUNCH_CHECK();
    for ( int a = 0; a < 3; ++a )
    {
        int rc = ghost_update( m, centers[a], st );
        if ( rc )
            return rc;
    }
    return TN_OK;
}

extern "C" int tn_fct_dt_stable_f64( const tn_mesh* m, const double* const* vel, const double* const* centers,
                                     double diffusivity, double* dt_stable, void* s )
{
    TN_CHECK_ARG( m && dt_stable, "tn_fct_dt_stable_f64: null argument" );
    FvGeom G{};
    int    rc;
    cudaStream_t st = as_stream( s );
    if ( ( rc = make_geom( m, vel, centers, G, st ) ) )
        return rc;
    unsigned long long* slot = reinterpret_cast< unsigned long long* >( m->d_red_result + 12 );
    const double        init = 1e300;
    TN_CUDA_TRY( cudaMemcpyAsync( slot, &init, sizeof( double ), cudaMemcpyHostToDevice, st ) );
    if ( diffusivity != 0.0 )
        dt_kernel< true ><<< cell_blocks( m ), kFvThreads, 0, st >>>( G, diffusivity, slot );
    else
        dt_kernel< false ><<< cell_blocks( m ), kFvThreads, 0, st >>>( G, diffusivity, slot );
    TN_LAUNCH_CHECK();
    TN_CUDA_TRY( cudaMemcpyAsync( dt_stable, slot, sizeof( double ), cudaMemcpyDeviceToHost, st ) );
    TN_CUDA_TRY( cudaStreamSynchronize( st ) );
    return TN_OK;
}

extern "C" int tn_fct_apply_dirichlet_f64( const tn_mesh* m, double* T, const tn_fct_dirichlet* bcs, void* s )
{
    TN_CHECK_ARG( m && T && bcs, "tn_fct_apply_dirichlet_f64: null argument" );
    const long long n = (long long) kDiamonds * m->N * m->N;
    dirichlet_kernel<<< unsigned( ( n + 255 ) / 256 ), 256, 0, as_stream( s ) >>>(
        m->N, T, bcs->T_cmb, bcs->T_surface, bcs->apply_cmb, bcs->apply_surface );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

extern "C" int tn_fct_step_f64( const tn_mesh* m, double* T, const double* const* vel, const double* const* centers,
                                double dt, double diffusivity, const double* source, int subtract_divergence,
                                const tn_fct_dirichlet* bcs, double* workspace, void* s )
{
    TN_CHECK_ARG( m && T && workspace, "tn_fct_step_f64: null argument" );
    FvGeom G{};
    int    rc;
    cudaStream_t st = as_stream( s );
    if ( ( rc = make_geom( m, vel, centers, G, st ) ) )
        return rc;
    const size_t nf = fv_size( m );
    double *     TL = workspace, *F = workspace + nf, *Rp = workspace + 7 * nf, *Rm = workspace + 8 * nf;
    TN_CUDA_TRY( cudaMemsetAsync( TL, 0, sizeof( double ) * nf, st ) );
    TN_CUDA_TRY( cudaMemsetAsync( Rp, 0, sizeof( double ) * 2 * nf, st ) );
    // predictor (fct_advection_diffusion.hpp:384-433) on T with fresh lateral ghosts
    if ( ( rc = ghost_update( m, T, st ) ) )
        return rc;
    if ( diffusivity != 0.0 )
        predictor_kernel< true ><<< cell_blocks( m ), kFvThreads, 0, st >>>( G, T, TL, F, dt, diffusivity, source,
                                                                             subtract_divergence );
    else
        predictor_kernel< false ><<< cell_blocks( m ), kFvThreads, 0, st >>>( G, T, TL, F, dt, diffusivity, source,
                                                                              subtract_divergence );
    TN_LAUNCH_CHECK();
    if ( bcs && ( rc = tn_fct_apply_dirichlet_f64( m, TL, bcs, s ) ) )
        return rc;
    // limiter (:539-566) and correction (:658-680)
    if ( ( rc = ghost_update( m, TL, st ) ) )
        return rc;
    limiter_kernel<<< cell_blocks( m ), kFvThreads, 0, st >>>( m->N, TL, F, Rp, Rm );
    TN_LAUNCH_CHECK();
    if ( ( rc = ghost_update( m, Rp, st ) ) || ( rc = ghost_update( m, Rm, st ) ) )
        return rc;
    correction_kernel<<< cell_blocks( m ), kFvThreads, 0, st >>>( m->N, TL, F, Rp, Rm, T );
    TN_LAUNCH_CHECK();
    return TN_OK;
}
