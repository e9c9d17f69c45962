// Shell mesh: geometry generation (host), masks, duplicated-node map and the
// additive halo kernel.
//
// Geometry follows grid/shell/spherical_shell.hpp: the 10 icosahedral diamonds
// (:420-559) are refined by recursive chord bisection, every new lateral point
// being normalize(p1 + p2) of its two parents (compute_node_recursive,
// :231-346); radii are uniform in [r_min, r_max] with the last one set exactly
// (uniform_shell_radii, :28).  Here the recursion is unrolled level by level,
// which computes each point once from the same parents and hence the same bits.
#include <math.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <mutex>

#include "common.cuh"

namespace tn {

static thread_local std::string g_last_error = "no error";
void set_error( const std::string& msg ) { g_last_error = msg; }

namespace {

struct V3
{
    double x, y, z;
};

V3 unit( V3 v )
{
    const double s = v.x * v.x + v.y * v.y + v.z * v.z;
    const double m = sqrt( s );
    if ( m > 1e-15 )
        v = { v.x / m, v.y / m, v.z / m };
    return v;
}

// The twelve icosahedron vertices: poles plus two staggered rings of five.
std::array< V3, 12 > icosahedron()
{
    std::array< V3, 12 > v{};
    const double         pi5 = 0.4 * asin( 1.0 );
    const double         w   = 2.0 * acos( 1.0 / ( 2.0 * sin( pi5 ) ) );
    const double         cw = cos( w ), sw = sin( w );
    v[0]  = { 0.0, 0.0, 1.0 };
    v[11] = { 0.0, 0.0, -1.0 };
    for ( int k = 1; k <= 5; ++k )
    {
        const double up = 2.0 * ( double( k ) - 0.5 ) * pi5;
        const double lo = 2.0 * ( double( k ) - 1 ) * pi5;
        v[k]            = { sw * cos( up ), sw * sin( up ), cw };
        v[k + 5]        = { sw * cos( lo ), sw * sin( lo ), -cw };
    }
    return v;
}

// Corner vertex ids of each diamond: pole, then counter-clockwise.
constexpr int kDiamondVerts[10][4] = { { 0, 5, 6, 1 },   { 0, 1, 7, 2 },  { 0, 2, 8, 3 },  { 0, 3, 9, 4 },
                                       { 0, 4, 10, 5 },  { 11, 7, 1, 6 }, { 11, 8, 2, 7 }, { 11, 9, 3, 8 },
                                       { 11, 10, 4, 9 }, { 11, 6, 5, 10 } };

void diamond_lateral_points( int diamond, int N, double* out /* [n1][n1][3] */ )
{
    const auto ico = icosahedron();
    const int  n1  = N + 1;
    auto       at  = [&]( int i, int j ) -> double* { return out + ( size_t( i ) * n1 + j ) * 3; };
    auto       put = [&]( int i, int j, V3 v ) {
        double* p = at( i, j );
        p[0] = v.x, p[1] = v.y, p[2] = v.z;
    };
    // northern diamonds run "left" = ring vertex 1, southern ones mirror it
    const int left = diamond < 5 ? 1 : 3, right = diamond < 5 ? 3 : 1;
    put( 0, 0, ico[kDiamondVerts[diamond][0]] );
    put( N, 0, ico[kDiamondVerts[diamond][left]] );
    put( N, N, ico[kDiamondVerts[diamond][2]] );
    put( 0, N, ico[kDiamondVerts[diamond][right]] );
    for ( int stride = N; stride >= 2; stride /= 2 )
    {
        const int h = stride / 2;
        for ( int i = 0; i <= N; i += h )
            for ( int j = 0; j <= N; j += h )
            {
                const int   ri = i % stride, rj = j % stride;
                const double *a = nullptr, *b = nullptr;
                if ( ri == 0 && rj == h ) // along a row
                    a = at( i, j - h ), b = at( i, j + h );
                else if ( ri == h && rj == 0 ) // along a column
                    a = at( i - h, j ), b = at( i + h, j );
                else if ( ri == h && rj == h ) // on the anti-diagonal
                    a = at( i - h, j + h ), b = at( i + h, j - h );
                else
                    continue;
                put( i, j, unit( { a[0] + b[0], a[1] + b[1], a[2] + b[2] } ) );
            }
    }
}

// a device copy of n host values (an empty array still gets a one-element allocation)
template < typename T >
int upload( const T* h, size_t n, T** d )
{
    TN_CUDA_TRY( cudaMalloc( d, std::max< size_t >( n, 1 ) * sizeof( T ) ) );
    if ( n )
        TN_CUDA_TRY( cudaMemcpy( *d, h, n * sizeof( T ), cudaMemcpyHostToDevice ) );
    return TN_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Halo kernel: one thread per (duplicate group, r, field); the copies are
// summed in ascending diamond order and the sum written to every copy.
// Coalesced along r (consecutive threads = consecutive r).
template < typename T >
__global__ void halo_sum_kernel( int n_groups, int n1, const int* __restrict__ offsets, const int* __restrict__ members,
                                 Ptr3< T > fields, int nfields )
{
    const long long tid   = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) n_groups * n1 * nfields;
    if ( tid >= total )
        return;
    const int r = int( tid % n1 );
    const int g = int( ( tid / n1 ) % n_groups );
    const int f = int( tid / ( (long long) n1 * n_groups ) );
    T*        v = fields.at( f );
    const int b = offsets[g], e = offsets[g + 1];
    T         s = 0;
    for ( int m = b; m < e; ++m )
        s += v[(size_t) members[m] * n1 + r];
    for ( int m = b; m < e; ++m )
        v[(size_t) members[m] * n1 + r] = s;
}

template < typename T >
int halo_sum( const tn_mesh* m, T* const* fields, int nfields, cudaStream_t st )
{
    TN_CHECK_ARG( m && fields && nfields >= 1 && nfields <= 3, "halo_sum: bad arguments" );
    Ptr3< T > f{};
    for ( int i = 0; i < nfields; ++i )
    {
        TN_CHECK_ARG( fields[i], "halo_sum: null field" );
        f.p[i] = fields[i];
    }
    const long long total = (long long) m->n_halo_groups * m->n1 * nfields;
    if ( total == 0 )
        return TN_OK;
    const int threads = 256;
    halo_sum_kernel< T ><<< unsigned( ( total + threads - 1 ) / threads ), threads, 0, st >>>(
        m->n_halo_groups, m->n1, m->d_halo_offsets, m->d_halo_members, f, nfields );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template int halo_sum< double >( const tn_mesh*, double* const*, int, cudaStream_t );
template int halo_sum< float >( const tn_mesh*, float* const*, int, cudaStream_t );

}  // namespace tn

using namespace tn;

extern "C" const char* tn_last_error( void ) { return tn::g_last_error.c_str(); }

namespace tn {

int shell_topology( int level, double r_min, double r_max, ShellTopology& t )
{
    TN_CHECK_ARG( level >= 1 && level <= 9, "tn_mesh_create: level must be in [1, 9]" );
    TN_CHECK_ARG( r_min < r_max, "tn_mesh_create: r_min must be strictly less than r_max" );
    t.level = level, t.N = 1 << level, t.n1 = t.N + 1;
    const int    n1 = t.n1, N = t.N;
    const size_t nlat = size_t( kDiamonds ) * n1 * n1;

    t.coords.resize( nlat * 3 );
    for ( int d = 0; d < kDiamonds; ++d )
        diamond_lateral_points( d, N, t.coords.data() + size_t( d ) * n1 * n1 * 3 );
    t.radii.resize( size_t( kDiamonds ) * n1 );
    const double step = ( r_max - r_min ) / N;
    for ( int d = 0; d < kDiamonds; ++d )
    {
        for ( int i = 0; i <= N; ++i )
            t.radii[d * n1 + i] = r_min + i * step;
        t.radii[d * n1 + N] = r_max;
    }

    // Duplicates: identical lateral points in different diamonds (the bisection
    // reproduces shared edges bit for bit).  Owner = lowest diamond id.
    std::map< std::array< uint64_t, 3 >, std::vector< int > > by_point;
    for ( size_t l = 0; l < nlat; ++l )
    {
        std::array< uint64_t, 3 > key;
        std::memcpy( key.data(), &t.coords[l * 3], 24 );
        by_point[key].push_back( int( l ) );
    }
    t.lat_owned.assign( nlat, 0 );
    t.offsets.assign( 1, 0 );
    t.members.clear();
    for ( auto& kv : by_point )
    {
        auto& v = kv.second; // lateral indices, ascending = ascending diamond id
        t.lat_owned[v[0]] = 1;
        if ( v.size() > 1 )
        {
            t.members.insert( t.members.end(), v.begin(), v.end() );
            t.offsets.push_back( int( t.members.size() ) );
        }
    }

    // FV ghost map: every lateral boundary face of a diamond is shared with
    // exactly one other diamond; both sides hold its two edge nodes bit for bit
    t.fv_ghost.assign( size_t( kDiamonds ) * 4 * N * 3, -1 );
    {
        using Key = std::array< uint64_t, 6 >;
        std::map< Key, std::vector< std::array< int, 3 > > > edges; // (diamond, side, i)
        auto edge_nodes = [&]( int side, int i, int& ax, int& ay, int& bx, int& by ) {
            if ( side < 2 )
                ax = bx = side == 0 ? 0 : N, ay = i, by = i + 1;
            else
                ay = by = side == 2 ? 0 : N, ax = i, bx = i + 1;
        };
        auto key_of = [&]( int d, int ax, int ay, int bx, int by ) {
            std::array< uint64_t, 3 > ka, kb;
            std::memcpy( ka.data(), &t.coords[( ( size_t( d ) * n1 + ax ) * n1 + ay ) * 3], 24 );
            std::memcpy( kb.data(), &t.coords[( ( size_t( d ) * n1 + bx ) * n1 + by ) * 3], 24 );
            if ( kb < ka )
                std::swap( ka, kb );
            return Key{ ka[0], ka[1], ka[2], kb[0], kb[1], kb[2] };
        };
        for ( int d = 0; d < kDiamonds; ++d )
            for ( int side = 0; side < 4; ++side )
                for ( int i = 0; i < N; ++i )
                {
                    int ax, ay, bx, by;
                    edge_nodes( side, i, ax, ay, bx, by );
                    edges[key_of( d, ax, ay, bx, by )].push_back( { d, side, i } );
                }
        for ( auto& kv : edges )
        {
            if ( kv.second.size() != 2 )
            {
                set_error( "tn_mesh_create: a diamond boundary edge is not shared by exactly two diamonds" );
                return TN_ERR_STATE;
            }
            for ( int k = 0; k < 2; ++k )
            {
                const auto& me = kv.second[k];
                const auto& ot = kv.second[1 - k];
                // the real cell of the other diamond adjacent to its boundary edge
                int x, y;
                if ( ot[1] == 0 )
                    x = 1, y = ot[2] + 1;
                else if ( ot[1] == 1 )
                    x = N, y = ot[2] + 1;
                else if ( ot[1] == 2 )
                    x = ot[2] + 1, y = 1;
                else
                    x = ot[2] + 1, y = N;
                int* e = &t.fv_ghost[( size_t( me[0] * 4 + me[1] ) * N + me[2] ) * 3];
                e[0] = ot[0], e[1] = x, e[2] = y;
            }
        }
    }

    // Gram matrix of the rigid rotations e_j x x over owned nodes, inverted:
    // the orthonormalised penalty modes m = C (e_j x x) satisfy C^T C = Gram^{-1}.
    double Gm[3][3] = { { 0 } };
    for ( size_t l = 0; l < nlat; ++l )
    {
        if ( !t.lat_owned[l] )
            continue;
        const int d = int( l / ( size_t( n1 ) * n1 ) );
        for ( int r = 0; r < n1; ++r )
        {
            const double rr = t.radii[d * n1 + r];
            const double x[3] = { t.coords[l * 3] * rr, t.coords[l * 3 + 1] * rr, t.coords[l * 3 + 2] * rr };
            const double x2   = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            for ( int i = 0; i < 3; ++i )
                for ( int j = 0; j < 3; ++j )
                    Gm[i][j] += ( i == j ? x2 : 0.0 ) - x[i] * x[j];
        }
    }
    {
        const double a = Gm[0][0], b = Gm[0][1], c = Gm[0][2], d = Gm[1][1], e = Gm[1][2], f = Gm[2][2];
        const double c00 = d * f - e * e, c01 = c * e - b * f, c02 = b * e - c * d;
        const double c11 = a * f - c * c, c12 = b * c - a * e, c22 = a * d - b * b;
        const double det = a * c00 + b * c01 + c * c02;
        const double inv[9] = { c00 / det, c01 / det, c02 / det, c01 / det, c11 / det, c12 / det, c02 / det, c12 / det, c22 / det };
        std::memcpy( t.gram_inv, inv, sizeof( inv ) );
    }
    return TN_OK;
}

int mesh_create_diamonds( const ShellTopology& t, double r_min, double r_max, int d0, int nd, tn_mesh** out )
{
    TN_CHECK_ARG( d0 >= 0 && nd >= 1 && d0 + nd <= kDiamonds, "mesh_create_diamonds: bad diamond range" );
    tn_mesh* m = new tn_mesh();
    m->level = t.level, m->N = t.N, m->n1 = t.n1;
    m->d0 = d0, m->nd = nd;
    m->r_min = r_min, m->r_max = r_max;
    const int    n1 = m->n1;
    const size_t per = size_t( n1 ) * n1, lat0 = size_t( d0 ) * per;
    m->nlat = size_t( nd ) * per;
    m->ns   = m->nlat * n1;

    m->h_coords.assign( t.coords.begin() + lat0 * 3, t.coords.begin() + ( lat0 + m->nlat ) * 3 );
    m->h_radii.assign( t.radii.begin() + size_t( d0 ) * n1, t.radii.begin() + size_t( d0 + nd ) * n1 );
    m->h_lat_owned.assign( t.lat_owned.begin() + lat0, t.lat_owned.begin() + lat0 + m->nlat );
    size_t owned = 0;
    for ( uint8_t o : m->h_lat_owned )
        owned += o;
    m->nu = owned * n1; // (10 N^2 + 2) n1 for the whole shell

    // the duplicate groups whose copies all lie in the range, as local lateral indices
    std::vector< int > offsets{ 0 }, members;
    const int          lo = int( lat0 ), hi = int( lat0 + m->nlat );
    for ( size_t g = 0; g + 1 < t.offsets.size(); ++g )
    {
        bool inside = true;
        for ( int k = t.offsets[g]; k < t.offsets[g + 1]; ++k )
            inside = inside && t.members[k] >= lo && t.members[k] < hi;
        if ( !inside )
            continue;
        for ( int k = t.offsets[g]; k < t.offsets[g + 1]; ++k )
            members.push_back( t.members[k] - lo );
        offsets.push_back( int( members.size() ) );
    }
    m->n_halo_groups = int( offsets.size() ) - 1;
    std::memcpy( m->penalty_gram_inv, t.gram_inv, sizeof( t.gram_inv ) );

    std::vector< int > lat_group( m->nlat, -1 );
    for ( int g = 0; g + 1 < int( offsets.size() ); ++g )
        for ( int k = offsets[g]; k < offsets[g + 1]; ++k )
            lat_group[members[k]] = g;

    std::vector< uint8_t > node_owned( m->ns );
    for ( size_t l = 0; l < m->nlat; ++l )
        std::memset( node_owned.data() + l * m->n1, m->h_lat_owned[l], m->n1 );
    int rc;
    std::vector< float > c32( m->h_coords.begin(), m->h_coords.end() ), r32( m->h_radii.begin(), m->h_radii.end() );
    if ( ( rc = upload( m->h_coords.data(), m->h_coords.size(), &m->d_coords ) ) ||
         ( rc = upload( m->h_radii.data(), m->h_radii.size(), &m->d_radii ) ) ||
         ( rc = upload( c32.data(), c32.size(), &m->d_coords32 ) ) ||
         ( rc = upload( r32.data(), r32.size(), &m->d_radii32 ) ) ||
         ( rc = upload( m->h_lat_owned.data(), m->h_lat_owned.size(), &m->d_lat_owned ) ) ||
         ( rc = upload( node_owned.data(), node_owned.size(), &m->d_node_owned ) ) ||
         ( rc = upload( offsets.data(), offsets.size(), &m->d_halo_offsets ) ) ||
         ( nd == kDiamonds && ( rc = upload( t.fv_ghost.data(), t.fv_ghost.size(), &m->d_fv_ghost ) ) ) ||
         ( rc = upload( members.data(), members.size(), &m->d_halo_members ) ) ||
         ( rc = upload( lat_group.data(), lat_group.size(), &m->d_lat_group ) ) )
    {
        tn_mesh_destroy( m );
        return rc;
    }
    if ( cudaMalloc( &m->d_red_partials, sizeof( double ) * kRedMaxBlocks * 8 ) != cudaSuccess ||
         cudaMalloc( &m->d_red_result, sizeof( double ) * 16 ) != cudaSuccess ||
         cudaMalloc( &m->d_red_counter, sizeof( unsigned int ) ) != cudaSuccess ||
         cudaMallocHost( &m->h_red_result, sizeof( double ) * 16 ) != cudaSuccess ||
         cudaMemset( m->d_red_counter, 0, sizeof( unsigned int ) ) != cudaSuccess ||
         cudaStreamCreateWithFlags( &m->side_stream, cudaStreamNonBlocking ) != cudaSuccess ||
         cudaEventCreateWithFlags( &m->ev_fork, cudaEventDisableTiming ) != cudaSuccess ||
         cudaEventCreateWithFlags( &m->ev_join, cudaEventDisableTiming ) != cudaSuccess )
    {
        set_error( "tn_mesh_create: device scratch, stream or event creation failed" );
        tn_mesh_destroy( m );
        return TN_ERR_NOMEM;
    }
    *out = m;
    return TN_OK;
}

}  // namespace tn

extern "C" int tn_mesh_create( int level, double r_min, double r_max, tn_mesh** out )
{
    TN_CHECK_ARG( out, "tn_mesh_create: out is NULL" );
    *out = nullptr;
    ShellTopology t;
    if ( const int rc = shell_topology( level, r_min, r_max, t ) )
        return rc;
    return mesh_create_diamonds( t, r_min, r_max, 0, kDiamonds, out );
}

extern "C" int tn_mesh_destroy( tn_mesh* m )
{
    if ( !m )
        return TN_OK;
    cudaFree( m->d_coords );
    cudaFree( m->d_radii );
    cudaFree( m->d_coords32 );
    cudaFree( m->d_radii32 );
    cudaFree( m->d_lat_owned );
    cudaFree( m->d_node_owned );
    cudaFree( m->d_halo_offsets );
    cudaFree( m->d_halo_members );
    cudaFree( m->d_lat_group );
    cudaFree( m->d_fv_ghost );
    cudaFree( m->d_fv_orient );
    cudaFree( m->d_grad_geom );
    cudaFree( m->d_stokes_geom );
    cudaFree( m->d_red_partials );
    cudaFree( m->d_red_result );
    cudaFree( m->d_red_counter );
    if ( m->h_red_result )
        cudaFreeHost( m->h_red_result );
    if ( m->side_stream )
        cudaStreamDestroy( m->side_stream );
    if ( m->ev_fork )
        cudaEventDestroy( m->ev_fork );
    if ( m->ev_join )
        cudaEventDestroy( m->ev_join );
    delete m;
    return TN_OK;
}

extern "C" int tn_mesh_dims( const tn_mesh* m, int* level, size_t* stored, size_t* unique )
{
    TN_CHECK_ARG( m, "tn_mesh_dims: mesh is NULL" );
    if ( level )
        *level = m->level;
    if ( stored )
        *stored = m->ns;
    if ( unique )
        *unique = m->nu;
    return TN_OK;
}

extern "C" int tn_mesh_geometry( const tn_mesh* m, double* coords, double* radii )
{
    TN_CHECK_ARG( m, "tn_mesh_geometry: mesh is NULL" );
    if ( coords )
        std::memcpy( coords, m->h_coords.data(), m->h_coords.size() * sizeof( double ) );
    if ( radii )
        std::memcpy( radii, m->h_radii.data(), m->h_radii.size() * sizeof( double ) );
    return TN_OK;
}

extern "C" int tn_mesh_masks( const tn_mesh* m, uint8_t* bmask, uint8_t* omask )
{
    TN_CHECK_ARG( m, "tn_mesh_masks: mesh is NULL" );
    const int n1 = m->n1;
    for ( size_t l = 0; l < m->nlat; ++l )
        for ( int r = 0; r < n1; ++r )
        {
            if ( bmask )
                bmask[l * n1 + r] = r == 0 ? 6 : ( r == n1 - 1 ? 10 : 1 );
            if ( omask )
                omask[l * n1 + r] = m->h_lat_owned[l];
        }
    return TN_OK;
}

extern "C" int tn_halo_sum_f64( const tn_mesh* m, double* const* f, int n, void* s )
{
    return halo_sum< double >( m, f, n, as_stream( s ) );
}
extern "C" int tn_halo_sum_f32( const tn_mesh* m, float* const* f, int n, void* s )
{
    return halo_sum< float >( m, f, n, as_stream( s ) );
}
