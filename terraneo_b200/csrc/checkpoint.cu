// XDMF output and checkpoint reading (io/xdmf.hpp): the reference's file
// format, written from device fields without a host round trip through the
// field layout.
//
// Format (io/xdmf.hpp:80-145): one directory per time series with
//  * geometry.bin  node coordinates (FP32 or FP64), topology.bin six node ids
//    per wedge (int32 or int64), both once, at the first write;
//  * checkpoint_metadata.bin  version 1, subdomain counts, subdomain sizes, the
//    radii, the points' scalar bytes, one (label, type, bytes, vec_dim) record
//    per grid, ordering 0 and the global subdomain ids in file order;
//  * <label>_<step>.bin per grid and write: the nodes subdomain by subdomain in
//    (r, y, x) order with x fastest and vector components interleaved;
//  * step_<step>.xmf  the XDMF description, written after the binary data.
// Grids are written in the reference's order: FP32 scalars, FP64 scalars,
// FP32 vectors, FP64 vectors, each group in the order added.
//
// The mesh here is one subdomain per diamond (subdomain refinement level 0,
// the mantle-circulation app's default), so a checkpoint has 10 subdomains
// with global ids diamond << 57.
//
// Device work: a tiled transpose (32 x 32 tiles of the (x, r) plane through
// shared memory) converts the r-fastest SoA fields to the file order and
// type on the caller's stream; the device-to-host copy runs on the writer's
// own stream and the files are written by a host thread, so the caller's
// stream continues as soon as the conversion kernels have run.
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <memory>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace tn {
namespace {

constexpr int kTile = 32;

template < typename T >
struct CPtr3
{
    const T* p[3];
    __device__ __forceinline__ const T* at( int c ) const { return c == 0 ? p[0] : ( c == 1 ? p[1] : p[2] ); }
};

// layout [10][x][y][r] (r fastest, C SoA components) -> file order
// [10][r][y][x][C] cast to Tout.  Block (32, 8): one 32 x 32 tile of (x, r)
// at one (diamond, y) per block.
template < typename Tin, typename Tout, int C >
__global__ void __launch_bounds__( 256 ) pack_nodes_kernel( int n1, CPtr3< Tin > src, Tout* __restrict__ dst )
{
    __shared__ Tin tile[C][kTile][kTile + 1];
    const int      r0 = blockIdx.x * kTile, x0 = blockIdx.y * kTile;
    const int      d = blockIdx.z / n1, y = blockIdx.z % n1;
    for ( int i = threadIdx.y; i < kTile; i += blockDim.y )
    {
        const int x = x0 + i, r = r0 + threadIdx.x;
        if ( x < n1 && r < n1 )
        {
            const size_t id = ( ( size_t( d ) * n1 + x ) * n1 + y ) * n1 + r;
#pragma unroll
            for ( int c = 0; c < C; ++c )
                tile[c][i][threadIdx.x] = src.at( c )[id];
        }
    }
    __syncthreads();
    for ( int j = threadIdx.y; j < kTile; j += blockDim.y )
    {
        const int r = r0 + j, x = x0 + threadIdx.x;
        if ( x < n1 && r < n1 )
        {
            const size_t o = ( ( size_t( d ) * n1 + r ) * n1 + y ) * n1 + x;
#pragma unroll
            for ( int c = 0; c < C; ++c )
                dst[o * C + c] = static_cast< Tout >( tile[c][threadIdx.x][j] );
        }
    }
}

// the inverse: file order (subdomains in diamond order) -> layout, cast
template < typename Tin, typename Tout, int C >
__global__ void __launch_bounds__( 256 ) unpack_nodes_kernel( int n1, const Tin* __restrict__ src, Ptr3< Tout > dst )
{
    __shared__ Tin tile[C][kTile][kTile + 1];
    const int      r0 = blockIdx.x * kTile, x0 = blockIdx.y * kTile;
    const int      d = blockIdx.z / n1, y = blockIdx.z % n1;
    for ( int j = threadIdx.y; j < kTile; j += blockDim.y )
    {
        const int r = r0 + j, x = x0 + threadIdx.x;
        if ( x < n1 && r < n1 )
        {
            const size_t o = ( ( size_t( d ) * n1 + r ) * n1 + y ) * n1 + x;
#pragma unroll
            for ( int c = 0; c < C; ++c )
                tile[c][threadIdx.x][j] = src[o * C + c];
        }
    }
    __syncthreads();
    for ( int i = threadIdx.y; i < kTile; i += blockDim.y )
    {
        const int x = x0 + i, r = r0 + threadIdx.x;
        if ( x < n1 && r < n1 )
        {
            const size_t id = ( ( size_t( d ) * n1 + x ) * n1 + y ) * n1 + r;
#pragma unroll
            for ( int c = 0; c < C; ++c )
                dst.at( c )[id] = static_cast< Tout >( tile[c][i][threadIdx.x] );
        }
    }
}

// node coordinates in file order for nodes [n0, n0 + count): the lateral
// unit-sphere point times the radius (grid::shell::coords,
// spherical_shell.hpp:2814-2838), computed in FP64 and cast
template < typename Tout >
__global__ void geometry_kernel( int n1, size_t n0, size_t count, const double* __restrict__ coords,
                                 const double* __restrict__ radii, Tout* __restrict__ out )
{
    for ( size_t t = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; t < count; t += size_t( gridDim.x ) * blockDim.x )
    {
        const size_t  g   = n0 + t;
        const int     x   = int( g % n1 ), y = int( ( g / n1 ) % n1 ), r = int( ( g / ( size_t( n1 ) * n1 ) ) % n1 );
        const int     d   = int( g / ( size_t( n1 ) * n1 * n1 ) );
        const double* u   = coords + ( ( size_t( d ) * n1 + x ) * n1 + y ) * 3;
        const double  rad = radii[size_t( d ) * n1 + r];
        out[3 * t + 0]    = static_cast< Tout >( u[0] * rad );
        out[3 * t + 1]    = static_cast< Tout >( u[1] * rad );
        out[3 * t + 2]    = static_cast< Tout >( u[2] * rad );
    }
}

// connectivity for hex cells [c0, c0 + count) in file order (diamond, r, y, x):
// the two wedges (v0, v1, v2, v4, v5, v6) and (v3, v2, v1, v7, v6, v5) of the
// cell's corners v0..v7 = (x, y, r) + (i & 1, (i >> 1) & 1, i >> 2)
// (io/xdmf.hpp:647-690)
template < typename Ti >
__global__ void topology_kernel( int n1, size_t c0, size_t count, Ti* __restrict__ out )
{
    const int N = n1 - 1;
    for ( size_t t = blockIdx.x * size_t( blockDim.x ) + threadIdx.x; t < count; t += size_t( gridDim.x ) * blockDim.x )
    {
        const size_t c = c0 + t;
        const int    x = int( c % N ), y = int( ( c / N ) % N ), r = int( ( c / ( size_t( N ) * N ) ) % N );
        const int    d = int( c / ( size_t( N ) * N * N ) );
        const long long s1 = (long long) n1 * n1;
        const long long v0 = (long long) d * s1 * n1 + r * s1 + (long long) y * n1 + x;
        const long long v4 = v0 + s1;
        const Ti        w[12] = { Ti( v0 ),          Ti( v0 + 1 ),      Ti( v0 + n1 ),      Ti( v4 ),
                                  Ti( v4 + 1 ),      Ti( v4 + n1 ),     Ti( v0 + n1 + 1 ),  Ti( v0 + n1 ),
                                  Ti( v0 + 1 ),      Ti( v4 + n1 + 1 ), Ti( v4 + n1 ),      Ti( v4 + 1 ) };
#pragma unroll
        for ( int k = 0; k < 12; ++k )
            out[12 * t + k] = w[k];
    }
}

unsigned grid_for( size_t n ) { return unsigned( std::min< size_t >( ( n + 255 ) / 256, 148 * 16 ) ); }

dim3 tile_grid( int n1 ) { return dim3( ( n1 + kTile - 1 ) / kTile, ( n1 + kTile - 1 ) / kTile, kDiamonds * n1 ); }

std::string escape_xml( const std::string& s )
{
    std::string o;
    for ( char c : s )
        switch ( c )
        {
        case '&': o += "&amp;"; break;
        case '"': o += "&quot;"; break;
        case '\'': o += "&apos;"; break;
        case '<': o += "&lt;"; break;
        case '>': o += "&gt;"; break;
        default: o += c;
        }
    return o;
}

bool write_file( const std::string& path, const void* p, size_t n, std::string& err )
{
    FILE* f = std::fopen( path.c_str(), "wb" );
    if ( !f )
    {
        err = "cannot open " + path + " for writing";
        return false;
    }
    const bool ok = std::fwrite( p, 1, n, f ) == n;
    if ( std::fclose( f ) != 0 || !ok )
    {
        err = "short write to " + path;
        return false;
    }
    return true;
}

}  // namespace
}  // namespace tn

using namespace tn;

struct tn_xdmf_output
{
    struct Grid
    {
        std::string label;
        int         in_bytes = 8, out_bytes = 4, vec = 1;
        const void* p[3]     = { nullptr, nullptr, nullptr };
        void*       d_stage  = nullptr;
        void*       h_stage  = nullptr;
        size_t      bytes    = 0;
    };

    const tn_mesh*      m = nullptr;
    std::string         dir;
    int                 pts = 4, conn = 8, device = 0;
    std::vector< Grid > grids; // in the order added
    std::vector< int >  order; // the reference's write order (set at the first write)
    int                 counter = 0;
    bool                first_done = false;
    cudaStream_t        copy_stream = nullptr;
    cudaEvent_t         ev_packed = nullptr, ev_copied = nullptr;
    std::thread         worker;
    std::string         worker_error;

    int join()
    {
        if ( worker.joinable() )
            worker.join();
        if ( !worker_error.empty() )
        {
            set_error( "XDMF write: " + worker_error );
            worker_error.clear();
            return TN_ERR_IO;
        }
        return TN_OK;
    }

    ~tn_xdmf_output()
    {
        if ( worker.joinable() )
            worker.join();
        for ( auto& g : grids )
        {
            if ( g.d_stage )
                cudaFree( g.d_stage );
            if ( g.h_stage )
                cudaFreeHost( g.h_stage );
        }
        if ( ev_packed )
            cudaEventDestroy( ev_packed );
        if ( ev_copied )
            cudaEventDestroy( ev_copied );
        if ( copy_stream )
            cudaStreamDestroy( copy_stream );
    }

    size_t nodes() const { return m->ns; }
    size_t elements() const { return size_t( kDiamonds ) * m->N * m->N * m->N * 2; }

    std::string xmf( const std::string& step ) const
    {
        const std::string nn = std::to_string( nodes() );
        std::string       s  = "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n";
        s += "<Xdmf Version=\"2.0\">\n  <Domain>\n    <Grid GridType=\"Uniform\" Name=\"Grid\">\n";
        s += "      <Geometry Type=\"XYZ\">\n        <DataItem DataType=\"Float\" Dimensions=\"" + nn +
             " 3\" Endian=\"Little\" Format=\"Binary\" Precision=\"" + std::to_string( pts ) +
             "\">geometry.bin</DataItem>\n      </Geometry>\n";
        s += "      <Topology NumberOfElements=\"" + std::to_string( elements() ) +
             "\" Type=\"Wedge\">\n        <DataItem DataType=\"Int\" Dimensions=\"" + std::to_string( 6 * elements() ) +
             "\" Endian=\"Little\" Format=\"Binary\" Precision=\"" + std::to_string( conn ) +
             "\">topology.bin</DataItem>\n      </Topology>\n";
        for ( int i : order )
        {
            const Grid& g = grids[i];
            s += std::string( "      <Attribute AttributeType=\"" ) + ( g.vec == 1 ? "Scalar" : "Vector" ) +
                 "\" Center=\"Node\" Name=\"" + escape_xml( g.label ) +
                 "\">\n        <DataItem DataType=\"Float\" Dimensions=\"" + nn + ( g.vec == 1 ? "" : " 3" ) +
                 "\" Endian=\"Little\" Format=\"Binary\" Precision=\"" + std::to_string( g.out_bytes ) + "\">" +
                 escape_xml( g.label + "_" + step + ".bin" ) + "</DataItem>\n      </Attribute>\n";
        }
        s += "    </Grid>\n  </Domain>\n</Xdmf>\n";
        return s;
    }

    std::string metadata() const
    {
        std::string s;
        auto        i32 = [&]( int32_t v ) { s.append( reinterpret_cast< const char* >( &v ), 4 ); };
        auto        i64 = [&]( int64_t v ) { s.append( reinterpret_cast< const char* >( &v ), 8 ); };
        auto        f64 = [&]( double v ) { s.append( reinterpret_cast< const char* >( &v ), 8 ); };
        i32( 1 ); // version
        i32( 1 ); // subdomains per diamond side
        i32( 1 ); // subdomains in the radial direction
        i32( m->n1 );
        i32( m->n1 );
        i32( m->n1 );
        for ( int r = 0; r < m->n1; ++r )
            f64( m->h_radii[r] );
        i32( pts );
        i32( int32_t( order.size() ) );
        for ( int i : order )
        {
            const Grid& g = grids[i];
            i32( int32_t( g.label.size() ) );
            s += g.label;
            i32( 2 ); // float
            i32( g.out_bytes );
            i32( g.vec );
        }
        i32( 0 ); // ordering 0: global subdomain ids in file order
        for ( int d = 0; d < kDiamonds; ++d )
            i64( int64_t( d ) << 57 );
        return s;
    }

    // geometry.bin and topology.bin, through a bounded device / pinned buffer pair, on stream st
    int write_mesh( cudaStream_t st )
    {
        const size_t chunk = size_t( 64 ) << 20;
        void *       d = nullptr, *h = nullptr;
        TN_CUDA_TRY( cudaMalloc( &d, chunk ) );
        if ( cudaMallocHost( &h, chunk ) != cudaSuccess )
        {
            cudaFree( d );
            set_error( "XDMF write: pinned host allocation failed" );
            return TN_ERR_NOMEM;
        }
        int         rc = TN_OK;
        std::string err;
        auto        stream_out = [&]( const std::string& path, size_t units, size_t unit_bytes, auto launch ) {
            FILE* f = std::fopen( path.c_str(), "wb" );
            if ( !f )
            {
                err = "cannot open " + path + " for writing";
                return false;
            }
            const size_t per = chunk / unit_bytes;
            bool         ok  = true;
            for ( size_t u0 = 0; u0 < units && ok; u0 += per )
            {
                const size_t n = std::min( per, units - u0 );
                launch( u0, n, d );
                ok = cudaGetLastError() == cudaSuccess &&
                     cudaMemcpyAsync( h, d, n * unit_bytes, cudaMemcpyDeviceToHost, st ) == cudaSuccess &&
                     cudaStreamSynchronize( st ) == cudaSuccess;
                if ( !ok )
                    err = "CUDA error while writing " + path;
                else if ( std::fwrite( h, 1, n * unit_bytes, f ) != n * unit_bytes )
                {
                    ok  = false;
                    err = "short write to " + path;
                }
            }
            if ( std::fclose( f ) != 0 && ok )
            {
                ok  = false;
                err = "short write to " + path;
            }
            return ok;
        };
        const int n1 = m->n1;
        bool      ok = stream_out( dir + "/geometry.bin", nodes(), 3 * size_t( pts ), [&]( size_t u0, size_t n, void* p ) {
            if ( pts == 4 )
                geometry_kernel< float ><<< grid_for( n ), 256, 0, st >>>( n1, u0, n, m->d_coords, m->d_radii, (float*) p );
            else
                geometry_kernel< double ><<< grid_for( n ), 256, 0, st >>>( n1, u0, n, m->d_coords, m->d_radii, (double*) p );
        } );
        const size_t cells = size_t( kDiamonds ) * m->N * m->N * m->N;
        ok = ok && stream_out( dir + "/topology.bin", cells, 12 * size_t( conn ), [&]( size_t u0, size_t n, void* p ) {
                 if ( conn == 4 )
                     topology_kernel< int32_t ><<< grid_for( n ), 256, 0, st >>>( n1, u0, n, (int32_t*) p );
                 else
                     topology_kernel< int64_t ><<< grid_for( n ), 256, 0, st >>>( n1, u0, n, (int64_t*) p );
             } );
        if ( !ok )
        {
            set_error( "XDMF write: " + err );
            rc = TN_ERR_IO;
        }
        cudaFree( d );
        cudaFreeHost( h );
        return rc;
    }
};

namespace {

template < typename Tin, typename Tout >
void launch_pack( const tn_xdmf_output::Grid& g, int n1, cudaStream_t st )
{
    CPtr3< Tin > s{ { (const Tin*) g.p[0], (const Tin*) g.p[1], (const Tin*) g.p[2] } };
    if ( g.vec == 1 )
        pack_nodes_kernel< Tin, Tout, 1 ><<< tile_grid( n1 ), dim3( kTile, 8 ), 0, st >>>( n1, s, (Tout*) g.d_stage );
    else
        pack_nodes_kernel< Tin, Tout, 3 ><<< tile_grid( n1 ), dim3( kTile, 8 ), 0, st >>>( n1, s, (Tout*) g.d_stage );
}

const char* kReadme =
    "# This directory contains the output of the XDMF writer (for visualization and checkpointing).\n"
    "\n"
    "Overview:\n"
    "- `geometry.bin`: cartesian node coordinates\n"
    "- `topology.bin`: connectivity/topology/elements (whatever you want to call it)\n"
    "- `checkpoint_metadata.bin`: metadata for checkpointing\n"
    "- `step_*.xmf`: xmf file (open this with Paraview for visualization) for each write() step\n"
    "- `<some_name>_*.bin`: binary grid data (per write() step)\n";

}  // namespace

extern "C" int tn_xdmf_output_create( const tn_mesh* m, const char* directory, int points_bytes,
                                      int connectivity_bytes, tn_xdmf_output** out )
{
    TN_CHECK_ARG( m && directory && out, "tn_xdmf_output_create: null argument" );
    TN_CHECK_ARG( points_bytes == 4 || points_bytes == 8, "tn_xdmf_output_create: points_bytes must be 4 or 8" );
    TN_CHECK_ARG( connectivity_bytes == 4 || connectivity_bytes == 8,
                  "tn_xdmf_output_create: connectivity_bytes must be 4 or 8" );
    *out  = nullptr;
    auto w = std::make_unique< tn_xdmf_output >();
    w->m   = m;
    w->dir = directory;
    w->pts = points_bytes;
    w->conn = connectivity_bytes;
    TN_CUDA_TRY( cudaGetDevice( &w->device ) );
    TN_CUDA_TRY( cudaStreamCreateWithFlags( &w->copy_stream, cudaStreamNonBlocking ) );
    TN_CUDA_TRY( cudaEventCreateWithFlags( &w->ev_packed, cudaEventDisableTiming ) );
    TN_CUDA_TRY( cudaEventCreateWithFlags( &w->ev_copied, cudaEventDisableTiming ) );
    *out = w.release();
    return TN_OK;
}

extern "C" int tn_xdmf_output_set_write_counter( tn_xdmf_output* w, int counter )
{
    TN_CHECK_ARG( w, "tn_xdmf_output_set_write_counter: null handle" );
    w->counter = counter;
    return TN_OK;
}

extern "C" int tn_xdmf_output_add( tn_xdmf_output* w, const char* label, int input_bytes, int vec_dim,
                                   const void* const* components, int output_bytes )
{
    TN_CHECK_ARG( w && label && components, "tn_xdmf_output_add: null argument" );
    TN_CHECK_ARG( !w->first_done, "XDMF::add(): Cannot add data after write() has been called." );
    TN_CHECK_ARG( input_bytes == 4 || input_bytes == 8, "XDMF::add(): Grid data type not supported (yet)." );
    TN_CHECK_ARG( output_bytes == 4 || output_bytes == 8, "tn_xdmf_output_add: output_bytes must be 4 or 8" );
    TN_CHECK_ARG( vec_dim == 1 || vec_dim == 3, "tn_xdmf_output_add: vec_dim must be 1 or 3" );
    for ( const auto& g : w->grids )
        TN_CHECK_ARG( g.label != label, std::string( "Cannot add data with label '" ) + label +
                                            "' - data with identical label has been added previously." );
    tn_xdmf_output::Grid g;
    g.label     = label;
    g.in_bytes  = input_bytes;
    g.out_bytes = output_bytes;
    g.vec       = vec_dim;
    for ( int c = 0; c < vec_dim; ++c )
    {
        TN_CHECK_ARG( components[c], "tn_xdmf_output_add: null component pointer" );
        g.p[c] = components[c];
    }
    g.bytes = w->nodes() * size_t( vec_dim ) * size_t( output_bytes );
    w->grids.push_back( g );
    return TN_OK;
}

extern "C" int tn_xdmf_output_write( tn_xdmf_output* w, void* s )
{
    TN_CHECK_ARG( w, "tn_xdmf_output_write: null handle" );
    int rc = w->join();
    if ( rc )
        return rc;
    cudaStream_t st = as_stream( s );
    const int    n1 = w->m->n1;
    if ( !w->first_done )
    {
        std::error_code ec;
        std::filesystem::create_directories( w->dir, ec );
        std::string err;
        if ( !write_file( w->dir + "/README.md", kReadme, std::strlen( kReadme ), err ) )
        {
            set_error( "XDMF write: " + err );
            return TN_ERR_IO;
        }
        w->order.clear();
        for ( int vec : { 1, 3 } )
            for ( int ib : { 4, 8 } )
                for ( int i = 0; i < int( w->grids.size() ); ++i )
                    if ( w->grids[i].vec == vec && w->grids[i].in_bytes == ib )
                        w->order.push_back( i );
        rc = w->write_mesh( st );
        if ( rc )
            return rc;
        const std::string md = w->metadata();
        if ( !write_file( w->dir + "/checkpoint_metadata.bin", md.data(), md.size(), err ) )
        {
            set_error( "XDMF write: " + err );
            return TN_ERR_IO;
        }
        for ( auto& g : w->grids )
        {
            TN_CUDA_TRY( cudaMalloc( &g.d_stage, g.bytes ) );
            TN_CUDA_TRY( cudaMallocHost( &g.h_stage, g.bytes ) );
        }
        w->first_done = true;
    }
    // conversion on the caller's stream, the copies on the writer's stream
    for ( int i : w->order )
    {
        const auto& g = w->grids[i];
        if ( g.in_bytes == 8 && g.out_bytes == 8 )
            launch_pack< double, double >( g, n1, st );
        else if ( g.in_bytes == 8 )
            launch_pack< double, float >( g, n1, st );
        else if ( g.out_bytes == 8 )
            launch_pack< float, double >( g, n1, st );
        else
            launch_pack< float, float >( g, n1, st );
        TN_LAUNCH_CHECK();
    }
    TN_CUDA_TRY( cudaEventRecord( w->ev_packed, st ) );
    TN_CUDA_TRY( cudaStreamWaitEvent( w->copy_stream, w->ev_packed, 0 ) );
    for ( int i : w->order )
    {
        const auto& g = w->grids[i];
        TN_CUDA_TRY( cudaMemcpyAsync( g.h_stage, g.d_stage, g.bytes, cudaMemcpyDeviceToHost, w->copy_stream ) );
    }
    TN_CUDA_TRY( cudaEventRecord( w->ev_copied, w->copy_stream ) );
    const std::string step = std::to_string( w->counter );
    std::string       xmf  = w->xmf( step );
    w->counter++;
    tn_xdmf_output* self = w;
    w->worker            = std::thread( [self, step, xmf]() {
        cudaSetDevice( self->device );
        if ( cudaEventSynchronize( self->ev_copied ) != cudaSuccess )
        {
            self->worker_error = "device-to-host copy failed";
            return;
        }
        std::string err;
        for ( int i : self->order )
        {
            const auto& g = self->grids[i];
            if ( !write_file( self->dir + "/" + g.label + "_" + step + ".bin", g.h_stage, g.bytes, err ) )
            {
                self->worker_error = err;
                return;
            }
        }
        // the step description last: its presence marks a complete step
        if ( !write_file( self->dir + "/step_" + step + ".xmf", xmf.data(), xmf.size(), err ) )
            self->worker_error = err;
    } );
    return TN_OK;
}

extern "C" int tn_xdmf_output_wait( tn_xdmf_output* w )
{
    TN_CHECK_ARG( w, "tn_xdmf_output_wait: null handle" );
    return w->join();
}

extern "C" int tn_xdmf_output_destroy( tn_xdmf_output* w )
{
    if ( !w )
        return TN_OK;
    const int rc = w->join();
    delete w;
    return rc;
}

// ---------------------------------------------------------------------------
// Checkpoint reading (io/xdmf.hpp:1117-1500).  Error texts are the reference's.

namespace {

struct GridFile
{
    std::string label;
    int32_t     type = 0, bytes = 0, vec = 0;
};

struct Metadata
{
    tn_checkpoint_info      info{};
    std::vector< double >   radii;
    std::vector< GridFile > files;
    std::vector< int64_t >  ids;
};

// read_xdmf_checkpoint_metadata (io/xdmf.hpp:1162-1268); "" on success, else the error
std::string read_metadata( const std::string& dir, Metadata& md )
{
    const std::string path = dir + "/checkpoint_metadata.bin";
    FILE*             f    = std::fopen( path.c_str(), "rb" );
    if ( !f )
        return "Could not find file: " + path;
    std::string buf;
    char        tmp[65536];
    size_t      n;
    while ( ( n = std::fread( tmp, 1, sizeof( tmp ), f ) ) > 0 )
        buf.append( tmp, n );
    std::fclose( f );
    size_t     pos = 0;
    auto       get = [&]( void* p, size_t k ) {
        if ( pos + k > buf.size() )
            return false;
        std::memcpy( p, buf.data() + pos, k );
        pos += k;
        return true;
    };
    const std::string err = "Failed to read from input stream.";
    auto&             I   = md.info;
    int32_t           v[6];
    for ( int i = 0; i < 6; ++i )
        if ( !get( &v[i], 4 ) )
            return err;
    I.version = v[0];
    I.subdomains_lateral = v[1];
    I.subdomains_radial  = v[2];
    I.size_x = v[3];
    I.size_y = v[4];
    I.size_r = v[5];
    const long long nr = (long long) I.subdomains_radial * ( I.size_r - 1 ) + 1;
    for ( long long i = 0; i < nr; ++i )
    {
        double r;
        if ( !get( &r, 8 ) )
            return err;
        if ( i > 0 && r <= md.radii.back() )
            return "Radii are not sorted correctly in checkpoint.";
        md.radii.push_back( r );
    }
    I.num_radii = int( md.radii.size() );
    if ( I.version > 0 && !get( &I.grid_scalar_bytes, 4 ) )
        return err;
    int32_t nf;
    if ( !get( &nf, 4 ) || nf < 0 )
        return err;
    for ( int i = 0; i < nf; ++i )
    {
        GridFile g;
        int32_t  len;
        if ( !get( &len, 4 ) || len < 0 || pos + size_t( len ) > buf.size() )
            return err;
        g.label.assign( buf.data() + pos, size_t( len ) );
        pos += size_t( len );
        if ( !get( &g.type, 4 ) || !get( &g.bytes, 4 ) || !get( &g.vec, 4 ) )
            return err;
        md.files.push_back( g );
    }
    I.num_grid_data_files = nf;
    if ( !get( &I.ordering, 4 ) )
        return err;
    if ( I.ordering == 0 )
    {
        const long long ns = 10LL * I.subdomains_lateral * I.subdomains_lateral * I.subdomains_radial;
        for ( long long i = 0; i < ns; ++i )
        {
            int64_t id;
            if ( !get( &id, 8 ) )
                return err + " (global_subdomain_id reading error)";
            md.ids.push_back( id );
        }
    }
    I.num_subdomain_ids = int( md.ids.size() );
    return "";
}

template < typename Tin, typename Tout >
void launch_unpack( int n1, const void* src, int vec, void* const* dst, cudaStream_t st )
{
    Ptr3< Tout > d{ { (Tout*) dst[0], (Tout*) ( vec == 3 ? dst[1] : nullptr ), (Tout*) ( vec == 3 ? dst[2] : nullptr ) } };
    if ( vec == 1 )
        unpack_nodes_kernel< Tin, Tout, 1 ><<< tile_grid( n1 ), dim3( kTile, 8 ), 0, st >>>( n1, (const Tin*) src, d );
    else
        unpack_nodes_kernel< Tin, Tout, 3 ><<< tile_grid( n1 ), dim3( kTile, 8 ), 0, st >>>( n1, (const Tin*) src, d );
}

}  // namespace

extern "C" int tn_read_xdmf_checkpoint_metadata( const char* directory, tn_checkpoint_info* info, double* radii,
                                                 int radii_capacity, long long* subdomain_ids, int ids_capacity )
{
    TN_CHECK_ARG( directory && info, "tn_read_xdmf_checkpoint_metadata: null argument" );
    Metadata          md;
    const std::string e = read_metadata( directory, md );
    if ( !e.empty() )
    {
        set_error( e );
        return TN_ERR_IO;
    }
    *info = md.info;
    for ( int i = 0; radii && i < std::min( radii_capacity, int( md.radii.size() ) ); ++i )
        radii[i] = md.radii[i];
    for ( int i = 0; subdomain_ids && i < std::min( ids_capacity, int( md.ids.size() ) ); ++i )
        subdomain_ids[i] = md.ids[i];
    return TN_OK;
}

extern "C" int tn_xdmf_checkpoint_grid_data_file( const char* directory, int index, char* label, int label_capacity,
                                                  int* scalar_data_type, int* scalar_bytes, int* vec_dim )
{
    TN_CHECK_ARG( directory, "tn_xdmf_checkpoint_grid_data_file: null argument" );
    Metadata          md;
    const std::string e = read_metadata( directory, md );
    if ( !e.empty() )
    {
        set_error( e );
        return TN_ERR_IO;
    }
    TN_CHECK_ARG( index >= 0 && index < int( md.files.size() ), "tn_xdmf_checkpoint_grid_data_file: index out of range" );
    const GridFile& g = md.files[index];
    if ( label )
    {
        TN_CHECK_ARG( label_capacity > int( g.label.size() ), "tn_xdmf_checkpoint_grid_data_file: label buffer too small" );
        std::memcpy( label, g.label.c_str(), g.label.size() + 1 );
    }
    if ( scalar_data_type )
        *scalar_data_type = g.type;
    if ( scalar_bytes )
        *scalar_bytes = g.bytes;
    if ( vec_dim )
        *vec_dim = g.vec;
    return TN_OK;
}

extern "C" int tn_read_xdmf_checkpoint_grid( const tn_mesh* m, const char* directory, const char* label, int step,
                                             int dst_bytes, int vec_dim, void* const* dst, void* s )
{
    TN_CHECK_ARG( m && directory && label && dst, "tn_read_xdmf_checkpoint_grid: null argument" );
    TN_CHECK_ARG( dst_bytes == 4 || dst_bytes == 8, "tn_read_xdmf_checkpoint_grid: dst_bytes must be 4 or 8" );
    TN_CHECK_ARG( vec_dim == 1 || vec_dim == 3, "tn_read_xdmf_checkpoint_grid: vec_dim must be 1 or 3" );
    for ( int c = 0; c < vec_dim; ++c )
        TN_CHECK_ARG( dst[c], "tn_read_xdmf_checkpoint_grid: null component pointer" );
    auto fail = [&]( const std::string& msg ) {
        set_error( msg );
        return TN_ERR_IO;
    };
    Metadata          md;
    const std::string e = read_metadata( directory, md );
    if ( !e.empty() )
        return fail( "Could not read checkpoint metadata: " + e );
    if ( !( md.info.version == 0 || md.info.version == 1 ) )
        return fail( "Supported checkpoint verions: 0, 1. This checkpoint has version " +
                     std::to_string( md.info.version ) + "." );
    const GridFile* g = nullptr;
    for ( const auto& f : md.files )
        if ( f.label == label )
        {
            g = &f;
            break;
        }
    if ( !g )
        return fail( std::string( "Could not find requested data (" ) + label + ") in checkpoint" );
    const std::string path = std::string( directory ) + "/" + label + "_" + std::to_string( step ) + ".bin";
    FILE*             f    = std::fopen( path.c_str(), "rb" );
    if ( !f )
        return fail( "Could not find checkpoint data file for requested label and step." );
    std::unique_ptr< FILE, int ( * )( FILE* ) > guard( f, std::fclose );
    const int n1 = m->n1;
    if ( md.info.size_x != n1 || md.info.size_y != n1 || md.info.size_r != n1 )
        return fail( "Grid data extents do not match metadata." );
    if ( md.info.ordering != 0 )
        return fail( "Checkpoint ordering type is not 0. Not supported." );
    if ( !( g->type == 2 && ( g->bytes == 4 || g->bytes == 8 ) ) )
        return fail( "Unsupported data type in checkpoint." );
    if ( vec_dim == 1 && g->vec != 1 )
        return fail( "Checkpoint is scalar, passed grid data view dims do not match." );
    if ( vec_dim == 3 && g->vec != 3 )
        return fail( "Checkpoint is vector-valued, passed grid data view dims do not match." );
    // the chunk of each diamond, wherever the writer put it
    const size_t chunk = size_t( n1 ) * n1 * n1 * size_t( vec_dim ) * size_t( g->bytes );
    void *       h = nullptr, *d = nullptr;
    TN_CUDA_TRY( cudaMallocHost( &h, chunk * kDiamonds ) );
    std::unique_ptr< void, cudaError_t ( * )( void* ) > hguard( h, cudaFreeHost );
    for ( int dd = 0; dd < kDiamonds; ++dd )
    {
        const int64_t id = int64_t( dd ) << 57;
        size_t        k  = 0;
        while ( k < md.ids.size() && md.ids[k] != id )
            ++k;
        if ( k == md.ids.size() )
            return fail( "Subdomain of diamond " + std::to_string( dd ) + " not found in checkpoint." );
        if ( fseeko( f, off_t( k * chunk ), SEEK_SET ) != 0 ||
             std::fread( (char*) h + dd * chunk, 1, chunk, f ) != chunk )
            return fail( "Checkpoint data file " + path + " is shorter than its metadata says." );
    }
    cudaStream_t st = as_stream( s );
    TN_CUDA_TRY( cudaMallocAsync( &d, chunk * kDiamonds, st ) );
    TN_CUDA_TRY( cudaMemcpyAsync( d, h, chunk * kDiamonds, cudaMemcpyHostToDevice, st ) );
    if ( g->bytes == 8 && dst_bytes == 8 )
        launch_unpack< double, double >( n1, d, vec_dim, dst, st );
    else if ( g->bytes == 8 )
        launch_unpack< double, float >( n1, d, vec_dim, dst, st );
    else if ( dst_bytes == 8 )
        launch_unpack< float, double >( n1, d, vec_dim, dst, st );
    else
        launch_unpack< float, float >( n1, d, vec_dim, dst, st );
    TN_LAUNCH_CHECK();
    TN_CUDA_TRY( cudaFreeAsync( d, st ) );
    // the pinned buffer is freed on return: wait for the copy
    TN_CUDA_TRY( cudaStreamSynchronize( st ) );
    return TN_OK;
}
