// Shared definitions of the terraneo_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/terraneo_b200.h"

namespace tn {

constexpr int kDiamonds = 10;

// Per-thread error text returned by tn_last_error().
void set_error( const std::string& msg );

#define TN_CUDA_TRY( expr )                                                                              \
    do                                                                                                   \
    {                                                                                                    \
        cudaError_t err_ = ( expr );                                                                     \
        if ( err_ != cudaSuccess )                                                                       \
        {                                                                                                \
            ::tn::set_error( std::string( #expr ) + ": " + cudaGetErrorString( err_ ) );                 \
            (void) cudaGetLastError(); /* the status is returned: clear a non-sticky error */            \
            return TN_ERR_CUDA;                                                                          \
        }                                                                                                \
    } while ( 0 )

#define TN_CHECK_ARG( cond, msg )                                                                        \
    do                                                                                                   \
    {                                                                                                    \
        if ( !( cond ) )                                                                                 \
        {                                                                                                \
            ::tn::set_error( msg );                                                                      \
            return TN_ERR_ARG;                                                                           \
        }                                                                                                \
    } while ( 0 )

// Launch-error check after a kernel launch.
#define TN_LAUNCH_CHECK() TN_CUDA_TRY( cudaGetLastError() )

// Launch settings cached per device (the SM count, a kernel's shared-memory limit, a cluster size): indexed by
// the calling thread's current device, so one process may drive several GPUs.
constexpr int kMaxDevices = 64;
inline int current_device()
{
    int d = 0;
    if ( cudaGetDevice( &d ) != cudaSuccess || d < 0 || d >= kMaxDevices )
    {
        (void) cudaGetLastError();
        return 0;
    }
    return d;
}

inline cudaStream_t as_stream( void* s ) { return reinterpret_cast< cudaStream_t >( s ); }

template < typename T >
struct Ptr3
{
    T* p[3];
    // component c with compile-time indices only: a kernel that indexes its
    // parameter array with a run-time c gets the array copied to its stack
    __host__ __device__ __forceinline__ T* at( int c ) const { return c == 0 ? p[0] : ( c == 1 ? p[1] : p[2] ); }
};

}  // namespace tn

namespace tn {

// Host-side topology of the whole 10-diamond shell (no device calls): what a
// mesh of any subset of the diamonds is cut from.
struct ShellTopology
{
    int                    level = 0, N = 0, n1 = 0;
    std::vector< double >  coords;    // [10][n1][n1][3]
    std::vector< double >  radii;     // [10][n1]
    std::vector< uint8_t > lat_owned; // [10][n1][n1], owner = lowest diamond id of a duplicated point
    // duplicated lateral points, CSR over global lateral indices (d n1 + x) n1 + y,
    // members ascending (= ascending diamond id), groups ordered by point
    std::vector< int > offsets, members;
    std::vector< int > fv_ghost; // finite-volume lateral ghost map of the whole shell
    double             gram_inv[9] = { 0 };
};

int shell_topology( int level, double r_min, double r_max, ShellTopology& t );

// The diamonds [d0, d0 + nd) of the shell as a mesh (stored compactly, local
// diamond index = global - d0); the halo groups kept are those whose copies all
// lie in the range.  d0 = 0, nd = 10 is the whole shell.
int mesh_create_diamonds( const ShellTopology& t, double r_min, double r_max, int d0, int nd, tn_mesh** out );

}  // namespace tn

// The mesh object behind the opaque tn_mesh handle.
struct tn_mesh
{
    int    level = 0, N = 0, n1 = 0;
    int    d0 = 0, nd = tn::kDiamonds; // global id of the first stored diamond, number of stored diamonds
    double r_min = 0, r_max = 0;
    size_t ns = 0, nu = 0, nlat = 0;

    std::vector< double > h_coords;    // [nd][n1][n1][3]
    std::vector< double > h_radii;     // [nd][n1]
    std::vector< uint8_t > h_lat_owned; // [nd][n1][n1]

    double*  d_coords   = nullptr;
    double*  d_radii    = nullptr;
    float*   d_coords32 = nullptr;
    float*   d_radii32  = nullptr;
    uint8_t* d_lat_owned = nullptr; // lateral ownership (same for every r)
    uint8_t* d_node_owned = nullptr; // per stored node, for flat reductions

    // duplicated lateral positions, CSR: members of group g are
    // halo_members[halo_offsets[g] .. halo_offsets[g+1]) as lateral indices
    int  n_halo_groups    = 0;
    int* d_halo_offsets   = nullptr;
    int* d_halo_members   = nullptr;
    int* d_lat_group      = nullptr; // halo group of each lateral position, -1 if not duplicated

    // finite-volume lateral ghost map: entry (d * 4 + side) * N + i gives the
    // (diamond, x, y) FV cell across the face of ghost cell i on side
    // (x = 0, x = N+1, y = 0, y = N+1) of diamond d (whole shell only)
    int* d_fv_ghost = nullptr;
    // per FV cell (with ghosts, fv index): bit n set when face n's geometric normal points into the cell and is
    // flipped (the orientation test against the neighbour's centre), built on first use
    uint8_t* d_fv_orient = nullptr;

    // lateral quadrature tables of the gradient-form operators (Laplace,
    // DivKGrad, VectorLaplace), built on first use: [10][N][N][2 wedges][105]
    std::mutex      geom_mutex;
    double*         d_grad_geom = nullptr;
    double*         d_stokes_geom = nullptr; // Divergence / Gradient, this mesh as the velocity mesh

    // fs/fs penalty: the orthonormalised modes are m = C (e_j x x); G = C^T C
    double penalty_gram_inv[9] = { 0 };

    // device scratch: reduction partials + counters
    double*       d_red_partials = nullptr; // kRedMaxBlocks * 8 doubles
    double*       d_red_result   = nullptr; // 16 doubles
    unsigned int* d_red_counter  = nullptr;
    double*       h_red_result   = nullptr; // pinned, 16 doubles

    // side stream for work that overlaps a kernel of the caller's stream
    // (forked from and joined back into that stream with the two events)
    cudaStream_t side_stream = nullptr;
    cudaEvent_t  ev_fork = nullptr, ev_join = nullptr;
};

namespace tn {
constexpr int kRedMaxBlocks = 1184; // 148 SMs x 8
}
