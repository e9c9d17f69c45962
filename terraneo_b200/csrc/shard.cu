// Sharded shell: one rank's diamonds, and the cross-rank half of the additive
// halo.
//
// The reference distributes 10 x 2^(3 l_sd) subdomains over its MPI ranks
// (DistributedDomain::create_uniform, grid/shell/spherical_shell.hpp:2566-2590)
// with subdomain_to_rank_iterate_diamond_subdomains (:717-745).  At subdomain
// refinement level 0 a subdomain is a diamond and that map gives every rank a
// contiguous block of diamonds, the first 10 % P ranks one more than the
// others.  A shard here is such a block, stored compactly (local diamond index
// = global id - first diamond), so every cell-local kernel runs on it
// unchanged.  The additive halo of an apply (communication/shell/
// communication.hpp:242-747: pack, send/recv, unpack with SUM) splits in two:
// duplicate groups whose copies all lie on this rank are summed by the mesh's
// halo kernel; every group with copies on two or more ranks is a "cross" group:
// tn_shard_pack writes, per cross group, the sum of this rank's copies into a
// buffer whose layout [field][cross group][r] is the same on every rank, the
// caller's communicator sums the buffers (an all-reduce: NCCL over NVLink
// through torch.distributed, or MPI_Allreduce in the reference app), and
// tn_shard_unpack writes the total to every local copy.
#include <algorithm>
#include <set>
#include <vector>

#include "common.cuh"

namespace tn {

template < typename T >
int epsdivdiv_apply( const tn_mesh*, const tn_epsdivdiv_params*, const T*, const T* const*, T* const*, cudaStream_t,
                     const double* );
template < typename T >
int penalty_dots( const tn_mesh*, const T* const*, double*, cudaStream_t );
template < typename T >
int prolong_constant( const tn_mesh*, const tn_mesh*, int, int, const T* const*, T* const*, cudaStream_t );
template < typename T >
int restrict_constant( const tn_mesh*, const tn_mesh*, int, int, const T* const*, T* const*, cudaStream_t );

namespace {

// subdomain_to_rank_iterate_diamond_subdomains at one subdomain per diamond:
// the subdomain's global index is its diamond id.
int rank_of_diamond( int d, int num_ranks )
{
    const int div = kDiamonds / num_ranks, rem = kDiamonds % num_ranks;
    if ( d < ( div + 1 ) * rem )
        return d / ( div + 1 );
    return rem + ( d - ( div + 1 ) * rem ) / div;
}

int partition( int num_ranks, int rank, int* first, int* count )
{
    TN_CHECK_ARG( num_ranks >= 1 && num_ranks <= kDiamonds,
                  "tn_shell_partition: num_ranks must be in [1, 10] (one diamond per rank at most 10 ranks)" );
    TN_CHECK_ARG( rank >= 0 && rank < num_ranks, "tn_shell_partition: rank must be in [0, num_ranks)" );
    int f = -1, c = 0;
    for ( int d = 0; d < kDiamonds; ++d )
        if ( rank_of_diamond( d, num_ranks ) == rank )
        {
            if ( f < 0 )
                f = d;
            ++c;
        }
    *first = f, *count = c;
    return TN_OK;
}

// Local (cross = false) or cross-rank (cross = true) duplicate groups of a
// rank, CSR over local lateral indices.  Cross groups come in the topology's
// group order, which every rank shares, and a rank without a copy of one
// keeps it as an empty group.
int halo_plan( const ShellTopology& t, int num_ranks, int rank, bool cross, std::vector< int >& offsets,
               std::vector< int >& members )
{
    int d0, nd;
    if ( const int rc = partition( num_ranks, rank, &d0, &nd ) )
        return rc;
    const int per = t.n1 * t.n1, lo = d0 * per, hi = ( d0 + nd ) * per;
    offsets.assign( 1, 0 );
    members.clear();
    for ( size_t g = 0; g + 1 < t.offsets.size(); ++g )
    {
        std::set< int > ranks;
        for ( int k = t.offsets[g]; k < t.offsets[g + 1]; ++k )
            ranks.insert( rank_of_diamond( t.members[k] / per, num_ranks ) );
        const bool is_cross = ranks.size() > 1;
        if ( is_cross != cross || ( !cross && !ranks.count( rank ) ) )
            continue;
        for ( int k = t.offsets[g]; k < t.offsets[g + 1]; ++k )
            if ( t.members[k] >= lo && t.members[k] < hi )
                members.push_back( t.members[k] - lo );
        offsets.push_back( int( members.size() ) );
    }
    return TN_OK;
}

// One thread per (cross group, r, field): buf = sum of this rank's copies.
template < typename T >
__global__ void shard_pack_kernel( int n_groups, int n1, const int* __restrict__ offsets,
                                   const int* __restrict__ members, Ptr3< const T > fields, int nfields,
                                   T* __restrict__ buf )
{
    const long long tid   = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) n_groups * n1 * nfields;
    if ( tid >= total )
        return;
    const int r = int( tid % n1 );
    const int g = int( ( tid / n1 ) % n_groups );
    const int f = int( tid / ( (long long) n1 * n_groups ) );
    const T*  v = fields.at( f );
    T         s = 0;
    for ( int m = offsets[g]; m < offsets[g + 1]; ++m )
        s += v[(size_t) members[m] * n1 + r];
    buf[tid] = s;
}

// One thread per (cross group, r, field): every local copy = the reduced buf.
template < typename T >
__global__ void shard_unpack_kernel( int n_groups, int n1, const int* __restrict__ offsets,
                                     const int* __restrict__ members, const T* __restrict__ buf, Ptr3< T > fields,
                                     int nfields )
{
    const long long tid   = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    const long long total = (long long) n_groups * n1 * nfields;
    if ( tid >= total )
        return;
    const int r = int( tid % n1 );
    const int g = int( ( tid / n1 ) % n_groups );
    const int f = int( tid / ( (long long) n1 * n_groups ) );
    T*        v = fields.at( f );
    const T   s = buf[tid];
    for ( int m = offsets[g]; m < offsets[g + 1]; ++m )
        v[(size_t) members[m] * n1 + r] = s;
}

}  // namespace
}  // namespace tn

struct tn_shard
{
    tn_mesh* mesh      = nullptr;
    int      num_ranks = 1, rank = 0;
    int      n_cross   = 0; // cross groups (the same number on every rank)
    int*     d_offsets = nullptr;
    int*     d_members = nullptr;
};

using namespace tn;

namespace {

template < typename T >
int shard_pack( const tn_shard* s, const T* const* fields, int nfields, T* buf, cudaStream_t st )
{
    TN_CHECK_ARG( s && fields && nfields >= 1 && nfields <= 3, "tn_shard_pack: bad arguments" );
    TN_CHECK_ARG( buf || s->n_cross == 0, "tn_shard_pack: exchange buffer is NULL" );
    Ptr3< const T > f{};
    for ( int i = 0; i < nfields; ++i )
    {
        TN_CHECK_ARG( fields[i], "tn_shard_pack: null field" );
        f.p[i] = fields[i];
    }
    const long long total = (long long) s->n_cross * s->mesh->n1 * nfields;
    if ( total == 0 )
        return TN_OK;
    shard_pack_kernel< T ><<< unsigned( ( total + 255 ) / 256 ), 256, 0, st >>>(
        s->n_cross, s->mesh->n1, s->d_offsets, s->d_members, f, nfields, buf );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template < typename T >
int shard_unpack( const tn_shard* s, const T* buf, T* const* fields, int nfields, cudaStream_t st )
{
    TN_CHECK_ARG( s && fields && nfields >= 1 && nfields <= 3, "tn_shard_unpack: bad arguments" );
    TN_CHECK_ARG( buf || s->n_cross == 0, "tn_shard_unpack: exchange buffer is NULL" );
    Ptr3< T > f{};
    for ( int i = 0; i < nfields; ++i )
    {
        TN_CHECK_ARG( fields[i], "tn_shard_unpack: null field" );
        f.p[i] = fields[i];
    }
    const long long total = (long long) s->n_cross * s->mesh->n1 * nfields;
    if ( total == 0 )
        return TN_OK;
    shard_unpack_kernel< T ><<< unsigned( ( total + 255 ) / 256 ), 256, 0, st >>>(
        s->n_cross, s->mesh->n1, s->d_offsets, s->d_members, buf, f, nfields );
    TN_LAUNCH_CHECK();
    return TN_OK;
}

template < typename T >
int shard_apply( const tn_shard* s, const tn_epsdivdiv_params* p, const T* k, const T* const* src, T* const* dst,
                 cudaStream_t st )
{
    TN_CHECK_ARG( s && p, "tn_shard_epsdivdiv_apply: null argument" );
    TN_CHECK_ARG( p->diagonal || !( p->bc_cmb == TN_BC_FREESLIP && p->bc_surface == TN_BC_FREESLIP ) ||
                      s->num_ranks == 1,
                  "tn_shard_epsdivdiv_apply: free-slip on both radii needs the whole shell's rotation dots; with two "
                  "or more ranks use tn_shard_penalty_dots and tn_shard_epsdivdiv_apply_fsfs" );
    return epsdivdiv_apply< T >( s->mesh, p, k, src, dst, st, nullptr );
}

template < typename T >
int shard_apply_fsfs( const tn_shard* s, const tn_epsdivdiv_params* p, const T* k, const T* const* src, T* const* dst,
                      const double* dots, cudaStream_t st )
{
    TN_CHECK_ARG( s && p && dots, "tn_shard_epsdivdiv_apply_fsfs: null argument" );
    TN_CHECK_ARG( !p->diagonal && p->bc_cmb == TN_BC_FREESLIP && p->bc_surface == TN_BC_FREESLIP,
                  "tn_shard_epsdivdiv_apply_fsfs: free-slip on both radii, non-diagonal only" );
    return epsdivdiv_apply< T >( s->mesh, p, k, src, dst, st, dots );
}

}  // namespace

extern "C" int tn_shell_partition( int num_ranks, int rank, int* first_diamond, int* num_diamonds )
{
    TN_CHECK_ARG( first_diamond && num_diamonds, "tn_shell_partition: null output" );
    return partition( num_ranks, rank, first_diamond, num_diamonds );
}

extern "C" int tn_shard_halo_plan( int level, int num_ranks, int rank, int cross, int* n_groups, int* n_members,
                                   int* offsets, int* members )
{
    TN_CHECK_ARG( n_groups && n_members, "tn_shard_halo_plan: null count output" );
    ShellTopology t;
    if ( const int rc = shell_topology( level, 0.5, 1.0, t ) ) // the radii do not enter the plan
        return rc;
    std::vector< int > off, mem;
    if ( const int rc = halo_plan( t, num_ranks, rank, cross != 0, off, mem ) )
        return rc;
    *n_groups  = int( off.size() ) - 1;
    *n_members = int( mem.size() );
    if ( offsets )
        std::copy( off.begin(), off.end(), offsets );
    if ( members )
        std::copy( mem.begin(), mem.end(), members );
    return TN_OK;
}

extern "C" int tn_shard_create( int level, double r_min, double r_max, int num_ranks, int rank, tn_shard** out )
{
    TN_CHECK_ARG( out, "tn_shard_create: out is NULL" );
    *out = nullptr;
    int d0, nd;
    if ( const int rc = partition( num_ranks, rank, &d0, &nd ) )
        return rc;
    ShellTopology t;
    if ( const int rc = shell_topology( level, r_min, r_max, t ) )
        return rc;
    std::vector< int > off, mem;
    if ( const int rc = halo_plan( t, num_ranks, rank, true, off, mem ) )
        return rc;
    tn_shard* s = new tn_shard();
    s->num_ranks = num_ranks, s->rank = rank;
    s->n_cross   = int( off.size() ) - 1;
    if ( const int rc = mesh_create_diamonds( t, r_min, r_max, d0, nd, &s->mesh ) )
    {
        delete s;
        return rc;
    }
    if ( cudaMalloc( &s->d_offsets, off.size() * sizeof( int ) ) != cudaSuccess ||
         cudaMalloc( &s->d_members, std::max< size_t >( mem.size(), 1 ) * sizeof( int ) ) != cudaSuccess ||
         cudaMemcpy( s->d_offsets, off.data(), off.size() * sizeof( int ), cudaMemcpyHostToDevice ) != cudaSuccess ||
         ( !mem.empty() &&
           cudaMemcpy( s->d_members, mem.data(), mem.size() * sizeof( int ), cudaMemcpyHostToDevice ) != cudaSuccess ) )
    {
        set_error( "tn_shard_create: device allocation of the exchange plan failed" );
        tn_shard_destroy( s );
        return TN_ERR_NOMEM;
    }
    *out = s;
    return TN_OK;
}

extern "C" int tn_shard_destroy( tn_shard* s )
{
    if ( !s )
        return TN_OK;
    tn_mesh_destroy( s->mesh );
    cudaFree( s->d_offsets );
    cudaFree( s->d_members );
    delete s;
    return TN_OK;
}

extern "C" int tn_shard_dims( const tn_shard* s, int* first_diamond, int* num_diamonds, size_t* stored,
                              size_t* owned, size_t* exchange_values )
{
    TN_CHECK_ARG( s, "tn_shard_dims: shard is NULL" );
    if ( first_diamond )
        *first_diamond = s->mesh->d0;
    if ( num_diamonds )
        *num_diamonds = s->mesh->nd;
    if ( stored )
        *stored = s->mesh->ns;
    if ( owned )
        *owned = s->mesh->nu;
    if ( exchange_values )
        *exchange_values = size_t( s->n_cross ) * s->mesh->n1;
    return TN_OK;
}

extern "C" int tn_shard_geometry( const tn_shard* s, double* coords, double* radii )
{
    TN_CHECK_ARG( s, "tn_shard_geometry: shard is NULL" );
    return tn_mesh_geometry( s->mesh, coords, radii );
}

extern "C" int tn_shard_masks( const tn_shard* s, uint8_t* bmask, uint8_t* omask )
{
    TN_CHECK_ARG( s, "tn_shard_masks: shard is NULL" );
    return tn_mesh_masks( s->mesh, bmask, omask );
}

extern "C" int tn_shard_epsdivdiv_apply_f64( const tn_shard* s, const tn_epsdivdiv_params* p, const double* k,
                                             const double* const* src, double* const* dst, void* st )
{
    return shard_apply< double >( s, p, k, src, dst, as_stream( st ) );
}
extern "C" int tn_shard_epsdivdiv_apply_f32( const tn_shard* s, const tn_epsdivdiv_params* p, const float* k,
                                             const float* const* src, float* const* dst, void* st )
{
    return shard_apply< float >( s, p, k, src, dst, as_stream( st ) );
}

extern "C" int tn_shard_pack_f64( const tn_shard* s, const double* const* fields, int nfields, double* buf, void* st )
{
    return shard_pack< double >( s, fields, nfields, buf, as_stream( st ) );
}
extern "C" int tn_shard_pack_f32( const tn_shard* s, const float* const* fields, int nfields, float* buf, void* st )
{
    return shard_pack< float >( s, fields, nfields, buf, as_stream( st ) );
}
extern "C" int tn_shard_unpack_f64( const tn_shard* s, const double* buf, double* const* fields, int nfields, void* st )
{
    return shard_unpack< double >( s, buf, fields, nfields, as_stream( st ) );
}
extern "C" int tn_shard_unpack_f32( const tn_shard* s, const float* buf, float* const* fields, int nfields, void* st )
{
    return shard_unpack< float >( s, buf, fields, nfields, as_stream( st ) );
}

extern "C" int tn_shard_vec_dot_f64( const tn_shard* s, int ncomp, const double* const* a, const double* const* b,
                                     double* result, void* st )
{
    TN_CHECK_ARG( s, "tn_shard_vec_dot_f64: shard is NULL" );
    return tn_vec_dot_f64( s->mesh, ncomp, a, b, result, st );
}

extern "C" int tn_shard_vec_lincomb_f64( const tn_shard* s, int ncomp, double* const* y, double c0, int nx,
                                         const double* c, const double* const* x, void* st )
{
    TN_CHECK_ARG( s, "tn_shard_vec_lincomb_f64: shard is NULL" );
    return tn_vec_lincomb_f64( s->mesh, ncomp, y, c0, nx, c, x, st );
}

// ---------------------------------------------------------------------------
// Multigrid on shards: every level's shard holds the same diamonds (the rank map does not depend on the level), so
// the transfers stay within the rank; the restriction's coarse halo covers the rank's own copies and the caller
// completes it with the coarse shard's exchange, as after an apply.

static int same_ranks( const tn_shard* f, const tn_shard* c )
{
    TN_CHECK_ARG( f && c, "shard transfer: null shard" );
    TN_CHECK_ARG( f->num_ranks == c->num_ranks && f->rank == c->rank,
                  "shard transfer: the shards must belong to the same rank of the same partition" );
    return TN_OK;
}

extern "C" int tn_shard_prolongation_constant_f64( const tn_shard* fine, const tn_shard* coarse, int ncomp,
                                                   int apply_mode, const double* const* src, double* const* dst,
                                                   void* st )
{
    if ( const int rc = same_ranks( fine, coarse ) )
        return rc;
    TN_CHECK_ARG( src && dst, "tn_shard_prolongation_constant_f64: null argument" );
    return prolong_constant< double >( fine->mesh, coarse->mesh, ncomp, apply_mode, src, dst, as_stream( st ) );
}

extern "C" int tn_shard_restriction_constant_f64( const tn_shard* fine, const tn_shard* coarse, int ncomp,
                                                  const double* const* src, double* const* dst, void* st )
{
    if ( const int rc = same_ranks( fine, coarse ) )
        return rc;
    TN_CHECK_ARG( src && dst, "tn_shard_restriction_constant_f64: null argument" );
    return restrict_constant< double >( fine->mesh, coarse->mesh, ncomp, TN_APPLY_REPLACE, src, dst, as_stream( st ) );
}

extern "C" int tn_shard_injection_f64( const tn_shard* fine, const tn_shard* coarse, int ncomp, const double* const* src,
                                       double* const* dst, void* st )
{
    if ( const int rc = same_ranks( fine, coarse ) )
        return rc;
    return tn_injection_f64( fine->mesh, coarse->mesh, ncomp, src, dst, st );
}

extern "C" int tn_shard_vec_invert_f64( const tn_shard* s, int ncomp, double* const* y, void* st )
{
    TN_CHECK_ARG( s, "tn_shard_vec_invert_f64: shard is NULL" );
    return tn_vec_invert_f64( s->mesh, ncomp, y, st );
}

extern "C" int tn_shard_vec_chebyshev_step_f64( const tn_shard* s, int ncomp, double* const* x, double* const* d,
                                                const double* const* b, const double* const* ax,
                                                const double* const* inv_diag, double alpha, double beta, void* st )
{
    TN_CHECK_ARG( s, "tn_shard_vec_chebyshev_step_f64: shard is NULL" );
    return tn_vec_chebyshev_step_f64( s->mesh, ncomp, x, d, b, ax, inv_diag, alpha, beta, st );
}

extern "C" int tn_shard_vec_mult_f64( const tn_shard* s, int ncomp, double* const* y, const double* const* x, void* st )
{
    TN_CHECK_ARG( s, "tn_shard_vec_mult_f64: shard is NULL" );
    return tn_vec_mult_f64( s->mesh, ncomp, y, x, st );
}

// ---------------------------------------------------------------------------
// Free-slip on both radii over shards: the rigid-rotation penalty (kerngen :287-408, :585-606) needs three dot
// products over the whole shell's owned nodes; each rank forms its part, the caller sums them over the ranks, and
// the apply forms the penalty vector from the sums (the shell's Gram matrix is the same on every rank).

extern "C" int tn_shard_penalty_dots_f64( const tn_shard* s, const double* const* src, double* dots, void* st )
{
    TN_CHECK_ARG( s, "tn_shard_penalty_dots_f64: shard is NULL" );
    return penalty_dots< double >( s->mesh, src, dots, as_stream( st ) );
}
extern "C" int tn_shard_penalty_dots_f32( const tn_shard* s, const float* const* src, double* dots, void* st )
{
    TN_CHECK_ARG( s, "tn_shard_penalty_dots_f32: shard is NULL" );
    return penalty_dots< float >( s->mesh, src, dots, as_stream( st ) );
}
extern "C" int tn_shard_epsdivdiv_apply_fsfs_f64( const tn_shard* s, const tn_epsdivdiv_params* p, const double* k,
                                                  const double* const* src, double* const* dst, const double* dots,
                                                  void* st )
{
    return shard_apply_fsfs< double >( s, p, k, src, dst, dots, as_stream( st ) );
}
extern "C" int tn_shard_epsdivdiv_apply_fsfs_f32( const tn_shard* s, const tn_epsdivdiv_params* p, const float* k,
                                                  const float* const* src, float* const* dst, const double* dots,
                                                  void* st )
{
    return shard_apply_fsfs< float >( s, p, k, src, dst, dots, as_stream( st ) );
}
