/* Single-rank MPI stand-in used only to compile the reference for the oracle
 * (test infrastructure; never part of the product).
 *
 * The reference needs MPI at compile time (src/terra/mpi/mpi.hpp:3) but this
 * image has no MPI.  With one rank, every collective is a copy (honouring
 * MPI_IN_PLACE), rank = 0, size = 1, and point-to-point calls are never
 * reached because same-rank subdomain pairs use local device copies
 * (src/terra/communication/shell/communication.hpp:256).  MPI-IO is only used
 * by the XDMF writer and checkpoint reader: single-rank stdio files below.
 *
 * A datatype handle encodes its element size in bytes in the low byte. */
#ifndef TN_ORACLE_MPI_STUB_H
#define TN_ORACLE_MPI_STUB_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef int MPI_Errhandler;
typedef int MPI_File;
typedef long long MPI_Offset;
typedef ptrdiff_t MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MAX_ERROR_STRING 64
#define MPI_COMM_WORLD 1
#define MPI_INFO_NULL 0
#define MPI_ERRORS_RETURN 0
#define MPI_IN_PLACE ((void*) 1)
#define MPI_STATUS_IGNORE ((MPI_Status*) 0)
#define MPI_STATUSES_IGNORE ((MPI_Status*) 0)
#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_CREATE 1

/* datatype = (id << 8) | size_in_bytes */
#define MPI_DATATYPE_NULL 0
#define MPI_CHAR ((1 << 8) | 1)
#define MPI_SIGNED_CHAR ((2 << 8) | 1)
#define MPI_UNSIGNED_CHAR ((3 << 8) | 1)
#define MPI_BYTE ((4 << 8) | 1)
#define MPI_CXX_BOOL ((5 << 8) | 1)
#define MPI_SHORT ((6 << 8) | 2)
#define MPI_UNSIGNED_SHORT ((7 << 8) | 2)
#define MPI_INT ((8 << 8) | 4)
#define MPI_UNSIGNED ((9 << 8) | 4)
#define MPI_FLOAT ((10 << 8) | 4)
#define MPI_LONG ((11 << 8) | 8)
#define MPI_UNSIGNED_LONG ((12 << 8) | 8)
#define MPI_LONG_LONG ((13 << 8) | 8)
#define MPI_UNSIGNED_LONG_LONG ((14 << 8) | 8)
#define MPI_DOUBLE ((15 << 8) | 8)
#define MPI_LONG_DOUBLE ((16 << 8) | 16)
#define MPI_INT64_T ((17 << 8) | 8)

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_LOR 4

static inline size_t tn_mpi_stub_size( MPI_Datatype t ) { return (size_t) ( t & 0xff ); }

static int tn_mpi_stub_state = 0; /* 0 = fresh, 1 = initialised, 2 = finalised */

static inline int MPI_Init( int* argc, char*** argv )
{
    (void) argc;
    (void) argv;
    tn_mpi_stub_state = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Finalize( void )
{
    tn_mpi_stub_state = 2;
    return MPI_SUCCESS;
}
static inline int MPI_Initialized( int* flag )
{
    *flag = tn_mpi_stub_state >= 1;
    return MPI_SUCCESS;
}
static inline int MPI_Finalized( int* flag )
{
    *flag = tn_mpi_stub_state == 2;
    return MPI_SUCCESS;
}
/* the communicator's size and this process's rank: 1 and 0 unless a driver poses as rank q of P to build that
 * rank's part of a distributed domain (no message is ever delivered) */
static int tn_mpi_stub_world_size = 1, tn_mpi_stub_rank = 0;
static inline int MPI_Comm_rank( MPI_Comm c, int* r )
{
    (void) c;
    *r = tn_mpi_stub_rank;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_size( MPI_Comm c, int* s )
{
    (void) c;
    *s = tn_mpi_stub_world_size;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_set_errhandler( MPI_Comm c, MPI_Errhandler e )
{
    (void) c;
    (void) e;
    return MPI_SUCCESS;
}
static inline int MPI_Error_string( int err, char* s, int* len )
{
    const char* msg = err == MPI_SUCCESS ? "success" : "single-rank MPI stand-in: unsupported call";
    *len            = (int) strlen( msg );
    memcpy( s, msg, (size_t) *len );
    return MPI_SUCCESS;
}
static inline int MPI_Barrier( MPI_Comm c )
{
    (void) c;
    return MPI_SUCCESS;
}
static inline int MPI_Bcast( void* b, int n, MPI_Datatype t, int root, MPI_Comm c )
{
    (void) b;
    (void) n;
    (void) t;
    (void) root;
    (void) c;
    return MPI_SUCCESS;
}
static inline int tn_mpi_stub_copy( const void* s, void* r, int n, MPI_Datatype t )
{
    if ( s != MPI_IN_PLACE && s != r )
        memcpy( r, s, (size_t) n * tn_mpi_stub_size( t ) );
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce( const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c )
{
    (void) op;
    (void) c;
    return tn_mpi_stub_copy( s, r, n, t );
}
static inline int MPI_Reduce( const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c )
{
    (void) op;
    (void) root;
    (void) c;
    return tn_mpi_stub_copy( s, r, n, t );
}
static inline int MPI_Scan( const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c )
{
    (void) op;
    (void) c;
    return tn_mpi_stub_copy( s, r, n, t );
}
static inline int MPI_Isend( const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* q )
{
    (void) b, (void) n, (void) t, (void) d, (void) tag, (void) c;
    *q = 0;
    return MPI_ERR_OTHER;
}
static inline int MPI_Irecv( void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request* q )
{
    (void) b, (void) n, (void) t, (void) s, (void) tag, (void) c;
    *q = 0;
    return MPI_ERR_OTHER;
}
static inline int MPI_Waitall( int n, MPI_Request* q, MPI_Status* st )
{
    (void) n, (void) q, (void) st;
    return MPI_SUCCESS;
}
/* Single-rank MPI-IO over stdio (the XDMF writer and checkpoint reader,
 * io/xdmf.hpp).  A file handle indexes a small table of open files, each
 * with its view displacement and file type; a derived (hindexed) type is an
 * index into a table of block lists and reads its blocks in order.  Opening
 * with MPI_MODE_CREATE does not truncate an existing file (MPI semantics). */
#include <stdio.h>
#include <stdlib.h>

#define TN_STUB_MAX_FILES 16
#define TN_STUB_MAX_TYPES 16
#define TN_STUB_TYPE_BASE 0x100000

typedef struct { FILE* f; long long disp; MPI_Datatype ftype; } tn_stub_file;
typedef struct { int n; int* len; MPI_Aint* off; } tn_stub_type;
static tn_stub_file tn_stub_files[TN_STUB_MAX_FILES];
static tn_stub_type tn_stub_types[TN_STUB_MAX_TYPES];

static inline int MPI_Type_create_hindexed( int n, const int* l, const MPI_Aint* d, MPI_Datatype o, MPI_Datatype* t )
{
    if ( o != MPI_CHAR && o != MPI_BYTE )
        return MPI_ERR_OTHER;
    for ( int i = 0; i < TN_STUB_MAX_TYPES; ++i )
        if ( !tn_stub_types[i].len )
        {
            tn_stub_types[i].n   = n;
            tn_stub_types[i].len = (int*) malloc( sizeof( int ) * ( n > 0 ? n : 1 ) );
            tn_stub_types[i].off = (MPI_Aint*) malloc( sizeof( MPI_Aint ) * ( n > 0 ? n : 1 ) );
            for ( int k = 0; k < n; ++k )
            {
                tn_stub_types[i].len[k] = l[k];
                tn_stub_types[i].off[k] = d[k];
            }
            *t = ( ( TN_STUB_TYPE_BASE + i ) << 8 ) | 1;
            return MPI_SUCCESS;
        }
    return MPI_ERR_OTHER;
}
static inline tn_stub_type* tn_stub_derived( MPI_Datatype t )
{
    const int i = ( t >> 8 ) - TN_STUB_TYPE_BASE;
    return ( i >= 0 && i < TN_STUB_MAX_TYPES && tn_stub_types[i].len ) ? &tn_stub_types[i] : (tn_stub_type*) 0;
}
static inline int MPI_Type_commit( MPI_Datatype* t ) { return tn_stub_derived( *t ) ? MPI_SUCCESS : MPI_ERR_OTHER; }
static inline int MPI_Type_free( MPI_Datatype* t )
{
    tn_stub_type* d = tn_stub_derived( *t );
    if ( d )
    {
        free( d->len );
        free( d->off );
        d->len = 0;
        d->off = 0;
    }
    *t = MPI_DATATYPE_NULL;
    return MPI_SUCCESS;
}
static inline tn_stub_file* tn_stub_fh( MPI_File fh )
{
    return ( fh >= 1 && fh <= TN_STUB_MAX_FILES && tn_stub_files[fh - 1].f ) ? &tn_stub_files[fh - 1] : (tn_stub_file*) 0;
}
static inline int MPI_File_open( MPI_Comm c, const char* f, int m, MPI_Info i, MPI_File* fh )
{
    (void) c, (void) i;
    *fh = 0;
    FILE* fp = 0;
    if ( m & MPI_MODE_RDONLY )
        fp = fopen( f, "rb" );
    else
    {
        fp = fopen( f, "r+b" );
        if ( !fp && ( m & MPI_MODE_CREATE ) )
            fp = fopen( f, "w+b" );
    }
    if ( !fp )
        return MPI_ERR_OTHER;
    for ( int k = 0; k < TN_STUB_MAX_FILES; ++k )
        if ( !tn_stub_files[k].f )
        {
            tn_stub_files[k].f     = fp;
            tn_stub_files[k].disp  = 0;
            tn_stub_files[k].ftype = MPI_CHAR;
            *fh                    = k + 1;
            return MPI_SUCCESS;
        }
    fclose( fp );
    return MPI_ERR_OTHER;
}
static inline int MPI_File_close( MPI_File* fh )
{
    tn_stub_file* f = tn_stub_fh( *fh );
    if ( !f )
        return MPI_ERR_OTHER;
    fclose( f->f );
    f->f = 0;
    *fh  = 0;
    return MPI_SUCCESS;
}
static inline int MPI_File_set_view( MPI_File fh, MPI_Offset o, MPI_Datatype e, MPI_Datatype t, const char* rep, MPI_Info i )
{
    (void) e, (void) rep, (void) i;
    tn_stub_file* f = tn_stub_fh( fh );
    if ( !f )
        return MPI_ERR_OTHER;
    f->disp  = o;
    f->ftype = t;
    return MPI_SUCCESS;
}
static inline int MPI_File_write_all( MPI_File fh, const void* b, int n, MPI_Datatype t, MPI_Status* st )
{
    (void) st;
    tn_stub_file* f = tn_stub_fh( fh );
    if ( !f || tn_stub_derived( f->ftype ) || fseeko( f->f, (off_t) f->disp, SEEK_SET ) )
        return MPI_ERR_OTHER;
    const size_t bytes = (size_t) n * tn_mpi_stub_size( t );
    return fwrite( b, 1, bytes, f->f ) == bytes ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_File_read_all( MPI_File fh, void* b, int n, MPI_Datatype t, MPI_Status* st )
{
    (void) st;
    tn_stub_file* f = tn_stub_fh( fh );
    if ( !f )
        return MPI_ERR_OTHER;
    size_t        left = (size_t) n * tn_mpi_stub_size( t );
    char*         p    = (char*) b;
    tn_stub_type* d    = tn_stub_derived( f->ftype );
    if ( !d )
    {
        if ( fseeko( f->f, (off_t) f->disp, SEEK_SET ) )
            return MPI_ERR_OTHER;
        return fread( p, 1, left, f->f ) == left ? MPI_SUCCESS : MPI_ERR_OTHER;
    }
    for ( int k = 0; k < d->n && left > 0; ++k )
    {
        size_t len = (size_t) d->len[k] < left ? (size_t) d->len[k] : left;
        if ( fseeko( f->f, (off_t) ( f->disp + d->off[k] ), SEEK_SET ) || fread( p, 1, len, f->f ) != len )
            return MPI_ERR_OTHER;
        p += len;
        left -= len;
    }
    return left == 0 ? MPI_SUCCESS : MPI_ERR_OTHER;
}
static inline int MPI_File_get_size( MPI_File fh, MPI_Offset* s )
{
    tn_stub_file* f = tn_stub_fh( fh );
    *s              = 0;
    if ( !f || fseeko( f->f, 0, SEEK_END ) )
        return MPI_ERR_OTHER;
    *s = (MPI_Offset) ftello( f->f );
    return MPI_SUCCESS;
}

#endif
