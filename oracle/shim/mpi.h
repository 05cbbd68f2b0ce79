/*
 * oracle/shim/mpi.h -- single-rank stand-in for the MPI calls the reference
 * makes, so that the reference's own, unmodified sources compile into the
 * checker binary oracle/_ref/BECMPI_ref.  TEST INFRASTRUCTURE ONLY.
 *
 * Semantics are those of MPI with exactly one rank (MPI_COMM_WORLD size 1):
 * collectives copy, Scatterv copies the root's segment, Isend/Irecv to self
 * match by tag, MPI-IO maps to POSIX file I/O with one file pointer.
 * Call sites: src/CosmoBEC_MPI.cpp:29-30,318-320,377; src/gadget_IC.h:484-510,
 * 538-544,624-627,724-741; src/write3D.h:38-52,69-76,95.
 */
#ifndef IFDM_SHIM_MPI_H
#define IFDM_SHIM_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; long long count; } MPI_Status;
typedef int MPI_Request;
typedef struct ifdm_shim_file *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0

#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_FLOAT 104
#define MPI_DOUBLE 108
#define MPI_LONG_LONG 208

#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3

#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_MODE_APPEND 128

#define MPI_SEEK_SET 600
#define MPI_SEEK_CUR 602
#define MPI_SEEK_END 604

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Scatterv(const void *sendbuf, const int sendcounts[], const int displs[], MPI_Datatype sendtype,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status *statuses);

int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char *datarep, MPI_Info info);
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype dt, MPI_Status *status);
int MPI_File_write_ordered(MPI_File fh, const void *buf, int count, MPI_Datatype dt, MPI_Status *status);
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype dt, MPI_Status *status);
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence);

#ifdef __cplusplus
}
#endif
#endif
