/* Test infrastructure (oracle). Single-rank MPI stub: the reference's
 * decs_MPI.h declares MPI-typed globals; most host oracle builds link none of
 * the MPI code paths and only need the types. The file functions below are
 * implemented over stdio by ref_dumpio.c, so that the reference's own dump
 * and restart writers (dump.c, restart.c) can run on one rank. */
#ifndef HAMR_REF_MPI_STUB_H
#define HAMR_REF_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_File;
typedef int MPI_Info;
typedef long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

/* datatypes carry their size in bytes */
#define MPI_INT 4
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 2
#define MPI_INFO_NULL 0
#define MPI_SEEK_SET 0
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_COMM_WORLD 0
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

#ifdef __cplusplus
extern "C" {
#endif
int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence);
int MPI_File_iwrite(MPI_File fh, const void *buf, int count, MPI_Datatype type, MPI_Request *req);
int MPI_File_iwrite_all(MPI_File fh, const void *buf, int count, MPI_Datatype type, MPI_Request *req);
int MPI_File_close(MPI_File *fh);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Barrier(MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
#ifdef __cplusplus
}
#endif
#endif
