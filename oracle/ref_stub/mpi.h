/* Test infrastructure (oracle). Single-rank MPI type stub: the reference's
 * decs_MPI.h declares MPI-typed globals; the host oracle build links none of
 * the MPI code paths, it only needs the types to exist. */
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
#endif
