/* Stand-in declarations (TEST INFRASTRUCTURE): the host set-up sources of the
 * reference's CUDA code (mesh.c, cerjan.c, grid.c through pmcl3d.h) include
 * mpi.h.  On one rank (PX = PY = 1) inimesh reads the media file with fread
 * and calls MPI only to reduce the media extremes over ranks, which
 * gpusgt_ref_stubs.c does for a single rank; the rest abort if called. */
#ifndef REFINC_GPUSGT_MPI_H
#define REFINC_GPUSGT_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_File;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef struct { int source; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_FLOAT 1
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_ORDER_C 0
#define MPI_MODE_RDONLY 0
#define MPI_INFO_NULL 0
int MPI_Comm_rank(MPI_Comm, int *);
int MPI_Allreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm);
int MPI_Type_create_subarray(int, const int *, const int *, const int *, int, MPI_Datatype, MPI_Datatype *);
int MPI_Type_commit(MPI_Datatype *);
int MPI_File_open(MPI_Comm, const char *, int, MPI_Info, MPI_File *);
int MPI_File_set_view(MPI_File, MPI_Offset, MPI_Datatype, MPI_Datatype, const char *, MPI_Info);
int MPI_File_read_all(MPI_File, void *, int, MPI_Datatype, MPI_Status *);
int MPI_File_close(MPI_File *);
int MPI_Abort(MPI_Comm, int);
#endif
