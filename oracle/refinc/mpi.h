/* Stand-in declarations (TEST INFRASTRUCTURE): DirectSynth's jbsim sources
 * include mpi.h; the functions the synthesis oracle calls use no MPI. */
#ifndef REFINC_MPI_H
#define REFINC_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_File;
typedef long long MPI_Offset;
typedef int MPI_Info;
typedef int MPI_Request;
typedef struct { int source; } MPI_Status;
#endif
