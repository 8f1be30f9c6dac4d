/*
 * gpusgt_ref_stubs.c -- TEST INFRASTRUCTURE: single-rank stand-ins for the MPI
 * calls of the reference's host set-up sources (mesh.c).  MPI_Allreduce over
 * one rank copies its input; the parallel-read calls are never reached with
 * PX = PY = 1 and abort if they are.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mpi.h"

static int never(const char *what)
{
    fprintf(stderr, "set-up reference driver: %s is not on the one-rank path\n", what);
    abort();
    return 1;
}

int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }

int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op, (void)c;
    if (t != MPI_FLOAT) return never("MPI_Allreduce of a type other than MPI_FLOAT");
    memcpy(out, in, sizeof(float) * (size_t)n);
    return 0;
}

int MPI_Type_create_subarray(int a, const int *b, const int *c, const int *d, int e, MPI_Datatype f, MPI_Datatype *g)
{
    (void)a, (void)b, (void)c, (void)d, (void)e, (void)f, (void)g;
    return never("MPI_Type_create_subarray");
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return never("MPI_Type_commit"); }
int MPI_File_open(MPI_Comm c, const char *n, int m, MPI_Info i, MPI_File *f)
{
    (void)c, (void)n, (void)m, (void)i, (void)f;
    return never("MPI_File_open");
}
int MPI_File_set_view(MPI_File f, MPI_Offset o, MPI_Datatype a, MPI_Datatype b, const char *r, MPI_Info i)
{
    (void)f, (void)o, (void)a, (void)b, (void)r, (void)i;
    return never("MPI_File_set_view");
}
int MPI_File_read_all(MPI_File f, void *b, int n, MPI_Datatype t, MPI_Status *s)
{
    (void)f, (void)b, (void)n, (void)t, (void)s;
    return never("MPI_File_read_all");
}
int MPI_File_close(MPI_File *f) { (void)f; return never("MPI_File_close"); }
int MPI_Abort(MPI_Comm c, int e) { (void)c, (void)e; return never("MPI_Abort"); }
