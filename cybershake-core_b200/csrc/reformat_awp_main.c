/*
 * reformat_awp -- an AWP SGT file ([point][6][timesteps], AWP component
 * order) rewritten in RWG order, with the command line of SgtHead's serial
 * reformat_awp (SgtHead/src/reformat_awp.c:8-35):
 *
 *   reformat_awp <input AWP SGT> <timesteps> <output SGT> [-z]
 *
 * The reordering runs on the GPU (awp_sgt_reorder_rwg), a slab of points at a
 * time; a trailing partial record is dropped, as the reference does.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/awp_sgt.h"

int main(int argc, char **argv)
{
    if (argc < 4) {
        printf("Usage: %s <input AWP SGT> <timesteps> <output AWP SGT> <-z>", argv[0]);
        return 1;
    }
    const int z = argc == 5 && strcmp(argv[4], "-z") == 0;
    if (z) printf("Will double all SGTs since they're the Z source\n");
    const int nt = atoi(argv[2]);
    if (nt < 1) {
        fprintf(stderr, "reformat_awp: timesteps must be >= 1\n");
        return 1;
    }
    FILE *in = fopen(argv[1], "rb");
    FILE *out = in ? fopen(argv[3], "wb") : NULL;
    if (!in || !out) {
        fprintf(stderr, "reformat_awp: cannot open %s\n", in ? argv[3] : argv[1]);
        if (in) fclose(in);
        return 1;
    }
    const size_t rec = (size_t)6 * nt;
    size_t slab = ((size_t)256 << 20) / (rec * sizeof(float));     /* about 256 MB of points */
    if (slab < 1) slab = 1;
    float *a = (float *)malloc(slab * rec * sizeof(float));
    float *b = (float *)malloc(slab * rec * sizeof(float));
    int rc = a && b ? 0 : 1;
    while (rc == 0) {
        const size_t got = fread(a, sizeof(float) * rec, slab, in);
        if (got == 0) break;
        if (awp_sgt_reorder_rwg(a, (int64_t)got, nt, z, b) != AWP_OK) {
            fprintf(stderr, "reformat_awp: %s\n", awp_last_error());
            rc = 1;
        } else if (fwrite(b, sizeof(float) * rec, got, out) != got) {
            fprintf(stderr, "reformat_awp: write failed\n");
            rc = 1;
        }
        if (got < slab) break;
    }
    free(a);
    free(b);
    fclose(in);
    if (fclose(out) != 0) rc = 1;
    return rc;
}
