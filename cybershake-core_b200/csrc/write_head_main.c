/*
 * write_head -- the RWG SGT header file for an AWP SGT run, with the command
 * line of SgtHead's write_head (SgtHead/src/write_head.c:12-37):
 *
 *   write_head <modelbox> <coordfile> <fdloc> <gridout> <spacing> <nt> <dt>
 *              <time decimation> <component> <moment> <max_freq>
 *              <awp_media_file> <outfile> [-c]
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/awp_sgt.h"

int main(int argc, char **argv)
{
    if (argc < 14) {
        printf("Usage: %s <modelbox_file> <coordfile> <fdloc_file> <gridout_file> <spacing> <nt> <dt> "
               "<time decimation> <component> <moment> <max_freq> <awp_media_file> <outfile> [-c]\n",
               argv[0]);
        return 1;
    }
    awp_sgthead_args a;
    memset(&a, 0, sizeof a);
    a.modelbox = argv[1];
    a.coordfile = argv[2];
    a.fdloc = argv[3];
    a.gridout = argv[4];
    a.spacing = (float)atof(argv[5]);
    a.nt = atoi(argv[6]);
    a.dt = (float)atof(argv[7]);
    a.sgt_tinc = atoi(argv[8]);
    a.component = argv[9];
    a.moment = (float)atof(argv[10]);
    a.flo = (float)atof(argv[11]);
    a.media_file = argv[12];
    a.mu_corr = argc == 15 && strcmp(argv[14], "-c") == 0;
    if (a.mu_corr) printf("Using unrelaxed/corrected mu.\n");
    const awp_status st = awp_write_sgt_header(&a, argv[13]);
    if (st != AWP_OK) {
        fprintf(stderr, "write_head: %s\n", awp_last_error());
        return 1;
    }
    return 0;
}
