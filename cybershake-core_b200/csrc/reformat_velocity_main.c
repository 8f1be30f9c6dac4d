/*
 * reformat_velocity -- the AWP media file from RWG velocity volumes, with the
 * command line of SgtHead's reformat_velocity (SgtHead/src/reformat_velocity.c:4-22):
 *
 *   reformat_velocity <nx> <ny> <nz> <velocity file prefix> <awp velocity out>
 *
 * reads prefix.p, prefix.s, prefix.d and transposes them on the GPU.
 */
#include <stdio.h>
#include <stdlib.h>

#include "../../include/awp_sgt.h"

int main(int argc, char **argv)
{
    if (argc < 6) {
        printf("Usage: %s <nx> <ny> <nz> <velocity file prefix> <awp velocity out>", argv[0]);
        return 0;
    }
    const awp_status st = awp_reformat_velocity(atoi(argv[1]), atoi(argv[2]), atoi(argv[3]), argv[4], argv[5]);
    if (st != AWP_OK) {
        fprintf(stderr, "reformat_velocity: %s\n", awp_last_error());
        return 1;
    }
    return 0;
}
