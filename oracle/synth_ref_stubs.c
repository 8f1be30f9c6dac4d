/*
 * synth_ref_stubs.c -- TEST INFRASTRUCTURE: link-time stand-ins for the
 * libraries and DirectSynth files that the compiled jbsim sources reference
 * outside the synthesis path (memcached SGT-header cache, cfuhash master
 * list, Fortran FFT resampling, MPI-era file helpers).  None is called by
 * synth_ref_driver.c; each aborts if it ever is, so a run that reached one
 * could not pass silently.
 */
#include <stdio.h>
#include <stdlib.h>

int debug = 0;

static void never(const char *what)
{
    fprintf(stderr, "synthesis reference driver: %s is not on the synthesis path\n", what);
    abort();
}

void write_log(char *s) { (void)s; }

void *check_malloc(size_t n)
{
    void *p = malloc(n ? n : 1);
    if (!p) never("check_malloc (out of memory)");
    return p;
}

#define NEVER(name) \
    void name(void) { never(#name); }
NEVER(cfuhash_destroy)
NEVER(cfuhash_destroy_with_free_fn)
NEVER(cfuhash_get)
NEVER(cfuhash_new_with_initial_size)
NEVER(cfuhash_put)
NEVER(fcroptrfile)
NEVER(fopfile_ro)
NEVER(fourg_)
NEVER(freed)
NEVER(frite)
NEVER(makedir)
NEVER(memcached_create)
NEVER(memcached_free)
NEVER(memcached_get)
NEVER(memcached_server_free)
NEVER(memcached_server_list_append)
NEVER(memcached_server_push)
NEVER(memcached_set)
NEVER(memcached_strerror)
