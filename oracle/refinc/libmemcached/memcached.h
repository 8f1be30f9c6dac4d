/* Stand-in declarations (TEST INFRASTRUCTURE) of the memcached client the
 * SGT header cache uses (get_sgtpars); not on the synthesis path. */
#ifndef REFINC_MEMCACHED_H
#define REFINC_MEMCACHED_H
#include <stddef.h>
#include <stdint.h>
#include <time.h>
typedef enum { MEMCACHED_SUCCESS = 0 } memcached_return;
typedef struct memcached_st memcached_st;
typedef struct memcached_server_st memcached_server_st;
memcached_st *memcached_create(memcached_st *ptr);
void memcached_free(memcached_st *ptr);
memcached_server_st *memcached_server_list_append(memcached_server_st *l, const char *host, unsigned int port,
                                                  memcached_return *e);
memcached_return memcached_server_push(memcached_st *p, memcached_server_st *l);
void memcached_server_free(memcached_server_st *l);
char *memcached_get(memcached_st *p, const char *key, size_t klen, size_t *vlen, uint32_t *flags, memcached_return *e);
memcached_return memcached_set(memcached_st *p, const char *key, size_t klen, const char *v, size_t vlen, time_t exp,
                               uint32_t flags);
const char *memcached_strerror(memcached_st *p, memcached_return rc);
#endif
