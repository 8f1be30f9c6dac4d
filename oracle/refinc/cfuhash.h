/* Stand-in declarations (TEST INFRASTRUCTURE) of the hash table library that
 * DirectSynth's SGT master list uses; not on the synthesis path. */
#ifndef REFINC_CFUHASH_H
#define REFINC_CFUHASH_H
#include <stddef.h>
typedef struct cfuhash_table cfuhash_table_t;
cfuhash_table_t *cfuhash_new_with_initial_size(size_t size);
void *cfuhash_get(cfuhash_table_t *ht, const char *key);
void *cfuhash_put(cfuhash_table_t *ht, const char *key, void *data);
int cfuhash_destroy(cfuhash_table_t *ht);
int cfuhash_destroy_with_free_fn(cfuhash_table_t *ht, void (*ff)(void *));
#endif
