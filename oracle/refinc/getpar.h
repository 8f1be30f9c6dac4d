/* Stand-in declarations (TEST INFRASTRUCTURE) of the parameter parser
 * DirectSynth uses; not on the synthesis path. */
#ifndef REFINC_GETPAR_H
#define REFINC_GETPAR_H
int getpar(const char *name, const char *type, void *val);
int mstpar(const char *name, const char *type, void *val);
int setpar(int argc, char **argv);
int endpar(void);
#endif
