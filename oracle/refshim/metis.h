/* Stand-in declaration for the one METIS call the reference makes; it is only reached with
 * more than one rank, never in oracle runs.  TEST INFRASTRUCTURE ONLY. */
#ifndef FG_REFSHIM_METIS_H
#define FG_REFSHIM_METIS_H
static inline int METIS_PartGraphRecursive(int *a, int *b, int *c, int *d, int *e, int *f, int *g, int *h,
                                           void *i, void *j, void *k, int *l, int *m) {
    (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h; (void)i; (void)j; (void)k; (void)l; (void)m;
    return -1;
}
#endif
