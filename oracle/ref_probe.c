/* ORACLE TEST INFRASTRUCTURE -- not part of the shipped library.
 *
 * Exposes static helpers of the reference core so that the restatement in
 * speigs_oracle.py and the device kernels can be pinned against the
 * reference's own code bit for bit.  The reference source is included from
 * the reference tree at build time (oracle/Makefile); nothing is copied.
 *   rand_vec        src/speigs_core.c:52-54
 *   orth_block      src/speigs_core.c:122-132
 *   check_symmetry  src/speigs_core.c:363-401
 *   find_components src/speigs_core.c:445-466
 */
#include "speigs_core.c"

void probe_rand_vec(uint64_t seed, speigs_int n, double *v, uint64_t *seed_after) {
    uint64_t s = seed;
    rand_vec(&s, n, v);
    *seed_after = s;
}

void probe_orth_block(speigs_int n, speigs_int m, const double *B, double *w, double *hout) {
    double *tmp = (double *)calloc((size_t)(m > 4 ? m : 4), sizeof(double));
    orth_block(n, m, B, w, hout, tmp);
    free(tmp);
}

int probe_check_symmetry(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                         const double *Ax) {
    return check_symmetry(n, Ap, Ai, Ax);
}

speigs_int probe_find_components(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                                 const double *Ax, speigs_int *comp) {
    return find_components(n, Ap, Ai, Ax, comp);
}
