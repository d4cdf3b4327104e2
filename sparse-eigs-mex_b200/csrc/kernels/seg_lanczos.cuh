// Segmented thick-restart Lanczos: many independent components in lockstep.
//
// The components of a block-diagonal matrix are stored as contiguous row
// segments of one vector space; one operator application (a solve with the
// factor of the whole forest, or one SpMV) serves every component at once,
// and the vector work of the reference's lanczos() (src/speigs_core.c:146-315)
// runs segment by segment, one thread block per component: Gram-Schmidt with
// the projected-matrix column, breakdown re-injection from the component's
// own random stream, the Ritz vectors and true residuals, and the thick
// restart with the per-vector drop test.  Each component keeps its own
// recurrence state (step, basis size, random-stream position), so its
// arithmetic is the reference's for that component alone; components that
// have converged or stopped are skipped.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace spx {

struct SegArgs {
    int nseg;
    const int32_t *off;        // [nseg + 1] first row of each segment
    int ncv;                   // basis columns allocated per segment (the largest m)
    int k, l;                  // wanted pairs; Ritz vectors kept at a restart
    int64_t ldv;
    double *V, *Vn;            // ldv x (ncv + 1)
    double *H;                 // nseg blocks of ncv x ncv (ld ncv)
    double *theta, *S;         // nseg x ncv, nseg x ncv x ncv (the batched eigensolver's)
    int *ord;                  // nseg x ncv
    int *j, *m;                // per segment: next column to extend, basis size
    int *ext;                  // per segment: 1 while its basis is being extended
    int *live;                 // per segment: 1 while it iterates
    int *ops;                  // per segment: operator applications
    int *stop;                 // per segment: 1 when a restart found no continuation
    uint64_t *seed;            // per segment: random-stream state
    const double *bthr;        // per segment: breakdown threshold 1e-13 max(||A_c||_1, 1)
    const double *rtol;        // per segment: tol max(||A_c||_1, 1)
    double *x, *w;             // operator input and output (n rows)
    double *X, *AX;            // Ritz vectors and A times them: ldv x k
    double *lam, *r2;          // nseg x k
    int *nconv;                // per segment
    int *err;                  // set when a start vector has zero norm
    const uint64_t *jt;        // xorshift64* jump table (64 x 64 words)
};

// start vectors (every segment draws from the same seed, as a separate
// call would) and the per-segment state
void launch_seg_start(const SegArgs &a, uint64_t seed, cudaStream_t st);
// one Lanczos step of every extending segment, after w = Op x
void launch_seg_step(const SegArgs &a, cudaStream_t st);
// the k wanted Ritz vectors of every live segment into X (normalised)
void launch_seg_ritz(const SegArgs &a, cudaStream_t st);
// Rayleigh quotients, residual norms and converged counts from X, AX
void launch_seg_resid(const SegArgs &a, cudaStream_t st);
// thick restart of every live segment
void launch_seg_restart(const SegArgs &a, cudaStream_t st);

}  // namespace spx
