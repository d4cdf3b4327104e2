// Host-side interface between the C API driver (driver.cpp, plain C++) and
// the device engine (engine.cu).  No CUDA types cross this header.
#pragma once

#include <stdint.h>

#include "../../include/speigs.h"
#include "../../include/speigs_b200.h"
#include "host/symbolic.h"

namespace spx {

// Full symmetric CSR built on the host from the upper triangle of the
// caller's CSC (the reference reads only the upper triangle: stype = 1 at
// src/speigs_core.c:836).
struct HostCSR {
    int32_t  n = 0;
    int64_t *rowptr = nullptr;   // n+1
    int32_t *col = nullptr;      // nnz
    double  *val = nullptr;      // nnz
    int64_t  nnz() const { return rowptr ? rowptr[n] : 0; }
};
int  build_full_csr(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                    HostCSR *out);
// The same CSR for an input whose pattern is symmetric with both triangles
// stored and strictly increasing row indices in every column (as the
// parallel symmetry check establishes): row i is column i, with the values
// of the upper triangle; built by parallel passes.
int  build_full_csr_sorted(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                           HostCSR *out);
void free_csr(HostCSR *A);

// Extended results not in speigs_info (device-side phase times in ms).
struct EngineStats {
    double ms_factor = 0, ms_op = 0, ms_ortho = 0, ms_resid = 0, ms_ritz = 0;
    int    factor_attempts = 0;
    int64_t solve_bytes = 0;     // algorithmic bytes of one shift-invert solve
    double factor_flops = 0;
};

// 'sm' (shift-invert) or 'lm' (direct) Lanczos on the device for a
// connected matrix: the part of the reference's speigs() from the operator
// set-up (:829-986) through lanczos() (:146-315).  lambda/V/resid are host
// buffers; entries are written for the converged-or-final Ritz pairs, in the
// Lanczos order (the caller sorts).  Returns 0 or SPEIGS_ERR_*.
// A is consumed (its host arrays are freed by the call).
// ext (may be NULL) selects the operator precision; einfo (may be NULL)
// receives the extension diagnostics.
// banded: the input passed the reference's banded-route gate; the route is
// reported as SPEIGS_PATH_BANDED (the band is factored by the supernodal
// code under nested dissection, which cuts it into independent segments).
int device_krylov(HostCSR &A, int64_t k, speigs_which which, const speigs_opts &o,
                  double anorm, double *lambda, double *V, double *resid, speigs_info *info,
                  EngineStats *stats, const speigs_ext_opts *ext = nullptr,
                  speigs_ext_info *einfo = nullptr, bool banded = false);

// Host set-up helpers shared by the C API entry points (driver.cpp).
int    host_check_symmetry(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax);
double host_norm1_upper(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax);

// Structure fast paths on the device.
int device_diag_path(int64_t n, const double *diag, int64_t k, speigs_which which,
                     double *lambda, double *V, double *resid, speigs_info *info);
int device_dense_path(const HostCSR &A, int64_t k, speigs_which which, double *lambda,
                      double *V, double *resid, speigs_info *info);

// The calling thread's current CUDA device (0 when it cannot be read), and
// making `dev` current on the calling thread.  Host worker threads start on
// device 0, so a pool that solves on the caller's GPU adopts its device
// first.
int  current_device();
void use_device(int dev);

// Complex eigenvectors from the real 2n x 2n embedding of a Hermitian
// matrix: V2 (host, 2n x kk column-major) holds the embedded eigenvectors
// in speigs() order; each candidate [a; b] is taken as a + i b, made
// orthogonal on the device to the vectors already accepted (complex
// Gram-Schmidt, twice) and kept when its norm stays above 0.1 -- the
// candidates dropped are complex multiples of accepted ones.  Up to k
// vectors are accepted: lambda/resid (host) from lam2/res2, Vr/Vi (host,
// n x k; may be NULL) their real and imaginary parts, zero past *nacc.
int device_hermitian_recover(int64_t n, int64_t kk, int64_t k, const double *V2,
                             const double *lam2, const double *res2, double *lambda, double *Vr,
                             double *Vi, double *resid, int64_t *nacc);

// Many components in lockstep: A is the CSR of their block-diagonal matrix
// with component c on rows [off[c], off[c+1]) (host, consumed); anorm[c] is
// ||A_c||_1.  Per component c: lam_out/res_out[c*k .. c*k+k) in Lanczos
// order (zero past min(k, its basis)), nconv/nops/restarts/flag; X_out (host,
// n x k column-major, may be NULL) the Ritz vectors on each component's rows.
// Returns 0, a negative code, or 1 when the forest needs a shift or the
// indefinite route (solve those components one by one instead).
// handed (per segment, may be NULL): set to 1 for the components still
// iterating when the lockstep loop stops early -- once the live components
// hold at most 1/handoff of the forest's rows, every lockstep step would
// still solve the whole forest for them, so they are handed back to be
// solved one by one (their other outputs are then not set).  With handed
// NULL or handoff <= 0 the loop runs every component to the end.
struct BatchedStats {
    double t_analyze = 0, t_factor = 0, t_iter = 0, t_total = 0;
    int64_t steps = 0, cycles = 0, handed = 0;
    bool graph = false;
};
int device_batched_krylov(HostCSR &A, int nseg, const int32_t *off, int64_t k,
                          speigs_which which, const speigs_opts &o, const double *anorm,
                          double *lam_out, double *res_out, double *X_out, int64_t *nconv_out,
                          int64_t *nops_out, int64_t *restarts_out, int *flag_out,
                          BatchedStats *bst, int *handed = nullptr, int handoff = 0);

// The factorization cache of the Krylov route (speigs_b200_factor_cache).
int factor_cache_configure(int entries);
int factor_cache_size();

// Thread-local text of the last CUDA failure seen by the engine.
const char *last_cuda_error();

}  // namespace spx
