// Device multifrontal supernodal Cholesky and the shift-invert solve.
//
// Replaces cholmod_l_factorize_p (reference src/speigs_core.c:940, :966) and
// cholmod_l_solve2 (:96) for the 'sm' operator.  The host symbolic analysis
// (host/symbolic.h) fixes the supernodes and tree levels; this file owns the
// device copy of that structure, the tile task lists, and the kernels.
//
// Storage.  Every supernode s has a dense front of r x r doubles (column
// major, rows in the supernode's row-list order) that lives only during the
// factorization, and a persistent r x c panel
//     G_s = [ inv(L11) ; L21 * inv(L11) ]
// that replaces the usual [L11 ; L21].  With G, both triangular solves are a
// single dense (transposed) product per supernode, so every supernode of a
// tree level is solved in parallel with no sequential substitution.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../host/symbolic.h"

namespace spx {

constexpr int kTile = 32;

enum MfTaskKind { MF_ASSEMBLE = 0, MF_DIAG, MF_ROWS, MF_UPD_NEXT, MF_UPDATE, MF_INV_T,
                  MF_INV_X, MF_WMUL, MF_TINY, MF_NKIND };

struct MfLaunch {
    int     kind;
    int64_t off;     // first task
    int64_t count;   // tasks
};

// Real is the storage type of the fronts and of the panels G: double for
// the plain FP64 operator, float for the mixed-precision one (FP32 factor,
// trailing updates on the TF32 tensor cores with an FP32-accurate 3-term
// split; the caller refines each solve in FP64).  Vectors are FP64 always.
template <class Real>
class MultifrontalPlanT {
public:
    MultifrontalPlanT() = default;
    ~MultifrontalPlanT();
    MultifrontalPlanT(const MultifrontalPlanT &) = delete;
    MultifrontalPlanT &operator=(const MultifrontalPlanT &) = delete;

    // Upload the symbolic structure and build the task lists.  rowptr/col
    // are the host copy of the full symmetric CSR (original numbering) whose
    // values live on the device at the same positions.  Returns 0 or a
    // negative SPEIGS_ERR_* code.
    int init(const spx_symbolic &S, const int64_t *rowptr, const int32_t *col,
             cudaStream_t st);

    // Numeric factorization of A + shift*I from the device CSR values.
    // A pivot <= pivtol counts as not positive.  Returns 0, 1 when a pivot
    // was not positive (A + shift*I not PD), or a negative error code.
    int factorize(const double *d_val, double shift, double pivtol, cudaStream_t st);

    // x = (A + shift I)^{-1} b  (b, x device vectors in the original order).
    // When `skip` is given and *skip is nonzero on the device, the launch
    // does nothing (refinement steps that are no longer needed).
    void solve(const double *b, double *x, cudaStream_t st, const int *skip = nullptr);

    // X = (A + shift I)^{-1} B for nr <= 32 right-hand sides at once: B and X
    // are column-major n x nr device arrays in the original order (leading
    // dimensions ldb, ldx).  One persistent launch runs the same task queue
    // as solve() with every vector entry widened to nr columns, so the panel
    // and the level structure are paid once for all columns.  `skip` as in
    // solve(); with `accumulate`, X += the solution instead of X = it.
    // Returns 0 or a negative code (device buffers for the block are
    // allocated on first use).
    int solve_block(const double *B, int64_t ldb, double *X, int64_t ldx, int nr,
                    cudaStream_t st, const int *skip = nullptr, bool accumulate = false);

    void release(cudaStream_t st);

    // device word set when a solve's dependency wait gave up (0 otherwise)
    int *error_word() const;

    int64_t n() const { return n_; }
    double factor_flops() const { return flops_; }
    int64_t panel_entries() const { return g_total_; }
    int64_t solve_bytes() const;      // algorithmic bytes of one solve pair
    int levels() const { return nlevels_; }

private:
    void launch_factor(const double *d_val, cudaStream_t st);
    int32_t n_ = 0, ns_ = 0, nlevels_ = 0;
    double flops_ = 0.0;
    int64_t front_total_ = 0, g_total_ = 0, u_total_ = 0, nrows_total_ = 0;
    // device symbolic
    int32_t *d_perm_ = nullptr, *d_sfirst_ = nullptr, *d_rows_ = nullptr, *d_relmap_ = nullptr;
    int32_t *d_child_ptr_ = nullptr, *d_child_list_ = nullptr;
    int64_t *d_rowptr_ = nullptr, *d_frontptr_ = nullptr, *d_gptr_ = nullptr, *d_uptr_ = nullptr;
    int32_t *d_acolptr_ = nullptr;   // [n+1] assembly entries per new column
    int32_t *d_atpos_ = nullptr;     // row position within the front
    int32_t *d_asrc_ = nullptr;      // index into the CSR values
    int32_t *d_cbnd_ = nullptr;      // child bounds per parent 32-row tile
    int64_t *d_cbnd_ptr_ = nullptr;
    int4 *d_tasks_ = nullptr;
    std::vector<MfLaunch> launches_;
    // solve: per-level task offsets (4 lists), tasks, gather lists
    void *d_meta_ = nullptr;         // per-supernode solve metadata
    void *d_stask_ = nullptr;        // solve task queue
    int32_t *d_bundle_ = nullptr;
    int32_t *d_cptr_ = nullptr, *d_cidx_ = nullptr, *d_chunks_ = nullptr;
    double *d_fpart_ = nullptr, *d_bpart_ = nullptr;
    int *d_cnt_ = nullptr, *d_sync_ = nullptr;
    int32_t nfc_ = 0, nbc_ = 0;
    int ntasks_ = 0;                 // block tasks of the solve queue
    int nfw_ = 0, nbw_ = 0;          // warp tasks after them: forward, then backward
    size_t sync_ints_ = 0;
    int solve_grid_ = 0;
    size_t solve_smem_ = 0;
    // numeric
    Real *d_front_ = nullptr;
    Real *d_G_ = nullptr;
    double *d_u_ = nullptr, *d_yf_ = nullptr, *d_x_ = nullptr;
    int *d_status_ = nullptr;
    double *d_params_ = nullptr;     // shift, pivot tolerance (read by the graph)
    // block solve: buffers for rows of up to bw_ doubles (8, 16, 24 or 32)
    // for the right-hand sides, the result, yf, x, the update vectors and
    // the chunk partials; a solve of width NR <= bw_ uses them with stride NR
    int bw_ = 0;
    int32_t fslots_ = 0, bslots_ = 0;
    double *d_byf_ = nullptr, *d_bx_ = nullptr,
           *d_bu_ = nullptr, *d_bfp_ = nullptr, *d_bbp_ = nullptr;
    int bgrid_[4] = {0, 0, 0, 0};          // per width NR = 8 (q + 1): grid, 0 = not set up
    size_t bsmem_[4] = {0, 0, 0, 0};
    cudaGraphExec_t fgraph_ = nullptr;
    bool use_side_ = false;                    // some front has >= 2 column blocks
    cudaStream_t fside_ = nullptr;             // second branch of the factor graph
    cudaEvent_t fev_[2] = {nullptr, nullptr};  // [0] column kb+1 updated, [1] step kb's panel done
    const double *fgraph_val_ = nullptr;
    const double *direct_val_ = nullptr;       // values last factored by direct launches
    int max_rows_ = 0;
};

using MultifrontalPlan = MultifrontalPlanT<double>;
using MultifrontalPlan32 = MultifrontalPlanT<float>;

// The members are defined in multifrontal.cu, which is compiled once per
// storage type; each translation unit specialises them for its type.
#define SPX_MF_DECLARE(R)                                                                    \
    template <> MultifrontalPlanT<R>::~MultifrontalPlanT();                                \
    template <> int MultifrontalPlanT<R>::init(const spx_symbolic &, const int64_t *,      \
                                               const int32_t *, cudaStream_t);             \
    template <> int MultifrontalPlanT<R>::factorize(const double *, double, double,        \
                                                    cudaStream_t);                         \
    template <> void MultifrontalPlanT<R>::solve(const double *, double *, cudaStream_t,   \
                                                 const int *);                            \
    template <> int MultifrontalPlanT<R>::solve_block(const double *, int64_t, double *,   \
                                                      int64_t, int, cudaStream_t,         \
                                                      const int *, bool);                 \
    template <> void MultifrontalPlanT<R>::release(cudaStream_t);                          \
    template <> int *MultifrontalPlanT<R>::error_word() const;                             \
    template <> int64_t MultifrontalPlanT<R>::solve_bytes() const;                         \
    template <> void MultifrontalPlanT<R>::launch_factor(const double *, cudaStream_t);
SPX_MF_DECLARE(double)
SPX_MF_DECLARE(float)
#undef SPX_MF_DECLARE

}  // namespace spx
