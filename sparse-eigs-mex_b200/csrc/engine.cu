// Device engine: thick-restart Lanczos with full reorthogonalisation over a
// pluggable operator, run on one GPU.
//
// The control flow is the reference's lanczos() (src/speigs_core.c:146-315)
// step for step -- same ncv/maxit/tol defaults, same start-vector stream,
// same breakdown threshold and re-injection, same convergence test and
// thick-restart rule -- with every vector operation on the device.  The host
// only reads back the scalars the reference branches on (a step's beta, the
// number of converged pairs, a restart vector's norm).
#include "engine.h"
#include "host/parallel.h"
#include "../../include/speigs_b200.h"
#include "kernels/krylov.cuh"
#include "kernels/multifrontal.cuh"
#include "kernels/block_krylov.cuh"
#include "kernels/dense_lu.cuh"
#include "kernels/seg_lanczos.cuh"
#include "counters.h"
#include "host/syev_host.h"

#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

namespace spx {


// cudaMemcpyAsync that feeds the transfer counters
static cudaError_t copy_async(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind,
                              cudaStream_t st) {
    if (kind == cudaMemcpyHostToDevice) note_h2d((long long)bytes);
    else if (kind == cudaMemcpyDeviceToHost) note_d2h((long long)bytes);
    return cudaMemcpyAsync(dst, src, bytes, kind, st);
}

static thread_local char g_err[256] = "";
const char *last_cuda_error() { return g_err; }
const char *set_last_error_text(const char *msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return g_err;
}

int current_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return dev;
}

void use_device(int dev) {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur == dev) return;
    if (cudaSetDevice(dev) != cudaSuccess) cudaGetLastError();
}

static int cuda_fail(cudaError_t e, const char *where) {
    snprintf(g_err, sizeof g_err, "%s: %s", where, cudaGetErrorString(e));
    cudaGetLastError();
    return SPEIGS_ERR_INTERNAL;
}

// ---------------------------------------------- projected eigenproblem --
// The Lanczos loops' projected problem (order m = the basis size) is solved on
// the host, as the reference solves it with LAPACK: H is read back, solved by
// syev_host, and theta, S, ord and the status word are written back in the
// layout the device Jacobi (launch_syev_small) uses.  The pinned staging
// buffers are reused from call to call: a call's first act is a synchronous
// read-back on the same stream, after which the previous call's uploads have
// completed.
struct SyevStage {
    double *buf = nullptr;
    size_t cap = 0;
    ~SyevStage() {
        if (buf) cudaFreeHost(buf);   // an error at process exit is harmless
    }
};
static int syev_projected(int m, const double *dH, int ldh, double *dtheta, double *dS, int *dord,
                          int *dstat, cudaStream_t st, int nvec = -1) {
    thread_local SyevStage sg;
    const size_t need = 2 * (size_t)m * m + 2 * (size_t)m + 8;
    if (sg.cap < need) {
        double *nb = nullptr;
        if (cudaMallocHost(&nb, sizeof(double) * need) != cudaSuccess) {
            cudaGetLastError();
            return SPEIGS_ERR_MEM;
        }
        if (sg.buf) cudaFreeHost(sg.buf);
        sg.buf = nb;
        sg.cap = need;
    }
    double *hH = sg.buf, *hS = hH + (size_t)m * m, *hth = hS + (size_t)m * m;
    int *hord = reinterpret_cast<int *>(hth + m);
    int *hst = reinterpret_cast<int *>(hth + 2 * m);
    note_d2h((long long)sizeof(double) * m * m);
    cudaMemcpy2DAsync(hH, sizeof(double) * m, dH, sizeof(double) * ldh, sizeof(double) * m, m,
                      cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "projected problem read-back");
    // nvec >= 0: eigenvectors only for the nvec wanted Ritz values (the
    // rest of S is zero); the eigenvalues are those of the full solver
    const int steps = (nvec >= 0 && nvec < m) ? syev_host_select(m, hH, m, nvec, hth, hS, hord)
                                              : syev_host(m, hH, m, hth, hS, hord);
    hst[0] = steps < 0 ? -1 : steps + 1;
    hst[1] = 0;
    copy_async(dtheta, hth, sizeof(double) * m, cudaMemcpyHostToDevice, st);
    copy_async(dS, hS, sizeof(double) * m * m, cudaMemcpyHostToDevice, st);
    copy_async(dord, hord, sizeof(int) * m, cudaMemcpyHostToDevice, st);
    copy_async(dstat, hst, sizeof(int) * 2, cudaMemcpyHostToDevice, st);
    return 0;
}

// ------------------------------------------------------------- resources --
// One memory pool per device with a high release threshold, so repeated calls
// reuse device memory instead of returning it to the driver at every sync.
cudaMemPool_t device_pool(int dev) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &thr);
        pools[dev] = p;
    }
    return pools[dev];
}

struct Stream {
    cudaStream_t s = nullptr;
    cudaError_t err = cudaSuccess;
    Stream() { err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking); }
    ~Stream() {
        if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    }
};

class Arena {
public:
    explicit Arena(cudaStream_t st) : st_(st) {
        int dev = 0;
        cudaGetDevice(&dev);
        pool_ = device_pool(dev);
    }
    ~Arena() {
        for (void *p : ptrs_) cudaFreeAsync(p, st_);
    }
    template <class T>
    T *alloc(size_t cnt) {
        void *p = nullptr;
        size_t bytes = (cnt ? cnt : 1) * sizeof(T);
        cudaError_t e = pool_ ? cudaMallocFromPoolAsync(&p, bytes, pool_, st_)
                              : cudaMallocAsync(&p, bytes, st_);
        if (e != cudaSuccess) { cudaGetLastError(); failed = true; return nullptr; }
        ptrs_.push_back(p);
        return (T *)p;
    }
    bool failed = false;

private:
    cudaStream_t st_;
    cudaMemPool_t pool_ = nullptr;
    std::vector<void *> ptrs_;
};

// Device-side phase timer: event pairs resolved at host syncs.  Events come
// from a pool that is recycled as pairs are resolved, so a long iteration
// creates only as many events as are in flight between two syncs.
class PhaseTimer {
public:
    explicit PhaseTimer(cudaStream_t st) : st_(st) {}
    ~PhaseTimer() {
        for (auto &p : pairs_) {
            if (p.a) cudaEventDestroy(p.a);
            if (p.b) cudaEventDestroy(p.b);
        }
        for (auto e : free_) cudaEventDestroy(e);
    }
    int begin() {
        int id;
        if (!free_ids_.empty()) { id = free_ids_.back(); free_ids_.pop_back(); }
        else { id = (int)pairs_.size(); pairs_.push_back({}); }
        Pair &p = pairs_[id];
        p.a = mk();
        p.b = nullptr;
        p.acc = nullptr;
        p.live = true;
        cudaEventRecord(p.a, st_);
        return id;
    }
    void end(int id, double *acc) {
        pairs_[id].b = mk();
        pairs_[id].acc = acc;
        cudaEventRecord(pairs_[id].b, st_);
    }
    void resolve() {   // after a stream sync: every ended pair is complete
        for (int id = 0; id < (int)pairs_.size(); id++) {
            Pair &p = pairs_[id];
            if (!p.live || !p.b) continue;
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) *p.acc += ms;
            else cudaGetLastError();
            free_.push_back(p.a);
            free_.push_back(p.b);
            p.a = p.b = nullptr;
            p.live = false;
            free_ids_.push_back(id);
        }
    }

private:
    struct Pair { cudaEvent_t a = nullptr, b = nullptr; double *acc = nullptr; bool live = false; };
    cudaEvent_t mk() {
        if (!free_.empty()) { cudaEvent_t e = free_.back(); free_.pop_back(); return e; }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    cudaStream_t st_;
    std::vector<Pair> pairs_;
    std::vector<int> free_ids_;
    std::vector<cudaEvent_t> free_;
};

// ------------------------------------------------------------ operators --
// The pluggable operator of the reference (speigs_op / op_apply,
// src/speigs_core.c:57-116): mode 0 is y = A x, mode 1 the Cholesky solve.
struct Operator {
    virtual ~Operator() = default;
    virtual void apply(const double *x, double *y, cudaStream_t st) = 0;
    // device word that becomes nonzero if an application failed (or null)
    virtual const int *error_word() const { return nullptr; }
    int64_t nops = 0;
};

struct DevA {
    int n;
    const int32_t *rp, *ci;
    const double *va;
};

// The numeric factor in the storage precision the plan was created with:
// FP64 (the drop-in operator) or FP32 (mixed precision, refined in FP64).
struct Factor {
    MultifrontalPlan f64;
    MultifrontalPlan32 f32;
    bool mixed = false;
    int init(const spx_symbolic &S, const int64_t *rp, const int32_t *ci, cudaStream_t st) {
        return mixed ? f32.init(S, rp, ci, st) : f64.init(S, rp, ci, st);
    }
    int factorize(const double *val, double shift, double pivtol, cudaStream_t st) {
        return mixed ? f32.factorize(val, shift, pivtol, st) : f64.factorize(val, shift, pivtol, st);
    }
    void solve(const double *b, double *x, cudaStream_t st, const int *skip = nullptr) {
        if (mixed) f32.solve(b, x, st, skip);
        else f64.solve(b, x, st, skip);
    }
    int solve_block(const double *B, int64_t ldb, double *X, int64_t ldx, int nr, cudaStream_t st,
                    const int *skip = nullptr, bool accumulate = false) {
        return mixed ? f32.solve_block(B, ldb, X, ldx, nr, st, skip, accumulate)
                     : f64.solve_block(B, ldb, X, ldx, nr, st, skip, accumulate);
    }
    int *error_word() const { return mixed ? f32.error_word() : f64.error_word(); }
    double factor_flops() const { return mixed ? f32.factor_flops() : f64.factor_flops(); }
    int64_t solve_bytes() const { return mixed ? f32.solve_bytes() : f64.solve_bytes(); }
    int64_t panel_entries() const { return mixed ? f32.panel_entries() : f64.panel_entries(); }
    void release(cudaStream_t st) { f64.release(st); f32.release(st); }
};

// Device state of the FP64 refinement of a mixed-precision solve.
struct RefineState {
    double *r = nullptr, *d = nullptr;
    int *flag = nullptr, *count = nullptr;
    ReduceScratch rs;
    int max_steps = 10;
    double tol = 1e-14;
};

struct SpmvOperator : Operator {
    DevA A;
    explicit SpmvOperator(const DevA &a) : A(a) {}
    void apply(const double *x, double *y, cudaStream_t st) override {
        nops++;
        launch_spmv(A.n, A.rp, A.ci, A.va, x, y, st);
    }
};

// The indefinite route: y = A^{-1} x with the dense inverse (reference
// operator mode 2, src/speigs_core.c:111-115).
struct DenseInvOperator : Operator {
    int n;
    const double *M;
    DenseInvOperator(int n_, const double *m) : n(n_), M(m) {}
    void apply(const double *x, double *y, cudaStream_t st) override {
        nops++;
        launch_dense_apply(n, M, x, y, st);
    }
};

struct CholOperator : Operator {
    Factor *plan;
    explicit CholOperator(Factor *p) : plan(p) {}
    void apply(const double *x, double *y, cudaStream_t st) override {
        nops++;
        plan->solve(x, y, st);
    }
    const int *error_word() const override { return plan->error_word(); }
};

// Mixed precision: y = (A + shift I)^{-1} x with the FP32 factor, refined
// in FP64 -- r = x - (A + shift I) y, y += M^{-1} r -- until the backward
// error test of launch_refine_residual holds or max_steps corrections were
// made.  The loop is launched in full every time; steps after convergence
// return at once on the device flag, so the host never waits.
struct MixedCholOperator : Operator {
    Factor *plan;
    DevA A;
    double shift, anorm;
    RefineState *rf;
    MixedCholOperator(Factor *p, const DevA &a, double sh, double an, RefineState *r)
        : plan(p), A(a), shift(sh), anorm(an), rf(r) {}
    void apply(const double *x, double *y, cudaStream_t st) override {
        nops++;
        plan->solve(x, y, st);
        cudaMemsetAsync(rf->flag, 0, sizeof(int), st);
        for (int it = 0; it <= rf->max_steps; it++) {
            launch_refine_residual(A.n, A.rp, A.ci, A.va, shift, x, y, rf->r, rf->tol, anorm,
                                   rf->flag, rf->count, rf->rs, st);
            if (it == rf->max_steps) break;
            plan->solve(rf->r, rf->d, st, rf->flag);
            launch_axpy_unless(A.n, y, rf->d, rf->flag, st);
        }
    }
    const int *error_word() const override { return plan->error_word(); }
};

// Operator on a block of b <= 32 vectors: W = Op V (column-major, leading
// dimensions ldv, ldw).  The block Lanczos counts block applications and the
// vectors they carry.
struct BlockOperator {
    virtual ~BlockOperator() = default;
    virtual int apply(const double *V, int64_t ldv, double *W, int64_t ldw, int b,
                      cudaStream_t st) = 0;
    virtual const int *error_word() const { return nullptr; }
    // A device word set when an application fell short of its accuracy
    // target with the work queued for it (the caller redoes that work with
    // set_full(true)); nullptr when every application is complete.
    virtual int *short_word() const { return nullptr; }
    virtual void set_full(bool) {}
    int64_t napps = 0, nvecs = 0;
    // optional: device time of the block solves (layout conversions
    // included), accumulated into *ms_solve by tm
    PhaseTimer *tm = nullptr;
    double *ms_solve = nullptr;
    double ms_solve_acc = 0;
    int64_t solve_calls = 0;
    int timed_solve(Factor *plan, const double *B, int64_t ldb, double *X, int64_t ldx, int nr,
                    cudaStream_t st, const int *skip = nullptr, bool accumulate = false) {
        solve_calls++;
        const int t = tm ? tm->begin() : -1;
        const int rc = plan->solve_block(B, ldb, X, ldx, nr, st, skip, accumulate);
        if (tm) tm->end(t, ms_solve);
        return rc;
    }
};

struct BlockCholOperator : BlockOperator {
    Factor *plan;
    explicit BlockCholOperator(Factor *p) : plan(p) {}
    int apply(const double *V, int64_t ldv, double *W, int64_t ldw, int b,
              cudaStream_t st) override {
        napps++;
        nvecs += b;
        return timed_solve(plan, V, ldv, W, ldw, b, st);
    }
    const int *error_word() const override { return plan->error_word(); }
};

// Device state of the FP64 refinement of a mixed-precision block solve.
struct BlockRefineState {
    double *R = nullptr, *part = nullptr;
    int64_t ld = 0;
    int *flag = nullptr, *count = nullptr;
    int *short_word = nullptr;   // set when a solve was left unconverged within `budget`
    unsigned *counter = nullptr;
    int max_steps = 10;
    int budget = 0;              // corrections queued per solve (0: max_steps)
    double tol = 1e-14;
};

__global__ void flag_if_unset_kernel(const int *flag, int *word) {
    if (!*(volatile const int *)flag) *word = 1;
}

// Mixed precision on a block: X = M^{-1} B with the FP32 factor, then
// R = B - (A + shift I) X and X += M^{-1} R (the correction solve adds its
// result into X) until every column passes the backward-error test or
// max_steps corrections were made.  As for one vector, the whole loop is
// queued; once the flag is set, the remaining solves return at once on the
// device.
struct BlockMixedOperator : BlockOperator {
    Factor *plan;
    DevA A;
    double shift, anorm;
    BlockRefineState *rf;
    BlockMixedOperator(Factor *p, const DevA &a, double sh, double an, BlockRefineState *r)
        : plan(p), A(a), shift(sh), anorm(an), rf(r) {}
    int apply(const double *V, int64_t ldv, double *W, int64_t ldw, int b,
              cudaStream_t st) override {
        napps++;
        nvecs += b;
        int rc = timed_solve(plan, V, ldv, W, ldw, b, st);
        if (rc) return rc;
        cudaMemsetAsync(rf->flag, 0, sizeof(int), st);
        // With a budget, only that many corrections are queued (the rest of
        // max_steps would return at once on the device flag but still cost
        // their launches); a solve still unconverged after them sets
        // short_word, and the caller redoes its work with the full loop.
        const int steps = (rf->budget > 0 && rf->short_word && !full)
                              ? std::min(rf->budget, rf->max_steps) : rf->max_steps;
        for (int it = 0; it <= steps; it++) {
            launch_block_refine_residual(A.n, A.rp, A.ci, A.va, shift, V, ldv, W, ldw, rf->R,
                                         rf->ld, b, rf->tol, anorm, rf->flag, rf->count,
                                         rf->part, rf->counter, st);
            if (it == steps) break;
            rc = timed_solve(plan, rf->R, rf->ld, W, ldw, b, st, rf->flag, true);
            if (rc) return rc;
        }
        if (steps < rf->max_steps) {
            flag_if_unset_kernel<<<1, 1, 0, st>>>(rf->flag, rf->short_word);
            note_launch();
        }
        return 0;
    }
    const int *error_word() const override { return plan->error_word(); }
    int *short_word() const override { return rf->budget > 0 ? rf->short_word : nullptr; }
    void set_full(bool f) override { full = f; }
    bool full = false;
};

// ------------------------------------------------------------- Lanczos --
namespace {

struct LanczosBufs {
    int n = 0, ncv0 = 0, kk = 0;
    int64_t ldv = 0;
    double *V = nullptr, *Vn = nullptr, *H = nullptr, *S = nullptr, *theta = nullptr,
           *thsave = nullptr, *w = nullptr, *X = nullptr, *AX = nullptr, *lam = nullptr,
           *r2 = nullptr, *xn2 = nullptr, *h1 = nullptr, *h2 = nullptr, *nrm2 = nullptr;
    int *ord = nullptr, *jstat = nullptr, *dflag = nullptr;
    ReduceScratch rs;
};

__global__ void thsave_kernel(const double *theta, const int *ord, int t, double *thsave,
                              int nret) {
    thsave[nret] = theta[ord[t]];
}

// dst = src * (1/sqrt(nrm2)) ; used for the normalisations the reference does
// with dnrm2 + dscal
inline void normalise(int n, const double *src, const double *nrm2, double *dst,
                      cudaStream_t st) {
    launch_scale_by_invnorm(n, src, nrm2, dst, st);
}

// w <- (I - B B^T) w twice (reference orth_block, src/speigs_core.c:122-132);
// leaves ||w||^2 in nrm2[0].  hcol: optional projected-matrix column.
inline void orth_block(const LanczosBufs &b, const double *B, int m, double *w, double *hcol,
                       cudaStream_t st) {
    if (m > 0) {
        launch_ts_dot(B, b.ldv, b.n, m, w, b.h1, hcol, hcol ? 1 : 0, b.rs, st);
        launch_ts_update_dot(B, b.ldv, b.n, m, w, b.h1, b.h2, hcol, hcol ? 2 : 0, b.rs, st);
        launch_ts_update_norm(B, b.ldv, b.n, m, w, b.h2, b.nrm2, b.rs, st);
    } else {
        launch_ts_norm(b.n, w, b.nrm2, b.rs, st);
    }
}

}  // namespace

// Results: lambda/resid (host, the last Rayleigh-Ritz's nout pairs in Lanczos
// order) and *Xdev (device, their Ritz vectors, leading dimension *ldx).
static int lanczos_device(Operator &op, const DevA &A, int n, int64_t k, const speigs_opts &o,
                          double anorm, double *lambda, double *resid, const double **Xdev,
                          int64_t *ldx, int *nout, speigs_info *info, EngineStats *stats,
                          Arena &ar, double *pinned, cudaStream_t st,
                          const double *warm = nullptr, int64_t warm_cols = 0,
                          int64_t *warm_used = nullptr) {
    int64_t ncv = o.ncv ? o.ncv : std::max<int64_t>(2 * k + 1, 20);
    if (ncv > n) ncv = n;
    if (ncv <= k) ncv = std::min<int64_t>(n, k + 1);
    if (ncv < 2) ncv = std::min<int64_t>(n, 2);
    const int64_t maxit = o.maxit ? o.maxit : 300;
    const double tol = o.tol > 0 ? o.tol : 1e-14;
    const double rtol = tol * std::max(anorm, 1.0);
    const double bthr = 1e-13 * std::max(anorm, 1.0);

    LanczosBufs b;
    b.n = n;
    b.ncv0 = (int)ncv;
    b.kk = (int)std::min<int64_t>(k, ncv);
    b.ldv = ((int64_t)n + 31) & ~(int64_t)31;
    const int ldh = (int)ncv;     // H keeps the leading dimension it was allocated with
    b.V = ar.alloc<double>((size_t)b.ldv * (ncv + 1));
    b.Vn = ar.alloc<double>((size_t)b.ldv * (ncv + 1));
    b.H = ar.alloc<double>((size_t)ncv * ncv);
    b.S = ar.alloc<double>((size_t)ncv * ncv);
    b.theta = ar.alloc<double>(ncv);
    b.thsave = ar.alloc<double>(ncv);
    b.w = ar.alloc<double>(b.ldv);
    b.X = ar.alloc<double>((size_t)b.ldv * b.kk);
    b.AX = ar.alloc<double>((size_t)b.ldv * b.kk);
    b.lam = ar.alloc<double>(b.kk);
    b.r2 = ar.alloc<double>(b.kk);
    b.xn2 = ar.alloc<double>(std::max<int64_t>(ncv + 1, b.kk));
    b.h1 = ar.alloc<double>(ncv + 1);
    b.h2 = ar.alloc<double>(ncv + 1);
    b.nrm2 = ar.alloc<double>(4);
    b.ord = ar.alloc<int>(ncv);
    b.jstat = ar.alloc<int>(2);
    b.dflag = ar.alloc<int>(1);
    const int nblk = (n + 511) / 512 + 1;
    const int maxcols = (int)std::max<int64_t>(ncv + 1, b.kk) + 1;
    b.rs.part = ar.alloc<double>((size_t)nblk * maxcols);
    b.rs.counter = ar.alloc<unsigned>(1);
    b.rs.max_blocks = nblk;
    b.rs.max_cols = maxcols;
    if (ar.failed) return SPEIGS_ERR_MEM;
    cudaMemsetAsync(b.rs.counter, 0, sizeof(unsigned), st);
    cudaMemsetAsync(b.H, 0, sizeof(double) * ncv * ncv, st);

    // pinned scalars read back by the host (the caller's buffer holds >= 2k+16):
    // Ritz values and residuals, a norm and the operator's error word, the
    // betas and error words of two pipelined steps, the restart flag
    double *hs = pinned;
    double *h_lam = hs, *h_r2 = hs + b.kk, *h_nrm = hs + 2 * b.kk;
    double *h_beta = h_nrm + 4;
    int *h_sterr = reinterpret_cast<int *>(h_nrm + 6);
    int *h_rflag = reinterpret_cast<int *>(h_nrm + 7);

    PhaseTimer tm(st);
    double ms_op = 0, ms_ortho = 0, ms_resid = 0, ms_ritz = 0;
    const int *op_err = op.error_word();
    int *h_operr = reinterpret_cast<int *>(h_nrm + 2);
    auto read_nrm = [&](double *out) -> int {
        copy_async(h_nrm, b.nrm2, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (op_err) copy_async(h_operr, op_err, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "lanczos sync");
        tm.resolve();
        if (op_err && *h_operr) {
            set_last_error_text("operator application failed: a solve dependency wait ran out");
            return SPEIGS_ERR_INTERNAL;
        }
        *out = sqrt(h_nrm[0]);
        return 0;
    };

    uint64_t seed = o.seed ? o.seed : 88172645463325252ULL;
    auto rand_vec = [&](double *dst) {
        launch_rand_vec(n, seed, dst, st);
        seed = rng_advance(seed, (uint64_t)n);
    };

    int64_t j = 0, restarts = 0, nconv = 0;
    if (warm_used) *warm_used = 0;
    const int64_t pmax = std::min<int64_t>(warm_cols, ncv - 2);
    if (warm && pmax >= 1) {
        // Start subspace Y (device, n x warm_cols, leading dimension n): the
        // start vector becomes the normalised sum of an orthonormal basis of
        // Y plus a 1e-8 share of the reference's random start (so no
        // eigenvector is missing from it), and the reference's algorithm runs
        // unchanged from there.  Seeding the recurrence with a vector keeps
        // the thick-restart invariant (a rank-one residual), which a set of
        // retained vectors taken from Y would break.  Dependent columns of Y
        // are dropped.
        int q = 0;
        double *acc = b.Vn + (size_t)ncv * b.ldv;   // running sum of the basis
        launch_fill(n, 0.0, acc, st);
        for (int i = 0; i < (int)pmax; i++) {
            double *dst = b.Vn + (size_t)q * b.ldv;
            launch_copy(n, warm + (size_t)i * n, dst, st);
            launch_ts_norm(n, dst, b.nrm2, b.rs, st);
            double n0 = 0;
            if (int e = read_nrm(&n0)) return e;
            if (!(n0 > 0.0)) continue;
            orth_block(b, b.Vn, q, dst, nullptr, st);
            double n1 = 0;
            if (int e = read_nrm(&n1)) return e;
            if (!(n1 > 1e-8 * n0)) continue;
            normalise(n, dst, b.nrm2, dst, st);
            launch_axpby(n, 1.0, dst, 1.0, acc, st);
            q++;
        }
        if (q >= 1) {
            rand_vec(b.w);
            launch_ts_norm(n, b.w, b.nrm2, b.rs, st);
            double nr = 0;
            if (int e = read_nrm(&nr)) return e;
            launch_axpby(n, 1.0 / std::sqrt((double)q), acc, 1e-8 / nr, b.w, st);
            launch_ts_norm(n, b.w, b.nrm2, b.rs, st);
            if (int e = read_nrm(&nr)) return e;
            normalise(n, b.w, b.nrm2, b.V, st);
            j = -1;   // start vector in place
            if (warm_used) *warm_used = q;
        }
    }
    if (j == -1) {
        j = 0;
    } else {
        // start vector (reference :187-191)
        rand_vec(b.w);
        launch_ts_norm(n, b.w, b.nrm2, b.rs, st);
        double nr0 = 0;
        if (int e = read_nrm(&nr0)) return e;
        if (nr0 == 0.0) return SPEIGS_ERR_INTERNAL;
        normalise(n, b.w, b.nrm2, b.V, st);
    }

    // Step jj of the recurrence: operator application, orthogonalisation,
    // and the read-back of beta_jj, complete when evb[jj & 1] is.  The host
    // tests beta_j for breakdown one step late: step j+1 is queued, on the
    // assumption that beta_j passes, before the host waits for beta_j, so
    // the device never idles while the host decides.  A breakdown (rare)
    // drains the stream, runs the reference's recovery and queues step j+1
    // again; everything the speculative step wrote is written again.
    struct StepEvents {
        cudaEvent_t e[2] = {nullptr, nullptr};
        ~StepEvents() { for (auto x : e) if (x) cudaEventDestroy(x); }
    } evb;
    for (auto &x : evb.e)
        if (cudaEventCreateWithFlags(&x, cudaEventDisableTiming) != cudaSuccess)
            return cuda_fail(cudaGetLastError(), "event");
    auto issue_step = [&](int64_t jj) {
        double *vj = b.V + (size_t)jj * b.ldv;
        int t0 = tm.begin();
        op.apply(vj, b.w, st);
        tm.end(t0, &ms_op);
        int t1 = tm.begin();
        orth_block(b, b.V, (int)(jj + 1), b.w, b.H + (size_t)jj * ldh, st);
        tm.end(t1, &ms_ortho);
        copy_async(h_beta + (jj & 1), b.nrm2, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (op_err) copy_async(h_sterr + (jj & 1), op_err, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaEventRecord(evb.e[jj & 1], st);
    };
    auto wait_beta = [&](int64_t jj, double *beta) -> int {
        cudaError_t e = cudaEventSynchronize(evb.e[jj & 1]);
        if (e != cudaSuccess) return cuda_fail(e, "lanczos sync");
        if (op_err && h_sterr[jj & 1]) {
            set_last_error_text("operator application failed: a solve dependency wait ran out");
            return SPEIGS_ERR_INTERNAL;
        }
        *beta = sqrt(h_beta[jj & 1]);
        return 0;
    };
    auto drain = [&]() -> int {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "lanczos sync");
        tm.resolve();
        return 0;
    };

    int rc = SPEIGS_OK;
    int last_nwant = 0;   // Ritz vectors of the last Rayleigh-Ritz stay in X
    for (;;) {
        // ---- extend the basis from j to ncv (reference :197-229)
        if (j < ncv) issue_step(j);
        for (; j < ncv; j++) {
            normalise(n, b.w, b.nrm2, b.V + (size_t)(j + 1) * b.ldv, st);
            if (j + 1 < ncv) {
                launch_set_beta(b.H, ldh, (int)(j + 1), (int)j, b.nrm2, 0, st);
                issue_step(j + 1);
            }
            double beta = 0;
            if (int e = wait_beta(j, &beta)) return e;
            if (beta > bthr) continue;
            // breakdown at step j (reference :205-216); the speculative step
            // j+1 does not count as an operator application
            if (int e = drain()) return e;
            if (j + 1 < ncv) op.nops--;
            for (int att = 0; att < 3 && beta <= bthr; att++) {
                rand_vec(b.w);
                orth_block(b, b.V, (int)(j + 1), b.w, nullptr, st);
                if (int e = read_nrm(&beta)) return e;
            }
            if (beta <= bthr) {
                // column j+1 holds the speculative normalisation, which is
                // not part of the basis
                launch_fill(n, 0.0, b.V + (size_t)(j + 1) * b.ldv, st);
                ncv = j + 1;
                break;
            }
            normalise(n, b.w, b.nrm2, b.V + (size_t)(j + 1) * b.ldv, st);
            if (j + 1 < ncv) {
                launch_set_beta(b.H, ldh, (int)(j + 1), (int)j, b.nrm2, 1, st);
                issue_step(j + 1);
            }
        }

        // ---- projected eigenproblem (reference :231-240)
        const int m = (int)ncv;
        int tr = tm.begin();
        if (int e = syev_projected(m, b.H, ldh, b.theta, b.S, b.ord, b.jstat, st)) return e;

        // ---- true residuals of the wanted Ritz pairs (reference :242-265)
        const int nwant = (int)std::min<int64_t>(k, m);
        launch_ritz_vectors(b.V, b.ldv, n, m, b.S, m, b.ord, 0, nwant, b.X, b.ldv, b.xn2, b.rs, st);
        launch_scale_cols(n, nwant, b.X, b.ldv, b.xn2, st);
        for (int t = 0; t < nwant; t++)
            launch_spmv(A.n, A.rp, A.ci, A.va, b.X + (size_t)t * b.ldv, b.AX + (size_t)t * b.ldv, st);
        launch_rayleigh_resid(n, nwant, b.X, b.ldv, b.AX, b.ldv, b.lam, b.r2, b.rs, st);
        tm.end(tr, &ms_resid);
        int jst[2] = {0, 0};
        copy_async(h_lam, b.lam, sizeof(double) * nwant, cudaMemcpyDeviceToHost, st);
        copy_async(h_r2, b.r2, sizeof(double) * nwant, cudaMemcpyDeviceToHost, st);
        copy_async(jst, b.jstat, sizeof(int), cudaMemcpyDeviceToHost, st);
        {
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cuda_fail(e, "residual sync");
            tm.resolve();
        }
        if (jst[0] < 0) { rc = SPEIGS_ERR_LAPACK; break; }
        nconv = 0;
        for (int t = 0; t < nwant; t++) {
            const double r = sqrt(h_r2[t]);
            lambda[t] = h_lam[t];
            if (resid) resid[t] = r;
            if (r <= rtol) nconv++;
        }
        last_nwant = nwant;

        if (nconv >= std::min<int64_t>(k, m) || restarts >= maxit || m < ncv) break;
        restarts++;

        // ---- thick restart: keep the top-l Ritz vectors (reference :270-303)
        int64_t l = std::min<int64_t>(k + 5, ncv - 1);
        if (l < 1) l = 1;
        // The retained vectors are queued without host reads; a vector that
        // orthogonalisation leaves with norm < 1e-10 raises dflag, and then
        // the loop is redone with the reference's per-vector test, which
        // skips such vectors.
        int nret = 0;
        double nr = 0;
        auto continuation = [&]() -> int {
            // the (m+1)-th Lanczos vector continues the recurrence
            launch_copy(n, b.V + (size_t)m * b.ldv, b.w, st);
            orth_block(b, b.Vn, nret, b.w, nullptr, st);
            return read_nrm(&nr);
        };
        bool per_vector = l > m;
        if (!per_vector) {
            int tk = tm.begin();
            cudaMemsetAsync(b.dflag, 0, sizeof(int), st);
            // all l Ritz vectors in one pass over V (each column is summed
            // in the same order as when it is formed alone)
            launch_ritz_vectors(b.V, b.ldv, n, m, b.S, m, b.ord, 0, (int)l, b.Vn, b.ldv, b.xn2,
                                b.rs, st);
            for (int t = 0; t < (int)l; t++) {
                double *dst = b.Vn + (size_t)t * b.ldv;
                orth_block(b, b.Vn, t, dst, nullptr, st);
                launch_flag_if_below(b.nrm2, 1e-20, b.dflag, st);
                normalise(n, dst, b.nrm2, dst, st);
                thsave_kernel<<<1, 1, 0, st>>>(b.theta, b.ord, t, b.thsave, t);
                note_launch();
            }
            copy_async(h_rflag, b.dflag, sizeof(int), cudaMemcpyDeviceToHost, st);
            tm.end(tk, &ms_ritz);
            nret = (int)l;
            if (int e = continuation()) return e;
            per_vector = *h_rflag != 0;
        }
        if (per_vector) {
            nret = 0;
            int tk = tm.begin();
            for (int t = 0; t < m && nret < l; t++) {
                double *dst = b.Vn + (size_t)nret * b.ldv;
                launch_ritz_vectors(b.V, b.ldv, n, m, b.S, m, b.ord, t, 1, dst, b.ldv, b.xn2, b.rs,
                                    st);
                orth_block(b, b.Vn, nret, dst, nullptr, st);
                double nv = 0;
                if (int e = read_nrm(&nv)) return e;
                if (nv < 1e-10) continue;
                normalise(n, dst, b.nrm2, dst, st);
                thsave_kernel<<<1, 1, 0, st>>>(b.theta, b.ord, t, b.thsave, nret);
                note_launch();
                nret++;
            }
            tm.end(tk, &ms_ritz);
            if (int e = continuation()) return e;
        }
        if (nr < 1e-10) {
            rand_vec(b.w);
            orth_block(b, b.Vn, nret, b.w, nullptr, st);
            if (int e = read_nrm(&nr)) return e;
        }
        if (nr < 1e-10) break;
        normalise(n, b.w, b.nrm2, b.Vn + (size_t)nret * b.ldv, st);
        std::swap(b.V, b.Vn);
        launch_set_diag(ldh, nret, b.thsave, b.H, st);
        j = nret;
    }
    if (rc) return rc;
    *Xdev = b.X;
    *ldx = b.ldv;
    *nout = last_nwant;
    {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "lanczos end");
        tm.resolve();
    }
    info->nconv = nconv;
    info->restarts = restarts;
    info->nops = op.nops;
    info->flag = (nconv >= std::min<int64_t>(k, ncv)) ? 0 : 1;
    info->t_op += ms_op * 1e-3;
    info->t_ortho += ms_ortho * 1e-3;
    info->t_resid += ms_resid * 1e-3;
    info->t_ritz += ms_ritz * 1e-3;
    if (stats) {
        stats->ms_op += ms_op; stats->ms_ortho += ms_ortho;
        stats->ms_resid += ms_resid; stats->ms_ritz += ms_ritz;
    }
    return SPEIGS_OK;
}

// ------------------------------------------------------- block Lanczos --
// Block thick-restart Lanczos for the shift-invert operator: the Rayleigh-
// Ritz projection of Op on a basis grown a block of b vectors at a time,
// restarted from the l = k + 5 wanted Ritz vectors plus the current
// residual block.  It starts from a block -- the caller's start subspace
// (the learned proposal), completed with the reference's random stream --
// so a proposal that already holds the wanted eigenvectors is used in full,
// and every block application reads the factor once for b vectors.
//
// Layout: V is n x (mmax + b) column-major (ld padded to 32); after a block
// at columns [jc, jc + b) is applied, H[0 : jc + b, jc : jc + b] = V^T Op V
// (two Gram-Schmidt passes, both summed) and the orthonormalised residual
// becomes the next block at [jc + b, jc + 2b).  H is read from its upper
// triangle, so it is exactly the projection V^T Op V whatever the block
// structure; dependent residual columns are replaced by vectors of the
// random stream.  Convergence is decided as in the reference: true
// residuals ||A x - lambda x|| <= tol max(||A||_1, 1) with lambda the
// Rayleigh quotient of A, for the k Ritz vectors of largest |theta|.  The
// projected problem is solved at the end of each cycle (and once after the
// first block of a start subspace); the residual of the block recurrence
// (cheap: a b x b Gram matrix) decides whether the true-residual test runs
// before the cycle's last check.
namespace {

struct BlockLanczosBufs {
    int n = 0, b = 0, mmax = 0;
    int64_t ldv = 0;
    double *V = nullptr, *Vn = nullptr, *H = nullptr, *S = nullptr, *theta = nullptr,
           *hb = nullptr, *G = nullptr, *Gres = nullptr, *Rinv = nullptr, *est2 = nullptr,
           *X = nullptr, *AX = nullptr, *lam = nullptr, *r2 = nullptr, *xn2 = nullptr;
    int *ord = nullptr, *jstat = nullptr, *cstat = nullptr;
    ReduceScratch rs;
    BlockScratch bs;
};

}  // namespace

static int block_lanczos_device(BlockOperator &op, const DevA &A, int n, int64_t k, int b,
                                const speigs_opts &o, double anorm, double shift, double *lambda,
                                double *resid, const double **Xdev, int64_t *ldx, int *nout,
                                speigs_info *info, EngineStats *stats, Arena &ar, double *pinned,
                                cudaStream_t st, const double *Y, int64_t p, int64_t *warm_used) {
    const int64_t maxit = o.maxit ? o.maxit : 300;
    const double tol = o.tol > 0 ? o.tol : 1e-14;
    const double rtol = tol * std::max(anorm, 1.0);
    const double bthr = 1e-13 * std::max(anorm, 1.0);
    const int64_t ncv_ref = o.ncv ? o.ncv : std::max<int64_t>(2 * k + 1, 20);
    const int kk = (int)k;
    const int l0 = (int)std::min<int64_t>(k + 5, n);
    int mmax = (int)std::max<int64_t>(ncv_ref, l0 + 3 * b);
    mmax = std::min(mmax, kBlockMaxM);
    mmax = std::min<int>(mmax, n - b);
    if (mmax < l0 + b || mmax < kk) return SPEIGS_ERR_ARG;

    BlockLanczosBufs B;
    B.n = n;
    B.b = b;
    B.mmax = mmax;
    B.ldv = ((int64_t)n + 31) & ~(int64_t)31;
    const int ldh = mmax;
    const int cols = mmax + b;
    B.V = ar.alloc<double>((size_t)B.ldv * cols);
    B.Vn = ar.alloc<double>((size_t)B.ldv * cols);
    B.H = ar.alloc<double>((size_t)ldh * ldh);
    B.S = ar.alloc<double>((size_t)ldh * ldh);
    B.theta = ar.alloc<double>(ldh);
    B.hb = ar.alloc<double>((size_t)ldh * b);
    B.G = ar.alloc<double>((size_t)b * b);
    B.Gres = ar.alloc<double>((size_t)b * b);
    B.Rinv = ar.alloc<double>((size_t)b * b);
    B.est2 = ar.alloc<double>(kk);
    B.X = ar.alloc<double>((size_t)B.ldv * kk);
    B.AX = ar.alloc<double>((size_t)B.ldv * kk);
    B.lam = ar.alloc<double>(kk);
    B.r2 = ar.alloc<double>(kk);
    B.xn2 = ar.alloc<double>(std::max(cols, kk));
    B.ord = ar.alloc<int>(ldh);
    B.jstat = ar.alloc<int>(2);
    B.cstat = ar.alloc<int>(4);
    const int nblk = (n + 511) / 512 + 1;
    const int maxc = std::max(cols, kk) + 1;
    B.rs.part = ar.alloc<double>((size_t)nblk * maxc);
    B.rs.counter = ar.alloc<unsigned>(1);
    B.rs.max_blocks = nblk;
    B.rs.max_cols = maxc;
    B.bs.max_parts = tsb_parts(n);
    B.bs.part = ar.alloc<double>((size_t)B.bs.max_parts * kBlockMaxM * kBlockMaxB);
    if (ar.failed) return SPEIGS_ERR_MEM;
    cudaMemsetAsync(B.rs.counter, 0, sizeof(unsigned), st);
    cudaMemsetAsync(B.H, 0, sizeof(double) * ldh * ldh, st);

    // pinned read-back: lam[k], r2[k], est2[k], theta of the wanted[k],
    // a status pair and the operator's error word
    double *h_lam = pinned, *h_r2 = pinned + kk, *h_est = pinned + 2 * kk,
           *h_th = pinned + 3 * kk;
    int *h_stat = reinterpret_cast<int *>(pinned + 4 * kk);
    int *h_jst = h_stat + 2;
    int *h_operr = h_stat + 4;
    const int *op_err = op.error_word();

    PhaseTimer tm(st);
    double ms_op = 0, ms_ortho = 0, ms_resid = 0, ms_ritz = 0;
    // the operator times its block solves with this loop's timer (resolved
    // at each sync) until the loop returns
    struct TimerLink {
        BlockOperator &o;
        ~TimerLink() { o.tm = nullptr; }
    } tlink{op};
    op.tm = &tm;
    op.ms_solve = &op.ms_solve_acc;
    auto sync = [&](const char *where) -> int {
        if (op_err) copy_async(h_operr, op_err, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, where);
        tm.resolve();
        if (op_err && *h_operr) {
            set_last_error_text("operator application failed: a solve dependency wait ran out");
            return SPEIGS_ERR_INTERNAL;
        }
        return 0;
    };

    uint64_t seed = o.seed ? o.seed : 88172645463325252ULL;
    auto rand_col = [&](double *dst) {
        launch_rand_vec(n, seed, dst, st);
        seed = rng_advance(seed, (uint64_t)n);
    };
    // W (b columns at Wp) <- (I - V V^T) W twice against V[:, 0:m]; with
    // hcol, the two passes' coefficients are summed into H[0:m, hcol..];
    // with gram, the Gram matrix W^T W of the result is left in B.G.
    // Returns whether it was (m > 0).
    auto cgs2 = [&](double *Wp, int m, double *hcol, bool gram) -> bool {
        if (m <= 0) return false;
        double *V = B.V;
        // pass 1's update and pass 2's product share one sweep over V, and
        // pass 2's update the sweep that forms the Gram matrix
        double *h1 = hcol ? hcol : B.hb;
        launch_tsb_tn(V, B.ldv, n, m, Wp, B.ldv, b, h1, ldh, 0, B.bs, st);
        launch_tsb_sub_tn(V, B.ldv, n, m, h1, ldh, Wp, B.ldv, b, B.hb, ldh, 0, B.bs, st);
        if (gram) launch_tsb_sub_gram(V, B.ldv, n, m, B.hb, ldh, Wp, B.ldv, b, B.G, B.bs, st);
        else launch_tsb_nn_sub(V, B.ldv, n, m, B.hb, ldh, Wp, B.ldv, b, st);
        if (hcol) launch_block_axpy_unless(m, b, hcol, ldh, B.hb, ldh, nullptr, st);
        return gram;
    };
    // Orthonormalise the block at Wp against V[:, 0:m] (already projected
    // out) and within itself by two Cholesky QR passes.  Columns found
    // dependent are replaced by random vectors and the block is projected
    // again (up to three times).  *replaced gets the columns replaced in the
    // first test; returns 1 when the block stays dependent (no extension).
    // With spec, the dependency test is not read back: the first pass goes
    // on as if no column were dependent, and the Cholesky kernel's sticky
    // flag (cstat[2]) tells the caller later whether the step must be redone.
    // gram_ready: B.G already holds W^T W (left there by cgs2).
    auto orthonormalise = [&](double *Wp, int m, unsigned *replaced, bool keep_gram,
                              bool spec, bool gram_ready = false) -> int {
        unsigned first_mask = 0;
        if (spec) {
            if (!gram_ready) launch_tsb_tn(Wp, B.ldv, n, b, Wp, B.ldv, b, B.G, b, 0, B.bs, st);
            if (keep_gram)
                cudaMemcpyAsync(B.Gres, B.G, sizeof(double) * b * b, cudaMemcpyDeviceToDevice, st);
            launch_block_chol(b, B.G, b, B.Rinv, bthr, 1e-14, B.cstat, st);
        }
        for (int att = 0; !spec; att++) {
            if (!(gram_ready && att == 0))
                launch_tsb_tn(Wp, B.ldv, n, b, Wp, B.ldv, b, B.G, b, 0, B.bs, st);
            if (keep_gram && att == 0)
                cudaMemcpyAsync(B.Gres, B.G, sizeof(double) * b * b, cudaMemcpyDeviceToDevice, st);
            launch_block_chol(b, B.G, b, B.Rinv, bthr, 1e-14, B.cstat, st);
            copy_async(h_stat, B.cstat, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
            if (int e = sync("block orthonormalisation")) return e;
            const unsigned mask = (unsigned)h_stat[0];
            if (att == 0) first_mask = mask;
            if (!h_stat[1]) break;
            if (att == 3) {
                if (replaced) *replaced = first_mask;
                return 1;
            }
            for (int c = 0; c < b; c++)
                if ((mask >> c) & 1u) rand_col(Wp + (size_t)c * B.ldv);
            cgs2(Wp, m, nullptr, false);
        }
        // the first Cholesky QR step and the second step's Gram matrix
        launch_tsb_mul_gram(n, b, Wp, B.ldv, B.Rinv, B.G, B.bs, st);
        launch_block_chol(b, B.G, b, B.Rinv, 0.0, 0.0, B.cstat, st);
        launch_tsb_right_mul(n, b, Wp, B.ldv, B.Rinv, st);
        if (replaced) *replaced = first_mask;
        return 0;
    };

    // ---- start block: the proposal's columns, completed with random ones.
    // A proposal wider than the block is first reduced to its b best
    // directions: the Rayleigh-Ritz vectors of A on span(Y) whose Ritz values
    // lie nearest the wanted end (smallest |theta + shift|), formed from the
    // orthonormalised proposal (b SpMV columns at a time would do too; one
    // SpMV per column is cheap beside a block solve).
    if (warm_used) *warm_used = 0;
    const double *Ysrc = Y;
    int64_t psrc = Y ? p : 0;
    bool compressed = false;
    if (Y && p > b && p <= kBlockMaxB) {
        const int q = (int)p;
        double *Yp = ar.alloc<double>((size_t)B.ldv * q), *AY = ar.alloc<double>((size_t)B.ldv * q);
        double *G32 = ar.alloc<double>((size_t)q * q), *R32 = ar.alloc<double>((size_t)q * q);
        double *Hq = ar.alloc<double>((size_t)q * q), *Sq = ar.alloc<double>((size_t)q * b);
        int *cst = ar.alloc<int>(4);
        if (ar.failed) return SPEIGS_ERR_MEM;
        for (int c = 0; c < q; c++) launch_copy(n, Y + (size_t)c * n, Yp + (size_t)c * B.ldv, st);
        for (int pass = 0; pass < 2; pass++) {
            launch_tsb_tn(Yp, B.ldv, n, q, Yp, B.ldv, q, G32, q, 0, B.bs, st);
            launch_block_chol(q, G32, q, R32, bthr, 1e-14, cst, st);
            launch_tsb_right_mul(n, q, Yp, B.ldv, R32, st);
        }
        for (int c = 0; c < q; c++)
            launch_spmv(A.n, A.rp, A.ci, A.va, Yp + (size_t)c * B.ldv, AY + (size_t)c * B.ldv, st);
        launch_tsb_tn(Yp, B.ldv, n, q, AY, B.ldv, q, Hq, q, 0, B.bs, st);
        std::vector<double> hH((size_t)q * q), th(q), hS((size_t)q * q), sel((size_t)q * b);
        std::vector<int> ordv(q);
        int hst[4] = {0, 0, 0, 0};
        copy_async(hst, cst, sizeof(int) * 2, cudaMemcpyDeviceToHost, st);
        copy_async(hH.data(), Hq, sizeof(double) * q * q, cudaMemcpyDeviceToHost, st);
        if (int e = sync("start subspace")) return e;
        if (!hst[1] && syev_host(q, hH.data(), q, th.data(), hS.data(), ordv.data()) >= 0) {
            std::vector<int> idx(q);
            for (int i = 0; i < q; i++) idx[i] = i;
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
                return std::fabs(th[x] + shift) < std::fabs(th[y] + shift);
            });
            for (int c = 0; c < b; c++)
                std::memcpy(sel.data() + (size_t)c * q, hS.data() + (size_t)idx[c] * q,
                            sizeof(double) * q);
            copy_async(Sq, sel.data(), sizeof(double) * q * b, cudaMemcpyHostToDevice, st);
            // V[:, 0:b] = Yp * S_sel (the product reads Yp only)
            launch_tsb_right_mul_into(n, q, Yp, B.ldv, Sq, q, B.V, B.ldv, b, st);
            if (int e = sync("start subspace")) return e;      // the host vectors die here
            compressed = true;
            psrc = b;
        }
    }
    const int pp = (int)std::min<int64_t>(psrc, b);
    for (int c = 0; c < b && !compressed; c++) {
        double *dst = B.V + (size_t)c * B.ldv;
        if (c < pp) launch_copy(n, Ysrc + (size_t)c * n, dst, st);
        else rand_col(dst);
    }
    {
        unsigned rep = 0;
        int e = orthonormalise(B.V, 0, &rep, false, false);
        if (e < 0) return e;
        if (e == 1) return SPEIGS_ERR_INTERNAL;
        int used = 0;
        for (int c = 0; c < pp; c++) used += ((rep >> c) & 1u) ? 0 : 1;
        if (warm_used) *warm_used = used;
    }

    int jc = 0, mm = 0;
    // Cycles run speculatively (no host read per block step); the state a
    // cycle starts from -- V[:, 0:jc + b] and H[:, 0:jc] -- is not written
    // during the cycle, so a cycle in which a block lost rank is redone from
    // it with the per-step test.
    int *h_dep = h_stat + 6;
    int jc_cycle = 0;
    int64_t napps_cycle = 0, nvecs_cycle = 0;
    bool spec_cycle = true;
    auto start_cycle = [&]() {
        jc_cycle = jc;
        napps_cycle = op.napps;
        nvecs_cycle = op.nvecs;
        spec_cycle = true;
        op.set_full(false);
        cudaMemsetAsync(B.cstat + 2, 0, sizeof(int), st);
    };
    start_cycle();
    int64_t restarts = 0, nconv = 0;
    int last_nwant = 0;
    int rc = SPEIGS_OK;
    bool have_result = false;
    for (;;) {
        // ---- apply Op to the block at [jc, jc + b); project; orthonormalise
        double *Vb = B.V + (size_t)jc * B.ldv;
        double *Wp = B.V + (size_t)(jc + b) * B.ldv;
        int t0 = tm.begin();
        if (int e = op.apply(Vb, B.ldv, Wp, B.ldv, b, st)) return e;
        tm.end(t0, &ms_op);
        mm = jc + b;
        int t1 = tm.begin();
        const bool gram = cgs2(Wp, mm, B.H + (size_t)jc * ldh, true);
        unsigned rep = 0;
        const int stuck = orthonormalise(Wp, mm, &rep, true, spec_cycle, gram);
        if (stuck < 0) return stuck;
        tm.end(t1, &ms_ortho);
        const bool cycle_end = stuck == 1 || mm + b > mmax;
        // The projected problem is solved where the reference solves it, at
        // the end of a cycle, and also after the first block application of
        // a start subspace: a proposal that already holds the wanted
        // eigenvectors is then finished by one block solve.
        const bool first_warm = (restarts == 0 && jc == 0 && pp > 0);
        if (!cycle_end && !first_warm) {
            jc = mm;
            continue;
        }
        if (spec_cycle || op.short_word()) {
            // a block that lost rank in this cycle, or an application that
            // fell short of its accuracy: redo the cycle from its start, with
            // the dependency test read after every step and the full
            // refinement loop
            copy_async(h_dep, B.cstat + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
            h_dep[1] = 0;
            if (op.short_word())
                copy_async(h_dep + 1, op.short_word(), sizeof(int), cudaMemcpyDeviceToHost, st);
            if (int e = sync("block step check")) return e;
            if ((spec_cycle && h_dep[0]) || h_dep[1]) {
                cudaMemsetAsync(B.cstat + 2, 0, sizeof(int), st);
                if (op.short_word()) cudaMemsetAsync(op.short_word(), 0, sizeof(int), st);
                op.napps = napps_cycle;
                op.nvecs = nvecs_cycle;
                jc = jc_cycle;
                spec_cycle = false;
                op.set_full(true);
                continue;
            }
        }

        // ---- Rayleigh-Ritz on H[0:mm, 0:mm]; the recurrence's residual
        // estimates gate the true-residual test
        const int nwant = std::min(kk, mm);
        int tr = tm.begin();
        // the Ritz vectors read later are the nwant wanted ones and the l
        // kept at a restart
        if (int e = syev_projected(mm, B.H, ldh, B.theta, B.S, B.ord, B.jstat, st,
                                   std::max(nwant, std::min(l0, mm))))
            return e;
        launch_block_ritz_est(nwant, b, B.S, mm, jc, B.ord, B.Gres, b, B.est2, st);
        tm.end(tr, &ms_ritz);
        {
            // theta of the wanted pairs, in ord order
            copy_async(h_est, B.est2, sizeof(double) * nwant, cudaMemcpyDeviceToHost, st);
            copy_async(h_jst, B.jstat, sizeof(int), cudaMemcpyDeviceToHost, st);
            std::vector<int> ordh(nwant);
            std::vector<double> thh(mm);
            copy_async(ordh.data(), B.ord, sizeof(int) * nwant, cudaMemcpyDeviceToHost, st);
            copy_async(thh.data(), B.theta, sizeof(double) * mm, cudaMemcpyDeviceToHost, st);
            if (int e = sync("block ritz")) return e;
            if (h_jst[0] < 0) { rc = SPEIGS_ERR_LAPACK; break; }
            for (int t = 0; t < nwant; t++) h_th[t] = thh[ordh[t]];
        }
        bool gate = nwant >= kk;
        for (int t = 0; t < nwant && gate; t++) {
            const double th = std::fabs(h_th[t]);
            const double est = std::sqrt(std::max(h_est[t], 0.0)) * (anorm + std::fabs(shift)) /
                               std::max(th, 1e-300);
            if (!(est <= 10.0 * rtol)) gate = false;
        }
        if (gate || cycle_end) {
            int t2 = tm.begin();
            launch_ritz_vectors(B.V, B.ldv, n, mm, B.S, mm, B.ord, 0, nwant, B.X, B.ldv, B.xn2,
                                B.rs, st);
            launch_scale_cols(n, nwant, B.X, B.ldv, B.xn2, st);
            for (int t = 0; t < nwant; t++)
                launch_spmv(A.n, A.rp, A.ci, A.va, B.X + (size_t)t * B.ldv,
                            B.AX + (size_t)t * B.ldv, st);
            launch_rayleigh_resid(n, nwant, B.X, B.ldv, B.AX, B.ldv, B.lam, B.r2, B.rs, st);
            tm.end(t2, &ms_resid);
            copy_async(h_lam, B.lam, sizeof(double) * nwant, cudaMemcpyDeviceToHost, st);
            copy_async(h_r2, B.r2, sizeof(double) * nwant, cudaMemcpyDeviceToHost, st);
            if (int e = sync("block residuals")) return e;
            nconv = 0;
            for (int t = 0; t < nwant; t++) {
                const double r = std::sqrt(h_r2[t]);
                lambda[t] = h_lam[t];
                if (resid) resid[t] = r;
                if (r <= rtol) nconv++;
            }
            last_nwant = nwant;
            have_result = true;
            if (nconv >= kk) break;
        }
        if (!cycle_end) {
            jc = mm;
            continue;
        }
        if (restarts >= maxit || stuck == 1) break;
        restarts++;

        // ---- thick restart: the l wanted Ritz vectors and the residual block
        const int l = std::min(l0, std::min(mm, mmax - b));
        int tk = tm.begin();
        launch_ritz_vectors(B.V, B.ldv, n, mm, B.S, mm, B.ord, 0, l, B.Vn, B.ldv, B.xn2, B.rs, st);
        launch_scale_cols(n, l, B.Vn, B.ldv, B.xn2, st);
        launch_block_copy(n, b, B.V + (size_t)mm * B.ldv, B.ldv, B.Vn + (size_t)l * B.ldv, B.ldv,
                          st);
        std::swap(B.V, B.Vn);
        launch_block_set_diag(ldh, mmax, l, B.theta, B.ord, B.H, st);
        tm.end(tk, &ms_ritz);
        jc = l;
        start_cycle();
    }
    if (rc) return rc;
    if (!have_result) return SPEIGS_ERR_INTERNAL;
    *Xdev = B.X;
    *ldx = B.ldv;
    *nout = last_nwant;
    if (int e = sync("block lanczos end")) return e;
    info->nconv = nconv;
    info->restarts = restarts;
    info->nops = op.nvecs;
    info->flag = (nconv >= kk) ? 0 : 1;
    info->t_op += ms_op * 1e-3;
    info->t_ortho += ms_ortho * 1e-3;
    info->t_resid += ms_resid * 1e-3;
    info->t_ritz += ms_ritz * 1e-3;
    if (stats) {
        stats->ms_op += ms_op; stats->ms_ortho += ms_ortho;
        stats->ms_resid += ms_resid; stats->ms_ritz += ms_ritz;
    }
    return SPEIGS_OK;
}

// ----------------------------------------------------------- host CSR --
int build_full_csr(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                   HostCSR *out) {
    if (n <= 0 || n > INT32_MAX) return SPEIGS_ERR_ARG;
    int64_t *cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    if (!cnt) return SPEIGS_ERR_MEM;
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            const int64_t r = Ai[q];
            if (r > c) continue;
            cnt[r + 1]++;
            if (r != c) cnt[c + 1]++;
        }
    for (int64_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
    const int64_t nnz = cnt[n];
    if (nnz > INT32_MAX) { free(cnt); return SPEIGS_ERR_MEM; }
    int32_t *ci = (int32_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(int32_t));
    double *cx = (double *)malloc((size_t)(nnz ? nnz : 1) * sizeof(double));
    int64_t *fill = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    if (!ci || !cx || !fill) { free(cnt); free(ci); free(cx); free(fill); return SPEIGS_ERR_MEM; }
    memcpy(fill, cnt, (size_t)n * sizeof(int64_t));
    // pass 1: entries (r, c) with r <= c go to row r in increasing c;
    // pass 2: their mirrors (c, r), r < c, go to row c in increasing r.
    // Row i then holds columns < i from pass 2 after columns >= i from pass 1.
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            const int64_t r = Ai[q];
            if (r > c) continue;
            const int64_t d = fill[r]++;
            ci[d] = (int32_t)c; cx[d] = Ax[q];
        }
    for (int64_t c = 0; c < n; c++)
        for (int64_t q = Ap[c]; q < Ap[c + 1]; q++) {
            const int64_t r = Ai[q];
            if (r >= c) continue;
            const int64_t d = fill[c]++;
            ci[d] = (int32_t)r; cx[d] = Ax[q];
        }
    free(fill);
    // rotate each row so its columns are ascending: [>= i part][< i part]
    std::vector<int32_t> tc;
    std::vector<double> tx;
    for (int64_t i = 0; i < n; i++) {
        const int64_t a = cnt[i], e = cnt[i + 1];
        int64_t split = a;
        while (split < e && ci[split] >= i) split++;
        if (split == a || split == e) continue;
        tc.assign(ci + split, ci + e);
        tx.assign(cx + split, cx + e);
        tc.insert(tc.end(), ci + a, ci + split);
        tx.insert(tx.end(), cx + a, cx + split);
        std::copy(tc.begin(), tc.end(), ci + a);
        std::copy(tx.begin(), tx.end(), cx + a);
    }
    out->n = (int32_t)n;
    out->rowptr = cnt;
    out->col = ci;
    out->val = cx;
    return SPEIGS_OK;
}

int build_full_csr_sorted(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
                          HostCSR *out) {
    if (n <= 0 || n > INT32_MAX) return SPEIGS_ERR_ARG;
    const int64_t nnz = Ap[n];
    if (nnz > INT32_MAX) return SPEIGS_ERR_MEM;
    int64_t *rp = (int64_t *)malloc((size_t)(n + 1) * sizeof(int64_t));
    int32_t *ci = (int32_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(int32_t));
    double *cx = (double *)malloc((size_t)(nnz ? nnz : 1) * sizeof(double));
    if (!rp || !ci || !cx) { free(rp); free(ci); free(cx); return SPEIGS_ERR_MEM; }
    memcpy(rp, Ap, (size_t)(n + 1) * sizeof(int64_t));
    parallel_ranges(n, 8192, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; i++)
            for (int64_t q = Ap[i]; q < Ap[i + 1]; q++) {
                const int64_t r = Ai[q];
                ci[q] = (int32_t)r;
                if (r <= i) {
                    cx[q] = Ax[q];                       // (r, i) is in the upper triangle
                } else {
                    // the upper-triangle mirror (i, r) sits in column r
                    const int64_t *f = std::lower_bound(Ai + Ap[r], Ai + Ap[r + 1], i);
                    cx[q] = Ax[f - Ai];
                }
            }
    });
    out->n = (int32_t)n;
    out->rowptr = rp;
    out->col = ci;
    out->val = cx;
    return SPEIGS_OK;
}

void free_csr(HostCSR *A) {
    free(A->rowptr); free(A->col); free(A->val);
    A->rowptr = nullptr; A->col = nullptr; A->val = nullptr; A->n = 0;
}

static double wall() {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

// ------------------------------------------------------------- the plan --
}  // namespace spx

struct speigs_plan_s {
    spx::Stream stream;
    spx::HostCSR A;                  // full symmetric CSR (host copy of the pattern)
    std::vector<int64_t> csc2csr;    // per CSC entry: CSR position(s) it feeds, or -1
    int64_t csc_nnz = 0;
    std::vector<int64_t> Ap_copy;    // CSC column pointers given at creation
    std::vector<int64_t> Ai_copy;
    speigs_which which = SPEIGS_SM;
    speigs_opts opts;
    double anorm = 1.0;
    double shift = 0.0;
    bool factored = false;
    int32_t *d_rp = nullptr, *d_ci = nullptr;
    double *d_va = nullptr;
    spx::Factor mf;
    bool banded = false;              // reported as the reference's banded route
    bool reuse_factor = false;        // factor cache hit: the numeric factor is current
    bool lu = false;                  // indefinite route: the dense inverse below
    double *d_ainv = nullptr;         // n x n, allocated on first use
    spx::RefineState refine;          // mixed precision only
    double refine_tol_user = 0;       // speigs_ext_opts.refine_tol (0: from opts.tol)
    int64_t refine_reported = 0;      // corrections already reported
    int64_t last_refine = 0;          // corrections of the last solve
    int64_t last_ops = 0;             // operator applications of the last solve
    const double *ext_warm = nullptr; // start subspace (host, n x ext_warm_cols)
    int64_t ext_warm_cols = 0;
    int64_t last_warm = 0;            // start-subspace columns used by the last solve
    int ext_block = 0;                // speigs_ext_opts.block
    int last_block = 0;               // block size of the last solve (0: single vector)
    int64_t last_block_solves = 0;    // its block solves (applications + corrections)
    double last_t_block_solve = 0;    // device time of its block solves (s)
    int64_t last_block_solve_calls = 0;   // block solves queued (corrections skipped on
                                          // the device included)
    double t_analyze = 0;
    std::vector<void *> owned;
};

namespace spx {

static int plan_upload_values(speigs_plan_s *p) {
    const int64_t nnz = p->A.nnz();
    cudaError_t e = copy_async(p->d_va, p->A.val, sizeof(double) * nnz,
                                    cudaMemcpyHostToDevice, p->stream.s);
    if (e != cudaSuccess) return cuda_fail(e, "upload values");
    e = cudaStreamSynchronize(p->stream.s);
    if (e != cudaSuccess) return cuda_fail(e, "upload values");
    p->factored = false;
    return 0;
}

static int plan_alloc(speigs_plan_s *p, void **ptr, size_t bytes) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPool_t pool = device_pool(dev);
    cudaError_t e = pool ? cudaMallocFromPoolAsync(ptr, bytes ? bytes : 1, pool, p->stream.s)
                         : cudaMallocAsync(ptr, bytes ? bytes : 1, p->stream.s);
    if (e != cudaSuccess) { cudaGetLastError(); return SPEIGS_ERR_MEM; }
    p->owned.push_back(*ptr);
    return 0;
}

// Build the plan from an already expanded full CSR (takes ownership of A).
int plan_from_csr(HostCSR &A, speigs_which which, const speigs_opts &o, double anorm,
                  const speigs_ext_opts *ext, speigs_plan_s **out) {
    g_err[0] = 0;
    int ndev = 0;
    cudaError_t e0 = cudaGetDeviceCount(&ndev);
    if (e0 != cudaSuccess || ndev == 0) {
        cuda_fail(e0 != cudaSuccess ? e0 : cudaErrorNoDevice, "no CUDA device");
        free_csr(&A);
        return SPEIGS_ERR_INTERNAL;
    }
    speigs_plan_s *p = new (std::nothrow) speigs_plan_s;
    if (!p) { free_csr(&A); return SPEIGS_ERR_MEM; }
    p->A = A;
    A = HostCSR();
    p->which = which;
    p->opts = o;
    p->anorm = anorm;
    p->mf.mixed = (which == SPEIGS_SM && ext && ext->precision == SPEIGS_B200_MIXED);
    if (ext && ext->refine_max > 0) p->refine.max_steps = ext->refine_max;
    if (ext && ext->refine_tol > 0) p->refine_tol_user = ext->refine_tol;
    if (p->stream.err != cudaSuccess) { int rc = cuda_fail(p->stream.err, "stream"); speigs_plan_destroy(p); return rc; }
    cudaStream_t st = p->stream.s;
    const int n = p->A.n;
    const int64_t nnz = p->A.nnz();
    int rc = 0;
    rc = rc ? rc : plan_alloc(p, (void **)&p->d_rp, sizeof(int32_t) * (n + 1));
    rc = rc ? rc : plan_alloc(p, (void **)&p->d_ci, sizeof(int32_t) * nnz);
    rc = rc ? rc : plan_alloc(p, (void **)&p->d_va, sizeof(double) * nnz);
    if (rc) { speigs_plan_destroy(p); return rc; }
    std::vector<int32_t> rp32(n + 1);
    for (int i = 0; i <= n; i++) rp32[i] = (int32_t)p->A.rowptr[i];
    copy_async(p->d_rp, rp32.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, st);
    copy_async(p->d_ci, p->A.col, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st);
    rc = plan_upload_values(p);
    if (rc) { speigs_plan_destroy(p); return rc; }
    if (which == SPEIGS_SM) {
        const double ta = wall();
        spx_symbolic S;
        const int ord = o.ordering == 1 ? SPX_ORDER_MINDEG : o.ordering == 2 ? SPX_ORDER_ND
                                                                            : SPX_ORDER_AUTO;
        int arc = spx_analyze(n, p->A.rowptr, p->A.col, ord, &S);
        if (arc) { speigs_plan_destroy(p); return arc == -2 ? SPEIGS_ERR_MEM : SPEIGS_ERR_FACTOR; }
        rc = p->mf.init(S, p->A.rowptr, p->A.col, st);
        spx_symbolic_free(&S);
        p->t_analyze = wall() - ta;
        if (rc) { speigs_plan_destroy(p); return rc; }
        if (p->mf.mixed) {
            RefineState &rf = p->refine;
            const int nblk = (n + 127) / 128;
            rc = rc ? rc : plan_alloc(p, (void **)&rf.r, sizeof(double) * n);
            rc = rc ? rc : plan_alloc(p, (void **)&rf.d, sizeof(double) * n);
            rc = rc ? rc : plan_alloc(p, (void **)&rf.flag, sizeof(int) * 2);
            rc = rc ? rc : plan_alloc(p, (void **)&rf.count, sizeof(int) * 2);
            rc = rc ? rc : plan_alloc(p, (void **)&rf.rs.part, sizeof(double) * 3 * (size_t)nblk);
            rc = rc ? rc : plan_alloc(p, (void **)&rf.rs.counter, sizeof(unsigned) * 2);
            if (rc) { speigs_plan_destroy(p); return rc; }
            rf.rs.max_blocks = nblk;
            rf.rs.max_cols = 3;
            cudaMemsetAsync(rf.count, 0, sizeof(int) * 2, st);
            cudaMemsetAsync(rf.rs.counter, 0, sizeof(unsigned) * 2, st);
        }
    }
    *out = p;
    return 0;
}

// Numeric factorization with the reference's capped shift escalation
// (src/speigs_core.c:938-970).  Returns 0, SPEIGS_ERR_FACTOR when A stays
// indefinite, or another negative code.
// The indefinite route's operator: A^{-1} formed on the device (the
// reference's UMFPACK LU at sigma = 0, src/speigs_core.c:972-984).
static int plan_dense_inverse(speigs_plan_s *p) {
    cudaStream_t st = p->stream.s;
    const int n = p->A.n;
    if (n > kLuDenseMax) {
        snprintf(g_err, sizeof g_err, "matrix is indefinite and its order %d exceeds the %d of "
                 "the device's dense indefinite route", n, kLuDenseMax);
        return SPEIGS_ERR_FACTOR;
    }
    if (!p->d_ainv) {
        int rc = plan_alloc(p, (void **)&p->d_ainv, sizeof(double) * (size_t)n * n);
        if (rc) return rc;
    }
    Arena ar(st);
    double *rowbuf = ar.alloc<double>(n), *colbuf = ar.alloc<double>(n);
    int *ipiv = ar.alloc<int>(n), *flags = ar.alloc<int>(2);
    if (ar.failed) return SPEIGS_ERR_MEM;
    launch_dense_inverse(n, p->d_rp, p->d_ci, p->d_va, p->anorm, p->d_ainv, rowbuf, colbuf, ipiv,
                         flags, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "dense inverse");
    return 0;
}

static int plan_factor(speigs_plan_s *p, EngineStats *stats) {
    cudaStream_t st = p->stream.s;
    const speigs_opts &o = p->opts;
    double delta = 0.0;
    p->lu = false;
    // A pivot that is rounding noise on the scale of ||A||_1 is treated as
    // not positive, so an exactly singular PSD matrix takes the shift route
    // deterministically instead of by the sign of its last rounding error.
    const double pivtol = 128.0 * (p->mf.mixed ? 1.1920928955078125e-07 : 2.220446049250313e-16) *
                          p->anorm;
    int fr = p->mf.factorize(p->d_va, 0.0, pivtol, st);
    int attempts = 1;
    if (fr == 1) {
        const double d0 = p->anorm * (o.shift0 > 0 ? o.shift0 : 1e-6);
        double dcap = p->anorm * 1e-3;
        if (d0 > dcap) dcap = d0;
        for (delta = d0; delta <= dcap * 1.0000001; delta *= 10.0) {
            fr = p->mf.factorize(p->d_va, delta, pivtol, st);
            attempts++;
            if (fr != 1) break;
        }
        if (fr == 1) delta = 0.0;
    }
    if (stats) {
        stats->factor_attempts = attempts;
        stats->factor_flops = p->mf.factor_flops();
        stats->solve_bytes = p->mf.solve_bytes();
    }
    if (fr < 0) return fr;
    if (fr == 1) {
        // still indefinite: like the reference (:975-984), the Lanczos runs on
        // A^{-1} at sigma = 0, the eigenvalues nearest zero
        int rc = plan_dense_inverse(p);
        if (rc) return rc;
        p->lu = true;
        p->shift = 0.0;
        p->factored = true;
        return 0;
    }
    p->shift = delta;
    p->factored = true;
    return 0;
}

struct Cand2 { double key; int idx; };

// Page-locked host scalars that a solve reads back, one buffer per host
// thread, grown on demand and kept for the thread's life: cudaMallocHost and
// cudaFreeHost are slow and synchronise the device, so they are not paid per
// call (which matters when several threads solve components at once).
// The calling thread's page-locked read-back buffer, released when the
// thread exits (the batched path solves on short-lived worker threads).
struct PinnedScalars {
    double *buf = nullptr;
    size_t cap = 0;
    ~PinnedScalars() {
        if (buf) cudaFreeHost(buf);   // an error at process exit is harmless
    }
};
static double *pinned_scalars(size_t need) {
    thread_local PinnedScalars ps;
    if (ps.cap >= need) return ps.buf;
    size_t want = std::max<size_t>(need, 256);
    double *nb = nullptr;
    if (cudaMallocHost(&nb, sizeof(double) * want) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (ps.buf) cudaFreeHost(ps.buf);
    ps.buf = nb;
    ps.cap = want;
    return ps.buf;
}

// Factor (if 'sm') and iterate; results sorted by |lambda| into host or
// device buffers.
static int plan_solve(speigs_plan_s *p, int64_t k, double *lambda, double *V, double *resid,
                      speigs_info *info, bool on_device, EngineStats *stats) {
    g_err[0] = 0;
    cudaStream_t st = p->stream.s;
    const int n = p->A.n;
    if (k <= 0 || k > n) return SPEIGS_ERR_ARG;
    info->anorm = p->anorm;
    info->ncomp = 0;
    info->t_analyze = p->reuse_factor ? 0.0 : p->t_analyze;
    DevA dA{n, p->d_rp, p->d_ci, p->d_va};
    // the refinement's backward-error target: the caller's, else two orders
    // below the Lanczos tolerance, within [1e-14, 1e-12] -- a solve refined
    // that far perturbs the operator by less than the residual test admits
    {
        const double t = p->opts.tol > 0 ? p->opts.tol : 1e-14;
        p->refine.tol = p->refine_tol_user > 0 ? p->refine_tol_user
                                               : std::min(1e-12, std::max(1e-14, 1e-2 * t));
    }
    SpmvOperator spmv_op(dA);
    CholOperator chol_op(&p->mf);
    MixedCholOperator mixed_op(&p->mf, dA, 0.0, p->anorm, &p->refine);
    DenseInvOperator lu_op(n, nullptr);
    Operator *op = &spmv_op;
    if (p->which == SPEIGS_LM) {
        info->path = SPEIGS_PATH_DIRECT;
    } else {
        const double tf = wall();
        int rc = (p->reuse_factor && p->factored) ? 0 : plan_factor(p, stats);
        info->t_factor = wall() - tf;
        if (rc) return rc;
        mixed_op.shift = p->shift;
        lu_op.M = p->d_ainv;
        op = p->lu ? (Operator *)&lu_op
                   : p->mf.mixed ? (Operator *)&mixed_op : (Operator *)&chol_op;
        info->shift = p->shift;
        info->path = p->lu ? SPEIGS_PATH_LU : p->banded ? SPEIGS_PATH_BANDED
                                                         : SPEIGS_PATH_SHIFTINV;
    }
    std::vector<double> lam_h(k, 0.0), res_h(k, 0.0);
    int rc = 0;
    const size_t need = 4 * (size_t)k + 16;
    double *pinbuf = pinned_scalars(need);
    if (!pinbuf) return SPEIGS_ERR_MEM;
    {
        Arena ar(st);
        const double *X = nullptr;
        int64_t ldx = 0;
        int nout = 0;
        // start subspace (host, n x ext_warm_cols) to the device; like the
        // matrix, it is input staging, so the iteration clock starts once it
        // has landed
        const double *dwarm = nullptr;
        const int64_t wcols = p->ext_warm ? std::min<int64_t>(p->ext_warm_cols, 64) : 0;
        if (wcols > 0) {
            double *dw = ar.alloc<double>((size_t)n * wcols);
            if (ar.failed) return SPEIGS_ERR_MEM;
            // the subspace may be host or device memory (a proposal computed
            // on the device need not go through the host)
            cudaMemcpyKind kind = on_device ? cudaMemcpyDefault : cudaMemcpyHostToDevice;
            cudaPointerAttributes pa{};
            if (cudaPointerGetAttributes(&pa, p->ext_warm) == cudaSuccess &&
                (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged))
                kind = cudaMemcpyDeviceToDevice;
            cudaGetLastError();
            copy_async(dw, p->ext_warm, sizeof(double) * (size_t)n * wcols, kind, st);
            if (cudaError_t e = cudaStreamSynchronize(st)) return cuda_fail(e, "start subspace upload");
            dwarm = dw;
        }
        const double ti = wall();
        int64_t wused = 0;
        // block method ('sm'): explicit block size, or the start subspace's width
        int bsz = 0;
        if (p->which == SPEIGS_SM && !p->lu) {
            if (p->ext_block > 0) bsz = std::min(p->ext_block, kBlockMaxB);
            else if (p->ext_block == 0 && wcols > 0) bsz = (int)std::min<int64_t>(wcols, kBlockMaxB);
            if (bsz > 0) {
                // room for the basis: l + b <= mmax <= n - b (else the single-vector method)
                const int64_t ncv_ref = p->opts.ncv ? p->opts.ncv : std::max<int64_t>(2 * k + 1, 20);
                const int64_t l0 = std::min<int64_t>(k + 5, n);
                int64_t mmax = std::min<int64_t>(std::max<int64_t>(ncv_ref, l0 + 3 * bsz), kBlockMaxM);
                mmax = std::min<int64_t>(mmax, n - bsz);
                if (mmax < l0 + bsz || mmax < k) bsz = 0;
            }
        }
        p->last_block = bsz;
        p->last_block_solves = 0;
        if (bsz > 0) {
            BlockRefineState brf;
            if (p->mf.mixed) {
                brf.ld = ((int64_t)n + 31) & ~(int64_t)31;
                brf.R = ar.alloc<double>((size_t)brf.ld * bsz);
                brf.part = ar.alloc<double>((size_t)3 * kBlockMaxB * ((n + 255) / 256));
                brf.flag = ar.alloc<int>(1);
                brf.count = ar.alloc<int>(1);
                brf.short_word = ar.alloc<int>(1);
                brf.counter = ar.alloc<unsigned>(1);
                if (ar.failed) return SPEIGS_ERR_MEM;
                cudaMemsetAsync(brf.count, 0, sizeof(int), st);
                cudaMemsetAsync(brf.short_word, 0, sizeof(int), st);
                cudaMemsetAsync(brf.counter, 0, sizeof(unsigned), st);
                brf.max_steps = p->refine.max_steps;
                brf.tol = p->refine.tol;
                // two corrections are queued per block solve; a cycle in which
                // one fell short is redone with the full loop
                brf.budget = 2;
            }
            BlockCholOperator bchol(&p->mf);
            BlockMixedOperator bmixed(&p->mf, dA, p->shift, p->anorm, &brf);
            BlockOperator &bop = p->mf.mixed ? (BlockOperator &)bmixed : (BlockOperator &)bchol;
            rc = block_lanczos_device(bop, dA, n, k, bsz, p->opts, p->anorm, p->shift,
                                      lam_h.data(), res_h.data(), &X, &ldx, &nout, info, stats,
                                      ar, pinbuf, st, dwarm, wcols, &wused);
            p->last_warm = wused;
            p->last_ops = bop.nvecs;
            int cnt = 0;
            if (rc == 0 && p->mf.mixed) {
                cudaMemcpyAsync(&cnt, brf.count, sizeof(int), cudaMemcpyDeviceToHost, st);
                note_d2h(sizeof(int));
                cudaStreamSynchronize(st);
            }
            p->last_refine = cnt;
            p->last_block_solves = bop.napps + cnt;
            p->last_t_block_solve = bop.ms_solve_acc * 1e-3;
            p->last_block_solve_calls = bop.solve_calls;
        } else {
        rc = lanczos_device(*op, dA, n, k, p->opts, p->anorm, lam_h.data(), res_h.data(), &X,
                            &ldx, &nout, info, stats, ar, pinbuf, st, dwarm, wcols, &wused);
        p->last_warm = wused;
        p->last_ops = op->nops;
        }
        if (rc == 0 && p->mf.mixed && bsz == 0 && !p->lu) {
            int cnt = 0;
            cudaMemcpyAsync(&cnt, p->refine.count, sizeof(int), cudaMemcpyDeviceToHost, st);
            note_d2h(sizeof(int));
            cudaStreamSynchronize(st);
            p->last_refine = cnt - p->refine_reported;
            p->refine_reported = cnt;
        } else if (bsz == 0) {
            p->last_refine = 0;
        }
        if (rc == 0) {
            // sort by |lambda|: ascending for 'sm', descending for 'lm'
            // (reference :994-1012); entries past nout keep the caller's memory
            std::vector<Cand2> ord(nout);
            for (int i = 0; i < nout; i++) ord[i] = {fabs(lam_h[i]), i};
            std::stable_sort(ord.begin(), ord.end(), [&](const Cand2 &a, const Cand2 &b) {
                return p->which == SPEIGS_SM ? a.key < b.key : a.key > b.key;
            });
            std::vector<double> ls(nout), rs(nout);
            for (int t = 0; t < nout; t++) { ls[t] = lam_h[ord[t].idx]; rs[t] = res_h[ord[t].idx]; }
            const cudaMemcpyKind kv = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
            const cudaMemcpyKind ks = on_device ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost;
            if (V)
                for (int t = 0; t < nout; t++)
                    copy_async(V + (size_t)t * n, X + (size_t)ord[t].idx * ldx,
                                    sizeof(double) * n, kv, st);
            if (on_device) {
                copy_async(lambda, ls.data(), sizeof(double) * nout, ks, st);
                if (resid) copy_async(resid, rs.data(), sizeof(double) * nout, ks, st);
            } else {
                memcpy(lambda, ls.data(), sizeof(double) * nout);
                if (resid) memcpy(resid, rs.data(), sizeof(double) * nout);
            }
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = cuda_fail(e, "copy out");
        }
        info->t_iter = wall() - ti;
    }
    return rc;
}

static void fill_ext_info(const speigs_plan_s *p, speigs_ext_info *e) {
    if (!e) return;
    memset(e, 0, sizeof *e);
    e->precision = p->mf.mixed ? SPEIGS_B200_MIXED : SPEIGS_B200_FP64;
    e->refine_steps = p->last_refine;
    e->factor_solves = p->which == SPEIGS_SM ? p->last_ops + p->last_refine : 0;
    e->warm_cols = p->last_warm;
    e->block = p->last_block;
    e->block_solves = p->last_block_solves;
    e->t_block_solve = p->last_t_block_solve;
    e->block_solve_calls = p->last_block_solve_calls;
    if (p->last_block > 0)
        e->factor_solves = p->which == SPEIGS_SM ? p->last_ops + (int64_t)p->last_refine *
                                                                     p->last_block : 0;
}

// ------------------------------------------------------ factor cache --
// Opt-in, process-wide: the device plans (matrix, symbolic analysis, numeric
// factor) of the last `capacity` distinct operators the Krylov route saw,
// so a parameter sweep or a continuation loop over one matrix skips the
// analysis and the factorization (the reference's planned cache keyed by
// matrix contents).  The key is the full symmetric CSR built from the
// caller's upper triangle, the route ('sm'/'lm'), the factor options
// (ordering, shift0), the precision and the device; a 64-bit hash finds
// candidates and the arrays are then compared in full.  An entry in use by
// one call is not shared with a concurrent one (that call builds its own
// plan).  Least recently used entries are released first.
namespace {

struct CacheEntry {
    uint64_t hash = 0;
    int dev = 0, which = 0, precision = 0, ordering = 0;
    double shift0 = 0.0;
    speigs_plan_s *plan = nullptr;
    bool busy = false;
    uint64_t last_use = 0;
};

struct FactorCache {
    std::mutex mu;
    int capacity = 0;
    uint64_t clock = 0;
    std::vector<CacheEntry> entries;
};

FactorCache &factor_cache() {
    static FactorCache *c = new FactorCache;   // kept for the process's life
    return *c;
}

uint64_t mix64(uint64_t h, uint64_t v) {
    h ^= v + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
    return h;
}

uint64_t csr_hash(const HostCSR &A) {
    uint64_t h = mix64(0, (uint64_t)A.n);
    const int64_t nnz = A.nnz();
    for (int32_t i = 0; i <= A.n; i++) h = mix64(h, (uint64_t)A.rowptr[i]);
    for (int64_t q = 0; q < nnz; q++) {
        uint64_t bits;
        memcpy(&bits, &A.val[q], sizeof bits);
        h = mix64(mix64(h, (uint64_t)(uint32_t)A.col[q]), bits);
    }
    return h;
}

bool same_csr(const HostCSR &a, const HostCSR &b) {
    if (a.n != b.n || a.nnz() != b.nnz()) return false;
    const int64_t nnz = a.nnz();
    return memcmp(a.rowptr, b.rowptr, sizeof(int64_t) * ((size_t)a.n + 1)) == 0 &&
           memcmp(a.col, b.col, sizeof(int32_t) * (size_t)nnz) == 0 &&
           memcmp(a.val, b.val, sizeof(double) * (size_t)nnz) == 0;
}

void evict_over_capacity(FactorCache &fc, std::vector<speigs_plan_s *> &drop) {
    for (;;) {
        int idle = 0;
        for (auto &e : fc.entries) idle += !e.busy;
        if ((int)fc.entries.size() <= fc.capacity || idle == 0) return;
        size_t victim = fc.entries.size();
        for (size_t i = 0; i < fc.entries.size(); i++)
            if (!fc.entries[i].busy &&
                (victim == fc.entries.size() || fc.entries[i].last_use < fc.entries[victim].last_use))
                victim = i;
        drop.push_back(fc.entries[victim].plan);
        fc.entries.erase(fc.entries.begin() + (long)victim);
    }
}

}  // namespace

int device_krylov(HostCSR &A, int64_t k, speigs_which which, const speigs_opts &o,
                  double anorm, double *lambda, double *V, double *resid, speigs_info *info,
                  EngineStats *stats, const speigs_ext_opts *ext, speigs_ext_info *einfo,
                  bool banded) {
    FactorCache &fc = factor_cache();
    int cap = 0;
    {
        std::lock_guard<std::mutex> lk(fc.mu);
        cap = fc.capacity;
    }
    const int precision = (which == SPEIGS_SM && ext && ext->precision == SPEIGS_B200_MIXED)
                              ? SPEIGS_B200_MIXED : SPEIGS_B200_FP64;
    const int dev = current_device();
    uint64_t key = 0;
    speigs_plan_s *p = nullptr;
    if (cap > 0) {
        key = csr_hash(A);
        std::lock_guard<std::mutex> lk(fc.mu);
        for (auto &e : fc.entries)
            if (!e.busy && e.hash == key && e.dev == dev && e.which == (int)which &&
                e.precision == precision && e.ordering == o.ordering && e.shift0 == o.shift0 &&
                same_csr(e.plan->A, A)) {
                e.busy = true;
                e.last_use = ++fc.clock;
                p = e.plan;
                break;
            }
    }
    const double t0 = wall();
    double t_setup = 0.0;
    if (p) {
        // a cache hit: the caller's copy of the matrix is not needed
        free_csr(&A);
        p->opts = o;
        p->anorm = anorm;
        p->reuse_factor = true;
    } else {
        int rc = plan_from_csr(A, which, o, anorm, ext, &p);
        if (rc) return rc;
        t_setup = wall() - t0 - p->t_analyze;
    }
    p->ext_warm = ext ? ext->warm : nullptr;
    p->ext_warm_cols = ext ? ext->warm_cols : 0;
    p->ext_block = ext ? ext->block : 0;
    p->banded = banded;
    int rc = plan_solve(p, k, lambda, V, resid, info, false, stats);
    fill_ext_info(p, einfo);
    const double t1 = wall();
    std::vector<speigs_plan_s *> drop;
    bool keep = false;
    if (cap > 0 && rc == 0 && p->factored) {
        std::lock_guard<std::mutex> lk(fc.mu);
        p->reuse_factor = true;
        bool found = false;
        for (auto &e : fc.entries)
            if (e.plan == p) { e.busy = false; e.last_use = ++fc.clock; found = true; }
        if (!found) {
            CacheEntry e;
            e.hash = key;
            e.dev = dev;
            e.which = (int)which;
            e.precision = precision;
            e.ordering = o.ordering;
            e.shift0 = o.shift0;
            e.plan = p;
            e.last_use = ++fc.clock;
            fc.entries.push_back(e);
        }
        keep = true;
        evict_over_capacity(fc, drop);
    } else if (cap > 0) {
        // a failed solve leaves no entry behind
        std::lock_guard<std::mutex> lk(fc.mu);
        for (size_t i = 0; i < fc.entries.size(); i++)
            if (fc.entries[i].plan == p) {
                fc.entries.erase(fc.entries.begin() + (long)i);
                break;
            }
    }
    if (!keep) speigs_plan_destroy(p);
    for (speigs_plan_s *q : drop) speigs_plan_destroy(q);
    if (einfo) {
        einfo->t_setup = t_setup;
        einfo->t_release = wall() - t1;
    }
    return rc;
}

int factor_cache_configure(int entries) {
    if (entries < 0) return SPEIGS_ERR_ARG;
    FactorCache &fc = factor_cache();
    std::vector<speigs_plan_s *> drop;
    {
        std::lock_guard<std::mutex> lk(fc.mu);
        fc.capacity = entries;
        evict_over_capacity(fc, drop);
    }
    for (speigs_plan_s *q : drop) speigs_plan_destroy(q);
    return SPEIGS_OK;
}

int factor_cache_size() {
    FactorCache &fc = factor_cache();
    std::lock_guard<std::mutex> lk(fc.mu);
    return (int)fc.entries.size();
}

// ---------------------------------------------------- batched Lanczos --
// Many components in lockstep (speigs_batched).  A is the full CSR of the
// components' block-diagonal matrix with component c on rows [off[c],
// off[c+1]); one plan holds the whole forest: one analysis, one
// factorization, and every operator application is one solve (or SpMV) for
// all components.  The step pair (operator, segmented Gram-Schmidt step) is
// captured once into a CUDA graph and replayed; the host reads the
// per-component state once per restart cycle.
int device_batched_krylov(HostCSR &A, int nseg, const int32_t *off_h, int64_t k,
                          speigs_which which, const speigs_opts &o, const double *anorm_h,
                          double *lam_out, double *res_out, double *X_out, int64_t *nconv_out,
                          int64_t *nops_out, int64_t *restarts_out, int *flag_out,
                          BatchedStats *bst, int *handed, int handoff) {
    g_err[0] = 0;
    const int n = A.n;
    if (handed) std::fill(handed, handed + nseg, 0);
    double amax = 1.0;
    for (int c = 0; c < nseg; c++) amax = std::max(amax, anorm_h[c]);
    // per-component basis size by the reference's rules
    int ncv = 0;
    std::vector<int> mh(nseg);
    for (int c = 0; c < nseg; c++) {
        const int64_t nc = off_h[c + 1] - off_h[c];
        int64_t v = o.ncv ? o.ncv : std::max<int64_t>(2 * k + 1, 20);
        if (v > nc) v = nc;
        if (v <= k) v = std::min<int64_t>(nc, k + 1);
        if (v < 2) v = std::min<int64_t>(nc, 2);
        mh[c] = (int)v;
        ncv = std::max(ncv, (int)v);
    }
    if (ncv > syev_small_smem_limit() || ncv > 128) { free_csr(&A); return 1; }
    const std::vector<int> m0 = mh;
    const int64_t maxit = o.maxit ? o.maxit : 300;
    const double tol = o.tol > 0 ? o.tol : 1e-14;
    const double t0 = wall();
    speigs_plan_s *p = nullptr;
    int rc = plan_from_csr(A, which, o, amax, nullptr, &p);
    if (rc) return rc;
    struct PlanGuard {
        speigs_plan_s *p;
        ~PlanGuard() { speigs_plan_destroy(p); }
    } guard{p};
    if (bst) bst->t_analyze = p->t_analyze;
    cudaStream_t st = p->stream.s;
    if (which == SPEIGS_SM) {
        const double tf = wall();
        rc = plan_factor(p, nullptr);
        if (bst) bst->t_factor = wall() - tf;
        if (rc) return rc == SPEIGS_ERR_FACTOR ? 1 : rc;
        // a shifted or indefinite forest goes component by component (each
        // component takes its own shift in the reference)
        if (p->shift != 0.0 || p->lu) return 1;
    }
    const double ti = wall();
    Arena ar(st);
    SegArgs a;
    a.nseg = nseg;
    a.ncv = ncv;
    a.k = (int)k;
    a.l = (int)std::min<int64_t>(k + 5, ncv - 1);
    a.ldv = ((int64_t)n + 31) & ~(int64_t)31;
    int32_t *d_off = ar.alloc<int32_t>(nseg + 1);
    a.off = d_off;
    a.V = ar.alloc<double>((size_t)a.ldv * (ncv + 1));
    a.Vn = ar.alloc<double>((size_t)a.ldv * (ncv + 1));
    a.H = ar.alloc<double>((size_t)nseg * ncv * ncv);
    a.theta = ar.alloc<double>((size_t)nseg * ncv);
    a.S = ar.alloc<double>((size_t)nseg * ncv * ncv);
    a.ord = ar.alloc<int>((size_t)nseg * ncv);
    int *d_jst = ar.alloc<int>((size_t)2 * nseg);
    a.j = ar.alloc<int>(nseg);
    a.m = ar.alloc<int>(nseg);
    a.ext = ar.alloc<int>(nseg);
    a.live = ar.alloc<int>(nseg);
    a.ops = ar.alloc<int>(nseg);
    a.stop = ar.alloc<int>(nseg);
    a.nconv = ar.alloc<int>(nseg);
    a.seed = ar.alloc<uint64_t>(nseg);
    double *d_bthr = ar.alloc<double>(nseg), *d_rtol = ar.alloc<double>(nseg);
    a.bthr = d_bthr;
    a.rtol = d_rtol;
    a.x = ar.alloc<double>(a.ldv);
    a.w = ar.alloc<double>(a.ldv);
    a.X = ar.alloc<double>((size_t)a.ldv * k);
    a.AX = ar.alloc<double>((size_t)a.ldv * k);
    a.lam = ar.alloc<double>((size_t)nseg * k);
    a.r2 = ar.alloc<double>((size_t)nseg * k);
    a.err = ar.alloc<int>(1);
    uint64_t *d_jt = ar.alloc<uint64_t>(64 * 64);
    a.jt = d_jt;
    if (ar.failed) return SPEIGS_ERR_MEM;
    {
        std::vector<double> bt(nseg), rt(nseg);
        for (int c = 0; c < nseg; c++) {
            bt[c] = 1e-13 * std::max(anorm_h[c], 1.0);
            rt[c] = tol * std::max(anorm_h[c], 1.0);
        }
        copy_async(d_off, off_h, sizeof(int32_t) * (nseg + 1), cudaMemcpyHostToDevice, st);
        copy_async(a.m, mh.data(), sizeof(int) * nseg, cudaMemcpyHostToDevice, st);
        copy_async(d_bthr, bt.data(), sizeof(double) * nseg, cudaMemcpyHostToDevice, st);
        copy_async(d_rtol, rt.data(), sizeof(double) * nseg, cudaMemcpyHostToDevice, st);
        copy_async(d_jt, rng_jump_table(), sizeof(uint64_t) * 64 * 64, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(a.err, 0, sizeof(int), st);
        cudaMemsetAsync(a.X, 0, sizeof(double) * (size_t)a.ldv * k, st);
        cudaMemsetAsync(a.x, 0, sizeof(double) * (size_t)a.ldv, st);
        cudaError_t e = cudaStreamSynchronize(st);   // the host vectors die here
        if (e != cudaSuccess) return cuda_fail(e, "batched set-up");
    }
    const uint64_t seed = o.seed ? o.seed : 88172645463325252ULL;
    launch_seg_start(a, seed, st);

    // one step for every component: w = Op x, then the segmented step
    DevA dA{n, p->d_rp, p->d_ci, p->d_va};
    auto issue_step = [&]() {
        if (which == SPEIGS_SM) p->mf.solve(a.x, a.w, st);
        else launch_spmv(n, dA.rp, dA.ci, dA.va, a.x, a.w, st);
        launch_seg_step(a, st);
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    struct GraphGuard {
        cudaGraph_t &g;
        cudaGraphExec_t &x;
        ~GraphGuard() {
            if (x) cudaGraphExecDestroy(x);
            if (g) cudaGraphDestroy(g);
        }
    } gg{graph, gexec};
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        issue_step();
        if (cudaStreamEndCapture(st, &graph) != cudaSuccess ||
            cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess) {
            cudaGetLastError();
            gexec = nullptr;
        }
    } else {
        cudaGetLastError();
    }
    const int *op_err = (which == SPEIGS_SM) ? p->mf.error_word() : nullptr;
    std::vector<int> jh(nseg, 0), liveh(nseg, 1), nconvh(nseg, 0), jsth(2 * nseg);
    std::vector<int64_t> resth(nseg, 0);
    std::vector<double> lamh((size_t)nseg * k, 0.0), r2h((size_t)nseg * k, 0.0);
    std::vector<double> lam_last((size_t)nseg * k, 0.0), r2_last((size_t)nseg * k, 0.0);
    std::vector<int> nwant_last(nseg, 0);
    int herr[2] = {0, 0};
    auto sync_read = [&](const char *where) -> int {
        copy_async(&herr[0], a.err, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (op_err) copy_async(&herr[1], op_err, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, where);
        if (herr[0]) { set_last_error_text("a start vector has zero norm"); return SPEIGS_ERR_INTERNAL; }
        if (herr[1]) {
            set_last_error_text("operator application failed: a solve dependency wait ran out");
            return SPEIGS_ERR_INTERNAL;
        }
        return 0;
    };
    int64_t restarts = 0, steps_total = 0;
    for (;;) {
        int nsteps = 0;
        for (int c = 0; c < nseg; c++)
            if (liveh[c]) nsteps = std::max(nsteps, mh[c] - jh[c]);
        for (int sidx = 0; sidx < nsteps; sidx++) {
            if (gexec) {
                if (cudaGraphLaunch(gexec, st) != cudaSuccess)
                    return cuda_fail(cudaGetLastError(), "batched step");
                note_launch(2);
            } else {
                issue_step();
            }
        }
        steps_total += nsteps;
        // projected eigenproblems, Ritz vectors, true residuals of every live component
        launch_syev_batched(nseg, ncv, a.m, a.H, ncv, (int64_t)ncv * ncv, a.theta, a.S, a.ord,
                            d_jst, a.live, st);
        launch_seg_ritz(a, st);
        for (int64_t t = 0; t < k; t++)
            launch_spmv(n, dA.rp, dA.ci, dA.va, a.X + (size_t)t * a.ldv, a.AX + (size_t)t * a.ldv,
                        st);
        launch_seg_resid(a, st);
        copy_async(nconvh.data(), a.nconv, sizeof(int) * nseg, cudaMemcpyDeviceToHost, st);
        copy_async(mh.data(), a.m, sizeof(int) * nseg, cudaMemcpyDeviceToHost, st);
        copy_async(jsth.data(), d_jst, sizeof(int) * 2 * nseg, cudaMemcpyDeviceToHost, st);
        copy_async(lamh.data(), a.lam, sizeof(double) * nseg * k, cudaMemcpyDeviceToHost, st);
        copy_async(r2h.data(), a.r2, sizeof(double) * nseg * k, cudaMemcpyDeviceToHost, st);
        if (int e = sync_read("batched check")) return e;
        int nlive = 0;
        for (int c = 0; c < nseg; c++) {
            if (!liveh[c]) continue;
            if (jsth[2 * c] < 0) return SPEIGS_ERR_LAPACK;
            const int nw = (int)std::min<int64_t>(k, mh[c]);
            nwant_last[c] = nw;
            for (int t = 0; t < nw; t++) {
                lam_last[(size_t)c * k + t] = lamh[(size_t)c * k + t];
                r2_last[(size_t)c * k + t] = r2h[(size_t)c * k + t];
            }
            // the reference stops at convergence, at maxit, or when the basis
            // ended early (m < ncv)
            const bool done = nconvh[c] >= nw || restarts >= maxit || mh[c] < m0[c];
            if (done) liveh[c] = 0;
            else nlive++;
        }
        if (nlive == 0) break;
        if (handed && handoff > 0) {
            int64_t live_rows = 0;
            for (int c = 0; c < nseg; c++)
                if (liveh[c]) live_rows += off_h[c + 1] - off_h[c];
            if ((int64_t)handoff * live_rows <= (int64_t)n) {
                for (int c = 0; c < nseg; c++)
                    if (liveh[c]) {
                        handed[c] = 1;
                        liveh[c] = 0;
                    }
                if (bst) bst->handed = nlive;
                break;
            }
        }
        restarts++;
        for (int c = 0; c < nseg; c++)
            if (liveh[c]) resth[c]++;
        copy_async(a.live, liveh.data(), sizeof(int) * nseg, cudaMemcpyHostToDevice, st);
        launch_seg_restart(a, st);
        copy_async(jh.data(), a.j, sizeof(int) * nseg, cudaMemcpyDeviceToHost, st);
        copy_async(liveh.data(), a.live, sizeof(int) * nseg, cudaMemcpyDeviceToHost, st);
        if (int e = sync_read("batched restart")) return e;
        bool any = false;
        for (int c = 0; c < nseg; c++) any |= liveh[c] != 0;
        if (!any) break;
    }
    // results in Lanczos order, as the reference leaves them; the caller sorts
    std::vector<int> opsh(nseg);
    copy_async(opsh.data(), a.ops, sizeof(int) * nseg, cudaMemcpyDeviceToHost, st);
    if (X_out)
        for (int64_t t = 0; t < k; t++)
            copy_async(X_out + (size_t)t * n, a.X + (size_t)t * a.ldv, sizeof(double) * n,
                       cudaMemcpyDeviceToHost, st);
    if (int e = sync_read("batched results")) return e;
    for (int c = 0; c < nseg; c++) {
        const int nw = nwant_last[c];
        int conv = 0;
        for (int t = 0; t < k; t++) {
            const double r = t < nw ? std::sqrt(r2_last[(size_t)c * k + t]) : 0.0;
            lam_out[(size_t)c * k + t] = t < nw ? lam_last[(size_t)c * k + t] : 0.0;
            if (res_out) res_out[(size_t)c * k + t] = r;
            if (t < nw && r <= tol * std::max(anorm_h[c], 1.0)) conv++;
        }
        nconv_out[c] = conv;
        nops_out[c] = opsh[c];
        restarts_out[c] = resth[c];
        flag_out[c] = conv >= nw ? 0 : 1;
    }
    if (bst) {
        bst->t_iter = wall() - ti;
        bst->steps = steps_total;
        bst->cycles = restarts + 1;
        bst->graph = gexec != nullptr;
        bst->t_total = wall() - t0;
    }
    return SPEIGS_OK;
}

// -------------------------------------------------- Hermitian recovery --
__global__ void times_i_kernel(int n, const double *w, double *dst) {
    // dst = i w in the real embedding: [x; y] -> [-y; x]
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        dst[i] = -w[n + i];
        dst[n + i] = w[i];
    }
}

int device_hermitian_recover(int64_t n64, int64_t kk, int64_t k, const double *V2,
                             const double *lam2, const double *res2, double *lambda, double *Vr,
                             double *Vi, double *resid, int64_t *nacc_out) {
    g_err[0] = 0;
    if (2 * n64 > INT32_MAX) return SPEIGS_ERR_ARG;
    const int n = (int)n64, n2 = 2 * n;
    Stream stream;
    if (stream.err != cudaSuccess) return cuda_fail(stream.err, "stream");
    cudaStream_t st = stream.s;
    int64_t nacc = 0;
    std::vector<int64_t> src;   // candidate column behind each accepted vector
    {
        Arena ar(st);
        const int64_t ldq = ((int64_t)n2 + 31) & ~(int64_t)31;
        double *C = ar.alloc<double>((size_t)n2 * kk);           // the candidates
        double *Q = ar.alloc<double>((size_t)ldq * 2 * k);       // accepted u, i u pairs
        double *w = ar.alloc<double>(ldq);
        double *h1 = ar.alloc<double>(2 * k + 1), *h2 = ar.alloc<double>(2 * k + 1);
        double *nrm2 = ar.alloc<double>(4);
        const int nblk = (n2 + 511) / 512 + 1;
        ReduceScratch rs;
        rs.part = ar.alloc<double>((size_t)nblk * (2 * k + 2));
        rs.counter = ar.alloc<unsigned>(1);
        rs.max_blocks = nblk;
        rs.max_cols = (int)(2 * k + 2);
        double *hn = pinned_scalars(16);
        if (ar.failed || !hn) return SPEIGS_ERR_MEM;
        cudaMemsetAsync(rs.counter, 0, sizeof(unsigned), st);
        copy_async(C, V2, sizeof(double) * (size_t)n2 * kk, cudaMemcpyHostToDevice, st);
        auto read_nrm = [&](double *out) -> int {
            copy_async(hn, nrm2, sizeof(double), cudaMemcpyDeviceToHost, st);
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cuda_fail(e, "hermitian recovery");
            *out = std::sqrt(hn[0]);
            return 0;
        };
        for (int64_t c = 0; c < kk && nacc < k; c++) {
            // the candidate [a; b] as a unit complex vector a + i b
            launch_copy(n2, C + (size_t)c * n2, w, st);
            launch_ts_norm(n2, w, nrm2, rs, st);
            double nr = 0.0;
            if (int e = read_nrm(&nr)) return e;
            if (!(nr > 0.0)) continue;
            launch_scale_by_invnorm(n2, w, nrm2, w, st);
            // complex Gram-Schmidt against the accepted u = real Gram-Schmidt
            // against u and i u, twice
            const int m = (int)(2 * nacc);
            if (m > 0) {
                launch_ts_dot(Q, ldq, n2, m, w, h1, nullptr, 0, rs, st);
                launch_ts_update_dot(Q, ldq, n2, m, w, h1, h2, nullptr, 0, rs, st);
                launch_ts_update_norm(Q, ldq, n2, m, w, h2, nrm2, rs, st);
            } else {
                launch_ts_norm(n2, w, nrm2, rs, st);
            }
            double wn = 0.0;
            if (int e = read_nrm(&wn)) return e;
            if (wn <= 0.1) continue;   // a complex multiple of an accepted vector
            double *u = Q + (size_t)(2 * nacc) * ldq;
            launch_scale_by_invnorm(n2, w, nrm2, u, st);
            times_i_kernel<<<std::max(1, std::min(1024, (n + 255) / 256)), 256, 0, st>>>(
                n, u, u + ldq);
            note_launch();
            src.push_back(c);
            nacc++;
        }
        for (int64_t a = 0; a < nacc; a++) {
            const double *u = Q + (size_t)(2 * a) * ldq;
            if (Vr) copy_async(Vr + (size_t)a * n, u, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
            if (Vi) copy_async(Vi + (size_t)a * n, u + n, sizeof(double) * n,
                               cudaMemcpyDeviceToHost, st);
        }
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "hermitian recovery");
    }
    for (int64_t a = 0; a < nacc; a++) {
        lambda[a] = lam2[src[a]];
        if (resid) resid[a] = res2[src[a]];
    }
    if (Vr) memset(Vr + (size_t)nacc * n, 0, sizeof(double) * (size_t)(k - nacc) * n);
    if (Vi) memset(Vi + (size_t)nacc * n, 0, sizeof(double) * (size_t)(k - nacc) * n);
    *nacc_out = nacc;
    return SPEIGS_OK;
}

// ------------------------------------------------------------ diag path --
__global__ void absbits_kernel(int n, const double *d, unsigned long long *key, int *idx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        key[i] = (unsigned long long)__double_as_longlong(fabs(d[i]));
        idx[i] = i;
    }
}

int device_diag_path(int64_t n64, const double *diag, int64_t k, speigs_which which,
                     double *lambda, double *V, double *resid, speigs_info *info) {
    g_err[0] = 0;
    if (n64 > INT32_MAX) return SPEIGS_ERR_ARG;
    const int n = (int)n64;
    Stream stream;
    if (stream.err != cudaSuccess) return cuda_fail(stream.err, "stream");
    cudaStream_t st = stream.s;
    std::vector<int> ord(k);
    {
        Arena ar(st);
        double *d = ar.alloc<double>(n);
        unsigned long long *k0 = ar.alloc<unsigned long long>(n), *k1 = ar.alloc<unsigned long long>(n);
        int *i0 = ar.alloc<int>(n), *i1 = ar.alloc<int>(n);
        if (ar.failed) return SPEIGS_ERR_MEM;
        copy_async(d, diag, sizeof(double) * n, cudaMemcpyHostToDevice, st);
        absbits_kernel<<<std::min(1024, (n + 255) / 256), 256, 0, st>>>(n, d, k0, i0);
        note_launch();
        size_t tb = 0;
        if (which == SPEIGS_SM)
            cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, i0, i1, n, 0, 64, st);
        else
            cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, k0, k1, i0, i1, n, 0, 64, st);
        void *tmp = ar.alloc<char>(tb);
        if (ar.failed) return SPEIGS_ERR_MEM;
        if (which == SPEIGS_SM)
            cub::DeviceRadixSort::SortPairs(tmp, tb, k0, k1, i0, i1, n, 0, 64, st);
        else
            cub::DeviceRadixSort::SortPairsDescending(tmp, tb, k0, k1, i0, i1, n, 0, 64, st);
        copy_async(ord.data(), i1, sizeof(int) * k, cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "diag sort");
    }
    for (int64_t t = 0; t < k; t++) {
        const int i = ord[t];
        lambda[t] = diag[i];
        if (V) { memset(V + (size_t)t * n, 0, (size_t)n * sizeof(double)); V[(size_t)t * n + i] = 1.0; }
        if (resid) resid[t] = 0.0;
    }
    info->nconv = k;
    info->flag = 0;
    info->path = SPEIGS_PATH_DIAG;
    return SPEIGS_OK;
}

// ----------------------------------------------------------- dense path --
__global__ void densify_kernel(int n, const int32_t *rp, const int32_t *ci, const double *va,
                               double *D) {
    for (int r = blockIdx.x; r < n; r += gridDim.x)
        for (int q = rp[r] + threadIdx.x; q < rp[r + 1]; q += blockDim.x)
            D[(size_t)r + (size_t)ci[q] * n] = va[q];
}

int device_dense_path(const HostCSR &A, int64_t k, speigs_which which, double *lambda,
                      double *V, double *resid, speigs_info *info) {
    g_err[0] = 0;
    const int n = A.n;
    const int64_t nnz = A.nnz();
    Stream stream;
    if (stream.err != cudaSuccess) return cuda_fail(stream.err, "stream");
    cudaStream_t st = stream.s;
    std::vector<double> theta(n);
    std::vector<int> ordd(n);
    std::vector<int32_t> rp32(n + 1);
    for (int i = 0; i <= n; i++) rp32[i] = (int32_t)A.rowptr[i];
    {
        Arena ar(st);
        int32_t *d_rp = ar.alloc<int32_t>(n + 1);
        int32_t *d_ci = ar.alloc<int32_t>(nnz);
        double *d_va = ar.alloc<double>(nnz);
        double *D = ar.alloc<double>((size_t)n * n);
        double *th = ar.alloc<double>(n);
        double *S = ar.alloc<double>((size_t)n * n);
        int *od = ar.alloc<int>(n);
        int *stt = ar.alloc<int>(2);
        const int me = (n + 1) & ~1;
        double *work = (n > syev_small_smem_limit()) ? ar.alloc<double>((size_t)2 * me * me) : nullptr;
        if (ar.failed) return SPEIGS_ERR_MEM;
        copy_async(d_rp, rp32.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, st);
        copy_async(d_ci, A.col, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st);
        copy_async(d_va, A.val, sizeof(double) * nnz, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(D, 0, sizeof(double) * n * n, st);
        densify_kernel<<<std::min(n, 4096), 32, 0, st>>>(n, d_rp, d_ci, d_va, D);
        note_launch();
        launch_syev_small(n, D, n, th, S, od, work, stt, st);
        int hst[2] = {0, 0};
        copy_async(theta.data(), th, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
        copy_async(hst, stt, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "dense path");
        if (hst[0] < 0) return SPEIGS_ERR_LAPACK;
        // order by |theta| ascending ('sm') or descending ('lm'), stable
        for (int i = 0; i < n; i++) ordd[i] = i;
        std::stable_sort(ordd.begin(), ordd.end(), [&](int a, int b) {
            return which == SPEIGS_SM ? fabs(theta[a]) < fabs(theta[b])
                                      : fabs(theta[a]) > fabs(theta[b]);
        });
        if (V)
            for (int64_t t = 0; t < k; t++)
                copy_async(V + (size_t)t * n, S + (size_t)ordd[t] * n, sizeof(double) * n,
                                cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "dense path copy");
    }
    for (int64_t t = 0; t < k; t++) {
        lambda[t] = theta[ordd[t]];
        if (resid) resid[t] = 0.0;
    }
    info->nconv = k;
    info->flag = 0;
    info->path = SPEIGS_PATH_DENSE;
    return SPEIGS_OK;
}

}  // namespace spx

// ================================================================ C API ==
using spx::HostCSR;

extern "C" {

int speigs_plan_create(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                       const double *Ax, speigs_which which, const speigs_opts *opts,
                       speigs_plan *plan) {
    return speigs_plan_create_ex(n, Ap, Ai, Ax, which, opts, nullptr, plan);
}

void speigs_default_ext_opts(speigs_ext_opts *e) {
    if (!e) return;
    memset(e, 0, sizeof *e);
    e->precision = SPEIGS_B200_FP64;
}

int speigs_plan_ext_info(speigs_plan p, speigs_ext_info *e) {
    if (!p || !e) return SPEIGS_ERR_ARG;
    spx::fill_ext_info(p, e);
    return SPEIGS_OK;
}

int speigs_plan_create_ex(speigs_int n, const speigs_int *Ap, const speigs_int *Ai,
                          const double *Ax, speigs_which which, const speigs_opts *opts,
                          const speigs_ext_opts *ext, speigs_plan *plan) {
    if (!plan) return SPEIGS_ERR_ARG;
    *plan = nullptr;
    speigs_opts defo;
    if (!opts) { speigs_default_opts(&defo); opts = &defo; }
    if (n <= 0 || !Ap || !Ai || !Ax) return SPEIGS_ERR_ARG;
    if (opts->check_sym != 0 && spx::host_check_symmetry(n, Ap, Ai, Ax) == 0)
        return SPEIGS_ERR_NOTSYM;
    double anorm = spx::host_norm1_upper(n, Ap, Ai, Ax);
    if (anorm <= 0) anorm = 1.0;
    HostCSR A;
    int rc = spx::build_full_csr(n, Ap, Ai, Ax, &A);
    if (rc) return rc;
    speigs_plan_s *p = nullptr;
    rc = spx::plan_from_csr(A, which, *opts, anorm, ext, &p);
    if (rc) return rc;
    p->Ap_copy.assign(Ap, Ap + n + 1);
    p->Ai_copy.assign(Ai, Ai + Ap[n]);
    p->ext_warm = ext ? ext->warm : nullptr;
    p->ext_warm_cols = ext ? ext->warm_cols : 0;
    p->ext_block = ext ? ext->block : 0;
    *plan = p;
    return SPEIGS_OK;
}

int speigs_plan_set_values(speigs_plan p, const double *Ax) {
    if (!p || !Ax) return SPEIGS_ERR_ARG;
    const int64_t n = p->A.n;
    HostCSR B;
    int rc = spx::build_full_csr(n, p->Ap_copy.data(), p->Ai_copy.data(), Ax, &B);
    if (rc) return rc;
    std::swap(p->A.val, B.val);
    spx::free_csr(&B);
    double anorm = spx::host_norm1_upper(n, p->Ap_copy.data(), p->Ai_copy.data(), Ax);
    p->anorm = anorm > 0 ? anorm : 1.0;
    return spx::plan_upload_values(p);
}

int speigs_plan_solve_device(speigs_plan p, speigs_int k, double *lambda, double *V,
                             double *resid, speigs_info *info) {
    if (!p || !lambda) return SPEIGS_ERR_ARG;
    speigs_info li;
    if (!info) info = &li;
    memset(info, 0, sizeof *info);
    return spx::plan_solve(p, k, lambda, V, resid, info, true, nullptr);
}

int speigs_plan_factor(speigs_plan p, double *shift) {
    if (!p) return SPEIGS_ERR_ARG;
    if (p->which != SPEIGS_SM) return SPEIGS_ERR_ARG;
    int rc = spx::plan_factor(p, nullptr);
    if (shift) *shift = p->shift;
    return rc;
}

int speigs_plan_apply_device(speigs_plan p, const double *x, double *y) {
    if (!p || !x || !y) return SPEIGS_ERR_ARG;
    cudaStream_t st = p->stream.s;
    if (p->which == SPEIGS_LM) {
        spx::launch_spmv(p->A.n, p->d_rp, p->d_ci, p->d_va, x, y, st);
    } else {
        if (!p->factored) {
            int rc = spx::plan_factor(p, nullptr);
            if (rc) return rc;
        }
        if (p->lu) {
            spx::launch_dense_apply(p->A.n, p->d_ainv, x, y, st);
        } else if (p->mf.mixed) {
            spx::DevA dA{p->A.n, p->d_rp, p->d_ci, p->d_va};
            spx::MixedCholOperator op(&p->mf, dA, p->shift, p->anorm, &p->refine);
            op.apply(x, y, st);
        } else {
            p->mf.solve(x, y, st);
        }
    }
    int herr = 0;
    if (p->which == SPEIGS_SM && !p->lu && p->mf.error_word())
        cudaMemcpyAsync(&herr, p->mf.error_word(), sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return spx::cuda_fail(e, "apply");
    if (herr) {
        spx::set_last_error_text("solve failed: a dependency wait ran out");
        return SPEIGS_ERR_INTERNAL;
    }
    return SPEIGS_OK;
}

int speigs_plan_apply_block_device(speigs_plan p, const double *x, int64_t ldx, double *y,
                                   int64_t ldy, int nr) {
    if (!p || !x || !y || nr < 1 || nr > spx::kBlockMaxB || ldx < p->A.n || ldy < p->A.n)
        return SPEIGS_ERR_ARG;
    cudaStream_t st = p->stream.s;
    const int n = p->A.n;
    int rc = 0;
    if (p->which == SPEIGS_LM) {
        for (int c = 0; c < nr; c++)
            spx::launch_spmv(n, p->d_rp, p->d_ci, p->d_va, x + (size_t)c * ldx, y + (size_t)c * ldy,
                             st);
    } else {
        if (!p->factored) {
            rc = spx::plan_factor(p, nullptr);
            if (rc) return rc;
        }
        if (p->lu) {
            for (int c = 0; c < nr; c++)
                spx::launch_dense_apply(n, p->d_ainv, x + (size_t)c * ldx, y + (size_t)c * ldy, st);
        } else if (p->mf.mixed) {
            spx::Arena ar(st);
            spx::BlockRefineState brf;
            brf.ld = ((int64_t)n + 31) & ~(int64_t)31;
            brf.R = ar.alloc<double>((size_t)brf.ld * nr);
            brf.part = ar.alloc<double>((size_t)3 * spx::kBlockMaxB * ((n + 255) / 256));
            brf.flag = ar.alloc<int>(1);
            brf.count = ar.alloc<int>(1);
            brf.counter = ar.alloc<unsigned>(1);
            if (ar.failed) return SPEIGS_ERR_MEM;
            cudaMemsetAsync(brf.count, 0, sizeof(int), st);
            cudaMemsetAsync(brf.counter, 0, sizeof(unsigned), st);
            brf.max_steps = p->refine.max_steps;
            brf.tol = p->refine.tol;
            spx::DevA dA{n, p->d_rp, p->d_ci, p->d_va};
            spx::BlockMixedOperator op(&p->mf, dA, p->shift, p->anorm, &brf);
            rc = op.apply(x, ldx, y, ldy, nr, st);
            cudaError_t e = cudaStreamSynchronize(st);   // before the arena returns its memory
            if (!rc && e != cudaSuccess) rc = spx::cuda_fail(e, "apply block");
        } else {
            rc = p->mf.solve_block(x, ldx, y, ldy, nr, st);
        }
        if (rc) return rc;
    }
    int herr = 0;
    if (p->which == SPEIGS_SM && !p->lu && p->mf.error_word())
        cudaMemcpyAsync(&herr, p->mf.error_word(), sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return spx::cuda_fail(e, "apply block");
    if (herr) {
        spx::set_last_error_text("solve failed: a dependency wait ran out");
        return SPEIGS_ERR_INTERNAL;
    }
    return SPEIGS_OK;
}

void *speigs_plan_stream(speigs_plan p) { return p ? (void *)p->stream.s : nullptr; }

int speigs_plan_costs(speigs_plan p, double *op_bytes, double *factor_flops, double *nnz_factor) {
    if (!p) return SPEIGS_ERR_ARG;
    const double n = p->A.n, nnz = (double)p->A.nnz();
    if (p->which == SPEIGS_LM) {
        if (op_bytes) *op_bytes = 12.0 * nnz + 4.0 * (n + 1) + 16.0 * n;
        if (factor_flops) *factor_flops = 0;
        if (nnz_factor) *nnz_factor = 0;
    } else {
        if (op_bytes) *op_bytes = (double)p->mf.solve_bytes();
        if (factor_flops) *factor_flops = p->mf.factor_flops();
        if (nnz_factor) *nnz_factor = (double)p->mf.panel_entries();
    }
    return SPEIGS_OK;
}

void speigs_plan_destroy(speigs_plan p) {
    if (!p) return;
    cudaStream_t st = p->stream.s;
    p->mf.release(st);
    for (void *q : p->owned) cudaFreeAsync(q, st);
    p->owned.clear();
    cudaStreamSynchronize(st);
    spx::free_csr(&p->A);
    delete p;
}

int speigs_b200_rand_vec(speigs_int n, uint64_t seed, double *v) {
    if (n <= 0 || n > INT32_MAX || !v) return SPEIGS_ERR_ARG;
    spx::Stream s;
    if (s.err != cudaSuccess) return spx::cuda_fail(s.err, "stream");
    double *d = nullptr;
    if (cudaMallocAsync(&d, sizeof(double) * n, s.s) != cudaSuccess) {
        cudaGetLastError();
        return SPEIGS_ERR_MEM;
    }
    spx::launch_rand_vec((int)n, seed, d, s.s);
    spx::copy_async(v, d, sizeof(double) * n, cudaMemcpyDeviceToHost, s.s);
    cudaFreeAsync(d, s.s);
    cudaError_t e = cudaStreamSynchronize(s.s);
    return e == cudaSuccess ? SPEIGS_OK : spx::cuda_fail(e, "rand_vec");
}

int speigs_b200_syev_small(int m, const double *H, double *theta, double *S, int *ord) {
    if (m <= 0 || !H || !theta || !S || !ord) return SPEIGS_ERR_ARG;
    spx::Stream s;
    if (s.err != cudaSuccess) return spx::cuda_fail(s.err, "stream");
    const size_t mm = (size_t)m * m, me = (size_t)((m + 1) & ~1);
    double *dH = nullptr, *dth = nullptr, *dS = nullptr, *dw = nullptr;
    int *dord = nullptr, *dst = nullptr;
    int rc = 0;
    if (cudaMallocAsync(&dH, sizeof(double) * mm, s.s) || cudaMallocAsync(&dth, sizeof(double) * m, s.s) ||
        cudaMallocAsync(&dS, sizeof(double) * mm, s.s) || cudaMallocAsync(&dw, sizeof(double) * 2 * me * me, s.s) ||
        cudaMallocAsync(&dord, sizeof(int) * m, s.s) || cudaMallocAsync(&dst, sizeof(int) * 2, s.s)) {
        cudaGetLastError();
        rc = SPEIGS_ERR_MEM;
    }
    int hst[2] = {0, 0};
    if (!rc) {
        spx::copy_async(dH, H, sizeof(double) * mm, cudaMemcpyHostToDevice, s.s);
        spx::launch_syev_small(m, dH, m, dth, dS, dord, dw, dst, s.s);
        spx::copy_async(theta, dth, sizeof(double) * m, cudaMemcpyDeviceToHost, s.s);
        spx::copy_async(S, dS, sizeof(double) * mm, cudaMemcpyDeviceToHost, s.s);
        spx::copy_async(ord, dord, sizeof(int) * m, cudaMemcpyDeviceToHost, s.s);
        spx::copy_async(hst, dst, sizeof(int), cudaMemcpyDeviceToHost, s.s);
    }
    void *ptrs[] = {dH, dth, dS, dw, dord, dst};
    for (void *q : ptrs) if (q) cudaFreeAsync(q, s.s);
    cudaError_t e = cudaStreamSynchronize(s.s);
    if (e != cudaSuccess) return spx::cuda_fail(e, "syev_small");
    if (!rc && hst[0] < 0) rc = SPEIGS_ERR_LAPACK;
    return rc;
}

int speigs_b200_factor_cache(int entries) { return spx::factor_cache_configure(entries); }

int speigs_b200_factor_cache_size(void) { return spx::factor_cache_size(); }

const char *speigs_b200_last_error(void) { return spx::last_cuda_error(); }

void speigs_b200_counters(long long *launches, long long *h2d_bytes, long long *d2h_bytes) {
    spx::Counters &c = spx::counters();
    if (launches) *launches = c.launches.load(std::memory_order_relaxed);
    if (h2d_bytes) *h2d_bytes = c.h2d.load(std::memory_order_relaxed);
    if (d2h_bytes) *d2h_bytes = c.d2h.load(std::memory_order_relaxed);
}

}  // extern "C"
