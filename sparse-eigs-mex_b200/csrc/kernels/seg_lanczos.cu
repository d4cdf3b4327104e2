// Segmented thick-restart Lanczos kernels (seg_lanczos.cuh): one thread
// block per component, every vector operation of the reference's lanczos()
// (src/speigs_core.c:146-315) restricted to the component's row segment.
#include "seg_lanczos.cuh"
#include "../common.cuh"
#include "../counters.h"

namespace spx {

namespace {

constexpr int kSegThreads = 256;

// xorshift64* state after `steps` draws (the jump table holds M^(2^b))
SPX_DEV uint64_t rng_jump(uint64_t s, uint64_t steps, const uint64_t *jt) {
    for (int b = 0; steps; b++, steps >>= 1) {
        if (!(steps & 1ull)) continue;
        const uint64_t *col = jt + (size_t)b * 64;
        uint64_t y = 0;
        for (int q = 0; q < 64; q++) y ^= col[q] & (0ull - ((s >> q) & 1ull));
        s = y;
    }
    return s;
}

// dst[i] = draw i + 1 of the stream from `seed`, U[-0.5, 0.5) (reference
// rand_vec, :52-54); each thread jumps to its own run of 64 draws
SPX_DEV void seg_rand(double *dst, int nr, uint64_t seed, const uint64_t *jt) {
    for (int first = threadIdx.x * 64; first < nr; first += blockDim.x * 64) {
        uint64_t s = rng_jump(seed, (uint64_t)first, jt);
        const int last = min(nr, first + 64);
        for (int i = first; i < last; i++) {
            s ^= s >> 12; s ^= s << 25; s ^= s >> 27;
            const uint64_t out = s * 0x2545F4914F6CDD1DULL;
            dst[i] = (double)(out >> 11) / 9007199254740992.0 - 0.5;
        }
    }
    __syncthreads();
}

// h[0:nc) = V[:, 0:nc]^T w over the segment's nr rows, eight columns at a time
SPX_DEV void seg_dots(const double *V, int64_t ldv, int nr, int nc, const double *w, double *h,
                      double *red) {
    for (int c0 = 0; c0 < nc; c0 += 8) {
        double p[8];
#pragma unroll
        for (int q = 0; q < 8; q++) p[q] = 0.0;
        for (int r = threadIdx.x; r < nr; r += blockDim.x) {
            const double wr = w[r];
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (c0 + q < nc) p[q] += V[r + (int64_t)(c0 + q) * ldv] * wr;
        }
        const double t = block_sum8(p, red);
        if (threadIdx.x < 8 && c0 + (int)threadIdx.x < nc) h[c0 + threadIdx.x] = t;
        __syncthreads();
    }
}

// w -= V[:, 0:nc] h
SPX_DEV void seg_update(const double *V, int64_t ldv, int nr, int nc, const double *h, double *w) {
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < nc; i++) s += V[r + (int64_t)i * ldv] * h[i];
        w[r] -= s;
    }
    __syncthreads();
}

SPX_DEV double seg_norm2(const double *w, int nr, double *red) {
    double s = 0.0;
    for (int r = threadIdx.x; r < nr; r += blockDim.x) s += w[r] * w[r];
    return block_sum(s, red);
}

// w <- (I - V V^T) w twice against nc columns (reference orth_block); h1 and
// h2 keep the two passes' coefficients; returns ||w||^2
SPX_DEV double seg_cgs2(const double *V, int64_t ldv, int nr, int nc, double *w, double *h1,
                        double *h2, double *red) {
    if (nc > 0) {
        seg_dots(V, ldv, nr, nc, w, h1, red);
        seg_update(V, ldv, nr, nc, h1, w);
        seg_dots(V, ldv, nr, nc, w, h2, red);
        seg_update(V, ldv, nr, nc, h2, w);
    }
    return seg_norm2(w, nr, red);
}

// shared memory: h1, h2, thsave [ncv + 1] each, reduction scratch
struct SegSmem {
    double *h1, *h2, *ths, *red;
};
SPX_DEV SegSmem seg_smem(double *sh, int ncv) {
    SegSmem s;
    s.h1 = sh;
    s.h2 = sh + (ncv + 1);
    s.ths = sh + 2 * (ncv + 1);
    s.red = sh + 3 * (ncv + 1);
    return s;
}

__global__ void __launch_bounds__(kSegThreads) seg_start_kernel(SegArgs a, uint64_t seed) {
    extern __shared__ double sh[];
    const SegSmem sm = seg_smem(sh, a.ncv);
    const int c = blockIdx.x;
    const int o = a.off[c], nr = a.off[c + 1] - o;
    double *v0 = a.V + o;
    seg_rand(v0, nr, seed, a.jt);
    const double n2 = seg_norm2(v0, nr, sm.red);
    double *H = a.H + (size_t)c * a.ncv * a.ncv;
    for (int e = threadIdx.x; e < a.ncv * a.ncv; e += blockDim.x) H[e] = 0.0;
    if (n2 == 0.0) {
        if (threadIdx.x == 0) {
            atomicExch(a.err, 1);
            a.live[c] = 0;
            a.ext[c] = 0;
        }
        return;
    }
    const double s = 1.0 / sqrt(n2);
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        const double v = v0[r] * s;
        v0[r] = v;
        a.x[o + r] = v;
    }
    if (threadIdx.x == 0) {
        a.seed[c] = rng_jump(seed, (uint64_t)nr, a.jt);
        a.j[c] = 0;
        a.ext[c] = 1;
        a.live[c] = 1;
        a.ops[c] = 0;
        a.stop[c] = 0;
    }
}

// one step of the extension loop (reference :197-229) after w = Op x
__global__ void __launch_bounds__(kSegThreads) seg_step_kernel(SegArgs a) {
    extern __shared__ double sh[];
    __shared__ uint64_t s_seed;
    const int c = blockIdx.x;
    if (!a.ext[c]) return;
    const SegSmem sm = seg_smem(sh, a.ncv);
    const int o = a.off[c], nr = a.off[c + 1] - o;
    const int jj = a.j[c], m = a.m[c];
    const double *V = a.V + o;
    double *w = a.w + o;
    double *H = a.H + (size_t)c * a.ncv * a.ncv;
    double beta = sqrt(seg_cgs2(V, a.ldv, nr, jj + 1, w, sm.h1, sm.h2, sm.red));
    // the projected-matrix column: both passes' coefficients
    for (int i = threadIdx.x; i <= jj; i += blockDim.x)
        H[i + (int64_t)jj * a.ncv] = sm.h1[i] + sm.h2[i];
    double brec = beta;
    const double thr = a.bthr[c];
    bool dead = false;
    if (beta <= thr) {
        // invariant subspace: fresh vectors from the component's stream
        brec = 0.0;
        if (threadIdx.x == 0) s_seed = a.seed[c];
        __syncthreads();
        for (int att = 0; att < 3 && beta <= thr; att++) {
            const uint64_t sd = s_seed;
            seg_rand(w, nr, sd, a.jt);
            if (threadIdx.x == 0) s_seed = rng_jump(sd, (uint64_t)nr, a.jt);
            beta = sqrt(seg_cgs2(V, a.ldv, nr, jj + 1, w, sm.h1, sm.h2, sm.red));
        }
        if (threadIdx.x == 0) a.seed[c] = s_seed;
        dead = !(beta > thr);
    }
    if (threadIdx.x == 0) a.ops[c] += 1;
    if (dead) {
        if (threadIdx.x == 0) {
            a.m[c] = jj + 1;       // the basis ends here (reference: ncv = j + 1)
            a.ext[c] = 0;
        }
        return;
    }
    const double s = 1.0 / beta;
    double *vn = a.V + o + (int64_t)(jj + 1) * a.ldv;
    const bool more = jj + 1 < m;
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        const double v = w[r] * s;
        vn[r] = v;
        if (more) a.x[o + r] = v;
    }
    if (threadIdx.x == 0) {
        if (more) {
            H[(jj + 1) + (int64_t)jj * a.ncv] = brec;
            H[jj + (int64_t)(jj + 1) * a.ncv] = brec;
        }
        a.j[c] = jj + 1;
        if (!more) a.ext[c] = 0;
    }
}

// x = V[:, 0:m] s over the segment
SPX_DEV void seg_combine(const double *V, int64_t ldv, int nr, int m, const double *s, double *x) {
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        double acc = 0.0;
        for (int q = 0; q < m; q++) acc += V[r + (int64_t)q * ldv] * s[q];
        x[r] = acc;
    }
    __syncthreads();
}

// the wanted Ritz vectors (reference :245-251): x = V s_i, normalised
__global__ void __launch_bounds__(kSegThreads) seg_ritz_kernel(SegArgs a) {
    extern __shared__ double sh[];
    const int c = blockIdx.x;
    if (!a.live[c]) return;
    const SegSmem sm = seg_smem(sh, a.ncv);
    const int o = a.off[c], nr = a.off[c + 1] - o;
    const int m = a.m[c], nwant = min(a.k, m);
    const double *S = a.S + (size_t)c * a.ncv * a.ncv;    // ld m
    const int *ord = a.ord + (size_t)c * a.ncv;
    for (int t = 0; t < nwant; t++) {
        double *x = a.X + (int64_t)t * a.ldv + o;
        seg_combine(a.V + o, a.ldv, nr, m, S + (size_t)ord[t] * m, x);
        const double xn2 = seg_norm2(x, nr, sm.red);
        if (xn2 > 0.0) {
            const double s = 1.0 / sqrt(xn2);
            for (int r = threadIdx.x; r < nr; r += blockDim.x) x[r] *= s;
        }
        __syncthreads();
    }
}

// Rayleigh quotients and true residuals (reference :252-263)
__global__ void __launch_bounds__(kSegThreads) seg_resid_kernel(SegArgs a) {
    extern __shared__ double sh[];
    const int c = blockIdx.x;
    if (!a.live[c]) return;
    const SegSmem sm = seg_smem(sh, a.ncv);
    const int o = a.off[c], nr = a.off[c + 1] - o;
    const int m = a.m[c], nwant = min(a.k, m);
    int conv = 0;
    for (int t = 0; t < nwant; t++) {
        const double *x = a.X + (int64_t)t * a.ldv + o, *ax = a.AX + (int64_t)t * a.ldv + o;
        double d = 0.0;
        for (int r = threadIdx.x; r < nr; r += blockDim.x) d += x[r] * ax[r];
        const double lam = block_sum(d, sm.red);
        double q = 0.0;
        for (int r = threadIdx.x; r < nr; r += blockDim.x) {
            const double e = ax[r] - lam * x[r];
            q += e * e;
        }
        const double r2 = block_sum(q, sm.red);
        if (threadIdx.x == 0) {
            a.lam[(size_t)c * a.k + t] = lam;
            a.r2[(size_t)c * a.k + t] = r2;
        }
        conv += (sqrt(r2) <= a.rtol[c]) ? 1 : 0;
    }
    if (threadIdx.x == 0) a.nconv[c] = conv;
}

// thick restart (reference :270-303): keep the top-l Ritz vectors that stay
// independent, continue from the (m+1)-th Lanczos vector
__global__ void __launch_bounds__(kSegThreads) seg_restart_kernel(SegArgs a) {
    extern __shared__ double sh[];
    __shared__ uint64_t s_seed;
    const int c = blockIdx.x;
    if (!a.live[c]) return;
    const SegSmem sm = seg_smem(sh, a.ncv);
    const int o = a.off[c], nr = a.off[c + 1] - o;
    const int m = a.m[c];
    int l = min(a.l, m - 1);
    if (l < 1) l = 1;
    const double *V = a.V + o;
    double *Vn = a.Vn + o;
    const double *S = a.S + (size_t)c * a.ncv * a.ncv;
    const double *th = a.theta + (size_t)c * a.ncv;
    const int *ord = a.ord + (size_t)c * a.ncv;
    int nret = 0;
    for (int t = 0; t < m && nret < l; t++) {
        const int i = ord[t];
        double *y = Vn + (int64_t)nret * a.ldv;
        seg_combine(V, a.ldv, nr, m, S + (size_t)i * m, y);
        const double nrm = sqrt(seg_cgs2(Vn, a.ldv, nr, nret, y, sm.h1, sm.h2, sm.red));
        if (nrm < 1e-10) continue;                // collapsed: dropped
        const double s = 1.0 / nrm;
        for (int r = threadIdx.x; r < nr; r += blockDim.x) y[r] *= s;
        if (threadIdx.x == 0) sm.ths[nret] = th[i];
        __syncthreads();
        nret++;
    }
    double *w = a.w + o;
    for (int r = threadIdx.x; r < nr; r += blockDim.x) w[r] = V[r + (int64_t)m * a.ldv];
    __syncthreads();
    double nrm = sqrt(seg_cgs2(Vn, a.ldv, nr, nret, w, sm.h1, sm.h2, sm.red));
    if (nrm < 1e-10) {
        if (threadIdx.x == 0) s_seed = a.seed[c];
        __syncthreads();
        const uint64_t sd = s_seed;
        seg_rand(w, nr, sd, a.jt);
        if (threadIdx.x == 0) a.seed[c] = rng_jump(sd, (uint64_t)nr, a.jt);
        nrm = sqrt(seg_cgs2(Vn, a.ldv, nr, nret, w, sm.h1, sm.h2, sm.red));
    }
    if (nrm < 1e-10) {
        // no continuation: the component stops with its last results
        if (threadIdx.x == 0) {
            a.live[c] = 0;
            a.stop[c] = 1;
            a.ext[c] = 0;
        }
        return;
    }
    const double s = 1.0 / nrm;
    double *vc = Vn + (int64_t)nret * a.ldv;
    for (int r = threadIdx.x; r < nr; r += blockDim.x) vc[r] = w[r] * s;
    __syncthreads();
    double *Vw = a.V + o;
    for (int q = 0; q <= nret; q++)
        for (int r = threadIdx.x; r < nr; r += blockDim.x)
            Vw[r + (int64_t)q * a.ldv] = Vn[r + (int64_t)q * a.ldv];
    for (int r = threadIdx.x; r < nr; r += blockDim.x) a.x[o + r] = vc[r];
    double *H = a.H + (size_t)c * a.ncv * a.ncv;
    for (int e = threadIdx.x; e < a.ncv * a.ncv; e += blockDim.x) {
        const int rr = e % a.ncv, cc = e / a.ncv;
        H[e] = (rr == cc && rr < nret) ? sm.ths[rr] : 0.0;
    }
    if (threadIdx.x == 0) {
        a.j[c] = nret;
        a.ext[c] = 1;
    }
}

size_t seg_smem_bytes(int ncv) { return sizeof(double) * (3 * (size_t)(ncv + 1) + 64); }

}  // namespace

void launch_seg_start(const SegArgs &a, uint64_t seed, cudaStream_t st) {
    seg_start_kernel<<<a.nseg, kSegThreads, seg_smem_bytes(a.ncv), st>>>(a, seed);
    note_launch();
}
void launch_seg_step(const SegArgs &a, cudaStream_t st) {
    seg_step_kernel<<<a.nseg, kSegThreads, seg_smem_bytes(a.ncv), st>>>(a);
    note_launch();
}
void launch_seg_ritz(const SegArgs &a, cudaStream_t st) {
    seg_ritz_kernel<<<a.nseg, kSegThreads, seg_smem_bytes(a.ncv), st>>>(a);
    note_launch();
}
void launch_seg_resid(const SegArgs &a, cudaStream_t st) {
    seg_resid_kernel<<<a.nseg, kSegThreads, seg_smem_bytes(a.ncv), st>>>(a);
    note_launch();
}
void launch_seg_restart(const SegArgs &a, cudaStream_t st) {
    seg_restart_kernel<<<a.nseg, kSegThreads, seg_smem_bytes(a.ncv), st>>>(a);
    note_launch();
}

}  // namespace spx
