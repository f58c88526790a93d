// solve_multi.cu -- kernel-ridge solves with several right-hand sides at once:
// (H + shift I) X = B by block-lockstep conjugate gradients (hmg_cg_multi_*,
// hmg_cg_solve_multi).
//
// No reference counterpart (hmglib has no solver; the diagonal `regularization` of
// its assemblers, kernel_system_assembler.h:47-48, is the shift).  Every column runs
// its own CG recurrence; the columns share one multi-vector product per iteration
// (hmg_matvec_multi reads the stored H-matrix once for all of them).  Vectors, inner
// products, step lengths and stopping tests are FP64 and computed on the device: one
// iteration is a product plus seven small kernels, and nothing waits for the host.
// Converged columns are frozen (alpha = beta = 0).
//
// Refinement (refine != 0) targets the stored operator applied exactly, as
// hmg_cg_solve does for one vector: the true residual R = B - (H + shift I) X is
// computed with FP64-arithmetic products; the inner CG (on the correction) uses
// FP64-arithmetic products while its largest relative residual is above
// 0.1 tol / 2e-7 and the handle's arithmetic after that (relaxed inexact Krylov);
// when every column's recurrence residual is below tol |b| the correction is added
// to X and the true residual is recomputed (at most 20 times).
//
// The host drives the state machine in hmg_cg_multi_advance: it enqueues work and
// reads residual norms back through pinned buffers and events, so a serving loop can
// interleave solve iterations with other work on the same stream.  Deterministic:
// the reductions run in a fixed order.
#include <algorithm>
#include <cmath>
#include <new>

#include "hmg_matrix.cuh"

namespace hmg {

static constexpr int MR_THREADS = 256;
static constexpr int MR_BLOCKS = 148;    // partial sums per column
static constexpr int MR_INFLIGHT = 2;     // iterations enqueued ahead of the last completed check
static constexpr int MR_MAX_OUTER = 20;   // true-residual restarts
static constexpr double MR_FP32_PRODUCT_ERR = 2e-7;  // FP32-arithmetic product error (see solve.cu)
static constexpr double MR_RELAX = 0.1;

// part[j * MR_BLOCKS + b] = partial of column j's a_j . b_j
__global__ void k_mr_dot_partial(const double* a, long long lda, const double* b, long long ldb, long long n,
                                 double* part)
{
    __shared__ double sh[MR_THREADS / 32];
    const int j = blockIdx.y;
    const double* aj = a + (size_t)j * lda;
    const double* bj = b + (size_t)j * ldb;
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * MR_THREADS + threadIdx.x; i < n; i += (long long)gridDim.x * MR_THREADS)
        acc = fma(aj[i], bj[i], acc);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < MR_THREADS / 32; w++) s += sh[w];
        part[(size_t)j * gridDim.x + blockIdx.x] = s;
    }
}

// out[j] = sum of column j's partials, in order
__global__ void k_mr_dot_final(const double* part, int np, int k, double* out)
{
    const int j = threadIdx.x;
    if (j >= k) return;
    double s = 0.0;
    for (int i = 0; i < np; i++) s += part[(size_t)j * np + i];
    out[j] = s;
}

// Column scalars of the recurrence, one thread per column.
struct MrScal {
    double *bb, *rr, *rrn, *pq, *alpha, *beta;
    int* active;  // 1 while the column iterates
    int* bad;     // set when p.Ap <= 0 on an active column
};

__global__ void k_mr_alpha(MrScal s, int k)
{
    const int j = threadIdx.x;
    if (j >= k) return;
    double a = 0.0;
    if (s.active[j]) {
        if (s.pq[j] > 0.0) a = s.rr[j] / s.pq[j];
        else *s.bad = 1;
    }
    s.alpha[j] = a;
}

// beta from the new residual norms; a column stops once |r| <= tol |b| (tol2 = tol^2)
__global__ void k_mr_beta(MrScal s, int k, double tol2)
{
    const int j = threadIdx.x;
    if (j >= k) return;
    double b = 0.0;
    if (s.active[j]) {
        b = s.rr[j] > 0.0 ? s.rrn[j] / s.rr[j] : 0.0;
        s.rr[j] = s.rrn[j];
        if (!(s.rrn[j] > tol2 * s.bb[j])) s.active[j] = 0;
    }
    s.beta[j] = b;
}

// inner CG start: active where the true residual is above tol |b|
__global__ void k_mr_start(MrScal s, int k, double tol2)
{
    const int j = threadIdx.x;
    if (j >= k) return;
    s.active[j] = s.rr[j] > tol2 * s.bb[j] ? 1 : 0;
}

// D += alpha P, R -= alpha Q (ld n)
__global__ void k_mr_axpy2(const double* alpha, const double* P, const double* Q, double* D, double* R, long long n,
                           int k)
{
    const long long tot = n * k;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const double a = alpha[e / n];
        if (a != 0.0) {
            D[e] = fma(a, P[e], D[e]);
            R[e] = fma(-a, Q[e], R[e]);
        }
    }
}

// P = R + beta P on active columns
__global__ void k_mr_xpby(const double* beta, const int* active, const double* R, double* P, long long n, int k)
{
    const long long tot = n * k;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / n);
        if (active[j]) P[e] = fma(beta[j], P[e], R[e]);
    }
}

// Q += shift P
__global__ void k_mr_shift(double shift, const double* P, double* Q, long long n, int k)
{
    const long long tot = n * k;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x)
        Q[e] = fma(shift, P[e], Q[e]);
}

// R = B - Y (B with leading dimension ldb, R and Y with n)
__global__ void k_mr_resid(const double* B, long long ldb, const double* Y, double* R, long long n, int k)
{
    const long long tot = n * k;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const long long j = e / n, i = e - j * n;
        R[e] = B[j * ldb + i] - Y[e];
    }
}

// X += D (X with leading dimension ldx)
__global__ void k_mr_addx(const double* D, double* X, long long ldx, long long n, int k)
{
    const long long tot = n * k;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const long long j = e / n, i = e - j * n;
        X[j * ldx + i] += D[e];
    }
}

// X copied to a dense n x k work array (ld n)
__global__ void k_mr_pack(const double* X, long long ldx, double* W, long long n, int k)
{
    const long long tot = n * k;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const long long j = e / n, i = e - j * n;
        W[e] = X[j * ldx + i];
    }
}

}  // namespace hmg

using namespace hmg;

// A check: residual norms and activity flags at one point of the recurrence, copied
// to pinned host memory behind an event.
struct MrCheck {
    cudaEvent_t ev = nullptr;
    double* rr = nullptr;   // pinned [k]: |r_j|^2
    double* bb = nullptr;   // pinned [k]: |b_j|^2
    int* active = nullptr;  // pinned [k + 1]: activity flags, then the "not positive definite" flag
    int iter = 0;           // iterations enqueued when it was taken
    bool resid = false;     // a true-residual check
};

enum { MR_RESID = 0, MR_WAIT_RESID = 1, MR_ITER = 2, MR_DONE = 3 };
static constexpr int MR_HIST = 8;  // per-iteration check results kept (indexed by iteration mod 8)

// Decisions are made from the check of iteration m - 1 when iteration m + 1 is about
// to be enqueued (or from the true residual for the first two iterations of an inner
// loop), never from whichever checks happen to have completed: the sequence of
// product arithmetics and the stopping iteration do not depend on GPU timing.
struct hmg_cg_multi {
    hmg_matrix* h = nullptr;
    int k = 0;
    long long n = 0;
    double shift = 0.0, tol = 0.0;
    int maxit = 0, refine = 0;
    const double* B = nullptr;
    long long ldb = 0;
    double* X = nullptr;
    long long ldx = 0;
    double *R = nullptr, *P = nullptr, *Q = nullptr, *D = nullptr, *W = nullptr, *part = nullptr, *sc = nullptr;
    int* flags = nullptr;  // active[k], then the bad flag
    MrScal s{};
    MrCheck checks[MR_INFLIGHT + 1];
    int nchecks = 0, head = 0;  // checks in flight: a queue in `checks`
    int state = MR_RESID;
    int iters = 0, outer = 0;
    int inner_start = 0;        // iterations enqueued when the current inner loop began
    int consumed = 0;           // iteration of the latest consumed iteration check
    bool resid_ready = false;   // the last true-residual check has been consumed
    double resid_worst = HUGE_VAL;    // largest relative true residual of the last restart
    double worst_hist[MR_HIST];       // per iteration: largest relative residual of the active columns
    int act_hist[MR_HIST];            // per iteration: active columns after it
    double relres[64];                // latest true relative residual per column
};

static hmg_status mr_dot(hmg_cg_multi* c, const double* a, const double* b, double* out)
{
    cudaStream_t st = c->h->stream;
    k_mr_dot_partial<<<dim3(MR_BLOCKS, c->k), MR_THREADS, 0, st>>>(a, c->n, b, c->n, c->n, c->part);
    HMG_LAUNCH_CHECK();
    k_mr_dot_final<<<1, 64, 0, st>>>(c->part, MR_BLOCKS, c->k, out);
    HMG_LAUNCH_CHECK();
    return HMG_OK;
}

static int mr_grid(long long tot) { return (int)std::min<long long>((tot + MR_THREADS - 1) / MR_THREADS, 4 * 148); }

// Q = (H + shift I) P for all k columns; fp64: FP64-arithmetic products
static hmg_status mr_apply(hmg_cg_multi* c, const double* P, double* Q, bool fp64)
{
    hmg_matrix* h = c->h;
    hmg_status st;
    if (fp64) {
        for (int j = 0; j < c->k; j++)
            if ((st = matvec_device(h, P + (size_t)j * c->n, Q + (size_t)j * c->n, true))) return st;
    } else if ((st = matvec_multi(h, c->k, P, (int)c->n, Q, (int)c->n))) {
        return st;
    }
    if (c->shift != 0.0) {
        k_mr_shift<<<mr_grid(c->n * c->k), MR_THREADS, 0, h->stream>>>(c->shift, P, Q, c->n, c->k);
        HMG_LAUNCH_CHECK();
    }
    return HMG_OK;
}

static hmg_status mr_push_check(hmg_cg_multi* c, bool resid)
{
    cudaStream_t st = c->h->stream;
    MrCheck& ck = c->checks[(c->head + c->nchecks) % (MR_INFLIGHT + 1)];
    HMG_CUDA_TRY(cudaMemcpyAsync(ck.rr, c->s.rr, sizeof(double) * c->k, cudaMemcpyDeviceToHost, st));
    HMG_CUDA_TRY(cudaMemcpyAsync(ck.bb, c->s.bb, sizeof(double) * c->k, cudaMemcpyDeviceToHost, st));
    HMG_CUDA_TRY(cudaMemcpyAsync(ck.active, c->flags, sizeof(int) * (c->k + 1), cudaMemcpyDeviceToHost, st));
    HMG_CUDA_TRY(cudaEventRecord(ck.ev, st));
    ck.iter = c->iters;
    ck.resid = resid;
    c->nchecks++;
    return HMG_OK;
}

// R = B - (H + shift I) X and rr = |R|^2 (FP64-arithmetic products when refining)
static hmg_status mr_true_residual(hmg_cg_multi* c)
{
    cudaStream_t st = c->h->stream;
    hmg_status e;
    k_mr_pack<<<mr_grid(c->n * c->k), MR_THREADS, 0, st>>>(c->X, c->ldx, c->W, c->n, c->k);
    HMG_LAUNCH_CHECK();
    if ((e = mr_apply(c, c->W, c->Q, c->refine != 0))) return e;
    k_mr_resid<<<mr_grid(c->n * c->k), MR_THREADS, 0, st>>>(c->B, c->ldb, c->Q, c->R, c->n, c->k);
    HMG_LAUNCH_CHECK();
    if ((e = mr_dot(c, c->R, c->R, c->s.rr))) return e;
    c->resid_ready = false;
    return mr_push_check(c, true);
}

// inner CG on the correction D from the true residual in R: P = R, D = 0, the columns
// above tol |b| active
static hmg_status mr_start_inner(hmg_cg_multi* c)
{
    cudaStream_t st = c->h->stream;
    HMG_CUDA_TRY(cudaMemcpyAsync(c->P, c->R, sizeof(double) * c->n * c->k, cudaMemcpyDeviceToDevice, st));
    HMG_CUDA_TRY(cudaMemsetAsync(c->D, 0, sizeof(double) * c->n * c->k, st));
    k_mr_start<<<1, 64, 0, st>>>(c->s, c->k, c->tol * c->tol);
    HMG_LAUNCH_CHECK();
    c->inner_start = c->iters;
    return HMG_OK;
}

// one CG iteration of every active column; worst: the largest relative residual the
// product arithmetic is chosen from
static hmg_status mr_iterate(hmg_cg_multi* c, double worst)
{
    cudaStream_t st = c->h->stream;
    hmg_status e;
    const double rel_fp64 = MR_RELAX * c->tol / MR_FP32_PRODUCT_ERR;
    const bool fp64 = c->refine && worst > rel_fp64;
    if ((e = mr_apply(c, c->P, c->Q, fp64))) return e;
    if ((e = mr_dot(c, c->P, c->Q, c->s.pq))) return e;
    k_mr_alpha<<<1, 64, 0, st>>>(c->s, c->k);
    HMG_LAUNCH_CHECK();
    k_mr_axpy2<<<mr_grid(c->n * c->k), MR_THREADS, 0, st>>>(c->s.alpha, c->P, c->Q, c->D, c->R, c->n, c->k);
    HMG_LAUNCH_CHECK();
    if ((e = mr_dot(c, c->R, c->R, c->s.rrn))) return e;
    k_mr_beta<<<1, 64, 0, st>>>(c->s, c->k, c->tol * c->tol);
    HMG_LAUNCH_CHECK();
    k_mr_xpby<<<mr_grid(c->n * c->k), MR_THREADS, 0, st>>>(c->s.beta, c->s.active, c->R, c->P, c->n, c->k);
    HMG_LAUNCH_CHECK();
    c->iters++;
    return mr_push_check(c, false);
}

// consume the completed checks, oldest first (wait: block for the oldest one)
static hmg_status mr_poll(hmg_cg_multi* c, bool wait)
{
    while (c->nchecks > 0) {
        MrCheck& ck = c->checks[c->head];
        if (wait) {
            HMG_CUDA_TRY(cudaEventSynchronize(ck.ev));
            wait = false;
        } else {
            const cudaError_t q = cudaEventQuery(ck.ev);
            if (q == cudaErrorNotReady) return HMG_OK;
            if (q != cudaSuccess) {
                set_error("hmg_cg_multi: %s", cudaGetErrorString(q));
                return HMG_ERR_CUDA;
            }
        }
        c->head = (c->head + 1) % (MR_INFLIGHT + 1);
        c->nchecks--;
        if (ck.active[c->k]) {
            set_error("hmg_cg_multi: the operator is not positive definite along a search direction (p.Ap <= 0)");
            return HMG_ERR_INVALID;
        }
        double worst = 0.0;
        int act = 0;
        for (int j = 0; j < c->k; j++) {
            const double rel = ck.bb[j] > 0.0 ? std::sqrt(ck.rr[j] / ck.bb[j]) : 0.0;
            if (ck.resid) {
                c->relres[j] = rel;
                worst = std::max(worst, rel);
            } else if (ck.active[j]) {
                worst = std::max(worst, rel);
                act++;
            }
        }
        if (ck.resid) {
            c->resid_worst = worst;
            c->resid_ready = true;
        } else {
            c->worst_hist[ck.iter % MR_HIST] = worst;
            c->act_hist[ck.iter % MR_HIST] = act;
            c->consumed = ck.iter;
        }
    }
    return HMG_OK;
}

static void mr_free(hmg_cg_multi* c)
{
    if (!c) return;
    cudaStream_t s = c->h ? c->h->stream : nullptr;
    if (s) cudaStreamSynchronize(s);
    dfree(c->R, s); dfree(c->P, s); dfree(c->Q, s); dfree(c->D, s); dfree(c->W, s);
    dfree(c->part, s); dfree(c->sc, s); dfree(c->flags, s);
    for (MrCheck& ck : c->checks) {
        if (ck.ev) cudaEventDestroy(ck.ev);
        if (ck.rr) cudaFreeHost(ck.rr);
        if (ck.bb) cudaFreeHost(ck.bb);
        if (ck.active) cudaFreeHost(ck.active);
    }
    delete c;
}

// Enqueues the next piece of work, if any can go; *enqueued = 1 if it did.
static hmg_status mr_advance(hmg_cg_multi* c, int* enqueued)
{
    *enqueued = 0;
    hmg_status e;
    if ((e = mr_poll(c, false))) return e;
    for (;;) {
        switch (c->state) {
        case MR_RESID:
            if ((e = mr_true_residual(c))) return e;
            c->state = MR_WAIT_RESID;
            *enqueued = 1;
            return HMG_OK;
        case MR_WAIT_RESID: {
            if (!c->resid_ready) return HMG_OK;
            bool all = true;
            for (int j = 0; j < c->k; j++) all &= c->relres[j] <= c->tol;
            if (all || c->iters >= c->maxit || c->outer >= MR_MAX_OUTER) {
                c->state = MR_DONE;
                return HMG_OK;
            }
            if ((e = mr_start_inner(c))) return e;
            c->state = MR_ITER;
            break;
        }
        case MR_ITER: {
            // iteration m + 1 is decided from the check of iteration m - 1
            const int m = c->iters, ref = m - 1;
            bool stop = m >= c->maxit;
            double worst = c->resid_worst;
            if (!stop && ref > c->inner_start) {
                if (c->consumed < ref) return HMG_OK;  // wait for it
                stop = c->act_hist[ref % MR_HIST] == 0;
                worst = c->worst_hist[ref % MR_HIST];
            }
            if (stop) {
                // the correction joins X (after every iteration in flight), then the
                // true residual decides
                k_mr_addx<<<mr_grid(c->n * c->k), MR_THREADS, 0, c->h->stream>>>(c->D, c->X, c->ldx, c->n, c->k);
                HMG_LAUNCH_CHECK();
                c->outer++;
                c->state = MR_RESID;
                break;
            }
            if ((e = mr_iterate(c, worst))) return e;
            *enqueued = 1;
            return HMG_OK;
        }
        default:
            return HMG_OK;
        }
    }
}

extern "C" {

hmg_status hmg_cg_multi_begin(hmg_cg_multi** out, hmg_matrix* h, int nrhs, double shift, const double* B, int ldb,
                              double* X, int ldx, double tol, int maxit, int refine)
{
    if (!out || !h || !B || !X) {
        set_error("hmg_cg_multi_begin: NULL argument");
        return HMG_ERR_INVALID;
    }
    *out = nullptr;
    if (h->n[0] != h->n[1]) {
        set_error("hmg_cg_multi_begin: the matrix must be square (n1 == n2)");
        return HMG_ERR_INVALID;
    }
    if (nrhs < 1 || nrhs > 64 || ldb < h->n[0] || ldx < h->n[0]) {
        set_error("hmg_cg_multi_begin: nrhs %d outside 1..64 or leading dimension below n", nrhs);
        return HMG_ERR_INVALID;
    }
    if (!std::isfinite(shift) || !std::isfinite(tol) || !(tol > 0.0) || maxit < 0) {
        set_error("hmg_cg_multi_begin: bad shift / tol / maxit");
        return HMG_ERR_INVALID;
    }
    if (!h->setup_done || !h->kernel_set || (h->naca > 0 && h->far_prec < 0)) {
        set_error("hmg_cg_multi_begin: the H-matrix is not compressed (hmg_setup, hmg_set_kernel, hmg_precompute_aca)");
        return HMG_ERR_STATE;
    }
    hmg_cg_multi* c = new (std::nothrow) hmg_cg_multi();
    if (!c) {
        set_error("hmg_cg_multi_begin: out of host memory");
        return HMG_ERR_NOMEM;
    }
    c->h = h;
    c->k = nrhs;
    c->n = h->n[0];
    c->shift = shift;
    c->tol = tol;
    c->maxit = maxit;
    c->refine = refine;
    c->B = B;
    c->ldb = ldb;
    c->X = X;
    c->ldx = ldx;
    cudaStream_t s = h->stream;
    const size_t nk = (size_t)c->n * nrhs;
    hmg_status st;
    if ((st = dalloc(&c->R, nk, s)) || (st = dalloc(&c->P, nk, s)) || (st = dalloc(&c->Q, nk, s)) ||
        (st = dalloc(&c->D, nk, s)) || (st = dalloc(&c->W, nk, s)) ||
        (st = dalloc(&c->part, (size_t)MR_BLOCKS * nrhs, s)) || (st = dalloc(&c->sc, (size_t)6 * 64, s)) ||
        (st = dalloc(&c->flags, (size_t)65, s))) {
        mr_free(c);
        return st;
    }
    c->s = MrScal{c->sc, c->sc + 64, c->sc + 128, c->sc + 192, c->sc + 256, c->sc + 320, c->flags, c->flags + 64};
    // the bad flag sits after the k activity flags in the copies: keep it at flags[k]
    c->s.bad = c->flags + nrhs;
    for (MrCheck& ck : c->checks) {
        if (cudaEventCreateWithFlags(&ck.ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost((void**)&ck.rr, sizeof(double) * 64) != cudaSuccess ||
            cudaMallocHost((void**)&ck.bb, sizeof(double) * 64) != cudaSuccess ||
            cudaMallocHost((void**)&ck.active, sizeof(int) * 65) != cudaSuccess) {
            cudaGetLastError();
            mr_free(c);
            set_error("hmg_cg_multi_begin: cannot create events / pinned buffers");
            return HMG_ERR_CUDA;
        }
    }
    if (cudaMemsetAsync(c->flags, 0, sizeof(int) * 65, s) != cudaSuccess ||
        cudaMemsetAsync(c->sc, 0, sizeof(double) * 6 * 64, s) != cudaSuccess) {
        mr_free(c);
        set_error("hmg_cg_multi_begin: cudaMemsetAsync failed");
        return HMG_ERR_CUDA;
    }
    // |b_j|^2 once
    k_mr_pack<<<mr_grid((long long)nk), MR_THREADS, 0, s>>>(B, ldb, c->W, c->n, nrhs);
    if ((st = mr_dot(c, c->W, c->W, c->s.bb))) {
        mr_free(c);
        return st;
    }
    for (int j = 0; j < 64; j++) c->relres[j] = HUGE_VAL;
    *out = c;
    return HMG_OK;
}

hmg_status hmg_cg_multi_advance(hmg_cg_multi* c, int* enqueued)
{
    if (!c) {
        set_error("hmg_cg_multi_advance: NULL state");
        return HMG_ERR_INVALID;
    }
    int e = 0;
    hmg_status st = mr_advance(c, &e);
    if (enqueued) *enqueued = e;
    if (st) c->state = MR_DONE;
    return st;
}

hmg_status hmg_cg_multi_poll(hmg_cg_multi* c, int* done, int* iters, double* relres)
{
    if (!c) {
        set_error("hmg_cg_multi_poll: NULL state");
        return HMG_ERR_INVALID;
    }
    hmg_status st = mr_poll(c, false);
    if (done) *done = c->state == MR_DONE;
    if (iters) *iters = c->iters;
    if (relres)
        for (int j = 0; j < c->k; j++) relres[j] = c->relres[j];
    return st;
}

hmg_status hmg_cg_multi_end(hmg_cg_multi* c)
{
    mr_free(c);
    return HMG_OK;
}

hmg_status hmg_cg_solve_multi(hmg_matrix* h, int nrhs, double shift, const double* B, int ldb, double* X, int ldx,
                              double tol, int maxit, int refine, int* iters, double* relres)
{
    hmg_cg_multi* c = nullptr;
    hmg_status st = hmg_cg_multi_begin(&c, h, nrhs, shift, B, ldb, X, ldx, tol, maxit, refine);
    if (st) return st;
    for (;;) {
        int enq = 0;
        if ((st = mr_advance(c, &enq))) break;
        if (c->state == MR_DONE) break;
        if (!enq) {
            if (c->nchecks == 0) {  // nothing in flight and nothing to enqueue: no progress possible
                set_error("hmg_cg_solve_multi: solver state machine stalled (state %d)", c->state);
                st = HMG_ERR_STATE;
                break;
            }
            if ((st = mr_poll(c, true))) break;  // wait for the oldest check
        }
    }
    if (!st) {
        if (iters) *iters = c->iters;
        if (relres)
            for (int j = 0; j < nrhs; j++) relres[j] = c->relres[j];
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
            set_error("hmg_cg_solve_multi: stream synchronisation failed");
            st = HMG_ERR_CUDA;
        }
    }
    mr_free(c);
    return st;
}

}  // extern "C"
