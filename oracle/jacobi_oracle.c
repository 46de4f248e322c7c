/*
 * FP64 host oracle for the one-sided (Hestenes) Jacobi SVD.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests, the smoke
 * check and the CPU-baseline leg of the benchmark call it.  No product code
 * path links it or falls back to it.
 *
 * It restates the arithmetic of kleedaisuki/jacobi-svd-cuda src/kernels.cu
 * on the CPU, operation by operation, so that a GPU implementation that keeps
 * the same reduction order can be compared bit for bit:
 *
 *   - round-robin schedule ............ src/kernels.cu:637-678
 *   - pair statistics (a_pp,a_qq,a_pq)  src/kernels.cu:412-472
 *       T "virtual lanes": lane t sums rows t, t+T, ... with a fused
 *       multiply-add chain (nvcc contracts `x += a*b`), then a halving
 *       tree  s[t] += s[t+stride], stride = T/2 .. 1.
 *   - rotation parameters ............. src/kernels.cu:485-521
 *   - rotation of A and V columns ..... src/kernels.cu:534-575
 *   - convergence (no rotation in a whole sweep) src/kernels.cu:889-981
 *   - U and Sigma (unsorted, absolute eps cut) src/kernels.cu:586-629
 *
 * Where nvcc is free to choose how a*b - c*d is contracted into one fused
 * multiply-add, the choice is a run-time "variant" (see JO_VARIANT_*), pinned
 * against the reference binary's own outputs by tests/golden/make_golden.py.
 *
 * Build: gcc -O2 -ffp-contract=off (no implicit contraction; every fused
 * operation below is an explicit fma()).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---- arithmetic variants ------------------------------------------------ */
/* p' = c*x - s*y */
#define JO_P_PLAIN 0  /* round(c*x) - round(s*y)            */
#define JO_P_FMA_CX 1 /* fma(c, x, -round(s*y))             */
#define JO_P_FMA_SY 2 /* fma(-s, y, round(c*x))             */
/* q' = s*x + c*y */
#define JO_Q_PLAIN 0  /* round(s*x) + round(c*y)            */
#define JO_Q_FMA_SX 1 /* fma(s, x, round(c*y))              */
#define JO_Q_FMA_CY 2 /* fma(c, y, round(s*x))              */
/* variant = p_form | (q_form << 2) | (no_param_fma << 4) | (no_dot_fma << 5) */

static inline double rot_p(double c, double s, double x, double y, int form)
{
    switch (form) {
    case JO_P_FMA_CX: return fma(c, x, -(s * y));
    case JO_P_FMA_SY: return fma(-s, y, c * x);
    default: return c * x - s * y;
    }
}

static inline double rot_q(double c, double s, double x, double y, int form)
{
    switch (form) {
    case JO_Q_FMA_SX: return fma(s, x, c * y);
    case JO_Q_FMA_CY: return fma(c, y, s * x);
    default: return s * x + c * y;
    }
}

/* ---- schedule ------------------------------------------------------------ */

/* Number of rounds per sweep: n_even - 1 (0 for n < 2). */
int jo_schedule_rounds(int n)
{
    if (n < 2) return 0;
    int ne = (n % 2) ? n + 1 : n;
    return ne - 1;
}

/*
 * Fixed-head circle method, src/kernels.cu:637-678.  pairs_out holds
 * rounds * (n_even/2) (p,q) pairs; count_out[r] is the number of real pairs
 * of round r (pairs touching the dummy column of an odd n are dropped).
 * Pair i of a round is (circle[i], circle[n_even-1-i]) - not normalised.
 */
int jo_schedule(int n, int *pairs_out, int *count_out)
{
    if (n < 2) return 0;
    const int ne = (n % 2) ? n + 1 : n;
    int *circle = (int *)malloc(sizeof(int) * (size_t)ne);
    if (!circle) return -1;
    for (int i = 0; i < ne; ++i) circle[i] = (i < n) ? i : -1;
    const int half = ne / 2;
    for (int r = 0; r < ne - 1; ++r) {
        int cnt = 0;
        for (int i = 0; i < half; ++i) {
            int lhs = circle[i], rhs = circle[ne - 1 - i];
            if (lhs >= 0 && rhs >= 0) {
                pairs_out[((size_t)r * half + cnt) * 2 + 0] = lhs;
                pairs_out[((size_t)r * half + cnt) * 2 + 1] = rhs;
                ++cnt;
            }
        }
        count_out[r] = cnt;
        int last = circle[ne - 1];
        for (int i = ne - 1; i > 1; --i) circle[i] = circle[i - 1];
        circle[1] = last;
    }
    free(circle);
    return ne - 1;
}

/* ---- reductions ------------------------------------------------------- */

/* Halving tree over partial sums s[0..T) (T a power of two). */
static inline double tree_reduce(double *s, int T)
{
    for (int stride = T / 2; stride > 0; stride >>= 1)
        for (int t = 0; t < stride; ++t) s[t] += s[t + stride];
    return s[0];
}

/*
 * Pair statistics of two contiguous columns x, y of length m with T virtual
 * lanes (src/kernels.cu:412-472).
 */
static void pair_stats(const double *x, const double *y, long m, int T, int no_dot_fma,
                       double *scratch, double *pp, double *qq, double *pq)
{
    double *spp = scratch, *sqq = scratch + T, *spq = scratch + 2 * T;
    for (int t = 0; t < T; ++t) {
        double lpp = 0.0, lqq = 0.0, lpq = 0.0;
        for (long r = t; r < m; r += T) {
            double a = x[r], b = y[r];
            if (no_dot_fma) {
                lpp += a * a; lqq += b * b; lpq += a * b;
            } else {
                lpp = fma(a, a, lpp); lqq = fma(b, b, lqq); lpq = fma(a, b, lpq);
            }
        }
        spp[t] = lpp; sqq[t] = lqq; spq[t] = lpq;
    }
    *pp = tree_reduce(spp, T);
    *qq = tree_reduce(sqq, T);
    *pq = tree_reduce(spq, T);
}

/*
 * Rotation parameters, src/kernels.cu:485-521.  Returns 1 when the pair
 * rotates.
 */
static int rotation_params(double pp, double qq, double pq, double eps, int no_param_fma,
                           double *c, double *s)
{
    const double rhs = eps * sqrt(fmax(pp, 0.0) * fmax(qq, 0.0));
    if (fabs(pq) > rhs && fabs(pq) > 1.0e-300) {
        const double tau = (qq - pp) / (2.0 * pq);
        const double h = no_param_fma ? (1.0 + tau * tau) : fma(tau, tau, 1.0);
        const double t = (tau >= 0.0) ? (1.0 / (tau + sqrt(h))) : (-1.0 / (-tau + sqrt(h)));
        const double g = no_param_fma ? (1.0 + t * t) : fma(t, t, 1.0);
        const double cs = 1.0 / sqrt(g);
        *c = cs;
        *s = t * cs;
        return 1;
    }
    *c = 1.0;
    *s = 0.0;
    return 0;
}

/* ---- threaded round executor ---------------------------------------------- */

typedef struct {
    /* shared problem state */
    double *a;  /* column-major m x n working copy      */
    double *v;  /* column-major n x n (column j = V[:,j]) */
    long m, n;
    int T, variant;
    double eps;
    const int *pairs;
    const int *counts;
    int rounds, half;
    int max_sweeps;
    /* progress */
    int nthreads;
    pthread_barrier_t bar;
    int *rotated; /* per thread, per sweep */
    int sweeps_done;
    int stop;
} jo_plain_ctx;

typedef struct {
    jo_plain_ctx *ctx;
    int tid;
} jo_worker_arg;

static void rotate_cols(double *x, double *y, long len, double c, double s, int variant)
{
    const int pf = variant & 3, qf = (variant >> 2) & 3;
    for (long r = 0; r < len; ++r) {
        double xv = x[r], yv = y[r];
        x[r] = rot_p(c, s, xv, yv, pf);
        y[r] = rot_q(c, s, xv, yv, qf);
    }
}

static void *plain_worker(void *argp)
{
    jo_worker_arg *arg = (jo_worker_arg *)argp;
    jo_plain_ctx *ctx = arg->ctx;
    const int tid = arg->tid, P = ctx->nthreads;
    const int no_param_fma = (ctx->variant >> 4) & 1, no_dot_fma = (ctx->variant >> 5) & 1;
    double *scratch = (double *)malloc(sizeof(double) * 3 * (size_t)ctx->T);
    for (int sweep = 0; sweep < ctx->max_sweeps; ++sweep) {
        int any = 0;
        for (int r = 0; r < ctx->rounds; ++r) {
            const int cnt = ctx->counts[r];
            for (int i = tid; i < cnt; i += P) {
                const int p = ctx->pairs[((size_t)r * ctx->half + i) * 2 + 0];
                const int q = ctx->pairs[((size_t)r * ctx->half + i) * 2 + 1];
                double *ap = ctx->a + (size_t)p * ctx->m, *aq = ctx->a + (size_t)q * ctx->m;
                double pp, qq, pq, c, s;
                pair_stats(ap, aq, ctx->m, ctx->T, no_dot_fma, scratch, &pp, &qq, &pq);
                if (rotation_params(pp, qq, pq, ctx->eps, no_param_fma, &c, &s)) {
                    any = 1;
                    rotate_cols(ap, aq, ctx->m, c, s, ctx->variant);
                    rotate_cols(ctx->v + (size_t)p * ctx->n, ctx->v + (size_t)q * ctx->n, ctx->n, c, s,
                                ctx->variant);
                }
                /* A pair that does not rotate is left unchanged: the reference
                 * multiplies by c = 1, s = 0, which reproduces every finite value
                 * (up to the sign of an exact zero). */
            }
            if (P > 1) pthread_barrier_wait(&ctx->bar);
        }
        ctx->rotated[tid] = any;
        if (P > 1) pthread_barrier_wait(&ctx->bar);
        if (tid == 0) {
            int tot = 0;
            for (int k = 0; k < P; ++k) tot |= ctx->rotated[k];
            ctx->sweeps_done = sweep + 1;
            ctx->stop = !tot;
        }
        if (P > 1) pthread_barrier_wait(&ctx->bar);
        if (ctx->stop) break;
    }
    free(scratch);
    return NULL;
}

/* U and Sigma from the converged working copy, src/kernels.cu:586-629. */
static void build_u_sigma(const double *a, long m, long n, int T, int no_dot_fma, double eps,
                          double *u_rowmajor, double *sigma)
{
    double *s = (double *)malloc(sizeof(double) * (size_t)T);
    for (long j = 0; j < n; ++j) {
        const double *col = a + (size_t)j * m;
        for (int t = 0; t < T; ++t) {
            double acc = 0.0;
            for (long r = t; r < m; r += T) acc = no_dot_fma ? acc + col[r] * col[r] : fma(col[r], col[r], acc);
            s[t] = acc;
        }
        const double sg = sqrt(fmax(tree_reduce(s, T), 0.0));
        sigma[j] = sg;
        for (long r = 0; r < m; ++r) u_rowmajor[(size_t)r * n + j] = (sg > eps) ? (col[r] / sg) : 0.0;
    }
    free(s);
}

/*
 * Plain one-sided Jacobi SVD with the reference's arithmetic.
 *   a        row-major m x n input (m >= n >= 1)
 *   lanes    reduction width T (power of two, 32..1024); the reference's
 *            threads_per_block
 *   variant  FMA placement, see JO_VARIANT comment above
 *   threads  host threads for the pairs of a round (>= 1)
 *   u        row-major m x n, sigma n, v row-major n x n (any may be NULL)
 * Returns 0 on success, negative on invalid arguments.
 */
int jo_plain_svd(const double *a, long m, long n, double eps, int max_sweeps, int lanes, int variant,
                 int threads, double *u, double *sigma, double *v, int *sweeps)
{
    if (m <= 0 || n <= 0 || m < n || eps <= 0.0 || max_sweeps <= 0) return -1;
    if (lanes < 1 || (lanes & (lanes - 1)) != 0) return -2;
    if (threads < 1) threads = 1;
    double *aw = (double *)malloc(sizeof(double) * (size_t)m * (size_t)n);
    double *vw = (double *)calloc((size_t)n * (size_t)n, sizeof(double));
    const int rounds = jo_schedule_rounds((int)n);
    const int ne = (n % 2) ? (int)n + 1 : (int)n;
    const int half = ne / 2;
    int *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)(rounds > 0 ? rounds : 1) * (size_t)half);
    int *counts = (int *)malloc(sizeof(int) * (size_t)(rounds > 0 ? rounds : 1));
    double *sg = (double *)malloc(sizeof(double) * (size_t)n);
    double *uu = (double *)malloc(sizeof(double) * (size_t)m * (size_t)n);
    if (!aw || !vw || !pairs || !counts || !sg || !uu) return -3;
    for (long r = 0; r < m; ++r)
        for (long c = 0; c < n; ++c) aw[(size_t)c * m + r] = a[(size_t)r * n + c];
    for (long j = 0; j < n; ++j) vw[(size_t)j * n + j] = 1.0;
    jo_schedule((int)n, pairs, counts);

    jo_plain_ctx ctx;
    memset(&ctx, 0, sizeof(ctx));
    ctx.a = aw; ctx.v = vw; ctx.m = m; ctx.n = n; ctx.T = lanes; ctx.variant = variant; ctx.eps = eps;
    ctx.pairs = pairs; ctx.counts = counts; ctx.rounds = rounds; ctx.half = half;
    ctx.max_sweeps = max_sweeps;
    if (threads > half) threads = half > 0 ? half : 1;
    ctx.nthreads = threads;
    ctx.rotated = (int *)calloc((size_t)threads, sizeof(int));
    if (threads > 1) pthread_barrier_init(&ctx.bar, NULL, (unsigned)threads);
    jo_worker_arg *args = (jo_worker_arg *)malloc(sizeof(jo_worker_arg) * (size_t)threads);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int k = 0; k < threads; ++k) {
        args[k].ctx = &ctx;
        args[k].tid = k;
        if (k > 0) pthread_create(&th[k], NULL, plain_worker, &args[k]);
    }
    plain_worker(&args[0]);
    for (int k = 1; k < threads; ++k) pthread_join(th[k], NULL);
    if (threads > 1) pthread_barrier_destroy(&ctx.bar);
    if (rounds == 0) ctx.sweeps_done = 1; /* n == 1: one empty sweep, as the reference */

    build_u_sigma(aw, m, n, lanes, (variant >> 5) & 1, eps, uu, sg);
    if (u) memcpy(u, uu, sizeof(double) * (size_t)m * (size_t)n);
    if (sigma) memcpy(sigma, sg, sizeof(double) * (size_t)n);
    if (v)
        for (long r = 0; r < n; ++r)
            for (long c = 0; c < n; ++c) v[(size_t)r * n + c] = vw[(size_t)c * n + r];
    if (sweeps) *sweeps = ctx.sweeps_done;
    free(aw); free(vw); free(pairs); free(counts); free(sg); free(uu);
    free(ctx.rotated); free(args); free(th);
    return 0;
}

/* ---- batch over independent matrices --------------------------------------- */

typedef struct {
    int count;
    const long *ms, *ns;
    const long *a_off, *u_off, *s_off, *v_off;
    const double *a;
    double *u, *sigma, *v;
    int *sweeps;
    double eps;
    int max_sweeps, lanes, variant;
    int next;
    pthread_mutex_t mu;
} jo_batch_ctx;

static void *batch_worker(void *p)
{
    jo_batch_ctx *b = (jo_batch_ctx *)p;
    for (;;) {
        pthread_mutex_lock(&b->mu);
        int k = b->next++;
        pthread_mutex_unlock(&b->mu);
        if (k >= b->count) break;
        jo_plain_svd(b->a + b->a_off[k], b->ms[k], b->ns[k], b->eps, b->max_sweeps, b->lanes, b->variant, 1,
                     b->u ? b->u + b->u_off[k] : NULL, b->sigma ? b->sigma + b->s_off[k] : NULL,
                     b->v ? b->v + b->v_off[k] : NULL, b->sweeps ? b->sweeps + k : NULL);
    }
    return NULL;
}

/*
 * Solve `count` independent matrices with `threads` host threads (one matrix
 * per thread at a time).  Offsets index the packed row-major buffers; u may be
 * NULL (sigma and V only).
 */
int jo_batch_svd(int count, const long *ms, const long *ns, const long *a_off, const double *a,
                 const long *u_off, double *u, const long *s_off, double *sigma, const long *v_off,
                 double *v, int *sweeps, double eps, int max_sweeps, int lanes, int variant, int threads)
{
    jo_batch_ctx b;
    memset(&b, 0, sizeof(b));
    b.count = count; b.ms = ms; b.ns = ns; b.a_off = a_off; b.u_off = u_off; b.s_off = s_off; b.v_off = v_off;
    b.a = a; b.u = u; b.sigma = sigma; b.v = v; b.sweeps = sweeps;
    b.eps = eps; b.max_sweeps = max_sweeps; b.lanes = lanes; b.variant = variant;
    pthread_mutex_init(&b.mu, NULL);
    if (threads < 1) threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int k = 1; k < threads; ++k) pthread_create(&th[k], NULL, batch_worker, &b);
    batch_worker(&b);
    for (int k = 1; k < threads; ++k) pthread_join(th[k], NULL);
    pthread_mutex_destroy(&b.mu);
    free(th);
    return 0;
}

/*
 * One sweep only (for timing extrapolation on very large inputs): applies
 * rounds [0, rounds) of one sweep in place on a column-major working copy.
 * Returns 1 if any pair rotated.
 */
int jo_plain_partial_sweep(double *a_colmajor, double *v_colmajor, long m, long n, double eps, int lanes,
                           int variant, int rounds_to_run, int threads)
{
    const int rounds = jo_schedule_rounds((int)n);
    const int ne = (n % 2) ? (int)n + 1 : (int)n;
    const int half = ne / 2;
    if (rounds_to_run > rounds) rounds_to_run = rounds;
    int *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)(rounds > 0 ? rounds : 1) * (size_t)half);
    int *counts = (int *)malloc(sizeof(int) * (size_t)(rounds > 0 ? rounds : 1));
    jo_schedule((int)n, pairs, counts);
    jo_plain_ctx ctx;
    memset(&ctx, 0, sizeof(ctx));
    ctx.a = a_colmajor; ctx.v = v_colmajor; ctx.m = m; ctx.n = n; ctx.T = lanes; ctx.variant = variant;
    ctx.eps = eps; ctx.pairs = pairs; ctx.counts = counts; ctx.rounds = rounds_to_run; ctx.half = half;
    ctx.max_sweeps = 1;
    if (threads < 1) threads = 1;
    if (threads > half) threads = half > 0 ? half : 1;
    ctx.nthreads = threads;
    ctx.rotated = (int *)calloc((size_t)threads, sizeof(int));
    if (threads > 1) pthread_barrier_init(&ctx.bar, NULL, (unsigned)threads);
    jo_worker_arg *args = (jo_worker_arg *)malloc(sizeof(jo_worker_arg) * (size_t)threads);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int k = 0; k < threads; ++k) {
        args[k].ctx = &ctx;
        args[k].tid = k;
        if (k > 0) pthread_create(&th[k], NULL, plain_worker, &args[k]);
    }
    plain_worker(&args[0]);
    for (int k = 1; k < threads; ++k) pthread_join(th[k], NULL);
    if (threads > 1) pthread_barrier_destroy(&ctx.bar);
    int any = !ctx.stop;
    free(pairs); free(counts); free(ctx.rotated); free(args); free(th);
    return any;
}
