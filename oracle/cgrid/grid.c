/* FP64 gridding oracle in C (TEST INFRASTRUCTURE ONLY): Kaiser-Bessel spreading of non-uniform
 * samples onto the periodic fine grid and interpolation from it.
 *
 * It restates, for large sizes, the same arithmetic as oracle/gridding.py (GridPlan.spread /
 * GridPlan.interp): the finufft-style gridding that the reference delegates to cufinufft
 * (cpp/corelib/lib/fft/nufft.cppm:205-250), with the Kaiser-Bessel kernel
 *     phi(z) = I0(beta sqrt(1 - (2z/w)^2)) / I0(beta),  |z| < w/2,
 * coordinates folded to the fine grid in float32 exactly as the device plan does (so both choose
 * the same first cell i0 = ceil(u - w/2)), and weights evaluated in double. Work is split over
 * POSIX threads (hbo_set_threads; default: the online processor count).
 *
 * Layouts: coordinates x[a][M] (float32, radians, axis a pairs with grid axis a); transforms
 * c[T][M] and grids g[T][nf0][nf1][nf2] as interleaved complex double (re, im). Unit leading
 * axes express 1-D / 2-D (nf = 1 and x = NULL on those axes).
 *
 * Spreading is deterministic: points are bucketed by the block of slabs (axis 0) holding their
 * first cell, even blocks run in parallel, then odd blocks; a block is at least w slabs wide so
 * blocks of one phase never touch the same cell.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define HBO_PI 3.14159265358979323846

#include <unistd.h>

static int g_threads = 0;

void hbo_set_threads(int n) { g_threads = n; }

static int nthreads(void) {
    if (g_threads > 0) return g_threads;
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

/* parallel for over [0, n): body(ctx, i); items are handed out one at a time */
typedef void (*body_fn)(void* ctx, int64_t i);
typedef struct {
    body_fn body;
    void* ctx;
    int64_t n;
    int64_t next;
    pthread_mutex_t mu;
} pfor_t;

static void* pfor_worker(void* arg) {
    pfor_t* p = (pfor_t*)arg;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        const int64_t i = p->next++;
        pthread_mutex_unlock(&p->mu);
        if (i >= p->n) break;
        p->body(p->ctx, i);
    }
    return NULL;
}

static void parallel_for(int64_t n, body_fn body, void* ctx) {
    pfor_t p = {body, ctx, n, 0, PTHREAD_MUTEX_INITIALIZER};
    int nt = nthreads();
    if (nt > n) nt = (int)n;
    if (nt <= 1) {
        for (int64_t i = 0; i < n; ++i) body(ctx, i);
        return;
    }
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nt);
    int started = 0;
    for (; started < nt; ++started)
        if (pthread_create(&th[started], NULL, pfor_worker, &p) != 0) break;
    pfor_worker(&p);
    for (int k = 0; k < started; ++k) pthread_join(th[k], NULL);
    free(th);
}

static double bessel_i0(double x) {
    /* power series sum_k ((x/2)^k / k!)^2, to double rounding */
    double q = 0.25 * x * x, term = 1.0, sum = 1.0;
    for (int k = 1; k < 500; ++k) {
        term *= q / ((double)k * (double)k);
        sum += term;
        if (term < 1e-17 * sum) break;
    }
    return sum;
}

static float fold(float x, float scale, float fnf) {
    float u = x * scale;
    float q = floorf(u / fnf);
    u = u - q * fnf;
    if (u < 0.0f) u = u + fnf;
    if (u >= fnf) u = u - fnf;
    return u;
}

typedef struct {
    int64_t nf[3];
    int w;
    double beta, i0b;
} plan_t;

/* first cell (unwrapped) and the w weights of one point along one axis */
static int64_t axis_taps(const plan_t* p, int a, float x, double* wt) {
    const int64_t nf = p->nf[a];
    const float scale = (float)((double)nf / (2.0 * HBO_PI));
    const float fnf = (float)nf;
    const float u = fold(x, scale, fnf);
    const float hw = 0.5f * (float)p->w;
    const int64_t i0 = (int64_t)ceilf(u - hw);
    for (int d = 0; d < p->w; ++d) {
        const double z = (double)(i0 + d) - (double)u;
        const double r = 2.0 * z / p->w;
        const double s = 1.0 - r * r;
        wt[d] = s >= 0.0 ? bessel_i0(p->beta * sqrt(s)) / p->i0b : 0.0;
    }
    return i0;
}

static inline int64_t wrap(int64_t i, int64_t n) {
    i %= n;
    return i < 0 ? i + n : i;
}

typedef struct {
    int64_t cell[3][16];
    double wt[3][16];
    int n[3];
} taps_t;

static void point_taps(const plan_t* p, const float* const x[3], int64_t j, taps_t* t) {
    for (int a = 0; a < 3; ++a) {
        if (p->nf[a] == 1) {
            t->n[a] = 1;
            t->cell[a][0] = 0;
            t->wt[a][0] = 1.0;
            continue;
        }
        const int64_t i0 = axis_taps(p, a, x[a][j], t->wt[a]);
        t->n[a] = p->w;
        for (int d = 0; d < p->w; ++d) t->cell[a][d] = wrap(i0 + d, p->nf[a]);
    }
}

static void spread_point(const plan_t* p, const taps_t* t, int64_t j, int64_t M, int T, const double* c, double* g) {
    const int64_t n = p->nf[0] * p->nf[1] * p->nf[2];
    for (int a0 = 0; a0 < t->n[0]; ++a0) {
        for (int a1 = 0; a1 < t->n[1]; ++a1) {
            const double w01 = t->wt[0][a0] * t->wt[1][a1];
            const int64_t base = (t->cell[0][a0] * p->nf[1] + t->cell[1][a1]) * p->nf[2];
            for (int a2 = 0; a2 < t->n[2]; ++a2) {
                const double wv = w01 * t->wt[2][a2];
                const int64_t cell = base + t->cell[2][a2];
                for (int tr = 0; tr < T; ++tr) {
                    const double* v = c + 2 * ((int64_t)tr * M + j);
                    double* o = g + 2 * ((int64_t)tr * n + cell);
                    o[0] += wv * v[0];
                    o[1] += wv * v[1];
                }
            }
        }
    }
}

typedef struct {
    const plan_t* p;
    const float* x[3];
    int64_t M;
    int T;
    const double* c;
    double* g;
    const int64_t* start;
    const int64_t* order;
    int phase;
} spread_ctx_t;

static void spread_block(void* arg, int64_t i) {
    const spread_ctx_t* s = (const spread_ctx_t*)arg;
    const int64_t b = 2 * i + s->phase;
    taps_t t;
    for (int64_t k = s->start[b]; k < s->start[b + 1]; ++k) {
        const int64_t j = s->order[k];
        point_taps(s->p, s->x, j, &t);
        spread_point(s->p, &t, j, s->M, s->T, s->c, s->g);
    }
}

/* g[T][nf] += sum_j c[t][j] phi(cell - u_j); returns 0, or -1 on bad arguments / no memory */
int hbo_spread(int64_t nf0, int64_t nf1, int64_t nf2, int w, double beta, int64_t M, const float* x0,
               const float* x1, const float* x2, int T, const double* c, double* g) {
    if (w < 2 || w > 16 || M < 0 || T < 1) return -1;
    plan_t p = {{nf0, nf1, nf2}, w, beta, bessel_i0(beta)};
    const float* x[3] = {x0, x1, x2};
    /* slab axis: the first non-unit axis */
    int sa = 0;
    while (sa < 2 && p.nf[sa] == 1) ++sa;
    const int64_t ns = p.nf[sa];
    int64_t nblk = ns / w;
    if (nblk % 2) --nblk;
    if (nblk < 2) {
        taps_t t;
        for (int64_t j = 0; j < M; ++j) {
            point_taps(&p, x, j, &t);
            spread_point(&p, &t, j, M, T, c, g);
        }
        return 0;
    }
    /* bucket points by the block of their first slab */
    int64_t* start = (int64_t*)calloc((size_t)nblk + 1, sizeof(int64_t));
    int64_t* blk = (int64_t*)malloc(sizeof(int64_t) * (size_t)(M ? M : 1));
    int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(M ? M : 1));
    if (!start || !blk || !order) {
        free(start);
        free(blk);
        free(order);
        return -1;
    }
    const float scale = (float)((double)ns / (2.0 * HBO_PI));
    for (int64_t j = 0; j < M; ++j) {
        const float u = fold(x[sa][j], scale, (float)ns);
        const int64_t i0 = wrap((int64_t)ceilf(u - 0.5f * (float)w), ns);
        int64_t b = i0 * nblk / ns;
        while (b + 1 < nblk && (b + 1) * ns / nblk <= i0) ++b;
        while (b > 0 && b * ns / nblk > i0) --b;
        blk[j] = b;
        start[b + 1]++;
    }
    for (int64_t b = 0; b < nblk; ++b) start[b + 1] += start[b];
    {
        int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)nblk);
        memcpy(fill, start, sizeof(int64_t) * (size_t)nblk);
        for (int64_t j = 0; j < M; ++j) order[fill[blk[j]]++] = j;
        free(fill);
    }
    spread_ctx_t ctx = {&p, {x[0], x[1], x[2]}, M, T, c, g, start, order, 0};
    for (int phase = 0; phase < 2; ++phase) {
        ctx.phase = phase;
        parallel_for((nblk - phase + 1) / 2, spread_block, &ctx);
    }
    free(start);
    free(blk);
    free(order);
    return 0;
}

typedef struct {
    const plan_t* p;
    const float* x[3];
    int64_t M;
    int T;
    const double* g;
    double* out;
} interp_ctx_t;

static void interp_chunk(void* arg, int64_t chunk) {
    const interp_ctx_t* s = (const interp_ctx_t*)arg;
    const plan_t* p = s->p;
    const int64_t n = p->nf[0] * p->nf[1] * p->nf[2];
    const int64_t j1 = (chunk + 1) * 4096 < s->M ? (chunk + 1) * 4096 : s->M;
    for (int64_t j = chunk * 4096; j < j1; ++j) {
        taps_t t;
        point_taps(p, s->x, j, &t);
        for (int tr = 0; tr < s->T; ++tr) {
            double re = 0.0, im = 0.0;
            const double* gt = s->g + 2 * (int64_t)tr * n;
            for (int a0 = 0; a0 < t.n[0]; ++a0) {
                for (int a1 = 0; a1 < t.n[1]; ++a1) {
                    const double w01 = t.wt[0][a0] * t.wt[1][a1];
                    const int64_t base = (t.cell[0][a0] * p->nf[1] + t.cell[1][a1]) * p->nf[2];
                    for (int a2 = 0; a2 < t.n[2]; ++a2) {
                        const double wv = w01 * t.wt[2][a2];
                        const double* v = gt + 2 * (base + t.cell[2][a2]);
                        re += wv * v[0];
                        im += wv * v[1];
                    }
                }
            }
            s->out[2 * ((int64_t)tr * s->M + j)] = re;
            s->out[2 * ((int64_t)tr * s->M + j) + 1] = im;
        }
    }
}

/* out[T][M] = sum over the footprint of g[t][cell] phi(cell - u_j) */
int hbo_interp(int64_t nf0, int64_t nf1, int64_t nf2, int w, double beta, int64_t M, const float* x0,
               const float* x1, const float* x2, int T, const double* g, double* out) {
    if (w < 2 || w > 16 || M < 0 || T < 1) return -1;
    plan_t p = {{nf0, nf1, nf2}, w, beta, bessel_i0(beta)};
    const float* x[3] = {x0, x1, x2};
    interp_ctx_t ctx = {&p, {x[0], x[1], x[2]}, M, T, g, out};
    parallel_for((M + 4095) / 4096, interp_chunk, &ctx);
    return 0;
}
