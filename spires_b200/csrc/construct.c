/*
 * construct.c -- host construction of a reservoir model.
 *
 * Weights are drawn with the C library's rand() in exactly the order the
 * reference draws them, so a caller that seeds srand() gets the same W, W_in
 * and W_out from this library as from the reference:
 *
 *   1. W_in, n*din draws of generate_weight          src/reservoir.c:378-383
 *   2. recurrent topology                           src/reservoir.c:385-537
 *   3. PSC_HETEROGENEOUS per-edge tau               src/synapses/psc_heterogeneous.c:60-89
 *   4. spectral-radius rescale (no draws)           src/reservoir.c:548-557
 *   5. W_out, n*dout draws of generate_weight(0.5)  src/reservoir.c:559-571
 *
 * The reference materialises a dense n x n scratch (3.2 GB at n = 20000) and an
 * n x n byte adjacency for scale-free graphs; here rows are produced directly
 * in CSR order and the Barabasi-Albert roulette runs on a prefix-sum tree. Both
 * choices give the same picks: the roulette totals are sums of small integers,
 * which double arithmetic holds exactly, so "first u with r <= prefix(u)" is
 * the same integer search either way.
 *
 * All libm-derived constants used by the dynamics (pow, exp, log, tgamma, sin,
 * cos) are computed here with the same expressions the reference evaluates, so
 * the device only ever sees their bits.
 */
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "sp_model.h"

/* (int)x as x86-64's truncating conversion performs it -- NaN and values
 * outside the int range give INT_MIN, which is what the reference's casts of
 * configuration values produce there -- without the undefined behaviour of
 * the C cast. */
static int trunc_int(double x)
{
    return (x > -2147483649.0 && x < 2147483648.0) ? (int)x : INT_MIN;
}

/* ---------------------------------------------------------------- draws -- */

/* Private generator with the sequence of glibc's srand(seed) + rand():
 * the additive lagged-Fibonacci generator of glibc's random_r (TYPE_3,
 * degree 31, separation 3): r[0] = seed (0 becomes 1), r[i] = 16807 r[i-1]
 * mod (2^31 - 1) for i < 31 (Schrage's decomposition, on signed 32-bit words
 * as glibc keeps them), then r[f] += r[b] modulo 2^32 with the front index
 * three ahead of the back one, output r[f] >> 1, and the first 310 outputs
 * discarded. It lets worker threads build independently seeded reservoirs at
 * the same time, each drawing what srand(seed) + rand() would give it. */
void sp_rand_seed(sp_rand_state *s, unsigned seed)
{
    int32_t word = (int32_t)(seed == 0 ? 1u : seed);
    s->r[0] = word;
    for (int i = 1; i < 31; i++) {
        const long hi = word / 127773, lo = word % 127773; /* 127773 = m / 16807 */
        long v = 16807 * lo - 2836 * hi;                   /* 2836 = m % 16807 */
        if (v < 0)
            v += 2147483647;
        word = (int32_t)v;
        s->r[i] = word;
    }
    s->f = 3;
    s->b = 0;
    for (int i = 0; i < 310; i++)
        (void)sp_rand_next(s);
}

int sp_rand_next(sp_rand_state *s)
{
    const uint32_t v = (uint32_t)s->r[s->f] + (uint32_t)s->r[s->b];
    s->r[s->f] = (int32_t)v;
    s->f = s->f == 30 ? 0 : s->f + 1;
    s->b = s->b == 30 ? 0 : s->b + 1;
    return (int)(v >> 1);
}

/* Block reader over a private generator: the same draws, produced a block at
 * a time, and open to loops that look at several upcoming draws at once. It
 * keeps the raw words x[q] = x[q-31] + x[q-3] (mod 2^32), the draws being
 * x[q] >> 1, with the 31 words before the unread ones in front of them (the
 * generator's state at any position is just the 31 raw words before it, the
 * front index on the oldest, the back index three behind the front). */
#define SP_STREAM_BLOCK 4096
typedef struct {
    uint32_t x[31 + SP_STREAM_BLOCK];
    int pos; /* the next unread word, >= 31 */
    int end; /* words held */
} draw_stream;

static void ds_open(draw_stream *d, const sp_rand_state *g)
{
    for (int k = 0; k < 31; k++) /* oldest first: it sits at the front index */
        d->x[k] = (uint32_t)g->r[(g->f + k) % 31];
    d->pos = d->end = 31;
}

/* keep the unread words and the 31 before them, then fill the block */
static void ds_refill(draw_stream *d)
{
    const int from = d->pos - 31, keep = d->end - from;
    memmove(d->x, d->x + from, (size_t)keep * sizeof(uint32_t));
    d->pos = 31;
    /* the last three words ride in registers: three independent add chains */
    uint32_t a = d->x[keep - 3], b = d->x[keep - 2], c = d->x[keep - 1];
    int q = keep;
    for (; q + 3 <= 31 + SP_STREAM_BLOCK; q += 3) {
        a += d->x[q - 31];
        b += d->x[q - 30];
        c += d->x[q - 29];
        d->x[q] = a;
        d->x[q + 1] = b;
        d->x[q + 2] = c;
    }
    for (; q < 31 + SP_STREAM_BLOCK; q++)
        d->x[q] = d->x[q - 31] + d->x[q - 3];
    d->end = 31 + SP_STREAM_BLOCK;
}

static inline int ds_next(draw_stream *d)
{
    if (d->pos == d->end)
        ds_refill(d);
    return (int)(d->x[d->pos++] >> 1);
}

/* The draw source of the current thread's build: the C library's rand()
 * (the reference behaviour) unless sp_model_build_seeded installed a reader
 * over a private generator. Hot loops read the pointer once and draw through
 * draw_from. */
static __thread draw_stream *tl_stream;
static inline int draw_from(draw_stream *d) { return d ? ds_next(d) : rand(); }
static int draw_int(void) { return draw_from(tl_stream); }

/* (double)rand()/RAND_MAX, src/reservoir.c:330-333 */
static double urand01(void) { return (double)draw_int() / (double)RAND_MAX; }

/* magnitude first, then the sign draw; src/reservoir.c:308-317 */
static double draw_weight(double ei_ratio)
{
    double magnitude = (double)draw_int() / RAND_MAX;
    if (((double)draw_int() / RAND_MAX) < ei_ratio)
        return magnitude;
    return -magnitude;
}

/* The smallest K with (double)K / RAND_MAX >= c. The correctly rounded
 * division is monotone in the numerator, so urand01() < c holds exactly when
 * the draw is below K: a comparison of draws needs no division. */
static long long draw_threshold(double c)
{
    long long lo = 0, hi = (long long)RAND_MAX + 1;
    while (lo < hi) {
        const long long mid = lo + (hi - lo) / 2;
        if ((double)mid / (double)RAND_MAX < c)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/* urand01() from a given source */
static inline double urand01_from(draw_stream *d) { return (double)draw_from(d) / (double)RAND_MAX; }

/* draw_weight(ei_ratio) from a given source, with the sign test as a draw
 * comparison against K_ei = draw_threshold(ei_ratio): the same two draws,
 * the same value */
static inline double weight_from(draw_stream *d, long long K_ei)
{
    const double magnitude = (double)draw_from(d) / RAND_MAX;
    return (long long)draw_from(d) < K_ei ? magnitude : -magnitude;
}

/* ------------------------------------------------------------------ CSR -- */

/* a graph with no edges: every row empty */
static int csr_empty(sp_host_model *m)
{
    m->row_ptr = calloc(m->n + 1, sizeof(int64_t));
    m->col = malloc(sizeof(int32_t));
    m->w = malloc(sizeof(double));
    m->nnz = 0;
    return (m->row_ptr && m->col && m->w) ? SP_OK : SP_EALLOC;
}

/* ------------------------------------------------------------ topologies -- */

/* Erdos-Renyi directed, no self loops; src/reservoir.c:386-397. Rows come
 * out in order and columns ascending, so the CSR is written directly (zero
 * weights dropped, as csr_build_from_dense does), with the draws in the
 * reference's order: the edge test, then the weight's two draws. */
static int er_reserve(sp_host_model *m, size_t *cap, size_t need)
{
    if (need <= *cap)
        return SP_OK;
    size_t nc = *cap + *cap / 2 + 1024;
    if (nc < need)
        nc = need;
    int32_t *col = realloc(m->col, nc * sizeof(int32_t));
    if (!col)
        return SP_EALLOC;
    m->col = col;
    double *w = realloc(m->w, nc * sizeof(double));
    if (!w)
        return SP_EALLOC;
    m->w = w;
    *cap = nc;
    return SP_OK;
}

static int topo_random(sp_host_model *m)
{
    const size_t n = m->n;
    const double density = m->connectivity > 0.0 ? (m->connectivity < 1.0 ? m->connectivity : 1.0)
                                                 : 0.0; /* NaN: no edges */
    size_t cap = (size_t)((double)n * (double)n * density * 1.05) + 1024;
    m->row_ptr = calloc(n + 1, sizeof(int64_t));
    m->col = malloc(cap * sizeof(int32_t));
    m->w = malloc(cap * sizeof(double));
    if (!m->row_ptr || !m->col || !m->w)
        return SP_EALLOC;
    /* the edge test and the weight's sign test as draw comparisons */
    const long long K = draw_threshold(m->connectivity);
    const long long K_ei = draw_threshold(m->ei_ratio);
    draw_stream *ds = tl_stream;
    size_t e = 0;
    if (ds) {
        /* Private generator: a pair takes one draw, or three when it is an
         * edge. Reading them from a block, the pairs up to the next edge are
         * a run of draws at or above K, found by a scan that does not branch
         * per pair on the random outcome; rows are crossed by counting. */
        const size_t per_row = n - 1; /* pairs (i, j), j != i, of a row */
        size_t i = 0, jj = 0;         /* the next pair: row i, its jj-th column */
        int pos = ds->pos, end = ds->end; /* local: the stores below may alias */
        while (i < n) {
            if (pos == end) {
                ds->pos = pos;
                ds_refill(ds);
                pos = ds->pos;
                end = ds->end;
            }
            const size_t left = per_row - jj, avail = (size_t)(end - pos);
            const size_t span = left < avail ? left : avail;
            const uint32_t *x = ds->x + pos;
            size_t q = 0;
            while (q < span && (long long)(x[q] >> 1) >= K)
                q++;
            pos += (int)q;
            jj += q;
            if (q < span) { /* an edge: its test draw, then the weight's two */
                pos++;
                if (end - pos < 2) {
                    ds->pos = pos;
                    ds_refill(ds);
                    pos = ds->pos;
                    end = ds->end;
                }
                const int mag_draw = (int)(ds->x[pos] >> 1);
                const long long sign_draw = (long long)(ds->x[pos + 1] >> 1);
                pos += 2;
                if (mag_draw != 0) { /* a zero weight is dropped, either sign */
                    if (e == cap && er_reserve(m, &cap, e + 1))
                        return SP_EALLOC;
                    const double mag = (double)mag_draw / RAND_MAX;
                    m->col[e] = (int32_t)(jj + (jj >= i));
                    m->w[e] = sign_draw < K_ei ? mag : -mag;
                    e++;
                }
                jj++;
            }
            if (jj == per_row) {
                i++;
                jj = 0;
                if (i < n)
                    m->row_ptr[i] = (int64_t)e;
            }
        }
        ds->pos = pos;
    } else {
        for (size_t i = 0; i < n; i++) {
            m->row_ptr[i] = (int64_t)e;
            for (size_t j = 0; j < n; j++) {
                if (i == j)
                    continue;
                if ((long long)rand() < K) {
                    const double v = weight_from(NULL, K_ei);
                    if (v == 0.0)
                        continue;
                    if (er_reserve(m, &cap, e + 1))
                        return SP_EALLOC;
                    m->col[e] = (int32_t)j;
                    m->w[e] = v;
                    e++;
                }
            }
        }
    }
    m->row_ptr[n] = (int64_t)e;
    m->nnz = e;
    return SP_OK;
}

static void sort_i32_small(int32_t *v, int k)
{
    for (int a = 1; a < k; a++) { /* insertion sort: a row's rewired targets */
        const int32_t x = v[a];
        int c = a - 1;
        while (c >= 0 && v[c] > x) {
            v[c + 1] = v[c];
            c--;
        }
        v[c + 1] = x;
    }
}

/* Watts-Strogatz on a directed ring; src/reservoir.c:399-443. The ring pass
 * draws every ring weight before any rewiring draw, so ring weights are kept
 * per row and each row is then rewired against its own dense scratch row.
 * A row's columns are its ring targets -- two ascending runs, 0..i+half-n
 * when the ring wraps and i+1..min(i+half, n-1) -- and its rewired targets,
 * sorted on their own; merging the three gives the row's columns ascending,
 * written straight to CSR (zero weights, the rewired-away ring edges among
 * them, dropped as csr_build_from_dense drops them). A row never holds more
 * than half entries: each rewiring removes one and adds at most one. */
static int topo_small_world(sp_host_model *m)
{
    size_t n = m->n;
    if (n < 3)
        return csr_empty(m);
    int K = trunc_int((m->connectivity) * (double)(n - 1) + 0.5);
    if (K < 2)
        K = 2;
    if (K % 2)
        K++;
    if (K >= (int)n)
        K = (int)n - 1;
    const double p = 0.1;
    draw_stream *ds = tl_stream;
    const long long K_ei = draw_threshold(m->ei_ratio);
    const int half = K / 2;
    const size_t cap = n * (size_t)half;

    double *ring = malloc((cap ? cap : 1) * sizeof(double));
    double *row = calloc(n, sizeof(double));
    int32_t *added = malloc(((size_t)half + 1) * sizeof(int32_t));
    m->row_ptr = calloc(n + 1, sizeof(int64_t));
    m->col = malloc((cap + 1) * sizeof(int32_t)); /* + 1: see the merge below */
    m->w = malloc((cap + 1) * sizeof(double));
    if (!ring || !row || !added || !m->row_ptr || !m->col || !m->w) {
        free(ring);
        free(row);
        free(added);
        return SP_EALLOC;
    }
    for (size_t i = 0; i < n; i++)
        for (int s = 1; s <= half; s++)
            ring[i * half + (s - 1)] = weight_from(ds, K_ei);

    size_t e = 0;
    for (size_t i = 0; i < n; i++) {
        for (int s = 1; s <= half; s++)
            row[(i + (size_t)s) % n] = ring[i * half + (s - 1)];
        int na = 0;
        for (int s = 1; s <= half; s++) {
            size_t j_old = (i + (size_t)s) % n;
            if (urand01_from(ds) < p) {
                row[j_old] = 0.0;
                size_t j_new;
                long long attempts = 0;
                do {
                    j_new = (size_t)(urand01_from(ds) * (double)n);
                    if (j_new >= n)
                        j_new = n - 1;
                    if (++attempts > 10 * (long long)n)
                        break;
                } while (j_new == i || row[j_new] != 0.0);
                if (j_new != i) {
                    row[j_new] = weight_from(ds, K_ei);
                    added[na++] = (int32_t)j_new;
                }
            }
        }
        sort_i32_small(added, na);
        /* The ring runs in ascending order -- [0, top - n] after the wrap (if
         * any), then [i + 1, min(top, n - 1)] -- with the sorted rewired
         * targets merged in. Every column is written and kept (e advanced)
         * only when its weight is nonzero and it is not a repeat; the one
         * spare slot of the arrays absorbs a last write that is not kept. */
        const size_t top = i + (size_t)half;
        const int64_t runs[2][2] = {{0, top < n ? -1 : (int64_t)(top - n)},
                                    {(int64_t)i + 1, (int64_t)(top < n ? top : n - 1)}};
        int k = 0;         /* next rewired target */
        int64_t last = -1; /* last column looked at */
        int32_t *col = m->col;
        double *w = m->w;
        for (int rr = 0; rr < 2; rr++)
            for (int64_t c = runs[rr][0]; c <= runs[rr][1]; c++) {
                for (; k < na && added[k] < c; k++) {
                    const int64_t a = added[k];
                    const double v = row[a];
                    col[e] = (int32_t)a;
                    w[e] = v;
                    e += (size_t)((v != 0.0) & (a != last));
                    last = a;
                }
                const double v = row[c];
                col[e] = (int32_t)c;
                w[e] = v;
                e += (size_t)((v != 0.0) & (c != last));
                last = c;
            }
        for (; k < na; k++) {
            const int64_t a = added[k];
            const double v = row[a];
            col[e] = (int32_t)a;
            w[e] = v;
            e += (size_t)((v != 0.0) & (a != last));
            last = a;
        }
        for (int s = 1; s <= half; s++)
            row[(i + (size_t)s) % n] = 0.0;
        for (int a2 = 0; a2 < na; a2++)
            row[added[a2]] = 0.0;
        m->row_ptr[i + 1] = (int64_t)e;
    }
    m->nnz = e;
    free(ring);
    free(row);
    free(added);
    return SP_OK;
}

/* The Barabasi-Albert roulette: weights deg[u] + 1 per node, a point update
 * per pick and the search for the first node whose prefix sum reaches a
 * target. The path of that search is random, so it is the latency of its
 * dependent loads that sets the pace.
 *
 * Main form: a tree of int32 inclusive prefix sums -- 16-ary levels, one
 * 64-byte node per 16 children, up to a single root node of at most 64
 * entries (8000 nodes: 500 and 32 nodes of 16, a root of 32; 34 KB,
 * cache-resident). A level costs one node load and its comparisons in 4-lane
 * vectors, against one load per level of a binary tree; the wide root saves
 * a level. Graphs whose totals could pass INT32_MAX use a Fenwick tree over
 * int64 instead. Both return the same node for the same target. */
typedef int32_t sp_v4i __attribute__((vector_size(16)));

#define SP_ROOT_MAX 64

typedef struct {
    int32_t *e;        /* 16 entries per node, levels stored leaf-parents first */
    size_t off[16];    /* first entry of each level */
    int levels;        /* 16-ary levels, then the root */
    int root_w;        /* root entries, a multiple of 4, <= SP_ROOT_MAX */
    int64_t *t;        /* Fenwick form: t[1..tn], tn a power of two */
    size_t tn;
} roulette;

static int rl_init(roulette *r, size_t n, int64_t max_total)
{
    memset(r, 0, sizeof(*r));
    if (max_total <= INT32_MAX) {
        size_t total = 0, count = n; /* units below the level being added */
        int l = 0;
        while (count > SP_ROOT_MAX) {
            const size_t nodes = (count + 15) / 16;
            r->off[l++] = total;
            total += nodes * 16;
            count = nodes;
        }
        r->root_w = (int)((count + 3) / 4 * 4);
        r->off[l++] = total;
        total += (size_t)r->root_w;
        r->levels = l;
        if (posix_memalign((void **)&r->e, 64, total * sizeof(int32_t)))
            return SP_EALLOC;
        memset(r->e, 0, total * sizeof(int32_t));
        return SP_OK;
    }
    r->tn = 1;
    while (r->tn < n)
        r->tn <<= 1;
    r->t = calloc(r->tn + 1, sizeof(int64_t));
    return r->t ? SP_OK : SP_EALLOC;
}

static void rl_free(roulette *r)
{
    free(r->e);
    free(r->t);
}

static void rl_add(roulette *r, size_t u, int64_t d)
{
    if (r->e) {
        const sp_v4i i0 = {0, 1, 2, 3}, i1 = {4, 5, 6, 7}, i2 = {8, 9, 10, 11},
                     i3 = {12, 13, 14, 15}, four = {4, 4, 4, 4};
        const int32_t d32 = (int32_t)d;
        const sp_v4i dd = {d32, d32, d32, d32};
        const int top = r->levels - 1;
        for (int l = 0; l < top; l++) {
            sp_v4i *x = (sp_v4i *)(r->e + r->off[l] + (u >> (4 * (l + 1))) * 16);
            const int32_t slot = (int32_t)((u >> (4 * l)) & 15);
            const sp_v4i sl = {slot, slot, slot, slot};
            x[0] += (i0 >= sl) & dd; /* the entries from the slot on hold u */
            x[1] += (i1 >= sl) & dd;
            x[2] += (i2 >= sl) & dd;
            x[3] += (i3 >= sl) & dd;
        }
        sp_v4i *x = (sp_v4i *)(r->e + r->off[top]);
        const int32_t slot = (int32_t)(u >> (4 * top));
        const sp_v4i sl = {slot, slot, slot, slot};
        sp_v4i idx = i0;
        for (int q = 0; q < r->root_w / 4; q++, idx += four)
            x[q] += (idx >= sl) & dd;
        return;
    }
    for (size_t k = u + 1; k <= r->tn; k += k & (~k + 1))
        r->t[k] += d;
}

/* The smallest 0-based u with prefix(u) >= target, for 1 <= target <= total. */
static size_t rl_pick(const roulette *r, int64_t target)
{
    if (r->e) {
        int32_t tg = (int32_t)target;
        const int top = r->levels - 1;
        /* entries are nondecreasing: the count below the target is the child
         * holding it */
        const int32_t *p = r->e + r->off[top];
        sp_v4i t = {tg, tg, tg, tg};
        sp_v4i below = {0, 0, 0, 0};
        for (int q = 0; q < r->root_w / 4; q++)
            below += ((const sp_v4i *)p)[q] < t;
        int32_t c = -(below[0] + below[1] + below[2] + below[3]);
        tg -= c ? p[c - 1] : 0;
        size_t node = (size_t)c;
        for (int l = top - 1; l >= 0; l--) {
            p = r->e + r->off[l] + node * 16;
            const sp_v4i *x = (const sp_v4i *)p;
            t = (sp_v4i){tg, tg, tg, tg};
            below = (x[0] < t) + (x[1] < t) + (x[2] < t) + (x[3] < t);
            c = -(below[0] + below[1] + below[2] + below[3]);
            tg -= c ? p[c - 1] : 0;
            node = node * 16 + (size_t)c;
        }
        return node;
    }
    size_t pos = 0;
    for (size_t step = r->tn >> 1; step; step >>= 1) {
        const int64_t t = r->t[pos + step];
        const int64_t mask = -(int64_t)(t < target); /* a mask, not a branch */
        pos += step & (size_t)mask;
        target -= t & mask;
    }
    return pos;
}

static int cmp_i32(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* Barabasi-Albert with initial attractiveness A = 1 and random orientation;
 * src/reservoir.c:445-536. The CSR is written directly. */
static int topo_scale_free(sp_host_model *m)
{
    size_t n = m->n;
    if (n < 2)
        return csr_empty(m);
    int mm = trunc_int((m->connectivity) * (double)(n - 1) + 0.5);
    if (mm < 1)
        mm = 1;
    if (mm >= (int)n)
        mm = (int)n - 1;
    int m0 = mm > 2 ? mm : 2;
    if (m0 >= (int)n)
        m0 = (int)n - 1;

    int rc = SP_EALLOC;
    draw_stream *ds = tl_stream;
    int64_t *deg = calloc(n, sizeof(int64_t));
    size_t max_edges = (size_t)m0 * (size_t)(m0 - 1) / 2 + (n - (size_t)m0) * (size_t)mm;
    roulette rl;
    /* totals never pass sum (deg + 1) = 2 edges + n */
    const int rl_rc = rl_init(&rl, n, 2 * (int64_t)max_edges + (int64_t)n);
    int32_t *eu = malloc((max_edges ? max_edges : 1) * sizeof(int32_t));
    int32_t *ev = malloc((max_edges ? max_edges : 1) * sizeof(int32_t));
    int32_t *picks = malloc((size_t)mm * sizeof(int32_t));
    int64_t *stamp = malloc(n * sizeof(int64_t)); /* stamp[u] = last v that picked u */
    int64_t *adj_off = NULL, *fill = NULL;
    int32_t *adj = NULL;
    unsigned char *fwd = NULL;
    double *wv = NULL;
    size_t ne = 0;
    if (rl_rc || !deg || !eu || !ev || !picks || !stamp)
        goto done;
    for (size_t u = 0; u < n; u++)
        stamp[u] = -1;

    /* seed clique on m0 nodes */
    for (int u = 0; u < m0; u++)
        for (int v = u + 1; v < m0; v++) {
            eu[ne] = u;
            ev[ne] = v;
            ne++;
            deg[u]++;
            deg[v]++;
        }
    for (size_t u = 0; u < (size_t)m0; u++)
        rl_add(&rl, u, deg[u] + 1);
    int64_t degsum = 0;
    for (int u = 0; u < m0; u++)
        degsum += deg[u];

    /* The roulette holds deg[u] + 1 for every u < v, and so sums to degsum + v,
     * the roulette total (an exact integer in double, at least v > 0). The
     * draw r = urand01() * total never exceeds it, so ceil(r) is a valid
     * target of the descent: the first u with r <= acc(u), acc(u) being
     * integral, is the first with acc(u) >= ceil(r). */
    for (size_t v = (size_t)m0; v < n; v++) {
        int added = 0;
        long long guard = 0;
        /* The attempts carry no branch on their random outcome: a repeated
         * pick is written again and adds zero. The target of an attempt,
         * ceil(urand01() * total), depends on whether the previous pick was
         * kept (total + 1) or not, so both candidates are formed from the
         * previous total while that pick is still being searched, and the
         * outcome only selects one. */
        int64_t total = degsum + (int64_t)v; /* the previous attempt's total */
        int kept = 0;                         /* ... and whether it kept its pick */
        while (added < mm && guard < 50LL * mm) {
            const double r01 = urand01_from(ds);
            const int64_t t_same = (int64_t)ceil(r01 * (double)total);
            const int64_t t_more = (int64_t)ceil(r01 * (double)(total + 1));
            const int64_t target = kept ? t_more : t_same;
            total += kept;
            size_t pick = rl_pick(&rl, target); /* a zero target gives node 0 */
            pick = (pick < v) ? pick : 0;
            kept = stamp[pick] != (int64_t)v; /* not yet picked for v */
            stamp[pick] = (int64_t)v;
            picks[added] = (int32_t)pick;
            added += kept;
            deg[v] += kept;
            deg[pick] += kept;
            degsum += kept; /* only deg[pick] counts in totals for u < v */
            rl_add(&rl, pick, kept);
            guard++;
        }
        while (added < mm) {
            size_t pick = (size_t)(urand01_from(ds) * (double)v);
            if (pick >= v)
                pick = v - 1;
            const int dup = stamp[pick] == (int64_t)v; /* already picked for v */
            if (pick != v && !dup) {
                stamp[pick] = (int64_t)v;
                picks[added++] = (int32_t)pick;
                deg[v]++;
                deg[pick]++;
                degsum += 1;
                rl_add(&rl, pick, 1);
            }
        }
        for (int a = 0; a < added; a++) {
            eu[ne] = picks[a];
            ev[ne] = (int32_t)v;
            ne++;
        }
        /* node v joins the roulette for later nodes with weight deg[v] + A */
        rl_add(&rl, v, deg[v] + 1);
        degsum += deg[v];
    }

    /* Neighbours above each node, ascending: the edges (a, b), a < b, are
     * bucketed by a. They were generated in nondecreasing order of b (the seed
     * clique row by row, then node by node), so a stable bucket fill leaves
     * every bucket ascending -- the same lists a sort of the full undirected
     * adjacency would give for the j > i part the orientation pass reads. */
    adj_off = calloc(n + 1, sizeof(int64_t));
    adj = malloc((ne > 0 ? ne : 1) * sizeof(int32_t));
    fill = malloc(n * sizeof(int64_t));
    if (!adj_off || !adj || !fill)
        goto done;
    for (size_t e = 0; e < ne; e++) {
        const int32_t lo = eu[e] < ev[e] ? eu[e] : ev[e];
        adj_off[lo + 1]++;
    }
    for (size_t u = 0; u < n; u++)
        adj_off[u + 1] += adj_off[u];
    memcpy(fill, adj_off, n * sizeof(int64_t));
    for (size_t e = 0; e < ne; e++) {
        const int32_t lo = eu[e] < ev[e] ? eu[e] : ev[e];
        const int32_t hi = eu[e] < ev[e] ? ev[e] : eu[e];
        adj[fill[lo]++] = hi;
    }
    for (size_t u = 0; u < n; u++) /* guard: keep the ascending order exact */
        for (int64_t k = adj_off[u] + 1; k < adj_off[u + 1]; k++)
            if (adj[k] < adj[k - 1]) {
                qsort(adj + adj_off[u], (size_t)(adj_off[u + 1] - adj_off[u]), sizeof(int32_t),
                      cmp_i32);
                break;
            }
    free(eu);
    free(ev);
    eu = ev = NULL;

    /* Orientation in row-major order over i < j (the bucket order): per edge
     * the orientation draw (urand01() < 0.5 keeps i -> j), then the weight's
     * two draws. Orientations and weights are kept per edge and the rows
     * counted; zero weights are dropped as csr_build_from_dense drops them. */
    fwd = malloc(ne > 0 ? ne : 1);
    wv = malloc((ne > 0 ? ne : 1) * sizeof(double));
    m->row_ptr = calloc(n + 1, sizeof(int64_t));
    if (!fwd || !wv || !m->row_ptr)
        goto done;
    {
        const long long K_half = draw_threshold(0.5);
        const long long K_ei = draw_threshold(m->ei_ratio);
        for (size_t i = 0; i < n; i++)
            for (int64_t k = adj_off[i]; k < adj_off[i + 1]; k++) {
                const int f = (long long)draw_from(ds) < K_half;
                const double w = weight_from(ds, K_ei);
                const size_t r = f ? i : (size_t)adj[k];
                fwd[k] = (unsigned char)f;
                wv[k] = w;
                m->row_ptr[r + 1] += (w != 0.0);
            }
    }
    for (size_t i = 0; i < n; i++)
        m->row_ptr[i + 1] += m->row_ptr[i];
    m->nnz = (size_t)m->row_ptr[n];
    m->col = malloc((m->nnz ? m->nnz : 1) * sizeof(int32_t));
    m->w = malloc((m->nnz ? m->nnz : 1) * sizeof(double));
    if (!m->col || !m->w)
        goto done;
    memcpy(fill, m->row_ptr, n * sizeof(int64_t));
    /* One pass with i ascending: row r receives its columns below r while
     * i < r (edges (i, r) oriented r -> i), then its columns above r at i = r
     * (its own bucket, ascending), and nothing later -- ascending columns with
     * no sort. The orientation is random, so the row and column are selected
     * rather than branched on. */
    for (size_t i = 0; i < n; i++)
        for (int64_t k = adj_off[i]; k < adj_off[i + 1]; k++) {
            if (wv[k] == 0.0)
                continue;
            const size_t j = (size_t)adj[k];
            const int f = fwd[k];
            const int64_t at = fill[f ? i : j]++;
            m->col[at] = (int32_t)(f ? j : i);
            m->w[at] = wv[k];
        }
    rc = SP_OK;
done:
    free(deg);
    rl_free(&rl);
    free(eu);
    free(ev);
    free(picks);
    free(stamp);
    free(adj_off);
    free(adj);
    free(fill);
    free(fwd);
    free(wv);
    return rc;
}

/* -------------------------------------------------------- power iteration -- */

/* csr_spectral_radius, src/sparse.c:93-127 (max-abs normalised power
 * iteration, tol 1e-6, at most 1000 iterations, x0 = 1). */
/* edge count from which the power iteration runs on the device */
#define SP_DEVICE_SR_MIN_NNZ ((size_t)1 << 15)

/* y[i] = the row-i sum over its edges in ascending order, for rows [i0, i1).
 * Four rows at a time, each with its own accumulator, keep four add chains in
 * flight where one row alone would wait on each addition; every row's sum
 * keeps its order and so its bits. */
static void csr_matvec_rows(const int64_t *rp, const int32_t *col, const double *w,
                            const double *x, double *y, size_t i0, size_t i1)
{
    size_t i = i0;
    for (; i + 4 <= i1; i += 4) {
        int64_t a0 = rp[i], a1 = rp[i + 1], a2 = rp[i + 2], a3 = rp[i + 3];
        const int64_t e0 = a1, e1 = a2, e2 = a3, e3 = rp[i + 4];
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int64_t common = e0 - a0;
        common = e1 - a1 < common ? e1 - a1 : common;
        common = e2 - a2 < common ? e2 - a2 : common;
        common = e3 - a3 < common ? e3 - a3 : common;
        for (int64_t t = 0; t < common; t++) {
            s0 += w[a0 + t] * x[col[a0 + t]];
            s1 += w[a1 + t] * x[col[a1 + t]];
            s2 += w[a2 + t] * x[col[a2 + t]];
            s3 += w[a3 + t] * x[col[a3 + t]];
        }
        for (a0 += common; a0 < e0; a0++)
            s0 += w[a0] * x[col[a0]];
        for (a1 += common; a1 < e1; a1++)
            s1 += w[a1] * x[col[a1]];
        for (a2 += common; a2 < e2; a2++)
            s2 += w[a2] * x[col[a2]];
        for (a3 += common; a3 < e3; a3++)
            s3 += w[a3] * x[col[a3]];
        y[i] = s0;
        y[i + 1] = s1;
        y[i + 2] = s2;
        y[i + 3] = s3;
    }
    for (; i < i1; i++) {
        double s = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; k++)
            s += w[k] * x[col[k]];
        y[i] = s;
    }
}

double sp_csr_spectral_radius(size_t n, const int64_t *row_ptr, const int32_t *col,
                              const double *w)
{
    const unsigned int max_iter = 1000;
    const double tol = 1e-6;
    double *x = malloc((n ? n : 1) * sizeof(double));
    double *y = malloc((n ? n : 1) * sizeof(double));
    if (!x || !y) {
        free(x);
        free(y);
        return NAN;
    }
    for (size_t i = 0; i < n; i++)
        x[i] = 1.0;
    double lambda_old = 0.0, lambda_new = 0.0;
    /* Rows are independent and each row sums in ascending edge order, and the
     * maximum is exact in any order, so splitting the rows over threads gives
     * the same bits as the serial loop. */
    const int par = row_ptr[n] > 65536;
    const size_t blk = 256, nblk = (n + blk - 1) / blk;
    for (unsigned int it = 0; it < max_iter; it++) {
#pragma omp parallel for schedule(static) if (par)
        for (size_t b = 0; b < nblk; b++)
            csr_matvec_rows(row_ptr, col, w, x, y, b * blk, (b + 1) * blk < n ? (b + 1) * blk : n);
        lambda_new = 0.0;
        for (size_t i = 0; i < n; i++) {
            double a = fabs(y[i]);
            if (a > lambda_new)
                lambda_new = a;
        }
#pragma omp parallel for schedule(static) if (par)
        for (size_t i = 0; i < n; i++)
            x[i] = y[i] / lambda_new;
        if (fabs(lambda_new - lambda_old) < tol)
            break;
        lambda_old = lambda_new;
    }
    free(x);
    free(y);
    return lambda_new;
}

/* ---------------------------------------------------------- validation -- */

int sp_validate_config(size_t n, size_t din, size_t dout, double dt, int conn_type,
                       int neuron_type, const double *neuron_params, int syn_type,
                       int syn_backend)
{
    (void)din;
    (void)dout;
    /* any topology and backend value is accepted, as in the reference: an
     * unknown topology draws no recurrent edges, and every backend other than
     * SPARSE stores dense */
    (void)conn_type;
    (void)syn_backend;
    if (n == 0 || n > (size_t)INT32_MAX)
        return SP_EINVAL;
    if (neuron_type < SP_LIF_DISCRETE || neuron_type > SP_FLIF_DIFFUSIVE)
        return SP_EINVAL;
    if (syn_type < SP_SYN_SIMPLE || syn_type > SP_SYN_FRAC_MEXP)
        return SP_EINVAL;
    if (!neuron_params)
        return SP_EINVAL;
    if (!(dt > 0.0))
        return SP_EINVAL;
    return SP_OK;
}

/* ------------------------------------------------------ neuron constants -- */

/* GL coefficients, src/neuron.c:14-21: note the (float) cast of k. */
static void gl_coeffs_float_k(double *c, double alpha, int L)
{
    c[0] = 1.0;
    for (int k = 1; k < L; k++)
        c[k] = c[k - 1] * (1.0 - (alpha + 1.0) / (float)k);
}

int sp_model_derive_neuron(sp_host_model *m)
{
    const double *p = m->neuron_params;
    const double dt = m->dt;
    sp_neuron_consts nc;
    memset(&nc, 0, sizeof(nc));
    if (!p)
        return SP_EINVAL;
    switch (m->neuron_type) {
    case SP_LIF_DISCRETE: /* src/neurons/lif_discrete.c:12-41 */
        nc.a = p[0];
        nc.b = p[1];
        nc.c = 1.0 - p[2];
        nc.d = p[3];
        nc.v_init = p[0];
        break;
    case SP_LIF_BIO: /* src/neurons/lif_bio.c:4-29 */
        nc.a = p[0];
        nc.b = p[1];
        nc.c = p[2];
        nc.d = p[3];
        nc.v_init = p[0];
        break;
    case SP_FLIF_GL: { /* src/neurons/flif_gl.c:7-49, src/neuron.c:36-54 */
        double T_mem = p[5];
        int L = (T_mem > 0 && dt > 0) ? trunc_int(T_mem / dt) : 2000;
        if (L > SP_MAX_MEM_LEN)
            L = SP_MAX_MEM_LEN;
        if (L < 1)
            return SP_EINVAL; /* the reference divides by zero (step % 0) */
        if (m->coef && m->nc.L != L)
            return SP_EINVAL; /* ring length is fixed at creation */
        nc.a = p[0];
        nc.b = p[1];
        nc.c = p[2];
        nc.d = p[3];
        nc.e = p[6];
        nc.f = p[7];
        nc.g = pow(dt, p[4]);
        nc.v_init = p[2];
        nc.tprev_init = p[7] + dt;
        nc.L = L;
        if (!m->coef) { /* computed once, with the creation-time alpha */
            m->coef = malloc((size_t)L * sizeof(double));
            if (!m->coef)
                return SP_EALLOC;
            gl_coeffs_float_k(m->coef, p[4], L);
        }
        break;
    }
    case SP_FLIF_CAPUTO: { /* src/neurons/flif_caputo.c:5-40 */
        double T_mem = p[8];
        int mem_len = (T_mem > 0) ? trunc_int(T_mem / dt) : SP_MAX_MEM_LEN;
        if (mem_len > SP_MAX_MEM_LEN)
            mem_len = SP_MAX_MEM_LEN;
        int D = mem_len - 2;
        if (D < 1)
            return SP_EINVAL; /* the reference writes past a zero-length array */
        if (m->coef && m->nc.L != D)
            return SP_EINVAL;
        double alpha = p[6];
        nc.a = p[3];
        nc.b = p[4];
        nc.c = p[1];
        nc.d = p[2];
        nc.e = p[0];
        nc.f = p[7];
        nc.g = pow(dt, alpha) * tgamma(2.0 - alpha);
        nc.v_init = p[4];
        nc.tprev_init = 2 * p[7];
        nc.L = D;
        if (!m->coef) {
            m->coef = malloc((size_t)D * sizeof(double));
            if (!m->coef)
                return SP_EALLOC;
        }
        /* every neuron recomputes its weights at init, so reset re-reads alpha */
        for (int i = 0; i < D; i++) {
            double x = i + 2;
            m->coef[i] = pow(x, 1.0 - alpha) - pow(x - 1.0, 1.0 - alpha);
        }
        break;
    }
    case SP_FLIF_DIFFUSIVE: { /* src/neurons/flif_diffusive.c:67-136 */
        double tau_m = p[3], alpha = p[4], P6 = p[5], ddt = dt;
        if (tau_m <= 0.0)
            tau_m = 1.0;
        if (ddt <= 0.0)
            ddt = 1e-3;
        if (alpha < 0.0)
            alpha = 0.0;
        if (alpha > 1.0)
            alpha = 1.0;
        nc.a = p[0];
        nc.b = p[1];
        nc.c = p[2];
        nc.d = p[6];
        nc.e = ddt / tau_m;
        nc.v_init = p[2];
        if (alpha < 1.0) {
            double t_min = 1.0 * ddt;
            double t_max = (P6 > 0.0) ? P6 : 100.0 * tau_m;
            if (t_max <= t_min)
                t_max = t_min * 2.0;
            nc.f = t_min;
            nc.g = t_max;
            nc.h = ddt;
            nc.i = pow(alpha, 2.0);
            nc.j = 6.0 * alpha;
            nc.k = pow(t_min, 1.0 - nc.j);
            nc.l = pow(t_max, 1.0 - nc.j);
            nc.diff_stochastic = 1;
        } else {
            double t_ref = (P6 > 0.0) ? P6 : 0.0;
            long s = 0;
            if (t_ref > 0.0) {
                s = (long)ceil(t_ref / ddt);
                if (s < 0)
                    s = 0;
            }
            nc.h = t_ref;
            nc.det_refr_steps = (int)s;
            nc.diff_stochastic = 0;
        }
        break;
    }
    default:
        return SP_EINVAL;
    }
    m->nc = nc;
    return SP_OK;
}

/* ----------------------------------------------------- synapse constants -- */

/* GL derivative coefficients of the fractional synapse (double k),
 * src/synapses/fractional.c:95-101 */
static void gl_coeffs_double_k(double *c, double alpha, int L)
{
    c[0] = 1.0;
    for (int k = 1; k < L; k++)
        c[k] = c[k - 1] * (1.0 - (alpha + 1.0) / (double)k);
}

static double log_uniform_tau(double tau_min, double tau_max)
{
    double log_min = log(tau_min);
    double log_max = log(tau_max);
    return exp(log_min + urand01() * (log_max - log_min));
}

/* Per-type constants and draws of synapse_build_from_dense (src/synapse.c:3-30). */
int sp_model_build_synapse(sp_host_model *m, const double *unused)
{
    (void)unused;
    const double *sp = m->synapse_params;
    const double dt = m->dt;
    sp_synapse_consts sc;
    memset(&sc, 0, sizeof(sc));
    switch (m->syn_type) {
    case SP_SYN_SIMPLE:
        break;
    case SP_SYN_PSC_HOM: { /* src/synapses/psc_homogeneous.c:25-84 */
        double tau = sp ? sp[0] : 1.0;
        double decay = exp(-dt / tau);
        sc.decay = decay;
        sc.omd = 1.0 - decay;
        break;
    }
    case SP_SYN_PSC_HET: { /* src/synapses/psc_heterogeneous.c:34-89,206-229 */
        double tmin = sp ? sp[0] : 1.0, tmax = sp ? sp[1] : 1.0;
        size_t nnz = m->nnz, n = m->n;
        m->edge_tau = malloc((nnz ? nnz : 1) * sizeof(double));
        m->edge_decay = malloc((nnz ? nnz : 1) * sizeof(double));
        m->edge_omd = malloc((nnz ? nnz : 1) * sizeof(double));
        if (!m->edge_tau || !m->edge_decay || !m->edge_omd)
            return SP_EALLOC;
        if (m->syn_backend == 0) {
            for (size_t k = 0; k < nnz; k++)
                m->edge_tau[k] = log_uniform_tau(tmin, tmax);
        } else {
            /* dense storage draws a tau for every one of the n*n entries */
            for (size_t i = 0; i < n; i++) {
                int64_t k = m->row_ptr[i], kend = m->row_ptr[i + 1];
                for (size_t j = 0; j < n; j++) {
                    double t = log_uniform_tau(tmin, tmax);
                    if (k < kend && (size_t)m->col[k] == j)
                        m->edge_tau[k++] = t;
                }
            }
        }
        for (size_t k = 0; k < nnz; k++) {
            double decay = exp(-dt / m->edge_tau[k]);
            m->edge_decay[k] = decay;
            m->edge_omd[k] = 1.0 - decay;
        }
        break;
    }
    case SP_SYN_FRAC: { /* src/synapses/fractional.c:40-61,103-142 */
        double alpha = sp ? sp[0] : 1.0;
        double tau = sp ? sp[1] : 1.0;
        double T_mem = sp ? sp[2] : 10.0;
        int L = (T_mem > 0 && dt > 0) ? trunc_int(T_mem / dt) : 2000;
        if (L > SP_MAX_MEM_LEN)
            L = SP_MAX_MEM_LEN;
        if (L < 1)
            L = 1;
        m->syn_coef = malloc((size_t)L * sizeof(double));
        if (!m->syn_coef)
            return SP_EALLOC;
        gl_coeffs_double_k(m->syn_coef, alpha, L);
        sc.frac_L = L;
        sc.frac_dta = pow(dt, alpha);
        sc.frac_tau = tau;
        break;
    }
    case SP_SYN_FRAC_MEXP: { /* src/synapses/fractional_multiexp.c:21-90,136-157 */
        const double PI_ = 3.14159265358979323846;
        double alpha = sp ? sp[0] : 0.5;
        double tau_syn = sp ? sp[1] : 1.0;
        double tau_min = sp ? sp[2] : 1.0;
        double tau_max = sp ? sp[3] : 20.0;
        int N = sp ? trunc_int(sp[4] + 0.5) : 8;
        if (N < 1)
            N = 1;
        double sin_apia = sin(alpha * PI_);
        int degenerate = fabs(sin_apia) < 1e-9;
        int Nc = degenerate ? 1 : N;
        m->mexp_tau = malloc((size_t)Nc * sizeof(double));
        m->mexp_c = malloc((size_t)Nc * sizeof(double));
        m->mexp_decay = malloc((size_t)Nc * sizeof(double));
        m->mexp_omd = malloc((size_t)Nc * sizeof(double));
        double *raw = malloc((size_t)Nc * sizeof(double));
        if (!m->mexp_tau || !m->mexp_c || !m->mexp_decay || !m->mexp_omd || !raw) {
            free(raw);
            return SP_EALLOC;
        }
        if (degenerate) {
            m->mexp_tau[0] = tau_syn;
            m->mexp_c[0] = 1.0;
        } else {
            double log_tau_min = log(tau_min);
            double log_tau_max = log(tau_max);
            double d_log_tau = (N > 1) ? (log_tau_max - log_tau_min) / (N - 1) : 0.0;
            double cos_apia = cos(alpha * PI_);
            double sum_raw = 0.0;
            for (int i = 0; i < N; i++) {
                double log_tau_i = log_tau_min + i * d_log_tau;
                double tau_i = exp(log_tau_i);
                double x = tau_syn / tau_i;
                double K = (1.0 / PI_) * pow(x, alpha - 1.0) * sin_apia /
                           (pow(x, 2.0 * alpha) + 2.0 * pow(x, alpha) * cos_apia + 1.0);
                double wq = K * x * d_log_tau;
                if (wq < 0.0)
                    wq = 0.0;
                raw[i] = wq * tau_i;
                m->mexp_tau[i] = tau_i;
                sum_raw += raw[i];
            }
            for (int i = 0; i < N; i++)
                m->mexp_c[i] = (sum_raw > 0.0) ? raw[i] / sum_raw : 1.0 / N;
        }
        free(raw);
        for (int c = 0; c < Nc; c++) {
            double decay = exp(-dt / m->mexp_tau[c]);
            m->mexp_decay[c] = decay;
            m->mexp_omd[c] = 1.0 - decay;
        }
        sc.mexp_N = Nc;
        break;
    }
    default:
        return SP_EINVAL;
    }
    m->sc = sc;
    return SP_OK;
}

/* ------------------------------------------------------------- top level -- */

static double wall_ms(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return 1e3 * (double)t.tv_sec + 1e-6 * (double)t.tv_nsec;
}

int sp_model_build(sp_host_model *m)
{
    int rc;
    size_t n = m->n;
    m->micro_steps = (int)llround(1.0 / m->dt);

    /* the reference initialises neurons before drawing weights; neuron init
     * draws nothing, so the order does not matter for rand() */
    rc = sp_model_derive_neuron(m);
    if (rc)
        return rc;

    m->W_in = malloc(((n) * (m->din) > 0 ? (n) * (m->din) : 1) * sizeof(double));
    m->W_out = malloc(((n) * (m->dout) > 0 ? (n) * (m->dout) : 1) * sizeof(double));
    if (!m->W_in || !m->W_out)
        return SP_EALLOC;

    for (size_t k = 0; k < n * m->din; k++)
        m->W_in[k] = draw_weight(m->ei_ratio);

    const double t_topo = wall_ms();
    switch (m->conn_type) {
    case SP_CONN_RANDOM:
        rc = topo_random(m);
        break;
    case SP_CONN_SMALL_WORLD:
        rc = topo_small_world(m);
        break;
    case SP_CONN_SCALE_FREE:
        rc = topo_scale_free(m);
        break;
    default: /* the reference's switch has no default: no recurrent edges */
        rc = csr_empty(m);
    }
    m->topology_ms = wall_ms() - t_topo;
    if (rc)
        return rc;

    rc = sp_model_build_synapse(m, NULL);
    if (rc)
        return rc;

    /* rescale_weights, src/reservoir.c:548-557 */
    /* large matrices: the device runs the same iteration bit for bit */
    const double t_sr = wall_ms();
    double sr = 0.0;
    const char *host_env = getenv("SPIRES_HOST_SPECTRAL_RADIUS");
    if (m->host_only || m->nnz < SP_DEVICE_SR_MIN_NNZ || (host_env && host_env[0] == '1') ||
        sp_dev_spectral_radius(n, m->row_ptr, m->col, m->w, &sr) != SP_OK)
        sr = sp_csr_spectral_radius(n, m->row_ptr, m->col, m->w);
    m->spectral_radius_before = sr;
    if (sr > 1e-9) {
        double f = m->spectral_radius / sr;
        for (size_t k = 0; k < m->nnz; k++)
            m->w[k] = f * m->w[k];
    }
    m->spectral_ms = wall_ms() - t_sr;

    /* randomize_output_layer, src/reservoir.c:559-571 */
    for (size_t k = 0; k < n * m->dout; k++)
        m->W_out[k] = draw_weight(0.5);

    /* FLIF_DIFFUSIVE seeds: the reference hashes the heap address of each
     * neuron (flif_diffusive.c:119-126), which no caller can reproduce; this
     * library hashes the parameter bits and the neuron index instead. */
    {
        uint64_t s = 0x9E3779B97F4A7C15ULL;
        for (int i = 0; i < 7 && m->neuron_type == SP_FLIF_DIFFUSIVE; i++) {
            uint64_t bits;
            memcpy(&bits, &m->neuron_params[i], sizeof(bits));
            s ^= bits + 0x9E3779B97F4A7C15ULL + (s << 6) + (s >> 2);
        }
        m->diffusive_seed = s;
    }
    return SP_OK;
}

void sp_model_free(sp_host_model *m)
{
    if (!m)
        return;
    free(m->W_in);
    free(m->W_out);
    free(m->row_ptr);
    free(m->col);
    free(m->w);
    free(m->coef);
    free(m->edge_decay);
    free(m->edge_omd);
    free(m->edge_tau);
    free(m->syn_coef);
    free(m->mexp_decay);
    free(m->mexp_omd);
    free(m->mexp_c);
    free(m->mexp_tau);
    memset(m, 0, sizeof(*m));
}

/* Recurrent weights from a dense row-major matrix, then the synapse build
 * (synapse_build_from_dense, src/synapse.c:3-30; PSC_HETEROGENEOUS draws its
 * per-edge tau here). Used by coarse-graining, which builds its merged matrix
 * densely (src/reservoir.c:951). */
int sp_model_set_dense_weights(sp_host_model *m, const double *dense)
{
    size_t n = m->n, nnz = 0;
    for (size_t k = 0; k < n * n; k++)
        if (dense[k] != 0.0)
            nnz++;
    m->row_ptr = calloc(n + 1, sizeof(int64_t));
    m->col = malloc((nnz ? nnz : 1) * sizeof(int32_t));
    m->w = malloc((nnz ? nnz : 1) * sizeof(double));
    if (!m->row_ptr || !m->col || !m->w)
        return SP_EALLOC;
    size_t idx = 0;
    for (size_t i = 0; i < n; i++) {
        m->row_ptr[i] = (int64_t)idx;
        for (size_t j = 0; j < n; j++) {
            double v = dense[i * n + j];
            if (v != 0.0) {
                m->col[idx] = (int32_t)j;
                m->w[idx] = v;
                idx++;
            }
        }
    }
    m->row_ptr[n] = (int64_t)idx;
    m->nnz = nnz;
    return sp_model_build_synapse(m, NULL);
}

int sp_model_build_seeded(sp_host_model *m, unsigned seed)
{
    sp_rand_state st;
    sp_rand_seed(&st, seed);
    draw_stream *ds = malloc(sizeof(*ds));
    if (!ds)
        return SP_EALLOC;
    ds_open(ds, &st);
    draw_stream *prev = tl_stream;
    tl_stream = ds;
    const int rc = sp_model_build(m);
    tl_stream = prev;
    free(ds);
    return rc;
}
