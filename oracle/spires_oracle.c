/*
 * oracle/spires_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker).
 *
 * Plain-C, single-threaded restatement of the reference reservoir step and
 * readouts. Each function cites the reference lines it follows. Compiled with
 * -ffp-contract=off so each product and sum rounds once, in source order, as
 * the reference does on x86-64. Constants the reference takes from libm are
 * evaluated with the same expressions here.
 *
 * Sum orders that define bit parity:
 *   W_in u        netlib dgemv: t = sum_j w_ij u_j ascending from +0;
 *                 ext_i = 0 + gamma t            (src/reservoir.c:132-136)
 *   recurrent     CSR row, ascending column, from +0 (src/sparse.c:68-76)
 *   GL history    ascending lag k = 1..limit     (src/neurons/flif_gl.c:67-72)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "spires_oracle.h"

#define MAX_MEM 20000
#define PI_ 3.14159265358979323846

struct orc_state {
    orc_model m;
    int micro;
    /* neuron constants */
    double p[12];
    int L;               /* GL ring length / Caputo register depth */
    double *coef;        /* GL or Caputo weights */
    double dta, kr;
    /* neuron state */
    double *V, *spike, *tprev;
    double *ring;        /* n x L, neuron-major as in the reference */
    long *nstep;         /* per-neuron internal step */
    long *refr_until;
    uint64_t *rng;
    /* synapse */
    double decay;                 /* PSC_HOM */
    double *trace;                /* PSC_HOM [n], PSC_HET [nnz] */
    double *edge_decay;
    int Ls;
    double *scoef, sdta, stau, *Ihist, *I;
    long sstep;
    int Nc;
    double *mtau, *mc, *mtr, *mcomb;
    /* scratch */
    double *ext, *last, *next;
};

static double ddot_rows(const orc_state *s, int i, const double *x)
{
    double sum = 0.0;
    for (int64_t k = s->m.row_ptr[i]; k < s->m.row_ptr[i + 1]; k++)
        sum += s->m.val[k] * x[s->m.col[k]];
    return sum;
}

/* neuron init, src/neurons/<model>.c init functions and src/neuron.c:23-60 */
static void neurons_init(orc_state *s, int first)
{
    const double *p = s->m.neuron_params;
    const double dt = s->m.dt;
    const int n = s->m.n;
    switch (s->m.neuron_type) {
    case 0: /* lif_discrete.c:12-21: [V_0, V_th, leak, bias] */
        for (int i = 0; i < n; i++) {
            s->V[i] = p[0];
            s->spike[i] = 0.0;
        }
        break;
    case 1: /* lif_bio.c:4-12: [V_0, V_th, tau, bias] */
        for (int i = 0; i < n; i++) {
            s->V[i] = p[0];
            s->spike[i] = 0.0;
        }
        break;
    case 2: { /* flif_caputo.c:5-40 */
        double T_mem = p[8];
        int mem = (T_mem > 0) ? (int)(T_mem / dt) : MAX_MEM;
        if (mem > MAX_MEM)
            mem = MAX_MEM;
        int D = mem - 2;
        if (first) {
            s->L = D;
            s->ring = calloc((size_t)n * D, sizeof(double));
            s->coef = malloc((size_t)D * sizeof(double));
        }
        for (int i = 0; i < D; i++) {
            double x = i + 2;
            s->coef[i] = pow(x, 1.0 - p[6]) - pow(x - 1.0, 1.0 - p[6]);
        }
        s->kr = pow(dt, p[6]) * tgamma(2.0 - p[6]);
        memset(s->ring, 0, (size_t)n * D * sizeof(double));
        for (int i = 0; i < n; i++) {
            s->V[i] = p[4];
            s->spike[i] = 0.0;
            s->tprev[i] = 2 * p[7];
        }
        break;
    }
    case 3: { /* flif_gl.c:7-49; coefficients once, neuron.c:36-54 */
        double T_mem = p[5];
        int L = (T_mem > 0 && dt > 0) ? (int)(T_mem / dt) : 2000;
        if (L > MAX_MEM)
            L = MAX_MEM;
        if (first) {
            s->L = L;
            s->ring = malloc((size_t)n * L * sizeof(double));
            s->coef = malloc((size_t)L * sizeof(double));
            s->coef[0] = 1.0;
            for (int k = 1; k < L; k++)
                s->coef[k] = s->coef[k - 1] * (1.0 - (p[4] + 1.0) / (float)k);
        }
        s->dta = pow(dt, p[4]);
        for (int i = 0; i < n; i++) {
            s->V[i] = p[2];
            s->spike[i] = 0.0;
            s->tprev[i] = p[7] + dt;
            s->nstep[i] = 0;
            for (int k = 0; k < s->L; k++)
                s->ring[(size_t)i * s->L + k] = p[2];
        }
        break;
    }
    case 4: { /* flif_diffusive.c:67-127 (seeded by index instead of address) */
        for (int i = 0; i < n; i++) {
            s->V[i] = p[2];
            s->spike[i] = 0.0;
            s->nstep[i] = 0;
            s->refr_until[i] = -1;
            /* SplitMix64 state after one discarded draw: the draw only
             * advances the state by the golden-ratio increment */
            uint64_t z = s->m.diffusive_seed ^ (0xD1B54A32D192ED03ULL * (uint64_t)(i + 1));
            s->rng[i] = z + 0x9E3779B97F4A7C15ULL;
        }
        break;
    }
    }
}

static uint64_t splitmix(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

orc_state *orc_create(const orc_model *m)
{
    orc_state *s = calloc(1, sizeof(*s));
    s->m = *m;
    const int n = m->n;
    const double dt = m->dt;
    s->micro = (int)llround(1.0 / dt);
    s->V = calloc(n, sizeof(double));
    s->spike = calloc(n, sizeof(double));
    s->tprev = calloc(n, sizeof(double));
    s->nstep = calloc(n, sizeof(long));
    s->refr_until = calloc(n, sizeof(long));
    s->rng = calloc(n, sizeof(uint64_t));
    s->ext = calloc(n, sizeof(double));
    s->last = calloc(n, sizeof(double));
    s->next = calloc(n, sizeof(double));
    neurons_init(s, 1);

    const double *sp = m->synapse_params;
    const size_t nnz = (size_t)m->row_ptr[n];
    switch (m->synapse_type) {
    case 1: /* psc_homogeneous.c:25-38,71-84 */
        s->decay = exp(-dt / (sp ? sp[0] : 1.0));
        s->trace = calloc(n, sizeof(double));
        break;
    case 2: /* psc_heterogeneous.c:206-229 */
        s->trace = calloc(nnz ? nnz : 1, sizeof(double));
        s->edge_decay = malloc((nnz ? nnz : 1) * sizeof(double));
        for (size_t k = 0; k < nnz; k++)
            s->edge_decay[k] = exp(-dt / m->edge_tau[k]);
        break;
    case 3: { /* fractional.c:40-61,103-142 */
        double alpha = sp ? sp[0] : 1.0;
        s->stau = sp ? sp[1] : 1.0;
        double T_mem = sp ? sp[2] : 10.0;
        int L = (T_mem > 0 && dt > 0) ? (int)(T_mem / dt) : 2000;
        if (L > MAX_MEM)
            L = MAX_MEM;
        if (L < 1)
            L = 1;
        s->Ls = L;
        s->scoef = malloc((size_t)L * sizeof(double));
        s->scoef[0] = 1.0;
        for (int k = 1; k < L; k++)
            s->scoef[k] = s->scoef[k - 1] * (1.0 - (alpha + 1.0) / (double)k);
        s->sdta = pow(dt, alpha);
        s->Ihist = calloc((size_t)n * L, sizeof(double));
        s->I = calloc(n, sizeof(double));
        break;
    }
    case 4: { /* fractional_multiexp.c:21-90,136-157 */
        double alpha = sp ? sp[0] : 0.5, tau_syn = sp ? sp[1] : 1.0;
        double tmin = sp ? sp[2] : 1.0, tmax = sp ? sp[3] : 20.0;
        int N = sp ? (int)(sp[4] + 0.5) : 8;
        if (N < 1)
            N = 1;
        double sa = sin(alpha * PI_);
        if (fabs(sa) < 1e-9) {
            s->Nc = 1;
            s->mtau = malloc(sizeof(double));
            s->mc = malloc(sizeof(double));
            s->mtau[0] = tau_syn;
            s->mc[0] = 1.0;
        } else {
            s->Nc = N;
            s->mtau = malloc(N * sizeof(double));
            s->mc = malloc(N * sizeof(double));
            double lmin = log(tmin), lmax = log(tmax);
            double dl = (N > 1) ? (lmax - lmin) / (N - 1) : 0.0;
            double ca = cos(alpha * PI_), tot = 0.0;
            for (int i = 0; i < N; i++) {
                double ti = exp(lmin + i * dl);
                double x = tau_syn / ti;
                double K = (1.0 / PI_) * pow(x, alpha - 1.0) * sa /
                           (pow(x, 2.0 * alpha) + 2.0 * pow(x, alpha) * ca + 1.0);
                double wq = K * x * dl;
                if (wq < 0.0)
                    wq = 0.0;
                s->mc[i] = wq * ti;
                s->mtau[i] = ti;
                tot += s->mc[i];
            }
            for (int i = 0; i < N; i++)
                s->mc[i] = (tot > 0.0) ? s->mc[i] / tot : 1.0 / N;
        }
        s->mtr = calloc((size_t)s->Nc * n, sizeof(double));
        s->mcomb = calloc(n, sizeof(double));
        break;
    }
    }
    return s;
}

void orc_free(orc_state *s)
{
    if (!s)
        return;
    free(s->V); free(s->spike); free(s->tprev); free(s->nstep); free(s->refr_until);
    free(s->rng); free(s->ring); free(s->coef); free(s->trace); free(s->edge_decay);
    free(s->scoef); free(s->Ihist); free(s->I); free(s->mtau); free(s->mc); free(s->mtr);
    free(s->mcomb); free(s->ext); free(s->last); free(s->next);
    free(s);
}

void orc_reset(orc_state *s) { neurons_init(s, 0); }

/* synapse_prepare, src/synapse.c:145-160 and the per-type prepare functions */
static const double *prepare(orc_state *s, const double *spk)
{
    const int n = s->m.n;
    const double dt = s->m.dt;
    switch (s->m.synapse_type) {
    case 1:
        for (int i = 0; i < n; i++)
            s->trace[i] = s->trace[i] * s->decay + (1.0 - s->decay) * spk[i];
        return s->trace;
    case 2:
        for (int i = 0; i < n; i++)
            for (int64_t k = s->m.row_ptr[i]; k < s->m.row_ptr[i + 1]; k++) {
                double d = s->edge_decay[k];
                s->trace[k] = s->trace[k] * d + (1.0 - d) * spk[s->m.col[k]];
            }
        return NULL;
    case 3: {
        const int L = s->Ls;
        const long st = s->sstep;
        const int head = (int)(st % L);
        const int lim = (st < L) ? (int)st : L - 1;
        for (int i = 0; i < n; i++) {
            double *h = s->Ihist + (size_t)i * L;
            double Ip = h[(head - 1 + L) % L];
            double hs = 0.0;
            for (int k = 1; k <= lim; k++)
                hs += s->scoef[k] * h[(head - k + L) % L];
            double rhs = (-Ip + spk[i]) / s->stau;
            double In = s->sdta * rhs - hs;
            h[head] = In;
            s->I[i] = In;
        }
        s->sstep++;
        (void)dt;
        return s->I;
    }
    case 4:
        for (int c = 0; c < s->Nc; c++) {
            double d = exp(-dt / s->mtau[c]);
            double *tr = s->mtr + (size_t)c * n;
            for (int i = 0; i < n; i++)
                tr[i] = tr[i] * d + (1.0 - d) * spk[i];
        }
        for (int i = 0; i < n; i++) {
            double sum = 0.0;
            for (int c = 0; c < s->Nc; c++)
                sum += s->mc[c] * s->mtr[(size_t)c * n + i];
            s->mcomb[i] = sum;
        }
        return s->mcomb;
    default:
        return spk;
    }
}

static double row_input(const orc_state *s, int i, const double *x)
{
    if (s->m.synapse_type == 2) {
        double sum = 0.0;
        for (int64_t k = s->m.row_ptr[i]; k < s->m.row_ptr[i + 1]; k++)
            sum += s->m.val[k] * s->trace[k];
        return sum;
    }
    return ddot_rows(s, i, x);
}

/* update_neuron for one neuron, src/neurons/<model>.c update functions */
static void update(orc_state *s, int i, double in)
{
    const double *p = s->m.neuron_params;
    const double dt = s->m.dt;
    double V = s->V[i];
    double spike = 0.0;
    switch (s->m.neuron_type) {
    case 0: /* lif_discrete.c:22-34 */
        V = (1.0 - p[2]) * V + in + p[3];
        if (V > p[1]) {
            V = p[0];
            spike = 1.0;
        }
        break;
    case 1: /* lif_bio.c:16-29 */ {
        double dV = (-V + in + p[3]) / p[2];
        V += dV * dt;
        if (V >= p[1]) {
            V = p[0];
            spike = 1.0;
        }
        break;
    }
    case 2: /* flif_caputo.c:43-71 */ {
        const int D = s->L;
        double *dm = s->ring + (size_t)i * D;
        if (s->tprev[i] > p[7]) {
            double dV = (-p[1] * (V - p[2]) + in) / p[0];
            double markov = s->kr * dV;
            for (int q = D - 1; q > 0; q--)
                dm[q] = dm[q - 1];
            dm[0] = V - p[4];
            double mem = 0;
            for (int q = 0; q < D; q++)
                mem += s->coef[q] * dm[q];
            V += markov - mem;
            if (V >= p[3]) {
                V = p[4];
                spike = 1.0;
                s->tprev[i] = 0.0;
            }
        } else {
            V = p[4];
        }
        s->tprev[i] += dt;
        break;
    }
    case 3: /* flif_gl.c:50-100 */ {
        const int L = s->L;
        double *h = s->ring + (size_t)i * L;
        const long st = s->nstep[i];
        const int head = (int)(st % L);
        if (s->tprev[i] > p[7]) {
            double Vp = h[(head - 1 + L) % L];
            double hs = 0.0;
            const int lim = (st < L) ? (int)st : L - 1;
            for (int k = 1; k <= lim; k++)
                hs += s->coef[k] * h[(head - k + L) % L];
            double rhs = (-(Vp - p[2]) / p[3]) + in + p[6];
            V = s->dta * rhs - hs;
            if (V >= p[0]) {
                V = p[1];
                spike = 1.0;
                s->tprev[i] = 0.0;
            }
        } else {
            V = p[1];
        }
        h[head] = V;
        s->nstep[i]++;
        s->tprev[i] += dt;
        break;
    }
    case 4: /* flif_diffusive.c:140-175 */ {
        double tau = p[3] > 0.0 ? p[3] : 1.0;
        double alpha = p[4] < 0.0 ? 0.0 : (p[4] > 1.0 ? 1.0 : p[4]);
        double g = dt / tau;
        double rhs = -(V - p[2]) + in + p[6];
        V = V + g * rhs;
        if (s->nstep[i] >= s->refr_until[i] && V >= p[0]) {
            V = p[1];
            spike = 1.0;
            long steps = 0;
            if (alpha < 1.0) {
                double tmin = dt, tmax = (p[5] > 0.0) ? p[5] : 100.0 * tau;
                if (tmax <= tmin)
                    tmax = tmin * 2.0;
                double m = pow(alpha, 2.0), q = 6.0 * alpha, W;
                double u0 = (splitmix(&s->rng[i]) >> 11) * (1.0 / 9007199254740992.0);
                if (u0 < m) {
                    W = dt;
                } else {
                    double u1 = (splitmix(&s->rng[i]) >> 11) * (1.0 / 9007199254740992.0);
                    if (tmax <= tmin)
                        W = tmin;
                    else if (q <= 1e-12)
                        W = tmin + u1 * (tmax - tmin);
                    else if (fabs(q - 1.0) < 1e-12)
                        W = tmin * pow(tmax / tmin, u1);
                    else
                        W = pow((1.0 - u1) * pow(tmin, 1.0 - q) + u1 * pow(tmax, 1.0 - q),
                                1.0 / (1.0 - q));
                }
                steps = (W <= 0.0) ? 0 : (long)ceil(W / dt);
                if (steps < 1)
                    steps = 1;
            } else {
                double tr = (p[5] > 0.0) ? p[5] : 0.0;
                steps = (tr <= 0.0) ? 0 : (long)ceil(tr / dt);
            }
            s->refr_until[i] = s->nstep[i] + steps;
        }
        s->nstep[i]++;
        break;
    }
    }
    s->V[i] = V;
    s->spike[i] = spike;
}

/* step_reservoir, src/reservoir.c:113-165 */
void orc_step(orc_state *s, const double *u)
{
    const int n = s->m.n, din = s->m.din;
    for (int i = 0; i < n; i++) {
        double t = 0.0;
        if (u && din > 0 && s->m.input_strength != 0.0) {
            for (int j = 0; j < din; j++)
                t = t + s->m.w_in[(size_t)i * din + j] * u[j];
            s->ext[i] = 0.0 + s->m.input_strength * t;
        } else {
            s->ext[i] = 0.0;
        }
    }
    memcpy(s->last, s->spike, n * sizeof(double));
    for (int mstep = 0; mstep < s->micro; mstep++) {
        const double *eff = prepare(s, s->last);
        for (int i = 0; i < n; i++) {
            double rec = row_input(s, i, eff);
            update(s, i, s->ext[i] + rec);
            s->next[i] = s->spike[i];
        }
        memcpy(s->last, s->next, n * sizeof(double));
    }
}

void orc_state_read(const orc_state *s, double *V, double *spikes)
{
    if (V)
        memcpy(V, s->V, s->m.n * sizeof(double));
    if (spikes)
        memcpy(spikes, s->spike, s->m.n * sizeof(double));
}

/* compute_output, src/reservoir.c:169-192 (sequential dot per output) */
void orc_output(const orc_state *s, double *y)
{
    for (int o = 0; o < s->m.dout; o++) {
        double t = 0.0;
        for (int i = 0; i < s->m.n; i++)
            t = t + s->m.w_out[(size_t)o * s->m.n + i] * s->V[i];
        y[o] = 0.0 + 1.0 * t;
    }
}

void orc_run(orc_state *s, const double *u, size_t T, double *phi, uint8_t *raster, double *y)
{
    const int n = s->m.n;
    for (size_t t = 0; t < T; t++) {
        orc_step(s, u ? u + t * s->m.din : NULL);
        if (phi)
            memcpy(phi + t * n, s->V, n * sizeof(double));
        if (raster)
            for (int i = 0; i < n; i++)
                raster[t * n + i] = s->spike[i] != 0.0;
        if (y)
            orc_output(s, y + t * s->m.dout);
    }
}

/* train_output_ridge_regression, src/reservoir.c:573-679: normal equations
 * and one LU solve with partial pivoting per output (dgesv). */
int orc_ridge(const double *X, const double *Y, size_t T, size_t w0, int n, int dout, double lam,
              double *w_out)
{
    double *A = calloc((size_t)n * n, sizeof(double));
    double *LU = malloc((size_t)n * n * sizeof(double));
    double *b = malloc((size_t)n * sizeof(double));
    int *piv = malloc((size_t)n * sizeof(int));
    int rc = 0;
    for (size_t t = w0; t < T; t++) {
        const double *x = X + t * n;
        for (int i = 0; i < n; i++) {
            double xi = x[i];
            if (xi == 0.0)
                continue;
            double *Ai = A + (size_t)i * n;
            for (int j = 0; j < n; j++)
                Ai[j] += xi * x[j];
        }
    }
    for (int i = 0; i < n; i++)
        A[(size_t)i * n + i] += lam;
    memcpy(LU, A, (size_t)n * n * sizeof(double));
    for (int j = 0; j < n; j++) {
        int p = j;
        double best = fabs(LU[(size_t)j * n + j]);
        for (int i = j + 1; i < n; i++)
            if (fabs(LU[(size_t)i * n + j]) > best) {
                best = fabs(LU[(size_t)i * n + j]);
                p = i;
            }
        piv[j] = p;
        if (LU[(size_t)p * n + j] == 0.0) {
            rc = j + 1;
            break;
        }
        if (p != j)
            for (int c = 0; c < n; c++) {
                double tmp = LU[(size_t)j * n + c];
                LU[(size_t)j * n + c] = LU[(size_t)p * n + c];
                LU[(size_t)p * n + c] = tmp;
            }
        for (int i = j + 1; i < n; i++) {
            double l = LU[(size_t)i * n + j] / LU[(size_t)j * n + j];
            LU[(size_t)i * n + j] = l;
            if (l != 0.0)
                for (int c = j + 1; c < n; c++)
                    LU[(size_t)i * n + c] -= l * LU[(size_t)j * n + c];
        }
    }
    for (int o = 0; o < dout && rc == 0; o++) {
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (size_t t = w0; t < T; t++)
                s += X[t * n + i] * Y[t * dout + o];
            b[i] = s;
        }
        for (int j = 0; j < n; j++)
            if (piv[j] != j) {
                double tmp = b[j];
                b[j] = b[piv[j]];
                b[piv[j]] = tmp;
            }
        for (int i = 0; i < n; i++) {
            double s = b[i];
            for (int c = 0; c < i; c++)
                s -= LU[(size_t)i * n + c] * b[c];
            b[i] = s;
        }
        for (int i = n - 1; i >= 0; i--) {
            double s = b[i];
            for (int c = i + 1; c < n; c++)
                s -= LU[(size_t)i * n + c] * b[c];
            b[i] = s / LU[(size_t)i * n + i];
        }
        memcpy(w_out + (size_t)o * n, b, (size_t)n * sizeof(double));
    }
    free(A);
    free(LU);
    free(b);
    free(piv);
    return rc;
}

/* train_output_iteratively, src/reservoir.c:244-280: prediction by the
 * sequential readout, then W_out row o += (lr * error_o) * state. */
void orc_train_online(orc_state *s, const double *target, double lr, double *w_out)
{
    const int n = s->m.n, dout = s->m.dout;
    for (int o = 0; o < dout; o++) {
        double t = 0.0;
        for (int i = 0; i < n; i++)
            t = t + w_out[(size_t)o * n + i] * s->V[i];
        double pred = 0.0 + 1.0 * t;
        double a = lr * (target[o] - pred);
        for (int i = 0; i < n; i++)
            w_out[(size_t)o * n + i] = w_out[(size_t)o * n + i] + a * s->V[i];
    }
}

/* train_output_rls, src/reservoir.c:681-767 (netlib-order BLAS steps). */
int orc_train_rls(orc_state *s, const double *u, const double *y, size_t T, double delta,
                  double lambda, double *w_out)
{
    const int n = s->m.n, dout = s->m.dout, din = s->m.din;
    double *P = calloc((size_t)n * n, sizeof(double));
    double *Px = malloc((size_t)n * sizeof(double));
    double *Wx = malloc((size_t)(dout ? dout : 1) * sizeof(double));
    if (!P || !Px || !Wx) {
        free(P); free(Px); free(Wx);
        return -1;
    }
    double inv_delta = 1.0 / delta;
    for (int i = 0; i < n; i++)
        P[(size_t)i * n + i] = inv_delta;
    memset(w_out, 0, (size_t)dout * n * sizeof(double));
    orc_reset(s);
    for (size_t t = 0; t < T; t++) {
        orc_step(s, u + t * din);
        const double *x = s->V;
        for (int i = 0; i < n; i++) { /* Px = P x */
            double acc = 0.0;
            for (int j = 0; j < n; j++)
                acc = acc + P[(size_t)i * n + j] * x[j];
            Px[i] = 0.0 + 1.0 * acc;
        }
        double dd = 0.0;
        for (int i = 0; i < n; i++)
            dd = dd + x[i] * Px[i];
        double denom = lambda + dd;
        double sc = 1.0 / denom;
        for (int i = 0; i < n; i++)
            Px[i] = sc * Px[i];
        for (int o = 0; o < dout; o++) {
            double acc = 0.0;
            for (int i = 0; i < n; i++)
                acc = acc + w_out[(size_t)o * n + i] * x[i];
            Wx[o] = y[t * dout + o] - (0.0 + 1.0 * acc);
        }
        for (int o = 0; o < dout; o++) /* W_out += e k^T */
            for (int i = 0; i < n; i++)
                if (Px[i] != 0.0)
                    w_out[(size_t)o * n + i] = w_out[(size_t)o * n + i] + Wx[o] * (1.0 * Px[i]);
        for (int j = 0; j < n; j++) { /* P += (-denom) k k^T */
            if (Px[j] == 0.0)
                continue;
            double tmp = -denom * Px[j];
            for (int i = 0; i < n; i++)
                P[(size_t)i * n + j] = P[(size_t)i * n + j] + Px[i] * tmp;
        }
        if (lambda != 1.0) {
            double il = 1.0 / lambda;
            for (size_t k = 0; k < (size_t)n * n; k++)
                P[k] = il * P[k];
        }
    }
    free(P);
    free(Px);
    free(Wx);
    return 0;
}
