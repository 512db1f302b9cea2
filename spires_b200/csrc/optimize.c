/*
 * optimize.c -- spires_optimize: AGILE hyper-parameter search over the public
 * API (src/spires_api.c:263-498, src/spires_opt_agile.c, src/agile.c).
 *
 * The search logic is the reference's, step for step, so that a caller gets
 * the same sequence of candidate configurations for the same losses:
 *   - PCG32 generator with the reference's increment (src/agile.c:10-23);
 *   - two-point SPSA with Rademacher signs, clamped probes (src/agile.c:114-142);
 *   - truncated power-law (Levy) step length on [eta_min, eta_max]
 *     (src/agile.c:99-110), reflection at the bounds (src/agile.c:32-49);
 *   - exploration with patience (x0.9 per improvement, floor 1), then SPSA
 *     gradient-descent refinement from the best point (src/agile.c:217-335);
 *   - one AGILE run per budget, warm-started from the previous best, 8-D theta
 *     with the reference's bounds, start point and options
 *     (src/spires_opt_agile.c:47-190).
 * Every loss evaluation builds, trains and validates reservoirs through this
 * library, so the simulation and ridge solves run on the GPU. The validation
 * pass (src/spires_api.c:298-342) runs as one launch with the readout fused
 * in; its per-step outputs are the same bits spires_step + spires_compute_output
 * would produce.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "../../include/spires.h"
#include "../../include/spires_ext.h"
#include "sp_api_internal.h"

#define SPIRES_EXPORT __attribute__((visibility("default")))

static int verbose(void) { return getenv("SPIRES_VERBOSE") != NULL; }

/* ------------------------------------------------------------ generator -- */

static uint32_t pcg32_next(uint64_t *s)
{
    uint64_t old = *s;
    *s = old * 6364136223846793005ULL + 0xda3e39cb94b95bdbULL;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}

static double pcg_uniform(uint64_t *s) { return pcg32_next(s) * (1.0 / 4294967296.0); }

/* -------------------------------------------------------------- AGILE core -- */

typedef double (*loss_fn)(const double *theta, int dim, void *ctx);

typedef struct {
    double mu, eta_min, eta_max, patience0, patience_decay;
    double refine_step;
    int refine_max_iters, refine_no_improve;
    double spsa_eps;
    int reflect;
    uint64_t seed;
} agile_opts;

typedef struct {
    double best_loss;
    int best_iter, total_evals, total_iters, refined;
} agile_report;

static double clampd(double x, double a, double b) { return x < a ? a : (x > b ? b : x); }

static void project(double *x, const double *lo, const double *hi, int d, int reflect)
{
    for (int i = 0; i < d; i++) {
        if (!reflect) {
            x[i] = clampd(x[i], lo[i], hi[i]);
        } else if (x[i] < lo[i]) {
            double over = lo[i] - x[i], span = hi[i] - lo[i];
            double k = floor(over / span);
            x[i] = lo[i] + (over - k * span);
        } else if (x[i] > hi[i]) {
            double over = x[i] - hi[i], span = hi[i] - lo[i];
            double k = floor(over / span);
            x[i] = hi[i] - (over - k * span);
        }
    }
}

static void spsa(const double *th, const double *lo, const double *hi, int d, double eps,
                 loss_fn f, void *ctx, uint64_t *rng, double *g)
{
    double delta[64] = {0}, tp[64] = {0}, tm[64] = {0};
    for (int i = 0; i < d; i++) {
        delta[i] = (pcg32_next(rng) & 1) ? 1.0 : -1.0;
        tp[i] = clampd(th[i] + eps * delta[i], lo[i], hi[i]);
        tm[i] = clampd(th[i] - eps * delta[i], lo[i], hi[i]);
    }
    double fp = f(tp, d, ctx);
    double fm = f(tm, d, ctx);
    double scale = (fp - fm) / (2.0 * eps);
    for (int i = 0; i < d; i++)
        g[i] = scale * delta[i];
}

static double levy_step(double mu, double a, double b, uint64_t *rng)
{
    if (mu <= 1.0)
        mu = 1.000001;
    double u = pcg_uniform(rng);
    double c1 = pow(a, 1.0 - mu), c2 = pow(b, 1.0 - mu);
    return pow(c1 + (c2 - c1) * u, 1.0 / (1.0 - mu));
}

static int agile_run(const double *theta0, const double *lo, const double *hi, int d, loss_fn f,
                     void *ctx, const agile_opts *o, double *best_theta, agile_report *rep)
{
    if (d > 64)
        return -1;
    double th[64], cand[64], g[64], dir[64];
    double refine_step = o->refine_step > 0.0 ? o->refine_step : o->eta_min;
    uint64_t rng = o->seed ? o->seed : 0xA57B17E5ULL;

    memcpy(th, theta0, (size_t)d * sizeof(double));
    project(th, lo, hi, d, o->reflect);
    double loss = f(th, d, ctx);
    double best = loss;
    memcpy(best_theta, th, (size_t)d * sizeof(double));
    int evals = 1, iters = 0, best_iter = 0, refined = 0;
    double patience = o->patience0;
    int since = 0;

    for (;;) {
        iters++;
        spsa(th, lo, hi, d, o->spsa_eps, f, ctx, &rng, g);
        evals += 2;
        double s = 0.0;
        for (int i = 0; i < d; i++)
            s += g[i] * g[i];
        double gn = sqrt(s);
        if (gn > 1e-18) {
            for (int i = 0; i < d; i++)
                dir[i] = (-1.0 / gn) * g[i];
        } else {
            double ss = 0.0;
            for (int i = 0; i < d; i++) {
                double z = pcg_uniform(&rng) * 2.0 - 1.0;
                dir[i] = z;
                ss += z * z;
            }
            double nn = sqrt(ss) + 1e-18;
            for (int i = 0; i < d; i++)
                dir[i] /= nn;
        }
        double eta = levy_step(o->mu, o->eta_min, o->eta_max, &rng);
        for (int i = 0; i < d; i++)
            cand[i] = th[i] + eta * dir[i];
        project(cand, lo, hi, d, o->reflect);
        double cl = f(cand, d, ctx);
        evals++;
        if (cl < loss) {
            memcpy(th, cand, (size_t)d * sizeof(double));
            loss = cl;
            since = 0;
            patience *= o->patience_decay;
            if (patience < 1.0)
                patience = 1.0;
            if (loss < best) {
                best = loss;
                best_iter = iters;
                memcpy(best_theta, th, (size_t)d * sizeof(double));
            }
            if (verbose())
                printf("[AGILE] iter %d improved: loss=%.6g, patience=%.2f\n", iters, loss,
                       patience);
        } else {
            since++;
        }
        if (since >= (int)ceil(patience)) {
            refined = 1;
            break;
        }
        if (iters > 1000000)
            break;
    }

    if (refined) {
        memcpy(th, best_theta, (size_t)d * sizeof(double));
        loss = best;
        int no_imp = 0;
        for (int k = 0; k < o->refine_max_iters; ++k) {
            iters++;
            spsa(th, lo, hi, d, o->spsa_eps, f, ctx, &rng, g);
            evals += 2;
            for (int i = 0; i < d; i++)
                th[i] += -refine_step * g[i];
            project(th, lo, hi, d, o->reflect);
            double nl = f(th, d, ctx);
            evals++;
            if (nl < loss - 1e-12) {
                loss = nl;
                if (loss < best) {
                    best = loss;
                    best_iter = iters;
                    memcpy(best_theta, th, (size_t)d * sizeof(double));
                }
                no_imp = 0;
            } else {
                no_imp++;
            }
            if (no_imp >= o->refine_no_improve)
                break;
        }
    }
    if (rep) {
        rep->best_loss = best;
        rep->best_iter = best_iter;
        rep->total_evals = evals;
        rep->total_iters = iters;
        rep->refined = refined;
    }
    return 0;
}

/* ------------------------------------------------------ spires objective -- */

static size_t snap_n(double x)
{
    static const size_t choices[] = {200, 400, 800, 1200};
    size_t best = choices[0];
    double bd = fabs(x - (double)choices[0]);
    for (size_t i = 1; i < 4; i++) {
        double dd = fabs(x - (double)choices[i]);
        if (dd < bd) {
            bd = dd;
            best = choices[i];
        }
    }
    return best;
}

static int snap_topo(double t)
{
    int k = (int)llround(t);
    if (k < 0)
        k = 0;
    if (k > 2)
        k = 2;
    return k;
}

typedef struct {
    double alpha, rho, gain, conn, ei, log10_ridge, n_cont, topo_cont;
} opt_params;

typedef struct {
    double data_fraction;
    int num_seeds;
} budget;

typedef struct {
    const spires_reservoir_config *base;
    const double *x, *y;
    size_t n;
    int alpha_index;
    const budget *bud;
    double lambda_var, lambda_cost;
} opt_ctx;

/* mean squared error of one-step readouts over [off, off+len) */
static double validation_mse(spires_reservoir *r, const double *x, const double *y, size_t off,
                             size_t len, size_t din, size_t dout)
{
    if (len == 0 || dout == 0)
        return INFINITY;
    double *yhat = malloc(len * dout * sizeof(double));
    if (!yhat)
        return INFINITY;
    if (spires_ext_run_record(r, x + off * din, len, NULL, NULL, yhat) != SPIRES_OK) {
        free(yhat);
        return INFINITY;
    }
    const double *yb = y + off * dout;
    double se = 0.0;
    for (size_t t = 0; t < len; t++)
        for (size_t o = 0; o < dout; o++) {
            double e = yb[t * dout + o] - yhat[t * dout + o];
            se += e * e;
        }
    free(yhat);
    return se / (double)(len * dout);
}

static int evaluate(const opt_params *pr, const budget *b, const opt_ctx *ctx, double *mean_out,
                    double *std_out, double *cost_out, int *feasible)
{
    spires_reservoir_config cfg = *ctx->base;
    cfg.num_neurons = snap_n(pr->n_cont);
    cfg.spectral_radius = pr->rho;
    cfg.input_strength = pr->gain;
    cfg.connectivity = pr->conn;
    cfg.ei_ratio = pr->ei;
    cfg.connectivity_type = (spires_connectivity_type)snap_topo(pr->topo_cont);
    double local_params[8] = {0};
    if (!cfg.neuron_params)
        cfg.neuron_params = local_params;
    /* written through the caller's array, as src/spires_api.c:362-365 does */
    cfg.neuron_params[ctx->alpha_index] = pr->alpha;

    const size_t din = cfg.num_inputs ? cfg.num_inputs : 1;
    const size_t dout = cfg.num_outputs ? cfg.num_outputs : 1;
    size_t n_train = (size_t)((double)ctx->n * fmax(0.0, fmin(1.0, b->data_fraction)));
    if (n_train < 8 || ctx->n <= n_train) {
        *feasible = 0;
        *mean_out = 0.0;
        *std_out = 1.0;
        *cost_out = 1.0;
        return 0;
    }
    size_t n_valid = ctx->n - n_train;
    const int seeds = b->num_seeds > 0 ? b->num_seeds : 1;
    double sum = 0.0, sum2 = 0.0;
    int ok = 0;
    for (int s = 0; s < seeds; s++) {
        spires_reservoir *r = NULL;
        if (spires_reservoir_create(&cfg, &r) != SPIRES_OK || !r)
            continue;
        double lambda = pow(10.0, pr->log10_ridge);
        if (spires_train_ridge(r, ctx->x, ctx->y, n_train, lambda) != SPIRES_OK) {
            spires_reservoir_destroy(r);
            continue;
        }
        if (spires_reservoir_reset(r) != SPIRES_OK) {
            spires_reservoir_destroy(r);
            continue;
        }
        double mse = validation_mse(r, ctx->x, ctx->y, n_train, n_valid, din, dout);
        spires_reservoir_destroy(r);
        if (!isfinite(mse) || mse < 0.0)
            continue;
        double metric = 1.0 / (1.0 + mse);
        sum += metric;
        sum2 += metric * metric;
        ok++;
    }
    if (ok == 0) {
        *feasible = 0;
        *mean_out = 0.0;
        *std_out = 1.0;
        *cost_out = 1.0;
        return 0;
    }
    double mean = sum / (double)ok;
    double var = fmax(0.0, (sum2 / (double)ok) - mean * mean);
    *mean_out = mean;
    *std_out = sqrt(var);
    double sparsity = cfg.connectivity > 1e-8 ? cfg.connectivity : 1e-8;
    *cost_out = (double)cfg.num_neurons * (1.0 / sparsity) * 1e-6;
    *feasible = 1;
    return 0;
}

static void theta_to_params(const double *th, opt_params *p)
{
    p->alpha = th[0];
    p->rho = th[1];
    p->gain = th[2];
    p->conn = th[3];
    p->ei = th[4];
    p->log10_ridge = th[5];
    p->n_cont = th[6];
    p->topo_cont = th[7];
}

static double objective(const double *theta, int dim, void *vctx)
{
    (void)dim;
    const opt_ctx *ctx = (const opt_ctx *)vctx;
    opt_params p;
    theta_to_params(theta, &p);
    p.n_cont = (double)snap_n(p.n_cont);
    p.topo_cont = (double)snap_topo(p.topo_cont);
    double mean = 0, sd = 0, cost = 0;
    int feasible = 1;
    int rc = evaluate(&p, ctx->bud, ctx, &mean, &sd, &cost, &feasible);
    if (rc != 0 || !feasible)
        return 1e6;
    return -(mean - ctx->lambda_var * sd - ctx->lambda_cost * cost);
}

SPIRES_EXPORT int spires_optimize(const spires_reservoir_config *base_config,
                                  const struct spires_opt_budget *budgets_pub, int num_budgets,
                                  const struct spires_opt_score *score_pub,
                                  struct spires_opt_result *out_pub, const double *input_series,
                                  const double *target_series, size_t series_length)
{
    if (verbose())
        printf("[SPIRES] spires_optimize entered\n");
    if (!base_config || !budgets_pub || num_budgets <= 0 || !score_pub || !out_pub)
        return -1;
    budget *buds = calloc((size_t)num_budgets, sizeof(budget));
    if (!buds)
        return -2;
    for (int i = 0; i < num_budgets; i++) {
        buds[i].data_fraction = budgets_pub[i].data_fraction;
        buds[i].num_seeds = budgets_pub[i].num_seeds;
    }
    opt_ctx ctx = {base_config, input_series, target_series, series_length, 4, NULL,
                   score_pub->lambda_var, score_pub->lambda_cost};

    enum { D = 8 };
    const double lo[D] = {0.05, 0.75, 0.20, 0.08, 0.70, -5.0, 200.0, 0.0};
    const double hi[D] = {1.0, 1.05, 1.50, 0.35, 1.10, -1.0, 1200.0, 2.0};
    double th0[D] = {0.55, 0.90, 1.00, 0.20, 0.80, -2.0, 400.0, 0.0};
    double thb[D];
    agile_opts o = {1.3, 1e-3, 0.3, 100.0, 0.9, 1e-2, 600, 60, 1e-3, 1, 0xA91EULL};
    for (int i = 0; i < num_budgets; i++) {
        ctx.bud = &buds[i];
        agile_report rep;
        if (agile_run(th0, lo, hi, D, objective, &ctx, &o, thb, &rep) != 0) {
            free(buds);
            return -1;
        }
        if (verbose())
            printf("[AGILE] budget %d: best loss %.6g after %d evaluations\n", i, rep.best_loss,
                   rep.total_evals);
        memcpy(th0, thb, sizeof(th0));
    }

    opt_params pb;
    theta_to_params(thb, &pb);
    pb.n_cont = (double)snap_n(pb.n_cont);
    pb.topo_cont = (double)snap_topo(pb.topo_cont);
    double mean = 0, sd = 0, cost = 0;
    int feasible = 1;
    (void)evaluate(&pb, &buds[num_budgets - 1], &ctx, &mean, &sd, &cost, &feasible);
    free(buds);

    out_pub->best_config = *base_config;
    out_pub->best_config.num_neurons = snap_n(pb.n_cont);
    out_pub->best_config.spectral_radius = pb.rho;
    out_pub->best_config.input_strength = pb.gain;
    out_pub->best_config.connectivity = pb.conn;
    out_pub->best_config.ei_ratio = pb.ei;
    out_pub->best_config.connectivity_type = (spires_connectivity_type)snap_topo(pb.topo_cont);
    out_pub->best_log10_ridge = pb.log10_ridge;
    out_pub->metric_mean = mean;
    out_pub->metric_std = sd;
    out_pub->best_score = mean - score_pub->lambda_var * sd - score_pub->lambda_cost * cost;
    return 0;
}

SPIRES_EXPORT spires_status spires_ext_agile_minimize(const double *theta0, const double *lower,
                                                     const double *upper, int dim,
                                                     spires_ext_loss_fn loss, void *ctx,
                                                     const spires_ext_agile_opts *opts,
                                                     double *theta_best,
                                                     spires_ext_agile_report *report)
{
    if (!theta0 || !lower || !upper || !loss || !theta_best || dim <= 0 || dim > 64)
        return SPIRES_ERR_INVALID_ARG;
    /* defaults of src/agile.c:158-166 when no options are given */
    agile_opts o = {1.3, 1e-3, 5e-1, 100.0, 0.9, 0.0, 200, 30, 1e-3, 1, 0xC0FFEEULL};
    if (opts) {
        o.mu = opts->mu;
        o.eta_min = opts->eta_min;
        o.eta_max = opts->eta_max;
        o.patience0 = opts->patience0;
        o.patience_decay = opts->patience_decay;
        o.refine_step = opts->refine_step;
        o.refine_max_iters = opts->refine_max_iters;
        o.refine_no_improve = opts->refine_no_improve;
        o.spsa_eps = opts->spsa_eps;
        o.reflect = opts->reflect_at_bounds;
        o.seed = opts->seed;
    }
    agile_report rep;
    if (agile_run(theta0, lower, upper, dim, (loss_fn)loss, ctx, &o, theta_best, &rep) != 0)
        return SPIRES_ERR_INVALID_ARG;
    if (report) {
        report->best_loss = rep.best_loss;
        report->best_iter = rep.best_iter;
        report->total_evals = rep.total_evals;
        report->total_iters = rep.total_iters;
        report->exited_refinement = rep.refined;
    }
    return SPIRES_OK;
}

/* ---- AGILE in ask/tell form: many chains advanced in lockstep ---------------
 * agile_run above drives one chain through a callback. Here each chain is a
 * state machine with the same arithmetic and the same PCG32 draws in the same
 * order; a caller asks every live chain for the points it needs next (two for
 * an SPSA gradient, one for a candidate or refinement step), evaluates them
 * all together (one batched simulation) and tells the losses back. A chain
 * driven this way visits exactly the points agile_run visits with the same
 * options and seed. */
enum { CH_INIT, CH_EXP_A, CH_EXP_B, CH_REF_A, CH_REF_B, CH_DONE };

typedef struct {
    int d, state;
    agile_opts o;
    double lo[64], hi[64];
    double th[64], cand[64], g[64], dir[64], tp[64], tm[64], delta[64], best_theta[64];
    double loss, best, patience, refine_step;
    int since, iters, evals, best_iter, refined, no_imp, k;
    uint64_t rng;
} agile_chain;

/* draws of spsa() before its two evaluations */
static void chain_spsa_points(agile_chain *c)
{
    for (int i = 0; i < c->d; i++) {
        c->delta[i] = (pcg32_next(&c->rng) & 1) ? 1.0 : -1.0;
        c->tp[i] = clampd(c->th[i] + c->o.spsa_eps * c->delta[i], c->lo[i], c->hi[i]);
        c->tm[i] = clampd(c->th[i] - c->o.spsa_eps * c->delta[i], c->lo[i], c->hi[i]);
    }
}

/* rest of spsa() after its evaluations */
static void chain_spsa_grad(agile_chain *c, double fp, double fm)
{
    double scale = (fp - fm) / (2.0 * c->o.spsa_eps);
    for (int i = 0; i < c->d; i++)
        c->g[i] = scale * c->delta[i];
}

static void chain_enter_refine(agile_chain *c)
{
    c->refined = 1;
    memcpy(c->th, c->best_theta, (size_t)c->d * sizeof(double));
    c->loss = c->best;
    c->no_imp = 0;
    c->k = 0;
    if (c->o.refine_max_iters > 0) {
        c->iters++;
        chain_spsa_points(c);
        c->state = CH_REF_A;
    } else {
        c->state = CH_DONE;
    }
}

static void chain_init(agile_chain *c, const double *theta0, const double *lo, const double *hi,
                       int d, const agile_opts *o)
{
    memset(c, 0, sizeof(*c));
    c->d = d;
    c->o = *o;
    memcpy(c->lo, lo, (size_t)d * sizeof(double));
    memcpy(c->hi, hi, (size_t)d * sizeof(double));
    c->refine_step = o->refine_step > 0.0 ? o->refine_step : o->eta_min;
    c->rng = o->seed ? o->seed : 0xA57B17E5ULL;
    memcpy(c->th, theta0, (size_t)d * sizeof(double));
    project(c->th, lo, hi, d, o->reflect);
    c->patience = o->patience0;
    c->state = CH_INIT;
}

/* points the chain needs evaluated now (0, 1 or 2), written to pts */
static int chain_ask(const agile_chain *c, double *pts)
{
    const size_t b = (size_t)c->d * sizeof(double);
    switch (c->state) {
    case CH_INIT:
        memcpy(pts, c->th, b);
        return 1;
    case CH_EXP_A:
    case CH_REF_A:
        memcpy(pts, c->tp, b);
        memcpy(pts + c->d, c->tm, b);
        return 2;
    case CH_EXP_B:
        memcpy(pts, c->cand, b);
        return 1;
    case CH_REF_B:
        memcpy(pts, c->th, b);
        return 1;
    default:
        return 0;
    }
}

static void chain_tell(agile_chain *c, const double *f)
{
    const int d = c->d;
    switch (c->state) {
    case CH_INIT:
        c->loss = f[0];
        c->best = f[0];
        memcpy(c->best_theta, c->th, (size_t)d * sizeof(double));
        c->evals = 1;
        c->iters++;
        chain_spsa_points(c);
        c->state = CH_EXP_A;
        break;
    case CH_EXP_A: {
        chain_spsa_grad(c, f[0], f[1]);
        c->evals += 2;
        double s = 0.0;
        for (int i = 0; i < d; i++)
            s += c->g[i] * c->g[i];
        double gn = sqrt(s);
        if (gn > 1e-18) {
            for (int i = 0; i < d; i++)
                c->dir[i] = (-1.0 / gn) * c->g[i];
        } else {
            double ss = 0.0;
            for (int i = 0; i < d; i++) {
                double z = pcg_uniform(&c->rng) * 2.0 - 1.0;
                c->dir[i] = z;
                ss += z * z;
            }
            double nn = sqrt(ss) + 1e-18;
            for (int i = 0; i < d; i++)
                c->dir[i] /= nn;
        }
        double eta = levy_step(c->o.mu, c->o.eta_min, c->o.eta_max, &c->rng);
        for (int i = 0; i < d; i++)
            c->cand[i] = c->th[i] + eta * c->dir[i];
        project(c->cand, c->lo, c->hi, d, c->o.reflect);
        c->state = CH_EXP_B;
        break;
    }
    case CH_EXP_B: {
        double cl = f[0];
        c->evals++;
        if (cl < c->loss) {
            memcpy(c->th, c->cand, (size_t)d * sizeof(double));
            c->loss = cl;
            c->since = 0;
            c->patience *= c->o.patience_decay;
            if (c->patience < 1.0)
                c->patience = 1.0;
            if (c->loss < c->best) {
                c->best = c->loss;
                c->best_iter = c->iters;
                memcpy(c->best_theta, c->th, (size_t)d * sizeof(double));
            }
        } else {
            c->since++;
        }
        if (c->since >= (int)ceil(c->patience)) {
            chain_enter_refine(c);
        } else if (c->iters > 1000000) {
            c->state = CH_DONE;
        } else {
            c->iters++;
            chain_spsa_points(c);
            c->state = CH_EXP_A;
        }
        break;
    }
    case CH_REF_A:
        chain_spsa_grad(c, f[0], f[1]);
        c->evals += 2;
        for (int i = 0; i < d; i++)
            c->th[i] += -c->refine_step * c->g[i];
        project(c->th, c->lo, c->hi, d, c->o.reflect);
        c->state = CH_REF_B;
        break;
    case CH_REF_B: {
        double nl = f[0];
        c->evals++;
        if (nl < c->loss - 1e-12) {
            c->loss = nl;
            if (c->loss < c->best) {
                c->best = c->loss;
                c->best_iter = c->iters;
                memcpy(c->best_theta, c->th, (size_t)d * sizeof(double));
            }
            c->no_imp = 0;
        } else {
            c->no_imp++;
        }
        c->k++;
        if (c->no_imp >= c->o.refine_no_improve || c->k >= c->o.refine_max_iters) {
            c->state = CH_DONE;
        } else {
            c->iters++;
            chain_spsa_points(c);
            c->state = CH_REF_A;
        }
        break;
    }
    default:
        break;
    }
}

struct spires_ext_agile_batch {
    int chains, dim;
    agile_chain *c;
    int *asked; /* points each chain was asked for in the last ask */
};

static void opts_from_public(agile_opts *o, const spires_ext_agile_opts *p)
{
    agile_opts def = {1.3, 1e-3, 5e-1, 100.0, 0.9, 0.0, 200, 30, 1e-3, 1, 0xC0FFEEULL};
    *o = def;
    if (p) {
        o->mu = p->mu;
        o->eta_min = p->eta_min;
        o->eta_max = p->eta_max;
        o->patience0 = p->patience0;
        o->patience_decay = p->patience_decay;
        o->refine_step = p->refine_step;
        o->refine_max_iters = p->refine_max_iters;
        o->refine_no_improve = p->refine_no_improve;
        o->spsa_eps = p->spsa_eps;
        o->reflect = p->reflect_at_bounds;
        o->seed = p->seed;
    }
}

SPIRES_EXPORT spires_status spires_ext_agile_batch_create(int chains, int dim,
                                                          const double *theta0,
                                                          const double *lower,
                                                          const double *upper,
                                                          const spires_ext_agile_opts *opts,
                                                          const uint64_t *seeds,
                                                          spires_ext_agile_batch **out)
{
    if (!out || chains <= 0 || dim <= 0 || dim > 64 || !theta0 || !lower || !upper)
        return SPIRES_ERR_INVALID_ARG;
    spires_ext_agile_batch *b = calloc(1, sizeof(*b));
    if (!b)
        return SPIRES_ERR_ALLOC;
    b->chains = chains;
    b->dim = dim;
    b->c = calloc((size_t)chains, sizeof(agile_chain));
    b->asked = calloc((size_t)chains, sizeof(int));
    if (!b->c || !b->asked) {
        free(b->c);
        free(b->asked);
        free(b);
        return SPIRES_ERR_ALLOC;
    }
    for (int k = 0; k < chains; k++) {
        agile_opts o;
        opts_from_public(&o, opts);
        if (seeds)
            o.seed = seeds[k];
        chain_init(&b->c[k], theta0 + (size_t)k * dim, lower, upper, dim, &o);
    }
    *out = b;
    return SPIRES_OK;
}

SPIRES_EXPORT void spires_ext_agile_batch_destroy(spires_ext_agile_batch *b)
{
    if (!b)
        return;
    free(b->c);
    free(b->asked);
    free(b);
}

SPIRES_EXPORT int spires_ext_agile_batch_ask(spires_ext_agile_batch *b, double *points,
                                             int *owner)
{
    if (!b || !points)
        return -1;
    int n = 0;
    for (int k = 0; k < b->chains; k++) {
        const int m = chain_ask(&b->c[k], points + (size_t)n * b->dim);
        b->asked[k] = m;
        for (int j = 0; j < m; j++)
            if (owner)
                owner[n + j] = k;
        n += m;
    }
    return n;
}

SPIRES_EXPORT spires_status spires_ext_agile_batch_tell(spires_ext_agile_batch *b,
                                                        const double *losses)
{
    if (!b || !losses)
        return SPIRES_ERR_INVALID_ARG;
    int n = 0;
    for (int k = 0; k < b->chains; k++) {
        if (b->asked[k] > 0)
            chain_tell(&b->c[k], losses + n);
        n += b->asked[k];
        b->asked[k] = 0;
    }
    return SPIRES_OK;
}

SPIRES_EXPORT spires_status spires_ext_agile_batch_best(const spires_ext_agile_batch *b, int chain,
                                                        double *theta,
                                                        spires_ext_agile_report *report)
{
    if (!b || chain < 0 || chain >= b->chains)
        return SPIRES_ERR_INVALID_ARG;
    const agile_chain *c = &b->c[chain];
    if (theta)
        memcpy(theta, c->best_theta, (size_t)c->d * sizeof(double));
    if (report) {
        report->best_loss = c->best;
        report->best_iter = c->best_iter;
        report->total_evals = c->evals;
        report->total_iters = c->iters;
        report->exited_refinement = c->refined;
    }
    return SPIRES_OK;
}

int sp_default_gram_mode(void)
{
    const char *e = getenv("SPIRES_RIDGE_GRAM");
    if (e && (!strcmp(e, "bf16x3") || !strcmp(e, "1")))
        return 1;
    if (e && (!strcmp(e, "tf32x3") || !strcmp(e, "2")))
        return 2;
    if (e && (!strcmp(e, "int8") || !strcmp(e, "3")))
        return 3;
    return 0;
}
