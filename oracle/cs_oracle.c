/*
 * cs_oracle.c -- CPU oracle for the B200 sweep.  TEST INFRASTRUCTURE ONLY: the
 * product library never links this file; tests, the smoke check and bench.py's
 * CPU-baseline leg load it as the checker.
 *
 * Sequential restatement of the reference's per-timestep sweep.  Each function
 * cites the reference code it follows.  Where the GPU design changes *how* a draw is
 * made while keeping its distribution, this file makes the same change so that the
 * two agree state for state:
 *   - random numbers come from counter-based Philox streams keyed by
 *     (seed, step, entity, purpose) instead of per-thread MRG streams;
 *   - a place group's Binomial(n, p) count plus sample without replacement
 *     (src/Sweep.cpp:463-470) is drawn as the equivalent n independent Bernoulli(p)
 *     trials, enumerated by geometric skips;
 *   - a cell's Poisson(sum of spatial infectiousness) contacts with a binary-search
 *     infector choice (src/Sweep.cpp:698-740) is drawn as the equivalent independent
 *     Poisson count per infector;
 *   - the dense cell-to-cell cum_trans/max_trans tables (src/CovidSim.cpp:2779-2800)
 *     are replaced by a block-level proposal with rejection, which samples the same
 *     target distribution (slot chosen with probability proportional to K(d)) without
 *     O(cells^2) storage;
 *   - several infectors reaching one susceptible in a step: the lowest
 *     (infector, infection type) key infects (the reference lets the first queued
 *     infect and the last queued label, src/Sweep.cpp:860-880);
 *   - cell list updates apply the reference's swap-with-block-end rule
 *     (src/Update.cpp:1402-1579) in descending list-position order;
 *   - writes that one person's transition makes to another household member
 *     (adult carer absence, household quarantine) run after all per-person
 *     transitions of the step, once per household.
 */
#include "cs_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define USHRT_MAX_M1 65534
#define MAX_SPATIAL_TRIES 100000
#define MAX_LOOP 1000

/* src/Constants.h:10-58: EARTHRADIUS = (1852*60*360 / PI) / 2 with PI = 3.1415926535 */
static const double ORACLE_PI = 3.1415926535;
#define EARTH_RADIUS (((double)40003200) / 3.1415926535 / 2)

typedef struct place_arrays {
    int32_t n;
    int32_t *mcell, *member_ofs, *members, *group_ofs, *group_start, *group_size;
    float *x, *y;
    uint16_t *close_start, *close_end;
    float* prob_close;
} place_arrays;

struct cs_cpu_ctx {
    cs_params P;
    char err[256];
    /* population */
    int32_t N, NH, NC, NM, NPT, NAD;
    int32_t *hh, *mcell, *place, *hh_first, *mcell_cell, *mcell_adunit, *cell_grid, *cell_start,
        *cell_members;
    uint16_t *group, *hh_nh, *hh_nhr;
    uint8_t *age, *pflags;
    float *hh_x, *hh_y;
    place_arrays pl[CS_MAX_PLACE_TYPES];
    int blanket;                 /* blanket movement restrictions in place this step */
    int cur_ts;                  /* the infect sweep's timestep (false-positive draws) */
    uint8_t* fc;                 /* [N] a false-positive entry this step */
    double rad_origin[2];        /* where infection radii are measured from */
    double *klookup, *khires;
    float *klookup_f, *khires_f;   /* the kernel tables rounded to FP32 (the spatial acceptance test) */
    /* dynamic per person */
    int8_t* inf;
    uint8_t *sev, *dflags;
    uint16_t *infection_time, *latent_time, *recovery_time, *sari_time, *critical_time,
        *stepdown_time, *absent_start, *absent_stop, *isolation_start, *quar_start, *detected_time;
    float *infness, *susc, *prob_absent, *prob_care;
    int32_t *infector, *listpos;
    int16_t* infect_type;
    /* dynamic per cell */
    int32_t *S, *L, *I, *R, *D, *S0, *slots;
    double* tot_prob;
    uint8_t* mark;
    /* microcell interventions */
    uint8_t *socdist, *moverest;
    double ci_dur, hq_dur;
    double *ci_start, *hq_start;   /* [max(1, NAD)]: AdUnits[a].CaseIsolationTimeStart, HQuarantineTimeStart */
    /* spatial proposal blocks */
    int32_t bs, nbx, nby, NB;
    int32_t *cell_block, *block_cell_ofs, *block_cells, *block_cum;
    int64_t* block_S0;
    double* block_row_cum; /* [NB][NB] */
    float* bound_c;        /* [nby][nby][nbx] bound by (row of b, row of B, column distance), FP32 rounded up */
    int bounds_static;     /* 1: bound_c holds every bound; 0: bounds are evaluated per call */
    /* per step scratch */
    uint64_t* claim;
    uint8_t *hh_carer, *hh_hq;
    uint16_t *carer_start, *carer_stop;   /* [NH] place-closure carers' windows (start > stop: none) */
    /* run */
    uint64_t seed;
    int run_started;
    cs_counters C;
};

/* ---------------------------------------------------------------- errors -- */
static int fail(cs_cpu_ctx* c, int code, const char* msg)
{
    if (c) snprintf(c->err, sizeof(c->err), "%s", msg);
    return code;
}
const char* cs_cpu_last_error(const cs_cpu_ctx* c) { return c ? c->err : "null context"; }

/* ------------------------------------------------------------ Philox RNG -- */
static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo)
{
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

void cs_cpu_philox(uint32_t key0, uint32_t key1, const uint32_t ctr[4], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    for (int r = 0; r < 10; r++) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ key0, n1 = lo1, n2 = hi0 ^ c3 ^ key1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        key0 += 0x9E3779B9u;
        key1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

typedef struct stream {
    uint32_t k0, k1, c1, c2, c3, block;
    double buf[2];
    int idx;
} stream;

static void stream_init(stream* s, uint64_t seed, int purpose, uint32_t ts, uint32_t entity, uint32_t sub)
{
    s->k0 = (uint32_t)seed;
    s->k1 = (uint32_t)(seed >> 32);
    s->c1 = entity;
    s->c2 = (ts & 0xffffu) | ((uint32_t)purpose << 16);
    s->c3 = sub;
    s->block = 0;
    s->idx = 2;
}

static double stream_next(stream* s)
{
    if (s->idx >= 2) {
        uint32_t ctr[4] = {s->block++, s->c1, s->c2, s->c3}, x[4];
        cs_cpu_philox(s->k0, s->k1, ctr, x);
        uint64_t a = ((uint64_t)x[1] << 32) | x[0];
        uint64_t b = ((uint64_t)x[3] << 32) | x[2];
        s->buf[0] = (double)(a >> 11) * (1.0 / 9007199254740992.0);
        s->buf[1] = (double)(b >> 11) * (1.0 / 9007199254740992.0);
        s->idx = 0;
    }
    return s->buf[s->idx++];
}

/* -------------------------------------------------------------- samplers -- */
/* Poisson: inversion below 10, else PTRS (Hormann 1993, "The transformed rejection
 * method for generating Poisson random variables").  Same distribution as the
 * reference's ignpoi_mt (Ahrens-Dieter, src/Rand.cpp:170-402). */
static int32_t sample_poisson(stream* s, double lambda, int64_t* err)
{
    if (!(lambda > 0)) return 0;
    if (lambda < 10.0) {
        double u = stream_next(s);
        double p = exp(-lambda), F = p;
        int32_t k = 0;
        while (u > F && k < MAX_LOOP) {
            k++;
            p = p * lambda / (double)k;
            F = F + p;
        }
        return k;
    }
    double slam = sqrt(lambda), loglam = log(lambda);
    double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
    double invalpha = 1.1239 + 1.1328 / (b - 3.4), vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int it = 0; it < MAX_LOOP; it++) {
        double U = stream_next(s) - 0.5;
        double V = stream_next(s);
        double us = 0.5 - fabs(U);
        double k = floor((2.0 * a / us + b) * U + lambda + 0.43);
        if (us >= 0.07 && V <= vr) return (int32_t)k;
        if (k < 0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lambda + k * loglam - lgamma(k + 1.0))
            return (int32_t)k;
    }
    (*err)++;
    return (int32_t)lambda;
}

/* Standard normal by Marsaglia's polar method. */
static double sample_normal(stream* s, int64_t* err)
{
    for (int it = 0; it < MAX_LOOP; it++) {
        double v1 = 2.0 * stream_next(s) - 1.0;
        double v2 = 2.0 * stream_next(s) - 1.0;
        double r = v1 * v1 + v2 * v2;
        if (r > 0.0 && r < 1.0) return v1 * sqrt(-2.0 * log(r) / r);
    }
    (*err)++;
    return 0.0;
}

/* Gamma(shape alpha, rate beta) by Marsaglia-Tsang, as gen_gamma_mt (src/Rand.cpp:1025-1096). */
static double sample_gamma(stream* s, double beta, double alpha, int64_t* err)
{
    double a = (alpha >= 1.0) ? alpha : alpha + 1.0;
    double d = a - (1.0 / 3.0);
    double c = 1.0 / (3.0 * sqrt(d));
    double u, z, v;
    int it = 0;
    do {
        u = stream_next(s);
        z = sample_normal(s, err);
        v = 1.0 + z * c;
        v = v * v * v;
        if (++it > MAX_LOOP) { (*err)++; break; }
    } while ((z <= (-1.0 / c)) || (log(u) >= (0.5 * z * z + d - d * v + d * log(v))));
    double g = (beta != 1.0) ? (d * v) / beta : d * v;
    if (alpha < 1.0) g = g * pow(stream_next(s), 1.0 / alpha);
    return g;
}

/* InverseCdf::choose (src/InverseCdf.cpp:60-74) with its uniform passed in. */
uint16_t cs_cpu_icdf_choose(const cs_icdf* icdf, double mean, double u, double steps_per_day)
{
    double q;
    int i = (int)floor(q = u * CS_CDF_RES);
    q -= (double)i;
    double ti = -mean * log(q * icdf->v[i + 1] + (1.0 - q) * icdf->v[i]);
    return (uint16_t)floor(0.5 + (ti * steps_per_day));
}

static uint16_t choose(const cs_icdf* icdf, double mean, stream* s, double spd)
{
    return cs_cpu_icdf_choose(icdf, mean, stream_next(s), spd);
}

/* ------------------------------------------------------- kernel & distance -- */
static double kernel_eval(int type, double scale, double shape, double p3, double p4, double r2)
{
    /* KernelStruct::* (src/Kernels.cpp:68-106) */
    double t, d;
    switch (type) {
    case 1: return exp(-sqrt(r2) / scale);
    case 2: t = -shape * log(sqrt(r2) / scale + 1.0); return (t < -690.0) ? 0.0 : exp(t);
    case 3: return exp(-r2 / (scale * scale));
    case 4: return (r2 > scale * scale) ? 0.0 : 1.0;
    case 5: t = 0.5 * shape * log(r2 / (scale * scale)); return (t > 690.0) ? 0.0 : (1.0 / (exp(t) + 1.0));
    case 6: t = log(sqrt(r2) / scale + 1.0); return (t < -690.0) ? 0.0 : (exp(-shape * t) + p3 * exp(-p4 * t)) / (1.0 + p3);
    case 7:
        d = sqrt(r2);
        t = -shape * log(d / scale + 1.0);
        return (t < -690.0) ? 0.0 : exp(t - pow(d / p3, p4));
    default: return -1.0;
    }
}

int cs_cpu_build_kernel_table(int kernel_type, double scale, double shape, double p3, double p4,
                              double longest_d2, int size, int expansion, double* lookup_out,
                              double* hi_res_out, double* delta_out)
{
    /* KernelLookup::setup + init(1.0, kernel) (src/Kernels.cpp:8-46) */
    if (kernel_type < 1 || kernel_type > 7 || size < 1 || expansion < 1) return CS_E_ARG;
    double delta = longest_d2 / size;
    for (int i = 0; i <= size; i++) {
        lookup_out[i] = kernel_eval(kernel_type, scale, shape, p3, p4, i * delta) / 1.0;
        hi_res_out[i] = kernel_eval(kernel_type, scale, shape, p3, p4, i * delta / expansion) / 1.0;
    }
    *delta_out = delta;
    return CS_OK;
}

/* KernelLookup::num (src/Kernels.cpp:108-129). */
static double knum(const double* lk, const double* hr, int size, int expansion, double delta, double r2, int64_t* err)
{
    double t = r2 / delta;
    if (t > size) { (*err)++; return 0.0; }
    double s = t * expansion;
    if (s < size) {
        t = s - floor(s);
        t = (1.0 - t) * hr[(int)s] + t * hr[(int)(s + 1.0)];
    } else {
        int i0 = (int)t, i1 = (int)(t + 1.0);
        if (i1 > size) i1 = size;
        s = t - floor(t);
        t = (1.0 - s) * lk[i0] + s * lk[i1];
    }
    return t;
}

double cs_cpu_kernel_num(const cs_cpu_ctx* c, double r2)
{
    int64_t e = 0;
    return knum(c->klookup, c->khires, c->P.kernel_size, c->P.kernel_expansion, c->P.kernel_delta, r2, &e);
}

/* dist2UTM (src/Dist.cpp:23-48). */
static double dist2_utm(const cs_params* P, double x1, double y1, double x2, double y2)
{
    double x, y, cy1, cy2, yt, xi, yi;
    x = fabs(x1 - x2) / 2;
    y = fabs(y1 - y2) / 2;
    xi = floor(x);
    yi = floor(y);
    x -= xi;
    y -= yi;
    x = (1 - x) * P->sinx[(int)xi] + x * P->sinx[((int)xi) + 1];
    y = (1 - y) * P->sinx[(int)yi] + y * P->sinx[((int)yi) + 1];
    yt = fabs(y1 + P->bbox_bottom_left_y);
    yi = floor(yt);
    cy1 = yt - yi;
    cy1 = (1 - cy1) * P->cosx[((int)yi)] + cy1 * P->cosx[((int)yi) + 1];
    yt = fabs(y2 + P->bbox_bottom_left_y);
    yi = floor(yt);
    cy2 = yt - yi;
    cy2 = (1 - cy2) * P->cosx[((int)yi)] + cy2 * P->cosx[((int)yi) + 1];
    x = fabs(1000 * (y * y + x * x * cy1 * cy2));
    xi = floor(x);
    x -= xi;
    y = (1 - x) * P->asin2sqx[((int)xi)] + x * P->asin2sqx[((int)xi) + 1];
    return 4 * EARTH_RADIUS * EARTH_RADIUS * y;
}

/* periodic_xy (src/Dist.cpp:13-21). */
static double periodic_xy(const cs_params* P, double x, double y)
{
    if (P->DoPeriodicBoundaries) {
        if (x > P->width_deg * 0.5) x = P->width_deg - x;
        if (y > P->height_deg * 0.5) y = P->height_deg - y;
    }
    return x * x + y * y;
}

/* dist2_raw (src/Dist.cpp:162-169). */
double cs_cpu_dist2_raw(const cs_params* P, double ax, double ay, double bx, double by)
{
    if (P->DoUTM_coords) return dist2_utm(P, ax, ay, bx, by);
    return periodic_xy(P, fabs(ax - bx), fabs(ay - by));
}

/* dist2(Person*, Person*) (src/Dist.cpp:49-61): household locations are floats; the
 * planar branch subtracts in float. */
static double dist2_hh(const cs_cpu_ctx* c, int32_t ha, int32_t hb)
{
    if (c->P.DoUTM_coords) return dist2_utm(&c->P, c->hh_x[ha], c->hh_y[ha], c->hh_x[hb], c->hh_y[hb]);
    float dx = c->hh_x[ha] - c->hh_x[hb];
    float dy = c->hh_y[ha] - c->hh_y[hb];
    return periodic_xy(&c->P, fabs(dx), fabs(dy));
}

/* dist2_raw (src/Dist.cpp:163-170) from household ha to a point, in double. */
static double dist2_hh_pt(const cs_cpu_ctx* c, int32_t ha, double bx, double by)
{
    return cs_cpu_dist2_raw(&c->P, c->hh_x[ha], c->hh_y[ha], bx, by);
}

/* dist2_cc_min (src/Dist.cpp:78-144) on grid cell indices. */
double cs_cpu_dist2_cc_min(const cs_params* P, int l, int m)
{
    int nch = P->nch, i = l, j = m;
    double x, y;
    if (P->DoUTM_coords) {
        if (P->cell_width * ((double)abs(m / nch - l / nch)) > ORACLE_PI) {
            if (m / nch > l / nch) j += nch;
            else if (m / nch < l / nch) i += nch;
        } else {
            if (m / nch > l / nch) i += nch;
            else if (m / nch < l / nch) j += nch;
        }
        if (m % nch > l % nch) i++;
        else if (m % nch < l % nch) j++;
        return dist2_utm(P, P->cell_width * fabs((double)(i / nch)), P->cell_height * fabs((double)(i % nch)),
                         P->cell_width * fabs((double)(j / nch)), P->cell_height * fabs((double)(j % nch)));
    }
    if ((P->DoPeriodicBoundaries) && (P->cell_width * ((double)abs(m / nch - l / nch)) > P->width_deg * 0.5)) {
        if (m / nch > l / nch) j += nch;
        else if (m / nch < l / nch) i += nch;
    } else {
        if (m / nch > l / nch) i += nch;
        else if (m / nch < l / nch) j += nch;
    }
    if ((P->DoPeriodicBoundaries) && (P->height_deg * ((double)abs(m % nch - l % nch)) > P->height_deg * 0.5)) {
        if (m % nch > l % nch) j++;
        else if (m % nch < l % nch) i++;
    } else {
        if (m % nch > l % nch) i++;
        else if (m % nch < l % nch) j++;
    }
    x = P->cell_width * fabs((double)(i / nch - j / nch));
    y = P->cell_height * fabs((double)(i % nch - j % nch));
    return periodic_xy(P, x, y);
}

/* Upper bound of K(d) for any pair of points in proposal blocks b and B: the kernel
 * at the blocks' closest-corner distance (the block analogue of dist2_cc_min),
 * shrunk by 2% in d^2 so that table interpolation can never push K(d)/bound above 1. */
static double block_bound(const cs_cpu_ctx* c, int b, int B, int64_t* err)
{
    const cs_params* P = &c->P;
    if (P->DoPeriodicBoundaries) return knum(c->klookup, c->khires, P->kernel_size, P->kernel_expansion, P->kernel_delta, 0.0, err);
    int bx = b / c->nby, by = b % c->nby, Bx = B / c->nby, By = B % c->nby;
    int bs = c->bs;
    int xa, xb, ya, yb;
    if (Bx > bx) { xa = (bx + 1) * bs; xb = Bx * bs; }
    else if (Bx < bx) { xa = bx * bs; xb = (Bx + 1) * bs; }
    else { xa = xb = bx * bs; }
    if (By > by) { ya = (by + 1) * bs; yb = By * bs; }
    else if (By < by) { ya = by * bs; yb = (By + 1) * bs; }
    else { ya = yb = by * bs; }
    double d2;
    if (P->DoUTM_coords)
        d2 = dist2_utm(P, P->cell_width * (double)xa, P->cell_height * (double)ya, P->cell_width * (double)xb, P->cell_height * (double)yb);
    else {
        double x = P->cell_width * fabs((double)(xa - xb)), y = P->cell_height * fabs((double)(ya - yb));
        d2 = x * x + y * y;
    }
    d2 = d2 * 0.98;
    return knum(c->klookup, c->khires, P->kernel_size, P->kernel_expansion, P->kernel_delta, d2, err);
}

/* The same bound by (row of b, row of B, column distance dx in blocks), as the GPU
 * library tabulates it once per geometry: the closest corners are dx - 1 blocks
 * apart in x (none for dx = 0) and at the rows' facing edges in y. */
static double block_bound_rel(const cs_cpu_ctx* c, int by, int By, int dx, int64_t* err)
{
    const cs_params* P = &c->P;
    if (P->DoPeriodicBoundaries) return knum(c->klookup, c->khires, P->kernel_size, P->kernel_expansion, P->kernel_delta, 0.0, err);
    const int bs = c->bs, g = dx > 0 ? (dx - 1) * bs : 0;
    int ya, yb;
    if (By > by) { ya = (by + 1) * bs; yb = By * bs; }
    else if (By < by) { ya = by * bs; yb = (By + 1) * bs; }
    else { ya = yb = by * bs; }
    double d2;
    if (P->DoUTM_coords)
        d2 = dist2_utm(P, P->cell_width * (double)g, P->cell_height * (double)ya, 0.0, P->cell_height * (double)yb);
    else {
        double x = P->cell_width * (double)g, y = P->cell_height * fabs((double)(ya - yb));
        d2 = x * x + y * y;
    }
    d2 = d2 * 0.98;
    return knum(c->klookup, c->khires, P->kernel_size, P->kernel_expansion, P->kernel_delta, d2, err);
}

/* Round up to FP32: the nearest float, or the next one up when that is below v. */
static float f32_up(double v)
{
    float f = (float)v;
    if ((double)f < v) f = nextafterf(f, INFINITY);
    return f;
}

/* Tabulate the bounds of the geometry; if any distance falls outside the kernel
 * table they are evaluated (and counted) per call instead, as the GPU library does. */
static void build_bound_table(cs_cpu_ctx* c)
{
    int64_t err = 0;
    const size_t n = (size_t)c->nby * c->nby * c->nbx;
    free(c->bound_c);
    c->bound_c = (float*)calloc(n + 1, sizeof(float));
    for (size_t e = 0; e < n; e++) {
        const int dx = (int)(e % c->nbx), By = (int)((e / c->nbx) % c->nby), by = (int)(e / ((size_t)c->nbx * c->nby));
        c->bound_c[e] = f32_up(block_bound_rel(c, by, By, dx, &err));
    }
    c->bounds_static = err == 0;
}

/* bound(b, B) for the proposal and the acceptance test alike. */
static double bound_of(const cs_cpu_ctx* c, int b, int B, int64_t* err)
{
    if (c->bounds_static) {
        const int bx = b / c->nby, by = b % c->nby, Bx = B / c->nby, By = B % c->nby;
        return (double)c->bound_c[((size_t)by * c->nby + By) * c->nbx + (bx > Bx ? bx - Bx : Bx - bx)];
    }
    return block_bound(c, b, B, err);
}

/* KernelLookup::num over FP32 copies of the tables, interpolated in double. */
static double knum_f32_tab(const float* lk, const float* hr, int size, int expansion, double delta, double r2,
                           int64_t* err)
{
    double t = r2 / delta;
    if (t > size) { (*err)++; return 0.0; }
    double s = t * expansion;
    if (s < size) {
        t = s - floor(s);
        t = (1.0 - t) * (double)hr[(int)s] + t * (double)hr[(int)(s + 1.0)];
    } else {
        int i0 = (int)t, i1 = (int)(t + 1.0);
        if (i1 > size) i1 = size;
        s = t - floor(t);
        t = (1.0 - s) * (double)lk[i0] + s * (double)lk[i1];
    }
    return t;
}

static double knum_f32(const cs_cpu_ctx* c, double r2, int64_t* err)
{
    const cs_params* P = &c->P;
    return knum_f32_tab(c->klookup_f, c->khires_f, P->kernel_size, P->kernel_expansion, P->kernel_delta, r2, err);
}

double cs_cpu_block_bound(const cs_cpu_ctx* c, int b, int B)
{
    int64_t e = 0;
    return bound_of(c, b, B, &e);
}

void cs_cpu_block_geometry(const cs_cpu_ctx* c, int32_t* out)
{
    out[0] = c->bs; out[1] = c->nbx; out[2] = c->nby; out[3] = c->bounds_static;
}

double cs_cpu_kernel_num_f32(const float* lookup, const float* hi_res, int size, int expansion, double delta, double r2)
{
    int64_t e = 0;
    return knum_f32_tab(lookup, hi_res, size, expansion, delta, r2, &e);
}

/* ---------------------------------------------------------- state macros -- */
/* src/ModelMacros.h:6-20 */
static inline int age_group(const cs_cpu_ctx* c, int p) { return c->age[p] / CS_AGE_GROUP_WIDTH; }
static inline int host_absent(const cs_cpu_ctx* c, int p, int ts) { return c->absent_start[p] <= ts && c->absent_stop[p] > ts; }
static inline int quar_comply(const cs_cpu_ctx* c, int p) { return (c->dflags[p] & CS_DF_QUAR_COMPLY_MASK) >> CS_DF_QUAR_COMPLY_SHIFT; }
static inline int host_quarantined(const cs_cpu_ctx* c, int p, int ts)
{
    return quar_comply(c, p) == 1 && (int)c->quar_start[p] + (int)c->P.usHQuarantineHouseDuration > ts && c->quar_start[p] <= ts;
}
static inline int host_to_be_quarantined(const cs_cpu_ctx* c, int p, int ts)
{
    return (int)c->quar_start[p] + (int)c->P.usHQuarantineHouseDuration > ts && quar_comply(c, p) < 2;
}
static inline int host_isolated(const cs_cpu_ctx* c, int p, int ts)
{
    int s = (int)c->isolation_start[p] + (int)c->P.usCaseIsolationDelay;
    return s <= ts && s + (int)c->P.usCaseIsolationDuration > ts;
}
static inline int place_closed(const cs_cpu_ctx* c, int pt, int pl, int ts)
{
    return c->pl[pt].close_start[pl] <= ts && c->pl[pt].close_end[pl] > ts;
}
static inline int is_ch(const cs_cpu_ctx* c, int p) { return (c->pflags[p] & CS_PF_CARE_HOME_RESIDENT) != 0; }
static inline int is_alive(const cs_cpu_ctx* c, int p) { return c->inf[p] != CS_INF_DEAD_WAS_ASYMP && c->inf[p] != CS_INF_DEAD_WAS_SYMP; }
static inline int link_of(const cs_cpu_ctx* c, int pt, int p) { return c->place[(size_t)pt * c->N + p]; }
static inline int group_of(const cs_cpu_ctx* c, int pt, int p) { return c->group[(size_t)pt * c->N + p]; }
static inline int cell_of(const cs_cpu_ctx* c, int p) { return c->mcell_cell[c->mcell[p]]; }

/* ------------------------------------------------ CalcInfSusc (src/CalcInfSusc.cpp) */
/* Factors that are exactly 1.0 in this sweep (digital contact tracing, treatment,
 * vaccination) are omitted: multiplying by 1.0 is exact, so the products agree bit
 * for bit with the reference's. */
static double calc_person_inf(const cs_cpu_ctx* c, int p, int ts)
{
    return fabs(c->infness[p]) * c->P.infectiousness[ts - c->latent_time[p] - 1];
}
static double calc_house_inf(const cs_cpu_ctx* c, int p, int ts)
{
    const cs_params* P = &c->P;
    int iso = host_isolated(c, p, ts);
    double infn = P->NoInfectiousnessSDinHH ? ((c->infness[p] < 0) ? P->SymptInfectiousness : P->AsymptInfectiousness) : fabs(c->infness[p]);
    return (iso ? P->Efficacies[CS_NPI_CASE_ISOLATION][CS_SETTING_HOUSE] : 1.0)
        * ((host_quarantined(c, p, ts) && !iso) ? P->Efficacies[CS_NPI_HOME_QUARANTINE][CS_SETTING_HOUSE] : 1.0)
        * P->HouseholdDenomLookup[c->hh_nhr[c->hh[p]] - 1]
        * (is_ch(c, p) ? P->CareHomeResidentHouseholdScaling : 1.0)
        * infn
        * P->infectiousness[ts - c->latent_time[p] - 1];
}
static double calc_place_inf(const cs_cpu_ctx* c, int p, int pt, int ts)
{
    const cs_params* P = &c->P;
    int iso = host_isolated(c, p, ts), ch = is_ch(c, p);
    return (iso ? P->Efficacies[CS_NPI_CASE_ISOLATION][pt] : 1.0)
        * ((host_quarantined(c, p, ts) && !ch && !iso) ? P->Efficacies[CS_NPI_HOME_QUARANTINE][pt] : 1.0)
        * ((c->inf[p] == CS_INF_CASE && !ch) ? P->SymptPlaceTypeContactRate[pt] : 1.0)
        * P->PlaceTypeTrans[pt] / P->PlaceTypeGroupSizeParam1[pt] * calc_person_inf(c, p, ts);
}
static double calc_spatial_inf(const cs_cpu_ctx* c, int p, int ts)
{
    const cs_params* P = &c->P;
    int iso = host_isolated(c, p, ts), ch = is_ch(c, p);
    return (iso ? P->Efficacies[CS_NPI_CASE_ISOLATION][CS_SETTING_SPATIAL] : 1.0)
        * ((host_quarantined(c, p, ts) && !ch && !iso) ? P->Efficacies[CS_NPI_HOME_QUARANTINE][CS_SETTING_SPATIAL] : 1.0)
        * ((c->inf[p] == CS_INF_CASE) ? P->SymptSpatialContactRate : 1.0)
        * P->RelativeSpatialContact[age_group(c, p)]
        * calc_person_inf(c, p, ts);
}
static double calc_person_susc(const cs_cpu_ctx* c, int p, int infector)
{
    const cs_params* P = &c->P;
    return P->WAIFW_Matrix[age_group(c, p)][age_group(c, infector)] * P->AgeSusceptibility[age_group(c, p)] * c->susc[p];
}
static double socdist_factor(const cs_cpu_ctx* c, int p, int setting)
{
    if (c->socdist[c->mcell[p]] != CS_TREAT_TREATED) return 1.0;
    return (c->pflags[p] & CS_PF_ESOCDIST_COMPLY) ? c->P.Efficacies[CS_NPI_ENHANCED_SOCIAL_DISTANCING][setting]
                                                  : c->P.Efficacies[CS_NPI_SOCIAL_DISTANCING][setting];
}
static double calc_house_susc(const cs_cpu_ctx* c, int p, int ts, int infector)
{
    (void)ts;
    return calc_person_susc(c, p, infector) * socdist_factor(c, p, CS_SETTING_HOUSE)
        * (is_ch(c, p) ? c->P.CareHomeResidentHouseholdScaling : 1.0);
}
static double calc_place_susc(const cs_cpu_ctx* c, int p, int pt, int ts)
{
    return ((host_quarantined(c, p, ts) && !is_ch(c, p)) ? c->P.Efficacies[CS_NPI_HOME_QUARANTINE][pt] : 1.0)
        * socdist_factor(c, p, pt);
}
static double calc_spatial_susc(const cs_cpu_ctx* c, int p, int ts)
{
    return ((host_quarantined(c, p, ts) && !is_ch(c, p)) ? c->P.Efficacies[CS_NPI_HOME_QUARANTINE][CS_SETTING_SPATIAL] : 1.0)
        * socdist_factor(c, p, CS_SETTING_SPATIAL)
        * c->P.RelativeSpatialContactSusc[age_group(c, p)];
}
static int moverest_differs(const cs_cpu_ctx* c, int ma, int mb)
{
    return c->moverest[ma] != c->moverest[mb] && (c->moverest[ma] == CS_TREAT_TREATED || c->moverest[mb] == CS_TREAT_TREATED);
}

/* --------------------------------------------------------------- setup -- */
#define DUP(dst, src, n, T) do { dst = (T*)malloc(sizeof(T) * (size_t)(n) + 1); if ((n) > 0) memcpy(dst, src, sizeof(T) * (size_t)(n)); } while (0)
#define ALLOC(dst, n, T) do { dst = (T*)calloc((size_t)(n) + 1, sizeof(T)); } while (0)

static void build_blocks(cs_cpu_ctx* c)
{
    const cs_params* P = &c->P;
    /* Proposal blocks: the smallest square of cells that keeps the block-pair table
     * at or below 4096 x 4096 entries, unless the parameters fix the size. */
    int bs = P->block_cells;
    if (bs <= 0) {
        bs = 1;
        while (((P->ncw + bs - 1) / bs) * ((P->nch + bs - 1) / bs) > 4096) bs++;
    }
    c->bs = bs;
    c->nbx = (P->ncw + bs - 1) / bs;
    c->nby = (P->nch + bs - 1) / bs;
    c->NB = c->nbx * c->nby;
    ALLOC(c->cell_block, c->NC, int32_t);
    ALLOC(c->block_cell_ofs, c->NB + 1, int32_t);
    ALLOC(c->block_cells, c->NC, int32_t);
    ALLOC(c->block_cum, c->NC, int32_t);
    ALLOC(c->block_S0, c->NB, int64_t);
    c->block_row_cum = (double*)calloc((size_t)c->NB * c->NB + 1, sizeof(double));
    for (int m = 0; m < c->NC; m++) {
        int g = c->cell_grid[m], x = g / P->nch, y = g % P->nch;
        c->cell_block[m] = (x / bs) * c->nby + (y / bs);
        c->block_cell_ofs[c->cell_block[m] + 1]++;
    }
    for (int b = 0; b < c->NB; b++) c->block_cell_ofs[b + 1] += c->block_cell_ofs[b];
    int32_t* fill = (int32_t*)calloc((size_t)c->NB + 1, sizeof(int32_t));
    for (int m = 0; m < c->NC; m++) {
        int b = c->cell_block[m];
        c->block_cells[c->block_cell_ofs[b] + fill[b]++] = m;
    }
    free(fill);
    c->klookup_f = (float*)calloc((size_t)P->kernel_size + 2, sizeof(float));
    c->khires_f = (float*)calloc((size_t)P->kernel_size + 2, sizeof(float));
    for (int i = 0; i <= P->kernel_size; i++) {
        c->klookup_f[i] = (float)c->klookup[i];
        c->khires_f[i] = (float)c->khires[i];
    }
    build_bound_table(c);
}

int cs_cpu_create(const cs_population* pop, const cs_params* params, cs_cpu_ctx** out)
{
    if (!pop || !params || !out) return CS_E_ARG;
    cs_cpu_ctx* c = (cs_cpu_ctx*)calloc(1, sizeof(cs_cpu_ctx));
    c->P = *params;
    c->rad_origin[0] = params->LocationInitialInfection[0];
    c->rad_origin[1] = params->LocationInitialInfection[1];
    c->N = pop->n_people; c->NH = pop->n_households; c->NC = pop->n_cells; c->NM = pop->n_mcells;
    c->NPT = pop->num_place_types; c->NAD = pop->n_adunits;
    if (c->NPT > CS_MAX_PLACE_TYPES || c->NPT != params->NumPlaceTypes) { *out = c; return fail(c, CS_E_ARG, "place type count mismatch"); }
    DUP(c->hh, pop->person_hh, c->N, int32_t);
    DUP(c->mcell, pop->person_mcell, c->N, int32_t);
    DUP(c->age, pop->person_age, c->N, uint8_t);
    DUP(c->pflags, pop->person_flags, c->N, uint8_t);
    DUP(c->place, pop->person_place, (size_t)c->NPT * c->N, int32_t);
    DUP(c->group, pop->person_group, (size_t)c->NPT * c->N, uint16_t);
    DUP(c->hh_first, pop->hh_first, c->NH, int32_t);
    DUP(c->hh_nh, pop->hh_nh, c->NH, uint16_t);
    DUP(c->hh_nhr, pop->hh_nhr, c->NH, uint16_t);
    DUP(c->hh_x, pop->hh_x, c->NH, float);
    DUP(c->hh_y, pop->hh_y, c->NH, float);
    DUP(c->mcell_cell, pop->mcell_cell, c->NM, int32_t);
    DUP(c->mcell_adunit, pop->mcell_adunit, c->NM, int32_t);
    DUP(c->cell_grid, pop->cell_grid, c->NC, int32_t);
    DUP(c->cell_start, pop->cell_start, c->NC + 1, int32_t);
    DUP(c->cell_members, pop->cell_members, c->N, int32_t);
    for (int t = 0; t < c->NPT; t++) {
        place_arrays* p = &c->pl[t];
        p->n = pop->n_places[t];
        int nm = pop->place_member_ofs[t][p->n], ng = pop->place_group_ofs[t][p->n];
        DUP(p->mcell, pop->place_mcell[t], p->n, int32_t);
        DUP(p->x, pop->place_x[t], p->n, float);
        DUP(p->y, pop->place_y[t], p->n, float);
        DUP(p->member_ofs, pop->place_member_ofs[t], p->n + 1, int32_t);
        DUP(p->members, pop->place_members[t], nm, int32_t);
        DUP(p->group_ofs, pop->place_group_ofs[t], p->n + 1, int32_t);
        DUP(p->group_start, pop->group_start[t], ng, int32_t);
        DUP(p->group_size, pop->group_size[t], ng, int32_t);
        ALLOC(p->close_start, p->n, uint16_t);
        ALLOC(p->close_end, p->n, uint16_t);
        ALLOC(p->prob_close, p->n, float);
    }
    DUP(c->klookup, pop->kernel_lookup, params->kernel_size + 1, double);
    DUP(c->khires, pop->kernel_hi_res, params->kernel_size + 1, double);
    ALLOC(c->inf, c->N, int8_t); ALLOC(c->sev, c->N, uint8_t); ALLOC(c->dflags, c->N, uint8_t);
    ALLOC(c->infection_time, c->N, uint16_t); ALLOC(c->latent_time, c->N, uint16_t);
    ALLOC(c->recovery_time, c->N, uint16_t); ALLOC(c->sari_time, c->N, uint16_t);
    ALLOC(c->critical_time, c->N, uint16_t); ALLOC(c->stepdown_time, c->N, uint16_t);
    ALLOC(c->absent_start, c->N, uint16_t); ALLOC(c->absent_stop, c->N, uint16_t);
    ALLOC(c->isolation_start, c->N, uint16_t); ALLOC(c->quar_start, c->N, uint16_t);
    ALLOC(c->detected_time, c->N, uint16_t);
    ALLOC(c->infness, c->N, float); ALLOC(c->susc, c->N, float);
    ALLOC(c->prob_absent, c->N, float); ALLOC(c->prob_care, c->N, float);
    ALLOC(c->infector, c->N, int32_t); ALLOC(c->listpos, c->N, int32_t); ALLOC(c->infect_type, c->N, int16_t);
    ALLOC(c->S, c->NC, int32_t); ALLOC(c->L, c->NC, int32_t); ALLOC(c->I, c->NC, int32_t);
    ALLOC(c->R, c->NC, int32_t); ALLOC(c->D, c->NC, int32_t); ALLOC(c->S0, c->NC, int32_t);
    ALLOC(c->tot_prob, c->NC, double); ALLOC(c->slots, c->N, int32_t); ALLOC(c->mark, c->N, uint8_t);
    ALLOC(c->socdist, c->NM, uint8_t); ALLOC(c->moverest, c->NM, uint8_t);
    ALLOC(c->claim, c->N, uint64_t);
    ALLOC(c->hh_carer, c->NH, uint8_t); ALLOC(c->hh_hq, c->NH, uint8_t);
    ALLOC(c->fc, c->N, uint8_t);
    ALLOC(c->carer_start, c->NH, uint16_t); ALLOC(c->carer_stop, c->NH, uint16_t);
    for (int h = 0; h < c->NH; h++) c->carer_start[h] = 0xFFFF;
    ALLOC(c->ci_start, c->NAD, double); ALLOC(c->hq_start, c->NAD, double);
    for (int a = 0; a <= c->NAD; a++) c->ci_start[a] = c->hq_start[a] = 1e10;
    for (int i = 0; i < c->N; i++) c->claim[i] = UINT64_MAX;
    build_blocks(c);
    *out = c;
    return CS_OK;
}

void cs_cpu_destroy(cs_cpu_ctx* c)
{
    if (!c) return;
    void* ptrs[] = {c->hh, c->mcell, c->age, c->pflags, c->place, c->group, c->hh_first, c->hh_nh, c->hh_nhr,
                    c->hh_x, c->hh_y, c->mcell_cell, c->mcell_adunit, c->cell_grid, c->cell_start, c->cell_members,
                    c->klookup, c->khires, c->inf, c->sev, c->dflags, c->infection_time, c->latent_time,
                    c->recovery_time, c->sari_time, c->critical_time, c->stepdown_time, c->absent_start,
                    c->absent_stop, c->isolation_start, c->quar_start, c->detected_time, c->infness, c->susc,
                    c->prob_absent, c->prob_care, c->infector, c->listpos, c->infect_type, c->S, c->L, c->I,
                    c->R, c->D, c->S0, c->tot_prob, c->slots, c->mark, c->socdist, c->moverest, c->claim,
                    c->hh_carer, c->hh_hq, c->cell_block, c->block_cell_ofs, c->block_cells, c->block_cum,
                    c->block_S0, c->block_row_cum, c->ci_start, c->hq_start, c->carer_start, c->carer_stop,
                    c->klookup_f, c->khires_f, c->bound_c, c->fc};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    for (int t = 0; t < c->NPT; t++) {
        place_arrays* p = &c->pl[t];
        free(p->mcell); free(p->x); free(p->y); free(p->member_ofs); free(p->members); free(p->group_ofs);
        free(p->group_start); free(p->group_size); free(p->close_start); free(p->close_end); free(p->prob_close);
    }
    free(c);
}

int cs_cpu_set_params(cs_cpu_ctx* c, const cs_params* params)
{
    if (params->kernel_size != c->P.kernel_size || params->NumPlaceTypes != c->P.NumPlaceTypes)
        return fail(c, CS_E_ARG, "set_params may not change the kernel table or place types");
    c->P = *params;
    build_bound_table(c);   /* the bounds depend on the geometry the parameters carry */
    return CS_OK;
}

/* Proposal tables from the current S0: per block its S0 total and the running S0
 * of its cells; per source block the running sum over target blocks of
 * S0_B * bound(b, B). */
static void rebuild_block_tables(cs_cpu_ctx* c)
{
    int64_t err = 0;
    for (int B = 0; B < c->NB; B++) {
        int64_t s = 0;
        for (int k = c->block_cell_ofs[B]; k < c->block_cell_ofs[B + 1]; k++) {
            s += c->S0[c->block_cells[k]];
            c->block_cum[k] = (int32_t)s;
        }
        c->block_S0[B] = s;
    }
    for (int b = 0; b < c->NB; b++) {
        double* row = c->block_row_cum + (size_t)b * c->NB;
        double s = 0.0;
        for (int B = 0; B < c->NB; B++) {
            double w = (c->block_S0[B] > 0) ? (double)c->block_S0[B] * bound_of(c, b, B, &err) : 0.0;
            s = s + w;
            row[B] = s;
        }
    }
    c->C.err_kernel_range += err;
}

/* --------------------------------------------------------- UpdateProbs -- */
/* Kmax between source row yl and target row ym at column distance dx: the
 * closest-corner rule of dist2_cc_min (src/Dist.cpp:78-144) written in terms of
 * (dx, yl, ym), which is all the distance depends on. */
static double row_kernel(const cs_cpu_ctx* c, int dx, int yl, int ym, int64_t* err)
{
    const cs_params* P = &c->P;
    int y1 = yl, y2 = ym;
    if (ym > yl) y1 = yl + 1;
    else if (ym < yl) y2 = ym + 1;
    double d2;
    if (P->DoUTM_coords) {
        int cx = (dx == 0) ? 0 : ((P->cell_width * (double)dx > ORACLE_PI) ? dx + 1 : dx - 1);
        d2 = dist2_utm(P, 0.0, P->cell_height * (double)y1, P->cell_width * (double)cx, P->cell_height * (double)y2);
    } else {
        int cx = (dx == 0) ? 0 : (((P->DoPeriodicBoundaries) && (P->cell_width * (double)dx > P->width_deg * 0.5)) ? dx + 1 : dx - 1);
        int dy = abs(ym - yl), cy = (dy == 0) ? 0 : dy - 1;
        if ((P->DoPeriodicBoundaries) && (P->height_deg * (double)dy > P->height_deg * 0.5)) cy = dy + 1;
        d2 = periodic_xy(P, P->cell_width * (double)cx, P->cell_height * (double)cy);
    }
    return (double)(float)knum(c->klookup, c->khires, P->kernel_size, P->kernel_expansion, P->kernel_delta, d2, err);
}

/* UpdateProbs (src/CovidSim.cpp:2752-2802): S0 per cell, then
 * tot_prob = sum_m S0_m Kmax(l,m) / sum_m n_m Kmax(l,m) with
 * Kmax = (float)num(dist2_cc_min), summed in float (as the reference's float
 * cum_trans sums, src/CovidSim.cpp:2785-2795) in a fixed order: over target
 * rows ym ascending, each row's sum over target columns xm ascending formed first
 * with fused multiply-adds (one rounding per term); row sums added within chunks
 * of TOT_PROB_ROW_CHUNK rows, chunk sums added in ascending order; zero terms are
 * skipped (adding +0.0 changes nothing). */
#define TOT_PROB_ROW_CHUNK 32
int cs_cpu_update_probs(cs_cpu_ctx* c, int do_place)
{
    const cs_params* P = &c->P;
    int64_t err = 0;
    for (int j = 0; j < c->NC; j++) {
        int n = c->cell_start[j + 1] - c->cell_start[j];
        if (!do_place) {
            c->S0[j] = c->S[j] + c->L[j] + c->I[j];
            if (P->DoDeathCountsInS0) {
                c->S0[j] += n / 5;
                if ((n < 100) || (c->S0[j] > n)) c->S0[j] = n;
            }
        } else c->S0[j] = c->S[j];
    }
    int ncw = P->ncw, nch = P->nch;
    size_t G = (size_t)ncw * nch;
    float* S0g = (float*)calloc(G, sizeof(float));
    float* Ng = (float*)calloc(G, sizeof(float));
    float* krow = (float*)malloc(sizeof(float) * ncw);
    for (int m = 0; m < c->NC; m++) {
        S0g[c->cell_grid[m]] = (float)c->S0[m];
        Ng[c->cell_grid[m]] = (float)(c->cell_start[m + 1] - c->cell_start[m]);
    }
    for (int l = 0; l < c->NC; l++) {
        int xl = c->cell_grid[l] / nch, yl = c->cell_grid[l] % nch;
        float A = 0.f, B = 0.f;
        for (int q0 = 0; q0 < nch; q0 += TOT_PROB_ROW_CHUNK) {
            float a = 0.f, b = 0.f;
            int q1 = q0 + TOT_PROB_ROW_CHUNK < nch ? q0 + TOT_PROB_ROW_CHUNK : nch;
            for (int ym = q0; ym < q1; ym++) {
                int anyS = 0, anyN = 0;
                for (int xm = 0; xm < ncw; xm++) {
                    anyS |= S0g[(size_t)xm * nch + ym] != 0.f;
                    anyN |= Ng[(size_t)xm * nch + ym] != 0.f;
                }
                if (!anyS && !anyN) continue;
                for (int k = 0; k < ncw; k++) krow[k] = (float)row_kernel(c, k, yl, ym, &err);
                float s = 0.f, sb = 0.f;
                for (int xm = 0; xm < ncw; xm++) {
                    int dd = xm > xl ? xm - xl : xl - xm;
                    float sv = S0g[(size_t)xm * nch + ym], nv = Ng[(size_t)xm * nch + ym];
                    if (sv != 0.f) s = fmaf(sv, krow[dd], s);
                    if (nv != 0.f) sb = fmaf(nv, krow[dd], sb);
                }
                if (anyS) a = a + s;
                if (anyN) b = b + sb;
            }
            A = A + a;
            B = B + b;
        }
        c->tot_prob[l] = (B > 0) ? (double)A / (double)B : 0.0;
    }
    free(S0g);
    free(Ng);
    free(krow);
    rebuild_block_tables(c);
    c->C.err_kernel_range += err;
    return CS_OK;
}

/* ------------------------------------------------------------ run start -- */
static void partition_block(cs_cpu_ctx* c, int cell, int b0, int n, int* removed_out);
static void do_detected_case(cs_cpu_ctx* c, int p, double t, int ts);

/* ToInfected + DoInfect (src/Update.cpp:100-195, 1531-1538) for one person, without
 * the cell-list move (done per cell afterwards). */
static void do_infect(cs_cpu_ctx* c, int p, double t, int ts, int32_t infector, int16_t infect_type)
{
    const cs_params* P = &c->P;
    c->inf[p] = CS_INF_LATENT;
    c->infection_time[p] = (uint16_t)ts;
    c->infector[p] = infector;
    c->infect_type[p] = infect_type;
    int cell = cell_of(c, p);
    c->S[cell]--; c->L[cell]++;
    c->mark[c->cell_start[cell] + c->listpos[p]] = 1;
    c->C.cumI++;
    if (infector != -2) {   /* a seed's radius is 0: the origin moved to it */
        const double x = (double)c->hh_x[c->hh[p]] - c->rad_origin[0], y = (double)c->hh_y[c->hh[p]] - c->rad_origin[1];
        const double r2 = x * x + y * y;
        int64_t bits;
        c->C.sumRad2_q += (int64_t)(r2 * 4294967296.0);
        memcpy(&bits, &r2, sizeof bits);
        if (bits > c->C.maxRad2_bits) c->C.maxRad2_bits = bits;
    }
    c->C.cumItype[infect_type % CS_INFECT_TYPE_MASK]++;
    c->C.cumIa[age_group(c, p)]++;
    c->C.cumI_keyworker[(c->pflags[p] & CS_PF_KEYWORKER) ? 1 : 0]++;
    int ad = c->mcell_adunit[c->mcell[p]];
    if (ad >= 0 && ad < CS_MAX_ADUNITS) c->C.cumI_adunit[ad]++;
    if (P->DoLatent) {
        stream s;
        stream_init(&s, c->seed, CS_RNG_LATENT, (uint32_t)ts, (uint32_t)p, 0);
        double q;
        int i = (int)floor((q = stream_next(&s) * CS_CDF_RES));
        q -= (double)i;
        c->latent_time[p] = (uint16_t)floor(0.5 + (t - P->LatentPeriod * log(q * P->latent_icdf.v[i + 1] + (1.0 - q) * P->latent_icdf.v[i])) * P->TimeStepsPerDay);
    } else
        c->latent_time[p] = (uint16_t)(t * P->TimeStepsPerDay);
    if (infector >= 0) {
        c->C.cumTG += ((int)c->infection_time[p]) - ((int)c->infection_time[infector]);
        c->C.cumSI += ((int)c->latent_time[p]) - ((int)c->latent_time[infector]);
        c->C.nTG++;
    }
    c->C.work_new_infections++;
}

/* Move every marked slot of the S block of each touched cell to the front of its
 * latent block (SusceptibleToLatent + UpdateCell, src/Update.cpp:128-136). */
static void partition_S_blocks(cs_cpu_ctx* c, const int32_t* touched, int ntouched)
{
    c->C.work_cells_touched += ntouched;
    for (int k = 0; k < ntouched; k++) {
        int cell = touched[k];
        /* S has already been decremented; the pre-update S block is S + L_new_marks,
         * recovered as the range that still holds marks: S_old = S + (#marks). */
        int b0 = c->cell_start[cell];
        int nmark = 0;
        int n = c->cell_start[cell + 1] - b0;
        for (int i = 0; i < n; i++) nmark += c->mark[b0 + i];
        partition_block(c, cell, b0, c->S[cell] + nmark, NULL);
    }
}

int cs_cpu_seed_infections(cs_cpu_ctx* c, double t, const int32_t* people, int n)
{
    int ts = (int)(uint16_t)(c->P.TimeStepsPerDay * t);
    int32_t* touched = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
    int nt = 0;
    for (int k = 0; k < n; k++) {
        int p = people[k];
        if (p < 0 || p >= c->N) { free(touched); return fail(c, CS_E_ARG, "seed person out of range"); }
        if (c->inf[p] != CS_INF_SUSCEPTIBLE) continue;
        do_infect(c, p, t, ts, -2, (int16_t)(CS_INFECT_TYPE_MASK - 1));
        touched[nt++] = cell_of(c, p);
    }
    /* radii are measured from the last seed's household (src/CovidSim.cpp:1358-1359) */
    if (n > 0) {
        c->rad_origin[0] = (double)c->hh_x[c->hh[people[n - 1]]];
        c->rad_origin[1] = (double)c->hh_y[c->hh[people[n - 1]]];
    }
    /* unique cells */
    for (int i = 0; i < nt; i++)
        for (int j = i + 1; j < nt; j++)
            if (touched[j] == touched[i]) { touched[j] = touched[--nt]; j--; }
    partition_S_blocks(c, touched, nt);
    free(touched);
    return CS_OK;
}

/* Run-level state outside the per-person view, as InitModel sets it: place
 * closures and each place's closure threshold (src/CovidSim.cpp:1110-1125),
 * social-distancing and movement flags, intervention windows. */
static void reset_run_level(cs_cpu_ctx* c, uint64_t seed)
{
    for (int t = 0; t < c->NPT; t++)
        for (int l = 0; l < c->pl[t].n; l++) {
            stream s;
            stream_init(&s, seed, CS_RNG_PLACE_INIT, 0, (uint32_t)l, (uint32_t)t);
            c->pl[t].close_start[l] = USHRT_MAX_M1;
            c->pl[t].close_end[l] = 0;
            c->pl[t].prob_close[l] = (float)stream_next(&s);
        }
    memset(c->socdist, 0, (size_t)c->NM);
    memset(c->moverest, 0, (size_t)c->NM);
    for (int a = 0; a <= c->NAD; a++) c->ci_start[a] = c->hq_start[a] = 1e10;
    c->ci_dur = c->hq_dur = 0;
}

int cs_cpu_begin_run(cs_cpu_ctx* c, uint64_t seed, const int32_t* seed_people, int n_seed, int update_probs)
{
    c->seed = seed;
    memset(&c->C, 0, sizeof(c->C));
    /* InitModel person resets (src/CovidSim.cpp:1006-1040) */
    for (int p = 0; p < c->N; p++) {
        stream s;
        stream_init(&s, seed, CS_RNG_RUN_INIT, 0, (uint32_t)p, 0);
        c->inf[p] = CS_INF_SUSCEPTIBLE;
        c->sev[p] = CS_SEV_ASYMPTOMATIC | (CS_SEV_ASYMPTOMATIC << 4);
        c->dflags[p] = (uint8_t)(2u << CS_DF_QUAR_COMPLY_SHIFT);
        c->infection_time[p] = 0; c->latent_time[p] = 0; c->recovery_time[p] = 0;
        c->sari_time[p] = c->critical_time[p] = c->stepdown_time[p] = USHRT_MAX_M1;
        c->absent_start[p] = USHRT_MAX_M1; c->absent_stop[p] = 0;
        c->isolation_start[p] = USHRT_MAX_M1; c->quar_start[p] = USHRT_MAX_M1; c->detected_time[p] = 0;
        c->infness[p] = 0.0f;
        c->susc[p] = 1.0f;
        c->prob_absent[p] = (float)stream_next(&s);
        c->prob_care[p] = (float)stream_next(&s);
        c->infector[p] = -1; c->infect_type[p] = 0;
    }
    /* cell lists (src/CovidSim.cpp:1042-1094) */
    for (int j = 0; j < c->NC; j++) {
        int b0 = c->cell_start[j], n = c->cell_start[j + 1] - b0;
        for (int i = 0; i < n; i++) {
            c->slots[b0 + i] = c->cell_members[b0 + i];
            c->listpos[c->cell_members[b0 + i]] = i;
            c->mark[b0 + i] = 0;
        }
        c->S[j] = n; c->L[j] = c->I[j] = c->R[j] = c->D[j] = 0;
        c->S0[j] = n;
        c->tot_prob[j] = 1.0;
    }
    reset_run_level(c, seed);
    c->run_started = 1;
    /* At a run start every cell is wholly susceptible, so UpdateProbs(0) gives
     * S0 = n and tot_prob = 1 exactly; only the proposal tables need rebuilding. */
    (void)update_probs;
    rebuild_block_tables(c);
    return cs_cpu_seed_infections(c, 0.0, seed_people, n_seed);
}

/* ------------------------------------------------------- cell list moves -- */
/* Remove every marked slot of block [b0, b0+n) by swapping it with the block's last
 * element, visiting positions from high to low: the sequence of UpdateCell calls the
 * reference makes (src/Update.cpp:128-136, 509-516, 918-925, 964-969) when the
 * transitions of a cell are processed in descending list order.  Marks are cleared. */
static void partition_block(cs_cpu_ctx* c, int cell, int b0, int n, int* removed_out)
{
    int base = c->cell_start[cell];
    int cur = n, removed = 0;
    for (int pos = b0 + n - 1; pos >= b0; pos--) {
        if (!c->mark[pos]) continue;
        cur--;
        removed++;
        int end = b0 + cur;
        if (pos < end) {
            int a = c->slots[pos], e = c->slots[end];
            c->slots[pos] = e;
            c->listpos[e] = pos - base;
            c->slots[end] = a;
            c->listpos[a] = end - base;
            c->mark[end] = 0;
        }
        c->mark[pos] = 0;
        c->mark[end] = 0;
    }
    if (removed_out) *removed_out = removed;
}

/* ------------------------------------------------------------- InfectSweep -- */
/* AddInfections (src/Sweep.cpp:2031-2065): with probability FalsePositiveRate the
 * entry is a false positive (DoFalseCase for the person) instead of an infection,
 * one draw per entry keyed by (infector, infectee, infection type). */
static inline void claim(cs_cpu_ctx* c, int person, int infector, int code)
{
    if (c->P.FalsePositiveRate > 0) {
        stream s;
        stream_init(&s, c->seed, CS_RNG_FALSE_POSITIVE, (uint32_t)c->cur_ts, (uint32_t)infector, (uint32_t)person);
        s.block = (uint32_t)code;
        if (stream_next(&s) < c->P.FalsePositiveRate) {
            c->fc[person] = 1;
            return;
        }
    }
    uint64_t key = ((uint64_t)(uint32_t)infector << 8) | (uint64_t)code;
    if (key < c->claim[person]) c->claim[person] = key;
}

/* Geometric-skip enumeration of n Bernoulli(p) trials: returns the next success
 * position after `pos` (or >= n when exhausted). */
static double next_success(stream* s, double pos, double logq)
{
    double u = stream_next(s);
    return pos + 1.0 + floor(log(u) / logq);
}

static void place_candidates(cs_cpu_ctx* c, int i, int pt, int link, double Pinf, int between, int ts, int mc_place)
{
    const cs_params* P = &c->P;
    const place_arrays* pl = &c->pl[pt];
    int base = pl->member_ofs[link], n;
    int gi = group_of(c, pt, i);
    if (!between) {
        int g = pl->group_ofs[link] + gi;
        base += pl->group_start[g];
        n = pl->group_size[g];
    } else
        n = pl->member_ofs[link + 1] - pl->member_ofs[link];
    double p = Pinf;
    if (p <= 0 || n <= 0) return;
    stream s;
    stream_init(&s, c->seed, between ? CS_RNG_PLACE_BETWEEN : CS_RNG_PLACE_GROUP, (uint32_t)ts, (uint32_t)i, (uint32_t)pt);
    double logq = (p < 1.0) ? log1p(-p) : 0.0;
    double pos = -1.0;
    for (;;) {
        if (p >= 1.0) pos = pos + 1.0;
        else pos = next_success(&s, pos, logq);
        if (!(pos < (double)n)) break;
        int m = pl->members[base + (int)pos];
        c->C.work_place_candidates++;
        double sc = calc_place_susc(c, m, pt, ts);
        if (between && is_ch(c, i) && is_ch(c, m) && group_of(c, pt, i) != group_of(c, pt, m))
            sc *= P->CareHomeResidentPlaceScaling;
        if ((pt == P->CareHomePlaceType) && ((!is_ch(c, i)) || (!is_ch(c, m)))) sc *= P->CareHomeWorkerGroupScaling;
        if (c->inf[m] == CS_INF_SUSCEPTIBLE && !host_absent(c, m, ts)) {
            sc *= calc_person_susc(c, m, i) * p / p;
            if (c->blanket) {
                if (dist2_hh_pt(c, c->hh[m], pl->x[link], pl->y[link]) > P->MoveRestrRadius2) sc *= P->MoveRestrEffect;
            } else if (moverest_differs(c, c->mcell[m], mc_place))
                sc *= P->MoveRestrEffect;
            if ((sc == 1) || (stream_next(&s) < sc)) claim(c, m, i, between ? 2 + pt + CS_MAX_PLACE_TYPES : 2 + pt);
        }
    }
}

/* Spatial contact j of infector i (src/Sweep.cpp:742-856 for one contact).
 * Draw t of the rejection loop reads its uniforms from Philox blocks 2t and 2t+1
 * of the contact's stream (at most four: target block, slot, acceptance, and for
 * the accepted draw the susceptibility test), so every draw's numbers are fixed
 * in advance whatever the earlier draws consumed; the first accepted draw wins. */
#define SPATIAL_BLOCKS_PER_DRAW 2
static int spatial_draw(cs_cpu_ctx* c, stream* s, int b, int hi_, const double* row, double total,
                        int* m_out, int* slot_out, int* p_out, int64_t* err)
{
    double target = stream_next(s) * total;
    int lo = 0, hi = c->NB - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (target < row[mid]) hi = mid; else lo = mid + 1;
    }
    int B = lo;
    if (c->block_S0[B] <= 0) return 0;
    double r = floor(stream_next(s) * (double)c->block_S0[B]);
    int k0 = c->block_cell_ofs[B], k1 = c->block_cell_ofs[B + 1] - 1;
    while (k0 < k1) {
        int mid = (k0 + k1) >> 1;
        if (r < (double)c->block_cum[mid]) k1 = mid; else k0 = mid + 1;
    }
    int m = c->block_cells[k0];
    int slot = (int)(r - (double)(c->block_cum[k0] - c->S0[m]));
    int p = c->slots[c->cell_start[m] + slot];
    double d2 = dist2_hh(c, hi_, c->hh[p]);
    double accept = knum_f32(c, d2, err) / bound_of(c, b, B, err);
    if ((stream_next(s) >= accept) || !is_alive(c, p)) return 0;
    *m_out = m; *slot_out = slot; *p_out = p;
    return 1;
}

static void spatial_contact(cs_cpu_ctx* c, int i, int ci, int j, int closed_i, int ts)
{
    const cs_params* P = &c->P;
    int b = c->cell_block[ci];
    const double* row = c->block_row_cum + (size_t)b * c->NB;
    double total = row[c->NB - 1];
    int64_t err = 0;
    if (!(total > 0)) { c->C.err_spatial_tries++; return; }
    stream s;
    int hi_ = c->hh[i];
    int m = 0, slot = 0, p = 0, t;
    for (t = 0; t < MAX_SPATIAL_TRIES; t++) {
        stream_init(&s, c->seed, CS_RNG_SPATIAL_CONTACT, (uint32_t)ts, (uint32_t)i, (uint32_t)j);
        s.block = (uint32_t)(SPATIAL_BLOCKS_PER_DRAW * t);
        if (spatial_draw(c, &s, b, hi_, row, total, &m, &slot, &p, &err)) break;
    }
    c->C.work_spatial_draws += (t < MAX_SPATIAL_TRIES) ? t + 1 : t;
    c->C.err_kernel_range += err;
    if (t >= MAX_SPATIAL_TRIES) { c->C.err_spatial_tries++; return; }
    if ((ci != m) || (c->hh[p] != hi_)) {
        double ss = calc_spatial_susc(c, p, ts);
        if (is_ch(c, p) || is_ch(c, i)) ss *= P->CareHomeResidentSpatialScaling;
        if (slot < c->S[m]) {
            ss *= calc_person_susc(c, p, i);
            ss *= P->WAIFW_Matrix_SpatialOnly[age_group(c, p)][age_group(c, i)];
            if (c->blanket) {
                if (dist2_hh_pt(c, hi_, c->hh_x[c->hh[p]], c->hh_y[c->hh[p]]) > P->MoveRestrRadius2) ss *= P->MoveRestrEffect;
            } else if (moverest_differs(c, c->mcell[p], c->mcell[i]))
                ss *= P->MoveRestrEffect;
            if ((!closed_i) && host_absent(c, p, ts)) {
                int f = 0;
                for (int pt = 0; (pt < c->NPT) && (!f); pt++)
                    if (link_of(c, pt, p) >= 0) f = place_closed(c, pt, link_of(c, pt, p), ts);
                if (f) ss *= P->Efficacies[CS_NPI_PLACE_CLOSURE][CS_SETTING_SPATIAL];
            }
            if ((ss == 1) || (stream_next(&s) < ss))
                if (c->inf[p] == CS_INF_SUSCEPTIBLE) claim(c, p, i, 2 + 2 * CS_MAX_PLACE_TYPES);
        }
    }
}

/* One infector's household, place and spatial passes (src/Sweep.cpp:314-691). */
static void infector_pass(cs_cpu_ctx* c, int i, int ci, double hh_beta, double sp_beta, double fp, double seas, int ts)
{
    const cs_params* P = &c->P;
    c->C.work_infectors++;
    int h = c->hh[i];
    /* household (src/Sweep.cpp:331-377) */
    if (hh_beta > 0 && c->hh_nh[h] > 1) {
        int f0 = c->hh_first[h], f1 = f0 + c->hh_nh[h];
        double HI = hh_beta * calc_house_inf(c, i, ts);
        int absent = 0;
        for (int m = f0; (m < f1) && (!absent); m++)
            for (int pt = 0; (pt < c->NPT) && (!absent); pt++)
                if (link_of(c, pt, m) >= 0) absent = place_closed(c, pt, link_of(c, pt, m), ts) && host_absent(c, m, ts);
        if (absent) HI *= P->Efficacies[CS_NPI_PLACE_CLOSURE][CS_SETTING_HOUSE];
        stream s;
        stream_init(&s, c->seed, CS_RNG_HOUSEHOLD, (uint32_t)ts, (uint32_t)i, 0);
        for (int m = f0; m < f1; m++) {
            c->C.work_hh_members++;
            if (c->inf[m] == CS_INF_SUSCEPTIBLE) {
                double foi = HI * calc_house_susc(c, m, ts, i);
                if (stream_next(&s) < foi) claim(c, m, i, 1);
            }
        }
    }
    /* places (src/Sweep.cpp:379-647) */
    if (P->DoPlaces && !host_absent(c, i, ts)) {
        for (int pt = 0; pt < c->NPT; pt++) {
            int link = link_of(c, pt, i);
            if (link < 0) continue;
            double PI = fp * seas * calc_place_inf(c, i, pt, ts);
            int mc_place = c->pl[pt].mcell[link];
            if (c->blanket) {
                if (dist2_hh_pt(c, h, c->pl[pt].x[link], c->pl[pt].y[link]) > P->MoveRestrRadius2) PI *= P->MoveRestrEffect;
            } else if (moverest_differs(c, c->mcell[i], mc_place))
                PI *= P->MoveRestrEffect;
            if (pt != P->HotelPlaceType) {
                double p1 = PI;
                if (p1 > 1) p1 = 1;
                place_candidates(c, i, pt, link, p1, 0, ts, mc_place);
            }
            {
                int n = c->pl[pt].member_ofs[link + 1] - c->pl[pt].member_ofs[link];
                double p2 = PI * (P->PlaceTypePropBetweenGroupLinks[pt] * P->PlaceTypeGroupSizeParam1[pt] / ((double)n));
                if (p2 > 1) p2 = 1;
                place_candidates(c, i, pt, link, p2, 1, ts, mc_place);
            }
        }
    }
    /* spatial (src/Sweep.cpp:656-856, per-infector Poisson split) */
    if (sp_beta > 0) {
        double si = calc_spatial_inf(c, i, ts);
        int closed = 0;
        if (P->DoPlaces)
            for (int pt = 0; (pt < c->NPT) && (!closed); pt++)
                if (link_of(c, pt, i) >= 0) closed = place_closed(c, pt, link_of(c, pt, i), ts);
        int closed_i = 0;
        if (closed && host_absent(c, i, ts)) { si *= P->Efficacies[CS_NPI_PLACE_CLOSURE][CS_SETTING_SPATIAL]; closed_i = 1; }
        double lambda = si * sp_beta * c->tot_prob[ci];
        stream s;
        stream_init(&s, c->seed, CS_RNG_SPATIAL_COUNT, (uint32_t)ts, (uint32_t)i, 0);
        int64_t err = 0;
        int k = sample_poisson(&s, lambda, &err);
        c->C.err_spatial_tries += err;
        c->C.work_spatial_contacts += k;
        for (int j = 0; j < k; j++) spatial_contact(c, i, ci, j, closed_i, ts);
    }
}

int cs_cpu_infect_sweep(cs_cpu_ctx* c, double t, int run)
{
    (void)run;
    const cs_params* P = &c->P;
    if (!c->run_started) return fail(c, CS_E_STATE, "infect sweep before begin_run");
    int ts = (int)(uint16_t)(P->TimeStepsPerDay * t);
    c->cur_ts = ts;
    double fp = P->ModelTimeStep / (1 - P->FalsePositiveRate);
    double seas = P->Seasonality;
    c->blanket = P->DoBlanketMoveRestr && (t >= P->MoveRestrTimeStart) && (t < P->MoveRestrTimeStart + P->MoveRestrDuration);
    double sp_beta = (P->DoSpatial ? seas * fp * P->LocalBeta : 0.0);
    double hh_beta = P->DoHouseholds ? seas * fp * P->HouseholdTrans : 0;
    for (int ci = 0; ci < c->NC; ci++) {
        int b0 = c->cell_start[ci] + c->S[ci] + c->L[ci];
        for (int k = 0; k < c->I[ci]; k++) infector_pass(c, c->slots[b0 + k], ci, hh_beta, sp_beta, fp, seas, ts);
    }
    /* queue drain: DoInfect for every claimed person (src/Sweep.cpp:860-880) */
    int32_t* touched = (int32_t*)malloc(sizeof(int32_t) * ((size_t)c->NC + 1));
    uint8_t* seen = (uint8_t*)calloc((size_t)c->NC + 1, 1);
    int nt = 0;
    for (int p = 0; p < c->N; p++) {
        if (c->claim[p] == UINT64_MAX) continue;
        uint64_t key = c->claim[p];
        c->claim[p] = UINT64_MAX;
        int infector = (int)(key >> 8), code = (int)(key & 0xff);
        int16_t it = (int16_t)(code + CS_INFECT_TYPE_MASK * (1 + c->infect_type[infector] / CS_INFECT_TYPE_MASK));
        do_infect(c, p, t, ts, infector, it);
        int cell = cell_of(c, p);
        if (!seen[cell]) { seen[cell] = 1; touched[nt++] = cell; }
    }
    partition_S_blocks(c, touched, nt);
    free(touched);
    free(seen);
    /* DoFalseCase (src/Update.cpp:896-905) for every person with a false-positive
     * entry, after the step's infections; a person the step did not infect takes
     * the false entry's labels (src/Sweep.cpp:866-869) */
    if (P->FalsePositiveRate > 0)
        for (int p = 0; p < c->N; p++) {
            if (!c->fc[p]) continue;
            c->fc[p] = 0;
            if (c->inf[p] == CS_INF_SUSCEPTIBLE) {
                c->infector[p] = -1;
                c->infect_type[p] = -1;
            }
            stream s;
            stream_init(&s, c->seed, CS_RNG_FALSE_CASE, (uint32_t)ts, (uint32_t)p, 0);
            if ((P->ControlPropCasesId == 1) || (stream_next(&s) < P->ControlPropCasesId)) {
                if (P->cumDC_at_sample >= P->CaseOrDeathThresholdBeforeAlert) c->C.cumDC++;
                do_detected_case(c, p, t, ts);
            }
            c->C.cumFC++;
        }
    return CS_OK;
}

/* ------------------------------------------------------ IncubRecoverySweep -- */
static void sev_add(cs_cpu_ctx* c, int p, int which, int delta, int cum)
{
    int ad = c->mcell_adunit[c->mcell[p]];
    int adok = ad >= 0 && ad < CS_MAX_ADUNITS;
    switch (which) {
    case CS_SEV_MILD: c->C.Mild += delta; if (cum) c->C.cumMild++; break;
    case CS_SEV_ILI: c->C.ILI += delta; if (cum) c->C.cumILI++; break;
    case CS_SEV_SARI: c->C.SARI += delta; if (cum) c->C.cumSARI++; break;
    case CS_SEV_CRITICAL:
        c->C.Critical += delta;
        if (adok) c->C.Critical_adunit[ad] += delta;
        if (cum) { c->C.cumCritical++; if (adok) c->C.cumCritical_adunit[ad]++; }
        break;
    case CS_SEV_STEPDOWN: c->C.CritRecov += delta; if (cum) c->C.cumCritRecov++; break;
    default: break;
    }
}
static inline int sev_cur(const cs_cpu_ctx* c, int p) { return c->sev[p] & 0x0f; }
static inline int sev_fin(const cs_cpu_ctx* c, int p) { return c->sev[p] >> 4; }
static inline void set_cur(cs_cpu_ctx* c, int p, int v) { c->sev[p] = (uint8_t)((c->sev[p] & 0xf0) | v); }
static inline void set_fin(cs_cpu_ctx* c, int p, int v) { c->sev[p] = (uint8_t)((c->sev[p] & 0x0f) | (v << 4)); }

/* DoIncub (src/Update.cpp:408-523) without the cell-list move. */
static void do_incub(cs_cpu_ctx* c, int p, int ts)
{
    const cs_params* P = &c->P;
    int age = age_group(c, p);
    if (age >= CS_NUM_AGE_GROUPS) age = CS_NUM_AGE_GROUPS - 1;
    stream s;
    stream_init(&s, c->seed, CS_RNG_INCUB, (uint32_t)ts, (uint32_t)p, 0);
    int64_t err = 0;
    float infn = (float)P->AgeInfectiousness[age];
    if (P->InfectiousnessSD > 0) {
        double k = 1 / (P->InfectiousnessSD * P->InfectiousnessSD);
        infn *= (float)sample_gamma(&s, k, k, &err);
    }
    double psym = P->ProportionSymptomatic[age];
    if (stream_next(&s) < psym) {
        c->inf[p] = CS_INF_INFECTIOUS_ALMOST_SYMPTOMATIC;
        infn *= (float)(-P->SymptInfectiousness);
    } else {
        c->inf[p] = CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE;
        infn *= (float)P->AsymptInfectiousness;
    }
    c->infness[p] = infn;
    double spd = P->TimeStepsPerDay;
    if (!P->DoSeverity || c->inf[p] == CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE) {
        if (P->DoInfectiousnessProfile)
            c->recovery_time[p] = (uint16_t)(c->latent_time[p] + (uint16_t)(P->InfectiousPeriod * spd));
        else
            c->recovery_time[p] = (uint16_t)(c->latent_time[p] + choose(&P->infectious_icdf, P->InfectiousPeriod, &s, spd));
    } else {
        int CaseTime = c->latent_time[p] + ((int)(P->LatentToSymptDelay / P->ModelTimeStep));
        /* ChooseFinalDiseaseSeverity (src/Update.cpp:1377-1389) */
        double x = stream_next(&s);
        int fin;
        if (x < P->Prop_ILI_ByAge[age]) fin = CS_SEV_ILI;
        else if (x < P->Prop_ILI_ByAge[age] + P->Prop_SARI_ByAge[age]) fin = CS_SEV_SARI;
        else if (x < P->Prop_ILI_ByAge[age] + P->Prop_SARI_ByAge[age] + P->Prop_Critical_ByAge[age]) fin = CS_SEV_CRITICAL;
        else fin = CS_SEV_MILD;
        set_fin(c, p, fin);
        /* DecideIfPersonDies (src/Update.cpp:388-406) */
        int to_die = 0;
        if (fin == CS_SEV_CRITICAL) { if (stream_next(&s) < (P->CFR_Critical_ByAge[age] * P->CFR_Critical_Scale_Current)) to_die = 1; }
        else if (fin == CS_SEV_SARI) { if (stream_next(&s) < (P->CFR_SARI_ByAge[age] * P->CFR_SARI_Scale_Current)) to_die = 1; }
        else if (fin == CS_SEV_ILI) { if (stream_next(&s) < (P->CFR_ILI_ByAge[age] * P->CFR_ILI_Scale_Current)) to_die = 1; }
        if (is_ch(c, p) && ((fin == CS_SEV_CRITICAL) || (fin == CS_SEV_SARI)) && (stream_next(&s) > P->CareHomeRelProbHosp)) {
            to_die = 1;
            fin = CS_SEV_ILI;
            set_fin(c, p, fin);
        }
        if (to_die) c->dflags[p] |= CS_DF_TO_DIE;
        if (fin == CS_SEV_MILD)
            c->recovery_time[p] = (uint16_t)(CaseTime + choose(&P->MildToRecovery_icdf, P->Mean_MildToRecovery[age], &s, spd));
        else if (fin == CS_SEV_CRITICAL) {
            c->sari_time[p] = (uint16_t)(CaseTime + choose(&P->ILIToSARI_icdf, P->Mean_ILIToSARI[age], &s, spd));
            c->critical_time[p] = (uint16_t)(c->sari_time[p] + choose(&P->SARIToCritical_icdf, P->Mean_SARIToCritical[age], &s, spd));
            if (to_die) {
                if (P->IncludeStepDownToDeath == 1) {
                    c->stepdown_time[p] = (uint16_t)(c->critical_time[p] + choose(&P->CriticalToCritRecov_icdf, P->Mean_CriticalToCritRecov[age], &s, spd));
                    c->recovery_time[p] = (uint16_t)(c->stepdown_time[p] + choose(&P->StepdownToDeath_icdf, P->Mean_StepdownToDeath[age], &s, spd));
                } else
                    c->recovery_time[p] = (uint16_t)(c->critical_time[p] + choose(&P->CriticalToDeath_icdf, P->Mean_CriticalToDeath[age], &s, spd));
            } else {
                c->stepdown_time[p] = (uint16_t)(c->critical_time[p] + choose(&P->CriticalToCritRecov_icdf, P->Mean_CriticalToCritRecov[age], &s, spd));
                c->recovery_time[p] = (uint16_t)(c->stepdown_time[p] + choose(&P->CritRecovToRecov_icdf, P->Mean_CritRecovToRecov[age], &s, spd));
            }
        } else if (fin == CS_SEV_SARI) {
            c->sari_time[p] = (uint16_t)(CaseTime + choose(&P->ILIToSARI_icdf, P->Mean_ILIToSARI[age], &s, spd));
            if (to_die)
                c->recovery_time[p] = (uint16_t)(c->sari_time[p] + choose(&P->SARIToDeath_icdf, P->Mean_SARIToDeath[age], &s, spd));
            else
                c->recovery_time[p] = (uint16_t)(c->sari_time[p] + choose(&P->SARIToRecovery_icdf, P->Mean_SARIToRecovery[age], &s, spd));
        } else {
            if (to_die)
                c->recovery_time[p] = (uint16_t)(CaseTime + choose(&P->ILIToDeath_icdf, P->Mean_ILIToDeath[age], &s, spd));
            else
                c->recovery_time[p] = (uint16_t)(CaseTime + choose(&P->ILIToRecovery_icdf, P->Mean_ILIToRecovery[age], &s, spd));
        }
    }
    if (c->inf[p] == CS_INF_INFECTIOUS_ALMOST_SYMPTOMATIC && ((P->ControlPropCasesId == 1) || (stream_next(&s) < P->ControlPropCasesId))) {
        c->dflags[p] |= CS_DF_DETECTED;
        c->detected_time[p] = (uint16_t)(ts + (uint16_t)(P->LatentToSymptDelay * spd));
    }
    c->C.err_spatial_tries += err;
}

/* Child-carer check of DoCase/DoDetectedCase (src/Update.cpp:736-763, 843-868): is
 * there an adult at home already?  Evaluated once per household after the step's
 * per-person transitions. */
static void carer_pass(cs_cpu_ctx* c, int h, int ts, int mode_ci)
{
    const cs_params* P = &c->P;
    int j1 = c->hh_first[h], j2 = j1 + c->hh_nh[h];
    int wp = P->PlaceTypeNoAirNum - 1;
    int f = 0;
    for (int j = j1; (j < j2) && (!f); j++)
        f = (is_alive(c, j) && (c->age[j] >= P->CaseAbsentChildAgeCutoff) &&
             ((link_of(c, wp, j) < 0) || host_absent(c, j, ts) || host_quarantined(c, j, ts)));
    if (f) return;
    int k = -1;
    for (int j = j1; j < j2; j++)
        if ((c->age[j] >= P->CaseAbsentChildAgeCutoff) && is_alive(c, j)) { k = j; break; }
    if (k < 0) return;
    if (mode_ci || !host_absent(c, k, ts)) c->absent_start[k] = (uint16_t)(ts + P->usCaseIsolationDelay);
    c->absent_stop[k] = (uint16_t)(ts + P->usCaseIsolationDelay + P->usCaseIsolationDuration);
    c->C.cumAA++;
}

/* Household quarantine of DoDetectedCase (src/Update.cpp:676-708), once per household. */
static void hq_pass(cs_cpu_ctx* c, int h, int ts)
{
    const cs_params* P = &c->P;
    int j1 = c->hh_first[h], j2 = j1 + c->hh_nh[h];
    if (host_to_be_quarantined(c, j1, ts) && !P->DoHQretrigger) return;
    stream s;
    stream_init(&s, c->seed, CS_RNG_HQ, (uint32_t)ts, (uint32_t)h, 0);
    c->quar_start[j1] = (uint16_t)(ts + ((uint16_t)(P->TimeStepsPerDay * P->HQuarantineDelay)));
    int k = (stream_next(&s) < P->HQuarantinePropHouseCompliant) ? 1 : 0;
    if (k) c->C.cumHQ++;
    for (int j = j1; j < j2; j++) {
        if (j > j1) c->quar_start[j] = c->quar_start[j1];
        int comply = (k == 0) ? 0 : ((stream_next(&s) < P->HQuarantinePropIndivCompliant) ? 1 : 0);
        c->dflags[j] = (uint8_t)((c->dflags[j] & ~CS_DF_QUAR_COMPLY_MASK) | (comply << CS_DF_QUAR_COMPLY_SHIFT));
    }
}

/* DoDetectedCase (src/Update.cpp:525-792): the case isolation and household
 * quarantine branches; household quarantine is deferred to hq_pass. */
static void do_detected_case(cs_cpu_ctx* c, int p, double t, int ts)
{
    const cs_params* P = &c->P;
    int ad = c->mcell_adunit[c->mcell[p]];
    if (ad >= 0 && ad < CS_MAX_ADUNITS) c->C.cumDC_adunit[ad]++;
    const int aw = (ad >= 0 && ad < c->NAD) ? ad : 0;   /* the person's admin unit's windows */
    const double hq0 = c->hq_start[aw], ci0 = c->ci_start[aw];
    if (P->DoHouseholds && t >= hq0 && t < hq0 + c->hq_dur) c->hh_hq[c->hh[p]] = 1;
    if (t >= ci0 && t < ci0 + c->ci_dur) {
        stream s;
        stream_init(&s, c->seed, CS_RNG_DETECTED, (uint32_t)ts, (uint32_t)p, 0);
        if ((P->CaseIsolationProp == 1) || (stream_next(&s) < P->CaseIsolationProp)) {
            c->isolation_start[p] = (uint16_t)ts;
            if (host_absent(c, p, ts)) {
                if (c->absent_stop[p] < ts + P->usCaseAbsenteeismDelay + P->usCaseIsolationDuration)
                    c->absent_stop[p] = (uint16_t)(ts + P->usCaseAbsenteeismDelay + P->usCaseIsolationDuration);
            } else if (P->DoRealSymptWithdrawal) {
                c->absent_start[p] = (uint16_t)(ts + P->usCaseIsolationDelay);
                c->absent_stop[p] = (uint16_t)(ts + P->usCaseIsolationDelay + P->usCaseIsolationDuration);
                if (P->DoPlaces && !host_quarantined(c, p, ts) && link_of(c, P->PlaceTypeNoAirNum - 1, p) >= 0 && c->age[p] >= P->CaseAbsentChildAgeCutoff)
                    c->C.cumAC++;
                if (P->DoHouseholds && P->DoPlaces && c->age[p] < P->CaseAbsentChildAgeCutoff) {
                    if (!host_quarantined(c, p, ts)) c->C.cumACS++;
                    if (c->prob_care[p] < P->CaseAbsentChildPropAdultCarers) c->hh_carer[c->hh[p]] |= 2;
                }
            }
        }
    }
}

/* DoCase (src/Update.cpp:794-894). */
static void do_case(cs_cpu_ctx* c, int p, double t, int ts)
{
    const cs_params* P = &c->P;
    int age = age_group(c, p);
    if (age >= CS_NUM_AGE_GROUPS) age = CS_NUM_AGE_GROUPS - 1;
    if (c->inf[p] != CS_INF_INFECTIOUS_ALMOST_SYMPTOMATIC) return;
    c->inf[p] = CS_INF_CASE;
    if (host_absent(c, p, ts)) {
        if (c->absent_stop[p] < ts + P->usCaseAbsenteeismDelay + P->usCaseAbsenteeismDuration)
            c->absent_stop[p] = (uint16_t)(ts + P->usCaseAbsenteeismDelay + P->usCaseAbsenteeismDuration);
    } else if ((P->DoRealSymptWithdrawal) && (P->DoPlaces)) {
        stream s;
        stream_init(&s, c->seed, CS_RNG_CASE, (uint32_t)ts, (uint32_t)p, 0);
        c->absent_start[p] = USHRT_MAX_M1;
        for (int j = 0; j < c->NPT; j++)
            if ((link_of(c, j, p) >= 0) && (j != P->HotelPlaceType) && (!host_absent(c, p, ts)) && (P->SymptPlaceTypeWithdrawalProp[j] > 0)) {
                if ((!is_ch(c, p)) && ((P->SymptPlaceTypeWithdrawalProp[j] == 1) || (stream_next(&s) < P->SymptPlaceTypeWithdrawalProp[j]))) {
                    c->absent_start[p] = (uint16_t)(ts + P->usCaseAbsenteeismDelay);
                    c->absent_stop[p] = (uint16_t)(ts + P->usCaseAbsenteeismDelay + P->usCaseAbsenteeismDuration);
                    if ((!host_quarantined(c, p, ts)) && (link_of(c, P->PlaceTypeNoAirNum - 1, p) >= 0) && (c->age[p] >= P->CaseAbsentChildAgeCutoff))
                        c->C.cumAC++;
                    if ((P->DoHouseholds) && (c->age[p] < P->CaseAbsentChildAgeCutoff)) {
                        if (!host_quarantined(c, p, ts)) c->C.cumACS++;
                        if (c->prob_care[p] < P->CaseAbsentChildPropAdultCarers) c->hh_carer[c->hh[p]] |= 1;
                    }
                }
            }
    }
    if (c->dflags[p] & CS_DF_DETECTED) {
        c->C.cumDC++;
        do_detected_case(c, p, t, ts);
    }
    c->C.cumC++;
    c->C.cumCa[age]++;
    c->C.cumC_keyworker[(c->pflags[p] & CS_PF_KEYWORKER) ? 1 : 0]++;
    int ad = c->mcell_adunit[c->mcell[p]];
    if (ad >= 0 && ad < CS_MAX_ADUNITS) c->C.cumC_adunit[ad]++;
    if (P->DoSeverity) {
        if (sev_fin(c, p) == CS_SEV_MILD) {
            if (sev_cur(c, p) == CS_SEV_ASYMPTOMATIC) { set_cur(c, p, CS_SEV_MILD); sev_add(c, p, CS_SEV_MILD, 1, 1); }
        } else {
            if (sev_cur(c, p) == CS_SEV_ASYMPTOMATIC) { set_cur(c, p, CS_SEV_ILI); sev_add(c, p, CS_SEV_ILI, 1, 1); }
        }
    }
}

/* The infectious-person loop body of IncubRecoverySweep (src/Sweep.cpp:929-977). */
static void infectious_events(cs_cpu_ctx* c, int p, double t, int ts)
{
    const cs_params* P = &c->P;
    int CaseTime = c->latent_time[p] + ((int)(P->LatentToSymptDelay / P->ModelTimeStep));
    if (P->DoSymptoms && ts == (uint16_t)CaseTime) do_case(c, p, t, ts);
    int to_die = (c->dflags[p] & CS_DF_TO_DIE) != 0;
    int ad = c->mcell_adunit[c->mcell[p]];
    int adok = ad >= 0 && ad < CS_MAX_ADUNITS;
    if (P->DoSeverity) {
        if (ts == c->sari_time[p] && sev_cur(c, p) == CS_SEV_ILI) {
            set_cur(c, p, CS_SEV_SARI); sev_add(c, p, CS_SEV_ILI, -1, 0); sev_add(c, p, CS_SEV_SARI, 1, 1);
        }
        if (ts == c->critical_time[p] && sev_cur(c, p) == CS_SEV_SARI) {
            set_cur(c, p, CS_SEV_CRITICAL); sev_add(c, p, CS_SEV_SARI, -1, 0); sev_add(c, p, CS_SEV_CRITICAL, 1, 1);
        }
        if (ts == c->stepdown_time[p] && sev_cur(c, p) == CS_SEV_CRITICAL && !to_die) {
            set_cur(c, p, CS_SEV_STEPDOWN); sev_add(c, p, CS_SEV_CRITICAL, -1, 0); sev_add(c, p, CS_SEV_STEPDOWN, 1, 1);
        }
        if (ts == c->recovery_time[p]) {
            int cur = sev_cur(c, p);
            if (to_die) {
                if (cur == CS_SEV_CRITICAL) { sev_add(c, p, CS_SEV_CRITICAL, -1, 0); c->C.cumDeath_Critical++; set_cur(c, p, CS_SEV_DEAD); }
                else if (cur == CS_SEV_SARI) { sev_add(c, p, CS_SEV_SARI, -1, 0); c->C.cumDeath_SARI++; set_cur(c, p, CS_SEV_DEAD); }
                else if (cur == CS_SEV_ILI) { sev_add(c, p, CS_SEV_ILI, -1, 0); c->C.cumDeath_ILI++; set_cur(c, p, CS_SEV_DEAD); }
            } else if (c->inf[p] == CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE || c->inf[p] == CS_INF_CASE) {
                if (cur == CS_SEV_MILD) { sev_add(c, p, CS_SEV_MILD, -1, 0); set_cur(c, p, CS_SEV_RECOVERED); }
                else if (cur == CS_SEV_ILI) { sev_add(c, p, CS_SEV_ILI, -1, 0); set_cur(c, p, CS_SEV_RECOVERED); }
                else if (cur == CS_SEV_SARI) { sev_add(c, p, CS_SEV_SARI, -1, 0); set_cur(c, p, CS_SEV_RECOVERED); }
                else if (cur == CS_SEV_STEPDOWN) { sev_add(c, p, CS_SEV_STEPDOWN, -1, 0); set_cur(c, p, CS_SEV_RECOVERED); }
            }
        }
    }
    if (ts == c->recovery_time[p]) {
        if (c->inf[p] == CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE || c->inf[p] == CS_INF_CASE) {
            int cell = cell_of(c, p);
            c->mark[c->cell_start[cell] + c->listpos[p]] = 1;
            c->I[cell]--;
            c->C.work_transitions++;
            if (!to_die) {
                c->inf[p] = (c->inf[p] == CS_INF_CASE) ? CS_INF_RECOVERED_FROM_SYMP : CS_INF_RECOVERED_FROM_ASYMP;
                c->R[cell]++;
                c->C.cumR++;
            } else {
                c->inf[p] = (c->inf[p] == CS_INF_CASE) ? CS_INF_DEAD_WAS_SYMP : CS_INF_DEAD_WAS_ASYMP;
                c->D[cell]++;
                c->C.cumD++;
                c->C.cumDa[age_group(c, p)]++;
                if (adok) c->C.cumD_adunit[ad]++;
            }
        }
    }
}

int cs_cpu_incub_recovery_sweep(cs_cpu_ctx* c, double t)
{
    const cs_params* P = &c->P;
    if (!c->run_started) return fail(c, CS_E_STATE, "incub sweep before begin_run");
    int ts = (int)(uint16_t)(P->TimeStepsPerDay * t);
    for (int ci = 0; ci < c->NC; ci++) c->C.work_incub_people += c->L[ci] + c->I[ci];
    /* latent -> infectious (src/Sweep.cpp:924-927) */
    for (int ci = 0; ci < c->NC; ci++) {
        int b0 = c->cell_start[ci] + c->S[ci];
        int L = c->L[ci], moved = 0;
        for (int k = 0; k < L; k++) {
            int p = c->slots[b0 + k];
            if (ts == c->latent_time[p]) {
                do_incub(c, p, ts);
                c->mark[b0 + k] = 1;
                moved++;
                c->C.work_transitions++;
            }
        }
        if (moved) {
            partition_block(c, ci, b0, L, NULL);
            c->L[ci] -= moved;
            c->I[ci] += moved;
        }
    }
    /* infectious events (src/Sweep.cpp:929-977) */
    for (int ci = 0; ci < c->NC; ci++) {
        int b0 = c->cell_start[ci] + c->S[ci] + c->L[ci];
        int I = c->I[ci];
        for (int k = 0; k < I; k++) infectious_events(c, c->slots[b0 + k], t, ts);
        int nm = 0;
        for (int k = 0; k < I; k++) nm += c->mark[b0 + k];
        if (nm) partition_block(c, ci, b0, I, NULL);
    }
    /* deferred household actions */
    for (int h = 0; h < c->NH; h++) {
        if (c->hh_carer[h]) { carer_pass(c, h, ts, (c->hh_carer[h] & 2) != 0); c->hh_carer[h] = 0; }
        if (c->hh_hq[h]) { hq_pass(c, h, ts); c->hh_hq[h] = 0; }
    }
    return CS_OK;
}

int cs_cpu_step(cs_cpu_ctx* c, double t, int run)
{
    int r = cs_cpu_infect_sweep(c, t, run);
    if (r) return r;
    return cs_cpu_incub_recovery_sweep(c, t);
}

/* --------------------------------------------------------- interventions -- */
int cs_cpu_set_interventions(cs_cpu_ctx* c, const cs_interventions* iv)
{
    for (int a = 0; a < (c->NAD > 0 ? c->NAD : 1); a++) {
        c->ci_start[a] = iv->adunit_CaseIsolationTimeStart ? iv->adunit_CaseIsolationTimeStart[a] : iv->CaseIsolationTimeStart;
        c->hq_start[a] = iv->adunit_HQuarantineTimeStart ? iv->adunit_HQuarantineTimeStart[a] : iv->HQuarantineTimeStart;
    }
    c->ci_dur = iv->CaseIsolationPolicyDuration;
    c->hq_dur = iv->HQuarantinePolicyDuration;
    if (iv->mcell_socdist) memcpy(c->socdist, iv->mcell_socdist, (size_t)c->NM);
    if (iv->mcell_moverest) memcpy(c->moverest, iv->mcell_moverest, (size_t)c->NM);
    return CS_OK;
}

/* Is a living adult at home already (no workplace link, or quarantined)?  The test
 * DoPlaceClose and DoPlaceOpen make before sending an adult home with a child
 * (src/Update.cpp:1211-1215, 1278-1281). */
static int adult_home_for_child(const cs_cpu_ctx* c, int h, int ts)
{
    const cs_params* P = &c->P;
    const int wp = P->PlaceTypeNoAirNum - 1;
    for (int j = c->hh_first[h]; j < c->hh_first[h] + c->hh_nh[h]; j++)
        if (is_alive(c, j) && c->age[j] >= P->CaseAbsentChildAgeCutoff &&
            (wp < 0 || link_of(c, wp, j) < 0 || host_quarantined(c, j, ts)))
            return 1;
    return 0;
}

/* The host closure queue of DoPlaceClose (src/Update.cpp:1218-1231), one window per
 * household merged by min/max, and its application by UpdateHostClosure
 * (src/Update.cpp:1243-1258) to the household's first living adult. */
static void queue_carer(cs_cpu_ctx* c, int h, uint16_t ws, uint16_t we)
{
    if (ws >= we) return;
    if (c->carer_start[h] > ws) c->carer_start[h] = ws;
    if (c->carer_stop[h] < we) c->carer_stop[h] = we;
}

static void carer_queue_apply(cs_cpu_ctx* c)
{
    const cs_params* P = &c->P;
    for (int h = 0; h < c->NH; h++) {
        if (c->carer_start[h] >= c->carer_stop[h]) continue;
        const uint16_t ws = c->carer_start[h], we = c->carer_stop[h];
        c->carer_start[h] = 0xFFFF;
        c->carer_stop[h] = 0;
        for (int j = c->hh_first[h]; j < c->hh_first[h] + c->hh_nh[h]; j++)
            if (c->age[j] >= P->CaseAbsentChildAgeCutoff && is_alive(c, j)) {
                if (c->absent_start[j] > ws) c->absent_start[j] = ws;
                if (c->absent_stop[j] < we) c->absent_stop[j] = we;
                break;
            }
    }
}

/* DoPlaceClose's loop over the members of a place that closed (src/Update.cpp:
 * 1196-1240) at timestep ts with absence window [ws, we). */
static void close_place_members(cs_cpu_ctx* c, int pt, int l, int ts, uint16_t ws, uint16_t we)
{
    const cs_params* P = &c->P;
    place_arrays* pl = &c->pl[pt];
    const double att = P->PlaceClosePropAttending[pt];
    for (int k = pl->member_ofs[l]; k < pl->member_ofs[l + 1]; k++) {
        const int w = pl->members[k];
        if (!((att == 0) || (c->prob_absent[w] >= att))) continue;
        if (!host_absent(c, w, ts) && !host_quarantined(c, w, ts) && c->age[w] < P->CaseAbsentChildAgeCutoff &&
            c->prob_care[w] < P->CaseAbsentChildPropAdultCarers && !adult_home_for_child(c, c->hh[w], ts))
            queue_carer(c, c->hh[w], ws, we);
        if (c->absent_start[w] > ws) c->absent_start[w] = ws;
        if (c->absent_stop[w] < we) c->absent_stop[w] = we;
    }
}

/* DoPlaceOpen (src/Update.cpp:1260-1294) for place l of type pt, whose closure ends
 * at ce > ts. */
static void open_place_members(cs_cpu_ctx* c, int pt, int l, int ts, uint16_t ce)
{
    const cs_params* P = &c->P;
    place_arrays* pl = &c->pl[pt];
    for (int k = pl->member_ofs[l]; k < pl->member_ofs[l + 1]; k++) {
        const int ai = pl->members[k];
        if (c->absent_stop[ai] == ce) c->absent_stop[ai] = (uint16_t)ts;
        if (!(c->prob_care[ai] < P->CaseAbsentChildPropAdultCarers)) continue;
        if (c->age[ai] >= P->CaseAbsentChildAgeCutoff || host_quarantined(c, ai, ts) || adult_home_for_child(c, c->hh[ai], ts))
            continue;
        for (int j = c->hh_first[c->hh[ai]]; j < c->hh_first[c->hh[ai]] + c->hh_nh[c->hh[ai]]; j++)
            if (c->age[j] >= P->CaseAbsentChildAgeCutoff && is_alive(c, j) && host_absent(c, j, ts) && c->absent_stop[j] == ce)
                c->absent_stop[j] = (uint16_t)ts;
    }
}

/* DoPlaceClose (src/Update.cpp:1095-1240) with DoAnyway = 1 for the listed
 * microcells: close the place if its ProbClose passes the efficacy, run the member
 * loop (symptomatic withdrawal model) at timestep `start`, then the carers. */
int cs_cpu_close_places(cs_cpu_ctx* c, int pt, const int32_t* mcells, int n_mcells, uint16_t start, uint16_t stop)
{
    const cs_params* P = &c->P;
    if (pt < 0 || pt >= c->NPT) return fail(c, CS_E_ARG, "bad place type");
    uint8_t* sel = NULL;
    if (mcells) {
        sel = (uint8_t*)calloc((size_t)c->NM + 1, 1);
        for (int k = 0; k < n_mcells; k++) if (mcells[k] >= 0 && mcells[k] < c->NM) sel[mcells[k]] = 1;
    }
    place_arrays* pl = &c->pl[pt];
    for (int l = 0; l < pl->n; l++) {
        if (sel && !sel[pl->mcell[l]]) continue;
        if (!(pl->close_end[l] < stop)) continue;
        if (pl->prob_close[l] >= P->Efficacies[CS_NPI_PLACE_CLOSURE][pt]) {
            if (pl->close_start[l] > start) pl->close_start[l] = start;
            pl->close_end[l] = stop;
            if (P->DoRealSymptWithdrawal) close_place_members(c, pt, l, start, start, stop);
        } else
            pl->close_start[l] = pl->close_end[l] = stop;
    }
    carer_queue_apply(c);
    free(sel);
    return CS_OK;
}

/* The outcomes of a host TreatSweep's DoPlaceClose / DoPlaceOpen calls, in the order
 * the GPU library applies them: opens, then closes, each place type by place type
 * (events of one kind and type in the order given), then the closures' carers. */
int cs_cpu_place_events(cs_cpu_ctx* c, const cs_place_event* ev, int n)
{
    const cs_params* P = &c->P;
    if (n < 0 || (n > 0 && !ev)) return fail(c, CS_E_ARG, "bad event list");
    for (int i = 0; i < n; i++) {
        if (ev[i].place_type >= c->NPT || ev[i].place < 0 || ev[i].place >= c->pl[ev[i].place_type].n)
            return fail(c, CS_E_ARG, "place event out of range");
        if (ev[i].kind != CS_PLACE_EV_CLOSE && ev[i].kind != CS_PLACE_EV_OPEN && ev[i].kind != CS_PLACE_EV_HOLIDAY)
            return fail(c, CS_E_ARG, "bad place event kind");
    }
    int closes = 0;
    /* opens, closes, then holidays (the holiday part of IncubRecoverySweep,
     * src/Sweep.cpp:889-918); closes' carers after the last close */
    static const int kinds[3] = {CS_PLACE_EV_OPEN, CS_PLACE_EV_CLOSE, CS_PLACE_EV_HOLIDAY};
    for (int kind = 0; kind < 3; kind++) {
        if (kind == 2 && closes) { carer_queue_apply(c); closes = 0; }
        for (int pt = 0; pt < c->NPT; pt++)
            for (int i = 0; i < n; i++) {
                const cs_place_event* e = ev + i;
                if (e->place_type != pt || e->kind != kinds[kind]) continue;
                place_arrays* pl = &c->pl[pt];
                if (e->kind == CS_PLACE_EV_HOLIDAY) {
                    if (pl->close_start[e->place] > e->win_start) pl->close_start[e->place] = e->win_start;
                    if (pl->close_end[e->place] < e->win_stop) pl->close_end[e->place] = e->win_stop;
                    for (int k = pl->member_ofs[e->place]; k < pl->member_ofs[e->place + 1]; k++) {
                        const int w = pl->members[k];
                        if (c->absent_start[w] > e->win_start) c->absent_start[w] = e->win_start;
                        if (c->absent_stop[w] < e->win_stop) c->absent_stop[w] = e->win_stop;
                    }
                } else if (e->kind == CS_PLACE_EV_CLOSE) {
                    closes = 1;
                    pl->close_start[e->place] = e->close_start;
                    pl->close_end[e->place] = e->close_end;
                    if (e->members && P->DoRealSymptWithdrawal) close_place_members(c, pt, e->place, e->ts, e->win_start, e->win_stop);
                } else {
                    const uint16_t ce = pl->close_end[e->place];
                    if (e->ts < ce) {
                        if (P->DoRealSymptWithdrawal) open_place_members(c, pt, e->place, e->ts, ce);
                        pl->close_end[e->place] = e->ts;
                    }
                }
            }
    }
    if (closes) carer_queue_apply(c);
    return CS_OK;
}

int cs_cpu_set_mcell_status(cs_cpu_ctx* c, const int32_t* mcells, const uint8_t* socdist, const uint8_t* moverest, int n)
{
    if (n < 0 || (n > 0 && !mcells)) return fail(c, CS_E_ARG, "bad microcell list");
    for (int k = 0; k < n; k++) {
        if (mcells[k] < 0 || mcells[k] >= c->NM) return fail(c, CS_E_ARG, "microcell out of range");
        if (socdist) c->socdist[mcells[k]] = socdist[k];
        if (moverest) c->moverest[mcells[k]] = moverest[k];
    }
    return CS_OK;
}

/* --------------------------------------------------------------- readout -- */
int cs_cpu_download_state(cs_cpu_ctx* c, const cs_state_view* v)
{
    size_t N = (size_t)c->N, NC = (size_t)c->NC;
#define CP(dst, src, n) do { if (v->dst) memcpy(v->dst, c->src, sizeof(*c->src) * (n)); } while (0)
    CP(inf, inf, N); CP(severity, sev, N); CP(flags, dflags, N);
    CP(infection_time, infection_time, N); CP(latent_time, latent_time, N);
    CP(recovery_or_death_time, recovery_time, N); CP(SARI_time, sari_time, N);
    CP(Critical_time, critical_time, N); CP(Stepdown_time, stepdown_time, N);
    CP(absent_start_time, absent_start, N); CP(absent_stop_time, absent_stop, N);
    CP(isolation_start_time, isolation_start, N); CP(quar_start_time, quar_start, N);
    CP(detected_time, detected_time, N); CP(infectiousness, infness, N); CP(susc, susc, N);
    CP(ProbAbsent, prob_absent, N); CP(ProbCare, prob_care, N); CP(infector, infector, N);
    CP(infect_type, infect_type, N); CP(listpos, listpos, N);
    CP(cell_S, S, NC); CP(cell_L, L, NC); CP(cell_I, I, NC); CP(cell_R, R, NC); CP(cell_D, D, NC);
    CP(cell_S0, S0, NC); CP(cell_tot_prob, tot_prob, NC); CP(cell_slots, slots, N);
#undef CP
    return CS_OK;
}

int cs_cpu_get_counters(cs_cpu_ctx* c, cs_counters* out)
{
    *out = c->C;
    int64_t S = 0, L = 0, I = 0, R = 0, D = 0;
    for (int j = 0; j < c->NC; j++) { S += c->S[j]; L += c->L[j]; I += c->I[j]; R += c->R[j]; D += c->D[j]; }
    out->S = S; out->L = L; out->I = I; out->R = R; out->D = D;
    return CS_OK;
}

/* ------------------------------------------------------ test-only exports -- */
int cs_cpu_upload_state(cs_cpu_ctx* c, uint64_t seed, const cs_state_view* v)
{
    size_t N = (size_t)c->N, NC = (size_t)c->NC;
    c->rad_origin[0] = c->P.LocationInitialInfection[0];
    c->rad_origin[1] = c->P.LocationInitialInfection[1];
#define CPI(src, dst, n) do { if (v->src) memcpy(c->dst, v->src, sizeof(*c->dst) * (n)); } while (0)
    CPI(inf, inf, N); CPI(severity, sev, N); CPI(flags, dflags, N);
    CPI(infection_time, infection_time, N); CPI(latent_time, latent_time, N);
    CPI(recovery_or_death_time, recovery_time, N); CPI(SARI_time, sari_time, N);
    CPI(Critical_time, critical_time, N); CPI(Stepdown_time, stepdown_time, N);
    CPI(absent_start_time, absent_start, N); CPI(absent_stop_time, absent_stop, N);
    CPI(isolation_start_time, isolation_start, N); CPI(quar_start_time, quar_start, N);
    CPI(detected_time, detected_time, N); CPI(infectiousness, infness, N); CPI(susc, susc, N);
    CPI(ProbAbsent, prob_absent, N); CPI(ProbCare, prob_care, N); CPI(infector, infector, N);
    CPI(infect_type, infect_type, N); CPI(listpos, listpos, N);
    CPI(cell_S, S, NC); CPI(cell_L, L, NC); CPI(cell_I, I, NC); CPI(cell_R, R, NC); CPI(cell_D, D, NC);
    CPI(cell_S0, S0, NC); CPI(cell_tot_prob, tot_prob, NC); CPI(cell_slots, slots, N);
#undef CPI
    memset(c->mark, 0, N);
    memset(&c->C, 0, sizeof(c->C));
    c->seed = seed;
    reset_run_level(c, seed);
    rebuild_block_tables(c);
    c->run_started = 1;
    return CS_OK;
}

/* The infectiousness/susceptibility products of src/CalcInfSusc.cpp for person p
 * (infector q, place type pt) at timestep ts:
 * kind 0 house_inf, 1 place_inf, 2 spatial_inf, 3 person_inf, 4 house_susc,
 * 5 place_susc, 6 spatial_susc, 7 person_susc. */
double cs_cpu_calc(const cs_cpu_ctx* c, int kind, int p, int q, int pt, int ts)
{
    switch (kind) {
    case 0: return calc_house_inf(c, p, ts);
    case 1: return calc_place_inf(c, p, pt, ts);
    case 2: return calc_spatial_inf(c, p, ts);
    case 3: return calc_person_inf(c, p, ts);
    case 4: return calc_house_susc(c, p, ts, q);
    case 5: return calc_place_susc(c, p, pt, ts);
    case 6: return calc_spatial_susc(c, p, ts);
    case 7: return calc_person_susc(c, p, q);
    default: return NAN;
    }
}

/* n draws of a sampler from stream (seed, purpose 0, entity k) for k = 0..n-1:
 * kind 0 Poisson(a); 1 Gamma(shape a, rate b); 2 successes among round(a)
 * Bernoulli(b) trials enumerated by geometric skips. */
int cs_cpu_sample_many(int kind, uint64_t seed, double a, double b, int n, double* out)
{
    int64_t err = 0;
    for (int k = 0; k < n; k++) {
        stream s;
        stream_init(&s, seed, 0, 0, (uint32_t)k, 0);
        if (kind == 0) out[k] = sample_poisson(&s, a, &err);
        else if (kind == 1) out[k] = sample_gamma(&s, b, a, &err);
        else if (kind == 2) {
            int trials = (int)a, cnt = 0;
            double logq = (b < 1.0) ? log1p(-b) : 0.0, pos = -1.0;
            for (;;) {
                if (b >= 1.0) pos = pos + 1.0;
                else pos = next_success(&s, pos, logq);
                if (!(pos < (double)trials)) break;
                cnt++;
            }
            out[k] = cnt;
        } else return CS_E_ARG;
    }
    return err ? CS_E_OVERFLOW : CS_OK;
}

/* ================================================================== set-up ==
 * Population set-up (the GPU's cs_gpu_setup_*), restated sequentially: the steps
 * of the reference's SetupModel that build the sweep's inputs -- microcell
 * populations (src/SetupModel.cpp:1137-1156), people numbered cell by cell
 * (:1163-1185), households and their locations (:1224-1290), people assigned to
 * places (:1989-2466) -- on the same counter-based streams as the device, with
 * the same arithmetic, so the two agree array for array. */
typedef struct cs_cpu_setup {
    char err[256];
    cs_setup_out o;              /* sizes and arrays (owned) */
} cs_cpu_setup;

static int setup_fail(cs_cpu_setup* s, int code, const char* msg)
{
    snprintf(s->err, sizeof s->err, "%s", msg);
    return code;
}

static uint64_t setup_rand64(uint64_t seed, int purpose, uint32_t ts, uint32_t entity, uint32_t sub)
{
    uint32_t ctr[4] = {0u, entity, (ts & 0xffffu) | ((uint32_t)purpose << 16), sub}, x[4];
    cs_cpu_philox((uint32_t)seed, (uint32_t)(seed >> 32), ctr, x);
    return ((uint64_t)x[1] << 32) | x[0];
}

static uint64_t mulhi64(uint64_t a, uint64_t b)
{
    return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
}

static double setup_knum(const double* lk, const double* hr, const cs_params* P, double r2)
{
    double t = r2 / P->kernel_delta;
    if (t > P->kernel_size) return 0.0;
    double s = t * P->kernel_expansion;
    if (s < P->kernel_size) {
        t = s - floor(s);
        return (1.0 - t) * hr[(int)s] + t * hr[(int)(s + 1.0)];
    }
    int i0 = (int)t, i1 = (int)(t + 1.0);
    if (i1 > P->kernel_size) i1 = P->kernel_size;
    s = t - floor(t);
    return (1.0 - s) * lk[i0] + s * lk[i1];
}

static double setup_dist2(const cs_params* P, float ax, float ay, float bx, float by)
{
    if (P->DoUTM_coords) return dist2_utm(P, ax, ay, bx, by);
    float dx = ax - bx, dy = ay - by;
    return periodic_xy(P, fabs(dx), fabs(dy));
}

static int setup_hh_size(stream* s, const double* cdf, int k, int n)
{
    double u = stream_next(s);
    int m = 1;
    while ((u > cdf[m - 1]) && (k + m < n) && (m < CS_MAX_HOUSEHOLD_SIZE)) m++;
    return m;
}

static int64_t setup_place_size(uint64_t seed, int t, int i, const cs_setup_place_type* T, int64_t* err)
{
    stream s;
    stream_init(&s, seed, CS_RNG_SETUP_PLACE_SIZE, 0, (uint32_t)i, (uint32_t)t);
    double v;
    if (T->size_kind == CS_SETUP_SIZE_POWER) {
        double u = 1.0 - stream_next(&s);
        v = floor((T->size_offset + 1.0) * pow(u, -1.0 / T->size_power) - T->size_offset);
        v = fmin(fmax(v, 1.0), T->size_max);
    } else {
        v = floor(sample_gamma(&s, 4.0 / T->mean_size, 4.0, err) + 0.5);
        v = fmax(v, 1.0);
    }
    return (int64_t)v;
}

typedef struct { double d2; int32_t pl; } setup_cand;

static int setup_cand_less(double d2, int pl, const setup_cand* c)
{
    return d2 < c->d2 || (d2 == c->d2 && pl < c->pl);
}

typedef struct { uint64_t key; int32_t a; } setup_key;

static int setup_key_cmp(const void* x, const void* y)
{
    const setup_key* a = (const setup_key*)x;
    const setup_key* b = (const setup_key*)y;
    if (a->key != b->key) return a->key < b->key ? -1 : 1;
    return (a->a > b->a) - (a->a < b->a);
}

#define SETUP_ALLOC(p, n, T)                                                   \
    do {                                                                       \
        (p) = (T*)calloc((size_t)((n) > 0 ? (n) : 1), sizeof(T));              \
        if (!(p)) { rc = setup_fail(s, CS_E_ARG, "setup: out of memory"); goto done; } \
    } while (0)

static int setup_run(cs_cpu_setup* s, const cs_setup_spec* S, const cs_params* P)
{
    int rc = CS_OK;
    int64_t err = 0;
    const uint64_t seed = S->seed;
    const int nmcl = S->nmcl, nch = S->nch, ncw = S->ncw;
    const int th = nch * nmcl, tw = ncw * nmcl;
    const int64_t M = (int64_t)tw * th;
    const int G = ncw * nch, N = S->n_people;
    const double mcw = S->cell_width / nmcl, mch = S->cell_height / nmcl;
    cs_setup_out* o = &s->o;
    uint64_t *q = NULL, *qb = NULL, *pref = NULL;
    int32_t *cnt = NULL, *mcell_start = NULL, *mcell_n = NULL;
    uint8_t* taken_p = NULL;
    int32_t* list = NULL;
    double bl[CS_SETUP_MAX_BLOBS][4];
    if (N <= 0 || ncw <= 0 || nch <= 0 || nmcl <= 0) return setup_fail(s, CS_E_ARG, "setup: bad sizes");
    if (S->n_blobs < 0 || S->n_blobs > CS_SETUP_MAX_BLOBS) return setup_fail(s, CS_E_ARG, "setup: bad n_blobs");
    if (S->num_place_types < 0 || S->num_place_types > CS_MAX_PLACE_TYPES)
        return setup_fail(s, CS_E_ARG, "setup: bad num_place_types");
    for (int t = 0; t < S->num_place_types; t++)
        if (S->pt[t].nearest < 1 || S->pt[t].nearest > CS_SETUP_MAX_NEAREST)
            return setup_fail(s, CS_E_ARG, "setup: bad nearest");
    o->n_people = N;
    o->num_place_types = S->num_place_types;
    o->n_adunits = S->adunit_grid > 0 ? S->adunit_grid * S->adunit_grid : 1;

    /* 1. microcell weights (lognormal, optionally blended with blobs), integer prefix */
    for (int k = 0; k < S->n_blobs; k++) {
        stream b;
        stream_init(&b, seed, CS_RNG_SETUP_BLOB, 0, (uint32_t)k, 0);
        bl[k][0] = 0.05 + 0.9 * stream_next(&b);
        bl[k][1] = 0.05 + 0.9 * stream_next(&b);
        bl[k][2] = 0.004 + 0.016 * stream_next(&b);
        bl[k][3] = exp(0.7 * sample_normal(&b, &err));
    }
    SETUP_ALLOC(q, M, uint64_t);
    SETUP_ALLOC(pref, M, uint64_t);
    if (S->n_blobs > 0) SETUP_ALLOC(qb, M, uint64_t);
    for (int64_t j = 0; j < M; j++) {
        stream d;
        stream_init(&d, seed, CS_RNG_SETUP_DENSITY, 0, (uint32_t)j, 0);
        double w = exp(S->sigma * sample_normal(&d, &err));
        q[j] = (uint64_t)floor(w * 1048576.0);
        if (S->n_blobs > 0) {
            const double xs = ((double)(j / th) + 0.5) / (double)tw;
            const double ys = ((double)(j % th) + 0.5) / (double)th;
            double b = 0.0;
            for (int k = 0; k < S->n_blobs; k++) {
                const double ax = (xs - bl[k][0]) / bl[k][2], ay = (ys - bl[k][1]) / bl[k][2];
                b = b + bl[k][3] * exp(-0.5 * ax * ax) * exp(-0.5 * ay * ay);
            }
            qb[j] = (uint64_t)floor(b * 1048576.0);
        }
    }
    if (S->n_blobs > 0) {
        uint64_t QW = 0, QB = 0;
        for (int64_t j = 0; j < M; j++) { QW += q[j]; QB += qb[j]; }
        for (int64_t j = 0; j < M; j++) {
            const double a = (double)q[j] / (double)QW, b = (double)qb[j] / (double)QB;
            q[j] = (uint64_t)floor(((1.0 - S->blob_share) * a + S->blob_share * b) * 4503599627370496.0);
        }
    }
    {
        uint64_t run = 0;
        for (int64_t j = 0; j < M; j++) pref[j] = run += q[j];
    }
    if (pref[M - 1] == 0) { rc = setup_fail(s, CS_E_ARG, "setup: every microcell weight is zero"); goto done; }

    /* 2. people to microcells */
    SETUP_ALLOC(cnt, M, int32_t);
    for (int k = 0; k < N; k++) {
        const uint64_t r = mulhi64(setup_rand64(seed, CS_RNG_SETUP_PERSON, 0, (uint32_t)k, 0), pref[M - 1]);
        int64_t lo = 0, hi = M - 1;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (pref[mid] > r) hi = mid; else lo = mid + 1;
        }
        cnt[lo]++;
    }

    /* 3. populated cells and microcells, the reference's order */
    {
        int NC = 0, NM = 0;
        for (int c = 0; c < G; c++) {
            int n = 0;
            for (int l = 0; l < nmcl; l++)
                for (int m = 0; m < nmcl; m++) {
                    int v = cnt[(int64_t)((c / nch) * nmcl + l) * th + (int64_t)(c % nch) * nmcl + m];
                    n += v;
                    NM += v > 0;
                }
            NC += n > 0;
        }
        o->n_cells = NC;
        o->n_mcells = NM;
        SETUP_ALLOC(o->cell_grid, NC, int32_t);
        SETUP_ALLOC(o->cell_start, NC + 1, int32_t);
        SETUP_ALLOC(o->mcell_cell, NM, int32_t);
        SETUP_ALLOC(o->mcell_grid, NM, int64_t);
        SETUP_ALLOC(o->mcell_adunit, NM, int32_t);
        SETUP_ALLOC(mcell_start, NM, int32_t);
        SETUP_ALLOC(mcell_n, NM, int32_t);
        int pid = 0, mid = 0, run = 0;
        for (int c = 0; c < G; c++) {
            const int first_mid = mid, first_run = run;
            for (int l = 0; l < nmcl; l++)
                for (int m = 0; m < nmcl; m++) {
                    const int64_t j = (int64_t)((c / nch) * nmcl + l) * th + (int64_t)(c % nch) * nmcl + m;
                    const int v = cnt[j];
                    if (v == 0) continue;
                    o->mcell_cell[mid] = pid;
                    o->mcell_grid[mid] = j;
                    mcell_start[mid] = run;
                    mcell_n[mid] = v;
                    int au = 0;
                    if (S->adunit_grid > 0) {
                        const int64_t mx = j / th, my = j % th;
                        int64_t ax = (mx * S->adunit_grid) / tw, ay = (my * S->adunit_grid) / th;
                        if (ax > S->adunit_grid - 1) ax = S->adunit_grid - 1;
                        if (ay > S->adunit_grid - 1) ay = S->adunit_grid - 1;
                        au = (int)(ax * S->adunit_grid + ay);
                    }
                    o->mcell_adunit[mid] = au;
                    run += v;
                    mid++;
                }
            if (run > first_run) {
                o->cell_grid[pid] = c;
                o->cell_start[pid] = first_run;
                pid++;
            }
            (void)first_mid;
        }
        o->cell_start[NC] = N;
    }

    /* 4. households */
    {
        const int NM = o->n_mcells;
        int NH = 0;
        for (int i = 0; i < NM; i++) {
            stream h;
            stream_init(&h, seed, CS_RNG_SETUP_HH, 0, (uint32_t)o->mcell_grid[i], 0);
            int k = 0;
            while (k < mcell_n[i]) { k += setup_hh_size(&h, S->hh_cdf, k, mcell_n[i]); NH++; }
        }
        o->n_households = NH;
        SETUP_ALLOC(o->hh_first, NH, int32_t);
        SETUP_ALLOC(o->hh_nh, NH, uint16_t);
        SETUP_ALLOC(o->hh_x, NH, float);
        SETUP_ALLOC(o->hh_y, NH, float);
        SETUP_ALLOC(o->person_hh, N, int32_t);
        SETUP_ALLOC(o->person_mcell, N, int32_t);
        int hh = 0;
        for (int i = 0; i < NM; i++) {
            const int64_t j = o->mcell_grid[i];
            stream h;
            stream_init(&h, seed, CS_RNG_SETUP_HH, 0, (uint32_t)j, 0);
            const int n = mcell_n[i], first = mcell_start[i];
            const double x = (double)(j / th), y = (double)(j % th);
            int k = 0;
            uint32_t ord = 0;
            while (k < n) {
                const int m = setup_hh_size(&h, S->hh_cdf, k, n);
                stream sl;
                stream_init(&sl, seed, CS_RNG_SETUP_HH_LOC, 0, (uint32_t)j, ord++);
                const double ux = stream_next(&sl), uy = stream_next(&sl);
                o->hh_first[hh] = first + k;
                o->hh_nh[hh] = (uint16_t)m;
                o->hh_x[hh] = (float)(mcw * (ux + x));
                o->hh_y[hh] = (float)(mch * (uy + y));
                for (int r = 0; r < m; r++) {
                    o->person_hh[first + k + r] = hh;
                    o->person_mcell[first + k + r] = i;
                }
                k += m;
                hh++;
            }
        }
    }

    /* 5. ages */
    SETUP_ALLOC(o->person_age, N, uint8_t);
    for (int p = 0; p < N; p++) {
        stream a;
        stream_init(&a, seed, CS_RNG_SETUP_AGE, 0, (uint32_t)p, 0);
        const double u = stream_next(&a);
        int b = 0;
        while (b < CS_NUM_AGE_GROUPS - 1 && !(u < S->age_cdf[b])) b++;
        int age = b * CS_AGE_GROUP_WIDTH + (int)floor(stream_next(&a) * CS_AGE_GROUP_WIDTH);
        o->person_age[p] = (uint8_t)(age < 84 ? age : 84);
    }

    /* 6. places */
    {
        const int npt = S->num_place_types;
        SETUP_ALLOC(o->person_place, (int64_t)(npt > 0 ? npt : 1) * N, int32_t);
        SETUP_ALLOC(o->person_group, (int64_t)(npt > 0 ? npt : 1) * N, uint16_t);
        for (int64_t i = 0; i < (int64_t)npt * N; i++) o->person_place[i] = -1;
        SETUP_ALLOC(taken_p, N, uint8_t);
        SETUP_ALLOC(list, N, int32_t);
        for (int t = 0; t < npt; t++) {
            const cs_setup_place_type* T = &S->pt[t];
            int n_att = 0;
            for (int p = 0; p < N; p++) {
                if (taken_p[p]) continue;
                const double a = (double)o->person_age[p];
                int f = 0;
                for (int b = 0; b < 3 && !f; b++) {
                    if (!(T->band_prop[b] > 0) || a < T->band_lo[b] || !(a < T->band_hi[b])) continue;
                    stream sa;
                    stream_init(&sa, seed, CS_RNG_SETUP_ATTEND, 0, (uint32_t)p, (uint32_t)(4 * t + b));
                    if (stream_next(&sa) < T->band_prop[b]) f = 1;
                }
                if (f) { taken_p[p] = 1; list[n_att++] = p; }
            }
            o->n_attendees[t] = n_att;
            if (n_att == 0) {
                o->n_places[t] = 0;
                SETUP_ALLOC(o->place_member_ofs[t], 1, int32_t);
                SETUP_ALLOC(o->place_group_ofs[t], 1, int32_t);
                continue;
            }
            /* sizes until they cover the attendees */
            int n_est = (int)((double)n_att / T->mean_size * 1.2) + 8;
            if (n_est < 1) n_est = 1;
            int64_t* sz = (int64_t*)calloc((size_t)n_est, sizeof(int64_t));
            int64_t* cum = (int64_t*)calloc((size_t)n_est, sizeof(int64_t));
            if (!sz || !cum) { free(sz); free(cum); rc = setup_fail(s, CS_E_ARG, "setup: out of memory"); goto done; }
            int64_t run = 0;
            for (int i = 0; i < n_est; i++) { sz[i] = setup_place_size(seed, t, i, T, &err); cum[i] = run += sz[i]; }
            int lo = 0, hi = n_est;
            while (lo < hi) { int mid = (lo + hi) >> 1; if (cum[mid] >= n_att) hi = mid; else lo = mid + 1; }
            const int npl = (lo < n_est) ? lo + 1 : n_est + 1;
            o->n_places[t] = npl;
            int32_t* rem = (int32_t*)calloc((size_t)npl, sizeof(int32_t));
            SETUP_ALLOC(o->place_mcell[t], npl, int32_t);
            SETUP_ALLOC(o->place_x[t], npl, float);
            SETUP_ALLOC(o->place_y[t], npl, float);
            for (int i = 0; i < npl; i++) {
                int64_t size;
                if (i < n_est) { size = sz[i]; if (cum[i] > n_att) size -= cum[i] - n_att; }
                else size = n_att - cum[n_est - 1];
                rem[i] = (int32_t)ceil((double)size * T->capacity_slack);
                const uint64_t r = mulhi64(setup_rand64(seed, CS_RNG_SETUP_PLACE_LOC, 0, (uint32_t)i, (uint32_t)t),
                                           (uint64_t)N);
                const int mid = o->person_mcell[r];
                const int64_t j = o->mcell_grid[mid];
                stream sp;
                stream_init(&sp, seed, CS_RNG_SETUP_PLACE_LOC, 0, (uint32_t)i, (uint32_t)t);
                sp.block = 1;
                const double ux = stream_next(&sp), uy = stream_next(&sp);
                o->place_mcell[t][i] = mid;
                o->place_x[t][i] = (float)(mcw * ((double)(j / th) + ux));
                o->place_y[t][i] = (float)(mch * ((double)(j % th) + uy));
            }
            free(sz);
            free(cum);
            /* buckets of about four places (order within a bucket is immaterial) */
            int bs = (int)floor(sqrt(4.0 * (double)G / (double)npl));
            if (bs < 1) bs = 1;
            const int nbx = (ncw + bs - 1) / bs, nby = (nch + bs - 1) / bs, NBK = nbx * nby;
            int32_t* bstart = (int32_t*)calloc((size_t)NBK + 1, sizeof(int32_t));
            int32_t* items = (int32_t*)calloc((size_t)npl, sizeof(int32_t));
            int32_t* pb = (int32_t*)calloc((size_t)npl, sizeof(int32_t));
            int32_t* link = (int32_t*)malloc(sizeof(int32_t) * (size_t)n_att);
            int32_t* prop = (int32_t*)malloc(sizeof(int32_t) * (size_t)n_att);
            int32_t* nprop = (int32_t*)calloc((size_t)npl, sizeof(int32_t));
            int32_t* taken = (int32_t*)calloc((size_t)npl, sizeof(int32_t));
            for (int i = 0; i < npl; i++) {
                int cx = (int)(o->place_x[t][i] / S->cell_width), cy = (int)(o->place_y[t][i] / S->cell_height);
                cx = cx < 0 ? 0 : (cx > ncw - 1 ? ncw - 1 : cx);
                cy = cy < 0 ? 0 : (cy > nch - 1 ? nch - 1 : cy);
                pb[i] = (cx / bs) * nby + (cy / bs);
                bstart[pb[i] + 1]++;
            }
            for (int b = 0; b < NBK; b++) bstart[b + 1] += bstart[b];
            {
                int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (size_t)NBK);
                memcpy(cur, bstart, sizeof(int32_t) * (size_t)NBK);
                for (int i = 0; i < npl; i++) items[cur[pb[i]]++] = i;
                free(cur);
            }
            for (int a = 0; a < n_att; a++) link[a] = -1;
            int forced = 0;
            const int nn = T->nearest;
            for (int rd = 0; rd <= S->rounds; rd++) {
                const int free_round = rd == S->rounds;
                for (int a = 0; a < n_att; a++) {
                    prop[a] = -1;
                    if (link[a] >= 0) continue;
                    const int p = list[a];
                    const int h = o->person_hh[p];
                    const float hx = o->hh_x[h], hy = o->hh_y[h];
                    int cx = (int)(hx / S->cell_width), cy = (int)(hy / S->cell_height);
                    cx = cx < 0 ? 0 : (cx > ncw - 1 ? ncw - 1 : cx);
                    cy = cy < 0 ? 0 : (cy > nch - 1 ? nch - 1 : cy);
                    const int bx = cx / bs, by = cy / bs;
                    setup_cand top[CS_SETUP_MAX_NEAREST];
                    int ntop = 0, found = 0, extra = -1;
                    const int rmax = nbx > nby ? nbx : nby;
                    for (int r = 0; r < rmax && extra != 0; r++) {
                        /* the square ring at Chebyshev distance r, any order */
                        for (int x = bx - r; x <= bx + r; x++)
                            for (int y = by - r; y <= by + r; y++) {
                                if (x != bx - r && x != bx + r && y != by - r && y != by + r) continue;
                                if (x < 0 || y < 0 || x >= nbx || y >= nby) continue;
                                const int bk = x * nby + y;
                                for (int e = bstart[bk]; e < bstart[bk + 1]; e++) {
                                    const int pl = items[e];
                                    if (!free_round && rem[pl] <= 0) continue;
                                    found++;
                                    const double d2 = setup_dist2(P, hx, hy, o->place_x[t][pl], o->place_y[t][pl]);
                                    if (ntop == nn && !setup_cand_less(d2, pl, &top[nn - 1])) continue;
                                    int k = (ntop < nn) ? ntop++ : nn - 1;
                                    while (k > 0 && setup_cand_less(d2, pl, &top[k - 1])) { top[k] = top[k - 1]; k--; }
                                    top[k].d2 = d2;
                                    top[k].pl = pl;
                                }
                            }
                        if (extra > 0) extra--;
                        else if (extra < 0 && found >= nn) extra = 1;
                    }
                    if (ntop == 0) continue;
                    double w[CS_SETUP_MAX_NEAREST], tot = 0.0;
                    for (int k = 0; k < ntop; k++) {
                        w[k] = setup_knum(T->kernel_lookup, T->kernel_hi_res, P, top[k].d2) *
                               (free_round ? 1.0 : (double)rem[top[k].pl]);
                        tot = tot + w[k];
                    }
                    int k = 0;
                    if (tot > 0) {
                        stream sc;
                        stream_init(&sc, seed, CS_RNG_SETUP_CHOOSE, (uint32_t)rd, (uint32_t)p, (uint32_t)t);
                        double u = stream_next(&sc) * tot;
                        while (k + 1 < ntop && u >= w[k]) { u -= w[k]; k++; }
                    } else if (!free_round) {
                        continue;
                    }
                    prop[a] = top[k].pl;
                }
                for (int a = 0; a < n_att; a++)
                    if (prop[a] >= 0) nprop[prop[a]]++;
                for (int a = 0; a < n_att; a++) {
                    const int pl = prop[a];
                    if (pl < 0) continue;
                    int ok = 1;
                    if (!free_round && nprop[pl] > rem[pl]) {
                        stream sa;
                        stream_init(&sa, seed, CS_RNG_SETUP_ACCEPT, (uint32_t)rd, (uint32_t)list[a], (uint32_t)t);
                        ok = stream_next(&sa) * (double)nprop[pl] < (double)rem[pl];
                    }
                    if (!ok) continue;
                    link[a] = pl;
                    taken[pl]++;
                    if (free_round) forced++;
                }
                for (int i = 0; i < npl; i++) {
                    rem[i] = rem[i] - taken[i] > 0 ? rem[i] - taken[i] : 0;
                    taken[i] = 0;
                    nprop[i] = 0;
                }
            }
            o->forced[t] = forced;
            /* member lists by (place, random key), then groups */
            setup_key* keys = (setup_key*)malloc(sizeof(setup_key) * (size_t)n_att);
            int32_t* mcount = (int32_t*)calloc((size_t)npl, sizeof(int32_t));
            for (int a = 0; a < n_att; a++)
                if (link[a] < 0) { rc = setup_fail(s, CS_E_OVERFLOW, "setup: an attendee has no place"); goto done; }
            for (int a = 0; a < n_att; a++) {
                const int p = list[a];
                const uint32_t hsh = (uint32_t)setup_rand64(seed, CS_RNG_SETUP_SHUFFLE, 0, (uint32_t)p, (uint32_t)t);
                keys[a].key = ((uint64_t)(uint32_t)link[a] << 32) | hsh;
                keys[a].a = a;
                mcount[link[a]]++;
                o->person_place[(int64_t)t * N + p] = link[a];
            }
            qsort(keys, (size_t)n_att, sizeof(setup_key), setup_key_cmp);
            SETUP_ALLOC(o->place_members[t], n_att, int32_t);
            for (int a = 0; a < n_att; a++) o->place_members[t][a] = list[keys[a].a];
            free(keys);
            SETUP_ALLOC(o->place_member_ofs[t], npl + 1, int32_t);
            SETUP_ALLOC(o->place_group_ofs[t], npl + 1, int32_t);
            int ngt = 0;
            for (int i = 0; i < npl; i++) {
                o->place_member_ofs[t][i + 1] = o->place_member_ofs[t][i] + mcount[i];
                int g = (int)floor((double)mcount[i] / (double)T->group_size + 0.5);
                if (g < 1) g = 1;
                o->place_group_ofs[t][i + 1] = o->place_group_ofs[t][i] + g;
                ngt += g;
            }
            o->n_groups[t] = ngt;
            SETUP_ALLOC(o->group_start[t], ngt, int32_t);
            SETUP_ALLOC(o->group_size[t], ngt, int32_t);
            for (int i = 0; i < npl; i++) {
                const int64_t n = mcount[i], g = o->place_group_ofs[t][i + 1] - o->place_group_ofs[t][i];
                for (int64_t k = 0; k < g; k++) {
                    const int64_t st = (k * n) / g, en = ((k + 1) * n) / g;
                    o->group_start[t][o->place_group_ofs[t][i] + k] = (int32_t)st;
                    o->group_size[t][o->place_group_ofs[t][i] + k] = (int32_t)(en - st);
                    for (int64_t r = st; r < en; r++)
                        o->person_group[(int64_t)t * N + o->place_members[t][o->place_member_ofs[t][i] + r]] =
                            (uint16_t)k;
                }
            }
            free(mcount);
            free(rem);
            free(bstart);
            free(items);
            free(pb);
            free(link);
            free(prop);
            free(nprop);
            free(taken);
        }
    }
    if (err) rc = setup_fail(s, CS_E_OVERFLOW, "setup: a bounded sampling loop gave up");
done:
    free(q);
    free(qb);
    free(pref);
    free(cnt);
    free(mcell_start);
    free(mcell_n);
    free(taken_p);
    free(list);
    return rc;
}

int cs_cpu_setup_run(const cs_setup_spec* spec, const cs_params* params, cs_cpu_setup** out)
{
    if (!out) return CS_E_ARG;
    *out = NULL;
    if (!spec || !params) return CS_E_ARG;
    cs_cpu_setup* s = (cs_cpu_setup*)calloc(1, sizeof(cs_cpu_setup));
    if (!s) return CS_E_ARG;
    *out = s;
    return setup_run(s, spec, params);
}

int cs_cpu_setup_sizes(cs_cpu_setup* s, cs_setup_out* o)
{
    if (!s || !o) return CS_E_ARG;
    const cs_setup_out* a = &s->o;
    o->n_people = a->n_people;
    o->n_households = a->n_households;
    o->n_cells = a->n_cells;
    o->n_mcells = a->n_mcells;
    o->n_adunits = a->n_adunits;
    o->num_place_types = a->num_place_types;
    for (int t = 0; t < CS_MAX_PLACE_TYPES; t++) {
        o->n_places[t] = a->n_places[t];
        o->n_groups[t] = a->n_groups[t];
        o->n_attendees[t] = a->n_attendees[t];
        o->forced[t] = a->forced[t];
    }
    o->device_ms = 0;
    return CS_OK;
}

static void setup_get(void* dst, const void* src, size_t bytes)
{
    if (dst && src && bytes) memcpy(dst, src, bytes);
}

int cs_cpu_setup_download(cs_cpu_setup* s, const cs_setup_out* o)
{
    if (!s || !o) return CS_E_ARG;
    const cs_setup_out* a = &s->o;
    const size_t N = (size_t)a->n_people, NH = (size_t)a->n_households, NM = (size_t)a->n_mcells,
                 NC = (size_t)a->n_cells, npt = (size_t)a->num_place_types;
    setup_get(o->person_hh, a->person_hh, 4 * N);
    setup_get(o->person_mcell, a->person_mcell, 4 * N);
    setup_get(o->person_age, a->person_age, N);
    setup_get(o->person_place, a->person_place, 4 * N * npt);
    setup_get(o->person_group, a->person_group, 2 * N * npt);
    setup_get(o->hh_first, a->hh_first, 4 * NH);
    setup_get(o->hh_nh, a->hh_nh, 2 * NH);
    setup_get(o->hh_x, a->hh_x, 4 * NH);
    setup_get(o->hh_y, a->hh_y, 4 * NH);
    setup_get(o->mcell_cell, a->mcell_cell, 4 * NM);
    setup_get(o->mcell_adunit, a->mcell_adunit, 4 * NM);
    setup_get(o->mcell_grid, a->mcell_grid, 8 * NM);
    setup_get(o->cell_grid, a->cell_grid, 4 * NC);
    setup_get(o->cell_start, a->cell_start, 4 * (NC + 1));
    for (size_t t = 0; t < npt; t++) {
        const size_t np = (size_t)a->n_places[t], na = (size_t)a->n_attendees[t], ng = (size_t)a->n_groups[t];
        setup_get(o->place_mcell[t], a->place_mcell[t], 4 * np);
        setup_get(o->place_x[t], a->place_x[t], 4 * np);
        setup_get(o->place_y[t], a->place_y[t], 4 * np);
        setup_get(o->place_member_ofs[t], a->place_member_ofs[t], 4 * (np + 1));
        setup_get(o->place_members[t], a->place_members[t], 4 * na);
        setup_get(o->place_group_ofs[t], a->place_group_ofs[t], 4 * (np + 1));
        setup_get(o->group_start[t], a->group_start[t], 4 * ng);
        setup_get(o->group_size[t], a->group_size[t], 4 * ng);
    }
    return CS_OK;
}

const char* cs_cpu_setup_last_error(const cs_cpu_setup* s)
{
    return s ? s->err : "null set-up handle";
}

void cs_cpu_setup_destroy(cs_cpu_setup* s)
{
    if (!s) return;
    cs_setup_out* a = &s->o;
    free(a->person_hh); free(a->person_mcell); free(a->person_age); free(a->person_place); free(a->person_group);
    free(a->hh_first); free(a->hh_nh); free(a->hh_x); free(a->hh_y);
    free(a->mcell_cell); free(a->mcell_adunit); free(a->mcell_grid); free(a->cell_grid); free(a->cell_start);
    for (int t = 0; t < CS_MAX_PLACE_TYPES; t++) {
        free(a->place_mcell[t]); free(a->place_x[t]); free(a->place_y[t]); free(a->place_member_ofs[t]);
        free(a->place_members[t]); free(a->place_group_ofs[t]); free(a->group_start[t]); free(a->group_size[t]);
    }
    free(s);
}

/* S, L, I, R, D of every cell as 16-bit values side by side (cs_gpu_get_sample16). */
int cs_cpu_get_cells16(cs_cpu_ctx* c, uint16_t* out)
{
    const int NC = c->NC;
    for (int k = 0; k < NC; k++) {
        if (c->cell_start[k + 1] - c->cell_start[k] > 65535) return fail(c, CS_E_RANGE, "a cell holds more than 65535 people");
        out[k] = (uint16_t)c->S[k];
        out[NC + k] = (uint16_t)c->L[k];
        out[2 * NC + k] = (uint16_t)c->I[k];
        out[3 * NC + k] = (uint16_t)c->R[k];
        out[4 * NC + k] = (uint16_t)c->D[k];
    }
    return CS_OK;
}

size_t cs_cpu_sample_packed_bytes(const cs_cpu_ctx* c)
{
    return sizeof(cs_counters) + sizeof(uint16_t) * 5 * (size_t)c->NC;
}
