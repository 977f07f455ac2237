// Device-side building blocks of the sweep: random streams, samplers, the spatial
// kernel lookup, distances and the infectiousness / susceptibility products.
//
// The library is compiled with --fmad=false so that every floating-point
// expression rounds exactly as written (no fused multiply-adds); together with
// counter-based random streams this makes a run's results a function of
// (population, parameters, seed) alone.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "covidsim_b200.h"
#include "cs_state.h"

namespace csb {

constexpr int kMaxLoop = 1000;
constexpr int kMaxSpatialTries = 100000;
constexpr uint16_t kNever = 65534;  // USHRT_MAX - 1

// src/Constants.h:10-58: EARTHRADIUS = (1852*60*360 / PI) / 2 with PI = 3.1415926535.
#define CSB_EARTH_RADIUS (((double)40003200) / 3.1415926535 / 2)
#define CSB_REF_PI 3.1415926535

// ----------------------------------------------------------------- Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
__device__ __forceinline__ void philox4x32_10(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1,
                                              uint32_t c2, uint32_t c3, uint32_t out[4])
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// One counter-based stream: {block, entity, ts | purpose << 16, sub} under the run key.
struct Stream {
    uint32_t k0, k1, c1, c2, c3, block;
    double buf[2];
    int idx;

    __device__ __forceinline__ Stream(uint64_t seed, int purpose, uint32_t ts, uint32_t entity, uint32_t sub)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), c1(entity),
          c2((ts & 0xffffu) | ((uint32_t)purpose << 16)), c3(sub), block(0), idx(2) {}

    __device__ __forceinline__ double next()
    {
        if (idx >= 2) {
            uint32_t x[4];
            philox4x32_10(k0, k1, block++, c1, c2, c3, x);
            uint64_t a = ((uint64_t)x[1] << 32) | x[0];
            uint64_t b = ((uint64_t)x[3] << 32) | x[2];
            buf[0] = (double)(a >> 11) * (1.0 / 9007199254740992.0);
            buf[1] = (double)(b >> 11) * (1.0 / 9007199254740992.0);
            idx = 0;
        }
        return buf[idx++];
    }
};

// ------------------------------------------------------------------ samplers
// Poisson: inversion below 10, else PTRS (Hormann 1993, "The transformed rejection
// method for generating Poisson random variables"); the reference's ignpoi_mt
// (src/Rand.cpp:170-402) samples the same distribution by Ahrens-Dieter.
__device__ inline int32_t sample_poisson(Stream& s, double lambda, unsigned long long* err)
{
    if (!(lambda > 0)) return 0;
    if (lambda < 10.0) {
        double u = s.next();
        double p = exp(-lambda), F = p;
        int32_t k = 0;
        while (u > F && k < kMaxLoop) {
            k++;
            p = p * lambda / (double)k;
            F = F + p;
        }
        return k;
    }
    double slam = sqrt(lambda), loglam = log(lambda);
    double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
    double invalpha = 1.1239 + 1.1328 / (b - 3.4), vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int it = 0; it < kMaxLoop; it++) {
        double U = s.next() - 0.5;
        double V = s.next();
        double us = 0.5 - fabs(U);
        double k = floor((2.0 * a / us + b) * U + lambda + 0.43);
        if (us >= 0.07 && V <= vr) return (int32_t)k;
        if (k < 0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -lambda + k * loglam - lgamma(k + 1.0))
            return (int32_t)k;
    }
    atomicAdd(err, 1ull);
    return (int32_t)lambda;
}

// Standard normal, Marsaglia's polar method.
__device__ inline double sample_normal(Stream& s, unsigned long long* err)
{
    for (int it = 0; it < kMaxLoop; it++) {
        double v1 = 2.0 * s.next() - 1.0;
        double v2 = 2.0 * s.next() - 1.0;
        double r = v1 * v1 + v2 * v2;
        if (r > 0.0 && r < 1.0) return v1 * sqrt(-2.0 * log(r) / r);
    }
    atomicAdd(err, 1ull);
    return 0.0;
}

// Gamma(shape alpha, rate beta), Marsaglia-Tsang as gen_gamma_mt (src/Rand.cpp:1025-1096).
__device__ inline double sample_gamma(Stream& s, double beta, double alpha, unsigned long long* err)
{
    double a = (alpha >= 1.0) ? alpha : alpha + 1.0;
    double d = a - (1.0 / 3.0);
    double c = 1.0 / (3.0 * sqrt(d));
    double u, z, v;
    int it = 0;
    do {
        u = s.next();
        z = sample_normal(s, err);
        v = 1.0 + z * c;
        v = v * v * v;
        if (++it > kMaxLoop) { atomicAdd(err, 1ull); break; }
    } while ((z <= (-1.0 / c)) || (log(u) >= (0.5 * z * z + d - d * v + d * log(v))));
    double g = (beta != 1.0) ? (d * v) / beta : d * v;
    if (alpha < 1.0) g = g * pow(s.next(), 1.0 / alpha);
    return g;
}

// InverseCdf::choose (src/InverseCdf.cpp:60-74).
__device__ __forceinline__ uint16_t icdf_choose(const cs_icdf& icdf, double mean, double u, double spd)
{
    double q;
    int i = (int)floor(q = u * CS_CDF_RES);
    q -= (double)i;
    double ti = -mean * log(q * icdf.v[i + 1] + (1.0 - q) * icdf.v[i]);
    return (uint16_t)floor(0.5 + (ti * spd));
}

// ------------------------------------------------------- kernel & distance
// KernelLookup::num (src/Kernels.cpp:108-129); out-of-table distances count as errors.
__device__ __forceinline__ double knum(const DevPop& d, const cs_params& P, double r2, unsigned long long* err)
{
    double t = r2 / P.kernel_delta;
    if (t > P.kernel_size) { atomicAdd(err, 1ull); return 0.0; }
    double s = t * P.kernel_expansion;
    if (s < P.kernel_size) {
        t = s - floor(s);
        t = (1.0 - t) * __ldg(d.khires + (int)s) + t * __ldg(d.khires + (int)(s + 1.0));
    } else {
        int i0 = (int)t, i1 = (int)(t + 1.0);
        if (i1 > P.kernel_size) i1 = P.kernel_size;
        s = t - floor(t);
        t = (1.0 - s) * __ldg(d.klookup + i0) + s * __ldg(d.klookup + i1);
    }
    return t;
}

// KernelLookup::num over the FP32 copies of the tables (values within 2^-24
// relative of the doubles), interpolated in double; an out-of-table distance sets
// *oor instead of counting an error.  The spatial pass's acceptance test reads it:
// half the bytes of the double tables per random lookup.
__device__ __forceinline__ double knum_f32(const DevPop& d, const cs_params& P, double r2, int* oor)
{
    double t = r2 / P.kernel_delta;
    if (t > P.kernel_size) { *oor = 1; return 0.0; }
    double s = t * P.kernel_expansion;
    if (s < P.kernel_size) {
        t = s - floor(s);
        t = (1.0 - t) * (double)__ldg(d.khires_f + (int)s) + t * (double)__ldg(d.khires_f + (int)(s + 1.0));
    } else {
        int i0 = (int)t, i1 = (int)(t + 1.0);
        if (i1 > P.kernel_size) i1 = P.kernel_size;
        s = t - floor(t);
        t = (1.0 - s) * (double)__ldg(d.klookup_f + i0) + s * (double)__ldg(d.klookup_f + i1);
    }
    return t;
}

// KernelLookup::num for a caller that decides later whether the evaluation counts:
// an out-of-table distance sets *oor instead of counting an error.
__device__ __forceinline__ double knum_flag(const DevPop& d, const cs_params& P, double r2, int* oor)
{
    double t = r2 / P.kernel_delta;
    if (t > P.kernel_size) { *oor = 1; return 0.0; }
    double s = t * P.kernel_expansion;
    if (s < P.kernel_size) {
        t = s - floor(s);
        t = (1.0 - t) * __ldg(d.khires + (int)s) + t * __ldg(d.khires + (int)(s + 1.0));
    } else {
        int i0 = (int)t, i1 = (int)(t + 1.0);
        if (i1 > P.kernel_size) i1 = P.kernel_size;
        s = t - floor(t);
        t = (1.0 - s) * __ldg(d.klookup + i0) + s * __ldg(d.klookup + i1);
    }
    return t;
}

// dist2UTM (src/Dist.cpp:23-48).
__device__ inline double dist2_utm(const cs_params& P, double x1, double y1, double x2, double y2)
{
    double x, y, cy1, cy2, yt, xi, yi;
    x = fabs(x1 - x2) / 2;
    y = fabs(y1 - y2) / 2;
    xi = floor(x);
    yi = floor(y);
    x -= xi;
    y -= yi;
    x = (1 - x) * P.sinx[(int)xi] + x * P.sinx[((int)xi) + 1];
    y = (1 - y) * P.sinx[(int)yi] + y * P.sinx[((int)yi) + 1];
    yt = fabs(y1 + P.bbox_bottom_left_y);
    yi = floor(yt);
    cy1 = yt - yi;
    cy1 = (1 - cy1) * P.cosx[((int)yi)] + cy1 * P.cosx[((int)yi) + 1];
    yt = fabs(y2 + P.bbox_bottom_left_y);
    yi = floor(yt);
    cy2 = yt - yi;
    cy2 = (1 - cy2) * P.cosx[((int)yi)] + cy2 * P.cosx[((int)yi) + 1];
    x = fabs(1000 * (y * y + x * x * cy1 * cy2));
    xi = floor(x);
    x -= xi;
    y = (1 - x) * P.asin2sqx[((int)xi)] + x * P.asin2sqx[((int)xi) + 1];
    return 4 * CSB_EARTH_RADIUS * CSB_EARTH_RADIUS * y;
}

// periodic_xy (src/Dist.cpp:13-21).
__device__ __forceinline__ double periodic_xy(const cs_params& P, double x, double y)
{
    if (P.DoPeriodicBoundaries) {
        if (x > P.width_deg * 0.5) x = P.width_deg - x;
        if (y > P.height_deg * 0.5) y = P.height_deg - y;
    }
    return x * x + y * y;
}

// dist2(Person*, Person*) (src/Dist.cpp:49-61) between two households.
__device__ __forceinline__ double dist2_hh(const DevPop& d, const cs_params& P, int32_t ha, int32_t hb)
{
    float2 a = __ldg(reinterpret_cast<const float2*>(d.hhr + ha));
    float2 b = __ldg(reinterpret_cast<const float2*>(d.hhr + hb));
    float ax = a.x, ay = a.y, bx = b.x, by = b.y;
    if (P.DoUTM_coords) return dist2_utm(P, ax, ay, bx, by);
    float dx = ax - bx, dy = ay - by;
    return periodic_xy(P, fabs(dx), fabs(dy));
}

// dist2_raw (src/Dist.cpp:163-170), in double from float locations: from a
// household to a point (a place), and between two households.
__device__ __forceinline__ double dist2_raw(const cs_params& P, double ax, double ay, double bx, double by)
{
    if (P.DoUTM_coords) return dist2_utm(P, ax, ay, bx, by);
    return periodic_xy(P, fabs(ax - bx), fabs(ay - by));
}
__device__ __forceinline__ double dist2_hh_pt(const DevPop& d, const cs_params& P, int32_t ha, float bx, float by)
{
    float2 a = __ldg(reinterpret_cast<const float2*>(d.hhr + ha));
    return dist2_raw(P, a.x, a.y, bx, by);
}
__device__ __forceinline__ double dist2_hh_raw(const DevPop& d, const cs_params& P, int32_t ha, int32_t hb)
{
    float2 b = __ldg(reinterpret_cast<const float2*>(d.hhr + hb));
    return dist2_hh_pt(d, P, ha, b.x, b.y);
}

// dist2_cc_min (src/Dist.cpp:78-144) on grid cell indices.
__device__ inline double dist2_cc_min(const cs_params& P, int l, int m)
{
    int nch = P.nch, i = l, j = m;
    if (P.DoUTM_coords) {
        if (P.cell_width * ((double)abs(m / nch - l / nch)) > CSB_REF_PI) {
            if (m / nch > l / nch) j += nch;
            else if (m / nch < l / nch) i += nch;
        } else {
            if (m / nch > l / nch) i += nch;
            else if (m / nch < l / nch) j += nch;
        }
        if (m % nch > l % nch) i++;
        else if (m % nch < l % nch) j++;
        return dist2_utm(P, P.cell_width * fabs((double)(i / nch)), P.cell_height * fabs((double)(i % nch)),
                         P.cell_width * fabs((double)(j / nch)), P.cell_height * fabs((double)(j % nch)));
    }
    if ((P.DoPeriodicBoundaries) && (P.cell_width * ((double)abs(m / nch - l / nch)) > P.width_deg * 0.5)) {
        if (m / nch > l / nch) j += nch;
        else if (m / nch < l / nch) i += nch;
    } else {
        if (m / nch > l / nch) i += nch;
        else if (m / nch < l / nch) j += nch;
    }
    if ((P.DoPeriodicBoundaries) && (P.height_deg * ((double)abs(m % nch - l % nch)) > P.height_deg * 0.5)) {
        if (m % nch > l % nch) j++;
        else if (m % nch < l % nch) i++;
    } else {
        if (m % nch > l % nch) i++;
        else if (m % nch < l % nch) j++;
    }
    double x = P.cell_width * fabs((double)(i / nch - j / nch));
    double y = P.cell_height * fabs((double)(i % nch - j % nch));
    return periodic_xy(P, x, y);
}

// Upper bound of K(d) over all point pairs in proposal blocks b and B: the kernel
// at the blocks' closest-corner distance, d^2 shrunk by 2% so table interpolation
// never lifts K(d)/bound above 1.
__device__ inline double block_bound(const DevPop& d, const cs_params& P, int b, int B, unsigned long long* err)
{
    if (P.DoPeriodicBoundaries) return knum(d, P, 0.0, err);
    int bx = b / d.nby, by = b % d.nby, Bx = B / d.nby, By = B % d.nby, bs = d.bs;
    int xa, xb, ya, yb;
    if (Bx > bx) { xa = (bx + 1) * bs; xb = Bx * bs; }
    else if (Bx < bx) { xa = bx * bs; xb = (Bx + 1) * bs; }
    else { xa = xb = bx * bs; }
    if (By > by) { ya = (by + 1) * bs; yb = By * bs; }
    else if (By < by) { ya = by * bs; yb = (By + 1) * bs; }
    else { ya = yb = by * bs; }
    double d2;
    if (P.DoUTM_coords)
        d2 = dist2_utm(P, P.cell_width * (double)xa, P.cell_height * (double)ya, P.cell_width * (double)xb, P.cell_height * (double)yb);
    else {
        double x = P.cell_width * fabs((double)(xa - xb)), y = P.cell_height * fabs((double)(ya - yb));
        d2 = x * x + y * y;
    }
    d2 = d2 * 0.98;
    return knum(d, P, d2, err);
}

// The same bound by (row of b, row of B, column distance dx in blocks): the
// closest corners are dx - 1 blocks apart in x (none for dx = 0) and at the rows'
// facing edges in y; the great-circle distance depends on x only through the
// difference and on y through both latitudes.
__device__ inline double block_bound_rel(const DevPop& d, const cs_params& P, int by, int By, int dx, unsigned long long* err)
{
    if (P.DoPeriodicBoundaries) return knum(d, P, 0.0, err);
    const int bs = d.bs, g = dx > 0 ? (dx - 1) * bs : 0;
    int ya, yb;
    if (By > by) { ya = (by + 1) * bs; yb = By * bs; }
    else if (By < by) { ya = by * bs; yb = (By + 1) * bs; }
    else { ya = yb = by * bs; }
    double d2;
    if (P.DoUTM_coords)
        d2 = dist2_utm(P, P.cell_width * (double)g, P.cell_height * (double)ya, 0.0, P.cell_height * (double)yb);
    else {
        double x = P.cell_width * (double)g, y = P.cell_height * fabs((double)(ya - yb));
        d2 = x * x + y * y;
    }
    d2 = d2 * 0.98;
    return knum(d, P, d2, err);
}

// bound(b, B) for the proposal and the acceptance test alike, so that their
// product stays exactly K(d): the compact FP32 table, or the per-call table.
__device__ __forceinline__ double bound_of(const DevPop& d, int b, int B)
{
    if (d.bounds_static) {
        const int bx = b / d.nby, by = b % d.nby, Bx = B / d.nby, By = B % d.nby;
        return (double)__ldg(d.bound_c + ((size_t)by * d.nby + By) * d.nbx + (bx > Bx ? bx - Bx : Bx - bx));
    }
    return d.block_bound_tab[(size_t)b * d.NB + B];
}

// ------------------------------------------------------------- state macros
// src/ModelMacros.h:6-20 over the device person record.
__device__ __forceinline__ int age_group(const PersonHot& h) { return h.age / CS_AGE_GROUP_WIDTH; }
__device__ __forceinline__ bool host_absent(const PersonHot& h, int ts) { return h.absent_start <= ts && h.absent_stop > ts; }
__device__ __forceinline__ int quar_comply(const PersonHot& h) { return (h.dflags & CS_DF_QUAR_COMPLY_MASK) >> CS_DF_QUAR_COMPLY_SHIFT; }
__device__ __forceinline__ bool host_quarantined(const PersonHot& h, const cs_params& P, int ts)
{
    return quar_comply(h) == 1 && (int)h.quar_start + (int)P.usHQuarantineHouseDuration > ts && h.quar_start <= ts;
}
__device__ __forceinline__ bool host_to_be_quarantined(const PersonHot& h, const cs_params& P, int ts)
{
    return (int)h.quar_start + (int)P.usHQuarantineHouseDuration > ts && quar_comply(h) < 2;
}
__device__ __forceinline__ bool host_isolated(const PersonHot& h, const cs_params& P, int ts)
{
    int s = (int)h.isolation_start + (int)P.usCaseIsolationDelay;
    return s <= ts && s + (int)P.usCaseIsolationDuration > ts;
}
__device__ __forceinline__ bool is_ch(const PersonHot& h) { return (h.pflags & CS_PF_CARE_HOME_RESIDENT) != 0; }
__device__ __forceinline__ bool is_alive(int8_t inf) { return inf != CS_INF_DEAD_WAS_ASYMP && inf != CS_INF_DEAD_WAS_SYMP; }
__device__ __forceinline__ bool place_closed(const DevPop& d, int pt, int pl, int ts)
{
    return d.pl[pt].close_start[pl] <= ts && d.pl[pt].close_end[pl] > ts;
}
// False when no place can be closed at ts, so the per-place checks can be skipped.
__device__ __forceinline__ bool closures_possible(const DevPop& d, int ts)
{
    return d.close_window[0] <= ts && ts < d.close_window[1];
}
__device__ __forceinline__ int link_of(const DevPop& d, int pt, int p) { return __ldg(&d.links[p].link[pt]); }
__device__ __forceinline__ int group_of(const DevPop& d, int pt, int p) { return __ldg(&d.links[p].group[pt]); }
// Whole records, as two and one 16-byte loads.
__device__ __forceinline__ PersonLinks load_links(const DevPop& d, int p)
{
    const int4* q = reinterpret_cast<const int4*>(d.links + p);
    int4 a = __ldg(q), b = __ldg(q + 1);
    PersonLinks r;
    static_assert(sizeof(r) == 2 * sizeof(int4), "layout");
    reinterpret_cast<int4*>(&r)[0] = a;
    reinterpret_cast<int4*>(&r)[1] = b;
    return r;
}
__device__ __forceinline__ HouseholdRec load_household(const DevPop& d, int h)
{
    int4 a = __ldg(reinterpret_cast<const int4*>(d.hhr + h));
    HouseholdRec r;
    reinterpret_cast<int4*>(&r)[0] = a;
    return r;
}

// --------------------------------------- CalcInfSusc (src/CalcInfSusc.cpp)
// Factors that are exactly 1.0 here (digital contact tracing, treatment,
// vaccination) are left out; multiplying by 1.0 is exact.
__device__ __forceinline__ double calc_person_inf(const PersonHot& h, const cs_params& P, int ts)
{
    return fabs(h.infness) * P.infectiousness[ts - h.latent_time - 1];
}
__device__ __forceinline__ double calc_house_inf(const PersonHot& h, uint16_t nhr, const cs_params& P, int ts)
{
    bool iso = host_isolated(h, P, ts);
    double infn = P.NoInfectiousnessSDinHH ? ((h.infness < 0) ? P.SymptInfectiousness : P.AsymptInfectiousness) : fabs(h.infness);
    return (iso ? P.Efficacies[CS_NPI_CASE_ISOLATION][CS_SETTING_HOUSE] : 1.0)
        * ((host_quarantined(h, P, ts) && !iso) ? P.Efficacies[CS_NPI_HOME_QUARANTINE][CS_SETTING_HOUSE] : 1.0)
        * P.HouseholdDenomLookup[nhr - 1]
        * (is_ch(h) ? P.CareHomeResidentHouseholdScaling : 1.0)
        * infn
        * P.infectiousness[ts - h.latent_time - 1];
}
__device__ __forceinline__ double calc_place_inf(const PersonHot& h, const cs_params& P, int pt, int ts)
{
    bool iso = host_isolated(h, P, ts), ch = is_ch(h);
    return (iso ? P.Efficacies[CS_NPI_CASE_ISOLATION][pt] : 1.0)
        * ((host_quarantined(h, P, ts) && !ch && !iso) ? P.Efficacies[CS_NPI_HOME_QUARANTINE][pt] : 1.0)
        * ((h.inf == CS_INF_CASE && !ch) ? P.SymptPlaceTypeContactRate[pt] : 1.0)
        * P.PlaceTypeTrans[pt] / P.PlaceTypeGroupSizeParam1[pt] * calc_person_inf(h, P, ts);
}
__device__ __forceinline__ double calc_spatial_inf(const PersonHot& h, const cs_params& P, int ts)
{
    bool iso = host_isolated(h, P, ts), ch = is_ch(h);
    return (iso ? P.Efficacies[CS_NPI_CASE_ISOLATION][CS_SETTING_SPATIAL] : 1.0)
        * ((host_quarantined(h, P, ts) && !ch && !iso) ? P.Efficacies[CS_NPI_HOME_QUARANTINE][CS_SETTING_SPATIAL] : 1.0)
        * ((h.inf == CS_INF_CASE) ? P.SymptSpatialContactRate : 1.0)
        * P.RelativeSpatialContact[age_group(h)]
        * calc_person_inf(h, P, ts);
}
__device__ __forceinline__ double calc_person_susc(const PersonHot& h, int infector_age_group, const cs_params& P)
{
    int a = age_group(h);
    return P.WAIFW_Matrix[a][infector_age_group] * P.AgeSusceptibility[a] * h.susc;
}
__device__ __forceinline__ double socdist_factor(const DevPop& d, const PersonHot& h, const cs_params& P, int setting)
{
    if (d.socdist[h.mcell] != CS_TREAT_TREATED) return 1.0;
    return (h.pflags & CS_PF_ESOCDIST_COMPLY) ? P.Efficacies[CS_NPI_ENHANCED_SOCIAL_DISTANCING][setting]
                                             : P.Efficacies[CS_NPI_SOCIAL_DISTANCING][setting];
}
__device__ __forceinline__ double calc_house_susc(const DevPop& d, const PersonHot& h, int infector_age_group, const cs_params& P)
{
    return calc_person_susc(h, infector_age_group, P) * socdist_factor(d, h, P, CS_SETTING_HOUSE)
        * (is_ch(h) ? P.CareHomeResidentHouseholdScaling : 1.0);
}
__device__ __forceinline__ double calc_place_susc(const DevPop& d, const PersonHot& h, const cs_params& P, int pt, int ts)
{
    return ((host_quarantined(h, P, ts) && !is_ch(h)) ? P.Efficacies[CS_NPI_HOME_QUARANTINE][pt] : 1.0)
        * socdist_factor(d, h, P, pt);
}
__device__ __forceinline__ double calc_spatial_susc(const DevPop& d, const PersonHot& h, const cs_params& P, int ts)
{
    return ((host_quarantined(h, P, ts) && !is_ch(h)) ? P.Efficacies[CS_NPI_HOME_QUARANTINE][CS_SETTING_SPATIAL] : 1.0)
        * socdist_factor(d, h, P, CS_SETTING_SPATIAL)
        * P.RelativeSpatialContactSusc[age_group(h)];
}
__device__ __forceinline__ bool moverest_differs(const DevPop& d, int ma, int mb)
{
    uint8_t a = d.moverest[ma], b = d.moverest[mb];
    return a != b && (a == CS_TREAT_TREATED || b == CS_TREAT_TREATED);
}

}  // namespace csb
