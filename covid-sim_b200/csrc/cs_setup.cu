// Population set-up on the GPU (cs_gpu_setup_*): the steps of the reference's
// SetupModel that build the sweep's inputs -- microcell populations
// (src/SetupModel.cpp:1137-1156), people numbered cell by cell (:1163-1185),
// households and their locations (:1224-1290), and the assignment of people to
// places (AssignPeopleToPlaces, :1989-2466) -- as parallel kernels on the
// counter-based streams.  Every random draw is keyed by (seed, purpose, entity),
// every sum is an integer sum or has a fixed order, and the only atomics are
// integer counts, so the result is a function of the spec alone.
//
// Work is one thread per microcell, person, household or place; the passes that
// need an order (people per cell, households per microcell, places' member lists)
// take it from exclusive scans and one stable radix sort, written below.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdarg>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "covidsim_b200.h"
#include "cs_device.cuh"

using namespace csb;

namespace {

constexpr int kT = 256;          // threads per block
constexpr int kItems = 8;        // items per thread in scans and the radix sort
constexpr int kTile = kT * kItems;

struct Blob { double cx, cy, rad, wt; };

// ------------------------------------------------------------ random helpers
// 64 random bits: block 0 of the stream {0, entity, ts | purpose << 16, sub}.
__device__ __forceinline__ uint64_t rand64(uint64_t seed, int purpose, uint32_t ts, uint32_t entity, uint32_t sub)
{
    uint32_t x[4];
    philox4x32_10((uint32_t)seed, (uint32_t)(seed >> 32), 0u, entity, (ts & 0xffffu) | ((uint32_t)purpose << 16),
                  sub, x);
    return ((uint64_t)x[1] << 32) | x[0];
}

// KernelLookup::num (src/Kernels.cpp:108-129) over a place type's tables.
__device__ __forceinline__ double knum_tab(const double* lk, const double* hr, const cs_params& P, double r2)
{
    double t = r2 / P.kernel_delta;
    if (t > P.kernel_size) return 0.0;
    double s = t * P.kernel_expansion;
    if (s < P.kernel_size) {
        t = s - floor(s);
        return (1.0 - t) * hr[(int)s] + t * hr[(int)(s + 1.0)];
    }
    int i0 = (int)t, i1 = (int)(t + 1.0);
    if (i1 > P.kernel_size) i1 = P.kernel_size;
    s = t - floor(t);
    return (1.0 - s) * lk[i0] + s * lk[i1];
}

// Household-to-place distance^2 as the sweep measures distances (dist2_raw).
__device__ __forceinline__ double dist2_pts(const cs_params& P, float ax, float ay, float bx, float by)
{
    if (P.DoUTM_coords) return dist2_utm(P, ax, ay, bx, by);
    float dx = ax - bx, dy = ay - by;
    return periodic_xy(P, fabs(dx), fabs(dy));
}

// ------------------------------------------------------------------- scans
// Exclusive (or inclusive) prefix sums of integer arrays, in three passes: block
// totals, a one-block scan of the totals, and the scan of each tile from its
// block's offset.  Integer addition is associative, so the result does not depend
// on the tiling.
template <typename T>
__device__ __forceinline__ T block_exclusive(T v, T* sh, T* total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        T s = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : (T)0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < (int)(blockDim.x >> 5)) sh[lane] = s;   // inclusive over warps
    }
    __syncthreads();
    T warp_ofs = (w > 0) ? sh[w - 1] : (T)0;
    *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();   // sh is reused by the caller's next call
    return warp_ofs + x - v;
}

template <typename Tin, typename T>
__global__ void __launch_bounds__(kT) k_scan_reduce(const Tin* __restrict__ in, long long n, T* __restrict__ bsum)
{
    __shared__ T sh[32];
    long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kItems;
    T s = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++)
        if (base + k < n) s += (T)in[base + k];
    T tot;
    block_exclusive<T>(s, sh, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

template <typename T>
__global__ void __launch_bounds__(1024) k_scan_totals(T* __restrict__ bsum, long long nb, T* __restrict__ grand)
{
    __shared__ T sh[32];
    T carry = 0;
    for (long long b0 = 0; b0 < nb; b0 += blockDim.x) {
        long long i = b0 + threadIdx.x;
        T v = (i < nb) ? bsum[i] : (T)0;
        T tot;
        T ex = block_exclusive<T>(v, sh, &tot);
        if (i < nb) bsum[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && grand) *grand = carry;
}

template <typename Tin, typename T>
__global__ void __launch_bounds__(kT) k_scan_apply(const Tin* __restrict__ in, long long n, const T* __restrict__ bsum,
                                                   T* __restrict__ out, int inclusive)
{
    __shared__ T sh[32];
    long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kItems;
    T v[kItems];
    T s = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        v[k] = (base + k < n) ? (T)in[base + k] : (T)0;
        s += v[k];
    }
    T tot;
    T run = bsum[blockIdx.x] + block_exclusive<T>(s, sh, &tot);
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        if (base + k < n) out[base + k] = inclusive ? run + v[k] : run;
        run += v[k];
    }
}

// ------------------------------------------------------------ radix sort
// Stable LSD radix sort of (key, value) pairs, 8 bits per pass.  Each block owns a
// tile of kTile consecutive pairs; the per-(digit, block) counts are scanned digit-
// major, so a pair's destination is the count of smaller digits, plus that of its
// digit in earlier blocks, plus its rank among equal digits earlier in its tile.
__global__ void __launch_bounds__(kT) k_radix_hist(const uint64_t* __restrict__ keys, long long n, int shift,
                                                  uint32_t* __restrict__ hist, long long nb)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kTile;
    for (int k = threadIdx.x; k < kTile; k += kT) {
        long long i = base + k;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(long long)threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kT) k_radix_scatter(const uint64_t* __restrict__ kin, const int32_t* __restrict__ vin,
                                                     long long n, int shift, const uint32_t* __restrict__ ofs,
                                                     long long nb, uint64_t* __restrict__ kout,
                                                     int32_t* __restrict__ vout)
{
    __shared__ uint32_t base_d[256];
    __shared__ uint32_t wcnt[kT / 32][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    base_d[threadIdx.x] = ofs[(long long)threadIdx.x * nb + blockIdx.x];
    __syncthreads();
    const long long tile = (long long)blockIdx.x * kTile;
    for (int it = 0; it < kItems; it++) {
        const long long i = tile + (long long)it * kT + threadIdx.x;
        const bool valid = i < n;
        uint64_t key = valid ? kin[i] : 0;
        int32_t val = valid ? vin[i] : 0;
        const int digit = valid ? (int)((key >> shift) & 255u) : 256 + lane;   // invalid lanes: no peers
        for (int k = lane; k < 256; k += 32) wcnt[w][k] = 0;
        __syncthreads();
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank == 0) wcnt[w][digit] = (uint32_t)__popc(peers);
        __syncthreads();
        {   // thread d: running offsets of digit d over the warps, in warp order
            const int d = threadIdx.x;
            uint32_t run = base_d[d];
            for (int ww = 0; ww < kT / 32; ww++) {
                uint32_t c = wcnt[ww][d];
                wcnt[ww][d] = run;
                run += c;
            }
            base_d[d] = run;
        }
        __syncthreads();
        if (valid) {
            const uint32_t dst = wcnt[w][digit] + (uint32_t)rank;
            kout[dst] = key;
            vout[dst] = val;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------- density and people
__global__ void k_blobs(uint64_t seed, int nb, Blob* __restrict__ out, unsigned long long* err)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    Stream s(seed, CS_RNG_SETUP_BLOB, 0, (uint32_t)k, 0);
    Blob b;
    b.cx = 0.05 + 0.9 * s.next();
    b.cy = 0.05 + 0.9 * s.next();
    b.rad = 0.004 + 0.016 * s.next();
    b.wt = exp(0.7 * sample_normal(s, err));
    out[k] = b;
}

// Microcell weights: lognormal(0, sigma) quantised to integers (w * 2^20), and the
// blobs' weight the same way.
__global__ void k_density(uint64_t seed, double sigma, long long M, int tw, int th, const Blob* __restrict__ blobs,
                          int nb, uint64_t* __restrict__ q, uint64_t* __restrict__ qb, unsigned long long* err)
{
    long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    Stream s(seed, CS_RNG_SETUP_DENSITY, 0, (uint32_t)j, 0);
    double w = exp(sigma * sample_normal(s, err));
    q[j] = (uint64_t)floor(w * 1048576.0);
    if (nb > 0) {
        const double xs = ((double)(j / th) + 0.5) / (double)tw;
        const double ys = ((double)(j % th) + 0.5) / (double)th;
        double b = 0.0;
        for (int k = 0; k < nb; k++) {
            const Blob bl = blobs[k];
            const double ax = (xs - bl.cx) / bl.rad, ay = (ys - bl.cy) / bl.rad;
            b = b + bl.wt * exp(-0.5 * ax * ax) * exp(-0.5 * ay * ay);
        }
        qb[j] = (uint64_t)floor(b * 1048576.0);
    }
}

// Blend: (1 - share) of the lognormal weight and share of the blobs', each
// normalised by its integer total, at 2^52 resolution.
__global__ void k_blend(long long M, double share, const uint64_t* __restrict__ QW, const uint64_t* __restrict__ QB,
                        uint64_t* __restrict__ q, const uint64_t* __restrict__ qb)
{
    long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    const double a = (double)q[j] / (double)*QW, b = (double)qb[j] / (double)*QB;
    q[j] = (uint64_t)floor(((1.0 - share) * a + share * b) * 4503599627370496.0);
}

// Each person draws its microcell: r in [0, total) from 64 random bits, then the
// first microcell whose inclusive prefix exceeds r.
__global__ void k_people_to_mcells(uint64_t seed, int N, const uint64_t* __restrict__ pref, long long M,
                                   int32_t* __restrict__ cnt)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const uint64_t tot = pref[M - 1];
    const uint64_t r = __umul64hi(rand64(seed, CS_RNG_SETUP_PERSON, 0, (uint32_t)k, 0), tot);
    long long lo = 0, hi = M - 1;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (pref[mid] > r) hi = mid; else lo = mid + 1;
    }
    atomicAdd(cnt + lo, 1);
}

// The microcell grid index of microcell (l, m) of grid cell c, in the reference's
// order within a cell (src/SetupModel.cpp:1166-1172): x offset l outer, y offset m.
__device__ __forceinline__ long long mcell_of(int c, int l, int m, int nch, int nmcl, int th)
{
    return (long long)((c / nch) * nmcl + l) * th + (long long)(c % nch) * nmcl + m;
}

__global__ void k_cell_sums(int G, int nch, int nmcl, int th, const int32_t* __restrict__ cnt,
                            int32_t* __restrict__ cell_n, int32_t* __restrict__ cell_pm, int32_t* __restrict__ cell_pop)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= G) return;
    int n = 0, pm = 0;
    for (int l = 0; l < nmcl; l++)
        for (int m = 0; m < nmcl; m++) {
            int v = cnt[mcell_of(c, l, m, nch, nmcl, th)];
            n += v;
            pm += v > 0;
        }
    cell_n[c] = n;
    cell_pm[c] = pm;
    cell_pop[c] = n > 0;
}

// Populated cells and microcells in the reference's order, with person offsets.
__global__ void k_cells(int G, int nch, int nmcl, int th, int tw, int adunit_grid, const int32_t* __restrict__ cnt,
                        const int32_t* __restrict__ cell_n, const int32_t* __restrict__ cell_person_ofs,
                        const int32_t* __restrict__ cell_mc_ofs, const int32_t* __restrict__ cell_id_ofs,
                        int32_t* __restrict__ cell_grid, int32_t* __restrict__ cell_start,
                        int32_t* __restrict__ mcell_cell, int64_t* __restrict__ mcell_grid,
                        int32_t* __restrict__ mcell_start, int32_t* __restrict__ mcell_n,
                        int32_t* __restrict__ mcell_adunit)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= G || cell_n[c] == 0) return;
    const int pid = cell_id_ofs[c];
    cell_grid[pid] = c;
    int run = cell_person_ofs[c];
    cell_start[pid] = run;
    int mid = cell_mc_ofs[c];
    for (int l = 0; l < nmcl; l++)
        for (int m = 0; m < nmcl; m++) {
            const long long j = mcell_of(c, l, m, nch, nmcl, th);
            const int v = cnt[j];
            if (v == 0) continue;
            mcell_cell[mid] = pid;
            mcell_grid[mid] = j;
            mcell_start[mid] = run;
            mcell_n[mid] = v;
            int au = 0;
            if (adunit_grid > 0) {
                const long long mx = j / th, my = j % th;
                const int ax = (int)min((mx * adunit_grid) / tw, (long long)adunit_grid - 1);
                const int ay = (int)min((my * adunit_grid) / th, (long long)adunit_grid - 1);
                au = ax * adunit_grid + ay;
            }
            mcell_adunit[mid] = au;
            run += v;
            mid++;
        }
}

// ---------------------------------------------------------------- households
// src/SetupModel.cpp:1224-1253: a size drawn from the cumulative distribution, cut
// at the microcell's remaining people and at the maximum size.
struct HhRule {
    double cdf[CS_MAX_HOUSEHOLD_SIZE];
};

__device__ __forceinline__ int hh_size(Stream& s, const HhRule& R, int k, int n)
{
    double u = s.next();
    int m = 1;
    while ((u > R.cdf[m - 1]) && (k + m < n) && (m < CS_MAX_HOUSEHOLD_SIZE)) m++;
    return m;
}

__global__ void k_hh_count(uint64_t seed, int NM, HhRule R, const int64_t* __restrict__ mcell_grid,
                           const int32_t* __restrict__ mcell_n, int32_t* __restrict__ hh_cnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NM) return;
    Stream s(seed, CS_RNG_SETUP_HH, 0, (uint32_t)mcell_grid[i], 0);
    const int n = mcell_n[i];
    int k = 0, c = 0;
    while (k < n) {
        k += hh_size(s, R, k, n);
        c++;
    }
    hh_cnt[i] = c;
}

__global__ void k_hh_fill(uint64_t seed, int NM, HhRule R, int th, double mcw, double mch,
                          const int64_t* __restrict__ mcell_grid, const int32_t* __restrict__ mcell_n,
                          const int32_t* __restrict__ mcell_start, const int32_t* __restrict__ hh_ofs,
                          int32_t* __restrict__ hh_first, uint16_t* __restrict__ hh_nh, float* __restrict__ hh_x,
                          float* __restrict__ hh_y, int32_t* __restrict__ person_hh, int32_t* __restrict__ person_mcell)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NM) return;
    const long long j = mcell_grid[i];
    Stream s(seed, CS_RNG_SETUP_HH, 0, (uint32_t)j, 0);
    const int n = mcell_n[i], first = mcell_start[i];
    const double x = (double)(j / th), y = (double)(j % th);
    int k = 0, h = hh_ofs[i];
    uint32_t ord = 0;
    while (k < n) {
        const int m = hh_size(s, R, k, n);
        Stream sl(seed, CS_RNG_SETUP_HH_LOC, 0, (uint32_t)j, ord++);
        const double ux = sl.next(), uy = sl.next();
        hh_first[h] = first + k;
        hh_nh[h] = (uint16_t)m;
        hh_x[h] = (float)(mcw * (ux + x));
        hh_y[h] = (float)(mch * (uy + y));
        for (int q = 0; q < m; q++) {
            person_hh[first + k + q] = h;
            person_mcell[first + k + q] = i;
        }
        k += m;
        h++;
    }
}

struct AgeRule {
    double cdf[CS_NUM_AGE_GROUPS];
};

__global__ void k_ages(uint64_t seed, int N, AgeRule R, uint8_t* __restrict__ age)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    Stream s(seed, CS_RNG_SETUP_AGE, 0, (uint32_t)p, 0);
    const double u = s.next();
    int b = 0;
    while (b < CS_NUM_AGE_GROUPS - 1 && !(u < R.cdf[b])) b++;
    int a = b * CS_AGE_GROUP_WIDTH + (int)floor(s.next() * CS_AGE_GROUP_WIDTH);
    age[p] = (uint8_t)min(a, 84);
}

// -------------------------------------------------------------------- places
struct Bands {
    double lo[3], hi[3], prop[3];
};

// Attendance of place type t: at most one place per person, types in order.
__global__ void k_attend(uint64_t seed, int N, int t, Bands B, const uint8_t* __restrict__ age,
                         uint8_t* __restrict__ taken, int32_t* __restrict__ att)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    int f = 0;
    if (!taken[p]) {
        const double a = (double)age[p];
        for (int b = 0; b < 3 && !f; b++) {
            if (!(B.prop[b] > 0) || a < B.lo[b] || !(a < B.hi[b])) continue;
            Stream s(seed, CS_RNG_SETUP_ATTEND, 0, (uint32_t)p, (uint32_t)(4 * t + b));
            if (s.next() < B.prop[b]) f = 1;
        }
        if (f) taken[p] = 1;
    }
    att[p] = f;
}

__global__ void k_att_list(int N, const int32_t* __restrict__ att, const int32_t* __restrict__ pos,
                           int32_t* __restrict__ list)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < N && att[p]) list[pos[p]] = p;
}

struct SizeRule {
    int kind;
    double mean, offset, power, max;
};

__device__ __forceinline__ int64_t place_size(uint64_t seed, int t, int i, const SizeRule& R, unsigned long long* err)
{
    Stream s(seed, CS_RNG_SETUP_PLACE_SIZE, 0, (uint32_t)i, (uint32_t)t);
    double v;
    if (R.kind == CS_SETUP_SIZE_POWER) {
        const double u = 1.0 - s.next();   // in (0, 1]
        v = floor((R.offset + 1.0) * pow(u, -1.0 / R.power) - R.offset);
        v = fmin(fmax(v, 1.0), R.max);
    } else {
        v = floor(sample_gamma(s, 4.0 / R.mean, 4.0, err) + 0.5);
        v = fmax(v, 1.0);
    }
    return (int64_t)v;
}

__global__ void k_place_sizes(uint64_t seed, int t, int n, SizeRule R, int64_t* __restrict__ sz,
                              unsigned long long* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sz[i] = place_size(seed, t, i, R, err);
}

// The places: sizes until they cover the attendees (the last cut to fit), one
// more if the draws fall short.  cum: inclusive prefix of the draws.
__global__ void k_place_cut(const int64_t* __restrict__ cum, int n_est, long long n_att, int32_t* __restrict__ n_places)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int lo = 0, hi = n_est;   // first index with cum >= n_att, n_est if none
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (cum[mid] >= n_att) hi = mid; else lo = mid + 1;
    }
    *n_places = (lo < n_est) ? lo + 1 : n_est + 1;
}

__global__ void k_place_init(uint64_t seed, int t, int npl, int n_est, long long n_att, double slack, int N,
                             int th, double mcw, double mch, const int64_t* __restrict__ sz,
                             const int64_t* __restrict__ cum, const int32_t* __restrict__ person_mcell,
                             const int64_t* __restrict__ mcell_grid, int32_t* __restrict__ place_mcell,
                             float* __restrict__ px, float* __restrict__ py, int32_t* __restrict__ rem)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npl) return;
    int64_t size;
    if (i < n_est) {
        size = sz[i];
        if (cum[i] > n_att) size -= cum[i] - n_att;
    } else {
        size = n_att - cum[n_est - 1];
    }
    rem[i] = (int32_t)ceil((double)size * slack);
    // located in the microcell of a person drawn uniformly: microcells in
    // proportion to their people
    const uint64_t r = __umul64hi(rand64(seed, CS_RNG_SETUP_PLACE_LOC, 0, (uint32_t)i, (uint32_t)t), (uint64_t)N);
    const int mid = person_mcell[r];
    const long long j = mcell_grid[mid];
    Stream s(seed, CS_RNG_SETUP_PLACE_LOC, 0, (uint32_t)i, (uint32_t)t);
    s.block = 1;   // block 0 gave the 64-bit draw
    const double ux = s.next(), uy = s.next();
    place_mcell[i] = mid;
    px[i] = (float)(mcw * ((double)(j / th) + ux));
    py[i] = (float)(mch * ((double)(j % th) + uy));
}

struct Buckets {
    int bs, nbx, nby;            // bucket side in cells, buckets per side
    double cw, ch;               // cell size
    int ncw, nch;
};

__device__ __forceinline__ int bucket_of(const Buckets& B, float x, float y)
{
    int cx = min(max((int)(x / B.cw), 0), B.ncw - 1);
    int cy = min(max((int)(y / B.ch), 0), B.nch - 1);
    return (cx / B.bs) * B.nby + (cy / B.bs);
}

__global__ void k_bucket_count(int npl, Buckets B, const float* __restrict__ px, const float* __restrict__ py,
                               int32_t* __restrict__ pb, int32_t* __restrict__ bcnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npl) return;
    int b = bucket_of(B, px[i], py[i]);
    pb[i] = b;
    atomicAdd(bcnt + b, 1);
}

__global__ void k_bucket_fill(int npl, const int32_t* __restrict__ pb, int32_t* __restrict__ cursor,
                              int32_t* __restrict__ items)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < npl) items[atomicAdd(cursor + pb[i], 1)] = i;   // order within a bucket is immaterial
}

struct Cand { double d2; int32_t pl; };

// (d2, place) ascending: the candidates' order does not depend on the visit order.
__device__ __forceinline__ bool cand_less(double d2, int pl, const Cand& c)
{
    return d2 < c.d2 || (d2 == c.d2 && pl < c.pl);
}

// One round of proposals: attendee a (person p) without a place gathers the nn
// nearest places with room (rings of buckets until nn are in hand, then one ring
// more) and proposes to one with probability proportional to K(d) * room (K alone
// in the capacity-free round).
__global__ void __launch_bounds__(128) k_propose(uint64_t seed, int t, int round, int free_round, int n_att, int nn,
                                                 Buckets B, const cs_params* __restrict__ Pp,
                                                 const double* __restrict__ lk, const double* __restrict__ hr,
                                                 const int32_t* __restrict__ list, const int32_t* __restrict__ person_hh,
                                                 const float* __restrict__ hh_x, const float* __restrict__ hh_y,
                                                 const float* __restrict__ px, const float* __restrict__ py,
                                                 const int32_t* __restrict__ bstart, const int32_t* __restrict__ items,
                                                 const int32_t* __restrict__ rem, const int32_t* __restrict__ link,
                                                 int32_t* __restrict__ prop)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_att) return;
    prop[a] = -1;
    if (link[a] >= 0) return;
    const cs_params& P = *Pp;
    const int p = list[a];
    const int h = person_hh[p];
    const float hx = hh_x[h], hy = hh_y[h];
    const int b0 = bucket_of(B, hx, hy);
    const int bx = b0 / B.nby, by = b0 % B.nby;
    Cand top[CS_SETUP_MAX_NEAREST];
    int ntop = 0, found = 0, extra = -1;
    const int rmax = max(B.nbx, B.nby);
    for (int r = 0; r < rmax && extra != 0; r++) {
        // the ring's buckets: the square's perimeter at Chebyshev distance r
        const int side = (r == 0) ? 1 : 8 * r;
        for (int q = 0; q < side; q++) {
            int x, y;
            if (r == 0) { x = bx; y = by; }
            else if (q < 2 * r + 1) { x = bx - r + q; y = by - r; }                    // bottom row
            else if (q < 4 * r + 2) { x = bx - r + (q - 2 * r - 1); y = by + r; }      // top row
            else if (q < 6 * r + 1) { x = bx - r; y = by - r + 1 + (q - 4 * r - 2); }  // left column
            else { x = bx + r; y = by - r + 1 + (q - 6 * r - 1); }                      // right column
            if (x < 0 || y < 0 || x >= B.nbx || y >= B.nby) continue;
            const int bk = x * B.nby + y;
            for (int e = bstart[bk]; e < bstart[bk + 1]; e++) {
                const int pl = items[e];
                if (!free_round && rem[pl] <= 0) continue;
                found++;
                const double d2 = dist2_pts(P, hx, hy, px[pl], py[pl]);
                if (ntop == nn && !cand_less(d2, pl, top[nn - 1])) continue;
                int k = (ntop < nn) ? ntop++ : nn - 1;
                while (k > 0 && cand_less(d2, pl, top[k - 1])) { top[k] = top[k - 1]; k--; }
                top[k].d2 = d2;
                top[k].pl = pl;
            }
        }
        if (extra > 0) extra--;
        else if (extra < 0 && found >= nn) extra = 1;
    }
    if (ntop == 0) return;
    double w[CS_SETUP_MAX_NEAREST];
    double tot = 0.0;
    for (int k = 0; k < ntop; k++) {
        w[k] = knum_tab(lk, hr, P, top[k].d2) * (free_round ? 1.0 : (double)rem[top[k].pl]);
        tot = tot + w[k];
    }
    int k = 0;
    if (tot > 0) {
        Stream s(seed, CS_RNG_SETUP_CHOOSE, (uint32_t)round, (uint32_t)p, (uint32_t)t);
        double u = s.next() * tot;
        while (k + 1 < ntop && u >= w[k]) { u -= w[k]; k++; }
    } else if (!free_round) {
        return;   // every place in reach is beyond the kernel: wait for the last round
    }
    prop[a] = top[k].pl;
}

__global__ void k_count_props(int n_att, const int32_t* __restrict__ prop, int32_t* __restrict__ nprop)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < n_att && prop[a] >= 0) atomicAdd(nprop + prop[a], 1);
}

__global__ void k_accept(uint64_t seed, int t, int round, int free_round, int n_att, const int32_t* __restrict__ list,
                         const int32_t* __restrict__ prop, const int32_t* __restrict__ nprop,
                         const int32_t* __restrict__ rem, int32_t* __restrict__ link, int32_t* __restrict__ taken,
                         int32_t* __restrict__ forced)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_att) return;
    const int pl = prop[a];
    if (pl < 0) return;
    bool ok = true;
    if (!free_round) {
        const int n = nprop[pl], r = rem[pl];
        if (n > r) {
            Stream s(seed, CS_RNG_SETUP_ACCEPT, (uint32_t)round, (uint32_t)list[a], (uint32_t)t);
            ok = s.next() * (double)n < (double)r;
        }
    }
    if (!ok) return;
    link[a] = pl;
    atomicAdd(taken + pl, 1);
    if (free_round) atomicAdd(forced, 1);
}

__global__ void k_take(int npl, int32_t* __restrict__ rem, int32_t* __restrict__ taken, int32_t* __restrict__ nprop)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npl) return;
    rem[i] = max(rem[i] - taken[i], 0);
    taken[i] = 0;
    nprop[i] = 0;
}

// Member lists: attendees sorted by (place, random key); person_place too.
__global__ void k_member_keys(uint64_t seed, int t, int n_att, const int32_t* __restrict__ list,
                              const int32_t* __restrict__ link, uint64_t* __restrict__ keys,
                              int32_t* __restrict__ vals, int32_t* __restrict__ mcount,
                              int32_t* __restrict__ person_place, unsigned long long* err)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_att) return;
    const int p = list[a], pl = link[a];
    if (pl < 0) {   // the last round reaches every place, so this does not happen; counted if it does
        atomicAdd(err, 1ull);
        return;
    }
    const uint32_t h = (uint32_t)rand64(seed, CS_RNG_SETUP_SHUFFLE, 0, (uint32_t)p, (uint32_t)t);
    keys[a] = ((uint64_t)(uint32_t)pl << 32) | h;
    vals[a] = p;
    atomicAdd(mcount + pl, 1);
    person_place[p] = pl;
}

__global__ void k_group_counts(int npl, int g1, const int32_t* __restrict__ mcount, int32_t* __restrict__ ng)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < npl) ng[i] = max(1, (int)floor((double)mcount[i] / (double)g1 + 0.5));
}

// Group k of a place of n members covers members [k n / ng, (k+1) n / ng).
__global__ void k_groups(int npl, const int32_t* __restrict__ mcount, const int32_t* __restrict__ mofs,
                         const int32_t* __restrict__ ng, const int32_t* __restrict__ gofs,
                         const int32_t* __restrict__ members, int32_t* __restrict__ gstart,
                         int32_t* __restrict__ gsize, uint16_t* __restrict__ person_group)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npl) return;
    const long long n = mcount[i], g = ng[i];
    for (long long k = 0; k < g; k++) {
        const long long s = (k * n) / g, e = ((k + 1) * n) / g;
        gstart[gofs[i] + k] = (int32_t)s;
        gsize[gofs[i] + k] = (int32_t)(e - s);
        for (long long q = s; q < e; q++) person_group[members[mofs[i] + q]] = (uint16_t)k;
    }
}

__global__ void k_fill_i32(int32_t* p, long long n, int32_t v)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

inline unsigned nblk(long long n, int t = kT) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ================================================================ host side
struct PlaceOut {
    int32_t n_places = 0, n_groups = 0, n_att = 0, forced = 0;
    int32_t *mcell = nullptr, *member_ofs = nullptr, *members = nullptr, *group_ofs = nullptr, *gstart = nullptr,
            *gsize = nullptr;
    float *x = nullptr, *y = nullptr;
};

struct cs_setup {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::vector<void*> allocs;
    int32_t N = 0, NH = 0, NC = 0, NM = 0, n_adunits = 1, npt = 0;
    double device_ms = 0;
    int32_t *person_hh = nullptr, *person_mcell = nullptr, *person_place = nullptr, *hh_first = nullptr,
            *mcell_cell = nullptr, *mcell_adunit = nullptr, *cell_grid = nullptr, *cell_start = nullptr;
    int64_t* mcell_grid = nullptr;
    uint8_t* person_age = nullptr;
    uint16_t *person_group = nullptr, *hh_nh = nullptr;
    float *hh_x = nullptr, *hh_y = nullptr;
    PlaceOut pl[CS_MAX_PLACE_TYPES];
};

namespace {

int fail(cs_setup* s, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    s->err = buf;
    return code;
}

#define SK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(s, CS_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define SLAUNCH(kern, grid, block, ...)                                                          \
    do {                                                                                         \
        if ((grid) > 0) kern<<<(grid), (block), 0, s->stream>>>(__VA_ARGS__);                    \
        cudaError_t e_ = cudaGetLastError();                                                     \
        if (e_ != cudaSuccess) return fail(s, CS_E_CUDA, "%s: %s", #kern, cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int dalloc(cs_setup* s, T** p, long long n)
{
    void* q = nullptr;
    SK(cudaMalloc(&q, (size_t)std::max(n, 1LL) * sizeof(T)));
    s->allocs.push_back(q);
    *p = (T*)q;
    return CS_OK;
}

#define SALLOC(p, n)                       \
    do {                                   \
        int r_ = dalloc(s, &(p), (n));     \
        if (r_) return r_;                 \
    } while (0)

// out[i] = exclusive (or inclusive) prefix of in; *total (device, may be null) the sum.
template <typename Tin, typename T>
int scan(cs_setup* s, const Tin* in, long long n, T* out, bool inclusive, T* total_dev)
{
    if (n <= 0) return CS_OK;
    const long long nb = (n + kTile - 1) / kTile;
    T* bsum;
    SALLOC(bsum, nb);
    k_scan_reduce<Tin, T><<<(unsigned)nb, kT, 0, s->stream>>>(in, n, bsum);
    SK(cudaGetLastError());
    k_scan_totals<T><<<1, 1024, 0, s->stream>>>(bsum, nb, total_dev);
    SK(cudaGetLastError());
    k_scan_apply<Tin, T><<<(unsigned)nb, kT, 0, s->stream>>>(in, n, bsum, out, inclusive ? 1 : 0);
    SK(cudaGetLastError());
    return CS_OK;
}
#define SSCAN(in, n, out, inc, tot)                      \
    do {                                                 \
        int r_ = scan(s, (in), (n), (out), (inc), (tot)); \
        if (r_) return r_;                               \
    } while (0)

template <typename T>
int read1(cs_setup* s, const T* dev, T* host)
{
    SK(cudaMemcpyAsync(host, dev, sizeof(T), cudaMemcpyDeviceToHost, s->stream));
    SK(cudaStreamSynchronize(s->stream));
    return CS_OK;
}
#define SREAD(dev, host)              \
    do {                              \
        int r_ = read1(s, (dev), (host)); \
        if (r_) return r_;            \
    } while (0)

// Stable sort of (key, value) pairs by the low `bits` bits of the key.
int radix_sort(cs_setup* s, uint64_t* keys, int32_t* vals, long long n, int bits)
{
    if (n <= 1) return CS_OK;
    const long long nb = (n + kTile - 1) / kTile;
    uint64_t* k2;
    int32_t* v2;
    uint32_t *hist, *ofs;
    SALLOC(k2, n);
    SALLOC(v2, n);
    SALLOC(hist, 256 * nb);
    SALLOC(ofs, 256 * nb);
    uint64_t* ka = keys;
    int32_t* va = vals;
    uint64_t* kb = k2;
    int32_t* vb = v2;
    int passes = (bits + 7) / 8;
    for (int ps = 0; ps < passes; ps++) {
        SLAUNCH(k_radix_hist, (unsigned)nb, kT, ka, n, 8 * ps, hist, nb);
        SSCAN(hist, 256 * nb, ofs, false, (uint32_t*)nullptr);
        SLAUNCH(k_radix_scatter, (unsigned)nb, kT, ka, va, n, 8 * ps, ofs, nb, kb, vb);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    if (ka != keys) {
        SK(cudaMemcpyAsync(keys, ka, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s->stream));
        SK(cudaMemcpyAsync(vals, va, n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s->stream));
    }
    return CS_OK;
}

int check_spec(cs_setup* s, const cs_setup_spec& S, const cs_params& P)
{
    if (S.n_people <= 0 || S.ncw <= 0 || S.nch <= 0 || S.nmcl <= 0)
        return fail(s, CS_E_ARG, "setup: n_people, ncw, nch and nmcl must be positive");
    if ((long long)S.ncw * S.nmcl * S.nch * S.nmcl > 0x7fffffffLL)
        return fail(s, CS_E_ARG, "setup: %d x %d cells of %d x %d microcells exceed 2^31 microcells", S.ncw, S.nch,
                    S.nmcl, S.nmcl);
    if (S.n_blobs < 0 || S.n_blobs > CS_SETUP_MAX_BLOBS)
        return fail(s, CS_E_ARG, "setup: n_blobs %d outside [0, %d]", S.n_blobs, CS_SETUP_MAX_BLOBS);
    if (S.n_blobs > 0 && !(S.blob_share > 0 && S.blob_share <= 1))
        return fail(s, CS_E_ARG, "setup: blob_share must be in (0, 1] with blobs");
    if (S.num_place_types < 0 || S.num_place_types > CS_MAX_PLACE_TYPES)
        return fail(s, CS_E_ARG, "setup: num_place_types %d outside [0, %d]", S.num_place_types, CS_MAX_PLACE_TYPES);
    if (S.adunit_grid < 0 || S.adunit_grid * S.adunit_grid > CS_MAX_ADUNITS)
        return fail(s, CS_E_ARG, "setup: adunit_grid %d gives more than %d admin units", S.adunit_grid, CS_MAX_ADUNITS);
    if (S.rounds < 0 || S.rounds > 64) return fail(s, CS_E_ARG, "setup: rounds %d outside [0, 64]", S.rounds);
    if (!(P.cell_width > 0) || P.ncw != S.ncw || P.nch != S.nch)
        return fail(s, CS_E_ARG, "setup: params describe another grid (%d x %d)", P.ncw, P.nch);
    for (int t = 0; t < S.num_place_types; t++) {
        const cs_setup_place_type& T = S.pt[t];
        if (T.nearest < 1 || T.nearest > CS_SETUP_MAX_NEAREST)
            return fail(s, CS_E_ARG, "setup: place type %d: nearest %d outside [1, %d]", t, T.nearest,
                        CS_SETUP_MAX_NEAREST);
        if (!(T.mean_size >= 1) || T.group_size < 1 || !(T.capacity_slack >= 1))
            return fail(s, CS_E_ARG, "setup: place type %d: mean_size >= 1, group_size >= 1, slack >= 1 needed", t);
        if (T.size_kind == CS_SETUP_SIZE_POWER && !(T.size_power > 0 && T.size_max >= 1))
            return fail(s, CS_E_ARG, "setup: place type %d: power-law sizes need power > 0, max >= 1", t);
        if (!T.kernel_lookup || !T.kernel_hi_res) return fail(s, CS_E_ARG, "setup: place type %d: no kernel table", t);
    }
    return CS_OK;
}

int run_setup(cs_setup* s, const cs_setup_spec& S, const cs_params& P)
{
    int r = check_spec(s, S, P);
    if (r) return r;
    SK(cudaSetDevice(s->device));
    SK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    SK(cudaEventCreate(&e0));
    SK(cudaEventCreate(&e1));
    SK(cudaEventRecord(e0, s->stream));
    const uint64_t seed = S.seed;
    const int nmcl = S.nmcl, nch = S.nch, ncw = S.ncw;
    const int th = nch * nmcl, tw = ncw * nmcl;
    const long long M = (long long)tw * th;
    const int G = ncw * nch;
    const int N = S.n_people;
    const double mcw = S.cell_width / nmcl, mch = S.cell_height / nmcl;
    s->N = N;
    s->npt = S.num_place_types;
    s->n_adunits = S.adunit_grid > 0 ? S.adunit_grid * S.adunit_grid : 1;

    cs_params* Pd;
    SALLOC(Pd, 1);
    SK(cudaMemcpyAsync(Pd, &P, sizeof(cs_params), cudaMemcpyHostToDevice, s->stream));
    unsigned long long* err;
    SALLOC(err, 1);
    SK(cudaMemsetAsync(err, 0, sizeof(unsigned long long), s->stream));

    // 1. microcell weights and their integer prefix sums
    uint64_t *q, *qb = nullptr, *pref, *QW, *QB;
    SALLOC(q, M);
    SALLOC(pref, M);
    SALLOC(QW, 1);
    SALLOC(QB, 1);
    Blob* blobs = nullptr;
    if (S.n_blobs > 0) {
        SALLOC(qb, M);
        SALLOC(blobs, S.n_blobs);
        SLAUNCH(k_blobs, 1u, 64, seed, S.n_blobs, blobs, err);
    }
    SLAUNCH(k_density, nblk(M), kT, seed, S.sigma, M, tw, th, blobs, S.n_blobs, q, qb, err);
    if (S.n_blobs > 0) {
        SSCAN(q, M, pref, true, QW);
        SSCAN(qb, M, pref, true, QB);
        SLAUNCH(k_blend, nblk(M), kT, M, S.blob_share, QW, QB, q, qb);
    }
    SSCAN(q, M, pref, true, QW);
    uint64_t qtot = 0;
    SREAD(QW, &qtot);
    if (qtot == 0) return fail(s, CS_E_ARG, "setup: every microcell weight is zero");

    // 2. people to microcells
    int32_t* cnt;
    SALLOC(cnt, M);
    SK(cudaMemsetAsync(cnt, 0, M * sizeof(int32_t), s->stream));
    SLAUNCH(k_people_to_mcells, nblk(N), kT, seed, N, pref, M, cnt);

    // 3. populated cells and microcells in the reference's order
    int32_t *cell_n, *cell_pm, *cell_pop, *cell_person_ofs, *cell_mc_ofs, *cell_id_ofs, *tot32;
    SALLOC(cell_n, G);
    SALLOC(cell_pm, G);
    SALLOC(cell_pop, G);
    SALLOC(cell_person_ofs, G);
    SALLOC(cell_mc_ofs, G);
    SALLOC(cell_id_ofs, G);
    SALLOC(tot32, 4);
    SLAUNCH(k_cell_sums, nblk(G), kT, G, nch, nmcl, th, cnt, cell_n, cell_pm, cell_pop);
    SSCAN(cell_n, G, cell_person_ofs, false, (int32_t*)nullptr);
    SSCAN(cell_pm, G, cell_mc_ofs, false, tot32 + 0);
    SSCAN(cell_pop, G, cell_id_ofs, false, tot32 + 1);
    int32_t NM = 0, NC = 0;
    SREAD(tot32 + 0, &NM);
    SREAD(tot32 + 1, &NC);
    s->NM = NM;
    s->NC = NC;
    int32_t *mcell_start, *mcell_n;
    SALLOC(s->cell_grid, NC);
    SALLOC(s->cell_start, NC + 1);
    SALLOC(s->mcell_cell, NM);
    SALLOC(s->mcell_grid, NM);
    SALLOC(mcell_start, NM);
    SALLOC(mcell_n, NM);
    SALLOC(s->mcell_adunit, NM);
    SLAUNCH(k_cells, nblk(G), kT, G, nch, nmcl, th, tw, S.adunit_grid, cnt, cell_n, cell_person_ofs, cell_mc_ofs,
            cell_id_ofs, s->cell_grid, s->cell_start, s->mcell_cell, s->mcell_grid, mcell_start, mcell_n,
            s->mcell_adunit);
    SK(cudaMemcpyAsync(s->cell_start + NC, &s->N, sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));

    // 4. households
    HhRule hr;
    for (int k = 0; k < CS_MAX_HOUSEHOLD_SIZE; k++) hr.cdf[k] = S.hh_cdf[k];
    int32_t *hh_cnt, *hh_ofs;
    SALLOC(hh_cnt, NM);
    SALLOC(hh_ofs, NM);
    SLAUNCH(k_hh_count, nblk(NM), kT, seed, NM, hr, s->mcell_grid, mcell_n, hh_cnt);
    SSCAN(hh_cnt, NM, hh_ofs, false, tot32 + 2);
    int32_t NH = 0;
    SREAD(tot32 + 2, &NH);
    s->NH = NH;
    SALLOC(s->hh_first, NH);
    SALLOC(s->hh_nh, NH);
    SALLOC(s->hh_x, NH);
    SALLOC(s->hh_y, NH);
    SALLOC(s->person_hh, N);
    SALLOC(s->person_mcell, N);
    SLAUNCH(k_hh_fill, nblk(NM), kT, seed, NM, hr, th, mcw, mch, s->mcell_grid, mcell_n, mcell_start, hh_ofs,
            s->hh_first, s->hh_nh, s->hh_x, s->hh_y, s->person_hh, s->person_mcell);

    // 5. ages
    AgeRule ar;
    for (int k = 0; k < CS_NUM_AGE_GROUPS; k++) ar.cdf[k] = S.age_cdf[k];
    SALLOC(s->person_age, N);
    SLAUNCH(k_ages, nblk(N), kT, seed, N, ar, s->person_age);

    // 6. places.  The spec's kernel tables are host arrays: each distinct one is
    // copied to the device once.
    const int npt = S.num_place_types;
    const size_t ktab = (size_t)P.kernel_size + 1;
    const double* klk[CS_MAX_PLACE_TYPES] = {};
    const double* khr[CS_MAX_PLACE_TYPES] = {};
    for (int t = 0; t < npt; t++) {
        for (int u = 0; u < t && !klk[t]; u++)
            if (S.pt[u].kernel_lookup == S.pt[t].kernel_lookup && S.pt[u].kernel_hi_res == S.pt[t].kernel_hi_res) {
                klk[t] = klk[u];
                khr[t] = khr[u];
            }
        if (klk[t]) continue;
        double *a, *b;
        SALLOC(a, ktab);
        SALLOC(b, ktab);
        SK(cudaMemcpyAsync(a, S.pt[t].kernel_lookup, sizeof(double) * ktab, cudaMemcpyHostToDevice, s->stream));
        SK(cudaMemcpyAsync(b, S.pt[t].kernel_hi_res, sizeof(double) * ktab, cudaMemcpyHostToDevice, s->stream));
        klk[t] = a;
        khr[t] = b;
    }
    SALLOC(s->person_place, (long long)std::max(npt, 1) * N);
    SALLOC(s->person_group, (long long)std::max(npt, 1) * N);
    SLAUNCH(k_fill_i32, nblk((long long)npt * N), kT, s->person_place, (long long)npt * N, -1);
    SK(cudaMemsetAsync(s->person_group, 0, sizeof(uint16_t) * (size_t)std::max(npt, 1) * N, s->stream));
    uint8_t* taken_p;
    int32_t *att, *att_pos, *list;
    SALLOC(taken_p, N);
    SALLOC(att, N);
    SALLOC(att_pos, N);
    SALLOC(list, N);
    SK(cudaMemsetAsync(taken_p, 0, N, s->stream));
    for (int t = 0; t < npt; t++) {
        const cs_setup_place_type& T = S.pt[t];
        PlaceOut& O = s->pl[t];
        Bands bd;
        for (int b = 0; b < 3; b++) { bd.lo[b] = T.band_lo[b]; bd.hi[b] = T.band_hi[b]; bd.prop[b] = T.band_prop[b]; }
        SLAUNCH(k_attend, nblk(N), kT, seed, N, t, bd, s->person_age, taken_p, att);
        SSCAN(att, N, att_pos, false, tot32 + 3);
        int32_t n_att = 0;
        SREAD(tot32 + 3, &n_att);
        O.n_att = n_att;
        SLAUNCH(k_att_list, nblk(N), kT, N, att, att_pos, list);
        if (n_att == 0) {
            O.n_places = 0;
            SALLOC(O.member_ofs, 1);
            SALLOC(O.group_ofs, 1);
            SK(cudaMemsetAsync(O.member_ofs, 0, sizeof(int32_t), s->stream));
            SK(cudaMemsetAsync(O.group_ofs, 0, sizeof(int32_t), s->stream));
            continue;
        }
        // sizes
        const int n_est = std::max(1, (int)((double)n_att / T.mean_size * 1.2) + 8);
        SizeRule sr{T.size_kind, T.mean_size, T.size_offset, T.size_power, T.size_max};
        int64_t *sz, *cum;
        SALLOC(sz, n_est);
        SALLOC(cum, n_est);
        SLAUNCH(k_place_sizes, nblk(n_est), kT, seed, t, n_est, sr, sz, err);
        SSCAN(sz, n_est, cum, true, (int64_t*)nullptr);
        int32_t* npl_d;
        SALLOC(npl_d, 1);
        SLAUNCH(k_place_cut, 1u, 1, cum, n_est, (long long)n_att, npl_d);
        int32_t npl = 0;
        SREAD(npl_d, &npl);
        O.n_places = npl;
        int32_t* rem;
        SALLOC(O.mcell, npl);
        SALLOC(O.x, npl);
        SALLOC(O.y, npl);
        SALLOC(rem, npl);
        SLAUNCH(k_place_init, nblk(npl), kT, seed, t, npl, n_est, (long long)n_att, T.capacity_slack, N, th, mcw, mch,
                sz, cum, s->person_mcell, s->mcell_grid, O.mcell, O.x, O.y, rem);
        // buckets of about four places
        Buckets B;
        B.ncw = ncw;
        B.nch = nch;
        B.cw = S.cell_width;
        B.ch = S.cell_height;
        B.bs = std::max(1, (int)floor(sqrt(4.0 * (double)G / (double)npl)));
        B.nbx = (ncw + B.bs - 1) / B.bs;
        B.nby = (nch + B.bs - 1) / B.bs;
        const int NBK = B.nbx * B.nby;
        int32_t *pb, *bcnt, *bstart, *cursor, *items;
        SALLOC(pb, npl);
        SALLOC(bcnt, NBK + 1);
        SALLOC(bstart, NBK + 1);
        SALLOC(cursor, NBK + 1);
        SALLOC(items, npl);
        SK(cudaMemsetAsync(bcnt, 0, sizeof(int32_t) * (NBK + 1), s->stream));
        SLAUNCH(k_bucket_count, nblk(npl), kT, npl, B, O.x, O.y, pb, bcnt);
        SSCAN(bcnt, NBK + 1, bstart, false, (int32_t*)nullptr);
        SK(cudaMemcpyAsync(cursor, bstart, sizeof(int32_t) * (NBK + 1), cudaMemcpyDeviceToDevice, s->stream));
        SLAUNCH(k_bucket_fill, nblk(npl), kT, npl, pb, cursor, items);
        // rounds of proposals
        int32_t *link, *prop, *nprop, *taken, *forced;
        SALLOC(link, n_att);
        SALLOC(prop, n_att);
        SALLOC(nprop, npl);
        SALLOC(taken, npl);
        SALLOC(forced, 1);
        SLAUNCH(k_fill_i32, nblk(n_att), kT, link, (long long)n_att, -1);
        SK(cudaMemsetAsync(nprop, 0, sizeof(int32_t) * npl, s->stream));
        SK(cudaMemsetAsync(taken, 0, sizeof(int32_t) * npl, s->stream));
        SK(cudaMemsetAsync(forced, 0, sizeof(int32_t), s->stream));
        for (int rd = 0; rd <= S.rounds; rd++) {
            const int free_round = rd == S.rounds;
            SLAUNCH(k_propose, nblk(n_att, 128), 128, seed, t, rd, free_round, n_att, T.nearest, B, Pd, klk[t],
                    khr[t], list, s->person_hh, s->hh_x, s->hh_y, O.x, O.y, bstart, items, rem, link, prop);
            SLAUNCH(k_count_props, nblk(n_att), kT, n_att, prop, nprop);
            SLAUNCH(k_accept, nblk(n_att), kT, seed, t, rd, free_round, n_att, list, prop, nprop, rem, link, taken,
                    forced);
            SLAUNCH(k_take, nblk(npl), kT, npl, rem, taken, nprop);
        }
        SREAD(forced, &O.forced);
        // members: by (place, random key)
        uint64_t* keys;
        int32_t *vals, *mcount, *ng;
        SALLOC(keys, n_att);
        SALLOC(vals, n_att);
        SALLOC(mcount, npl);
        SALLOC(ng, npl);
        SALLOC(O.member_ofs, npl + 1);
        SALLOC(O.group_ofs, npl + 1);
        SK(cudaMemsetAsync(mcount, 0, sizeof(int32_t) * npl, s->stream));
        SLAUNCH(k_member_keys, nblk(n_att), kT, seed, t, n_att, list, link, keys, vals, mcount,
                s->person_place + (long long)t * N, err);
        int bits = 32;
        while (bits < 64 && ((uint64_t)npl >> (bits - 32)) != 0) bits++;
        r = radix_sort(s, keys, vals, n_att, bits);
        if (r) return r;
        O.members = vals;
        // offsets and groups (the extra last entry of each scan input is zero)
        int32_t *mc1, *ng1;
        SALLOC(mc1, npl + 1);
        SALLOC(ng1, npl + 1);
        SK(cudaMemsetAsync(mc1 + npl, 0, sizeof(int32_t), s->stream));
        SK(cudaMemsetAsync(ng1 + npl, 0, sizeof(int32_t), s->stream));
        SK(cudaMemcpyAsync(mc1, mcount, sizeof(int32_t) * npl, cudaMemcpyDeviceToDevice, s->stream));
        SLAUNCH(k_group_counts, nblk(npl), kT, npl, T.group_size, mcount, ng);
        SK(cudaMemcpyAsync(ng1, ng, sizeof(int32_t) * npl, cudaMemcpyDeviceToDevice, s->stream));
        SSCAN(mc1, npl + 1, O.member_ofs, false, (int32_t*)nullptr);
        SSCAN(ng1, npl + 1, O.group_ofs, false, tot32 + 3);
        SREAD(tot32 + 3, &O.n_groups);
        SALLOC(O.gstart, O.n_groups);
        SALLOC(O.gsize, O.n_groups);
        SLAUNCH(k_groups, nblk(npl), kT, npl, mcount, O.member_ofs, ng, O.group_ofs, O.members, O.gstart, O.gsize,
                s->person_group + (long long)t * N);
    }
    SK(cudaEventRecord(e1, s->stream));
    SK(cudaStreamSynchronize(s->stream));
    float ms = 0;
    SK(cudaEventElapsedTime(&ms, e0, e1));
    s->device_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    unsigned long long nerr = 0;
    SK(cudaMemcpy(&nerr, err, sizeof nerr, cudaMemcpyDeviceToHost));
    if (nerr) return fail(s, CS_E_OVERFLOW, "setup: %llu bounded sampling loops gave up", nerr);
    return CS_OK;
}

}  // namespace

extern "C" size_t cs_sizeof_setup_spec(void) { return sizeof(cs_setup_spec); }
extern "C" size_t cs_sizeof_setup_out(void) { return sizeof(cs_setup_out); }

extern "C" int cs_gpu_setup_run(const cs_setup_spec* spec, const cs_params* params, int device, cs_setup** out)
{
    if (!out) return CS_E_ARG;
    *out = nullptr;
    if (!spec || !params) return CS_E_ARG;
    cs_setup* s = new cs_setup();
    s->device = device;
    *out = s;
    return run_setup(s, *spec, *params);
}

extern "C" int cs_gpu_setup_sizes(cs_setup* s, cs_setup_out* o)
{
    if (!s || !o) return CS_E_ARG;
    o->n_people = s->N;
    o->n_households = s->NH;
    o->n_cells = s->NC;
    o->n_mcells = s->NM;
    o->n_adunits = s->n_adunits;
    o->num_place_types = s->npt;
    for (int t = 0; t < CS_MAX_PLACE_TYPES; t++) {
        o->n_places[t] = s->pl[t].n_places;
        o->n_groups[t] = s->pl[t].n_groups;
        o->n_attendees[t] = s->pl[t].n_att;
        o->forced[t] = s->pl[t].forced;
    }
    o->device_ms = s->device_ms;
    return CS_OK;
}

extern "C" int cs_gpu_setup_download(cs_setup* s, const cs_setup_out* o)
{
    if (!s || !o) return CS_E_ARG;
    SK(cudaSetDevice(s->device));
    auto get = [&](void* dst, const void* src, size_t bytes) -> int {
        if (!dst || !src || bytes == 0) return CS_OK;
        SK(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
        return CS_OK;
    };
    const size_t N = (size_t)s->N, NH = (size_t)s->NH, NM = (size_t)s->NM, NC = (size_t)s->NC;
    int r = 0;
    r |= get(o->person_hh, s->person_hh, 4 * N);
    r |= get(o->person_mcell, s->person_mcell, 4 * N);
    r |= get(o->person_age, s->person_age, N);
    r |= get(o->person_place, s->person_place, 4 * N * s->npt);
    r |= get(o->person_group, s->person_group, 2 * N * s->npt);
    r |= get(o->hh_first, s->hh_first, 4 * NH);
    r |= get(o->hh_nh, s->hh_nh, 2 * NH);
    r |= get(o->hh_x, s->hh_x, 4 * NH);
    r |= get(o->hh_y, s->hh_y, 4 * NH);
    r |= get(o->mcell_cell, s->mcell_cell, 4 * NM);
    r |= get(o->mcell_adunit, s->mcell_adunit, 4 * NM);
    r |= get(o->mcell_grid, s->mcell_grid, 8 * NM);
    r |= get(o->cell_grid, s->cell_grid, 4 * NC);
    r |= get(o->cell_start, s->cell_start, 4 * (NC + 1));
    for (int t = 0; t < s->npt; t++) {
        const PlaceOut& O = s->pl[t];
        const size_t np = (size_t)O.n_places, na = (size_t)O.n_att, ng = (size_t)O.n_groups;
        r |= get(o->place_mcell[t], O.mcell, 4 * np);
        r |= get(o->place_x[t], O.x, 4 * np);
        r |= get(o->place_y[t], O.y, 4 * np);
        r |= get(o->place_member_ofs[t], O.member_ofs, 4 * (np + 1));
        r |= get(o->place_members[t], O.members, 4 * na);
        r |= get(o->place_group_ofs[t], O.group_ofs, 4 * (np + 1));
        r |= get(o->group_start[t], O.gstart, 4 * ng);
        r |= get(o->group_size[t], O.gsize, 4 * ng);
    }
    return r ? CS_E_CUDA : CS_OK;
}

extern "C" const char* cs_gpu_setup_last_error(const cs_setup* s)
{
    return s ? s->err.c_str() : "null set-up handle";
}

extern "C" void cs_gpu_setup_destroy(cs_setup* s)
{
    if (!s) return;
    cudaSetDevice(s->device);
    for (void* p : s->allocs) cudaFree(p);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}
