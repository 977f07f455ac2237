// B200 (sm_100a) implementation of CovidSim's per-timestep sweep behind the C ABI
// of include/covidsim_b200.h.
//
// One timestep = InfectSweep + IncubRecoverySweep (src/Sweep.cpp:283-979).  The
// reference walks cells on CPU threads and pushes infections through per-thread
// queues; here each phase is a handful of grid-stride kernels over compact lists
// built on the device, with no host round trip inside a step (so a step can be
// replayed as a CUDA graph):
//
//   InfectSweep
//     k_build_active         infectious people of every cell, one list
//     k_infector_hh_spatial  household pass and spatial Poisson count per infector;
//                            reserves each infector's entries of the contact map
//     k_infector_places      place passes, one thread per (infector, place type)
//     k_spatial              spatial contacts: block proposal + rejection, eight
//                            draws of a contact evaluated together
//     k_apply_infections     DoInfect for every claimed person (lowest key wins)
//     k_partition_S          S -> L cell-list moves, one warp per touched cell
//   IncubRecoverySweep
//     k_incub_gather         the latent and infectious people with an event this step,
//                            read from the cells' lists
//     k_incub_events         DoIncub / DoCase / severity / recovery / death per person
//     k_incub_finish         L -> I and I -> R/D cell-list moves per touched cell, then
//                            the deferred adult-carer absence and household quarantine
//
// Determinism: all random numbers come from Philox streams keyed by
// (seed, step, entity, purpose); conflicting infections resolve by atomicMin on a
// 64-bit key; counters are integer atomics; every floating-point reduction runs
// in a fixed order.  Results therefore do not depend on launch geometry.
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "covidsim_b200.h"
#include "cs_device.cuh"
#include "cs_state.h"

namespace cg = cooperative_groups;
using namespace csb;

// ------------------------------------------------------------------ helpers
#define CSB_CTR(field) ((unsigned long long*)&d.C->field)

// Per-block staging of the counters in shared memory, for kernels whose threads
// hit the same few counters (severity tallies, per-age and per-admin-unit sums):
// with many items, adds go to shared memory and each block adds its non-zero
// totals to the global counters once, at its end; with few items the zeroing and
// flushing would cost more than they save, so adds go straight to the global
// counters.  CSB_STAGED is valid between stage_begin() and stage_flush() only.
constexpr int kCtrWords = (int)(sizeof(cs_counters) / sizeof(unsigned long long));
static_assert(sizeof(cs_counters) % sizeof(unsigned long long) == 0, "counters are 64-bit words");
constexpr int kStageMinItems = 16384;
__shared__ unsigned long long s_ctr[kCtrWords];
__shared__ unsigned long long* s_ctr_base;
#define CSB_STAGED(field) ((unsigned long long*)((char*)s_ctr_base + offsetof(cs_counters, field)))

__device__ __forceinline__ void stage_begin(cs_counters* C, bool staged)
{
    if (staged)
        for (int i = threadIdx.x; i < kCtrWords; i += blockDim.x) s_ctr[i] = 0ull;
    if (threadIdx.x == 0) s_ctr_base = staged ? s_ctr : reinterpret_cast<unsigned long long*>(C);
    __syncthreads();
}
__device__ __forceinline__ void stage_flush(cs_counters* C, bool staged)
{
    if (!staged) return;
    __syncthreads();
    unsigned long long* g = reinterpret_cast<unsigned long long*>(C);
    for (int i = threadIdx.x; i < kCtrWords; i += blockDim.x)
        if (s_ctr[i]) atomicAdd(g + i, s_ctr[i]);
}

__device__ __forceinline__ void cnt_add(unsigned long long* p, long long v) { atomicAdd(p, (unsigned long long)v); }

// Adds every calling thread's v with one atomic per warp, skipping zero sums: the
// end-of-kernel work tallies would otherwise put one atomic per thread on a
// single address.
__device__ __forceinline__ void cnt_add_warp(unsigned long long* p, long long v)
{
    cg::coalesced_group g = cg::coalesced_threads();
    long long sum = cg::reduce(g, v, cg::plus<long long>());
    if (g.thread_rank() == 0 && sum != 0) atomicAdd(p, (unsigned long long)sum);
}

// Warp-aggregated append to a device list.
__device__ __forceinline__ int32_t append(int32_t* count)
{
    cg::coalesced_group g = cg::coalesced_threads();
    int32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(count, (int32_t)g.size());
    base = g.shfl(base, 0);
    return base + (int32_t)g.thread_rank();
}

// Reserves na entries of list A and nb entries of list B for every thread of the
// block, with one atomic per list per block.  Every thread of the block must call
// it at the same point (block-uniform control flow); blockDim.x is a multiple of 32.
__device__ __forceinline__ int2 block_reserve2(int32_t* count_a, int32_t na, int32_t* count_b, int32_t nb)
{
    __shared__ int2 warp_base[32];
    __shared__ int2 block_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    int32_t ia = na, ib = nb;
    for (int o = 1; o < 32; o <<= 1) {
        int32_t ya = __shfl_up_sync(0xffffffffu, ia, o), yb = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= o) { ia += ya; ib += yb; }
    }
    if (lane == 31) warp_base[warp] = make_int2(ia, ib);
    __syncthreads();
    if (warp == 0) {
        int2 v = lane < nwarps ? warp_base[lane] : make_int2(0, 0);
        int32_t xa = v.x, xb = v.y;
        for (int o = 1; o < 32; o <<= 1) {
            int32_t ya = __shfl_up_sync(0xffffffffu, xa, o), yb = __shfl_up_sync(0xffffffffu, xb, o);
            if (lane >= o) { xa += ya; xb += yb; }
        }
        int32_t ta = __shfl_sync(0xffffffffu, xa, 31), tb = __shfl_sync(0xffffffffu, xb, 31);
        if (lane == 0)
            block_base = make_int2(ta && count_a ? atomicAdd(count_a, ta) : 0, tb && count_b ? atomicAdd(count_b, tb) : 0);
        if (lane < nwarps) warp_base[lane] = make_int2(xa - v.x, xb - v.y);
    }
    __syncthreads();
    int2 r = make_int2(block_base.x + warp_base[warp].x + ia - na, block_base.y + warp_base[warp].y + ib - nb);
    __syncthreads();   // the shared slots are reused by the next call
    return r;
}

__device__ __forceinline__ void mark_cell(const DevPop& d, int c)
{
    // cell_flag is a byte array; use the containing 32-bit word for the atomic.
    unsigned int* w = (unsigned int*)(d.cell_flag + (c & ~3));
    unsigned int bit = 1u << ((c & 3) * 8);
    unsigned int old = atomicOr(w, bit);
    if (!(old & bit)) d.touched[append(d.counts + kCntTouched)] = c;
}

__device__ __forceinline__ bool flag_household(const DevPop& d, int h, uint8_t f)
{
    unsigned int* w = (unsigned int*)(d.hh_flag + (h & ~3));
    unsigned int sh = (h & 3) * 8;
    unsigned int old = atomicOr(w, (unsigned int)f << sh);
    if (((old >> sh) & 0xffu) == 0) d.hh_list[append(d.counts + kCntHH)] = h;
    return true;
}

constexpr int kThreads = 256;

// close_window of a run in which no place has been closed
static const int32_t kNoClosures[2] = {INT32_MAX, 0};

// ------------------------------------------------------------- contexts
// Device arrays of a population that never change during runs (households,
// place memberships, cell lists, kernel tables, proposal-block layout, the
// UpdateProbs kernel rows and denominators).  Contexts made by
// cs_gpu_create_replica share one store; the last one destroyed frees it.
struct StaticStore {
    int device = 0;
    std::vector<void*> allocs;
    float* Gtab = nullptr;
    ~StaticStore()
    {
        cudaSetDevice(device);
        for (void* p : allocs) cudaFree(p);
        if (Gtab) cudaFree(Gtab);
    }
};

struct DayCtl;

struct cs_gpu_ctx {
    int device = 0;
    std::shared_ptr<StaticStore> stat;     // static population arrays (possibly shared)
    std::vector<void*>* alloc_to = nullptr;  // where dalloc records allocations (null: allocs)
    int max_cell_people = 0;   // the largest cell's population (cs_gpu_get_sample16's limit)
    void* pack16 = nullptr;    // device staging of cs_gpu_get_sample16
    void* packed = nullptr;    // device staging of cs_gpu_get_sample_packed
    cudaStream_t own_stream = nullptr;     // the context's stream while a batch lends it another
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;           // the place pass's branch beside the spatial pass
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    char err[512] = {0};
    long long launches = 0;
    DevPop d{};
    cs_params hp{};                 // host copy of the parameters
    std::vector<void*> allocs;      // every cudaMalloc of the context
    cs_params* dP = nullptr;
    DevIv* dIv = nullptr;
    double *iv_ci = nullptr, *iv_hq = nullptr;   // the windows' per-admin-unit start times
    cs_counters* dC = nullptr;
    int32_t* d_seed_list = nullptr;
    unsigned long long* d_seed = nullptr;   // device copy of seed (DevPop::seed_src)
    int seed_cap = 0;
    // dense-grid buffers of UpdateProbs' normaliser
    float *S0g = nullptr, *Ng = nullptr, *Ag = nullptr, *Bg = nullptr;
    uint8_t *rowS = nullptr, *rowN = nullptr;
    float* Gtab = nullptr;   // kernel rows of every (source row, target row) pair, or null
    void* xfer = nullptr;    // state-transfer staging (XferSlices)
    float *Apart = nullptr, *Bpart = nullptr;   // per row-chunk partial sums
    uint64_t seed = 0;
    bool run_started = false;
    int grid = 148 * 8;
    int spatial_lanes = 8;   // lanes per spatial contact (2, 4, 8 or 16)
    // one timestep captured as a CUDA graph and replayed
    bool use_graph = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<cudaGraphNode_t> set_step_nodes;
    std::vector<cudaKernelNodeParams> set_step_params;   // their launch parameters, read once at capture
    long long graph_launches = 0;
    // device-side run loop: one graph per day (cs_gpu_run)
    DayCtl* d_ctl = nullptr;
    int32_t* d_clock = nullptr;
    cs_counters* d_series = nullptr;
    int series_cap = 0;
    int day_every_step = -1;    // the probs_every_step the day graph was captured with
    long long geometry_gen = 0; // bumped when set_params replaces the kernel-row table
    size_t tp_smem[2] = {0, 0}; // dynamic shared memory enabled for k_tot_prob_rows<false>, <true>
    // staging of cs_gpu_place_events / cs_gpu_set_mcell_status
    cs_place_event* d_ev = nullptr;
    int ev_cap = 0;
    size_t people_sent = 0;   // people whose arrays cs_gpu_upload_people has queued
    void* d_mc = nullptr;
    size_t mc_cap = 0;
    cudaGraph_t day_graph = nullptr;
    cudaGraphExec_t day_exec = nullptr;
    long long day_launches = 0;
    // optional per-launch timing with events on the context's stream
    bool prof = false;
    struct Rec { const char* name; cudaEvent_t a, b; };
    std::vector<Rec> ring;
    size_t ring_used = 0;
    std::vector<const char*> prof_names;
    std::vector<double> prof_ms;
    std::vector<long long> prof_n;
    // per-kernel timing inside a captured day graph: event-record nodes around each
    // kernel, read after every replay, so that the times are device times between
    // back-to-back graph launches rather than eager launches with host gaps
    bool capturing_prof = false;
    bool day_graph_prof = false;
    std::vector<cudaEvent_t> graph_events;   // pool, reused by later captures
    std::vector<Rec> graph_recs;             // the captured day graph's timed kernels
};

static void drop_day_graph(cs_gpu_ctx* c)
{
    if (c->day_exec) cudaGraphExecDestroy(c->day_exec);
    if (c->day_graph) cudaGraphDestroy(c->day_graph);
    c->day_exec = nullptr;
    c->day_graph = nullptr;
}

static void prof_flush(cs_gpu_ctx* c)
{
    if (!c->ring_used) return;
    cudaEventSynchronize(c->ring[c->ring_used - 1].b);
    for (size_t i = 0; i < c->ring_used; i++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ring[i].a, c->ring[i].b);
        size_t k = 0;
        while (k < c->prof_names.size() && std::strcmp(c->prof_names[k], c->ring[i].name) != 0) k++;
        if (k == c->prof_names.size()) { c->prof_names.push_back(c->ring[i].name); c->prof_ms.push_back(0); c->prof_n.push_back(0); }
        c->prof_ms[k] += ms;
        c->prof_n[k]++;
    }
    c->ring_used = 0;
}

static cudaEvent_t graph_event(cs_gpu_ctx* c, size_t i)
{
    while (c->graph_events.size() <= i) {
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        c->graph_events.push_back(e);
    }
    return c->graph_events[i];
}

static void prof_begin(cs_gpu_ctx* c, const char* name)
{
    if (c->capturing_prof) {   // an event-record node before the kernel's node
        const size_t i = 2 * c->graph_recs.size();
        cs_gpu_ctx::Rec r{name, graph_event(c, i), graph_event(c, i + 1)};
        cudaEventRecordWithFlags(r.a, c->stream, cudaEventRecordExternal);
        c->graph_recs.push_back(r);
        return;
    }
    if (c->ring_used == c->ring.size()) prof_flush(c);
    cs_gpu_ctx::Rec& r = c->ring[c->ring_used];
    r.name = name;
    cudaEventRecord(r.a, c->stream);
}

static void prof_end(cs_gpu_ctx* c)
{
    if (c->capturing_prof) {
        cudaEventRecordWithFlags(c->graph_recs.back().b, c->stream, cudaEventRecordExternal);
        return;
    }
    cudaEventRecord(c->ring[c->ring_used].b, c->stream);
    c->ring_used++;
}

// After a replay of a day graph captured with timing nodes: add its kernels' times.
static void prof_graph_collect(cs_gpu_ctx* c)
{
    if (c->graph_recs.empty()) return;
    cudaEventSynchronize(c->graph_recs.back().b);
    for (const auto& r : c->graph_recs) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        size_t k = 0;
        while (k < c->prof_names.size() && std::strcmp(c->prof_names[k], r.name) != 0) k++;
        if (k == c->prof_names.size()) { c->prof_names.push_back(r.name); c->prof_ms.push_back(0); c->prof_n.push_back(0); }
        c->prof_ms[k] += ms;
        c->prof_n[k]++;
    }
}

static int set_err(cs_gpu_ctx* c, int code, const char* fmt, ...)
{
    if (c) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(c->err, sizeof(c->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return set_err(c, CS_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define LAUNCH(kernel, grid, block, ...)                                                           \
    do {                                                                                           \
        if (c->prof) prof_begin(c, #kernel);                                                       \
        kernel<<<(grid), (block), 0, c->stream>>>(__VA_ARGS__);                                    \
        if (c->prof) prof_end(c);                                                                  \
        c->launches++;                                                                             \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess) return set_err(c, CS_E_CUDA, "launch %s: %s", #kernel, cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
static int dalloc(cs_gpu_ctx* c, T** p, size_t n)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * (n ? n : 1));
    if (e != cudaSuccess) return set_err(c, CS_E_CUDA, "cudaMalloc(%zu bytes): %s", sizeof(T) * n, cudaGetErrorString(e));
    (c->alloc_to ? c->alloc_to : &c->allocs)->push_back(q);
    *p = (T*)q;
    return CS_OK;
}

template <typename T>
static int dupload(cs_gpu_ctx* c, T** p, const T* src, size_t n)
{
    int r = dalloc(c, p, n);
    if (r) return r;
    if (n && src) {
        cudaError_t e = cudaMemcpyAsync(*p, src, sizeof(T) * n, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return set_err(c, CS_E_CUDA, "upload: %s", cudaGetErrorString(e));
    }
    return CS_OK;
}

extern "C" {
static int tot_prob_pass(cs_gpu_ctx* c, bool denominators);
static int build_kernel_rows(cs_gpu_ctx* c);
static int build_block_bounds(cs_gpu_ctx* c);
}

// ================================================================ run start
__global__ void k_reset_people(DevPop d, uint64_t seed)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) *d.ev_init = 1;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.N; p += gridDim.x * blockDim.x) {
        Stream s(seed, CS_RNG_RUN_INIT, 0, (uint32_t)p, 0);
        PersonHot h = d.hot[p];
        h.inf = CS_INF_SUSCEPTIBLE;
        h.sev = CS_SEV_ASYMPTOMATIC | (CS_SEV_ASYMPTOMATIC << 4);
        h.dflags = (uint8_t)(2u << CS_DF_QUAR_COMPLY_SHIFT);
        h.latent_time = 0;
        h.absent_start = kNever;
        h.absent_stop = 0;
        h.isolation_start = kNever;
        h.quar_start = kNever;
        h.infness = 0.0f;
        h.susc = 1.0f;
        d.hot[p] = h;
        d.infection_time[p] = 0;
        d.recovery_time[p] = 0;
        d.sari_time[p] = d.critical_time[p] = d.stepdown_time[p] = kNever;
        d.next_ev[p] = 0xFFFF;
        d.detected_time[p] = 0;
        d.prob_absent[p] = (float)s.next();
        d.prob_care[p] = (float)s.next();
        d.infector[p] = -1;
        d.infect_type[p] = 0;
        d.pstep[p] = 0;
        d.claim[p] = ~0ull;
    }
}

__global__ void k_reset_slots(DevPop d)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.NC; c += gridDim.x * blockDim.x) {
        int b0 = d.cell_start[c], n = d.cell_start[c + 1] - b0;
        d.S[c] = n;
        d.L[c] = d.I[c] = d.R[c] = d.D[c] = 0;
        d.S0[c] = n;
        d.tot_prob[c] = 1.0;
        d.cell_flag[c] = 0;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.N; i += gridDim.x * blockDim.x) {
        int p = d.cell_members[i];
        d.slots[i] = p;
        d.mark[i] = 0;
    }
}

__global__ void k_reset_listpos(DevPop d)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.NC; c += gridDim.x * blockDim.x) {
        int b0 = d.cell_start[c], n = d.cell_start[c + 1] - b0;
        for (int i = 0; i < n; i++) d.listpos[d.cell_members[b0 + i]] = i;
    }
}

__global__ void k_reset_places(DevPop d, int pt, uint64_t seed)
{
    DevPlaces pl = d.pl[pt];
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < pl.n; l += gridDim.x * blockDim.x) {
        Stream s(seed, CS_RNG_PLACE_INIT, 0, (uint32_t)l, (uint32_t)pt);
        pl.close_start[l] = kNever;
        pl.close_end[l] = 0;
        pl.prob_close[l] = (float)s.next();
    }
}

// ============================================================ UpdateProbs
__global__ void k_update_S0(DevPop d, int do_place)
{
    if (d.gate && !*d.gate) return;
    const cs_params& P = *d.P;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.NC; j += gridDim.x * blockDim.x) {
        int n = d.cell_start[j + 1] - d.cell_start[j];
        int s0;
        if (!do_place) {
            s0 = d.S[j] + d.L[j] + d.I[j];
            if (P.DoDeathCountsInS0) {
                s0 += n / 5;
                if ((n < 100) || (s0 > n)) s0 = n;
            }
        } else
            s0 = d.S[j];
        d.S0[j] = s0;
    }
}

// tot_prob of src/CovidSim.cpp:2779-2791 without the dense Ncells^2 tables.
//
// tot_prob_l = A_l / B_l with A_l = sum_m S0_m Kmax(l,m), B_l = sum_m n_m Kmax(l,m)
// and Kmax(l,m) = (float)num(dist2_cc_min(l, m)).  The closest-corner distance
// between two cells depends only on their column distance |dx| and their two rows,
// so a block owning source row yl and a run of source columns evaluates the
// kernel once per (target row ym, |dx|) into shared memory and every thread sums
// its own source cells from there.  Order of summation (restated by the oracle):
//   A_l = sum over ym ascending of ( sum over xm ascending of S0(xm,ym) * G(|xm-xl|) ),
// the inner sum by fused multiply-adds (one rounding per term), zero terms
// skipped (adding +0.0 changes nothing).
__device__ double row_kernel(const DevPop& d, const cs_params& P, int dx, int yl, int ym, unsigned long long* err)
{
    int y1 = yl, y2 = ym;
    if (ym > yl) y1 = yl + 1;
    else if (ym < yl) y2 = ym + 1;
    double d2;
    if (P.DoUTM_coords) {
        int cx = (dx == 0) ? 0 : ((P.cell_width * (double)dx > CSB_REF_PI) ? dx + 1 : dx - 1);
        d2 = dist2_utm(P, 0.0, P.cell_height * (double)y1, P.cell_width * (double)cx, P.cell_height * (double)y2);
    } else {
        int cx = (dx == 0) ? 0 : (((P.DoPeriodicBoundaries) && (P.cell_width * (double)dx > P.width_deg * 0.5)) ? dx + 1 : dx - 1);
        int dy = abs(ym - yl), cy = (dy == 0) ? 0 : dy - 1;
        if ((P.DoPeriodicBoundaries) && (P.height_deg * (double)dy > P.height_deg * 0.5)) cy = dy + 1;
        d2 = periodic_xy(P, P.cell_width * (double)cx, P.cell_height * (double)cy);
    }
    return (double)(float)knum(d, P, d2, err);
}

// The kernel rows are geometry only, so they are evaluated once per context:
// Gtab[(yl * nch + ym) * ncw + dx] = row_kernel(dx, yl, ym), exact in float since
// row_kernel rounds through float.  *oor counts distances beyond the kernel table.
__global__ void k_kernel_rows(DevPop d, float* Gtab, unsigned long long* oor)
{
    const cs_params& P = *d.P;
    const size_t ncw = P.ncw, nch = P.nch, n = nch * nch * ncw;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        int dx = (int)(e % ncw);
        size_t pair = e / ncw;
        int ym = (int)(pair % nch), yl = (int)(pair / nch);
        Gtab[e] = (float)row_kernel(d, P, dx, yl, ym, oor);
    }
}

__global__ void k_grid_values(DevPop d, float* S0g, float* Ng, uint8_t* rowS, uint8_t* rowN)
{
    if (d.gate && !*d.gate) return;
    int nch = d.P->nch;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.NC; c += gridDim.x * blockDim.x) {
        int g = d.cell_grid[c];
        S0g[g] = (float)d.S0[c];
        if (d.S0[c] > 0) rowS[g % nch] = 1;
        if (Ng) {
            int n = d.cell_start[c + 1] - d.cell_start[c];
            Ng[g] = (float)n;
            if (n > 0) rowN[g % nch] = 1;
        }
    }
}

// Each thread owns kTotProbCols = 8 consecutive source columns xl0..xl0+7 of
// source row yl.  Shared memory holds the kernel row mirrored, Gm[off + dx] =
// G(|dx|), so target column xm of output j reads Gm[off + xm - xl0 - j]: for
// sixteen targets xm0..xm0+15 a thread reads one window of 23 values, w[q] =
// Gm[off - 7 + xm0 - xl0 + q], and does 128 fused multiply-adds from registers.
// Gm is stored with one pad slot after every 8 values, so the windows of the 32
// lanes of a warp (9 slots apart) fall in distinct banks.
//
// Arithmetic: FP32, as the reference's float cum_trans sums (src/CovidSim.cpp:2785-2795).
// Summation order, restated by the oracle: for each output, the row sum over xm
// ascending (fused multiply-adds, one rounding per term); row sums added in
// ascending ym within chunks of kTotProbRowChunk target rows; chunk sums added in
// ascending chunk order.  A zero S0 adds +0.0, which changes nothing.  Blocks
// cover `chunks_per_block` chunks each: the sweep uses one chunk per block
// (partial sums, then k_tot_prob_reduce) for parallelism, and the fixed-scratch
// entry point all chunks in one block; both give the same bits.
constexpr int kTotProbCols = 8;
constexpr int kTotProbSpan = 16;          // target columns per register window
constexpr int kTotProbRowChunk = 32;

__host__ __device__ constexpr int tp_phys(int i) { return i + (i >> 3); }

struct TotProbGeom {
    int ncwR;   // target columns rounded up to a multiple of 16 (tail S0 = 0)
    int off;    // Gm index of dx = 0: ncwR + 7, so off - 7 is a multiple of 8
    int gphys;  // values in the padded Gm array
    int nchunks;           // ceil(nch / kTotProbRowChunk)
    int chunks_per_block;  // 1 (partial sums) or nchunks (final sums)
    int need;              // threads per source row: ceil(ncw / 8)
    int rpb;               // source rows per block: 2 when two rows fit 256 threads, else 1
    size_t smem(bool denominators) const
    {
        return sizeof(float) * ((size_t)rpb * gphys + (denominators ? 2 : 1) * (size_t)ncwR);
    }
};

static TotProbGeom tot_prob_geom(int ncw, int nch, bool partial)
{
    TotProbGeom g;
    g.ncwR = (ncw + kTotProbSpan - 1) / kTotProbSpan * kTotProbSpan;
    g.off = g.ncwR + 7;
    g.gphys = tp_phys(g.off + g.ncwR + kTotProbSpan) + 2;
    g.gphys += g.gphys & 1;   // keep the arrays after Gm 8-byte aligned (float2 reads)
    g.nchunks = (nch + kTotProbRowChunk - 1) / kTotProbRowChunk;
    g.chunks_per_block = partial ? 1 : g.nchunks;
    g.need = (ncw + kTotProbCols - 1) / kTotProbCols;
    g.rpb = (2 * g.need <= 256) ? 2 : 1;
    return g;
}

// Out[(z * ncw + xl) * nch + yl] for block z of the chunk dimension.
template <bool kDenominators>
__global__ void __launch_bounds__(256) k_tot_prob_rows(DevPop d, const float* S0g, const float* Ng,
                                                       const uint8_t* rowS, const uint8_t* rowN,
                                                       float* Aout, float* Bout, TotProbGeom gm,
                                                       const float* __restrict__ Gtab)
{
    if (d.gate && !*d.gate) return;
    const cs_params& P = *d.P;
    const int ncw = P.ncw, nch = P.nch;
    extern __shared__ __align__(16) float sh[];
    float* Srow = sh + gm.rpb * gm.gphys;   // ncwR
    float* Nrow = Srow + gm.ncwR;           // ncwR (denominator pass only)
    // rpb == 2: threads [0, need) own source row 2*blockIdx.y, [need, 2*need) the
    // next one, each with its own kernel row Gp; the rest only help fill shared memory
    const int sub = gm.rpb == 2 ? (int)threadIdx.x / gm.need : 0;
    const int jcol = gm.rpb == 2 ? (int)threadIdx.x % gm.need : (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int yl0 = blockIdx.y * gm.rpb;
    const int yl = yl0 + sub;
    float* Gp = sh + (size_t)min(sub, gm.rpb - 1) * gm.gphys;   // this thread's padded, mirrored kernel row
    const int xl0 = (sub < gm.rpb && yl < nch) ? jcol * kTotProbCols : ncw;   // ncw: no outputs
    const int q0 = blockIdx.z * gm.chunks_per_block;
    const int q1 = min(q0 + gm.chunks_per_block, gm.nchunks);
    for (int k = threadIdx.x; k < gm.rpb * gm.gphys; k += blockDim.x) sh[k] = 0.f;
    for (int k = ncw + threadIdx.x; k < gm.ncwR; k += blockDim.x) {
        Srow[k] = 0.f;
        if (kDenominators) Nrow[k] = 0.f;
    }
    float A[kTotProbCols], B[kTotProbCols];
#pragma unroll
    for (int j = 0; j < kTotProbCols; j++) A[j] = B[j] = 0.f;
    // window start of this thread for xm0 = 0, in padded units: phys(off - 7 - xl0 + q)
    // = 9 * (off - 7 - xl0) / 8 + q + q / 8, with off - 7 - xl0 a multiple of 8
    const int t0 = 9 * ((gm.off - 7 - xl0) / 8);
    for (int q = q0; q < q1; q++) {
        float a[kTotProbCols], b[kTotProbCols];
#pragma unroll
        for (int j = 0; j < kTotProbCols; j++) a[j] = b[j] = 0.f;
        const int ym1 = min(nch, (q + 1) * kTotProbRowChunk);
        for (int ym = q * kTotProbRowChunk; ym < ym1; ym++) {
            const bool useS = rowS[ym] != 0, useN = kDenominators && rowN[ym] != 0;
            if (!useS && !useN) continue;
            __syncthreads();
            for (int e = threadIdx.x; e < gm.rpb * ncw; e += blockDim.x) {
                const int r = e / ncw, k = e % ncw, ylr = yl0 + r;
                if (ylr < nch) {
                    float v = Gtab ? Gtab[((size_t)ylr * nch + ym) * ncw + k]
                                   : (float)row_kernel(d, P, k, ylr, ym, CSB_CTR(err_kernel_range));
                    float* G = sh + (size_t)r * gm.gphys;
                    G[tp_phys(gm.off + k)] = v;
                    G[tp_phys(gm.off - k)] = v;
                }
                if (r == 0) {
                    Srow[k] = S0g[(size_t)k * nch + ym];
                    if (kDenominators) Nrow[k] = Ng[(size_t)k * nch + ym];
                }
            }
            __syncthreads();
            if (xl0 >= ncw) continue;
            float sa[kTotProbCols], sb[kTotProbCols];
#pragma unroll
            for (int j = 0; j < kTotProbCols; j++) sa[j] = sb[j] = 0.f;
            for (int xm0 = 0, t = t0; xm0 < gm.ncwR; xm0 += kTotProbSpan, t += 18) {
                float w[kTotProbSpan + kTotProbCols - 1];
#pragma unroll
                for (int r = 0; r < kTotProbSpan + kTotProbCols - 1; r++) w[r] = Gp[t + r + (r >> 3)];
                if (useS) {
                    const float2* s2 = reinterpret_cast<const float2*>(Srow + xm0);
#pragma unroll
                    for (int u2 = 0; u2 < kTotProbSpan / 2; u2++) {
                        const float2 sv = s2[u2];
#pragma unroll
                        for (int j = 0; j < kTotProbCols; j++) sa[j] = fmaf(sv.x, w[2 * u2 - j + 7], sa[j]);
#pragma unroll
                        for (int j = 0; j < kTotProbCols; j++) sa[j] = fmaf(sv.y, w[2 * u2 + 1 - j + 7], sa[j]);
                    }
                }
                if (kDenominators && useN) {
                    const float2* n2 = reinterpret_cast<const float2*>(Nrow + xm0);
#pragma unroll
                    for (int u2 = 0; u2 < kTotProbSpan / 2; u2++) {
                        const float2 nv = n2[u2];
#pragma unroll
                        for (int j = 0; j < kTotProbCols; j++) sb[j] = fmaf(nv.x, w[2 * u2 - j + 7], sb[j]);
#pragma unroll
                        for (int j = 0; j < kTotProbCols; j++) sb[j] = fmaf(nv.y, w[2 * u2 + 1 - j + 7], sb[j]);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < kTotProbCols; j++) {
                if (useS) a[j] = a[j] + sa[j];
                if (kDenominators && useN) b[j] = b[j] + sb[j];
            }
        }
#pragma unroll
        for (int j = 0; j < kTotProbCols; j++) {
            A[j] = A[j] + a[j];
            if (kDenominators) B[j] = B[j] + b[j];
        }
    }
    const size_t zofs = (size_t)blockIdx.z * ncw * nch;
#pragma unroll
    for (int j = 0; j < kTotProbCols; j++) {
        int xl = xl0 + j;
        if (xl < ncw) {
            Aout[zofs + (size_t)xl * nch + yl] = A[j];
            if (kDenominators) Bout[zofs + (size_t)xl * nch + yl] = B[j];
        }
    }
}

// Chunk sums added in ascending chunk order: out[g] = sum over z of part[z][g].
__global__ void k_tot_prob_reduce(const float* __restrict__ part, int nparts, size_t G, float* __restrict__ out,
                                  const int32_t* gate)
{
    if (gate && !*gate) return;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < G; g += (size_t)gridDim.x * blockDim.x) {
        float A = 0.f;
        for (int z = 0; z < nparts; z++) A = A + part[(size_t)z * G + g];
        out[g] = A;
    }
}

// Launch shape of k_tot_prob_rows: ceil(ncw / 8) threads per source row, in
// blocks of up to 256 threads (whole warps).
static void tot_prob_launch_shape(int ncw, int nch, const TotProbGeom& gm, dim3* grid, int* threads)
{
    (void)ncw;
    int tpb = ((gm.rpb * gm.need + 31) / 32) * 32;
    if (tpb > 256) tpb = 256;
    *threads = tpb;
    const int xblocks = gm.rpb == 2 ? 1 : (gm.need + tpb - 1) / tpb;
    *grid = dim3(xblocks, (nch + gm.rpb - 1) / gm.rpb, gm.nchunks / gm.chunks_per_block);
}

__global__ void k_tot_prob_finish(DevPop d, const float* Ag, const float* Bg)
{
    if (d.gate && !*d.gate) return;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.NC; c += gridDim.x * blockDim.x) {
        int g = d.cell_grid[c];
        const double b = (double)Bg[g];
        d.tot_prob[c] = (b > 0) ? (double)Ag[g] / b : 0.0;
    }
}

__global__ void k_block_S0(DevPop d)
{
    if (d.gate && !*d.gate) return;
    for (int B = blockIdx.x * blockDim.x + threadIdx.x; B < d.NB; B += gridDim.x * blockDim.x) {
        long long s = 0;
        int k0 = d.block_cell_ofs[B], k1 = d.block_cell_ofs[B + 1];
        for (int k = k0; k < k1; k++) {
            int m = d.block_cells[k], s0 = d.S0[m];
            s += s0;
            d.block_cell_info[k] = BlockCell{(int32_t)s, m, d.cell_start[m], s0};
        }
        d.block_info[B] = BlockInfo{s, k0, k1};
        // cut points of the block's cells: entry k0+q = first cell whose running S0
        // exceeds q/nc of the block total
        int nc = k1 - k0, j = k0;
        for (int q = 0; q < nc; q++) {
            double thr = (double)q * (double)s / (double)nc;
            while (j < k1 - 1 && (double)d.block_cell_info[j].cum <= thr) j++;
            d.cell_guide[k0 + q] = (int16_t)(j - k0);
        }
    }
}

// Every bound of the geometry by (row of b, row of B, column distance), once per
// population, rounded up to FP32 so that it still bounds K; *oor counts distances
// beyond the kernel table (then the bounds are evaluated per call instead, so that
// the error counts stay those of the per-call evaluation).
__global__ void k_block_bounds_all(DevPop d, float* bound_c, unsigned long long* oor)
{
    const cs_params& P = *d.P;
    const size_t n = (size_t)d.nby * d.nby * d.nbx;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int dx = (int)(e % d.nbx), By = (int)((e / d.nbx) % d.nby), by = (int)(e / ((size_t)d.nbx * d.nby));
        bound_c[e] = __double2float_ru(block_bound_rel(d, P, by, By, dx, oor));
    }
}

// Row b of the proposal table: running sum over B of S0_B * bound(b, B), added in
// B order so the doubles round exactly as a sequential loop.
__global__ void k_block_rows(DevPop d)
{
    if (d.gate && !*d.gate) return;
    const cs_params& P = *d.P;
    int lane = threadIdx.x & 31;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int b = warp; b < d.NB; b += nwarps) {
        double* row = d.block_row_cum + (size_t)b * d.NB;
        double* btab = d.bounds_static ? nullptr : d.block_bound_tab + (size_t)b * d.NB;
        double s = 0.0;
        for (int B0 = 0; B0 < d.NB; B0 += 32) {
            int B = B0 + lane;
            double w = 0.0;
            if (B < d.NB && d.block_info[B].S0 > 0) {
                double bound;
                if (d.bounds_static) bound = bound_of(d, b, B);
                else btab[B] = bound = block_bound(d, P, b, B, CSB_CTR(err_kernel_range));
                w = (double)d.block_info[B].S0 * bound;
            }
            for (int k = 0; k < 32; k++) {
                double wk = __shfl_sync(0xffffffffu, w, k);
                if (B0 + k < d.NB) {
                    s = s + wk;
                    if (lane == k) row[B] = s;
                }
            }
        }
        // guide[k] = first B whose running weight exceeds k/NB of the row total (the
        // last block if none): thresholds and the row both ascend, so each lane
        // finds its entries by binary search
        __syncwarp();
        int16_t* guide = d.block_guide + (size_t)b * d.NB;
        const double total = s;
        for (int k = lane; k < d.NB; k += 32) {
            double thr = (double)k * total / (double)d.NB;
            int lo = 0, hi = d.NB - 1;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (row[mid] <= thr) lo = mid + 1; else hi = mid;
            }
            guide[k] = (int16_t)lo;
        }
    }
}

// ======================================================== active-list build
// The step's active people, cell by cell: infectious, slots [S+L, S+L+I) (mode 0),
// or latent and infectious, slots [S, S+L+I) (mode 1).  The cells come in tiles of
// blockDim.x; Q = gridDim.x / tiles blocks share a tile, block q copying its chunks
// q, q + Q, ... of blockDim.x entries (entry j by the thread whose turn it is), so a
// cell with thousands of active people costs no more than its share and the launch
// has the parallelism of the list.  Each chunk reserves its entries at once, so the
// list's order varies from launch to launch; nothing that reads it depends on the
// order (random streams are keyed by person and contact, conflicting claims resolve
// by key, tallies are integer sums, and cell lists are reordered by position).
__device__ __forceinline__ void k_build_active_body(const DevPop& d, int mode)
{
    __shared__ int s_first[kThreads], s_ofs[kThreads], s_n[kThreads];
    const int ntiles = (d.NC + blockDim.x - 1) / blockDim.x;
    const int Q = max(1, (int)gridDim.x / ntiles), part = blockIdx.x % Q;
    for (int tile = blockIdx.x / Q; tile < ntiles; tile += max(1, (int)gridDim.x / Q)) {
        const int c0 = tile * blockDim.x;
        const int c = c0 + threadIdx.x;
        int first = 0, n = 0;
        if (c < d.NC) {
            first = d.cell_start[c] + d.S[c] + (mode == 0 ? d.L[c] : 0);
            n = mode == 0 ? d.I[c] : d.L[c] + d.I[c];
        }
        const int o = block_reserve2(nullptr, n, nullptr, 0).x;   // the block's own prefix of n
        s_first[threadIdx.x] = first;
        s_ofs[threadIdx.x] = o;
        s_n[threadIdx.x] = n;
        __syncthreads();
        const int total = s_ofs[blockDim.x - 1] + s_n[blockDim.x - 1];
        for (int j0 = part * blockDim.x; j0 < total; j0 += Q * blockDim.x) {   // block-uniform: every thread reserves
            const int j = j0 + (int)threadIdx.x;
            const bool valid = j < total;
            int p = 0, cell = 0;
            if (valid) {
                int lo = 0, hi = blockDim.x - 1;   // the last cell whose entries start at or before j
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (s_ofs[mid] <= j) lo = mid; else hi = mid - 1;
                }
                p = d.slots[s_first[lo] + (j - s_ofs[lo])];
                cell = c0 + lo;
            }
            const int e = block_reserve2(d.counts + kCntAct, valid ? 1 : 0, nullptr, 0).x;
            if (valid) {
                d.act[e] = p;
                d.act_cell[e] = cell;
            }
        }
        __syncthreads();   // the shared arrays are refilled for the next cells
    }
}
__global__ void k_build_active(DevPop d, int mode) { k_build_active_body(d, mode); }
__global__ void k_build_active_multi(const DevPop* __restrict__ pops, int mode) { k_build_active_body(pops[blockIdx.y], mode); }

// =============================================================== InfectSweep
typedef DevStep StepScalars;

// AddInfections (src/Sweep.cpp:2031-2065): with probability FalsePositiveRate the
// entry is a false positive (DoFalseCase for the person) instead of an infection.
// The draw is keyed by (infector, infectee, infection type), one per entry.
__device__ __forceinline__ void claim_infection(const DevPop& d, const cs_params& P, const StepScalars& st, int person,
                                                int infector, int code)
{
    if (P.FalsePositiveRate > 0) {
        Stream s(st.seed, CS_RNG_FALSE_POSITIVE, (uint32_t)st.ts, (uint32_t)infector, (uint32_t)person);
        s.block = (uint32_t)code;
        if (s.next() < P.FalsePositiveRate) {
            const uint32_t bit = 1u << (person & 31);
            if (!(atomicOr(d.fc_flag + (person >> 5), bit) & bit)) d.fc_queue[append(d.counts + kCntFalse)] = person;
            return;
        }
    }
    unsigned long long key = ((unsigned long long)(uint32_t)infector << 8) | (unsigned long long)code;
    unsigned long long old = atomicMin(d.claim + person, key);
    if (old == ~0ull) d.queue[append(d.counts + kCntQueue)] = person;
}

// The step's scalars from the parameters, on the device (src/Sweep.cpp:292-301).
__device__ __forceinline__ void k_set_step_body(const DevPop& d, double t, unsigned long long seed)
{
    const cs_params& P = *d.P;
    if (d.t_src) t = *d.t_src;
    if (d.step_clock) {
        int k = *d.step_clock;
        t = (double)k * P.ModelTimeStep;
        *d.step_clock = k + 1;
    }
    if (d.seed_src) seed = *d.seed_src;
    DevStep st;
    st.t = t;
    st.ts = (int)(uint16_t)(P.TimeStepsPerDay * t);
    st.blanket = P.DoBlanketMoveRestr && (t >= P.MoveRestrTimeStart) && (t < P.MoveRestrTimeStart + P.MoveRestrDuration);
    st.fp = P.ModelTimeStep / (1 - P.FalsePositiveRate);
    st.seas = P.Seasonality;
    st.sp_beta = P.DoSpatial ? st.seas * st.fp * P.LocalBeta : 0.0;
    st.hh_beta = P.DoHouseholds ? st.seas * st.fp * P.HouseholdTrans : 0.0;
    st.seed = seed;
    *d.step = st;
}
__global__ void k_set_step(DevPop d, double t, unsigned long long seed) { k_set_step_body(d, t, seed); }
__global__ void k_set_step_multi(const DevPop* __restrict__ pops, double t, unsigned long long seed) { k_set_step_body(pops[blockIdx.y], t, seed); }

// Geometric-skip enumeration of the Bernoulli(p) trials over a member list
// (equivalent to the reference's Binomial count + sample without replacement,
// src/Sweep.cpp:463-470 and 563-566).
__device__ void place_candidates(const DevPop& d, const cs_params& P, const StepScalars& st, int i, const PersonHot& hi,
                                 int pt, int link, double p, bool between, uint64_t seed)
{
    const DevPlaces& pl = d.pl[pt];
    int base = pl.member_ofs[link], n;
    int gi = group_of(d, pt, i);
    if (!between) {
        int g = pl.group_ofs[link] + gi;
        base += pl.group_start[g];
        n = pl.group_size[g];
    } else
        n = pl.member_ofs[link + 1] - pl.member_ofs[link];
    if (p <= 0 || n <= 0) return;
    int mc_place = pl.mcell[link];
    Stream s(seed, between ? CS_RNG_PLACE_BETWEEN : CS_RNG_PLACE_GROUP, (uint32_t)st.ts, (uint32_t)i, (uint32_t)pt);
    double logq = (p < 1.0) ? log1p(-p) : 0.0;
    double pos = -1.0;
    int iag = age_group(hi);
    bool ich = is_ch(hi);
    long long ncand = 0;
    for (;;) {
        if (p >= 1.0) pos = pos + 1.0;
        else pos = pos + 1.0 + floor(log(s.next()) / logq);
        if (!(pos < (double)n)) break;
        int m = pl.members[base + (int)pos];
        ncand++;
        PersonHot hm = d.hot[m];
        if (hm.inf == CS_INF_SUSCEPTIBLE && !host_absent(hm, st.ts)) {
            // the susceptibility is formed only for a candidate it can matter to (the
            // same factors in the same order as for every candidate)
            double sc = calc_place_susc(d, hm, P, pt, st.ts);
            if (between && ich && is_ch(hm) && gi != group_of(d, pt, m)) sc *= P.CareHomeResidentPlaceScaling;
            if ((pt == P.CareHomePlaceType) && ((!ich) || (!is_ch(hm)))) sc *= P.CareHomeWorkerGroupScaling;
            sc *= calc_person_susc(hm, iag, P) * p / p;
            if (st.blanket) {
                if (dist2_hh_pt(d, P, hm.hh, pl.x[link], pl.y[link]) > P.MoveRestrRadius2) sc *= P.MoveRestrEffect;
            } else if (moverest_differs(d, hm.mcell, mc_place))
                sc *= P.MoveRestrEffect;
            if ((sc == 1) || (s.next() < sc)) claim_infection(d, P, st, m, i, between ? 2 + pt + CS_MAX_PLACE_TYPES : 2 + pt);
        }
    }
    cnt_add_warp(CSB_CTR(work_place_candidates), ncand);
}

// Household pass and spatial Poisson count of one infector (src/Sweep.cpp:331-377,
// 656-698); one thread per infector.
__device__ __forceinline__ void k_infector_hh_spatial_body(const DevPop& d)
{
    const cs_params& P = *d.P;
    const StepScalars st = *d.step;
    const uint64_t seed = st.seed;
    int nact = d.counts[kCntAct];
    const bool anyc = closures_possible(d, st.ts);
    long long hh_members = 0;
    // block-uniform loop: every thread takes part in the list reservations
    for (int base = blockIdx.x * blockDim.x; base < nact; base += gridDim.x * blockDim.x) {
        const int idx = base + threadIdx.x;
        int links[CS_MAX_PLACE_TYPES];
        int nwork = 0, k = 0;
        uint8_t closed_i = 0;
        bool absent_i = true;
        if (idx < nact) {
            int i = d.act[idx], ci = d.act_cell[idx];
            PersonHot hi = d.hot[i];
            int h = hi.hh;
            int iag = age_group(hi);
            const HouseholdRec hr = load_household(d, h);
            uint16_t nh = hr.nh;
            if (st.hh_beta > 0 && nh > 1) {
                int f0 = hr.first, f1 = f0 + nh;
                double HI = st.hh_beta * calc_house_inf(hi, hr.nhr, P, st.ts);
                bool absent = false;
                for (int m = f0; anyc && (m < f1) && (!absent); m++) {
                    // a member counts only when absent: its places are read only then
                    if (!host_absent(d.hot[m], st.ts)) continue;
                    for (int pt = 0; (pt < d.NPT) && (!absent); pt++) {
                        int lk = link_of(d, pt, m);
                        if (lk >= 0) absent = place_closed(d, pt, lk, st.ts);
                    }
                }
                if (absent) HI *= P.Efficacies[CS_NPI_PLACE_CLOSURE][CS_SETTING_HOUSE];
                Stream s(seed, CS_RNG_HOUSEHOLD, (uint32_t)st.ts, (uint32_t)i, 0);
                for (int m = f0; m < f1; m++) {
                    hh_members++;
                    PersonHot hm = d.hot[m];
                    if (hm.inf == CS_INF_SUSCEPTIBLE) {
                        double foi = HI * calc_house_susc(d, hm, iag, P);
                        if (s.next() < foi) claim_infection(d, P, st, m, i, 1);
                    }
                }
            }
            // the infector's place passes: one work entry per place it attends today
            absent_i = host_absent(hi, st.ts);
            const PersonLinks pli = load_links(d, i);
            for (int pt = 0; pt < d.NPT; pt++) {
                links[pt] = P.DoPlaces ? pli.link[pt] : -1;
                if (links[pt] >= 0 && !absent_i) nwork++;
            }
            if (st.sp_beta > 0) {
                double si = calc_spatial_inf(hi, P, st.ts);
                bool closed = false;   // counts only for an absent infector
                for (int pt = 0; anyc && absent_i && (pt < d.NPT) && (!closed); pt++)
                    if (links[pt] >= 0) closed = place_closed(d, pt, links[pt], st.ts);
                if (closed && absent_i) { si *= P.Efficacies[CS_NPI_PLACE_CLOSURE][CS_SETTING_SPATIAL]; closed_i = 1; }
                double lambda = si * st.sp_beta * d.tot_prob[ci];
                Stream s(seed, CS_RNG_SPATIAL_COUNT, (uint32_t)st.ts, (uint32_t)i, 0);
                k = sample_poisson(s, lambda, CSB_CTR(err_spatial_tries));
            }
        }
        // place-work entries [ow, ow + nwork) and contact-map entries [oc, oc + k)
        const int2 o = block_reserve2(d.counts + kCntPlaceWork, nwork, d.counts + kCntContacts, k);
        if (idx < nact) {
            int ow = o.x;
            for (int pt = 0; pt < d.NPT; pt++)
                if (links[pt] >= 0 && !absent_i) d.place_work[ow++] = make_int2((idx << 3) | pt, links[pt]);
            d.cnt_ofs[idx] = o.y;
            for (int jj = 0; jj < k && o.y + jj < d.cmap_cap; jj++) d.cmap[o.y + jj] = idx;
            d.act_closed[idx] = closed_i;
        }
    }
    cnt_add_warp(CSB_CTR(work_hh_members), hh_members);
}
__global__ void __launch_bounds__(kThreads) k_infector_hh_spatial(DevPop d) { k_infector_hh_spatial_body(d); }
__global__ void __launch_bounds__(kThreads) k_infector_hh_spatial_multi(const DevPop* __restrict__ pops) { k_infector_hh_spatial_body(pops[blockIdx.y]); }

// Place passes (src/Sweep.cpp:379-647): one thread per (infector, place) work
// entry, i.e. per place type the infector attends and is not absent from.
__device__ __forceinline__ void k_infector_places_body(const DevPop& d)
{
    const cs_params& P = *d.P;
    const StepScalars st = *d.step;
    const uint64_t seed = st.seed;
    int n = d.counts[kCntPlaceWork];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        int2 e = d.place_work[t];
        int idx = e.x >> 3, pt = e.x & 7, link = e.y;
        int i = d.act[idx];
        PersonHot hi = d.hot[i];
        double PI = st.fp * st.seas * calc_place_inf(hi, P, pt, st.ts);
        if (st.blanket) {
            if (dist2_hh_pt(d, P, hi.hh, d.pl[pt].x[link], d.pl[pt].y[link]) > P.MoveRestrRadius2)
                PI *= P.MoveRestrEffect;
        } else if (moverest_differs(d, hi.mcell, d.pl[pt].mcell[link]))
            PI *= P.MoveRestrEffect;
        if (pt != P.HotelPlaceType) {
            double p1 = PI;
            if (p1 > 1) p1 = 1;
            place_candidates(d, P, st, i, hi, pt, link, p1, false, seed);
        }
        int np = d.pl[pt].member_ofs[link + 1] - d.pl[pt].member_ofs[link];
        double p2 = PI * (P.PlaceTypePropBetweenGroupLinks[pt] * P.PlaceTypeGroupSizeParam1[pt] / ((double)np));
        if (p2 > 1) p2 = 1;
        place_candidates(d, P, st, i, hi, pt, link, p2, true, seed);
    }
}
__global__ void __launch_bounds__(kThreads) k_infector_places(DevPop d) { k_infector_places_body(d); }
__global__ void __launch_bounds__(kThreads) k_infector_places_multi(const DevPop* __restrict__ pops) { k_infector_places_body(pops[blockIdx.y]); }

// Spatial contacts (src/Sweep.cpp:742-856): pick a target block from the infector's
// block row, a slot uniformly among the block's S0 slots, accept with K(d)/bound,
// redraw on rejection or a dead target.  Draw t of a contact reads its uniforms
// from Philox blocks 2t and 2t+1 of the contact's stream, so the draws are
// independent of one another: LANES lanes (4, 8 or 16, a tuning choice that does
// not change results) evaluate draws t0..t0+LANES-1 together and the lowest
// accepted one wins, exactly as a sequential loop would.
constexpr uint32_t kSpatialBlocksPerDraw = 2;

// One rejection draw; true when accepted (target alive, u < K(d)/bound).
__device__ __forceinline__ bool spatial_draw(const DevPop& d, const cs_params& P, Stream& s, int b,
                                             const double* row, const int16_t* guide_row, double total,
                                             int hh_inf, int& m_out, int& slot_out, int& p_out,
                                             PersonHot& hp_out, double& d2_out, int* oor)
{
    // smallest B with target < row[B]: guide-table start, then walk
    double u1 = s.next();
    double target = u1 * total;
    int B = guide_row[min((int)(u1 * (double)d.NB), d.NB - 1)];
    while (B > 0 && row[B - 1] > target) B--;
    while (B < d.NB - 1 && !(target < row[B])) B++;
    const BlockInfo bi = d.block_info[B];
    long long bS0 = bi.S0;
    if (bS0 <= 0) return false;
    double u2 = s.next();
    double r = floor(u2 * (double)bS0);
    // smallest cell k in block B with r < cum[k], the same way
    int kb = bi.kb, ke = bi.ke - 1;
    int k0 = kb + d.cell_guide[kb + min((int)(u2 * (double)(ke - kb + 1)), ke - kb)];
    while (k0 > kb && r < (double)d.block_cell_info[k0 - 1].cum) k0--;
    while (k0 < ke && !(r < (double)d.block_cell_info[k0].cum)) k0++;
    const BlockCell bc = d.block_cell_info[k0];
    int m = bc.m;
    int slot = (int)(r - (double)(bc.cum - bc.s0));
    int p = d.slots[bc.start + slot];
    PersonHot hp = d.hot[p];
    double d2 = dist2_hh(d, P, hh_inf, hp.hh);
    double accept = knum_f32(d, P, d2, oor) / bound_of(d, b, B);
    if ((s.next() >= accept) || !is_alive(hp.inf)) return false;
    m_out = m; slot_out = slot; p_out = p; hp_out = hp; d2_out = d2;
    return true;
}

template <int kSpatialLanes>
__device__ __forceinline__ void k_spatial_body(const DevPop& d)
{
    const cs_params& P = *d.P;
    const StepScalars st = *d.step;
    const uint64_t seed = st.seed;
    int nact = d.counts[kCntAct];
    int nres = d.counts[kCntContacts];
    int ncont = min(nres, d.cmap_cap);   // contacts beyond the map are counted as overflow
    auto tile = cg::tiled_partition<kSpatialLanes>(cg::this_thread_block());
    const int lane = (int)tile.thread_rank();
    const int group = (blockIdx.x * blockDim.x + threadIdx.x) / kSpatialLanes;
    const int ngroups = (gridDim.x * blockDim.x) / kSpatialLanes;
    long long draws = 0, oor_count = 0, give_ups = 0;
    for (int cidx = group; cidx < ncont; cidx += ngroups) {
        int idx = d.cmap[cidx];            // the infector owning contact cidx
        int j = cidx - d.cnt_ofs[idx];
        int i = d.act[idx], ci = d.act_cell[idx];
        bool closed_i = d.act_closed[idx] != 0;
        PersonHot hinf = d.hot[i];
        int b = d.cell_block[ci];
        const double* row = d.block_row_cum + (size_t)b * d.NB;
        const int16_t* guide_row = d.block_guide + (size_t)b * d.NB;
        double total = row[d.NB - 1];
        if (!(total > 0)) { if (lane == 0) give_ups++; continue; }
        int m = 0, slot = 0, p = 0, won = -1;
        double d2w = 0.0;
        PersonHot hp;
        Stream s(seed, CS_RNG_SPATIAL_CONTACT, (uint32_t)st.ts, (uint32_t)i, (uint32_t)j);
        for (int t0 = 0; t0 < kMaxSpatialTries; t0 += kSpatialLanes) {
            int t = t0 + lane, oor = 0;
            s = Stream(seed, CS_RNG_SPATIAL_CONTACT, (uint32_t)st.ts, (uint32_t)i, (uint32_t)j);
            s.block = kSpatialBlocksPerDraw * (uint32_t)t;
            bool acc = (t < kMaxSpatialTries) && spatial_draw(d, P, s, b, row, guide_row, total, hinf.hh,
                                                              m, slot, p, hp, d2w, &oor);
            unsigned mask = tile.ballot(acc);
            int w = mask ? __ffs(mask) - 1 : kSpatialLanes;
            if (lane < w) oor_count += oor;   // draws up to the winner count, as in a sequential loop
            if (lane == w) oor_count += oor;
            if (mask) { won = t0 + w; break; }
        }
        if (lane == 0) draws += (won >= 0) ? won + 1 : kMaxSpatialTries;
        if (won < 0) { if (lane == 0) give_ups++; continue; }
        if (lane != won % kSpatialLanes) continue;
        if ((ci != m) || (hp.hh != hinf.hh)) {
            int iag = age_group(hinf);
            double ss = calc_spatial_susc(d, hp, P, st.ts);
            if (is_ch(hp) || is_ch(hinf)) ss *= P.CareHomeResidentSpatialScaling;
            if (slot < d.S[m]) {
                ss *= calc_person_susc(hp, iag, P);
                ss *= P.WAIFW_Matrix_SpatialOnly[age_group(hp)][iag];
                if (st.blanket) {   // the draw's distance is dist2_raw's with UTM coordinates
                    const double d2b = P.DoUTM_coords ? d2w : dist2_hh_raw(d, P, hinf.hh, hp.hh);
                    if (d2b > P.MoveRestrRadius2) ss *= P.MoveRestrEffect;
                } else if (moverest_differs(d, hp.mcell, hinf.mcell))
                    ss *= P.MoveRestrEffect;
                if ((!closed_i) && closures_possible(d, st.ts) && host_absent(hp, st.ts)) {
                    bool f = false;
                    for (int pt = 0; (pt < d.NPT) && (!f); pt++) {
                        int lk = link_of(d, pt, p);
                        if (lk >= 0) f = place_closed(d, pt, lk, st.ts);
                    }
                    if (f) ss *= P.Efficacies[CS_NPI_PLACE_CLOSURE][CS_SETTING_SPATIAL];
                }
                if ((ss == 1) || (s.next() < ss))
                    if (hp.inf == CS_INF_SUSCEPTIBLE) claim_infection(d, P, st, p, i, 2 + 2 * CS_MAX_PLACE_TYPES);
            }
        }
    }
    cnt_add_warp(CSB_CTR(work_spatial_draws), draws);
    cnt_add_warp(CSB_CTR(err_kernel_range), oor_count);
    cnt_add_warp(CSB_CTR(err_spatial_tries), give_ups);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cnt_add(CSB_CTR(work_infectors), nact);
        cnt_add(CSB_CTR(work_spatial_contacts), ncont);
        if (nres > ncont) cnt_add(CSB_CTR(err_queue_overflow), nres - ncont);
    }
}
template <int kSpatialLanes>
__global__ void __launch_bounds__(kThreads, 3) k_spatial(DevPop d) { k_spatial_body<kSpatialLanes>(d); }
template <int kSpatialLanes>
__global__ void __launch_bounds__(kThreads, 3) k_spatial_multi(const DevPop* __restrict__ pops) { k_spatial_body<kSpatialLanes>(pops[blockIdx.y]); }

// DoInfect (src/Update.cpp:100-195) for every person claimed this step.
__device__ __forceinline__ void k_apply_infections_body(const DevPop& d)
{
    const cs_params& P = *d.P;
    const double t = d.step->t;
    const int ts = d.step->ts;
    const uint64_t seed = d.step->seed;
    int nq = d.counts[kCntQueue];
    if (blockIdx.x * blockDim.x >= nq) return;   // a block without work stages nothing
    const bool staged = nq >= kStageMinItems;
    stage_begin(d.C, staged);
    // single-address tallies, summed per thread and added once per warp
    long long n_inf = 0, n_kw = 0, n_tg = 0, sum_tg = 0, sum_si = 0, rad_q = 0, rad_max = 0;
    const double ox = d.rad_origin[0], oy = d.rad_origin[1];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        int p = d.queue[q];
        unsigned long long key = d.claim[p];
        d.claim[p] = ~0ull;
        int32_t infector = (int32_t)(uint32_t)(key >> 8);
        int code = (int)(key & 0xff);
        int16_t it = (infector >= 0)
            ? (int16_t)(code + CS_INFECT_TYPE_MASK * (1 + d.infect_type[infector] / CS_INFECT_TYPE_MASK))
            : (int16_t)code;
        PersonHot h = d.hot[p];
        h.inf = CS_INF_LATENT;
        d.infection_time[p] = (uint16_t)ts;
        d.infector[p] = infector;
        d.infect_type[p] = it;
        int cell = d.mcell_cell[h.mcell];
        atomicSub(d.S + cell, 1);
        atomicAdd(d.L + cell, 1);
        d.mark[d.cell_start[cell] + d.listpos[p]] = 1;
        atomicAdd(d.cnt + cell, 1);  // transitions out of this cell's S block
        mark_cell(d, cell);
        n_inf++;
        if (infector != -2) {   // a seed's radius is 0 (the origin moved to it)
            const HouseholdRec hr = load_household(d, h.hh);
            const double x = (double)hr.x - ox, y = (double)hr.y - oy;
            const double r2 = x * x + y * y;
            rad_q += (long long)(r2 * 4294967296.0);
            rad_max = max(rad_max, __double_as_longlong(r2));
        }
        cnt_add(CSB_STAGED(cumItype[it % CS_INFECT_TYPE_MASK]), 1);
        cnt_add(CSB_STAGED(cumIa[age_group(h)]), 1);
        if (h.pflags & CS_PF_KEYWORKER) n_kw++;
        int ad = d.mcell_adunit[h.mcell];
        if (ad >= 0 && ad < CS_MAX_ADUNITS) cnt_add(CSB_STAGED(cumI_adunit[ad]), 1);
        if (P.DoLatent) {
            Stream s(seed, CS_RNG_LATENT, (uint32_t)ts, (uint32_t)p, 0);
            double qq;
            int i = (int)floor((qq = s.next() * CS_CDF_RES));
            qq -= (double)i;
            h.latent_time = (uint16_t)floor(0.5 + (t - P.LatentPeriod * log(qq * P.latent_icdf.v[i + 1] + (1.0 - qq) * P.latent_icdf.v[i])) * P.TimeStepsPerDay);
        } else
            h.latent_time = (uint16_t)(t * P.TimeStepsPerDay);
        d.hot[p] = h;
        d.next_ev[p] = h.latent_time;
        if (infector >= 0) {
            sum_tg += ((int)(uint16_t)ts) - ((int)d.infection_time[infector]);
            sum_si += ((int)h.latent_time) - ((int)d.hot[infector].latent_time);
            n_tg++;
        }
    }
    cnt_add_warp(CSB_CTR(cumI), n_inf);
    cnt_add_warp(CSB_CTR(cumI_keyworker[1]), n_kw);
    cnt_add_warp(CSB_CTR(cumI_keyworker[0]), n_inf - n_kw);
    cnt_add_warp(CSB_CTR(cumTG), sum_tg);
    cnt_add_warp(CSB_CTR(cumSI), sum_si);
    cnt_add_warp(CSB_CTR(nTG), n_tg);
    cnt_add_warp(CSB_CTR(sumRad2_q), rad_q);
    {
        long long m = rad_max;
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0 && m > 0) atomicMax((long long*)CSB_CTR(maxRad2_bits), m);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt_add(CSB_STAGED(work_new_infections), nq);
    stage_flush(d.C, staged);
}
__global__ void k_apply_infections(DevPop d) { k_apply_infections_body(d); }
__global__ void k_apply_infections_multi(const DevPop* __restrict__ pops) { k_apply_infections_body(pops[blockIdx.y]); }

// Swap-with-block-end removal of marked slots, high to low (src/Update.cpp:1402-1579
// UpdateCell sequence).  Moved people get their new listpos.  One warp per block:
// the warp reads the marks 32 positions at a time from the top and lane 0 applies
// the swaps in descending position order, as a serial scan would.  A swap writes
// only at its own position and above, so the marks the warp read for the positions
// still below are the ones a serial scan would find there.
__device__ void partition_block_warp(const DevPop& d, int base, int b0, int n, int nmarked, uint8_t want,
                                     bool relay_exit)
{
    const int lane = threadIdx.x & 31;
    int cur = n, removed = 0;
    for (int top = b0 + n - 1; top >= b0 && removed < nmarked; top -= 32) {
        const int pos = top - lane;
        unsigned hits = __ballot_sync(0xffffffffu, pos >= b0 && d.mark[pos] == want);
        if (lane == 0) {
            while (hits && removed < nmarked) {
                const int p = top - (__ffs(hits) - 1);   // lowest lane: highest position
                hits &= hits - 1;
                cur--;
                removed++;
                const int end = b0 + cur;
                if (p < end) {
                    int a = d.slots[p], e = d.slots[end];
                    d.slots[p] = e;
                    d.listpos[e] = p - base;
                    d.slots[end] = a;
                    d.listpos[a] = end - base;
                }
                d.mark[p] = 0;
                d.mark[end] = 0;
                if (relay_exit) {
                    int a = d.slots[end];
                    if (d.pstep[a] & kStepItoRD) d.mark[end] = 2;
                }
            }
        }
        removed = __shfl_sync(0xffffffffu, removed, 0);
        __syncwarp();
    }
}

// S -> L list moves for every cell that gained latent people this step, one warp
// per cell.
__device__ __forceinline__ void k_partition_S_body(const DevPop& d)
{
    int nt = d.counts[kCntTouched];
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt_add(CSB_CTR(work_cells_touched), nt);
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < nt; k += warps) {
        int c = d.touched[k];
        int moved = d.cnt[c];
        int base = d.cell_start[c];
        partition_block_warp(d, base, base, d.S[c] + moved, moved, 1, false);
        if ((threadIdx.x & 31) == 0) {
            d.cnt[c] = 0;
            d.cell_flag[c] = 0;
        }
    }
}
__global__ void k_partition_S(DevPop d) { k_partition_S_body(d); }
__global__ void k_partition_S_multi(const DevPop* __restrict__ pops) { k_partition_S_body(pops[blockIdx.y]); }

// ====================================================== IncubRecoverySweep
__device__ __forceinline__ void sev_add(const DevPop& d, int ad, int which, int delta, bool cum)
{
    bool adok = ad >= 0 && ad < CS_MAX_ADUNITS;
    switch (which) {
    case CS_SEV_MILD: cnt_add(CSB_STAGED(Mild), delta); if (cum) cnt_add(CSB_STAGED(cumMild), 1); break;
    case CS_SEV_ILI: cnt_add(CSB_STAGED(ILI), delta); if (cum) cnt_add(CSB_STAGED(cumILI), 1); break;
    case CS_SEV_SARI: cnt_add(CSB_STAGED(SARI), delta); if (cum) cnt_add(CSB_STAGED(cumSARI), 1); break;
    case CS_SEV_CRITICAL:
        cnt_add(CSB_STAGED(Critical), delta);
        if (adok) cnt_add(CSB_STAGED(Critical_adunit[ad]), delta);
        if (cum) { cnt_add(CSB_STAGED(cumCritical), 1); if (adok) cnt_add(CSB_STAGED(cumCritical_adunit[ad]), 1); }
        break;
    case CS_SEV_STEPDOWN: cnt_add(CSB_STAGED(CritRecov), delta); if (cum) cnt_add(CSB_STAGED(cumCritRecov), 1); break;
    default: break;
    }
}

// An infectious person's times that IncubRecoverySweep tests besides case onset
// (latent_time + delay), held in registers through the person's transitions.
struct PersonTimes {
    uint16_t rec, sari, crit, sd;
};

__device__ __forceinline__ PersonTimes load_times(const DevPop& d, const cs_params& P, int p)
{
    PersonTimes tm;
    tm.rec = d.recovery_time[p];
    if (P.DoSeverity) {
        tm.sari = d.sari_time[p];
        tm.crit = d.critical_time[p];
        tm.sd = d.stepdown_time[p];
    } else {
        tm.sari = tm.crit = tm.sd = 0xFFFF;
    }
    return tm;
}

// DoIncub (src/Update.cpp:408-523) for one person, on a register copy of the record;
// tm returns the person's times as written.
__device__ void do_incub(const DevPop& d, const cs_params& P, int p, PersonHot& h, int ts, uint64_t seed, PersonTimes& tm)
{
    if (P.DoSeverity) {   // the times this call leaves unset keep their values
        tm.sari = d.sari_time[p];
        tm.crit = d.critical_time[p];
        tm.sd = d.stepdown_time[p];
    } else {
        tm.sari = tm.crit = tm.sd = 0xFFFF;
    }
    int age = age_group(h);
    if (age >= CS_NUM_AGE_GROUPS) age = CS_NUM_AGE_GROUPS - 1;
    Stream s(seed, CS_RNG_INCUB, (uint32_t)ts, (uint32_t)p, 0);
    unsigned long long* err = CSB_CTR(err_spatial_tries);
    float infn = (float)P.AgeInfectiousness[age];
    if (P.InfectiousnessSD > 0) {
        double k = 1 / (P.InfectiousnessSD * P.InfectiousnessSD);
        infn *= (float)sample_gamma(s, k, k, err);
    }
    if (s.next() < P.ProportionSymptomatic[age]) {
        h.inf = CS_INF_INFECTIOUS_ALMOST_SYMPTOMATIC;
        infn *= (float)(-P.SymptInfectiousness);
    } else {
        h.inf = CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE;
        infn *= (float)P.AsymptInfectiousness;
    }
    h.infness = infn;
    double spd = P.TimeStepsPerDay;
    if (!P.DoSeverity || h.inf == CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE) {
        if (P.DoInfectiousnessProfile)
            d.recovery_time[p] = tm.rec = (uint16_t)(h.latent_time + (uint16_t)(P.InfectiousPeriod * spd));
        else
            d.recovery_time[p] = tm.rec = (uint16_t)(h.latent_time + icdf_choose(P.infectious_icdf, P.InfectiousPeriod, s.next(), spd));
    } else {
        int CaseTime = h.latent_time + ((int)(P.LatentToSymptDelay / P.ModelTimeStep));
        double x = s.next();
        int fin;
        if (x < P.Prop_ILI_ByAge[age]) fin = CS_SEV_ILI;
        else if (x < P.Prop_ILI_ByAge[age] + P.Prop_SARI_ByAge[age]) fin = CS_SEV_SARI;
        else if (x < P.Prop_ILI_ByAge[age] + P.Prop_SARI_ByAge[age] + P.Prop_Critical_ByAge[age]) fin = CS_SEV_CRITICAL;
        else fin = CS_SEV_MILD;
        bool to_die = false;
        if (fin == CS_SEV_CRITICAL) { if (s.next() < (P.CFR_Critical_ByAge[age] * P.CFR_Critical_Scale_Current)) to_die = true; }
        else if (fin == CS_SEV_SARI) { if (s.next() < (P.CFR_SARI_ByAge[age] * P.CFR_SARI_Scale_Current)) to_die = true; }
        else if (fin == CS_SEV_ILI) { if (s.next() < (P.CFR_ILI_ByAge[age] * P.CFR_ILI_Scale_Current)) to_die = true; }
        if (is_ch(h) && ((fin == CS_SEV_CRITICAL) || (fin == CS_SEV_SARI)) && (s.next() > P.CareHomeRelProbHosp)) {
            to_die = true;
            fin = CS_SEV_ILI;
        }
        h.sev = (uint8_t)((h.sev & 0x0f) | (fin << 4));
        if (to_die) h.dflags |= CS_DF_TO_DIE;
        uint16_t rec;
        if (fin == CS_SEV_MILD)
            rec = (uint16_t)(CaseTime + icdf_choose(P.MildToRecovery_icdf, P.Mean_MildToRecovery[age], s.next(), spd));
        else if (fin == CS_SEV_CRITICAL) {
            uint16_t sari = (uint16_t)(CaseTime + icdf_choose(P.ILIToSARI_icdf, P.Mean_ILIToSARI[age], s.next(), spd));
            uint16_t crit = (uint16_t)(sari + icdf_choose(P.SARIToCritical_icdf, P.Mean_SARIToCritical[age], s.next(), spd));
            d.sari_time[p] = tm.sari = sari;
            d.critical_time[p] = tm.crit = crit;
            if (to_die) {
                if (P.IncludeStepDownToDeath == 1) {
                    uint16_t sd = (uint16_t)(crit + icdf_choose(P.CriticalToCritRecov_icdf, P.Mean_CriticalToCritRecov[age], s.next(), spd));
                    d.stepdown_time[p] = tm.sd = sd;
                    rec = (uint16_t)(sd + icdf_choose(P.StepdownToDeath_icdf, P.Mean_StepdownToDeath[age], s.next(), spd));
                } else
                    rec = (uint16_t)(crit + icdf_choose(P.CriticalToDeath_icdf, P.Mean_CriticalToDeath[age], s.next(), spd));
            } else {
                uint16_t sd = (uint16_t)(crit + icdf_choose(P.CriticalToCritRecov_icdf, P.Mean_CriticalToCritRecov[age], s.next(), spd));
                d.stepdown_time[p] = tm.sd = sd;
                rec = (uint16_t)(sd + icdf_choose(P.CritRecovToRecov_icdf, P.Mean_CritRecovToRecov[age], s.next(), spd));
            }
        } else if (fin == CS_SEV_SARI) {
            uint16_t sari = (uint16_t)(CaseTime + icdf_choose(P.ILIToSARI_icdf, P.Mean_ILIToSARI[age], s.next(), spd));
            d.sari_time[p] = tm.sari = sari;
            if (to_die) rec = (uint16_t)(sari + icdf_choose(P.SARIToDeath_icdf, P.Mean_SARIToDeath[age], s.next(), spd));
            else rec = (uint16_t)(sari + icdf_choose(P.SARIToRecovery_icdf, P.Mean_SARIToRecovery[age], s.next(), spd));
        } else {
            if (to_die) rec = (uint16_t)(CaseTime + icdf_choose(P.ILIToDeath_icdf, P.Mean_ILIToDeath[age], s.next(), spd));
            else rec = (uint16_t)(CaseTime + icdf_choose(P.ILIToRecovery_icdf, P.Mean_ILIToRecovery[age], s.next(), spd));
        }
        d.recovery_time[p] = tm.rec = rec;
    }
    if (h.inf == CS_INF_INFECTIOUS_ALMOST_SYMPTOMATIC && ((P.ControlPropCasesId == 1) || (s.next() < P.ControlPropCasesId))) {
        h.dflags |= CS_DF_DETECTED;
        d.detected_time[p] = (uint16_t)(ts + (uint16_t)(P.LatentToSymptDelay * spd));
    }
}

// DoDetectedCase (src/Update.cpp:525-792): case isolation now, household
// quarantine deferred to the per-household pass.
__device__ void do_detected_case(const DevPop& d, const cs_params& P, const DevIv& iv, int p, PersonHot& h, double t, int ts,
                                 uint64_t seed)
{
    int ad = d.mcell_adunit[h.mcell];
    if (ad >= 0 && ad < CS_MAX_ADUNITS) cnt_add(CSB_STAGED(cumDC_adunit[ad]), 1);
    const int aw = (ad >= 0 && ad < d.NA) ? ad : 0;   // the person's admin unit's windows
    const double hq0 = iv.hq_start[aw], ci0 = iv.ci_start[aw];
    if (P.DoHouseholds && t >= hq0 && t < hq0 + iv.hq_dur) flag_household(d, h.hh, 4);
    if (t >= ci0 && t < ci0 + iv.ci_dur) {
        Stream s(seed, CS_RNG_DETECTED, (uint32_t)ts, (uint32_t)p, 0);
        if ((P.CaseIsolationProp == 1) || (s.next() < P.CaseIsolationProp)) {
            h.isolation_start = (uint16_t)ts;
            if (host_absent(h, ts)) {
                if (h.absent_stop < ts + P.usCaseAbsenteeismDelay + P.usCaseIsolationDuration)
                    h.absent_stop = (uint16_t)(ts + P.usCaseAbsenteeismDelay + P.usCaseIsolationDuration);
            } else if (P.DoRealSymptWithdrawal) {
                h.absent_start = (uint16_t)(ts + P.usCaseIsolationDelay);
                h.absent_stop = (uint16_t)(ts + P.usCaseIsolationDelay + P.usCaseIsolationDuration);
                if (P.DoPlaces && !host_quarantined(h, P, ts) && link_of(d, P.PlaceTypeNoAirNum - 1, p) >= 0 && h.age >= P.CaseAbsentChildAgeCutoff)
                    cnt_add(CSB_STAGED(cumAC), 1);
                if (P.DoHouseholds && P.DoPlaces && h.age < P.CaseAbsentChildAgeCutoff) {
                    if (!host_quarantined(h, P, ts)) cnt_add(CSB_STAGED(cumACS), 1);
                    if (d.prob_care[p] < P.CaseAbsentChildPropAdultCarers) flag_household(d, h.hh, 2);
                }
            }
        }
    }
}

// DoCase (src/Update.cpp:794-894).
__device__ void do_case(const DevPop& d, const cs_params& P, const DevIv& iv, int p, PersonHot& h, double t, int ts, uint64_t seed)
{
    int age = age_group(h);
    if (age >= CS_NUM_AGE_GROUPS) age = CS_NUM_AGE_GROUPS - 1;
    if (h.inf != CS_INF_INFECTIOUS_ALMOST_SYMPTOMATIC) return;
    h.inf = CS_INF_CASE;
    if (host_absent(h, ts)) {
        if (h.absent_stop < ts + P.usCaseAbsenteeismDelay + P.usCaseAbsenteeismDuration)
            h.absent_stop = (uint16_t)(ts + P.usCaseAbsenteeismDelay + P.usCaseAbsenteeismDuration);
    } else if ((P.DoRealSymptWithdrawal) && (P.DoPlaces)) {
        Stream s(seed, CS_RNG_CASE, (uint32_t)ts, (uint32_t)p, 0);
        h.absent_start = kNever;
        for (int j = 0; j < d.NPT; j++)
            if ((link_of(d, j, p) >= 0) && (j != P.HotelPlaceType) && (!host_absent(h, ts)) && (P.SymptPlaceTypeWithdrawalProp[j] > 0)) {
                if ((!is_ch(h)) && ((P.SymptPlaceTypeWithdrawalProp[j] == 1) || (s.next() < P.SymptPlaceTypeWithdrawalProp[j]))) {
                    h.absent_start = (uint16_t)(ts + P.usCaseAbsenteeismDelay);
                    h.absent_stop = (uint16_t)(ts + P.usCaseAbsenteeismDelay + P.usCaseAbsenteeismDuration);
                    if ((!host_quarantined(h, P, ts)) && (link_of(d, P.PlaceTypeNoAirNum - 1, p) >= 0) && (h.age >= P.CaseAbsentChildAgeCutoff))
                        cnt_add(CSB_STAGED(cumAC), 1);
                    if ((P.DoHouseholds) && (h.age < P.CaseAbsentChildAgeCutoff)) {
                        if (!host_quarantined(h, P, ts)) cnt_add(CSB_STAGED(cumACS), 1);
                        if (d.prob_care[p] < P.CaseAbsentChildPropAdultCarers) flag_household(d, h.hh, 1);
                    }
                }
            }
    }
    if (h.dflags & CS_DF_DETECTED) {
        cnt_add(CSB_STAGED(cumDC), 1);
        do_detected_case(d, P, iv, p, h, t, ts, seed);
    }
    cnt_add(CSB_STAGED(cumC), 1);
    cnt_add(CSB_STAGED(cumCa[age]), 1);
    cnt_add(CSB_STAGED(cumC_keyworker[(h.pflags & CS_PF_KEYWORKER) ? 1 : 0]), 1);
    int ad = d.mcell_adunit[h.mcell];
    if (ad >= 0 && ad < CS_MAX_ADUNITS) cnt_add(CSB_STAGED(cumC_adunit[ad]), 1);
    if (P.DoSeverity) {
        int cur = h.sev & 0x0f, fin = h.sev >> 4;
        if (cur == CS_SEV_ASYMPTOMATIC) {
            int to = (fin == CS_SEV_MILD) ? CS_SEV_MILD : CS_SEV_ILI;
            h.sev = (uint8_t)((h.sev & 0xf0) | to);
            sev_add(d, ad, to, 1, true);
        }
    }
}

// The infectious-person body of IncubRecoverySweep (src/Sweep.cpp:929-977).
// Returns bit 0 when the person leaves the infectious block this step and bit 1
// when any event fired (the record must be written back).
__device__ int infectious_events(const DevPop& d, const cs_params& P, const DevIv& iv, int p, PersonHot& h, int cell,
                                 double t, int ts, uint64_t seed, const PersonTimes& tm)
{
    int CaseTime = h.latent_time + ((int)(P.LatentToSymptDelay / P.ModelTimeStep));
    const uint16_t rec = tm.rec;
    bool any = (ts == (uint16_t)CaseTime) || (ts == rec) ||
               (P.DoSeverity && (ts == tm.sari || ts == tm.crit || ts == tm.sd));
    if (!any) return 0;
    if (P.DoSymptoms && ts == (uint16_t)CaseTime) do_case(d, P, iv, p, h, t, ts, seed);
    bool to_die = (h.dflags & CS_DF_TO_DIE) != 0;
    int ad = d.mcell_adunit[h.mcell];
    if (P.DoSeverity) {
        int cur = h.sev & 0x0f;
        if (ts == tm.sari && cur == CS_SEV_ILI) { cur = CS_SEV_SARI; sev_add(d, ad, CS_SEV_ILI, -1, false); sev_add(d, ad, CS_SEV_SARI, 1, true); }
        if (ts == tm.crit && cur == CS_SEV_SARI) { cur = CS_SEV_CRITICAL; sev_add(d, ad, CS_SEV_SARI, -1, false); sev_add(d, ad, CS_SEV_CRITICAL, 1, true); }
        if (ts == tm.sd && cur == CS_SEV_CRITICAL && !to_die) { cur = CS_SEV_STEPDOWN; sev_add(d, ad, CS_SEV_CRITICAL, -1, false); sev_add(d, ad, CS_SEV_STEPDOWN, 1, true); }
        if (ts == rec) {
            if (to_die) {
                if (cur == CS_SEV_CRITICAL) { sev_add(d, ad, CS_SEV_CRITICAL, -1, false); cnt_add(CSB_STAGED(cumDeath_Critical), 1); cur = CS_SEV_DEAD; }
                else if (cur == CS_SEV_SARI) { sev_add(d, ad, CS_SEV_SARI, -1, false); cnt_add(CSB_STAGED(cumDeath_SARI), 1); cur = CS_SEV_DEAD; }
                else if (cur == CS_SEV_ILI) { sev_add(d, ad, CS_SEV_ILI, -1, false); cnt_add(CSB_STAGED(cumDeath_ILI), 1); cur = CS_SEV_DEAD; }
            } else if (h.inf == CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE || h.inf == CS_INF_CASE) {
                if (cur == CS_SEV_MILD) { sev_add(d, ad, CS_SEV_MILD, -1, false); cur = CS_SEV_RECOVERED; }
                else if (cur == CS_SEV_ILI) { sev_add(d, ad, CS_SEV_ILI, -1, false); cur = CS_SEV_RECOVERED; }
                else if (cur == CS_SEV_SARI) { sev_add(d, ad, CS_SEV_SARI, -1, false); cur = CS_SEV_RECOVERED; }
                else if (cur == CS_SEV_STEPDOWN) { sev_add(d, ad, CS_SEV_STEPDOWN, -1, false); cur = CS_SEV_RECOVERED; }
            }
        }
        h.sev = (uint8_t)((h.sev & 0xf0) | cur);
    }
    if (ts == rec && (h.inf == CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE || h.inf == CS_INF_CASE)) {
        atomicSub(d.I + cell, 1);
        cnt_add(CSB_STAGED(work_transitions), 1);
        if (!to_die) {
            h.inf = (h.inf == CS_INF_CASE) ? CS_INF_RECOVERED_FROM_SYMP : CS_INF_RECOVERED_FROM_ASYMP;
            atomicAdd(d.R + cell, 1);
            cnt_add(CSB_STAGED(cumR), 1);
        } else {
            h.inf = (h.inf == CS_INF_CASE) ? CS_INF_DEAD_WAS_SYMP : CS_INF_DEAD_WAS_ASYMP;
            atomicAdd(d.D + cell, 1);
            cnt_add(CSB_STAGED(cumD), 1);
            cnt_add(CSB_STAGED(cumDa[age_group(h)]), 1);
            if (ad >= 0 && ad < CS_MAX_ADUNITS) cnt_add(CSB_STAGED(cumD_adunit[ad]), 1);
        }
        return 3;
    }
    return 2;
}

// An infectious person's next transition time after (strict) or from step ts: the
// least of the times infectious_events tests that is above (or at) ts, 0xFFFF when
// none is.  The times are compared as IncubRecoverySweep compares them, 16-bit.
__device__ __forceinline__ uint16_t next_infectious_time(const cs_params& P, uint16_t latent_time, const PersonTimes& tm,
                                                         int ts, bool strict)
{
    const int lo = strict ? ts + 1 : ts;
    const int delay = (int)(P.LatentToSymptDelay / P.ModelTimeStep);
    int best = 0xFFFF;
    auto take = [&](int x) { if (x >= lo && x < best) best = x; };
    take((uint16_t)(latent_time + delay));
    take(tm.rec);
    if (P.DoSeverity) {
        take(tm.sari);
        take(tm.crit);
        take(tm.sd);
    }
    return (uint16_t)best;
}

// The gather's test from the person's own times, forming next_ev on the way (the
// first gather after an upload or reset); kept out of line, off the common path.
// (The arrays come as pointers: a DevPop passed by reference to an out-of-line
// function would be copied to every thread's stack.)
__device__ __noinline__ bool gather_test_from_times(const cs_params* __restrict__ P, const PersonHot* hot,
                                                    const uint16_t* const* times, uint16_t* next_ev, int p, int ts)
{
    const int delay = (int)(P->LatentToSymptDelay / P->ModelTimeStep);
    const PersonHot h = hot[p];
    if (h.inf == CS_INF_LATENT) {
        next_ev[p] = h.latent_time;
        return h.latent_time == ts;
    }
    // times: recovery, SARI, critical, stepdown
    const int v[5] = {(uint16_t)(h.latent_time + delay), times[0][p], P->DoSeverity ? times[1][p] : 0xFFFF,
                      P->DoSeverity ? times[2][p] : 0xFFFF, P->DoSeverity ? times[3][p] : 0xFFFF};
    int best = 0xFFFF;
    bool ev = false;
    for (int k = 0; k < 5; k++) {
        if (k >= 2 && !P->DoSeverity) break;
        if (v[k] == ts) ev = true;
        if (v[k] >= ts && v[k] < best) best = v[k];
    }
    next_ev[p] = (uint16_t)best;
    return ev;
}

// Which latent / infectious people have an event this step (latent period ends,
// case onset, severity change, recovery or death): a light scan that compacts
// them so the heavy transition kernel runs only on those.
// IncubRecoverySweep's scan (src/Sweep.cpp:920-977) over the cells' lists: every
// latent and infectious person (slots [S, S+L+I) of each cell, read block-
// cooperatively as k_build_active reads a cell's slots, so a dense cell costs no more
// than its share of the block) joins the step's event list when one of its times is
// now.  The cells come in tiles of blockDim.x; Q = gridDim.x / tiles blocks share a
// tile, block q taking its chunks q, q + Q, ... of blockDim.x entries, so the launch
// has the parallelism of a flat list without building one.  The lists hold (person,
// cell) in act / act_cell, latent people from the front and infectious people from
// the back, in no particular order within each: k_incub_events treats each person on
// its own.
__device__ __forceinline__ void k_incub_gather_body(const DevPop& d)
{
    const int ts = d.step->ts;
    const bool init = *d.ev_init != 0;   // next_ev is formed from the people's own times
    __shared__ int s_first[kThreads], s_ofs[kThreads], s_n[kThreads], s_L[kThreads];
    long long people = 0;
    const int ntiles = (d.NC + blockDim.x - 1) / blockDim.x;
    const int Q = max(1, (int)gridDim.x / ntiles), part = blockIdx.x % Q;
    for (int tile = blockIdx.x / Q; tile < ntiles; tile += max(1, (int)gridDim.x / Q)) {
        const int c0 = tile * blockDim.x;
        const int c = c0 + threadIdx.x;
        int first = 0, n = 0, nl = 0;
        if (c < d.NC) {
            first = d.cell_start[c] + d.S[c];
            nl = d.L[c];
            n = nl + d.I[c];
        }
        const int o = block_reserve2(nullptr, n, nullptr, 0).x;   // the block's own prefix of n
        s_first[threadIdx.x] = first;
        s_ofs[threadIdx.x] = o;
        s_n[threadIdx.x] = n;
        s_L[threadIdx.x] = nl;
        __syncthreads();
        const int total = s_ofs[blockDim.x - 1] + s_n[blockDim.x - 1];
        if (threadIdx.x == 0 && part == 0) people += total;
        for (int j0 = part * blockDim.x; j0 < total; j0 += Q * blockDim.x) {   // block-uniform: every thread reserves
            const int j = j0 + (int)threadIdx.x;
            bool ev = false, latent = false;
            int p = 0, cell = 0;
            if (j < total) {
                int lo = 0, hi = blockDim.x - 1;   // the last cell whose entries start at or before j
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (s_ofs[mid] <= j) lo = mid; else hi = mid - 1;
                }
                latent = j - s_ofs[lo] < s_L[lo];   // the cell's slots run latent, then infectious
                p = d.slots[s_first[lo] + (j - s_ofs[lo])];
                cell = c0 + lo;
                if (init) {
                    const uint16_t* times[4] = {d.recovery_time, d.sari_time, d.critical_time, d.stepdown_time};
                    ev = gather_test_from_times(d.P, d.hot, times, d.next_ev, p, ts);
                } else {
                    ev = d.next_ev[p] == ts;
                }
            }
            const int2 e = block_reserve2(d.counts + kCntEvents, (ev && latent) ? 1 : 0, d.counts + kCntEventsInf,
                                          (ev && !latent) ? 1 : 0);
            if (ev) {
                const int at = latent ? e.x : d.N - 1 - e.y;
                d.act[at] = p;
                d.act_cell[at] = cell;
            }
        }
        __syncthreads();   // the shared arrays are refilled for the next cells
    }
    if (threadIdx.x == 0 && people) cnt_add(CSB_CTR(work_incub_people), people);
}
__global__ void __launch_bounds__(kThreads) k_incub_gather(DevPop d) { k_incub_gather_body(d); }
__global__ void __launch_bounds__(kThreads) k_incub_gather_multi(const DevPop* __restrict__ pops) { k_incub_gather_body(pops[blockIdx.y]); }

// DoFalseCase (src/Update.cpp:896-905) for every person with a false-positive
// entry this step, after the step's infections: detected with probability
// ControlPropCasesId (counted once the detected cases at the last sample reached
// the alert threshold) and then treated as a detected case; every false case is
// counted.  A person the step did not infect takes the false entry's labels
// (infector and infection type -1, as the reference's queue drain writes them,
// src/Sweep.cpp:866-869); an infected one keeps the infection's.
__device__ __forceinline__ void k_apply_false_cases_body(const DevPop& d)
{
    const cs_params& P = *d.P;
    const double t = d.step->t;
    const int ts = d.step->ts;
    const uint64_t seed = d.step->seed;
    const DevIv iv = *d.iv;
    const int n = d.counts[kCntFalse];
    if (blockIdx.x * blockDim.x >= n) return;
    stage_begin(d.C, false);
    long long nfc = 0, ndc = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int p = d.fc_queue[q];
        d.fc_flag[p >> 5] = 0;   // every flagged person of the word is in the queue
        PersonHot h = d.hot[p];
        if (h.inf == CS_INF_SUSCEPTIBLE) {
            d.infector[p] = -1;
            d.infect_type[p] = -1;
        }
        Stream s(seed, CS_RNG_FALSE_CASE, (uint32_t)ts, (uint32_t)p, 0);
        if ((P.ControlPropCasesId == 1) || (s.next() < P.ControlPropCasesId)) {
            if (P.cumDC_at_sample >= P.CaseOrDeathThresholdBeforeAlert) ndc++;
            do_detected_case(d, P, iv, p, h, t, ts, seed);
            d.hot[p] = h;
        }
        nfc++;
    }
    cnt_add_warp(CSB_CTR(cumFC), nfc);
    cnt_add_warp(CSB_CTR(cumDC), ndc);
    stage_flush(d.C, false);
}
__global__ void k_apply_false_cases(DevPop d) { k_apply_false_cases_body(d); }
__global__ void k_apply_false_cases_multi(const DevPop* __restrict__ pops) { k_apply_false_cases_body(pops[blockIdx.y]); }

// cnt[c] low 16 bits: L -> I moves of cell c; high 16 bits: I -> R/D moves.
__device__ __forceinline__ void k_incub_events_body(const DevPop& d)
{
    const cs_params& P = *d.P;
    const double t = d.step->t;
    const int ts = d.step->ts;
    const uint64_t seed = d.step->seed;
    const DevIv iv = *d.iv;
    const int nlat = d.counts[kCntEvents], nev = nlat + d.counts[kCntEventsInf];
    if (blockIdx.x == 0 && threadIdx.x == 0) *d.ev_init = 0;   // the gather before this formed next_ev
    if (blockIdx.x * blockDim.x >= nev) return;   // a block without work stages nothing
    const bool staged = nev >= kStageMinItems;
    stage_begin(d.C, staged);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nev; e += gridDim.x * blockDim.x) {
        const int at = e < nlat ? e : d.N - 1 - (e - nlat);   // latent events, then infectious ones
        const int p = d.act[at], c = d.act_cell[at];
        PersonHot h = d.hot[p];
        int pos = d.cell_start[c] + d.listpos[p];
        if (h.inf == CS_INF_LATENT) {
            if (h.latent_time != ts) continue;
            PersonTimes tm;
            do_incub(d, P, p, h, ts, seed, tm);
            atomicSub(d.L + c, 1);
            atomicAdd(d.I + c, 1);
            int add = 1;
            d.mark[pos] = 1;
            cnt_add(CSB_STAGED(work_transitions), 1);
            if (infectious_events(d, P, iv, p, h, c, t, ts, seed, tm) & 1) {
                d.pstep[p] = kStepItoRD;
                add += 1 << 16;
                d.next_ev[p] = 0xFFFF;
            } else {
                d.next_ev[p] = next_infectious_time(P, h.latent_time, tm, ts, true);
            }
            d.hot[p] = h;
            atomicAdd(d.cnt + c, add);
            mark_cell(d, c);
        } else {
            const PersonTimes tm = load_times(d, P, p);
            int r = infectious_events(d, P, iv, p, h, c, t, ts, seed, tm);
            if (r & 2) d.hot[p] = h;
            if (r & 1) {
                d.mark[pos] = 2;
                atomicAdd(d.cnt + c, 1 << 16);
                mark_cell(d, c);
                d.next_ev[p] = 0xFFFF;
            } else {
                d.next_ev[p] = next_infectious_time(P, h.latent_time, tm, ts, true);
            }
        }
    }
    stage_flush(d.C, staged);
}
__global__ void __launch_bounds__(kThreads, 3) k_incub_events(DevPop d) { k_incub_events_body(d); }
__global__ void __launch_bounds__(kThreads, 3) k_incub_events_multi(const DevPop* __restrict__ pops) { k_incub_events_body(pops[blockIdx.y]); }

__device__ __forceinline__ void k_partition_LI_body(const DevPop& d)
{
    int nt = d.counts[kCntTouched];
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < nt; k += warps) {
        int c = d.touched[k];
        int v = d.cnt[c];
        int nLI = v & 0xffff, nIR = (v >> 16) & 0xffff;
        int base = d.cell_start[c];
        int S = d.S[c], L = d.L[c], I = d.I[c];
        if (nLI) partition_block_warp(d, base, base + S, L + nLI, nLI, 1, true);
        if (nIR) partition_block_warp(d, base, base + S + L, I + nIR, nIR, 2, false);
        if ((threadIdx.x & 31) == 0) {
            d.cnt[c] = 0;
            d.cell_flag[c] = 0;
        }
    }
}
__global__ void k_partition_LI(DevPop d) { k_partition_LI_body(d); }
__global__ void k_partition_LI_multi(const DevPop* __restrict__ pops) { k_partition_LI_body(pops[blockIdx.y]); }

// Deferred household actions, once per household, after every per-person
// transition of the step: the adult-carer absence of DoCase/DoDetectedCase
// (src/Update.cpp:736-763, 843-868) and household quarantine (src/Update.cpp:676-708).
__device__ __forceinline__ void k_household_after_body(const DevPop& d)
{
    const cs_params& P = *d.P;
    const int ts = d.step->ts;
    const uint64_t seed = d.step->seed;
    // the step's transition flags are only set on event people: clear them
    const int nlat = d.counts[kCntEvents], nev = nlat + d.counts[kCntEventsInf];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nev; e += gridDim.x * blockDim.x)
        d.pstep[d.act[e < nlat ? e : d.N - 1 - (e - nlat)]] = 0;
    int nh = d.counts[kCntHH];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nh; k += gridDim.x * blockDim.x) {
        int h = d.hh_list[k];
        uint8_t f = d.hh_flag[h];
        d.hh_flag[h] = 0;
        const HouseholdRec hr = load_household(d, h);
        int j1 = hr.first, j2 = j1 + hr.nh;
        if (f & 3) {
            int wp = P.PlaceTypeNoAirNum - 1;
            bool ok = false;
            for (int j = j1; (j < j2) && (!ok); j++) {
                PersonHot hj = d.hot[j];
                ok = (is_alive(hj.inf) && (hj.age >= P.CaseAbsentChildAgeCutoff) &&
                      ((link_of(d, wp, j) < 0) || host_absent(hj, ts) || host_quarantined(hj, P, ts)));
            }
            if (!ok) {
                int kk = -1;
                for (int j = j1; j < j2; j++) {
                    PersonHot hj = d.hot[j];
                    if ((hj.age >= P.CaseAbsentChildAgeCutoff) && is_alive(hj.inf)) { kk = j; break; }
                }
                if (kk >= 0) {
                    PersonHot hk = d.hot[kk];
                    if ((f & 2) || !host_absent(hk, ts)) d.hot[kk].absent_start = (uint16_t)(ts + P.usCaseIsolationDelay);
                    d.hot[kk].absent_stop = (uint16_t)(ts + P.usCaseIsolationDelay + P.usCaseIsolationDuration);
                    cnt_add(CSB_CTR(cumAA), 1);
                }
            }
        }
        if (f & 4) {
            if (host_to_be_quarantined(d.hot[j1], P, ts) && !P.DoHQretrigger) continue;
            Stream s(seed, CS_RNG_HQ, (uint32_t)ts, (uint32_t)h, 0);
            uint16_t qs = (uint16_t)(ts + ((uint16_t)(P.TimeStepsPerDay * P.HQuarantineDelay)));
            int kc = (s.next() < P.HQuarantinePropHouseCompliant) ? 1 : 0;
            if (kc) cnt_add(CSB_CTR(cumHQ), 1);
            for (int j = j1; j < j2; j++) {
                int comply = (kc == 0) ? 0 : ((s.next() < P.HQuarantinePropIndivCompliant) ? 1 : 0);
                PersonHot hj = d.hot[j];
                hj.quar_start = qs;
                hj.dflags = (uint8_t)((hj.dflags & ~CS_DF_QUAR_COMPLY_MASK) | (comply << CS_DF_QUAR_COMPLY_SHIFT));
                d.hot[j] = hj;
            }
        }
    }
}
__global__ void k_household_after(DevPop d) { k_household_after_body(d); }
__global__ void k_household_after_multi(const DevPop* __restrict__ pops) { k_household_after_body(pops[blockIdx.y]); }

// The cell-list moves and the household actions in one launch: the moves touch the
// cells' slots and list positions, the household actions people's absences and
// quarantine, flags and household lists, so neither waits for the other.
__global__ void k_incub_finish(DevPop d)
{
    k_partition_LI_body(d);
    k_household_after_body(d);
}
__global__ void k_incub_finish_multi(const DevPop* __restrict__ pops)
{
    k_partition_LI_body(pops[blockIdx.y]);
    k_household_after_body(pops[blockIdx.y]);
}

// ============================================================ seeding
__global__ void k_seed_claims(DevPop d, const int32_t* list, int n)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int p = list[k];
        if (p < 0 || p >= d.N) continue;
        if (d.hot[p].inf != CS_INF_SUSCEPTIBLE) continue;
        unsigned long long key = ((unsigned long long)(uint32_t)(-2) << 8) | (unsigned long long)(CS_INFECT_TYPE_MASK - 1);
        if (atomicCAS(d.claim + p, ~0ull, key) == ~0ull) d.queue[append(d.counts + kCntQueue)] = p;
        // radii are measured from the last seed's household (src/CovidSim.cpp:1358-1359)
        if (k == n - 1) {
            const HouseholdRec hr = load_household(d, d.hot[p].hh);
            d.rad_origin[0] = (double)hr.x;
            d.rad_origin[1] = (double)hr.y;
        }
    }
}

// ============================================================ interventions
// No intervention windows: every admin unit's start times at 1e10, durations 0.
__global__ void k_iv_reset(DevIv* iv, int na)
{
    for (int a = threadIdx.x; a < na; a += blockDim.x) iv->ci_start[a] = iv->hq_start[a] = 1e10;
    if (threadIdx.x == 0) iv->ci_dur = iv->hq_dur = 0.0;
}

// State of the device-side run loop (cs_gpu_run): its policy, the host loop's
// variables between timesteps (src/CovidSim.cpp:1517-1526 PreviousProportionSusceptible,
// the ICU trigger's switch state) and what the day's logic decided for the
// kernels gated on it.
struct DayCtl {
    cs_run_policy pol;
    cs_counters* series;        // [days] counters at each day's end
    double prev_prop_s, on_until;
    int32_t day, started;
    int32_t update;             // UpdateProbs runs (gate of its kernels)
    int32_t socd_write;         // every microcell's social-distancing flag becomes socd_value
    int32_t close;              // places of the policy's types close over [close_start, close_stop)
    uint16_t close_start, close_stop;   // per admin unit: the envelope of the units' windows
    uint8_t socd_value, pad[3];
    // per admin unit triggers (pol.per_adunit)
    int32_t a_started[CS_MAX_ADUNITS];
    double a_on_until[CS_MAX_ADUNITS];
    int8_t a_switch[CS_MAX_ADUNITS];    // this day: -1 none, 1 on, 0 off
    uint16_t a_close_start[CS_MAX_ADUNITS], a_close_stop[CS_MAX_ADUNITS];
};

// ------------------------------------------------------------ place closure
// Is a living adult at home already (no workplace link, or quarantined)?  The test
// DoPlaceClose and DoPlaceOpen make before sending an adult home with a child
// (src/Update.cpp:1211-1215, 1278-1281).  It reads no absence times, so the
// closures of one call may run in any order.
__device__ bool adult_home_for_child(const DevPop& d, const cs_params& P, int hh, int ts)
{
    const HouseholdRec r = d.hhr[hh];
    const int wp = P.PlaceTypeNoAirNum - 1;
    for (int j = r.first; j < r.first + r.nh; j++) {
        const PersonHot m = d.hot[j];
        if (is_alive(m.inf) && m.age >= P.CaseAbsentChildAgeCutoff &&
            (wp < 0 || link_of(d, wp, j) < 0 || host_quarantined(m, P, ts)))
            return true;
    }
    return false;
}

// Queue household hh for an adult carer over [ws, we): the host closure queue of
// DoPlaceClose (src/Update.cpp:1218-1231).  Windows of several closures merge as
// UpdateHostClosure's min/max does; the household is listed once.
__device__ void flag_carer(const DevPop& d, int hh, uint16_t ws, uint16_t we)
{
    if (ws >= we) return;
    uint32_t* w = d.carer_win + hh;
    const uint32_t add = ((uint32_t)(0xFFFFu - ws) << 16) | we;
    uint32_t old = *w, assumed;
    bool first = false;
    do {
        assumed = old;
        const uint32_t nv = max(assumed & 0xFFFF0000u, add & 0xFFFF0000u) | max(assumed & 0xFFFFu, add & 0xFFFFu);
        if (nv == assumed) break;
        old = atomicCAS(w, assumed, nv);
        first = (old == assumed) && assumed == 0u;
    } while (old != assumed);
    if (first) d.carer_list[append(d.counts + kCntCarer)] = hh;
}

// UpdateHostClosure (src/Update.cpp:1243-1258) for the households flag_carer
// listed: the first living adult's absence covers the window.
__device__ __forceinline__ void k_carer_pass_body(const DevPop& d)
{
    const cs_params& P = *d.P;
    const int n = d.counts[kCntCarer];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int hh = d.carer_list[k];
        const uint32_t win = d.carer_win[hh];
        d.carer_win[hh] = 0u;
        const uint16_t ws = (uint16_t)(0xFFFFu - (win >> 16)), we = (uint16_t)(win & 0xFFFFu);
        const HouseholdRec r = d.hhr[hh];
        for (int j = r.first; j < r.first + r.nh; j++) {
            PersonHot* m = d.hot + j;
            if (m->age >= P.CaseAbsentChildAgeCutoff && is_alive(m->inf)) {
                if (m->absent_start > ws) m->absent_start = ws;
                if (m->absent_stop < we) m->absent_stop = we;
                break;
            }
        }
    }
}
__global__ void k_carer_pass(DevPop d) { k_carer_pass_body(d); }
__global__ void k_carer_pass_multi(const DevPop* __restrict__ pops) { k_carer_pass_body(pops[blockIdx.y]); }
__global__ void k_carer_reset(DevPop d) { d.counts[kCntCarer] = 0; }
__global__ void k_carer_reset_multi(const DevPop* __restrict__ pops) { pops[blockIdx.x].counts[kCntCarer] = 0; }

// DoPlaceClose's loop over the members of a place that closed (src/Update.cpp:
// 1196-1240) at timestep ts with absence window [ws, we), one block per place.  A
// person is a member of one place per type, so the blocks of one launch (one place
// type) write disjoint people; carers are only queued here.
__device__ void close_place_members(const DevPop& d, const cs_params& P, int pt, int l, int ts, uint16_t ws, uint16_t we)
{
    const DevPlaces& pl = d.pl[pt];
    const double att = P.PlaceClosePropAttending[pt];
    for (int k = pl.member_ofs[l] + threadIdx.x; k < pl.member_ofs[l + 1]; k += blockDim.x) {
        const int w = pl.members[k];
        if (!((att == 0) || (d.prob_absent[w] >= att))) continue;
        PersonHot* hw = d.hot + w;
        const PersonHot h = *hw;
        if (!host_absent(h, ts) && !host_quarantined(h, P, ts) && h.age < P.CaseAbsentChildAgeCutoff &&
            d.prob_care[w] < P.CaseAbsentChildPropAdultCarers && !adult_home_for_child(d, P, h.hh, ts))
            flag_carer(d, h.hh, ws, we);
        if (h.absent_start > ws) hw->absent_start = ws;
        if (h.absent_stop < we) hw->absent_stop = we;
    }
}

// DoPlaceOpen (src/Update.cpp:1260-1294) for place l of type pt, whose closure
// ends at ce > ts: absences that ended with the closure end at ts, also those of
// adults who stayed home with a child of the place.
__device__ void open_place_members(const DevPop& d, const cs_params& P, int pt, int l, int ts, uint16_t ce)
{
    const DevPlaces& pl = d.pl[pt];
    for (int k = pl.member_ofs[l] + threadIdx.x; k < pl.member_ofs[l + 1]; k += blockDim.x) {
        const int ai = pl.members[k];
        PersonHot* ha = d.hot + ai;
        if (ha->absent_stop == ce) ha->absent_stop = (uint16_t)ts;
        if (!(d.prob_care[ai] < P.CaseAbsentChildPropAdultCarers)) continue;
        const PersonHot h = *ha;
        if (h.age >= P.CaseAbsentChildAgeCutoff || host_quarantined(h, P, ts) || adult_home_for_child(d, P, h.hh, ts)) continue;
        const HouseholdRec r = d.hhr[h.hh];
        for (int j = r.first; j < r.first + r.nh; j++) {
            PersonHot* m = d.hot + j;
            const PersonHot mh = *m;
            if (mh.age >= P.CaseAbsentChildAgeCutoff && is_alive(mh.inf) && host_absent(mh, ts) && mh.absent_stop == ce)
                m->absent_stop = (uint16_t)ts;
        }
    }
}

__device__ void k_close_places_body(const DevPop& d, int pt, const uint8_t* sel, uint16_t start, uint16_t stop,
                                    const DayCtl* ctl)
{
    if (ctl) {   // a day graph's closure: only on the day a trigger fired, window from the device
        if (!ctl->close || !((ctl->pol.close_place_types >> pt) & 1u)) return;
        start = ctl->close_start;
        stop = ctl->close_stop;
    }
    const bool per_unit = ctl && ctl->pol.per_adunit;
    const cs_params& P = *d.P;
    DevPlaces pl = d.pl[pt];
    // every place closed at ts afterwards has close_start >= start and close_end <= stop
    const uint16_t start0 = start, stop0 = stop;
    if (blockIdx.x == 0 && threadIdx.x == 0 && start0 < stop0) {
        atomicMin(d.close_window, (int32_t)start0);
        atomicMax(d.close_window + 1, (int32_t)stop0);
    }
    for (int l = blockIdx.x; l < pl.n; l += gridDim.x) {
        if (sel && !sel[pl.mcell[l]]) continue;
        uint16_t ws = start0, we = stop0;   // this place's closure window
        if (per_unit) {   // the window of the place's admin unit, if it switched on today
            const int a = d.mcell_adunit[pl.mcell[l]];
            if (a < 0 || a >= CS_MAX_ADUNITS || ctl->a_switch[a] != 1) continue;
            ws = ctl->a_close_start[a];
            we = ctl->a_close_stop[a];
        }
        __shared__ int do_members;
        if (threadIdx.x == 0) {
            do_members = 0;
            if (pl.close_end[l] < we) {
                if (pl.prob_close[l] >= P.Efficacies[CS_NPI_PLACE_CLOSURE][pt]) {
                    if (pl.close_start[l] > ws) pl.close_start[l] = ws;
                    pl.close_end[l] = we;
                    do_members = P.DoRealSymptWithdrawal;
                } else
                    pl.close_start[l] = pl.close_end[l] = we;
            }
        }
        __syncthreads();
        if (do_members) close_place_members(d, P, pt, l, ws, ws, we);
        __syncthreads();
    }
}

// Outcomes of a host's DoPlaceClose / DoPlaceOpen calls and holiday closures
// (cs_gpu_place_events), one block per event; every event of one launch has the
// same kind and place type.
__global__ void k_place_events(DevPop d, const cs_place_event* __restrict__ ev, int n)
{
    const cs_params& P = *d.P;
    for (int e = blockIdx.x; e < n; e += gridDim.x) {
        const cs_place_event E = ev[e];
        const DevPlaces& pl = d.pl[E.place_type];
        if (E.kind == CS_PLACE_EV_HOLIDAY) {   // src/Sweep.cpp:904-913
            if (threadIdx.x == 0) {
                if (pl.close_start[E.place] > E.win_start) pl.close_start[E.place] = E.win_start;
                if (pl.close_end[E.place] < E.win_stop) pl.close_end[E.place] = E.win_stop;
                if (pl.close_start[E.place] < pl.close_end[E.place]) {
                    atomicMin(d.close_window, (int32_t)pl.close_start[E.place]);
                    atomicMax(d.close_window + 1, (int32_t)pl.close_end[E.place]);
                }
            }
            for (int k = pl.member_ofs[E.place] + threadIdx.x; k < pl.member_ofs[E.place + 1]; k += blockDim.x) {
                PersonHot* hw = d.hot + pl.members[k];
                if (hw->absent_start > E.win_start) hw->absent_start = E.win_start;
                if (hw->absent_stop < E.win_stop) hw->absent_stop = E.win_stop;
            }
        } else if (E.kind == CS_PLACE_EV_CLOSE) {
            if (threadIdx.x == 0) {
                pl.close_start[E.place] = E.close_start;
                pl.close_end[E.place] = E.close_end;
                if (E.close_start < E.close_end) {
                    atomicMin(d.close_window, (int32_t)E.close_start);
                    atomicMax(d.close_window + 1, (int32_t)E.close_end);
                }
            }
            if (E.members && P.DoRealSymptWithdrawal) close_place_members(d, P, E.place_type, E.place, E.ts, E.win_start, E.win_stop);
        } else {
            const uint16_t ce = pl.close_end[E.place];
            __syncthreads();
            if (E.ts < ce) {
                if (P.DoRealSymptWithdrawal) open_place_members(d, P, E.place_type, E.place, E.ts, ce);
                if (threadIdx.x == 0) pl.close_end[E.place] = E.ts;
            }
        }
        __syncthreads();
    }
}

// Microcell status from a host's TreatSweep (cs_gpu_set_mcell_status).
__global__ void k_mcell_status(DevPop d, const int32_t* __restrict__ m, const uint8_t* __restrict__ sd,
                               const uint8_t* __restrict__ mr, int n)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        if (sd) d.socdist[m[k]] = sd[k];
        if (mr) d.moverest[m[k]] = mr[k];
    }
}
__global__ void k_close_places(DevPop d, int pt, const uint8_t* sel, uint16_t start, uint16_t stop, const DayCtl* ctl)
{
    k_close_places_body(d, pt, sel, start, stop, ctl);
}
__global__ void k_close_places_multi(const DevPop* __restrict__ pops, int pt, DayCtl* const* ctls)
{
    const DevPop& d = pops[blockIdx.y];
    if (pt < d.NPT) k_close_places_body(d, pt, nullptr, 0, 0, ctls[blockIdx.y]);
}

// The test after a timestep whether the susceptible fraction fell by more than 0.2
// since UpdateProbs last ran (src/CovidSim.cpp:1520-1526); S is fresh from k_cell_totals.
__device__ __forceinline__ void k_probs_check_body(const DevPop& d, DayCtl* ctl, int day_end)
{
    if (!day_end && !ctl->pol.probs_every_step) {   // this realisation tests at day ends only
        ctl->update = 0;
        return;
    }
    const double prop_s = (double)d.C->S / (double)d.N;
    int up = 0;
    if (ctl->prev_prop_s - prop_s > 0.2) {
        ctl->prev_prop_s = prop_s;
        up = 1;
    }
    ctl->update = up;
}
__global__ void k_probs_check(DevPop d, DayCtl* ctl, int day_end) { k_probs_check_body(d, ctl, day_end); }
__global__ void k_probs_check_multi(const DevPop* __restrict__ pops, DayCtl* const* ctls, int day_end)
{
    k_probs_check_body(pops[blockIdx.x], ctls[blockIdx.x], day_end);
}

// End of a day of the run loop: the day's counters into the series, and the global
// ICU trigger (src/CovidSim.cpp:3150-3159 with global thresholds) switching case
// isolation, household quarantine, social distancing and place closure on for
// pol.duration days, then off.  The switch takes effect from the next timestep.
// One trigger (the global one, or one admin unit's) at the end of a day, as the host
// loop decides it: 1 switches on (for pol.duration days), 0 switches off, -1 nothing.
// A global trigger fires at recent >= threshold (src/Sweep.cpp:1476), an admin unit's
// at recent > threshold (src/Sweep.cpp:1478-1482).
__device__ __forceinline__ int trigger_step(const cs_run_policy& pol, long long recent, double tn, int32_t& started,
                                            double& on_until, bool strict)
{
    if (!started && (strict ? recent > pol.icu_threshold : recent >= pol.icu_threshold)) {
        started = 1;
        on_until = tn + pol.duration;
        return 1;
    }
    if (started && on_until > 0 && tn >= on_until) {
        on_until = -1.0;
        return 0;
    }
    return -1;
}

__device__ void k_day_logic_body(const DevPop& d, DayCtl* ctl, const int32_t* clock, DevIv* iv)
{
    __shared__ int s_sw, s_any, s_cmin, s_cmax;
    const int day = ctl->day;
    {
        const unsigned long long* src = (const unsigned long long*)d.C;
        unsigned long long* dst = (unsigned long long*)(ctl->series + day);
        for (int k = threadIdx.x; k < (int)(sizeof(cs_counters) / 8); k += blockDim.x) dst[k] = src[k];
    }
    const cs_params& P = *d.P;
    const cs_run_policy& pol = ctl->pol;
    const double t = (double)(*clock - 1) * P.ModelTimeStep;   // the day's last timestep
    const double tn = t + P.ModelTimeStep;
    const int w = pol.icu_window;
    const cs_counters* past = day + 1 > w ? ctl->series + (day - w) : nullptr;
    const int ts = (int)(tn * P.TimeStepsPerDay);
    const int stop = min(65533, ts + (int)(pol.duration * P.TimeStepsPerDay));
    if (threadIdx.x == 0) {
        ctl->socd_write = 0;
        ctl->close = 0;
        s_sw = -1;
        s_any = 0;
        s_cmin = INT_MAX;
        s_cmax = 0;
        if (pol.icu_trigger && !pol.per_adunit) {
            const long long recent = (long long)d.C->cumCritical - (past ? (long long)past->cumCritical : 0ll);
            s_sw = trigger_step(pol, recent, tn, ctl->started, ctl->on_until, false);
        }
    }
    __syncthreads();
    if (pol.icu_trigger && !pol.per_adunit && s_sw >= 0) {   // every admin unit's windows
        const int sw = s_sw;
        for (int a = threadIdx.x; a < d.NA; a += blockDim.x) {
            iv->ci_start[a] = (sw && pol.case_isolation) ? tn : 1e10;
            iv->hq_start[a] = (sw && pol.household_quarantine) ? tn : 1e10;
        }
        if (threadIdx.x == 0) {
            iv->ci_dur = iv->hq_dur = pol.duration;
            ctl->socd_write = 1;
            ctl->socd_value = (sw && pol.social_distancing) ? CS_TREAT_TREATED : CS_TREAT_UNTREATED;
            if (sw) {
                ctl->close = 1;
                ctl->close_start = (uint16_t)ts;
                ctl->close_stop = (uint16_t)stop;
            }
        }
    }
    if (pol.icu_trigger && pol.per_adunit) {   // one trigger per admin unit
        const int na = min(d.NA, CS_MAX_ADUNITS);
        for (int a = threadIdx.x; a < CS_MAX_ADUNITS; a += blockDim.x) {
            int sw = -1;
            if (a < na) {
                const long long recent = (long long)d.C->cumCritical_adunit[a] -
                                         (past ? (long long)past->cumCritical_adunit[a] : 0ll);
                sw = trigger_step(pol, recent, tn, ctl->a_started[a], ctl->a_on_until[a], true);
            }
            ctl->a_switch[a] = (int8_t)sw;
            if (sw < 0) continue;
            iv->ci_start[a] = (sw && pol.case_isolation) ? tn : 1e10;
            iv->hq_start[a] = (sw && pol.household_quarantine) ? tn : 1e10;
            atomicOr(&s_any, 1);
            if (sw) {
                ctl->a_close_start[a] = (uint16_t)ts;
                ctl->a_close_stop[a] = (uint16_t)stop;
                if ((uint16_t)ts < (uint16_t)stop) {
                    atomicMin(&s_cmin, (int)(uint16_t)ts);
                    atomicMax(&s_cmax, (int)(uint16_t)stop);
                }
                atomicOr(&s_any, 2);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_any) {
            iv->ci_dur = iv->hq_dur = pol.duration;
            ctl->socd_write = 1;
            if (s_any & 2) {
                ctl->close = 1;
                ctl->close_start = (uint16_t)(s_cmin == INT_MAX ? 0 : s_cmin);
                ctl->close_stop = (uint16_t)s_cmax;
            }
        }
    }
    if (threadIdx.x == 0) ctl->day = day + 1;
}
__global__ void k_day_logic(DevPop d, DayCtl* ctl, const int32_t* clock, DevIv* iv) { k_day_logic_body(d, ctl, clock, iv); }
// one block per member; the window struct is the member's own (written only here and
// by cs_gpu_set_interventions)
__global__ void k_day_logic_multi(const DevPop* __restrict__ pops, DayCtl* const* ctls)
{
    const DevPop& d = pops[blockIdx.x];
    k_day_logic_body(d, ctls[blockIdx.x], d.step_clock, const_cast<DevIv*>(d.iv));
}

__device__ __forceinline__ void k_socdist_fill_body(const DevPop& d, const DayCtl* ctl)
{
    if (!ctl->socd_write) return;
    const bool per_unit = ctl->pol.per_adunit != 0;
    const uint8_t on = ctl->pol.social_distancing ? CS_TREAT_TREATED : CS_TREAT_UNTREATED;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < d.NM; m += gridDim.x * blockDim.x) {
        if (!per_unit) {
            d.socdist[m] = ctl->socd_value;
            continue;
        }
        const int a = d.mcell_adunit[m];
        if (a < 0 || a >= CS_MAX_ADUNITS || ctl->a_switch[a] < 0) continue;
        d.socdist[m] = ctl->a_switch[a] ? on : (uint8_t)CS_TREAT_UNTREATED;
    }
}
__global__ void k_socdist_fill(DevPop d, const DayCtl* ctl) { k_socdist_fill_body(d, ctl); }
__global__ void k_socdist_fill_multi(const DevPop* __restrict__ pops, DayCtl* const* ctls)
{
    k_socdist_fill_body(pops[blockIdx.y], ctls[blockIdx.y]);
}

__device__ __forceinline__ void k_cell_totals_body(const DevPop& d)
{
    long long s = 0, l = 0, i = 0, r = 0, dd = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.NC; c += gridDim.x * blockDim.x) {
        s += d.S[c]; l += d.L[c]; i += d.I[c]; r += d.R[c]; dd += d.D[c];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        l += __shfl_down_sync(0xffffffffu, l, o);
        i += __shfl_down_sync(0xffffffffu, i, o);
        r += __shfl_down_sync(0xffffffffu, r, o);
        dd += __shfl_down_sync(0xffffffffu, dd, o);
    }
    if ((threadIdx.x & 31) == 0) {
        cnt_add(CSB_CTR(S), s); cnt_add(CSB_CTR(L), l); cnt_add(CSB_CTR(I), i);
        cnt_add(CSB_CTR(R), r); cnt_add(CSB_CTR(D), dd);
    }
}
__global__ void k_cell_totals(DevPop d) { k_cell_totals_body(d); }
__global__ void k_cell_totals_multi(const DevPop* __restrict__ pops) { k_cell_totals_body(pops[blockIdx.y]); }
// S..D of each member's counter block to zero before k_cell_totals_multi
__global__ void k_zero_totals_multi(const DevPop* __restrict__ pops)
{
    if (threadIdx.x < 5) (&pops[blockIdx.x].C->S)[threadIdx.x] = 0;
}

// ================================================================ host API
extern "C" {

int cs_abi_version(void) { return CS_ABI_VERSION; }
size_t cs_sizeof_params(void) { return sizeof(cs_params); }
size_t cs_sizeof_population(void) { return sizeof(cs_population); }
size_t cs_sizeof_counters(void) { return sizeof(cs_counters); }
size_t cs_sizeof_interventions(void) { return sizeof(cs_interventions); }
size_t cs_sizeof_run_policy(void) { return sizeof(cs_run_policy); }

const char* cs_gpu_last_error(const cs_gpu_ctx* c) { return c ? c->err : "null context"; }

int cs_kernel_arch(int* binary_version, int* ptx_version)
{
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, (const void*)k_apply_infections) != cudaSuccess) {
        (void)cudaGetLastError();
        return CS_E_CUDA;
    }
    if (binary_version) *binary_version = a.binaryVersion;
    if (ptx_version) *ptx_version = a.ptxVersion;
    return CS_OK;
}
void* cs_gpu_stream(cs_gpu_ctx* c) { return c ? (void*)c->stream : nullptr; }
int64_t cs_gpu_launch_count(const cs_gpu_ctx* c) { return c ? c->launches : 0; }

static int check_params(cs_gpu_ctx* c, const cs_params* P)
{
    if (!(P->FalsePositiveRate >= 0 && P->FalsePositiveRate < 1)) return set_err(c, CS_E_ARG, "FalsePositiveRate outside [0, 1)");
    if (P->NumPlaceTypes < 0 || P->NumPlaceTypes > CS_MAX_PLACE_TYPES) return set_err(c, CS_E_ARG, "NumPlaceTypes out of range");
    if (P->kernel_size < 2 || P->kernel_expansion < 1 || !(P->kernel_delta > 0)) return set_err(c, CS_E_ARG, "kernel table not set");
    if (P->ncw <= 0 || P->nch <= 0) return set_err(c, CS_E_ARG, "grid size not set");
    return CS_OK;
}

// Dynamic state of one realisation and the per-step scratch, for a context whose
// static arrays (c->stat, and the static pointers in c->d) are in place.
static int alloc_dynamic(cs_gpu_ctx* c)
{
    DevPop& d = c->d;
    int r;
    const size_t N = d.N, NH = d.NH, NC = d.NC, NM = d.NM, NPT = d.NPT;
    const cs_params* params = &c->hp;
#define UP(field, src, n) do { if ((r = dupload(c, &field, src, n))) return r; } while (0)
#define AL(field, n) do { if ((r = dalloc(c, &field, n))) return r; } while (0)
    for (size_t pt = 0; pt < NPT; pt++) {
        DevPlaces& pl = d.pl[pt];
        AL(pl.close_start, (size_t)pl.n); AL(pl.close_end, (size_t)pl.n); AL(pl.prob_close, (size_t)pl.n);
    }
    AL(d.infection_time, N); AL(d.recovery_time, N); AL(d.sari_time, N); AL(d.critical_time, N);
    AL(d.stepdown_time, N); AL(d.detected_time, N); AL(d.prob_absent, N); AL(d.prob_care, N);
    AL(d.infector, N); AL(d.listpos, N); AL(d.infect_type, N); AL(d.pstep, N);
    AL(d.next_ev, N); AL(d.ev_init, 1);
    CK(cudaMemsetAsync(d.ev_init, 0xff, sizeof(int32_t), c->stream));
    {   // S, L, I, R, D side by side, so that a host can copy all five at once
        int32_t* cells5;
        AL(cells5, 5 * NC);
        d.S = cells5; d.L = cells5 + NC; d.I = cells5 + 2 * NC; d.R = cells5 + 3 * NC; d.D = cells5 + 4 * NC;
    }
    AL(d.S0, NC);
    AL(d.tot_prob, NC); AL(d.slots, N); AL(d.mark, N);
    AL(d.socdist, NM); AL(d.moverest, NM);
    CK(cudaMemsetAsync(d.socdist, 0, NM, c->stream));
    CK(cudaMemsetAsync(d.moverest, 0, NM, c->stream));
    AL(d.block_cell_info, NC); AL(d.block_info, (size_t)d.NB); AL(d.block_row_cum, (size_t)d.NB * d.NB);
    if (!d.bounds_static) AL(d.block_bound_tab, (size_t)d.NB * d.NB);   // else shared, filled once
    AL(d.block_guide, (size_t)d.NB * d.NB); AL(d.cell_guide, NC);
    {
        size_t G = (size_t)params->ncw * params->nch;
        AL(c->S0g, G); AL(c->Ag, G);
        const size_t nchunks = (params->nch + kTotProbRowChunk - 1) / kTotProbRowChunk;
        AL(c->Apart, nchunks * G);
        AL(c->rowS, (size_t)params->nch);
    }
    AL(d.claim, N); AL(d.queue, N); AL(d.counts, kCntN); AL(d.touched, NC); AL(d.cell_flag, NC + 4);
    AL(d.act, N); AL(d.act_cell, N); AL(d.cnt, NC); AL(d.cnt_ofs, N);
    AL(d.cmap, 2 * N); d.cmap_cap = (int32_t)(2 * N);
    AL(d.act_closed, N); AL(d.hh_flag, NH + 4); AL(d.hh_list, NH);
    AL(d.carer_win, NH); AL(d.carer_list, NH);
    CK(cudaMemsetAsync(d.carer_win, 0, sizeof(uint32_t) * NH, c->stream));
    AL(d.place_work, N * (size_t)(NPT > 0 ? NPT : 1));
    AL(d.close_window, 2);
    CK(cudaMemcpyAsync(d.close_window, kNoClosures, sizeof(kNoClosures), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(d.claim, 0xff, sizeof(unsigned long long) * N, c->stream));
    CK(cudaMemsetAsync(d.counts, 0, sizeof(int32_t) * kCntN, c->stream));
    CK(cudaMemsetAsync(d.cell_flag, 0, NC + 4, c->stream));
    CK(cudaMemsetAsync(d.hh_flag, 0, NH + 4, c->stream));
    CK(cudaMemsetAsync(d.cnt, 0, sizeof(int32_t) * NC, c->stream));
    CK(cudaMemsetAsync(d.pstep, 0, N, c->stream));
    { cs_params* t; UP(t, params, 1); c->dP = t; d.P = t; }
    {
        double *ci, *hq;
        AL(ci, d.NA); AL(hq, d.NA);
        DevIv iv{0, 0, ci, hq};
        DevIv* t; UP(t, &iv, 1); c->dIv = t; d.iv = t;
        c->iv_ci = ci; c->iv_hq = hq;
        LAUNCH(k_iv_reset, 1, kThreads, t, d.NA);
    }
    { DevStep* t; AL(t, 1); d.step = t; CK(cudaMemsetAsync(t, 0, sizeof(DevStep), c->stream)); }
    { unsigned long long* t; AL(t, 1); c->d_seed = t; d.seed_src = t; CK(cudaMemsetAsync(t, 0, sizeof(*t), c->stream)); }
    d.t_src = nullptr;
    { cs_counters* t; AL(t, 1); c->dC = t; d.C = t; CK(cudaMemsetAsync(t, 0, sizeof(cs_counters), c->stream)); }
    { double* t; UP(t, params->LocationInitialInfection, 2); d.rad_origin = t; }
    AL(d.fc_flag, N / 32 + 1); AL(d.fc_queue, N);
    CK(cudaMemsetAsync(d.fc_flag, 0, sizeof(uint32_t) * (N / 32 + 1), c->stream));
#undef UP
#undef AL
    CK(cudaStreamSynchronize(c->stream));   // the parameter and window copies came from the stack
    return CS_OK;
}

int cs_gpu_create(const cs_population* pop, const cs_params* params, int device, cs_gpu_ctx** out)
{
    if (!out) return CS_E_ARG;
    cs_gpu_ctx* c = new cs_gpu_ctx();
    *out = c;
    if (!pop || !params) return set_err(c, CS_E_ARG, "null population or parameters");
    int r = check_params(c, params);
    if (r) return r;
    if (pop->num_place_types != params->NumPlaceTypes) return set_err(c, CS_E_ARG, "place type count mismatch");
    c->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    c->grid = nsm * 8;
    c->hp = *params;
    c->stat = std::make_shared<StaticStore>();
    c->stat->device = device;
    DevPop& d = c->d;
    d.N = pop->n_people; d.NH = pop->n_households; d.NC = pop->n_cells; d.NM = pop->n_mcells; d.NPT = pop->num_place_types;
    d.NA = pop->n_adunits > 0 ? pop->n_adunits : 1;
    size_t N = d.N, NH = d.NH, NC = d.NC, NM = d.NM, NPT = d.NPT;
    if (d.NPT < 0 || d.NPT > CS_MAX_PLACE_TYPES) return set_err(c, CS_E_ARG, "num_place_types out of range");
    if (N >= (1u << 28)) return set_err(c, CS_E_UNSUPPORTED, "at most 2^28 - 1 people (place work entries pack index << 3)");
    if (N == 0 || NC == 0) return set_err(c, CS_E_ARG, "empty population");
#define UP(field, src, n) do { if ((r = dupload(c, &field, src, n))) return r; } while (0)
#define AL(field, n) do { if ((r = dalloc(c, &field, n))) return r; } while (0)
    // people: the record mixes static fields (household, microcell, age, flags)
    // with dynamic ones, so each realisation holds its own copy
    {
        std::vector<PersonHot> hot(N);
        for (size_t p = 0; p < N; p++) {
            PersonHot h{};
            h.hh = pop->person_hh[p];
            h.mcell = pop->person_mcell[p];
            h.age = pop->person_age[p];
            h.pflags = pop->person_flags ? pop->person_flags[p] : 0;
            h.absent_start = kNever;
            h.isolation_start = kNever;
            h.quar_start = kNever;
            h.susc = 1.0f;
            h.dflags = (uint8_t)(2u << CS_DF_QUAR_COMPLY_SHIFT);
            hot[p] = h;
        }
        PersonHot* ph;
        UP(ph, hot.data(), N);
        d.hot = ph;
        CK(cudaStreamSynchronize(c->stream));
    }
    // ---- static arrays, kept in the (shareable) static store
    c->alloc_to = &c->stat->allocs;
    {
        std::vector<PersonLinks> lk(N);
        for (size_t p = 0; p < N; p++) {
            PersonLinks& q = lk[p];
            for (int pt = 0; pt < CS_MAX_PLACE_TYPES; pt++) {
                q.link[pt] = pt < (int)NPT ? pop->person_place[pt * N + p] : -1;
                q.group[pt] = pt < (int)NPT ? pop->person_group[pt * N + p] : 0;
            }
            q.pad = 0;
        }
        PersonLinks* t;
        UP(t, lk.data(), N);
        d.links = t;
        CK(cudaStreamSynchronize(c->stream));
    }
    {
        std::vector<HouseholdRec> hh(NH);
        for (size_t h = 0; h < NH; h++)
            hh[h] = HouseholdRec{pop->hh_x[h], pop->hh_y[h], pop->hh_first[h], pop->hh_nh[h], pop->hh_nhr[h]};
        HouseholdRec* t;
        UP(t, hh.data(), NH);
        d.hhr = t;
        CK(cudaStreamSynchronize(c->stream));
    }
    { int32_t* t; UP(t, pop->mcell_cell, NM); d.mcell_cell = t; }
    { int32_t* t; UP(t, pop->mcell_adunit, NM); d.mcell_adunit = t; }
    { int32_t* t; UP(t, pop->cell_grid, NC); d.cell_grid = t; }
    { int32_t* t; UP(t, pop->cell_start, NC + 1); d.cell_start = t; }
    for (size_t m = 0; m < NC; m++)
        c->max_cell_people = std::max(c->max_cell_people, pop->cell_start[m + 1] - pop->cell_start[m]);
    { int32_t* t; UP(t, pop->cell_members, N); d.cell_members = t; }
    size_t ksz = (size_t)params->kernel_size + 1;
    { double* t; UP(t, pop->kernel_lookup, ksz); d.klookup = t; }
    { double* t; UP(t, pop->kernel_hi_res, ksz); d.khires = t; }
    {
        std::vector<float> f(ksz), g(ksz);
        for (size_t i = 0; i < ksz; i++) f[i] = (float)pop->kernel_lookup[i];
        for (size_t i = 0; i < ksz; i++) g[i] = (float)pop->kernel_hi_res[i];
        { float* t; UP(t, f.data(), ksz); d.klookup_f = t; }
        { float* t; UP(t, g.data(), ksz); d.khires_f = t; }
        CK(cudaStreamSynchronize(c->stream));   // before f and g go out of scope
    }
    for (size_t pt = 0; pt < NPT; pt++) {
        DevPlaces& pl = d.pl[pt];
        pl.n = pop->n_places[pt];
        size_t np = pl.n;
        size_t nm = pop->place_member_ofs[pt][np], ng = pop->place_group_ofs[pt][np];
        { int32_t* t; UP(t, pop->place_mcell[pt], np); pl.mcell = t; }
        { int32_t* t; UP(t, pop->place_member_ofs[pt], np + 1); pl.member_ofs = t; }
        { int32_t* t; UP(t, pop->place_members[pt], nm); pl.members = t; }
        { int32_t* t; UP(t, pop->place_group_ofs[pt], np + 1); pl.group_ofs = t; }
        { int32_t* t; UP(t, pop->group_start[pt], ng); pl.group_start = t; }
        { int32_t* t; UP(t, pop->group_size[pt], ng); pl.group_size = t; }
        { float* t; UP(t, pop->place_x[pt], np); pl.x = t; }
        { float* t; UP(t, pop->place_y[pt], np); pl.y = t; }
    }
    // proposal blocks
    int bs = params->block_cells;
    if (bs <= 0) {
        bs = 1;
        while (((params->ncw + bs - 1) / bs) * ((params->nch + bs - 1) / bs) > 4096) bs++;
    }
    d.bs = bs;
    d.nbx = (params->ncw + bs - 1) / bs;
    d.nby = (params->nch + bs - 1) / bs;
    d.NB = d.nbx * d.nby;
    // guide tables index blocks and a block's cells with 16-bit entries
    if (d.NB > 32767 || (long long)bs * bs > 32767)
        return set_err(c, CS_E_UNSUPPORTED, "proposal blocks: at most 32767 blocks of at most 32767 cells");
    {
        std::vector<int32_t> cb(NC), ofs(d.NB + 1, 0), cells(NC), fill(d.NB, 0);
        for (size_t m = 0; m < NC; m++) {
            int g = pop->cell_grid[m], x = g / params->nch, y = g % params->nch;
            cb[m] = (x / bs) * d.nby + (y / bs);
            ofs[cb[m] + 1]++;
        }
        for (int b = 0; b < d.NB; b++) ofs[b + 1] += ofs[b];
        for (size_t m = 0; m < NC; m++) cells[ofs[cb[m]] + fill[cb[m]]++] = (int32_t)m;
        { int32_t* t; UP(t, cb.data(), NC); d.cell_block = t; }
        { int32_t* t; UP(t, ofs.data(), (size_t)d.NB + 1); d.block_cell_ofs = t; }
        { int32_t* t; UP(t, cells.data(), NC); d.block_cells = t; }
        CK(cudaStreamSynchronize(c->stream));
    }
    {   // UpdateProbs denominators and the buffers only their pass uses
        size_t G = (size_t)params->ncw * params->nch;
        AL(c->Ng, G); AL(c->Bg, G);
        const size_t nchunks = (params->nch + kTotProbRowChunk - 1) / kTotProbRowChunk;
        AL(c->Bpart, nchunks * G);
        AL(c->rowN, (size_t)params->nch);
    }
    { float* t; AL(t, (size_t)d.nby * d.nby * d.nbx); d.bound_c = t; }
    d.block_bound_tab = nullptr;
    d.bounds_static = 1;
    c->alloc_to = nullptr;
#undef UP
#undef AL
    // ---- dynamic state of this realisation
    r = alloc_dynamic(c);
    if (r) return r;
    r = build_block_bounds(c);
    if (r) return r;
    r = build_kernel_rows(c);
    if (r) return r;
    r = tot_prob_pass(c, true);  // the n-weighted denominators never change
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

int cs_gpu_create_replica(const cs_gpu_ctx* base, cs_gpu_ctx** out)
{
    if (!out) return CS_E_ARG;
    cs_gpu_ctx* c = new cs_gpu_ctx();
    *out = c;
    if (!base || !base->stat) return set_err(c, CS_E_ARG, "replica of a null or unfinished context");
    int r;
    c->device = base->device;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    c->grid = base->grid;
    c->hp = base->hp;
    c->stat = base->stat;
    c->d = base->d;           // static pointers and sizes; dynamic ones are replaced below
    c->Ng = base->Ng; c->Bg = base->Bg; c->Bpart = base->Bpart; c->rowN = base->rowN;
    c->Gtab = base->Gtab;
    c->max_cell_people = base->max_cell_people;
    DevPop& d = c->d;
    {
        PersonHot* ph;
        if ((r = dalloc(c, &ph, (size_t)d.N))) return r;
        // static fields of the base's records; begin_run resets the dynamic ones
        CK(cudaMemcpyAsync(ph, base->d.hot, sizeof(PersonHot) * d.N, cudaMemcpyDeviceToDevice, c->stream));
        d.hot = ph;
    }
    r = alloc_dynamic(c);
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

void cs_gpu_destroy(cs_gpu_ctx* c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& r : c->ring) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (cudaEvent_t e : c->graph_events) cudaEventDestroy(e);
    if (c->side) { cudaStreamSynchronize(c->side); cudaStreamDestroy(c->side); }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->day_exec) cudaGraphExecDestroy(c->day_exec);
    if (c->day_graph) cudaGraphDestroy(c->day_graph);
    if (c->d_ctl) cudaFree(c->d_ctl);
    if (c->d_clock) cudaFree(c->d_clock);
    if (c->d_series) cudaFree(c->d_series);
    for (void* p : c->allocs) cudaFree(p);
    c->stat.reset();   // frees the static arrays when no replica still uses them
    if (c->xfer) cudaFree(c->xfer);
    if (c->d_seed_list) cudaFree(c->d_seed_list);
    if (c->d_ev) cudaFree(c->d_ev);
    if (c->d_mc) cudaFree(c->d_mc);
    if (c->pack16) cudaFree(c->pack16);
    if (c->packed) cudaFree(c->packed);
    cudaStream_t own = c->own_stream ? c->own_stream : c->stream;   // never a batch's stream
    if (own) cudaStreamDestroy(own);
    delete c;
}

int cs_gpu_set_params(cs_gpu_ctx* c, const cs_params* params)
{
    if (!c || !params) return CS_E_ARG;
    int r = check_params(c, params);
    if (r) return r;
    if (params->kernel_size != c->hp.kernel_size || params->NumPlaceTypes != c->hp.NumPlaceTypes || params->ncw != c->hp.ncw ||
        params->nch != c->hp.nch)
        return set_err(c, CS_E_ARG, "set_params may not change the kernel table, grid or place types");
    const cs_params& o = c->hp;
    const bool geometry = params->DoUTM_coords != o.DoUTM_coords || params->DoPeriodicBoundaries != o.DoPeriodicBoundaries ||
                          params->cell_width != o.cell_width || params->cell_height != o.cell_height ||
                          params->width_deg != o.width_deg || params->height_deg != o.height_deg ||
                          params->bbox_bottom_left_y != o.bbox_bottom_left_y || params->kernel_delta != o.kernel_delta ||
                          params->kernel_expansion != o.kernel_expansion ||
                          memcmp(params->sinx, o.sinx, sizeof(o.sinx)) || memcmp(params->cosx, o.cosx, sizeof(o.cosx)) ||
                          memcmp(params->asin2sqx, o.asin2sqx, sizeof(o.asin2sqx));
    if (geometry && c->stat.use_count() > 1)
        return set_err(c, CS_E_UNSUPPORTED, "set_params may not change the geometry of a population shared by replicas");
    drop_day_graph(c);   // captured with this kernel-row table and steps per day
    if ((params->FalsePositiveRate > 0) != (o.FalsePositiveRate > 0) && c->graph_exec) {
        // the captured step has the false-case pass only while false positives are on
        CK(cudaStreamSynchronize(c->stream));
        cudaGraphExecDestroy(c->graph_exec);
        cudaGraphDestroy(c->graph);
        c->graph_exec = nullptr;
        c->graph = nullptr;
    }
    c->hp = *params;
    CK(cudaMemcpyAsync(c->dP, params, sizeof(cs_params), cudaMemcpyHostToDevice, c->stream));
    if (geometry) {   // the kernel rows and the n-weighted denominators depend on it
        c->geometry_gen++;
        CK(cudaStreamSynchronize(c->stream));
        if (c->stat->Gtab) cudaFree(c->stat->Gtab);
        c->stat->Gtab = c->Gtab = nullptr;
        r = build_kernel_rows(c);
        if (r == CS_OK) r = build_block_bounds(c);
        if (r == CS_OK) r = tot_prob_pass(c, true);
        if (r) return r;
        CK(cudaStreamSynchronize(c->stream));
    }
    return CS_OK;
}

// bound(b, B) for every pair of proposal blocks, into the table the population's
// contexts share.  If a distance falls outside the kernel table, this context
// evaluates the bounds per call into its own table instead.
static int build_block_bounds(cs_gpu_ctx* c)
{
    DevPop& d = c->d;
    if (!d.bounds_static) return CS_OK;
    unsigned long long* oor = nullptr;
    CK(cudaMalloc(&oor, sizeof(unsigned long long)));
    CK(cudaMemsetAsync(oor, 0, sizeof(unsigned long long), c->stream));
    LAUNCH(k_block_bounds_all, c->grid, kThreads, d, (float*)d.bound_c, oor);
    unsigned long long h = 0;
    CK(cudaMemcpyAsync(&h, oor, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    cudaFree(oor);
    if (h) {
        d.bounds_static = 0;
        int r = dalloc(c, &d.block_bound_tab, (size_t)d.NB * d.NB);
        if (r) return r;
    }
    return CS_OK;
}

// Kernel rows for UpdateProbs, when they fit in kGtabMaxBytes.  If any distance
// falls outside the kernel table the rows are dropped again, so that UpdateProbs
// evaluates (and counts) them on every call as before.
constexpr size_t kGtabMaxBytes = (size_t)16 << 30;

static int build_kernel_rows(cs_gpu_ctx* c)
{
    const cs_params& P = c->hp;
    size_t n = (size_t)P.nch * P.nch * P.ncw;
    if (n * sizeof(float) > kGtabMaxBytes) return CS_OK;
    if (cudaMalloc(&c->stat->Gtab, n * sizeof(float)) != cudaSuccess) {
        (void)cudaGetLastError();
        c->stat->Gtab = c->Gtab = nullptr;
        return CS_OK;   // not enough memory: evaluate on the fly
    }
    c->Gtab = c->stat->Gtab;
    unsigned long long* oor = nullptr;
    CK(cudaMalloc(&oor, sizeof(unsigned long long)));
    CK(cudaMemsetAsync(oor, 0, sizeof(unsigned long long), c->stream));
    LAUNCH(k_kernel_rows, c->grid, kThreads, c->d, c->Gtab, oor);
    unsigned long long h = 0;
    CK(cudaMemcpyAsync(&h, oor, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    cudaFree(oor);
    if (h) {
        cudaFree(c->stat->Gtab);
        c->stat->Gtab = c->Gtab = nullptr;
    }
    return CS_OK;
}

// bytes of p to zero (a kernel rather than a memset so that a day graph can gate it)
__global__ void k_zero_gated(unsigned char* p, size_t bytes, const int32_t* gate)
{
    if (gate && !*gate) return;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < bytes; e += (size_t)gridDim.x * blockDim.x) p[e] = 0;
}

// The dynamic shared memory the row kernel needs, raised above the default before
// its first launch (and so never inside a graph capture that follows one).
static int tot_prob_smem(cs_gpu_ctx* c, bool denominators, size_t smem)
{
    size_t& have = c->tp_smem[denominators ? 1 : 0];
    if (smem <= 48 * 1024 || smem <= have) return CS_OK;
    if (denominators) CK(cudaFuncSetAttribute(k_tot_prob_rows<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else CK(cudaFuncSetAttribute(k_tot_prob_rows<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    have = smem;
    return CS_OK;
}

static int tot_prob_prepare(cs_gpu_ctx* c)
{
    const cs_params& P = c->hp;
    const TotProbGeom gm = tot_prob_geom(P.ncw, P.nch, true);
    return tot_prob_smem(c, false, gm.smem(false));
}

// One pass of the tot_prob row kernel: A from the current S0 (and, at creation,
// B from the cell populations).
static int tot_prob_pass(cs_gpu_ctx* c, bool denominators)
{
    DevPop& d = c->d;
    const cs_params& P = c->hp;
    size_t G = (size_t)P.ncw * P.nch;
    if (d.gate) {
        LAUNCH(k_zero_gated, c->grid, kThreads, (unsigned char*)c->S0g, sizeof(float) * G, d.gate);
        LAUNCH(k_zero_gated, 4, kThreads, c->rowS, (size_t)P.nch, d.gate);
    } else {
        CK(cudaMemsetAsync(c->S0g, 0, sizeof(float) * G, c->stream));
        CK(cudaMemsetAsync(c->rowS, 0, P.nch, c->stream));
    }
    if (denominators) {
        CK(cudaMemsetAsync(c->Ng, 0, sizeof(float) * G, c->stream));
        CK(cudaMemsetAsync(c->rowN, 0, P.nch, c->stream));
    }
    LAUNCH(k_grid_values, (d.NC + kThreads - 1) / kThreads, kThreads, d, c->S0g, denominators ? c->Ng : nullptr, c->rowS, c->rowN);
    const TotProbGeom gm = tot_prob_geom(P.ncw, P.nch, true);
    dim3 grid;
    int tpb;
    tot_prob_launch_shape(P.ncw, P.nch, gm, &grid, &tpb);
    const size_t smem = gm.smem(denominators);
    int r = tot_prob_smem(c, denominators, smem);
    if (r) return r;
    if (c->prof) prof_begin(c, "k_tot_prob_rows");
    if (denominators) {
        k_tot_prob_rows<true><<<grid, tpb, smem, c->stream>>>(d, c->S0g, c->Ng, c->rowS, c->rowN, c->Apart, c->Bpart, gm, c->Gtab);
    } else {
        k_tot_prob_rows<false><<<grid, tpb, smem, c->stream>>>(d, c->S0g, nullptr, c->rowS, nullptr, c->Apart, nullptr, gm, c->Gtab);
    }
    if (c->prof) prof_end(c);
    c->launches++;
    CK(cudaGetLastError());
    const int rgrid = (int)((G + kThreads - 1) / kThreads);
    LAUNCH(k_tot_prob_reduce, rgrid, kThreads, c->Apart, gm.nchunks, G, c->Ag, d.gate);
    if (denominators) LAUNCH(k_tot_prob_reduce, rgrid, kThreads, c->Bpart, gm.nchunks, G, c->Bg, d.gate);
    return CS_OK;
}

static int rebuild_blocks(cs_gpu_ctx* c)
{
    DevPop& d = c->d;
    LAUNCH(k_block_S0, (d.NB + kThreads - 1) / kThreads, kThreads, d);
    LAUNCH(k_block_rows, (d.NB * 32 + kThreads - 1) / kThreads, kThreads, d);
    return CS_OK;
}

int cs_gpu_update_probs(cs_gpu_ctx* c, int do_place)
{
    if (!c) return CS_E_ARG;
    DevPop& d = c->d;
    LAUNCH(k_update_S0, (d.NC + kThreads - 1) / kThreads, kThreads, d, do_place);
    int r = tot_prob_pass(c, false);
    if (r) return r;
    LAUNCH(k_tot_prob_finish, (d.NC + kThreads - 1) / kThreads, kThreads, d, c->Ag, c->Bg);
    return rebuild_blocks(c);
}

static int apply_queue(cs_gpu_ctx* c)
{
    DevPop& d = c->d;
    LAUNCH(k_apply_infections, c->grid, kThreads, d);
    LAUNCH(k_partition_S, c->grid, kThreads, d);
    if (c->hp.FalsePositiveRate > 0) LAUNCH(k_apply_false_cases, c->grid, kThreads, d);
    // every sweep leaves its list counters at zero for the next one; the household
    // list (last) is the incub sweep's
    CK(cudaMemsetAsync(d.counts, 0, sizeof(int32_t) * (kCntN - 1), c->stream));
    return CS_OK;
}

int cs_gpu_seed_infections(cs_gpu_ctx* c, double t, const int32_t* people, int n)
{
    if (!c) return CS_E_ARG;
    if (!c->run_started) return set_err(c, CS_E_STATE, "seed_infections before begin_run");
    if (n <= 0) return CS_OK;
    if (n > c->seed_cap) {
        if (c->d_seed_list) cudaFree(c->d_seed_list);
        c->d_seed_list = nullptr;
        CK(cudaMalloc(&c->d_seed_list, sizeof(int32_t) * n));
        c->seed_cap = n;
    }
    CK(cudaMemcpyAsync(c->d_seed_list, people, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream));
    LAUNCH(k_set_step, 1, 1, c->d, t, (unsigned long long)c->seed);
    LAUNCH(k_seed_claims, (n + kThreads - 1) / kThreads, kThreads, c->d, c->d_seed_list, n);
    return apply_queue(c);
}

// Run-level state outside the per-person view, as InitModel sets it: place
// closures and each place's closure threshold (src/CovidSim.cpp:1110-1125),
// social-distancing and movement flags, intervention windows.
static int reset_run_level(cs_gpu_ctx* c, uint64_t seed)
{
    DevPop& d = c->d;
    for (int pt = 0; pt < d.NPT; pt++) LAUNCH(k_reset_places, c->grid, kThreads, d, pt, seed);
    CK(cudaMemcpyAsync(d.close_window, kNoClosures, sizeof(kNoClosures), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(d.socdist, 0, d.NM, c->stream));
    CK(cudaMemsetAsync(d.moverest, 0, d.NM, c->stream));
    LAUNCH(k_iv_reset, 1, kThreads, c->dIv, d.NA);
    return CS_OK;
}

int cs_gpu_begin_run(cs_gpu_ctx* c, uint64_t seed, const int32_t* seed_people, int n_seed, int update_probs)
{
    if (!c) return CS_E_ARG;
    (void)update_probs;  // a fresh run has S0 = n and tot_prob = 1 exactly
    DevPop& d = c->d;
    c->seed = seed;
    CK(cudaMemcpyAsync(c->d_seed, &c->seed, sizeof(c->seed), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(d.C, 0, sizeof(cs_counters), c->stream));
    CK(cudaMemsetAsync(d.counts, 0, sizeof(int32_t) * kCntN, c->stream));
    CK(cudaMemsetAsync(d.cnt, 0, sizeof(int32_t) * d.NC, c->stream));
    LAUNCH(k_reset_people, c->grid, kThreads, d, seed);
    LAUNCH(k_reset_slots, c->grid, kThreads, d);
    LAUNCH(k_reset_listpos, (d.NC + kThreads - 1) / kThreads, kThreads, d);
    int r = reset_run_level(c, seed);
    if (r) return r;
    r = rebuild_blocks(c);
    if (r) return r;
    c->run_started = true;
    return cs_gpu_seed_infections(c, 0.0, seed_people, n_seed);
}

static int build_active(cs_gpu_ctx* c, int mode)
{
    DevPop& d = c->d;
    // the list counters are zero here: every sweep (and begin_run, upload_state,
    // seed_infections) ends by zeroing them
    const int ntiles = (d.NC + kThreads - 1) / kThreads;
    LAUNCH(k_build_active, ntiles * std::max(1, c->grid / ntiles), kThreads, d, mode);
    return CS_OK;
}

int cs_gpu_infect_sweep(cs_gpu_ctx* c, double t, int run)
{
    (void)run;
    if (!c) return CS_E_ARG;
    if (!c->run_started) return set_err(c, CS_E_STATE, "infect_sweep before begin_run");
    DevPop& d = c->d;
    LAUNCH(k_set_step, 1, 1, d, t, (unsigned long long)c->seed);
    int r = build_active(c, 0);
    if (r) return r;
    LAUNCH(k_infector_hh_spatial, c->grid, kThreads, d);
    // The place pass and the spatial pass both read the infector pass's lists and
    // only claim infections (atomicMin on the claim key) and add to counters, so the
    // place pass runs on the side stream beside the spatial pass (a branch of the
    // captured graphs).  While profiling they run one after the other.
    const bool fork = c->side && !c->prof;
    if (fork) {
        CK(cudaEventRecord(c->ev_fork, c->stream));
        CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
        k_infector_places<<<c->grid, kThreads, 0, c->side>>>(d);
        c->launches++;
        CK(cudaGetLastError());
        CK(cudaEventRecord(c->ev_join, c->side));
    } else {
        LAUNCH(k_infector_places, c->grid, kThreads, d);
    }
    switch (c->spatial_lanes) {
    case 2: LAUNCH(k_spatial<2>, c->grid, kThreads, d); break;
    case 4: LAUNCH(k_spatial<4>, c->grid, kThreads, d); break;
    case 16: LAUNCH(k_spatial<16>, c->grid, kThreads, d); break;
    default: LAUNCH(k_spatial<8>, c->grid, kThreads, d); break;
    }
    if (fork) CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    return apply_queue(c);
}

// IncubRecoverySweep; set_step false when the infect sweep of the same timestep has
// just written the step's scalars.
static int incub_sweep(cs_gpu_ctx* c, double t, bool set_step)
{
    DevPop& d = c->d;
    if (set_step) LAUNCH(k_set_step, 1, 1, d, t, (unsigned long long)c->seed);
    {   // every tile of kThreads cells shared by enough blocks to fill the grid
        const int ntiles = (d.NC + kThreads - 1) / kThreads;
        LAUNCH(k_incub_gather, ntiles * std::max(1, c->grid / ntiles), kThreads, d);
    }
    LAUNCH(k_incub_events, c->grid, kThreads, d);
    LAUNCH(k_incub_finish, c->grid, kThreads, d);
    CK(cudaMemsetAsync(d.counts, 0, sizeof(int32_t) * kCntN, c->stream));   // all list counters
    return CS_OK;
}

int cs_gpu_incub_recovery_sweep(cs_gpu_ctx* c, double t)
{
    if (!c) return CS_E_ARG;
    if (!c->run_started) return set_err(c, CS_E_STATE, "incub_recovery_sweep before begin_run");
    return incub_sweep(c, t, true);
}

static int step_eager(cs_gpu_ctx* c, double t, int run)
{
    int r = cs_gpu_infect_sweep(c, t, run);
    if (r) return r;
    return incub_sweep(c, t, false);
}

// Capture one whole timestep (both sweeps: ten kernels and two memsets, one more
// kernel with false positives on) as a CUDA graph.  Every kernel reads the step's
// scalars from device memory written by k_set_step, so a replay only needs the
// k_set_step node's arguments changed.
static int capture_step(cs_gpu_ctx* c, double t, int run)
{
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    long long l0 = c->launches;
    int r = step_eager(c, t, run);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (r || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        c->use_graph = false;  // fall back to eager launches for this context
        return r ? r : set_err(c, CS_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    }
    size_t n = 0;
    CK(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    CK(cudaGraphGetNodes(g, nodes.data(), &n));
    c->set_step_nodes.clear();
    c->set_step_params.clear();
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        CK(cudaGraphNodeGetType(nd, &ty));
        if (ty != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        CK(cudaGraphKernelNodeGetParams(nd, &kp));
        if (kp.func == (void*)k_set_step) {
            c->set_step_nodes.push_back(nd);
            c->set_step_params.push_back(kp);
        }
    }
    CK(cudaGraphInstantiate(&c->graph_exec, g, 0));
    c->graph = g;
    c->graph_launches = c->launches - l0;
    c->launches = l0;
    return CS_OK;
}

int cs_gpu_step(cs_gpu_ctx* c, double t, int run)
{
    if (!c) return CS_E_ARG;
    if (!c->run_started) return set_err(c, CS_E_STATE, "step before begin_run");
    if (!c->use_graph || c->prof) return step_eager(c, t, run);
    if (!c->graph_exec) {
        int r = capture_step(c, t, run);
        if (r) return r;
    }
    DevPop d = c->d;
    unsigned long long seed = c->seed;
    for (size_t k = 0; k < c->set_step_nodes.size(); k++) {
        void* args[] = {&d, &t, &seed};
        cudaKernelNodeParams kp = c->set_step_params[k];
        kp.kernelParams = args;
        kp.extra = nullptr;
        CK(cudaGraphExecKernelNodeSetParams(c->graph_exec, c->set_step_nodes[k], &kp));
    }
    CK(cudaGraphLaunch(c->graph_exec, c->stream));
    c->launches += c->graph_launches;
    return CS_OK;
}

int cs_gpu_set_grid(cs_gpu_ctx* c, int blocks)
{
    if (!c || blocks <= 0) return CS_E_ARG;
    CK(cudaStreamSynchronize(c->stream));
    c->grid = blocks;
    drop_day_graph(c);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
    return CS_OK;
}

int cs_gpu_grid(const cs_gpu_ctx* c) { return c ? c->grid : 0; }

int cs_gpu_set_spatial_lanes(cs_gpu_ctx* c, int lanes)
{
    if (!c) return CS_E_ARG;
    if (lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16) return set_err(c, CS_E_ARG, "spatial lanes must be 2, 4, 8 or 16");
    CK(cudaStreamSynchronize(c->stream));
    c->spatial_lanes = lanes;
    drop_day_graph(c);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
    return CS_OK;
}

int cs_gpu_use_graphs(cs_gpu_ctx* c, int enable)
{
    if (!c) return CS_E_ARG;
    c->use_graph = enable != 0;
    return CS_OK;
}

// ------------------------------------------------------- device run loop
// S..D of the counter block from the cells, as cs_gpu_get_counters does.
static int enqueue_totals(cs_gpu_ctx* c)
{
    CK(cudaMemsetAsync(c->d.C, 0, 5 * sizeof(int64_t), c->stream));
    LAUNCH(k_cell_totals, 64, kThreads, c->d);
    return CS_OK;
}

// One day of the run loop on the context's stream.  c->d carries the step clock
// (k_set_step takes t from it) and the UpdateProbs gate (&ctl->update), so the
// same launches serve every day and can be captured once.  Order as the host loop:
// the timesteps; after each (or the day's last) the counters and the UpdateProbs
// test; at the day's end the series and the trigger, then the gated UpdateProbs,
// and the switch's social-distancing flags and closures.
static int enqueue_day(cs_gpu_ctx* c, int spd, bool every_step)
{
    DevPop& d = c->d;
    for (int s = 0; s < spd; s++) {
        int r = step_eager(c, 0.0, 0);
        if (r) return r;
        if (!every_step && s < spd - 1) continue;
        r = enqueue_totals(c);
        if (r) return r;
        LAUNCH(k_probs_check, 1, 1, d, c->d_ctl, s == spd - 1 ? 1 : 0);
        if (s == spd - 1) LAUNCH(k_day_logic, 1, kThreads, d, c->d_ctl, (const int32_t*)c->d_clock, c->dIv);
        r = cs_gpu_update_probs(c, 0);
        if (r) return r;
    }
    const int mgrid = std::max(1, std::min(c->grid, (d.NM + kThreads - 1) / kThreads));
    LAUNCH(k_socdist_fill, mgrid, kThreads, d, (const DayCtl*)c->d_ctl);
    for (int pt = 0; pt < d.NPT; pt++)
        LAUNCH(k_close_places, c->grid, kThreads, d, pt, (const uint8_t*)nullptr, (uint16_t)0, (uint16_t)0, (const DayCtl*)c->d_ctl);
    if (d.NPT > 0) {
        LAUNCH(k_carer_pass, 64, kThreads, d);
        LAUNCH(k_carer_reset, 1, 1, d);
    }
    return CS_OK;
}

static int capture_day(cs_gpu_ctx* c, int spd, bool every_step)
{
    int r = tot_prob_prepare(c);
    if (r) return r;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    long long l0 = c->launches;
    r = enqueue_day(c, spd, every_step);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (r || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        c->launches = l0;
        return r ? r : set_err(c, CS_E_CUDA, "day graph capture: %s", cudaGetErrorString(e));
    }
    cudaError_t ei = cudaGraphInstantiate(&c->day_exec, g, 0);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        c->day_exec = nullptr;
        c->launches = l0;
        return set_err(c, CS_E_CUDA, "day graph instantiate: %s", cudaGetErrorString(ei));
    }
    c->day_graph = g;
    c->day_launches = c->launches - l0;
    c->day_every_step = every_step ? 1 : 0;
    c->launches = l0;
    return CS_OK;
}

static int run_days(cs_gpu_ctx* c, int days, int spd, bool every_step)
{
    const bool graph = c->use_graph;
    if (graph && (!c->day_exec || c->day_every_step != (every_step ? 1 : 0) || c->day_graph_prof != c->prof)) {
        drop_day_graph(c);
        prof_flush(c);
        c->graph_recs.clear();
        c->capturing_prof = c->prof;
        int r = capture_day(c, spd, every_step);
        c->capturing_prof = false;
        c->day_graph_prof = c->prof && r == CS_OK;
        if (r) return r;
    }
    for (int k = 0; k < days; k++) {
        if (graph) {
            CK(cudaGraphLaunch(c->day_exec, c->stream));
            c->launches += c->day_launches;
            if (c->day_graph_prof) prof_graph_collect(c);
        } else {
            int r = enqueue_day(c, spd, every_step);
            if (r) return r;
        }
    }
    return CS_OK;
}

// Timesteps per day of the context's parameters, or 0 when not a whole number.
static int steps_per_day(const cs_gpu_ctx* c)
{
    const int spd = (int)std::lround(c->hp.TimeStepsPerDay);
    return (spd >= 1 && (double)spd == c->hp.TimeStepsPerDay) ? spd : 0;
}

// The run loop's device state for a run of `days` days from t = 0 under pol: the
// control block, the step clock at 0, and room for the day-end series.
static int day_ctl_start(cs_gpu_ctx* c, int days, const cs_run_policy& pol)
{
    if (pol.icu_trigger && pol.icu_window < 1) return set_err(c, CS_E_ARG, "icu_window must be at least 1 day");
    if (!c->d_ctl) {
        CK(cudaMalloc(&c->d_ctl, sizeof(DayCtl)));
        CK(cudaMalloc(&c->d_clock, sizeof(int32_t)));
    }
    if (days > c->series_cap) {
        CK(cudaStreamSynchronize(c->stream));
        if (c->d_series) cudaFree(c->d_series);
        c->d_series = nullptr;
        c->series_cap = 0;
        CK(cudaMalloc(&c->d_series, sizeof(cs_counters) * (size_t)days));
        c->series_cap = days;
    }
    DayCtl h{};
    h.pol = pol;
    h.series = c->d_series;
    h.prev_prop_s = 1.0;
    h.on_until = -1.0;
    const int32_t zero = 0;
    CK(cudaMemcpyAsync(c->d_ctl, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_clock, &zero, sizeof(zero), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));   // h and zero live on this stack frame
    return CS_OK;
}

// The day-end series of a finished run into daily (may be NULL); the stream is
// synchronised afterwards, so *last holds the final day's counters.
static int day_series_out(cs_gpu_ctx* c, int days, cs_counters* daily, cs_counters* last)
{
    CK(cudaMemcpyAsync(last, c->d_series + (days - 1), sizeof(*last), cudaMemcpyDeviceToHost, c->stream));
    if (daily) CK(cudaMemcpyAsync(daily, c->d_series, sizeof(cs_counters) * (size_t)days, cudaMemcpyDeviceToHost, c->stream));
    return CS_OK;
}

static int check_give_ups(cs_gpu_ctx* c, const cs_counters& last)
{
    if (last.err_queue_overflow || last.err_spatial_tries || last.err_kernel_range)
        return set_err(c, CS_E_OVERFLOW, "bounded device loop gave up (spatial %lld, queue %lld, kernel range %lld)",
                       (long long)last.err_spatial_tries, (long long)last.err_queue_overflow, (long long)last.err_kernel_range);
    return CS_OK;
}

int cs_gpu_run(cs_gpu_ctx* c, int days, const cs_run_policy* policy, cs_counters* daily)
{
    if (!c || days < 0) return CS_E_ARG;
    if (!c->run_started) return set_err(c, CS_E_STATE, "run before begin_run");
    if (days == 0) return CS_OK;
    const int spd = steps_per_day(c);
    if (!spd) return set_err(c, CS_E_ARG, "the run loop needs a whole number of timesteps per day");
    cs_run_policy pol{};
    if (policy) pol = *policy;
    int r = day_ctl_start(c, days, pol);
    if (r) return r;
    c->d.step_clock = c->d_clock;
    c->d.gate = &c->d_ctl->update;
    r = run_days(c, days, spd, pol.probs_every_step != 0);
    c->d.step_clock = nullptr;
    c->d.gate = nullptr;
    if (r) return r;
    cs_counters last;
    r = day_series_out(c, days, daily, &last);
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    return check_give_ups(c, last);
}

// List counters of every member of a batch back to zero (the end-of-sweep reset).
__global__ void k_zero_counts_multi(const DevPop* __restrict__ pops, int n)
{
    if (threadIdx.x < n) pops[blockIdx.x].counts[threadIdx.x] = 0;
}

// ------------------------------------------------------------ batched steps
// A batch steps many realisations (contexts, each with its own population or a
// replica sharing one) with one CUDA graph per timestep.  Each of the step's
// kernels is launched once for all members: blockIdx.y selects the member, whose
// DevPop the kernel reads from a device array, so a timestep is the same 11
// kernels and 2 counter resets whatever the number of members.  While the batch
// exists every member's work goes to the batch's stream, which keeps a member's
// own calls (UpdateProbs, interventions, counters) ordered with the batched steps.
struct cs_gpu_batch {
    int device = 0;
    std::vector<cs_gpu_ctx*> members;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> member_launches;
    double* d_t = nullptr;   // the timestep's t, read by every member's k_set_step
    DevPop* d_pops = nullptr; // members' DevPop (t taken from d_t)
    int lanes = 8;            // spatial lanes of the batched launches
    // device run loop (cs_gpu_batch_run): members' DevPop with step clocks and
    // UpdateProbs gates, their control blocks, one graph per day
    DevPop* d_pops_day = nullptr;
    DayCtl** d_ctls = nullptr;
    cudaGraph_t day_graph = nullptr;
    cudaGraphExec_t day_exec = nullptr;
    int day_every_step = -1;
    int day_spd = 0;
    std::vector<long long> day_geometry;       // members' geometry_gen when the day graph was captured
    std::vector<long long> member_day_launches;
    static constexpr int kSide = 8;            // streams the members' UpdateProbs chains fan out to
    cudaStream_t side[kSide] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kSide] = {};
    char err[512] = {0};
};

static int batch_err(cs_gpu_batch* b, int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b->err, sizeof(b->err), fmt, ap);
    va_end(ap);
    return code;
}

#define BCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return batch_err(b, CS_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

static void batch_drop_graph(cs_gpu_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    if (b->day_exec) cudaGraphExecDestroy(b->day_exec);
    if (b->day_graph) cudaGraphDestroy(b->day_graph);
    b->day_exec = nullptr;
    b->day_graph = nullptr;
}

int cs_gpu_batch_create(cs_gpu_ctx* const* members, int n, cs_gpu_batch** out)
{
    if (!out || !members || n <= 0) return CS_E_ARG;
    cs_gpu_batch* b = new cs_gpu_batch();
    *out = b;
    b->device = members[0] ? members[0]->device : 0;
    for (int k = 0; k < n; k++) {
        cs_gpu_ctx* m = members[k];
        if (!m) return batch_err(b, CS_E_ARG, "member %d is null", k);
        if (m->device != b->device) return batch_err(b, CS_E_ARG, "member %d is on device %d, not %d", k, m->device, b->device);
        if (m->own_stream) return batch_err(b, CS_E_STATE, "member %d already belongs to a batch", k);
        for (int j = 0; j < k; j++)
            if (members[j] == m) return batch_err(b, CS_E_ARG, "member %d appears twice", k);
    }
    BCK(cudaSetDevice(b->device));
    BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    BCK(cudaMalloc(&b->d_t, sizeof(double)));
    BCK(cudaMalloc(&b->d_pops, sizeof(DevPop) * n));
    b->members.assign(members, members + n);
    b->member_launches.assign(n, 0);
    for (int k = 0; k < n; k++) {
        cs_gpu_ctx* m = b->members[k];
        BCK(cudaStreamSynchronize(m->stream));
        m->own_stream = m->stream;
        m->stream = b->stream;
    }
    return CS_OK;
}

const char* cs_gpu_batch_last_error(const cs_gpu_batch* b) { return b ? b->err : "null batch"; }

#define BLAUNCH(kernel, grid, block, ...)                                                          \
    do {                                                                                           \
        kernel<<<(grid), (block), 0, b->stream>>>(__VA_ARGS__);                                    \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess) return batch_err(b, CS_E_CUDA, "launch %s: %s", #kernel, cudaGetErrorString(e_)); \
    } while (0)

// The batched timestep, in the order of step_eager (InfectSweep, then
// IncubRecoverySweep without a second k_set_step).
static int batch_enqueue(cs_gpu_batch* b, const DevPop* pops)
{
    const int R = (int)b->members.size();
    const int grid = b->members[0]->grid;
    const dim3 g(grid, R), one(1, R);
    BLAUNCH(k_set_step_multi, one, 1, pops, 0.0, 0ull);
    BLAUNCH(k_build_active_multi, g, kThreads, pops, 0);
    BLAUNCH(k_infector_hh_spatial_multi, g, kThreads, pops);
    BLAUNCH(k_infector_places_multi, g, kThreads, pops);
    switch (b->lanes) {
    case 2: BLAUNCH(k_spatial_multi<2>, g, kThreads, pops); break;
    case 4: BLAUNCH(k_spatial_multi<4>, g, kThreads, pops); break;
    case 16: BLAUNCH(k_spatial_multi<16>, g, kThreads, pops); break;
    default: BLAUNCH(k_spatial_multi<8>, g, kThreads, pops); break;
    }
    BLAUNCH(k_apply_infections_multi, g, kThreads, pops);
    BLAUNCH(k_partition_S_multi, g, kThreads, pops);
    bool fpr = false;
    for (const cs_gpu_ctx* m : b->members) fpr |= m->hp.FalsePositiveRate > 0;
    if (fpr) BLAUNCH(k_apply_false_cases_multi, g, kThreads, pops);
    BLAUNCH(k_zero_counts_multi, R, 32, pops, (int)(kCntN - 1));   // the household list is the incub sweep's
    BLAUNCH(k_incub_gather_multi, g, kThreads, pops);
    BLAUNCH(k_incub_events_multi, g, kThreads, pops);
    BLAUNCH(k_incub_finish_multi, g, kThreads, pops);
    BLAUNCH(k_zero_counts_multi, R, 32, pops, (int)kCntN);
    return CS_OK;
}

static int batch_same_grid(cs_gpu_batch* b)
{
    for (size_t k = 1; k < b->members.size(); k++)
        if (b->members[k]->grid != b->members[0]->grid)
            return batch_err(b, CS_E_ARG, "members use different launch shapes; set one with cs_gpu_batch_set_grid");
    return CS_OK;
}

static int batch_capture(cs_gpu_batch* b, double t, int run)
{
    (void)t;
    (void)run;
    const int n = (int)b->members.size();
    if (int r = batch_same_grid(b)) return r;
    // members' DevPop, each taking t from the batch
    std::vector<DevPop> hp(n);
    for (int k = 0; k < n; k++) {
        hp[k] = b->members[k]->d;
        hp[k].t_src = b->d_t;
    }
    BCK(cudaMemcpyAsync(b->d_pops, hp.data(), sizeof(DevPop) * n, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int r = batch_enqueue(b, b->d_pops);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (r || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return r ? r : batch_err(b, CS_E_CUDA, "batch capture: %s", cudaGetErrorString(e));
    }
    BCK(cudaGraphInstantiate(&b->exec, g, 0));
    b->graph = g;
    for (int k = 0; k < n; k++) b->member_launches[k] = 11;   // kernels run for each member per step
    return CS_OK;
}

int cs_gpu_batch_step(cs_gpu_batch* b, double t, int run)
{
    if (!b) return CS_E_ARG;
    for (size_t k = 0; k < b->members.size(); k++)
        if (!b->members[k]->run_started) return batch_err(b, CS_E_STATE, "member %zu: step before begin_run", k);
    if (!b->exec) {
        int r = batch_capture(b, t, run);
        if (r) return r;
    }
    // every member's k_set_step reads t (and its run's seed) from device memory
    BCK(cudaMemcpyAsync(b->d_t, &t, sizeof(double), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaGraphLaunch(b->exec, b->stream));
    for (size_t k = 0; k < b->members.size(); k++) b->members[k]->launches += b->member_launches[k];
    return CS_OK;
}

// Launch shape of every member's grid-stride kernels (blocks); the batch graph is
// captured again at the next step.  Results do not depend on it.
int cs_gpu_batch_set_grid(cs_gpu_batch* b, int blocks)
{
    if (!b || blocks <= 0) return CS_E_ARG;
    BCK(cudaStreamSynchronize(b->stream));
    for (cs_gpu_ctx* m : b->members) {
        m->grid = blocks;
        drop_day_graph(m);
        if (m->graph_exec) cudaGraphExecDestroy(m->graph_exec);
        if (m->graph) cudaGraphDestroy(m->graph);
        m->graph_exec = nullptr;
        m->graph = nullptr;
    }
    batch_drop_graph(b);
    return CS_OK;
}

int cs_gpu_batch_set_spatial_lanes(cs_gpu_batch* b, int lanes)
{
    if (!b) return CS_E_ARG;
    if (lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16) return batch_err(b, CS_E_ARG, "spatial lanes must be 2, 4, 8 or 16");
    BCK(cudaStreamSynchronize(b->stream));
    b->lanes = lanes;
    batch_drop_graph(b);
    return CS_OK;
}

void* cs_gpu_batch_stream(cs_gpu_batch* b) { return b ? (void*)b->stream : nullptr; }

int cs_gpu_batch_sync(cs_gpu_batch* b)
{
    if (!b) return CS_E_ARG;
    BCK(cudaStreamSynchronize(b->stream));
    return CS_OK;
}

// ------------------------------------------------------- batched run loop
// The single-context day (enqueue_day) for every member at once: the batched
// timesteps, then the members' totals, UpdateProbs tests and day logic as one
// launch each (blockIdx selects the member), and each member's gated UpdateProbs
// chain on one of kSide side streams, forked from and joined back into the
// batch's stream, so that the chains' mostly empty launches overlap.
static int batch_updates(cs_gpu_batch* b)
{
    BCK(cudaEventRecord(b->ev_fork, b->stream));
    for (int i = 0; i < cs_gpu_batch::kSide; i++) BCK(cudaStreamWaitEvent(b->side[i], b->ev_fork, 0));
    int r = CS_OK;
    for (size_t k = 0; k < b->members.size() && !r; k++) {
        cs_gpu_ctx* m = b->members[k];
        m->stream = b->side[k % cs_gpu_batch::kSide];
        const long long l0 = m->launches;
        r = cs_gpu_update_probs(m, 0);
        b->member_day_launches[k] += m->launches - l0;
        m->launches = l0;
        m->stream = b->stream;
        if (r) batch_err(b, r, "member %zu UpdateProbs: %s", k, m->err);
    }
    // joined even after an error, so that the capture can end
    for (int i = 0; i < cs_gpu_batch::kSide; i++) {
        cudaEventRecord(b->ev_join[i], b->side[i]);
        cudaStreamWaitEvent(b->stream, b->ev_join[i], 0);
    }
    return r;
}

static int batch_enqueue_day(cs_gpu_batch* b, int spd, bool every_step)
{
    const int R = (int)b->members.size();
    const DevPop* pops = b->d_pops_day;
    int npt = 0;
    for (cs_gpu_ctx* m : b->members) npt = std::max(npt, m->d.NPT);
    for (int s = 0; s < spd; s++) {
        int r = batch_enqueue(b, pops);
        if (r) return r;
        for (int k = 0; k < R; k++) b->member_day_launches[k] += 11;
        if (!every_step && s < spd - 1) continue;
        const int day_end = s == spd - 1 ? 1 : 0;
        BLAUNCH(k_zero_totals_multi, R, 32, pops);
        BLAUNCH(k_cell_totals_multi, dim3(64, R), kThreads, pops);
        BLAUNCH(k_probs_check_multi, R, 1, pops, b->d_ctls, day_end);
        if (day_end) BLAUNCH(k_day_logic_multi, R, kThreads, pops, b->d_ctls);
        for (int k = 0; k < R; k++) b->member_day_launches[k] += 2 + day_end;
        r = batch_updates(b);
        if (r) return r;
    }
    const dim3 g(b->members[0]->grid, R);
    BLAUNCH(k_socdist_fill_multi, g, kThreads, pops, b->d_ctls);
    for (int pt = 0; pt < npt; pt++) BLAUNCH(k_close_places_multi, g, kThreads, pops, pt, b->d_ctls);
    if (npt > 0) {
        BLAUNCH(k_carer_pass_multi, dim3(64, R), kThreads, pops);
        BLAUNCH(k_carer_reset_multi, R, 1, pops);
    }
    for (int k = 0; k < R; k++) b->member_day_launches[k] += 1 + b->members[k]->d.NPT + (npt > 0 ? 2 : 0);
    return CS_OK;
}

static int batch_capture_day(cs_gpu_batch* b, int spd, bool every_step)
{
    const int n = (int)b->members.size();
    if (!b->ev_fork) {
        BCK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
        for (int i = 0; i < cs_gpu_batch::kSide; i++) {
            BCK(cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking));
            BCK(cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming));
        }
    }
    for (cs_gpu_ctx* m : b->members)
        if (int r = tot_prob_prepare(m)) return batch_err(b, r, "%s", m->err);
    b->member_day_launches.assign(n, 0);
    // the members' own launches (their UpdateProbs chains) read the clock and gate too
    for (cs_gpu_ctx* m : b->members) {
        m->d.step_clock = m->d_clock;
        m->d.gate = &m->d_ctl->update;
    }
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int r = batch_enqueue_day(b, spd, every_step);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    for (cs_gpu_ctx* m : b->members) {
        m->d.step_clock = nullptr;
        m->d.gate = nullptr;
    }
    if (r || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return r ? r : batch_err(b, CS_E_CUDA, "batch day graph capture: %s", cudaGetErrorString(e));
    }
    cudaError_t ei = cudaGraphInstantiate(&b->day_exec, g, 0);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        b->day_exec = nullptr;
        return batch_err(b, CS_E_CUDA, "batch day graph instantiate: %s", cudaGetErrorString(ei));
    }
    b->day_graph = g;
    b->day_every_step = every_step ? 1 : 0;
    b->day_spd = spd;
    b->day_geometry.resize(n);
    for (int k = 0; k < n; k++) b->day_geometry[k] = b->members[k]->geometry_gen;
    return CS_OK;
}

int cs_gpu_batch_run(cs_gpu_batch* b, int days, const cs_run_policy* policies, cs_counters* daily)
{
    if (!b || days < 0) return CS_E_ARG;
    const int n = (int)b->members.size();
    for (int k = 0; k < n; k++)
        if (!b->members[k]->run_started) return batch_err(b, CS_E_STATE, "member %d: run before begin_run", k);
    if (days == 0) return CS_OK;
    if (int r = batch_same_grid(b)) return r;
    for (int k = 0; k < n; k++)
        if (b->members[k]->prof) return batch_err(b, CS_E_STATE, "member %d has per-launch timing on", k);
    const int spd = steps_per_day(b->members[0]);
    for (int k = 0; k < n; k++)
        if (!spd || steps_per_day(b->members[k]) != spd)
            return batch_err(b, CS_E_ARG, "the batched run loop needs the same whole number of timesteps per day in every member");
    bool every = false;
    for (int k = 0; k < n; k++) {
        cs_gpu_ctx* m = b->members[k];
        cs_run_policy pol{};
        if (policies) pol = policies[k];
        every = every || pol.probs_every_step;
        if (int r = day_ctl_start(m, days, pol)) return batch_err(b, r, "member %d: %s", k, m->err);
    }
    if (!b->d_pops_day) {
        BCK(cudaMalloc(&b->d_pops_day, sizeof(DevPop) * n));
        BCK(cudaMalloc(&b->d_ctls, sizeof(DayCtl*) * n));
    }
    std::vector<DevPop> hp(n);
    std::vector<DayCtl*> hc(n);
    for (int k = 0; k < n; k++) {
        cs_gpu_ctx* m = b->members[k];
        hp[k] = m->d;
        hp[k].step_clock = m->d_clock;
        hp[k].gate = &m->d_ctl->update;
        hc[k] = m->d_ctl;
    }
    BCK(cudaMemcpyAsync(b->d_pops_day, hp.data(), sizeof(DevPop) * n, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->d_ctls, hc.data(), sizeof(DayCtl*) * n, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    bool stale = !b->day_exec || b->day_every_step != (every ? 1 : 0) || b->day_spd != spd;
    for (int k = 0; k < n && !stale; k++) stale = b->day_geometry[k] != b->members[k]->geometry_gen;
    if (stale) {
        if (b->day_exec) cudaGraphExecDestroy(b->day_exec);
        if (b->day_graph) cudaGraphDestroy(b->day_graph);
        b->day_exec = nullptr;
        b->day_graph = nullptr;
        if (int r = batch_capture_day(b, spd, every)) return r;
    }
    for (int d = 0; d < days; d++) BCK(cudaGraphLaunch(b->day_exec, b->stream));
    for (int k = 0; k < n; k++) b->members[k]->launches += b->member_day_launches[k] * days;
    std::vector<cs_counters> last(n);
    for (int k = 0; k < n; k++)
        if (int r = day_series_out(b->members[k], days, daily ? daily + (size_t)k * days : nullptr, &last[k]))
            return batch_err(b, r, "member %d: %s", k, b->members[k]->err);
    BCK(cudaStreamSynchronize(b->stream));
    for (int k = 0; k < n; k++)
        if (int r = check_give_ups(b->members[k], last[k])) return batch_err(b, r, "member %d: %s", k, b->members[k]->err);
    return CS_OK;
}

void cs_gpu_batch_destroy(cs_gpu_batch* b)
{
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    for (int i = 0; i < cs_gpu_batch::kSide; i++) {
        if (b->side[i]) cudaStreamDestroy(b->side[i]);
        if (b->ev_join[i]) cudaEventDestroy(b->ev_join[i]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->d_pops_day) cudaFree(b->d_pops_day);
    if (b->d_ctls) cudaFree(b->d_ctls);
    for (cs_gpu_ctx* m : b->members)
        if (m && m->own_stream) {
            m->stream = m->own_stream;
            m->own_stream = nullptr;
        }
    if (b->d_t) cudaFree(b->d_t);
    if (b->d_pops) cudaFree(b->d_pops);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int cs_gpu_set_interventions(cs_gpu_ctx* c, const cs_interventions* iv)
{
    if (!c || !iv) return CS_E_ARG;
    const int na = c->d.NA;
    std::vector<double> ci(na), hq(na);
    for (int a = 0; a < na; a++) {
        ci[a] = iv->adunit_CaseIsolationTimeStart ? iv->adunit_CaseIsolationTimeStart[a] : iv->CaseIsolationTimeStart;
        hq[a] = iv->adunit_HQuarantineTimeStart ? iv->adunit_HQuarantineTimeStart[a] : iv->HQuarantineTimeStart;
    }
    DevIv div{iv->CaseIsolationPolicyDuration, iv->HQuarantinePolicyDuration, c->iv_ci, c->iv_hq};
    CK(cudaMemcpyAsync(c->iv_ci, ci.data(), sizeof(double) * na, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->iv_hq, hq.data(), sizeof(double) * na, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->dIv, &div, sizeof(div), cudaMemcpyHostToDevice, c->stream));
    if (iv->mcell_socdist) CK(cudaMemcpyAsync(c->d.socdist, iv->mcell_socdist, c->d.NM, cudaMemcpyHostToDevice, c->stream));
    if (iv->mcell_moverest) CK(cudaMemcpyAsync(c->d.moverest, iv->mcell_moverest, c->d.NM, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

int cs_gpu_close_places(cs_gpu_ctx* c, int pt, const int32_t* mcells, int n_mcells, uint16_t start, uint16_t stop)
{
    if (!c) return CS_E_ARG;
    if (pt < 0 || pt >= c->d.NPT) return set_err(c, CS_E_ARG, "bad place type %d", pt);
    uint8_t* sel = nullptr;
    if (mcells) {
        std::vector<uint8_t> h(c->d.NM, 0);
        for (int k = 0; k < n_mcells; k++) if (mcells[k] >= 0 && mcells[k] < c->d.NM) h[mcells[k]] = 1;
        CK(cudaMalloc(&sel, c->d.NM));
        CK(cudaMemcpyAsync(sel, h.data(), c->d.NM, cudaMemcpyHostToDevice, c->stream));
    }
    LAUNCH(k_close_places, c->grid, kThreads, c->d, pt, sel, start, stop, (const DayCtl*)nullptr);
    LAUNCH(k_carer_pass, 64, kThreads, c->d);
    LAUNCH(k_carer_reset, 1, 1, c->d);
    if (sel) {
        CK(cudaStreamSynchronize(c->stream));
        cudaFree(sel);
    }
    return CS_OK;
}

// Outcomes of a host TreatSweep's DoPlaceClose / DoPlaceOpen calls: opens first,
// then closes, each kind place type by place type, so that one launch never has two
// places of a person; the closures' carers follow the last close launch.
int cs_gpu_place_events(cs_gpu_ctx* c, const cs_place_event* ev, int n)
{
    if (!c) return CS_E_ARG;
    if (n < 0 || (n > 0 && !ev)) return set_err(c, CS_E_ARG, "bad event list");
    if (n == 0) return CS_OK;
    std::vector<cs_place_event> v(ev, ev + n);
    for (const cs_place_event& e : v) {
        if (e.place_type >= c->d.NPT || e.place < 0 || e.place >= c->d.pl[e.place_type].n)
            return set_err(c, CS_E_ARG, "place event: place %d of type %d out of range", e.place, (int)e.place_type);
        if (e.kind != CS_PLACE_EV_CLOSE && e.kind != CS_PLACE_EV_OPEN && e.kind != CS_PLACE_EV_HOLIDAY)
            return set_err(c, CS_E_ARG, "place event: bad kind %d", (int)e.kind);
    }
    // opens, closes, holidays; each kind place type by place type
    auto key = [](const cs_place_event& e) {
        return (e.kind == CS_PLACE_EV_OPEN ? 0 : e.kind == CS_PLACE_EV_CLOSE ? 16 : 32) + (int)e.place_type;
    };
    std::stable_sort(v.begin(), v.end(), [&](const cs_place_event& a, const cs_place_event& b) { return key(a) < key(b); });
    if (c->ev_cap < n) {
        if (c->d_ev) cudaFree(c->d_ev);
        c->d_ev = nullptr;
        c->ev_cap = 0;
        CK(cudaMalloc(&c->d_ev, sizeof(cs_place_event) * (size_t)n));
        c->ev_cap = n;
    }
    CK(cudaMemcpyAsync(c->d_ev, v.data(), sizeof(cs_place_event) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    bool closes = false;
    for (int i0 = 0; i0 < n;) {
        int i1 = i0;
        while (i1 < n && key(v[i1]) == key(v[i0])) i1++;
        if (v[i0].kind == CS_PLACE_EV_HOLIDAY && closes) {   // the closures' carers before the holidays
            LAUNCH(k_carer_pass, 64, kThreads, c->d);
            LAUNCH(k_carer_reset, 1, 1, c->d);
            closes = false;
        }
        LAUNCH(k_place_events, std::min(c->grid, i1 - i0), kThreads, c->d, c->d_ev + i0, i1 - i0);
        closes |= v[i0].kind == CS_PLACE_EV_CLOSE;
        i0 = i1;
    }
    if (closes) {
        LAUNCH(k_carer_pass, 64, kThreads, c->d);
        LAUNCH(k_carer_reset, 1, 1, c->d);
    }
    CK(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

int cs_gpu_set_mcell_status(cs_gpu_ctx* c, const int32_t* mcells, const uint8_t* socdist, const uint8_t* moverest, int n)
{
    if (!c) return CS_E_ARG;
    if (n < 0 || (n > 0 && !mcells)) return set_err(c, CS_E_ARG, "bad microcell list");
    if (n == 0 || (!socdist && !moverest)) return CS_OK;
    for (int k = 0; k < n; k++)
        if (mcells[k] < 0 || mcells[k] >= c->d.NM) return set_err(c, CS_E_ARG, "microcell %d out of range", mcells[k]);
    const size_t need = (size_t)n * (4 + 2);
    if (c->mc_cap < need) {
        if (c->d_mc) cudaFree(c->d_mc);
        c->d_mc = nullptr;
        c->mc_cap = 0;
        CK(cudaMalloc(&c->d_mc, need));
        c->mc_cap = need;
    }
    int32_t* dm = (int32_t*)c->d_mc;
    uint8_t* dsd = (uint8_t*)(dm + n);
    uint8_t* dmr = dsd + n;
    CK(cudaMemcpyAsync(dm, mcells, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    if (socdist) CK(cudaMemcpyAsync(dsd, socdist, (size_t)n, cudaMemcpyHostToDevice, c->stream));
    if (moverest) CK(cudaMemcpyAsync(dmr, moverest, (size_t)n, cudaMemcpyHostToDevice, c->stream));
    LAUNCH(k_mcell_status, std::max(1, std::min(c->grid, (n + kThreads - 1) / kThreads)), kThreads, c->d, dm,
           socdist ? (const uint8_t*)dsd : nullptr, moverest ? (const uint8_t*)dmr : nullptr, n);
    CK(cudaStreamSynchronize(c->stream));
    return CS_OK;
}


int cs_gpu_profile(cs_gpu_ctx* c, int enable)
{
    if (!c) return CS_E_ARG;
    if (enable && c->ring.empty()) {
        c->ring.resize(4096);
        for (auto& r : c->ring) {
            CK(cudaEventCreate(&r.a));
            CK(cudaEventCreate(&r.b));
        }
    }
    if (!enable) prof_flush(c);
    c->prof = enable != 0;
    if (enable == 2) { c->prof_names.clear(); c->prof_ms.clear(); c->prof_n.clear(); c->ring_used = 0; }
    return CS_OK;
}

int cs_gpu_profile_entry(cs_gpu_ctx* c, int i, char* name, int cap, double* total_ms, int64_t* launches)
{
    if (!c) return CS_E_ARG;
    prof_flush(c);
    if (i < 0 || i >= (int)c->prof_names.size()) return CS_E_RANGE;
    if (name && cap > 0) snprintf(name, cap, "%s", c->prof_names[i]);
    if (total_ms) *total_ms = c->prof_ms[i];
    if (launches) *launches = c->prof_n[i];
    return CS_OK;
}

int cs_gpu_sync(cs_gpu_ctx* c)
{
    if (!c) return CS_E_ARG;
    CK(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

int cs_gpu_get_counters(cs_gpu_ctx* c, cs_counters* out)
{
    if (!c || !out) return CS_E_ARG;
    DevPop& d = c->d;
    CK(cudaMemsetAsync(d.C, 0, 5 * sizeof(int64_t), c->stream));  // S..D recomputed below
    LAUNCH(k_cell_totals, 64, kThreads, d);
    CK(cudaMemcpyAsync(out, d.C, sizeof(cs_counters), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (out->err_queue_overflow || out->err_spatial_tries || out->err_kernel_range)
        return set_err(c, CS_E_OVERFLOW, "bounded device loop gave up (spatial %lld, queue %lld, kernel range %lld)",
                       (long long)out->err_spatial_tries, (long long)out->err_queue_overflow, (long long)out->err_kernel_range);
    return CS_OK;
}

// The cell counts and the counter block together, waited for once: what the
// reference's RecordSample reads at every output step.  From page-locked buffers
// (cs_host_alloc) the six copies run at the link's rate.
int cs_gpu_get_sample(cs_gpu_ctx* c, int32_t* S, int32_t* L, int32_t* I, int32_t* R, int32_t* D, cs_counters* out)
{
    if (!c || !out) return CS_E_ARG;
    DevPop& d = c->d;
    const size_t n = sizeof(int32_t) * d.NC;
    if (S && L == S + d.NC && I == L + d.NC && R == I + d.NC && D == R + d.NC) {
        CK(cudaMemcpyAsync(S, d.S, 5 * n, cudaMemcpyDeviceToHost, c->stream));   // the five arrays lie side by side
    } else {
        if (S) CK(cudaMemcpyAsync(S, d.S, n, cudaMemcpyDeviceToHost, c->stream));
        if (L) CK(cudaMemcpyAsync(L, d.L, n, cudaMemcpyDeviceToHost, c->stream));
        if (I) CK(cudaMemcpyAsync(I, d.I, n, cudaMemcpyDeviceToHost, c->stream));
        if (R) CK(cudaMemcpyAsync(R, d.R, n, cudaMemcpyDeviceToHost, c->stream));
        if (D) CK(cudaMemcpyAsync(D, d.D, n, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaMemsetAsync(d.C, 0, 5 * sizeof(int64_t), c->stream));  // S..D recomputed below
    LAUNCH(k_cell_totals, 64, kThreads, d);
    CK(cudaMemcpyAsync(out, d.C, sizeof(cs_counters), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (out->err_queue_overflow || out->err_spatial_tries || out->err_kernel_range)
        return set_err(c, CS_E_OVERFLOW, "bounded device loop gave up (spatial %lld, queue %lld, kernel range %lld)",
                       (long long)out->err_spatial_tries, (long long)out->err_queue_overflow, (long long)out->err_kernel_range);
    return CS_OK;
}

// S, L, I, R, D of every cell as 16-bit values side by side: half the bytes of
// cs_gpu_get_sample's copy, for populations whose cells hold at most 65,535 people.
__global__ void k_pack_cells16(DevPop d, uint16_t* __restrict__ out)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.NC; c += gridDim.x * blockDim.x) {
        out[c] = (uint16_t)d.S[c];
        out[d.NC + c] = (uint16_t)d.L[c];
        out[2 * d.NC + c] = (uint16_t)d.I[c];
        out[3 * d.NC + c] = (uint16_t)d.R[c];
        out[4 * d.NC + c] = (uint16_t)d.D[c];
    }
}

// The counter block (S..D left 0) followed by S, L, I, R, D of every cell as 16-bit
// values, written by one kernel into one device buffer: one copy per sample.
__global__ void k_pack_sample(DevPop d, unsigned char* __restrict__ out)
{
    if (blockIdx.x == 0) {   // the counters, 8-byte words, S..D (the first five) zero
        const int64_t* src = reinterpret_cast<const int64_t*>(d.C);
        int64_t* dst = reinterpret_cast<int64_t*>(out);
        for (int k = threadIdx.x; k < (int)(sizeof(cs_counters) / 8); k += blockDim.x) dst[k] = k < 5 ? 0 : src[k];
    }
    uint16_t* cells = reinterpret_cast<uint16_t*>(out + sizeof(cs_counters));
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.NC; c += gridDim.x * blockDim.x) {
        cells[c] = (uint16_t)d.S[c];
        cells[d.NC + c] = (uint16_t)d.L[c];
        cells[2 * d.NC + c] = (uint16_t)d.I[c];
        cells[3 * d.NC + c] = (uint16_t)d.R[c];
        cells[4 * d.NC + c] = (uint16_t)d.D[c];
    }
}

size_t cs_gpu_sample_packed_bytes(const cs_gpu_ctx* c)
{
    return c ? sizeof(cs_counters) + sizeof(uint16_t) * 5 * (size_t)c->d.NC : 0;
}

int cs_gpu_sample_packed_begin(cs_gpu_ctx* c, void* buf, size_t bytes)
{
    if (!c || !buf) return CS_E_ARG;
    DevPop& d = c->d;
    const size_t need = cs_gpu_sample_packed_bytes(c);
    if (bytes < need) return set_err(c, CS_E_ARG, "sample_packed: %zu bytes, %zu needed", bytes, need);
    if (c->max_cell_people > 65535)
        return set_err(c, CS_E_RANGE, "sample_packed: a cell holds %d people, more than 16 bits count",
                       c->max_cell_people);
    if (!c->packed) CK(cudaMalloc(&c->packed, need));
    LAUNCH(k_pack_sample, (d.NC + kThreads - 1) / kThreads, kThreads, d, (unsigned char*)c->packed);
    CK(cudaMemcpyAsync(buf, c->packed, need, cudaMemcpyDeviceToHost, c->stream));
    return CS_OK;
}

int cs_gpu_sample_packed_end(cs_gpu_ctx* c, const void* buf)
{
    if (!c || !buf) return CS_E_ARG;
    CK(cudaStreamSynchronize(c->stream));
    const cs_counters* out = (const cs_counters*)buf;
    if (out->err_queue_overflow || out->err_spatial_tries || out->err_kernel_range)
        return set_err(c, CS_E_OVERFLOW, "bounded device loop gave up (spatial %lld, queue %lld, kernel range %lld)",
                       (long long)out->err_spatial_tries, (long long)out->err_queue_overflow, (long long)out->err_kernel_range);
    return CS_OK;
}

int cs_gpu_get_sample_packed(cs_gpu_ctx* c, void* buf, size_t bytes)
{
    const int r = cs_gpu_sample_packed_begin(c, buf, bytes);
    return r ? r : cs_gpu_sample_packed_end(c, buf);
}

int cs_gpu_get_sample16(cs_gpu_ctx* c, uint16_t* cells, cs_counters* out)
{
    if (!c || !cells || !out) return CS_E_ARG;
    DevPop& d = c->d;
    if (c->max_cell_people > 65535)
        return set_err(c, CS_E_RANGE, "get_sample16: a cell holds %d people, more than 16 bits count",
                       c->max_cell_people);
    if (!c->pack16) CK(cudaMalloc(&c->pack16, sizeof(uint16_t) * 5 * (size_t)d.NC));
    LAUNCH(k_pack_cells16, (d.NC + kThreads - 1) / kThreads, kThreads, d, (uint16_t*)c->pack16);
    CK(cudaMemcpyAsync(cells, c->pack16, sizeof(uint16_t) * 5 * (size_t)d.NC, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemsetAsync(d.C, 0, 5 * sizeof(int64_t), c->stream));  // S..D recomputed below
    LAUNCH(k_cell_totals, 64, kThreads, d);
    CK(cudaMemcpyAsync(out, d.C, sizeof(cs_counters), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (out->err_queue_overflow || out->err_spatial_tries || out->err_kernel_range)
        return set_err(c, CS_E_OVERFLOW, "bounded device loop gave up (spatial %lld, queue %lld, kernel range %lld)",
                       (long long)out->err_spatial_tries, (long long)out->err_queue_overflow, (long long)out->err_kernel_range);
    return CS_OK;
}

void* cs_host_alloc(size_t bytes)
{
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
    return p;
}

void cs_host_free(void* p)
{
    if (p) cudaFreeHost(p);
}

int cs_gpu_get_cell_counts(cs_gpu_ctx* c, int32_t* S, int32_t* L, int32_t* I, int32_t* R, int32_t* D)
{
    if (!c) return CS_E_ARG;
    size_t n = sizeof(int32_t) * c->d.NC;
    if (S) CK(cudaMemcpyAsync(S, c->d.S, n, cudaMemcpyDeviceToHost, c->stream));
    if (L) CK(cudaMemcpyAsync(L, c->d.L, n, cudaMemcpyDeviceToHost, c->stream));
    if (I) CK(cudaMemcpyAsync(I, c->d.I, n, cudaMemcpyDeviceToHost, c->stream));
    if (R) CK(cudaMemcpyAsync(R, c->d.R, n, cudaMemcpyDeviceToHost, c->stream));
    if (D) CK(cudaMemcpyAsync(D, c->d.D, n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CS_OK;
}

// ------------------------------------------------------- state transfer
__global__ void k_unpack_hot(DevPop d, int8_t* inf, uint8_t* sev, uint8_t* fl, uint16_t* lt, uint16_t* as, uint16_t* ae,
                             uint16_t* iso, uint16_t* qs, float* infn, float* susc)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.N; p += gridDim.x * blockDim.x) {
        PersonHot h = d.hot[p];
        if (inf) inf[p] = h.inf;
        if (sev) sev[p] = h.sev;
        if (fl) fl[p] = h.dflags;
        if (lt) lt[p] = h.latent_time;
        if (as) as[p] = h.absent_start;
        if (ae) ae[p] = h.absent_stop;
        if (iso) iso[p] = h.isolation_start;
        if (qs) qs[p] = h.quar_start;
        if (infn) infn[p] = h.infness;
        if (susc) susc[p] = h.susc;
    }
}

__global__ void k_pack_hot(DevPop d, const int8_t* inf, const uint8_t* sev, const uint8_t* fl, const uint16_t* lt,
                           const uint16_t* as, const uint16_t* ae, const uint16_t* iso, const uint16_t* qs,
                           const float* infn, const float* susc)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.N; p += gridDim.x * blockDim.x) {
        PersonHot h = d.hot[p];
        h.inf = inf[p]; h.sev = sev[p]; h.dflags = fl[p]; h.latent_time = lt[p]; h.absent_start = as[p];
        h.absent_stop = ae[p]; h.isolation_start = iso[p]; h.quar_start = qs[p]; h.infness = infn[p]; h.susc = susc[p];
        d.hot[p] = h;
    }
}

// Device staging of the ten per-person fields that PersonHot packs, for state
// transfers: one buffer per context, allocated on first use and kept, so repeated
// uploads and downloads allocate nothing.
struct XferSlices {
    int8_t* inf; uint8_t* sev; uint8_t* fl; uint16_t *lt, *as, *ae, *iso, *qs; float *infn, *susc;
};

static int xfer_slices(cs_gpu_ctx* c, XferSlices* x)
{
    const size_t N = c->d.N;
    const size_t sizes[10] = {N, N, N, 2 * N, 2 * N, 2 * N, 2 * N, 2 * N, 4 * N, 4 * N};
    size_t ofs[10], total = 0;
    for (int k = 0; k < 10; k++) { ofs[k] = total; total += (sizes[k] + 255) / 256 * 256; }
    if (!c->xfer) CK(cudaMalloc(&c->xfer, total));
    char* b = (char*)c->xfer;
    x->inf = (int8_t*)(b + ofs[0]); x->sev = (uint8_t*)(b + ofs[1]); x->fl = (uint8_t*)(b + ofs[2]);
    x->lt = (uint16_t*)(b + ofs[3]); x->as = (uint16_t*)(b + ofs[4]); x->ae = (uint16_t*)(b + ofs[5]);
    x->iso = (uint16_t*)(b + ofs[6]); x->qs = (uint16_t*)(b + ofs[7]);
    x->infn = (float*)(b + ofs[8]); x->susc = (float*)(b + ofs[9]);
    return CS_OK;
}

int cs_gpu_download_state(cs_gpu_ctx* c, const cs_state_view* v)
{
    if (!c || !v) return CS_E_ARG;
    DevPop& d = c->d;
    size_t N = d.N, NC = d.NC;
    // person record fields go through the staging slices (10 fields)
    XferSlices x;
    int r0 = xfer_slices(c, &x);
    if (r0) return r0;
    int8_t* dinf = v->inf ? x.inf : nullptr;
    uint8_t* dsev = v->severity ? x.sev : nullptr;
    uint8_t* dfl = v->flags ? x.fl : nullptr;
    uint16_t* dlt = v->latent_time ? x.lt : nullptr;
    uint16_t* das = v->absent_start_time ? x.as : nullptr;
    uint16_t* dae = v->absent_stop_time ? x.ae : nullptr;
    uint16_t* diso = v->isolation_start_time ? x.iso : nullptr;
    uint16_t* dqs = v->quar_start_time ? x.qs : nullptr;
    float* dinfn = v->infectiousness ? x.infn : nullptr;
    float* dsusc = v->susc ? x.susc : nullptr;
    k_unpack_hot<<<c->grid, kThreads, 0, c->stream>>>(d, dinf, dsev, dfl, dlt, das, dae, diso, dqs, dinfn, dsusc);
    c->launches++;
    int rc = CS_OK;
#define DL(dst, src, bytes) do { if (v->dst && src) { cudaError_t e_ = cudaMemcpyAsync(v->dst, src, bytes, cudaMemcpyDeviceToHost, c->stream); if (e_ != cudaSuccess) rc = set_err(c, CS_E_CUDA, "download: %s", cudaGetErrorString(e_)); } } while (0)
    DL(inf, dinf, N); DL(severity, dsev, N); DL(flags, dfl, N); DL(latent_time, dlt, 2 * N);
    DL(absent_start_time, das, 2 * N); DL(absent_stop_time, dae, 2 * N); DL(isolation_start_time, diso, 2 * N);
    DL(quar_start_time, dqs, 2 * N); DL(infectiousness, dinfn, 4 * N); DL(susc, dsusc, 4 * N);
    DL(infection_time, d.infection_time, 2 * N); DL(recovery_or_death_time, d.recovery_time, 2 * N);
    DL(SARI_time, d.sari_time, 2 * N); DL(Critical_time, d.critical_time, 2 * N); DL(Stepdown_time, d.stepdown_time, 2 * N);
    DL(detected_time, d.detected_time, 2 * N); DL(ProbAbsent, d.prob_absent, 4 * N); DL(ProbCare, d.prob_care, 4 * N);
    DL(infector, d.infector, 4 * N); DL(infect_type, d.infect_type, 2 * N); DL(listpos, d.listpos, 4 * N);
    DL(cell_S, d.S, 4 * NC); DL(cell_L, d.L, 4 * NC); DL(cell_I, d.I, 4 * NC); DL(cell_R, d.R, 4 * NC);
    DL(cell_D, d.D, 4 * NC); DL(cell_S0, d.S0, 4 * NC); DL(cell_tot_prob, d.tot_prob, 8 * NC); DL(cell_slots, d.slots, 4 * N);
#undef DL
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return set_err(c, CS_E_CUDA, "download sync: %s", cudaGetErrorString(e));
    return rc;
}

// The per-person arrays of a state upload for people [first, first + n), queued on
// the context's stream from the view's host arrays: the record fields into the
// staging slices (k_pack_hot packs them later), the rest into place.
static int upload_people_slice(cs_gpu_ctx* c, const cs_state_view* v, const XferSlices& x, size_t first, size_t n)
{
    DevPop& d = c->d;
    if (n == 0) return CS_OK;
#define SL(dst, src, w)                                                                                       \
    CK(cudaMemcpyAsync((char*)(dst) + (size_t)(w) * first, (const char*)v->src + (size_t)(w) * first,        \
                       (size_t)(w) * n, cudaMemcpyHostToDevice, c->stream))
    SL(x.inf, inf, 1); SL(x.sev, severity, 1); SL(x.fl, flags, 1); SL(x.lt, latent_time, 2);
    SL(x.as, absent_start_time, 2); SL(x.ae, absent_stop_time, 2); SL(x.iso, isolation_start_time, 2);
    SL(x.qs, quar_start_time, 2); SL(x.infn, infectiousness, 4); SL(x.susc, susc, 4);
    SL(d.infection_time, infection_time, 2); SL(d.recovery_time, recovery_or_death_time, 2);
    SL(d.sari_time, SARI_time, 2); SL(d.critical_time, Critical_time, 2); SL(d.stepdown_time, Stepdown_time, 2);
    SL(d.detected_time, detected_time, 2); SL(d.prob_absent, ProbAbsent, 4); SL(d.prob_care, ProbCare, 4);
    SL(d.infector, infector, 4); SL(d.infect_type, infect_type, 2); SL(d.listpos, listpos, 4);
#undef SL
    return CS_OK;
}

static bool people_fields(const cs_state_view* v)
{
    return v->inf && v->severity && v->flags && v->latent_time && v->absent_start_time && v->absent_stop_time &&
           v->isolation_start_time && v->quar_start_time && v->infectiousness && v->susc && v->infection_time &&
           v->recovery_or_death_time && v->SARI_time && v->Critical_time && v->Stepdown_time && v->detected_time &&
           v->ProbAbsent && v->ProbCare && v->infector && v->infect_type && v->listpos;
}

int cs_gpu_upload_people(cs_gpu_ctx* c, const cs_state_view* v, int64_t first, int64_t n)
{
    if (!c || !v) return CS_E_ARG;
    if (!people_fields(v)) return set_err(c, CS_E_ARG, "upload_people needs every per-person field of the view");
    if (first != (int64_t)c->people_sent || n < 0 || first + n > (int64_t)c->d.N)
        return set_err(c, CS_E_ARG, "upload_people: people [%lld, %lld) do not follow the %zu sent (of %d)",
                       (long long)first, (long long)(first + n), c->people_sent, c->d.N);
    XferSlices x;
    int r = xfer_slices(c, &x);
    if (r) return r;
    r = upload_people_slice(c, v, x, (size_t)first, (size_t)n);
    if (r) return r;
    c->people_sent += (size_t)n;
    return CS_OK;
}

int cs_gpu_upload_state(cs_gpu_ctx* c, uint64_t seed, const cs_state_view* v)
{
    if (!c || !v) return CS_E_ARG;
    DevPop& d = c->d;
    size_t N = d.N, NC = d.NC;
    if (!v->inf || !v->severity || !v->flags || !v->latent_time || !v->absent_start_time || !v->absent_stop_time ||
        !v->isolation_start_time || !v->quar_start_time || !v->infectiousness || !v->susc || !v->infection_time ||
        !v->recovery_or_death_time || !v->SARI_time || !v->Critical_time || !v->Stepdown_time || !v->detected_time ||
        !v->ProbAbsent || !v->ProbCare || !v->infector || !v->infect_type || !v->listpos || !v->cell_S || !v->cell_L ||
        !v->cell_I || !v->cell_R || !v->cell_D || !v->cell_S0 || !v->cell_tot_prob || !v->cell_slots)
        return set_err(c, CS_E_ARG, "upload_state needs every field of the view");
    XferSlices x;
    int r0 = xfer_slices(c, &x);
    if (r0) return r0;
    {   // the people cs_gpu_upload_people has not sent yet
        const size_t sent = c->people_sent;
        c->people_sent = 0;
        if (sent > N) return set_err(c, CS_E_STATE, "upload_state: %zu people sent ahead, %zu in the population", sent, N);
        r0 = upload_people_slice(c, v, x, sent, N - sent);
        if (r0) return r0;
    }
    int8_t* dinf = x.inf; uint8_t* dsev = x.sev; uint8_t* dfl = x.fl;
    uint16_t *dlt = x.lt, *das = x.as, *dae = x.ae, *diso = x.iso, *dqs = x.qs;
    float *dinfn = x.infn, *dsusc = x.susc;
    k_pack_hot<<<c->grid, kThreads, 0, c->stream>>>(d, dinf, dsev, dfl, dlt, das, dae, diso, dqs, dinfn, dsusc);
    c->launches++;
#define UL(src, dst, bytes) CK(cudaMemcpyAsync(dst, v->src, bytes, cudaMemcpyHostToDevice, c->stream))
    UL(cell_S, d.S, 4 * NC); UL(cell_L, d.L, 4 * NC); UL(cell_I, d.I, 4 * NC); UL(cell_R, d.R, 4 * NC);
    UL(cell_D, d.D, 4 * NC); UL(cell_S0, d.S0, 4 * NC); UL(cell_tot_prob, d.tot_prob, 8 * NC); UL(cell_slots, d.slots, 4 * N);
#undef UL
    CK(cudaMemsetAsync(d.mark, 0, N, c->stream));
    CK(cudaMemsetAsync(d.counts, 0, sizeof(int32_t) * kCntN, c->stream));
    CK(cudaMemsetAsync(d.cnt, 0, sizeof(int32_t) * d.NC, c->stream));
    CK(cudaMemsetAsync(d.C, 0, sizeof(cs_counters), c->stream));
    CK(cudaMemsetAsync(d.ev_init, 0xff, sizeof(int32_t), c->stream));   // next_ev from the uploaded times
    // the host seeded the run: its LocationInitialInfection is where radii start
    CK(cudaMemcpyAsync(d.rad_origin, c->hp.LocationInitialInfection, sizeof(double) * 2, cudaMemcpyHostToDevice,
                       c->stream));
    c->seed = seed;
    CK(cudaMemcpyAsync(c->d_seed, &c->seed, sizeof(c->seed), cudaMemcpyHostToDevice, c->stream));
    int r = reset_run_level(c, seed);
    if (r == CS_OK) r = rebuild_blocks(c);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (r) return r;
    if (e != cudaSuccess) return set_err(c, CS_E_CUDA, "upload sync: %s", cudaGetErrorString(e));
    c->run_started = true;
    return CS_OK;
}

}  // extern "C"

// ================================================ UpdateProbs without allocation
// cs_gpu_update_probs_static computes what cs_gpu_update_probs computes, with the
// same kernels in the same order, but takes its two grid-sized scratch arrays (S0
// laid out on the cell grid, and the per-cell numerators) and the row-used flags
// from one file-scope device array instead of the context's allocations.  It is
// for callers that must not allocate device memory when UpdateProbs runs: a
// process whose device memory is already reserved by another allocator's pool,
// where a further allocation fails; and a caller running beside other streams,
// where freeing scratch would synchronise the whole device.  Nothing in it calls
// an allocating routine; its limit is the fixed size of that array.
namespace {
constexpr size_t kStaticCells = CS_STATIC_MAX_GRID_CELLS;
constexpr size_t kStaticRows = CS_STATIC_MAX_GRID_ROWS;
constexpr size_t kStaticBytes = 2 * sizeof(float) * kStaticCells + kStaticRows;
}  // namespace

// [S0 on the grid: kStaticCells floats][numerators: kStaticCells floats][row flags]
static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

extern "C" int cs_gpu_update_probs_static(cs_gpu_ctx* c, int do_place)
{
    if (!c) return CS_E_ARG;
    DevPop& d = c->d;
    const cs_params& P = c->hp;
    const size_t G = (size_t)P.ncw * P.nch;
    if (G > kStaticCells || (size_t)P.nch > kStaticRows)
        return set_err(c, CS_E_RANGE,
                       "update_probs_static: %d x %d grid cells exceed its fixed scratch (%zu cells, %zu rows); "
                       "use cs_gpu_update_probs", P.ncw, P.nch, kStaticCells, kStaticRows);
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev != c->device)
        return set_err(c, CS_E_STATE, "update_probs_static: device %d is current, the context is on device %d",
                       dev, c->device);
    // The array's device address in the current context, looked up on every call
    // (the lookup allocates nothing): a context made after a device reset, or
    // another context on the same device, holds its own copy of the module.  The
    // first lookup in a context loads the library's module there, which is why the
    // first call should come before any stream capture.
    void* base = nullptr;
    {
        cudaError_t e = cudaGetSymbolAddress(&base, g_static_scratch);
        if (e != cudaSuccess || !base)
            return set_err(c, CS_E_CUDA, "update_probs_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    }
    float* S0g = (float*)base;
    float* Ag = S0g + kStaticCells;
    uint8_t* rowS = (uint8_t*)(Ag + kStaticCells);
    // The array still holds the previous call's values.  Grid positions without a
    // populated cell and rows without susceptibles must read zero; the numerators
    // are written in full by the row kernel.
    CK(cudaMemsetAsync(S0g, 0, sizeof(float) * G, c->stream));
    CK(cudaMemsetAsync(rowS, 0, P.nch, c->stream));
    const int cgrid = (d.NC + kThreads - 1) / kThreads;
    LAUNCH(k_update_S0, cgrid, kThreads, d, do_place);
    LAUNCH(k_grid_values, cgrid, kThreads, d, S0g, (float*)nullptr, rowS, (uint8_t*)nullptr);
    // All row chunks of a column block run in one block (grid z = 1): the chunked
    // form's per-chunk partial sums would need nchunks x G more floats of scratch.
    const TotProbGeom gm = tot_prob_geom(P.ncw, P.nch, false);
    dim3 grid;
    int tpb;
    tot_prob_launch_shape(P.ncw, P.nch, gm, &grid, &tpb);
    const size_t smem = gm.smem(false);
    int r = tot_prob_smem(c, false, smem);
    if (r) return r;
    if (c->prof) prof_begin(c, "k_tot_prob_rows_static");
    k_tot_prob_rows<false><<<grid, tpb, smem, c->stream>>>(d, S0g, nullptr, rowS, nullptr, Ag, nullptr, gm, c->Gtab);
    if (c->prof) prof_end(c);
    c->launches++;
    CK(cudaGetLastError());
    LAUNCH(k_tot_prob_finish, cgrid, kThreads, d, Ag, c->Bg);
    LAUNCH(k_block_S0, (d.NB + kThreads - 1) / kThreads, kThreads, d);
    LAUNCH(k_block_rows, (d.NB * 32 + kThreads - 1) / kThreads, kThreads, d);
    return CS_OK;
}
