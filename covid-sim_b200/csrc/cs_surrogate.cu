// Scenario surrogate: a small network mapping 8 intervention/transmission
// parameters to 365 days x 4 daily outputs, trained on trajectories of the GPU
// simulator and used to screen scenario sweeps.  No counterpart in the
// reference, which has no learned model; the layer definitions follow
// oracle/surrogate_ref.py, which the tests use as the reference.
//
//   x [B, 8] -> 4 x (Linear 512 + ReLU) -> Linear 256 + ReLU -> Linear 2944 + ReLU
//   -> [B, 46, 64] -> 3 x (nearest upsample x2 -> Conv1d k=5 pad 2) 64 -> 64 -> 32 -> 4
//      (ReLU after the first two) -> first 365 time points -> y [B, 365, 4]
//
// Every matrix product (the linear layers, and the convolutions as products of
// im2col columns with the weights) runs on the tensor cores in BF16 with FP32
// accumulation: C[M,N] = A[M,K] * B[N,K]^T, both operands row-major BF16 with
// every dimension padded to a multiple of 64 (pads hold zeros, so they add
// nothing).  Master weights, gradients and Adam moments are FP32; the BF16
// weight copies are refreshed after each update.  Gradients are deterministic:
// every reduction has a fixed order.
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "covidsim_b200.h"

typedef __nv_bfloat16 bf16;

namespace sur {

constexpr int kIn = 8, kWidth = 512, kLatent = 256, kT0 = 46, kC0 = 64, kTap = 5;
constexpr int kTOut = 365, kNOut = 4, kCh = 64;   // conv activations keep 64 channel slots

inline int up64(int x) { return (x + 63) / 64 * 64; }

// ------------------------------------------------------------------- GEMM
// C[M,N] = A[M,K] * B[N,K]^T (+ bias[n]) (ReLU), FP32 out and/or BF16 out.
// M, N multiples of 64; K multiple of 32; leading dimensions multiples of 8.
// 128 threads: a 2 x 2 grid of warps, each a 32 x 32 tile of m16n8k16 products.
__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Split K (gridDim.z > 1): slice z covers k in [z * kchunk, min(K, (z + 1) * kchunk))
// and writes its partial product to C + z * cstride (no bias, ReLU or BF16 output).
__global__ void __launch_bounds__(128) k_gemm_nt(const bf16* __restrict__ A, int lda, const bf16* __restrict__ B, int ldb,
                                                 float* __restrict__ C, int ldc, bf16* __restrict__ Cb, int ldcb,
                                                 const float* __restrict__ bias, int relu, int K, int kchunk, size_t cstride)
{
    if (gridDim.z > 1) {
        const int z = blockIdx.z;
        A += (size_t)z * kchunk;
        B += (size_t)z * kchunk;
        C += (size_t)z * cstride;
        K = min(kchunk, K - z * kchunk);
    }
    __shared__ __align__(16) bf16 As[64][40];
    __shared__ __align__(16) bf16 Bs[64][40];
    const int bm = blockIdx.y * 64, bn = blockIdx.x * 64;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, tq = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;
    for (int k0 = 0; k0 < K; k0 += 32) {
        for (int i = threadIdx.x; i < 256; i += 128) {
            int r = i >> 2, c = (i & 3) * 8;
            *reinterpret_cast<uint4*>(&As[r][c]) = *reinterpret_cast<const uint4*>(A + (size_t)(bm + r) * lda + k0 + c);
            *reinterpret_cast<uint4*>(&Bs[r][c]) = *reinterpret_cast<const uint4*>(B + (size_t)(bn + r) * ldb + k0 + c);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 32; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; mi++) {
                int r = wm + mi * 16 + g;
                a[mi][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + tq * 2]);
                a[mi][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + tq * 2]);
                a[mi][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + tq * 2 + 8]);
                a[mi][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + tq * 2 + 8]);
            }
#pragma unroll
            for (int ni = 0; ni < 4; ni++) {
                int n = wn + ni * 8 + g;
                b[ni][0] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + tq * 2]);
                b[ni][1] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + tq * 2 + 8]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++) mma_bf16(acc[mi][ni], a[mi], b[ni]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int r = bm + wm + mi * 16 + g + h * 8;
                int c = bn + wn + ni * 8 + tq * 2;
                float v0 = acc[mi][ni][2 * h], v1 = acc[mi][ni][2 * h + 1];
                if (bias) { v0 += bias[c]; v1 += bias[c + 1]; }
                if (relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
                if (C) { C[(size_t)r * ldc + c] = v0; C[(size_t)r * ldc + c + 1] = v1; }
                if (Cb) *reinterpret_cast<__nv_bfloat162*>(Cb + (size_t)r * ldcb + c) = __floats2bfloat162_rn(v0, v1);
            }
}

// ------------------------------------------------------- tcgen05 GEMM
// The same product on the 5th-generation tensor cores.  A block computes a 128 x BN
// tile: its 128 threads stage 64-wide K slices of A and B in shared memory in the
// K-major 128-byte-swizzled layout (two stages, so the loads of slice k+1 overlap
// the products of slice k), one thread issues the tcgen05.mma instructions
// (M = 128, N = BN, K = 16 each, BF16 in, FP32 accumulator in tensor memory) and
// commits them to the stage's mbarrier, and after the last slice every warp reads
// its 32 accumulator rows from tensor memory for the epilogue (bias, ReLU, FP32
// and/or BF16 stores).  Rows of A past M are staged as zeros and not stored.
// Every wait is bounded: on a give-up the block records it in *err, waits (bounded)
// for its issued products, frees its tensor memory and returns.
namespace tc {

constexpr int BM = 128, BK = 64;          // BK bf16 = 128 bytes, one swizzle row
constexpr unsigned kSpin = 1u << 22;      // try_wait rounds before a wait gives up

__host__ __device__ constexpr size_t smem_bytes(int BN) { return 1024 + 2 * (size_t)(BM + BN) * BK * 2; }

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand: start
// address, leading offset 16 B (unused by this layout), 8-row groups 1024 B apart,
// descriptor version 1, layout SWIZZLE_128B.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(saddr(bar)), "r"(parity) : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    for (unsigned i = 0; i < kSpin; i++)
        if (mbar_try(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                 :: "r"(d_tmem), "l"(a), "l"(b), "r"(id), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ void ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// rows x 64 BF16 of a row-major matrix (row stride ld elements, rows from r0, k from
// k0) into a 128-byte-swizzled stage: 16-byte chunk j of row r lands at
// r * 128 + ((j ^ (r & 7)) * 16).  Rows at or past nrows are zero.
__device__ __forceinline__ void stage_rows(unsigned char* dst, const bf16* __restrict__ src, int ld, int r0, int nrows,
                                           int k0, int rows)
{
    for (int i = threadIdx.x; i < rows * 8; i += blockDim.x) {
        const int r = i >> 3, j = i & 7;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (r0 + r < nrows) v = *reinterpret_cast<const uint4*>(src + (size_t)(r0 + r) * ld + k0 + j * 8);
        *reinterpret_cast<uint4*>(dst + r * 128 + ((j ^ (r & 7)) << 4)) = v;
    }
}

// The A operand of a convolution read straight from its input H [Bn*T, kCh] (no
// column matrix): row m = b*2T + t, column k = tap*Cin + c holds
// H[b*T + (t+tap-2)/2, c] when 0 <= t+tap-2 < 2T, else zero (as k_im2col_up).  Cin is
// a multiple of 8, so a 16-byte chunk never straddles two taps.
__device__ __forceinline__ void stage_conv_rows(unsigned char* dst, const bf16* __restrict__ H, int T, int Cin, int r0,
                                                int nrows, int k0)
{
    for (int i = threadIdx.x; i < BM * 8; i += blockDim.x) {
        const int r = i >> 3, j = i & 7;
        uint4 v = make_uint4(0, 0, 0, 0);
        const int m = r0 + r, k = k0 + j * 8;
        const int tap = k / Cin;
        if (m < nrows && tap < kTap) {
            const int b = m / (2 * T), t = m - b * 2 * T, u = t + tap - kTap / 2;
            if (u >= 0 && u < 2 * T)
                v = *reinterpret_cast<const uint4*>(H + ((size_t)b * T + (u >> 1)) * kCh + (k - tap * Cin));
        }
        *reinterpret_cast<uint4*>(dst + r * 128 + ((j ^ (r & 7)) << 4)) = v;
    }
}

}  // namespace tc

// C[M,N] = A[M,K] B[N,K]^T (+ bias) (ReLU) on tcgen05; N a multiple of BN, K of 64;
// split K as k_gemm_nt (gridDim.z slices of kchunk, partial products at C + z * cstride).
// With H set, A is the column matrix of a convolution of H (hT time points, hCin
// channels), generated while staging (not split).
template <int BN>
__global__ void __launch_bounds__(128) k_gemm_tc(const bf16* __restrict__ A, int lda, const bf16* __restrict__ B, int ldb,
                                                 float* __restrict__ C, int ldc, bf16* __restrict__ Cb, int ldcb,
                                                 const float* __restrict__ bias, int relu, int M, int K, int kchunk,
                                                 size_t cstride, int* err, const bf16* __restrict__ H, int hT, int hCin)
{
    using namespace tc;
    extern __shared__ unsigned char smem_raw[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tmem_base;
    __shared__ int s_ok;
    unsigned char* base = smem_raw + ((1024 - (saddr(smem_raw) & 1023)) & 1023);
    unsigned char* As = base;                          // [2][BM * 128 B]
    unsigned char* Bs = base + 2 * BM * BK * 2;        // [2][BN * 128 B]
    if (gridDim.z > 1) {
        const int z = blockIdx.z;
        A += (size_t)z * kchunk;
        B += (size_t)z * kchunk;
        C += (size_t)z * cstride;
        K = min(kchunk, K - z * kchunk);
    }
    const int bm = blockIdx.y * BM, bn = blockIdx.x * BN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(saddr(&tmem_base)), "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(saddr(&bar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(saddr(&bar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_ok = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tm = tmem_base;
    const int nk = K / BK;
    int issued = 0;                    // slices whose products were committed
    for (int kc = 0; kc < nk; kc++) {
        const int st = kc & 1;
        if (kc >= 2) {                 // the products that read this stage are done
            if (threadIdx.x == 0 && !mbar_wait(&bar[st], ((kc - 2) >> 1) & 1)) s_ok = 0;
            __syncthreads();
            if (!s_ok) break;
        }
        if (H) stage_conv_rows(As + st * BM * 128, H, hT, hCin, bm, M, kc * BK);
        else stage_rows(As + st * BM * 128, A, lda, bm, M, kc * BK, BM);
        stage_rows(Bs + st * BN * 128, B, ldb, bn, 1 << 30, kc * BK, BN);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = saddr(As + st * BM * 128), b0 = saddr(Bs + st * BN * 128);
#pragma unroll
            for (int k = 0; k < BK / 16; k++)
                tc::mma(tm, sdesc(a0 + 32 * k), sdesc(b0 + 32 * k), idesc(BM, BN), (kc | k) != 0);
            commit(&bar[st]);
        }
        issued = kc + 1;
    }
    // the last committed slice's barrier completes after all earlier products
    if (threadIdx.x == 0 && issued > 0 && !mbar_wait(&bar[(issued - 1) & 1], ((issued - 1) >> 1) & 1)) s_ok = 0;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (s_ok && issued == nk) {
        const int row = bm + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            uint32_t r[32];
            ld32(tm + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            if (row < M) {
                const int col = bn + c0;
#pragma unroll
                for (int j = 0; j < 32; j += 2) {
                    float v0 = __uint_as_float(r[j]), v1 = __uint_as_float(r[j + 1]);
                    if (nk == 0) v0 = v1 = 0.f;
                    if (bias) { v0 += bias[col + j]; v1 += bias[col + j + 1]; }
                    if (relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
                    if (C) *reinterpret_cast<float2*>(C + (size_t)row * ldc + col + j) = make_float2(v0, v1);
                    if (Cb) *reinterpret_cast<__nv_bfloat162*>(Cb + (size_t)row * ldcb + col + j) = __floats2bfloat162_rn(v0, v1);
                }
            }
        }
    } else if (threadIdx.x == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tm), "r"(BN));
}

// C[r, c] = sum over the slices z, in ascending order, of part[z][r, c] ([M, N] each),
// then the product's epilogue (bias, ReLU, FP32 and/or BF16 stores).
__global__ void k_splitk_reduce(const float* __restrict__ part, int nsplit, int M, int N, float* __restrict__ C, int ldc,
                                bf16* __restrict__ Cb, int ldcb, const float* __restrict__ bias, int relu)
{
    const size_t MN = (size_t)M * N;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < MN; e += (size_t)gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int z = 0; z < nsplit; z++) acc += part[z * MN + e];
        const size_t r = e / N, c = e % N;
        if (bias) acc += bias[c];
        if (relu) acc = fmaxf(acc, 0.f);
        if (C) C[r * ldc + c] = acc;
        if (Cb) Cb[r * ldcb + c] = __float2bfloat16_rn(acc);
    }
}

// out[c, r] = in[r, c] for an R x Cc block (both multiples of 32).
__global__ void k_transpose(const bf16* __restrict__ in, int ldi, bf16* __restrict__ out, int ldo, int R, int Cc)
{
    __shared__ bf16 t[32][33];
    int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) t[i][threadIdx.x] = in[(size_t)(r0 + i) * ldi + c0 + threadIdx.x];
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) out[(size_t)(c0 + i) * ldo + r0 + threadIdx.x] = t[threadIdx.x][i];
}

// Columns of the x2 upsampled, zero-padded input: cols[b*2T + t, k*Cin + c] =
// H[b*T + (t+k-2)/2, c] for 0 <= t+k-2 < 2T (channel stride kCh), zero elsewhere
// (and in the pad columns up to ldc).
__global__ void k_im2col_up(const bf16* __restrict__ H, int Bn, int T, int Cin, bf16* __restrict__ cols, int ldc)
{
    const size_t rows = (size_t)Bn * 2 * T;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < rows * ldc; e += (size_t)gridDim.x * blockDim.x) {
        size_t row = e / ldc;
        int col = (int)(e % ldc);
        bf16 v = __float2bfloat16(0.f);
        if (col < kTap * Cin) {
            int k = col / Cin, c = col % Cin;
            int b = (int)(row / (2 * T)), t = (int)(row % (2 * T));
            int u = t + k - kTap / 2;
            if (u >= 0 && u < 2 * T) v = H[((size_t)b * T + (u >> 1)) * kCh + c];
        }
        cols[e] = v;
    }
}

// The transposed column matrix, colsT[k, m] = cols[m, k] of k_im2col_up, for m < M
// (= Bn*2T) and k < ldk (columns past kTap*Cin zero), through a 32 x 32 shared tile
// so that both the reads of H and the writes are coalesced.
__global__ void k_im2colT_up(const bf16* __restrict__ H, int T, int Cin, bf16* __restrict__ colsT, int M)
{
    __shared__ bf16 tile[32][34];
    const int m0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const int m = m0 + q, k = k0 + threadIdx.x;
        bf16 v = __float2bfloat16(0.f);
        const int tap = k / Cin;
        if (tap < kTap) {
            const int b = m / (2 * T), t = m - b * 2 * T, u = t + tap - kTap / 2;
            if (u >= 0 && u < 2 * T) v = H[((size_t)b * T + (u >> 1)) * kCh + (k - tap * Cin)];
        }
        tile[q][threadIdx.x] = v;
    }
    __syncthreads();
    for (int q = threadIdx.y; q < 32; q += blockDim.y)
        colsT[(size_t)(k0 + q) * M + m0 + threadIdx.x] = tile[threadIdx.x][q];
}

// Adjoint of k_im2col_up, fused with the ReLU mask of H: for channel c < Cin,
// dz[b*T+s, c] = (H > 0) * sum over u in {2s, 2s+1}, k of dcols[b*2T + u-k+2, k*Cin + c];
// FP32 and BF16 copies; channels >= Cin are zero.
__global__ void k_col2im_up_relu(const float* __restrict__ dcols, int ldd, int Bn, int T, int Cin,
                                 const bf16* __restrict__ H, float* __restrict__ dz, bf16* __restrict__ dzb)
{
    const size_t n = (size_t)Bn * T * kCh;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        int c = (int)(e % kCh);
        size_t bs = e / kCh;
        int b = (int)(bs / T), s = (int)(bs % T);
        float acc = 0.f;
        if (c < Cin) {
            for (int du = 0; du < 2; du++) {
                int u = 2 * s + du;
                for (int k = 0; k < kTap; k++) {
                    int t = u - k + kTap / 2;
                    if (t >= 0 && t < 2 * T) acc += dcols[((size_t)b * 2 * T + t) * ldd + k * Cin + c];
                }
            }
            if (!(__bfloat162float(H[e]) > 0.f)) acc = 0.f;
        }
        dz[e] = acc;
        dzb[e] = __float2bfloat16(acc);
    }
}

// dz = dh * (h > 0), FP32 and BF16 copies (dense [rows, ld]).
__global__ void k_relu_back(const float* __restrict__ dh, const bf16* __restrict__ h, size_t n, float* __restrict__ dz,
                            bf16* __restrict__ dzb)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        float v = __bfloat162float(h[e]) > 0.f ? dh[e] : 0.f;
        dz[e] = v;
        dzb[e] = __float2bfloat16(v);
    }
}

// Column sums of dz [rows, ld] in a fixed order: part[chunk, col] over row chunks
// of 256, then the chunks in ascending order.
// Column sums of dz [rows, ld] in a fixed order.  Block (x, y) covers 32 columns
// and row chunk y of kColChunk rows; its 8 row lanes each sum every 8th row, then
// a shared-memory tree adds the lanes: part[y, col].  The final pass adds the
// chunks the same way.
constexpr int kColChunk = 2048;
__device__ __forceinline__ float lanes_tree(float v, float (*sh)[33])
{
    sh[threadIdx.y][threadIdx.x] = v;
    __syncthreads();
    for (int o = 4; o > 0; o >>= 1) {
        if ((int)threadIdx.y < o) sh[threadIdx.y][threadIdx.x] += sh[threadIdx.y + o][threadIdx.x];
        __syncthreads();
    }
    return sh[0][threadIdx.x];
}
__global__ void k_colsum_part(const float* __restrict__ dz, int rows, int ld, float* __restrict__ part)
{
    __shared__ float sh[8][33];
    const int col = blockIdx.x * 32 + threadIdx.x;
    const int r0 = blockIdx.y * kColChunk, r1 = min(rows, r0 + kColChunk);
    float v = 0.f;
    if (col < ld)
        for (int r = r0 + threadIdx.y; r < r1; r += 8) v += dz[(size_t)r * ld + col];
    v = lanes_tree(v, sh);
    if (threadIdx.y == 0 && col < ld) part[(size_t)blockIdx.y * ld + col] = v;
}
__global__ void k_colsum_final(const float* __restrict__ part, int nchunks, int ld, float* __restrict__ out)
{
    __shared__ float sh[8][33];
    const int col = blockIdx.x * 32 + threadIdx.x;
    float v = 0.f;
    if (col < ld)
        for (int q = threadIdx.y; q < nchunks; q += 8) v += part[(size_t)q * ld + col];
    v = lanes_tree(v, sh);
    if (threadIdx.y == 0 && col < ld) out[col] = v;
}

// Loss terms and the output gradient: y is [B*368, 64] (channels < 4 used), target
// [n, 365, 4]; rows of samples >= n and time points >= 365 get zero gradient.
__global__ void k_mse(const float* __restrict__ y, const float* __restrict__ target, int n, int Bp, float scale,
                      float* __restrict__ dy, float* __restrict__ sq)
{
    const int T = 2 * 2 * 2 * kT0;   // 368
    const size_t total = (size_t)Bp * T * kCh;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int c = (int)(e % kCh);
        size_t bt = e / kCh;
        int b = (int)(bt / T), t = (int)(bt % T);
        float g = 0.f;
        if (c < kNOut && t < kTOut && b < n) {
            float d = y[e] - target[((size_t)b * kTOut + t) * kNOut + c];
            g = 2.f * d * scale;
            sq[((size_t)b * kTOut + t) * kNOut + c] = d * d;
        }
        dy[e] = g;
    }
}

// Adam (Kingma & Ba, 2015) on FP32 master weights; refreshes the BF16 copy.
// Sum of v[0..n) in a fixed order: block b sums its contiguous range (strided by
// thread, then a shared-memory tree), the final pass adds the blocks in order.
__global__ void k_sum_part(const float* __restrict__ v, size_t n, double* __restrict__ part)
{
    __shared__ double sh[256];
    const size_t per = (n + gridDim.x - 1) / gridDim.x, b0 = blockIdx.x * per, e0 = min(n, b0 + per);
    double acc = 0.0;
    for (size_t e = b0 + threadIdx.x; e < e0; e += blockDim.x) acc += v[e];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_sum_final(const double* __restrict__ part, int n, double* __restrict__ out)
{
    __shared__ double sh[256];
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a += part[i];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                       bf16* __restrict__ wb, size_t n, float lr, float b1, float b2, float eps, float c1, float c2, float wd)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        float gi = g[e];
        float mi = b1 * m[e] + (1.f - b1) * gi;
        float vi = b2 * v[e] + (1.f - b2) * gi * gi;
        m[e] = mi;
        v[e] = vi;
        // decoupled weight decay (Loshchilov & Hutter, "Decoupled weight decay regularization", 2019)
        float wi = w[e] * (1.f - lr * wd) - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[e] = wi;
        if (wb) wb[e] = __float2bfloat16(wi);
    }
}

__global__ void k_to_bf16(const float* __restrict__ in, bf16* __restrict__ out, size_t n)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        out[e] = __float2bfloat16(in[e]);
}

// x [n, 8] -> BF16 [Bp, 64] (zeros beyond)
__global__ void k_load_x(const float* __restrict__ x, int n, int Bp, bf16* __restrict__ xb)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Bp * 64; e += gridDim.x * blockDim.x) {
        int b = e / 64, c = e % 64;
        xb[e] = __float2bfloat16((b < n && c < kIn) ? x[b * kIn + c] : 0.f);
    }
}

// y [B*368, 64] -> out [n, 365, 4]
__global__ void k_store_y(const float* __restrict__ y, int n, float* __restrict__ out)
{
    const int T = 8 * kT0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * kTOut * kNOut; e += gridDim.x * blockDim.x) {
        int c = e % kNOut, t = (e / kNOut) % kTOut, b = e / (kNOut * kTOut);
        out[e] = y[((size_t)b * T + t) * kCh + c];
    }
}

}  // namespace sur

using namespace sur;

struct Layer {
    int out, in;        // logical
    int outP, inP;      // padded (64)
    bool conv;
    int T;              // conv: output time points; linear: 0
    int cin;            // conv: input channels (logical)
    bool relu;
    size_t wofs, bofs;  // offsets in the padded parameter arrays
};

struct cs_sur {
    int device = 0;
    int bmax = 0;       // batch capacity (multiple of 64)
    cudaStream_t stream = nullptr;
    char err[512] = {0};
    std::vector<Layer> L;
    size_t np = 0;                          // padded parameter count (weights + biases)
    float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;   // FP32, padded layout
    bf16* wb = nullptr;                     // BF16 weights (and biases, unused)
    long long t = 0;                        // Adam step
    // activations and scratch sized for bmax
    std::vector<bf16*> act;                 // act[0] = input, act[l+1] = output of layer l (BF16)
    float* yout = nullptr;                  // last layer output FP32 [bmax*368, 64]
    bf16 *cols[3] = {nullptr, nullptr, nullptr};
    bf16 *colsT = nullptr, *dzT = nullptr, *wT = nullptr, *hT = nullptr;
    float *dz = nullptr, *dh = nullptr, *dcols = nullptr, *part = nullptr;
    float* kpart = nullptr;                 // split-K partial products
    size_t kpart_n = 0;
    double *lpart = nullptr, *lsum = nullptr;   // loss reduction
    int* d_err = nullptr;                   // set by a tensor-core GEMM whose wait gave up
    int gemm_impl = 0;                      // 0: tcgen05, 1: mma.sync
    bf16* dzb = nullptr;
    float *xdev = nullptr, *tdev = nullptr, *sq = nullptr, *ydev = nullptr;
    std::vector<void*> allocs;
};

static int sur_err(cs_sur* s, int code, const char* fmt, ...)
{
    if (s) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(s->err, sizeof(s->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

#define SCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return sur_err(s, CS_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
static int salloc(cs_sur* s, T** p, size_t n)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * (n ? n : 1));
    if (e != cudaSuccess) return sur_err(s, CS_E_CUDA, "cudaMalloc(%zu bytes): %s", sizeof(T) * n, cudaGetErrorString(e));
    s->allocs.push_back(q);
    SCK(cudaMemsetAsync(q, 0, sizeof(T) * (n ? n : 1), s->stream));
    *p = (T*)q;
    return CS_OK;
}

static void build_layers(cs_sur* s)
{
    s->L.clear();
    const int lin[6][2] = {{kWidth, kIn}, {kWidth, kWidth}, {kWidth, kWidth}, {kWidth, kWidth}, {kLatent, kWidth}, {kT0 * kC0, kLatent}};
    size_t ofs = 0;
    for (int i = 0; i < 6; i++) {
        Layer l{lin[i][0], lin[i][1], up64(lin[i][0]), up64(lin[i][1]), false, 0, 0, true, 0, 0};
        l.wofs = ofs; ofs += (size_t)l.outP * l.inP;
        l.bofs = ofs; ofs += l.outP;
        s->L.push_back(l);
    }
    const int conv[3][3] = {{64, 64, 1}, {64, 32, 1}, {32, 4, 0}};
    int T = kT0;
    for (int i = 0; i < 3; i++) {
        T *= 2;
        Layer l{conv[i][1], kTap * conv[i][0], up64(conv[i][1]), up64(kTap * conv[i][0]), true, T, conv[i][0], conv[i][2] != 0, 0, 0};
        l.wofs = ofs; ofs += (size_t)l.outP * l.inP;
        l.bofs = ofs; ofs += l.outP;
        s->L.push_back(l);
    }
    s->np = ofs;
}

constexpr int kLossBlocks = 296;

// One product (or, with nsplit > 1, its K slices of kchunk) on the selected path.
static int gemm_launch(cs_sur* s, const bf16* A, int lda, const bf16* B, int ldb, float* C, int ldc, bf16* Cb, int ldcb,
                       const float* bias, int relu, int M, int N, int K, int nsplit, int kchunk, size_t cstride)
{
    if (s->gemm_impl == 0 && K % 64 == 0 && kchunk % 64 == 0) {
        dim3 grid(N / 64, (M + tc::BM - 1) / tc::BM, nsplit);
        k_gemm_tc<64><<<grid, 128, tc::smem_bytes(64), s->stream>>>(A, lda, B, ldb, C, ldc, Cb, ldcb, bias, relu, M, K,
                                                                    kchunk, cstride, s->d_err, nullptr, 0, 0);
    } else {
        dim3 grid(N / 64, M / 64, nsplit);
        sur::k_gemm_nt<<<grid, 128, 0, s->stream>>>(A, lda, B, ldb, C, ldc, Cb, ldcb, bias, relu, K, kchunk, cstride);
    }
    SCK(cudaGetLastError());
    return CS_OK;
}

// C = A B^T (+ bias) (ReLU).  A product with few output tiles and a long K (the
// convolutions' weight gradients, K = batch x time points; the linear layers at
// batch sizes of a few hundred) is split along K so that about two blocks per SM
// run; the slices' partial products are then summed in a fixed order and the
// epilogue applied.
constexpr int kMaxSplit = 64;

static int gemm(cs_sur* s, const bf16* A, int lda, const bf16* B, int ldb, float* C, int ldc, bf16* Cb, int ldcb,
                const float* bias, int relu, int M, int N, int K)
{
    if (M % 64 || N % 64 || K % 32) return sur_err(s, CS_E_ARG, "gemm shape %d x %d x %d not padded", M, N, K);
    const int tiles = (s->gemm_impl == 0 ? (M + tc::BM - 1) / tc::BM : M / 64) * (N / 64);
    int nsplit = tiles < 74 ? std::min(kMaxSplit, std::max(1, std::min(K / 128, 296 / tiles))) : 1;
    if (nsplit > 1 && K % 64 == 0) {
        const int kchunk = ((K + nsplit - 1) / nsplit + 63) / 64 * 64;
        nsplit = (K + kchunk - 1) / kchunk;
        if (nsplit > 1 && (size_t)nsplit * M * N <= s->kpart_n) {
            int r = gemm_launch(s, A, lda, B, ldb, s->kpart, N, nullptr, 0, nullptr, 0, M, N, K, nsplit, kchunk,
                                (size_t)M * N);
            if (r) return r;
            const int rg = (int)std::min<size_t>(1184, ((size_t)M * N + 255) / 256);
            sur::k_splitk_reduce<<<rg, 256, 0, s->stream>>>(s->kpart, nsplit, M, N, C, ldc, Cb, ldcb, bias, relu);
            SCK(cudaGetLastError());
            return CS_OK;
        }
    }
    return gemm_launch(s, A, lda, B, ldb, C, ldc, Cb, ldcb, bias, relu, M, N, K, 1, K, 0);
}


static int transpose(cs_sur* s, const bf16* in, int ldi, bf16* out, int ldo, int R, int Cc)
{
    dim3 grid(Cc / 32, R / 32), block(32, 8);
    sur::k_transpose<<<grid, block, 0, s->stream>>>(in, ldi, out, ldo, R, Cc);
    SCK(cudaGetLastError());
    return CS_OK;
}

static size_t act_elems(const cs_sur* s, int li, int Bp)
{
    // act[li] is the input of layer li: [Bp, inP] for linear layers, [Bp*T_in, 64] for convs
    if (li == 0) return (size_t)Bp * 64;
    const Layer& p = s->L[li - 1];
    return p.conv ? (size_t)Bp * p.T * kCh : (size_t)Bp * p.outP;
}

extern "C" {

size_t cs_sur_num_params(void)
{
    // logical (unpadded) weights and biases, in the flat order of the host interface
    size_t n = 0;
    const int shapes[9][2] = {{kWidth, kIn}, {kWidth, kWidth}, {kWidth, kWidth}, {kWidth, kWidth}, {kLatent, kWidth},
                              {kT0 * kC0, kLatent}, {64, kTap * 64}, {32, kTap * 64}, {4, kTap * 32}};
    for (auto& sh : shapes) n += (size_t)sh[0] * sh[1] + sh[0];
    return n;
}

int cs_sur_create(int max_batch, int device, cs_sur** out)
{
    if (!out) return CS_E_ARG;
    cs_sur* s = new cs_sur();
    *out = s;
    if (max_batch <= 0) return sur_err(s, CS_E_ARG, "max_batch must be positive");
    s->device = device;
    s->bmax = up64(max_batch);
    SCK(cudaSetDevice(device));
    SCK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    build_layers(s);
    int r;
#define SA(p, n) do { if ((r = salloc(s, &p, n))) return r; } while (0)
    SA(s->w, s->np); SA(s->m, s->np); SA(s->v, s->np); SA(s->g, s->np); SA(s->wb, s->np);
    const int B = s->bmax;
    s->act.assign(s->L.size() + 1, nullptr);
    size_t maxc = 0, maxcol = 0, maxw = 0;
    for (size_t li = 0; li <= s->L.size(); li++) {
        size_t n = act_elems(s, (int)li, B);
        SA(s->act[li], n);
        maxc = std::max(maxc, n);
    }
    for (int i = 0; i < 3; i++) {
        const Layer& l = s->L[6 + i];
        size_t n = (size_t)B * l.T * l.inP;
        SA(s->cols[i], n);
        maxcol = std::max(maxcol, n);
    }
    for (auto& l : s->L) maxw = std::max(maxw, (size_t)l.outP * l.inP);
    SA(s->yout, (size_t)B * 8 * kT0 * kCh);
    SA(s->colsT, maxcol);
    SA(s->dcols, maxcol);
    size_t maxz = std::max(maxc, (size_t)B * 8 * kT0 * kCh);
    SA(s->dz, maxz); SA(s->dzb, maxz); SA(s->dzT, maxz); SA(s->dh, maxz); SA(s->hT, maxz);
    SA(s->wT, maxw);
    SA(s->part, (size_t)((B * 8 * kT0 + 255) / 256 + 1) * 3000);
    {
        size_t mn = 0;
        for (int i = 0; i < 3; i++) mn = std::max(mn, (size_t)s->L[6 + i].outP * s->L[6 + i].inP);
        s->kpart_n = std::max(mn * kMaxSplit, (size_t)4 << 20);
        SA(s->kpart, s->kpart_n);
    }
    SA(s->lpart, (size_t)kLossBlocks); SA(s->lsum, (size_t)1); SA(s->d_err, (size_t)1);
    SCK(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
    SCK(cudaFuncSetAttribute(k_gemm_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::smem_bytes(64)));
    SA(s->xdev, (size_t)B * kIn); SA(s->tdev, (size_t)B * kTOut * kNOut); SA(s->sq, (size_t)B * kTOut * kNOut);
    SA(s->ydev, (size_t)B * kTOut * kNOut);
#undef SA
    SCK(cudaStreamSynchronize(s->stream));
    return CS_OK;
}

void cs_sur_destroy(cs_sur* s)
{
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (void* p : s->allocs) cudaFree(p);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

const char* cs_sur_last_error(const cs_sur* s) { return s ? s->err : "null surrogate"; }

int cs_sur_set_params(cs_sur* s, const float* flat)
{
    if (!s || !flat) return CS_E_ARG;
    std::vector<float> h(s->np, 0.f);
    size_t k = 0;
    for (auto& l : s->L) {
        for (int o = 0; o < l.out; o++)
            for (int i = 0; i < l.in; i++) h[l.wofs + (size_t)o * l.inP + i] = flat[k++];
        for (int o = 0; o < l.out; o++) h[l.bofs + o] = flat[k++];
    }
    SCK(cudaMemcpyAsync(s->w, h.data(), sizeof(float) * s->np, cudaMemcpyHostToDevice, s->stream));
    SCK(cudaMemsetAsync(s->m, 0, sizeof(float) * s->np, s->stream));
    SCK(cudaMemsetAsync(s->v, 0, sizeof(float) * s->np, s->stream));
    sur::k_to_bf16<<<256, 256, 0, s->stream>>>(s->w, s->wb, s->np);
    SCK(cudaGetLastError());
    s->t = 0;
    SCK(cudaStreamSynchronize(s->stream));
    return CS_OK;
}

int cs_sur_get_params(cs_sur* s, float* flat)
{
    if (!s || !flat) return CS_E_ARG;
    std::vector<float> h(s->np);
    SCK(cudaMemcpyAsync(h.data(), s->w, sizeof(float) * s->np, cudaMemcpyDeviceToHost, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    size_t k = 0;
    for (auto& l : s->L) {
        for (int o = 0; o < l.out; o++)
            for (int i = 0; i < l.in; i++) flat[k++] = h[l.wofs + (size_t)o * l.inP + i];
        for (int o = 0; o < l.out; o++) flat[k++] = h[l.bofs + o];
    }
    return CS_OK;
}

}  // extern "C"

// Forward pass of Bp rows (x already in act[0]); leaves y in s->yout.
static int forward(cs_sur* s, int Bp)
{
    int r;
    for (int li = 0; li < 6; li++) {
        const Layer& l = s->L[li];
        if ((r = gemm(s, s->act[li], l.inP, s->wb + l.wofs, l.inP, nullptr, 0, s->act[li + 1], l.outP,
                      s->w + l.bofs, 1, Bp, l.outP, l.inP))) return r;
    }
    int T = kT0;
    for (int ci = 0; ci < 3; ci++) {
        const Layer& l = s->L[6 + ci];
        const bool last = ci == 2;
        float* C = last ? s->yout : nullptr;
        bf16* Cb = last ? nullptr : s->act[7 + ci];
        const int M = Bp * 2 * T;
        if (s->gemm_impl == 0) {   // the column matrix is generated while staging
            dim3 grid(l.outP / 64, (M + tc::BM - 1) / tc::BM, 1);
            k_gemm_tc<64><<<grid, 128, tc::smem_bytes(64), s->stream>>>(nullptr, 0, s->wb + l.wofs, l.inP, C, kCh, Cb, kCh,
                                                                        s->w + l.bofs, l.relu ? 1 : 0, M, l.inP, l.inP, 0,
                                                                        s->d_err, s->act[6 + ci], T, l.cin);
            SCK(cudaGetLastError());
        } else {
            sur::k_im2col_up<<<1184, 256, 0, s->stream>>>(s->act[6 + ci], Bp, T, l.cin, s->cols[ci], l.inP);
            SCK(cudaGetLastError());
            if ((r = gemm(s, s->cols[ci], l.inP, s->wb + l.wofs, l.inP, C, kCh, Cb, kCh, s->w + l.bofs, l.relu ? 1 : 0,
                          M, l.outP, l.inP))) return r;
        }
        T *= 2;
    }
    return CS_OK;
}

static int colsum(cs_sur* s, const float* dz, int rows, int ld, float* out)
{
    const int nch = (rows + kColChunk - 1) / kColChunk;
    const dim3 blk(32, 8);
    sur::k_colsum_part<<<dim3((ld + 31) / 32, nch), blk, 0, s->stream>>>(dz, rows, ld, s->part);
    sur::k_colsum_final<<<(ld + 31) / 32, blk, 0, s->stream>>>(s->part, nch, ld, out);
    SCK(cudaGetLastError());
    return CS_OK;
}

// Backward pass from dy (in s->dh as [Bp*368, 64] FP32) to gradients in s->g.
static int backward(cs_sur* s, int Bp)
{
    int r;
    // ---- convolutions, last to first
    // dz of the last conv is dy (no ReLU)
    {
        size_t n = (size_t)Bp * 8 * kT0 * kCh;
        sur::k_to_bf16<<<1184, 256, 0, s->stream>>>(s->dh, s->dzb, n);
        SCK(cudaMemcpyAsync(s->dz, s->dh, sizeof(float) * n, cudaMemcpyDeviceToDevice, s->stream));
    }
    int T = 8 * kT0;
    for (int ci = 2; ci >= 0; ci--) {
        const Layer& l = s->L[6 + ci];
        const int M = Bp * T;
        // dW = dz^T cols: A = dz^T [outP, M], B = cols^T [inP, M]
        if ((r = transpose(s, s->dzb, kCh, s->dzT, M, M, l.outP))) return r;
        {   // the transposed column matrix of this convolution's input, from the input itself
            dim3 grid(l.inP / 32, M / 32), blk(32, 8);
            sur::k_im2colT_up<<<grid, blk, 0, s->stream>>>(s->act[6 + ci], T / 2, l.cin, s->colsT, M);
            SCK(cudaGetLastError());
        }
        if ((r = gemm(s, s->dzT, M, s->colsT, M, s->g + l.wofs, l.inP, nullptr, 0, nullptr, 0, l.outP, l.inP, M))) return r;
        if ((r = colsum(s, s->dz, M, kCh, s->g + l.bofs))) return r;
        // dcols = dz W: A = dz [M, outP], B = W^T [inP, outP]
        if ((r = transpose(s, s->wb + l.wofs, l.inP, s->wT, l.outP, l.outP, l.inP))) return r;
        if ((r = gemm(s, s->dzb, kCh, s->wT, l.outP, s->dcols, l.inP, nullptr, 0, nullptr, 0, M, l.inP, l.outP))) return r;
        // dz of the layer below: col2im with the ReLU mask of this conv's input
        T /= 2;
        sur::k_col2im_up_relu<<<1184, 256, 0, s->stream>>>(s->dcols, l.inP, Bp, T, l.cin, s->act[6 + ci], s->dz, s->dzb);
        SCK(cudaGetLastError());
    }
    // ---- linear layers, last to first; s->dz/dzb hold dz of layer li's output
    for (int li = 5; li >= 0; li--) {
        const Layer& l = s->L[li];
        if ((r = transpose(s, s->dzb, l.outP, s->dzT, Bp, Bp, l.outP))) return r;
        if ((r = transpose(s, s->act[li], l.inP, s->hT, Bp, Bp, l.inP))) return r;
        if ((r = gemm(s, s->dzT, Bp, s->hT, Bp, s->g + l.wofs, l.inP, nullptr, 0, nullptr, 0, l.outP, l.inP, Bp))) return r;
        if ((r = colsum(s, s->dz, Bp, l.outP, s->g + l.bofs))) return r;
        if (li == 0) break;
        if ((r = transpose(s, s->wb + l.wofs, l.inP, s->wT, l.outP, l.outP, l.inP))) return r;
        if ((r = gemm(s, s->dzb, l.outP, s->wT, l.outP, s->dh, l.inP, nullptr, 0, nullptr, 0, Bp, l.inP, l.outP))) return r;
        sur::k_relu_back<<<1184, 256, 0, s->stream>>>(s->dh, s->act[li], (size_t)Bp * l.inP, s->dz, s->dzb);
        SCK(cudaGetLastError());
    }
    return CS_OK;
}

// Wait for the stream; an error if a tensor-core GEMM's bounded wait gave up.
static int sync_check(cs_sur* s)
{
    int e = 0;
    SCK(cudaMemcpyAsync(&e, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    if (e) {
        SCK(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream));
        return sur_err(s, CS_E_CUDA, "a tensor-core GEMM gave up waiting for its products");
    }
    return CS_OK;
}

static int load_batch(cs_sur* s, const float* x, const float* target, int n, int* Bp)
{
    if (n <= 0 || n > s->bmax) return sur_err(s, CS_E_RANGE, "batch of %d outside 1..%d", n, s->bmax);
    *Bp = up64(n);
    SCK(cudaMemcpyAsync(s->xdev, x, sizeof(float) * n * kIn, cudaMemcpyHostToDevice, s->stream));
    sur::k_load_x<<<(*Bp * 64 + 255) / 256, 256, 0, s->stream>>>(s->xdev, n, *Bp, s->act[0]);
    SCK(cudaGetLastError());
    if (target) SCK(cudaMemcpyAsync(s->tdev, target, sizeof(float) * n * kTOut * kNOut, cudaMemcpyHostToDevice, s->stream));
    return CS_OK;
}

static int loss_grad(cs_sur* s, const float* x, const float* target, int n, float* loss)
{
    int Bp, r;
    if ((r = load_batch(s, x, target, n, &Bp))) return r;
    if ((r = forward(s, Bp))) return r;
    const float scale = 1.f / ((float)n * kTOut * kNOut);
    sur::k_mse<<<1184, 256, 0, s->stream>>>(s->yout, s->tdev, n, Bp, scale, s->dh, s->sq);
    SCK(cudaGetLastError());
    if ((r = backward(s, Bp))) return r;
    if (loss) {
        const size_t nsq = (size_t)n * kTOut * kNOut;
        sur::k_sum_part<<<kLossBlocks, 256, 0, s->stream>>>(s->sq, nsq, s->lpart);
        sur::k_sum_final<<<1, 256, 0, s->stream>>>(s->lpart, kLossBlocks, s->lsum);
        SCK(cudaGetLastError());
        double acc = 0.0;
        SCK(cudaMemcpyAsync(&acc, s->lsum, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        if ((r = sync_check(s))) return r;
        *loss = (float)(acc / (double)nsq);
    }
    return CS_OK;
}

extern "C" {

int cs_sur_forward(cs_sur* s, const float* x, int n, float* y)
{
    if (!s || !x || !y) return CS_E_ARG;
    for (int b0 = 0; b0 < n; b0 += s->bmax) {
        int nb = std::min(s->bmax, n - b0), Bp, r;
        if ((r = load_batch(s, x + (size_t)b0 * kIn, nullptr, nb, &Bp))) return r;
        if ((r = forward(s, Bp))) return r;
        sur::k_store_y<<<512, 256, 0, s->stream>>>(s->yout, nb, s->ydev);
        SCK(cudaGetLastError());
        SCK(cudaMemcpyAsync(y + (size_t)b0 * kTOut * kNOut, s->ydev, sizeof(float) * nb * kTOut * kNOut,
                            cudaMemcpyDeviceToHost, s->stream));
    }
    return sync_check(s);
}

int cs_sur_loss_grad(cs_sur* s, const float* x, const float* target, int n, float* loss, float* grad)
{
    if (!s || !x || !target) return CS_E_ARG;
    int r = loss_grad(s, x, target, n, loss);
    if (r) return r;
    if (grad) {
        std::vector<float> h(s->np);
        SCK(cudaMemcpyAsync(h.data(), s->g, sizeof(float) * s->np, cudaMemcpyDeviceToHost, s->stream));
        if ((r = sync_check(s))) return r;
        size_t k = 0;
        for (auto& l : s->L) {
            for (int o = 0; o < l.out; o++)
                for (int i = 0; i < l.in; i++) grad[k++] = h[l.wofs + (size_t)o * l.inP + i];
            for (int o = 0; o < l.out; o++) grad[k++] = h[l.bofs + o];
        }
    }
    return CS_OK;
}

int cs_sur_train_step(cs_sur* s, const float* x, const float* target, int n, float lr, float weight_decay, float* loss)
{
    if (!s || !x || !target) return CS_E_ARG;
    int r = loss_grad(s, x, target, n, loss);
    if (r) return r;
    s->t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)s->t), c2 = 1.f - powf(b2, (float)s->t);
    sur::k_adam<<<1184, 256, 0, s->stream>>>(s->w, s->m, s->v, s->g, s->wb, s->np, lr, b1, b2, 1e-8f, c1, c2, weight_decay);
    SCK(cudaGetLastError());
    if (!loss) return sync_check(s);
    return CS_OK;
}

int cs_sur_set_gemm(cs_sur* s, int impl)
{
    if (!s) return CS_E_ARG;
    if (impl != 0 && impl != 1) return sur_err(s, CS_E_ARG, "GEMM path must be 0 (tcgen05) or 1 (mma.sync)");
    SCK(cudaStreamSynchronize(s->stream));
    s->gemm_impl = impl;
    return CS_OK;
}

}  // extern "C"
