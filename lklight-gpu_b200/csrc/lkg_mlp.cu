// Learned pose-energy surrogate: a 64 -> 256 -> 256 -> 256 -> 1 ReLU MLP with
// BF16 weights and activations and FP32 accumulation, trained online on the
// exact scorer's energies and used to screen candidate GSO moves.
//
// Kernels (all hand-written; the GEMM layers on tcgen05 by default, the
// mma.sync m16n8k16 bf16 kernel k_gemm kept as the second backend):
//   k_features   pose parameters + far-field potential and receptor atom
//                counts at 16 ligand anchor atoms -> 64 bf16 features
//   k_gemm       C = A * B^T tiles of 64 x 64, K step 32, four warps; A / B
//                read [rows][k] or transposed from global; epilogues: bias +
//                ReLU -> bf16 (forward), x ReLU'(H) -> bf16 (backward data),
//                split-K atomic FP32 (weight gradients)
//   k_gemm_tc    tcgen05 + TMA layers (forward, backward data): 128-row tiles,
//                K-major SW128 operands, FP32 accumulator in TMEM
//   k_wgrad_tc   tcgen05 + TMA weight gradients: MN-major SW128 operands,
//                reduction over the batch split across CTAs
//   k_head       last layer (256 -> 1) dot products, FP32 (prediction)
//   k_loss_head  training: the last layer, MSE on the standardised target,
//                dy, dH3 and the head-gradient partials
//   k_grad_adam  every gradient summed from its partials in a fixed order,
//                then Adam on the FP32 master weights (one launch), which
//                also refreshes both BF16 layouts of the GEMM weights
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include <cmath>
#include <cstring>
#include <vector>

#include "lkg_runtime.h"
#include "lkg_score.cuh"

namespace lkg {
namespace mlp {

constexpr int IN = 64, H = 256, NA = 16;   // features, width, anchors

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------
// per pose: [w, x, y, z, tx/s, ty/s, tz/s, then per anchor a:
//            phi(x_a) * 100, log1p(receptor atoms in the anchor's 3x3x3
//            fine cells), log1p(atoms in its own cell)], 1.0, zero padding
// Training batches also write the standardised targets (tgt not null):
// t = (asinh(score / e_scale) - mu) / sd.
struct TargetArgs {
    const double* scores;
    float e_scale, mu, sd;
    float* t;
};

__global__ void k_features(const ComplexDev* __restrict__ cxs, int cid, const double* __restrict__ poses, int n,
                           const int* __restrict__ anchors, float tscale, __nv_bfloat16* __restrict__ feat,
                           TargetArgs tgt) {
    const ComplexDev& c = cxs[cid];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int pose = t / NA, a = t % NA;
    if (pose >= n) return;
    const double* pq = poses + 7 * (size_t)pose;
    const Rot rot = pose_matrix(pq);
    __nv_bfloat16* f = feat + (size_t)pose * IN;
    if (a == 0) {
        if (tgt.t) tgt.t[pose] = (asinhf((float)(tgt.scores[pose] / tgt.e_scale)) - tgt.mu) / tgt.sd;
        for (int k = 0; k < 4; ++k) f[k] = __float2bfloat16((float)pq[k]);
        for (int k = 0; k < 3; ++k) f[4 + k] = __float2bfloat16((float)(pq[4 + k] / tscale));
        f[7 + 3 * NA] = __float2bfloat16(1.0f);
        for (int k = 8 + 3 * NA; k < IN; ++k) f[k] = __float2bfloat16(0.0f);
    }
    const int j = anchors[a];
    const float4 b = __ldg(c.lpos + j);
    double xd, yd, zd;
    apply(rot, (double)b.x, (double)b.y, (double)b.z, xd, yd, zd);
    const float x = (float)xd, y = (float)yd, z = (float)zd;
    float phi = c.phi ? sample_phi(c, x, y, z) : 0.f;
    // receptor atom counts in the 3 x 3 x 3 cells of edge h around the atom
    // and in its own cell (x sub-cells merged; bounds-clamped)
    const int xs = (int)(c.h * c.inv_hx + 0.5f);
    const int cx = (int)floorf((x - c.ox) * c.inv_h), cy = (int)floorf((y - c.oy) * c.inv_h),
              cz = (int)floorf((z - c.oz) * c.inv_h);
    int n27 = 0, n1 = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy) {
            const int zz = cz + dz, yy = cy + dy;
            if (zz < 0 || zz >= c.ncz || yy < 0 || yy >= c.ncy) continue;
            const int row = (zz * c.ncy + yy) * c.ncx;
            const int x0 = max((cx - 1) * xs, 0), x1 = min((cx + 2) * xs - 1, c.ncx - 1);
            if (x0 <= x1) n27 += __ldg(c.cell_start + row + x1 + 1) - __ldg(c.cell_start + row + x0);
            const int y0 = max(cx * xs, 0), y1 = min((cx + 1) * xs - 1, c.ncx - 1);
            if (dz == 0 && dy == 0 && y0 <= y1)
                n1 = __ldg(c.cell_start + row + y1 + 1) - __ldg(c.cell_start + row + y0);
        }
    f[7 + 3 * a] = __float2bfloat16(phi * 100.0f);
    f[8 + 3 * a] = __float2bfloat16(log1pf((float)n27));
    f[9 + 3 * a] = __float2bfloat16(log1pf((float)n1));
}

// ---------------------------------------------------------------------------
// GEMM: C[M x N] = sum_k A(m, k) * B(n, k)
//   A(m, k) = TA ? A[k * lda + m] : A[m * lda + k]
//   B(n, k) = TB ? B[k * ldb + n] : B[n * ldb + k]
// ---------------------------------------------------------------------------
enum { EPI_FWD = 0, EPI_BWD = 1, EPI_WGRAD = 2 };
constexpr int BM = 64, BN = 64, BK = 32;

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                                              const __nv_bfloat16* __restrict__ B, int ldb, float* __restrict__ Cf,
                                              __nv_bfloat16* __restrict__ Cb, int ldc, const float* __restrict__ bias,
                                              const __nv_bfloat16* __restrict__ Hmask, int k_chunk) {
    __shared__ __align__(16) __nv_bfloat16 sA[BM][BK + 8];
    __shared__ __align__(16) __nv_bfloat16 sB[BN][BK + 8];
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kb = blockIdx.z * k_chunk, ke = min(K, kb + k_chunk);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;   // warp sub-tile 32 x 32
    const int g = lane >> 2, tq = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = kb; k0 < ke; k0 += BK) {
        // tile loads (bounds-checked; zero fill)
        for (int e = threadIdx.x; e < BM * BK; e += 128) {
            int mm, kk;
            if (TA) { mm = e % BM; kk = e / BM; } else { kk = e % BK; mm = e / BK; }
            const int gm = m0 + mm, gk = k0 + kk;
            sA[mm][kk] = (gm < M && gk < ke) ? (TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]) : zero;
        }
        for (int e = threadIdx.x; e < BN * BK; e += 128) {
            int nn, kk;
            if (TB) { nn = e % BN; kk = e / BN; } else { kk = e % BK; nn = e / BK; }
            const int gn = n0 + nn, gk = k0 + kk;
            sB[nn][kk] = (gn < N && gk < ke) ? (TB ? B[(size_t)gk * ldb + gn] : B[(size_t)gn * ldb + gk]) : zero;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < BK; ks += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + g;
                af[i][0] = *(const uint32_t*)&sA[r][ks + 2 * tq];
                af[i][1] = *(const uint32_t*)&sA[r + 8][ks + 2 * tq];
                af[i][2] = *(const uint32_t*)&sA[r][ks + 2 * tq + 8];
                af[i][3] = *(const uint32_t*)&sA[r + 8][ks + 2 * tq + 8];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int cc = wn + j * 8 + g;
                bf[j][0] = *(const uint32_t*)&sB[cc][ks + 2 * tq];
                bf[j][1] = *(const uint32_t*)&sB[cc][ks + 2 * tq + 8];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bf[j]);
        }
        __syncthreads();
    }
    // epilogue
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int gm = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0);
                const int gn = n0 + wn + j * 8 + 2 * tq + (r & 1);
                if (gm >= M || gn >= N) continue;
                float v = acc[i][j][r];
                if (EPI == EPI_FWD) {
                    v += bias[gn];
                    Cb[(size_t)gm * ldc + gn] = __float2bfloat16(v > 0.f ? v : 0.f);
                } else if (EPI == EPI_BWD) {
                    const float hm = __bfloat162float(Hmask[(size_t)gm * ldc + gn]);
                    Cb[(size_t)gm * ldc + gn] = __float2bfloat16(hm > 0.f ? v : 0.f);
                } else {   // split blockIdx.z's partial tile; k_grad_adam adds the splits in order
                    Cf[(size_t)blockIdx.z * M * ldc + (size_t)gm * ldc + gn] = v;
                }
            }
}

// ---------------------------------------------------------------------------
// Layers on the 5th-generation tensor cores (tcgen05, sm_100a):
//   Y[M x 256] = epi(A[M x K] B^T), A [M x K] and B [256 x K] both K-major
//   bf16 (K = 64 or 256), FP32 accumulation; epilogues: EPI_FWD (+ bias,
//   ReLU; B = W, a forward layer) and EPI_BWD (x ReLU'(Hm); B = W^T, the
//   backward-data product dA_in = dC W).
// One CTA (4 warps) per 128-row tile and the full width N = 256.  The
// operands arrive by TMA: one 2D tiled copy per 64-element K slab of A (128
// rows) and of B (256 rows), 128-byte swizzled, into 1024-byte aligned
// shared memory, all completing on one mbarrier (expect_tx); rows past M
// are zero-filled by the copy.  One elected thread then issues K / 16
// tcgen05.mma (M = 128, N = 256, K = 16, BF16 in, FP32 accumulate) with
// SW128 K-major descriptors (8-row groups 1024 B apart; a K step of 16 moves
// the start address by 32 B inside the swizzle atom) into a 128-lane x
// 256-column TMEM accumulator and commits them to a second mbarrier; each
// warp reads its 32 TMEM lanes (rows) back with tcgen05.ld and applies the
// epilogue.  Both waits are bounded: a wait that runs out sets status bit 2,
// the CTA skips the rest, waits (bounded again) for the copies or MMAs it
// still has in flight, and the accumulator is still freed.
// ---------------------------------------------------------------------------
constexpr int TC_BM = 128, TC_N = 256, TC_KMAX = 256, TC_KS = 64;   // K slab of one TMA copy (128 B)
constexpr size_t TC_SMEM = (size_t)(TC_BM + TC_N) * TC_KMAX * 2 + 1024;   // A, B slabs + alignment slack

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, 128-byte swizzle: SBO = 1024 B (next 8 rows), LBO unused (1),
// version 1 (bits 46-47), layout type SWIZZLE_128B (2, bits 61-63)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3fff) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred P1;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}\n"
                     : "=r"(ok) : "r"(bar), "r"(phase) : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar) : "memory");
}

// TN: output columns of a CTA (256, or 128 with blockIdx.y picking the half
// when the row tiles alone would leave most SMs idle)
template <int EPI, int TN>
__global__ void __launch_bounds__(128, 1)
k_gemm_tc(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int M, int K,
          const float* __restrict__ bias, const __nv_bfloat16* __restrict__ Hm, __nv_bfloat16* __restrict__ Y,
          int* __restrict__ status) {
    static_assert(TN == 128 || TN == 256, "tile width");
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long bars[2];   // operands loaded, accumulator ready
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * TN, nslab = K / TC_KS;
    const uint32_t base = (smem_u32(tc_smem) + 1023u) & ~1023u;   // SW128 atoms are 1024-byte aligned
    const uint32_t sA = base, sB = base + (uint32_t)(nslab * TC_BM * 128);
    const uint32_t bar_ld = smem_u32(&bars[0]), bar_mma = smem_u32(&bars[1]);
    // 1. TMEM: 256 columns (the FP32 accumulator); barriers; the TMA copies
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_slot)), "r"(TN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar_ld), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar_mma), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        const uint32_t bytes = (uint32_t)(nslab * (TC_BM + TN) * 128);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar_ld), "r"(bytes) : "memory");
        for (int sl = 0; sl < nslab; ++sl) {
            tma_load_2d(sA + (uint32_t)(sl * TC_BM * 128), &mapA, sl * TC_KS, m0, bar_ld);
            tma_load_2d(sB + (uint32_t)(sl * TN * 128), &mapB, sl * TC_KS, n0, bar_ld);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const bool ld_ok = mbar_wait(bar_ld, 0);
    // 2. one thread issues the MMAs and commits them to the second barrier
    if (ld_ok && tid == 0) {
        // kind::f16 descriptor: D f32 (bits 4-5 = 1), A bf16 (7-9 = 1), B bf16
        // (10-12 = 1), both K-major, N >> 3 at 17-22, M >> 4 at 24-28
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                               ((uint32_t)(TC_BM >> 4) << 24);
        for (int sl = 0; sl < nslab; ++sl)
            for (int ks = 0; ks < TC_KS / 16; ++ks) {
                const uint64_t ad = tc_desc(sA + (uint32_t)(sl * TC_BM * 128 + ks * 32));
                const uint64_t bd = tc_desc(sB + (uint32_t)(sl * TN * 128 + ks * 32));
                const uint32_t acc = (sl | ks) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(bar_mma) : "memory");
    }
    // 3. bounded wait for the accumulator
    const bool ok = ld_ok && mbar_wait(bar_mma, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (lane == 0) atomicOr(status, 4);
    } else {
        // 4. epilogue: warp w holds rows 32w .. 32w + 31 (TMEM lanes)
        const int row = m0 + warp * 32 + lane;
        for (int cl = 0; cl < TN; cl += 32) {
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cl;
            const int c0 = n0 + cl;   // output column
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                         "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                         "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                           "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
                           "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
                           "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
                __align__(16) __nv_bfloat16 o[32];
                if (EPI == EPI_FWD) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const float v = __uint_as_float(r[j]) + bias[c0 + j];
                        o[j] = __float2bfloat16(v > 0.f ? v : 0.f);
                    }
                } else {
                    __align__(16) __nv_bfloat16 hm[32];
                    const uint4* src = reinterpret_cast<const uint4*>(Hm + (size_t)row * TC_N + c0);
#pragma unroll
                    for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(hm)[q] = src[q];
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        o[j] = __float2bfloat16(__bfloat162float(hm[j]) > 0.f ? __uint_as_float(r[j]) : 0.f);
                }
                uint4* dst = reinterpret_cast<uint4*>(Y + (size_t)row * TC_N + c0);
#pragma unroll
                for (int q = 0; q < 4; ++q) dst[q] = reinterpret_cast<const uint4*>(o)[q];
            }
        }
    }
    // 5. free the accumulator.  After a wait that ran out, first wait out
    //    (bounded again) what this CTA still has in flight: the TMA copies
    //    into its shared memory, or the MMAs into its TMEM
    if (!ld_ok) mbar_wait(bar_ld, 0);
    else if (!ok) mbar_wait(bar_mma, 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TN));
    }
}

// ---------------------------------------------------------------------------
// Forward layer for large predictions: a persistent, warp-specialised
// tcgen05 GEMM.  Each CTA (one per SM) keeps the layer's weights B
// [256 x K] resident in shared memory and walks row tiles t = blockIdx.x,
// + gridDim.x, ...:
//   warp 0, one lane:  TMA producer; 128-row x 64-K slabs of A into a ring
//                      of PP_ST stages (full / empty mbarriers per stage)
//   warp 1, one lane:  MMA issuer; per slab four tcgen05.mma (M 128, N 256,
//                      K 16) into one of two TMEM accumulators, the slab's
//                      stage freed by tcgen05.commit, the tile's accumulator
//                      announced by a second commit
//   warps 2-5:         epilogue; each warp reads its TMEM lane quarter
//                      (warp % 4), adds the bias, applies ReLU, stores bf16,
//                      and frees the accumulator for the tile after next
// so the next tile's copies and MMAs run under the current tile's epilogue.
// The MMAs are the same as k_gemm_tc's (same descriptors, same K order), so
// the outputs are too.  Every wait is bounded: one that runs out sets status
// bit 4 and an abort flag that ends every role's loop; the producer and the
// MMA issuer then wait (bounded) for their copies and MMAs still in flight
// before the accumulators are freed.
// ---------------------------------------------------------------------------
constexpr int PP_ST = 4;                          // A ring stages (16 KB each)
constexpr int PP_THREADS = 192;
constexpr size_t PP_SMEM = (size_t)TC_N * TC_KMAX * 2 + (size_t)PP_ST * TC_BM * 128 + 1024;

__device__ __forceinline__ bool pp_wait(uint32_t bar, uint32_t phase, volatile int* abort) {
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred P1;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}\n"
                     : "=r"(ok) : "r"(bar), "r"(phase) : "memory");
        if (ok) return true;
        if ((it & 255) == 255 && abort && *abort) return false;
    }
    return false;
}

__global__ void __launch_bounds__(PP_THREADS, 1)
k_gemm_tc_pp(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int M, int K,
             const float* __restrict__ bias, __nv_bfloat16* __restrict__ Y, int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long full[PP_ST], empty[PP_ST], accf[2], acce[2], bfull;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nslab = K / TC_KS, tiles = (M + TC_BM - 1) / TC_BM;
    const uint32_t base = (smem_u32(tc_smem) + 1023u) & ~1023u;   // SW128 atoms are 1024-byte aligned
    const uint32_t sB = base, sA = base + (uint32_t)(TC_N * TC_KMAX * 2);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_slot)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        abort_flag = 0;
        for (int i = 0; i < PP_ST; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&full[i])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&empty[i])), "r"(1));
        }
        for (int i = 0; i < 2; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&accf[i])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&acce[i])), "r"(4));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&bfull)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    if (warp == 0) {
        if (lane == 0) {
            // the weights, once; then the A slabs of every tile through the ring
            const uint32_t bb = smem_u32(&bfull);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                         :: "r"(bb), "r"((uint32_t)(nslab * TC_N * 128)) : "memory");
            for (int sl = 0; sl < nslab; ++sl) tma_load_2d(sB + (uint32_t)(sl * TC_N * 128), &mapB, sl * TC_KS, 0, bb);
            int it = 0;
            for (int t = blockIdx.x; t < tiles && !abort_flag; t += gridDim.x)
                for (int sl = 0; sl < nslab; ++sl, ++it) {
                    const int s = it % PP_ST, round = it / PP_ST;
                    if (round > 0 && !pp_wait(smem_u32(&empty[s]), (uint32_t)((round - 1) & 1), &abort_flag)) {
                        atomicOr(status, 4);
                        abort_flag = 1;
                        break;
                    }
                    const uint32_t fb = smem_u32(&full[s]);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                                 :: "r"(fb), "r"((uint32_t)(TC_BM * 128)) : "memory");
                    tma_load_2d(sA + (uint32_t)(s * TC_BM * 128), &mapA, sl * TC_KS, t * TC_BM, fb);
                }
            // every copy issued has landed before the CTA ends (the last
            // round of each stage; bounded)
            for (int s = 0; s < PP_ST && s < it; ++s) {
                const int last = s + ((it - 1 - s) / PP_ST) * PP_ST;
                pp_wait(smem_u32(&full[s]), (uint32_t)((last / PP_ST) & 1), nullptr);
            }
            pp_wait(smem_u32(&bfull), 0u, nullptr);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                                   ((uint32_t)(TC_BM >> 4) << 24);
            int it = 0, lt = 0, last_s = -1, last_round = 0;
            bool ok = pp_wait(smem_u32(&bfull), 0u, &abort_flag);
            for (int t = blockIdx.x; ok && t < tiles && !abort_flag; t += gridDim.x, ++lt) {
                const int buf = lt & 1, use = lt >> 1;
                if (use > 0 && !pp_wait(smem_u32(&acce[buf]), (uint32_t)((use - 1) & 1), &abort_flag)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc_addr = tmem + (uint32_t)(buf * TC_N);
                for (int sl = 0; sl < nslab; ++sl, ++it) {
                    const int s = it % PP_ST, round = it / PP_ST;
                    if (!pp_wait(smem_u32(&full[s]), (uint32_t)(round & 1), &abort_flag)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    for (int ks = 0; ks < TC_KS / 16; ++ks) {
                        const uint64_t ad = tc_desc(sA + (uint32_t)(s * TC_BM * 128 + ks * 32));
                        const uint64_t bd = tc_desc(sB + (uint32_t)(sl * TC_N * 128 + ks * 32));
                        const uint32_t acc = (sl | ks) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                            :: "r"(acc_addr), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u),
                               "r"(0u));
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                 :: "r"(smem_u32(&empty[s])) : "memory");
                    last_s = s;
                    last_round = round;
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             :: "r"(smem_u32(&accf[buf])) : "memory");
            }
            if (!ok) {
                atomicOr(status, 4);
                abort_flag = 1;
            }
            // the MMAs issued have completed before the accumulators are
            // freed (the last commit covers every earlier MMA; bounded)
            if (last_s >= 0) pp_wait(smem_u32(&empty[last_s]), (uint32_t)(last_round & 1), nullptr);
        }
    } else {
        const int q = warp & 3;   // the TMEM lane quarter this warp may read
        int lt = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++lt) {
            const int buf = lt & 1, use = lt >> 1;
            // one decision for the whole warp (its TMEM loads are warp-wide)
            if (!__all_sync(0xffffffffu, pp_wait(smem_u32(&accf[buf]), (uint32_t)(use & 1), &abort_flag))) {
                if (lane == 0) {
                    atomicOr(status, 4);
                    abort_flag = 1;
                }
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int row = t * TC_BM + q * 32 + lane;
            for (int cl = 0; cl < TC_N; cl += 32) {
                uint32_t r[32];
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * TC_N + cl);
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                             "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                             "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                               "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                               "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
                               "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
                               "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
                               "=r"(r[31])
                             : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (row < M) {
                    __align__(16) __nv_bfloat16 o[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const float v = __uint_as_float(r[j]) + bias[cl + j];
                        o[j] = __float2bfloat16(v > 0.f ? v : 0.f);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(Y + (size_t)row * TC_N + cl);
#pragma unroll
                    for (int qq = 0; qq < 4; ++qq) dst[qq] = reinterpret_cast<const uint4*>(o)[qq];
                }
            }
            // this warp is done with the accumulator: the tile after next may use it
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(&acce[buf])) : "memory");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(512));
    }
}

// ---------------------------------------------------------------------------
// Weight gradients on tcgen05: dW[o][i] = sum_r dC[r][o] * A_in[r][i] over
// the batch rows r.  Both operands are stored row by row ([r][o], [r][i]),
// so for the reduction over r they are MN-major: A (M = o, 128 per CTA)
// and B (N = i: 64 or 256) arrive by TMA as boxes of 64 contiguous
// elements x 64 batch rows, 128-byte swizzled (8 rows per 1024-byte atom).
// The descriptors are MN-major SW128: SBO = 1024 B to the next 8 rows (K),
// LBO = 64 rows x 128 B to the next 64 elements (MN); one K step of 16 rows
// moves the start address by 2048 B (two whole atoms).  Each CTA reduces a
// chunk of TCW_ROWS batch rows (all its slabs resident, one expect_tx
// barrier) and writes its FP32 partial tile to part[split][o][i]; the
// splits are added in order afterwards (k_grad_adam), so training stays
// bitwise reproducible.  Waits are bounded as in k_gemm_tc.
// ---------------------------------------------------------------------------
constexpr int TCW_ROWS = 128;                       // batch rows per CTA (two 64-row slabs)
constexpr int TCW_SLAB = 64;                        // batch rows per TMA box
constexpr size_t TCW_SMEM = (size_t)(TC_BM + TC_N) * TCW_ROWS * 2 + 1024;

__device__ __forceinline__ uint64_t tc_desc_mn(uint32_t saddr, uint32_t lbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3fff) | ((uint64_t)((lbo_bytes >> 4) & 0x3fff) << 16) |
           ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

template <int TN>
__global__ void __launch_bounds__(128, 1)
k_wgrad_tc(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, int rows,
           float* __restrict__ part, int* __restrict__ status) {
    static_assert(TN == 64 || TN == 256, "input width");
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long bars[2];
    __shared__ uint32_t tmem_slot;
    constexpr int NSLAB = TCW_ROWS / TCW_SLAB;
    constexpr uint32_t A_SLAB = TC_BM * TCW_SLAB * 2, B_SLAB = TN * TCW_SLAB * 2;   // bytes per slab
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_BM, r0 = blockIdx.y * TCW_ROWS;
    const uint32_t base = (smem_u32(tc_smem) + 1023u) & ~1023u;
    const uint32_t sA = base, sB = base + (uint32_t)NSLAB * A_SLAB;
    const uint32_t bar_ld = smem_u32(&bars[0]), bar_mma = smem_u32(&bars[1]);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_slot)), "r"(TN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar_ld), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar_mma), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     :: "r"(bar_ld), "r"((uint32_t)NSLAB * (A_SLAB + B_SLAB)) : "memory");
        // slab sl: A boxes of 64 output rows (o) and B boxes of 64 inputs (i),
        // 64 batch rows each; box b of a slab sits b x 64 x 128 B in
        for (int sl = 0; sl < NSLAB; ++sl) {
            const int y = r0 + sl * TCW_SLAB;
            for (int b = 0; b < TC_BM / 64; ++b)
                tma_load_2d(sA + (uint32_t)sl * A_SLAB + (uint32_t)b * (TCW_SLAB * 128), &mapA, m0 + 64 * b, y, bar_ld);
            for (int b = 0; b < TN / 64; ++b)
                tma_load_2d(sB + (uint32_t)sl * B_SLAB + (uint32_t)b * (TCW_SLAB * 128), &mapB, 64 * b, y, bar_ld);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const bool ld_ok = mbar_wait(bar_ld, 0);
    if (ld_ok && tid == 0) {
        // kind::f16: D f32, A and B bf16, both MN-major (bits 15, 16), N >> 3, M >> 4
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                               ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
        for (int sl = 0; sl < NSLAB; ++sl)
            for (int ks = 0; ks < TCW_SLAB / 16; ++ks) {
                const uint64_t ad = tc_desc_mn(sA + (uint32_t)sl * A_SLAB + (uint32_t)ks * 2048, TCW_SLAB * 128);
                const uint64_t bd = tc_desc_mn(sB + (uint32_t)sl * B_SLAB + (uint32_t)ks * 2048, TCW_SLAB * 128);
                const uint32_t acc = (sl | ks) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(bar_mma) : "memory");
    }
    const bool ok = ld_ok && mbar_wait(bar_mma, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (lane == 0) atomicOr(status, 4);
    } else {
        // warp w: output rows o = m0 + 32 w + lane (TMEM lanes), 32 columns at a time
        float* out = part + (size_t)blockIdx.y * H * TN + (size_t)(m0 + warp * 32 + lane) * TN;
        for (int cl = 0; cl < TN; cl += 32) {
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cl;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                         "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                         "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                           "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
                           "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
                           "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float4* dst = reinterpret_cast<float4*>(out + cl);
#pragma unroll
            for (int q = 0; q < 8; ++q)
                dst[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                     __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
        }
    }
    if (!ld_ok) mbar_wait(bar_ld, 0);
    else if (!ok) mbar_wait(bar_mma, 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TN));
    }
}

// last layer: y[n] = H3[n] . w3 + b3
__global__ void k_head(const __nv_bfloat16* __restrict__ H3, int n, const float* __restrict__ w3, const float* b3,
                       float* __restrict__ y) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= n) return;
    float s = 0.f;
    for (int k = lane; k < H; k += 32) s += __bfloat162float(H3[(size_t)row * H + k]) * w3[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[row] = s + b3[0];
}

// Every reduction of the backward pass adds its terms in a fixed order
// (partials per block of rows or per split, then the partials in order), so
// training is bitwise reproducible.
constexpr int RB = 32;   // rows per partial sum (bias gradients)
constexpr int RL = 32;   // rows per partial sum of the loss kernel (each warp four rows of the head)

// training, per block of RL rows (one thread per column): the head
// y = H3 . w3 + b3 (a warp per row, as k_head; y is also stored), the loss
// terms d = y - t, dy = 2 d / n, dH3 = dy w3 x ReLU'(H3), and the partial
// sums over the block's rows of dy h (the w3 gradient, H columns), of dy
// (b3) and of d^2 / n (the loss) -> part[blk][H + 2]
__global__ void __launch_bounds__(H) k_loss_head(const float* __restrict__ t, const __nv_bfloat16* __restrict__ H3,
                                                int n, const float* __restrict__ w3, const float* __restrict__ b3,
                                                float* __restrict__ y, __nv_bfloat16* __restrict__ dH3,
                                                float* __restrict__ part) {
    static_assert(RL % (H / 32) == 0, "whole rows per warp");
    __shared__ float s_y[RL];
    const int k = threadIdx.x, r0 = blockIdx.x * RL, r1 = min(n, r0 + RL);
    for (int rr = k >> 5; rr < RL; rr += H / 32) {
        const int row = r0 + rr, lane = k & 31;
        if (row < r1) {
            float sy = 0.f;
            for (int c = lane; c < H; c += 32) sy += __bfloat162float(H3[(size_t)row * H + c]) * w3[c];
            for (int o = 16; o > 0; o >>= 1) sy += __shfl_xor_sync(0xffffffffu, sy, o);
            if (lane == 0) {
                s_y[rr] = sy + b3[0];
                y[row] = sy + b3[0];
            }
        }
    }
    __syncthreads();
    float gw = 0.f, gb = 0.f, ls = 0.f;
#pragma unroll
    for (int r = r0; r < r0 + RL; ++r) {
        if (r >= r1) break;
        const float d = s_y[r - r0] - t[r];
        const float dy = 2.f * d / (float)n;
        const float h = __bfloat162float(H3[(size_t)r * H + k]);
        dH3[(size_t)r * H + k] = __float2bfloat16(h > 0.f ? dy * w3[k] : 0.f);
        gw += dy * h;
        gb += dy;
        ls += d * d / (float)n;
    }
    float* p = part + (size_t)blockIdx.x * (H + 2);
    p[k] = gw;
    if (k == 0) { p[H] = gb; p[H + 1] = ls; }
}

// bias-gradient partials of the three layers in one launch: column sums
// of dC_L [n x H] per block of RB rows -> part[L][blk][H] (blockIdx.y = L)
struct ColSums {
    const __nv_bfloat16* dC[3];
    float* part;
};
__global__ void __launch_bounds__(H) k_colsum3(ColSums a, int n) {
    const int col = threadIdx.x, blk = blockIdx.x, L = blockIdx.y, r0 = blk * RB, r1 = min(n, r0 + RB);
    const __nv_bfloat16* dC = a.dC[L];
    float s = 0.f;
    for (int r = r0; r < r1; ++r) s += __bfloat162float(dC[(size_t)r * H + col]);
    a.part[((size_t)L * gridDim.x + blk) * H + col] = s;
}

// the three GEMM layers inside the flat parameter vector
struct AdamLayers {
    int off[3], cols[3];
    __nv_bfloat16* wt[3];
    __nv_bfloat16* w[3];
};

// The whole gradient and the Adam step in one launch.  Every parameter's
// gradient is summed in a fixed order: a weight over the weight-gradient
// splits in split order; a bias over k_colsum3's row blocks in order; w3
// and b3 over k_loss_head's row blocks in order.  g receives the sums, and the loss sum is added to
// the running loss.  Nothing depends on thread timing, so training repeats
// bit for bit.  apply = 0: gradients only (no update).  The step count t
// (1-based) lives on the device so that training steps can be replayed from
// a CUDA graph: step[0] is t, step[1] counts finished blocks, and the last
// block to finish advances t (after every block has read it).
struct GradSums {
    const float* wpart[3];           // per layer: nz[L] partial [H x cols] tiles
    int nz[3];
    const float* cpart;              // k_colsum3 partials [3][nblk][H]
    int nblk;
    const float* lpart;              // k_loss_head partials [nlblk][H + 2]
    int nlblk;
    float* loss;                     // running loss sum
};
__global__ void k_grad_adam(float* __restrict__ p, float* __restrict__ gr, float* __restrict__ m1,
                            float* __restrict__ m2, int n, float lr, float b1, float b2, float eps,
                            int* __restrict__ step, AdamLayers L, GradSums G, int apply) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float t = 0.f;
    if (apply) {
        t = (float)*reinterpret_cast<volatile int*>(step);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const unsigned v = atomicAdd(reinterpret_cast<unsigned*>(step + 1), 1u);
            if (v == gridDim.x - 1) {
                step[0] += 1;
                step[1] = 0;
            }
        }
    }
    if (i >= n) return;
    float gg = 0.f;
    const int off_w3 = L.off[2] + H * L.cols[2] + H;
    if (i >= off_w3) {   // w3 [H], b3 (and the loss, with b3)
        const int k = i - off_w3;
        #pragma unroll 8
        for (int b = 0; b < G.nlblk; ++b) gg += G.lpart[(size_t)b * (H + 2) + k];
        if (k == H) {
            float ls = 0.f;
            for (int b = 0; b < G.nlblk; ++b) ls += G.lpart[(size_t)b * (H + 2) + H + 1];
            *G.loss += ls;
        }
    } else {
        int l = 2;
        while (i < L.off[l]) --l;
        const int j = i - L.off[l], nw = H * L.cols[l];
        if (j < nw) {
            const float* part = G.wpart[l];
            #pragma unroll 8
            for (int z = 0; z < G.nz[l]; ++z) gg += part[(size_t)z * nw + j];
        } else {   // bias o of layer l: the row blocks' column sums in order
            const float* part = G.cpart + (size_t)l * G.nblk * H + (j - nw);
            #pragma unroll 8
            for (int b = 0; b < G.nblk; ++b) gg += part[(size_t)b * H];
        }
    }
    gr[i] = gg;
    if (!apply) return;
    const float bc1 = 1.f - powf(b1, t), bc2 = 1.f - powf(b2, t);
    const float a = b1 * m1[i] + (1.f - b1) * gg, v = b2 * m2[i] + (1.f - b2) * gg * gg;
    m1[i] = a;
    m2[i] = v;
    const float np = p[i] - lr * (a / bc1) / (sqrtf(v / bc2) + eps);
    p[i] = np;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int j = i - L.off[k];
        if (j >= 0 && j < H * L.cols[k]) {
            const int r = j / L.cols[k], c = j % L.cols[k];   // [rows = out][cols = in]
            L.wt[k][j] = __float2bfloat16(np);
            L.w[k][(size_t)c * H + r] = __float2bfloat16(np);
        }
    }
}

__global__ void k_f2bf(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = __float2bfloat16(src[i]);
}

__global__ void k_f2bf_t(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, int rows, int cols) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < rows * cols) dst[(size_t)(i % cols) * rows + i / cols] = __float2bfloat16(src[i]);
}

}  // namespace mlp
}  // namespace lkg

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace lkg;
using namespace lkg::mlp;

struct lkg_surrogate {
    lkg_ctx* ctx = nullptr;
    int cid = -1;
    float tscale = 50.f;
    float t_mu = 0.f, t_sd = 1.f, e_scale = 100.f;   // target standardisation
    DBuf anchors;
    // parameters: FP32 master, Adam moments, gradients (flat)
    //   W0 [H x IN], b0 [H], W1 [H x H], b1, W2 [H x H], b2, w3 [H], b3 [1]
    DBuf p, g, m1, m2;
    DBuf wt[3], w[3];   // BF16 layouts per GEMM layer
    // activations for a batch
    DBuf X, H1, H2, H3, dH1, dH2, dH3, y, t, loss;
    DBuf wpart, rpart;   // backward partial sums: per layer and split (weight gradients), per row block (loss)
    size_t wsplits = 0;  // splits each layer's region of wpart holds
    int wnz[3] = {0, 0, 0};   // splits the last backward wrote per layer
    DBuf cpart;          // bias-gradient partials [3][row blocks][H]
    DBuf Xtr, ttr;       // training: features and standardised targets of the whole training set
    int cap_tr = 0;
    int cap = 0;     // rows of X, H1..H3, y, t (forward)
    int cap_b = 0;   // rows of dH1..dH3 (backward)
    DBuf d_step;   // Adam step count (device, 1-based) and the Adam kernel's block counter
    int tc = 1;    // GEMM layers (forward, backward data, weight gradients) on tcgen05 (1, default) or mma.sync (0)
    DBuf d_status; // tcgen05 wait time-outs (bit 2)
    size_t off[9];   // block offsets of W0 b0 W1 b1 W2 b2 w3 b3, and the total
};

namespace {

constexpr size_t NPARAM = (size_t)H * IN + H + 2 * ((size_t)H * H + H) + H + 1;

// predictions run in chunks of at most this many rows, so the inference
// buffers stay bounded and are sized once
constexpr int PRED_CHUNK = 65536;

// weight gradients reduce over the batch: split it so that the 16 output
// tiles of a layer still fill the GPU
int wgrad_splits(int n) { return std::max(1, std::min(64, n / 64)); }

// activation buffers for n rows: forward ones always, backward ones when
// `bwd` (training); growing reallocates (and so synchronises the device),
// so callers that know their sizes reserve them up front
int sur_reserve(lkg_surrogate* S, int n, bool bwd) {
    if (n > S->cap) {
        const int m = S->cap > 0 ? std::max(n, S->cap + S->cap / 2) : n;   // grow geometrically
        const size_t nb = (size_t)m * sizeof(__nv_bfloat16);
        LKG_CK(S->X.reserve(nb * IN), "surrogate alloc");
        LKG_CK(S->H1.reserve(nb * H), "surrogate alloc");
        LKG_CK(S->H2.reserve(nb * H), "surrogate alloc");
        LKG_CK(S->H3.reserve(nb * H), "surrogate alloc");
        LKG_CK(S->y.reserve((size_t)m * sizeof(float)), "surrogate alloc");
        LKG_CK(S->t.reserve((size_t)m * sizeof(float)), "surrogate alloc");
        S->cap = m;
    }
    if (bwd && n > S->cap_b) {
        const int m = S->cap_b > 0 ? std::max(n, S->cap_b + S->cap_b / 2) : n;
        const size_t nb = (size_t)m * sizeof(__nv_bfloat16);
        LKG_CK(S->dH1.reserve(nb * H), "surrogate alloc");
        LKG_CK(S->dH2.reserve(nb * H), "surrogate alloc");
        LKG_CK(S->dH3.reserve(nb * H), "surrogate alloc");
        const size_t splits = std::max<size_t>(wgrad_splits(m), (size_t)(m + TCW_ROWS - 1) / TCW_ROWS);
        LKG_CK(S->wpart.reserve(splits * H * (IN + 2 * H) * sizeof(float)), "surrogate alloc");
        S->wsplits = splits;
        LKG_CK(S->rpart.reserve((size_t)((m + RL - 1) / RL) * (H + 2) * sizeof(float)), "surrogate alloc");
        LKG_CK(S->cpart.reserve((size_t)3 * ((m + RB - 1) / RB) * H * sizeof(float)), "surrogate alloc");
        S->cap_b = m;
    }
    return 0;
}

// split-K: rows of K per split (a multiple of BK) and the number of splits
int split_chunk(int K, int splits) { return ((K + splits - 1) / splits + BK - 1) / BK * BK; }
int split_count(int K, int splits) { return (K + split_chunk(K, splits) - 1) / split_chunk(K, splits); }

template <bool TA, bool TB, int EPI>
cudaError_t gemm(cudaStream_t s, int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
                 float* Cf, __nv_bfloat16* Cb, int ldc, const float* bias, const __nv_bfloat16* Hm, int splits = 1) {
    const int kc = split_chunk(K, splits);
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, split_count(K, splits));
    k_gemm<TA, TB, EPI><<<grid, 128, 0, s>>>(M, N, K, A, lda, B, ldb, Cf, Cb, ldc, bias, Hm, kc);
    return cudaGetLastError();
}

float* P(lkg_surrogate* S, int k) { return S->p.as<float>() + S->off[k]; }
// layer L's region of the weight-gradient partials (layers 0, 1, 2 in turn)
float* wpart_of(lkg_surrogate* S, int L) {
    return S->wpart.as<float>() + S->wsplits * H * (L == 0 ? 0 : (size_t)IN + (size_t)(L - 1) * H);
}

// forward of n feature rows already in S->X; y in S->y
// 2D tiled tensor map of a row-major [rows x K] bf16 matrix for the tcgen05
// kernel: boxes of 64 K elements x box_rows rows, 128-byte swizzled; the
// rows past `rows` read as zeros
bool tc_map(CUtensorMap* m, const void* base, int rows, int K, int box_rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    const cuuint32_t box[2] = {(cuuint32_t)TC_KS, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Y[n x 256] = epi(A[n x K] B^T), B [256 x K]
template <int EPI>
cudaError_t gemm_tc(lkg_surrogate* S, int n, int K, const __nv_bfloat16* A, const __nv_bfloat16* B, const float* b,
                    const __nv_bfloat16* Hm, __nv_bfloat16* Y) {
    if (n <= 0) return cudaSuccess;
    const int tiles = (n + TC_BM - 1) / TC_BM;
    if (EPI == EPI_FWD && tiles > S->ctx->sm_count && K % TC_KS == 0 && K <= TC_KMAX) {
        // more row tiles than SMs (large predictions): the persistent,
        // pipelined kernel, one CTA per SM
        alignas(64) CUtensorMap ma, mb;
        if (!tc_map(&ma, A, n, K, TC_BM) || !tc_map(&mb, B, TC_N, K, TC_N)) return cudaErrorInvalidValue;
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tc_pp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PP_SMEM);
        if (e != cudaSuccess) return e;
        k_gemm_tc_pp<<<S->ctx->sm_count, PP_THREADS, PP_SMEM, S->ctx->stream>>>(ma, mb, n, K, b, Y,
                                                                              S->d_status.as<int>());
        return cudaGetLastError();
    }
    // few row tiles (training batches): two CTAs of 128 columns per tile
    const bool split = 2 * tiles <= S->ctx->sm_count;
    const int tn = split ? 128 : TC_N;
    alignas(64) CUtensorMap ma, mb;
    if (K % TC_KS || K > TC_KMAX || !tc_map(&ma, A, n, K, TC_BM) || !tc_map(&mb, B, TC_N, K, tn))
        return cudaErrorInvalidValue;
    auto kern = split ? k_gemm_tc<EPI, 128> : k_gemm_tc<EPI, 256>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    if (e != cudaSuccess) return e;
    kern<<<dim3(tiles, TC_N / tn), 128, TC_SMEM, S->ctx->stream>>>(ma, mb, n, K, b, Hm, Y, S->d_status.as<int>());
    return cudaGetLastError();
}

// dW[H x kin] partials: part[split][o][i] = sum over the split's batch rows r
// of dC[r][o] * A_in[r][i]; returns the number of splits
cudaError_t wgrad_tc(lkg_surrogate* S, int n, int kin, const __nv_bfloat16* dC, const __nv_bfloat16* Ain, float* part,
                     int* nsplit) {
    const int splits = (n + TCW_ROWS - 1) / TCW_ROWS;
    *nsplit = splits;
    alignas(64) CUtensorMap ma, mb;
    if ((kin != 64 && kin != H) || !tc_map(&ma, dC, n, H, TCW_SLAB) || !tc_map(&mb, Ain, n, kin, TCW_SLAB))
        return cudaErrorInvalidValue;
    auto kern = kin == H ? k_wgrad_tc<256> : k_wgrad_tc<64>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TCW_SMEM);
    if (e != cudaSuccess) return e;
    kern<<<dim3(H / TC_BM, splits), 128, TCW_SMEM, S->ctx->stream>>>(ma, mb, n, part, S->d_status.as<int>());
    return cudaGetLastError();
}

// forward of n feature rows (X, default S->X): H1..H3, and with `head`
// the output y (training fuses the head into the loss kernel instead)
int forward(lkg_surrogate* S, int n, const __nv_bfloat16* X = nullptr, bool head = true) {
    cudaStream_t s = S->ctx->stream;
    if (!X) X = S->X.as<__nv_bfloat16>();
    if (S->tc) {
        LKG_CK(gemm_tc<EPI_FWD>(S, n, IN, X, S->wt[0].as<__nv_bfloat16>(), P(S, 1), nullptr,
                                S->H1.as<__nv_bfloat16>()), "mlp fwd tc");
        LKG_CK(gemm_tc<EPI_FWD>(S, n, H, S->H1.as<__nv_bfloat16>(), S->wt[1].as<__nv_bfloat16>(), P(S, 3), nullptr,
                                S->H2.as<__nv_bfloat16>()), "mlp fwd tc");
        LKG_CK(gemm_tc<EPI_FWD>(S, n, H, S->H2.as<__nv_bfloat16>(), S->wt[2].as<__nv_bfloat16>(), P(S, 5), nullptr,
                                S->H3.as<__nv_bfloat16>()), "mlp fwd tc");
    } else {
        LKG_CK((gemm<false, false, EPI_FWD>(s, n, H, IN, X, IN, S->wt[0].as<__nv_bfloat16>(), IN, nullptr,
                                            S->H1.as<__nv_bfloat16>(), H, P(S, 1), nullptr)), "mlp fwd");
        LKG_CK((gemm<false, false, EPI_FWD>(s, n, H, H, S->H1.as<__nv_bfloat16>(), H, S->wt[1].as<__nv_bfloat16>(), H,
                                            nullptr, S->H2.as<__nv_bfloat16>(), H, P(S, 3), nullptr)), "mlp fwd");
        LKG_CK((gemm<false, false, EPI_FWD>(s, n, H, H, S->H2.as<__nv_bfloat16>(), H, S->wt[2].as<__nv_bfloat16>(), H,
                                            nullptr, S->H3.as<__nv_bfloat16>(), H, P(S, 5), nullptr)), "mlp fwd");
    }
    S->ctx->launches += 3;
    if (head) {
        k_head<<<(n + 7) / 8, 256, 0, s>>>(S->H3.as<__nv_bfloat16>(), n, P(S, 6), P(S, 7), S->y.as<float>());
        LKG_CK(cudaGetLastError(), "mlp head");
        S->ctx->launches += 1;
    }
    return 0;
}

// backward of n rows after forward(head = false): the fused head and loss
// (y, dH3, the loss partials), then per layer the weight-gradient partials
// (each layer into its own region of wpart) and the backward-data product,
// then the bias partials of all three layers.
// X, t: the rows' features and standardised targets (default S->X, S->t).
// grad_step sums every gradient afterwards.
int backward(lkg_surrogate* S, int n, const __nv_bfloat16* X = nullptr, const float* t = nullptr) {
    cudaStream_t s = S->ctx->stream;
    if (!X) X = S->X.as<__nv_bfloat16>();
    if (!t) t = S->t.as<float>();
    const int nlblk = (n + RL - 1) / RL;
    k_loss_head<<<nlblk, H, 0, s>>>(t, S->H3.as<__nv_bfloat16>(), n, P(S, 6), P(S, 7), S->y.as<float>(),
                                    S->dH3.as<__nv_bfloat16>(), S->rpart.as<float>());
    LKG_CK(cudaGetLastError(), "mlp loss");
    const int splits = wgrad_splits(n);
    const __nv_bfloat16* acts[3] = {S->H1.as<__nv_bfloat16>(), S->H2.as<__nv_bfloat16>(), S->H3.as<__nv_bfloat16>()};
    __nv_bfloat16* dacts[3] = {S->dH1.as<__nv_bfloat16>(), S->dH2.as<__nv_bfloat16>(), S->dH3.as<__nv_bfloat16>()};
    for (int L = 2; L >= 0; --L) {
        const int kin = L == 0 ? IN : H;
        const __nv_bfloat16* ain = L == 0 ? X : acts[L - 1];
        // dW_L[o][i] = sum_n dC[n][o] * A_in[n][i]   (A = dC^T, B = A_in^T)
        int nz = 0;
        if (S->tc) {
            LKG_CK(wgrad_tc(S, n, kin, dacts[L], ain, wpart_of(S, L), &nz), "mlp wgrad tc");
        } else {
            LKG_CK((gemm<true, true, EPI_WGRAD>(s, H, kin, n, dacts[L], H, ain, kin, wpart_of(S, L), nullptr, kin,
                                                nullptr, nullptr, splits)), "mlp wgrad");
            nz = split_count(n, splits);
        }
        S->wnz[L] = nz;
        if (L > 0) {
            // dA_in[n][i] = (sum_o dC[n][o] W_L[o][i]) x ReLU'(A_in); w[L] is W_L^T [in x out]
            if (S->tc)
                LKG_CK(gemm_tc<EPI_BWD>(S, n, H, dacts[L], S->w[L].as<__nv_bfloat16>(), nullptr, acts[L - 1],
                                        dacts[L - 1]), "mlp bwd tc");
            else
                LKG_CK((gemm<false, false, EPI_BWD>(s, n, H, H, dacts[L], H, S->w[L].as<__nv_bfloat16>(), H, nullptr,
                                                    dacts[L - 1], H, nullptr, acts[L - 1])), "mlp bwd");
        }
    }
    const ColSums cs{{S->dH1.as<__nv_bfloat16>(), S->dH2.as<__nv_bfloat16>(), S->dH3.as<__nv_bfloat16>()},
                     S->cpart.as<float>()};
    k_colsum3<<<dim3((n + RB - 1) / RB, 3), H, 0, s>>>(cs, n);
    LKG_CK(cudaGetLastError(), "mlp bias grad");
    S->ctx->launches += 7;   // head and loss, 3 x weight-gradient partials, 2 x backward data, bias partials
    return 0;
}

// every gradient summed from the partials of backward(n rows) into S->g,
// the batch's loss added to S->loss, and with `apply` the Adam step (one
// launch)
int grad_step(lkg_surrogate* S, int n, bool apply, float lr = 0.f) {
    cudaStream_t s = S->ctx->stream;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    AdamLayers L;
    GradSums G;
    for (int k = 0; k < 3; ++k) {
        L.off[k] = (int)S->off[2 * k];
        L.cols[k] = k == 0 ? IN : H;
        L.wt[k] = S->wt[k].as<__nv_bfloat16>();
        L.w[k] = S->w[k].as<__nv_bfloat16>();
        G.wpart[k] = wpart_of(S, k);
        G.nz[k] = S->wnz[k];
    }
    G.cpart = S->cpart.as<float>();
    G.nblk = (n + RB - 1) / RB;
    G.lpart = S->rpart.as<float>();
    G.nlblk = (n + RL - 1) / RL;
    G.loss = S->loss.as<float>();
    const int np = (int)NPARAM;
    k_grad_adam<<<(np + 255) / 256, 256, 0, s>>>(S->p.as<float>(), S->g.as<float>(), S->m1.as<float>(),
                                                 S->m2.as<float>(), np, lr, b1, b2, eps, S->d_step.as<int>(), L, G,
                                                 apply ? 1 : 0);
    LKG_CK(cudaGetLastError(), "mlp grad / adam");
    S->ctx->launches += 1;
    return 0;
}

int refresh_bf16(lkg_surrogate* S) {
    cudaStream_t s = S->ctx->stream;
    for (int L = 0; L < 3; ++L) {
        const int k = 2 * L, cols = (L == 0) ? IN : H, n = H * cols;
        k_f2bf<<<(n + 255) / 256, 256, 0, s>>>(P(S, k), S->wt[L].as<__nv_bfloat16>(), n);
        k_f2bf_t<<<(n + 255) / 256, 256, 0, s>>>(P(S, k), S->w[L].as<__nv_bfloat16>(), H, cols);
    }
    LKG_CK(cudaGetLastError(), "mlp bf16 refresh");
    return 0;
}

// features of n device poses into S->X; with d_scores also their
// standardised targets into S->t (training)
// (into X_out / t_out instead when given: the training set's buffers)
int features(lkg_surrogate* S, int n, const double* d_poses, const double* d_scores = nullptr,
             __nv_bfloat16* X_out = nullptr, float* t_out = nullptr) {
    if (!X_out && sur_reserve(S, n, false)) return lkg_last_status();
    int st = sync_descriptors(S->ctx);
    if (st) return st;
    if (!X_out) X_out = S->X.as<__nv_bfloat16>();
    if (!t_out) t_out = S->t.as<float>();
    const int threads = 256, blocks = (int)(((size_t)n * NA + threads - 1) / threads);
    const TargetArgs tgt{d_scores, S->e_scale, S->t_mu, S->t_sd, d_scores ? t_out : nullptr};
    k_features<<<blocks, threads, 0, S->ctx->stream>>>(S->ctx->d_cx.as<ComplexDev>(), S->cid, d_poses, n,
                                                       S->anchors.as<int>(), S->tscale, X_out, tgt);
    LKG_CK(cudaGetLastError(), "features");
    S->ctx->launches++;
    return 0;
}

// predictions back to score units: the inverse of the standardised target
// t = (asinh(score / e_scale) - mu) / sd that k_features writes in training
__global__ void k_untarget(const float* __restrict__ y, int n, float e_scale, float mu, float sd, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)(sinhf(y[i] * sd + mu) * e_scale);
}

}  // namespace

extern "C" {

int lkg_surrogate_create(lkg_ctx* ctx, int complex_id, uint64_t seed, lkg_surrogate** out) {
    if (!ctx || !out || complex_id < 0 || complex_id >= (int)ctx->cx.size())
        return set_error(LKG_ERR_ARG, "bad surrogate arguments");
    cudaSetDevice(ctx->device);
    auto* S = new lkg_surrogate();
    S->ctx = ctx;
    S->cid = complex_id;
    const ComplexRec& cr = *ctx->cx[complex_id];
    // anchors: 16 ligand atoms spread by farthest-point sampling over the
    // (sorted) ligand reference coordinates
    const int nl = cr.d.nl;
    std::vector<float4> lp(nl);
    cudaMemcpy(lp.data(), cr.d.lpos, nl * sizeof(float4), cudaMemcpyDeviceToHost);
    std::vector<int> anc;
    std::vector<float> dmin(nl, 1e30f);
    int cur = 0;
    float rmax = 0.f;
    for (int i = 0; i < nl; ++i) rmax = std::max(rmax, std::sqrt(lp[i].x * lp[i].x + lp[i].y * lp[i].y + lp[i].z * lp[i].z));
    for (int a = 0; a < NA; ++a) {
        anc.push_back(cur);
        int best = 0;
        float bd = -1.f;
        for (int i = 0; i < nl; ++i) {
            float dx = lp[i].x - lp[cur].x, dy = lp[i].y - lp[cur].y, dz = lp[i].z - lp[cur].z;
            dmin[i] = std::min(dmin[i], dx * dx + dy * dy + dz * dz);
            if (dmin[i] > bd) { bd = dmin[i]; best = i; }
        }
        cur = best;
    }
    // translation scale: far-field box half-extent (receptor size + 30 A)
    S->tscale = std::max(20.f, 0.25f * (float)cr.d.fnx * (float)cr.d.fsp64);
    size_t sizes[8] = {(size_t)H * IN, H, (size_t)H * H, H, (size_t)H * H, H, H, 1};
    S->off[0] = 0;
    for (int k = 0; k < 8; ++k) S->off[k + 1] = S->off[k] + sizes[k];
    std::vector<float> p(NPARAM, 0.f);
    // He-uniform initialisation (deterministic LCG from `seed`)
    uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto u = [&]() {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return (double)(st >> 11) * (1.0 / 9007199254740992.0);
    };
    const int fan[4] = {IN, H, H, H};
    for (int L = 0; L < 4; ++L) {
        const double lim = std::sqrt(6.0 / fan[L]) * (L == 3 ? 0.5 : 1.0);
        for (size_t i = S->off[2 * L]; i < S->off[2 * L + 1]; ++i) p[i] = (float)((2.0 * u() - 1.0) * lim);
    }
    int rc = 0;
    cudaError_t e;
    if ((e = S->p.reserve(NPARAM * 4)) != cudaSuccess || (e = S->g.reserve(NPARAM * 4)) != cudaSuccess ||
        (e = S->m1.reserve(NPARAM * 4)) != cudaSuccess || (e = S->m2.reserve(NPARAM * 4)) != cudaSuccess ||
        (e = S->anchors.reserve(NA * sizeof(int))) != cudaSuccess || (e = S->loss.reserve(sizeof(float))) != cudaSuccess ||
        (e = S->d_step.reserve(2 * sizeof(int))) != cudaSuccess || (e = S->d_status.reserve(sizeof(int))) != cudaSuccess) {
        delete S;
        return set_error(cuda_to_status(e), "surrogate alloc: %s", cudaGetErrorString(e));
    }
    for (int L = 0; L < 3; ++L) {
        const size_t n = (size_t)H * (L == 0 ? IN : H) * sizeof(__nv_bfloat16);
        if ((e = S->wt[L].reserve(n)) != cudaSuccess || (e = S->w[L].reserve(n)) != cudaSuccess) {
            delete S;
            return set_error(cuda_to_status(e), "surrogate alloc: %s", cudaGetErrorString(e));
        }
    }
    cudaMemcpy(S->p.p, p.data(), NPARAM * 4, cudaMemcpyHostToDevice);
    cudaMemset(S->m1.p, 0, NPARAM * 4);
    cudaMemset(S->m2.p, 0, NPARAM * 4);
    const int one = 1;
    const int step0[2] = {one, 0};   // t = 1, no block done
    cudaMemcpy(S->d_step.p, step0, sizeof(step0), cudaMemcpyHostToDevice);
    cudaMemset(S->d_status.p, 0, sizeof(int));
    cudaMemcpy(S->anchors.p, anc.data(), NA * sizeof(int), cudaMemcpyHostToDevice);
    if ((rc = refresh_bf16(S))) { delete S; return rc; }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) {
        delete S;
        return set_error(cuda_to_status(e), "surrogate init: %s", cudaGetErrorString(e));
    }
    *out = S;
    return set_ok();
}

int lkg_surrogate_destroy(lkg_surrogate* S) {
    if (S) { cudaSetDevice(S->ctx->device); cudaStreamSynchronize(S->ctx->stream); }
    delete S;
    return set_ok();
}

// Fit the target standardisation to a set of exact scores (host array).
int lkg_surrogate_set_target_scale(lkg_surrogate* S, int n, const double* scores) {
    if (!S || n <= 0 || !scores) return set_error(LKG_ERR_ARG, "bad scale args");
    double e = 0.0;
    std::vector<double> a(n);
    for (int i = 0; i < n; ++i) a[i] = std::fabs(scores[i]);
    std::nth_element(a.begin(), a.begin() + n / 2, a.end());
    e = std::max(1.0, a[n / 2]);
    double mu = 0.0, sd = 0.0;
    for (int i = 0; i < n; ++i) mu += std::asinh(scores[i] / e);
    mu /= n;
    for (int i = 0; i < n; ++i) { double d = std::asinh(scores[i] / e) - mu; sd += d * d; }
    sd = std::sqrt(sd / n);
    S->e_scale = (float)e;
    S->t_mu = (float)mu;
    S->t_sd = (float)std::max(sd, 1e-3);
    return set_ok();
}

// Predicted scores (same units as lkg_score) for n device poses.
int lkg_surrogate_predict(lkg_surrogate* S, int n, const double* d_poses, double* d_pred) {
    if (!S || n < 0 || (n && (!d_poses || !d_pred))) return set_error(LKG_ERR_ARG, "bad predict args");
    if (n == 0) return set_ok();
    cudaSetDevice(S->ctx->device);
    int st;
    for (int b0 = 0; b0 < n; b0 += PRED_CHUNK) {
        const int m = std::min(PRED_CHUNK, n - b0);
        if ((st = features(S, m, d_poses + 7 * (size_t)b0))) return st;
        if ((st = forward(S, m))) return st;
        k_untarget<<<(m + 255) / 256, 256, 0, S->ctx->stream>>>(S->y.as<float>(), m, S->e_scale, S->t_mu, S->t_sd,
                                                                d_pred + b0);
        LKG_CK(cudaGetLastError(), "predict");
        S->ctx->launches++;
    }
    return set_ok();
}

// Buffers for predictions of up to n_predict poses per call and training
// batches of train_batch rows, allocated now rather than on first use.
int lkg_surrogate_reserve(lkg_surrogate* S, int n_predict, int train_batch) {
    if (!S || n_predict < 0 || train_batch < 0) return set_error(LKG_ERR_ARG, "bad reserve args");
    cudaSetDevice(S->ctx->device);
    const int nf = std::max(std::min(n_predict, PRED_CHUNK), train_batch);
    if (nf > 0 && sur_reserve(S, nf, false)) return lkg_last_status();
    if (train_batch > 0 && sur_reserve(S, train_batch, true)) return lkg_last_status();
    return set_ok();
}

// `epochs` passes of minibatch Adam over n device poses with exact scores;
// returns the last epoch's mean loss in *loss (standardised units).
int lkg_surrogate_train(lkg_surrogate* S, int n, const double* d_poses, const double* d_scores, int epochs,
                        int batch, float lr, float* loss_out) {
    if (!S || n <= 0 || !d_poses || !d_scores || epochs <= 0 || batch <= 0)
        return set_error(LKG_ERR_ARG, "bad train args");
    cudaSetDevice(S->ctx->device);
    cudaStream_t s = S->ctx->stream;
    batch = std::min(batch, n);
    int st;
    double last = 0.0;
    const int nb = n / batch;
    if ((st = sur_reserve(S, batch, true)) || (st = sync_descriptors(S->ctx))) return st ? st : lkg_last_status();
    // the features and targets of the whole set, once (they do not change
    // between epochs); then one epoch = per batch the forward layers, the
    // backward and one gradient / Adam launch (the loss is summed on the
    // device), captured once in a CUDA graph and replayed `epochs` times
    if (n > S->cap_tr) {
        LKG_CK(S->Xtr.reserve((size_t)n * IN * sizeof(__nv_bfloat16)), "surrogate alloc");
        LKG_CK(S->ttr.reserve((size_t)n * sizeof(float)), "surrogate alloc");
        S->cap_tr = n;
    }
    __nv_bfloat16* Xtr = S->Xtr.as<__nv_bfloat16>();
    float* ttr = S->ttr.as<float>();
    if ((st = features(S, n, d_poses, d_scores, Xtr, ttr))) return st;
    auto epoch = [&]() -> int {
        LKG_CK(cudaMemsetAsync(S->loss.p, 0, sizeof(float), s), "mlp loss clear");
        for (int b0 = 0; b0 + batch <= n; b0 += batch) {
            const __nv_bfloat16* xb = Xtr + (size_t)b0 * IN;
            int r;
            if ((r = forward(S, batch, xb, false))) return r;
            if ((r = backward(S, batch, xb, ttr + b0))) return r;
            if ((r = grad_step(S, batch, true, lr))) return r;
        }
        return 0;
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graphed = false;
    if (epochs > 1 && cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int r = epoch();
        const cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (r) { if (graph) cudaGraphDestroy(graph); return r; }
        if (e == cudaSuccess && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) graphed = true;
        else cudaGetLastError();
    }
    for (int ep = 0; ep < epochs; ++ep) {
        if (graphed) {
            const cudaError_t e = cudaGraphLaunch(exec, s);
            if (e != cudaSuccess) {
                cudaGraphExecDestroy(exec);
                cudaGraphDestroy(graph);
                return set_error(cuda_to_status(e), "training graph: %s", cudaGetErrorString(e));
            }
        } else if ((st = epoch())) {
            return st;
        }
    }
    float l = 0.f;
    cudaError_t e = cudaMemcpyAsync(&l, S->loss.p, sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_error(cuda_to_status(e), "train: %s", cudaGetErrorString(e));
    last = nb ? (double)l / nb : 0.0;
    if (loss_out) *loss_out = (float)last;
    return set_ok();
}

// Forward layers on tcgen05 (1, default) or on the mma.sync kernel (0).
int lkg_surrogate_set_backend(lkg_surrogate* S, int tcgen05) {
    if (!S) return set_error(LKG_ERR_ARG, "null surrogate");
    S->tc = tcgen05 ? 1 : 0;
    return set_ok();
}

// Kernel status bits since the last call (4: a tcgen05 accumulator wait ran
// out); cleared by the call.
int lkg_surrogate_status(lkg_surrogate* S, int* bits) {
    if (!S || !bits) return set_error(LKG_ERR_ARG, "bad status args");
    cudaSetDevice(S->ctx->device);
    LKG_CK(cudaStreamSynchronize(S->ctx->stream), "surrogate status");
    LKG_CK(cudaMemcpy(bits, S->d_status.p, sizeof(int), cudaMemcpyDeviceToHost), "surrogate status");
    LKG_CK(cudaMemset(S->d_status.p, 0, sizeof(int)), "surrogate status");
    return set_ok();
}

// Parameters (FP32 master, flat order W0 b0 W1 b1 W2 b2 w3 b3; W are [out][in]).
int64_t lkg_surrogate_nparams(void) { return (int64_t)NPARAM; }
int lkg_surrogate_get_params(lkg_surrogate* S, float* out) {
    if (!S || !out) return set_error(LKG_ERR_ARG, "bad args");
    LKG_CK(cudaMemcpy(out, S->p.p, NPARAM * 4, cudaMemcpyDeviceToHost), "get params");
    return set_ok();
}
int lkg_surrogate_set_params(lkg_surrogate* S, const float* in) {
    if (!S || !in) return set_error(LKG_ERR_ARG, "bad args");
    LKG_CK(cudaMemcpy(S->p.p, in, NPARAM * 4, cudaMemcpyHostToDevice), "set params");
    int st = refresh_bf16(S);
    if (st) return st;
    LKG_CK(cudaStreamSynchronize(S->ctx->stream), "set params");
    return set_ok();
}

// One forward + backward on n host feature rows (bf16 bit patterns) with
// host targets (already standardised): writes the standardised outputs,
// the flat gradient and the loss (for the gradient check against FP64).
int lkg_surrogate_grad(lkg_surrogate* S, int n, const uint16_t* feats, const float* targets, float* y_out,
                       float* grad_out, float* loss_out) {
    if (!S || n <= 0 || !feats || !targets) return set_error(LKG_ERR_ARG, "bad grad args");
    cudaSetDevice(S->ctx->device);
    if (sur_reserve(S, n, true)) return lkg_last_status();
    LKG_CK(cudaMemcpy(S->X.p, feats, (size_t)n * IN * 2, cudaMemcpyHostToDevice), "grad upload");
    LKG_CK(cudaMemcpy(S->t.p, targets, (size_t)n * 4, cudaMemcpyHostToDevice), "grad upload");
    LKG_CK(cudaMemsetAsync(S->loss.p, 0, sizeof(float), S->ctx->stream), "grad loss clear");
    int st;
    if ((st = forward(S, n, nullptr, false)) || (st = backward(S, n)) || (st = grad_step(S, n, false))) return st;
    LKG_CK(cudaStreamSynchronize(S->ctx->stream), "grad");
    if (y_out) LKG_CK(cudaMemcpy(y_out, S->y.p, (size_t)n * 4, cudaMemcpyDeviceToHost), "grad read");
    if (grad_out) LKG_CK(cudaMemcpy(grad_out, S->g.p, NPARAM * 4, cudaMemcpyDeviceToHost), "grad read");
    if (loss_out) LKG_CK(cudaMemcpy(loss_out, S->loss.p, 4, cudaMemcpyDeviceToHost), "grad read");
    return set_ok();
}

// Features of n device poses into a host array of bf16 bit patterns.
int lkg_surrogate_features(lkg_surrogate* S, int n, const double* d_poses, uint16_t* out) {
    if (!S || n <= 0 || !d_poses || !out) return set_error(LKG_ERR_ARG, "bad args");
    cudaSetDevice(S->ctx->device);
    int st = features(S, n, d_poses);
    if (st) return st;
    LKG_CK(cudaStreamSynchronize(S->ctx->stream), "features");
    LKG_CK(cudaMemcpy(out, S->X.p, (size_t)n * IN * 2, cudaMemcpyDeviceToHost), "features read");
    return set_ok();
}

}  // extern "C"
