// Warp-independent fused scorer (f32 fast path, dna / pydock / vdw and the
// reference-compatible flag combinations).
//
// Every warp fetches its own work units from the global counter; there is
// no block-level barrier inside the loop, so a warp that meets a crowded
// interface never holds up the warps beside it.  A work unit is a tile of
// `p.tile` ligand atoms of one pose, split into groups of G consecutive
// atoms (spatially compact: the ligand is ordered by recursive coordinate
// bisection in groups of G) whose bounding sphere (centre, radius rho, in the
// ligand frame) is computed on the host.  Per group:
//   1. lanes 0..G-1 transform their atom in f64 (kept as an f32 value plus
//      the rounding residual), add the far-field term q * phi(x'), and park
//      position and parameters in one of two slot sets in shared memory
//      (the sets alternate between groups, so hits of one group can still be
//      queued while the next group is set up);
//   2. the receptor rows (z, y cells of edge h) within 10 A + rho of the
//      posed centre are enumerated 32 at a time (one per lane), trimmed in x
//      to sub-cells of edge h / xsub, and turned into contiguous atom spans;
//   3. 32 candidates at a time (lane -> span by a binary search over the
//      warp's exclusive prefix of span lengths, coalesced float4 loads, the
//      next chunk loaded while this one is tested) are tested against the G
//      slot atoms (broadcast shared-memory reads), slot by slot; a ballot
//      per slot appends that slot's hits (slot << 26 | receptor index) to
//      the warp's ring buffer in lane order;
//   4. while 32 or more hits are pending, each lane takes one and evaluates
//      the pair terms with compensated distances and the exact d^2 <= 100
//      test, accumulating in f64: the expensive math always runs on 32 lanes.
// The warp's sums are reduced by shuffles into one partial per work unit;
// the last unit of a pose sums the partials in tile order (deterministic:
// the hit order is fixed by the algorithm, not by scheduling).
#pragma once
#include "lkg_score.cuh"

namespace lkg {

constexpr int WK_THREADS = 128;   // 4 independent warps per block

// hit buffer: fewer than 64 pending hits (a batch of the plain kernel is 64
// hits, two a lane) are moved to its front after each candidate chunk, so
// the pending hits + the 32 x G hits of one chunk always fit
template <int G> struct WRing { static constexpr int N = 32 * G + 64; };

// resident blocks per SM the register budget is sized for: 64 registers a
// thread for G = 8, 72 for G = 16 (measured 1.4 % faster than 80 at 6
// blocks, 64 at 8 blocks 1.3 % slower), 80 for G = 32
template <int G> struct WOcc { static constexpr int N = (G <= 8) ? 8 : (G == 16 ? 7 : 6); };

// per-warp desolvation state of the two slot sets (cpydock): the slot
// atoms' f64 positions, their running minimum d^2 to non-excluded receptor
// atoms (f64 bits; non-negative doubles order like their bit patterns) and
// whether the ligand atom itself is excluded
template <int G>
struct WDes {
    double lx[2 * G], ly[2 * G], lz[2 * G];
    unsigned long long lmin[2 * G];
    int lf[2 * G];
};

// interface words a warp collects in shared memory before merging them into
// the pose's bits (larger sets go to HBM directly)
constexpr int W_IBUF = 32;
// hits of the packed pair path whose f32 d^2 lies within NEAR_BAND of the
// 10 A cutoff wait here for the f64 decision (the scalar pair path), which
// runs before their slot set is reused
constexpr int W_DEFER = 64;
// plain and interface kernels: candidates of the current group within its
// sphere (x, y, z relative to the group centre, receptor index in w), tested
// 32 at a time: a ring of 64, since fewer than 32 wait when a chunk of 32
// more arrives
constexpr int W_CQ = 64;
struct WQueue {
    float4 a[W_CQ];
};

template <int G>
struct WSlots {
    Rot rot;                    // pose of the current work unit
    float4 lpos[2 * G];         // x, y, z (f32 part), q
    float4 lres[2 * G];         // x, y, z residuals, sqrt eps
    float4 ltest[2 * G];        // candidate test: -2 l', |l'|^2 - 100.01 (l' = l - group centre)
    float2 lpar[2 * G];         // r, heavy
    int ltag[2 * G];            // IFACE: restraint bit of the slot atom, -1 = none
    unsigned* ibits;            // IFACE: interface bits of the current pose in HBM (null: none)
    unsigned* iset;             // IFACE: where pairs set them: ibuf, or ibits when the pose has more words
    unsigned ibuf[W_IBUF];      // IFACE: the unit's bits, merged into ibits once at the unit's end
    unsigned hit[WRing<G>::N];  // (slot << 26) | receptor index, pending hits first
    unsigned defer[W_DEFER];    // plain kernel: hits within f32 rounding of the cutoff, decided in f64 later
    int ndefer;
};

// Staged candidates (the plain kernel's TMA variant, selected per context):
// a window of STAGE_WIN receptor atoms (their float4 positions) copied from
// the row spans into shared memory by bulk copies (cp.async.bulk, no
// multicast) that complete on the warp's mbarrier.
constexpr int STAGE_WIN = 64;
struct WStage {
    float4 a[STAGE_WIN];
    unsigned long long bar;
    unsigned phase;   // parity of the barrier's current phase
};

__device__ __forceinline__ uint32_t w_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// bounded wait for phase `parity` of the mbarrier at `bar` (false: ran out)
__device__ __forceinline__ bool w_bar_wait(uint32_t bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred P1;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}\n"
                     : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

// Receptor-side minima of the fast cpydock kernel: one 64-bit word per slot,
// the minimum d^2 quantised to 37 bits (0 .. SOLV2_D in steps of 3e-10 A^2)
// above the 27-bit receptor index, so one atomicMin updates a slot (the key
// bits are equal) and a slot costs 8 bytes of shared memory instead of 12.
// Only pairs with d^2 <= SOLV2_D are inserted; the receptor term's
// sqrt(d^2) then moves by < 1e-10 A.
// Spill: a pose that touches more receptor atoms within 6.4 A than the
// shared table holds (a ligand sunk into a large receptor) continues in the
// block's own table in global memory, of more slots than the complex has
// receptor atoms, so an insert there always finds its key or an empty slot.
// A key enters the global table only after the shared table was found full
// without it, and a full shared table stays full, so the two tables hold
// disjoint keys and the receptor sum runs over both.  The block empties the
// global slots it used when it sums them.
struct MinHash64 {
    static constexpr unsigned long long EMPTY = ~0ull;
    static constexpr unsigned long long KEY_MASK = (1ull << 27) - 1;
    static constexpr double SCALE = (double)((1ull << 37) - 1) / SOLV2_D;
    unsigned long long* slot;
    int cap;
    unsigned long long* spill;   // the block's global table (all EMPTY between poses), or null
    int spill_cap;
    int* spilled;                // shared flag: the pose used the global table
    __device__ void init(char* smem, int cap_, unsigned long long* spill_, int spill_cap_, int* spilled_) {
        cap = cap_;
        slot = reinterpret_cast<unsigned long long*>(smem);
        spill = spill_;
        spill_cap = spill_cap_;
        spilled = spilled_;
        for (int s = threadIdx.x; s < cap; s += blockDim.x) slot[s] = EMPTY;
        if (threadIdx.x == 0) *spilled = 0;
    }
    // linear probing over tab[0..n) (n a power of two); false when full.
    // GLOBAL: the table is in global memory, where the atomics act in L2:
    // plain reads there bypass L1 (__ldcg), which could hold a stale line
    template <bool GLOBAL>
    __device__ static bool put(unsigned long long* tab, int n, int k, unsigned long long w) {
        unsigned h = ((unsigned)k * 2654435761u) & (unsigned)(n - 1);
        for (int probe = 0; probe < n; ++probe) {
            unsigned long long v = GLOBAL ? __ldcg(tab + h) : tab[h];
            if (v == EMPTY) {
                v = atomicCAS(tab + h, EMPTY, w);
                if (v == EMPTY) return true;
            }
            if ((v & KEY_MASK) == (unsigned long long)k) {
                atomicMin(tab + h, w);
                return true;
            }
            h = (h + 1) & (unsigned)(n - 1);
        }
        return false;
    }
    // k < 2^26 (the receptor index limit); 0 <= d2 <= SOLV2_D
    __device__ bool insert(int k, double d2) {
        const unsigned long long w = (__double2ull_rn(d2 * SCALE) << 27) | (unsigned long long)k;
        if (put<false>(slot, cap, k, w)) return true;
        if (!spill) return false;
        *spilled = 1;
        return put<true>(spill, spill_cap, k, w);
    }
    __device__ static int key_of(unsigned long long v) { return v == EMPTY ? -1 : (int)(v & KEY_MASK); }
    __device__ static double value_of(unsigned long long v) { return fmin((double)(v >> 27) / SCALE, SOLV2_D); }
    __device__ int key(int s) const { return key_of(slot[s]); }
    __device__ double value(int s) const { return value_of(slot[s]); }
};

// IFACE: start a unit of pose bits `bits` (lane 0; the caller syncs the
// warp after): collect in the warp's buffer when the pose fits in it
template <int G>
__device__ __forceinline__ void w_iface_begin(WSlots<G>& W, const ComplexDev& c, unsigned* bits) {
    W.ibits = bits;
    W.iset = !bits ? nullptr : (c.iface_words <= W_IBUF ? W.ibuf : bits);
}

// IFACE: merge the warp's buffer into the pose's bits and clear it (all
// lanes); the buffer is all zero between units
template <int G>
__device__ __forceinline__ void w_iface_flush(WSlots<G>& W, const ComplexDev& c) {
    __syncwarp();
    if (W.iset == W.ibuf)
        for (int w = (int)(threadIdx.x & 31); w < c.iface_words; w += 32) {
            const unsigned v = W.ibuf[w];
            if (v) { atomicOr(W.ibits + w, v); W.ibuf[w] = 0u; }
        }
    __syncwarp();
}

// 1 / x and 1 / sqrt(x) by the MUFU approximations alone (PTX rcp.approx /
// rsqrt.approx, flush-to-zero): the pair distances are far from f32
// denormals (d^2 >= ~1 A^2 for any real pair, <= 100 here), where these
// are within a few ulp, the budget of the f32 pair math
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// pair terms of one queued hit: the exact d^2 <= 100 test on the
// compensated d^2, then the reference formulas (those of pair_fast, with
// the LJ power taken as (rr^2 / d^2)^3) and the clash term selected instead
// of branched on.  DESOLV: pairs that can lie within 6.4 A also update both
// atoms' minimum distance in f64 (cpydock.rs:615-668), the ligand atom's in
// its slot, the receptor atom's in the block's hash.  IFACE: pairs that can
// lie within 3.9 A and involve a tagged atom are re-tested in f64 (the slot
// position as f32 value + residual, ~2^-48 relative) and set the pose's
// interface bits.
template <int G, bool DESOLV, bool IFACE>
__device__ __forceinline__ void w_pair(const ComplexDev& c, const WSlots<G>& W, WDes<G>* D, MinHash64* hash,
                                       int* status, unsigned e, unsigned flags, unsigned* iset, double& elec,
                                       double& vdw, int& np) {
    const int l = (int)(e >> 26), k = (int)(e & 0x3ffffffu);
    const float4 a = __ldg(c.rpos + k);
    const float4 pr = __ldg(c.rpar + k);
    const float4 lp = W.lpos[l], lr = W.lres[l];
    const float2 lq = W.lpar[l];
    const float dx = (lp.x - a.x) + lr.x, dy = (lp.y - a.y) + lr.y, dz = (lp.z - a.z) + lr.z;
    const float d2 = dx * dx + dy * dy + dz * dz;
    const bool in = fabsf(d2 - 100.f) < NEAR_BAND ? near_exact(c, k, lp.x, lr.x, lp.y, lr.y, lp.z, lr.z)
                                                  : d2 <= 100.f;
    if (!in) return;
    ++np;
    const float ir2 = rcp_approx(d2);
    if (flags & F_ELEC) {
        float ae = lp.w * a.w * ir2;
        ae = fminf(fmaxf(ae, -ES_CAP_F), ES_CAP_F);
        elec += (double)ae;
    }
    const float sv = lr.w * pr.x;
    const float rr = lq.x + pr.y;
    const float t = rr * rr * ir2;
    const float p6 = t * t * t;
    float vp = fminf(sv * p6 * (p6 - 2.f), 1.0f);
    if (flags & F_CLASH) {   // uniform per complex: the other families skip the distance
        const float d = d2 * rsqrt_approx(d2), dmin = 0.75f * rr;
        const bool clash = lq.y != 0.f && pr.z != 0.f && d < dmin;
        vp = clash ? vp + 6.f * (dmin - d) : vp;
    }
    vdw += (double)vp;
    if (DESOLV && !D->lf[l] && pr.w == 0.f && d2 <= SOLV2_F * 1.001f) {
        const double4 a64 = c.rpos64[k];
        const double ex = D->lx[l] - a64.x, ey = D->ly[l] - a64.y, ez = D->lz[l] - a64.z;
        const double d2d = ex * ex + ey * ey + ez * ez;
        atomicMin(&D->lmin[l], (unsigned long long)__double_as_longlong(d2d));
        if (d2d <= SOLV2_D && !hash->insert(k, d2d)) atomicOr(status, 1);
    }
    // tagged atoms carry the sign bit on their heavy flag (receptor: rpar.z,
    // set with the restraints; ligand slot: lpar.y), which the != 0 tests
    // above do not see: untagged pairs cost one test
    if (IFACE && iset && d2 <= IFACE2_F && ((__float_as_uint(pr.z) | __float_as_uint(lq.y)) >> 31)) {
        const int2 rt = __ldg(c.rtag + k);
        const int lt = W.ltag[l];
        {
            const double4 a64 = c.rpos64[k];
            double ex, ey, ez;
            if (DESOLV) { ex = D->lx[l] - a64.x; ey = D->ly[l] - a64.y; ez = D->lz[l] - a64.z; }
            else {
                ex = ((double)lp.x + (double)lr.x) - a64.x;
                ey = ((double)lp.y + (double)lr.y) - a64.y;
                ez = ((double)lp.z + (double)lr.z) - a64.z;
            }
            if (ex * ex + ey * ey + ez * ez <= IFACE2_D) {
                iface_set(iset, rt.x);
                iface_set(iset, rt.y);
                iface_set(iset, lt);
            }
        }
    }
}

// Packed pairs of f32 (Blackwell's f32x2 FADD / FMUL / FFMA: one instruction
// computes both lanes of the pair, each rounded as the scalar operation)
struct F2 { unsigned long long v; };
__device__ __forceinline__ F2 f2(float a, float b) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_get(F2 x, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v)); }
__device__ __forceinline__ F2 add2(F2 a, F2 b) { F2 r; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ F2 sub2(F2 a, F2 b) { F2 r; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ F2 mul2(F2 a, F2 b) { F2 r; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
    F2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}

// two queued hits a lane (the plain kernel, no desolvation, no interface
// bits): the pair terms of w_pair for hits e0 and e1 computed side by side
// on packed f32 pairs, which halves the FP32 instructions of the pair math.
// e1 counts only when v1 (a partial batch).  Same formulas as w_pair, per
// hit; d^2 is summed as (dx^2 + dy^2) + dz^2 with the squares of (x, y)
// taken as one packed pair, a difference of a few ulps from w_pair's
// fused chain (the f64 decision near the cutoff sees through it).
template <int G>
__device__ __forceinline__ void w_pair2(const ComplexDev& c, WSlots<G>& W, unsigned e0, unsigned e1, bool v1,
                                        unsigned flags, double& elec, double& vdw, int& np) {
    const int l0 = (int)(e0 >> 26), k0 = (int)(e0 & 0x3ffffffu);
    const int l1 = (int)(e1 >> 26), k1 = (int)(e1 & 0x3ffffffu);
    const float4 a0 = __ldg(c.rpos + k0), a1 = __ldg(c.rpos + k1);
    const float4 p0 = __ldg(c.rpar + k0), p1 = __ldg(c.rpar + k1);
    const float4 lp0 = W.lpos[l0], lp1 = W.lpos[l1], lr0 = W.lres[l0], lr1 = W.lres[l1];
    const float2 lq0 = W.lpar[l0], lq1 = W.lpar[l1];
    // per hit: (x, y) as one packed pair (the float4s' aligned halves), z scalar
    const F2 dxy0 = add2(sub2(f2(lp0.x, lp0.y), f2(a0.x, a0.y)), f2(lr0.x, lr0.y));
    const F2 dxy1 = add2(sub2(f2(lp1.x, lp1.y), f2(a1.x, a1.y)), f2(lr1.x, lr1.y));
    const float dz0 = (lp0.z - a0.z) + lr0.z, dz1 = (lp1.z - a1.z) + lr1.z;
    float sx0, sy0, sx1, sy1;
    f2_get(mul2(dxy0, dxy0), sx0, sy0);
    f2_get(mul2(dxy1, dxy1), sx1, sy1);
    const float d20 = fmaf(dz0, dz0, sy0 + sx0), d21 = fmaf(dz1, dz1, sy1 + sx1);
    const F2 d2 = f2(d20, d21);
    bool ok0 = d20 <= 100.f, ok1 = v1 && d21 <= 100.f;
    // a hit within f32 rounding of the cutoff leaves this path for the
    // deferred list (w_flush_deferred decides it in f64); were the list full
    // (W_DEFER such hits before their slot set is reused) it keeps the f32
    // decision
    if (__builtin_expect(fabsf(d20 - 100.f) < NEAR_BAND, 0)) {
        const int i = atomicAdd(&W.ndefer, 1);
        if (i < W_DEFER) { W.defer[i] = e0; ok0 = false; }
    }
    if (__builtin_expect(v1 && fabsf(d21 - 100.f) < NEAR_BAND, 0)) {
        const int i = atomicAdd(&W.ndefer, 1);
        if (i < W_DEFER) { W.defer[i] = e1; ok1 = false; }
    }
    np += (int)ok0 + (int)ok1;
    const F2 ir2 = f2(rcp_approx(d20), rcp_approx(d21));
    if (flags & F_ELEC) {
        float e0f, e1f;
        f2_get(mul2(mul2(f2(lp0.w, lp1.w), f2(a0.w, a1.w)), ir2), e0f, e1f);
        e0f = fminf(fmaxf(e0f, -ES_CAP_F), ES_CAP_F);
        e1f = fminf(fmaxf(e1f, -ES_CAP_F), ES_CAP_F);
        if (ok0) elec += (double)e0f;
        if (ok1) elec += (double)e1f;
    }
    const F2 sv = mul2(f2(lr0.w, lr1.w), f2(p0.x, p1.x));
    const F2 rr = add2(f2(lq0.x, lq1.x), f2(p0.y, p1.y));
    const F2 t = mul2(mul2(rr, rr), ir2);
    const F2 p6 = mul2(mul2(t, t), t);
    float v0, vv1;
    f2_get(mul2(mul2(sv, p6), sub2(p6, f2(2.f, 2.f))), v0, vv1);
    v0 = fminf(v0, 1.0f);
    vv1 = fminf(vv1, 1.0f);
    if (flags & F_CLASH) {
        const F2 d = mul2(d2, f2(rsqrt_approx(d20), rsqrt_approx(d21)));
        const F2 dmin = mul2(f2(0.75f, 0.75f), rr);
        float dd0, dd1, m0, m1, c0, c1;
        f2_get(d, dd0, dd1);
        f2_get(dmin, m0, m1);
        f2_get(fma2(f2(6.f, 6.f), sub2(dmin, d), f2(v0, vv1)), c0, c1);
        v0 = (lq0.y != 0.f && p0.z != 0.f && dd0 < m0) ? c0 : v0;
        vv1 = (lq1.y != 0.f && p1.z != 0.f && dd1 < m1) ? c1 : vv1;
    }
    if (ok0) vdw += (double)v0;
    if (ok1) vdw += (double)vv1;
}

// the deferred hits through the scalar pair path (which decides the cutoff
// in f64 near it); out of line: it runs only when such hits exist
template <int G>
__device__ __noinline__ void w_flush_deferred(const ComplexDev& c, WSlots<G>& W, unsigned flags, double& elec,
                                              double& vdw, int& np) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    const int n = min(W.ndefer, W_DEFER);
    for (int i = lane; i < n; i += 32)
        w_pair<G, false, false>(c, W, nullptr, nullptr, nullptr, W.defer[i], flags, nullptr, elec, vdw, np);
    __syncwarp();
    if (lane == 0) W.ndefer = 0;
    __syncwarp();
}

// receptor atom of candidate kk of the current rows: the span is the last
// row whose exclusive prefix is <= kk (empty rows never qualify ahead of the
// non-empty row that follows them); far away when kk is past the end
__device__ __forceinline__ void w_fetch(const ComplexDev& c, int st, int excl, int total, int kk, float4& a,
                                        int& ridx) {
    int rr = 0;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const int v = __shfl_sync(0xffffffffu, excl, rr + s);
        if (v <= kk) rr += s;
    }
    const int rst = __shfl_sync(0xffffffffu, st, rr), rex = __shfl_sync(0xffffffffu, excl, rr);
    ridx = rst + (kk - rex);
    a = kk < total ? __ldg(c.rpos + ridx) : make_float4(3e30f, 3e30f, 3e30f, 0.f);
}

constexpr unsigned long long W_NOMIN = 0x7fefffffffffffffull;   // largest finite double

// lower bound of the distance from (x, y, z) to the nearest receptor atom
// (ComplexDev::rlb; rlb_m outside its grid)
__device__ __forceinline__ float w_receptor_bound(const ComplexDev& c, float x, float y, float z) {
    const int ix = (int)floorf((x - c.rlbox) * c.rlb_inv);
    const int iy = (int)floorf((y - c.rlboy) * c.rlb_inv);
    const int iz = (int)floorf((z - c.rlboz) * c.rlb_inv);
    if (ix < 0 || iy < 0 || iz < 0 || ix >= c.rlbx || iy >= c.rlby || iz >= c.rlbz) return c.rlb_m;
    return __ldg(c.rlb + ((size_t)iz * c.rlby + iy) * c.rlbx + ix);
}


// The warp's sums over its groups.
struct WAcc {
    double elec = 0.0, vdw = 0.0, solv = 0.0;
    int np = 0;
};

// Scores groups g_first, g_first + g_step, ... (< g_end) of one pose whose
// rotation is in W.rot, into acc (per lane).  DESOLV also adds each slot
// atom's g(min d^2) * des to acc.solv once its hits are all evaluated.
template <int G, bool DESOLV, bool IFACE, bool STAGE = false>
__device__ __forceinline__ void w_groups(const ComplexDev& c, WSlots<G>& W, WDes<G>* D, MinHash64* hash, int* status,
                                         int g_first, int g_end, int g_step, WAcc& acc, WQueue* Q,
                                         WStage* S = nullptr, bool far_sep = false) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const unsigned flags = c.flags;
    const int nl = c.nl;
    unsigned* const iset = IFACE ? W.iset : nullptr;   // set by the caller for the unit
    // hits [head, tail) are pending; hits [head, prev_start) belong to the
    // group before the previous one (whose slot set the next group reuses)
    int head = 0, tail = 0, prev_start = 0;
    int jdes0 = -1, jdes1 = -1;   // DESOLV: this lane's slot atom in set 0 / set 1
    // the plain kernel evaluates 64 hits a batch (two a lane, packed f32
    // pairs); the desolvation and interface kernels 32 (one a lane)
    constexpr bool PAIR2 = !DESOLV && !IFACE;
    constexpr int BATCH = PAIR2 ? 64 : 32;
    auto drain_partial = [&]() {
        const int n = tail - head;
        if (n > lane) {
            if (PAIR2)
                w_pair2<G>(c, W, W.hit[head + lane], lane + 32 < n ? W.hit[head + 32 + lane] : W.hit[head + lane],
                           lane + 32 < n, flags, acc.elec, acc.vdw, acc.np);
            else
                w_pair<G, DESOLV, IFACE>(c, W, D, hash, status, W.hit[head + lane], flags, iset, acc.elec, acc.vdw,
                                         acc.np);
        }
        head = tail;
    };
    auto finalize = [&](int set) {   // DESOLV: the slot set's minima are final
        const int j = set ? jdes1 : jdes0;
        if (DESOLV && lane < G && j >= 0) {
            const double2 ls = c.lsolv64[j];
            acc.solv += solv_term(__longlong_as_double((long long)D->lmin[set + lane]), ls.y) * ls.x;
        }
        if (set) jdes1 = -1; else jdes0 = -1;
    };
    int it = 0;
    for (int grp = g_first; grp < g_end; grp += g_step, ++it) {
        const int set = (it & 1) * G;
        // slot set `set` last served the group before the previous one, whose
        // hits were queued before the previous group started: evaluate any
        // still pending
        if (prev_start > head) drain_partial();
        if (PAIR2) {   // the deferred hits, before their slot set is reused
            __syncwarp();
            if (W.ndefer) w_flush_deferred<G>(c, W, flags, acc.elec, acc.vdw, acc.np);
        }
        prev_start = tail;
        __syncwarp();
        finalize(set);
        // 1. the group's ligand atoms
        if (lane < G) {
            const int j = grp * G + lane;
            const bool valid = j < nl;
            const float4 b4 = valid ? __ldg(c.lpos + j) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 lp4 = valid ? __ldg(c.lpar + j) : make_float4(0.f, 0.f, 0.f, 0.f);
            double xd, yd, zd;
            {   // from the f64 base coordinates, as the reference transforms them
                const double4 b64 = valid ? c.lpos64[j] : make_double4(0.0, 0.0, 0.0, 0.0);
                apply(W.rot, b64.x, b64.y, b64.z, xd, yd, zd);
            }
            float x = (float)xd, y = (float)yd, z = (float)zd;
            const float4 res = make_float4((float)(xd - (double)x), (float)(yd - (double)y),
                                           (float)(zd - (double)z), lp4.x);
            // far field with the reference's f64 interpolation (a per-atom
            // cost; f32 here would add up over thousands of charged atoms)
            // (the cpydock kernel takes it from k_far_poses instead when
            // that pass ran: far_sep)
            if (valid && (flags & F_FAR) && !(DESOLV && far_sep) && b4.w != 0.f)
                acc.elec += c.lpos64[j].w * sample_phi(c, xd, yd, zd);
            if (!valid) { x = y = z = 1e30f; }   // never within reach of a receptor atom
            W.lpos[set + lane] = make_float4(x, y, z, b4.w);
            W.lres[set + lane] = res;
            const int ltg = (IFACE && valid && c.ltag) ? __ldg(c.ltag + j) : -1;
            W.lpar[set + lane] = make_float2(lp4.y, ltg >= 0 ? -lp4.z : lp4.z);   // -0 or -1 when tagged
            if (IFACE) W.ltag[set + lane] = ltg;
            if (DESOLV) {
                D->lx[set + lane] = xd; D->ly[set + lane] = yd; D->lz[set + lane] = zd;
                D->lmin[set + lane] = W_NOMIN;
                D->lf[set + lane] = lp4.w != 0.f;
                if (set) jdes1 = valid ? j : -1; else jdes0 = valid ? j : -1;
            }
        }
        // 2. receptor rows within reach of the group sphere
        const float4 gs = __ldg(c.lgrp + grp);
        double cxd, cyd, czd;
        apply(W.rot, (double)gs.x, (double)gs.y, (double)gs.z, cxd, cyd, czd);
        const float gx = (float)cxd, gy = (float)cyd, gz = (float)czd;
        if (lane < G) {
            // candidate test |a' - l'|^2 <= 100.01 as |a'|^2 - 2 a'.l' +
            // |l'|^2 in the group frame (|a'| <= ~20 A: rounding ~1e-4,
            // far inside the 0.01 margin); invalid slots never pass
            const float4 lp = W.lpos[set + lane];
            const float lx = lp.x - gx, ly = lp.y - gy, lz = lp.z - gz;
            const bool far_slot = !(lp.x < 1e29f);
            W.ltest[set + lane] = far_slot ? make_float4(0.f, 0.f, 0.f, 3e30f)
                                           : make_float4(-2.f * lx, -2.f * ly, -2.f * lz,
                                                         lx * lx + ly * ly + lz * lz - 100.01f);
        }
        __syncwarp();
        const float R = SCAN_R + gs.w, R2 = R * R;
        // cpydock kernel: no receptor atom within R of the centre, so the
        // group has no candidate and its rows are not enumerated (most groups
        // of a large ligand at the interface: with a 12,000-atom ligand on a
        // 101,000-atom receptor the step is 4.5 % faster; the plain kernel,
        // whose ligands are smaller, measured 1 % slower with the test)
        if (DESOLV && c.rlb && R < c.rlb_m && w_receptor_bound(c, gx, gy, gz) > R) continue;
        const int cz0 = max(0, (int)floorf((gz - R - c.oz) * c.inv_h));
        const int cz1 = min(c.ncz - 1, (int)floorf((gz + R - c.oz) * c.inv_h));
        const int cy0 = max(0, (int)floorf((gy - R - c.oy) * c.inv_h));
        const int cy1 = min(c.ncy - 1, (int)floorf((gy + R - c.oy) * c.inv_h));
        const int nyr = cy1 - cy0 + 1, nzr = cz1 - cz0 + 1;
        const int nbox = (nyr > 0 && nzr > 0) ? nyr * nzr : 0;
        const float inv_nyr = 1.0f / (float)max(nyr, 1);
        const unsigned enc_set = (unsigned)set << 26;
        // 3. queued candidates, 32 a time: each lane tests its candidate
        //    (relative to the group centre) against the group's slots and
        //    appends its hits
        auto test_chunk = [&](const float ax, const float ay, const float az, const int ridx) {
            const float aa = ax * ax + ay * ay + az * az;
            // the lane's candidate against every slot: a bit per hit
            unsigned m = 0;
#pragma unroll
            for (int l = 0; l < G; ++l) {
                const float4 t = W.ltest[set + l];
                // |a'|^2 - 2 a'.l' <= -(|l'|^2 - 100.01): three FMAs, the
                // slot's constant on the right (invalid slots: -3e30)
                const float q = fmaf(ax, t.x, fmaf(ay, t.y, fmaf(az, t.z, aa)));
                m |= (q <= -t.w ? 1u : 0u) << l;
            }
            // lane-major append: each lane writes its hits (slot order)
            // at the warp's exclusive prefix of the hit counts
            const int nh = __popc(m);
            int inc = nh;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, inc, o);
                if (lane >= o) inc += v;
            }
            const int chunk_hits = __shfl_sync(FULL, inc, 31);
            if (chunk_hits == 0) return;
            unsigned* dst = W.hit + tail + (inc - nh);
            const unsigned enc = (unsigned)ridx | enc_set;
#pragma unroll
            for (int l = 0; l < G; ++l)
                if (m & (1u << l)) *dst++ = enc + ((unsigned)l << 26);
            tail += chunk_hits;
            __syncwarp();
            // 4. full batches
            while (tail - head >= BATCH) {
                if (PAIR2)
                    w_pair2<G>(c, W, W.hit[head + lane], W.hit[head + 32 + lane], true, flags, acc.elec,
                               acc.vdw, acc.np);
                else
                    w_pair<G, DESOLV, IFACE>(c, W, D, hash, status, W.hit[head + lane], flags, iset, acc.elec,
                                             acc.vdw, acc.np);
                head += BATCH;
            }
            // keep the buffer linear: the < BATCH pending hits move to its front
            if (head > 0) {
                const int rem = tail - head;
                const unsigned v = lane < rem ? W.hit[head + lane] : 0u;
                const unsigned v2 = (PAIR2 && lane + 32 < rem) ? W.hit[head + 32 + lane] : 0u;
                __syncwarp();
                if (lane < rem) W.hit[lane] = v;
                if (PAIR2 && lane + 32 < rem) W.hit[32 + lane] = v2;
                __syncwarp();
                prev_start = max(prev_start - head, 0);
                tail = rem;
                head = 0;
            }
        };
        // a candidate farther than R from the group centre is more than 10 A
        // from every slot atom (|l'| <= rho).  The plain and interface
        // kernels queue only the candidates within R (the row spans' corners
        // outside the sphere, about 40 % of the candidates with 6 A cells,
        // then cost no slot tests); the cpydock kernel, short of shared
        // memory and L1, tests whole chunks and skips those with none within R
        int q_head = 0, q_tail = 0;
        auto chunk = [&](const float4 a, const int ridx) {
            const float ax = a.x - gx, ay = a.y - gy, az = a.z - gz;
            const bool in = ax * ax + ay * ay + az * az <= R2;
            if (DESOLV) {
                if (__any_sync(FULL, in)) test_chunk(ax, ay, az, ridx);
                return;
            }
            const unsigned b = __ballot_sync(FULL, in);
            if (in)
                Q->a[(q_tail + __popc(b & lt_mask)) & (W_CQ - 1)] = make_float4(ax, ay, az, __int_as_float(ridx));
            q_tail += __popc(b);
            if (q_tail - q_head >= 32) {
                __syncwarp();
                const float4 q = Q->a[(q_head + lane) & (W_CQ - 1)];
                q_head += 32;
                test_chunk(q.x, q.y, q.z, __float_as_int(q.w));
            }
        };
        for (int r0 = 0; r0 < nbox; r0 += 32) {
            const int r = r0 + lane;
            int st = 0, len = 0;
            if (r < nbox) {
                // r = zz * nyr + yy; (r + 0.5) / nyr is at least 0.5 / nyr
                // away from an integer, far above the f32 rounding error
                const int zz = (int)(((float)r + 0.5f) * inv_nyr), yy = r - zz * nyr;
                const int cz = cz0 + zz, cy = cy0 + yy;
                const float zlo = c.oz + cz * c.h, ylo = c.oy + cy * c.h;
                const float dzm = fmaxf(0.f, fmaxf(zlo - gz, gz - (zlo + c.h)));
                const float dym = fmaxf(0.f, fmaxf(ylo - gy, gy - (ylo + c.h)));
                const float rem = R2 - dzm * dzm - dym * dym;
                if (rem >= 0.f) {
                    const float wx = sqrtf(rem);
                    const int cx0 = max(0, (int)floorf((gx - wx - c.ox) * c.inv_hx));
                    const int cx1 = min(c.ncx - 1, (int)floorf((gx + wx - c.ox) * c.inv_hx));
                    if (cx0 <= cx1) {
                        const int row = (cz * c.ncy + cy) * c.ncx;
                        st = __ldg(c.cell_start + row + cx0);
                        len = __ldg(c.cell_start + row + cx1 + 1) - st;
                    }
                }
            }
            int inc = len;   // inclusive prefix of the span lengths
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, inc, o);
                if (lane >= o) inc += v;
            }
            const int total = __shfl_sync(FULL, inc, 31);
            const int excl = inc - len;
            if (!STAGE) {
                // the next chunk's receptor atoms are fetched (through L1)
                // while the current one is tested
                float4 an = make_float4(3e30f, 3e30f, 3e30f, 0.f);
                int rn = 0;
                if (total > 0) w_fetch(c, st, excl, total, lane, an, rn);
                for (int k0 = 0; k0 < total; k0 += 32) {
                    const float4 a = an;
                    const int ridx = rn;
                    if (k0 + 32 < total) w_fetch(c, st, excl, total, k0 + 32 + lane, an, rn);
                    chunk(a, ridx);
                }
            } else {
                // windows of STAGE_WIN candidates: every row span's part of
                // the window is bulk-copied into shared memory by its lane
                const uint32_t bar = w_smem_u32(&S->bar);
                for (int w0 = 0; w0 < total; w0 += STAGE_WIN) {
                    const int wn = min(STAGE_WIN, total - w0);
                    const int lo = max(excl, w0), hi = min(excl + len, w0 + wn);
                    __syncwarp();   // the previous window is read
                    if (lane == 0)
                        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                                     :: "r"(bar), "r"((uint32_t)wn * 16u) : "memory");
                    __syncwarp();
                    if (hi > lo) {
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        asm volatile(
                            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                            :: "r"(w_smem_u32(S->a + (lo - w0))),
                               "l"(reinterpret_cast<uint64_t>(c.rpos + st + (lo - excl))),
                               "r"((uint32_t)(hi - lo) * 16u), "r"(bar) : "memory");
                    }
                    const unsigned ph = S->phase;
                    if (!w_bar_wait(bar, ph)) {
                        // ran out: report, and wait (bounded again) for the copies in flight
                        if (lane == 0) atomicOr(status, 8);
                        w_bar_wait(bar, ph);
                    }
                    __syncwarp();
                    if (lane == 0) S->phase = ph ^ 1u;
                    __syncwarp();
                    for (int k0 = w0; k0 < w0 + wn; k0 += 32) {
                        const int kk = k0 + lane;
                        int rr = 0;
#pragma unroll
                        for (int sft = 16; sft > 0; sft >>= 1) {
                            const int v = __shfl_sync(FULL, excl, rr + sft);
                            if (v <= kk) rr += sft;
                        }
                        const int ridx = __shfl_sync(FULL, st, rr) + (kk - __shfl_sync(FULL, excl, rr));
                        const float4 a = kk < w0 + wn ? S->a[kk - w0] : make_float4(3e30f, 3e30f, 3e30f, 0.f);
                        chunk(a, ridx);
                    }
                }
            }
        }
        // the queue's remainder (the lanes past it test a far candidate)
        if (!DESOLV && q_tail > q_head) {
            __syncwarp();
            const int n = q_tail - q_head;
            const float4 q = lane < n ? Q->a[(q_head + lane) & (W_CQ - 1)] : make_float4(3e30f, 3e30f, 3e30f, 0.f);
            test_chunk(q.x, q.y, q.z, __float_as_int(q.w));
        }
    }
    __syncwarp();
    drain_partial();
    __syncwarp();
    if (PAIR2 && W.ndefer) w_flush_deferred<G>(c, W, flags, acc.elec, acc.vdw, acc.np);
    finalize(0);
    finalize(G);
}

// STAGE: the candidates reach shared memory by bulk copies (WStage) instead
// of L1 loads (selected per context; the measured alternative)
template <int G, bool IFACE, bool STAGE = false>
__global__ void __launch_bounds__(WK_THREADS, WOcc<G>::N) k_score_warp(LaunchParams p) {
    static_assert(G == 4 || G == 8 || G == 16 || G == 32, "group size");
    static_assert(!(STAGE && IFACE), "the staged variant is the plain kernel's");
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char wk_smem[];
    const int lane = threadIdx.x & 31;
    WSlots<G>& W = reinterpret_cast<WSlots<G>*>(wk_smem)[threadIdx.x >> 5];
    WQueue* Q = reinterpret_cast<WQueue*>(wk_smem + (WK_THREADS / 32) * sizeof(WSlots<G>)) + (threadIdx.x >> 5);
    WStage* S = STAGE ? reinterpret_cast<WStage*>(wk_smem + (WK_THREADS / 32) * (sizeof(WSlots<G>) + sizeof(WQueue))) +
                            (threadIdx.x >> 5)
                      : nullptr;
    if (STAGE) {
        if (lane == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(w_smem_u32(&S->bar)), "r"(1));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            S->phase = 0u;
        }
        __syncwarp();
    }
    if (IFACE) W.ibuf[lane] = 0u;
    if (lane == 0) W.ndefer = 0;
    __syncwarp();
    for (;;) {
        unsigned long long wq = 0;
        if (lane == 0) wq = atomicAdd(p.work_counter, 1ull);
        const long long w = (long long)__shfl_sync(FULL, wq, 0);
        if (w >= p.total_work) break;
        const int b = find_item(p.item_work0, p.n_items, w);
        const ComplexDev& c = p.cx[__ldg(p.item_complex + b)];
        const long long local = w - __ldg(p.item_work0 + b);
        const int ntiles = c.ntiles;
        const int pose = (int)(local / ntiles), tile = (int)(local % ntiles);
        const long long g = (long long)__ldg(p.item_pose0 + b) + pose;
        if (p.pose_mask && !p.pose_mask[g]) continue;   // pose skipped: keeps its score
        __syncwarp();   // readers of the previous unit's pose are done
        if (lane == 0) {
            W.rot = pose_matrix(p.poses + 7 * g);
            if (IFACE) w_iface_begin(W, c, iface_bits(p, c, g));
            else if (c.iface_words) atomicOr(p.status, 2);   // a launch without room for the bits
        }
        __syncwarp();
        const int gpt = p.tile / G;
        const int g0 = tile * gpt, g1 = min(g0 + gpt, (c.nl + G - 1) / G);
        WAcc acc;
        w_groups<G, false, IFACE, STAGE>(c, W, nullptr, nullptr, p.status, g0, g1, 1, acc, Q, S);
        if (IFACE && W.ibits) {
            w_iface_flush(W, c);
            __threadfence();   // interface bits before the unit is published
        }
        const double elec = warp_sum(acc.elec), vdw = warp_sum(acc.vdw);
        const long long npl = warp_sum((long long)acc.np);
        if (lane == 0) {
            // partial of work unit w; the pose's units are w - tile .. w - tile + ntiles - 1
            double* part = p.partials + (size_t)w * 4;
            part[0] = elec; part[1] = vdw; part[2] = 0.0; part[3] = (double)npl;
            __threadfence();
            const int done = atomicAdd(p.pose_counter + g, 1);
            if (done == ntiles - 1) {
                __threadfence();
                double e = 0.0, vv = 0.0, nps = 0.0;
                const double* pp = p.partials + (size_t)(w - tile) * 4;
                for (int t = 0; t < ntiles; ++t) {
                    e += __ldcg(pp + 4 * t); vv += __ldcg(pp + 4 * t + 1); nps += __ldcg(pp + 4 * t + 3);
                }
                write_pose(p, c, g, e, vv, 0.0, nps, IFACE ? W.ibits : nullptr);
                p.pose_counter[g] = 0;
            }
        }
    }
    __syncthreads();   // every warp of the block has left the work loop
    finish_launch(p);
}

// cpydock: one block per pose (the receptor-side minima live in the block's
// shared-memory hash); warp k takes the pose's groups k, k + NW, ... (a fixed
// assignment: the sums do not depend on scheduling).  Block layout of the
// dynamic shared memory: hash (hcap x 8 B), then NW x WSlots, NW x WDes.
// 8 warps a block, three blocks an SM (24 warps resident, 80 registers):
// the block's warps wait for one another at the end of every pose, and
// with 8 warps a pose instead of 12 that wait is shorter (a 12,000-atom
// ligand on a 101,000-atom receptor: 30.9 against 32.3 ms a step; 4 warps
// at 5 blocks: 34.2 ms).
constexpr int WD_THREADS = 256;
constexpr int WD_BLOCKS = 3;

template <int G>
__host__ __device__ constexpr size_t wd_smem(int hcap) {
    return (size_t)hcap * sizeof(unsigned long long) + (size_t)(WD_THREADS / 32) * (sizeof(WSlots<G>) + sizeof(WDes<G>));
}

template <int G, bool IFACE>
__global__ void __launch_bounds__(WD_THREADS, WD_BLOCKS) k_score_warp_desolv(LaunchParams p) {
    constexpr int NW = WD_THREADS / 32;
    extern __shared__ __align__(16) unsigned char wd_smem_raw[];
    __shared__ long long s_work;
    __shared__ double s_red[4][32];
    __shared__ long long s_fix[32];
    __shared__ int s_spilled;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long* const spill =
        p.spill ? reinterpret_cast<unsigned long long*>(p.spill + (size_t)blockIdx.x * p.spill_cap * SPILL_SLOT_BYTES)
                : nullptr;
    for (;;) {
        if (threadIdx.x == 0) s_work = (long long)atomicAdd(p.work_counter, 1ull);
        __syncthreads();
        const long long w = s_work;
        __syncthreads();
        if (w >= p.total_work) break;
        const int b = find_item(p.item_work0, p.n_items, w);
        const ComplexDev& c = p.cx[__ldg(p.item_complex + b)];
        const int pose = (int)(w - __ldg(p.item_work0 + b));
        const long long g = (long long)__ldg(p.item_pose0 + b) + pose;
        if (p.pose_mask && !p.pose_mask[g]) continue;   // block-uniform: pose skipped
        MinHash64 hash;
        hash.init(reinterpret_cast<char*>(wd_smem_raw), c.hcap, spill, p.spill_cap, &s_spilled);
        unsigned char* base = wd_smem_raw + (size_t)c.hcap * sizeof(unsigned long long);
        WSlots<G>& W = reinterpret_cast<WSlots<G>*>(base)[wid];
        WDes<G>* D = reinterpret_cast<WDes<G>*>(base + (size_t)NW * sizeof(WSlots<G>)) + wid;
        if (IFACE) W.ibuf[lane] = 0u;   // the slots move with the complex's hash size
        if (lane == 0) {
            W.rot = pose_matrix(p.poses + 7 * g);
            if (IFACE) w_iface_begin(W, c, iface_bits(p, c, g));
            else if (c.iface_words) atomicOr(p.status, 2);
        }
        __syncthreads();   // hash cleared, poses set
        WAcc acc;
        w_groups<G, true, IFACE>(c, W, D, &hash, p.status, wid, (c.nl + G - 1) / G, NW, acc, nullptr, nullptr,
                                 p.far != nullptr);
        if (IFACE && W.ibits) w_iface_flush(W, c);   // before the block's barrier below
        __syncthreads();   // every pair has updated the hash
        // receptor side: fixed-point (2^-40) sum over hash slots; slot order
        // depends on insertion races, integer sums do not
        long long fix = 0;
        for (int s = threadIdx.x; s < c.hcap; s += blockDim.x) {
            const int k = hash.key(s);
            if (k < 0) continue;
            const double2 rs = c.rsolv64[k];
            fix += __double2ll_rn(solv_term(hash.value(s), rs.y) * rs.x * 1099511627776.0);
        }
        if (s_spilled)   // block-uniform: read after the barrier above
            for (int s = threadIdx.x; s < p.spill_cap; s += blockDim.x) {
                const unsigned long long v = __ldcg(spill + s);
                if (v == MinHash64::EMPTY) continue;
                __stcg(spill + s, MinHash64::EMPTY);   // empty again for the block's next pose
                const int k = MinHash64::key_of(v);
                const double2 rs = c.rsolv64[k];
                fix += __double2ll_rn(solv_term(MinHash64::value_of(v), rs.y) * rs.x * 1099511627776.0);
            }
        fix = warp_sum(fix);
        if (lane == 0) s_fix[wid] = fix;
        double v[4] = {acc.elec, acc.vdw, acc.solv, (double)acc.np};
        block_sum<4>(v, s_red);   // contains __syncthreads: s_fix is complete
        if (threadIdx.x == 0) {
            long long f = 0;
            for (int i = 0; i < NW; ++i) f += s_fix[i];
            const double far = p.far ? __ldcg(p.far + g) : 0.0;   // k_far_poses' far field, when it ran
            write_pose(p, c, g, p.solv_only ? 0.0 : v[0] + far, p.solv_only ? 0.0 : v[1],
                       v[2] + (double)f * (1.0 / 1099511627776.0), v[3], IFACE ? W.ibits : nullptr);
        }
        __syncthreads();
    }
    finish_launch(p);
}

// The far field of the cpydock launch group as its own pass, before the
// fused kernel: one block per pose, each thread a fixed stride of ligand
// atoms (the f64 transform of the f64 base coordinates and the reference's
// f64 interpolation, as the fused kernel does it), then a block sum in a
// fixed order into far[pose] (deterministic).  Inside the fused kernel the
// 8 grid gathers of every charged atom waited on memory with only 24 warps
// per SM resident; here every thread has independent gathers in flight.
// Skipped (masked) poses are left alone.
constexpr int FAR_THREADS = 256;
__global__ void __launch_bounds__(FAR_THREADS, 4) k_far_poses(LaunchParams p) {
    __shared__ double s_red[4][32];
    for (long long w = blockIdx.x; w < p.total_work; w += gridDim.x) {
        const int b = find_item(p.item_work0, p.n_items, w);
        const ComplexDev& c = p.cx[__ldg(p.item_complex + b)];
        const long long g = (long long)__ldg(p.item_pose0 + b) + (w - __ldg(p.item_work0 + b));
        if (p.pose_mask && !p.pose_mask[g]) continue;   // block-uniform
        double v[1] = {0.0};
        if (c.flags & F_FAR) {
            const Rot rot = pose_matrix(p.poses + 7 * g);
            for (int j = threadIdx.x; j < c.nl; j += FAR_THREADS) {
                if (__ldg(&c.lpos[j].w) == 0.f) continue;
                const double4 b64 = c.lpos64[j];
                double xd, yd, zd;
                apply(rot, b64.x, b64.y, b64.z, xd, yd, zd);
                v[0] += b64.w * sample_phi(c, xd, yd, zd);
            }
        }
        block_sum<1>(v, s_red);
        if (threadIdx.x == 0) p.far[g] = v[0];
    }
}

}  // namespace lkg
