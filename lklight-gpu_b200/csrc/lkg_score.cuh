// Fused pose-scoring kernels (sm_100a).
//
// One work unit = one tile of ligand atoms of one pose of one complex; one
// thread per ligand atom.  Per atom, in one pass:
//   (a) rigid transform x' = R(q) x + t in f64 (full_score.cu:255-268);
//   (b) far field q_j * phi(x') by trilinear interpolation
//       (full_score.cu:27-51 / grid_dna.rs:159-197);
//   (c) near scan over receptor atoms within 10 A: the fine cell grid turns
//       every (z, y) cell row inside the 10 A sphere into one contiguous span
//       of position-sorted receptor atoms, trimmed in x to the sphere, read
//       as coalesced float4 through the read-only path; for d^2 <= 100 the
//       clamped electrostatics, the capped Lennard-Jones and the heavy-atom
//       clash penalty (full_score.cu:296-315, dna.rs:947-968);
//   (d) cpydock only: the ligand atom's minimum distance to non-excluded
//       receptor atoms in registers and the receptor atoms' minima in a
//       shared-memory hash (atomicMin), reduced in the same kernel
//       (full_score.cu:477-569 merged; cpydock.rs:615-668).
// Per-pose sums: registers -> warp shuffles -> one shared array per block ->
// per-tile partials; the last tile of a pose to finish sums the partials in
// tile order, so results do not depend on scheduling (bitwise reproducible).
// Work units are fetched from a global counter by persistent blocks; the
// counters reset themselves at the end of each launch.
#pragma once
#include "lkg_internal.h"

namespace lkg {

// ------------------------------------------------------------------------
// precision traits
// ------------------------------------------------------------------------
template <typename R> struct Tr;
template <> struct Tr<float> {
    __device__ static float4 rpos(const ComplexDev& c, int k) { return __ldg(c.rpos + k); }
    __device__ static float4 rpar(const ComplexDev& c, int k) { return __ldg(c.rpar + k); }
    __device__ static float2 rsolv(const ComplexDev& c, int k) { return __ldg(c.rsolv + k); }
    __device__ static float4 lpos(const ComplexDev& c, int j) { return __ldg(c.lpos + j); }
    __device__ static float4 lpar(const ComplexDev& c, int j) { return __ldg(c.lpar + j); }
    __device__ static float2 lsolv(const ComplexDev& c, int j) { return __ldg(c.lsolv + j); }
};
template <> struct Tr<double> {
    __device__ static double4 rpos(const ComplexDev& c, int k) { return c.rpos64[k]; }
    __device__ static double4 rpar(const ComplexDev& c, int k) { return c.rpar64[k]; }
    __device__ static double2 rsolv(const ComplexDev& c, int k) { return c.rsolv64[k]; }
    __device__ static double4 lpos(const ComplexDev& c, int j) { return c.lpos64[j]; }
    __device__ static double4 lpar(const ComplexDev& c, int j) { return c.lpar64[j]; }
    __device__ static double2 lsolv(const ComplexDev& c, int j) { return c.lsolv64[j]; }
};

// ------------------------------------------------------------------------
// transform
// ------------------------------------------------------------------------
struct Rot { double m00, m01, m02, m10, m11, m12, m20, m21, m22, tx, ty, tz; };

__device__ __forceinline__ Rot pose_matrix(const double* __restrict__ pq) {
    // qt.rs:67-74 / full_score.cu:259-265; no normalisation (as the reference)
    double w = pq[0], x = pq[1], y = pq[2], z = pq[3];
    Rot r;
    r.m00 = 1. - 2. * (y * y + z * z); r.m01 = 2. * (x * y - w * z); r.m02 = 2. * (x * z + w * y);
    r.m10 = 2. * (x * y + w * z); r.m11 = 1. - 2. * (x * x + z * z); r.m12 = 2. * (y * z - w * x);
    r.m20 = 2. * (x * z - w * y); r.m21 = 2. * (y * z + w * x); r.m22 = 1. - 2. * (x * x + y * y);
    r.tx = pq[4]; r.ty = pq[5]; r.tz = pq[6];
    return r;
}

__device__ __forceinline__ void apply(const Rot& r, double vx, double vy, double vz,
                                      double& x, double& y, double& z) {
    // rot3_apply (qt.rs:122-128) then + t, left to right
    x = r.m00 * vx + r.m01 * vy + r.m02 * vz + r.tx;
    y = r.m10 * vx + r.m11 * vy + r.m12 * vz + r.ty;
    z = r.m20 * vx + r.m21 * vy + r.m22 * vz + r.tz;
}

// ------------------------------------------------------------------------
// far field
// ------------------------------------------------------------------------
// The grid is stored in bricks of 4 x 4 x 4 points (256 bytes: two 128-byte
// lines), bricks x-fastest, points x-fastest inside a brick.  A sample's 8
// corners then sit in one brick (or a few neighbouring ones), on 1-2 lines
// instead of the 4 rows of the x-fastest layout, and the samples of a
// compact ligand group share bricks.  Returns the offset of corner
// (ix, iy, iz) and the steps to its +x, +y and +z neighbours.
__device__ __forceinline__ size_t phi_brick_offsets(const ComplexDev& c, int ix, int iy, int iz, size_t& ox,
                                                    size_t& oy, size_t& oz) {
    const size_t bx = (size_t)c.fbx, bxy = (size_t)c.fbx * c.fby;
    ox = (ix & 3) == 3 ? 64 - 3 : 1;
    oy = (iy & 3) == 3 ? bx * 64 - 12 : 4;
    oz = (iz & 3) == 3 ? bxy * 64 - 48 : 16;
    return (((size_t)(iz >> 2) * bxy + (size_t)(iy >> 2) * bx + (size_t)(ix >> 2)) << 6) +
           (size_t)(((iz & 3) << 4) | ((iy & 3) << 2) | (ix & 3));
}
__device__ __forceinline__ float sample_phi(const ComplexDev& c, float x, float y, float z) {
    float fx = (x - c.fox) / c.fsp, fy = (y - c.foy) / c.fsp, fz = (z - c.foz) / c.fsp;
    // in the box iff 0 <= f < n - 1 per axis (ix + 1 < n); compared in float
    // so that inf / NaN / huge coordinates never reach the integer index
    if (!(fx >= 0.f && fy >= 0.f && fz >= 0.f && fx < (float)(c.fnx - 1) && fy < (float)(c.fny - 1) &&
          fz < (float)(c.fnz - 1)))
        return 0.f;
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    if (ix + 1 >= c.fnx || iy + 1 >= c.fny || iz + 1 >= c.fnz) return 0.f;
    float tx = fx - ix, ty = fy - iy, tz = fz - iz;
    size_t ox, oy, oz;
    const float* p = c.phi + phi_brick_offsets(c, ix, iy, iz, ox, oy, oz);
    float c000 = __ldg(p), c100 = __ldg(p + ox), c010 = __ldg(p + oy), c110 = __ldg(p + oy + ox);
    float c001 = __ldg(p + oz), c101 = __ldg(p + oz + ox), c011 = __ldg(p + oz + oy), c111 = __ldg(p + oz + oy + ox);
    float c00 = c000 * (1.f - tx) + c100 * tx, c10 = c010 * (1.f - tx) + c110 * tx;
    float c01 = c001 * (1.f - tx) + c101 * tx, c11 = c011 * (1.f - tx) + c111 * tx;
    float c0 = c00 * (1.f - ty) + c10 * ty, c1 = c01 * (1.f - ty) + c11 * ty;
    return c0 * (1.f - tz) + c1 * tz;
}

__device__ __forceinline__ double sample_phi(const ComplexDev& c, double x, double y, double z) {
    // grid_dna.rs:159-197 including the `tx as f32` weights
    double s = c.fsp64;
    double fx, fy, fz;
    if (c.finv64 != 0.0) {   // power-of-two spacing (0.5 A): the same quotient, no divisions
        fx = (x - c.fox64) * c.finv64; fy = (y - c.foy64) * c.finv64; fz = (z - c.foz64) * c.finv64;
    } else {
        fx = (x - c.fox64) / s; fy = (y - c.foy64) / s; fz = (z - c.foz64) / s;
    }
    double ix = floor(fx), iy = floor(fy), iz = floor(fz);
    if (ix < 0.0 || iy < 0.0 || iz < 0.0) return 0.0;
    if (!(ix < (double)(c.fnx - 1) && iy < (double)(c.fny - 1) && iz < (double)(c.fnz - 1))) return 0.0;
    long long ix0 = (long long)ix, iy0 = (long long)iy, iz0 = (long long)iz;
    if (ix0 + 1 >= c.fnx || iy0 + 1 >= c.fny || iz0 + 1 >= c.fnz) return 0.0;
    double tx = (double)(float)(fx - ix), ty = (double)(float)(fy - iy), tz = (double)(float)(fz - iz);
    size_t ox, oy, oz;
    const float* p = c.phi + phi_brick_offsets(c, (int)ix0, (int)iy0, (int)iz0, ox, oy, oz);
    double c000 = p[0], c100 = p[ox], c010 = p[oy], c110 = p[oy + ox];
    double c001 = p[oz], c101 = p[oz + ox], c011 = p[oz + oy], c111 = p[oz + oy + ox];
    double c00 = c000 * (1.0 - tx) + c100 * tx;
    double c10 = c010 * (1.0 - tx) + c110 * tx;
    double c01 = c001 * (1.0 - tx) + c101 * tx;
    double c11 = c011 * (1.0 - tx) + c111 * tx;
    double c0 = c00 * (1.0 - ty) + c10 * ty;
    double c1 = c01 * (1.0 - ty) + c11 * ty;
    return c0 * (1.0 - tz) + c1 * tz;
}

// ------------------------------------------------------------------------
// near scan: visit every receptor atom whose fine cell intersects the
// SCAN_R sphere around (x, y, z); rows are trimmed to the sphere.
// ------------------------------------------------------------------------
template <typename F>
__device__ __forceinline__ void scan_rows(const ComplexDev& c, float x, float y, float z, F&& visit) {
    const float R = SCAN_R, R2 = SCAN_R * SCAN_R;
    int cz0 = max(0, (int)floorf((z - R - c.oz) * c.inv_h));
    int cz1 = min(c.ncz - 1, (int)floorf((z + R - c.oz) * c.inv_h));
    for (int cz = cz0; cz <= cz1; ++cz) {
        float zlo = c.oz + cz * c.h;
        float dzm = fmaxf(0.f, fmaxf(zlo - z, z - (zlo + c.h)));
        float remz = R2 - dzm * dzm;
        if (remz < 0.f) continue;
        float wy = sqrtf(remz);
        int cy0 = max(0, (int)floorf((y - wy - c.oy) * c.inv_h));
        int cy1 = min(c.ncy - 1, (int)floorf((y + wy - c.oy) * c.inv_h));
        for (int cy = cy0; cy <= cy1; ++cy) {
            float ylo = c.oy + cy * c.h;
            float dym = fmaxf(0.f, fmaxf(ylo - y, y - (ylo + c.h)));
            float rem = remz - dym * dym;
            if (rem < 0.f) continue;
            float wx = sqrtf(rem);
            int cx0 = max(0, (int)floorf((x - wx - c.ox) * c.inv_hx));
            int cx1 = min(c.ncx - 1, (int)floorf((x + wx - c.ox) * c.inv_hx));
            if (cx0 > cx1) continue;
            int row = (cz * c.ncy + cy) * c.ncx;
            int b = __ldg(c.cell_start + row + cx0), e = __ldg(c.cell_start + row + cx1 + 1);
            for (int k = b; k < e; ++k) visit(k);
        }
    }
}

// ------------------------------------------------------------------------
// pair terms
// ------------------------------------------------------------------------
// The 10 A cutoff is the one discontinuity of the pair terms (a Coulomb
// term there is up to ~0.5 kcal/mol), so a pair whose f32 d^2 lies within
// NEAR_BAND of 100 is decided in f64, as the reference decides it: the slot
// atom's f64 position (its f32 value + rounding residual, ~2^-48 relative)
// against the receptor atom's f64 coordinates, without contraction.  The
// compensated f32 d^2 is off by ~1e-5 A^2 at most, far inside the band.
constexpr float NEAR_BAND = 1e-3f;
static __device__ __noinline__ bool near_exact(const ComplexDev& c, int k, float x, float xr, float y, float yr, float z,
                                           float zr) {
    const double4 a = c.rpos64[k];
    const double dx = __dsub_rn(__dadd_rn((double)x, (double)xr), a.x);
    const double dy = __dsub_rn(__dadd_rn((double)y, (double)yr), a.y);
    const double dz = __dsub_rn(__dadd_rn((double)z, (double)zr), a.z);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)) <= 100.0;
}

struct AtomAcc {
    double elec, vdw;   // per-atom sums
    int np;             // near pairs
};

__device__ __forceinline__ void pair_fast(unsigned flags, float qj, float svj, float rj, bool hj,
                                          const float4& a, const float4& pr, float d2,
                                          double& elec, double& vdw) {
    float ir2 = __fdividef(1.0f, d2);   // ~2 ulp; the f32 path's budget is ~1e-7 relative per term
    if (flags & F_ELEC) {
        // a clamped term is the exact f64 cap, as in the reference: its f32
        // rounding would otherwise add up over the many clamped pairs of a
        // clashing pose
        const float ae = qj * a.w * ir2;
        elec += ae >= ES_CAP_F ? ES_CAP_D : (ae <= -ES_CAP_F ? -ES_CAP_D : (double)ae);
    }
    float sv = svj * pr.x;
    float rr = rj + pr.y;
    float rr2 = rr * rr;
    float p6 = rr2 * rr2 * rr2 * (ir2 * ir2 * ir2);
    // (sv*p6)*(p6-2): finite for sv == 0 even where p6^2 would overflow
    float vp = fminf(sv * p6 * (p6 - 2.f), 1.0f);
    if ((flags & F_CLASH) && hj && pr.z != 0.f) {
        float d = d2 * rsqrtf(d2);
        float dmin = 0.75f * rr;
        if (d < dmin) vp += 6.f * (dmin - d);
    }
    vdw += (double)vp;
}

__device__ __forceinline__ double powi6(double x) { double x2 = x * x; double x4 = x2 * x2; return x2 * x4; }
__device__ __forceinline__ double powi3(double x) { double x2 = x * x; return x * x2; }

__device__ __forceinline__ void pair_exact(unsigned flags, int lj_form, double qj, double svj, double rj,
                                           double epsj, bool hj, const double4& a, const double4& pr,
                                           double d2, double& elec, double& vdw) {
    // dna.rs:947-968, pydock.rs:415-424, vdw.rs:129-137, cpydock.rs:630-639
    if (flags & F_ELEC) {
        double ae = qj * a.w / d2;
        if (ae < -ES_CAP_D) ae = -ES_CAP_D;
        if (ae > ES_CAP_D) ae = ES_CAP_D;
        elec += ae;
    }
    if (lj_form == LJ_SVDW) {
        double vdw_e = svj * pr.x;
        double vdw_r = rj + pr.y;
        double p6 = powi6(vdw_r) / powi3(d2);
        double v = fmin(vdw_e * (p6 * p6 - 2.0 * p6), 1.0);
        if ((flags & F_CLASH) && hj && pr.w != 0.0) {
            double d = sqrt(d2);
            double dmin = 0.75 * vdw_r;
            if (d < dmin) v += 6.0 * (dmin - d);
        }
        vdw += v;
    } else {
        double ve = sqrt(epsj * pr.z);
        double vr = rj + pr.y;
        double p6 = (lj_form == LJ_POW) ? pow(vr, 6.0) / pow(d2, 3.0) : powi6(vr) / powi3(d2);
        double k = ve * (p6 * p6 - 2.0 * p6);
        vdw += (k > 1.0) ? 1.0 : k;
    }
}

// g(min d^2) of the desolvation sum (cpydock.rs:648-668), asa > 0 atoms;
// the constant contribution of asa < 0 atoms is added on the host side
__device__ __forceinline__ double solv_term(double d2, double asa) {
    double sv = 0.0;
    if (d2 <= SOLV2_D && d2 > 0.0 && asa > 0.0) sv = -10.0 * sqrt(d2) + 65.0;
    if (sv > asa && asa > 0.0) sv = asa;
    return sv;
}

// receptor-minimum hash in shared memory (open addressing, bounded probes):
// key = position-sorted receptor index, value = f64 bits of the minimum d^2
// (non-negative doubles order like their bit patterns, so atomicMin works).
// Spill: as the fast kernel's table (MinHash64), a pose that fills the
// shared table continues in the block's global table (values, then keys;
// more slots than receptor atoms), whose keys are disjoint from the shared
// table's; the block empties the global slots when it sums them.
struct MinHash {
    static constexpr unsigned long long NOMIN = 0x7fefffffffffffffull;
    int* keys; unsigned long long* vals; int cap;
    int* skeys; unsigned long long* svals; int scap;   // the block's global table, or null
    int* spilled;
    __device__ void init(char* smem, int cap_, unsigned char* spill, int spill_cap, int* spilled_) {
        cap = cap_; vals = (unsigned long long*)smem; keys = (int*)(vals + cap);
        for (int s = threadIdx.x; s < cap; s += blockDim.x) { keys[s] = -1; vals[s] = NOMIN; }
        svals = spill ? reinterpret_cast<unsigned long long*>(spill) : nullptr;
        skeys = spill ? reinterpret_cast<int*>(svals + spill_cap) : nullptr;
        scap = spill_cap;
        spilled = spilled_;
        if (threadIdx.x == 0) *spilled = 0;
    }
    __device__ static bool put(int* kt, unsigned long long* vt, int n, int k, double d2) {
        unsigned h = ((unsigned)k * 2654435761u) & (unsigned)(n - 1);
        for (int probe = 0; probe < n; ++probe) {
            int prev = atomicCAS(kt + h, -1, k);
            if (prev == -1 || prev == k) {
                atomicMin(vt + h, (unsigned long long)__double_as_longlong(d2));
                return true;
            }
            h = (h + 1) & (unsigned)(n - 1);
        }
        return false;
    }
    __device__ bool insert(int k, double d2) {
        if (put(keys, vals, cap, k, d2)) return true;
        if (!skeys) return false;
        *spilled = 1;
        return put(skeys, svals, scap, k, d2);
    }
    __device__ double value(int s) const { return __longlong_as_double((long long)vals[s]); }
};

// ------------------------------------------------------------------------
// interface flags (restraints and membrane; dna.rs:885-897,970-973,
// scoring.rs:83-108): a pair within INTERFACE_CUTOFF sets the bits of both
// atoms' restraint residues and of the receptor atom's membrane bead
// ------------------------------------------------------------------------
// the pose's interface bits, or null when its complex has none; a launch
// without room for them flags status bit 2 (the host reports it)
__device__ __forceinline__ unsigned* iface_bits(const LaunchParams& p, const ComplexDev& c, long long g) {
    if (!c.iface_words) return nullptr;
    if (!p.iface || c.iface_words > p.iface_stride) { atomicOr(p.status, 2); return nullptr; }
    return p.iface + (size_t)g * p.iface_stride;
}

__device__ __forceinline__ void iface_set(unsigned* bits, int b) {
    if (b >= 0) atomicOr(bits + (b >> 5), 1u << (b & 31));
}

// receptor atom k (sorted order) and a ligand atom with tag lt at squared
// distance d2 (f64)
__device__ __forceinline__ void iface_mark(const ComplexDev& c, unsigned* bits, int k, int lt, double d2) {
    if (!(d2 <= IFACE2_D)) return;
    const int2 rt = c.rtag[k];
    iface_set(bits, rt.x);
    iface_set(bits, rt.y);
    iface_set(bits, lt);
}

// set bits in [a, b)
__device__ __forceinline__ int iface_count(const unsigned* bits, int a, int b) {
    int n = 0;
    for (int w = a >> 5; a < b && w <= ((b - 1) >> 5); ++w) {
        unsigned m = __ldcg(bits + w);
        const int lo = w * 32;
        if (a > lo) m &= ~0u << (a - lo);
        if (b < lo + 32) m &= (1u << (b - lo)) - 1u;
        n += __popc(m);
    }
    return n;
}

// the pose's restraint fractions and membrane intersection
// (satisfied_restraints, membrane_intersection: scoring.rs:83-108) applied
// to score s in the family's operation order, without contraction; the
// bits are cleared for the next launch.  f (optional): pr, pl, intersection
__device__ __forceinline__ double iface_apply(const ComplexDev& c, unsigned* bits, double s, double* f) {
    const int nr = c.nres_r, nl = c.nres_l, nm = c.nmem;
    const int cr = iface_count(bits, 0, nr), cl = iface_count(bits, nr, nr + nl);
    const int cm = iface_count(bits, nr + nl, nr + nl + nm);
    for (int w = 0; w < c.iface_words; ++w) bits[w] = 0u;
    const double pr = nr ? (double)cr / (double)nr : 0.0;
    const double pl = nl ? (double)cl / (double)nl : 0.0;
    const double inter = nm ? (double)cm / (double)nm : 0.0;
    const double pen = inter > 0.0 ? __dmul_rn(MEMBRANE_PENALTY, inter) : 0.0;
    if (f) { f[0] = pr; f[1] = pl; f[2] = inter; }
    switch (c.iface_form) {
        case IF_DNA: return __dadd_rn(s, __dsub_rn(__dadd_rn(__dmul_rn(pr, s), __dmul_rn(pl, s)), pen));
        case IF_VDW: return __dadd_rn(__dadd_rn(s, __dmul_rn(pr, s)), __dmul_rn(pl, s));
        default: return __dsub_rn(__dadd_rn(__dadd_rn(s, __dmul_rn(pr, s)), __dmul_rn(pl, s)), pen);
    }
}

// ------------------------------------------------------------------------
// per-atom work
// ------------------------------------------------------------------------
template <typename R> struct Atom;

// f32 path: f64 transform cast to f32 as the reference kernel does
template <> struct Atom<float> {
    template <bool DESOLV>
    __device__ static void run(const ComplexDev& c, const Rot& rot, int j, AtomAcc& acc,
                               double& min_l, MinHash* hash, int* status,
                               float* out_e, float* out_v, unsigned* ibits) {
        float4 b = Tr<float>::lpos(c, j);
        float4 lp = Tr<float>::lpar(c, j);
        double xd, yd, zd;
        {   // from the f64 base coordinates, as the reference transforms them
            const double4 b64 = c.lpos64[j];
            apply(rot, b64.x, b64.y, b64.z, xd, yd, zd);
        }
        // the f64 position as a float plus its rounding residual: x - a.x is
        // (nearly) exact for nearby atoms, so adding the residual keeps the
        // pair distance accurate to f32 rounding of the *difference*
        float x = (float)xd, y = (float)yd, z = (float)zd;
        const float xl = (float)(xd - (double)x), yl = (float)(yd - (double)y), zl = (float)(zd - (double)z);
        const float qj = b.w, svj = lp.x, rj = lp.y;
        const bool hj = lp.z != 0.f, lf = lp.w != 0.f;
        const unsigned flags = c.flags;
        double elec = 0.0, vdw = 0.0;
        // far field with the reference's f64 interpolation (per atom, cheap)
        if ((flags & F_FAR) && qj != 0.f) elec += c.lpos64[j].w * sample_phi(c, xd, yd, zd);
        int np = 0;
        const int lt = ibits ? c.ltag[j] : -1;
        scan_rows(c, x, y, z, [&](int k) {
            float4 a = Tr<float>::rpos(c, k);
            float dx = (x - a.x) + xl, dy = (y - a.y) + yl, dz = (z - a.z) + zl;
            float d2 = dx * dx + dy * dy + dz * dz;
            const bool in = fabsf(d2 - 100.f) < NEAR_BAND ? near_exact(c, k, x, xl, y, yl, z, zl) : d2 <= 100.f;
            if (in) {
                float4 pr = Tr<float>::rpar(c, k);
                ++np;
                pair_fast(flags, qj, svj, rj, hj, a, pr, d2, elec, vdw);
                // desolvation minima in f64 (the g(d^2) step at 6.4 A makes
                // f32 distances too coarse near the threshold); only pairs
                // that can be within 6.4 A pay for it
                if (DESOLV && !lf && pr.w == 0.f && d2 <= SOLV2_F * 1.001f) {
                    double4 a64 = c.rpos64[k];
                    double ex = xd - a64.x, ey = yd - a64.y, ez = zd - a64.z;
                    double d2d = ex * ex + ey * ey + ez * ez;
                    min_l = fmin(min_l, d2d);
                    if (d2d <= SOLV2_D && !hash->insert(k, d2d)) atomicOr(status, 1);
                }
                if (ibits && d2 <= IFACE2_F && ((__float_as_uint(pr.z) >> 31) || lt >= 0)) {
                    const double4 a64 = c.rpos64[k];
                    const double ex = xd - a64.x, ey = yd - a64.y, ez = zd - a64.z;
                    iface_mark(c, ibits, k, lt, ex * ex + ey * ey + ez * ez);
                }
            }
        });
        acc.elec += elec;
        acc.vdw += vdw;
        acc.np += np;
        if (out_e) { int o = c.lorig[j]; out_e[o] = (float)elec; out_v[o] = (float)vdw; }
    }
};

// f64 path: the reference CPU grid arithmetic
template <> struct Atom<double> {
    template <bool DESOLV>
    __device__ static void run(const ComplexDev& c, const Rot& rot, int j, AtomAcc& acc,
                               double& min_l, MinHash* hash, int* status,
                               float* out_e, float* out_v, unsigned* ibits) {
        double4 b = Tr<double>::lpos(c, j);
        double4 lp = Tr<double>::lpar(c, j);
        double x, y, z;
        apply(rot, b.x, b.y, b.z, x, y, z);
        const double qj = b.w, svj = lp.x, rj = lp.y, epsj = lp.z;
        const bool hj = lp.w != 0.0;
        const bool lf = DESOLV ? (Tr<float>::lpar(c, j).w != 0.f) : false;
        const unsigned flags = c.flags;
        const int lj_form = c.lj_form;
        double elec = 0.0, vdw = 0.0, far = 0.0;
        if ((flags & F_FAR) && qj != 0.0) far = qj * sample_phi(c, x, y, z);
        int np = 0;
        const int lt = ibits ? c.ltag[j] : -1;
        scan_rows(c, (float)x, (float)y, (float)z, [&](int k) {
            double4 a = Tr<double>::rpos(c, k);
            double dx = x - a.x, dy = y - a.y, dz = z - a.z;
            double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 <= 100.0) {
                double4 pr = Tr<double>::rpar(c, k);
                ++np;
                pair_exact(flags, lj_form, qj, svj, rj, epsj, hj, a, pr, d2, elec, vdw);
                if (DESOLV && !lf && __ldg(&c.rpar[k].w) == 0.f) {
                    min_l = fmin(min_l, d2);
                    if (d2 <= SOLV2_D && !hash->insert(k, d2)) atomicOr(status, 1);
                }
                if (ibits) iface_mark(c, ibits, k, lt, d2);
            }
        });
        acc.elec += elec + far;
        acc.vdw += vdw;
        acc.np += np;
        if (out_e) { int o = c.lorig[j]; out_e[o] = (float)(elec + far); out_v[o] = (float)vdw; }
    }
};

// ------------------------------------------------------------------------
// reductions
// ------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ long long warp_sum(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block sum of NV doubles into thread 0 (fixed order -> deterministic)
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*sred)[32]) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
    if (lane == 0)
#pragma unroll
        for (int i = 0; i < NV; ++i) sred[i][wid] = v[i];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += sred[i][w];
            v[i] = s;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ int find_item(const long long* __restrict__ work0, int n_items, long long w) {
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(work0 + mid) <= w) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// final per-pose output (family combination: gpu_score.rs:326-331,
// gpu_family.rs:283-308, cpydock.rs:789-791; CPU-grid cpydock adds the
// constant asa<0 term, cpydock.rs:648-668)
// With interface bits (ibits) the score is combined with the restraint
// fractions and the membrane penalty (iface_apply).
__device__ __forceinline__ void write_pose(const LaunchParams& p, const ComplexDev& c, long long g,
                                           double elec, double vdw, double solv, double np,
                                           unsigned* ibits = nullptr) {
    if (p.raw_pairs || p.solv_only) {
        if (p.raw_pairs) { p.scores[2 * g] = elec; p.scores[2 * g + 1] = vdw; }
        else p.scores[g] = solv;
        if (ibits) for (int w = 0; w < c.iface_words; ++w) ibits[w] = 0u;
    } else {
        double s;
        double ek = elec * FACTOR / EPSILON;
        if (c.flags & F_DESOLV) {
            double st = solv + c.solv_const;
            s = (ek + 0.1 * vdw - st) * -1.0;
            solv = st;
        } else if (!(c.flags & F_ELEC)) {
            s = vdw * -1.0;
        } else {
            s = -(ek + vdw);
        }
        if (ibits) s = iface_apply(c, ibits, s, p.iface_out ? p.iface_out + 3 * g : nullptr);
        p.scores[g] = s;
    }
    if (p.parts) {
        p.parts[4 * g] = elec; p.parts[4 * g + 1] = vdw; p.parts[4 * g + 2] = solv; p.parts[4 * g + 3] = np;
    }
}

__device__ __forceinline__ void finish_launch(const LaunchParams& p) {
    if (threadIdx.x == 0) {
        unsigned long long d = atomicAdd(p.work_counter + 1, 1ull);
        if (d == gridDim.x - 1) { p.work_counter[0] = 0ull; p.work_counter[1] = 0ull; }
    }
}

// ------------------------------------------------------------------------
// kernel 1: tiles of ligand atoms (dna / pydock / vdw and compat flags)
// ------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_score_tiles(LaunchParams p) {
    __shared__ long long s_work;
    __shared__ double s_red[4][32];
    for (;;) {
        if (threadIdx.x == 0) s_work = (long long)atomicAdd(p.work_counter, 1ull);
        __syncthreads();
        const long long w = s_work;
        __syncthreads();
        if (w >= p.total_work) break;
        const int b = find_item(p.item_work0, p.n_items, w);
        const ComplexDev& c = p.cx[__ldg(p.item_complex + b)];
        const long long local = w - __ldg(p.item_work0 + b);
        const int pose = (int)(local / c.ntiles), tile = (int)(local % c.ntiles);
        const long long g = (long long)__ldg(p.item_pose0 + b) + pose;
        if (p.pose_mask && !p.pose_mask[g]) continue;   // block-uniform: pose skipped
        const int j = tile * p.tile + threadIdx.x;
        AtomAcc acc{0.0, 0.0, 0};
        unsigned* ibits = iface_bits(p, c, g);
        if (j < c.nl && threadIdx.x < p.tile) {
            const Rot rot = pose_matrix(p.poses + 7 * g);
            double dummy_min = 0.0;
            const bool atom_out = p.atom_elec && b == 0 && pose == 0;
            Atom<R>::template run<false>(c, rot, j, acc, dummy_min, nullptr, p.status,
                                         atom_out ? p.atom_elec : nullptr, atom_out ? p.atom_vdw : nullptr, ibits);
        }
        if (ibits) __threadfence();   // interface bits before the unit is published
        double v[3] = {acc.elec, acc.vdw, (double)acc.np};
        block_sum<3>(v, s_red);
        if (threadIdx.x == 0) {
            // partial of work unit w; the pose's units are w - tile .. w - tile + ntiles - 1
            double* part = p.partials + (size_t)w * 4;
            part[0] = v[0]; part[1] = v[1]; part[2] = 0.0; part[3] = v[2];
            __threadfence();
            int done = atomicAdd(p.pose_counter + g, 1);
            if (done == c.ntiles - 1) {
                __threadfence();
                double e = 0.0, vv = 0.0, np = 0.0;
                const double* pp = p.partials + (size_t)(w - tile) * 4;
                for (int t = 0; t < c.ntiles; ++t) {
                    e += __ldcg(pp + 4 * t); vv += __ldcg(pp + 4 * t + 1); np += __ldcg(pp + 4 * t + 3);
                }
                write_pose(p, c, g, e, vv, 0.0, np, ibits);
                p.pose_counter[g] = 0;
            }
        }
    }
    finish_launch(p);
}

// ------------------------------------------------------------------------
// kernel 2: one block per pose, cpydock desolvation fused
// ------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(512) k_score_desolv(LaunchParams p) {
    extern __shared__ __align__(16) char smem[];
    __shared__ long long s_work;
    __shared__ double s_red[4][32];
    __shared__ long long s_fix[32];
    __shared__ int s_spilled;
    unsigned char* const spill = p.spill ? p.spill + (size_t)blockIdx.x * p.spill_cap * SPILL_SLOT_BYTES : nullptr;
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
        MinHash hash;
        hash.init(smem, c.hcap, spill, p.spill_cap, &s_spilled);
        __syncthreads();
        const Rot rot = pose_matrix(p.poses + 7 * g);
        unsigned* ibits = iface_bits(p, c, g);
        AtomAcc acc{0.0, 0.0, 0};
        double solv_l = 0.0;
        const bool want_pairs = !p.solv_only;
        for (int j = threadIdx.x; j < c.nl; j += blockDim.x) {
            double min_l = 1e300;
            AtomAcc a1{0.0, 0.0, 0};
            Atom<R>::template run<true>(c, rot, j, a1, min_l, &hash, p.status, nullptr, nullptr, ibits);
            if (want_pairs) { acc.elec += a1.elec; acc.vdw += a1.vdw; }
            acc.np += a1.np;
            double2 ls = c.lsolv64[j];
            solv_l += solv_term(min_l, ls.y) * ls.x;
        }
        __syncthreads();
        // receptor side: fixed-point (2^-40) sum over hash slots; slot order
        // depends on insertion races, integer sums do not
        long long fix = 0;
        for (int s = threadIdx.x; s < c.hcap; s += blockDim.x) {
            int k = hash.keys[s];
            if (k < 0) continue;
            double2 rs = c.rsolv64[k];
            fix += __double2ll_rn(solv_term(hash.value(s), rs.y) * rs.x * 1099511627776.0);
        }
        if (s_spilled)   // block-uniform: read after the barrier above
            for (int s = threadIdx.x; s < hash.scap; s += blockDim.x) {
                // the atomics acted in L2: read around L1
                const int k = __ldcg(hash.skeys + s);
                if (k < 0) continue;
                const double d2 = __longlong_as_double((long long)__ldcg(hash.svals + s));
                __stcg(hash.skeys + s, -1);                 // empty again for the block's next pose
                __stcg(hash.svals + s, MinHash::NOMIN);
                double2 rs = c.rsolv64[k];
                fix += __double2ll_rn(solv_term(d2, rs.y) * rs.x * 1099511627776.0);
            }
        fix = warp_sum(fix);
        if ((threadIdx.x & 31) == 0) s_fix[threadIdx.x >> 5] = fix;
        double v[4] = {acc.elec, acc.vdw, solv_l, (double)acc.np};
        block_sum<4>(v, s_red);   // contains __syncthreads: s_fix is complete
        if (threadIdx.x == 0) {
            long long f = 0;
            for (int i = 0; i < (int)((blockDim.x + 31) >> 5); ++i) f += s_fix[i];
            double solv = v[2] + (double)f * (1.0 / 1099511627776.0);
            write_pose(p, c, g, v[0], v[1], solv, v[3], ibits);
        }
        __syncthreads();
    }
    finish_launch(p);
}

}  // namespace lkg
