// Oracle: CPU restatement of LKlight's CPU grid scoring path, GSO and RNG.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h).  Written to follow the reference's
// arithmetic operation by operation so that results match its f64 code to the
// last bit where the reference is deterministic:
//   * no FMA contraction (built with -ffp-contract=off), left-to-right sums;
//   * f64::powi(x, n) restated as LLVM expands it (binary method:
//     x^6 = x^2 * x^4, x^3 = x * x^2);
//   * f64::min / f64::clamp NaN semantics (fmin ignores NaN, clamp keeps it);
//   * the far field's f32 accumulation order (atom by atom) and its
//     `tx as f32` interpolation weights.
// Paths cited below are relative to the LKlight-GPU source tree.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <unordered_map>
#include <vector>
#include <immintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// rand 0.7.3 StdRng = rand_chacha 0.2 ChaCha20 (djb variant: 64-bit block
// counter, 64-bit stream id = 0), seeded by rand_core 0.5.1 seed_from_u64,
// which fills the 32-byte key with 8 PCG32 (XSH-RR) outputs.  Restated from
// the published ChaCha20 and PCG32 descriptions; pinned by qt.rs:474-488.
// ---------------------------------------------------------------------------
struct Rng {
    uint32_t key[8];
    uint64_t counter = 0;      // next block to generate
    uint32_t buf[64];          // 4 blocks, as rand_chacha buffers them
    int idx = 64;
};

inline uint32_t rotl32(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }

void chacha_block(const uint32_t key[8], uint64_t ctr, uint32_t out[16]) {
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                      key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                      (uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u};
    uint32_t x[16];
    memcpy(x, s, sizeof(x));
#define QR(a, b, c, d)                       \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16); \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12); \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);  \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
    for (int r = 0; r < 10; ++r) {
        QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
        QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
    }
#undef QR
    for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

void rng_seed(Rng& r, uint64_t state) {
    const uint64_t MUL = 6364136223846793005ull, INC = 11634580027462260723ull;
    for (int i = 0; i < 8; ++i) {
        state = state * MUL + INC;
        uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
        uint32_t rot = (uint32_t)(state >> 59);
        r.key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
    }
    r.counter = 0;
    r.idx = 64;
}

void rng_refill(Rng& r) {
    for (int b = 0; b < 4; ++b) chacha_block(r.key, r.counter + b, r.buf + 16 * b);
    r.counter += 4;
    r.idx = 0;
}

uint64_t rng_u64(Rng& r) {  // rand_core BlockRng::next_u64 (even index path)
    if (r.idx >= 64) rng_refill(r);
    if (r.idx == 63) {          // straddle (only after an odd number of u32 reads)
        uint64_t lo = r.buf[63];
        rng_refill(r);
        uint64_t hi = r.buf[0];
        r.idx = 1;
        return (hi << 32) | lo;
    }
    uint64_t lo = r.buf[r.idx], hi = r.buf[r.idx + 1];
    r.idx += 2;
    return (hi << 32) | lo;
}

double rng_f64(Rng& r) {  // rand 0.7 Standard for f64: 53 high bits * 2^-53
    return (double)(rng_u64(r) >> 11) * (1.0 / 9007199254740992.0);
}

// ---------------------------------------------------------------------------
// Quaternion helpers (src/qt.rs)
// ---------------------------------------------------------------------------
struct Quat { double w, x, y, z; };

void q_normalize(Quat& q) {  // qt.rs:36-46
    double n = std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    q.w /= n; q.x /= n; q.y /= n; q.z /= n;
}

Quat q_slerp(Quat q1, Quat q2, double t) {  // qt.rs:80-104
    q_normalize(q1);
    q_normalize(q2);
    double dot = q1.w * q2.w + q1.x * q2.x + q1.y * q2.y + q1.z * q2.z;
    if (dot < 0.0) {
        q1 = Quat{-q1.w, -q1.x, -q1.y, -q1.z};
        dot *= -1.0;
    }
    if (dot > 0.9995) {  // LINEAR_THRESHOLD (constants.rs:11)
        Quat r{q1.w + (q2.w - q1.w) * t, q1.x + (q2.x - q1.x) * t,
               q1.y + (q2.y - q1.y) * t, q1.z + (q2.z - q1.z) * t};
        q_normalize(r);
        return r;
    }
    dot = std::fmax(std::fmin(dot, 1.0), -1.0);
    double omega = std::acos(dot);
    double so = std::sin(omega);
    double a = std::sin((1.0 - t) * omega) / so;
    double b = std::sin(t * omega) / so;
    return Quat{q1.w * a + q2.w * b, q1.x * a + q2.x * b, q1.y * a + q2.y * b, q1.z * a + q2.z * b};
}

void q_matrix(const Quat& q, double m[3][3]) {  // qt.rs:67-74
    double w = q.w, x = q.x, y = q.y, z = q.z;
    m[0][0] = 1. - 2. * (y * y + z * z); m[0][1] = 2. * (x * y - w * z); m[0][2] = 2. * (x * z + w * y);
    m[1][0] = 2. * (x * y + w * z); m[1][1] = 1. - 2. * (x * x + z * z); m[1][2] = 2. * (y * z - w * x);
    m[2][0] = 2. * (x * z - w * y); m[2][1] = 2. * (y * z + w * x); m[2][2] = 1. - 2. * (x * x + y * y);
}

inline void rot3_apply(const double m[3][3], const double v[3], double out[3]) {  // qt.rs:122-128
    out[0] = m[0][0] * v[0] + m[0][1] * v[1] + m[0][2] * v[2];
    out[1] = m[1][0] * v[0] + m[1][1] * v[1] + m[1][2] * v[2];
    out[2] = m[2][0] * v[0] + m[2][1] * v[1] + m[2][2] * v[2];
}

// f64::powi as LLVM expands a constant exponent (binary method)
inline double powi6(double x) { double x2 = x * x; double x4 = x2 * x2; return x2 * x4; }
inline double powi3(double x) { double x2 = x * x; return x * x2; }
// f64::clamp: NaN passes through
inline double clampd(double v, double lo, double hi) { if (v < lo) v = lo; if (v > hi) v = hi; return v; }

// ---------------------------------------------------------------------------
// Receptor far field (src/grid_dna.rs:25-209)
// ---------------------------------------------------------------------------
const double CLOSE_DIST = 10.0;
const double FIELD_RMAX = 30.0;
const double SPACING = 0.5;

struct Field {
    double origin[3];
    int64_t n[3];
    double spacing;
    int fp64;
    std::vector<float> phi;
    std::vector<double> phi64;
};

// Grid extent of ReceptorField::new (grid_dna.rs:44-70): 30 A + 2 spacings
// beyond the atoms, floored / ceiled to whole Angstroms.
void field_extent(const double* coords, int64_t na, double lo[3], int64_t n[3]) {
    double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int a = 0; a < 3; ++a) lo[a] = INFINITY;
    for (int64_t i = 0; i < na; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::fmin(lo[a], coords[3 * i + a]);
            hi[a] = std::fmax(hi[a], coords[3 * i + a]);
        }
    for (int a = 0; a < 3; ++a) {
        lo[a] = std::floor(lo[a] - FIELD_RMAX - 2.0 * SPACING);
        hi[a] = std::ceil(hi[a] + FIELD_RMAX + 2.0 * SPACING);
    }
    for (int a = 0; a < 3; ++a) n[a] = (int64_t)((hi[a] - lo[a]) / SPACING) + 1;
}

// One grid row of one atom: points xl..xh, 10 < d <= 30, += (T)(q / d^2),
// with the reference's expressions: dx = lo + (double)ix * s - c,
// d2 = dx * dx + dyz^2.  On hosts with AVX2 four points go at a time: the
// same IEEE operations lane by lane ((double)ix as an exact f64 counter),
// and a point outside the shell adds +0, which leaves its value's bits
// unchanged (a grid value is never -0: it starts at +0 and every term is
// nonzero), so both versions give the same bits.
template <typename T>
inline void field_row_scalar(T* row, int64_t xl, int64_t xh, double lo0, double s, double c0, double dyz2,
                             double qk) {
    const double r2min = CLOSE_DIST * CLOSE_DIST, r2max = FIELD_RMAX * FIELD_RMAX;
    for (int64_t ix = xl; ix <= xh; ++ix) {
        double dx = lo0 + (double)ix * s - c0;
        double d2 = dx * dx + dyz2;
        if (d2 > r2min && d2 <= r2max) row[ix] += (T)(qk / d2);
    }
}

template <typename T>
__attribute__((target("avx2"))) void field_row_avx2(T* row, int64_t xl, int64_t xh, double lo0, double s,
                                                     double c0, double dyz2, double qk) {
    const __m256d vlo = _mm256_set1_pd(lo0), vs = _mm256_set1_pd(s), vc = _mm256_set1_pd(c0);
    const __m256d vyz = _mm256_set1_pd(dyz2), vq = _mm256_set1_pd(qk), four = _mm256_set1_pd(4.0);
    const __m256d vmin = _mm256_set1_pd(CLOSE_DIST * CLOSE_DIST), vmax = _mm256_set1_pd(FIELD_RMAX * FIELD_RMAX);
    __m256d fx = _mm256_setr_pd((double)xl, (double)(xl + 1), (double)(xl + 2), (double)(xl + 3));
    int64_t ix = xl;
    for (; ix + 3 <= xh; ix += 4) {
        const __m256d dx = _mm256_sub_pd(_mm256_add_pd(vlo, _mm256_mul_pd(fx, vs)), vc);
        const __m256d d2 = _mm256_add_pd(_mm256_mul_pd(dx, dx), vyz);
        const __m256d in = _mm256_and_pd(_mm256_cmp_pd(d2, vmin, _CMP_GT_OQ), _mm256_cmp_pd(d2, vmax, _CMP_LE_OQ));
        const __m256d t = _mm256_and_pd(_mm256_div_pd(vq, d2), in);
        if constexpr (sizeof(T) == 4) {
            float* p = reinterpret_cast<float*>(row) + ix;
            _mm_storeu_ps(p, _mm_add_ps(_mm_loadu_ps(p), _mm256_cvtpd_ps(t)));
        } else {
            double* p = reinterpret_cast<double*>(row) + ix;
            _mm256_storeu_pd(p, _mm256_add_pd(_mm256_loadu_pd(p), t));
        }
        fx = _mm256_add_pd(fx, four);
    }
    field_row_scalar(row, ix, xh, lo0, s, c0, dyz2, qk);
}

const bool HAVE_AVX2 = __builtin_cpu_supports("avx2");

template <typename T>
inline void field_row(T* row, int64_t xl, int64_t xh, double lo0, double s, double c0, double dyz2, double qk) {
    if (HAVE_AVX2) field_row_avx2(row, xl, xh, lo0, s, c0, dyz2, qk);
    else field_row_scalar(row, xl, xh, lo0, s, c0, dyz2, qk);
}

// One atom's contribution to the grid points of the box [b0, b1] (inclusive
// per axis), exactly as the per-atom scatter of grid_dna.rs:71-149 visits
// them: the atom's +-spread box, the row test dyz^2 < 30^2, the row's x
// range from sqrt(30^2 - dyz^2), then 10 < d <= 30 per point, adding
// (qk / d^2) as f32 (or f64).  Restricting the scatter to a box changes
// neither the set of points an atom reaches nor the value added there.
template <typename T, bool SCALAR = false>
inline void field_atom_into(T* phi, const double lo[3], const int64_t n[3], const double* c, double qk,
                            const int64_t b0[3], const int64_t b1[3]) {
    const double s = SPACING;
    const int64_t spread = (int64_t)std::ceil(FIELD_RMAX / s) + 2;
    const double r2max = FIELD_RMAX * FIELD_RMAX;
    int64_t gi[3], gh[3];
    for (int a = 0; a < 3; ++a) {
        int64_t fl = (int64_t)std::floor((c[a] - lo[a]) / s);
        gi[a] = std::max<int64_t>(fl - spread, 0);
        gh[a] = std::min<int64_t>(fl + spread, n[a] - 1);
    }
    const int64_t zlo = std::max(gi[2], b0[2]), zhi = std::min(gh[2], b1[2]);
    const int64_t ylo = std::max(gi[1], b0[1]), yhi = std::min(gh[1], b1[1]);
    if (zlo > zhi || ylo > yhi || gi[0] > b1[0] || gh[0] < b0[0]) return;
    const double cxi_f = (c[0] - lo[0]) / s;
    const int64_t nx = n[0], ny = n[1];
    for (int64_t iz = zlo; iz <= zhi; ++iz) {
        double zz = lo[2] + (double)iz * s;
        double dz = zz - c[2];
        for (int64_t iy = ylo; iy <= yhi; ++iy) {
            double yy = lo[1] + (double)iy * s;
            double dy = yy - c[1];
            double dyz2 = dy * dy + dz * dz;
            if (dyz2 >= r2max) continue;
            double b = std::sqrt(r2max - dyz2);
            int64_t xl = std::max<int64_t>((int64_t)std::floor(cxi_f - b / s) - 1, gi[0]);
            int64_t xh = std::min<int64_t>((int64_t)std::ceil(cxi_f + b / s) + 1, gh[0]);
            if (xl > gh[0] || xh < gi[0]) continue;
            xl = std::max(std::max(xl, gi[0]), b0[0]);
            xh = std::min(std::min(xh, gh[0]), b1[0]);
            T* row = phi + (iz * ny + iy) * nx;
            if (SCALAR) field_row_scalar(row, xl, xh, lo[0], s, c[0], dyz2, qk);
            else field_row(row, xl, xh, lo[0], s, c[0], dyz2, qk);
        }
    }
}

// ReceptorField::build (grid_dna.rs:44-149).  The reference scatters atom by
// atom; every grid point therefore receives its q/d^2 terms in atom order,
// and that order fixes the f32 bits.  Here the grid is cut into bricks of
// 32^3 points (128 KB of f32, cache resident) built in parallel; each brick
// walks the atoms in index order and applies the scatter restricted to
// itself, so every point still adds its terms in atom order: the result is
// bitwise the reference's (checked against the plain scatter,
// field_build_scatter, in tests/test_oracle.py).
#ifndef BX
#define BX 128
#define BY 16
#define BZ 16
#endif
Field* field_build(const double* coords, const double* q, int64_t na, int fp64) {
    Field* f = new Field();
    f->fp64 = fp64;
    double lo[3];
    int64_t n[3];
    field_extent(coords, na, lo, n);
    size_t total = (size_t)n[0] * n[1] * n[2];
    if (fp64) f->phi64.assign(total, 0.0); else f->phi.assign(total, 0.0f);
    const double s = SPACING;
    const int64_t spread = (int64_t)std::ceil(FIELD_RMAX / s) + 2;
    // charged atoms with their grid cell, for the per-brick atom test
    std::vector<int64_t> idx;
    std::vector<int64_t> cell;
    for (int64_t k = 0; k < na; ++k) {
        if (q[k] == 0.0) continue;
        idx.push_back(k);
        for (int a = 0; a < 3; ++a) cell.push_back((int64_t)std::floor((coords[3 * k + a] - lo[a]) / s));
    }
    const int64_t B[3] = {BX, BY, BZ};
    const int64_t nb[3] = {(n[0] + B[0] - 1) / B[0], (n[1] + B[1] - 1) / B[1], (n[2] + B[2] - 1) / B[2]};
    const int64_t nbricks = nb[0] * nb[1] * nb[2];
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t br = 0; br < nbricks; ++br) {
        const int64_t bx = br % nb[0], by = (br / nb[0]) % nb[1], bz = br / (nb[0] * nb[1]);
        const int64_t b0[3] = {bx * B[0], by * B[1], bz * B[2]};
        const int64_t b1[3] = {std::min(b0[0] + B[0], n[0]) - 1, std::min(b0[1] + B[1], n[1]) - 1,
                               std::min(b0[2] + B[2], n[2]) - 1};
        for (size_t m = 0; m < idx.size(); ++m) {
            const int64_t* cl = &cell[3 * m];
            // the atom's +-spread box misses the brick: no point of it is reached
            if (cl[0] + spread < b0[0] || cl[0] - spread > b1[0] || cl[1] + spread < b0[1] ||
                cl[1] - spread > b1[1] || cl[2] + spread < b0[2] || cl[2] - spread > b1[2])
                continue;
            const int64_t k = idx[m];
            if (fp64) field_atom_into(f->phi64.data(), lo, n, coords + 3 * k, q[k], b0, b1);
            else field_atom_into(f->phi.data(), lo, n, coords + 3 * k, q[k], b0, b1);
        }
    }
    for (int a = 0; a < 3; ++a) { f->origin[a] = lo[a]; f->n[a] = n[a]; }
    f->spacing = s;
    return f;
}

// The plain per-atom scatter of grid_dna.rs:71-149 (single thread, scalar
// rows), kept as the check of field_build's brick order and AVX2 rows.
Field* field_build_scatter(const double* coords, const double* q, int64_t na, int fp64) {
    Field* f = new Field();
    f->fp64 = fp64;
    double lo[3];
    int64_t n[3];
    field_extent(coords, na, lo, n);
    size_t total = (size_t)n[0] * n[1] * n[2];
    if (fp64) f->phi64.assign(total, 0.0); else f->phi.assign(total, 0.0f);
    const int64_t b0[3] = {0, 0, 0}, b1[3] = {n[0] - 1, n[1] - 1, n[2] - 1};
    for (int64_t k = 0; k < na; ++k) {
        if (q[k] == 0.0) continue;
        if (fp64) field_atom_into<double, true>(f->phi64.data(), lo, n, coords + 3 * k, q[k], b0, b1);
        else field_atom_into<float, true>(f->phi.data(), lo, n, coords + 3 * k, q[k], b0, b1);
    }
    for (int a = 0; a < 3; ++a) { f->origin[a] = lo[a]; f->n[a] = n[a]; }
    f->spacing = SPACING;
    return f;
}

inline double field_at(const Field* f, int64_t ix, int64_t iy, int64_t iz) {
    size_t k = (size_t)((iz * f->n[1] + iy) * f->n[0] + ix);
    return f->fp64 ? f->phi64[k] : (double)f->phi[k];
}

double field_sample(const Field* f, double x, double y, double z) {  // grid_dna.rs:159-197
    double s = f->spacing;
    double fx = (x - f->origin[0]) / s, fy = (y - f->origin[1]) / s, fz = (z - f->origin[2]) / s;
    double ix = std::floor(fx), iy = std::floor(fy), iz = std::floor(fz);
    if (ix < 0.0 || iy < 0.0 || iz < 0.0) return 0.0;
    int64_t ix0 = (int64_t)ix, iy0 = (int64_t)iy, iz0 = (int64_t)iz;
    if (ix0 + 1 >= f->n[0] || iy0 + 1 >= f->n[1] || iz0 + 1 >= f->n[2]) return 0.0;
    double tx, ty, tz;
    if (f->fp64) { tx = fx - ix; ty = fy - iy; tz = fz - iz; }
    else { tx = (double)(float)(fx - ix); ty = (double)(float)(fy - iy); tz = (double)(float)(fz - iz); }
    double c000 = field_at(f, ix0, iy0, iz0), c100 = field_at(f, ix0 + 1, iy0, iz0);
    double c010 = field_at(f, ix0, iy0 + 1, iz0), c110 = field_at(f, ix0 + 1, iy0 + 1, iz0);
    double c001 = field_at(f, ix0, iy0, iz0 + 1), c101 = field_at(f, ix0 + 1, iy0, iz0 + 1);
    double c011 = field_at(f, ix0, iy0 + 1, iz0 + 1), c111 = field_at(f, ix0 + 1, iy0 + 1, iz0 + 1);
    double c00 = c000 * (1.0 - tx) + c100 * tx;
    double c10 = c010 * (1.0 - tx) + c110 * tx;
    double c01 = c001 * (1.0 - tx) + c101 * tx;
    double c11 = c011 * (1.0 - tx) + c111 * tx;
    double c0 = c00 * (1.0 - ty) + c10 * ty;
    double c1 = c01 * (1.0 - ty) + c11 * ty;
    return c0 * (1.0 - tz) + c1 * tz;
}

// ---------------------------------------------------------------------------
// Cell lists
// ---------------------------------------------------------------------------
// CudaReceptor::build (src/gpu_score.rs:75-144): used by the DNA CPU path.
struct Crec {
    int32_t nc[3];
    double lo[3];        // f32-rounded origin, widened back to f64 (dna.rs:906-909)
    double sp;
    std::vector<int32_t> cell_start, cell_atoms;
};

void crec_build(const double* coords, int64_t n, Crec& c, float origin_f[3]) {
    const double cell = CLOSE_DIST;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::fmin(lo[a], coords[3 * i + a]);
            hi[a] = std::fmax(hi[a], coords[3 * i + a]);
        }
    for (int a = 0; a < 3; ++a) lo[a] = std::floor(lo[a] - 0.01);
    for (int a = 0; a < 3; ++a) c.nc[a] = std::max<int32_t>((int32_t)std::floor((hi[a] - lo[a]) / cell) + 1, 1);
    size_t ncells = (size_t)(c.nc[0] + 1) * (c.nc[1] + 1) * (c.nc[2] + 1);
    c.cell_start.assign(ncells, 0);
    std::vector<size_t> cell_of(n);
    for (int64_t k = 0; k < n; ++k) {
        int64_t ix = std::clamp<int64_t>((int64_t)std::floor((coords[3 * k] - lo[0]) / cell), 0, c.nc[0] - 1);
        int64_t iy = std::clamp<int64_t>((int64_t)std::floor((coords[3 * k + 1] - lo[1]) / cell), 0, c.nc[1] - 1);
        int64_t iz = std::clamp<int64_t>((int64_t)std::floor((coords[3 * k + 2] - lo[2]) / cell), 0, c.nc[2] - 1);
        size_t cl = (size_t)((iz * c.nc[1] + iy) * c.nc[0] + ix);
        cell_of[k] = cl;
        c.cell_start[cl] += 1;
    }
    int32_t acc = 0;
    for (auto& v : c.cell_start) { int32_t t = v; v = acc; acc += t; }
    c.cell_start.push_back(acc);
    c.cell_atoms.assign(n, 0);
    std::vector<int32_t> cursor(c.cell_start);
    for (int64_t k = 0; k < n; ++k) c.cell_atoms[cursor[cell_of[k]]++] = (int32_t)k;
    for (int a = 0; a < 3; ++a) {
        origin_f[a] = (float)lo[a];
        c.lo[a] = (double)origin_f[a];
    }
    c.sp = (double)(float)cell;
}

// NearCells (src/nearcell.rs:22-112): used by the vdw/pydock/cpydock CPU paths.
struct NearCells {
    double cell;
    double lo[3];
    int64_t n[3];
    std::vector<int64_t> cell_start, cell_atoms;
    int64_t n_atoms;

    void build(const double* coords, int64_t na, double cell_) {
        n_atoms = na;
        if (na == 0 || cell_ <= 0.0) {
            cell = std::fmax(cell_, 1e-6);
            lo[0] = lo[1] = lo[2] = 0.0;
            n[0] = n[1] = n[2] = 1;
            cell_start.assign(2, 0);
            cell_atoms.clear();
            return;
        }
        cell = cell_;
        double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int64_t i = 0; i < na; ++i)
            for (int d = 0; d < 3; ++d) {
                double v = coords[3 * i + d];
                if (v < mn[d]) mn[d] = v;
                if (v > mx[d]) mx[d] = v;
            }
        for (int d = 0; d < 3; ++d) lo[d] = mn[d] - 1.0;
        for (int d = 0; d < 3; ++d) {
            double span = mx[d] - lo[d] + 1.0;
            n[d] = std::max<int64_t>((int64_t)std::ceil(span / cell), 1);
        }
        size_t total = (size_t)(n[0] * n[1] * n[2]);
        cell_start.assign(total + 1, 0);
        auto key = [&](const double* c) -> size_t {
            int64_t ix = std::clamp<int64_t>((int64_t)std::floor((c[0] - lo[0]) / cell), 0, n[0] - 1);
            int64_t iy = std::clamp<int64_t>((int64_t)std::floor((c[1] - lo[1]) / cell), 0, n[1] - 1);
            int64_t iz = std::clamp<int64_t>((int64_t)std::floor((c[2] - lo[2]) / cell), 0, n[2] - 1);
            return (size_t)((iz * n[1] + iy) * n[0] + ix);
        };
        for (int64_t i = 0; i < na; ++i) cell_start[key(coords + 3 * i) + 1] += 1;
        for (size_t i = 0; i < total; ++i) cell_start[i + 1] += cell_start[i];
        cell_atoms.assign(na, 0);
        std::vector<int64_t> cursor(cell_start);
        for (int64_t i = 0; i < na; ++i) cell_atoms[cursor[key(coords + 3 * i)]++] = i;
    }

    template <class F>
    void for_each_near(double x, double y, double z, F&& f) const {
        if (n_atoms == 0) return;
        int64_t cx = std::clamp<int64_t>((int64_t)std::floor((x - lo[0]) / cell), 0, n[0] - 1);
        int64_t cy = std::clamp<int64_t>((int64_t)std::floor((y - lo[1]) / cell), 0, n[1] - 1);
        int64_t cz = std::clamp<int64_t>((int64_t)std::floor((z - lo[2]) / cell), 0, n[2] - 1);
        for (int64_t dz = -1; dz <= 1; ++dz) {
            int64_t iz = cz + dz;
            if (iz < 0 || iz >= n[2]) continue;
            for (int64_t dy = -1; dy <= 1; ++dy) {
                int64_t iy = cy + dy;
                if (iy < 0 || iy >= n[1]) continue;
                for (int64_t dx = -1; dx <= 1; ++dx) {
                    int64_t ix = cx + dx;
                    if (ix < 0 || ix >= n[0]) continue;
                    size_t cl = (size_t)((iz * n[1] + iy) * n[0] + ix);
                    for (int64_t p = cell_start[cl]; p < cell_start[cl + 1]; ++p) f((size_t)cell_atoms[p]);
                }
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Scoring families
// ---------------------------------------------------------------------------
const double EPSILON = 4.0, FACTOR = 332.0;
const double ELEC_MAX_CUTOFF = 1.0 * EPSILON / FACTOR, ELEC_MIN_CUTOFF = -1.0 * EPSILON / FACTOR;
const double VDW_CUTOFF = 1.0;
const double CLOSE_DIST2 = CLOSE_DIST * CLOSE_DIST;     // == VDW_DIST_CUTOFF2
const double ELEC_DIST_CUTOFF2 = 30.0 * 30.0;
const double CLASH_PENALTY_W = 6.0, CLASH_PENALTY_FRAC = 0.75;  // dna.rs:32-33
const double SOLVATION_DISTANCE2 = 6.4 * 6.4;                   // cpydock.rs:44
const double INTERFACE_CUTOFF2 = 3.9 * 3.9;                     // constants.rs:14-15
const double MEMBRANE_PENALTY_SCORE = 999.0;                    // constants.rs:21
const double VDW_WEIGHT = 0.1;                                   // cpydock.rs:45
const double HUGE_DIST = 10000.0;                               // cpydock.rs:412

struct Mol {
    int64_t n = 0;
    std::vector<double> c, q, vdw, svdw, rad, des, asa;
    std::vector<uint8_t> heavy;
    std::vector<int32_t> hyd;
    void load(int64_t n_, const double* c_, const double* q_, const double* v_, const double* r_,
              const uint8_t* h_, const int32_t* hy_, const double* d_, const double* a_) {
        n = n_;
        c.assign(c_, c_ + 3 * n);
        q.assign(q_, q_ + n);
        vdw.assign(v_, v_ + n);
        svdw.resize(n);
        for (int64_t i = 0; i < n; ++i) svdw[i] = std::sqrt(vdw[i]);
        rad.assign(r_, r_ + n);
        heavy.assign(n, 0);
        if (h_) heavy.assign(h_, h_ + n);
        hyd.assign(n, 0);
        if (hy_) hyd.assign(hy_, hy_ + n);
        des.assign(n, 0.0);
        if (d_) des.assign(d_, d_ + n);
        asa.assign(n, 0.0);
        if (a_) asa.assign(a_, a_ + n);
    }
    // cpydock C-binary exclusion view (cpydock.rs:808-819)
    bool flag(int64_t i) const { return (i % 2 == 0) && hyd[i / 2] != 0; }
};

struct Model {
    int family;
    Mol rec, lig;
    Field* field[2] = {nullptr, nullptr};
    Crec crec;
    float crec_origin[3];
    NearCells cells;
    bool built_cells = false;
    // active restraints (restraint residue index per atom, -1 = none) and
    // receptor membrane beads; the reference keeps residue -> atoms maps
    // (pydock.rs:30-32), which count the same satisfied residues
    std::vector<int32_t> rres, lres, mem;
    int nres_r = 0, nres_l = 0;
    bool need_iface() const { return nres_r > 0 || nres_l > 0 || !mem.empty(); }

    const Field* get_field(int fp64) {
        int k = fp64 ? 1 : 0;
        if (!field[k]) field[k] = field_build(rec.c.data(), rec.q.data(), rec.n, fp64);
        return field[k];
    }
    void build_cells() {
        if (built_cells) return;
        if (family == ORC_DNA) crec_build(rec.c.data(), rec.n, crec, crec_origin);
        else cells.build(rec.c.data(), rec.n, 10.0);
        built_cells = true;
    }
    ~Model() { delete field[0]; delete field[1]; }
};

void transform_ligand(const Mol& lig, const double t[3], const double qv[4], std::vector<double>& out) {
    Quat q{qv[0], qv[1], qv[2], qv[3]};
    double m[3][3];
    q_matrix(q, m);
    out.resize(3 * lig.n);
    for (int64_t j = 0; j < lig.n; ++j) {
        double r[3];
        rot3_apply(m, &lig.c[3 * j], r);
        out[3 * j] = r[0] + t[0];
        out[3 * j + 1] = r[1] + t[1];
        out[3 * j + 2] = r[2] + t[2];
    }
}

// DNA::energy_grid CPU branch (src/dna.rs:834-998); ir / il (when not null)
// receive the interface flags of dna.rs:970-973
double dna_grid(Model& M, const std::vector<double>& L, const Field* fld, double parts[5], uint8_t* ir,
                uint8_t* il) {
    const Mol& R = M.rec; const Mol& G = M.lig; const Crec& c = M.crec;
    double e_sum = 0.0, v_sum = 0.0, npairs = 0.0;
    const double csp = c.sp, cox = c.lo[0], coy = c.lo[1], coz = c.lo[2];
    const int64_t ncx = c.nc[0], ncy = c.nc[1], ncz = c.nc[2];
    for (int64_t j = 0; j < G.n; ++j) {
        double x = L[3 * j], y = L[3 * j + 1], z = L[3 * j + 2];
        double qj = G.q[j], svdwj = G.svdw[j], vdwrj = G.rad[j];
        bool hj = G.heavy[j] != 0;
        int64_t cxi = std::clamp<int64_t>((int64_t)std::floor((x - cox) / csp), 0, ncx - 1);
        int64_t cyi = std::clamp<int64_t>((int64_t)std::floor((y - coy) / csp), 0, ncy - 1);
        int64_t czi = std::clamp<int64_t>((int64_t)std::floor((z - coz) / csp), 0, ncz - 1);
        for (int64_t dz = -1; dz <= 1; ++dz) {
            int64_t iz = czi + dz;
            if (iz < 0 || iz >= ncz) continue;
            for (int64_t dy = -1; dy <= 1; ++dy) {
                int64_t iy = cyi + dy;
                if (iy < 0 || iy >= ncy) continue;
                for (int64_t dx = -1; dx <= 1; ++dx) {
                    int64_t ix = cxi + dx;
                    if (ix < 0 || ix >= ncx) continue;
                    size_t cell = (size_t)((iz * ncy + iy) * ncx + ix);
                    for (int32_t p = c.cell_start[cell]; p < c.cell_start[cell + 1]; ++p) {
                        size_t i = (size_t)c.cell_atoms[p];
                        double ddx = x - R.c[3 * i], ddy = y - R.c[3 * i + 1], ddz = z - R.c[3 * i + 2];
                        double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        if (d2 <= CLOSE_DIST2) {
                            e_sum += clampd(qj * R.q[i] / d2, ELEC_MIN_CUTOFF, ELEC_MAX_CUTOFF);
                            double vdw_e = svdwj * R.svdw[i];
                            double vdw_r = vdwrj + R.rad[i];
                            double p6 = powi6(vdw_r) / powi3(d2);
                            double v = std::fmin(vdw_e * (p6 * p6 - 2.0 * p6), VDW_CUTOFF);
                            if (hj && R.heavy[i]) {
                                double d = std::sqrt(d2);
                                double dmin = CLASH_PENALTY_FRAC * vdw_r;
                                if (d < dmin) v += CLASH_PENALTY_W * (dmin - d);
                            }
                            v_sum += v;
                            npairs += 1.0;
                        }
                        if (ir && d2 <= INTERFACE_CUTOFF2) { ir[i] = 1; il[j] = 1; }
                    }
                }
            }
        }
    }
    double e_far = 0.0;  // ReceptorField::far_field_energy (grid_dna.rs:201-209)
    for (int64_t j = 0; j < G.n; ++j)
        if (G.q[j] != 0.0) e_far += G.q[j] * field_sample(fld, L[3 * j], L[3 * j + 1], L[3 * j + 2]);
    double total_elec = (e_sum + e_far) * FACTOR / EPSILON;
    if (parts) { parts[0] = e_sum; parts[1] = e_far; parts[2] = v_sum; parts[3] = 0.0; parts[4] = npairs; }
    return -(total_elec + v_sum);
}

// PYDOCK::energy_grid (src/pydock.rs:353-447) and VDW::energy_grid
// (src/vdw.rs:73-151); interface flags as pydock.rs:427-430, vdw.rs:139-142
double pydock_vdw_grid(Model& M, const std::vector<double>& L, const Field* fld, double parts[5], uint8_t* ir,
                       uint8_t* il) {
    const Mol& R = M.rec; const Mol& G = M.lig;
    const bool vdw_only = (M.family == ORC_VDW);
    double e_near = 0.0, total_vdw = 0.0, npairs = 0.0;
    for (int64_t j = 0; j < G.n; ++j) {
        double x = L[3 * j], y = L[3 * j + 1], z = L[3 * j + 2];
        double qj = G.q[j], svdwj = G.svdw[j], vcj = G.vdw[j], vdwrj = G.rad[j];
        M.cells.for_each_near(x, y, z, [&](size_t i) {
            double dx = x - R.c[3 * i], dy = y - R.c[3 * i + 1], dz = z - R.c[3 * i + 2];
            double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 <= CLOSE_DIST2) {
                npairs += 1.0;
                if (vdw_only) {  // vdw.rs:129-137
                    double vdw_energy = std::sqrt(R.vdw[i] * vcj);
                    double vdw_radius = R.rad[i] + vdwrj;
                    double p6 = powi6(vdw_radius) / powi3(d2);
                    double k = vdw_energy * (p6 * p6 - 2.0 * p6);
                    if (k > VDW_CUTOFF) k = VDW_CUTOFF;
                    total_vdw += k;
                } else {         // pydock.rs:415-424
                    e_near += clampd(qj * R.q[i] / d2, ELEC_MIN_CUTOFF, ELEC_MAX_CUTOFF);
                    double vdw_e = svdwj * R.svdw[i];
                    double vdw_r = vdwrj + R.rad[i];
                    double p6 = powi6(vdw_r) / powi3(d2);
                    total_vdw += std::fmin(vdw_e * (p6 * p6 - 2.0 * p6), VDW_CUTOFF);
                }
            }
            if (ir && d2 <= INTERFACE_CUTOFF2) { ir[i] = 1; il[j] = 1; }
        });
    }
    if (vdw_only) {
        if (parts) { parts[0] = 0; parts[1] = 0; parts[2] = total_vdw; parts[3] = 0; parts[4] = npairs; }
        return total_vdw * -1.0;
    }
    double e_far = 0.0;
    for (int64_t j = 0; j < G.n; ++j)
        if (G.q[j] != 0.0) e_far += G.q[j] * field_sample(fld, L[3 * j], L[3 * j + 1], L[3 * j + 2]);
    double total_elec = (e_near + e_far) * FACTOR / EPSILON;
    if (parts) { parts[0] = e_near; parts[1] = e_far; parts[2] = total_vdw; parts[3] = 0; parts[4] = npairs; }
    return -(total_elec + total_vdw);
}

// CPYDOCK::energy_grid (src/cpydock.rs:556-676); interface flags as
// cpydock.rs:639-642
double cpydock_grid(Model& M, const std::vector<double>& L, const Field* fld, double parts[5], uint8_t* ir,
                    uint8_t* il) {
    const Mol& R = M.rec; const Mol& G = M.lig;
    std::vector<double> min_rec(R.n, HUGE_DIST), min_lig(G.n, HUGE_DIST);
    double e_near = 0.0, total_vdw = 0.0, npairs = 0.0;
    for (int64_t j = 0; j < G.n; ++j) {
        double x = L[3 * j], y = L[3 * j + 1], z = L[3 * j + 2];
        double qj = G.q[j], vdwqj = G.vdw[j], vdwrj = G.rad[j];
        bool lf = G.flag(j);
        M.cells.for_each_near(x, y, z, [&](size_t i) {
            double dx = x - R.c[3 * i], dy = y - R.c[3 * i + 1], dz = z - R.c[3 * i + 2];
            double d2 = dx * dx + dy * dy + dz * dz;
            if (!R.flag((int64_t)i) && !lf) {
                if (d2 < min_rec[i]) min_rec[i] = d2;
                if (d2 < min_lig[j]) min_lig[j] = d2;
            }
            if (d2 <= CLOSE_DIST2) {
                npairs += 1.0;
                e_near += clampd(qj * R.q[i] / d2, ELEC_MIN_CUTOFF, ELEC_MAX_CUTOFF);
                double vdw_e = std::sqrt(vdwqj * R.vdw[i]);
                double vdw_r = vdwrj + R.rad[i];
                double p6 = std::pow(vdw_r, 6.0) / std::pow(d2, 3.0);
                double k = vdw_e * (p6 * p6 - 2.0 * p6);
                total_vdw += (k > VDW_CUTOFF) ? VDW_CUTOFF : k;
            }
            if (ir && d2 <= INTERFACE_CUTOFF2) { ir[i] = 1; il[j] = 1; }
        });
    }
    double e_far = 0.0;
    for (int64_t j = 0; j < G.n; ++j)
        if (G.q[j] != 0.0) e_far += G.q[j] * field_sample(fld, L[3 * j], L[3 * j + 1], L[3 * j + 2]);
    double total_elec_kcal = (e_near + e_far) * FACTOR / EPSILON;
    double total_solv = 0.0;
    for (int64_t i = 0; i < R.n; ++i) {
        double sv = 0.0;
        if (min_rec[i] <= SOLVATION_DISTANCE2 && min_rec[i] > 0.0 && R.asa[i] > 0.0)
            sv = -10.0 * std::sqrt(min_rec[i]) + 65.0;
        if (sv > R.asa[i]) sv = R.asa[i];
        total_solv += sv * R.des[i];
    }
    for (int64_t j = 0; j < G.n; ++j) {
        double sv = 0.0;
        if (min_lig[j] <= SOLVATION_DISTANCE2 && min_lig[j] > 0.0 && G.asa[j] > 0.0)
            sv = -10.0 * std::sqrt(min_lig[j]) + 65.0;
        if (sv > G.asa[j]) sv = G.asa[j];
        total_solv += sv * G.des[j];
    }
    if (parts) { parts[0] = e_near; parts[1] = e_far; parts[2] = total_vdw; parts[3] = total_solv; parts[4] = npairs; }
    return (total_elec_kcal + VDW_WEIGHT * total_vdw - total_solv) * -1.0;
}

// satisfied_restraints (scoring.rs:83-98): restraint residues with at least
// one interface atom over all residues of the map
double satisfied_restraints(const std::vector<uint8_t>& iface, const std::vector<int32_t>& res, int nres) {
    if (nres == 0) return 0.0;
    std::vector<char> sat(nres, 0);
    for (size_t i = 0; i < res.size(); ++i)
        if (res[i] >= 0 && iface[i] == 1) sat[res[i]] = 1;
    int n = 0;
    for (char c : sat) n += c;
    return (double)n / (double)nres;
}

// membrane_intersection (scoring.rs:100-108)
double membrane_intersection(const std::vector<uint8_t>& iface, const std::vector<int32_t>& mem) {
    if (mem.empty()) return 0.0;
    int64_t n = 0;
    for (int32_t i : mem) n += iface[i];
    return (double)n / (double)mem.size();
}

// iface (optional): pr, pl, membrane intersection
double energy_grid(Model& M, const double t[3], const double q[4], int fp64, double parts[5],
                   double iface[3] = nullptr) {
    std::vector<double> L;
    transform_ligand(M.lig, t, q, L);
    const Field* fld = (M.family == ORC_VDW) ? nullptr : M.get_field(fp64);
    const bool need = M.need_iface();
    std::vector<uint8_t> ir(need ? M.rec.n : 0, 0), il(need ? M.lig.n : 0, 0);
    uint8_t* pr_ = need ? ir.data() : nullptr;
    uint8_t* pl_ = need ? il.data() : nullptr;
    double score;
    switch (M.family) {
        case ORC_DNA: score = dna_grid(M, L, fld, parts, pr_, pl_); break;
        case ORC_CPYDOCK: score = cpydock_grid(M, L, fld, parts, pr_, pl_); break;
        default: score = pydock_vdw_grid(M, L, fld, parts, pr_, pl_); break;
    }
    if (iface) iface[0] = iface[1] = iface[2] = 0.0;
    if (!need) return score;
    const double perc_r = satisfied_restraints(ir, M.rres, M.nres_r);
    const double perc_l = satisfied_restraints(il, M.lres, M.nres_l);
    const double intersection = membrane_intersection(ir, M.mem);
    const double penalty = intersection > 0.0 ? MEMBRANE_PENALTY_SCORE * intersection : 0.0;
    if (iface) { iface[0] = perc_r; iface[1] = perc_l; iface[2] = intersection; }
    switch (M.family) {
        case ORC_DNA: score += perc_r * score + perc_l * score - penalty; break;   // dna.rs:989-995
        case ORC_VDW: score = score + perc_r * score + perc_l * score; break;      // vdw.rs:146-149
        default: score = score + perc_r * score + perc_l * score - penalty; break; // pydock.rs:440-445, cpydock.rs:670-675
    }
    return score;
}

// energy_exact, all pairs (dna.rs:668-819 without the Z-window sort, which
// changes only the summation order; pydock.rs:221-338; vdw.rs:153-248;
// cpydock.rs:386-552).  Receptor-major loop as in the reference.
double energy_exact(Model& M, const double t[3], const double qv[4]) {
    std::vector<double> L;
    transform_ligand(M.lig, t, qv, L);
    const Mol& R = M.rec; const Mol& G = M.lig;
    double te = 0.0, tv = 0.0;
    std::vector<double> min_rec, min_lig;
    if (M.family == ORC_CPYDOCK) { min_rec.assign(R.n, HUGE_DIST); min_lig.assign(G.n, HUGE_DIST); }
    for (int64_t i = 0; i < R.n; ++i) {
        double ei = 0.0, vi = 0.0;
        double rx = R.c[3 * i], ry = R.c[3 * i + 1], rz = R.c[3 * i + 2];
        for (int64_t j = 0; j < G.n; ++j) {
            double dx = rx - L[3 * j], dy = ry - L[3 * j + 1], dz = rz - L[3 * j + 2];
            double d2 = dx * dx + dy * dy + dz * dz;
            if (M.family == ORC_CPYDOCK && !R.flag(i) && !G.flag(j)) {
                if (d2 < min_rec[i]) min_rec[i] = d2;
                if (d2 < min_lig[j]) min_lig[j] = d2;
            }
            if (M.family != ORC_VDW && d2 <= ELEC_DIST_CUTOFF2)
                ei += clampd(R.q[i] * G.q[j] / d2, ELEC_MIN_CUTOFF, ELEC_MAX_CUTOFF);
            if (d2 <= CLOSE_DIST2) {
                if (M.family == ORC_VDW) {
                    double ve = std::sqrt(R.vdw[i] * G.vdw[j]);
                    double vr = R.rad[i] + G.rad[j];
                    double p6 = powi6(vr) / powi3(d2);
                    double k = ve * (p6 * p6 - 2.0 * p6);
                    vi += (k > VDW_CUTOFF) ? VDW_CUTOFF : k;
                } else if (M.family == ORC_CPYDOCK) {
                    double ve = std::sqrt(R.vdw[i] * G.vdw[j]);
                    double vr = R.rad[i] + G.rad[j];
                    double p6 = std::pow(vr, 6.0) / std::pow(d2, 3.0);
                    double k = ve * (p6 * p6 - 2.0 * p6);
                    vi += (k > VDW_CUTOFF) ? VDW_CUTOFF : k;
                } else {
                    double ve = R.svdw[i] * G.svdw[j];
                    double vr = R.rad[i] + G.rad[j];
                    double p6 = powi6(vr) / powi3(d2);
                    double v = std::fmin(ve * (p6 * p6 - 2.0 * p6), VDW_CUTOFF);
                    if (M.family == ORC_DNA && R.heavy[i] && G.heavy[j]) {
                        double d = std::sqrt(d2);
                        double dmin = CLASH_PENALTY_FRAC * vr;
                        if (d < dmin) v += CLASH_PENALTY_W * (dmin - d);
                    }
                    vi += v;
                }
            }
        }
        te += ei;
        tv += vi;
    }
    if (M.family == ORC_VDW) return tv * -1.0;
    double total_elec = te * FACTOR / EPSILON;
    if (M.family != ORC_CPYDOCK) return -(total_elec + tv);
    double solv = 0.0;
    for (int64_t i = 0; i < R.n; ++i) {
        double sv = 0.0;
        if (min_rec[i] <= SOLVATION_DISTANCE2 && min_rec[i] > 0.0 && R.asa[i] > 0.0)
            sv = -10.0 * std::sqrt(min_rec[i]) + 65.0;
        if (sv > R.asa[i]) sv = R.asa[i];
        solv += sv * R.des[i];
    }
    for (int64_t j = 0; j < G.n; ++j) {
        double sv = 0.0;
        if (min_lig[j] <= SOLVATION_DISTANCE2 && min_lig[j] > 0.0 && G.asa[j] > 0.0)
            sv = -10.0 * std::sqrt(min_lig[j]) + 65.0;
        if (sv > G.asa[j]) sv = G.asa[j];
        solv += sv * G.des[j];
    }
    return (total_elec + VDW_WEIGHT * tv - solv) * -1.0;
}

// ---------------------------------------------------------------------------
// GSO (src/lib.rs:47-78, src/swarm.rs:70-230, src/glowworm.rs)
// ---------------------------------------------------------------------------
struct Glow {
    uint32_t id;
    double t[3];
    Quat r;
    double rho = 0.5, gamma = 0.4, beta = 0.08, luciferin = 5.0;   // glowworm.rs:45-51
    double vision = 0.2, max_vision = 5.0;
    int max_neighbors = 5;
    std::vector<uint32_t> nb;
    std::vector<double> prob;
    double scoring = 0.0;
    bool moved = false;
    uint32_t step = 0;
};

struct Gso {
    Model* model;
    std::vector<Glow> g;
    Rng rng;
    int fp64, threads;
    int64_t scored = 0;
};

void gso_update_luciferin(Gso& S) {  // swarm.rs:70-103 / glowworm.rs:61-72
    std::vector<int64_t> need;
    for (size_t i = 0; i < S.g.size(); ++i)
        if (S.g[i].moved || S.g[i].step == 0) need.push_back((int64_t)i);
    int64_t nn = (int64_t)need.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(S.threads)
    for (int64_t k = 0; k < nn; ++k) {
        Glow& gw = S.g[need[k]];
        double q[4] = {gw.r.w, gw.r.x, gw.r.y, gw.r.z};
        gw.scoring = energy_grid(*S.model, gw.t, q, S.fp64, nullptr);
    }
    S.scored += nn;
    for (auto& gw : S.g) {
        gw.luciferin = (1.0 - gw.rho) * gw.luciferin + gw.gamma * gw.scoring;
        gw.step += 1;
    }
}

void gso_movement(Gso& S) {  // swarm.rs:105-174
    size_t n = S.g.size();
    if (n == 0) return;
    std::vector<double> pos(3 * n);
    std::vector<Quat> rot(n);
    for (size_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) pos[3 * i + a] = S.g[i].t[a];
        rot[i] = S.g[i].r;
    }
    // neighbour lists: id-ordered scan (the spatial hash of swarm.rs:181-230
    // returns the same id-sorted lists)
    std::vector<double> luc(n);
    for (size_t i = 0; i < n; ++i) luc[i] = S.g[i].luciferin;
    for (size_t i = 0; i < n; ++i) {
        Glow& g1 = S.g[i];
        double vr2 = g1.vision * g1.vision;
        g1.nb.clear();
        for (size_t k = 0; k < n; ++k) {
            const Glow& g2 = S.g[k];
            if (g2.id == g1.id || !(g1.luciferin < g2.luciferin)) continue;
            double dx = g1.t[0] - g2.t[0], dy = g1.t[1] - g2.t[1], dz = g1.t[2] - g2.t[2];
            if (dx * dx + dy * dy + dz * dz < vr2) g1.nb.push_back(g2.id);
        }
        // compute_probability_moving_toward_neighbor (glowworm.rs:114-128)
        g1.prob.clear();
        double total = 0.0;
        for (uint32_t nid : g1.nb) {
            double diff = luc[nid] - g1.luciferin;
            g1.prob.push_back(diff);
            total += diff;
        }
        for (auto& p : g1.prob) p /= total;
    }
    std::vector<double> randoms(n);
    for (size_t i = 0; i < n; ++i) randoms[i] = rng_f64(S.rng);
    for (size_t i = 0; i < n; ++i) {
        Glow& gw = S.g[i];
        // select_random_neighbor (glowworm.rs:130-142)
        uint32_t nid = gw.id;
        if (!gw.nb.empty()) {
            double sum = 0.0;
            size_t k = 0;
            while (sum < randoms[i] && k < gw.prob.size()) { sum += gw.prob[k]; ++k; }
            nid = gw.nb[k == 0 ? 0 : k - 1];
        }
        // move_towards (glowworm.rs:144-182), DEFAULT_*_STEP = 0.5
        gw.moved = gw.id != nid;
        if (gw.moved) {
            double dx = pos[3 * nid] - gw.t[0], dy = pos[3 * nid + 1] - gw.t[1], dz = pos[3 * nid + 2] - gw.t[2];
            double norm = std::sqrt(dx * dx + dy * dy + dz * dz);
            double coef = 0.5 / norm;
            gw.t[0] += dx * coef;
            gw.t[1] += dy * coef;
            gw.t[2] += dz * coef;
            gw.r = q_slerp(gw.r, rot[nid], 0.5);
            q_normalize(gw.r);
        }
        // update_vision_range (glowworm.rs:107-112)
        double v = gw.vision + gw.beta * (double)(gw.max_neighbors - (int)gw.nb.size());
        gw.vision = std::fmin(gw.max_vision, std::fmax(0.0, v));
    }
}

// ---------------------------------------------------------------------------
// Synthetic receptor chain for the CPU reference arm of the benchmark, so
// that its inputs are made without the product library.  Same algorithm and
// std::mt19937_64 stream as liblkg's lkg_synth_chain (a seeded
// self-avoiding walk, not reference code): bond vectors uniform on the
// sphere, rejected outside radius R or within min_sep of an atom more than
// two bonds back; every 200 consecutive rejections the end is either given
// 0.5 A more radius (stuck at the boundary with no new length for
// `patience` attempts) or backed off by 1, 2, 4, ... atoms.  Checked bit
// for bit against the library's generator in tests/test_host.py.
// ---------------------------------------------------------------------------
struct ChainGrid {
    double cs;
    std::unordered_map<int64_t, std::vector<int>> cells;
    static int64_t pack(int64_t ix, int64_t iy, int64_t iz) {
        return ((ix + (1 << 20)) << 42) | ((iy + (1 << 20)) << 21) | (iz + (1 << 20));
    }
    int64_t cell_of(double x, double y, double z) const {
        return pack((int64_t)std::floor(x / cs), (int64_t)std::floor(y / cs), (int64_t)std::floor(z / cs));
    }
};

int synth_chain(uint64_t seed, int32_t n, double r0, double bond, double min_sep, int32_t patience,
                double* coords, double* r_final) {
    if (n <= 0 || !coords || r0 <= 0 || bond <= 0 || min_sep < 0 || patience <= 0) return -1;
    std::mt19937_64 gen(seed);
    auto unit = [&]() { return (double)(gen() >> 11) * (1.0 / 9007199254740992.0); };
    const double two_pi = 2.0 * M_PI;
    double R = r0;
    ChainGrid G{std::max(min_sep, 1.0), {}};
    std::vector<double> c{0.0, 0.0, 0.0};
    c.reserve(3 * (size_t)n);
    G.cells[G.cell_of(0, 0, 0)].push_back(0);
    int fails = 0, longest = 1, back = 1;
    long long tries = 0, since_longest = 0;
    const long long max_tries = 4000LL * n + 100000000LL;
    const double sep2 = min_sep * min_sep;
    while ((int)(c.size() / 3) < n) {
        const int k = (int)(c.size() / 3);
        const double u = 2.0 * unit() - 1.0;
        const double phi = two_pi * unit();
        const double sn = std::sqrt(std::max(0.0, 1.0 - u * u));
        const double* e = &c[3 * (k - 1)];
        const double x = e[0] + bond * sn * std::cos(phi), y = e[1] + bond * sn * std::sin(phi), z = e[2] + bond * u;
        bool ok = x * x + y * y + z * z <= R * R;
        if (ok) {
            const int64_t bx = (int64_t)std::floor(x / G.cs), by = (int64_t)std::floor(y / G.cs),
                          bz = (int64_t)std::floor(z / G.cs);
            for (int64_t dz = -1; dz <= 1 && ok; ++dz)
                for (int64_t dy = -1; dy <= 1 && ok; ++dy)
                    for (int64_t dx = -1; dx <= 1 && ok; ++dx) {
                        auto it = G.cells.find(ChainGrid::pack(bx + dx, by + dy, bz + dz));
                        if (it == G.cells.end()) continue;
                        for (int a : it->second) {
                            if (a >= k - 2) continue;
                            const double ex = x - c[3 * a], ey = y - c[3 * a + 1], ez = z - c[3 * a + 2];
                            if (ex * ex + ey * ey + ez * ez < sep2) { ok = false; break; }
                        }
                    }
        }
        if (ok) {
            c.insert(c.end(), {x, y, z});
            G.cells[G.cell_of(x, y, z)].push_back(k);
            fails = 0;
            if (k + 1 > longest) { longest = k + 1; since_longest = 0; back = 1; }
            continue;
        }
        if (++tries > max_tries) return -1;
        if (++fails % 200 == 0 && k > 1) {
            const double* t = &c[3 * (k - 1)];
            const double rt = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
            if (rt > R - 2.0 * min_sep && since_longest >= patience) {
                R += 0.5;
                since_longest = 0;
            } else {
                const int m = std::min(back, k - 1);
                for (int i = 0; i < m; ++i) {
                    const int last = (int)(c.size() / 3) - 1;
                    auto& v = G.cells[G.cell_of(c[3 * last], c[3 * last + 1], c[3 * last + 2])];
                    v.erase(std::remove(v.begin(), v.end(), last), v.end());
                    c.resize(c.size() - 3);
                }
                back = std::min(back * 2, 256);
            }
            fails = 0;
        }
        ++since_longest;
    }
    std::copy(c.begin(), c.end(), coords);
    if (r_final) *r_final = R;
    return 0;
}

// ---------------------------------------------------------------------------
// Lee & Richards solvent-accessible surface area (src/lr_sasa.rs:27-291, the
// freesasa 2.2 algorithm with probe 1.4 A and 20 slices), restated here
// independently of liblkg's copy so that the cpydock reference areas are
// checked against the reference's own algorithm.
// ---------------------------------------------------------------------------
struct LrNb {
    std::vector<std::vector<int>> idx;       // neighbours of each atom, in discovery order
    std::vector<std::vector<double>> dxy;    // sqrt(dx^2 + dy^2)
    std::vector<std::vector<double>> dx, dy; // neighbour minus atom
};

// lr_sasa.rs:27-145: cells of edge 2 max(R), atoms in index order per cell,
// each cell paired with the neighbouring cells whose offset sums to >= 0
// (and itself, from the next atom on), pairs kept when d^2 < (Ri + Rj)^2
LrNb lr_neighbours(const double* c, const std::vector<double>& R) {
    const int n = (int)R.size();
    LrNb nb;
    nb.idx.resize(n); nb.dxy.resize(n); nb.dx.resize(n); nb.dy.resize(n);
    double rmax = 0.0;
    for (double r : R) rmax = std::fmax(rmax, r);
    const double d = 2.0 * rmax;
    double lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[0], c[1], c[2]};
    for (int i = 1; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::fmin(lo[a], c[3 * i + a]);
            hi[a] = std::fmax(hi[a], c[3 * i + a]);
        }
    int64_t nc[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] -= d / 2.0;
        hi[a] += d / 2.0;
        nc[a] = (int64_t)std::ceil((hi[a] - lo[a]) / d);
    }
    auto cell_index = [&](int64_t ix, int64_t iy, int64_t iz) { return ix + nc[0] * (iy + nc[1] * iz); };
    std::vector<std::vector<int>> cell(nc[0] * nc[1] * nc[2]);
    for (int i = 0; i < n; ++i) {
        int64_t g[3];
        for (int a = 0; a < 3; ++a)
            g[a] = std::min<int64_t>(std::max<int64_t>((int64_t)((c[3 * i + a] - lo[a]) / d), 0), nc[a] - 1);
        cell[cell_index(g[0], g[1], g[2])].push_back(i);
    }
    for (int64_t iz = 0; iz < nc[2]; ++iz)
        for (int64_t iy = 0; iy < nc[1]; ++iy)
            for (int64_t ix = 0; ix < nc[0]; ++ix) {
                const std::vector<int>& A = cell[cell_index(ix, iy, iz)];
                // neighbour cells in x-outer, z-inner order, as lr_sasa.rs:84-102 lists them
                for (int64_t jx = std::max<int64_t>(ix - 1, 0); jx <= std::min(ix + 1, nc[0] - 1); ++jx)
                    for (int64_t jy = std::max<int64_t>(iy - 1, 0); jy <= std::min(iy + 1, nc[1] - 1); ++jy)
                        for (int64_t jz = std::max<int64_t>(iz - 1, 0); jz <= std::min(iz + 1, nc[2] - 1); ++jz) {
                            if ((jx - ix) + (jy - iy) + (jz - iz) < 0) continue;
                            const bool same = jx == ix && jy == iy && jz == iz;
                            const std::vector<int>& B = cell[cell_index(jx, jy, jz)];
                            for (size_t ii = 0; ii < A.size(); ++ii) {
                                const int a = A[ii];
                                for (size_t jj = same ? ii + 1 : 0; jj < B.size(); ++jj) {
                                    const int b = B[jj];
                                    const double cut2 = (R[a] + R[b]) * (R[a] + R[b]);
                                    const double ex = c[3 * b] - c[3 * a], ey = c[3 * b + 1] - c[3 * a + 1],
                                                 ez = c[3 * b + 2] - c[3 * a + 2];
                                    if (ex * ex + ey * ey + ez * ez < cut2) {
                                        const double exy = std::sqrt(ex * ex + ey * ey);
                                        nb.idx[a].push_back(b); nb.idx[b].push_back(a);
                                        nb.dxy[a].push_back(exy); nb.dxy[b].push_back(exy);
                                        nb.dx[a].push_back(ex); nb.dx[b].push_back(-ex);
                                        nb.dy[a].push_back(ey); nb.dy[b].push_back(-ey);
                                    }
                                }
                            }
                        }
            }
    return nb;
}

// exposed length of the full circle given m buried intervals (start, end)
// in arc[0 .. 2m): intervals sorted by start (insertion sort), then the gaps
// between the running union's end and the next start are summed
// (lr_sasa.rs:150-185)
double lr_exposed(std::vector<double>& arc, int m) {
    const double two_pi = 2.0 * M_PI;
    if (m == 0) return two_pi;
    for (int i = 2; i < 2 * m; i += 2) {
        const double s0 = arc[i], s1 = arc[i + 1];
        int j = i;
        for (; j > 0 && arc[j - 2] > s0; j -= 2) {
            arc[j] = arc[j - 2];
            arc[j + 1] = arc[j - 1];
        }
        arc[j] = s0;
        arc[j + 1] = s1;
    }
    double total = arc[0], end = arc[1];
    for (int i = 2; i < 2 * m; i += 2) {
        if (end < arc[i]) total += arc[i] - end;
        if (arc[i + 1] > end) end = arc[i + 1];
    }
    return total + two_pi - end;
}

// area of atom i: n_slices planes across its sphere, each plane's exposed
// arc of the atom's circle times delta * R_i (lr_sasa.rs:187-268)
double lr_area(int i, const double* c, const std::vector<double>& R, const LrNb& nb, int n_slices) {
    const double two_pi = 2.0 * M_PI;
    const std::vector<int>& J = nb.idx[i];
    const int m = (int)J.size();
    const double zi = c[3 * i + 2], ri = R[i];
    const double delta = 2.0 * ri / n_slices;
    double z = zi - ri - 0.5 * delta, area = 0.0;
    std::vector<double> arc(4 * std::max(m, 1));
    for (int s = 0; s < n_slices; ++s) {
        z += delta;
        const double di = std::fabs(zi - z);
        const double ri_p2 = ri * ri - di * di;
        if (ri_p2 < 0.0) continue;
        const double ri_p = std::sqrt(ri_p2);
        if (ri_p <= 0.0) continue;
        int arcs = 0;
        bool buried = false;
        for (int k = 0; k < m; ++k) {
            const double dj = std::fabs(c[3 * J[k] + 2] - z);
            const double rj = R[J[k]];
            if (!(dj < rj)) continue;
            const double rj_p2 = rj * rj - dj * dj;
            const double rj_p = std::sqrt(rj_p2);
            const double dij = nb.dxy[i][k];
            if (dij >= ri_p + rj_p) continue;                // circles apart
            if (dij + ri_p < rj_p) { buried = true; break; }  // circle i inside circle j
            if (dij + rj_p < ri_p) continue;                  // circle j inside circle i
            const double alpha = std::acos((ri_p2 + dij * dij - rj_p2) / (2.0 * ri_p * dij));
            const double beta = std::atan2(nb.dy[i][k], nb.dx[i][k]) + M_PI;
            double a0 = beta - alpha, a1 = beta + alpha;
            if (a0 < 0.0) a0 += two_pi;
            if (a1 > 2.0 * M_PI) a1 -= two_pi;
            if (a1 < a0) {   // the interval wraps through 0: two pieces
                arc[2 * arcs] = 0.0; arc[2 * arcs + 1] = a1;
                arc[2 * arcs + 2] = a0; arc[2 * arcs + 3] = two_pi;
                arcs += 2;
            } else {
                arc[2 * arcs] = a0; arc[2 * arcs + 1] = a1;
                arcs += 1;
            }
        }
        if (!buried) area += delta * ri * lr_exposed(arc, arcs);
    }
    return area;
}

}  // namespace


// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void orc_lr_sasa(const double* coords, const double* radii, int32_t n, double* out) {
    if (n <= 0) return;
    std::vector<double> R(n);
    for (int i = 0; i < n; ++i) R[i] = radii[i] + 1.4;   // probe radius
    const LrNb nb = lr_neighbours(coords, R);
    for (int i = 0; i < n; ++i) out[i] = lr_area(i, coords, R, nb, 20);
}

int orc_synth_chain(uint64_t seed, int32_t n, double r0, double bond, double min_sep, int32_t patience,
                    double* coords, double* r_final) {
    return synth_chain(seed, n, r0, bond, min_sep, patience, coords, r_final);
}

void* orc_rng_new(uint64_t seed) { Rng* r = new Rng(); rng_seed(*r, seed); return r; }
void orc_rng_free(void* r) { delete (Rng*)r; }
double orc_rng_f64(void* r) { return rng_f64(*(Rng*)r); }
uint64_t orc_rng_u64(void* r) { return rng_u64(*(Rng*)r); }

void orc_quat_random(void* rng, double out[4]) {  // qt.rs:106-117
    Rng& r = *(Rng*)rng;
    double u1 = rng_f64(r), u2 = rng_f64(r), u3 = rng_f64(r);
    const double PI = 3.14159265358979323846;
    out[0] = std::sqrt(1.0 - u1) * std::sin(2.0 * PI * u2);
    out[1] = std::sqrt(1.0 - u1) * std::cos(2.0 * PI * u2);
    out[2] = std::sqrt(u1) * std::sin(2.0 * PI * u3);
    out[3] = std::sqrt(u1) * std::cos(2.0 * PI * u3);
}

void orc_quat_slerp(const double a[4], const double b[4], double t, double out[4]) {
    Quat r = q_slerp(Quat{a[0], a[1], a[2], a[3]}, Quat{b[0], b[1], b[2], b[3]}, t);
    out[0] = r.w; out[1] = r.x; out[2] = r.y; out[3] = r.z;
}

void orc_quat_normalize(double q[4]) {
    Quat r{q[0], q[1], q[2], q[3]};
    q_normalize(r);
    q[0] = r.w; q[1] = r.x; q[2] = r.y; q[3] = r.z;
}

void* orc_field_new(const double* coords, const double* q, int64_t n, int fp64) {
    return field_build(coords, q, n, fp64);
}
void* orc_field_new_scatter(const double* coords, const double* q, int64_t n, int fp64) {
    return field_build_scatter(coords, q, n, fp64);
}
void orc_field_info(const void* fv, double origin[3], int64_t dims[3], double* spacing) {
    const Field* f = (const Field*)fv;
    for (int a = 0; a < 3; ++a) { origin[a] = f->origin[a]; dims[a] = f->n[a]; }
    *spacing = f->spacing;
}
const float* orc_field_phi32(const void* f) { return ((const Field*)f)->phi.data(); }
const double* orc_field_phi64(const void* f) { return ((const Field*)f)->phi64.data(); }
double orc_field_sample(const void* f, double x, double y, double z) { return field_sample((const Field*)f, x, y, z); }
void orc_field_free(void* f) { delete (Field*)f; }

int64_t orc_crec_build(const double* coords, int64_t n, int32_t nc[3], float origin[3],
                       float* cell_sp, int32_t* cell_start, int32_t* cell_atoms) {
    Crec c;
    crec_build(coords, n, c, origin);
    for (int a = 0; a < 3; ++a) nc[a] = c.nc[a];
    *cell_sp = (float)c.sp;
    if (cell_start) memcpy(cell_start, c.cell_start.data(), c.cell_start.size() * sizeof(int32_t));
    if (cell_atoms) memcpy(cell_atoms, c.cell_atoms.data(), c.cell_atoms.size() * sizeof(int32_t));
    return (int64_t)c.cell_start.size();
}

int64_t orc_nearcell_pair_count(const double* coords, int64_t n, double cell) {
    NearCells nc;
    nc.build(coords, n, cell);
    std::vector<std::pair<int64_t, int64_t>> near;
    double cut2 = cell * cell;
    for (int64_t j = 0; j < n; ++j) {
        const double* c = coords + 3 * j;
        nc.for_each_near(c[0], c[1], c[2], [&](size_t i) {
            double dx = c[0] - coords[3 * i], dy = c[1] - coords[3 * i + 1], dz = c[2] - coords[3 * i + 2];
            if ((int64_t)i != j && dx * dx + dy * dy + dz * dz <= cut2)
                near.emplace_back(std::min<int64_t>(i, j), std::max<int64_t>(i, j));
        });
    }
    std::sort(near.begin(), near.end());
    near.erase(std::unique(near.begin(), near.end()), near.end());
    return (int64_t)near.size();
}

int64_t orc_allpairs_count(const double* coords, int64_t n, double cut) {
    int64_t cnt = 0;
    double cut2 = cut * cut;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = i + 1; j < n; ++j) {
            double dx = coords[3 * i] - coords[3 * j], dy = coords[3 * i + 1] - coords[3 * j + 1],
                   dz = coords[3 * i + 2] - coords[3 * j + 2];
            if (dx * dx + dy * dy + dz * dz <= cut2) ++cnt;
        }
    return cnt;
}

void* orc_model_new(int family,
                    int64_t nr, const double* rc, const double* rq, const double* rvdw,
                    const double* rrad, const uint8_t* rheavy, const int32_t* rhyd,
                    const double* rdes, const double* rasa,
                    int64_t nl, const double* lc, const double* lq, const double* lvdw,
                    const double* lrad, const uint8_t* lheavy, const int32_t* lhyd,
                    const double* ldes, const double* lasa) {
    Model* m = new Model();
    m->family = family;
    m->rec.load(nr, rc, rq, rvdw, rrad, rheavy, rhyd, rdes, rasa);
    m->lig.load(nl, lc, lq, lvdw, lrad, lheavy, lhyd, ldes, lasa);
    m->build_cells();
    return m;
}

void orc_model_free(void* m) { delete (Model*)m; }

const void* orc_model_field(void* m, int fp64) { return ((Model*)m)->get_field(fp64); }

double orc_energy_grid(void* m, const double t[3], const double q[4], int fp64, double parts[5]) {
    return energy_grid(*(Model*)m, t, q, fp64, parts);
}

double orc_energy_exact(void* m, const double t[3], const double q[4]) {
    return energy_exact(*(Model*)m, t, q);
}

void orc_model_set_restraints(void* mv, const int32_t* rres, int nres_r, const int32_t* lres, int nres_l,
                              const int32_t* mem, int64_t nmem) {
    Model& M = *(Model*)mv;
    M.nres_r = nres_r;
    M.nres_l = nres_l;
    M.rres.assign(M.rec.n, -1);
    M.lres.assign(M.lig.n, -1);
    if (nres_r && rres) M.rres.assign(rres, rres + M.rec.n);
    if (nres_l && lres) M.lres.assign(lres, lres + M.lig.n);
    M.mem.assign(mem ? mem : nullptr, mem ? mem + nmem : nullptr);
}

void orc_batch_energy_grid_iface(void* mv, int64_t N, const double* poses, int fp64, int threads,
                                 double* out, double* iface) {
    Model& M = *(Model*)mv;
    if (M.family != ORC_VDW) M.get_field(fp64);
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#else
    int nt = 1; (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t k = 0; k < N; ++k) {
        const double* p = poses + 7 * k;
        double q[4] = {p[0], p[1], p[2], p[3]};
        double t[3] = {p[4], p[5], p[6]};
        out[k] = energy_grid(M, t, q, fp64, nullptr, iface ? iface + 3 * k : nullptr);
    }
}

void orc_batch_energy_grid(void* mv, int64_t N, const double* poses, int fp64, int threads,
                           double* out, double* parts) {
    Model& M = *(Model*)mv;
    if (M.family != ORC_VDW) M.get_field(fp64);
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#else
    int nt = 1; (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t k = 0; k < N; ++k) {
        const double* p = poses + 7 * k;
        double q[4] = {p[0], p[1], p[2], p[3]};
        double t[3] = {p[4], p[5], p[6]};
        out[k] = energy_grid(M, t, q, fp64, parts ? parts + 5 * k : nullptr);
    }
}

void* orc_gso_new(void* model, int64_t n, const double* positions, uint64_t seed, int fp64, int threads) {
    Gso* S = new Gso();
    S->model = (Model*)model;
    S->fp64 = fp64;
#ifdef _OPENMP
    S->threads = threads > 0 ? threads : omp_get_max_threads();
#else
    S->threads = 1; (void)threads;
#endif
    rng_seed(S->rng, seed);
    if (S->model->family != ORC_VDW) S->model->get_field(fp64);
    S->g.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        Glow& g = S->g[i];
        const double* p = positions + 7 * i;
        g.id = (uint32_t)i;
        g.t[0] = p[0]; g.t[1] = p[1]; g.t[2] = p[2];
        g.r = Quat{p[3], p[4], p[5], p[6]};
    }
    return S;
}

void orc_gso_run(void* gv, int steps) {  // lib.rs:66-78 (file output omitted)
    Gso& S = *(Gso*)gv;
    for (int s = 1; s <= steps; ++s) {
        gso_update_luciferin(S);
        gso_movement(S);
    }
}

void orc_gso_state(const void* gv, double* trans, double* rot, double* luc, double* scoring,
                   double* vision, int32_t* nneigh, uint8_t* moved) {
    const Gso& S = *(const Gso*)gv;
    for (size_t i = 0; i < S.g.size(); ++i) {
        const Glow& g = S.g[i];
        if (trans) for (int a = 0; a < 3; ++a) trans[3 * i + a] = g.t[a];
        if (rot) { rot[4 * i] = g.r.w; rot[4 * i + 1] = g.r.x; rot[4 * i + 2] = g.r.y; rot[4 * i + 3] = g.r.z; }
        if (luc) luc[i] = g.luciferin;
        if (scoring) scoring[i] = g.scoring;
        if (vision) vision[i] = g.vision;
        if (nneigh) nneigh[i] = (int32_t)g.nb.size();
        if (moved) moved[i] = g.moved ? 1 : 0;
    }
}

int64_t orc_gso_scored(const void* g) { return ((const Gso*)g)->scored; }
void orc_gso_free(void* g) { delete (Gso*)g; }

}  // extern "C"
