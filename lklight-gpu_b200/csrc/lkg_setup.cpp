// Setup-time host helpers: Lee & Richards SASA (cpydock reference areas) and
// the self-avoiding random chain used to synthesise benchmark receptors.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <unordered_map>
#include <vector>

#include "lkg_runtime.h"

using namespace lkg;

namespace {

// ---------------------------------------------------------------------------
// Lee & Richards SASA (lr_sasa.rs, a port of freesasa 2.2 nb.c + sasa_lr.c):
// probe 1.4 A, 20 slices; cell-list neighbours, per-slice exposed arcs.
// ---------------------------------------------------------------------------
const double TWOPI = 2.0 * M_PI;

struct Nb {
    std::vector<std::vector<int>> nb;
    std::vector<std::vector<double>> xyd, xd, yd;
};

Nb neighbours(const double* c, const std::vector<double>& r, int n) {  // lr_sasa.rs:27-145
    Nb o;
    o.nb.resize(n); o.xyd.resize(n); o.xd.resize(n); o.yd.resize(n);
    double rmax = 0.0;
    for (double v : r) rmax = std::max(rmax, v);
    const double d = 2.0 * rmax;
    double mn[3] = {c[0], c[1], c[2]}, mx[3] = {c[0], c[1], c[2]};
    for (int i = 1; i < n; ++i)
        for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], c[3 * i + a]); mx[a] = std::max(mx[a], c[3 * i + a]); }
    for (int a = 0; a < 3; ++a) { mn[a] -= d / 2.0; mx[a] += d / 2.0; }
    int nc[3];
    for (int a = 0; a < 3; ++a) nc[a] = std::max(1, (int)std::ceil((mx[a] - mn[a]) / d));
    const int ncell = nc[0] * nc[1] * nc[2];
    std::vector<std::vector<int>> cell(ncell);
    auto cell_of = [&](const double* p) {
        int ix = std::min(std::max((int)((p[0] - mn[0]) / d), 0), nc[0] - 1);
        int iy = std::min(std::max((int)((p[1] - mn[1]) / d), 0), nc[1] - 1);
        int iz = std::min(std::max((int)((p[2] - mn[2]) / d), 0), nc[2] - 1);
        return ix + nc[0] * (iy + nc[1] * iz);
    };
    for (int i = 0; i < n; ++i) cell[cell_of(c + 3 * i)].push_back(i);
    for (int icx = 0; icx < nc[0]; ++icx)
        for (int icy = 0; icy < nc[1]; ++icy)
            for (int icz = 0; icz < nc[2]; ++icz) {
                int ic = icx + nc[0] * (icy + nc[1] * icz);
                int x0 = icx > 0 ? icx - 1 : 0, x1 = icx < nc[0] - 1 ? icx + 1 : icx;
                int y0 = icy > 0 ? icy - 1 : 0, y1 = icy < nc[1] - 1 ? icy + 1 : icy;
                int z0 = icz > 0 ? icz - 1 : 0, z1 = icz < nc[2] - 1 ? icz + 1 : icz;
                for (int i = x0; i <= x1; ++i)
                    for (int j = y0; j <= y1; ++j)
                        for (int k = z0; k <= z1; ++k) {
                            if ((i - icx) + (j - icy) + (k - icz) < 0) continue;
                            int jc = i + nc[0] * (j + nc[1] * k);
                            const auto& ai = cell[ic];
                            const auto& aj = cell[jc];
                            for (size_t ii = 0; ii < ai.size(); ++ii) {
                                int ia = ai[ii];
                                size_t start = (ic == jc) ? ii + 1 : 0;
                                for (size_t jj = start; jj < aj.size(); ++jj) {
                                    int ja = aj[jj];
                                    double cut2 = (r[ia] + r[ja]) * (r[ia] + r[ja]);
                                    double dx = c[3 * ja] - c[3 * ia], dy = c[3 * ja + 1] - c[3 * ia + 1],
                                           dz = c[3 * ja + 2] - c[3 * ia + 2];
                                    if (dx * dx + dy * dy + dz * dz < cut2) {
                                        double dxy = std::sqrt(dx * dx + dy * dy);
                                        o.nb[ia].push_back(ja); o.nb[ja].push_back(ia);
                                        o.xyd[ia].push_back(dxy); o.xyd[ja].push_back(dxy);
                                        o.xd[ia].push_back(dx); o.xd[ja].push_back(-dx);
                                        o.yd[ia].push_back(dy); o.yd[ja].push_back(-dy);
                                    }
                                }
                            }
                        }
            }
    return o;
}

double exposed_arc(std::vector<double>& arc, int n) {  // lr_sasa.rs:150-186
    if (n == 0) return TWOPI;
    for (int i = 2; i < 2 * n; i += 2) {
        double t0 = arc[i], t1 = arc[i + 1];
        int j = i;
        while (j > 0 && arc[j - 2] > t0) { arc[j] = arc[j - 2]; arc[j + 1] = arc[j - 1]; j -= 2; }
        arc[j] = t0; arc[j + 1] = t1;
    }
    double sum = arc[0], sup = arc[1];
    for (int i2 = 2; i2 < 2 * n; i2 += 2) {
        if (sup < arc[i2]) sum += arc[i2] - sup;
        if (arc[i2 + 1] > sup) sup = arc[i2 + 1];
    }
    return sum + TWOPI - sup;
}

double atom_area(int i, const double* c, const std::vector<double>& r, const Nb& nb, int nslices) {  // :190-269
    const int nn = (int)nb.nb[i].size();
    const double zi = c[3 * i + 2], ri = r[i];
    const double delta = 2.0 * ri / nslices;
    double z = zi - ri - 0.5 * delta, sasa = 0.0;
    std::vector<double> arc(4 * std::max(nn, 1));
    for (int s = 0; s < nslices; ++s) {
        z += delta;
        double di = std::fabs(zi - z);
        double ri_p2 = ri * ri - di * di;
        if (ri_p2 < 0.0) continue;
        double ri_p = std::sqrt(ri_p2);
        if (ri_p <= 0.0) continue;
        int narc = 0;
        bool buried = false;
        for (int j = 0; j < nn; ++j) {
            int nbj = nb.nb[i][j];
            double zj = c[3 * nbj + 2], dj = std::fabs(zj - z), rj = r[nbj];
            if (dj < rj) {
                double rj_p2 = rj * rj - dj * dj, rj_p = std::sqrt(rj_p2), dij = nb.xyd[i][j];
                if (dij >= ri_p + rj_p) continue;
                if (dij + ri_p < rj_p) { buried = true; break; }
                if (dij + rj_p < ri_p) continue;
                double alpha = std::acos((ri_p2 + dij * dij - rj_p2) / (2.0 * ri_p * dij));
                double beta = std::atan2(nb.yd[i][j], nb.xd[i][j]) + M_PI;
                double inf = beta - alpha, sup = beta + alpha;
                if (inf < 0.0) inf += TWOPI;
                if (sup > 2.0 * M_PI) sup -= TWOPI;
                if (sup < inf) {
                    arc[2 * narc] = 0.0; arc[2 * narc + 1] = sup; arc[2 * narc + 2] = inf; arc[2 * narc + 3] = TWOPI;
                    narc += 2;
                } else {
                    arc[2 * narc] = inf; arc[2 * narc + 1] = sup;
                    narc += 1;
                }
            }
        }
        if (!buried) sasa += delta * ri * exposed_arc(arc, narc);
    }
    return sasa;
}

inline double u01(std::mt19937_64& g) { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

extern "C" {

int lkg_lr_sasa(const double* coords, const double* radii, int32_t n, double* out) {
    if (n < 0 || (n > 0 && (!coords || !radii || !out))) return set_error(LKG_ERR_ARG, "bad sasa args");
    if (n == 0) return set_ok();
    std::vector<double> r(n);
    for (int i = 0; i < n; ++i) r[i] = radii[i] + 1.4;
    Nb nb = neighbours(coords, r, n);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) out[i] = atom_area(i, coords, r, nb, 20);
    return set_ok();
}

// Self-avoiding random chain: bond `bond` A in a uniformly random direction,
// rejected if it leaves the sphere of radius R or comes within `min_sep` A of
// any atom more than two bonds back.  Every 200 consecutive rejections the
// end is trapped: if it sits at the boundary and `patience` attempts have
// passed without the chain reaching a new length, R grows by 0.5 A;
// otherwise the last atoms are removed (1, 2, 4, ... while no new length is
// reached).  Bounded: fails with LKG_ERR_ARG after
// 4000 n + 1e8 attempts.  Deterministic for a seed (std::mt19937_64).
// Writes n x 3 coords and the final radius.
int lkg_synth_chain(uint64_t seed, int32_t n, double r0, double bond, double min_sep, int32_t patience,
                    double* coords, double* r_final) {
    if (n <= 0 || !coords || r0 <= 0 || bond <= 0 || min_sep < 0 || patience <= 0)
        return set_error(LKG_ERR_ARG, "bad chain args");
    std::mt19937_64 g(seed);
    double R = r0;
    const double cs = std::max(min_sep, 1.0);
    std::unordered_map<int64_t, std::vector<int>> grid;
    auto key = [&](double x, double y, double z) {
        int64_t ix = (int64_t)std::floor(x / cs) + (1 << 20), iy = (int64_t)std::floor(y / cs) + (1 << 20),
                iz = (int64_t)std::floor(z / cs) + (1 << 20);
        return (ix << 42) | (iy << 21) | iz;
    };
    std::vector<double> c;
    c.reserve(3 * (size_t)n);
    c.insert(c.end(), {0.0, 0.0, 0.0});
    grid[key(0, 0, 0)].push_back(0);
    int fails = 0, best = 1, pop = 1;
    long long attempts_total = 0, since_best = 0;
    const long long max_attempts = 4000LL * n + 100000000LL;
    const int backtrack_every = 200;
    const double sep2 = min_sep * min_sep;
    while ((int)(c.size() / 3) < n) {
        const int k = (int)(c.size() / 3);
        double u = 2.0 * u01(g) - 1.0, phi = TWOPI * u01(g), s = std::sqrt(std::max(0.0, 1.0 - u * u));
        double x = c[3 * (k - 1)] + bond * s * std::cos(phi), y = c[3 * (k - 1) + 1] + bond * s * std::sin(phi),
               z = c[3 * (k - 1) + 2] + bond * u;
        bool ok = x * x + y * y + z * z <= R * R;
        if (ok) {
            int64_t bx = (int64_t)std::floor(x / cs), by = (int64_t)std::floor(y / cs), bz = (int64_t)std::floor(z / cs);
            for (int64_t dz = -1; dz <= 1 && ok; ++dz)
                for (int64_t dy = -1; dy <= 1 && ok; ++dy)
                    for (int64_t dx = -1; dx <= 1 && ok; ++dx) {
                        auto it = grid.find(((bx + dx + (1 << 20)) << 42) | ((by + dy + (1 << 20)) << 21) | (bz + dz + (1 << 20)));
                        if (it == grid.end()) continue;
                        for (int a : it->second) {
                            if (a >= k - 2) continue;
                            double ex = x - c[3 * a], ey = y - c[3 * a + 1], ez = z - c[3 * a + 2];
                            if (ex * ex + ey * ey + ez * ez < sep2) { ok = false; break; }
                        }
                    }
        }
        if (ok) {
            c.insert(c.end(), {x, y, z});
            grid[key(x, y, z)].push_back(k);
            fails = 0;
            if (k + 1 > best) { best = k + 1; since_best = 0; pop = 1; }
            continue;
        }
        if (++attempts_total > max_attempts)
            return set_error(LKG_ERR_ARG, "random chain did not fit (%d of %d atoms placed)", k, n);
        ++fails;
        if (fails % backtrack_every == 0 && k > 1) {
            // the end is trapped: remove the last `pop` atoms (doubling while
            // no new length is reached) and retry from there
            const double* e = &c[3 * (k - 1)];
            double re = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            if (re > R - 2.0 * min_sep && since_best >= patience) {
                R += 0.5;  // crowded at the boundary: make room
                since_best = 0;
            } else {
                int m = std::min(pop, k - 1);
                for (int t = 0; t < m; ++t) {
                    const int last = (int)(c.size() / 3) - 1;
                    const double* p = &c[3 * last];
                    auto& v = grid[key(p[0], p[1], p[2])];
                    v.erase(std::remove(v.begin(), v.end(), last), v.end());
                    c.resize(c.size() - 3);
                }
                pop = std::min(pop * 2, 256);
            }
            fails = 0;
        }
        ++since_best;
    }
    std::copy(c.begin(), c.end(), coords);
    if (r_final) *r_final = R;
    return set_ok();
}

}  // extern "C"
