// Receptor far field phi(x) = sum_{i: 10 < |x - r_i| <= 30} q_i / |x - r_i|^2
// on the 0.5 A grid of ReceptorField (grid_dna.rs:44-149), built on the GPU
// with the same bits as the reference's host builder.
//
// The reference scatters atom by atom and accumulates in f32, so each grid
// point receives its (q/d^2 as f32) terms in ascending atom order.  Here one
// thread owns one grid point (a block owns an 8 x 8 x 4 brick) and gathers:
// charged atoms are streamed in index order in chunks of blockDim, each
// chunk is compacted in order to the atoms whose distance to the brick can
// fall in (10, 30] A, and every thread then walks that list in order and
// applies the reference's exact write test
//      dyz2 < 30^2  and  10^2 < d2 <= 30^2
// with dx = (lo0 + ix*s) - cx, dy = (lo1 + iy*s) - cy, dz = (lo2 + iz*s) - cz,
// dyz2 = dy*dy + dz*dz, d2 = dx*dx + dyz2, all in f64 without contraction
// (this file is compiled with --fmad=false), then phi += (float)(q / d2).
// The reference's per-atom scatter window (+-62 points) and its x-slab pruning
// never exclude a point that passes this test, so the write set, the values
// and their order per point are the reference's.
#include "lkg_internal.h"

namespace lkg {

namespace {

constexpr int BX = 8, BY = 8, BZ = 4, BT = BX * BY * BZ;

__global__ void __launch_bounds__(BT) k_field(const double4* __restrict__ atoms, int n,
                                              double lo0, double lo1, double lo2, double s,
                                              int nx, int ny, int nz, float* __restrict__ phi) {
    __shared__ double4 s_list[BT];
    __shared__ int s_cnt[BT / 32];
    const int bx = blockIdx.x * BX, by = blockIdx.y * BY, bz = blockIdx.z * BZ;
    const int tx = threadIdx.x % BX, ty = (threadIdx.x / BX) % BY, tz = threadIdx.x / (BX * BY);
    const int ix = bx + tx, iy = by + ty, iz = bz + tz;
    const double r2min = 100.0, r2max = 900.0;
    // brick bounds (grid coordinates are exactly lo + i*s)
    const double xa = lo0 + (double)bx * s, xb = lo0 + (double)min(bx + BX - 1, nx - 1) * s;
    const double ya = lo1 + (double)by * s, yb = lo1 + (double)min(by + BY - 1, ny - 1) * s;
    const double za = lo2 + (double)bz * s, zb = lo2 + (double)min(bz + BZ - 1, nz - 1) * s;
    const double px = lo0 + (double)ix * s, py = lo1 + (double)iy * s, pz = lo2 + (double)iz * s;
    float acc = 0.0f;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < n; base += BT) {
        const int a = base + threadIdx.x;
        bool keep = false;
        double4 at = make_double4(0, 0, 0, 0);
        if (a < n) {
            at = atoms[a];
            double ex = fmax(fmax(xa - at.x, at.x - xb), 0.0);
            double ey = fmax(fmax(ya - at.y, at.y - yb), 0.0);
            double ez = fmax(fmax(za - at.z, at.z - zb), 0.0);
            double near2 = ex * ex + ey * ey + ez * ez;
            double fx = fmax(fabs(xa - at.x), fabs(xb - at.x));
            double fy = fmax(fabs(ya - at.y), fabs(yb - at.y));
            double fz = fmax(fabs(za - at.z), fabs(zb - at.z));
            double far2 = fx * fx + fy * fy + fz * fz;
            keep = near2 <= r2max * (1.0 + 1e-9) && far2 > r2min * (1.0 - 1e-9);
        }
        // order-preserving compaction of the chunk
        unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_cnt[wid] = __popc(m);
        __syncthreads();
        int off = 0, tot = 0;
        for (int w = 0; w < BT / 32; ++w) { if (w < wid) off += s_cnt[w]; tot += s_cnt[w]; }
        if (keep) s_list[off + __popc(m & ((1u << lane) - 1u))] = at;
        __syncthreads();
        for (int k = 0; k < tot; ++k) {
            const double4 c = s_list[k];
            const double dz = pz - c.z;
            const double dy = py - c.y;
            const double dyz2 = dy * dy + dz * dz;
            const double dx = px - c.x;
            const double d2 = dx * dx + dyz2;
            if (dyz2 < r2max && d2 > r2min && d2 <= r2max) acc += (float)(c.w / d2);
        }
        __syncthreads();
    }
    if (ix < nx && iy < ny && iz < nz) phi[((size_t)iz * ny + iy) * nx + ix] = acc;
}

__global__ void k_far_sum(const float* __restrict__ phi, int nx, int ny, int nz, float ox, float oy,
                          float oz, float sp, const float* __restrict__ xyz, const float* __restrict__ q,
                          int n, double* __restrict__ out) {
    // far_field.cu:43-57 semantics: one thread per atom, trilinear sample
    __shared__ double s_red[32];
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (j < n && q[j] != 0.f) {
        float x = xyz[3 * j], y = xyz[3 * j + 1], z = xyz[3 * j + 2];
        float fx = (x - ox) / sp, fy = (y - oy) / sp, fz = (z - oz) / sp;
        if (fx >= 0.f && fy >= 0.f && fz >= 0.f && fx < (float)(nx - 1) && fy < (float)(ny - 1) &&
            fz < (float)(nz - 1)) {
            int ix = (int)fx, iy = (int)fy, iz = (int)fz;
            if (ix + 1 < nx && iy + 1 < ny && iz + 1 < nz) {
                float tx = fx - ix, ty = fy - iy, tz = fz - iz;
                size_t sy = nx, sz = (size_t)nx * ny;
                const float* p = phi + iz * sz + iy * sy + ix;
                float c00 = p[0] * (1.f - tx) + p[1] * tx, c10 = p[sy] * (1.f - tx) + p[sy + 1] * tx;
                float c01 = p[sz] * (1.f - tx) + p[sz + 1] * tx;
                float c11 = p[sz + sy] * (1.f - tx) + p[sz + sy + 1] * tx;
                float c0 = c00 * (1.f - ty) + c10 * ty, c1 = c01 * (1.f - ty) + c11 * ty;
                v = (double)(q[j] * (c0 * (1.f - tz) + c1 * tz));
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += s_red[w];
        atomicAdd(out, s);
    }
}

}  // namespace

cudaError_t build_field_device(const double* d_atoms, const double* /*unused*/, int n,
                               const double lo[3], const int dims[3], double spacing,
                               float* d_phi, cudaStream_t s) {
    dim3 grid((dims[0] + BX - 1) / BX, (dims[1] + BY - 1) / BY, (dims[2] + BZ - 1) / BZ);
    k_field<<<grid, BT, 0, s>>>((const double4*)d_atoms, n, lo[0], lo[1], lo[2], spacing,
                                dims[0], dims[1], dims[2], d_phi);
    return cudaGetLastError();
}

cudaError_t launch_far_field_sum(const float* phi, int nx, int ny, int nz, float ox, float oy,
                                 float oz, float sp, const float* coords, const float* q, int n,
                                 double* d_result, cudaStream_t s) {
    int t = 256, b = (n + t - 1) / t;
    if (b < 1) b = 1;
    k_far_sum<<<b, t, 0, s>>>(phi, nx, ny, nz, ox, oy, oz, sp, coords, q, n, d_result);
    return cudaGetLastError();
}

__global__ void k_phi_bricks(const float* __restrict__ src, int nx, int ny, int nz, int nbx, int nby,
                             float* __restrict__ dst, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const size_t b = i >> 6;
    const int l = (int)(i & 63);
    const int x = (int)(b % nbx) * 4 + (l & 3);
    const int y = (int)((b / nbx) % nby) * 4 + ((l >> 2) & 3);
    const int z = (int)(b / ((size_t)nbx * nby)) * 4 + (l >> 4);
    dst[i] = (x < nx && y < ny && z < nz) ? src[((size_t)z * ny + y) * nx + x] : 0.f;
}

cudaError_t phi_to_bricks(const float* src, int nx, int ny, int nz, float* dst, cudaStream_t s) {
    const int nbx = (nx + 3) / 4, nby = (ny + 3) / 4, nbz = (nz + 3) / 4;
    const size_t total = (size_t)nbx * nby * nbz * 64;
    k_phi_bricks<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(src, nx, ny, nz, nbx, nby, dst, total);
    return cudaGetLastError();
}

}  // namespace lkg
