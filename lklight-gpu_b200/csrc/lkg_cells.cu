// Receptor set-up on the GPU: the fine cell grid's counting sort and the
// packing of the position-sorted device arrays (the GPU cell list of
// src/gpu_score.rs:75-144, on this library's finer grid).
//
//   1. k_cell_of     cell of every atom, from its f32 coordinates by the same
//                    f32 operations as the host build (floor((x - o) / edge),
//                    clamped), and the per-cell counts (atomicAdd)
//   2. scan          exclusive prefix of the counts -> cell_start (ncell + 1)
//   3. k_scatter     every atom to a slot of its cell (atomic cursor: the
//                    order inside a cell is arbitrary here)
//   4. k_cell_order  each cell's atoms sorted by index (insertion sort: cells
//                    hold a few atoms), so the order is the host build's
//                    stable counting sort, bit for bit
//   5. k_pack        f32 / f64 atom arrays in cell order and the
//                    sorted -> caller index map
// The host build (lkg_runtime.cu build_receptor) stays as the check: a GPU
// test scores the same poses on complexes set up both ways and requires
// equal bits.
#include "lkg_runtime.h"

namespace lkg {
namespace {

__global__ void k_cell_of(const double* __restrict__ c, int n, float ox, float oy, float oz, float ix, float iy,
                          float iz, int nx, int ny, int nz, int* __restrict__ cell, int* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cx = min(max((int)floorf(((float)c[3 * i] - ox) * ix), 0), nx - 1);
    const int cy = min(max((int)floorf(((float)c[3 * i + 1] - oy) * iy), 0), ny - 1);
    const int cz = min(max((int)floorf(((float)c[3 * i + 2] - oz) * iz), 0), nz - 1);
    const int k = (cz * ny + cy) * nx + cx;
    cell[i] = k;
    atomicAdd(count + k, 1);
}

// exclusive scan of n ints, 2048 a block (two a thread), block totals out
constexpr int SCAN_T = 1024, SCAN_B = 2 * SCAN_T;

__global__ void k_scan_block(const int* __restrict__ in, int* __restrict__ out, size_t n, int* __restrict__ sums) {
    __shared__ int s[SCAN_B];
    const size_t base = (size_t)blockIdx.x * SCAN_B;
    const int t = threadIdx.x;
    s[2 * t] = base + 2 * t < n ? in[base + 2 * t] : 0;
    s[2 * t + 1] = base + 2 * t + 1 < n ? in[base + 2 * t + 1] : 0;
    // work-efficient scan (up-sweep, down-sweep) of the block's 2048 values
    int off = 1;
    for (int d = SCAN_T; d > 0; d >>= 1, off <<= 1) {
        __syncthreads();
        if (t < d) {
            const int a = off * (2 * t + 1) - 1, b = off * (2 * t + 2) - 1;
            s[b] += s[a];
        }
    }
    __syncthreads();
    if (t == 0) {
        if (sums) sums[blockIdx.x] = s[SCAN_B - 1];
        s[SCAN_B - 1] = 0;
    }
    for (int d = 1; d <= SCAN_T; d <<= 1) {
        off >>= 1;
        __syncthreads();
        if (t < d) {
            const int a = off * (2 * t + 1) - 1, b = off * (2 * t + 2) - 1;
            const int v = s[a];
            s[a] = s[b];
            s[b] += v;
        }
    }
    __syncthreads();
    if (base + 2 * t < n) out[base + 2 * t] = s[2 * t];
    if (base + 2 * t + 1 < n) out[base + 2 * t + 1] = s[2 * t + 1];
}

__global__ void k_scan_add(int* __restrict__ out, size_t n, const int* __restrict__ offs) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offs[i / SCAN_B];
}

// exclusive scan of in[0..n) into out[0..n), levels of 2048-value blocks
cudaError_t scan_exclusive(const int* in, int* out, size_t n, DBuf* tmp, int level, cudaStream_t s) {
    const size_t blocks = (n + SCAN_B - 1) / SCAN_B;
    if (blocks == 1) {
        k_scan_block<<<1, SCAN_T, 0, s>>>(in, out, n, nullptr);
        return cudaGetLastError();
    }
    if (level >= 3) return cudaErrorInvalidValue;   // 2048^4 values: beyond any grid built here
    cudaError_t e = tmp[2 * level].reserve(blocks * sizeof(int));
    if (e == cudaSuccess) e = tmp[2 * level + 1].reserve(blocks * sizeof(int));
    if (e != cudaSuccess) return e;
    int* sums = tmp[2 * level].as<int>();
    int* offs = tmp[2 * level + 1].as<int>();
    k_scan_block<<<(unsigned)blocks, SCAN_T, 0, s>>>(in, out, n, sums);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = scan_exclusive(sums, offs, blocks, tmp, level + 1, s)) != cudaSuccess) return e;
    k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, offs);
    return cudaGetLastError();
}

__global__ void k_scatter(const int* __restrict__ cell, int n, int* __restrict__ cursor, int* __restrict__ order) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) order[atomicAdd(cursor + cell[i], 1)] = i;
}

__global__ void k_cell_order(const int* __restrict__ cs, size_t ncell, int* __restrict__ order) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ncell) return;
    const int b = cs[k], e = cs[k + 1];
    for (int i = b + 1; i < e; ++i) {
        const int v = order[i];
        int j = i - 1;
        while (j >= b && order[j] > v) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = v;
    }
}

struct MolDev {
    const double *c, *q, *svdw, *rad, *eps, *des, *asa;
    const uint8_t *heavy, *excl;
};

__global__ void k_pack(MolDev m, const int* __restrict__ order, int n, float4* __restrict__ pos,
                       float4* __restrict__ par, float2* __restrict__ sol, double4* __restrict__ pos64,
                       double4* __restrict__ par64, double2* __restrict__ sol64, int* __restrict__ rorig) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = order[k];
    const double x = m.c[3 * i], y = m.c[3 * i + 1], z = m.c[3 * i + 2];
    pos[k] = make_float4((float)x, (float)y, (float)z, (float)m.q[i]);
    par[k] = make_float4((float)m.svdw[i], (float)m.rad[i], m.heavy[i] ? 1.f : 0.f, m.excl[i] ? 1.f : 0.f);
    sol[k] = make_float2((float)m.des[i], (float)m.asa[i]);
    pos64[k] = make_double4(x, y, z, m.q[i]);
    par64[k] = make_double4(m.svdw[i], m.rad[i], m.eps[i], m.heavy[i] ? 1.0 : 0.0);
    sol64[k] = make_double2(m.des[i], m.asa[i]);
    rorig[k] = i;
}

template <class T>
cudaError_t up(DBuf& b, const std::vector<T>& v, cudaStream_t s) {
    cudaError_t e = b.reserve(std::max<size_t>(v.size(), 1) * sizeof(T));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

}  // namespace

// The receptor's cell-sorted device arrays and cell_start (ncell + 1), built
// on the GPU for grid origin o, cells nc (x counts sub-cells) and inverse
// cell edges inv_e; the same arrays, bit for bit, as the host build.
int build_receptor_device(lkg_ctx* ctx, const MolIn& R, ComplexRec& cr, const float o[3], const int nc[3],
                          const float inv_e[3]) {
    const int n = R.n;
    const size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
    cudaStream_t s = ctx->stream;
    DBuf c, q, svdw, rad, eps, des, asa, heavy, excl, cell, count, cursor, order, tmp[6];
    LKG_CK(up(c, R.c, s), "receptor upload");
    LKG_CK(up(q, R.q, s), "receptor upload");
    LKG_CK(up(svdw, R.svdw, s), "receptor upload");
    LKG_CK(up(rad, R.rad, s), "receptor upload");
    LKG_CK(up(eps, R.eps, s), "receptor upload");
    LKG_CK(up(des, R.des, s), "receptor upload");
    LKG_CK(up(asa, R.asa, s), "receptor upload");
    LKG_CK(up(heavy, R.heavy, s), "receptor upload");
    LKG_CK(up(excl, R.excl, s), "receptor upload");
    LKG_CK(cell.reserve(std::max(n, 1) * sizeof(int)), "receptor cells");
    LKG_CK(count.reserve((ncell + 1) * sizeof(int)), "receptor cells");
    LKG_CK(cursor.reserve((ncell + 1) * sizeof(int)), "receptor cells");
    LKG_CK(order.reserve(std::max(n, 1) * sizeof(int)), "receptor cells");
    LKG_CK(cr.cell_start.reserve((ncell + 1) * sizeof(int)), "receptor cells");
    LKG_CK(cudaMemsetAsync(count.p, 0, (ncell + 1) * sizeof(int), s), "receptor cells");
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (n > 0) {
        k_cell_of<<<nb, 256, 0, s>>>(c.as<double>(), n, o[0], o[1], o[2], inv_e[0], inv_e[1], inv_e[2], nc[0], nc[1],
                                     nc[2], cell.as<int>(), count.as<int>());
        LKG_CK(cudaGetLastError(), "receptor cells");
    }
    // cell_start[k] = atoms in cells < k, for k = 0 .. ncell (the count of the
    // extra cell ncell is 0, so its prefix is n)
    LKG_CK(scan_exclusive(count.as<int>(), cr.cell_start.as<int>(), ncell + 1, tmp, 0, s), "receptor cells");
    LKG_CK(cudaMemcpyAsync(cursor.p, cr.cell_start.p, (ncell + 1) * sizeof(int), cudaMemcpyDeviceToDevice, s),
           "receptor cells");
    LKG_CK(cr.rpos.reserve(std::max(n, 1) * sizeof(float4)), "receptor arrays");
    LKG_CK(cr.rpar.reserve(std::max(n, 1) * sizeof(float4)), "receptor arrays");
    LKG_CK(cr.rsolv.reserve(std::max(n, 1) * sizeof(float2)), "receptor arrays");
    LKG_CK(cr.rpos64.reserve(std::max(n, 1) * sizeof(double4)), "receptor arrays");
    LKG_CK(cr.rpar64.reserve(std::max(n, 1) * sizeof(double4)), "receptor arrays");
    LKG_CK(cr.rsolv64.reserve(std::max(n, 1) * sizeof(double2)), "receptor arrays");
    LKG_CK(cr.rorig.reserve(std::max(n, 1) * sizeof(int)), "receptor arrays");
    if (n > 0) {
        k_scatter<<<nb, 256, 0, s>>>(cell.as<int>(), n, cursor.as<int>(), order.as<int>());
        k_cell_order<<<(unsigned)((ncell + 255) / 256), 256, 0, s>>>(cr.cell_start.as<int>(), ncell, order.as<int>());
        const MolDev m{c.as<double>(), q.as<double>(), svdw.as<double>(), rad.as<double>(), eps.as<double>(),
                       des.as<double>(), asa.as<double>(), heavy.as<uint8_t>(), excl.as<uint8_t>()};
        k_pack<<<nb, 256, 0, s>>>(m, order.as<int>(), n, cr.rpos.as<float4>(), cr.rpar.as<float4>(),
                                  cr.rsolv.as<float2>(), cr.rpos64.as<double4>(), cr.rpar64.as<double4>(),
                                  cr.rsolv64.as<double2>(), cr.rorig.as<int>());
        LKG_CK(cudaGetLastError(), "receptor pack");
        ctx->launches += 5;
    }
    // the staging buffers are freed on return: wait for the kernels first
    LKG_CK(cudaStreamSynchronize(s), "receptor set-up");
    return set_ok();
}

}  // namespace lkg
