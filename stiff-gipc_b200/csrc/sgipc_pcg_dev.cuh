// sgipc_pcg_dev.cuh — device pieces shared by the PCG kernels: matrix / hierarchy views, the
// block SpMV row kernel and block reductions.
#pragma once
#include "sgipc_internal.cuh"

namespace sgipc {

template <class T>
struct MatView {
    const T* fval;   // full symmetric static blocks
    const T* uc;     // unique contact blocks (upper)
    const T* cl;     // the same blocks transposed, in the order of the transposed lists
};

struct Topo {
    int n;
    const int* frow_ptr;
    const int* fcol;
    const int* cu_ptr;
    const int* uc_col;
    const int* cl_ptr;
    const int* cl_col;
};

struct MasView {
    const int* table;
    int L;
    int npos;
    const int* info;
    const int* part_map;
    const int* up;
};

inline Topo topo_of(SgipcCtx* c) {
    Topo t;
    t.n = c->n;
    t.frow_ptr = c->frow_ptr;
    t.fcol = c->fcol;
    t.cu_ptr = c->cu_ptr;
    t.uc_col = c->uc_col;
    t.cl_ptr = c->cl_ptr;
    t.cl_col = c->cl_col;
    return t;
}

// ---- block reduction helpers ---------------------------------------------------------------
template <int NR>
__device__ __forceinline__ void block_sum(double (&v)[NR], double* smem /*[NR*32]*/) {
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[r] += __shfl_down_sync(0xffffffffu, v[r], o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int r = 0; r < NR; r++) smem[r * 32 + w] = v[r];
    __syncthreads();
    if (w == 0) {
        // the warps' sums by warp 0: lane k takes warp k's, then a fixed xor tree (all NR
        // values side by side; a serial loop in one thread waited out each load in turn)
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int r = 0; r < NR; r++) {
            double s = lane < nw ? smem[r * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[r] = s;
        }
    }
}

// ---- SpMV core ------------------------------------------------------------------------------
// Operand gather: x_j (plain vector) or p_j = z_j + beta p_old_j (direction formed on the fly)
template <class T, int NR, bool kL2 = false>
struct Operand {
    const T* a;       // x, or z
    const T* b;       // nullptr, or p_old
    T beta[NR];
    __device__ __forceinline__ void load(int j, T (&xj)[NR][3]) const {
        T va[3][NR], vb[3][NR];
#pragma unroll
        for (int q = 0; q < 3; q++) ldn<kL2, T, NR>(a + (size_t)(3 * j + q) * NR, va[q]);
        if (b) {
#pragma unroll
            for (int q = 0; q < 3; q++) ldn<kL2, T, NR>(b + (size_t)(3 * j + q) * NR, vb[q]);
#pragma unroll
            for (int q = 0; q < 3; q++)
#pragma unroll
                for (int r = 0; r < NR; r++) xj[r][q] = va[q][r] + beta[r] * vb[q][r];
        } else {
#pragma unroll
            for (int q = 0; q < 3; q++)
#pragma unroll
                for (int r = 0; r < NR; r++) xj[r][q] = va[q][r];
        }
    }
};

// Rows are processed by groups of kSpG lanes: lane g of a group takes every kSpG-th block of
// the row's lists (full static row, contact upper, contact transposed) and the group adds
// its partial results with shuffles.
constexpr int kSpG = 4;
inline int spmv_grid(int n) { return nblk((long long)n * kSpG, 256); }

template <class T, int NR, class Op>
__device__ __forceinline__ void row_mv(const Topo& tp, const MatView<T>& A, const Op& x, int i, int g,
                                       T (&acc)[NR][3]) {
#pragma unroll
    for (int r = 0; r < NR; r++) acc[r][0] = acc[r][1] = acc[r][2] = 0;
    if (i < tp.n) {
        // One virtual list per row: the full static row, then its contact blocks, then its
        // transposed contact blocks (stored transposed).  The six bounds are loaded together,
        // and each lane issues every load of a batch of kB entries before the first use (a
        // row is ~13 blocks: one FP32 batch of kB = 4 covers most rows; smaller batches keep
        // FP64 and multi-RHS operands in registers).
        const int s0 = tp.frow_ptr[i], s1 = tp.frow_ptr[i + 1];
        const int u0 = tp.cu_ptr[i], u1 = tp.cu_ptr[i + 1];
        const int k0 = tp.cl_ptr[i], k1 = tp.cl_ptr[i + 1];
        const int ns = s1 - s0, nsu = ns + (u1 - u0), len = nsu + (k1 - k0);
        constexpr int kB = NR == 1 ? (sizeof(T) == 4 ? 4 : 2) : (sizeof(T) == 4 ? 2 : 1);
        for (int e0 = g; e0 < len; e0 += kB * kSpG) {
            int cj[kB];
            T bv[kB][9];
            T xb[kB][NR][3];
#pragma unroll
            for (int u = 0; u < kB; u++) {
                const int e = e0 + u * kSpG;
                const T* src = nullptr;
                cj[u] = -1;
                if (e < ns) {
                    cj[u] = __ldg(tp.fcol + s0 + e);
                    src = A.fval + 9 * (size_t)(s0 + e);
                } else if (e < nsu) {
                    cj[u] = __ldg(tp.uc_col + u0 + (e - ns));
                    src = A.uc + 9 * (size_t)(u0 + (e - ns));
                } else if (e < len) {
                    cj[u] = __ldg(tp.cl_col + k0 + (e - nsu));
                    src = A.cl + 9 * (size_t)(k0 + (e - nsu));
                }
                if (src)
#pragma unroll
                    for (int q = 0; q < 9; q++) bv[u][q] = __ldg(src + q);
            }
#pragma unroll
            for (int u = 0; u < kB; u++)
                if (cj[u] >= 0) x.load(cj[u], xb[u]);
#pragma unroll
            for (int u = 0; u < kB; u++) {
                if (cj[u] < 0) continue;
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const T x0 = xb[u][r][0], x1 = xb[u][r][1], x2 = xb[u][r][2];
                    acc[r][0] += bv[u][0] * x0 + bv[u][1] * x1 + bv[u][2] * x2;
                    acc[r][1] += bv[u][3] * x0 + bv[u][4] * x1 + bv[u][5] * x2;
                    acc[r][2] += bv[u][6] * x0 + bv[u][7] * x1 + bv[u][8] * x2;
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int q = 0; q < 3; q++)
#pragma unroll
            for (int o = 1; o < kSpG; o <<= 1) acc[r][q] += __shfl_xor_sync(0xffffffffu, acc[r][q], o, kSpG);
}

// host-side views of a context
inline MasView mas_view(SgipcCtx* c) {
    MasView m;
    m.table = c->mas.table;
    m.L = c->mas.levelnum;
    m.npos = c->mas.npos;
    m.info = c->mas.info;
    m.part_map = c->mas.part_map;
    m.up = c->mas.up;
    return m;
}

template <class T>
inline MatView<T> mat_view(SgipcCtx* c);
template <>
inline MatView<double> mat_view<double>(SgipcCtx* c) {
    return {c->fval64, c->uc64, c->cl64};
}
template <>
inline MatView<float> mat_view<float>(SgipcCtx* c) {
    return {c->fval32, c->uc32, c->cl32};
}


}  // namespace sgipc
