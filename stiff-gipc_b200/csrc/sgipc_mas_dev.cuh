// sgipc_mas_dev.cuh — device helpers of the MAS restriction shared by the MAS and PCG units.
//
// Every level-(l+1) node is a connected component inside ONE bank of 16 level-l nodes, so
// restricting a vector to the next level is a bank-local reduction: the 16 lanes of a
// half-warp hold one bank, each lane sums the values of the lanes that share its parent
// and the lowest such lane stores the sum.  No atomics, a fixed summation order, and each
// coarse entry written exactly once (replacing the atomic restriction of
// __buildMultiLevelR_optimized_new, StiffGIPC/MASPreconditioner.cu:729-847).
#pragma once
#include "sgipc_internal.cuh"

namespace sgipc {

// All 16 lanes of a half-warp call this together (values of idle lanes: parent = -1).
// v[NR*3] holds this node's value; s receives the sum over the lanes of the half-warp with
// the same parent (a butterfly when the half-warp is one group, else added in lane order);
// returns true on the lowest such lane.
template <class M, int NR>
__device__ __forceinline__ bool bank_group_sum(int parent, const M (&v)[NR * 3], M (&s)[NR * 3]) {
    // Each half-warp (one bank) decides for itself, with half-warp masks, so that a bank's
    // sums never depend on the bank beside it: one group (a connected bank, the common
    // case) adds by a butterfly, several groups in lane order.
    const unsigned half = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
    const bool one = __all_sync(half, parent == __shfl_sync(half, parent, 0, 16));
    if (one) {
#pragma unroll
        for (int k = 0; k < NR * 3; k++) {
            s[k] = v[k];
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) s[k] += __shfl_xor_sync(half, s[k], o, 16);
        }
        return (threadIdx.x & 15) == 0;
    }
#pragma unroll
    for (int k = 0; k < NR * 3; k++) s[k] = 0;
    int leader = -1;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        int pj = __shfl_sync(half, parent, j, 16);
        bool same = pj == parent;
        if (same && leader < 0) leader = j;
#pragma unroll
        for (int k = 0; k < NR * 3; k++) {
            M vj = __shfl_sync(half, v[k], j, 16);
            if (same) s[k] += vj;
        }
    }
    return (int)(threadIdx.x & 15) == leader;
}

// The group sum above, stored at R[3*parent+q][r] (when parent >= 0) by the group's leader.
template <class M, int NR>
__device__ __forceinline__ void bank_reduce_store(int parent, const M (&v)[NR * 3], M* __restrict__ R) {
    M s[NR * 3];
    const bool lead = bank_group_sum<M, NR>(parent, v, s);
    if (parent >= 0 && lead) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            M o[NR];
#pragma unroll
            for (int r = 0; r < NR; r++) o[r] = s[r * 3 + q];
            stn<M, NR>(R + (size_t)(3 * parent + q) * NR, o);
        }
    }
}

// Levels l_first .. L-2 -> l_first+1 .. L-1, run by ONE CTA (levels >= 1 are at most npos/16
// nodes).
// kL2: level 1 was written by other CTAs of the same kernel (read it through L2).
template <class M, int NR, bool kL2 = false>
__device__ __forceinline__ void restrict_coarse_cta(const int* __restrict__ info, const int* __restrict__ up, int L,
                                                    M* __restrict__ R, int l_first = 1) {
    for (int l = l_first; l + 1 < L; l++) {
        const int count = info[8 + l], start = info[l];
        for (int base = 0; base < count; base += blockDim.x) {
            const int a = base + threadIdx.x;
            M v[NR * 3];
            int par = -1;
            if (a < count) {
                const int g = start + a;
                par = up[g];
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    M t[NR];
                    ldn<kL2, M, NR>(R + (size_t)(3 * g + q) * NR, t);
#pragma unroll
                    for (int r = 0; r < NR; r++) v[r * 3 + q] = t[r];
                }
            } else {
#pragma unroll
                for (int k = 0; k < NR * 3; k++) v[k] = 0;
            }
            bank_reduce_store<M, NR>(par, v, R);
        }
        __syncthreads();
    }
}

}  // namespace sgipc
