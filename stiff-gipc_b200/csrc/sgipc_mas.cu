// sgipc_mas.cu — multilevel additive Schwarz (MAS) preconditioner.
//
// Semantics of StiffGIPC's MASPreconditioner (MASPreconditioner.cu:29-2262):
//   level 0   : the partition positions; a domain is a bank of 16 consecutive positions;
//   level l+1 : the connected components, inside each level-l bank, of the graph made of
//               mesh edges (StiffGIPC/load_mesh.cpp:934-1040) and of every vertex pair of
//               every contact pair (_buildCollisionConnection_new, :1132); components are
//               numbered bank by bank, by their lowest lane (_buildLevel1_new, _prefixSumLx);
//   levels    : computeNumLevels (:1724-1743), at most 6;
//   matrices  : the bank-diagonal 48x48 blocks of P_l^T A P_l over the FEM block rows
//               (PrepareHessian_bcoo, :1816-2093), a zero diagonal entry replaced by 1 and
//               inverted by Gauss-Jordan without pivoting (__inverse6_P96x96, :630-726);
//   apply     : z = sum_l P_l A_l^-1 P_l^T r (__buildMultiLevelR_optimized_new,
//               _schwarzLocalXSym6, __collectFinalZ_new, :729-1027).
// The B200 version keeps every level's bookkeeping on the device (no per-level host
// copy), builds the per-level masks with one thread per vertex / per contact pair and
// resolves a bank's components with one thread per bank.
#include <cub/cub.cuh>
#include <mutex>
#include <vector>

#include "sgipc_internal.cuh"
#include "sgipc_mas_dev.cuh"

using namespace sgipc;

namespace {

__global__ void k_init_level0(int nv, const int* __restrict__ real_map, int L, int* __restrict__ node,
                              int* __restrict__ table, int* __restrict__ info, int npos, int* __restrict__ up) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v == 0) {
        info[0] = 0;     // start of level 0
        info[8] = npos;  // count of level 0 (positions, padding included)
        if (L == 1) info[16] = npos;
    }
    if (v < npos) up[v] = -1;  // padding positions have no parent
    if (v >= nv) return;
    int p = real_map[v];
    node[v] = p;
    table[(size_t)v * L] = p;
}

// OR `bit` into mask[a]; lanes of a warp with the same target combine their bits first
// (at coarse levels most edges of a warp land on the same few nodes)
__device__ __forceinline__ void mask_or_warp(uint32_t* mask, int a, uint32_t bit) {
    const unsigned grp = __match_any_sync(0xffffffffu, a);
    const uint32_t bits = __reduce_or_sync(grp, bit);
    if (a >= 0 && bits && (int)(threadIdx.x & 31) == __ffs(grp) - 1) atomicOr(mask + a, bits);
}

// one thread per neighbour-list slot (row[k] is the slot's vertex)
__global__ void k_mask_edges(int nnz, const int* __restrict__ row, const int* __restrict__ nbr,
                             const int* __restrict__ node, uint32_t* __restrict__ mask) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    int a = -1;
    uint32_t bit = 0;
    if (k < nnz) {
        a = node[row[k]];
        const int b = node[nbr[k]];
        if (a != b && (a >> 4) == (b >> 4)) bit = 1u << (b & 15);
    }
    mask_or_warp(mask, bit ? a : -1, bit);
}

// The connectivity bits of one contact pair (its decoded vertices, all ordered pairs inside
// one bank); every lane of the warp calls it (idle lanes: e = nullptr).
__device__ __forceinline__ void mask_pair_warp(const int4* e_ptr, int nv, const int* __restrict__ node,
                                               uint32_t* __restrict__ mask) {
    int v[4] = {-1, -1, -1, -1}, n = 0;
    if (e_ptr) {
        const int4 e = *e_ptr;
        if (e.x >= 0) {
            v[0] = e.x; v[1] = e.y; v[2] = e.z; v[3] = e.w < 0 ? -e.w - 1 : e.w; n = 4;
        } else {
            v[0] = -e.x - 1;
            if (e.z < 0) {
                if (e.y < 0) { v[1] = -e.y - 1; v[2] = -e.z - 1; v[3] = -e.w - 1; n = 4; }
                else { v[1] = e.y; n = 2; }
            } else if (e.w < 0) {
                if (e.y < 0) { v[1] = -e.y - 1; v[2] = e.z; v[3] = -e.w - 1; n = 4; }
                else { v[1] = e.y; v[2] = e.z; n = 3; }
            } else { v[1] = e.y; v[2] = e.z; v[3] = e.w; n = 4; }
        }
    }
    int a[4] = {-1, -1, -1, -1};
    for (int i = 0; i < n; i++) a[i] = (v[i] >= 0 && v[i] < nv) ? node[v[i]] : -1;
    // the 12 ordered vertex pairs, each one warp-aggregated OR
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (i == j) continue;
            const int x = a[i], y = a[j];
            const bool on = x >= 0 && y >= 0 && x != y && (x >> 4) == (y >> 4);
            mask_or_warp(mask, on ? x : -1, on ? 1u << (y & 15) : 0u);
        }
}

__global__ void k_mask_pairs(int np, const int4* __restrict__ pairs, int nv, const int* __restrict__ node,
                             uint32_t* __restrict__ mask) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    mask_pair_warp(p < np ? pairs + p : nullptr, nv, node, mask);
}

// Half a warp per bank (bk; all 32 lanes call it), writing its nodes' component ranks and
// its component count (bank_cnt[bk], for bk <= bank_last; zero beyond the level's banks).
__device__ __forceinline__ void bank_components_half(int bk, int bank_last, int count, int level,
                                                     const uint32_t* __restrict__ mask,
                                                     const int* __restrict__ part_map, int* __restrict__ rank,
                                                     int* __restrict__ bank_cnt) {
    const int i = threadIdx.x & 15;
    const int nbank = (count + 15) >> 4;
    const int lo = bk << 4;
    const bool inb = bk < nbank;
    const bool real = inb && lo + i < count && (level > 0 || part_map[lo + i] >= 0);
    uint32_t m = real ? (mask[lo + i] | (1u << i)) : 0u;
#pragma unroll 1
    for (int it = 0; it < 5; it++) {
        uint32_t acc = m;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint32_t mj = __shfl_sync(0xffffffffu, m, j, 16);
            if (m & (1u << j)) acc |= mj;
        }
        m = acc;
    }
    const int lead = __ffs(m) - 1;
    const uint32_t leaders = (__ballot_sync(0xffffffffu, real && lead == i) >> (threadIdx.x & 16)) & 0xffffu;
    if (inb && lo + i < count) rank[lo + i] = lead < 0 ? 0 : __popc(leaders & ((1u << lead) - 1u));
    if (i == 0 && bk <= bank_last) bank_cnt[bk] = inb ? __popc(leaders) : 0;
}

// Half a warp per bank, lane i holding node i's connectivity row: components by repeated
// squaring of the reachability rows (each round doubles the path length, so five rounds
// close 16 nodes), numbered by their lowest lane.  At level 0 the padding positions
// (part_map < 0) are no node and form no component (_preparePrefixSumL0_new /
// _buildLevel1_new skip them, MASPreconditioner.cu:157-270).
__global__ void k_bank_components(int nbank_cap, const int* __restrict__ info, int level,
                                  const uint32_t* __restrict__ mask, const int* __restrict__ part_map,
                                  int* __restrict__ rank, int* __restrict__ bank_cnt) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    bank_components_half(gt >> 4, nbank_cap, info[8 + level], level, mask, part_map, rank, bank_cnt);
}

__global__ void k_assign(int nv, int L, int level, const int* __restrict__ bank_off, const int* __restrict__ rank,
                         int* __restrict__ node, int* __restrict__ table, int* __restrict__ info,
                         int* __restrict__ up) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int count = info[8 + level];
    const int start = info[level];
    const int start_next = start + ((count + 15) & ~15);
    if (v == 0) {
        int nbank = (count + 15) >> 4;
        info[level + 1] = start_next;
        info[8 + level + 1] = bank_off[nbank];
        if (level + 2 == L) info[16] = start_next + ((bank_off[nbank] + 15) & ~15);
    }
    if (v >= nv) return;
    int a = node[v];
    int nn = bank_off[a >> 4] + rank[a];
    node[v] = nn;
    table[(size_t)v * L + level + 1] = start_next + nn;
    up[start + a] = start_next + nn;  // every vertex of node a writes the same parent
    if (level + 2 == L) up[start_next + nn] = -1;
}

// Scatter one 3x3 block B at (r,c) (and B^T at (c,r)) into every level from l_first on whose
// bank holds both endpoints.  Lanes of a warp whose blocks land on the same coarse entry
// add them first (match + shuffles) so that one lane issues the atomics.  The groups nest
// (blocks with the same (cluster(r), cluster(c)) at level l share it at level l + 1), so
// each level adds only the previous level's group sums, carried by their leaders: a few
// per warp at the coarse levels, where nearly every block of the warp lands on one entry.
// Levels l >= l_top (at most kTopLevels of them, each one domain of <= 16 nodes) go to the
// CTA's shared copies s_top[l - l_top] of their domains instead (flushed by flush_top).
constexpr int kTopLevels = 2;
__device__ __forceinline__ void scatter_block_warp(double* dom, const int* __restrict__ table, int L, int r, int c,
                                                   const double (&B)[9], bool valid, int l_first, int l_top,
                                                   double (*s_top)[2304]) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    double V[9];
#pragma unroll
    for (int q = 0; q < 9; q++) V[q] = valid ? B[q] : 0.0;
    unsigned carriers = __ballot_sync(full, valid);  // lanes holding a partial sum
    const unsigned long long diag = r == c ? 1ull : 0ull;
    // the clusters of r and c at every level, loaded together up front (one round trip)
    int tr[SGIPC_MAX_LEVELS], tc[SGIPC_MAX_LEVELS];
#pragma unroll
    for (int l = 0; l < SGIPC_MAX_LEVELS; l++) {
        const bool in = valid && l >= l_first && l < L;
        tr[l] = in ? table[(size_t)r * L + l] : -1;
        tc[l] = in ? table[(size_t)c * L + l] : -1;
    }
#pragma unroll
    for (int l = 0; l < SGIPC_MAX_LEVELS; l++) {
        if (l < l_first || l >= L) continue;  // warp-uniform
        int ga = -1, gb = -1;
        if (valid) {
            ga = tr[l];
            gb = tc[l];
        }
        // target (ga, gb) and whether the block is a diagonal one
        const unsigned long long key =
            valid ? (((unsigned long long)(unsigned)ga << 33) | ((unsigned long long)(unsigned)gb << 1) | diag) : ~0ull;
        const unsigned grp = __match_any_sync(full, key);
        const bool lead = lane == __ffs(grp) - 1;
        double S[9];
#pragma unroll
        for (int q = 0; q < 9; q++) S[q] = 0.0;
        unsigned m = grp & carriers;
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
#pragma unroll
            for (int q = 0; q < 9; q++) S[q] += __shfl_sync(grp, V[q], j);
        }
        if (valid && lead && (ga >> 4) == (gb >> 4)) {
            double* D = l >= l_top ? s_top[l - l_top] : dom + (size_t)(ga >> 4) * 2304;
            int ra = 3 * (ga & 15), cb = 3 * (gb & 15);
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    double v = S[3 * i + j];
                    if (v == 0.0) continue;
                    atomicAdd(D + (ra + i) * 48 + cb + j, v);
                    if (r != c) atomicAdd(D + (cb + j) * 48 + ra + i, v);
                }
        }
#pragma unroll
        for (int q = 0; q < 9; q++) V[q] = lead ? S[q] : 0.0;
        carriers = __ballot_sync(full, valid && lead);
    }
}

// The top levels' domain copies of the CTA: zeroed, filled by scatter_block_warp, then added
// to the global domains (one atomic per non-zero entry and CTA instead of one per warp
// group: every block of the grid lands on the few entries of these levels).
// levels l >= l_top accumulated per CTA: the top levels (at most kTopLevels) whose nodes
// form one domain starting on a domain boundary (info[l] = first node, info[8 + l] = count)
__device__ __forceinline__ int top_levels_dev(const int* __restrict__ info, int L) {
    int l = L;
    while (l > 1 && L - (l - 1) <= kTopLevels && info[8 + l - 1] <= 16 && (info[l - 1] & 15) == 0) l--;
    return l;
}

__device__ __forceinline__ void zero_top(int ntop, double (*s_top)[2304]) {
    for (int k = threadIdx.x; k < ntop * 2304; k += blockDim.x) s_top[k / 2304][k % 2304] = 0.0;
    __syncthreads();
}

__device__ __forceinline__ void flush_top(const int* __restrict__ info, int l_top, int ntop, double (*s_top)[2304],
                                          double* __restrict__ dom) {
    __syncthreads();
    for (int k = threadIdx.x; k < ntop * 2304; k += blockDim.x) {
        const double v = s_top[k / 2304][k % 2304];
        if (v != 0.0) atomicAdd(dom + (size_t)(info[l_top + k / 2304] >> 4) * 2304 + k % 2304, v);
    }
}

__global__ void k_scatter_static(int nnz, const int* __restrict__ slot_row, const int* __restrict__ col,
                                 const double* __restrict__ val, const int* __restrict__ table, int L,
                                 const int* __restrict__ info, double* __restrict__ dom) {
    __shared__ double s_top[kTopLevels][2304];
    if (info[21]) return;  // aborted hierarchy build: the host rejects its tables
    const int l_top = top_levels_dev(info, L), ntop = L - l_top;
    zero_top(ntop, s_top);
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = s < nnz;
    double B[9];
#pragma unroll
    for (int q = 0; q < 9; q++) B[q] = valid ? val[9 * (size_t)s + q] : 0.0;
    scatter_block_warp(dom, table, L, valid ? slot_row[s] : 0, valid ? col[s] : 0, B, valid, 1, l_top, s_top);
    flush_top(info, l_top, ntop, s_top, dom);
}

// Level 0 of the static blocks, without atomics: the level-0 domains are the banks of the
// fixed position map, so each entry (a, b) of domain d takes one static block (or its
// transpose, or nothing) known at creation.  One thread per 3x3 entry writes it whole.
// The grid also zeroes the coarser domains [nd0, info[16] / 16) that the scatters add to
// (at most ndom_cap domains in all).  Nothing is written after an aborted hierarchy build
// (info[21] set), whose tables the host rejects.
__global__ void k_fill_level0(int nd0, int ndom_cap, const int* __restrict__ map0, const double* __restrict__ val,
                              const int* __restrict__ info, double* __restrict__ dom) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (info[21]) return;
    {
        const int ndom = min(info[16] / 16, ndom_cap);
        const size_t n2 = ndom > nd0 ? (size_t)(ndom - nd0) * (2304 / 2) : 0;
        double2* coarse = reinterpret_cast<double2*>(dom + (size_t)nd0 * 2304);
        for (size_t e = t; e < n2; e += (size_t)gridDim.x * blockDim.x) coarse[e] = make_double2(0.0, 0.0);
    }
    if (t >= nd0 * 256) return;
    const int d = t >> 8, a = (t >> 4) & 15, b = t & 15;
    const int m = map0[t];
    double B[9];
#pragma unroll
    for (int q = 0; q < 9; q++) B[q] = 0.0;
    if (m > 0) {
#pragma unroll
        for (int q = 0; q < 9; q++) B[q] = val[9 * (size_t)(m - 1) + q];
    } else if (m < 0) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) B[3 * i + j] = val[9 * (size_t)(-m - 1) + 3 * j + i];
    }
    double* D = dom + (size_t)d * 2304 + (3 * a) * 48 + 3 * b;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) D[i * 48 + j] = B[3 * i + j];
}

__global__ void k_scatter_contact(int cap, const int* __restrict__ nuc, const int* __restrict__ ur,
                                  const int* __restrict__ uc, const double* __restrict__ val,
                                  const int* __restrict__ table, int L, const int* __restrict__ info,
                                  double* __restrict__ dom) {
    __shared__ double s_top[kTopLevels][2304];
    const int l_top = top_levels_dev(info, L);
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x * blockDim.x >= nuc[0]) return;  // whole block beyond the unique blocks
    const int ntop = L - l_top;
    zero_top(ntop, s_top);
    bool valid = u < cap && u < nuc[0];
    double B[9];
#pragma unroll
    for (int q = 0; q < 9; q++) B[q] = valid ? val[9 * (size_t)u + q] : 0.0;
    scatter_block_warp(dom, table, L, valid ? ur[u] : 0, valid ? uc[u] : 0, B, valid, 0, l_top, s_top);
    flush_top(info, l_top, ntop, s_top, dom);
}

// Gauss-Jordan inversion without pivoting, in place, one 48x48 domain per 64-thread CTA.
// Thread 8 r + c holds the 6 x 6 tile of rows 6r.., columns 6c.. in registers.  For pivot k
// with p = A(k,k):  A(i,j) -= A(i,k) A(k,j) / p  (i, j != k);  A(k,j) = A(k,j) / p;
// A(i,k) = -A(i,k) / p;  A(k,k) = 1 / p.  The owners publish row k and column k to shared
// memory (double-buffered: one barrier per step), and the pivot loop is unrolled by 6 so that
// row k's and column k's offsets inside a tile are compile-time constants.  Six domains per
// SM (three warps per scheduler, up to 170 registers, no spills) measured faster than one warp
// per domain or eight two-warp domains per SM (128 registers, spilling).
__global__ void __launch_bounds__(64, 6) k_invert(int ndom, double* __restrict__ dom, float* __restrict__ dom32,
                                                  int write64, int write32) {
    __shared__ __align__(16) double srow[2][48], scol[2][48];
    const int d = blockIdx.x;
    if (d >= ndom) return;
    const int r = threadIdx.x >> 3, c = threadIdx.x & 7;
    const int i0 = 6 * r, j0 = 6 * c;
    const double* D = dom + (size_t)d * 2304;
    double t[6][6];
#pragma unroll
    for (int a = 0; a < 6; a++)
#pragma unroll
        for (int b = 0; b < 6; b += 2) {
            const double2 v = *reinterpret_cast<const double2*>(D + (i0 + a) * 48 + j0 + b);
            // a zero diagonal (padding node) becomes 1
            t[a][b] = (i0 + a == j0 + b && v.x == 0.0) ? 1.0 : v.x;
            t[a][b + 1] = (i0 + a == j0 + b + 1 && v.y == 0.0) ? 1.0 : v.y;
        }
#pragma unroll 1
    for (int kk = 0; kk < 8; kk++) {  // pivots 6 kk .. 6 kk + 5: row group and column group kk
#pragma unroll
        for (int j = 0; j < 6; j++) {
            const int q = j & 1;
            if (r == kk)  // row k = 6 kk + j as it is before this step
#pragma unroll
                for (int b = 0; b < 6; b += 2)
                    *reinterpret_cast<double2*>(&srow[q][j0 + b]) = make_double2(t[j][b], t[j][b + 1]);
            if (c == kk)  // column k
#pragma unroll
                for (int a = 0; a < 6; a += 2)
                    *reinterpret_cast<double2*>(&scol[q][i0 + a]) = make_double2(t[a][j], t[a + 1][j]);
            __syncthreads();
            double rk[6], ck[6];
#pragma unroll
            for (int b = 0; b < 6; b += 2) {
                const double2 v = *reinterpret_cast<const double2*>(&srow[q][j0 + b]);
                rk[b] = v.x;
                rk[b + 1] = v.y;
            }
#pragma unroll
            for (int a = 0; a < 6; a += 2) {
                const double2 v = *reinterpret_cast<const double2*>(&scol[q][i0 + a]);
                ck[a] = v.x;
                ck[a + 1] = v.y;
            }
            const double ip = 1.0 / srow[q][6 * kk + j];
#pragma unroll
            for (int b = 0; b < 6; b++) rk[b] *= ip;
#pragma unroll
            for (int a = 0; a < 6; a++)
#pragma unroll
                for (int b = 0; b < 6; b++) t[a][b] -= ck[a] * rk[b];
            if (r == kk)  // the pivot row is set instead of updated
#pragma unroll
                for (int b = 0; b < 6; b++) t[j][b] = rk[b];
            if (c == kk)  // and so is the pivot column
#pragma unroll
                for (int a = 0; a < 6; a++) t[a][j] = (r == kk && a == j) ? ip : -ck[a] * ip;
        }
    }
    double* Dw = dom + (size_t)d * 2304;
    float* Dw32 = dom32 + (size_t)d * 2304;
#pragma unroll
    for (int a = 0; a < 6; a++)
#pragma unroll
        for (int b = 0; b < 6; b += 2) {
            const int o = (i0 + a) * 48 + j0 + b;
            if (write64) *reinterpret_cast<double2*>(Dw + o) = make_double2(t[a][b], t[a][b + 1]);
            if (write32) *reinterpret_cast<float2*>(Dw32 + o) = make_float2((float)t[a][b], (float)t[a][b + 1]);
        }
}

}  // namespace

// ------------------------------------------------------------------------------------------
// apply kernels (also used by the fused PCG kernels through the templates below)
// ------------------------------------------------------------------------------------------
namespace sgipc {

// level 0 and level 1 of the restriction: one thread per position
template <class T, class M>
__global__ void k_restrict01(int npos, const T* __restrict__ r, const int* __restrict__ part_map,
                             const int* __restrict__ up, M* __restrict__ R) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    int v = p < npos ? part_map[p] : -1;
    M val[3] = {0, 0, 0};
    if (v >= 0) {
        val[0] = (M)r[3 * v];
        val[1] = (M)r[3 * v + 1];
        val[2] = (M)r[3 * v + 2];
    }
    if (p < npos) {
        R[3 * p] = val[0];
        R[3 * p + 1] = val[1];
        R[3 * p + 2] = val[2];
    }
    bank_reduce_store<M, 1>(v >= 0 ? up[p] : -1, val, R);
}

template <class M>
__global__ void __launch_bounds__(1024) k_restrict_coarse(const int* __restrict__ info, const int* __restrict__ up,
                                                          int L, M* __restrict__ R) {
    restrict_coarse_cta<M, 1>(info, up, L, R);
}

// Z_d = A_d^-1 R_d, four domains per 192-thread CTA
template <class M>
__global__ void __launch_bounds__(192) k_domain_mv(const int* __restrict__ info, const M* __restrict__ inv,
                                                   const M* __restrict__ R, M* __restrict__ Z) {
    __shared__ M sR[4][48];
    const int ndom = info[16] >> 4;
    const int ld = threadIdx.x / 48, i = threadIdx.x % 48;
    const int d = blockIdx.x * 4 + ld;
    if (d < ndom) sR[ld][i] = R[48 * (size_t)d + i];
    __syncthreads();
    if (d >= ndom) return;
    const M* Ad = inv + (size_t)d * 2304;
    M acc = 0;
#pragma unroll 8
    for (int j = 0; j < 48; j++) acc += Ad[j * 48 + i] * sR[ld][j];
    Z[48 * (size_t)d + i] = acc;
}

template <class T, class M>
__global__ void k_prolong(int nv, const int* __restrict__ table, int L, const M* __restrict__ Z, T* __restrict__ z) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const int* tv = table + (size_t)v * L;
    M x = 0, y = 0, w = 0;
    for (int l = 0; l < L; l++) {
        int g = tv[l];
        x += Z[3 * g];
        y += Z[3 * g + 1];
        w += Z[3 * g + 2];
    }
    z[3 * v] = (T)x;
    z[3 * v + 1] = (T)y;
    z[3 * v + 2] = (T)w;
}

template <class T>
SgipcStatus mas_apply_t(SgipcCtx* c, const T* r, T* z, int fp32_inv, cudaStream_t s) {
    MasWork& m = c->mas;
    if (!m.built) return SGIPC_NOT_READY;
    const int L = m.levelnum;
    const int ndom = m.h_info[16] / 16;
    SG_COUNT(c, 4);
    if (fp32_inv) {
        k_restrict01<T, float><<<nblk(m.npos), SGIPC_BLOCK, 0, s>>>(m.npos, r, m.part_map, m.up, m.R32);
        k_restrict_coarse<float><<<1, 1024, 0, s>>>(m.info, m.up, L, m.R32);
        k_domain_mv<float><<<(ndom + 3) / 4, 192, 0, s>>>(m.info, m.dom32, m.R32, m.Z32);
        k_prolong<T, float><<<nblk(c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, m.table, L, m.Z32, z);
    } else {
        k_restrict01<T, double><<<nblk(m.npos), SGIPC_BLOCK, 0, s>>>(m.npos, r, m.part_map, m.up, m.R64);
        k_restrict_coarse<double><<<1, 1024, 0, s>>>(m.info, m.up, L, m.R64);
        k_domain_mv<double><<<(ndom + 3) / 4, 192, 0, s>>>(m.info, m.dom64, m.R64, m.Z64);
        k_prolong<T, double><<<nblk(c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, m.table, L, m.Z64, z);
    }
    SG_LAUNCH_CHECK(c, "mas apply");
    return SGIPC_OK;
}

template SgipcStatus mas_apply_t<double>(SgipcCtx*, const double*, double*, int, cudaStream_t);
template SgipcStatus mas_apply_t<float>(SgipcCtx*, const float*, float*, int, cudaStream_t);

// First of the coarsest levels (at most kTopLevels, each with <= 16 nodes, i.e. one domain
// starting at a multiple of 16) that the scatter accumulates per CTA; L when none.
static int num_levels(int nodes) {
    int nLevel = 1;
    int levelSz = (nodes + 15) / 16 * 16;
    while (levelSz > 16) {
        levelSz /= 16;
        nLevel++;
        levelSz = (levelSz + 15) / 16 * 16;
    }
    nLevel = nLevel + 1;
    return nLevel > SGIPC_MAX_LEVELS ? SGIPC_MAX_LEVELS : nLevel;
}

// ---- the whole hierarchy as one cooperative launch -------------------------------------------
// The phases of the per-level kernels below (level-0 init; per level: mask reset, edge and
// pair masks, bank components, the exclusive scan of the component counts, assignment;
// then the level-1 bank ranges) separated by grid barriers: one launch instead of about
// thirty runtime calls, which matters because the hierarchy is enqueued beside the
// assembly and the host's enqueue time is on the critical path.  Barrier words live in
// info[20] (arrivals) and info[21] (abort, set when a wait exceeds its limit).
constexpr int kHierThreads = 256;
constexpr int kHierMaxCtas = 296;      // the largest grid the build may take (hier_part size)
// its grid beside the assembly (SGIPC_HIER_CTAS overrides): measured on the two-cube bench step,
// the MAS build ends at 0.41 ms with 32 CTAs, 0.36 ms with 74 and 0.41 ms with 148 (the
// assembly's kernels then lose their SMs)
constexpr int kHierDefaultCtas = 74;
constexpr long long kHierSpinLimit = 1LL << 24;

struct HierArgs {
    int nv, npos, L, nnbr, npairs;
    const int* real_map;
    const int* part_map;
    const int* nbr_row;
    const int* nbr;
    const int4* pairs;
    int* node;
    int* table;
    int* up;
    int* info;
    uint32_t* mask;
    int* rank;
    int* bank_cnt;
    int* bank_off;
    int* part;      // [gridDim.x] chunk totals of the scan (bank_off's tail beyond the banks)
    int* l1_first;
    int* l1_last;
    long long spin_limit;  // polls of a barrier wait before the build gives up
};

__device__ bool hier_barrier(int* info, unsigned int& epoch, long long limit) {
    __shared__ int s_ok;
    __syncthreads();
    epoch++;
    if (threadIdx.x == 0) {
        unsigned int* cnt = reinterpret_cast<unsigned int*>(info + 20);
        volatile unsigned int* abort = reinterpret_cast<volatile unsigned int*>(info + 21);
        // release add / acquire poll (the CTA barriers around them carry the order to the
        // CTA's other threads), as the persistent PCG's barrier: no separate fences
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(cnt), "r"(1u) : "memory");
        const unsigned int target = epoch * gridDim.x;
        int ok = 1;
        for (long long k = 0;; k++) {
            unsigned int seen;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(cnt) : "memory");
            if ((int)(seen - target) >= 0) break;
            if (*abort) {
                ok = 0;
                break;
            }
            if (k > limit) {
                atomicExch(reinterpret_cast<unsigned int*>(info + 21), 1u);
                ok = 0;
                break;
            }
            if (k > 64) __nanosleep(64);
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__global__ void __launch_bounds__(kHierThreads) k_hierarchy(HierArgs h) {
    typedef cub::BlockScan<int, kHierThreads> Scan;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ int s_carry;
    unsigned int epoch = 0;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const int gw = tid >> 5, nw = nth >> 5;  // global warp index / count
    int* info = h.info;
    // level 0: positions
    if (tid == 0) {
        info[0] = 0;
        info[8] = h.npos;
        if (h.L == 1) info[16] = h.npos;
    }
    for (int v = tid; v < max(h.nv, h.npos); v += nth) {
        if (v < h.npos) {
            h.up[v] = -1;     // padding positions have no parent
            h.mask[v] = 0u;   // level 0's connection masks start empty
        }
        if (v < h.nv) {
            const int p = h.real_map[v];
            h.node[v] = p;
            h.table[(size_t)v * h.L] = p;
        }
    }
    if (!hier_barrier(info, epoch, h.spin_limit)) return;
    for (int l = 0; l + 1 < h.L; l++) {
        const int count = info[8 + l], start = info[l];
        const int nbank = (count + 15) >> 4;
        // (the masks of this level were zeroed by the previous phase)
        // edge masks (one lane per neighbour slot) and contact-pair masks, warp-aggregated
        for (int k0 = gw * 32; k0 < h.nnbr; k0 += nw * 32) {
            const int k = k0 + lane;
            int a = -1;
            uint32_t bit = 0;
            if (k < h.nnbr) {
                a = h.node[h.nbr_row[k]];
                const int b = h.node[h.nbr[k]];
                if (a != b && (a >> 4) == (b >> 4)) bit = 1u << (b & 15);
            }
            mask_or_warp(h.mask, bit ? a : -1, bit);
        }
        for (int p0 = gw * 32; p0 < h.npairs; p0 += nw * 32)
            mask_pair_warp(p0 + lane < h.npairs ? h.pairs + p0 + lane : nullptr, h.nv, h.node, h.mask);
        if (!hier_barrier(info, epoch, h.spin_limit)) return;
        // components, half a warp per bank; bank nbank gets a zero count (the scan's total)
        for (int b0 = gw * 2; b0 <= nbank; b0 += nw * 2)
            bank_components_half(b0 + (lane >> 4), nbank, count, l, h.mask, h.part_map, h.rank, h.bank_cnt);
        if (!hier_barrier(info, epoch, h.spin_limit)) return;
        // exclusive scan of bank_cnt[0 .. nbank]: per CTA a chunk, then the chunk offsets
        const int n1 = nbank + 1, cs = (n1 + gridDim.x - 1) / gridDim.x;
        const int c0 = min(n1, (int)blockIdx.x * cs), c1 = min(n1, c0 + cs);
        if (threadIdx.x == 0) s_carry = 0;
        __syncthreads();
        for (int t0 = c0; t0 < c1; t0 += blockDim.x) {
            const int i = t0 + threadIdx.x;
            int x = i < c1 ? h.bank_cnt[i] : 0, y, agg;
            Scan(scan_tmp).ExclusiveSum(x, y, agg);
            const int carry = s_carry;
            if (i < c1) h.bank_off[i] = y + carry;
            __syncthreads();
            if (threadIdx.x == 0) s_carry = carry + agg;
            __syncthreads();
        }
        if (threadIdx.x == 0) h.part[blockIdx.x] = s_carry;
        if (!hier_barrier(info, epoch, h.spin_limit)) return;
        if (threadIdx.x < 32) {
            int o = 0;
            for (int k = threadIdx.x; k < (int)blockIdx.x; k += 32) o += h.part[k];
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) o += __shfl_xor_sync(0xffffffffu, o, d);
            if (threadIdx.x == 0) s_carry = o;
        }
        __syncthreads();
        for (int i = c0 + threadIdx.x; i < c1; i += blockDim.x) h.bank_off[i] += s_carry;
        if (!hier_barrier(info, epoch, h.spin_limit)) return;
        // assignment of the next level's ids
        const int start_next = start + ((count + 15) & ~15);
        if (tid == 0) {
            info[l + 1] = start_next;
            info[8 + l + 1] = h.bank_off[nbank];
            if (l + 2 == h.L) info[16] = start_next + ((h.bank_off[nbank] + 15) & ~15);
        }
        for (int v = tid; v < h.nv; v += nth) {
            const int a = h.node[v];
            const int nn = h.bank_off[a >> 4] + h.rank[a];
            h.node[v] = nn;
            h.table[(size_t)v * h.L + l + 1] = start_next + nn;
            h.up[start + a] = start_next + nn;  // every vertex of node a writes the same parent
            if (l + 2 == h.L) h.up[start_next + nn] = -1;
        }
        // the next level's masks start empty (nothing reads the masks in this phase)
        if (l + 2 < h.L)
            for (int k = tid; k < h.bank_off[nbank]; k += nth) h.mask[k] = 0u;
        if (!hier_barrier(info, epoch, h.spin_limit)) return;
    }
    if (h.L >= 3) {
        const int nb0 = h.npos >> 4;
        for (int k = tid; k < nb0 + 2; k += nth) {
            h.l1_first[k] = 0x7f7f7f7f;
            h.l1_last[k] = -1;
        }
        if (!hier_barrier(info, epoch, h.spin_limit)) return;
        const int start1 = info[1];
        for (int b = tid; b < nb0; b += nth) {
            int lo = 0x7fffffff, hi = -1;
            for (int k = 0; k < 16; k++) {
                const int g = h.up[16 * b + k];
                if (g < 0) continue;
                lo = min(lo, (g - start1) >> 4);
                hi = max(hi, (g - start1) >> 4);
            }
            for (int m = lo; m <= hi; m++) {
                atomicMin(h.l1_first + m, b);
                atomicMax(h.l1_last + m, b);
            }
        }
    }
}

// For each level-1 bank m (nodes 16 m .. 16 m + 15): the first and last level-0 bank whose
// positions have a parent in it.  Level-1 ids grow with the level-0 bank (components are
// numbered bank by bank), so the banks in between feed m as well.
// One thread per level-0 bank: its components span at most two level-1 banks.
__global__ void k_l1_ranges(int npos, const int* __restrict__ up, const int* __restrict__ info,
                            int* __restrict__ first, int* __restrict__ last) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= (npos >> 4)) return;
    const int start1 = info[1];
    int lo = 0x7fffffff, hi = -1;
    for (int k = 0; k < 16; k++) {
        const int g = up[16 * b + k];
        if (g < 0) continue;
        lo = min(lo, (g - start1) >> 4);
        hi = max(hi, (g - start1) >> 4);
    }
    for (int m = lo; m <= hi; m++) {
        atomicMin(first + m, b);
        atomicMax(last + m, b);
    }
}

SgipcStatus mas_create(SgipcCtx* c, const SgipcTopology* t) {
    MasWork& m = c->mas;
    m.npos = t->part_map_size;
    m.levelnum = num_levels(m.npos > c->nv ? m.npos : c->nv);
    m.total_cap = m.levelnum * m.npos;
    const int nv = c->nv;
    std::vector<int> pm(t->partId_map_real, t->partId_map_real + m.npos);
    std::vector<int> rm(t->real_map_partId, t->real_map_partId + nv);
    for (int i = 0; i < m.npos; i++)
        if (pm[i] >= nv) return SGIPC_BAD_INPUT;
    for (int v = 0; v < nv; v++)
        if (rm[v] < 0 || rm[v] >= m.npos || pm[rm[v]] != v) return SGIPC_BAD_INPUT;
    std::vector<int> ptr(nv + 1), nb(t->neighborStart[nv]), nrow(t->neighborStart[nv]);
    for (int i = 0; i <= nv; i++) ptr[i] = (int)t->neighborStart[i];
    for (size_t k = 0; k < nb.size(); k++) {
        nb[k] = (int)t->neighborList[k];
        if (nb[k] < 0 || nb[k] >= nv) return SGIPC_BAD_INPUT;
    }
    for (int v = 0; v < nv; v++)
        for (int k = ptr[v]; k < ptr[v + 1]; k++) nrow[k] = v;
    m.nnbr = (int)nb.size();
    const size_t ndom_cap = (size_t)m.total_cap / 16;
    const size_t rhs = (size_t)c->max_rhs;
    auto A = [&](void** p, size_t bytes) -> bool { return cudaMalloc(p, bytes ? bytes : 4) == cudaSuccess; };
    if (!A((void**)&m.part_map, sizeof(int) * m.npos) || !A((void**)&m.real_map, sizeof(int) * nv) ||
        !A((void**)&m.nbr_ptr, sizeof(int) * (nv + 1)) || !A((void**)&m.nbr, sizeof(int) * nb.size()) ||
        !A((void**)&m.nbr_row, sizeof(int) * nb.size()) ||
        !A((void**)&m.table, sizeof(int) * (size_t)nv * m.levelnum) || !A((void**)&m.node, sizeof(int) * nv) ||
        !A((void**)&m.up, sizeof(int) * (size_t)m.total_cap) ||
        !A((void**)&m.mask, sizeof(uint32_t) * m.npos) || !A((void**)&m.comp_rank, sizeof(int) * m.npos) ||
        !A((void**)&m.bank_cnt, sizeof(int) * (m.npos / 16 + 2)) ||
        !A((void**)&m.bank_off, sizeof(int) * (m.npos / 16 + 2)) || !A((void**)&m.info, sizeof(int) * 32) ||
        !A((void**)&m.map0, sizeof(int) * (size_t)(m.npos / 16) * 256) ||
        !A((void**)&m.l1_first, sizeof(int) * (m.npos / 16 + 2)) ||
        !A((void**)&m.l1_last, sizeof(int) * (m.npos / 16 + 2)) ||
        !A((void**)&m.dom64, sizeof(double) * ndom_cap * 2304) || !A((void**)&m.dom32, sizeof(float) * ndom_cap * 2304) ||
        !A((void**)&m.R64, sizeof(double) * 3 * m.total_cap * rhs) ||
        !A((void**)&m.Z64, sizeof(double) * 3 * m.total_cap * rhs) ||
        !A((void**)&m.R32, sizeof(float) * 3 * m.total_cap * rhs) ||
        !A((void**)&m.Z32, sizeof(float) * 3 * m.total_cap * rhs)) {
        snprintf(c->err, sizeof(c->err), "MAS workspace allocation failed");
        return SGIPC_CUDA_ERROR;
    }
    SG_CHECK(c, cudaMemcpy(m.part_map, pm.data(), sizeof(int) * m.npos, cudaMemcpyHostToDevice));
    SG_CHECK(c, cudaMemcpy(m.real_map, rm.data(), sizeof(int) * nv, cudaMemcpyHostToDevice));
    SG_CHECK(c, cudaMemcpy(m.nbr_ptr, ptr.data(), sizeof(int) * (nv + 1), cudaMemcpyHostToDevice));
    if (!nb.empty()) SG_CHECK(c, cudaMemcpy(m.nbr, nb.data(), sizeof(int) * nb.size(), cudaMemcpyHostToDevice));
    if (!nb.empty()) SG_CHECK(c, cudaMemcpy(m.nbr_row, nrow.data(), sizeof(int) * nb.size(), cudaMemcpyHostToDevice));
    {
        // static slot of every level-0 domain entry (the static pattern is on the device)
        std::vector<int> srow(c->nnz), scol(c->nnz), map0((size_t)(m.npos / 16) * 256, 0);
        if (c->nnz) {
            SG_CHECK(c, cudaMemcpy(srow.data(), c->slot_row, sizeof(int) * c->nnz, cudaMemcpyDeviceToHost));
            SG_CHECK(c, cudaMemcpy(scol.data(), c->col, sizeof(int) * c->nnz, cudaMemcpyDeviceToHost));
        }
        for (int k = 0; k < c->nnz; k++) {
            const int pa = rm[srow[k]], pb = rm[scol[k]];
            if ((pa >> 4) != (pb >> 4)) continue;
            const size_t d = (size_t)(pa >> 4) * 256;
            map0[d + (pa & 15) * 16 + (pb & 15)] = k + 1;
            if (pa != pb) map0[d + (pb & 15) * 16 + (pa & 15)] = -(k + 1);
        }
        SG_CHECK(c, cudaMemcpy(m.map0, map0.data(), sizeof(int) * map0.size(), cudaMemcpyHostToDevice));
    }
    SG_CHECK(c, cudaMemset(m.R64, 0, sizeof(double) * 3 * m.total_cap * rhs));
    SG_CHECK(c, cudaMemset(m.R32, 0, sizeof(float) * 3 * m.total_cap * rhs));
    SG_CHECK(c, cudaMemset(m.info, 0, sizeof(int) * 32));
    SG_CHECK(c, cudaStreamCreateWithFlags(&m.side, cudaStreamNonBlocking));
    SG_CHECK(c, cudaEventCreateWithFlags(&m.ev_start, cudaEventDisableTiming));
    SG_CHECK(c, cudaEventCreateWithFlags(&m.ev_hier, cudaEventDisableTiming));
    SG_CHECK(c, cudaEventCreateWithFlags(&m.ev_static, cudaEventDisableTiming));
    SG_CHECK(c, cudaEventCreateWithFlags(&m.ev_pre, cudaEventDisableTiming));
    SG_CHECK(c, cudaMallocHost((void**)&m.h_info_pinned, sizeof(int) * 32));
    SG_CHECK(c, cudaMalloc((void**)&m.hier_part, sizeof(int) * kHierMaxCtas));
    {
        int coop = 0, nsm = 0, per = 0;
        SG_CHECK(c, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device));
        SG_CHECK(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
        SG_CHECK(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_hierarchy, kHierThreads, 0));
        // the build runs beside the assembly's kernels: a small grid leaves them the SMs
        int want = kHierDefaultCtas;
        const char* e = getenv("SGIPC_HIER_CTAS");
        if (e && atoi(e) > 0) want = atoi(e) < kHierMaxCtas ? atoi(e) : kHierMaxCtas;
        m.hier_grid = coop && per > 0 ? (nsm * per < want ? nsm * per : want) : 0;
    }
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, m.bank_cnt, m.bank_off, m.npos / 16 + 2);
    m.scan_tmp_bytes = tb + 256;
    SG_CHECK(c, cudaMalloc(&m.scan_tmp, m.scan_tmp_bytes));
    return SGIPC_OK;
}

void mas_destroy(SgipcCtx* c) {
    MasWork& m = c->mas;
    if (m.side) {
        cudaStreamSynchronize(m.side);  // a prebuild may still read the caller's pairs
        cudaStreamDestroy(m.side);
    }
    if (m.ev_start) cudaEventDestroy(m.ev_start);
    if (m.ev_hier) cudaEventDestroy(m.ev_hier);
    if (m.ev_static) cudaEventDestroy(m.ev_static);
    if (m.ev_pre) cudaEventDestroy(m.ev_pre);
    if (m.h_info_pinned) cudaFreeHost(m.h_info_pinned);
    if (m.hier_part) cudaFree(m.hier_part);
    void* ptrs[] = {m.part_map, m.real_map, m.nbr_ptr, m.nbr, m.nbr_row, m.table, m.up, m.node, m.mask, m.comp_rank, m.bank_cnt,
                    m.bank_off, m.map0, m.l1_first, m.l1_last, m.info, m.dom64, m.dom32, m.R64, m.Z64, m.R32, m.Z32,
                    m.scan_tmp};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

// The hierarchy (levels, cluster tables, parents, level-1 bank ranges) for these contacts
// on stream s; the level counts land in the pinned buffer (read after s reaches them).
static SgipcStatus mas_hierarchy(SgipcCtx* c, const SgipcContacts* con, cudaStream_t s) {
    MasWork& m = c->mas;
    const int nv = c->nv, L = m.levelnum;
    const int nbank_cap = m.npos / 16 + 1;
    if (m.hier_grid > 0) {  // one cooperative launch
        HierArgs h;
        h.nv = nv;
        h.npos = m.npos;
        h.L = L;
        h.nnbr = m.nnbr;
        h.npairs = con && con->pair_num > 0 ? con->pair_num : 0;
        h.real_map = m.real_map;
        h.part_map = m.part_map;
        h.nbr_row = m.nbr_row;
        h.nbr = m.nbr;
        h.pairs = h.npairs ? (const int4*)con->pairs : nullptr;
        h.node = m.node;
        h.table = m.table;
        h.up = m.up;
        h.info = m.info;
        h.mask = m.mask;
        h.rank = m.comp_rank;
        h.bank_cnt = m.bank_cnt;
        h.bank_off = m.bank_off;
        h.part = m.hier_part;
        h.l1_first = m.l1_first;
        h.l1_last = m.l1_last;
        h.spin_limit = c->wait_limit > 0 ? c->wait_limit : kHierSpinLimit;
        SG_CHECK(c, cudaMemsetAsync(m.info + 20, 0, 2 * sizeof(int), s));
        void* args[] = {&h};
        SG_COUNT(c, 1);
        SG_CHECK(c, cudaLaunchCooperativeKernel((const void*)k_hierarchy, dim3(m.hier_grid), dim3(kHierThreads), args,
                                                0, s));
        SG_CHECK(c, cudaMemcpyAsync(m.h_info_pinned, m.info, sizeof(int) * 22, cudaMemcpyDeviceToHost, s));
        return SGIPC_OK;
    }
    k_init_level0<<<nblk(nv > m.npos ? nv : m.npos), SGIPC_BLOCK, 0, s>>>(nv, m.real_map, L, m.node, m.table,
                                                                          m.info, m.npos, m.up);
    SG_COUNT(c, 1 + (L - 1) * (3 + (con && con->pair_num > 0)) + (L >= 3));
    for (int l = 0; l + 1 < L; l++) {
        SG_CHECK(c, cudaMemsetAsync(m.mask, 0, sizeof(uint32_t) * m.npos, s));
        if (m.nnbr > 0) k_mask_edges<<<nblk(m.nnbr), SGIPC_BLOCK, 0, s>>>(m.nnbr, m.nbr_row, m.nbr, m.node, m.mask);
        if (con && con->pair_num > 0)
            k_mask_pairs<<<nblk(con->pair_num), SGIPC_BLOCK, 0, s>>>(con->pair_num, (const int4*)con->pairs, nv,
                                                                     m.node, m.mask);
        k_bank_components<<<nblk(16LL * (nbank_cap + 1), 128), 128, 0, s>>>(nbank_cap, m.info, l, m.mask, m.part_map,
                                                                           m.comp_rank, m.bank_cnt);
        size_t tb = m.scan_tmp_bytes;
        SG_CHECK(c, cub::DeviceScan::ExclusiveSum(m.scan_tmp, tb, m.bank_cnt, m.bank_off, nbank_cap + 1, s));
        k_assign<<<nblk(nv), SGIPC_BLOCK, 0, s>>>(nv, L, l, m.bank_off, m.comp_rank, m.node, m.table, m.info, m.up);
    }
    if (L >= 3) {
        // level-0 bank range of every level-1 bank (the persistent solve restricts a level-1
        // bank to level 2 inside one CTA)
        SG_CHECK(c, cudaMemsetAsync(m.l1_first, 0x7f, sizeof(int) * (m.npos / 16 + 2), s));
        SG_CHECK(c, cudaMemsetAsync(m.l1_last, 0xff, sizeof(int) * (m.npos / 16 + 2), s));
        k_l1_ranges<<<nblk(m.npos / 16), SGIPC_BLOCK, 0, s>>>(m.npos, m.up, m.info, m.l1_first, m.l1_last);
    }
    SG_LAUNCH_CHECK(c, "mas hierarchy");
    SG_CHECK(c, cudaMemsetAsync(m.info + 21, 0, sizeof(int), s));
    SG_CHECK(c, cudaMemcpyAsync(m.h_info_pinned, m.info, sizeof(int) * 22, cudaMemcpyDeviceToHost, s));
    return SGIPC_OK;
}

static bool same_pairs(const MasWork& m, const SgipcContacts* con) {
    const void* p = con && con->pair_num > 0 ? (const void*)con->pairs : nullptr;
    const int n = con && con->pair_num > 0 ? con->pair_num : 0;
    return p == m.hier_pairs && n == m.hier_pair_num;
}

SgipcStatus mas_mark_start(SgipcCtx* c, cudaStream_t s) {
    SG_CHECK(c, cudaEventRecord(c->mas.ev_start, s));
    return SGIPC_OK;
}

SgipcStatus mas_prebuild(SgipcCtx* c, const SgipcContacts* con, cudaStream_t s) {
    MasWork& m = c->mas;
    (void)s;
    // the side stream rewrites the tables only after the work queued before the assembly
    // (a previous solve reads them)
    SG_CHECK(c, cudaStreamWaitEvent(m.side, m.ev_start, 0));
    SgipcStatus st = mas_hierarchy(c, con, m.side);
    if (st != SGIPC_OK) return st;
    SG_CHECK(c, cudaEventRecord(m.ev_hier, m.side));
    SG_CHECK(c, cudaEventRecord(m.ev_pre, m.side));  // the last work on `side` (moved by a prescatter)
    m.hier_pending = 1;
    m.hier_pairs = con && con->pair_num > 0 ? (const void*)con->pairs : nullptr;
    m.hier_pair_num = con && con->pair_num > 0 ? con->pair_num : 0;
    return SGIPC_OK;
}

SgipcStatus mas_prescatter(SgipcCtx* c, cudaStream_t s) {
    MasWork& m = c->mas;
    m.pre_scattered = 0;
    if (!m.hier_pending) return SGIPC_OK;
    const int nd0 = m.npos / 16;
    SG_CHECK(c, cudaEventRecord(m.ev_static, s));
    SG_CHECK(c, cudaStreamWaitEvent(m.side, m.ev_static, 0));
    SG_COUNT(c, 2);
    k_fill_level0<<<nblk(256LL * nd0), SGIPC_BLOCK, 0, m.side>>>(nd0, m.total_cap / 16, m.map0, c->val64, m.info,
                                                                 m.dom64);
    k_scatter_static<<<nblk(c->nnz), SGIPC_BLOCK, 0, m.side>>>(c->nnz, c->slot_row, c->col, c->val64, m.table,
                                                               m.levelnum, m.info, m.dom64);
    SG_LAUNCH_CHECK(c, "mas static scatter");
    SG_CHECK(c, cudaEventRecord(m.ev_pre, m.side));
    m.pre_scattered = 1;
    return SGIPC_OK;
}

SgipcStatus mas_build(SgipcCtx* c, const SgipcContacts* con, SgipcPrecision prec, cudaStream_t s) {
    MasWork& m = c->mas;
    if (!c->assembled) return SGIPC_NOT_READY;
    const int L = m.levelnum;
    const bool reuse = m.hier_pending && same_pairs(m, con);
    const bool pre = reuse && m.pre_scattered;
    if (m.hier_pending) {
        // the prebuilt hierarchy and static scatter (or, for other contacts or a stale scatter,
        // their end before this build rewrites them)
        SG_CHECK(c, cudaStreamWaitEvent(s, m.ev_pre, 0));
        SG_CHECK(c, cudaEventSynchronize(m.ev_hier));
    }
    if (!reuse) {
        SgipcStatus st = mas_hierarchy(c, con, s);
        if (st != SGIPC_OK) return st;
        SG_CHECK(c, cudaStreamSynchronize(s));
    }
    m.hier_pending = 0;
    m.pre_scattered = 0;
    if (m.h_info_pinned[21]) {
        snprintf(c->err, sizeof(c->err), "mas: a grid barrier of the hierarchy build exceeded its wait limit");
        return SGIPC_CUDA_ERROR;
    }
    memcpy(m.h_info, m.h_info_pinned, sizeof(int) * 17);
    const int total = m.h_info[16];
    if (total > m.total_cap || total <= 0) {
        snprintf(c->err, sizeof(c->err), "MAS cluster count %d exceeds capacity %d", total, m.total_cap);
        return SGIPC_CAPACITY;
    }
    const int ndom = total / 16, nd0 = m.npos / 16;
    // restricted vectors: entries outside the current levels' nodes must read as zero
    SG_CHECK(c, cudaMemsetAsync(m.R64, 0, sizeof(double) * 3 * (size_t)total * c->max_rhs, s));
    SG_CHECK(c, cudaMemsetAsync(m.R32, 0, sizeof(float) * 3 * (size_t)total * c->max_rhs, s));
    if (!pre) {
        // level 0 written whole and the coarser domains zeroed, then the static blocks added
        SG_COUNT(c, 2);
        k_fill_level0<<<nblk(256LL * nd0), SGIPC_BLOCK, 0, s>>>(nd0, m.total_cap / 16, m.map0, c->val64, m.info,
                                                                m.dom64);
        k_scatter_static<<<nblk(c->nnz), SGIPC_BLOCK, 0, s>>>(c->nnz, c->slot_row, c->col, c->val64, m.table, L,
                                                              m.info, m.dom64);
    }
    SG_COUNT(c, 2);
    k_scatter_contact<<<nblk(c->cap_cblk), SGIPC_BLOCK, 0, s>>>(c->cap_cblk, c->nuc, c->uc_row, c->uc_col, c->uc64,
                                                               m.table, L, m.info, m.dom64);
    const int w64 = prec == SGIPC_FP64 ? 1 : 0, w32 = prec == SGIPC_FP64 ? 0 : 1;
    k_invert<<<ndom, 64, 0, s>>>(ndom, m.dom64, m.dom32, w64, w32);
    SG_LAUNCH_CHECK(c, "mas matrices");
    m.built = (int)prec + 1;
    return SGIPC_OK;
}

}  // namespace sgipc

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------
extern "C" SgipcStatus sgipc_mas_build(SgipcCtx* c, const SgipcContacts* con, SgipcPrecision prec, void* stream) {
    if (!c) return SGIPC_BAD_INPUT;
    if (con && con->pair_num > 0 && !con->pairs) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    SgipcStatus st = mas_build(c, con, prec, (cudaStream_t)stream);
    if (st == SGIPC_OK) {
        c->mas_con = con ? *con : SgipcContacts{};
        c->mas_has_con = con != nullptr;
    }
    return st;
}

namespace sgipc {
SgipcStatus mas_time_hook(SgipcCtx* c, const char* name, cudaStream_t s, double* bytes) {
    MasWork& m = c->mas;
    if (strncmp(name, "mas_", 4)) return SGIPC_NOT_READY;
    if (!m.built) return SGIPC_NOT_READY;
    const int L = m.levelnum, total = m.h_info[16], ndom = total / 16;
    SG_COUNT(c, 1);
    if (!strcmp(name, "mas_scatter")) {  // static blocks: level-0 fill + coarser levels' scatter
        SG_COUNT(c, 1);
        k_fill_level0<<<nblk(256LL * (m.npos / 16)), SGIPC_BLOCK, 0, s>>>(m.npos / 16, m.total_cap / 16, m.map0,
                                                                         c->val64, m.info, m.dom64);
        k_scatter_static<<<nblk(c->nnz), SGIPC_BLOCK, 0, s>>>(c->nnz, c->slot_row, c->col, c->val64, m.table, L,
                                                               m.info, m.dom64);
        *bytes = (double)c->nnz * (72 + 8) + (double)c->nv * L * 4 + (double)ndom * 2304 * 8;
    } else if (!strcmp(name, "mas_invert")) {
        k_invert<<<ndom, 64, 0, s>>>(ndom, m.dom64, m.dom32, 1, 1);
        *bytes = (double)ndom * 2304 * (8 + 8 + 4);
    } else if (!strcmp(name, "mas_domain64") || !strcmp(name, "mas_domain32")) {
        const bool f32 = name[10] == '3';
        if (f32)
            k_domain_mv<float><<<(ndom + 3) / 4, 192, 0, s>>>(m.info, m.dom32, m.R32, m.Z32);
        else
            k_domain_mv<double><<<(ndom + 3) / 4, 192, 0, s>>>(m.info, m.dom64, m.R64, m.Z64);
        // algorithmic: packed symmetric domain inverse (136 3x3 blocks) + R in + Z out
        const double sm = f32 ? 4 : 8;
        *bytes = (double)ndom * (136 * 9 * sm + 2 * 48 * sm);
    } else {
        return SGIPC_NOT_READY;
    }
    SG_LAUNCH_CHECK(c, name);
    return SGIPC_OK;
}
}  // namespace sgipc

extern "C" SgipcStatus sgipc_mas_apply(SgipcCtx* c, const double* r, double* z, void* stream) {
    if (!c || !r || !z) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    return mas_apply_t<double>(c, r, z, c->mas.built == SGIPC_FP64 + 1 ? 0 : 1, (cudaStream_t)stream);
}

extern "C" SgipcStatus sgipc_mas_info(SgipcCtx* c, int32_t* levelnum, int32_t* level_counts, int32_t* total) {
    if (!c) return SGIPC_BAD_INPUT;
    if (!c->mas.built) return SGIPC_NOT_READY;
    if (levelnum) *levelnum = c->mas.levelnum;
    if (level_counts)
        for (int l = 0; l < c->mas.levelnum; l++) level_counts[l] = c->mas.h_info[8 + l];
    if (total) *total = c->mas.h_info[16];
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_mas_export_tables(SgipcCtx* c, int32_t* table) {
    if (!c || !table) return SGIPC_BAD_INPUT;
    if (!c->mas.built) return SGIPC_NOT_READY;
    SG_DEVICE(c);
    SG_CHECK(c, cudaDeviceSynchronize());
    SG_CHECK(c, cudaMemcpy(table, c->mas.table, sizeof(int) * (size_t)c->nv * c->mas.levelnum, cudaMemcpyDeviceToHost));
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_mas_export_domains(SgipcCtx* c, double* out) {
    if (!c || !out) return SGIPC_BAD_INPUT;
    if (!c->mas.built) return SGIPC_NOT_READY;
    SG_DEVICE(c);
    SG_CHECK(c, cudaDeviceSynchronize());
    const size_t n = (size_t)(c->mas.h_info[16] / 16) * 2304;
    if (c->mas.built == SGIPC_FP64 + 1) {
        SG_CHECK(c, cudaMemcpy(out, c->mas.dom64, n * sizeof(double), cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(n);
        SG_CHECK(c, cudaMemcpy(tmp.data(), c->mas.dom32, n * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < n; k++) out[k] = tmp[k];
    }
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_mas_restrict(SgipcCtx* c, const double* r, double* out) {
    if (!c || !r || !out) return SGIPC_BAD_INPUT;
    if (!c->mas.built) return SGIPC_NOT_READY;
    SG_DEVICE(c);
    MasWork& m = c->mas;
    SG_CHECK(c, cudaDeviceSynchronize());
    k_restrict01<double, double><<<nblk(m.npos), SGIPC_BLOCK>>>(m.npos, r, m.part_map, m.up, m.R64);
    k_restrict_coarse<double><<<1, 1024>>>(m.info, m.up, m.levelnum, m.R64);
    SG_COUNT(c, 2);
    SG_LAUNCH_CHECK(c, "mas restrict");
    SG_CHECK(c, cudaDeviceSynchronize());
    SG_CHECK(c, cudaMemcpy(out, m.R64, sizeof(double) * 3 * (size_t)m.h_info[16], cudaMemcpyDeviceToHost));
    return SGIPC_OK;
}

// ------------------------------------------------------------------------------------------
// MAS apply without any allocation
// ------------------------------------------------------------------------------------------
// Some hosts cannot let a call allocate device memory: a solver step running inside a
// plugin whose host owns every device allocation through its own pool (a cudaMalloc there
// would bypass the pool's accounting or fail under its memory cap), or a real-time loop in
// which an allocation's implicit device synchronisation would stall other streams.  For
// them sgipc_mas_apply_noalloc keeps the restricted residual R and the domain solutions Z
// of the apply in a fixed array compiled into this library instead of the context's own
// buffers.  The array exists once per device that loads the library and stays there until
// the process exits; every call on that device shares it.

// Largest hierarchy it serves, in clusters summed over all levels (padding included):
// R and Z, 3 values each per cluster, FP64 = 2 * 3 * 65536 * 8 B = 3 MiB per device.
#define SGIPC_NOALLOC_MAX_CLUSTERS 65536
static __device__ __align__(256) double g_mas_noalloc_scratch[2 * 3 * SGIPC_NOALLOC_MAX_CLUSTERS];

namespace {
// Device address of the array, looked up once per device.  In host code the array's name
// only stands for it and must never be handed to a kernel.
constexpr int kNoAllocMaxDevices = 64;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_mu;
}  // namespace

extern "C" SgipcStatus sgipc_mas_apply_noalloc(SgipcCtx* c, const double* r, double* z, void* stream) {
    if (!c || !r || !z) return SGIPC_BAD_INPUT;
    MasWork& m = c->mas;
    if (!m.built) return SGIPC_NOT_READY;
    const int total = m.h_info[16];
    if (total > SGIPC_NOALLOC_MAX_CLUSTERS) {
        snprintf(c->err, sizeof(c->err),
                 "mas_apply_noalloc: the hierarchy has %d clusters, the static scratch holds at most %d", total,
                 SGIPC_NOALLOC_MAX_CLUSTERS);
        return SGIPC_CAPACITY;
    }
    if (c->device < 0 || c->device >= kNoAllocMaxDevices) {
        snprintf(c->err, sizeof(c->err), "mas_apply_noalloc: device %d beyond the %d supported", c->device,
                 kNoAllocMaxDevices);
        return SGIPC_BAD_INPUT;
    }
    // the context's device is current until this call returns; the caller's is restored then
    SG_DEVICE(c);
    // set-up on the first call on this device (with the device current): resolve the
    // array's device address
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_addr[c->device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_mas_noalloc_scratch);
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaGetSymbolAddress(g_mas_noalloc_scratch)");
            g_noalloc_addr[c->device] = p;
        }
        base = g_noalloc_addr[c->device];
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int L = m.levelnum;
    const int ndom = total / 16;
    const size_t n3 = 3 * (size_t)total;
    // the restriction never writes the padding slots of levels >= 1, and the domain solve
    // reads them: R must start at zero (the last call left its own values there).  Z is
    // written in full by the domain solve.
    if (m.built == SGIPC_FP64 + 1) {
        double* R = (double*)base;
        double* Z = R + n3;
        SG_CHECK(c, cudaMemsetAsync(R, 0, n3 * sizeof(double), s));
        SG_COUNT(c, 4);
        k_restrict01<double, double><<<nblk(m.npos), SGIPC_BLOCK, 0, s>>>(m.npos, r, m.part_map, m.up, R);
        k_restrict_coarse<double><<<1, 1024, 0, s>>>(m.info, m.up, L, R);
        k_domain_mv<double><<<(ndom + 3) / 4, 192, 0, s>>>(m.info, m.dom64, R, Z);
        k_prolong<double, double><<<nblk(c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, m.table, L, Z, z);
    } else {
        float* R = (float*)base;
        float* Z = R + n3;
        SG_CHECK(c, cudaMemsetAsync(R, 0, n3 * sizeof(float), s));
        SG_COUNT(c, 4);
        k_restrict01<double, float><<<nblk(m.npos), SGIPC_BLOCK, 0, s>>>(m.npos, r, m.part_map, m.up, R);
        k_restrict_coarse<float><<<1, 1024, 0, s>>>(m.info, m.up, L, R);
        k_domain_mv<float><<<(ndom + 3) / 4, 192, 0, s>>>(m.info, m.dom32, R, Z);
        k_prolong<double, float><<<nblk(c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, m.table, L, Z, z);
    }
    SG_LAUNCH_CHECK(c, "mas apply noalloc");
    return SGIPC_OK;
}
