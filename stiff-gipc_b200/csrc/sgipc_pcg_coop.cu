// sgipc_pcg_coop.cu — the whole MAS-preconditioned CG solve as ONE persistent kernel.
//
// Same algorithm and stop rules as the graph of sgipc_pcg.cu (PCGSolver::pcg,
// StiffGIPC/linear_system/solver/pcg_solver.cu:174-267), but the iteration never leaves
// the GPU: a cooperative launch keeps every CTA resident, and the phases of an iteration
// are separated by grid barriers instead of kernel boundaries.  At the sizes of one Newton
// system (~20k block rows, ~25 MB of matrix, hierarchy and vectors, all L2-resident) an
// iteration is a handful of dependent L2 round trips, so the design minimises round trips
// per phase and barrier latency.  Per iteration, with three or more MAS levels:
//   spmv    p = z + beta p_old (ping-pong buffers), Ap = A p, p.Ap          -> barrier + sum
//   update  x += alpha p, r_new = r_old - alpha Ap (two residual buffers), r.r, restriction
//           to MAS levels 0, 1 and 2: CTAs aligned to level-1 banks (phase_positions_l2)
//                                                                         -> barrier + sum
//   mas     level-0..2 domain solves on all CTAs but the last, which restricts 2 -> 3 ->
//           ... and solves the few domains above                           -> barrier
//   prolong z = sum_l Z, r.z                                               -> barrier + sum
// With one or two levels the update restricts to levels 0/1 only and the MAS takes two
// phases (level 0/1 domains with the restriction 1 -> 2; then the coarser levels).  The
// mixed solve's FP32 instance ends with the refinement epilogue (x64 += x, the FP64
// residual, its r.z and r.r).  Shared memory holds each CTA's SpMV rows, their contact
// blocks and its first level-0/1 domain inverses for the whole solve.
// Barrier: one monotonic arrival counter (release add; acquire polling until it reaches
// epoch x grid).  Dot products: every CTA stores its partial before arriving; after the
// barrier every CTA adds all partials in the same fixed order, so all CTAs take identical
// decisions from identical numbers (partials are double-buffered by epoch parity).  Values
// written by one CTA and read by another inside the kernel are loaded through L2
// (ld.global.cg) or, after the barrier's acquire, through L1.  Waits are bounded:
// past the limit a CTA raises the abort word, every CTA leaves, and the solve reports
// SGIPC_CUDA_ERROR.
#include <cstdlib>

#include "sgipc_internal.cuh"
#include "sgipc_mas_dev.cuh"
#include "sgipc_pcg_dev.cuh"

namespace sgipc {

constexpr int kCoopThreads = 512;
constexpr int kDomPerCta = kCoopThreads / 48;  // 10 domains of 48 rows per round
constexpr int kCoopMaxCtasPerSm = 2;
constexpr long long kSpinLimit = 1LL << 25;    // polls (~50 ns each once sleeping): ~2 s

// dynamic shared memory of the persistent solve: [rp (rows + 1)] [columns] [block values]
// [domain inverses], each part 16-byte aligned
__host__ __device__ constexpr int coop_pad4(int n) { return (n + 3) & ~3; }
__host__ __device__ constexpr size_t coop_rows_bytes(int rows, int ecap, int tsize) {
    return ecap > 0 ? (size_t)(coop_pad4(rows + 1) + coop_pad4(ecap)) * 4 + (((size_t)9 * ecap * tsize + 15) & ~(size_t)15)
                    : 0;
}

// contact part: [ru (rows + 1)] [rl (rows + 1)] [columns] [block values]
__host__ __device__ constexpr size_t coop_contact_bytes(int rows, int kcap, int tsize) {
    return kcap > 0 ? (size_t)(2 * coop_pad4(rows + 1) + coop_pad4(kcap)) * 4 + (((size_t)9 * kcap * tsize + 15) & ~(size_t)15)
                    : 0;
}
constexpr int kContactSlots = 768;  // contact entries per CTA held in shared memory

// dst[k] = src[k] for k < n by the whole CTA, eight loads in flight per thread (a plain
// strided loop waits out one L2 round trip per element a thread copies)
template <class T>
__device__ __forceinline__ void smem_fill(T* dst, const T* __restrict__ src, int n) {
    constexpr int kU = 8;
    for (int k0 = threadIdx.x; k0 < n; k0 += kU * (int)blockDim.x) {
        T v[kU];
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const int k = k0 + u * (int)blockDim.x;
            if (k < n) v[u] = __ldg(src + k);
        }
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const int k = k0 + u * (int)blockDim.x;
            if (k < n) dst[k] = v[u];
        }
    }
}

struct GridBarrier {
    unsigned int* count;  // arrivals since launch (zeroed before the launch)
    unsigned int* abort;
    long long spin_limit;  // polls of one wait before the solve gives up
    // phase profile (nullptr: off): per CTA and barrier epoch e < stamp_epochs, the
    // %globaltimer values when the CTA arrives at barrier e and when it leaves it, at
    // stamps[(cta * stamp_epochs + e) * 2 + {0, 1}]; epoch 0 holds the kernel's start and
    // the end of its shared-memory loads
    unsigned long long* stamps;
    int stamp_epochs;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void stamp(const GridBarrier& br, unsigned int epoch, int which) {
    if (br.stamps && epoch < (unsigned int)br.stamp_epochs)
        br.stamps[((size_t)blockIdx.x * br.stamp_epochs + epoch) * 2 + which] = global_ns();
}

// the phase that ends at a barrier, recorded with the profile (after the stamps of all
// gridDim.x CTAs: stamps[gridDim.x * stamp_epochs * 2 + epoch])
enum PhaseTag : int {
    kPhInit = 1,       // r = b, x = 0, restriction
    kPhMas = 2,        // domain solves (levels 0..2, or 0..1)
    kPhMasCoarse = 3,  // domain solves of the coarser levels (one- and two-level-restriction mode)
    kPhProlong = 4,    // z = sum of the levels' Z, r.z
    kPhSpmv = 5,       // p = z + beta p, Ap, p.Ap
    kPhUpdate = 6,     // x, r, restriction, r.r
    kPhAcc64 = 7,      // refinement: x64 += x (no longer a phase of its own: kept for the tag numbering)
    kPhRes64 = 8,      // refinement: r64 = b64 - A x64
    kPhRestr64 = 9,    // refinement: restriction of r64
    kPhProlong64 = 10,  // refinement: r64 . M r64
    kPhFusedA = 11,     // fused: z at the columns, w = A z, r.z, z.w, z.Ap_old
    kPhFusedB = 12      // fused: p, Ap, x, r, restriction, own level-0/1 domains; r.r, p.Ap
};

__device__ __forceinline__ void tag_phase(const GridBarrier& br, unsigned int epoch, int tag) {
    if (br.stamps && blockIdx.x == 0 && epoch < (unsigned int)br.stamp_epochs)
        br.stamps[(size_t)gridDim.x * br.stamp_epochs * 2 + epoch] = (unsigned long long)tag;
}

template <class T, class M, int NR>
struct CoopArgs {
    Topo tp;
    MatView<T> A;
    MasView mv;
    const M* inv;
    M* R;
    M* Z;
    const double* b;
    T* x;
    T* r;
    T* r2;             // second residual buffer (level-1-aligned passes read the old one)
    T* z;
    T* p0;
    T* p1;
    T* Ap;
    PcgScalars* sc;
    double* partial;   // [2][stride][gridDim.x] (stride: NR values, three NR in the fused solve)
    GridBarrier br;
    int nv;
    int nd01;          // domains of levels 0 and 1
    int nd2;           // domains of levels 0..2
    int ndom;          // all domains
    int max_iter;
    int crit;
    double tol;
    // shared-memory residency (0 = off): static rows of the CTA's SpMV rows (up to ecap
    // blocks) and the first dcap of its level-0/1 domain inverses, loaded once per solve
    int ecap;
    int kcap;
    int dcap;
    // >= 3 levels: position passes aligned to level-1 banks restrict to level 2 in the CTA,
    // and one MAS phase solves levels 0..2 while one CTA takes the levels above
    int l2mode;
    const int* l1_first;
    const int* l1_last;
    // refinement epilogue (FP32 inner solve, one right-hand side; x64 == nullptr: none)
    int x64_assign;  // x64 = x instead of x64 += x (the first refinement)
    const int* input_flag;  // copied into the scalars at the end (one read-back for both)
    double* x64;
    const double* b64;
    double* r64;
    MatView<double> A64;
    // fused iteration (k_pcg_fused): w = A z, the second Ap buffer, and per CTA the sorted
    // distinct columns of its rows (cs_cols[cs_ptr[c] ..]), each static entry's slot among
    // them (cs_lcol, by full-pattern index) and each row's own slot (cs_dslot); ccap bounds
    // a CTA's count
    T* w;
    T* Ap2;
    const int* cs_ptr;
    const int* cs_cols;
    const int* cs_lcol;
    const int* cs_dslot;
    int ccap;
    int zextra;  // further z slots for the columns of resident contact entries outside the set
};

__device__ __forceinline__ void red_add_release_gpu(unsigned int* p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier number `epoch` (1, 2, ...).  All threads of every CTA call it.
__device__ bool grid_barrier(const GridBarrier& br, unsigned int epoch, int tag) {
    __shared__ int s_ok;
    __syncthreads();  // the CTA's writes of this phase precede thread 0's release
    if (threadIdx.x == 0) {
        const unsigned int target = epoch * gridDim.x;
        stamp(br, epoch, 0);
        tag_phase(br, epoch, tag);
        red_add_release_gpu(br.count, 1u);
        int ok = 1;
        for (long long k = 0;; k++) {
            if ((int)(ld_acquire_gpu(br.count) - target) >= 0) break;
            if ((k & 63) == 63 && *(volatile unsigned int*)br.abort) {
                ok = 0;
                break;
            }
            if (k > br.spin_limit) {
                atomicExch(br.abort, 1u);
                ok = 0;
                break;
            }
            if (k > 256) __nanosleep(32);
        }
        // No fence here: the acquire load that saw the count orders every later access of
        // this thread after the other CTAs' released writes, and the __syncthreads below
        // extends that order to the CTA's other threads (the memory model's causality
        // order is transitive through CTA barriers), so their ordinary loads, L1-cached
        // ones included, see those writes.  (A fence here measured 0.9 us per iteration.)
        stamp(br, epoch, 1);
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

constexpr int kReduceLoads = 10;  // partial loads per lane issued together: grids up to 320 CTAs

// Barrier + sum over CTAs: v[r] is this thread's contribution; on return out[r] holds the
// grid total in every thread.  The partial buffer of parity epoch & 1 is rewritten two
// barriers later at the earliest, after every CTA has read it.
// `stride` (>= NR) is the number of values per CTA that each parity half of the buffer holds
// (the same for every reduction of a kernel, so that the halves never overlap).
template <int NR, int S>
__device__ bool grid_reduce(const GridBarrier& br, unsigned int epoch, int tag, double (&v)[NR], double* partial,
                            double (&smem)[S], double (&out)[NR], int stride = NR) {
    static_assert(S >= NR * 32, "block_sum needs 32 doubles of shared memory per value");
    __shared__ double s_tot[NR];
    double* part = partial + (size_t)(epoch & 1) * stride * gridDim.x;
    block_sum<NR>(v, smem);
    if (threadIdx.x == 0)
#pragma unroll
        for (int r = 0; r < NR; r++) part[r * gridDim.x + blockIdx.x] = v[r];
    const bool ok = grid_barrier(br, epoch, tag);
    // warp r adds the partials of value r: lane l takes CTAs l, l + 32, ... in that order
    // (all its loads issued together, and all warps side by side: one L2 round trip), then a
    // fixed xor tree, so every CTA computes the same total
    static_assert(NR <= kCoopThreads / 32, "one warp per reduced value");
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w < NR) {
        const int G = gridDim.x;
        const double* pr = part + (size_t)w * G;
        double t[kReduceLoads];
#pragma unroll
        for (int j = 0; j < kReduceLoads; j++) {
            const int k = lane + 32 * j;
            t[j] = k < G ? __ldcg(pr + k) : 0.0;
        }
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < kReduceLoads; j++) acc += t[j];
        for (int k = lane + 32 * kReduceLoads; k < G; k += 32) acc += __ldcg(pr + k);  // grids beyond 320 CTAs
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) s_tot[w] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; r++) out[r] = s_tot[r];
    __syncthreads();  // s_tot is reused by the next call
    return ok;
}

// ---- phases ---------------------------------------------------------------------------------
// Loops over MAS positions and level-1 nodes are warp-mapped over the whole grid with
// warp-uniform bounds, so that every 16-lane bank is a half-warp of consecutive entries
// (bank_reduce_store needs all 32 lanes).
__device__ __forceinline__ int grid_warp() { return (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); }
__device__ __forceinline__ int grid_warps() { return (int)((gridDim.x * blockDim.x) >> 5); }
// The same warps numbered CTA-fastest: a phase with fewer warps of work than the grid holds
// (one warp per 32 MAS positions or vertices) spreads over every SM instead of filling the
// first CTAs
__device__ __forceinline__ int spread_warp() { return (int)((threadIdx.x >> 5) * gridDim.x + blockIdx.x); }

// R at MAS position p (level 0) from the per-(rhs, component) values val[r * 3 + q]
template <class M, int NR>
__device__ __forceinline__ void store_levels01(M* R, int p, const M (&val)[NR * 3]) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
        M o[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) o[r] = val[r * 3 + q];
        stn<M, NR>(R + (size_t)(3 * p + q) * NR, o);
    }
}

// r = b, x = 0, R (levels 0 and 1) = restriction of r, ||b||^2
template <class T, class M, int NR>
__device__ void phase_init(const CoopArgs<T, M, NR>& a, double (&bb)[NR]) {
    const MasView& mv = a.mv;
    const int lane = threadIdx.x & 31;
    for (int pb = spread_warp() * 32; pb < mv.npos; pb += grid_warps() * 32) {
        const int p = pb + lane;
        const int v = p < mv.npos ? mv.part_map[p] : -1;
        M val[NR * 3];
#pragma unroll
        for (int k = 0; k < NR * 3; k++) val[k] = 0;
        if (v >= 0) {
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const size_t k = (size_t)(3 * v + q) * NR;
                double bv[NR];
                ldn<false, double, NR>(a.b + k, bv);
                T tr[NR], tx[NR];
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    tr[r] = (T)bv[r];
                    tx[r] = 0;
                    val[r * 3 + q] = (M)tr[r];
                    bb[r] += bv[r] * bv[r];
                }
                stn<T, NR>(a.r + k, tr);
                stn<T, NR>(a.x + k, tx);
            }
        }
        if (p < mv.npos) store_levels01<M, NR>(a.R, p, val);
        bank_reduce_store<M, NR>(v >= 0 ? mv.up[p] : -1, val, a.R);
    }
}

// Z_d = A_d^-1 R_d: 48-thread slot `threadIdx.x / 48` of the CTA takes domain d0 + slot
// when it is below `hi`.  All loads of a row of the product are issued together.
template <class M, int NR>
__device__ __forceinline__ void solve_domains(const M* __restrict__ inv, const M* R, M* Z, int d0, int hi,
                                              M (*sR)[48 * NR], const M* cache = nullptr, int ncached = 0) {
    const int ld = threadIdx.x / 48, i = threadIdx.x % 48;
    const int d = d0 + ld;
    const bool act = ld < kDomPerCta && d < hi;
    if (act) {
        M t[NR];
        ldn<true, M, NR>(R + (48 * (size_t)d + i) * NR, t);
        stn<M, NR>(&sR[ld][i * NR], t);
    }
    __syncthreads();
    if (act) {
        const bool sm = ld < ncached;  // this slot's inverse is resident in shared memory
        const M* Ad = sm ? cache + (size_t)ld * 2304 : inv + (size_t)d * 2304;
        M acc[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) acc[r] = 0;
        constexpr int kU = sizeof(M) == 4 ? (NR == 1 ? 24 : 12) : (NR == 1 ? 12 : 6);  // loads in flight
#pragma unroll
        for (int j0 = 0; j0 < 48; j0 += kU) {
            M w[kU];
#pragma unroll
            for (int j = 0; j < kU; j++) w[j] = sm ? Ad[(j0 + j) * 48 + i] : __ldg(Ad + (j0 + j) * 48 + i);
#pragma unroll
            for (int j = 0; j < kU; j++) {
                M rj[NR];
                ldn<false, M, NR>(&sR[ld][(j0 + j) * NR], rj);
#pragma unroll
                for (int r = 0; r < NR; r++) acc[r] += w[j] * rj[r];
            }
        }
        stn<M, NR>(Z + (48 * (size_t)d + i) * NR, acc);
    }
    __syncthreads();
}

// domains [lo, hi) over CTAs first .. first+ncta-1 (block-uniform loop bounds)
// (the first round may read `ncached` inverses from `cache`)
template <class M, int NR>
__device__ __forceinline__ void solve_domain_range(const M* inv, const M* R, M* Z, int lo, int hi, int first,
                                                   int ncta, M (*sR)[48 * NR], const M* cache = nullptr,
                                                   int ncached = 0) {
    const int c = (int)blockIdx.x - first;
    if (c < 0 || c >= ncta) return;
    for (int d0 = lo + c * kDomPerCta; d0 < hi; d0 += ncta * kDomPerCta) {
        solve_domains<M, NR>(inv, R, Z, d0, hi, sR, cache, ncached);
        ncached = 0;
    }
}

// restriction level 1 -> 2, one half-warp per level-1 bank, taken by the LAST warps of the
// grid (the level-0/1 domain solves fill the first CTAs)
template <class M, int NR>
__device__ void restrict_level1(const MasView& mv, M* R) {
    const int count = mv.info[9], start = mv.info[1];
    const int lane = threadIdx.x & 31;
    for (int ab = (grid_warps() - 1 - grid_warp()) * 32; ab < count; ab += grid_warps() * 32) {
        const int aa = ab + lane;
        M v[NR * 3];
        int par = -1;
        if (aa < count) {
            const int g = start + aa;
            par = mv.up[g];
#pragma unroll
            for (int q = 0; q < 3; q++) {
                M t[NR];
                ldn<true, M, NR>(R + (size_t)(3 * g + q) * NR, t);
#pragma unroll
                for (int r = 0; r < NR; r++) v[r * 3 + q] = t[r];
            }
        } else {
#pragma unroll
            for (int k = 0; k < NR * 3; k++) v[k] = 0;
        }
        bank_reduce_store<M, NR>(par, v, R);
    }
}

// z = M^-1 r given R at levels 0 and 1: two phases and two barriers (one when L <= 2)
template <class T, class M, int NR>
__device__ bool phase_mas(const CoopArgs<T, M, NR>& a, M (*sR)[48 * NR], unsigned int& epoch, const M* dcache,
                          int ndc) {
    const int L = a.mv.L, G = gridDim.x;
    if (a.l2mode) {
        // levels 0..2 are complete: the grid solves their domains; with more levels the last
        // CTA restricts 2 -> 3 -> ... and solves the (few) domains above
        if (L > 3 && blockIdx.x == G - 1) {
            restrict_coarse_cta<M, NR, true>(a.mv.info, a.mv.up, L, a.R, 2);
            solve_domain_range<M, NR>(a.inv, a.R, a.Z, a.nd2, a.ndom, G - 1, 1, sR);
        } else {
            solve_domain_range<M, NR>(a.inv, a.R, a.Z, 0, a.nd2, 0, L > 3 ? G - 1 : G, sR, dcache, ndc);
        }
        return grid_barrier(a.br, ++epoch, kPhMas);
    }
    if (L > 2) restrict_level1<M, NR>(a.mv, a.R);
    solve_domain_range<M, NR>(a.inv, a.R, a.Z, 0, a.nd01, 0, G, sR, dcache, ndc);
    if (!grid_barrier(a.br, ++epoch, kPhMas)) return false;
    if (L <= 2) return true;
    if (blockIdx.x == 0) {
        restrict_coarse_cta<M, NR, true>(a.mv.info, a.mv.up, L, a.R, 2);
        solve_domain_range<M, NR>(a.inv, a.R, a.Z, a.nd2, a.ndom, 0, 1, sR);
    }
    if (G > 1)
        solve_domain_range<M, NR>(a.inv, a.R, a.Z, a.nd01, a.nd2, 1, G - 1, sR);
    else
        solve_domain_range<M, NR>(a.inv, a.R, a.Z, a.nd01, a.nd2, 0, 1, sR);
    return grid_barrier(a.br, ++epoch, kPhMasCoarse);
}

// z = sum over levels of Z at the vertex's clusters; r.z
template <class T, class M, int NR>
__device__ void phase_prolong(const CoopArgs<T, M, NR>& a, const T* rcur, const bool (&run)[NR], double (&rz)[NR]) {
    const MasView& mv = a.mv;
    for (int v = spread_warp() * 32 + (int)(threadIdx.x & 31); v < a.nv; v += gridDim.x * blockDim.x) {
        const int* tv = mv.table + (size_t)v * mv.L;
        int gl[SGIPC_MAX_LEVELS];
#pragma unroll
        for (int l = 0; l < SGIPC_MAX_LEVELS; l++) gl[l] = l < mv.L ? __ldg(tv + l) : -1;
        // every right-hand side is summed and stored (vector accesses); a stopped one's z
        // is never used, and only running ones add to r.z
        M sq[3][NR];
#pragma unroll
        for (int q = 0; q < 3; q++)
#pragma unroll
            for (int r = 0; r < NR; r++) sq[q][r] = 0;
#pragma unroll
        for (int l = 0; l < SGIPC_MAX_LEVELS; l++) {
            if (gl[l] < 0) continue;
#pragma unroll
            for (int q = 0; q < 3; q++) {
                M t[NR];
                ldn<false, M, NR>(a.Z + (size_t)(3 * gl[l] + q) * NR, t);  // coarse clusters are shared: L1 reuse
#pragma unroll
                for (int r = 0; r < NR; r++) sq[q][r] += t[r];
            }
        }
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const size_t k = (size_t)(3 * v + q) * NR;
            T zz[NR], rv[NR];
            ldn<true, T, NR>(rcur + k, rv);
#pragma unroll
            for (int r = 0; r < NR; r++) {
                zz[r] = (T)sq[q][r];
                if (run[r]) rz[r] += (double)rv[r] * (double)zz[r];
            }
            stn<T, NR>(a.z + k, zz);
        }
    }
}

// p = z + beta p_old (p = z on the first iteration), Ap = A p, p.Ap
// The static rows of this CTA's first SpMV pass, resident in shared memory: local row
// pointers rp[0..rows], column indices and block values of entries [rp[0], rp[rows]).
template <class T>
struct RowCache {
    const int* rp;
    const int* col;
    const T* val;
    int r0, r1;  // rows held (r0 == r1: none)
    // contact entries of the same rows (constant during a solve) when they fit: per row the
    // upper entries [ru[li], ru[li+1]) and the transposed ones [rl[li], rl[li+1]) of kcol/kval
    const int* ru;
    const int* rl;
    const int* kcol;
    const T* kval;
};

// row_mv with the static part read from shared memory; the (few) contact entries of the
// row come from global memory, their bounds loaded before the static work
template <class T, int NR, class Op>
__device__ __forceinline__ void row_mv_resident(const Topo& tp, const MatView<T>& A, const Op& x, int i, int g,
                                                const RowCache<T>& rc, T (&acc)[NR][3]) {
#pragma unroll
    for (int r = 0; r < NR; r++) acc[r][0] = acc[r][1] = acc[r][2] = 0;
    if (i < tp.n && rc.kcol) {
        // everything of the row in shared memory: one virtual list (static, contact,
        // transposed contact), only the gathers of x touch global memory
        const int li = i - rc.r0;
        const int s0 = rc.rp[li], ns = rc.rp[li + 1] - s0;
        const int u0 = rc.ru[li], nu = rc.ru[li + 1] - u0;
        const int l0 = rc.rl[li], nl = rc.rl[li + 1] - l0;
        const int len = ns + nu + nl;
        constexpr int kB = NR == 1 ? (sizeof(T) == 4 ? 4 : 2) : 1;
        for (int e0 = g; e0 < len; e0 += kB * kSpG) {
            int cj[kB];
            const T* bp[kB];
            T xb[kB][NR][3];
#pragma unroll
            for (int u = 0; u < kB; u++) {
                const int e = e0 + u * kSpG;
                cj[u] = -1;
                bp[u] = nullptr;
                if (e < ns) {
                    cj[u] = rc.col[s0 + e];
                    bp[u] = rc.val + 9 * (s0 + e);
                } else if (e < ns + nu) {
                    cj[u] = rc.kcol[u0 + e - ns];
                    bp[u] = rc.kval + 9 * (u0 + e - ns);
                } else if (e < len) {
                    cj[u] = rc.kcol[l0 + e - ns - nu];
                    bp[u] = rc.kval + 9 * (l0 + e - ns - nu);
                }
            }
#pragma unroll
            for (int u = 0; u < kB; u++)
                if (cj[u] >= 0) x.load(cj[u], xb[u]);
#pragma unroll
            for (int u = 0; u < kB; u++) {
                if (cj[u] < 0) continue;
                const T* bv = bp[u];
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const T x0 = xb[u][r][0], x1 = xb[u][r][1], x2 = xb[u][r][2];
                    acc[r][0] += bv[0] * x0 + bv[1] * x1 + bv[2] * x2;
                    acc[r][1] += bv[3] * x0 + bv[4] * x1 + bv[5] * x2;
                    acc[r][2] += bv[6] * x0 + bv[7] * x1 + bv[8] * x2;
                }
            }
        }
    } else if (i < tp.n) {
        const int u0 = tp.cu_ptr[i], u1 = tp.cu_ptr[i + 1];
        const int k0 = tp.cl_ptr[i], k1 = tp.cl_ptr[i + 1];
        const int li = i - rc.r0;
        const int s0 = rc.rp[li], s1 = rc.rp[li + 1];
        constexpr int kB = NR == 1 ? (sizeof(T) == 4 ? 4 : 2) : 1;
        for (int e0 = s0 + g; e0 < s1; e0 += kB * kSpG) {
            int cj[kB];
            T xb[kB][NR][3];
#pragma unroll
            for (int u = 0; u < kB; u++) {
                const int e = e0 + u * kSpG;
                cj[u] = e < s1 ? rc.col[e] : -1;
            }
#pragma unroll
            for (int u = 0; u < kB; u++)
                if (cj[u] >= 0) x.load(cj[u], xb[u]);
#pragma unroll
            for (int u = 0; u < kB; u++) {
                if (cj[u] < 0) continue;
                const T* bv = rc.val + 9 * (e0 + u * kSpG);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const T x0 = xb[u][r][0], x1 = xb[u][r][1], x2 = xb[u][r][2];
                    acc[r][0] += bv[0] * x0 + bv[1] * x1 + bv[2] * x2;
                    acc[r][1] += bv[3] * x0 + bv[4] * x1 + bv[5] * x2;
                    acc[r][2] += bv[6] * x0 + bv[7] * x1 + bv[8] * x2;
                }
            }
        }
        const int nu = u1 - u0, len = nu + (k1 - k0);
        for (int e = g; e < len; e += kSpG) {
            const bool up = e < nu;
            const int cj = up ? __ldg(tp.uc_col + u0 + e) : __ldg(tp.cl_col + k0 + (e - nu));
            const T* src = up ? A.uc + 9 * (size_t)(u0 + e) : A.cl + 9 * (size_t)(k0 + (e - nu));
            T bv[9], xb[NR][3];
#pragma unroll
            for (int q = 0; q < 9; q++) bv[q] = __ldg(src + q);
            x.load(cj, xb);
#pragma unroll
            for (int r = 0; r < NR; r++) {
                acc[r][0] += bv[0] * xb[r][0] + bv[1] * xb[r][1] + bv[2] * xb[r][2];
                acc[r][1] += bv[3] * xb[r][0] + bv[4] * xb[r][1] + bv[5] * xb[r][2];
                acc[r][2] += bv[6] * xb[r][0] + bv[7] * xb[r][1] + bv[8] * xb[r][2];
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

template <class T, class M, int NR>
__device__ void phase_spmv(const CoopArgs<T, M, NR>& a, bool first, const double (&beta)[NR], const T* pold, T* pnew,
                           const bool (&run)[NR], double (&pAp)[NR], const RowCache<T>& rc) {
    Operand<T, NR, false> op;  // L1-cached gathers: each x_j serves ~13 rows of the same CTA
    op.a = a.z;
    op.b = first ? nullptr : pold;
#pragma unroll
    for (int r = 0; r < NR; r++) op.beta[r] = (T)beta[r];
    constexpr int gpw = 32 / kSpG;  // rows per warp and pass
    const int lane = threadIdx.x & 31;
    const int n = a.tp.n;
    for (int i0 = grid_warp() * gpw; i0 < n; i0 += grid_warps() * gpw) {  // warp-uniform bound
        const int i = i0 + lane / kSpG, g = lane % kSpG;
        T pi[NR][3];
        if (i < n && g == 0) op.load(i, pi);  // issued before the row's gathers
        T acc[NR][3];
        if (i0 >= rc.r0 && i0 < rc.r1)  // warp-uniform: the warp's rows are resident
            row_mv_resident<T, NR>(a.tp, a.A, op, i, g, rc, acc);
        else
            row_mv<T, NR>(a.tp, a.A, op, i, g, acc);
        if (i < n && g == 0) {
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const size_t k = (size_t)(3 * i + q) * NR;
                T pv[NR], av[NR];
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    pv[r] = pi[r][q];
                    av[r] = acc[r][q];
                    if (run[r]) pAp[r] += (double)pi[r][q] * (double)acc[r][q];
                }
                stn<T, NR>(pnew + k, pv);
                stn<T, NR>(a.Ap + k, av);
            }
        }
    }
}

// x += alpha p, r -= alpha Ap, restriction of r to levels 0 and 1, r.r
template <class T, class M, int NR>
__device__ void phase_update(const CoopArgs<T, M, NR>& a, const double (&alpha)[NR], const T* p,
                             const bool (&run)[NR], double (&rr)[NR]) {
    const MasView& mv = a.mv;
    const int lane = threadIdx.x & 31;
    for (int pb = spread_warp() * 32; pb < mv.npos; pb += grid_warps() * 32) {
        const int pos = pb + lane;
        const int v = pos < mv.npos ? mv.part_map[pos] : -1;
        M val[NR * 3];
#pragma unroll
        for (int k = 0; k < NR * 3; k++) val[k] = 0;
        if (v >= 0) {
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const size_t k = (size_t)(3 * v + q) * NR;
                T xv[NR], pv[NR], rv[NR], av[NR];
                ldn<true, T, NR>(a.x + k, xv);
                ldn<true, T, NR>(p + k, pv);
                ldn<true, T, NR>(a.r + k, rv);
                ldn<true, T, NR>(a.Ap + k, av);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    // a stopped right-hand side keeps x and r (selected, not multiplied by 0,
                    // so that non-finite p of a broken-down one cannot leak in)
                    const T al = (T)alpha[r];
                    if (run[r]) {
                        xv[r] = xv[r] + al * pv[r];
                        rv[r] = rv[r] - al * av[r];
                        rr[r] += (double)rv[r] * (double)rv[r];
                    }
                    val[r * 3 + q] = run[r] ? (M)rv[r] : (M)0;
                }
                stn<T, NR>(a.x + k, xv);
                stn<T, NR>(a.r + k, rv);
            }
        }
        if (pos < mv.npos) store_levels01<M, NR>(a.R, pos, val);
        bank_reduce_store<M, NR>(v >= 0 ? mv.up[pos] : -1, val, a.R);
    }
}

// Position pass aligned to level-1 banks (l2mode), for the initial restriction (kInit:
// r = b, x = 0) and for the update (x += alpha p, r_new = r_old - alpha Ap).  CTA c takes
// level-1 banks m = c, c + G, ...; for each, the level-0 banks l1_first[m] .. l1_last[m]
// that feed it, two per warp.  A level-0 bank belongs to the level-1 bank of its first
// component: only there are x, r and its level-0 R written and r.r accumulated.  A bank
// whose components straddle two level-1 banks is recomputed by the second one from the
// old residual (identical arithmetic), so that every CTA holds its level-1 bank complete
// (level-1 sums: the same 16-lane groups and order as bank_reduce_store), keeps it in shared
// memory and restricts it to level 2 itself.
// kMode: 0 update, 1 init (r = b, x = 0), 2 restriction of the FP64 vector r_src only
template <class T, class M, int NR, int kMode>
__device__ void phase_positions_l2(const CoopArgs<T, M, NR>& a, const double (&alpha)[NR], const T* p,
                                   const T* r_old, T* r_new, const bool (&run)[NR], double (&acc)[NR],
                                   M (*s_l1)[3 * NR]) {
    const MasView& mv = a.mv;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int start1 = mv.info[1], count1 = mv.info[9];
    const int nb1 = (count1 + 15) >> 4;
    for (int m = blockIdx.x; m < nb1; m += gridDim.x) {  // block-uniform
        const int b_lo = __ldg(a.l1_first + m), b_hi = __ldg(a.l1_last + m);
        const int id_lo = 16 * m, id_hi = min(16 * m + 16, count1);
        for (int b0 = b_lo + 2 * w; b0 <= b_hi; b0 += 2 * (kCoopThreads / 32)) {  // warp-uniform
            const int bank = b0 + (lane >> 4);
            const int pos = bank * 16 + (lane & 15);
            const int v = bank <= b_hi ? __ldg(mv.part_map + pos) : -1;
            const int par = v >= 0 ? __ldg(mv.up + pos) - start1 : -1;  // local level-1 id
            int first = par >= 0 ? par : 0x7fffffff;  // the bank's first component
#pragma unroll
            for (int o = 1; o < 16; o <<= 1) first = min(first, __shfl_xor_sync(0xffffffffu, first, o, 16));
            const bool own = first >= id_lo;
            M val[NR * 3];
#pragma unroll
            for (int k = 0; k < NR * 3; k++) val[k] = 0;
            if (v >= 0) {
                T pq[3][NR];
                if (kMode == 0)
#pragma unroll
                    for (int q = 0; q < 3; q++) ldn<true, T, NR>(p + (size_t)(3 * v + q) * NR, pq[q]);
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const size_t k = (size_t)(3 * v + q) * NR;
                    T rv[NR];
                    if (kMode == 2) {
                        double sv[NR];
                        ldn<true, double, NR>(a.r64 + k, sv);
#pragma unroll
                        for (int r = 0; r < NR; r++) rv[r] = (T)sv[r];
                    } else if (kMode == 1) {
                        double bv[NR];
                        ldn<false, double, NR>(a.b + k, bv);
                        T tx[NR];
#pragma unroll
                        for (int r = 0; r < NR; r++) {
                            rv[r] = (T)bv[r];
                            tx[r] = 0;
                            if (own) acc[r] += bv[r] * bv[r];
                        }
                        if (own) {
                            stn<T, NR>(r_new + k, rv);
                            stn<T, NR>(a.x + k, tx);
                        }
                    } else {
                        T xv[NR], av[NR];
#pragma unroll
                        for (int r = 0; r < NR; r++) xv[r] = 0;
                        ldn<true, T, NR>(r_old + k, rv);
                        ldn<true, T, NR>(a.Ap + k, av);
                        if (own) ldn<true, T, NR>(a.x + k, xv);
#pragma unroll
                        for (int r = 0; r < NR; r++) {
                            const T al = (T)alpha[r];
                            if (run[r]) {
                                rv[r] = rv[r] - al * av[r];
                                xv[r] = xv[r] + al * pq[q][r];
                                if (own) acc[r] += (double)rv[r] * (double)rv[r];
                            }
                        }
                        if (own) {
                            stn<T, NR>(a.x + k, xv);
                            stn<T, NR>(r_new + k, rv);
                        }
                    }
#pragma unroll
                    for (int r = 0; r < NR; r++) val[r * 3 + q] = (kMode != 0 || run[r]) ? (M)rv[r] : (M)0;
                }
            }
            if (own && bank <= b_hi) store_levels01<M, NR>(a.R, pos, val);
            // level-1 sums of this bank's components inside [id_lo, id_hi)
            const int gp = (par >= id_lo && par < id_hi) ? par : -1;
            M sum[NR * 3];
            const bool lead = bank_group_sum<M, NR>(gp, val, sum);
            if (lead && gp >= 0) {
#pragma unroll
                for (int k = 0; k < NR * 3; k++) s_l1[gp - id_lo][k] = sum[k];
                store_levels01<M, NR>(a.R, start1 + gp, sum);
            }
        }
        __syncthreads();
        if (w == 0) {  // level 1 -> 2 for this bank (same groups and order as restrict_level1)
            const int a1 = id_lo + (lane & 15);
            const bool ok = lane < 16 && a1 < id_hi;
            M v1[NR * 3];
#pragma unroll
            for (int k = 0; k < NR * 3; k++) v1[k] = ok ? s_l1[lane & 15][k] : (M)0;
            bank_reduce_store<M, NR>(ok ? __ldg(mv.up + start1 + a1) : -1, v1, a.R);
        }
        __syncthreads();  // s_l1 is rewritten for the next bank
    }
}

// ---- fused iteration (three levels or more, every row resident) -----------------------------
// One iteration in three phases and three grid barriers instead of four:
//   A  z = M^-1 r prolonged at the columns of the CTA's rows (into shared memory), w = A z
//      from shared memory, and the dots r.z, z.w, z.Ap_old;
//   B  beta, alpha from those dots; p = z + beta p_old, Ap = w + beta Ap_old (A symmetric:
//      p.Ap = z.w + 2 beta z.Ap_old + beta^2 p_old.Ap_old), x += alpha p, r -= alpha Ap,
//      restriction to levels 0..2; r.r and p.Ap;
//   C  the MAS domain solves (levels 0..2 over the grid, the levels above on the last CTA).
// The prolongation needs no phase of its own, and the SpMV reads z from shared memory
// instead of gathering z and p_old.  p.Ap enters the recurrence from the previous iteration's
// direct dot.  (Solving each CTA's level-0/1 domains inside B, whose residuals are complete
// in the CTA, was measured slower: B grew by 6.7 us while C stayed bound by the last CTA's
// coarse chain.)
constexpr int kFusedMaxCols = 1024;  // distinct columns of one CTA's rows held in shared memory
// the column sets are built with the static pattern for CTAs of 128 rows (sgipc_ctx.cu)
static_assert(kCoopThreads / kSpG == 128, "fused column sets assume 128 rows per CTA");

// shared-memory part of the column set: [table rows (cols x SGIPC_MAX_LEVELS)] [z values]
__host__ __device__ constexpr size_t fused_cols_bytes(int ccap, int tsize, int nr) {
    return ccap > 0 ? (size_t)coop_pad4(ccap * SGIPC_MAX_LEVELS) * 4 + (((size_t)ccap * 3 * nr * tsize + 15) & ~(size_t)15)
                    : 0;
}

template <class T, int NR>
struct FusedCache {
    const int* tab;   // [nc][SGIPC_MAX_LEVELS] cluster of each column at each level
    T* zs;            // [nc][3][NR] z at the columns
    const int* dsl;   // [rows] slot of each row's own column
    int nc;           // the CTA's static columns (slots 0 .. nc-1)
    int nz;           // slots in use: nc + the contact columns outside the static set
};

// z at vertex j: the sum over levels of Z at j's clusters (the order of phase_prolong)
template <class T, class M, int NR>
__device__ __forceinline__ void prolong_at(const MasView& mv, const M* Z, int j, T (&xj)[NR][3]) {
    int gl[SGIPC_MAX_LEVELS];
#pragma unroll
    for (int l = 0; l < SGIPC_MAX_LEVELS; l++) gl[l] = l < mv.L ? __ldg(mv.table + (size_t)j * mv.L + l) : -1;
    M sq[3][NR];
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int r = 0; r < NR; r++) sq[q][r] = 0;
#pragma unroll
    for (int l = 0; l < SGIPC_MAX_LEVELS; l++) {
        if (gl[l] < 0) continue;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            M t[NR];
            ldn<false, M, NR>(Z + (size_t)(3 * gl[l] + q) * NR, t);
#pragma unroll
            for (int r = 0; r < NR; r++) sq[q][r] += t[r];
        }
    }
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
        for (int r = 0; r < NR; r++) xj[r][q] = (T)sq[q][r];
}

// phase A.  dots[r] += r.z, dots[NR + r] += z.w, dots[2 NR + r] += z.Ap_old (not on the first
// iteration); z and w of the CTA's rows go to a.z and a.w.
template <class T, class M, int NR>
__device__ void phase_fused_spmv(const CoopArgs<T, M, NR>& a, const RowCache<T>& rc, const FusedCache<T, NR>& fc,
                                 const T* rcur, const T* ap_old, bool first, const bool (&run)[NR],
                                 double (&dots)[3 * NR]) {
    const MasView& mv = a.mv;
    constexpr int gpw = 32 / kSpG;
    const int lane = threadIdx.x & 31, g = lane % kSpG;
    const int i = rc.r0 + (int)(threadIdx.x >> 5) * gpw + lane / kSpG;
    // r and Ap_old of the row, issued before the z gathers (they do not depend on them)
    T rpre[3][NR], apre[3][NR];
    if (i < rc.r1 && g == 0) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const size_t k = (size_t)(3 * i + q) * NR;
            ldn<true, T, NR>(rcur + k, rpre[q]);
            if (!first) ldn<true, T, NR>(ap_old + k, apre[q]);
        }
    }
    // z at the CTA's columns (their cluster tables are resident)
    for (int s = threadIdx.x; s < fc.nz; s += blockDim.x) {
        M sq[3][NR];
#pragma unroll
        for (int q = 0; q < 3; q++)
#pragma unroll
            for (int r = 0; r < NR; r++) sq[q][r] = 0;
#pragma unroll
        for (int l = 0; l < SGIPC_MAX_LEVELS; l++) {
            if (l >= mv.L) break;
            const int g = fc.tab[s * SGIPC_MAX_LEVELS + l];
#pragma unroll
            for (int q = 0; q < 3; q++) {
                M t[NR];
                ldn<false, M, NR>(a.Z + (size_t)(3 * g + q) * NR, t);
#pragma unroll
                for (int r = 0; r < NR; r++) sq[q][r] += t[r];
            }
        }
#pragma unroll
        for (int q = 0; q < 3; q++) {
            T zz[NR];
#pragma unroll
            for (int r = 0; r < NR; r++) zz[r] = (T)sq[q][r];
            stn<T, NR>(fc.zs + ((size_t)s * 3 + q) * NR, zz);
        }
    }
    __syncthreads();
    // w = A z over the CTA's rows: static entries from shared memory, contact entries from
    // their z slots (or prolonged at their columns)
    T acc[NR][3];
#pragma unroll
    for (int r = 0; r < NR; r++) acc[r][0] = acc[r][1] = acc[r][2] = 0;
    if (i < rc.r1) {
        const int li = i - rc.r0;
        const int s0 = rc.rp[li], s1 = rc.rp[li + 1];
        for (int e = s0 + g; e < s1; e += kSpG) {
            const T* bv = rc.val + 9 * e;
            const T* zp = fc.zs + (size_t)rc.col[e] * 3 * NR;
            T x3[3][NR];
#pragma unroll
            for (int q = 0; q < 3; q++) ldn<false, T, NR>(zp + q * NR, x3[q]);
#pragma unroll
            for (int r = 0; r < NR; r++) {
                acc[r][0] += bv[0] * x3[0][r] + bv[1] * x3[1][r] + bv[2] * x3[2][r];
                acc[r][1] += bv[3] * x3[0][r] + bv[4] * x3[1][r] + bv[5] * x3[2][r];
                acc[r][2] += bv[6] * x3[0][r] + bv[7] * x3[1][r] + bv[8] * x3[2][r];
            }
        }
        int u0, nu, l0, nl;
        const int* kc;
        const T* kv;
        if (rc.kcol) {
            u0 = rc.ru[li], nu = rc.ru[li + 1] - u0, l0 = rc.rl[li], nl = rc.rl[li + 1] - l0;
            kc = rc.kcol, kv = rc.kval;
        } else {
            u0 = a.tp.cu_ptr[i], nu = a.tp.cu_ptr[i + 1] - u0, l0 = a.tp.cl_ptr[i], nl = a.tp.cl_ptr[i + 1] - l0;
            kc = nullptr, kv = nullptr;
        }
        for (int e = g; e < nu + nl; e += kSpG) {
            const bool up = e < nu;
            int cj;
            const T* src;
            if (kc) {  // resident: a z slot (>= 0), or -(column + 1) beyond the slots
                const int k = up ? u0 + e : l0 + (e - nu);
                cj = kc[k];
                src = kv + 9 * (size_t)k;
            } else {
                cj = -1 - (up ? __ldg(a.tp.uc_col + u0 + e) : __ldg(a.tp.cl_col + l0 + (e - nu)));
                src = up ? a.A.uc + 9 * (size_t)(u0 + e) : a.A.cl + 9 * (size_t)(l0 + (e - nu));
            }
            T xb[NR][3];
            if (cj >= 0) {
                const T* zp = fc.zs + (size_t)cj * 3 * NR;
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    T t3[NR];
                    ldn<false, T, NR>(zp + q * NR, t3);
#pragma unroll
                    for (int r = 0; r < NR; r++) xb[r][q] = t3[r];
                }
            } else {
                prolong_at<T, M, NR>(mv, a.Z, -1 - cj, xb);
            }
            T bv[9];
#pragma unroll
            for (int q = 0; q < 9; q++) bv[q] = kc ? src[q] : __ldg(src + q);
#pragma unroll
            for (int r = 0; r < NR; r++) {
                acc[r][0] += bv[0] * xb[r][0] + bv[1] * xb[r][1] + bv[2] * xb[r][2];
                acc[r][1] += bv[3] * xb[r][0] + bv[4] * xb[r][1] + bv[5] * xb[r][2];
                acc[r][2] += bv[6] * xb[r][0] + bv[7] * xb[r][1] + bv[8] * xb[r][2];
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int q = 0; q < 3; q++)
#pragma unroll
            for (int o = 1; o < kSpG; o <<= 1) acc[r][q] += __shfl_xor_sync(0xffffffffu, acc[r][q], o, kSpG);
    if (i < rc.r1 && g == 0) {
        const T* zp = fc.zs + (size_t)fc.dsl[i - rc.r0] * 3 * NR;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const size_t k = (size_t)(3 * i + q) * NR;
            T zv[NR], wv[NR];
            ldn<false, T, NR>(zp + q * NR, zv);
#pragma unroll
            for (int r = 0; r < NR; r++) {
                wv[r] = acc[r][q];
                if (run[r]) {
                    dots[r] += (double)rpre[q][r] * (double)zv[r];
                    dots[NR + r] += (double)zv[r] * (double)wv[r];
                    if (!first) dots[2 * NR + r] += (double)zv[r] * (double)apre[q][r];
                }
            }
            stn<T, NR>(a.z + k, zv);
            stn<T, NR>(a.w + k, wv);
        }
    }
}

// The CTA's first level-1 bank m = blockIdx.x as the update pass reads it, kept in shared
// memory for the solve (the hierarchy is fixed during a solve): its level-0 bank range, the
// vertex and local level-1 parent of each position of the first kPosBanks banks of the range,
// and the level-2 parent of each of its level-1 nodes.
constexpr int kPosBanks = 32;
struct PosCache {
    int b_lo, b_hi;
    const int* v;    // [kPosBanks * 16]
    const int* par;  // [kPosBanks * 16] local level-1 id (up - start1), -1 without a vertex
    const int* up1;  // [16]
    bool valid;
};

// Phase B: the position pass of phase_positions_l2 (update mode) on the fused recurrence.
// acc[r] += r.r, acc[NR + r] += p.Ap (owners).  A stopped right-hand side keeps x, r, p and
// Ap (selected, never multiplied).
template <class T, class M, int NR>
__device__ void phase_fused_update(const CoopArgs<T, M, NR>& a, const double (&alpha)[NR], const double (&beta)[NR],
                                   bool first, const T* p_old, T* p_new, const T* ap_old, T* ap_new, const T* r_old,
                                   T* r_new, const bool (&run)[NR], double (&acc)[2 * NR], M (*s_l1)[3 * NR],
                                   const PosCache& pc) {
    // components of a vertex loaded together: all three with one right-hand side (with four,
    // the 72 values spill and the batched solve measured slower)
    constexpr int kQ = NR == 1 ? 3 : 1;
    const MasView& mv = a.mv;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int start1 = mv.info[1], count1 = mv.info[9];
    const int nb1 = (count1 + 15) >> 4;
    for (int m = blockIdx.x; m < nb1; m += gridDim.x) {  // block-uniform
        const bool cached = pc.valid && m == (int)blockIdx.x;
        const int b_lo = cached ? pc.b_lo : __ldg(a.l1_first + m), b_hi = cached ? pc.b_hi : __ldg(a.l1_last + m);
        const int id_lo = 16 * m, id_hi = min(16 * m + 16, count1);
        for (int b0 = b_lo + 2 * w; b0 <= b_hi; b0 += 2 * (kCoopThreads / 32)) {  // warp-uniform
            const int bank = b0 + (lane >> 4);
            const int pos = bank * 16 + (lane & 15);
            int v, par;
            if (cached && bank - b_lo < kPosBanks) {
                v = bank <= b_hi ? pc.v[pos - 16 * b_lo] : -1;
                par = bank <= b_hi ? pc.par[pos - 16 * b_lo] : -1;
            } else {
                v = bank <= b_hi ? __ldg(mv.part_map + pos) : -1;
                par = v >= 0 ? __ldg(mv.up + pos) - start1 : -1;
            }
            int firstc = par >= 0 ? par : 0x7fffffff;
#pragma unroll
            for (int o = 1; o < 16; o <<= 1) firstc = min(firstc, __shfl_xor_sync(0xffffffffu, firstc, o, 16));
            const bool own = firstc >= id_lo;
            M val[NR * 3];
#pragma unroll
            for (int k = 0; k < NR * 3; k++) val[k] = 0;
            if (v >= 0) {
                // the loads of kQ components go out together, ahead of their stores: the
                // compiler cannot move a load above a store to another array (it may alias),
                // so component by component would cost one L2 round trip each
#pragma unroll
                for (int q0 = 0; q0 < 3; q0 += kQ) {
                    T zv[kQ][NR], wv[kQ][NR], po[kQ][NR], ao[kQ][NR], rv[kQ][NR], xv[kQ][NR];
#pragma unroll
                    for (int j = 0; j < kQ; j++) {
                        const size_t k = (size_t)(3 * v + q0 + j) * NR;
                        ldn<true, T, NR>(a.z + k, zv[j]);
                        ldn<true, T, NR>(a.w + k, wv[j]);
                        ldn<true, T, NR>(r_old + k, rv[j]);
                        if (!first) {
                            ldn<true, T, NR>(p_old + k, po[j]);
                            ldn<true, T, NR>(ap_old + k, ao[j]);
                        } else {
#pragma unroll
                            for (int r = 0; r < NR; r++) po[j][r] = ao[j][r] = 0;
                        }
#pragma unroll
                        for (int r = 0; r < NR; r++) xv[j][r] = 0;
                        if (own) ldn<true, T, NR>(a.x + k, xv[j]);
                    }
#pragma unroll
                    for (int j = 0; j < kQ; j++) {
                        const int q = q0 + j;
                        const size_t k = (size_t)(3 * v + q) * NR;
                        T pn[NR], an[NR];
#pragma unroll
                        for (int r = 0; r < NR; r++) {
                            const T al = (T)alpha[r], be = (T)beta[r];
                            pn[r] = po[j][r];
                            an[r] = ao[j][r];
                            if (run[r]) {
                                pn[r] = first ? zv[j][r] : zv[j][r] + be * po[j][r];
                                an[r] = first ? wv[j][r] : wv[j][r] + be * ao[j][r];
                                rv[j][r] = rv[j][r] - al * an[r];
                                xv[j][r] = xv[j][r] + al * pn[r];
                                if (own) {
                                    acc[r] += (double)rv[j][r] * (double)rv[j][r];
                                    acc[NR + r] += (double)pn[r] * (double)an[r];
                                }
                            }
                            val[r * 3 + q] = run[r] ? (M)rv[j][r] : (M)0;
                        }
                        if (own) {
                            stn<T, NR>(a.x + k, xv[j]);
                            stn<T, NR>(r_new + k, rv[j]);
                            stn<T, NR>(p_new + k, pn);
                            stn<T, NR>(ap_new + k, an);
                        }
                    }
                }
            }
            if (own && bank <= b_hi) store_levels01<M, NR>(a.R, pos, val);
            const int gp = (par >= id_lo && par < id_hi) ? par : -1;
            M sum[NR * 3];
            const bool lead = bank_group_sum<M, NR>(gp, val, sum);
            if (lead && gp >= 0) {
#pragma unroll
                for (int k = 0; k < NR * 3; k++) s_l1[gp - id_lo][k] = sum[k];
                store_levels01<M, NR>(a.R, start1 + gp, sum);
            }
        }
        __syncthreads();
        if (w == 0) {
            const int a1 = id_lo + (lane & 15);
            const bool ok = lane < 16 && a1 < id_hi;
            M v1[NR * 3];
#pragma unroll
            for (int k = 0; k < NR * 3; k++) v1[k] = ok ? s_l1[lane & 15][k] : (M)0;
            bank_reduce_store<M, NR>(ok ? (cached ? pc.up1[lane & 15] : __ldg(mv.up + start1 + a1)) : -1, v1, a.R);
        }
        __syncthreads();
    }
}

// The coarse chain in shared memory: R of levels >= 3 lives in `cb` (the CTA's staging
// array, 160 nodes), restricted from R2 with the half-warp groups of restrict_coarse_cta (the
// same sums), and the domains of levels >= 3 are solved from it, their inverses from `cache`
// (ncache of them, from domain nd2 on) or global memory.  Only Z is written.  Returns false
// (nothing done) when the levels above 2 hold more than 160 nodes.  `cb` was zeroed once at
// the start of the solve: every node with children is overwritten by each call, and the
// padding nodes stay zero.  upc: the parents of the nodes from level 2 on (up[info[2] + k]),
// kept in shared memory for the solve, or nullptr (read from global memory).
template <class T, class M, int NR>
__device__ bool coarse_chain_smem(const CoopArgs<T, M, NR>& a, M* cb, const M* cache, int ncache, const int* upc) {
    const int* info = a.mv.info;
    const int L = a.mv.L;
    const int start3 = info[3], start2 = info[2];
    const int ntop = info[16] - start3;  // nodes of levels >= 3, padding included
    if (ntop > 160 || ntop <= 0) return false;
    for (int l = 2; l + 1 < L; l++) {
        const int count = info[8 + l], start = info[l];
        for (int base = 0; base < count; base += blockDim.x) {
            const int aa = base + threadIdx.x;
            M v[NR * 3];
            int par = -1;
            if (aa < count) {
                const int g = start + aa;
                par = upc ? upc[g - start2] : __ldg(a.mv.up + g);
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    M t[NR];
                    if (l == 2) ldn<true, M, NR>(a.R + (size_t)(3 * g + q) * NR, t);
                    else ldn<false, M, NR>(cb + (size_t)(3 * (g - start3) + q) * NR, t);
#pragma unroll
                    for (int r = 0; r < NR; r++) v[r * 3 + q] = t[r];
                }
            } else {
#pragma unroll
                for (int k = 0; k < NR * 3; k++) v[k] = 0;
            }
            M sum[NR * 3];
            const bool lead = bank_group_sum<M, NR>(par, v, sum);
            if (par >= 0 && lead) {
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    M o[NR];
#pragma unroll
                    for (int r = 0; r < NR; r++) o[r] = sum[r * 3 + q];
                    stn<M, NR>(cb + (size_t)(3 * (par - start3) + q) * NR, o);
                }
            }
        }
        __syncthreads();
    }
    // Z = A_d^-1 R_d for the domains of levels >= 3, kDomPerCta per round
    const int ld = threadIdx.x / 48, i = threadIdx.x % 48;
    for (int d0 = a.nd2; d0 < a.ndom; d0 += kDomPerCta) {
        const int d = d0 + ld;
        if (ld < kDomPerCta && d < a.ndom) {
            const int slot = d - a.nd2;
            const bool sm = slot < ncache;
            const M* Ad = sm ? cache + (size_t)slot * 2304 : a.inv + (size_t)d * 2304;
            const M* Rd = cb + (size_t)(48 * d - 3 * start3) * NR;
            M acc[NR];
#pragma unroll
            for (int r = 0; r < NR; r++) acc[r] = 0;
            constexpr int kU = sizeof(M) == 4 ? (NR == 1 ? 24 : 12) : (NR == 1 ? 12 : 6);
#pragma unroll
            for (int j0 = 0; j0 < 48; j0 += kU) {
                M wv[kU];
#pragma unroll
                for (int j = 0; j < kU; j++) wv[j] = sm ? Ad[(j0 + j) * 48 + i] : __ldg(Ad + (j0 + j) * 48 + i);
#pragma unroll
                for (int j = 0; j < kU; j++) {
                    M rj[NR];
                    ldn<false, M, NR>(Rd + (size_t)(j0 + j) * NR, rj);
#pragma unroll
                    for (int r = 0; r < NR; r++) acc[r] += wv[j] * rj[r];
                }
            }
            stn<M, NR>(a.Z + (48 * (size_t)d + i) * NR, acc);
        }
    }
    __syncthreads();  // cb is the staging array of the next phase's solves
    return true;
}

// Phase C: the MAS domain solves, levels 0..2 over the grid while (with more levels) the
// last CTA restricts 2 -> 3 -> ... and solves the domains above, in shared memory where the
// levels above 2 fit (coarse_chain_smem), else as the MAS phase of k_pcg_coop.
template <class T, class M, int NR>
__device__ void phase_fused_mas(const CoopArgs<T, M, NR>& a, M (*sR)[48 * NR], const M* dcache, int ndc,
                                const int* upc) {
    const int L = a.mv.L, G = gridDim.x;
    if (L > 3 && blockIdx.x == G - 1) {
        if (!coarse_chain_smem<T, M, NR>(a, &sR[0][0], dcache, ndc, upc)) {
            restrict_coarse_cta<M, NR, true>(a.mv.info, a.mv.up, L, a.R, 2);
            solve_domain_range<M, NR>(a.inv, a.R, a.Z, a.nd2, a.ndom, G - 1, 1, sR);
        }
    } else {
        solve_domain_range<M, NR>(a.inv, a.R, a.Z, 0, a.nd2, 0, L > 3 ? G - 1 : G, sR, dcache, ndc);
    }
}

// ---- refinement epilogue of the mixed solve (FP32 inner solve, one right-hand side) --------
// The refined iterate x64 + x at column j, formed where the residual reads it (x64 is updated
// only after every CTA has read it; on the first refinement x64 is not read)
template <class T>
struct RefineOperand {
    const double* x64;
    const T* x;
    int assign;
    __device__ __forceinline__ void load(int j, double (&xj)[1][3]) const {
        double xa[3], xb[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            xa[q] = assign ? 0.0 : __ldcg(x64 + 3 * (size_t)j + q);
            xb[q] = (double)__ldcg(x + 3 * (size_t)j + q);
        }
#pragma unroll
        for (int q = 0; q < 3; q++) xj[0][q] = xa[q] + xb[q];
    }
};

// x64 += x (the inner solve's correction)
template <class T, class M, int NR>
__device__ void phase_accumulate64(const CoopArgs<T, M, NR>& a) {
    const int n3 = 3 * a.tp.n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += gridDim.x * blockDim.x)
        a.x64[k] = (a.x64_assign ? 0.0 : a.x64[k]) + (double)__ldcg(a.x + k);
}

// r64 = b64 - A x64 with the FP64 matrix, r64 . r64
template <class T, class M, int NR>
__device__ void phase_residual64(const CoopArgs<T, M, NR>& a, double& rr) {
    RefineOperand<T> op{a.x64, a.x, a.x64_assign};
    constexpr int gpw = 32 / kSpG;
    const int lane = threadIdx.x & 31, n = a.tp.n;
    for (int i0 = grid_warp() * gpw; i0 < n; i0 += grid_warps() * gpw) {  // warp-uniform bound
        const int i = i0 + lane / kSpG, g = lane % kSpG;
        double acc[1][3];
        row_mv<double, 1>(a.tp, a.A64, op, i, g, acc);
        if (i < n && g == 0)
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const double r = a.b64[3 * (size_t)i + q] - acc[0][q];
                a.r64[3 * (size_t)i + q] = r;
                rr += r * r;
            }
    }
}

// r64 . z with z = M r64 from the current Z (as the prolongation, z in T)
template <class T, class M, int NR>
__device__ void phase_prolong_ref(const CoopArgs<T, M, NR>& a, double& rz) {
    const MasView& mv = a.mv;
    for (int v = spread_warp() * 32 + (int)(threadIdx.x & 31); v < a.nv; v += gridDim.x * blockDim.x) {
        const int* tv = mv.table + (size_t)v * mv.L;
        // the vertex's clusters first, then all their Z values (two round trips, not two per
        // level); the sums in level order
        int gl[SGIPC_MAX_LEVELS];
#pragma unroll
        for (int l = 0; l < SGIPC_MAX_LEVELS; l++) gl[l] = l < mv.L ? __ldg(tv + l) : -1;
        M zl[SGIPC_MAX_LEVELS][3];
#pragma unroll
        for (int l = 0; l < SGIPC_MAX_LEVELS; l++)
#pragma unroll
            for (int q = 0; q < 3; q++) zl[l][q] = gl[l] >= 0 ? a.Z[3 * (size_t)gl[l] + q] : (M)0;
        M s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
        for (int l = 0; l < SGIPC_MAX_LEVELS; l++)
            if (gl[l] >= 0) {
                s0 += zl[l][0];
                s1 += zl[l][1];
                s2 += zl[l][2];
            }
        const size_t k = 3 * (size_t)v;
        rz += __ldcg(a.r64 + k) * (double)(T)s0 + __ldcg(a.r64 + k + 1) * (double)(T)s1 +
              __ldcg(a.r64 + k + 2) * (double)(T)s2;
    }
}

// per right-hand-side scalars of the solve (shared memory, see k_pcg_coop)
template <int NR>
struct RhsState {
    double rz0[NR], rz[NR], bn2[NR], rr[NR], beta[NR], alpha[NR];
    int iters[NR], status[NR];
    bool run[NR], stop_rz[NR];
};

// ---- the solve ------------------------------------------------------------------------------
template <class T, class M, int NR>
__global__ void __launch_bounds__(kCoopThreads) k_pcg_coop(CoopArgs<T, M, NR> a) {
    __shared__ double smem[NR * 32];
    __shared__ __align__(16) M sR[kDomPerCta][48 * NR];
    extern __shared__ __align__(16) unsigned char dsm[];
    unsigned int epoch = 0;
    if (threadIdx.x == 0) stamp(a.br, 0, 0);

    // ---- shared-memory residency of this CTA's static rows and level-0/1 domain inverses
    // (constant for the whole solve): loaded once, read every iteration
    constexpr int rpc = kCoopThreads / kSpG;  // rows of one CTA in one SpMV pass
    // held in shared memory (uniform over the CTA) rather than in every thread's registers
    __shared__ RowCache<T> rcs;
    RowCache<T> rc{nullptr, nullptr, nullptr, 0, 0, nullptr, nullptr, nullptr, nullptr};
    const M* dcache = nullptr;
    int ndc = 0;
    {
        int* rp = reinterpret_cast<int*>(dsm);
        int* ccol = rp + coop_pad4(rpc + 1);
        T* cval = reinterpret_cast<T*>(ccol + coop_pad4(a.ecap));
        M* dom = reinterpret_cast<M*>(dsm + coop_rows_bytes(rpc, a.ecap, sizeof(T)) +
                                      coop_contact_bytes(rpc, a.kcap, sizeof(T)));
        if (a.ecap > 0) {
            const int r0 = blockIdx.x * rpc, r1 = min(a.tp.n, r0 + rpc);
            if (r0 < r1) {
                const int e0 = __ldg(a.tp.frow_ptr + r0), e1 = __ldg(a.tp.frow_ptr + r1);
                for (int k = threadIdx.x; k <= r1 - r0; k += blockDim.x) rp[k] = __ldg(a.tp.frow_ptr + r0 + k) - e0;
                smem_fill(ccol, a.tp.fcol + e0, e1 - e0);
                smem_fill(cval, a.A.fval + 9 * (size_t)e0, 9 * (e1 - e0));
                rc = RowCache<T>{rp, ccol, cval, r0, r1, nullptr, nullptr, nullptr, nullptr};
                // the rows' contact entries, when they fit the kcap slots
                int* ru = reinterpret_cast<int*>(dsm + coop_rows_bytes(rpc, a.ecap, sizeof(T)));
                int* rl = ru + coop_pad4(rpc + 1);
                int* kcol = rl + coop_pad4(rpc + 1);
                T* kval = reinterpret_cast<T*>(kcol + coop_pad4(a.kcap));
                const int u0 = __ldg(a.tp.cu_ptr + r0), u1 = __ldg(a.tp.cu_ptr + r1);
                const int q0 = __ldg(a.tp.cl_ptr + r0), q1 = __ldg(a.tp.cl_ptr + r1);
                const int nu = u1 - u0, nl = q1 - q0;
                if (a.kcap > 0 && nu + nl <= a.kcap) {
                    for (int k = threadIdx.x; k <= r1 - r0; k += blockDim.x) {
                        ru[k] = __ldg(a.tp.cu_ptr + r0 + k) - u0;
                        rl[k] = __ldg(a.tp.cl_ptr + r0 + k) - q0 + nu;
                    }
                    smem_fill(kcol, a.tp.uc_col + u0, nu);
                    smem_fill(kcol + nu, a.tp.cl_col + q0, nl);
                    smem_fill(kval, a.A.uc + 9 * (size_t)u0, 9 * nu);
                    smem_fill(kval + 9 * nu, a.A.cl + 9 * (size_t)q0, 9 * nl);
                    rc.ru = ru;
                    rc.rl = rl;
                    rc.kcol = kcol;
                    rc.kval = kval;
                }
            }
        }
        if (a.dcap > 0) {
            const int d0 = blockIdx.x * kDomPerCta;
            ndc = max(0, min(a.dcap, a.nd01 - d0));
            smem_fill(dom, a.inv + 2304 * (size_t)d0, ndc * 2304);
            dcache = dom;
        }
        if (threadIdx.x == 0) rcs = rc;
        __syncthreads();
        if (threadIdx.x == 0) stamp(a.br, 0, 1);
    }
    // Per right-hand-side state in shared memory: thread 0 updates it from the grid totals
    // (identical in every CTA) after each reduction, the CTA reads it after a __syncthreads.
    // Kept out of the threads' registers, which the phases need for their loads in flight.
    __shared__ RhsState<NR> S;
    if (threadIdx.x == 0)
#pragma unroll
        for (int r = 0; r < NR; r++) {
            S.run[r] = true;
            S.stop_rz[r] = false;
            S.iters[r] = 0;
            S.status[r] = SGIPC_OK;
            S.rz0[r] = S.rz[r] = S.rr[r] = S.bn2[r] = S.beta[r] = S.alpha[r] = 0.0;
        }
    double v[NR], t[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) v[r] = 0.0;
    // ---- r = b, x = 0, z = M r, rz0 = r.z
    // (level-1-aligned passes keep the residual in two buffers: rcur holds the current one)
    __shared__ M s_l1[16][3 * NR];
    T* rcur = a.r;
    T* ralt = a.r2;
    if (a.l2mode)
        phase_positions_l2<T, M, NR, 1>(a, S.alpha, nullptr, nullptr, rcur, S.run, v, s_l1);
    else
        phase_init(a, v);
    bool ok = grid_reduce<NR>(a.br, ++epoch, kPhInit, v, a.partial, smem, t);  // starts with __syncthreads
    if (threadIdx.x == 0)
#pragma unroll
        for (int r = 0; r < NR; r++) S.bn2[r] = t[r];
    ok = ok && phase_mas(a, sR, epoch, dcache, ndc);
    if (ok) {
#pragma unroll
        for (int r = 0; r < NR; r++) v[r] = 0.0;
        phase_prolong(a, rcur, S.run, v);
        ok = grid_reduce<NR>(a.br, ++epoch, kPhProlong, v, a.partial, smem, t);
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (int r = 0; r < NR; r++) {
            const double rz0 = ok ? t[r] : 0.0;
            S.rz0[r] = S.rz[r] = rz0;
            S.rr[r] = S.bn2[r];
            if (!(rz0 > 0.0) || !isfinite(rz0)) {
                // b = 0 (or an indefinite preconditioner): nothing to iterate
                S.run[r] = false;
                if (!isfinite(rz0) || rz0 < 0.0) S.status[r] = SGIPC_BREAKDOWN;
            }
        }
    __syncthreads();
    bool any = false;
#pragma unroll
    for (int r = 0; r < NR; r++) any |= S.run[r];
    // ---- iterations k = 1 .. max_iter-1
    for (int k = 1; ok && any && k < a.max_iter; k++) {
        T* pnew = (k & 1) ? a.p1 : a.p0;
        const T* pold = (k & 1) ? a.p0 : a.p1;
#pragma unroll
        for (int r = 0; r < NR; r++) v[r] = 0.0;
        phase_spmv(a, k == 1, S.beta, pold, pnew, S.run, v, rcs);
        if (!(ok = grid_reduce<NR>(a.br, ++epoch, kPhSpmv, v, a.partial, smem, t))) break;
        if (threadIdx.x == 0)
#pragma unroll
            for (int r = 0; r < NR; r++) {
                S.stop_rz[r] = false;
                S.alpha[r] = 0.0;
                if (!S.run[r]) continue;
                S.iters[r] = k;
                const double pAp = t[r], rz = S.rz[r];
                if (!(pAp > 0.0) || !isfinite(pAp) || !isfinite(rz)) {
                    S.run[r] = false;
                    S.status[r] = SGIPC_BREAKDOWN;
                    continue;
                }
                S.alpha[r] = rz / pAp;
                // the reference tests the r.z of the current iterate and stops after its update
                S.stop_rz[r] = a.crit == SGIPC_CRIT_RZ && fabs(rz) <= a.tol * S.rz0[r];
            }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < NR; r++) v[r] = 0.0;
        if (a.l2mode) {
            phase_positions_l2<T, M, NR, 0>(a, S.alpha, pnew, rcur, ralt, S.run, v, s_l1);
            T* t2 = rcur;
            rcur = ralt;
            ralt = t2;
        } else {
            phase_update(a, S.alpha, pnew, S.run, v);
        }
        if (!(ok = grid_reduce<NR>(a.br, ++epoch, kPhUpdate, v, a.partial, smem, t))) break;
        if (threadIdx.x == 0)
#pragma unroll
            for (int r = 0; r < NR; r++) {
                if (!S.run[r]) continue;
                S.rr[r] = t[r];
                if (S.stop_rz[r] || (a.crit == SGIPC_CRIT_TRUE && t[r] <= a.tol * a.tol * S.bn2[r])) S.run[r] = false;
            }
        __syncthreads();
        any = false;
#pragma unroll
        for (int r = 0; r < NR; r++) any |= S.run[r];
        if (!any || k + 1 >= a.max_iter) break;  // converged, or the iteration cap
        if (!(ok = phase_mas(a, sR, epoch, dcache, ndc))) break;
#pragma unroll
        for (int r = 0; r < NR; r++) v[r] = 0.0;
        phase_prolong(a, rcur, S.run, v);
        if (!(ok = grid_reduce<NR>(a.br, ++epoch, kPhProlong, v, a.partial, smem, t))) break;
        if (threadIdx.x == 0)
#pragma unroll
            for (int r = 0; r < NR; r++) {
                if (!S.run[r]) continue;
                S.beta[r] = t[r] / S.rz[r];
                S.rz[r] = t[r];
            }
        __syncthreads();
    }
    double rz_ref = 0.0, rr_ref = 0.0;
    if constexpr (sizeof(T) == 4 && NR == 1) {
        if (ok && a.x64 && a.l2mode) {
            // r64 = b64 - A (x64 + x); r64 . r64; x64 += x (after every CTA has read it);
            // M r64 (FP32 MAS); r64 . M r64
            v[0] = 0.0;
            phase_residual64(a, v[0]);
            ok = grid_reduce<NR>(a.br, ++epoch, kPhRes64, v, a.partial, smem, t);
            rr_ref = t[0];
            if (ok) phase_accumulate64(a);
            v[0] = 0.0;
            if (ok) phase_positions_l2<T, M, NR, 2>(a, S.alpha, nullptr, nullptr, nullptr, S.run, v, s_l1);
            ok = ok && grid_barrier(a.br, ++epoch, kPhRestr64);
            ok = ok && phase_mas(a, sR, epoch, dcache, ndc);
            v[0] = 0.0;
            if (ok) phase_prolong_ref(a, v[0]);
            ok = ok && grid_reduce<NR>(a.br, ++epoch, kPhProlong64, v, a.partial, smem, t);
            rz_ref = t[0];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
        for (int r = 0; r < NR; r++) {
            PcgScalars& sc = a.sc[r];
            sc.rz_ref = rz_ref;
            sc.rr_ref = rr_ref;
            sc.iter = S.iters[r];
            sc.rz0 = S.rz0[r];
            sc.rz = S.rz[r];
            sc.rz_next = S.rz[r];
            sc.bnorm2 = S.bn2[r];
            sc.rr = S.rr[r];
            sc.bodies = 0;
            sc.halt = 1;
            sc.input_flag = a.input_flag ? *(volatile const int*)a.input_flag : 0;
            // state 0 = still running when the iteration cap was reached
            sc.state = ok ? (S.run[r] ? 0 : 2) : 2;
            sc.status = ok ? S.status[r] : SGIPC_CUDA_ERROR;
        }
    }
}


// ---- the fused solve ------------------------------------------------------------------------
template <int NR>
struct FusedState {
    double rz0[NR], rz[NR], bn2[NR], rr[NR], beta[NR], alpha[NR], pap[NR];
    int iters[NR], status[NR];
    bool run[NR], stop_rz[NR];
};
// values per CTA in each parity half of the partial buffer (phase A's three dots).  (Sending
// phase B's two dots with the next phase A's instead, so that B ends at a plain barrier, measured
// 0.6 us per iteration slower.)
template <int NR>
constexpr int kFusedStride = 3 * NR;

template <class T, class M, int NR>
__global__ void __launch_bounds__(kCoopThreads) k_pcg_fused(CoopArgs<T, M, NR> a) {
    __shared__ double smem[kFusedStride<NR> * 32];  // block_sum of up to three values per right-hand side
    __shared__ __align__(16) M sR[kDomPerCta][48 * NR];
    __shared__ __align__(16) M s_l1[16][3 * NR];
    extern __shared__ __align__(16) unsigned char dsm[];
    unsigned int epoch = 0;
    if (threadIdx.x == 0) stamp(a.br, 0, 0);
    constexpr int rpc = kCoopThreads / kSpG;
    __shared__ RowCache<T> rcs;
    __shared__ FusedCache<T, NR> fcs;
    __shared__ int s_pv[kPosBanks * 16], s_ppar[kPosBanks * 16], s_pup1[16];
    __shared__ PosCache pcs;
    __shared__ const int* s_chain_up;
    const M* dcache = nullptr;
    int ndc = 0;
    {
        // the update pass's view of the first level-1 bank (PosCache)
        {
            const int start1 = a.mv.info[1], count1 = a.mv.info[9];
            const int m = blockIdx.x;
            PosCache pc{0, -1, s_pv, s_ppar, s_pup1, false};
            if (m < ((count1 + 15) >> 4)) {
                pc.b_lo = __ldg(a.l1_first + m);
                pc.b_hi = __ldg(a.l1_last + m);
                pc.valid = true;
                const int nb = min(kPosBanks, pc.b_hi - pc.b_lo + 1);
                for (int k = threadIdx.x; k < nb * 16; k += blockDim.x) {
                    const int pos = 16 * pc.b_lo + k;
                    const int v = __ldg(a.mv.part_map + pos);
                    s_pv[k] = v;
                    s_ppar[k] = v >= 0 ? __ldg(a.mv.up + pos) - start1 : -1;
                }
                if (threadIdx.x < 16) {
                    const int a1 = 16 * m + threadIdx.x;
                    s_pup1[threadIdx.x] = a1 < count1 ? __ldg(a.mv.up + start1 + a1) : -1;
                }
            }
            if (threadIdx.x == 0) pcs = pc;
        }
        // rows (static entries with their column slots), contact entries, the column set
        // (cluster tables, z slots), each row's own slot, the own domain inverses
        int* rp = reinterpret_cast<int*>(dsm);
        int* ccol = rp + coop_pad4(rpc + 1);
        T* cval = reinterpret_cast<T*>(ccol + coop_pad4(a.ecap));
        unsigned char* after_rows = dsm + coop_rows_bytes(rpc, a.ecap, sizeof(T));
        int* ru = reinterpret_cast<int*>(after_rows);
        int* rl = ru + coop_pad4(rpc + 1);
        int* kcol = rl + coop_pad4(rpc + 1);
        T* kval = reinterpret_cast<T*>(kcol + coop_pad4(a.kcap));
        unsigned char* after_con = after_rows + coop_contact_bytes(rpc, a.kcap, sizeof(T));
        const int zcap = a.ccap + a.zextra;
        int* tab = reinterpret_cast<int*>(after_con);
        T* zs = reinterpret_cast<T*>(tab + coop_pad4(zcap * SGIPC_MAX_LEVELS));
        unsigned char* after_cols = after_con + fused_cols_bytes(zcap, sizeof(T), NR);
        int* dsl = reinterpret_cast<int*>(after_cols);
        M* dom = reinterpret_cast<M*>(after_cols + (size_t)coop_pad4(rpc) * 4);
        RowCache<T> rc{rp, ccol, cval, 0, 0, nullptr, nullptr, nullptr, nullptr};
        FusedCache<T, NR> fc{tab, zs, dsl, 0, 0};
        __shared__ int s_extra;
        const int r0 = blockIdx.x * rpc, r1 = min(a.tp.n, r0 + rpc);
        if (r0 < r1) {
            const int e0 = __ldg(a.tp.frow_ptr + r0), e1 = __ldg(a.tp.frow_ptr + r1);
            for (int k = threadIdx.x; k <= r1 - r0; k += blockDim.x) rp[k] = __ldg(a.tp.frow_ptr + r0 + k) - e0;
            smem_fill(ccol, a.cs_lcol + e0, e1 - e0);
            smem_fill(cval, a.A.fval + 9 * (size_t)e0, 9 * (e1 - e0));
            for (int k = threadIdx.x; k < r1 - r0; k += blockDim.x) dsl[k] = __ldg(a.cs_dslot + r0 + k);
            rc.r0 = r0;
            rc.r1 = r1;
            const int u0 = __ldg(a.tp.cu_ptr + r0), u1 = __ldg(a.tp.cu_ptr + r1);
            const int q0 = __ldg(a.tp.cl_ptr + r0), q1 = __ldg(a.tp.cl_ptr + r1);
            const int nu = u1 - u0, nl = q1 - q0;
            if (a.kcap > 0 && nu + nl <= a.kcap) {
                for (int k = threadIdx.x; k <= r1 - r0; k += blockDim.x) {
                    ru[k] = __ldg(a.tp.cu_ptr + r0 + k) - u0;
                    rl[k] = __ldg(a.tp.cl_ptr + r0 + k) - q0 + nu;
                }
                smem_fill(kcol, a.tp.uc_col + u0, nu);
                smem_fill(kcol + nu, a.tp.cl_col + q0, nl);
                smem_fill(kval, a.A.uc + 9 * (size_t)u0, 9 * nu);
                smem_fill(kval + 9 * nu, a.A.cl + 9 * (size_t)q0, 9 * nl);
                rc.ru = ru;
                rc.rl = rl;
                rc.kcol = kcol;
                rc.kval = kval;
            }
            const int c0 = __ldg(a.cs_ptr + blockIdx.x);
            fc.nc = __ldg(a.cs_ptr + blockIdx.x + 1) - c0;
            // (a gather through the column list: four elements per thread in flight)
            for (int k0 = threadIdx.x; k0 < fc.nc * SGIPC_MAX_LEVELS; k0 += 4 * (int)blockDim.x) {
                int col[4], tv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int k = k0 + u * (int)blockDim.x;
                    col[u] = k < fc.nc * SGIPC_MAX_LEVELS ? __ldg(a.cs_cols + c0 + k / SGIPC_MAX_LEVELS) : -1;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int k = k0 + u * (int)blockDim.x, l = k % SGIPC_MAX_LEVELS;
                    tv[u] = col[u] >= 0 && l < a.mv.L ? __ldg(a.mv.table + (size_t)col[u] * a.mv.L + l) : -1;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int k = k0 + u * (int)blockDim.x;
                    if (k < fc.nc * SGIPC_MAX_LEVELS) tab[k] = tv[u];
                }
            }
            // resident contact entries: the slot of their column in the static set, or a slot of
            // their own (the z values, not the slot numbers, enter the products: the atomic
            // order of the extra slots changes nothing), or -(column + 1) beyond the slots
            fc.nz = fc.nc;
            if (rc.kcol) {
                int* scol = reinterpret_cast<int*>(zs);  // the sorted set, during this set-up only
                for (int k = threadIdx.x; k < fc.nc; k += blockDim.x) scol[k] = __ldg(a.cs_cols + c0 + k);
                if (threadIdx.x == 0) s_extra = 0;
                __syncthreads();
                for (int k = threadIdx.x; k < nu + nl; k += blockDim.x) {
                    const int col = kcol[k];
                    int lo = 0, hi = fc.nc;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (scol[mid] < col) lo = mid + 1;
                        else hi = mid;
                    }
                    int slot;
                    if (lo < fc.nc && scol[lo] == col) {
                        slot = lo;
                    } else {
                        const int x = atomicAdd(&s_extra, 1);
                        slot = x < a.zextra ? fc.nc + x : -1 - col;
                        if (x < a.zextra)
                            for (int l = 0; l < SGIPC_MAX_LEVELS; l++)
                                tab[(size_t)(fc.nc + x) * SGIPC_MAX_LEVELS + l] =
                                    l < a.mv.L ? __ldg(a.mv.table + (size_t)col * a.mv.L + l) : -1;
                    }
                    kcol[k] = slot;
                }
                __syncthreads();
                fc.nz = fc.nc + min(s_extra, a.zextra);
            }
        }
        // the first round of the CTA's level-0..2 domains in the MAS phase (as k_pcg_coop);
        // with more than three levels the last CTA takes the domains above level 2 instead
        if (a.dcap > 0) {
            const bool chain = a.mv.L > 3 && blockIdx.x == gridDim.x - 1;
            const int d0 = chain ? a.nd2 : (int)blockIdx.x * kDomPerCta;
            ndc = max(0, min(a.dcap, (chain ? a.ndom : a.nd2) - d0));
            smem_fill(dom, a.inv + 2304 * (size_t)d0, ndc * 2304);
            dcache = dom;
        }
        // the coarse chain's CTA: its staging array zeroed once (the chain overwrites every node
        // with children and leaves the padding nodes at zero), and the parents of the nodes
        // from level 2 on cached in the update pass's position arrays, which this CTA does not
        // use when it holds no level-1 bank
        if (a.mv.L > 3 && blockIdx.x == gridDim.x - 1) {
            for (int k = threadIdx.x; k < kDomPerCta * 48 * NR; k += blockDim.x) (&sR[0][0])[k] = 0;
            const int nup = a.mv.info[16] - a.mv.info[2];
            const bool no_bank = (int)blockIdx.x >= ((a.mv.info[9] + 15) >> 4);  // s_pv unused
            const bool room = no_bank && nup > 0 && nup <= kPosBanks * 16;
            if (room)
                for (int k = threadIdx.x; k < nup; k += blockDim.x) s_pv[k] = __ldg(a.mv.up + a.mv.info[2] + k);
            if (threadIdx.x == 0) s_chain_up = room ? s_pv : nullptr;
        } else if (threadIdx.x == 0) {
            s_chain_up = nullptr;
        }
        if (threadIdx.x == 0) {
            rcs = rc;
            fcs = fc;
        }
        __syncthreads();
        if (threadIdx.x == 0) stamp(a.br, 0, 1);
    }
    __shared__ FusedState<NR> S;
    if (threadIdx.x == 0)
#pragma unroll
        for (int r = 0; r < NR; r++) {
            S.run[r] = true;
            S.stop_rz[r] = false;
            S.iters[r] = 0;
            S.status[r] = SGIPC_OK;
            S.rz0[r] = S.rz[r] = S.rr[r] = S.bn2[r] = S.beta[r] = S.alpha[r] = S.pap[r] = 0.0;
        }
    double v[NR], t[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) v[r] = 0.0;
    // ---- r = b, x = 0, R at levels 0..2, the CTA's level-0/1 domain solves; ||b||^2
    T* rcur = a.r;
    T* ralt = a.r2;
    T* pcur = a.p0;
    T* palt = a.p1;
    T* acur = a.Ap;
    T* aalt = a.Ap2;
    phase_positions_l2<T, M, NR, 1>(a, S.alpha, nullptr, nullptr, rcur, S.run, v, s_l1);
    bool ok = grid_reduce<NR>(a.br, ++epoch, kPhInit, v, a.partial, smem, t, kFusedStride<NR>);
    if (threadIdx.x == 0)
#pragma unroll
        for (int r = 0; r < NR; r++) S.bn2[r] = S.rr[r] = t[r];
    if (ok) phase_fused_mas<T, M, NR>(a, sR, dcache, ndc, s_chain_up);
    ok = ok && grid_barrier(a.br, ++epoch, kPhMas);
    for (int k = 1; ok; k++) {
        // ---- A: z, w = A z, r.z, z.w, z.Ap_old
        double d3[3 * NR], t3[3 * NR];
#pragma unroll
        for (int q = 0; q < 3 * NR; q++) d3[q] = 0.0;
        __syncthreads();  // S read below is settled
        phase_fused_spmv<T, M, NR>(a, rcs, fcs, rcur, acur, k == 1, S.run, d3);
        if (!(ok = grid_reduce<3 * NR>(a.br, ++epoch, kPhFusedA, d3, a.partial, smem, t3, kFusedStride<NR>))) break;
        if (threadIdx.x == 0)
#pragma unroll
            for (int r = 0; r < NR; r++) {
                S.stop_rz[r] = false;
                S.alpha[r] = 0.0;
                if (!S.run[r]) continue;
                const double rz = t3[r], zw = t3[NR + r], zap = t3[2 * NR + r];
                if (k == 1) {
                    S.rz0[r] = S.rz[r] = rz;
                    if (!(rz > 0.0) || !isfinite(rz)) {
                        // b = 0 (or an indefinite preconditioner): nothing to iterate
                        S.run[r] = false;
                        if (!isfinite(rz) || rz < 0.0) S.status[r] = SGIPC_BREAKDOWN;
                        continue;
                    }
                }
                if (k >= a.max_iter) continue;  // the iteration cap: no update
                const double beta = k == 1 ? 0.0 : rz / S.rz[r];
                const double pAp = k == 1 ? zw : zw + 2.0 * beta * zap + beta * beta * S.pap[r];
                S.iters[r] = k;
                if (!(pAp > 0.0) || !isfinite(pAp) || !isfinite(rz)) {
                    S.run[r] = false;
                    S.status[r] = SGIPC_BREAKDOWN;
                    continue;
                }
                S.beta[r] = beta;
                S.alpha[r] = rz / pAp;
                S.rz[r] = rz;
                // the reference tests the r.z of the current iterate and stops after its update
                S.stop_rz[r] = a.crit == SGIPC_CRIT_RZ && fabs(rz) <= a.tol * S.rz0[r];
            }
        __syncthreads();
        bool any = false;
#pragma unroll
        for (int r = 0; r < NR; r++) any |= S.run[r];
        if (!any || k >= a.max_iter) break;
        // ---- B: p, Ap, x, r, restriction to levels 0..2; r.r, p.Ap
        double d2[2 * NR], t2[2 * NR];
#pragma unroll
        for (int q = 0; q < 2 * NR; q++) d2[q] = 0.0;
        phase_fused_update<T, M, NR>(a, S.alpha, S.beta, k == 1, pcur, palt, acur, aalt, rcur, ralt, S.run, d2, s_l1,
                                     pcs);
        T* tmp = rcur;
        rcur = ralt;
        ralt = tmp;
        tmp = pcur;
        pcur = palt;
        palt = tmp;
        tmp = acur;
        acur = aalt;
        aalt = tmp;
        if (!(ok = grid_reduce<2 * NR>(a.br, ++epoch, kPhFusedB, d2, a.partial, smem, t2, kFusedStride<NR>))) break;
        if (threadIdx.x == 0)
#pragma unroll
            for (int r = 0; r < NR; r++) {
                if (!S.run[r]) continue;
                S.rr[r] = t2[r];
                S.pap[r] = t2[NR + r];
                if (S.stop_rz[r] || (a.crit == SGIPC_CRIT_TRUE && t2[r] <= a.tol * a.tol * S.bn2[r])) S.run[r] = false;
            }
        __syncthreads();
        any = false;
#pragma unroll
        for (int r = 0; r < NR; r++) any |= S.run[r];
        if (!any || k + 1 >= a.max_iter) break;  // converged, or the iteration cap
        // ---- C: the MAS domain solves
        phase_fused_mas<T, M, NR>(a, sR, dcache, ndc, s_chain_up);
        if (!(ok = grid_barrier(a.br, ++epoch, kPhMas))) break;
    }
    double rz_ref = 0.0, rr_ref = 0.0;
    if constexpr (sizeof(T) == 4 && NR == 1) {
        if (ok && a.x64) {
            // r64 = b64 - A (x64 + x); r64 . r64; x64 += x (after every CTA has read it);
            // M r64 (FP32 MAS); r64 . M r64
            v[0] = 0.0;
            phase_residual64(a, v[0]);
            ok = grid_reduce<NR>(a.br, ++epoch, kPhRes64, v, a.partial, smem, t, kFusedStride<NR>);
            rr_ref = t[0];
            if (ok) phase_accumulate64(a);
            v[0] = 0.0;
            if (ok) phase_positions_l2<T, M, NR, 2>(a, S.alpha, nullptr, nullptr, nullptr, S.run, v, s_l1);
            ok = ok && grid_barrier(a.br, ++epoch, kPhRestr64);
            if (ok) phase_fused_mas<T, M, NR>(a, sR, dcache, ndc, s_chain_up);
            ok = ok && grid_barrier(a.br, ++epoch, kPhMas);
            v[0] = 0.0;
            if (ok) phase_prolong_ref(a, v[0]);
            ok = ok && grid_reduce<NR>(a.br, ++epoch, kPhProlong64, v, a.partial, smem, t, kFusedStride<NR>);
            rz_ref = t[0];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
        for (int r = 0; r < NR; r++) {
            PcgScalars& sc = a.sc[r];
            sc.rz_ref = rz_ref;
            sc.rr_ref = rr_ref;
            sc.iter = S.iters[r];
            sc.rz0 = S.rz0[r];
            sc.rz = S.rz[r];
            sc.rz_next = S.rz[r];
            sc.bnorm2 = S.bn2[r];
            sc.rr = S.rr[r];
            sc.bodies = 0;
            sc.halt = 1;
            sc.input_flag = a.input_flag ? *(volatile const int*)a.input_flag : 0;
            sc.state = ok ? (S.run[r] ? 0 : 2) : 2;
            sc.status = ok ? S.status[r] : SGIPC_CUDA_ERROR;
        }
    }
}

// ---- host launcher ----------------------------------------------------------------------------
// Launch configuration of one instance on this context (device attributes, shared-memory
// residency sizes, occupancy): computed once, it depends only on the device and the static
// pattern.  usable = 0 when the device cannot co-schedule the grid.
template <class T, class M, int NR>
SgipcStatus coop_configure(SgipcCtx* c, SgipcCtx::CoopCfg& cfg) {
    cfg = SgipcCtx::CoopCfg{};
    int coop = 0, nsm = 0, per = 0, optin = 0;
    SG_CHECK(c, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device));
    SG_CHECK(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    SG_CHECK(c, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    cfg.valid = 1;
    if (!coop) return SGIPC_OK;
    // shared-memory residency with one CTA per SM: the static rows of each CTA's SpMV pass
    // (when one pass covers all rows) first, then as many of its level-0/1 domain
    // inverses as still fit (the first round of a CTA's domains)
    const void* fn = (const void*)k_pcg_coop<T, M, NR>;
    cudaFuncAttributes fa;
    SG_CHECK(c, cudaFuncGetAttributes(&fa, fn));
    const long long budget = (long long)optin - (long long)fa.sharedSizeBytes - 1024;
    constexpr int rpc = kCoopThreads / kSpG;
    int ecap = 0, dcap = 0;
    size_t dyn = 0;
    if (budget > 0 && c->h_frow_ptr && c->n <= (long long)nsm * rpc) {
        for (int b = 0; b * rpc < c->n; b++) {
            const int r0 = b * rpc, r1 = r0 + rpc < c->n ? r0 + rpc : c->n;
            const int e = c->h_frow_ptr[r1] - c->h_frow_ptr[r0];
            if (e > ecap) ecap = e;
        }
        if ((long long)coop_rows_bytes(rpc, ecap, sizeof(T)) > budget) ecap = 0;
    }
    int kcap = 0;
    if (ecap > 0 && (long long)(coop_rows_bytes(rpc, ecap, sizeof(T)) +
                                coop_contact_bytes(rpc, kContactSlots, sizeof(T))) <= budget)
        kcap = kContactSlots;
    const size_t rows_bytes = coop_rows_bytes(rpc, ecap, sizeof(T)) + coop_contact_bytes(rpc, kcap, sizeof(T));
    if (budget > 0) {
        long long left = budget - (long long)rows_bytes;
        dcap = left > 0 ? (int)(left / (2304 * (long long)sizeof(M))) : 0;
        if (dcap > kDomPerCta) dcap = kDomPerCta;
    }
    dyn = rows_bytes + (size_t)dcap * 2304 * sizeof(M);
    if (dyn > 0) SG_CHECK(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    SG_CHECK(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_coop<T, M, NR>, kCoopThreads, dyn));
    if (per < 1 && dyn > 0) {  // residency does not fit next to the kernel: run without it
        ecap = kcap = dcap = 0;
        dyn = 0;
        SG_CHECK(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_coop<T, M, NR>, kCoopThreads, 0));
    }
    if (per < 1) return SGIPC_OK;
    if (per > kCoopMaxCtasPerSm) per = kCoopMaxCtasPerSm;
    int grid = dyn > 0 ? nsm : nsm * per;  // residency assumes the one-CTA-per-SM mapping
    if (grid > c->pcg64.coop_cap) grid = c->pcg64.coop_cap;
    if (grid > c->pcg32.coop_cap) grid = c->pcg32.coop_cap;
    cfg.usable = 1;
    cfg.grid = grid;
    cfg.ecap = ecap;
    cfg.kcap = kcap;
    cfg.dcap = dcap;
    cfg.dyn = dyn;
    return SGIPC_OK;
}

// The fused solve's configuration: one CTA per SM, every row resident (static and, when they
// fit, contact entries), the column sets of the context (built for this grid), then as many of
// the CTA's first round of MAS domain inverses as still fit.  usable = 0 sends the solve to
// k_pcg_coop.
template <class T, class M, int NR>
SgipcStatus fused_configure(SgipcCtx* c, SgipcCtx::CoopCfg& cfg) {
    cfg = SgipcCtx::CoopCfg{};
    cfg.valid = 1;
    int coop = 0, nsm = 0, per = 0, optin = 0;
    SG_CHECK(c, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device));
    SG_CHECK(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    SG_CHECK(c, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    constexpr int rpc = kCoopThreads / kSpG;
    if (!coop || !c->cs_ptr || c->cs_grid != nsm || c->cs_cap > kFusedMaxCols || !c->h_frow_ptr ||
        (long long)nsm * rpc < c->n || nsm > c->pcg64.coop_cap || nsm > c->pcg32.coop_cap)
        return SGIPC_OK;
    const void* fn = (const void*)k_pcg_fused<T, M, NR>;
    cudaFuncAttributes fa;
    SG_CHECK(c, cudaFuncGetAttributes(&fa, fn));
    const long long budget = (long long)optin - (long long)fa.sharedSizeBytes - 1024;
    int ecap = 0;
    for (int b = 0; b * rpc < c->n; b++) {
        const int r0 = b * rpc, r1 = r0 + rpc < c->n ? r0 + rpc : c->n;
        const int e = c->h_frow_ptr[r1] - c->h_frow_ptr[r0];
        if (e > ecap) ecap = e;
    }
    const int ccap = c->cs_cap;
    const size_t fixed = coop_rows_bytes(rpc, ecap, sizeof(T)) + fused_cols_bytes(ccap, sizeof(T), NR) +
                         (size_t)coop_pad4(rpc) * 4;
    if ((long long)fixed > budget) return SGIPC_OK;
    const int kcap = (long long)(fixed + coop_contact_bytes(rpc, kContactSlots, sizeof(T))) <= budget ? kContactSlots : 0;
    // z slots for contact columns outside the static set, up to one per resident contact
    // entry, as far as they fit
    int zextra = 0;
    if (kcap > 0) {
        const long long room = budget - (long long)(fixed + coop_contact_bytes(rpc, kcap, sizeof(T)));
        const long long per = SGIPC_MAX_LEVELS * 4 + 3LL * NR * (long long)sizeof(T);
        zextra = room > 64 ? (int)((room - 64) / per) : 0;
        if (zextra > kcap) zextra = kcap;
    }
    const size_t base = coop_rows_bytes(rpc, ecap, sizeof(T)) + fused_cols_bytes(ccap + zextra, sizeof(T), NR) +
                        (size_t)coop_pad4(rpc) * 4 + coop_contact_bytes(rpc, kcap, sizeof(T));
    long long left = budget - (long long)base;
    int dcap = left > 0 ? (int)(left / (2304 * (long long)sizeof(M))) : 0;
    if (dcap > kDomPerCta) dcap = kDomPerCta;
    const size_t dyn = base + (size_t)dcap * 2304 * sizeof(M);
    SG_CHECK(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    SG_CHECK(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_fused<T, M, NR>, kCoopThreads, dyn));
    if (per < 1) return SGIPC_OK;
    cfg.usable = 1;
    cfg.grid = nsm;
    cfg.ecap = ecap;
    cfg.kcap = kcap;
    cfg.dcap = dcap;
    cfg.ccap = ccap;
    cfg.zextra = zextra;
    cfg.dyn = dyn;
    return SGIPC_OK;
}

template <class T, class M, int NR>
SgipcStatus run_pcg_coop(SgipcCtx* c, PcgWork& w, int fp32_mas, const double* b, double tol, int max_iter, int crit,
                         cudaStream_t s, bool* used, RefineArgs* ref) {
    *used = false;
    const char* e = getenv("SGIPC_PCG_GRAPH");
    if (e && e[0] == '1') return SGIPC_OK;  // the graph of per-phase kernels instead
    constexpr int inst = (sizeof(T) == 8 ? (sizeof(M) == 8 ? 0 : 1) : 2) + (NR == 4 ? 3 : 0);
    SgipcCtx::CoopCfg& cfg = c->coop_cfg[inst];
    if (!cfg.valid) {
        SgipcStatus st = coop_configure<T, M, NR>(c, cfg);
        if (st != SGIPC_OK) return st;
    }
    if (!cfg.usable) return SGIPC_OK;  // the graph of per-phase kernels instead
    MasWork& m = c->mas;
    const int* h = m.h_info;
    const int L = m.levelnum;
    const int ndom = h[16] / 16;
    const int nd01 = L > 2 ? h[2] / 16 : ndom;
    // the fused iteration where it applies (three levels or more, every row resident);
    // SGIPC_PCG_FUSED=0 keeps the four-phase iteration
    const char* fz = getenv("SGIPC_PCG_FUSED");
    SgipcCtx::CoopCfg& fcfg = c->fused_cfg[inst];
    bool fused = false;
    // (FP64 vectors with four right-hand sides measured slower fused: kept four-phase)
    if (L >= 3 && !(fz && fz[0] == '0') && !(sizeof(T) == 8 && sizeof(M) == 8 && NR == 4)) {
        if (!fcfg.valid) {
            SgipcStatus st = fused_configure<T, M, NR>(c, fcfg);
            if (st != SGIPC_OK) return st;
        }
        fused = fcfg.usable != 0;
    }
    const SgipcCtx::CoopCfg& use = fused ? fcfg : cfg;
    const int grid = use.grid, ecap = use.ecap, kcap = use.kcap, dcap = use.dcap;
    const size_t dyn = use.dyn;
    const void* fn = fused ? (const void*)k_pcg_fused<T, M, NR> : (const void*)k_pcg_coop<T, M, NR>;
    CoopArgs<T, M, NR> a;
    a.tp = topo_of(c);
    a.A = mat_view<T>(c);
    a.mv = mas_view(c);
    a.inv = fp32_mas ? (const M*)m.dom32 : (const M*)m.dom64;
    a.R = fp32_mas ? (M*)m.R32 : (M*)m.R64;
    a.Z = fp32_mas ? (M*)m.Z32 : (M*)m.Z64;
    a.b = b;
    a.x = (T*)w.x;
    a.r = (T*)w.r;
    a.r2 = (T*)w.r2;
    a.z = (T*)w.z;
    a.p0 = (T*)w.p;
    a.p1 = (T*)w.p2;
    a.Ap = (T*)w.Ap;
    a.sc = w.sc;
    a.partial = w.coop;
    a.br = {w.ticket + 4, w.ticket + 5, c->wait_limit > 0 ? c->wait_limit : kSpinLimit, c->stamps, c->stamp_epochs};
    a.nv = c->nv;
    a.ndom = ndom;
    a.nd01 = nd01;
    a.nd2 = L > 3 ? h[3] / 16 : a.ndom;
    a.ecap = ecap;
    a.kcap = kcap;
    a.dcap = dcap;
    a.l2mode = L >= 3 && grid >= 2;
    a.l1_first = m.l1_first;
    a.l1_last = m.l1_last;
    const bool refine = ref && sizeof(T) == 4 && NR == 1 && a.l2mode;
    a.x64 = refine ? ref->x64 : nullptr;
    a.x64_assign = refine && ref->assign ? 1 : 0;
    a.input_flag = c->dflag;
    a.b64 = refine ? ref->b64 : nullptr;
    a.r64 = refine ? ref->r64 : nullptr;
    a.A64 = mat_view<double>(c);
    if (ref) ref->done = refine;
    a.max_iter = max_iter;
    a.crit = crit;
    a.tol = tol;
    a.w = (T*)w.w;
    a.Ap2 = (T*)w.Ap2;
    a.cs_ptr = c->cs_ptr;
    a.cs_cols = c->cs_cols;
    a.cs_lcol = c->cs_lcol;
    a.cs_dslot = c->cs_dslot;
    a.ccap = fused ? use.ccap : 0;
    a.zextra = fused ? use.zextra : 0;
    SG_CHECK(c, cudaMemsetAsync(w.ticket + 4, 0, 2 * sizeof(unsigned int), s));
    // level-1-aligned passes write the level-0 entries of the banks that hold vertices only:
    // the others must read as zero in every solve, whatever the right-hand-side count
    if (a.l2mode) SG_CHECK(c, cudaMemsetAsync(a.R, 0, sizeof(M) * 3 * (size_t)m.npos * NR, s));
    void* args[] = {&a};
    SG_COUNT(c, 1);
    SG_CHECK(c, cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kCoopThreads), args, dyn, s));
    *used = true;
    return SGIPC_OK;
}

#define SGIPC_COOP_INST(T, M, NR)                                                                             \
    template SgipcStatus run_pcg_coop<T, M, NR>(SgipcCtx*, PcgWork&, int, const double*, double, int, int, \
                                                cudaStream_t, bool*, RefineArgs*);
SGIPC_COOP_INST(double, double, 1)
SGIPC_COOP_INST(double, float, 1)
SGIPC_COOP_INST(float, float, 1)
SGIPC_COOP_INST(double, double, 4)
SGIPC_COOP_INST(double, float, 4)
SGIPC_COOP_INST(float, float, 4)

int coop_max_grid(int device) {
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    return nsm * kCoopMaxCtasPerSm;
}

}  // namespace sgipc
