// sgipc_broad.cu — the contact pairs of a Newton iterate and the lagged friction set-up on the GPU.
//
// GIPC::buildCP (StiffGIPC/GIPC.cu:9065-9083) finds, through two LBVHs (mlbvh.cu), every
// surface point closer than d-hat to a surface triangle and every pair of surface edges closer
// than d-hat, and encodes each as the int4 the barrier kernels read (_checkPTintersection /
// _checkEEintersection, mlbvh.cu:534-1059), with its CCD candidate, its MatIndex (the pair's rank
// among the pairs of its Hessian size) and the counters _cpNum[5] (total, -, two-, three- and
// four-vertex pairs); _GroundCollisionDetect (GIPC.cu:6433) lists the surface points near the
// ground.  The reference appends with atomics, so its order changes from run to run.
//
// Here a uniform grid replaces the trees.  The cell is wider than any triangle or edge box
// grown by the contact gap sqrt(d-hat), so each grown box covers at most 2 x 2 x 2 cells; the
// (cell, primitive) keys are radix-sorted once per call and a query binary-searches its cells.
// A point visits its own cell; an edge visits the cells of its grown box and reports a pair
// only in the cell holding the low corner of the two boxes' overlap, so every pair is found
// once.  Two passes (count, exclusive scan, write) give a deterministic order: point-triangle
// pairs by surface point, then by triangle; edge-edge pairs by (edge, other edge), sorted after
// the write.  MatIndex is the rank in that order.  The pair tests restate the reference's
// closest-feature classification and squared distances term for term; this file is compiled
// without contracting multiply-adds (-fmad=false), so a pair at the edge of d-hat, or of a
// feature region, is decided as the reference's own arithmetic decides it.
//
// The lagged friction set-up (_calFrictionLastH_DistAndTan / _calFrictionLastH_gd,
// GIPC.cu:8362-8499, run once per frame in GIPC.cu:8660-8696) maps every non-mollified pair to
// its normal force, closest-point coordinates and tangent basis (FrictionUtils.cuh:52-399);
// the outputs keep the input order.
#include <cub/cub.cuh>

#include "sgipc_geom.cuh"
#include "sgipc_internal.cuh"

namespace sgipc {

// per-context buffers of the pair search (grown when a call needs more)
struct BroadWork {
    int cap_tri = 0, cap_edge = 0, cap_q = 0, cap_rec = 0, cap_sv = 0;
    unsigned long long* tkey = nullptr;    // [8 * faces] cell keys of the grown triangle boxes
    unsigned long long* tkey_s = nullptr;
    int* tval = nullptr;
    int* tval_s = nullptr;
    unsigned long long* ekey = nullptr;    // [8 * edges]
    unsigned long long* ekey_s = nullptr;
    int* eval = nullptr;
    int* eval_s = nullptr;
    unsigned long long* bounds = nullptr;  // [8] ordered min xyz, max xyz, largest box extent
    double* grid = nullptr;                // [6] origin xyz, cell size, contact gap, error flag
    int* counts = nullptr;                 // [queries + 1]
    int* offs = nullptr;                   // [queries + 1]
    int* gflag = nullptr;                  // [surface points + 1]
    int* goff = nullptr;
    unsigned long long* reckey = nullptr;  // [records] (edge << 32 | other edge) of edge-edge records
    unsigned long long* reckey_s = nullptr;
    int* recidx = nullptr;
    int* recidx_s = nullptr;
    int4* rec_pair = nullptr;              // unsorted edge-edge records
    int4* rec_ccd = nullptr;
    unsigned long long* gscan = nullptr;   // [records] packed ranks per Hessian size
    unsigned int* d_counts = nullptr;      // [4] pairs, point-triangle pairs, ground pairs, grid error
    unsigned int* h_counts = nullptr;      // pinned copy
    void* cub = nullptr;
    size_t cub_bytes = 0;
};

}  // namespace sgipc

using namespace sgipc;

namespace {

constexpr int kCellBits = 21;
constexpr unsigned long long kNoKey = ~0ull;
constexpr int kGroupBits = 21;  // packed rank fields: three 21-bit counters in one 64-bit word
constexpr int kQueryThreads = 128;

// order-preserving map of doubles to unsigned integers (min / max by integer atomics)
__device__ __forceinline__ unsigned long long ord(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord(unsigned long long u) {
    return __longlong_as_double((long long)((u >> 63) ? (u & 0x7fffffffffffffffull) : ~u));
}

__device__ __forceinline__ d3 ldp(const double* x, unsigned v) { return {x[3 * v], x[3 * v + 1], x[3 * v + 2]}; }

// scene bounds of the surface points and the largest extent of a triangle or edge box;
// bounds[7] != 0 when an index names no vertex (nothing is loaded from such an index)
__global__ void k_bounds(const double* __restrict__ x, int nv, const unsigned* __restrict__ sv, int nsv,
                         const unsigned* __restrict__ faces, int nf, const unsigned* __restrict__ edges, int ne,
                         unsigned long long* bounds) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY}, ext = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsv + nf + ne; i += stride) {
        if (i < nsv) {
            if (sv[i] >= (unsigned)nv) {
                atomicOr(bounds + 7, 1ull);
                continue;
            }
            const d3 p = ldp(x, sv[i]);
            lo[0] = fmin(lo[0], p.x), lo[1] = fmin(lo[1], p.y), lo[2] = fmin(lo[2], p.z);
            hi[0] = fmax(hi[0], p.x), hi[1] = fmax(hi[1], p.y), hi[2] = fmax(hi[2], p.z);
        } else {
            const bool tri = i < nsv + nf;
            const int k = tri ? i - nsv : i - nsv - nf;
            const unsigned* v = tri ? faces + 3 * k : edges + 2 * k;
            if (v[0] >= (unsigned)nv || v[1] >= (unsigned)nv || (tri && v[2] >= (unsigned)nv)) {
                atomicOr(bounds + 7, 1ull);
                continue;
            }
            const d3 a = ldp(x, v[0]), b = ldp(x, v[1]), c = tri ? ldp(x, v[2]) : a;
            ext = fmax(ext, fmax(fmax(a.x, b.x), c.x) - fmin(fmin(a.x, b.x), c.x));
            ext = fmax(ext, fmax(fmax(a.y, b.y), c.y) - fmin(fmin(a.y, b.y), c.y));
            ext = fmax(ext, fmax(fmax(a.z, b.z), c.z) - fmin(fmin(a.z, b.z), c.z));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            lo[q] = fmin(lo[q], __shfl_xor_sync(0xffffffffu, lo[q], o));
            hi[q] = fmax(hi[q], __shfl_xor_sync(0xffffffffu, hi[q], o));
        }
        ext = fmax(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            atomicMin(bounds + q, ord(lo[q]));
            atomicMax(bounds + 3 + q, ord(hi[q]));
        }
        atomicMax(bounds + 6, ord(ext));
    }
}

// cell size and origin; grid[5] = 1 when the scene needs more than 2^21 cells along an axis,
// 2 when an index names no vertex (every later kernel then returns at once)
__global__ void k_grid(const unsigned long long* bounds, double gap, double* grid) {
    const double ext = unord(bounds[6]);
    const double h = (ext + 2.0 * gap) * 1.001 + 1e-12;
    int bad = 0;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const double lo = unord(bounds[q]), hi = unord(bounds[3 + q]);
        grid[q] = lo - gap - h;
        if (!(hi >= lo) || (hi - grid[q]) / h + 2.0 >= (double)(1 << kCellBits)) bad = 1;
    }
    grid[3] = h;
    grid[4] = gap;
    grid[5] = bounds[7] ? 2 : bad;
}

__device__ __forceinline__ int cell_of(double v, double o, double h) { return (int)floor((v - o) / h); }
__device__ __forceinline__ unsigned long long cell_key(int i, int j, int k) {
    return (unsigned long long)i | ((unsigned long long)j << kCellBits) | ((unsigned long long)k << (2 * kCellBits));
}

// grown box of a triangle (grow = gap) or an edge (grow = gap / 2)
struct Box {
    d3 lo, hi;
};
__device__ __forceinline__ Box grown_box(const double* x, const unsigned* v, int nvert, double grow) {
    d3 a = ldp(x, v[0]), lo = a, hi = a;
    for (int k = 1; k < nvert; k++) {
        const d3 b = ldp(x, v[k]);
        lo = {fmin(lo.x, b.x), fmin(lo.y, b.y), fmin(lo.z, b.z)};
        hi = {fmax(hi.x, b.x), fmax(hi.y, b.y), fmax(hi.z, b.z)};
    }
    return {{lo.x - grow, lo.y - grow, lo.z - grow}, {hi.x + grow, hi.y + grow, hi.z + grow}};
}

// keys of the (at most 8) cells a grown box covers; unused slots get kNoKey
__global__ void k_insert(const double* __restrict__ x, const unsigned* __restrict__ prim, int n, int nvert,
                         const double* __restrict__ grid, unsigned long long* key, int* val) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || grid[5] != 0.0) return;
    const double h = grid[3], gap = grid[4];
    const Box b = grown_box(x, prim + (size_t)nvert * p, nvert, nvert == 3 ? gap : 0.5 * gap);
    const int i0 = cell_of(b.lo.x, grid[0], h), j0 = cell_of(b.lo.y, grid[1], h), k0 = cell_of(b.lo.z, grid[2], h);
    const int i1 = cell_of(b.hi.x, grid[0], h), j1 = cell_of(b.hi.y, grid[1], h), k1 = cell_of(b.hi.z, grid[2], h);
#pragma unroll
    for (int s = 0; s < 8; s++) {
        const int i = i0 + (s & 1), j = j0 + ((s >> 1) & 1), k = k0 + (s >> 2);
        key[8 * (size_t)p + s] = (i <= i1 && j <= j1 && k <= k1) ? cell_key(i, j, k) : kNoKey;
        val[8 * (size_t)p + s] = p;
    }
}

// first index in sorted keys [0, n) not below k
__device__ __forceinline__ int lower_bound(const unsigned long long* __restrict__ keys, int n, unsigned long long k) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(keys + mid) < k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

struct PairOut {
    int4 pair, ccd;
    int group;  // 0: two vertices (6 x 6), 1: three (9 x 9), 2: four (12 x 12)
};

// _checkPTintersection (mlbvh.cu:534-645): point p against triangle (a, b, c)
__device__ __forceinline__ bool check_pt(const double* x, unsigned p, unsigned a, unsigned b, unsigned c, double dhat,
                                         PairOut& o) {
    const d3 v0 = ldp(x, p), v1 = ldp(x, a), v2 = ldp(x, b), v3 = ldp(x, c);
    const int t = pt_type(v0, v1, v2, v3);
    double d;
    switch (t) {
        case 0: d = pp_d2(v0, v1); break;
        case 1: d = pp_d2(v0, v2); break;
        case 2: d = pp_d2(v0, v3); break;
        case 3: d = pe_d2(v0, v1, v2); break;
        case 4: d = pe_d2(v0, v2, v3); break;
        case 5: d = pe_d2(v0, v3, v1); break;
        default: d = pplane_d2(v0, v1, v2, v3); break;
    }
    if (!(d < dhat)) return false;
    const int q = -(int)p - 1;
    o.ccd = make_int4(q, (int)a, (int)b, (int)c);
    switch (t) {
        case 0: o.pair = make_int4(q, (int)a, -1, -1), o.group = 0; break;
        case 1: o.pair = make_int4(q, (int)b, -1, -1), o.group = 0; break;
        case 2: o.pair = make_int4(q, (int)c, -1, -1), o.group = 0; break;
        case 3: o.pair = make_int4(q, (int)a, (int)b, -1), o.group = 1; break;
        case 4: o.pair = make_int4(q, (int)b, (int)c, -1), o.group = 1; break;
        case 5: o.pair = make_int4(q, (int)c, (int)a, -1), o.group = 1; break;
        default: o.pair = make_int4(q, (int)a, (int)b, (int)c), o.group = 2; break;
    }
    return true;
}

// _checkEEintersection (mlbvh.cu:685-1059): edge (i0, i1) against the other edge (i2, i3) of
// index other; nearly parallel edges mark their point-point / point-edge pair with
// w = -other - 2 (the mollified encodings are off in the reference, smooth = false)
__device__ __forceinline__ bool check_ee(const double* x, const double* rest, unsigned i0, unsigned i1, unsigned i2,
                                         unsigned i3, int other, double dhat, PairOut& o) {
    const d3 v0 = ldp(x, i0), v1 = ldp(x, i1), v2 = ldp(x, i2), v3 = ldp(x, i3);
    const int t = ee_type(v0, v1, v2, v3);
    double d;
    switch (t) {
        case 0: d = pp_d2(v0, v2); break;
        case 1: d = pp_d2(v0, v3); break;
        case 2: d = pe_d2(v0, v2, v3); break;
        case 3: d = pp_d2(v1, v2); break;
        case 4: d = pp_d2(v1, v3); break;
        case 5: d = pe_d2(v1, v2, v3); break;
        case 6: d = pe_d2(v2, v0, v1); break;
        case 7: d = pe_d2(v3, v0, v1); break;
        default: d = ll_d2(v0, v1, v2, v3); break;
    }
    if (!(d < dhat)) return false;
    const d3 r0 = ldp(rest, i0), r1 = ldp(rest, i1), r2 = ldp(rest, i2), r3 = ldp(rest, i3);
    const double cr = sq(cross(v0 - v1, v2 - v3));
    const double eps = 1e-3 * sq(r0 - r1) * sq(r2 - r3);
    const int add_e = cr < eps ? -other - 2 : -1;
    const int a = (int)i0, b = (int)i1, c = (int)i2, e = (int)i3;
    o.ccd = make_int4(a, b, c, e);
    switch (t) {
        case 0: o.pair = make_int4(-a - 1, c, -1, add_e), o.group = 0; break;
        case 1: o.pair = make_int4(-a - 1, e, -1, add_e), o.group = 0; break;
        case 2: o.pair = make_int4(-a - 1, c, e, add_e), o.group = 1; break;
        case 3: o.pair = make_int4(-b - 1, c, -1, add_e), o.group = 0; break;
        case 4: o.pair = make_int4(-b - 1, e, -1, add_e), o.group = 0; break;
        case 5: o.pair = make_int4(-b - 1, c, e, add_e), o.group = 1; break;
        case 6: o.pair = make_int4(-c - 1, a, b, add_e), o.group = 1; break;
        case 7: o.pair = make_int4(-e - 1, a, b, add_e), o.group = 1; break;
        default: o.pair = make_int4(a, b, c, e), o.group = 2; break;
    }
    return true;
}

struct QueryArgs {
    const double* x;
    const double* rest;
    const unsigned* sv;
    const unsigned* faces;
    const unsigned* edges;
    const int* body;
    const int* btype;
    int nsv, nf, ne;
    double dhat;
    const double* grid;
    const unsigned long long* tkey;
    const int* tval;
    const unsigned long long* ekey;
    const int* eval;
};

__device__ __forceinline__ bool all_fixed(const int* bt, unsigned a, unsigned b, unsigned c, unsigned d) {
    return bt && bt[a] >= 2 && bt[b] >= 2 && bt[c] >= 2 && bt[d] >= 2;
}

// Query q < nsv: surface point sv[q] against the triangles of its cell; q >= nsv: edge q - nsv
// against the edges of its grown box's cells.  kWrite = false counts into counts[q]; true
// writes the records from offs[q] on (edge-edge ones to the unsorted record buffers).
template <bool kWrite>
__global__ void k_query(QueryArgs a, int* counts, const int* offs, int4* pairs, int4* ccd, int* group,
                        int4* rec_pair, int4* rec_ccd, unsigned long long* reckey, int* recidx) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.nsv + a.ne || a.grid[5] != 0.0) return;
    const double h = a.grid[3], gap = a.grid[4];
    int found = 0;
    const int base = kWrite ? offs[q] : 0;
    PairOut o;
    if (q < a.nsv) {
        const unsigned p = a.sv[q];
        const d3 xp = ldp(a.x, p);
        const unsigned long long key = cell_key(cell_of(xp.x, a.grid[0], h), cell_of(xp.y, a.grid[1], h),
                                                cell_of(xp.z, a.grid[2], h));
        const int n8 = 8 * a.nf;
        for (int k = lower_bound(a.tkey, n8, key); k < n8 && __ldg(a.tkey + k) == key; k++) {
            const int f = __ldg(a.tval + k);
            const unsigned t0 = a.faces[3 * f], t1 = a.faces[3 * f + 1], t2 = a.faces[3 * f + 2];
            // _selfQuery_vf's filters (mlbvh.cu:1350-1362)
            if (!(a.body[p] != a.body[t0] || a.body[p] == -1)) continue;
            if (p == t0 || p == t1 || p == t2) continue;
            if (all_fixed(a.btype, p, t0, t1, t2)) continue;
            if (!check_pt(a.x, p, t0, t1, t2, a.dhat, o)) continue;
            if (kWrite) {
                pairs[base + found] = o.pair;
                ccd[base + found] = o.ccd;
                group[base + found] = o.group;
            }
            found++;
        }
    } else {
        const int s = q - a.nsv;
        const unsigned e0 = a.edges[2 * s], e1 = a.edges[2 * s + 1];
        const Box bs = grown_box(a.x, a.edges + 2 * s, 2, 0.5 * gap);
        const int i0 = cell_of(bs.lo.x, a.grid[0], h), j0 = cell_of(bs.lo.y, a.grid[1], h), k0 = cell_of(bs.lo.z, a.grid[2], h);
        const int i1 = cell_of(bs.hi.x, a.grid[0], h), j1 = cell_of(bs.hi.y, a.grid[1], h), k1 = cell_of(bs.hi.z, a.grid[2], h);
        const int n8 = 8 * a.ne;
        for (int c = 0; c < 8; c++) {
            const int ci = i0 + (c & 1), cj = j0 + ((c >> 1) & 1), ck = k0 + (c >> 2);
            if (ci > i1 || cj > j1 || ck > k1) continue;
            const unsigned long long key = cell_key(ci, cj, ck);
            for (int k = lower_bound(a.ekey, n8, key); k < n8 && __ldg(a.ekey + k) == key; k++) {
                const int other = __ldg(a.eval + k);
                if (other <= s) continue;  // each pair once, as (edge, larger edge) (mlbvh.cu:1550-1560)
                const Box bo = grown_box(a.x, a.edges + 2 * other, 2, 0.5 * gap);
                if (bo.lo.x > bs.hi.x || bs.lo.x > bo.hi.x || bo.lo.y > bs.hi.y || bs.lo.y > bo.hi.y ||
                    bo.lo.z > bs.hi.z || bs.lo.z > bo.hi.z)
                    continue;
                // the one cell that reports this pair: the one holding the overlap's low corner
                if (cell_of(fmax(bs.lo.x, bo.lo.x), a.grid[0], h) != ci ||
                    cell_of(fmax(bs.lo.y, bo.lo.y), a.grid[1], h) != cj ||
                    cell_of(fmax(bs.lo.z, bo.lo.z), a.grid[2], h) != ck)
                    continue;
                const unsigned f0 = a.edges[2 * other], f1 = a.edges[2 * other + 1];
                // _selfQuery_ee's filters (mlbvh.cu:1550-1566)
                if (!(a.body[e0] != a.body[f0] || a.body[e0] == -1)) continue;
                if (e0 == f0 || e0 == f1 || e1 == f0 || e1 == f1) continue;
                if (all_fixed(a.btype, e0, e1, f0, f1)) continue;
                if (!check_ee(a.x, a.rest, e0, e1, f0, f1, other, a.dhat, o)) continue;
                if (kWrite) {
                    const int r = base + found - offs[a.nsv];  // position among the edge-edge records
                    rec_pair[r] = o.pair;
                    rec_ccd[r] = o.ccd;
                    reckey[r] = ((unsigned long long)s << 32) | (unsigned)other;
                    recidx[r] = r;
                }
                found++;
            }
        }
    }
    if (!kWrite) counts[q] = found;
}

// edge-edge records in (edge, other edge) order after the sort; their Hessian-size group
__global__ void k_gather_ee(int n, int first, const int* __restrict__ idx, const int4* __restrict__ rp,
                            const int4* __restrict__ rc, int4* pairs, int4* ccd, int* group) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int r = idx[k];
    const int4 p = rp[r];
    pairs[first + k] = p;
    ccd[first + k] = rc[r];
    // point-point (z < 0, w at most -1), point-edge (w < 0), or edge-edge
    group[first + k] = p.x >= 0 ? 2 : (p.z < 0 ? 0 : 1);
}

__global__ void k_group_flags(int n, const int* __restrict__ group, unsigned long long* flags) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) flags[k] = 1ull << (kGroupBits * group[k]);
}

// MatIndex = rank among the pairs of the same group; cp_num = total, 0, per-group counts
__global__ void k_mat_index(int n, int* mat_index, const unsigned long long* __restrict__ flags,
                            const unsigned long long* __restrict__ scan, unsigned* cp_num) {
    // mat_index holds the group codes on entry; each thread rewrites only its own entry
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long m = (1ull << kGroupBits) - 1;
    if (k < n) mat_index[k] = (int)((scan[k] >> (kGroupBits * mat_index[k])) & m);
    if (k == 0) {
        const unsigned long long last = n > 0 ? scan[n - 1] + flags[n - 1] : 0ull;
        cp_num[0] = (unsigned)n;
        cp_num[1] = 0;
        for (int g = 0; g < 3; g++) cp_num[2 + g] = (unsigned)((last >> (kGroupBits * g)) & m);
    }
}

// _GroundCollisionDetect (GIPC.cu:6433-6450): surface points with (n.x - offset)^2 <= dHat
__global__ void k_ground_flags(const double* __restrict__ x, const unsigned* __restrict__ sv, int nsv, double offset,
                               double dhat, const double* __restrict__ grid, int* flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsv || grid[5] != 0.0) return;
    const double dist = x[3 * sv[i] + 1] - offset;  // normal +y
    flag[i] = dist * dist > dhat ? 0 : 1;
}
__global__ void k_ground_write(const unsigned* __restrict__ sv, int nsv, const int* __restrict__ flag,
                               const int* __restrict__ off, unsigned* out, unsigned* gp_num) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nsv && flag[i]) out[off[i]] = sv[i];
    if (i == nsv - 1) *gp_num = (unsigned)(off[i] + flag[i]);
}

__global__ void k_counts_out(const int* offs, int nsv, int nq, const int* goff, const int* gflag,
                             const double* grid, unsigned* counts) {
    unsigned* h_counts = counts;
    h_counts[0] = (unsigned)offs[nq];
    h_counts[1] = (unsigned)offs[nsv];
    h_counts[2] = nsv > 0 ? (unsigned)(goff[nsv - 1] + gflag[nsv - 1]) : 0u;
    h_counts[3] = (unsigned)grid[5];
}

// ------------------------------------------------------------------------------------------
// lagged friction set-up
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ d3 normalized(d3 v) {
    const double inv = 1.0 / sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x * inv, v.y * inv, v.z * inv};
}

// 2 x 2 inverse by Gauss-Jordan elimination with the reference's pivot rule (an entry below
// 1e-15 in magnitude is replaced by adding a later row; __Inverse2x2, gpu_eigen_libs.cu:1342-1411);
// a singular matrix gives zeros
__device__ inline void inverse2x2(const double A[2][2], double R[2][2]) {
    double m[2][4] = {{A[0][0], A[0][1], 1.0, 0.0}, {A[1][0], A[1][1], 0.0, 1.0}};
    R[0][0] = R[0][1] = R[1][0] = R[1][1] = 0.0;
    for (int i = 0; i < 2; i++) {
        if (fabs(m[i][i]) < 1e-15) {
            int j = i + 1;
            for (; j < 2; j++)
                if (fabs(m[j][i]) > 1e-15) break;
            if (j == 2) return;
            for (int r = i; r < 4; r++) m[i][r] += m[j][r];
        }
        const double ep = m[i][i];
        for (int r = i; r < 4; r++) m[i][r] /= ep;
        for (int j = i + 1; j < 2; j++) {
            const double e = -1 * (m[j][i] / m[i][i]);
            for (int r = i; r < 4; r++) m[j][r] += e * m[i][r];
        }
    }
    for (int i = 1; i >= 0; i--)
        for (int j = i - 1; j >= 0; j--) {
            const double e = -1 * (m[j][i] / m[i][i]);
            for (int r = i; r < 4; r++) m[j][r] += e * m[i][r];
        }
    for (int i = 0; i < 2; i++) R[i][0] = m[i][2], R[i][1] = m[i][3];
}

// (first tangent, second tangent) stored as the columns of a row-major 3 x 2 basis
__device__ __forceinline__ void store_basis(double* B, d3 c0, d3 c1) {
    B[0] = c0.x, B[1] = c1.x, B[2] = c0.y, B[3] = c1.y, B[4] = c0.z, B[5] = c1.z;
}

__device__ __forceinline__ bool in_mesh(int v, int nv) { return v >= 0 && v < nv; }

// flags: 1 when pair k takes part in friction (not mollified); a pair naming a vertex
// outside the mesh is left out and raises bad[0]
__global__ void k_fric_flags(const int4* __restrict__ pairs, int n, int nv, int* flag, unsigned* bad) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int4 p = pairs[k];
    int f;
    bool ok;
    if (p.x >= 0) {
        f = p.w >= 0;
        ok = !f || (in_mesh(p.x, nv) && in_mesh(p.y, nv) && in_mesh(p.z, nv) && in_mesh(p.w, nv));
    } else if (p.z < 0) {
        f = p.y >= 0;
        ok = !f || (in_mesh(-p.x - 1, nv) && in_mesh(p.y, nv));
    } else if (p.w < 0) {
        f = p.y >= 0;
        ok = !f || (in_mesh(-p.x - 1, nv) && in_mesh(p.y, nv) && in_mesh(p.z, nv));
    } else {
        f = 1;
        ok = in_mesh(-p.x - 1, nv) && in_mesh(p.y, nv) && in_mesh(p.z, nv) && in_mesh(p.w, nv);
    }
    if (!ok) {
        f = 0;
        atomicOr(bad, 1u);
    }
    flag[k] = f;
}

// _calFrictionLastH_DistAndTan (GIPC.cu:8388-8499) with the closest points and tangent bases
// of FrictionUtils.cuh:52-399; the lagged normal force is that of the RANK-2 barrier
__global__ void k_fric_setup(const double* __restrict__ x, const int4* __restrict__ pairs, int n,
                             const int* __restrict__ flag, const int* __restrict__ off, double dhat, double kappa,
                             int4* out_pairs, double* lambda, double* coord, double* basis, unsigned* cp_num_last) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || !flag[k]) return;
    const int4 p = pairs[k];
    const int o = off[k];
    double dis, c0 = 0.0, c1 = 0.0;
    double* B = basis + 6 * (size_t)o;
    int group;
    if (p.x >= 0) {  // edge-edge
        const d3 v0 = ldp(x, p.x), v1 = ldp(x, p.y), v2 = ldp(x, p.z), v3 = ldp(x, p.w);
        dis = ll_d2(v0, v1, v2, v3);
        const d3 e20 = v0 - v2, e01 = v1 - v0, e23 = v3 - v2;
        const double A[2][2] = {{sq(e01), -dot(e23, e01)}, {-dot(e23, e01), sq(e23)}};
        double R[2][2];
        inverse2x2(A, R);
        const double r0 = -dot(e20, e01), r1 = dot(e20, e23);
        c0 = R[0][0] * r0 + R[0][1] * r1;
        c1 = R[1][0] * r0 + R[1][1] * r1;
        store_basis(B, normalized(e01), normalized(cross(cross(e01, e23), e01)));
        group = 2;
    } else {
        const unsigned v = (unsigned)(-p.x - 1);
        const d3 v0 = ldp(x, v), v1 = ldp(x, p.y);
        if (p.z < 0) {  // point-point
            dis = pp_d2(v0, v1);
            const d3 v01 = v1 - v0;
            const d3 xc = {0.0, -v01.z, v01.y}, yc = {v01.z, 0.0, -v01.x};
            const d3 t0 = sq(xc) > sq(yc) ? xc : yc;
            store_basis(B, normalized(t0), normalized(cross(v01, t0)));
            group = 0;
        } else if (p.w < 0) {  // point-edge
            const d3 v2 = ldp(x, p.z);
            dis = pe_d2(v0, v1, v2);
            const d3 e12 = v2 - v1;
            c0 = dot(v0 - v1, e12) / sq(e12);
            store_basis(B, normalized(e12), normalized(cross(e12, v0 - v1)));
            group = 1;
        } else {  // point-triangle
            const d3 v2 = ldp(x, p.z), v3 = ldp(x, p.w);
            dis = pplane_d2(v0, v1, v2, v3);
            const d3 v12 = v2 - v1, v13 = v3 - v1, v10 = v0 - v1;
            const double A[2][2] = {{v12.x * v12.x + v12.y * v12.y + v12.z * v12.z, v12.x * v13.x + v12.y * v13.y + v12.z * v13.z},
                                    {v13.x * v12.x + v13.y * v12.y + v13.z * v12.z, v13.x * v13.x + v13.y * v13.y + v13.z * v13.z}};
            double R[2][2];
            inverse2x2(A, R);
            const double b0 = v12.x * v10.x + v12.y * v10.y + v12.z * v10.z;
            const double b1 = v13.x * v10.x + v13.y * v10.y + v13.z * v10.z;
            c0 = R[0][0] * b0 + R[0][1] * b1;
            c1 = R[1][0] * b0 + R[1][1] * b1;
            store_basis(B, normalized(v12), normalized(cross(cross(v12, v13), v12)));
            group = 2;
        }
    }
    const double l = log(dis / dhat);
    lambda[o] = -kappa * 2.0 * sqrt(dis) * (l * l * (2 * dis - 2 * dhat) + (2 * l * (dis - dhat) * (dis - dhat)) / dis);
    coord[2 * (size_t)o] = c0;
    coord[2 * (size_t)o + 1] = c1;
    out_pairs[o] = p;
    // integer counts: the same totals in any order
    atomicAdd(cp_num_last, 1u);
    atomicAdd(cp_num_last + 2 + group, 1u);
}

// _calFrictionLastH_gd (GIPC.cu:8362-8386): the ground pairs' normal forces (the RANK-1 form
// of the ground barrier, as the reference writes it)
__global__ void k_fric_ground(const double* __restrict__ x, int nv, const unsigned* __restrict__ gp, int n,
                              double offset, double dhat, double kappa, double* lambda, unsigned* out, unsigned* bad) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const unsigned g = gp[k];
    if (g >= (unsigned)nv) {
        atomicOr(bad, 1u);
        lambda[k] = 0.0;
        out[k] = g;
        return;
    }
    const double dist = x[3 * g + 1] - offset;
    const double dist2 = dist * dist;
    const double t = dist2 - dhat;
    const double g_b = t * log(dist2 / dhat) * -2.0 - (t * t) / dist2;
    lambda[k] = -kappa * 2.0 * sqrt(dist2) * g_b;
    out[k] = g;
}

// buffers for nsv points, nf triangles, ne edges and cap records
SgipcStatus broad_reserve(SgipcCtx* c, int nsv, int nf, int ne, int cap) {
    if (!c->broad) {
        c->broad = new BroadWork();
        BroadWork& w = *c->broad;
        SG_CHECK(c, cudaMalloc((void**)&w.bounds, sizeof(unsigned long long) * 8));
        SG_CHECK(c, cudaMalloc((void**)&w.grid, sizeof(double) * 8));
        SG_CHECK(c, cudaMalloc((void**)&w.d_counts, sizeof(unsigned) * 4));
        SG_CHECK(c, cudaMallocHost((void**)&w.h_counts, sizeof(unsigned) * 4));
    }
    BroadWork& w = *c->broad;
    bool cub_again = false;
    if (8 * nf > w.cap_tri) {
        const int m = 8 * nf;
        for (unsigned long long** p : {&w.tkey, &w.tkey_s}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(unsigned long long) * (size_t)(m > 0 ? m : 1)));
        }
        for (int** p : {&w.tval, &w.tval_s}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(int) * (size_t)(m > 0 ? m : 1)));
        }
        w.cap_tri = m;
        cub_again = true;
    }
    if (8 * ne > w.cap_edge) {
        const int m = 8 * ne;
        for (unsigned long long** p : {&w.ekey, &w.ekey_s}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(unsigned long long) * (size_t)(m > 0 ? m : 1)));
        }
        for (int** p : {&w.eval, &w.eval_s}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(int) * (size_t)(m > 0 ? m : 1)));
        }
        w.cap_edge = m;
        cub_again = true;
    }
    if (nsv + ne + 1 > w.cap_q) {
        const int m = nsv + ne + 1;
        for (int** p : {&w.counts, &w.offs}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(int) * (size_t)m));
        }
        w.cap_q = m;
        cub_again = true;
    }
    if (nsv + 1 > w.cap_sv) {
        const int m = nsv + 1;
        for (int** p : {&w.gflag, &w.goff}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(int) * (size_t)m));
        }
        w.cap_sv = m;
        cub_again = true;
    }
    if (cap > w.cap_rec) {
        const int m = cap > 1 ? cap : 1;
        for (unsigned long long** p : {&w.reckey, &w.reckey_s, &w.gscan}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(unsigned long long) * (size_t)m));
        }
        for (int** p : {&w.recidx, &w.recidx_s}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(int) * (size_t)m));
        }
        for (int4** p : {&w.rec_pair, &w.rec_ccd}) {
            if (*p) cudaFree(*p);
            SG_CHECK(c, cudaMalloc((void**)p, sizeof(int4) * (size_t)m));
        }
        w.cap_rec = m;
        cub_again = true;
    }
    if (cub_again) {
        size_t b = 0, t = 0;
        SG_CHECK(c, cub::DeviceRadixSort::SortPairs(nullptr, t, w.tkey, w.tkey_s, w.tval, w.tval_s, w.cap_tri));
        b = t > b ? t : b;
        SG_CHECK(c, cub::DeviceRadixSort::SortPairs(nullptr, t, w.ekey, w.ekey_s, w.eval, w.eval_s, w.cap_edge));
        b = t > b ? t : b;
        SG_CHECK(c, cub::DeviceRadixSort::SortPairs(nullptr, t, w.reckey, w.reckey_s, w.recidx, w.recidx_s,
                                                    w.cap_rec));
        b = t > b ? t : b;
        SG_CHECK(c, cub::DeviceScan::ExclusiveSum(nullptr, t, w.counts, w.offs, w.cap_q));
        b = t > b ? t : b;
        SG_CHECK(c, cub::DeviceScan::ExclusiveSum(nullptr, t, w.gscan, w.gscan, w.cap_rec));
        b = t > b ? t : b;
        if (b > w.cub_bytes) {
            if (w.cub) cudaFree(w.cub);
            SG_CHECK(c, cudaMalloc(&w.cub, b));
            w.cub_bytes = b;
        }
    }
    return SGIPC_OK;
}

}  // namespace

namespace sgipc {
void broad_destroy(SgipcCtx* c) {
    if (!c->broad) return;
    BroadWork& w = *c->broad;
    void* ps[] = {w.tkey, w.tkey_s, w.tval, w.tval_s, w.ekey, w.ekey_s, w.eval, w.eval_s, w.bounds, w.grid, w.d_counts,
                  w.counts, w.offs, w.gflag, w.goff, w.reckey, w.reckey_s, w.recidx, w.recidx_s, w.rec_pair,
                  w.rec_ccd, w.gscan, w.cub};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (w.h_counts) cudaFreeHost(w.h_counts);
    delete c->broad;
    c->broad = nullptr;
}
}  // namespace sgipc

extern "C" SgipcStatus sgipc_build_cp(SgipcCtx* c, const double* x, const double* rest, const SgipcSurface* surf,
                                      const int32_t* body_id, const int32_t* boundary_type, double dHat,
                                      double ground_offset, int32_t cap, int32_t* pairs, int32_t* ccd_pairs,
                                      int32_t* mat_index, uint32_t* cp_num, int32_t ground_cap, uint32_t* ground_pairs,
                                      uint32_t* gp_num, uint32_t* h_cp_num, uint32_t* h_gp_num, void* stream) {
    if (!c || !x || !rest || !surf || !body_id || !pairs || !ccd_pairs || !mat_index || !cp_num || !ground_pairs ||
        !gp_num || !h_cp_num || !h_gp_num || cap < 0 || ground_cap < 0 || !(dHat > 0.0))
        return SGIPC_BAD_INPUT;
    const int nsv = surf->surf_vert_num, nf = surf->face_num, ne = surf->edge_num;
    if (nsv < 0 || nf < 0 || ne < 0 || (nsv && !surf->surf_verts) || (nf && !surf->faces) || (ne && !surf->edges))
        return SGIPC_BAD_INPUT;
    if (cap >= (1 << kGroupBits)) {
        snprintf(c->err, sizeof(c->err), "build_cp: capacity %d beyond the %d pairs one call ranks", cap,
                 (1 << kGroupBits) - 1);
        return SGIPC_BAD_INPUT;
    }
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    SgipcStatus st = broad_reserve(c, nsv, nf, ne, cap);
    if (st != SGIPC_OK) return st;
    BroadWork& w = *c->broad;
    const int nq = nsv + ne;
    const double gap = sqrt(dHat);
    // bounds: min entries start at the largest key, max entries at 0
    SG_CHECK(c, cudaMemsetAsync(w.bounds, 0xff, sizeof(unsigned long long) * 3, s));
    SG_CHECK(c, cudaMemsetAsync(w.bounds + 3, 0, sizeof(unsigned long long) * 5, s));  // and the index flag
    SG_COUNT(c, 1);
    k_bounds<<<148, 256, 0, s>>>(x, c->nv, surf->surf_verts, nsv, surf->faces, nf, surf->edges, ne, w.bounds);
    SG_COUNT(c, 1);
    k_grid<<<1, 1, 0, s>>>(w.bounds, gap, w.grid);
    if (nf > 0) {
        SG_COUNT(c, 1);
        k_insert<<<nblk(nf), SGIPC_BLOCK, 0, s>>>(x, surf->faces, nf, 3, w.grid, w.tkey, w.tval);
        size_t t = w.cub_bytes;
        SG_CHECK(c, cub::DeviceRadixSort::SortPairs(w.cub, t, w.tkey, w.tkey_s, w.tval, w.tval_s, 8 * nf, 0, 64, s));
    }
    if (ne > 0) {
        SG_COUNT(c, 1);
        k_insert<<<nblk(ne), SGIPC_BLOCK, 0, s>>>(x, surf->edges, ne, 2, w.grid, w.ekey, w.eval);
        size_t t = w.cub_bytes;
        SG_CHECK(c, cub::DeviceRadixSort::SortPairs(w.cub, t, w.ekey, w.ekey_s, w.eval, w.eval_s, 8 * ne, 0, 64, s));
    }
    QueryArgs qa{x, rest, surf->surf_verts, surf->faces, surf->edges, body_id, boundary_type, nsv, nf, ne, dHat,
                 w.grid, w.tkey_s, w.tval_s, w.ekey_s, w.eval_s};
    SG_CHECK(c, cudaMemsetAsync(w.counts, 0, sizeof(int) * (size_t)(nq + 1), s));
    if (nq > 0) {
        SG_COUNT(c, 1);
        k_query<false><<<nblk(nq, kQueryThreads), kQueryThreads, 0, s>>>(qa, w.counts, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                nullptr, nullptr);
    }
    size_t t = w.cub_bytes;
    SG_CHECK(c, cub::DeviceScan::ExclusiveSum(w.cub, t, w.counts, w.offs, nq + 1, s));
    SG_CHECK(c, cudaMemsetAsync(w.gflag, 0, sizeof(int) * (size_t)(nsv + 1), s));
    if (nsv > 0) {
        SG_COUNT(c, 1);
        k_ground_flags<<<nblk(nsv), SGIPC_BLOCK, 0, s>>>(x, surf->surf_verts, nsv, ground_offset, dHat, w.grid,
                                                         w.gflag);
    }
    t = w.cub_bytes;
    SG_CHECK(c, cub::DeviceScan::ExclusiveSum(w.cub, t, w.gflag, w.goff, nsv + 1, s));
    SG_COUNT(c, 1);
    k_counts_out<<<1, 1, 0, s>>>(w.offs, nsv, nq, w.goff, w.gflag, w.grid, w.d_counts);
    SG_CHECK(c, cudaMemcpyAsync(w.h_counts, w.d_counts, sizeof(unsigned) * 4, cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    const int total = (int)w.h_counts[0], npt = (int)w.h_counts[1], ng = (int)w.h_counts[2];
    for (int k = 0; k < 5; k++) h_cp_num[k] = 0;
    h_cp_num[0] = (unsigned)total;
    *h_gp_num = (unsigned)ng;
    if (w.h_counts[3] == 2) {
        snprintf(c->err, sizeof(c->err), "build_cp: a surface point, triangle or edge names a vertex outside the mesh");
        return SGIPC_BAD_INPUT;
    }
    if (w.h_counts[3]) {
        snprintf(c->err, sizeof(c->err), "build_cp: the scene spans more than 2^%d grid cells along an axis",
                 kCellBits);
        return SGIPC_BAD_INPUT;
    }
    if (total > cap || ng > ground_cap) {
        snprintf(c->err, sizeof(c->err), "build_cp: %d pairs for capacity %d, %d ground pairs for capacity %d",
                 total, cap, ng, ground_cap);
        return SGIPC_CAPACITY;
    }
    int4* P = reinterpret_cast<int4*>(pairs);
    int4* Q = reinterpret_cast<int4*>(ccd_pairs);
    // group codes of the final order, kept in gscan (an int per record fits) until they move to
    // mat_index; gscan then takes the packed flags
    int* group = reinterpret_cast<int*>(w.gscan);
    if (nq > 0) {
        SG_COUNT(c, 1);
        k_query<true><<<nblk(nq, kQueryThreads), kQueryThreads, 0, s>>>(qa, nullptr, w.offs, P, Q, group, w.rec_pair, w.rec_ccd, w.reckey,
                                               w.recidx);
    }
    const int nee = total - npt;
    if (nee > 0) {
        t = w.cub_bytes;
        SG_CHECK(c, cub::DeviceRadixSort::SortPairs(w.cub, t, w.reckey, w.reckey_s, w.recidx, w.recidx_s, nee, 0, 64,
                                                    s));
        SG_COUNT(c, 1);
        k_gather_ee<<<nblk(nee), SGIPC_BLOCK, 0, s>>>(nee, npt, w.recidx_s, w.rec_pair, w.rec_ccd, P, Q, group);
    }
    // ranks per Hessian size: the group codes move to mat_index first (gscan is rewritten)
    if (total > 0) {
        SG_CHECK(c, cudaMemcpyAsync(mat_index, group, sizeof(int) * (size_t)total, cudaMemcpyDeviceToDevice, s));
        SG_COUNT(c, 1);
        k_group_flags<<<nblk(total), SGIPC_BLOCK, 0, s>>>(total, mat_index, w.gscan);
        t = w.cub_bytes;
        SG_CHECK(c, cub::DeviceScan::ExclusiveSum(w.cub, t, w.gscan, w.reckey, total, s));
    }
    SG_COUNT(c, 1);
    k_mat_index<<<nblk(total > 0 ? total : 1), SGIPC_BLOCK, 0, s>>>(total, mat_index, w.gscan, w.reckey, cp_num);
    if (nsv > 0) {
        SG_COUNT(c, 1);
        k_ground_write<<<nblk(nsv), SGIPC_BLOCK, 0, s>>>(surf->surf_verts, nsv, w.gflag, w.goff, ground_pairs, gp_num);
    } else {
        SG_CHECK(c, cudaMemsetAsync(gp_num, 0, sizeof(unsigned), s));
    }
    SG_LAUNCH_CHECK(c, "build_cp");
    SG_CHECK(c, cudaMemcpyAsync(h_cp_num, cp_num, sizeof(unsigned) * 5, cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_friction_setup(SgipcCtx* c, const double* x, const int32_t* pairs, int32_t pair_num,
                                            const uint32_t* ground_pairs, int32_t ground_num, double dHat,
                                            double kappa, double ground_offset, int32_t* fric_pairs,
                                            double* fric_lambda, double* fric_coord, double* fric_basis,
                                            uint32_t* cp_num_last, uint32_t* fric_gd_pairs, double* fric_gd_lambda,
                                            uint32_t* h_cp_num_last, void* stream) {
    if (!c || !x || pair_num < 0 || ground_num < 0 || !(dHat > 0.0) || !cp_num_last)
        return SGIPC_BAD_INPUT;
    if (pair_num > 0 && (!pairs || !fric_pairs || !fric_lambda || !fric_coord || !fric_basis)) return SGIPC_BAD_INPUT;
    if (ground_num > 0 && (!ground_pairs || !fric_gd_pairs || !fric_gd_lambda)) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    SgipcStatus st = broad_reserve(c, pair_num, 0, 0, pair_num);  // flags / offsets over the pairs
    if (st != SGIPC_OK) return st;
    BroadWork& w = *c->broad;
    SG_CHECK(c, cudaMemsetAsync(cp_num_last, 0, sizeof(unsigned) * 5, s));
    if (pair_num > 0) {
        const int4* P = reinterpret_cast<const int4*>(pairs);
        SG_COUNT(c, 2);
        k_fric_flags<<<nblk(pair_num), SGIPC_BLOCK, 0, s>>>(P, pair_num, c->nv, w.gflag, cp_num_last + 1);
        size_t t = w.cub_bytes;
        SG_CHECK(c, cub::DeviceScan::ExclusiveSum(w.cub, t, w.gflag, w.goff, pair_num, s));
        k_fric_setup<<<nblk(pair_num), SGIPC_BLOCK, 0, s>>>(x, P, pair_num, w.gflag, w.goff, dHat, kappa,
                                                            reinterpret_cast<int4*>(fric_pairs), fric_lambda,
                                                            fric_coord, fric_basis, cp_num_last);
    }
    if (ground_num > 0) {
        SG_COUNT(c, 1);
        k_fric_ground<<<nblk(ground_num), SGIPC_BLOCK, 0, s>>>(x, c->nv, ground_pairs, ground_num, ground_offset, dHat,
                                                               kappa, fric_gd_lambda, fric_gd_pairs, cp_num_last + 1);
    }
    SG_LAUNCH_CHECK(c, "friction_setup");
    if (h_cp_num_last) {
        SG_CHECK(c, cudaMemcpyAsync(h_cp_num_last, cp_num_last, sizeof(unsigned) * 5, cudaMemcpyDeviceToHost, s));
        SG_CHECK(c, cudaStreamSynchronize(s));
        if (h_cp_num_last[1]) {
            snprintf(c->err, sizeof(c->err), "friction_setup: a pair or ground pair names a vertex outside the mesh");
            return SGIPC_BAD_INPUT;
        }
    }
    return SGIPC_OK;
}
