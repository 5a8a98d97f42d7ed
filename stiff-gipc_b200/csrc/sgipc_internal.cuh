// sgipc_internal.cuh — context layout shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/sgipc.h"
#include "sgipc_math.cuh"

#define SGIPC_BANK 16
#define SGIPC_MAX_LEVELS 6
#define SGIPC_BLOCK 256

namespace sgipc {

struct BroadWork;  // buffers of the contact-pair search (sgipc_broad.cu)

// Device-resident PCG scalars (no host round trip per iteration).
struct PcgScalars {
    double rz;        // r.z of the current iterate (reference: rz)
    double rz_next;   // r.z after the latest preconditioner apply (rz_new)
    double rz0;
    double pAp;
    double alpha;
    double tol;
    double bnorm2;    // ||b||^2 (true-residual criterion)
    double rr;        // ||r||^2 of the current iterate
    int32_t iter;     // SpMVs performed
    int32_t max_iter;
    int32_t state;    // 0 running, 1 stop after this update, 2 stopped
    int32_t status;   // SgipcStatus
    int32_t crit;     // SgipcCriterion
    int32_t bodies;   // iteration bodies executed (hard bound on the graph's while loop)
    int32_t first;    // 1 until the first SpMV (p = z, no beta)
    int32_t pcur;     // which of the two p buffers holds the current direction
    int32_t halt;     // [rhs 0 only] set once the loop must stop; later bodies return at once
    int32_t input_flag;  // persistent solve: the assembly's bad-input flag, copied at its end
    double rz_ref;    // refinement epilogue: r64 . M r64 and r64 . r64 of the FP64 residual
    double rr_ref;
};

// Mixed-precision refinement run by the persistent FP32 solve as its epilogue: x64 += x,
// r64 = b64 - A x64 (FP64 matrix), then r64 . M r64 (FP32 MAS) and r64 . r64 into the
// solve's scalars.  done = true when the epilogue ran (else the caller refines itself).
struct RefineArgs {
    double* x64;
    const double* b64;
    double* r64;
    bool done;
    bool assign;  // first refinement: x64 = x (x64 is not read before)
};

// One precision's PCG workspace (T = double or float) for up to `nrhs` right-hand sides.
struct PcgWork {
    void* x;
    void* r;
    void* r2;                // second residual buffer of the persistent solve
    void* z;
    void* p;
    void* p2;                // second direction buffer (the SpMV forms p = z + beta p_old on the fly)
    void* Ap;
    void* Ap2;               // second A p buffer of the fused persistent solve
    void* w;                 // w = A z of the fused persistent solve
    PcgScalars* sc;          // [nrhs]
    double* partial;         // reduction partials [nrhs][max_blocks]
    unsigned int* ticket;    // [0..3] last-block counters; [4..5] grid barrier of the persistent solve
    double* coop;            // persistent solve: block partials [2][3 nrhs][coop_cap]
    int coop_cap;            // largest grid the persistent solve may use
    bool last_coop;          // the latest solve ran as the persistent kernel (its scalars carry input_flag)
    cudaGraphExec_t exec;    // captured iteration loop
    bool cond_graph;         // true: while-node graph (whole loop in one launch)
    long long captured_key;  // precision/rhs tag and domain count the graph was captured for
};

struct MasWork {
    int npos;                // level-0 positions (padded to 16)
    int levelnum;
    int total_cap;           // cluster capacity = levelnum * npos
    int* part_map;           // [npos] position -> vertex or -1
    int* real_map;           // [nv]
    int* nbr_ptr;            // [nv+1] mesh neighbour CSR
    int* nbr;                // [nnz]
    int* nbr_row;            // [nnz] vertex of each neighbour slot
    int nnbr;                // nnz
    int* table;              // [nv * levelnum] global cluster per level (level 0 = position)
    int* up;                 // [total_cap] global id of each cluster's parent at the next level (-1: none)
    int* node;               // [nv] node id at the level being built
    uint32_t* mask;          // [npos] bank-local connectivity
    int* comp_rank;          // [npos] new local id of the component a node belongs to
    int* bank_cnt;           // [npos/16 + 1]
    int* bank_off;           // [npos/16 + 1]
    int* map0;               // [npos/16 * 256] static slot of each level-0 domain entry (a, b):
                             //   s + 1 (block s), -(s + 1) (its transpose), 0 (none)
    int* l1_first;           // [npos/16 + 2] per level-1 bank: first and last level-0 bank holding
    int* l1_last;            //   one of its nodes' positions (levels >= 3)
    int* info;               // device: [0..7] level starts, [8..15] level counts, [16] total
    int h_info[17];          // host copy after build
    double* dom64;           // [total_cap/16][48*48] FP64 domain matrices / inverses
    float* dom32;            // [total_cap/16][48*48] FP32 inverses
    double* R64;             // [total_cap*3]
    double* Z64;
    float* R32;
    float* Z32;
    void* scan_tmp;
    size_t scan_tmp_bytes;
    int built;               // 0 none, else SgipcPrecision+1 of the stored inverses
    // hierarchy prebuilt by sgipc_assemble on `side` (it needs the contacts only, not the
    // matrix), overlapping the assembly; consumed by the next mas_build with the same pairs
    cudaStream_t side;
    cudaEvent_t ev_start, ev_hier;
    // static blocks scattered into the domains on `side` once the hierarchy and the static
    // matrix are ready (ev_static: static matrix written on the caller's stream; ev_pre: the
    // scatter done), overlapping the contact merge; consumed with the prebuilt hierarchy
    cudaEvent_t ev_static, ev_pre;
    int pre_scattered;
    int* h_info_pinned;      // [32] pinned landing area of the level counts (and [21]: abort)
    int* hier_part;          // [32] chunk totals of the fused hierarchy kernel's scan
    int hier_grid;           // CTAs of the fused hierarchy kernel (0: per-level kernels), -1 unset
    int hier_pending;
    const void* hier_pairs;
    int hier_pair_num;
};

}  // namespace sgipc

struct SgipcCtx {
    int device;
    int nv, nt, nf, nh, nsoft;
    int n;                    // block rows
    int max_pairs, max_ground, max_fric, max_fric_gd, max_rhs;
    char err[512];

    // ---- static symmetric-upper BSR ---------------------------------------------------
    int nnz;                  // static blocks (upper incl. diagonal)
    int* row_ptr;             // [n+1]
    int* col;                 // [nnz]
    int* slot_row;            // [nnz]
    int* diag_slot;           // [n]
    int* low_ptr;             // [n+1] lower (transposed) entries per row
    int* low_slot;            // [nnz - n]
    double* val64;            // [nnz*9]
    // full symmetric copy of the static blocks (both triangles) for the SpMV
    int nnz_full;             // 2*nnz - n
    int* frow_ptr;            // [n+1]
    int* h_frow_ptr;          // host copy (sizes the persistent solve's shared-memory residency)
    int* fcol;                // [nnz_full]
    int* fup;                 // [nnz] full index of upper slot s
    int* flo;                 // [nnz] full index of its transpose (-1 on the diagonal)
    double* fval64;           // [nnz_full*9]
    float* fval32;            // [nnz_full*9]
    // element blocks and their gather lists
    int n_eblk;               // 10 per tet, 6 per triangle, 10 per hinge
    double* eblk;             // [n_eblk*9] oriented element blocks
    int* contrib_ptr;         // [nnz+1]
    int* contrib;             // [n_eblk] element block ids sorted by slot
    int n_egrad;              // 4 per tet, 3 per triangle, 4 per hinge
    double* egrad;            // [n_egrad*3]
    int* vinc_ptr;            // [nv+1]
    int* vinc;                // [n_egrad] element gradient rows per vertex
    // topology
    uint32_t* tets;           // [nt*4]
    uint32_t* tris;           // [nf*3]
    uint32_t* hinges;         // [nh*2]
    int32_t* hinge_adj;       // [nh*2]
    uint32_t* soft_idx;       // [nsoft]
    // gradients and right-hand side
    double* shape_grads;      // [3nv]
    double* fb;               // [3nv]
    double* b;                // [3n]
    const int32_t* btype;     // last assembly's BoundaryType (caller-owned, device)

    // ---- dynamic contact blocks -------------------------------------------------------
    int cap_cblk;
    unsigned long long* ckey;     // [cap]
    unsigned long long* ckey_s;   // sorted
    int* cidx;                    // [cap]
    int* cidx_s;
    double* cval;                 // [cap*9]
    int* run_start;               // [cap+1] first sorted index of each unique block's run
    int* cflag;                   // [cap+1] segment heads -> unique ids
    int* nuc;                     // device: number of unique contact blocks
    int* uc_row;                  // [cap]
    int* uc_col;
    double* uc64;                 // [cap*9]
    float* uc32;
    int* cu_ptr;                  // [n+1] unique contact blocks by row (upper)
    int* cl_ptr;                  // [n+1] transposed entries by row
    int* cl_idx;                  // [cap] unique block of each transposed slot, in placement order
    int* cl_col;                  // [cap] column of each transposed entry (= uc_row of its block)
    double* cl64;                 // [cap*9] transposed copy of the block (SpMV reads it directly)
    float* cl32;
    int* lcount;                  // [2n+1] transposed entries per row [0, n], then fill cursors [n+1, 2n]
    int* lpos;                    // [cap] transposed slot of each unique block (-1: diagonal)
    void* cub_tmp;
    size_t cub_tmp_bytes;
    int key_bits;
    int assembled;
    int* dflag;                   // device: input errors found by kernels (bit 0: pair index)
    double* en_part;              // [en_cap] per-CTA partial sums of the line-search energy terms
    int en_cap;
    double* en_terms;             // [16] device: the nine terms and their total
    unsigned int* en_ticket;      // [1] device: CTAs of the energy launch done (0 between launches)
    double* h_en;                 // [16] pinned landing area of en_terms ([12], [13]: step sizes)
    double* ccd_part;             // [592] per-CTA maxima of the step-size kernels
    double* ccd_out;              // [2] the step (or speed) and the out-of-range flag
    int* ccd_bad;                 // [1] a candidate with an out-of-range vertex (0 between launches)
    unsigned int* ccd_ticket;     // [1] CTAs of a step-size launch done (0 between launches)
    // last inputs (for re-timing kernels against the current state)
    SgipcFemData last_fem;
    SgipcContacts last_con;
    SgipcParams last_prm;
    int last_has_con;
    SgipcContacts mas_con;        // contacts of the last MAS build (to rebuild after timing)
    int mas_has_con;
    long long launches;           // kernels of this library launched on the context
    sgipc::BroadWork* broad;      // contact-pair search buffers, made on its first call
    // polls a grid-barrier wait of the persistent solve or the hierarchy build makes before
    // it gives up (0: the kernels' defaults, about 2 s); sgipc_set_wait_limit
    long long wait_limit;
    // phase profile of the persistent solve (sgipc_profile_pcg; nullptr otherwise)
    unsigned long long* stamps;
    int stamp_epochs;
    // launch configuration of the persistent solve per (T, M, NR) instance, computed on its
    // first use (it depends on the device and the static pattern only)
    struct CoopCfg {
        int valid, usable, grid, ecap, kcap, dcap, ccap, zextra;
        size_t dyn;
    } coop_cfg[6], fused_cfg[6];
    // column sets of the fused persistent solve, built with the static pattern for a grid of
    // cs_grid CTAs of 128 rows: per CTA the sorted distinct columns of its rows
    // (cs_cols[cs_ptr[c] .. cs_ptr[c+1])), each full-pattern entry's slot among them
    // (cs_lcol) and each row's own slot (cs_dslot); cs_cap = the largest set
    // close constraints of the barrier-stiffness update (sgipc_close_record / _check): the
    // ground vertices and the pairs closer than dTol at the last record, with their values;
    // close_cnt [4] device counters (ground, pairs, the check's flag), close_num their host copy
    uint32_t* close_gid;
    double* close_gval;
    void* close_pid;  // int4
    double* close_pval;
    unsigned int* close_cnt;
    int close_num[2];
    int* cs_ptr;
    int* cs_cols;
    int* cs_lcol;
    int* cs_dslot;
    int cs_grid;
    int cs_cap;

    // ---- MAS and PCG ------------------------------------------------------------------
    sgipc::MasWork mas;
    sgipc::PcgWork pcg64;
    sgipc::PcgWork pcg32;
    double* tmp64;            // [3n * max_rhs] scratch vectors
    double* tmp64b;
    double* dot_partial;      // reduction scratch
    unsigned int* dot_ticket;
    double* dot_out;          // [16]
    double* h_pinned;         // host pinned scalars
    cudaStream_t cap_stream;  // capture stream
    // assembly: the contact kernels and their merge run on asm_stream beside the element
    // kernels on the caller's stream (joined before the right-hand side)
    cudaStream_t asm_stream;
    cudaEvent_t ev_asm[3];
    int max_blocks;           // reduction grid cap
};

namespace sgipc {

inline SgipcStatus cuda_fail(SgipcCtx* c, cudaError_t e, const char* what) {
    if (c) snprintf(c->err, sizeof(c->err), "%s: %s", what, cudaGetErrorString(e));
    return SGIPC_CUDA_ERROR;
}

#define SG_CHECK(ctx, call)                                          \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return sgipc::cuda_fail(ctx, e_, #call); \
    } while (0)

#define SG_LAUNCH_CHECK(ctx, name)                                   \
    do {                                                             \
        cudaError_t e_ = cudaGetLastError();                         \
        if (e_ != cudaSuccess) return sgipc::cuda_fail(ctx, e_, name); \
    } while (0)

// Makes `dev` current for the rest of the scope and gives the caller's current device back
// when the scope ends, so an entry point never leaves another device selected for its host.
struct DeviceScope {
    int prev = -1;
    bool switched = false;
    cudaError_t err;
    explicit DeviceScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        err = (prev == dev) ? cudaSuccess : cudaSetDevice(dev);
        switched = (prev != dev) && err == cudaSuccess;
    }
    ~DeviceScope() {
        if (switched && prev >= 0) cudaSetDevice(prev);
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
};

#define SG_DEVICE(ctx)                                                           \
    sgipc::DeviceScope sg_device_scope_((ctx)->device);                          \
    if (sg_device_scope_.err != cudaSuccess)                                     \
        return sgipc::cuda_fail(ctx, sg_device_scope_.err, "cudaSetDevice")

// Vector loads.  kL2 = true reads through L2 only (ld.global.cg): required for vectors that
// other CTAs of the same (persistent) kernel wrote, which a non-coherent L1 line could hide.
template <bool kL2, class T>
__device__ __forceinline__ T ldv(const T* p) {
    if constexpr (kL2)
        return __ldcg(p);
    else
        return *p;
}

// The NR right-hand-side values of one (row, component) are contiguous ([(3 v + q) * NR + r]):
// four floats move as one 16-byte access, four doubles as two (the arrays are allocation-
// aligned and 3 v + q steps by 16 or 32 bytes); other widths move as scalars.
template <bool kL2, class T, int NR>
__device__ __forceinline__ void ldn(const T* p, T (&v)[NR]) {
    if constexpr (NR == 4 && sizeof(T) == 4) {
        const float4 q = kL2 ? __ldcg(reinterpret_cast<const float4*>(p)) : *reinterpret_cast<const float4*>(p);
        v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
    } else if constexpr (NR == 4 && sizeof(T) == 8) {
        const double2* d = reinterpret_cast<const double2*>(p);
        const double2 q0 = kL2 ? __ldcg(d) : d[0], q1 = kL2 ? __ldcg(d + 1) : d[1];
        v[0] = q0.x, v[1] = q0.y, v[2] = q1.x, v[3] = q1.y;
    } else {
#pragma unroll
        for (int r = 0; r < NR; r++) v[r] = ldv<kL2>(p + r);
    }
}

template <class T, int NR>
__device__ __forceinline__ void stn(T* p, const T (&v)[NR]) {
    if constexpr (NR == 4 && sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (NR == 4 && sizeof(T) == 8) {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    } else {
#pragma unroll
        for (int r = 0; r < NR; r++) p[r] = v[r];
    }
}

inline int nblk(long long n, int b = SGIPC_BLOCK) { return (int)((n + b - 1) / b); }

// count `k` kernel launches of this library on the context
#define SG_COUNT(ctx, k) ((ctx)->launches += (k))

// Per-unit hooks for sgipc_time_kernel: launch the named kernel once against the current
// state; *bytes receives its algorithmic bytes per launch.  Returns SGIPC_NOT_READY when
// the unit does not own the name.
SgipcStatus assemble_time_hook(SgipcCtx* c, const char* name, cudaStream_t s, double* bytes);
SgipcStatus mas_time_hook(SgipcCtx* c, const char* name, cudaStream_t s, double* bytes);
SgipcStatus pcg_time_hook(SgipcCtx* c, const char* name, cudaStream_t s, double* bytes);

// ---- cross-unit entry points ------------------------------------------------------------
SgipcStatus mas_create(SgipcCtx* c, const SgipcTopology* t);
void broad_destroy(SgipcCtx* c);
void mas_destroy(SgipcCtx* c);
SgipcStatus mas_build(SgipcCtx* c, const SgipcContacts* con, SgipcPrecision prec, cudaStream_t s);
// Start the hierarchy for these contacts on the MAS side stream, after the work queued on
// s so far (called by sgipc_assemble: the hierarchy needs no matrix values).
SgipcStatus mas_prebuild(SgipcCtx* c, const SgipcContacts* con, cudaStream_t s);
// Record the point of s after which the side stream may rewrite the hierarchy.
SgipcStatus mas_mark_start(SgipcCtx* c, cudaStream_t s);
// after the static matrix is written on s: scatter it into the prebuilt hierarchy's domains
SgipcStatus mas_prescatter(SgipcCtx* c, cudaStream_t s);
// z = M^-1 r for T in {double, float}; r, z are [3n] vectors of T (rz accumulated into
// out_dot[0] when out_dot != nullptr, using r . z with r in T precision).
template <class T>
SgipcStatus mas_apply_t(SgipcCtx* c, const T* r, T* z, int fp32_inv, cudaStream_t s);
SgipcStatus pcg_create(SgipcCtx* c);
void pcg_destroy(SgipcCtx* c);
template <class T>
SgipcStatus spmv_t(SgipcCtx* c, const T* x, T* y, cudaStream_t s);
SgipcStatus dot64(SgipcCtx* c, const double* a, const double* b, int n, double* out_dev, cudaStream_t s);
// The whole PCG solve as one cooperative (persistent) kernel; *used = false when the device
// cannot co-schedule it (the caller then runs the graph of per-phase kernels).
template <class T, class M, int NR>
SgipcStatus run_pcg_coop(SgipcCtx* c, PcgWork& w, int fp32_mas, const double* b, double tol, int max_iter, int crit,
                         cudaStream_t s, bool* used, RefineArgs* ref = nullptr);
// largest grid run_pcg_coop launches on `device` (sizes its reduction buffers)
int coop_max_grid(int device);
// BAD_INPUT if a kernel flagged an invalid input since the last check (synchronises)
SgipcStatus check_device_flag(SgipcCtx* c, cudaStream_t s);

}  // namespace sgipc
