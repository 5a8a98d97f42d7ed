// sgipc_global.cu — the global FEM + ABD linear system: one PCG over [ABD | FEM] DOFs.
//
// Semantics of StiffGIPC's GlobalLinearSystem with its two subsystems (gipc/gipc.cu:42-70):
// the ABD subsystem comes first (12 DOFs = 4 block rows per body), the FEM subsystem after
// it (3 DOFs per vertex), offsets by an exclusive scan of the subsystem sizes
// (global_linear_system.cu:8-74).  The matrix is the symmetric upper BCOO of both
// (global_linear_system.cu:182-199, spmv.cu): here the FEM context's assembled matrix on
// the FEM rows and the ABD context's merged body-space blocks (body rows, and body x FEM
// coupling in FEM columns) used with their transposes.  The preconditioner is the identity
// overwritten by each local preconditioner on its own range (apply_preconditioner,
// global_linear_system.cu:152-166): ABDPreconditioner (12x12 block Jacobi) on the body
// rows, MAS_Preconditioner on the FEM rows.  PCGSolver::pcg (pcg_solver.cu:174-267) with
// its stop rule.  distribute_solution (global_linear_system.cu:76-87) hands the FEM part
// back as the FEM move direction and maps every body's dq to its points:
// dx = J(x_bar) dq (ABDLinearSubsystem::retrieve_solution, abd_linear_subsystem.cu:33-56,
// cal_x_from_q.cu:34-66 forms J q - J (q - dq), the same quantity).
//
// B200 layout: the FEM rows run the FEM context's SpMV and MAS unchanged; the body rows
// (a few thousand block rows at the C4 size) are one thread per block row over the row-
// sorted merged blocks and a column-sorted index of their transposes, so every output is
// summed in a fixed order (no atomics).  The loop's scalars (alpha, beta, the stop tests) live on
// the device: small kernels compute them from the dot products and the vector kernels read
// them, so the host reads the state back once per iteration, after the update and its stop
// tests (the reference reads two scalars back per iteration).  Enqueuing several iterations per
// read-back (the kernels after a stop return at once) measured slower on the affine-body bed:
// its solves take about six iterations, and the preconditioner and SpMV of the iterations past
// the stop cost more than the read-backs saved.
#include <cub/cub.cuh>

#include "sgipc_abd_ctx.cuh"

using namespace sgipc;

namespace {

__device__ __forceinline__ int lower_bound_i(const int* a, int n, int v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ int lower_bound_k(const unsigned long long* a, int n, unsigned long long v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// rptr[r] = first merged block of body row r (blocks are sorted by (row, col))
__global__ void k_g_rowptr(int nrows, const int* __restrict__ nu, const int* __restrict__ u_row, int* __restrict__ rptr) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r <= nrows) rptr[r] = lower_bound_i(u_row, nu[0], r);
}

// transposed index: the off-diagonal blocks keyed by (col, row); diagonal blocks and unused
// slots sort past every column
__global__ void k_g_tkeys(int cap, const int* __restrict__ nu, const int* __restrict__ u_row,
                          const int* __restrict__ u_col, unsigned long long* __restrict__ key, int* __restrict__ idx) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cap) return;
    const bool off = k < nu[0] && u_row[k] != u_col[k];
    key[k] = off ? (((unsigned long long)(unsigned)u_col[k] << 32) | (unsigned)u_row[k]) : ~0ull;
    idx[k] = k;
}

__global__ void k_g_colptr(int ncols, int m, const unsigned long long* __restrict__ key_s, int* __restrict__ cptr) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= ncols) cptr[c] = lower_bound_k(key_s, m, (unsigned long long)(unsigned)c << 32);
}

__device__ __forceinline__ void block_mv(const double* V, const double* x, double (&y)[3]) {
    y[0] += V[0] * x[0] + V[1] * x[1] + V[2] * x[2];
    y[1] += V[3] * x[0] + V[4] * x[1] + V[5] * x[2];
    y[2] += V[6] * x[0] + V[7] * x[1] + V[8] * x[2];
}

__device__ __forceinline__ void block_mtv(const double* V, const double* x, double (&y)[3]) {
    y[0] += V[0] * x[0] + V[3] * x[1] + V[6] * x[2];
    y[1] += V[1] * x[0] + V[4] * x[1] + V[7] * x[2];
    y[2] += V[2] * x[0] + V[5] * x[1] + V[8] * x[2];
}

// y[r] for the body rows: the row's blocks times x, then the transposed blocks whose column
// is r (global block indices; x, y global vectors)
__global__ void k_g_body_rows(int nrows, const int* __restrict__ rptr, const int* __restrict__ cptr,
                              const int* __restrict__ tidx, const int* __restrict__ u_row,
                              const int* __restrict__ u_col, const double* __restrict__ u_val,
                              const double* __restrict__ x, double* __restrict__ y) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrows) return;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int k = rptr[r]; k < rptr[r + 1]; k++) block_mv(u_val + 9 * (size_t)k, x + 3 * (size_t)u_col[k], acc);
    for (int j = cptr[r]; j < cptr[r + 1]; j++) {
        const int k = tidx[j];
        block_mtv(u_val + 9 * (size_t)k, x + 3 * (size_t)u_row[k], acc);
    }
    for (int q = 0; q < 3; q++) y[3 * (size_t)r + q] = acc[q];
}

// FEM rows: add the transposed coupling blocks (body row, FEM column) to the FEM SpMV's y
__global__ void k_g_fem_coupling(int nfem, int off, const int* __restrict__ cptr, const int* __restrict__ tidx,
                                 const int* __restrict__ u_row, const double* __restrict__ u_val,
                                 const double* __restrict__ x, double* __restrict__ y) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nfem) return;
    const int c = off + v;
    const int j0 = cptr[c], j1 = cptr[c + 1];
    if (j0 == j1) return;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int j = j0; j < j1; j++) {
        const int k = tidx[j];
        block_mtv(u_val + 9 * (size_t)k, x + 3 * (size_t)u_row[k], acc);
    }
    for (int q = 0; q < 3; q++) y[3 * (size_t)c + q] += acc[q];
}

// Device state of the loop (PCGSolver::pcg's scalars).  halt: 0 running, 1 stopped (converged
// or broken down), 2 stopped at the iteration cap.
struct GState {
    double rz0, rz, bn2, alpha, beta;
    int iters, halt, status, stop;
};
// dot-product slots: d[0] p.Ap, d[1] r.r, d[2] r.z (new), d[3] r0.z0, d[4] b.b, d[5] residual^2;
// the state from d + kStateOff
constexpr int kStateOff = 16;

__global__ void k_g_start(GState* st, const double* __restrict__ d) {
    const double rz0 = d[3];
    const bool run = rz0 > 0.0 && isfinite(rz0);
    st->rz0 = st->rz = rz0;
    st->bn2 = d[4];
    st->alpha = st->beta = 0.0;
    st->iters = 0;
    st->stop = 0;
    st->halt = run ? 0 : 1;
    st->status = (!run && (!isfinite(rz0) || rz0 < 0.0)) ? SGIPC_BREAKDOWN : SGIPC_OK;
}

// alpha = r.z / p.Ap of iteration k; the r.z test of the current iterate (the reference stops
// after this iteration's update)
__global__ void k_g_alpha(GState* st, const double* __restrict__ d, int k, int crit, double tol) {
    if (st->halt) return;
    const double pAp = d[0];
    st->iters = k;
    if (!(pAp > 0.0) || !isfinite(pAp)) {
        st->status = SGIPC_BREAKDOWN;
        st->halt = 1;
        return;
    }
    st->alpha = st->rz / pAp;
    st->stop = crit == SGIPC_CRIT_RZ && fabs(st->rz) <= tol * st->rz0;
}

// after the update: the true-residual test, or the r.z one decided before it; the cap
__global__ void k_g_after(GState* st, const double* __restrict__ d, int k, int crit, double tol, int max_iter) {
    if (st->halt) return;
    const bool stop = crit == SGIPC_CRIT_TRUE ? d[1] <= tol * tol * st->bn2 : st->stop != 0;
    if (stop) st->halt = 1;
    else if (k + 1 >= max_iter) st->halt = 2;
}

__global__ void k_g_beta(GState* st, const double* __restrict__ d) {
    if (st->halt) return;
    const double rz_new = d[2];
    st->beta = rz_new / st->rz;
    st->rz = rz_new;
}

__global__ void k_g_update(long long n, const GState* __restrict__ st, const double* __restrict__ p,
                           const double* __restrict__ Ap, double* __restrict__ x, double* __restrict__ r) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || st->halt) return;
    const double alpha = st->alpha;
    x[i] += alpha * p[i];
    r[i] -= alpha * Ap[i];
}

__global__ void k_g_direction(long long n, const GState* __restrict__ st, const double* __restrict__ z,
                              double* __restrict__ p) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !st->halt) p[i] = z[i] + st->beta * p[i];
}

__global__ void k_g_residual(long long n, const double* __restrict__ b, double* __restrict__ y) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = b[i] - y[i];
}

// dx of every ABD point: J(x_bar) dq of its body (translation + x_bar . da_r per row)
__global__ void k_g_point_dx(int P, const int* __restrict__ point_body, const double* __restrict__ x_bar,
                             const double* __restrict__ dq, double* __restrict__ dx) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const double* q = dq + 12 * (size_t)point_body[p];
    const double* xb = x_bar + 3 * (size_t)p;
    for (int r = 0; r < 3; r++)
        dx[3 * (size_t)p + r] = q[r] + xb[0] * q[3 + 3 * r] + xb[1] * q[4 + 3 * r] + xb[2] * q[5 + 3 * r];
}

template <class T>
SgipcStatus grow(SgipcCtx* f, T** p, size_t n) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    SG_CHECK(f, cudaMalloc((void**)p, sizeof(T) * (n > 0 ? n : 1)));
    return SGIPC_OK;
}

struct Global {
    SgipcCtx* f;
    SgipcAbdCtx* a;
    int nb;     // body block rows 4B
    int nfem;   // FEM block rows
    long long N;
    cudaStream_t s;
    int fp32_mas;
};

// y = A x over the global vector
SgipcStatus g_spmv(const Global& g, const double* x, double* y) {
    SgipcAbdCtx* a = g.a;
    SgipcStatus st = spmv_t<double>(g.f, x + 3 * (size_t)g.nb, y + 3 * (size_t)g.nb, g.s);
    if (st != SGIPC_OK) return st;
    SG_COUNT(g.f, 2);
    k_g_body_rows<<<nblk(g.nb, 128), 128, 0, g.s>>>(g.nb, a->g_rptr, a->g_cptr, a->g_tidx_s, a->u_row, a->u_col,
                                                     a->u_val, x, y);
    k_g_fem_coupling<<<nblk(g.nfem), SGIPC_BLOCK, 0, g.s>>>(g.nfem, g.nb, a->g_cptr, a->g_tidx_s, a->u_row,
                                                             a->u_val, x, y);
    SG_LAUNCH_CHECK(g.f, "global spmv");
    return SGIPC_OK;
}

// z = M^-1 r: ABD block Jacobi on the body rows, MAS on the FEM rows
SgipcStatus g_precond(const Global& g, const double* r, double* z) {
    SG_COUNT(g.f, 1);
    abd_precond_apply_async(g.a, r, z, g.s);
    SG_LAUNCH_CHECK(g.f, "abd block jacobi");
    return mas_apply_t<double>(g.f, r + 3 * (size_t)g.nb, z + 3 * (size_t)g.nb, g.fp32_mas, g.s);
}

// u . v into the device slot d[slot] (no read-back)
SgipcStatus g_dot(const Global& g, const double* u, const double* v, int slot) {
    return dot64(g.f, u, v, (int)g.N, g.a->g_dot + slot, g.s);
}

}  // namespace

extern "C" SgipcStatus sgipc_global_pcg_solve(SgipcCtx* f, SgipcAbdCtx* a, SgipcCriterion crit, double tol,
                                              int32_t max_iter, const double* b, double* x, double* abd_point_dx,
                                              SgipcSolveStats* stats, void* stream) {
    if (!f || !a || !b || !x || !(tol >= 0.0)) return SGIPC_BAD_INPUT;
    if (crit != SGIPC_CRIT_RZ && crit != SGIPC_CRIT_TRUE) return SGIPC_BAD_INPUT;
    if (a->device != f->device) {
        snprintf(f->err, sizeof(f->err), "global solve: the FEM and ABD contexts live on different devices");
        return SGIPC_BAD_INPUT;
    }
    if (!f->assembled || !f->mas.built || !a->assembled || !a->pbuilt) {
        snprintf(f->err, sizeof(f->err), "global solve: assemble both systems and build both preconditioners first");
        return SGIPC_NOT_READY;
    }
    SG_DEVICE(f);
    Global g{f, a, 4 * a->B, f->n, 3LL * (4LL * a->B + f->n), (cudaStream_t)stream, f->mas.built == SGIPC_FP64 + 1 ? 0 : 1};
    if (g.N > 0x7fffffffLL) return SGIPC_CAPACITY;
    if (max_iter <= 0) max_iter = (int)(0.3 * (double)g.N);
    if (max_iter < 2) max_iter = 2;
    // ---- buffers (grown on demand) and the merged blocks' row / column index
    int nu = 0;
    SG_CHECK(f, cudaMemcpyAsync(&nu, a->nu, sizeof(int), cudaMemcpyDeviceToHost, g.s));
    SG_CHECK(f, cudaStreamSynchronize(g.s));
    SgipcStatus st;
    const int ncols = g.nb + g.nfem;
    if (a->g_cap_blk < a->cap) {
        if ((st = grow(f, &a->g_tkey, a->cap)) || (st = grow(f, &a->g_tkey_s, a->cap)) ||
            (st = grow(f, &a->g_tidx, a->cap)) || (st = grow(f, &a->g_tidx_s, a->cap)))
            return st;
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, a->g_tkey, a->g_tkey_s, a->g_tidx, a->g_tidx_s, a->cap);
        if ((st = grow(f, (char**)&a->g_cub, tb))) return st;
        a->g_cub_bytes = tb;
        a->g_cap_blk = a->cap;
    }
    if (a->g_cap_ptr < ncols + 1) {
        if ((st = grow(f, &a->g_rptr, g.nb + 1)) || (st = grow(f, &a->g_cptr, ncols + 1))) return st;
        a->g_cap_ptr = ncols + 1;
    }
    if (a->g_cap_vec < (size_t)g.N) {
        if ((st = grow(f, &a->g_vec, 4 * (size_t)g.N)) || (st = grow(f, &a->g_dot, 32))) return st;
        a->g_cap_vec = (size_t)g.N;
    }
    SG_COUNT(f, 3);
    k_g_rowptr<<<nblk(g.nb + 1), SGIPC_BLOCK, 0, g.s>>>(g.nb, a->nu, a->u_row, a->g_rptr);
    k_g_tkeys<<<nblk(a->cap), SGIPC_BLOCK, 0, g.s>>>(a->cap, a->nu, a->u_row, a->u_col, a->g_tkey, a->g_tidx);
    size_t tb = a->g_cub_bytes;
    SG_CHECK(f, cub::DeviceRadixSort::SortPairs(a->g_cub, tb, a->g_tkey, a->g_tkey_s, a->g_tidx, a->g_tidx_s,
                                                nu > 0 ? nu : 1, 0, 64, g.s));
    k_g_colptr<<<nblk(ncols + 1), SGIPC_BLOCK, 0, g.s>>>(ncols, nu, a->g_tkey_s, a->g_cptr);
    SG_LAUNCH_CHECK(f, "global index");

    // ---- PCG (PCGSolver::pcg semantics, as the persistent FEM solve)
    double* r = a->g_vec;
    double* z = r + g.N;
    double* p = z + g.N;
    double* Ap = p + g.N;
    const int gb = nblk(g.N);
    double* d = a->g_dot;
    GState* gst = reinterpret_cast<GState*>(d + kStateOff);
    SG_CHECK(f, cudaMemsetAsync(x, 0, sizeof(double) * g.N, g.s));
    SG_CHECK(f, cudaMemcpyAsync(r, b, sizeof(double) * g.N, cudaMemcpyDeviceToDevice, g.s));
    if ((st = g_precond(g, r, z))) return st;
    if ((st = g_dot(g, r, z, 3)) || (st = g_dot(g, b, b, 4))) return st;
    SG_CHECK(f, cudaMemcpyAsync(p, z, sizeof(double) * g.N, cudaMemcpyDeviceToDevice, g.s));
    SG_COUNT(f, 1);
    k_g_start<<<1, 1, 0, g.s>>>(gst, d);
    GState hs{};
    SG_CHECK(f, cudaMemcpyAsync(&hs, gst, sizeof(hs), cudaMemcpyDeviceToHost, g.s));
    SG_CHECK(f, cudaStreamSynchronize(g.s));
    for (int k = 1; !hs.halt && k < max_iter; k++) {
        if ((st = g_spmv(g, p, Ap)) || (st = g_dot(g, p, Ap, 0))) return st;
        SG_COUNT(f, 2);
        k_g_alpha<<<1, 1, 0, g.s>>>(gst, d, k, (int)crit, tol);
        k_g_update<<<gb, SGIPC_BLOCK, 0, g.s>>>(g.N, gst, p, Ap, x, r);
        if (crit == SGIPC_CRIT_TRUE && (st = g_dot(g, r, r, 1))) return st;
        SG_COUNT(f, 1);
        k_g_after<<<1, 1, 0, g.s>>>(gst, d, k, (int)crit, tol, max_iter);
        SG_LAUNCH_CHECK(f, "global pcg");
        // the one read-back of the iteration: stopped (converged, broken down, at the cap)?
        SG_CHECK(f, cudaMemcpyAsync(&hs, gst, sizeof(hs), cudaMemcpyDeviceToHost, g.s));
        SG_CHECK(f, cudaStreamSynchronize(g.s));
        if (hs.halt) break;
        if ((st = g_precond(g, r, z)) || (st = g_dot(g, r, z, 2))) return st;
        SG_COUNT(f, 2);
        k_g_beta<<<1, 1, 0, g.s>>>(gst, d);
        k_g_direction<<<gb, SGIPC_BLOCK, 0, g.s>>>(g.N, gst, z, p);
    }
    int status = hs.status;
    // still running at the cap: not converged
    if (status == SGIPC_OK && hs.halt != 1) status = SGIPC_NOT_CONVERGED;
    // ---- true residual, distribute_solution
    if ((st = g_spmv(g, x, Ap))) return st;
    SG_COUNT(f, 1);
    k_g_residual<<<gb, SGIPC_BLOCK, 0, g.s>>>(g.N, b, Ap);
    if ((st = g_dot(g, Ap, Ap, 5))) return st;
    SG_CHECK(f, cudaMemcpyAsync(f->h_pinned, d + 5, sizeof(double), cudaMemcpyDeviceToHost, g.s));
    SG_CHECK(f, cudaStreamSynchronize(g.s));
    const double res2 = f->h_pinned[0], bn2 = hs.bn2;
    const double rel = bn2 > 0 ? std::sqrt(res2 / bn2) : std::sqrt(res2);
    const double rz0 = hs.rz0, rz = hs.rz;
    const int iters = hs.iters;
    if (abd_point_dx && a->P > 0) {
        SG_COUNT(f, 1);
        k_g_point_dx<<<nblk(a->P), SGIPC_BLOCK, 0, g.s>>>(a->P, a->point_body, a->x_bar, x, abd_point_dx);
        SG_LAUNCH_CHECK(f, "abd point dx");
    }
    if (stats) {
        *stats = SgipcSolveStats{};
        stats->iterations = iters;
        stats->rz0 = rz0;
        stats->rz = rz;
        stats->rel_residual = rel;
        stats->status = status;
    }
    return (SgipcStatus)status;
}
