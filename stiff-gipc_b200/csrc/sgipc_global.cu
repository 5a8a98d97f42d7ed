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
// summed in a fixed order (no atomics).  The loop is host-driven with device dot products
// (two scalar reads per iteration, as the reference's): the coupled system is the
// secondary path next to the persistent FEM solve.
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

__global__ void k_g_update(long long n, double alpha, const double* __restrict__ p, const double* __restrict__ Ap,
                           double* __restrict__ x, double* __restrict__ r) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] += alpha * p[i];
    r[i] -= alpha * Ap[i];
}

__global__ void k_g_direction(long long n, double beta, const double* __restrict__ z, double* __restrict__ p) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = z[i] + beta * p[i];
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

SgipcStatus g_dot(const Global& g, const double* u, const double* v, double* out) {
    SgipcStatus st = dot64(g.f, u, v, (int)g.N, g.a->g_dot, g.s);
    if (st != SGIPC_OK) return st;
    SG_CHECK(g.f, cudaMemcpyAsync(g.f->h_pinned, g.a->g_dot, sizeof(double), cudaMemcpyDeviceToHost, g.s));
    SG_CHECK(g.f, cudaStreamSynchronize(g.s));
    *out = g.f->h_pinned[0];
    return SGIPC_OK;
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
        if ((st = grow(f, &a->g_vec, 4 * (size_t)g.N)) || (st = grow(f, &a->g_dot, 8))) return st;
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
    SG_CHECK(f, cudaMemsetAsync(x, 0, sizeof(double) * g.N, g.s));
    SG_CHECK(f, cudaMemcpyAsync(r, b, sizeof(double) * g.N, cudaMemcpyDeviceToDevice, g.s));
    if ((st = g_precond(g, r, z))) return st;
    double rz0 = 0, bn2 = 0;
    if ((st = g_dot(g, r, z, &rz0))) return st;
    if ((st = g_dot(g, b, b, &bn2))) return st;
    SG_CHECK(f, cudaMemcpyAsync(p, z, sizeof(double) * g.N, cudaMemcpyDeviceToDevice, g.s));
    double rz = rz0;
    int iters = 0, status = SGIPC_OK;
    bool running = rz0 > 0.0 && std::isfinite(rz0);
    if (!running && (!std::isfinite(rz0) || rz0 < 0.0)) status = SGIPC_BREAKDOWN;
    for (int k = 1; running && k < max_iter; k++) {
        if ((st = g_spmv(g, p, Ap))) return st;
        double pAp = 0;
        if ((st = g_dot(g, p, Ap, &pAp))) return st;
        iters = k;
        if (!(pAp > 0.0) || !std::isfinite(pAp)) {
            status = SGIPC_BREAKDOWN;
            running = false;
            break;
        }
        const double alpha = rz / pAp;
        // the reference tests the r.z of the current iterate and stops after its update
        bool stop = crit == SGIPC_CRIT_RZ && std::fabs(rz) <= tol * rz0;
        SG_COUNT(f, 1);
        k_g_update<<<gb, SGIPC_BLOCK, 0, g.s>>>(g.N, alpha, p, Ap, x, r);
        if (crit == SGIPC_CRIT_TRUE) {
            double rr = 0;
            if ((st = g_dot(g, r, r, &rr))) return st;
            stop = rr <= tol * tol * bn2;
        }
        if (stop) {
            running = false;
            break;
        }
        if (k + 1 >= max_iter) break;
        if ((st = g_precond(g, r, z))) return st;
        double rz_new = 0;
        if ((st = g_dot(g, r, z, &rz_new))) return st;
        const double beta = rz_new / rz;
        rz = rz_new;
        SG_COUNT(f, 1);
        k_g_direction<<<gb, SGIPC_BLOCK, 0, g.s>>>(g.N, beta, z, p);
    }
    if (running && status == SGIPC_OK) status = SGIPC_NOT_CONVERGED;  // the iteration cap
    SG_LAUNCH_CHECK(f, "global pcg");
    // ---- true residual, distribute_solution
    double rel = 0;
    if ((st = g_spmv(g, x, Ap))) return st;
    SG_COUNT(f, 1);
    k_g_residual<<<gb, SGIPC_BLOCK, 0, g.s>>>(g.N, b, Ap);
    double res2 = 0;
    if ((st = g_dot(g, Ap, Ap, &res2))) return st;
    rel = bn2 > 0 ? std::sqrt(res2 / bn2) : std::sqrt(res2);
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
