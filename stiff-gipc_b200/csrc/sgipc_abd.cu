// sgipc_abd.cu — affine-body (ABD) gradients, Hessians and the ABD block-Jacobi
// preconditioner.
//
// Semantics of StiffGIPC's ABDSystem / ABDPreconditioner:
//   q = [p; a1; a2; a3] per body, a point with body-frame position x_bar sits at
//   x = J(x_bar) q = p + (x_bar.a1, x_bar.a2, x_bar.a3) (abd_jacobi_matrix.inl);
//   body energy: kinetic M (q - q_tilde) with the lumped dyadic mass M = sum m J^T J
//   (abd_jacobi_matrix.inl, abd_system.cu:527-600) and the orthogonality potential
//   kappa v dt^2 V_perp, V_perp = sum_i (a_i.a_i - 1)^2 + sum_{i != j} (a_i.a_j)^2, whose
//   9x9 Hessian is projected to PSD (abd_energy.inl:9-127, setup...cu:186-289);
//   contacts: point gradients g -> J^T g, point blocks H_ij -> J_i^T H_ij J_j between
//   bodies and J_i^T H_ij between a body and a FEM vertex (setup...cu:349-610);
//   preconditioner: the inverse of each body's 12x12 diagonal block (setup...cu:612-655).
// The B200 version: one thread per body for the body terms (the 9x9 projection by cyclic
// Jacobi in registers / local memory), one thread per point block for the mappings, a
// deterministic per-body gather of point gradients (points are numbered body by body), a
// keyed radix-sort merge of the body-space blocks, Gauss-Jordan inverses per body.
#include <cub/cub.cuh>
#include <vector>

#include "sgipc_abd_ctx.cuh"

using namespace sgipc;


namespace {

constexpr unsigned long long kNoKey = ~0ull;

SgipcStatus abd_fail(SgipcAbdCtx* c, cudaError_t e, const char* what) {
    if (c) snprintf(c->err, sizeof(c->err), "%s: %s", what, cudaGetErrorString(e));
    return SGIPC_CUDA_ERROR;
}
#define AB_CHECK(ctx, call)                                     \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return abd_fail(ctx, e_, #call); \
    } while (0)

__device__ __forceinline__ unsigned long long bkey(int r, int c) {
    return ((unsigned long long)(unsigned)r << 32) | (unsigned)c;
}

// M v for the dyadic mass (m, m x, m x x^T) of one body
__device__ void dyadic_mv(const double* dm, const double* v, double* out) {
    const double m = dm[0];
    const double* mx = dm + 1;
    const double* D = dm + 4;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const double* a = v + 3 + 3 * r;
        out[r] = mx[0] * a[0] + mx[1] * a[1] + mx[2] * a[2] + m * v[r];
#pragma unroll
        for (int c = 0; c < 3; c++)
            out[3 + 3 * r + c] = D[3 * c + 0] * a[0] + D[3 * c + 1] * a[1] + D[3 * c + 2] * a[2] + mx[c] * v[r];
    }
}

// cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major, in place:
// A -> diag(w)); V accumulates the eigenvectors as columns
template <int N>
__device__ void jacobi_eig(double (&A)[N][N], double (&V)[N][N]) {
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) V[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 20; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < N; i++) {
            diag += A[i][i] * A[i][i];
            for (int j = i + 1; j < N; j++) off += A[i][j] * A[i][j];
        }
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < N - 1; p++)
            for (int q = p + 1; q < N; q++) {
                const double apq = A[p][q];
                if (apq == 0.0) continue;
                const double th = (A[q][q] - A[p][p]) / (2.0 * apq);
                const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < N; k++) {  // A <- A R (columns p, q)
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = cs * akp - sn * akq;
                    A[k][q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < N; k++) {  // A <- R^T A (rows p, q)
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = cs * apk - sn * aqk;
                    A[q][k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < N; k++) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = cs * vkp - sn * vkq;
                    V[k][q] = sn * vkp + cs * vkq;
                }
            }
    }
}

// body terms: gradient (12) and the 10 upper 3x3 blocks of the 12x12 body Hessian
__global__ void k_abd_body(int B, const double* __restrict__ q, const double* __restrict__ qt,
                           const double* __restrict__ dmass, const double* __restrict__ vol,
                           const int* __restrict__ bt, double kappa, double dt, double* __restrict__ grad,
                           unsigned long long* __restrict__ key, int* __restrict__ idx, double* __restrict__ val) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const double* dm = dmass + 13 * (size_t)b;
    double qb[12], dq[12], G[12];
    for (int k = 0; k < 12; k++) {
        qb[k] = q[12 * (size_t)b + k];
        dq[k] = qb[k] - qt[12 * (size_t)b + k];
    }
    double H[12][12];
    for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++) H[i][j] = 0.0;
    // dyadic mass matrix
    for (int r = 0; r < 3; r++) {
        H[r][r] = dm[0];
        for (int c = 0; c < 3; c++) {
            H[r][3 + 3 * r + c] = dm[1 + c];
            H[3 + 3 * r + c][r] = dm[1 + c];
            for (int d = 0; d < 3; d++) H[3 + 3 * r + c][3 + 3 * r + d] = dm[4 + 3 * c + d];
        }
    }
    const bool fixed = bt[b] != 0;
    if (fixed) {
        for (int k = 0; k < 12; k++) G[k] = 0.0;
    } else {
        dyadic_mv(dm, dq, G);
        const double kvt2 = kappa * vol[b] * dt * dt;
        const double* a[3] = {qb + 3, qb + 6, qb + 9};
        double Hs[9][9], V[9][9];
        for (int i = 0; i < 3; i++) {
            const double aii = a[i][0] * a[i][0] + a[i][1] * a[i][1] + a[i][2] * a[i][2];
            for (int p = 0; p < 3; p++) {
                double g = 4.0 * (aii - 1.0) * a[i][p];
                for (int j = 0; j < 3; j++) {
                    if (j == i) continue;
                    const double aij = a[i][0] * a[j][0] + a[i][1] * a[j][1] + a[i][2] * a[j][2];
                    g += 4.0 * aij * a[j][p];
                }
                G[3 + 3 * i + p] += kvt2 * g;
            }
            for (int j = 0; j < 3; j++) {
                const double aij = a[i][0] * a[j][0] + a[i][1] * a[j][1] + a[i][2] * a[j][2];
                for (int p = 0; p < 3; p++)
                    for (int r = 0; r < 3; r++) {
                        double h;
                        if (i == j) {
                            h = 8.0 * a[i][p] * a[i][r] + (p == r ? 4.0 * (aii - 1.0) : 0.0);
                            for (int k = 0; k < 3; k++)
                                if (k != i) h += 4.0 * a[k][p] * a[k][r];
                        } else {
                            h = 4.0 * a[j][p] * a[i][r] + (p == r ? 4.0 * aij : 0.0);
                        }
                        Hs[3 * i + p][3 * j + r] = kvt2 * h;
                    }
            }
        }
        jacobi_eig<9>(Hs, V);
        for (int i = 0; i < 9; i++)
            for (int j = 0; j < 9; j++) {
                double s = 0.0;
                for (int k = 0; k < 9; k++)
                    if (Hs[k][k] > 0.0) s += V[i][k] * Hs[k][k] * V[j][k];
                H[3 + i][3 + j] += s;
            }
    }
    for (int k = 0; k < 12; k++) grad[12 * (size_t)b + k] = G[k];
    const int pa[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3}, pb[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
    for (int s = 0; s < 10; s++) {
        const size_t o = 10 * (size_t)b + s;
        key[o] = bkey(4 * b + pa[s], 4 * b + pb[s]);
        idx[o] = (int)o;
        for (int p = 0; p < 3; p++)
            for (int r = 0; r < 3; r++) val[9 * o + 3 * p + r] = H[3 * pa[s] + p][3 * pb[s] + r];
    }
}

// body gradient += J_p^T g_p over the body's points (deterministic order)
__global__ void k_abd_point_grad(int B, const int* __restrict__ body_ptr, const int* __restrict__ bt,
                                 const double* __restrict__ x_bar, const double* __restrict__ g,
                                 double* __restrict__ grad) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B || bt[b] != 0) return;
    double G[12];
    for (int k = 0; k < 12; k++) G[k] = 0.0;
    for (int p = body_ptr[b]; p < body_ptr[b + 1]; p++) {
        const double gx[3] = {g[3 * (size_t)p], g[3 * (size_t)p + 1], g[3 * (size_t)p + 2]};
        const double* x = x_bar + 3 * (size_t)p;
        for (int r = 0; r < 3; r++) {
            G[r] += gx[r];
            for (int c = 0; c < 3; c++) G[3 + 3 * r + c] += x[c] * gx[r];
        }
    }
    for (int k = 0; k < 12; k++) grad[12 * (size_t)b + k] += G[k];
}

// the (k, l) 3x3 block of J(x)^T H J(y): block rows/cols 0 = translation, 1+r = row a_r
__device__ __forceinline__ void jthj_block(const double* x, const double* y, const double (&H)[3][3], int k, int l,
                                           double* out /*9 row-major*/) {
    for (int p = 0; p < 3; p++)
        for (int r = 0; r < 3; r++) {
            double v;
            if (k == 0 && l == 0) v = H[p][r];
            else if (k == 0) v = H[p][l - 1] * y[r];          // H e_{l-1} y^T
            else if (l == 0) v = x[p] * H[k - 1][r];          // x H(k-1, :)
            else v = x[p] * y[r] * H[k - 1][l - 1];           // (x y^T) H(k-1, l-1)
            out[3 * p + r] = v;
        }
}

// ABD-ABD point blocks -> body-space blocks, 16 slots per input block
__global__ void k_abd_abd(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                          const double* __restrict__ vals, const int* __restrict__ point_body,
                          const int* __restrict__ bt, const double* __restrict__ x_bar, int P, int base,
                          unsigned long long* __restrict__ key, int* __restrict__ idx, double* __restrict__ val,
                          int* __restrict__ flag) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    int i = rows[e], j = cols[e];
    const size_t o0 = (size_t)base + 16 * (size_t)e;
    if (i < 0 || j < 0 || i >= P || j >= P) {
        atomicOr(flag, 1);
        for (int s = 0; s < 16; s++) {
            key[o0 + s] = kNoKey;
            idx[o0 + s] = (int)(o0 + s);
        }
        return;
    }
    double H[3][3];
    for (int p = 0; p < 3; p++)
        for (int r = 0; r < 3; r++) H[p][r] = vals[9 * (size_t)e + 3 * p + r];
    int bi = point_body[i], bj = point_body[j];
    const bool zero = bt[bi] != 0 || bt[bj] != 0;
    const double* x = x_bar + 3 * (size_t)i;
    const double* y = x_bar + 3 * (size_t)j;
    for (int s = 0; s < 16; s++) {
        const int k = s / 4, l = s % 4;
        const size_t o = o0 + s;
        idx[o] = (int)o;
        double blk[9], bt2[9];
        jthj_block(x, y, H, k, l, blk);
        int r = 4 * bi + k, c = 4 * bj + l;
        if (bi == bj) {
            // same body: the symmetric counterpart (j, i) of an off-diagonal point block
            // lands in the same group; keep the upper half of K + K^T (K itself when i == j)
            if (k > l) {
                key[o] = kNoKey;
                continue;
            }
            if (i != j) {
                jthj_block(x, y, H, l, k, bt2);  // K(l, k), to add transposed
                for (int p = 0; p < 3; p++)
                    for (int t = 0; t < 3; t++) blk[3 * p + t] += bt2[3 * t + p];
            }
        } else if (bi > bj) {  // keep upper storage: the block sits transposed at (c, r)
            const int rr = r;
            r = c;
            c = rr;
            for (int p = 0; p < 3; p++)
                for (int t = 0; t < 3; t++) bt2[3 * p + t] = blk[3 * t + p];
            for (int q = 0; q < 9; q++) blk[q] = bt2[q];
        }
        key[o] = bkey(r, c);
        for (int q = 0; q < 9; q++) val[9 * o + q] = zero ? 0.0 : blk[q];
    }
}

// ABD-FEM point blocks -> 4 body-row blocks in FEM column 4B + j
__global__ void k_abd_fem(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                          const double* __restrict__ vals, const int* __restrict__ point_body,
                          const int* __restrict__ bt, const double* __restrict__ x_bar, const int* __restrict__ fbt,
                          int P, int B, int base, unsigned long long* __restrict__ key, int* __restrict__ idx,
                          double* __restrict__ val, int* __restrict__ flag) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int i = rows[e], j = cols[e];
    const size_t o0 = (size_t)base + 4 * (size_t)e;
    if (i < 0 || i >= P || j < 0) {
        atomicOr(flag, 1);
        for (int s = 0; s < 4; s++) {
            key[o0 + s] = kNoKey;
            idx[o0 + s] = (int)(o0 + s);
        }
        return;
    }
    const int b = point_body[i];
    const bool zero = bt[b] != 0 || (fbt && fbt[j] != 0);
    const double* x = x_bar + 3 * (size_t)i;
    const double* H = vals + 9 * (size_t)e;
    for (int k = 0; k < 4; k++) {
        const size_t o = o0 + k;
        idx[o] = (int)o;
        key[o] = bkey(4 * b + k, 4 * B + j);
        for (int p = 0; p < 3; p++)
            for (int r = 0; r < 3; r++) {
                const double v = k == 0 ? H[3 * p + r] : x[p] * H[3 * (k - 1) + r];  // (J^T H) rows
                val[9 * o + 3 * p + r] = zero ? 0.0 : v;
            }
    }
}

__global__ void k_heads(int m, const unsigned long long* __restrict__ ks, int* __restrict__ flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    if (i == m) {
        flag[m] = 0;
        return;
    }
    const unsigned long long k = ks[i];
    flag[i] = (k != kNoKey && (i == 0 || ks[i - 1] != k)) ? 1 : 0;
}

__global__ void k_reduce(int m, const unsigned long long* __restrict__ ks, const int* __restrict__ is,
                         const int* __restrict__ uid, const double* __restrict__ val, int* __restrict__ ur,
                         int* __restrict__ uc, double* __restrict__ uv, int* __restrict__ nu) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) nu[0] = uid[m];
    if (i >= m) return;
    const unsigned long long k = ks[i];
    if (k == kNoKey || (i > 0 && ks[i - 1] == k)) return;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = i; j < m && ks[j] == k; j++)
        for (int q = 0; q < 9; q++) acc[q] += val[9 * (size_t)is[j] + q];
    const int u = uid[i];
    ur[u] = (int)(k >> 32);
    uc[u] = (int)(k & 0xffffffffull);
    for (int q = 0; q < 9; q++) uv[9 * (size_t)u + q] = acc[q];
}

// body diagonal groups of the merged matrix into dense 12x12 blocks (both triangles)
__global__ void k_pfill(const int* __restrict__ nu, const int* __restrict__ ur, const int* __restrict__ uc,
                        const double* __restrict__ uv, int B, double* __restrict__ Pm) {
    int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu[0]) return;
    const int r = ur[u], c = uc[u];
    if (r / 4 != c / 4 || r >= 4 * B) return;
    const int b = r / 4, k = r % 4, l = c % 4;
    double* M = Pm + 144 * (size_t)b;
    for (int p = 0; p < 3; p++)
        for (int t = 0; t < 3; t++) {
            const double v = uv[9 * (size_t)u + 3 * p + t];
            M[(3 * k + p) * 12 + 3 * l + t] = v;
            if (k != l) M[(3 * l + t) * 12 + 3 * k + p] = v;
        }
}

// in-place Gauss-Jordan inverse with partial pivoting, one thread per body
__global__ void k_pinv(int B, double* __restrict__ Pm) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    double A[12][24];
    const double* M = Pm + 144 * (size_t)b;
    for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++) {
            A[i][j] = M[12 * i + j];
            A[i][12 + j] = i == j ? 1.0 : 0.0;
        }
    for (int c = 0; c < 12; c++) {
        int piv = c;
        for (int i = c + 1; i < 12; i++)
            if (fabs(A[i][c]) > fabs(A[piv][c])) piv = i;
        if (piv != c)
            for (int j = 0; j < 24; j++) {
                const double t = A[c][j];
                A[c][j] = A[piv][j];
                A[piv][j] = t;
            }
        const double d = A[c][c];
        const double inv = d != 0.0 ? 1.0 / d : 0.0;
        for (int j = 0; j < 24; j++) A[c][j] *= inv;
        for (int i = 0; i < 12; i++) {
            if (i == c) continue;
            const double f = A[i][c];
            if (f == 0.0) continue;
            for (int j = 0; j < 24; j++) A[i][j] -= f * A[c][j];
        }
    }
    double* O = Pm + 144 * (size_t)b;
    for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++) O[12 * i + j] = A[i][12 + j];
}

__global__ void k_papply(int B, const double* __restrict__ Pm, const double* __restrict__ r, double* __restrict__ z) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 12 * B) return;
    const int b = t / 12, i = t % 12;
    const double* M = Pm + 144 * (size_t)b + 12 * i;
    const double* rb = r + 12 * (size_t)b;
    double s = 0.0;
    for (int j = 0; j < 12; j++) s += M[j] * rb[j];
    z[t] = s;
}

template <class T>
SgipcStatus dalloc(SgipcAbdCtx* c, T** p, size_t n) {
    AB_CHECK(c, cudaMalloc((void**)p, sizeof(T) * (n > 0 ? n : 1)));
    return SGIPC_OK;
}

template <class T>
SgipcStatus upload(SgipcAbdCtx* c, T** p, const T* h, size_t n) {
    SgipcStatus st = dalloc(c, p, n);
    if (st != SGIPC_OK) return st;
    if (n) AB_CHECK(c, cudaMemcpy(*p, h, sizeof(T) * n, cudaMemcpyHostToDevice));
    return SGIPC_OK;
}

}  // namespace

extern "C" const char* sgipc_abd_last_error(const SgipcAbdCtx* c) { return c ? c->err : "null context"; }

extern "C" SgipcStatus sgipc_abd_destroy(SgipcAbdCtx* c) {
    if (!c) return SGIPC_BAD_INPUT;
    sgipc::DeviceScope dev_scope(c->device);
    void* ps[] = {c->point_body, c->body_ptr, c->bt, c->x_bar, c->dmass, c->vol, c->key, c->key_s, c->idx,
                  c->idx_s, c->val, c->flag, c->nu, c->u_row, c->u_col, c->u_val, c->pinv, c->cub_tmp,
                  c->g_rptr, c->g_cptr, c->g_tkey, c->g_tkey_s, c->g_tidx, c->g_tidx_s, c->g_vec, c->g_dot,
                  c->g_cub};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete c;
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_abd_create(const SgipcAbdTopology* t, int device, SgipcAbdCtx** out) {
    if (!t || !out || t->body_num < 1 || t->point_num < 0 || t->max_abd_blocks < 0 || t->max_fem_blocks < 0)
        return SGIPC_BAD_INPUT;
    if (!t->dyadic_mass || !t->volume || !t->boundary_type || (t->point_num && (!t->point_body || !t->x_bar)))
        return SGIPC_BAD_INPUT;
    const int B = t->body_num, P = t->point_num;
    std::vector<int> ptr(B + 1, 0);
    for (int p = 0; p < P; p++) {
        const int b = t->point_body[p];
        if (b < 0 || b >= B || (p > 0 && b < t->point_body[p - 1])) return SGIPC_BAD_INPUT;  // numbered body by body
        ptr[b + 1]++;
    }
    for (int b = 0; b < B; b++) ptr[b + 1] += ptr[b];
    SgipcAbdCtx* c = new SgipcAbdCtx();
    memset(c, 0, sizeof(*c));
    c->device = device;
    c->B = B;
    c->P = P;
    c->max_abd = t->max_abd_blocks;
    c->max_fem = t->max_fem_blocks;
    c->cap = 10 * B + 16 * c->max_abd + 4 * c->max_fem;
    auto fail = [&](SgipcStatus st) {
        sgipc_abd_destroy(c);
        return st;
    };
    sgipc::DeviceScope dev_scope(device);
    if (dev_scope.err != cudaSuccess) return fail(SGIPC_CUDA_ERROR);
    SgipcStatus st;
    if ((st = upload(c, &c->point_body, t->point_body, P)) || (st = upload(c, &c->body_ptr, ptr.data(), B + 1)) ||
        (st = upload(c, &c->bt, t->boundary_type, B)) || (st = upload(c, &c->x_bar, t->x_bar, 3 * (size_t)P)) ||
        (st = upload(c, &c->dmass, t->dyadic_mass, 13 * (size_t)B)) || (st = upload(c, &c->vol, t->volume, B)) ||
        (st = dalloc(c, &c->key, c->cap)) || (st = dalloc(c, &c->key_s, c->cap)) || (st = dalloc(c, &c->idx, c->cap)) ||
        (st = dalloc(c, &c->idx_s, c->cap)) || (st = dalloc(c, &c->val, 9 * (size_t)c->cap)) ||
        (st = dalloc(c, &c->flag, c->cap + 1)) || (st = dalloc(c, &c->nu, 2)) || (st = dalloc(c, &c->u_row, c->cap)) ||
        (st = dalloc(c, &c->u_col, c->cap)) || (st = dalloc(c, &c->u_val, 9 * (size_t)c->cap)) ||
        (st = dalloc(c, &c->pinv, 144 * (size_t)B)))
        return fail(st);
    size_t a = 0, b2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, a, c->key, c->key_s, c->idx, c->idx_s, c->cap);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, c->flag, c->flag, c->cap + 1);
    c->cub_bytes = a > b2 ? a : b2;
    if ((st = dalloc(c, (char**)&c->cub_tmp, c->cub_bytes))) return fail(st);
    *out = c;
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_abd_grad_hess(SgipcAbdCtx* c, const double* q, const double* qt, double kappa, double dt,
                                           const double* point_grad, int32_t nabd, const int32_t* arows,
                                           const int32_t* acols, const double* avals, int32_t nfem,
                                           const int32_t* frows, const int32_t* fcols, const double* fvals,
                                           const int32_t* fbt, double* body_grad, void* stream) {
    if (!c || !q || !qt || !body_grad || !(dt > 0.0) || !(kappa >= 0.0) || nabd < 0 || nfem < 0) return SGIPC_BAD_INPUT;
    if ((nabd && (!arows || !acols || !avals)) || (nfem && (!frows || !fcols || !fvals))) return SGIPC_BAD_INPUT;
    if (nabd > c->max_abd || nfem > c->max_fem) {
        snprintf(c->err, sizeof(c->err), "contact blocks exceed the ABD context capacity");
        return SGIPC_CAPACITY;
    }
    cudaStream_t s = (cudaStream_t)stream;
    sgipc::DeviceScope dev_scope(c->device);
    AB_CHECK(c, dev_scope.err);
    const int B = c->B;
    AB_CHECK(c, cudaMemsetAsync(c->flag + c->cap, 0, sizeof(int), s));  // input-error word
    int* eflag = c->flag + c->cap;
    k_abd_body<<<nblk(B, 64), 64, 0, s>>>(B, q, qt, c->dmass, c->vol, c->bt, kappa, dt, body_grad, c->key, c->idx,
                                          c->val);
    if (point_grad && c->P)
        k_abd_point_grad<<<nblk(B, 128), 128, 0, s>>>(B, c->body_ptr, c->bt, c->x_bar, point_grad, body_grad);
    int base = 10 * B;
    if (nabd)
        k_abd_abd<<<nblk(nabd, 128), 128, 0, s>>>(nabd, arows, acols, avals, c->point_body, c->bt, c->x_bar, c->P,
                                                  base, c->key, c->idx, c->val, eflag);
    base += 16 * nabd;
    if (nfem)
        k_abd_fem<<<nblk(nfem, 128), 128, 0, s>>>(nfem, frows, fcols, fvals, c->point_body, c->bt, c->x_bar, fbt,
                                                  c->P, B, base, c->key, c->idx, c->val, eflag);
    base += 4 * nfem;
    const int m = base;
    c->m_last = m;
    size_t tb = c->cub_bytes;
    AB_CHECK(c, cub::DeviceRadixSort::SortPairs(c->cub_tmp, tb, c->key, c->key_s, c->idx, c->idx_s, m, 0, 64, s));
    // the scan input/output must not overlap the error word: heads for m entries + 1
    int hflag = 0;
    AB_CHECK(c, cudaMemcpyAsync(&hflag, eflag, sizeof(int), cudaMemcpyDeviceToHost, s));
    AB_CHECK(c, cudaStreamSynchronize(s));
    if (hflag) {
        snprintf(c->err, sizeof(c->err), "a contact block references a point outside the ABD points");
        return SGIPC_BAD_INPUT;
    }
    k_heads<<<nblk(m + 1), SGIPC_BLOCK, 0, s>>>(m, c->key_s, c->flag);
    tb = c->cub_bytes;
    AB_CHECK(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp, tb, c->flag, c->flag, m + 1, s));
    k_reduce<<<nblk(m), SGIPC_BLOCK, 0, s>>>(m, c->key_s, c->idx_s, c->flag, c->val, c->u_row, c->u_col, c->u_val,
                                             c->nu);
    AB_CHECK(c, cudaGetLastError());
    c->assembled = 1;
    c->pbuilt = 0;
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_abd_export_bcoo(SgipcAbdCtx* c, int32_t cap, int32_t* rows, int32_t* cols, double* vals,
                                             int32_t* count) {
    if (!c || !count) return SGIPC_BAD_INPUT;
    if (!c->assembled) return SGIPC_NOT_READY;
    sgipc::DeviceScope dev_scope(c->device);
    AB_CHECK(c, dev_scope.err);
    AB_CHECK(c, cudaDeviceSynchronize());
    int nu = 0;
    AB_CHECK(c, cudaMemcpy(&nu, c->nu, sizeof(int), cudaMemcpyDeviceToHost));
    *count = nu;
    if (!rows) return SGIPC_OK;
    if (!cols || !vals || cap < nu) return SGIPC_CAPACITY;
    AB_CHECK(c, cudaMemcpy(rows, c->u_row, sizeof(int) * nu, cudaMemcpyDeviceToHost));
    AB_CHECK(c, cudaMemcpy(cols, c->u_col, sizeof(int) * nu, cudaMemcpyDeviceToHost));
    AB_CHECK(c, cudaMemcpy(vals, c->u_val, sizeof(double) * 9 * nu, cudaMemcpyDeviceToHost));
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_abd_precond_build(SgipcAbdCtx* c, void* stream) {
    if (!c) return SGIPC_BAD_INPUT;
    if (!c->assembled) return SGIPC_NOT_READY;
    cudaStream_t s = (cudaStream_t)stream;
    sgipc::DeviceScope dev_scope(c->device);
    AB_CHECK(c, dev_scope.err);
    AB_CHECK(c, cudaMemsetAsync(c->pinv, 0, sizeof(double) * 144 * c->B, s));
    k_pfill<<<nblk(c->m_last > 0 ? c->m_last : 1), SGIPC_BLOCK, 0, s>>>(c->nu, c->u_row, c->u_col, c->u_val, c->B,
                                                                       c->pinv);
    k_pinv<<<nblk(c->B, 64), 64, 0, s>>>(c->B, c->pinv);
    AB_CHECK(c, cudaGetLastError());
    c->pbuilt = 1;
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_abd_precond_apply(SgipcAbdCtx* c, const double* r, double* z, void* stream) {
    if (!c || !r || !z) return SGIPC_BAD_INPUT;
    if (!c->assembled) return SGIPC_NOT_READY;
    sgipc::DeviceScope dev_scope(c->device);
    AB_CHECK(c, dev_scope.err);
    k_papply<<<nblk(12LL * c->B), SGIPC_BLOCK, 0, (cudaStream_t)stream>>>(c->B, c->pinv, r, z);
    AB_CHECK(c, cudaGetLastError());
    return SGIPC_OK;
}

void sgipc::abd_precond_apply_async(SgipcAbdCtx* c, const double* r, double* z, cudaStream_t s) {
    k_papply<<<nblk(12LL * c->B), SGIPC_BLOCK, 0, s>>>(c->B, c->pinv, r, z);
}
