// sgipc_assemble.cu — gradient and Hessian assembly of one Newton iteration.
//
// Follows GIPC::computeGradientAndHessian (StiffGIPC/GIPC.cu:10110-10344):
//   kinetic gradient M(x - x~)                          GIPC.cu:6339
//   IPC barrier, RANK 2, Gauss-Newton Hessian            GIPC.cu:3106-4945
//   lagged smoothed friction (pairs and ground)          GIPC.cu:1357-1800, 5047-5270
//   ground barrier, soft constraints                     GIPC.cu:6363-6514
//   stable Neo-Hookean tets with the analytic projection femEnergy.cu:1593-1857
//   Dirichlet zeroing, mass diagonal                     GIPC.cu:10295-10336
//   b = fb + shape_grads, Dirichlet rows zeroed          fem_linear_subsystem.cu:56-84
//
// Layout on the GPU (all FP64):
//   * static part: element kernels write oriented 3x3 blocks into per-element slots
//     (eblk) and per-vertex gradient rows (egrad); gather kernels sum them into the BSR
//     values and shape_grads through CSR lists built at context creation;
//   * dynamic part: every contact pair writes its upper blocks under a (row,col) key; one
//     radix sort plus a segmented sum gives the unique contact blocks, kept row-sorted
//     together with a transposed index list so that SpMV needs no atomics.
#include <cmath>

#include <cub/cub.cuh>

#include "sgipc_internal.cuh"

using namespace sgipc;

namespace {

constexpr unsigned long long kBadKey = ~0ull;

// ------------------------------------------------------------------------------------------
// kinetic gradient, reset of the contact gradient
// ------------------------------------------------------------------------------------------
__global__ void k_kinetic(int nv, const double* __restrict__ x, const double* __restrict__ xt,
                          const double* __restrict__ m, double* __restrict__ shape_grads, double* __restrict__ fb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * nv) return;
    shape_grads[i] = m[i / 3] * (x[i] - xt[i]);
    fb[i] = 0.0;
}

// ------------------------------------------------------------------------------------------
// stable Neo-Hookean tet (USE_SNK1): PK1 femEnergy.cu:432-459, eigensystem 1593-1717
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_snk(int nt, const uint32_t* __restrict__ tets, const double* __restrict__ x,
                                             const double* __restrict__ dminv, const double* __restrict__ vol,
                                             const double* __restrict__ lr, const double* __restrict__ vr, double dt2,
                                             double* __restrict__ eblk, double* __restrict__ egrad) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    uint4 tv = reinterpret_cast<const uint4*>(tets)[t];
    const uint32_t vid[4] = {tv.x, tv.y, tv.z, tv.w};
    d3 X0 = ld3(x, tv.x), X1 = ld3(x, tv.y), X2 = ld3(x, tv.z), X3 = ld3(x, tv.w);
    double Di[3][3];
#pragma unroll
    for (int k = 0; k < 9; k++) Di[k / 3][k % 3] = dminv[9 * (size_t)t + k];
    const double mu = lr[t], lam = vr[t], sc = dt2 * vol[t];
    d3 e1 = X1 - X0, e2 = X2 - X0, e3 = X3 - X0;
    double F[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double a = comp(e1, i), b = comp(e2, i), c = comp(e3, i);
#pragma unroll
        for (int j = 0; j < 3; j++) F[i][j] = a * Di[0][j] + b * Di[1][j] + c * Di[2][j];
    }
    d3 f0 = mk(F[0][0], F[1][0], F[2][0]), f1 = mk(F[0][1], F[1][1], F[2][1]), f2 = mk(F[0][2], F[1][2], F[2][2]);
    d3 g0 = cross(f1, f2), g1 = cross(f2, f0), g2 = cross(f0, f1);
    const double J = dot(f0, g0);
    const double ev = lam * (J - 1.0) - mu;  // evScale of the twist/flip pairs
    // P = mu F + (lam (J - 1) - mu) cof(F); gradient rows G = P Dm^-T
    d3 P0 = mu * f0 + ev * g0, P1 = mu * f1 + ev * g1, P2 = mu * f2 + ev * g2;
    d3 gr[4];
#pragma unroll
    for (int k = 0; k < 3; k++) gr[k + 1] = sc * (Di[k][0] * P0 + Di[k][1] * P1 + Di[k][2] * P2);
    gr[0] = -(gr[1] + gr[2] + gr[3]);
#pragma unroll
    for (int a = 0; a < 4; a++) {
        double* o = egrad + 3 * (4 * (size_t)t + a);
        o[0] = gr[a].x;
        o[1] = gr[a].y;
        o[2] = gr[a].z;
    }
    // analytic eigensystem of d2Psi/dF2 (Smith et al., "Analytic eigensystems for isotropic
    // distortion energies"): twist/flip pairs per axis plus a 3x3 scaling block
    double U[3][3], S[3], V[3][3];
    svd3_rv(F, U, S, V);
    double c1[3], c2[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double lt = fmax(mu + ev * S[k], 0.0), lf = fmax(mu - ev * S[k], 0.0);
        c1[k] = 0.5 * (lt + lf);
        c2[k] = 0.5 * (lf - lt);
    }
    double A[3][3], Q[3][3];
    const double es = lam * (2.0 * J - 1.0) - mu;
    A[0][0] = mu + lam * S[1] * S[1] * S[2] * S[2];
    A[1][1] = mu + lam * S[0] * S[0] * S[2] * S[2];
    A[2][2] = mu + lam * S[0] * S[0] * S[1] * S[1];
    A[0][1] = A[1][0] = es * S[2];
    A[0][2] = A[2][0] = es * S[1];
    A[1][2] = A[2][1] = es * S[0];
    sym_eig3(A, Q);
    double Sp[3][3];
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
        for (int q = 0; q < 3; q++) {
            double s = 0;
#pragma unroll
            for (int m = 0; m < 3; m++) s += fmax(A[m][m], 0.0) * Q[p][m] * Q[q][m];
            Sp[p][q] = s;
        }
    // d_a = V^T D(a,:)^T with D the rows of dF/dx
    double d[4][3];
#pragma unroll
    for (int p = 0; p < 3; p++) {
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double v = V[j][p];
            s1 += v * Di[0][j];
            s2 += v * Di[1][j];
            s3 += v * Di[2][j];
        }
        s0 = -(s1 + s2 + s3);
        d[0][p] = s0;
        d[1][p] = s1;
        d[2][p] = s2;
        d[3][p] = s3;
    }
    const int pa[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
    const int pb[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
    const int ax_i[3] = {1, 0, 0}, ax_j[3] = {2, 2, 1};
    // (unrolled: the vertex pair of each block is then a compile-time index into d, which a
    // rolled loop kept in local memory; 168 registers, measured 4 % faster than rolled)
#pragma unroll
    for (int k = 0; k < 10; k++) {
        const int a = pa[k], b = pb[k];
        double K[3][3];
#pragma unroll
        for (int p = 0; p < 3; p++)
#pragma unroll
            for (int q = 0; q < 3; q++) K[p][q] = Sp[p][q] * d[a][p] * d[b][q];
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const int i = ax_i[m], j = ax_j[m];
            K[j][j] += c1[m] * d[a][i] * d[b][i];
            K[i][i] += c1[m] * d[a][j] * d[b][j];
            K[j][i] += c2[m] * d[a][i] * d[b][j];
            K[i][j] += c2[m] * d[a][j] * d[b][i];
        }
        // H = sc * U K U^T, written transposed when the element's vertex order is reversed
        double UK[3][3];
#pragma unroll
        for (int p = 0; p < 3; p++)
#pragma unroll
            for (int q = 0; q < 3; q++) UK[p][q] = U[p][0] * K[0][q] + U[p][1] * K[1][q] + U[p][2] * K[2][q];
        const bool tr = vid[a] > vid[b];
        double* o = eblk + 9 * (10 * (size_t)t + k);
#pragma unroll
        for (int p = 0; p < 3; p++)
#pragma unroll
            for (int q = 0; q < 3; q++) {
                double h = sc * (UK[p][0] * U[q][0] + UK[p][1] * U[q][1] + UK[p][2] * U[q][2]);
                o[tr ? (3 * q + p) : (3 * p + q)] = h;
            }
    }
}

// ------------------------------------------------------------------------------------------
// cloth membrane: Baraff-Witkin stretch + shear (femEnergy.cu:351-403 stress, 535-707 the
// two projected Hessians, 2146-2215 the element kernel).  F = Ds Dm^-1 (3x2), columns
// f0, f1.  Energy density k_st (S(|f0|) + S(|f1|)) + k_sh (f0.f1)^2 with
// S(t) = (t-1)^2 + [t > 1] s (t-1)^3, times area*thickness*dt^2.  The reference projects
// the stretch and the shear Hessian separately and sums them; both projections have closed
// forms used here:
//   stretch, per column (n = f/t):  [t > 1] S'(t)/t (I - n n^T) + c n n^T, with
//     c = S''(t) for t > 1 and 2 otherwise (the negative transverse part clamped);
//   shear, E = I6^2 with I6 = f0.f1, g = [f1; f0], a = [f0; f1], swap S = [[0,I],[I,0]]:
//     the exact Hessian 2(g g^T + I6 S) has, in span{a, g}, the eigenpair
//     2 lambda0 with q ~ I6 a + lambda0 g, lambda0 = (I2 + sqrt(I2^2 + 12 I6^2)) / 2, and in
//     the complement +-2|I6| on the eigenspaces of S; the projection keeps
//     2 lambda0 q q^T + |I6| [[Pw, sg Pw], [sg Pw, Pw]], sg = sign(I6) (+1 at 0),
//     Pw = I - w w^T / |w|^2, w = f0 + sg f1 (the part of the sg-eigenspace outside span{a,g}).
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_tri_bw(int nf, const uint32_t* __restrict__ tris, const double* __restrict__ x,
                                                const double* __restrict__ dminv, const double* __restrict__ area,
                                                double kst, double ksh, double srate, double dt2, int eoff, int goff,
                                                double* __restrict__ eblk, double* __restrict__ egrad) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    int vid[3];
#pragma unroll
    for (int a = 0; a < 3; a++) vid[a] = (int)tris[3 * f + a];
    const d3 x0 = ld3(x, vid[0]), e1 = ld3(x, vid[1]) - x0, e2 = ld3(x, vid[2]) - x0;
    const double* Di = dminv + 4 * (size_t)f;  // row-major 2x2
    const d3 col[2] = {Di[0] * e1 + Di[2] * e2, Di[1] * e1 + Di[3] * e2};
    // dF(:,j)/dx_a = D[a][j] I
    const double D[3][2] = {{-(Di[0] + Di[2]), -(Di[1] + Di[3])}, {Di[0], Di[1]}, {Di[2], Di[3]}};
    const double scale = area[f] * dt2;

    // stress P (columns) and the 6x6 projected Hessian as 3x3 blocks Hq[j][k]
    d3 P[2];
    double Hq[2][2][3][3];
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
        for (int k = 0; k < 2; k++)
#pragma unroll
            for (int p = 0; p < 3; p++)
#pragma unroll
                for (int q = 0; q < 3; q++) Hq[j][k][p][q] = 0.0;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const d3 fj = col[j];
        const double t = sqrt(sq(fj));
        const double u = t - 1.0;
        const double dS = 2.0 * u + (t > 1.0 ? 3.0 * srate * u * u : 0.0);
        P[j] = (kst * dS / t) * fj;
        const double ct = t > 1.0 ? dS / t : 0.0;                    // transverse (clamped)
        const double cn = t > 1.0 ? 2.0 + 6.0 * srate * u : 2.0;     // along n
        const double n[3] = {fj.x / t, fj.y / t, fj.z / t};
#pragma unroll
        for (int p = 0; p < 3; p++)
#pragma unroll
            for (int q = 0; q < 3; q++)
                Hq[j][j][p][q] += kst * ((p == q ? ct : 0.0) + (cn - ct) * n[p] * n[q]);
    }
    {
        const d3 f0 = col[0], f1 = col[1];
        const double I6 = dot(f0, f1), I2 = sq(f0) + sq(f1);
        P[0] = P[0] + (2.0 * ksh * I6) * f1;
        P[1] = P[1] + (2.0 * ksh * I6) * f0;
        const double lam0 = 0.5 * (I2 + sqrt(I2 * I2 + 12.0 * I6 * I6));
        const d3 qa = I6 * f0 + lam0 * f1, qb = I6 * f1 + lam0 * f0;  // q = [qa; qb] unnormalised
        const double qn = sq(qa) + sq(qb);
        const double iq = qn > 0.0 ? 1.0 / qn : 0.0;
        const double sg = I6 >= 0.0 ? 1.0 : -1.0;
        const d3 w = f0 + sg * f1;
        const double ww = sq(w);
        const double iw = ww > 0.0 ? 1.0 / ww : 0.0;
        const double q0[2][3] = {{qa.x, qa.y, qa.z}, {qb.x, qb.y, qb.z}};
        const double wv[3] = {w.x, w.y, w.z};
        const double aI6 = fabs(I6);
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const double s = j == k ? 1.0 : sg;
#pragma unroll
                for (int p = 0; p < 3; p++)
#pragma unroll
                    for (int q = 0; q < 3; q++) {
                        const double Pw = (p == q ? 1.0 : 0.0) - wv[p] * wv[q] * iw;
                        Hq[j][k][p][q] += ksh * (2.0 * lam0 * q0[j][p] * q0[k][q] * iq + aI6 * s * Pw);
                    }
            }
    }
    // gradient rows and the 6 oriented upper blocks
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const d3 g = scale * (D[a][0] * P[0] + D[a][1] * P[1]);
        double* o = egrad + 3 * ((size_t)goff + 3 * (size_t)f + a);
        o[0] = g.x;
        o[1] = g.y;
        o[2] = g.z;
    }
    const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const int a = pa[k], b = pb[k];
        const bool tr = vid[a] > vid[b];
        double* o = eblk + 9 * ((size_t)eoff + 6 * (size_t)f + k);
#pragma unroll
        for (int p = 0; p < 3; p++)
#pragma unroll
            for (int q = 0; q < 3; q++) {
                double h = 0.0;
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int l = 0; l < 2; l++) h += D[a][j] * D[b][l] * Hq[j][l][p][q];
                o[tr ? (3 * q + p) : (3 * p + q)] = scale * h;
            }
    }
}

// ------------------------------------------------------------------------------------------
// quadratic bending (femEnergy.cu:2623-2753; Q from the rest shape, :2492-2618): per
// interior edge with vertices [e0, e1, opposite of triangle 1, opposite of triangle 2],
// E = 1/2 c x^T (Q (x) I3) x, c = |rest e0 - rest e1| * bendStiff * dt^2: gradient c Q x,
// constant Hessian c Q (x) I3.  Boundary edges (no second triangle) contribute nothing.
// ------------------------------------------------------------------------------------------
__global__ void k_hinge_quad(int nh, const uint32_t* __restrict__ edges, const int32_t* __restrict__ adj,
                             const double* __restrict__ x, const double* __restrict__ rest,
                             const double* __restrict__ Qcm, double kb_dt2, int eoff, int goff,
                             double* __restrict__ eblk, double* __restrict__ egrad) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= nh) return;
    const int v[4] = {(int)edges[2 * h], (int)edges[2 * h + 1], adj[2 * h], adj[2 * h + 1]};
    const bool boundary = v[2] < 0 || v[3] < 0;
    double Q[4][4];
    double c = 0.0;
    if (!boundary) {
        c = sqrt(sq(ld3(rest, v[0]) - ld3(rest, v[1]))) * kb_dt2;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) Q[i][j] = Qcm[16 * (size_t)h + 4 * j + i];  // column-major
    } else {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) Q[i][j] = 0.0;
    }
    d3 xv[4];
#pragma unroll
    for (int a = 0; a < 4; a++) xv[a] = boundary ? mk(0, 0, 0) : ld3(x, v[a]);
#pragma unroll
    for (int a = 0; a < 4; a++) {
        d3 g = mk(0, 0, 0);
#pragma unroll
        for (int b = 0; b < 4; b++) g = g + (c * Q[a][b]) * xv[b];
        double* o = egrad + 3 * ((size_t)goff + 4 * (size_t)h + a);
        o[0] = g.x;
        o[1] = g.y;
        o[2] = g.z;
    }
    const int pa[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3}, pb[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
#pragma unroll
    for (int k = 0; k < 10; k++) {
        // block (a, b) is c Q(a,b) I3; stored as the (min, max) block, i.e. from Q(b,a) when
        // the element's vertex order is reversed
        const bool tr = v[pa[k]] > v[pb[k]];
        const double d = c * (tr ? Q[pb[k]][pa[k]] : Q[pa[k]][pb[k]]);
        double* o = eblk + 9 * ((size_t)eoff + 10 * (size_t)h + k);
#pragma unroll
        for (int q = 0; q < 9; q++) o[q] = (q % 4 == 0) ? d : 0.0;
    }
}

// ------------------------------------------------------------------------------------------
// static gathers
// ------------------------------------------------------------------------------------------
struct StaticOut {
    double* v64;       // upper slots (the MAS scatter and the BCOO export read these)
    const int* fup;    // full-pattern index of each upper slot
    const int* flo;    // full-pattern index of its transpose (-1 on the diagonal)
    double* f64;       // full symmetric copy
    float* f32;
};

__global__ void k_gather_blocks(int nnz, const int* __restrict__ cptr, const int* __restrict__ contrib,
                                const double* __restrict__ eblk, const int* __restrict__ slot_row,
                                const int* __restrict__ col, const int32_t* __restrict__ btype,
                                const double* __restrict__ mass, StaticOut o) {
    long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 9LL * nnz) return;
    int s = (int)(tid / 9), q = (int)(tid % 9);
    int r = slot_row[s], c = col[s];
    const int k0 = cptr[s], k1 = cptr[s + 1];
    // the contributions four at a time, their index and value loads issued together (one by
    // one, each waited out two L2 round trips), added in list order as before; the boundary
    // test is applied after the loads
    double acc = 0.0;
    int k = k0;
    for (; k + 4 <= k1; k += 4) {
        int ix[4];
#pragma unroll
        for (int u = 0; u < 4; u++) ix[u] = contrib[k + u];
        double e[4];
#pragma unroll
        for (int u = 0; u < 4; u++) e[u] = eblk[9 * (size_t)ix[u] + q];
#pragma unroll
        for (int u = 0; u < 4; u++) acc += e[u];
    }
    for (; k < k1; k++) acc += eblk[9 * (size_t)contrib[k] + q];
    if (btype[r] != 0 || btype[c] != 0) acc = 0.0;
    if (r == c && (q == 0 || q == 4 || q == 8)) acc += mass[r];
    o.v64[tid] = acc;
    const size_t fu = 9 * (size_t)o.fup[s] + q;
    o.f64[fu] = acc;
    o.f32[fu] = (float)acc;
    const int fl = o.flo[s];
    if (fl >= 0) {
        const size_t ft = 9 * (size_t)fl + 3 * (q % 3) + q / 3;
        o.f64[ft] = acc;
        o.f32[ft] = (float)acc;
    }
}

static StaticOut static_out(SgipcCtx* c) {
    StaticOut o;
    o.v64 = c->val64;
    o.fup = c->fup;
    o.flo = c->flo;
    o.f64 = c->fval64;
    o.f32 = c->fval32;
    return o;
}

__global__ void k_gather_grad(int nv, const int* __restrict__ vptr, const int* __restrict__ vinc,
                              const double* __restrict__ egrad, double* __restrict__ shape_grads) {
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 3 * nv) return;
    int v = tid / 3, q = tid % 3;
    const int k0 = vptr[v], k1 = vptr[v + 1];
    double acc = 0.0;
    int k = k0;
    for (; k + 4 <= k1; k += 4) {  // four incident elements in flight, added in list order
        int ix[4];
#pragma unroll
        for (int u = 0; u < 4; u++) ix[u] = vinc[k + u];
        double e[4];
#pragma unroll
        for (int u = 0; u < 4; u++) e[u] = egrad[3 * (size_t)ix[u] + q];
#pragma unroll
        for (int u = 0; u < 4; u++) acc += e[u];
    }
    for (; k < k1; k++) acc += egrad[3 * (size_t)vinc[k] + q];
    shape_grads[tid] += acc;
}

__global__ void k_rhs(int nv, const double* __restrict__ fb, const double* __restrict__ sg,
                      const int32_t* __restrict__ btype, double* __restrict__ b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * nv) return;
    b[i] = btype[i / 3] != 0 ? 0.0 : fb[i] + sg[i];
}

// ------------------------------------------------------------------------------------------
// contact blocks
// ------------------------------------------------------------------------------------------
struct BlockSink {
    unsigned long long* key;
    int* idx;
    double* val;
    const int32_t* btype;  // Dirichlet flags (blocks touching a flagged vertex are zeroed); null: none
    int bits;
    int nv;
    int* flag;  // set to 1 when a pair names a vertex outside [0, nv)
};

__device__ __forceinline__ bool ids_ok(const BlockSink& bs, const int* v, int n) {
    for (int a = 0; a < n; a++)
        if (v[a] < 0 || v[a] >= bs.nv) {
            atomicOr(bs.flag, 1);
            return false;
        }
    return true;
}

// store up to 10 upper blocks of an nv-vertex pair: H_ab = sum_t coef_t u_t,a w_t,b^T
// expressed through a callback producing the 3x3 block for local (a,b)
template <class BlockFn>
__device__ __forceinline__ void emit_pair_blocks(const BlockSink& bs, int base, int nvp, const int* vid, BlockFn fn) {
    // unrolled: the per-vertex arrays of the pair's lambdas are then indexed at compile time
    // (rolled, they lived in local memory; friction terms 7 % faster)
    int k = 0;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = a; b < 4; b++, k++) {
            int slot = base + k;
            bs.idx[slot] = slot;
            if (a >= nvp || b >= nvp) {
                bs.key[slot] = kBadKey;
                continue;
            }
            int r = vid[a], c = vid[b];
            bool tr = r > c;
            int rr = tr ? c : r, cc = tr ? r : c;
            bs.key[slot] = ((unsigned long long)rr << bs.bits) | (unsigned long long)cc;
            double H[3][3];
            fn(a, b, H);
            bool dir = bs.btype && (bs.btype[r] != 0 || bs.btype[c] != 0);
            double* o = bs.val + 9 * (size_t)slot;
#pragma unroll
            for (int p = 0; p < 3; p++)
#pragma unroll
                for (int q = 0; q < 3; q++) o[3 * p + q] = dir ? 0.0 : (tr ? H[q][p] : H[p][q]);
        }
}

__device__ __forceinline__ void emit_diag_block(const BlockSink& bs, int slot, int v, const double H[3][3]) {
    bs.idx[slot] = slot;
    bs.key[slot] = ((unsigned long long)v << bs.bits) | (unsigned long long)v;
    bool dir = bs.btype && bs.btype[v] != 0;
    double* o = bs.val + 9 * (size_t)slot;
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
        for (int q = 0; q < 3; q++) o[3 * p + q] = dir ? 0.0 : H[p][q];
}

__device__ __forceinline__ void add_grad(double* fb, int v, d3 g) {
    atomicAdd(fb + 3 * v, g.x);
    atomicAdd(fb + 3 * v + 1, g.y);
    atomicAdd(fb + 3 * v + 2, g.z);
}

// Decoded barrier pair: kind 0 PP, 1 PE, 2 PT, 3 EE, 4 mollified EE, 5 mollified PE,
// 6 mollified PP (encoding of StiffGIPC/mlbvh.cu:560-1059, decoded as GIPC.cu:3131-4945)
__device__ __forceinline__ int decode_pair(int4 e, int* v, int& nvp) {
    if (e.x >= 0) {
        v[0] = e.x; v[1] = e.y; v[2] = e.z;
        if (e.w >= 0) { v[3] = e.w; nvp = 4; return 3; }
        v[3] = -e.w - 1; nvp = 4; return 4;
    }
    v[0] = -e.x - 1;
    if (e.z < 0) {
        if (e.y < 0) { v[1] = -e.y - 1; v[2] = -e.z - 1; v[3] = -e.w - 1; nvp = 4; return 6; }
        v[1] = e.y; v[2] = v[3] = 0; nvp = 2; return 0;
    }
    if (e.w < 0) {
        if (e.y < 0) { v[1] = -e.y - 1; v[2] = e.z; v[3] = -e.w - 1; nvp = 4; return 5; }
        v[1] = e.y; v[2] = e.z; v[3] = 0; nvp = 3; return 1;
    }
    v[1] = e.y; v[2] = e.z; v[3] = e.w; nvp = 4; return 2;
}

// squared distance and its gradient (hand-derived, see the derivation in each branch)
__device__ __forceinline__ double dist2_grad(int kind, const d3* X, d3* g) {
    if (kind == 0 || kind == 6) {  // |a - b|^2
        d3 d = X[0] - X[1];
        g[0] = 2.0 * d;
        g[1] = -2.0 * d;
        g[2] = g[3] = mk(0, 0, 0);
        return sq(d);
    }
    if (kind == 1 || kind == 5) {  // |(e0-p) x (e1-p)|^2 / |e1-e0|^2
        d3 p = X[0], e0 = X[1], e1 = X[2];
        d3 c = cross(e0 - p, e1 - p), e = e1 - e0;
        double L = sq(e), C = sq(c);
        d3 gp = 2.0 * cross(c, e), ge0 = 2.0 * cross(e1 - p, c), ge1 = 2.0 * cross(c, e0 - p);
        double iL = 1.0 / L, r = C * iL * iL;
        g[0] = iL * gp;
        g[1] = iL * ge0 + (2.0 * r) * e;
        g[2] = iL * ge1 - (2.0 * r) * e;
        g[3] = mk(0, 0, 0);
        return C * iL;
    }
    if (kind == 2) {  // s^2 / |n|^2, n = (t1-t0) x (t2-t0), s = (p - t0).n
        d3 p = X[0], t0 = X[1], t1 = X[2], t2 = X[3];
        d3 e1 = t1 - t0, e2 = t2 - t0, w = p - t0;
        d3 n = cross(e1, e2);
        double s = dot(w, n), N = sq(n), iN = 1.0 / N;
        d3 sp = n, s0 = cross(e1 - e2, w) - n, s1 = cross(e2, w), s2 = cross(w, e1);
        d3 N0 = 2.0 * cross(e1 - e2, n), N1 = 2.0 * cross(e2, n), N2 = 2.0 * cross(n, e1);
        double a = 2.0 * s * iN, b = s * s * iN * iN;
        g[0] = a * sp;
        g[1] = a * s0 - b * N0;
        g[2] = a * s1 - b * N1;
        g[3] = a * s2 - b * N2;
        return s * s * iN;
    }
    // EE: s^2/|n|^2, n = (a1-a0) x (b1-b0), s = (b0 - a0).n
    d3 a0 = X[0], a1 = X[1], b0 = X[2], b1 = X[3];
    d3 u = a1 - a0, v = b1 - b0, w = b0 - a0;
    d3 n = cross(u, v);
    double s = dot(w, n), N = sq(n), iN = 1.0 / N;
    d3 vw = cross(v, w), wu = cross(w, u), vn = cross(v, n), nu = cross(n, u);
    double a = 2.0 * s * iN, b = s * s * iN * iN;
    g[0] = a * (-1.0 * n - vw) + (2.0 * b) * vn;
    g[1] = a * vw - (2.0 * b) * vn;
    g[2] = a * (n - wu) + (2.0 * b) * nu;
    g[3] = a * wu - (2.0 * b) * nu;
    return s * s * iN;
}

// B(I) = c (I-1)^2 ln(I)^2 and its first two derivatives in I
__device__ __forceinline__ void barrier_s(double I, double c, double& B, double& dB, double& d2B) {
    double L = log(I), t = I - 1.0;
    B = c * t * t * L * L;
    dB = c * (2.0 * t * L * L + 2.0 * t * t * L / I);
    d2B = c * (2.0 * L * L + 8.0 * t * L / I + 2.0 * t * t * (1.0 - L) / (I * I));
}

__device__ __forceinline__ void barrier_one(int p, int np, const int4* __restrict__ pairs,
                                            const double* __restrict__ x, const double* __restrict__ rest,
                                            double dhat, double kappa, double* __restrict__ fb, BlockSink bs,
                                            int base) {
    int v[4], nvp;
    int kind = decode_pair(pairs[p], v, nvp);
    if (!ids_ok(bs, v, nvp)) {
        emit_pair_blocks(bs, base + 10 * p, 0, v, [&](int, int, double H[3][3]) {});
        return;
    }
    d3 X[4];
#pragma unroll
    for (int a = 0; a < 4; a++) X[a] = a < nvp ? ld3(x, v[a]) : mk(0, 0, 0);
    d3 gd2[4];
    double d2 = dist2_grad(kind, X, gd2);
    const double sdh = sqrt(dhat), dist = sqrt(d2);
    const double I = d2 / dhat, f = sqrt(I);
    d3 gf[4];
#pragma unroll
    for (int a = 0; a < 4; a++) gf[a] = (1.0 / (2.0 * dist * sdh)) * gd2[a];
    if (kind <= 3) {
        double B, dB, d2B;
        barrier_s(I, kappa * dhat * dhat, B, dB, d2B);
        double dBdf = 2.0 * f * dB;
        double Ic = d2 < 1e-6 * dhat ? 1e-6 : I;  // gassThreshold clamp (GIPC.cu:3258-3272)
        double Bc, dBc, d2Bc;
        barrier_s(Ic, kappa * dhat * dhat, Bc, dBc, d2Bc);
        double lam0 = 4.0 * Ic * d2Bc + 2.0 * dBc;
        for (int a = 0; a < 4; a++) if (a < nvp) add_grad(fb, v[a], dBdf * gf[a]);
        emit_pair_blocks(bs, base + 10 * p, nvp, v, [&](int a, int b, double H[3][3]) {
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) H[i][j] = lam0 * comp(gf[a], i) * comp(gf[b], j);
        });
        return;
    }
    // mollified pairs: b = kappa e(c^2) Bt(I), c = |edge0 x edge1|
    int ea0, ea1, eb0, eb1;
    if (kind == 4) { ea0 = 0; ea1 = 1; eb0 = 2; eb1 = 3; }
    else if (kind == 6) { ea0 = 0; ea1 = 2; eb0 = 1; eb1 = 3; }
    else { ea0 = 0; ea1 = 3; eb0 = 1; eb1 = 2; }
    d3 u = X[ea1] - X[ea0], w = X[eb1] - X[eb0];
    d3 n = cross(u, w);
    double I1 = sq(n);
    if (I1 == 0.0) {
        emit_pair_blocks(bs, base + 10 * p, 0, v, [&](int, int, double H[3][3]) {});
        return;
    }
    double c = sqrt(I1);
    d3 gc[4];
    {
        d3 wn = cross(w, n), nu = cross(n, u);
        double k = 1.0 / (2.0 * c);
        gc[ea0] = (-2.0 * k) * wn;
        gc[ea1] = (2.0 * k) * wn;
        gc[eb0] = (-2.0 * k) * nu;
        gc[eb1] = (2.0 * k) * nu;
    }
    d3 r0 = ld3(rest, v[ea0]), r1 = ld3(rest, v[ea1]), r2 = ld3(rest, v[eb0]), r3 = ld3(rest, v[eb1]);
    double ex = 1e-3 * sq(r0 - r1) * sq(r2 - r3);  // _compute_epx, mlbvh.cu:264
    double em = -I1 * I1 / (ex * ex) + 2.0 * I1 / ex;
    double dem = -2.0 * I1 / (ex * ex) + 2.0 / ex;
    double B, dB, d2B;
    barrier_s(I, dhat * dhat, B, dB, d2B);
    double dbdc = kappa * dem * 2.0 * c * B, dbdf = kappa * em * dB * 2.0 * f;
    for (int a = 0; a < 4; a++) add_grad(fb, v[a], dbdc * gc[a] + dbdf * gf[a]);
    double M00 = kappa * B * (-4.0 * (3.0 * I1 - ex) / (ex * ex));
    double M11 = kappa * em * (4.0 * I * d2B + 2.0 * dB);
    double M01 = kappa * dem * 2.0 * c * dB * 2.0 * f;
    make_pd2(M00, M01, M11);
    emit_pair_blocks(bs, base + 10 * p, 4, v, [&](int a, int b, double H[3][3]) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
                H[i][j] = M00 * comp(gc[a], i) * comp(gc[b], j) +
                          M01 * (comp(gc[a], i) * comp(gf[b], j) + comp(gf[a], i) * comp(gc[b], j)) +
                          M11 * comp(gf[a], i) * comp(gf[b], j);
    });
}

__global__ void __launch_bounds__(128) k_barrier(int np, const int4* __restrict__ pairs, const double* __restrict__ x,
                                                 const double* __restrict__ rest, double dhat, double kappa,
                                                 double* __restrict__ fb, BlockSink bs, int base) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    barrier_one(p, np, pairs, x, rest, dhat, kappa, fb, bs, base);
}

// friction pairs (FrictionUtils.cuh, GIPC.cu:1439-1800 and 5087-5270), C1 static clamping
__device__ __forceinline__ void friction_one(int p, int np, const int4* __restrict__ pairs,
                                             const double* __restrict__ x, const double* __restrict__ x0,
                                             const double* __restrict__ lam, const double* __restrict__ coord,
                                             const double* __restrict__ basis, double mu, double eps2,
                                             double* __restrict__ fb, BlockSink bs, int base) {
    int4 e = pairs[p];
    int v[4] = {0, 0, 0, 0}, nvp = 0;
    double cf[4] = {0, 0, 0, 0};
    double g1 = coord[2 * p], g2 = coord[2 * p + 1];
    if (e.x >= 0) {
        if (e.w >= 0) {
            v[0] = e.x; v[1] = e.y; v[2] = e.z; v[3] = e.w; nvp = 4;
            cf[0] = 1.0 - g1; cf[1] = g1; cf[2] = g2 - 1.0; cf[3] = -g2;
        }
    } else if (e.y >= 0) {
        v[0] = -e.x - 1;
        if (e.z < 0) { v[1] = e.y; nvp = 2; cf[0] = 1.0; cf[1] = -1.0; }
        else if (e.w < 0) { v[1] = e.y; v[2] = e.z; nvp = 3; cf[0] = 1.0; cf[1] = g1 - 1.0; cf[2] = -g1; }
        else { v[1] = e.y; v[2] = e.z; v[3] = e.w; nvp = 4; cf[0] = 1.0; cf[1] = -1.0 + g1 + g2; cf[2] = -g1; cf[3] = -g2; }
    }
    if (nvp == 0 || !ids_ok(bs, v, nvp)) {
        emit_pair_blocks(bs, base + 10 * p, 0, v, [&](int, int, double H[3][3]) {});
        return;
    }
    const double* Tb = basis + 6 * (size_t)p;  // 3x2 row-major
    d3 t0 = mk(Tb[0], Tb[2], Tb[4]), t1 = mk(Tb[1], Tb[3], Tb[5]);
    d3 rel = mk(0, 0, 0);
    for (int a = 0; a < nvp; a++) rel = rel + cf[a] * (ld3(x, v[a]) - ld3(x0, v[a]));
    double u0 = dot(t0, rel), u1 = dot(t1, rel);
    double un2 = u0 * u0 + u1 * u1, un = sqrt(un2), eps = sqrt(eps2);
    double f1d, M00, M01, M11;
    if (un2 > eps2) {
        f1d = 1.0 / un;
        double k = 1.0 / (un2 * un);
        M00 = f1d - k * u0 * u0; M01 = -k * u0 * u1; M11 = f1d - k * u1 * u1;
    } else {
        f1d = (-un + 2.0 * eps) / (eps * eps);
        double f2 = 2.0 * (eps - un) / (eps * eps);
        if (f2 != f1d && un2 != 0.0) {
            double k = (f1d - f2) / un2;
            M00 = f1d - k * u0 * u0; M01 = -k * u0 * u1; M11 = f1d - k * u1 * u1;
        } else {
            M00 = M11 = f1d; M01 = 0.0;
        }
    }
    make_pd2(M00, M01, M11);
    const double s = mu * lam[p];
    d3 gt = (s * f1d) * (u0 * t0 + u1 * t1);
    for (int a = 0; a < 4; a++) if (a < nvp) add_grad(fb, v[a], cf[a] * gt);
    // W = basis M basis^T
    double W[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double ti0 = comp(t0, i), ti1 = comp(t1, i), tj0 = comp(t0, j), tj1 = comp(t1, j);
            W[i][j] = s * (ti0 * (M00 * tj0 + M01 * tj1) + ti1 * (M01 * tj0 + M11 * tj1));
        }
    emit_pair_blocks(bs, base + 10 * p, nvp, v, [&](int a, int b, double H[3][3]) {
        double k = cf[a] * cf[b];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) H[i][j] = k * W[i][j];
    });
}

__global__ void __launch_bounds__(128) k_friction(int np, const int4* __restrict__ pairs, const double* __restrict__ x,
                                                  const double* __restrict__ x0, const double* __restrict__ lam,
                                                  const double* __restrict__ coord, const double* __restrict__ basis,
                                                  double mu, double eps2, double* __restrict__ fb, BlockSink bs,
                                                  int base) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    friction_one(p, np, pairs, x, x0, lam, coord, basis, mu, eps2, fb, bs, base);
}

// ground barrier (GIPC.cu:6463-6514), plane y = offset
__device__ __forceinline__ void ground_one(int p, int ng, const uint32_t* __restrict__ gp,
                                           const double* __restrict__ x, double offset, double dhat, double kappa,
                                           double* __restrict__ fb, BlockSink bs, int base) {
    int v = gp[p];
    if (!ids_ok(bs, &v, 1)) {
        bs.idx[base + p] = base + p;
        bs.key[base + p] = kBadKey;
        return;
    }
    double dist = x[3 * v + 1] - offset, d2 = dist * dist, t = d2 - dhat;
    double gb = t * log(d2 / dhat) * -2.0 - (t * t) / d2;
    double hb = (log(d2 / dhat) * -2.0 - t * 4.0 / d2) + 1.0 / (d2 * d2) * (t * t);
    atomicAdd(fb + 3 * v + 1, kappa * gb * 2.0 * dist);
    double H[3][3] = {{0, 0, 0}, {0, kappa * (4.0 * hb * d2 + 2.0 * gb), 0}, {0, 0, 0}};
    emit_diag_block(bs, base + p, v, H);
}


// ground friction (GIPC.cu:1357-1437, 5047-5085), normal +y
__device__ __forceinline__ void fric_ground_one(int p, int ng, const uint32_t* __restrict__ gp,
                                                const double* __restrict__ x, const double* __restrict__ x0,
                                                const double* __restrict__ lam, double mu, double eps2,
                                                double* __restrict__ fb, BlockSink bs, int base) {
    int v = gp[p];
    if (!ids_ok(bs, &v, 1)) {
        bs.idx[base + p] = base + p;
        bs.key[base + p] = kBadKey;
        return;
    }
    double vx = x[3 * v] - x0[3 * v], vz = x[3 * v + 2] - x0[3 * v + 2];
    double m2 = vx * vx + vz * vz, s = mu * lam[p], eps = sqrt(eps2);
    double H[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (m2 > eps2) {
        double m = sqrt(m2), k = s / (m2 * m);
        atomicAdd(fb + 3 * v, s * vx / m);
        atomicAdd(fb + 3 * v + 2, s * vz / m);
        double a = s / m - k * vx * vx, b = -k * vx * vz, c = s / m - k * vz * vz;
        make_pd2(a, b, c);
        H[0][0] = a; H[0][2] = b; H[2][0] = b; H[2][2] = c;
    } else {
        atomicAdd(fb + 3 * v, s * vx / eps);
        atomicAdd(fb + 3 * v + 2, s * vz / eps);
        H[0][0] = s / eps;
        H[2][2] = s / eps;
    }
    emit_diag_block(bs, base + p, v, H);
}


// All contact terms of a call in one launch: the CTAs take the barrier pairs, then the
// friction pairs, then the ground and the ground-friction vertices (128 threads each), so the
// four kinds run side by side instead of one after another.
struct ContactLaunch {
    int np, nf, ng, ngf;           // items of each kind (0: none)
    int cb, cf, cg;                // first CTA of friction, ground, ground friction
    const int4* pairs;
    const int4* fpairs;
    const uint32_t* gpairs;
    const uint32_t* gfpairs;
    const double* x;
    const double* x0;
    const double* rest;
    const double* flam;
    const double* fcoord;
    const double* fbasis;
    const double* gflam;
    double dhat, kappa, mu, gmu, eps2, offset;
    int base_b, base_f, base_g, base_gf;
};

__global__ void __launch_bounds__(128) k_contacts(ContactLaunch L, double* __restrict__ fb, BlockSink bs) {
    const int b = blockIdx.x;
    if (b < L.cb) {
        const int p = b * 128 + threadIdx.x;
        if (p < L.np) barrier_one(p, L.np, L.pairs, L.x, L.rest, L.dhat, L.kappa, fb, bs, L.base_b);
    } else if (b < L.cf) {
        const int p = (b - L.cb) * 128 + threadIdx.x;
        if (p < L.nf)
            friction_one(p, L.nf, L.fpairs, L.x, L.x0, L.flam, L.fcoord, L.fbasis, L.mu, L.eps2, fb, bs, L.base_f);
    } else if (b < L.cg) {
        const int p = (b - L.cf) * 128 + threadIdx.x;
        if (p < L.ng) ground_one(p, L.ng, L.gpairs, L.x, L.offset, L.dhat, L.kappa, fb, bs, L.base_g);
    } else {
        const int p = (b - L.cg) * 128 + threadIdx.x;
        if (p < L.ngf) fric_ground_one(p, L.ngf, L.gfpairs, L.x, L.x0, L.gflam, L.gmu, L.eps2, fb, bs, L.base_gf);
    }
}

// soft constraints (GIPC.cu:6363-6407)
__global__ void k_soft(int ns, const uint32_t* __restrict__ idx, const double* __restrict__ x,
                       const double* __restrict__ target, double k, double* __restrict__ sg, BlockSink bs, int base) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ns) return;
    int v = idx[p];
    for (int q = 0; q < 3; q++) atomicAdd(sg + 3 * v + q, k * (x[3 * v + q] - target[3 * p + q]));
    double H[3][3] = {{k, 0, 0}, {0, k, 0}, {0, 0, k}};
    emit_diag_block(bs, base + p, v, H);
}

// ---- contact block merge ------------------------------------------------------------------
// run heads of the sorted keys (the unused-slot key forms no run); flag[m] = 0
__global__ void k_run_heads(int m, const unsigned long long* __restrict__ ks, int* __restrict__ flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    if (i == m) {
        flag[m] = 0;
        return;
    }
    const unsigned long long k = ks[i];
    flag[i] = (k != kBadKey && (i == 0 || ks[i - 1] != k)) ? 1 : 0;
}

// after the exclusive scan flag[i] = run id of head i; start[u] = first sorted index of run
// u, start[nuc] = end of the last run; row / column of every unique block
__global__ void k_run_starts(int m, const unsigned long long* __restrict__ ks, const int* __restrict__ rid, int bits,
                             int* __restrict__ start, int* __restrict__ uc_row, int* __restrict__ uc_col,
                             int* __restrict__ nuc, int* __restrict__ lcount) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    // end of the last run: the first unused-slot key (sorted last), or m; written by the
    // thread at that boundary (a binary search by one thread took ~19 round trips)
    {
        const bool here = i == m ? (m == 0 || ks[m - 1] != kBadKey) : (ks[i] == kBadKey && (i == 0 || ks[i - 1] != kBadKey));
        if (here) {
            const int nu = rid[m];
            nuc[0] = nu;
            start[nu] = i;
        }
    }
    if (i == m) return;
    const unsigned long long k = ks[i];
    if (k == kBadKey || (i > 0 && ks[i - 1] == k)) return;
    const int u = rid[i];
    start[u] = i;
    const unsigned long long mask = (1ull << bits) - 1ull;
    const int row = (int)(k >> bits), col = (int)(k & mask);
    uc_row[u] = row;
    uc_col[u] = col;
    // off-diagonal blocks also appear transposed, in the list of row `col`
    if (row != col) atomicAdd(lcount + col, 1);
}

// ... and entry q of the transposed copy at slot lpos[u] gets entry q of the block, at its
// transposed place 3 (q % 3) + q / 3
// One warp per unique block (grid-stride over the blocks): lane l adds the run's slots l,
// l + 32, ... in order, then a fixed xor tree adds the lanes, so the sum is the same run to
// run; lanes 0..8 store the nine entries (upper and, transposed, lower copies).
__global__ void __launch_bounds__(256) k_run_sums(const int* __restrict__ nuc, const int* __restrict__ start,
                                                  const int* __restrict__ is, const double* __restrict__ cval,
                                                  const int* __restrict__ lpos, double* __restrict__ u64,
                                                  float* __restrict__ u32, double* __restrict__ l64,
                                                  float* __restrict__ l32) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int nu = nuc[0];
    for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < nu; u += nw) {
        const int j0 = start[u], j1 = start[u + 1];
        double acc[9];
#pragma unroll
        for (int q = 0; q < 9; q++) acc[q] = 0.0;
        for (int j = j0 + lane; j < j1; j += 32) {
            const double* v = cval + 9 * (size_t)is[j];
#pragma unroll
            for (int q = 0; q < 9; q++) acc[q] += v[q];
        }
#pragma unroll
        for (int q = 0; q < 9; q++)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        if (lane < 9) {
            double a = acc[0];
#pragma unroll
            for (int q = 1; q < 9; q++)
                if (lane == q) a = acc[q];
            u64[9 * (size_t)u + lane] = a;
            u32[9 * (size_t)u + lane] = (float)a;
            const int k = lpos[u];
            if (k >= 0) {
                const int qt = 3 * (lane % 3) + lane / 3;
                l64[9 * (size_t)k + qt] = a;
                l32[9 * (size_t)k + qt] = (float)a;
            }
        }
    }
}

// upper row pointers (thread i <= n: first unique block whose row >= i, by binary search over
// the row-sorted blocks) and placement of each off-diagonal block u in the transposed list of
// row uc_col[u], in the order the atomics hand out the slots
__global__ void k_lower_place(int m, int n, const int* __restrict__ nuc, const int* __restrict__ uc_row,
                              const int* __restrict__ uc_col, const int* __restrict__ cl_ptr, int* __restrict__ fill,
                              int* __restrict__ cu_ptr, int* __restrict__ cl_idx) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nu = nuc[0];
    if (t <= n) {
        // first block with row >= t: an 8-way search, seven probes in flight per step (five
        // round trips for 30 000 blocks instead of fifteen)
        int lo = 0, hi = nu;
        while (hi - lo > 8) {
            const int step = (hi - lo + 7) >> 3;
            int below = 0;  // probes lo + step .. lo + 7 step with row < t
#pragma unroll
            for (int j = 1; j < 8; j++) {
                const int p = lo + j * step;
                below += (p < hi && uc_row[p] < t) ? 1 : 0;
            }
            // the answer lies in (lo + below * step, lo + (below + 1) * step]
            const int nlo = lo + below * step, nhi = min(hi, lo + (below + 1) * step);
            lo = below > 0 ? nlo + 1 : lo;
            hi = nhi;
            if (below > 0 && lo > hi) lo = hi;
        }
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (uc_row[mid] < t) lo = mid + 1; else hi = mid;
        }
        cu_ptr[t] = lo;
    }
    if (t < nu) {
        const int col = uc_col[t];
        if (uc_row[t] != col) cl_idx[cl_ptr[col] + atomicAdd(fill + col, 1)] = t;
    }
}

// final slot of each off-diagonal block in its transposed list: its rank by row among the
// blocks of the same column, so that every transposed list is sorted by column whatever order
// the placement atomics took; lpos[u] = -1 for diagonal blocks
__global__ void k_lower_rank(const int* __restrict__ nuc, const int* __restrict__ uc_row,
                             const int* __restrict__ uc_col, const int* __restrict__ cl_ptr,
                             const int* __restrict__ cl_idx, int* __restrict__ lpos, int* __restrict__ cl_col) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nuc[0]) return;
    const int row = uc_row[u], col = uc_col[u];
    if (row == col) {
        lpos[u] = -1;
        return;
    }
    const int k0 = cl_ptr[col], k1 = cl_ptr[col + 1];
    int rank = 0;
    int k = k0;
    for (; k + 4 <= k1; k += 4) {  // four list entries in flight
        int ix[4];
#pragma unroll
        for (int u = 0; u < 4; u++) ix[u] = __ldg(cl_idx + k + u);
#pragma unroll
        for (int u = 0; u < 4; u++) rank += __ldg(uc_row + ix[u]) < row;
    }
    for (; k < k1; k++) rank += __ldg(uc_row + __ldg(cl_idx + k)) < row;
    lpos[u] = k0 + rank;
    cl_col[k0 + rank] = row;
}


// ------------------------------------------------------------------------------------------
// line-search energy (GIPC::computeEnergy, GIPC.cu:10520-10580; per-term reductions
// Energy_Add_Reduction_Algorithm, GIPC.cu:10347-10518).  Each kernel writes one partial sum
// per CTA; every sum runs in a fixed order, so the energy is the same bit for bit on every
// run.  The scalings of computeEnergy (dt^2 on the elastic terms, kappa, the friction rates)
// are applied per element, as in the gradient kernels above.
// ------------------------------------------------------------------------------------------
// fixed-order CTA sum of one value per thread into part[blockIdx.x]; every thread calls it
__device__ __forceinline__ void cta_energy(double e, double* __restrict__ part) {
    __shared__ double sw[SGIPC_BLOCK / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sw[w];
        part[blockIdx.x] = t;
    }
}

// kinetic 1/2 m |x - x_tilde|^2 (_getKineticEnergy_Reduction_3D)
__device__ __forceinline__ double en_kinetic(int gi, int nv, const double* __restrict__ x, const double* __restrict__ xt,
                             const double* __restrict__ m) {
    const int i = gi;
    double e = 0.0;
    if (i < nv) {
        const d3 d = ld3(x, i) - ld3(xt, i);
        e = 0.5 * m[i] * sq(d);
    }
    return e;
}

// stable Neo-Hookean: dt^2 vol 1/2 (mu (|F|^2 - 3) + lam (J - 1 - mu/lam)^2)
// (_getFEMEnergy_Reduction_3D; femEnergy.cu:1042-1050)
__device__ __forceinline__ double en_snk(int gi, int nt, const uint32_t* __restrict__ tets, const double* __restrict__ x,
                         const double* __restrict__ dminv, const double* __restrict__ vol,
                         const double* __restrict__ lr, const double* __restrict__ vr, double dt2) {
    const int t = gi;
    double e = 0.0;
    if (t < nt) {
        const uint4 tv = reinterpret_cast<const uint4*>(tets)[t];
        const d3 X0 = ld3(x, tv.x), e1 = ld3(x, tv.y) - X0, e2 = ld3(x, tv.z) - X0, e3 = ld3(x, tv.w) - X0;
        const double* Di = dminv + 9 * (size_t)t;
        double F[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) F[i][j] = comp(e1, i) * Di[j] + comp(e2, i) * Di[3 + j] + comp(e3, i) * Di[6 + j];
        double I2 = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) I2 += F[i][j] * F[i][j];
        const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                         F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                         F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
        const double mu = lr[t], lam = vr[t], Jm = J - 1.0 - mu / lam;
        e = 0.5 * (mu * (I2 - 3.0) + lam * Jm * Jm) * vol[t] * dt2;
    }
    return e;
}

// cloth membrane: dt^2 area (kst sum_j S(|f_j|) + ksh (f_0 . f_1)^2), S(t) = (t-1)^2 (+ srate
// (t-1)^3 when stretched) (_getFEMEnergy_Reduction_3D_triangle, femEnergy.cu:351-403)
__device__ __forceinline__ double en_tri(int gi, int nf, const uint32_t* __restrict__ tris, const double* __restrict__ x,
                         const double* __restrict__ dminv, const double* __restrict__ area, double kst, double ksh,
                         double srate, double dt2) {
    const int f = gi;
    double e = 0.0;
    if (f < nf) {
        const d3 x0 = ld3(x, tris[3 * f]), e1 = ld3(x, tris[3 * f + 1]) - x0, e2 = ld3(x, tris[3 * f + 2]) - x0;
        const double* Di = dminv + 4 * (size_t)f;
        const d3 col[2] = {Di[0] * e1 + Di[2] * e2, Di[1] * e1 + Di[3] * e2};
        double E = 0.0;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const double t = sqrt(sq(col[j])), u = t - 1.0;
            E += kst * (u * u + (t > 1.0 ? srate * u * u * u : 0.0));
        }
        const double I6 = dot(col[0], col[1]);
        E += ksh * I6 * I6;
        e = E * area[f] * dt2;
    }
    return e;
}

// quadratic bending: 1/2 c sum_ab Q_ab x_a . x_b, c = |rest e| bendStiff dt^2; boundary
// edges (a missing wing) carry none (femEnergy.cu:2623-2753)
__device__ __forceinline__ double en_hinge(int gi, int nh, const uint32_t* __restrict__ edges, const int32_t* __restrict__ adj,
                           const double* __restrict__ x, const double* __restrict__ rest,
                           const double* __restrict__ Qcm, double kb_dt2) {
    const int h = gi;
    double e = 0.0;
    if (h < nh && adj[2 * h] >= 0 && adj[2 * h + 1] >= 0) {
        const int v[4] = {(int)edges[2 * h], (int)edges[2 * h + 1], adj[2 * h], adj[2 * h + 1]};
        const double c = sqrt(sq(ld3(rest, v[0]) - ld3(rest, v[1]))) * kb_dt2;
        d3 xv[4];
#pragma unroll
        for (int a = 0; a < 4; a++) xv[a] = ld3(x, v[a]);
        double E = 0.0;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            d3 g = mk(0, 0, 0);
#pragma unroll
            for (int b = 0; b < 4; b++) g = g + Qcm[16 * (size_t)h + 4 * b + a] * xv[b];
            E += 0.5 * c * dot(xv[a], g);
        }
        e = E;
    }
    return e;
}

// soft constraints 1/2 k |x - target|^2, k = motionRate softRate^2 (GIPC.cu:6363-6407)
__device__ __forceinline__ double en_soft(int gi, int ns, const uint32_t* __restrict__ idx, const double* __restrict__ x,
                          const double* __restrict__ target, double k) {
    const int p = gi;
    double e = 0.0;
    if (p < ns) e = 0.5 * k * sq(ld3(x, idx[p]) - ld3(target, p));
    return e;
}

// barrier pairs: kappa dhat^2 (I-1)^2 ln^2 I, I = d^2/dhat; mollified EE / PE / PP pairs
// times e(c^2) (_getBarrierEnergy_Reduction_3D, GIPC.cu:701-958)
__device__ __forceinline__ double en_barrier(int gi, int np, int nv, const int4* __restrict__ pairs, const double* __restrict__ x,
                             const double* __restrict__ rest, double dhat, double kappa) {
    const int p = gi;
    double e = 0.0;
    if (p < np) {
        int v[4], nvp;
        const int kind = decode_pair(pairs[p], v, nvp);
        bool ok = true;
        for (int a = 0; a < nvp; a++) ok = ok && v[a] >= 0 && v[a] < nv;
        if (ok) {
            d3 X[4], gd2[4];
#pragma unroll
            for (int a = 0; a < 4; a++) X[a] = a < nvp ? ld3(x, v[a]) : mk(0, 0, 0);
            const double I = dist2_grad(kind, X, gd2) / dhat;
            double B, dB, d2B;
            if (kind <= 3) {
                barrier_s(I, kappa * dhat * dhat, B, dB, d2B);
                e = B;
            } else {
                int ea0, ea1, eb0, eb1;
                if (kind == 4) { ea0 = 0; ea1 = 1; eb0 = 2; eb1 = 3; }
                else if (kind == 6) { ea0 = 0; ea1 = 2; eb0 = 1; eb1 = 3; }
                else { ea0 = 0; ea1 = 3; eb0 = 1; eb1 = 2; }
                const double I1 = sq(cross(X[ea1] - X[ea0], X[eb1] - X[eb0]));
                if (I1 != 0.0) {
                    const double ex = 1e-3 * sq(ld3(rest, v[ea0]) - ld3(rest, v[ea1])) *
                                      sq(ld3(rest, v[eb0]) - ld3(rest, v[eb1]));
                    const double em = -I1 * I1 / (ex * ex) + 2.0 * I1 / ex;
                    barrier_s(I, dhat * dhat, B, dB, d2B);
                    e = kappa * em * B;
                }
            }
        }
    }
    return e;
}

// ground barrier -kappa (d^2 - dhat)^2 ln(d^2/dhat), d = y - offset (GIPC.cu:6463-6514)
__device__ __forceinline__ double en_ground(int gi, int ng, int nv, const uint32_t* __restrict__ gp, const double* __restrict__ x,
                            double offset, double dhat, double kappa) {
    const int p = gi;
    double e = 0.0;
    if (p < ng && (int)gp[p] < nv) {
        const double dist = x[3 * gp[p] + 1] - offset, d2 = dist * dist, t = d2 - dhat;
        e = -kappa * t * t * log(d2 / dhat);
    }
    return e;
}

// pair friction mu lambda f0(|u|): f0 = |u| beyond eps, else |u|^2 (eps - |u|/3) / eps^2 +
// eps/3 (_getFrictionEnergy_Reduction_3D, GIPC.cu:1252-1356)
__device__ __forceinline__ double en_friction(int gi, int np, int nv, const int4* __restrict__ pairs, const double* __restrict__ x,
                              const double* __restrict__ x0, const double* __restrict__ lam,
                              const double* __restrict__ coord, const double* __restrict__ basis, double mu,
                              double eps2) {
    const int p = gi;
    double e = 0.0;
    if (p < np) {
        const int4 q = pairs[p];
        int v[4] = {0, 0, 0, 0}, nvp = 0;
        double cf[4] = {0, 0, 0, 0};
        const double g1 = coord[2 * p], g2 = coord[2 * p + 1];
        if (q.x >= 0) {
            if (q.w >= 0) {
                v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w; nvp = 4;
                cf[0] = 1.0 - g1; cf[1] = g1; cf[2] = g2 - 1.0; cf[3] = -g2;
            }
        } else if (q.y >= 0) {
            v[0] = -q.x - 1;
            if (q.z < 0) { v[1] = q.y; nvp = 2; cf[0] = 1.0; cf[1] = -1.0; }
            else if (q.w < 0) { v[1] = q.y; v[2] = q.z; nvp = 3; cf[0] = 1.0; cf[1] = g1 - 1.0; cf[2] = -g1; }
            else { v[1] = q.y; v[2] = q.z; v[3] = q.w; nvp = 4; cf[0] = 1.0; cf[1] = -1.0 + g1 + g2; cf[2] = -g1; cf[3] = -g2; }
        }
        bool ok = nvp > 0;
        for (int a = 0; a < nvp; a++) ok = ok && v[a] >= 0 && v[a] < nv;
        if (ok) {
            const double* Tb = basis + 6 * (size_t)p;
            const d3 t0 = mk(Tb[0], Tb[2], Tb[4]), t1 = mk(Tb[1], Tb[3], Tb[5]);
            d3 rel = mk(0, 0, 0);
            for (int a = 0; a < nvp; a++) rel = rel + cf[a] * (ld3(x, v[a]) - ld3(x0, v[a]));
            const double u0 = dot(t0, rel), u1 = dot(t1, rel);
            const double un2 = u0 * u0 + u1 * u1, un = sqrt(un2), eps = sqrt(eps2);
            const double f0 = un2 > eps2 ? un : un2 * (-un / 3.0 + eps) / (eps * eps) + eps / 3.0;
            e = mu * lam[p] * f0;
        }
    }
    return e;
}

// ground friction mu lambda (|v| - eps/2) beyond eps, else mu lambda |v|^2 / (2 eps), v the
// tangential (x, z) step (_getFrictionEnergy_gd_Reduction_3D, GIPC.cu:1357-1437)
__device__ __forceinline__ double en_fric_ground(int gi, int ng, int nv, const uint32_t* __restrict__ gp, const double* __restrict__ x,
                                 const double* __restrict__ x0, const double* __restrict__ lam, double mu,
                                 double eps2) {
    const int p = gi;
    double e = 0.0;
    if (p < ng && (int)gp[p] < nv) {
        const int v = gp[p];
        const double vx = x[3 * v] - x0[3 * v], vz = x[3 * v + 2] - x0[3 * v + 2];
        const double m2 = vx * vx + vz * vz, s = mu * lam[p], eps = sqrt(eps2);
        e = m2 > eps2 ? s * (sqrt(m2) - eps * 0.5) : s * m2 / eps * 0.5;
    }
    return e;
}

// Everything in one launch: CTA b evaluates term t where off[t] <= b < off[t + 1] (its
// elements (b - off[t]) * blockDim + threadIdx), stores its partial, and the last CTA to
// finish (a ticket counter, reset by that CTA) sums each term's partials in order into
// terms[t] and their total into terms[9].
struct EnergyOffsets {
    int off[10];
};
struct EnergyArgs {
    int nv, nt, nf, nh, ns, npair, nground, nfric, nfg;
    const double *x, *xt, *m, *x0, *rest;
    const uint32_t *tets, *tris, *hinges, *soft_idx, *gp, *fgp;
    const int32_t* adj;
    const int4 *pairs, *fpairs;
    const double *dminv, *vol, *lr, *vr, *tdminv, *area, *Q, *target, *flam, *coord, *basis, *fglam;
    double dt2, kst, ksh, srate, kb_dt2, ksoft, dhat, kappa, offset, mu, mu_gd, eps2;
};
__global__ void __launch_bounds__(SGIPC_BLOCK) k_energy(EnergyArgs a, EnergyOffsets o, double* __restrict__ part,
                                                        double* __restrict__ terms, unsigned int* __restrict__ ticket) {
    int t = 0;
    while (t < 8 && (int)blockIdx.x >= o.off[t + 1]) t++;
    const int gi = ((int)blockIdx.x - o.off[t]) * blockDim.x + threadIdx.x;
    double e = 0.0;
    switch (t) {
        case 0: e = en_kinetic(gi, a.nv, a.x, a.xt, a.m); break;
        case 1: e = en_snk(gi, a.nt, a.tets, a.x, a.dminv, a.vol, a.lr, a.vr, a.dt2); break;
        case 2: e = en_tri(gi, a.nf, a.tris, a.x, a.tdminv, a.area, a.kst, a.ksh, a.srate, a.dt2); break;
        case 3: e = en_hinge(gi, a.nh, a.hinges, a.adj, a.x, a.rest, a.Q, a.kb_dt2); break;
        case 4: e = en_soft(gi, a.ns, a.soft_idx, a.x, a.target, a.ksoft); break;
        case 5: e = en_barrier(gi, a.npair, a.nv, a.pairs, a.x, a.rest, a.dhat, a.kappa); break;
        case 6: e = en_ground(gi, a.nground, a.nv, a.gp, a.x, a.offset, a.dhat, a.kappa); break;
        case 7: e = en_friction(gi, a.nfric, a.nv, a.fpairs, a.x, a.x0, a.flam, a.coord, a.basis, a.mu, a.eps2); break;
        default: e = en_fric_ground(gi, a.nfg, a.nv, a.fgp, a.x, a.x0, a.fglam, a.mu_gd, a.eps2); break;
    }
    cta_energy(e, part);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the terms' partials side by side: warp w adds terms w and w + 8 (lane l takes partials
    // l, l + 32, ... of a term, four loads in flight, then a fixed xor tree); thread 0 adds
    // the terms in order
    __shared__ double st[9];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = w; q < 9; q += (int)(blockDim.x >> 5)) {
        double sum = 0.0;
#pragma unroll 4
        for (int i = o.off[q] + lane; i < o.off[q + 1]; i += 32) sum += __ldcg(part + i);
#pragma unroll
        for (int k = 16; k > 0; k >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, k);
        if (lane == 0) st[q] = sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double total = 0.0;
        for (int q = 0; q < 9; q++) {
            terms[q] = st[q];
            total += st[q];
        }
        terms[9] = total;
        *ticket = 0u;
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
static SgipcStatus energy_launch(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k, const SgipcParams* p,
                                 cudaStream_t s, double* bytes);
static SgipcStatus check_inputs(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k, const SgipcParams* p) {
    if (!c || !f || !p) return SGIPC_BAD_INPUT;
    if (!f->vertexes || !f->xTilta || !f->masses || !f->BoundaryType) return SGIPC_BAD_INPUT;
    if (c->nt && (!f->DmInverses || !f->volum || !f->lengthRate || !f->volumeRate)) return SGIPC_BAD_INPUT;
    if (c->nf && (!f->triDmInverses || !f->area)) return SGIPC_BAD_INPUT;
    if (c->nh && (!f->quad_bending_Q || !f->rest_vertexes)) return SGIPC_BAD_INPUT;
    if (c->nsoft && !f->targetVert) return SGIPC_BAD_INPUT;
    if (!(p->dt > 0.0) || !(p->dHat > 0.0) || !(p->kappa >= 0.0)) return SGIPC_BAD_INPUT;
    if (k) {
        if (k->pair_num < 0 || k->ground_num < 0 || k->fric_num < 0 || k->fric_gd_num < 0) return SGIPC_BAD_INPUT;
        if (k->pair_num > c->max_pairs || k->ground_num > c->max_ground || k->fric_num > c->max_fric ||
            k->fric_gd_num > c->max_fric_gd) {
            snprintf(c->err, sizeof(c->err), "contact counts exceed the context capacity");
            return SGIPC_CAPACITY;
        }
        if ((k->pair_num && (!k->pairs || !f->rest_vertexes)) || (k->ground_num && !k->ground_pairs) ||
            (k->fric_num && (!k->fric_pairs || !k->fric_lambda || !k->fric_coord || !k->fric_basis || !f->o_vertexes)) ||
            (k->fric_gd_num && (!k->fric_gd_pairs || !k->fric_gd_lambda || !f->o_vertexes)))
            return SGIPC_BAD_INPUT;
    }
    return SGIPC_OK;
}

static BlockSink sink(SgipcCtx* c, const SgipcFemData* f) {
    BlockSink bs;
    bs.key = c->ckey;
    bs.idx = c->cidx;
    bs.val = c->cval;
    bs.btype = f->BoundaryType;
    bs.bits = c->key_bits;
    bs.nv = c->nv;
    bs.flag = c->dflag;
    return bs;
}

// contact block slots launch_contacts will use (soft constraints follow them)
static int contact_slots(const SgipcContacts* k, const SgipcParams* p) {
    if (!k) return 0;
    int m = 0;
    if (k->pair_num > 0) m += 10 * k->pair_num;
    if (k->fric_num > 0 && p->frictionRate > 0.0) m += 10 * k->fric_num;
    if (k->ground_num > 0) m += k->ground_num;
    if (k->fric_gd_num > 0 && p->gd_frictionRate > 0.0) m += k->fric_gd_num;
    return m;
}

// launch the contact kernels; returns the number of contact block slots used
static int launch_contacts(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k, const SgipcParams* p,
                           double* grad, cudaStream_t s, bool keep_dirichlet = false) {
    BlockSink bs = sink(c, f);
    if (keep_dirichlet) bs.btype = nullptr;
    if (!k) return 0;
    ContactLaunch L{};
    L.np = k->pair_num > 0 ? k->pair_num : 0;
    L.nf = k->fric_num > 0 && p->frictionRate > 0.0 ? k->fric_num : 0;
    L.ng = k->ground_num > 0 ? k->ground_num : 0;
    L.ngf = k->fric_gd_num > 0 && p->gd_frictionRate > 0.0 ? k->fric_gd_num : 0;
    L.cb = nblk(L.np, 128);
    L.cf = L.cb + nblk(L.nf, 128);
    L.cg = L.cf + nblk(L.ng, 128);
    const int grid = L.cg + nblk(L.ngf, 128);
    L.pairs = (const int4*)k->pairs;
    L.fpairs = (const int4*)k->fric_pairs;
    L.gpairs = k->ground_pairs;
    L.gfpairs = k->fric_gd_pairs;
    L.x = f->vertexes;
    L.x0 = f->o_vertexes;
    L.rest = f->rest_vertexes;
    L.flam = k->fric_lambda;
    L.fcoord = k->fric_coord;
    L.fbasis = k->fric_basis;
    L.gflam = k->fric_gd_lambda;
    L.dhat = p->dHat;
    L.kappa = p->kappa;
    L.mu = p->frictionRate;
    L.gmu = p->gd_frictionRate;
    L.eps2 = p->fDhat * p->dt * p->dt;
    L.offset = p->ground_offset;
    L.base_b = 0;
    L.base_f = 10 * L.np;
    L.base_g = L.base_f + 10 * L.nf;
    L.base_gf = L.base_g + L.ng;
    if (grid > 0) {
        SG_COUNT(c, 1);
        k_contacts<<<grid, 128, 0, s>>>(L, grad, bs);
    }
    return L.base_gf + L.ngf;
}

static SgipcStatus merge_contacts(SgipcCtx* c, int m, cudaStream_t s) {
    if (m == 0) {
        SG_CHECK(c, cudaMemsetAsync(c->nuc, 0, sizeof(int), s));
        SG_CHECK(c, cudaMemsetAsync(c->cu_ptr, 0, sizeof(int) * (c->n + 1), s));
        SG_CHECK(c, cudaMemsetAsync(c->cl_ptr, 0, sizeof(int) * (c->n + 1), s));
        return SGIPC_OK;
    }
    const int endbit = 2 * c->key_bits, n = c->n;
    SG_COUNT(c, 5);
    // keys sorted with their slot ids; runs of equal keys numbered by a scan of run heads;
    // each unique block summed by 9 threads (one per entry) over its run in sorted order
    // (deterministic), with every load of a run independent of the previous one.  The
    // transposed lists need no second sort: the run heads count the blocks of each column,
    // a scan of the counts gives the row pointers, and each block's rank by row within its
    // column gives its slot.
    SG_CHECK(c, cudaMemsetAsync(c->lcount, 0, sizeof(int) * (2 * (size_t)n + 1), s));
    size_t tb = c->cub_tmp_bytes;
    SG_CHECK(c, cub::DeviceRadixSort::SortPairs(c->cub_tmp, tb, c->ckey, c->ckey_s, c->cidx, c->cidx_s, m, 0, endbit, s));
    k_run_heads<<<nblk(m + 1), SGIPC_BLOCK, 0, s>>>(m, c->ckey_s, c->cflag);
    tb = c->cub_tmp_bytes;
    SG_CHECK(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp, tb, c->cflag, c->cflag, m + 1, s));
    k_run_starts<<<nblk(m + 1), SGIPC_BLOCK, 0, s>>>(m, c->ckey_s, c->cflag, c->key_bits, c->run_start, c->uc_row,
                                                     c->uc_col, c->nuc, c->lcount);
    tb = c->cub_tmp_bytes;
    SG_CHECK(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp, tb, c->lcount, c->cl_ptr, n + 1, s));
    k_lower_place<<<nblk(std::max(m, n + 1)), SGIPC_BLOCK, 0, s>>>(m, n, c->nuc, c->uc_row, c->uc_col, c->cl_ptr,
                                                                   c->lcount + n + 1, c->cu_ptr, c->cl_idx);
    k_lower_rank<<<nblk(m), SGIPC_BLOCK, 0, s>>>(c->nuc, c->uc_row, c->uc_col, c->cl_ptr, c->cl_idx, c->lpos,
                                                 c->cl_col);
    k_run_sums<<<std::min(nblk(32LL * m), 8 * 148), SGIPC_BLOCK, 0, s>>>(c->nuc, c->run_start, c->cidx_s, c->cval,
                                                                         c->lpos, c->uc64, c->uc32, c->cl64, c->cl32);
    SG_LAUNCH_CHECK(c, "contact merge");
    return SGIPC_OK;
}

static SgipcStatus launch_fem(SgipcCtx* c, const SgipcFemData* f, const SgipcParams* p, cudaStream_t s) {
    const double dt2 = p->dt * p->dt;
    if (c->nt > 0) {
        SG_COUNT(c, 1);
        k_snk<<<nblk(c->nt, 128), 128, 0, s>>>(c->nt, c->tets, f->vertexes, f->DmInverses, f->volum, f->lengthRate,
                                               f->volumeRate, dt2, c->eblk, c->egrad);
    }
    // element block / gradient row offsets: tets (10 / 4 each), triangles (6 / 3), hinges (10 / 4)
    if (c->nf > 0) {
        SG_COUNT(c, 1);
        k_tri_bw<<<nblk(c->nf, 128), 128, 0, s>>>(c->nf, c->tris, f->vertexes, f->triDmInverses, f->area,
                                                  p->stretchStiff, p->shearStiff, p->strainRate, dt2, 10 * c->nt,
                                                  4 * c->nt, c->eblk, c->egrad);
    }
    if (c->nh > 0) {
        SG_COUNT(c, 1);
        k_hinge_quad<<<nblk(c->nh), SGIPC_BLOCK, 0, s>>>(c->nh, c->hinges, c->hinge_adj, f->vertexes, f->rest_vertexes,
                                                         f->quad_bending_Q, p->bendStiff * dt2,
                                                         10 * c->nt + 6 * c->nf, 4 * c->nt + 3 * c->nf, c->eblk,
                                                         c->egrad);
    }
    SG_LAUNCH_CHECK(c, "fem element kernels");
    return SGIPC_OK;
}

static SgipcStatus gather_static(SgipcCtx* c, const SgipcFemData* f, cudaStream_t s) {
    c->mas.pre_scattered = 0;  // a scatter of the previous static matrix is stale
    SG_COUNT(c, 1 + (c->n_egrad > 0));
    k_gather_blocks<<<nblk(9LL * c->nnz), SGIPC_BLOCK, 0, s>>>(c->nnz, c->contrib_ptr, c->contrib, c->eblk, c->slot_row,
                                                                c->col, f->BoundaryType, f->masses, static_out(c));
    if (c->n_egrad > 0)
        k_gather_grad<<<nblk(3LL * c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, c->vinc_ptr, c->vinc, c->egrad, c->shape_grads);
    SG_LAUNCH_CHECK(c, "static gather");
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_assemble(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k,
                                      const SgipcParams* p, void* stream) {
    SgipcStatus st = check_inputs(c, f, k, p);
    if (st != SGIPC_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    SG_DEVICE(c);
    // the MAS hierarchy of these contacts on its own stream, first (it needs the contact
    // graph only; started before the assembly kernels, it runs beside them and
    // sgipc_mas_build reuses it)
    if ((st = mas_mark_start(c, s)) != SGIPC_OK) return st;
    if ((st = mas_prebuild(c, k, s)) != SGIPC_OK) return st;
    c->btype = f->BoundaryType;
    c->last_fem = *f;
    c->last_prm = *p;
    c->last_has_con = k != nullptr;
    if (k) c->last_con = *k;
    SG_COUNT(c, 2 + (c->nsoft > 0));
    k_kinetic<<<nblk(3LL * c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, f->vertexes, f->xTilta, f->masses, c->shape_grads, c->fb);
    // contacts (fb, contact block slots) on asm_stream, elements (element blocks, static
    // matrix, shape_grads) on s; the merge needs the soft-constraint slots from s, the
    // right-hand side both
    // (the soft constraints go first on s: the merge needs their block slots, and they add
    // to shape_grads before the element gradients do)
    cudaStream_t sc = c->asm_stream;
    const int m_con = contact_slots(k, p);
    if (c->nsoft > 0) {
        BlockSink bs = sink(c, f);
        k_soft<<<nblk(c->nsoft), SGIPC_BLOCK, 0, s>>>(c->nsoft, c->soft_idx, f->vertexes, f->targetVert,
                                                      p->motionRate * p->softRate * p->softRate, c->shape_grads, bs,
                                                      m_con);
    }
    SG_CHECK(c, cudaEventRecord(c->ev_asm[0], s));
    SG_CHECK(c, cudaStreamWaitEvent(sc, c->ev_asm[0], 0));
    int m = launch_contacts(c, f, k, p, c->fb, sc);
    SG_LAUNCH_CHECK(c, "contact kernels");
    m += c->nsoft;
    if ((st = merge_contacts(c, m, sc)) != SGIPC_OK) return st;
    if ((st = launch_fem(c, f, p, s)) != SGIPC_OK) return st;
    if ((st = gather_static(c, f, s)) != SGIPC_OK) return st;
    // the static blocks into the prebuilt hierarchy's domains, on the MAS stream beside the merge
    if ((st = mas_prescatter(c, s)) != SGIPC_OK) return st;
    SG_CHECK(c, cudaEventRecord(c->ev_asm[2], sc));
    SG_CHECK(c, cudaStreamWaitEvent(s, c->ev_asm[2], 0));
    k_rhs<<<nblk(3LL * c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, c->fb, c->shape_grads, f->BoundaryType, c->b);
    SG_LAUNCH_CHECK(c, "rhs");
    c->assembled = 1;
    c->mas.built = 0;
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_barrier_grad_hess(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k,
                                               const SgipcParams* p, double* grad, void* stream) {
    SgipcStatus st = check_inputs(c, f, k, p);
    if (st != SGIPC_OK) return st;
    if (!grad || !k) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    SgipcContacts only = *k;
    only.fric_num = 0;
    only.ground_num = 0;
    only.fric_gd_num = 0;
    int m = launch_contacts(c, f, &only, p, grad, s);
    SG_LAUNCH_CHECK(c, "barrier");
    return merge_contacts(c, m, s);
}

extern "C" SgipcStatus sgipc_friction_grad_hess(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k,
                                                const SgipcParams* p, double* grad, void* stream) {
    SgipcStatus st = check_inputs(c, f, k, p);
    if (st != SGIPC_OK) return st;
    if (!grad || !k) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    SgipcContacts only = *k;
    only.pair_num = 0;
    only.ground_num = 0;
    int m = launch_contacts(c, f, &only, p, grad, s);
    SG_LAUNCH_CHECK(c, "friction");
    return merge_contacts(c, m, s);
}

extern "C" SgipcStatus sgipc_fem_grad_hess(SgipcCtx* c, const SgipcFemData* f, const SgipcParams* p, double* grad,
                                           void* stream) {
    SgipcStatus st = check_inputs(c, f, nullptr, p);
    if (st != SGIPC_OK) return st;
    if (!grad) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    if ((st = launch_fem(c, f, p, s)) != SGIPC_OK) return st;
    if ((st = gather_static(c, f, s)) != SGIPC_OK) return st;
    // gather_static added the element gradient into shape_grads; hand it to the caller
    if (c->n_egrad > 0)
        k_gather_grad<<<nblk(3LL * c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, c->vinc_ptr, c->vinc, c->egrad, grad);
    SG_LAUNCH_CHECK(c, "fem gradient");
    return SGIPC_OK;
}

// ------------------------------------------------------------------------------------------
// timing hook
// ------------------------------------------------------------------------------------------
namespace sgipc {
// ---- class partition of the contact terms (affine-body points) ------------------------------
// slot s of the contact blocks: fa[s] = 1 for an ABD-ABD block, ff[s] = 1 for an ABD-FEM block
// (upper keys: r <= c, so an ABD-FEM block has r < af <= c)
__global__ void k_part_flags(int m, const unsigned long long* __restrict__ key, int bits, int af, int* __restrict__ fa,
                             int* __restrict__ ff) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > m) return;
    int a = 0, f = 0;
    if (s < m) {
        const unsigned long long k = key[s];
        if (k != kBadKey) {
            const int r = (int)(k >> bits), c = (int)(k & ((1ull << bits) - 1));
            a = r >= af;
            f = r < af && c >= af;
        }
    }
    fa[s] = a;
    ff[s] = f;
}

// emit the flagged blocks at their scanned positions (slot order): ABD-ABD as (point, point)
// with point ids counted from af, ABD-FEM as (point, FEM vertex) with the block transposed to
// that orientation
__global__ void k_part_emit(int m, const unsigned long long* __restrict__ key, const double* __restrict__ val, int bits,
                            int af, const int* __restrict__ oa, const int* __restrict__ of, int cap,
                            int32_t* __restrict__ arow, int32_t* __restrict__ acol, double* __restrict__ aval,
                            int32_t* __restrict__ frow, int32_t* __restrict__ fcol, double* __restrict__ fval) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= m) return;
    const unsigned long long k = key[s];
    if (k == kBadKey) return;
    const int r = (int)(k >> bits), c = (int)(k & ((1ull << bits) - 1));
    const double* v = val + 9 * (size_t)s;
    if (r >= af) {
        const int i = oa[s];
        if (i >= cap) return;
        arow[i] = r - af;
        acol[i] = c - af;
        for (int q = 0; q < 9; q++) aval[9 * (size_t)i + q] = v[q];
    } else if (c >= af) {
        const int i = of[s];
        if (i >= cap) return;
        frow[i] = c - af;
        fcol[i] = r;
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++) fval[9 * (size_t)i + 3 * p + q] = v[3 * q + p];
    }
}

__global__ void k_part_grad(int npt, int af, const double* __restrict__ g, double* __restrict__ pg) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 3 * npt) pg[k] = g[3 * (size_t)af + k];
}

extern "C" SgipcStatus sgipc_contact_partition(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k,
                                               const SgipcParams* p, int32_t abd_first, int32_t cap,
                                               int32_t* abd_rows, int32_t* abd_cols, double* abd_vals,
                                               int32_t* abd_count, int32_t* fem_rows, int32_t* fem_cols,
                                               double* fem_vals, int32_t* fem_count, double* point_grad,
                                               void* stream) {
    SgipcStatus st = check_inputs(c, f, k, p);
    if (st != SGIPC_OK) return st;
    if (abd_first < 0 || abd_first > c->nv || cap < 0 || !abd_count || !fem_count) {
        snprintf(c->err, sizeof(c->err), "contact_partition: abd_first %d outside [0, %d] or a missing count",
                 abd_first, c->nv);
        return SGIPC_BAD_INPUT;
    }
    if (cap > 0 && (!abd_rows || !abd_cols || !abd_vals || !fem_rows || !fem_cols || !fem_vals)) return SGIPC_BAD_INPUT;
    cudaStream_t s = (cudaStream_t)stream;
    SG_DEVICE(c);
    const int npt = c->nv - abd_first;
    SG_CHECK(c, cudaMemsetAsync(c->tmp64, 0, sizeof(double) * 3 * (size_t)c->nv, s));
    const int m = launch_contacts(c, f, k, p, c->tmp64, s, true);
    SG_LAUNCH_CHECK(c, "contact kernels (partition)");
    int* fa = c->cflag;
    int* ff = c->run_start;
    SG_COUNT(c, 2 + (npt > 0 && point_grad ? 1 : 0));
    k_part_flags<<<nblk(m + 1), SGIPC_BLOCK, 0, s>>>(m, c->ckey, c->key_bits, abd_first, fa, ff);
    size_t tb = c->cub_tmp_bytes;
    SG_CHECK(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp, tb, fa, fa, m + 1, s));
    tb = c->cub_tmp_bytes;
    SG_CHECK(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp, tb, ff, ff, m + 1, s));
    if (m > 0)
        k_part_emit<<<nblk(m), SGIPC_BLOCK, 0, s>>>(m, c->ckey, c->cval, c->key_bits, abd_first, fa, ff, cap, abd_rows,
                                                    abd_cols, abd_vals, fem_rows, fem_cols, fem_vals);
    if (npt > 0 && point_grad) k_part_grad<<<nblk(3LL * npt), SGIPC_BLOCK, 0, s>>>(npt, abd_first, c->tmp64, point_grad);
    SG_LAUNCH_CHECK(c, "contact partition");
    int cnt[2];
    SG_CHECK(c, cudaMemcpyAsync(&cnt[0], fa + m, sizeof(int), cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaMemcpyAsync(&cnt[1], ff + m, sizeof(int), cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    *abd_count = cnt[0];
    *fem_count = cnt[1];
    if (cnt[0] > cap || cnt[1] > cap) {
        snprintf(c->err, sizeof(c->err), "contact_partition: %d ABD-ABD and %d ABD-FEM blocks beyond the capacity %d",
                 cnt[0], cnt[1], cap);
        return SGIPC_CAPACITY;
    }
    return SGIPC_OK;
}

// ---- barrier stiffness adaptation (GIPC::initKappa / suggestKappa / upperBoundKappa,
// GIPC.cu:9850-9929; the close-constraint checks of GIPC::postLineSearch, GIPC.cu:10777-10806)
// shape_grads += the tet rows (the first 4 * nt element gradient rows) of each vertex
__global__ void k_gather_grad_tets(int nv, int limit, const int* __restrict__ vptr, const int* __restrict__ vinc,
                                   const double* __restrict__ egrad, double* __restrict__ out) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 3 * nv) return;
    const int v = tid / 3, q = tid % 3;
    double acc = 0.0;
    for (int k = vptr[v]; k < vptr[v + 1]; k++) {
        const int e = vinc[k];
        if (e < limit) acc += egrad[3 * (size_t)e + q];
    }
    out[tid] += acc;
}

// compute_H_b (GIPC.cu, used by suggestKappa / upperBoundKappa): the barrier's second
// derivative scale at d = 1e-16 bbox^2
static double kappa_hb(double bbox_diag2, double dhat) {
    const double d = 1.0e-16 * bbox_diag2, t = d - dhat;
    return (std::log(d / dhat) * -2.0 - t * 4.0 / d) + 1.0 / (d * d) * (t * t);
}

extern "C" SgipcStatus sgipc_init_kappa(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k,
                                        const SgipcParams* p, double mean_mass, double bbox_diag2,
                                        double min_kappa_coef, double* kappa, void* stream) {
    SgipcStatus st = check_inputs(c, f, k, p);
    if (st != SGIPC_OK) return st;
    if (!kappa || !(bbox_diag2 > 0.0)) return SGIPC_BAD_INPUT;
    if (!k || k->pair_num <= 0) return SGIPC_OK;  // the reference adapts only with contact pairs
    cudaStream_t s = (cudaStream_t)stream;
    SG_DEVICE(c);
    const int nv = c->nv;
    double* GE = c->tmp64;   // kinetic + tet elastic + soft-constraint gradient
    double* gc = c->tmp64b;  // barrier + ground gradient at kappa = 1
    SG_COUNT(c, 2 + (c->nsoft > 0));
    k_kinetic<<<nblk(3LL * nv), SGIPC_BLOCK, 0, s>>>(nv, f->vertexes, f->xTilta, f->masses, GE, gc);
    if ((st = launch_fem(c, f, p, s)) != SGIPC_OK) return st;
    k_gather_grad_tets<<<nblk(3LL * nv), SGIPC_BLOCK, 0, s>>>(nv, 4 * c->nt, c->vinc_ptr, c->vinc, c->egrad, GE);
    if (c->nsoft > 0) {
        BlockSink bs = sink(c, f);
        k_soft<<<nblk(c->nsoft), SGIPC_BLOCK, 0, s>>>(c->nsoft, c->soft_idx, f->vertexes, f->targetVert,
                                                      p->motionRate * p->softRate * p->softRate, GE, bs, 0);
    }
    SgipcContacts only = *k;
    only.fric_num = 0;
    only.fric_gd_num = 0;
    SgipcParams p1 = *p;
    p1.kappa = 1.0;
    p1.frictionRate = 0.0;
    p1.gd_frictionRate = 0.0;
    launch_contacts(c, f, &only, &p1, gc, s);
    SG_LAUNCH_CHECK(c, "init kappa gradients");
    if ((st = dot64(c, gc, GE, 3 * nv, c->dot_out, s)) != SGIPC_OK) return st;
    if ((st = dot64(c, gc, gc, 3 * nv, c->dot_out + 1, s)) != SGIPC_OK) return st;
    double h[2];
    SG_CHECK(c, cudaMemcpyAsync(h, c->dot_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    double K = *kappa;
    double minK = -h[0] / h[1];
    if (minK > 0.0) K = minK;
    const double hb = kappa_hb(bbox_diag2, p->dHat);
    // suggestKappa overwrites minKappa with its suggestion, which then bounds Kappa below
    minK = mean_mass == 0.0 ? min_kappa_coef / (4.0e-16 * bbox_diag2 * hb)
                            : min_kappa_coef * mean_mass / (4.0e-16 * bbox_diag2 * hb);
    if (K < minK) K = minK;
    double kmax = 100 * min_kappa_coef * mean_mass / (4.0e-16 * bbox_diag2 * hb);
    if (mean_mass == 0.0) kmax = 100 * min_kappa_coef / (4.0e-16 * bbox_diag2 * hb);
    if (K > kmax) K = kmax;
    *kappa = K;
    return SGIPC_OK;
}

// close constraints: ground vertices and pairs closer than dTol (squared), with their value
__global__ void k_close_ground_record(int ng, const uint32_t* __restrict__ gp, const double* __restrict__ x,
                                      double offset, double dtol, uint32_t* __restrict__ id,
                                      double* __restrict__ val, unsigned int* __restrict__ cnt) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ng) return;
    const uint32_t v = gp[p];
    const double d = x[3 * (size_t)v + 1] - offset, d2 = d * d;
    if (d2 < dtol) {
        const unsigned int i = atomicAdd(cnt, 1u);
        id[i] = v;
        val[i] = d2;
    }
}

__global__ void k_close_pair_record(int np, const int4* __restrict__ pairs, const double* __restrict__ x,
                                    double dtol, int4* __restrict__ id, double* __restrict__ val,
                                    unsigned int* __restrict__ cnt) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    int v[4], nvp;
    const int kind = decode_pair(pairs[p], v, nvp);
    d3 X[4], g[4];
#pragma unroll
    for (int a = 0; a < 4; a++) X[a] = a < nvp ? ld3(x, v[a]) : mk(0, 0, 0);
    const double d2 = dist2_grad(kind, X, g);
    if (d2 < dtol) {
        const unsigned int i = atomicAdd(cnt + 1, 1u);
        id[i] = pairs[p];
        val[i] = d2;
    }
}

// flag[0] = 1 when a recorded ground vertex or pair is closer now than when recorded
__global__ void k_close_check(int ng, int np, const uint32_t* __restrict__ gid, const double* __restrict__ gval,
                              const int4* __restrict__ pid, const double* __restrict__ pval,
                              const double* __restrict__ x, double offset, int* __restrict__ flag) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ng) {
        const double d = x[3 * (size_t)gid[t] + 1] - offset;
        if (d * d < gval[t]) *flag = 1;
    } else if (t < ng + np) {
        int v[4], nvp;
        const int kind = decode_pair(pid[t - ng], v, nvp);
        d3 X[4], g[4];
#pragma unroll
        for (int a = 0; a < 4; a++) X[a] = a < nvp ? ld3(x, v[a]) : mk(0, 0, 0);
        if (dist2_grad(kind, X, g) < pval[t - ng]) *flag = 1;
    }
}

extern "C" SgipcStatus sgipc_close_record(SgipcCtx* c, const double* x, const SgipcContacts* k, double dtol,
                                          double ground_offset, int32_t* counts, void* stream) {
    if (!c || !x || !k || (k->pair_num > 0 && !k->pairs) || (k->ground_num > 0 && !k->ground_pairs))
        return SGIPC_BAD_INPUT;
    if (k->pair_num > c->max_pairs || k->ground_num > c->max_ground) return SGIPC_CAPACITY;
    cudaStream_t s = (cudaStream_t)stream;
    SG_DEVICE(c);
    if (!c->close_cnt) {
        SG_CHECK(c, cudaMalloc((void**)&c->close_gid, sizeof(uint32_t) * (size_t)std::max(c->max_ground, 1)));
        SG_CHECK(c, cudaMalloc((void**)&c->close_gval, sizeof(double) * (size_t)std::max(c->max_ground, 1)));
        SG_CHECK(c, cudaMalloc((void**)&c->close_pid, sizeof(int4) * (size_t)std::max(c->max_pairs, 1)));
        SG_CHECK(c, cudaMalloc((void**)&c->close_pval, sizeof(double) * (size_t)std::max(c->max_pairs, 1)));
        SG_CHECK(c, cudaMalloc((void**)&c->close_cnt, sizeof(unsigned int) * 4));
    }
    SG_CHECK(c, cudaMemsetAsync(c->close_cnt, 0, sizeof(unsigned int) * 4, s));
    SG_COUNT(c, (k->ground_num > 0) + (k->pair_num > 0));
    if (k->ground_num > 0)
        k_close_ground_record<<<nblk(k->ground_num), SGIPC_BLOCK, 0, s>>>(
            k->ground_num, k->ground_pairs, x, ground_offset, dtol, c->close_gid, c->close_gval, c->close_cnt);
    if (k->pair_num > 0)
        k_close_pair_record<<<nblk(k->pair_num), SGIPC_BLOCK, 0, s>>>(
            k->pair_num, (const int4*)k->pairs, x, dtol, (int4*)c->close_pid, c->close_pval, c->close_cnt);
    SG_LAUNCH_CHECK(c, "close constraints");
    unsigned int h[2];
    SG_CHECK(c, cudaMemcpyAsync(h, c->close_cnt, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    c->close_num[0] = (int)h[0];
    c->close_num[1] = (int)h[1];
    if (counts) {
        counts[0] = (int32_t)h[0];
        counts[1] = (int32_t)h[1];
    }
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_close_check(SgipcCtx* c, const double* x, double ground_offset, int32_t* changed,
                                         void* stream) {
    if (!c || !x || !changed) return SGIPC_BAD_INPUT;
    *changed = 0;
    const int ng = c->close_cnt ? c->close_num[0] : 0, np = c->close_cnt ? c->close_num[1] : 0;
    if (ng + np == 0) return SGIPC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    SG_DEVICE(c);
    SG_CHECK(c, cudaMemsetAsync(c->close_cnt + 2, 0, sizeof(unsigned int), s));
    SG_COUNT(c, 1);
    k_close_check<<<nblk(ng + np), SGIPC_BLOCK, 0, s>>>(ng, np, c->close_gid, c->close_gval, (const int4*)c->close_pid,
                                                        c->close_pval, x, ground_offset,
                                                        reinterpret_cast<int*>(c->close_cnt + 2));
    SG_LAUNCH_CHECK(c, "close check");
    unsigned int h = 0;
    SG_CHECK(c, cudaMemcpyAsync(&h, c->close_cnt + 2, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    *changed = h != 0;
    return SGIPC_OK;
}

SgipcStatus assemble_time_hook(SgipcCtx* c, const char* name, cudaStream_t s, double* bytes) {
    const SgipcFemData* f = &c->last_fem;
    const SgipcParams* p = &c->last_prm;
    const SgipcContacts* k = c->last_has_con ? &c->last_con : nullptr;
    double* scratch = c->tmp64b;  // gradient sink that keeps fb untouched
    if (!strcmp(name, "energy")) return energy_launch(c, f, k, p, s, bytes);
    if (!strcmp(name, "snk")) {
        if (c->nt <= 0) return SGIPC_BAD_INPUT;
        SG_COUNT(c, 1);
        k_snk<<<nblk(c->nt, 128), 128, 0, s>>>(c->nt, c->tets, f->vertexes, f->DmInverses, f->volum, f->lengthRate,
                                               f->volumeRate, p->dt * p->dt, c->eblk, c->egrad);
        // positions, DmInv, volume, (mu, lambda), indices in; 10 FP64 blocks and 4 gradient rows out
        *bytes = (double)c->nt * (4 * 24 + 72 + 8 + 16 + 16 + 10 * 72 + 12 * 8);
    } else if (!strcmp(name, "gather_blocks")) {
        SG_COUNT(c, 1);
        k_gather_blocks<<<nblk(9LL * c->nnz), SGIPC_BLOCK, 0, s>>>(c->nnz, c->contrib_ptr, c->contrib, c->eblk,
                                                                    c->slot_row, c->col, f->BoundaryType, f->masses,
                                                                    static_out(c));
        // element blocks and their indices in; per upper slot its indices, flags and the FP64
        // upper value out, the full-pattern FP64 + FP32 copy, and the transposed copy off the
        // diagonal
        *bytes = (double)c->n_eblk * (72 + 4) + (double)c->nnz * (28 + 72 + 108) + (double)(c->nnz - c->n) * 108;
    } else if (!strcmp(name, "barrier")) {
        if (!k || k->pair_num <= 0) return SGIPC_BAD_INPUT;
        SG_COUNT(c, 1);
        BlockSink bs = sink(c, f);
        k_barrier<<<nblk(k->pair_num, 128), 128, 0, s>>>(k->pair_num, (const int4*)k->pairs, f->vertexes,
                                                          f->rest_vertexes, p->dHat, p->kappa, scratch, bs, 0);
        // pair + 4 positions (+ 4 rest positions) in; 10 keyed FP64 blocks and 12 gradient entries out
        *bytes = (double)k->pair_num * (16 + 4 * 24 + 4 * 24 + 10 * (72 + 8 + 4) + 12 * 8);
    } else if (!strcmp(name, "friction")) {
        if (!k || k->fric_num <= 0) return SGIPC_BAD_INPUT;
        SG_COUNT(c, 1);
        BlockSink bs = sink(c, f);
        k_friction<<<nblk(k->fric_num, 128), 128, 0, s>>>(k->fric_num, (const int4*)k->fric_pairs, f->vertexes,
                                                           f->o_vertexes, k->fric_lambda, k->fric_coord, k->fric_basis,
                                                           p->frictionRate, p->fDhat * p->dt * p->dt, scratch, bs,
                                                           10 * (k->pair_num > 0 ? k->pair_num : 0));
        *bytes = (double)k->fric_num * (16 + 8 + 16 + 48 + 8 * 24 + 10 * (72 + 8 + 4) + 12 * 8);
    } else {
        return SGIPC_NOT_READY;
    }
    SG_LAUNCH_CHECK(c, name);
    return SGIPC_OK;
}
}  // namespace sgipc

// ------------------------------------------------------------------------------------------
// line-search energy: host side
// ------------------------------------------------------------------------------------------
// Launch the energy kernels and the final sum into c->en_terms on s (no synchronisation).
// Terms: 0 kinetic, 1 tets, 2 triangles, 3 hinges, 4 soft, 5 barrier, 6 ground, 7 friction,
// 8 ground friction; 9 the total.  *bytes: algorithmic bytes of the launch sequence.
static SgipcStatus energy_launch(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k, const SgipcParams* p,
                                 cudaStream_t s, double* bytes) {
    const double dt2 = p->dt * p->dt, eps2 = p->fDhat * dt2;
    const int npair = k ? k->pair_num : 0, nground = k ? k->ground_num : 0;
    const int nfric = k && p->frictionRate > 0.0 ? k->fric_num : 0;
    const int nfg = k && p->gd_frictionRate > 0.0 ? k->fric_gd_num : 0;
    const int cnt[9] = {c->nv, c->nt, c->nf, c->nh, c->nsoft, npair, nground, nfric, nfg};
    EnergyOffsets o;
    o.off[0] = 0;
    for (int t = 0; t < 9; t++) o.off[t + 1] = o.off[t] + nblk(cnt[t]);
    if (o.off[9] > c->en_cap) {
        snprintf(c->err, sizeof(c->err), "energy: %d partial sums exceed the context's %d", o.off[9], c->en_cap);
        return SGIPC_CAPACITY;
    }
    EnergyArgs a;
    a.nv = c->nv; a.nt = c->nt; a.nf = c->nf; a.nh = c->nh; a.ns = c->nsoft;
    a.npair = npair; a.nground = nground; a.nfric = nfric; a.nfg = nfg;
    a.x = f->vertexes; a.xt = f->xTilta; a.m = f->masses; a.x0 = f->o_vertexes; a.rest = f->rest_vertexes;
    a.tets = c->tets; a.tris = c->tris; a.hinges = c->hinges; a.soft_idx = c->soft_idx;
    a.gp = k ? k->ground_pairs : nullptr; a.fgp = k ? k->fric_gd_pairs : nullptr; a.adj = c->hinge_adj;
    a.pairs = k ? (const int4*)k->pairs : nullptr; a.fpairs = k ? (const int4*)k->fric_pairs : nullptr;
    a.dminv = f->DmInverses; a.vol = f->volum; a.lr = f->lengthRate; a.vr = f->volumeRate;
    a.tdminv = f->triDmInverses; a.area = f->area; a.Q = f->quad_bending_Q; a.target = f->targetVert;
    a.flam = k ? k->fric_lambda : nullptr; a.coord = k ? k->fric_coord : nullptr; a.basis = k ? k->fric_basis : nullptr;
    a.fglam = k ? k->fric_gd_lambda : nullptr;
    a.dt2 = dt2; a.kst = p->stretchStiff; a.ksh = p->shearStiff; a.srate = p->strainRate; a.kb_dt2 = p->bendStiff * dt2;
    a.ksoft = p->motionRate * p->softRate * p->softRate; a.dhat = p->dHat; a.kappa = p->kappa;
    a.offset = p->ground_offset; a.mu = p->frictionRate; a.mu_gd = p->gd_frictionRate; a.eps2 = eps2;
    k_energy<<<o.off[9], SGIPC_BLOCK, 0, s>>>(a, o, c->en_part, c->en_terms, c->en_ticket);
    SG_COUNT(c, 1);
    SG_LAUNCH_CHECK(c, "energy");
    if (bytes)  // positions (and the per-element inputs) in, one partial per CTA out and back
        *bytes = (double)c->nv * (24 + 24 + 8) + (double)c->nt * (16 + 4 * 24 + 72 + 8 + 16) +
                 (double)c->nf * (12 + 3 * 24 + 32 + 8) + (double)c->nh * (16 + 4 * 24 + 2 * 24 + 128) +
                 (double)c->nsoft * (4 + 24 + 24) + (double)npair * (16 + 4 * 24 + 4 * 24) + (double)nground * (4 + 8) +
                 (double)nfric * (16 + 8 + 16 + 48 + 8 * 24) + (double)nfg * (4 + 8 + 48) + 2.0 * 8 * o.off[9];
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_compute_energy(SgipcCtx* c, const SgipcFemData* f, const SgipcContacts* k,
                                            const SgipcParams* p, double* energy, double* terms, void* stream) {
    SgipcStatus st = check_inputs(c, f, k, p);
    if (st != SGIPC_OK) return st;
    if (!energy) return SGIPC_BAD_INPUT;
    cudaStream_t s = (cudaStream_t)stream;
    SG_DEVICE(c);
    if ((st = energy_launch(c, f, k, p, s, nullptr)) != SGIPC_OK) return st;
    SG_CHECK(c, cudaMemcpyAsync(c->h_en, c->en_terms, sizeof(double) * 10, cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    *energy = c->h_en[9];
    if (terms)
        for (int t = 0; t < 9; t++) terms[t] = c->h_en[t];
    return SGIPC_OK;
}
