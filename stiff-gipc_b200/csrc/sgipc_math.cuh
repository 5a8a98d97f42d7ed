// sgipc_math.cuh — fixed-size FP64 math used by the element kernels.
//
// Own small value types replace the reference's __GEIGEN__ structs and device-side
// Eigen (StiffGIPC/eigen_data.h, gpu_eigen_libs.cu).  The symmetric 3x3 eigen-solver is a
// cyclic Jacobi iteration (Golub & Van Loan, "Matrix Computations", sec. 8.5) and the SVD
// is formed from it (F^T F = V S^2 V^T, U = F V S^-1 with the rotation-variant sign
// convention), written from those published methods.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace sgipc {

struct d3 {
    double x, y, z;
};
__host__ __device__ __forceinline__ d3 mk(double a, double b, double c) { return {a, b, c}; }
__host__ __device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ d3 operator-(d3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ d3 operator*(double s, d3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ d3 cross(d3 a, d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ double sq(d3 a) { return dot(a, a); }
__device__ __forceinline__ d3 ld3(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__host__ __device__ __forceinline__ double comp(d3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// 3x3 row-major
struct m3 {
    double m[3][3];
};

// Cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix.  On return A's diagonal
// holds the eigenvalues and V's columns the eigenvectors (A_in = V diag V^T).
__host__ __device__ inline void sym_eig3(double A[3][3], double V[3][3]) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) V[i][j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 12; sweep++) {
        double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= 1e-34 * dia || off == 0.0) break;
#pragma unroll
        for (int pq = 0; pq < 3; pq++) {
            const int p = pq == 2 ? 1 : 0;
            const int q = pq == 0 ? 1 : 2;
            double apq = A[p][q];
            if (fabs(apq) < 1e-300) continue;
            double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
            double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - s * akq;
                A[k][q] = s * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - s * aqk;
                A[q][k] = s * apk + c * aqk;
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq;
                V[k][q] = s * vkp + c * vkq;
            }
        }
    }
}

// Rotation-variant SVD F = U diag(S) V^T: U, V proper rotations, S sorted by magnitude
// descending, the sign of det F carried by S[2].
__host__ __device__ inline void svd3_rv(const double F[3][3], double U[3][3], double S[3], double V[3][3]) {
    double C[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C[i][j] = F[0][i] * F[0][j] + F[1][i] * F[1][j] + F[2][i] * F[2][j];
    sym_eig3(C, V);
    double e[3] = {C[0][0], C[1][1], C[2][2]};
    // sort descending (swap columns of V)
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 2 - a; b++)
            if (e[b] < e[b + 1]) {
                double t = e[b]; e[b] = e[b + 1]; e[b + 1] = t;
                for (int k = 0; k < 3; k++) { double tv = V[k][b]; V[k][b] = V[k][b + 1]; V[k][b + 1] = tv; }
            }
    double detV = V[0][0] * (V[1][1] * V[2][2] - V[1][2] * V[2][1]) - V[0][1] * (V[1][0] * V[2][2] - V[1][2] * V[2][0]) +
                  V[0][2] * (V[1][0] * V[2][1] - V[1][1] * V[2][0]);
    if (detV < 0)
        for (int k = 0; k < 3; k++) V[k][2] = -V[k][2];
    d3 fv[3];
    for (int c = 0; c < 3; c++)
        fv[c] = mk(F[0][0] * V[0][c] + F[0][1] * V[1][c] + F[0][2] * V[2][c],
                   F[1][0] * V[0][c] + F[1][1] * V[1][c] + F[1][2] * V[2][c],
                   F[2][0] * V[0][c] + F[2][1] * V[1][c] + F[2][2] * V[2][c]);
    double n0 = sqrt(sq(fv[0]));
    d3 u0 = n0 > 0 ? (1.0 / n0) * fv[0] : mk(1, 0, 0);
    d3 t1 = fv[1] - dot(fv[1], u0) * u0;
    double n1 = sqrt(sq(t1));
    d3 u1;
    if (n1 > 1e-300 && n1 > 1e-14 * n0) {
        u1 = (1.0 / n1) * t1;
    } else {
        d3 a = fabs(u0.x) < 0.9 ? mk(1, 0, 0) : mk(0, 1, 0);
        d3 t = cross(u0, a);
        u1 = (1.0 / sqrt(sq(t))) * t;
    }
    d3 u2 = cross(u0, u1);
    S[0] = dot(u0, fv[0]);
    S[1] = dot(u1, fv[1]);
    S[2] = dot(u2, fv[2]);
    U[0][0] = u0.x; U[1][0] = u0.y; U[2][0] = u0.z;
    U[0][1] = u1.x; U[1][1] = u1.y; U[2][1] = u1.z;
    U[0][2] = u2.x; U[1][2] = u2.y; U[2][2] = u2.z;
}

// PSD projection of a symmetric 2x2 [a b; b c] (makePDGeneral<2>, GIPC.cu:31-57):
// left untouched when already PSD, negative eigenvalues clamped otherwise.
__host__ __device__ inline void make_pd2(double& a, double& b, double& c) {
    double tr = 0.5 * (a + c);
    double df = 0.5 * (a - c);
    double r = sqrt(df * df + b * b);
    double l0 = tr - r, l1 = tr + r;
    if (l0 >= 0.0) return;
    if (l1 <= 0.0) { a = b = c = 0.0; return; }
    // eigenvector of l1
    double vx, vy;
    if (fabs(b) > 0.0) {
        vx = b; vy = l1 - a;
        double nn = sqrt(vx * vx + vy * vy);
        vx /= nn; vy /= nn;
    } else if (a >= c) { vx = 1; vy = 0; } else { vx = 0; vy = 1; }
    a = l1 * vx * vx;
    b = l1 * vx * vy;
    c = l1 * vy * vy;
}

}  // namespace sgipc
