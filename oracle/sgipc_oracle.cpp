// sgipc_oracle.cpp — CPU FP64 restatement of StiffGIPC's per-Newton-iteration linear
// system.  TEST INFRASTRUCTURE ONLY: it is the checker for the CUDA library (tests,
// the smoke check and bench.py's CPU-baseline leg); nothing in the product links it.
//
// Parity status: the reference ships no tests, golden vectors or fixtures for this path
// and cannot be built here (Eigen 3.4, GLUT/GLEW/OpenGL and nlohmann_json are absent),
// so this restatement is pinned by closed-form and finite-difference identities of the
// reference formulas (see tests/) rather than by reference outputs: parity unpinned.
//
// It is written independently of the CUDA kernels:
//   * distance derivatives come from forward-mode dual numbers, not hand derivations;
//   * the stable Neo-Hookean Hessian is the exact 9x9 second derivative projected by a
//     numeric Jacobi eigen-decomposition (the CUDA kernel uses the analytic
//     twist/flip/scaling eigensystem the reference uses);
//   * assembly merges plain COO triplets by sorting, as Converter::convert does.
//
// Reference files followed (paths inside the StiffGIPC project):
//   femEnergy.cu:432-459 (SNK1 PK1), 1042-1050 (energy), 1593-1717 (projected Hessian),
//   1719-1857 (tet kernel); GIPC.cu:31-57 (makePDGeneral), 701-958 (barrier energy),
//   1252-1800 (friction energy/Hessian), 3106-4945 (barrier gradient+Hessian),
//   5047-5270 (friction gradient), 6339-6514 (kinetic, soft, ground), 10110-10344
//   (assembly order, Dirichlet zeroing, mass diagonal); FrictionUtils.cuh:52-499;
//   mlbvh.cu:229-268 (distances, mollifier eps); converter.cu, spmv.cu (BCOO merge,
//   symmetric SpMV); pcg_solver.cu:174-267 (PCG); MASPreconditioner.cu:29-2262 (MAS).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------------------
// forward-mode dual numbers with N directions
// ---------------------------------------------------------------------------------------
template <int N>
struct Dual {
    double v;
    double d[N];
    Dual() : v(0) { std::fill(d, d + N, 0.0); }
    Dual(double c) : v(c) { std::fill(d, d + N, 0.0); }
    static Dual var(double c, int i) { Dual r(c); r.d[i] = 1.0; return r; }
};
template <int N> Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v + b.v; for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i]; return r; }
template <int N> Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v - b.v; for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i]; return r; }
template <int N> Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v * b.v; for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <int N> Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) { Dual<N> r; r.v = a.v / b.v; for (int i = 0; i < N; i++) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v); return r; }
template <int N> Dual<N> operator*(double s, const Dual<N>& a) { Dual<N> r; r.v = s * a.v; for (int i = 0; i < N; i++) r.d[i] = s * a.d[i]; return r; }
template <int N> Dual<N> dsqrt(const Dual<N>& a) { Dual<N> r; r.v = std::sqrt(a.v); for (int i = 0; i < N; i++) r.d[i] = a.d[i] / (2.0 * r.v); return r; }

template <class T> struct P3 { T x, y, z; };
template <class T> P3<T> sub(const P3<T>& a, const P3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> T dot(const P3<T>& a, const P3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> P3<T> cross(const P3<T>& a, const P3<T>& b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// squared distances by feature type (mlbvh.cu:229-262)
template <class T> T dist2_pp(const P3<T>& a, const P3<T>& b) { P3<T> d = sub(a, b); return dot(d, d); }
template <class T> T dist2_pe(const P3<T>& p, const P3<T>& e0, const P3<T>& e1) {
    P3<T> c = cross(sub(e0, p), sub(e1, p)); P3<T> e = sub(e1, e0); return dot(c, c) / dot(e, e); }
template <class T> T dist2_pt(const P3<T>& p, const P3<T>& t0, const P3<T>& t1, const P3<T>& t2) {
    P3<T> n = cross(sub(t1, t0), sub(t2, t0)); T s = dot(sub(p, t0), n); return s * s / dot(n, n); }
template <class T> T dist2_ee(const P3<T>& a0, const P3<T>& a1, const P3<T>& b0, const P3<T>& b1) {
    P3<T> n = cross(sub(a1, a0), sub(b1, b0)); T s = dot(sub(b0, a0), n); return s * s / dot(n, n); }

// ---------------------------------------------------------------------------------------
// symmetric eigen-decomposition (cyclic Jacobi) and PSD projection
// ---------------------------------------------------------------------------------------
void jacobi_eig(int n, const double* A_in, double* w, double* V) {
    std::vector<double> A(A_in, A_in + n * n);
    for (int i = 0; i < n * n; i++) V[i] = 0.0;
    for (int i = 0; i < n; i++) V[i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                tot += A[i * n + j] * A[i * n + j];
                if (i != j) off += A[i * n + j] * A[i * n + j];
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = A[p * n + q];
                if (std::fabs(apq) < 1e-300) continue;
                double app = A[p * n + p], aqq = A[q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < n; i++) w[i] = A[i * n + i];
}

// makePDGeneral (GIPC.cu:31-57): clamp negative eigenvalues to zero; untouched if PSD.
void make_pd(int n, double* A) {
    std::vector<double> w(n), V(n * n);
    jacobi_eig(n, A, w.data(), V.data());
    double mn = *std::min_element(w.begin(), w.end());
    if (mn >= 0.0) return;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int k = 0; k < n; k++)
                if (w[k] > 0.0) s += V[i * n + k] * w[k] * V[j * n + k];
            A[i * n + j] = s;
        }
}

// When 0, the SNK element Hessian is left unprojected (the exact second derivative), for
// checks of derivatives that need the true Jacobian of the gradient.
int g_project_snk = 1;

// ---------------------------------------------------------------------------------------
// stable Neo-Hookean tet (USE_SNK1)
// ---------------------------------------------------------------------------------------
// vec() is column-major: index 3*j + i holds F(i,j) (femEnergy.cu:1389-1435).
void snk_tet(const double* X /*4x3*/, const double* Dinv /*3x3 row-major*/, double vol,
             double mu, double lam, double dt2, double* energy, double* grad /*12*/,
             double* H12 /*144*/) {
    double Ds[3][3], F[3][3];
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) Ds[i][k] = X[(k + 1) * 3 + i] - X[i];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            F[i][j] = 0;
            for (int k = 0; k < 3; k++) F[i][j] += Ds[i][k] * Dinv[k * 3 + j];
        }
    double I2 = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) I2 += F[i][j] * F[i][j];
    double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
               F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    double Jm = J - 1.0 - mu / lam;
    if (energy) *energy = 0.5 * (mu * (I2 - 3.0) + lam * Jm * Jm) * vol * dt2;
    // columns f0,f1,f2 of F; dJ/dfj = f_{j+1} x f_{j+2}
    double f[3][3];
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) f[j][i] = F[i][j];
    double g[9];
    for (int j = 0; j < 3; j++) {
        const double* a = f[(j + 1) % 3];
        const double* b = f[(j + 2) % 3];
        g[3 * j + 0] = a[1] * b[2] - a[2] * b[1];
        g[3 * j + 1] = a[2] * b[0] - a[0] * b[2];
        g[3 * j + 2] = a[0] * b[1] - a[1] * b[0];
    }
    double P[9];
    for (int k = 0; k < 9; k++) P[k] = mu * f[k / 3][k % 3] + lam * Jm * g[k];
    // dF/dx (9x12): F(:,j) = sum_k (x_{k+1} - x_0) Dinv(k,j)
    double D[4][3];
    for (int j = 0; j < 3; j++) {
        D[0][j] = -(Dinv[0 * 3 + j] + Dinv[1 * 3 + j] + Dinv[2 * 3 + j]);
        for (int k = 0; k < 3; k++) D[k + 1][j] = Dinv[k * 3 + j];
    }
    double PF[9][12];
    std::memset(PF, 0, sizeof(PF));
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++)
            for (int a = 0; a < 4; a++) PF[3 * j + i][3 * a + i] = D[a][j];
    if (grad)
        for (int c = 0; c < 12; c++) {
            double s = 0;
            for (int r = 0; r < 9; r++) s += PF[r][c] * P[r];
            grad[c] = s * vol * dt2;
        }
    if (!H12) return;
    // exact Hessian in F: mu*I + lam*g g^T + lam*Jm * d2J/dF2
    double H[81];
    for (int r = 0; r < 9; r++)
        for (int c = 0; c < 9; c++) H[r * 9 + c] = (r == c ? mu : 0.0) + lam * g[r] * g[c];
    // d2J/(dF(:,j) dF(:,l)) for j != l: J = eps_abc f0_a f1_b f2_c
    const int eps[3][3][3] = {{{0, 0, 0}, {0, 0, 1}, {0, -1, 0}}, {{0, 0, -1}, {0, 0, 0}, {1, 0, 0}},
                              {{0, 1, 0}, {-1, 0, 0}, {0, 0, 0}}};
    for (int j = 0; j < 3; j++)
        for (int l = 0; l < 3; l++) {
            if (j == l) continue;
            int m = 3 - j - l;  // remaining column
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    double s = 0;
                    for (int c = 0; c < 3; c++) {
                        int idx[3];
                        idx[j] = a; idx[l] = b; idx[m] = c;
                        s += eps[idx[0]][idx[1]][idx[2]] * f[m][c];
                    }
                    H[(3 * j + a) * 9 + 3 * l + b] += lam * Jm * s;
                }
        }
    if (g_project_snk) make_pd(9, H);
    for (int r = 0; r < 12; r++)
        for (int c = 0; c < 12; c++) {
            double s = 0;
            for (int p = 0; p < 9; p++) {
                if (PF[p][r] == 0.0) continue;
                for (int q = 0; q < 9; q++) s += PF[p][r] * H[p * 9 + q] * PF[q][c];
            }
            H12[r * 12 + c] = s * vol * dt2;
        }
}

// ---------------------------------------------------------------------------------------
// Baraff-Witkin cloth membrane (femEnergy.cu:351-403 stress, 535-707 projected Hessians,
// 2146-2215 element kernel).  F = Ds Dm^-1 (3x2) with columns f0, f1;
//   E = area * dt^2 * [ k_st (S(|f0|) + S(|f1|)) + k_sh (f0.f1)^2 ],
//   S(t) = (t-1)^2 + [t > 1] s (t-1)^3.
// The reference projects the stretch Hessian (per column) and the shear Hessian to PSD
// separately and adds them; here each exact Hessian is built in closed form and projected
// by the numeric eigen-decomposition.  vec(F) is column-major (f0 then f1).
// ---------------------------------------------------------------------------------------
void tri_bw(const double* X /*3x3*/, const double* Dinv /*2x2 row-major*/, double area, double kst, double ksh,
            double srate, double dt2, double* energy, double* grad /*9*/, double* H9 /*81*/) {
    double f[2][3];
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < 3; i++)
            f[j][i] = (X[3 + i] - X[i]) * Dinv[0 * 2 + j] + (X[6 + i] - X[i]) * Dinv[1 * 2 + j];
    double E = 0, P[6] = {0}, Hf[36] = {0};
    for (int j = 0; j < 2; j++) {
        double t = std::sqrt(f[j][0] * f[j][0] + f[j][1] * f[j][1] + f[j][2] * f[j][2]);
        double u = t - 1.0;
        double S = u * u + (t > 1.0 ? srate * u * u * u : 0.0);
        double dS = 2.0 * u + (t > 1.0 ? 3.0 * srate * u * u : 0.0);
        double d2S = 2.0 + (t > 1.0 ? 6.0 * srate * u : 0.0);
        E += kst * S;
        double H3[9];
        for (int p = 0; p < 3; p++) {
            P[3 * j + p] += kst * dS / t * f[j][p];
            for (int q = 0; q < 3; q++) {
                double n2 = f[j][p] * f[j][q] / (t * t);
                H3[3 * p + q] = d2S * n2 + dS / t * ((p == q ? 1.0 : 0.0) - n2);
            }
        }
        make_pd(3, H3);
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++) Hf[(3 * j + p) * 6 + 3 * j + q] += kst * H3[3 * p + q];
    }
    // shear: E = I6^2, gradient 2 I6 g with g = [f1; f0], Hessian 2 (g g^T + I6 swap)
    double I6 = f[0][0] * f[1][0] + f[0][1] * f[1][1] + f[0][2] * f[1][2];
    E += ksh * I6 * I6;
    double g[6] = {f[1][0], f[1][1], f[1][2], f[0][0], f[0][1], f[0][2]};
    double Hs[36];
    for (int r = 0; r < 6; r++) {
        P[r] += ksh * 2.0 * I6 * g[r];
        for (int c = 0; c < 6; c++) Hs[r * 6 + c] = 2.0 * (g[r] * g[c] + ((c == (r + 3) % 6) ? I6 : 0.0));
    }
    make_pd(6, Hs);
    for (int k = 0; k < 36; k++) Hf[k] += ksh * Hs[k];
    // dF(:,j)/dx_a = D[a][j] I
    double D[3][2];
    for (int j = 0; j < 2; j++) {
        D[0][j] = -(Dinv[0 * 2 + j] + Dinv[1 * 2 + j]);
        D[1][j] = Dinv[0 * 2 + j];
        D[2][j] = Dinv[1 * 2 + j];
    }
    double sc = area * dt2;
    if (energy) *energy = E * sc;
    if (grad)
        for (int a = 0; a < 3; a++)
            for (int p = 0; p < 3; p++) grad[3 * a + p] = sc * (D[a][0] * P[p] + D[a][1] * P[3 + p]);
    if (H9)
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                for (int p = 0; p < 3; p++)
                    for (int q = 0; q < 3; q++) {
                        double h = 0;
                        for (int j = 0; j < 2; j++)
                            for (int l = 0; l < 2; l++) h += D[a][j] * D[b][l] * Hf[(3 * j + p) * 6 + 3 * l + q];
                        H9[(3 * a + p) * 9 + 3 * b + q] = sc * h;
                    }
}

// ---------------------------------------------------------------------------------------
// quadratic bending (femEnergy.cu:2623-2753): E = 1/2 c sum_ij Q_ij x_i . x_j with
// c = |rest e0 - rest e1| * bendStiff * dt^2, Q column-major 4x4 per hinge.
// ---------------------------------------------------------------------------------------
void hinge_quad(const double* X /*4x3*/, const double* Qcm, double c, double* energy, double* grad /*12*/,
                double* H12 /*144*/) {
    double E = 0;
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 3; k++) {
            double s = 0;
            for (int j = 0; j < 4; j++) s += Qcm[4 * j + i] * X[3 * j + k];
            if (grad) grad[3 * i + k] = c * s;
            E += 0.5 * c * X[3 * i + k] * s;
        }
    if (energy) *energy = E;
    if (H12)
        for (int r = 0; r < 12; r++)
            for (int cc = 0; cc < 12; cc++) H12[r * 12 + cc] = (r % 3 == cc % 3) ? c * Qcm[4 * (cc / 3) + r / 3] : 0.0;
}

// ---------------------------------------------------------------------------------------
// IPC barrier (RANK 2): b(I) = kappa * dhat^2 * (I-1)^2 * ln(I)^2, I = d^2 / dhat
// ---------------------------------------------------------------------------------------
struct BarrierScalars { double B, dB, d2B; };
BarrierScalars barrier_s(double I, double kappa, double dhat) {
    double L = std::log(I), c = kappa * dhat * dhat;
    BarrierScalars s;
    s.B = c * (I - 1) * (I - 1) * L * L;
    s.dB = c * (2 * (I - 1) * L * L + 2 * (I - 1) * (I - 1) * L / I);
    s.d2B = c * (2 * L * L + 8 * (I - 1) * L / I + 2 * (I - 1) * (I - 1) * (1 - L) / (I * I));
    return s;
}

// Decoded pair: vertex list and kind.
struct Pair {
    int kind;       // 0 PP, 1 PE, 2 PT, 3 EE, 4 mollified EE, 5 mollified PE, 6 mollified PP
    int nv;
    int v[4];
};
Pair decode(const int32_t* e) {
    Pair p;
    int x = e[0], y = e[1], z = e[2], w = e[3];
    if (x >= 0) {
        if (w >= 0) { p.kind = 3; p.nv = 4; p.v[0] = x; p.v[1] = y; p.v[2] = z; p.v[3] = w; }
        else { p.kind = 4; p.nv = 4; p.v[0] = x; p.v[1] = y; p.v[2] = z; p.v[3] = -w - 1; }
        return p;
    }
    int v0 = -x - 1;
    if (z < 0) {
        if (y < 0) { p.kind = 6; p.nv = 4; p.v[0] = v0; p.v[1] = -y - 1; p.v[2] = -z - 1; p.v[3] = -w - 1; }
        else { p.kind = 0; p.nv = 2; p.v[0] = v0; p.v[1] = y; p.v[2] = p.v[3] = -1; }
    } else if (w < 0) {
        if (y < 0) { p.kind = 5; p.nv = 4; p.v[0] = v0; p.v[1] = -y - 1; p.v[2] = z; p.v[3] = -w - 1; }
        else { p.kind = 1; p.nv = 3; p.v[0] = v0; p.v[1] = y; p.v[2] = z; p.v[3] = -1; }
    } else { p.kind = 2; p.nv = 4; p.v[0] = v0; p.v[1] = y; p.v[2] = z; p.v[3] = w; }
    return p;
}

typedef Dual<12> D12;
P3<D12> dvar(const double* x, int slot) {
    return {D12::var(x[0], 3 * slot), D12::var(x[1], 3 * slot + 1), D12::var(x[2], 3 * slot + 2)};
}

// squared distance of the pair's distance function, as a dual over its vertices
D12 pair_dist2(const Pair& p, const double* X) {
    P3<D12> a = dvar(X + 3 * p.v[0], 0), b = dvar(X + 3 * p.v[1], 1);
    switch (p.kind) {
        case 0: case 6: return dist2_pp(a, b);
        case 1: case 5: { P3<D12> c = dvar(X + 3 * p.v[2], 2); return dist2_pe(a, b, c); }
        case 2: { P3<D12> c = dvar(X + 3 * p.v[2], 2), d = dvar(X + 3 * p.v[3], 3); return dist2_pt(a, b, c, d); }
        default: { P3<D12> c = dvar(X + 3 * p.v[2], 2), d = dvar(X + 3 * p.v[3], 3); return dist2_ee(a, b, c, d); }
    }
}

// mollifier edge pair (c = |e0 x e1|) and rest-shape eps (GIPC.cu:3338-3360, 3640-3700, 4140-4200)
void moll_edges(const Pair& p, int e[4]) {
    if (p.kind == 4) { e[0] = 0; e[1] = 1; e[2] = 2; e[3] = 3; }        // (x,y) x (z,w)
    else if (p.kind == 6) { e[0] = 0; e[1] = 2; e[2] = 1; e[3] = 3; }   // (x,z) x (y,w)
    else { e[0] = 0; e[1] = 3; e[2] = 1; e[3] = 2; }                    // PE: (x,w) x (y,z)
}

// returns number of vertices; fills energy, grad (3*nv) and GN Hessian (3nv x 3nv, row-major 12 stride)
int barrier_pair(const int32_t* enc, const double* X, const double* R, double dhat, double kappa,
                 int* vid, double* energy, double* grad, double* H) {
    Pair p = decode(enc);
    for (int i = 0; i < 4; i++) vid[i] = p.v[i];
    for (int i = 0; i < 12; i++) grad[i] = 0;
    for (int i = 0; i < 144; i++) H[i] = 0;
    *energy = 0;
    D12 d2 = pair_dist2(p, X);
    double dsq = std::sqrt(dhat);
    // f = d / sqrt(dhat); grad f = grad(d^2) / (2 d sqrt(dhat))
    double dist = std::sqrt(d2.v);
    double gf[12];
    for (int i = 0; i < 12; i++) gf[i] = d2.d[i] / (2.0 * dist * dsq);
    double I = d2.v / dhat;
    if (p.kind <= 3) {
        BarrierScalars s = barrier_s(I, kappa, dhat);
        *energy = s.B;
        double f = std::sqrt(I);
        double dBdf = 2.0 * f * s.dB;
        double Ic = I;
        if (d2.v < 1e-6 * dhat) Ic = 1e-6;  // gassThreshold clamp (GIPC.cu:3258-3272)
        BarrierScalars sc = barrier_s(Ic, kappa, dhat);
        double lam0 = 4.0 * Ic * sc.d2B + 2.0 * sc.dB;
        for (int i = 0; i < 12; i++) grad[i] = dBdf * gf[i];
        for (int i = 0; i < 12; i++)
            for (int j = 0; j < 12; j++) H[i * 12 + j] = lam0 * gf[i] * gf[j];
        return p.nv;
    }
    // mollified: b = kappa * e(c^2) * Bt(I), e(s) = -s^2/eps^2 + 2 s/eps, Bt = dhat^2 (I-1)^2 ln^2 I
    int e[4];
    moll_edges(p, e);
    P3<D12> q0 = dvar(X + 3 * p.v[e[0]], e[0]), q1 = dvar(X + 3 * p.v[e[1]], e[1]);
    P3<D12> q2 = dvar(X + 3 * p.v[e[2]], e[2]), q3 = dvar(X + 3 * p.v[e[3]], e[3]);
    P3<D12> cr = cross(sub(q1, q0), sub(q3, q2));
    D12 c2 = dot(cr, cr);
    if (c2.v == 0.0) return p.nv;
    D12 c = dsqrt(c2);
    const double* r0 = R + 3 * p.v[e[0]]; const double* r1 = R + 3 * p.v[e[1]];
    const double* r2 = R + 3 * p.v[e[2]]; const double* r3 = R + 3 * p.v[e[3]];
    double l01 = 0, l23 = 0;
    for (int k = 0; k < 3; k++) { l01 += (r0[k] - r1[k]) * (r0[k] - r1[k]); l23 += (r2[k] - r3[k]) * (r2[k] - r3[k]); }
    double ex = 1e-3 * l01 * l23;
    double I1 = c2.v;
    double em = -I1 * I1 / (ex * ex) + 2.0 * I1 / ex;
    double dem = -2.0 * I1 / (ex * ex) + 2.0 / ex;
    BarrierScalars s = barrier_s(I, 1.0, dhat);
    *energy = kappa * em * s.B;
    double f = std::sqrt(I);
    double dbdc = kappa * dem * 2.0 * c.v * s.B;
    double dbdf = kappa * em * s.dB * 2.0 * f;
    for (int i = 0; i < 12; i++) grad[i] = dbdc * c.d[i] + dbdf * gf[i];
    double M[4];
    M[0] = kappa * s.B * (-4.0 * (3.0 * I1 - ex) / (ex * ex));                  // d2b/dc2
    M[3] = kappa * em * (4.0 * I * s.d2B + 2.0 * s.dB);                        // d2b/df2
    M[1] = M[2] = kappa * dem * 2.0 * c.v * s.dB * 2.0 * f;                    // d2b/dcdf
    make_pd(2, M);
    for (int i = 0; i < 12; i++)
        for (int j = 0; j < 12; j++)
            H[i * 12 + j] = M[0] * c.d[i] * c.d[j] + M[1] * (c.d[i] * gf[j] + gf[i] * c.d[j]) + M[3] * gf[i] * gf[j];
    return p.nv;
}

// ---------------------------------------------------------------------------------------
// friction (lagged, SFCLAMPING_ORDER 1)
// ---------------------------------------------------------------------------------------
// T (3nv x 2): lifts the 2D tangent relative displacement to the pair's vertices.
int friction_T(const int32_t* enc, const double* coord, const double* basis /*3x2 row-major*/,
               int* vid, double T[12][2]) {
    std::memset(T, 0, sizeof(double) * 24);
    int x = enc[0], y = enc[1], z = enc[2], w = enc[3];
    double coef[4];
    int nv;
    if (x >= 0) {
        vid[0] = x; vid[1] = y; vid[2] = z; vid[3] = w; nv = 4;
        coef[0] = 1.0 - coord[0]; coef[1] = coord[0]; coef[2] = coord[1] - 1.0; coef[3] = -coord[1];
    } else {
        int v0 = -x - 1;
        if (z < 0) { vid[0] = v0; vid[1] = y; vid[2] = vid[3] = -1; nv = 2; coef[0] = 1; coef[1] = -1; }
        else if (w < 0) { vid[0] = v0; vid[1] = y; vid[2] = z; vid[3] = -1; nv = 3;
            coef[0] = 1; coef[1] = coord[0] - 1.0; coef[2] = -coord[0]; }
        else { vid[0] = v0; vid[1] = y; vid[2] = z; vid[3] = w; nv = 4;
            coef[0] = 1; coef[1] = -1.0 + coord[0] + coord[1]; coef[2] = -coord[0]; coef[3] = -coord[1]; }
    }
    for (int a = 0; a < nv; a++)
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 2; c++) T[3 * a + k][c] = coef[a] * basis[k * 2 + c];
    return nv;
}

int friction_pair(const int32_t* enc, const double* X, const double* X0, const double* coord,
                  const double* basis, double lastH, double mu, double eps2, int* vid,
                  double* energy, double* grad, double* H) {
    for (int i = 0; i < 12; i++) grad[i] = 0;
    for (int i = 0; i < 144; i++) H[i] = 0;
    *energy = 0;
    if (enc[0] < 0 && enc[1] < 0) { vid[0] = vid[1] = vid[2] = vid[3] = -1; return 0; }  // mollified: skipped
    if (enc[0] >= 0 && enc[3] < 0) { vid[0] = vid[1] = vid[2] = vid[3] = -1; return 0; }
    double T[12][2];
    int nv = friction_T(enc, coord, basis, vid, T);
    double u[2] = {0, 0};
    for (int a = 0; a < nv; a++)
        for (int k = 0; k < 3; k++) {
            double dx = X[3 * vid[a] + k] - X0[3 * vid[a] + k];
            u[0] += T[3 * a + k][0] * dx;
            u[1] += T[3 * a + k][1] * dx;
        }
    double eps = std::sqrt(eps2);
    double un2 = u[0] * u[0] + u[1] * u[1], un = std::sqrt(un2);
    double f0, f1_div, M[4];
    if (un2 > eps2) {
        f0 = un; f1_div = 1.0 / un;
        M[0] = 1.0 / un - u[0] * u[0] / (un2 * un); M[1] = M[2] = -u[0] * u[1] / (un2 * un);
        M[3] = 1.0 / un - u[1] * u[1] / (un2 * un);
    } else {
        f0 = un2 * (-un / 3.0 + eps) / (eps * eps) + eps / 3.0;
        f1_div = (-un + 2.0 * eps) / (eps * eps);
        double f2 = 2.0 * (eps - un) / (eps * eps);
        if (f2 != f1_div && un2 != 0.0) {
            double k = (f1_div - f2) / un2;
            M[0] = f1_div - k * u[0] * u[0]; M[1] = M[2] = -k * u[0] * u[1]; M[3] = f1_div - k * u[1] * u[1];
        } else { M[0] = M[3] = f1_div; M[1] = M[2] = 0; }
    }
    make_pd(2, M);
    double s = mu * lastH;
    *energy = s * f0;
    for (int r = 0; r < 3 * nv; r++) grad[r] = s * f1_div * (T[r][0] * u[0] + T[r][1] * u[1]);
    for (int r = 0; r < 3 * nv; r++)
        for (int c = 0; c < 3 * nv; c++) {
            double tm0 = T[r][0] * M[0] + T[r][1] * M[2], tm1 = T[r][0] * M[1] + T[r][1] * M[3];
            H[r * 12 + c] = s * (tm0 * T[c][0] + tm1 * T[c][1]);
        }
    return nv;
}

// ground friction (normal +y): _calFrictionHessian_gd (GIPC.cu:1357-1437), gradient GIPC.cu:5047
void friction_ground(const double* x, const double* x0, double lastH, double mu, double eps2,
                     double* energy, double* g, double* H) {
    double v[3] = {x[0] - x0[0], 0.0, x[2] - x0[2]};
    double m2 = v[0] * v[0] + v[2] * v[2];
    double eps = std::sqrt(eps2), s = mu * lastH;
    for (int i = 0; i < 9; i++) H[i] = 0;
    if (m2 > eps2) {
        double m = std::sqrt(m2);
        *energy = s * (m - eps * 0.5);
        g[0] = s * v[0] / m; g[1] = 0; g[2] = s * v[2] / m;
        double M[4] = {s / m - s * v[0] * v[0] / (m2 * m), -s * v[0] * v[2] / (m2 * m),
                       -s * v[0] * v[2] / (m2 * m), s / m - s * v[2] * v[2] / (m2 * m)};
        make_pd(2, M);
        H[0] = M[0]; H[2] = M[1]; H[6] = M[2]; H[8] = M[3];
    } else {
        *energy = s * m2 / eps * 0.5;
        g[0] = s * v[0] / eps; g[1] = 0; g[2] = s * v[2] / eps;
        H[0] = s / eps; H[8] = s / eps;
    }
}

// ---------------------------------------------------------------------------------------
// COO accumulation
// ---------------------------------------------------------------------------------------
struct Coo {
    std::vector<int64_t> key;
    std::vector<double> val;  // 9 per block
    void add(int r, int c, const double* b /*row-major 3x3*/) {
        key.push_back(((int64_t)r << 32) | (uint32_t)c);
        val.insert(val.end(), b, b + 9);
    }
};

// write the upper blocks of a (3nv x 3nv, stride 12) pair Hessian following the contact
// rules of computeGradientAndHessian (GIPC.cu:10183-10214): keep blocks with
// row <= col, zero blocks touching a Dirichlet vertex
void push_pair_blocks(Coo& coo, int nv, const int* vid, const double* H, const int32_t* btype) {
    for (int a = 0; a < nv; a++)
        for (int b = 0; b < nv; b++) {
            int r = vid[a], c = vid[b];
            if (r > c) continue;
            double blk[9];
            bool dir = btype && (btype[r] != 0 || btype[c] != 0);
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) blk[i * 3 + j] = dir ? 0.0 : H[(3 * a + i) * 12 + 3 * b + j];
            coo.add(r, c, blk);
        }
}

// upper blocks (a <= b by position in the element) of an element Hessian with stride 3nv,
// oriented (min, max) by vertex id, zeroed when they touch a Dirichlet vertex
void push_elem_blocks(Coo& coo, int nv, const int32_t* vid, const double* H, const int32_t* btype) {
    const int st = 3 * nv;
    for (int a = 0; a < nv; a++)
        for (int b = a; b < nv; b++) {
            int r = vid[a], c = vid[b];
            bool tr = r > c;
            bool dir = btype[r] != 0 || btype[c] != 0;
            double blk[9];
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    double v = tr ? H[(3 * b + i) * st + 3 * a + j] : H[(3 * a + i) * st + 3 * b + j];
                    blk[i * 3 + j] = dir ? 0.0 : v;
                }
            if (tr) coo.add(c, r, blk); else coo.add(r, c, blk);
        }
}

// ---------------------------------------------------------------------------------------
// affine bodies (abd_system/: abd_energy.inl:9-127, abd_jacobi_matrix.inl,
// setup_abd_system_gradient_and_hessian.cu:162-610).  Written with explicit J matrices:
// J(x) is 3x12 with J[r][r] = 1 and J[r][3 + 3r + c] = x_c (x = J q = p + A x_bar, the rows
// of A being a1, a2, a3).
// ---------------------------------------------------------------------------------------
void abd_J(const double* x, double J[3][12]) {
    for (int r = 0; r < 3; r++) {
        for (int k = 0; k < 12; k++) J[r][k] = 0.0;
        J[r][r] = 1.0;
        for (int c = 0; c < 3; c++) J[r][3 + 3 * r + c] = x[c];
    }
}

// orthogonality potential V = sum_i (|a_i|^2 - 1)^2 + sum_{i != j} (a_i . a_j)^2 and its
// exact 9x9 Hessian, by forward-mode dual numbers over the 9 entries of A
void abd_shape(const double* q, double* V, double* g9, double* H9) {
    // gradient by duals; Hessian by differentiating the dual gradient expression again
    // (each gradient component is a cubic polynomial: its derivative is taken with duals)
    auto grad_dual = [&](const Dual<9>* a, Dual<9>* g) {
        for (int i = 0; i < 3; i++) {
            Dual<9> ai2 = a[3 * i] * a[3 * i] + a[3 * i + 1] * a[3 * i + 1] + a[3 * i + 2] * a[3 * i + 2];
            for (int p = 0; p < 3; p++) {
                Dual<9> gi = 4.0 * ((ai2 - Dual<9>(1.0)) * a[3 * i + p]);
                for (int j = 0; j < 3; j++) {
                    if (j == i) continue;
                    Dual<9> aij = a[3 * i] * a[3 * j] + a[3 * i + 1] * a[3 * j + 1] + a[3 * i + 2] * a[3 * j + 2];
                    gi = gi + 4.0 * (aij * a[3 * j + p]);
                }
                g[3 * i + p] = gi;
            }
        }
    };
    Dual<9> a[9], g[9];
    for (int k = 0; k < 9; k++) a[k] = Dual<9>::var(q[3 + k], k);
    grad_dual(a, g);
    double v = 0;
    for (int i = 0; i < 3; i++) {
        double ai2 = q[3 + 3 * i] * q[3 + 3 * i] + q[4 + 3 * i] * q[4 + 3 * i] + q[5 + 3 * i] * q[5 + 3 * i];
        v += (ai2 - 1) * (ai2 - 1);
        for (int j = 0; j < 3; j++) {
            if (j == i) continue;
            double aij = q[3 + 3 * i] * q[3 + 3 * j] + q[4 + 3 * i] * q[4 + 3 * j] + q[5 + 3 * i] * q[5 + 3 * j];
            v += aij * aij;
        }
    }
    if (V) *V = v;
    for (int k = 0; k < 9; k++) {
        if (g9) g9[k] = g[k].v;
        if (H9)
            for (int l = 0; l < 9; l++) H9[9 * k + l] = g[k].d[l];
    }
}

}  // namespace

extern "C" {

// --------------------------------- element-level API ----------------------------------

void or_snk_tet(const double* X, const double* Dinv, double vol, double mu, double lam, double dt2,
                double* energy, double* grad, double* H12) {
    snk_tet(X, Dinv, vol, mu, lam, dt2, energy, grad, H12);
}

int or_barrier_pair(const int32_t* enc, const double* X, const double* R, double dhat, double kappa,
                    int* vid, double* energy, double* grad, double* H) {
    return barrier_pair(enc, X, R, dhat, kappa, vid, energy, grad, H);
}

int or_friction_pair(const int32_t* enc, const double* X, const double* X0, const double* coord,
                     const double* basis, double lastH, double mu, double eps2, int* vid,
                     double* energy, double* grad, double* H) {
    return friction_pair(enc, X, X0, coord, basis, lastH, mu, eps2, vid, energy, grad, H);
}

void or_friction_ground(const double* x, const double* x0, double lastH, double mu, double eps2,
                        double* energy, double* g, double* H) {
    friction_ground(x, x0, lastH, mu, eps2, energy, g, H);
}

void or_make_pd(int n, double* A) { make_pd(n, A); }
void or_set_snk_projection(int on) { g_project_snk = on; }

// body gradient (12 per body) and the merged upper body-space BCOO; returns the block
// count, fills rows/cols/vals when rows != NULL (cap entries at most)
int or_abd_assemble(int B, int P, const int32_t* point_body, const double* x_bar, const double* dmass,
                    const double* vol, const int32_t* bt, const double* q, const double* qt, double kappa, double dt,
                    const double* point_grad, int nabd, const int32_t* arows, const int32_t* acols,
                    const double* avals, int nfem, const int32_t* frows, const int32_t* fcols, const double* fvals,
                    const int32_t* fbt, double* body_grad, int cap, int32_t* rows, int32_t* cols, double* vals) {
    Coo coo;
    auto add12 = [&](int rb, int cb, const double (*K)[12], bool upper_only) {
        for (int k = 0; k < 4; k++)
            for (int l = 0; l < 4; l++) {
                if (upper_only && k > l) continue;
                double blk[9];
                for (int p = 0; p < 3; p++)
                    for (int t = 0; t < 3; t++) blk[3 * p + t] = K[3 * k + p][3 * l + t];
                int r = 4 * rb + k, c = 4 * cb + l;
                if (r <= c) coo.add(r, c, blk);
                else {
                    double bt2[9];
                    for (int p = 0; p < 3; p++)
                        for (int t = 0; t < 3; t++) bt2[3 * p + t] = blk[3 * t + p];
                    coo.add(c, r, bt2);
                }
            }
    };
    for (int b = 0; b < B; b++) {
        const double* dm = dmass + 13 * b;
        // M = m J(0)^T J(0) generalised: entries 1, x_c, x_c x_d -> m, m x_c, m x_c x_d
        double M[12][12] = {{0}};
        for (int r = 0; r < 3; r++) {
            M[r][r] = dm[0];
            for (int c = 0; c < 3; c++) {
                M[r][3 + 3 * r + c] = M[3 + 3 * r + c][r] = dm[1 + c];
                for (int d = 0; d < 3; d++) M[3 + 3 * r + c][3 + 3 * r + d] = dm[4 + 3 * c + d];
            }
        }
        double G[12] = {0}, H[12][12];
        for (int i = 0; i < 12; i++)
            for (int j = 0; j < 12; j++) H[i][j] = M[i][j];
        if (bt[b] == 0) {
            for (int i = 0; i < 12; i++)
                for (int j = 0; j < 12; j++) G[i] += M[i][j] * (q[12 * b + j] - qt[12 * b + j]);
            double kvt2 = kappa * vol[b] * dt * dt, g9[9], H9[81];
            abd_shape(q + 12 * b, nullptr, g9, H9);
            for (int k = 0; k < 81; k++) H9[k] *= kvt2;
            make_pd(9, H9);
            for (int i = 0; i < 9; i++) {
                G[3 + i] += kvt2 * g9[i];
                for (int j = 0; j < 9; j++) H[3 + i][3 + j] += H9[9 * i + j];
            }
            // point barrier gradients: J^T g
            if (point_grad)
                for (int p = 0; p < P; p++) {
                    if (point_body[p] != b) continue;
                    double J[3][12];
                    abd_J(x_bar + 3 * p, J);
                    for (int k = 0; k < 12; k++)
                        for (int r = 0; r < 3; r++) G[k] += J[r][k] * point_grad[3 * p + r];
                }
        }
        for (int k = 0; k < 12; k++) body_grad[12 * b + k] = G[k];
        add12(b, b, H, true);
    }
    // ABD-ABD blocks: J_i^T H J_j (and its transpose for a same-body off-diagonal block)
    for (int e = 0; e < nabd; e++) {
        int i = arows[e], j = acols[e], bi = point_body[i], bj = point_body[j];
        double Ji[3][12], Jj[3][12], K[12][12];
        abd_J(x_bar + 3 * i, Ji);
        abd_J(x_bar + 3 * j, Jj);
        const double* Hp = avals + 9 * e;
        bool zero = bt[bi] != 0 || bt[bj] != 0;
        for (int k = 0; k < 12; k++)
            for (int l = 0; l < 12; l++) {
                double s = 0;
                for (int p = 0; p < 3; p++)
                    for (int t = 0; t < 3; t++) s += Ji[p][k] * Hp[3 * p + t] * Jj[t][l];
                K[k][l] = zero ? 0.0 : s;
            }
        if (bi == bj) {
            if (i != j) {
                double S[12][12];
                for (int k = 0; k < 12; k++)
                    for (int l = 0; l < 12; l++) S[k][l] = K[k][l] + K[l][k];
                add12(bi, bi, S, true);
            } else {
                add12(bi, bi, K, true);
            }
        } else {
            add12(bi, bj, K, false);
        }
    }
    // ABD-FEM blocks: J_i^T H into FEM column 4B + j
    for (int e = 0; e < nfem; e++) {
        int i = frows[e], j = fcols[e], b = point_body[i];
        double Ji[3][12];
        abd_J(x_bar + 3 * i, Ji);
        const double* Hp = fvals + 9 * e;
        bool zero = bt[b] != 0 || (fbt && fbt[j] != 0);
        for (int k = 0; k < 4; k++) {
            double blk[9];
            for (int p = 0; p < 3; p++)
                for (int t = 0; t < 3; t++) {
                    double s = 0;
                    for (int r = 0; r < 3; r++) s += Ji[r][3 * k + p] * Hp[3 * r + t];
                    blk[3 * p + t] = zero ? 0.0 : s;
                }
            coo.add(4 * b + k, 4 * B + j, blk);
        }
    }
    // merge
    std::vector<size_t> order(coo.key.size());
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](size_t a, size_t c) { return coo.key[a] < coo.key[c] || (coo.key[a] == coo.key[c] && a < c); });
    int nu = 0;
    for (size_t i = 0; i < order.size();) {
        size_t j = i;
        double acc[9] = {0};
        while (j < order.size() && coo.key[order[j]] == coo.key[order[i]]) {
            for (int k = 0; k < 9; k++) acc[k] += coo.val[9 * order[j] + k];
            j++;
        }
        if (rows && nu < cap) {
            rows[nu] = (int32_t)(coo.key[order[i]] >> 32);
            cols[nu] = (int32_t)(coo.key[order[i]] & 0xffffffff);
            std::memcpy(vals + 9 * nu, acc, sizeof(acc));
        }
        nu++;
        i = j;
    }
    return nu;
}
void or_tri_bw(const double* X, const double* Dinv, double area, double kst, double ksh, double srate, double dt2,
               double* energy, double* grad, double* H9) {
    tri_bw(X, Dinv, area, kst, ksh, srate, dt2, energy, grad, H9);
}

// Geometry of a barrier pair: f = d / sqrt(dhat) and its gradient over the pair's
// vertices (the last column of the reference's pFpx_* Jacobians), and for mollified
// pairs c = |e0 x e1| with its gradient (column 4 of pFpx_pee/ppe/ppp).  Returns nv.
int or_pair_geom(const int32_t* enc, const double* X, double dhat, double* f, double* gf, double* c, double* gc) {
    Pair p = decode(enc);
    D12 d2 = pair_dist2(p, X);
    double dist = std::sqrt(d2.v), dsq = std::sqrt(dhat);
    *f = dist / dsq;
    for (int i = 0; i < 12; i++) gf[i] = d2.d[i] / (2.0 * dist * dsq);
    *c = 0;
    for (int i = 0; i < 12; i++) gc[i] = 0;
    if (p.kind >= 4) {
        int e[4];
        moll_edges(p, e);
        P3<D12> q0 = dvar(X + 3 * p.v[e[0]], e[0]), q1 = dvar(X + 3 * p.v[e[1]], e[1]);
        P3<D12> q2 = dvar(X + 3 * p.v[e[2]], e[2]), q3 = dvar(X + 3 * p.v[e[3]], e[3]);
        P3<D12> cr = cross(sub(q1, q0), sub(q3, q2));
        D12 cc = dsqrt(dot(cr, cr));
        *c = cc.v;
        for (int i = 0; i < 12; i++) gc[i] = cc.d[i];
    }
    return p.nv;
}

void or_eig(int n, const double* A, double* w, double* V) { jacobi_eig(n, A, w, V); }

// --------------------------------- system assembly -----------------------------------

// Scene description (host arrays), mirrors device_TetraData + contacts.
typedef struct OrScene {
    int nv, nt, npairs, nground, nfric, nfric_gd, nsoft;
    const double* x;        // [nv*3]
    const double* x0;       // start of step
    const double* rest;
    const double* xt;       // xTilta
    const double* mass;
    const int32_t* btype;
    const int32_t* tets;    // [nt*4]
    const double* dminv;    // [nt*9]
    const double* vol;
    const double* lr;
    const double* vr;
    const int32_t* pairs;   // [npairs*4]
    const int32_t* gpairs;
    const int32_t* fpairs;
    const double* flam;
    const double* fcoord;
    const double* fbasis;   // [nfric*6]
    const int32_t* fgpairs;
    const double* fglam;
    const int32_t* soft_idx;
    const double* soft_target;
    double dt, dhat, kappa, fdhat, mu, mu_gd, ground_offset, motion_rate, soft_rate;
    // cloth: triangles (membrane) and hinges (quadratic bending)
    int nf, nh;
    const int32_t* tris;     // [nf*3]
    const double* tdminv;    // [nf*4] row-major 2x2
    const double* tarea;     // area * thickness
    const int32_t* hinges;   // [nh*2]
    const int32_t* hadj;     // [nh*2], -1 = boundary
    const double* hq;        // [nh*16] column-major
    double stretch, shear, strain_rate, bend;
} OrScene;

// Assemble gradient b (Dirichlet rows zeroed) and the merged upper BCOO.  Returns the
// number of unique blocks; if rows == NULL only counts.  Also returns the total energy.
int or_assemble(const OrScene* s, double* b, int cap, int32_t* rows, int32_t* cols, double* vals,
                double* energy_out) {
    int nv = s->nv;
    std::vector<double> grad(3 * nv, 0.0);
    double energy = 0.0;
    // kinetic (GIPC.cu:6339) -- energy 0.5*m*|x - xt|^2
    for (int i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) {
            double d = s->x[3 * i + k] - s->xt[3 * i + k];
            grad[3 * i + k] += s->mass[i] * d;
            energy += 0.5 * s->mass[i] * d * d;
        }
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    std::vector<Coo> coos(nth);
    std::vector<std::vector<double>> grads(nth, std::vector<double>(3 * nv, 0.0));
    std::vector<double> energies(nth, 0.0);
    double dt2 = s->dt * s->dt;
    double eps2 = s->fdhat * dt2;
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        Coo& coo = coos[tid];
        std::vector<double>& g = grads[tid];
        double& en = energies[tid];
        double e, gr[12], H[144];
        int vid[4];
        // barrier pairs
#pragma omp for schedule(static)
        for (int p = 0; p < s->npairs; p++) {
            int nvp = barrier_pair(s->pairs + 4 * p, s->x, s->rest, s->dhat, s->kappa, vid, &e, gr, H);
            en += e;
            for (int a = 0; a < nvp; a++)
                for (int k = 0; k < 3; k++) g[3 * vid[a] + k] += gr[3 * a + k];
            push_pair_blocks(coo, nvp, vid, H, s->btype);
        }
        // friction pairs
#pragma omp for schedule(static)
        for (int p = 0; p < s->nfric; p++) {
            int nvp = friction_pair(s->fpairs + 4 * p, s->x, s->x0, s->fcoord + 2 * p, s->fbasis + 6 * p,
                                    s->flam[p], s->mu, eps2, vid, &e, gr, H);
            en += e;
            for (int a = 0; a < nvp; a++)
                for (int k = 0; k < 3; k++) g[3 * vid[a] + k] += gr[3 * a + k];
            push_pair_blocks(coo, nvp, vid, H, s->btype);
        }
        // ground friction
#pragma omp for schedule(static)
        for (int p = 0; p < s->nfric_gd; p++) {
            int v = s->fgpairs[p];
            double H3[9], g3[3];
            friction_ground(s->x + 3 * v, s->x0 + 3 * v, s->fglam[p], s->mu_gd, eps2, &e, g3, H3);
            en += e;
            for (int k = 0; k < 3; k++) g[3 * v + k] += g3[k];
            if (s->btype[v] != 0) for (int k = 0; k < 9; k++) H3[k] = 0;
            coo.add(v, v, H3);
        }
        // ground barrier (GIPC.cu:6463-6514), RANK-1 form in d^2
#pragma omp for schedule(static)
        for (int p = 0; p < s->nground; p++) {
            int v = s->gpairs[p];
            double dist = s->x[3 * v + 1] - s->ground_offset;
            double d2 = dist * dist, t = d2 - s->dhat;
            double gb = t * std::log(d2 / s->dhat) * -2.0 - (t * t) / d2;
            double hb = (std::log(d2 / s->dhat) * -2.0 - t * 4.0 / d2) + 1.0 / (d2 * d2) * (t * t);
            en += -s->kappa * t * t * std::log(d2 / s->dhat);
            g[3 * v + 1] += s->kappa * gb * 2.0 * dist;
            double param = 4.0 * hb * d2 + 2.0 * gb;
            double H3[9] = {0, 0, 0, 0, s->kappa * param, 0, 0, 0, 0};
            if (s->btype[v] != 0) H3[4] = 0;
            coo.add(v, v, H3);
        }
        // soft constraints (GIPC.cu:6363-6407)
#pragma omp for schedule(static)
        for (int p = 0; p < s->nsoft; p++) {
            int v = s->soft_idx[p];
            double k = s->motion_rate * s->soft_rate * s->soft_rate;
            for (int c = 0; c < 3; c++) {
                double d = s->x[3 * v + c] - s->soft_target[3 * p + c];
                g[3 * v + c] += k * d;
                en += 0.5 * k * d * d;
            }
            double H3[9] = {k, 0, 0, 0, k, 0, 0, 0, k};
            if (s->btype[v] != 0) for (int c = 0; c < 9; c++) H3[c] = 0;
            coo.add(v, v, H3);
        }
        // stable Neo-Hookean tets: 10 upper blocks each
#pragma omp for schedule(static)
        for (int t = 0; t < s->nt; t++) {
            const int32_t* tv = s->tets + 4 * t;
            double X[12];
            for (int a = 0; a < 4; a++)
                for (int k = 0; k < 3; k++) X[3 * a + k] = s->x[3 * tv[a] + k];
            snk_tet(X, s->dminv + 9 * t, s->vol[t], s->lr[t], s->vr[t], dt2, &e, gr, H);
            en += e;
            for (int a = 0; a < 4; a++)
                for (int k = 0; k < 3; k++) g[3 * tv[a] + k] += gr[3 * a + k];
            for (int a = 0; a < 4; a++)
                for (int bb = a; bb < 4; bb++) {
                    int r = tv[a], c = tv[bb];
                    bool tr = r > c;
                    double blk[9];
                    bool dir = s->btype[r] != 0 || s->btype[c] != 0;
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) {
                            double v = tr ? H[(3 * bb + i) * 12 + 3 * a + j] : H[(3 * a + i) * 12 + 3 * bb + j];
                            blk[i * 3 + j] = dir ? 0.0 : v;
                        }
                    if (tr) coo.add(c, r, blk); else coo.add(r, c, blk);
                }
        }
        // cloth membrane: 6 upper blocks per triangle; quadratic bending: 10 per hinge
#pragma omp for schedule(static)
        for (int f = 0; f < s->nf; f++) {
            const int32_t* tv = s->tris + 3 * f;
            double X[9], H9[81];
            for (int a = 0; a < 3; a++)
                for (int k = 0; k < 3; k++) X[3 * a + k] = s->x[3 * tv[a] + k];
            tri_bw(X, s->tdminv + 4 * f, s->tarea[f], s->stretch, s->shear, s->strain_rate, dt2, &e, gr, H9);
            en += e;
            for (int a = 0; a < 3; a++)
                for (int k = 0; k < 3; k++) g[3 * tv[a] + k] += gr[3 * a + k];
            push_elem_blocks(coo, 3, tv, H9, s->btype);
        }
#pragma omp for schedule(static)
        for (int h = 0; h < s->nh; h++) {
            const int32_t hv[4] = {s->hinges[2 * h], s->hinges[2 * h + 1], s->hadj[2 * h], s->hadj[2 * h + 1]};
            if (hv[2] < 0 || hv[3] < 0) continue;  // boundary edge: no bending term
            double X[12], R0[3];
            for (int a = 0; a < 4; a++)
                for (int k = 0; k < 3; k++) X[3 * a + k] = s->x[3 * hv[a] + k];
            for (int k = 0; k < 3; k++) R0[k] = s->rest[3 * hv[0] + k] - s->rest[3 * hv[1] + k];
            double c = std::sqrt(R0[0] * R0[0] + R0[1] * R0[1] + R0[2] * R0[2]) * s->bend * dt2;
            hinge_quad(X, s->hq + 16 * h, c, &e, gr, H);
            en += e;
            for (int a = 0; a < 4; a++)
                for (int k = 0; k < 3; k++) g[3 * hv[a] + k] += gr[3 * a + k];
            push_elem_blocks(coo, 4, hv, H, s->btype);
        }
    }
    for (int t = 0; t < nth; t++) {
        energy += energies[t];
        for (int i = 0; i < 3 * nv; i++) grad[i] += grads[t][i];
    }
    // mass diagonal (added after the Dirichlet zeroing, GIPC.cu:10317-10336)
    Coo mass;
    for (int i = 0; i < nv; i++) {
        double blk[9] = {s->mass[i], 0, 0, 0, s->mass[i], 0, 0, 0, s->mass[i]};
        mass.add(i, i, blk);
    }
    // merge: sort keys, sum duplicates (Converter::convert, converter.cu:23-196)
    std::vector<int64_t> key;
    std::vector<const double*> src;
    for (auto* c : {&mass}) for (size_t i = 0; i < c->key.size(); i++) { key.push_back(c->key[i]); src.push_back(&c->val[9 * i]); }
    for (auto& c : coos) for (size_t i = 0; i < c.key.size(); i++) { key.push_back(c.key[i]); src.push_back(&c.val[9 * i]); }
    std::vector<size_t> order(key.size());
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](size_t a, size_t bq) { return key[a] < key[bq] || (key[a] == key[bq] && a < bq); });
    int nu = 0;
    for (size_t i = 0; i < order.size();) {
        size_t j = i;
        double acc[9] = {0};
        while (j < order.size() && key[order[j]] == key[order[i]]) {
            for (int k = 0; k < 9; k++) acc[k] += src[order[j]][k];
            j++;
        }
        if (rows && nu < cap) {
            rows[nu] = (int32_t)(key[order[i]] >> 32);
            cols[nu] = (int32_t)(key[order[i]] & 0xffffffff);
            std::memcpy(vals + 9 * nu, acc, sizeof(acc));
        }
        nu++;
        i = j;
    }
    if (b)
        for (int i = 0; i < nv; i++)
            for (int k = 0; k < 3; k++) b[3 * i + k] = s->btype[i] != 0 ? 0.0 : grad[3 * i + k];
    if (energy_out) *energy_out = energy;
    return nu;
}

// y = A x with A symmetric, given by its upper BCOO (spmv.cu:8-133)
void or_spmv(int nb, const int32_t* rows, const int32_t* cols, const double* vals, int n,
             const double* x, double* y) {
    std::fill(y, y + 3 * n, 0.0);
    for (int k = 0; k < nb; k++) {
        int r = rows[k], c = cols[k];
        const double* B = vals + 9 * k;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                y[3 * r + i] += B[i * 3 + j] * x[3 * c + j];
                if (r != c) y[3 * c + j] += B[i * 3 + j] * x[3 * r + i];
            }
    }
}

// --------------------------------- MAS preconditioner --------------------------------

// Level count (MASPreconditioner::computeNumLevels, MASPreconditioner.cu:1724-1743)
int or_mas_num_levels(int nodes) {
    int nLevel = 1;
    int levelSz = (nodes + 15) / 16 * 16;
    while (levelSz > 16) {
        levelSz /= 16;
        nLevel++;
        levelSz = (levelSz + 15) / 16 * 16;
    }
    nLevel = nLevel + 1;
    return nLevel > 6 ? 6 : nLevel;
}

typedef struct OrMas {
    int nv, npos, levelnum, total;
    int level_start[8];
    int level_count[8];
    std::vector<int>* table;    // [nv * levelnum] global cluster index per level (level 0 = position)
    std::vector<double>* inv;   // [total/16][48*48] dense inverses
} OrMas;

// Connected components of the bank-local graph given by per-node 16-bit masks; returns
// the new node id of every node (numbered bank by bank, components ordered by their
// lowest lane) and the number of new nodes.  Nodes with real[i] == 0 (padding positions
// of level 0) are no node: they are skipped, as _preparePrefixSumL0_new and
// _buildLevel1_new skip partId_map_real < 0 (MASPreconditioner.cu:157-270).
static int bank_components(int count, const std::vector<uint32_t>& mask, const std::vector<char>& real,
                           std::vector<int>& next) {
    next.assign(count, -1);
    int nid = 0;
    int nbank = (count + 15) / 16;
    for (int bk = 0; bk < nbank; bk++) {
        int lo = bk * 16, hi = std::min(count, lo + 16);
        // transitive closure of masks within the bank
        std::vector<uint32_t> comp(16, 0);
        for (int i = lo; i < hi; i++) comp[i - lo] = real[i] ? (mask[i] | (1u << (i - lo))) : 0u;
        bool changed = true;
        while (changed) {
            changed = false;
            for (int i = 0; i < hi - lo; i++) {
                uint32_t m = comp[i];
                for (int j = 0; j < 16; j++)
                    if (m & (1u << j)) m |= comp[j];
                if (m != comp[i]) { comp[i] = m; changed = true; }
            }
        }
        // symmetric closure: j in comp[i] => i in comp[j]
        for (int it = 0; it < 16; it++) {
            bool ch = false;
            for (int i = 0; i < hi - lo; i++)
                for (int j = 0; j < hi - lo; j++)
                    if ((comp[i] >> j & 1) && comp[j] != comp[i]) { comp[j] |= comp[i]; comp[i] |= comp[j]; ch = true; }
            if (!ch) break;
        }
        for (int i = lo; i < hi; i++) {
            if (!real[i]) continue;
            int lead = __builtin_ctz(comp[i - lo]);
            if (lead == i - lo) next[i] = nid++;
        }
        for (int i = lo; i < hi; i++)
            if (real[i]) next[i] = next[lo + __builtin_ctz(comp[i - lo])];
    }
    return nid;
}

// Build the hierarchy (ReorderRealtime, MASPreconditioner.cu:1772-1813) with the
// connectivity of mesh edges and of every vertex pair of every contact pair, then the
// domain matrices P_l^T A P_l restricted to 16-node banks (PrepareHessian_bcoo,
// MASPreconditioner.cu:1816-2093) and their Gauss-Jordan inverses
// (__inverse6_P96x96, MASPreconditioner.cu:630-726).
void* or_mas_build(int nv, int npos, const int32_t* part_map, const int32_t* real_map,
                   const uint32_t* nbr_start, const uint32_t* nbr_list, int npairs,
                   const int32_t* pairs, int nb, const int32_t* rows, const int32_t* cols,
                   const double* vals) {
    OrMas* M = new OrMas();
    M->nv = nv;
    M->npos = npos;
    M->levelnum = or_mas_num_levels(std::max(npos, nv));
    int L = M->levelnum;
    M->table = new std::vector<int>((size_t)nv * L, -1);
    std::vector<int>& tab = *M->table;
    // edge list: mesh + contact cliques
    std::vector<std::pair<int, int>> edges;
    for (int v = 0; v < nv; v++)
        for (uint32_t k = nbr_start[v]; k < nbr_start[v + 1]; k++) edges.push_back({v, (int)nbr_list[k]});
    for (int p = 0; p < npairs; p++) {
        const int32_t* e = pairs + 4 * p;
        int v[4];
        int x = e[0], y = e[1], z = e[2], w = e[3];
        int n = 0;
        if (x >= 0) { v[0] = x; v[1] = y; v[2] = z; v[3] = w < 0 ? -w - 1 : w; n = 4; }
        else {
            v[0] = -x - 1;
            if (z < 0) {
                if (y < 0) { v[1] = -y - 1; v[2] = -z - 1; v[3] = -w - 1; n = 4; }
                else { v[1] = y; n = 2; }
            } else if (w < 0) {
                if (y < 0) { v[1] = -y - 1; v[2] = z; v[3] = -w - 1; n = 4; }
                else { v[1] = y; v[2] = z; n = 3; }
            } else { v[1] = y; v[2] = z; v[3] = w; n = 4; }
        }
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++)
                if (v[i] >= 0 && v[j] >= 0 && v[i] < nv && v[j] < nv && v[i] != v[j]) {
                    edges.push_back({v[i], v[j]});
                    edges.push_back({v[j], v[i]});
                }
    }
    // level 0: positions
    for (int v = 0; v < nv; v++) tab[(size_t)v * L + 0] = real_map[v];
    M->level_start[0] = 0;
    M->level_count[0] = npos;
    std::vector<int> node(nv);  // node id (level-local) per vertex at the current level
    for (int v = 0; v < nv; v++) node[v] = real_map[v];
    int count = npos;
    int start = 0;
    int padded = npos;
    for (int l = 0; l < L - 1; l++) {
        std::vector<uint32_t> mask(count, 0);
        for (auto& e : edges) {
            int a = node[e.first], b = node[e.second];
            if (a != b && a / 16 == b / 16) mask[a] |= 1u << (b % 16);
        }
        std::vector<int> next;
        std::vector<char> real(count, 1);
        if (l == 0)
            for (int p = 0; p < count; p++) real[p] = part_map[p] >= 0;
        int nnext = bank_components(count, mask, real, next);
        start += padded;
        padded = (nnext + 15) / 16 * 16;
        M->level_start[l + 1] = start;
        M->level_count[l + 1] = nnext;
        for (int v = 0; v < nv; v++) {
            node[v] = next[node[v]];
            tab[(size_t)v * L + l + 1] = start + node[v];
        }
        count = nnext;
    }
    M->total = start + padded;
    int ndom = M->total / 16;
    M->inv = new std::vector<double>((size_t)ndom * 48 * 48, 0.0);
    std::vector<double>& A = *M->inv;
    auto addblk = [&](int ga, int gb, const double* B, bool transpose) {
        // ga, gb global cluster ids in the same bank; add B (or B^T) at (ga, gb)
        int d = ga / 16, la = ga % 16, lb = gb % 16;
        double* D = &A[(size_t)d * 2304];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) D[(3 * la + i) * 48 + 3 * lb + j] += transpose ? B[j * 3 + i] : B[i * 3 + j];
    };
    for (int k = 0; k < nb; k++) {
        int r = rows[k], c = cols[k];
        if (r >= nv || c >= nv || r < 0 || c < 0) continue;
        const double* B = vals + 9 * k;
        for (int l = 0; l < L; l++) {
            int ga = tab[(size_t)r * L + l], gb = tab[(size_t)c * L + l];
            if (ga / 16 != gb / 16) continue;
            addblk(ga, gb, B, false);
            if (r != c) addblk(gb, ga, B, true);
        }
    }
    // Gauss-Jordan without pivoting; a zero diagonal becomes 1
    for (int d = 0; d < ndom; d++) {
        double* D = &A[(size_t)d * 2304];
        for (int i = 0; i < 48; i++)
            if (D[i * 48 + i] == 0.0) D[i * 48 + i] = 1.0;
        std::vector<double> I(2304, 0.0);
        for (int i = 0; i < 48; i++) I[i * 48 + i] = 1.0;
        for (int j = 0; j < 48; j++) {
            double piv = D[j * 48 + j];
            for (int c = 0; c < 48; c++) { D[j * 48 + c] /= piv; I[j * 48 + c] /= piv; }
            for (int r = 0; r < 48; r++) {
                if (r == j) continue;
                double f = D[r * 48 + j];
                if (f == 0.0) continue;
                for (int c = 0; c < 48; c++) { D[r * 48 + c] -= f * D[j * 48 + c]; I[r * 48 + c] -= f * I[j * 48 + c]; }
            }
        }
        std::memcpy(D, I.data(), sizeof(double) * 2304);
    }
    return M;
}

void or_mas_free(void* h) {
    OrMas* M = (OrMas*)h;
    delete M->table;
    delete M->inv;
    delete M;
}

void or_mas_info(void* h, int* levelnum, int* starts, int* counts, int* total) {
    OrMas* M = (OrMas*)h;
    *levelnum = M->levelnum;
    for (int l = 0; l < M->levelnum; l++) { starts[l] = M->level_start[l]; counts[l] = M->level_count[l]; }
    *total = M->total;
}

void or_mas_domains(void* h, double* out) {
    OrMas* M = (OrMas*)h;
    std::copy(M->inv->begin(), M->inv->end(), out);
}

void or_mas_table(void* h, int32_t* out) {
    OrMas* M = (OrMas*)h;
    std::copy(M->table->begin(), M->table->end(), out);
}

// z = sum_l P_l^T A_l^-1 P_l r; single_inv rounds the inverses and vectors to FP32 as the
// reference's shipping configuration stores them (MasMatrixSymf, float3 Z).
void or_mas_apply(void* h, const double* r, double* z, int single) {
    OrMas* M = (OrMas*)h;
    int L = M->levelnum, nv = M->nv;
    std::vector<double> R((size_t)M->total * 3, 0.0), Z((size_t)M->total * 3, 0.0);
    for (int v = 0; v < nv; v++)
        for (int l = 0; l < L; l++) {
            int g = (*M->table)[(size_t)v * L + l];
            for (int k = 0; k < 3; k++) R[3 * g + k] += single ? (double)(float)r[3 * v + k] : r[3 * v + k];
        }
    if (single)
        for (auto& q : R) q = (double)(float)q;
    int ndom = M->total / 16;
#pragma omp parallel for schedule(static)
    for (int d = 0; d < ndom; d++) {
        const double* D = &(*M->inv)[(size_t)d * 2304];
        for (int i = 0; i < 48; i++) {
            double s = 0;
            for (int j = 0; j < 48; j++) {
                double a = single ? (double)(float)D[i * 48 + j] : D[i * 48 + j];
                s += a * R[48 * d + j];
            }
            Z[48 * d + i] = s;
        }
    }
    for (int v = 0; v < nv; v++)
        for (int k = 0; k < 3; k++) {
            double s = 0;
            for (int l = 0; l < L; l++) s += Z[3 * (*M->table)[(size_t)v * L + l] + k];
            z[3 * v + k] = s;
        }
}

// Reference PCG (pcg_solver.cu:174-267) with the MAS preconditioner; returns iterations.
int or_pcg(int nb, const int32_t* rows, const int32_t* cols, const double* vals, int n,
           void* mas, int single, const double* b, double* x, double tol, int max_iter,
           double* rz0_out, double* rz_out) {
    int N = 3 * n;
    std::vector<double> r(b, b + N), z(N), p(N), Ap(N);
    std::fill(x, x + N, 0.0);
    auto dotv = [&](const std::vector<double>& a, const std::vector<double>& c) {
        double s = 0;
        for (int i = 0; i < N; i++) s += a[i] * c[i];
        return s;
    };
    or_mas_apply(mas, r.data(), z.data(), single);
    double rz = dotv(r, z);
    p = z;
    double rz0 = rz;
    int k;
    for (k = 1; k < max_iter; ++k) {
        or_spmv(nb, rows, cols, vals, n, p.data(), Ap.data());
        double pAp = dotv(p, Ap);
        double alpha = rz / pAp;
        for (int i = 0; i < N; i++) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        if (std::fabs(rz) <= tol * rz0) break;
        or_mas_apply(mas, r.data(), z.data(), single);
        double rz_new = dotv(r, z);
        double beta = rz_new / rz;
        for (int i = 0; i < N; i++) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
    if (rz0_out) *rz0_out = rz0;
    if (rz_out) *rz_out = rz;
    return k;
}


// ---------------------------------------------------------------------------------------
// line-search step bounds (test infrastructure): additive CCD of point-triangle and
// edge-edge candidates (StiffGIPC/ACCD.cu:15-535, Li, Kaufman and Jiang 2021), the
// reference's per-candidate reduction (GIPC.cu:7052, self_largestFeasibleStepSize
// :8880-8914) and the ground plane bound (GIPC.cu:6902, ground_largestFeasibleStepSize
// :8986-9025).  Scalar FP64 loops over plain arrays.
// ---------------------------------------------------------------------------------------
namespace ccd {
struct V3 { double v[3]; };
static V3 sub(const V3& a, const V3& b) { return {{a.v[0] - b.v[0], a.v[1] - b.v[1], a.v[2] - b.v[2]}}; }
static V3 add(const V3& a, const V3& b) { return {{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2]}}; }
static V3 scl(double s, const V3& a) { return {{s * a.v[0], s * a.v[1], s * a.v[2]}}; }
static double dt(const V3& a, const V3& b) { return a.v[0] * b.v[0] + a.v[1] * b.v[1] + a.v[2] * b.v[2]; }
static V3 cr(const V3& a, const V3& b) {
    return {{a.v[1] * b.v[2] - a.v[2] * b.v[1], a.v[2] * b.v[0] - a.v[0] * b.v[2], a.v[0] * b.v[1] - a.v[1] * b.v[0]}};
}
static double n2(const V3& a) { return dt(a, a); }
// 3x3 determinant of the columns a, b, c
static double det3(const V3& a, const V3& b, const V3& c) {
    return a.v[0] * (b.v[1] * c.v[2] - b.v[2] * c.v[1]) - b.v[0] * (a.v[1] * c.v[2] - a.v[2] * c.v[1]) +
           c.v[0] * (a.v[1] * b.v[2] - a.v[2] * b.v[1]);
}
static double d_pp(const V3& a, const V3& b) { return n2(sub(a, b)); }
static double d_pe(const V3& p, const V3& e0, const V3& e1) { return n2(cr(sub(e0, p), sub(e1, p))) / n2(sub(e1, e0)); }
static double d_pplane(const V3& p, const V3& t0, const V3& t1, const V3& t2) {
    V3 n = cr(sub(t1, t0), sub(t2, t0));
    double s = dt(sub(p, t0), n);
    return s * s / n2(n);
}
static double d_ll(const V3& a0, const V3& a1, const V3& b0, const V3& b1) {
    V3 n = cr(sub(a1, a0), sub(b1, b0));
    double s = dt(sub(b0, a0), n);
    return s * s / n2(n);
}
static double d_pt(const V3& p, const V3& t0, const V3& t1, const V3& t2) {
    V3 n = cr(sub(t1, t0), sub(t2, t0));
    const V3* A[3] = {&t0, &t1, &t2};
    const V3* B[3] = {&t1, &t2, &t0};
    double s[3];
    for (int i = 0; i < 3; i++) {
        V3 e = sub(*B[i], *A[i]), f = cr(e, n), w = sub(p, *A[i]);
        double D = det3(e, f, n);
        s[i] = det3(w, f, n) / D;
        double h = det3(e, w, n) / D;
        if (s[i] > 0.0 && s[i] < 1.0 && h >= 0.0) return d_pe(p, *A[i], *B[i]);
    }
    if (s[0] <= 0.0 && s[2] >= 1.0) return d_pp(p, t0);
    if (s[1] <= 0.0 && s[0] >= 1.0) return d_pp(p, t1);
    if (s[2] <= 0.0 && s[1] >= 1.0) return d_pp(p, t2);
    return d_pplane(p, t0, t1, t2);
}
static double d_ee(const V3& a0, const V3& a1, const V3& b0, const V3& b1) {
    V3 u = sub(a1, a0), v = sub(b1, b0), w = sub(a0, b0);
    double a = n2(u), b = dt(u, v), c = n2(v), d = dt(u, w), e = dt(v, w);
    double D = a * c - b * b, sN = b * e - c * d, tN, tD = D;
    int kind = 8;
    if (sN <= 0.0) { tN = e; tD = c; kind = 2; }
    else if (sN >= D) { tN = e + b; tD = c; kind = 5; }
    else {
        tN = a * e - b * d;
        V3 uv = cr(u, v);
        if (tN > 0.0 && tN < tD && (dt(w, uv) == 0.0 || n2(uv) < 1.0e-20 * a * c)) {
            if (sN < D / 2) { tN = e; tD = c; kind = 2; }
            else { tN = e + b; tD = c; kind = 5; }
        }
    }
    if (tN <= 0.0) kind = (-d <= 0.0) ? 0 : ((-d >= a) ? 3 : 6);
    else if (tN >= tD) kind = (b - d <= 0.0) ? 1 : ((b - d >= a) ? 4 : 7);
    switch (kind) {
        case 0: return d_pp(a0, b0);
        case 1: return d_pp(a0, b1);
        case 2: return d_pe(a0, b0, b1);
        case 3: return d_pp(a1, b0);
        case 4: return d_pp(a1, b1);
        case 5: return d_pe(a1, b0, b1);
        case 6: return d_pe(b0, a0, a1);
        case 7: return d_pe(b1, a0, a1);
        default: return d_ll(a0, a1, b0, b1);
    }
}
// additive CCD: X[4] positions, M[4] displacements, eta the separation ratio kept
static double accd(bool ee, V3 X[4], V3 M[4], double eta) {
    V3 mov = ee ? scl(-0.25, add(add(M[0], M[1]), add(M[2], M[3]))) : scl(-0.25, add(add(M[1], M[2]), add(M[3], M[0])));
    for (int a = 0; a < 4; a++) M[a] = add(M[a], mov);
    double L = ee ? std::sqrt(std::max(n2(M[0]), n2(M[1]))) + std::sqrt(std::max(n2(M[2]), n2(M[3])))
                  : std::sqrt(n2(M[0])) + std::sqrt(std::max(n2(M[1]), std::max(n2(M[2]), n2(M[3]))));
    if (L == 0.0) return 1.0;
    auto dist2 = [&]() {
        double d2 = ee ? d_ee(X[0], X[1], X[2], X[3]) : d_pt(X[0], X[1], X[2], X[3]);
        if (ee && d2 <= 0.0)
            d2 = std::min(std::min(d_pp(X[0], X[2]), d_pp(X[0], X[3])), std::min(d_pp(X[1], X[2]), d_pp(X[1], X[3])));
        return d2;
    };
    double d2 = dist2(), d = std::sqrt(d2);
    const double gap = eta * d2 / d;
    double toc = 0.0;
    for (int it = 0; it < 50000; it++) {
        double step = (1.0 - eta) * d2 / (d * L);
        for (int a = 0; a < 4; a++) X[a] = add(X[a], scl(step, M[a]));
        d2 = dist2();
        d = std::sqrt(d2);
        if (toc != 0.0 && d2 / d < gap) return toc;
        toc += step;
        if (toc > 1.0) return 1.0;
    }
    return toc;
}
}  // namespace ccd

// step along -dir keeping every candidate (int32[4]: x < 0 point -x-1 vs triangle y z w,
// else edge x y vs edge z w) apart; toi (optional) per candidate
double or_self_step(const double* x, const double* dir, const int32_t* pairs, int n, double slackness, double* toi) {
    double vmax = 1.0;
    for (int i = 0; i < n; i++) {
        int v[4] = {pairs[4 * i], pairs[4 * i + 1], pairs[4 * i + 2], pairs[4 * i + 3]};
        bool ee = v[0] >= 0;
        if (!ee) v[0] = -v[0] - 1;
        ccd::V3 X[4], M[4];
        for (int a = 0; a < 4; a++)
            for (int k = 0; k < 3; k++) {
                X[a].v[k] = x[3 * v[a] + k];
                M[a].v[k] = -dir[3 * v[a] + k];
            }
        double t = ccd::accd(ee, X, M, 1.0 - slackness);
        if (toi) toi[i] = t;
        vmax = std::max(vmax, 1.0 / t);
    }
    return 1.0 / vmax;
}

// one additive-CCD time of impact: x12 / d12 the four positions and displacements (point,
// triangle or edge, edge), eta the separation ratio kept (point_triangle_ccd /
// edge_edge_ccd, ACCD.cu:373-535, thickness 0)
double or_accd(int ee, const double* x12, const double* d12, double eta) {
    ccd::V3 X[4], M[4];
    for (int a = 0; a < 4; a++)
        for (int k = 0; k < 3; k++) {
            X[a].v[k] = x12[3 * a + k];
            M[a].v[k] = d12[3 * a + k];
        }
    return ccd::accd(ee != 0, X, M, eta);
}

// step bound of vertices verts against the plane y = offset, normal +y
double or_ground_step(const double* x, const double* dir, const uint32_t* verts, int n, double offset,
                      double slackness) {
    double vmax = 1.0;
    for (int i = 0; i < n; i++) {
        uint32_t v = verts[i];
        double coef = dir[3 * v + 1];
        if (coef > 0.0) vmax = std::max(vmax, coef / ((x[3 * v + 1] - offset) * slackness));
    }
    return 1.0 / vmax;
}

// largest |dir| over the vertices verts (GIPC.cu:7157, cfl_largestSpeed :8916-8944)
double or_cfl_speed(const double* dir, const uint32_t* verts, int n) {
    double m = 0.0;
    for (int i = 0; i < n; i++) {
        const double* d = dir + 3 * verts[i];
        m = std::max(m, std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
    }
    return m;
}

int or_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
