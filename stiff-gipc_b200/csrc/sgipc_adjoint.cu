// sgipc_adjoint.cu — parameter derivatives for the implicit-step adjoint (no counterpart
// in the reference).
//
// The implicit step x*(theta) solves g(x*; theta) = 0 with g the assembled gradient
// (StiffGIPC/GIPC.cu:10110-10344).  For a loss L(x*), the implicit function theorem gives
//     dL/dtheta = -lambda^T dg/dtheta,   A lambda = dL/dx*,
// where A is the same projected BSR Hessian the Newton solve uses (solved with the same
// MAS-PCG).  Two parameter families are differentiated here:
//   * Young's modulus E_t of every tet: the stable Neo-Hookean PK1
//     P = mu F + (lam (J-1) - mu) cof F (femEnergy.cu:432-459) is linear in (mu, lam) and
//     mu = 4/3 * E/(2(1+nu)), lam = E nu/((1+nu)(1-2nu)) + 5/6 * E/(2(1+nu))
//     (StiffGIPC/gl_main.cu:609-617), so dg_t/dE_t = dt^2 vol_t dF/dx^T vec(dP/dE);
//   * initial velocity v0_i: g_kin = M (x - x_prev - dt v0 - dt^2 g) (GIPC.cu:6339,
//     8073-8097), so dg_i/dv0_i = -dt m_i I and dL/dv0_i = dt m_i lambda_i.
// Element quantities are recomputed from x rather than stored.
#include "sgipc_internal.cuh"

using namespace sgipc;

namespace {

__global__ void k_dLdE(int nt, int nrhs, int nv, const uint32_t* __restrict__ tets, const double* __restrict__ x,
                       const double* __restrict__ dminv, const double* __restrict__ vol, const int32_t* __restrict__ bt,
                       double amu, double alam, double dt2, const double* __restrict__ lambda, double* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    uint4 tv = reinterpret_cast<const uint4*>(tets)[t];
    const int vid[4] = {(int)tv.x, (int)tv.y, (int)tv.z, (int)tv.w};
    d3 X0 = ld3(x, vid[0]);
    d3 e[3] = {ld3(x, vid[1]) - X0, ld3(x, vid[2]) - X0, ld3(x, vid[3]) - X0};
    double Di[3][3];
#pragma unroll
    for (int k = 0; k < 9; k++) Di[k / 3][k % 3] = dminv[9 * (size_t)t + k];
    d3 f[3];
#pragma unroll
    for (int j = 0; j < 3; j++) f[j] = Di[0][j] * e[0] + Di[1][j] * e[1] + Di[2][j] * e[2];
    d3 g0 = cross(f[1], f[2]), g1 = cross(f[2], f[0]), g2 = cross(f[0], f[1]);
    double J = dot(f[0], g0);
    double ev = alam * (J - 1.0) - amu;
    d3 P0 = amu * f[0] + ev * g0, P1 = amu * f[1] + ev * g1, P2 = amu * f[2] + ev * g2;
    const double sc = dt2 * vol[t];
    d3 gr[4];
#pragma unroll
    for (int k = 0; k < 3; k++) gr[k + 1] = sc * (Di[k][0] * P0 + Di[k][1] * P1 + Di[k][2] * P2);
    gr[0] = -(gr[1] + gr[2] + gr[3]);
    for (int r = 0; r < nrhs; r++) {
        const double* lam = lambda + (size_t)r * 3 * nv;
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < 4; a++)
            if (bt[vid[a]] == 0) s += dot(gr[a], ld3(lam, vid[a]));
        out[(size_t)r * nt + t] = -s;
    }
}

__global__ void k_dLdv0(int nv, int nrhs, const double* __restrict__ m, const int32_t* __restrict__ bt, double dt,
                        const double* __restrict__ lambda, double* __restrict__ out) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3LL * nv * nrhs) return;
    int v = (int)((k % (3LL * nv)) / 3);
    out[k] = bt[v] == 0 ? dt * m[v] * lambda[k] : 0.0;
}

}  // namespace

extern "C" SgipcStatus sgipc_adjoint_param_grads(SgipcCtx* c, const SgipcFemData* f, const SgipcParams* p,
                                                 double poisson, int32_t nrhs, const double* lambda, double* dLdE,
                                                 double* dLdv0, void* stream) {
    if (!c || !f || !p || !lambda || nrhs < 1) return SGIPC_BAD_INPUT;
    if (!f->vertexes || !f->masses || !f->BoundaryType || (c->nt && (!f->DmInverses || !f->volum)))
        return SGIPC_BAD_INPUT;
    if (!(poisson > -1.0 && poisson < 0.5)) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    const double shear = 1.0 / (2.0 * (1.0 + poisson));
    const double amu = 4.0 * shear / 3.0;
    const double alam = poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson)) + 5.0 * shear / 6.0;
    if (dLdE && c->nt > 0)
        k_dLdE<<<nblk(c->nt), SGIPC_BLOCK, 0, s>>>(c->nt, nrhs, c->nv, c->tets, f->vertexes, f->DmInverses, f->volum,
                                                   f->BoundaryType, amu, alam, p->dt * p->dt, lambda, dLdE);
    if (dLdv0)
        k_dLdv0<<<nblk(3LL * c->nv * nrhs), SGIPC_BLOCK, 0, s>>>(c->nv, nrhs, f->masses, f->BoundaryType, p->dt,
                                                                  lambda, dLdv0);
    SG_LAUNCH_CHECK(c, "adjoint parameter gradients");
    return SGIPC_OK;
}
