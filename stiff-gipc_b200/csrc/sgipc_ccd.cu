// sgipc_ccd.cu — line-search step bounds: additive CCD over point-triangle and edge-edge
// candidates, and the ground plane.
//
// The reference bounds the Newton step before its line search by
//   GIPC::self_largestFeasibleStepSize   (GIPC.cu:8880-8914, per pair
//                                         _reduct_min_selfTimeStep_to_double GIPC.cu:7052)
//   GIPC::ground_largestFeasibleStepSize (GIPC.cu:8986-9025, per vertex
//                                         _reduct_min_groundTimeStep_to_double GIPC.cu:6902)
// with the additive CCD (ACD) of Li, Kaufman and Jiang, "Codimensional Incremental Potential
// Contact" (2021), as StiffGIPC/ACCD.cu:373-535 applies it: remove the pair's mean
// displacement, then advance by the conservative step (1 - eta) (d^2 - t^2) / ((d + t) L),
// L the largest relative displacement, until the separation falls below eta times the
// initial one.  The squared distances classify the closest features first (point-triangle:
// vertex / edge / face; edge-edge: the segment-segment closest-point cases of D. Sunday,
// "Distance between segments"), as ACCD.cu:15-372 does.  The step of the whole set is
// 1 / max(1 / toi) as in the reference; a max is exact, so the result does not depend on the
// reduction order.
#include <algorithm>

#include "sgipc_geom.cuh"
#include "sgipc_internal.cuh"

using namespace sgipc;

namespace {

constexpr int kCcdMaxIter = 50000;  // per pair, as ACCD.cu

__device__ double pt_d2(d3 p, d3 t0, d3 t1, d3 t2) {
    switch (pt_type(p, t0, t1, t2)) {
        case 0: return pp_d2(p, t0);
        case 1: return pp_d2(p, t1);
        case 2: return pp_d2(p, t2);
        case 3: return pe_d2(p, t0, t1);
        case 4: return pe_d2(p, t1, t2);
        case 5: return pe_d2(p, t2, t0);
        default: return pplane_d2(p, t0, t1, t2);
    }
}

__device__ double ee_d2(d3 a0, d3 a1, d3 b0, d3 b1) {
    switch (ee_type(a0, a1, b0, b1)) {
        case 0: return pp_d2(a0, b0);
        case 1: return pp_d2(a0, b1);
        case 2: return pe_d2(a0, b0, b1);
        case 3: return pp_d2(a1, b0);
        case 4: return pp_d2(a1, b1);
        case 5: return pe_d2(a1, b0, b1);
        case 6: return pe_d2(b0, a0, a1);
        case 7: return pe_d2(b1, a0, a1);
        default: return ll_d2(a0, a1, b0, b1);
    }
}

// Additive CCD of one pair: the four vertices X[0..3] move by D[0..3] over the unit step.
// Point-triangle (ee false): X[0] the point; edge-edge: X[0]X[1] against X[2]X[3].  eta is
// the separation kept (1 - slackness), thick the thickness.
__device__ double accd(bool ee, d3* X, d3* D, double eta, double thick) {
    // mean displacement, summed as (edge a) + (edge b) / (triangle's first two) + (rest)
    const d3 mean = ee ? -0.25 * ((D[0] + D[1]) + (D[2] + D[3])) : -0.25 * ((D[1] + D[2]) + (D[3] + D[0]));
#pragma unroll
    for (int a = 0; a < 4; a++) D[a] = D[a] + mean;
    double L;
    if (ee)
        L = sqrt(fmax(sq(D[0]), sq(D[1]))) + sqrt(fmax(sq(D[2]), sq(D[3])));
    else
        L = sqrt(sq(D[0])) + sqrt(fmax(sq(D[1]), fmax(sq(D[2]), sq(D[3]))));
    if (L == 0.0) return 1.0;
    const double t2 = thick * thick;
    // the current separation d^2 - t^2 (edge-edge: endpoint distances once it is not positive)
    auto sep = [&](double& d2) {
        d2 = ee ? ee_d2(X[0], X[1], X[2], X[3]) : pt_d2(X[0], X[1], X[2], X[3]);
        double f = d2 - t2;
        if (ee && f <= 0.0) {
            d2 = fmin(fmin(pp_d2(X[0], X[2]), pp_d2(X[0], X[3])), fmin(pp_d2(X[1], X[2]), pp_d2(X[1], X[3])));
            f = d2 - t2;
        }
        return f;
    };
    double d2, f = sep(d2), d = sqrt(d2);
    const double gap = eta * f / (d + thick);
    double toc = 0.0;
    for (int it = 0; it < kCcdMaxIter; it++) {
        const double step = (1.0 - eta) * f / ((d + thick) * L);
#pragma unroll
        for (int a = 0; a < 4; a++) X[a] = X[a] + step * D[a];
        f = sep(d2);
        d = sqrt(d2);
        if (toc != 0.0 && f / (d + thick) < gap) return toc;
        toc += step;
        if (toc > 1.0) return 1.0;
    }
    return toc;
}

// fixed-size grid of the step-size kernels (grid-stride loops over the candidates)
constexpr int kCcdGrid = 148 * 4;

// How a step-size launch ends: the last CTA to finish (ticket) takes m = max(init, every
// CTA's maximum), writes out[0] = 1 / m (step sizes) or m (speeds) and out[1] = the
// out-of-range flag, and resets the flag and the ticket for the next launch.
struct StepFinish {
    double init;
    int invert;
    double* out;
    int* bad;
    unsigned int* ticket;
};

// max over the CTA of v into part[blockIdx.x], then the finish above (every thread calls it)
__device__ __forceinline__ void cta_max(double v, double* __restrict__ part, const StepFinish& fin) {
    __shared__ double sw[SGIPC_BLOCK / 32];
    __shared__ bool last;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = sw[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sw[w]);
        part[blockIdx.x] = m;
        __threadfence();
        last = atomicAdd(fin.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x >= 32) return;
    __threadfence();
    double m = fin.init;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) m = fmax(m, __ldcg(part + i));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) {
        fin.out[0] = fin.invert ? 1.0 / m : m;
        fin.out[1] = (double)atomicExch(fin.bad, 0);
        *fin.ticket = 0u;
    }
}

// per candidate 1 / toi along -dir (the reference passes -moveDir as the displacement);
// candidates with a vertex index outside [0, nv) set bad[0] and count as 1
__global__ void __launch_bounds__(SGIPC_BLOCK) k_self_step(int np, int nv, const int4* __restrict__ pairs,
                                                           const double* __restrict__ x,
                                                           const double* __restrict__ dir, double eta,
                                                           double* __restrict__ toi, double* __restrict__ part,
                                                           StepFinish fin) {
    double vmax = 1.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        int4 q = pairs[i];
        const bool ee = q.x >= 0;
        if (!ee) q.x = -q.x - 1;
        const int v[4] = {q.x, q.y, q.z, q.w};
        bool ok = true;
#pragma unroll
        for (int a = 0; a < 4; a++) ok = ok && v[a] >= 0 && v[a] < nv;
        double inv = 1.0;
        if (ok) {
            d3 X[4], D[4];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                X[a] = ld3(x, v[a]);
                D[a] = -ld3(dir, v[a]);
            }
            const double t = accd(ee, X, D, eta, 0.0);
            inv = 1.0 / t;
            if (toi) toi[i] = t;
        } else {
            atomicOr(fin.bad, 1);
            if (toi) toi[i] = 1.0;
        }
        vmax = fmax(vmax, inv);
    }
    cta_max(vmax, part, fin);
}

// per surface vertex approaching the plane y = offset (dir . n > 0 with n = +y):
// dir_y / ((y - offset) slackness), else 1
__global__ void __launch_bounds__(SGIPC_BLOCK) k_ground_step(int ns, int nv, const uint32_t* __restrict__ verts,
                                                             const double* __restrict__ x,
                                                             const double* __restrict__ dir, double offset,
                                                             double slackness, double* __restrict__ part,
                                                             StepFinish fin) {
    double vmax = 1.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
        const uint32_t v = verts[i];
        if (v >= (uint32_t)nv) {
            atomicOr(fin.bad, 1);
            continue;
        }
        const double coef = dir[3 * v + 1];
        if (coef > 0.0) vmax = fmax(vmax, coef / ((x[3 * v + 1] - offset) * slackness));
    }
    cta_max(vmax, part, fin);
}

// largest |dir| over the vertices verts (_reduct_max_cfl_to_double, GIPC.cu:7157)
__global__ void __launch_bounds__(SGIPC_BLOCK) k_cfl_speed(int ns, int nv, const uint32_t* __restrict__ verts,
                                                           const double* __restrict__ dir, double* __restrict__ part,
                                                           StepFinish fin) {
    double vmax = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
        const uint32_t v = verts[i];
        if (v >= (uint32_t)nv) {
            atomicOr(fin.bad, 1);
            continue;
        }
        vmax = fmax(vmax, sqrt(sq(ld3(dir, (int)v))));
    }
    cta_max(vmax, part, fin);
}

StepFinish step_finish(SgipcCtx* c, bool speed) {
    return {speed ? 0.0 : 1.0, speed ? 0 : 1, c->ccd_out, c->ccd_bad, c->ccd_ticket};
}

SgipcStatus read_step(SgipcCtx* c, cudaStream_t s, double* value, const char* what) {
    SG_COUNT(c, 1);
    SG_LAUNCH_CHECK(c, what);
    SG_CHECK(c, cudaMemcpyAsync(c->h_en + 12, c->ccd_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    if (c->h_en[13] != 0.0) {
        snprintf(c->err, sizeof(c->err), "%s: a candidate names a vertex outside [0, %d)", what, c->nv);
        return SGIPC_BAD_INPUT;
    }
    *value = c->h_en[12];
    return SGIPC_OK;
}

// x = x_base - alpha dir for the free vertices (all with move_boundary), GIPC.cu:7937
__global__ void k_step_forward(int nv, double* __restrict__ x, const double* __restrict__ xb,
                               const double* __restrict__ dir, const int* __restrict__ btype, double alpha,
                               int move_boundary) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * nv) return;
    // product and difference rounded separately (no fused multiply-add), as the reference's
    // __minus(x, __s_vec_multiply(dir, alpha)) evaluates it: the trial positions are bitwise the same
    if (move_boundary || btype[i / 3] == 0) x[i] = __dsub_rn(xb[i], __dmul_rn(dir[i], alpha));
}

}  // namespace

extern "C" SgipcStatus sgipc_step_forward(SgipcCtx* c, double* x, const double* x_base, const double* move_dir,
                                          const int32_t* boundary_type, double alpha, int32_t move_boundary,
                                          void* stream) {
    if (!c || !x || !x_base || !move_dir || (!move_boundary && !boundary_type)) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    SG_COUNT(c, 1);
    k_step_forward<<<nblk(3LL * c->nv), SGIPC_BLOCK, 0, s>>>(c->nv, x, x_base, move_dir, boundary_type, alpha,
                                                             move_boundary);
    SG_LAUNCH_CHECK(c, "step forward");
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_self_step_size(SgipcCtx* c, const double* x, const double* move_dir,
                                            const int32_t* pairs, int32_t npairs, double slackness, double* alpha,
                                            double* toi, void* stream) {
    if (!c || !x || !move_dir || !alpha || npairs < 0 || (npairs > 0 && !pairs)) return SGIPC_BAD_INPUT;
    if (!(slackness > 0.0 && slackness <= 1.0)) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = std::max(1, std::min(nblk(npairs), kCcdGrid));
    k_self_step<<<grid, SGIPC_BLOCK, 0, s>>>(npairs, c->nv, (const int4*)pairs, x, move_dir, 1.0 - slackness, toi,
                                             c->ccd_part, step_finish(c, false));
    return read_step(c, s, alpha, "self step size");
}

extern "C" SgipcStatus sgipc_ground_step_size(SgipcCtx* c, const double* x, const double* move_dir,
                                              const uint32_t* verts, int32_t nverts, double ground_offset,
                                              double slackness, double* alpha, void* stream) {
    if (!c || !x || !move_dir || !alpha || nverts < 0 || (nverts > 0 && !verts)) return SGIPC_BAD_INPUT;
    if (!(slackness > 0.0 && slackness <= 1.0)) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = std::max(1, std::min(nblk(nverts), kCcdGrid));
    k_ground_step<<<grid, SGIPC_BLOCK, 0, s>>>(nverts, c->nv, verts, x, move_dir, ground_offset, slackness,
                                               c->ccd_part, step_finish(c, false));
    return read_step(c, s, alpha, "ground step size");
}

extern "C" SgipcStatus sgipc_cfl_largest_speed(SgipcCtx* c, const double* move_dir, const uint32_t* verts,
                                               int32_t nverts, double* speed, void* stream) {
    if (!c || !move_dir || !speed || nverts < 0 || (nverts > 0 && !verts)) return SGIPC_BAD_INPUT;
    SG_DEVICE(c);
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = std::max(1, std::min(nblk(nverts), kCcdGrid));
    k_cfl_speed<<<grid, SGIPC_BLOCK, 0, s>>>(nverts, c->nv, verts, move_dir, c->ccd_part, step_finish(c, true));
    return read_step(c, s, speed, "cfl speed");
}
