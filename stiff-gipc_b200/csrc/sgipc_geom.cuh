// sgipc_geom.cuh — squared distances and closest-feature classification of point-triangle
// and edge-edge primitives, shared by the line-search CCD (sgipc_ccd.cu) and the contact-pair
// search (sgipc_broad.cu).
//
// The classifications are the reference's _dType_PT / _dType_EE (StiffGIPC/mlbvh.cu:288-530),
// which ACCD.cu:15-262 repeats for the CCD; the distances are _d_PP / _d_PE / _d_PT / _d_EE
// (mlbvh.cu:229-260): point-line, point-plane and line-line squared distances.
#pragma once
#include "sgipc_math.cuh"

namespace {
using sgipc::d3;
using sgipc::cross;
using sgipc::dot;
using sgipc::sq;

__device__ __forceinline__ double pp_d2(d3 a, d3 b) { return sq(a - b); }
// squared distance of p to the line through e0, e1
__device__ __forceinline__ double pe_d2(d3 p, d3 e0, d3 e1) { return sq(cross(e0 - p, e1 - p)) / sq(e1 - e0); }
// squared distance of p to the plane of t0, t1, t2
__device__ __forceinline__ double pplane_d2(d3 p, d3 t0, d3 t1, d3 t2) {
    const d3 n = cross(t1 - t0, t2 - t0);
    const double s = dot(p - t0, n);
    return s * s / sq(n);
}
// squared distance between the lines through a0, a1 and b0, b1
__device__ __forceinline__ double ll_d2(d3 a0, d3 a1, d3 b0, d3 b1) {
    const d3 n = cross(a1 - a0, b1 - b0);
    const double s = dot(b0 - a0, n);
    return s * s / sq(n);
}

// det of the 3x3 matrix with columns a, b, c, expanded term by term in the order of the
// reference's __Determiant (gpu_eigen_libs.cu:1193-1201), so that the classification below
// rounds as the reference's does
__device__ __forceinline__ double det_cols(d3 a, d3 b, d3 c) {
    return a.x * b.y * c.z + a.y * b.z * c.x + a.z * b.x * c.y - a.z * b.y * c.x - a.x * c.y * b.z -
           b.x * a.y * c.z;
}

// Closest feature of triangle (t0, t1, t2) to p: 0-2 a vertex, 3-5 the edge t0t1 / t1t2 /
// t2t0, 6 the face.  For each edge (a, b), (s, h) solve [e, e x n, n] (s, h, k) = p - a by
// Cramer's rule; the edge is closest when 0 < s < 1 and h >= 0.
__device__ __forceinline__ int pt_type(d3 p, d3 t0, d3 t1, d3 t2) {
    const d3 n = cross(t1 - t0, t2 - t0);
    const d3 a[3] = {t0, t1, t2}, b[3] = {t1, t2, t0};
    double s[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const d3 e = b[i] - a[i], f = cross(e, n), w = p - a[i];
        const double D = det_cols(e, f, n);
        s[i] = det_cols(w, f, n) / D;
        const double h = det_cols(e, w, n) / D;
        if (s[i] > 0.0 && s[i] < 1.0 && h >= 0.0) return 3 + i;
    }
    if (s[0] <= 0.0 && s[2] >= 1.0) return 0;
    if (s[1] <= 0.0 && s[0] >= 1.0) return 1;
    if (s[2] <= 0.0 && s[1] >= 1.0) return 2;
    return 6;
}

// Closest features of segments a0a1 and b0b1 (Sunday's clamped closest-point parameters
// s on a, t on b): 0 a0-b0, 1 a0-b1, 2 a0-segment b, 3 a1-b0, 4 a1-b1, 5 a1-segment b,
// 6 b0-segment a, 7 b1-segment a, 8 the two lines.  Nearly parallel segments (a zero or
// tiny |u x v|) take an endpoint case instead of the lines.
__device__ __forceinline__ int ee_type(d3 a0, d3 a1, d3 b0, d3 b1) {
    const d3 u = a1 - a0, v = b1 - b0, w = a0 - b0;
    const double a = sq(u), b = dot(u, v), c = sq(v), d = dot(u, w), e = dot(v, w);
    const double D = a * c - b * b;
    const double sN = b * e - c * d;
    double tN, tD = D;
    int res = 8;
    if (sN <= 0.0) {  // s clamped to 0
        tN = e;
        tD = c;
        res = 2;
    } else if (sN >= D) {  // s clamped to 1
        tN = e + b;
        tD = c;
        res = 5;
    } else {
        tN = a * e - b * d;
        const d3 uv = cross(u, v);
        if (tN > 0.0 && tN < tD && (dot(w, uv) == 0.0 || sq(uv) < 1.0e-20 * a * c)) {
            if (sN < D / 2) {
                tN = e;
                tD = c;
                res = 2;
            } else {
                tN = e + b;
                tD = c;
                res = 5;
            }
        }
    }
    if (tN <= 0.0) {  // t clamped to 0: b0 against segment a
        if (-d <= 0.0) return 0;
        if (-d >= a) return 3;
        return 6;
    }
    if (tN >= tD) {  // t clamped to 1: b1 against segment a
        if (b - d <= 0.0) return 1;
        if (b - d >= a) return 4;
        return 7;
    }
    return res;
}

}  // namespace
