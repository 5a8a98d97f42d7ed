// sgipc_abd_ctx.cuh — the affine-body context, shared by the ABD unit (sgipc_abd.cu) and the
// global FEM + ABD solve (sgipc_global.cu).
#pragma once
#include "sgipc_internal.cuh"

struct SgipcAbdCtx {
    int device;
    int B, P, max_abd, max_fem, cap;
    char err[256];
    int* point_body;
    int* body_ptr;       // [B+1] points of each body
    int* bt;             // [B]
    double* x_bar;       // [3P]
    double* dmass;       // [13B]
    double* vol;         // [B]
    // merge
    unsigned long long* key;
    unsigned long long* key_s;
    int* idx;
    int* idx_s;
    double* val;         // [9 cap]
    int* flag;           // [cap+1]
    int* nu;             // device: unique blocks
    int* u_row;
    int* u_col;
    double* u_val;
    int m_last;          // emitted slots of the last call
    double* pinv;        // [144 B]
    int assembled;
    int pbuilt;          // block-Jacobi inverses of the current assembly
    void* cub_tmp;
    size_t cub_bytes;
    // global FEM + ABD solve (sgipc_global_pcg_solve): row pointers of the merged blocks,
    // their transposed (column-sorted) index and the PCG vectors; allocated on first use
    int g_cap_blk, g_cap_ptr;
    size_t g_cap_vec;
    int* g_rptr;         // [4B + 1]
    int* g_cptr;         // [4B + n + 1]
    unsigned long long* g_tkey;
    unsigned long long* g_tkey_s;
    int* g_tidx;
    int* g_tidx_s;
    double* g_vec;       // r, z, p, Ap of the global vector
    double* g_dot;       // device scalars
    void* g_cub;
    size_t g_cub_bytes;
};

namespace sgipc {
// z_b = P_b^-1 r_b for every body (the ABD block Jacobi of the last precond build), on s
void abd_precond_apply_async(SgipcAbdCtx* c, const double* r, double* z, cudaStream_t s);
}  // namespace sgipc
