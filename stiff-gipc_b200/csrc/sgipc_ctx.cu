// sgipc_ctx.cu — context creation: the static symmetric-upper BSR pattern, element ->
// slot gather lists and every workspace.
//
// Replaces, at init time, what StiffGIPC re-derives every Newton iteration: the triplet
// buffers sized in GIPC::init (GIPC.cu:8593-8640) and the per-iteration radix sort /
// segmented reduce of Converter::convert (linear_system/utils/converter.cu:23-196).  The
// FEM connectivity never changes, so its block pattern is computed once here; element
// kernels then write straight into per-element block slots that a gather sums into the
// BSR values, deterministically and without atomics.
#include <algorithm>
#include <cub/cub.cuh>
#include <numeric>
#include <vector>

#include "sgipc_internal.cuh"

using namespace sgipc;

namespace {

template <class T>
SgipcStatus dalloc(SgipcCtx* c, T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc");
    return SGIPC_OK;
}

template <class T>
SgipcStatus upload(SgipcCtx* c, T** p, const std::vector<T>& h) {
    SgipcStatus s = dalloc(c, p, h.size());
    if (s != SGIPC_OK) return s;
    if (!h.empty()) SG_CHECK(c, cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SGIPC_OK;
}

#define SG_TRY(x)                          \
    do {                                   \
        SgipcStatus s_ = (x);              \
        if (s_ != SGIPC_OK) return s_;     \
    } while (0)

// local upper block pairs of a 4-vertex element, in the reference's write order
// (femEnergy.cu:1840-1856)
const int kPair4[10][2] = {{0, 0}, {0, 1}, {0, 2}, {0, 3}, {1, 1}, {1, 2}, {1, 3}, {2, 2}, {2, 3}, {3, 3}};
const int kPair3[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};

}  // namespace

static SgipcStatus build_static(SgipcCtx* c, const SgipcTopology* t) {
    const int nv = t->vertex_num;
    // element block keys: tets (10), triangles (6), hinges (10)
    std::vector<std::pair<int, int>> eb;  // (min, max) per element block, in element order
    eb.reserve((size_t)t->tet_num * 10 + (size_t)t->tri_num * 6 + (size_t)t->tri_edge_num * 10);
    std::vector<int> egv;                 // vertex of each element gradient row
    egv.reserve((size_t)t->tet_num * 4 + (size_t)t->tri_num * 3 + (size_t)t->tri_edge_num * 4);
    for (int e = 0; e < t->tet_num; e++) {
        const uint32_t* v = t->tetrahedras + 4 * e;
        for (int k = 0; k < 10; k++) {
            int a = v[kPair4[k][0]], b = v[kPair4[k][1]];
            eb.push_back({std::min(a, b), std::max(a, b)});
        }
        for (int a = 0; a < 4; a++) egv.push_back(v[a]);
    }
    for (int e = 0; e < t->tri_num; e++) {
        const uint32_t* v = t->triangles + 3 * e;
        for (int k = 0; k < 6; k++) {
            int a = v[kPair3[k][0]], b = v[kPair3[k][1]];
            eb.push_back({std::min(a, b), std::max(a, b)});
        }
        for (int a = 0; a < 3; a++) egv.push_back(v[a]);
    }
    for (int e = 0; e < t->tri_edge_num; e++) {
        int v[4] = {(int)t->tri_edges[2 * e], (int)t->tri_edges[2 * e + 1], t->tri_edge_adj_vertex[2 * e],
                    t->tri_edge_adj_vertex[2 * e + 1]};
        bool boundary = v[2] < 0 || v[3] < 0;
        for (int k = 0; k < 10; k++) {
            int a = v[kPair4[k][0]], b = v[kPair4[k][1]];
            if (boundary) a = b = v[0];  // boundary hinges contribute zero blocks (femEnergy.cu:2640-2660)
            eb.push_back({std::min(a, b), std::max(a, b)});
        }
        for (int a = 0; a < 4; a++) egv.push_back(boundary ? v[0] : v[a]);
    }
    for (auto& p : eb)
        if (p.first < 0 || p.second >= nv) {
            snprintf(c->err, sizeof(c->err), "element vertex index out of range");
            return SGIPC_BAD_INPUT;
        }
    // pattern: element blocks + the full diagonal (mass)
    std::vector<uint64_t> keys;
    keys.reserve(eb.size() + nv);
    for (auto& p : eb) keys.push_back(((uint64_t)p.first << 32) | (uint32_t)p.second);
    for (int i = 0; i < nv; i++) keys.push_back(((uint64_t)i << 32) | (uint32_t)i);
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    const int n = c->n, nnz = (int)keys.size();
    c->nnz = nnz;
    std::vector<int> row_ptr(n + 1, 0), col(nnz), slot_row(nnz), diag(n, -1);
    for (int s = 0; s < nnz; s++) {
        int r = (int)(keys[s] >> 32), cc = (int)(keys[s] & 0xffffffffu);
        row_ptr[r + 1]++;
        col[s] = cc;
        slot_row[s] = r;
        if (r == cc) diag[r] = s;
    }
    for (int i = 0; i < n; i++) row_ptr[i + 1] += row_ptr[i];
    // lower lists: slot (r, c) with r < c appears transposed in row c
    std::vector<int> low_ptr(n + 1, 0);
    for (int s = 0; s < nnz; s++)
        if (slot_row[s] != col[s]) low_ptr[col[s] + 1]++;
    for (int i = 0; i < n; i++) low_ptr[i + 1] += low_ptr[i];
    std::vector<int> low_slot(std::max(low_ptr[n], 1)), fill(low_ptr.begin(), low_ptr.end() - 1);
    for (int s = 0; s < nnz; s++)
        if (slot_row[s] != col[s]) low_slot[fill[col[s]]++] = s;
    // element block -> slot, then gather CSR by slot
    c->n_eblk = (int)eb.size();
    std::vector<int> eslot(eb.size());
    for (size_t e = 0; e < eb.size(); e++) {
        uint64_t k = ((uint64_t)eb[e].first << 32) | (uint32_t)eb[e].second;
        eslot[e] = (int)(std::lower_bound(keys.begin(), keys.end(), k) - keys.begin());
    }
    std::vector<int> cptr(nnz + 1, 0);
    for (int s : eslot) cptr[s + 1]++;
    for (int s = 0; s < nnz; s++) cptr[s + 1] += cptr[s];
    std::vector<int> contrib(std::max((size_t)1, eb.size())), cf(cptr.begin(), cptr.end() - 1);
    for (size_t e = 0; e < eb.size(); e++) contrib[cf[eslot[e]]++] = (int)e;
    // element gradient rows -> vertex gather CSR
    c->n_egrad = (int)egv.size();
    std::vector<int> vptr(nv + 1, 0);
    for (int v : egv) vptr[v + 1]++;
    for (int i = 0; i < nv; i++) vptr[i + 1] += vptr[i];
    std::vector<int> vinc(std::max((size_t)1, egv.size())), vf(vptr.begin(), vptr.end() - 1);
    for (size_t e = 0; e < egv.size(); e++) vinc[vf[egv[e]]++] = (int)e;

    // full symmetric pattern: row i holds its upper slots and the transposes of the
    // upper slots (j, i), j < i; every block sits contiguously with its column index
    std::vector<int> frow(n + 1, 0);
    for (int i = 0; i < n; i++) frow[i + 1] = (row_ptr[i + 1] - row_ptr[i]) + (low_ptr[i + 1] - low_ptr[i]);
    for (int i = 0; i < n; i++) frow[i + 1] += frow[i];
    c->nnz_full = frow[n];
    c->h_frow_ptr = (int*)malloc(sizeof(int) * (n + 1));
    if (!c->h_frow_ptr) return SGIPC_CUDA_ERROR;
    std::copy(frow.begin(), frow.end(), c->h_frow_ptr);
    std::vector<int> fcol(std::max(c->nnz_full, 1)), fup(nnz), flo(nnz, -1);
    for (int i = 0; i < n; i++) {
        int k = frow[i];
        for (int q = low_ptr[i]; q < low_ptr[i + 1]; q++) {  // (j, i) with j < i, as B^T
            int s = low_slot[q];
            fcol[k] = slot_row[s];
            flo[s] = k++;
        }
        for (int s = row_ptr[i]; s < row_ptr[i + 1]; s++) {
            fcol[k] = col[s];
            fup[s] = k++;
        }
    }
    SG_TRY(upload(c, &c->frow_ptr, frow));
    SG_TRY(upload(c, &c->fcol, fcol));
    SG_TRY(upload(c, &c->fup, fup));
    SG_TRY(upload(c, &c->flo, flo));
    // column sets of the fused persistent solve: CTA b of a one-CTA-per-SM grid takes rows
    // [128 b, 128 b + 128); its z values are prolonged once per iteration at the distinct
    // columns of those rows
    {
        int nsm = 0;
        SG_CHECK(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
        constexpr int rpc = 128;
        if (nsm > 0 && (long long)nsm * rpc >= n) {
            std::vector<int> cptr2(nsm + 1, 0), ccols, lcol(std::max(c->nnz_full, 1), 0), dslot(std::max(n, 1), 0);
            int cap = 0;
            for (int b = 0; b < nsm; b++) {
                const int r0 = std::min(n, b * rpc), r1 = std::min(n, r0 + rpc);
                std::vector<int> set(fcol.begin() + frow[r0], fcol.begin() + frow[r1]);
                std::sort(set.begin(), set.end());
                set.erase(std::unique(set.begin(), set.end()), set.end());
                cap = std::max(cap, (int)set.size());
                for (int e = frow[r0]; e < frow[r1]; e++)
                    lcol[e] = (int)(std::lower_bound(set.begin(), set.end(), fcol[e]) - set.begin());
                for (int i = r0; i < r1; i++) dslot[i] = (int)(std::lower_bound(set.begin(), set.end(), i) - set.begin());
                ccols.insert(ccols.end(), set.begin(), set.end());
                cptr2[b + 1] = (int)ccols.size();
            }
            if (ccols.empty()) ccols.push_back(0);
            SG_TRY(upload(c, &c->cs_ptr, cptr2));
            SG_TRY(upload(c, &c->cs_cols, ccols));
            SG_TRY(upload(c, &c->cs_lcol, lcol));
            SG_TRY(upload(c, &c->cs_dslot, dslot));
            c->cs_grid = nsm;
            c->cs_cap = cap;
        }
    }
    SG_TRY(dalloc(c, &c->fval64, (size_t)c->nnz_full * 9));
    SG_TRY(dalloc(c, &c->fval32, (size_t)c->nnz_full * 9));
    SG_TRY(upload(c, &c->row_ptr, row_ptr));
    SG_TRY(upload(c, &c->col, col));
    SG_TRY(upload(c, &c->slot_row, slot_row));
    SG_TRY(upload(c, &c->diag_slot, diag));
    SG_TRY(upload(c, &c->low_ptr, low_ptr));
    SG_TRY(upload(c, &c->low_slot, low_slot));
    SG_TRY(upload(c, &c->contrib_ptr, cptr));
    SG_TRY(upload(c, &c->contrib, contrib));
    SG_TRY(upload(c, &c->vinc_ptr, vptr));
    SG_TRY(upload(c, &c->vinc, vinc));
    SG_TRY(dalloc(c, &c->val64, (size_t)nnz * 9));
    SG_TRY(dalloc(c, &c->eblk, (size_t)c->n_eblk * 9));
    SG_TRY(dalloc(c, &c->egrad, (size_t)c->n_egrad * 3));
    return SGIPC_OK;
}

// A host copy of a topology array the caller passed in device memory (the reference keeps
// its connectivity in device_TetraData); host, pinned and managed arrays are read in place.
template <class T>
static const T* host_view(const T* p, size_t n, std::vector<T>& keep, cudaError_t& err) {
    if (!p || n == 0) return p;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();  // an unregistered host pointer on older runtimes
        return p;
    }
    if (a.type != cudaMemoryTypeDevice) return p;
    keep.resize(n);
    cudaError_t e = cudaMemcpy(keep.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) err = e;
    return keep.data();
}

extern "C" SgipcStatus sgipc_create(const SgipcTopology* t_in, int device, SgipcCtx** out) {
    if (!t_in || !out) return SGIPC_BAD_INPUT;
    *out = nullptr;
    {
        const SgipcTopology* t = t_in;  // counts and pointers, before any CUDA call
        if (t->vertex_num <= 0 || t->tet_num < 0 || t->tri_num < 0 || t->tri_edge_num < 0 || t->soft_num < 0 ||
            t->max_pairs < 0 || t->max_ground < 0 || t->max_fric_pairs < 0 || t->max_fric_ground < 0)
            return SGIPC_BAD_INPUT;
        if ((t->tet_num && !t->tetrahedras) || (t->tri_num && !t->triangles) ||
            (t->tri_edge_num && (!t->tri_edges || !t->tri_edge_adj_vertex)) || !t->partId_map_real ||
            !t->real_map_partId || !t->neighborStart || (t->soft_num && !t->targetIndex))
            return SGIPC_BAD_INPUT;
        if (t->part_map_size < t->vertex_num || t->part_map_size % SGIPC_BANK) return SGIPC_BAD_INPUT;
    }
    // the topology arrays as host arrays, wherever the caller keeps them
    SgipcTopology th = *t_in;
    std::vector<uint32_t> k_tets, k_tris, k_hin, k_soft, k_nstart, k_nlist;
    std::vector<int32_t> k_hadj, k_pm, k_rm;
    {
        sgipc::DeviceScope scope(device);
        if (scope.err != cudaSuccess) return SGIPC_CUDA_ERROR;
        cudaError_t err = cudaSuccess;
        const size_t nv = th.vertex_num > 0 ? (size_t)th.vertex_num : 0;
        th.tetrahedras = host_view(th.tetrahedras, 4 * (size_t)std::max(th.tet_num, 0), k_tets, err);
        th.triangles = host_view(th.triangles, 3 * (size_t)std::max(th.tri_num, 0), k_tris, err);
        th.tri_edges = host_view(th.tri_edges, 2 * (size_t)std::max(th.tri_edge_num, 0), k_hin, err);
        th.tri_edge_adj_vertex = host_view(th.tri_edge_adj_vertex, 2 * (size_t)std::max(th.tri_edge_num, 0), k_hadj, err);
        th.targetIndex = host_view(th.targetIndex, (size_t)std::max(th.soft_num, 0), k_soft, err);
        th.partId_map_real = host_view(th.partId_map_real, (size_t)std::max(th.part_map_size, 0), k_pm, err);
        th.real_map_partId = host_view(th.real_map_partId, nv, k_rm, err);
        th.neighborStart = host_view(th.neighborStart, nv + 1, k_nstart, err);
        if (err == cudaSuccess && th.neighborStart && nv > 0)
            th.neighborList = host_view(th.neighborList, (size_t)th.neighborStart[nv], k_nlist, err);
        if (err != cudaSuccess) return SGIPC_CUDA_ERROR;
    }
    const SgipcTopology* t = &th;
    SgipcCtx* c = new SgipcCtx();
    memset(c, 0, sizeof(SgipcCtx));
    c->device = device;
    sgipc::DeviceScope dev_scope(device);
    cudaError_t e = dev_scope.err;
    if (e != cudaSuccess) {
        delete c;
        return SGIPC_CUDA_ERROR;
    }
    c->nv = t->vertex_num;
    c->nt = t->tet_num;
    c->nf = t->tri_num;
    c->nh = t->tri_edge_num;
    c->nsoft = t->soft_num;
    c->n = t->vertex_num;
    c->max_pairs = t->max_pairs;
    c->max_ground = t->max_ground;
    c->max_fric = t->max_fric_pairs;
    c->max_fric_gd = t->max_fric_ground;
    c->max_rhs = t->max_rhs < 1 ? 1 : t->max_rhs;
    SgipcStatus st = build_static(c, t);
    auto fail = [&](SgipcStatus s) {
        sgipc_destroy(c);
        return s;
    };
    if (st != SGIPC_OK) return fail(st);
    // topology copies
    std::vector<uint32_t> tets(t->tetrahedras, t->tetrahedras + 4 * (size_t)t->tet_num);
    std::vector<uint32_t> tris(t->triangles ? t->triangles : nullptr,
                               t->triangles ? t->triangles + 3 * (size_t)t->tri_num : nullptr);
    std::vector<uint32_t> hin(t->tri_edges ? t->tri_edges : nullptr,
                              t->tri_edges ? t->tri_edges + 2 * (size_t)t->tri_edge_num : nullptr);
    std::vector<int32_t> hadj(t->tri_edge_adj_vertex ? t->tri_edge_adj_vertex : nullptr,
                              t->tri_edge_adj_vertex ? t->tri_edge_adj_vertex + 2 * (size_t)t->tri_edge_num : nullptr);
    std::vector<uint32_t> soft(t->targetIndex ? t->targetIndex : nullptr,
                               t->targetIndex ? t->targetIndex + t->soft_num : nullptr);
    for (uint32_t s : soft)
        if ((int)s >= c->nv) return fail(SGIPC_BAD_INPUT);
    if ((st = upload(c, &c->tets, tets)) != SGIPC_OK) return fail(st);
    if ((st = upload(c, &c->tris, tris)) != SGIPC_OK) return fail(st);
    if ((st = upload(c, &c->hinges, hin)) != SGIPC_OK) return fail(st);
    if ((st = upload(c, &c->hinge_adj, hadj)) != SGIPC_OK) return fail(st);
    if ((st = upload(c, &c->soft_idx, soft)) != SGIPC_OK) return fail(st);
    const int n = c->n;
    if ((st = dalloc(c, &c->shape_grads, 3 * (size_t)c->nv)) != SGIPC_OK) return fail(st);
    if ((st = dalloc(c, &c->fb, 3 * (size_t)c->nv)) != SGIPC_OK) return fail(st);
    if ((st = dalloc(c, &c->b, 3 * (size_t)n)) != SGIPC_OK) return fail(st);
    // contact block capacity: 10 upper blocks per barrier pair and per friction pair,
    // one per ground barrier / ground friction / soft constraint
    long long cap = 10LL * c->max_pairs + 10LL * c->max_fric + c->max_ground + c->max_fric_gd + c->nsoft + 1;
    if (cap > (1LL << 30)) return fail(SGIPC_CAPACITY);
    c->cap_cblk = (int)cap;
    if ((st = dalloc(c, &c->ckey, cap)) || (st = dalloc(c, &c->ckey_s, cap)) || (st = dalloc(c, &c->cidx, cap)) ||
        (st = dalloc(c, &c->cidx_s, cap)) || (st = dalloc(c, &c->cval, cap * 9)) ||
        (st = dalloc(c, &c->run_start, cap + 1)) ||
        (st = dalloc(c, &c->cflag, cap + 1)) || (st = dalloc(c, &c->nuc, 4)) || (st = dalloc(c, &c->uc_row, cap)) ||
        (st = dalloc(c, &c->uc_col, cap)) || (st = dalloc(c, &c->uc64, cap * 9)) ||
        (st = dalloc(c, &c->uc32, cap * 9)) || (st = dalloc(c, &c->cu_ptr, n + 1)) ||
        (st = dalloc(c, &c->cl_ptr, n + 1)) || (st = dalloc(c, &c->cl_idx, cap)) || (st = dalloc(c, &c->lcount, 2 * (size_t)n + 1)) ||
        (st = dalloc(c, &c->cl_col, cap)) || (st = dalloc(c, &c->cl64, cap * 9)) || (st = dalloc(c, &c->cl32, cap * 9)) ||
        (st = dalloc(c, &c->lpos, cap)) || (st = dalloc(c, &c->dflag, 4)))
        return fail(st);
    SG_CHECK(c, cudaMemset(c->dflag, 0, 4 * sizeof(int)));
    // energy partial sums: one per CTA of every term's kernel at the context's capacities
    {
        const long long cnt[9] = {c->nv, c->nt, c->nf, c->nh, c->nsoft, c->max_pairs, c->max_ground, c->max_fric,
                                  c->max_fric_gd};
        long long ecap = 1;
        for (long long v : cnt) ecap += nblk(v);
        c->en_cap = (int)ecap;
        if ((st = dalloc(c, &c->en_part, ecap)) || (st = dalloc(c, &c->en_terms, 16)) ||
            (st = dalloc(c, &c->ccd_part, 148 * 4)) || (st = dalloc(c, &c->ccd_out, 2)) ||
            (st = dalloc(c, &c->ccd_bad, 1)) || (st = dalloc(c, &c->en_ticket, 1)) ||
            (st = dalloc(c, &c->ccd_ticket, 1)))
            return fail(st);
        SG_CHECK(c, cudaMemset(c->ccd_bad, 0, sizeof(int)));
        SG_CHECK(c, cudaMemset(c->ccd_ticket, 0, sizeof(unsigned int)));
        SG_CHECK(c, cudaMemset(c->en_ticket, 0, sizeof(unsigned int)));
        SG_CHECK(c, cudaMallocHost((void**)&c->h_en, sizeof(double) * 16));
    }
    // contact block keys are (row << bits) | col with row, col < 2^bits - 1, so that the
    // all-ones key of an unused slot sorts after every real block
    int bits = 1;
    while ((1LL << bits) < (long long)n + 2) bits++;
    c->key_bits = bits;
    // CUB temporary storage: radix sort of cap pairs, exclusive scans of cap + 1 and n + 1 ints
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b1, c->ckey, c->ckey_s, c->cidx, c->cidx_s, (int)cap, 0, 64);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, c->cflag, c->cflag, (int)cap + 1);
    cub::DeviceScan::ExclusiveSum(nullptr, b3, c->lcount, c->cl_ptr, n + 1);
    c->cub_tmp_bytes = std::max(std::max(b1, b2), b3) + 256;
    if ((st = dalloc(c, (char**)&c->cub_tmp, c->cub_tmp_bytes)) != SGIPC_OK) return fail(st);
    SG_CHECK(c, cudaMemset(c->nuc, 0, 4 * sizeof(int)));
    if ((st = mas_create(c, t)) != SGIPC_OK) return fail(st);
    if ((st = pcg_create(c)) != SGIPC_OK) return fail(st);
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(cuda_fail(c, e, "cudaDeviceSynchronize"));
    *out = c;
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_destroy(SgipcCtx* c) {
    if (!c) return SGIPC_OK;
    sgipc::DeviceScope dev_scope(c->device);
    broad_destroy(c);
    pcg_destroy(c);
    mas_destroy(c);
    void* ptrs[] = {c->row_ptr, c->col, c->slot_row, c->diag_slot, c->low_ptr, c->low_slot, c->val64,
                    c->eblk, c->contrib_ptr, c->contrib, c->egrad, c->vinc_ptr, c->vinc, c->tets, c->tris,
                    c->hinges, c->hinge_adj, c->soft_idx, c->shape_grads, c->fb, c->b, c->ckey, c->ckey_s,
                    c->cidx, c->cidx_s, c->cval, c->cflag, c->nuc, c->uc_row, c->uc_col, c->uc64, c->uc32,
                    c->cu_ptr, c->cl_ptr, c->cl_idx, c->lcount, c->lpos, c->cub_tmp, c->dflag,
                    c->frow_ptr, c->fcol, c->fup, c->flo, c->fval64, c->fval32, c->cl_col, c->cl64, c->cl32, c->run_start, c->en_part, c->en_terms, c->ccd_part, c->ccd_out, c->ccd_bad, c->en_ticket, c->ccd_ticket,
                    c->cs_ptr, c->cs_cols, c->cs_lcol, c->cs_dslot, c->close_gid, c->close_gval, c->close_pid,
                    c->close_pval, c->close_cnt};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->h_en) cudaFreeHost(c->h_en);
    free(c->h_frow_ptr);
    delete c;
    return SGIPC_OK;
}

extern "C" const char* sgipc_status_string(SgipcStatus s) {
    switch (s) {
        case SGIPC_OK: return "ok";
        case SGIPC_CUDA_ERROR: return "cuda error";
        case SGIPC_NOT_CONVERGED: return "not converged";
        case SGIPC_BREAKDOWN: return "pcg breakdown";
        case SGIPC_BAD_INPUT: return "bad input";
        case SGIPC_CAPACITY: return "capacity exceeded";
        case SGIPC_NOT_READY: return "not ready";
    }
    return "unknown";
}

extern "C" const char* sgipc_last_error(const SgipcCtx* c) { return c ? c->err : ""; }

extern "C" SgipcStatus sgipc_set_wait_limit(SgipcCtx* c, int64_t polls) {
    if (!c || polls < 0) return SGIPC_BAD_INPUT;
    c->wait_limit = polls;
    return SGIPC_OK;
}

extern "C" SgipcStatus sgipc_get_rhs(SgipcCtx* c, double* b, void* stream) {
    if (!c || !b) return SGIPC_BAD_INPUT;
    if (!c->assembled) return SGIPC_NOT_READY;
    SG_DEVICE(c);
    SG_CHECK(c, cudaMemcpyAsync(b, c->b, 3 * sizeof(double) * c->n, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return SGIPC_OK;
}

namespace sgipc {
SgipcStatus check_device_flag(SgipcCtx* c, cudaStream_t s) {
    int h = 0;
    SG_CHECK(c, cudaMemcpyAsync(&h, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, s));
    SG_CHECK(c, cudaStreamSynchronize(s));
    if (h) {
        SG_CHECK(c, cudaMemsetAsync(c->dflag, 0, sizeof(int), s));
        snprintf(c->err, sizeof(c->err), "a contact pair names a vertex outside [0, vertex_num); it was skipped");
        return SGIPC_BAD_INPUT;
    }
    return SGIPC_OK;
}
}  // namespace sgipc

extern "C" SgipcStatus sgipc_export_bcoo(SgipcCtx* c, int32_t cap, int32_t* rows, int32_t* cols, double* vals,
                                         int32_t* count) {
    if (!c || !count) return SGIPC_BAD_INPUT;
    if (!c->assembled) return SGIPC_NOT_READY;
    SG_DEVICE(c);
    SG_CHECK(c, cudaDeviceSynchronize());
    {
        SgipcStatus fs = check_device_flag(c, 0);
        if (fs != SGIPC_OK) return fs;
    }
    int nuc = 0;
    SG_CHECK(c, cudaMemcpy(&nuc, c->nuc, sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> sr(c->nnz), sc(c->nnz), ur(nuc), ucc(nuc);
    std::vector<double> sv((size_t)c->nnz * 9), uv((size_t)nuc * 9);
    SG_CHECK(c, cudaMemcpy(sr.data(), c->slot_row, sizeof(int) * c->nnz, cudaMemcpyDeviceToHost));
    SG_CHECK(c, cudaMemcpy(sc.data(), c->col, sizeof(int) * c->nnz, cudaMemcpyDeviceToHost));
    SG_CHECK(c, cudaMemcpy(sv.data(), c->val64, sizeof(double) * 9 * c->nnz, cudaMemcpyDeviceToHost));
    if (nuc) {
        SG_CHECK(c, cudaMemcpy(ur.data(), c->uc_row, sizeof(int) * nuc, cudaMemcpyDeviceToHost));
        SG_CHECK(c, cudaMemcpy(ucc.data(), c->uc_col, sizeof(int) * nuc, cudaMemcpyDeviceToHost));
        SG_CHECK(c, cudaMemcpy(uv.data(), c->uc64, sizeof(double) * 9 * nuc, cudaMemcpyDeviceToHost));
    }
    // merge the two sorted lists, summing equal keys
    int i = 0, j = 0, k = 0;
    auto key = [](int r, int cc) { return ((uint64_t)r << 32) | (uint32_t)cc; };
    while (i < c->nnz || j < nuc) {
        uint64_t ki = i < c->nnz ? key(sr[i], sc[i]) : ~0ull;
        uint64_t kj = j < nuc ? key(ur[j], ucc[j]) : ~0ull;
        uint64_t kk = std::min(ki, kj);
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (ki == kk) {
            for (int q = 0; q < 9; q++) acc[q] += sv[(size_t)9 * i + q];
            i++;
        }
        if (kj == kk) {
            for (int q = 0; q < 9; q++) acc[q] += uv[(size_t)9 * j + q];
            j++;
        }
        if (rows && k < cap) {
            rows[k] = (int)(kk >> 32);
            cols[k] = (int)(kk & 0xffffffffu);
            for (int q = 0; q < 9; q++) vals[(size_t)9 * k + q] = acc[q];
        }
        k++;
    }
    *count = k;
    return (rows && k > cap) ? SGIPC_CAPACITY : SGIPC_OK;
}
