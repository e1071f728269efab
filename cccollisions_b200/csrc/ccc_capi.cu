// ccc_capi.cu — C ABI of the B200 collision engine (declarations in include/ccc_b200.h).
//
// Host orchestration only: argument checks, workspace carving, launches on the caller's
// stream.  No host-device synchronisation happens inside an operation; the device
// status word is read back only by ccc_read_status.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <atomic>

#include "../../include/ccc_b200.h"
#include "ccc_kernels.cuh"
#include "ccc_runtime.cuh"

using namespace ccc;

namespace ccc {

int g_num_sms[64] = {0};

int num_sms() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (g_num_sms[dev] == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        g_num_sms[dev] = n > 0 ? n : 148;
    }
    return g_num_sms[dev];
}

// ---- launch accounting and optional per-kernel event timing ----
std::atomic<int64_t> g_launches{0};
// elementary functions of the continuous-collision solver (MathLib); CUDA's own by default,
// which is what the reference calls
int g_math_lib = LIB_REFERENCE;
bool g_timing = false;
constexpr int MAX_TIMED = 8192;
struct Timed { const char* name; cudaEvent_t a, b; };
Timed g_timed[MAX_TIMED];
int g_ntimed = 0;
cudaEvent_t g_pool[2 * MAX_TIMED];
int g_pool_init = 0;

bool timing_active() { return g_timing; }

void timing_before(const char* name, cudaStream_t s, int* slot) {
    *slot = -1;
    if (!g_timing || g_ntimed >= MAX_TIMED) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
    int i = g_ntimed++;
    if (g_pool_init <= 2 * i + 1) {
        while (g_pool_init <= 2 * i + 1) cudaEventCreate(&g_pool[g_pool_init++]);
    }
    g_timed[i].name = name;
    g_timed[i].a = g_pool[2 * i];
    g_timed[i].b = g_pool[2 * i + 1];
    cudaEventRecord(g_timed[i].a, s);
    *slot = i;
}
void timing_after(int slot, cudaStream_t s) {
    ++g_launches;
    if (slot >= 0) cudaEventRecord(g_timed[slot].b, s);
}

}  // namespace ccc

namespace {

// Workspace layout (every section 256-byte aligned):
//   [header 64 B][mesh counters M][visit counters total-M]   <- zeroed per call
//   [mesh table: count, offsets M+1, data offsets M, slot ids M][rightmost total-M]
//   [nodes total x 64 B (mesh m's F-1 nodes from slot m*F)][candidates cap x 8 B]
struct Layout {
    int64_t hdr, mesh_cnt, visits, zero_end, moff, table, rmk, nodes, cand, end;
    int64_t cand_cap;
};

Layout layout(int64_t B, int64_t F, int64_t maxc, bool need_nodes) {
    Layout L;
    int64_t total = B * F;
    int64_t internal = total - B;
    L.hdr = 0;
    L.mesh_cnt = align_up(L.hdr + (int64_t)sizeof(WsHeader), 256);
    L.visits = align_up(L.mesh_cnt + B * 4, 256);
    L.zero_end = align_up(L.visits + internal * 4, 256);
    L.moff = L.zero_end;
    L.table = align_up(L.moff + (B + 1) * 4, 256);
    L.rmk = align_up(L.table + (3 * B + 4) * 4, 256);
    L.nodes = need_nodes ? align_up(L.rmk + internal * 4, 256) : L.rmk;
    L.cand = need_nodes ? align_up(L.nodes + total * (int64_t)sizeof(TNode), 256) : L.nodes;
    L.cand_cap = need_nodes ? total * maxc : 0;
    L.end = align_up(L.cand + L.cand_cap * 8, 256);
    return L;
}

// one wave of resident narrow-phase blocks (the kernels' launch bounds); the kernels loop
// over their work
inline int narrow_grid() { return num_sms() * NARROW_MIN_BLOCKS; }

int check_common(int dtype, int64_t B, int64_t F) {
    if (dtype != 0 && dtype != 1) return CCC_ERR_INVALID_ARG;
    if (B < 1 || F < 2) return CCC_ERR_INVALID_ARG;
    // int32 indexing inside the kernels (and headroom for the Karras range doubling); each
    // factor is bounded first so that the product cannot wrap
    const int64_t lim = (int64_t)1 << 28;
    if (B >= lim || F >= lim || B * F >= lim) return CCC_ERR_INVALID_ARG;
    return CCC_OK;
}

// True when B * F * per * k rows stay below 2^31 (int32 row indices in the kernels).  The
// test divides instead of multiplying, so a huge per-triangle capacity cannot wrap the
// product; B * F < 2^28 (check_common) and k <= 15 keep the divisor in range.
bool rows_fit(int64_t B, int64_t F, int64_t per, int64_t k = 1) {
    if (per < 1) return false;
    return per <= ((((int64_t)1 << 31) - 1) / (B * F * k));
}

struct Prepared {
    char* base;
    Layout L;
    WsHeader* hdr;
    int* mesh_cnt;
    int* visits;
    int* moff;
    int* rmk;
    TNode* nodes;
    int2* cand;
    int* table;
    Forest forest;
};

int prepare(void* ws, int64_t ws_bytes, int64_t B, int64_t F, int64_t maxc, bool need_nodes, cudaStream_t s,
            Prepared& P) {
    P.L = layout(B, F, maxc, need_nodes);
    if (ws == nullptr || ws_bytes < P.L.end) return CCC_ERR_WORKSPACE;
    P.base = (char*)ws;
    P.hdr = (WsHeader*)(P.base + P.L.hdr);
    P.mesh_cnt = (int*)(P.base + P.L.mesh_cnt);
    P.visits = (int*)(P.base + P.L.visits);
    P.moff = (int*)(P.base + P.L.moff);
    P.rmk = (int*)(P.base + P.L.rmk);
    P.nodes = (TNode*)(P.base + P.L.nodes);
    P.cand = (int2*)(P.base + P.L.cand);
    P.table = (int*)(P.base + P.L.table);
    // the packed table is stored twice over: moff (= voff) feeds the tensor-layout kernels
    P.forest.nm = P.table;
    P.forest.voff = P.moff;
    P.forest.poff = P.table + 4;
    P.forest.sid = P.table + 4 + B;
    if (cudaMemsetAsync(P.base, 0, (size_t)P.L.zero_end, s) != cudaSuccess) return CCC_ERR_CUDA;
    CCC_LAUNCH("k_uniform_offsets", s, k_uniform_offsets<<<grid_for(B + 1, 256), 256, 0, s>>>(
        P.table, P.moff, P.table + 4, P.table + 4 + B, (int)B, (int)F));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

// import + traversal shared by every query operation; candidates land in P.cand
template <class T>
int run_broad_phase(const void* bboxes, const int64_t* tree, const uint8_t* mask, int64_t B, int64_t F, T th,
                    bool exact_f32, Prepared& P, cudaStream_t s) {
    const T* bb = (const T*)bboxes;
    const long long* tr = (const long long*)tree;
    int M = (int)B;
    int total = (int)(B * F);
    int internal = total - M;
    CCC_LAUNCH("k_import_nodes", s, k_import_nodes<T><<<grid_for(internal, 256), 256, 0, s>>>(P.moff, M, internal, bb, tr, P.nodes, &P.hdr->status));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_import_rightmost", s, k_import_rightmost<<<grid_for(total, 256), 256, 0, s>>>(P.moff, M, total, tr, P.nodes, P.visits, P.rmk,
                                                            &P.hdr->status));
    CCC_LAUNCH_CHECK();
    int g = grid_for(total, TRAV_THREADS);
    int cap = (int)P.L.cand_cap;
    TensorLeaves<T> lv{bb, tr};
    if (mask) {
        if (exact_f32)
            CCC_LAUNCH("k_traverse", s, k_traverse<T, true, true><<<g, TRAV_THREADS, 0, s>>>(P.nodes, lv, P.forest, mask, th,
                                                                                             P.cand, cap, P.hdr, nullptr));
        else
            CCC_LAUNCH("k_traverse", s, k_traverse<T, true, false><<<g, TRAV_THREADS, 0, s>>>(P.nodes, lv, P.forest, mask, th,
                                                                                              P.cand, cap, P.hdr, nullptr));
    } else {
        if (exact_f32)
            CCC_LAUNCH("k_traverse", s, k_traverse<T, false, true><<<g, TRAV_THREADS, 0, s>>>(P.nodes, lv, P.forest, mask, th,
                                                                                              P.cand, cap, P.hdr, nullptr));
        else
            CCC_LAUNCH("k_traverse", s, k_traverse<T, false, false><<<g, TRAV_THREADS, 0, s>>>(P.nodes, lv, P.forest, mask,
                                                                                               th, P.cand, cap, P.hdr, nullptr));
    }
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T> constexpr bool is_f32() { return sizeof(T) == 4; }

template <class T>
int bvh_impl(const void* tri, const void* tri_next, int64_t B, int64_t F, void* bboxes, int64_t* tree, void* ws,
             int64_t ws_bytes, cudaStream_t s) {
    Prepared P;
    int rc = prepare(ws, ws_bytes, B, F, 0, false, s, P);
    if (rc) return rc;
    int M = (int)B, total = (int)(B * F), internal = total - M;
    long long* tr = (long long*)tree;
    CCC_LAUNCH("k_leaf_rows", s, k_leaf_rows<T><<<grid_for(total, 256), 256, 0, s>>>((const T*)tri, (const T*)tri_next, P.moff, M, total,
                                                         (T*)bboxes, tr));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_karras_identity", s, k_karras_identity<<<grid_for(internal, 256), 256, 0, s>>>(P.moff, M, internal, tr));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_refit", s, k_refit<T><<<grid_for(total, 256), 256, 0, s>>>(P.moff, M, total, (T*)bboxes, tr, P.visits, &P.hdr->status));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T>
int static_impl(const void* bboxes, const int64_t* tree, const void* tri, int64_t B, int64_t F, double threshold,
                int64_t max_collisions, int64_t* out, void* ws, int64_t ws_bytes, cudaStream_t s) {
    Prepared P;
    int rc = prepare(ws, ws_bytes, B, F, max_collisions, true, s, P);
    if (rc) return rc;
    // the reference passes a float threshold into T-typed kernels
    T th = (T)(float)threshold;
    rc = run_broad_phase<T>(bboxes, tree, nullptr, B, F, th, is_f32<T>() && th == 0, P, s);
    if (rc) return rc;
    CCC_LAUNCH("k_static_narrow", s, k_static_narrow<T><<<narrow_grid(), NARROW_THREADS, 0, s>>>(P.cand, (int)P.L.cand_cap, P.hdr, (const T*)tri, P.forest,
                                                                th, (long long*)out, (int)max_collisions, P.mesh_cnt));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T, int OP>
int te_impl(const void* bboxes, const int64_t* tree, const void* tri, int64_t B, int64_t F, int64_t max_collisions,
            int64_t* rows, void* coefs, int32_t* masks, void* ws, int64_t ws_bytes, cudaStream_t s) {
    Prepared P;
    int rc = prepare(ws, ws_bytes, B, F, max_collisions, true, s, P);
    if (rc) return rc;
    // the reference's triangle-edge queries traverse and intersect with threshold 0
    rc = run_broad_phase<T>(bboxes, tree, nullptr, B, F, (T)0, is_f32<T>(), P, s);
    if (rc) return rc;
    if (OP == TE_COLLISIONS) {
        CCC_WITH_LIB(CCC_LAUNCH("k_te_narrow", s, k_te_narrow<T, OP, LIBV><<<narrow_grid(), NARROW_THREADS, 0, s>>>(
            P.cand, (int)P.L.cand_cap, P.hdr, (const T*)tri, P.forest, (long long*)rows, (T*)coefs, (int*)masks,
            (int)max_collisions, P.mesh_cnt)));
    } else {
        CCC_LAUNCH("k_te_narrow", s, k_te_narrow<T, OP, LIB_PORTABLE><<<narrow_grid(), NARROW_THREADS, 0, s>>>(
            P.cand, (int)P.L.cand_cap, P.hdr, (const T*)tri, P.forest, (long long*)rows, (T*)coefs, (int*)masks,
            (int)max_collisions, P.mesh_cnt));
    }
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <int OP>
int te_entry(int dtype, const void* bboxes, const int64_t* tree, const void* triangles, int64_t B, int64_t F,
             int64_t max_collisions, int64_t* rows, void* coefs, int32_t* masks, void* ws, int64_t ws_bytes,
             void* stream) {
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (!bboxes || !tree || !triangles || !rows || max_collisions < 1) return CCC_ERR_INVALID_ARG;
    if (OP == TE_COLLISIONS && !coefs) return CCC_ERR_INVALID_ARG;
    if (OP == TE_CANDIDATES2 && !masks) return CCC_ERR_INVALID_ARG;
    if (!rows_fit(B, F, max_collisions)) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == 0 ? te_impl<float, OP>(bboxes, tree, triangles, B, F, max_collisions, rows, coefs, masks, ws,
                                           ws_bytes, s)
                      : te_impl<double, OP>(bboxes, tree, triangles, B, F, max_collisions, rows, coefs, masks, ws,
                                            ws_bytes, s);
}

template <class T>
int ccd_impl(const void* bboxes, const int64_t* tree, const void* x0, const void* x1, const uint8_t* mask, int64_t B,
             int64_t F, int64_t maxc, int64_t maxcol, int64_t* rows, void* times, void* ws, int64_t ws_bytes,
             cudaStream_t s) {
    Prepared P;
    int rc = prepare(ws, ws_bytes, B, F, maxc, true, s, P);
    if (rc) return rc;
    rc = run_broad_phase<T>(bboxes, tree, mask, B, F, (T)0, is_f32<T>(), P, s);
    if (rc) return rc;
    cudaError_t le = cudaSuccess;
    CCC_WITH_LIB(CCC_LAUNCH("k_ccd_narrow", s, le = launch_ccd_narrow<T, CCD_ROWS, CornerSink<T>, LIBV, SRC_CANDIDATES>(
        num_sms() * CCD_MIN_BLOCKS, s, P.cand, (int)P.L.cand_cap, P.hdr, (const T*)x0, (const T*)x1, P.forest, (long long*)rows,
        (T*)times, (int)maxcol, P.mesh_cnt, Weld{}, CornerSink<T>{})));
    if (le != cudaSuccess) return CCC_ERR_CUDA;
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T>
int mincol_impl(const void* bboxes, const int64_t* tree, const void* x0, const void* x1, int64_t B, int64_t F,
                int64_t maxc, int64_t* rows, void* ws, int64_t ws_bytes, cudaStream_t s) {
    Prepared P;
    int rc = prepare(ws, ws_bytes, B, F, maxc, true, s, P);
    if (rc) return rc;
    rc = run_broad_phase<T>(bboxes, tree, nullptr, B, F, (T)0, is_f32<T>(), P, s);
    if (rc) return rc;
    cudaError_t le = cudaSuccess;
    CCC_LAUNCH("k_ccd_narrow", s, le = launch_ccd_narrow<T, CCD_MINCOL, CornerSink<T>, LIB_PORTABLE, SRC_CANDIDATES>(
        num_sms() * CCD_MIN_BLOCKS, s, P.cand, (int)P.L.cand_cap, P.hdr, (const T*)x0, (const T*)x1, P.forest, (long long*)rows,
        nullptr, (int)(maxc * 15), P.mesh_cnt, Weld{}, CornerSink<T>{}));
    if (le != cudaSuccess) return CCC_ERR_CUDA;
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T>
int prox_impl(const void* bboxes, const int64_t* tree, const void* tri, int64_t B, int64_t F, double threshold,
              int64_t maxc, int64_t* rows, void* ws, int64_t ws_bytes, cudaStream_t s) {
    Prepared P;
    int rc = prepare(ws, ws_bytes, B, F, maxc, true, s, P);
    if (rc) return rc;
    T th = (T)(float)threshold;
    rc = run_broad_phase<T>(bboxes, tree, nullptr, B, F, th, is_f32<T>() && th == 0, P, s);
    if (rc) return rc;
    CCC_LAUNCH("k_prox_narrow", s, k_prox_narrow<T><<<narrow_grid(), NARROW_THREADS, 0, s>>>(P.cand, (int)P.L.cand_cap, P.hdr, (const T*)tri, P.forest,
                                                              th, (long long*)rows, (int)maxc, P.mesh_cnt));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T>
int impulses_impl(const void* bboxes, const int64_t* tree, const void* x0, const void* x1, const void* masses,
                  const uint8_t* mask, int64_t B, int64_t F, int64_t maxc, void* dv, void* dx, int32_t* cnt, void* ws,
                  int64_t ws_bytes, cudaStream_t s) {
    Prepared P;
    int rc = prepare(ws, ws_bytes, B, F, maxc, true, s, P);
    if (rc) return rc;
    rc = run_broad_phase<T>(bboxes, tree, mask, B, F, (T)0, is_f32<T>(), P, s);
    if (rc) return rc;
    cudaError_t le = cudaSuccess;
    CCC_WITH_LIB(CCC_LAUNCH("k_ccd_narrow", s, le = launch_ccd_narrow<T, CCD_IMPULSES, CornerSink<T>, LIBV, SRC_CANDIDATES>(
        num_sms() * CCD_MIN_BLOCKS, s, P.cand, (int)P.L.cand_cap, P.hdr, (const T*)x0, (const T*)x1, P.forest, nullptr, nullptr, 0,
        P.mesh_cnt, Weld{}, CornerSink<T>{(const T*)masses, (T*)dv, (T*)dx, (int*)cnt})));
    if (le != cudaSuccess) return CCC_ERR_CUDA;
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T>
int from_rows_impl(const int64_t* rows, const void* roots, int64_t B, int64_t N, const void* x0, const void* x1,
                   const void* masses, int64_t F, void* dv, void* dx, int32_t* cnt, void* ws, int64_t ws_bytes,
                   cudaStream_t s) {
    Prepared P;
    int rc = prepare(ws, ws_bytes, B, F, 0, false, s, P);
    if (rc) return rc;
    if (B * N == 0) return CCC_OK;
    int g = (int)std::min<int64_t>(grid_for(B * N, NARROW_THREADS), (int64_t)narrow_grid());
    CCC_WITH_LIB(CCC_LAUNCH("k_impulses_from_rows", s, k_impulses_from_rows<T, LIBV><<<g, NARROW_THREADS, 0, s>>>(
        (const long long*)rows, (const T*)roots, (int)B, N, (int)F, (const T*)x0, (const T*)x1, (const T*)masses,
        (T*)dv, (T*)dx, (int*)cnt, P.hdr)));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

}  // namespace

extern "C" {

int ccc_version(void) { return 1; }

int64_t ccc_kernel_launches(void) { return g_launches; }

int ccc_set_math_library(int lib) {
    if (lib != LIB_REFERENCE && lib != LIB_PORTABLE) return CCC_ERR_INVALID_ARG;
    g_math_lib = lib;
    return CCC_OK;
}

int ccc_get_math_library(void) { return g_math_lib; }

int ccc_debug_stage(int op, int lib, const double* in, int in_stride, double* out, int out_stride, int64_t n,
                    void* stream) {
    if (op < 0 || op > 5 || (lib != LIB_REFERENCE && lib != LIB_PORTABLE) || n < 0 || n >= ((int64_t)1 << 31))
        return CCC_ERR_INVALID_ARG;
    const int need_in[6] = {24, 4, 26, 30, 4, 1}, need_out[6] = {4, 3, 1, 6, 3, 3};
    if (in_stride < need_in[op] || out_stride < need_out[op]) return CCC_ERR_INVALID_ARG;
    if (n == 0) return CCC_OK;
    if (!in || !out) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    CCC_LAUNCH("k_debug_stage", s, e = launch_debug_stage(op, lib, in, in_stride, out, out_stride, (int)n, s));
    return e == cudaSuccess ? CCC_OK : CCC_ERR_CUDA;
}

int ccc_debug_math(int op, const double* in, double* out, int64_t n, void* stream) {
    if (op < 0 || op > 11 || n < 0 || (n > 0 && (!in || !out)) || n >= ((int64_t)1 << 31)) return CCC_ERR_INVALID_ARG;
    if (n == 0) return CCC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    CCC_LAUNCH("k_debug_math", s, e = launch_debug_math(op, in, out, (int)n, s));
    return e == cudaSuccess ? CCC_OK : CCC_ERR_CUDA;
}

int ccc_timing_begin(void) {
    g_timing = true;
    g_ntimed = 0;
    return CCC_OK;
}

int ccc_timing_end(int max_kernels, char* names, int name_len, float* total_ms, int32_t* count) {
    g_timing = false;
    int nk = 0;
    if (g_ntimed > 0 && cudaEventSynchronize(g_timed[g_ntimed - 1].b) != cudaSuccess) return -CCC_ERR_CUDA;
    for (int i = 0; i < g_ntimed; ++i) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, g_timed[i].a, g_timed[i].b) != cudaSuccess) return -CCC_ERR_CUDA;
        int k = 0;
        while (k < nk && strncmp(names + k * name_len, g_timed[i].name, name_len - 1) != 0) ++k;
        if (k == nk) {
            if (nk >= max_kernels) continue;
            strncpy(names + k * name_len, g_timed[i].name, name_len - 1);
            names[k * name_len + name_len - 1] = 0;
            total_ms[k] = 0.f;
            count[k] = 0;
            ++nk;
        }
        total_ms[k] += ms;
        count[k] += 1;
    }
    g_ntimed = 0;
    return nk;
}

const char* ccc_error_string(int code) {
    switch (code) {
        case CCC_OK: return "ok";
        case CCC_ERR_INVALID_ARG: return "invalid argument";
        case CCC_ERR_WORKSPACE: return "workspace too small";
        case CCC_ERR_CUDA: return "CUDA launch error";
        case CCC_ERR_TOO_LARGE: return "problem larger than the fixed scratch of the no-allocation entry point";
        default: return "unknown error";
    }
}

int64_t ccc_workspace_size(int op, int64_t B, int64_t F, int64_t maxc) {
    if (check_common(0, B, F) != CCC_OK) return -1;
    bool nodes = !(op == CCC_OP_BVH);
    int64_t per = nodes ? std::max<int64_t>(maxc, 1) : 0;
    if (nodes && !rows_fit(B, F, per)) return -1;
    return layout(B, F, per, nodes).end;
}

int ccc_read_status(const void* ws, int64_t n_mesh, int32_t* out, void* stream) {
    if (!ws || !out || n_mesh < 0) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const char* base = (const char*)ws;
    if (cudaMemcpyAsync(out, base, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CCC_ERR_CUDA;
    if (n_mesh > 0) {
        Layout L = layout(1, 2, 1, true);   // mesh counter offset does not depend on sizes
        if (cudaMemcpyAsync(out + 2, base + L.mesh_cnt, (size_t)n_mesh * sizeof(int32_t), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess)
            return CCC_ERR_CUDA;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return CCC_ERR_CUDA;
    return CCC_OK;
}

int ccc_read_counters(const void* ws, int32_t* out, void* stream) {
    if (!ws || !out) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemcpyAsync(out, ws, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CCC_ERR_CUDA;
    return CCC_OK;
}

int ccc_bvh(int dtype, const void* triangles, const void* triangles_next, int64_t B, int64_t F, void* bboxes,
            int64_t* tree, void* ws, int64_t ws_bytes, void* stream) {
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (!triangles || !bboxes || !tree) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == 0 ? bvh_impl<float>(triangles, triangles_next, B, F, bboxes, tree, ws, ws_bytes, s)
                      : bvh_impl<double>(triangles, triangles_next, B, F, bboxes, tree, ws, ws_bytes, s);
}

int ccc_find_collisions(int dtype, const void* bboxes, const int64_t* tree, const void* triangles, int64_t B,
                        int64_t F, double threshold, int64_t max_collisions, int64_t* out, void* ws,
                        int64_t ws_bytes, void* stream) {
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (!bboxes || !tree || !triangles || !out || max_collisions < 1) return CCC_ERR_INVALID_ARG;
    if (!rows_fit(B, F, max_collisions)) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == 0 ? static_impl<float>(bboxes, tree, triangles, B, F, threshold, max_collisions, out, ws, ws_bytes, s)
                      : static_impl<double>(bboxes, tree, triangles, B, F, threshold, max_collisions, out, ws, ws_bytes, s);
}

int ccc_find_triangle_edge_collisions(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                      int64_t B, int64_t F, int64_t max_collisions, int64_t* out_rows,
                                      void* out_coefs, void* ws, int64_t ws_bytes, void* stream) {
    return te_entry<TE_COLLISIONS>(dtype, bboxes, tree, triangles, B, F, max_collisions, out_rows, out_coefs, nullptr,
                                   ws, ws_bytes, stream);
}

int ccc_find_triangle_edge_candidates(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                      int64_t B, int64_t F, int64_t max_collisions, int64_t* out_rows, void* ws,
                                      int64_t ws_bytes, void* stream) {
    return te_entry<TE_CANDIDATES>(dtype, bboxes, tree, triangles, B, F, max_collisions, out_rows, nullptr, nullptr,
                                   ws, ws_bytes, stream);
}

int ccc_find_triangle_edge_candidates2(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                       int64_t B, int64_t F, int64_t max_collisions, int64_t* out_pairs,
                                       int32_t* out_binmasks, void* ws, int64_t ws_bytes, void* stream) {
    return te_entry<TE_CANDIDATES2>(dtype, bboxes, tree, triangles, B, F, max_collisions, out_pairs, nullptr,
                                    out_binmasks, ws, ws_bytes, stream);
}

int ccc_find_collisions_continuous(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                   const void* triangles_next, const uint8_t* mask, int64_t B, int64_t F,
                                   int64_t maxc, int64_t maxcol, int64_t* out_rows, void* out_times, void* ws,
                                   int64_t ws_bytes, void* stream) {
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (!bboxes || !tree || !triangles || !triangles_next || !out_rows || !out_times || maxc < 1 || maxcol < 1)
        return CCC_ERR_INVALID_ARG;
    if (!rows_fit(B, F, maxc) || !rows_fit(B, F, maxcol)) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == 0 ? ccd_impl<float>(bboxes, tree, triangles, triangles_next, mask, B, F, maxc, maxcol, out_rows,
                                        out_times, ws, ws_bytes, s)
                      : ccd_impl<double>(bboxes, tree, triangles, triangles_next, mask, B, F, maxc, maxcol, out_rows,
                                         out_times, ws, ws_bytes, s);
}

int ccc_find_mincol_cand(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                         const void* triangles_next, int64_t B, int64_t F, int64_t max_collisions, int64_t* out_rows,
                         void* ws, int64_t ws_bytes, void* stream) {
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (!bboxes || !tree || !triangles || !triangles_next || !out_rows || max_collisions < 1) return CCC_ERR_INVALID_ARG;
    if (!rows_fit(B, F, max_collisions, 15)) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == 0 ? mincol_impl<float>(bboxes, tree, triangles, triangles_next, B, F, max_collisions, out_rows, ws,
                                           ws_bytes, s)
                      : mincol_impl<double>(bboxes, tree, triangles, triangles_next, B, F, max_collisions, out_rows, ws,
                                            ws_bytes, s);
}

int ccc_find_proximity(int dtype, const void* bboxes, const int64_t* tree, const void* triangles, int64_t B,
                       int64_t F, double threshold, int64_t maxc, int64_t* out_rows, void* ws, int64_t ws_bytes,
                       void* stream) {
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (!bboxes || !tree || !triangles || !out_rows || maxc < 1) return CCC_ERR_INVALID_ARG;
    if (!rows_fit(B, F, maxc)) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == 0 ? prox_impl<float>(bboxes, tree, triangles, B, F, threshold, maxc, out_rows, ws, ws_bytes, s)
                      : prox_impl<double>(bboxes, tree, triangles, B, F, threshold, maxc, out_rows, ws, ws_bytes, s);
}

int ccc_compute_impulses(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                         const void* triangles_next, const void* masses, const uint8_t* mask, int64_t B, int64_t F,
                         int64_t maxc, int64_t maxcol, void* dv, void* dx, int32_t* counter, void* ws,
                         int64_t ws_bytes, void* stream) {
    (void)maxcol;   // the reference does not cap the contacts that feed the impulses
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (!bboxes || !tree || !triangles || !triangles_next || !masses || !dv || !dx || !counter || maxc < 1)
        return CCC_ERR_INVALID_ARG;
    if (!rows_fit(B, F, maxc)) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == 0 ? impulses_impl<float>(bboxes, tree, triangles, triangles_next, masses, mask, B, F, maxc, dv, dx,
                                             counter, ws, ws_bytes, s)
                      : impulses_impl<double>(bboxes, tree, triangles, triangles_next, masses, mask, B, F, maxc, dv, dx,
                                              counter, ws, ws_bytes, s);
}

int ccc_compute_impulses_from_collisions(int dtype, const int64_t* collisions, const void* roots, int64_t B,
                                         int64_t N, const void* triangles, const void* triangles_next,
                                         const void* masses, int64_t F, void* dv, void* dx, int32_t* counter,
                                         void* ws, int64_t ws_bytes, void* stream) {
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (N < 0 || (N > 0 && (!collisions || !roots)) || !triangles || !triangles_next || !masses || !dv || !dx ||
        !counter)
        return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == 0 ? from_rows_impl<float>(collisions, roots, B, N, triangles, triangles_next, masses, F, dv, dx,
                                              counter, ws, ws_bytes, s)
                      : from_rows_impl<double>(collisions, roots, B, N, triangles, triangles_next, masses, F, dv, dx,
                                               counter, ws, ws_bytes, s);
}

// ---------------------------------------------------------------------------------------
// Continuous collisions without any caller-provided or library-allocated scratch.
//
// Some callers cannot allocate device memory at all: plugins running inside a host
// framework that owns every byte of the GPU through its own pool, or real-time step loops
// whose policy forbids allocations after start-up.  For them the scratch of
// ccc_find_collisions_continuous lives in a fixed file-scope device array of
// CCC_STATIC_SCRATCH_BYTES, which every GPU that loads this library holds until the
// process exits.  The array's name is only a host-side stand-in in host code, so its
// device address is looked up with cudaGetSymbolAddress, with the calling device current,
// on every call: after a cudaDeviceReset (or in another context) the module's data is
// loaded again at a different address, so a cached address could point at someone else's
// memory.  The first call on a device also loads the module's data there, so it should
// come before any stream capture.  Every call shares the array: calls whose work overlaps
// on the GPU (different streams or threads without ordering) race on it.  Each call clears
// the parts that must start at zero; the rest is fully rewritten before it is read.

#define CCC_STATIC_SCRATCH_BYTES (64ll << 20)

static __device__ __align__(256) unsigned char g_ccc_static_scratch[CCC_STATIC_SCRATCH_BYTES];

// device address of the array on the current device (nullptr on a CUDA error)
static void* static_scratch_base() {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_ccc_static_scratch) != cudaSuccess) return nullptr;
    return p;
}

int64_t ccc_static_scratch_bytes(void) { return CCC_STATIC_SCRATCH_BYTES; }

int ccc_find_collisions_continuous_static(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                          const void* triangles_next, const uint8_t* mask, int64_t B, int64_t F,
                                          int64_t maxc, int64_t maxcol, int64_t* out_rows, void* out_times,
                                          void* stream) {
    int rc = check_common(dtype, B, F);
    if (rc) return rc;
    if (!rows_fit(B, F, maxc) || !rows_fit(B, F, maxcol)) return CCC_ERR_INVALID_ARG;
    int64_t need = layout(B, F, maxc, true).end;
    if (need > CCC_STATIC_SCRATCH_BYTES) return CCC_ERR_TOO_LARGE;
    void* base = static_scratch_base();
    if (base == nullptr) return CCC_ERR_CUDA;
    return ccc_find_collisions_continuous(dtype, bboxes, tree, triangles, triangles_next, mask, B, F, maxc, maxcol,
                                          out_rows, out_times, base, CCC_STATIC_SCRATCH_BYTES, stream);
}

int ccc_static_scratch_read_status(int64_t n_mesh, int32_t* out, void* stream) {
    void* base = static_scratch_base();
    if (base == nullptr) return CCC_ERR_CUDA;
    return ccc_read_status(base, n_mesh, out, stream);
}

int ccc_static_scratch_read_counters(int32_t* out, void* stream) {
    void* base = static_scratch_base();
    if (base == nullptr) return CCC_ERR_CUDA;
    return ccc_read_counters(base, out, stream);
}

}  // extern "C"
