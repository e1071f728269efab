// ccc_engine.cu — host side of the resident multi-mesh engine (include/ccc_engine.h).
//
// Slot bookkeeping (first-fit ranges of the triangle and vertex arenas), the device mesh
// tables, and the launch sequences of the build, collision and impulse-loop steps.  Every
// step kernel is a grid-stride loop of a fixed grid that reads its sizes from the device
// mesh table, so a sequence captured as a CUDA graph stays valid when the active set
// changes.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/ccc_b200.h"
#include "../../include/ccc_engine.h"
#include "ccc_engine.cuh"
#include "ccc_runtime.cuh"

using namespace ccc;

namespace {

constexpr int TAB_HDR = 4;
constexpr int ITEM_THREADS = 256;

int64_t tab_words(int64_t mc) { return TAB_HDR + (mc + 1) + mc + mc + (mc + 1) + mc; }

struct Tables {
    Forest f;
    VertTable vt;
};

Tables tables_at(const int* tab, int64_t mc) {
    Tables t;
    t.f.nm = tab;
    t.f.voff = tab + TAB_HDR;
    t.f.poff = t.f.voff + mc + 1;
    t.f.sid = t.f.poff + mc;
    t.vt.vvoff = t.f.sid + mc;
    t.vt.vpoff = t.vt.vvoff + mc + 1;
    return t;
}

// Block layout, every section 256-byte aligned.  The state span [hdr, flags] is read back
// in one copy; [hdr, contacts] is cleared before every step.
struct EngineLayout {
    int64_t hdr, mesh_cnt, contacts, iters, flags, state_end;
    int64_t tab, btab, bounds;
    int64_t x0, x1, masses, faces;
    int64_t leaf_tri, lparent, nparent, visits, nodes, qnodes, qcode, qleaf, nrange, front;
    int64_t rows, times, cand;
    int64_t keys0, keys1, vals0, vals1, hist;
    int64_t verts0, verts1, vel, acc;
    int64_t wtab, vidc, wcnt, fan_end, fan, fan_tmp, vid4, twin4, third4, pending, live, end;
    int64_t zero_bytes, hist_len, cand_cap;
};

EngineLayout engine_layout(int64_t tsz, int64_t tc, int64_t vc, int64_t mc, int64_t maxc, int64_t maxcol) {
    EngineLayout L;
    int64_t o = 0;
    auto take = [&](int64_t bytes) {
        int64_t at = o;
        o = align_up(o + bytes, 256);
        return at;
    };
    L.hdr = take(sizeof(WsHeader));
    L.mesh_cnt = take(mc * 4);
    L.contacts = take(mc * 4);
    L.zero_bytes = o;
    L.iters = take(mc * 4);
    L.flags = take(mc * 4);
    L.state_end = o;
    L.tab = take(tab_words(mc) * 4);
    L.btab = take(tab_words(mc) * 4);
    L.bounds = take(mc * 6 * 4);
    L.x0 = take(tc * 9 * tsz);
    L.x1 = take(tc * 9 * tsz);
    L.masses = take(tc * 3 * tsz);
    L.faces = take(tc * 3 * 4);
    L.leaf_tri = take(tc * 4);
    L.lparent = take(tc * 4);
    L.nparent = take(tc * 4);
    L.visits = take(tc * 4);
    L.nodes = take(tc * (int64_t)sizeof(TNode));
    L.qnodes = take(tc * (int64_t)sizeof(QNode));
    L.qcode = take(tc * 4);
    L.qleaf = take(tc * 4);
    L.nrange = take(tc * 8);
    L.front = take(tc * 8);
    L.rows = take(tc * maxcol * 3 * 8);
    L.times = take(tc * maxcol * tsz);
    L.cand_cap = tc * maxc;
    L.cand = take(L.cand_cap * 8);
    L.keys0 = take(tc * 8);
    L.keys1 = take(tc * 8);
    L.vals0 = take(tc * 4);
    L.vals1 = take(tc * 4);
    L.hist_len = 256 * ((tc + SORT_TILE - 1) / SORT_TILE);
    L.hist = take((L.hist_len + 256) * 4);    // tile counts, then the digits' totals
    L.verts0 = take(vc * 3 * tsz);
    L.verts1 = take(vc * 3 * tsz);
    L.vel = take(vc * 3 * tsz);
    L.acc = take(vc * 8 * 8);
    // corner classes (Weld): table (then the classes' first member entries), per-corner-id
    // arrays (4 ids per slot), member list
    L.wtab = take(tc * 6 * 4);
    L.vidc = take(tc * 4 * 4);
    L.wcnt = take(tc * 4 * 4);
    L.fan_end = take(tc * 4 * 4);
    L.fan = take(tc * 3 * 16);
    L.fan_tmp = take(tc * 3 * 16);      // the member list in order of arrival
    L.vid4 = take(tc * 16);
    L.twin4 = take(tc * 16);
    L.third4 = take(tc * 16);
    L.pending = take(L.cand_cap * 16);
    L.live = take(L.cand_cap * 16);
    L.end = o;
    return L;
}

struct MeshRec {
    bool used = false;
    bool built = false;      // tree topology exists for the current slot range
    int64_t F = 0, V = 0, poff = 0, vpoff = 0;
};

// first-fit allocator over [0, capacity)
struct Ranges {
    std::map<int64_t, int64_t> free;   // start -> length
    void init(int64_t cap) {
        free.clear();
        if (cap > 0) free[0] = cap;
    }
    int64_t alloc(int64_t len) {
        if (len == 0) return 0;
        for (auto it = free.begin(); it != free.end(); ++it) {
            if (it->second >= len) {
                int64_t at = it->first, rest = it->second - len;
                free.erase(it);
                if (rest) free[at + len] = rest;
                return at;
            }
        }
        return -1;
    }
    void release(int64_t at, int64_t len) {
        if (len == 0) return;
        auto it = free.emplace(at, len).first;
        auto nx = std::next(it);
        if (nx != free.end() && at + it->second == nx->first) {
            it->second += nx->second;
            free.erase(nx);
        }
        if (it != free.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free.erase(it);
            }
        }
    }
    int64_t largest() const {
        int64_t b = 0;
        for (auto& kv : free) b = std::max(b, kv.second);
        return b;
    }
};

// launch shapes: traversal blocks per SM, narrow-phase blocks per SM (one is resident at
// a time; more blocks split the work finer), the traversal's schedule (0: one query per
// thread, k_traverse_q; 1: 32 queries per warp walking together, k_traverse_w) and, for
// k_traverse_q, the tree levels below the root each block copies into shared memory (0-2),
// and the narrow phase's batch (1: 256 sub-tests, 2: 512)
struct Shape {
    int trav, narrow, warp, stage, batch;
};
constexpr Shape SHAPES[] = {{4, 1, 0, 0, 1},  {8, 1, 0, 0, 1},  {16, 1, 0, 0, 1}, {4, 2, 0, 0, 1},  {8, 2, 0, 0, 1},
                            {16, 2, 0, 0, 1}, {8, 4, 0, 0, 1},  {16, 4, 0, 0, 1}, {32, 8, 0, 0, 1}, {4, 2, 1, 0, 1},
                            {8, 2, 1, 0, 1},  {16, 2, 1, 0, 1}, {32, 2, 1, 0, 1}, {16, 2, 0, 1, 1}, {16, 2, 0, 2, 1},
                            {32, 8, 0, 1, 1}, {32, 8, 0, 2, 1}, {16, 1, 0, 0, 2}, {16, 2, 0, 0, 2}, {32, 4, 0, 0, 2},
                            {32, 8, 0, 0, 2}};
constexpr int NSHAPES = sizeof(SHAPES) / sizeof(SHAPES[0]);
constexpr int DEFAULT_SHAPE = 4;

std::mutex g_tune_mu;
std::map<std::pair<int, int>, int> g_tune_cache;    // (dtype, log2 of active triangles) -> shape

}  // namespace

struct ccc_engine {
    int dtype = 1;
    int64_t tsz = 8, tri_cap = 0, vert_cap = 0, mesh_cap = 0, maxc = 16, maxcol = 16;
    char* base = nullptr;
    EngineLayout L;
    std::vector<MeshRec> mesh;
    Ranges tri_free, vert_free;
    int64_t active_tris = 0;
    std::vector<int32_t> active_ids;
    int* h_stage = nullptr;      // pinned staging of the two tables
    char* h_state = nullptr;     // pinned copy of the state span
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    // second stream of a collision step: the corner classes are rebuilt on it while the
    // refit runs on the caller's stream (fork and join through the two events)
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int64_t graph_kernels[2] = {0, 0};
    int graph_max_iter = 0;
    int shape = DEFAULT_SHAPE;

    template <class P> P* at(int64_t off) const { return reinterpret_cast<P*>(base + off); }
    Tables active() const { return tables_at(at<int>(L.tab), mesh_cap); }
    Tables building() const { return tables_at(at<int>(L.btab), mesh_cap); }
    WsHeader* hdr() const { return at<WsHeader>(L.hdr); }
};

namespace {

inline int item_grid() { return num_sms() * 8; }

// Fill a table (which = 0 active, 1 build) for the given slot ids, ordered by triangle slot,
// and upload it.  Returns the triangle count through ntri.
int upload_table(ccc_engine* e, int which, const int32_t* ids, int64_t n, cudaStream_t s, int64_t* ntri) {
    if (n < 0 || n > e->mesh_cap || (n > 0 && !ids)) return CCC_ERR_INVALID_ARG;
    std::vector<int32_t> v(ids, ids + n);
    std::vector<char> seen(e->mesh_cap, 0);
    for (int32_t id : v) {
        if (id < 0 || id >= e->mesh_cap || !e->mesh[id].used || seen[id]) return CCC_ERR_INVALID_ARG;
        seen[id] = 1;
    }
    std::sort(v.begin(), v.end(), [&](int32_t a, int32_t b) { return e->mesh[a].poff < e->mesh[b].poff; });
    int64_t words = tab_words(e->mesh_cap);
    int* h = e->h_stage + which * words;
    if (cudaEventSynchronize(e->stage_ev[which]) != cudaSuccess) return CCC_ERR_CUDA;
    int64_t mc = e->mesh_cap;
    int* voff = h + TAB_HDR;
    int* poff = voff + mc + 1;
    int* sid = poff + mc;
    int* vvoff = sid + mc;
    int* vpoff = vvoff + mc + 1;
    h[0] = (int)n;
    int64_t t = 0, vv = 0;
    for (int64_t i = 0; i < n; ++i) {
        const MeshRec& r = e->mesh[v[i]];
        voff[i] = (int)t;
        vvoff[i] = (int)vv;
        poff[i] = (int)r.poff;
        vpoff[i] = (int)r.vpoff;
        sid[i] = v[i];
        t += r.F;
        vv += r.V;
    }
    voff[n] = (int)t;
    vvoff[n] = (int)vv;
    if (ntri) *ntri = t;
    int* d = e->at<int>(which ? e->L.btab : e->L.tab);
    if (cudaMemcpyAsync(d, h, words * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return CCC_ERR_CUDA;
    if (cudaEventRecord(e->stage_ev[which], s) != cudaSuccess) return CCC_ERR_CUDA;
    return CCC_OK;
}

// The refit's climbs are chains of dependent L2 round trips, so it runs about one leaf per
// thread (up to 64 blocks per SM) rather than a grid-stride loop over few threads.
inline int refit_grid(const ccc_engine* e) {
    return (int)std::min<int64_t>(grid_for(e->tri_cap, REFIT_THREADS), (int64_t)num_sms() * 64);
}

template <class T> int refit(ccc_engine* e, const Tables& t, const int* flags, cudaStream_t s) {
    if (cudaMemsetAsync(&e->hdr()->front, 0, sizeof(int), s) != cudaSuccess) return CCC_ERR_CUDA;
    CCC_LAUNCH("k_engine_refit", s, k_engine_refit_local<T><<<refit_grid(e), REFIT_THREADS, 0, s>>>(
        t.f, e->at<T>(e->L.x0), e->at<T>(e->L.x1), e->at<int>(e->L.leaf_tri), e->at<int>(e->L.lparent),
        e->at<int>(e->L.nparent), e->at<int>(e->L.qcode), e->at<int>(e->L.qleaf), e->at<int2>(e->L.nrange),
        e->at<TNode>(e->L.nodes), e->at<QNode>(e->L.qnodes), e->at<int2>(e->L.front), (int)e->tri_cap, flags,
        e->hdr()));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_engine_refit_front", s, k_engine_refit_front<<<num_sms() * 8, 256, 0, s>>>(
        t.f, e->at<int>(e->L.nparent), e->at<int>(e->L.qcode), e->at<QNode>(e->L.qnodes),
        e->at<unsigned>(e->L.visits), e->at<int2>(e->L.front), (int)e->tri_cap, e->hdr()));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

// vid: the corner classes of the step (pairs sharing a vertex are not emitted), or null
template <class T> int traverse(ccc_engine* e, const Tables& t, const int* flags, const int4* vid, cudaStream_t s) {
    int g = num_sms() * SHAPES[e->shape].trav;
    if (SHAPES[e->shape].warp)
        CCC_LAUNCH("k_traverse", s, k_traverse_w<<<g, TRAV_THREADS, 0, s>>>(
            e->at<QNode>(e->L.qnodes), e->at<int>(e->L.qleaf), e->at<int>(e->L.leaf_tri), t.f, e->at<int2>(e->L.cand),
            (int)e->L.cand_cap, e->hdr(), flags, vid));
    else if (SHAPES[e->shape].stage == 0)
        CCC_LAUNCH("k_traverse", s, k_traverse_q<0><<<g, TRAV_THREADS, 0, s>>>(
            e->at<QNode>(e->L.qnodes), e->at<int>(e->L.qleaf), e->at<int>(e->L.leaf_tri), t.f, e->at<int2>(e->L.cand),
            (int)e->L.cand_cap, e->hdr(), flags, vid));
    else if (SHAPES[e->shape].stage == 1)
        CCC_LAUNCH("k_traverse", s, k_traverse_q<1><<<g, TRAV_THREADS, 0, s>>>(
            e->at<QNode>(e->L.qnodes), e->at<int>(e->L.qleaf), e->at<int>(e->L.leaf_tri), t.f, e->at<int2>(e->L.cand),
            (int)e->L.cand_cap, e->hdr(), flags, vid));
    else
        CCC_LAUNCH("k_traverse", s, k_traverse_q<2><<<g, TRAV_THREADS, 0, s>>>(
            e->at<QNode>(e->L.qnodes), e->at<int>(e->L.qleaf), e->at<int>(e->L.leaf_tri), t.f, e->at<int2>(e->L.cand),
            (int)e->L.cand_cap, e->hdr(), flags, vid));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

// corner classes of the active meshes' current positions (k_weld_*)
template <class T> int weld(ccc_engine* e, const Tables& t, cudaStream_t s) {
    const EngineLayout& L = e->L;
    if (cudaMemsetAsync(e->base + L.wtab, 0xff, e->tri_cap * 6 * 4, s) != cudaSuccess ||
        cudaMemsetAsync(e->base + L.wcnt, 0, e->tri_cap * 4 * 4, s) != cudaSuccess)
        return CCC_ERR_CUDA;
    const T* x0 = e->at<T>(L.x0);
    const T* x1 = e->at<T>(L.x1);
    int* vidc = e->at<int>(L.vidc);
    int* cnt = e->at<int>(L.wcnt);
    int* fan_end = e->at<int>(L.fan_end);
    CCC_LAUNCH("k_weld_insert", s, k_weld_insert<T><<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, x0, x1, e->at<int>(L.wtab), vidc, cnt, e->hdr()));
    CCC_LAUNCH_CHECK();
    // (the table is not read after k_weld_insert: its space holds the classes' first entries)
    int* fan_start = e->at<int>(L.wtab);
    CCC_LAUNCH("k_weld_alloc", s, k_weld_alloc<<<item_grid(), WELD_THREADS, 0, s>>>(
        t.f, vidc, cnt, fan_start, fan_end, e->hdr()));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_weld_fill", s, k_weld_fill<<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, vidc, fan_start, fan_end, e->at<int4>(L.fan_tmp)));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_weld_rank", s, k_weld_rank<<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, vidc, fan_start, cnt, e->at<int4>(L.fan_tmp), e->at<int4>(L.fan)));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_weld_tri", s, k_weld_tri<<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, vidc, cnt, fan_start, e->at<int4>(L.fan), e->at<int4>(L.vid4), e->at<int4>(L.twin4),
        e->at<int4>(L.third4)));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

Weld engine_weld(ccc_engine* e) {
    const EngineLayout& L = e->L;
    // (the records for k_ccd_expand take the pending list's space, free once staging ends)
    return Weld{e->at<int4>(L.vid4), e->at<int4>(L.fan), e->at<int4>(L.twin4), e->at<int4>(L.third4),
                e->at<int4>(L.live), e->at<int4>(L.pending), (int)L.cand_cap};
}

// the sub-tests of every candidate pair, for the narrow phase (k_ccd_stage_*)
template <class T> int stage(ccc_engine* e, cudaStream_t s) {
    CCC_LAUNCH("k_ccd_stage_mask", s, k_ccd_stage_mask<T><<<num_sms() * 3, STAGE_THREADS, 0, s>>>(
        e->at<int2>(e->L.cand), (int)e->L.cand_cap, e->hdr(), e->at<T>(e->L.x0), e->at<T>(e->L.x1), engine_weld(e),
        e->at<int4>(e->L.live), e->at<int4>(e->L.pending)));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_ccd_stage_pending", s, k_ccd_stage_pending<<<num_sms() * 8, STAGE_THREADS, 0, s>>>(
        (int)e->L.cand_cap, e->hdr(), engine_weld(e), e->at<int4>(e->L.pending), e->at<int4>(e->L.live)));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T> int ccd_step(ccc_engine* e, cudaStream_t s) {
    if (cudaMemsetAsync(e->base, 0, e->L.zero_bytes, s) != cudaSuccess) return CCC_ERR_CUDA;
    Tables t = e->active();
    // the corner classes on the side stream, the refit on s (independent); joined before
    // the traversal, which drops pairs by class.  Under per-kernel timing both run on s, so
    // that each kernel is timed alone.
    const bool fork = !timing_active();
    if (fork && (cudaEventRecord(e->fork_ev, s) != cudaSuccess ||
                 cudaStreamWaitEvent(e->side, e->fork_ev, 0) != cudaSuccess))
        return CCC_ERR_CUDA;
    int rc = weld<T>(e, t, fork ? e->side : s);
    if (rc) return rc;
    rc = refit<T>(e, t, nullptr, s);
    if (rc) return rc;
    if (fork && (cudaEventRecord(e->join_ev, e->side) != cudaSuccess ||
                 cudaStreamWaitEvent(s, e->join_ev, 0) != cudaSuccess))
        return CCC_ERR_CUDA;
    rc = traverse<T>(e, t, nullptr, e->at<int4>(e->L.vid4), s);
    if (rc) return rc;
    rc = stage<T>(e, s);
    if (rc) return rc;
    int g = num_sms() * ccd_min_blocks(SRC_STAGED, SHAPES[e->shape].batch) * SHAPES[e->shape].narrow;
    cudaError_t le = cudaSuccess;
    if (SHAPES[e->shape].batch == 2)
        CCC_WITH_LIB(CCC_LAUNCH("k_ccd_narrow", s, le = launch_ccd_narrow<T, CCD_ROWS, CornerSink<T>, LIBV, SRC_STAGED, 2>(
            g, s, e->at<int2>(e->L.cand), (int)e->L.cand_cap, e->hdr(), e->at<T>(e->L.x0), e->at<T>(e->L.x1), t.f,
            e->at<long long>(e->L.rows), e->at<T>(e->L.times), (int)e->maxcol, e->at<int>(e->L.mesh_cnt),
            engine_weld(e), CornerSink<T>{})));
    else
        CCC_WITH_LIB(CCC_LAUNCH("k_ccd_narrow", s, le = launch_ccd_narrow<T, CCD_ROWS, CornerSink<T>, LIBV, SRC_STAGED>(
            g, s, e->at<int2>(e->L.cand), (int)e->L.cand_cap, e->hdr(), e->at<T>(e->L.x0), e->at<T>(e->L.x1), t.f,
            e->at<long long>(e->L.rows), e->at<T>(e->L.times), (int)e->maxcol, e->at<int>(e->L.mesh_cnt),
            engine_weld(e), CornerSink<T>{})));
    if (le != cudaSuccess) return CCC_ERR_CUDA;
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_ccd_expand", s, k_ccd_expand<T><<<num_sms() * 8, EXPAND_THREADS, 0, s>>>(
        e->hdr(), engine_weld(e), t.f, e->at<long long>(e->L.rows), e->at<T>(e->L.times), (int)e->maxcol,
        e->at<int>(e->L.mesh_cnt)));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

template <class T> int loop_step(ccc_engine* e, int max_iter, cudaStream_t s) {
    if (cudaMemsetAsync(e->base, 0, e->L.zero_bytes, s) != cudaSuccess) return CCC_ERR_CUDA;
    Tables t = e->active();
    int* flags = e->at<int>(e->L.flags);
    int* contacts = e->at<int>(e->L.contacts);
    // (repeated sub-tests are not shared here: a loop iteration's narrow phase is mostly
    // contacts, which every pair computes with its own masses, and the class rebuild and
    // staging cost more than the solves they save)
    int rc = refit<T>(e, t, flags, s);
    if (rc) return rc;
    rc = traverse<T>(e, t, flags, nullptr, s);
    if (rc) return rc;
    int g = num_sms() * CCD_MIN_BLOCKS * SHAPES[e->shape].narrow;
    const Weld W{};
    LoopSink<T> sink{e->at<T>(e->L.masses), e->at<int>(e->L.faces), t.vt, e->at<long long>(e->L.acc), contacts};
    cudaError_t le = cudaSuccess;
    CCC_WITH_LIB(CCC_LAUNCH("k_ccd_narrow", s, le = launch_ccd_narrow<T, CCD_IMPULSES, LoopSink<T>, LIBV, SRC_EXACT>(
        g, s, e->at<int2>(e->L.cand), (int)e->L.cand_cap, e->hdr(), e->at<T>(e->L.x0), e->at<T>(e->L.x1), t.f,
        nullptr, nullptr, 0, e->at<int>(e->L.mesh_cnt), W, sink)));
    if (le != cudaSuccess) return CCC_ERR_CUDA;
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_loop_update", s, k_loop_update<<<grid_for(e->mesh_cap, ITEM_THREADS), ITEM_THREADS, 0, s>>>(
        t.f, contacts, e->at<int>(e->L.iters), flags, max_iter));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_loop_apply", s, k_loop_apply<T><<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, t.vt, contacts, e->at<long long>(e->L.acc), e->at<T>(e->L.verts1), e->at<T>(e->L.vel)));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_gather_soup", s, k_gather_soup<T><<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, t.vt, contacts, e->at<int>(e->L.faces), e->at<T>(e->L.verts1), e->at<T>(e->L.x1), &e->hdr()->status));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

// tree topology of the build table's meshes (ntri triangles in nb meshes), then a refit
template <class T> int build_trees(ccc_engine* e, int64_t ntri, int64_t nb, cudaStream_t s) {
    if (ntri == 0) return CCC_OK;
    Tables t = e->building();
    unsigned* bounds = e->at<unsigned>(e->L.bounds);
    CCC_LAUNCH("k_reset_bounds", s, k_reset_bounds<<<grid_for(e->mesh_cap, ITEM_THREADS), ITEM_THREADS, 0, s>>>(t.f, bounds));
    CCC_LAUNCH_CHECK();
    unsigned long long* keys[2] = {e->at<unsigned long long>(e->L.keys0), e->at<unsigned long long>(e->L.keys1)};
    int* vals[2] = {e->at<int>(e->L.vals0), e->at<int>(e->L.vals1)};
    // the centroids pass from k_mesh_bounds to k_morton in the second key and value buffers
    // (8 + 4 bytes an item), which the sort first writes after k_morton
    float2* cxy = reinterpret_cast<float2*>(keys[1]);
    float* cz = reinterpret_cast<float*>(vals[1]);
    CCC_LAUNCH("k_mesh_bounds", s, k_mesh_bounds<T><<<item_grid(), ITEM_THREADS, 0, s>>>(t.f, e->at<T>(e->L.x0),
                                                                                        e->at<T>(e->L.x1), bounds,
                                                                                        cxy, cz));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_morton", s, k_morton<<<item_grid(), ITEM_THREADS, 0, s>>>(t.f, cxy, cz, bounds, keys[0], vals[0]));
    CCC_LAUNCH_CHECK();
    int mesh_bits = 0;
    while (((int64_t)1 << mesh_bits) < nb) ++mesh_bits;
    int passes = (30 + mesh_bits + 7) / 8;
    int n = (int)ntri;
    int nblk = (int)((ntri + SORT_TILE - 1) / SORT_TILE);
    int* hist = e->at<int>(e->L.hist);
    int cur = 0;
    for (int p = 0; p < passes; ++p) {
        int shift = 8 * p;
        CCC_LAUNCH("k_radix_hist", s, k_radix_hist<<<nblk, SORT_THREADS, 0, s>>>(keys[cur], n, shift, hist, nblk));
        CCC_LAUNCH_CHECK();
        int* rowtot = hist + e->L.hist_len;
        CCC_LAUNCH("k_radix_rowscan", s, k_radix_rowscan<<<256, SORT_THREADS, 0, s>>>(hist, nblk, rowtot));
        CCC_LAUNCH_CHECK();
        CCC_LAUNCH("k_radix_scatter", s, k_radix_scatter<<<nblk, SORT_THREADS, 0, s>>>(keys[cur], vals[cur], keys[1 - cur],
                                                                                   vals[1 - cur], n, shift, hist,
                                                                                   rowtot, nblk));
        CCC_LAUNCH_CHECK();
        cur = 1 - cur;
    }
    CCC_LAUNCH("k_karras_build", s, k_karras_build<<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, keys[cur], vals[cur], e->at<TNode>(e->L.nodes), e->at<int>(e->L.nparent), e->at<int>(e->L.lparent),
        e->at<int>(e->L.leaf_tri), e->at<unsigned>(e->L.visits), e->at<int2>(e->L.nrange), &e->hdr()->status));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_qtree_depth", s, k_qtree_depth<<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, e->at<int>(e->L.nparent), e->at<int>(e->L.qcode), &e->hdr()->status));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_qtree_slots", s, k_qtree_slots<<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, e->at<TNode>(e->L.nodes), e->at<int>(e->L.qcode), e->at<int>(e->L.qleaf), e->at<QNode>(e->L.qnodes),
        &e->hdr()->status));
    CCC_LAUNCH_CHECK();
    return refit<T>(e, t, nullptr, s);
}

template <class T> int loop_prepare(ccc_engine* e, int64_t ntri, int64_t nb, cudaStream_t s) {
    Tables t = e->building();
    CCC_LAUNCH("k_loop_reset", s, k_loop_reset<<<grid_for(e->mesh_cap, ITEM_THREADS), ITEM_THREADS, 0, s>>>(
        t.f, e->at<int>(e->L.iters), e->at<int>(e->L.flags)));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_zero_acc", s, k_zero_acc<<<item_grid(), ITEM_THREADS, 0, s>>>(t.f, t.vt, e->at<long long>(e->L.acc)));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_gather_soup", s, k_gather_soup<T><<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, t.vt, nullptr, e->at<int>(e->L.faces), e->at<T>(e->L.verts0), e->at<T>(e->L.x0), &e->hdr()->status));
    CCC_LAUNCH_CHECK();
    CCC_LAUNCH("k_gather_soup", s, k_gather_soup<T><<<item_grid(), ITEM_THREADS, 0, s>>>(
        t.f, t.vt, nullptr, e->at<int>(e->L.faces), e->at<T>(e->L.verts1), e->at<T>(e->L.x1), &e->hdr()->status));
    CCC_LAUNCH_CHECK();
    return build_trees<T>(e, ntri, nb, s);
}

// steps need the trees of every active mesh
bool active_built(const ccc_engine* e) {
    for (int32_t id : e->active_ids)
        if (!e->mesh[id].used || !e->mesh[id].built) return false;
    return true;
}

// shared-memory attributes of the narrow-phase kernels an engine launches, set before any
// stream capture
template <class T> bool prepare_kernels() {
    return prepare_ccd_narrow<T, CCD_ROWS, CornerSink<T>, LIB_REFERENCE, SRC_STAGED>() == cudaSuccess &&
           prepare_ccd_narrow<T, CCD_ROWS, CornerSink<T>, LIB_PORTABLE, SRC_STAGED>() == cudaSuccess &&
           prepare_ccd_narrow<T, CCD_IMPULSES, LoopSink<T>, LIB_REFERENCE, SRC_EXACT>() == cudaSuccess &&
           prepare_ccd_narrow<T, CCD_IMPULSES, LoopSink<T>, LIB_PORTABLE, SRC_EXACT>() == cudaSuccess &&
           prepare_ccd_narrow<T, CCD_ROWS, CornerSink<T>, LIB_REFERENCE, SRC_STAGED, 2>() == cudaSuccess &&
           prepare_ccd_narrow<T, CCD_ROWS, CornerSink<T>, LIB_PORTABLE, SRC_STAGED, 2>() == cudaSuccess;
}

int run_op(ccc_engine* e, int op, int max_iter, cudaStream_t s) {
    if (!active_built(e)) return CCC_ERR_INVALID_ARG;
    if (op == CCC_ENGINE_OP_CCD) return e->dtype ? ccd_step<double>(e, s) : ccd_step<float>(e, s);
    if (op == CCC_ENGINE_OP_LOOP_STEP)
        return e->dtype ? loop_step<double>(e, max_iter, s) : loop_step<float>(e, max_iter, s);
    return CCC_ERR_INVALID_ARG;
}

int ilog2(int64_t x) {
    int b = 0;
    while (x > 1) {
        x >>= 1;
        ++b;
    }
    return b;
}

}  // namespace

extern "C" {

int64_t ccc_engine_bytes(int dtype, int64_t tc, int64_t vc, int64_t mc, int64_t maxc, int64_t maxcol) {
    if ((dtype != 0 && dtype != 1) || tc < 2 || vc < 0 || mc < 1 || maxc < 1 || maxcol < 1) return -1;
    if (tc >= ((int64_t)1 << 28) || vc >= ((int64_t)1 << 28) || mc >= ((int64_t)1 << 24)) return -1;
    if (tc * maxc >= ((int64_t)1 << 31)) return -1;
    return engine_layout(dtype ? 8 : 4, tc, vc, mc, maxc, maxcol).end;
}

int ccc_engine_create(int dtype, int64_t tc, int64_t vc, int64_t mc, int64_t maxc, int64_t maxcol, void* block,
                      int64_t block_bytes, void* stream, ccc_engine** out) {
    if (!out) return CCC_ERR_INVALID_ARG;
    *out = nullptr;
    int64_t need = ccc_engine_bytes(dtype, tc, vc, mc, maxc, maxcol);
    if (need < 0) return CCC_ERR_INVALID_ARG;
    if (!block || ((uintptr_t)block & 255) || block_bytes < need) return CCC_ERR_WORKSPACE;
    ccc_engine* e = new ccc_engine();
    e->dtype = dtype;
    e->tsz = dtype ? 8 : 4;
    e->tri_cap = tc;
    e->vert_cap = vc;
    e->mesh_cap = mc;
    e->maxc = maxc;
    e->maxcol = maxcol;
    e->base = (char*)block;
    e->L = engine_layout(e->tsz, tc, vc, mc, maxc, maxcol);
    e->mesh.assign(mc, MeshRec());
    e->tri_free.init(tc);
    e->vert_free.init(vc);
    cudaStream_t s = (cudaStream_t)stream;
    int64_t words = tab_words(mc);
    bool ok = cudaHostAlloc((void**)&e->h_stage, 2 * words * 4, cudaHostAllocDefault) == cudaSuccess &&
              cudaHostAlloc((void**)&e->h_state, e->L.state_end, cudaHostAllocDefault) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->stage_ev[0], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->stage_ev[1], cudaEventDisableTiming) == cudaSuccess &&
              cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->fork_ev, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->join_ev, cudaEventDisableTiming) == cudaSuccess;
    if (ok) ok = dtype ? prepare_kernels<double>() : prepare_kernels<float>();
    if (ok) {
        memset(e->h_stage, 0, 2 * words * 4);
        // state, tables (empty), refit counters, topology and accumulators start cleared
        ok = cudaMemsetAsync(e->base, 0, e->L.bounds, s) == cudaSuccess &&
             cudaMemsetAsync(e->base + e->L.visits, 0, tc * 4, s) == cudaSuccess &&
             cudaMemsetAsync(e->base + e->L.acc, 0, vc * 64, s) == cudaSuccess &&
             cudaStreamSynchronize(s) == cudaSuccess;
    }
    if (!ok) {
        ccc_engine_destroy(e);
        return CCC_ERR_CUDA;
    }
    *out = e;
    return CCC_OK;
}

int ccc_engine_destroy(ccc_engine* e) {
    if (!e) return CCC_ERR_INVALID_ARG;
    for (int i = 0; i < 2; ++i) {
        if (e->graph[i]) cudaGraphExecDestroy(e->graph[i]);
        if (e->stage_ev[i]) {
            cudaEventSynchronize(e->stage_ev[i]);
            cudaEventDestroy(e->stage_ev[i]);
        }
    }
    if (e->side) {
        cudaStreamSynchronize(e->side);
        cudaStreamDestroy(e->side);
    }
    if (e->fork_ev) cudaEventDestroy(e->fork_ev);
    if (e->join_ev) cudaEventDestroy(e->join_ev);
    if (e->h_stage) cudaFreeHost(e->h_stage);
    if (e->h_state) cudaFreeHost(e->h_state);
    delete e;
    return CCC_OK;
}

int ccc_engine_add_mesh(ccc_engine* e, int64_t F, int64_t V, int32_t* slot_id) {
    if (!e || !slot_id || F < 2 || V < 0) return CCC_ERR_INVALID_ARG;
    int32_t sid = -1;
    for (int64_t i = 0; i < e->mesh_cap; ++i)
        if (!e->mesh[i].used) {
            sid = (int32_t)i;
            break;
        }
    if (sid < 0) return CCC_ERR_WORKSPACE;
    int64_t p = e->tri_free.alloc(F);
    if (p < 0) return CCC_ERR_WORKSPACE;
    int64_t vp = e->vert_free.alloc(V);
    if (vp < 0) {
        e->tri_free.release(p, F);
        return CCC_ERR_WORKSPACE;
    }
    MeshRec& r = e->mesh[sid];
    r.used = true;
    r.F = F;
    r.V = V;
    r.poff = p;
    r.vpoff = vp;
    *slot_id = sid;
    return CCC_OK;
}

int ccc_engine_remove_mesh(ccc_engine* e, int32_t sid) {
    if (!e || sid < 0 || sid >= e->mesh_cap || !e->mesh[sid].used) return CCC_ERR_INVALID_ARG;
    MeshRec& r = e->mesh[sid];
    e->tri_free.release(r.poff, r.F);
    e->vert_free.release(r.vpoff, r.V);
    r = MeshRec();
    // a removed mesh leaves the active set on the host side; the device table keeps it until
    // the next ccc_engine_set_active, and steps refuse to run until then
    return CCC_OK;
}

int ccc_engine_mesh_view(ccc_engine* e, int32_t sid, ccc_mesh_view* out) {
    if (!e || !out || sid < 0 || sid >= e->mesh_cap || !e->mesh[sid].used) return CCC_ERR_INVALID_ARG;
    const MeshRec& r = e->mesh[sid];
    const EngineLayout& L = e->L;
    out->F = r.F;
    out->V = r.V;
    out->x0 = e->base + L.x0 + r.poff * 9 * e->tsz;
    out->x1 = e->base + L.x1 + r.poff * 9 * e->tsz;
    out->masses = e->base + L.masses + r.poff * 3 * e->tsz;
    out->faces = (int32_t*)(e->base + L.faces + r.poff * 3 * 4);
    out->verts0 = r.V ? e->base + L.verts0 + r.vpoff * 3 * e->tsz : nullptr;
    out->verts1 = r.V ? e->base + L.verts1 + r.vpoff * 3 * e->tsz : nullptr;
    out->vel = r.V ? e->base + L.vel + r.vpoff * 3 * e->tsz : nullptr;
    out->rows = (int64_t*)(e->base + L.rows + r.poff * e->maxcol * 3 * 8);
    out->times = e->base + L.times + r.poff * e->maxcol * e->tsz;
    return CCC_OK;
}

int ccc_engine_free_slots(ccc_engine* e, int64_t* tris, int64_t* verts) {
    if (!e) return CCC_ERR_INVALID_ARG;
    if (tris) *tris = e->tri_free.largest();
    if (verts) *verts = e->vert_free.largest();
    return CCC_OK;
}

int ccc_engine_set_active(ccc_engine* e, const int32_t* ids, int64_t n, void* stream) {
    if (!e) return CCC_ERR_INVALID_ARG;
    int64_t t = 0;
    int rc = upload_table(e, 0, ids, n, (cudaStream_t)stream, &t);
    if (rc == CCC_OK) {
        e->active_tris = t;
        e->active_ids.assign(ids, ids + n);
    }
    return rc;
}

int ccc_engine_build(ccc_engine* e, const int32_t* ids, int64_t n, void* stream) {
    if (!e) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int64_t t = 0;
    int rc = upload_table(e, 1, ids, n, s, &t);
    if (rc) return rc;
    rc = e->dtype ? build_trees<double>(e, t, n, s) : build_trees<float>(e, t, n, s);
    if (rc == CCC_OK)
        for (int64_t i = 0; i < n; ++i) e->mesh[ids[i]].built = true;
    return rc;
}

int ccc_engine_ccd(ccc_engine* e, void* stream) {
    if (!e) return CCC_ERR_INVALID_ARG;
    return run_op(e, CCC_ENGINE_OP_CCD, 0, (cudaStream_t)stream);
}

int ccc_engine_loop_prepare(ccc_engine* e, const int32_t* ids, int64_t n, void* stream) {
    if (!e) return CCC_ERR_INVALID_ARG;
    for (int64_t i = 0; i < n; ++i)
        if (ids && ids[i] >= 0 && ids[i] < e->mesh_cap && e->mesh[ids[i]].used && e->mesh[ids[i]].V == 0)
            return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int64_t t = 0;
    int rc = upload_table(e, 1, ids, n, s, &t);
    if (rc) return rc;
    rc = e->dtype ? loop_prepare<double>(e, t, n, s) : loop_prepare<float>(e, t, n, s);
    if (rc == CCC_OK)
        for (int64_t i = 0; i < n; ++i) e->mesh[ids[i]].built = true;
    return rc;
}

int ccc_engine_loop_step(ccc_engine* e, int32_t max_iter, void* stream) {
    if (!e || max_iter < 1) return CCC_ERR_INVALID_ARG;
    return run_op(e, CCC_ENGINE_OP_LOOP_STEP, max_iter, (cudaStream_t)stream);
}

int ccc_engine_capture(ccc_engine* e, int op, int32_t max_iter, void* stream) {
    if (!e || !stream || (op != CCC_ENGINE_OP_CCD && op != CCC_ENGINE_OP_LOOP_STEP)) return CCC_ERR_INVALID_ARG;
    if (op == CCC_ENGINE_OP_LOOP_STEP && max_iter < 1) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int64_t launches0 = g_launches;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return CCC_ERR_CUDA;
    int rc = run_op(e, op, max_iter, s);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    g_launches = launches0;
    if (rc || ce != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        return rc ? rc : CCC_ERR_CUDA;
    }
    cudaGraphExec_t x = nullptr;
    size_t nn = 0;
    bool ok = cudaGraphInstantiate(&x, g, 0) == cudaSuccess && cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess;
    int64_t kernels = 0;
    if (ok) {
        std::vector<cudaGraphNode_t> nodes(nn);
        ok = cudaGraphGetNodes(g, nodes.data(), &nn) == cudaSuccess;
        for (size_t i = 0; ok && i < nn; ++i) {
            cudaGraphNodeType ty;
            if (cudaGraphNodeGetType(nodes[i], &ty) != cudaSuccess) ok = false;
            else if (ty == cudaGraphNodeTypeKernel) ++kernels;
        }
    }
    cudaGraphDestroy(g);
    if (!ok) {
        if (x) cudaGraphExecDestroy(x);
        return CCC_ERR_CUDA;
    }
    if (e->graph[op]) cudaGraphExecDestroy(e->graph[op]);
    e->graph[op] = x;
    e->graph_kernels[op] = kernels;
    if (op == CCC_ENGINE_OP_LOOP_STEP) e->graph_max_iter = max_iter;
    return CCC_OK;
}

int ccc_engine_replay(ccc_engine* e, int op, void* stream) {
    if (!e || (op != CCC_ENGINE_OP_CCD && op != CCC_ENGINE_OP_LOOP_STEP) || !e->graph[op]) return CCC_ERR_INVALID_ARG;
    if (!active_built(e)) return CCC_ERR_INVALID_ARG;
    if (cudaGraphLaunch(e->graph[op], (cudaStream_t)stream) != cudaSuccess) return CCC_ERR_CUDA;
    g_launches += e->graph_kernels[op];
    return CCC_OK;
}

int ccc_engine_autotune(ccc_engine* e, void* stream, int32_t* choice) {
    if (!e) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    std::pair<int, int> key(e->dtype, ilog2(std::max<int64_t>(e->active_tris, 1)));
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            e->shape = it->second;
            if (choice) *choice = e->shape;
            return CCC_OK;
        }
    }
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return CCC_ERR_CUDA;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return CCC_ERR_CUDA;
    }
    int best = DEFAULT_SHAPE;
    float best_ms = 1e30f;
    int rc = CCC_OK;
    for (int i = 0; i < NSHAPES && rc == CCC_OK; ++i) {
        e->shape = i;
        rc = run_op(e, CCC_ENGINE_OP_CCD, 0, s);      // warm-up
        float tot = 0.f;
        for (int r = 0; r < 2 && rc == CCC_OK; ++r) {
            cudaEventRecord(a, s);
            rc = run_op(e, CCC_ENGINE_OP_CCD, 0, s);
            cudaEventRecord(b, s);
            float ms = 0.f;
            if (rc == CCC_OK && (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess))
                rc = CCC_ERR_CUDA;
            tot += ms;
        }
        if (rc == CCC_OK && tot < best_ms) {
            best_ms = tot;
            best = i;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    e->shape = best;
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = best;
    }
    if (choice) *choice = best;
    return CCC_OK;
}

int ccc_engine_schedule_count(void) { return NSHAPES; }

int ccc_engine_schedule_info(int32_t choice, int32_t* out) {
    if (choice < 0 || choice >= NSHAPES || !out) return CCC_ERR_INVALID_ARG;
    out[0] = SHAPES[choice].trav;
    out[1] = SHAPES[choice].narrow;
    out[2] = SHAPES[choice].warp;
    out[3] = SHAPES[choice].stage;
    out[4] = SHAPES[choice].batch;
    return CCC_OK;
}

int ccc_engine_set_schedule(ccc_engine* e, int32_t choice) {
    if (!e || choice < 0 || choice >= NSHAPES) return CCC_ERR_INVALID_ARG;
    e->shape = choice;
    return CCC_OK;
}

int ccc_engine_pack_rows(ccc_engine* e, int64_t* out_rows, void* out_times, int64_t capacity, int32_t* out_meta,
                         void* stream) {
    if (!e || !out_rows || !out_times || !out_meta || capacity < 0) return CCC_ERR_INVALID_ARG;
    if (e->tri_cap * e->maxcol >= ((int64_t)1 << 31)) return CCC_ERR_INVALID_ARG;   // int32 offsets
    cudaStream_t s = (cudaStream_t)stream;
    Forest F = e->active().f;
    CCC_LAUNCH("k_pack_offsets", s, k_pack_offsets<<<1, PACK_SCAN_THREADS, 0, s>>>(
        F, e->at<int>(e->L.mesh_cnt), (int)e->maxcol, &e->hdr()->status, out_meta));
    CCC_LAUNCH_CHECK();
    if (capacity == 0) return CCC_OK;
    int64_t work = std::min<int64_t>(capacity, e->active_tris * e->maxcol);
    int g = (int)std::max<int64_t>(1, std::min<int64_t>(grid_for(work, 256), (int64_t)num_sms() * 8));
    if (e->dtype)
        CCC_LAUNCH("k_pack_rows", s, k_pack_rows<double><<<g, 256, 0, s>>>(
            F, out_meta, e->at<long long>(e->L.rows), e->at<double>(e->L.times), (int)e->maxcol, (long long*)out_rows,
            (double*)out_times, capacity, &e->hdr()->status));
    else
        CCC_LAUNCH("k_pack_rows", s, k_pack_rows<float><<<g, 256, 0, s>>>(
            F, out_meta, e->at<long long>(e->L.rows), e->at<float>(e->L.times), (int)e->maxcol, (long long*)out_rows,
            (float*)out_times, capacity, &e->hdr()->status));
    CCC_LAUNCH_CHECK();
    return CCC_OK;
}

int ccc_engine_counters(ccc_engine* e, int32_t* out, void* stream) {
    if (!e || !out) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    WsHeader h;
    if (cudaMemcpyAsync(&h, e->base + e->L.hdr, sizeof(WsHeader), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CCC_ERR_CUDA;
    out[0] = h.status;
    out[1] = h.cand_count;
    out[2] = h.subtests;
    out[3] = h.roots;
    out[4] = h.solved;
    out[5] = h.live_count;
    return CCC_OK;
}

int ccc_engine_read_state(ccc_engine* e, const int32_t* ids, int64_t n, int32_t* status, int32_t* rows,
                          int32_t* contacts, int32_t* iterations, int32_t* flags, void* stream) {
    if (!e || n < 0 || (n > 0 && !ids)) return CCC_ERR_INVALID_ARG;
    for (int64_t i = 0; i < n; ++i)
        if (ids[i] < 0 || ids[i] >= e->mesh_cap) return CCC_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemcpyAsync(e->h_state, e->base, e->L.state_end, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CCC_ERR_CUDA;
    const WsHeader* h = (const WsHeader*)(e->h_state + e->L.hdr);
    if (status) *status = h->status;
    const int* mc = (const int*)(e->h_state + e->L.mesh_cnt);
    const int* ct = (const int*)(e->h_state + e->L.contacts);
    const int* it = (const int*)(e->h_state + e->L.iters);
    const int* fl = (const int*)(e->h_state + e->L.flags);
    for (int64_t i = 0; i < n; ++i) {
        if (rows) rows[i] = std::min<int64_t>(mc[ids[i]], e->mesh[ids[i]].F * e->maxcol);
        if (contacts) contacts[i] = ct[ids[i]];
        if (iterations) iterations[i] = it[ids[i]];
        if (flags) flags[i] = fl[ids[i]];
    }
    return CCC_OK;
}

}  // extern "C"
