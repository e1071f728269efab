// ccc_kernels.cuh — sm_100a kernels of the collision pipeline.
//
// Meshes are processed as a "forest": M meshes concatenated, mesh m owning triangles
// [moff[m], moff[m+1]).  The exported tree tensors use the reference layout per mesh
// (src/build_bvh.cu:309-378): rows 0..F-2 internal nodes, rows F-1..2F-2 leaves in sorted
// position order, bboxes row = (min xyz, max xyz), tree row = (parent, left, right, tri id),
// -1 for "none".  Mesh m's rows start at 2*moff[m] - m.
//
// Traversal works on a compact copy of the internal nodes (TNode, 64 B): both child boxes
// rounded outward to fp32 plus child references, so one node visit is four 16-byte loads.
#pragma once

#include <atomic>

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cooperative_groups/scan.h>
#include "ccc_geom.cuh"

namespace cg = cooperative_groups;

namespace ccc {

enum StatusBits {
    ST_CAND_OVERFLOW = 1,     // more candidate pairs than max_candidates_per_triangle * F
    ST_OUT_OVERFLOW = 2,      // more result rows than the output tensor holds
    ST_STACK_OVERFLOW = 4,    // traversal deeper than the 64-entry stack
    ST_MALFORMED_TREE = 8,    // child / parent index out of range or a cycle in the tree
};

// per-mesh state flags of the resident engine's impulse loop
enum MeshFlags {
    MF_DONE = 1,         // the impulse loop has stopped for this mesh
    MF_CONVERGED = 2,    // ... because a collision check found no contact
};

// Workspace header (int32 words) shared by all operations.
struct WsHeader {
    int status;
    int cand_count;
    int subtests;      // continuous sub-tests (pair, type) whose swept sub-boxes overlap
    int roots;         // roots in [0, 1] filtered
    int front;         // engine refit: climbs handed from the block pass to the global pass
    int solved;        // sub-tests solved (fewer than subtests when repeated ones are shared)
    int fan_cursor;    // engine corner classes: member list slots handed out
    int live_count;    // engine staging: pairs with sub-tests to solve (Weld.live)
    int pending_count; // engine staging: pairs left with vertex-face sub-tests to place
    int expand_count;  // engine narrow phase: records for k_ccd_expand (Weld.expand)
    int pad[6];
};

struct __align__(16) TNode {
    float4 a;   // left  lo.x lo.y lo.z hi.x
    float4 b;   // left  hi.y hi.z | right lo.x lo.y
    float4 c;   // right lo.z hi.x hi.y hi.z
    int4 d;     // left ref, right ref, left aux, right aux
};
// ref >= 0: internal node (mesh-local index); ref < 0: leaf at position ~ref.
// aux: internal child -> rightmost leaf position of its subtree; leaf child -> triangle id.

static constexpr int TRAV_THREADS = 128;
static constexpr int STACK_DEPTH = 64;        // STACK_SIZE (flags.h:26-29)
static constexpr int NARROW_THREADS = 128;
// resident blocks per SM of the static and proximity narrow phases
static constexpr int NARROW_MIN_BLOCKS = 4;

// mesh containing element g where base(m) = off[m] - m * shift (shift 0: triangles,
// shift 1: internal nodes); off has M + 1 entries
__device__ __forceinline__ int find_mesh(const int* __restrict__ off, int M, long long g, int shift) {
    int lo = 0, hi = M - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        long long b = (long long)__ldg(off + mid) - (long long)mid * shift;
        if (b <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Mesh table of the traversal and narrow-phase kernels.  Mesh m (0 <= m < *nm) owns the
// work items [voff[m], voff[m+1]) (a dense prefix that assigns threads to meshes) and the
// data slots [poff[m], poff[m] + F_m) of the triangle, node, leaf and per-triangle output
// arrays (ascending and non-overlapping; poff = voff for a packed batch).  sid[m] is the
// mesh's stable slot id, which indexes its per-mesh counters and state.  All four live in
// device memory, so a captured launch sequence serves whatever table is current.
struct Forest {
    const int* nm;
    const int* voff;
    const int* poff;
    const int* sid;
};

__device__ __forceinline__ int forest_size(const Forest& f) { return __ldg(f.nm); }

// mesh owning data slot g (the last m with poff[m] <= g)
__device__ __forceinline__ int forest_slot_mesh(const Forest& f, int M, long long g) {
    return find_mesh(f.poff, M, g, 0);
}

// ---------------------------------------------------------------------------------------
// packed mesh table for the reference API (B meshes of F triangles): nm = B,
// voff[i] = poff[i] = i * F, sid[i] = i
static __global__ void k_uniform_offsets(int* nm, int* voff, int* poff, int* sid, int M, int F) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *nm = M;
    if (i <= M) voff[i] = i * F;
    if (i < M) {
        poff[i] = i * F;
        sid[i] = i;
    }
}

// ---------------------------------------------------------------------------------------
// Build (reference order): leaf boxes, Karras topology, bottom-up box refit.
// The reference's scene box is reduced from AABB() = (-MAX, +MAX) (aabb.cu:25-34,
// build_bvh.cu:243-244), which makes every Morton code 0; with all keys equal the stable
// sort keeps the input order, so leaf position p holds triangle p and the Karras prefix
// delta(i, j) reduces to 32 + clz(i ^ j).

// leaf rows: box of triangle p (swept over t0/t1 for motion), tree row (parent set later,
// -1, -1, p)
template <class T>
__global__ void k_leaf_rows(const T* __restrict__ x0, const T* __restrict__ x1, const int* __restrict__ moff, int M,
                            int total, T* __restrict__ bboxes, long long* __restrict__ tree) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int m = find_mesh(moff, M, g, 0);
    int F = moff[m + 1] - moff[m];
    int p = g - moff[m];
    long long row = 2LL * moff[m] - m + (F - 1) + p;
    Box<T> b = tri_box(load_tri(x0, g));
    if (x1) b = merge(b, tri_box(load_tri(x1, g)));      // MergeTriBoundingBoxes (452-460)
    store_box(bboxes + row * 6, b);
    tree[row * 4 + 1] = -1;
    tree[row * 4 + 2] = -1;
    tree[row * 4 + 3] = p;
}

// delta for all-equal keys and identity ids (LongestCommonPrefix, bvh.cu:65-89)
__device__ __forceinline__ int delta_id(int i, int j, int n) {
    if (j < 0 || j > n - 1) return -1;
    return 32 + __clz(i ^ j);
}

// BuildRadixTree (build_bvh.cu:74-143) for identity order.  The split search is the
// standard Karras one (steps ceil(l/2), ceil(l/4), ..., 1), which reaches the same split
// as the reference's loop.
static __global__ void k_karras_identity(const int* __restrict__ moff, int M, int total_internal, long long* __restrict__ tree) {
    int gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= total_internal) return;
    int m = find_mesh(moff, M, gi, 1);
    int n = moff[m + 1] - moff[m];
    int i = gi - (moff[m] - m);
    long long base = 2LL * moff[m] - m;
    int dnext = delta_id(i, i + 1, n), dlast = delta_id(i, i - 1, n);
    int d = (dnext - dlast >= 0) ? 1 : -1;
    int dmin = delta_id(i, i - d, n);
    int lmax = 2;
    while (delta_id(i, i + lmax * d, n) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta_id(i, i + (l + t) * d, n) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta_id(i, j, n);
    int s = 0;
    for (int div = 2;; div *= 2) {
        int t = (l + div - 1) / div;
        if (delta_id(i, i + (s + t) * d, n) > dnode) s += t;
        if (t <= 1) break;
    }
    int split = i + s * d + min(d, 0);
    long long lc = (min(i, j) == split) ? (long long)(n - 1 + split) : (long long)split;
    long long rc = (max(i, j) == split + 1) ? (long long)(n - 1 + split + 1) : (long long)(split + 1);
    tree[(base + i) * 4 + 1] = lc;
    tree[(base + i) * 4 + 2] = rc;
    tree[(base + i) * 4 + 3] = -1;
    tree[(base + lc) * 4 + 0] = i;
    tree[(base + rc) * 4 + 0] = i;
    if (i == 0) tree[base * 4 + 0] = -1;
}

// CreateHierarchy (build_bvh.cu:145-209): each leaf climbs; the second thread to reach a
// node writes the union of its children's boxes and continues.
template <class T>
__global__ void k_refit(const int* __restrict__ moff, int M, int total, T* bboxes, const long long* __restrict__ tree,
                        int* __restrict__ visits, int* status) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int m = find_mesh(moff, M, g, 0);
    int n = moff[m + 1] - moff[m];
    if (n < 2) return;
    int p = g - moff[m];
    long long base = 2LL * moff[m] - m;
    int* vis = visits + (moff[m] - m);
    long long node = tree[(base + n - 1 + p) * 4 + 0];
    for (int guard = 0; guard < n; ++guard) {
        if (node < 0 || node >= n - 1) { atomicOr(status, ST_MALFORMED_TREE); return; }
        __threadfence();
        if (atomicAdd(vis + node, 1) == 0) return;
        long long lc = tree[(base + node) * 4 + 1], rc = tree[(base + node) * 4 + 2];
        const T* lb = bboxes + (base + lc) * 6;
        const T* rb = bboxes + (base + rc) * 6;
        Box<T> L, R;
        L.lo = mk<T>(__ldcg(lb + 0), __ldcg(lb + 1), __ldcg(lb + 2));
        L.hi = mk<T>(__ldcg(lb + 3), __ldcg(lb + 4), __ldcg(lb + 5));
        R.lo = mk<T>(__ldcg(rb + 0), __ldcg(rb + 1), __ldcg(rb + 2));
        R.hi = mk<T>(__ldcg(rb + 3), __ldcg(rb + 4), __ldcg(rb + 5));
        store_box(bboxes + (base + node) * 6, merge(L, R));
        if (node == 0) return;
        node = tree[(base + node) * 4 + 0];
    }
    atomicOr(status, ST_MALFORMED_TREE);
}

// ---------------------------------------------------------------------------------------
// Import of exported tensors into traversal nodes (build_bvh_from_array_tree 667-705 and
// set_rightmost_nodes 707-743).

template <class T> __device__ __forceinline__ void box_to_f32(const T* p, float lo[3], float hi[3]) {
    if (sizeof(T) == 4) {
        for (int c = 0; c < 3; ++c) { lo[c] = (float)p[c]; hi[c] = (float)p[3 + c]; }
    } else {
        for (int c = 0; c < 3; ++c) {
            lo[c] = __double2float_rd((double)p[c]);
            hi[c] = __double2float_ru((double)p[3 + c]);
        }
    }
}

template <class T>
__global__ void k_import_nodes(const int* __restrict__ moff, int M, int total_internal, const T* __restrict__ bboxes,
                               const long long* __restrict__ tree, TNode* __restrict__ nodes, int* status) {
    int gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= total_internal) return;
    int m = find_mesh(moff, M, gi, 1);
    int n = moff[m + 1] - moff[m];
    int k = gi - (moff[m] - m);
    long long base = 2LL * moff[m] - m;
    long long ch[2] = {tree[(base + k) * 4 + 1], tree[(base + k) * 4 + 2]};
    float lo[2][3], hi[2][3];
    int ref[2], aux[2];
    for (int s = 0; s < 2; ++s) {
        long long c = ch[s];
        if (c <= 0 || c >= 2LL * n - 1) {
            atomicOr(status, ST_MALFORMED_TREE);
            c = 2LL * n - 2;     // keep the record pointing at a valid leaf
        }
        box_to_f32<T>(bboxes + (base + c) * 6, lo[s], hi[s]);
        if (c >= n - 1) {
            ref[s] = ~(int)(c - (n - 1));
            long long id = tree[(base + c) * 4 + 3];
            if (id < 0 || id >= n) {
                atomicOr(status, ST_MALFORMED_TREE);
                id = 0;
            }
            aux[s] = (int)id;
        } else {
            ref[s] = (int)c;
            aux[s] = -1;
        }
    }
    TNode t;
    t.a = make_float4(lo[0][0], lo[0][1], lo[0][2], hi[0][0]);
    t.b = make_float4(hi[0][1], hi[0][2], lo[1][0], lo[1][1]);
    t.c = make_float4(lo[1][2], hi[1][0], hi[1][1], hi[1][2]);
    t.d = make_int4(ref[0], ref[1], aux[0], aux[1]);
    nodes[moff[m] + k] = t;      // mesh m's nodes start at its first triangle slot
}

// rightmost leaf position of every internal subtree, written into the parent's aux slot
static __global__ void k_import_rightmost(const int* __restrict__ moff, int M, int total, const long long* __restrict__ tree,
                                   TNode* nodes, int* __restrict__ visits, int* __restrict__ rmk, int* status) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int m = find_mesh(moff, M, g, 0);
    int n = moff[m + 1] - moff[m];
    if (n < 2) return;
    int p = g - moff[m];
    long long base = 2LL * moff[m] - m;
    int ioff = moff[m] - m;
    TNode* nd = nodes + moff[m];
    long long node = tree[(base + n - 1 + p) * 4 + 0];
    for (int guard = 0; guard < n; ++guard) {
        if (node < 0 || node >= n - 1) { atomicOr(status, ST_MALFORMED_TREE); return; }
        __threadfence();
        if (atomicAdd(visits + ioff + node, 1) == 0) return;
        int4 d = nd[node].d;
        int rl = d.x < 0 ? ~d.x : __ldcg(rmk + ioff + d.x);
        int rr = d.y < 0 ? ~d.y : __ldcg(rmk + ioff + d.y);
        int r = max(rl, rr);
        rmk[ioff + node] = r;
        long long par = tree[(base + node) * 4 + 0];
        if (par >= 0 && par < n - 1) {
            int4 pd = nd[par].d;
            if (pd.x == (int)node) nd[par].d.z = r;
            else nd[par].d.w = r;
        }
        if (node == 0) return;
        node = par;
    }
    atomicOr(status, ST_MALFORMED_TREE);
}

// ---------------------------------------------------------------------------------------
// Traversal (traverseBVH, collisions_static.cu:10-103; traverseBVHPartial,
// collisions_continuous.cu:127-230).  One thread per query leaf, an explicit stack in
// shared memory, fp32 child-box tests with outward rounding, then the exact
// reference-precision leaf test for every fp32 hit.  Emits global triangle indices.

__device__ __forceinline__ float nudge_down(float x) { return nextafterf(x, -INFINITY); }
__device__ __forceinline__ float nudge_up(float x) { return nextafterf(x, INFINITY); }

// Where traversal finds the leaves of mesh m (n triangles) in the reference's exported
// tensors (mesh m's rows start at 2 voff[m] - m): the query's exact box and triangle id, and
// the exact box of a hit leaf, by sorted leaf position.
template <class T> struct TensorLeaves {
    const T* bboxes;
    const long long* tree;
    __device__ __forceinline__ long long row(int m, int vo, int n, int pos) const {
        return 2LL * vo - m + (n - 1) + pos;
    }
    __device__ __forceinline__ Box<T> box(int m, int vo, int po, int n, int pos) const {
        return load_box(bboxes + row(m, vo, n, pos) * 6);
    }
    __device__ __forceinline__ long long id(int m, int vo, int po, int n, int pos) const {
        return tree[row(m, vo, n, pos) * 4 + 3];
    }
};

// Traversal kernels pass candidates through a per-thread buffer of TRAV_BUF pairs and
// reserve TRAV_BUF slots per thread of a coalesced group with one atomic on the shared
// counter, which every SM contends for.
static constexpr int TRAV_BUF = 16;

// the first n buffered pairs of thread tid to cand[base ..]; pairs past the capacity are
// dropped and reported
__device__ __forceinline__ void flush_candidates(int2 (*cbuf)[TRAV_THREADS], int tid, int n, int base,
                                                 int2* __restrict__ cand, int cand_cap, WsHeader* hdr) {
    for (int i = 0; i < n; ++i) {
        const long long slot = (long long)base + i;
        if (base >= 0 && slot < cand_cap) cand[slot] = cbuf[i][tid];
        else atomicOr(&hdr->status, ST_CAND_OVERFLOW);
    }
}

// the remaining buffered pairs of every thread of the calling coalesced group, with one
// atomic for the group (exclusive scan of the counts)
__device__ __forceinline__ void flush_rest(int2 (*cbuf)[TRAV_THREADS], int tid, int n, int2* __restrict__ cand,
                                           int cand_cap, WsHeader* hdr) {
    cg::coalesced_group grp = cg::coalesced_threads();
    int incl = n;
    for (int o = 1; o < (int)grp.size(); o <<= 1) {
        int y = grp.shfl_up(incl, o);
        if ((int)grp.thread_rank() >= o) incl += y;
    }
    int total = grp.shfl(incl, grp.size() - 1);
    int base = 0;
    if (grp.thread_rank() == 0) base = atomicAdd(&hdr->cand_count, total);
    base = grp.shfl(base, 0) + incl - n;
    flush_candidates(cbuf, tid, n, base, cand, cand_cap, hdr);
}

template <class T, bool MASKED, bool EXACT_F32, class Leaves>
__global__ void __launch_bounds__(TRAV_THREADS)
k_traverse(const TNode* __restrict__ nodes, Leaves leaves, Forest F, const uint8_t* __restrict__ mask, T th,
           int2* __restrict__ cand, int cand_cap, WsHeader* hdr, const int* __restrict__ mflags) {
    int stack[STACK_DEPTH];          // per-thread, in local memory (L1): shared memory holds the buffer
    __shared__ int2 cbuf[TRAV_BUF][TRAV_THREADS];
    int nbuf = 0;
    const int tid = threadIdx.x;
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    for (int v = blockIdx.x * blockDim.x + tid; v < total; v += gridDim.x * blockDim.x) {
        int m = find_mesh(F.voff, M, v, 0);
        int vo = __ldg(F.voff + m), po = __ldg(F.poff + m);
        int n = __ldg(F.voff + m + 1) - vo;
        int p = v - vo;
        if (n < 2) continue;
        if (MASKED && !mask[po + p]) continue;
        if (mflags && (__ldg(mflags + __ldg(F.sid + m)) & MF_DONE)) continue;
        const TNode* nd = nodes + po;
        long long qid64 = leaves.id(m, vo, po, n, p);
        if (qid64 < 0 || qid64 >= n) {
            atomicOr(&hdr->status, ST_MALFORMED_TREE);
            continue;
        }
        int qid = (int)qid64;
        // conservative fp32 query box: threshold folded in, rounded outward, nudged one more ulp
        float qlo[3], qhi[3];
        Box<T> q = leaves.box(m, vo, po, n, p);
        {
            T lo[3] = {q.lo.x, q.lo.y, q.lo.z}, hi[3] = {q.hi.x, q.hi.y, q.hi.z};
            for (int c = 0; c < 3; ++c) {
                if (EXACT_F32) {
                    qlo[c] = (float)lo[c];
                    qhi[c] = (float)hi[c];
                } else {
                    qlo[c] = nudge_down(__double2float_rd((double)lo[c] - (double)th));
                    qhi[c] = nudge_up(__double2float_ru((double)hi[c] + (double)th));
                }
            }
        }
        int sp = 0;
        int node = 0;
        const int limit = 4 * n + 64;
        for (int it = 0;; ++it) {
            if (it > limit) { atomicOr(&hdr->status, ST_MALFORMED_TREE); break; }
            const float4* np = reinterpret_cast<const float4*>(nd + node);
            float4 A = __ldg(np + 0), B = __ldg(np + 1), C = __ldg(np + 2);
            int4 D = __ldg(reinterpret_cast<const int4*>(np + 3));
            // child references inside this mesh: internal < n - 1, leaf position < n
            if (D.x >= n - 1 || D.y >= n - 1 || ~D.x >= n || ~D.y >= n) {
                atomicOr(&hdr->status, ST_MALFORMED_TREE);
                break;
            }
            bool ol = (qlo[0] <= A.w) && (qhi[0] >= A.x) && (qlo[1] <= B.x) && (qhi[1] >= A.y) && (qlo[2] <= B.y) &&
                      (qhi[2] >= A.z);
            bool orr = (qlo[0] <= C.y) && (qhi[0] >= B.z) && (qlo[1] <= C.z) && (qhi[1] >= B.w) && (qlo[2] <= C.w) &&
                       (qhi[2] >= C.x);
            if (!MASKED) {
                int rml = D.x < 0 ? ~D.x : D.z;
                int rmr = D.y < 0 ? ~D.y : D.w;
                if (p >= rml) ol = false;
                if (p >= rmr) orr = false;
            }
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                int ref = s ? D.y : D.x;
                bool hit = (s ? orr : ol) && ref < 0;
                if (hit) {
                    int cpos = ~ref;
                    int cid = s ? D.w : D.z;
                    if (MASKED && mask[po + cid] && !(qid < cid)) hit = false;
                    if (hit && !EXACT_F32) hit = overlap(q, leaves.box(m, vo, po, n, cpos), th);
                    if (hit) {
                        cbuf[nbuf++][tid] = make_int2(po + min(qid, cid), po + max(qid, cid));
                        if (nbuf == TRAV_BUF) {
                            cg::coalesced_group grp = cg::coalesced_threads();
                            int base = 0;
                            if (grp.thread_rank() == 0) base = atomicAdd(&hdr->cand_count, TRAV_BUF * (int)grp.size());
                            base = grp.shfl(base, 0) + TRAV_BUF * (int)grp.thread_rank();
                            flush_candidates(cbuf, tid, TRAV_BUF, base, cand, cand_cap, hdr);
                            nbuf = 0;
                        }
                    }
                }
            }
            bool tl = ol && D.x >= 0, tr = orr && D.y >= 0;
            if (!tl && !tr) {
                if (sp == 0) break;
                node = stack[--sp];
            } else {
                node = tl ? D.x : D.y;
                if (tl && tr) {
                    if (sp >= STACK_DEPTH) { atomicOr(&hdr->status, ST_STACK_OVERFLOW); break; }
                    stack[sp++] = D.y;
                }
            }
        }
    }
    if (nbuf > 0) flush_rest(cbuf, tid, nbuf, cand, cand_cap, hdr);
}

// ---------------------------------------------------------------------------------------
// Narrow phases.  Grid-stride over the candidate buffer; the count is read on the device.

// Output region of the mesh that owns data slot g: rows [poff[m] * per_tri, ... + F_m * per_tri)
struct OutRegion {
    int m;              // table index
    int po;             // first data slot
    long long cap;      // F_m * per_tri
};
__device__ __forceinline__ OutRegion out_region(const Forest& F, int M, long long g, int per_tri) {
    OutRegion r;
    r.m = forest_slot_mesh(F, M, g);
    r.po = __ldg(F.poff + r.m);
    r.cap = (long long)(__ldg(F.voff + r.m + 1) - __ldg(F.voff + r.m)) * per_tri;
    return r;
}

// per-mesh append of one row; returns the row index within the mesh region or -1 when full
__device__ __forceinline__ long long append_row(int* mesh_counters, const Forest& F, int m, long long cap,
                                                int* status) {
    cg::coalesced_group act = cg::coalesced_threads();
    cg::coalesced_group grp = cg::labeled_partition(act, m);
    int slot = 0;
    if (grp.thread_rank() == 0) slot = atomicAdd(mesh_counters + __ldg(F.sid + m), (int)grp.size());
    slot = grp.shfl(slot, 0) + grp.thread_rank();
    if ((long long)slot >= cap) {
        atomicOr(status, ST_OUT_OVERFLOW);
        return -1;
    }
    return slot;
}

// find_collisions: SAT + shared-vertex count (collisions_static.cu:123-159)
template <class T>
__global__ void __launch_bounds__(NARROW_THREADS)
k_static_narrow(const int2* __restrict__ cand, int cand_cap, WsHeader* hdr, const T* __restrict__ tri, Forest F,
                T th, long long* __restrict__ rows, int max_per_tri, int* __restrict__ mesh_counters) {
    const int M = forest_size(F);
    int n = min(hdr->cand_count, cand_cap);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int2 pr = cand[c];
        Tri<T> a = load_tri(tri, pr.x), b = load_tri(tri, pr.y);
        bool keep = sat(a, b, th) && !(count_shared(a, b) > 0);
        if (keep) {
            OutRegion R = out_region(F, M, pr.x, max_per_tri);
            long long r = append_row(mesh_counters, F, R.m, R.cap, &hdr->status);
            if (r >= 0) {
                long long o = (long long)R.po * max_per_tri + r;
                rows[o * 2 + 0] = pr.x - R.po;
                rows[o * 2 + 1] = pr.y - R.po;
            }
        }
    }
}

// find_triangle_edge_collisions (OP 0), _candidates (OP 1), _candidates2 (OP 2)
// (collisions_static.cu:588-942, icontour.cu:113-281): candidate pairs that intersect
// (separating axes, threshold 0) and share at most one vertex (none for OP 0), then the six
// edge sub-tests of each pair.  OP 0 / 1 append a row (i, j, cid, flag) per listed sub-test
// (OP 0 with the edge coefficient); OP 2 appends one row (i, j) per pair with its masks
// (bit cid set in x when the sub-test is listed, in y when it is a loop node).
enum TeOp { TE_COLLISIONS = 0, TE_CANDIDATES = 1, TE_CANDIDATES2 = 2 };

template <class T, int OP, int LIB>
__global__ void __launch_bounds__(NARROW_THREADS)
k_te_narrow(const int2* __restrict__ cand, int cand_cap, WsHeader* hdr, const T* __restrict__ tri, Forest F,
            long long* __restrict__ rows, T* __restrict__ coefs, int* __restrict__ masks, int max_per_tri,
            int* __restrict__ mesh_counters) {
    const int M = forest_size(F);
    int n = min(hdr->cand_count, cand_cap);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int2 pr = cand[c];
        Tri<T> a = load_tri(tri, pr.x), b = load_tri(tri, pr.y);
        if (!(sat(a, b, (T)0) && !(count_shared(a, b) > (OP == TE_COLLISIONS ? 0 : 1)))) continue;
        OutRegion R = out_region(F, M, pr.x, max_per_tri);
        int mx = 0, my = 0;
        for (int cid = 0; cid < 6; ++cid) {
            Tri<T> face;
            V3<T> p0, p1;
            int e;
            te_edge(a, b, cid, face, p0, p1, e);
            int flag = -1;
            T coef = (T)-1;
            if (OP == TE_COLLISIONS) {
                if (!te_intersect<T, LIB>(face, p0, p1, cid, flag, coef)) continue;
            } else {
                int r = te_candidate(face, p0, p1, cid, e);
                if (!r) continue;
                if (OP == TE_CANDIDATES2) {
                    mx |= 1 << cid;
                    if (r & 2) my |= 1 << cid;
                    continue;
                }
                flag = (r & 2) ? 0 : -1;
            }
            long long r = append_row(mesh_counters, F, R.m, R.cap, &hdr->status);
            if (r >= 0) {
                long long o = (long long)R.po * max_per_tri + r;
                rows[o * 4 + 0] = pr.x - R.po;
                rows[o * 4 + 1] = pr.y - R.po;
                rows[o * 4 + 2] = cid;
                rows[o * 4 + 3] = flag;
                if (OP == TE_COLLISIONS) coefs[o] = coef;
            }
        }
        if (OP == TE_CANDIDATES2) {
            long long r = append_row(mesh_counters, F, R.m, R.cap, &hdr->status);
            if (r >= 0) {
                long long o = (long long)R.po * max_per_tri + r;
                rows[o * 2 + 0] = pr.x - R.po;
                rows[o * 2 + 1] = pr.y - R.po;
                masks[o * 2 + 0] = mx;
                masks[o * 2 + 1] = my;
            }
        }
    }
}

enum CcdMode { CCD_ROWS = 0, CCD_IMPULSES = 1, CCD_MINCOL = 2 };
// where the continuous narrow phase takes its pairs from: the candidate buffer (the
// reference-format operations), the candidate buffer with the pairs' exact leaf boxes
// tested as well (the engine's impulse loop, whose candidates come from fp32 boxes rounded
// outward), or the engine's staged list (shared sub-tests)
enum CcdSource { SRC_CANDIDATES = 0, SRC_EXACT = 1, SRC_STAGED = 2 };

// Receiver of the impulses of CCD_IMPULSES: per-corner sums and counters (F, 3, 3) / (F, 3)
// of the reference's compute_impulses.  Per-corner masses (F, 3) feed the contact.
template <class T> struct CornerSink {
    const T* masses;
    T* dv;
    T* dx;
    int* cnt;
    __device__ __forceinline__ void add(const MTet<T>& tet, long long gi, long long gj, int k, T root,
                                        const Contact<T>& ct, const Forest&, int, int*) const {
        apply_impulse(tet, gi, gj, k, root, ct, dv, dx, cnt);
    }
};

// Continuous narrow phase (collisions_continuous.cu:14-765, collisions_impulses.cu:24-1067),
// block-synchronous.  Blocks of CCD_BLOCK threads loop over chunks of CCD_BLOCK candidate
// pairs.  Every thread runs the shared-vertex test and the 15 swept sub-box tests of its
// pair, and the surviving (pair, type) sub-tests are appended to a ring queue in shared
// memory.  Whenever a full batch of CCD_BATCH sub-tests is queued (and once more at the end
// for the remainder), the block solves it in three phases separated by barriers, so that
// every warp of the block runs the same phase's code at the same time:
//   (1) cubic coefficients and the solver prefix of every sub-test, which classifies it;
//   (2) the roots, with the sub-tests ordered by solver branch;
//   (3) the root filter and the output of every root in [0, 1], edge-edge roots first and
//       vertex-face roots after them, so that a warp runs one of the two filters.
// Sub-tests take different branches and have 0 to 3 roots: solved in arrival order they
// leave most lanes idle, and a kernel whose warps are in different phases needs all of its
// code in the instruction cache at once.  Queued batches are always full, so no phase runs
// with a partly empty round of threads.
#ifndef CCC_CCD_BLOCK
#define CCC_CCD_BLOCK 256
#endif
#ifndef CCC_CCD_MIN_BLOCKS
#define CCC_CCD_MIN_BLOCKS 3
#endif
#ifndef CCC_CCD_BATCH_MULT
#define CCC_CCD_BATCH_MULT 1
#endif
static constexpr int CCD_BLOCK = CCC_CCD_BLOCK;
static constexpr int CCD_MIN_BLOCKS = CCC_CCD_MIN_BLOCKS;      // resident blocks per SM
// the engine's staged kernel with batches of 256 needs no more than 64 registers, so four
// of its blocks fit an SM
static constexpr int CCD_MIN_BLOCKS_STAGED = 4;
constexpr int ccd_min_blocks(int src, int bm) {
    return src == SRC_STAGED && bm == 1 ? CCD_MIN_BLOCKS_STAGED : CCD_MIN_BLOCKS;
}
static constexpr int CCD_BATCH = CCC_CCD_BATCH_MULT * CCD_BLOCK;
static_assert(CCD_BLOCK % 32 == 0 && CCD_BLOCK <= 1024 && 3 * CCD_BATCH <= 65536, "CCD_BLOCK");

constexpr size_t align16(size_t x) { return (x + 15) / 16 * 16; }

// dynamic shared memory of one block (byte offsets) for batches of NB sub-tests
template <class T, int NB = CCD_BATCH> struct CcdLayout {
    static constexpr int QUEUE = NB + 15 * CCD_BLOCK;     // a partial batch plus a chunk's worst case
    static constexpr size_t rec = 0;                                                   // double [6][NB]
    static constexpr size_t root_val = rec + 6 * NB * sizeof(double);                  // T [3 NB]
    static constexpr size_t items = align16(root_val + 3 * NB * sizeof(T));            // int2 [QUEUE]
    static constexpr size_t clist = items + QUEUE * sizeof(int2);                      // u16 [NB]
    static constexpr size_t root_rec = clist + NB * 2;                                 // u16 [3 NB]
    static constexpr size_t rec_cls = root_rec + 3 * NB * 2;                           // u8 [NB]
    static constexpr size_t rec_pos = align16(rec_cls + NB);                           // u16 [NB]
    static constexpr size_t spairs = align16(rec_pos + NB * 2);                        // int2 [BLOCK]
    static constexpr size_t pbuf = spairs + CCD_BLOCK * sizeof(int2);                   // u16 [BLOCK / 32][64]
    static constexpr size_t ints = align16(pbuf + (CCD_BLOCK / 32) * 64 * 2);          // int [64]
    static constexpr size_t bytes = ints + 64 * sizeof(int);
    static_assert(3 * NB <= 65536, "batch indices are 16-bit");
};

// slots of the small int area
// (class counts and root counts come in two sets, used by alternate batches; each set of
// root counts holds the edge-edge and the vertex-face count)
// (the live-pair counter of a chunk also comes in two, used by alternate chunks)
enum CcdInts { CI_WARP = 0, CI_TOTAL = 32, CI_COUNT = 33, CI_ROOTS = 41, CI_LIVE = 45 };

// a queued sub-test: triangle slots i and j, type k in the top bits of j (slots < 2^28),
// bit 28 of i set when the sub-test stands for all its repeats (see Weld)
constexpr int SLOT_MASK = 0x0fffffff;
__device__ __forceinline__ int2 pack_subtest(int i, int j, int k, int shared = 0) {
    return make_int2(i | (shared << 28), j | (k << 28));
}

// Repeated sub-tests (resident engine only).  On a mesh a vertex-face sub-test (v, face B)
// is the sub-test of every pair (A', B) whose triangle A' has a corner at v, and an
// edge-edge sub-test belongs to every pair of triangles carrying the two edges with their
// corners in the same order: the tetrahedra are bit for bit the same, and so are their
// roots, filter decisions and contacts.  The pairs that produce one of them are known from
// the corner classes alone:
//  * the corners of a mesh whose start positions are equal (==, the reference's
//    shared-vertex relation, figures.cu:527-544) form a class; a pair shares a vertex
//    exactly when its triangles have a class in common;
//  * every such pair is live (shares no vertex), is a candidate pair of the reference (a
//    vertex's swept sub-box lies in its triangle's leaf box, the merge of the triangle's
//    boxes at both ends of the step, when x0 + (x1 - x0) == x1 for its coordinates), and
//    has the sub-test's sub-box bit (the boxes of the same points);
//  * for vertex-face types 12..14 (vertex of the first triangle) they are the pairs
//    (A', B) with A' < B over the class's corners, for 9..11 the pairs (A, B') with
//    B' > A; for edge-edge types the pairs over each edge and its twin, the other
//    triangle edge whose corners are the same classes in the same order.
// The smallest of those (slot, slot, type) triples solves the sub-test and emits the rows
// or contacts of all of them; the others drop it.  A class is excluded (CLS_NODEDUP) when
// its corners are not bit-identical at both ends of the step, when x0 + (x1 - x0) != x1 for
// one of its coordinates, or when it has more than WELD_FANCAP corners; an edge with more
// than one twin is excluded too.  A sub-test touching an excluded class or edge is solved
// by each of its pairs, as without the classes.  Every pair finds the same members, so
// each repeat is solved exactly once.  Pairs with a rigid motion have no sub-test with a
// root (ccd_pair_subbox_mask), so it does not matter which of them is the smallest.
constexpr int CLS_MASK = (1 << 30) - 1;
constexpr int CLS_NODEDUP = 1 << 30;
constexpr int TWIN_NONE = -1, TWIN_MANY = -2;
constexpr int WELD_FANCAP = 16;
struct Weld {
    const int4* vid;       // per triangle slot: the class of each corner (its first entry in
                           // fan) | CLS_NODEDUP; in w the three class sizes (bits 5c..5c+4,
                           // sizes above 31 as 31) and whether each edge e has no twin, one
                           // or more (bits 15+2e..16+2e: 0, 1, 2); null: no classes
    const int4* fan;       // the classes' members, class by class in ascending corner id:
                           // (corner id 4 * slot + corner, the classes of its triangle)
    const int4* twin;      // per triangle slot and edge {01, 02, 12}: 4 * slot + edge of its
                           // twin, TWIN_NONE or TWIN_MANY
    const int4* third;     // per triangle slot and edge: the class of the twin's third corner
    const int4* live;      // the pairs with sub-tests to solve (hdr->live_count of them, from
                           // k_ccd_stage_*): slots i, j and the sub-tests it solves (bits
                           // 0..14) with those that stand for their repeats (bits 15..29)
    int4* expand;          // the roots that passed the filter, for k_ccd_expand
                           // (hdr->expand_count, at most expand_cap): slots i | shared << 28,
                           // j | type << 28, the root as a double (low, high words); null:
                           // k_ccd_narrow writes the rows itself
    int expand_cap;
};

__device__ __forceinline__ int int4_at(int4 v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }
__device__ __forceinline__ bool classes_meet(int4 a, int4 b) {
    const int a0 = a.x & CLS_MASK, a1 = a.y & CLS_MASK, a2 = a.z & CLS_MASK;
    const int b0 = b.x & CLS_MASK, b1 = b.y & CLS_MASK, b2 = b.z & CLS_MASK;
    return a0 == b0 || a0 == b1 || a0 == b2 || a1 == b0 || a1 == b1 || a1 == b2 || a2 == b0 || a2 == b1 ||
           a2 == b2;
}
__device__ __forceinline__ int class_size(int4 v, int c) { return (v.w >> (5 * c)) & 31; }
__device__ __forceinline__ int twin_kind(int4 v, int e) { return (v.w >> (15 + 2 * e)) & 3; }

// The edge-edge pairs of sub-test 3e + f of pair (A, B): over the edges' twins ta, tb
// (4 * slot + edge, or TWIN_NONE) whose third corners have classes ha, hb, the pairs
// (a < b) that share no vertex, the pair itself first.
template <class Fn>
__device__ __forceinline__ void weld_ee_members(int A, int B, int e, int f, int4 VA, int4 VB, int ta, int tb, int ha,
                                                int hb, Fn&& fn) {
    // edge {01, 02, 12}[e]: corners e > 1 ? 1 : 0 and e > 0 ? 2 : 1
    const int4 TA = make_int4(int4_at(VA, e > 1), int4_at(VA, e > 0 ? 2 : 1), ha, 0);
    const int4 TB = make_int4(int4_at(VB, f > 1), int4_at(VB, f > 0 ? 2 : 1), hb, 0);
    for (int i = 0; i < 2; ++i) {
        if (i == 1 && ta < 0) break;
        const int a = i ? ta >> 2 : A, sa = i ? ta & 3 : e;
        for (int j = 0; j < 2; ++j) {
            if (j == 1 && tb < 0) break;
            const int b = j ? tb >> 2 : B, sb = j ? tb & 3 : f;
            if (a >= b) continue;
            if ((i | j) && classes_meet(i ? TA : VA, j ? TB : VB)) continue;
            fn(a, b, 3 * sa + sb);
        }
    }
}

// Calls fn(a, b, type) for every pair that has sub-test k of pair (A, B) (A < B, live), the
// pair itself included, and returns true; returns false without a call when the sub-test
// is solved by each of its pairs.  VA, VB: W.vid[A], W.vid[B].
template <class Fn>
__device__ __forceinline__ bool weld_members(const Weld& W, int A, int B, int k, int4 VA, int4 VB, Fn&& fn) {
    if (k >= 9) {
        const bool vf = k >= 12;                 // vertex of A, face of B (else face of A)
        const int4 Vface = vf ? VB : VA;
        const int4 Vvert = vf ? VA : VB;
        const int c = vf ? k - 12 : k - 9;
        const int v = int4_at(Vvert, c);
        // (a class of one corner: the pair is the sub-test's only one)
        if (((v | Vface.x | Vface.y | Vface.z) & CLS_NODEDUP) || class_size(Vvert, c) < 2) return false;
        const int end = v + class_size(Vvert, c);
        for (int i = v; i < end; ++i) {
            const int4 en = __ldg(W.fan + i);
            const int t = en.x >> 2, cc = en.x & 3;
            if (vf ? t >= B : t <= A) continue;
            if (classes_meet(make_int4(en.y, en.z, en.w, 0), Vface)) continue;
            if (vf) fn(t, B, 12 + cc);
            else fn(A, t, 9 + cc);
        }
        return true;
    }
    const int e = k / 3, f = k - 3 * e;
    // (edges without a twin: the pair is the sub-test's only one)
    const int ka = twin_kind(VA, e), kb = twin_kind(VB, f);
    if (ka == 2 || kb == 2 || (ka | kb) == 0) return false;
    if ((int4_at(VA, e > 1) | int4_at(VA, e > 0 ? 2 : 1) | int4_at(VB, f > 1) | int4_at(VB, f > 0 ? 2 : 1)) &
        CLS_NODEDUP)
        return false;
    weld_ee_members(A, B, e, f, VA, VB, ka ? int4_at(__ldg(W.twin + A), e) : TWIN_NONE,
                    kb ? int4_at(__ldg(W.twin + B), f) : TWIN_NONE, ka ? int4_at(__ldg(W.third + A), e) : 0,
                    kb ? int4_at(__ldg(W.third + B), f) : 0, fn);
    return true;
}

// Whether pair (A, B) solves its sub-test k: true when the sub-test is not shared or when
// (A, B, k) is the smallest of its pairs; *shared tells which.  The members of a class are
// in ascending corner id, so a vertex-face scan stops at the first pair that has the
// sub-test.
__device__ __forceinline__ bool weld_solves(const Weld& W, int A, int B, int k, int4 VA, int4 VB, bool* shared) {
    *shared = false;
    if (k >= 9) {
        const bool vf = k >= 12;
        const int4 Vface = vf ? VB : VA;
        const int4 Vvert = vf ? VA : VB;
        const int c = vf ? k - 12 : k - 9;
        const int v = int4_at(Vvert, c);
        if (((v | Vface.x | Vface.y | Vface.z) & CLS_NODEDUP) || class_size(Vvert, c) < 2) return true;
        *shared = true;
        const int end = v + class_size(Vvert, c);
        for (int i = v; i < end; ++i) {
            const int4 en = __ldg(W.fan + i);
            const int t = en.x >> 2, cc = en.x & 3;
            if (vf ? t >= B : t <= A) {
                if (vf) break;             // the remaining corners are on later triangles
                continue;
            }
            if (classes_meet(make_int4(en.y, en.z, en.w, 0), Vface)) continue;
            return vf ? (t == A && cc == c) : (t == B && cc == c);
        }
        return true;    // (not reached: the pair itself has the sub-test)
    }
    int ma = A, mb = B, mk = k;
    const bool sh = weld_members(W, A, B, k, VA, VB, [&](int a, int b, int kk) {
        if (a < ma || (a == ma && (b < mb || (b == mb && kk < mk)))) {
            ma = a;
            mb = b;
            mk = kk;
        }
    });
    *shared = sh;
    return !sh || (ma == A && mb == B && mk == k);
}

// The pairs of sub-test k of pair (A, B) in (ma, mb, mk), at most WELD_FANCAP of them (a
// shared vertex-face sub-test has one per corner of its class, an edge-edge one at most
// four); the pair alone when the sub-test is not shared.  Returns their number.
__device__ __forceinline__ int weld_list(const Weld& W, int A, int B, int k, bool shared, int* ma, int* mb, int* mk) {
    int n = 0;
    if (shared)
        weld_members(W, A, B, k, __ldg(W.vid + A), __ldg(W.vid + B), [&](int a, int b, int kk) {
            if (n < WELD_FANCAP) {
                ma[n] = a;
                mb[n] = b;
                mk[n] = kk;
                ++n;
            }
        });
    if (n == 0) {
        ma[0] = A;
        mb[0] = B;
        mk[0] = k;
        n = 1;
    }
    return n;
}

__device__ __forceinline__ int warp_inclusive_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// Row reservation for the lanes of mask, which call it together: each lane's nm rows in the
// region of its mesh m, with one atomic per mesh among them; returns the lane's first row
// (its prefix of the counts of the lanes in its mesh).  A whole warp in one mesh, the usual
// case, takes plain warp scans.
__device__ __forceinline__ int reserve_rows(int* mesh_counters, const Forest& F, int m, int nm, unsigned mask) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    __syncwarp(mask);
    if (mask == FULL && __all_sync(FULL, m == __shfl_sync(FULL, m, 0))) {
        const int incl = warp_inclusive_scan(nm, lane);
        int base = 0;
        if (lane == 31) base = atomicAdd(mesh_counters + __ldg(F.sid + m), incl);
        return __shfl_sync(FULL, base, 31) + incl - nm;
    }
    cg::coalesced_group g = cg::labeled_partition(cg::coalesced_threads(), m);
    const int before = cg::exclusive_scan(g, nm);
    const int all = cg::reduce(g, nm, cg::plus<int>());
    int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(mesh_counters + __ldg(F.sid + m), all);
    return g.shfl(base, 0) + before;
}

// Staging of the resident engine's candidate pairs for k_ccd_narrow: the list Weld.live of
// the pairs with sub-tests to solve, in two kernels.
//  * k_ccd_stage_mask: pairs whose triangles share a vertex (a corner class in common, the
//    same relation as the reference's coordinate test) are dropped; the others queue per
//    warp in shared memory and are taken 32 at a time, for the sub-box mask with the exact
//    leaf-box test (the engine's candidates come from fp32 boxes rounded outward) and the
//    choice of the pair that solves each sub-test wherever the triangles' own records tell
//    it: every edge-edge sub-test (classes, twins and the twins' third corners) and the
//    vertex-face sub-tests that are not shared.  A pair left with shared vertex-face
//    sub-tests goes to the pending list, the others with work to the live list.
//    hdr->subtests counts the sub-tests of the masks.
//  * k_ccd_stage_pending: the pending pairs' vertex-face sub-tests, spread over the lanes
//    of a warp (a scan of the vertex's class each); then the pairs go to the live list.
// Records: (slot i, slot j, the sub-tests to solve in bits 0..14 with the shared ones in
// bits 15..29, pending vertex-face sub-tests).
static constexpr int STAGE_THREADS = 256;
static constexpr int STAGE_WARPS = STAGE_THREADS / 32;

// the pair that solves edge-edge sub-test k of pair (A, B) from the records of A and B
__device__ __forceinline__ bool weld_ee_solves(int A, int B, int k, int4 VA, int4 VB, int4 TWA, int4 TWB, int4 THA,
                                               int4 THB, bool* shared) {
    const int e = k / 3, f = k - 3 * e;
    const int ka = twin_kind(VA, e), kb = twin_kind(VB, f);
    *shared = false;
    if (ka == 2 || kb == 2 || (ka | kb) == 0) return true;
    if ((int4_at(VA, e > 1) | int4_at(VA, e > 0 ? 2 : 1) | int4_at(VB, f > 1) | int4_at(VB, f > 0 ? 2 : 1)) &
        CLS_NODEDUP)
        return true;
    *shared = true;
    int ma = A, mb = B, mk = k;
    weld_ee_members(A, B, e, f, VA, VB, ka ? int4_at(TWA, e) : TWIN_NONE, kb ? int4_at(TWB, f) : TWIN_NONE,
                    int4_at(THA, e), int4_at(THB, f), [&](int a, int b, int kk) {
                        if (a < ma || (a == ma && (b < mb || (b == mb && kk < mk)))) {
                            ma = a;
                            mb = b;
                            mk = kk;
                        }
                    });
    return ma == A && mb == B && mk == k;
}

// a record to the live list (work, no pending) or the pending list, warp-aggregated
__device__ __forceinline__ void stage_emit(WsHeader* hdr, int4* live, int4* pending, int2 pr, unsigned word,
                                           unsigned pend, bool valid) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const bool to_live = valid && pend == 0u && word != 0u, to_pend = valid && pend != 0u;
    const unsigned ml = __ballot_sync(FULL, to_live), mp = __ballot_sync(FULL, to_pend);
    int bl = 0, bp = 0;
    if (lane == 0 && ml) bl = atomicAdd(&hdr->live_count, __popc(ml));
    if (lane == 0 && mp) bp = atomicAdd(&hdr->pending_count, __popc(mp));
    bl = __shfl_sync(FULL, bl, 0) + __popc(ml & lt);
    bp = __shfl_sync(FULL, bp, 0) + __popc(mp & lt);
    // (at most one record per candidate in either list)
    if (to_live) live[bl] = make_int4(pr.x, pr.y, (int)word, 0);
    if (to_pend) pending[bp] = make_int4(pr.x, pr.y, (int)word, (int)pend);
}

template <class T>
__global__ void __launch_bounds__(STAGE_THREADS, 3)
k_ccd_stage_mask(const int2* __restrict__ cand, int cand_cap, WsHeader* hdr, const T* __restrict__ x0,
                 const T* __restrict__ x1, Weld W, int4* __restrict__ live, int4* __restrict__ pending) {
    __shared__ int2 q_pr[STAGE_WARPS][64];
    __shared__ int4 q_va[STAGE_WARPS][64], q_vb[STAGE_WARPS][64];
    const int n = min(*(volatile int*)&hdr->cand_count, cand_cap);
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int warps = gridDim.x * STAGE_WARPS;
    int masked = 0, qn = 0;             // qn: queued live pairs of this warp (warp-uniform)
    for (int base = (blockIdx.x * STAGE_WARPS + wq) * 32;; base += warps * 32) {
        const bool more = base < n;
        if (!more && qn == 0) break;
        if (more) {
            const int c = base + lane;
            int2 pr = make_int2(0, 0);
            int4 VA = make_int4(0, 0, 0, 0), VB = VA;
            bool lv = false;
            if (c < n) {
                pr = cand[c];
                VA = __ldg(W.vid + pr.x);
                VB = __ldg(W.vid + pr.y);
                lv = !classes_meet(VA, VB);
            }
            const unsigned m = __ballot_sync(FULL, lv);
            if (lv) {
                const int at = qn + __popc(m & lt);
                q_pr[wq][at] = pr;
                q_va[wq][at] = VA;
                q_vb[wq][at] = VB;
            }
            qn += __popc(m);
            __syncwarp();
        }
        while (qn >= 32 || (!more && qn > 0)) {
            const bool valid = lane < qn;
            int2 pr = make_int2(0, 0);
            unsigned word = 0u, pend = 0u;
            if (valid) {
                pr = q_pr[wq][lane];
                const int4 VA = q_va[wq][lane], VB = q_vb[wq][lane];
                const unsigned bits = ccd_pair_subbox_mask<T, true, true>(x0, x1, pr.x, pr.y);
                masked += __popc(bits);
                const unsigned ee = bits & 0x1ffu;
                int4 TWA = make_int4(0, 0, 0, 0), TWB = TWA, THA = TWA, THB = TWA;
                if (ee && ((VA.w | VB.w) >> 15)) {
                    TWA = __ldg(W.twin + pr.x);
                    TWB = __ldg(W.twin + pr.y);
                    THA = __ldg(W.third + pr.x);
                    THB = __ldg(W.third + pr.y);
                }
                for (unsigned b = bits; b; b &= b - 1) {
                    const int k = __ffs(b) - 1;
                    bool sh = false, solve = true;
                    if (k < 9) {
                        solve = weld_ee_solves(pr.x, pr.y, k, VA, VB, TWA, TWB, THA, THB, &sh);
                    } else {
                        const bool vf = k >= 12;
                        const int4 Vface = vf ? VB : VA, Vvert = vf ? VA : VB;
                        const int c = vf ? k - 12 : k - 9;
                        if (!((int4_at(Vvert, c) | Vface.x | Vface.y | Vface.z) & CLS_NODEDUP) &&
                            class_size(Vvert, c) >= 2) {
                            pend |= 1u << k;
                            solve = false;
                        }
                    }
                    if (solve) word |= (1u << k) | (sh ? 1u << (15 + k) : 0u);
                }
            }
            stage_emit(hdr, live, pending, pr, word, pend, valid);
            // the queue's second half moves to the front
            __syncwarp();
            if (lane + 32 < qn) {
                q_pr[wq][lane] = q_pr[wq][lane + 32];
                q_va[wq][lane] = q_va[wq][lane + 32];
                q_vb[wq][lane] = q_vb[wq][lane + 32];
            }
            qn = qn > 32 ? qn - 32 : 0;
            __syncwarp();
        }
    }
    masked = __reduce_add_sync(FULL, masked);
    if (lane == 0 && masked) atomicAdd(&hdr->subtests, masked);
}

static __global__ void __launch_bounds__(STAGE_THREADS, 8)
k_ccd_stage_pending(int cand_cap, WsHeader* hdr, Weld W, const int4* __restrict__ pending, int4* __restrict__ live) {
    // per warp: 32 pending pairs, their classes, pending sub-tests, the prefix of their
    // counts and the sub-tests they solve; the lanes take the sub-tests 32 at a time
    __shared__ int2 s_pr[STAGE_THREADS];
    __shared__ int4 s_va[STAGE_THREADS], s_vb[STAGE_THREADS];
    __shared__ unsigned s_bits[STAGE_THREADS], s_word[STAGE_THREADS];
    __shared__ int s_pre[STAGE_THREADS];
    const int n = min(*(volatile int*)&hdr->pending_count, cand_cap);
    const int tid = threadIdx.x, lane = tid & 31, w0 = tid & ~31;
    const unsigned FULL = 0xffffffffu;
    const int warps = gridDim.x * STAGE_WARPS;
    for (int base = (blockIdx.x * STAGE_WARPS + (tid >> 5)) * 32; base < n; base += warps * 32) {
        const int c = base + lane;
        unsigned pend = 0u, word = 0u;
        int2 pr = make_int2(0, 0);
        if (c < n) {
            const int4 rec = pending[c];
            pr = make_int2(rec.x, rec.y);
            word = (unsigned)rec.z;
            pend = (unsigned)rec.w;
            s_va[tid] = __ldg(W.vid + pr.x);
            s_vb[tid] = __ldg(W.vid + pr.y);
        }
        s_pr[tid] = pr;
        s_bits[tid] = pend;
        s_word[tid] = word;
        const int incl = warp_inclusive_scan(__popc(pend), lane);
        s_pre[tid] = incl;
        const int total = __shfl_sync(FULL, incl, 31);
        __syncwarp();
        for (int r = lane; r < total; r += 32) {
            int lo = 0, hi = 31;                       // the pair: first prefix above r
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (s_pre[w0 + mid] > r) hi = mid;
                else lo = mid + 1;
            }
            const int p = w0 + lo;
            const int k = __fns(s_bits[p], 0, r - (lo ? s_pre[p - 1] : 0) + 1);
            bool sh = false;
            if (weld_solves(W, s_pr[p].x, s_pr[p].y, k, s_va[p], s_vb[p], &sh))
                atomicOr(&s_word[p], (1u << k) | (sh ? 1u << (15 + k) : 0u));
        }
        __syncwarp();
        word = s_word[tid];
        stage_emit(hdr, live, nullptr, pr, word, 0u, c < n);
        __syncwarp();
    }
}

// The continuous narrow phase is compiled in one translation unit only, ccc_narrow.cu, with
// nvcc's default multiply-add contraction as the reference is compiled (CUDA's pow, which the
// solver calls, computes slightly different results on rare arguments under -fmad=false);
// every operation of this library's own in it is contraction-proof (mulrn / addrn / subrn,
// fmaT).  The other units see only the launcher's declaration; ccc_narrow.cu instantiates
// the (type, mode, sink, math library) combinations the library launches.
template <class T, int MODE, class Sink, int LIB, int SRC, int BM = 1>
cudaError_t launch_ccd_narrow(int grid, cudaStream_t s, const int2* cand, int cand_cap, WsHeader* hdr, const T* x0,
                              const T* x1, Forest F, long long* rows, T* times, int max_per_tri, int* mesh_counters,
                              Weld W, Sink sink);
template <class T, int MODE, class Sink, int LIB, int SRC, int BM = 1> cudaError_t prepare_ccd_narrow();

#ifdef CCC_NARROW_TU
template <class T, int MODE, class Sink, int LIB, int SRC, int BM>
__global__ void __launch_bounds__(CCD_BLOCK, ccd_min_blocks(SRC, BM))
k_ccd_narrow(const int2* __restrict__ cand, int cand_cap, WsHeader* hdr, const T* __restrict__ x0,
             const T* __restrict__ x1, Forest F, long long* __restrict__ rows, T* __restrict__ times, int max_per_tri,
             int* __restrict__ mesh_counters, Weld W, Sink sink) {
    extern __shared__ __align__(16) unsigned char smem[];
    using L = CcdLayout<T, BM * CCD_BLOCK>;
    constexpr bool STAGED = SRC == SRC_STAGED;
    double* rec = reinterpret_cast<double*>(smem + L::rec);
    T* root_val = reinterpret_cast<T*>(smem + L::root_val);
    int2* items = reinterpret_cast<int2*>(smem + L::items);
    unsigned short* clist = reinterpret_cast<unsigned short*>(smem + L::clist);
    unsigned short* root_rec = reinterpret_cast<unsigned short*>(smem + L::root_rec);
    unsigned char* rec_cls = smem + L::rec_cls;
    unsigned short* rec_pos = reinterpret_cast<unsigned short*>(smem + L::rec_pos);
    int2* spairs = reinterpret_cast<int2*>(smem + L::spairs);
    unsigned short* pbuf = reinterpret_cast<unsigned short*>(smem + L::pbuf);
    int* ints = reinterpret_cast<int*>(smem + L::ints);
    constexpr int NW = CCD_BLOCK / 32;
    constexpr int NB = BM * CCD_BLOCK;
    constexpr int Q = L::QUEUE;
    const int M = forest_size(F);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned FULL = 0xffffffffu;
    const unsigned lt = (1u << lane) - 1u;
    const int n = min(*(volatile int*)(STAGED ? &hdr->live_count : &hdr->cand_count), cand_cap);
    int head = 0, queued = 0;           // ring queue of sub-tests (block-uniform)
    int masked = 0;                     // this thread's sub-tests before repeats are shared
    // class counts and root count of a batch, two sets used by alternate batches: a batch
    // clears the other set at its end, when every read of that set is two barriers back
    // (the staging barriers order the initial clearing before the first batch)
    int par = 0, cpar = 0;
    if (tid < 8) ints[CI_COUNT + tid] = 0;
    if (tid < 4) ints[CI_ROOTS + tid] = 0;
    if (tid < 2) ints[CI_LIVE + tid] = 0;
    __syncthreads();
    for (long long base = (long long)blockIdx.x * CCD_BLOCK;; base += (long long)gridDim.x * CCD_BLOCK) {
        const bool more = base < n;
        if (!more && queued == 0) break;
        if (more) {
            int2 pr = make_int2(0, 0);
            uint32_t bits = 0;
            unsigned shared_bits = 0;
            if constexpr (STAGED) {
                // the resident engine's pairs come staged by k_ccd_stage_*: the pairs with
                // sub-tests to solve, which ones, and which of them stand for their repeats
                const long long c = base + tid;
                if (c < n) {
                    const int4 rec = W.live[c];
                    pr = make_int2(rec.x, rec.y);
                    bits = (unsigned)rec.z & 0x7fffu;
                    shared_bits = ((unsigned)rec.z >> 15) & 0x7fffu;
                }
            } else {
                // about half of the candidate pairs are mesh neighbours that share a vertex:
                // the chunk's other pairs are gathered first (block-wide), so that the 15
                // swept sub-box tests run on full warps
                long long c = base + tid;
                bool live = false;
                if (c < n) {
                    pr = cand[c];
                    live = !ccd_pair_shares_vertex<T>(x0, pr.x, pr.y) &&
                           (SRC != SRC_EXACT || ccd_pair_leaf_overlap<T>(x0, x1, pr.x, pr.y));
                }
                const unsigned lb = __ballot_sync(FULL, live);
                int lbase = 0;
                if (lane == 0 && lb) lbase = atomicAdd(&ints[CI_LIVE + cpar], __popc(lb));
                lbase = __shfl_sync(FULL, lbase, 0);
                if (live) spairs[lbase + __popc(lb & lt)] = pr;
                __syncthreads();
                const int nlive = ints[CI_LIVE + cpar];
                // the other chunk parity's counter was last read before the barrier above
                if (tid == 0) ints[CI_LIVE + (cpar ^ 1)] = 0;
                cpar ^= 1;
                pr = make_int2(0, 0);
                if (tid < nlive) {
                    pr = spairs[tid];
                    bits = ccd_pair_subbox_mask<T, MODE != CCD_MINCOL>(x0, x1, pr.x, pr.y);
                }
                if (MODE != CCD_MINCOL) masked += __popc(bits);
                if (MODE == CCD_MINCOL) {
                    while (bits) {
                        int k = __ffs(bits) - 1;
                        bits &= bits - 1;
                        OutRegion R = out_region(F, M, pr.x, max_per_tri);
                        long long r = append_row(mesh_counters, F, R.m, R.cap, &hdr->status);
                        if (r >= 0) {
                            long long o = (long long)R.po * max_per_tri + r;
                            rows[o * 3 + 0] = pr.x - R.po;
                            rows[o * 3 + 1] = pr.y - R.po;
                            rows[o * 3 + 2] = k;
                        }
                    }
                    // the next chunk reuses spairs and the other live counter
                    __syncthreads();
                    continue;
                }
            }
            // append the chunk's sub-tests (block-wide exclusive scan of the counts)
            const int cnt = __popc(bits);
            const int incl = warp_inclusive_scan(cnt, lane);
            if (lane == 31) ints[CI_WARP + warp] = incl;
            __syncthreads();
            if (warp == 0) {
                int v = lane < NW ? ints[CI_WARP + lane] : 0;
                int sc = warp_inclusive_scan(v, lane);
                if (lane < NW) ints[CI_WARP + lane] = sc - v;
                if (lane == 31) ints[CI_TOTAL] = sc;
            }
            __syncthreads();
            int pos = head + queued + ints[CI_WARP + warp] + incl - cnt;
            const int total = ints[CI_TOTAL];
            while (bits) {
                int k = __ffs(bits) - 1;
                bits &= bits - 1;
                items[pos % Q] = pack_subtest(pr.x, pr.y, k, (shared_bits >> k) & 1u);
                ++pos;
            }
            if (tid == 0 && total) atomicAdd(&hdr->solved, total);
            queued += total;
            __syncthreads();
        }
        // solve full batches (and, after the last chunk, the remainder)
        while (queued >= NB || (!more && queued > 0)) {
            const int nb = min(NB, queued);
            // (1) coefficients and solver prefix; each sub-test takes its place in its class
            for (int ri = tid; ri < nb; ri += CCD_BLOCK) {
                int2 it = items[(head + ri) % Q];
                int k = (it.y >> 28) & 15;
                MTet<T> tet = load_tet(x0, x1, it.x & SLOT_MASK, it.y & SLOT_MASK, k);
                T cf[4];
                cubic_coeffs(tet, cf);
                rec[0 * NB + ri] = (double)cf[0];
                rec[1 * NB + ri] = (double)cf[1];
                rec[2 * NB + ri] = (double)cf[2];
                rec[3 * NB + ri] = (double)cf[3];
                double g, h;
                int cls = cubic_prefix<LIB>((double)cf[0], (double)cf[1], (double)cf[2], (double)cf[3], g, h);
                rec[4 * NB + ri] = g;
                rec[5 * NB + ri] = h;
                rec_cls[ri] = (unsigned char)cls;
                if (cls != CUBIC_NONE) rec_pos[ri] = (unsigned short)atomicAdd(&ints[CI_COUNT + 4 * par + cls - 1], 1);
            }
            __syncthreads();
            // sub-tests ordered by class (every thread forms the class offsets itself)
            const int* counts = ints + CI_COUNT + 4 * par;
            const int o1 = counts[0];
            const int o2 = o1 + counts[1];
            const int o3 = o2 + counts[2];
            const int nsolve = o3 + counts[3];
            for (int ri = tid; ri < nb; ri += CCD_BLOCK) {
                int cls = rec_cls[ri];
                if (cls != CUBIC_NONE) {
                    int off = cls == 1 ? 0 : (cls == 2 ? o1 : (cls == 3 ? o2 : o3));
                    clist[off + rec_pos[ri]] = (unsigned short)ri;
                }
            }
            __syncthreads();
            // (2) roots; the ones in [0, 1] go to the root list, edge-edge roots from its
            // front and vertex-face roots from its back
            for (int j0 = 0; j0 < nsolve; j0 += CCD_BLOCK) {
                const int j = j0 + tid;
                T rr[3] = {(T)-1, (T)-1, (T)-1};
                int ri = 0;
                bool ee = false;
                if (j < nsolve) {
                    ri = clist[j];
                    ee = ((items[(head + ri) % Q].y >> 28) & 15) < 9;
                    int cc = (j >= o1) + (j >= o2) + (j >= o3);
                    class_roots<T, LIB>(cc + 1, rec[0 * NB + ri], rec[1 * NB + ri], rec[2 * NB + ri],
                                        rec[3 * NB + ri], rec[4 * NB + ri], rec[5 * NB + ri], rr);
                }
#pragma unroll
                for (int s = 0; s < 3; ++s) {
                    bool keep = j < nsolve && (rr[s] >= 0 && rr[s] <= 1);
                    unsigned me = __ballot_sync(FULL, keep && ee);
                    unsigned mf = __ballot_sync(FULL, keep && !ee);
                    int ae = 0, af = 0;
                    if (lane == 0 && me) ae = atomicAdd(&ints[CI_ROOTS + 2 * par], __popc(me));
                    if (lane == 0 && mf) af = atomicAdd(&ints[CI_ROOTS + 2 * par + 1], __popc(mf));
                    ae = __shfl_sync(FULL, ae, 0) + __popc(me & lt);
                    af = __shfl_sync(FULL, af, 0) + __popc(mf & lt);
                    if (keep) {
                        const int at = ee ? ae : 3 * NB - 1 - af;
                        root_rec[at] = (unsigned short)ri;
                        root_val[at] = rr[s];
                    }
                }
            }
            __syncthreads();
            const int nee = ints[CI_ROOTS + 2 * par];
            const int nroots = nee + ints[CI_ROOTS + 2 * par + 1];
            if (tid == 0 && nroots) atomicAdd(&hdr->roots, nroots);
            // (3) filter and output
            if (MODE == CCD_ROWS) {
                // about one root in twelve passes the filter: those are buffered per warp and
                // their rows written 32 at a time, so that the mesh lookup and the row append
                // run on full warps rather than on the few lanes that passed
                unsigned short* pb = pbuf + warp * 64;
                int np = 0;                        // buffered roots of this warp (warp-uniform)
                // (mask: the lanes that call it together)
                auto emit = [&](int j, unsigned mask) {
                    const int2 it = items[(head + root_rec[j]) % Q];
                    const int qx = it.x & SLOT_MASK, qy = it.y & SLOT_MASK, k = (it.y >> 28) & 15;
                    const T tv = root_val[j];
                    // every pair of a shared sub-test is in the mesh of (qx, qy)
                    const OutRegion R = out_region(F, M, qx, max_per_tri);
                    auto row = [&](int a, int b, int kk) {
                        long long r = append_row(mesh_counters, F, R.m, R.cap, &hdr->status);
                        if (r >= 0) {
                            long long o = (long long)R.po * max_per_tri + r;
                            rows[o * 3 + 0] = a - R.po;
                            rows[o * 3 + 1] = b - R.po;
                            rows[o * 3 + 2] = kk;
                            times[o] = tv;
                        }
                    };
                    if constexpr (STAGED) {
                        // each passing root leaves a record for k_ccd_expand, which writes its
                        // rows (every pair's, for a shared sub-test); the roots that do not
                        // fit in the record list are written here
                        unsigned rest = mask;
                        if (W.expand) {
                            const int leader = __ffs(mask) - 1;
                            int b0 = 0;
                            if (lane == leader) b0 = atomicAdd(&hdr->expand_count, __popc(mask));
                            b0 = __shfl_sync(mask, b0, leader) + __popc(mask & lt);
                            const bool fits = b0 < W.expand_cap;
                            rest = __ballot_sync(mask, !fits);
                            if (fits) {
                                const double tw = (double)tv;
                                W.expand[b0] = make_int4(it.x, it.y, __double2loint(tw), __double2hiint(tw));
                                return;
                            }
                        }
                        int ma[WELD_FANCAP], mb[WELD_FANCAP], mk[WELD_FANCAP];
                        const int nm = weld_list(W, qx, qy, k, (it.x >> 28) & 1, ma, mb, mk);
                        // the rows of all the lanes in one mesh are reserved with one atomic
                        const int base = reserve_rows(mesh_counters, F, R.m, nm, rest);
                        for (int i = 0; i < nm; ++i) {
                            const long long r = (long long)base + i;
                            if (r >= R.cap) {
                                atomicOr(&hdr->status, ST_OUT_OVERFLOW);
                                break;
                            }
                            const long long o = (long long)R.po * max_per_tri + r;
                            rows[o * 3 + 0] = ma[i] - R.po;
                            rows[o * 3 + 1] = mb[i] - R.po;
                            rows[o * 3 + 2] = mk[i];
                            times[o] = tv;
                        }
                    } else {
                        row(qx, qy, k);
                    }
                };
                for (int b0 = warp * 32; b0 < nroots; b0 += CCD_BLOCK) {
                    const int jj = b0 + lane;
                    int j = 0;
                    bool pass = false;
                    if (jj < nroots) {
                        j = jj < nee ? jj : 3 * NB - 1 - (jj - nee);
                        const int2 it = items[(head + root_rec[j]) % Q];
                        const int k = (it.y >> 28) & 15;
                        MTet<T> tet = load_tet(x0, x1, it.x & SLOT_MASK, it.y & SLOT_MASK, k);
                        pass = ccd_filter(tet, k, root_val[j]);
                    }
                    const unsigned pm = __ballot_sync(FULL, pass);
                    if (pass) pb[np + __popc(pm & lt)] = (unsigned short)j;
                    np += __popc(pm);
                    if (np >= 32) {
                        __syncwarp();
                        emit(pb[lane], FULL);
                        __syncwarp();
                        if (lane < np - 32) pb[lane] = pb[32 + lane];
                        __syncwarp();
                        np -= 32;
                    }
                }
                __syncwarp();
                if (lane < np) emit(pb[lane], (1u << np) - 1u);     // (np < 32 here)
            } else {
                for (int jj = tid; jj < nroots; jj += CCD_BLOCK) {
                    const int j = jj < nee ? jj : 3 * NB - 1 - (jj - nee);
                    int2 it = items[(head + root_rec[j]) % Q];
                    int k = (it.y >> 28) & 15;
                    int2 q = make_int2(it.x & SLOT_MASK, it.y & SLOT_MASK);
                    T root = root_val[j];
                    MTet<T> tet = load_tet(x0, x1, q.x, q.y, k);
                    if (!ccd_filter(tet, k, root)) continue;
                    // the contact of every pair with this sub-test (its own corner masses)
                    int ma[STAGED ? WELD_FANCAP : 1], mb[STAGED ? WELD_FANCAP : 1], mk[STAGED ? WELD_FANCAP : 1];
                    int nm = 1;
                    if constexpr (STAGED) nm = weld_list(W, q.x, q.y, k, (it.x >> 28) & 1, ma, mb, mk);
                    else {
                        ma[0] = q.x;
                        mb[0] = q.y;
                        mk[0] = k;
                    }
                    for (int i = 0; i < nm; ++i) {
                        const int a = ma[i], b = mb[i], kk = mk[i];
                        T mq[4];
#pragma unroll
                        for (int pt = 0; pt < 4; ++pt)
                            mq[pt] = sink.masses[(long long)(tet_side(kk, pt) ? b : a) * 3 + tet_corner(kk, pt)];
                        Contact<T> ct = contact<T, LIB>(tet, kk, root, mq);
                        sink.add(tet, a, b, kk, root, ct, F, M, &hdr->status);
                    }
                }
            }
            if (tid < 4) ints[CI_COUNT + 4 * (par ^ 1) + tid] = 0;
            if (tid >= 4 && tid < 6) ints[CI_ROOTS + 2 * (par ^ 1) + tid - 4] = 0;
            par ^= 1;
            head = (head + nb) % Q;
            queued -= nb;
            __syncthreads();
        }
    }
    // (the loop ends for the whole block at once)
    if (MODE != CCD_MINCOL) {
        const int ws = __reduce_add_sync(FULL, masked);
        if (lane == 0 && ws) atomicAdd(&hdr->subtests, ws);
    }
}

// Launch of k_ccd_narrow with its dynamic shared memory (the size is raised once per
// instantiation and device; prepare_ccd_narrow does it ahead of any stream capture).
// The flags are atomic because host threads may launch on different streams at once; two
// first calls may both set the attribute, which is harmless.
template <class T, int MODE, class Sink, int LIB, int SRC, int BM> cudaError_t prepare_ccd_narrow() {
    static std::atomic<bool> done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && done[dev].load(std::memory_order_acquire)) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_ccd_narrow<T, MODE, Sink, LIB, SRC, BM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)CcdLayout<T, BM * CCD_BLOCK>::bytes);
    if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev].store(true, std::memory_order_release);
    return e;
}

template <class T, int MODE, class Sink, int LIB, int SRC, int BM>
cudaError_t launch_ccd_narrow(int grid, cudaStream_t s, const int2* cand, int cand_cap, WsHeader* hdr, const T* x0,
                              const T* x1, Forest F, long long* rows, T* times, int max_per_tri, int* mesh_counters,
                              Weld W, Sink sink) {
    cudaError_t e = prepare_ccd_narrow<T, MODE, Sink, LIB, SRC, BM>();
    if (e != cudaSuccess) return e;
    k_ccd_narrow<T, MODE, Sink, LIB, SRC, BM><<<grid, CCD_BLOCK, CcdLayout<T, BM * CCD_BLOCK>::bytes, s>>>(
        cand, cand_cap, hdr, x0, x1, F, rows, times, max_per_tri, mesh_counters, W, sink);
    return cudaSuccess;
}

#endif  // CCC_NARROW_TU

// The rows of the roots that passed the filter in k_ccd_narrow (its records in Weld.expand),
// every pair's for a shared sub-test: one record a thread, the rows of a warp's lanes
// reserved with one atomic per mesh.
static constexpr int EXPAND_THREADS = 256;
template <class T>
__global__ void __launch_bounds__(EXPAND_THREADS)
k_ccd_expand(WsHeader* hdr, Weld W, Forest F, long long* __restrict__ rows, T* __restrict__ times, int max_per_tri,
             int* __restrict__ mesh_counters) {
    const unsigned FULL = 0xffffffffu;
    const int M = forest_size(F);
    const int n = min(*(volatile int*)&hdr->expand_count, W.expand_cap);
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (EXPAND_THREADS / 32);
    for (int base = ((blockIdx.x * EXPAND_THREADS + threadIdx.x) >> 5) * 32; base < n; base += nwarps * 32) {
        const int c = base + lane;
        int ma[WELD_FANCAP], mb[WELD_FANCAP], mk[WELD_FANCAP];
        int nm = 0, m = 0, po = 0;
        long long cap = 0;
        T tv = T(0);
        if (c < n) {
            const int4 rec = W.expand[c];
            const int qx = rec.x & SLOT_MASK, qy = rec.y & SLOT_MASK, k = (rec.y >> 28) & 15;
            tv = (T)__hiloint2double(rec.w, rec.z);
            const OutRegion R = out_region(F, M, qx, max_per_tri);
            m = R.m;
            po = R.po;
            cap = R.cap;
            nm = weld_list(W, qx, qy, k, (rec.x >> 28) & 1, ma, mb, mk);
        }
        const unsigned has = __ballot_sync(FULL, nm > 0);
        if (nm > 0) {
            const int first = reserve_rows(mesh_counters, F, m, nm, has);
            for (int i = 0; i < nm; ++i) {
                const long long r = (long long)first + i;
                if (r >= cap) {
                    atomicOr(&hdr->status, ST_OUT_OVERFLOW);
                    break;
                }
                const long long o = (long long)po * max_per_tri + r;
                rows[o * 3 + 0] = ma[i] - po;
                rows[o * 3 + 1] = mb[i] - po;
                rows[o * 3 + 2] = mk[i];
                times[o] = tv;
            }
        }
    }
}

// proximity (proximity_static.cu:11-508)
template <class T>
__global__ void __launch_bounds__(NARROW_THREADS)
k_prox_narrow(const int2* __restrict__ cand, int cand_cap, WsHeader* hdr, const T* __restrict__ tri, Forest F, T th,
              long long* __restrict__ rows, int max_per_tri, int* __restrict__ mesh_counters) {
    const int M = forest_size(F);
    int n = min(hdr->cand_count, cand_cap);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int2 pr = cand[c];
        Tri<T> a = load_tri(tri, pr.x), b = load_tri(tri, pr.y);
        if (share_vertex(a.v, b.v)) continue;
        for (int k = 0; k < 15; ++k) {
            if (!prox_subbox(a, b, k, th)) continue;
            T d = prox_distance(a, b, k);
            if (!(d <= th && d >= 0)) continue;
            OutRegion R = out_region(F, M, pr.x, max_per_tri);
            long long r = append_row(mesh_counters, F, R.m, R.cap, &hdr->status);
            if (r >= 0) {
                long long o = (long long)R.po * max_per_tri + r;
                rows[o * 3 + 0] = pr.x - R.po;
                rows[o * 3 + 1] = pr.y - R.po;
                rows[o * 3 + 2] = k;
            }
        }
    }
}

// compute_impulses_from_collisions (collisions_impulses.cu:1738-1880) on caller rows.
// Rows with an index outside [0, F) or a type outside [0, 15) are skipped (the reference
// reads out of bounds on its -1 padding rows).
template <class T, int LIB>
__global__ void __launch_bounds__(NARROW_THREADS)
k_impulses_from_rows(const long long* __restrict__ rows, const T* __restrict__ roots, int B, long long N, int F,
                     const T* __restrict__ x0, const T* __restrict__ x1, const T* __restrict__ masses,
                     T* __restrict__ dv_out, T* __restrict__ dx_out, int* __restrict__ cnt_out, WsHeader* hdr) {
    long long total = (long long)B * N;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < total;
         r += (long long)gridDim.x * blockDim.x) {
        long long b = r / N;
        long long i = rows[r * 3 + 0], j = rows[r * 3 + 1], kk = rows[r * 3 + 2];
        if (i < 0 || j < 0 || i >= F || j >= F || kk < 0 || kk >= 15) continue;
        int k = (int)kk;
        long long gi = b * F + i, gj = b * F + j;
        T root = roots[r];
        MTet<T> tet = load_tet(x0, x1, gi, gj, k);
        T mq[4];
        for (int pt = 0; pt < 4; ++pt) mq[pt] = masses[(tet_side(k, pt) ? gj : gi) * 3 + tet_corner(k, pt)];
        Contact<T> ct = contact<T, LIB>(tet, k, root, mq);
        apply_impulse(tet, gi, gj, k, root, ct, dv_out, dx_out, cnt_out);
    }
}

// Test hooks of the solver's arithmetic (k_debug_math, k_debug_stage), compiled in
// ccc_narrow.cu with the continuous narrow phase, so that they compute what it computes.
cudaError_t launch_debug_math(int op, const double* in, double* out, int n, cudaStream_t s);
cudaError_t launch_debug_stage(int op, int lib, const double* in, int in_stride, double* out, int out_stride, int n,
                               cudaStream_t s);

}  // namespace ccc
