// ccc_oracle.cpp — CPU restatement of the reference collision pipeline.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only the test
// suite, the smoke check and the benchmark's CPU-baseline leg may load it.  The product
// library never links or calls it.
//
// It restates, one function per reference routine, the semantics of Dolorousrtur/
// CCCollisions (file:line citations are relative to that project's root):
//   * LBVH build  (src/build_bvh.cu, src/bvh.cu, src/aabb.cu, src/figures.cu)
//   * BVH traversal with the "rightmost" ordering rule (src/collisions_static.cu:10-120)
//     and its masked variant (src/collisions_continuous.cu:127-230, 1079-1099)
//   * static triangle-triangle separating-axis test (src/figures.cu:378-576,
//     src/collisions_static.cu:123-159)
//   * continuous collision: 15 sub-tests, tetrahedra, cubic coefficients, Cardano solve,
//     root flattening and inside/segment filters (src/collisions_continuous.cu:14-765)
//   * impulses (src/collisions_impulses.cu:24-1067)
//   * proximity (src/proximity_static.cu:11-508)
//   * triangle-edge helpers (src/collisions_static.cu:345-942, src/icontour.cu:11-281)
//
// Arithmetic: IEEE-754 float/double in the reference's evaluation order, term by term.
// The reference is compiled by nvcc with its default fused multiply-add contraction, so
// the restatement writes those fusions out explicitly (fmaT) where nvcc forms them:
// a*b + c -> fma(a, b, c); c + a*b -> fma(a, b, c); a*b + c*d and a*b - c*d fuse the first
// product; dot / cross / norm2 become fixed fma chains.  This model reproduces the
// reference's cubic coefficients and root filters bit for bit (tests/test_golden.py).
// Nothing else is contracted (built with -ffp-contract=off).  The
// transcendental calls of the cubic solver go through ccc_libm.h and the CAMPARY products
// through ccc_ddmul.h, which the CUDA path includes too, so results agree to the bit.
//
// Parity pin: the reference ships no tests or golden vectors.  This restatement is pinned
// by hand-derived known-answer tests (tests/test_oracle_kat.py), brute-force O(F^2)
// enumeration, and fixtures written by the reference extension itself where available.

#include <stdint.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <vector>
#include <algorithm>
#include <atomic>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../cccollisions_b200/csrc/ccc_libm.h"
#include "../cccollisions_b200/csrc/ccc_ddmul.h"

namespace orc {

template <class T> struct V3 { T x, y, z; };
template <class T> static inline V3<T> mk(T x, T y, T z) { V3<T> r; r.x = x; r.y = y; r.z = z; return r; }
template <class T> static inline V3<T> operator+(V3<T> a, V3<T> b) { return mk<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> static inline V3<T> operator-(V3<T> a, V3<T> b) { return mk<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> static inline V3<T> operator*(V3<T> a, T s) { return mk<T>(a.x * s, a.y * s, a.z * s); }
template <class T> static inline V3<T> operator/(V3<T> a, T s) { return mk<T>(a.x / s, a.y / s, a.z / s); }
static inline float fmaT(float a, float b, float c) { return fmaf(a, b, c); }
static inline double fmaT(double a, double b, double c) { return fma(a, b, c); }
// a.x*b.x + a.y*b.y + a.z*b.z  ->  fma(a.z, b.z, fma(a.x, b.x, a.y*b.y))
template <class T> static inline T dot(V3<T> a, V3<T> b) { return fmaT(a.z, b.z, fmaT(a.x, b.x, a.y * b.y)); }
template <class T> static inline T dot_zyx(V3<T> a, V3<T> b) { return fmaT(a.z, b.z, fmaT(a.y, b.y, a.x * b.x)); }
// a.y*b.z - a.z*b.y  ->  fma(a.y, b.z, -(a.z*b.y)), and cyclically
template <class T> static inline V3<T> cross(V3<T> a, V3<T> b) {
    return mk<T>(fmaT(a.y, b.z, -(a.z * b.y)), fmaT(a.z, b.x, -(a.x * b.z)), fmaT(a.x, b.y, -(a.y * b.x)));
}
template <class T> static inline T norm2(V3<T> a) { return fmaT(a.z, a.z, fmaT(a.x, a.x, a.y * a.y)); }
// v + d * t  ->  fma(d, t, v) per component
template <class T> static inline V3<T> axpy(V3<T> v, V3<T> d, T t) {
    return mk<T>(fmaT(d.x, t, v.x), fmaT(d.y, t, v.y), fmaT(d.z, t, v.z));
}
// a*u + b*v + c*w  ->  fma(c, w, fma(a, u, b*v)) per component
template <class T> static inline V3<T> lin3(V3<T> a, T u, V3<T> b, T v, V3<T> c, T w) {
    return mk<T>(fmaT(c.x, w, fmaT(a.x, u, b.x * v)), fmaT(c.y, w, fmaT(a.y, u, b.y * v)),
                 fmaT(c.z, w, fmaT(a.z, u, b.z * v)));
}
// a*b - c*d  ->  fma(a, b, -(c*d))
template <class T> static inline T fms2(T a, T b, T c, T d) { return fmaT(a, b, -(c * d)); }
// CUDA min/max on floating point follow fmin/fmax (a NaN operand yields the other one)
template <class T> static inline T fmn(T a, T b) { return (T)fmin(a, b); }
template <class T> static inline T fmx(T a, T b) { return (T)fmax(a, b); }

template <class T> struct Box { V3<T> lo, hi; };
// AABB::operator+ (aabb.cu:51-56)
template <class T> static inline Box<T> merge(const Box<T>& a, const Box<T>& b) {
    Box<T> r;
    r.lo = mk<T>(fmn(a.lo.x, b.lo.x), fmn(a.lo.y, b.lo.y), fmn(a.lo.z, b.lo.z));
    r.hi = mk<T>(fmx(a.hi.x, b.hi.x), fmx(a.hi.y, b.hi.y), fmx(a.hi.z, b.hi.z));
    return r;
}
// checkOverlap (aabb.cu:101-111): inclusive, threshold widens the second box
template <class T> static inline bool overlap(const Box<T>& a, const Box<T>& b, T th) {
    return (a.lo.x <= (b.hi.x + th)) && (a.hi.x >= (b.lo.x - th)) &&
           (a.lo.y <= (b.hi.y + th)) && (a.hi.y >= (b.lo.y - th)) &&
           (a.lo.z <= (b.hi.z + th)) && (a.hi.z >= (b.lo.z - th));
}

template <class T> struct Tri { V3<T> v[3]; };
template <class T> static inline Tri<T> load_tri(const T* p, int64_t i) {
    Tri<T> t;
    for (int c = 0; c < 3; ++c) t.v[c] = mk<T>(p[i * 9 + c * 3 + 0], p[i * 9 + c * 3 + 1], p[i * 9 + c * 3 + 2]);
    return t;
}
// Triangle::ComputeBBox (figures.cu:37-41)
template <class T> static inline Box<T> tri_box(const Tri<T>& t) {
    Box<T> b;
    b.lo = mk<T>(fmn(t.v[0].x, fmn(t.v[1].x, t.v[2].x)), fmn(t.v[0].y, fmn(t.v[1].y, t.v[2].y)),
                 fmn(t.v[0].z, fmn(t.v[1].z, t.v[2].z)));
    b.hi = mk<T>(fmx(t.v[0].x, fmx(t.v[1].x, t.v[2].x)), fmx(t.v[0].y, fmx(t.v[1].y, t.v[2].y)),
                 fmx(t.v[0].z, fmx(t.v[1].z, t.v[2].z)));
    return b;
}

// ---------------------------------------------------------------------------------------
// LBVH build
// ---------------------------------------------------------------------------------------

// expandBits / morton3D (bvh.cu:29-62)
static inline uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
template <class T> static inline uint32_t morton3d(T x, T y, T z) {
    // x * 1024.0f is evaluated in T; min/max with fmin/fmax semantics, then truncation
    x = fmn<T>(fmx<T>(x * (T)1024.0f, (T)0.0f), (T)1023.0f);
    y = fmn<T>(fmx<T>(y * (T)1024.0f, (T)0.0f), (T)1023.0f);
    z = fmn<T>(fmx<T>(z * (T)1024.0f, (T)0.0f), (T)1023.0f);
    return expand_bits((uint32_t)x) * 4 + expand_bits((uint32_t)y) * 2 + expand_bits((uint32_t)z);
}

static inline int nthr(int n) {
#ifdef _OPENMP
    return n > 0 ? n : omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

static inline int clz32(uint32_t v) { return v == 0 ? 32 : __builtin_clz(v); }

// LongestCommonPrefix (bvh.cu:65-89)
static inline int lcp(int i, int j, const uint32_t* codes, int n, const int* ids) {
    if (i < 0 || i > n - 1 || j < 0 || j > n - 1) return -1;
    uint32_t k1 = codes[i], k2 = codes[j];
    if (k1 == k2) return clz32(k1 ^ k2) + clz32((uint32_t)(ids[i] ^ ids[j]));
    return clz32(k1 ^ k2);
}

// Tree in the reference's exported numbering: node k < F-1 internal, k >= F-1 leaf
// (leaf position k - (F-1)).  Arrays are sized 2F-1.
struct Topo {
    std::vector<int> parent, left, right, rightmost;
};

// BuildRadixTree (build_bvh.cu:74-143) over sorted codes; writes children / parents in the
// exported numbering.
static void karras(const uint32_t* codes, const int* ids, int n, Topo& tp) {
    tp.parent.assign(2 * n - 1, -1);
    tp.left.assign(2 * n - 1, -1);
    tp.right.assign(2 * n - 1, -1);
    for (int idx = 0; idx < n - 1; ++idx) {
        int dnext = lcp(idx, idx + 1, codes, n, ids);
        int dlast = lcp(idx, idx - 1, codes, n, ids);
        int dir = dnext - dlast >= 0 ? 1 : -1;
        int dmin = lcp(idx, idx - dir, codes, n, ids);
        int lmax = 2;
        while (lcp(idx, idx + lmax * dir, codes, n, ids) > dmin) lmax *= 2;
        int l = 0;
        int div = 2;
        for (int t = lmax / div; t >= 1; div *= 2) {
            if (lcp(idx, idx + (l + t) * dir, codes, n, ids) > dmin) l = l + t;
            t = lmax / div;
        }
        int j = idx + l * dir;
        int nd = lcp(idx, j, codes, n, ids);
        // The reference's split search uses ceil(l / div), which never reaches 0: on the GPU
        // the loop ends only when the 32-bit divider overflows (after div = 2^30).  Every
        // extra pass has t == 1 and is idempotent once the monotone predicate has failed, so
        // stopping at div = 2^30 gives the reference's split (= the standard Karras split).
        int s = 0;
        long long ldiv = 2;
        for (int t = (int)((l + (ldiv - 1)) / ldiv); t >= 1 && ldiv <= (1LL << 30); ldiv *= 2) {
            if (lcp(idx, idx + (s + t) * dir, codes, n, ids) > nd) s = s + t;
            t = (int)((l + (ldiv - 1)) / ldiv);
        }
        int split = idx + s * dir + std::min(dir, 0);
        int lc = (std::min(idx, j) == split) ? (n - 1 + split) : split;
        int rc = (std::max(idx, j) == split + 1) ? (n - 1 + split + 1) : (split + 1);
        tp.left[idx] = lc;
        tp.right[idx] = rc;
        tp.parent[lc] = idx;
        tp.parent[rc] = idx;
    }
}

// Subtree boxes and rightmost leaf position, bottom-up (CreateHierarchy build_bvh.cu:145-209
// and set_rightmost_nodes 707-743 compute the same values with atomic counters).
template <class T>
static void refit(int n, const Topo& tp, std::vector<Box<T>>& box, std::vector<int>& rm) {
    rm.assign(2 * n - 1, -1);
    for (int p = 0; p < n; ++p) rm[n - 1 + p] = p;
    // post-order by explicit stack from the root
    std::vector<int> order;
    order.reserve(2 * n);
    std::vector<int> st;
    st.push_back(0);
    while (!st.empty()) {
        int k = st.back();
        st.pop_back();
        order.push_back(k);
        if (k < n - 1) {
            st.push_back(tp.left[k]);
            st.push_back(tp.right[k]);
        }
    }
    for (int i = (int)order.size() - 1; i >= 0; --i) {
        int k = order[i];
        if (k >= n - 1) continue;
        box[k] = merge(box[tp.left[k]], box[tp.right[k]]);
        rm[k] = std::max(rm[tp.left[k]], rm[tp.right[k]]);
    }
}

// build_bvh (build_bvh.cu:221-306, 381-449) and its motion overload (476-648).
// spatial == 0 restates the reference literally: the scene box is reduced from the
// initial AABB() = (-MAX, +MAX) (aabb.cu:25-34, build_bvh.cu:243), so it is unbounded,
// every normalised centroid divides by an infinite extent, and every Morton code is 0;
// the stable sort then keeps the input order.  spatial == 1 starts the reduction from the
// empty box instead, giving real Morton codes (a spatially sorted tree; the pairs found
// do not depend on the tree).
template <class T>
static void build(const T* tri, const T* tri_next, int n, int spatial, T* bboxes_out, int64_t* tree_out,
                  uint32_t* codes_out) {
    std::vector<Box<T>> lb(n);
    for (int i = 0; i < n; ++i) {
        Box<T> b = tri_box(load_tri(tri, i));
        if (tri_next) b = merge(b, tri_box(load_tri(tri_next, i)));    // MergeTriBoundingBoxes 452-460
        lb[i] = b;
    }
    const T MX = sizeof(T) == 4 ? (T)FLT_MAX : (T)DBL_MAX;
    Box<T> scene;
    if (spatial) { scene.lo = mk<T>(MX, MX, MX); scene.hi = mk<T>(-MX, -MX, -MX); }
    else { scene.lo = mk<T>(-MX, -MX, -MX); scene.hi = mk<T>(MX, MX, MX); }
    for (int i = 0; i < n; ++i) scene = merge(scene, lb[i]);
    std::vector<uint32_t> codes(n);
    for (int i = 0; i < n; ++i) {
        Tri<T> t = load_tri(tri, i);
        V3<T> c = ((t.v[0] + t.v[1]) + t.v[2]) / (T)3.0;       // ComputeMortonCodes 26-46
        if (tri_next) {                                         // motion version 48-71
            Tri<T> t2 = load_tri(tri_next, i);
            V3<T> c2 = ((t2.v[0] + t2.v[1]) + t2.v[2]) / (T)3.0;
            c = (c + c2) / (T)2.0;
        }
        T x = (c.x - scene.lo.x) / (scene.hi.x - scene.lo.x);
        T y = (c.y - scene.lo.y) / (scene.hi.y - scene.lo.y);
        T z = (c.z - scene.lo.z) / (scene.hi.z - scene.lo.z);
        codes[i] = morton3d<T>(x, y, z);
    }
    // thrust::sequence + stable sort_by_key (build_bvh.cu:268-279)
    std::vector<int> ids(n);
    for (int i = 0; i < n; ++i) ids[i] = i;
    std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return codes[a] < codes[b]; });
    std::vector<uint32_t> sc(n);
    for (int i = 0; i < n; ++i) sc[i] = codes[ids[i]];
    if (codes_out) memcpy(codes_out, codes.data(), sizeof(uint32_t) * n);
    Topo tp;
    karras(sc.data(), ids.data(), n, tp);
    std::vector<Box<T>> box(2 * n - 1);
    for (int p = 0; p < n; ++p) box[n - 1 + p] = lb[ids[p]];   // leaf box = bboxes[tri_id] (161)
    std::vector<int> rm;
    refit(n, tp, box, rm);
    // CreateBboxesTree (309-378)
    for (int k = 0; k < 2 * n - 1; ++k) {
        T* bo = bboxes_out + (int64_t)k * 6;
        bo[0] = box[k].lo.x; bo[1] = box[k].lo.y; bo[2] = box[k].lo.z;
        bo[3] = box[k].hi.x; bo[4] = box[k].hi.y; bo[5] = box[k].hi.z;
        int64_t* to = tree_out + (int64_t)k * 4;
        to[0] = tp.parent[k];
        to[1] = tp.left[k];
        to[2] = tp.right[k];
        to[3] = (k >= n - 1) ? ids[k - (n - 1)] : -1;
    }
}

// ---------------------------------------------------------------------------------------
// Traversal
// ---------------------------------------------------------------------------------------

// Tree imported from the exported tensors (build_bvh_from_array_tree 667-705 +
// set_rightmost_nodes 707-743).
template <class T> struct Forest {
    int n;
    std::vector<Box<T>> box;
    std::vector<int> left, right, rm, idx;
    bool ok = true;
};

template <class T> static void import_tree(const T* bboxes, const int64_t* tree, int n, Forest<T>& f) {
    f.n = n;
    f.box.resize(2 * n - 1);
    f.left.assign(2 * n - 1, -1);
    f.right.assign(2 * n - 1, -1);
    f.idx.assign(2 * n - 1, -1);
    for (int k = 0; k < 2 * n - 1; ++k) {
        const T* b = bboxes + (int64_t)k * 6;
        f.box[k].lo = mk<T>(b[0], b[1], b[2]);
        f.box[k].hi = mk<T>(b[3], b[4], b[5]);
        f.left[k] = (int)tree[k * 4 + 1];
        f.right[k] = (int)tree[k * 4 + 2];
        f.idx[k] = (int)tree[k * 4 + 3];
    }
    // rightmost via the same post-order walk (boxes are kept as imported)
    f.rm.assign(2 * n - 1, -1);
    for (int p = 0; p < n; ++p) f.rm[n - 1 + p] = p;
    std::vector<int> order, st;
    st.push_back(0);
    size_t guard = 0;
    while (!st.empty()) {
        int k = st.back();
        st.pop_back();
        if (k < 0 || k >= 2 * n - 1 || ++guard > (size_t)(4 * n)) { f.ok = false; return; }
        order.push_back(k);
        if (k < n - 1) { st.push_back(f.left[k]); st.push_back(f.right[k]); }
    }
    for (int i = (int)order.size() - 1; i >= 0; --i) {
        int k = order[i];
        if (k < n - 1) f.rm[k] = std::max(f.rm[f.left[k]], f.rm[f.right[k]]);
    }
}

// traverseBVH (collisions_static.cu:10-103) / traverseBVHPartial
// (collisions_continuous.cu:127-230) for one query leaf position p.  Appends (min id,
// max id) pairs.  mask == nullptr: full query with the ordering rule; otherwise the masked
// variant: the query runs only if mask[p] (mask indexed by leaf POSITION, 1090), ordering
// is disabled, and a hit leaf c is kept if !mask[id_c] (indexed by triangle ID, 174) or
// id_p < id_c.
template <class T>
static int traverse_one(const Forest<T>& f, int p, T th, const uint8_t* mask, std::vector<int64_t>& out) {
    const int n = f.n;
    const int leaf = n - 1 + p;
    const Box<T>& q = f.box[leaf];
    const int qid = f.idx[leaf];
    const bool ordering = (mask == nullptr);
    int stack[64];
    int sp = 0;
    stack[sp++] = -1;
    int node = 0;
    int depth_fail = 0;
    do {
        int cl = f.left[node], cr = f.right[node];
        bool ol = overlap(q, f.box[cl], th);
        bool orr = overlap(q, f.box[cr], th);
        if (ordering) {
            if (p >= f.rm[cl]) ol = false;
            if (p >= f.rm[cr]) orr = false;
        }
        bool ll = cl >= n - 1, rl = cr >= n - 1;
        if (ol && ll) {
            int cid = f.idx[cl];
            if (!mask || !mask[cid] || qid < cid) {
                out.push_back(std::min(qid, cid));
                out.push_back(std::max(qid, cid));
            }
        }
        if (orr && rl) {
            int cid = f.idx[cr];
            if (!mask || !mask[cid] || qid < cid) {
                out.push_back(std::min(qid, cid));
                out.push_back(std::max(qid, cid));
            }
        }
        bool tl = ol && !ll, tr = orr && !rl;
        if (!tl && !tr) {
            node = stack[--sp];
        } else {
            node = tl ? cl : cr;
            if (tl && tr) {
                if (sp >= 64) { depth_fail = 1; break; }
                stack[sp++] = cr;
            }
        }
    } while (node != -1);
    return depth_fail;
}

template <class T>
static int64_t candidates(const Forest<T>& f, T th, const uint8_t* mask, std::vector<int64_t>& pairs, int nthreads) {
    const int n = f.n;
    pairs.clear();
    int bad = 0;
#ifdef _OPENMP
    int nt = nthr(nthreads);
    std::vector<std::vector<int64_t>> loc(nt);
#pragma omp parallel num_threads(nt) reduction(| : bad)
    {
        std::vector<int64_t>& mine = loc[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 256)
        for (int p = 0; p < n; ++p) {
            if (mask && !mask[p]) continue;
            bad |= traverse_one(f, p, th, mask, mine);
        }
    }
    for (auto& v : loc) pairs.insert(pairs.end(), v.begin(), v.end());
#else
    (void)nthreads;
    for (int p = 0; p < n; ++p) {
        if (mask && !mask[p]) continue;
        bad |= traverse_one(f, p, th, mask, pairs);
    }
#endif
    return bad ? -1 : (int64_t)(pairs.size() / 2);
}

// ---------------------------------------------------------------------------------------
// Static narrow phase
// ---------------------------------------------------------------------------------------

// isect_interval / TriangleTriangleOverlap (figures.cu:378-427)
template <class T> static inline bool axis_overlap(const Tri<T>& a, const Tri<T>& b, V3<T> ax, T th) {
    T d = dot(ax, a.v[0]);
    T alo = d, ahi = d;
    d = dot(ax, a.v[1]); alo = fmn(alo, d); ahi = fmx(ahi, d);
    d = dot(ax, a.v[2]); alo = fmn(alo, d); ahi = fmx(ahi, d);
    d = dot(ax, b.v[0]);
    T blo = d, bhi = d;
    d = dot(ax, b.v[1]); blo = fmn(blo, d); bhi = fmx(bhi, d);
    d = dot(ax, b.v[2]); blo = fmn(blo, d); bhi = fmx(bhi, d);
    return (alo <= bhi + th) && (ahi >= blo - th);
}

// TriangleTriangleIsectSepAxis (figures.cu:446-509)
template <class T> static bool sat(const Tri<T>& a, const Tri<T>& b, T th) {
    V3<T> a0 = a.v[1] - a.v[0], a1 = a.v[2] - a.v[0], a2 = a.v[2] - a.v[1];
    V3<T> an = cross(a1, a2);
    V3<T> b0 = b.v[1] - b.v[0], b1 = b.v[2] - b.v[0], b2 = b.v[2] - b.v[1];
    V3<T> bn = cross(b1, b2);
    V3<T> axes[17] = {an, bn,
                      cross(a0, b0), cross(a0, b1), cross(a0, b2),
                      cross(a1, b0), cross(a1, b1), cross(a1, b2),
                      cross(a2, b0), cross(a2, b1), cross(a2, b2),
                      cross(an, a0), cross(an, a1), cross(an, a2),
                      cross(an, b0), cross(an, b1), cross(an, b2)};
    bool ok = true;
    for (int i = 0; i < 17; ++i) ok = ok && axis_overlap(a, b, axes[i], th);
    return ok;
}

template <class T> static inline bool veq(V3<T> a, V3<T> b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// countSharedVerts (figures.cu:548-576)
template <class T> static int count_shared(const Tri<T>& a, const Tri<T>& b) {
    int c = 0;
    for (int i = 0; i < 3; ++i)
        if (veq(a.v[i], b.v[0]) || veq(a.v[i], b.v[1]) || veq(a.v[i], b.v[2])) ++c;
    return c;
}
// shareVertex (figures.cu:527-544, 578-596)
template <class T> static bool share_vertex(const Tri<T>& a, const Tri<T>& b) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (veq(a.v[i], b.v[j])) return true;
    return false;
}

// ---------------------------------------------------------------------------------------
// Continuous collision
// ---------------------------------------------------------------------------------------

template <class T> struct MTri { V3<T> v[3], dv[3]; };
// MovingTriangle(Triangle, Triangle) (figures.cu:307-314): dv = x1 - x0
template <class T> static inline MTri<T> load_mtri(const T* x0, const T* x1, int64_t i) {
    Tri<T> a = load_tri(x0, i), b = load_tri(x1, i);
    MTri<T> m;
    for (int c = 0; c < 3; ++c) { m.v[c] = a.v[c]; m.dv[c] = b.v[c] - a.v[c]; }
    return m;
}
// MovingTriangle::ComputeBBoxVertex (346-351): box of v and v + dv
template <class T> static inline Box<T> mvbox(const MTri<T>& t, int i) {
    V3<T> a = t.v[i], b = t.v[i] + t.dv[i];
    Box<T> r;
    r.lo = mk<T>(fmn(a.x, b.x), fmn(a.y, b.y), fmn(a.z, b.z));
    r.hi = mk<T>(fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z));
    return r;
}
// static boxes (Triangle::ComputeBBoxVertex 58-61) as degenerate boxes
template <class T> static inline Box<T> svbox(const Tri<T>& t, int i) {
    Box<T> r;
    r.lo = t.v[i];
    r.hi = t.v[i];
    return r;
}

// edge table {01, 02, 12} used by types 0..8 (collisions_continuous.cu:36-124, 234-318)
static const int EA[3] = {0, 0, 1};
static const int EB[3] = {1, 2, 2};

// corner indices of the four tetrahedron points for type k: side (0 = first triangle of
// the pair, 1 = second) and corner.
static inline void type_points(int k, int side[4], int corner[4]) {
    if (k < 9) {
        int e0 = k / 3, e1 = k % 3;
        side[0] = 0; corner[0] = EA[e0];
        side[1] = 0; corner[1] = EB[e0];
        side[2] = 1; corner[2] = EA[e1];
        side[3] = 1; corner[3] = EB[e1];
    } else if (k < 12) {
        side[0] = 0; corner[0] = 0;
        side[1] = 0; corner[1] = 1;
        side[2] = 0; corner[2] = 2;
        side[3] = 1; corner[3] = k - 9;
    } else {
        side[0] = 0; corner[0] = k - 12;
        side[1] = 1; corner[1] = 0;
        side[2] = 1; corner[2] = 1;
        side[3] = 1; corner[3] = 2;
    }
}

// check_minimal_bbox_overlap (collisions_continuous.cu:234-318): swept sub-boxes, no threshold
template <class T> static bool ccd_subbox(const MTri<T>& a, const MTri<T>& b, int k) {
    Box<T> b0, b1;
    if (k < 9) {
        int e0 = k / 3, e1 = k % 3;
        b0 = merge(mvbox(a, EA[e0]), mvbox(a, EB[e0]));
        b1 = merge(mvbox(b, EA[e1]), mvbox(b, EB[e1]));
    } else if (k < 12) {
        b0 = merge(merge(mvbox(a, 0), mvbox(a, 1)), mvbox(a, 2));
        b1 = mvbox(b, k - 9);
    } else {
        b0 = mvbox(a, k - 12);
        b1 = merge(merge(mvbox(b, 0), mvbox(b, 1)), mvbox(b, 2));
    }
    return overlap(b0, b1, (T)0);
}

template <class T> struct MTet { V3<T> v[4], dv[4]; };
template <class T> static inline MTet<T> make_tet(const MTri<T>& a, const MTri<T>& b, int k) {
    int side[4], corner[4];
    type_points(k, side, corner);
    MTet<T> t;
    for (int i = 0; i < 4; ++i) {
        const MTri<T>& s = side[i] ? b : a;
        t.v[i] = s.v[corner[i]];
        t.dv[i] = s.dv[corner[i]];
    }
    return t;
}

// MovingTetraMatrix coef3..coef0 (figures.cu:122-293), exact term order, summed from 0
template <class T> static void cubic_coeffs(const MTet<T>& t, T c[4]) {
    V3<T> v0 = t.v[0] - t.v[3], v1 = t.v[1] - t.v[3], v2 = t.v[2] - t.v[3];
    V3<T> dv0 = t.dv[0] - t.dv[3], dv1 = t.dv[1] - t.dv[3], dv2 = t.dv[2] - t.dv[3];
    // SCALE == 1 (flags.h:57-59): multiplying by it is exact and omitted
    T k3 = 0;
    k3 = fmaT(dv2.z * dv1.y, dv0.x, k3);
    k3 = fmaT(-dv1.z * dv2.y, dv0.x, k3);
    k3 = fmaT(-dv2.z * dv0.y, dv1.x, k3);
    k3 = fmaT(dv0.z * dv2.y, dv1.x, k3);
    k3 = fmaT(dv1.z * dv0.y, dv2.x, k3);
    k3 = fmaT(-dv0.z * dv1.y, dv2.x, k3);
    T k2 = 0;
    k2 = fmaT(v2.z * dv1.y, dv0.x, k2);
    k2 = fmaT(dv2.z * v1.y, dv0.x, k2);
    k2 = fmaT(dv2.z * dv1.y, v0.x, k2);
    k2 = fmaT(-v1.z * dv2.y, dv0.x, k2);
    k2 = fmaT(-dv1.z * v2.y, dv0.x, k2);
    k2 = fmaT(-dv1.z * dv2.y, v0.x, k2);
    k2 = fmaT(-v2.z * dv0.y, dv1.x, k2);
    k2 = fmaT(-dv2.z * v0.y, dv1.x, k2);
    k2 = fmaT(-dv2.z * dv0.y, v1.x, k2);
    k2 = fmaT(v0.z * dv2.y, dv1.x, k2);
    k2 = fmaT(dv0.z * v2.y, dv1.x, k2);
    k2 = fmaT(dv0.z * dv2.y, v1.x, k2);
    k2 = fmaT(v1.z * dv0.y, dv2.x, k2);
    k2 = fmaT(dv1.z * v0.y, dv2.x, k2);
    k2 = fmaT(dv1.z * dv0.y, v2.x, k2);
    k2 = fmaT(-v0.z * dv1.y, dv2.x, k2);
    k2 = fmaT(-dv0.z * v1.y, dv2.x, k2);
    k2 = fmaT(-dv0.z * dv1.y, v2.x, k2);
    T k1 = 0;
    k1 = fmaT(v2.z * v1.y, dv0.x, k1);
    k1 = fmaT(v2.z * dv1.y, v0.x, k1);
    k1 = fmaT(dv2.z * v1.y, v0.x, k1);
    k1 = fmaT(-v1.z * v2.y, dv0.x, k1);
    k1 = fmaT(-v1.z * dv2.y, v0.x, k1);
    k1 = fmaT(-dv1.z * v2.y, v0.x, k1);
    k1 = fmaT(-v2.z * v0.y, dv1.x, k1);
    k1 = fmaT(-v2.z * dv0.y, v1.x, k1);
    k1 = fmaT(-dv2.z * v0.y, v1.x, k1);
    k1 = fmaT(v0.z * v2.y, dv1.x, k1);
    k1 = fmaT(v0.z * dv2.y, v1.x, k1);
    k1 = fmaT(dv0.z * v2.y, v1.x, k1);
    k1 = fmaT(v1.z * v0.y, dv2.x, k1);
    k1 = fmaT(v1.z * dv0.y, v2.x, k1);
    k1 = fmaT(dv1.z * v0.y, v2.x, k1);
    k1 = fmaT(-v0.z * v1.y, dv2.x, k1);
    k1 = fmaT(-v0.z * dv1.y, v2.x, k1);
    k1 = fmaT(-dv0.z * v1.y, v2.x, k1);
    T k0 = 0;
    k0 = fmaT(v2.z * v1.y, v0.x, k0);
    k0 = fmaT(-v1.z * v2.y, v0.x, k0);
    k0 = fmaT(-v2.z * v0.y, v1.x, k0);
    k0 = fmaT(v0.z * v2.y, v1.x, k0);
    k0 = fmaT(v1.z * v0.y, v2.x, k0);
    k0 = fmaT(-v0.z * v1.y, v2.x, k0);
    c[0] = k3; c[1] = k2; c[2] = k1; c[3] = k0;
}

static const double EPS = 1e-16;   // EPSILON (flags.h:36-38)

// add_root (collisions_continuous.cu:448-464): keep roots in [-EPS, 1+EPS], at most 3 slots
// the root is converted to the storage type T before the window test (the parameter is T)
template <class T> static inline void add_root(T r[3], T x, int& nr) {
    if (x < -EPS || x > 1 + EPS) return;
    if (nr < 3) r[nr] = x;
    nr++;
}

// solveCubic + computeG + computeH (collisions_continuous.cu:472-613); roots start at -1
template <class T> static void solve_cubic(double a, double b, double c, double d, T r[3]) {
    r[0] = r[1] = r[2] = -1;
    int nr = 0;
    if (a == 0 && b == 0) {
        // linear case: the reference computes -d/c into a local and never stores it
        return;
    } else if (fabs(a) < EPS) {
        double D = fmaT(c, c, -(4.0 * b * d));
        if (D >= 0) {
            D = ccc_sqrt(D);
            double x1 = (-c + D) / (2.0 * b);
            double x2 = (-c - D) / (2.0 * b);
            add_root<T>(r, (T)x1, nr);
            add_root<T>(r, (T)x2, nr);
        }
    } else {
        double f = ((3.0 * c / a) - ((b * b) / (a * a))) / 3.0;
        // computeG
        double b3 = 2 * ccc_cube_hi(b);
        ccc_dd a2dd = ccc_sq_dd(a);
        double a2 = a2dd.hi;
        double a3 = ccc_certmul2_hi(a2dd.hi, a2dd.lo, a);
        double p1 = b3 / a3;
        double p2 = (b * c * 9) / a2;
        double p3 = 27.0 * d / a;
        double g = (p1 - p2 + p3) / 27.0;
        // computeH: pow(g, 2) taken as g * g
        double f3 = ccc_cube_hi(f);
        double h = g * g / 4.0 + f3 / 27.0;
        if (f == 0 && g == 0 && h == 0) {
            float k = (float)(d / a);
            double x1;
            if (k >= 0) x1 = (double)(ccc_cbrtf(k) * -1);
            else x1 = (double)ccc_cbrtf(-k);
            add_root<T>(r, (T)x1, nr);
        } else if (h <= 0) {
            double i = ccc_sqrt(((g * g) / 4.0) - h);
            double j = ccc_cbrt(i);
            double k = ccc_acos(-(g / (2 * i)));
            double L = j * -1;
            double M = ccc_cos(k / 3.0);
            // N = sqrt(3) * sin(k/3) feeds M + N and M - N, and nvcc fuses both (and each
            // result into L * (.) + P); the first root is rounded twice, as compiled
            double sn = ccc_sin(k / 3.0);
            double P = (b / (3.0 * a)) * -1;
            double x1 = (2 * j) * ccc_cos(k / 3.0) - (b / (3.0 * a));
            double x2 = fmaT(L, fmaT(ccc_sqrt(3.0), sn, M), P);
            double x3 = fmaT(L, fmaT(-ccc_sqrt(3.0), sn, M), P);
            add_root<T>(r, (T)x1, nr);
            add_root<T>(r, (T)x2, nr);
            add_root<T>(r, (T)x3, nr);
        } else {
            double R = -(g / 2.0) + ccc_sqrt(h);
            double S, U;
            if (R >= 0) S = ccc_cbrt(R);
            else S = -ccc_cbrt(-R);
            double V = -(g / 2.0) - ccc_sqrt(h);
            if (V >= 0) U = ccc_cbrt(V);
            else U = -ccc_cbrt(-V);
            double x1 = (S + U) - (b / (3.0 * a));
            add_root<T>(r, (T)x1, nr);
        }
    }
}

// is_inside (collisions_continuous.cu:615-637); NaN passes
template <class T> static bool is_inside(V3<T> v0, V3<T> v1, V3<T> v2, V3<T> vt) {
    V3<T> e1 = v0 - v1, e2 = v2 - v1, ep = vt - v1;
    T d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(ep, e1), d21 = dot(ep, e2);
    T denom = fms2(d00, d11, d01, d01);
    T v = fms2(d11, d20, d01, d21) / denom;
    T w = fms2(d00, d21, d01, d20) / denom;
    T u = 1 - v - w;
    if (v < 0 || v > 1) return false;
    if (w < 0 || w > 1) return false;
    if (u < 0 || u > 1) return false;
    return true;
}

template <class T> static inline V3<T> at_time(const MTet<T>& t, int i, T root) { return axpy(t.v[i], t.dv[i], root); }

// filterCollisions (collisions_continuous.cu:640-684)
template <class T> static bool ccd_filter(const MTet<T>& tet, int k, T root) {
    if (root < -(T)EPS) return false;
    V3<T> p0 = at_time(tet, 0, root), p1 = at_time(tet, 1, root), p2 = at_time(tet, 2, root), p3 = at_time(tet, 3, root);
    if (k < 9) {
        V3<T> da = p1 - p0, db = p3 - p2, dc = p2 - p0;
        T s = dot(cross(dc, db), cross(da, db)) / norm2(cross(da, db));
        T p = dot(cross(dc, da), cross(da, db)) / norm2(cross(da, db));
        if (s < 0 || s > 1 || p < 0 || p > 1) return false;
        return true;
    } else if (k < 12) {
        return is_inside(p0, p1, p2, p3);
    }
    return is_inside(p1, p2, p3, p0);
}

struct Hit { int64_t i, j; int k; double t; };

// The continuous narrow phase for one candidate pair (i < j): every emitted row.
// make_moving_triangles .. copy_filtered_collisions (collisions_continuous.cu:14-765).
template <class T>
static void ccd_pair(const T* x0, const T* x1, int64_t i, int64_t j, std::vector<Hit>& out, bool need_filter = true) {
    MTri<T> a = load_mtri(x0, x1, i), b = load_mtri(x0, x1, j);
    Tri<T> sa, sb;
    for (int c = 0; c < 3; ++c) { sa.v[c] = a.v[c]; sb.v[c] = b.v[c]; }
    if (share_vertex(sa, sb)) return;
    for (int k = 0; k < 15; ++k) {
        if (!ccd_subbox(a, b, k)) continue;
        MTet<T> tet = make_tet(a, b, k);
        T c[4];
        cubic_coeffs(tet, c);
        T r[3];
        solve_cubic<T>((double)c[0], (double)c[1], (double)c[2], (double)c[3], r);
        for (int s = 0; s < 3; ++s) {
            T root = r[s];
            if (!(root >= 0 && root <= 1)) continue;     // flatten_cubic_roots 743-764
            if (need_filter && !ccd_filter(tet, k, root)) continue;
            Hit h;
            h.i = i; h.j = j; h.k = k; h.t = (double)root;
            out.push_back(h);
        }
    }
}

// ---------------------------------------------------------------------------------------
// Impulses (collisions_impulses.cu)
// ---------------------------------------------------------------------------------------

static const double THICKNESS = 2e-3;   // collisions_impulses.cu:12-14

template <class T> static inline V3<T> vnormalize(V3<T> a) {
    // normalize(double3) = a * rsqrt(|a|^2) (utils.cu:91-93); taken as a * (1 / sqrt(|a|^2))
    T n = norm2(a);
    T inv = (T)1 / (T)sqrt((double)n);
    return a * inv;
}

// masses2quad (collisions_impulses.cu:24-123): the four per-corner masses of the tetrahedron
template <class T> static inline void mass_quad(const T* masses, int64_t i, int64_t j, int k, T q[4]) {
    int side[4], corner[4];
    type_points(k, side, corner);
    for (int p = 0; p < 4; ++p) q[p] = masses[(side[p] ? j : i) * 3 + corner[p]];
}

template <class T> struct Contact {
    V3<T> n;    // normal direction after orientation (and inversion for types 12..14)
    T vn;       // normal relative velocity
    T m0, m1;   // mass pair
};

// compute_coeficients_and_directions (collisions_impulses.cu:162-543)
template <class T> static Contact<T> contact(const MTet<T>& tet, int k, T root, const T q[4]) {
    Contact<T> ct;
    MTet<T> thz;
    for (int i = 0; i < 4; ++i) { thz.v[i] = at_time(tet, i, root); thz.dv[i] = tet.dv[i]; }
    if (k < 9) {
        // compute_coeficients_edge_edge (306-328)
        V3<T> da = thz.v[1] - thz.v[0], db = thz.v[3] - thz.v[2], dc = thz.v[2] - thz.v[0];
        T denom = norm2(cross(da, db));
        T s, t;
        if (fabs((double)denom) < 1e-15) { s = (T)0.5; t = (T)0.5; }
        else {
            s = dot(cross(dc, db), cross(da, db)) / norm2(cross(da, db));
            t = dot(cross(dc, da), cross(da, db)) / norm2(cross(da, db));
        }
        // compute_normal_direction_edge_edge (330-447), on the t = 0 tetrahedron
        const V3<T>* v = tet.v;
        const V3<T>* dv = tet.dv;
        V3<T> p0 = axpy(v[0], v[1] - v[0], s);
        V3<T> p1 = axpy(v[2], v[3] - v[2], t);
        V3<T> dp0 = axpy(dv[0], dv[1] - dv[0], s);
        V3<T> dp1 = axpy(dv[2], dv[3] - dv[2], t);
        V3<T> c0 = axpy(v[0], dv[0], root), c1 = axpy(v[1], dv[1], root), c2 = axpy(v[2], dv[2], root);
        V3<T> nd = vnormalize(cross(c1 - c0, c2 - c0));
        if (dot(p1 - p0, nd) < 0) nd = nd * (T)-1;
        ct.n = nd;
        ct.vn = dot(dp1 - dp0, nd);
        // compute_masses_edge_edge (449-454)
        ct.m0 = fmaT(q[0], 1 - s, q[1] * s);
        ct.m1 = fmaT(q[2], 1 - t, q[3] * t);
        return ct;
    }
    // triangle-vertex: types 9..11 face = points 0,1,2, vertex = 3; types 12..14 face =
    // points 1,2,3, vertex = 0 and the normal is inverted at the end (503-535)
    bool inv = k >= 12;
    int f0 = inv ? 1 : 0, f1 = inv ? 2 : 1, f2 = inv ? 3 : 2, fv = inv ? 0 : 3;
    // compute_coeficients_triangle_vertex (162-193), at the collision time
    V3<T> e1 = thz.v[f0] - thz.v[f1], e2 = thz.v[f2] - thz.v[f1], ep = thz.v[fv] - thz.v[f1];
    T d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(ep, e1), d21 = dot(ep, e2);
    T denom = fms2(d00, d11, d01, d01);
    T u, w, vv;
    if (fabs((double)denom) < 1e-15) { u = (T)(1. / 3.); w = (T)(1. / 3.); }
    else {
        u = fms2(d11, d20, d01, d21) / denom;
        w = fms2(d00, d21, d01, d20) / denom;
    }
    vv = 1 - u - w;
    // compute_normal_direction_triangle_vertex (196-304)
    const V3<T>* v = tet.v;
    const V3<T>* dv = tet.dv;
    V3<T> pt = lin3(v[f0], u, v[f1], vv, v[f2], w);
    V3<T> dpt = lin3(dv[f0], u, dv[f1], vv, dv[f2], w);
    V3<T> c0 = axpy(v[f0], dv[f0], root), c1 = axpy(v[f1], dv[f1], root), c2 = axpy(v[f2], dv[f2], root);
    V3<T> nd = vnormalize(cross(c1 - c0, c2 - c0));
    if (dot(v[fv] - pt, nd) < 0) nd = nd * (T)-1;
    ct.vn = dot(dv[fv] - dpt, nd);
    if (inv) nd = nd * (T)-1;
    ct.n = nd;
    // compute_masses_triangle_vertex (456-468)
    if (inv) {
        ct.m0 = q[0];
        ct.m1 = fmaT(q[3], w, fmaT(q[1], u, q[2] * vv));
    } else {
        ct.m0 = fmaT(q[2], w, fmaT(q[0], u, q[1] * vv));
        ct.m1 = q[3];
    }
    return ct;
}

// extrapolate_impulses + extrapolate_impulses_dv (collisions_impulses.cu:609-1067):
// accumulate into dv/dx (F,3,3) and counters (F,3).
template <class T>
static void apply_impulse(const MTet<T>& tet, int64_t i, int64_t j, int k, T root, const Contact<T>& ct, T* dv_out,
                          T* dx_out, int32_t* cnt_out) {
    T offset;
    if (fabs((double)ct.vn) < 1e-15) offset = (T)0.1;
    else offset = (T)((2 * THICKNESS) / (double)(-ct.vn));
    offset = (T)fmin(fmax((double)offset, 0.), 1.);
    T msum = ct.m0 + ct.m1;
    T mf0, mf1;
    if (fabs((double)msum) < 1e-15) { mf0 = (T)0.5; mf1 = (T)0.5; }
    else { mf0 = ct.m0 / msum; mf1 = 1 - mf0; }
    T mag0 = ct.vn * mf1;
    T mag1 = -ct.vn * mf0;
    T mags[4];
    if (k < 9) { mags[0] = mag0; mags[1] = mag0; mags[2] = mag1; mags[3] = mag1; }
    else if (k < 12) { mags[0] = mag0; mags[1] = mag0; mags[2] = mag0; mags[3] = mag1; }
    else { mags[0] = mag0; mags[1] = mag1; mags[2] = mag1; mags[3] = mag1; }
    T ro = (T)fmax((double)(root - offset), 0.);
    int side[4], corner[4];
    type_points(k, side, corner);
    for (int p = 0; p < 4; ++p) {
        V3<T> imp = ct.n * mags[p];
        V3<T> nv = tet.dv[p] + imp;
        V3<T> idx = (nv - tet.dv[p]) * (1 - ro);
        int64_t tri = side[p] ? j : i;
        T* d = dv_out + tri * 9 + corner[p] * 3;
        d[0] += imp.x; d[1] += imp.y; d[2] += imp.z;
        T* x = dx_out + tri * 9 + corner[p] * 3;
        x[0] += idx.x; x[1] += idx.y; x[2] += idx.z;
        cnt_out[tri * 3 + corner[p]] += 1;
    }
}

// ---------------------------------------------------------------------------------------
// Proximity (proximity_static.cu)
// ---------------------------------------------------------------------------------------

// static sub-boxes with threshold (11-98)
template <class T> static bool prox_subbox(const Tri<T>& a, const Tri<T>& b, int k, T th) {
    Box<T> b0, b1;
    if (k < 9) {
        int e0 = k / 3, e1 = k % 3;
        b0 = merge(svbox(a, EA[e0]), svbox(a, EB[e0]));
        b1 = merge(svbox(b, EA[e1]), svbox(b, EB[e1]));
    } else if (k < 12) {
        b0 = tri_box(a);
        b1 = svbox(b, k - 9);
    } else {
        b0 = svbox(a, k - 12);
        b1 = tri_box(b);
    }
    return overlap(b0, b1, th);
}

// vec_sq_diff returns float (utils.cu:57-61); sqrt is then taken in float
template <class T> static inline float sq_diff_f(V3<T> a, V3<T> b) { V3<T> d = a - b; return (float)dot(d, d); }

// distance_point_to_segment (205-228)
template <class T> static void pt_seg(V3<T> p, V3<T> a, V3<T> b, T dc[3], bool set_s, T second) {
    V3<T> ab = b - a, ap = p - a;
    T t = dot(ap, ab) / dot(ab, ab);
    if (t < 0.0) t = 0.0;
    if (t > 1.0) t = 1.0;
    V3<T> c = mk<T>(fmaT(t, ab.x, a.x), fmaT(t, ab.y, a.y), fmaT(t, ab.z, a.z));
    T nd = (T)sqrtf(sq_diff_f(p, c));
    if (nd < dc[0]) {
        dc[0] = nd;
        if (set_s) { dc[1] = t; dc[2] = second; }
        else { dc[2] = t; dc[1] = second; }
    }
}

// compute_distance_edge_edge (239-332) / compute_distance_triangle_node (334-433):
// returns the distance, -1 when the closest points fall outside the features
template <class T> static T prox_distance(const Tri<T>& a, const Tri<T>& b, int k) {
    int side[4], corner[4];
    type_points(k, side, corner);
    V3<T> v[4];
    for (int p = 0; p < 4; ++p) v[p] = (side[p] ? b : a).v[corner[p]];
    if (k < 9) {
        V3<T> da = v[1] - v[0], db = v[3] - v[2], dc = v[2] - v[0];
        T s = dot(cross(dc, db), cross(da, db)) / norm2(cross(da, db));
        T t = dot(cross(dc, da), cross(da, db)) / norm2(cross(da, db));
        if (s != s || t != t) {
            T d3[3] = {(T)FLT_MAX, (T)-1., (T)-1.};
            pt_seg(v[0], v[2], v[3], d3, false, (T)0.);
            pt_seg(v[1], v[2], v[3], d3, false, (T)1.);
            pt_seg(v[2], v[0], v[1], d3, true, (T)0.);
            pt_seg(v[3], v[0], v[1], d3, true, (T)1.);
            s = d3[1];
            t = d3[2];
        }
        bool sv = (s >= 0 && s <= 1), tv = (t >= 0 && t <= 1);
        if (!sv || !tv) return (T)-1;
        return (T)sqrtf(sq_diff_f(axpy(v[0], da, s), axpy(v[2], db, t)));
    }
    int f0 = k < 12 ? 0 : 1, f1 = k < 12 ? 1 : 2, f2 = k < 12 ? 2 : 3, fv = k < 12 ? 3 : 0;
    V3<T> e1 = v[f0] - v[f1], e2 = v[f2] - v[f1], ep = v[fv] - v[f1];
    T d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(ep, e1), d21 = dot(ep, e2);
    T denom = fms2(d00, d11, d01, d01);
    T u = fms2(d11, d20, d01, d21) / denom;
    T w = fms2(d00, d21, d01, d20) / denom;
    T vv = 1 - w - u;
    bool ok = (vv >= 0 && vv <= 1) && (w >= 0 && w <= 1) && (u >= 0 && u <= 1);
    if (!ok) return (T)-1;
    V3<T> pt = lin3(v[f0], u, v[f1], vv, v[f2], w);
    return (T)sqrtf(sq_diff_f(v[fv], pt));
}

}  // namespace orc

using namespace orc;

// =======================================================================================
// C entry points (ctypes).  dtype: 0 = float32, 1 = float64.  All tensors are one mesh.
// Return values >= 0 are counts; -1 = capacity overflow or malformed tree.
// =======================================================================================
#define ORC_API extern "C"

// Self-check of the double-double short paths (ccc_ddmul.h): n operand sets drawn by a
// splitmix64 stream from `seed` in one of four families (0: random significands over
// exponents +-600; 1: significands of 1..30 bits, which make exact and tied products;
// 2: neighbours of powers of two; 3: zeros, signed zeros, subnormals, huge values, inf and
// NaN mixed in).  Each set checks certifiedMul<1,1,2> (both terms) and the leading term of
// certifiedMul<2,1,2> against the bin algorithm.  out: [mismatches, short-path uses].
static uint64_t sm64(uint64_t& s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static double draw(uint64_t& st, int family) {
    uint64_t r = sm64(st);
    int sign = (int)(r & 1);
    int ex = (int)((r >> 1) % 1201) - 600;
    uint64_t mant = sm64(st) & 0x000fffffffffffffull;
    if (family == 1) {
        int bits = 1 + (int)((r >> 20) % 30);
        mant &= ~((1ull << (52 - bits + 1)) - 1) & 0x000fffffffffffffull;
    } else if (family == 2) {
        uint64_t k = (r >> 24) % 4;
        mant = (r >> 40) & 1 ? k : (0x000fffffffffffffull - k);
        ex = (int)((r >> 28) % 401) - 200;
    } else if (family == 3) {
        switch ((r >> 30) % 8) {
            case 0: return sign ? -0.0 : 0.0;
            case 1: return ccc_dfrombits(sm64(st) & 0x000fffffffffffffull);          // subnormal
            case 2: return ccc_dfrombits(((uint64_t)(2000 + (r >> 33) % 46) << 52) | mant);
            case 3: return sign ? -INFINITY : INFINITY;
            case 4: return NAN;
            default: ex = (int)((r >> 1) % 2001) - 1000;
        }
    }
    uint64_t u = ((uint64_t)sign << 63) | ((uint64_t)(ex + 1023) << 52) | mant;
    return ccc_dfrombits(u);
}
static bool same(double a, double b) { return ccc_dbits(a) == ccc_dbits(b) || (a != a && b != b); }

ORC_API int orc_ddmul_check(int64_t n, uint64_t seed, int family, int64_t* out) {
    int64_t bad = 0, fast = 0;
#pragma omp parallel for reduction(+ : bad, fast) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        uint64_t st = seed * 0x100000001b3ull + (uint64_t)i * 0x9e3779b97f4a7c15ull;
        double x = draw(st, family), y = draw(st, family), z = draw(st, family);
        ccc_dd g = ccc_certmul_k<1>(x, 0.0, y);
        ccc_dd f = ccc_certmul1(x, y);
        if (!same(g.hi, f.hi) || !same(g.lo, f.lo)) ++bad;
        if (ccc_dbits(f.hi) == ccc_dbits(x * y) && !(x == 0.0 || y == 0.0)) ++fast;
        // K = 2 on a normalised expansion (a square, as in the solver) and on (x, lo) pairs
        ccc_dd sq = ccc_certmul_k<1>(x, 0.0, x);
        if (!same(ccc_certmul_k<2>(sq.hi, sq.lo, z).hi, ccc_certmul2_hi(sq.hi, sq.lo, z))) ++bad;
        ccc_dd pr = ccc_certmul_k<1>(y, 0.0, z);
        if (!same(ccc_certmul_k<2>(pr.hi, pr.lo, x).hi, ccc_certmul2_hi(pr.hi, pr.lo, x))) ++bad;
        if (!same(ccc_cube_hi(x), ccc_certmul_k<2>(sq.hi, sq.lo, x).hi)) ++bad;
    }
    out[0] = bad;
    out[1] = fast;
    return 0;
}

ORC_API int orc_bvh(int dtype, const void* tri, const void* tri_next, int n, int spatial, void* bboxes, int64_t* tree,
            uint32_t* codes) {
    if (n < 2) return -1;
    if (dtype == 0) build<float>((const float*)tri, (const float*)tri_next, n, spatial, (float*)bboxes, tree, codes);
    else build<double>((const double*)tri, (const double*)tri_next, n, spatial, (double*)bboxes, tree, codes);
    return 0;
}

template <class T>
static int64_t cand_impl(const T* bboxes, const int64_t* tree, int n, double th, const uint8_t* mask, int64_t* out,
                         int64_t cap, int nthreads) {
    Forest<T> f;
    import_tree(bboxes, tree, n, f);
    if (!f.ok) return -1;
    std::vector<int64_t> pairs;
    int64_t c = candidates(f, (T)th, mask, pairs, nthreads);
    if (c < 0) return -1;
    int64_t w = std::min(c, cap);
    if (out) memcpy(out, pairs.data(), sizeof(int64_t) * 2 * w);
    return c;
}

// All candidate pairs (min id, max id) of one mesh; returns the total count (only `cap`
// rows are written).
ORC_API int64_t orc_candidates(int dtype, const void* bboxes, const int64_t* tree, int n, double th, const uint8_t* mask,
                       int64_t* out, int64_t cap, int nthreads) {
    if (dtype == 0) return cand_impl<float>((const float*)bboxes, tree, n, th, mask, out, cap, nthreads);
    return cand_impl<double>((const double*)bboxes, tree, n, th, mask, out, cap, nthreads);
}

template <class T>
static int64_t static_impl(const T* bboxes, const int64_t* tree, const T* tri, int n, double th_f, int64_t* out,
                           int64_t cap, int nthreads) {
    Forest<T> f;
    import_tree(bboxes, tree, n, f);
    if (!f.ok) return -1;
    // the reference passes the float threshold into a T-typed kernel argument
    T th = (T)(float)th_f;
    std::vector<int64_t> pairs;
    if (candidates(f, th, nullptr, pairs, nthreads) < 0) return -1;
    int64_t nc = (int64_t)pairs.size() / 2;
    std::vector<uint8_t> keep(nc, 0);
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthr(nthreads))
    for (int64_t c = 0; c < nc; ++c) {
        Tri<T> a = load_tri(tri, pairs[2 * c]), b = load_tri(tri, pairs[2 * c + 1]);
        keep[c] = sat(a, b, th) && !(count_shared(a, b) > 0);
    }
    int64_t w = 0;
    for (int64_t c = 0; c < nc; ++c) {
        if (!keep[c]) continue;
        if (w < cap) { out[2 * w] = pairs[2 * c]; out[2 * w + 1] = pairs[2 * c + 1]; }
        ++w;
    }
    return w;
}

// find_collisions (collisions_static.cu:206-342): intersecting pairs (i, j)
ORC_API int64_t orc_find_collisions(int dtype, const void* bboxes, const int64_t* tree, const void* tri, int n, double th,
                            int64_t* out, int64_t cap, int nthreads) {
    if (dtype == 0) return static_impl<float>((const float*)bboxes, tree, (const float*)tri, n, th, out, cap, nthreads);
    return static_impl<double>((const double*)bboxes, tree, (const double*)tri, n, th, out, cap, nthreads);
}

// ---------------------------------------------------------------------------------------
// Triangle-edge helpers (collisions_static.cu:345-942, icontour.cu:11-281)
// ---------------------------------------------------------------------------------------

// hasVertex (figures.cu:598-609): exact coordinate equality with one of the corners
template <class T> static inline bool has_vertex(const Tri<T>& t, V3<T> p) {
    return veq(t.v[0], p) || veq(t.v[1], p) || veq(t.v[2], p);
}

// Sub-test cid (0..5) of a pair (a, b): cid < 3 takes edge cid % 3 of a against face b,
// cid >= 3 edge cid % 3 of b against face a; edge e runs from corner e to corner (e + 1) % 3
// (collectTEIntersections / collectTECandidates, collisions_static.cu:465-586).
template <class T>
static inline void te_edge(const Tri<T>& a, const Tri<T>& b, int cid, Tri<T>& face, V3<T>& p0, V3<T>& p1, int& e) {
    const Tri<T>& t1 = cid < 3 ? a : b;
    face = cid < 3 ? b : a;
    e = cid % 3;
    p0 = t1.v[e];
    p1 = t1.v[(e + 1) % 3];
}

// addTECollsion (collisions_static.cu:345-462): 1 and (flag, coefficient) when edge p0-p1
// crosses the face; flag 0 / coefficient 0 for an edge that starts at a corner of the face
// (cid < 3 only), -1 / the edge parameter t of the crossing otherwise.  NaN passes the
// range tests, as in the reference.
template <class T>
static inline int te_intersect(const Tri<T>& face, V3<T> p0, V3<T> p1, int cid, int& flag, T& coef) {
    V3<T> e1 = face.v[1] - face.v[0], e2 = face.v[2] - face.v[0];
    V3<T> nrm = vnormalize(cross(e1, e2));
    bool s0 = has_vertex(face, p0), s1 = has_vertex(face, p1);
    if (s0 || s1) {
        if (cid > 2 || !s0) return 0;
        flag = 0;
        coef = (T)0;
        return 1;
    }
    V3<T> dir = p1 - p0;
    T en = dot(dir, nrm);
    if (en == 0) return 0;
    T d = dot(nrm, face.v[0]);
    T t = (d - dot(nrm, p0)) / en;
    if (t < 0 || t > 1) return 0;
    V3<T> x = axpy(p0, dir, t);
    V3<T> ep = x - face.v[0];
    // the reference's float build contracts the dot products of the face's edges as
    // fma(z, z', fma(y, y', x x')); its double build, and both builds for the ones with ep,
    // as dot()
    const bool f32 = sizeof(T) == 4;
    T d00 = f32 ? dot_zyx(e1, e1) : dot(e1, e1), d01 = f32 ? dot_zyx(e1, e2) : dot(e1, e2),
      d11 = f32 ? dot_zyx(e2, e2) : dot(e2, e2), d20 = dot(ep, e1), d21 = dot(ep, e2);
    T denom = fms2(d00, d11, d01, d01);
    if ((double)denom < 1e-15) return 0;
    T v = fms2(d11, d20, d01, d21) / denom;
    T w = fms2(d00, d21, d01, d20) / denom;
    T u = (T)(1.0 - (double)v - (double)w);  // `1.0 - v - w`: a double expression for float T
    if (u < 0 || v < 0 || w < 0) return 0;
    flag = -1;
    coef = t;
    return 1;
}

// collectTECandidates / collectTECandidates2 (collisions_static.cu:525-586, icontour.cu:11-110):
// bit 0 = the sub-test is listed, bit 1 = it is listed as a loop node (edge starting at a
// corner of the face).  The box test compares the face's box with the box of the face's
// own edge e (not the tested edge), as the reference does.
template <class T> static inline int te_candidate(const Tri<T>& face, V3<T> p0, V3<T> p1, int cid, int e) {
    if (has_vertex(face, p0)) return cid < 3 ? 3 : 0;
    if (has_vertex(face, p1)) return 0;
    const V3<T>& q0 = face.v[e];
    const V3<T>& q1 = face.v[(e + 1) % 3];
    Box<T> b1;
    b1.lo = mk<T>(fmn(q0.x, q1.x), fmn(q0.y, q1.y), fmn(q0.z, q1.z));
    b1.hi = mk<T>(fmx(q0.x, q1.x), fmx(q0.y, q1.y), fmx(q0.z, q1.z));
    return overlap(tri_box(face), b1, (T)0) ? 1 : 0;
}

// find_triangle_edge_collisions (op 0), _candidates (op 1), _candidates2 (op 2)
// (collisions_static.cu:588-942, icontour.cu:113-281): candidate pairs that intersect
// (separating axes, threshold 0) sharing at most `allow` vertices (0 for op 0, 1 otherwise),
// then the six edge sub-tests of each.  Ops 0 / 1 write rows (i, j, cid, flag) (+ the
// coefficient, op 0) and return the row count; op 2 writes (i, j) and (mask_x, mask_y) per
// pair and returns the pair count.  At most `cap` rows are written.
template <class T>
static int64_t te_impl(const T* bboxes, const int64_t* tree, const T* tri, int n, int op, int64_t* rows, T* coefs,
                       int32_t* masks, int64_t cap, int nthreads) {
    Forest<T> f;
    import_tree(bboxes, tree, n, f);
    if (!f.ok) return -1;
    std::vector<int64_t> pairs;
    if (candidates(f, (T)0, nullptr, pairs, nthreads) < 0) return -1;
    const int allow = op == 0 ? 0 : 1;
    int64_t nc = (int64_t)pairs.size() / 2;
    int64_t w = 0;
    for (int64_t c = 0; c < nc; ++c) {
        int64_t i = pairs[2 * c], j = pairs[2 * c + 1];
        Tri<T> a = load_tri(tri, i), b = load_tri(tri, j);
        if (!(sat(a, b, (T)0) && !(count_shared(a, b) > allow))) continue;
        int32_t mx = 0, my = 0;
        for (int cid = 0; cid < 6; ++cid) {
            Tri<T> face;
            V3<T> p0, p1;
            int e;
            te_edge(a, b, cid, face, p0, p1, e);
            int flag = -1;
            T coef = (T)-1;
            if (op == 0) {
                if (!te_intersect(face, p0, p1, cid, flag, coef)) continue;
            } else {
                int r = te_candidate(face, p0, p1, cid, e);
                if (!r) continue;
                flag = (r & 2) ? 0 : -1;
                if (op == 2) {
                    mx |= 1 << cid;
                    if (r & 2) my |= 1 << cid;
                    continue;
                }
            }
            if (w < cap) {
                rows[4 * w + 0] = i; rows[4 * w + 1] = j; rows[4 * w + 2] = cid; rows[4 * w + 3] = flag;
                if (coefs) coefs[w] = coef;
            }
            ++w;
        }
        if (op == 2) {
            if (w < cap) {
                rows[2 * w] = i; rows[2 * w + 1] = j;
                masks[2 * w] = mx; masks[2 * w + 1] = my;
            }
            ++w;
        }
    }
    return w;
}

ORC_API int64_t orc_triangle_edge(int dtype, const void* bboxes, const int64_t* tree, const void* tri, int n, int op,
                                  int64_t* rows, void* coefs, int32_t* masks, int64_t cap, int nthreads) {
    if (op < 0 || op > 2) return -1;
    if (dtype == 0)
        return te_impl<float>((const float*)bboxes, tree, (const float*)tri, n, op, rows, (float*)coefs, masks, cap,
                              nthreads);
    return te_impl<double>((const double*)bboxes, tree, (const double*)tri, n, op, rows, (double*)coefs, masks, cap,
                           nthreads);
}

template <class T>
static int64_t ccd_impl(const T* bboxes, const int64_t* tree, const T* x0, const T* x1, int n, const uint8_t* mask,
                        int64_t* rows, double* times, int64_t cap, int nthreads, int filter) {
    Forest<T> f;
    import_tree(bboxes, tree, n, f);
    if (!f.ok) return -1;
    std::vector<int64_t> pairs;
    if (candidates(f, (T)0, mask, pairs, nthreads) < 0) return -1;
    int64_t nc = (int64_t)pairs.size() / 2;
    std::vector<Hit> hits;
#ifdef _OPENMP
    int nt = nthr(nthreads);
    std::vector<std::vector<Hit>> loc(nt);
#pragma omp parallel num_threads(nt)
    {
        std::vector<Hit>& mine = loc[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 1024)
        for (int64_t c = 0; c < nc; ++c) ccd_pair(x0, x1, pairs[2 * c], pairs[2 * c + 1], mine, filter != 0);
    }
    for (auto& v : loc) hits.insert(hits.end(), v.begin(), v.end());
#else
    for (int64_t c = 0; c < nc; ++c) ccd_pair(x0, x1, pairs[2 * c], pairs[2 * c + 1], hits, filter != 0);
#endif
    int64_t w = 0;
    for (const Hit& h : hits) {
        if (w < cap) {
            rows[3 * w] = h.i; rows[3 * w + 1] = h.j; rows[3 * w + 2] = h.k;
            if (times) times[w] = h.t;
        }
        ++w;
    }
    return w;
}

// find_collisions_continuous (collisions_continuous.cu:814-1076) and its partial variant
// (1103-1376) when mask != NULL: rows (i, j, k) and times of impact (as double).
ORC_API int64_t orc_ccd(int dtype, const void* bboxes, const int64_t* tree, const void* x0, const void* x1, int n,
                const uint8_t* mask, int64_t* rows, double* times, int64_t cap, int nthreads) {
    if (dtype == 0)
        return ccd_impl<float>((const float*)bboxes, tree, (const float*)x0, (const float*)x1, n, mask, rows, times, cap,
                               nthreads, 1);
    return ccd_impl<double>((const double*)bboxes, tree, (const double*)x0, (const double*)x1, n, mask, rows, times,
                            cap, nthreads, 1);
}

template <class T>
static int64_t mincol_impl(const T* bboxes, const int64_t* tree, const T* x0, const T* x1, int n, int64_t* rows,
                           int64_t cap) {
    Forest<T> f;
    import_tree(bboxes, tree, n, f);
    if (!f.ok) return -1;
    std::vector<int64_t> pairs;
    if (candidates(f, (T)0, nullptr, pairs, 1) < 0) return -1;
    int64_t w = 0;
    for (size_t c = 0; c < pairs.size() / 2; ++c) {
        MTri<T> a = load_mtri(x0, x1, pairs[2 * c]), b = load_mtri(x0, x1, pairs[2 * c + 1]);
        Tri<T> sa, sb;
        for (int q = 0; q < 3; ++q) { sa.v[q] = a.v[q]; sb.v[q] = b.v[q]; }
        if (share_vertex(sa, sb)) continue;
        for (int k = 0; k < 15; ++k) {
            if (!ccd_subbox(a, b, k)) continue;
            if (w < cap) { rows[3 * w] = pairs[2 * c]; rows[3 * w + 1] = pairs[2 * c + 1]; rows[3 * w + 2] = k; }
            ++w;
        }
    }
    return w;
}

// find_mincol_cand (collisions_continuous.cu:1379-1519): (i, j, k) sub-tests whose swept
// sub-boxes overlap
ORC_API int64_t orc_mincol(int dtype, const void* bboxes, const int64_t* tree, const void* x0, const void* x1, int n,
                   int64_t* rows, int64_t cap) {
    if (dtype == 0) return mincol_impl<float>((const float*)bboxes, tree, (const float*)x0, (const float*)x1, n, rows, cap);
    return mincol_impl<double>((const double*)bboxes, tree, (const double*)x0, (const double*)x1, n, rows, cap);
}

template <class T>
static void impulses_from_rows(const T* x0, const T* x1, const T* masses, const int64_t* rows, const double* times,
                               int64_t nrows, T* dv, T* dx, int32_t* cnt) {
    for (int64_t r = 0; r < nrows; ++r) {
        int64_t i = rows[3 * r], j = rows[3 * r + 1];
        int k = (int)rows[3 * r + 2];
        T root = (T)times[r];
        MTri<T> a = load_mtri(x0, x1, i), b = load_mtri(x0, x1, j);
        MTet<T> tet = make_tet(a, b, k);
        T q[4];
        mass_quad(masses, i, j, k, q);
        Contact<T> ct = contact(tet, k, root, q);
        apply_impulse(tet, i, j, k, root, ct, dv, dx, cnt);
    }
}

// compute_impulses_from_collisions (collisions_impulses.cu:1738-1880): rows must be valid
ORC_API int orc_impulses_from_rows(int dtype, const void* x0, const void* x1, const void* masses, int n, const int64_t* rows,
                           const double* times, int64_t nrows, void* dv, void* dx, int32_t* cnt) {
    (void)n;
    if (dtype == 0)
        impulses_from_rows<float>((const float*)x0, (const float*)x1, (const float*)masses, rows, times, nrows,
                                  (float*)dv, (float*)dx, cnt);
    else
        impulses_from_rows<double>((const double*)x0, (const double*)x1, (const double*)masses, rows, times, nrows,
                                   (double*)dv, (double*)dx, cnt);
    return 0;
}

// compute_impulses (collisions_impulses.cu:1069-1397) and its partial variant
// (1402-1734): CCD rows, then impulses accumulated per triangle corner.
// Returns the number of contacts.
ORC_API int64_t orc_impulses(int dtype, const void* bboxes, const int64_t* tree, const void* x0, const void* x1,
                     const void* masses, int n, const uint8_t* mask, void* dv, void* dx, int32_t* cnt, int nthreads) {
    int64_t cap = 1 << 26;
    std::vector<int64_t> rows;
    std::vector<double> times;
    int64_t c = orc_ccd(dtype, bboxes, tree, x0, x1, n, mask, nullptr, nullptr, 0, nthreads);
    if (c < 0) return c;
    rows.resize(3 * (size_t)std::max<int64_t>(c, 1));
    times.resize(std::max<int64_t>(c, 1));
    c = orc_ccd(dtype, bboxes, tree, x0, x1, n, mask, rows.data(), times.data(), std::min(c, cap), nthreads);
    orc_impulses_from_rows(dtype, x0, x1, masses, n, rows.data(), times.data(), c, dv, dx, cnt);
    return c;
}

// ---------------------------------------------------------------------------------------
// Impulse loop of the resident engine (no counterpart in the reference, whose caller owns
// the loop): collision check with impulses, per-vertex average of the corner corrections,
// repeat until a check finds no contact or max_iter iterations.  Impulses are summed per
// vertex in 2^-56 fixed point (int64), so the sums do not depend on contact order and the
// GPU engine's loop matches this one bit for bit.
// ---------------------------------------------------------------------------------------
static const double FIX_SCALE = 72057594037927936.0;   // 2^56
static const double FIX_INV = 1.3877787807814457e-17;  // 2^-56

static inline bool to_fix(double x, int64_t& q) {
    if (!(fabs(x) < 64.0)) return false;
    q = (int64_t)nearbyint(x * FIX_SCALE);
    return true;
}

template <class T>
static void gather_soup(const T* verts, const int32_t* faces, int64_t F, T* soup) {
    for (int64_t f = 0; f < F; ++f)
        for (int c = 0; c < 3; ++c)
            for (int d = 0; d < 3; ++d) soup[f * 9 + c * 3 + d] = verts[(int64_t)faces[f * 3 + c] * 3 + d];
}

// one contact's four point impulses into the fixed-point vertex sums (8 words per vertex:
// dx xyz, dv xyz, count); returns false if a value was non-finite or out of range
template <class T>
static bool loop_contact(const MTet<T>& tet, int64_t i, int64_t j, int k, T root, const Contact<T>& ct,
                         const int32_t* faces, int64_t* acc) {
    T offset;
    if (fabs((double)ct.vn) < 1e-15) offset = (T)0.1;
    else offset = (T)((2 * THICKNESS) / (double)(-ct.vn));
    offset = (T)fmin(fmax((double)offset, 0.), 1.);
    T msum = ct.m0 + ct.m1;
    T mf0, mf1;
    if (fabs((double)msum) < 1e-15) { mf0 = (T)0.5; mf1 = (T)0.5; }
    else { mf0 = ct.m0 / msum; mf1 = 1 - mf0; }
    T mag0 = ct.vn * mf1;
    T mag1 = -ct.vn * mf0;
    T mags[4];
    if (k < 9) { mags[0] = mag0; mags[1] = mag0; mags[2] = mag1; mags[3] = mag1; }
    else if (k < 12) { mags[0] = mag0; mags[1] = mag0; mags[2] = mag0; mags[3] = mag1; }
    else { mags[0] = mag0; mags[1] = mag1; mags[2] = mag1; mags[3] = mag1; }
    T keep = 1 - (T)fmax((double)(root - offset), 0.);
    int side[4], corner[4];
    type_points(k, side, corner);
    bool all_ok = true;
    for (int p = 0; p < 4; ++p) {
        V3<T> imp = ct.n * mags[p];
        V3<T> nv = tet.dv[p] + imp;
        V3<T> idx = (nv - tet.dv[p]) * keep;
        int64_t q[6];
        bool ok = to_fix((double)idx.x, q[0]) && to_fix((double)idx.y, q[1]) && to_fix((double)idx.z, q[2]) &&
                  to_fix((double)imp.x, q[3]) && to_fix((double)imp.y, q[4]) && to_fix((double)imp.z, q[5]);
        if (!ok) {
            all_ok = false;
            continue;
        }
        int64_t tri = side[p] ? j : i;
        int64_t* a = acc + (int64_t)faces[tri * 3 + corner[p]] * 8;
        for (int c = 0; c < 6; ++c) a[c] = (int64_t)((uint64_t)a[c] + (uint64_t)q[c]);
        a[6] += 1;
    }
    return all_ok;
}

template <class T>
static int loop_impl(const T* verts0, T* verts1, T* vel, const int32_t* faces, const T* masses, int64_t F, int64_t V,
                     int max_iter, int32_t* contacts_per_iter, int nthreads, int* converged) {
    std::vector<T> x0(F * 9), x1(F * 9), bb((2 * F - 1) * 6);
    std::vector<int64_t> tree((2 * F - 1) * 4);
    std::vector<int64_t> acc(V * 8);
    gather_soup(verts0, faces, F, x0.data());
    int it = 0;
    *converged = 0;
    for (;;) {
        gather_soup(verts1, faces, F, x1.data());
        build<T>(x0.data(), x1.data(), (int)F, 1, bb.data(), tree.data(), nullptr);
        int64_t c = ccd_impl<T>(bb.data(), tree.data(), x0.data(), x1.data(), (int)F, nullptr, nullptr, nullptr, 0,
                                nthreads, 1);
        if (c < 0) return -1;
        if (contacts_per_iter) contacts_per_iter[it] = (int32_t)c;
        if (c == 0) {
            *converged = 1;
            break;
        }
        std::vector<int64_t> rows(3 * c);
        std::vector<double> times(c);
        ccd_impl<T>(bb.data(), tree.data(), x0.data(), x1.data(), (int)F, nullptr, rows.data(), times.data(), c,
                    nthreads, 1);
        std::fill(acc.begin(), acc.end(), 0);
        for (int64_t r = 0; r < c; ++r) {
            int64_t i = rows[3 * r], j = rows[3 * r + 1];
            int k = (int)rows[3 * r + 2];
            T root = (T)times[r];
            MTri<T> a = load_mtri(x0.data(), x1.data(), i), b = load_mtri(x0.data(), x1.data(), j);
            MTet<T> tet = make_tet(a, b, k);
            T q[4];
            mass_quad(masses, i, j, k, q);
            Contact<T> ct = contact(tet, k, root, q);
            loop_contact(tet, i, j, k, root, ct, faces, acc.data());
        }
        for (int64_t v = 0; v < V; ++v) {
            const int64_t* a = acc.data() + v * 8;
            if (a[6] == 0) continue;
            double cnt = (double)a[6];
            for (int d = 0; d < 3; ++d) {
                double dx = ((double)a[d] * FIX_INV) / cnt;
                double dv = ((double)a[3 + d] * FIX_INV) / cnt;
                verts1[v * 3 + d] = (T)((double)verts1[v * 3 + d] + dx);
                vel[v * 3 + d] = (T)((double)vel[v * 3 + d] + dv);
            }
        }
        ++it;
        if (it >= max_iter) break;
    }
    return it;
}

// Impulse loop on one mesh (vertices, faces, per-corner masses); verts1 and vel are updated
// in place.  Returns the iterations applied (or -1), writes the contact count of every
// collision check to contacts_per_iter (max_iter + 1 entries) and whether the last check
// found no contact.
ORC_API int orc_impulse_loop(int dtype, const void* verts0, void* verts1, void* vel, const int32_t* faces,
                             const void* masses, int64_t F, int64_t V, int max_iter, int32_t* contacts_per_iter,
                             int nthreads, int* converged) {
    if (F < 2 || V < 1 || max_iter < 1) return -1;
    for (int64_t f = 0; f < 3 * F; ++f)
        if (faces[f] < 0 || faces[f] >= V) return -1;
    if (dtype == 0)
        return loop_impl<float>((const float*)verts0, (float*)verts1, (float*)vel, faces, (const float*)masses, F, V,
                                max_iter, contacts_per_iter, nthreads, converged);
    return loop_impl<double>((const double*)verts0, (double*)verts1, (double*)vel, faces, (const double*)masses, F, V,
                             max_iter, contacts_per_iter, nthreads, converged);
}

template <class T>
static int64_t prox_impl(const T* bboxes, const int64_t* tree, const T* tri, int n, double th_f, int64_t* rows,
                         double* dist, int64_t cap) {
    Forest<T> f;
    import_tree(bboxes, tree, n, f);
    if (!f.ok) return -1;
    T th = (T)(float)th_f;
    std::vector<int64_t> pairs;
    if (candidates(f, th, nullptr, pairs, 1) < 0) return -1;
    int64_t w = 0;
    for (size_t c = 0; c < pairs.size() / 2; ++c) {
        Tri<T> a = load_tri(tri, pairs[2 * c]), b = load_tri(tri, pairs[2 * c + 1]);
        if (share_vertex(a, b)) continue;
        for (int k = 0; k < 15; ++k) {
            if (!prox_subbox(a, b, k, th)) continue;
            T d = prox_distance(a, b, k);
            if (!(d <= th && d >= 0)) continue;
            if (w < cap) {
                rows[3 * w] = pairs[2 * c]; rows[3 * w + 1] = pairs[2 * c + 1]; rows[3 * w + 2] = k;
                if (dist) dist[w] = (double)d;
            }
            ++w;
        }
    }
    return w;
}

// find_proximity (proximity_static.cu:510-694): (i, j, k) rows closer than threshold
ORC_API int64_t orc_proximity(int dtype, const void* bboxes, const int64_t* tree, const void* tri, int n, double th,
                      int64_t* rows, double* dist, int64_t cap) {
    if (dtype == 0) return prox_impl<float>((const float*)bboxes, tree, (const float*)tri, n, th, rows, dist, cap);
    return prox_impl<double>((const double*)bboxes, tree, (const double*)tri, n, th, rows, dist, cap);
}

// ---- primitive probes for known-answer tests ----
ORC_API int orc_solve_cubic(double a, double b, double c, double d, double* roots) {
    solve_cubic<double>(a, b, c, d, roots);
    return 0;
}
ORC_API uint32_t orc_morton(double x, double y, double z) { return morton3d<double>(x, y, z); }
ORC_API uint32_t orc_morton_f(float x, float y, float z) { return morton3d<float>(x, y, z); }
ORC_API void orc_certmul(const double* x, int k, double y, double* r) {
    ccc_dd d = ccc_certmul(x[0], k > 1 ? x[1] : 0.0, k, y);
    r[0] = d.hi;
    r[1] = d.lo;
}
ORC_API double orc_cbrt(double x) { return ccc_cbrt(x); }
ORC_API double orc_acos(double x) { return ccc_acos(x); }
ORC_API double orc_cos(double x) { return ccc_cos(x); }
ORC_API double orc_sin(double x) { return ccc_sin(x); }
ORC_API void orc_cubic_coeffs(const double* tet /* v0..v3, dv0..dv3: 24 doubles */, double* c) {
    MTet<double> t;
    for (int i = 0; i < 4; ++i) {
        t.v[i] = mk<double>(tet[3 * i], tet[3 * i + 1], tet[3 * i + 2]);
        t.dv[i] = mk<double>(tet[12 + 3 * i], tet[12 + 3 * i + 1], tet[12 + 3 * i + 2]);
    }
    cubic_coeffs(t, c);
}
// root filter and contact kinematics of one tetrahedron (v0..v3, dv0..dv3) of type k
ORC_API int orc_filter(const double* tet, int k, double root) {
    MTet<double> t;
    for (int i = 0; i < 4; ++i) {
        t.v[i] = mk<double>(tet[3 * i], tet[3 * i + 1], tet[3 * i + 2]);
        t.dv[i] = mk<double>(tet[12 + 3 * i], tet[12 + 3 * i + 1], tet[12 + 3 * i + 2]);
    }
    return ccd_filter(t, k, root) ? 1 : 0;
}
ORC_API void orc_contact(const double* tet, int k, double root, const double* q, double* out) {
    MTet<double> t;
    for (int i = 0; i < 4; ++i) {
        t.v[i] = mk<double>(tet[3 * i], tet[3 * i + 1], tet[3 * i + 2]);
        t.dv[i] = mk<double>(tet[12 + 3 * i], tet[12 + 3 * i + 1], tet[12 + 3 * i + 2]);
    }
    Contact<double> c = contact(t, k, root, q);
    out[0] = c.n.x; out[1] = c.n.y; out[2] = c.n.z; out[3] = c.vn; out[4] = c.m0; out[5] = c.m1;
}
ORC_API int orc_sat(int dtype, const void* a, const void* b, double th) {
    if (dtype == 0) {
        Tri<float> x = load_tri((const float*)a, 0), y = load_tri((const float*)b, 0);
        return sat(x, y, (float)th) ? 1 : 0;
    }
    Tri<double> x = load_tri((const double*)a, 0), y = load_tri((const double*)b, 0);
    return sat(x, y, th) ? 1 : 0;
}
ORC_API int orc_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

