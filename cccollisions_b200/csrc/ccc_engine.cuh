// ccc_engine.cuh — kernels of the resident multi-mesh engine.
//
// The engine keeps many meshes of uneven size on the device at once, each in its own
// slot range of one arena, and runs every step over a device-resident mesh table
// (Forest), so one captured launch sequence serves whatever meshes are active.
//
// Per mesh, the tree is a Karras radix tree over 30-bit Morton codes of the triangles'
// swept centroids, normalised by the mesh's own centroid bounds, sorted by a stable LSD
// radix sort (keys: mesh index above the code, so one sort orders every mesh at once).
// Topology is built once (the binary tree, then four-wide traversal nodes, QNode, over it);
// every step only refits the boxes, bottom-up, straight into the QNode slots (fp32 rounded
// outward); a leaf's query box is its own slot box.  The candidate pairs are therefore a
// superset of the pairs whose T-precision swept boxes overlap; the continuous narrow phase
// re-tests every pair's swept sub-boxes exactly, so its output is that of the reference's
// exact candidate set.
//
// The impulse loop adds a vertex arena: faces map triangle corners to vertices, contacts
// add their impulses to per-vertex fixed-point accumulators (integer atomics, so the sums
// do not depend on the order the contacts arrive in), and the averaged corrections move
// the vertices, after which the end-of-step triangle soup is regathered.
#pragma once

#include "ccc_kernels.cuh"

namespace ccc {

// non-finite impulse skipped by the loop accumulators
static constexpr int ST_NONFINITE = 16;

// Vertex arena of the mesh table: dense vertex prefix (M + 1) and vertex data bases (M).
struct VertTable {
    const int* vvoff;
    const int* vpoff;
};

// ---------------------------------------------------------------------------------------
// Tree build

// order-preserving map of floats to unsigned ints, for atomicMin / atomicMax
__device__ __forceinline__ unsigned f2ord(float f) {
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

template <class T> __device__ __forceinline__ float3 swept_centroid(const T* x0, const T* x1, long long slot) {
    const T* a = x0 + slot * 9;
    const T* b = x1 + slot * 9;
    T c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) c[d] = ((a[d] + a[3 + d] + a[6 + d]) + (b[d] + b[3 + d] + b[6 + d])) / (T)6;
    return make_float3((float)c[0], (float)c[1], (float)c[2]);
}

// per-mesh centroid bounds (6 ordered words per slot id: min xyz, max xyz; the caller sets
// the min words to 0xffffffff and the max words to 0 first), and the centroids of the work
// items for k_morton (x, y in cxy, z in cz).  Each warp takes BOUNDS_CHUNK consecutive items;
// a lane keeps running bounds while its mesh stays the same (the items are in mesh order),
// and the warp's lanes are reduced once a chunk, so that the words see one atomic a chunk
// rather than one a warp of items.
static constexpr int BOUNDS_CHUNK = 256;
template <class T>
__global__ void k_mesh_bounds(Forest F, const T* __restrict__ x0, const T* __restrict__ x1,
                              unsigned* __restrict__ bounds, float2* __restrict__ cxy, float* __restrict__ cz) {
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    auto flush = [&](int m, const float* lo, const float* hi) {
        unsigned* b = bounds + 6 * __ldg(F.sid + m);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            atomicMin(b + d, f2ord(lo[d]));
            atomicMax(b + 3 + d, f2ord(hi[d]));
        }
    };
    for (long long base = (long long)((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * BOUNDS_CHUNK; base < total;
         base += nwarps * BOUNDS_CHUNK) {
        int cm = -1;                         // the mesh of this lane's running bounds
        float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
        for (int r = 0; r < BOUNDS_CHUNK / 32; ++r) {
            const long long v = base + r * 32 + lane;
            if (v >= total) break;
            const int m = find_mesh(F.voff, M, v, 0);
            const float3 c = swept_centroid(x0, x1, (long long)__ldg(F.poff + m) + (v - __ldg(F.voff + m)));
            cxy[v] = make_float2(c.x, c.y);
            cz[v] = c.z;
            const float cc[3] = {c.x, c.y, c.z};
            if (m != cm) {
                if (cm >= 0) flush(cm, lo, hi);
                cm = m;
#pragma unroll
                for (int d = 0; d < 3; ++d) lo[d] = hi[d] = cc[d];
            } else {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    lo[d] = fminf(lo[d], cc[d]);
                    hi[d] = fmaxf(hi[d], cc[d]);
                }
            }
        }
        // (every lane takes part in the shuffle: a lane past the end has cm < 0)
        const int m0 = __shfl_sync(FULL, cm, 0);
        if (__all_sync(FULL, cm >= 0 && cm == m0)) {
            // the whole warp in one mesh: butterfly reduction, one atomic per word
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    lo[d] = fminf(lo[d], __shfl_xor_sync(FULL, lo[d], o));
                    hi[d] = fmaxf(hi[d], __shfl_xor_sync(FULL, hi[d], o));
                }
            if (lane == 0) flush(cm, lo, hi);
        } else if (cm >= 0) {
            flush(cm, lo, hi);
        }
    }
}

// 10 bits of x spread to every third bit (bit i -> bit 3i)
__device__ __forceinline__ unsigned spread3(unsigned x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__device__ __forceinline__ unsigned quantize1024(float c, float lo, float hi) {
    float ext = hi - lo;
    float t = ext > 0.f ? (c - lo) / ext : 0.f;
    float q = fminf(fmaxf(t * 1024.f, 0.f), 1023.f);
    return (unsigned)q;
}

// sort keys (mesh index << 30 | Morton code) and values (mesh-local triangle id), from the
// centroids that k_mesh_bounds left
static __global__ void k_morton(Forest F, const float2* __restrict__ cxy, const float* __restrict__ cz,
                         const unsigned* __restrict__ bounds, unsigned long long* __restrict__ keys,
                         int* __restrict__ vals) {
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        int m = find_mesh(F.voff, M, v, 0);
        int local = v - __ldg(F.voff + m);
        const float2 cv = cxy[v];
        const float3 c = make_float3(cv.x, cv.y, cz[v]);
        const unsigned* b = bounds + 6 * __ldg(F.sid + m);
        unsigned qx = quantize1024(c.x, ord2f(b[0]), ord2f(b[3]));
        unsigned qy = quantize1024(c.y, ord2f(b[1]), ord2f(b[4]));
        unsigned qz = quantize1024(c.z, ord2f(b[2]), ord2f(b[5]));
        unsigned code = (spread3(qx) << 2) | (spread3(qy) << 1) | spread3(qz);
        keys[v] = ((unsigned long long)m << 30) | code;
        vals[v] = local;
    }
}

// ---- stable LSD radix sort, 8-bit digits: histogram, scan, scatter per pass ----
static constexpr int SORT_THREADS = 256;
static constexpr int SORT_ROUNDS = 8;
static constexpr int SORT_TILE = SORT_THREADS * SORT_ROUNDS;

// counts[d * nblk + b] = number of keys of tile b with digit d
static __global__ void __launch_bounds__(SORT_THREADS)
k_radix_hist(const unsigned long long* __restrict__ keys, int n, int shift, int* __restrict__ counts, int nblk) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * SORT_TILE;
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        long long i = base + r * SORT_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255], 1);
    }
    __syncthreads();
    counts[(long long)threadIdx.x * nblk + blockIdx.x] = h[threadIdx.x];
}

// exclusive prefix of v over the SORT_THREADS threads of the block, with the block's sum in
// *total (wsum: SORT_THREADS / 32 + 1 ints of shared memory, free again on return)
__device__ __forceinline__ int sort_block_exclusive_scan(int v, int* wsum, int* total) {
    constexpr int WARPS = SORT_THREADS / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int incl = warp_inclusive_scan(v, lane);
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int x = lane < WARPS ? wsum[lane] : 0;
        const int sc = warp_inclusive_scan(x, lane);
        if (lane < WARPS) wsum[lane] = sc - x;
        if (lane == 31) wsum[WARPS] = sc;
    }
    __syncthreads();
    const int r = wsum[w] + incl - v;
    *total = wsum[WARPS];
    __syncthreads();
    return r;
}

// One block a digit d: row d of counts (the tiles' counts of digit d, in tile order) becomes
// its exclusive prefix, in place, and rowtot[d] the row's sum.  k_radix_scatter adds the
// prefix of the row sums (the keys of the smaller digits) itself.
static constexpr int ROWSCAN_ITEMS = 4;
static __global__ void __launch_bounds__(SORT_THREADS)
k_radix_rowscan(int* __restrict__ counts, int nblk, int* __restrict__ rowtot) {
    __shared__ int wsum[SORT_THREADS / 32 + 1];
    int* row = counts + (long long)blockIdx.x * nblk;
    int carry = 0;                                   // (the same in every thread)
    for (int base = 0; base < nblk; base += SORT_THREADS * ROWSCAN_ITEMS) {
        const int at = base + threadIdx.x * ROWSCAN_ITEMS;
        int v[ROWSCAN_ITEMS], sum = 0;
#pragma unroll
        for (int i = 0; i < ROWSCAN_ITEMS; ++i) {
            v[i] = at + i < nblk ? row[at + i] : 0;
            sum += v[i];
        }
        int total;
        int run = carry + sort_block_exclusive_scan(sum, wsum, &total);
#pragma unroll
        for (int i = 0; i < ROWSCAN_ITEMS; ++i) {
            if (at + i < nblk) row[at + i] = run;
            run += v[i];
        }
        carry += total;
    }
    if (threadIdx.x == 0) rowtot[blockIdx.x] = carry;
}

// stable scatter: keys of tile b with digit d go to (the keys of the digits below d) +
// offs[d * nblk + b] onwards, in input order; offs and rowtot from k_radix_rowscan
static __global__ void __launch_bounds__(SORT_THREADS)
k_radix_scatter(const unsigned long long* __restrict__ kin, const int* __restrict__ vin,
                unsigned long long* __restrict__ kout, int* __restrict__ vout, int n, int shift,
                const int* __restrict__ offs, const int* __restrict__ rowtot, int nblk) {
    constexpr int WARPS = SORT_THREADS / 32;
    __shared__ int whist[WARPS][256];
    __shared__ int base[256];
    __shared__ int round_total[256];
    __shared__ int wsum[WARPS + 1];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    int all;
    base[t] = sort_block_exclusive_scan(rowtot[t], wsum, &all) + offs[(long long)t * nblk + blockIdx.x];
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < SORT_ROUNDS; ++r) {
        long long i = (long long)blockIdx.x * SORT_TILE + r * SORT_THREADS + t;
        bool valid = i < n;
        unsigned long long key = valid ? kin[i] : 0ull;
        int d = valid ? (int)((key >> shift) & 255) : 256;
        for (int j = t; j < WARPS * 256; j += SORT_THREADS) (&whist[0][0])[j] = 0;
        __syncthreads();
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int rank = __popc(peers & lt);
        if (valid && rank == 0) whist[w][d] = __popc(peers);
        __syncthreads();
        {
            int run = 0;
            for (int ww = 0; ww < WARPS; ++ww) {
                int c = whist[ww][t];
                whist[ww][t] = run;
                run += c;
            }
            round_total[t] = run;
        }
        __syncthreads();
        if (valid) {
            int pos = base[d] + whist[w][d] + rank;
            kout[pos] = key;
            vout[pos] = vin[i];
        }
        __syncthreads();
        base[t] += round_total[t];
        __syncthreads();
    }
}

// Karras radix tree over the sorted codes of each mesh (Karras 2012, "Maximizing Parallelism
// in the Construction of BVHs, Octrees, and k-d Trees"), equal codes ordered by position.
// Writes the child references of every internal node (ref >= 0 internal node, ~pos leaf),
// their aux words (rightmost leaf position of an internal child, triangle id of a leaf),
// the parent codes ((parent << 1) | side) of nodes and leaves and the leaf -> triangle map,
// and clears the refit counters.
__device__ __forceinline__ int karras_delta(const unsigned long long* k, int n, int i, int j) {
    if (j < 0 || j > n - 1) return -1;
    unsigned a = (unsigned)(k[i] & 0x3fffffffull), b = (unsigned)(k[j] & 0x3fffffffull);
    return a == b ? 32 + __clz(i ^ j) : __clz(a ^ b);
}

static __global__ void k_karras_build(Forest F, const unsigned long long* __restrict__ keys,
                                      const int* __restrict__ vals, TNode* __restrict__ nodes,
                                      int* __restrict__ nparent, int* __restrict__ lparent,
                                      int* __restrict__ leaf_tri, unsigned* __restrict__ visits,
                                      int2* __restrict__ nrange, int* __restrict__ status) {
    const int M = forest_size(F);
    const int total_internal = __ldg(F.voff + M) - M;
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < total_internal; gi += gridDim.x * blockDim.x) {
        int m = find_mesh(F.voff, M, gi, 1);
        int vo = __ldg(F.voff + m), po = __ldg(F.poff + m);
        int n = __ldg(F.voff + m + 1) - vo;
        int i = gi - (vo - m);
        const unsigned long long* k = keys + vo;
        int d = (karras_delta(k, n, i, i + 1) - karras_delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = karras_delta(k, n, i, i - d);
        int lmax = 2;
        for (int g = 0; g < 32 && karras_delta(k, n, i, i + lmax * d) > dmin; ++g) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (karras_delta(k, n, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = karras_delta(k, n, i, j);
        int s = 0;
        for (int t = l;;) {
            t = (t + 1) >> 1;
            if (karras_delta(k, n, i, i + (s + t) * d) > dnode) s += t;
            if (t <= 1) break;
        }
        int split = i + s * d + min(d, 0);
        int lo = min(i, j), hi = max(i, j);
        if (split < lo || split + 1 > hi) {      // cannot happen for a valid sort
            atomicOr(status, ST_MALFORMED_TREE);
            continue;
        }
        int lref, rref, laux, raux;
        if (lo == split) {
            lref = ~split;
            laux = __ldg(vals + vo + split);
            lparent[po + split] = (i << 1) | 0;
            leaf_tri[po + split] = laux;
        } else {
            lref = split;
            laux = split;
            nparent[po + split] = (i << 1) | 0;
        }
        if (hi == split + 1) {
            rref = ~(split + 1);
            raux = __ldg(vals + vo + split + 1);
            lparent[po + split + 1] = (i << 1) | 1;
            leaf_tri[po + split + 1] = raux;
        } else {
            rref = split + 1;
            raux = hi;
            nparent[po + split + 1] = (i << 1) | 1;
        }
        nodes[po + i].d = make_int4(lref, rref, laux, raux);
        nrange[po + i] = make_int2(lo, hi);
        visits[po + i] = 0u;
        if (i == 0) nparent[po] = -1;
    }
}

// ---------------------------------------------------------------------------------------
// Four-wide nodes.  Every even-depth internal node b of the binary tree (the root has depth
// 0) heads a QNode whose 2 to 4 slots are b's children, where a child that is itself an
// internal node (odd depth) is replaced by its two children.  A slot holds a child box
// (fp32, rounded outward), a reference (>= 0: the QNode of an even-depth internal node;
// ~pos: the leaf at sorted position pos) and an aux word (the rightmost leaf position below
// an internal slot, the triangle id of a leaf slot).  Unused slots hold an empty box.
// QNodes are indexed by their binary node.  One QNode visit covers two binary levels, so a
// tree walk needs half as many dependent node fetches.
struct __align__(16) QNode {
    float4 lox, loy, loz, hix, hiy, hiz;
    int4 ref, aux;
};
static constexpr int Q_EMPTY = 0x7fffffff;
// qcode of an internal node: (QNode << 2) | slot for an even-depth node below the root;
// QCODE_ROOT for the root; for an odd-depth node, which has no slot of its own,
// QCODE_ODD - ((QNode << 2) | first slot) locates the two adjacent slots of its children
static constexpr int QCODE_ROOT = -1;
static constexpr int QCODE_ODD = -2;

// depth parity of every internal node (a climb to the root); even nodes other than the root
// get their slot code from k_qtree_slots
static __global__ void k_qtree_depth(Forest F, const int* __restrict__ nparent, int* __restrict__ qcode,
                                     int* __restrict__ status) {
    const int M = forest_size(F);
    const int total_internal = __ldg(F.voff + M) - M;
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < total_internal; gi += gridDim.x * blockDim.x) {
        int m = find_mesh(F.voff, M, gi, 1);
        int vo = __ldg(F.voff + m), po = __ldg(F.poff + m);
        int n = __ldg(F.voff + m + 1) - vo;
        int i = gi - (vo - m);
        int depth = 0, x = i;
        for (int guard = 0; x != 0 && guard < n; ++guard) {
            int code = __ldg(nparent + po + x);
            if (code < 0 || (code >> 1) >= n - 1) { atomicOr(status, ST_MALFORMED_TREE); break; }
            x = code >> 1;
            ++depth;
        }
        qcode[po + i] = i == 0 ? QCODE_ROOT : ((depth & 1) ? QCODE_ODD : 0);
    }
}

// slots of every QNode: references, aux words, empty boxes (the refit fills them), and the
// slot code of every leaf (qleaf) and even-depth internal node (qcode) they hold
static __global__ void k_qtree_slots(Forest F, const TNode* __restrict__ nodes, int* __restrict__ qcode,
                                     int* __restrict__ qleaf, QNode* __restrict__ qnodes, int* __restrict__ status) {
    const int M = forest_size(F);
    const int total_internal = __ldg(F.voff + M) - M;
    for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < total_internal; gi += gridDim.x * blockDim.x) {
        int m = find_mesh(F.voff, M, gi, 1);
        int vo = __ldg(F.voff + m), po = __ldg(F.poff + m);
        int n = __ldg(F.voff + m + 1) - vo;
        int i = gi - (vo - m);
        if (qcode[po + i] <= QCODE_ODD) continue;
        int4 d = nodes[po + i].d;
        int ref[4] = {Q_EMPTY, Q_EMPTY, Q_EMPTY, Q_EMPTY}, aux[4] = {0, 0, 0, 0};
        int ns = 0;
        bool ok = true;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            int r = side ? d.y : d.x, a = side ? d.w : d.z;
            if (r < 0) {
                ok = ok && ~r < n;
                ref[ns] = r;
                aux[ns] = a;
                ++ns;
            } else if (r < n - 1) {
                int4 dc = nodes[po + r].d;     // odd-depth child: its two children take its place
                qcode[po + r] = QCODE_ODD - ((i << 2) | ns);
                ref[ns] = dc.x;
                aux[ns] = dc.z;
                ++ns;
                ref[ns] = dc.y;
                aux[ns] = dc.w;
                ++ns;
            } else {
                ok = false;
            }
        }
        for (int sl = 0; sl < ns && ok; ++sl) {
            int r = ref[sl];
            if (r < 0) {
                if (~r >= n) { ok = false; break; }
                qleaf[po + ~r] = (i << 2) | sl;
            } else {
                if (r >= n - 1) { ok = false; break; }
                qcode[po + r] = (i << 2) | sl;
            }
        }
        if (!ok) {
            atomicOr(status, ST_MALFORMED_TREE);
            continue;
        }
        QNode q;
        const float inf = __int_as_float(0x7f800000);
        q.lox = q.loy = q.loz = make_float4(inf, inf, inf, inf);
        q.hix = q.hiy = q.hiz = make_float4(-inf, -inf, -inf, -inf);
        q.ref = make_int4(ref[0], ref[1], ref[2], ref[3]);
        q.aux = make_int4(aux[0], aux[1], aux[2], aux[3]);
        qnodes[po + i] = q;
    }
}

// ---------------------------------------------------------------------------------------
// Corner classes of the active meshes (Weld, for the narrow phase's repeated sub-tests),
// rebuilt in every step because the caller may rewrite the positions between steps.  Mesh
// m owns the part [6 poff[m], 6 (poff[m] + F_m)) of an open-addressing table of corner ids
// (4 * slot + corner), twice its corner count, cleared to -1 before k_weld_insert:
//  * k_weld_insert: every corner looks for an entry with its start position (compared with
//    ==, so -0 meets +0 and NaN meets nothing) and claims an empty one otherwise; the
//    claiming corner is the class's representative; the class sizes (cnt, zeroed before),
//    and CLS_NODEDUP on a class with a corner that differs from the representative in a bit
//    of either position or whose coordinates do not come back from their displacement
//    (x0 + (x1 - x0) != x1);
//  * k_weld_alloc: each class's range of the member list (a block-wide scan and one atomic
//    per block), k_weld_fill: the members with their triangles' classes, in order of
//    arrival, k_weld_rank: each class's members in ascending corner id;
//  * k_weld_tri: each triangle's classes, named by their first entry in the member list,
//    with CLS_NODEDUP also for classes of more than WELD_FANCAP corners and the three class
//    sizes, and the twin of each edge with the class of the twin's third corner.
// The classes are a function of the positions; which corner represents a class depends on
// the order of arrival, which no result depends on.

__device__ __forceinline__ unsigned long long weld_mix(unsigned long long z) {     // SplitMix64 finaliser
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
template <class T> __device__ __forceinline__ unsigned long long weld_key(T v) {
    const T z = v + (T)0;    // -0 + 0 = +0
    return sizeof(T) == 4 ? (unsigned long long)__float_as_uint((float)z)
                          : (unsigned long long)__double_as_longlong((double)z);
}
template <class T> __device__ __forceinline__ unsigned long long weld_bits(T v) {
    return sizeof(T) == 4 ? (unsigned long long)__float_as_uint((float)v)
                          : (unsigned long long)__double_as_longlong((double)v);
}

// the mesh and data slot of work item v (triangle position) of the active table
struct WeldItem {
    int m, n, po;
    long long slot;
};
__device__ __forceinline__ WeldItem weld_item(const Forest& F, int M, int v) {
    WeldItem w;
    w.m = find_mesh(F.voff, M, v, 0);
    const int vo = __ldg(F.voff + w.m);
    w.po = __ldg(F.poff + w.m);
    w.n = __ldg(F.voff + w.m + 1) - vo;
    w.slot = (long long)w.po + (v - vo);
    return w;
}

template <class T>
__global__ void k_weld_insert(Forest F, const T* __restrict__ x0, const T* __restrict__ x1, int* tab,
                              int* __restrict__ vidc, int* cnt, WsHeader* hdr) {
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        const WeldItem w = weld_item(F, M, v);
        int* part = tab + 6LL * w.po;
        const unsigned long long size = 6ull * (unsigned long long)w.n;
        for (int c = 0; c < 3; ++c) {
            const T* p = x0 + w.slot * 9 + 3 * c;
            const T px = __ldg(p), py = __ldg(p + 1), pz = __ldg(p + 2);
            const unsigned long long h = weld_mix(weld_key(px) ^ weld_mix(weld_key(py) ^ weld_mix(weld_key(pz))));
            unsigned long long at = __umul64hi(h, size);
            const int id = (int)(4 * w.slot + c);
            int rep = -1;
            for (unsigned long long probe = 0; probe < size; ++probe) {
                int cur = __ldcg(part + at);
                if (cur == -1) {
                    cur = atomicCAS(part + at, -1, id);
                    if (cur == -1) {
                        rep = id;
                        break;
                    }
                }
                const T* q = x0 + (long long)(cur >> 2) * 9 + 3 * (cur & 3);
                if (__ldg(q) == px && __ldg(q + 1) == py && __ldg(q + 2) == pz) {
                    rep = cur;
                    break;
                }
                if (++at == size) at = 0;
            }
            // (the table has twice the mesh's corners, so every corner finds its entry)
            if (rep < 0) {
                atomicOr(&hdr->status, ST_MALFORMED_TREE);
                rep = id;
            }
            vidc[id] = rep;
            // the class's size, and whether this corner keeps it from being shared
            const T* p1 = x1 + w.slot * 9 + 3 * c;
            const T* r0 = x0 + (long long)(rep >> 2) * 9 + 3 * (rep & 3);
            const T* r1 = x1 + (long long)(rep >> 2) * 9 + 3 * (rep & 3);
            const T pc[3] = {px, py, pz};
            bool ok = true;
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                const T a0 = pc[ax], a1 = __ldg(p1 + ax);
                const T d = a1 - a0;
                ok = ok && (a0 + d) == a1;     // MovingTriangle::ComputeBBoxVertex's v + dv
                ok = ok && weld_bits(a0) == weld_bits(__ldg(r0 + ax)) && weld_bits(a1) == weld_bits(__ldg(r1 + ax));
            }
            atomicAdd(cnt + rep, 1);
            if (!ok) atomicOr(cnt + rep, CLS_NODEDUP);
        }
    }
}

static constexpr int WELD_THREADS = 256;

static __global__ void __launch_bounds__(WELD_THREADS)
k_weld_alloc(Forest F, const int* __restrict__ vidc, const int* __restrict__ cnt, int* __restrict__ fan_start,
             int* __restrict__ fan_end, WsHeader* hdr) {
    __shared__ int wsum[WELD_THREADS / 32];
    __shared__ int base_s;
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b0 = blockIdx.x * WELD_THREADS; b0 < total; b0 += gridDim.x * WELD_THREADS) {
        const int v = b0 + threadIdx.x;
        int sz[3] = {0, 0, 0};
        long long slot = 0;
        if (v < total) {
            slot = weld_item(F, M, v).slot;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int id = (int)(4 * slot + c);
                if (__ldg(vidc + id) == id) sz[c] = __ldg(cnt + id) & CLS_MASK;
            }
        }
        const int mine = sz[0] + sz[1] + sz[2];
        const int incl = warp_inclusive_scan(mine, lane);
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const int x = lane < WELD_THREADS / 32 ? wsum[lane] : 0;
            const int sc = warp_inclusive_scan(x, lane);
            if (lane < WELD_THREADS / 32) wsum[lane] = sc - x;
            if (lane == 31) base_s = sc ? atomicAdd(&hdr->fan_cursor, sc) : 0;
        }
        __syncthreads();
        int at = base_s + wsum[warp] + incl - mine;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (sz[c]) {
                fan_start[4 * slot + c] = at;
                fan_end[4 * slot + c] = at;       // k_weld_fill moves it to the end
                at += sz[c];
            }
        __syncthreads();
    }
}

static __global__ void k_weld_fill(Forest F, const int* __restrict__ vidc, const int* __restrict__ fan_start,
                                   int* fan_end, int4* __restrict__ fan) {
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        const long long slot = weld_item(F, M, v).slot;
        const int r0 = __ldg(vidc + 4 * slot), r1 = __ldg(vidc + 4 * slot + 1), r2 = __ldg(vidc + 4 * slot + 2);
        const int4 en = make_int4(0, __ldg(fan_start + r0), __ldg(fan_start + r1), __ldg(fan_start + r2));
        for (int c = 0; c < 3; ++c) {
            const int pos = atomicAdd(fan_end + (c == 0 ? r0 : (c == 1 ? r1 : r2)), 1);
            fan[pos] = make_int4((int)(4 * slot + c), en.y, en.z, en.w);
        }
    }
}

// each class's members in ascending corner id (classes of at most WELD_FANCAP corners; the
// larger ones, whose order no kernel reads, keep their places): k_weld_fill's entries (tmp)
// go to the place of their rank in their class, one thread an entry
static __global__ void k_weld_rank(Forest F, const int* __restrict__ vidc, const int* __restrict__ fan_start,
                                   const int* __restrict__ cnt, const int4* __restrict__ tmp, int4* __restrict__ fan) {
    const int M = forest_size(F);
    const long long entries = 3LL * __ldg(F.voff + M);       // every corner is in one class
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < entries;
         e += (long long)gridDim.x * blockDim.x) {
        const int4 en = tmp[e];
        const int rep = __ldg(vidc + en.x);
        const int n = __ldg(cnt + rep) & CLS_MASK;
        long long at = e;
        if (n >= 2 && n <= WELD_FANCAP) {
            const int s0 = __ldg(fan_start + rep);
            int rank = 0;
            for (int j = 0; j < n; ++j) rank += __ldg(&tmp[s0 + j].x) < en.x;
            at = s0 + rank;
        }
        fan[at] = en;
    }
}

static __global__ void k_weld_tri(Forest F, const int* __restrict__ vidc, const int* __restrict__ cnt,
                                  const int* __restrict__ fan_start, const int4* __restrict__ fan,
                                  int4* __restrict__ vid, int4* __restrict__ twin, int4* __restrict__ third) {
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        const long long slot = weld_item(F, M, v).slot;
        int st[3], n[3], fl[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int r = __ldg(vidc + 4 * slot + c);
            const int cv = __ldg(cnt + r);
            st[c] = __ldg(fan_start + r);
            n[c] = cv & CLS_MASK;
            fl[c] = ((cv & CLS_NODEDUP) || n[c] > WELD_FANCAP) ? CLS_NODEDUP : 0;
        }
        int tw[3], th[3];
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const int a0 = e > 1, a1 = e > 0 ? 2 : 1;
            tw[e] = TWIN_NONE;
            th[e] = 0;
            if (fl[a0] | fl[a1]) continue;      // no sub-test over this edge is shared
            const int u1 = st[a1];
            int found = 0;
            for (int i = st[a0]; i < st[a0] + n[a0]; ++i) {
                const int4 en = __ldg(fan + i);
                const int t = en.x >> 2, ca = en.x & 3;
                for (int cb = ca + 1; cb < 3; ++cb) {
                    if ((long long)t == slot && ca == a0 && cb == a1) continue;    // the edge itself
                    if ((cb == 1 ? en.z : en.w) == u1) {
                        ++found;
                        tw[e] = 4 * t + (ca + cb - 1);
                        const int oc = 3 - ca - cb;            // the twin's third corner
                        th[e] = oc == 0 ? en.y : (oc == 1 ? en.z : en.w);
                    }
                }
            }
            if (found > 1) tw[e] = TWIN_MANY;
        }
        int w = min(n[0], 31) | (min(n[1], 31) << 5) | (min(n[2], 31) << 10);
#pragma unroll
        for (int e = 0; e < 3; ++e) w |= (tw[e] == TWIN_NONE ? 0 : (tw[e] == TWIN_MANY ? 2 : 1)) << (15 + 2 * e);
        vid[slot] = make_int4(st[0] | fl[0], st[1] | fl[1], st[2] | fl[2], w);
        twin[slot] = make_int4(tw[0], tw[1], tw[2], 0);
        third[slot] = make_int4(th[0], th[1], th[2], 0);
    }
}

// ---------------------------------------------------------------------------------------
// Refit: swept leaf boxes rounded outward to fp32 into their slots, then bottom-up the box of
// every even-depth node into its own slot.

template <class T> __device__ __forceinline__ void box_outward_f32(const Box<T>& b, float lo[3], float hi[3]) {
    T l[3] = {b.lo.x, b.lo.y, b.lo.z}, h[3] = {b.hi.x, b.hi.y, b.hi.z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (sizeof(T) == 4) {
            lo[c] = (float)l[c];
            hi[c] = (float)h[c];
        } else {
            lo[c] = __double2float_rd((double)l[c]);
            hi[c] = __double2float_ru((double)h[c]);
        }
    }
}

__device__ __forceinline__ void write_qslot(QNode* qn, int code, const float lo[3], const float hi[3]) {
    float* f = reinterpret_cast<float*>(qn + (code >> 2));
    const int sl = code & 3;
    f[0 + sl] = lo[0];
    f[4 + sl] = lo[1];
    f[8 + sl] = lo[2];
    f[12 + sl] = hi[0];
    f[16 + sl] = hi[1];
    f[20 + sl] = hi[2];
}

// one slot's box, read through L2 (written by other blocks)
__device__ __forceinline__ void read_qslot(const QNode* qn, int code, float lo[3], float hi[3]) {
    const float* f = reinterpret_cast<const float*>(qn + (code >> 2));
    const int sl = code & 3;
    lo[0] = __ldcg(f + 0 + sl);
    lo[1] = __ldcg(f + 4 + sl);
    lo[2] = __ldcg(f + 8 + sl);
    hi[0] = __ldcg(f + 12 + sl);
    hi[1] = __ldcg(f + 16 + sl);
    hi[2] = __ldcg(f + 20 + sl);
}

__device__ __forceinline__ float hmin4(float4 v) { return fminf(fminf(v.x, v.y), fminf(v.z, v.w)); }
__device__ __forceinline__ float hmax4(float4 v) { return fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)); }

// Refit: every leaf writes its swept box (fp32, rounded outward) into its QNode slot and
// climbs; at each binary node the second arrival (the one that finds the node's other
// subtree done) unions the children and goes on, the first stops.  Two passes:
//  * pass 1 (k_engine_refit_local): a block takes REFIT_THREADS consecutive leaf positions
//    and refits every node whose leaf range lies inside them, in shared memory, round by
//    round; an item whose parent reaches outside the block hands that arrival to pass 2
//    through the frontier list;
//  * pass 2 (k_engine_refit_front) finishes those climbs with device-scope fences, global
//    arrival counters and L2 reads.  The global counters only ever grow and the arrival
//    that finds an odd count is the second one, so they are never cleared (a node refit in
//    pass 1 leaves its counter alone).  The kernel boundary makes every box written in
//    pass 1 visible to pass 2.
// Most nodes lie inside one block's range, so most of the refit is shared-memory work
// instead of device fences and L2 round trips.  Meshes with MF_DONE set in mflags (when
// given) are skipped.
static constexpr int REFIT_THREADS = 256;

// pass 1: a block's leaf positions [base, base + REFIT_THREADS) and the internal nodes of
// each mesh whose leaf range lies inside them ("local" nodes; a node's index lies in its
// range, so these are the nodes at the same positions).  The boxes live in shared memory,
// indexed by position - base: the leaves' from the soups, the local nodes' computed in
// rounds (a node whose two children were done in earlier rounds takes the union of their
// boxes; fminf / fmaxf skip NaN, so the order of the unions does not matter).  Then every
// leaf and every local even-depth node writes its box into its QNode slot, and each whose
// parent is not local hands that arrival to pass 2 through the frontier list.
template <class T>
__global__ void __launch_bounds__(REFIT_THREADS)
k_engine_refit_local(Forest F, const T* __restrict__ x0, const T* __restrict__ x1, const int* __restrict__ leaf_tri,
                     const int* __restrict__ lparent, const int* __restrict__ nparent,
                     const int* __restrict__ qcode, const int* __restrict__ qleaf, const int2* __restrict__ nrange,
                     const TNode* __restrict__ nodes, QNode* qnodes, int2* __restrict__ front, int front_cap,
                     const int* __restrict__ mflags, WsHeader* hdr) {
    __shared__ float s_llo[3][REFIT_THREADS], s_lhi[3][REFIT_THREADS];    // leaf boxes
    __shared__ float s_nlo[3][REFIT_THREADS], s_nhi[3][REFIT_THREADS];    // local node boxes
    __shared__ unsigned short s_done[REFIT_THREADS];    // round a local node was done in (0: not yet)
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    const int t = threadIdx.x;
    for (int base = blockIdx.x * REFIT_THREADS; base < total; base += gridDim.x * REFIT_THREADS) {
        const int v = base + t;
        bool live = false, node_local = false;
        int m = 0, vo = 0, po = 0, n = 0, p = 0, cl = 0, cr = 0;
        if (v < total) {
            m = find_mesh(F.voff, M, v, 0);
            vo = __ldg(F.voff + m);
            po = __ldg(F.poff + m);
            n = __ldg(F.voff + m + 1) - vo;
            p = v - vo;
            live = n >= 2 && !(mflags && (__ldg(mflags + __ldg(F.sid + m)) & MF_DONE));
        }
        const int blo = base - vo, bhi = base + REFIT_THREADS - 1 - vo;     // the block in mesh positions
        if (live) {
            // the leaf at position p
            const int tri = __ldg(leaf_tri + po + p);
            if (tri < 0 || tri >= n) {
                atomicOr(&hdr->status, ST_MALFORMED_TREE);
                live = false;
            } else {
                const long long slot = (long long)po + tri;
                const Box<T> b = merge(tri_box(load_tri(x0, slot)), tri_box(load_tri(x1, slot)));
                float lo[3], hi[3];
                box_outward_f32(b, lo, hi);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    s_llo[c][t] = lo[c];
                    s_lhi[c][t] = hi[c];
                }
            }
            // the internal node at position p, when its range lies inside the block
            if (live && p < n - 1) {
                const int2 r = __ldg(nrange + po + p);
                if (r.x >= blo && r.y <= bhi) {
                    const int4 d = __ldg(&nodes[po + p].d);
                    cl = d.x;
                    cr = d.y;
                    node_local = (cl < 0 ? ~cl < n : cl < n - 1) && (cr < 0 ? ~cr < n : cr < n - 1);
                    if (!node_local) atomicOr(&hdr->status, ST_MALFORMED_TREE);
                }
            }
        }
        s_done[t] = 0;
        __syncthreads();
        // rounds: children indices (position - base) of a local node lie in the block
        const int il = node_local ? (cl < 0 ? vo + ~cl : vo + cl) - base : 0;
        const int ir = node_local ? (cr < 0 ? vo + ~cr : vo + cr) - base : 0;
        bool pending = node_local;
#pragma unroll 1
        for (int round = 1; round <= REFIT_THREADS; ++round) {
            if (pending) {
                const bool dl = cl < 0 || (s_done[il] != 0 && s_done[il] < round);
                const bool dr = cr < 0 || (s_done[ir] != 0 && s_done[ir] < round);
                if (dl && dr) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const float a0 = cl < 0 ? s_llo[c][il] : s_nlo[c][il], a1 = cl < 0 ? s_lhi[c][il] : s_nhi[c][il];
                        const float b0 = cr < 0 ? s_llo[c][ir] : s_nlo[c][ir], b1 = cr < 0 ? s_lhi[c][ir] : s_nhi[c][ir];
                        s_nlo[c][t] = fminf(a0, b0);
                        s_nhi[c][t] = fmaxf(a1, b1);
                    }
                    s_done[t] = (unsigned short)round;
                    pending = false;
                }
            }
            if (!__syncthreads_or(pending)) break;
        }
        if (pending) atomicOr(&hdr->status, ST_MALFORMED_TREE);     // (a cycle: not reached)
        // slots and the hand-over to pass 2
        if (live) {
            QNode* qn = qnodes + po;
            const int lq = __ldg(qleaf + po + p);
            if (lq < 0 || (lq >> 2) >= n - 1) {
                atomicOr(&hdr->status, ST_MALFORMED_TREE);
            } else {
                const float lo[3] = {s_llo[0][t], s_llo[1][t], s_llo[2][t]};
                const float hi[3] = {s_lhi[0][t], s_lhi[1][t], s_lhi[2][t]};
                write_qslot(qn, lq, lo, hi);
            }
            // each item whose parent is not local hands the arrival at the parent to pass 2
            for (int item = 0; item < 2; ++item) {
                if (item == 1 && (!node_local || pending)) break;
                if (item == 1) {
                    const int qc = __ldg(qcode + po + p);
                    if (qc >= 0) {
                        if ((qc >> 2) >= n - 1) {
                            atomicOr(&hdr->status, ST_MALFORMED_TREE);
                        } else {
                            const float lo[3] = {s_nlo[0][t], s_nlo[1][t], s_nlo[2][t]};
                            const float hi[3] = {s_nhi[0][t], s_nhi[1][t], s_nhi[2][t]};
                            write_qslot(qn, qc, lo, hi);
                        }
                    }
                }
                const int code = __ldg((item ? nparent : lparent) + po + p);
                if (code < 0) continue;                           // the root
                const int par = code >> 1;
                if (par >= n - 1) {
                    atomicOr(&hdr->status, ST_MALFORMED_TREE);
                    continue;
                }
                const int2 r = __ldg(nrange + po + par);
                if (r.x >= blo && r.y <= bhi) continue;           // a local parent: done here
                const int f = atomicAdd(&hdr->front, 1);
                if (f < front_cap) front[f] = make_int2(m, code);
                else atomicOr(&hdr->status, ST_MALFORMED_TREE);
            }
        }
        __syncthreads();
    }
}

// pass 2: the climbs handed over by pass 1, from the node they reached (global protocol)
static __global__ void k_engine_refit_front(Forest F, const int* __restrict__ nparent, const int* __restrict__ qcode,
                                            QNode* qnodes, unsigned* visits, const int2* __restrict__ front,
                                            int front_cap, WsHeader* hdr) {
    const int nf = min(*(volatile int*)&hdr->front, front_cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
        const int2 e = front[i];
        const int m = e.x;
        const int vo = __ldg(F.voff + m), po = __ldg(F.poff + m);
        const int n = __ldg(F.voff + m + 1) - vo;
        QNode* qn = qnodes + po;
        int code = e.y;
        float lo[3], hi[3];
        for (int guard = 0; guard < n; ++guard) {
            const int node = code >> 1;
            if (code < 0 || node >= n - 1) { atomicOr(&hdr->status, ST_MALFORMED_TREE); break; }
            __threadfence();
            if ((atomicAdd(visits + po + node, 1u) & 1u) == 0u) break;     // first arrival
            const int qc = __ldg(qcode + po + node);
            if (qc <= QCODE_ODD) {
                const int c0 = QCODE_ODD - qc;
                if ((c0 >> 2) >= n - 1 || (c0 & 3) > 2) { atomicOr(&hdr->status, ST_MALFORMED_TREE); break; }
                float l2[3], h2[3];
                read_qslot(qn, c0, lo, hi);
                read_qslot(qn, c0 + 1, l2, h2);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    lo[c] = fminf(lo[c], l2[c]);
                    hi[c] = fmaxf(hi[c], h2[c]);
                }
            } else {
                const float4* f = reinterpret_cast<const float4*>(qn + node);
                lo[0] = hmin4(__ldcg(f + 0));
                lo[1] = hmin4(__ldcg(f + 1));
                lo[2] = hmin4(__ldcg(f + 2));
                hi[0] = hmax4(__ldcg(f + 3));
                hi[1] = hmax4(__ldcg(f + 4));
                hi[2] = hmax4(__ldcg(f + 5));
                if (qc == QCODE_ROOT) break;
                if (qc < 0 || (qc >> 2) >= n - 1) { atomicOr(&hdr->status, ST_MALFORMED_TREE); break; }
                write_qslot(qn, qc, lo, hi);
            }
            code = __ldg(nparent + po + node);
            if (code < 0) break;
        }
    }
}

// Continuous-collision candidates of resident trees: one query leaf per thread walks the
// QNodes with an explicit per-thread stack (local memory), tests the 4 slot boxes of a node at once
// (fp32; the query box is the leaf's own outward-rounded slot box), keeps the reference's
// order rule (a slot is skipped when its rightmost leaf position is not after the query's,
// so each unordered pair is found once) and emits (min id, max id) in data slots.  Candidates
// are the pairs whose fp32 boxes overlap, a superset of the exact ones; the continuous
// narrow phase re-tests every pair's swept sub-boxes exactly.  With the corner classes
// (vid, the collision step), pairs whose triangles share a vertex, which the narrow phase
// drops, are not emitted.
//
// SD > 0: the top SD + 1 levels of the mesh of a block's first query (at most 1 + 4 + 16
// QNodes) are copied into shared memory at every step of the block's loop, breadth first,
// and every reference from one copied node to another is rewritten to TRAV_STAGED | its
// index among the copies; the block's queries of that mesh start at the copied root and read
// those nodes from shared memory.  The other queries (a block spanning two meshes) walk
// the global nodes.
static constexpr int TRAV_STAGED = 1 << 30;
__device__ __forceinline__ int trav_stage_count(int sd) { return sd == 0 ? 0 : (sd == 1 ? 5 : 21); }

template <int SD>
static __global__ void __launch_bounds__(TRAV_THREADS)
k_traverse_q(const QNode* __restrict__ qnodes, const int* __restrict__ qleaf, const int* __restrict__ leaf_tri,
             Forest F, int2* __restrict__ cand, int cand_cap, WsHeader* hdr, const int* __restrict__ mflags,
             const int4* __restrict__ vid) {
    int stack[STACK_DEPTH];          // per-thread, in local memory (L1): shared memory holds the buffer
    __shared__ int2 cbuf[TRAV_BUF][TRAV_THREADS];     // candidate buffer (see flush_candidates)
    __shared__ QNode top[SD > 0 ? (SD == 1 ? 5 : 21) : 1];
    __shared__ int top_src[SD > 0 ? (SD == 1 ? 5 : 21) : 1];    // global index of each copy
    __shared__ int top_n, top_mesh;
    int nbuf = 0;
    const int tid = threadIdx.x;
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    for (int base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
        if (SD > 0) {
            // copy the top levels of the first query's mesh (block-uniform steps)
            __syncthreads();       // the previous step's walks are done with the copies
            if (tid == 0) {
                const int m0 = find_mesh(F.voff, M, base, 0);
                const int n0 = __ldg(F.voff + m0 + 1) - __ldg(F.voff + m0);
                const bool ok = n0 >= 2 && !(mflags && (__ldg(mflags + __ldg(F.sid + m0)) & MF_DONE));
                top_mesh = ok ? m0 : -1;
                top_n = ok ? 1 : 0;
                top_src[0] = 0;
            }
            __syncthreads();
            const int m0 = top_mesh;
            const QNode* qn0 = qnodes + (m0 >= 0 ? __ldg(F.poff + m0) : 0);
            const int n0 = m0 >= 0 ? __ldg(F.voff + m0 + 1) - __ldg(F.voff + m0) : 0;
            int lo = 0;                                 // first copy of the current level
#pragma unroll 1
            for (int lev = 0; lev <= SD && m0 >= 0; ++lev) {
                const int hi = top_n;                   // copies [lo, hi) are this level's
                // copy the level's nodes, 8 threads a node (16 bytes each)
                for (int w = tid; w < (hi - lo) * 8; w += blockDim.x) {
                    const int i = lo + w / 8, part = w % 8;
                    reinterpret_cast<int4*>(top + i)[part] =
                        __ldg(reinterpret_cast<const int4*>(qn0 + top_src[i]) + part);
                }
                __syncthreads();
                if (lev < SD && tid == 0) {
                    // the next level: the copies' internal children, rewritten to their copies
                    int cnt = hi;
                    for (int i = lo; i < hi; ++i) {
                        int* rr = reinterpret_cast<int*>(&top[i].ref);
                        for (int sl = 0; sl < 4; ++sl) {
                            const int r = rr[sl];
                            if (r == Q_EMPTY || r < 0 || r >= n0 - 1) continue;    // leaf, empty or bad
                            top_src[cnt] = r;
                            rr[sl] = TRAV_STAGED | cnt;
                            ++cnt;
                        }
                    }
                    top_n = cnt;
                }
                __syncthreads();
                lo = hi;
            }
        }
        const int v = base + tid;
        if (v < total) {
            const int m = find_mesh(F.voff, M, v, 0);
            const int vo = __ldg(F.voff + m), po = __ldg(F.poff + m);
            const int n = __ldg(F.voff + m + 1) - vo;
            const int p = v - vo;
            bool go = n >= 2 && !(mflags && (__ldg(mflags + __ldg(F.sid + m)) & MF_DONE));
            const QNode* qn = qnodes + po;
            const int qid = go ? __ldg(leaf_tri + po + p) : 0;
            const int lq = go ? __ldg(qleaf + po + p) : 0;
            if (go && (qid < 0 || qid >= n || lq < 0 || (lq >> 2) >= n - 1)) {
                atomicOr(&hdr->status, ST_MALFORMED_TREE);
                go = false;
            }
            if (go) {
                // (the query triangle's corner classes: pairs that share a vertex are not emitted)
                const int4 VQ = vid ? __ldg(vid + po + qid) : make_int4(0, 0, 0, 0);
                float qlo[3], qhi[3];
                {
                    const float* f = reinterpret_cast<const float*>(qn + (lq >> 2));
                    const int sl = lq & 3;
                    qlo[0] = __ldg(f + 0 + sl);
                    qlo[1] = __ldg(f + 4 + sl);
                    qlo[2] = __ldg(f + 8 + sl);
                    qhi[0] = __ldg(f + 12 + sl);
                    qhi[1] = __ldg(f + 16 + sl);
                    qhi[2] = __ldg(f + 20 + sl);
                }
                int sp = 0;
                int node = (SD > 0 && m == top_mesh) ? TRAV_STAGED : 0;
                const int limit = 2 * n + 64;
                for (int it = 0;; ++it) {
                    if (it > limit) {
                        atomicOr(&hdr->status, ST_MALFORMED_TREE);
                        break;
                    }
                    float4 LX, LY, LZ, HX, HY, HZ;
                    int4 R, A;
                    if (SD > 0 && (node & TRAV_STAGED)) {
                        const QNode& t = top[node & 0xff];
                        LX = t.lox; LY = t.loy; LZ = t.loz; HX = t.hix; HY = t.hiy; HZ = t.hiz; R = t.ref; A = t.aux;
                    } else {
                        const float4* f = reinterpret_cast<const float4*>(qn + node);
                        LX = __ldg(f + 0); LY = __ldg(f + 1); LZ = __ldg(f + 2);
                        HX = __ldg(f + 3); HY = __ldg(f + 4); HZ = __ldg(f + 5);
                        R = __ldg(reinterpret_cast<const int4*>(f + 6));
                        A = __ldg(reinterpret_cast<const int4*>(f + 7));
                    }
                    const float lx[4] = {LX.x, LX.y, LX.z, LX.w}, ly[4] = {LY.x, LY.y, LY.z, LY.w};
                    const float lz[4] = {LZ.x, LZ.y, LZ.z, LZ.w}, hx[4] = {HX.x, HX.y, HX.z, HX.w};
                    const float hy[4] = {HY.x, HY.y, HY.z, HY.w}, hz[4] = {HZ.x, HZ.y, HZ.z, HZ.w};
                    const int rr[4] = {R.x, R.y, R.z, R.w}, aa[4] = {A.x, A.y, A.z, A.w};
                    int next = -1;
                    bool bad = false, deep = false;
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        const int ref = rr[s];
                        if (ref == Q_EMPTY) continue;
                        const bool staged = SD > 0 && ref >= 0 && (ref & TRAV_STAGED);
                        if (!staged && (ref >= n - 1 || (ref < 0 && ~ref >= n))) { bad = true; continue; }
                        bool hit = (qlo[0] <= hx[s]) && (qhi[0] >= lx[s]) && (qlo[1] <= hy[s]) && (qhi[1] >= ly[s]) &&
                                   (qlo[2] <= hz[s]) && (qhi[2] >= lz[s]);
                        const int rightmost = ref < 0 ? ~ref : aa[s];
                        if (p >= rightmost) hit = false;
                        if (!hit) continue;
                        if (ref < 0) {
                            const int cid = aa[s];
                            if (vid && classes_meet(VQ, __ldg(vid + po + cid))) continue;
                            cbuf[nbuf++][tid] = make_int2(po + min(qid, cid), po + max(qid, cid));
                            if (nbuf == TRAV_BUF) {
                                cg::coalesced_group grp = cg::coalesced_threads();
                                int b0 = 0;
                                if (grp.thread_rank() == 0) b0 = atomicAdd(&hdr->cand_count, TRAV_BUF * (int)grp.size());
                                b0 = grp.shfl(b0, 0) + TRAV_BUF * (int)grp.thread_rank();
                                flush_candidates(cbuf, tid, TRAV_BUF, b0, cand, cand_cap, hdr);
                                nbuf = 0;
                            }
                        } else if (next < 0) {
                            next = ref;
                        } else if (sp < STACK_DEPTH) {
                            stack[sp++] = ref;
                        } else {
                            deep = true;
                        }
                    }
                    if (bad || deep) {
                        atomicOr(&hdr->status, bad ? ST_MALFORMED_TREE : ST_STACK_OVERFLOW);
                        break;
                    }
                    if (next >= 0) {
                        node = next;
                    } else {
                        if (sp == 0) break;
                        node = stack[--sp];
                    }
                }
            }
        }
    }
    if (nbuf > 0) flush_rest(cbuf, tid, nbuf, cand, cand_cap, hdr);
}

// Warp-cooperative form of k_traverse_q (collisions_static.cu:10-103): the 32 lanes of a warp
// take 32 consecutive query leaves and walk the QNode tree together with one stack, held
// across the lanes' registers (entry e in lane e % 32, word e / 32).  Each visited QNode is
// staged once per warp in shared memory (one coalesced 128-byte load, a word per lane) and
// read from there by every lane, instead of being fetched once per lane; every lane tests
// its own query against the node's four slots, and an internal slot is descended into when
// any lane's query reaches it.  A lane
// emits exactly the pairs of the per-thread walk: it emits leaf L when its box overlaps L's
// and its position is before L's (the order rule), and then it also overlaps every slot box
// above L (a slot box contains the boxes below it) and is before their rightmost leaves, so
// the warp, which descends wherever some lane's walk would, reaches L.  Lanes of a warp whose
// leaves lie in two meshes walk mesh by mesh.
static __global__ void __launch_bounds__(TRAV_THREADS)
k_traverse_w(const QNode* __restrict__ qnodes, const int* __restrict__ qleaf, const int* __restrict__ leaf_tri,
             Forest F, int2* __restrict__ cand, int cand_cap, WsHeader* hdr, const int* __restrict__ mflags,
             const int4* __restrict__ vid) {
    __shared__ int2 cbuf[TRAV_BUF][TRAV_THREADS];     // candidate buffer (see flush_candidates)
    __shared__ __align__(16) int nbuf_s[TRAV_THREADS / 32][32];    // each warp's staged QNode
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31;
    int nbuf = 0;
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    const int wpb = TRAV_THREADS / 32;
    int* stage = nbuf_s[tid >> 5];
    const float4* sf = reinterpret_cast<const float4*>(stage);
    const long long wstride = (long long)gridDim.x * wpb * 32;
    for (long long base = ((long long)blockIdx.x * wpb + (tid >> 5)) * 32; base < total; base += wstride) {
        const int v = (int)base + lane;
        const bool valid = v < total;
        const int m = valid ? find_mesh(F.voff, M, v, 0) : -1;
        unsigned pending = __ballot_sync(FULL, valid);
        while (pending) {
            const int mm = __shfl_sync(FULL, m, __ffs(pending) - 1);
            const bool mine = valid && m == mm;
            pending &= ~__ballot_sync(FULL, mine);
            const int vo = __ldg(F.voff + mm), po = __ldg(F.poff + mm);
            const int n = __ldg(F.voff + mm + 1) - vo;
            if (n < 2) continue;
            if (mflags && (__ldg(mflags + __ldg(F.sid + mm)) & MF_DONE)) continue;
            const QNode* qn = qnodes + po;
            const int p = v - vo;
            bool act = mine;
            int qid = 0;
            int4 VQ = make_int4(0, 0, 0, 0);
            float qlo[3] = {0.f, 0.f, 0.f}, qhi[3] = {0.f, 0.f, 0.f};
            if (act) {
                qid = __ldg(leaf_tri + po + p);
                const int lq = __ldg(qleaf + po + p);
                if (qid < 0 || qid >= n || lq < 0 || (lq >> 2) >= n - 1) {
                    atomicOr(&hdr->status, ST_MALFORMED_TREE);
                    act = false;
                } else {
                    if (vid) VQ = __ldg(vid + po + qid);
                    const float* f = reinterpret_cast<const float*>(qn + (lq >> 2));
                    const int sl = lq & 3;
                    qlo[0] = __ldg(f + 0 + sl);
                    qlo[1] = __ldg(f + 4 + sl);
                    qlo[2] = __ldg(f + 8 + sl);
                    qhi[0] = __ldg(f + 12 + sl);
                    qhi[1] = __ldg(f + 16 + sl);
                    qhi[2] = __ldg(f + 20 + sl);
                }
            }
            if (!__any_sync(FULL, act)) continue;
            int s0 = 0, s1 = 0;          // the warp's stack, entry e in lane e % 32, word e / 32
            int sp = 0, node = 0;
            const int limit = 2 * n + 64;
            for (int it = 0;; ++it) {
                if (it > limit) {
                    if (lane == 0) atomicOr(&hdr->status, ST_MALFORMED_TREE);
                    break;
                }
                // stage the node: word `lane` of its 128 bytes from each lane
                __syncwarp();
                stage[lane] = __ldg(reinterpret_cast<const int*>(qn + node) + lane);
                __syncwarp();
                const float4 LX = sf[0], LY = sf[1], LZ = sf[2], HX = sf[3], HY = sf[4], HZ = sf[5];
                const int4 R = reinterpret_cast<const int4*>(sf)[6];
                const int4 A = reinterpret_cast<const int4*>(sf)[7];
                const float lx[4] = {LX.x, LX.y, LX.z, LX.w}, ly[4] = {LY.x, LY.y, LY.z, LY.w};
                const float lz[4] = {LZ.x, LZ.y, LZ.z, LZ.w}, hx[4] = {HX.x, HX.y, HX.z, HX.w};
                const float hy[4] = {HY.x, HY.y, HY.z, HY.w}, hz[4] = {HZ.x, HZ.y, HZ.z, HZ.w};
                const int rr[4] = {R.x, R.y, R.z, R.w}, aa[4] = {A.x, A.y, A.z, A.w};
                int next = -1;
                bool bad = false, deep = false;
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int ref = rr[s];
                    if (ref == Q_EMPTY) continue;
                    if (ref >= n - 1 || (ref < 0 && ~ref >= n)) { bad = true; continue; }
                    const int rightmost = ref < 0 ? ~ref : aa[s];
                    const bool hit = act && p < rightmost && (qlo[0] <= hx[s]) && (qhi[0] >= lx[s]) &&
                                     (qlo[1] <= hy[s]) && (qhi[1] >= ly[s]) && (qlo[2] <= hz[s]) && (qhi[2] >= lz[s]);
                    if (ref < 0) {
                        if (hit && !(vid && classes_meet(VQ, __ldg(vid + po + aa[s])))) {
                            const int cid = aa[s];
                            cbuf[nbuf++][tid] = make_int2(po + min(qid, cid), po + max(qid, cid));
                            if (nbuf == TRAV_BUF) {
                                cg::coalesced_group grp = cg::coalesced_threads();
                                int b0 = 0;
                                if (grp.thread_rank() == 0) b0 = atomicAdd(&hdr->cand_count, TRAV_BUF * (int)grp.size());
                                b0 = grp.shfl(b0, 0) + TRAV_BUF * (int)grp.thread_rank();
                                flush_candidates(cbuf, tid, TRAV_BUF, b0, cand, cand_cap, hdr);
                                nbuf = 0;
                            }
                        }
                    } else if (__any_sync(FULL, hit)) {
                        if (next < 0) {
                            next = ref;
                        } else if (sp < STACK_DEPTH) {
                            if (lane == (sp & 31)) {
                                if (sp < 32) s0 = ref;
                                else s1 = ref;
                            }
                            ++sp;
                        } else {
                            deep = true;
                        }
                    }
                }
                if (bad || deep) {
                    if (lane == 0) atomicOr(&hdr->status, bad ? ST_MALFORMED_TREE : ST_STACK_OVERFLOW);
                    break;
                }
                if (next >= 0) {
                    node = next;
                } else {
                    if (sp == 0) break;
                    --sp;
                    const int w0 = __shfl_sync(FULL, s0, sp & 31), w1 = __shfl_sync(FULL, s1, sp & 31);
                    node = sp < 32 ? w0 : w1;
                }
            }
        }
    }
    if (nbuf > 0) flush_rest(cbuf, tid, nbuf, cand, cand_cap, hdr);
}

// ---------------------------------------------------------------------------------------
// Impulse loop

static constexpr double FIX_SCALE = 72057594037927936.0;        // 2^56
static constexpr double FIX_INV = 1.3877787807814457e-17;       // 2^-56
static constexpr double FIX_LIMIT = 64.0;

// fixed-point value of one impulse component (|x| < 64), 0 and false when out of range
__device__ __forceinline__ bool to_fix(double x, long long& q) {
    if (!(fabs(x) < FIX_LIMIT)) return false;
    q = __double2ll_rn(x * FIX_SCALE);
    return true;
}

// the contact's four point impulses, added to the vertices they move
template <class T>
__device__ __forceinline__ void loop_impulse(const MTet<T>& tet, long long gi, long long gj, int k, T root,
                                             const Contact<T>& ct, int m, const int* faces, const VertTable& vt,
                                             long long* acc, int* status) {
    ImpulseScale<T> sc = impulse_scale(ct, root);
    const int vbase = __ldg(vt.vpoff + m);
    const int nv = __ldg(vt.vvoff + m + 1) - __ldg(vt.vvoff + m);
#pragma unroll 1
    for (int pt = 0; pt < 4; ++pt) {
        V3<T> imp, idx;
        impulse_point(tet, k, pt, ct, sc, imp, idx);
        long long tri = tet_side(k, pt) ? gj : gi;
        int corner = tet_corner(k, pt);
        long long q[6];
        bool ok = to_fix((double)idx.x, q[0]) && to_fix((double)idx.y, q[1]) && to_fix((double)idx.z, q[2]) &&
                  to_fix((double)imp.x, q[3]) && to_fix((double)imp.y, q[4]) && to_fix((double)imp.z, q[5]);
        if (!ok) {
            atomicOr(status, ST_NONFINITE);
            continue;
        }
        int vid = __ldg(faces + tri * 3 + corner);
        if (vid < 0 || vid >= nv) {
            atomicOr(status, ST_MALFORMED_TREE);
            continue;
        }
        long long vslot = (long long)vbase + vid;
        unsigned long long* a = reinterpret_cast<unsigned long long*>(acc + vslot * 8);
#pragma unroll
        for (int c = 0; c < 6; ++c) atomicAdd(a + c, (unsigned long long)q[c]);
        atomicAdd(a + 6, 1ull);
    }
}

// Receiver of the impulses of the engine's loop iteration: counts the contacts of each mesh
// and adds their impulses to the per-vertex accumulators.
template <class T> struct LoopSink {
    const T* masses;       // 3 per triangle slot
    const int* faces;      // 3 mesh-local vertex ids per triangle slot
    VertTable vt;
    long long* acc;        // 8 words per vertex slot: dx xyz, dv xyz, count, unused
    int* contacts;         // per slot id
    __device__ __forceinline__ void add(const MTet<T>& tet, long long gi, long long gj, int k, T root,
                                        const Contact<T>& ct, const Forest& F, int M, int* status) const {
        int m = forest_slot_mesh(F, M, gi);
        atomicAdd(contacts + __ldg(F.sid + m), 1);
        loop_impulse(tet, gi, gj, k, root, ct, m, faces, vt, acc, status);
    }
};

// after a loop iteration's collision check: a mesh without contacts has converged; one with
// contacts takes this iteration's corrections and stops at max_iter iterations
static __global__ void k_loop_update(Forest F, const int* __restrict__ contacts, int* __restrict__ iters,
                                     int* __restrict__ flags, int max_iter) {
    const int M = forest_size(F);
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        int sid = __ldg(F.sid + m);
        int f = flags[sid];
        if (f & MF_DONE) continue;
        if (contacts[sid] == 0) {
            flags[sid] = f | MF_DONE | MF_CONVERGED;
        } else {
            int it = iters[sid] + 1;
            iters[sid] = it;
            if (it >= max_iter) flags[sid] = f | MF_DONE;
        }
    }
}

// average correction of every vertex touched this iteration; clears the accumulators
template <class T>
__global__ void k_loop_apply(Forest F, VertTable vt, const int* __restrict__ contacts, long long* __restrict__ acc,
                             T* __restrict__ verts1, T* __restrict__ vel) {
    const int M = forest_size(F);
    const int total = __ldg(vt.vvoff + M);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        int m = find_mesh(vt.vvoff, M, v, 0);
        if (__ldg(contacts + __ldg(F.sid + m)) == 0) continue;
        long long vs = (long long)__ldg(vt.vpoff + m) + (v - __ldg(vt.vvoff + m));
        long long* a = acc + vs * 8;
        long long cnt = a[6];
        if (cnt == 0) continue;
        double c = (double)cnt;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double dx = ((double)a[d] * FIX_INV) / c;
            double dv = ((double)a[3 + d] * FIX_INV) / c;
            verts1[vs * 3 + d] = (T)((double)verts1[vs * 3 + d] + dx);
            vel[vs * 3 + d] = (T)((double)vel[vs * 3 + d] + dv);
        }
#pragma unroll
        for (int d = 0; d < 8; ++d) a[d] = 0;
    }
}

// triangle soup of the vertices (all meshes in the table, or only those with contacts
// this iteration when contacts is given)
template <class T>
__global__ void k_gather_soup(Forest F, VertTable vt, const int* __restrict__ contacts, const int* __restrict__ faces,
                              const T* __restrict__ verts, T* __restrict__ soup, int* status) {
    const int M = forest_size(F);
    const int total = __ldg(F.voff + M);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        int m = find_mesh(F.voff, M, v, 0);
        if (contacts && __ldg(contacts + __ldg(F.sid + m)) == 0) continue;
        long long slot = (long long)__ldg(F.poff + m) + (v - __ldg(F.voff + m));
        long long vb = __ldg(vt.vpoff + m);
        int nv = __ldg(vt.vvoff + m + 1) - __ldg(vt.vvoff + m);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            int vid = __ldg(faces + slot * 3 + c);
            if (vid < 0 || vid >= nv) {
                atomicOr(status, ST_MALFORMED_TREE);
                continue;
            }
            long long vs = vb + vid;
#pragma unroll
            for (int d = 0; d < 3; ++d) soup[slot * 9 + c * 3 + d] = verts[vs * 3 + d];
        }
    }
}

// ---------------------------------------------------------------------------------------
// Per-mesh resets over a table

// centroid bounds of every mesh in the table to (empty): min words high, max words low
static __global__ void k_reset_bounds(Forest F, unsigned* __restrict__ bounds) {
    const int M = forest_size(F);
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        unsigned* b = bounds + 6 * __ldg(F.sid + m);
        b[0] = b[1] = b[2] = 0xffffffffu;
        b[3] = b[4] = b[5] = 0u;
    }
}

// loop counters and flags of every mesh in the table
static __global__ void k_loop_reset(Forest F, int* __restrict__ iters, int* __restrict__ flags) {
    const int M = forest_size(F);
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        int sid = __ldg(F.sid + m);
        iters[sid] = 0;
        flags[sid] = 0;
    }
}

// vertex accumulators of every mesh in the table
static __global__ void k_zero_acc(Forest F, VertTable vt, long long* __restrict__ acc) {
    const int M = forest_size(F);
    const int total = __ldg(vt.vvoff + M);
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < total; v += gridDim.x * blockDim.x) {
        int m = find_mesh(vt.vvoff, M, v, 0);
        long long vs = (long long)__ldg(vt.vpoff + m) + (v - __ldg(vt.vvoff + m));
#pragma unroll
        for (int d = 0; d < 8; ++d) acc[vs * 8 + d] = 0;
    }
}

// ---------------------------------------------------------------------------------------
// Packed copy of the active meshes' collision rows, for one device-to-host copy per step.
// meta = [offsets (M + 1) | slot ids (M) | status word] in table order: offsets[m] = rows of
// the active meshes before m, each mesh's count capped at its capacity F_m * maxcol.  One block.
static constexpr int PACK_SCAN_THREADS = 1024;
static __global__ void __launch_bounds__(PACK_SCAN_THREADS)
k_pack_offsets(Forest F, const int* __restrict__ mesh_cnt, int maxcol, const int* status, int* __restrict__ meta) {
    __shared__ int warp_sum[PACK_SCAN_THREADS / 32];
    __shared__ int carry;
    const int M = forest_size(F);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < M; base += PACK_SCAN_THREADS) {
        const int m = base + threadIdx.x;
        int n = 0;
        if (m < M) {
            int sid = __ldg(F.sid + m);
            long long cap = (long long)(__ldg(F.voff + m + 1) - __ldg(F.voff + m)) * maxcol;
            n = (int)min((long long)max(mesh_cnt[sid], 0), cap);
            meta[M + 1 + m] = sid;
        }
        int incl = warp_inclusive_scan(n, lane);
        if (lane == 31) warp_sum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int v = warp_sum[lane];
            int sc = warp_inclusive_scan(v, lane);
            warp_sum[lane] = sc - v;
        }
        __syncthreads();
        const int c0 = carry;
        if (m < M) meta[m] = c0 + warp_sum[warp] + incl - n;
        __syncthreads();
        if (threadIdx.x == PACK_SCAN_THREADS - 1) carry = c0 + warp_sum[warp] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        meta[M] = carry;
        meta[2 * M + 1] = *(volatile const int*)status;
    }
}

// rows and times of every active mesh, back to back in table order (the first `capacity`
// rows; ST_OUT_OVERFLOW when there are more)
template <class T>
static __global__ void k_pack_rows(Forest F, const int* __restrict__ meta, const long long* __restrict__ rows,
                                   const T* __restrict__ times, int maxcol, long long* __restrict__ out_rows,
                                   T* __restrict__ out_times, long long capacity, int* status) {
    const int M = forest_size(F);
    const long long total = __ldg(meta + M);
    const long long n = min(total, capacity);
    if (blockIdx.x == 0 && threadIdx.x == 0 && total > capacity) atomicOr(status, ST_OUT_OVERFLOW);
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
         r += (long long)gridDim.x * blockDim.x) {
        int m = find_mesh(meta, M, r, 0);
        long long src = (long long)__ldg(F.poff + m) * maxcol + (r - __ldg(meta + m));
        out_rows[r * 3 + 0] = __ldg(rows + src * 3 + 0);
        out_rows[r * 3 + 1] = __ldg(rows + src * 3 + 1);
        out_rows[r * 3 + 2] = __ldg(rows + src * 3 + 2);
        out_times[r] = __ldg(times + src);
    }
}

}  // namespace ccc
