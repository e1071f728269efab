// ccc_geom.cuh — device geometry for the collision pipeline.
//
// Every expression keeps the reference's evaluation order (Dolorousrtur/CCCollisions
// src/figures.cu, src/aabb.cu, src/collisions_continuous.cu, src/collisions_impulses.cu,
// src/proximity_static.cu).  The reference is compiled with nvcc's default multiply-add
// contraction; this library is compiled with -fmad=false and writes the same fusions out
// explicitly (fmaT): a*b + c -> fma(a, b, c), c + a*b -> fma(a, b, c), a*b +- c*d fuses
// the first product, dot / cross / norm2 are fixed fma chains.  Every other operation is
// a single IEEE-754 rounding, so the CPU oracle (same model with std::fma) matches.
#pragma once

#include <stdint.h>
#include <float.h>
#include "ccc_libm.h"
#include "ccc_ddmul.h"

namespace ccc {

template <class T> struct V3 { T x, y, z; };
template <class T> __device__ __forceinline__ V3<T> mk(T x, T y, T z) { V3<T> r; r.x = x; r.y = y; r.z = z; return r; }
template <class T> __device__ __forceinline__ V3<T> operator+(V3<T> a, V3<T> b) { return mk<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> __device__ __forceinline__ V3<T> operator-(V3<T> a, V3<T> b) { return mk<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> __device__ __forceinline__ V3<T> operator*(V3<T> a, T s) { return mk<T>(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
// a.x*b.x + a.y*b.y + a.z*b.z  ->  fma(a.z, b.z, fma(a.x, b.x, a.y*b.y))
template <class T> __device__ __forceinline__ T dot(V3<T> a, V3<T> b) { return fmaT(a.z, b.z, fmaT(a.x, b.x, a.y * b.y)); }
template <class T> __device__ __forceinline__ T dot_zyx(V3<T> a, V3<T> b) { return fmaT(a.z, b.z, fmaT(a.y, b.y, a.x * b.x)); }
// a.y*b.z - a.z*b.y  ->  fma(a.y, b.z, -(a.z*b.y)), and cyclically
template <class T> __device__ __forceinline__ V3<T> cross(V3<T> a, V3<T> b) {
    return mk<T>(fmaT(a.y, b.z, -(a.z * b.y)), fmaT(a.z, b.x, -(a.x * b.z)), fmaT(a.x, b.y, -(a.y * b.x)));
}
template <class T> __device__ __forceinline__ T norm2(V3<T> a) { return fmaT(a.z, a.z, fmaT(a.x, a.x, a.y * a.y)); }
// v + d * t  ->  fma(d, t, v) per component
template <class T> __device__ __forceinline__ V3<T> axpy(V3<T> v, V3<T> d, T t) {
    return mk<T>(fmaT(d.x, t, v.x), fmaT(d.y, t, v.y), fmaT(d.z, t, v.z));
}
// a*u + b*v + c*w  ->  fma(c, w, fma(a, u, b*v)) per component
template <class T> __device__ __forceinline__ V3<T> lin3(V3<T> a, T u, V3<T> b, T v, V3<T> c, T w) {
    return mk<T>(fmaT(c.x, w, fmaT(a.x, u, b.x * v)), fmaT(c.y, w, fmaT(a.y, u, b.y * v)),
                 fmaT(c.z, w, fmaT(a.z, u, b.z * v)));
}
// a*b - c*d  ->  fma(a, b, -(c*d))
template <class T> __device__ __forceinline__ T fms2(T a, T b, T c, T d) { return fmaT(a, b, -(c * d)); }
// A rounded product, sum or difference that the compiler never fuses with a neighbouring
// operation.  The continuous narrow phase is compiled with multiply-add contraction on (as
// the reference is: it must call CUDA's pow as the reference's build compiles it), so every
// product of this library's own that feeds a sum is written with these (or inside an
// explicit fmaT, whose operands are never fused either): the code rounds as written under
// either setting.
__device__ __forceinline__ float mulrn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulrn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float addrn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double addrn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float subrn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double subrn(double a, double b) { return __dsub_rn(a, b); }

// Elementary functions of the cubic solver and of normalize(): CUDA's own (the reference's
// calls: cbrt, cbrtf, acos, cos, sin, pow(x, 2), rsqrt) or this library's portable ones,
// which the CPU oracle shares bit for bit.
enum MathLib { LIB_REFERENCE = 0, LIB_PORTABLE = 1 };
__device__ __forceinline__ float fmn(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float fmx(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fmn(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double fmx(double a, double b) { return fmax(a, b); }

template <class T> struct Box { V3<T> lo, hi; };
template <class T> __device__ __forceinline__ Box<T> merge(const Box<T>& a, const Box<T>& b) {
    Box<T> r;
    r.lo = mk<T>(fmn(a.lo.x, b.lo.x), fmn(a.lo.y, b.lo.y), fmn(a.lo.z, b.lo.z));
    r.hi = mk<T>(fmx(a.hi.x, b.hi.x), fmx(a.hi.y, b.hi.y), fmx(a.hi.z, b.hi.z));
    return r;
}
// checkOverlap (aabb.cu:101-111)
template <class T> __device__ __forceinline__ bool overlap(const Box<T>& a, const Box<T>& b, T th) {
    return (a.lo.x <= (b.hi.x + th)) && (a.hi.x >= (b.lo.x - th)) &&
           (a.lo.y <= (b.hi.y + th)) && (a.hi.y >= (b.lo.y - th)) &&
           (a.lo.z <= (b.hi.z + th)) && (a.hi.z >= (b.lo.z - th));
}
template <class T> __device__ __forceinline__ Box<T> load_box(const T* p) {
    Box<T> b;
    b.lo = mk<T>(p[0], p[1], p[2]);
    b.hi = mk<T>(p[3], p[4], p[5]);
    return b;
}
template <class T> __device__ __forceinline__ void store_box(T* p, const Box<T>& b) {
    p[0] = b.lo.x; p[1] = b.lo.y; p[2] = b.lo.z; p[3] = b.hi.x; p[4] = b.hi.y; p[5] = b.hi.z;
}

template <class T> struct Tri { V3<T> v[3]; };
template <class T> __device__ __forceinline__ Tri<T> load_tri(const T* __restrict__ p, int64_t i) {
    Tri<T> t;
    const T* q = p + i * 9;
#pragma unroll
    for (int c = 0; c < 3; ++c) t.v[c] = mk<T>(__ldg(q + 3 * c), __ldg(q + 3 * c + 1), __ldg(q + 3 * c + 2));
    return t;
}
// Triangle::ComputeBBox (figures.cu:37-41)
template <class T> __device__ __forceinline__ Box<T> tri_box(const Tri<T>& t) {
    Box<T> b;
    b.lo = mk<T>(fmn(t.v[0].x, fmn(t.v[1].x, t.v[2].x)), fmn(t.v[0].y, fmn(t.v[1].y, t.v[2].y)),
                 fmn(t.v[0].z, fmn(t.v[1].z, t.v[2].z)));
    b.hi = mk<T>(fmx(t.v[0].x, fmx(t.v[1].x, t.v[2].x)), fmx(t.v[0].y, fmx(t.v[1].y, t.v[2].y)),
                 fmx(t.v[0].z, fmx(t.v[1].z, t.v[2].z)));
    return b;
}

template <class T> __device__ __forceinline__ bool veq(V3<T> a, V3<T> b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
// shareVertex (figures.cu:527-544, 578-596): equality of coordinates
template <class T> __device__ __forceinline__ bool share_vertex(const V3<T>* a, const V3<T>* b) {
    bool s = false;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) s = s || veq(a[i], b[j]);
    return s;
}
// countSharedVerts (figures.cu:548-576)
template <class T> __device__ __forceinline__ int count_shared(const Tri<T>& a, const Tri<T>& b) {
    int c = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (veq(a.v[i], b.v[0]) || veq(a.v[i], b.v[1]) || veq(a.v[i], b.v[2])) ++c;
    return c;
}

// isect_interval + TriangleTriangleOverlap (figures.cu:378-427)
template <class T> __device__ __forceinline__ bool axis_overlap(const Tri<T>& a, const Tri<T>& b, V3<T> ax, T th) {
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
// TriangleTriangleIsectSepAxis (figures.cu:446-509); the reference ANDs all 17 axes
// without early exit, which is the same predicate as stopping at the first failure
template <class T> __device__ __forceinline__ bool sat(const Tri<T>& a, const Tri<T>& b, T th) {
    V3<T> a0 = a.v[1] - a.v[0], a1 = a.v[2] - a.v[0], a2 = a.v[2] - a.v[1];
    V3<T> an = cross(a1, a2);
    V3<T> b0 = b.v[1] - b.v[0], b1 = b.v[2] - b.v[0], b2 = b.v[2] - b.v[1];
    V3<T> bn = cross(b1, b2);
    if (!axis_overlap(a, b, an, th)) return false;
    if (!axis_overlap(a, b, bn, th)) return false;
    if (!axis_overlap(a, b, cross(a0, b0), th)) return false;
    if (!axis_overlap(a, b, cross(a0, b1), th)) return false;
    if (!axis_overlap(a, b, cross(a0, b2), th)) return false;
    if (!axis_overlap(a, b, cross(a1, b0), th)) return false;
    if (!axis_overlap(a, b, cross(a1, b1), th)) return false;
    if (!axis_overlap(a, b, cross(a1, b2), th)) return false;
    if (!axis_overlap(a, b, cross(a2, b0), th)) return false;
    if (!axis_overlap(a, b, cross(a2, b1), th)) return false;
    if (!axis_overlap(a, b, cross(a2, b2), th)) return false;
    if (!axis_overlap(a, b, cross(an, a0), th)) return false;
    if (!axis_overlap(a, b, cross(an, a1), th)) return false;
    if (!axis_overlap(a, b, cross(an, a2), th)) return false;
    if (!axis_overlap(a, b, cross(an, b0), th)) return false;
    if (!axis_overlap(a, b, cross(an, b1), th)) return false;
    if (!axis_overlap(a, b, cross(an, b2), th)) return false;
    return true;
}

// ------------------------------------------------------------------ continuous collision

// MovingTriangle (figures.cu:295-366): positions at t = 0 and displacement x1 - x0
template <class T> struct MTri { V3<T> v[3], dv[3]; };
template <class T> __device__ __forceinline__ MTri<T> load_mtri(const T* __restrict__ x0, const T* __restrict__ x1, int64_t i) {
    Tri<T> a = load_tri(x0, i), b = load_tri(x1, i);
    MTri<T> m;
#pragma unroll
    for (int c = 0; c < 3; ++c) { m.v[c] = a.v[c]; m.dv[c] = b.v[c] - a.v[c]; }
    return m;
}
// MovingTriangle::ComputeBBoxVertex (346-351): box of v and v + dv
template <class T> __device__ __forceinline__ Box<T> mvbox(const MTri<T>& t, int i) {
    V3<T> a = t.v[i], b = t.v[i] + t.dv[i];
    Box<T> r;
    r.lo = mk<T>(fmn(a.x, b.x), fmn(a.y, b.y), fmn(a.z, b.z));
    r.hi = mk<T>(fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z));
    return r;
}
template <class T> __device__ __forceinline__ Box<T> svbox(const Tri<T>& t, int i) {
    Box<T> r;
    r.lo = t.v[i];
    r.hi = t.v[i];
    return r;
}

// Point table of the 15 sub-tests (collisions_continuous.cu:36-124): bits per point p:
// side (first/second triangle of the pair) and corner.  Types 0..8 edge-edge with edges
// {01, 02, 12}[k/3] and [k%3]; 9..11 face of the first vs vertex k-9 of the second;
// 12..14 vertex k-12 of the first vs face of the second.
__device__ __forceinline__ void type_points(int k, int side[4], int corner[4]) {
    if (k < 9) {
        int e0 = k / 3, e1 = k - 3 * (k / 3);
        side[0] = 0; corner[0] = e0 == 2 ? 1 : 0;
        side[1] = 0; corner[1] = e0 == 0 ? 1 : 2;
        side[2] = 1; corner[2] = e1 == 2 ? 1 : 0;
        side[3] = 1; corner[3] = e1 == 0 ? 1 : 2;
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
template <class T> __device__ __forceinline__ bool ccd_subbox(const MTri<T>& a, const MTri<T>& b, int k) {
    int side[4], corner[4];
    type_points(k, side, corner);
    Box<T> b0, b1;
    if (k < 9) {
        b0 = merge(mvbox(a, corner[0]), mvbox(a, corner[1]));
        b1 = merge(mvbox(b, corner[2]), mvbox(b, corner[3]));
    } else if (k < 12) {
        b0 = merge(merge(mvbox(a, 0), mvbox(a, 1)), mvbox(a, 2));
        b1 = mvbox(b, k - 9);
    } else {
        b0 = mvbox(a, k - 12);
        b1 = merge(merge(mvbox(b, 0), mvbox(b, 1)), mvbox(b, 2));
    }
    return overlap(b0, b1, (T)0);
}

// all 15 swept sub-box tests as a bit mask; the three per-vertex swept boxes of each
// triangle are computed once
template <class T> __device__ __forceinline__ uint32_t ccd_subbox_mask(const MTri<T>& a, const MTri<T>& b) {
    Box<T> va[3], vb[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) { va[i] = mvbox(a, i); vb[i] = mvbox(b, i); }
    Box<T> ea[3], eb[3];
    ea[0] = merge(va[0], va[1]); ea[1] = merge(va[0], va[2]); ea[2] = merge(va[1], va[2]);
    eb[0] = merge(vb[0], vb[1]); eb[1] = merge(vb[0], vb[2]); eb[2] = merge(vb[1], vb[2]);
    Box<T> fa = merge(merge(va[0], va[1]), va[2]);
    Box<T> fb = merge(merge(vb[0], vb[1]), vb[2]);
    uint32_t m = 0;
#pragma unroll
    for (int e0 = 0; e0 < 3; ++e0)
#pragma unroll
        for (int e1 = 0; e1 < 3; ++e1)
            if (overlap(ea[e0], eb[e1], (T)0)) m |= 1u << (3 * e0 + e1);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (overlap(fa, vb[i], (T)0)) m |= 1u << (9 + i);
        if (overlap(va[i], fb, (T)0)) m |= 1u << (12 + i);
    }
    return m;
}

// The shared-vertex test and the 15 swept sub-box tests of a candidate pair (i, j), read
// straight from the soups one axis at a time: both are conjunctions over the axes (equal
// coordinates; intervals that overlap), so the per-axis results are ANDed.  Same boxes and
// comparisons as share_vertex + ccd_subbox_mask (v and v + dv with dv = x1 - x0, min / max
// merges, inclusive bounds), with a third of the live values.

// shareVertex of the start positions (figures.cu:527-544): any vertex of i equal to one of
// j on every axis
template <class T>
__device__ __forceinline__ bool ccd_pair_shares_vertex(const T* __restrict__ x0, long long i, long long j) {
    const T* a0 = x0 + i * 9;
    const T* b0 = x0 + j * 9;
    uint32_t eq = 0x1ffu;       // vertex pairs (ia, jb) equal on every axis so far: bit 3 ia + jb
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        T av[3], bv[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            av[c] = __ldg(a0 + 3 * c + ax);
            bv[c] = __ldg(b0 + 3 * c + ax);
        }
#pragma unroll
        for (int ia = 0; ia < 3; ++ia)
#pragma unroll
            for (int jb = 0; jb < 3; ++jb)
                if (!(av[ia] == bv[jb])) eq &= ~(1u << (3 * ia + jb));
    }
    return eq != 0u;
}

// The mask of sub-tests whose swept boxes overlap, for a pair that shares no vertex
// (REJECT_RIGID: 0 as well for a pair whose sub-tests can have no root, see the end; LEAF: 0
// as well for a pair whose leaf boxes do not overlap, the test of ccd_pair_leaf_overlap
// made from the same loads).
template <class T, bool REJECT_RIGID = true, bool LEAF = false>
__device__ __forceinline__ uint32_t ccd_pair_subbox_mask(const T* __restrict__ x0, const T* __restrict__ x1,
                                                         long long i, long long j) {
    const T* a0 = x0 + i * 9;
    const T* a1 = x1 + i * 9;
    const T* b0 = x0 + j * 9;
    const T* b1 = x1 + j * 9;
    uint32_t m = 0x7fffu;
    bool rigid = true;          // every vertex moves by the same displacement (on all axes so far)
    bool leaf = true;           // the leaf boxes overlap (on all axes so far)
    auto axis = [&](int ax) {
        T alo[3], ahi[3], blo[3], bhi[3], dv[6];
        T la = T(0), ha = T(0), lb = T(0), hb = T(0);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T av = __ldg(a0 + 3 * c + ax);
            const T aw = __ldg(a1 + 3 * c + ax);
            dv[c] = aw - av;
            T ae = av + dv[c];
            alo[c] = fmn(av, ae);
            ahi[c] = fmx(av, ae);
            T bv = __ldg(b0 + 3 * c + ax);
            const T bw = __ldg(b1 + 3 * c + ax);
            dv[3 + c] = bw - bv;
            T be = bv + dv[3 + c];
            blo[c] = fmn(bv, be);
            bhi[c] = fmx(bv, be);
            if constexpr (LEAF) {
                la = c ? fmn(la, fmn(av, aw)) : fmn(av, aw);
                ha = c ? fmx(ha, fmx(av, aw)) : fmx(av, aw);
                lb = c ? fmn(lb, fmn(bv, bw)) : fmn(bv, bw);
                hb = c ? fmx(hb, fmx(bv, bw)) : fmx(bv, bw);
            }
        }
        if constexpr (LEAF) leaf = leaf && la <= hb && ha >= lb;
        // the same displacement at all six vertices, finite, and start positions below half the
        // largest finite value so that every difference of two of them is finite too (the range
        // tests only where the displacements agree, which deforming pairs seldom do)
        bool same = true;
#pragma unroll
        for (int c = 1; c < 6; ++c) same = same && dv[c] == dv[0];
        rigid = rigid && same;
        if (rigid) {
            const T half_max = sizeof(T) == 4 ? T(1.7e38) : T(8.9e307);
            rigid = fabs(dv[0]) <= half_max;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                rigid = rigid && fabs(__ldg(a0 + 3 * c + ax)) <= half_max && fabs(__ldg(b0 + 3 * c + ax)) <= half_max;
        }
        // edges 01, 02, 12 and the face
        const T ealo[3] = {fmn(alo[0], alo[1]), fmn(alo[0], alo[2]), fmn(alo[1], alo[2])};
        const T eahi[3] = {fmx(ahi[0], ahi[1]), fmx(ahi[0], ahi[2]), fmx(ahi[1], ahi[2])};
        const T eblo[3] = {fmn(blo[0], blo[1]), fmn(blo[0], blo[2]), fmn(blo[1], blo[2])};
        const T ebhi[3] = {fmx(bhi[0], bhi[1]), fmx(bhi[0], bhi[2]), fmx(bhi[1], bhi[2])};
        const T falo = fmn(fmn(alo[0], alo[1]), alo[2]), fahi = fmx(fmx(ahi[0], ahi[1]), ahi[2]);
        const T fblo = fmn(fmn(blo[0], blo[1]), blo[2]), fbhi = fmx(fmx(bhi[0], bhi[1]), bhi[2]);
        uint32_t ma = 0;
#pragma unroll
        for (int e0 = 0; e0 < 3; ++e0)
#pragma unroll
            for (int e1 = 0; e1 < 3; ++e1)
                if (ealo[e0] <= ebhi[e1] && eahi[e0] >= eblo[e1]) ma |= 1u << (3 * e0 + e1);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (falo <= bhi[c] && fahi >= blo[c]) ma |= 1u << (9 + c);
            if (alo[c] <= fbhi && ahi[c] >= fblo) ma |= 1u << (12 + c);
        }
        m &= ma;
    };
    // (with the leaf test the axes go one at a time, which keeps the registers of a kernel
    // with several blocks an SM)
    if constexpr (LEAF) {
#pragma unroll 1
        for (int ax = 0; ax < 3; ++ax) axis(ax);
    } else {
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) axis(ax);
    }
    // A pair whose six vertices all move by the same finite displacement (a static or rigidly
    // translating piece), with finite position differences, has in every sub-test
    // displacement differences of exactly zero: the t^3 and t^2 coefficients are exactly 0
    // (every term has such a factor and finite other factors), and the reference drops the
    // root of that linear case (collisions_continuous.cu:531-535), so no sub-test of the pair
    // can give a row or a contact.
    return (REJECT_RIGID && rigid) || !leaf ? 0u : m;
}

// Whether the pair's leaf boxes (each triangle's boxes at x0 and x1 merged,
// MergeTriBoundingBoxes, build_bvh.cu:452-460) overlap (checkOverlap, aabb.cu:107-111), one
// axis at a time; fmin / fmax skip NaN and the comparisons do not tell -0 from +0, so the
// order of the reductions does not change the answer.
template <class T>
__device__ __forceinline__ bool ccd_pair_leaf_overlap(const T* __restrict__ x0, const T* __restrict__ x1, long long i,
                                                      long long j) {
    bool ov = true;
#pragma unroll 1
    for (int ax = 0; ax < 3; ++ax) {
        T la = __ldg(x0 + i * 9 + ax), ha = la, lb = __ldg(x0 + j * 9 + ax), hb = lb;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T a0 = __ldg(x0 + i * 9 + 3 * c + ax), a1 = __ldg(x1 + i * 9 + 3 * c + ax);
            const T b0 = __ldg(x0 + j * 9 + 3 * c + ax), b1 = __ldg(x1 + j * 9 + 3 * c + ax);
            la = fmn(la, fmn(a0, a1));
            ha = fmx(ha, fmx(a0, a1));
            lb = fmn(lb, fmn(b0, b1));
            hb = fmx(hb, fmx(b0, b1));
        }
        ov = ov && la <= hb && ha >= lb;
    }
    return ov;
}

// 0 when the triangles share a vertex, else ccd_pair_subbox_mask
template <class T, bool REJECT_RIGID = true>
__device__ __forceinline__ uint32_t ccd_pair_mask(const T* __restrict__ x0, const T* __restrict__ x1, long long i,
                                                  long long j) {
    if (ccd_pair_shares_vertex<T>(x0, i, j)) return 0u;
    return ccd_pair_subbox_mask<T, REJECT_RIGID>(x0, x1, i, j);
}

// The same table packed into constants, so a runtime type k selects points without
// indexing local arrays: side(k, p) = bit 4k + p of CCD_SIDE_TABLE, corner(k, p) = the
// 2-bit field 8 (k % 8) + 2p of CCD_CORNER_TABLE[k / 8].
constexpr int ccd_side_of(int k, int p) { return k < 9 ? (p >= 2) : (k < 12 ? (p == 3) : (p >= 1)); }
constexpr int ccd_corner_of(int k, int p) {
    return k < 9 ? (p == 0 ? (k / 3 == 2 ? 1 : 0) : p == 1 ? (k / 3 == 0 ? 1 : 2)
                    : p == 2 ? (k % 3 == 2 ? 1 : 0) : (k % 3 == 0 ? 1 : 2))
         : k < 12 ? (p < 3 ? p : k - 9)
                  : (p == 0 ? k - 12 : p - 1);
}
constexpr unsigned long long ccd_side_table() {
    unsigned long long t = 0;
    for (int k = 0; k < 15; ++k)
        for (int p = 0; p < 4; ++p) t |= (unsigned long long)ccd_side_of(k, p) << (4 * k + p);
    return t;
}
constexpr unsigned long long ccd_corner_table(int half) {
    unsigned long long t = 0;
    for (int k = 8 * half; k < 15 && k < 8 * half + 8; ++k)
        for (int p = 0; p < 4; ++p) t |= (unsigned long long)ccd_corner_of(k, p) << (8 * (k - 8 * half) + 2 * p);
    return t;
}
constexpr unsigned long long CCD_SIDE_TABLE = ccd_side_table();
constexpr unsigned long long CCD_CORNER_TABLE0 = ccd_corner_table(0);
constexpr unsigned long long CCD_CORNER_TABLE1 = ccd_corner_table(1);
__device__ __forceinline__ int tet_side(int k, int p) { return (int)((CCD_SIDE_TABLE >> (4 * k + p)) & 1ull); }
__device__ __forceinline__ int tet_corner(int k, int p) {
    unsigned long long t = k < 8 ? CCD_CORNER_TABLE0 : CCD_CORNER_TABLE1;
    return (int)((t >> (8 * (k & 7) + 2 * p)) & 3ull);
}

template <class T> struct MTet { V3<T> v[4], dv[4]; };

// tetrahedron of sub-test k read straight from the two soups: the four points at t = 0 and
// their displacements x1 - x0 (make_tetrahedron, collisions_continuous.cu:36-124)
template <class T>
__device__ __forceinline__ MTet<T> load_tet(const T* __restrict__ x0, const T* __restrict__ x1, long long gi,
                                            long long gj, int k) {
    MTet<T> t;
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        long long o = (tet_side(k, p) ? gj : gi) * 9 + tet_corner(k, p) * 3;
        V3<T> a = mk<T>(__ldg(x0 + o), __ldg(x0 + o + 1), __ldg(x0 + o + 2));
        V3<T> b = mk<T>(__ldg(x1 + o), __ldg(x1 + o + 1), __ldg(x1 + o + 2));
        t.v[p] = a;
        t.dv[p] = b - a;
    }
    return t;
}

template <class T> __device__ __forceinline__ MTet<T> make_tet(const MTri<T>& a, const MTri<T>& b, int k) {
    int side[4], corner[4];
    type_points(k, side, corner);
    MTet<T> t;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const MTri<T>& s = side[i] ? b : a;
        t.v[i] = s.v[corner[i]];
        t.dv[i] = s.dv[corner[i]];
    }
    return t;
}

// MovingTetraMatrix::coef3..coef0 (figures.cu:122-293): exact term order, summed from 0
template <class T> __device__ __forceinline__ void cubic_coeffs(const MTet<T>& t, T c[4]) {
    V3<T> v0 = t.v[0] - t.v[3], v1 = t.v[1] - t.v[3], v2 = t.v[2] - t.v[3];
    V3<T> dv0 = t.dv[0] - t.dv[3], dv1 = t.dv[1] - t.dv[3], dv2 = t.dv[2] - t.dv[3];
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

#define CCC_EPS 1e-16   // EPSILON (flags.h:36-38)

// add_root (collisions_continuous.cu:448-464): the root arrives converted to T
template <class T> __device__ __forceinline__ void add_root(T r[3], T x, int& nr) {
    if (x < -CCC_EPS || x > 1 + CCC_EPS) return;
    if (nr < 3) r[nr] = x;
    nr++;
}

// solveCubic with computeG / computeH (collisions_continuous.cu:472-613), in two parts: the
// prefix classifies (c3, c2, c1, c0) = (a, b, c, d) and computes g and h, and one function
// per branch produces its roots.  solve_cubic chains them; the continuous narrow phase
// calls the parts separately so that a warp solves one branch at a time.
// lib (MathLib) is a template parameter so that each kernel carries one solver variant.
enum CubicClass {
    CUBIC_NONE = 0,      // linear: the reference never stores its root
    CUBIC_QUAD = 1,      // |a| < EPSILON
    CUBIC_TRIPLE = 2,    // f = g = h = 0
    CUBIC_THREE = 3,     // h <= 0: three real roots (trigonometric form)
    CUBIC_ONE = 4,       // h > 0 (or NaN): one real root
};

template <int lib>
__device__ __forceinline__ int cubic_prefix(double a, double b, double c, double d, double& g, double& h) {
    g = h = 0.0;
    if (a == 0 && b == 0) return CUBIC_NONE;
    if (fabs(a) < CCC_EPS) return CUBIC_QUAD;
    double f = ((3.0 * c / a) - ((b * b) / (a * a))) / 3.0;
    double b3 = 2 * ccc_cube_hi(b);
    ccc_dd a2dd = ccc_sq_dd(a);
    double a2 = a2dd.hi;
    double a3 = ccc_certmul2_hi(a2dd.hi, a2dd.lo, a);
    double p1 = b3 / a3;
    double p2 = (b * c * 9) / a2;
    double p3 = 27.0 * d / a;
    g = (p1 - p2 + p3) / 27.0;
    double f3 = ccc_cube_hi(f);
    // the reference's pow(g, 2) resolves (through std::pow's promotion) to CUDA's general
    // pow(double, double), which is not always the rounded square
    // the reference's pow(g, 2) resolves (through std::pow's promotion) to CUDA's general
    // pow(double, double), which is not always the rounded square; CUDA's pow itself depends
    // on the contraction setting it is compiled with, and the narrow phase is compiled with
    // the reference's (ccc_narrow.cu).  g2 / 4 is exact.
    double g2 = lib == LIB_REFERENCE ? pow(g, 2.0) : mulrn(g, g);
    h = addrn(mulrn(g2, 0.25), f3 / 27.0);
    if (f == 0 && g == 0 && h == 0) return CUBIC_TRIPLE;
    return h <= 0 ? CUBIC_THREE : CUBIC_ONE;
}

template <class T> __device__ __forceinline__ void quad_roots(double b, double c, double d, T r[3], int& nr) {
    double D = fmaT(c, c, -(4.0 * b * d));
    if (D >= 0) {
        D = ccc_sqrt(D);
        double x1 = (-c + D) / (2.0 * b);
        double x2 = (-c - D) / (2.0 * b);
        add_root<T>(r, (T)x1, nr);
        add_root<T>(r, (T)x2, nr);
    }
}

template <class T, int lib> __device__ __forceinline__ void triple_roots(double a, double d, T r[3], int& nr) {
    float k = (float)(d / a);
    double x1;
    float cr = lib == LIB_REFERENCE ? cbrtf(k >= 0 ? k : -k) : ccc_cbrtf(k >= 0 ? k : -k);
    if (k >= 0) x1 = (double)(cr * -1);
    else x1 = (double)cr;
    add_root<T>(r, (T)x1, nr);
}

template <class T, int lib>
__device__ __forceinline__ void three_roots(double a, double b, double g, double h, T r[3], int& nr) {
    double i = ccc_sqrt(subrn(mulrn(mulrn(g, g), 0.25), h));
    double j, k, M, sn;
    if (lib == LIB_REFERENCE) {
        j = cbrt(i);
        k = acos(-(g / (2 * i)));
        M = cos(k / 3.0);
        sn = sin(k / 3.0);
    } else {
        j = ccc_cbrt(i);
        k = ccc_acos(-(g / (2 * i)));
        M = ccc_cos(k / 3.0);
        sn = ccc_sin(k / 3.0);
    }
    // N = sqrt(3) * sin(k/3) is fused into M + N and M - N and each result into
    // L * (.) + P; the first root 2 j cos(k/3) - b/(3a) is rounded twice (unfused)
    const double r3 = ccc_sqrt(3.0);
    double L = j * -1;
    double P = (b / (3.0 * a)) * -1;
    double x1 = subrn(mulrn(2 * j, M), b / (3.0 * a));
    double x2 = fmaT(L, fmaT(r3, sn, M), P);
    double x3 = fmaT(L, fmaT(-r3, sn, M), P);
    add_root<T>(r, (T)x1, nr);
    add_root<T>(r, (T)x2, nr);
    add_root<T>(r, (T)x3, nr);
}

template <class T, int lib>
__device__ __forceinline__ void one_root(double a, double b, double g, double h, T r[3], int& nr) {
    const double hg = mulrn(g, 0.5);      // g / 2, exact
    double R = addrn(-hg, ccc_sqrt(h));
    double S, U;
    double Ra = R >= 0 ? R : -R;
    S = lib == LIB_REFERENCE ? cbrt(Ra) : ccc_cbrt(Ra);
    if (R < 0) S = -S;
    double V = subrn(-hg, ccc_sqrt(h));
    double Va = V >= 0 ? V : -V;
    U = lib == LIB_REFERENCE ? cbrt(Va) : ccc_cbrt(Va);
    if (V < 0) U = -U;
    double x1 = (S + U) - (b / (3.0 * a));
    add_root<T>(r, (T)x1, nr);
}

// roots of one class; r starts at -1
template <class T, int lib>
__device__ __forceinline__ void class_roots(int cls, double a, double b, double c, double d, double g, double h,
                                            T r[3]) {
    r[0] = r[1] = r[2] = (T)-1;
    int nr = 0;
    switch (cls) {
        case CUBIC_QUAD: quad_roots<T>(b, c, d, r, nr); break;
        case CUBIC_TRIPLE: triple_roots<T, lib>(a, d, r, nr); break;
        case CUBIC_THREE: three_roots<T, lib>(a, b, g, h, r, nr); break;
        case CUBIC_ONE: one_root<T, lib>(a, b, g, h, r, nr); break;
        default: break;
    }
}

template <class T, int lib> __device__ __noinline__ void solve_cubic(double a, double b, double c, double d, T r[3]) {
    double g, h;
    int cls = cubic_prefix<lib>(a, b, c, d, g, h);
    class_roots<T, lib>(cls, a, b, c, d, g, h, r);
}

// is_inside (collisions_continuous.cu:615-637)
template <class T> __device__ __forceinline__ bool is_inside(V3<T> v0, V3<T> v1, V3<T> v2, V3<T> vt) {
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

template <class T> __device__ __forceinline__ V3<T> at_time(const MTet<T>& t, int i, T root) { return axpy(t.v[i], t.dv[i], root); }

// filterCollisions (collisions_continuous.cu:640-684)
template <class T> __device__ __forceinline__ bool ccd_filter(const MTet<T>& tet, int k, T root) {
    if (root < -(T)CCC_EPS) return false;
    V3<T> p0 = at_time(tet, 0, root), p1 = at_time(tet, 1, root), p2 = at_time(tet, 2, root), p3 = at_time(tet, 3, root);
    if (k < 9) {
        V3<T> da = p1 - p0, db = p3 - p2, dc = p2 - p0;
        T s = dot(cross(dc, db), cross(da, db)) / norm2(cross(da, db));
        T p = dot(cross(dc, da), cross(da, db)) / norm2(cross(da, db));
        if (s < 0 || s > 1 || p < 0 || p > 1) return false;
        return true;
    }
    // face then vertex: (p0, p1, p2 | p3) for k < 12, (p1, p2, p3 | p0) after, picked by
    // selects so that both kinds run one code path
    const bool inv = k >= 12;
    return is_inside(inv ? p1 : p0, inv ? p2 : p1, inv ? p3 : p2, inv ? p0 : p3);
}

// ------------------------------------------------------------------ impulses

#define CCC_THICKNESS 2e-3   // collisions_impulses.cu:12-14

// normalize(double3) = a * rsqrt(|a|^2) (utils.cu:91-93); the portable form uses 1 / sqrt
template <int lib> __device__ __forceinline__ float rsqrt_lib(float n) { return lib == LIB_REFERENCE ? rsqrtf(n) : 1.0f / sqrtf(n); }
template <int lib> __device__ __forceinline__ double rsqrt_lib(double n) { return lib == LIB_REFERENCE ? rsqrt(n) : 1.0 / ccc_sqrt(n); }
template <int lib, class T> __device__ __forceinline__ V3<T> vnormalize(V3<T> a) {
    T n = norm2(a);
    return a * rsqrt_lib<lib>(n);
}

template <class T> struct Contact { V3<T> n; T vn, m0, m1; };

// compute_coeficients_and_directions and helpers (collisions_impulses.cu:162-543).
// q holds the masses of the four tetrahedron points.  For vertex-face types the points
// are first put in (face 0, face 1, face 2, vertex) order with selects: types 9..11 are
// already in that order, types 12..14 have the vertex first.
template <class T, int lib> __device__ __forceinline__ Contact<T> contact(const MTet<T>& tet, int k, T root, const T q[4]) {
    Contact<T> ct;
    if (k < 9) {
        V3<T> th0 = at_time(tet, 0, root), th1 = at_time(tet, 1, root), th2 = at_time(tet, 2, root),
              th3 = at_time(tet, 3, root);
        V3<T> da = th1 - th0, db = th3 - th2, dc = th2 - th0;
        T denom = norm2(cross(da, db));
        T s, t;
        if (fabs((double)denom) < 1e-15) { s = (T)0.5; t = (T)0.5; }
        else {
            s = dot(cross(dc, db), cross(da, db)) / norm2(cross(da, db));
            t = dot(cross(dc, da), cross(da, db)) / norm2(cross(da, db));
        }
        const V3<T>* v = tet.v;
        const V3<T>* dv = tet.dv;
        V3<T> p0 = axpy(v[0], v[1] - v[0], s);
        V3<T> p1 = axpy(v[2], v[3] - v[2], t);
        V3<T> dp0 = axpy(dv[0], dv[1] - dv[0], s);
        V3<T> dp1 = axpy(dv[2], dv[3] - dv[2], t);
        V3<T> c0 = axpy(v[0], dv[0], root), c1 = axpy(v[1], dv[1], root), c2 = axpy(v[2], dv[2], root);
        V3<T> nd = vnormalize<lib>(cross(c1 - c0, c2 - c0));
        if (dot(p1 - p0, nd) < 0) nd = nd * (T)-1;
        ct.n = nd;
        ct.vn = dot(dp1 - dp0, nd);
        ct.m0 = fmaT(q[0], 1 - s, q[1] * s);
        ct.m1 = fmaT(q[2], 1 - t, q[3] * t);
        return ct;
    }
    const bool inv = k >= 12;
    V3<T> F0 = inv ? tet.v[1] : tet.v[0], F1 = inv ? tet.v[2] : tet.v[1], F2 = inv ? tet.v[3] : tet.v[2],
          FV = inv ? tet.v[0] : tet.v[3];
    V3<T> D0 = inv ? tet.dv[1] : tet.dv[0], D1 = inv ? tet.dv[2] : tet.dv[1], D2 = inv ? tet.dv[3] : tet.dv[2],
          DV = inv ? tet.dv[0] : tet.dv[3];
    T q0 = inv ? q[1] : q[0], q1 = inv ? q[2] : q[1], q2 = inv ? q[3] : q[2], qv = inv ? q[0] : q[3];
    V3<T> t0 = axpy(F0, D0, root), t1 = axpy(F1, D1, root), t2 = axpy(F2, D2, root), tv = axpy(FV, DV, root);
    V3<T> e1 = t0 - t1, e2 = t2 - t1, ep = tv - t1;
    T d00 = dot(e1, e1), d01 = dot(e1, e2), d11 = dot(e2, e2), d20 = dot(ep, e1), d21 = dot(ep, e2);
    T denom = fms2(d00, d11, d01, d01);
    T u, w, vv;
    if (fabs((double)denom) < 1e-15) { u = (T)(1. / 3.); w = (T)(1. / 3.); }
    else {
        u = fms2(d11, d20, d01, d21) / denom;
        w = fms2(d00, d21, d01, d20) / denom;
    }
    vv = 1 - u - w;
    V3<T> pt = lin3(F0, u, F1, vv, F2, w);
    V3<T> dpt = lin3(D0, u, D1, vv, D2, w);
    V3<T> c0 = axpy(F0, D0, root), c1 = axpy(F1, D1, root), c2 = axpy(F2, D2, root);
    V3<T> nd = vnormalize<lib>(cross(c1 - c0, c2 - c0));
    if (dot(FV - pt, nd) < 0) nd = nd * (T)-1;
    ct.vn = dot(DV - dpt, nd);
    if (inv) nd = nd * (T)-1;
    ct.n = nd;
    T mface = fmaT(q2, w, fmaT(q0, u, q1 * vv));
    ct.m0 = inv ? qv : mface;
    ct.m1 = inv ? mface : qv;
    return ct;
}

// ------------------------------------------------------------------ triangle-edge helpers

// hasVertex (figures.cu:598-609): exact coordinate equality with one of the corners
template <class T> __device__ __forceinline__ bool has_vertex(const Tri<T>& t, V3<T> p) {
    return veq(t.v[0], p) || veq(t.v[1], p) || veq(t.v[2], p);
}

// Sub-test cid (0..5) of a candidate pair (a, b): cid < 3 takes edge cid % 3 of a against
// face b, cid >= 3 edge cid % 3 of b against face a; edge e runs from corner e to corner
// (e + 1) % 3 (collectTEIntersections / collectTECandidates, collisions_static.cu:465-586).
template <class T>
__device__ __forceinline__ void te_edge(const Tri<T>& a, const Tri<T>& b, int cid, Tri<T>& face, V3<T>& p0,
                                        V3<T>& p1, int& e) {
    const bool first = cid < 3;
    e = first ? cid : cid - 3;
    const int e1 = e == 2 ? 0 : e + 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) face.v[c] = first ? b.v[c] : a.v[c];
    const Tri<T>& t1 = first ? a : b;
    p0 = e == 0 ? t1.v[0] : (e == 1 ? t1.v[1] : t1.v[2]);
    p1 = e1 == 0 ? t1.v[0] : (e1 == 1 ? t1.v[1] : t1.v[2]);
}

// addTECollsion (collisions_static.cu:345-462): true, with (flag, coefficient), when edge
// p0-p1 crosses the face: flag 0 / coefficient 0 for an edge that starts at a corner of
// the face (cid < 3 only), flag -1 / the edge parameter t of the crossing otherwise.  NaN
// passes the range tests, as in the reference.
template <class T, int lib>
__device__ __forceinline__ bool te_intersect(const Tri<T>& face, V3<T> p0, V3<T> p1, int cid, int& flag, T& coef) {
    V3<T> e1 = face.v[1] - face.v[0], e2 = face.v[2] - face.v[0];
    bool s0 = has_vertex(face, p0), s1 = has_vertex(face, p1);
    if (s0 || s1) {
        if (cid > 2 || !s0) return false;
        flag = 0;
        coef = (T)0;
        return true;
    }
    V3<T> nrm = vnormalize<lib>(cross(e1, e2));
    V3<T> dir = p1 - p0;
    T en = dot(dir, nrm);
    if (en == 0) return false;
    T d = dot(nrm, face.v[0]);
    T t = (d - dot(nrm, p0)) / en;
    if (t < 0 || t > 1) return false;
    V3<T> x = axpy(p0, dir, t);
    V3<T> ep = x - face.v[0];
    // The reference's float build contracts the three dot products of the face's edges the
    // other way round, fma(z, z', fma(y, y', x x')), and the two with ep as dot() does; its
    // double build uses dot() for all five.  (Matched against the reference's rows on seeded
    // folds, where many crossings pass exactly through a triangle edge.)
    const bool f32 = sizeof(T) == 4;
    T d00 = f32 ? dot_zyx(e1, e1) : dot(e1, e1), d01 = f32 ? dot_zyx(e1, e2) : dot(e1, e2),
      d11 = f32 ? dot_zyx(e2, e2) : dot(e2, e2), d20 = dot(ep, e1), d21 = dot(ep, e2);
    T denom = fms2(d00, d11, d01, d01);
    if ((double)denom < 1e-15) return false;
    T v = fms2(d11, d20, d01, d21) / denom;
    T w = fms2(d00, d21, d01, d20) / denom;
    T u = (T)(1.0 - (double)v - (double)w);     // `1.0 - v - w`: a double expression for float T
    if (u < 0 || v < 0 || w < 0) return false;
    flag = -1;
    coef = t;
    return true;
}

// collectTECandidates / collectTECandidates2 (collisions_static.cu:525-586, icontour.cu:11-110):
// bit 0 = the sub-test is listed, bit 1 = listed as a loop node (the edge starts at a corner
// of the face).  The box test compares the face's box with the box of the face's own edge e
// (not of the tested edge), as the reference does.
template <class T> __device__ __forceinline__ int te_candidate(const Tri<T>& face, V3<T> p0, V3<T> p1, int cid, int e) {
    if (has_vertex(face, p0)) return cid < 3 ? 3 : 0;
    if (has_vertex(face, p1)) return 0;
    const int e1 = e == 2 ? 0 : e + 1;
    V3<T> q0 = e == 0 ? face.v[0] : (e == 1 ? face.v[1] : face.v[2]);
    V3<T> q1 = e1 == 0 ? face.v[0] : (e1 == 1 ? face.v[1] : face.v[2]);
    Box<T> b1;
    b1.lo = mk<T>(fmn(q0.x, q1.x), fmn(q0.y, q1.y), fmn(q0.z, q1.z));
    b1.hi = mk<T>(fmx(q0.x, q1.x), fmx(q0.y, q1.y), fmx(q0.z, q1.z));
    return overlap(tri_box(face), b1, (T)0) ? 1 : 0;
}

// extrapolate_impulses + extrapolate_impulses_dv (collisions_impulses.cu:609-1067): impulses of
// one contact added to the per-corner dv / dx sums and counters (F, 3, 3) / (F, 3)
// Impulse magnitudes of one contact: mag0 on the face / edge-0 side, mag1 on the other,
// and keep = 1 - max(root - offset, 0), the share of the step left after the contact.
template <class T> struct ImpulseScale { T mag0, mag1, keep; };

template <class T> __device__ __forceinline__ ImpulseScale<T> impulse_scale(const Contact<T>& ct, T root) {
    T offset;
    if (fabs((double)ct.vn) < 1e-15) offset = (T)0.1;
    else offset = (T)((2 * CCC_THICKNESS) / (double)(-ct.vn));
    offset = (T)fmin(fmax((double)offset, 0.), 1.);
    T msum = ct.m0 + ct.m1;
    T mf0, mf1;
    if (fabs((double)msum) < 1e-15) { mf0 = (T)0.5; mf1 = (T)0.5; }
    else { mf0 = ct.m0 / msum; mf1 = 1 - mf0; }
    ImpulseScale<T> sc;
    sc.mag0 = ct.vn * mf1;
    sc.mag1 = -ct.vn * mf0;
    sc.keep = 1 - (T)fmax((double)(root - offset), 0.);
    return sc;
}

// velocity change imp and position change idx of tetrahedron point pt
template <class T>
__device__ __forceinline__ void impulse_point(const MTet<T>& tet, int k, int pt, const Contact<T>& ct,
                                              const ImpulseScale<T>& sc, V3<T>& imp, V3<T>& idx) {
    T mag = (k < 9) ? (pt < 2 ? sc.mag0 : sc.mag1) : (k < 12 ? (pt < 3 ? sc.mag0 : sc.mag1) : (pt < 1 ? sc.mag0 : sc.mag1));
    imp = mk<T>(mulrn(ct.n.x, mag), mulrn(ct.n.y, mag), mulrn(ct.n.z, mag));
    // the point's displacement by value selects: a run-time index into tet would move the
    // whole tetrahedron to local memory
    const V3<T> d = pt == 0 ? tet.dv[0] : (pt == 1 ? tet.dv[1] : (pt == 2 ? tet.dv[2] : tet.dv[3]));
    V3<T> nv = d + imp;
    idx = (nv - d) * sc.keep;
}

// extrapolate_impulses + extrapolate_impulses_dv (collisions_impulses.cu:609-1067): impulses of
// one contact added to the per-corner dv / dx sums and counters (F, 3, 3) / (F, 3)
template <class T>
__device__ __forceinline__ void apply_impulse(const MTet<T>& tet, long long gi, long long gj, int k, T root,
                                              const Contact<T>& ct, T* dv_out, T* dx_out, int* cnt_out) {
    ImpulseScale<T> sc = impulse_scale(ct, root);
#pragma unroll
    for (int pt = 0; pt < 4; ++pt) {
        V3<T> imp, idx;
        impulse_point(tet, k, pt, ct, sc, imp, idx);
        long long tri = tet_side(k, pt) ? gj : gi;
        int corner = tet_corner(k, pt);
        T* d = dv_out + tri * 9 + corner * 3;
        atomicAdd(d + 0, imp.x); atomicAdd(d + 1, imp.y); atomicAdd(d + 2, imp.z);
        T* x = dx_out + tri * 9 + corner * 3;
        atomicAdd(x + 0, idx.x); atomicAdd(x + 1, idx.y); atomicAdd(x + 2, idx.z);
        atomicAdd(cnt_out + tri * 3 + corner, 1);
    }
}

// ------------------------------------------------------------------ proximity

template <class T> __device__ __forceinline__ bool prox_subbox(const Tri<T>& a, const Tri<T>& b, int k, T th) {
    int side[4], corner[4];
    type_points(k, side, corner);
    Box<T> b0, b1;
    if (k < 9) {
        b0 = merge(svbox(a, corner[0]), svbox(a, corner[1]));
        b1 = merge(svbox(b, corner[2]), svbox(b, corner[3]));
    } else if (k < 12) {
        b0 = tri_box(a);
        b1 = svbox(b, k - 9);
    } else {
        b0 = svbox(a, k - 12);
        b1 = tri_box(b);
    }
    return overlap(b0, b1, th);
}

// vec_sq_diff returns float (utils.cu:57-61); the distance is sqrt in float
template <class T> __device__ __forceinline__ float sq_diff_f(V3<T> a, V3<T> b) { V3<T> d = a - b; return (float)dot(d, d); }

template <class T> __device__ __forceinline__ void pt_seg(V3<T> p, V3<T> a, V3<T> b, T dc[3], bool set_s, T second) {
    V3<T> ab = b - a, ap = p - a;
    T t = dot(ap, ab) / dot(ab, ab);
    if (t < (T)0.0) t = (T)0.0;
    if (t > (T)1.0) t = (T)1.0;
    V3<T> c = mk<T>(fmaT(t, ab.x, a.x), fmaT(t, ab.y, a.y), fmaT(t, ab.z, a.z));
    T nd = (T)__fsqrt_rn(sq_diff_f(p, c));
    if (nd < dc[0]) {
        dc[0] = nd;
        if (set_s) { dc[1] = t; dc[2] = second; }
        else { dc[2] = t; dc[1] = second; }
    }
}

// compute_distance_edge_edge / compute_distance_triangle_node (proximity_static.cu:205-433)
template <class T> __device__ __forceinline__ T prox_distance(const Tri<T>& a, const Tri<T>& b, int k) {
    int side[4], corner[4];
    type_points(k, side, corner);
    V3<T> v[4];
#pragma unroll
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
        return (T)__fsqrt_rn(sq_diff_f(axpy(v[0], da, s), axpy(v[2], db, t)));
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
    return (T)__fsqrt_rn(sq_diff_f(v[fv], pt));
}

}  // namespace ccc
