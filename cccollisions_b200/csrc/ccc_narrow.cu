// ccc_narrow.cu — the continuous narrow phase (k_ccd_narrow) and the solver's test hooks.
//
// This translation unit alone is compiled with nvcc's default multiply-add contraction
// (-fmad=true), as the reference extension is: the solver calls CUDA's pow, whose result on
// rare arguments depends on that setting (pow(g, 2.0) in the cubic's h differs by an ulp on
// about 6 in a million arguments under -fmad=false, which moved a root near t = 0 of a nearly
// coplanar sub-test).  The solver's other CUDA functions (cbrt, acos, cos, sin, cbrtf,
// rsqrt, rsqrtf) gave the same bits under both settings on 2^28 arguments each.  Every
// operation of this library's own reached from here rounds as written under either setting:
// products that feed sums are explicitly rounded (mulrn / addrn / subrn, ccc_mul / ccc_add /
// ccc_sub) or operands of explicit fused multiply-adds (fmaT / ccc_fma), which are never
// fused further.  The rest of the library is compiled with -fmad=false.
#define CCC_NARROW_TU
#include "../../include/ccc_b200.h"
#include "ccc_kernels.cuh"
#include "ccc_engine.cuh"
#include "ccc_runtime.cuh"

namespace ccc {

// the combinations the library launches: (type, mode, sink, math library)
#define CCC_NARROW_INSTANCE(T, MODE, SINK, LIB, SRC, BM)                                                         \
    template cudaError_t launch_ccd_narrow<T, MODE, SINK, LIB, SRC, BM>(int, cudaStream_t, const int2*, int,        \
                                                                           WsHeader*, const T*, const T*, Forest,      \
                                                                           long long*, T*, int, int*, Weld, SINK);     \
    template cudaError_t prepare_ccd_narrow<T, MODE, SINK, LIB, SRC, BM>();
#define CCC_NARROW_TYPES(MODE, SINK, LIB, SRC, BM)                                                              \
    CCC_NARROW_INSTANCE(float, MODE, SINK<float>, LIB, SRC, BM)                                                  \
    CCC_NARROW_INSTANCE(double, MODE, SINK<double>, LIB, SRC, BM)
// the reference-format operations (pairs from the candidate buffer), batches of 256
CCC_NARROW_TYPES(CCD_ROWS, CornerSink, LIB_REFERENCE, SRC_CANDIDATES, 1)
CCC_NARROW_TYPES(CCD_ROWS, CornerSink, LIB_PORTABLE, SRC_CANDIDATES, 1)
CCC_NARROW_TYPES(CCD_IMPULSES, CornerSink, LIB_REFERENCE, SRC_CANDIDATES, 1)
CCC_NARROW_TYPES(CCD_IMPULSES, CornerSink, LIB_PORTABLE, SRC_CANDIDATES, 1)
CCC_NARROW_TYPES(CCD_MINCOL, CornerSink, LIB_PORTABLE, SRC_CANDIDATES, 1)
// the resident engine's collision step (staged pairs, shared sub-tests), batches of 256 or
// 512, and its impulse loop (candidate buffer, the exact leaf-box test)
CCC_NARROW_TYPES(CCD_ROWS, CornerSink, LIB_REFERENCE, SRC_STAGED, 1)
CCC_NARROW_TYPES(CCD_ROWS, CornerSink, LIB_PORTABLE, SRC_STAGED, 1)
CCC_NARROW_TYPES(CCD_ROWS, CornerSink, LIB_REFERENCE, SRC_STAGED, 2)
CCC_NARROW_TYPES(CCD_ROWS, CornerSink, LIB_PORTABLE, SRC_STAGED, 2)
CCC_NARROW_TYPES(CCD_IMPULSES, LoopSink, LIB_REFERENCE, SRC_EXACT, 1)
CCC_NARROW_TYPES(CCD_IMPULSES, LoopSink, LIB_PORTABLE, SRC_EXACT, 1)

// Element-wise evaluation of the solver's arithmetic building blocks, for tests that compare
// them bit for bit with the CPU oracle and against CUDA's own elementary functions.
// op 0 cbrt, 1 acos, 2 cos, 3 sin, 4 certified product (in: x0, x1, k, y; out: r0, r1),
// 5 solve_cubic (in: a, b, c, d; out: three roots), 6 CUDA cbrt, 7 CUDA acos, 8 CUDA cos,
// 9 CUDA sin.  in has 4 doubles per element, out 3.
static __global__ void k_debug_math(int op, const double* __restrict__ in, double* __restrict__ out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* a = in + 4 * i;
    double* o = out + 3 * i;
    o[0] = o[1] = o[2] = 0.0;
    switch (op) {
        case 0: o[0] = ccc_cbrt(a[0]); break;
        case 1: o[0] = ccc_acos(a[0]); break;
        case 2: o[0] = ccc_cos(a[0]); break;
        case 3: o[0] = ccc_sin(a[0]); break;
        case 4: {
            ccc_dd d = ccc_certmul(a[0], a[1], (int)a[2], a[3]);
            o[0] = d.hi;
            o[1] = d.lo;
            break;
        }
        case 5: solve_cubic<double, LIB_PORTABLE>(a[0], a[1], a[2], a[3], o); break;
        case 6: o[0] = cbrt(a[0]); break;
        case 7: o[0] = acos(a[0]); break;
        case 8: o[0] = cos(a[0]); break;
        case 9: o[0] = sin(a[0]); break;
        case 10: case 11: {
            double A = a[0], Bc = a[1], Cc = a[2], Dc = a[3];
            double f = ((3.0 * Cc / A) - ((Bc * Bc) / (A * A))) / 3.0;
            double b3 = 2 * ccc_cube_hi(Bc);
            ccc_dd a2dd = ccc_sq_dd(A);
            double a3 = ccc_certmul(a2dd.hi, a2dd.lo, 2, A).hi;
            double g = (b3 / a3 - (Bc * Cc * 9) / a2dd.hi + 27.0 * Dc / A) / 27.0;
            double h = addrn(mulrn(mulrn(g, g), 0.25), ccc_cube_hi(f) / 27.0);
            if (op == 10) { o[0] = f; o[1] = g; o[2] = h; }
            else { o[0] = b3; o[1] = a2dd.hi; o[2] = a3; }
            break;
        }
        default: break;
    }
}

// Stages of the continuous narrow phase on caller tetrahedra (v0..v3, dv0..dv3 = 24
// doubles per element), for tests against the reference's own kernels and the oracle.
// op 0: cubic coefficients -> 4 doubles; op 1: cubic solve (in: 4 coefficients) -> 3
// roots; op 2: root filter (in: tet, type, root) -> 1.0 / 0.0; op 3: contact kinematics
// (in: tet, type, root, 4 masses) -> normal (3), normal velocity, mass pair (2).
// lib selects the elementary functions (MathLib).
static __global__ void k_debug_stage(int op, int lib, const double* __restrict__ in, int in_stride,
                              double* __restrict__ out, int out_stride, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* a = in + (long long)i * in_stride;
    double* o = out + (long long)i * out_stride;
    MTet<double> t;
    if (op != 1) {
        for (int p = 0; p < 4; ++p) {
            t.v[p] = mk<double>(a[3 * p], a[3 * p + 1], a[3 * p + 2]);
            t.dv[p] = mk<double>(a[12 + 3 * p], a[12 + 3 * p + 1], a[12 + 3 * p + 2]);
        }
    }
    if (op == 0) {
        cubic_coeffs(t, o);
    } else if (op == 1) {
        if (lib == LIB_REFERENCE) solve_cubic<double, LIB_REFERENCE>(a[0], a[1], a[2], a[3], o);
        else solve_cubic<double, LIB_PORTABLE>(a[0], a[1], a[2], a[3], o);
    } else if (op == 2) {
        o[0] = ccd_filter(t, (int)a[24], a[25]) ? 1.0 : 0.0;
    } else if (op == 4) {
        // (f, g, h) of the solver prefix for coefficients (c3, c2, c1, c0)
        double A = a[0], B = a[1], Cc = a[2], D = a[3];
        double f = ((3.0 * Cc / A) - ((B * B) / (A * A))) / 3.0;
        double b3 = 2 * ccc_cube_hi(B);
        ccc_dd a2dd = ccc_sq_dd(A);
        double a3 = ccc_certmul(a2dd.hi, a2dd.lo, 2, A).hi;
        double g = (b3 / a3 - (B * Cc * 9) / a2dd.hi + 27.0 * D / A) / 27.0;
        double g2 = lib == LIB_REFERENCE ? pow(g, 2.0) : mulrn(g, g);
        o[0] = f;
        o[1] = g;
        o[2] = addrn(mulrn(g2, 0.25), ccc_cube_hi(f) / 27.0);
    } else if (op == 5) {
        // squares of a[0]: pow(x, 2), pow(x, 2.0), x * x
        double x = a[0];
        volatile int two = 2;
        o[0] = pow(x, two);
        o[1] = pow(x, (double)two);
        o[2] = x * x;
    } else if (op == 3) {
        double q[4] = {a[26], a[27], a[28], a[29]};
        Contact<double> ct = lib == LIB_REFERENCE ? contact<double, LIB_REFERENCE>(t, (int)a[24], a[25], q)
                                                  : contact<double, LIB_PORTABLE>(t, (int)a[24], a[25], q);
        o[0] = ct.n.x; o[1] = ct.n.y; o[2] = ct.n.z; o[3] = ct.vn; o[4] = ct.m0; o[5] = ct.m1;
    }
}


cudaError_t launch_debug_math(int op, const double* in, double* out, int n, cudaStream_t s) {
    k_debug_math<<<grid_for(n, 128), 128, 0, s>>>(op, in, out, n);
    return cudaGetLastError();
}

cudaError_t launch_debug_stage(int op, int lib, const double* in, int in_stride, double* out, int out_stride, int n,
                               cudaStream_t s) {
    k_debug_stage<<<grid_for(n, 128), 128, 0, s>>>(op, lib, in, in_stride, out, out_stride, n);
    return cudaGetLastError();
}

}  // namespace ccc
