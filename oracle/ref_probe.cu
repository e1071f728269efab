// ref_probe.cu — TEST INFRASTRUCTURE: runs single stages of the reference's own device code.
//
// Compiled by oracle/build_ref.py together with the reference's sources (src/out.cu,
// included from the reference checkout) into oracle/_ref/libref_probe.so, with the
// reference's build flags (nvcc defaults: fused multiply-add contraction on).  Each entry
// point launches one reference kernel on caller device buffers and synchronises, so a
// script can record the reference's arithmetic stage by stage (cubic coefficients, roots,
// filters, contact kinematics) for tests/golden/.  Only straight-line kernels are exposed.
#include "out.cu"

// CAMPARY certifiedMul<1,1,2> / <2,1,2> and the solver's computeG / computeH
// (collisions_continuous.cu:472-507) on caller values
__global__ void probe_certmul(const double* in, double* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* a = in + 4 * i;
    double x[2] = {a[0], a[1]};
    double y = a[3];
    double r[2];
    if ((int)a[2] == 1) certifiedMul<1, 1, 2>(x, &y, r);
    else certifiedMul<2, 1, 2>(x, &y, r);
    out[2 * i] = r[0];
    out[2 * i + 1] = r[1];
}

__global__ void probe_fgh(const double* in, double* out, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = in[4 * i], b = in[4 * i + 1], c = in[4 * i + 2], d = in[4 * i + 3];
    double temp1[2], temp2[2];
    double f = ((3.0 * c / a) - ((b * b) / (a * a))) / 3.0;
    double g = computeG(a, b, c, d, &temp1[0], &temp2[0]);
    double h = computeH(g, f, &temp1[0], &temp2[0]);
    out[3 * i] = f;
    out[3 * i + 1] = g;
    out[3 * i + 2] = h;
}

extern "C" {

int ref_certmul(const double* in, double* out, int n) {
    probe_certmul<<<(n + 127) / 128, 128>>>(in, out, n);
    return (int)cudaDeviceSynchronize();
}

int ref_fgh(const double* in, double* out, int n) {
    probe_fgh<<<(n + 127) / 128, 128>>>(in, out, n);
    return (int)cudaDeviceSynchronize();
}

// getCubicCoeffs (collisions_continuous.cu:409-445): tets n x 24 doubles (MovingTetrahedron),
// coefs n x 4 (c3, c2, c1, c0)
int ref_cubic_coeffs(const double* tets, double* coefs, long long* scratch3, int n) {
    getCubicCoeffs<double><<<(n + 127) / 128, 128>>>((MovingTetrahedron<double>*)tets, (double4*)coefs,
                                                     (long3*)scratch3, n);
    return (int)cudaDeviceSynchronize();
}

// solveCubic (collisions_continuous.cu:511-613): coefs n x 4, roots n x 3 (pre-filled -1)
int ref_solve_cubic(const double* coefs, double* roots, int n) {
    solveCubic<double><<<(n + 127) / 128, 128>>>((double4*)coefs, (double3*)roots, n);
    return (int)cudaDeviceSynchronize();
}

// filterCollisions (collisions_continuous.cu:640-684): tets n x 24, tids n x 3 (type in z),
// roots n, valid n bools (pre-filled 0)
int ref_filter(const double* tets, const long long* tids, const double* roots, bool* valid, int n) {
    filterCollisions<double><<<(n + 127) / 128, 128>>>((MovingTetrahedron<double>*)tets, (long3*)tids,
                                                       (double*)roots, valid, n);
    return (int)cudaDeviceSynchronize();
}

// compute_coeficients_and_directions (collisions_impulses.cu:470-543)
int ref_contact(const double* tets, const long long* tids, const double* roots, const double* mass_quads,
                double* coefficients, double* normals, double* vn, double* vn_end, double* mass_pairs, int n) {
    compute_coeficients_and_directions<double><<<(n + 127) / 128, 128>>>(
        (MovingTetrahedron<double>*)tets, (long3*)tids, (double*)roots, (double4*)mass_quads, (double3*)coefficients,
        (double3*)normals, vn, vn_end, (double2*)mass_pairs, n);
    return (int)cudaDeviceSynchronize();
}

}  // extern "C"
