/* ccc_b200.h — C ABI of the B200 collision engine.
 *
 * Each entry point replaces one host routine of the reference torch extension
 * (Dolorousrtur/CCCollisions, src/cccollisions.cpp and the L2 host functions it calls).
 * Conventions shared by every call:
 *   - dtype: 0 = float32, 1 = float64 (the reference dispatches on both,
 *     AT_DISPATCH_FLOATING_TYPES).
 *   - All array arguments are DEVICE pointers to contiguous arrays in the reference's
 *     tensor layouts: triangles (B, F, 3, 3); bboxes (B, 2F-1, 6) of dtype; tree
 *     (B, 2F-1, 4) int64 with rows (parent, left, right, triangle id); masks (B, F) uint8.
 *   - Outputs are written in place.  Row outputs must be pre-filled with -1 by the caller
 *     (the reference allocates them as -1 * ones); impulse outputs must be zeroed.
 *   - ws / ws_bytes: caller-provided device scratch of at least the size returned by the
 *     matching *_workspace_size call.  The library makes no device allocations at run time;
 *     it does keep one fixed module-data array of ccc_static_scratch_bytes() (64 MiB) on
 *     every device where it is loaded (the scratch of ccc_find_collisions_continuous_static),
 *     which device-memory budgets should leave room for.
 *   - stream: a cudaStream_t (NULL = legacy default stream).  Calls are asynchronous;
 *     ccc_read_status() synchronises the stream and returns the device status word.
 *   - Return value: 0 on success or a CCC_ERR_* code for argument / launch errors.
 *     Capacity overflows are reported through the status word (bits below), as the
 *     reference prints a warning and truncates.
 *   - Threads: the entry points may be called from several host threads at once, each
 *     with its own workspace (and stream); ccc_find_collisions_continuous_static shares one
 *     device array between its calls.  The math-library mode and the timing hooks are
 *     process-wide settings: set them while no other thread is launching.  The launch
 *     count is exact when one thread launches at a time.
 */
#ifndef CCC_B200_H
#define CCC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* return codes */
#define CCC_OK 0
#define CCC_ERR_INVALID_ARG 1
#define CCC_ERR_WORKSPACE 2
#define CCC_ERR_CUDA 3
#define CCC_ERR_TOO_LARGE 4

/* status word bits (device side, read with ccc_read_status) */
#define CCC_ST_CAND_OVERFLOW 1   /* more candidate pairs than F * max_candidates_per_triangle */
#define CCC_ST_OUT_OVERFLOW 2    /* more result rows than the output holds (rows truncated)   */
#define CCC_ST_STACK_OVERFLOW 4  /* traversal deeper than the 64-entry stack                  */
#define CCC_ST_MALFORMED_TREE 8  /* tree tensor indices out of range or cyclic                */

/* operation ids for ccc_workspace_size */
#define CCC_OP_BVH 0
#define CCC_OP_FIND_COLLISIONS 1
#define CCC_OP_CONTINUOUS 2
#define CCC_OP_PROXIMITY 3
#define CCC_OP_IMPULSES 4
#define CCC_OP_MINCOL 5

int ccc_version(void);
const char* ccc_error_string(int code);

/* Instrumentation (no counterpart in the reference, which has no tracing): the number of
 * kernels this library has launched since load, and optional per-kernel CUDA-event timing.
 * Between ccc_timing_begin and ccc_timing_end every launch is bracketed by events on its
 * stream; ccc_timing_end synchronises on the last event and returns the number of distinct
 * kernels, writing their names (name_len bytes each), summed milliseconds and launch counts. */
int64_t ccc_kernel_launches(void);
int ccc_timing_begin(void);
int ccc_timing_end(int max_kernels, char* names, int name_len, float* total_ms, int32_t* count);

/* Elementary functions used by the continuous-collision solver and the impulse normals
 * (no counterpart in the reference, which always uses CUDA's): CCC_LIB_REFERENCE (default)
 * calls CUDA's cbrt, acos, cos, sin, pow and rsqrt exactly where the reference does;
 * CCC_LIB_PORTABLE uses this library's own implementations, which the CPU oracle shares
 * bit for bit.  Process-wide; returns CCC_ERR_INVALID_ARG for other values. */
#define CCC_LIB_REFERENCE 0
#define CCC_LIB_PORTABLE 1
int ccc_set_math_library(int lib);
int ccc_get_math_library(void);

/* Test hook (no counterpart in the reference): one stage of the continuous narrow phase on
 * caller tetrahedra (device arrays; rows of in_stride / out_stride doubles).  op 0: cubic
 * coefficients of (v0..v3, dv0..dv3) -> (c3, c2, c1, c0); op 1: cubic solve of
 * (c3, c2, c1, c0) -> three roots (-1 = none); op 2: root filter of (tet, type, root) ->
 * 1 / 0; op 3: contact kinematics of (tet, type, root, four masses) -> (normal, normal
 * velocity, mass pair).  lib: CCC_LIB_REFERENCE or CCC_LIB_PORTABLE. */
int ccc_debug_stage(int op, int lib, const double* in, int in_stride, double* out, int out_stride, int64_t n,
                    void* stream);

/* Test hook (no counterpart in the reference): evaluates the continuous-collision solver's
 * arithmetic element-wise on the device so tests can compare it with the CPU oracle.
 * op: 0 cbrt, 1 acos, 2 cos, 3 sin (the library's own), 4 certified product
 * (in x0, x1, k, y -> out r0, r1), 5 cubic solve (in a, b, c, d -> out three roots,
 * -1 = none), 6..9 CUDA's cbrt, acos, cos, sin.  in: n x 4 doubles, out: n x 3 doubles
 * (device pointers). */
int ccc_debug_math(int op, const double* in, double* out, int64_t n, void* stream);

/* Bytes of device scratch an operation needs for B meshes of F triangles with the given
 * per-triangle candidate capacity (ignored by CCC_OP_BVH). */
int64_t ccc_workspace_size(int op, int64_t B, int64_t F, int64_t max_candidates_per_triangle);

/* Copies the status word, the candidate count and up to n_mesh per-mesh row counts from
 * the workspace to host memory (synchronises the stream).  out must hold 2 + n_mesh ints. */
int ccc_read_status(const void* ws, int64_t n_mesh, int32_t* out, void* stream);

/* Work counters of the last operation on a workspace (no counterpart in the reference):
 * synchronises the stream and writes 4 ints: status word, candidate pairs, continuous
 * sub-tests solved, roots in [0, 1] filtered. */
int ccc_read_counters(const void* ws, int32_t* out, void* stream);

/* bvh / bvh_motion — replaces build_bvh(triangles[, triangles_next], &bboxes, &tree)
 * (src/build_bvh.cu:381-449, 570-648; bindings src/cccollisions.cpp:102-132).
 * triangles_next may be NULL (static build).  Writes every row of bboxes and tree in the
 * reference's order: the reference's unbounded scene box gives all-zero Morton codes, so
 * leaf position p holds triangle p. */
int ccc_bvh(int dtype, const void* triangles, const void* triangles_next, int64_t B, int64_t F, void* bboxes,
            int64_t* tree, void* ws, int64_t ws_bytes, void* stream);

/* find_collisions — replaces find_collisions_from_bbox_tree (src/collisions_static.cu:
 * 206-342; binding src/cccollisions.cpp:134-148).  out: (B, F*max_collisions, 2) int64,
 * pre-filled with -1; intersecting pairs (i, j), i < j, are packed at the front. */
int ccc_find_collisions(int dtype, const void* bboxes, const int64_t* tree, const void* triangles, int64_t B,
                        int64_t F, double threshold, int64_t max_collisions, int64_t* out, void* ws,
                        int64_t ws_bytes, void* stream);

/* find_triangle_edge_collisions — replaces find_triangle_edge_collisions_from_bbox_tree
 * (src/collisions_static.cu:588-720, kernels 345-522; binding src/cccollisions.cpp:151-173).
 * Candidate pairs with threshold 0, kept when they intersect and share no vertex; then six
 * edge sub-tests per pair (cid 0..2: edge (v0v1, v1v2, v2v0)[cid] of triangle i against
 * face j; 3..5: edge cid-3 of j against face i).  out_rows (B, F*max_collisions, 4) int64
 * (i, j, cid, flag) and out_coefs (B, F*max_collisions, 1) of dtype (edge parameter of the
 * crossing), both pre-filled with -1; rows are packed at the front of each mesh's slice.
 * The reference copies item b's rows to offset b*F*max_collisions*3 of the 4-wide tensor
 * (collisions_static.cu:763) and copies 6 rows per intersecting pair even past the tensor's
 * end; here each item has its own slice, and rows past the capacity are dropped with
 * CCC_ST_OUT_OVERFLOW in the status word. */
int ccc_find_triangle_edge_collisions(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                      int64_t B, int64_t F, int64_t max_collisions, int64_t* out_rows,
                                      void* out_coefs, void* ws, int64_t ws_bytes, void* stream);

/* find_triangle_edge_candidates — replaces find_triangle_edge_candidates
 * (src/collisions_static.cu:723-942, kernel 525-586; binding src/cccollisions.cpp:176-194).
 * Pairs sharing at most one vertex; per sub-test a row (i, j, cid, 0) when the edge starts
 * at a corner of the face (cid < 3 only), else (i, j, cid, -1) when the face's box overlaps
 * the box of the face's own edge cid % 3.  out_rows (B, F*max_collisions, 4), pre-filled -1. */
int ccc_find_triangle_edge_candidates(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                      int64_t B, int64_t F, int64_t max_collisions, int64_t* out_rows, void* ws,
                                      int64_t ws_bytes, void* stream);

/* find_triangle_edge_candidates2 — replaces find_triangle_edge_candidates2
 * (src/icontour.cu:113-281, kernel 11-110; binding src/cccollisions.cpp:197-218).  The
 * pairs of find_triangle_edge_candidates, one row each: out_pairs (B, F*max_collisions, 2)
 * int64 pre-filled with -1, out_binmasks (B, F*max_collisions, 2) int32 pre-filled with 0:
 * bit cid of x when sub-test cid is listed, of y when it is a loop node. */
int ccc_find_triangle_edge_candidates2(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                       int64_t B, int64_t F, int64_t max_collisions, int64_t* out_pairs,
                                       int32_t* out_binmasks, void* ws, int64_t ws_bytes, void* stream);

/* find_collisions_continuous / find_collisions_continuous_partial — replaces
 * find_collisions_from_bbox_tree (CCD overload, src/collisions_continuous.cu:814-1076) and
 * find_collisions_from_bbox_tree_partial (1103-1376); bindings src/cccollisions.cpp:220-273.
 * mask: NULL, or (B, F) uint8 triangles_to_check.  out_rows (B, F*max_col, 3) int64 and
 * out_times (B, F*max_col, 1) of dtype, both pre-filled with -1. */
int ccc_find_collisions_continuous(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                   const void* triangles_next, const uint8_t* mask, int64_t B, int64_t F,
                                   int64_t max_candidates_per_triangle, int64_t max_collisions_per_triangle,
                                   int64_t* out_rows, void* out_times, void* ws, int64_t ws_bytes, void* stream);

/* find_mincol_cand — replaces find_minimal_candidates_from_bbox_tree
 * (src/collisions_continuous.cu:1379-1519; binding src/cccollisions.cpp:405-423).
 * out_rows (B, F*max_collisions*15, 3) int64, pre-filled with -1. */
int ccc_find_mincol_cand(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                         const void* triangles_next, int64_t B, int64_t F, int64_t max_collisions, int64_t* out_rows,
                         void* ws, int64_t ws_bytes, void* stream);

/* find_proximity — replaces find_proximity_from_bbox_tree (src/proximity_static.cu:510-694;
 * binding src/cccollisions.cpp:276-296).  out_rows (B, F*max_cand, 3) int64, pre-filled -1. */
int ccc_find_proximity(int dtype, const void* bboxes, const int64_t* tree, const void* triangles, int64_t B,
                       int64_t F, double threshold, int64_t max_candidates_per_triangle, int64_t* out_rows, void* ws,
                       int64_t ws_bytes, void* stream);

/* compute_impulses / compute_impulses_partial — replaces collision_impulses_from_bbox_tree
 * (src/collisions_impulses.cu:1069-1397) and its _partial variant (1402-1734); bindings
 * src/cccollisions.cpp:299-370.  masses (B, F, 3) of dtype; mask NULL or (B, F) uint8.
 * dv, dx (B, F, 3, 3) of dtype and counter (B, F, 3) int32, all zero-filled. */
int ccc_compute_impulses(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                         const void* triangles_next, const void* masses, const uint8_t* mask, int64_t B, int64_t F,
                         int64_t max_candidates_per_triangle, int64_t max_collisions_per_triangle, void* dv, void* dx,
                         int32_t* counter, void* ws, int64_t ws_bytes, void* stream);

/* compute_impulses_from_collisions — replaces collision_impulses_from_continuous_collisions
 * (src/collisions_impulses.cu:1738-1880; binding src/cccollisions.cpp:374-403).
 * collisions (B, N, 3) int64, roots (B, N, 1) of dtype.  Rows with out-of-range indices
 * (such as the -1 padding) are skipped. */
int ccc_compute_impulses_from_collisions(int dtype, const int64_t* collisions, const void* roots, int64_t B,
                                         int64_t N, const void* triangles, const void* triangles_next,
                                         const void* masses, int64_t F, void* dv, void* dx, int32_t* counter,
                                         void* ws, int64_t ws_bytes, void* stream);

/* find_collisions_continuous without any scratch allocation — no counterpart in the
 * reference.  For callers that cannot allocate device memory (a plugin inside a host
 * framework that owns the GPU's memory through its own pool, or a real-time step loop that
 * forbids allocations): the same computation and outputs as ccc_find_collisions_continuous,
 * with its scratch in a fixed device array of ccc_static_scratch_bytes() bytes (64 MiB)
 * that every GPU loading this library holds until exit.  Problems whose scratch
 * (ccc_workspace_size(CCC_OP_CONTINUOUS, B, F, max_candidates_per_triangle)) exceeds it
 * return CCC_ERR_TOO_LARGE before any device work.  Every call looks up the array's device
 * address on the current device (cudaGetSymbolAddress, a host-side lookup, so a
 * cudaDeviceReset in between is harmless); the first call on a device also loads the
 * module's data there, so make it before any stream capture.  All calls share the array:
 * calls that overlap on the GPU race.  Outputs as for ccc_find_collisions_continuous
 * (pre-filled with -1 by the caller). */
int64_t ccc_static_scratch_bytes(void);
int ccc_find_collisions_continuous_static(int dtype, const void* bboxes, const int64_t* tree, const void* triangles,
                                          const void* triangles_next, const uint8_t* mask, int64_t B, int64_t F,
                                          int64_t max_candidates_per_triangle, int64_t max_collisions_per_triangle,
                                          int64_t* out_rows, void* out_times, void* stream);

/* ccc_read_status / ccc_read_counters for the last ccc_find_collisions_continuous_static
 * call on the current device (no counterpart in the reference): the status word (candidate
 * or output overflow, stack overflow, malformed tree), the candidate count and up to n_mesh
 * per-mesh row counts; or the four work counters.  They read the shared array, so call them
 * before the next static call is queued.  Synchronise the stream. */
int ccc_static_scratch_read_status(int64_t n_mesh, int32_t* out, void* stream);
int ccc_static_scratch_read_counters(int32_t* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CCC_B200_H */
