/* ccc_engine.h — resident multi-mesh collision engine (C ABI).
 *
 * The reference extension (src/cccollisions.cpp) handles one batch of equal-size meshes per
 * call and rebuilds and re-imports every tree on every call (src/build_bvh.cu:570-648,
 * 745-763).  The engine keeps meshes of uneven size resident on the device instead, each in
 * its own slot range of one caller-provided block of device memory, and runs each step
 * over all active meshes at once:
 *
 *   - ccc_engine_build: per-mesh LBVH topology (30-bit Morton codes of the swept centroids,
 *     device radix sort, Karras radix tree), once per mesh;
 *   - ccc_engine_ccd: refit + traversal + continuous narrow phase for every active mesh,
 *     rows and times of impact per mesh (the reference's find_collisions_continuous rows);
 *   - ccc_engine_loop_*: the impulse loop (compute impulses, apply them to the vertices,
 *     repeat until a collision check finds no contact or max_iter iterations), per mesh.
 *
 * The active set lives in a device-side mesh table, so a step captured once as a CUDA graph
 * (ccc_engine_capture) replays for any active set (ccc_engine_replay).  The library
 * allocates no device memory: the caller provides the block (ccc_engine_bytes).
 *
 * Shared conventions: dtype 0 = float32, 1 = float64 for positions; every call returns
 * CCC_OK (0) or a CCC_ERR_* code from ccc_b200.h; device errors (capacity overflow, bad face
 * indices) are reported in the status word of ccc_engine_read_state.  An engine is not
 * thread-safe; calls on one engine must be ordered on one stream.
 */
#ifndef CCC_ENGINE_H
#define CCC_ENGINE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ccc_engine ccc_engine;

/* device pointers of one resident mesh, for the caller to fill or read */
typedef struct ccc_mesh_view {
    int64_t F, V;          /* triangles, vertices (0 for a collision-only mesh)            */
    void* x0;              /* (F, 3, 3) triangle positions at the start of the step        */
    void* x1;              /* (F, 3, 3) triangle positions at the end of the step          */
    void* masses;          /* (F, 3) per-corner masses (impulse loop)                      */
    int32_t* faces;        /* (F, 3) mesh-local vertex ids (impulse loop)                  */
    void* verts0;          /* (V, 3) vertex positions at the start of the step             */
    void* verts1;          /* (V, 3) vertex positions at the end of the step (updated)     */
    void* vel;             /* (V, 3) vertex velocities (updated by the loop)               */
    int64_t* rows;         /* (F * max_collisions_per_triangle, 3) rows (i, j, type)      */
    void* times;           /* (F * max_collisions_per_triangle) times of impact            */
} ccc_mesh_view;

/* per-mesh state flags (ccc_engine_read_state) */
#define CCC_MESH_DONE 1       /* the impulse loop has stopped for this mesh          */
#define CCC_MESH_CONVERGED 2  /* ... because a collision check found no contact       */

/* extra status bit of the engine (besides CCC_ST_* of ccc_b200.h) */
#define CCC_ST_NONFINITE 16   /* a non-finite impulse was left out of the loop sums    */

/* operations for capture / replay */
#define CCC_ENGINE_OP_CCD 0
#define CCC_ENGINE_OP_LOOP_STEP 1

/* Device bytes of an engine with room for tri_capacity triangles and vert_capacity vertices
 * in at most mesh_capacity meshes; -1 for invalid sizes. */
int64_t ccc_engine_bytes(int dtype, int64_t tri_capacity, int64_t vert_capacity, int64_t mesh_capacity,
                         int64_t max_candidates_per_triangle, int64_t max_collisions_per_triangle);

/* Create an engine in the caller's device block (at least ccc_engine_bytes, 256-byte
 * aligned).  Clears the block's state on `stream` and synchronises it. */
int ccc_engine_create(int dtype, int64_t tri_capacity, int64_t vert_capacity, int64_t mesh_capacity,
                      int64_t max_candidates_per_triangle, int64_t max_collisions_per_triangle, void* block,
                      int64_t block_bytes, void* stream, ccc_engine** out);
int ccc_engine_destroy(ccc_engine* e);

/* Reserve slots for a mesh of F >= 2 triangles and V vertices (V = 0: collision only).
 * Writes the mesh's slot id; CCC_ERR_WORKSPACE when the block has no room left. */
int ccc_engine_add_mesh(ccc_engine* e, int64_t F, int64_t V, int32_t* slot_id);
int ccc_engine_remove_mesh(ccc_engine* e, int32_t slot_id);
int ccc_engine_mesh_view(ccc_engine* e, int32_t slot_id, ccc_mesh_view* out);
/* free triangle and vertex slots (largest contiguous run of each) */
int ccc_engine_free_slots(ccc_engine* e, int64_t* tris, int64_t* verts);

/* Select the meshes the next steps process (uploaded to the device mesh table on stream). */
int ccc_engine_set_active(ccc_engine* e, const int32_t* slot_ids, int64_t n, void* stream);

/* Build the trees of the given meshes from their current x0 / x1. */
int ccc_engine_build(ccc_engine* e, const int32_t* slot_ids, int64_t n, void* stream);

/* Continuous collisions of every active mesh: refit, traversal, narrow phase.  Rows of
 * mesh s are written to its view's rows / times; their count is read back by
 * ccc_engine_read_state. */
int ccc_engine_ccd(ccc_engine* e, void* stream);

/* Start the impulse loop of the given meshes: triangle soups from verts0 / verts1 through
 * faces, tree build, iteration counters and flags cleared. */
int ccc_engine_loop_prepare(ccc_engine* e, const int32_t* slot_ids, int64_t n, void* stream);

/* One iteration for every active mesh that has not stopped: collision check with impulses
 * (the reference's compute_impulses), then every touched vertex moves by the average of
 * the position corrections of its corners (and its velocity by the average velocity
 * change), and the mesh stops when the check found no contact or after max_iter
 * iterations. */
int ccc_engine_loop_step(ccc_engine* e, int32_t max_iter, void* stream);

/* Capture one operation (CCC_ENGINE_OP_*) on a non-default stream as a CUDA graph, and
 * replay it.  Replays use the device mesh table as it is at replay time. */
int ccc_engine_capture(ccc_engine* e, int op, int32_t max_iter, void* stream);
int ccc_engine_replay(ccc_engine* e, int op, void* stream);

/* Launch-shape autotuner: times the collision step of the active set for each candidate
 * schedule (traversal and narrow-phase grid sizes, traversal form, tree levels staged in
 * shared memory, narrow-phase batch size), keeps the fastest and returns its index.  It
 * only recomputes collision rows.  Choices are cached per (dtype, size class). */
int ccc_engine_autotune(ccc_engine* e, void* stream, int32_t* choice);

/* The autotuner's candidate schedules (no counterpart in the reference): their number;
 * the parameters of one in out[5] (out[0] traversal blocks per SM, out[1] narrow-phase
 * blocks per SM in units of the resident count, out[2] traversal form: 0 one query per
 * thread, 1 32 queries per warp walking the tree together, out[3] tree levels below the
 * root that each block of the one-query-per-thread form copies into shared memory, 0-2,
 * out[4] the narrow phase's batch in units of 256 sub-tests, 1 or 2); and fixing the
 * engine to one of them. */
int ccc_engine_schedule_count(void);
int ccc_engine_schedule_info(int32_t choice, int32_t* out);
int ccc_engine_set_schedule(ccc_engine* e, int32_t choice);

/* Synchronise the stream and read the status word and, for each given mesh, its row
 * count, contacts of the last loop iteration, iterations and flags (NULL to skip). */
int ccc_engine_read_state(ccc_engine* e, const int32_t* slot_ids, int64_t n, int32_t* status, int32_t* rows,
                          int32_t* contacts, int32_t* iterations, int32_t* flags, void* stream);

/* Pack the rows and times of the last ccc_engine_ccd of every active mesh back to back into
 * out_rows (capacity x 3 int64) and out_times (capacity, of the engine's dtype), so that one
 * device-to-host copy fetches a whole step (no counterpart in the reference, which returns
 * one fixed-size tensor per call).  Device-only, no synchronisation.  out_meta (device,
 * 2 * M + 2 int32 for M active meshes) receives, in the engine's table order (ascending
 * triangle slot), the row offset of each mesh, the total at [M], the mesh slot ids at
 * [M + 1 .. 2M] and the step's status word at [2M + 1].  Rows past capacity are dropped
 * with CCC_ST_OUT_OVERFLOW; a capacity of the active triangles x
 * max_collisions_per_triangle always suffices. */
int ccc_engine_pack_rows(ccc_engine* e, int64_t* out_rows, void* out_times, int64_t capacity, int32_t* out_meta,
                         void* stream);

/* Synchronise the stream and read the work counters of the last step into out[6]: status
 * word, candidate pairs (in a collision step, those whose triangles share no vertex: the
 * others are dropped during the traversal), continuous sub-tests (pair, type) whose swept
 * sub-boxes overlap,
 * roots in [0, 1] filtered, sub-tests solved, and candidate pairs with sub-tests to solve.
 * A sub-test that several pairs of a mesh have with the same tetrahedron (a vertex-face
 * test over the triangles around the vertex, an edge-edge test over the two triangles of an
 * edge) is solved once, and its rows or contacts are written for each of those pairs. */
int ccc_engine_counters(ccc_engine* e, int32_t* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CCC_ENGINE_H */
