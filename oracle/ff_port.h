/*
 * CPU restatement of fastfusion's depth-fusion hot path (the oracle).
 *
 * ORACLE INFRASTRUCTURE ONLY: tests/, the smoke check and bench.py's CPU
 * baseline leg load oracle/_ref/libffport.so as the checker.  The product
 * (fastfusion_b200/) never links or calls it.
 *
 * It restates, in plain C and in the reference's operation order:
 *   - FusionMipMapCPU::addMap for uint16 depth
 *       (reference src/fusion/geometryfusion_mipmap_cpu.cpp:1603-2034)
 *   - the traversal / brick allocation
 *       (traversal_wrapper_functions.cpp:576-694, traversal_functions.cpp:185-211,308-395)
 *   - the first-frame volume (geometryfusion_mipmap_cpu.cpp:1186-1233,1270-1303)
 *   - grow() (geometryfusion_mipmap_cpu.cpp:3071-3319, treeandbrick.cpp:419-440)
 *   - the SDF/weight/colour update (update_functions.cpp:1187-1444, 1633-1732)
 *
 * The update runs with round-toward-zero like the reference (MXCSR RZ,
 * update_functions.cpp:1678-1679) but replaces the reference's approximate
 * _mm256_rcp_ps by an exact reciprocal, so the result is defined bit for bit
 * (the GPU reproduces it with __frcp_rz).  ffp_set_update_mode(m, mode):
 *   1 (default) round-toward-zero, exact reciprocal -- the defined target;
 *   2 round-toward-zero with the host CPU's RCPPS -- the reference's own
 *     instruction, used only to check this restatement against the compiled
 *     reference on the same machine;
 *   0 round-to-nearest, exact reciprocal (rounding-sensitivity tests);
 *   3 the FP64 oracle: the same allocation, and the update's geometry and
 *     running averages in double precision from the double pose (no float
 *     camera parameters, exact reciprocals, round-to-nearest) into separate
 *     double SDF/weight arrays (ffp_bricks64) -- the reference against which
 *     the FP32 and FP16-storage results state their error.
 */
#ifndef FF_PORT_H
#define FF_PORT_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFP_BRANCHINIT 0xFFFFFFFEu

typedef struct ffp_map ffp_map;

ffp_map *ffp_create(float scale, float threshold, int color, uint32_t leaves_total, uint32_t branches_total);
void ffp_destroy(ffp_map *m);
void ffp_set_update_mode(ffp_map *m, int mode);
/* Per-pixel confidence multiplying the weight increment (borrowed; NULL: off). */
void ffp_set_confidence(ffp_map *m, const float *conf);
/* SDF and weight stored at half precision (round to nearest even after each
 * update), as the GPU's FP16 storage keeps them. */
void ffp_set_storage_fp16(ffp_map *m, int on);
/* The value the FP16 storage keeps for f (for tests of the rounding). */
float ffp_half_round(float f);

/* One depth frame (uint16, depth*scaling = metres) with BGR colour.
 * K = {fx, fy, cx, cy}; R (row-major 3x3) and t map camera to world.
 * Returns the number of queued (updated) leaves, like addMap. */
int ffp_add_map(ffp_map *m, const uint16_t *depth, const uint8_t *bgr, int w, int h, const double *K,
                const double *R, const double *t, float scaling, float maxcam);

/* State accessors. ints: n, leaves_used, branches_used, queued, leaves_total,
 * branches_total, frames, bandwidth, meshing_ok, grow_count. */
void ffp_state(const ffp_map *m, int64_t *ints, float *offset);
void ffp_leaves(const ffp_map *m, uint16_t *pos, uint16_t *scale, uint32_t *parent);
void ffp_queue(const ffp_map *m, uint32_t *q);
void ffp_tree(const ffp_map *m, uint32_t *tree);
/* Brick contents of leaves [0, n): 512 SDF, 512 weights, 512 x 3 colour (R, G, B) each. */
void ffp_bricks(const ffp_map *m, int64_t n, float *dist, float *wgt, uint16_t *col);
/* FP64-oracle brick contents of leaves [0, n) (update mode 3 only). */
void ffp_bricks64(const ffp_map *m, int64_t n, double *dist, double *wgt);
/* Replace brick contents (used to start the update from a given state). */
void ffp_set_bricks(ffp_map *m, int64_t n, const float *dist, const float *wgt, const uint16_t *col);

/* Meshing (ff_port_mesh.c): every cell re-meshed from the current voxels.
 * Returns the number of cells; cells are sorted by (type, quirk, size, origin). */
int64_t ffp_update_meshes(ffp_map *m);
void ffp_mesh_counts(const ffp_map *m, int64_t *ncells, int64_t *nv, int64_t *nf);
/* cells: 14 int32 each (type, quirk, ox, oy, oz, size, L0..L7);
 * ranges: per cell first vertex, vertex count, first face, face count. */
void ffp_mesh_copy(const ffp_map *m, int32_t *cells, int64_t *ranges, float *xyz, uint8_t *rgb, uint32_t *faces);
int ffp_set_state(ffp_map *m, uint32_t n, const float *offset, const uint32_t *tree, uint32_t branches_used,
                  const uint16_t *pos, const uint16_t *scale, const uint32_t *parent, uint32_t leaves_used,
                  const float *dist, const float *wgt, const uint16_t *col);

#ifdef __cplusplus
}
#endif
#endif
