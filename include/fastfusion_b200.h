/*
 * fastfusion_b200 -- C ABI of the B200 depth-fusion + incremental-meshing path.
 *
 * One handle is one map: the reference's FusionMipMapCPU object
 * (tum-vision/fastfusion src/fusion/geometryfusion_mipmap_cpu.hpp:111-534).
 * Every entry point returns ff_status; ff_last_error() describes the last
 * failure on a handle.  A handle is used by one host thread at a time; its
 * device work is ordered on one CUDA stream (ff_set_stream).
 *
 * Plain pointers and sizes only: no CUDA, C++ or torch types in signatures.
 */
#ifndef FASTFUSION_B200_H
#define FASTFUSION_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ff_status {
  FF_OK = 0,
  FF_ERR_BAD_ARG = 1,   /* NULL handle/pointer, bad size, bad config */
  FF_ERR_CUDA = 2,      /* a CUDA runtime call failed (message in ff_last_error) */
  FF_ERR_OOM_POOL = 3,  /* device memory for the brick pool could not be had */
  FF_ERR_OOM_MESH = 4,  /* mesh output larger than the mesh buffers allow */
  FF_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up */
  FF_ERR_STATE = 6,     /* call not valid in the current state */
  FF_ERR_NO_DEVICE = 7  /* no CUDA device / library built without one */
} ff_status;

/* Voxel storage of the brick pool. */
enum { FF_STORAGE_FP32 = 0, FF_STORAGE_FP16 = 1 };

/* Reciprocal of the voxel update.  The reference runs its update with the
 * approximate x86 RCPPS instruction (update_functions.cpp:1246,1373,1386),
 * whose result bits depend on the CPU model.
 *   FF_RCP_HOST:  reproduce the RCPPS of the CPU this library runs on (a
 *                 table measured from the instruction at ff_create over all
 *                 2^23 mantissas, stored by the leading mantissa bits the
 *                 result depends on: 8 KB on recent Intel cores, at most
 *                 32 MB); results are bit-identical to the reference binary
 *                 on the same host.  x86-64 only.
 *   FF_RCP_EXACT: exact round-toward-zero reciprocal; host-independent. */
enum { FF_RCP_HOST = 0, FF_RCP_EXACT = 1 };

typedef struct ff_config {
  float scale;             /* voxel edge in metres (FusionMipMapCPU ctor `scale`) */
  float threshold;         /* truncation distance in metres (ctor `distanceThreshold`) */
  int color;               /* fuse colour (ctor `color`); must be 1 like the reference's AVX update */
  uint32_t leaves_max;     /* brick pool capacity in 8^3 bricks; 0 = derive from pool_bytes */
  uint32_t branches_max;   /* octree capacity in uint32 entries (16 per branch); 0 = 4 x leaves_max x 16 / 8 */
  uint64_t pool_bytes;     /* used when leaves_max == 0 */
  int device;              /* CUDA device ordinal */
  int storage;             /* FF_STORAGE_FP32 (reference layout) or FF_STORAGE_FP16 */
  int rcp_mode;            /* FF_RCP_HOST (default, reference bits) or FF_RCP_EXACT */
} ff_config;

typedef struct ff_handle ff_handle;

/* Counters of the map; field names follow the reference's members. */
typedef struct ff_stats {
  uint32_t n;                  /* _n: side of the octree volume in voxels */
  float offset[3];             /* _offset: world position of voxel (0,0,0), metres */
  uint32_t leaves_used;        /* _nLeavesUsed (may exceed leaves_max after overflow) */
  uint32_t leaves_max;         /* _nLeavesTotal */
  uint32_t branches_used;      /* _nBranchesUsed (entries) */
  uint32_t branches_max;       /* _nBranchesTotal */
  uint32_t queued;             /* _nLeavesQueuedSurface of the last frame */
  uint32_t frames;             /* _framesAdded */
  uint32_t meshing_ok;         /* _performIncrementalMeshing */
  uint32_t grows;              /* number of grow() events */
  uint64_t mesh_vertices;      /* size of the current mesh */
  uint64_t mesh_faces;
  uint64_t mesh_cells;         /* mesh cells of the last update */
  uint64_t mesh_cells_dirty;   /* cells re-meshed by the last update */
  uint32_t processed_pixels;   /* pixels that passed the row/column de-duplication */
  uint32_t new_leaves;         /* leaves allocated by the last frame */
  uint32_t dedupe_rounds;      /* rounds the last frame's de-duplication took to settle */
  uint32_t graph_replays;      /* batched calls led by this map that replayed a recorded CUDA graph */
  uint32_t update_batch;       /* frames one deferred voxel-update pass takes (ff_set_update_batch) */
  uint64_t fused_bricks;       /* bricks read and written by the voxel updates so far (a pass counts a brick once,
                                  whatever the number of its frames; as of the last finished pass) */
  uint64_t fused_frame_bricks; /* queued bricks summed over the frames updated so far (the reference reads and
                                  writes each of them once per frame) */
  uint64_t mesh_cells_generated; /* cells the last update's octree traversal produced (the rest were kept from
                                    the update before; all of them after a full generation) */
  uint32_t mesh_top_kept;      /* 1: the last update's traversal started from the items of its first levels kept
                                  from an earlier update (no frame since created anything near the root) */
} ff_stats;

/* Create a map.  Replaces `new FusionMipMapCPU(0,0,0,scale,threshold,0,color)`
 * (geometryfusion_mipmap_cpu.cpp:420-640). */
ff_status ff_create(const ff_config *cfg, ff_handle **out);

/* Destroy a map and free its device memory (~FusionMipMapCPU). */
ff_status ff_destroy(ff_handle *h);

/* Order this map's device work on the given cudaStream_t (NULL = the
 * library's own stream). */
ff_status ff_set_stream(ff_handle *h, void *cuda_stream);

/* Wait for this map's outstanding device work (the last frame's placement
 * of new bricks and voxel update, which an add-map call does not wait for). */
ff_status ff_sync(ff_handle *h);

/* Fuse one frame.  Replaces FusionMipMapCPU::addMap(const cv::Mat &depth
 * CV_16UC1, CameraInfo, const cv::Mat &rgb CV_8UC3 BGR, float scaling, float
 * maxcamdistance) (geometryfusion_mipmap_cpu.hpp:122-123, .cpp:1603-2034).
 * depth/bgr are HOST buffers, borrowed for the call; pitches in bytes
 * (0 = tightly packed).  K = {fx, fy, cx, cy}; R (row-major) and t are the
 * camera-to-world pose (CameraInfo rotation/translation).  *queued (may be
 * NULL) receives addMap's return value, the number of bricks updated. */
ff_status ff_add_map_u16(ff_handle *h, const uint16_t *depth, int width, int height, size_t depth_pitch,
                         const uint8_t *bgr, size_t bgr_pitch, const double K[4], const double R[9],
                         const double t[3], float scaling, float maxcam, int32_t *queued);

/* Same as ff_add_map_u16 with depth/bgr already in device memory (tightly
 * packed).  No host<->device copy of the images.  The call returns once the
 * frame's bricks are counted; the placement of its new bricks may still be
 * running on a second stream of the map (every later call on this handle is
 * ordered after it), and its voxel update is deferred (ff_set_update_batch).
 * The images are read by the call itself (and copied for the deferred
 * update), so they are free when it returns; they must be ready in the order
 * of the map's stream (ff_set_stream).  With deferral off
 * (ff_set_update_batch(h, 1)) the update runs on the second stream and reads
 * the images: they must then stay unchanged until the next call on this
 * handle returns or ff_sync(h). */
ff_status ff_add_map_u16_device(ff_handle *h, const uint16_t *d_depth, const uint8_t *d_bgr, int width, int height,
                                const double K[4], const double R[9], const double t[3], float scaling,
                                float maxcam, int32_t *queued);

/* A sequence of n frames of one map, all W x H, in device memory; the same
 * results as n calls of ff_add_map_u16_device (queued[k] = frame k's count).
 * The frames' de-duplication (which reads no octree) runs for all of them in
 * one set of cooperative launches; their inserts and leaf finalisations run
 * frame after frame on the device without returning to the host (each
 * finalisation hands the next frame its branch count and leaf base); one
 * read-back of all frames' counters follows.  When a frame must grow the
 * volume, the frames after it were de-duplicated in the old volume: they are
 * halted on the device and run again after the growth.  Their voxel update
 * runs as one deferred pass before the call returns, so the images are free
 * then.  K + 4k, R + 9k, t + 3k: frame k's camera, as in ff_add_map_u16.
 * On an error the frames before the failing one are fused and queued[] of
 * the later ones is left unset.  The reference fuses one frame per call
 * (geometryfusion_mipmap_cpu.cpp:1603-2034); this is the frame-batched form. */
ff_status ff_add_map_sequence_u16_device(ff_handle *h, int n, const uint16_t *const *d_depth,
                                         const uint8_t *const *d_bgr, int width, int height, const double *K,
                                         const double *R, const double *t, float scaling, float maxcam,
                                         int32_t *queued);

/* The same with the n frames in HOST memory: the reference's several-frames
 * addMap(std::vector<cv::Mat> depthImages, std::vector<CameraInfo>,
 * std::vector<cv::Mat> rgbImages) (geometryfusion_mipmap_cpu.hpp:125-129,
 * .cpp:2116-2240), which adds the frames one after another.  All frames'
 * depth images are copied to the device first, their colour images on a
 * second stream while the frames are allocated; frames are taken 32 at a
 * time.  Pitches in bytes (0 = tightly packed).  The images are free when the
 * call returns; page-locked memory (ff_alloc_host) lets the copies run
 * without the host. */
ff_status ff_add_map_sequence_u16(ff_handle *h, int n, const uint16_t *const *depth, const uint8_t *const *bgr,
                                  int width, int height, size_t depth_pitch, size_t bgr_pitch, const double *K,
                                  const double *R, const double *t, float scaling, float maxcam, int32_t *queued);

/* Several independent maps fuse one frame each, in one set of launches (the
 * de-duplication of all frames in one cooperative launch, their inserts,
 * leaf finalisations and voxel updates in one launch each) -- for many maps
 * of uneven size on one GPU.  Same results as ff_add_map_u16_device on each
 * map in turn.  maps: n distinct handles on one device with the same storage
 * and reciprocal mode, n <= 32; per map i: device images d_depth[i], d_bgr[i]
 * of width[i] x height[i], K + 4i, R + 9i, t + 3i, scaling[i], maxcam[i];
 * queued[i] (may be NULL) receives each map's count.  The work runs on
 * maps[0]'s stream.  The reference fuses one map per call; this is the
 * batched form of its addMap (geometryfusion_mipmap_cpu.cpp:1603-2034). */
ff_status ff_add_maps_u16_device(ff_handle *const *maps, int n, const uint16_t *const *d_depth,
                                 const uint8_t *const *d_bgr, const int *width, const int *height, const double *K,
                                 const double *R, const double *t, const float *scaling, const float *maxcam,
                                 int32_t *queued);

/* Launch shapes of the per-frame kernels (what the autotuner chooses; 0 in
 * a field = the default).  dedupe_rows: height of a de-duplication tile, 8,
 * 16 or 32 (default: 16 when all tiles of the call fit one cooperative launch;
 * 8 only where they fit);
 * fuse_shape: block shape of the voxel update, 0..3 = (1 brick per 512-thread
 * block, registers for 4 blocks per SM), (1, 3), (2 bricks per 1024-thread
 * block, 2), (2, 1); fuse_blocks_per_sm: grid of the update in blocks per SM
 * (default 8 for one brick per block, 4 for two); insert_block: threads per
 * block of the octree insert (default 256); graph: 1 = ff_add_maps_u16_device
 * records its launches once as a CUDA graph and replays it while the maps
 * and image sizes stay the same (no effect while profiling).  Launch shapes
 * never change results. */
typedef struct {
  int dedupe_rows;
  int fuse_shape;
  int fuse_blocks_per_sm;
  int insert_block;
  int graph;
} ff_tuning;

/* Make this map one of `shards` parts of a larger map, one part per GPU
 * (call before its first frame; no counterpart in the reference, which fuses
 * one map on one machine).  Every part is given every frame and holds the
 * whole map's octree and leaf table (the same allocation as the whole map:
 * identical leaf indices, queues and counts).  The voxel updates and the
 * meshing are divided: a part updates the bricks it owns and meshes the mesh
 * cells it owns, each owner a hash of the object's origin in units of its
 * edge (in coordinates that volume growth does not move) and of its edge.
 * Before a part meshes, the bricks the other parts changed must reach it:
 * each part exports the bricks it owns that changed since its last export
 * (ff_halo_export), the caller moves the records between the GPUs (an NCCL
 * all-gather, say: records land in each GPU's own memory) and each part
 * imports the others' (ff_halo_import).  Each part's mesh then holds the
 * meshes of its cells, exactly as the whole map meshes them; together the
 * parts' meshes are the whole map's mesh. */
ff_status ff_set_shard(ff_handle *h, int shard, int shards);

/* ---- Loop closure: removing fused frames (the reference's deleteOldLoopPoses) ----
 *
 * When a trajectory is corrected, the reference's loop closure removes the
 * contribution of already fused frames: a second set of voxel arrays ("loop
 * arrays") for at most `capacity` bricks (MAX_LOOP_CLOSURE_LEAVES = 100,000
 * there, definitions.h:124) receives, per frame, the update of
 * update8AddLoopSSESingleDeleteloop (loopclosure.cpp:15-228) -- the frame's
 * depth (float metres, NaN where there is none) and colour planes, projected
 * with the frame's corrected pose, with the weight fall-off's sign turned --
 * over the bricks the frame queued when it was fused; each brick gets the
 * next free slot in queue order the first time (updateWrapper_deleteloop,
 * loopclosure.cpp:232-309).  The voxel values equal the reference's bit for
 * bit with FF_RCP_HOST.
 *
 * ff_loop_begin: (re)start with zeroed loop arrays for `capacity` bricks and
 * no brick mapped (updateArraysForLoopClosure,
 * geometryfusion_mipmap_cpu.cpp:3910-3931).  ff_loop_delete_frame: one frame
 * (device memory: depth float[h][w], red/green/blue uint8[h][w], the queue of
 * the frame's leaves -- ff_get_queue after its addMap); *complete = 0 when the
 * slots ran out (the entry that found none and every later one are left out,
 * as the reference returns there).  ff_loop_get: slots in use; per leaf its
 * slot (0xFFFFFFFE: none; leaf_slot[leaves_used]); and the loop arrays of the
 * slots in use as ff_get_bricks lays out bricks (any pointer may be NULL). */
ff_status ff_loop_begin(ff_handle *h, uint32_t capacity);
ff_status ff_loop_delete_frame(ff_handle *h, const float *d_depth, const uint8_t *d_red, const uint8_t *d_green,
                               const uint8_t *d_blue, int width, int height, const double K[4], const double R[9],
                               const double t[3], const uint32_t *d_queue, uint32_t n_queue, int *complete);
ff_status ff_loop_get(ff_handle *h, uint32_t *n_mapped, uint32_t *leaf_slot, float *sdf, float *weight,
                      uint16_t *rgb);

/* Halo export of a part of a sharded map: the bricks this part owns whose
 * voxels changed since its last export (with a buffer), as records of
 * *record_bytes bytes each -- uint32 leaf index, 12 bytes of padding, then
 * the brick's SDF and weight (float, or half with FP16 storage) and its three
 * uint16 colour planes, 512 voxels each -- written to device memory d_records
 * with room for `capacity` records.  With d_records NULL only *n_records is
 * set (call again with a buffer that large); more records than capacity is
 * FF_ERR_BAD_ARG and nothing is written.  The waiting voxel updates run first.
 * On an unsharded map every changed brick is exported. */
ff_status ff_halo_export(ff_handle *h, void *d_records, uint64_t capacity, uint64_t *n_records,
                         uint64_t *record_bytes);

/* Halo import: write the bricks of n_records records (as ff_halo_export
 * writes them, from another part of the same map; device memory) into this
 * part's pool.  Records whose leaf index lies past this map's pool are
 * skipped. */
ff_status ff_halo_import(ff_handle *h, const void *d_records, uint64_t n_records);

/* Set the launch shapes used by calls that this map leads (the map itself,
 * or a batch whose maps[0] it is). */
ff_status ff_set_tuning(ff_handle *h, const ff_tuning *t);

/* Frames whose voxel update is deferred to one pass (at most
 * FF_UPDATE_BATCH_MAX, default 16; 1 = every frame updated by itself).  The
 * reference updates each queued brick once per frame
 * (update_functions.cpp:1633-1732); here a single-map frame only marks its
 * bricks, and one pass later reads and writes each marked brick once,
 * applying its frames in order with the same operations -- the voxel values
 * are bit-identical to frame-by-frame updates.  The pass runs when the batch
 * is full, before the volume grows, and before anything reads or replaces
 * voxel state (ff_update_meshes, ff_get_bricks, ff_set_bricks, ff_set_state,
 * ff_raycast_depth, ff_sync, ff_set_stream, a batched call).  The waiting
 * frames' images are copies the map keeps (a ring of frames x W x H x 5
 * bytes, x 9 with the learned weight), so device images given to
 * ff_add_map_u16_device are free when the call returns.  No counterpart in
 * the reference. */
#define FF_UPDATE_BATCH_MAX 32
ff_status ff_set_update_batch(ff_handle *h, int frames);

/* Bound of every device-side wait of this map (the grid barriers of the
 * de-duplication and of the mesh-cell traversal, the lock wait of the octree
 * insert), in polling iterations; default FF_SPIN_LIMIT_DEFAULT.  A wait
 * that runs out sets an error flag and returns instead of waiting on; the
 * call then returns FF_ERR_TIMEOUT: after a de-duplication wait the frame is
 * left out and the map is as it was before the call; after an insert wait
 * the bricks found so far are allocated but the frame's voxel update is
 * skipped; after a traversal wait ff_update_meshes leaves the mesh of the
 * previous update, and the next update meshes every change since then.  The
 * handle stays usable either way.  No counterpart in the reference (its traversal
 * is sequential and has no waits). */
#define FF_SPIN_LIMIT_DEFAULT (1u << 22)
ff_status ff_set_spin_limit(ff_handle *h, uint32_t iterations);

/* How ff_update_meshes finds the mesh cells.  FF_CELLS_INCREMENTAL (the
 * default): only the parts of the octree that gained a branch or a leaf
 * since the previous update are traversed again; the cells elsewhere are
 * kept from the previous update's list (like the reference's
 * updateMeshCellStructure, geometryfusion_mipmap_cpu.cpp:2488-2616, which
 * adds cells only for new octree slots).  FF_CELLS_FULL: every cell is
 * generated again from the whole octree at every update.  Both give the same
 * cell list in the same order; the first update, a growth of the volume and
 * ff_set_state always generate every cell. */
#define FF_CELLS_INCREMENTAL 0
#define FF_CELLS_FULL 1
ff_status ff_set_cell_generation(ff_handle *h, int mode);

/* Failure injection for tests of the error paths (no counterpart in the
 * reference).  FF_INJECT_CONFIDENCE_TIMEOUT: the next frame reports that a
 * bounded wait of the confidence network gave up, exactly as the network
 * reports it on the device (its error word is set); the frame's bricks are
 * allocated, its voxel update is skipped and the call returns
 * FF_ERR_TIMEOUT.  0 cancels a pending injection. */
enum { FF_INJECT_CONFIDENCE_TIMEOUT = 1 };
ff_status ff_inject_error(ff_handle *h, int what);

/* Re-mesh the cells touched since the last update and rebuild the
 * interleaved mesh.  Replaces FusionMipMapCPU::updateMeshes()
 * (geometryfusion_mipmap_cpu.cpp:2884-2954) with threaded meshing off;
 * *updated = 1 like its `true` return. */
ff_status ff_update_meshes(ff_handle *h, int *updated);

/* Size of the mesh of the last update (MeshInterleaved vertices/faces). */
ff_status ff_get_mesh_counts(ff_handle *h, uint64_t *n_vertices, uint64_t *n_faces);

/* Copy the mesh of the last update to HOST buffers: xyz float[3*nv] (world
 * metres), rgb uint8[3*nv], faces uint32[3*nf].  Replaces
 * getMeshInterleavedMarchingCubes() (geometryfusion_mipmap_cpu.cpp:3359-3374). */
ff_status ff_get_mesh(ff_handle *h, float *xyz, uint8_t *rgb, uint32_t *faces);

/* ff_get_mesh without waiting: the copies are queued on a copy stream of the
 * map behind the last update's device work and the call returns at once, so
 * the copy overlaps what the caller issues next (the next frames).  The
 * buffers (page-locked memory, ff_alloc_host, lets the copy run without the
 * host) hold the mesh when ff_mesh_wait returns; they must stay allocated
 * until then.  A later ff_update_meshes orders its writes after the copy on
 * the device, without blocking the host.  No counterpart in the reference
 * (its mesh is returned by value). */
ff_status ff_get_mesh_async(ff_handle *h, float *xyz, uint8_t *rgb, uint32_t *faces);

/* Wait for the copies of the last ff_get_mesh_async (returns at once if there
 * are none). */
ff_status ff_mesh_wait(ff_handle *h);

/* Page-locked host memory for ff_get_mesh / ff_add_map_u16 buffers: copies
 * to and from it run at full PCIe/C2C speed.  Not a counterpart of a
 * reference call (the reference has no device). */
ff_status ff_alloc_host(size_t bytes, void **out);
ff_status ff_free_host(void *p);

/* The mesh cells of the last update (ff_stats.mesh_cells of them), in mesh
 * order: 14 int32 each -- type (0 interior, 1-3 wall x/y/z, 4-6 edge x/y/z,
 * 7 corner), quirk flag, origin x/y/z, size (voxels), the leaf of each side
 * (8 entries, 0xFFFFFFFE past the cell's side count) -- the reference's
 * MeshCell (treeandbrick_incremental.hpp:71-93); and 4 int64 each: first
 * vertex, vertex count, first face, face count of the cell's part of the mesh. */
ff_status ff_get_mesh_cells(ff_handle *h, int32_t *cells, int64_t *ranges);

/* ff_get_mesh_cells for callers that cannot allocate device memory during the
 * call: a fixed memory budget, an allocator they do not own, or code where
 * cudaMalloc is not allowed.  It has no counterpart in the reference.  The
 * cells are staged in a fixed device buffer that is part of the library
 * (FF_NOALLOC_MAX_CELLS cells, 5.8 MB, held on every GPU that loads the
 * library until the process exits); the call allocates nothing.  A mesh with
 * more cells is rejected with FF_ERR_BAD_ARG and a message, and nothing is
 * written.  Every call looks up the buffer's device address on the current
 * device (the first call on a device may load the library's device code:
 * make that first call before any stream capture).  Every call on one device uses the same buffer,
 * so calls whose GPU work overlaps (maps on different streams) race: order
 * them on the host or on one stream. */
#define FF_NOALLOC_MAX_CELLS 65536
ff_status ff_get_mesh_cells_noalloc(ff_handle *h, int32_t *cells, int64_t *ranges);

/* Device pointers to the same mesh, valid until the next ff_update_meshes. */
ff_status ff_get_mesh_device(ff_handle *h, const float **xyz, const uint8_t **rgb, const uint32_t **faces);

ff_status ff_get_stats(ff_handle *h, ff_stats *out);

/* Leaf table of leaves [0, min(leaves_used, leaves_max)): position (3 x
 * uint16 voxels), scale (voxel spacing of the brick) and parent leaf
 * (0xFFFFFFFE if none) -- the reference's _leafPos/_leafScale/_leafParent. */
ff_status ff_get_leaves(ff_handle *h, uint16_t *pos, uint16_t *scale, uint32_t *parent);

/* Bricks updated by the last frame (leaf indices, unordered). */
ff_status ff_get_queue(ff_handle *h, uint32_t *leaves);

/* Brick contents of leaves [first, first+count) as the reference stores
 * them: SDF float[512], weight float[512], colour uint16[512][3] (R,G,B x256)
 * per brick, voxel index (z*8+y)*8+x. */
ff_status ff_get_bricks(ff_handle *h, uint32_t first, uint32_t count, float *sdf, float *weight, uint16_t *rgb);
ff_status ff_set_bricks(ff_handle *h, uint32_t first, uint32_t count, const float *sdf, const float *weight,
                        const uint16_t *rgb);

/* The octree array (branches_used entries): 16 per branch, [0..7] leaf index
 * per octant, [8..15] child branch -- the reference's _tree layout. */
ff_status ff_get_tree(ff_handle *h, uint32_t *tree);

/* Replace the whole map state (snapshot restore): octree, leaf table, bricks,
 * volume side n and offset.  Used to resume and to mesh a given voxel state. */
ff_status ff_set_state(ff_handle *h, uint32_t n, const float offset[3], const uint32_t *tree, uint32_t branches_used,
                       const uint16_t *pos, const uint16_t *scale, const uint32_t *parent, uint32_t leaves_used,
                       const float *sdf, const float *weight, const uint16_t *rgb);

/* Device-time profile per stage, measured with CUDA events on the map's
 * stream.  ff_profile(h, 1) resets and starts recording; ff_profile_read
 * returns, per stage, the summed milliseconds, the algorithmic bytes (bytes
 * the stage must move at minimum: e.g. 14,336 B per fused FP32 brick) and the
 * number of launches.  Stages, in order: grow (volume extension), dedupe
 * (projection and de-duplication of the pixels), insert, finalize (leaf
 * indices and parents), fuse, mesh_cells (cell generation and sort),
 * mesh_count, mesh_emit, confidence (the learned weight's network). */
#define FF_PROFILE_STAGES 9
ff_status ff_profile(ff_handle *h, int enable);
ff_status ff_profile_read(ff_handle *h, double *ms, double *bytes, uint64_t *launches);

/* Process-wide counts, since the library was loaded, of this library's own
 * kernel launches and of its calls into CUB (sort and scan, each of which
 * launches a few library kernels). */
ff_status ff_kernel_launches(uint64_t *own, uint64_t *library);

/* ---- Learned per-pixel confidence weight (no counterpart in the reference) ----
 *
 * The reference weights every pixel's update by the same distance ramp
 * (update_functions.cpp:1187-1444).  With a confidence network set, each
 * frame's pixels first go through a 3-layer 5x5 CNN (16 channels; BF16
 * weights and activations, FP32 accumulation) that predicts the pixel's
 * depth error r; the ramp's weight increment of every voxel the pixel
 * updates is multiplied by c = (1 - r/tau)^2 for r < tau, else 0.
 *
 * Parameters (FF_CNN_PARAMS floats, in order): W1[16][5][25] b1[16]
 * W2[16][16][25] b2[16] W3[1][16][25] b3[1]; W[out][in][ky*5+kx] of a 'same'
 * 5x5 correlation, ReLU after layers 1 and 2.  Input per pixel (8 channels,
 * 5 used): depth z (m), the unit normal from central differences of the
 * back-projected 4-neighbours (zero unless all are valid), validity.  Output:
 * the predicted |depth error| in centimetres. */
#define FF_CNN_PARAMS 8833
#define FF_CNN_FEAT_CH 8
#define FF_CNN_HIDDEN 16
#define FF_CNN_PACKED_BYTES 33280

/* Turn the learned weight on for this map (params: FF_CNN_PARAMS floats,
 * rounded to BF16; tau in metres), or off with params NULL. */
ff_status ff_set_confidence(ff_handle *h, const float *params, int n_params, float tau_m);

/* The confidence map of the last frame (width x height floats, host memory). */
ff_status ff_get_confidence_map(ff_handle *h, float *out, int *width, int *height);

/* Depth along each pixel's ray of the first surface of the fused map within
 * +-window_m of the pixel's measured depth (the SDF of the finest brick,
 * trilinear inside a brick, sampled every step_m of depth): 0 for pixels
 * without depth, -1 where no surface lies in the window.  d_depth and d_out are
 * device memory (uint16 and float, width x height); pose as in ff_add_map_u16. */
ff_status ff_raycast_depth(ff_handle *h, const double K[4], const double R[9], const double t[3],
                           const uint16_t *d_depth, int width, int height, float scaling, float window_m,
                           float step_m, float *d_out);

/* Training and inference kernels of the network on caller-owned device
 * memory (stream: a cudaStream_t, NULL for the default stream).  n images of
 * width x height; feat bf16 [n][h][w][8]; a1, a2 bf16 [n][h][w][16]; pred /
 * dpred / target float [n][h][w]; g1, g2 float [n][h][w][16] (scratch);
 * params bf16 and grads / master / m / v float [FF_CNN_PARAMS]; packed:
 * FF_CNN_PACKED_BYTES of scratch that ff_cnn_forward fills with the weights
 * laid out as tensor-core operands (one per concurrent call).
 * ff_cnn_forward writes the confidence when tau_m > 0, else the prediction.
 * ff_cnn_backward adds the parameter gradients of d(loss)/d(pred) to grads.
 * ff_cnn_mse: loss += sum over target >= 0 of (pred - target)^2 * inv_count,
 * dpred = 2 (pred - target) * inv_count (0 where target < 0).
 * ff_cnn_adam: one Adam step of master, BF16 copy into params, grads cleared. */
ff_status ff_cnn_features(const uint16_t *d_depth, int n, int width, int height, float scaling, const double K[4],
                          void *d_feat, void *stream);
ff_status ff_cnn_forward(const void *d_params, void *d_packed, const void *d_feat, int n, int width, int height,
                         void *d_a1, void *d_a2, float *d_out, float tau_m, void *stream);
ff_status ff_cnn_backward(const void *d_params, const void *d_feat, const void *d_a1, const void *d_a2,
                          const float *d_dpred, int n, int width, int height, float *d_g1, float *d_g2,
                          float *d_grads, void *stream);
ff_status ff_cnn_mse(const float *d_pred, const float *d_target, int64_t count, float inv_count, float *d_dpred,
                     double *d_loss, void *stream);
ff_status ff_cnn_adam(float *d_master, void *d_params, float *d_grads, float *d_m, float *d_v, float lr,
                      float beta1, float beta2, float eps, int step, void *stream);

/* Message of the last failure on this handle (or of ff_create when h is NULL). */
const char *ff_last_error(const ff_handle *h);

/* Library build/version string. */
const char *ff_version(void);

#ifdef __cplusplus
}
#endif
#endif
