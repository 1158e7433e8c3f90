/*
 * bvhcd.h -- C ABI of the B200 collision pipeline (LBVH + BVTT front +
 * triangle-triangle narrow phase).
 *
 * The entry points replace the reference's two module classes and its
 * scheduler; each declaration names the reference interface it stands in for
 * (paths inside littlemine/BVH-based-Collision-Detection-Scheme,
 * Mine/ = Source/Project/Mine/).  Plain pointers and sizes only: positions
 * are float[3] per vertex, faces int[3] per triangle, pairs int[2].  Streams
 * are cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Every function returns a bvhcd_status; nothing prints or exits.  Work is
 * enqueued asynchronously on the given stream; functions that return counts
 * to the host synchronise that stream and say so.
 */
#ifndef BVHCD_H_
#define BVHCD_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    BVHCD_OK = 0,
    BVHCD_INVALID_ARG = 1,
    BVHCD_OUT_OF_MEMORY = 2,
    BVHCD_CAPACITY_EXCEEDED = 3, /* a front / pair buffer overflowed; see stats */
    BVHCD_CUDA_ERROR = 4,
    BVHCD_TIMEOUT = 5,
    BVHCD_NOT_READY = 6          /* e.g. front maintained before any BVH build */
} bvhcd_status;

/* LBvhFixedDeformableMaintenance {BUILD, REFIT, UPDATE}
 * (Mine/collision/lbvh/LBvhFixedDeformable.h:20-21). */
typedef enum { BVHCD_BVH_BUILD = 0, BVHCD_BVH_REFIT = 1, BVHCD_BVH_UPDATE = 2 } bvhcd_bvh_op;

/* BvttFrontLooseIntraMaintenance {PURE_BVH_CD, GENERATE, UPDATE, REORDER,
 * KEEP, RESTRUCTURE} (Mine/collision/bvtt_front/BvttFrontLooseIntra.h:20-22). */
typedef enum {
    BVHCD_FRONT_PURE_BVH_CD = 0,
    BVHCD_FRONT_GENERATE = 1,
    BVHCD_FRONT_UPDATE = 2,
    BVHCD_FRONT_REORDER = 3,
    BVHCD_FRONT_KEEP = 4,
    BVHCD_FRONT_RESTRUCTURE = 5
} bvhcd_front_op;

/* LBvhBuildConfig{primSize, extSize, intSize} (Mine/setting/BvhSettings.h:49-54)
 * plus the CDBenchmarkSettings switches (Mine/setting/CDBenchmarkSettings.h:33-35). */
typedef struct {
    int32_t prim_capacity;   /* max triangles (reference default 150000) */
    int32_t vert_capacity;   /* max vertices */
    int32_t enable_restr;    /* quality-triggered restructuring (reference: on) */
    int32_t node_box_fp16;   /* precision mode: the front traversals read internal-node
                                boxes stored as FP16 rounded outward (16-byte records
                                instead of 32-byte ones); leaf tests stay FP32, so the
                                pair set is the same.  Fronts may differ (looser boxes). */
    int32_t reserved[4];
} bvhcd_bvh_config;

/* BvttFrontIntraBuildConfig{intFrontSize, extFrontSize, cpNum}
 * (Mine/setting/BvttFrontSettings.h:52-63). */
typedef struct {
    int64_t int_front_capacity;  /* reference default 2,300,000 */
    int64_t ext_front_capacity;  /* reference default 2,300,000 */
    int64_t pair_capacity;       /* reference default 1,600,000 */
    int32_t cull_adjacent;       /* drop pairs sharing a vertex id (covertex) */
    int32_t narrow_phase;        /* run the tri-tri test after the broad phase */
    int32_t auto_grow;           /* what an overflow of a front, pair or hit buffer does:
                                    0: nothing (reported in the stats; the front and the
                                       results of that maintain and of the ones working
                                       from its front are incomplete until a GENERATE);
                                    1: grow the buffers and replay the stage in the same
                                       call -- complete results every call, but each
                                       maintain reads the counters back (synchronises);
                                    2: deferred -- no synchronisation: each maintain copies
                                       its counters to pinned host memory with an event,
                                       and a later maintain that finds a completed copy
                                       showing an overflow grows the buffers and
                                       regenerates the front; the maintains in between
                                       report the overflow (stats, CAPACITY_EXCEEDED from
                                       bvhcd_front_pairs) */
    int32_t precision;           /* 0: the reference's FP32 narrow phase; 1: FP32 where
                                    certain, FP64 for the pairs it flags (hits equal an
                                    FP64 evaluation of every pair), FP64 contact points /
                                    distances where FP32 is ill-conditioned */
    int32_t reserved[4];
} bvhcd_front_config;

/* SceneData{pos, fids} (Mine/world/Scene.h:16-20).  Every maintain that
 * reads new positions also writes them into the BVH's own 16-byte records
 * (x, y, z, 0; 16 bytes of device memory per vertex of capacity), which the
 * FP32 narrow phase reads; the precision mode's narrow phase, the contacts
 * and the proximity queries read the positions given to the last maintain. */
typedef struct {
    const float *pos;      /* V x 3 */
    const int32_t *faces;  /* T x 3 vertex ids */
    int32_t num_vertices;
    int32_t num_faces;
    int32_t on_device;     /* 1: device pointers, read in place; 0: host pointers, copied */
    int32_t faces_static;  /* 1: faces unchanged since the last call (skip their copy) */
} bvhcd_scene;

/* A scene given as one axis-aligned box per primitive instead of triangles:
 * ARCSimSceneData{fsize, faces, boxes} (Mine/world/Scene.h:39-45), boxes a
 * simulator computed itself (for instance swept over its time step).  The
 * boxes take the place of the triangles' boxes everywhere (scene box, Morton
 * codes of their centres, leaves, refit, restructure); the faces give the
 * vertex ids for adjacency culling and the original ids of the pairs.  There
 * are no positions, so a front over such a BVH runs the broad phase only
 * (narrow_phase = 0). */
typedef struct {
    const void *boxes;     /* T x 6: min x, y, z, max x, y, z; FP32, or FP64 with boxes_f64 */
    const int32_t *faces;  /* T x 3 vertex ids */
    int32_t num_faces;
    int32_t boxes_f64;     /* 1: FP64 boxes, rounded outward to FP32 (min down, max up), so the
                              FP32 box contains the given one; the reference converts to nearest */
    int32_t on_device;     /* 1: device pointers (FP32 boxes read in place); 0: host, copied */
    int32_t faces_static;  /* 1: faces unchanged since the last call (skip their copy) */
} bvhcd_box_scene;

/* Stats the reference logs per frame in inspectResults
 * (Mine/collision/bvtt_front/BvttFrontLooseIntra.cu:50-61). */
typedef struct {
    int64_t int_front;       /* F_int */
    int64_t ext_front;       /* F_ext */
    int64_t broad_pairs;     /* cpNum */
    int64_t narrow_hits;     /* actualCpNum */
    int32_t overflow;        /* this maintain: bit0 int front, bit1 ext front, bit2 pairs,
                                bit3 hits, bit4 traversal bound, bit5 sprout work list,
                                bit6 the front it worked from had lost entries (bits 0,
                                1, 4, 5 carry over from maintain to maintain until a
                                GENERATE) */
    int32_t bvh_opt_tag;     /* 0 refit, 1 restructure, 2 build (BvhRestrLog.h:59) */
    int32_t front_op_run;    /* the front operation that actually ran */
    int32_t restr_pending;   /* quality check marked the BVH for restructuring */
    int32_t num_rt_subtrees; /* restructure decision inputs (LBvhFixedDeformable.cu:240-241) */
    int32_t num_rt_int_nodes;
    int32_t flagged;         /* precision mode: pairs the narrow phase re-decided in FP64 */
    int32_t keep_tested;     /* entries the last KEEP tested: all of them, or those whose
                                expiry had come (the others cannot have changed state) */
    int32_t overflow_any;    /* the overflow bits of every maintain since the front was
                                created (sticky; a replay of auto_grow = 1 clears its own) */
    int32_t nonfinite_input; /* 1: the last maintain of the front's BVH (either BVH of an
                                inter front) was given a NaN or infinite coordinate; the
                                frame's tree, front and pairs mean nothing, and
                                bvhcd_front_pairs returns BVHCD_INVALID_ARG.  The reference
                                does not check (its CUDA error checks exit the process,
                                Mine/utility/CudaThrustUtils.hpp:9-11). */
    int32_t reserved[2];
} bvhcd_front_stats;

typedef struct bvhcd_bvh bvhcd_bvh;
typedef struct bvhcd_front bvhcd_front;

const char *bvhcd_status_string(bvhcd_status s);
/* 1 when the library was built with device code for this device. */
bvhcd_status bvhcd_device_check(int32_t device, int32_t *ok);

/* ---- BVH module: replaces LBvhFixedDeformable
 * ctor  (Mine/collision/lbvh/LBvhFixedDeformable.cu:20-55, .h:30),
 * dtor  (.cu:57-66),
 * maintain(scheme, SceneData) (.cu:68-87),
 * getPrimNodeSize/getExtNodeSize/getIntNodeSize, bvhOptTag (.h:37-50). */
bvhcd_status bvhcd_bvh_create(const bvhcd_bvh_config *cfg, bvhcd_bvh **out);
bvhcd_status bvhcd_bvh_destroy(bvhcd_bvh *bvh);
bvhcd_status bvhcd_bvh_maintain(bvhcd_bvh *bvh, bvhcd_bvh_op op, const bvhcd_scene *scene,
                                void *stream);
/* maintain(scheme, const ARCSimSceneData&) (Mine/collision/lbvh/
 * LBvhFixedDeformable.cu:89-112, with the *ARCSim kernels of
 * LBvhBuildKernels.cu:10-52 and LBvhUpdateKernels.cu:11-32): the same
 * operations on a box scene.  A handle may switch between box and triangle
 * scenes at a BUILD. */
bvhcd_status bvhcd_bvh_maintain_boxes(bvhcd_bvh *bvh, bvhcd_bvh_op op, const bvhcd_box_scene *scene,
                                      void *stream);
bvhcd_status bvhcd_bvh_sizes(const bvhcd_bvh *bvh, int32_t *prims, int32_t *ext_nodes,
                             int32_t *int_nodes);
/* Copies the next frame's positions (host memory, num_vertices x 3 floats;
 * pinned memory lets the copy run asynchronously) into one of two device
 * staging buffers of the handle, on copy_stream, and returns the buffer's
 * device address in *staged.  A bvhcd_bvh_maintain or bvhcd_frame whose
 * scene has pos == that address (on_device = 1, faces on the device) first
 * makes its own stream wait for the copy, so the upload of frame f + 1 runs
 * while frame f computes; a buffer is refilled only after the frames that
 * read it.  One staged frame may be outstanding: a second call before a
 * maintain used the first returns BVHCD_NOT_READY.  Not for
 * bvhcd_frame_graph (its scene pointers are fixed).  The reference uploads
 * each frame's positions before the frame runs
 * (Mine/Frameworks/CudaProject/CudaProjectApp.cpp:49-52, Scene::getFormatedData). */
bvhcd_status bvhcd_bvh_stage_positions(bvhcd_bvh *bvh, const float *host_pos, int32_t num_vertices,
                                       void *copy_stream, const float **staged);
bvhcd_status bvhcd_bvh_opt_tag(const bvhcd_bvh *bvh, int32_t *tag);
/* Marks subtrees (internal nodes by DFS id, host array) as degraded, the
 * marks the front-quality check leaves in BvhRestrLog
 * (Mine/collision/bvtt_front/BvttFrontGenerateKernels.cu:45-47); the next
 * bvhcd_bvh_maintain applies the reference's restructure decision
 * (Mine/collision/lbvh/LBvhFixedDeformable.cu:210-352) to them.  Used by
 * schedulers that pick subtrees themselves.  Ignored when enable_restr = 0. */
bvhcd_status bvhcd_bvh_request_restructure(bvhcd_bvh *bvh, const int32_t *roots, int32_t n,
                                           void *stream);
/* Copies the tree to host arrays for invariant checks (the reference's
 * debug kernels checkBVHIntegrity / checkPrimmap,
 * Mine/collision/lbvh/LBvhBuildKernels.cu:228-293).  Synchronises `stream`.
 * inode: 6 ints per internal node in DFS order (lc, rc, par, mark, rangex,
 * rangey); ibox, lbox: 6 floats per node; leaf: 4 ints per Morton slot (orig
 * triangle id, parent, mark, lca); lca: T+1 ints; codes: T; primmap: T.
 * Any pointer may be NULL. */
bvhcd_status bvhcd_bvh_export(const bvhcd_bvh *bvh, int32_t *inode, float *ibox, int32_t *leaf,
                              float *lbox, int32_t *lca, uint32_t *codes, int32_t *primmap,
                              void *stream);

/* ---- Front module: replaces BvttFrontLooseIntra
 * ctor  (Mine/collision/bvtt_front/BvttFrontLooseIntra.cu:16-38), borrows the BVH,
 * dtor  (:40-48),
 * maintain(scheme) (:69-126),
 * inspectResults (:50-61) -> bvhcd_front_stats,
 * applyCpResults(uint*, uint2*) (:63-67) -> bvhcd_front_pairs(which = 0). */
bvhcd_status bvhcd_front_create(bvhcd_bvh *bvh, const bvhcd_front_config *cfg,
                                bvhcd_front **out);
/* Inter-object front: replaces BvttFrontLooseInter
 * (Mine/collision/bvtt_front/BvttFrontLooseInter.cu:16-331) over a deformable
 * BVH and a rigid one (LBvhRigid, Mine/collision/lbvh/LBvhRigid.cu: the same
 * build and refit without restructuring -- an ordinary BVH handle here).  The
 * rigid BVH's triangles traverse the deformable BVH; every front operation of
 * bvhcd_front_maintain applies (RESTRUCTURE, and a build or restructure of
 * either BVH, regenerate the front).  Pairs are (deformable triangle id, rigid
 * triangle id), as the reference writes them; every rigid triangle takes part
 * (the reference's generation skips the last one).  narrow_phase runs the
 * triangle test across the two meshes (the reference's inter front has no
 * narrow phase); cull_adjacent does not apply; precision must be 0.  Both
 * BVHs must hold one scene and stay alive, unmoved, while the front lives;
 * not for bvhcd_frame_graph, bvhcd_front_contacts, bvhcd_front_copy_state or
 * the learner. */
bvhcd_status bvhcd_front_create_inter(bvhcd_bvh *deformable, bvhcd_bvh *rigid, const bvhcd_front_config *cfg,
                                      bvhcd_front **out);
bvhcd_status bvhcd_front_destroy(bvhcd_front *front);
bvhcd_status bvhcd_front_maintain(bvhcd_front *front, bvhcd_front_op op, void *stream);
/* Synchronises `stream`. */
bvhcd_status bvhcd_front_stats_get(bvhcd_front *front, bvhcd_front_stats *stats, void *stream);
/* Copies pairs of original triangle ids.  which = 0: broad-phase candidate
 * pairs (applyCpResults); 1: pairs whose triangles intersect (the narrow
 * result the reference keeps in d_orderedCdpairs).  out_on_device selects a
 * device or host destination.  *count receives the full count even when it
 * exceeds cap (then only cap pairs are written and CAPACITY_EXCEEDED is
 * returned).  Synchronises `stream`. */
bvhcd_status bvhcd_front_pairs(bvhcd_front *front, int32_t which, int32_t *out, int64_t cap,
                               int64_t *count, int32_t out_on_device, void *stream);
/* Device pointer of the current hit list (pairs of original triangle ids)
 * and of two device-side int64 counts {broad pairs, hits}, both written by
 * the last maintain on its stream; valid until the next maintain.  No sync. */
bvhcd_status bvhcd_front_device_results(bvhcd_front *front, const int32_t **hit_pairs,
                                        const int64_t **counts);
/* Asynchronous read-back: enqueues on `stream` a kernel that writes the pairs
 * (which as in bvhcd_front_pairs, the same order) and their count straight
 * into host memory from bvhcd_host_alloc, so nothing synchronises and the
 * next frame can be enqueued at once; the results are valid once the stream
 * has passed this point (an event).  At most cap pairs are written;
 * *host_count receives the full count.  No counterpart in the reference,
 * whose applyCpResults / inspectResults copy synchronously
 * (BvttFrontLooseIntra.cu:50-67). */
bvhcd_status bvhcd_front_pairs_async(bvhcd_front *front, int32_t which, int32_t *host_out, int64_t cap,
                                     int64_t *host_count, void *stream);
/* Pinned host memory mapped into the device's address space (for
 * bvhcd_front_pairs_async), and its release. */
bvhcd_status bvhcd_host_alloc(int64_t bytes, void **ptr);
bvhcd_status bvhcd_host_free(void *ptr);
/* Copies the current front (sorted-prim, node) entries; which = 0 internal,
 * 1 external.  Synchronises `stream`. */
bvhcd_status bvhcd_front_export(bvhcd_front *front, int32_t which, int32_t *out, int64_t cap,
                                int64_t *count, void *stream);

/* ---- Stage timing: the reference's Logger::recordSection GPU sections
 * (Mine/utility/CudaTimer.hpp:43-53, e.g. "refit_bvh", "broad_phase_cd_update",
 * "narrow_phase").  When enabled, the library records a CUDA event pair on
 * the work stream around each stage (no synchronisation); reading the times
 * synchronises the events and accumulates them per stage. */
typedef enum {
    BVHCD_STAGE_BVH_BUILD = 0,
    BVHCD_STAGE_BVH_REFIT = 1,
    BVHCD_STAGE_BVH_RESTRUCTURE = 2,
    BVHCD_STAGE_FRONT_GENERATE = 3,
    BVHCD_STAGE_FRONT_UPDATE = 4,
    BVHCD_STAGE_FRONT_KEEP = 5,
    BVHCD_STAGE_FRONT_BALANCE = 6,
    BVHCD_STAGE_FRONT_REORDER = 7,
    BVHCD_STAGE_NARROW = 8,
    BVHCD_STAGE_QUALITY = 9,
    BVHCD_STAGE_PURE_BVH_CD = 10,
    BVHCD_STAGE_FRONT_RESTRUCTURE = 11,  /* an inter front re-sprouting restructured subtrees
                                            ("broad_phase_restr_front") */
    BVHCD_STAGE_COUNT = 12
} bvhcd_stage;

bvhcd_status bvhcd_profile_enable(bvhcd_bvh *bvh, int32_t on);
/* ms[i] = summed milliseconds of stage i since the last reset, calls[i] =
 * number of timed calls.  reset != 0 clears the sums after reading. */
bvhcd_status bvhcd_profile_read(bvhcd_bvh *bvh, double *ms, int64_t *calls, int32_t reset);

/* Number of kernels this library has launched in this process (a counter
 * for benchmarks; no reference counterpart beyond the per-kernel timers of
 * Mine/system/CudaDevice/CudaKernelLauncher.cu:54-69). */
bvhcd_status bvhcd_launch_count(int64_t *n);

/* Fault injection for tests (no counterpart in the reference, whose
 * allocation failures end the process in checkCudaErrors): the n-th device
 * allocation the library makes from now on (n >= 1) fails as if the device
 * were out of memory, so the call that makes it returns BVHCD_OUT_OF_MEMORY;
 * n = 0 cancels a planned fault.  Host-side only: nothing reaches the GPU. */
bvhcd_status bvhcd_debug_fail_alloc(int64_t n);

/* ---- Morton order without device allocation.  No counterpart in the
 * reference.  For callers that may not allocate device memory once they are
 * running -- a simulator that hands the whole device to its own memory pool,
 * or a real-time loop in which cudaMalloc's implicit device synchronisation
 * is not allowed -- this computes what a BVH build starts with: the scene
 * box, the 30-bit Morton code of every triangle and the stable sort by code.
 * codes[s] receives the s-th smallest code, order[s] the original triangle
 * id in Morton slot s (ties keep the original order), the same codes and
 * order bvhcd_bvh_maintain(BUILD) produces.  All pointers are device
 * pointers the caller owns; the temporaries live in one fixed device array of
 * the library (about 9.2 MB, present on every GPU that loads the library
 * until the process exits), so num_faces is limited to
 * BVHCD_NOALLOC_MAX_FACES; larger requests return BVHCD_CAPACITY_EXCEEDED
 * without touching the GPU.  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress); make that first call before any
 * stream capture.  Under CUDA's lazy module loading the library's device code,
 * and with it the array, is loaded on a device at the first use of any of its
 * kernels there -- possibly this call -- which allocates and synchronises
 * once: make the first call during initialisation, not in the loop that must
 * not allocate.  Calls share the array: two calls whose work overlaps on
 * the GPU (different streams, or different host threads) race and must be
 * serialised by the caller.  Asynchronous on `stream`. */
#define BVHCD_NOALLOC_MAX_FACES 1048576
bvhcd_status bvhcd_morton_order_noalloc(const float *pos, const int32_t *faces, int32_t num_faces,
                                        uint32_t *codes, int32_t *order, void *stream);

/* ---- Batched scenes.  No counterpart in the reference, which builds one
 * tree over all meshes of a SceneData (Mine/world/Scene.cpp:31-40).  The
 * num_faces triangles of every bvhcd_scene given to this BVH are num_scenes
 * independent scenes: scene s owns triangles [tri_offsets[s],
 * tri_offsets[s+1]) (a host array of num_scenes + 1 ints, tri_offsets[0] = 0,
 * at least 2 triangles per scene when num_scenes > 1; faces keep global
 * vertex ids).  Each scene gets its own tree -- the tree it would get on its
 * own, with its Morton slots shifted by tri_offsets[s] and its internal-node
 * ids by tri_offsets[s] - s -- no pair crosses scenes, and every stage runs
 * over all scenes in one launch.  Pairs carry global triangle ids;
 * bvhcd_bvh_sizes reports num_faces - num_scenes internal nodes.  Requires
 * enable_restr = 0.  num_scenes = 1 returns to a single scene; the next
 * maintain rebuilds either way. */
bvhcd_status bvhcd_bvh_set_scenes(bvhcd_bvh *bvh, int32_t num_scenes, const int32_t *tri_offsets);

/* ---- Proximities of the broad pairs (no counterpart in the reference's
 * pipeline: it carries signed_vf_distance and signed_ee_distance,
 * Mine/utility/CudaDeviceUtils.cu:163-193, the measures a cloth solver builds
 * its repulsion constraints from, but never calls them).  For every broad
 * pair, in the order of bvhcd_front_pairs(which = 0), every vertex-face and
 * edge-edge feature pair of the two triangles whose signed distance is within
 * `thickness` and whose closest points lie inside both features (all
 * barycentric weights non-negative), skipping feature pairs that share a
 * vertex id.  FP64 from the FP32 positions.  Records come ordered by pair,
 * then kind, then feature. */
typedef struct {
    int32_t pair;    /* index of the pair in bvhcd_front_pairs(which = 0) order */
    int32_t kind;    /* 0: vertex fa of the first triangle against the second's face;
                        1: vertex fb of the second triangle against the first's face;
                        2: edge fa of the first (its vertices fa, fa + 1 mod 3) against edge fb of the second */
    int32_t fa, fb;  /* feature indices, -1 where the kind has none */
    double dist;     /* signed distance along n (vertex minus face / first edge minus second) */
    double n[3];     /* unit normal: the face's for kinds 0 and 1, the two edges' cross product for 2 */
    double w[4];     /* weights as signed_vf_distance (1, -b0, -b1, -b2 over the face) and
                        signed_ee_distance (a0, a1 on the first edge, -b0, -b1 on the second) give them */
} bvhcd_proximity;
/* pos: device positions (V x 3 FP32) of the front's BVH, or NULL for the
 * positions of its last maintain (required for a box scene, which has none;
 * NULL for an inter front, which uses each BVH's own).  out: host, or device
 * with out_on_device; *count receives the full count (CAPACITY_EXCEEDED and
 * the first cap records when it exceeds cap).  Synchronises `stream`. */
bvhcd_status bvhcd_front_proximity(bvhcd_front *front, const float *pos, double thickness, bvhcd_proximity *out,
                                   int64_t cap, int64_t *count, int32_t out_on_device, void *stream);

/* ---- Mesh files.  Reads a Wavefront OBJ file -- the format of the reference's
 * benchmark frames, loaded per frame by Scene::update / addMesh
 * (Mine/world/Scene.cpp:14-43) through assimp with triangulation
 * (Mine/utility/ModelReader.hpp:23-27) -- into positions (V x 3) and faces
 * (T x 3, 0-based): v records and f records (v, v/vt, v//vn, v/vt/vn corners,
 * negative ids relative to the vertices read so far), polygons split into a
 * fan around their first corner, other records skipped.  Vertex ids stay as
 * the file shares them (assimp's OBJ import gives every face corner its own
 * vertex, which leaves nothing for adjacency culling).  With pos / faces NULL
 * only the counts are returned; CAPACITY_EXCEEDED when a count exceeds its
 * capacity (the first vcap / fcap records are written).  INVALID_ARG for a
 * missing file or a malformed v or f record.  Host only. */
bvhcd_status bvhcd_obj_read(const char *path, float *pos, int32_t vcap, int32_t *faces, int32_t fcap,
                            int32_t *num_vertices, int32_t *num_faces);

/* ---- Contact points and distances (precision mode extension; the
 * reference's narrow phase returns a hit flag only, narrow_phase.cu:8-24).
 * which = 0: for every hit, in the order bvhcd_front_pairs(which = 1) returns
 * them, the midpoint (x, y, z) and length (w) of the two triangles'
 * intersection segment (NaN point for coplanar pairs); which = 1: for every
 * broad-phase pair, in the order of bvhcd_front_pairs(which = 0), the distance
 * between the two triangles (w; 0 for intersecting pairs).  Computed in FP32,
 * or in FP64 with precision = 1; written as FP32.  out: 4 floats per item
 * (host, or device with out_on_device); flagged (may be NULL) receives how
 * many items were computed in FP64.  Synchronises `stream`. */
bvhcd_status bvhcd_front_contacts(bvhcd_front *front, int32_t which, float *out, int64_t cap, int64_t *count,
                                  int64_t *flagged, int32_t out_on_device, void *stream);
/* The same computed and written in FP64: 4 doubles per item.  FP32 results
 * carry the FP32 rounding of absolute coordinates -- half an ulp of a
 * coordinate near 1 is about 1e-5 of a 2e-3 triangle -- which this form does
 * not. */
bvhcd_status bvhcd_front_contacts64(bvhcd_front *front, int32_t which, double *out, int64_t cap, int64_t *count,
                                    int32_t out_on_device, void *stream);

/* ---- State copies.  No counterpart in the reference.  dst becomes a copy of
 * src -- tree, restructure log, counters, fronts, pairs and their host-side
 * state -- so the two continue independently from the same frame (the
 * learned scheduler's counterfactual runs fork this way).  dst must have the
 * configuration src has (the same enable_restr; a front bound to another BVH
 * handle, itself a copy of src's BVH).  Device input that src reads in place
 * is read in place by dst too.  Asynchronous on `stream`. */
bvhcd_status bvhcd_bvh_copy_state(bvhcd_bvh *dst, const bvhcd_bvh *src, void *stream);
bvhcd_status bvhcd_front_copy_state(bvhcd_front *dst, const bvhcd_front *src, void *stream);

/* ---- Learned scheduler.  No counterpart in the reference, whose schedule is
 * the static cycle of BenchmarkLogic::maintainScheme plus the front-quality
 * check (Mine/system/Logic/BenchmarkLogic.hpp:90-156,
 * Mine/collision/bvtt_front/BvttFrontGenerateKernels.cu:34-49).
 *
 * The tree is cut into disjoint subtrees (internal nodes with at most
 * max_subtree_leaves leaves whose parent has more).  Every frame the GPU
 * computes 16 features per subtree (subtree size and depth, SAH ratio, box
 * volume and area growth since the last build, mean / max / large leaf
 * displacement since the last build in mean leaf diagonals, front entries and
 * their int/ext balance against the last front generation, front density,
 * frames since build and since generation, tree size, a constant) and a
 * 16-64-64-3 MLP (BF16 weight matrices, FP32 biases and accumulation) votes
 * per subtree: 0 refit, 1 restructure, 2 regenerate the front.  The votes
 * become the reference's own operations: restructure marks on the voted
 * subtrees (applied by the next BVH maintain with the reference's restructure
 * decision), and a front GENERATE in the next frame when subtrees holding more
 * than half of the cut's leaves vote for it.  Pair sets never depend on it.
 * The BVH must have enable_restr = 1 and one scene; the learner turns the
 * front's own quality check off.  The weights live on the device: set them
 * (BVHCD_MLP_PARAMS floats: W1[16][64], b1[64], W2[64][64], b2[64],
 * W3[64][3], b3[3], row-major, input index first) or train them with
 * bvhcd_mlp_train. */
#define BVHCD_MLP_PARAMS 5443
typedef struct bvhcd_learner bvhcd_learner;
bvhcd_status bvhcd_learner_create(bvhcd_bvh *bvh, bvhcd_front *front, int32_t max_subtree_leaves,
                                  bvhcd_learner **out);
bvhcd_status bvhcd_learner_destroy(bvhcd_learner *learner);
bvhcd_status bvhcd_learner_set_params(bvhcd_learner *learner, const float *params);
bvhcd_status bvhcd_learner_get_params(const bvhcd_learner *learner, float *params);
/* One learned frame: BVH refit (build on frame 0; a restructure when a
 * decision marked subtrees), then KEEP -- or, with a front cycle of c > 0
 * frames set (bvhcd_learner_set_front_cycle), the reference's cycle (UPDATE at
 * frame % c == 0, REORDER at c - 1, KEEP otherwise) -- or GENERATE after a
 * rebuild or a regenerate vote.  Every `decide_every` frames (default 3) it queues a
 * decision -- features, votes, marks and counts on the device, an event --
 * and the first frame that finds the event complete applies it; the host never
 * waits for it.  A decision voted on a tree that has changed since is dropped.
 * bvh_tag receives the reference's opt tag (0 refit, 1 restructure, 2 build),
 * front_op the op run; either may be NULL. */
bvhcd_status bvhcd_learner_set_decide_every(bvhcd_learner *learner, int32_t frames);
/* The front operations between decisions: 0 (the default) keeps the front
 * until a vote or a tree change regenerates it; c > 0 runs the reference's
 * front cycle of c frames (BvttFrontSettings.h:49 uses 6). */
bvhcd_status bvhcd_learner_set_front_cycle(bvhcd_learner *learner, int32_t frames);
bvhcd_status bvhcd_learner_frame(bvhcd_learner *learner, const bvhcd_scene *scene, int32_t frame,
                                 int32_t *bvh_tag, int32_t *front_op, void *stream);
/* Trace recording under another schedule: after each frame's maintains, tell
 * the learner whether the tree was rebuilt or restructured and whether the
 * front was generated (it recomputes the cut and its references). */
bvhcd_status bvhcd_learner_observe(bvhcd_learner *learner, int32_t tree_changed, int32_t front_generated,
                                   void *stream);
/* The cut's subtree roots (DFS ids) to host memory; roots may be NULL to ask
 * for the count. */
bvhcd_status bvhcd_learner_cut(const bvhcd_learner *learner, int32_t *roots, int32_t cap, int32_t *n, void *stream);
/* The features of the current frame (n rows of 16 floats) to host memory; X
 * may be NULL to compute them on the device only. */
bvhcd_status bvhcd_learner_features(bvhcd_learner *learner, float *X, int32_t cap_rows, int32_t *n, void *stream);
/* Front entries per cut subtree in `front` (any front over a tree that shares
 * this learner's cut ranges: a copy, or one restructured inside them). */
bvhcd_status bvhcd_learner_work(bvhcd_learner *learner, const bvhcd_front *front, int64_t *out, int32_t cap,
                                void *stream);
/* Training on the GPU.  X (n x 16 floats) and y (n labels in {0,1,2}) are
 * device arrays, class_weight 3 host floats; the loss is the class-weighted
 * mean cross-entropy (1/n) sum_r w[y_r] CE_r.  gradient: the loss gradient of
 * all n rows at the current weights, to host memory (BVHCD_MLP_PARAMS floats,
 * d loss / d master weight, the BF16 rounding passed straight through).
 * train: `epochs` passes of Adam (beta 0.9 / 0.999, eps 1e-8) over minibatches
 * of `batch` rows in a seeded shuffle; last_loss receives the mean minibatch
 * loss of the last epoch.  predict: logits (n x 3) and votes of device rows;
 * either output may be NULL. */
bvhcd_status bvhcd_mlp_gradient(bvhcd_learner *learner, const float *X, const int32_t *y, int32_t n,
                                const float *class_weight, float *grad, float *loss, void *stream);
bvhcd_status bvhcd_mlp_train(bvhcd_learner *learner, const float *X, const int32_t *y, int32_t n,
                             const float *class_weight, int32_t epochs, int32_t batch, float lr, uint32_t seed,
                             float *last_loss, void *stream);
bvhcd_status bvhcd_mlp_predict(bvhcd_learner *learner, const float *X, int32_t n, float *logits, int32_t *vote,
                               void *stream);

/* ---- Launch shapes of the front stages.  No counterpart in the reference,
 * whose launcher derives one block size per kernel from occupancy
 * (Mine/system/CudaDevice/CudaDevice.cu:86-95).  unroll: front entries one
 * thread tests per step (1, 2 or 4; read by the four front scans); block:
 * threads per block (128, 256 or 512).  Results never depend on the shapes. */
enum {
    BVHCD_SHAPE_KEEP = 0,       /* keep scan */
    BVHCD_SHAPE_PRUNE_INT = 1,  /* prune/sprout update, internal entries */
    BVHCD_SHAPE_PRUNE_EXT = 2,  /* prune/sprout update, external entries */
    BVHCD_SHAPE_BALANCE = 3,    /* balance scan */
    BVHCD_SHAPE_SPROUT = 4,     /* traversal below overlapping front nodes */
    BVHCD_SHAPE_NARROW = 5,     /* narrow phase */
    BVHCD_SHAPE_COUNT = 6
};
typedef struct {
    int32_t unroll[BVHCD_SHAPE_COUNT];
    int32_t block[BVHCD_SHAPE_COUNT];
} bvhcd_launch_shapes;
bvhcd_status bvhcd_front_get_shapes(const bvhcd_front *front, bvhcd_launch_shapes *shapes);
/* Values outside the sets above return BVHCD_INVALID_ARG. */
bvhcd_status bvhcd_front_set_shapes(bvhcd_front *front, const bvhcd_launch_shapes *shapes);
/* Autotuner: on the front's current tree and front (it needs a generated
 * front: BVHCD_NOT_READY otherwise), times each stage in every candidate
 * shape -- 9 for the scans, 3 block sizes for sprout and the narrow phase --
 * `repeats` times after one untimed run, and keeps the fastest.  The stages
 * run on the real front without committing it; at the end the front is
 * regenerated from the current tree (a GENERATE, pairs and hits included), so
 * the next frame continues from a consistent state.  `chosen` (may be NULL)
 * receives the shapes, `best_ms` (may be NULL, BVHCD_SHAPE_COUNT doubles)
 * the mean time per run of each stage in its chosen shape.  Synchronises
 * `stream`. */
bvhcd_status bvhcd_front_autotune(bvhcd_front *front, int32_t repeats, bvhcd_launch_shapes *chosen,
                                  double *best_ms, void *stream);

/* ---- Graph-launched frame.  No counterpart in the reference.  Runs
 * bvhcd_bvh_maintain(bvh_op) then bvhcd_front_maintain(front_op) on
 * `stream` (not the legacy default stream).  The first call runs ordinary
 * launches (it sizes every buffer); afterwards each distinct (bvh_op,
 * front_op, host-side state of both handles) is captured once as a CUDA
 * graph, launched, and replayed by later calls with the same key.  The scene
 * must be device-resident (on_device = 1) and use the same pointers and sizes
 * on every call: the graphs read it in place, so the caller writes each
 * frame's positions into that buffer before the call.  Requires
 * enable_restr = 0 on the BVH and auto_grow = 0 on the front (capacities are
 * fixed inside a graph; an overflow still shows in bvhcd_front_stats).
 * Another scene pointer or size, bvhcd_bvh_set_scenes, or a change of
 * launch shapes drops the captured graphs.  The stage profiler does not time graph-launched frames. */
bvhcd_status bvhcd_frame_graph(bvhcd_bvh *bvh, bvhcd_front *front, const bvhcd_scene *scene,
                               int32_t bvh_op, int32_t front_op, void *stream);

/* ---- Scheduler: BenchmarkLogic::maintainScheme, STATIC_MANDATORY with
 * divergent marks (Mine/system/Logic/BenchmarkLogic.hpp:90-156). */
bvhcd_status bvhcd_schedule_heuristic(int32_t frame, int32_t start_frame, int32_t *bvh_op,
                                      int32_t *front_op);

/* ---- One-call frame: schedule + BVH maintain + front maintain, the body of
 * CudaProjectApp::Main's loop (Mine/Frameworks/CudaProject/CudaProjectApp.cpp:49-52). */
bvhcd_status bvhcd_frame(bvhcd_bvh *bvh, bvhcd_front *front, int32_t frame, int32_t start_frame,
                         const bvhcd_scene *scene, void *stream);

#ifdef __cplusplus
}
#endif
#endif
