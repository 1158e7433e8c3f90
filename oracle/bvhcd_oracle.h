/*
 * bvhcd_oracle.h -- CPU restatement of the reference collision path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  It is the checker that the CUDA path is compared with
 * (tests/, __graft_entry__.smoke()) and the CPU baseline timed by bench.py.
 *
 * Parity pin: the reference ships no tests, fixtures or golden vectors.  This
 * restatement is pinned by (a) an independent sweep-and-prune enumeration of
 * the FP32 AABB-overlap pair set (orc_brute_pairs), which the front pipeline
 * must reproduce exactly, (b) the gProximity tri-tri predicate compiled from
 * the reference's own header into oracle/_ref (oracle/ref_build.sh), which the
 * FP32 SAT restatement must agree with bit for bit, and (c) the exact
 * expansion-arithmetic tri-tri predicate in exact_tritri.c.
 *
 * Every stage cites the reference kernel it restates, by path inside the
 * reference project (Mine/ = Source/Project/Mine/).
 */
#ifndef BVHCD_ORACLE_H_
#define BVHCD_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Maintenance options, same order as the reference enums
 * (Mine/collision/lbvh/LBvhFixedDeformable.h:20-21,
 *  Mine/collision/bvtt_front/BvttFrontLooseIntra.h:20-22). */
enum { ORC_BVH_BUILD = 0, ORC_BVH_REFIT = 1, ORC_BVH_UPDATE = 2 };
enum { ORC_FRONT_PURE_BVH_CD = 0, ORC_FRONT_GENERATE = 1, ORC_FRONT_UPDATE = 2,
       ORC_FRONT_REORDER = 3, ORC_FRONT_KEEP = 4, ORC_FRONT_RESTRUCTURE = 5 };

typedef struct orc_pipe orc_pipe;

/* A pipeline = LBvhFixedDeformable + BvttFrontLooseIntra + narrow phase. */
orc_pipe *orc_pipe_create(int restr_enabled, int cull_adjacent, int narrow_enabled);
void orc_pipe_destroy(orc_pipe *p);
/* Runs one frame: BVH maintain then front maintain (+ narrow phase). */
int orc_pipe_frame(orc_pipe *p, int T, const int *faces, int V, const float *verts,
                   int bvh_op, int front_op);
/* info[0..15]: T, F_int, F_ext, P (broad pairs), H (narrow hits), opt tag,
 * restr-log-updated, numRtSubtree, numRtIntNode, front op actually run,
 * narrow ran (0/1). */
void orc_pipe_info(const orc_pipe *p, int64_t *info);
/* which = 0: broad-phase pairs (orig ids, emission order), 1: narrow hits. */
int64_t orc_pipe_pairs(const orc_pipe *p, int which, int *out, int64_t cap);
/* which = 0: internal front, 1: external front; entries (sorted prim, node). */
int64_t orc_pipe_front(const orc_pipe *p, int which, int *out, int64_t cap);
/* Tree export (DFS order internal nodes, Morton-order leaves).
 * inode: 6 ints per internal node (lc, rc, par, mark, rangex, rangey)
 * ibox : 6 floats per internal node, leaf: 4 ints per leaf (orig id, par,
 * mark, lca), lca has T+1 entries (last = -1) -> stored in leaf_lca. */
int orc_pipe_tree(const orc_pipe *p, int *inode, float *ibox, int *leaf,
                  float *lbox, int *leaf_lca, unsigned *codes, int *primmap);
/* Per-node front counts and begins as the log holds them now. */
int orc_pipe_log(const orc_pipe *p, unsigned *intcnt, unsigned *extcnt,
                 unsigned *intbeg, unsigned *extbeg);
void orc_set_threads(int n);
/* Test pinning only: restructure with the reference's own primitive-map
 * update (LBvhRestructureKernels.cu:68-120) run in thread order. */
void orc_pipe_set_reference_permutation(orc_pipe *p, int on);
void orc_pipe_mark_restructure(orc_pipe *p, const int *roots, int n);

/* Standalone stages. */
void orc_scene_box(int T, const int *faces, const float *verts, float *box6);
void orc_morton_codes(int T, const int *faces, const float *verts, const float *box6,
                      unsigned *codes);
/* All unordered pairs (i<j by orig id) whose FP32 AABBs overlap (touching
 * counts), optionally without pairs sharing a vertex id.  Sweep and prune. */
int64_t orc_brute_pairs(int T, const int *faces, const float *verts, int cull,
                        int *out, int64_t cap);
int orc_tritri_sat32(const float *p9, const float *q9);
int orc_tritri_exact(const float *p9, const float *q9);
/* Batch forms over pairs of orig triangle ids. */
void orc_narrow_sat32(int64_t n, const int *pairs, const int *faces, const float *verts,
                      unsigned char *hit);
void orc_narrow_exact(int64_t n, const int *pairs, const int *faces, const float *verts,
                      unsigned char *hit);
void orc_schedule(int frame, int start, int *bvh_op, int *front_op);

/* Precision mode references (precision_oracle.c): FP64 SAT, intersection
 * segment (midpoint xyz, length; returns 1, 0 = none, 2 = coplanar), triangle
 * distance, and all three over a pair list (any output may be NULL). */
int orc_tritri_sat64(const float *p9, const float *q9);
int orc_contact64(const float *p9, const float *q9, double *out4);
double orc_tri_distance64(const float *p9, const float *q9);
void orc_precision_pairs(int64_t n, const int *pairs, const int *faces, const float *verts,
                         unsigned char *hit64, double *contact4, double *dist);

/* Proximities of a pair list (proximity_oracle.c): the layout of
 * bvhcd_proximity.  Pairs index faces fa (first) and fb (second); returns the
 * count and writes up to cap records in the kernel's order. */
typedef struct {
    int32_t pair, kind, fa, fb;
    double dist, n[3], w[4];
} orc_prox;
int64_t orc_proximity(int64_t n, const int *pairs, const int *fa, const float *va, const int *fb, const float *vb,
                      int same_mesh, double h, orc_prox *out, int64_t cap);

#ifdef __cplusplus
}
#endif
#endif
