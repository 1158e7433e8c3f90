/*
 * bvhcd_oracle.c -- CPU restatement of the reference collision path
 * (LBVH build / refit / restructure, BVTT front generate / prune-sprout /
 * keep / reorder / balance, quality check, FP32 SAT narrow phase).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py.  The product library never links it.
 *
 * Each function names the reference kernel it restates (paths inside the
 * reference project, Mine/ = Source/Project/Mine/).  Parallel loops use
 * OpenMP; emission order is therefore not deterministic, exactly like the
 * reference's atomicAdd emission, so callers compare fronts and pair lists
 * as sorted multisets.  Per-node counts, begins, the tree and the restructure
 * decision are deterministic.
 *
 * Deviations from the reference, each deliberate:
 *  - restructure permutes the restructured primitives by the sort
 *    permutation (the reference's updatePrimMap, LBvhRestructureKernels.cu:68-77,
 *    applies its inverse and reads the slot->triangle map while other threads
 *    write it, so that map can stop being a permutation: triangles vanish
 *    from the leaves and others appear twice).  orc_pipe_set_reference_
 *    permutation() switches to the reference's update run in thread order,
 *    which reproduces the reference bit for bit on a restructure that starts
 *    from a consistent tree; it exists to pin the rest of the restructure
 *    against the reference and is not what the product computes;
 *  - the narrow phase runs on every frame (the reference skips it on frames
 *    whose BVH was restructured, BvttFrontLooseIntra.cu:84-109).
 */
#include "bvhcd_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float mn[3], mx[3]; } obox;

/* ------------------------------------------------------------------ */
/* growable int-pair vector                                           */
typedef struct { int *d; int64_t n, cap; } pvec;

static void pv_reserve(pvec *v, int64_t cap) {
    if (cap <= v->cap) return;
    int64_t nc = v->cap ? v->cap : 1024;
    while (nc < cap) nc *= 2;
    v->d = (int *)realloc(v->d, sizeof(int) * 2 * (size_t)nc);
    v->cap = nc;
}
static inline void pv_push(pvec *v, int a, int b) {
    if (v->n == v->cap) pv_reserve(v, v->n + 1);
    v->d[2 * v->n] = a;
    v->d[2 * v->n + 1] = b;
    v->n++;
}
static void pv_free(pvec *v) { free(v->d); v->d = NULL; v->n = v->cap = 0; }

/* per-thread emission buffers merged after each parallel loop */
#define ORC_MAX_THREADS 256
typedef struct { pvec intf, extf, pairs; } emitbuf;

static int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
static int orc_tid(void) {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ */
/* boxes: AABB::empty/combines/overlaps (Mine/base/Bv.h:27-45,80-84)   */
static inline void box_empty(obox *b) {
    b->mn[0] = b->mn[1] = b->mn[2] = FLT_MAX;
    b->mx[0] = b->mx[1] = b->mx[2] = -FLT_MAX;
}
static inline void box_add(obox *b, const float *v) {
    for (int k = 0; k < 3; k++) {
        b->mn[k] = fminf(b->mn[k], v[k]);
        b->mx[k] = fmaxf(b->mx[k], v[k]);
    }
}
static inline void box_merge(obox *o, const obox *a, const obox *b) {
    for (int k = 0; k < 3; k++) {
        o->mn[k] = fminf(a->mn[k], b->mn[k]);
        o->mx[k] = fmaxf(a->mx[k], b->mx[k]);
    }
}
/* BvhBvCompletePort::overlaps (Mine/collision/lbvh/BvhBV.h:54-59); touching overlaps */
static inline int box_overlap(const obox *node, const obox *b) {
    if (b->mn[0] > node->mx[0] || b->mx[0] < node->mn[0]) return 0;
    if (b->mn[1] > node->mx[1] || b->mx[1] < node->mn[1]) return 0;
    if (b->mn[2] > node->mx[2] || b->mx[2] < node->mn[2]) return 0;
    return 1;
}
static inline void tri_box(obox *b, const int *faces, const float *verts, int t) {
    box_empty(b);
    box_add(b, verts + 3 * (size_t)faces[3 * (size_t)t + 0]);
    box_add(b, verts + 3 * (size_t)faces[3 * (size_t)t + 1]);
    box_add(b, verts + 3 * (size_t)faces[3 * (size_t)t + 2]);
}

/* covertex (Mine/utility/CudaDeviceUtils.cu:153-157) */
static inline int covertex(const int *a, const int *b) {
    return a[0] == b[0] || a[0] == b[1] || a[0] == b[2] || a[1] == b[0] || a[1] == b[1] ||
           a[1] == b[2] || a[2] == b[0] || a[2] == b[1] || a[2] == b[2];
}

/* ------------------------------------------------------------------ */
/* Morton codes: expandBits / morton3D (Mine/utility/CudaDeviceUtils.cu:82-130)
 * and calcMCs (Mine/collision/lbvh/LBvhBuildKernels.cu:76-91).        */
static inline unsigned expand10(unsigned v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
static inline unsigned quant1024(float x) {
    x = fminf(fmaxf(x * 1024.0f, 0.0f), 1023.0f);
    return (unsigned)x;
}
static inline unsigned morton_of_box(const obox *b, const obox *scene) {
    float c[3], o[3];
    for (int k = 0; k < 3; k++) {
        c[k] = (float)((double)(b->mn[k] + b->mx[k]) * 0.5); /* AABB::center, Bv.h:65-67 */
        o[k] = c[k] - scene->mn[k];
    }
    float w = scene->mx[0] - scene->mn[0];
    float h = scene->mx[1] - scene->mn[1];
    float d = scene->mx[2] - scene->mn[2];
    unsigned xx = expand10(quant1024(o[0] / w));
    unsigned yy = expand10(quant1024(o[1] / h));
    unsigned zz = expand10(quant1024(o[2] / d));
    return xx * 4 + yy * 2 + zz;
}

/* calcMaxBV (LBvhBuildKernels.cu:55-74): scene box over triangle boxes */
void orc_scene_box(int T, const int *faces, const float *verts, float *box6) {
    obox s;
    box_empty(&s);
    for (int t = 0; t < T; t++) {
        obox b;
        tri_box(&b, faces, verts, t);
        box_merge(&s, &s, &b);
    }
    memcpy(box6, s.mn, 3 * sizeof(float));
    memcpy(box6 + 3, s.mx, 3 * sizeof(float));
}

void orc_morton_codes(int T, const int *faces, const float *verts, const float *box6,
                      unsigned *codes) {
    obox s;
    memcpy(s.mn, box6, 3 * sizeof(float));
    memcpy(s.mx, box6 + 3, 3 * sizeof(float));
#pragma omp parallel for schedule(static)
    for (int t = 0; t < T; t++) {
        obox b;
        tri_box(&b, faces, verts, t);
        codes[t] = morton_of_box(&b, &s);
    }
}

/* stable LSD radix sort of (key, val) pairs, the thrust::sort_by_key the
 * reference calls (LBvhFixedDeformable.cu:355-363, :300) */
static void radix_sort_u32(int n, unsigned *key, int *val) {
    unsigned *k2 = (unsigned *)malloc(sizeof(unsigned) * (size_t)(n > 0 ? n : 1));
    int *v2 = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int shift = 0; shift < 32; shift += 8) {
        int64_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (int i = 0; i < n; i++) cnt[((key[i] >> shift) & 255) + 1]++;
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (int i = 0; i < n; i++) {
            int64_t pos = cnt[(key[i] >> shift) & 255]++;
            k2[pos] = key[i];
            v2[pos] = val[i];
        }
        memcpy(key, k2, sizeof(unsigned) * (size_t)n);
        memcpy(val, v2, sizeof(int) * (size_t)n);
    }
    free(k2);
    free(v2);
}
static void radix_sort_u64(int n, uint64_t *key, int *val) {
    uint64_t *k2 = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    int *v2 = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int shift = 0; shift < 64; shift += 8) {
        int64_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (int i = 0; i < n; i++) cnt[((key[i] >> shift) & 255) + 1]++;
        for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
        for (int i = 0; i < n; i++) {
            int64_t pos = cnt[(key[i] >> shift) & 255]++;
            k2[pos] = key[i];
            v2[pos] = val[i];
        }
        memcpy(key, k2, sizeof(uint64_t) * (size_t)n);
        memcpy(val, v2, sizeof(int) * (size_t)n);
    }
    free(k2);
    free(v2);
}

static inline int split_metric(unsigned a, unsigned b) {
    unsigned x = a ^ b;
    return x ? 32 - __builtin_clz(x) : 0; /* 32 - __clz(x), __clz(0) = 32 */
}

/* ------------------------------------------------------------------ */
/* pipeline state                                                      */
struct orc_pipe {
    int restr_enabled, cull, narrow_enabled;
    int ref_perm;             /* restructure permutes as the reference does (test pinning) */
    int T, V, cap;            /* T prims, capacity of per-node arrays */
    const int *faces;         /* borrowed for the frame */
    const float *verts;
    /* leaves in Morton order (BvhPrimitiveNode + BvhExtNode) */
    obox *lbox;
    int *lidx, *lvid, *lpar, *lmark, *lca, *primmap, *metric;
    unsigned *code;
    /* internal nodes in DFS order (BvhIntNode) */
    int *lc, *rc, *par, *rx, *ry;
    unsigned *mark;
    obox *ibox;
    obox scene;
    /* scratch for builds */
    int *ulc, *urc, *upar, *urx, *ury, *ulca, *uflag, *ulpar, *tkmap, *seq, *vals;
    unsigned *umark, *depth, *offs;
    obox *ubox;
    /* restructure log (BvhRestrLog) */
    int *intrange, *rtroot, *intmark, *extrange, *extmark, *leafroot, *prevlbd, *gathermap;
    int updated, opt_tag, num_rt_subtree, num_rt_int;
    /* front log (FlOrderLog) */
    unsigned *intcnt, *extcnt, *intbeg, *extbeg, *intback, *extback;
    int log_stale;            /* counts split by a balance; begins still hold */
    float *snapshot;
    /* fronts (current) and pairs */
    pvec intf, extf, pairs, hits;
    int last_front_op, narrow_ran, built;
};

static void *xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

static void pipe_alloc(orc_pipe *p, int T) {
    if (p->lbox && T + 2 <= p->cap) return;
    int c = T + 2;
#define RE(ptr, type, n) ptr = (type *)realloc(ptr, sizeof(type) * (size_t)(n))
    RE(p->lbox, obox, c); RE(p->lidx, int, c); RE(p->lvid, int, 3 * c); RE(p->lpar, int, c);
    RE(p->lmark, int, c); RE(p->lca, int, c + 1); RE(p->primmap, int, c); RE(p->metric, int, c);
    RE(p->code, unsigned, c);
    RE(p->lc, int, c); RE(p->rc, int, c); RE(p->par, int, c); RE(p->rx, int, c); RE(p->ry, int, c);
    RE(p->mark, unsigned, c); RE(p->ibox, obox, c);
    RE(p->ulc, int, c); RE(p->urc, int, c); RE(p->upar, int, c); RE(p->urx, int, c);
    RE(p->ury, int, c); RE(p->ulca, int, c); RE(p->uflag, int, c); RE(p->ulpar, int, c);
    RE(p->tkmap, int, c); RE(p->seq, int, c); RE(p->vals, int, c);
    RE(p->umark, unsigned, c); RE(p->depth, unsigned, c + 1); RE(p->offs, unsigned, c + 1);
    RE(p->ubox, obox, c);
    RE(p->intrange, int, c); RE(p->rtroot, int, c); RE(p->intmark, int, c);
    RE(p->extrange, int, c + 1); RE(p->extmark, int, c + 1); RE(p->leafroot, int, c + 1);
    RE(p->prevlbd, int, c); RE(p->gathermap, int, c + 1);
    RE(p->intcnt, unsigned, c + 1); RE(p->extcnt, unsigned, c + 1); RE(p->intbeg, unsigned, c + 1);
    RE(p->extbeg, unsigned, c + 1); RE(p->intback, unsigned, c + 1); RE(p->extback, unsigned, c + 1);
    RE(p->snapshot, float, c);
#undef RE
    memset(p->umark, 0, sizeof(unsigned) * (size_t)c);
    memset(p->uflag, 0, sizeof(int) * (size_t)c);
    memset(p->intcnt, 0, sizeof(unsigned) * (size_t)(c + 1));
    memset(p->extcnt, 0, sizeof(unsigned) * (size_t)(c + 1));
    memset(p->intbeg, 0, sizeof(unsigned) * (size_t)(c + 1));
    memset(p->extbeg, 0, sizeof(unsigned) * (size_t)(c + 1));
    memset(p->intback, 0, sizeof(unsigned) * (size_t)(c + 1));
    memset(p->extback, 0, sizeof(unsigned) * (size_t)(c + 1));
    memset(p->snapshot, 0, sizeof(float) * (size_t)c);
    p->cap = c;
}

orc_pipe *orc_pipe_create(int restr_enabled, int cull_adjacent, int narrow_enabled) {
    orc_pipe *p = (orc_pipe *)xcalloc(1, sizeof(orc_pipe));
    p->restr_enabled = restr_enabled;
    p->cull = cull_adjacent;
    p->narrow_enabled = narrow_enabled;
    p->last_front_op = -1;
    return p;
}

void orc_pipe_destroy(orc_pipe *p) {
    if (!p) return;
    void *ptrs[] = {p->lbox, p->lidx, p->lvid, p->lpar, p->lmark, p->lca, p->primmap, p->metric,
                    p->code, p->lc, p->rc, p->par, p->rx, p->ry, p->mark, p->ibox, p->ulc,
                    p->urc, p->upar, p->urx, p->ury, p->ulca, p->uflag, p->ulpar, p->tkmap,
                    p->seq, p->vals, p->umark, p->depth, p->offs, p->ubox, p->intrange,
                    p->rtroot, p->intmark, p->extrange, p->extmark, p->leafroot, p->prevlbd,
                    p->gathermap, p->intcnt, p->extcnt, p->intbeg, p->extbeg, p->intback,
                    p->extback, p->snapshot};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    pv_free(&p->intf); pv_free(&p->extf); pv_free(&p->pairs); pv_free(&p->hits);
    free(p);
}

/* ------------------------------------------------------------------ */
/* Bottom-up construction, shared by build and restructure.
 * buildIntNodes (LBvhBuildKernels.cu:135-172) and restrIntNodes
 * (LBvhRestructureKernels.cu:122-166): a node covering leaves (l, r]
 * becomes the right child of split l when metric[l] < metric[r], else the
 * left child of split r.  In a restructure the boundary of a subtree acts as
 * an infinitely dissimilar split (bdmark).  Nodes are indexed by split.
 * seg == NULL: whole tree.  Leaves are processed in increasing order; the
 * structure does not depend on the order (the atomic flag picks the second
 * arrival, which only decides who merges). */
static void climb_build(orc_pipe *p, const int *leaves, int nleaves, const int *seg) {
    const int T = p->T;
    for (int k = 0; k < nleaves; k++) {
        int idx = leaves ? leaves[k] : k;
        p->ulca[idx] = -1;
        p->depth[idx] = 0;
    }
    for (int k = 0; k < nleaves; k++) {
        int idx = leaves ? leaves[k] : k;
        int sub = seg ? seg[idx] : 0;
        int l = idx - 1, r = idx, mark, bd = 0;
        if (seg) bd = ((l < 0 || seg[l] != sub) << 1) | (r == T - 1 || seg[r + 1] != sub);
        if (bd) mark = bd & 1;
        else mark = (l >= 0) ? (p->metric[l] < p->metric[r]) : 0;
        if (!seg && l < 0) mark = 0;
        int cur = mark ? l : r;
        p->ulpar[idx] = cur;
        if (mark) { p->urc[cur] = idx; p->ury[cur] = idx; p->umark[cur] |= 2u; p->lmark[idx] = 7; }
        else      { p->ulc[cur] = idx; p->urx[cur] = idx; p->umark[cur] |= 1u; p->lmark[idx] = 3; }
        while (p->uflag[cur]++ == 1) {
            /* BvhIntNodeCompletePort::refit(i, lvs) (BvhIntNode.h:59-74) */
            unsigned m = p->umark[cur];
            const obox *a = (m & 1u) ? &p->lbox[p->ulc[cur]] : &p->ubox[p->ulc[cur]];
            const obox *b = (m & 2u) ? &p->lbox[p->urc[cur]] : &p->ubox[p->urc[cur]];
            box_merge(&p->ubox[cur], a, b);
            p->umark[cur] &= 7u;
            l = p->urx[cur] - 1;
            r = p->ury[cur];
            p->ulca[l + 1] = cur;
            p->depth[l + 1]++;
            if (seg) bd = ((l < 0 || seg[l] != sub) << 1) | (r == T - 1 || seg[r + 1] != sub);
            if (bd) mark = bd & 1;
            else mark = (l >= 0) ? (p->metric[l] < p->metric[r]) : 0;
            int is_root = seg ? (bd == 3) : (l + 1 == 0 && r == T - 1);
            if (is_root) {
                p->upar[cur] = -1;
                if (!seg) p->umark[cur] &= ~4u;
                else if (p->mark[sub] & 4u) p->umark[cur] |= 4u;   /* keep relation with father */
                else p->umark[cur] &= ~4u;
                break;
            }
            int pr = mark ? l : r;
            p->upar[cur] = pr;
            if (mark) { p->urc[pr] = cur; p->ury[pr] = r; p->umark[pr] &= ~2u; p->umark[cur] |= 4u; }
            else      { p->ulc[pr] = cur; p->urx[pr] = l + 1; p->umark[pr] &= ~1u; p->umark[cur] &= ~4u; }
            cur = pr;
        }
    }
}

/* refit: refitExtNode (LBvhUpdateKernels.cu:35-61) then refitIntNode (:63-74).
 * Internal nodes are merged in decreasing DFS id (children follow parents in
 * DFS pre-order), which gives the same exact min/max as the atomic climb. */
static void orc_refit_leaves(orc_pipe *p) {
    const int T = p->T;
#pragma omp parallel for schedule(static)
    for (int t = 0; t < T; t++) {
        obox b;
        tri_box(&b, p->faces, p->verts, t);
        p->lbox[p->primmap[t]] = b;
    }
}
static void orc_refit_internal(orc_pipe *p) {
    for (int d = p->T - 2; d >= 0; d--) {
        unsigned m = p->mark[d];
        const obox *a = (m & 1u) ? &p->lbox[p->lc[d]] : &p->ibox[p->lc[d]];
        const obox *b = (m & 2u) ? &p->lbox[p->rc[d]] : &p->ibox[p->rc[d]];
        box_merge(&p->ibox[d], a, b);
    }
}

/* build (LBvhFixedDeformable.cu:121-178) */
static void orc_build(orc_pipe *p) {
    const int T = p->T;
    float s6[6];
    orc_scene_box(T, p->faces, p->verts, s6);
    memcpy(p->scene.mn, s6, 12);
    memcpy(p->scene.mx, s6 + 3, 12);
    unsigned *keys = (unsigned *)malloc(sizeof(unsigned) * (size_t)(T > 0 ? T : 1));
    orc_morton_codes(T, p->faces, p->verts, s6, keys);
    for (int i = 0; i < T; i++) p->vals[i] = i;
    radix_sort_u32(T, keys, p->vals);
    /* calcInverseMapping (CudaKernelUtils.cu:28-32) + buildPrimitives (LBvhBuildKernels.cu:114-133) */
    for (int i = 0; i < T; i++) {
        int t = p->vals[i];
        p->primmap[t] = i;
        p->code[i] = keys[i];
        p->lidx[i] = t;
        for (int k = 0; k < 3; k++) p->lvid[3 * i + k] = p->faces[3 * (size_t)t + k];
        tri_box(&p->lbox[i], p->faces, p->verts, t);
    }
    free(keys);
    /* calcExtNodeSplitMetrics (BvhExtNode.cu:128-134) */
    for (int i = 0; i < T; i++) p->metric[i] = (i != T - 1) ? split_metric(p->code[i], p->code[i + 1]) : 33;
    p->lca[T] = -1;
    if (T < 2) {
        if (T == 1) { p->lca[0] = 1; p->lpar[0] = -1; p->lmark[0] = 7; }
        p->built = 1;
        return;
    }
    memset(p->uflag, 0, sizeof(int) * (size_t)T);
    memset(p->umark, 0, sizeof(unsigned) * (size_t)T);
    climb_build(p, NULL, T, NULL);
    /* reorderIntNodes (LBvhFixedDeformable.cu:365-380): DFS pre-order ids
     * from prefix sums of left-chain lengths (calcIntNodeOrders :174-185) */
    unsigned run = 0;
    for (int i = 0; i < T; i++) { p->offs[i] = run; run += p->depth[i]; }
    for (int i = 0; i < T; i++) {
        int node = p->ulca[i];
        unsigned id = p->offs[i];
        if (node != -1)
            for (unsigned d = p->depth[i]; d--; node = p->ulc[node]) p->tkmap[node] = (int)id++;
    }
    /* updateBvhExtNodeLinks (:187-200) */
    for (int i = 0; i < T; i++) {
        p->lpar[i] = p->tkmap[p->ulpar[i]];
        p->lca[i] = (p->ulca[i] != -1) ? (p->tkmap[p->ulca[i]] << 1) : ((i << 1) | 1);
    }
    /* reorderIntNode (:202-217) */
    for (int k = 0; k < T - 1; k++) {
        int n = p->tkmap[k];
        unsigned m = p->umark[k];
        p->lc[n] = (m & 1u) ? p->ulc[k] : p->tkmap[p->ulc[k]];
        p->rc[n] = (m & 2u) ? p->urc[k] : p->tkmap[p->urc[k]];
        p->mark[n] = m;
        p->par[n] = p->upar[k] != -1 ? p->tkmap[p->upar[k]] : -1;
        p->rx[n] = p->urx[k];
        p->ry[n] = p->ury[k];
        p->ibox[n] = p->ubox[k];
    }
    p->built = 1;
}

/* restructure (LBvhFixedDeformable.cu:210-352, LBvhRestructureKernels.cu) */
static void orc_restructure(orc_pipe *p) {
    const int T = p->T, I = T - 1;
    /* 1: int node marks = inclusive scan of intrange */
    int run = 0;
    for (int i = 0; i < I; i++) { run += p->intrange[i]; p->intmark[i] = run; }
    /* 2-3: calibrateLeafRangeMarks (:9-17) + scan */
    memset(p->extrange, 0, sizeof(int) * (size_t)(T + 1));
    for (int i = 0; i < T; i++) {
        int rt = p->rtroot[i];
        if (rt != INT_MAX && p->intmark[rt] == 1) { p->extrange[i]++; p->extrange[p->ry[rt] + 1]--; }
    }
    run = 0;
    for (int i = 0; i <= T; i++) { run += p->extrange[i]; p->extmark[i] = run; }
    /* 4: calibrateRestrRoots (:19-35) */
    memset(p->extrange, 0, sizeof(int) * (size_t)(T + 1));
    p->num_rt_subtree = 0;
    p->num_rt_int = 0;
    for (int i = 0; i < T; i++) {
        int rt = p->rtroot[i];
        if (rt != INT_MAX && p->intmark[rt] == 1) {
            p->extrange[i] += rt;
            p->extrange[p->ry[rt] + 1] -= rt;
            p->num_rt_int += p->ry[rt] - p->rx[rt];
            p->num_rt_subtree++;
        }
    }
    if (p->num_rt_int > (I >> 1)) { orc_build(p); p->opt_tag = 2; return; }
    if (p->num_rt_int < (I >> 3)) {
        orc_refit_leaves(p);
        orc_refit_internal(p);
        p->opt_tag = 0;
        return;
    }
    for (int i = 0; i < I; i++) p->prevlbd[i] = p->rx[i];
    /* 5: per-leaf subtree root */
    run = 0;
    for (int i = 0; i <= T; i++) { run += p->extrange[i]; p->leafroot[i] = run; }
    /* 6-7: scene box, Morton codes of restructured primitives, (root, code)
     * keys, segmented sort (calcRestrMCs :37-55, selectPrimitives :57-66) */
    float s6[6];
    orc_scene_box(T, p->faces, p->verts, s6);
    memcpy(p->scene.mn, s6, 12);
    memcpy(p->scene.mx, s6 + 3, 12);
    int nr = 0;
    for (int i = 0; i < T; i++) if (p->leafroot[i] > 0) nr++;
    uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nr > 0 ? nr : 1));
    int *task = (int *)malloc(sizeof(int) * (size_t)(nr > 0 ? nr : 1));
    int *sorted = (int *)malloc(sizeof(int) * (size_t)(nr > 0 ? nr : 1));
    int *oldidx = (int *)malloc(sizeof(int) * (size_t)(nr > 0 ? nr : 1));
    int k = 0;
    for (int i = 0; i < T; i++) {
        if (p->leafroot[i] > 0) {
            obox b;
            tri_box(&b, p->faces, p->verts, p->lidx[i]);
            unsigned c = morton_of_box(&b, &p->scene);
            keys[k] = ((uint64_t)(unsigned)p->leafroot[i] << 32) | c;
            task[k] = i;
            sorted[k] = i;
            k++;
        }
    }
    radix_sort_u64(nr, keys, sorted);
    if (p->ref_perm) {
        /* 8-9 as the reference runs them under one sequential schedule
         * (thread index order): updatePrimMap (:68-77) moves the triangle of
         * slot task[k] to slot sorted[k] -- the inverse of the sort
         * permutation -- reading the slot->triangle map while it writes it,
         * so a slot written by an earlier thread is read back already
         * overwritten and the map stops being a permutation;
         * updatePrimAndExtNode (:79-120) then writes each triangle's box, and
         * for restructured slots its vertex ids and Morton code, to
         * primmap[t] (last writer wins, unwritten slots keep their old
         * values), and refitIntNode refits the old topology. */
        for (k = 0; k < nr; k++) {
            int val = p->lidx[task[k]];
            p->primmap[val] = sorted[k];
            p->lidx[sorted[k]] = val;
        }
        for (int t = 0; t < T; t++) {
            int pid = p->primmap[t];
            tri_box(&p->lbox[pid], p->faces, p->verts, t);
            if (p->extmark[pid]) {
                for (int j = 0; j < 3; j++) p->lvid[3 * pid + j] = p->faces[3 * (size_t)t + j];
                p->code[pid] = morton_of_box(&p->lbox[pid], &p->scene);
            }
        }
        free(keys); free(sorted); free(oldidx);
        orc_refit_internal(p);
    } else {
        /* 8: permutation inside each subtree: slot task[k] receives the
         * triangle that sorts k-th (the reference's updatePrimMap :68-77
         * applies the inverse permutation; see the file header). */
        for (k = 0; k < nr; k++) oldidx[k] = p->lidx[sorted[k]];
        for (k = 0; k < nr; k++) {
            int slot = task[k], t = oldidx[k];
            p->lidx[slot] = t;
            p->primmap[t] = slot;
            for (int j = 0; j < 3; j++) p->lvid[3 * slot + j] = p->faces[3 * (size_t)t + j];
            p->code[slot] = (unsigned)(keys[k] & 0xffffffffu);
        }
        free(keys); free(sorted); free(oldidx);
        /* 9: boxes of every primitive, then refit with the old topology
         * (updatePrimAndExtNode :79-120, refitIntNode) */
        orc_refit_leaves(p);
        orc_refit_internal(p);
    }
    /* 10: split metrics and confined rebuild (restrIntNodes :122-166) */
    for (int i = 0; i < T; i++) p->metric[i] = (i != T - 1) ? split_metric(p->code[i], p->code[i + 1]) : 33;
    memset(p->depth, 0, sizeof(unsigned) * (size_t)(T + 1));
    memset(p->uflag, 0, sizeof(int) * (size_t)T);
    climb_build(p, task, nr, p->leafroot);
    /* calcRestrIntNodeOrders (:168-195): DFS ids inside each subtree slot */
    unsigned acc = 0;
    for (int i = 0; i <= T; i++) { p->offs[i] = acc; acc += p->depth[i]; }
    int nseq = 0;
    for (k = 0; k < nr; k++) {
        int idx = task[k];
        int node = p->ulca[idx];
        if (node != -1) {
            int root = p->leafroot[idx];
            int newid = root + (int)p->offs[idx] - (int)p->offs[p->prevlbd[root]];
            if ((p->mark[root] & 4u) || idx != p->prevlbd[root]) p->lca[idx] = newid << 1;
            for (unsigned d = p->depth[idx]; d--; node = p->ulc[node]) {
                if (p->umark[node] & 2u) p->lpar[p->urc[node]] = newid;
                p->tkmap[node] = newid++;
                p->seq[nseq++] = node;
            }
            p->lpar[idx] = newid - 1;
        } else {
            p->lca[idx] = (idx << 1) | 1;
        }
    }
    /* reorderRestrIntNodes (:197-215) */
    for (int q = 0; q < nseq; q++) {
        int u = p->seq[q], n = p->tkmap[u];
        unsigned m = p->umark[u];
        p->mark[n] = m;
        p->lc[n] = (m & 1u) ? p->ulc[u] : p->tkmap[p->ulc[u]];
        p->rc[n] = (m & 2u) ? p->urc[u] : p->tkmap[p->urc[u]];
        if (p->upar[u] != -1) p->par[n] = p->tkmap[p->upar[u]];
        p->rx[n] = p->urx[u];
        p->ry[n] = p->ury[u];
        p->ibox[n] = p->ubox[u];
    }
    free(task);
    p->opt_tag = 1;
}

/* LBvhFixedDeformable::maintain (LBvhFixedDeformable.cu:68-87) */
static void orc_bvh_maintain(orc_pipe *p, int op) {
    p->opt_tag = 0;
    if (p->restr_enabled && p->updated && p->built && p->T >= 2) {
        orc_restructure(p);
        return;
    }
    if (op == ORC_BVH_BUILD || !p->built) {
        orc_build(p);
    } else { /* REFIT; UPDATE = refit (the reference marks it deprecated, LBvhUpdateKernels.cu:88) */
        orc_refit_leaves(p);
        if (p->T >= 2) orc_refit_internal(p);
    }
}

/* ------------------------------------------------------------------ */
/* front log helpers (FlOrderLog.cu:7-12, FlOrderLog.cpp clear)        */
static void log_clear(orc_pipe *p) {
    size_t n = (size_t)p->T + 1;
    memset(p->intcnt, 0, sizeof(unsigned) * n);
    memset(p->extcnt, 0, sizeof(unsigned) * n);
    memset(p->intback, 0, sizeof(unsigned) * n);
    memset(p->extback, 0, sizeof(unsigned) * n);
}
static void log_prepare(orc_pipe *p) {
    unsigned a = 0;
    for (int i = 0; i < p->T; i++) { p->intbeg[i] = a; a += p->intcnt[i]; }
    p->intbeg[p->T] = a;
    a = 0;
    for (int i = 0; i <= p->T; i++) { p->extbeg[i] = a; a += p->extcnt[i]; }
}

static emitbuf *emit_alloc(void) {
    int nt = orc_threads();
    if (nt > ORC_MAX_THREADS) nt = ORC_MAX_THREADS;
    return (emitbuf *)xcalloc((size_t)nt, sizeof(emitbuf));
}
static void emit_merge(emitbuf *eb, pvec *intf, pvec *extf, pvec *pairs) {
    int nt = orc_threads();
    if (nt > ORC_MAX_THREADS) nt = ORC_MAX_THREADS;
    for (int t = 0; t < nt; t++) {
        if (intf) { pv_reserve(intf, intf->n + eb[t].intf.n);
            memcpy(intf->d + 2 * intf->n, eb[t].intf.d, sizeof(int) * 2 * (size_t)eb[t].intf.n);
            intf->n += eb[t].intf.n; }
        if (extf) { pv_reserve(extf, extf->n + eb[t].extf.n);
            memcpy(extf->d + 2 * extf->n, eb[t].extf.d, sizeof(int) * 2 * (size_t)eb[t].extf.n);
            extf->n += eb[t].extf.n; }
        if (pairs) { pv_reserve(pairs, pairs->n + eb[t].pairs.n);
            memcpy(pairs->d + 2 * pairs->n, eb[t].pairs.d, sizeof(int) * 2 * (size_t)eb[t].pairs.n);
            pairs->n += eb[t].pairs.n; }
        pv_free(&eb[t].intf); pv_free(&eb[t].extf); pv_free(&eb[t].pairs);
    }
    free(eb);
}

#define ATOMIC_INC(x) __atomic_fetch_add(&(x), 1u, __ATOMIC_RELAXED)

static inline void emit_pair(orc_pipe *p, emitbuf *e, int i, int j) {
    if (p->cull && covertex(p->lvid + 3 * i, p->lvid + 3 * j)) return;
    pv_push(&e->pairs, p->lidx[i], p->lidx[j]);
}

/* Stackless DFS over the DFS-ordered tree starting at tagged node `st`
 * until tagged node `stop`.  The left spine below an internal node is
 * walked by incrementing the DFS id up to the parent of the leftmost leaf
 * (lpar); a node that stops overlapping is left through the escape link
 * lca[rangey + 1].  mode bit0: emit front entries + counts, bit1: emit pairs.
 * This is the loop body shared by genLooseIntraFrontsWithLog
 * (BvttFrontGenerateKernels.cu:51-90), the sprout half of
 * maintainIntLooseIntraFrontsWithLog (BvttFrontPruneSproutKernels.cu:32-56),
 * keepIntLooseIntraFronts (BvttFrontKeepKernels.cu:21-42), the overlap half
 * of reorderIntLooseIntraFrontsWithLog (BvttFrontReorderKernels.cu:43-62)
 * and pureBvhSelfCD (BvhCDKernels.cu:17-49). */
static void traverse(orc_pipe *p, emitbuf *e, int prim, int st, int stop, int front) {
    const obox *bv = &p->lbox[prim];
    do {
        int t = st & 1, lbd;
        st >>= 1;
        if (!t) {
            for (t = p->lpar[lbd = p->rx[st]]; st <= t && box_overlap(&p->ibox[st], bv); st++)
                ;
        } else {
            t = st - 1;
            lbd = st;
        }
        if (st == t + 1) {
            if (box_overlap(&p->lbox[lbd], bv)) emit_pair(p, e, prim, lbd);
            if (front) { pv_push(&e->extf, prim, lbd); ATOMIC_INC(p->extcnt[lbd]); }
            st = p->lca[lbd + 1];
        } else {
            if (front) { pv_push(&e->intf, prim, st); ATOMIC_INC(p->intcnt[st]); }
            st = p->lca[p->ry[st] + 1];
        }
    } while (st != stop);
}

/* reorderFronts (BvttFrontLooseIntra.cu:140-170): counting sort by node */
static void orc_reorder_fronts(orc_pipe *p) {
    log_prepare(p);
    log_clear(p);
    pvec ni = {0}, ne = {0};
    pv_reserve(&ni, p->intf.n);
    pv_reserve(&ne, p->extf.n);
    ni.n = p->intf.n;
    ne.n = p->extf.n;
    /* pureReorderLooseFrontsWithLog (BvttFrontReorderKernels.cu:12-24),
     * sequential so the order inside a bucket is deterministic here */
    for (int64_t q = 0; q < p->intf.n; q++) {
        int a = p->intf.d[2 * q], n = p->intf.d[2 * q + 1];
        unsigned pos = p->intbeg[n] + p->intcnt[n]++;
        ni.d[2 * pos] = a; ni.d[2 * pos + 1] = n;
    }
    for (int64_t q = 0; q < p->extf.n; q++) {
        int a = p->extf.d[2 * q], n = p->extf.d[2 * q + 1];
        unsigned pos = p->extbeg[n] + p->extcnt[n]++;
        ne.d[2 * pos] = a; ne.d[2 * pos + 1] = n;
    }
    pv_free(&p->intf); pv_free(&p->extf);
    p->intf = ni;
    p->extf = ne;
    p->log_stale = 0;
}

/* frontSnapshot (BvttFrontGenerateKernels.cu:26-32) */
static void orc_snapshot(orc_pipe *p) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < p->T - 1; i++) {
        int x = p->rx[i], y = p->ry[i];
        unsigned ic = p->intbeg[i + y - x] - p->intbeg[i];
        unsigned ec = p->extbeg[y + 1] - p->extbeg[x] + 1u;
        p->snapshot[i] = (float)(1.0 * ic / ec);
    }
}

/* checkQuality + checkFrontQuality (BvttFrontLooseIntra.cu:219-228,
 * BvttFrontGenerateKernels.cu:34-49) */
static void orc_check_quality(orc_pipe *p) {
    const int T = p->T;
    for (int i = 0; i < T; i++) p->rtroot[i] = INT_MAX; /* BvhRestrLog::clear */
    memset(p->intrange, 0, sizeof(int) * (size_t)T);
    unsigned total = p->intbeg[T - 1];
    for (int i = 0; i < T - 1; i++) {
        int x = p->rx[i], y = p->ry[i];
        int ic = (int)(p->intbeg[i + y - x] - p->intbeg[i]);
        int ec = (int)(p->extbeg[y + 1] - p->extbeg[x]);
        double lhs = 1.0 * ic / ec;
        double rhs = (double)p->snapshot[i] + 1 - 0.7 * ic / total;
        if (lhs > rhs) {
            p->intrange[i] += 1;
            p->intrange[i + y - x] -= 1;
            if (i < p->rtroot[x]) p->rtroot[x] = i;
        }
    }
    p->updated = 1;
}

static void orc_generate(orc_pipe *p) {
    log_clear(p);
    p->intf.n = p->extf.n = p->pairs.n = 0;
    emitbuf *eb = emit_alloc();
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < p->T - 1; i++)
        traverse(p, &eb[orc_tid()], i, p->lca[i + 1], -1, 1);
    emit_merge(eb, &p->intf, &p->extf, &p->pairs);
    orc_reorder_fronts(p);
    if (p->restr_enabled) orc_snapshot(p);
}

static void orc_pure_bvh(orc_pipe *p) {
    p->pairs.n = 0;
    emitbuf *eb = emit_alloc();
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < p->T - 1; i++)
        traverse(p, &eb[orc_tid()], i, p->lca[i + 1], -1, 0);
    emit_merge(eb, NULL, NULL, &p->pairs);
}

/* pruneSprout (BvttFrontLooseIntra.cu:254-283) with
 * maintainIntLooseIntraFrontsWithLog / maintainExtLooseIntraFrontsWithLog
 * (BvttFrontPruneSproutKernels.cu:12-93) */
static void orc_prune_sprout(orc_pipe *p) {
    log_clear(p);
    p->pairs.n = 0;
    pvec oi = p->intf, oe = p->extf;
    memset(&p->intf, 0, sizeof(pvec));
    memset(&p->extf, 0, sizeof(pvec));
    emitbuf *eb = emit_alloc();
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t q = 0; q < oi.n; q++) {
        emitbuf *e = &eb[orc_tid()];
        int prim = oi.d[2 * q], st = oi.d[2 * q + 1];
        const obox *bv = &p->lbox[prim];
        if (!box_overlap(&p->ibox[st], bv)) { /* prune */
            int t = p->lca[p->rx[st]] >> 1;
            for (st--; st >= t && !box_overlap(&p->ibox[st], bv); st--)
                ;
            if (st < t && (st + 1 > 0 && !box_overlap(&p->ibox[p->par[st + 1]], bv))) continue;
            pv_push(&e->intf, prim, st + 1);
            ATOMIC_INC(p->intcnt[st + 1]);
            continue;
        }
        int stop = p->lca[p->ry[st] + 1]; /* sprout */
        int start = (p->lc[st] << 1) | (int)(p->mark[st] & 1u);
        traverse(p, e, prim, start, stop, 1);
    }
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t q = 0; q < oe.n; q++) {
        emitbuf *e = &eb[orc_tid()];
        int prim = oe.d[2 * q], st = oe.d[2 * q + 1];
        const obox *bv = &p->lbox[prim];
        if (!box_overlap(&p->lbox[st], bv)) {
            int gfa = p->lpar[st];
            if (box_overlap(&p->ibox[gfa], bv)) {
                pv_push(&e->extf, prim, st);
                ATOMIC_INC(p->extcnt[st]);
                continue;
            }
            if ((p->lmark[st] & 4) == 4) continue;
            int leaf = st;
            for (st = gfa - 1, gfa = p->lca[leaf] >> 1; st >= gfa && !box_overlap(&p->ibox[st], bv); st--)
                ;
            if (st < gfa && (st + 1 > 0 && !box_overlap(&p->ibox[p->par[st + 1]], bv))) continue;
            pv_push(&e->intf, prim, st + 1);
            ATOMIC_INC(p->intcnt[st + 1]);
        } else {
            pv_push(&e->extf, prim, st);
            ATOMIC_INC(p->extcnt[st]);
            emit_pair(p, e, prim, st);
        }
    }
    emit_merge(eb, &p->intf, &p->extf, &p->pairs);
    pv_free(&oi);
    pv_free(&oe);
    if (p->restr_enabled) orc_check_quality(p);
    orc_reorder_fronts(p);
}

/* keep (BvttFrontLooseIntra.cu:314-328): keepInt/ExtLooseIntraFronts */
static void orc_keep(orc_pipe *p) {
    p->pairs.n = 0;
    emitbuf *eb = emit_alloc();
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t q = 0; q < p->intf.n; q++) {
        int prim = p->intf.d[2 * q], st = p->intf.d[2 * q + 1];
        if (!box_overlap(&p->ibox[st], &p->lbox[prim])) continue;
        int stop = p->lca[p->ry[st] + 1];
        int start = (p->lc[st] << 1) | (int)(p->mark[st] & 1u);
        if (start != stop) traverse(p, &eb[orc_tid()], prim, start, stop, 0);
    }
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < p->extf.n; q++) {
        int prim = p->extf.d[2 * q], st = p->extf.d[2 * q + 1];
        if (box_overlap(&p->lbox[prim], &p->lbox[st])) emit_pair(p, &eb[orc_tid()], prim, st);
    }
    emit_merge(eb, NULL, NULL, &p->pairs);
}

/* balance (BvttFrontLooseIntra.cu:285-312) with
 * reorderIntLooseIntraFrontsWithLog (BvttFrontReorderKernels.cu:27-63):
 * non-overlapping entries fill each node bucket from the front, overlapping
 * ones from the back and are traversed; the external front is kept. */
static void orc_balance(orc_pipe *p) {
    /* A balance splits each node's count into front and back halves and
     * clears the external counts without moving an entry to another node,
     * so the begins it started from still hold for a following balance
     * (the reference rescans the split counts there, :286, and overlaps
     * entries; its schedules never run two balances in a row). */
    if (!p->log_stale) log_prepare(p);
    log_clear(p);
    p->log_stale = 1;
    p->pairs.n = 0;
    pvec ni = {0};
    pv_reserve(&ni, p->intf.n);
    ni.n = p->intf.n;
    for (int64_t q = 0; q < p->intf.n; q++) {
        int prim = p->intf.d[2 * q], st = p->intf.d[2 * q + 1];
        unsigned pos;
        if (!box_overlap(&p->ibox[st], &p->lbox[prim])) pos = p->intbeg[st] + p->intcnt[st]++;
        else pos = p->intbeg[st + 1] - 1 - p->intback[st]++;
        ni.d[2 * pos] = prim;
        ni.d[2 * pos + 1] = st;
    }
    emitbuf *eb = emit_alloc();
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t q = 0; q < p->intf.n; q++) {
        int prim = p->intf.d[2 * q], st = p->intf.d[2 * q + 1];
        if (!box_overlap(&p->ibox[st], &p->lbox[prim])) continue;
        int stop = p->lca[p->ry[st] + 1];
        int start = (p->lc[st] << 1) | (int)(p->mark[st] & 1u);
        if (start != stop) traverse(p, &eb[orc_tid()], prim, start, stop, 0);
    }
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < p->extf.n; q++) {
        int prim = p->extf.d[2 * q], st = p->extf.d[2 * q + 1];
        if (box_overlap(&p->lbox[prim], &p->lbox[st])) emit_pair(p, &eb[orc_tid()], prim, st);
    }
    emit_merge(eb, NULL, NULL, &p->pairs);
    pv_free(&p->intf);
    p->intf = ni;
}

/* ------------------------------------------------------------------ */
/* FP32 17-axis SAT: the tri-tri test of Gottschalk's separating-axis
 * method as gProximity's triangleIntersection2 applies it
 * (Source/Externals/inc/gProximity/cuda_intersect_tritri.h:247-266,349-433):
 * translate by P1, edges e/f, normals n/m, 9 edge-edge axes, 6 in-plane edge
 * normals; an axis separates when the projected intervals are strictly
 * disjoint.  Evaluated without contraction (compile with -ffp-contract=off). */
typedef struct { float x, y, z; } f3;
static inline f3 f3sub(f3 a, f3 b) { f3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline f3 f3cross(f3 a, f3 b) {
    f3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline float f3dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline int axis_overlap(f3 ax, f3 p1, f3 p2, f3 p3, f3 q1, f3 q2, f3 q3) {
    float P1 = f3dot(ax, p1), P2 = f3dot(ax, p2), P3 = f3dot(ax, p3);
    float Q1 = f3dot(ax, q1), Q2 = f3dot(ax, q2), Q3 = f3dot(ax, q3);
    float mx1 = fmaxf(fmaxf(P1, P2), P3), mn1 = fminf(fminf(P1, P2), P3);
    float mx2 = fmaxf(fmaxf(Q1, Q2), Q3), mn2 = fminf(fminf(Q1, Q2), Q3);
    if (mn1 > mx2) return 0;
    if (mn2 > mx1) return 0;
    return 1;
}
int orc_tritri_sat32(const float *P, const float *Q) {
    f3 P1 = {P[0], P[1], P[2]}, P2 = {P[3], P[4], P[5]}, P3 = {P[6], P[7], P[8]};
    f3 Q1 = {Q[0], Q[1], Q[2]}, Q2 = {Q[3], Q[4], Q[5]}, Q3 = {Q[6], Q[7], Q[8]};
    f3 p1 = {0.f, 0.f, 0.f};
    f3 p2 = f3sub(P2, P1), p3 = f3sub(P3, P1);
    f3 q1 = f3sub(Q1, P1), q2 = f3sub(Q2, P1), q3 = f3sub(Q3, P1);
    f3 e[3] = {f3sub(p2, p1), f3sub(p3, p2), f3sub(p1, p3)};
    f3 f[3] = {f3sub(q2, q1), f3sub(q3, q2), f3sub(q1, q3)};
    f3 n = f3cross(e[0], e[1]), m = f3cross(f[0], f[1]);
    if (!axis_overlap(n, p1, p2, p3, q1, q2, q3)) return 0;
    if (!axis_overlap(m, p1, p2, p3, q1, q2, q3)) return 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (!axis_overlap(f3cross(e[i], f[j]), p1, p2, p3, q1, q2, q3)) return 0;
    for (int i = 0; i < 3; i++)
        if (!axis_overlap(f3cross(e[i], n), p1, p2, p3, q1, q2, q3)) return 0;
    for (int j = 0; j < 3; j++)
        if (!axis_overlap(f3cross(f[j], m), p1, p2, p3, q1, q2, q3)) return 0;
    return 1;
}

static void load_tri(const int *faces, const float *verts, int t, float *o9) {
    for (int k = 0; k < 3; k++) memcpy(o9 + 3 * k, verts + 3 * (size_t)faces[3 * (size_t)t + k], 12);
}

void orc_narrow_sat32(int64_t n, const int *pairs, const int *faces, const float *verts,
                      unsigned char *hit) {
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; q++) {
        float a[9], b[9];
        load_tri(faces, verts, pairs[2 * q], a);
        load_tri(faces, verts, pairs[2 * q + 1], b);
        hit[q] = (unsigned char)orc_tritri_sat32(a, b);
    }
}
void orc_narrow_exact(int64_t n, const int *pairs, const int *faces, const float *verts,
                      unsigned char *hit) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t q = 0; q < n; q++) {
        float a[9], b[9];
        load_tri(faces, verts, pairs[2 * q], a);
        load_tri(faces, verts, pairs[2 * q + 1], b);
        hit[q] = (unsigned char)orc_tritri_exact(a, b);
    }
}

/* proximityQuery / simpleNarrowPhase (BvttFrontLooseIntra.cu:128-138,
 * narrow_phase.cu:8-24): keep the pairs whose triangles intersect */
static void orc_narrow(orc_pipe *p) {
    p->hits.n = 0;
    int64_t n = p->pairs.n;
    unsigned char *h = (unsigned char *)xcalloc((size_t)n, 1);
    orc_narrow_sat32(n, p->pairs.d, p->faces, p->verts, h);
    pv_reserve(&p->hits, n);
    for (int64_t q = 0; q < n; q++)
        if (h[q]) pv_push(&p->hits, p->pairs.d[2 * q], p->pairs.d[2 * q + 1]);
    free(h);
}

/* BvttFrontLooseIntra::maintain (BvttFrontLooseIntra.cu:69-126) */
static void orc_front_maintain(orc_pipe *p, int op) {
    p->updated = 0;
    int run = op;
    if (p->restr_enabled && (p->opt_tag == 2 || p->opt_tag == 1)) run = ORC_FRONT_GENERATE;
    if (p->T < 2) {
        p->intf.n = p->extf.n = p->pairs.n = 0;
        run = op;
    } else {
        switch (run) {
        case ORC_FRONT_PURE_BVH_CD: orc_pure_bvh(p); break;
        case ORC_FRONT_GENERATE: orc_generate(p); break;
        case ORC_FRONT_UPDATE: orc_prune_sprout(p); break;
        case ORC_FRONT_REORDER: orc_balance(p); break;
        case ORC_FRONT_KEEP: orc_keep(p); break;
        default: orc_generate(p); run = ORC_FRONT_GENERATE; break;
        }
    }
    p->last_front_op = run;
    p->narrow_ran = 0;
    if (p->narrow_enabled) { orc_narrow(p); p->narrow_ran = 1; }
}

int orc_pipe_frame(orc_pipe *p, int T, const int *faces, int V, const float *verts, int bvh_op,
                   int front_op) {
    if (!p || T < 0 || V < 0) return -1;
    if (p->built && T != p->T) { p->built = 0; p->updated = 0; }
    pipe_alloc(p, T);
    p->T = T;
    p->V = V;
    p->faces = faces;
    p->verts = verts;
    orc_bvh_maintain(p, bvh_op);
    orc_front_maintain(p, front_op);
    return 0;
}

/* Marks subtrees (DFS roots) as degraded exactly as checkFrontQuality does
 * (BvttFrontGenerateKernels.cu:45-47); the next BVH maintain restructures. */
void orc_pipe_set_reference_permutation(orc_pipe *p, int on) { p->ref_perm = on; }

void orc_pipe_mark_restructure(orc_pipe *p, const int *roots, int n) {
    const int T = p->T;
    if (T < 2) return;
    if (!p->updated) {
        for (int i = 0; i < T; i++) p->rtroot[i] = INT_MAX;
        memset(p->intrange, 0, sizeof(int) * (size_t)T);
    }
    for (int k = 0; k < n; k++) {
        int i = roots[k];
        if (i < 0 || i >= T - 1) continue;
        int x = p->rx[i], y = p->ry[i];
        p->intrange[i] += 1;
        p->intrange[i + y - x] -= 1;
        if (i < p->rtroot[x]) p->rtroot[x] = i;
    }
    p->updated = 1;
}

void orc_pipe_info(const orc_pipe *p, int64_t *info) {
    memset(info, 0, sizeof(int64_t) * 16);
    info[0] = p->T; info[1] = p->intf.n; info[2] = p->extf.n; info[3] = p->pairs.n;
    info[4] = p->hits.n; info[5] = p->opt_tag; info[6] = p->updated;
    info[7] = p->num_rt_subtree; info[8] = p->num_rt_int; info[9] = p->last_front_op;
    info[10] = p->narrow_ran;
}

int64_t orc_pipe_pairs(const orc_pipe *p, int which, int *out, int64_t cap) {
    const pvec *v = which ? &p->hits : &p->pairs;
    int64_t n = v->n < cap ? v->n : cap;
    if (out && n > 0) memcpy(out, v->d, sizeof(int) * 2 * (size_t)n);
    return v->n;
}
int64_t orc_pipe_front(const orc_pipe *p, int which, int *out, int64_t cap) {
    const pvec *v = which ? &p->extf : &p->intf;
    int64_t n = v->n < cap ? v->n : cap;
    if (out && n > 0) memcpy(out, v->d, sizeof(int) * 2 * (size_t)n);
    return v->n;
}

int orc_pipe_tree(const orc_pipe *p, int *inode, float *ibox, int *leaf, float *lbox,
                  int *leaf_lca, unsigned *codes, int *primmap) {
    const int T = p->T;
    for (int i = 0; i < T - 1; i++) {
        if (inode) {
            inode[6 * i + 0] = p->lc[i]; inode[6 * i + 1] = p->rc[i]; inode[6 * i + 2] = p->par[i];
            inode[6 * i + 3] = (int)p->mark[i]; inode[6 * i + 4] = p->rx[i]; inode[6 * i + 5] = p->ry[i];
        }
        if (ibox) { memcpy(ibox + 6 * i, p->ibox[i].mn, 12); memcpy(ibox + 6 * i + 3, p->ibox[i].mx, 12); }
    }
    for (int i = 0; i < T; i++) {
        if (leaf) {
            leaf[4 * i + 0] = p->lidx[i]; leaf[4 * i + 1] = p->lpar[i];
            leaf[4 * i + 2] = p->lmark[i]; leaf[4 * i + 3] = p->lca[i];
        }
        if (lbox) { memcpy(lbox + 6 * i, p->lbox[i].mn, 12); memcpy(lbox + 6 * i + 3, p->lbox[i].mx, 12); }
        if (codes) codes[i] = p->code[i];
        if (primmap) primmap[i] = p->primmap[i];
    }
    if (leaf_lca) for (int i = 0; i <= T; i++) leaf_lca[i] = p->lca[i];
    return T;
}

int orc_pipe_log(const orc_pipe *p, unsigned *intcnt, unsigned *extcnt, unsigned *intbeg,
                 unsigned *extbeg) {
    size_t n = (size_t)p->T + 1;
    if (intcnt) memcpy(intcnt, p->intcnt, sizeof(unsigned) * n);
    if (extcnt) memcpy(extcnt, p->extcnt, sizeof(unsigned) * n);
    if (intbeg) memcpy(intbeg, p->intbeg, sizeof(unsigned) * n);
    if (extbeg) memcpy(extbeg, p->extbeg, sizeof(unsigned) * n);
    return p->T;
}

/* ------------------------------------------------------------------ */
/* Brute force: sweep and prune on min.x over FP32 triangle boxes.      */
typedef struct { float key; int id; } sap_item;
static int sap_cmp(const void *a, const void *b) {
    const sap_item *x = (const sap_item *)a, *y = (const sap_item *)b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return x->id - y->id;
}
int64_t orc_brute_pairs(int T, const int *faces, const float *verts, int cull, int *out,
                        int64_t cap) {
    obox *b = (obox *)malloc(sizeof(obox) * (size_t)(T > 0 ? T : 1));
    sap_item *it = (sap_item *)malloc(sizeof(sap_item) * (size_t)(T > 0 ? T : 1));
    for (int t = 0; t < T; t++) {
        tri_box(&b[t], faces, verts, t);
        it[t].key = b[t].mn[0];
        it[t].id = t;
    }
    qsort(it, (size_t)T, sizeof(sap_item), sap_cmp);
    int64_t total = 0;
    emitbuf *eb = emit_alloc();
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
    for (int a = 0; a < T; a++) {
        const obox *A = &b[it[a].id];
        for (int c = a + 1; c < T && !(it[c].key > A->mx[0]); c++) {
            const obox *B = &b[it[c].id];
            if (!box_overlap(A, B)) continue;
            int i = it[a].id, j = it[c].id;
            if (cull && covertex(faces + 3 * (size_t)i, faces + 3 * (size_t)j)) continue;
            pv_push(&eb[orc_tid()].pairs, i < j ? i : j, i < j ? j : i);
            total++;
        }
    }
    pvec all = {0};
    emit_merge(eb, NULL, NULL, &all);
    int64_t n = all.n < cap ? all.n : cap;
    if (out && n > 0) memcpy(out, all.d, sizeof(int) * 2 * (size_t)n);
    pv_free(&all);
    free(b);
    free(it);
    return total;
}

/* BenchmarkLogic::maintainScheme, STATIC_MANDATORY with divergent marks
 * (Mine/system/Logic/BenchmarkLogic.hpp:102-117), cycles 12 (BvhSettings.h:45)
 * and 6 (BvttFrontSettings.h:49). */
void orc_schedule(int frame, int start, int *bvh_op, int *front_op) {
    int f = frame - start;
    int b = (f % 12) ? ORC_BVH_REFIT : ORC_BVH_BUILD;
    int k = f % 6, fr;
    if (k == 0) fr = (frame == start) ? ORC_FRONT_GENERATE : ORC_FRONT_UPDATE;
    else if (k == 5) fr = ORC_FRONT_REORDER;
    else fr = ORC_FRONT_KEEP;
    if (b == ORC_BVH_BUILD) fr = ORC_FRONT_GENERATE;
    if ((f + 1) % 12 == 0) fr = ORC_FRONT_KEEP;
    *bvh_op = b;
    *front_op = fr;
}
