// lbvh.cu -- LBVH build, refit and quality-triggered subtree restructuring.
//
// Build follows the reference's construction rule (Apetrei-style bottom-up
// climb; a node covering leaves (l, r] is the right child of split l when
// metric[l] < metric[r], else the left child of split r;
// Mine/collision/lbvh/LBvhBuildKernels.cu:135-172) so the topology, the DFS
// numbering and the escape links are the reference's.  The DFS ids are
// computed without the reference's sequential chain walk
// (calcIntNodeOrders, :174-185): every node records its distance from the
// bottom of its left chain during the climb, the chain top records the chain
// length, and one scan over chain lengths gives every id in parallel.
#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_fp16.h>

#include "pipeline.h"
#include "prims.cuh"

namespace bvhcd {

bvhcd_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return BVHCD_OK;
    if (e == cudaErrorMemoryAllocation) return BVHCD_OUT_OF_MEMORY;
    return BVHCD_CUDA_ERROR;
}

#define BV_TRY(x)                                  \
    do {                                           \
        cudaError_t e__ = (x);                     \
        if (e__ != cudaSuccess) return cuda_status(e__); \
    } while (0)

namespace {

constexpr int kThreads = 256;
constexpr int kBoxTile = 4096;  // triangles per block of the per-scene box reduction
inline unsigned grid_for(int64_t n, int per = kThreads) {
    int64_t g = (n + per - 1) / per;
    if (g < 1) g = 1;
    if (g > 65535LL * 64) g = 65535LL * 64;
    return (unsigned)g;
}

__device__ __forceinline__ int split_metric(unsigned a, unsigned b) {
    return 32 - __clz(a ^ b);  // __clz(0) == 32 -> 0
}

// ---------------------------------------------------------------- scene box
// Block-wide min/max of three coordinates; the result lands in out[0..5]
// (shared) for threads 0..5 after the call.
__device__ __forceinline__ void block_box(float (&mn)[3], float (&mx)[3], float *out) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    __shared__ float s[kThreads / 32][6];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; k++) { s[w][k] = mn[k]; s[w][3 + k] = mx[k]; }
    __syncthreads();
    if (threadIdx.x < 6) {
        float v = s[0][threadIdx.x];
        for (int q = 1; q < kThreads / 32; q++)
            v = threadIdx.x < 3 ? fminf(v, s[q][threadIdx.x]) : fmaxf(v, s[q][threadIdx.x]);
        out[threadIdx.x] = v;
    }
}

__device__ __forceinline__ void box_of_range(int first, int end, int step, const PrimSrc &p, float (&mn)[3],
                                             float (&mx)[3]) {
    for (int t = first; t < end; t += step) {
        float4 lo, hi;
        prim_box(p, t, lo, hi);
        mn[0] = fminf(mn[0], lo.x); mn[1] = fminf(mn[1], lo.y); mn[2] = fminf(mn[2], lo.z);
        mx[0] = fmaxf(mx[0], hi.x); mx[1] = fmaxf(mx[1], hi.y); mx[2] = fmaxf(mx[2], hi.z);
    }
}

__global__ void __launch_bounds__(kThreads) k_box_partial(int T, PrimSrc p, float *partial) {
    float mn[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float mx[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    box_of_range(blockIdx.x * blockDim.x + threadIdx.x, T, gridDim.x * blockDim.x, p, mn, mx);
    __shared__ float out[6];
    block_box(mn, mx, out);
    if (threadIdx.x < 6) partial[6 * blockIdx.x + threadIdx.x] = out[threadIdx.x];
}

__global__ void __launch_bounds__(kThreads) k_box_final(int n, const float *partial, float *scene) {
    float mn[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float mx[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    for (int q = threadIdx.x; q < n; q += blockDim.x)
        for (int k = 0; k < 3; k++) {
            mn[k] = fminf(mn[k], partial[6 * q + k]);
            mx[k] = fmaxf(mx[k], partial[6 * q + 3 + k]);
        }
    __shared__ float out[6];
    block_box(mn, mx, out);
    if (threadIdx.x < 6) scene[threadIdx.x] = out[threadIdx.x];
}

// ---------------------------------------------------------------- batched scenes
// A batch of independent scenes is built as one forest.  Scene s owns the
// input triangles [off[s], off[s+1]) and, in the tree, the leaves
// [off[s], off[s+1]) sorted by (scene, Morton code) and the internal nodes
// with DFS ids [off[s] - s, off[s+1] - s - 1).  Each scene's subtree is the
// tree the scene would get on its own, shifted by those offsets: its own box
// normalises its codes, a scene boundary is a split no climb crosses (the
// confined rebuild of a restructure, with scenes as the subtrees), and the
// escape after a scene's last leaf ends the traversal.

// Exact float min/max through integer atomics on the bit pattern: non-negative
// floats order like their bits as signed ints, negative ones in reverse of
// their bits as unsigned ints.
__device__ __forceinline__ void atomic_min_f32(float *a, float v) {
    if (v >= 0.f) atomicMin(reinterpret_cast<int *>(a), __float_as_int(v));
    else atomicMax(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f32(float *a, float v) {
    if (v >= 0.f) atomicMax(reinterpret_cast<int *>(a), __float_as_int(v));
    else atomicMin(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}

__global__ void k_sbox_init(int S, float *sbox) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * S; i += gridDim.x * blockDim.x)
        sbox[i] = (i % 6) < 3 ? 3.402823466e+38f : -3.402823466e+38f;
}

// Per-scene boxes: one block per tile {scene, first, end} of one scene's
// triangles; the tile's box is merged into its scene's with the atomics above
// (min/max are exact, so the box equals the scene's own reduction).
__global__ void __launch_bounds__(kThreads) k_sbox_tiles(const int4 *__restrict__ tiles, PrimSrc p,
                                                         float *sbox) {
    const int4 tl = tiles[blockIdx.x];
    float mn[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float mx[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    box_of_range(tl.y + threadIdx.x, tl.z, blockDim.x, p, mn, mx);
    __shared__ float out[6];
    block_box(mn, mx, out);
    if (threadIdx.x < 3) atomic_min_f32(sbox + 6 * tl.x + threadIdx.x, out[threadIdx.x]);
    else if (threadIdx.x < 6) atomic_max_f32(sbox + 6 * tl.x + threadIdx.x, out[threadIdx.x]);
}

// 64-bit keys (scene << 30 | 30-bit code of the triangle in its scene's box).
__global__ void k_morton_seg(int T, PrimSrc p, const int *__restrict__ scene_of, const float *__restrict__ sbox,
                             unsigned long long *keys, int *vals) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const int sc = __ldg(scene_of + t);
        float4 lo, hi;
        prim_box(p, t, lo, hi);
        float box[6];
#pragma unroll
        for (int k = 0; k < 6; k++) box[k] = __ldg(sbox + 6 * sc + k);
        keys[t] = ((unsigned long long)sc << 30) | morton_box(lo, hi, box);
        vals[t] = t;
    }
}

// ---------------------------------------------------------------- build
__global__ void k_morton(int T, PrimSrc p, const float *__restrict__ scene, unsigned *keys, int *vals) {
    __shared__ float s[6];
    if (threadIdx.x < 6) s[threadIdx.x] = scene[threadIdx.x];
    __syncthreads();
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        float4 lo, hi;
        prim_box(p, t, lo, hi);
        keys[t] = morton_box(lo, hi, s);
        vals[t] = t;
    }
}

// Morton-ordered primitives and leaves (calcInverseMapping,
// Mine/utility/CudaKernelUtils.cu:28-32; buildPrimitives,
// LBvhBuildKernels.cu:114-133, here storing the vertex ids too;
// calcExtNodeSplitMetrics, Mine/collision/lbvh/BvhExtNode.cu:128-134).
__device__ __forceinline__ void write_leaf(int i, int t, unsigned k, int metric_i, const PrimSrc &p,
                                           int4 *sface, int *primmap, unsigned *code, int *metric,
                                           float4 *lrec) {
    int4 f = make_int4(__ldg(p.faces + 3 * (size_t)t), __ldg(p.faces + 3 * (size_t)t + 1),
                       __ldg(p.faces + 3 * (size_t)t + 2), t);
    sface[i] = f;
    primmap[t] = i;
    code[i] = k;
    metric[i] = metric_i;
    float4 lo, hi;
    face_box(p, f, lo, hi);
    lrec[2 * i] = lo;
    lrec[2 * i + 1] = hi;
}

__global__ void k_leaves(int T, const unsigned *__restrict__ keys, const int *__restrict__ vals, PrimSrc p,
                         int4 *sface, int *primmap, unsigned *code, int *metric, float4 *lrec) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        const unsigned k = keys[i];
        write_leaf(i, vals[i], k, (i != T - 1) ? split_metric(k, keys[i + 1]) : 33, p, sface, primmap, code,
                   metric, lrec);
    }
}

// Leaves of a forest: the scene id of every slot goes to leafscene (the
// metric across a scene boundary is never read: the boundary decides).
__global__ void k_leaves_seg(int T, const unsigned long long *__restrict__ keys, const int *__restrict__ vals,
                             PrimSrc p, int4 *sface, int *primmap, unsigned *code, int *metric, float4 *lrec,
                             int *leafscene) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        const unsigned c = (unsigned)(k & 0x3fffffffu);
        leafscene[i] = (int)(k >> 30);
        const int m = (i != T - 1) ? split_metric(c, (unsigned)(keys[i + 1] & 0x3fffffffu)) : 33;
        write_leaf(i, vals[i], c, m, p, sface, primmap, code, metric, lrec);
    }
}

// FP64 primitive boxes (min xyz, max xyz) to FP32, rounded outward
__global__ void k_boxes_f64(int64_t n, const double *__restrict__ in, float *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (i % 6) < 3 ? __double2float_rd(in[i]) : __double2float_ru(in[i]);
}

__global__ void k_single_leaf(int *lca, float4 *lrec) {
    if (threadIdx.x == 0) {
        lca[0] = 1;
        lca[1] = -1;
        lrec[0].w = __int_as_float(-1);
        lrec[1].w = __int_as_float(-1);
    }
}

__global__ void k_metrics(int T,const unsigned *__restrict__ code, int *metric) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x)
        metric[i] = (i != T - 1) ? split_metric(code[i], code[i + 1]) : 33;
}

struct Climb {
    int *ulc, *urc, *upar, *urx, *ury;
    unsigned *umark;
    float4 *ubox;
    unsigned *uflag;
    int *posb, *clen, *ulpar;
    int *uheight;  // node height (leaves 0), for the refit plan
};

// Arrival at a parent: an exchange with acquire-release semantics at device
// scope.  The first child to arrive leaves its tagged reference (+1, so that
// 0 means nobody yet) and stops; the second gets that reference back, and
// the release by the first makes the data it wrote before (its box, range,
// chain position, height) visible to the second's loads.
__device__ __forceinline__ unsigned arrive_exch(unsigned *p, unsigned v) {
    unsigned old;
    asm volatile("atom.exch.acq_rel.gpu.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Bottom-up construction (buildIntNodes, LBvhBuildKernels.cu:135-172; with
// kSeg the confined rebuild of restrIntNodes,
// Mine/collision/lbvh/LBvhRestructureKernels.cu:122-166, over the listed
// leaves, or over all leaves of a forest when `leaves` is null, with
// `prev_topo` null: a scene root has no father).  Internal nodes are
// indexed by split.  The second thread to reach a node merges the child
// boxes, records its height and posb = distance from the bottom of its left
// chain and, at a chain top, the chain length of the chain's leftmost leaf.
//
// A thread carries the node it stands for in registers (tagged reference
// node << 1 or leaf << 1 | 1, box, leaf range, posb, height) and writes the
// node's results before it arrives at the parent; the second arrival loads
// only the sibling's box and the two of its fields it needs, all at once.  One
// exchange per level orders everything (the uflag words start at 0).
template <bool kSeg>
__global__ void __launch_bounds__(kThreads) k_climb(int T, int n, const int *__restrict__ leaves,
                                                    const int *__restrict__ seg,
                                                    const int *__restrict__ metric,
                                                    const float4 *__restrict__ lrec,
                                                    const int4 *__restrict__ prev_topo, Climb c) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int idx = (kSeg && leaves) ? leaves[k] : k;
        const int sub = kSeg ? seg[idx] : 0;
        int l = idx - 1, r = idx, bd = 0;
        bool right;  // the node is the right child of its parent
        if (kSeg) bd = ((l < 0 || seg[l] != sub) ? 2 : 0) | ((r == T - 1 || seg[r + 1] != sub) ? 1 : 0);
        if (bd) right = bd & 1;
        else right = (l >= 0) && (metric[l] < metric[r]);
        int cur = right ? l : r;  // the parent split
        c.ulpar[idx] = cur;
        if (right) c.clen[idx] = 0;
        int ref = (idx << 1) | 1, rx = idx, ry = idx, pb = 0, h = 0;
        float4 lo = __ldg(&lrec[2 * idx]), hi = __ldg(&lrec[2 * idx + 1]);
        while (true) {
            const unsigned old = arrive_exch(&c.uflag[cur], (unsigned)ref + 1u);
            if (old == 0u) break;  // first arrival: the sibling's thread goes on
            const int sref = (int)old - 1, sib = sref >> 1;
            float4 slo, shi;
            int sbound = sib, spb = 0, sh = 0;
            if (sref & 1) {
                slo = __ldcg(&lrec[2 * sib]);
                shi = __ldcg(&lrec[2 * sib + 1]);
            } else {
                slo = __ldcg(&c.ubox[2 * sib]);
                shi = __ldcg(&c.ubox[2 * sib + 1]);
                sbound = right ? __ldcg(&c.urx[sib]) : __ldcg(&c.ury[sib]);
                spb = __ldcg(&c.posb[sib]);
                sh = __ldcg(&c.uheight[sib]);
            }
            const int lref = right ? sref : ref, rref = right ? ref : sref;
            const unsigned m = (unsigned)(lref & 1) | ((unsigned)(rref & 1) << 1);
            const int nrx = right ? sbound : rx, nry = right ? ry : sbound;
            lo = make_float4(fminf(lo.x, slo.x), fminf(lo.y, slo.y), fminf(lo.z, slo.z), 0.f);
            hi = make_float4(fmaxf(hi.x, shi.x), fmaxf(hi.y, shi.y), fmaxf(hi.z, shi.z), 0.f);
            pb = (m & 1u) ? 0 : (right ? spb : pb) + 1;
            h = 1 + max(h, sh);
            c.ulc[cur] = lref >> 1;
            c.urc[cur] = rref >> 1;
            c.urx[cur] = nrx;
            c.ury[cur] = nry;
            c.ubox[2 * cur] = lo;
            c.ubox[2 * cur + 1] = hi;
            c.posb[cur] = pb;
            c.uheight[cur] = h;
            rx = nrx;
            ry = nry;
            l = rx - 1;
            r = ry;
            if (kSeg) bd = ((l < 0 || seg[l] != sub) ? 2 : 0) | ((r == T - 1 || seg[r + 1] != sub) ? 1 : 0);
            const bool is_root = kSeg ? (bd == 3) : (l + 1 == 0 && r == T - 1);
            if (is_root) {
                c.upar[cur] = -1;
                const bool rflag = (kSeg && prev_topo) ? ((prev_topo[sub].w & 4) != 0) : false;
                c.umark[cur] = m | (rflag ? 4u : 0u);
                c.clen[rx] = pb + 1;
                break;
            }
            if (bd) right = bd & 1;
            else right = (l >= 0) && (metric[l] < metric[r]);
            const int par = right ? l : r;
            c.upar[cur] = par;
            c.umark[cur] = m | (right ? 4u : 0u);
            if (right) c.clen[rx] = pb + 1;
            ref = cur << 1;
            cur = par;
        }
    }
}

// DFS id of every internal node: chain offset of its leftmost leaf plus its
// position from the chain top (calcIntNodeOrders, LBvhBuildKernels.cu:174-185).
// In a forest the split after a scene's last leaf is no node (`leafscene`
// non-null marks those splits).
__device__ __forceinline__ bool scene_end(const int *leafscene, int s, int T) {
    return leafscene && s + 1 < T && __ldg(leafscene + s + 1) != __ldg(leafscene + s);
}

__global__ void k_dfs_ids(int nint, const int *__restrict__ urx, const int *__restrict__ posb,
                          const unsigned *__restrict__ coff, const int *__restrict__ clen,
                          const int *__restrict__ leafscene, int *dfs) {
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nint; u += gridDim.x * blockDim.x) {
        if (scene_end(leafscene, u, nint + 1)) continue;
        int rx = urx[u];
        dfs[u] = (int)coff[rx] + clen[rx] - 1 - posb[u];
    }
}

__device__ __forceinline__ int lca_of(int s, int T, const unsigned *coff, const int *clen) {
    if (s >= T) return -1;
    return clen[s] > 0 ? (int)(coff[s] << 1) : ((s << 1) | 1);
}

// Escape links and leaf parents (updateBvhExtNodeLinks, LBvhBuildKernels.cu:187-200).
__global__ void k_leaf_links(int T, const unsigned *__restrict__ coff, const int *__restrict__ clen,
                             const int *__restrict__ ulpar, const int *__restrict__ dfs,
                             const int *__restrict__ leafscene, int *lca, float4 *lrec) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < T; s += gridDim.x * blockDim.x) {
        lca[s] = lca_of(s, T, coff, clen);
        if (s == 0) lca[T] = -1;
        reinterpret_cast<float *>(lrec)[8 * (size_t)s + 3] = __int_as_float(dfs[ulpar[s]]);
        const int esc = scene_end(leafscene, s, T) ? -1 : lca_of(s + 1, T, coff, clen);
        reinterpret_cast<float *>(lrec)[8 * (size_t)s + 7] = __int_as_float(esc);
    }
}

// Internal nodes in DFS order (reorderIntNode, LBvhBuildKernels.cu:202-217).
__global__ void k_write_nodes(int nint, int T, Climb c, const int *__restrict__ dfs,
                              const unsigned *__restrict__ coff, const int *__restrict__ clen,
                              const int *__restrict__ leafscene, float4 *nrec, int4 *topo, int2 *nrange,
                              int *height) {
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nint; u += gridDim.x * blockDim.x) {
        if (scene_end(leafscene, u, T)) continue;
        int d = dfs[u];
        unsigned m = c.umark[u];
        int lc = c.ulc[u], rc = c.urc[u], p = c.upar[u];
        int rx = c.urx[u], ry = c.ury[u];
        topo[d] = make_int4((m & 1u) ? lc : dfs[lc], (m & 2u) ? rc : dfs[rc], p < 0 ? -1 : dfs[p], (int)m);
        nrange[d] = make_int2(rx, ry);
        height[d] = c.uheight[u];
        float4 lo = c.ubox[2 * u], hi = c.ubox[2 * u + 1];
        lo.w = __int_as_float(rx | ((m & 1u) ? (int)0x80000000 : 0));  // bit 31: the left child is leaf rx
        hi.w = __int_as_float(scene_end(leafscene, ry, T) ? -1 : lca_of(ry + 1, T, coff, clen));
        nrec[2 * d] = lo;
        nrec[2 * d + 1] = hi;
    }
}

// ---------------------------------------------------------------- refit
// refitExtNode + refitIntNode (Mine/collision/lbvh/LBvhUpdateKernels.cu:35-74):
// leaf boxes from the three vertices, then every internal box as the union of
// its children's, bottom-up.
//
// A climb over the whole tree with one arrival counter per node pays a
// device-scope atomic and fence per level on its longest leaf-to-root chain,
// and those chains set its time.  This refit runs level by level instead, in
// node height order (a parent is higher than its children), in shared
// memory, with CTA barriers between levels:
//  - the leaves are cut into blocks of kRefitW; a node whose leaf range lies
//    in one block is local to it, the others (the top of the tree and the
//    spines above each block boundary) cross;
//  - one CTA per leaf block computes its leaf boxes, then its local nodes
//    from a level-sorted list, and exports the boxes the crossing nodes need
//    (those of its local subtree roots and boundary leaves) to a compact
//    array;
//  - the CTA that finishes last (a counter after a fence; nothing waits)
//    computes the crossing nodes level by level from that array.
// Every record is written whole (box and links) in one 256-bit store: the
// links come from the plan, so no record is read.  Min and max are exact,
// so the boxes equal those of any bottom-up order.  The plan (splits,
// heights, lists, links, exports) depends on the topology only; refit_plan
// rebuilds it after every build and restructure.
constexpr int kRefitW = 4096;        // leaves per local block
constexpr int kRefitThreads = 1024;  // threads per refit CTA
constexpr int kRefitSlots = kRefitW / kRefitThreads;
constexpr int kMaxLevels = 64;       // levels a level-sorted list holds (deeper: one pass per height)
// per list: level count L (or -1), level offsets 0..L+1, then at fixed places
// the node count (crossing list) or export count (block list), the list
// length, and the first narrow level
constexpr int kLevelHdr = kMaxLevels + 6;
constexpr int kHdrCount = kLevelHdr - 3, kHdrLen = kLevelHdr - 2, kHdrNarrow = kLevelHdr - 1;
constexpr int kLevelThreads = 256;  // threads that run the wide levels of a list
// boxes of the block's leaves and nodes, then its level-sorted work list; the
// last CTA reuses it for the crossing nodes' boxes and list
constexpr size_t kLocalSmem = (size_t)2 * kRefitW * 6 * sizeof(float) + (size_t)kRefitW * sizeof(int);

// Node heights (leaves 0, a node one above its higher child), bottom-up with
// arrival counters: run once per topology, so its fences do not matter.
__global__ void __launch_bounds__(kThreads) k_heights(int T, const float4 *__restrict__ lrec,
                                                      const int4 *__restrict__ topo, unsigned *flag, int *height) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < T; s += gridDim.x * blockDim.x) {
        int p = __float_as_int(__ldg(reinterpret_cast<const float *>(lrec) + 8 * (size_t)s + 3));
        int h = 0;
        for (int guard = T; p >= 0 && guard > 0; --guard) {
            atomicMax(&height[p], h + 1);
            __threadfence();
            if (atomicAdd(&flag[p], 1u) == 0u) break;
            __threadfence();
            h = __ldcg(&height[p]);
            p = __ldg(&topo[p]).z;
        }
    }
}

// split of each internal node (the last leaf of its left subtree: every
// internal node has its own) and whether its leaf range crosses a block
__global__ void k_plan_split(int nint, const int4 *__restrict__ topo, const int2 *__restrict__ nrange, int *split,
                             unsigned *cross) {
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nint; d += gridDim.x * blockDim.x) {
        const int4 t = topo[d];
        split[d] = (t.w & 1) ? t.x : nrange[t.x].y;
        const int2 r = nrange[d];
        cross[d] = (r.x / kRefitW) != (r.y / kRefitW) ? 1u : 0u;
    }
}

__device__ __forceinline__ void box_empty(float4 &lo, float4 &hi) {
    lo = make_float4(3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f, 0.f);
    hi = make_float4(-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f, 0.f);
}
// boxes as 6 floats (24 bytes, 8-byte aligned): three 64-bit accesses
// |b - a| rounded up
__device__ __forceinline__ float box_change(float a, float b) { return fmaxf(__fsub_ru(b, a), __fsub_ru(a, b)); }
__device__ __forceinline__ void box_store6(float *b, const float4 &lo, const float4 &hi) {
    float2 *q = reinterpret_cast<float2 *>(b);
    q[0] = make_float2(lo.x, lo.y);
    q[1] = make_float2(lo.z, hi.x);
    q[2] = make_float2(hi.y, hi.z);
}
__device__ __forceinline__ void box_load6(const float *b, float4 &lo, float4 &hi) {
    const float2 *q = reinterpret_cast<const float2 *>(b);
    const float2 u = q[0], v = q[1], w = q[2];
    lo = make_float4(u.x, u.y, v.x, 0.f);
    hi = make_float4(v.y, w.x, w.y, 0.f);
}
__device__ __forceinline__ void box_union(float4 &lo, float4 &hi, const float4 &clo, const float4 &chi) {
    lo.x = fminf(lo.x, clo.x); lo.y = fminf(lo.y, clo.y); lo.z = fminf(lo.z, clo.z);
    hi.x = fmaxf(hi.x, chi.x); hi.y = fmaxf(hi.y, chi.y); hi.z = fmaxf(hi.z, chi.z);
}
__device__ __forceinline__ void box_union6(const float *b, float4 &lo, float4 &hi) {
    float4 clo, chi;
    box_load6(b, clo, chi);
    box_union(lo, hi, clo, chi);
}
// the box fields of a 32-byte record ({lo.xyz, link}, {hi.xyz, link}); the
// links stay (the deep-tree forms only)
__device__ __forceinline__ void rec_store_box(float4 *rec, const float4 &lo, const float4 &hi) {
    float *w = reinterpret_cast<float *>(rec);
    w[0] = lo.x; w[1] = lo.y; w[2] = lo.z;
    w[4] = hi.x; w[5] = hi.y; w[6] = hi.z;
}

// plan[split(d)] = {d, or -1 if d crosses; left ref; right ref; height},
// refs (leaf << 1 | 1) or (split << 1).  top[k] for the k-th crossing node
// = {d; left ref; right ref; height}, refs (leaf << 2 | 1), (local node << 2)
// or (crossing k << 2 | 2).  A non-crossing child of crossing node k on side
// c is marked for export to slot 2k + c (lexp per leaf, nexp per node); a
// crossing child's export slot holds the empty box.
__global__ void k_plan_write(int nint, const int4 *__restrict__ topo, const int *__restrict__ split,
                             const unsigned *__restrict__ cross, const unsigned *__restrict__ topk,
                             const int *__restrict__ height, int4 *plan, int4 *top, int *lexp, int *nexp,
                             float *gext) {
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nint; d += gridDim.x * blockDim.x) {
        const int4 t = topo[d];
        const bool lleaf = (t.w & 1) != 0, rleaf = (t.w & 2) != 0;
        const bool c = cross[d] != 0;
        const int h = height[d];
        plan[split[d]] = make_int4(c ? -1 : d, lleaf ? (t.x << 1) | 1 : split[t.x] << 1,
                                   rleaf ? (t.y << 1) | 1 : split[t.y] << 1, h);
        if (!c) continue;
        const int k = (int)topk[d];
        auto ref = [&](int ch, bool leaf) {
            return leaf ? (ch << 2) | 1 : cross[ch] ? (int)(topk[ch] << 2) | 2 : ch << 2;
        };
        top[k] = make_int4(d, ref(t.x, lleaf), ref(t.y, rleaf), h);
        const int ch[2] = {t.x, t.y};
        const bool leaf[2] = {lleaf, rleaf};
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const int slot = 2 * k + side;
            if (leaf[side]) lexp[ch[side]] = slot;
            else if (!cross[ch[side]]) nexp[ch[side]] = slot;
            else {
                float4 lo, hi;
                box_empty(lo, hi);
                box_store6(gext + 6 * (size_t)slot, lo, hi);
            }
        }
    }
}

// Level-sorted work lists, built once per topology by one CTA per list:
// count per level, offsets, scatter.  hdr[0] = number of levels L (or -1
// when the heights span more than kMaxLevels), hdr[1 + h] = offset of level
// h, h = 0..L + 1, hdr[kHdrLen] = the list length, hdr[kHdrNarrow] = the
// first level from which every level has at most 32 nodes (one warp runs
// those, with warp barriers).
__device__ void level_sort_begin(int *cnt) {
    if (threadIdx.x <= kMaxLevels) cnt[threadIdx.x] = 0;
}
__device__ void level_sort_offsets(const int *cnt, int *cur, int L, int *hdr) {
    if (threadIdx.x != 0) return;
    int acc = 0;
    hdr[0] = L;
    for (int h = 0; h <= L; h++) {
        hdr[1 + h] = acc;
        cur[h] = acc;
        acc += cnt[h];
    }
    hdr[2 + L] = acc;
    hdr[kHdrLen] = acc;
    int lw = L + 1;
    while (lw > 0 && cnt[lw - 1] <= 32) lw--;
    hdr[kHdrNarrow] = lw;
}

// Local lists: for leaf block b, its local nodes by height (level h - 1 holds
// height h).  A node's box slot is kRefitW + its list position; the entry is
// {node, left child slot << 16 | right child slot, node links (rangex,
// escape)}; a leaf's slot is its index in the block.  llink holds every
// leaf's links (parent, escape).  lexport[b * kRefitW + x] = {export slot,
// box slot with the list, box slot without it (kRefitW + split - L0)},
// hdr[kHdrCount] their count.
__global__ void __launch_bounds__(kRefitThreads) k_plan_local(int T, const int4 *__restrict__ plan,
                                                              const float4 *__restrict__ lrec,
                                                              const float4 *__restrict__ nrec,
                                                              const int *__restrict__ lexp,
                                                              const int *__restrict__ nexp, int4 *llist,
                                                              int2 *llink, int4 *lexport, int *lhdr) {
    __shared__ int cnt[kMaxLevels + 1], cur[kMaxLevels + 1], hmax, nex, pos_of[kRefitW];
    const int L0 = blockIdx.x * kRefitW, nl = min(kRefitW, T - L0);
    int *hdr = lhdr + (size_t)blockIdx.x * kLevelHdr;
    level_sort_begin(cnt);
    if (threadIdx.x == 0) { hmax = 0; nex = 0; }
    __syncthreads();
    int4 e[kRefitSlots];
    int hm = 0;
#pragma unroll
    for (int i = 0; i < kRefitSlots; i++) {
        const int j = threadIdx.x + i * kRefitThreads;
        e[i] = (j < nl && L0 + j < T - 1) ? __ldg(&plan[L0 + j]) : make_int4(-1, -1, -1, 0);
        if (e[i].x >= 0) hm = max(hm, e[i].w);
        if (j < nl) {
            float4 lo, hi;
            ldg8(lrec + 2 * (size_t)(L0 + j), lo, hi);
            llink[L0 + j] = make_int2(__float_as_int(lo.w), __float_as_int(hi.w));
        }
    }
    atomicMax(&hmax, hm);
    __syncthreads();
    const int H = hmax;
    const bool listed = H <= kMaxLevels;
    if (listed) {
#pragma unroll
        for (int i = 0; i < kRefitSlots; i++)
            if (e[i].x >= 0) atomicAdd(&cnt[e[i].w - 1], 1);
        __syncthreads();
        level_sort_offsets(cnt, cur, max(H - 1, 0), hdr);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kRefitSlots; i++)
            if (e[i].x >= 0) pos_of[threadIdx.x + i * kRefitThreads] = atomicAdd(&cur[e[i].w - 1], 1);
        __syncthreads();
        auto slot = [&](int ref) { return (ref & 1) ? (ref >> 1) - L0 : kRefitW + pos_of[(ref >> 1) - L0]; };
#pragma unroll
        for (int i = 0; i < kRefitSlots; i++) {
            if (e[i].x < 0) continue;
            float4 lo, hi;
            ldg8(nrec + 2 * (size_t)e[i].x, lo, hi);
            llist[L0 + pos_of[threadIdx.x + i * kRefitThreads]] = make_int4(
                e[i].x, (slot(e[i].y) << 16) | slot(e[i].z), __float_as_int(lo.w), __float_as_int(hi.w));
        }
    } else if (threadIdx.x == 0) {
        hdr[0] = -1;
    }
#pragma unroll
    for (int i = 0; i < kRefitSlots; i++) {
        const int j = threadIdx.x + i * kRefitThreads;
        if (j >= nl) continue;
        const int le = __ldg(&lexp[L0 + j]);
        if (le >= 0) lexport[(size_t)L0 + atomicAdd(&nex, 1)] = make_int4(le, j, j, 0);
        if (e[i].x < 0) continue;
        const int ne = __ldg(&nexp[e[i].x]);
        if (ne >= 0)
            lexport[(size_t)L0 + atomicAdd(&nex, 1)] = make_int4(ne, listed ? kRefitW + pos_of[j] : -1, kRefitW + j, 0);
    }
    __syncthreads();
    if (threadIdx.x == 0) hdr[kHdrCount] = nex;
}

// Top list: the crossing nodes that have a crossing child, by height (level
// h - H0, H0 the lowest crossing height), as {k, crossing child k or -1, the
// other or -1, 0}; tlink[k] = node k's links (rangex, escape); thdr[kHdrCount]
// = the number of crossing nodes.
__global__ void __launch_bounds__(kRefitThreads) k_plan_top(const unsigned *__restrict__ ctr,
                                                            const int4 *__restrict__ top,
                                                            const float4 *__restrict__ nrec, int4 *tlist,
                                                            int2 *tlink, int *thdr) {
    __shared__ int cnt[kMaxLevels + 1], cur[kMaxLevels + 1], hlo, hhi;
    const int K = (int)ctr[C_TOPK];
    level_sort_begin(cnt);
    if (threadIdx.x == 0) { hlo = INT_MAX; hhi = 0; }
    __syncthreads();
    int h0 = INT_MAX, h1 = 0;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int4 e = __ldg(&top[k]);
        h0 = min(h0, e.w);
        h1 = max(h1, e.w);
        float4 lo, hi;
        ldg8(nrec + 2 * (size_t)e.x, lo, hi);
        tlink[k] = make_int2(__float_as_int(lo.w), __float_as_int(hi.w));
    }
    atomicMin(&hlo, h0);
    atomicMax(&hhi, h1);
    if (threadIdx.x == 0) { thdr[kHdrCount] = K; thdr[kHdrLen] = 0; }
    __syncthreads();
    const int H0 = hlo, H1 = hhi;
    if (H1 - H0 > kMaxLevels) {
        if (threadIdx.x == 0) thdr[0] = -1;
        return;
    }
    auto pending = [](const int4 &e) { return (e.y & 3) == 2 || (e.z & 3) == 2; };
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int4 e = __ldg(&top[k]);
        if (pending(e)) atomicAdd(&cnt[e.w - H0], 1);
    }
    __syncthreads();
    level_sort_offsets(cnt, cur, H1 - H0, thdr);
    __syncthreads();
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int4 e = __ldg(&top[k]);
        if (!pending(e)) continue;
        const int pos = atomicAdd(&cur[e.w - H0], 1);
        tlist[pos] = make_int4(k, (e.y & 3) == 2 ? e.y >> 2 : -1, (e.z & 3) == 2 ? e.z >> 2 : -1, 0);
    }
}

// Levels 0..L of a level-sorted list: the wide ones by the first kN threads
// with a named barrier among them (kN = the CTA: the CTA barrier), from level
// lw on (each at most 32 nodes) by warp 0 with warp barriers.  work(t)
// handles list position t.  Every thread of the CTA calls it.
template <int kN, typename F>
__device__ __forceinline__ void run_levels(const int *ofs, int L, int lw, F work) {
    if (threadIdx.x < kN) {
        for (int h = 0; h < lw && h <= L; h++) {
            for (int t = ofs[h] + threadIdx.x; t < ofs[h + 1]; t += kN) work(t);
            if (kN == kRefitThreads) __syncthreads();
            else asm volatile("bar.sync 1, %0;" ::"n"(kN) : "memory");
        }
    }
    if (threadIdx.x < 32) {
        for (int h = lw; h <= L; h++) {
            const int t = ofs[h] + threadIdx.x;
            if (t < ofs[h + 1]) work(t);
            __syncwarp();
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void top_level_work(const int4 &q, float *box) {
    float *b = box + 6 * (size_t)q.x;
    float4 lo, hi;
    box_load6(b, lo, hi);
    if (q.y >= 0) box_union6(box + 6 * (size_t)q.y, lo, hi);
    if (q.z >= 0) box_union6(box + 6 * (size_t)q.z, lo, hi);
    box_store6(b, lo, hi);
}

struct RefitTop {
    const int4 *top, *tlist;
    const int2 *tlink;
    const int *thdr;
    const float *gext;  // 2 export slots per crossing node
    float *gbox;        // crossing-node slots when shared memory is too small
    unsigned *done;     // leaf blocks finished
    unsigned *delta;    // largest leaf box change of this refit (FP32 bits)
    unsigned *motion;   // accumulated leaf box change (FP32 bits)
    unsigned *nf_acc;   // a block saw a non-finite input coordinate
    unsigned *nonfinite;  // the refit's verdict (written by the last block)
    float4 *v4;           // the positions as 16-byte records (null for a box scene)
    int V;
};

// The crossing nodes, run by the CTA that finished last: a node's slot
// starts as the union of its two export slots (the final boxes of its
// non-crossing children; empty for a crossing child), then the nodes with
// crossing children take those in level by level.  Slots and list in
// shared memory when they fit, else in global scratch (the CTA barrier
// orders both); without a list (heights spanning more than kMaxLevels) one
// pass per height.
__device__ void refit_top(const RefitTop &g, float4 *nrec, float *smem, int *sofs) {
    // the header at fixed places: one round trip
    const int L = __ldg(&g.thdr[0]);
    const int K = __ldg(&g.thdr[kHdrCount]);
    const int npend = __ldg(&g.thdr[kHdrLen]);
    const int lw = __ldg(&g.thdr[kHdrNarrow]);
    const int ofs_t = threadIdx.x <= kMaxLevels + 1 ? __ldg(&g.thdr[1 + threadIdx.x]) : 0;
    if (K <= 0) return;
    const size_t box_floats = ((size_t)6 * K + 3) & ~(size_t)3;
    const bool in_smem = box_floats * sizeof(float) + (size_t)npend * sizeof(int4) <= kLocalSmem;
    float *box = in_smem ? smem : g.gbox;
    int4 *slist = reinterpret_cast<int4 *>(smem + box_floats);
    if (L >= 0 && threadIdx.x <= L + 1) sofs[threadIdx.x] = ofs_t;
    for (int k0 = 0; k0 < K; k0 += 2 * kRefitThreads) {
        // this round's loads first: two nodes' export slots and list entries
        float2 x[2][6];
        int4 q[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int k = k0 + u * kRefitThreads + threadIdx.x;
            const float2 *src = reinterpret_cast<const float2 *>(g.gext + 12 * (size_t)min(k, K - 1));
#pragma unroll
            for (int c = 0; c < 6; c++) x[u][c] = __ldcg(src + c);
            q[u] = (in_smem && k < npend) ? __ldg(&g.tlist[k]) : make_int4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int k = k0 + u * kRefitThreads + threadIdx.x;
            if (k >= K) continue;
            float4 lo = make_float4(fminf(x[u][0].x, x[u][3].x), fminf(x[u][0].y, x[u][3].y),
                                    fminf(x[u][1].x, x[u][4].x), 0.f);
            float4 hi = make_float4(fmaxf(x[u][1].y, x[u][4].y), fmaxf(x[u][2].x, x[u][5].x),
                                    fmaxf(x[u][2].y, x[u][5].y), 0.f);
            box_store6(box + 6 * (size_t)k, lo, hi);
            if (in_smem && k < npend) slist[k] = q[u];
        }
    }
    __syncthreads();
    if (L >= 0) {
        if (in_smem) run_levels<kLevelThreads>(sofs, L, lw, [&](int t) { top_level_work(slist[t], box); });
        else run_levels<kLevelThreads>(sofs, L, lw, [&](int t) { top_level_work(__ldg(&g.tlist[t]), box); });
    } else {
        int hmin = INT_MAX, hmax = 0;
        for (int k = 0; k < K; k++) {
            const int h = __ldg(&g.top[k]).w;
            hmin = min(hmin, h);
            hmax = max(hmax, h);
        }
        for (int h = hmin; h <= hmax; h++) {
            for (int k = threadIdx.x; k < K; k += blockDim.x) {
                const int4 e = __ldg(&g.top[k]);
                if (e.w != h || ((e.y & 3) != 2 && (e.z & 3) != 2)) continue;
                top_level_work(make_int4(k, (e.y & 3) == 2 ? e.y >> 2 : -1, (e.z & 3) == 2 ? e.z >> 2 : -1, 0), box);
            }
            __syncthreads();
        }
    }
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int d = __ldg(&g.top[k]).x;
        const int2 lk = __ldg(&g.tlink[k]);
        float4 lo, hi;
        box_load6(box + 6 * (size_t)k, lo, hi);
        lo.w = __int_as_float(lk.x);
        hi.w = __int_as_float(lk.y);
        stg8(nrec + 2 * (size_t)d, lo, hi);
    }
}

// One CTA per block of kRefitW leaves: leaf boxes, then the block's local
// nodes level by level from its level-sorted list, all in shared memory,
// then its exports; the last CTA to finish runs the crossing nodes.
__global__ void __launch_bounds__(kRefitThreads, 1) k_refit(int T, const int4 *__restrict__ sface, PrimSrc p,
                                                            const int4 *__restrict__ plan,
                                                            const int4 *__restrict__ llist,
                                                            const int2 *__restrict__ llink,
                                                            const int4 *__restrict__ lexport,
                                                            const int *__restrict__ lhdr, float4 *lrec,
                                                            float4 *nrec, float *gext, RefitTop g) {
    extern __shared__ __align__(16) float sb[];  // boxes: the block's leaves, then its nodes
    int *slist = reinterpret_cast<int *>(sb + 12 * kRefitW);
    __shared__ int sofs[kLevelHdr], hmax, last;
    __shared__ unsigned sdelta, snf;
    const int L0 = blockIdx.x * kRefitW;
    const int nl = min(kRefitW, T - L0);
    const int *hdr = lhdr + (size_t)blockIdx.x * kLevelHdr;
    if (threadIdx.x == 0) {
        hmax = 0;
        sdelta = 0u;
        snf = 0u;
    }
    const int L = __ldg(&hdr[0]);
    const int nloc = L >= 0 ? __ldg(&hdr[2 + L]) : 0;
    if (L >= 0 && threadIdx.x <= L + 1) sofs[threadIdx.x] = __ldg(&hdr[1 + threadIdx.x]);
    // the positions as 16-byte records for the narrow phase: a contiguous
    // share of the vertices per CTA, read and written coalesced
    if (g.v4) {
        const int per = (g.V + (int)gridDim.x - 1) / (int)gridDim.x;
        const int v1 = min(g.V, (int)blockIdx.x * per + per);
        for (int v = blockIdx.x * per + threadIdx.x; v < v1; v += kRefitThreads) {
            const float *x = p.verts + 3 * (size_t)v;
            g.v4[v] = make_float4(__ldg(x), __ldg(x + 1), __ldg(x + 2), 0.f);
        }
    }
    int4 w[kRefitSlots];
    // the largest change of a leaf box coordinate, rounded up: a bound on how
    // far any box of the tree moved (a node's box is a min / max of leaf boxes)
    float dmax = 0.f;
    bool nonfin = false;  // a NaN or infinite input coordinate
#pragma unroll
    for (int i = 0; i < kRefitSlots; i++) {
        const int t = threadIdx.x + i * kRefitThreads;
        w[i] = t < nloc ? __ldg(&llist[L0 + t]) : make_int4(-1, 0, 0, 0);
        if (t < nloc) slist[t] = w[i].y;
        if (t >= nl) continue;
        const int4 f = __ldg(&sface[L0 + t]);
        const int2 lk = __ldg(&llink[L0 + t]);
        const float4 olo = __ldcg(lrec + 2 * (size_t)(L0 + t)), ohi = __ldcg(lrec + 2 * (size_t)(L0 + t) + 1);
        float4 lo, hi;
        nonfin |= !face_box_fin(p, f, lo, hi);
        dmax = fmaxf(dmax, fmaxf(box_change(olo.x, lo.x), fmaxf(box_change(olo.y, lo.y), box_change(olo.z, lo.z))));
        dmax = fmaxf(dmax, fmaxf(box_change(ohi.x, hi.x), fmaxf(box_change(ohi.y, hi.y), box_change(ohi.z, hi.z))));
        box_store6(sb + 6 * t, lo, hi);
        lo.w = __int_as_float(lk.x);
        hi.w = __int_as_float(lk.y);
        stg8(lrec + 2 * (size_t)(L0 + t), lo, hi);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&sdelta, __float_as_uint(dmax));  // non-negative: bit order
    if (__any_sync(0xffffffffu, nonfin) && (threadIdx.x & 31) == 0) atomicOr(&snf, 1u);
    __syncthreads();
    if (L >= 0) {
        run_levels<kRefitThreads>(sofs, L, __ldg(&hdr[kHdrNarrow]), [&](int t) {
            const int q = slist[t];
            float4 lo, hi;
            box_load6(sb + 6 * (q >> 16), lo, hi);
            box_union6(sb + 6 * (q & 0xffff), lo, hi);
            box_store6(sb + 6 * (kRefitW + t), lo, hi);
        });
#pragma unroll
        for (int i = 0; i < kRefitSlots; i++) {
            if (w[i].x < 0) continue;
            float4 lo, hi;
            box_load6(sb + 6 * (kRefitW + threadIdx.x + i * kRefitThreads), lo, hi);
            lo.w = __int_as_float(w[i].z);
            hi.w = __int_as_float(w[i].w);
            stg8(nrec + 2 * (size_t)w[i].x, lo, hi);
        }
    } else {
        // a block with a chain of more than kMaxLevels local nodes: one pass
        // per height over the block's splits (slot kRefitW + split - L0)
        int4 e[kRefitSlots];
        int hm = 0;
#pragma unroll
        for (int i = 0; i < kRefitSlots; i++) {
            const int j = threadIdx.x + i * kRefitThreads;
            e[i] = (j < nl && L0 + j < T - 1) ? __ldg(&plan[L0 + j]) : make_int4(-1, -1, -1, 0);
            if (e[i].x >= 0) hm = max(hm, e[i].w);
        }
        atomicMax(&hmax, hm);
        __syncthreads();
        const int Hm = hmax;
        auto slot = [&](int ref) { return (ref & 1) ? (ref >> 1) - L0 : kRefitW + (ref >> 1) - L0; };
        for (int h = 1; h <= Hm; h++) {
#pragma unroll
            for (int i = 0; i < kRefitSlots; i++) {
                if (e[i].x < 0 || e[i].w != h) continue;
                float4 lo, hi;
                box_load6(sb + 6 * slot(e[i].y), lo, hi);
                box_union6(sb + 6 * slot(e[i].z), lo, hi);
                box_store6(sb + 6 * (kRefitW + threadIdx.x + i * kRefitThreads), lo, hi);
            }
            __syncthreads();
        }
#pragma unroll
        for (int i = 0; i < kRefitSlots; i++) {
            if (e[i].x < 0) continue;
            float4 lo, hi;
            box_load6(sb + 6 * (kRefitW + threadIdx.x + i * kRefitThreads), lo, hi);
            rec_store_box(nrec + 2 * (size_t)e[i].x, lo, hi);
        }
    }
    if (gridDim.x == 1) {  // one block: no node crosses
        if (threadIdx.x == 0) {
            *g.motion = __float_as_uint(__fadd_ru(__uint_as_float(*g.motion), __uint_as_float(sdelta)));
            *g.nonfinite = snf;
        }
        return;
    }
    const int nex = __ldg(&hdr[kHdrCount]);
    for (int x = threadIdx.x; x < nex; x += blockDim.x) {
        const int4 ex = __ldg(&lexport[(size_t)L0 + x]);
        float4 lo, hi;
        box_load6(sb + 6 * (L >= 0 ? ex.y : ex.z), lo, hi);
        float2 *q = reinterpret_cast<float2 *>(gext + 6 * (size_t)ex.x);
        __stcg(q, make_float2(lo.x, lo.y));
        __stcg(q + 1, make_float2(lo.z, hi.x));
        __stcg(q + 2, make_float2(hi.y, hi.z));
    }
    // the last CTA to finish runs the crossing nodes
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicMax(g.delta, sdelta);
        if (snf) atomicOr(g.nf_acc, 1u);
        __threadfence();
        last = atomicAdd(g.done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // the kernel after the refit may start now (a front maintain's first
    // kernels wait for the refit's end before they read what it writes)
    pdl_release();
    __threadfence();
    refit_top(g, nrec, sb, sofs);
    if (threadIdx.x == 0) {
        *g.done = 0u;
        const float d = __uint_as_float(atomicExch(g.delta, 0u));
        *g.motion = __float_as_uint(__fadd_ru(__uint_as_float(*g.motion), d));
        *g.nonfinite = atomicExch(g.nf_acc, 0u);
    }
}

// Finiteness of a build's or restructure's input (the refit checks its own
// inline): every coordinate of the n floats (positions, or a box scene's FP32
// boxes); the last block to finish writes the verdict and clears the
// accumulator, so the check needs no clearing launch.
__global__ void __launch_bounds__(kThreads) k_check_finite(int64_t n, const float *__restrict__ x, unsigned *ctr,
                                                           float4 *v4) {
    __shared__ unsigned snf;
    __shared__ bool last;
    if (threadIdx.x == 0) snf = 0u;
    __syncthreads();
    bool bad = false;
    if (v4) {  // triangle positions (n = 3 V), also written as 16-byte records
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n / 3;
             i += (int64_t)gridDim.x * blockDim.x) {
            const float a = __ldg(x + 3 * i), b = __ldg(x + 3 * i + 1), c = __ldg(x + 3 * i + 2);
            bad |= !finite1(a) || !finite1(b) || !finite1(c);
            v4[i] = make_float4(a, b, c, 0.f);
        }
    } else {
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            bad |= !finite1(__ldg(x + i));
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&snf, 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (snf) atomicOr(ctr + C_NF_ACC, 1u);
        __threadfence();
        last = atomicAdd(ctr + C_NF_DONE, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        ctr[C_NF_DONE] = 0u;
        ctr[C_NONFINITE] = atomicExch(ctr + C_NF_ACC, 0u);
    }
}

// ---------------------------------------------------------------- FP16 node records
// {min.xyz rounded down, max.xyz rounded up to FP16, escape}: 16 bytes per
// internal node for the front traversals (the FP32 records stay the master).
__global__ void k_node_fp16(int nint, const float4 *__restrict__ nrec, uint4 *nrec16) {
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nint; d += gridDim.x * blockDim.x) {
        const float4 lo = nrec[2 * d], hi = nrec[2 * d + 1];
        auto h = [](__half x) { return (unsigned)__half_as_ushort(x); };
        uint4 r;
        r.x = h(__float2half_rd(lo.x)) | (h(__float2half_rd(lo.y)) << 16);
        r.y = h(__float2half_rd(lo.z)) | (h(__float2half_ru(hi.x)) << 16);
        r.z = h(__float2half_ru(hi.y)) | (h(__float2half_ru(hi.z)) << 16);
        r.w = (unsigned)__float_as_int(hi.w);
        nrec16[d] = r;
    }
}

// ---------------------------------------------------------------- restructure
// calibrateLeafRangeMarks (LBvhRestructureKernels.cu:9-17)
__global__ void k_rs_leaf_marks(int T, const int *__restrict__ rtroot, const int *__restrict__ intmark,
                                const int2 *__restrict__ nrange, int *extrange) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        int rt = rtroot[i];
        if (rt != INT_MAX && intmark[rt] == 1) {
            atomicAdd(extrange + i, 1);
            atomicAdd(extrange + nrange[rt].y + 1, -1);
        }
    }
}
// calibrateRestrRoots (:19-35)
__global__ void k_rs_roots(int T, const int *__restrict__ rtroot, const int *__restrict__ intmark,
                           const int2 *__restrict__ nrange, int *rootmark, unsigned *ctr) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        int rt = rtroot[i];
        if (rt != INT_MAX && intmark[rt] == 1) {
            int2 rg = nrange[rt];
            atomicAdd(rootmark + i, rt);
            atomicAdd(rootmark + rg.y + 1, -rt);
            atomicAdd(ctr + C_RT_INTNODES, (unsigned)(rg.y - rg.x));
            atomicAdd(ctr + C_RT_SUBTREES, 1u);
        }
    }
}
__global__ void k_rs_flags(int T, const int *__restrict__ leafroot, unsigned *flag) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < T; s += gridDim.x * blockDim.x)
        flag[s] = leafroot[s] > 0 ? 1u : 0u;
}
// calcRestrMCs + selectPrimitives (:37-66): (subtree root, Morton) keys
__global__ void k_rs_select(int T, const int *__restrict__ leafroot, const unsigned *__restrict__ pos,
                            const int4 *__restrict__ sface, PrimSrc p,
                            const float *__restrict__ scene, unsigned long long *keys, int *task,
                            int *vals) {
    __shared__ float sc[6];
    if (threadIdx.x < 6) sc[threadIdx.x] = scene[threadIdx.x];
    __syncthreads();
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < T; s += gridDim.x * blockDim.x) {
        int rt = leafroot[s];
        if (rt > 0) {
            int4 f = sface[s];
            float4 lo, hi;
            face_box(p, f, lo, hi);
            unsigned q = pos[s];
            keys[q] = ((unsigned long long)(unsigned)rt << 32) | morton_box(lo, hi, sc);
            task[q] = s;
            vals[q] = s;
        }
    }
}
// For each restructured subtree R (root DFS id R > 0): the DFS id of the old
// parent of its leftmost leaf, i.e. the end of R's old left spine R, R + 1,
// ...  Read before the confined rebuild rewrites the links.  A complete cut
// of the old subtree holds exactly one node of that spine or the leftmost
// leaf itself, which is what an inter front's restructure keys on.
__global__ void k_rs_oldlast(int T, const int *__restrict__ leafroot, const float4 *__restrict__ lrec,
                             int *oldlast) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < T; s += gridDim.x * blockDim.x) {
        const int R = leafroot[s];
        if (R > 0 && (s == 0 || leafroot[s - 1] != R)) oldlast[R] = __float_as_int(lrec[2 * (size_t)s].w);
    }
}

// updatePrimMap (:68-77), applying the sort permutation: slot task[k]
// receives the primitive that sorts k-th inside its subtree.
__global__ void k_rs_gather(int nr, const int *__restrict__ sorted, const int4 *__restrict__ sface,
                            int4 *tmp) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nr; k += gridDim.x * blockDim.x)
        tmp[k] = sface[sorted[k]];
}
__global__ void k_rs_scatter(int nr, const int *__restrict__ task, const int4 *__restrict__ tmp,
                             const unsigned long long *__restrict__ keys, int4 *sface, int *primmap,
                             unsigned *code) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nr; k += gridDim.x * blockDim.x) {
        int s = task[k];
        int4 f = tmp[k];
        sface[s] = f;
        primmap[f.w] = s;
        code[s] = (unsigned)(keys[k] & 0xffffffffull);
    }
}
// calcRestrIntNodeOrders (:168-195), ids part: DFS ids inside each subtree slot
__global__ void k_rs_dfs(int nr, int T, const int *__restrict__ task, const int *__restrict__ leafroot,
                         const int2 *__restrict__ nrange, const unsigned *__restrict__ coff,
                         const int *__restrict__ clen, const int *__restrict__ posb,
                         const int *__restrict__ urx, int *dfs) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nr; k += gridDim.x * blockDim.x) {
        int s = task[k];
        int root = leafroot[s];
        if (s + 1 < T && leafroot[s + 1] == root) {
            int rxr = nrange[root].x, rx = urx[s];
            dfs[s] = root + (int)(coff[rx] - coff[rxr]) + clen[rx] - 1 - posb[s];
        }
    }
}
// calcRestrIntNodeOrders, link part: new escape links inside the subtrees.
// The subtree root keeps its DFS id; when it is a left child the chain of
// its leftmost leaf continues above it, so that leaf's link is unchanged.
__global__ void k_rs_lca(int nr, const int *__restrict__ task, const int *__restrict__ leafroot,
                         const int2 *__restrict__ nrange, const int4 *__restrict__ topo,
                         const unsigned *__restrict__ coff, const int *__restrict__ clen, int *lca) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nr; k += gridDim.x * blockDim.x) {
        int s = task[k];
        int root = leafroot[s];
        int rxr = nrange[root].x;
        if (clen[s] > 0) {
            bool keep = (s == rxr) && !(topo[root].w & 4);
            if (!keep) lca[s] = (root + (int)(coff[s] - coff[rxr])) << 1;
        } else {
            lca[s] = (s << 1) | 1;
        }
    }
}
// reorderRestrIntNodes (:197-215) and the leaf links of restructured leaves
__global__ void k_rs_write(int nr, int T, const int *__restrict__ task, const int *__restrict__ leafroot,
                           Climb c, const int *__restrict__ dfs, const int *__restrict__ lca,
                           float4 *nrec, int4 *topo, int2 *nrange, float4 *lrec) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nr; k += gridDim.x * blockDim.x) {
        int s = task[k];
        reinterpret_cast<float *>(lrec)[8 * (size_t)s + 3] = __int_as_float(dfs[c.ulpar[s]]);
        reinterpret_cast<float *>(lrec)[8 * (size_t)s + 7] = __int_as_float(lca[s + 1]);
        if (s + 1 < T && leafroot[s + 1] == leafroot[s]) {
            int u = s, d = dfs[u];
            unsigned m = c.umark[u];
            int lc = c.ulc[u], rc = c.urc[u], p = c.upar[u];
            int rx = c.urx[u], ry = c.ury[u];
            int par = p < 0 ? topo[d].z : dfs[p];
            topo[d] = make_int4((m & 1u) ? lc : dfs[lc], (m & 2u) ? rc : dfs[rc], par, (int)m);
            nrange[d] = make_int2(rx, ry);
            float4 lo = c.ubox[2 * u], hi = c.ubox[2 * u + 1];
            lo.w = __int_as_float(rx | ((m & 1u) ? (int)0x80000000 : 0));  // bit 31: the left child is leaf rx
            hi.w = __int_as_float(lca[ry + 1]);
            nrec[2 * d] = lo;
            nrec[2 * d + 1] = hi;
        }
    }
}

// checkFrontQuality's marking step (BvttFrontGenerateKernels.cu:45-47) for
// subtrees chosen by the caller
__global__ void k_mark_roots(int n, int nint, const int *__restrict__ roots, const int2 *__restrict__ nrange,
                             int *intrange, int *rtroot) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int i = roots[k];
        if (i < 0 || i >= nint) continue;
        int2 r = nrange[i];
        atomicAdd(intrange + i, 1);
        atomicAdd(intrange + i + r.y - r.x, -1);
        atomicMin(rtroot + r.x, i);
    }
}
__global__ void k_fill(int n, int *p, int v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// Export helpers
__global__ void k_export(int T, const float4 *__restrict__ nrec, const int4 *__restrict__ topo,
                         const int2 *__restrict__ nrange, const float4 *__restrict__ lrec,
                         const int4 *__restrict__ sface, const int *__restrict__ lca,
                         int *inode, float *ibox, int *leaf, float *lbox) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        if (i < T - 1) {
            int4 t = topo[i];
            int2 r = nrange[i];
            inode[6 * i + 0] = t.x; inode[6 * i + 1] = t.y; inode[6 * i + 2] = t.z;
            inode[6 * i + 3] = t.w; inode[6 * i + 4] = r.x; inode[6 * i + 5] = r.y;
            float4 lo = nrec[2 * i], hi = nrec[2 * i + 1];
            ibox[6 * i + 0] = lo.x; ibox[6 * i + 1] = lo.y; ibox[6 * i + 2] = lo.z;
            ibox[6 * i + 3] = hi.x; ibox[6 * i + 4] = hi.y; ibox[6 * i + 5] = hi.z;
        }
        float4 lo = lrec[2 * i], hi = lrec[2 * i + 1];
        int l = lca[i];
        leaf[4 * i + 0] = sface[i].w;
        leaf[4 * i + 1] = __float_as_int(lo.w);
        leaf[4 * i + 2] = (l & 1) ? 7 : 3;
        leaf[4 * i + 3] = l;
        lbox[6 * i + 0] = lo.x; lbox[6 * i + 1] = lo.y; lbox[6 * i + 2] = lo.z;
        lbox[6 * i + 3] = hi.x; lbox[6 * i + 4] = hi.y; lbox[6 * i + 5] = hi.z;
    }
}

}  // namespace

// ====================================================================== host
Profiler::~Profiler() {
    for (auto &p : pending_) { pool_.push_back(p.a); pool_.push_back(p.b); }
    for (cudaEvent_t e : open_) if (e) pool_.push_back(e);
    for (cudaEvent_t e : pool_) cudaEventDestroy(e);
}

cudaEvent_t Profiler::get() {
    if (!pool_.empty()) {
        cudaEvent_t e = pool_.back();
        pool_.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void Profiler::begin(int stage, cudaStream_t s) {
    if (open_[stage]) pool_.push_back(open_[stage]);
    open_[stage] = get();
    cudaEventRecord(open_[stage], s);
}

void Profiler::end(int stage, cudaStream_t s) {
    if (!open_[stage]) return;
    cudaEvent_t b = get();
    cudaEventRecord(b, s);
    pending_.push_back({stage, open_[stage], b});
    open_[stage] = nullptr;
}

bvhcd_status Profiler::read(double *ms, int64_t *calls, bool reset) {
    for (auto &p : pending_) {
        cudaError_t e = cudaEventSynchronize(p.b);
        if (e != cudaSuccess) return cuda_status(e);
        float t = 0.f;
        e = cudaEventElapsedTime(&t, p.a, p.b);
        if (e != cudaSuccess) return cuda_status(e);
        ms_[p.stage] += t;
        calls_[p.stage] += 1;
        pool_.push_back(p.a);
        pool_.push_back(p.b);
    }
    pending_.clear();
    for (int i = 0; i < BVHCD_STAGE_COUNT; i++) {
        if (ms) ms[i] = ms_[i];
        if (calls) calls[i] = calls_[i];
        if (reset) { ms_[i] = 0; calls_[i] = 0; }
    }
    return BVHCD_OK;
}

LBvh::~LBvh() {
    DBuf *bufs[] = {&verts_, &faces_, &nrec_, &lrec_, &topo_, &nrange_, &lca_, &sface_, &primmap_,
                    &code_, &refit_flag_, &keys_, &vals_, &keys2_, &vals2_, &k64_, &k64b_, &metric_,
                    &ulc_, &urc_, &upar_, &urx_, &ury_, &umark_, &ubox_, &uflag_, &posb_, &clen_,
                    &coff_, &dfs_, &ulpar_, &scene_, &partial_, &scratch_, &task_, &tmpface_,
                    &intrange_, &rtroot_, &intmark_, &extrange_, &extmark_, &leafroot_, &rs_oldlast_, &flagbuf_,
                    &ctr_, &scene_of_, &leafscene_, &sbox_, &tiles_, &nrec16_, &split_, &cross_, &topk_,
                    &plan_, &top_, &gbox_, &height_, &llist_, &lhdr_, &tlist_,
                    &thdr_, &llink_, &tlink_, &lexp_, &nexp_, &lexport_, &gext_, &uheight_};
    for (DBuf *b : bufs) b->release();
    for (int k = 0; k < 2; k++) {
        stage_[k].release();
        if (stage_ready_[k]) cudaEventDestroy(stage_ready_[k]);
        if (stage_free_[k]) cudaEventDestroy(stage_free_[k]);
    }
    if (h_ctr_) cudaFreeHost(h_ctr_);
}

// Double-buffered position upload (see bvhcd_bvh_stage_positions).  Buffer k
// is free once the stream that used it has passed the start of the maintain
// that took the other buffer (stage_free_[k], recorded there).
bvhcd_status LBvh::stage_positions(const float *host, int nv, cudaStream_t copy, const float **staged) {
    if (!staged || nv < 0 || (nv > 0 && !host)) return BVHCD_INVALID_ARG;
    if (stage_pending_) return BVHCD_NOT_READY;
    for (int k = 0; k < 2; k++) {
        if (!stage_ready_[k]) BV_TRY(cudaEventCreateWithFlags(&stage_ready_[k], cudaEventDisableTiming));
        if (!stage_free_[k]) BV_TRY(cudaEventCreateWithFlags(&stage_free_[k], cudaEventDisableTiming));
    }
    const int k = stage_next_;
    const size_t bytes = sizeof(float) * 3 * (size_t)(nv > 0 ? nv : 1);
    if (stage_[k].bytes < bytes) {
        BV_TRY(cudaStreamSynchronize(copy));
        BV_TRY(cudaEventSynchronize(stage_free_[k]));
        stage_[k].release();
        BV_TRY(stage_[k].reserve(bytes));
    }
    BV_TRY(cudaStreamWaitEvent(copy, stage_free_[k], 0));
    if (nv > 0)
        BV_TRY(cudaMemcpyAsync(stage_[k].p, host, sizeof(float) * 3 * (size_t)nv, cudaMemcpyHostToDevice, copy));
    BV_TRY(cudaEventRecord(stage_ready_[k], copy));
    *staged = stage_[k].as<float>();
    stage_next_ = 1 - k;
    stage_pending_ = true;
    return BVHCD_OK;
}

bvhcd_status LBvh::init() {
    if (cfg_.prim_capacity < 0 || cfg_.vert_capacity < 0) return BVHCD_INVALID_ARG;
    BV_TRY(ctr_.reserve(sizeof(unsigned) * C_NUM));
    BV_TRY(cudaMemset(ctr_.p, 0, sizeof(unsigned) * C_NUM));
    BV_TRY(scene_.reserve(64));
    BV_TRY(cudaMallocHost(&h_ctr_, sizeof(unsigned) * C_NUM));
    int T = cfg_.prim_capacity > 0 ? cfg_.prim_capacity : 1;
    int V = cfg_.vert_capacity > 0 ? cfg_.vert_capacity : 3 * T;
    return ensure_capacity(T, V);
}

bvhcd_status LBvh::ensure_capacity(int T, int V) {
    if (V > capV_) {
        BV_TRY(verts_.reserve(sizeof(float) * 3 * (size_t)V));
        BV_TRY(verts4_.reserve(sizeof(float4) * (size_t)V));
        capV_ = V;
    }
    if (T <= capT_) return BVHCD_OK;
    size_t n = (size_t)T + 2;
    BV_TRY(faces_.reserve(sizeof(int) * 3 * n));
    BV_TRY(nrec_.reserve(sizeof(float4) * 2 * n));
    BV_TRY(lrec_.reserve(sizeof(float4) * 2 * n));
    BV_TRY(topo_.reserve(sizeof(int4) * n));
    BV_TRY(nrange_.reserve(sizeof(int2) * n));
    BV_TRY(lca_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(sface_.reserve(sizeof(int4) * n));
    BV_TRY(primmap_.reserve(sizeof(int) * n));
    BV_TRY(code_.reserve(sizeof(unsigned) * n));
    BV_TRY(refit_flag_.reserve(sizeof(unsigned) * n));
    BV_TRY(split_.reserve(sizeof(int) * n));
    BV_TRY(cross_.reserve(sizeof(unsigned) * n));
    BV_TRY(topk_.reserve(sizeof(unsigned) * n));
    BV_TRY(plan_.reserve(sizeof(int4) * n));
    BV_TRY(top_.reserve(sizeof(int4) * n));
    BV_TRY(gbox_.reserve(sizeof(float) * 6 * n));
    BV_TRY(height_.reserve(sizeof(int) * n));
    BV_TRY(uheight_.reserve(sizeof(int) * n));
    BV_TRY(llist_.reserve(sizeof(int4) * (n + kRefitW)));
    BV_TRY(lhdr_.reserve(sizeof(int) * kLevelHdr * (n / kRefitW + 2)));
    BV_TRY(tlist_.reserve(sizeof(int4) * n));
    BV_TRY(thdr_.reserve(sizeof(int) * kLevelHdr));
    BV_TRY(llink_.reserve(sizeof(int2) * n));
    BV_TRY(lexp_.reserve(sizeof(int) * n));
    BV_TRY(nexp_.reserve(sizeof(int) * n));
    BV_TRY(lexport_.reserve(sizeof(int4) * (n + kRefitW)));
    BV_TRY(gext_.reserve(sizeof(float) * 12 * n));
    BV_TRY(tlink_.reserve(sizeof(int2) * n));
    BV_TRY(keys_.reserve(sizeof(unsigned) * n));
    BV_TRY(vals_.reserve(sizeof(int) * n));
    BV_TRY(keys2_.reserve(sizeof(unsigned) * n));
    BV_TRY(vals2_.reserve(sizeof(int) * n));
    BV_TRY(k64_.reserve(sizeof(unsigned long long) * n));
    BV_TRY(k64b_.reserve(sizeof(unsigned long long) * n));
    BV_TRY(metric_.reserve(sizeof(int) * n));
    BV_TRY(ulc_.reserve(sizeof(int) * n));
    BV_TRY(urc_.reserve(sizeof(int) * n));
    BV_TRY(upar_.reserve(sizeof(int) * n));
    BV_TRY(urx_.reserve(sizeof(int) * n));
    BV_TRY(ury_.reserve(sizeof(int) * n));
    BV_TRY(umark_.reserve(sizeof(unsigned) * n));
    BV_TRY(ubox_.reserve(sizeof(float4) * 2 * n));
    BV_TRY(uflag_.reserve(sizeof(unsigned) * n));
    BV_TRY(posb_.reserve(sizeof(int) * n));
    BV_TRY(clen_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(coff_.reserve(sizeof(unsigned) * (n + 1)));
    BV_TRY(dfs_.reserve(sizeof(int) * n));
    BV_TRY(ulpar_.reserve(sizeof(int) * n));
    BV_TRY(partial_.reserve(sizeof(float) * 6 * 4096));
    size_t scr = sort_scratch_bytes((int64_t)n);
    size_t scr2 = scan_scratch_bytes((int64_t)n + 1);
    BV_TRY(scratch_.reserve(scr > scr2 ? scr : scr2));
    BV_TRY(task_.reserve(sizeof(int) * n));
    BV_TRY(tmpface_.reserve(sizeof(int4) * n));
    BV_TRY(intrange_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(rtroot_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(intmark_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(extrange_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(extmark_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(leafroot_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(rs_oldlast_.reserve(sizeof(int) * (n + 1)));
    BV_TRY(flagbuf_.reserve(sizeof(unsigned) * (n + 1)));
    capT_ = T;
    return BVHCD_OK;
}

Tree LBvh::tree() const {
    Tree t;
    t.nrec = nrec_.as<float4>();
    t.lrec = lrec_.as<float4>();
    t.topo = topo_.as<int4>();
    t.nrange = nrange_.as<int2>();
    t.lca = lca_.as<int>();
    t.sface = sface_.as<int4>();
    t.primmap = primmap_.as<int>();
    t.code = code_.as<unsigned>();
    t.nrec16 = cfg_.node_box_fp16 ? nrec16_.as<uint4>() : nullptr;
    t.T = T_;
    return t;
}

bvhcd_status LBvh::upload(const bvhcd_scene &sc, cudaStream_t s) {
    if (sc.num_faces < 0 || sc.num_vertices < 0) return BVHCD_INVALID_ARG;
    if (sc.num_faces > 0 && (!sc.pos || !sc.faces)) return BVHCD_INVALID_ARG;
    bvhcd_status st = ensure_capacity(sc.num_faces, sc.num_vertices);
    if (st != BVHCD_OK) return st;
    if (sc.on_device) {
        if (is_staged(sc.pos)) {
            const int k = sc.pos == stage_[0].as<float>() ? 0 : 1;
            BV_TRY(cudaStreamWaitEvent(s, stage_ready_[k], 0));
            BV_TRY(cudaEventRecord(stage_free_[1 - k], s));
            stage_pending_ = false;
        }
        vptr_ = sc.pos;
        if (fptr_ != sc.faces || !sc.faces_static) faces_epoch_++;
        fptr_ = sc.faces;
    } else {
        if (sc.num_vertices)
            BV_TRY(cudaMemcpyAsync(verts_.p, sc.pos, sizeof(float) * 3 * (size_t)sc.num_vertices,
                                   cudaMemcpyHostToDevice, s));
        bool same = sc.faces_static && built_ && fptr_ == faces_.as<int>() && T_ == sc.num_faces;
        if (!same) faces_epoch_++;
        if (!same && sc.num_faces)
            BV_TRY(cudaMemcpyAsync(faces_.p, sc.faces, sizeof(int) * 3 * (size_t)sc.num_faces,
                                   cudaMemcpyHostToDevice, s));
        vptr_ = verts_.as<float>();
        fptr_ = faces_.as<int>();
    }
    // a tree built over a box scene is rebuilt for triangles
    if (built_ && (sc.num_faces != T_ || box_input_)) built_ = false;
    box_input_ = false;
    bptr_ = nullptr;
    T_ = sc.num_faces;
    V_ = sc.num_vertices;
    return BVHCD_OK;
}

// ARCSimSceneData input (LBvhFixedDeformable::maintain(scheme, const
// ARCSimSceneData&), LBvhFixedDeformable.cu:89-112): the primitives' boxes
// are given.  FP64 boxes are rounded outward, so the FP32 box the tree holds
// contains the given one (the reference converts to nearest,
// buildPrimitivesARCSim / refitExtNodeARCSim, LBvhBuildKernels.cu:35-50,
// LBvhUpdateKernels.cu:11-22).
bvhcd_status LBvh::upload_boxes(const bvhcd_box_scene &sc, cudaStream_t s) {
    if (sc.num_faces < 0) return BVHCD_INVALID_ARG;
    if (sc.num_faces > 0 && (!sc.boxes || !sc.faces)) return BVHCD_INVALID_ARG;
    bvhcd_status st = ensure_capacity(sc.num_faces, 0);
    if (st != BVHCD_OK) return st;
    const size_t T = (size_t)sc.num_faces;
    const bool convert = sc.boxes_f64 != 0;
    if (convert || !sc.on_device) BV_TRY(boxes_.reserve(sizeof(float) * 6 * (T > 0 ? T : 1)));
    if (sc.on_device) {
        if (fptr_ != sc.faces || !sc.faces_static) faces_epoch_++;
        fptr_ = sc.faces;
        if (convert && T) {
            k_boxes_f64<<<grid_for((int64_t)(6 * T)), kThreads, 0, s>>>((int64_t)(6 * T),
                                                                       static_cast<const double *>(sc.boxes),
                                                                       boxes_.as<float>()); note_launch();
            BV_TRY(cudaGetLastError());
        }
        bptr_ = convert ? boxes_.as<float>() : static_cast<const float *>(sc.boxes);
    } else {
        bool same = sc.faces_static && built_ && fptr_ == faces_.as<int>() && T_ == sc.num_faces;
        if (!same) faces_epoch_++;
        if (!same && T)
            BV_TRY(cudaMemcpyAsync(faces_.p, sc.faces, sizeof(int) * 3 * T, cudaMemcpyHostToDevice, s));
        fptr_ = faces_.as<int>();
        if (convert && T) {
            BV_TRY(boxes64_.reserve(sizeof(double) * 6 * T));
            BV_TRY(cudaMemcpyAsync(boxes64_.p, sc.boxes, sizeof(double) * 6 * T, cudaMemcpyHostToDevice, s));
            k_boxes_f64<<<grid_for((int64_t)(6 * T)), kThreads, 0, s>>>((int64_t)(6 * T), boxes64_.as<double>(),
                                                                       boxes_.as<float>()); note_launch();
            BV_TRY(cudaGetLastError());
        } else if (T) {
            BV_TRY(cudaMemcpyAsync(boxes_.p, sc.boxes, sizeof(float) * 6 * T, cudaMemcpyHostToDevice, s));
        }
        bptr_ = boxes_.as<float>();
    }
    // a tree built over triangles is rebuilt for boxes
    if (built_ && (sc.num_faces != T_ || !box_input_)) built_ = false;
    box_input_ = true;
    vptr_ = nullptr;
    T_ = sc.num_faces;
    V_ = 0;
    return BVHCD_OK;
}

bvhcd_status LBvh::scene_box(cudaStream_t s) {
    int g = (int)grid_for(T_);
    if (g > 4096) g = 4096;
    k_box_partial<<<g, kThreads, 0, s>>>(T_, src(), partial_.as<float>()); note_launch();
    k_box_final<<<1, kThreads, 0, s>>>(g, partial_.as<float>(), scene_.as<float>()); note_launch();
    return cuda_status(cudaGetLastError());
}

static Climb make_climb(const DBuf &ulc, const DBuf &urc, const DBuf &upar, const DBuf &urx,
                        const DBuf &ury, const DBuf &umark, const DBuf &ubox, const DBuf &uflag,
                        const DBuf &posb, const DBuf &clen, const DBuf &ulpar, const DBuf &uheight) {
    Climb c;
    c.ulc = ulc.as<int>(); c.urc = urc.as<int>(); c.upar = upar.as<int>();
    c.urx = urx.as<int>(); c.ury = ury.as<int>(); c.umark = umark.as<unsigned>();
    c.ubox = ubox.as<float4>(); c.uflag = uflag.as<unsigned>(); c.posb = posb.as<int>();
    c.clen = clen.as<int>(); c.ulpar = ulpar.as<int>(); c.uheight = uheight.as<int>();
    return c;
}

bvhcd_status LBvh::build(cudaStream_t s) {
    StageScope prof_scope(&prof_, BVHCD_STAGE_BVH_BUILD, s);
    const int T = T_;
    built_ = false;
    // a new topology: the accumulated box motion starts again
    BV_TRY(cudaMemsetAsync(ctr_.as<unsigned>() + C_DELTA, 0, 2 * sizeof(unsigned), s));
    if (T == 0) { built_ = true; return BVHCD_OK; }
    int *leafscene = nullptr;
    if (S_ > 1) {
        // a forest of S_ scenes: per-scene boxes, (scene, code) keys
        if (T != h_off_[S_]) return BVHCD_INVALID_ARG;
        k_sbox_init<<<1, kThreads, 0, s>>>(S_, sbox_.as<float>()); note_launch();
        k_sbox_tiles<<<ntiles_, kThreads, 0, s>>>(tiles_.as<int4>(), src(), sbox_.as<float>()); note_launch();
        k_morton_seg<<<grid_for(T), kThreads, 0, s>>>(T, src(), scene_of_.as<int>(), sbox_.as<float>(),
                                                      k64_.as<unsigned long long>(), vals_.as<int>()); note_launch();
        int sbits = 0;
        while ((1 << sbits) < S_) sbits++;
        BV_TRY(radix_sort_u64(k64_.as<unsigned long long>(), vals_.as<int>(), k64b_.as<unsigned long long>(),
                              vals2_.as<int>(), T, 30 + sbits, scratch_.p, s));
        leafscene = leafscene_.as<int>();
        k_leaves_seg<<<grid_for(T), kThreads, 0, s>>>(T, k64_.as<unsigned long long>(), vals_.as<int>(), src(),
                                                      sface_.as<int4>(), primmap_.as<int>(),
                                                      code_.as<unsigned>(), metric_.as<int>(),
                                                      lrec_.as<float4>(), leafscene); note_launch();
    } else {
        bvhcd_status st = scene_box(s);
        if (st != BVHCD_OK) return st;
        k_morton<<<grid_for(T), kThreads, 0, s>>>(T, src(), scene_.as<float>(), keys_.as<unsigned>(),
                                                  vals_.as<int>()); note_launch();
        BV_TRY(radix_sort_u32(keys_.as<unsigned>(), vals_.as<int>(), keys2_.as<unsigned>(), vals2_.as<int>(),
                              T, 30, scratch_.p, s));
        k_leaves<<<grid_for(T), kThreads, 0, s>>>(T, keys_.as<unsigned>(), vals_.as<int>(), src(),
                                                  sface_.as<int4>(), primmap_.as<int>(), code_.as<unsigned>(),
                                                  metric_.as<int>(), lrec_.as<float4>()); note_launch();
        if (T == 1) {
            // a single leaf: no internal node, lca = {leaf 0, end}, no parent
            k_single_leaf<<<1, 32, 0, s>>>(lca_.as<int>(), lrec_.as<float4>()); note_launch();
            BV_TRY(cudaGetLastError());
            built_ = true;
            topo_epoch_++;
            return refit_plan(s, true);
        }
    }
    Climb c = make_climb(ulc_, urc_, upar_, urx_, ury_, umark_, ubox_, uflag_, posb_, clen_, ulpar_, uheight_);
    BV_TRY(cudaMemsetAsync(uflag_.p, 0, sizeof(unsigned) * (size_t)T, s));
    BV_TRY(cudaMemsetAsync(clen_.as<int>() + T, 0, sizeof(int), s));
    if (leafscene)
        k_climb<true><<<grid_for(T), kThreads, 0, s>>>(T, T, nullptr, leafscene, metric_.as<int>(),
                                                       lrec_.as<float4>(), nullptr, c);
    else
        k_climb<false><<<grid_for(T), kThreads, 0, s>>>(T, T, nullptr, nullptr, metric_.as<int>(),
                                                        lrec_.as<float4>(), nullptr, c);
    note_launch();
    BV_TRY(scan_u32(clen_.as<unsigned>(), coff_.as<unsigned>(), T + 1, false, nullptr, scratch_.p, s));
    k_dfs_ids<<<grid_for(T - 1), kThreads, 0, s>>>(T - 1, urx_.as<int>(), posb_.as<int>(),
                                                   coff_.as<unsigned>(), clen_.as<int>(), leafscene,
                                                   dfs_.as<int>()); note_launch();
    k_leaf_links<<<grid_for(T), kThreads, 0, s>>>(T, coff_.as<unsigned>(), clen_.as<int>(), ulpar_.as<int>(),
                                                  dfs_.as<int>(), leafscene, lca_.as<int>(),
                                                  lrec_.as<float4>()); note_launch();
    k_write_nodes<<<grid_for(T - 1), kThreads, 0, s>>>(T - 1, T, c, dfs_.as<int>(), coff_.as<unsigned>(),
                                                       clen_.as<int>(), leafscene, nrec_.as<float4>(),
                                                       topo_.as<int4>(), nrange_.as<int2>(), height_.as<int>()); note_launch();
    BV_TRY(cudaGetLastError());
    built_ = true;
    topo_epoch_++;
    return refit_plan(s, true);
}

bvhcd_status LBvh::copy_state_from(const LBvh &src, cudaStream_t s) {
    if (&src == this) return BVHCD_OK;
    if (src.cfg_.enable_restr != cfg_.enable_restr || src.cfg_.node_box_fp16 != cfg_.node_box_fp16)
        return BVHCD_INVALID_ARG;
    const DBuf *from[] = {&src.verts_, &src.verts4_, &src.faces_, &src.boxes_, &src.nrec_, &src.lrec_, &src.topo_, &src.nrange_, &src.lca_,
                          &src.sface_, &src.primmap_, &src.code_, &src.refit_flag_, &src.intrange_, &src.rtroot_,
                          &src.intmark_, &src.extrange_, &src.extmark_, &src.leafroot_, &src.ctr_,
                          &src.scene_of_, &src.leafscene_, &src.sbox_, &src.tiles_, &src.scene_, &src.nrec16_,
                          &src.split_, &src.cross_, &src.topk_, &src.plan_, &src.top_,
                          &src.height_, &src.llist_, &src.lhdr_, &src.tlist_, &src.thdr_,
                          &src.llink_, &src.tlink_, &src.lexport_, &src.gext_};
    DBuf *to[] = {&verts_, &verts4_, &faces_, &boxes_, &nrec_, &lrec_, &topo_, &nrange_, &lca_, &sface_, &primmap_, &code_,
                  &refit_flag_, &intrange_, &rtroot_, &intmark_, &extrange_, &extmark_, &leafroot_, &ctr_,
                  &scene_of_, &leafscene_, &sbox_, &tiles_, &scene_, &nrec16_, &split_, &cross_, &topk_,
                  &plan_, &top_, &height_, &llist_, &lhdr_, &tlist_, &thdr_, &llink_, &tlink_,
                  &lexport_, &gext_};
    bvhcd_status st = ensure_capacity(src.capT_, src.capV_);
    if (st != BVHCD_OK) return st;
    for (size_t k = 0; k < sizeof(to) / sizeof(to[0]); k++) BV_TRY(to[k]->copy_from(*from[k], s));
    T_ = src.T_; V_ = src.V_;
    built_ = src.built_; updated_ = src.updated_;
    opt_tag_ = src.opt_tag_; rt_subtrees_ = src.rt_subtrees_; rt_intnodes_ = src.rt_intnodes_;
    // input read in place stays where it is; an owned copy maps to this handle's copy
    vptr_ = src.vptr_ == src.verts_.as<float>() ? verts_.as<float>() : src.vptr_;
    fptr_ = src.fptr_ == src.faces_.as<int>() ? faces_.as<int>() : src.fptr_;
    bptr_ = src.bptr_ && src.bptr_ == src.boxes_.as<float>() ? boxes_.as<float>() : src.bptr_;
    box_input_ = src.box_input_;
    S_ = src.S_; ntiles_ = src.ntiles_; h_off_ = src.h_off_;
    epoch_++;
    topo_epoch_++;
    faces_epoch_++;
    return cuda_status(cudaGetLastError());
}

// Batched scenes (see the forest kernels above).  The layout is static: the
// per-triangle scene ids and the box tiles are uploaded once here.
bvhcd_status LBvh::set_scenes(int S, const int32_t *off) {
    if (S < 1 || !off || off[0] != 0) return BVHCD_INVALID_ARG;
    if (S > 1 && restr_enabled()) return BVHCD_INVALID_ARG;
    if (S > (1 << 22)) return BVHCD_INVALID_ARG;
    for (int k = 0; k < S; k++)
        if (off[k + 1] - off[k] < (S > 1 ? 2 : 0)) return BVHCD_INVALID_ARG;
    const int T = off[S];
    std::vector<int> scene_of((size_t)T);
    std::vector<int4> tiles;
    for (int k = 0; k < S; k++) {
        for (int t = off[k]; t < off[k + 1]; t++) scene_of[(size_t)t] = k;
        for (int t = off[k]; t < off[k + 1]; t += kBoxTile)
            tiles.push_back(make_int4(k, t, t + kBoxTile < off[k + 1] ? t + kBoxTile : off[k + 1], 0));
    }
    h_off_.assign(off, off + S + 1);
    S_ = S;
    epoch_++;
    built_ = false;
    if (S == 1) return BVHCD_OK;
    BV_TRY(scene_of_.reserve(sizeof(int) * (size_t)(T > 0 ? T : 1)));
    BV_TRY(leafscene_.reserve(sizeof(int) * (size_t)(T > 0 ? T : 1)));
    BV_TRY(sbox_.reserve(sizeof(float) * 6 * (size_t)S));
    BV_TRY(tiles_.reserve(sizeof(int4) * tiles.size()));
    BV_TRY(cudaMemcpy(scene_of_.p, scene_of.data(), sizeof(int) * (size_t)T, cudaMemcpyHostToDevice));
    BV_TRY(cudaMemcpy(tiles_.p, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice));
    ntiles_ = (int)tiles.size();
    return BVHCD_OK;
}

// The refit plan of the current topology (see k_heights, k_plan_split,
// k_plan_write, k_plan_local, k_plan_top).  heights_known: the build's climb
// has written every node's height already.
bvhcd_status LBvh::refit_plan(cudaStream_t s, bool heights_known) {
    const int nint = T_ - S_;  // internal nodes: one tree of n - 1 per scene of n leaves
    const int nb = (T_ + kRefitW - 1) / kRefitW;
    if (T_ <= 0) return BVHCD_OK;
    BV_TRY(cudaMemsetAsync(lexp_.p, 0xFF, sizeof(int) * (size_t)T_, s));
    BV_TRY(cudaMemsetAsync(ctr_.as<unsigned>() + C_REFIT_DONE, 0, sizeof(unsigned), s));
    if (nint > 0) {
        BV_TRY(cudaMemsetAsync(nexp_.p, 0xFF, sizeof(int) * (size_t)nint, s));
        BV_TRY(cudaMemsetAsync(plan_.p, 0xFF, sizeof(int4) * (size_t)T_, s));
        if (!heights_known) {
            BV_TRY(cudaMemsetAsync(height_.p, 0, sizeof(int) * (size_t)nint, s));
            BV_TRY(cudaMemsetAsync(refit_flag_.p, 0, sizeof(unsigned) * (size_t)nint, s));
            k_heights<<<grid_for(T_), kThreads, 0, s>>>(T_, lrec_.as<float4>(), topo_.as<int4>(),
                                                        refit_flag_.as<unsigned>(), height_.as<int>()); note_launch();
        }
        k_plan_split<<<grid_for(nint), kThreads, 0, s>>>(nint, topo_.as<int4>(), nrange_.as<int2>(),
                                                         split_.as<int>(), cross_.as<unsigned>()); note_launch();
        BV_TRY(scan_u32(cross_.as<unsigned>(), topk_.as<unsigned>(), nint, false, ctr_.as<unsigned>() + C_TOPK,
                        scratch_.p, s));
        k_plan_write<<<grid_for(nint), kThreads, 0, s>>>(nint, topo_.as<int4>(), split_.as<int>(),
                                                         cross_.as<unsigned>(), topk_.as<unsigned>(),
                                                         height_.as<int>(), plan_.as<int4>(), top_.as<int4>(),
                                                         lexp_.as<int>(), nexp_.as<int>(), gext_.as<float>()); note_launch();
    }
    k_plan_local<<<nb, kRefitThreads, 0, s>>>(T_, plan_.as<int4>(), lrec_.as<float4>(), nrec_.as<float4>(),
                                               lexp_.as<int>(), nexp_.as<int>(), llist_.as<int4>(), llink_.as<int2>(),
                                               lexport_.as<int4>(), lhdr_.as<int>()); note_launch();
    if (nb > 1) {
        k_plan_top<<<1, kRefitThreads, 0, s>>>(ctr_.as<unsigned>(), top_.as<int4>(), nrec_.as<float4>(),
                                                tlist_.as<int4>(), tlink_.as<int2>(), thdr_.as<int>()); note_launch();
    }
    return cuda_status(cudaGetLastError());
}

bvhcd_status LBvh::refit(cudaStream_t s) {
    StageScope prof_scope(&prof_, BVHCD_STAGE_BVH_REFIT, s);
    const int T = T_;
    if (T == 0) {
        BV_TRY(cudaMemsetAsync(ctr_.as<unsigned>() + C_NONFINITE, 0, sizeof(unsigned), s));
        return BVHCD_OK;
    }
    static const bool attrs = [] {
        cudaFuncSetAttribute(k_refit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLocalSmem);
        return true;
    }();
    (void)attrs;
    RefitTop g;
    g.top = top_.as<int4>();
    g.tlist = tlist_.as<int4>();
    g.tlink = tlink_.as<int2>();
    g.thdr = thdr_.as<int>();
    g.gext = gext_.as<float>();
    g.gbox = gbox_.as<float>();
    g.done = ctr_.as<unsigned>() + C_REFIT_DONE;
    g.delta = ctr_.as<unsigned>() + C_DELTA;
    g.motion = ctr_.as<unsigned>() + C_MOTION;
    g.nf_acc = ctr_.as<unsigned>() + C_NF_ACC;
    g.nonfinite = ctr_.as<unsigned>() + C_NONFINITE;
    g.v4 = box_input_ ? nullptr : verts4_.as<float4>();
    g.V = V_;
    const int nb = (T + kRefitW - 1) / kRefitW;
    k_refit<<<nb, kRefitThreads, kLocalSmem, s>>>(T, sface_.as<int4>(), src(), plan_.as<int4>(), llist_.as<int4>(),
                                                  llink_.as<int2>(), lexport_.as<int4>(), lhdr_.as<int>(),
                                                  lrec_.as<float4>(), nrec_.as<float4>(), gext_.as<float>(), g); note_launch();
    return cuda_status(cudaGetLastError());
}

// LBvhFixedDeformable::restructure (LBvhFixedDeformable.cu:210-352)
bvhcd_status LBvh::restructure(cudaStream_t s) {
    StageScope prof_scope(&prof_, BVHCD_STAGE_BVH_RESTRUCTURE, s);
    const int T = T_, I = T - 1;
    unsigned *ctr = ctr_.as<unsigned>();
    // 1 int node marks, 2-3 leaf range marks, 4 subtree roots
    BV_TRY(scan_i32(intrange_.as<int>(), intmark_.as<int>(), I, true, nullptr, scratch_.p, s));
    BV_TRY(cudaMemsetAsync(extrange_.p, 0, sizeof(int) * (size_t)(T + 1), s));
    k_rs_leaf_marks<<<grid_for(T), kThreads, 0, s>>>(T, rtroot_.as<int>(), intmark_.as<int>(),
                                                     nrange_.as<int2>(), extrange_.as<int>()); note_launch();
    BV_TRY(scan_i32(extrange_.as<int>(), extmark_.as<int>(), T + 1, true, nullptr, scratch_.p, s));
    BV_TRY(cudaMemsetAsync(extrange_.p, 0, sizeof(int) * (size_t)(T + 1), s));
    BV_TRY(cudaMemsetAsync(ctr + C_RT_SUBTREES, 0, sizeof(unsigned) * 2, s));
    k_rs_roots<<<grid_for(T), kThreads, 0, s>>>(T, rtroot_.as<int>(), intmark_.as<int>(), nrange_.as<int2>(),
                                                extrange_.as<int>(), ctr); note_launch();
    BV_TRY(cudaMemcpyAsync(h_ctr_ + C_RT_SUBTREES, ctr + C_RT_SUBTREES, sizeof(unsigned) * 2,
                           cudaMemcpyDeviceToHost, s));
    BV_TRY(cudaStreamSynchronize(s));
    rt_subtrees_ = (int)h_ctr_[C_RT_SUBTREES];
    rt_intnodes_ = (int)h_ctr_[C_RT_INTNODES];
    // the reference's thresholds (LBvhFixedDeformable.cu:245, :257)
    if (rt_intnodes_ > (I >> 1)) {
        bvhcd_status st = build(s);
        opt_tag_ = 2;
        return st;
    }
    if (rt_intnodes_ < (I >> 3)) {
        opt_tag_ = 0;
        return refit(s);
    }
    // 5 per-leaf subtree root
    BV_TRY(scan_i32(extrange_.as<int>(), leafroot_.as<int>(), T + 1, true, nullptr, scratch_.p, s));
    k_rs_oldlast<<<grid_for(T), kThreads, 0, s>>>(T, leafroot_.as<int>(), lrec_.as<float4>(), rs_oldlast_.as<int>());
    note_launch();
    // 6-7 keys of the restructured primitives
    bvhcd_status st = scene_box(s);
    if (st != BVHCD_OK) return st;
    unsigned *flag = flagbuf_.as<unsigned>();
    unsigned *pos = keys2_.as<unsigned>();
    k_rs_flags<<<grid_for(T), kThreads, 0, s>>>(T, leafroot_.as<int>(), flag); note_launch();
    BV_TRY(scan_u32(flag, pos, T, false, ctr + C_RT_SUBTREES + 2, scratch_.p, s));
    k_rs_select<<<grid_for(T), kThreads, 0, s>>>(T, leafroot_.as<int>(), pos, sface_.as<int4>(), src(),
                                                 scene_.as<float>(), k64_.as<unsigned long long>(),
                                                 task_.as<int>(), vals_.as<int>()); note_launch();
    const int nr = rt_intnodes_ + rt_subtrees_;  // leaves = internal nodes + subtrees
    int bits = 32;
    while ((1LL << (bits - 32)) <= (long long)T && bits < 64) bits++;
    BV_TRY(radix_sort_u64(k64_.as<unsigned long long>(), vals_.as<int>(), k64b_.as<unsigned long long>(),
                          vals2_.as<int>(), nr, bits, scratch_.p, s));
    // 8 permutation
    k_rs_gather<<<grid_for(nr), kThreads, 0, s>>>(nr, vals_.as<int>(), sface_.as<int4>(), tmpface_.as<int4>()); note_launch();
    k_rs_scatter<<<grid_for(nr), kThreads, 0, s>>>(nr, task_.as<int>(), tmpface_.as<int4>(),
                                                   k64_.as<unsigned long long>(), sface_.as<int4>(),
                                                   primmap_.as<int>(), code_.as<unsigned>()); note_launch();
    // 9 boxes + refit with the old topology
    st = refit(s);
    if (st != BVHCD_OK) return st;
    // 10 confined rebuild
    k_metrics<<<grid_for(T), kThreads, 0, s>>>(T, code_.as<unsigned>(), metric_.as<int>()); note_launch();
    Climb c = make_climb(ulc_, urc_, upar_, urx_, ury_, umark_, ubox_, uflag_, posb_, clen_, ulpar_, uheight_);
    BV_TRY(cudaMemsetAsync(uflag_.p, 0, sizeof(unsigned) * (size_t)T, s));
    BV_TRY(cudaMemsetAsync(clen_.p, 0, sizeof(int) * (size_t)(T + 1), s));
    k_climb<true><<<grid_for(nr), kThreads, 0, s>>>(T, nr, task_.as<int>(), leafroot_.as<int>(),
                                                    metric_.as<int>(), lrec_.as<float4>(), topo_.as<int4>(), c); note_launch();
    BV_TRY(scan_u32(clen_.as<unsigned>(), coff_.as<unsigned>(), T + 1, false, nullptr, scratch_.p, s));
    k_rs_dfs<<<grid_for(nr), kThreads, 0, s>>>(nr, T, task_.as<int>(), leafroot_.as<int>(), nrange_.as<int2>(),
                                               coff_.as<unsigned>(), clen_.as<int>(), posb_.as<int>(),
                                               urx_.as<int>(), dfs_.as<int>()); note_launch();
    k_rs_lca<<<grid_for(nr), kThreads, 0, s>>>(nr, task_.as<int>(), leafroot_.as<int>(), nrange_.as<int2>(),
                                               topo_.as<int4>(), coff_.as<unsigned>(), clen_.as<int>(),
                                               lca_.as<int>()); note_launch();
    k_rs_write<<<grid_for(nr), kThreads, 0, s>>>(nr, T, task_.as<int>(), leafroot_.as<int>(), c, dfs_.as<int>(),
                                                 lca_.as<int>(), nrec_.as<float4>(), topo_.as<int4>(),
                                                 nrange_.as<int2>(), lrec_.as<float4>()); note_launch();
    BV_TRY(cudaGetLastError());
    opt_tag_ = 1;
    topo_epoch_++;
    rs_epoch_ = topo_epoch_;  // leafroot_, intmark_ and rs_oldlast_ describe this change
    // a new topology (the refit above saw leaves change slots): the
    // accumulated box motion starts again
    BV_TRY(cudaMemsetAsync(ctr_.as<unsigned>() + C_DELTA, 0, 2 * sizeof(unsigned), s));
    // the confined rebuild can change the heights of the subtrees' ancestors
    return refit_plan(s, false);
}

bvhcd_status LBvh::node_fp16(cudaStream_t s) {
    if (!cfg_.node_box_fp16 || T_ < 2 || !built_) return BVHCD_OK;
    BV_TRY(nrec16_.reserve(sizeof(uint4) * (size_t)(capT_ + 2)));
    k_node_fp16<<<grid_for(T_ - 1), kThreads, 0, s>>>(T_ - 1, nrec_.as<float4>(), nrec16_.as<uint4>()); note_launch();
    return cuda_status(cudaGetLastError());
}

// LBvhFixedDeformable::maintain (LBvhFixedDeformable.cu:68-87)
bvhcd_status LBvh::maintain(bvhcd_bvh_op op, const bvhcd_scene &scene, cudaStream_t s) {
    bvhcd_status st = maintain_tree(op, scene, s);
    if (st != BVHCD_OK) return st;
    return node_fp16(s);
}

bvhcd_status LBvh::maintain_tree(bvhcd_bvh_op op, const bvhcd_scene &scene, cudaStream_t s) {
    if (op < BVHCD_BVH_BUILD || op > BVHCD_BVH_UPDATE) return BVHCD_INVALID_ARG;
    if (S_ > 1 && scene.num_faces != h_off_[S_]) return BVHCD_INVALID_ARG;
    int prevT = T_;
    bool was_built = built_;
    bvhcd_status st = upload(scene, s);
    if (st != BVHCD_OK) return st;
    return maintain_ops(op, prevT, was_built, s);
}

bvhcd_status LBvh::maintain_boxes(bvhcd_bvh_op op, const bvhcd_box_scene &scene, cudaStream_t s) {
    if (op < BVHCD_BVH_BUILD || op > BVHCD_BVH_UPDATE) return BVHCD_INVALID_ARG;
    if (S_ > 1 && scene.num_faces != h_off_[S_]) return BVHCD_INVALID_ARG;
    int prevT = T_;
    bool was_built = built_;
    bvhcd_status st = upload_boxes(scene, s);
    if (st != BVHCD_OK) return st;
    st = maintain_ops(op, prevT, was_built, s);
    if (st != BVHCD_OK) return st;
    return node_fp16(s);
}

bvhcd_status LBvh::maintain_ops(bvhcd_bvh_op op, int prevT, bool was_built, cudaStream_t s) {
    opt_tag_ = 0;
    if (cfg_.enable_restr && updated_ && was_built && built_ && prevT == T_ && T_ >= 2) {
        bvhcd_status st = check_finite(s);
        return st != BVHCD_OK ? st : restructure(s);
    }
    if (op == BVHCD_BVH_BUILD || !built_) {
        bvhcd_status st = check_finite(s);
        return st != BVHCD_OK ? st : build(s);
    }
    return refit(s);  // UPDATE is refit: the reference marks updateIntNode deprecated (LBvhUpdateKernels.cu:88)
}

// The input of a build or restructure checked for NaN / infinite coordinates
// (a refit checks inline); the verdict goes to the counter C_NONFINITE, which
// the front's stats and pair export read.
bvhcd_status LBvh::check_finite(cudaStream_t s) {
    const float *x = box_input_ ? bptr_ : vptr_;
    const int64_t n = box_input_ ? 6 * (int64_t)T_ : 3 * (int64_t)V_;
    if (!x || n <= 0) {
        BV_TRY(cudaMemsetAsync(ctr_.as<unsigned>() + C_NONFINITE, 0, sizeof(unsigned), s));
        return BVHCD_OK;
    }
    int64_t g = (n + kThreads - 1) / kThreads;
    if (g > kSms * 4) g = kSms * 4;
    k_check_finite<<<(unsigned)g, kThreads, 0, s>>>(n, x, ctr_.as<unsigned>(),
                                                    box_input_ ? nullptr : verts4_.as<float4>()); note_launch();
    return cuda_status(cudaGetLastError());
}

bvhcd_status LBvh::request_restructure(const int32_t *roots, int32_t n, cudaStream_t s) {
    if (n < 0 || (n > 0 && !roots)) return BVHCD_INVALID_ARG;
    if (!built_) return BVHCD_NOT_READY;
    if (!cfg_.enable_restr || T_ < 2 || n == 0) return BVHCD_OK;
    const int T = T_;
    if (!updated_) {
        k_fill<<<grid_for(T), kThreads, 0, s>>>(T, rtroot_.as<int>(), INT_MAX); note_launch();
        BV_TRY(cudaMemsetAsync(intrange_.p, 0, sizeof(int) * (size_t)T, s));
    }
    DBuf tmp;
    BV_TRY(tmp.reserve(sizeof(int) * (size_t)n));
    BV_TRY(cudaMemcpyAsync(tmp.p, roots, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
    k_mark_roots<<<grid_for(n), kThreads, 0, s>>>(n, T - 1, tmp.as<int>(), nrange_.as<int2>(), intrange_.as<int>(),
                                                  rtroot_.as<int>()); note_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    tmp.release();
    BV_TRY(e);
    updated_ = true;
    return BVHCD_OK;
}

bvhcd_status LBvh::request_restructure_device(const int32_t *roots, int32_t n, cudaStream_t s) {
    if (n < 0 || (n > 0 && !roots)) return BVHCD_INVALID_ARG;
    if (!built_) return BVHCD_NOT_READY;
    if (!cfg_.enable_restr || T_ < 2 || n == 0) return BVHCD_OK;
    const int T = T_;
    if (!updated_) {
        k_fill<<<grid_for(T), kThreads, 0, s>>>(T, rtroot_.as<int>(), INT_MAX); note_launch();
        BV_TRY(cudaMemsetAsync(intrange_.p, 0, sizeof(int) * (size_t)T, s));
    }
    k_mark_roots<<<grid_for(n), kThreads, 0, s>>>(n, T - 1, roots, nrange_.as<int2>(), intrange_.as<int>(),
                                                  rtroot_.as<int>()); note_launch();
    BV_TRY(cudaGetLastError());
    updated_ = true;
    return BVHCD_OK;
}

bvhcd_status LBvh::export_tree(int32_t *inode, float *ibox, int32_t *leaf, float *lbox, int32_t *lca,
                               uint32_t *codes, int32_t *primmap, cudaStream_t s) const {
    const int T = T_;
    if (!built_) return BVHCD_NOT_READY;
    if (T == 0) return BVHCD_OK;
    DBuf tmp;
    size_t nb = sizeof(int) * 6 * (size_t)T * 2 + sizeof(int) * 4 * (size_t)T + sizeof(float) * 6 * (size_t)T;
    BV_TRY(tmp.reserve(nb));
    int *d_inode = tmp.as<int>();
    float *d_ibox = reinterpret_cast<float *>(d_inode + 6 * (size_t)T);
    int *d_leaf = reinterpret_cast<int *>(d_ibox + 6 * (size_t)T);
    float *d_lbox = reinterpret_cast<float *>(d_leaf + 4 * (size_t)T);
    k_export<<<grid_for(T), kThreads, 0, s>>>(T, nrec_.as<float4>(), topo_.as<int4>(), nrange_.as<int2>(),
                                              lrec_.as<float4>(), sface_.as<int4>(), lca_.as<int>(), d_inode,
                                              d_ibox, d_leaf, d_lbox); note_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && inode && T > 1)
        e = cudaMemcpyAsync(inode, d_inode, sizeof(int) * 6 * (size_t)(T - 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && ibox && T > 1)
        e = cudaMemcpyAsync(ibox, d_ibox, sizeof(float) * 6 * (size_t)(T - 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && leaf)
        e = cudaMemcpyAsync(leaf, d_leaf, sizeof(int) * 4 * (size_t)T, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && lbox)
        e = cudaMemcpyAsync(lbox, d_lbox, sizeof(float) * 6 * (size_t)T, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && lca)
        e = cudaMemcpyAsync(lca, lca_.p, sizeof(int) * (size_t)(T + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && codes)
        e = cudaMemcpyAsync(codes, code_.p, sizeof(unsigned) * (size_t)T, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && primmap)
        e = cudaMemcpyAsync(primmap, primmap_.p, sizeof(int) * (size_t)T, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    DBuf &t = const_cast<DBuf &>(tmp);
    t.release();
    return cuda_status(e);
}

// ---------------------------------------------------------------- Morton order
// without allocation.  Same kernels as the build's first half (scene box,
// Morton codes, stable radix sort), for callers that may not allocate device
// memory: the temporaries live in one fixed file-scope device array.
namespace {
constexpr size_t kNaPartialBytes = 4096 * 6 * sizeof(float);  // box partials, one per block
constexpr size_t kNaSceneBytes = 256;                          // scene box
constexpr size_t kNaKeysBytes = sizeof(unsigned) * BVHCD_NOALLOC_MAX_FACES;  // sort ping-pong keys
constexpr size_t kNaValsBytes = sizeof(int) * BVHCD_NOALLOC_MAX_FACES;       // sort ping-pong values
constexpr size_t kNaSortBytes = 1u << 20;                      // histograms + scan sums
constexpr size_t kNaTotal = kNaPartialBytes + kNaSceneBytes + kNaKeysBytes + kNaValsBytes + kNaSortBytes;
}  // namespace

// Loaded into every device context that uses this library and held there
// until the process exits (about 9.2 MB).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaTotal];

static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[256] = {};

// The symbol's device address for the current device, looked up once per
// device.  In host code the array's name only stands in for the symbol.
static cudaError_t noalloc_scratch(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_noalloc_ptr[dev]);
    return cudaSuccess;
}

bvhcd_status morton_order_noalloc(const float *verts, const int *faces, int T, unsigned *codes, int *order,
                                  cudaStream_t s) {
    if (T < 0 || (T > 0 && (!verts || !faces || !codes || !order))) return BVHCD_INVALID_ARG;
    if ((int64_t)T > (int64_t)BVHCD_NOALLOC_MAX_FACES || sort_scratch_bytes(T) > kNaSortBytes)
        return BVHCD_CAPACITY_EXCEEDED;
    if (T == 0) return BVHCD_OK;
    unsigned char *base = nullptr;
    BV_TRY(noalloc_scratch(&base));
    float *partial = reinterpret_cast<float *>(base);
    float *scene = reinterpret_cast<float *>(base + kNaPartialBytes);
    unsigned *keys_alt = reinterpret_cast<unsigned *>(base + kNaPartialBytes + kNaSceneBytes);
    int *vals_alt = reinterpret_cast<int *>(base + kNaPartialBytes + kNaSceneBytes + kNaKeysBytes);
    void *sort_scratch = base + kNaPartialBytes + kNaSceneBytes + kNaKeysBytes + kNaValsBytes;
    // every scratch word read below is written earlier in the same call
    int g = (int)grid_for(T);
    if (g > 4096) g = 4096;
    k_box_partial<<<g, kThreads, 0, s>>>(T, PrimSrc{faces, verts, nullptr}, partial); note_launch();
    k_box_final<<<1, kThreads, 0, s>>>(g, partial, scene); note_launch();
    k_morton<<<grid_for(T), kThreads, 0, s>>>(T, PrimSrc{faces, verts, nullptr}, scene, codes, order); note_launch();
    BV_TRY(cudaGetLastError());
    BV_TRY(radix_sort_u32(codes, order, keys_alt, vals_alt, T, 30, sort_scratch, s));
    return BVHCD_OK;
}

}  // namespace bvhcd
