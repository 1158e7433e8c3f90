// front.cu -- BVTT front generation, maintenance (prune / sprout), keep,
// ordering (counting sort by node) and balance, the front-quality metric, and
// the triangle-triangle narrow phase.
//
// Every kernel reads its work size from a device counter and walks it with a
// grid-stride loop, so a frame is a fixed launch sequence with no host round
// trip.  Emission reserves output slots in per-thread chunks and checks
// capacity before writing.
#include <climits>
#include <cstdlib>
#include <utility>

#include <cuda_fp16.h>

#include "pipeline.h"
#include "tritri.cuh"
#include "proximity.cuh"
#include "prims.cuh"

namespace bvhcd {

#define FR_TRY(x)                                        \
    do {                                                 \
        cudaError_t e__ = (x);                           \
        if (e__ != cudaSuccess) return cuda_status(e__); \
    } while (0)

namespace {

constexpr int kThreads = 256;
// resident blocks for the grid-stride kernels: a multiple of the SM count
constexpr int kFrontBlocks = kSms * 8;

inline unsigned grid_for(int64_t n) {
    int64_t g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    if (g > kFrontBlocks * 4) g = kFrontBlocks * 4;
    return (unsigned)g;
}

struct FArgs {
    const float4 *nrec, *lrec;
    // records of the traversing primitives: the tree's own leaves (an intra
    // front), or the leaves of another BVH (an inter front, whose primitives
    // start at the root, root_tag, instead of their own leaf's escape link)
    const float4 *prec;
    int nprim, inter, root_tag;
    const uint4 *nrec16;   // FP16 node records, or null for the FP32 ones
    const int2 *nrange;
    const int4 *topo;
    const int *lca;
    const int4 *sface;
    FrontLog log;
    unsigned *ctr;
    const int2 *in_int, *in_ext;
    int2 *out_int, *out_ext;
    int in_int_slot, in_ext_slot, out_int_slot, out_ext_slot;
    unsigned cap_int, cap_ext;
    int2 *pairs;
    unsigned cap_pairs;
    int2 *work;
    unsigned cap_work;
    int cull;
    int T;
    // keep-time expiries (keep only): motion is the tree's accumulated box
    // motion (FP32 bits); the _in arrays give each entry's expiry (read by
    // k_keep_select), the _out arrays receive the expiries of the entries
    // tested; ksel lists the entries to test (indices into [0, F_int + F_ext)),
    // or is null to test every entry
    const unsigned *motion;
    const float *iexp_in, *xexp_in;
    float *iexp_out, *xexp_out;
    const unsigned *ksel;
    // an inter front's restructure (k_restr_scan): the traversed BVH's last
    // restructure -- per internal node a non-zero mark inside a restructured
    // subtree, per leaf slot its subtree root (0 outside), per root the old
    // end of its left spine
    const int *rs_mark, *rs_root, *rs_last;
    // keep: the scan's last block records the pair count in C_PAIRS_SCAN
    int snap_scan;
};

// A node's box and escape link: from the FP32 record ({lo.xyz, rangex |
// leftleaf << 31}, {hi.xyz, escape}), or, with FP16 node boxes, from the 16-byte record {min.xyz,
// max.xyz as halves rounded outward, escape}.  The FP16 box contains the FP32
// one, so a traversal on it visits a superset of the nodes and still tests
// every overlapping leaf in FP32: the pair set does not change.
__device__ __forceinline__ float half_lo(unsigned w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xffffu))); }
__device__ __forceinline__ float half_hi(unsigned w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); }
__device__ __forceinline__ void node_rec(const FArgs &a, int n, float4 &lo, float4 &hi) {
    if (a.nrec16) {
        const uint4 r = __ldg(a.nrec16 + n);
        lo = make_float4(half_lo(r.x), half_hi(r.x), half_lo(r.y), __int_as_float(-1));
        hi = make_float4(half_hi(r.y), half_lo(r.z), half_hi(r.z), __int_as_float((int)r.w));
    } else {
        ldg8(a.nrec + 2 * n, lo, hi);
    }
}
// the node's leftmost leaf (lo.w of the FP32 record without its bit 31)
__device__ __forceinline__ int node_rangex(const FArgs &a, int n, const float4 &lo) {
    return a.nrec16 ? __ldg(&a.nrange[n]).x : (__float_as_int(lo.w) & 0x7fffffff);
}

// Per-node counter increment aggregated over the converged lanes of a warp
// that hit the same node: one atomic per distinct node instead of one per
// entry.  Nodes near the root sit in the fronts of a large share of all
// primitives, so unaggregated increments serialise on a few L2 addresses.
// Returns this lane's rank among the increments of its node (old value +
// rank within the group).
__device__ __forceinline__ unsigned node_add(unsigned *cnt, unsigned key, int node) {
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(cnt + node, (unsigned)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

// Output slots are handed out in per-thread chunks: a thread reserves kChunk
// consecutive slots of a stream with one atomic (shared by the converged
// lanes that need a chunk at the same time) and fills them as it emits.  The
// slots it has not filled when it finishes are closed with the hole marker
// (-1, -1), which every consumer skips.  Without chunks the traversal kernels
// serialise on the one counter per stream.  The stream counters therefore
// count reserved slots; true sizes come from the per-node counts (fronts) and
// from the narrow phase's count of valid pairs.
constexpr unsigned kChunk = 8;
struct Chunk {
    unsigned base = 0, left = 0;
};
struct Em {
    Chunk fi, fe, pr, wk;  // internal front, external front, pairs, sprout work
};

// Returns whether the entry was stored (false: past the capacity, flagged).
__device__ __forceinline__ bool chunk_put(int2 *buf, unsigned *ctr, unsigned cap, Chunk &c, const int2 &v,
                                          unsigned *ovf, unsigned bit) {
    if (c.left == 0) {
        cg::coalesced_group g = cg::coalesced_threads();
        unsigned b = 0;
        if (g.thread_rank() == 0) b = atomicAdd(ctr, kChunk * g.size());
        c.base = g.shfl(b, 0) + kChunk * g.thread_rank();
        c.left = kChunk;
    }
    const unsigned slot = c.base++;
    --c.left;
    if (slot < cap) {
        buf[slot] = v;
        return true;
    }
    atomicOr(ovf, bit);
    return false;
}
__device__ __forceinline__ void chunk_close(int2 *buf, unsigned cap, Chunk &c) {
    for (; c.left > 0; --c.left) {
        const unsigned slot = c.base++;
        if (slot < cap) buf[slot] = make_int2(-1, -1);
    }
}

// Only stored entries are counted: the per-node counts place the entries in
// the ordered front (reorder, balance), so after an overflow the ordered
// front holds exactly the entries that were kept and no unwritten slot.
__device__ __forceinline__ void emit_int(const FArgs &a, Em &em, int prim, int node) {
    if (chunk_put(a.out_int, a.ctr + a.out_int_slot, a.cap_int, em.fi, make_int2(prim, node), a.ctr + C_OVERFLOW, 1u))
        node_add(a.log.intcnt, (unsigned)node, node);
}
__device__ __forceinline__ void emit_ext(const FArgs &a, Em &em, int prim, int leaf) {
    if (chunk_put(a.out_ext, a.ctr + a.out_ext_slot, a.cap_ext, em.fe, make_int2(prim, leaf), a.ctr + C_OVERFLOW, 2u))
        node_add(a.log.extcnt, (unsigned)leaf, leaf);
}
// Returns whether the pair was stored (not culled, within the capacity).
__device__ __forceinline__ bool emit_pair(const FArgs &a, Em &em, int prim, const int4 &pf, int leaf) {
    if (a.cull && covertex(pf, __ldg(&a.sface[leaf]))) return false;
    return chunk_put(a.pairs, a.ctr + C_PAIRS, a.cap_pairs, em.pr, make_int2(prim, leaf), a.ctr + C_OVERFLOW, 4u);
}
__device__ __forceinline__ void emit_work(const FArgs &a, Em &em, const int2 &e) {
    chunk_put(a.work, a.ctr + C_WORK, a.cap_work, em.wk, e, a.ctr + C_OVERFLOW, 32u);
}
__device__ __forceinline__ void em_close(const FArgs &a, Em &em) {
    if (a.out_int) chunk_close(a.out_int, a.cap_int, em.fi);
    if (a.out_ext) chunk_close(a.out_ext, a.cap_ext, em.fe);
    if (a.pairs) chunk_close(a.pairs, a.cap_pairs, em.pr);
    if (a.work) chunk_close(a.work, a.cap_work, em.wk);
}

// The front scans walk their n entries grid-stride (the whole grid then works
// on a narrow window of the node-sorted front at any time, which keeps the
// records it reads in L2), but with no more lanes than n / kScanMinPer:
// chunked emission leaves up to kChunk - 1 reserved but unused slots per
// emitting lane and stream, and those holes count against the capacity.  With
// at least kScanMinPer entries per lane they stay below 7/32 of the input
// however small the front is next to the grid (one entry per lane would
// reserve eight slots per entry).  The traversal kernels (generation, sprout)
// keep one work item per lane: an item is a whole traversal, and their holes
// are at most seven per item and stream.
constexpr unsigned kScanMinPer = 32;
struct Spread {
    unsigned start, stride;  // this lane's first item (n: none); the lanes at work
};
template <unsigned kMin>
__device__ __forceinline__ Spread spread(unsigned n) {
    const unsigned grid = gridDim.x * blockDim.x;
    unsigned lanes = ((n + kMin - 1) / kMin + 31u) & ~31u;
    lanes = lanes < 32u ? 32u : lanes < grid ? lanes : grid;
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    return Spread{t < lanes ? t : n, lanes};
}

// left child of internal node d, tagged: the FP32 record carries it (bit 31
// of lo.w set: the left child is the leaf rangex; clear: it is node d + 1,
// the next id in DFS order); the FP16 record does not, so there it comes
// from the range and the leaf's parent
__device__ __forceinline__ int left_child_tagged(const FArgs &a, int d, const float4 &lo) {
    if (!a.nrec16) {
        const int w = __float_as_int(lo.w);
        return w < 0 ? (((w & 0x7fffffff) << 1) | 1) : ((d + 1) << 1);
    }
    const int rx = __ldg(&a.nrange[d]).x;
    const int last = __float_as_int(__ldg(reinterpret_cast<const float *>(a.lrec) + 8 * (size_t)rx + 3));
    return last == d ? ((rx << 1) | 1) : ((d + 1) << 1);
}

// Stackless traversal from tagged node `st` until tagged node `stop`
// (the loop shared by genLooseIntraFrontsWithLog,
// Mine/collision/bvtt_front/BvttFrontGenerateKernels.cu:65-88, the sprout
// half of maintainIntLooseIntraFrontsWithLog,
// BvttFrontPruneSproutKernels.cu:34-56, keepIntLooseIntraFronts,
// BvttFrontKeepKernels.cu:26-42, and pureBvhSelfCD, BvhCDKernels.cu:30-47):
// walk the left spine of an internal node by DFS id while the box overlaps,
// up to the parent of its leftmost leaf; a node that stops overlapping is a
// front node and is left through its escape link.  (A loop body of one
// record per step for both kinds of node was measured slower: 0.88 against
// 0.64 ms per generation on the 562,742-triangle scene -- the spine loop
// keeps consecutive records in a tight dependent chain.)
// An overlapping leaf is passed to on_pair (the pair's emission).
template <bool kFront, typename PairFn>
__device__ __forceinline__ void traverse_with(const FArgs &a, Em &em, int prim, const float4 &plo,
                                              const float4 &phi, int st, int stop, PairFn on_pair) {
    // a valid tree is left after at most 2T - 1 visits; the bound only turns
    // a corrupted tree into an error flag instead of an endless loop
    int guard = 2 * a.T + 2;
    while (st != stop) {
        if (--guard < 0) {
            atomicOr(a.ctr + C_OVERFLOW, 16u);
            return;
        }
        int leaf;
        float4 llo, lhi;
        if (st & 1) {
            leaf = st >> 1;
            ldg8(a.lrec + 2 * leaf, llo, lhi);
        } else {
            int n = st >> 1;
            float4 nlo, nhi;
            node_rec(a, n, nlo, nhi);
            leaf = node_rangex(a, n, nlo);
            ldg8(a.lrec + 2 * leaf, llo, lhi);
            const int last = __float_as_int(llo.w);  // parent of the leftmost leaf
            bool stopped = false;
            while (true) {
                if (!overlap(nlo, nhi, plo, phi)) { stopped = true; break; }
                if (n >= last) break;
                ++n;
                node_rec(a, n, nlo, nhi);
            }
            if (stopped) {
                if (kFront) emit_int(a, em, prim, n);
                st = __float_as_int(nhi.w);
                continue;
            }
        }
        if (overlap(llo, lhi, plo, phi)) on_pair(leaf);
        if (kFront) emit_ext(a, em, prim, leaf);
        st = __float_as_int(lhi.w);
    }
}
template <bool kFront>
__device__ __forceinline__ void traverse(const FArgs &a, Em &em, int prim, const float4 &plo,
                                         const float4 &phi, const int4 &pf, int st, int stop) {
    traverse_with<kFront>(a, em, prim, plo, phi, st, stop, [&](int leaf) { emit_pair(a, em, prim, pf, leaf); });
}

__device__ __forceinline__ int4 prim_face(const FArgs &a, int prim) {
    return a.cull ? __ldg(&a.sface[prim]) : make_int4(0, 0, 0, 0);
}

// genLooseIntraFrontsWithLog (BvttFrontGenerateKernels.cu:51-90) /
// pureBvhSelfCD (BvhCDKernels.cu:17-49)
template <bool kFront>
__global__ void __launch_bounds__(kThreads) k_generate(FArgs a) {
    Em em;
    // an intra front: primitive i traverses from its own leaf's escape link
    // (the primitives to its right); an inter front: every primitive of the
    // other BVH from the root (genLooseInterFrontsWithLog,
    // BvttFrontGenerateKernels.cu:92-124, which skips the last one)
    const int n = a.inter ? a.nprim : a.T - 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 plo, phi;
        ldg8(a.prec + 2 * i, plo, phi);
        traverse<kFront>(a, em, i, plo, phi, prim_face(a, i), a.inter ? a.root_tag : __float_as_int(phi.w), -1);
    }
    em_close(a, em);
}

// Walk up the left chain above node `n` (exclusive) while nodes do not
// overlap; returns the node to emit or -1 to drop (prune half of
// BvttFrontPruneSproutKernels.cu:24-30 and :76-82).
__device__ __forceinline__ int prune_up(const FArgs &a, int n, int top, const float4 &plo,
                                        const float4 &phi) {
    for (; n >= top; --n) {
        float4 lo, hi;
        node_rec(a, n, lo, hi);
        if (overlap(lo, hi, plo, phi)) break;
    }
    if (n < top && n + 1 > 0) {
        // the chain top's parent decides, unless the top is a root (node 0,
        // or the root of one scene of a forest)
        int p = __ldg(&a.topo[n + 1]).z;
        if (p >= 0) {
            float4 lo, hi;
            node_rec(a, p, lo, hi);
            if (!overlap(lo, hi, plo, phi)) return -1;
        }
    }
    return n + 1;
}

// Batched front scans.  The common case of every front operation is a test
// of one front entry (primitive record against node record) that ends the
// entry's work; the rare overlapping internal entry needs a traversal below
// its node.  The scans below test kU entries per thread per step with all
// their loads issued together (memory-level parallelism instead of one
// dependent chain per entry), keep the register count low, and append the
// overlapping internal entries to a work list that k_sprout traverses.
template <int kU>
struct Batch {
    int2 e[kU];
    unsigned qi[kU];  // the entry's index in [0, F_int + F_ext)
    bool v[kU], in_int[kU];
    float4 plo[kU], phi[kU], nlo[kU], nhi[kU];
};

// entries q0 + k*stride (internal ones first in the index space, then
// external ones)
template <int kU, bool kKeep = false>
__device__ __forceinline__ void load_ents(const FArgs &a, unsigned q0, unsigned stride, unsigned ni,
                                          unsigned total, Batch<kU> &b) {
#pragma unroll
    for (int k = 0; k < kU; k++) {
        const unsigned p = q0 + k * stride;
        b.v[k] = p < total;
        const unsigned q = (kKeep && a.ksel && b.v[k]) ? __ldg(a.ksel + p) : p;
        if (kKeep) b.qi[k] = q;
        b.in_int[k] = q < ni;
        b.e[k] = b.v[k] ? (b.in_int[k] ? __ldcs(&a.in_int[q]) : __ldcs(&a.in_ext[q - ni])) : make_int2(0, 0);
    }
}
// the primitive and node records of the batch's entries
template <int kU>
__device__ __forceinline__ void load_recs(const FArgs &a, Batch<kU> &b) {
#pragma unroll
    for (int k = 0; k < kU; k++) {
        if (!b.v[k]) continue;
        ldg8(a.prec + 2 * b.e[k].x, b.plo[k], b.phi[k]);
        if (b.in_int[k]) {
            node_rec(a, b.e[k].y, b.nlo[k], b.nhi[k]);
        } else {
            ldg8(a.lrec + 2 * b.e[k].y, b.nlo[k], b.nhi[k]);
        }
    }
}
template <int kU, bool kKeep = false>
__device__ __forceinline__ void take_ents(Batch<kU> &dst, const Batch<kU> &src) {
#pragma unroll
    for (int k = 0; k < kU; k++) {
        dst.e[k] = src.e[k];
        if (kKeep) dst.qi[k] = src.qi[k];
        dst.v[k] = src.v[k];
        dst.in_int[k] = src.in_int[k];
    }
}
// The scans walk the entry stream software-pipelined: the next batch's
// entries are requested before the current batch's records, so a step waits
// for one round trip (the records) instead of two (entries, then records).



// Traversal below overlapping internal front nodes (the sprout half of
// maintainIntLooseIntraFrontsWithLog, BvttFrontPruneSproutKernels.cu:32-56,
// with kFront; keepIntLooseIntraFronts, BvttFrontKeepKernels.cu:21-42, and the
// overlap half of reorderIntLooseIntraFrontsWithLog,
// BvttFrontReorderKernels.cu:43-62, without).
template <bool kFront, int kB>
__global__ void __launch_bounds__(kB) k_sprout(FArgs a) {
    pdl_wait();
    Em em;
    const unsigned n = min(a.ctr[C_WORK], a.cap_work);
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int2 e = a.work[q];
        if (e.x < 0) continue;  // hole
        float4 plo, phi;
        ldg8(a.prec + 2 * e.x, plo, phi);
        const int node = e.y < 0 ? ~e.y : e.y;
        float4 nlo, nhi;
        node_rec(a, node, nlo, nhi);
        // e.y = ~R: the whole restructured subtree R, R itself first (an inter
        // front's restructure); else below the overlapping node e.y
        traverse<kFront>(a, em, e.x, plo, phi, prim_face(a, e.x),
                         e.y < 0 ? (node << 1) : left_child_tagged(a, node, nlo), __float_as_int(nhi.w));
    }
    em_close(a, em);
}

// maintainIntLooseIntraFrontsWithLog (BvttFrontPruneSproutKernels.cu:12-57):
// non-overlapping entries are pruned here, overlapping ones go to k_sprout<true>.
// Five CTAs of 256 per SM: the scan fits 48 registers without spilling, and
// the extra warps hide more of its dependent loads (the left-chain walks).
template <int kU, int kB>
__global__ void __launch_bounds__(kB, 1280 / kB) k_maintain_int_scan(FArgs a) {
    pdl_wait();
    Em em;
    const unsigned ni = min(a.ctr[a.in_int_slot], a.cap_int);
    const Spread sp = spread<kScanMinPer>(ni);
    Batch<kU> b, nb;
    load_ents(a, sp.start, sp.stride, ni, ni, b);
    for (unsigned q0 = sp.start; q0 < ni; q0 += kU * sp.stride, take_ents(b, nb)) {
        load_ents(a, q0 + kU * sp.stride, sp.stride, ni, ni, nb);
        load_recs(a, b);
#pragma unroll
        for (int k = 0; k < kU; k++) {
            if (!b.v[k]) continue;
            if (overlap(b.nlo[k], b.nhi[k], b.plo[k], b.phi[k])) {
                emit_work(a, em, b.e[k]);
                continue;
            }
            const int top = __ldg(&a.lca[node_rangex(a, b.e[k].y, b.nlo[k])]) >> 1;
            const int m = prune_up(a, b.e[k].y - 1, top, b.plo[k], b.phi[k]);
            if (m >= 0) emit_int(a, em, b.e[k].x, m);
        }
    }
    em_close(a, em);
}

// maintainExtLooseIntraFrontsWithLog (BvttFrontPruneSproutKernels.cu:60-93)
// (five CTAs of 256 per SM, as the internal scan: 48 registers with a few
// bytes of spills, still faster)
template <int kU, int kB>
__global__ void __launch_bounds__(kB, 1280 / kB) k_maintain_ext(FArgs a) {
    pdl_wait();
    Em em;
    const unsigned ne = min(a.ctr[a.in_ext_slot], a.cap_ext);
    const Spread sp = spread<kScanMinPer>(ne);
    Batch<kU> b, nb;
    load_ents(a, sp.start, sp.stride, 0, ne, b);
    for (unsigned q0 = sp.start; q0 < ne; q0 += kU * sp.stride, take_ents(b, nb)) {
        load_ents(a, q0 + kU * sp.stride, sp.stride, 0, ne, nb);
        load_recs(a, b);
#pragma unroll
        for (int k = 0; k < kU; k++) {
            if (!b.v[k]) continue;
            const int prim = b.e[k].x, st = b.e[k].y;
            if (overlap(b.nlo[k], b.nhi[k], b.plo[k], b.phi[k])) {
                emit_ext(a, em, prim, st);
                emit_pair(a, em, prim, prim_face(a, prim), st);
                continue;
            }
            const int gfa = __float_as_int(b.nlo[k].w);
            float4 glo, ghi;
            node_rec(a, gfa, glo, ghi);
            if (overlap(glo, ghi, b.plo[k], b.phi[k])) {
                emit_ext(a, em, prim, st);
                continue;
            }
            const int l = __ldg(&a.lca[st]);
            if (l & 1) continue;  // right child: the parent's left chain handles it
            const int m = prune_up(a, gfa - 1, l >> 1, b.plo[k], b.phi[k]);
            if (m >= 0) emit_int(a, em, prim, m);
        }
    }
    em_close(a, em);
}

// An inter front after its traversed BVH restructured subtrees
// (BvttFrontLooseInter::restructure, BvttFrontLooseInter.cu:252-318, with
// separateInt/ExtLooseInterFrontWithLog, BvttFrontReorderKernels.cu:171-198,
// filterInt/ExtFrontCnts, FlOrderLog.cu:36-73, and
// restructureInt/ExtLooseInterFrontWithLog, BvttFrontRestructureKernels.cu:
// 99-157), in one pass over both fronts.  An entry outside every
// restructured subtree is valid: an internal one that overlaps goes to the
// sprout work list, the others are kept as they are (no prune here: a prune
// could drop an entry whose left sibling's entries are being replaced); an
// external one is kept and gives its pair.  The entries of a primitive inside
// a restructured subtree R were a complete cut of R's old subtree, which
// holds exactly one node of R's old left spine (DFS ids R .. old end) or R's
// leftmost leaf: that entry becomes the work item (primitive, ~R), which
// k_sprout<true> traverses from R itself; the others are dropped.
template <int kU, int kB>
__global__ void __launch_bounds__(kB) k_restr_scan(FArgs a) {
    pdl_wait();
    Em em;
    const unsigned ni = min(a.ctr[a.in_int_slot], a.cap_int);
    const unsigned ne = min(a.ctr[a.in_ext_slot], a.cap_ext);
    const Spread sp = spread<kScanMinPer>(ni + ne);
    Batch<kU> b, nb;
    load_ents(a, sp.start, sp.stride, ni, ni + ne, b);
    for (unsigned q0 = sp.start; q0 < ni + ne; q0 += kU * sp.stride, take_ents(b, nb)) {
        load_ents(a, q0 + kU * sp.stride, sp.stride, ni, ni + ne, nb);
        load_recs(a, b);
#pragma unroll
        for (int k = 0; k < kU; k++) {
            if (!b.v[k]) continue;
            const int prim = b.e[k].x, node = b.e[k].y;
            if (b.in_int[k]) {
                if (__ldg(&a.rs_mark[node]) > 0) {
                    const int R = __ldg(&a.rs_root[node_rangex(a, node, b.nlo[k])]);
                    if (node <= __ldg(&a.rs_last[R])) emit_work(a, em, make_int2(prim, ~R));
                    continue;
                }
                if (overlap(b.nlo[k], b.nhi[k], b.plo[k], b.phi[k])) emit_work(a, em, b.e[k]);
                else emit_int(a, em, prim, node);
                continue;
            }
            const int R = __ldg(&a.rs_root[node]);
            if (R > 0) {
                if (node == __ldg(&a.nrange[R]).x) emit_work(a, em, make_int2(prim, ~R));
                continue;
            }
            emit_ext(a, em, prim, node);
            if (overlap(b.nlo[k], b.nhi[k], b.plo[k], b.phi[k])) emit_pair(a, em, prim, prim_face(a, prim), node);
        }
    }
    em_close(a, em);
}

// Keep-time expiries.  Between two refits every box of a tree moves by at
// most the largest change of a leaf box coordinate (a node's box is a min /
// max of leaf boxes); the refit sums those changes, rounded up, into the
// tree's motion M.  A keep that finds an entry's boxes apart by a gap g (a
// lower bound, rounded down, along their most separated axis) gives it the
// expiry M + g / 2: while the motion stays below it the boxes stay apart and
// the entry has nothing to emit.  An external entry of two triangles that
// share a vertex never gives a pair while the faces stay the same (expiry
// +inf); an entry that overlaps is tested every time (expiry -1).
__device__ __forceinline__ float box_gap(const float4 &alo, const float4 &ahi, const float4 &blo, const float4 &bhi) {
    float g = fmaxf(__fsub_rd(blo.x, ahi.x), __fsub_rd(alo.x, bhi.x));
    g = fmaxf(g, fmaxf(__fsub_rd(blo.y, ahi.y), __fsub_rd(alo.y, bhi.y)));
    return fmaxf(g, fmaxf(__fsub_rd(blo.z, ahi.z), __fsub_rd(alo.z, bhi.z)));
}

// The entries whose expiry the motion has reached, as a list of indices into
// [0, F_int + F_ext), in index order.  The expiries are read as a stream of
// 16-byte loads and nothing else of a waiting entry is touched.  The two
// arrays are tiled apart (a tile starts on a 16-byte boundary of its own
// array): a block takes tiles of 2048 entries, a warp two runs of 128, a lane
// four consecutive entries per run.  A warp scan places each lane's picks in
// its warp, a block scan in shared memory places the warps, one atomic per
// tile reserves the tile's run of the list.
constexpr int kSelRuns = 2;  // (the list positions below are written for two)
constexpr unsigned kSelTile = kSelRuns * 4 * kThreads;
__global__ void __launch_bounds__(kThreads) k_keep_select(FArgs a, unsigned *list, unsigned *count) {
    __shared__ unsigned wsum[kThreads / 32], tbase;
    const unsigned ni = min(a.ctr[a.in_int_slot], a.cap_int);
    const unsigned ne = min(a.ctr[a.in_ext_slot], a.cap_ext);
    const unsigned nti = (ni + kSelTile - 1) / kSelTile, ntiles = nti + (ne + kSelTile - 1) / kSelTile;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float4 ex[kSelRuns];
    auto load_tile = [&](unsigned k) {  // every load of the tile in flight at once
        const bool ext = k >= nti;
        const float *src = ext ? a.xexp_in : a.iexp_in;
        const unsigned n = ext ? ne : ni;
        const unsigned base = (ext ? k - nti : k) * kSelTile + warp * (kSelRuns * 128u) + lane * 4u;
#pragma unroll
        for (int r = 0; r < kSelRuns; r++) {
            const unsigned i = base + r * 128u;
            if (i + 4u <= n) {
                ex[r] = __ldcs(reinterpret_cast<const float4 *>(src + i));
            } else {
                ex[r].x = i < n ? __ldcs(src + i) : 0.f;
                ex[r].y = i + 1u < n ? __ldcs(src + i + 1u) : 0.f;
                ex[r].z = i + 2u < n ? __ldcs(src + i + 2u) : 0.f;
                ex[r].w = 0.f;
            }
        }
    };
    // the front sizes and the expiries come from earlier maintains: the first
    // tile is loaded before the wait for the kernels just before (the refit
    // that accumulates the motion, the prologue that zeroes the count)
    if (blockIdx.x < ntiles) load_tile(blockIdx.x);
    pdl_wait();
    const float M = __uint_as_float(*a.motion);
    for (unsigned k = blockIdx.x; k < ntiles; k += gridDim.x) {
        const bool ext = k >= nti;
        const unsigned n = ext ? ne : ni;
        const unsigned qoff = ext ? ni : 0u;
        const unsigned base = (ext ? k - nti : k) * kSelTile + warp * (kSelRuns * 128u) + lane * 4u;
        if (k != blockIdx.x) load_tile(k);
        // picks per lane and run (past the end nothing is picked, whatever
        // the motion: an infinite input coordinate makes it infinite)
        unsigned bits[kSelRuns], packed = 0;
#pragma unroll
        for (int r = 0; r < kSelRuns; r++) {
            const unsigned i = base + r * 128u;
            bits[r] = ((i < n && !(M < ex[r].x)) ? 1u : 0u) | ((i + 1u < n && !(M < ex[r].y)) ? 2u : 0u) |
                      ((i + 2u < n && !(M < ex[r].z)) ? 4u : 0u) | ((i + 3u < n && !(M < ex[r].w)) ? 8u : 0u);
            packed += (unsigned)__popc(bits[r]) << (16 * r);
        }
        // both runs' counts scanned at once, one per half-word
        unsigned incl = packed;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += u;
        }
        const unsigned wtot = __shfl_sync(0xffffffffu, incl, 31);
        const unsigned excl = incl - packed;
        if (lane == 0) wsum[warp] = (wtot & 0xffffu) + (wtot >> 16);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned acc = 0;
            for (int w = 0; w < kThreads / 32; w++) {
                const unsigned c = wsum[w];
                wsum[w] = acc;
                acc += c;
            }
            tbase = acc ? atomicAdd(count, acc) : 0u;
        }
        __syncthreads();
        unsigned pos[kSelRuns] = {tbase + wsum[warp] + (excl & 0xffffu),
                                  tbase + wsum[warp] + (wtot & 0xffffu) + (excl >> 16)};
#pragma unroll
        for (int r = 0; r < kSelRuns; r++) {
            const unsigned q = qoff + base + r * 128u;
#pragma unroll
            for (int j = 0; j < 4; j++)
                if ((bits[r] >> j) & 1u) list[pos[r]++] = q + j;
        }
        __syncthreads();  // wsum and tbase are reused by the next tile
    }
}

// An emission without per-lane chunks: the converged lanes that emit at the
// same time take consecutive slots with one atomic, so nothing is reserved
// unused (the selected keep runs few entries per lane, where chunks would
// leave holes in most slots).
__device__ __forceinline__ void put_dense(int2 *buf, unsigned *ctr, unsigned cap, const int2 &v, unsigned *ovf,
                                          unsigned bit) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned b = 0;
    if (g.thread_rank() == 0) b = atomicAdd(ctr, g.size());
    const unsigned slot = g.shfl(b, 0) + g.thread_rank();
    if (slot < cap) buf[slot] = v;
    else atomicOr(ovf, bit);
}

// keepIntLooseIntraFronts / keepExtLooseIntraFronts (BvttFrontKeepKernels.cu:11-58)
// in one index space: [0, F_int) internal entries, then external ones; with
// a selection list, only the listed entries, spread over every lane and
// emitted densely.  With expiries out, every entry tested gets its new
// expiry.
template <int kU, int kB>
__global__ void __launch_bounds__(kB) k_keep_scan(FArgs a) {
    pdl_wait();
    Em em;
    const unsigned ni = min(a.ctr[a.in_int_slot], a.cap_int);
    const unsigned ne = min(a.ctr[a.in_ext_slot], a.cap_ext);
    const unsigned total = a.ksel ? min(a.ctr[C_KSEL], ni + ne) : ni + ne;
    const float M = a.motion ? __uint_as_float(*a.motion) : 0.f;
    const Spread sp = a.ksel ? spread<1>(total) : spread<kScanMinPer>(total);
    Batch<kU> b, nb;
    load_ents<kU, true>(a, sp.start, sp.stride, ni, total, b);
    for (unsigned q0 = sp.start; q0 < total; q0 += kU * sp.stride, take_ents<kU, true>(b, nb)) {
        load_ents<kU, true>(a, q0 + kU * sp.stride, sp.stride, ni, total, nb);
        load_recs(a, b);
#pragma unroll
        for (int k = 0; k < kU; k++) {
            if (!b.v[k]) continue;
            const bool ov = overlap(b.nlo[k], b.nhi[k], b.plo[k], b.phi[k]);
            if (b.in_int[k]) {
                if (a.iexp_out)
                    a.iexp_out[b.qi[k]] =
                        ov ? -1.f : __fadd_rd(M, __fmul_rd(box_gap(b.plo[k], b.phi[k], b.nlo[k], b.nhi[k]), 0.5f));
                if (ov) {
                    if (a.ksel) put_dense(a.work, a.ctr + C_WORK, a.cap_work, b.e[k], a.ctr + C_OVERFLOW, 32u);
                    else emit_work(a, em, b.e[k]);
                }
                continue;
            }
            if (!a.xexp_out) {
                if (ov) emit_pair(a, em, b.e[k].x, prim_face(a, b.e[k].x), b.e[k].y);
                continue;
            }
            // (faces are read only for overlapping entries; a separated one waits on its gap)
            const bool adj = ov && a.cull && covertex(prim_face(a, b.e[k].x), __ldg(&a.sface[b.e[k].y]));
            a.xexp_out[b.qi[k] - ni] =
                adj ? 3.402823466e+38f
                    : (ov ? -1.f : __fadd_rd(M, __fmul_rd(box_gap(b.plo[k], b.phi[k], b.nlo[k], b.nhi[k]), 0.5f)));
            if (ov && !adj) {
                if (a.ksel) put_dense(a.pairs, a.ctr + C_PAIRS, a.cap_pairs, b.e[k], a.ctr + C_OVERFLOW, 4u);
                else chunk_put(a.pairs, a.ctr + C_PAIRS, a.cap_pairs, em.pr, b.e[k], a.ctr + C_OVERFLOW, 4u);
            }
        }
    }
    em_close(a, em);
    if (a.snap_scan) {  // the last block records the scan's pair count (the keep's tail reads it)
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(a.ctr + C_SCAN_DONE, 1u) == gridDim.x - 1) {
                __threadfence();
                a.ctr[C_PAIRS_SCAN] = atomicAdd(a.ctr + C_PAIRS, 0u);
                a.ctr[C_SCAN_DONE] = 0u;
            }
        }
    }
}

// balance: reorderIntLooseIntraFrontsWithLog (BvttFrontReorderKernels.cu:27-63)
// + keepExtLooseIntraFronts for the external front.  Non-overlapping entries
// fill their node's bucket from the front, overlapping ones from the back
// and are traversed by k_sprout<false>.
template <int kU, int kB>
__global__ void __launch_bounds__(kB) k_balance_scan(FArgs a) {
    pdl_wait();
    Em em;
    const unsigned ni = min(a.ctr[a.in_int_slot], a.cap_int);
    const unsigned ne = min(a.ctr[a.in_ext_slot], a.cap_ext);
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctr[a.out_int_slot] = a.ctr[a.in_int_slot];
    const Spread sp = spread<kScanMinPer>(ni + ne);
    Batch<kU> b, nb;
    load_ents(a, sp.start, sp.stride, ni, ni + ne, b);
    for (unsigned q0 = sp.start; q0 < ni + ne; q0 += kU * sp.stride, take_ents(b, nb)) {
        load_ents(a, q0 + kU * sp.stride, sp.stride, ni, ni + ne, nb);
        load_recs(a, b);
#pragma unroll
        for (int k = 0; k < kU; k++) {
            if (!b.v[k]) continue;
            const int2 e = b.e[k];
            const bool ov = overlap(b.nlo[k], b.nhi[k], b.plo[k], b.phi[k]);
            if (b.in_int[k]) {
                const unsigned key = ((unsigned)e.y << 1) | (ov ? 1u : 0u);
                unsigned pos = ov ? a.log.intbeg[e.y + 1] - 1u - node_add(a.log.intback, key, e.y)
                                  : a.log.intbeg[e.y] + node_add(a.log.intcnt, key, e.y);
                if (pos < a.cap_int) a.out_int[pos] = e;
                if (ov) emit_work(a, em, e);
            } else if (ov) {
                emit_pair(a, em, e.x, prim_face(a, e.x), e.y);
            }
        }
    }
    em_close(a, em);
}

// pureReorderLooseFrontsWithLog (BvttFrontReorderKernels.cu:12-24): a
// counting sort scatter of both fronts by node.  Holes left by chunked
// emission are skipped; the sorted fronts' sizes are the per-node count
// totals.
//
// The sort key is the node's group of 2^kReorderShift consecutive DFS ids,
// not the node itself: the order only serves the locality of the scans that
// read the front next (their node records then come from a few lines per
// warp), and the per-node counts the emission kept are what the quality
// check, the snapshot and a balance's buckets use.  A group's run starts at
// the begin of its first node (the scan of the per-node counts), so no count
// is recomputed and the counts stay as the emission left them.
//
// Tiles of kReorderTile entries: each CTA first groups its tile by key
// (group, internal or external front) in a shared-memory hash table, taking
// each entry's rank within its key and listing the slots it filled; then one
// global atomic per distinct key reserves the key's run in the sorted front;
// then every entry is written at run start + rank.  Neighbouring primitives
// share most front nodes and a group holds several nodes, so a tile holds
// far fewer keys than entries: the cursor atomics (which serialise on the
// groups near the root) drop by that factor, and a key's entries land next to
// each other.  Only the listed slots are visited to place the runs and to
// clear the table for the next tile (a tile fills a few hundred of its
// slots), and the table is cleared whole once per CTA.
#ifndef BVHCD_REORDER_THREADS
#define BVHCD_REORDER_THREADS 256
#endif
constexpr int kReorderThreads = BVHCD_REORDER_THREADS;
constexpr int kReorderPer = 8;                                   // entries per thread per tile
constexpr int kReorderTile = kReorderThreads * kReorderPer;
constexpr int kReorderSlots = 2 * kReorderTile;                  // hash slots (load factor <= 1/2)
constexpr int kReorderHashShift = 32 - (kReorderThreads == 512 ? 13 : 12);
static_assert(kReorderSlots == (1 << (32 - kReorderHashShift)), "hash width");
constexpr unsigned kEmptyKey = 0xffffffffu;

#ifndef BVHCD_REORDER_SHIFT
#define BVHCD_REORDER_SHIFT 2
#endif
constexpr int kReorderShift = BVHCD_REORDER_SHIFT;  // 4 nodes (128 bytes of node records) per group

inline size_t reorder_groups(int T) { return ((size_t)T >> kReorderShift) + 2; }

__global__ void __launch_bounds__(kReorderThreads) k_reorder(FArgs a, unsigned *cur_int, unsigned *cur_ext) {
    extern __shared__ unsigned rsm[];
    unsigned *skey = rsm, *scnt = rsm + kReorderSlots, *sbase = rsm + 2 * kReorderSlots;
    unsigned short *sused = reinterpret_cast<unsigned short *>(rsm + 3 * kReorderSlots);  // filled slots (< 2^16)
    __shared__ unsigned nused[2];
    const unsigned ni = min(a.ctr[a.in_int_slot], a.cap_int);
    const unsigned ne = min(a.ctr[a.in_ext_slot], a.cap_ext);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.ctr[a.out_int_slot] = a.log.intbeg[a.T];
        a.ctr[a.out_ext_slot] = a.log.extbeg[a.T];
    }
    for (int i = threadIdx.x; i < kReorderSlots; i += kReorderThreads) {
        skey[i] = kEmptyKey;
        scnt[i] = 0u;
    }
    if (threadIdx.x == 0) nused[0] = nused[1] = 0u;
    __syncthreads();
    const unsigned total = ni + ne;
    const unsigned ntiles = (total + kReorderTile - 1) / kReorderTile;
    unsigned par = 0;
    for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x, par ^= 1u) {
        int2 e[kReorderPer];
        unsigned slot[kReorderPer], rank[kReorderPer];
#pragma unroll
        for (int j = 0; j < kReorderPer; j++) {
            const unsigned q = tile * kReorderTile + j * kReorderThreads + threadIdx.x;
            e[j] = q < total ? (q < ni ? __ldcs(&a.in_int[q]) : __ldcs(&a.in_ext[q - ni])) : make_int2(-1, -1);
            if (e[j].x >= 0) e[j].x |= (q < ni ? 0 : (int)0x80000000);  // front tag in the sign bit, for now
        }
#pragma unroll
        for (int j = 0; j < kReorderPer; j++) {
            slot[j] = kEmptyKey;
            if (e[j].x == -1) continue;  // hole (a tagged entry is never -1: its index is below 2^31 - 1)
            const unsigned key = (((unsigned)e[j].y >> kReorderShift) << 1) | ((unsigned)e[j].x >> 31);
            unsigned h = (key * 2654435761u) >> kReorderHashShift;
            // a filled slot keeps its key until the table is cleared, so a plain
            // load finds the key (most entries: a tile holds far fewer keys than
            // entries) and only an empty slot needs the compare-and-swap
            for (int probe = 0; probe < kReorderSlots; probe++, h = (h + 1) & (kReorderSlots - 1)) {
                unsigned prev = *reinterpret_cast<volatile unsigned *>(&skey[h]);
                if (prev == kEmptyKey) {
                    prev = atomicCAS(&skey[h], kEmptyKey, key);
                    if (prev == kEmptyKey) sused[atomicAdd(&nused[par], 1u)] = (unsigned short)h;
                }
                if (prev == kEmptyKey || prev == key) break;
            }
            slot[j] = h;
            rank[j] = atomicAdd(&scnt[h], 1u);
        }
        if (threadIdx.x == 0) nused[par ^ 1u] = 0u;  // the next tile's list (last read before this tile's first barrier)
        __syncthreads();
        const unsigned nu = nused[par];
        for (unsigned i = threadIdx.x; i < nu; i += kReorderThreads) {
            const unsigned h = sused[i];
            const unsigned key = skey[h];
            const unsigned g = key >> 1;
            const unsigned first = g << kReorderShift;
            if (key & 1u) sbase[h] = a.log.extbeg[first] + atomicAdd(cur_ext + g, scnt[h]);
            else sbase[h] = a.log.intbeg[first] + atomicAdd(cur_int + g, scnt[h]);
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kReorderPer; j++) {
            if (slot[j] == kEmptyKey) continue;
            const bool is_ext = e[j].x < 0;
            const int2 v = make_int2(e[j].x & 0x7fffffff, e[j].y);
            const unsigned pos = sbase[slot[j]] + rank[j];
            if (!is_ext) {
                if (pos < a.cap_int) a.out_int[pos] = v;
            } else if (pos < a.cap_ext) {
                a.out_ext[pos] = v;
            }
        }
        // the filled slots are emptied for the next tile (the scatter reads only sbase)
        for (unsigned i = threadIdx.x; i < nu; i += kReorderThreads) {
            const unsigned h = sused[i];
            skey[h] = kEmptyKey;
            scnt[h] = 0u;
        }
        __syncthreads();
    }
}

constexpr size_t kReorderSmem = sizeof(unsigned) * 3 * kReorderSlots + sizeof(unsigned short) * kReorderTile;
static_assert(kReorderSlots <= 65536, "slot indices are listed as 16-bit values");

// frontSnapshot (BvttFrontGenerateKernels.cu:26-32)
__global__ void k_snapshot(int nint, const int2 *__restrict__ nrange, const unsigned *__restrict__ intbeg,
                           const unsigned *__restrict__ extbeg, float *snap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nint; i += gridDim.x * blockDim.x) {
        int2 r = nrange[i];
        unsigned ic = intbeg[i + r.y - r.x] - intbeg[i];
        unsigned ec = extbeg[r.y + 1] - extbeg[r.x] + 1u;
        snap[i] = __double2float_rn(__ddiv_rn(__dmul_rn(1.0, (double)ic), (double)ec));
    }
}

__global__ void k_fill_i32(int n, int *p, int v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// checkFrontQuality (BvttFrontGenerateKernels.cu:34-49): a subtree whose
// internal/external front ratio grew past snapshot + 1 - 0.7 * share is
// marked (+1/-1 range markers in DFS order and the shallowest root per
// leftmost leaf).  Double precision, IEEE operations, as the reference.
__global__ void k_check_quality(int nint, const int2 *__restrict__ nrange,
                                const unsigned *__restrict__ intbeg, const unsigned *__restrict__ extbeg,
                                const float *__restrict__ snap, int *intrange, int *rtroot) {
    const unsigned total = intbeg[nint];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nint; i += gridDim.x * blockDim.x) {
        int2 r = nrange[i];
        int ic = (int)(intbeg[i + r.y - r.x] - intbeg[i]);
        int ec = (int)(extbeg[r.y + 1] - extbeg[r.x]);
        double lhs = __ddiv_rn((double)ic, (double)ec);
        double rhs = __dsub_rn(__dadd_rn((double)snap[i], 1.0), __ddiv_rn(__dmul_rn(0.7, (double)ic), (double)total));
        if (lhs > rhs) {
            atomicAdd(intrange + i, 1);
            atomicAdd(intrange + i + r.y - r.x, -1);
            atomicMin(rtroot + r.x, i);
        }
    }
}

// ---------------------------------------------------------------- narrow phase
// FP32 17-axis separating-axis test (Gottschalk's triangle SAT as
// gProximity's triangleIntersection2 applies it,
// Source/Externals/inc/gProximity/cuda_intersect_tritri.h:247-266,349-433):
// translate by P1, face normals, nine edge x edge axes, six in-plane edge
// normals; intervals strictly apart separate.  Explicit round-to-nearest
// intrinsics keep the compiler from contracting into FMAs, so the result is
// bit-identical to the same sequence evaluated on the CPU.
struct v3 { float x, y, z; };
__device__ __forceinline__ v3 vsub(v3 a, v3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ v3 vcross(v3 a, v3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ __forceinline__ float vdot(v3 a, v3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ bool axis_overlap(v3 ax, v3 p2, v3 p3, v3 q1, v3 q2, v3 q3) {
    const v3 p1 = {0.f, 0.f, 0.f};
    float P1 = vdot(ax, p1), P2 = vdot(ax, p2), P3 = vdot(ax, p3);
    float Q1 = vdot(ax, q1), Q2 = vdot(ax, q2), Q3 = vdot(ax, q3);
    float mx1 = fmaxf(fmaxf(P1, P2), P3), mn1 = fminf(fminf(P1, P2), P3);
    float mx2 = fmaxf(fmaxf(Q1, Q2), Q3), mn2 = fminf(fminf(Q1, Q2), Q3);
    return !(mn1 > mx2) && !(mn2 > mx1);
}
__device__ bool tritri_sat32(v3 P1, v3 P2, v3 P3, v3 Q1, v3 Q2, v3 Q3) {
    const v3 z = {0.f, 0.f, 0.f};
    v3 p2 = vsub(P2, P1), p3 = vsub(P3, P1);
    v3 q1 = vsub(Q1, P1), q2 = vsub(Q2, P1), q3 = vsub(Q3, P1);
    v3 e0 = vsub(p2, z), e1 = vsub(p3, p2), e2 = vsub(z, p3);
    v3 f0 = vsub(q2, q1), f1 = vsub(q3, q2), f2 = vsub(q1, q3);
    v3 n = vcross(e0, e1), m = vcross(f0, f1);
    if (!axis_overlap(n, p2, p3, q1, q2, q3)) return false;
    if (!axis_overlap(m, p2, p3, q1, q2, q3)) return false;
    const v3 e[3] = {e0, e1, e2}, f[3] = {f0, f1, f2};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            if (!axis_overlap(vcross(e[i], f[j]), p2, p3, q1, q2, q3)) return false;
#pragma unroll
    for (int i = 0; i < 3; i++)
        if (!axis_overlap(vcross(e[i], n), p2, p3, q1, q2, q3)) return false;
#pragma unroll
    for (int j = 0; j < 3; j++)
        if (!axis_overlap(vcross(f[j], m), p2, p3, q1, q2, q3)) return false;
    return true;
}

__device__ __forceinline__ v3 vload(const float *v, int i) {
    const float *p = v + 3 * (size_t)i;
    return {__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}
__device__ __forceinline__ v3 vload(const float4 *v, int i) {
    const float4 p = __ldg(v + i);
    return {p.x, p.y, p.z};
}

// The block of the narrow phase that finishes last writes the valid pair and
// hit counts as 64-bit values (the counts the C ABI exports) and clears the
// finish counter for the next launch.
__device__ __forceinline__ void narrow_done(unsigned *ctr, unsigned cap_pairs, unsigned cap_hits, int64_t *out) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(ctr + C_NARROW_DONE, 1u) == gridDim.x - 1) {
            __threadfence();
            out[0] = min(__ldcg(ctr + C_PAIRS_VALID), cap_pairs);
            out[1] = min(__ldcg(ctr + C_HITS), cap_hits);
            ctr[C_NARROW_DONE] = 0u;
        }
    }
}

// simpleNarrowPhase (Mine/collision/narrow_phase/narrow_phase.cu:8-24):
// keeps the pairs whose triangles intersect, as original triangle ids, and
// counts the valid broad-phase pairs (the pair list has holes).  Without
// kTest it only counts.  A pair is (traversing primitive, leaf): the
// primitive's triangle from (psface, pverts), the leaf's from (sface, verts)
// -- the same mesh for an intra front, the other BVH's for an inter front,
// whose hits are written leaf first (the reference's inter pair order).
__device__ __forceinline__ void narrow_test(const NarrowArgs &n, const int2 &p) {
    const int4 a = __ldg(&n.psface[p.x]), b = __ldg(&n.sface[p.y]);
    if (tritri_sat32(vload(n.pverts, a.x), vload(n.pverts, a.y), vload(n.pverts, a.z), vload(n.verts, b.x),
                     vload(n.verts, b.y), vload(n.verts, b.z)))
        emit(n.hits, n.ctr + C_HITS, n.cap_hits, n.leaf_first ? make_int2(b.w, a.w) : make_int2(a.w, b.w),
             n.ctr + C_OVERFLOW, 8u);
}
__device__ __forceinline__ void count_valid(unsigned *ctr, unsigned valid) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) valid += __shfl_xor_sync(0xffffffffu, valid, o);
    if ((threadIdx.x & 31) == 0 && valid) atomicAdd(ctr + C_PAIRS_VALID, valid);
}

template <bool kTest, int kB>
__global__ void __launch_bounds__(kB) k_narrow(const int2 *__restrict__ pairs, NarrowArgs na) {
    pdl_wait();
    const unsigned n = min(na.ctr[C_PAIRS], na.cap_pairs);
    unsigned valid = 0;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int2 p = pairs[q];
        if (p.x < 0) continue;  // hole
        ++valid;
        if (kTest) narrow_test(na, p);
    }
    count_valid(na.ctr, valid);
    narrow_done(na.ctr, na.cap_pairs, na.cap_hits, na.counts64);
}

// The end of a keep, sprout and narrow phase in one launch.  The first
// blocks run the traversals below the overlapping internal entries (the
// sprout half of keepIntLooseIntraFronts, BvttFrontKeepKernels.cu:21-42)
// and test each pair they emit at once; the other blocks test the pairs the
// keep scan emitted, [0, the count its last block recorded).  The pair list
// is the same as with k_sprout followed by k_narrow (the scan's pairs, then
// the traversals'), and so are the hits and counts.
template <bool kTest, int kB>
__global__ void __launch_bounds__(kB) k_keep_tail(FArgs a, NarrowArgs na) {
    pdl_wait();
    Em em;
    unsigned valid = 0;
    const unsigned nwork = min(a.ctr[C_WORK], a.cap_work);
    const unsigned na_blocks = min((nwork + kB - 1) / kB, gridDim.x - 1u);
    if (blockIdx.x < na_blocks) {
        for (unsigned q = blockIdx.x * kB + threadIdx.x; q < nwork; q += na_blocks * kB) {
            const int2 e = a.work[q];
            if (e.x < 0) continue;  // hole
            float4 plo, phi;
            ldg8(a.prec + 2 * e.x, plo, phi);
            const int node = e.y < 0 ? ~e.y : e.y;  // (as k_sprout: ~R only comes from an inter restructure)
            float4 nlo, nhi;
            node_rec(a, node, nlo, nhi);
            const int4 pf = prim_face(a, e.x);
            traverse_with<false>(a, em, e.x, plo, phi, e.y < 0 ? (node << 1) : left_child_tagged(a, node, nlo),
                                 __float_as_int(nhi.w),
                                 [&](int leaf) {
                                     if (!emit_pair(a, em, e.x, pf, leaf)) return;
                                     ++valid;
                                     if (kTest) narrow_test(na, make_int2(e.x, leaf));
                                 });
        }
        em_close(a, em);
    } else {
        const unsigned ns = min(a.ctr[C_PAIRS_SCAN], na.cap_pairs);
        for (unsigned q = (blockIdx.x - na_blocks) * kB + threadIdx.x; q < ns; q += (gridDim.x - na_blocks) * kB) {
            const int2 p = a.pairs[q];
            if (p.x < 0) continue;  // hole
            ++valid;
            if (kTest) narrow_test(na, p);
        }
    }
    count_valid(na.ctr, valid);
    narrow_done(na.ctr, na.cap_pairs, na.cap_hits, na.counts64);
}

// The precision mode's narrow phase: the FP32 test decides where it is
// certain, the FP64 test where it is not (the flagged pairs, counted), so the
// hits are those of an FP64 evaluation of every pair (tritri.cuh).
template <bool kUnused, int kB>
__global__ void __launch_bounds__(kB) k_narrow_prec(const int2 *__restrict__ pairs, const int4 *__restrict__ sface,
                                                     const float *__restrict__ verts, unsigned *ctr,
                                                     unsigned cap_pairs, int2 *hits, unsigned cap_hits,
                                                     int64_t *counts64) {
    pdl_wait();
    const unsigned n = min(ctr[C_PAIRS], cap_pairs);
    unsigned valid = 0, flagged = 0;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        int2 p = pairs[q];
        if (p.x < 0) continue;  // hole
        ++valid;
        int4 a = __ldg(&sface[p.x]), b = __ldg(&sface[p.y]);
        const v3 A0 = vload(verts, a.x), A1 = vload(verts, a.y), A2 = vload(verts, a.z);
        const v3 B0 = vload(verts, b.x), B1 = vload(verts, b.y), B2 = vload(verts, b.z);
        int hit = prec::tritri_sat32_certain(prec::fk(A0.x, A0.y, A0.z), prec::fk(A1.x, A1.y, A1.z),
                                             prec::fk(A2.x, A2.y, A2.z), prec::fk(B0.x, B0.y, B0.z),
                                             prec::fk(B1.x, B1.y, B1.z), prec::fk(B2.x, B2.y, B2.z));
        if (hit < 0) {
            ++flagged;
            hit = prec::tritri_sat64(prec::mk(A0.x, A0.y, A0.z), prec::mk(A1.x, A1.y, A1.z),
                                     prec::mk(A2.x, A2.y, A2.z), prec::mk(B0.x, B0.y, B0.z),
                                     prec::mk(B1.x, B1.y, B1.z), prec::mk(B2.x, B2.y, B2.z))
                      ? 1
                      : 0;
        }
        if (hit) emit(hits, ctr + C_HITS, cap_hits, make_int2(a.w, b.w), ctr + C_OVERFLOW, 8u);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        valid += __shfl_xor_sync(0xffffffffu, valid, o);
        flagged += __shfl_xor_sync(0xffffffffu, flagged, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (valid) atomicAdd(ctr + C_PAIRS_VALID, valid);
        if (flagged) atomicAdd(ctr + C_FLAGGED, flagged);
    }
    narrow_done(ctr, cap_pairs, cap_hits, counts64);
}

// Contact points of hits (kDist false: midpoint xyz and length of the
// intersection segment; NaN for coplanar pairs) or distances of broad pairs
// (kDist true: w = distance), over pairs of original triangle ids.  With
// kPrec, ill-conditioned cases are evaluated in FP64: nearly parallel planes
// (sin^2 of their angle below 1e-6) for contact points, distances below a
// thousandth of the pair's size for distances.
template <bool kDist, bool kPrec, bool kF64>
__global__ void k_contacts(const int2 *__restrict__ list, const unsigned *__restrict__ count, unsigned cap,
                           const int *__restrict__ faces, const float *__restrict__ verts, void *out_,
                           unsigned *nflag) {
    // kF64: FP64 arithmetic and FP64 results (double4 per item); else float4
    // results, FP64 arithmetic in the precision mode and FP32 otherwise
    constexpr bool kD = kPrec || kF64;
    const unsigned n = min(*count, cap);
    unsigned fl = 0;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int2 pr = list[q];
        prec::V<float> P[3], Q[3];
        for (int k = 0; k < 3; k++) {
            const v3 a = vload(verts, __ldg(faces + 3 * (size_t)pr.x + k));
            const v3 b = vload(verts, __ldg(faces + 3 * (size_t)pr.y + k));
            P[k] = prec::V<float>{a.x, a.y, a.z};
            Q[k] = prec::V<float>{b.x, b.y, b.z};
        }
        prec::V<double> Pd[3], Qd[3];
        if (kD)
            for (int k = 0; k < 3; k++) {
                Pd[k] = prec::V<double>{P[k].x, P[k].y, P[k].z};
                Qd[k] = prec::V<double>{Q[k].x, Q[k].y, Q[k].z};
            }
        double r[4];
        if (!kDist) {
            int st;
            if (kD) {
                double cd = 0.0;
                st = prec::contact_point(Pd, Qd, r, &cd);
                ++fl;
            } else {
                float o[4], cond = 0.f;
                st = prec::contact_point(P, Q, o, &cond);
                for (int k = 0; k < 4; k++) r[k] = o[k];
            }
            if (st != 1) {
                const double nan = __longlong_as_double(0x7ff8000000000000ll);
                r[0] = r[1] = r[2] = nan;
                r[3] = 0.0;
            }
        } else {
            // intersecting pairs are at distance 0 (decided as the narrow phase decides)
            int hit;
            if (kPrec) {
                hit = prec::tritri_sat32_certain(prec::fk(P[0].x, P[0].y, P[0].z), prec::fk(P[1].x, P[1].y, P[1].z),
                                                 prec::fk(P[2].x, P[2].y, P[2].z), prec::fk(Q[0].x, Q[0].y, Q[0].z),
                                                 prec::fk(Q[1].x, Q[1].y, Q[1].z), prec::fk(Q[2].x, Q[2].y, Q[2].z));
                if (hit < 0)
                    hit = prec::tritri_sat64(prec::mk(P[0].x, P[0].y, P[0].z), prec::mk(P[1].x, P[1].y, P[1].z),
                                             prec::mk(P[2].x, P[2].y, P[2].z), prec::mk(Q[0].x, Q[0].y, Q[0].z),
                                             prec::mk(Q[1].x, Q[1].y, Q[1].z), prec::mk(Q[2].x, Q[2].y, Q[2].z));
            } else {
                hit = tritri_sat32(v3{P[0].x, P[0].y, P[0].z}, v3{P[1].x, P[1].y, P[1].z}, v3{P[2].x, P[2].y, P[2].z},
                                   v3{Q[0].x, Q[0].y, Q[0].z}, v3{Q[1].x, Q[1].y, Q[1].z}, v3{Q[2].x, Q[2].y, Q[2].z});
            }
            double d = 0.0;
            if (!hit && kD) {
                d = prec::tri_distance(Pd, Qd, 2.2250738585072014e-308);
                ++fl;
            } else if (!hit) {
                d = prec::tri_distance(P, Q, 1.17549435e-38f);
            }
            r[0] = r[1] = r[2] = 0.0;
            r[3] = d;
        }
        if (kF64) static_cast<double4 *>(out_)[q] = make_double4(r[0], r[1], r[2], r[3]);
        else static_cast<float4 *>(out_)[q] = make_float4((float)r[0], (float)r[1], (float)r[2], (float)r[3]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) fl += __shfl_xor_sync(0xffffffffu, fl, o);
    if ((threadIdx.x & 31) == 0 && fl) atomicAdd(nflag, fl);
}

// Order-preserving compaction of the broad pairs past their holes, into
// original ids: flags, an exclusive scan, a scatter.  Every export of the same
// frame lists the pairs in the same order (their slot order).
__global__ void k_pair_flags(const int2 *__restrict__ pairs, const unsigned *__restrict__ ctr, unsigned cap,
                             unsigned n_all, unsigned *flags) {
    const unsigned n = min(ctr[C_PAIRS], cap);
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < n_all; q += gridDim.x * blockDim.x)
        flags[q] = (q < n && pairs[q].x >= 0) ? 1u : 0u;
}
__global__ void k_pair_scatter(const int2 *__restrict__ pairs, const int4 *__restrict__ psface,
                               const int4 *__restrict__ sface, int leaf_first, const unsigned *__restrict__ ctr,
                               unsigned cap, const unsigned *__restrict__ flags, const unsigned *__restrict__ pos,
                               int2 *out) {
    const unsigned n = min(ctr[C_PAIRS], cap);
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
        if (flags[q]) {
            const int2 p = pairs[q];
            const int a = __ldg(&psface[p.x]).w, b = __ldg(&sface[p.y]).w;
            out[pos[q]] = leaf_first ? make_int2(b, a) : make_int2(a, b);
        }
}

// Start of a maintain: the previous maintain's overflow bits join the sticky
// record, and the bits that say the current front is incomplete (an entry or
// a traversal was lost: bits 0, 1, 4, 5) carry over when this maintain works
// from that front (keep, update, balance), since its results are then
// incomplete too; a generation starts clean.
// The carried bits are joined by bit 6, which says that this maintain's own
// results (pairs, hits) are incomplete because its input front was.
constexpr unsigned kFrontLossBits = 1u | 2u | 16u | 32u | 64u;
// Lane k < C_NUM also zeroes counter k when bit k of `zero` is set (the
// maintain's first attempt starts its stage and narrow-phase counters here
// instead of in a memset each).
__global__ void k_ovf_roll(unsigned *ctr, unsigned carry, unsigned zero) {
    // the next kernel may start at once (it waits for this one); this one
    // waits for the kernel before it, so completion stays in order
    pdl_release();
    pdl_wait();
    if (threadIdx.x == 0) {
        const unsigned o = ctr[C_OVERFLOW];
        ctr[C_OVF_STICKY] |= o;
        ctr[C_OVERFLOW] = (o & carry) ? ((o & carry) | 64u) : 0u;
    }
    if (threadIdx.x < C_NUM && ((zero >> threadIdx.x) & 1u)) ctr[threadIdx.x] = 0u;
}

__global__ void k_counts64(const unsigned *__restrict__ ctr, unsigned cap_pairs, unsigned cap_hits,
                           int64_t *out) {
    if (threadIdx.x == 0) {
        out[0] = min(ctr[C_PAIRS_VALID], cap_pairs);
        out[1] = min(ctr[C_HITS], cap_hits);
    }
}

unsigned resident_blocks(const void *kernel, int block = kThreads) {
    int nb = 0, dev = 0, sms = kSms;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, 0);
    return (unsigned)((nb > 0 ? nb : 1) * sms);
}

}  // namespace

// A launch, with programmatic stream serialisation when `pdl` (the kernel
// then waits with pdl_wait before it reads what earlier kernels wrote).
template <typename... KArgs, typename... Args>
void launch_k(bool pdl, void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
              Args &&...args) {
    if (!pdl) {
        k<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

// One resident wave of blocks (blocks per SM at this kernel's occupancy x SM
// count): the grid-stride kernels then run without a tail wave.
#define RESIDENT(K) ([]() { static unsigned g_ = 0; if (!g_) g_ = resident_blocks((const void *)(K)); return g_; }())
#define RESIDENT_B(K, B) \
    ([]() { static unsigned g_ = 0; if (!g_) g_ = resident_blocks((const void *)(K), B); return g_; }())
// Front scans in a launch shape: entries per thread step (1, 2, 4) x threads
// per block (128, 256, 512).
#define SCAN_AT(KERNEL, U, B, S, ARG) launch_k(pdl_, KERNEL<U, B>, RESIDENT_B((KERNEL<U, B>), B), B, 0, S, ARG)
#define SCAN_U(KERNEL, U, B, S, ARG)                 \
    do {                                             \
        if ((U) == 1) SCAN_AT(KERNEL, 1, B, S, ARG); \
        else if ((U) == 4) SCAN_AT(KERNEL, 4, B, S, ARG); \
        else SCAN_AT(KERNEL, 2, B, S, ARG);          \
    } while (0)
#define LAUNCH_SCAN(KERNEL, SH, S, ARG)                            \
    do {                                                           \
        if ((SH).b == 128) SCAN_U(KERNEL, (SH).u, 128, S, ARG);      \
        else if ((SH).b == 512) SCAN_U(KERNEL, (SH).u, 512, S, ARG); \
        else SCAN_U(KERNEL, (SH).u, 256, S, ARG);                    \
        note_launch();                                             \
    } while (0)
// Per-item kernels (sprout, narrow phase) in a block size.
#define ITEM_AT(KERNEL, F, B, S, ...) launch_k(pdl_, KERNEL<F, B>, RESIDENT_B((KERNEL<F, B>), B), B, 0, S, __VA_ARGS__)
#define LAUNCH_ITEM(KERNEL, F, SH, S, ...)                                \
    do {                                                                  \
        if ((SH).b == 128) ITEM_AT(KERNEL, F, 128, S, __VA_ARGS__);         \
        else if ((SH).b == 512) ITEM_AT(KERNEL, F, 512, S, __VA_ARGS__);    \
        else ITEM_AT(KERNEL, F, 256, S, __VA_ARGS__);                       \
        note_launch();                                                    \
    } while (0)

// ====================================================================== host
Front::~Front() {
    for (auto &set : front_)
        for (auto &b : set) b.release();
    DBuf *bufs[] = {&pairs_, &hits_, &outbuf_, &work_, &logcnt_, &intbeg_, &extbeg_,
                    &snapshot_, &scratch_, &counts64_, &cbuf_, &cflag_, &cscratch_, &fctr_, &rcur_,
                    &pxbuf_, &pxout_, &iexp_, &xexp_, &ksel_};
    for (DBuf *b : bufs) b->release();
    for (int k = 0; k < kSnap; k++)
        if (snap_ev_[k]) cudaEventDestroy(snap_ev_[k]);
    if (h_snap_) cudaFreeHost(h_snap_);
}

bvhcd_status Front::init() {
    if (const char *u = getenv("BVHCD_FRONT_UNROLL")) {
        const int v = atoi(u);
        for (int k = 0; k < BVHCD_SHAPE_COUNT; k++)
            if (v == 1 || v == 2 || v == 4) shape_[k].u = v;
    }
    if (cfg_.int_front_capacity <= 0 || cfg_.ext_front_capacity <= 0 || cfg_.pair_capacity <= 0)
        return BVHCD_INVALID_ARG;
    if (cfg_.auto_grow < 0 || cfg_.auto_grow > 2) return BVHCD_INVALID_ARG;
    if (cfg_.int_front_capacity > 0x7fffffffLL || cfg_.ext_front_capacity > 0x7fffffffLL ||
        cfg_.pair_capacity > 0x7fffffffLL)
        return BVHCD_INVALID_ARG;
    fcap_[0] = cfg_.int_front_capacity;
    fcap_[1] = cfg_.ext_front_capacity;
    pcap_ = cfg_.pair_capacity;
    for (int set = 0; set < 2; set++)
        for (int k = 0; k < 2; k++) FR_TRY(front_[set][k].reserve(sizeof(int2) * (size_t)fcap_[k]));
    FR_TRY(pairs_.reserve(sizeof(int2) * (size_t)pcap_));
    FR_TRY(hits_.reserve(sizeof(int2) * (size_t)pcap_));
    FR_TRY(work_.reserve(sizeof(int2) * (size_t)fcap_[0]));
    FR_TRY(iexp_.reserve(sizeof(float) * (size_t)fcap_[0]));
    FR_TRY(xexp_.reserve(sizeof(float) * (size_t)fcap_[1]));
    FR_TRY(ksel_.reserve(sizeof(unsigned) * (size_t)(fcap_[0] + fcap_[1])));
    FR_TRY(counts64_.reserve(sizeof(int64_t) * 2));
    FR_TRY(fctr_.reserve(sizeof(unsigned) * C_NUM));
    FR_TRY(cudaMemset(fctr_.p, 0, sizeof(unsigned) * C_NUM));
    return ensure_node_capacity(bvh_->T() > 0 ? bvh_->T() : 1);
}

bvhcd_status Front::ensure_node_capacity(int T) {
    if (T <= capT_) return BVHCD_OK;
    size_t n = (size_t)T + 2;
    FR_TRY(logcnt_.reserve(sizeof(unsigned) * 4 * n));
    FR_TRY(intbeg_.reserve(sizeof(unsigned) * n));
    FR_TRY(extbeg_.reserve(sizeof(unsigned) * n));
    FR_TRY(snapshot_.reserve(sizeof(float) * n));
    FR_TRY(scratch_.reserve(scan_scratch_bytes((int64_t)n)));
    FR_TRY(rcur_.reserve(sizeof(unsigned) * 2 * reorder_groups(T)));
    FR_TRY(cudaMemset(logcnt_.p, 0, sizeof(unsigned) * 4 * n));
    logn_ = n;
    FR_TRY(cudaMemset(intbeg_.p, 0, sizeof(unsigned) * n));
    FR_TRY(cudaMemset(extbeg_.p, 0, sizeof(unsigned) * n));
    FR_TRY(cudaMemset(snapshot_.p, 0, sizeof(float) * n));
    capT_ = T;
    return BVHCD_OK;
}

FrontLog Front::log() const {
    FrontLog l;
    unsigned *c = logcnt_.as<unsigned>();
    l.intcnt = c;
    l.extcnt = c + logn_;
    l.intback = c + 2 * logn_;
    l.extback = c + 3 * logn_;
    l.intbeg = intbeg_.as<unsigned>();
    l.extbeg = extbeg_.as<unsigned>();
    return l;
}

// The work list's capacity is what its buffer holds, never a front capacity
// that may have grown past it.
static FArgs make_args(const LBvh *bvh, const LBvh *trav, unsigned *ctr, const FrontLog &log, int cull,
                       const DBuf &work) {
    const int64_t cap_work = (int64_t)(work.bytes / sizeof(int2));
    Tree t = bvh->tree();
    FArgs a;
    a.nrec = t.nrec; a.lrec = t.lrec; a.topo = t.topo; a.lca = t.lca; a.sface = t.sface;
    a.nrec16 = t.nrec16; a.nrange = t.nrange;
    a.prec = trav ? trav->tree().lrec : t.lrec;
    a.nprim = trav ? trav->T() : t.T;
    a.inter = trav ? 1 : 0;
    a.root_tag = t.T >= 2 ? 0 : 1;  // internal node 0, or the single leaf
    a.log = log;
    a.ctr = ctr;
    a.in_int = a.in_ext = nullptr;
    a.out_int = a.out_ext = nullptr;
    a.in_int_slot = C_INT0; a.in_ext_slot = C_EXT0; a.out_int_slot = C_INT1; a.out_ext_slot = C_EXT1;
    a.cap_int = a.cap_ext = 0;
    a.pairs = nullptr;
    a.cap_pairs = 0;
    a.work = work.as<int2>();
    a.cap_work = (unsigned)(cap_work < 0xffffffffLL ? cap_work : 0xffffffffLL);
    a.cull = trav ? 0 : cull;  // vertex sharing means nothing across two meshes
    a.T = t.T;
    a.motion = nullptr;
    a.iexp_in = a.xexp_in = nullptr;
    a.iexp_out = a.xexp_out = nullptr;
    a.ksel = nullptr;
    a.rs_mark = a.rs_root = a.rs_last = nullptr;
    a.snap_scan = 0;
    return a;
}

// log clear (FlOrderLog.cpp clear): counts and back counts, one memset
cudaError_t Front::log_clear(cudaStream_t s) const {
    return cudaMemsetAsync(logcnt_.p, 0, sizeof(unsigned) * 4 * logn_, s);
}

// FlOrderLog::prepare (FlOrderLog.cu:7-12): begins from counts
static cudaError_t log_prepare(const FrontLog &l, int T, void *scratch, cudaStream_t s) {
    return scan2_u32(l.intcnt, l.intbeg, l.extcnt, l.extbeg, T + 1, scratch, s);
}

bvhcd_status Front::reorder(cudaStream_t s) {
    StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_FRONT_REORDER, s);
    const int T = bvh_->T();
    FrontLog l = log();
    FR_TRY(log_prepare(l, T, scratch_.p, s));
    exp_valid_ = false;  // the fronts move
    const size_t ng = reorder_groups(T);
    FR_TRY(cudaMemsetAsync(rcur_.p, 0, sizeof(unsigned) * 2 * ng, s));
    FArgs a = make_args(bvh_, trav_, counters(), l, cfg_.cull_adjacent, work_);
    const int nx = 1 - cur_;
    a.in_int = front_[nx][0].as<int2>(); a.in_ext = front_[nx][1].as<int2>();
    a.out_int = front_[cur_][0].as<int2>(); a.out_ext = front_[cur_][1].as<int2>();
    a.in_int_slot = 2 * nx; a.in_ext_slot = 2 * nx + 1;
    a.out_int_slot = 2 * cur_; a.out_ext_slot = 2 * cur_ + 1;
    a.cap_int = (unsigned)fcap_[0]; a.cap_ext = (unsigned)fcap_[1];
    static const unsigned grid = [] {
        cudaFuncSetAttribute(k_reorder, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kReorderSmem);
        int nb = 0, dev = 0, sms = kSms;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_reorder, kReorderThreads, kReorderSmem);
        return (unsigned)((nb > 0 ? nb : 1) * sms);
    }();
    k_reorder<<<grid, kReorderThreads, kReorderSmem, s>>>(a, rcur_.as<unsigned>(), rcur_.as<unsigned>() + ng);
    note_launch();
    log_counted_ = true;  // the emission before it counted every entry
    return cuda_status(cudaGetLastError());
}

// Emission into the other buffer set; the caller reorders back.
bvhcd_status Front::generate(cudaStream_t s, bool pure) {
    const int T = bvh_->T();
    unsigned *ctr = counters();
    FrontLog l = log();
    FArgs a = make_args(bvh_, trav_, counters(), l, cfg_.cull_adjacent, work_);
    a.pairs = pairs_.as<int2>();
    a.cap_pairs = (unsigned)pcap_;
    if (!zeroed_) FR_TRY(cudaMemsetAsync(ctr + C_PAIRS, 0, sizeof(unsigned), s));
    if (pure) {
        StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_PURE_BVH_CD, s);
        k_generate<false><<<grid_for(a.inter ? a.nprim : T), kThreads, 0, s>>>(a); note_launch();
        return cuda_status(cudaGetLastError());
    }
    FR_TRY(log_clear(s));
    const int nx = 1 - cur_;
    a.out_int = front_[nx][0].as<int2>(); a.out_ext = front_[nx][1].as<int2>();
    a.out_int_slot = 2 * nx; a.out_ext_slot = 2 * nx + 1;
    a.cap_int = (unsigned)fcap_[0]; a.cap_ext = (unsigned)fcap_[1];
    if (!zeroed_) FR_TRY(cudaMemsetAsync(ctr + 2 * nx, 0, 2 * sizeof(unsigned), s));
    {
        StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_FRONT_GENERATE, s);
        k_generate<true><<<grid_for(a.inter ? a.nprim : T), kThreads, 0, s>>>(a); note_launch();
    }
    FR_TRY(cudaGetLastError());
    bvhcd_status st = reorder(s);
    if (st != BVHCD_OK) return st;
    has_front_ = true;
    seen_epoch_[0] = bvh_->topo_epoch();
    seen_epoch_[1] = trav()->topo_epoch();
    if (bvh_->restr_enabled() && !inter()) return snapshot(s);
    return BVHCD_OK;
}

bvhcd_status Front::snapshot(cudaStream_t s) {
    const int T = bvh_->T();
    Tree t = bvh_->tree();
    k_snapshot<<<grid_for(T), kThreads, 0, s>>>(T - 1, t.nrange, intbeg_.as<unsigned>(), extbeg_.as<unsigned>(),
                                                snapshot_.as<float>()); note_launch();
    return cuda_status(cudaGetLastError());
}

bvhcd_status Front::check_quality(cudaStream_t s) {
    StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_QUALITY, s);
    const int T = bvh_->T();
    Tree t = bvh_->tree();
    k_fill_i32<<<grid_for(T), kThreads, 0, s>>>(T, bvh_->rtroot(), INT_MAX); note_launch();
    FR_TRY(cudaMemsetAsync(bvh_->intrange(), 0, sizeof(int) * (size_t)T, s));
    k_check_quality<<<grid_for(T), kThreads, 0, s>>>(T - 1, t.nrange, intbeg_.as<unsigned>(),
                                                     extbeg_.as<unsigned>(), snapshot_.as<float>(),
                                                     bvh_->intrange(), bvh_->rtroot()); note_launch();
    FR_TRY(cudaGetLastError());
    bvh_->set_updated(true);
    return BVHCD_OK;
}

// pruneSprout (BvttFrontLooseIntra.cu:254-283): the update kernels write the
// new front into the other buffer set, then the quality check and the
// reorder back.
bvhcd_status Front::update_kernels(cudaStream_t s) {
    const int T = bvh_->T();
    unsigned *ctr = counters();
    FrontLog l = log();
    FR_TRY(log_clear(s));
    FArgs a = make_args(bvh_, trav_, counters(), l, cfg_.cull_adjacent, work_);
    const int nx = 1 - cur_;
    a.in_int = front_[cur_][0].as<int2>(); a.in_ext = front_[cur_][1].as<int2>();
    a.in_int_slot = 2 * cur_; a.in_ext_slot = 2 * cur_ + 1;
    a.out_int = front_[nx][0].as<int2>(); a.out_ext = front_[nx][1].as<int2>();
    a.out_int_slot = 2 * nx; a.out_ext_slot = 2 * nx + 1;
    a.cap_int = (unsigned)fcap_[0]; a.cap_ext = (unsigned)fcap_[1];
    a.pairs = pairs_.as<int2>();
    a.cap_pairs = (unsigned)pcap_;
    if (!zeroed_) {
        FR_TRY(cudaMemsetAsync(ctr + 2 * nx, 0, 2 * sizeof(unsigned), s));
        FR_TRY(cudaMemsetAsync(ctr + C_PAIRS, 0, sizeof(unsigned), s));
        FR_TRY(cudaMemsetAsync(ctr + C_WORK, 0, sizeof(unsigned), s));
    }
    {
        StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_FRONT_UPDATE, s);
        LAUNCH_SCAN(k_maintain_int_scan, shape_[BVHCD_SHAPE_PRUNE_INT], s, a);
        LAUNCH_SCAN(k_maintain_ext, shape_[BVHCD_SHAPE_PRUNE_EXT], s, a);
        LAUNCH_ITEM(k_sprout, true, shape_[BVHCD_SHAPE_SPROUT], s, a);
    }
    return cuda_status(cudaGetLastError());
}

// BvttFrontLooseInter::restructure (BvttFrontLooseInter.cu:252-318): the
// traversed BVH restructured subtrees since this inter front was last made or
// restructured; valid entries are kept (or sprouted), the entries inside each
// restructured subtree are replaced by one traversal of the new subtree per
// primitive (k_restr_scan), then the usual ordering.  The reference also
// prunes right after; here the next UPDATE does.
bvhcd_status Front::restructure_inter(cudaStream_t s) {
    const int T = bvh_->T();
    unsigned *ctr = counters();
    FrontLog l = log();
    FR_TRY(log_clear(s));
    FArgs a = make_args(bvh_, trav_, counters(), l, cfg_.cull_adjacent, work_);
    const int nx = 1 - cur_;
    a.in_int = front_[cur_][0].as<int2>(); a.in_ext = front_[cur_][1].as<int2>();
    a.in_int_slot = 2 * cur_; a.in_ext_slot = 2 * cur_ + 1;
    a.out_int = front_[nx][0].as<int2>(); a.out_ext = front_[nx][1].as<int2>();
    a.out_int_slot = 2 * nx; a.out_ext_slot = 2 * nx + 1;
    a.cap_int = (unsigned)fcap_[0]; a.cap_ext = (unsigned)fcap_[1];
    a.pairs = pairs_.as<int2>();
    a.cap_pairs = (unsigned)pcap_;
    a.rs_mark = bvh_->rs_intmark();
    a.rs_root = bvh_->rs_leafroot();
    a.rs_last = bvh_->rs_oldlast();
    FR_TRY(cudaMemsetAsync(ctr + 2 * nx, 0, 2 * sizeof(unsigned), s));
    FR_TRY(cudaMemsetAsync(ctr + C_PAIRS, 0, sizeof(unsigned), s));
    FR_TRY(cudaMemsetAsync(ctr + C_WORK, 0, sizeof(unsigned), s));
    {
        StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_FRONT_RESTRUCTURE, s);
        LAUNCH_SCAN(k_restr_scan, shape_[BVHCD_SHAPE_PRUNE_INT], s, a);
        LAUNCH_ITEM(k_sprout, true, shape_[BVHCD_SHAPE_SPROUT], s, a);
    }
    FR_TRY(cudaGetLastError());
    bvhcd_status st = reorder(s);
    if (st != BVHCD_OK) return st;
    seen_epoch_[0] = bvh_->topo_epoch();
    seen_epoch_[1] = trav()->topo_epoch();
    return BVHCD_OK;
}

bvhcd_status Front::prune_sprout(cudaStream_t s) {
    bvhcd_status st = update_kernels(s);
    if (st != BVHCD_OK) return st;
    if (bvh_->restr_enabled() && quality_check_ && !inter()) {
        st = check_quality(s);
        if (st != BVHCD_OK) return st;
    }
    return reorder(s);
}

bvhcd_status Front::keep(cudaStream_t s) {
    StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_FRONT_KEEP, s);
    unsigned *ctr = counters();
    FArgs a = make_args(bvh_, trav_, counters(), log(), cfg_.cull_adjacent, work_);
    a.in_int = front_[cur_][0].as<int2>(); a.in_ext = front_[cur_][1].as<int2>();
    a.in_int_slot = 2 * cur_; a.in_ext_slot = 2 * cur_ + 1;
    a.cap_int = (unsigned)fcap_[0]; a.cap_ext = (unsigned)fcap_[1];
    a.pairs = pairs_.as<int2>();
    a.cap_pairs = (unsigned)pcap_;
    if (!zeroed_) {
        FR_TRY(cudaMemsetAsync(ctr + C_PAIRS, 0, sizeof(unsigned), s));
        FR_TRY(cudaMemsetAsync(ctr + C_WORK, 0, sizeof(unsigned), s));
    }
    // expiries: an intra front over FP32 node boxes (an inter front's
    // primitives move with another tree; FP16 boxes move by their rounding too)
    const bool expiries = !inter() && !cfg_.precision && !bvh_->tree().nrec16;
    if (exp_epoch_ != bvh_->topo_epoch() || exp_faces_ != bvh_->faces_epoch()) exp_valid_ = false;
    if (expiries) {
        a.motion = bvh_->counters() + C_MOTION;
        a.iexp_out = iexp_.as<float>();
        a.xexp_out = xexp_.as<float>();
        if (exp_valid_) {
            a.iexp_in = iexp_.as<float>();
            a.xexp_in = xexp_.as<float>();
            if (!zeroed_) FR_TRY(cudaMemsetAsync(ctr + C_KSEL, 0, sizeof(unsigned), s));
            launch_k(pdl_, k_keep_select, RESIDENT(k_keep_select), kThreads, 0, s, a, ksel_.as<unsigned>(),
                     ctr + C_KSEL);
            note_launch();
            a.ksel = ksel_.as<unsigned>();
        }
    }
    last_keep_sel_ = a.ksel != nullptr;
    a.snap_scan = keep_tail_ ? 1 : 0;
    LAUNCH_SCAN(k_keep_scan, shape_[BVHCD_SHAPE_KEEP], s, a);
    if (expiries) {
        exp_valid_ = true;
        exp_epoch_ = bvh_->topo_epoch();
        exp_faces_ = bvh_->faces_epoch();
    }
    if (keep_tail_) {
        // the narrow phase's counters start at zero (the maintain's prologue
        // zeroed them on its first attempt)
        if (!zeroed_) {
            FR_TRY(cudaMemsetAsync(ctr + C_HITS, 0, sizeof(unsigned), s));
            FR_TRY(cudaMemsetAsync(ctr + C_PAIRS_VALID, 0, sizeof(unsigned), s));
            FR_TRY(cudaMemsetAsync(ctr + C_FLAGGED, 0, sizeof(unsigned), s));
        }
        // (timed as part of the keep stage)
        // (in the keep stage's block size: most of the tail's work is the scan's
        // pairs, not sprouts)
        const Shape tail{1, shape_[BVHCD_SHAPE_KEEP].b};
        if (cfg_.narrow_phase) LAUNCH_ITEM(k_keep_tail, true, tail, s, a, narrow_args());
        else LAUNCH_ITEM(k_keep_tail, false, tail, s, a, narrow_args());
        tail_ran_ = true;
        return cuda_status(cudaGetLastError());
    }
    LAUNCH_ITEM(k_sprout, false, shape_[BVHCD_SHAPE_SPROUT], s, a);
    return cuda_status(cudaGetLastError());
}

// balance (BvttFrontLooseIntra.cu:285-312).  The external front stays where
// it is; only the internal front moves to the other buffer.
bvhcd_status Front::balance_kernels(cudaStream_t s) {
    const int T = bvh_->T();
    unsigned *ctr = counters();
    FrontLog l = log();
    // A balance leaves a node's entries counted in two halves (intcnt from
    // the front of its bucket, intback from the back) and the external counts
    // cleared, but it moves no entry to another node: the begins it started
    // from still hold, and a balance that follows one (with only keeps in
    // between) starts from them again.  The reference scans the counts every
    // time (BvttFrontLooseIntra.cu:286), which places a second balance's
    // entries over one another; its schedules never run two in a row.
    if (log_counted_) FR_TRY(log_prepare(l, T, scratch_.p, s));
    FR_TRY(log_clear(s));
    log_counted_ = false;
    exp_valid_ = false;  // the internal front moves
    FArgs a = make_args(bvh_, trav_, counters(), l, cfg_.cull_adjacent, work_);
    const int nx = 1 - cur_;
    a.in_int = front_[cur_][0].as<int2>(); a.in_ext = front_[cur_][1].as<int2>();
    a.in_int_slot = 2 * cur_; a.in_ext_slot = 2 * cur_ + 1;
    a.out_int = front_[nx][0].as<int2>();
    a.out_int_slot = 2 * nx;
    a.cap_int = (unsigned)fcap_[0]; a.cap_ext = (unsigned)fcap_[1];
    a.pairs = pairs_.as<int2>();
    a.cap_pairs = (unsigned)pcap_;
    FR_TRY(cudaMemsetAsync(ctr + C_PAIRS, 0, sizeof(unsigned), s));
    FR_TRY(cudaMemsetAsync(ctr + C_WORK, 0, sizeof(unsigned), s));
    LAUNCH_SCAN(k_balance_scan, shape_[BVHCD_SHAPE_BALANCE], s, a);
    LAUNCH_ITEM(k_sprout, false, shape_[BVHCD_SHAPE_SPROUT], s, a);
    return cuda_status(cudaGetLastError());
}

bvhcd_status Front::balance(cudaStream_t s) {
    StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_FRONT_BALANCE, s);
    bvhcd_status st = balance_kernels(s);
    if (st != BVHCD_OK) return st;
    unsigned *ctr = counters();
    const int nx = 1 - cur_;
    // swap the internal front buffers of the two sets, keep the external one
    std::swap(front_[0][0], front_[1][0]);
    int_swapped_ = !int_swapped_;
    FR_TRY(cudaMemcpyAsync(ctr + 2 * cur_, ctr + 2 * nx, sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
    return BVHCD_OK;
}

NarrowArgs Front::narrow_args() {
    NarrowArgs n;
    n.psface = trav()->tree().sface;
    n.pverts = trav()->verts4();
    n.sface = bvh_->tree().sface;
    n.verts = bvh_->verts4();
    n.leaf_first = inter() ? 1 : 0;
    n.ctr = counters();
    n.hits = hits_.as<int2>();
    n.cap_pairs = (unsigned)pcap_;
    n.cap_hits = (unsigned)pcap_;
    n.counts64 = counts64_.as<int64_t>();
    return n;
}

bvhcd_status Front::narrow(cudaStream_t s, bool test) {
    StageScope prof_scope(bvh_->profiler(), BVHCD_STAGE_NARROW, s);
    unsigned *ctr = counters();
    if (!zeroed_) {
        FR_TRY(cudaMemsetAsync(ctr + C_HITS, 0, sizeof(unsigned), s));
        FR_TRY(cudaMemsetAsync(ctr + C_PAIRS_VALID, 0, sizeof(unsigned), s));
        FR_TRY(cudaMemsetAsync(ctr + C_FLAGGED, 0, sizeof(unsigned), s));
    }
    const Shape sh = shape_[BVHCD_SHAPE_NARROW];
    int64_t *c64 = counts64_.as<int64_t>();
    if (test && cfg_.precision)
        LAUNCH_ITEM(k_narrow_prec, true, sh, s, pairs_.as<int2>(), bvh_->tree().sface, bvh_->verts(), ctr,
                    (unsigned)pcap_, hits_.as<int2>(), (unsigned)pcap_, c64);
    else if (test)
        LAUNCH_ITEM(k_narrow, true, sh, s, pairs_.as<int2>(), narrow_args());
    else
        LAUNCH_ITEM(k_narrow, false, sh, s, pairs_.as<int2>(), narrow_args());
    return cuda_status(cudaGetLastError());
}

bvhcd_status Front::run(bvhcd_front_op op, cudaStream_t s) {
    switch (op) {
    case BVHCD_FRONT_PURE_BVH_CD: return generate(s, true);
    case BVHCD_FRONT_GENERATE: return generate(s, false);
    case BVHCD_FRONT_UPDATE: return prune_sprout(s);
    case BVHCD_FRONT_REORDER: return balance(s);
    case BVHCD_FRONT_KEEP: return keep(s);
    case BVHCD_FRONT_RESTRUCTURE: return restructure_inter(s);
    default: return generate(s, false);
    }
}

bvhcd_status Front::grow_and_check(cudaStream_t s, unsigned *ovf_bits) {
    unsigned h[C_NUM];
    FR_TRY(cudaMemcpyAsync(h, counters(), sizeof(h), cudaMemcpyDeviceToHost, s));
    FR_TRY(cudaStreamSynchronize(s));
    *ovf_bits = h[C_OVERFLOW];
    if (!*ovf_bits) return BVHCD_OK;
    bvhcd_status st = grow_from(h, s);
    if (st != BVHCD_OK) return st;
    FR_TRY(cudaMemsetAsync(counters() + C_OVERFLOW, 0, sizeof(unsigned), s));
    return BVHCD_OK;
}

// Deferred capacity check (auto_grow = 2): the counters of each of the last
// kSnap maintains are copied into pinned host memory on the work stream, each
// copy with an event.  A maintain looks at the copies whose events have
// completed (it waits only for the slot it is about to reuse, a maintain
// kSnap - 1 calls back); one that shows an overflow in a maintain made since
// the last regeneration grows the buffers from its counts and makes this
// maintain regenerate the front.  No synchronisation in the steady state;
// the frames between the overflow and the regeneration report it.
bvhcd_status Front::deferred_check(cudaStream_t s, bool *regen) {
    *regen = false;
    if (!h_snap_) {
        FR_TRY(cudaMallocHost(reinterpret_cast<void **>(&h_snap_), sizeof(unsigned) * C_NUM * kSnap));
        for (int k = 0; k < kSnap; k++) FR_TRY(cudaEventCreateWithFlags(&snap_ev_[k], cudaEventDisableTiming));
    }
    const int reuse = (int)(seq_ % kSnap);
    for (int k = 0; k < kSnap; k++) {
        if (snap_seq_[k] < 0) continue;
        cudaError_t q = cudaEventQuery(snap_ev_[k]);
        if (q == cudaErrorNotReady && k == reuse) q = cudaEventSynchronize(snap_ev_[k]);
        if (q == cudaErrorNotReady) continue;
        FR_TRY(q);
        const unsigned *h = h_snap_ + (size_t)k * C_NUM;
        if (h[C_OVERFLOW] != 0 && snap_seq_[k] >= regen_seq_) {
            bvhcd_status st = grow_from(h, s);  // (synchronises s: rare)
            if (st != BVHCD_OK) return st;
            *regen = true;
        }
        snap_seq_[k] = -1;
    }
    if (*regen) regen_seq_ = seq_;
    return BVHCD_OK;
}

bvhcd_status Front::deferred_snapshot(cudaStream_t s) {
    const int k = (int)(seq_ % kSnap);
    FR_TRY(cudaMemcpyAsync(h_snap_ + (size_t)k * C_NUM, counters(), sizeof(unsigned) * C_NUM,
                           cudaMemcpyDeviceToHost, s));
    FR_TRY(cudaEventRecord(snap_ev_[k], s));
    snap_seq_[k] = seq_++;
    return BVHCD_OK;
}

// Buffers grown to the sizes the counters `h` of an overflowed maintain ask
// for (reserved slots, so at least the true sizes), half as much again.
bvhcd_status Front::grow_from(const unsigned *h, cudaStream_t s) {
    int64_t need_int = (int64_t)(h[C_INT0] > h[C_INT1] ? h[C_INT0] : h[C_INT1]);
    int64_t need_ext = (int64_t)(h[C_EXT0] > h[C_EXT1] ? h[C_EXT0] : h[C_EXT1]);
    int64_t need_pairs = (int64_t)(h[C_PAIRS] > h[C_HITS] ? h[C_PAIRS] : h[C_HITS]);
    auto grow = [](int64_t need, int64_t cur) {
        int64_t g = need + need / 2 + 1024;
        if (g > 0x7fffffffLL) g = 0x7fffffffLL;
        return g > cur ? g : cur;
    };
    const int64_t nc[2] = {grow(need_int, fcap_[0]), grow(need_ext, fcap_[1])};
    const int64_t npc = grow(need_pairs, pcap_);
    const bool gf[2] = {nc[0] > fcap_[0], nc[1] > fcap_[1]}, gp = npc > pcap_;
    // Every grown buffer is allocated before the handle changes: if one
    // allocation fails the others are released and the front keeps its old,
    // consistent buffers (no capacity ever exceeds the buffer behind it).
    DBuf nf[2][2], nwork, niexp, nxexp, nksel, npairs, nhits;
    DBuf *tmp[] = {&nf[0][0], &nf[0][1], &nf[1][0], &nf[1][1], &nwork, &niexp, &nxexp, &nksel, &npairs, &nhits};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; k++)
        for (int set = 0; set < 2 && gf[k] && e == cudaSuccess; set++) e = nf[set][k].reserve(sizeof(int2) * (size_t)nc[k]);
    // every work item comes from one internal entry of the input front
    if (e == cudaSuccess && gf[0]) e = nwork.reserve(sizeof(int2) * (size_t)nc[0]);
    if (e == cudaSuccess && gf[0]) e = niexp.reserve(sizeof(float) * (size_t)nc[0]);
    if (e == cudaSuccess && gf[1]) e = nxexp.reserve(sizeof(float) * (size_t)nc[1]);
    if (e == cudaSuccess && (gf[0] || gf[1])) e = nksel.reserve(sizeof(unsigned) * (size_t)(nc[0] + nc[1]));
    if (e == cudaSuccess && gp) e = npairs.reserve(sizeof(int2) * (size_t)npc);
    if (e == cudaSuccess && gp) e = nhits.reserve(sizeof(int2) * (size_t)npc);
    // the current front survives in set cur_: copied into its grown buffers
    for (int k = 0; k < 2 && e == cudaSuccess; k++)
        if (gf[k]) e = cudaMemcpyAsync(nf[cur_][k].p, front_[cur_][k].p, sizeof(int2) * (size_t)fcap_[k],
                                       cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // nothing queued still reads the old buffers
    if (e != cudaSuccess) {
        for (DBuf *b : tmp) b->release();
        return cuda_status(e);
    }
    auto swap_in = [](DBuf &dst, DBuf &src) {
        dst.release();
        dst = src;
        src = DBuf{};
    };
    for (int k = 0; k < 2; k++) {
        if (!gf[k]) continue;
        for (int set = 0; set < 2; set++) swap_in(front_[set][k], nf[set][k]);
        fcap_[k] = nc[k];
        exp_valid_ = false;
    }
    if (gf[0]) {
        swap_in(work_, nwork);
        swap_in(iexp_, niexp);
    }
    if (gf[1]) swap_in(xexp_, nxexp);
    if (gf[0] || gf[1]) swap_in(ksel_, nksel);
    if (gp) {
        swap_in(pairs_, npairs);
        swap_in(hits_, nhits);
        pcap_ = npc;
    }
    return BVHCD_OK;
}

// BvttFrontLooseIntra::maintain (BvttFrontLooseIntra.cu:69-126)
bvhcd_status Front::maintain(bvhcd_front_op op, cudaStream_t s) {
    if (op < BVHCD_FRONT_PURE_BVH_CD || op > BVHCD_FRONT_RESTRUCTURE) return BVHCD_INVALID_ARG;
    if (!bvh_->built() || !trav()->built()) return BVHCD_NOT_READY;
    if (inter() && (bvh_->num_scenes() != 1 || trav_->num_scenes() != 1)) return BVHCD_INVALID_ARG;
    // a box scene has no triangles to test
    if (cfg_.narrow_phase && (bvh_->box_input() || trav()->box_input())) return BVHCD_INVALID_ARG;
    const int T = bvh_->T();
    bvhcd_status st = ensure_node_capacity(T);
    if (st != BVHCD_OK) return st;
    if (!inter()) bvh_->set_updated(false);  // an inter front leaves the deformable BVH's restructure marks alone
    bool regen = false;
    if (cfg_.auto_grow == 2) {
        st = deferred_check(s, &regen);
        if (st != BVHCD_OK) return st;
    }
    bvhcd_front_op run_op = op;
    // front override after a BVH build or restructure (:75-110): the front
    // is regenerated in both cases
    if (bvh_->restr_enabled() && (bvh_->opt_tag() == 2 || bvh_->opt_tag() == 1)) run_op = BVHCD_FRONT_GENERATE;
    // an inter front's entries name both trees' nodes: after a restructure of
    // the traversed BVH -- the only change of either tree since the front was
    // last made -- it is restructured (re-sprouted inside the restructured
    // subtrees, BvttFrontLooseInter.cu:77-83); after any other change of
    // either tree (a build; the rigid one too, which the reference does not
    // check) it is regenerated
    const bool topo_changed =
        inter() && has_front_ && (seen_epoch_[0] != bvh_->topo_epoch() || seen_epoch_[1] != trav_->topo_epoch());
    const bool resprout = topo_changed && seen_epoch_[1] == trav_->topo_epoch() &&
                          seen_epoch_[0] + 1 == bvh_->topo_epoch() && bvh_->rs_epoch() == bvh_->topo_epoch();
    if (topo_changed && run_op != BVHCD_FRONT_PURE_BVH_CD)
        run_op = resprout ? BVHCD_FRONT_RESTRUCTURE : BVHCD_FRONT_GENERATE;
    if (op == BVHCD_FRONT_RESTRUCTURE && !resprout) run_op = BVHCD_FRONT_GENERATE;
    // a front operation needs a front: the first one is generated
    if (!has_front_ && (run_op == BVHCD_FRONT_UPDATE || run_op == BVHCD_FRONT_REORDER || run_op == BVHCD_FRONT_KEEP))
        run_op = BVHCD_FRONT_GENERATE;
    // a deformable BVH of one leaf has no internal node for the front
    // operations to climb to: its inter front is generated every frame
    if (inter() && T == 1 && run_op != BVHCD_FRONT_PURE_BVH_CD) run_op = BVHCD_FRONT_GENERATE;
    // a deferred check found an earlier overflow: the buffers have grown, the
    // front is made again
    if (regen && run_op != BVHCD_FRONT_PURE_BVH_CD) run_op = BVHCD_FRONT_GENERATE;
    unsigned *ctr = counters();
    const bool from_front = run_op == BVHCD_FRONT_UPDATE || run_op == BVHCD_FRONT_REORDER ||
                            run_op == BVHCD_FRONT_KEEP || run_op == BVHCD_FRONT_RESTRUCTURE;
    // the first attempt's keep and narrow-phase counters start at zero here
    const unsigned nxs = 1u << (2 * (1 - cur_)) | 1u << (2 * (1 - cur_) + 1);  // the other set's front sizes
    unsigned zero = (1u << C_HITS) | (1u << C_PAIRS_VALID) | (1u << C_FLAGGED);
    if (run_op == BVHCD_FRONT_KEEP) zero |= (1u << C_PAIRS) | (1u << C_WORK) | (1u << C_KSEL);
    if (run_op == BVHCD_FRONT_GENERATE) zero |= (1u << C_PAIRS) | nxs;
    if (run_op == BVHCD_FRONT_PURE_BVH_CD) zero |= 1u << C_PAIRS;
    if (run_op == BVHCD_FRONT_UPDATE) zero |= (1u << C_PAIRS) | (1u << C_WORK) | nxs;
    static_assert(C_NUM <= 32, "counter slots zeroed by lane");
    // kernels of this maintain may start before the one before them ends
    // (programmatic dependent launch), except inside a stream capture
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    FR_TRY(cudaStreamIsCapturing(s, &cs));
    struct PdlScope {
        bool &on;
        ~PdlScope() { on = false; }
    } pdl_scope{pdl_};
    pdl_ = cs == cudaStreamCaptureStatusNone;
    launch_k(pdl_, k_ovf_roll, 1u, 32u, 0, s, ctr, from_front ? kFrontLossBits : 0u, zero); note_launch();
    if (inter() ? (T < 1 || trav_->T() < 1) : T < 2) {
        FR_TRY(cudaMemsetAsync(ctr, 0, sizeof(unsigned) * 6, s));
        FR_TRY(cudaMemsetAsync(ctr + C_PAIRS_VALID, 0, sizeof(unsigned), s));
        last_op_ = run_op;
        if (run_op != BVHCD_FRONT_PURE_BVH_CD) has_front_ = true;
        return cfg_.auto_grow == 2 ? deferred_snapshot(s) : BVHCD_OK;
    }
    // With auto_grow the stage is replayed after growing the buffers.  The
    // stage's input (the tree and the front in set cur_) is intact when an
    // emission overflows because outputs go to the other set, except for the
    // reorder scatter, which is checked before it runs.
    for (int attempt = 0; attempt < 4; attempt++) {
        zeroed_ = attempt == 0;
        // a keep's sprout and narrow phase run as one launch (not in the
        // precision mode, whose narrow phase has its own kernel)
        keep_tail_ = run_op == BVHCD_FRONT_KEEP && !cfg_.precision;
        tail_ran_ = false;
        st = run(run_op, s);
        keep_tail_ = false;
        // without the test the narrow phase only counts the pairs
        if (st == BVHCD_OK && !tail_ran_) st = narrow(s, cfg_.narrow_phase != 0);
        zeroed_ = false;
        if (st != BVHCD_OK) return st;
        if (cfg_.auto_grow != 1) break;
        unsigned ovf = 0;
        st = grow_and_check(s, &ovf);
        if (st != BVHCD_OK) return st;
        if (!ovf) break;
        // an UPDATE or a balance overwrote the front, or the front this
        // maintain started from had lost entries: start again from a
        // generated front
        if (run_op == BVHCD_FRONT_UPDATE || run_op == BVHCD_FRONT_REORDER || run_op == BVHCD_FRONT_RESTRUCTURE ||
            (ovf & (1u | 2u | 16u | 64u)))
            run_op = BVHCD_FRONT_GENERATE;
    }
    last_op_ = run_op;
    FR_TRY(cudaGetLastError());
    return cfg_.auto_grow == 2 ? deferred_snapshot(s) : BVHCD_OK;
}

bvhcd_status Front::copy_state_from(const Front &src, cudaStream_t s) {
    if (&src == this) return BVHCD_OK;
    bvhcd_status st = ensure_node_capacity(src.capT_);
    if (st != BVHCD_OK) return st;
    const DBuf *from[] = {&src.front_[0][0], &src.front_[0][1], &src.front_[1][0], &src.front_[1][1], &src.pairs_,
                          &src.hits_, &src.work_, &src.intbeg_, &src.extbeg_,
                          &src.snapshot_, &src.counts64_, &src.fctr_};
    DBuf *to[] = {&front_[0][0], &front_[0][1], &front_[1][0], &front_[1][1], &pairs_, &hits_, &work_,
                  &intbeg_, &extbeg_, &snapshot_, &counts64_, &fctr_};
    for (size_t k = 0; k < sizeof(to) / sizeof(to[0]); k++) FR_TRY(to[k]->copy_from(*from[k], s));
    // the log sections, src.logn_ words each (this front's are at least as long)
    for (size_t k = 0; k < 4; k++)
        FR_TRY(cudaMemcpyAsync(logcnt_.as<unsigned>() + k * logn_, src.logcnt_.as<unsigned>() + k * src.logn_,
                               sizeof(unsigned) * src.logn_, cudaMemcpyDeviceToDevice, s));
    fcap_[0] = src.fcap_[0];
    fcap_[1] = src.fcap_[1];
    pcap_ = src.pcap_;
    cur_ = src.cur_;
    last_op_ = src.last_op_;
    has_front_ = src.has_front_;
    int_swapped_ = src.int_swapped_;
    log_counted_ = src.log_counted_;
    exp_valid_ = false;
    for (int k = 0; k < BVHCD_SHAPE_COUNT; k++) shape_[k] = src.shape_[k];
    shape_epoch_++;
    return cuda_status(cudaGetLastError());
}

void Front::get_shapes(bvhcd_launch_shapes *sh) const {
    for (int k = 0; k < BVHCD_SHAPE_COUNT; k++) {
        sh->unroll[k] = shape_[k].u;
        sh->block[k] = shape_[k].b;
    }
}

bvhcd_status Front::set_shapes(const bvhcd_launch_shapes &sh) {
    for (int k = 0; k < BVHCD_SHAPE_COUNT; k++) {
        const int u = sh.unroll[k], b = sh.block[k];
        if ((u != 1 && u != 2 && u != 4) || (b != 128 && b != 256 && b != 512)) return BVHCD_INVALID_ARG;
    }
    for (int k = 0; k < BVHCD_SHAPE_COUNT; k++) shape_[k] = Shape{sh.unroll[k], sh.block[k]};
    shape_epoch_++;
    return BVHCD_OK;
}

// Mean device time of `repeats` runs of fn on stream s, after one untimed run.
template <typename Fn>
static bvhcd_status time_runs(Fn fn, int repeats, cudaStream_t s, double *ms) {
    bvhcd_status st = fn();
    if (st != BVHCD_OK) return st;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) e = cudaEventRecord(a, s);
    for (int r = 0; r < repeats && e == cudaSuccess && st == BVHCD_OK; r++) st = fn();
    if (e == cudaSuccess) e = cudaEventRecord(b, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float f = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, a, b);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (st != BVHCD_OK) return st;
    if (e != cudaSuccess) return cuda_status(e);
    *ms = (double)f / repeats;
    return BVHCD_OK;
}

// Autotuner over the launch shapes (see bvhcd_front_autotune).  Each stage's
// kernels run on the real front and tree; none commits its output (keep and
// the narrow phase only rewrite pairs and hits, the update and balance
// kernels write the other buffer set), and a final GENERATE leaves the front
// consistent.
bvhcd_status Front::autotune(int repeats, bvhcd_launch_shapes *chosen, double *best_ms, cudaStream_t s) {
    if (repeats < 1 || repeats > 1000) return BVHCD_INVALID_ARG;
    if (!bvh_->built() || !has_front_) return BVHCD_NOT_READY;
    if (best_ms)
        for (int k = 0; k < BVHCD_SHAPE_COUNT; k++) best_ms[k] = 0.0;
    if (bvh_->T() >= 2) {
        Profiler *prof = bvh_->profiler();
        const bool prof_on = prof->on;
        prof->on = false;
        static const int kUs[3] = {1, 2, 4}, kBs[3] = {128, 256, 512};
        bvhcd_status st = BVHCD_OK;
        auto tune = [&](int stage, bool scan, auto fn) {
            Shape best = shape_[stage];
            double bt = 1e300;
            for (int ui = 0; ui < (scan ? 3 : 1) && st == BVHCD_OK; ui++)
                for (int bi = 0; bi < 3 && st == BVHCD_OK; bi++) {
                    shape_[stage] = Shape{scan ? kUs[ui] : shape_[stage].u, kBs[bi]};
                    double ms = 0.0;
                    st = time_runs(fn, repeats, s, &ms);
                    if (st == BVHCD_OK && ms < bt) {
                        bt = ms;
                        best = shape_[stage];
                    }
                }
            shape_[stage] = best;
            if (best_ms) best_ms[stage] = bt;
        };
        const bool test = cfg_.narrow_phase != 0;
        tune(BVHCD_SHAPE_KEEP, true, [&] { return keep(s); });
        tune(BVHCD_SHAPE_SPROUT, false, [&] { return keep(s); });
        tune(BVHCD_SHAPE_NARROW, false, [&] { return narrow(s, test); });
        tune(BVHCD_SHAPE_PRUNE_INT, true, [&] { return update_kernels(s); });
        tune(BVHCD_SHAPE_PRUNE_EXT, true, [&] { return update_kernels(s); });
        tune(BVHCD_SHAPE_BALANCE, true, [&] { return balance_kernels(s); });
        if (st == BVHCD_OK) st = generate(s, false);
        if (st == BVHCD_OK) st = narrow(s, test);
        prof->on = prof_on;
        if (st != BVHCD_OK) return st;
        last_op_ = BVHCD_FRONT_GENERATE;
        k_counts64<<<1, 32, 0, s>>>(counters(), (unsigned)pcap_, (unsigned)pcap_, counts64_.as<int64_t>());
        note_launch();
        FR_TRY(cudaGetLastError());
        FR_TRY(cudaStreamSynchronize(s));
    }
    shape_epoch_++;
    if (chosen) get_shapes(chosen);
    return BVHCD_OK;
}

// 1 when the last maintain of this front's BVH (or, for an inter front, of
// either BVH) was given a NaN or infinite coordinate; enqueued copies only
static cudaError_t nonfinite_read(const LBvh *a, const LBvh *b, unsigned *h2, cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(h2, a->nonfinite_flag(), sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h2 + 1, b->nonfinite_flag(), sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    return e;
}

bvhcd_status Front::stats(bvhcd_front_stats *st, cudaStream_t s) {
    unsigned h[C_NUM], nf[2] = {0u, 0u};
    FR_TRY(cudaMemcpyAsync(h, counters(), sizeof(h), cudaMemcpyDeviceToHost, s));
    FR_TRY(nonfinite_read(bvh_, trav(), nf, s));
    FR_TRY(cudaStreamSynchronize(s));
    *st = bvhcd_front_stats{};
    st->int_front = h[2 * cur_];
    st->ext_front = h[2 * cur_ + 1];
    st->broad_pairs = h[C_PAIRS_VALID];
    st->narrow_hits = h[C_HITS];
    st->overflow = (int32_t)h[C_OVERFLOW];
    st->overflow_any = (int32_t)(h[C_OVERFLOW] | h[C_OVF_STICKY]);
    st->nonfinite_input = (nf[0] | nf[1]) ? 1 : 0;
    st->bvh_opt_tag = bvh_->opt_tag();
    st->front_op_run = last_op_;
    st->restr_pending = bvh_->updated() ? 1 : 0;
    st->num_rt_subtrees = bvh_->last_rt_subtrees();
    st->num_rt_int_nodes = bvh_->last_rt_intnodes();
    st->flagged = (int32_t)h[C_FLAGGED];
    st->keep_tested = last_keep_sel_ ? (int32_t)h[C_KSEL] : (int32_t)(h[2 * cur_] + h[2 * cur_ + 1]);
    return BVHCD_OK;
}

bvhcd_status Front::compact_pairs(cudaStream_t s) {
    const size_t n = (size_t)(pcap_ > 0 ? pcap_ : 1);
    FR_TRY(outbuf_.reserve(sizeof(int2) * n));
    FR_TRY(cflag_.reserve(sizeof(unsigned) * 2 * n));
    FR_TRY(cscratch_.reserve(scan_scratch_bytes((int64_t)n)));
    unsigned *flags = cflag_.as<unsigned>(), *pos = flags + n;
    unsigned *ctr = counters();
    k_pair_flags<<<grid_for((int64_t)n), kThreads, 0, s>>>(pairs_.as<int2>(), ctr, (unsigned)pcap_, (unsigned)n, flags);
    note_launch();
    FR_TRY(scan_u32(flags, pos, (int64_t)n, false, ctr + C_COMPACT, cscratch_.p, s));
    k_pair_scatter<<<kFrontBlocks, kThreads, 0, s>>>(pairs_.as<int2>(), trav()->tree().sface, bvh_->tree().sface,
                                                     inter() ? 1 : 0, ctr, (unsigned)pcap_, flags, pos,
                                                     outbuf_.as<int2>());
    note_launch();
    return cuda_status(cudaGetLastError());
}

bvhcd_status Front::pairs(int which, int32_t *out, int64_t cap, int64_t *count, bool out_dev,
                          cudaStream_t s) {
    const int2 *src = hits_.as<int2>();
    if (!which) {
        // compact the broad pairs past their holes into original ids first
        bvhcd_status st = compact_pairs(s);
        if (st != BVHCD_OK) return st;
        src = outbuf_.as<int2>();
    }
    unsigned h[C_NUM], nf[2] = {0u, 0u};
    FR_TRY(cudaMemcpyAsync(h, counters(), sizeof(h), cudaMemcpyDeviceToHost, s));
    FR_TRY(nonfinite_read(bvh_, trav(), nf, s));
    FR_TRY(cudaStreamSynchronize(s));
    // NaN / infinite input: no tree, front or pair of this frame means anything
    if (nf[0] | nf[1]) {
        if (count) *count = 0;
        return BVHCD_INVALID_ARG;
    }
    int64_t n = which ? (int64_t)h[C_HITS] : (int64_t)h[C_COMPACT];
    if (n > pcap_) n = pcap_;
    if (count) *count = n;
    if (!out || cap <= 0) return n > cap ? BVHCD_CAPACITY_EXCEEDED : BVHCD_OK;
    int64_t m = n < cap ? n : cap;
    if (m > 0)
        FR_TRY(cudaMemcpyAsync(out, src, sizeof(int2) * (size_t)m,
                               out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    FR_TRY(cudaStreamSynchronize(s));
    // lost pairs or hits, or a front (this maintain's input or its traversals) that lost entries
    if (h[C_OVERFLOW] & (which ? (4u | 8u | 16u | 32u | 64u) : (4u | 16u | 32u | 64u))) return BVHCD_CAPACITY_EXCEEDED;
    return n > cap ? BVHCD_CAPACITY_EXCEEDED : BVHCD_OK;
}

namespace {
// Proximities of the compacted broad pairs (bvhcd_front_proximity): a first
// pass counts each pair's records (0 past the last pair, up to the capacity),
// a scan turns the counts into offsets, a second pass writes the records
// there, so they come ordered by pair and, inside a pair, by feature.
template <bool kWrite>
__global__ void k_proximity(const int2 *__restrict__ list, const unsigned *__restrict__ cnt, unsigned cap,
                            const int *__restrict__ fa, const float *__restrict__ va, const int *__restrict__ fb,
                            const float *__restrict__ vb, int same_mesh, double h, unsigned *counts,
                            const unsigned *__restrict__ offs, bvhcd_proximity *out, unsigned long long ocap) {
    const unsigned n = min(*cnt, cap);
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < cap; q += gridDim.x * blockDim.x) {
        if (q >= n) {
            if (!kWrite) counts[q] = 0u;
            continue;
        }
        if (kWrite && counts[q] == 0u) continue;  // most pairs have no proximity
        const int2 p = list[q];
        int ia[3], ib[3];
        prec::d3 pa[3], pb[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            ia[k] = __ldg(fa + 3 * (size_t)p.x + k);
            ib[k] = __ldg(fb + 3 * (size_t)p.y + k);
            const float3 x = load_vert(va, ia[k]), y = load_vert(vb, ib[k]);
            pa[k] = prec::mk(x.x, x.y, x.z);
            pb[k] = prec::mk(y.x, y.y, y.z);
        }
        if (!kWrite) {
            unsigned c = 0;
            prox::triangle_pair(ia, pa, ib, pb, same_mesh != 0, h, [&](const prox::Hit &) { ++c; });
            counts[q] = c;
        } else {
            unsigned long long o = offs[q];
            prox::triangle_pair(ia, pa, ib, pb, same_mesh != 0, h, [&](const prox::Hit &r) {
                if (o < ocap) {
                    bvhcd_proximity &x = out[o];
                    x.pair = (int)q;
                    x.kind = r.kind;
                    x.fa = r.fa;
                    x.fb = r.fb;
                    x.dist = r.d;
                    x.n[0] = r.n.x;
                    x.n[1] = r.n.y;
                    x.n[2] = r.n.z;
                    for (int k = 0; k < 4; k++) x.w[k] = r.w[k];
                }
                ++o;
            });
        }
    }
}
}  // namespace

bvhcd_status Front::proximity(const float *pos, double h, bvhcd_proximity *out, int64_t cap, int64_t *count,
                              bool out_dev, cudaStream_t s) {
    if (cap < 0 || !(h >= 0.0) || (inter() && pos)) return BVHCD_INVALID_ARG;
    if (!bvh_->built() || !trav()->built() || !has_front_) return BVHCD_NOT_READY;
    const float *va = pos ? pos : bvh_->verts();
    const float *vb = inter() ? trav_->verts() : va;
    if (!va || !vb) return BVHCD_INVALID_ARG;  // a box scene has no positions of its own
    if (count) *count = 0;
    if (pcap_ <= 0) return BVHCD_OK;
    bvhcd_status st = compact_pairs(s);
    if (st != BVHCD_OK) return st;
    const size_t n = (size_t)pcap_;
    FR_TRY(pxbuf_.reserve(sizeof(unsigned) * (2 * n + 1)));
    FR_TRY(cscratch_.reserve(scan_scratch_bytes((int64_t)n)));
    unsigned *counts = pxbuf_.as<unsigned>(), *offs = counts + n, *total = offs + n;
    const int2 *list = outbuf_.as<int2>();
    const unsigned *cnt = counters() + C_COMPACT;
    const unsigned g = RESIDENT((k_proximity<false>));
    k_proximity<false><<<g, kThreads, 0, s>>>(list, cnt, (unsigned)pcap_, bvh_->faces(), va, trav()->faces(), vb,
                                              inter() ? 0 : 1, h, counts, nullptr, nullptr, 0ull);
    note_launch();
    FR_TRY(cudaGetLastError());
    FR_TRY(scan_u32(counts, offs, (int64_t)n, false, total, cscratch_.p, s));
    unsigned htot = 0;
    FR_TRY(cudaMemcpyAsync(&htot, total, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    FR_TRY(cudaStreamSynchronize(s));
    if (count) *count = (int64_t)htot;
    const int64_t m = (int64_t)htot < cap ? (int64_t)htot : cap;
    if (out && m > 0) {
        bvhcd_proximity *dst = out;
        if (!out_dev) {
            FR_TRY(pxout_.reserve(sizeof(bvhcd_proximity) * (size_t)m));
            dst = pxout_.as<bvhcd_proximity>();
        }
        k_proximity<true><<<g, kThreads, 0, s>>>(list, cnt, (unsigned)pcap_, bvh_->faces(), va, trav()->faces(), vb,
                                                 inter() ? 0 : 1, h, counts, offs, dst, (unsigned long long)m);
        note_launch();
        FR_TRY(cudaGetLastError());
        if (!out_dev)
            FR_TRY(cudaMemcpyAsync(out, dst, sizeof(bvhcd_proximity) * (size_t)m, cudaMemcpyDeviceToHost, s));
        FR_TRY(cudaStreamSynchronize(s));
    }
    return (int64_t)htot > cap ? BVHCD_CAPACITY_EXCEEDED : BVHCD_OK;
}

// Contact points of the hits (which = 0) or distances of the broad pairs
// (which = 1), in the order bvhcd_front_pairs returns them.
bvhcd_status Front::contacts(int which, void *out, int64_t cap, int64_t *count, int64_t *flagged, bool out_dev,
                             bool f64, cudaStream_t s) {
    if (which < 0 || which > 1 || cap < 0 || inter() || bvh_->box_input()) return BVHCD_INVALID_ARG;
    const int2 *list = hits_.as<int2>();
    unsigned *ctr = counters();
    const unsigned *cnt = ctr + C_HITS;
    if (which == 1) {
        bvhcd_status st = compact_pairs(s);
        if (st != BVHCD_OK) return st;
        list = outbuf_.as<int2>();
        cnt = ctr + C_COMPACT;
    }
    const size_t item = f64 ? sizeof(double4) : sizeof(float4);
    const size_t nres = (size_t)(pcap_ > 0 ? pcap_ : 1);
    FR_TRY(cbuf_.reserve(item * nres + 16));
    void *res = cbuf_.p;
    unsigned *nflag = reinterpret_cast<unsigned *>(static_cast<char *>(cbuf_.p) + item * nres);
    FR_TRY(cudaMemsetAsync(nflag, 0, sizeof(unsigned), s));
    const int *faces = bvh_->faces();
    const float *verts = bvh_->verts();
    const unsigned g = RESIDENT((k_contacts<false, false, false>));
    const unsigned pc = (unsigned)pcap_;
    const bool pr = cfg_.precision != 0;
#define KC(D, P, F) k_contacts<D, P, F><<<g, kThreads, 0, s>>>(list, cnt, pc, faces, verts, res, nflag)
    if (f64) {
        if (which == 0) KC(false, false, true);
        else if (pr) KC(true, true, true);
        else KC(true, false, true);
    } else if (which == 0) {
        if (pr) KC(false, true, false);
        else KC(false, false, false);
    } else {
        if (pr) KC(true, true, false);
        else KC(true, false, false);
    }
#undef KC
    note_launch();
    FR_TRY(cudaGetLastError());
    unsigned h[C_NUM], hf = 0;
    FR_TRY(cudaMemcpyAsync(h, ctr, sizeof(h), cudaMemcpyDeviceToHost, s));
    FR_TRY(cudaMemcpyAsync(&hf, nflag, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    FR_TRY(cudaStreamSynchronize(s));
    int64_t n = which ? (int64_t)h[C_COMPACT] : (int64_t)h[C_HITS];
    if (n > pcap_) n = pcap_;
    if (count) *count = n;
    if (flagged) *flagged = hf;
    int64_t m = n < cap ? n : cap;
    if (out && m > 0) {
        FR_TRY(cudaMemcpyAsync(out, res, item * (size_t)m,
                               out_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
        FR_TRY(cudaStreamSynchronize(s));
    }
    return n > cap ? BVHCD_CAPACITY_EXCEEDED : BVHCD_OK;
}

bvhcd_status Front::export_front(int which, int32_t *out, int64_t cap, int64_t *count, cudaStream_t s) {
    if (which < 0 || which > 1) return BVHCD_INVALID_ARG;
    unsigned h[C_NUM];
    FR_TRY(cudaMemcpyAsync(h, counters(), sizeof(h), cudaMemcpyDeviceToHost, s));
    FR_TRY(cudaStreamSynchronize(s));
    int64_t n = h[2 * cur_ + which];
    if (n > fcap_[which]) n = fcap_[which];
    if (count) *count = n;
    int64_t m = n < cap ? n : cap;
    if (out && m > 0) {
        FR_TRY(cudaMemcpyAsync(out, front_[cur_][which].p, sizeof(int2) * (size_t)m, cudaMemcpyDeviceToHost, s));
        FR_TRY(cudaStreamSynchronize(s));
    }
    return n > cap ? BVHCD_CAPACITY_EXCEEDED : BVHCD_OK;
}

namespace {
// The pairs and their count into mapped host memory (bvhcd_front_pairs_async).
__global__ void k_pairs_to_host(const int2 *__restrict__ src, const unsigned *__restrict__ cnt, unsigned pcap,
                                int2 *out, int64_t cap, int64_t *count) {
    const unsigned n = min(*cnt, pcap);
    const int64_t m = (int64_t)n < cap ? (int64_t)n : cap;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x)
        out[q] = src[q];
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = (int64_t)n;
}
}  // namespace

bvhcd_status Front::pairs_async(int which, int32_t *host_out, int64_t cap, int64_t *host_count, cudaStream_t s) {
    if (which < 0 || which > 1 || cap < 0 || !host_count || (cap > 0 && !host_out)) return BVHCD_INVALID_ARG;
    void *dout = nullptr, *dcnt = nullptr;
    if (cudaHostGetDevicePointer(&dcnt, host_count, 0) != cudaSuccess) {
        cudaGetLastError();
        return BVHCD_INVALID_ARG;  // not mapped host memory
    }
    if (cap > 0 && cudaHostGetDevicePointer(&dout, host_out, 0) != cudaSuccess) {
        cudaGetLastError();
        return BVHCD_INVALID_ARG;
    }
    const int2 *src = hits_.as<int2>();
    const unsigned *cnt = counters() + C_HITS;
    if (!which) {
        bvhcd_status st = compact_pairs(s);
        if (st != BVHCD_OK) return st;
        src = outbuf_.as<int2>();
        cnt = counters() + C_COMPACT;
    }
    k_pairs_to_host<<<kFrontBlocks, kThreads, 0, s>>>(src, cnt, (unsigned)pcap_, static_cast<int2 *>(dout), cap,
                                                      static_cast<int64_t *>(dcnt));
    note_launch();
    return cuda_status(cudaGetLastError());
}

bvhcd_status Front::device_results(const int32_t **hits, const int64_t **counts) {
    if (hits) *hits = hits_.as<int32_t>();
    if (counts) *counts = counts64_.as<int64_t>();
    return BVHCD_OK;
}

}  // namespace bvhcd
