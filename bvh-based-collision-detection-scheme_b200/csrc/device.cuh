// device.cuh -- data layout in HBM and the device helpers shared by the
// LBVH, front and narrow-phase kernels.
//
// Layout (T triangles, Morton-ordered "slots" s = 0..T-1, internal nodes in
// DFS pre-order d = 0..T-2):
//   lrec[2s], lrec[2s+1]  leaf record, one 32-byte sector:
//                         {min.xyz, parent}, {max.xyz, escape}
//                         parent = DFS id of the leaf's parent (for a left
//                         child this is the bottom of the left chain that
//                         starts at s); escape = lca[s+1], the next node in
//                         DFS order after the leaf.
//   nrec[2d], nrec[2d+1]  internal record, one 32-byte sector:
//                         {min.xyz, rangex | leftleaf << 31}, {max.xyz, escape}
//                         escape = lca[rangey+1]; leftleaf = the left child is
//                         the leaf rangex (else it is node d + 1).
//   sface[s]              int4 {v0, v1, v2, original triangle id}
//   lca[0..T]             tagged DFS entry per leaf (node<<1, or leaf<<1|1),
//                         lca[T] = -1, the reference's escape links
//                         (Mine/collision/lbvh/LBvhBuildKernels.cu:187-200)
//   topo[d]               int4 {lc, rc, par, mark}; mark bit0/bit1: left /
//                         right child is a leaf, bit2: node is a right child
//                         (LBvhBuildKernels.cu:147-148,168-169)
// A traversal step therefore needs one internal sector per node on the left
// spine and one leaf sector per chain; the integer fields ride in the .w lanes.
#pragma once

#include <cooperative_groups.h>
#include <cuda/atomic>
#include <cuda_runtime.h>
#include <stdint.h>

namespace bvhcd {
namespace cg = cooperative_groups;

constexpr int kSms = 148;

struct Tree {
    float4 *nrec;      // 2 (T-1)
    float4 *lrec;      // 2 T
    int4 *topo;        // T-1
    int2 *nrange;      // T-1 (rangex, rangey)
    int *lca;          // T+1
    int4 *sface;       // T
    int *primmap;      // T (orig -> slot)
    unsigned *code;    // T
    uint4 *nrec16;     // T-1 FP16 node records {6 outward-rounded halves, escape}, or null
    int T;
};

struct FrontLog {      // FlOrderLog (Mine/collision/auxiliary/FlOrderLog.h:19-50)
    unsigned *intcnt;  // T+1
    unsigned *extcnt;  // T+1
    unsigned *intbeg;  // T+1
    unsigned *extbeg;  // T+1
    unsigned *intback; // T+1
    unsigned *extback; // T+1
};

// The narrow phase's inputs and outputs (front.cu).
struct NarrowArgs {
    const int4 *psface;
    const float4 *pverts;  // positions as 16-byte records (x, y, z, 0)
    const int4 *sface;
    const float4 *verts;
    int leaf_first;
    unsigned *ctr;
    int2 *hits;
    unsigned cap_pairs, cap_hits;
    int64_t *counts64;
};

// Counters kept on the device so no stage needs a host round trip.
enum CounterSlot {
    C_INT0 = 0, C_EXT0 = 1,   // front sizes, buffer set 0
    C_INT1 = 2, C_EXT1 = 3,   // front sizes, buffer set 1
    C_PAIRS = 4, C_HITS = 5,
    C_OVERFLOW = 6,           // bit0 int front, bit1 ext front, bit2 pairs, bit3 hits,
                              // bit4 traversal bound hit, bit5 sprout work list
    C_RT_SUBTREES = 7, C_RT_INTNODES = 8,
    C_KSEL = 9,               // keep: front entries selected for a test (the rest wait on their expiries)
    C_WORK = 10,              // overlapping internal entries queued for traversal
    C_PAIRS_VALID = 11,       // broad-phase pairs (C_PAIRS counts reserved slots, holes included)
    C_COMPACT = 12,           // compaction cursor of the pair export
    C_FLAGGED = 13,           // precision mode: pairs re-decided in FP64
    C_TOPK = 14,              // refit plan: nodes whose leaf range crosses a refit block
    C_REFIT_DONE = 15,        // refit: leaf blocks finished (the last one runs the crossing nodes)
    C_DELTA = 16,             // refit: largest change of a leaf box coordinate (FP32 bits, rounded up)
    C_MOTION = 17,            // refit: sum of those changes since the last build (FP32 bits, rounded up)
    C_OVF_STICKY = 18,        // C_OVERFLOW bits of every maintain since the front was created
    C_NF_ACC = 19,            // BVH: non-finite input seen by the blocks of the running check
    C_NONFINITE = 20,         // BVH: 1 when the last maintain's input held a NaN or infinite coordinate
    C_NF_DONE = 21,           // BVH: blocks of the build-time finiteness check finished
    C_NARROW_DONE = 22,       // narrow phase: blocks finished (the last one writes the 64-bit counts)
    C_PAIRS_SCAN = 23,        // keep: the pairs the scan emitted (recorded by its last block)
    C_SCAN_DONE = 24,         // keep: scan blocks finished
    C_NUM = 25
};

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while the previous kernel of the stream runs; it
// waits here before it touches anything that kernel (or one before it)
// writes, and every such kernel waits before it ends, so completion stays in
// stream order.  Without the launch attribute the wait returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// lets the next kernel (launched with the attribute) start before this one ends
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ float4 ldg4(const float4 *p) { return __ldg(p); }
__device__ __forceinline__ float4 ldcg4(const float4 *p) { return __ldcg(p); }
// A 32-byte record {lo, hi} (32-byte aligned, read-only for the kernel's
// lifetime) in one 256-bit load: a gather of records then costs one request
// per warp instead of two.
__device__ __forceinline__ void ldg8(const float4 *p, float4 &lo, float4 &hi) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(lo.x), "=f"(lo.y), "=f"(lo.z), "=f"(lo.w), "=f"(hi.x), "=f"(hi.y), "=f"(hi.z), "=f"(hi.w)
        : "l"(p));
}
// the same record stored whole in one 256-bit store (a whole 32-byte sector:
// no partial-sector write for the memory to merge)
__device__ __forceinline__ void stg8(float4 *p, const float4 &lo, const float4 &hi) {
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(lo.x), "f"(lo.y),
                 "f"(lo.z), "f"(lo.w), "f"(hi.x), "f"(hi.y), "f"(hi.z), "f"(hi.w)
                 : "memory");
}

// AABB overlap, touching counts (BvhBvCompletePort::overlaps,
// Mine/collision/lbvh/BvhBV.h:54-65).  n = node box, b = query box.
__device__ __forceinline__ bool overlap(const float4 &nlo, const float4 &nhi, const float4 &blo,
                                        const float4 &bhi) {
    return !((blo.x > nhi.x) | (bhi.x < nlo.x) | (blo.y > nhi.y) | (bhi.y < nlo.y) |
             (blo.z > nhi.z) | (bhi.z < nlo.z));
}

// covertex (Mine/utility/CudaDeviceUtils.cu:153-157)
__device__ __forceinline__ bool covertex(const int4 &a, const int4 &b) {
    return (a.x == b.x) | (a.x == b.y) | (a.x == b.z) | (a.y == b.x) | (a.y == b.y) |
           (a.y == b.z) | (a.z == b.x) | (a.z == b.y) | (a.z == b.z);
}

// A vertex in two loads: its 12 bytes start on an 8-byte boundary (x, y as
// one 8-byte load, then z) or 4 bytes past one (x, then y, z as one 8-byte
// load); the choice is a select, not a branch, so a warp issues two load
// instructions whatever its lanes' parities.  Needs only the 4-byte
// alignment any float array has.
__device__ __forceinline__ float3 load_vert(const float *v, int i) {
    const float *p = v + 3 * (size_t)i;
    const bool even = (reinterpret_cast<uintptr_t>(p) & 7u) == 0;
    const float2 w = __ldg(reinterpret_cast<const float2 *>(even ? p : p + 1));
    const float s = __ldg(even ? p + 2 : p);
    return even ? make_float3(w.x, w.y, s) : make_float3(s, w.x, w.y);
}

// Triangle box: AABB::empty then three combines (Mine/base/Bv.h:27-34,80-84).
__device__ __forceinline__ void tri_box(const float3 &a, const float3 &b, const float3 &c,
                                        float4 &lo, float4 &hi) {
    lo.x = fminf(fminf(fminf(3.402823466e+38f, a.x), b.x), c.x);
    lo.y = fminf(fminf(fminf(3.402823466e+38f, a.y), b.y), c.y);
    lo.z = fminf(fminf(fminf(3.402823466e+38f, a.z), b.z), c.z);
    hi.x = fmaxf(fmaxf(fmaxf(-3.402823466e+38f, a.x), b.x), c.x);
    hi.y = fmaxf(fmaxf(fmaxf(-3.402823466e+38f, a.y), b.y), c.y);
    hi.z = fmaxf(fmaxf(fmaxf(-3.402823466e+38f, a.z), b.z), c.z);
}

// Where the primitives' boxes come from: triangles (vertex ids and vertex
// positions), or a scene given as one FP32 box per primitive (min xyz, max
// xyz; the reference's ARCSimSceneData, Mine/world/Scene.h:39-45), whose
// faces only give the vertex ids for adjacency culling.
struct PrimSrc {
    const int *faces;
    const float *verts;  // null for a box scene
    const float *boxes;  // null for triangles
};
// box of primitive t (its original id)
__device__ __forceinline__ void prim_box(const PrimSrc &p, int t, float4 &lo, float4 &hi) {
    if (p.boxes) {
        const float *b = p.boxes + 6 * (size_t)t;
        lo = make_float4(__ldg(b), __ldg(b + 1), __ldg(b + 2), 0.f);
        hi = make_float4(__ldg(b + 3), __ldg(b + 4), __ldg(b + 5), 0.f);
    } else {
        tri_box(load_vert(p.verts, __ldg(p.faces + 3 * (size_t)t)), load_vert(p.verts, __ldg(p.faces + 3 * (size_t)t + 1)),
                load_vert(p.verts, __ldg(p.faces + 3 * (size_t)t + 2)), lo, hi);
    }
}
// the same from a slot's stored face (x, y, z vertex ids, w original id)
__device__ __forceinline__ void face_box(const PrimSrc &p, const int4 &f, float4 &lo, float4 &hi) {
    if (p.boxes) prim_box(p, f.w, lo, hi);
    else tri_box(load_vert(p.verts, f.x), load_vert(p.verts, f.y), load_vert(p.verts, f.z), lo, hi);
}
// |x| <= FLT_MAX: false for NaN and for +-inf
__device__ __forceinline__ bool finite1(float x) { return fabsf(x) <= 3.402823466e+38f; }
__device__ __forceinline__ bool finite3(const float3 &v) { return finite1(v.x) & finite1(v.y) & finite1(v.z); }
// face_box that also says whether every input coordinate was finite (the
// box's min / max would drop a NaN, so the inputs themselves are tested)
__device__ __forceinline__ bool face_box_fin(const PrimSrc &p, const int4 &f, float4 &lo, float4 &hi) {
    if (p.boxes) {
        prim_box(p, f.w, lo, hi);
        return finite1(lo.x) & finite1(lo.y) & finite1(lo.z) & finite1(hi.x) & finite1(hi.y) & finite1(hi.z);
    }
    const float3 a = load_vert(p.verts, f.x), b = load_vert(p.verts, f.y), c = load_vert(p.verts, f.z);
    tri_box(a, b, c, lo, hi);
    return finite3(a) & finite3(b) & finite3(c);
}

// 30-bit Morton code of a box centre normalised by the scene box
// (calcMCs, LBvhBuildKernels.cu:76-91; morton3D/expandBits,
// Mine/utility/CudaDeviceUtils.cu:82-130).  IEEE operations only, no
// contraction, so the code is bit-identical to the reference's.
__device__ __forceinline__ unsigned expand10(unsigned v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ unsigned quant1024(float x) {
    x = fminf(fmaxf(__fmul_rn(x, 1024.0f), 0.0f), 1023.0f);
    return (unsigned)x;
}
__device__ __forceinline__ unsigned morton_box(const float4 &lo, const float4 &hi,
                                               const float *scene) {
    float cx = __fmul_rn(__fadd_rn(lo.x, hi.x), 0.5f);
    float cy = __fmul_rn(__fadd_rn(lo.y, hi.y), 0.5f);
    float cz = __fmul_rn(__fadd_rn(lo.z, hi.z), 0.5f);
    float ox = __fsub_rn(cx, scene[0]), oy = __fsub_rn(cy, scene[1]), oz = __fsub_rn(cz, scene[2]);
    float w = __fsub_rn(scene[3], scene[0]);
    float h = __fsub_rn(scene[4], scene[1]);
    float d = __fsub_rn(scene[5], scene[2]);
    unsigned xx = expand10(quant1024(__fdiv_rn(ox, w)));
    unsigned yy = expand10(quant1024(__fdiv_rn(oy, h)));
    unsigned zz = expand10(quant1024(__fdiv_rn(oz, d)));
    return xx * 4u + yy * 2u + zz;
}

// Warp-aggregated reservation: the converged threads that call it take
// consecutive slots with one atomic.  Returns the slot; writes only when the
// slot is below capacity, otherwise raises the overflow bit (the counter keeps
// counting so the required size is known).
template <typename T>
__device__ __forceinline__ void emit(T *buf, unsigned *ctr, unsigned cap, const T &v,
                                     unsigned *ovf, unsigned bit) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, (unsigned)g.size());
    base = g.shfl(base, 0) + g.thread_rank();
    if (base < cap) buf[base] = v;
    else atomicOr(ovf, bit);
}

}  // namespace bvhcd
