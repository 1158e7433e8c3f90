// pipeline.h -- host classes behind the C ABI.  LBvh mirrors
// LBvhFixedDeformable (Mine/collision/lbvh/LBvhFixedDeformable.h:27-108) and
// Front mirrors BvttFrontLooseIntra (Mine/collision/bvtt_front/BvttFrontLooseIntra.h:27-80):
// same maintenance options, same per-frame state machine, but every size
// stays on the device and every call only enqueues work on a stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <vector>

#include "../../include/bvhcd.h"
#include "device.cuh"

namespace bvhcd {

// Host-side fault injection for the tests (bvhcd_debug_fail_alloc): true when
// the device allocation about to be made is the one chosen to fail.
bool alloc_fault_due();

// Device buffer owned by a handle.
struct DBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t n) {
        if (n <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = alloc_fault_due() ? cudaErrorMemoryAllocation : cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T>
    T *as() const { return reinterpret_cast<T *>(p); }
    // this buffer becomes a device copy of `src` (grown to its size)
    cudaError_t copy_from(const DBuf &src, cudaStream_t s) {
        if (!src.p) return cudaSuccess;
        cudaError_t e = reserve(src.bytes);
        if (e != cudaSuccess) return e;
        return cudaMemcpyAsync(p, src.p, src.bytes, cudaMemcpyDeviceToDevice, s);
    }
};

bvhcd_status cuda_status(cudaError_t e);
bvhcd_status morton_order_noalloc(const float *verts, const int *faces, int T, unsigned *codes, int *order,
                                  cudaStream_t s);

// Stage timer: CUDA event pairs recorded on the work stream, resolved when
// read (the reference's Logger::recordSection, Mine/utility/CudaTimer.hpp:43-53).
class Profiler {
  public:
    ~Profiler();
    bool on = false;
    void begin(int stage, cudaStream_t s);
    void end(int stage, cudaStream_t s);
    bvhcd_status read(double *ms, int64_t *calls, bool reset);

  private:
    struct Pending { int stage; cudaEvent_t a, b; };
    cudaEvent_t get();
    std::vector<cudaEvent_t> pool_;
    std::vector<Pending> pending_;
    cudaEvent_t open_[BVHCD_STAGE_COUNT] = {};
    double ms_[BVHCD_STAGE_COUNT] = {};
    int64_t calls_[BVHCD_STAGE_COUNT] = {};
};

// RAII stage scope
struct StageScope {
    Profiler *p;
    int stage;
    cudaStream_t s;
    StageScope(Profiler *p_, int st, cudaStream_t s_) : p(p_), stage(st), s(s_) {
        if (p->on) p->begin(stage, s);
    }
    ~StageScope() {
        if (p->on) p->end(stage, s);
    }
};

class LBvh {
  public:
    explicit LBvh(const bvhcd_bvh_config &cfg) : cfg_(cfg) {}
    ~LBvh();
    bvhcd_status init();
    bvhcd_status maintain(bvhcd_bvh_op op, const bvhcd_scene &scene, cudaStream_t s);
    bvhcd_status maintain_tree(bvhcd_bvh_op op, const bvhcd_scene &scene, cudaStream_t s);
    // the same for a scene of primitive boxes (no positions)
    bvhcd_status maintain_boxes(bvhcd_bvh_op op, const bvhcd_box_scene &scene, cudaStream_t s);
    bool box_input() const { return box_input_; }
    bvhcd_status stage_positions(const float *host, int nv, cudaStream_t copy, const float **staged);
    bool is_staged(const float *p) const { return p && (p == stage_[0].as<float>() || p == stage_[1].as<float>()); }
    bvhcd_status export_tree(int32_t *inode, float *ibox, int32_t *leaf, float *lbox, int32_t *lca,
                             uint32_t *codes, int32_t *primmap, cudaStream_t s) const;
    bvhcd_status request_restructure(const int32_t *roots, int32_t n, cudaStream_t s);
    // the same with the roots already on the device; enqueued only
    bvhcd_status request_restructure_device(const int32_t *roots, int32_t n, cudaStream_t s);
    bvhcd_status set_scenes(int S, const int32_t *tri_offsets);
    // Device and host state of `src` (same configuration) copied into this
    // handle: a fork point for counterfactual runs.
    bvhcd_status copy_state_from(const LBvh &src, cudaStream_t s);
    int num_scenes() const { return S_; }
    int layout_epoch() const { return epoch_; }  // bumped by every set_scenes

    // Host-side state a maintain() call advances; a captured frame graph
    // restores the state its capture ended with after every replay.
    struct HostState {
        int T, V, opt_tag, rt_subtrees, rt_intnodes;
        bool built, updated, box_input;
        const float *vptr, *bptr;
        const int *fptr;
    };
    HostState host_state() const {
        return HostState{T_, V_, opt_tag_, rt_subtrees_, rt_intnodes_, built_, updated_, box_input_, vptr_, bptr_,
                         fptr_};
    }
    void set_host_state(const HostState &h) {
        T_ = h.T; V_ = h.V; opt_tag_ = h.opt_tag; rt_subtrees_ = h.rt_subtrees; rt_intnodes_ = h.rt_intnodes;
        built_ = h.built; updated_ = h.updated; box_input_ = h.box_input; vptr_ = h.vptr; bptr_ = h.bptr;
        fptr_ = h.fptr;
    }

    Tree tree() const;
    int T() const { return T_; }
    int V() const { return V_; }
    bool built() const { return built_; }
    int opt_tag() const { return opt_tag_; }
    // advances whenever the topology (and so the leaf order) changes: build,
    // restructure, state copy
    int topo_epoch() const { return topo_epoch_; }
    // The last restructure: the topology epoch it produced, and per internal
    // node a non-zero mark inside a restructured subtree, per leaf slot the
    // subtree's root (0 outside), per root the old end of its left spine.
    // Valid while rs_epoch() == topo_epoch().
    int rs_epoch() const { return rs_epoch_; }
    const int *rs_intmark() const { return intmark_.as<int>(); }
    const int *rs_leafroot() const { return leafroot_.as<int>(); }
    const int *rs_oldlast() const { return rs_oldlast_.as<int>(); }
    // advances whenever the faces (vertex ids) may have changed
    int faces_epoch() const { return faces_epoch_; }
    const float *verts() const { return vptr_; }
    // The positions as 16-byte records (x, y, z, 0), one load per vertex for
    // the narrow phase's gathers; written by every maintain that reads new
    // triangle positions (inside the refit, or by the finiteness check ahead
    // of a build or restructure).
    const float4 *verts4() const { return verts4_.as<float4>(); }
    const int *faces() const { return fptr_; }
    bool restr_enabled() const { return cfg_.enable_restr != 0; }

    // BvhRestrLog (Mine/collision/auxiliary/BvhRestrLog.h:57-80): written by
    // the front's quality check, consumed by the next maintain.
    int *intrange() const { return intrange_.as<int>(); }
    int *rtroot() const { return rtroot_.as<int>(); }
    void set_updated(bool u) { updated_ = u; }
    bool updated() const { return updated_; }
    unsigned *counters() const { return ctr_.as<unsigned>(); }
    // this BVH's device word saying the last maintain's input held a NaN or
    // infinite coordinate
    const unsigned *nonfinite_flag() const { return ctr_.as<unsigned>() + C_NONFINITE; }
    int last_rt_subtrees() const { return rt_subtrees_; }
    int last_rt_intnodes() const { return rt_intnodes_; }
    Profiler *profiler() { return &prof_; }

  private:
    bvhcd_status ensure_capacity(int T, int V);
    bvhcd_status upload(const bvhcd_scene &scene, cudaStream_t s);
    bvhcd_status upload_boxes(const bvhcd_box_scene &scene, cudaStream_t s);
    bvhcd_status maintain_ops(bvhcd_bvh_op op, int prevT, bool was_built, cudaStream_t s);
    PrimSrc src() const { return PrimSrc{fptr_, vptr_, bptr_}; }
    bvhcd_status build(cudaStream_t s);
    bvhcd_status refit(cudaStream_t s);
    bvhcd_status refit_plan(cudaStream_t s, bool heights_known);
    bvhcd_status restructure(cudaStream_t s);
    bvhcd_status scene_box(cudaStream_t s);
    bvhcd_status climb_and_order(cudaStream_t s);
    bvhcd_status node_fp16(cudaStream_t s);
    bvhcd_status check_finite(cudaStream_t s);

    bvhcd_bvh_config cfg_;
    int T_ = 0, V_ = 0, capT_ = 0, capV_ = 0;
    bool built_ = false, updated_ = false;
    int opt_tag_ = 0, rt_subtrees_ = 0, rt_intnodes_ = 0;
    const float *vptr_ = nullptr;
    const int *fptr_ = nullptr;
    const float *bptr_ = nullptr;  // FP32 primitive boxes of a box scene
    bool box_input_ = false;
    // owned copies of host input (boxes_: a box scene's FP32 boxes, boxes64_:
    // its FP64 boxes before rounding)
    DBuf verts_, faces_, boxes_, boxes64_;
    DBuf verts4_;  // 16-byte position records (verts4())
    // tree
    DBuf nrec_, lrec_, topo_, nrange_, lca_, sface_, primmap_, code_, refit_flag_, nrec16_;
    // refit plan (a function of the topology): split of each internal node,
    // crossing flags and ranks, per-split local entries, crossing-node
    // entries, node heights, level-sorted lists (per leaf block and for the
    // crossing nodes) with their level offsets, record links (leaves, crossing
    // nodes), export marks and lists with the export slots, and the top
    // pass's global storage when the crossing nodes exceed shared memory
    DBuf split_, cross_, topk_, plan_, top_, gbox_, height_, llist_, lhdr_, tlist_, thdr_, llink_, tlink_, lexp_,
        nexp_, lexport_, gext_, uheight_;
    // build scratch
    DBuf keys_, vals_, keys2_, vals2_, k64_, k64b_, metric_, ulc_, urc_, upar_, urx_, ury_, umark_,
        ubox_, uflag_, posb_, clen_, coff_, dfs_, ulpar_, scene_, partial_, scratch_, task_, tmpface_;
    // restructure log
    DBuf intrange_, rtroot_, intmark_, extrange_, extmark_, leafroot_, flagbuf_;
    // old end of each restructured subtree's left spine (see k_rs_oldlast), and
    // the topology epoch the restructure arrays describe (-1: none)
    DBuf rs_oldlast_;
    int rs_epoch_ = -1;
    // batched scenes: S_ scenes, triangle offsets, per-triangle scene id,
    // per-slot scene id, per-scene boxes, box-reduction tiles
    int S_ = 1, ntiles_ = 0, epoch_ = 0, topo_epoch_ = 0, faces_epoch_ = 0;
    std::vector<int> h_off_;
    DBuf scene_of_, leafscene_, sbox_, tiles_;
    DBuf ctr_;
    unsigned *h_ctr_ = nullptr;  // pinned
    // double-buffered position uploads: copy done / buffer free events
    DBuf stage_[2];
    cudaEvent_t stage_ready_[2] = {nullptr, nullptr}, stage_free_[2] = {nullptr, nullptr};
    int stage_next_ = 0;
    bool stage_pending_ = false;
    Profiler prof_;
};

class Front {
  public:
    // trav: null for an intra front (the BVH's own triangles traverse it), or
    // the BVH whose triangles traverse `bvh` (an inter front)
    Front(LBvh *bvh, const bvhcd_front_config &cfg, LBvh *trav = nullptr) : bvh_(bvh), trav_(trav), cfg_(cfg) {}
    ~Front();
    bvhcd_status init();
    bvhcd_status maintain(bvhcd_front_op op, cudaStream_t s);
    bvhcd_status stats(bvhcd_front_stats *st, cudaStream_t s);
    bvhcd_status pairs(int which, int32_t *out, int64_t cap, int64_t *count, bool out_dev,
                       cudaStream_t s);
    bvhcd_status export_front(int which, int32_t *out, int64_t cap, int64_t *count, cudaStream_t s);
    bvhcd_status proximity(const float *pos, double thickness, bvhcd_proximity *out, int64_t cap, int64_t *count,
                           bool out_dev, cudaStream_t s);
    bvhcd_status contacts(int which, void *out, int64_t cap, int64_t *count, int64_t *flagged, bool out_dev,
                          bool f64, cudaStream_t s);
    bvhcd_status device_results(const int32_t **hits, const int64_t **counts);
    bvhcd_status pairs_async(int which, int32_t *host_out, int64_t cap, int64_t *host_count, cudaStream_t s);

    // Host-side state a maintain() call advances (see LBvh::HostState);
    // int_swapped: balance() exchanged the internal-front buffers of the two
    // sets an odd number of times; log_counted: the log's per-node counts
    // describe the current front (a balance leaves only its begins valid).
    struct HostState {
        int cur, last_op, exp_epoch, exp_faces;
        bool has_front, int_swapped, log_counted, exp_valid;
    };
    HostState host_state() const {
        return HostState{cur_, last_op_, exp_epoch_, exp_faces_, has_front_, int_swapped_, log_counted_, exp_valid_};
    }
    void set_host_state(const HostState &h) {
        cur_ = h.cur;
        last_op_ = h.last_op;
        exp_epoch_ = h.exp_epoch;
        exp_faces_ = h.exp_faces;
        has_front_ = h.has_front;
        log_counted_ = h.log_counted;
        exp_valid_ = h.exp_valid;
        if (h.int_swapped != int_swapped_) {
            std::swap(front_[0][0], front_[1][0]);
            int_swapped_ = h.int_swapped;
        }
    }
    bool auto_grow() const { return cfg_.auto_grow != 0; }
    LBvh *bvh() const { return bvh_; }
    bool inter() const { return trav_ != nullptr; }
    const LBvh *trav() const { return trav_ ? trav_ : bvh_; }
    unsigned *counters() const { return fctr_.as<unsigned>(); }
    bvhcd_status copy_state_from(const Front &src, cudaStream_t s);
    const FrontLog front_log() const { return log(); }
    // the front-quality check of an UPDATE (checkFrontQuality) marks
    // subtrees for restructuring; a scheduler that marks them itself turns it off
    void set_quality_check(bool on) { quality_check_ = on; }
    bool has_front() const { return has_front_; }
    void get_shapes(bvhcd_launch_shapes *sh) const;
    bvhcd_status set_shapes(const bvhcd_launch_shapes &sh);
    bvhcd_status autotune(int repeats, bvhcd_launch_shapes *chosen, double *best_ms, cudaStream_t s);
    int shape_epoch() const { return shape_epoch_; }

  private:
    bvhcd_status ensure_node_capacity(int T);
    bvhcd_status run(bvhcd_front_op op, cudaStream_t s);
    bvhcd_status generate(cudaStream_t s, bool pure);
    bvhcd_status prune_sprout(cudaStream_t s);
    bvhcd_status restructure_inter(cudaStream_t s);
    bvhcd_status update_kernels(cudaStream_t s);
    bvhcd_status keep(cudaStream_t s);
    bvhcd_status balance(cudaStream_t s);
    bvhcd_status balance_kernels(cudaStream_t s);
    bvhcd_status reorder(cudaStream_t s);
    bvhcd_status narrow(cudaStream_t s, bool test);
    bvhcd_status check_quality(cudaStream_t s);
    bvhcd_status snapshot(cudaStream_t s);
    bvhcd_status grow_and_check(cudaStream_t s, unsigned *ovf_bits);
    bvhcd_status grow_from(const unsigned *h, cudaStream_t s);
    bvhcd_status deferred_check(cudaStream_t s, bool *regen);
    bvhcd_status deferred_snapshot(cudaStream_t s);
    bvhcd_status compact_pairs(cudaStream_t s);
    FrontLog log() const;

    LBvh *bvh_;
    LBvh *trav_ = nullptr;
    int seen_epoch_[2] = {-1, -1};  // topology epochs of bvh_ and trav() at the last generation
    DBuf fctr_;                     // this front's device counters (CounterSlot)
    bvhcd_front_config cfg_;
    int capT_ = 0;
    int cur_ = 0;  // which buffer set holds the current front
    int last_op_ = -1;
    // launch shape per front stage (BVHCD_SHAPE_*): entries per thread step
    // in the scans, threads per block
    struct Shape {
        int u, b;
    };
    // default launch shapes (unroll, block) per stage: keep, internal prune,
    // external prune, balance, sprout, narrow phase; bvhcd_front_set_shapes or
    // the autotuner replace them
    Shape shape_[BVHCD_SHAPE_COUNT] = {{2, 256}, {2, 256}, {1, 512}, {2, 256}, {1, 512}, {1, 256}};
    int shape_epoch_ = 0;
    bool has_front_ = false;
    bool int_swapped_ = false;
    bool log_counted_ = true;
    // keep-time expiries of the front entries (one float per entry of the
    // current set's internal / external front), valid until the fronts move,
    // the tree's topology changes or new faces arrive; ksel_: the entries a
    // keep selects for a test
    DBuf iexp_, xexp_, ksel_;
    bool exp_valid_ = false, last_keep_sel_ = false;
    // the running stage and narrow phase find their counters zeroed already
    // (the maintain's first attempt zeroes them in its prologue)
    bool zeroed_ = false;
    // the front scans, sprouts and narrow phase of the running maintain are
    // launched with programmatic stream serialisation
    bool pdl_ = false;
    // a KEEP of the running maintain ends in k_keep_tail (its sprout and the
    // narrow phase in one launch); the maintain then runs no narrow phase
    bool keep_tail_ = false, tail_ran_ = false;
    NarrowArgs narrow_args();
    int exp_epoch_ = -1, exp_faces_ = -1;
    bool quality_check_ = true;
    DBuf front_[2][2];  // [set][0 int, 1 ext] int2 entries
    int64_t fcap_[2] = {0, 0};
    DBuf pairs_, hits_, outbuf_, work_, cbuf_, cflag_, cscratch_;
    int64_t pcap_ = 0;
    // the per-node counts of the front log in one buffer (one clearing memset):
    // intcnt, extcnt, intback, extback, logn_ words apart
    DBuf logcnt_, intbeg_, extbeg_, snapshot_, scratch_, counts64_;
    size_t logn_ = 0;
    cudaError_t log_clear(cudaStream_t s) const;
    DBuf rcur_;  // reorder cursors, one per group of 2^kReorderShift nodes and front
    DBuf pxbuf_, pxout_;  // proximity counts / offsets / total; records for a host destination
    // deferred capacity check (auto_grow = 2): counter copies of the last
    // kSnap maintains in pinned host memory, one event each; the maintain
    // number of each copy (-1: looked at); maintains counted; the maintain
    // that last regenerated after an overflow
    static constexpr int kSnap = 3;
    unsigned *h_snap_ = nullptr;
    cudaEvent_t snap_ev_[kSnap] = {nullptr, nullptr, nullptr};
    long long snap_seq_[kSnap] = {-1, -1, -1};
    long long seq_ = 0, regen_seq_ = 0;
};

}  // namespace bvhcd
