// capi.cu -- extern "C" entry points declared in include/bvhcd.h.
#include <new>

#include <vector>

#include "learn.h"
#include "pipeline.h"
#include "prims.cuh"

struct bvhcd_bvh {
    bvhcd::LBvh impl;
    explicit bvhcd_bvh(const bvhcd_bvh_config &c) : impl(c) {}
};
// A frame (BVH op + front op) captured as a CUDA graph, keyed by the ops and
// by the host state the frame starts from; `after` is the host state its
// capture ended with, restored after every replay.
struct FrameGraph {
    int bvh_op, front_op;
    bvhcd::LBvh::HostState bvh_before, bvh_after;
    bvhcd::Front::HostState front_before, front_after;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
};

struct bvhcd_front {
    bvhcd::Front impl;
    // graph-launched frames (bvhcd_frame_graph)
    std::vector<FrameGraph> graphs;
    const float *g_pos = nullptr;
    const int32_t *g_faces = nullptr;
    int g_T = -1, g_V = -1, g_scenes = -1, g_shapes = -1;  // layout / launch-shape epochs
    bool g_warm = false;
    bvhcd_front(bvhcd::LBvh *b, const bvhcd_front_config &c, bvhcd::LBvh *trav = nullptr) : impl(b, c, trav) {}
    ~bvhcd_front() { drop_graphs(); }
    void drop_graphs() {
        for (FrameGraph &g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        graphs.clear();
        g_warm = false;
    }
};

struct bvhcd_learner {
    bvhcd::Learner impl;
    bvhcd_learner(bvhcd::LBvh *b, bvhcd::Front *f, int smax) : impl(b, f, smax) {}
};

namespace {
inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

bool same_state(const bvhcd::LBvh::HostState &a, const bvhcd::LBvh::HostState &b) {
    return a.T == b.T && a.V == b.V && a.opt_tag == b.opt_tag && a.built == b.built && a.updated == b.updated &&
           a.box_input == b.box_input && a.vptr == b.vptr && a.bptr == b.bptr && a.fptr == b.fptr;
}
bool same_state(const bvhcd::Front::HostState &a, const bvhcd::Front::HostState &b) {
    return a.cur == b.cur && a.last_op == b.last_op && a.has_front == b.has_front && a.int_swapped == b.int_swapped &&
           a.log_counted == b.log_counted && a.exp_valid == b.exp_valid;
}
}  // namespace

extern "C" {
#pragma GCC visibility push(default)

const char *bvhcd_status_string(bvhcd_status s) {
    switch (s) {
    case BVHCD_OK: return "ok";
    case BVHCD_INVALID_ARG: return "invalid argument";
    case BVHCD_OUT_OF_MEMORY: return "out of device memory";
    case BVHCD_CAPACITY_EXCEEDED: return "capacity exceeded";
    case BVHCD_CUDA_ERROR: return "CUDA error";
    case BVHCD_TIMEOUT: return "timeout";
    case BVHCD_NOT_READY: return "not ready";
    }
    return "unknown status";
}

bvhcd_status bvhcd_device_check(int32_t device, int32_t *ok) {
    if (!ok) return BVHCD_INVALID_ARG;
    *ok = 0;
    cudaDeviceProp p;
    cudaError_t e = cudaGetDeviceProperties(&p, device);
    if (e != cudaSuccess) return bvhcd::cuda_status(e);
    *ok = (p.major == 10 && p.minor == 0) ? 1 : 0;
    return BVHCD_OK;
}

bvhcd_status bvhcd_bvh_create(const bvhcd_bvh_config *cfg, bvhcd_bvh **out) {
    if (!cfg || !out) return BVHCD_INVALID_ARG;
    *out = nullptr;
    bvhcd_bvh *h = new (std::nothrow) bvhcd_bvh(*cfg);
    if (!h) return BVHCD_OUT_OF_MEMORY;
    bvhcd_status st = h->impl.init();
    if (st != BVHCD_OK) {
        delete h;
        return st;
    }
    *out = h;
    return BVHCD_OK;
}

bvhcd_status bvhcd_bvh_destroy(bvhcd_bvh *bvh) {
    if (!bvh) return BVHCD_INVALID_ARG;
    delete bvh;
    return BVHCD_OK;
}

bvhcd_status bvhcd_bvh_maintain(bvhcd_bvh *bvh, bvhcd_bvh_op op, const bvhcd_scene *scene, void *stream) {
    if (!bvh || !scene) return BVHCD_INVALID_ARG;
    return bvh->impl.maintain(op, *scene, as_stream(stream));
}

bvhcd_status bvhcd_bvh_maintain_boxes(bvhcd_bvh *bvh, bvhcd_bvh_op op, const bvhcd_box_scene *scene, void *stream) {
    if (!bvh || !scene) return BVHCD_INVALID_ARG;
    return bvh->impl.maintain_boxes(op, *scene, as_stream(stream));
}

bvhcd_status bvhcd_bvh_sizes(const bvhcd_bvh *bvh, int32_t *prims, int32_t *ext_nodes, int32_t *int_nodes) {
    if (!bvh) return BVHCD_INVALID_ARG;
    int T = bvh->impl.T();
    int S = bvh->impl.num_scenes();
    if (prims) *prims = T;
    if (ext_nodes) *ext_nodes = T;
    if (int_nodes) *int_nodes = T >= S ? T - S : 0;
    return BVHCD_OK;
}

bvhcd_status bvhcd_bvh_set_scenes(bvhcd_bvh *bvh, int32_t num_scenes, const int32_t *tri_offsets) {
    if (!bvh) return BVHCD_INVALID_ARG;
    return bvh->impl.set_scenes(num_scenes, tri_offsets);
}

bvhcd_status bvhcd_bvh_opt_tag(const bvhcd_bvh *bvh, int32_t *tag) {
    if (!bvh || !tag) return BVHCD_INVALID_ARG;
    *tag = bvh->impl.opt_tag();
    return BVHCD_OK;
}

bvhcd_status bvhcd_bvh_request_restructure(bvhcd_bvh *bvh, const int32_t *roots, int32_t n, void *stream) {
    if (!bvh) return BVHCD_INVALID_ARG;
    return bvh->impl.request_restructure(roots, n, as_stream(stream));
}

bvhcd_status bvhcd_bvh_export(const bvhcd_bvh *bvh, int32_t *inode, float *ibox, int32_t *leaf, float *lbox,
                              int32_t *lca, uint32_t *codes, int32_t *primmap, void *stream) {
    if (!bvh) return BVHCD_INVALID_ARG;
    return bvh->impl.export_tree(inode, ibox, leaf, lbox, lca, codes, primmap, as_stream(stream));
}

bvhcd_status bvhcd_front_create(bvhcd_bvh *bvh, const bvhcd_front_config *cfg, bvhcd_front **out) {
    if (!bvh || !cfg || !out) return BVHCD_INVALID_ARG;
    *out = nullptr;
    bvhcd_front *h = new (std::nothrow) bvhcd_front(&bvh->impl, *cfg);
    if (!h) return BVHCD_OUT_OF_MEMORY;
    bvhcd_status st = h->impl.init();
    if (st != BVHCD_OK) {
        delete h;
        return st;
    }
    *out = h;
    return BVHCD_OK;
}

bvhcd_status bvhcd_front_create_inter(bvhcd_bvh *deformable, bvhcd_bvh *rigid, const bvhcd_front_config *cfg,
                                      bvhcd_front **out) {
    if (!deformable || !rigid || !cfg || !out || deformable == rigid) return BVHCD_INVALID_ARG;
    if (cfg->precision || deformable->impl.num_scenes() != 1 || rigid->impl.num_scenes() != 1) return BVHCD_INVALID_ARG;
    *out = nullptr;
    bvhcd_front *h = new (std::nothrow) bvhcd_front(&deformable->impl, *cfg, &rigid->impl);
    if (!h) return BVHCD_OUT_OF_MEMORY;
    bvhcd_status st = h->impl.init();
    if (st != BVHCD_OK) {
        delete h;
        return st;
    }
    *out = h;
    return BVHCD_OK;
}

bvhcd_status bvhcd_front_destroy(bvhcd_front *front) {
    if (!front) return BVHCD_INVALID_ARG;
    delete front;
    return BVHCD_OK;
}

bvhcd_status bvhcd_front_maintain(bvhcd_front *front, bvhcd_front_op op, void *stream) {
    if (!front) return BVHCD_INVALID_ARG;
    return front->impl.maintain(op, as_stream(stream));
}

bvhcd_status bvhcd_front_stats_get(bvhcd_front *front, bvhcd_front_stats *stats, void *stream) {
    if (!front || !stats) return BVHCD_INVALID_ARG;
    return front->impl.stats(stats, as_stream(stream));
}

bvhcd_status bvhcd_front_pairs(bvhcd_front *front, int32_t which, int32_t *out, int64_t cap, int64_t *count,
                               int32_t out_on_device, void *stream) {
    if (!front || which < 0 || which > 1 || cap < 0) return BVHCD_INVALID_ARG;
    return front->impl.pairs(which, out, cap, count, out_on_device != 0, as_stream(stream));
}

bvhcd_status bvhcd_front_device_results(bvhcd_front *front, const int32_t **hit_pairs, const int64_t **counts) {
    if (!front) return BVHCD_INVALID_ARG;
    return front->impl.device_results(hit_pairs, counts);
}

bvhcd_status bvhcd_front_export(bvhcd_front *front, int32_t which, int32_t *out, int64_t cap, int64_t *count,
                                void *stream) {
    if (!front || cap < 0) return BVHCD_INVALID_ARG;
    return front->impl.export_front(which, out, cap, count, as_stream(stream));
}

bvhcd_status bvhcd_profile_enable(bvhcd_bvh *bvh, int32_t on) {
    if (!bvh) return BVHCD_INVALID_ARG;
    bvh->impl.profiler()->on = on != 0;
    return BVHCD_OK;
}

bvhcd_status bvhcd_profile_read(bvhcd_bvh *bvh, double *ms, int64_t *calls, int32_t reset) {
    if (!bvh) return BVHCD_INVALID_ARG;
    return bvh->impl.profiler()->read(ms, calls, reset != 0);
}

bvhcd_status bvhcd_morton_order_noalloc(const float *pos, const int32_t *faces, int32_t num_faces, uint32_t *codes,
                                        int32_t *order, void *stream) {
    return bvhcd::morton_order_noalloc(pos, faces, num_faces, codes, order, as_stream(stream));
}

// BenchmarkLogic::maintainScheme, STATIC_MANDATORY with divergent marks
// (Mine/system/Logic/BenchmarkLogic.hpp:102-117): BVH cycle 12
// (Mine/setting/BvhSettings.h:45), front cycle 6 (Mine/setting/BvttFrontSettings.h:49).
bvhcd_status bvhcd_schedule_heuristic(int32_t frame, int32_t start_frame, int32_t *bvh_op, int32_t *front_op) {
    if (!bvh_op || !front_op || frame < start_frame) return BVHCD_INVALID_ARG;
    const int f = frame - start_frame;
    int b = (f % 12) ? BVHCD_BVH_REFIT : BVHCD_BVH_BUILD;
    int k = f % 6, fr;
    if (k == 0) fr = (frame == start_frame) ? BVHCD_FRONT_GENERATE : BVHCD_FRONT_UPDATE;
    else if (k == 5) fr = BVHCD_FRONT_REORDER;
    else fr = BVHCD_FRONT_KEEP;
    if (b == BVHCD_BVH_BUILD) fr = BVHCD_FRONT_GENERATE;
    if ((f + 1) % 12 == 0) fr = BVHCD_FRONT_KEEP;
    *bvh_op = b;
    *front_op = fr;
    return BVHCD_OK;
}

bvhcd_status bvhcd_bvh_stage_positions(bvhcd_bvh *bvh, const float *host_pos, int32_t num_vertices,
                                       void *copy_stream, const float **staged) {
    if (!bvh) return BVHCD_INVALID_ARG;
    return bvh->impl.stage_positions(host_pos, num_vertices, as_stream(copy_stream), staged);
}

bvhcd_status bvhcd_frame(bvhcd_bvh *bvh, bvhcd_front *front, int32_t frame, int32_t start_frame,
                         const bvhcd_scene *scene, void *stream) {
    int32_t b, f;
    bvhcd_status st = bvhcd_schedule_heuristic(frame, start_frame, &b, &f);
    if (st != BVHCD_OK) return st;
    st = bvhcd_bvh_maintain(bvh, (bvhcd_bvh_op)b, scene, stream);
    if (st != BVHCD_OK) return st;
    return bvhcd_front_maintain(front, (bvhcd_front_op)f, stream);
}

bvhcd_status bvhcd_front_contacts(bvhcd_front *front, int32_t which, float *out, int64_t cap, int64_t *count,
                                  int64_t *flagged, int32_t out_on_device, void *stream) {
    if (!front) return BVHCD_INVALID_ARG;
    return front->impl.contacts(which, out, cap, count, flagged, out_on_device != 0, false, as_stream(stream));
}

bvhcd_status bvhcd_front_contacts64(bvhcd_front *front, int32_t which, double *out, int64_t cap, int64_t *count,
                                    int32_t out_on_device, void *stream) {
    if (!front) return BVHCD_INVALID_ARG;
    return front->impl.contacts(which, out, cap, count, nullptr, out_on_device != 0, true, as_stream(stream));
}

bvhcd_status bvhcd_front_pairs_async(bvhcd_front *front, int32_t which, int32_t *host_out, int64_t cap,
                                     int64_t *host_count, void *stream) {
    if (!front) return BVHCD_INVALID_ARG;
    return front->impl.pairs_async(which, host_out, cap, host_count, as_stream(stream));
}

bvhcd_status bvhcd_host_alloc(int64_t bytes, void **ptr) {
    if (!ptr || bytes < 0) return BVHCD_INVALID_ARG;
    *ptr = nullptr;
    cudaError_t e = cudaHostAlloc(ptr, (size_t)(bytes > 0 ? bytes : 1), cudaHostAllocMapped | cudaHostAllocPortable);
    return bvhcd::cuda_status(e);
}

bvhcd_status bvhcd_host_free(void *ptr) {
    if (!ptr) return BVHCD_OK;
    return bvhcd::cuda_status(cudaFreeHost(ptr));
}

bvhcd_status bvhcd_front_proximity(bvhcd_front *front, const float *pos, double thickness, bvhcd_proximity *out,
                                   int64_t cap, int64_t *count, int32_t out_on_device, void *stream) {
    if (!front) return BVHCD_INVALID_ARG;
    return front->impl.proximity(pos, thickness, out, cap, count, out_on_device != 0, as_stream(stream));
}

bvhcd_status bvhcd_bvh_copy_state(bvhcd_bvh *dst, const bvhcd_bvh *src, void *stream) {
    if (!dst || !src) return BVHCD_INVALID_ARG;
    return dst->impl.copy_state_from(src->impl, as_stream(stream));
}

bvhcd_status bvhcd_front_copy_state(bvhcd_front *dst, const bvhcd_front *src, void *stream) {
    if (!dst || !src) return BVHCD_INVALID_ARG;
    if (dst->impl.inter() || src->impl.inter()) return BVHCD_INVALID_ARG;
    dst->drop_graphs();
    return dst->impl.copy_state_from(src->impl, as_stream(stream));
}

bvhcd_status bvhcd_learner_create(bvhcd_bvh *bvh, bvhcd_front *front, int32_t max_subtree_leaves,
                                  bvhcd_learner **out) {
    if (!bvh || !front || !out || &bvh->impl != front->impl.bvh() || front->impl.inter()) return BVHCD_INVALID_ARG;
    bvhcd_learner *l = new (std::nothrow) bvhcd_learner(&bvh->impl, &front->impl, max_subtree_leaves);
    if (!l) return BVHCD_OUT_OF_MEMORY;
    bvhcd_status st = l->impl.init();
    if (st != BVHCD_OK) {
        delete l;
        return st;
    }
    *out = l;
    return BVHCD_OK;
}

bvhcd_status bvhcd_learner_destroy(bvhcd_learner *l) {
    delete l;
    return BVHCD_OK;
}

bvhcd_status bvhcd_learner_set_params(bvhcd_learner *l, const float *params) {
    if (!l || !params) return BVHCD_INVALID_ARG;
    return l->impl.set_params(params);
}

bvhcd_status bvhcd_learner_get_params(const bvhcd_learner *l, float *params) {
    if (!l || !params) return BVHCD_INVALID_ARG;
    return l->impl.get_params(params);
}

bvhcd_status bvhcd_learner_frame(bvhcd_learner *l, const bvhcd_scene *scene, int32_t frame, int32_t *bvh_tag,
                                 int32_t *front_op, void *stream) {
    if (!l || !scene) return BVHCD_INVALID_ARG;
    return l->impl.frame(*scene, frame, as_stream(stream), bvh_tag, front_op);
}

bvhcd_status bvhcd_learner_set_front_cycle(bvhcd_learner *l, int32_t frames) {
    if (!l || frames < 0) return BVHCD_INVALID_ARG;
    l->impl.set_front_cycle(frames);
    return BVHCD_OK;
}

bvhcd_status bvhcd_learner_set_decide_every(bvhcd_learner *l, int32_t frames) {
    if (!l || frames < 1) return BVHCD_INVALID_ARG;
    l->impl.set_decide_every(frames);
    return BVHCD_OK;
}

bvhcd_status bvhcd_learner_observe(bvhcd_learner *l, int32_t tree_changed, int32_t front_generated, void *stream) {
    if (!l) return BVHCD_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    l->impl.tick(tree_changed != 0, front_generated != 0);
    bvhcd_status st = BVHCD_OK;
    if (tree_changed) st = l->impl.on_tree_changed(s);
    if (st == BVHCD_OK && front_generated) st = l->impl.on_front_generated(s);
    return st;
}

bvhcd_status bvhcd_learner_cut(const bvhcd_learner *l, int32_t *roots, int32_t cap, int32_t *n, void *stream) {
    if (!l || !n || cap < 0) return BVHCD_INVALID_ARG;
    *n = l->impl.ncut();
    if (!roots) return BVHCD_OK;
    if (cap < *n) return BVHCD_CAPACITY_EXCEEDED;
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaMemcpyAsync(roots, l->impl.roots(), sizeof(int32_t) * (size_t)*n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return bvhcd::cuda_status(e);
}

bvhcd_status bvhcd_learner_features(bvhcd_learner *l, float *X, int32_t cap_rows, int32_t *n, void *stream) {
    if (!l || !n || cap_rows < 0) return BVHCD_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    bvhcd_status st = l->impl.features(s);
    if (st != BVHCD_OK) return st;
    *n = l->impl.ncut();
    if (!X) return BVHCD_OK;
    if (cap_rows < *n) return BVHCD_CAPACITY_EXCEEDED;
    cudaError_t e = cudaMemcpyAsync(X, l->impl.X(), sizeof(float) * 16 * (size_t)*n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return bvhcd::cuda_status(e);
}

bvhcd_status bvhcd_learner_work(bvhcd_learner *l, const bvhcd_front *front, int64_t *out, int32_t cap, void *stream) {
    if (!l || !front || !out || cap < l->impl.ncut()) return BVHCD_INVALID_ARG;
    return l->impl.work(front->impl, out, as_stream(stream));
}

bvhcd_status bvhcd_mlp_gradient(bvhcd_learner *l, const float *X, const int32_t *y, int32_t n,
                                const float *class_weight, float *grad, float *loss, void *stream) {
    if (!l || !X || !y || !class_weight || n <= 0) return BVHCD_INVALID_ARG;
    return l->impl.gradient(X, y, class_weight, n, grad, loss, as_stream(stream));
}

bvhcd_status bvhcd_mlp_train(bvhcd_learner *l, const float *X, const int32_t *y, int32_t n, const float *class_weight,
                             int32_t epochs, int32_t batch, float lr, uint32_t seed, float *last_loss, void *stream) {
    if (!l || !X || !y || !class_weight) return BVHCD_INVALID_ARG;
    return l->impl.train(X, y, n, class_weight, epochs, batch, lr, seed, last_loss, as_stream(stream));
}

bvhcd_status bvhcd_mlp_predict(bvhcd_learner *l, const float *X, int32_t n, float *logits, int32_t *vote,
                               void *stream) {
    if (!l || !X || n < 0) return BVHCD_INVALID_ARG;
    return l->impl.predict(X, n, logits, vote, as_stream(stream));
}

bvhcd_status bvhcd_front_get_shapes(const bvhcd_front *front, bvhcd_launch_shapes *shapes) {
    if (!front || !shapes) return BVHCD_INVALID_ARG;
    front->impl.get_shapes(shapes);
    return BVHCD_OK;
}

bvhcd_status bvhcd_front_set_shapes(bvhcd_front *front, const bvhcd_launch_shapes *shapes) {
    if (!front || !shapes) return BVHCD_INVALID_ARG;
    return front->impl.set_shapes(*shapes);
}

bvhcd_status bvhcd_front_autotune(bvhcd_front *front, int32_t repeats, bvhcd_launch_shapes *chosen,
                                  double *best_ms, void *stream) {
    if (!front) return BVHCD_INVALID_ARG;
    return front->impl.autotune(repeats, chosen, best_ms, as_stream(stream));
}

bvhcd_status bvhcd_frame_graph(bvhcd_bvh *bvh, bvhcd_front *front, const bvhcd_scene *scene, int32_t bvh_op,
                               int32_t front_op, void *stream) {
    if (!bvh || !front || !scene || !stream) return BVHCD_INVALID_ARG;
    if (&bvh->impl != front->impl.bvh()) return BVHCD_INVALID_ARG;
    if (!scene->on_device || bvh->impl.restr_enabled() || front->impl.auto_grow() || front->impl.inter())
        return BVHCD_INVALID_ARG;
    if (bvh->impl.is_staged(scene->pos)) return BVHCD_INVALID_ARG;  // staging buffers alternate
    if (bvh_op < BVHCD_BVH_BUILD || bvh_op > BVHCD_BVH_UPDATE) return BVHCD_INVALID_ARG;
    if (front_op < BVHCD_FRONT_PURE_BVH_CD || front_op > BVHCD_FRONT_RESTRUCTURE) return BVHCD_INVALID_ARG;
    cudaStream_t s = as_stream(stream);
    if (scene->pos != front->g_pos || scene->faces != front->g_faces || scene->num_faces != front->g_T ||
        scene->num_vertices != front->g_V || bvh->impl.layout_epoch() != front->g_scenes ||
        front->impl.shape_epoch() != front->g_shapes) {
        front->drop_graphs();
        front->g_pos = scene->pos;
        front->g_faces = scene->faces;
        front->g_T = scene->num_faces;
        front->g_V = scene->num_vertices;
        front->g_scenes = bvh->impl.layout_epoch();
        front->g_shapes = front->impl.shape_epoch();
    }
    bvhcd_status st;
    if (!front->g_warm) {
        // the first frame runs as ordinary launches: it sizes every buffer,
        // so no capture ever allocates
        st = bvh->impl.maintain((bvhcd_bvh_op)bvh_op, *scene, s);
        if (st == BVHCD_OK) st = front->impl.maintain((bvhcd_front_op)front_op, s);
        if (st == BVHCD_OK) front->g_warm = true;
        return st;
    }
    const bvhcd::LBvh::HostState hb = bvh->impl.host_state();
    const bvhcd::Front::HostState hf = front->impl.host_state();
    for (FrameGraph &g : front->graphs) {
        if (g.bvh_op != bvh_op || g.front_op != front_op || !same_state(g.bvh_before, hb) ||
            !same_state(g.front_before, hf))
            continue;
        cudaError_t e = cudaGraphLaunch(g.exec, s);
        if (e != cudaSuccess) return bvhcd::cuda_status(e);
        bvh->impl.set_host_state(g.bvh_after);
        front->impl.set_host_state(g.front_after);
        for (long long k = 0; k < g.launches; k++) bvhcd::note_launch();
        return BVHCD_OK;
    }
    // capture this frame, then launch it (capturing runs only the host side)
    bvhcd::Profiler *prof = bvh->impl.profiler();
    const bool prof_on = prof->on;
    prof->on = false;
    const long long n0 = bvhcd::launch_count();
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        prof->on = prof_on;
        return bvhcd::cuda_status(e);
    }
    st = bvh->impl.maintain((bvhcd_bvh_op)bvh_op, *scene, s);
    if (st == BVHCD_OK) st = front->impl.maintain((bvhcd_front_op)front_op, s);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(s, &graph);
    prof->on = prof_on;
    if (st != BVHCD_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        bvh->impl.set_host_state(hb);
        front->impl.set_host_state(hf);
        return st != BVHCD_OK ? st : bvhcd::cuda_status(e);
    }
    FrameGraph g;
    g.bvh_op = bvh_op;
    g.front_op = front_op;
    g.bvh_before = hb;
    g.front_before = hf;
    g.bvh_after = bvh->impl.host_state();
    g.front_after = front->impl.host_state();
    g.launches = bvhcd::launch_count() - n0;
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e == cudaSuccess) e = cudaGraphLaunch(g.exec, s);
    if (e != cudaSuccess) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        bvh->impl.set_host_state(hb);
        front->impl.set_host_state(hf);
        return bvhcd::cuda_status(e);
    }
    front->graphs.push_back(g);
    return BVHCD_OK;
}

}  // extern "C"

#include <atomic>
namespace bvhcd {
static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace bvhcd

namespace bvhcd {
// allocations left before the chosen one fails (0: no fault planned)
static std::atomic<long long> g_alloc_countdown{0};
bool alloc_fault_due() {
    long long c = g_alloc_countdown.load(std::memory_order_relaxed);
    while (c > 0) {
        if (g_alloc_countdown.compare_exchange_weak(c, c - 1, std::memory_order_relaxed)) return c == 1;
    }
    return false;
}
}  // namespace bvhcd

extern "C" __attribute__((visibility("default"))) bvhcd_status bvhcd_debug_fail_alloc(int64_t n) {
    if (n < 0) return BVHCD_INVALID_ARG;
    bvhcd::g_alloc_countdown.store((long long)n, std::memory_order_relaxed);
    return BVHCD_OK;
}

extern "C" __attribute__((visibility("default"))) bvhcd_status bvhcd_launch_count(int64_t *n) {
    if (!n) return BVHCD_INVALID_ARG;
    *n = bvhcd::launch_count();
    return BVHCD_OK;
}
