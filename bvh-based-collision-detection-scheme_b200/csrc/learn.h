// learn.h -- the learned scheduler's host class (see learn.cu).
#pragma once

#include <cuda_bf16.h>

#include "pipeline.h"

namespace bvhcd {

constexpr int kMlpParams = 16 * 64 + 64 + 64 * 64 + 64 + 64 * 3 + 3;  // 5443

class Learner {
  public:
    Learner(LBvh *bvh, Front *front, int smax) : bvh_(bvh), front_(front), smax_(smax) {}
    ~Learner();
    bvhcd_status init();
    bvhcd_status set_params(const float *host);
    bvhcd_status get_params(float *host) const;

    // bookkeeping after a maintain that rebuilt / restructured the tree, or
    // generated a front (frame() does both itself)
    bvhcd_status on_tree_changed(cudaStream_t s);
    bvhcd_status on_front_generated(cudaStream_t s);
    void tick(bool tree_changed, bool generated) {
        if (!tree_changed) since_build_++;
        if (!generated) since_gen_++;
    }

    bvhcd_status features(cudaStream_t s);
    bvhcd_status work(const Front &f, int64_t *host, cudaStream_t s);
    bvhcd_status predict(const float *X, int n, float *logits, int *vote, cudaStream_t s);
    bvhcd_status gradient(const float *X, const int *y, const float *cw, int n, float *grad_host, float *loss_host,
                          cudaStream_t s);
    bvhcd_status train(const float *X, const int *y, int n, const float *cw, int epochs, int batch, float lr,
                       unsigned seed, float *last_loss, cudaStream_t s);
    bvhcd_status decide(cudaStream_t s, int *n_restructure, double *regen_share);
    bvhcd_status decide_async(cudaStream_t s);
    void poll();
    void set_decide_every(int k) { decide_every_ = k > 0 ? k : 1; }
    void set_front_cycle(int c) { front_cycle_ = c > 0 ? c : 0; }
    long long decisions_applied() const { return decisions_applied_; }
    bvhcd_status frame(const bvhcd_scene &scene, int32_t frame_no, cudaStream_t s, int32_t *bvh_tag,
                       int32_t *front_op_run);

    int ncut() const { return ncut_; }
    const int *roots() const { return roots_.as<int>(); }
    const float *X() const { return X_.as<float>(); }
    int last_restructure() const { return last_restructure_; }
    double last_regen_share() const { return last_regen_share_; }

  private:
    LBvh *bvh_;
    Front *front_;
    int smax_;
    int ncut_ = 0, since_build_ = 0, since_gen_ = 0, adam_t_ = 0;
    bool regen_pending_ = false;
    double regen_threshold_ = 0.5, last_regen_share_ = 0.0;
    int last_restructure_ = 0;
    int decide_every_ = 3, tree_epoch_ = 0, pending_epoch_ = -1;
    int front_cycle_ = 0;  // 0: keep between decisions; c: the reference's front cycle of c frames
    bool pending_ = false;
    long long decisions_applied_ = 0;
    cudaEvent_t ev_ = nullptr;
    unsigned long long *h_act_ = nullptr;
    DBuf roots_, flag_, pos_, scratch_, av_b_, cen_b_, diag_, dpart_, gen_intbeg_, gen_extbeg_, X_, logits_, vote_,
        rt_roots_, act_, work_, p_, wq_, g_, m_, v_, loss_, bx_, by_, bidx_, cw_;
};

}  // namespace bvhcd
