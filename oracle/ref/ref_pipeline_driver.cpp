// ref_pipeline_driver.cpp -- runs the reference's own pipeline
// (LBvhFixedDeformable + BvttFrontLooseIntra, compiled unmodified from the
// reference tree as host C++ with every kernel run one thread at a time by
// oracle/ref/Makefile.refemu) on frames read from a file,
// with the reference's STATIC_MANDATORY / divergent-marks schedule
// (Mine/system/Logic/BenchmarkLogic.hpp:102-117), and writes per frame the
// broad-phase pair list (applyCpResults) and the tree arrays.  It replaces
// only the app shell and the assimp scene loader
// (Mine/Frameworks/CudaProject/CudaProjectApp.cpp:26-59, Mine/world/Scene.cpp).
//
// TEST INFRASTRUCTURE ONLY: it produces the golden fixtures under
// tests/golden/ (tests/golden/make_golden.py) and is never part of the product.
//
// Input file:  int32 magic 'BVHI', T, V, F; int32 faces[T*3]; float frames[F*V*3]
// Marks file (optional): per frame int32 n, int32 roots[n] -- subtrees marked
//   for restructuring just before that frame's BVH maintenance.
// Output file: per frame: int32 magic 'FRAM', frame, bvh op, front op,
//   opt tag, npairs, T; int32 pairs[npairs*2] (orig ids as emitted);
//   int32 leaf_lca[T+1], leaf_par[T], prim_idx[T], prim_map[T];
//   uint32 codes[T]; int32 int_par[T-1], int_lbd[T-1], int_rbd[T-1];
//   uint32 int_mark[T-1].
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "collision/bvtt_front/BVTTFront.h"
#include "collision/lbvh/LBvh.h"
#include "setting/BvhSettings.h"
#include "setting/BvttFrontSettings.h"
#include "system/CudaDevice/CudaDevice.h"
#include "system/Log/Logger.hpp"
#include "world/Scene.h"

using namespace mn;

// The reference's constructor leaves its restructure scratch vectors empty
// (Mine/collision/lbvh/LBvhFixedDeformable.cu:44-51 are commented out, "only
// used in the restructuring scheme") while restructuring is switched on
// (Mine/setting/CDBenchmarkSettings.h:54), so its first restructure writes
// through null pointers (calibrateRestrRoots,
// Mine/collision/lbvh/LBvhRestructureKernels.cu:32).  The driver sizes them
// as those commented lines state.  They are private members; an explicit
// instantiation names them, which the language exempts from access checks.
template <typename Tag, typename Tag::type M>
struct Expose {
    friend typename Tag::type member(Tag) { return M; }
};
#define EXPOSE(NAME, ELEM)                                                     \
    struct Tag_##NAME {                                                        \
        using type = thrust::device_vector<ELEM> LBvhFixedDeformable::*;       \
        friend type member(Tag_##NAME);                                        \
    };                                                                         \
    template struct Expose<Tag_##NAME, &LBvhFixedDeformable::NAME>;
EXPOSE(d_prevLbds, int)
EXPOSE(d_prevRbds, int)
EXPOSE(d_gatherMap, int)
EXPOSE(d_taskSequence, int)
EXPOSE(d_sequence, int)
EXPOSE(d_rtSubtrees, int)
EXPOSE(d_sizePerSubtree, uint)
EXPOSE(d_begPerSubtree, int)

static void size_restructure_scratch(LBvhFixedDeformable &b) {
    const int P = BvhSettings::prim_size(), I = BvhSettings::int_node_size();
    (b.*member(Tag_d_prevLbds{})).resize(I);
    (b.*member(Tag_d_prevRbds{})).resize(I);
    (b.*member(Tag_d_gatherMap{})).resize(P);
    (b.*member(Tag_d_taskSequence{})).resize(P);
    (b.*member(Tag_d_sequence{})).resize(P);
    (b.*member(Tag_d_rtSubtrees{})).resize((size_t)I << 1);
    (b.*member(Tag_d_sizePerSubtree{})).resize((size_t)I << 1);
    (b.*member(Tag_d_begPerSubtree{})).resize((size_t)I << 1);
}

static void schedule(int f, int *b, int *fr) {
    int bb = (f % 12) ? 1 : 0;  // REFIT : BUILD
    int k = f % 6, ff;
    if (k == 0) ff = (f == 0) ? 1 : 2;  // GENERATE : UPDATE
    else if (k == 5) ff = 3;            // REORDER
    else ff = 4;                        // KEEP
    if (bb == 0) ff = 1;
    if ((f + 1) % 12 == 0) ff = 4;
    *b = bb;
    *fr = ff;
}

template <typename T>
static std::vector<T> dev_copy(const T *d, size_t n) {
    std::vector<T> h(n);
    if (n) cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost);
    return h;
}

template <typename T>
static void put(FILE *o, const std::vector<T> &v) {
    if (!v.empty()) fwrite(v.data(), sizeof(T), v.size(), o);
}

// Marks the subtrees rooted at `roots` (DFS internal-node ids of the current
// tree) for restructuring through the reference's public BvhRestrLog
// interface, with the same three updates its quality check makes per
// flagged node (checkFrontQuality, Mine/collision/bvtt_front/
// BvttFrontGenerateKernels.cu:44-46) and the same clear-then-tag protocol
// (BvttFrontLooseIntra::checkQuality, Mine/collision/bvtt_front/
// BvttFrontLooseIntra.cu:219-228), so that the next maintain() takes the
// restructure branch (LBvhFixedDeformable::maintain, Mine/collision/lbvh/
// LBvhFixedDeformable.cu:69-80).
static void mark_restructure(LBvhFixedDeformable &b, const std::vector<int> &roots) {
    const int t = (int)b.getPrimNodeSize();
    if (t < 2 || roots.empty()) return;
    BvhRestrLog &log = b.restrLog();
    if (!log.getUpdateTag()) log.clear(t);
    std::vector<int> ir = dev_copy(log.getIntRange(), (size_t)t);
    std::vector<int> rr = dev_copy(log.getRestrBvhRoot(), (size_t)t);
    std::vector<int> lb = dev_copy(b.ctks().getLbds(), (size_t)t - 1);
    std::vector<int> rb = dev_copy(b.ctks().getRbds(), (size_t)t - 1);
    for (int i : roots) {
        if (i < 0 || i >= t - 1) continue;
        ir[i] += 1;
        ir[i + rb[i] - lb[i]] -= 1;
        if (i < rr[lb[i]]) rr[lb[i]] = i;
    }
    cudaMemcpy(log.getIntRange(), ir.data(), sizeof(int) * ir.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(log.getRestrBvhRoot(), rr.data(), sizeof(int) * rr.size(), cudaMemcpyHostToDevice);
    log.setUpdateTag(true);
}

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s frames.bin out.bin [marks.bin]\n", argv[0]);
        return 2;
    }
    FILE *in = fopen(argv[1], "rb");
    if (!in) return 2;
    int hdr[4];
    if (fread(hdr, sizeof(int), 4, in) != 4 || hdr[0] != 0x49485642) return 2;
    const int T = hdr[1], V = hdr[2], F = hdr[3];
    if (T < 2 || T > BvhSettings::prim_size()) {
        fprintf(stderr, "triangle count %d outside the reference's capacity\n", T);
        return 2;
    }
    std::vector<int3> faces(T);
    std::vector<float3> frames((size_t)F * V);
    if (fread(faces.data(), sizeof(int3), T, in) != (size_t)T) return 2;
    if (fread(frames.data(), sizeof(float3), frames.size(), in) != frames.size()) return 2;
    fclose(in);
    // optional marks file: per frame int32 n, then n int32 subtree roots
    std::vector<std::vector<int>> marks(F);
    if (argc > 3) {
        FILE *mk = fopen(argv[3], "rb");
        if (!mk) return 2;
        for (int f = 0; f < F; f++) {
            int n = 0;
            if (fread(&n, sizeof(int), 1, mk) != 1 || n < 0) return 2;
            marks[f].resize(n);
            if (n && fread(marks[f].data(), sizeof(int), n, mk) != (size_t)n) return 2;
        }
        fclose(mk);
    }

    CudaDevice::startup();
    Logger::startup();
    {
        LBvhKernelRegister lbvh_kernels;
        BvttFrontKernelRegister front_kernels;
        auto bvh = std::make_unique<LBvh<ModelType::FixedDeformableType>>(LBvhBuildConfig{});
        size_restructure_scratch(*bvh);
        auto fl = std::make_unique<BvttFront<BvttFrontType::LooseIntraType>>(
            BvttFrontIntraBuildConfig<LBvh<ModelType::FixedDeformableType>>(
                bvh.get(), BvttFrontType::LooseIntraType, BvttFrontSettings::ext_front_size(),
                BvttFrontSettings::int_front_size(), BvhSettings::ext_node_size(), BvhSettings::int_node_size()));
        uint *d_cnt = nullptr;
        uint2 *d_pairs = nullptr;
        cudaMalloc(&d_cnt, sizeof(uint));
        cudaMalloc(&d_pairs, sizeof(uint2) * BvttFrontSettings::collision_pair_num());
        FILE *out = fopen(argv[2], "wb");
        if (!out) return 2;
        SceneData sd;
        sd.fids = faces;
        for (int f = 0; f < F; f++) {
            sd.pos.assign(frames.begin() + (size_t)f * V, frames.begin() + (size_t)(f + 1) * V);
            int b, fr;
            schedule(f, &b, &fr);
            mark_restructure(*bvh, marks[f]);
            bvh->maintain((LBvhFixedDeformableMaintenance)b, sd);
            fl->maintain((BvttFrontLooseIntraMaintenance)fr);
            fl->applyCpResults(d_cnt, d_pairs);
            cudaDeviceSynchronize();
            uint n = 0;
            cudaMemcpy(&n, d_cnt, sizeof(uint), cudaMemcpyDeviceToHost);
            std::vector<int> pairs = dev_copy(reinterpret_cast<int *>(d_pairs), (size_t)n * 2);
            const int t = (int)bvh->getPrimNodeSize();
            int rec[7] = {0x4d415246, f, b, fr, bvh->bvhOptTag(), (int)n, t};
            fwrite(rec, sizeof(int), 7, out);
            put(out, pairs);
            put(out, dev_copy(bvh->clvs().getLcas(), (size_t)t + 1));
            put(out, dev_copy(bvh->clvs().getPars(), (size_t)t));
            put(out, dev_copy(bvh->clvs().getPrimitiveArray().getIdx(), (size_t)t));
            put(out, dev_copy(bvh->getPrimMap(), (size_t)t));
            put(out, dev_copy(bvh->clvs().getMtCodes(), (size_t)t));
            put(out, dev_copy(bvh->ctks().getPars(), (size_t)t - 1));
            put(out, dev_copy(bvh->ctks().getLbds(), (size_t)t - 1));
            put(out, dev_copy(bvh->ctks().getRbds(), (size_t)t - 1));
            put(out, dev_copy(bvh->ctks().getMarks(), (size_t)t - 1));
        }
        fclose(out);
        cudaFree(d_pairs);
        cudaFree(d_cnt);
    }
    Logger::shutdown();
    CudaDevice::shutdown();
    return 0;
}
