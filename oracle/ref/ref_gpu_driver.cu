// ref_gpu_driver.cu -- runs the reference's own CUDA pipeline
// (LBvhFixedDeformable + BvttFrontLooseIntra, compiled unmodified from the
// reference tree by oracle/ref/Makefile.refgpu) on frames read from a file,
// with the reference's STATIC_MANDATORY / divergent-marks schedule
// (Mine/system/Logic/BenchmarkLogic.hpp:102-117), and writes per frame the
// broad-phase pair list (applyCpResults) and the tree arrays.  It replaces
// only the app shell and the assimp scene loader
// (Mine/Frameworks/CudaProject/CudaProjectApp.cpp:26-59, Mine/world/Scene.cpp).
//
// TEST INFRASTRUCTURE ONLY: it produces the golden fixtures under
// tests/golden/ (oracle/ref/make_golden.py) and is never part of the product.
//
// Input file:  int32 magic 'BVHI', T, V, F; int32 faces[T*3]; float frames[F*V*3]
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

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s frames.bin out.bin\n", argv[0]);
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

    CudaDevice::startup();
    Logger::startup();
    {
        LBvhKernelRegister lbvh_kernels;
        BvttFrontKernelRegister front_kernels;
        auto bvh = std::make_unique<LBvh<ModelType::FixedDeformableType>>(LBvhBuildConfig{});
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
