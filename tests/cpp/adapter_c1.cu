// adapter_c1.cu -- the reference-side binding of INTEGRATION.md, compiled
// against the reference's own headers and driven by the reference's own
// scheduler, over the C ABI of libbvhcd.so.
//
// TEST INFRASTRUCTURE: built by tests/cpp/Makefile (only where the reference
// tree is present), run by tests/test_gpu_integration_adapter.py.
//
// The adapter classes (LBvhB200, BvttFrontB200, ...) are not written here:
// the Makefile extracts them from INTEGRATION.md into
// _build/integration_adapters.h, so this file proves that the code a
// maintainer would paste compiles against Mine/world/Scene.h and
// Mine/setting/BvhSettings.h and runs.  The frame loop is the reference app's
// (Mine/Frameworks/CudaProject/CudaProjectApp.cpp:49-52): the schedule comes
// from BenchmarkLogic::maintainScheme() (Mine/system/Logic/BenchmarkLogic.hpp:90-156)
// advanced by BenchmarkLogic::next() to the reference's STATIC_MANDATORY
// benchmark (Mine/setting/CDBenchmarkSettings.cpp), the broad pairs come back
// through applyCpResults and the sizes through inspectResults.
//
// Input file: int32 T, V, F; int32 faces[T][3]; float32 frames[F][V][3].
// Output file: per frame int32 count, int32 pairs[count][2].  Stdout: per
// frame the adapter's inspectResults line and the BVH's opt tag.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "integration_adapters.h"
#include "system/Logic/BenchmarkLogic.hpp"

using namespace mn;

static bool read_all(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }

int main(int argc, char **argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: adapter_c1 input output\n");
        return 2;
    }
    FILE *in = fopen(argv[1], "rb");
    if (!in) return 2;
    int hdr[3];
    if (!read_all(in, hdr, sizeof(hdr))) return 2;
    const int T = hdr[0], V = hdr[1], F = hdr[2];
    SceneData data;
    data.fids.resize(T);
    data.pos.resize(V);
    if (!read_all(in, data.fids.data(), sizeof(int3) * (size_t)T)) return 2;
    std::vector<float> frames((size_t)F * V * 3);
    if (!read_all(in, frames.data(), sizeof(float) * frames.size())) return 2;
    fclose(in);

    // the reference's scheduler, advanced to its STATIC_MANDATORY benchmark
    BenchmarkLogic logic;
    bool found = false;
    while (logic.next())
        if (CDBenchmarkSettings::benchmark(logic.currentBenchmarkId()).schemeOpt.type == CDSchemeType::STATIC_MANDATORY) {
            found = true;
            break;
        }
    if (!found) return 3;

    LBvhB200 bvh{LBvhBuildConfig{}};
    BvttFrontB200 front(&bvh, BvttFrontSettings::ext_front_size(), BvttFrontSettings::int_front_size(),
                        BvttFrontSettings::collision_pair_num());
    const int cap = BvttFrontSettings::collision_pair_num();
    uint *d_count = nullptr;
    uint2 *d_pairs = nullptr;
    if (cudaMalloc(&d_count, sizeof(uint)) != cudaSuccess || cudaMalloc(&d_pairs, sizeof(uint2) * cap) != cudaSuccess)
        return 4;
    std::vector<uint2> pairs(cap);
    FILE *out = fopen(argv[2], "wb");
    if (!out) return 2;
    for (int f = 0; f < F; f++) {
        for (int v = 0; v < V; v++) {
            const float *p = frames.data() + 3 * ((size_t)f * V + v);
            data.pos[v] = PointType{p[0], p[1], p[2]};
        }
        auto opts = logic.maintainScheme();
        bvh.maintain(opts.first, data);
        front.maintain(opts.second);
        printf("frame %d bvh_op %d front_op %d opt_tag %d ", f, (int)opts.first, (int)opts.second, bvh.bvhOptTag());
        front.inspectResults();
        front.applyCpResults(d_count, d_pairs);
        uint n = 0;
        if (cudaMemcpy(&n, d_count, sizeof(uint), cudaMemcpyDeviceToHost) != cudaSuccess) return 4;
        if ((int)n > cap) return 5;
        if (n && cudaMemcpy(pairs.data(), d_pairs, sizeof(uint2) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return 4;
        const int ni = (int)n;
        fwrite(&ni, sizeof(int), 1, out);
        fwrite(pairs.data(), sizeof(uint2), n, out);
        logic.next();
    }
    fclose(out);
    cudaFree(d_count);
    cudaFree(d_pairs);
    return 0;
}
