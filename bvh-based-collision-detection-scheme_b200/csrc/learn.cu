// learn.cu -- the learned scheduler.  No counterpart in the reference, whose
// scheduler is the static cycle of BenchmarkLogic::maintainScheme
// (Mine/system/Logic/BenchmarkLogic.hpp:90-156) plus the front-quality check
// (checkFrontQuality, Mine/collision/bvtt_front/BvttFrontGenerateKernels.cu:34-49).
//
// The tree is cut into disjoint subtrees (every internal node with at most
// smax leaves whose parent has more); per subtree 16 features are computed on
// the GPU every frame, a 16-64-64-3 MLP (BF16 weights, FP32 accumulation)
// votes refit / restructure / regenerate-the-front, and the votes become the
// reference's own maintenance operations: restructure marks on the voted
// subtrees (the BvhRestrLog marks checkFrontQuality would write), and a front
// GENERATE when subtrees holding most leaves vote for it.  None of this
// changes a result: every operation keeps the pair set exact.
//
// Training runs on the GPU as well: one kernel computes the loss gradient of
// a minibatch (forward and backward for 128 rows per block, outer-product
// sums in shared memory), one applies Adam to the FP32 master weights and
// writes the BF16 copy the forward passes read.
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "learn.h"
#include "prims.cuh"

namespace bvhcd {

#define LN_TRY(x)                                        \
    do {                                                 \
        cudaError_t e__ = (x);                           \
        if (e__ != cudaSuccess) return cuda_status(e__); \
    } while (0)

namespace {

constexpr int kThreads = 256;
inline unsigned blocks_for(int64_t n, int per = kThreads) {
    int64_t g = (n + per - 1) / per;
    if (g < 1) g = 1;
    if (g > 65535LL * 16) g = 65535LL * 16;
    return (unsigned)g;
}

// ---------------------------------------------------------------- tree cut
// cut roots: internal nodes with <= smax leaves whose parent has more (or
// that are the root)
__global__ void k_cut_flags(int nint, const int2 *__restrict__ nrange, const int4 *__restrict__ topo, int smax,
                            unsigned *flag) {
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nint; d += gridDim.x * blockDim.x) {
        const int2 r = nrange[d];
        const int size = r.y - r.x + 1;
        bool cut = size <= smax;
        if (cut) {
            const int p = topo[d].z;
            if (p >= 0) {
                const int2 q = nrange[p];
                cut = (q.y - q.x + 1) > smax;
            }
        }
        flag[d] = cut ? 1u : 0u;
    }
}

__global__ void k_cut_compact(int nint, const unsigned *__restrict__ flag, const unsigned *__restrict__ pos,
                              int *roots) {
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nint; d += gridDim.x * blockDim.x)
        if (flag[d]) roots[pos[d]] = d;
}

// ---------------------------------------------------------------- snapshots
__device__ __forceinline__ float box_area(const float4 &lo, const float4 &hi) {
    const float x = fmaxf(hi.x - lo.x, 0.f), y = fmaxf(hi.y - lo.y, 0.f), z = fmaxf(hi.z - lo.z, 0.f);
    return 2.f * (x * y + y * z + z * x);
}
__device__ __forceinline__ float box_volume(const float4 &lo, const float4 &hi) {
    return fmaxf(hi.x - lo.x, 0.f) * fmaxf(hi.y - lo.y, 0.f) * fmaxf(hi.z - lo.z, 0.f);
}

// per node {area, volume} and per leaf box centre, at the last build
__global__ void k_build_snapshot(int T, const float4 *__restrict__ nrec, const float4 *__restrict__ lrec,
                                 float2 *av, float4 *cen) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        if (i < T - 1) {
            const float4 lo = nrec[2 * i], hi = nrec[2 * i + 1];
            av[i] = make_float2(box_area(lo, hi), box_volume(lo, hi));
        }
        const float4 lo = lrec[2 * i], hi = lrec[2 * i + 1];
        cen[i] = make_float4(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z),
                             sqrtf((hi.x - lo.x) * (hi.x - lo.x) + (hi.y - lo.y) * (hi.y - lo.y) +
                                   (hi.z - lo.z) * (hi.z - lo.z)));
    }
}

// mean leaf-box diagonal at the build: a fixed-order two-level sum, so the
// features (and the votes) do not depend on the schedule
constexpr int kDiagBlocks = 256;
__global__ void __launch_bounds__(kThreads) k_diag_partial(int T, const float4 *__restrict__ cen, double *part) {
    const int per = (T + kDiagBlocks - 1) / kDiagBlocks;
    const int a = blockIdx.x * per, b = min(T, a + per);
    double v = 0.0;
    for (int i = a + threadIdx.x; i < b; i += blockDim.x) v += cen[i].w;
    __shared__ double s[kThreads];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}
__global__ void k_diag_final(int T, const double *__restrict__ part, float *diag) {
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int k = 0; k < kDiagBlocks; k++) v += part[k];
        const double m = T > 0 ? v / T : 1.0;
        diag[0] = (float)(m > 1e-30 ? m : 1e-30);
    }
}

// ---------------------------------------------------------------- features
// One warp per cut subtree.  The subtree of DFS node r with leaves [x, y]
// holds the internal nodes [r, r + y - x) and the leaves [x, y]; front
// entries per node are differences of the front log's begins.
__global__ void __launch_bounds__(kThreads) k_features(int ncut, const int *__restrict__ roots, Tree t,
                                                       const unsigned *__restrict__ intbeg,
                                                       const unsigned *__restrict__ extbeg,
                                                       const unsigned *__restrict__ gen_intbeg,
                                                       const unsigned *__restrict__ gen_extbeg,
                                                       const float2 *__restrict__ av_b,
                                                       const float4 *__restrict__ cen_b,
                                                       const float *__restrict__ diag, float since_build,
                                                       float since_gen, float *X) {
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const float inv_diag = 1.f / __ldg(diag);
    for (int c = w; c < ncut; c += nw) {
        const int r = roots[c];
        const int2 rg = t.nrange[r];
        const int size = rg.y - rg.x + 1;
        float sah_now = 0.f, sah_b = 0.f;
        for (int d = r + lane; d < r + size - 1; d += 32) {
            sah_now += box_area(t.nrec[2 * d], t.nrec[2 * d + 1]);
            sah_b += av_b[d].x;
        }
        float dsum = 0.f, dmax = 0.f, dbig = 0.f;
        for (int s = rg.x + lane; s <= rg.y; s += 32) {
            const float4 lo = t.lrec[2 * s], hi = t.lrec[2 * s + 1];
            const float4 cb = cen_b[s];
            const float dx = 0.5f * (lo.x + hi.x) - cb.x, dy = 0.5f * (lo.y + hi.y) - cb.y,
                        dz = 0.5f * (lo.z + hi.z) - cb.z;
            const float dd = sqrtf(dx * dx + dy * dy + dz * dz) * inv_diag;
            dsum += dd;
            dmax = fmaxf(dmax, dd);
            dbig += dd > 0.5f ? 1.f : 0.f;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sah_now += __shfl_xor_sync(0xffffffffu, sah_now, o);
            sah_b += __shfl_xor_sync(0xffffffffu, sah_b, o);
            dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
            dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
            dbig += __shfl_xor_sync(0xffffffffu, dbig, o);
        }
        if (lane == 0) {
            const float a_now = box_area(t.nrec[2 * r], t.nrec[2 * r + 1]);
            const float v_now = box_volume(t.nrec[2 * r], t.nrec[2 * r + 1]);
            const float2 ab = av_b[r];
            int depth = 0;
            for (int p = t.topo[r].z; p >= 0 && depth < 64; p = t.topo[p].z) depth++;
            const float ie = (float)(intbeg[r + size - 1] - intbeg[r]);
            const float ee = (float)(extbeg[rg.y + 1] - extbeg[rg.x]);
            const float ie0 = (float)(gen_intbeg[r + size - 1] - gen_intbeg[r]);
            const float ee0 = (float)(gen_extbeg[rg.y + 1] - gen_extbeg[rg.x]);
            const float inv = 1.f / (float)size;
            float *x = X + 16 * (size_t)c;
            x[0] = log2f((float)size) * (1.f / 16.f);
            x[1] = depth * (1.f / 32.f);
            x[2] = fminf((sah_now / fmaxf(a_now, 1e-30f)) / fmaxf(sah_b / fmaxf(ab.x, 1e-30f), 1e-30f), 16.f);
            x[3] = fminf(fmaxf(logf(fmaxf(v_now, 1e-30f) / fmaxf(ab.y, 1e-30f)), -8.f), 8.f);
            x[4] = fminf(a_now / fmaxf(ab.x, 1e-30f), 16.f);
            x[5] = fminf(dsum * inv, 16.f);
            x[6] = fminf(dmax, 16.f);
            x[7] = fminf((ie + ee) / fmaxf(ie0 + ee0, 1.f), 16.f);
            x[8] = fminf(fmaxf(ie / fmaxf(ee, 1.f) - ie0 / fmaxf(ee0, 1.f), -16.f), 16.f);
            x[9] = fminf(ee * inv, 64.f) * (1.f / 16.f);
            x[10] = fminf(ie * inv, 64.f) * (1.f / 16.f);
            x[11] = since_build * (1.f / 12.f);
            x[12] = since_gen * (1.f / 6.f);
            x[13] = dbig * inv;
            x[14] = log2f((float)t.T) * (1.f / 24.f);
            x[15] = 1.f;
        }
    }
}

// front entries per cut subtree, for counterfactual labelling
__global__ void k_work(int ncut, const int *__restrict__ roots, const int2 *__restrict__ nrange,
                       const unsigned *__restrict__ intbeg, const unsigned *__restrict__ extbeg, int64_t *out) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncut; c += gridDim.x * blockDim.x) {
        const int r = roots[c];
        const int2 rg = nrange[r];
        const int size = rg.y - rg.x + 1;
        out[c] = (int64_t)(intbeg[r + size - 1] - intbeg[r]) + (int64_t)(extbeg[rg.y + 1] - extbeg[rg.x]);
    }
}

// ---------------------------------------------------------------- MLP
// params (FP32 master, kMlpParams): W1[16][64], b1[64], W2[64][64], b2[64],
// W3[64][3], b3[3]; the forward reads the BF16 copy of the weight matrices
// and the FP32 biases.
constexpr int kIn = 16, kH = 64, kOut = 3;
constexpr int oW1 = 0, oB1 = oW1 + kIn * kH, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH * kOut;
static_assert(oB3 + kOut == kMlpParams, "parameter layout");

// The network runs on the tensor cores: mma.sync m16n8k16 with BF16
// operands and FP32 accumulation, one warp per tile of 16 rows.  Inputs,
// activations and back-propagated errors enter each product rounded to BF16
// (nearest even); accumulation, bias, ReLU, softmax and the loss are FP32.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// two values as BF16 in one register, the first in the low half
__device__ __forceinline__ unsigned pack2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned *>(&v);
}
__device__ __forceinline__ unsigned pack2h(unsigned short lo, unsigned short hi) {
    return (unsigned)lo | ((unsigned)hi << 16);
}

// Weights in shared memory as BF16, laid out for the B operands (the two K
// values a lane reads for one output column are adjacent), rows padded so the
// lanes of a warp hit distinct banks: w1t[n][k] = W1[k][n], w2t[n][k] =
// W2[k][n], w3t[c][k] = W3[k][c] (c < 3, zero to 8) for the forward; w2[i][j]
// = W2[i][j], w3p[j][c] = W3[j][c] (zero past 3) for the back-propagation.
constexpr int kS16 = 24, kS64 = 72;  // padded row lengths for K = 16 / 64
struct MlpW {
    __nv_bfloat16 w1t[kH * kS16];
    __nv_bfloat16 w2t[kH * kS64];
    __nv_bfloat16 w2[kH * kS64];
    __nv_bfloat16 w3t[8 * kS64];
    __nv_bfloat16 w3p[kH * kS16];
    float b1[kH], b2[kH], b3[4];
};
__device__ void load_mlp_weights(MlpW &w, const __nv_bfloat16 *__restrict__ wq, const float *__restrict__ p) {
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    for (int i = threadIdx.x; i < kIn * kH; i += blockDim.x) {
        const int k = i / kH, n = i % kH;
        w.w1t[n * kS16 + k] = wq[oW1 + i];
    }
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
        const int k = i / kH, n = i % kH;
        w.w2t[n * kS64 + k] = wq[oW2 + i];
        w.w2[k * kS64 + n] = wq[oW2 + i];
    }
    for (int i = threadIdx.x; i < 8 * kS64; i += blockDim.x) {
        const int c = i / kS64, k = i % kS64;
        w.w3t[i] = (c < kOut && k < kH) ? wq[oW3 + k * kOut + c] : zero;
    }
    for (int i = threadIdx.x; i < kH * kS16; i += blockDim.x) {
        const int j = i / kS16, c = i % kS16;
        w.w3p[i] = c < kOut ? wq[oW3 + j * kOut + c] : zero;
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        w.b1[i] = p[oB1 + i];
        w.b2[i] = p[oB2 + i];
    }
    if (threadIdx.x < 4) w.b3[threadIdx.x] = threadIdx.x < kOut ? p[oB3 + threadIdx.x] : 0.f;
}
// B fragment of n-tile nt, k-step kk from a [n][k] array with row length ld
__device__ __forceinline__ void bfrag(const __nv_bfloat16 *wt, int ld, int nt, int kk, int g, int t, unsigned &b0,
                                      unsigned &b1) {
    const __nv_bfloat16 *q = wt + (nt * 8 + g) * ld + kk * 16 + 2 * t;
    b0 = *reinterpret_cast<const unsigned *>(q);
    b1 = *reinterpret_cast<const unsigned *>(q + 8);
}

// Forward of one 16-row tile in a warp: h1, h2 (FP32, after ReLU) and the
// logits as accumulator fragments (lane g = lane / 4 holds rows g and g + 8,
// columns 2t, 2t + 1 of each 8-column tile, t = lane % 4).
struct Fwd {
    float h1[8][4], h2[8][4], z[4];
};
__device__ __forceinline__ void mlp_forward(const MlpW &w, const unsigned (&ax)[4], int g, int t, Fwd &o) {
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const float b0 = w.b1[nt * 8 + 2 * t], b1 = w.b1[nt * 8 + 2 * t + 1];
        float c[4] = {b0, b1, b0, b1};
        unsigned q0, q1;
        bfrag(w.w1t, kS16, nt, 0, g, t, q0, q1);
        mma_bf16(c, ax, q0, q1);
#pragma unroll
        for (int e = 0; e < 4; e++) o.h1[nt][e] = fmaxf(c[e], 0.f);
    }
    unsigned a[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {  // accumulator fragments of two column tiles = one A fragment
        a[kk][0] = pack2(o.h1[2 * kk][0], o.h1[2 * kk][1]);
        a[kk][1] = pack2(o.h1[2 * kk][2], o.h1[2 * kk][3]);
        a[kk][2] = pack2(o.h1[2 * kk + 1][0], o.h1[2 * kk + 1][1]);
        a[kk][3] = pack2(o.h1[2 * kk + 1][2], o.h1[2 * kk + 1][3]);
    }
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const float b0 = w.b2[nt * 8 + 2 * t], b1 = w.b2[nt * 8 + 2 * t + 1];
        float c[4] = {b0, b1, b0, b1};
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            unsigned q0, q1;
            bfrag(w.w2t, kS64, nt, kk, g, t, q0, q1);
            mma_bf16(c, a[kk], q0, q1);
        }
#pragma unroll
        for (int e = 0; e < 4; e++) o.h2[nt][e] = fmaxf(c[e], 0.f);
    }
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        a[kk][0] = pack2(o.h2[2 * kk][0], o.h2[2 * kk][1]);
        a[kk][1] = pack2(o.h2[2 * kk][2], o.h2[2 * kk][3]);
        a[kk][2] = pack2(o.h2[2 * kk + 1][0], o.h2[2 * kk + 1][1]);
        a[kk][3] = pack2(o.h2[2 * kk + 1][2], o.h2[2 * kk + 1][3]);
    }
    const float c0 = 2 * t < kOut ? w.b3[2 * t] : 0.f, c1 = 2 * t + 1 < kOut ? w.b3[2 * t + 1] : 0.f;
    o.z[0] = c0; o.z[1] = c1; o.z[2] = c0; o.z[3] = c1;
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        unsigned q0, q1;
        bfrag(w.w3t, kS64, 0, kk, g, t, q0, q1);
        mma_bf16(o.z, a[kk], q0, q1);
    }
}
// A fragment of the inputs of rows r0 + g, r0 + g + 8 (zero past n)
__device__ __forceinline__ void xfrag(const float *__restrict__ X, int n, int r0, int g, int t, unsigned (&ax)[4]) {
    float v[2][4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int r = r0 + g + 8 * h;
        const float *x = X + kIn * (size_t)r;
        const bool ok = r < n;
        v[h][0] = ok ? x[2 * t] : 0.f;
        v[h][1] = ok ? x[2 * t + 1] : 0.f;
        v[h][2] = ok ? x[2 * t + 8] : 0.f;
        v[h][3] = ok ? x[2 * t + 9] : 0.f;
    }
    ax[0] = pack2(v[0][0], v[0][1]);
    ax[1] = pack2(v[1][0], v[1][1]);
    ax[2] = pack2(v[0][2], v[0][3]);
    ax[3] = pack2(v[1][2], v[1][3]);
}

// logits and the argmax vote, one warp per 16-row tile
__global__ void __launch_bounds__(kThreads) k_mlp_infer(int n, const float *__restrict__ X,
                                                        const __nv_bfloat16 *__restrict__ wq,
                                                        const float *__restrict__ p, float *logits, int *vote) {
    __shared__ __align__(16) MlpW w;
    load_mlp_weights(w, wq, p);
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int tile = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 16 < n; tile += warps) {
        const int r0 = tile * 16;
        unsigned ax[4];
        xfrag(X, n, r0, g, t, ax);
        Fwd o;
        mlp_forward(w, ax, g, t, o);
        // column 2 of rows g and g + 8 sits in lane t = 1
        const float z2a = __shfl_down_sync(0xffffffffu, o.z[0], 1), z2b = __shfl_down_sync(0xffffffffu, o.z[2], 1);
        if (t == 0) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = r0 + g + 8 * h;
                if (r >= n) continue;
                const float zz[3] = {o.z[2 * h], o.z[2 * h + 1], h ? z2b : z2a};
                int best = 0;
#pragma unroll
                for (int c = 0; c < kOut; c++) {
                    if (logits) logits[kOut * (size_t)r + c] = zz[c];
                    if (zz[c] > zz[best]) best = c;
                }
                if (vote) vote[r] = best;
            }
        }
    }
}

// Minibatch gradient of the class-weighted cross-entropy
// L = (1/N) sum_r cw[y_r] CE(softmax(logits_r), y_r), accumulated into grad
// (FP32) and loss.  128 rows per block, 16 per warp.  Each warp runs the
// forward and the back-propagation of its rows on the tensor cores (the
// output error through W3 and W2, masked by the ReLUs), and leaves the BF16
// inputs, activations and errors of its rows in shared memory; then the
// block's weight gradients are products over its 128 rows, Actᵀ · Err, again
// on the tensor cores (44 output tiles of 16 x 8 shared by the 8 warps), and
// the bias gradients column sums of the errors.
constexpr int kRows = 128;
struct GradSmem {
    MlpW w;
    __nv_bfloat16 x[kRows * kS16];    // inputs, columns 0..15
    __nv_bfloat16 h1[kRows * kS64];
    __nv_bfloat16 h2[kRows * kS64];
    __nv_bfloat16 d1[kRows * kS64];   // errors at the first hidden layer's pre-activations
    __nv_bfloat16 d2[kRows * kS64];
    __nv_bfloat16 dl[kRows * kS16];   // errors at the logits, columns 0..2 (zero to 16)
};
// one 16 x 8 tile of Actᵀ · Err over the block's rows: rows m0..m0+15 of
// Actᵀ (feature columns of act), columns n0..n0+7 of err
__device__ __forceinline__ void wgrad_tile(const __nv_bfloat16 *act, int lda, const __nv_bfloat16 *err, int lde,
                                           int m0, int n0, int g, int t, float (&c)[4]) {
    const unsigned short *A = reinterpret_cast<const unsigned short *>(act);
    const unsigned short *E = reinterpret_cast<const unsigned short *>(err);
    c[0] = c[1] = c[2] = c[3] = 0.f;
#pragma unroll 2
    for (int k0 = 0; k0 < kRows; k0 += 16) {
        const int ra = k0 + 2 * t;
        unsigned a[4];
        a[0] = pack2h(A[ra * lda + m0 + g], A[(ra + 1) * lda + m0 + g]);
        a[1] = pack2h(A[ra * lda + m0 + g + 8], A[(ra + 1) * lda + m0 + g + 8]);
        a[2] = pack2h(A[(ra + 8) * lda + m0 + g], A[(ra + 9) * lda + m0 + g]);
        a[3] = pack2h(A[(ra + 8) * lda + m0 + g + 8], A[(ra + 9) * lda + m0 + g + 8]);
        const unsigned b0 = pack2h(E[ra * lde + n0 + g], E[(ra + 1) * lde + n0 + g]);
        const unsigned b1 = pack2h(E[(ra + 8) * lde + n0 + g], E[(ra + 9) * lde + n0 + g]);
        mma_bf16(c, a, b0, b1);
    }
}

__global__ void __launch_bounds__(kThreads) k_mlp_grad(int n, const float *__restrict__ X, const int *__restrict__ y,
                                                       const float *__restrict__ cw, float inv_n,
                                                       const __nv_bfloat16 *__restrict__ wq,
                                                       const float *__restrict__ p, float *grad, float *loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &sm = *reinterpret_cast<GradSmem *>(smem_raw);
    load_mlp_weights(sm.w, wq, p);
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    for (int i = threadIdx.x; i < kRows * kS16; i += blockDim.x) sm.dl[i] = zero;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int rb = blockIdx.x * kRows;         // the block's first row
    const int r0 = rb + warp * 16, l0 = warp * 16;  // the warp's first row, globally and in the block
    unsigned ax[4];
    xfrag(X, n, r0, g, t, ax);
    Fwd o;
    mlp_forward(sm.w, ax, g, t, o);
    // inputs and activations of the warp's rows, BF16 (what the products read)
    {
        unsigned *xs = reinterpret_cast<unsigned *>(sm.x);
        xs[((l0 + g) * kS16 + 2 * t) >> 1] = ax[0];
        xs[((l0 + g + 8) * kS16 + 2 * t) >> 1] = ax[1];
        xs[((l0 + g) * kS16 + 2 * t + 8) >> 1] = ax[2];
        xs[((l0 + g + 8) * kS16 + 2 * t + 8) >> 1] = ax[3];
        unsigned *h1s = reinterpret_cast<unsigned *>(sm.h1), *h2s = reinterpret_cast<unsigned *>(sm.h2);
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            h1s[((l0 + g) * kS64 + nt * 8 + 2 * t) >> 1] = pack2(o.h1[nt][0], o.h1[nt][1]);
            h1s[((l0 + g + 8) * kS64 + nt * 8 + 2 * t) >> 1] = pack2(o.h1[nt][2], o.h1[nt][3]);
            h2s[((l0 + g) * kS64 + nt * 8 + 2 * t) >> 1] = pack2(o.h2[nt][0], o.h2[nt][1]);
            h2s[((l0 + g + 8) * kS64 + nt * 8 + 2 * t) >> 1] = pack2(o.h2[nt][2], o.h2[nt][3]);
        }
    }
    // softmax cross-entropy of rows g and g + 8 in lane t = 0; their errors
    // at the logits (zero for rows past n), BF16 into shared memory
    const float z2a = __shfl_down_sync(0xffffffffu, o.z[0], 1), z2b = __shfl_down_sync(0xffffffffu, o.z[2], 1);
    float my_loss = 0.f;
    if (t == 0) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int r = r0 + g + 8 * h;
            const float zz[3] = {o.z[2 * h], o.z[2 * h + 1], h ? z2b : z2a};
            float d[3] = {0.f, 0.f, 0.f};
            if (r < n) {
                const float m = fmaxf(zz[0], fmaxf(zz[1], zz[2]));
                float e[kOut], s = 0.f;
#pragma unroll
                for (int c = 0; c < kOut; c++) {
                    e[c] = expf(zz[c] - m);
                    s += e[c];
                }
                const int lab = y[r];
                const float wt = cw[lab] * inv_n;
                my_loss += wt * (logf(s) + m - zz[lab]);
#pragma unroll
                for (int c = 0; c < kOut; c++) d[c] = wt * (e[c] / s - (c == lab ? 1.f : 0.f));
            }
#pragma unroll
            for (int c = 0; c < kOut; c++) sm.dl[(l0 + g + 8 * h) * kS16 + c] = __float2bfloat16_rn(d[c]);
        }
    }
    __syncwarp();
    // errors at the second hidden layer: (dl · W3ᵀ) masked by h2 > 0
    unsigned adl[4];
    {
        const unsigned *dls = reinterpret_cast<const unsigned *>(sm.dl);
        adl[0] = dls[((l0 + g) * kS16 + 2 * t) >> 1];
        adl[1] = dls[((l0 + g + 8) * kS16 + 2 * t) >> 1];
        adl[2] = dls[((l0 + g) * kS16 + 2 * t + 8) >> 1];
        adl[3] = dls[((l0 + g + 8) * kS16 + 2 * t + 8) >> 1];
    }
    float d2[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        unsigned q0, q1;
        bfrag(sm.w.w3p, kS16, nt, 0, g, t, q0, q1);
        mma_bf16(c, adl, q0, q1);
#pragma unroll
        for (int e = 0; e < 4; e++) d2[nt][e] = o.h2[nt][e] > 0.f ? c[e] : 0.f;
    }
    unsigned a[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        a[kk][0] = pack2(d2[2 * kk][0], d2[2 * kk][1]);
        a[kk][1] = pack2(d2[2 * kk][2], d2[2 * kk][3]);
        a[kk][2] = pack2(d2[2 * kk + 1][0], d2[2 * kk + 1][1]);
        a[kk][3] = pack2(d2[2 * kk + 1][2], d2[2 * kk + 1][3]);
    }
    {
        unsigned *d2s = reinterpret_cast<unsigned *>(sm.d2);
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            d2s[((l0 + g) * kS64 + 16 * kk + 2 * t) >> 1] = a[kk][0];
            d2s[((l0 + g + 8) * kS64 + 16 * kk + 2 * t) >> 1] = a[kk][1];
            d2s[((l0 + g) * kS64 + 16 * kk + 8 + 2 * t) >> 1] = a[kk][2];
            d2s[((l0 + g + 8) * kS64 + 16 * kk + 8 + 2 * t) >> 1] = a[kk][3];
        }
    }
    // errors at the first hidden layer: (d2 · W2ᵀ) masked by h1 > 0
    {
        unsigned *d1s = reinterpret_cast<unsigned *>(sm.d1);
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                unsigned q0, q1;
                bfrag(sm.w.w2, kS64, nt, kk, g, t, q0, q1);
                mma_bf16(c, a[kk], q0, q1);
            }
#pragma unroll
            for (int e = 0; e < 4; e++) c[e] = o.h1[nt][e] > 0.f ? c[e] : 0.f;
            d1s[((l0 + g) * kS64 + nt * 8 + 2 * t) >> 1] = pack2(c[0], c[1]);
            d1s[((l0 + g + 8) * kS64 + nt * 8 + 2 * t) >> 1] = pack2(c[2], c[3]);
        }
    }
    __syncthreads();
    // weight gradients: tiles 0..7 of dW1 (16 x 64), 8..39 of dW2 (64 x 64),
    // 40..43 of dW3 (64 x 3, padded to 8 columns)
    for (int tile = warp; tile < 44; tile += kThreads / 32) {
        float c[4];
        int base, ld, m0, n0, ncol;
        if (tile < 8) {
            m0 = 0; n0 = tile * 8;
            wgrad_tile(sm.x, kS16, sm.d1, kS64, m0, n0, g, t, c);
            base = oW1; ld = kH; ncol = kH;
        } else if (tile < 40) {
            m0 = ((tile - 8) >> 3) * 16; n0 = ((tile - 8) & 7) * 8;
            wgrad_tile(sm.h1, kS64, sm.d2, kS64, m0, n0, g, t, c);
            base = oW2; ld = kH; ncol = kH;
        } else {
            m0 = (tile - 40) * 16; n0 = 0;
            wgrad_tile(sm.h2, kS64, sm.dl, kS16, m0, n0, g, t, c);
            base = oW3; ld = kOut; ncol = kOut;
        }
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int row = m0 + g + ((e >> 1) << 3), col = n0 + 2 * t + (e & 1);
            if (col < ncol) atomicAdd(grad + base + row * ld + col, c[e]);
        }
    }
    // bias gradients: column sums of the BF16 errors
    for (int i = threadIdx.x; i < kH + kH + kOut; i += blockDim.x) {
        const __nv_bfloat16 *src;
        int ld, col, dst;
        if (i < kH) { src = sm.d1; ld = kS64; col = i; dst = oB1 + i; }
        else if (i < 2 * kH) { src = sm.d2; ld = kS64; col = i - kH; dst = oB2 + col; }
        else { src = sm.dl; ld = kS16; col = i - 2 * kH; dst = oB3 + col; }
        float gsum = 0.f;
        for (int r = 0; r < kRows; r++) gsum += __bfloat162float(src[r * ld + col]);
        atomicAdd(grad + dst, gsum);
    }
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, o2);
    if (lane == 0 && my_loss != 0.f) atomicAdd(loss, my_loss);
}

// Adam on the FP32 master weights (Kingma & Ba), then the BF16 copy.
__global__ void k_adam(int n, float *p, float *g, float *m, float *v, __nv_bfloat16 *wq, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        wq[i] = __float2bfloat16_rn(pi);
        g[i] = 0.f;
    }
}

__global__ void k_to_bf16(int n, const float *__restrict__ p, __nv_bfloat16 *wq) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        wq[i] = __float2bfloat16_rn(p[i]);
}

// gather rows `idx` of X / y into a contiguous minibatch
__global__ void k_gather_rows(int n, const int *__restrict__ idx, const float *__restrict__ X,
                              const int *__restrict__ y, float *Xb, int *yb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * kIn; i += gridDim.x * blockDim.x) {
        const int r = i / kIn, k = i % kIn;
        Xb[i] = X[kIn * (size_t)idx[r] + k];
        if (k == 0) yb[r] = y[idx[r]];
    }
}

// votes -> restructure root list and the leaf-weighted share of front
// regeneration votes: out[0] = restructure roots, out[1] = leaves voting
// regenerate, out[2] = leaves covered by the cut
__global__ void k_actions(int ncut, const int *__restrict__ roots, const int *__restrict__ vote,
                          const int2 *__restrict__ nrange, int *rt_roots, unsigned long long *out) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncut; c += gridDim.x * blockDim.x) {
        const int r = roots[c];
        const int2 rg = nrange[r];
        const unsigned long long size = (unsigned long long)(rg.y - rg.x + 1);
        atomicAdd(out + 2, size);
        if (vote[c] == 1) rt_roots[atomicAdd(out, 1ull)] = r;
        else if (vote[c] == 2) atomicAdd(out + 1, size);
    }
}

// restructure marks (the BvhRestrLog marks checkFrontQuality writes,
// BvttFrontGenerateKernels.cu:44-46) for the voted roots, count on the device;
// the log is reset first (no other marker runs beside the learner)
__global__ void k_mark_voted(int T, const unsigned long long *__restrict__ act, const int *__restrict__ roots,
                             const int2 *__restrict__ nrange, int *intrange, int *rtroot) {
    const int n = (int)act[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = roots[k];
        const int2 r = nrange[i];
        atomicAdd(intrange + i, 1);
        atomicAdd(intrange + i + r.y - r.x, -1);
        atomicMin(rtroot + r.x, i);
    }
}

__global__ void k_reset_marks(int T, int *intrange, int *rtroot) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < T; i += gridDim.x * blockDim.x) {
        intrange[i] = 0;
        rtroot[i] = INT_MAX;
    }
}

}  // namespace

// ====================================================================== host
Learner::~Learner() {
    DBuf *bufs[] = {&roots_, &flag_, &pos_, &scratch_, &av_b_, &cen_b_, &diag_, &dpart_, &gen_intbeg_,
                    &gen_extbeg_, &X_, &logits_, &vote_, &rt_roots_, &act_, &work_, &p_, &wq_, &g_, &m_, &v_,
                    &loss_, &bx_, &by_, &bidx_, &cw_};
    for (DBuf *b : bufs) b->release();
    if (h_act_) cudaFreeHost(h_act_);
    if (ev_) cudaEventDestroy(ev_);
}

bvhcd_status Learner::init() {
    // restructure marks need a BVH that restructures; a forest has no restructure
    if (smax_ < 2 || !bvh_->restr_enabled() || bvh_->num_scenes() != 1) return BVHCD_INVALID_ARG;
    front_->set_quality_check(false);
    LN_TRY(p_.reserve(sizeof(float) * kMlpParams));
    LN_TRY(wq_.reserve(sizeof(__nv_bfloat16) * kMlpParams));
    LN_TRY(g_.reserve(sizeof(float) * kMlpParams));
    LN_TRY(m_.reserve(sizeof(float) * kMlpParams));
    LN_TRY(v_.reserve(sizeof(float) * kMlpParams));
    LN_TRY(loss_.reserve(sizeof(float)));
    LN_TRY(act_.reserve(sizeof(unsigned long long) * 4));
    LN_TRY(diag_.reserve(sizeof(float)));
    LN_TRY(dpart_.reserve(sizeof(double) * kDiagBlocks));
    LN_TRY(cw_.reserve(sizeof(float) * 3));
    LN_TRY(cudaMallocHost(&h_act_, sizeof(unsigned long long) * 4));
    LN_TRY(cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming));
    // He-style initialisation from a fixed LCG, so an untrained network is reproducible
    std::vector<float> p(kMlpParams, 0.f);
    unsigned long long st = 0x9E3779B97F4A7C15ull;
    auto rnd = [&]() {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return ((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
    };
    for (int i = oW1; i < oB1; i++) p[i] = (float)(rnd() * std::sqrt(6.0 / kIn));
    for (int i = oW2; i < oB2; i++) p[i] = (float)(rnd() * std::sqrt(6.0 / kH));
    for (int i = oW3; i < oB3; i++) p[i] = (float)(rnd() * std::sqrt(6.0 / kH));
    return set_params(p.data());
}

bvhcd_status Learner::set_params(const float *host) {
    LN_TRY(cudaMemcpy(p_.p, host, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    k_to_bf16<<<blocks_for(kMlpParams), kThreads>>>(kMlpParams, p_.as<float>(), wq_.as<__nv_bfloat16>());
    note_launch();
    LN_TRY(cudaMemset(g_.p, 0, sizeof(float) * kMlpParams));
    LN_TRY(cudaMemset(m_.p, 0, sizeof(float) * kMlpParams));
    LN_TRY(cudaMemset(v_.p, 0, sizeof(float) * kMlpParams));
    adam_t_ = 0;
    LN_TRY(cudaDeviceSynchronize());
    return BVHCD_OK;
}

bvhcd_status Learner::get_params(float *host) const {
    LN_TRY(cudaMemcpy(host, p_.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
    return BVHCD_OK;
}

// After a build or a restructure: the cut and the build-time references.
bvhcd_status Learner::on_tree_changed(cudaStream_t s) {
    const int T = bvh_->T();
    ncut_ = 0;
    since_build_ = 0;
    tree_epoch_++;
    if (T < 2) return BVHCD_OK;
    Tree t = bvh_->tree();
    LN_TRY(flag_.reserve(sizeof(unsigned) * (size_t)(T + 1)));
    LN_TRY(pos_.reserve(sizeof(unsigned) * (size_t)(T + 1)));
    LN_TRY(roots_.reserve(sizeof(int) * (size_t)(T + 1)));
    LN_TRY(scratch_.reserve(scan_scratch_bytes((int64_t)T + 1)));
    LN_TRY(av_b_.reserve(sizeof(float2) * (size_t)T));
    LN_TRY(cen_b_.reserve(sizeof(float4) * (size_t)T));
    LN_TRY(cudaMemsetAsync(flag_.p, 0, sizeof(unsigned) * (size_t)(T + 1), s));
    k_cut_flags<<<blocks_for(T - 1), kThreads, 0, s>>>(T - 1, t.nrange, t.topo, smax_, flag_.as<unsigned>());
    note_launch();
    LN_TRY(scan_u32(flag_.as<unsigned>(), pos_.as<unsigned>(), T, false, nullptr, scratch_.p, s));
    k_cut_compact<<<blocks_for(T - 1), kThreads, 0, s>>>(T - 1, flag_.as<unsigned>(), pos_.as<unsigned>(),
                                                         roots_.as<int>());
    note_launch();
    k_build_snapshot<<<blocks_for(T), kThreads, 0, s>>>(T, t.nrec, t.lrec, av_b_.as<float2>(), cen_b_.as<float4>());
    note_launch();
    k_diag_partial<<<kDiagBlocks, kThreads, 0, s>>>(T, cen_b_.as<float4>(), dpart_.as<double>());
    note_launch();
    k_diag_final<<<1, 32, 0, s>>>(T, dpart_.as<double>(), diag_.as<float>());
    note_launch();
    unsigned n = 0;  // exclusive scan over T flags (flag[T-1] = 0): pos[T-1] counts every cut root
    LN_TRY(cudaMemcpyAsync(&n, pos_.as<unsigned>() + (T - 1), sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    LN_TRY(cudaStreamSynchronize(s));
    ncut_ = (int)n;
    LN_TRY(X_.reserve(sizeof(float) * 16 * (size_t)(ncut_ > 0 ? ncut_ : 1)));
    LN_TRY(logits_.reserve(sizeof(float) * 3 * (size_t)(ncut_ > 0 ? ncut_ : 1)));
    LN_TRY(vote_.reserve(sizeof(int) * (size_t)(ncut_ > 0 ? ncut_ : 1)));
    LN_TRY(rt_roots_.reserve(sizeof(int) * (size_t)(ncut_ > 0 ? ncut_ : 1)));
    LN_TRY(work_.reserve(sizeof(int64_t) * (size_t)(ncut_ > 0 ? ncut_ : 1)));
    return BVHCD_OK;
}

// After a front GENERATE: the per-node entry counts of the fresh front.
bvhcd_status Learner::on_front_generated(cudaStream_t s) {
    const int T = bvh_->T();
    since_gen_ = 0;
    if (T < 2) return BVHCD_OK;
    FrontLog l = front_->front_log();
    LN_TRY(gen_intbeg_.reserve(sizeof(unsigned) * (size_t)(T + 1)));
    LN_TRY(gen_extbeg_.reserve(sizeof(unsigned) * (size_t)(T + 1)));
    LN_TRY(cudaMemcpyAsync(gen_intbeg_.p, l.intbeg, sizeof(unsigned) * (size_t)(T + 1), cudaMemcpyDeviceToDevice, s));
    LN_TRY(cudaMemcpyAsync(gen_extbeg_.p, l.extbeg, sizeof(unsigned) * (size_t)(T + 1), cudaMemcpyDeviceToDevice, s));
    return BVHCD_OK;
}

bvhcd_status Learner::features(cudaStream_t s) {
    if (ncut_ == 0) return BVHCD_OK;
    if (!gen_intbeg_.p) return BVHCD_NOT_READY;
    FrontLog l = front_->front_log();
    k_features<<<blocks_for((int64_t)ncut_ * 32), kThreads, 0, s>>>(
        ncut_, roots_.as<int>(), bvh_->tree(), l.intbeg, l.extbeg, gen_intbeg_.as<unsigned>(),
        gen_extbeg_.as<unsigned>(), av_b_.as<float2>(), cen_b_.as<float4>(), diag_.as<float>(), (float)since_build_,
        (float)since_gen_, X_.as<float>());
    note_launch();
    return cuda_status(cudaGetLastError());
}

bvhcd_status Learner::work(const Front &f, int64_t *host, cudaStream_t s) {
    if (ncut_ == 0) return BVHCD_OK;
    FrontLog l = f.front_log();
    k_work<<<blocks_for(ncut_), kThreads, 0, s>>>(ncut_, roots_.as<int>(), bvh_->tree().nrange, l.intbeg, l.extbeg,
                                                 work_.as<int64_t>());
    note_launch();
    LN_TRY(cudaMemcpyAsync(host, work_.p, sizeof(int64_t) * (size_t)ncut_, cudaMemcpyDeviceToHost, s));
    LN_TRY(cudaStreamSynchronize(s));
    return BVHCD_OK;
}

bvhcd_status Learner::predict(const float *X, int n, float *logits, int *vote, cudaStream_t s) {
    if (n <= 0) return BVHCD_OK;
    k_mlp_infer<<<blocks_for(n), kThreads, 0, s>>>(n, X, wq_.as<__nv_bfloat16>(), p_.as<float>(), logits, vote);
    note_launch();
    return cuda_status(cudaGetLastError());
}

bvhcd_status Learner::gradient(const float *X, const int *y, const float *cw, int n, float *grad_host,
                               float *loss_host, cudaStream_t s) {
    if (n <= 0) return BVHCD_INVALID_ARG;
    LN_TRY(cudaMemsetAsync(g_.p, 0, sizeof(float) * kMlpParams, s));
    LN_TRY(cudaMemsetAsync(loss_.p, 0, sizeof(float), s));
    LN_TRY(cudaMemcpyAsync(cw_.p, cw, sizeof(float) * 3, cudaMemcpyHostToDevice, s));
    LN_TRY(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GradSmem)));
    k_mlp_grad<<<(n + kRows - 1) / kRows, kThreads, sizeof(GradSmem), s>>>(
        n, X, y, cw_.as<float>(), 1.f / n, wq_.as<__nv_bfloat16>(), p_.as<float>(), g_.as<float>(), loss_.as<float>());
    note_launch();
    LN_TRY(cudaGetLastError());
    if (grad_host) LN_TRY(cudaMemcpyAsync(grad_host, g_.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, s));
    if (loss_host) LN_TRY(cudaMemcpyAsync(loss_host, loss_.p, sizeof(float), cudaMemcpyDeviceToHost, s));
    LN_TRY(cudaStreamSynchronize(s));
    LN_TRY(cudaMemsetAsync(g_.p, 0, sizeof(float) * kMlpParams, s));
    return BVHCD_OK;
}

// Minibatch Adam over (X, y) resident on the device; minibatches follow a
// fixed-seed shuffle per epoch.  Returns the mean loss of the last epoch.
bvhcd_status Learner::train(const float *X, const int *y, int n, const float *cw, int epochs, int batch, float lr,
                            unsigned seed, float *last_loss, cudaStream_t s) {
    if (n <= 0 || epochs <= 0 || batch <= 0 || batch > (1 << 20)) return BVHCD_INVALID_ARG;
    LN_TRY(bx_.reserve(sizeof(float) * 16 * (size_t)batch));
    LN_TRY(by_.reserve(sizeof(int) * (size_t)batch));
    LN_TRY(bidx_.reserve(sizeof(int) * (size_t)n));
    LN_TRY(cudaMemcpyAsync(cw_.p, cw, sizeof(float) * 3, cudaMemcpyHostToDevice, s));
    LN_TRY(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GradSmem)));
    std::vector<int> order((size_t)n);
    unsigned long long st = 0x2545F4914F6CDD1Dull ^ seed;
    double epoch_loss = 0.0;
    for (int ep = 0; ep < epochs; ep++) {
        for (int i = 0; i < n; i++) order[(size_t)i] = i;
        for (int i = n - 1; i > 0; i--) {  // Fisher-Yates with an LCG
            st = st * 6364136223846793005ull + 1442695040888963407ull;
            const int j = (int)((st >> 33) % (unsigned long long)(i + 1));
            std::swap(order[(size_t)i], order[(size_t)j]);
        }
        LN_TRY(cudaMemcpyAsync(bidx_.p, order.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
        LN_TRY(cudaMemsetAsync(loss_.p, 0, sizeof(float), s));
        int nb = 0;
        for (int b0 = 0; b0 < n; b0 += batch, nb++) {
            const int m = n - b0 < batch ? n - b0 : batch;
            k_gather_rows<<<blocks_for((int64_t)m * 16), kThreads, 0, s>>>(m, bidx_.as<int>() + b0, X, y,
                                                                             bx_.as<float>(), by_.as<int>());
            note_launch();
            k_mlp_grad<<<(m + kRows - 1) / kRows, kThreads, sizeof(GradSmem), s>>>(
                m, bx_.as<float>(), by_.as<int>(), cw_.as<float>(), 1.f / m, wq_.as<__nv_bfloat16>(), p_.as<float>(),
                g_.as<float>(), loss_.as<float>());
            note_launch();
            adam_t_++;
            const float b1 = 0.9f, b2 = 0.999f;
            k_adam<<<blocks_for(kMlpParams), kThreads, 0, s>>>(kMlpParams, p_.as<float>(), g_.as<float>(), m_.as<float>(),
                                                             v_.as<float>(), wq_.as<__nv_bfloat16>(), lr, b1, b2, 1e-8f,
                                                             1.f - std::pow(b1, (float)adam_t_),
                                                             1.f - std::pow(b2, (float)adam_t_));
            note_launch();
        }
        float l = 0.f;
        LN_TRY(cudaMemcpyAsync(&l, loss_.p, sizeof(float), cudaMemcpyDeviceToHost, s));
        LN_TRY(cudaStreamSynchronize(s));
        epoch_loss = nb ? l / nb : 0.0;
    }
    if (last_loss) *last_loss = (float)epoch_loss;
    return cuda_status(cudaGetLastError());
}

// One decision: features -> votes -> restructure marks for the next BVH
// maintain and the regenerate flag for the next front op.
bvhcd_status Learner::decide(cudaStream_t s, int *n_restructure, double *regen_share) {
    *n_restructure = 0;
    *regen_share = 0.0;
    if (ncut_ == 0) return BVHCD_OK;
    bvhcd_status st = features(s);
    if (st != BVHCD_OK) return st;
    st = predict(X_.as<float>(), ncut_, nullptr, vote_.as<int>(), s);
    if (st != BVHCD_OK) return st;
    LN_TRY(cudaMemsetAsync(act_.p, 0, sizeof(unsigned long long) * 4, s));
    k_actions<<<blocks_for(ncut_), kThreads, 0, s>>>(ncut_, roots_.as<int>(), vote_.as<int>(), bvh_->tree().nrange,
                                                    rt_roots_.as<int>(), act_.as<unsigned long long>());
    note_launch();
    LN_TRY(cudaMemcpyAsync(h_act_, act_.p, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, s));
    LN_TRY(cudaStreamSynchronize(s));
    *n_restructure = (int)h_act_[0];
    *regen_share = h_act_[2] ? (double)h_act_[1] / (double)h_act_[2] : 0.0;
    if (*n_restructure > 0) {
        st = bvh_->request_restructure_device(rt_roots_.as<int>(), *n_restructure, s);
        if (st != BVHCD_OK) return st;
    }
    return BVHCD_OK;
}

// Decision without a host wait: the votes are turned into restructure marks
// and counts on the device, the counts copied to pinned memory and an event
// recorded; a later frame applies them once the event has completed, unless
// the tree changed in between (the marks name subtrees of the tree they were
// voted on).
bvhcd_status Learner::decide_async(cudaStream_t s) {
    if (pending_ || ncut_ == 0 || bvh_->updated()) return BVHCD_OK;
    bvhcd_status st = features(s);
    if (st != BVHCD_OK) return st;
    st = predict(X_.as<float>(), ncut_, nullptr, vote_.as<int>(), s);
    if (st != BVHCD_OK) return st;
    const int T = bvh_->T();
    LN_TRY(cudaMemsetAsync(act_.p, 0, sizeof(unsigned long long) * 4, s));
    k_actions<<<blocks_for(ncut_), kThreads, 0, s>>>(ncut_, roots_.as<int>(), vote_.as<int>(), bvh_->tree().nrange,
                                                    rt_roots_.as<int>(), act_.as<unsigned long long>());
    note_launch();
    k_reset_marks<<<blocks_for(T), kThreads, 0, s>>>(T, bvh_->intrange(), bvh_->rtroot());
    note_launch();
    k_mark_voted<<<blocks_for(ncut_), kThreads, 0, s>>>(T, act_.as<unsigned long long>(), rt_roots_.as<int>(),
                                                       bvh_->tree().nrange, bvh_->intrange(), bvh_->rtroot());
    note_launch();
    LN_TRY(cudaMemcpyAsync(h_act_, act_.p, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, s));
    LN_TRY(cudaEventRecord(ev_, s));
    pending_ = true;
    pending_epoch_ = tree_epoch_;
    return BVHCD_OK;
}

void Learner::poll() {
    if (!pending_ || cudaEventQuery(ev_) != cudaSuccess) return;
    pending_ = false;
    if (pending_epoch_ != tree_epoch_) return;
    last_restructure_ = (int)h_act_[0];
    last_regen_share_ = h_act_[2] ? (double)h_act_[1] / (double)h_act_[2] : 0.0;
    if (last_restructure_ > 0) bvh_->set_updated(true);
    regen_pending_ = last_regen_share_ > regen_threshold_;
    decisions_applied_++;
}

// The learned frame: apply a completed decision, BVH refit (a restructure
// when a decision marked subtrees; a build on the first frame), KEEP or the
// front op of the reference's cycle when one is set -- or GENERATE after a
// build or restructure, or when a decision voted it -- then, every
// decide_every frames, the next decision (queued, applied in a later frame).
bvhcd_status Learner::frame(const bvhcd_scene &scene, int32_t frame_no, cudaStream_t s, int32_t *bvh_op_run,
                            int32_t *front_op_run) {
    if (frame_no < 0) return BVHCD_INVALID_ARG;
    poll();
    const bool first = !bvh_->built() || frame_no == 0;
    if (first) pending_ = false;
    bvhcd_status st = bvh_->maintain(first ? BVHCD_BVH_BUILD : BVHCD_BVH_REFIT, scene, s);
    if (st != BVHCD_OK) return st;
    const int tag = bvh_->opt_tag();
    const bool rebuilt = first || tag == 1 || tag == 2;
    if (rebuilt) {
        st = on_tree_changed(s);
        if (st != BVHCD_OK) return st;
    } else {
        since_build_++;
    }
    bvhcd_front_op fop;
    const int k = front_cycle_ ? frame_no % front_cycle_ : 1;
    if (rebuilt || regen_pending_ || !front_->has_front()) fop = BVHCD_FRONT_GENERATE;
    else if (front_cycle_ && k == 0) fop = BVHCD_FRONT_UPDATE;
    else if (front_cycle_ && k == front_cycle_ - 1) fop = BVHCD_FRONT_REORDER;
    else fop = BVHCD_FRONT_KEEP;
    st = front_->maintain(fop, s);
    if (st != BVHCD_OK) return st;
    if (fop == BVHCD_FRONT_GENERATE) {
        st = on_front_generated(s);
        if (st != BVHCD_OK) return st;
    } else {
        since_gen_++;
    }
    if (bvh_op_run) *bvh_op_run = first ? 2 : tag;  // the reference's opt tag: 0 refit, 1 restructure, 2 build
    if (front_op_run) *front_op_run = (int32_t)fop;
    if (fop == BVHCD_FRONT_GENERATE) regen_pending_ = false;
    if (frame_no % decide_every_ == 0) return decide_async(s);
    return BVHCD_OK;
}

}  // namespace bvhcd
