// prims.cu -- device-wide scan (reduce / scan-of-sums / apply) and a stable
// LSD radix sort with 8-bit digits (tile histogram, scan, stable scatter with
// warp match ranking).
#include "prims.cuh"

namespace bvhcd {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

// Exclusive block scan of one value per thread (NT <= 1024); `total`
// receives the block sum.  Safe to call repeatedly in one kernel.
template <typename T, int NT>
__device__ __forceinline__ T block_excl_scan(T v, T &total) {
    __shared__ T s_w[NT / 32];
    __shared__ T s_tot;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T inc = warp_incl_scan(v);
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    if (w == 0) {
        T x = (lane < NT / 32) ? s_w[lane] : T(0);
        T xi = warp_incl_scan(x);
        if (lane < NT / 32) s_w[lane] = xi - x;
        if (lane == NT / 32 - 1) s_tot = xi;
    }
    __syncthreads();
    T r = s_w[w] + inc - v;
    total = s_tot;
    __syncthreads();
    return r;
}

// Grid barrier k (0, 1, ...) of the launch: the arrival counter (zeroed before
// the launch) reaches (k + 1) x gridDim.x.  The wait is bounded: a CTA that
// gives up raises *err and goes on (the sort's result is then not used).
__device__ __forceinline__ void coop_barrier(unsigned *bar, unsigned k, unsigned *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned goal = (k + 1u) * gridDim.x;
        unsigned v = 0;
        for (long long it = 0; it < (1ll << 26); it++) {
            asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if (v >= goal) break;
        }
        if (v < goal) atomicOr(err, 1u);
        __threadfence();
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const T *in, int64_t n, T *sums) {
    int64_t base = (int64_t)blockIdx.x * kScanTile;
    T acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + k * kScanThreads + threadIdx.x;
        if (i < n) acc += in[i];
    }
    T tot;
    block_excl_scan<T, kScanThreads>(acc, tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// single block: exclusive scan of the tile sums in place, total to *total
template <typename T>
__global__ void __launch_bounds__(1024) k_scan_sums(T *sums, int64_t m, T *total) {
    __shared__ T s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int64_t b = 0; b < m; b += 1024) {
        int64_t i = b + threadIdx.x;
        T v = (i < m) ? sums[i] : T(0);
        T tot;
        T ex = block_excl_scan<T, 1024>(v, tot);
        T carry = s_carry;
        if (i < m) sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = s_carry;
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_tile_apply(const T *in, T *out, int64_t n,
                                                             const T *sums, bool inclusive) {
    __shared__ T s[kScanTile];
    int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + k * kScanThreads + threadIdx.x;
        s[k * kScanThreads + threadIdx.x] = (i < n) ? in[i] : T(0);
    }
    __syncthreads();
    T v[kScanItems];
    T acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = s[threadIdx.x * kScanItems + k];
        acc += v[k];
    }
    T tot;
    T ex = block_excl_scan<T, kScanThreads>(acc, tot) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        T x = v[k];
        s[threadIdx.x * kScanItems + k] = inclusive ? ex + x : ex;
        ex += x;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        int64_t i = base + k * kScanThreads + threadIdx.x;
        if (i < n) out[i] = s[k * kScanThreads + threadIdx.x];
    }
}

template <typename T>
cudaError_t scan_impl(const T *in, T *out, int64_t n, bool inclusive, T *total, void *scratch,
                      cudaStream_t s) {
    if (n <= 0) {
        if (total) return cudaMemsetAsync(total, 0, sizeof(T), s);
        return cudaSuccess;
    }
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    T *sums = reinterpret_cast<T *>(scratch);
    k_tile_sums<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, sums); note_launch();
    k_scan_sums<T><<<1, 1024, 0, s>>>(sums, tiles, total); note_launch();
    k_tile_apply<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums, inclusive); note_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------------------ sort
constexpr int kSortThreads = 256;
constexpr int kSortRounds = 8;
constexpr int kSortTile = kSortThreads * kSortRounds;

template <typename K>
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const K *keys, int64_t n, int shift,
                                                            unsigned *hist, int64_t ntiles) {
    __shared__ unsigned s_h[256];
    s_h[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll
    for (int r = 0; r < kSortRounds; r++) {
        int64_t i = base + r * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&s_h[(unsigned)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = s_h[threadIdx.x];
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const K *keys, const int *vals,
                                                               K *okeys, int *ovals, int64_t n,
                                                               int shift, const unsigned *hist,
                                                               int64_t ntiles) {
    __shared__ unsigned s_run[256];
    __shared__ unsigned s_w[kSortThreads / 32][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    s_run[threadIdx.x] = hist[(int64_t)threadIdx.x * ntiles + blockIdx.x];
    int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kSortRounds; r++) {
#pragma unroll
        for (int q = 0; q < kSortThreads / 32; q++) s_w[q][threadIdx.x] = 0;
        __syncthreads();
        int64_t i = base + r * kSortThreads + threadIdx.x;
        bool valid = i < n;
        K key = valid ? keys[i] : K(0);
        int val = valid ? vals[i] : 0;
        unsigned d = valid ? ((unsigned)(key >> shift) & 255u) : 256u;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        unsigned lrank = __popc(peers & lt);
        if (valid && lrank == 0) s_w[w][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            unsigned pos = s_run[d] + lrank;
            for (int q = 0; q < w; q++) pos += s_w[q][d];
            okeys[pos] = key;
            ovals[pos] = val;
        }
        __syncthreads();
        unsigned add = 0;
#pragma unroll
        for (int q = 0; q < kSortThreads / 32; q++) add += s_w[q][threadIdx.x];
        s_run[threadIdx.x] += add;
        __syncthreads();
    }
}

// All passes in one cooperative launch (one CTA per SM, every CTA resident):
// CTA b owns the b-th slice of the keys; per pass it counts its slice's
// digits, a grid barrier, then every CTA reads all slices' counts (the
// digit's global offset plus the counts of the slices before its own), ranks
// its keys stably (rounds of 1024 in index order, warp match ranks, per-warp
// counts) and scatters them; a grid barrier ends the pass.  No look-back and
// no launch per step: 2 barriers per pass.
constexpr int kCoopThreads = 1024;
constexpr int kCoopWarps = kCoopThreads / 32;

__global__ void __launch_bounds__(kCoopThreads, 1) k_sort_coop(unsigned *keys, int *vals, unsigned *keys_alt,
                                                                int *vals_alt, int n, int passes,
                                                                unsigned *counts, unsigned *bar, unsigned *err) {
    __shared__ unsigned s_cnt[256], s_base[256], s_run[256];
    __shared__ unsigned short s_w[kCoopWarps][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int per = (n + (int)gridDim.x - 1) / (int)gridDim.x;
    const int lo = min(n, (int)blockIdx.x * per), hi = min(n, lo + per);
    unsigned *ks = keys, *kd = keys_alt;
    int *vs = vals, *vd = vals_alt;
    unsigned k = 0;  // barriers passed
    for (int p = 0; p < passes; p++, ks = (p & 1) ? keys_alt : keys, kd = (p & 1) ? keys : keys_alt,
             vs = (p & 1) ? vals_alt : vals, vd = (p & 1) ? vals : vals_alt) {
        const int shift = 8 * p;
        if (threadIdx.x < 256) s_cnt[threadIdx.x] = 0u;
        __syncthreads();
        for (int i = lo + threadIdx.x; i < hi; i += kCoopThreads) atomicAdd(&s_cnt[(__ldcg(ks + i) >> shift) & 255u], 1u);
        __syncthreads();
        if (threadIdx.x < 256) __stcg(counts + (size_t)blockIdx.x * 256 + threadIdx.x, s_cnt[threadIdx.x]);
        coop_barrier(bar, k++, err);
        // digit d: its global offset (all slices' counts of smaller digits)
        // and the counts of the slices before this one; four threads per
        // digit, each over every fourth slice
        if (threadIdx.x < 256) {
            s_cnt[threadIdx.x] = 0u;
            s_run[threadIdx.x] = 0u;
        }
        __syncthreads();
        {
            const unsigned d = threadIdx.x & 255u;
            unsigned tot = 0, before = 0;
#pragma unroll 8
            for (unsigned b = threadIdx.x >> 8; b < gridDim.x; b += kCoopThreads / 256) {
                const unsigned c = __ldcg(counts + (size_t)b * 256 + d);
                tot += c;
                before += b < blockIdx.x ? c : 0u;
            }
            atomicAdd(&s_cnt[d], tot);
            atomicAdd(&s_run[d], before);
        }
        __syncthreads();
        if (threadIdx.x < 32) {  // exclusive scan of the 256 digit totals by one warp
            unsigned v[8], acc = 0;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                v[j] = s_cnt[lane * 8 + j];
                acc += v[j];
            }
            unsigned incl = acc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned u = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += u;
            }
            unsigned ex = incl - acc;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                s_base[lane * 8 + j] = ex;
                ex += v[j];
            }
        }
        __syncthreads();
        if (threadIdx.x < 256) s_run[threadIdx.x] += s_base[threadIdx.x];
        // stable ranks, 1024 keys per round in index order
        for (int r0 = lo; r0 < hi; r0 += kCoopThreads) {
            for (int x = threadIdx.x; x < kCoopWarps * 256; x += kCoopThreads) (&s_w[0][0])[x] = 0;
            __syncthreads();
            const int i = r0 + threadIdx.x;
            const bool valid = i < hi;
            const unsigned key = valid ? __ldcg(ks + i) : 0u;
            const int val = valid ? __ldcg(vs + i) : 0;
            const unsigned d = valid ? ((key >> shift) & 255u) : 256u;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const unsigned lrank = __popc(peers & lt);
            if (valid && lrank == 0) s_w[w][d] = (unsigned short)__popc(peers);
            __syncthreads();
            if (valid) {
                unsigned pos = s_run[d] + lrank;
                for (int q = 0; q < w; q++) pos += s_w[q][d];
                kd[pos] = key;
                vd[pos] = val;
            }
            __syncthreads();
            if (threadIdx.x < 256) {
                unsigned add = 0;
#pragma unroll 8
                for (int q = 0; q < kCoopWarps; q++) add += s_w[q][threadIdx.x];
                s_run[threadIdx.x] += add;
            }
            __syncthreads();  // s_w is cleared by the next round
        }
        coop_barrier(bar, k++, err);
    }
}

template <typename K>
cudaError_t sort_impl(K *keys, int *vals, K *keys_alt, int *vals_alt, int64_t n, int key_bits,
                      void *scratch, cudaStream_t s) {
    if (n <= 1) return cudaSuccess;
    int64_t ntiles = (n + kSortTile - 1) / kSortTile;
    unsigned *hist = reinterpret_cast<unsigned *>(scratch);
    void *scan_scratch = hist + 256 * ntiles + 64;
    int passes = (key_bits + 7) / 8;
    K *ks = keys, *kd = keys_alt;
    int *vs = vals, *vd = vals_alt;
    for (int p = 0; p < passes; p++) {
        int shift = 8 * p;
        k_sort_hist<K><<<(unsigned)ntiles, kSortThreads, 0, s>>>(ks, n, shift, hist, ntiles); note_launch();
        cudaError_t e = scan_impl<unsigned>(hist, hist, 256 * ntiles, false, nullptr, scan_scratch, s);
        if (e != cudaSuccess) return e;
        k_sort_scatter<K><<<(unsigned)ntiles, kSortThreads, 0, s>>>(ks, vs, kd, vd, n, shift, hist,
                                                                    ntiles); note_launch();
        K *tk = ks; ks = kd; kd = tk;
        int *tv = vs; vs = vd; vd = tv;
    }
    if (ks != keys) {
        cudaMemcpyAsync(keys, ks, sizeof(K) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(vals, vs, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

// The cooperative sort of 32-bit keys when every CTA fits at once and the
// scratch holds the per-slice counts (n at least 1024 keys per SM, so each
// slice is at least one round); false: use the launch-per-step sort.  Not
// inside a stream capture.
bool sort_coop_u32(unsigned *keys, int *vals, unsigned *keys_alt, int *vals_alt, int64_t n, int key_bits,
                   void *scratch, size_t scratch_bytes, cudaStream_t s, cudaError_t *err_out) {
    static int sms = -1;
    if (sms < 0) {
        int dev = 0, coop = 0, nb = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_sort_coop, kCoopThreads, 0);
        if (!coop || nb < 1) sms = 0;
    }
    if (sms <= 0 || n < (int64_t)sms * kCoopThreads || n > INT32_MAX) return false;
    if ((size_t)sms * 256 * sizeof(unsigned) + 256 > scratch_bytes) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
    unsigned *counts = reinterpret_cast<unsigned *>(scratch);
    unsigned *bar = counts + (size_t)sms * 256;  // barrier counter, then the timeout flag
    cudaError_t e = cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s);
    if (e == cudaSuccess) {
        int nn = (int)n, passes = (key_bits + 7) / 8;
        unsigned *errp = bar + 1;
        void *args[] = {&keys, &vals, &keys_alt, &vals_alt, &nn, &passes, &counts, &bar, &errp};
        e = cudaLaunchCooperativeKernel((const void *)k_sort_coop, dim3(sms), dim3(kCoopThreads), args, 0, s);
        note_launch();
        if (e == cudaSuccess && (passes & 1)) {
            e = cudaMemcpyAsync(keys, keys_alt, sizeof(unsigned) * (size_t)n, cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(vals, vals_alt, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        }
    }
    *err_out = e;
    return true;
}

// One or two scans in one cooperative launch: every CTA sums its tiles
// (2048 values), a grid barrier, then every CTA adds the sums of the tiles
// before its own (one load per thread and a block reduction) and writes its
// tiles' scan.  Replaces the three launches of the tile-sum scan.
struct CoopScan {
    const unsigned *in;
    unsigned *out;
    int64_t n;
    unsigned *total;  // device, may be null
    int inclusive;
    unsigned tiles;   // ceil(n / kScanTile)
};

template <int NT>
__device__ __forceinline__ unsigned block_sum(unsigned v) {
    __shared__ unsigned s_w[NT / 32];
    v = warp_incl_scan(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 31) s_w[w] = v;
    __syncthreads();
    unsigned t = 0;
#pragma unroll
    for (int q = 0; q < NT / 32; q++) t += s_w[q];
    __syncthreads();
    return t;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_coop(CoopScan a, CoopScan b, unsigned *sums, unsigned *bar,
                                                             unsigned *err) {
    const unsigned ntot = a.tiles + b.tiles;
    for (unsigned t = blockIdx.x; t < ntot; t += gridDim.x) {
        const CoopScan &j = t < a.tiles ? a : b;
        const int64_t base = (int64_t)(t < a.tiles ? t : t - a.tiles) * kScanTile;
        unsigned acc = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            const int64_t i = base + k * kScanThreads + threadIdx.x;
            if (i < j.n) acc += j.in[i];
        }
        acc = block_sum<kScanThreads>(acc);
        if (threadIdx.x == 0) __stcg(sums + t, acc);
    }
    coop_barrier(bar, 0u, err);
    for (unsigned t = blockIdx.x; t < ntot; t += gridDim.x) {
        const bool first = t < a.tiles;
        const CoopScan &j = first ? a : b;
        const unsigned t0 = first ? 0u : a.tiles, lt = t - t0;
        // the sums of this job's tiles before this one
        unsigned before = 0;
        for (unsigned q = threadIdx.x; q < lt; q += kScanThreads) before += __ldcg(sums + t0 + q);
        before = block_sum<kScanThreads>(before);
        const int64_t base = (int64_t)lt * kScanTile;
        __shared__ unsigned sv[kScanTile];
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            const int64_t i = base + k * kScanThreads + threadIdx.x;
            sv[k * kScanThreads + threadIdx.x] = i < j.n ? j.in[i] : 0u;
        }
        __syncthreads();
        unsigned v[kScanItems], acc = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            v[k] = sv[threadIdx.x * kScanItems + k];
            acc += v[k];
        }
        unsigned tot;
        unsigned ex = block_excl_scan<unsigned, kScanThreads>(acc, tot) + before;
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            sv[threadIdx.x * kScanItems + k] = j.inclusive ? ex + v[k] : ex;
            ex += v[k];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            const int64_t i = base + k * kScanThreads + threadIdx.x;
            if (i < j.n) j.out[i] = sv[k * kScanThreads + threadIdx.x];
        }
        if (threadIdx.x == 0 && j.total && lt + 1 == j.tiles) *j.total = before + tot;
        __syncthreads();  // sv is the next tile's
    }
}

// The cooperative form of one or two scans when it applies (not inside a
// stream capture; every CTA resident; the scratch of a scan of the longer
// input holds both jobs' tile sums); false: use the three-launch form.
bool scan_coop(const CoopScan &a, const CoopScan &b, void *scratch, size_t scratch_bytes, cudaStream_t s,
               cudaError_t *err_out) {
    static int resident = -1;
    if (resident < 0) {
        int dev = 0, coop = 0, nb = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_scan_coop, kScanThreads, 0);
        resident = coop ? nb * sms : 0;
    }
    const unsigned ntot = a.tiles + b.tiles;
    if (resident <= 0 || ntot < 2) return false;
    if ((size_t)ntot * sizeof(unsigned) + 16 > scratch_bytes) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return false;
    unsigned *sums = reinterpret_cast<unsigned *>(scratch);
    unsigned *bar = sums + ntot;  // barrier counter, then the timeout flag
    cudaError_t e = cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s);
    if (e == cudaSuccess) {
        CoopScan ja = a, jb = b;
        unsigned *errp = bar + 1;
        void *args[] = {&ja, &jb, &sums, &bar, &errp};
        const unsigned grid = ntot < (unsigned)resident ? ntot : (unsigned)resident;
        e = cudaLaunchCooperativeKernel((const void *)k_scan_coop, dim3(grid), dim3(kScanThreads), args, 0, s);
        note_launch();
    }
    *err_out = e;
    return true;
}

inline CoopScan coop_job(const unsigned *in, unsigned *out, int64_t n, bool inclusive, unsigned *total) {
    return CoopScan{in, out, n, total, inclusive ? 1 : 0, (unsigned)((n + kScanTile - 1) / kScanTile)};
}

}  // namespace

size_t scan_scratch_bytes(int64_t n) {
    int64_t tiles = (n + kScanTile - 1) / kScanTile + 1;
    return (size_t)tiles * 8 + 256;
}

cudaError_t scan_u32(const unsigned *in, unsigned *out, int64_t n, bool inclusive, unsigned *total,
                     void *scratch, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    if (n > 0 && n <= INT32_MAX &&
        scan_coop(coop_job(in, out, n, inclusive, total), coop_job(nullptr, nullptr, 0, false, nullptr), scratch,
                  scan_scratch_bytes(n), s, &e))
        return e;
    return scan_impl<unsigned>(in, out, n, inclusive, total, scratch, s);
}
// (two's complement: the sums of int32 values are those of their bit patterns)
cudaError_t scan_i32(const int *in, int *out, int64_t n, bool inclusive, int *total, void *scratch,
                     cudaStream_t s) {
    return scan_u32(reinterpret_cast<const unsigned *>(in), reinterpret_cast<unsigned *>(out), n, inclusive,
                    reinterpret_cast<unsigned *>(total), scratch, s);
}
cudaError_t scan2_u32(const unsigned *in_a, unsigned *out_a, const unsigned *in_b, unsigned *out_b, int64_t n,
                      void *scratch, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    if (n > 0 && n <= INT32_MAX &&
        scan_coop(coop_job(in_a, out_a, n, false, nullptr), coop_job(in_b, out_b, n, false, nullptr), scratch,
                  scan_scratch_bytes(n), s, &e))
        return e;
    e = scan_impl<unsigned>(in_a, out_a, n, false, nullptr, scratch, s);
    if (e == cudaSuccess) e = scan_impl<unsigned>(in_b, out_b, n, false, nullptr, scratch, s);
    return e;
}

size_t sort_scratch_bytes(int64_t n) {
    int64_t ntiles = (n + kSortTile - 1) / kSortTile + 1;
    return (size_t)(256 * ntiles + 64) * 4 + scan_scratch_bytes(256 * ntiles) + 256;
}

cudaError_t radix_sort_u32(unsigned *keys, int *vals, unsigned *keys_alt, int *vals_alt, int64_t n,
                           int key_bits, void *scratch, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    if (sort_coop_u32(keys, vals, keys_alt, vals_alt, n, key_bits, scratch, sort_scratch_bytes(n), s, &e)) return e;
    return sort_impl<unsigned>(keys, vals, keys_alt, vals_alt, n, key_bits, scratch, s);
}
cudaError_t radix_sort_u64(unsigned long long *keys, int *vals, unsigned long long *keys_alt,
                           int *vals_alt, int64_t n, int key_bits, void *scratch, cudaStream_t s) {
    return sort_impl<unsigned long long>(keys, vals, keys_alt, vals_alt, n, key_bits, scratch, s);
}

}  // namespace bvhcd
