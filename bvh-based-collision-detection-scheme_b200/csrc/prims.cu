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

}  // namespace

size_t scan_scratch_bytes(int64_t n) {
    int64_t tiles = (n + kScanTile - 1) / kScanTile + 1;
    return (size_t)tiles * 8 + 256;
}

cudaError_t scan_u32(const unsigned *in, unsigned *out, int64_t n, bool inclusive, unsigned *total,
                     void *scratch, cudaStream_t s) {
    return scan_impl<unsigned>(in, out, n, inclusive, total, scratch, s);
}
cudaError_t scan_i32(const int *in, int *out, int64_t n, bool inclusive, int *total, void *scratch,
                     cudaStream_t s) {
    return scan_impl<int>(in, out, n, inclusive, total, scratch, s);
}

size_t sort_scratch_bytes(int64_t n) {
    int64_t ntiles = (n + kSortTile - 1) / kSortTile + 1;
    return (size_t)(256 * ntiles + 64) * 4 + scan_scratch_bytes(256 * ntiles) + 256;
}

cudaError_t radix_sort_u32(unsigned *keys, int *vals, unsigned *keys_alt, int *vals_alt, int64_t n,
                           int key_bits, void *scratch, cudaStream_t s) {
    return sort_impl<unsigned>(keys, vals, keys_alt, vals_alt, n, key_bits, scratch, s);
}
cudaError_t radix_sort_u64(unsigned long long *keys, int *vals, unsigned long long *keys_alt,
                           int *vals_alt, int64_t n, int key_bits, void *scratch, cudaStream_t s) {
    return sort_impl<unsigned long long>(keys, vals, keys_alt, vals_alt, n, key_bits, scratch, s);
}

}  // namespace bvhcd
