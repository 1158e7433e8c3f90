// prims.cuh -- device-wide scan and LSD radix sort used by the pipeline.
// The reference calls Thrust for these (thrust::exclusive_scan /
// inclusive_scan / sort_by_key, e.g. Mine/collision/lbvh/LBvhFixedDeformable.cu:216-300,
// Mine/collision/auxiliary/FlOrderLog.cu:7-12); this library carries its own.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bvhcd {

// Scratch bytes needed by scan_u32 / scan_i32 for n elements.
size_t scan_scratch_bytes(int64_t n);
// out[i] = sum(in[0..i)) (exclusive) or sum(in[0..i]) (inclusive), n
// elements; in and out may alias.  `total` (device, may be null) receives
// the sum of all n inputs.
cudaError_t scan_u32(const unsigned *in, unsigned *out, int64_t n, bool inclusive, unsigned *total,
                     void *scratch, cudaStream_t s);
cudaError_t scan_i32(const int *in, int *out, int64_t n, bool inclusive, int *total, void *scratch,
                     cudaStream_t s);
// Two exclusive scans of n elements each (scratch as for one scan of n).
cudaError_t scan2_u32(const unsigned *in_a, unsigned *out_a, const unsigned *in_b, unsigned *out_b, int64_t n,
                      void *scratch, cudaStream_t s);

// Stable LSD radix sort of (key, value) pairs; keys_alt / vals_alt are
// ping-pong buffers of the same size.  Sorts bits [0, key_bits).  The sorted
// result ends in (keys, vals) on return.
size_t sort_scratch_bytes(int64_t n);
cudaError_t radix_sort_u32(unsigned *keys, int *vals, unsigned *keys_alt, int *vals_alt, int64_t n,
                           int key_bits, void *scratch, cudaStream_t s);
cudaError_t radix_sort_u64(unsigned long long *keys, int *vals, unsigned long long *keys_alt,
                           int *vals_alt, int64_t n, int key_bits, void *scratch, cudaStream_t s);

}  // namespace bvhcd

namespace bvhcd {
// Process-wide count of kernels this library has launched.
void note_launch();
long long launch_count();
}  // namespace bvhcd
