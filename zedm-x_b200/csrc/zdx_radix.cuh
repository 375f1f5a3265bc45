// zdx_radix.cuh -- stable LSD radix sort of (uint32 key, int32 value) pairs on the device.
//
// Used for the cell binning of the broad phase (sort particles by hashed cell key) and for the
// transposed pair index of the force scatter (sort pair ids by their second particle).  Stability is
// what makes the scatter deterministic: ties keep the input order.  8-bit digits, one pass per digit
// that can be non-zero; each pass = per-tile digit histogram, one exclusive scan over (digit, tile),
// and a scatter that ranks equal digits inside a tile in input order (warp match + per-warp counts).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace zdx {

// Scratch bytes for sorting n elements (histograms).
size_t radix_scratch_bytes(int64_t n);
// Sorts (keys, vals) of length n; key_bits = number of low key bits that can be non-zero.  Results
// end in (keys, vals); kt/vt are same-size temporaries.  With n_dev, n is a capacity that sizes the
// launches and min(*n_dev, n) elements are sorted (graph-capturable: no host read of the count).
// Returns cudaSuccess or the launch error.
cudaError_t radix_sort_u32(uint32_t* keys, int32_t* vals, uint32_t* kt, int32_t* vt, int64_t n, int key_bits,
                           void* scratch, cudaStream_t s, const int64_t* n_dev = nullptr);

// Exclusive scan of counts into offsets, any size: off[0..n) and off[n] = total, n = ncap or, with
// n_dev, min(*n_dev, ncap) read on the device.  scratch: scan_scratch_bytes(ncap).
size_t scan_scratch_bytes(int64_t ncap);
// kernels one scan_offsets / radix_sort_u32 call launches (for the launch counters)
int scan_kernels(int64_t ncap);
int radix_kernels(int64_t n, int key_bits);
template <class T>
cudaError_t scan_offsets(const T* cnt, int64_t ncap, const int64_t* n_dev, int64_t* off, void* scratch, cudaStream_t s);

// Exclusive scan of n int32 counts into n+1 int64 offsets (one block, small n).
cudaError_t scan_counts_i32(const int32_t* cnt, int64_t n, int64_t* off, cudaStream_t s);

}  // namespace zdx
