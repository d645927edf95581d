// sort.cuh -- stable radix sort of (key, value) pairs on the device.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fmm2d {

// Stable sort of n (key, value) pairs by bits [lo_bit, key_bits) of key
// (8-bit digits from lo_bit up).  keys_tmp / vals_tmp are scratch arrays of
// n elements; the result is left in keys / vals.
void radix_sort_pairs(uint32_t *keys, uint32_t *vals, uint32_t *keys_tmp,
                      uint32_t *vals_tmp, int64_t n, int key_bits,
                      cudaStream_t s, int lo_bit = 0);

}  // namespace fmm2d
