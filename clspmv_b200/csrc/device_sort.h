// Device sort and scan building blocks (sort_device.cu), shared by the device COO sort
// and the device layout builds (layout_device.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace csp {

// Exclusive scan of a[0, n) in place on the stream.
int device_exclusive_scan(unsigned* a, size_t n, cudaStream_t st);

// Stable LSD radix sort of n 64-bit keys with 32-bit payloads over the low `bits` bits;
// k0/v0 hold the input, k1/v1 are scratch of the same sizes, and *kres/*vres receive
// the buffers that hold the result.
int device_radix_sort_pairs(uint64_t* k0, uint64_t* k1, unsigned* v0, unsigned* v1, long long n, int bits,
                            cudaStream_t st, uint64_t** kres, unsigned** vres);

}  // namespace csp
