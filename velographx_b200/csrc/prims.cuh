// Device primitives used by the graph and BFS kernels: stable LSD radix sort of
// 64-bit keys (optionally with 32-bit values), exclusive scans, and a scratch
// arena.  All launches are stream-ordered and allocate only through Scratch.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace vxh {

// Grow-only device scratch buffer.  Reuse across calls on one stream.
struct Scratch {
  void* ptr = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes);  // 0 on success, negative on allocation failure
  void release();
  ~Scratch() { release(); }
};

// Sort (keys, vals) ascending by the low `key_bits` bits of the keys; stable.
// keys/vals are double-buffered with keys_alt/vals_alt (same sizes).  On
// return *in_alt says whether the sorted data ended in the *_alt buffers.
// vals may be null (keys-only sort).
int radix_sort_u64(uint64_t* keys, uint64_t* keys_alt, uint32_t* vals, uint32_t* vals_alt, size_t n,
                   int key_bits, bool* in_alt, Scratch& scratch, cudaStream_t s);

// Scratch bytes radix_sort_u64 needs for n items.
size_t radix_sort_scratch_bytes(size_t n);

// out[i] = sum(in[0..i)); optionally writes the grand total to *total_dev.
int scan_exclusive_u32_to_u64(const uint32_t* in, uint64_t* out, size_t n, uint64_t* total_dev,
                              Scratch& scratch, cudaStream_t s);
int scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total_dev,
                       Scratch& scratch, cudaStream_t s);
size_t scan_scratch_bytes(size_t n);

// Number of SMs of the current device (cached).
int sm_count();

}  // namespace vxh
