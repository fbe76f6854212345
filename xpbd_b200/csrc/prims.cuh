// Device primitives used by the broad phases: a stable LSD radix sort of
// (uint64 key, uint32 value) pairs and an exclusive scan of int32 counts.
#pragma once
#include "engine.cuh"

namespace xpbd {

// Scratch sizes (bytes) for the primitives.
size_t sort_scratch_bytes(int n);   // two ping-pong buffers
size_t scan_scratch_bytes(int n);

// Stable sort of keys[0..n) with values; result in keys/vals.  `max_bits` bounds
// the significant key bits (passes beyond the largest key are skipped on the
// device).  `scratch` must hold sort_scratch_bytes(n).
int sort_pairs_u64(uint64_t* keys, uint32_t* vals, int n, void* scratch, int max_bits,
                   cudaStream_t stream);

// out[i] = sum(in[0..i)); *total = sum(in[0..n)) (device int), n >= 0.
int exclusive_scan_i32(const int* in, int* out, int n, int* total, void* scratch,
                       cudaStream_t stream);

}  // namespace xpbd
