// Device sort and scan of the plan builder: a stable LSD radix sort of
// (64-bit key, 32-bit value) pairs and a three-phase scan of int arrays.
// Both run on the caller's stream, allocate nothing and take their scratch
// from the caller (sizes from the *_tmp_bytes functions).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace yg {

enum ScanOp : int { SCAN_SUM = 0, SCAN_MIN = 1, SCAN_MAX = 2 };

// Scratch bytes of sort_pairs for n pairs.
size_t sort_pairs_tmp_bytes(long long n);
// Sorts the pairs (k0[i], v0[i]), i < n, by bits [0, end_bit) of the key,
// stably (equal keys keep their input order), 8 bits per pass, ping-ponging
// between (k0, v0) and (k1, v1).  *in_alt is set to 1 when the sorted pairs
// end in (k1, v1), else 0.  n < 2^31.
cudaError_t sort_pairs(unsigned long long* k0, unsigned long long* k1, unsigned int* v0, unsigned int* v1,
                       long long n, int end_bit, void* tmp, size_t tmp_bytes, cudaStream_t st, int* in_alt);

// Scratch bytes of scan_i32 for n elements.
size_t scan_tmp_bytes(long long n);
// out[i] = op(in[0..i]) (inclusive) or op(in[0..i-1]) with the operator's
// identity at i = 0 (exclusive); in == out is allowed.  n < 2^31.
cudaError_t scan_i32(const int* in, int* out, long long n, int op, bool exclusive, void* tmp, size_t tmp_bytes,
                     cudaStream_t st);

}  // namespace yg
