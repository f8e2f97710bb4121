// Device primitives written for this library: exclusive scan, stable LSD radix sort,
// segmented row sort and small reductions.  All are stream-ordered on the given stream.
#pragma once

#include "pb_common.cuh"

namespace pb {

// out[0..n] = exclusive prefix sums of in[0..n); out[n] = total.  in and out may alias.
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, cudaStream_t s);

// Stable LSD radix sort of (key, value) pairs on key bits [begin_bit, end_bit).  Sorted data
// ends in (keys, vals) or (keys_alt, vals_alt); the return value says which (true = alt).
// vals may be null (keys only).
bool radix_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, int64_t n,
                          int begin_bit, int end_bit, cudaStream_t s);
bool radix_sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, int64_t n,
                          int begin_bit, int end_bit, cudaStream_t s);

// Sorts every row r of a CSR (off[r]..off[r+1]) ascending by key, carrying an optional
// payload.  Keys within a row are distinct.  key_bits bounds the key values (< 2^key_bits).
void segmented_sort_rows(const uint32_t* off, int64_t nrows, uint32_t* keys, uint32_t* vals, int key_bits,
                         uint32_t max_row, cudaStream_t s);

// Sum / max reductions into a single device value (result written to *out, host-visible
// after stream sync).
void reduce_max_u32(const uint32_t* in, int64_t n, uint32_t* out_dev, cudaStream_t s);

// ids[0..count) of i in [0,n) with pred(flags[i]) — flags are uint8; returns via device count.
void compact_flags(const uint8_t* flags, int64_t n, uint32_t* ids_out, uint32_t* count_dev, cudaStream_t s);

}  // namespace pb
