// Device layout of one SBWT bitvector for rank queries ("rank blocks").
//
// The reference keeps each A/C/G/T bitvector plus a separate Poppy index
// (layer_0 per 2^32 bits, layer_1_2 per 1024 bits: src/Poppy/Poppy.h:19-27,
// rank in src/UtilityKernels/Rank.cuh:26-65), so one rank reads a 256-bit basic
// block of bits and an 8-byte layer_1_2 entry from another line.  Here the
// counts and the bits share one 32-byte DRAM sector, so a rank is ONE sector
// and a handful of instructions (one masked popcount):
//
//   block b (32 bytes, 32-byte aligned) covers positions [192 b, 192 b + 192):
//     w0, w1, w2 = payload bits 0..63, 64..127, 128..191
//     w3 = ones before the block, relative to its superchunk (bits 0..31)
//          | ones in w0 << 40 | ones in w0 and w1 << 48
//   superchunk s = blocks [2^24 s, 2^24 (s+1)) (3.2e9 positions);
//   l0[s] = ones before superchunk s (u64).
// There are floor(N / 192) + 1 blocks, so rank(v, N) (reached from an
// interval that ends at the last node) is defined and equals the total.
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#define SBWT_HD
#else
#define SBWT_HD __host__ __device__
#endif

namespace sbwt {

constexpr uint32_t kBlockBits = 192;
constexpr uint32_t kSuperchunkShift = 24;

struct Block {
  unsigned long long w0, w1, w2, w3;
};

// Device view of the SBWT used by the search kernels.
struct SbwtView {
  const Block *blocks[4];
  const uint64_t *l0[4];
  // the same arrays addressed arithmetically (vector c at base + c * stride),
  // so a per-lane char does not index a parameter array
  const Block *blocks0;
  uint64_t block_stride;  // in blocks
  const uint64_t *l00;
  uint64_t l0_stride;     // in entries
  uint64_t c_map[5];
  const uint64_t *presearch;  // pyramid of levels 1..presearch_max
  const uint64_t *suffix_group_starts;  // N bits or nullptr
  const uint64_t *key_marks;            // N bits or nullptr
  const uint64_t *kmer_table;  // (key, node) slots, or nullptr
  uint64_t kmer_table_mask;    // slots - 1
  const uint64_t *kmer_filter; // blocked Bloom filter of the table's keys, or nullptr
  uint64_t filter_words;       // 64-bit words of kmer_filter
  uint64_t num_bits;
  uint32_t k;
  uint32_t p;      // presearch depth used by this call
  uint32_t wide;   // presearch entries are (u64 l, u64 r) pairs
};

// Offset of presearch level j (1-based) in the pyramid, in entries.
SBWT_HD inline uint64_t presearch_level_offset(uint32_t j) {
  return ((1ULL << (2 * j)) - 4ULL) / 3ULL;
}

}  // namespace sbwt
