// Device-side rank / search primitives over the layout in device_layout.hpp.
#pragma once

#include <cstdint>

#include "device_layout.hpp"

namespace sbwt {

// One 256-bit read-only load (a single sector request on sm_100).
__device__ __forceinline__ Block load_block(const Block *p) {
  Block b;
  asm("ld.global.nc.v4.u64 {%0,%1,%2,%3}, [%4];"
               : "=l"(b.w0), "=l"(b.w1), "=l"(b.w2), "=l"(b.w3)
               : "l"(p));
  return b;
}

// L2 eviction-priority policies (createpolicy, sm_80+) for loads that give
// one: evict_last keeps a small working set that every step hits resident in
// L2 while large random or streaming traffic passes through; evict_first
// marks lines that are read once (random lookups in a table much larger
// than L2).
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// load_block with an L2 eviction policy and no L1 allocation (random sectors
// see no L1 reuse).
__device__ __forceinline__ Block load_block_hint(const Block *p, uint64_t policy) {
  Block b;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u64 {%0,%1,%2,%3}, [%4], %5;"
      : "=l"(b.w0), "=l"(b.w1), "=l"(b.w2), "=l"(b.w3)
      : "l"(p), "l"(policy));
  return b;
}

__device__ __forceinline__ unsigned long long low_mask(uint32_t t) {
  // bits [0, t) set, t in [0, 64]
  return t >= 64 ? ~0ULL : ((1ULL << t) - 1ULL);
}

__device__ __forceinline__ uint32_t clamp64(int t) {
  return t <= 0 ? 0u : (t >= 64 ? 64u : (uint32_t)t);
}

// Payload word of in-block offset q (q in [0, 192)).
__device__ __forceinline__ unsigned long long block_word(const Block &b, uint32_t q) {
  const uint32_t wi = q >> 6;
  return wi == 0 ? b.w0 : (wi == 1 ? b.w1 : b.w2);
}

// Ones of the block strictly before in-block offset q (q in [0, 192)),
// including the block's 32-bit count relative to its superchunk.
__device__ __forceinline__ uint64_t block_rank(const Block &b, uint32_t q) {
  const uint32_t hi = (uint32_t)(b.w3 >> 32);
  const uint32_t sub = (hi >> (8 * (q >> 6))) & 0xFFu;  // 0 for the first word
  return (uint32_t)b.w3 + sub +
         (uint32_t)__popcll(block_word(b, q) & ((1ULL << (q & 63)) - 1ULL));
}

__device__ __forceinline__ bool block_bit(const Block &b, uint32_t q) {
  return (block_word(b, q) >> (q & 63)) & 1ULL;
}

// Block of position i.  Indexes are < 2^37 (checked when an index is built),
// so i / 192 = (i >> 6) / 3 is a 32-bit division by a constant.
__device__ __forceinline__ uint64_t block_of(uint64_t i) {
  return (uint64_t)((uint32_t)(i >> 6) / 3u);
}

// Hash of a k-mer key: the SplitMix64 finalizer (Steele, Lea, Flood 2014).
// The k-mer table takes its bucket from the low bits, the k-mer filter its
// word from the high bits and its four bit positions from bits 0..23.
__device__ __forceinline__ uint64_t kmer_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// First slot of a key's probe sequence in the k-mer table (an even slot, so
// that one 32-byte sector holds the first two slots probed), from its hash.
__device__ __forceinline__ uint64_t kmer_table_slot(uint64_t z, uint64_t mask) {
  return z & mask & ~1ULL;
}

__device__ __forceinline__ uint64_t kmer_table_bucket(uint64_t key, uint64_t mask) {
  return kmer_table_slot(kmer_mix(key), mask);
}

// k-mer filter (a blocked Bloom filter with one 64-bit word per key): the
// word of a hash (multiply-shift range reduction of its high bits) and the
// four bits the key sets in it.  A key is absent when any of its bits is
// clear; a key whose bits are all set may be present (false positives at
// about 1.5 % with 10 bits per key).
__device__ __forceinline__ uint64_t kmer_filter_word(uint64_t z, uint64_t n_words) {
  return __umul64hi(z, n_words);
}
__device__ __forceinline__ uint64_t kmer_filter_bits(uint64_t z) {
  return (1ULL << (z & 63)) | (1ULL << ((z >> 6) & 63)) | (1ULL << ((z >> 12) & 63)) |
         (1ULL << ((z >> 18) & 63));
}

// rank_c(i): ones of vector c in [0, i), i in [0, N].
__device__ __forceinline__ uint64_t rank_full(const SbwtView &s, uint32_t c,
                                              uint64_t i) {
  const uint64_t b = block_of(i);
  const Block blk = load_block(s.blocks[c] + b);
  return s.l0[c][b >> kSuperchunkShift] +
         block_rank(blk, (uint32_t)(i - b * kBlockBits));
}

__device__ __forceinline__ void presearch_get(const SbwtView &s, uint32_t level,
                                              uint64_t x, uint64_t &l,
                                              uint64_t &r) {
  const uint64_t e = presearch_level_offset(level) + x;
  if (!s.wide) {
    uint64_t v = __ldg(s.presearch + e);
    l = v >> 32;
    r = v & 0xFFFFFFFFULL;
  } else {
    ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2 *>(s.presearch) + e);
    l = v.x;
    r = v.y;
  }
}

// One backward-search step on [l, r] with char c
// (src/IndexSearcher/IndexSearcher.cuh:52-54 of the reference); both rank
// blocks are loaded before either is used, and a shared block is loaded once.
__device__ __forceinline__ void sbwt_step(const SbwtView &s, uint32_t c,
                                          uint64_t &l, uint64_t &r) {
  const uint64_t bl = block_of(l);
  const uint64_t r1 = r + 1;
  const uint64_t br = block_of(r1);
  const Block *base = s.blocks[c];
  const Block Bl = load_block(base + bl);
  Block Br = Bl;
  if (br != bl) Br = load_block(base + br);
  const uint64_t cc = s.c_map[c];
  const uint64_t nl = cc + s.l0[c][bl >> kSuperchunkShift] +
                      block_rank(Bl, (uint32_t)(l - bl * kBlockBits));
  const uint64_t nr = cc + s.l0[c][br >> kSuperchunkShift] +
                      block_rank(Br, (uint32_t)(r1 - br * kBlockBits)) - 1;
  l = nl;
  r = nr;
}

}  // namespace sbwt
