// Index step on the B200: device SBWT (rank blocks + presearch pyramid),
// device SeqToBits / PositionsBuilder equivalents, and the search kernels.
//
// Reference behaviour restated (SBWT-Search, paths in its src/):
//   d_presearch            Presearcher/Presearcher.cuh:19-41
//   d_search<move_to_key>  IndexSearcher/IndexSearcher.cuh:22-72
//   CharToBits/convert_int SeqToBitsConverter/CharToBits.h:33-40,
//                          SeqToBitsConverter/ContinuousSeqToBitsConverter.cpp:91-107
//   build_positions        PositionsBuilder/PositionsBuilder.cpp:15-47
//   -1 / -2 mapping        IndexResultsPrinter/ContinuousIndexResultsPrinter.hpp:196-205
#include <cuda_runtime.h>
#include <emmintrin.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "common.hpp"
#include "formats.hpp"
#include "index_internal.hpp"
#include "rank_blocks.cuh"

namespace sbwt {

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Presearch pyramid, level j from level j-1: entry(x) for the j-char string
// x (first char in the top bits) = one step from entry(x >> 2) with char
// x & 3; level 1 = [c_map[c], c_map[c+1] - 1].  Same table as d_presearch,
// built in sum_j 4^j steps instead of p * 4^p.
__global__ void presearch_level_kernel(SbwtView s, uint64_t *pyr, uint32_t j) {
  const uint64_t n = 1ULL << (2 * j);
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < n;
       x += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t c = (uint32_t)(x & 3);
    uint64_t l, r;
    if (j == 1) {
      l = s.c_map[c];
      r = s.c_map[c + 1] - 1;
    } else {
      const uint64_t pe = presearch_level_offset(j - 1) + (x >> 2);
      if (!s.wide) {
        const uint64_t v = pyr[pe];
        l = v >> 32;
        r = v & 0xFFFFFFFFULL;
      } else {
        l = pyr[2 * pe];
        r = pyr[2 * pe + 1];
      }
      if (l <= r) sbwt_step(s, c, l, r);  // empty stays empty
    }
    const uint64_t e = presearch_level_offset(j) + x;
    if (!s.wide) {
      pyr[e] = (l << 32) | (r & 0xFFFFFFFFULL);
    } else {
      pyr[2 * e] = l;
      pyr[2 * e + 1] = r;
    }
  }
}

// ASCII -> 2-bit MSB-first words (A0 C1 G2 T3, either case) + invalid bits.
// One warp per 32 consecutive chars: coalesced byte loads, the word is
// assembled with warp reductions.  Chars at or past n pack as 0, valid.
__global__ void pack_kernel(const char *__restrict__ chars, uint64_t n,
                            uint64_t *__restrict__ packed,
                            uint32_t *__restrict__ invalid, uint64_t n_words) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warp0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = warp0; w < n_words; w += warps) {
    const uint64_t i = w * 32 + lane;
    uint32_t code = 0;
    bool bad = false;
    if (i < n) {
      const uint32_t ch = (uint8_t)chars[i];
      code = ((ch >> 1) ^ (ch >> 2)) & 3u;
      const uint32_t lower = ch | 0x20u;
      bad = !(lower == 'a' || lower == 'c' || lower == 'g' || lower == 't');
      if (bad) code = 0;
    }
    const uint32_t hi = lane < 16 ? code << (30 - 2 * lane) : 0u;
    const uint32_t lo = lane >= 16 ? code << (30 - 2 * (lane - 16)) : 0u;
    const uint32_t whi = __reduce_or_sync(0xFFFFFFFFu, hi);
    const uint32_t wlo = __reduce_or_sync(0xFFFFFFFFu, lo);
    const uint32_t inv = __ballot_sync(0xFFFFFFFFu, bad);
    if (lane == 0) {
      packed[w] = ((uint64_t)whi << 32) | wlo;
      invalid[w] = inv;
    }
  }
}

// The same packing from 16-byte loads (chars 16-byte aligned): byte-parallel
// codes and validity (SIMD byte compares).  pack_kernel's one 32-byte load
// per warp iteration left it latency-bound (0.4 TB/s on 1.7 GB of chars).
__device__ __forceinline__ void pack_4chars(uint32_t x, uint32_t &codes8, uint32_t &inv4) {
  const uint32_t lower = x | 0x20202020u;
  const uint32_t ok = __vcmpeq4(lower, 0x61616161u) | __vcmpeq4(lower, 0x63636363u) |
                      __vcmpeq4(lower, 0x67676767u) | __vcmpeq4(lower, 0x74747474u);
  const uint32_t c = ((x >> 1) ^ (x >> 2)) & 0x03030303u & ok;  // per byte: A0 C1 G2 T3
  codes8 = ((c & 0xFFu) << 6) | (((c >> 8) & 0xFFu) << 4) | (((c >> 16) & 0xFFu) << 2) |
           (c >> 24);  // first char on top
  const uint32_t bad = ~ok & 0x80808080u;
  inv4 = ((bad >> 7) & 1u) | ((bad >> 14) & 2u) | ((bad >> 21) & 4u) | ((bad >> 28) & 8u);
}

// One 64-bit word (32 chars, two 16-byte loads) per thread and two words per
// iteration, so four loads are in flight per thread.
__device__ __forceinline__ void pack_word(const char *__restrict__ chars, uint64_t n,
                                          uint64_t w, uint64_t &word, uint32_t &inv) {
  const uint64_t i0 = w * 32;
  uint32_t x[8];
  if (i0 + 32 <= n) {
    const uint4 a = __ldg(reinterpret_cast<const uint4 *>(chars + i0));
    const uint4 b = __ldg(reinterpret_cast<const uint4 *>(chars + i0 + 16));
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
  } else {  // the last word: chars past n pack as 'A' (code 0, valid)
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      x[q] = 0;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const uint64_t i = i0 + 4 * q + c;
        x[q] |= (uint32_t)(i < n ? (uint8_t)chars[i] : (uint8_t)'A') << (8 * c);
      }
    }
  }
  uint32_t hi = 0, lo = 0;
  inv = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    uint32_t c8, i4;
    pack_4chars(x[q], c8, i4);
    if (q < 4)
      hi |= c8 << (24 - 8 * q);
    else
      lo |= c8 << (24 - 8 * (q - 4));
    inv |= i4 << (4 * q);
  }
  word = ((uint64_t)hi << 32) | lo;
}

__global__ void pack16_kernel(const char *__restrict__ chars, uint64_t n,
                              uint64_t *__restrict__ packed, uint32_t *__restrict__ invalid,
                              uint64_t n_words) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n_words;
       w += 2 * step) {
    const uint64_t w2 = w + step;
    uint64_t a = 0, b = 0;
    uint32_t ia = 0, ib = 0;
    pack_word(chars, n, w, a, ia);
    if (w2 < n_words) pack_word(chars, n, w2, b, ib);
    packed[w] = a;
    invalid[w] = ia;
    if (w2 < n_words) {
      packed[w2] = b;
      invalid[w2] = ib;
    }
  }
}

// --- exclusive scan of per-read k-mer counts -> kmer_off[0..n_reads] ---------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr uint64_t kScanTile = (uint64_t)kScanThreads * kScanItems;

__device__ __forceinline__ uint64_t read_kmers(const uint64_t *ends, uint64_t r,
                                               uint64_t base, uint32_t k) {
  const uint64_t st = r ? ends[r - 1] : base;
  const uint64_t len = ends[r] - st;
  return len >= k ? len - k + 1 : 0;
}

template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *total) {
  __shared__ T warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    T s = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  const T warp_prefix = wid ? warp_sums[wid - 1] : 0;
  *total = warp_sums[kScanThreads / 32 - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

__global__ void scan_reduce_kernel(const uint64_t *ends, uint64_t n_reads,
                                   uint64_t base, uint32_t k, uint64_t n_chars,
                                   uint64_t *block_sums, uint32_t *err) {
  const uint64_t t0 = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint64_t s = 0;
  for (int i = 0; i < kScanItems; ++i)
    if (t0 + i < n_reads) {
      const uint64_t r = t0 + i;
      const uint64_t st = r ? ends[r - 1] : base;
      if (ends[r] < st || ends[r] - base > n_chars) atomicOr(err, 4u);
      s += read_kmers(ends, r, base, k);
    }
  uint64_t total;
  block_exclusive_scan<uint64_t>(s, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// A batch whose read ends failed the check (err bit 4) gets a total of 0 and
// all-zero k-mer offsets: the launches queued after the scan then do nothing
// (no host round trip is needed before them).
__global__ void scan_sums_kernel(uint64_t *block_sums, uint64_t n_blocks,
                                 uint64_t *grand_total, const uint32_t *err) {
  __shared__ uint64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint64_t b0 = 0; b0 < n_blocks; b0 += kScanThreads) {
    const uint64_t b = b0 + threadIdx.x;
    uint64_t v = b < n_blocks ? block_sums[b] : 0;
    uint64_t total;
    uint64_t ex = block_exclusive_scan<uint64_t>(v, &total);
    if (b < n_blocks) block_sums[b] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *grand_total = (*err & 4u) ? 0 : carry;
}

__global__ void scan_write_kernel(const uint64_t *ends, uint64_t n_reads,
                                  uint64_t base, uint32_t k,
                                  const uint64_t *block_sums, uint64_t *kmer_off,
                                  const uint32_t *err) {
  const uint64_t t0 = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  if (*err & 4u) {  // the same word for every thread: a uniform return
    for (int i = 0; i < kScanItems; ++i) {
      if (t0 + i < n_reads) kmer_off[t0 + i] = 0;
      if (t0 + i == n_reads - 1) kmer_off[n_reads] = 0;
    }
    return;
  }
  uint64_t v[kScanItems];
  uint64_t s = 0;
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (t0 + i < n_reads) ? read_kmers(ends, t0 + i, base, k) : 0;
    s += v[i];
  }
  uint64_t total;
  uint64_t ex = block_exclusive_scan<uint64_t>(s, &total) + block_sums[blockIdx.x];
  for (int i = 0; i < kScanItems; ++i) {
    if (t0 + i < n_reads) kmer_off[t0 + i] = ex;
    if (t0 + i == n_reads - 1) kmer_off[n_reads] = ex + v[i];
    ex += v[i];
  }
}

// --- search ------------------------------------------------------------------
__device__ __forceinline__ uint32_t char_at(const uint64_t *packed, uint64_t i) {
  return (uint32_t)((__ldg(packed + (i >> 5)) >> (62 - 2 * (i & 31))) & 3ULL);
}

// First `n` chars (n <= 32) from char i as an integer, first char on top.
__device__ __forceinline__ uint64_t chars_prefix(const uint64_t *packed, uint64_t i,
                                                 uint32_t n) {
  const uint64_t w = i >> 5;
  const uint32_t off = (uint32_t)(i & 31);
  uint64_t win = __ldg(packed + w) << (2 * off);
  if (off) win |= __ldg(packed + w + 1) >> (64 - 2 * off);
  return win >> (64 - 2 * n);
}

// Full search of the k-mer starting at char `pos`: presearch lookup of the
// first p chars, then one step per remaining char, stopping at the first
// empty interval (emptiness is preserved by every later step, so the answer
// is unchanged).  Returns the node or SBWT_NOT_FOUND.
__device__ __forceinline__ uint64_t full_search(const SbwtView &s,
                                                const uint64_t *packed,
                                                uint64_t pos) {
  uint64_t l, r;
  presearch_get(s, s.p, chars_prefix(packed, pos, s.p), l, r);
  if (l > r) return SBWT_NOT_FOUND;
  for (uint64_t i = pos + s.p; i < pos + s.k; ++i) {
    sbwt_step(s, char_at(packed, i), l, r);
    if (l > r) return SBWT_NOT_FOUND;
  }
  return l;
}

// full_search that also counts the distinct rank-block sectors it reads
// (one per step, two when l and r + 1 fall in different blocks).
__device__ __forceinline__ uint64_t full_search_counted(const SbwtView &s,
                                                        const uint64_t *packed,
                                                        uint64_t pos, uint64_t &sectors) {
  uint64_t l, r;
  presearch_get(s, s.p, chars_prefix(packed, pos, s.p), l, r);
  if (l > r) return SBWT_NOT_FOUND;
  for (uint64_t i = pos + s.p; i < pos + s.k; ++i) {
    sectors += (block_of(l) == block_of(r + 1)) ? 1 : 2;
    sbwt_step(s, char_at(packed, i), l, r);
    if (l > r) return SBWT_NOT_FOUND;
  }
  return l;
}

// Largest u <= v with suffix_group_starts[u] set (node 0, the root, always is).
__device__ __forceinline__ uint64_t group_start(const uint64_t *sg, uint64_t v) {
  uint64_t w = v >> 6;
  uint64_t m = __ldg(sg + w) & low_mask((uint32_t)(v & 63) + 1);
  while (m == 0 && w > 0) m = __ldg(sg + --w);
  if (m == 0) return 0;
  return w * 64 + 63 - __clzll(m);
}

// Successor of node v (a found k-mer x) by char c: the node of x[1..k) c, or
// SBWT_NOT_FOUND.  The edge bit lives at the first node of v's suffix group.
__device__ __forceinline__ uint64_t stream_step(const SbwtView &s, uint64_t v,
                                                uint32_t c) {
  uint64_t b = block_of(v);
  Block B = load_block(s.blocks[c] + b);
  uint32_t q = (uint32_t)(v - b * kBlockBits);
  if (!block_bit(B, q)) {
    const uint64_t u = group_start(s.suffix_group_starts, v);
    if (u == v) return SBWT_NOT_FOUND;
    const uint64_t bu = block_of(u);
    if (bu != b) {
      B = load_block(s.blocks[c] + bu);
      b = bu;
    }
    q = (uint32_t)(u - b * kBlockBits);
    if (!block_bit(B, q)) return SBWT_NOT_FOUND;
  }
  return s.c_map[c] + s.l0[c][b >> kSuperchunkShift] + block_rank(B, q);
}

// Forward walk of a found node to the next key k-mer
// (src/IndexSearcher/IndexSearcher.cuh:60-70): while the node is not a key
// k-mer, follow its first outgoing edge in A,C,G,T order.  Bounded: a node
// without an outgoing edge sets *err and returns the node unchanged.
constexpr uint32_t kMaxKeyWalk = 1u << 16;
__device__ __forceinline__ uint64_t key_walk(const SbwtView &s, uint64_t v,
                                             uint32_t *err) {
  for (uint32_t it = 0; it < kMaxKeyWalk; ++it) {
    if ((__ldg(s.key_marks + (v >> 6)) >> (v & 63)) & 1ULL) return v;
    bool moved = false;
    for (uint32_t c = 0; c < 4; ++c) {
      const uint64_t b = block_of(v);
      const Block B = load_block(s.blocks[c] + b);
      const uint32_t q = (uint32_t)(v - b * kBlockBits);
      if (block_bit(B, q)) {
        v = s.c_map[c] + s.l0[c][b >> kSuperchunkShift] + block_rank(B, q);
        moved = true;
        break;
      }
    }
    if (!moved) break;
  }
  atomicOr(err, 1u);
  return v;
}

// The reference seam: one k-mer per position, independent walks.
__global__ void __launch_bounds__(256) search_positions_kernel(
    SbwtView s, const uint64_t *__restrict__ packed, uint64_t n_chars_cap,
    const uint64_t *__restrict__ positions, uint64_t n, uint64_t *__restrict__ out,
    uint32_t move_to_key, uint32_t *err) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t pos = __ldg(positions + t);
    if (pos > n_chars_cap || n_chars_cap - pos < s.k) {  // k-mer past bit_seqs
      atomicOr(err, 2u);
      out[t] = SBWT_NOT_FOUND;
      continue;
    }
    uint64_t v = full_search(s, packed, pos);
    if (move_to_key && v != SBWT_NOT_FOUND) v = key_walk(s, v, err);
    out[t] = v;
  }
}

struct ReadsView {
  const uint64_t *packed;   // chunk chars, 2-bit packed (+1 pad word)
  const uint32_t *invalid;  // invalid-char bits, 32 per word
  const uint64_t *ends;     // exclusive read ends (absolute)
  const uint64_t *kmer_off; // n_reads + 1
  uint64_t base;            // absolute char offset of chunk char 0
  uint64_t n_reads;
  uint64_t n_kmers;
  uint64_t tile;            // k-mer slots per tile
  uint64_t n_tiles;
  uint64_t *out;
  uint64_t out_capacity;
  uint32_t probe_len;       // L of the absent-prefix probe (0 = off)
  const uint64_t *n_kmers_dev;  // if set, the k-mer total is read from here
  unsigned long long *queue;    // work-queue counter (tiles handed out), zeroed
  uint64_t n_kmers_bound;       // > every chunk position, slot and read number
  uint32_t *out32;  // walks kernel only: 32-bit results here instead of `out`
                    // (node, 0xFFFFFFFF not found, 0xFFFFFFFE invalid)
};

__device__ __forceinline__ bool invalid_at(const uint32_t *inv, uint64_t i) {
  return (__ldg(inv + (i >> 5)) >> (i & 31)) & 1u;
}

// Highest invalid char position in [a, b) (chunk-relative), or -1.
__device__ __forceinline__ int64_t last_invalid(const uint32_t *inv, uint64_t a,
                                                uint64_t b) {
  if (b <= a) return -1;
  int64_t w = (int64_t)((b - 1) >> 5);
  const int64_t wa = (int64_t)(a >> 5);
  uint32_t m = __ldg(inv + w);
  const uint32_t top = (uint32_t)((b - 1) & 31);
  if (top < 31) m &= (2u << top) - 1u;
  while (true) {
    if (w == wa) m &= ~((1u << (a & 31)) - 1u);
    if (m) return w * 32 + 31 - __clz(m);
    if (w == wa) return -1;
    m = __ldg(inv + --w);
  }
}

// 32-byte aligned chunk of a u64 array that holds word i, loaded as a block.
__device__ __forceinline__ const Block *chunk_of(const uint64_t *base, uint64_t i) {
  return reinterpret_cast<const Block *>(base + (i & ~3ULL));
}
__device__ __forceinline__ uint64_t chunk_word(const Block &b, uint64_t i) {
  const uint32_t j = (uint32_t)(i & 3);
  return j == 0 ? b.w0 : (j == 1 ? b.w1 : (j == 2 ? b.w2 : b.w3));
}

// *out = the first read r in [r0, n_reads) with ends[r] > limit (n_reads if
// none); one thread, binary search (ends are non-decreasing; the scan kernels
// check that).
__global__ void ends_upper_bound_kernel(const uint64_t *ends, uint64_t r0, uint64_t n_reads,
                                        uint64_t limit, uint64_t *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint64_t lo = r0, hi = n_reads;
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (ends[mid] > limit)
      hi = mid;
    else
      lo = mid + 1;
  }
  out[0] = lo;
  out[1] = lo > r0 ? ends[lo - 1] : limit;
}

// First read of every work tile: tile_read[t] = the read holding k-mer slot
// t * tile.  One thread per read; reads without k-mers own no tile.
__global__ void tile_reads_kernel(const uint64_t *kmer_off, uint64_t n_reads, uint64_t tile,
                                  uint64_t *tile_read) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n_reads;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a = kmer_off[r], b = kmer_off[r + 1];
    for (uint64_t t = (a + tile - 1) / tile; t * tile < b; ++t) tile_read[t] = r;
  }
}

// Fused index step over reads.
//
// Work unit = a tile of consecutive k-mer result slots.  Inside a read:
//  * a k-mer that follows a found k-mer is resolved by ONE step along the
//    successor edge of the previous node (stream step); the answer is the
//    same as a full search because a k-mer's node is unique;
//  * when a search fails at char f (the string x[pos..f] is not a suffix of
//    any node), the kernel probes the L-mer x[f-L+1..f].  If it is absent,
//    every k-mer starting in (pos, f-L+1] holds it as a prefix of its own
//    prefix x[j..f], and every prefix of a k-mer in the SBWT is a suffix of
//    some node, so all those k-mers are reported not found without a search.
//    This removes most of the full searches around sequencing errors.
//
// Every lane runs its own state machine; each loop iteration is one memory
// round trip per active lane: addresses are computed per lane, the warp
// reconverges (warp-uniform exit test) and issues the loads together, then
// ONE shared rank computation serves every mode.  Three of the modes are the
// same backward-search step (rank blocks of l and rr + 1 for the char at wi),
// so most lanes take one code path:
//   M_NEW    : the k-mer at `slot` needs its first load (stream step if the
//              previous k-mer was found, else the presearch entry);
//   M_WALK   : search walk (also the single step at a group start g);
//   M_STREAM : the step on [v, v] from the previous k-mer's node v; empty
//              means no edge at v itself, so the group scan follows;
//   M_SG     : suffix-group-start word u (bits <= ubit) below a failed stream
//              step;
//   M_PPRE   : probe, presearch entry of x[m..m+lvl);
//   M_PROBE  : probe walk up to probe_end (nothing is emitted);
//   M_HASH   : k-mer table lookup of the k-mer at `slot` (k <= 31, when the
//              index has the table): one 32-byte sector of two slots per
//              step, u = the first slot of the pair.
// Per-lane register window over the packed chars and invalid bits of a read:
// words wbase and wbase + 1, i.e. chunk positions [32 wbase, 32 wbase + 64).
// With k <= 33 every char the lane needs for the k-mer at pos (and for a probe
// started when that k-mer failed) lies in the window of wbase = pos / 32, so
// after the window moves the search reads no char from memory.
struct CharWindow {
  uint64_t w0, w1;   // packed words wbase, wbase + 1
  uint64_t inv;      // invalid bits of both words (word wbase in the low half)
  uint64_t wbase;
  __device__ __forceinline__ void init(const uint64_t *packed, const uint32_t *invalid) {
    wbase = ~1ULL;  // neither equal to nor one below any real word index
    w0 = w1 = inv = 0;
    (void)packed;
    (void)invalid;
  }
  __device__ __forceinline__ void move_to(const uint64_t *packed, const uint32_t *invalid,
                                          uint64_t pos) {
    const uint64_t wb = pos >> 5;
    if (wb == wbase) return;
    if (wb == wbase + 1) {
      w0 = w1;
      w1 = __ldg(packed + wb + 1);
      inv = (inv >> 32) | ((uint64_t)__ldg(invalid + wb + 1) << 32);
    } else {
      w0 = __ldg(packed + wb);
      w1 = __ldg(packed + wb + 1);
      inv = (uint64_t)__ldg(invalid + wb) | ((uint64_t)__ldg(invalid + wb + 1) << 32);
    }
    wbase = wb;
  }
  __device__ __forceinline__ uint32_t char_at(uint64_t i) const {
    const uint32_t off = (uint32_t)(i - 32 * wbase);
    const uint64_t w = off < 32 ? w0 : w1;
    return (uint32_t)((w >> (62 - 2 * (off & 31))) & 3ULL);
  }
  // first n chars (1 <= n <= 32) from position i, first char on top
  __device__ __forceinline__ uint64_t prefix(uint64_t i, uint32_t n) const {
    const uint32_t off = (uint32_t)(i - 32 * wbase);
    uint64_t v;
    if (off < 32) {
      v = w0 << (2 * off);
      if (off) v |= w1 >> (64 - 2 * off);
    } else {
      v = w1 << (2 * (off - 32));
    }
    return v >> (64 - 2 * n);
  }
  __device__ __forceinline__ bool invalid_at(uint64_t i) const {
    return (inv >> (uint32_t)(i - 32 * wbase)) & 1ULL;
  }
  // highest invalid position in [a, b) (b - a <= 63), or -1
  __device__ __forceinline__ int64_t last_invalid(uint64_t a, uint64_t b) const {
    if (b <= a) return -1;
    const uint32_t oa = (uint32_t)(a - 32 * wbase), ob = (uint32_t)(b - 32 * wbase);
    uint64_t m = inv & (ob >= 64 ? ~0ULL : ((1ULL << ob) - 1));
    m &= ~((1ULL << oa) - 1);
    return m ? (int64_t)(32 * wbase + 63 - __clzll(m)) : -1;
  }
};

// Lane modes: a new k-mer; the group-start scan of a failed stream step; the
// presearch of a probe; and three walks that share one step (the backward
// search step on [l, rr] with the char at wi): the walk of a k-mer search
// (also the single step of a group start), the stream step from the previous
// k-mer's node (an empty result sends the lane to the group scan), and the
// walk of a probe (its end proves k-mers absent or not; nothing is emitted).
enum : uint32_t { M_NEW = 0, M_SG = 1, M_PPRE = 2, M_HASH = 3, M_WALK = 4, M_STREAM = 5,
                  M_PROBE = 6 };
enum : uint32_t { K_NONE = 0, K_BLOCK = 1, K_PRE = 2, K_SGW = 3, K_HASH = 4 };
// SBWTs with fewer nodes than this use 32-bit node arithmetic in the search.
constexpr uint64_t kNarrowLimit = (uint64_t)kBlockBits << kSuperchunkShift;

#ifndef SBWT_SEARCH_MIN_BLOCKS
#define SBWT_SEARCH_MIN_BLOCKS 5  // 256-thread blocks per SM the register budget targets
#endif

// Index arithmetic of the search kernel: all 32-bit (nodes, chunk
// positions, k-mer slots, read numbers) when the SBWT has fewer than
// 192 * 2^24 nodes (one superchunk: no l0 table) and the batch fewer than
// 2^32 chars, else all 64-bit.
template <class I>
__device__ __forceinline__ I block_idx(I i) {
  return (I)((uint32_t)((uint64_t)i >> 6) / 3u);
}

// Per-lane register window over the packed chars and invalid bits (see
// CharWindow); index type I.
template <class I>
struct CharWin {
  uint64_t w0, w1, inv;
  I wbase;
  __device__ __forceinline__ void init() {
    wbase = (I)~(I)1;  // neither equal to nor one below any real word index
    w0 = w1 = inv = 0;
  }
  __device__ __forceinline__ void move_to(const uint64_t *packed, const uint32_t *invalid,
                                          I pos) {
    const I wb = pos >> 5;
    if (wb == wbase) return;
    if (wb == wbase + 1) {
      w0 = w1;
      w1 = __ldg(packed + wb + 1);
      inv = (inv >> 32) | ((uint64_t)__ldg(invalid + wb + 1) << 32);
    } else {
      w0 = __ldg(packed + wb);
      w1 = __ldg(packed + wb + 1);
      inv = (uint64_t)__ldg(invalid + wb) | ((uint64_t)__ldg(invalid + wb + 1) << 32);
    }
    wbase = wb;
  }
  __device__ __forceinline__ uint32_t char_at(I i) const {
    const uint32_t off = (uint32_t)(i - 32 * wbase);
    const uint64_t w = off < 32 ? w0 : w1;
    return (uint32_t)((w >> (62 - 2 * (off & 31))) & 3ULL);
  }
  __device__ __forceinline__ uint64_t prefix(I i, uint32_t n) const {
    const uint32_t off = (uint32_t)(i - 32 * wbase);
    uint64_t v;
    if (off < 32) {
      v = w0 << (2 * off);
      if (off) v |= w1 >> (64 - 2 * off);
    } else {
      v = w1 << (2 * (off - 32));
    }
    return v >> (64 - 2 * n);
  }
  __device__ __forceinline__ bool invalid_at(I i) const {
    return (inv >> (uint32_t)(i - 32 * wbase)) & 1ULL;
  }
  // 1 + highest invalid position in [a, b) (b - a <= 63), or 0
  __device__ __forceinline__ I last_invalid1(I a, I b) const {
    if (b <= a) return 0;
    const uint32_t oa = (uint32_t)(a - 32 * wbase), ob = (uint32_t)(b - 32 * wbase);
    uint64_t m = inv & (ob >= 64 ? ~0ULL : ((1ULL << ob) - 1));
    m &= ~((1ULL << oa) - 1);
    return m ? (I)(32 * wbase + 64 - __clzll(m)) : (I)0;
  }
};

template <bool STREAM, bool COUNT, bool SMALLK, class I>
__global__ void __launch_bounds__(256, SBWT_SEARCH_MIN_BLOCKS)
    search_reads_kernel(SbwtView s, ReadsView rv, const uint64_t *__restrict__ tile_read,
                        uint32_t move_to_key, uint32_t *err,
                        unsigned long long *counters) {
  constexpr I NONE = ~I(0);
  constexpr bool NARROW = sizeof(I) == 4;
  __shared__ I sh_cmap[4];
  if (threadIdx.x < 4) sh_cmap[threadIdx.x] = (I)s.c_map[threadIdx.x];
  __syncthreads();
  const uint32_t k = s.k;
  const uint32_t L = rv.probe_len;
  // presearch levels of a new k-mer and of a probe (fixed per launch)
  const uint32_t probe_lvl = min(L, s.p);
  const uint64_t pre_off = presearch_level_offset(s.p);
  const uint64_t probe_off = presearch_level_offset(max(probe_lvl, 1u));
  const uint32_t lane = threadIdx.x & 31;
  const I n_kmers = (I)(rv.n_kmers_dev ? *rv.n_kmers_dev : rv.n_kmers);
  const I tsize = (I)rv.tile;
  const I n_tiles = (n_kmers + tsize - 1) / tsize;
  const I base = (I)rv.base;
  uint64_t n_pre = 0, n_block = 0, n_sg = 0, n_probe = 0, n_iter = 0, n_lane = 0, n_known = 0,
           n_searched = 0, n_distinct = 0;
  uint64_t n_mode[6] = {0, 0, 0, 0, 0, 0};
  bool exhausted = false;  // the work queue is empty for this lane
  I slot = 0, slot_end = 0, r = 0, r_next = 0, pos = 0, skip_until = 0;
  I last_inv1 = 0;  // 1 + last invalid char position (0 = none)
  I v = NONE;       // node of the previous k-mer of this read
  I l = 0, rr = 0, u = 0;
  I wi = 0, probe_end = 0, probe_skip = 0, pu = 0;
  uint32_t mode = M_NEW, c = 0, ubit = 63;
  bool done = false;
  CharWin<I> cw;
  cw.init();
  while (true) {
    // ---- work queue (warp-collective): lanes out of k-mers take a new tile;
    // one atomic per warp hands out consecutive tiles.
    __syncwarp();
    const bool need = !exhausted && mode == M_NEW && slot >= slot_end;
    const unsigned need_mask = __ballot_sync(0xFFFFFFFFu, need);
    I new_tile = NONE;
    if (need_mask) {
      const int leader = __ffs(need_mask) - 1;
      unsigned long long qb = 0;
      if ((int)lane == leader) qb = atomicAdd(rv.queue, (unsigned long long)__popc(need_mask));
      qb = __shfl_sync(0xFFFFFFFFu, qb, leader);
      if (need) {
        const unsigned long long t = qb + __popc(need_mask & ((1u << lane) - 1u));
        if (t >= (unsigned long long)n_tiles) {
          exhausted = true;
        } else {
          new_tile = (I)t;
        }
      }
    }
    // ---- phase 1 (per lane): what to load --------------------------------
    uint32_t kind = K_NONE;
    I pa = 0, pb = 0;
    uint64_t pre_e = 0;
    I run_slot = 0, run_pos = 0;
    uint32_t run_n = 0;
    bool run_inv = false;
    if (!done) {
      if (mode == M_NEW) {
        bool ready = false;
        while (true) {
          if (slot >= slot_end) {  // next tile
            if (new_tile == NONE) {  // none this iteration
              done = exhausted;
              break;
            }
            slot = new_tile * tsize;
            new_tile = NONE;
            slot_end = min(slot + tsize, n_kmers);
            r = (I)__ldg(tile_read + slot / tsize);
            r_next = (I)__ldg(rv.kmer_off + r + 1);
            pos = (r ? (I)__ldg(rv.ends + r - 1) : base) - base +
                  (slot - (I)__ldg(rv.kmer_off + r));
            if (SMALLK) {
              cw.move_to(rv.packed, rv.invalid, pos);
              last_inv1 = cw.last_invalid1(pos, pos + k - 1);
            } else {
              last_inv1 = (I)(last_invalid(rv.invalid, pos, pos + k - 1) + 1);
            }
            v = NONE;
            skip_until = 0;
          } else if (slot == r_next) {  // next read
            do {
              r_next = (I)__ldg(rv.kmer_off + (++r) + 1);
            } while (r_next == slot);
            pos = (I)__ldg(rv.ends + r - 1) - base;
            if (SMALLK) {
              cw.move_to(rv.packed, rv.invalid, pos);
              last_inv1 = cw.last_invalid1(pos, pos + k - 1);
            } else {
              last_inv1 = (I)(last_invalid(rv.invalid, pos, pos + k - 1) + 1);
            }
            v = NONE;
            skip_until = 0;
          }
          const I newc = pos + k - 1;
          if (SMALLK) cw.move_to(rv.packed, rv.invalid, pos);
          if (SMALLK ? cw.invalid_at(newc) : invalid_at(rv.invalid, newc)) last_inv1 = newc + 1;
          const bool skip = slot < skip_until;
          if (last_inv1 <= pos && !skip) {
            ready = true;  // a k-mer to search
            break;
          }
          if (run_n) break;  // one run per iteration: this lane resumes next time
          // a run of k-mers whose results are known without a search (an
          // invalid char in each, or proven absent by the probe), up to the
          // read / tile end; the warp writes it below
          const I n = min(skip ? skip_until - slot : last_inv1 - pos, min(r_next, slot_end) - slot);
          run_inv = !skip;
          run_slot = slot;
          run_pos = pos;
          run_n = (uint32_t)n;
          if (COUNT) n_known += n;
          v = NONE;
          slot += n;
          pos += n;
          if (slot < min(r_next, slot_end)) {  // the window moved: its last invalid char
            if (SMALLK) {
              cw.move_to(rv.packed, rv.invalid, pos);
              last_inv1 = cw.last_invalid1(pos, pos + k - 1);
            } else {
              last_inv1 = (I)(last_invalid(rv.invalid, pos, pos + k - 1) + 1);
            }
          }
        }
        if (ready) {
          if (STREAM && v != NONE) {  // the stream step: one walk step on [v, v]
            l = rr = v;
            wi = pos + k - 1;
            mode = M_STREAM;
          } else if (SMALLK && s.kmer_table) {  // one k-mer table lookup
            u = (I)kmer_table_bucket(cw.prefix(pos, k), s.kmer_table_mask);
            mode = M_HASH;
          } else {
            kind = K_PRE;
            pre_e = pre_off +
                    (SMALLK ? cw.prefix(pos, s.p) : chars_prefix(rv.packed, pos, s.p));
          }
        }
      }
      if (mode >= M_WALK) {
        kind = K_BLOCK;
        c = SMALLK ? cw.char_at(wi) : char_at(rv.packed, wi);
        pa = l;
        pb = rr + 1;
      } else if (mode == M_SG) {
        kind = K_SGW;
      } else if (mode == M_HASH) {
        kind = K_HASH;
      } else if (mode == M_PPRE) {  // pu = probe start m
        kind = K_PRE;
        pre_e = probe_off +
                (SMALLK ? cw.prefix(pu, probe_lvl) : chars_prefix(rv.packed, pu, probe_lvl));
      }
    }
    // ---- known runs (converged): the warp writes each lane's run, 32 slots
    // per store; a probe-proven run is -1 except where a k-mer holds an
    // invalid char (-2 takes priority)
    for (unsigned runs = __ballot_sync(0xFFFFFFFFu, run_n != 0); runs; runs &= runs - 1) {
      const int q = __ffs(runs) - 1;
      const I q_slot = __shfl_sync(0xFFFFFFFFu, run_slot, q);
      const I q_pos = __shfl_sync(0xFFFFFFFFu, run_pos, q);
      const uint32_t q_n = __shfl_sync(0xFFFFFFFFu, run_n, q);
      const bool q_inv = __shfl_sync(0xFFFFFFFFu, (uint32_t)run_inv, q) != 0;
      for (uint32_t j = lane; j < q_n; j += 32) {
        const I p = q_pos + (I)j;
        const bool inv = q_inv || last_invalid(rv.invalid, p, p + k) >= 0;
        if (q_slot + j < rv.out_capacity)
          __stcs(rv.out + q_slot + j, (unsigned long long)(inv ? SBWT_INVALID : SBWT_NOT_FOUND));
      }
    }
    if (__all_sync(0xFFFFFFFFu, done)) break;
    // ---- phase 2 (converged): the loads ------------------------------------
    const I ba = block_idx(pa), bb = block_idx(pb);
    const Block *bc = s.blocks0 + (uint64_t)c * s.block_stride;
    const Block *addrA = nullptr, *addrB = nullptr;
    if (kind == K_BLOCK) {
      addrA = bc + ba;
      if (bb != ba) addrB = bc + bb;
    } else if (kind == K_PRE) {
      addrA = s.wide ? chunk_of(s.presearch, 2 * pre_e) : chunk_of(s.presearch, pre_e);
    } else if (kind == K_HASH) {
      addrA = reinterpret_cast<const Block *>(s.kmer_table + 2 * (uint64_t)u);
    } else if (kind == K_SGW) {
      addrA = chunk_of(s.suffix_group_starts, (uint64_t)u);
    }
    Block A = Block{0, 0, 0, 0}, B;
    if (addrA) A = load_block(addrA);
    B = A;
    if (addrB) B = load_block(addrB);
    if (COUNT) {
      n_pre += kind == K_PRE || kind == K_HASH;
      n_block += (kind == K_BLOCK) + (addrB != nullptr);
      n_sg += kind == K_SGW;
      n_probe += (mode == M_PPRE || mode == M_PROBE);
      n_iter += lane == 0;
      n_lane += kind != K_NONE;
      // phase-3 paths: stream step, presearch of a new k-mer, walk, group
      // scan, k-mer table lookup, probe (presearch or walk)
      const uint32_t path = kind == K_NONE ? 6u
                            : mode == M_STREAM ? 0u
                            : mode == M_NEW ? 1u
                            : mode == M_WALK ? 2u
                            : mode == M_SG ? 3u
                            : mode == M_HASH ? 4u : 5u;
      if (path < 6) ++n_mode[path];
      const uint32_t seen = __reduce_or_sync(0xFFFFFFFFu, path < 6 ? 1u << path : 0u);
      n_distinct += lane == 0 ? __popc(seen) : 0;
    }
    if (done || kind == K_NONE) continue;
    // ---- phase 3: one shared rank computation, then per-mode updates ------
    const uint32_t qa = (uint32_t)(pa - ba * kBlockBits), qb = (uint32_t)(pb - bb * kBlockBits);
    I ra = sh_cmap[c] + (I)block_rank(A, qa);
    I rb = sh_cmap[c] + (I)block_rank(B, qb);
    if (!NARROW) {
      const uint64_t *l0c = s.l00 + (uint64_t)c * s.l0_stride;
      ra += (I)l0c[(uint64_t)ba >> kSuperchunkShift];
      rb += (I)l0c[(uint64_t)bb >> kSuperchunkShift];
    }
    I pl = 0, pr = 0;
    if (kind == K_PRE) {
      if (!s.wide) {
        const uint64_t e = chunk_word(A, pre_e);
        pl = (I)(e >> 32);
        pr = (I)(e & 0xFFFFFFFFULL);
      } else {
        pl = (I)chunk_word(A, 2 * pre_e);
        pr = (I)chunk_word(A, 2 * pre_e + 1);
      }
    }
    I emit = 0;
    bool emitted = false;
    I fail_at = NONE;  // char where a search of this k-mer failed
    if (mode >= M_WALK) {  // one backward-search step (the common path)
      l = ra;
      rr = rb - 1;
      ++wi;
      if (l > rr) {
        if (mode == M_STREAM) {  // no edge at v itself: find v's group start
          u = v >> 6;
          ubit = (uint32_t)(v & 63);
          mode = M_SG;
        } else if (mode == M_PROBE) {  // x[m..probe_end] is absent
          skip_until = probe_skip;
          mode = M_NEW;
        } else {
          emit = NONE;
          emitted = true;
          fail_at = wi - 1;
        }
      } else if (wi == (mode == M_PROBE ? probe_end + 1 : pos + k)) {
        if (mode == M_PROBE) {
          mode = M_NEW;  // present: nothing to skip
        } else {
          emit = l;
          emitted = true;
        }
      }
    } else if (kind == K_PRE) {  // presearch of a new k-mer or of a probe
      const bool probe = mode == M_PPRE;
      if (pl > pr) {
        if (probe) {
          skip_until = probe_skip;
          mode = M_NEW;
        } else {
          emit = NONE;
          emitted = true;
        }
      } else {
        const I start = probe ? pu + probe_lvl : pos + s.p;
        const I end = probe ? probe_end + 1 : pos + k;
        if (start >= end) {  // the presearch covered every char
          if (probe) {
            mode = M_NEW;
          } else {
            emit = pl;
            emitted = true;
          }
        } else {
          l = pl;
          rr = pr;
          wi = start;
          mode = probe ? M_PROBE : M_WALK;
        }
      }
    } else if (kind == K_HASH) {  // slots u, u + 1: (key, node) each
      const uint64_t key = SMALLK ? cw.prefix(pos, k) : 0;
      if (A.w0 == key) {
        emit = (I)A.w1;
        emitted = true;
      } else if (A.w2 == key) {
        emit = (I)A.w3;
        emitted = true;
      } else if (A.w0 == ~0ULL || A.w2 == ~0ULL) {  // an empty slot: absent
        emit = NONE;
        emitted = true;
      } else {
        u = (I)(((uint64_t)u + 2) & s.kmer_table_mask);
      }
    } else {  // M_SG: suffix-group starts at or below v, one word per step
      const uint64_t w = chunk_word(A, (uint64_t)u) & low_mask(ubit + 1);
      if (w) {
        const I g = (I)((uint64_t)u * 64 + 63 - __clzll(w));
        if (g == v) {  // v starts its group and has no edge c
          emit = NONE;
          emitted = true;
          fail_at = pos + k - 1;
        } else {  // the edge bit of v's group lives at g: one step on [g, g]
          l = rr = g;
          wi = pos + k - 1;
          mode = M_WALK;
        }
      } else if (u == 0) {
        emit = NONE;  // no group start below v: malformed SBWT
        emitted = true;
      } else {
        --u;
        ubit = 63;
      }
    }
    if (emitted) {
      if (COUNT) ++n_searched;
      v = emit;
      uint64_t res = emit == NONE ? SBWT_NOT_FOUND : (uint64_t)emit;
      if (move_to_key && res != SBWT_NOT_FOUND) res = key_walk(s, res, err);
      if (slot < rv.out_capacity) __stcs(rv.out + slot, (unsigned long long)res);
      // a failed search may prove the next k-mers absent: probe x[m..f]
      if (L && fail_at != NONE && fail_at >= pos + L + 1) {
        const I m = fail_at - L + 1;  // > pos + 1
        probe_end = fail_at;
        probe_skip = slot + (m - pos) + 1;  // slots of k-mers starting at pos+1..m
        pu = m;
        mode = M_PPRE;
      } else {
        mode = M_NEW;
      }
      ++slot;
      ++pos;
      if (SMALLK && mode == M_PPRE) cw.move_to(rv.packed, rv.invalid, pos);
    }
  }
  if (COUNT) {
    atomicAdd(counters + 0, (unsigned long long)n_pre);
    atomicAdd(counters + 1, (unsigned long long)n_block);
    atomicAdd(counters + 2, (unsigned long long)n_sg);
    atomicAdd(counters + 3, (unsigned long long)n_probe);
    atomicAdd(counters + 4, (unsigned long long)n_iter);
    atomicAdd(counters + 5, (unsigned long long)n_lane);
    atomicAdd(counters + 6, (unsigned long long)n_known);
    atomicAdd(counters + 7, (unsigned long long)n_searched);
    for (int i = 0; i < 6; ++i) atomicAdd(counters + 8 + i, (unsigned long long)n_mode[i]);
    atomicAdd(counters + 14, (unsigned long long)n_distinct);
  }
}

// Read search for the common configuration: the index has its k-mer table
// (k <= 31) and suffix-group words, fewer than 192 * 2^24 nodes (32-bit node
// arithmetic), no key-k-mer walk.  The same tiles, work queue and result
// rules as search_reads_kernel, with three single-sector operations only:
//   T_STREAM : the k-mer follows a found k-mer v: bit c of v (c = the new
//              last char).  Set: the node is C[c] + rank_c(v) (v starts its
//              suffix group, where edge bits live).  Clear: the group scan.
//   T_SG     : highest suffix-group start g <= v, one 64-bit word per load;
//              g == v means no edge c (not found), else T_STEP at g.
//   T_STEP   : bit c of g: C[c] + rank_c(g), or not found.
//   T_HASH   : any other k-mer: its k-mer table pair of slots.
// A step on the single-node interval [x, x] is nonempty iff bit c of x is
// set (rank_c(x + 1) - rank_c(x) = bit), so one rank block answers it.  No
// presearch walk and no absent-prefix probe: every k-mer the stream cannot
// reach is one table lookup.  Keeping the lane state to these four modes
// keeps the per-iteration instruction count low (the general kernel is
// issue-bound on its state machine); the kernel then waits on its sectors,
// so the loads carry L2 eviction priorities that keep the rank blocks and
// group words resident against the table lookups and the result stream.
enum : uint32_t { T_NEW = 0, T_STREAM = 1, T_STEP = 2, T_SG = 3, T_HASH = 4 };

#ifndef SBWT_TABLE_MIN_BLOCKS
#define SBWT_TABLE_MIN_BLOCKS 5  // 256-thread blocks per SM the register budget targets
#endif

template <bool COUNT>
__global__ void __launch_bounds__(256, SBWT_TABLE_MIN_BLOCKS)
    search_table_kernel(SbwtView s, ReadsView rv, const uint64_t *__restrict__ tile_read,
                        unsigned long long *counters) {
  using I = uint32_t;
  constexpr I NONE = ~I(0);
  __shared__ uint32_t sh_cmap[4];
  if (threadIdx.x < 4) sh_cmap[threadIdx.x] = (uint32_t)s.c_map[threadIdx.x];
  __syncthreads();
  const uint32_t k = s.k;
  const uint32_t lane = threadIdx.x & 31;
  const I n_kmers = (I)(rv.n_kmers_dev ? *rv.n_kmers_dev : rv.n_kmers);
  const I tsize = (I)rv.tile;
  const I n_tiles = (n_kmers + tsize - 1) / tsize;
  const I base = (I)rv.base;
  const I out_cap = (I)min(rv.out_capacity, (uint64_t)NONE);
  uint64_t n_table = 0, n_block = 0, n_sg = 0, n_iter = 0, n_lane = 0, n_known = 0,
           n_searched = 0, n_distinct = 0, n_stream = 0, n_step = 0;
  bool exhausted = false;  // the work queue is empty for this lane
  bool done = false;
  I slot = 0, slot_end = 0, r = 0, r_next = 0, pos = 0;
  I last_inv1 = 0;  // 1 + last invalid char position (0 = none)
  I v = NONE;       // node of the previous k-mer of this read
  I x = 0;          // node of a step, or the word of the group scan
  uint32_t mode = T_NEW, ubit = 63;
  uint64_t key = 0, hslot = 0;
  // rank blocks and group words (every step, ~32 bytes per 192 nodes per
  // char) stay in L2; table lines (one random lookup each) leave first
  const uint64_t pol_last = l2_policy_evict_last(), pol_first = l2_policy_evict_first();
  CharWin<I> cw;
  cw.init();
  while (true) {
    // ---- work queue (warp-collective), as in search_reads_kernel
    __syncwarp();
    const bool need = !exhausted && mode == T_NEW && slot >= slot_end;
    const unsigned need_mask = __ballot_sync(0xFFFFFFFFu, need);
    I new_tile = NONE;
    if (need_mask) {
      const int leader = __ffs(need_mask) - 1;
      unsigned long long qb = 0;
      if ((int)lane == leader) qb = atomicAdd(rv.queue, (unsigned long long)__popc(need_mask));
      qb = __shfl_sync(0xFFFFFFFFu, qb, leader);
      if (need) {
        const unsigned long long t = qb + __popc(need_mask & ((1u << lane) - 1u));
        if (t >= (unsigned long long)n_tiles) {
          exhausted = true;
        } else {
          new_tile = (I)t;
        }
      }
    }
    // ---- phase 1 (per lane): the next k-mer and its load address
    I run_slot = 0;
    uint32_t run_n = 0;
    const Block *addr = nullptr;
    uint32_t c = 0;
    if (!done) {
      if (mode == T_NEW) {
        bool ready = false;
        while (true) {
          if (slot >= slot_end) {  // next tile
            if (new_tile == NONE) {
              done = exhausted;
              break;
            }
            slot = new_tile * tsize;
            new_tile = NONE;
            slot_end = min(slot + tsize, n_kmers);
            r = (I)__ldg(tile_read + slot / tsize);
            r_next = (I)__ldg(rv.kmer_off + r + 1);
            pos = (r ? (I)__ldg(rv.ends + r - 1) : base) - base +
                  (slot - (I)__ldg(rv.kmer_off + r));
            cw.move_to(rv.packed, rv.invalid, pos);
            last_inv1 = cw.last_invalid1(pos, pos + k - 1);
            v = NONE;
          } else if (slot == r_next) {  // next read
            do {
              r_next = (I)__ldg(rv.kmer_off + (++r) + 1);
            } while (r_next == slot);
            pos = (I)__ldg(rv.ends + r - 1) - base;
            cw.move_to(rv.packed, rv.invalid, pos);
            last_inv1 = cw.last_invalid1(pos, pos + k - 1);
            v = NONE;
          }
          const I newc = pos + k - 1;
          cw.move_to(rv.packed, rv.invalid, pos);
          if (cw.invalid_at(newc)) last_inv1 = newc + 1;
          if (last_inv1 <= pos) {
            ready = true;
            break;
          }
          if (run_n) break;  // one run per iteration
          // k-mers pos .. last_inv1 - 1 all hold the invalid char at
          // last_inv1 - 1: a run of -2 up to the read / tile end, written
          // by the warp below
          const I n = min(last_inv1 - pos, min(r_next, slot_end) - slot);
          run_slot = slot;
          run_n = (uint32_t)n;
          if (COUNT) n_known += n;
          v = NONE;
          slot += n;
          pos += n;
          if (slot < min(r_next, slot_end)) {
            cw.move_to(rv.packed, rv.invalid, pos);
            last_inv1 = cw.last_invalid1(pos, pos + k - 1);
          }
        }
        if (ready) {
          if (v != NONE) {
            x = v;
            mode = T_STREAM;
          } else {
            key = cw.prefix(pos, k);
            hslot = kmer_table_bucket(key, s.kmer_table_mask);
            mode = T_HASH;
          }
        }
      }
      if (mode == T_STREAM || mode == T_STEP) {
        c = cw.char_at(pos + k - 1);
        addr = s.blocks0 + (uint64_t)c * s.block_stride + block_idx(x);
      } else if (mode == T_HASH) {
        addr = reinterpret_cast<const Block *>(s.kmer_table + 2 * hslot);
      } else if (mode == T_SG) {
        addr = chunk_of(s.suffix_group_starts, (uint64_t)x);
      }
    }
    // ---- runs of -2 (converged): the warp writes each lane's run
    for (unsigned runs = __ballot_sync(0xFFFFFFFFu, run_n != 0); runs; runs &= runs - 1) {
      const int q = __ffs(runs) - 1;
      const I q_slot = __shfl_sync(0xFFFFFFFFu, run_slot, q);
      const uint32_t q_n = __shfl_sync(0xFFFFFFFFu, run_n, q);
      for (uint32_t j = lane; j < q_n; j += 32)
        if (q_slot + j < out_cap) __stcs(rv.out + q_slot + j, (unsigned long long)SBWT_INVALID);
    }
    if (__all_sync(0xFFFFFFFFu, done)) break;
    // ---- phase 2 (converged): one 32-byte load per active lane
    Block A = Block{0, 0, 0, 0};
    if (addr) A = load_block_hint(addr, mode == T_HASH ? pol_first : pol_last);
    if (COUNT) {
      n_iter += lane == 0;
      n_lane += addr != nullptr;
      const uint32_t path = addr == nullptr ? 0u : 1u << mode;
      if (addr) {
        n_table += mode == T_HASH;
        n_block += mode == T_STREAM || mode == T_STEP;
        n_sg += mode == T_SG;
        n_stream += mode == T_STREAM;
        n_step += mode == T_STEP;
      }
      const uint32_t seen = __reduce_or_sync(0xFFFFFFFFu, path);
      n_distinct += lane == 0 ? __popc(seen) : 0;
    }
    if (addr == nullptr) continue;
    // ---- phase 3 (per lane)
    I emit = NONE;
    bool emitted = false;
    if (mode == T_HASH) {  // slots hslot, hslot + 1: (key, node) each
      if (A.w0 == key) {
        emit = (I)A.w1;
        emitted = true;
      } else if (A.w2 == key) {
        emit = (I)A.w3;
        emitted = true;
      } else if (A.w0 == ~0ULL || A.w2 == ~0ULL) {  // an empty slot: absent
        emitted = true;
      } else {
        hslot = (hslot + 2) & s.kmer_table_mask;
      }
    } else if (mode == T_SG) {  // group starts at or below v in word x
      const uint64_t w = chunk_word(A, (uint64_t)x) & low_mask(ubit + 1);
      if (w) {
        const I g = x * 64 + 63 - (I)__clzll(w);
        if (g == v) {
          emitted = true;  // v starts its group and has no edge c
        } else {
          x = g;
          mode = T_STEP;
        }
      } else if (x == 0) {
        emitted = true;  // no group start below v: malformed SBWT
      } else {
        --x;
        ubit = 63;
      }
    } else {  // a step on [x, x] with the k-mer's last char
      const uint32_t q = x - block_idx(x) * kBlockBits;
      if (block_bit(A, q)) {
        emit = sh_cmap[c] + (I)block_rank(A, q);
        emitted = true;
      } else if (mode == T_STREAM) {  // no edge at v itself: v's group start
        ubit = x & 63;
        x >>= 6;
        mode = T_SG;
      } else {
        emitted = true;
      }
    }
    if (emitted) {
      if (COUNT) ++n_searched;
      v = emit;
      if (slot < out_cap)
        __stcs(rv.out + slot,
               (unsigned long long)(emit == NONE ? SBWT_NOT_FOUND : (uint64_t)emit));
      ++slot;
      ++pos;
      mode = T_NEW;
    }
  }
  if (COUNT) {
    atomicAdd(counters + 0, (unsigned long long)n_table);
    atomicAdd(counters + 1, (unsigned long long)n_block);
    atomicAdd(counters + 2, (unsigned long long)n_sg);
    atomicAdd(counters + 4, (unsigned long long)n_iter);
    atomicAdd(counters + 5, (unsigned long long)n_lane);
    atomicAdd(counters + 6, (unsigned long long)n_known);
    atomicAdd(counters + 7, (unsigned long long)n_searched);
    atomicAdd(counters + 8, (unsigned long long)n_stream);   // stream steps
    atomicAdd(counters + 10, (unsigned long long)n_step);    // steps at a group start
    atomicAdd(counters + 11, (unsigned long long)n_sg);      // group scan words
    atomicAdd(counters + 12, (unsigned long long)n_table);   // table lookups
    atomicAdd(counters + 14, (unsigned long long)n_distinct);
  }
}

// Read search with the k-mer table and its filter, W walks per lane (a walk
// = one work tile being searched).  The same tiles, work queue and result
// rules as search_table_kernel.  Each iteration first issues the loads of all
// W walks of the lane and then uses them, so a lane keeps W independent
// loads in flight (up to 4 W while its walks read filter words).  Walk modes:
//   WK_STREAM, WK_SG, WK_STEP : T_STREAM, T_SG and T_STEP of search_table_kernel;
//   WK_FILTER : the walk has no previous node (tile or read start, after an
//              absent k-mer or an invalid char): the filter words of the
//              next nb <= 4 k-mers of the read, loaded together.  K-mers the
//              filter rejects are absent (-1); the first one it passes goes
//              to WK_HASH.
//   WK_HASH   : the k-mer table pair of slots of that k-mer.
// The filter answers most k-mers a stream step cannot reach (those around
// read errors) from a structure 25x smaller than the table; a rejection is
// exact, so results equal the table kernel's.  Results pass through 4 slots
// per walk in shared memory and leave as one 32-byte store per 4 consecutive
// k-mer slots (tiles are multiples of 4 slots) when the output is 32-byte
// aligned.
enum : uint32_t { WK_NEW = 0, WK_STREAM = 1, WK_STEP = 2, WK_SG = 3, WK_FILTER = 4, WK_HASH = 5,
                  WK_DONE = 6 };
constexpr uint32_t kFilterBatch = 4;

__device__ __forceinline__ uint64_t load_u64_nc(const uint64_t *p) {
  uint64_t v;
  asm("ld.global.nc.L1::no_allocate.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

// load_u64_nc with an L2 eviction policy.
__device__ __forceinline__ uint64_t load_u64_hint(const uint64_t *p, uint64_t policy) {
  uint64_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u64 %0, [%1], %2;"
      : "=l"(v)
      : "l"(p), "l"(policy));
  return v;
}

__device__ __forceinline__ void store_u32x4_cs(uint32_t *p, uint32_t a, uint32_t b,
                                               uint32_t c, uint32_t d) {
  asm volatile("st.global.cs.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
}

// A 32-bit node of the narrow kernels as a 64-bit result (~0u: not found).
__device__ __forceinline__ uint64_t widen_node(uint32_t node) {
  return node == ~0u ? (uint64_t)SBWT_NOT_FOUND : (uint64_t)node;
}

__device__ __forceinline__ void store_sector_cs(uint64_t *p, uint64_t a, uint64_t b,
                                                uint64_t c, uint64_t d) {
  asm volatile("st.global.cs.v4.u64 [%0], {%1,%2,%3,%4};" ::"l"(p), "l"(a), "l"(b), "l"(c),
               "l"(d)
               : "memory");
}

// W walks per lane; MINB = 256-thread blocks per SM the register budget
// targets (W = 1: 5, or 6 for the lean 16-slot kernel without the filter,
// which fits 40 registers without spills; W = 2: 4 or 3, W = 4: 2).
// LEAN: no filter and no staging (a walk without a previous node goes to the
// table at once; each result is one 8-byte store), i.e. search_table_kernel's
// work with W walks per lane.
// LFILTER (with LEAN): the filter in front of the table, one k-mer at a time.
// LSTAGE (with LEAN, W = 1): results staged per lane in a shared-memory row
// of G slots (one group of G consecutive k-mer slots) and stored by the warp
// together: once per iteration, at a converged point, the lanes whose group
// is complete or left behind (the walk moved past it or ended) hand their
// rows to the warp, 32 / G rows per store instruction, each row one run of
// G consecutive results (G * 8 bytes, a full 128-byte line for G = 16).
// G: slots staged per walk before they are stored (4, 8 or 16); without
// LEAN, results leave as 32-byte stores of 4 slots per lane.
template <int W, int MINB, bool COUNT, bool LEAN = false, bool LFILTER = false,
          bool LSTAGE = false, int G = 4, int KC = 0>
__global__ void __launch_bounds__(256, MINB)
    search_walks_kernel(SbwtView s, ReadsView rv, const uint64_t *__restrict__ tile_read,
                        unsigned long long *counters) {
  using I = uint32_t;
  constexpr I NONE = ~I(0);
  __shared__ uint32_t sh_cmap[4];
  // staged results (32-bit nodes, NONE for not found): slot % G first for
  // the per-lane stores; one padded row per lane for the warp's stores (the
  // odd row stride keeps both the lanes' writes and a row read
  // conflict-free)
  // (row w * 256 + thread for walk w; a lean walk emits at most one result
  // per iteration, so one open group per walk suffices)
  constexpr bool COOP = LEAN && LSTAGE;
  __shared__ uint32_t sh_out[COOP ? 1 : G][W][256];
  __shared__ uint32_t sh_row[COOP ? 256 * W : 1][G + 1];
  constexpr uint32_t GFULL = (1u << G) - 1u;
  if (threadIdx.x < 4) sh_cmap[threadIdx.x] = (uint32_t)s.c_map[threadIdx.x];
  __syncthreads();
  const uint32_t k = KC ? (uint32_t)KC : s.k;  // KC: k known at compile time
  const uint32_t lane = threadIdx.x & 31;
  const I n_kmers = (I)(rv.n_kmers_dev ? *rv.n_kmers_dev : rv.n_kmers);
  const I tsize = (I)rv.tile;
  const I n_tiles = (n_kmers + tsize - 1) / tsize;
  const I base = (I)rv.base;
  const I out_cap = (I)min(rv.out_capacity, (uint64_t)NONE);
  const bool vec_out = ((uintptr_t)rv.out & 31) == 0;
  uint32_t *const out32 = rv.out32;
  const bool vec_out32 = ((uintptr_t)out32 & 15) == 0;
  uint64_t n_table = 0, n_block = 0, n_sg = 0, n_filter = 0, n_iter = 0, n_lane = 0,
           n_known = 0, n_searched = 0, n_stream = 0, n_step = 0, n_distinct = 0;
  I slot[W], slot_end[W], r[W], r_next[W], pos[W], last_inv1[W], v[W], x[W], hslot[W];
  I obase[W];
  uint32_t mode[W], ubit[W], nb[W], omask[W];
  CharWin<I> cw[W];
#pragma unroll
  for (int w = 0; w < W; ++w) {
    slot[w] = slot_end[w] = r[w] = r_next[w] = pos[w] = last_inv1[w] = x[w] = hslot[w] = 0;
    v[w] = NONE;
    obase[w] = 0;
    mode[w] = WK_NEW;
    ubit[w] = 63;
    nb[w] = 0;
    omask[w] = 0;
    cw[w].init();
  }
  const uint64_t pol_last = l2_policy_evict_last(), pol_first = l2_policy_evict_first();

  auto flush = [&](int w) {  // the staged slots of walk w's open group
   if constexpr (!COOP) {
    const I g = obase[w];
    const uint32_t t = threadIdx.x;
    const bool full = omask[w] == GFULL && g + G <= out_cap;
    if (out32) {  // 32-bit codes: the value's low word (markers stay markers)
      if (full && vec_out32) {
#pragma unroll
        for (int q = 0; q < G; q += 4)
          store_u32x4_cs(out32 + g + q, sh_out[q][w][t], sh_out[q + 1][w][t],
                         sh_out[q + 2][w][t], sh_out[q + 3][w][t]);
      } else {
#pragma unroll
        for (int q = 0; q < G; ++q)
          if (((omask[w] >> q) & 1u) && g + q < out_cap)
            __stcs(out32 + g + q, sh_out[q][w][t]);
      }
    } else if (full && vec_out) {
#pragma unroll
      for (int q = 0; q < G; q += 4)
        store_sector_cs(rv.out + g + q, widen_node(sh_out[q][w][t]),
                        widen_node(sh_out[q + 1][w][t]), widen_node(sh_out[q + 2][w][t]),
                        widen_node(sh_out[q + 3][w][t]));
    } else {
#pragma unroll
      for (int q = 0; q < G; ++q)
        if (((omask[w] >> q) & 1u) && g + q < out_cap)
          __stcs(rv.out + g + q, (unsigned long long)widen_node(sh_out[q][w][t]));
    }
    omask[w] = 0;
   }
  };
  auto emit = [&](int w, I sl, I node) {
    if constexpr (COOP) {  // the group of sl is obase[w] or none is open
      if (!omask[w]) obase[w] = sl & ~I(G - 1);
      sh_row[w * 256 + threadIdx.x][sl & (G - 1)] = node;
      omask[w] |= 1u << (sl & (G - 1));
      return;
    } else {
    if (LEAN && !LSTAGE) {
      if (sl < out_cap) {
        if (out32)
          __stcs(out32 + sl, (unsigned int)node);
        else
          __stcs(rv.out + sl,
                 node == NONE ? (unsigned long long)SBWT_NOT_FOUND : (unsigned long long)node);
      }
      return;
    }
    const I g = sl & ~I(G - 1);
    if (omask[w] && g != obase[w]) flush(w);
    obase[w] = g;
    sh_out[sl & (G - 1)][w][threadIdx.x] = node;
    omask[w] |= 1u << (sl & (G - 1));
    if (omask[w] == GFULL) flush(w);
    }
  };

  while (true) {
    // ---- work queue (warp-collective): one tile per walk that needs one
    I new_tile[W];
#pragma unroll
    for (int w = 0; w < W; ++w) new_tile[w] = NONE;
    if (W == 1) {  // one ballot: lanes in order take consecutive tiles
      const bool nd = mode[0] == WK_NEW && slot[0] >= slot_end[0];
      const unsigned nm = __ballot_sync(0xFFFFFFFFu, nd);
      if (nm) {
        const int leader = __ffs(nm) - 1;
        unsigned long long qb = 0;
        if ((int)lane == leader) qb = atomicAdd(rv.queue, (unsigned long long)__popc(nm));
        qb = __shfl_sync(0xFFFFFFFFu, qb, leader);
        if (nd) {
          const unsigned long long t = qb + __popc(nm & ((1u << lane) - 1u));
          if (t < (unsigned long long)n_tiles)
            new_tile[0] = (I)t;
          else
            mode[0] = WK_DONE;
        }
      }
    }
    uint32_t need = 0, incl = 0, total = 0;
    if (W > 1) {
#pragma unroll
      for (int w = 0; w < W; ++w) need += (mode[w] == WK_NEW && slot[w] >= slot_end[w]);
      incl = need;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if ((int)lane >= o) incl += t;
      }
      total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    if (total) {
      unsigned long long qb = 0;
      if (lane == 31) qb = atomicAdd(rv.queue, (unsigned long long)total);
      qb = __shfl_sync(0xFFFFFFFFu, qb, 31);
      unsigned long long t = qb + incl - need;
#pragma unroll
      for (int w = 0; w < W; ++w) {
        if (mode[w] == WK_NEW && slot[w] >= slot_end[w]) {
          if (t < (unsigned long long)n_tiles)
            new_tile[w] = (I)t;
          else
            mode[w] = WK_DONE;
          ++t;
        }
      }
    }
    // ---- phase 1 (per walk): the next k-mer, runs of -2, the walk's mode
    I run_slot[W];
    uint32_t run_n[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      run_slot[w] = 0;
      run_n[w] = 0;
      if (mode[w] != WK_NEW) continue;
      bool ready = false;
      while (true) {
        if (slot[w] >= slot_end[w]) {  // next tile
          if (new_tile[w] == NONE) break;
          slot[w] = new_tile[w] * tsize;
          new_tile[w] = NONE;
          slot_end[w] = min(slot[w] + tsize, n_kmers);
          r[w] = (I)__ldg(tile_read + slot[w] / tsize);
          r_next[w] = (I)__ldg(rv.kmer_off + r[w] + 1);
          pos[w] = (r[w] ? (I)__ldg(rv.ends + r[w] - 1) : base) - base +
                   (slot[w] - (I)__ldg(rv.kmer_off + r[w]));
          cw[w].move_to(rv.packed, rv.invalid, pos[w]);
          last_inv1[w] = cw[w].last_invalid1(pos[w], pos[w] + k - 1);
          v[w] = NONE;
        } else if (slot[w] == r_next[w]) {  // next read
          do {
            r_next[w] = (I)__ldg(rv.kmer_off + (++r[w]) + 1);
          } while (r_next[w] == slot[w]);
          pos[w] = (I)__ldg(rv.ends + r[w] - 1) - base;
          cw[w].move_to(rv.packed, rv.invalid, pos[w]);
          last_inv1[w] = cw[w].last_invalid1(pos[w], pos[w] + k - 1);
          v[w] = NONE;
        }
        const I newc = pos[w] + k - 1;
        cw[w].move_to(rv.packed, rv.invalid, pos[w]);
        if (cw[w].invalid_at(newc)) last_inv1[w] = newc + 1;
        if (last_inv1[w] <= pos[w]) {
          ready = true;
          break;
        }
        if (run_n[w]) break;  // one run per walk per iteration
        // k-mers pos .. last_inv1 - 1 all hold the invalid char at
        // last_inv1 - 1: a run of -2 up to the read / tile end
        const I n = min(last_inv1[w] - pos[w], min(r_next[w], slot_end[w]) - slot[w]);
        run_slot[w] = slot[w];
        run_n[w] = (uint32_t)n;
        if (COUNT) n_known += n;
        v[w] = NONE;
        slot[w] += n;
        pos[w] += n;
        if (slot[w] < min(r_next[w], slot_end[w])) {
          cw[w].move_to(rv.packed, rv.invalid, pos[w]);
          last_inv1[w] = cw[w].last_invalid1(pos[w], pos[w] + k - 1);
        }
      }
      if (ready) {
        if (v[w] != NONE) {
          x[w] = v[w];
          mode[w] = WK_STREAM;
        } else if (LEAN && LFILTER) {
          nb[w] = 1;
          mode[w] = WK_FILTER;
        } else if (LEAN) {
          hslot[w] = (I)kmer_table_bucket(cw[w].prefix(pos[w], k), s.kmer_table_mask);
          mode[w] = WK_HASH;
        } else {
          // k-mers pos .. pos + nb - 1 of this read and tile, in the char
          // window, whose chars after newc are valid
          const uint32_t off = pos[w] - 32 * cw[w].wbase;
          uint32_t lim = min(min(r_next[w], slot_end[w]) - slot[w], 65u - k - off);
          lim = min(lim, kFilterBatch);
          const uint32_t o1 = off + k;  // window offset of newc + 1
          const uint64_t m = (cw[w].inv >> o1) & low_mask(lim - 1);
          if (m) lim = min(lim, (uint32_t)__ffsll((long long)m));
          nb[w] = lim;
          mode[w] = WK_FILTER;
        }
      }
    }
    // ---- runs of -2 (converged): the warp writes each walk's run
#pragma unroll
    for (int w = 0; w < W; ++w) {
      for (unsigned runs = __ballot_sync(0xFFFFFFFFu, run_n[w] != 0); runs; runs &= runs - 1) {
        const int q = __ffs(runs) - 1;
        const I q_slot = __shfl_sync(0xFFFFFFFFu, run_slot[w], q);
        const uint32_t q_n = __shfl_sync(0xFFFFFFFFu, run_n[w], q);
        for (uint32_t j = lane; j < q_n; j += 32) {
          if (q_slot + j >= out_cap) continue;
          if (out32)
            __stcs(out32 + q_slot + j, 0xFFFFFFFEu);
          else
            __stcs(rv.out + q_slot + j, (unsigned long long)SBWT_INVALID);
        }
      }
    }
    if (COOP) {  // ---- the warp stores the rows of complete or left groups
     constexpr int P = 32 / G;  // rows per store instruction
     const int sub = (int)lane / G, q = (int)lane % G;
#pragma unroll
     for (int w = 0; w < W; ++w) {
      const bool nf = omask[w] && (mode[w] == WK_DONE || omask[w] == GFULL ||
                                   (slot[w] & ~I(G - 1)) != obase[w]);
      for (unsigned fm = __ballot_sync(0xFFFFFFFFu, nf); fm;) {
        int src = -1;
#pragma unroll
        for (int i = 0; i < P; ++i) {  // the sub-th lane left in fm
          if (i == sub && fm) src = __ffs(fm) - 1;
          fm &= fm - 1;
        }
        const int from = src < 0 ? (int)lane : src;
        const I gb = __shfl_sync(0xFFFFFFFFu, obase[w], from);
        const uint32_t gm = __shfl_sync(0xFFFFFFFFu, omask[w], from);
        if (src >= 0 && ((gm >> q) & 1u) && gb + (I)q < out_cap) {
          const uint32_t val = sh_row[w * 256 + (threadIdx.x & ~31u) + (unsigned)src][q];
          if (out32)
            __stcs(out32 + gb + q, val);
          else
            __stcs(rv.out + gb + q, (unsigned long long)widen_node(val));
        }
      }
      if (nf) omask[w] = 0;
     }
    }
    bool all_done = true;
#pragma unroll
    for (int w = 0; w < W; ++w) all_done &= mode[w] == WK_DONE;
    if (__all_sync(0xFFFFFFFFu, all_done)) break;
    // ---- phase 2: the loads of every walk, issued before any is used
    Block A[W];
    I step_base[W];      // a step's C[c] (its char's first node)
    uint32_t step_q[W];  // a step's offset of x in its rank block
    uint64_t fz[W];      // the filter's first k-mer hash
#pragma unroll
    for (int w = 0; w < W; ++w) {
      A[w] = Block{0, 0, 0, 0};
      step_base[w] = 0;
      step_q[w] = 0;
      fz[w] = 0;
      if (mode[w] == WK_STREAM || mode[w] == WK_STEP) {
        const uint32_t c = cw[w].char_at(pos[w] + k - 1);
        const I b = block_idx(x[w]);
        A[w] = load_block_hint(s.blocks0 + (uint64_t)c * s.block_stride + b, pol_last);
        step_base[w] = sh_cmap[c];
        step_q[w] = x[w] - b * kBlockBits;
      } else if (mode[w] == WK_SG) {
        A[w] = load_block_hint(chunk_of(s.suffix_group_starts, (uint64_t)x[w]), pol_last);
      } else if (mode[w] == WK_HASH) {
        A[w] = load_block_hint(reinterpret_cast<const Block *>(s.kmer_table + 2 * (uint64_t)hslot[w]),
                               pol_first);
      } else if ((!LEAN || LFILTER) && mode[w] == WK_FILTER) {  // no filter: never
        uint64_t z = kmer_mix(cw[w].prefix(pos[w], k));
        fz[w] = z;
        A[w].w0 = load_u64_hint(s.kmer_filter + kmer_filter_word(z, s.filter_words), pol_first);
        if (nb[w] > 1) {
          z = kmer_mix(cw[w].prefix(pos[w] + 1, k));
          A[w].w1 = load_u64_hint(s.kmer_filter + kmer_filter_word(z, s.filter_words), pol_first);
        }
        if (nb[w] > 2) {
          z = kmer_mix(cw[w].prefix(pos[w] + 2, k));
          A[w].w2 = load_u64_hint(s.kmer_filter + kmer_filter_word(z, s.filter_words), pol_first);
        }
        if (nb[w] > 3) {
          z = kmer_mix(cw[w].prefix(pos[w] + 3, k));
          A[w].w3 = load_u64_hint(s.kmer_filter + kmer_filter_word(z, s.filter_words), pol_first);
        }
      }
    }
    if (COUNT) {
      n_iter += lane == 0;
      uint32_t path = 0;
#pragma unroll
      for (int w = 0; w < W; ++w) {
        const uint32_t md = mode[w];
        n_lane += md >= WK_STREAM && md <= WK_HASH;
        path |= (md >= WK_STREAM && md <= WK_HASH) ? 1u << md : 0u;
        n_table += md == WK_HASH;
        n_block += md == WK_STREAM || md == WK_STEP;
        n_sg += md == WK_SG;
        n_filter += md == WK_FILTER ? nb[w] : 0;
        n_stream += md == WK_STREAM;
        n_step += md == WK_STEP;
      }
      const uint32_t seen = __reduce_or_sync(0xFFFFFFFFu, path);
      n_distinct += lane == 0 ? __popc(seen) : 0;
    }
    // ---- phase 3 (per walk)
#pragma unroll
    for (int w = 0; w < W; ++w) {
      const uint32_t md = mode[w];
      if ((!LEAN || LFILTER) && md == WK_FILTER) {
        // k-mers the filter rejects are absent; the first it passes is looked up
        uint32_t j = 0;
        for (; j < nb[w]; ++j) {
          const uint64_t z = j == 0 ? fz[w] : kmer_mix(cw[w].prefix(pos[w], k));
          const uint64_t word = j == 0 ? A[w].w0 : (j == 1 ? A[w].w1 : (j == 2 ? A[w].w2 : A[w].w3));
          const uint64_t bits = kmer_filter_bits(z);
          if ((word & bits) == bits) {
            hslot[w] = (I)kmer_table_slot(z, s.kmer_table_mask);
            mode[w] = WK_HASH;
            break;
          }
          if (COUNT) ++n_searched;
          emit(w, slot[w], NONE);
          ++slot[w];
          ++pos[w];
        }
        if (j == nb[w]) mode[w] = WK_NEW;  // v stays NONE
        continue;
      }
      if (md != WK_STREAM && md != WK_STEP && md != WK_SG && md != WK_HASH) continue;
      I res = NONE;
      bool emitted = false;
      if (md == WK_HASH) {  // slots hslot, hslot + 1: (key, node) each
        const uint64_t key = cw[w].prefix(pos[w], k);
        if (A[w].w0 == key) {
          res = (I)A[w].w1;
          emitted = true;
        } else if (A[w].w2 == key) {
          res = (I)A[w].w3;
          emitted = true;
        } else if (A[w].w0 == ~0ULL || A[w].w2 == ~0ULL) {  // an empty slot: absent
          emitted = true;
        } else {
          hslot[w] = (I)(((uint64_t)hslot[w] + 2) & s.kmer_table_mask);
        }
      } else if (md == WK_SG) {  // group starts at or below v in word x
        const uint64_t wd = chunk_word(A[w], (uint64_t)x[w]) & low_mask(ubit[w] + 1);
        if (wd) {
          const I g = x[w] * 64 + 63 - (I)__clzll(wd);
          if (g == v[w]) {
            emitted = true;  // v starts its group and has no edge c
          } else {
            x[w] = g;
            mode[w] = WK_STEP;
          }
        } else if (x[w] == 0) {
          emitted = true;  // no group start below v: malformed SBWT
        } else {
          --x[w];
          ubit[w] = 63;
        }
      } else {  // a step on [x, x] with the k-mer's last char
        const uint32_t q = step_q[w];
        if (block_bit(A[w], q)) {
          res = step_base[w] + (I)block_rank(A[w], q);
          emitted = true;
        } else if (md == WK_STREAM) {  // no edge at v itself: v's group start
          ubit[w] = x[w] & 63;
          x[w] >>= 6;
          mode[w] = WK_SG;
        } else {
          emitted = true;
        }
      }
      if (emitted) {
        if (COUNT) ++n_searched;
        v[w] = res;
        emit(w, slot[w], res);
        ++slot[w];
        ++pos[w];
        mode[w] = WK_NEW;
      }
    }
  }
  if (!COOP) {
#pragma unroll
    for (int w = 0; w < W; ++w)
      if (omask[w]) flush(w);
  }
  if (COUNT) {
    atomicAdd(counters + 0, (unsigned long long)n_table);
    atomicAdd(counters + 1, (unsigned long long)n_block);
    atomicAdd(counters + 2, (unsigned long long)n_sg);
    atomicAdd(counters + 3, (unsigned long long)n_filter);
    atomicAdd(counters + 4, (unsigned long long)n_iter);
    atomicAdd(counters + 5, (unsigned long long)n_lane);
    atomicAdd(counters + 6, (unsigned long long)n_known);
    atomicAdd(counters + 7, (unsigned long long)n_searched);
    atomicAdd(counters + 8, (unsigned long long)n_stream);   // stream steps
    atomicAdd(counters + 9, (unsigned long long)n_filter);   // filter words
    atomicAdd(counters + 10, (unsigned long long)n_step);    // steps at a group start
    atomicAdd(counters + 11, (unsigned long long)n_sg);      // group scan words
    atomicAdd(counters + 12, (unsigned long long)n_table);   // table lookups
    atomicAdd(counters + 14, (unsigned long long)n_distinct);
  }
}

// Tables up to this size stay in L2 (126 MB on B200) beside the filter and
// the streams of one launch: the k-mers kernels load their lines evict-last.
constexpr uint64_t kTableL2ResidentBytes = 96ULL << 20;

// Read search with every k-mer looked up on its own (k <= 31, k-mer table and
// filter): no stream steps, so no lane waits on the previous k-mer of its
// read.  A warp takes chunks of 32 * PER consecutive k-mer slots; lane j
// handles slots j, j + 32, ... of the chunk, so every warp store writes 32
// consecutive results.  Per slot: its read (from the tile table, a few steps
// forward), the k chars from the packed words, -2 if one is invalid, else the
// filter word (all PER issued together), and for the keys the filter passes
// the k-mer table pair of slots (probed to the first empty slot).  Results
// equal the other kernels' (the table holds exactly the SBWT's k-mers; a
// filter rejection is exact).  It beats the stream kernels when the table and
// filter stay in L2 and inside the address-translation reach (small indexes):
// all loads of a lane are independent.  FILT = false skips the filter: every
// valid k-mer goes to the table (one round trip fewer; for a table that stays
// in L2 an absent k-mer's probe costs about what its filter word does).
template <int PER, bool COUNT, bool FILT = true, int KC = 0>
__global__ void __launch_bounds__(256)
    search_kmers_kernel(SbwtView s, ReadsView rv, const uint64_t *__restrict__ tile_read,
                        unsigned long long *counters) {
  using I = uint32_t;
  constexpr I CH = 32 * PER;
  // reads of a chunk resolved from one round of loads (slots past them walk
  // on): 2 for chunks of 64 slots (0.155 against 0.171 ms with 5 on the
  // 1 Mbp case: fewer loads and selects per slot), 5 for chunks of 128
  constexpr int MR = PER <= 2 ? 2 : 5;
  const uint32_t k = KC ? (uint32_t)KC : s.k;  // KC: k known at compile time
  const uint32_t lane = threadIdx.x & 31;
  const I n_kmers = (I)(rv.n_kmers_dev ? *rv.n_kmers_dev : rv.n_kmers);
  const I n_reads = (I)rv.n_reads;
  const I base = (I)rv.base;
  const I out_cap = (I)min(rv.out_capacity, (uint64_t)~I(0));
  const I n_chunks = (n_kmers + CH - 1) / CH;
  const uint64_t warp0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  // table lines: evict-last when the table fits well inside L2 (its lines
  // are touched again by later k-mers), evict-first when it does not
  const uint64_t pol_table = (s.kmer_table_mask + 1) * 16 <= kTableL2ResidentBytes
                                 ? l2_policy_evict_last()
                                 : l2_policy_evict_first();
  uint64_t n_table = 0, n_filter = 0, n_known = 0;
  // Every phase below issues all its loads before it uses any (no load waits
  // on a branch over another's value), so one chunk costs about four
  // round trips: read offsets, chars, filter words, table.  The tile-table
  // entry of the next chunk is loaded one chunk ahead.
  I r_next = warp0 < n_chunks ? (I)__ldg(tile_read + (I)warp0 * CH / (I)rv.tile) : 0;
  for (uint64_t ch = warp0; ch < n_chunks; ch += warps) {
    const I c0 = (I)ch * CH;
    I r = r_next;
    if (ch + warps < n_chunks)
      r_next = (I)__ldg(tile_read + (I)(ch + warps) * CH / (I)rv.tile);
    // offsets and ends of reads r .. r + MR - 1 (one round of loads); the
    // chunk's first read is r itself when the tile size divides the chunk
    I ko[MR + 1], st[MR];
    while (true) {
#pragma unroll
      for (int j = 0; j <= MR; ++j) ko[j] = (I)__ldg(rv.kmer_off + min(r + j, n_reads));
#pragma unroll
      for (int j = 0; j < MR; ++j) {
        const I rr = min(r + j, n_reads);
        st[j] = (rr ? (I)__ldg(rv.ends + rr - 1) : base) - base;
      }
      if (ko[1] > c0 || r + 1 >= n_reads) break;
      // forward to the chunk's first read (tiles that do not divide chunks)
      while (r + 1 < n_reads && (I)__ldg(rv.kmer_off + r + 1) <= c0) ++r;
    }
    I slot[PER], pos[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      slot[t] = c0 + (I)t * 32 + lane;
      pos[t] = 0;
      if (slot[t] >= n_kmers) continue;
      int j = 0;
#pragma unroll
      for (int q = 1; q < MR; ++q) j += ko[q] <= slot[t] ? 1 : 0;
      if (ko[MR] <= slot[t]) {  // beyond the loaded reads: walk on (short reads)
        I rr = r + MR;
        while ((I)__ldg(rv.kmer_off + rr + 1) <= slot[t]) ++rr;
        pos[t] = (I)__ldg(rv.ends + rr - 1) - base + (slot[t] - (I)__ldg(rv.kmer_off + rr));
      } else {
        I ko_j = ko[0], st_j = st[0];
#pragma unroll
        for (int q = 1; q < MR; ++q)
          if (q == j) {
            ko_j = ko[q];
            st_j = st[q];
          }
        pos[t] = st_j + (slot[t] - ko_j);
      }
    }
    // chars and invalid bits of every k-mer of the lane
    uint64_t w0[PER], w1[PER], inv[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const I wi = pos[t] >> 5;
      const bool in = slot[t] < n_kmers;
      w0[t] = in ? __ldg(rv.packed + wi) : 0;
      w1[t] = in ? __ldg(rv.packed + wi + 1) : 0;
      inv[t] = in ? ((uint64_t)__ldg(rv.invalid + wi) |
                     ((uint64_t)__ldg(rv.invalid + wi + 1) << 32))
                  : 0;
    }
    uint64_t key[PER], z[PER], fw[PER];
    uint32_t state[PER];  // 0 none, 1 invalid, 2 filter
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const uint32_t off = pos[t] & 31;
      key[t] = 0;
      state[t] = slot[t] >= n_kmers ? 0u : (((inv[t] >> off) & low_mask(k)) ? 1u : 2u);
      const uint64_t v = off ? (w0[t] << (2 * off)) | (w1[t] >> (64 - 2 * off)) : w0[t];
      if (state[t] == 2) key[t] = v >> (64 - 2 * k);
    }
    // filter words, all issued before any is used
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      fw[t] = 0;
      z[t] = 0;
      if (state[t] == 2) {
        z[t] = kmer_mix(key[t]);
        if (FILT) fw[t] = load_u64_nc(s.kmer_filter + kmer_filter_word(z[t], s.filter_words));
      }
    }
    uint64_t res[PER];
    bool look[PER];
    I hs[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      res[t] = state[t] == 1 ? (uint64_t)SBWT_INVALID : (uint64_t)SBWT_NOT_FOUND;
      const uint64_t bits = kmer_filter_bits(z[t]);
      look[t] = state[t] == 2 && (!FILT || (fw[t] & bits) == bits);
      hs[t] = look[t] ? (I)kmer_table_slot(z[t], s.kmer_table_mask) : 0;
      if (COUNT) {
        n_filter += FILT && state[t] == 2;
        n_known += state[t] == 1;
      }
    }
    // table probes of the keys the filter passed, one round of loads at a time
    while (true) {
      bool any = false;
      Block A[PER];  // read only where look[t]
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        if (look[t]) {
          A[t] = load_block_hint(
              reinterpret_cast<const Block *>(s.kmer_table + 2 * (uint64_t)hs[t]), pol_table);
          any = true;
        }
      }
      if (!any) break;
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        if (!look[t]) continue;
        if (COUNT) ++n_table;
        if (A[t].w0 == key[t]) {
          res[t] = A[t].w1;
          look[t] = false;
        } else if (A[t].w2 == key[t]) {
          res[t] = A[t].w3;
          look[t] = false;
        } else if (A[t].w0 == ~0ULL || A[t].w2 == ~0ULL) {
          look[t] = false;  // an empty slot: absent
        } else {
          hs[t] = (I)(((uint64_t)hs[t] + 2) & s.kmer_table_mask);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      if (slot[t] >= n_kmers || slot[t] >= out_cap) continue;
      if (rv.out32)
        __stcs(rv.out32 + slot[t], (unsigned int)res[t]);
      else
        __stcs(rv.out + slot[t], (unsigned long long)res[t]);
    }
  }
  if (COUNT) {
    atomicAdd(counters + 0, (unsigned long long)n_table);
    atomicAdd(counters + 3, (unsigned long long)n_filter);
    atomicAdd(counters + 6, (unsigned long long)n_known);
    atomicAdd(counters + 9, (unsigned long long)n_filter);   // filter words
    atomicAdd(counters + 12, (unsigned long long)n_table);   // table lookups
  }
}

template <int PER, bool COUNT>
__global__ void __launch_bounds__(256)
    search_kmers_seq_kernel(SbwtView s, ReadsView rv, const uint64_t *__restrict__ tile_read,
                        unsigned long long *counters) {
  using I = uint32_t;
  constexpr I CH = 32 * PER;
  constexpr int MR = 5;  // reads of a chunk resolved from one round of loads
  const uint32_t k = s.k;
  const uint32_t lane = threadIdx.x & 31;
  const I n_kmers = (I)(rv.n_kmers_dev ? *rv.n_kmers_dev : rv.n_kmers);
  const I n_reads = (I)rv.n_reads;
  const I base = (I)rv.base;
  const I out_cap = (I)min(rv.out_capacity, (uint64_t)~I(0));
  const I n_chunks = (n_kmers + CH - 1) / CH;
  const uint64_t warp0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  // table lines: evict-last when the table fits well inside L2 (its lines
  // are touched again by later k-mers), evict-first when it does not
  const uint64_t pol_table = (s.kmer_table_mask + 1) * 16 <= kTableL2ResidentBytes
                                 ? l2_policy_evict_last()
                                 : l2_policy_evict_first();
  uint64_t n_table = 0, n_filter = 0, n_known = 0;
  // Every phase below issues all its loads before it uses any (no load waits
  // on a branch over another's value), so one chunk costs about four
  // round trips: read offsets, chars, filter words, table.  The tile-table
  // entry of the next chunk is loaded one chunk ahead.
  I r_next = warp0 < n_chunks ? (I)__ldg(tile_read + (I)warp0 * CH / (I)rv.tile) : 0;
  for (uint64_t ch = warp0; ch < n_chunks; ch += warps) {
    const I c0 = (I)ch * CH;
    I r = r_next;
    if (ch + warps < n_chunks)
      r_next = (I)__ldg(tile_read + (I)(ch + warps) * CH / (I)rv.tile);
    // offsets and ends of reads r .. r + MR - 1 (one round of loads); the
    // chunk's first read is r itself when the tile size divides the chunk
    I ko[MR + 1], st[MR];
    while (true) {
#pragma unroll
      for (int j = 0; j <= MR; ++j) ko[j] = (I)__ldg(rv.kmer_off + min(r + j, n_reads));
#pragma unroll
      for (int j = 0; j < MR; ++j) {
        const I rr = min(r + j, n_reads);
        st[j] = (rr ? (I)__ldg(rv.ends + rr - 1) : base) - base;
      }
      if (ko[1] > c0 || r + 1 >= n_reads) break;
      // forward to the chunk's first read (tiles that do not divide chunks)
      while (r + 1 < n_reads && (I)__ldg(rv.kmer_off + r + 1) <= c0) ++r;
    }
    I slot[PER], pos[PER];
    // this lane's PER consecutive slots; when they lie in one read their
    // chars come from one window of three packed words
    const I s0 = c0 + lane * (I)PER;
    bool one_read = false;
    {
      int j = 0;
#pragma unroll
      for (int q = 1; q < MR; ++q) j += ko[q] <= s0 ? 1 : 0;
      I kend = ko[MR];
#pragma unroll
      for (int q = 1; q < MR; ++q)
        if (q == j + 1) kend = ko[q];
      one_read = ko[MR] > s0 && s0 + (I)PER <= kend && s0 + (I)PER <= n_kmers;
    }
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      slot[t] = s0 + (I)t;
      pos[t] = 0;
      if (slot[t] >= n_kmers) continue;
      if (one_read && t > 0) {
        pos[t] = pos[0] + (I)t;
        continue;
      }
      int j = 0;
#pragma unroll
      for (int q = 1; q < MR; ++q) j += ko[q] <= slot[t] ? 1 : 0;
      if (ko[MR] <= slot[t]) {  // beyond the loaded reads: walk on (short reads)
        I rr = r + MR;
        while ((I)__ldg(rv.kmer_off + rr + 1) <= slot[t]) ++rr;
        pos[t] = (I)__ldg(rv.ends + rr - 1) - base + (slot[t] - (I)__ldg(rv.kmer_off + rr));
      } else {
        I ko_j = ko[0], st_j = st[0];
#pragma unroll
        for (int q = 1; q < MR; ++q)
          if (q == j) {
            ko_j = ko[q];
            st_j = st[q];
          }
        pos[t] = st_j + (slot[t] - ko_j);
      }
    }
    uint64_t key[PER], z[PER], fw[PER];
    uint32_t state[PER];  // 0 none, 1 invalid, 2 filter
    if (one_read) {  // one window: words pos0 >> 5 .. + 2
      const I wi = pos[0] >> 5;
      const uint64_t p0 = __ldg(rv.packed + wi), p1 = __ldg(rv.packed + wi + 1),
                     p2 = __ldg(rv.packed + wi + 2);
      const uint32_t i0 = __ldg(rv.invalid + wi), i1 = __ldg(rv.invalid + wi + 1),
                     i2 = __ldg(rv.invalid + wi + 2);
      const uint32_t off0 = pos[0] & 31;
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const uint32_t o = off0 + t;  // < 32 + PER
        const bool hi = o >= 32;
        const uint32_t oo = o & 31;
        const uint64_t a = hi ? p1 : p0, b = hi ? p2 : p1;
        const uint64_t iw = hi ? ((uint64_t)i1 | ((uint64_t)i2 << 32))
                               : ((uint64_t)i0 | ((uint64_t)i1 << 32));
        const uint64_t v = oo ? (a << (2 * oo)) | (b >> (64 - 2 * oo)) : a;
        state[t] = ((iw >> oo) & low_mask(k)) ? 1u : 2u;
        key[t] = state[t] == 2 ? v >> (64 - 2 * k) : 0;
      }
    } else {
      // chars and invalid bits of every k-mer of the lane
      uint64_t w0[PER], w1[PER], inv[PER];
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const I wi = pos[t] >> 5;
        const bool in = slot[t] < n_kmers;
        w0[t] = in ? __ldg(rv.packed + wi) : 0;
        w1[t] = in ? __ldg(rv.packed + wi + 1) : 0;
        inv[t] = in ? ((uint64_t)__ldg(rv.invalid + wi) |
                       ((uint64_t)__ldg(rv.invalid + wi + 1) << 32))
                    : 0;
      }
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        const uint32_t off = pos[t] & 31;
        key[t] = 0;
        state[t] = slot[t] >= n_kmers ? 0u : (((inv[t] >> off) & low_mask(k)) ? 1u : 2u);
        const uint64_t v = off ? (w0[t] << (2 * off)) | (w1[t] >> (64 - 2 * off)) : w0[t];
        if (state[t] == 2) key[t] = v >> (64 - 2 * k);
      }
    }
    // filter words, all issued before any is used
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      fw[t] = 0;
      z[t] = 0;
      if (state[t] == 2) {
        z[t] = kmer_mix(key[t]);
        fw[t] = load_u64_nc(s.kmer_filter + kmer_filter_word(z[t], s.filter_words));
      }
    }
    uint64_t res[PER];
    bool look[PER];
    I hs[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      res[t] = state[t] == 1 ? (uint64_t)SBWT_INVALID : (uint64_t)SBWT_NOT_FOUND;
      const uint64_t bits = kmer_filter_bits(z[t]);
      look[t] = state[t] == 2 && (fw[t] & bits) == bits;
      hs[t] = look[t] ? (I)kmer_table_slot(z[t], s.kmer_table_mask) : 0;
      if (COUNT) {
        n_filter += state[t] == 2;
        n_known += state[t] == 1;
      }
    }
    // table probes of the keys the filter passed, one round of loads at a time
    while (true) {
      bool any = false;
      Block A[PER];
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        A[t] = Block{0, 0, 0, 0};
        if (look[t]) {
          A[t] = load_block_hint(
              reinterpret_cast<const Block *>(s.kmer_table + 2 * (uint64_t)hs[t]), pol_table);
          any = true;
        }
      }
      if (!any) break;
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        if (!look[t]) continue;
        if (COUNT) ++n_table;
        if (A[t].w0 == key[t]) {
          res[t] = A[t].w1;
          look[t] = false;
        } else if (A[t].w2 == key[t]) {
          res[t] = A[t].w3;
          look[t] = false;
        } else if (A[t].w0 == ~0ULL || A[t].w2 == ~0ULL) {
          look[t] = false;  // an empty slot: absent
        } else {
          hs[t] = (I)(((uint64_t)hs[t] + 2) & s.kmer_table_mask);
        }
      }
    }
    if (PER == 4 && !rv.out32 && s0 + 4 <= n_kmers && s0 + 4 <= out_cap &&
        ((uintptr_t)(rv.out + s0) & 31) == 0) {
      store_sector_cs(rv.out + s0, res[0], res[1], res[PER > 2 ? 2 : 0], res[PER > 3 ? 3 : 0]);
    } else {
#pragma unroll
      for (int t = 0; t < PER; ++t) {
        if (slot[t] >= n_kmers || slot[t] >= out_cap) continue;
        if (rv.out32)
          __stcs(rv.out32 + slot[t], (unsigned int)res[t]);
        else
          __stcs(rv.out + slot[t], (unsigned long long)res[t]);
      }
    }
  }
  if (COUNT) {
    atomicAdd(counters + 0, (unsigned long long)n_table);
    atomicAdd(counters + 3, (unsigned long long)n_filter);
    atomicAdd(counters + 6, (unsigned long long)n_known);
    atomicAdd(counters + 9, (unsigned long long)n_filter);   // filter words
    atomicAdd(counters + 12, (unsigned long long)n_table);   // table lookups
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
// Optional instrumentation (off by default): CUDA-event time of every search
// kernel launch on its own stream, a count of this library's kernel
// launches, and (count mode) the work counters of the read search kernel.
struct Profile {
  std::mutex mu;
  bool enabled = false;
  bool count = false;
  double search_ms = 0;
  uint64_t search_launches = 0;
  uint64_t launches = 0;
  uint64_t counters[16] = {};
  DeviceBuffer d_counters;
};
static Profile &profile() {
  static Profile p;
  return p;
}
static void note_launches(uint64_t n) {
  Profile &p = profile();
  if (!p.enabled) return;
  std::lock_guard<std::mutex> g(p.mu);
  p.launches += n;
}

// Launch attributes of a search kernel: the persisting L2 window over the
// index's hot data when the device supports one.
struct LaunchAttrs {
  cudaLaunchAttribute attr[1];
  unsigned n = 0;
};
static LaunchAttrs search_attrs(const void *hot, u64 window_bytes, u64 persist_bytes) {
  LaunchAttrs a;
  if (hot && window_bytes && persist_bytes) {
    a.attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
    a.attr[0].val.accessPolicyWindow.base_ptr = const_cast<void *>(hot);
    a.attr[0].val.accessPolicyWindow.num_bytes = window_bytes;
    a.attr[0].val.accessPolicyWindow.hitRatio =
        (float)std::min(1.0, (double)persist_bytes / (double)window_bytes);
    a.attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    a.attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    a.n = 1;
  }
  return a;
}

template <class... KArgs, class... Args>
static void launch_ex(void (*kernel)(KArgs...), int grid, int threads, cudaStream_t st,
                      const LaunchAttrs &la, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cfg.attrs = const_cast<cudaLaunchAttribute *>(la.attr);
  cfg.numAttrs = la.n;
  SBWT_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
}

static int sm_count(int dev);

// launch_ex with the grid capped at one wave of resident blocks: for kernels
// that split their work statically over the grid (the k-mers kernels), a
// partial last wave would leave most SMs idle at the end.
template <typename... KArgs, typename... Args>
static void launch_one_wave(void (*kernel)(KArgs...), int grid, int threads, cudaStream_t st,
                            const LaunchAttrs &la, Args... args) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> per_sm;  // resident blocks per SM
  int nb = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = per_sm.find({(const void *)kernel, threads});
    if (it != per_sm.end()) {
      nb = it->second;
    } else {
      SBWT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, 0));
      per_sm[{(const void *)kernel, threads}] = nb;
    }
  }
  int dev = 0;
  SBWT_CUDA(cudaGetDevice(&dev));
  const int wave = std::max(1, nb) * sm_count(dev);
  launch_ex(kernel, std::min(grid, wave), threads, st, la, args...);
}

// kernel_mode: 0 = the general kernel; 1 = the table kernel; 2..5 = the
// walks kernel with (walks per lane, blocks per SM) = (1, 5), (2, 4), (2, 3),
// (4, 2) (the table kernel when the index has no k-mer filter); 6 = the
// k-mers kernel; 7 = 11 when the table and filter are small, else 17; 8, 9 =
// the walks kernel without filter and staging, 1 or 2 walks per lane; 10 =
// the same with the filter in front of the table, one k-mer at a time; 11,
// 12 = the k-mers kernel with 2 or 8 k-mers per lane (6: 4); 13, 14 = the
// lean walks kernel (1 walk) with staged stores, without and with the
// one-k-mer filter; 15 = the k-mers kernel with consecutive slots per lane;
// 16, 17 = 13 staging 8 or 16 slots per store group; 18 = 14 staging 16;
// 19 = 6 without the filter.
// Results never depend on it.
// Whether launch_search_kernel runs the walks kernel (the only one that can
// write 32-bit results, ReadsView::out32).
static bool walks_kernel_applies(const SbwtView &sv, const ReadsView &rv, bool stream,
                                 uint32_t mtk, uint32_t kernel_mode) {
  const bool narrow = sv.num_bits < kNarrowLimit && rv.n_kmers_bound < (1ULL << 32);
  return kernel_mode >= 2 && stream && narrow && sv.kmer_table && sv.kmer_filter &&
         sv.k <= 31 && mtk == 0 && sv.suffix_group_starts;
}

// The k-mers kernel (modes 6, 11) has the walks kernel's conditions.  Mode 7
// (automatic, the default) picks it, with 2 k-mers per lane (mode 11: 51
// registers, 5 blocks per SM; faster than 4 per lane at 3 blocks), when the
// table and filter fit kKmersKernelMaxBytes (they then stay in L2 and inside
// the translation reach, and independent lookups beat the chained stream
// steps), else the
// lean walks kernel with 16 staged slots per store group (mode 17: a large
// table, where the stream steps' rank blocks are the smaller random working
// set, a table lookup costs about what a filter probe does, and the staged
// 64-byte result stores spare the DRAM the partial writes of the table
// kernel's 8-byte stores).  Where the walks kernel does not apply, mode 17
// runs the table kernel.
constexpr u64 kKmersKernelMaxBytes = 256ULL << 20;
static uint32_t resolve_kernel_mode(const SbwtView &sv, uint32_t kernel_mode) {
  if (kernel_mode != 7) return kernel_mode;
  const u64 bytes = (sv.kmer_table_mask + 1) * 16 + sv.filter_words * 8;
  return sv.kmer_table && sv.kmer_filter && bytes <= kKmersKernelMaxBytes ? 11u : 17u;
}

// instrument = false keeps the launch free of the profiler's events and
// counter buffer (the allocation-free entry point).
static void launch_search_kernel(bool stream, const SbwtView &sv, const ReadsView &rv,
                                 const uint64_t *tile_read, uint32_t mtk, uint32_t *d_err,
                                 int grid, int threads, cudaStream_t st,
                                 const LaunchAttrs &la, uint32_t kernel_mode,
                                 bool instrument = true) {
  Profile &p = profile();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(st, &cap);
  const bool timed = instrument && p.enabled && cap == cudaStreamCaptureStatusNone;
  if (timed) {
    SBWT_CUDA(cudaEventCreate(&e0));
    SBWT_CUDA(cudaEventCreate(&e1));
    SBWT_CUDA(cudaEventRecord(e0, st));
  }
  unsigned long long *ctr = nullptr;
  if (timed && p.count) {
    std::lock_guard<std::mutex> g(p.mu);
    if (p.d_counters.size() == 0) {
      p.d_counters.resize(128);
      SBWT_CUDA(cudaMemset(p.d_counters.get(), 0, 128));
    }
    ctr = p.d_counters.get<unsigned long long>();
  }
  const bool small = sv.k <= 33;
  const bool narrow = sv.num_bits < kNarrowLimit && rv.n_kmers_bound < (1ULL << 32);
  const bool table = kernel_mode != 0 && stream && narrow && sv.kmer_table && sv.k <= 31 &&
                     mtk == 0 && sv.suffix_group_starts;
  kernel_mode = resolve_kernel_mode(sv, kernel_mode);
  const bool walks = walks_kernel_applies(sv, rv, stream, mtk, kernel_mode);
  if (rv.out32 && !walks)
    throw Error(SBWT_E_INVALID, "32-bit results need the walks kernel");
#define SBWT_LAUNCH(S_, C_, K_)                                                          \
  do {                                                                                   \
    if (narrow)                                                                          \
      launch_ex(search_reads_kernel<S_, C_, K_, uint32_t>, grid, threads, st, la, sv, rv, \
                tile_read, mtk, d_err, ctr);                                             \
    else                                                                                 \
      launch_ex(search_reads_kernel<S_, C_, K_, uint64_t>, grid, threads, st, la, sv, rv, \
                tile_read, mtk, d_err, ctr);                                             \
  } while (0)
  if (walks) {
#define SBWT_LEAN(W_, B_, F_)                                                              \
  do {                                                                                     \
    if (ctr)                                                                               \
      launch_ex(search_walks_kernel<W_, B_, true, true, F_>, grid, threads, st, la, sv, rv, \
                tile_read, ctr);                                                           \
    else                                                                                   \
      launch_ex(search_walks_kernel<W_, B_, false, true, F_>, grid, threads, st, la, sv,   \
                rv, tile_read, ctr);                                                       \
  } while (0)
#define SBWT_LEANS(W_, B_, F_)                                                             \
  do {                                                                                     \
    if (ctr)                                                                               \
      launch_ex(search_walks_kernel<W_, B_, true, true, F_, true>, grid, threads, st, la,  \
                sv, rv, tile_read, ctr);                                                   \
    else                                                                                   \
      launch_ex(search_walks_kernel<W_, B_, false, true, F_, true>, grid, threads, st, la, \
                sv, rv, tile_read, ctr);                                                   \
  } while (0)
#define SBWT_LEANSG(W_, B_, F_, G_)                                                        \
  do {                                                                                     \
    if (ctr)                                                                               \
      launch_ex(search_walks_kernel<W_, B_, true, true, F_, true, G_>, grid, threads, st,  \
                la, sv, rv, tile_read, ctr);                                               \
    else                                                                                   \
      launch_ex(search_walks_kernel<W_, B_, false, true, F_, true, G_>, grid, threads, st, \
                la, sv, rv, tile_read, ctr);                                               \
  } while (0)
#define SBWT_WALKS(W_, B_)                                                                 \
  do {                                                                                     \
    if (ctr)                                                                               \
      launch_ex(search_walks_kernel<W_, B_, true>, grid, threads, st, la, sv, rv, tile_read, \
                ctr);                                                                      \
    else                                                                                   \
      launch_ex(search_walks_kernel<W_, B_, false>, grid, threads, st, la, sv, rv, tile_read, \
                ctr);                                                                      \
  } while (0)
    if (kernel_mode == 2) SBWT_WALKS(1, 5);
    else if (kernel_mode == 3) SBWT_WALKS(2, 4);
    else if (kernel_mode == 4) SBWT_WALKS(2, 3);
    else if (kernel_mode == 5) SBWT_WALKS(4, 2);
    else if (kernel_mode == 8) SBWT_LEAN(1, 5, false);
    else if (kernel_mode == 9) SBWT_LEAN(2, 3, false);
    else if (kernel_mode == 10) SBWT_LEAN(1, 5, true);
    else if (kernel_mode == 15 && ctr)
      launch_one_wave(search_kmers_seq_kernel<4, true>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 15)
      launch_one_wave(search_kmers_seq_kernel<4, false>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 13) SBWT_LEANS(1, 5, false);
    else if (kernel_mode == 16) SBWT_LEANSG(1, 5, false, 8);
    else if (kernel_mode == 17 && sv.k == 31 && ctr)
      launch_ex(search_walks_kernel<1, 6, true, true, false, true, 16, 31>, grid, threads, st,
                la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 17 && sv.k == 31)
      launch_ex(search_walks_kernel<1, 6, false, true, false, true, 16, 31>, grid, threads, st,
                la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 17) SBWT_LEANSG(1, 6, false, 16);
    else if (kernel_mode == 18) SBWT_LEANSG(1, 5, true, 16);
    else if (kernel_mode == 14) SBWT_LEANS(1, 5, true);
    else if (kernel_mode == 11 && sv.k == 31 && ctr)
      launch_one_wave(search_kmers_kernel<2, true, true, 31>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 11 && sv.k == 31)
      launch_one_wave(search_kmers_kernel<2, false, true, 31>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 11 && ctr)
      launch_one_wave(search_kmers_kernel<2, true>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 11)
      launch_one_wave(search_kmers_kernel<2, false>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 19 && ctr)
      launch_one_wave(search_kmers_kernel<4, true, false>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 19)
      launch_one_wave(search_kmers_kernel<4, false, false>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 12 && ctr)
      launch_one_wave(search_kmers_kernel<8, true>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (kernel_mode == 12)
      launch_one_wave(search_kmers_kernel<8, false>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else if (ctr)
      launch_one_wave(search_kmers_kernel<4, true>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
    else
      launch_one_wave(search_kmers_kernel<4, false>,
                      grid, threads, st, la, sv, rv, tile_read, ctr);
#undef SBWT_WALKS
#undef SBWT_LEAN
#undef SBWT_LEANS
#undef SBWT_LEANSG
  } else if (table) {
    if (ctr)
      launch_ex(search_table_kernel<true>, grid, threads, st, la, sv, rv, tile_read, ctr);
    else
      launch_ex(search_table_kernel<false>, grid, threads, st, la, sv, rv, tile_read, ctr);
  } else if (ctr) {
    if (stream) {
      if (small) SBWT_LAUNCH(true, true, true); else SBWT_LAUNCH(true, true, false);
    } else {
      if (small) SBWT_LAUNCH(false, true, true); else SBWT_LAUNCH(false, true, false);
    }
  } else {
    if (stream) {
      if (small) SBWT_LAUNCH(true, false, true); else SBWT_LAUNCH(true, false, false);
    } else {
      if (small) SBWT_LAUNCH(false, false, true); else SBWT_LAUNCH(false, false, false);
    }
  }
#undef SBWT_LAUNCH
  SBWT_CUDA(cudaGetLastError());
  if (timed) {
    SBWT_CUDA(cudaEventRecord(e1, st));
    SBWT_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SBWT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> g(p.mu);
    p.search_ms += ms;
    p.search_launches += 1;
    p.launches += 1;
  }
}
static int sm_count(int dev) {
  int n = 148;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

// Builds the rank blocks of one bitvector (host), see device_layout.hpp.
void build_rank_blocks_host(const u64 *words, u64 num_bits,
                              std::vector<Block> &blocks, std::vector<u64> &l0,
                              u64 &total) {
  const u64 nb = num_bits / kBlockBits + 1;
  const u64 nw = (num_bits + 63) / 64;
  blocks.assign(nb, Block{0, 0, 0, 0});
  l0.assign((nb >> kSuperchunkShift) + 1, 0);
  auto get64 = [&](u64 bit) -> u64 {  // 64 bits from position `bit`, 0 past end
    u64 w = bit / 64, o = bit % 64;
    u64 a = w < nw ? words[w] : 0;
    u64 v = a >> o;
    if (o) {
      u64 b = (w + 1) < nw ? words[w + 1] : 0;
      v |= b << (64 - o);
    }
    return v;
  };
  auto clip = [&](u64 v, u64 bit0, u64 nbits) -> u64 {  // zero bits >= num_bits
    if (bit0 >= num_bits) return 0;
    u64 avail = num_bits - bit0;
    if (avail >= nbits) return v;
    return v & ((1ULL << avail) - 1);
  };
  u64 ones = 0, chunk_base = 0;
  for (u64 b = 0; b < nb; ++b) {
    if ((b & ((1ULL << kSuperchunkShift) - 1)) == 0) {
      l0[b >> kSuperchunkShift] = ones;
      chunk_base = ones;
    }
    const u64 s = b * kBlockBits;
    const u64 p0 = clip(get64(s), s, 64);
    const u64 p1 = clip(get64(s + 64), s + 64, 64);
    const u64 p2 = clip(get64(s + 128), s + 128, 64);
    const u64 c0 = __builtin_popcountll(p0), c1 = __builtin_popcountll(p1);
    Block &B = blocks[b];
    B.w0 = p0;
    B.w1 = p1;
    B.w2 = p2;
    B.w3 = ((ones - chunk_base) & 0xFFFFFFFFULL) | (c0 << 40) | ((c0 + c1) << 48);
    ones += c0 + c1 + __builtin_popcountll(p2);
  }
  total = ones;
}

IndexImpl::IndexImpl(const u64 *const acgt[4], u64 num_bits_, u32 k_,
                     const u64 *sg, const u64 *key_marks, int device_,
                     unsigned presearch_letters) {
  if (num_bits_ == 0) throw Error(SBWT_E_INVALID, "empty SBWT");
  if (num_bits_ >= (1ULL << 37))
    throw Error(SBWT_E_INVALID, "SBWTs of 2^37 or more nodes are not supported");
  if (k_ == 0) throw Error(SBWT_E_INVALID, "k must be positive");
  device = device_;
  DeviceGuard g(device);
  num_bits = num_bits_;
  k = k_;
  // default depth: 14 for large SBWTs (each extra letter replaces a search
  // step), the reference's 12 for small ones (whose deeper tables would only
  // move lookups from L2 to DRAM)
  p_max = presearch_letters ? presearch_letters
                            : (num_bits_ >= (1ULL << 26) ? kPresearchMaxLetters : 12u);
  if (p_max > kPresearchMaxLetters)
    throw Error(SBWT_E_INVALID, "presearch_letters must be <= 14");
  if (p_max > k) p_max = k;
  wide = num_bits >= (1ULL << 32) ? 1 : 0;
  // rank blocks, one host thread per vector
  std::vector<Block> hb[4];
  std::vector<u64> hl0[4];
  u64 totals[4];
  {
    std::vector<std::thread> th;
    for (int c = 0; c < 4; ++c)
      th.emplace_back([&, c] { build_rank_blocks_host(acgt[c], num_bits, hb[c], hl0[c], totals[c]); });
    for (auto &t : th) t.join();
  }
  view = SbwtView{};
  c_map[0] = 1;
  for (int c = 0; c < 4; ++c) c_map[c + 1] = c_map[c] + totals[c];
  for (int c = 0; c < 5; ++c) view.c_map[c] = c_map[c];
  // The rank blocks of A/C/G/T and the suffix-group-start words share one
  // allocation ("hot" data of every search step), so one L2 access-policy
  // window can keep them resident.
  const u64 nw = (num_bits + 63) / 64;
  u64 off[5];
  u64 hot_bytes = 0;
  for (int c = 0; c < 4; ++c) {
    off[c] = hot_bytes;
    hot_bytes += ((hb[c].size() * sizeof(Block) + 255) / 256) * 256;
  }
  off[4] = hot_bytes;
  if (sg) hot_bytes += (((nw + 8) * 8 + 255) / 256) * 256;
  hot.resize(hot_bytes);
  SBWT_CUDA(cudaMemset(hot.get(), 0, hot_bytes));
  unsigned char *hp = hot.get<unsigned char>();
  const u64 n_l0 = hl0[0].size();
  l0_all.resize(4 * n_l0 * 8);
  for (int c = 0; c < 4; ++c) {
    SBWT_CUDA(cudaMemcpy(hp + off[c], hb[c].data(), hb[c].size() * sizeof(Block),
                         cudaMemcpyHostToDevice));
    SBWT_CUDA(cudaMemcpy(l0_all.get<u64>() + c * n_l0, hl0[c].data(), n_l0 * 8,
                         cudaMemcpyHostToDevice));
    view.blocks[c] = reinterpret_cast<const Block *>(hp + off[c]);
    view.l0[c] = l0_all.get<u64>() + c * n_l0;
  }
  view.blocks0 = reinterpret_cast<const Block *>(hp);
  view.block_stride = off[1] / sizeof(Block);
  view.l00 = l0_all.get<u64>();
  view.l0_stride = n_l0;
  if (sg) {
    SBWT_CUDA(cudaMemcpy(hp + off[4], sg, nw * 8, cudaMemcpyHostToDevice));
    view.suffix_group_starts = reinterpret_cast<const u64 *>(hp + off[4]);
  }
  // An optional persisting-L2 window over the hot data (off by default: the
  // carve-out takes L2 away from the presearch table and the streams, and
  // measured slower on the 100 Mbp workload).
  {
    int max_window = 0;
    cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, device);
    window_bytes = std::min<u64>(hot_bytes, (u64)std::max(max_window, 0));
    cudaGetLastError();
  }
  if (key_marks) {
    key_buf.resize((nw + 1) * 8);
    SBWT_CUDA(cudaMemset(key_buf.get(), 0, (nw + 1) * 8));
    SBWT_CUDA(cudaMemcpy(key_buf.get(), key_marks, nw * 8, cudaMemcpyHostToDevice));
    view.key_marks = key_buf.get<u64>();
  }
  view.num_bits = num_bits;
  view.k = k;
  view.wide = wide;
  // presearch pyramid, levels 1..p_max
  const u64 entries = presearch_level_offset(p_max + 1);
  presearch.resize(entries * 8 * (wide ? 2 : 1) + 64);
  view.presearch = presearch.get<u64>();
  view.p = p_max;
  const int sms = sm_count(device);
  for (u32 j = 1; j <= p_max; ++j) {
    const u64 n = 1ULL << (2 * j);
    const int grid = (int)std::min<u64>((n + 255) / 256, (u64)sms * 16);
    presearch_level_kernel<<<grid, 256>>>(view, presearch.get<u64>(), j);
    SBWT_CUDA(cudaGetLastError());
  }
  SBWT_CUDA(cudaDeviceSynchronize());
  build_kmer_table();
  device_bytes = presearch.size() + hot.size() + key_buf.size() + l0_all.size() +
                 kmer_table.size() + kmer_filter.size();
}

SbwtView IndexImpl::view_for(u32 p) const {
  SbwtView v = view;
  v.p = (p == 0 || p > p_max) ? p_max : p;
  return v;
}

// Per-thread, per-device scratch (device buffers, streams, pinned error word).
struct Workspace {
  int device = -1;
  cudaStream_t streams[2] = {nullptr, nullptr};
  DeviceBuffer chars[2], ends[2], kmer_off[2], packed[2], invalid[2], results[2],
      block_sums[2], total[2], tile_read[2], queue[2], positions, bits, results32[2];
  uint32_t *err_host = nullptr;  // pinned: the error word, then (at +8 bytes) a k-mer count
  DeviceBuffer err_dev;
  cudaEvent_t done[2] = {nullptr, nullptr};
  uint32_t *stage[2] = {nullptr, nullptr};  // pinned: 32-bit results of a chunk
  u64 stage_cap[2] = {0, 0};
  uint32_t *staging(int b, u64 n) {
    if (stage_cap[b] < n) {
      if (stage[b]) cudaFreeHost(stage[b]);
      stage[b] = nullptr;
      stage_cap[b] = 0;
      SBWT_CUDA(cudaHostAlloc((void **)&stage[b], n * 4, cudaHostAllocDefault));
      stage_cap[b] = n;
    }
    return stage[b];
  }
  ~Workspace() {
    if (device < 0) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (auto &s : streams)
      if (s) cudaStreamDestroy(s);
    for (auto &e : done)
      if (e) cudaEventDestroy(e);
    if (err_host) cudaFreeHost(err_host);
    for (auto *p : stage)
      if (p) cudaFreeHost(p);
    cudaSetDevice(prev);
  }
};

// 32-bit result codes -> the API's u64 values (0xFFFFFFFF -> SBWT_NOT_FOUND,
// 0xFFFFFFFE -> SBWT_INVALID), on host threads, with streaming stores (the
// caller reads the results later, not now).
static inline u64 widen_code(uint32_t x) {
  return x >= 0xFFFFFFFEu ? (0xFFFFFFFF00000000ULL | x) : (u64)x;
}
static void widen_range(const uint32_t *src, u64 *dst, u64 n) {
  u64 i = 0;
  for (; i < n && ((uintptr_t)(dst + i) & 15); ++i) dst[i] = widen_code(src[i]);
  const __m128i m1 = _mm_set1_epi32(-1), m2 = _mm_set1_epi32(-2);
  for (; i + 4 <= n; i += 4) {
    const __m128i v = _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i));
    const __m128i hi = _mm_or_si128(_mm_cmpeq_epi32(v, m1), _mm_cmpeq_epi32(v, m2));
    _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i), _mm_unpacklo_epi32(v, hi));
    _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i + 2), _mm_unpackhi_epi32(v, hi));
  }
  for (; i < n; ++i) dst[i] = widen_code(src[i]);
  _mm_sfence();
}
static void widen_results(const uint32_t *src, u64 *dst, u64 n) {
  const u64 per = 4ULL << 20;  // k-mers per thread at least
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned T = (unsigned)std::min<u64>(std::min<u64>(hw, 32), std::max<u64>(n / per, 1));
  if (T <= 1) {
    widen_range(src, dst, n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(T);
  for (unsigned t = 0; t < T; ++t) {
    const u64 a = n * t / T, b = n * (t + 1) / T;
    th.emplace_back(widen_range, src + a, dst + a, b - a);
  }
  for (auto &x : th) x.join();
}

static Workspace &workspace(int device) {
  thread_local std::map<int, std::unique_ptr<Workspace>> ws;
  auto &p = ws[device];
  if (!p) {
    p = std::make_unique<Workspace>();
    p->device = device;
    for (auto &s : p->streams)
      SBWT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    for (auto &e : p->done) SBWT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SBWT_CUDA(cudaMallocHost(&p->err_host, 16));
    p->err_dev.resize(sizeof(uint32_t));
    SBWT_CUDA(cudaMemset(p->err_dev.get(), 0, sizeof(uint32_t)));
  }
  return *p;
}

static void check_err_word(Workspace &ws, cudaStream_t st) {
  SBWT_CUDA(cudaMemcpyAsync(ws.err_host, ws.err_dev.get(), 4, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaStreamSynchronize(st));
  const uint32_t e = *ws.err_host;
  if (e) {
    *ws.err_host = 0;
    SBWT_CUDA(cudaMemset(ws.err_dev.get(), 0, 4));
    if (e & 4u)
      throw Error(SBWT_E_INVALID, "read_ends are not non-decreasing within n_chars");
    if (e & 2u)
      throw Error(SBWT_E_INVALID, "a k-mer position lies past the end of bit_seqs");
    throw Error(SBWT_E_TIMEOUT,
                "key k-mer walk did not reach a key k-mer (node without an "
                "outgoing edge); results of those k-mers are unspecified");
  }
}

static int grid_for(int dev, u64 work, int threads, int per_sm) {
  const u64 g = std::min<u64>((work + threads - 1) / threads, (u64)sm_count(dev) * per_sm);
  return (int)std::max<u64>(g, 1);
}


// Length L of the absent-prefix probe: a random L-mer is a suffix of some
// node with probability about N / 4^L, so L = ceil(log4 N) + 3 makes a probe
// of an erroneous stretch come back absent most of the time.
static uint32_t probe_length(u64 num_bits, u32 k, const LaunchConfig &cfg) {
  if (cfg.probe_len == ~0u) return 0;
  uint32_t L = cfg.probe_len;
  if (L == 0) {
    uint32_t lg = 0;
    while (lg < 32 && (1ULL << (2 * lg)) < num_bits) ++lg;
    L = lg + 3;
  }
  return L < k ? L : 0;
}

static u64 tile_size(int device, u64 n_kmers, const LaunchConfig &cfg) {
  if (cfg.tile) return cfg.tile;
  const u64 resident = (u64)sm_count(device) * cfg.blocks_per_sm * cfg.block_threads;
  u64 tile = n_kmers / (resident * 8);
  // at most 128 slots: the tiles in flight then span less of the chars and
  // results (fewer pages and DRAM rows at a time; 10 % faster than 577 on the
  // 100 Mbp workload); a multiple of 16 slots: the walks kernels store
  // groups of up to 16 staged results
  return (std::min<u64>(std::max<u64>(tile, 16), 128) + 15) & ~15ULL;
}

// Scan of per-read k-mer counts and the packing of the chars (device-resident
// inputs).  The k-mer total lands in *sc.total.
static void launch_prepare(int device, u32 k, const char *d_chars, u64 n_chars,
                           const u64 *d_ends, u64 n_reads, u64 base,
                           const ReadsScratch &sc, cudaStream_t st) {
  const u64 n_words = (n_chars + 31) / 32;
  const u64 n_scan_blocks = (n_reads + kScanTile - 1) / kScanTile;
  scan_reduce_kernel<<<(unsigned)n_scan_blocks, kScanThreads, 0, st>>>(
      d_ends, n_reads, base, k, n_chars, sc.block_sums, sc.err);
  scan_sums_kernel<<<1, kScanThreads, 0, st>>>(sc.block_sums, n_scan_blocks, sc.total,
                                               sc.err);
  scan_write_kernel<<<(unsigned)n_scan_blocks, kScanThreads, 0, st>>>(
      d_ends, n_reads, base, k, sc.block_sums, sc.kmer_off, sc.err);
  SBWT_CUDA(cudaMemsetAsync(sc.packed + n_words, 0, 16, st));
  SBWT_CUDA(cudaMemsetAsync(sc.invalid + n_words, 0, 8, st));
  if (n_words && ((uintptr_t)d_chars & 15) == 0)
    pack16_kernel<<<grid_for(device, (n_words + 1) / 2, 256, 8), 256, 0, st>>>(
        d_chars, n_chars, sc.packed, sc.invalid, n_words);
  else if (n_words)
    pack_kernel<<<grid_for(device, n_words * 32, 256, 32), 256, 0, st>>>(
        d_chars, n_chars, sc.packed, sc.invalid, n_words);
  SBWT_CUDA(cudaGetLastError());
  note_launches(n_words ? 4 : 3);
}

// Tile table + the read search kernel over a prepared batch of n_kmers.
// With d_total the kernels read the k-mer count from device memory (the
// scan's total) and n_kmers is only an upper bound, for the tiling.
static void launch_search(const IndexImpl &ix, u64 n_chars, const u64 *d_ends, u64 n_reads,
                          u64 base,
                          u64 n_kmers, u64 *d_out, u64 out_capacity, u32 flags,
                          const LaunchConfig &cfg, const ReadsScratch &sc,
                          cudaStream_t st, uint32_t *d_out32 = nullptr,
                          const u64 *d_total = nullptr) {
  if (n_reads == 0 || n_kmers == 0) return;
  ReadsView rv{};
  rv.out32 = d_out32;
  rv.n_kmers_bound = std::max<u64>(n_chars, n_reads) + 64;
  rv.packed = sc.packed;
  rv.invalid = sc.invalid;
  rv.ends = d_ends;
  rv.kmer_off = sc.kmer_off;
  rv.base = base;
  rv.n_reads = n_reads;
  rv.n_kmers = n_kmers;
  rv.tile = tile_size(ix.device, n_kmers, cfg);
  rv.n_tiles = (n_kmers + rv.tile - 1) / rv.tile;
  rv.out = d_out;
  rv.out_capacity = out_capacity;
  rv.probe_len = probe_length(ix.num_bits, ix.k, cfg);
  rv.n_kmers_dev = d_total;
  rv.queue = sc.queue;
  SBWT_CUDA(cudaMemsetAsync(sc.queue, 0, 8, st));
  tile_reads_kernel<<<grid_for(ix.device, n_reads, 256, 16), 256, 0, st>>>(
      sc.kmer_off, n_reads, rv.tile, sc.tile_read);
  SBWT_CUDA(cudaGetLastError());
  note_launches(1);
  const int threads = (int)cfg.block_threads;
  const int grid = grid_for(ix.device, rv.n_tiles, threads, cfg.blocks_per_sm);
  const SbwtView sv = ix.view_for(cfg.presearch_letters);
  const bool stream = !(flags & SBWT_PER_KMER_WALK) && ix.view.suffix_group_starts;
  const u32 mtk = (flags & SBWT_MOVE_TO_KEY_KMER) ? 1u : 0u;
  u64 persist = 0;
  if (cfg.l2_window && ix.window_bytes) {  // sets the context's persisting L2 size
    int max_persist = 0;
    cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ix.device);
    size_t cur = 0;
    cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
    const size_t want = std::min<size_t>((size_t)std::max(max_persist, 0), ix.window_bytes);
    if (want > cur) cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want);
    cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize);
    cudaGetLastError();
    persist = cur;
  }
  launch_search_kernel(stream, sv, rv, sc.tile_read, mtk, sc.err, grid, threads, st,
                       persist ? search_attrs(ix.hot.get(), ix.window_bytes, persist)
                               : LaunchAttrs{},
                       cfg.table_kernel);
}

// The index step of one device-resident batch without any host
// synchronisation (capturable in a CUDA graph): scan, pack, tile table and
// the search kernel.  The k-mer total is taken from device memory inside the
// kernel; tiles are sized from max_kmers (an upper bound, e.g. n_chars) and
// the tile table must hold max_kmers / tile + 2 entries.
void enqueue_index_step(const IndexImpl &ix, const char *d_chars, u64 n_chars,
                        const u64 *d_ends, u64 n_reads, const ReadsScratch &sc, u64 *d_out,
                        u64 out_capacity, u64 max_kmers, u32 flags, const LaunchConfig &cfg,
                        cudaStream_t st) {
  SBWT_CUDA(cudaMemsetAsync(sc.err, 0, 4, st));
  SBWT_CUDA(cudaMemsetAsync(sc.queue, 0, 8, st));
  if (n_reads == 0) {
    SBWT_CUDA(cudaMemsetAsync(sc.total, 0, 8, st));
    return;
  }
  launch_prepare(ix.device, ix.k, d_chars, n_chars, d_ends, n_reads, 0, sc, st);
  ReadsView rv{};
  rv.n_kmers_bound = std::max<u64>(n_chars, n_reads) + 64;
  rv.packed = sc.packed;
  rv.invalid = sc.invalid;
  rv.ends = d_ends;
  rv.kmer_off = sc.kmer_off;
  rv.base = 0;
  rv.n_reads = n_reads;
  rv.n_kmers = 0;
  rv.n_kmers_dev = sc.total;
  rv.tile = tile_size(ix.device, std::max<u64>(max_kmers, 1), cfg);
  rv.n_tiles = 0;  // computed on the device from the total
  rv.out = d_out;
  rv.out_capacity = out_capacity;
  rv.probe_len = probe_length(ix.num_bits, ix.k, cfg);
  rv.queue = sc.queue;
  tile_reads_kernel<<<grid_for(ix.device, n_reads, 256, 16), 256, 0, st>>>(
      sc.kmer_off, n_reads, rv.tile, sc.tile_read);
  const int grid = (int)((u64)sm_count(ix.device) * cfg.blocks_per_sm);
  const SbwtView sv = ix.view_for(cfg.presearch_letters);
  const bool stream = !(flags & SBWT_PER_KMER_WALK) && ix.view.suffix_group_starts;
  const u32 mtk = (flags & SBWT_MOVE_TO_KEY_KMER) ? 1u : 0u;
  launch_search_kernel(stream, sv, rv, sc.tile_read, mtk, sc.err, grid,
                       (int)cfg.block_threads, st, LaunchAttrs{}, cfg.table_kernel);
  note_launches(1);
}

u64 index_tile_size(const IndexImpl &ix, u64 max_kmers, const LaunchConfig &cfg) {
  return tile_size(ix.device, std::max<u64>(max_kmers, 1), cfg);
}

// Grows the workspace buffers of slot b for a batch and returns raw pointers.
static ReadsScratch scratch_for(Workspace &ws, int b, u64 n_chars, u64 n_reads,
                                u64 n_kmers_max, u64 tile_min) {
  const u64 n_words = (n_chars + 31) / 32;
  ws.kmer_off[b].ensure((n_reads + 1) * 8);
  ws.packed[b].ensure((n_words + 2) * 8);
  ws.invalid[b].ensure((n_words + 2) * 4);
  ws.block_sums[b].ensure(((n_reads + kScanTile - 1) / kScanTile + 1) * 8);
  ws.total[b].ensure(8);
  ws.tile_read[b].ensure((n_kmers_max / tile_min + 2) * 8);
  ws.queue[b].ensure(8);
  return ReadsScratch{ws.kmer_off[b].get<u64>(), ws.packed[b].get<u64>(),
                      ws.invalid[b].get<uint32_t>(), ws.block_sums[b].get<u64>(),
                      ws.total[b].get<u64>(), ws.tile_read[b].get<u64>(),
                      ws.err_dev.get<uint32_t>(),
                      ws.queue[b].get<unsigned long long>()};
}

u64 count_kmers_host(const u64 *ends, u64 n_reads, u32 k, u64 base) {
  u64 n = 0, prev = base;
  for (u64 r = 0; r < n_reads; ++r) {
    if (ends[r] < prev) throw Error(SBWT_E_INVALID, "read_ends must be non-decreasing");
    const u64 len = ends[r] - prev;
    if (len >= k) n += len - k + 1;
    prev = ends[r];
  }
  return n;
}

void IndexImpl::search_reads_device_pieces(const char *chars, u64 n_chars,
                                           const u64 *read_ends, u64 n_reads, u64 *results,
                                           u64 capacity, u64 *n_results, u32 flags,
                                           cudaStream_t st, const LaunchConfig &cfg) const {
  Workspace &ws = workspace(device);
  // an explicit chunk size (a tuning and testing hook) sets the piece size
  const u64 kPieceChars = cfg.chunk_chars ? std::min<u64>(cfg.chunk_chars, 1ULL << 31)
                                          : (1ULL << 31);
  DeviceBuffer bound(16);
  u64 r0 = 0, c0 = 0, k_acc = 0;
  bool over = false;
  while (r0 < n_reads) {
    u64 hb[2] = {0, 0};
    ends_upper_bound_kernel<<<1, 32, 0, st>>>(read_ends, r0, n_reads, c0 + kPieceChars,
                                              bound.get<u64>());
    SBWT_CUDA(cudaGetLastError());
    SBWT_CUDA(cudaMemcpyAsync(hb, bound.get(), 16, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
    u64 r1 = hb[0], c1 = hb[1];
    if (r1 == r0) {  // one read longer than a piece: it is a piece of its own
      r1 = r0 + 1;
      SBWT_CUDA(cudaMemcpy(&c1, read_ends + r0, 8, cudaMemcpyDeviceToHost));
    }
    if (c1 < c0 || c1 > n_chars)
      throw Error(SBWT_E_INVALID, "read_ends are not non-decreasing within n_chars");
    const u64 nc = c1 - c0, nr = r1 - r0;
    const ReadsScratch sc = scratch_for(ws, 0, nc, nr, nc, 16);
    launch_prepare(device, k, chars + c0, nc, read_ends + r0, nr, c0, sc, st);
    u64 n_k = 0;
    SBWT_CUDA(cudaMemcpyAsync(&n_k, sc.total, 8, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
    check_err_word(ws, st);
    if (k_acc + n_k > capacity) over = true;
    if (!over)
      launch_search(*this, nc, read_ends + r0, nr, c0, n_k, results + k_acc,
                    capacity - k_acc, flags, cfg, sc, st);
    k_acc += n_k;
    r0 = r1;
    c0 = c1;
  }
  check_err_word(ws, st);
  if (n_results) *n_results = k_acc;
  if (over) throw Error(SBWT_E_CAPACITY, "results_capacity smaller than the k-mer count");
}

u32 IndexImpl::host_result_bytes(const LaunchConfig &cfg) const {
  ReadsView probe{};
  probe.n_kmers_bound = (64ULL << 20) + 64;
  const SbwtView sv = view_for(cfg.presearch_letters);
  return walks_kernel_applies(sv, probe, view.suffix_group_starts != nullptr, 0,
                              resolve_kernel_mode(sv, cfg.table_kernel))
             ? 4u
             : 8u;
}

void IndexImpl::search_reads(const char *chars, u64 n_chars, const u64 *read_ends,
                             u64 n_reads, u64 *results, u64 capacity,
                             u64 *n_results, u32 flags, cudaStream_t user_stream,
                             const LaunchConfig &cfg) const {
  DeviceGuard g(device);
  Workspace &ws = workspace(device);
  if (flags & SBWT_DEVICE_POINTERS) {
    // The 32-bit kernels index chars and k-mer slots of one launch in 32
    // bits: a batch of 2^32 or more chars on an index they serve runs as
    // consecutive launches of at most 2^31 chars each (whole reads).
    if (num_bits < kNarrowLimit && n_reads &&
        (n_chars + 64 >= (1ULL << 32) || (cfg.chunk_chars && n_chars > cfg.chunk_chars))) {
      search_reads_device_pieces(chars, n_chars, read_ends, n_reads, results, capacity,
                                 n_results, flags, user_stream, cfg);
      return;
    }
    // everything resident; the k-mer count (needed for the tiling and the
    // capacity check) comes from the device scan
    u64 n_k = 0;
    if (n_reads) {
      // k-mers <= chars, so a tile table sized for n_chars is always enough
      const ReadsScratch sc = scratch_for(ws, 0, n_chars, n_reads, n_chars, 16);
      // scan, packing, tile table and search queued back to back: the search
      // reads the k-mer count from the scan's total (a batch with bad read
      // ends has a total of 0), tiles are sized for n_chars (>= the count),
      // and no kernel writes at or past `capacity`.  The count and the error
      // word come back under one synchronisation (check_err_word's).
      launch_prepare(device, k, chars, n_chars, read_ends, n_reads, 0, sc, user_stream);
      launch_search(*this, n_chars, read_ends, n_reads, 0, n_chars, results, capacity, flags,
                    cfg, sc, user_stream, nullptr, sc.total);
      u64 *const total_host = reinterpret_cast<u64 *>(ws.err_host + 2);
      SBWT_CUDA(cudaMemcpyAsync(total_host, sc.total, 8, cudaMemcpyDeviceToHost, user_stream));
      check_err_word(ws, user_stream);
      n_k = *total_host;
      if (n_results) *n_results = n_k;
      if (n_k > capacity)
        throw Error(SBWT_E_CAPACITY, "results_capacity smaller than the k-mer count");
    } else if (n_results) {
      *n_results = 0;
    }
    return;
  }
  // host pointers: chunk the reads, double-buffer, overlap H2D/compute/D2H.
  // Each chunk is planned (its last read by binary search over the cumulative
  // ends, its k-mers and the ends' order checked over its own reads) while the
  // previous one is on the GPU, and its results are only copied back once
  // they fit the capacity.
  // A pinned results buffer receives u64 results by DMA.  A pageable one
  // would take them through the driver's staging copies; with the walks or
  // k-mers kernel the results of a chunk then cross PCIe as 32-bit codes into
  // a pinned staging buffer instead and are widened to u64 on host threads
  // while the next chunk runs (half the device-to-host bytes).
  const u64 chunk_chars = cfg.chunk_chars ? cfg.chunk_chars : (64ULL << 20);
  const bool pinned_in = is_host_pinned(chars) && is_host_pinned(read_ends);
  const bool pinned = pinned_in && is_host_pinned(results);
  const SbwtView sv_host = view_for(cfg.presearch_letters);
  const bool stream_host = !(flags & SBWT_PER_KMER_WALK) && view.suffix_group_starts;
  const u32 mtk_host = (flags & SBWT_MOVE_TO_KEY_KMER) ? 1u : 0u;
  struct Pending {
    int b = -1;
    u64 at = 0, n = 0;
  } pend;
  auto drain = [&]() {  // widens the chunk whose 32-bit results are in flight
    if (pend.b < 0) return;
    SBWT_CUDA(cudaEventSynchronize(ws.done[pend.b]));
    widen_results(ws.stage[pend.b], results + pend.at, pend.n);
    pend.b = -1;
  };
  u64 r = 0, kacc = 0, prev_end = 0;
  bool over = false, unordered = false;
  for (size_t i = 0; r < n_reads; ++i) {
    const u64 r0 = r, c0 = prev_end;
    u64 r1 = (u64)(std::upper_bound(read_ends + r0, read_ends + n_reads, c0 + chunk_chars) -
                   read_ends);
    r1 = std::max(r1, r0 + 1);
    u64 nk = 0, prev = c0;
    for (u64 q = r0; q < r1 && !unordered; ++q) {
      unordered = read_ends[q] < prev;
      const u64 len = read_ends[q] - prev;
      if (len >= k) nk += len - k + 1;
      prev = read_ends[q];
    }
    if (unordered) break;  // reported once the chunks in flight are done
    if (kacc + nk > capacity) {
      over = true;
      break;
    }
    const int b = (int)(i & 1);
    cudaStream_t st = ws.streams[b];
    const u64 nc = prev - c0, nr = r1 - r0;
    ReadsView probe{};
    probe.n_kmers_bound = std::max<u64>(nc, nr) + 64;
    const bool narrow = !pinned && walks_kernel_applies(sv_host, probe, stream_host, mtk_host,
                                                        resolve_kernel_mode(sv_host,
                                                                            cfg.table_kernel));
    ws.chars[b].ensure(nc + 16);
    ws.ends[b].ensure(nr * 8);
    if (narrow)
      ws.results32[b].ensure(std::max<u64>(nk, 1) * 4);
    else
      ws.results[b].ensure(std::max<u64>(nk, 1) * 8);
    const ReadsScratch sc = scratch_for(ws, b, nc, nr, nk, tile_size(device, nk, cfg));
    SBWT_CUDA(cudaMemcpyAsync(ws.chars[b].get(), chars + c0, nc, cudaMemcpyHostToDevice, st));
    SBWT_CUDA(cudaMemcpyAsync(ws.ends[b].get(), read_ends + r0, nr * 8,
                              cudaMemcpyHostToDevice, st));
    launch_prepare(device, k, ws.chars[b].get<char>(), nc, ws.ends[b].get<u64>(), nr, c0, sc,
                   st);
    if (narrow) {
      uint32_t *stage = ws.staging(b, std::max<u64>(nk, 1));
      launch_search(*this, nc, ws.ends[b].get<u64>(), nr, c0, nk, nullptr, nk, flags, cfg, sc,
                    st, ws.results32[b].get<uint32_t>());
      if (nk)
        SBWT_CUDA(cudaMemcpyAsync(stage, ws.results32[b].get(), nk * 4,
                                  cudaMemcpyDeviceToHost, st));
      SBWT_CUDA(cudaEventRecord(ws.done[b], st));
      drain();  // the previous chunk, while this one runs
      pend.b = b;
      pend.at = kacc;
      pend.n = nk;
      if (!pinned_in) drain();
    } else {
      drain();
      launch_search(*this, nc, ws.ends[b].get<u64>(), nr, c0, nk, ws.results[b].get<u64>(), nk,
                    flags, cfg, sc, st);
      if (nk)
        SBWT_CUDA(cudaMemcpyAsync(results + kacc, ws.results[b].get(), nk * 8,
                                  cudaMemcpyDeviceToHost, st));
      if (!pinned) SBWT_CUDA(cudaStreamSynchronize(st));
    }
    kacc += nk;
    r = r1;
    prev_end = prev;
  }
  drain();
  for (auto &s : ws.streams) SBWT_CUDA(cudaStreamSynchronize(s));
  if (unordered) throw Error(SBWT_E_INVALID, "read ends must be non-decreasing");
  if (over) {
    const u64 total_k = count_kmers_host(read_ends, n_reads, k, 0);
    if (n_results) *n_results = total_k;
    throw Error(SBWT_E_CAPACITY, "results_capacity smaller than the k-mer count");
  }
  if (n_results) *n_results = kacc;
  check_err_word(ws, ws.streams[0]);
}

void IndexImpl::search_positions(const u64 *bit_seqs, u64 n_words, const u64 *positions,
                                 u64 n, u64 *results, u32 flags, cudaStream_t st,
                                 const LaunchConfig &cfg) const {
  DeviceGuard g(device);
  Workspace &ws = workspace(device);
  if (n == 0) return;
  if ((flags & SBWT_MOVE_TO_KEY_KMER) && !view.key_marks)
    throw Error(SBWT_E_INVALID, "SBWT_MOVE_TO_KEY_KMER needs key k-mer marks");
  const SbwtView sv = view_for(cfg.presearch_letters);
  const u32 mtk = (flags & SBWT_MOVE_TO_KEY_KMER) ? 1u : 0u;
  const int grid = grid_for(device, n, 256, cfg.blocks_per_sm);
  if (flags & SBWT_DEVICE_POINTERS) {
    search_positions_kernel<<<grid, 256, 0, st>>>(sv, bit_seqs, n_words * 32, positions,
                                                   n, results, mtk, ws.err_dev.get<u32>());
    note_launches(1);
    SBWT_CUDA(cudaGetLastError());
    check_err_word(ws, st);
    return;
  }
  cudaStream_t s0 = ws.streams[0];
  ws.bits.ensure((n_words + 2) * 8);
  ws.positions.ensure(n * 8);
  ws.results[0].ensure(n * 8);
  SBWT_CUDA(cudaMemsetAsync(ws.bits.get<u64>() + n_words, 0, 16, s0));
  SBWT_CUDA(cudaMemcpyAsync(ws.bits.get(), bit_seqs, n_words * 8, cudaMemcpyHostToDevice, s0));
  SBWT_CUDA(cudaMemcpyAsync(ws.positions.get(), positions, n * 8, cudaMemcpyHostToDevice, s0));
  search_positions_kernel<<<grid, 256, 0, s0>>>(sv, ws.bits.get<u64>(), n_words * 32,
                                                 ws.positions.get<u64>(), n,
                                                 ws.results[0].get<u64>(), mtk,
                                                 ws.err_dev.get<u32>());
  note_launches(1);
  SBWT_CUDA(cudaGetLastError());
  SBWT_CUDA(cudaMemcpyAsync(results, ws.results[0].get(), n * 8, cudaMemcpyDeviceToHost, s0));
  check_err_word(ws, s0);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the fused read search
// ---------------------------------------------------------------------------
// Some callers may not allocate device memory themselves or through us: code
// that runs while another framework owns the device allocator (a caching
// allocator that must see every byte), latency-critical serving loops where a
// cudaMalloc / cudaFree would stall or implicitly synchronize the device, and
// hosts that have already sized their memory budget to the last byte.  For
// them sbwt_search_reads_noalloc runs the same pipeline (scan, pack, tile
// table, search kernel) with all its scratch in this fixed device array.
//
// Limits: at most kNoAllocMaxChars chars and kNoAllocMaxReads reads per call.
// The array (about 9 MiB) lives on every GPU that loads this library until
// the process exits.  All calls share it, so calls that overlap on the GPU
// (from several host threads or streams) race: serialize them.
constexpr u64 kNoAllocMaxChars = 8ULL << 20;
constexpr u64 kNoAllocMaxReads = 1ULL << 18;
constexpr u64 kNoAllocWords = kNoAllocMaxChars / 32;
constexpr u64 kNoAllocOffKmerOff = 0;
constexpr u64 kNoAllocOffPacked = kNoAllocOffKmerOff + (kNoAllocMaxReads + 1) * 8;
constexpr u64 kNoAllocOffInvalid = kNoAllocOffPacked + (kNoAllocWords + 2) * 8;
constexpr u64 kNoAllocOffBlockSums =
    ((kNoAllocOffInvalid + (kNoAllocWords + 2) * 4 + 255) / 256) * 256;
constexpr u64 kNoAllocOffTotal =
    kNoAllocOffBlockSums + ((kNoAllocMaxReads + kScanTile - 1) / kScanTile + 1) * 8;
constexpr u64 kNoAllocOffErr = kNoAllocOffTotal + 8;
constexpr u64 kNoAllocOffQueue = kNoAllocOffErr + 8;
constexpr u64 kNoAllocOffTileRead = kNoAllocOffErr + 248;  // keeps 8-byte alignment
constexpr u64 kNoAllocTileMin = 16;
constexpr u64 kNoAllocBytes =
    kNoAllocOffTileRead + (kNoAllocMaxChars / kNoAllocTileMin + 2) * 8;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch on `device`, looked up once per device
// (with that device current) on the first call there; later calls read it
// without a lock.
static unsigned char *noalloc_scratch_address(int device) {
  static const int n_dev = [] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
    return n;
  }();
  static std::unique_ptr<std::atomic<unsigned char *>[]> addr(
      new std::atomic<unsigned char *>[std::max(n_dev, 1)]());
  static std::mutex mu;
  if (device < 0 || device >= n_dev) throw Error(SBWT_E_INVALID, "device id out of range");
  unsigned char *a = addr[device].load(std::memory_order_acquire);
  if (a) return a;
  std::lock_guard<std::mutex> g(mu);
  a = addr[device].load(std::memory_order_relaxed);
  if (!a) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      throw Error(SBWT_E_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                   cudaGetErrorString(e));
    a = static_cast<unsigned char *>(p);
    addr[device].store(a, std::memory_order_release);
  }
  return a;
}

void IndexImpl::search_reads_noalloc(const char *d_chars, u64 n_chars, const u64 *d_ends,
                                     u64 n_reads, u64 *d_results, u64 capacity,
                                     u64 *n_results, u32 flags, cudaStream_t st,
                                     const LaunchConfig &cfg_in) const {
  if (n_chars > kNoAllocMaxChars || n_reads > kNoAllocMaxReads)
    throw Error(SBWT_E_INVALID,
                "sbwt_search_reads_noalloc takes at most " +
                    std::to_string(kNoAllocMaxChars) + " chars and " +
                    std::to_string(kNoAllocMaxReads) + " reads per call (got " +
                    std::to_string(n_chars) + " chars, " + std::to_string(n_reads) +
                    " reads); split the batch or use sbwt_search_reads");
  DeviceGuard g(device);
  unsigned char *base = noalloc_scratch_address(device);
  ReadsScratch sc{reinterpret_cast<u64 *>(base + kNoAllocOffKmerOff),
                  reinterpret_cast<u64 *>(base + kNoAllocOffPacked),
                  reinterpret_cast<uint32_t *>(base + kNoAllocOffInvalid),
                  reinterpret_cast<u64 *>(base + kNoAllocOffBlockSums),
                  reinterpret_cast<u64 *>(base + kNoAllocOffTotal),
                  reinterpret_cast<u64 *>(base + kNoAllocOffTileRead),
                  reinterpret_cast<uint32_t *>(base + kNoAllocOffErr),
                  reinterpret_cast<unsigned long long *>(base + kNoAllocOffQueue)};
  // the error word and the work-queue counter keep the last call's values:
  // clear them first
  SBWT_CUDA(cudaMemsetAsync(sc.err, 0, 4, st));
  SBWT_CUDA(cudaMemsetAsync(sc.queue, 0, 8, st));
  u64 n_k = 0;
  uint32_t err = 0;
  if (n_reads) {
    launch_prepare(device, k, d_chars, n_chars, d_ends, n_reads, 0, sc, st);
    SBWT_CUDA(cudaMemcpyAsync(&n_k, sc.total, 8, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaMemcpyAsync(&err, sc.err, 4, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
    if (err) throw Error(SBWT_E_INVALID, "read_ends are not non-decreasing within n_chars");
  }
  if (n_results) *n_results = n_k;
  if (n_k > capacity)
    throw Error(SBWT_E_CAPACITY, "results_capacity smaller than the k-mer count");
  if (n_k == 0) return;
  LaunchConfig cfg = cfg_in;  // the tile table is sized for tiles of >= 16
  if (cfg.tile && cfg.tile < kNoAllocTileMin) cfg.tile = kNoAllocTileMin;
  ReadsView rv{};
  rv.n_kmers_bound = std::max<u64>(n_chars, n_reads) + 64;
  rv.packed = sc.packed;
  rv.invalid = sc.invalid;
  rv.ends = d_ends;
  rv.kmer_off = sc.kmer_off;
  rv.base = 0;
  rv.n_reads = n_reads;
  rv.n_kmers = n_k;
  rv.tile = tile_size(device, n_k, cfg);
  rv.n_tiles = (n_k + rv.tile - 1) / rv.tile;
  rv.out = d_results;
  rv.out_capacity = capacity;
  rv.probe_len = probe_length(num_bits, k, cfg);
  rv.queue = sc.queue;
  tile_reads_kernel<<<grid_for(device, n_reads, 256, 16), 256, 0, st>>>(sc.kmer_off, n_reads,
                                                                        rv.tile, sc.tile_read);
  const int grid = grid_for(device, rv.n_tiles, (int)cfg.block_threads, cfg.blocks_per_sm);
  const SbwtView sv = view_for(cfg.presearch_letters);
  const u32 mtk = (flags & SBWT_MOVE_TO_KEY_KMER) ? 1u : 0u;
  const bool stream = !(flags & SBWT_PER_KMER_WALK) && view.suffix_group_starts;
  // the same kernel choice as sbwt_search_reads, without the profiler
  launch_search_kernel(stream, sv, rv, sc.tile_read, mtk, sc.err, grid,
                       (int)cfg.block_threads, st, LaunchAttrs{}, cfg.table_kernel,
                       /*instrument=*/false);
  SBWT_CUDA(cudaMemcpyAsync(&err, sc.err, 4, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaStreamSynchronize(st));
  if (err)
    throw Error(SBWT_E_TIMEOUT,
                "key k-mer walk did not reach a key k-mer (node without an outgoing "
                "edge); results of those k-mers are unspecified");
}

}  // namespace sbwt

extern "C" {
// Instrumentation hooks (not part of the reference-facing surface).
int sbwt_profile_enable(int enabled, int count_work) {
  sbwt::Profile &p = sbwt::profile();
  std::lock_guard<std::mutex> g(p.mu);
  p.enabled = enabled != 0;
  p.count = count_work != 0;
  return SBWT_OK;
}
// search_ms: summed CUDA-event time of the read/position search kernels;
// counters (count mode only): [0] presearch lookups, [1] rank-block sectors,
// [2] suffix-group words, [3] probe iterations, [4] warp iterations, [5] lane
// load steps, [6] k-mers written without a search (invalid or proven absent),
// [7] k-mers searched, [8..13] lane steps of each phase-3 path (stream step,
// presearch of a new k-mer, walk, group scan, k-mer table lookup, probe),
// [14] distinct paths per warp iteration, summed.  Resets the totals.
int sbwt_profile_read(double *search_ms, uint64_t *search_launches,
                      uint64_t *launches, uint64_t counters[16]) {
  sbwt::Profile &p = sbwt::profile();
  std::lock_guard<std::mutex> g(p.mu);
  if (search_ms) *search_ms = p.search_ms;
  if (search_launches) *search_launches = p.search_launches;
  if (launches) *launches = p.launches;
  if (counters) {
    uint64_t dc[16] = {};
    if (p.d_counters.size()) {
      cudaMemcpy(dc, p.d_counters.get(), 128, cudaMemcpyDeviceToHost);
      cudaMemset(p.d_counters.get(), 0, 128);
    }
    for (int i = 0; i < 16; ++i) counters[i] = dc[i];
  }
  p.search_ms = 0;
  p.search_launches = 0;
  p.launches = 0;
  return SBWT_OK;
}
}
