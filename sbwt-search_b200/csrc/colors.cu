// Colors step on the B200: per-read color counting and the tau threshold.
//
// Reference behaviour restated (SBWT-Search, paths in its src/):
//   d_color_search   ColorSearcher/ColorSearcher.cuh:68-206 (+ helpers :208-318)
//   d_post_process   ColorSearcher/ColorPostProcessor.cuh:21-43
//   threshold        ColorResultsPrinter/ContinuousColorResultsPrinter.hpp:235-263
//   .tcolors layout  ColorIndexBuilder/ColorIndexBuilder.cpp:23-86
//
// Semantics: count[r][c] = number of found k-mers of read r whose color set
// holds c.  The reference gets there with one thread per k-mer, a warp-wide
// loop over the color span and u8 per-(warp, color) partial counts summed by
// a second kernel into an R x C u64 matrix copied to the host.  Here one warp
// owns one read and one tile of up to 8192 colors (more colors -> more tiles
// per read): lane i owns colors [64 i, 64 i + 64) (and i + 32, ...) of the
// tile as bit-sliced counters in shared memory (plane j holds bit j of 64
// counters), a dense color row is added with a ripple-carry over the planes
// (no atomics, no conflicts), a sparse list is turned into the same per-lane
// row words with warp shuffles, the k-mers of a window that share a color set
// add it once with their multiplicity, and the threshold is a bit-sliced
// comparison; only the passing color bitmask leaves the kernel.  Each k-mer's
// set is one 8-byte record load from a per-node table when that table is
// resident (else rank over the key k-mer marks, color set index, record).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "colors_internal.hpp"
#include "common.hpp"
#include "formats.hpp"
#include "rank_blocks.cuh"

namespace sbwt {

constexpr int kColorWarps = 4;  // warps (reads in flight) per block

__device__ __forceinline__ uint64_t rec_start(uint64_t rec) { return rec >> (kRecLenBits + 1); }
__device__ __forceinline__ uint32_t rec_len(uint64_t rec) {
  return (uint32_t)(rec >> 1) & ((1u << kRecLenBits) - 1);
}

struct ColorsJob {
  const uint64_t *vals;     // SBWT indexes (markers allowed when counted)
  const uint64_t *offs;     // n_reads + 1
  const uint64_t *not_found;  // per read or nullptr
  const uint64_t *invalid;    // per read or nullptr
  uint64_t n_reads;
  double tau;
  uint32_t include_not_found, include_invalid;
  uint32_t planes;          // bit planes of the counters
  uint64_t *pass_bits;      // n_reads x row_words (mode 0)
  uint32_t *pass_count;     // n_reads (mode 0)
  uint32_t *counts;         // n_reads x num_colors (mode 1)
};

__device__ __forceinline__ uint64_t rank_key(const ColorsView &cv, uint64_t i) {
  const uint64_t b = i / kBlockBits;
  const Block B = load_block(cv.key_blocks + b);
  return cv.key_l0[b >> kSuperchunkShift] + block_rank(B, (uint32_t)(i - b * kBlockBits));
}

// The packed set record of SBWT index v < key_bits: the set of key k-mer
// number rank(key_marks, v), as the reference's ColorSearcher resolves it
// (rank of v among the key k-mer marks, then color_set_idxs).  kRecNone when
// the rank is past the last key k-mer.  DIRECT reads the per-node table that
// holds exactly these values.
template <bool DIRECT>
__device__ __forceinline__ uint64_t set_record(const ColorsView &cv, uint64_t v) {
  if (DIRECT) return __ldg(cv.node_rec + v);
  const uint64_t j = rank_key(cv, v);
  if (j >= cv.n_keys) return kRecNone;
  const uint32_t s = __ldg(cv.csi + j);
  return s < cv.n_sets ? __ldg(cv.recs + s) : kRecNone;
}

// out[i] = entry i of an sdsl int vector of `width` bits per entry (LSB-first
// in 64-bit words); entries >= limit set *err and read as 0.
__global__ void unpack_set_indexes_kernel(const uint64_t *words, uint64_t n, uint32_t width,
                                          uint64_t limit, uint32_t *out, uint32_t *err) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t mask = width >= 64 ? ~0ULL : (1ULL << width) - 1;
  uint32_t bad = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += step) {
    const uint64_t bit = i * width, w = bit >> 6, o = bit & 63;
    uint64_t v = words[w] >> o;
    if (o + width > 64) v |= words[w + 1] << (64 - o);
    v &= mask;
    if (v >= limit) {
      bad = 1;
      v = 0;
    }
    out[i] = (uint32_t)v;
  }
  if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, 1u);
}

// node_rec[v] = set_record(v) for every v < key_bits.
__global__ void node_record_kernel(ColorsView cv, uint64_t *out) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < cv.key_bits; v += step)
    out[v] = set_record<false>(cv, v);
}

// Adds x << j0 (one bit per color, shifted to plane j0) into the bit-sliced
// counters planes[j * stride] (j = 0..P-1): ripple carry, stops when the
// carry dies.  Counts never exceed 2^P - 1 (P covers the longest read), so
// no carry leaves plane P - 1.
__device__ __forceinline__ void add_word_at(uint64_t *planes, uint32_t stride, uint32_t j0,
                                            uint32_t P, uint64_t x) {
  for (uint32_t j = j0; j < P && x; ++j) {
    const uint64_t p = planes[j * stride];
    planes[j * stride] = p ^ x;
    x &= p;
  }
}

// Adds m copies of row word x: one ripple per set bit of m.
__device__ __forceinline__ void add_weighted(uint64_t *planes, uint32_t stride, uint32_t P,
                                             uint64_t x, uint32_t m) {
  while (m) {
    const uint32_t b = __ffs(m) - 1;
    m &= m - 1;
    add_word_at(planes, stride, b, P, x);
  }
}

// 2 rows in flight at a 14-blocks-per-SM register budget (32 registers):
// 17.6 ms against 17.9 ms at 12 blocks, 19.5 ms for 4 rows at 10 blocks
// (2 M reads of the 2000-genome workload); more rows in flight cost
// occupancy and were slower (8 rows: 2x)
#ifndef SBWT_COLORS_ROWS_IN_FLIGHT
#define SBWT_COLORS_ROWS_IN_FLIGHT 2
#endif
#ifndef SBWT_COLORS_BLOCKS_PER_SM
#define SBWT_COLORS_BLOCKS_PER_SM 14
#endif
constexpr int kRowsInFlight = SBWT_COLORS_ROWS_IN_FLIGHT;  // dense rows loaded before the adds
#ifndef SBWT_COLORS_WINDOWS
#define SBWT_COLORS_WINDOWS 4
#endif
constexpr int kWindows = SBWT_COLORS_WINDOWS;  // windows of 32 k-mers whose lookups overlap
constexpr int kColorBlocksPerSm = SBWT_COLORS_BLOCKS_PER_SM;

// Adds m copies of the sparse color list sparse[start, start + len) to this
// warp's counters for the row words [wbase, wbase + 32 * WL).  Warp-uniform.
// 32 ids at a time: each lane ORs its id's bit into the row word it falls in
// (stage: the warp's 32 * WL zeroed words in shared memory), then every lane
// adds its own staged words and zeroes them again.
__device__ __forceinline__ void add_sparse(const ColorsView &cv, uint64_t *planes,
                                           uint64_t *stage, uint32_t stride, uint32_t P,
                                           uint32_t WL, uint32_t wbase, uint32_t lane,
                                           uint64_t start, uint32_t len, uint32_t m) {
  const uint32_t span = 32 * WL;
  for (uint32_t c0 = 0; c0 < len; c0 += 32) {
    const bool in = c0 + lane < len;
    const uint32_t id = in ? __ldg(cv.sparse + start + c0 + lane) : 0xFFFFFFFFu;
    const uint32_t n = min(32u, len - c0);
    if (cv.tiles > 1 && cv.sparse_sorted) {  // ascending ids: skip chunks outside the tile
      if ((__shfl_sync(0xFFFFFFFFu, id, n - 1) >> 6) < wbase) continue;
      if ((__shfl_sync(0xFFFFFFFFu, id, 0) >> 6) >= wbase + span) break;
    }
    const uint32_t local = (id >> 6) - wbase;  // wraps above span when below the tile
    if (in && local < span) atomicOr((unsigned long long *)(stage + local), 1ULL << (id & 63));
    __syncwarp();
    for (uint32_t w = 0; w < WL; ++w) {
      const uint32_t li = lane + 32 * w;
      const uint64_t x = stage[li];
      if (x) {
        stage[li] = 0;
        add_weighted(planes + li, stride, P, x, m);
      }
    }
    __syncwarp();
  }
}

// One warp per work item (read r, color tile): tile t covers row words
// [t * 32 * WL, (t + 1) * 32 * WL), lane i owns words i, i + 32, ... of it.
// The k-mers are taken 32 * kWindows at a time: every lane issues the set
// record loads of its kWindows k-mers together, then each window of 32 adds
// its distinct records once with their multiplicity (__match_any_sync), rows
// kRowsInFlight at a time.  Counts are sums, so the order and grouping of the
// adds does not change them.
// mode 0: pass bitmask + count per read; mode 1: full counts.  WLC: the row
// words per lane when known at compile time (1: up to 2048 colors), else 0;
// PC: the counter planes when known (8: reads of at most 255 k-mers), else 0.
template <int MODE, bool DIRECT, int WLC, int PC>
__global__ void __launch_bounds__(32 * kColorWarps, kColorBlocksPerSm)
    colors_kernel(ColorsView cv, ColorsJob job, uint32_t *err) {
  constexpr uint32_t FULL = 0xFFFFFFFFu;
  extern __shared__ uint64_t smem[];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t WL = WLC ? (uint32_t)WLC : cv.words_per_lane;
  const uint32_t P = PC ? (uint32_t)PC : job.planes, T = cv.tiles;
  // per warp: P planes x (32 * WL) words, plane-major so lanes are contiguous,
  // then 32 * WL staging words for the sparse lists
  const uint32_t stride = 32 * WL;
  uint64_t *planes = smem + (uint64_t)wid * (P + 1) * stride;
  uint64_t *stage = planes + (uint64_t)P * stride;
  const uint64_t warps = (uint64_t)gridDim.x * kColorWarps;
  const uint64_t n_items = job.n_reads * T;
  for (uint64_t item = blockIdx.x * (uint64_t)kColorWarps + wid; item < n_items; item += warps) {
    const uint64_t r = T == 1 ? item : item / T;
    const uint32_t wbase = (uint32_t)(item - r * T) * stride;
    for (uint32_t q = lane; q < (P + 1) * stride; q += 32) planes[q] = 0;
    __syncwarp();
    const uint64_t o0 = job.offs[r], o1 = job.offs[r + 1];
    uint32_t found = 0, not_found = 0, invalid = 0;
    for (uint64_t base = o0; base < o1; base += 32 * kWindows) {
      // lookup phase: lane t classifies k-mers base + 32 l + t (l < kWindows)
      uint64_t v[kWindows], rec[kWindows];
      uint32_t cand = 0, bad = 0;
#pragma unroll
      for (int l = 0; l < kWindows; ++l) {
        const uint64_t t = base + 32 * l + lane;
        const bool in = t < o1;
        v[l] = in ? job.vals[t] : kRecNone;
        not_found += in && v[l] == SBWT_NOT_FOUND;
        invalid += in && v[l] == SBWT_INVALID;
        if (in && v[l] < SBWT_INVALID && v[l] >= cv.key_bits) bad = 1;
        if (in && v[l] < cv.key_bits) cand |= 1u << l;
      }
      found += __popc(cand);
#pragma unroll
      for (int l = 0; l < kWindows; ++l)
        rec[l] = (cand >> l) & 1u ? set_record<DIRECT>(cv, v[l]) : kRecNone;
#pragma unroll
      for (int l = 0; l < kWindows; ++l)
        if (((cand >> l) & 1u) && rec[l] == kRecNone) bad = 1;
      if (bad) atomicOr(err, 1u);
      // add phase, one window after the other (records rotate into rec[0])
#pragma unroll 1
      for (int l = 0; l < kWindows && base + 32 * l < o1; ++l) {
        const uint64_t r0 = rec[0];
#pragma unroll
        for (int q = 0; q + 1 < kWindows; ++q) rec[q] = rec[q + 1];
        const uint32_t group = __match_any_sync(FULL, r0);
        const uint32_t weight = __popc(group);
        uint32_t todo = __ballot_sync(FULL, r0 != kRecNone && __ffs(group) - 1 == (int)lane);
        while (todo) {
          uint64_t rr[kRowsInFlight];
          uint32_t wt[kRowsInFlight];
#pragma unroll
          for (int u = 0; u < kRowsInFlight; ++u) {
            const int src = todo ? __ffs(todo) - 1 : 0;
            const uint32_t live = todo ? 1u : 0u;
            todo &= todo - 1;
            rr[u] = __shfl_sync(FULL, r0, src);
            wt[u] = live * __shfl_sync(FULL, weight, src);
          }
          for (uint32_t w = 0; w < WL; ++w) {
            const uint32_t local = lane + 32 * w, word = wbase + local;
            uint64_t x[kRowsInFlight];
#pragma unroll
            for (int u = 0; u < kRowsInFlight; ++u)
              x[u] = (wt[u] && (rr[u] & 1ULL) && word < rec_len(rr[u]))
                         ? __ldg(cv.dense + rec_start(rr[u]) + word)
                         : 0;
#pragma unroll
            for (int u = 0; u < kRowsInFlight; ++u)
              if (x[u]) add_weighted(planes + local, stride, P, x[u], wt[u]);
          }
#pragma unroll
          for (int u = 0; u < kRowsInFlight; ++u)
            if (wt[u] && !(rr[u] & 1ULL))
              add_sparse(cv, planes, stage, stride, P, WL, wbase, lane, rec_start(rr[u]),
                         rec_len(rr[u]), wt[u]);
        }
      }
    }
    __syncwarp();
    // per-read sizes
    for (int o = 16; o; o >>= 1) {
      found += __shfl_xor_sync(FULL, found, o);
      not_found += __shfl_xor_sync(FULL, not_found, o);
      invalid += __shfl_xor_sync(FULL, invalid, o);
    }
    if (job.not_found) not_found += (uint32_t)job.not_found[r];
    if (job.invalid) invalid += (uint32_t)job.invalid[r];
    if (MODE == 0) {
      const uint64_t size = (uint64_t)found + (job.include_not_found ? not_found : 0) +
                            (job.include_invalid ? invalid : 0);
      const uint64_t minimum = (uint64_t)ceil((double)size * job.tau);
      uint32_t passing = 0;
      for (uint32_t w = 0; w < WL; ++w) {
        const uint32_t local = lane + 32 * w, word = wbase + local;
        uint64_t ge = 0;
        if (minimum > 0 && word < cv.row_words && (P >= 64 || (minimum >> P) == 0)) {
          uint64_t gt = 0, eq = ~0ULL;
          for (int j = (int)P - 1; j >= 0; --j) {
            const uint64_t pl = planes[(uint32_t)j * stride + local];
            if ((minimum >> j) & 1ULL) {
              eq &= pl;
            } else {
              gt |= eq & pl;
              eq &= ~pl;
            }
          }
          ge = gt | eq;
          const uint32_t rem = cv.num_colors - word * 64;
          if (rem < 64) ge &= (1ULL << rem) - 1ULL;
        }
        if (word < cv.row_words) job.pass_bits[r * cv.row_words + word] = ge;
        passing += __popcll(ge);
      }
      for (int o = 16; o; o >>= 1) passing += __shfl_xor_sync(FULL, passing, o);
      if (lane == 0) {
        if (T == 1)
          job.pass_count[r] = passing;
        else
          atomicAdd(job.pass_count + r, passing);  // zeroed before the launch
      }
    } else {
      for (uint32_t w = 0; w < WL; ++w) {
        const uint32_t local = lane + 32 * w, word = wbase + local;
        if (word >= cv.row_words) continue;
        for (uint32_t b = 0; b < 64; ++b) {
          const uint32_t c = word * 64 + b;
          if (c >= cv.num_colors) break;
          uint32_t cnt = 0;
          for (uint32_t j = 0; j < P; ++j)
            cnt |= (uint32_t)((planes[j * stride + local] >> b) & 1ULL) << j;
          job.counts[r * cv.num_colors + c] = cnt;
        }
      }
    }
    __syncwarp();
  }
}

// Expands each read's pass bitmask into ascending color ids at ids_off[r].
__global__ void emit_ids_kernel(const uint64_t *pass_bits, uint32_t row_words,
                                const uint64_t *ids_off, uint64_t n_reads,
                                uint32_t *ids, uint64_t capacity) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warp0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = warp0; r < n_reads; r += warps) {
    uint64_t out = ids_off[r];
    for (uint32_t w0 = 0; w0 < row_words; w0 += 32) {
      const uint32_t word = w0 + lane;
      uint64_t m = word < row_words ? pass_bits[r * row_words + word] : 0;
      const uint32_t cnt = __popcll(m);
      uint32_t incl = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      uint64_t pos = out + incl - cnt;
      while (m) {
        const uint32_t b = __ffsll(m) - 1;
        m &= m - 1;
        if (pos < capacity) ids[pos] = word * 64 + b;
        ++pos;
      }
      out += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
  }
}

// Exclusive scan of u32 counts into u64 offsets off[0..n] in three launches
// and no scratch: block b of the first launch leaves the total of counts
// [b * kScanSpan, (b + 1) * kScanSpan) in off[b * kScanSpan], one block
// scans those totals in place (and writes off[n]), and the last launch
// replaces every block's range with its offsets.
constexpr uint32_t kScanThreads = 1024, kScanPer = 4, kScanSpan = kScanThreads * kScanPer;

// Block-wide exclusive scan of one u64 per thread; the block total comes back
// through *total.  All threads of the block must call it.
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t *total) {
  __shared__ uint64_t wsum[32];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint64_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint64_t s = lane < blockDim.x / 32 ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  const uint64_t ex = (wid ? wsum[wid - 1] : 0) + x - v;
  *total = wsum[blockDim.x / 32 - 1];
  __syncthreads();  // wsum is reused by the next call
  return ex;
}

__global__ void __launch_bounds__(kScanThreads) scan_totals_kernel(const uint32_t *cnt, uint64_t n,
                                                                   uint64_t *off) {
  const uint64_t b0 = blockIdx.x * (uint64_t)kScanSpan;
  uint64_t v = 0;
  for (uint32_t k = 0; k < kScanPer; ++k) {
    const uint64_t i = b0 + k * kScanThreads + threadIdx.x;
    if (i < n) v += cnt[i];
  }
  uint64_t total = 0;
  block_exclusive_scan(v, &total);
  if (threadIdx.x == 0) off[b0] = total;
}

__global__ void __launch_bounds__(kScanThreads) scan_tops_kernel(uint64_t *off, uint64_t n,
                                                                 uint64_t n_blocks) {
  uint64_t carry = 0;
  for (uint64_t b = 0; b < n_blocks; b += kScanThreads) {
    const uint64_t i = b + threadIdx.x;
    const uint64_t v = i < n_blocks ? off[i * kScanSpan] : 0;
    uint64_t total = 0;
    const uint64_t ex = block_exclusive_scan(v, &total);
    if (i < n_blocks) off[i * kScanSpan] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) off[n] = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_write_kernel(const uint32_t *cnt, uint64_t n,
                                                                  uint64_t *off) {
  __shared__ uint64_t base;
  const uint64_t b0 = blockIdx.x * (uint64_t)kScanSpan;
  if (threadIdx.x == 0) base = off[b0];
  __syncthreads();
  const uint64_t i0 = b0 + (uint64_t)threadIdx.x * kScanPer;
  uint32_t c[kScanPer];
  uint64_t v = 0;
#pragma unroll
  for (uint32_t k = 0; k < kScanPer; ++k) {
    c[k] = i0 + k < n ? cnt[i0 + k] : 0;
    v += c[k];
  }
  uint64_t total = 0;
  uint64_t at = base + block_exclusive_scan(v, &total);
#pragma unroll
  for (uint32_t k = 0; k < kScanPer; ++k) {
    if (i0 + k < n) off[i0 + k] = at;
    at += c[k];
  }
}

static void enqueue_scan_counts(const uint32_t *d_cnt, uint64_t n, uint64_t *d_off,
                                cudaStream_t st) {
  if (n == 0) {
    SBWT_CUDA(cudaMemsetAsync(d_off, 0, 8, st));
    return;
  }
  const uint64_t nb = (n + kScanSpan - 1) / kScanSpan;
  scan_totals_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(d_cnt, n, d_off);
  scan_tops_kernel<<<1, kScanThreads, 0, st>>>(d_off, n, nb);
  scan_write_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(d_cnt, n, d_off);
  SBWT_CUDA(cudaGetLastError());
}

// out[0] = max over reads of offs[r + 1] - offs[r]; out[1] = 1 when some
// offset decreases.  out is zeroed before the launch.
__global__ void max_span_kernel(const uint64_t *offs, uint64_t n_reads,
                                unsigned long long *out) {
  unsigned long long m = 0, bad = 0;
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n_reads; r += step) {
    const uint64_t a = offs[r], b = offs[r + 1];
    if (b < a)
      bad = 1;
    else
      m = max(m, (unsigned long long)(b - a));
  }
  for (int o = 16; o; o >>= 1) {
    m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    bad |= __shfl_xor_sync(0xFFFFFFFFu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (m) atomicMax(out, m);
    if (bad) atomicOr(out + 1, bad);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
void build_rank_blocks_host(const u64 *words, u64 num_bits, std::vector<Block> &blocks,
                            std::vector<u64> &l0, u64 &total);

ColorsImpl::ColorsImpl(const TColorsFile &t, int device_) {
  device = device_;
  DeviceGuard g(device);
  num_colors = t.num_colors();
  if (num_colors == 0 || num_colors > (1u << 20))
    throw Error(SBWT_E_FORMAT, "number of colors out of range");
  const u64 n_sets = t.is_dense_marks.num_bits;
  const u64 n_keys = t.color_set_idxs.size();
  const HostColorSets h = prepare_color_sets(t);
  std::vector<Block> kb;
  std::vector<u64> kl0;
  u64 total_keys = 0;
  build_rank_blocks_host(t.key_kmer_marks.words.data(), t.key_kmer_marks.num_bits, kb, kl0,
                         total_keys);
  if (total_keys > n_keys)
    throw Error(SBWT_E_FORMAT, "more key k-mers than color set indexes");
  auto up = [&](DeviceBuffer &b, const void *src, size_t bytes) {
    b.resize(bytes);
    SBWT_CUDA(cudaMemcpy(b.get(), src, bytes, cudaMemcpyHostToDevice));
  };
  up(key_blocks, kb.data(), kb.size() * sizeof(Block));
  up(key_l0, kl0.data(), kl0.size() * 8);
  up(recs_buf, h.recs.data(), h.recs.size() * 8);
  up(dense_buf, h.dense_words.data(), h.dense_words.size() * 8);
  up(sparse_buf, h.sparse.data(), h.sparse.size() * 4);
  // color set indexes: the packed int vector goes up as it is and is widened
  // to u32 on the device
  csi_buf.resize(std::max<u64>(n_keys, 1) * 4);
  if (n_keys) {
    DeviceBuffer packed, err;
    up(packed, t.color_set_idxs.words.data(), t.color_set_idxs.words.size() * 8);
    err.resize(4);
    SBWT_CUDA(cudaMemset(err.get(), 0, 4));
    const u64 blocks = std::min<u64>((n_keys + 255) / 256, 148 * 16);
    unpack_set_indexes_kernel<<<(unsigned)blocks, 256>>>(
        packed.get<u64>(), n_keys, t.color_set_idxs.width, n_sets, csi_buf.get<uint32_t>(),
        err.get<uint32_t>());
    SBWT_CUDA(cudaGetLastError());
    uint32_t bad = 0;
    SBWT_CUDA(cudaMemcpy(&bad, err.get(), 4, cudaMemcpyDeviceToHost));
    if (bad) throw Error(SBWT_E_FORMAT, "color set index out of range");
  }
  view = ColorsView{};
  view.key_blocks = key_blocks.get<Block>();
  view.key_l0 = key_l0.get<u64>();
  view.key_bits = t.key_kmer_marks.num_bits;
  view.csi = csi_buf.get<uint32_t>();
  view.n_keys = n_keys;
  view.recs = recs_buf.get<u64>();
  view.n_sets = n_sets;
  view.dense = dense_buf.get<u64>();
  view.sparse = sparse_buf.get<uint32_t>();
  view.num_colors = (uint32_t)num_colors;
  view.row_words = (uint32_t)((num_colors + 63) / 64);
  // color tiles of at most 32 lanes x 4 words (8192 colors) per warp
  view.words_per_lane = std::min<uint32_t>((view.row_words + 31) / 32, 4);
  view.tiles = (view.row_words + 32 * view.words_per_lane - 1) / (32 * view.words_per_lane);
  view.sparse_sorted = h.sparse_sorted ? 1 : 0;
  set_node_table(true);
}

u64 ColorsImpl::device_footprint() const {
  return key_blocks.size() + key_l0.size() + csi_buf.size() + recs_buf.size() +
         dense_buf.size() + sparse_buf.size() + node_buf.size();
}

// The per-node record table turns the k-mer -> color set lookup (rank block,
// color set index, set record: three dependent random loads) into one load.
// It costs 8 bytes per SBWT node and is only built when that stays within
// kNodeTableMaxBytes and half of the free device memory.
bool ColorsImpl::set_node_table(bool enable) {
  DeviceGuard g(device);
  view.node_rec = nullptr;
  node_buf.release();
  if (enable) {
    const u64 bytes = std::max<u64>(view.key_bits, 1) * 8;
    size_t free_b = 0, total_b = 0;
    SBWT_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (bytes <= kNodeTableMaxBytes && bytes <= free_b / 2) {
      node_buf.resize(bytes);
      const u64 blocks = std::min<u64>((view.key_bits + 255) / 256, 148 * 16);
      node_record_kernel<<<(unsigned)std::max<u64>(blocks, 1), 256>>>(view, node_buf.get<u64>());
      SBWT_CUDA(cudaGetLastError());
      SBWT_CUDA(cudaDeviceSynchronize());
      view.node_rec = node_buf.get<u64>();
    }
  }
  device_bytes = device_footprint();
  return view.node_rec != nullptr;
}

struct ColorsWorkspace {
  int device = -1;
  DeviceBuffer vals, offs, nf, inv, pass_bits, pass_count, ids_off, ids, counts, err, span;
  cudaStream_t stream = nullptr;
  ~ColorsWorkspace() {
    if (stream) cudaStreamDestroy(stream);
  }
};

static ColorsWorkspace &colors_workspace(int device) {
  thread_local std::unique_ptr<ColorsWorkspace> ws[16];
  if (device < 0 || device >= 16) throw Error(SBWT_E_INVALID, "device id out of range");
  auto &p = ws[device];
  if (!p) {
    p = std::make_unique<ColorsWorkspace>();
    p->device = device;
    SBWT_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    p->err.resize(4);
    SBWT_CUDA(cudaMemset(p->err.get(), 0, 4));
  }
  return *p;
}

static uint32_t planes_for(u64 max_kmers) {
  uint32_t P = 1;
  while (P < 40 && (max_kmers >> P)) ++P;
  return P;
}

// Runs the colors kernel on device-resident arrays.  mode 0 -> pass bits +
// counts; mode 1 -> counts.  max_kmers bounds the per-read k-mer count.
void ColorsImpl::launch(const u64 *d_vals, const u64 *d_offs, const u64 *d_nf,
                        const u64 *d_inv, u64 n_reads, u64 max_kmers, double tau,
                        u32 flags, int mode, u64 *d_pass_bits, uint32_t *d_pass_count,
                        uint32_t *d_counts, uint32_t *d_err, cudaStream_t st) const {
  if (n_reads == 0) return;
  ColorsJob job{};
  job.vals = d_vals;
  job.offs = d_offs;
  job.not_found = d_nf;
  job.invalid = d_inv;
  job.n_reads = n_reads;
  job.tau = tau;
  job.include_not_found = (flags & SBWT_INCLUDE_NOT_FOUND) ? 1 : 0;
  job.include_invalid = (flags & SBWT_INCLUDE_INVALID) ? 1 : 0;
  job.planes = planes_for(max_kmers) <= 8 ? 8u : planes_for(max_kmers);
  if (mode == 0 && view.tiles > 1)  // tiles of a read add their passing counts
    SBWT_CUDA(cudaMemsetAsync(d_pass_count, 0, n_reads * 4, st));
  job.pass_bits = d_pass_bits;
  job.pass_count = d_pass_count;
  job.counts = d_counts;
  const size_t smem = (size_t)kColorWarps * (job.planes + 1) * 32 * view.words_per_lane * 8;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const u64 items = n_reads * view.tiles;
  const u64 blocks = std::min<u64>((items + kColorWarps - 1) / kColorWarps, (u64)sms * 32);
  const bool direct = view.node_rec != nullptr;
  auto go = [&](auto kernel) {
    SBWT_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    kernel<<<(unsigned)blocks, 32 * kColorWarps, smem, st>>>(view, job, d_err);
  };
  const bool wl1 = view.words_per_lane == 1, p8 = job.planes == 8;
  if (mode == 0 && wl1 && p8)
    direct ? go(colors_kernel<0, true, 1, 8>) : go(colors_kernel<0, false, 1, 8>);
  else if (mode == 0)
    direct ? go(colors_kernel<0, true, 0, 0>) : go(colors_kernel<0, false, 0, 0>);
  else if (wl1 && p8)
    direct ? go(colors_kernel<1, true, 1, 8>) : go(colors_kernel<1, false, 1, 8>);
  else
    direct ? go(colors_kernel<1, true, 0, 0>) : go(colors_kernel<1, false, 0, 0>);
  SBWT_CUDA(cudaGetLastError());
}

// The colors step of one device-resident batch without host synchronisation
// (capturable): per-read counting over `vals` (index-step results, -1/-2
// markers counted, not looked up) + threshold, scan of the per-read pass
// counts into d_ids_off (n_reads + 1), ids into d_ids (capacity bound checked
// on the device; d_ids_off[n_reads] is the required size).
void ColorsImpl::enqueue_pseudoalign(const u64 *d_vals, const u64 *d_offs, u64 n_reads,
                                     u64 max_kmers, double tau, u32 flags, u64 *d_pass_bits,
                                     uint32_t *d_pass_count, u64 *d_ids_off, uint32_t *d_ids,
                                     u64 ids_capacity, uint32_t *d_err,
                                     cudaStream_t st) const {
  if (n_reads == 0) {
    SBWT_CUDA(cudaMemsetAsync(d_ids_off, 0, 8, st));
    return;
  }
  launch(d_vals, d_offs, nullptr, nullptr, n_reads, max_kmers, tau, flags, 0, d_pass_bits,
         d_pass_count, nullptr, d_err, st);
  enqueue_scan_counts(d_pass_count, n_reads, d_ids_off, st);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const u64 blocks = std::min<u64>((n_reads + 7) / 8, (u64)sms * 16);
  emit_ids_kernel<<<(unsigned)std::max<u64>(blocks, 1), 256, 0, st>>>(
      d_pass_bits, view.row_words, d_ids_off, n_reads, d_ids, ids_capacity);
  SBWT_CUDA(cudaGetLastError());
}

void ColorsImpl::prepare_launch(u64 max_kmers) const {
  const uint32_t P = planes_for(max_kmers) <= 8 ? 8u : planes_for(max_kmers);
  const size_t smem = (size_t)kColorWarps * (P + 1) * 32 * view.words_per_lane * 8;
  for (auto kernel : {colors_kernel<0, true, 1, 8>, colors_kernel<0, false, 1, 8>,
                      colors_kernel<1, true, 1, 8>, colors_kernel<1, false, 1, 8>,
                      colors_kernel<0, true, 0, 0>, colors_kernel<0, false, 0, 0>,
                      colors_kernel<1, true, 0, 0>, colors_kernel<1, false, 0, 0>})
    SBWT_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
}

static u64 max_span(const u64 *offs, u64 n_reads) {
  u64 m = 0;
  for (u64 r = 0; r < n_reads; ++r) {
    if (offs[r + 1] < offs[r]) throw Error(SBWT_E_INVALID, "offsets must be non-decreasing");
    m = std::max(m, offs[r + 1] - offs[r]);
  }
  return m;
}

// Longest read of device-resident offsets (one small reduction, 16 bytes back).
static u64 device_max_span(ColorsWorkspace &ws, const u64 *d_offs, u64 n_reads,
                           cudaStream_t st) {
  ws.span.ensure(16);
  SBWT_CUDA(cudaMemsetAsync(ws.span.get(), 0, 16, st));
  const u64 blocks = std::min<u64>((n_reads + 255) / 256, 148 * 8);
  max_span_kernel<<<(unsigned)std::max<u64>(blocks, 1), 256, 0, st>>>(
      d_offs, n_reads, ws.span.get<unsigned long long>());
  SBWT_CUDA(cudaGetLastError());
  unsigned long long h[2] = {0, 0};
  SBWT_CUDA(cudaMemcpyAsync(h, ws.span.get(), 16, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaStreamSynchronize(st));
  if (h[1]) throw Error(SBWT_E_INVALID, "offsets must be non-decreasing");
  return h[0];
}

static void check_colors_err(ColorsWorkspace &ws, cudaStream_t st) {
  uint32_t e = 0;
  SBWT_CUDA(cudaMemcpyAsync(&e, ws.err.get(), 4, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaStreamSynchronize(st));
  if (e) {
    SBWT_CUDA(cudaMemset(ws.err.get(), 0, 4));
    throw Error(SBWT_E_INVALID, "an SBWT index is not a key k-mer of this color index");
  }
}

void ColorsImpl::counts(const u64 *vals, const u64 *offs, u64 n_reads, uint32_t *out,
                        u32 flags, cudaStream_t user_stream) const {
  DeviceGuard g(device);
  ColorsWorkspace &ws = colors_workspace(device);
  if (n_reads == 0) return;
  if (flags & SBWT_DEVICE_POINTERS) {
    launch(vals, offs, nullptr, nullptr, n_reads, device_max_span(ws, offs, n_reads, user_stream),
           0.0, 0, 1,
           nullptr, nullptr, out, ws.err.get<uint32_t>(), user_stream);
    check_colors_err(ws, user_stream);
    return;
  }
  const u64 mk = max_span(offs, n_reads);
  const u64 n_vals = offs[n_reads] - offs[0];
  cudaStream_t st = ws.stream;
  ws.vals.ensure(std::max<u64>(n_vals, 1) * 8);
  ws.offs.ensure((n_reads + 1) * 8);
  ws.counts.ensure(n_reads * num_colors * 4);
  // offsets are rebased to the first value
  std::vector<u64> ro(n_reads + 1);
  for (u64 r = 0; r <= n_reads; ++r) ro[r] = offs[r] - offs[0];
  if (n_vals)
    SBWT_CUDA(cudaMemcpyAsync(ws.vals.get(), vals + offs[0], n_vals * 8,
                              cudaMemcpyHostToDevice, st));
  SBWT_CUDA(cudaMemcpyAsync(ws.offs.get(), ro.data(), (n_reads + 1) * 8,
                            cudaMemcpyHostToDevice, st));
  launch(ws.vals.get<u64>(), ws.offs.get<u64>(), nullptr, nullptr, n_reads, mk, 0.0, 0, 1,
         nullptr, nullptr, ws.counts.get<uint32_t>(), ws.err.get<uint32_t>(), st);
  SBWT_CUDA(cudaMemcpyAsync(out, ws.counts.get(), n_reads * num_colors * 4,
                            cudaMemcpyDeviceToHost, st));
  check_colors_err(ws, st);
}

void ColorsImpl::pseudoalign(const u64 *vals, const u64 *offs, const u64 *nf,
                             const u64 *inv, u64 n_reads, double tau, u32 flags,
                             uint32_t *ids, u64 capacity, u64 *ids_offsets,
                             cudaStream_t user_stream) const {
  DeviceGuard g(device);
  ColorsWorkspace &ws = colors_workspace(device);
  const u32 rw = view.row_words;
  const bool dev = flags & SBWT_DEVICE_POINTERS;
  cudaStream_t st = dev ? user_stream : ws.stream;
  if (n_reads == 0) {
    if (dev) {
      SBWT_CUDA(cudaMemsetAsync(ids_offsets, 0, 8, st));
    } else {
      ids_offsets[0] = 0;
    }
    return;
  }
  const u64 *d_vals = vals, *d_offs = offs, *d_nf = nf, *d_inv = inv;
  u64 mk = 0;
  if (dev) {
    mk = device_max_span(ws, offs, n_reads, st);
  } else {
    mk = max_span(offs, n_reads);
    const u64 n_vals = offs[n_reads] - offs[0];
    ws.vals.ensure(std::max<u64>(n_vals, 1) * 8);
    ws.offs.ensure((n_reads + 1) * 8);
    std::vector<u64> ro(n_reads + 1);
    for (u64 r = 0; r <= n_reads; ++r) ro[r] = offs[r] - offs[0];
    if (n_vals)
      SBWT_CUDA(cudaMemcpyAsync(ws.vals.get(), vals + offs[0], n_vals * 8,
                                cudaMemcpyHostToDevice, st));
    SBWT_CUDA(cudaMemcpyAsync(ws.offs.get(), ro.data(), (n_reads + 1) * 8,
                              cudaMemcpyHostToDevice, st));
    d_vals = ws.vals.get<u64>();
    d_offs = ws.offs.get<u64>();
    d_nf = d_inv = nullptr;
    if (nf && (flags & SBWT_INCLUDE_NOT_FOUND)) {
      ws.nf.ensure(n_reads * 8);
      SBWT_CUDA(cudaMemcpyAsync(ws.nf.get(), nf, n_reads * 8, cudaMemcpyHostToDevice, st));
      d_nf = ws.nf.get<u64>();
    }
    if (inv && (flags & SBWT_INCLUDE_INVALID)) {
      ws.inv.ensure(n_reads * 8);
      SBWT_CUDA(cudaMemcpyAsync(ws.inv.get(), inv, n_reads * 8, cudaMemcpyHostToDevice, st));
      d_inv = ws.inv.get<u64>();
    }
  }
  if (!(flags & SBWT_INCLUDE_NOT_FOUND)) d_nf = nullptr;
  if (!(flags & SBWT_INCLUDE_INVALID)) d_inv = nullptr;
  ws.pass_bits.ensure(n_reads * rw * 8);
  ws.pass_count.ensure(n_reads * 4);
  ws.ids_off.ensure((n_reads + 1) * 8);
  launch(d_vals, d_offs, d_nf, d_inv, n_reads, mk, tau, flags, 0, ws.pass_bits.get<u64>(),
         ws.pass_count.get<uint32_t>(), nullptr, ws.err.get<uint32_t>(), st);
  u64 *d_ids_off = dev ? ids_offsets : ws.ids_off.get<u64>();
  enqueue_scan_counts(ws.pass_count.get<uint32_t>(), n_reads, d_ids_off, st);
  u64 total = 0;
  SBWT_CUDA(cudaMemcpyAsync(&total, d_ids_off + n_reads, 8, cudaMemcpyDeviceToHost, st));
  check_colors_err(ws, st);
  if (!dev) {
    SBWT_CUDA(cudaMemcpyAsync(ids_offsets, ws.ids_off.get(), (n_reads + 1) * 8,
                              cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
  }
  if (total > capacity) throw Error(SBWT_E_CAPACITY, "ids_capacity too small");
  uint32_t *d_ids = ids;
  if (!dev) {
    ws.ids.ensure(std::max<u64>(total, 1) * 4);
    d_ids = ws.ids.get<uint32_t>();
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const u64 blocks = std::min<u64>((n_reads + 7) / 8, (u64)sms * 16);
  emit_ids_kernel<<<(unsigned)std::max<u64>(blocks, 1), 256, 0, st>>>(
      ws.pass_bits.get<u64>(), rw, d_ids_off, n_reads, d_ids, capacity);
  SBWT_CUDA(cudaGetLastError());
  if (!dev) {
    if (total)
      SBWT_CUDA(cudaMemcpyAsync(ids, d_ids, total * 4, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
  }
}

}  // namespace sbwt
