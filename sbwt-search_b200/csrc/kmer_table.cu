// The k-mer table of an index: every k-mer of the SBWT (k <= 31) -> its node,
// in an open-addressing hash table on the device.  It extends the presearch
// idea (a table lookup replaces the first p search steps) to the whole
// k-mer: a read k-mer that cannot be reached by a stream step from the
// previous k-mer costs one table lookup instead of a presearch lookup and
// k - p backward-search steps.  (A failed stream step still starts the
// absent-prefix probe, which proves a run of the following k-mers absent
// with one presearch lookup.)  Results are identical: the table holds exactly
// the k-mers of the SBWT with their nodes.
//
// Labels are recovered from the SBWT itself: the last char of node v is the
// c with C[c] <= v < C[c + 1] (node 0 is the root, all '$'), and its
// predecessor (the node whose marked c-edge reaches v) is the
// (v - C[c])-th set bit of vector c.  k rounds of "char, then predecessor"
// over all nodes spell every label; a node whose chain reaches the root
// within k chars is a dummy ($-padded) and is not a k-mer.
//
// Table: 2^m slots of 16 bytes (key, node), key = the k chars with the first
// char on top (2 bits each), empty = ~0; a key's probe sequence starts at an
// even slot (so a 32-byte sector holds the first two slots it probes) and
// moves one slot at a time; at most half of the slots are used.
//
// Filter: beside the table, a blocked Bloom filter of the same keys, 10 bits
// per k-mer, one 64-bit word per key with four of its bits set
// (kmer_filter_word / kmer_filter_bits).  It is 25x smaller than the table
// (144 MB for 115 M k-mers against 4 GiB), so a read k-mer that is absent
// -- most k-mers that a stream step cannot reach -- is answered from a
// structure inside the GPU's address-translation reach and mostly in L2,
// and only k-mers the filter passes pay a table lookup.  A filter answer of
// "absent" is exact (no false negatives), so results do not change.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>

#include "index_internal.hpp"
#include "rank_blocks.cuh"

namespace sbwt {

namespace {

// Word w of a bitvector, read from its rank blocks (three payload words per
// block, in order).
__device__ __forceinline__ uint64_t vec_word(const Block *blocks, uint64_t w) {
  const Block &b = blocks[w / 3];
  const uint32_t j = (uint32_t)(w % 3);
  return j == 0 ? b.w0 : (j == 1 ? b.w1 : b.w2);
}

__global__ void word_ones_kernel(const Block *blocks, uint64_t n_words, uint64_t *cnt) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n_words; w += step)
    cnt[w] = __popcll(vec_word(blocks, w));
}

// positions of the set bits of one vector, in order
__global__ void ones_positions_kernel(const Block *blocks, uint64_t n_words,
                                      const uint64_t *off, uint64_t *pos) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n_words; w += step) {
    uint64_t m = vec_word(blocks, w), o = off[w];
    while (m) {
      pos[o++] = w * 64 + __ffsll((long long)m) - 1;
      m &= m - 1;
    }
  }
}

struct LabelView {
  const uint64_t *ones[4];
  uint64_t c_map[5];
};

// One round of label recovery: the char of cur[v] lands at bits 2t of key[v],
// and cur[v] moves to its predecessor; a chain that reaches the root marks a
// dummy (alive = 0).
__global__ void label_round_kernel(LabelView lv, uint64_t n, uint32_t t, uint64_t *cur,
                                   uint64_t *key, uint8_t *alive) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += step) {
    if (!alive[v]) continue;
    const uint64_t x = t == 0 ? v : cur[v];
    if (x == 0) {
      alive[v] = 0;
      continue;
    }
    uint32_t c = 0;
    while (c < 3 && x >= lv.c_map[c + 1]) ++c;
    key[v] = (t == 0 ? 0 : key[v]) | ((uint64_t)c << (2 * t));
    cur[v] = lv.ones[c][x - lv.c_map[c]];
  }
}

// k-mers (alive nodes), one atomic per warp
__global__ void count_alive_kernel(const uint8_t *alive, uint64_t n, unsigned long long *out) {
  unsigned long long c = 0;
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += step)
    c += alive[v];
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void table_insert_kernel(const uint64_t *key, const uint8_t *alive, uint64_t n,
                                    uint64_t *table, uint64_t mask, uint32_t *err) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += step) {
    if (!alive[v]) continue;
    const unsigned long long kk = key[v];
    uint64_t s = kmer_table_bucket(kk, mask);
    for (uint64_t tries = 0; tries <= mask; ++tries) {
      const unsigned long long old =
          atomicCAS((unsigned long long *)(table + 2 * s), ~0ULL, kk);
      if (old == ~0ULL) {
        table[2 * s + 1] = v;
        break;
      }
      if (old == kk) {  // a k-mer twice: the SBWT is malformed
        atomicOr(err, 1u);
        break;
      }
      s = (s + 1) & mask;
    }
  }
}

__global__ void filter_insert_kernel(const uint64_t *key, const uint8_t *alive, uint64_t n,
                                     unsigned long long *filter, uint64_t n_words) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += step) {
    if (!alive[v]) continue;
    const uint64_t z = kmer_mix(key[v]);
    atomicOr(filter + kmer_filter_word(z, n_words), (unsigned long long)kmer_filter_bits(z));
  }
}

unsigned grid_of(uint64_t n) {
  return (unsigned)std::max<uint64_t>(std::min<uint64_t>((n + 255) / 256, 148 * 32), 1);
}

}  // namespace

// Builds the table from the index's rank blocks.  Returns false (and builds
// nothing) when k > 31 or the table would not fit in kKmerTableMaxBytes or a
// quarter of the free device memory.
bool IndexImpl::build_kmer_table() {
  DeviceGuard g(device);
  drop_kmer_table();
  if (k > 31 || k < 2) return false;
  const u64 n = num_bits, nw = (num_bits + 63) / 64;
  // predecessor tables: positions of the ones of each vector
  DeviceBuffer cnt((nw + 1) * 8), ones[4];
  size_t tb = 0;
  DeviceBuffer tmp;
  LabelView lv{};
  for (int c = 0; c < 5; ++c) lv.c_map[c] = c_map[c];
  for (int c = 0; c < 4; ++c) {
    const u64 total = c_map[c + 1] - c_map[c];
    ones[c].resize(std::max<u64>(total, 1) * 8);
    word_ones_kernel<<<grid_of(nw), 256>>>(view.blocks[c], nw, cnt.get<u64>());
    SBWT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.get<u64>(), cnt.get<u64>(),
                                            (int64_t)nw));
    tmp.ensure(std::max<size_t>(tb, 1));
    SBWT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, cnt.get<u64>(), cnt.get<u64>(),
                                            (int64_t)nw));
    ones_positions_kernel<<<grid_of(nw), 256>>>(view.blocks[c], nw, cnt.get<u64>(),
                                                ones[c].get<u64>());
    SBWT_CUDA(cudaGetLastError());
    lv.ones[c] = ones[c].get<u64>();
  }
  cnt.release();
  // labels
  DeviceBuffer cur(n * 8), key(n * 8), alive(n);
  SBWT_CUDA(cudaMemset(alive.get(), 1, n));
  for (u32 t = 0; t < k; ++t)
    label_round_kernel<<<grid_of(n), 256>>>(lv, n, t, cur.get<u64>(), key.get<u64>(),
                                            alive.get<uint8_t>());
  SBWT_CUDA(cudaGetLastError());
  for (auto &o : ones) o.release();
  cur.release();
  // k-mer count -> table size (load <= 1/2)
  DeviceBuffer d_n(8);
  SBWT_CUDA(cudaMemset(d_n.get(), 0, 8));
  count_alive_kernel<<<grid_of(n), 256>>>(alive.get<uint8_t>(), n,
                                          d_n.get<unsigned long long>());
  SBWT_CUDA(cudaGetLastError());
  u64 n_kmers = 0;
  SBWT_CUDA(cudaMemcpy(&n_kmers, d_n.get(), 8, cudaMemcpyDeviceToHost));
  u64 slots = 2;
  while (slots < 2 * n_kmers) slots <<= 1;
  size_t free_b = 0, total_b = 0;
  SBWT_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const u64 filter_words = std::max<u64>((n_kmers * kFilterBitsPerKmer + 63) / 64, 1);
  if (slots > (1ULL << 32) || slots * 16 > kKmerTableMaxBytes ||
      slots * 16 + filter_words * 8 > free_b / 4)
    return false;
  kmer_table.resize(slots * 16);
  SBWT_CUDA(cudaMemset(kmer_table.get(), 0xFF, slots * 16));
  DeviceBuffer d_err(4);
  SBWT_CUDA(cudaMemset(d_err.get(), 0, 4));
  table_insert_kernel<<<grid_of(n), 256>>>(key.get<u64>(), alive.get<uint8_t>(), n,
                                           kmer_table.get<u64>(), slots - 1,
                                           d_err.get<uint32_t>());
  SBWT_CUDA(cudaGetLastError());
  uint32_t e = 0;
  SBWT_CUDA(cudaMemcpy(&e, d_err.get(), 4, cudaMemcpyDeviceToHost));
  if (e) {
    kmer_table.release();
    throw Error(SBWT_E_FORMAT, "an SBWT k-mer occurs twice");
  }
  kmer_filter.resize(filter_words * 8);
  SBWT_CUDA(cudaMemset(kmer_filter.get(), 0, filter_words * 8));
  filter_insert_kernel<<<grid_of(n), 256>>>(key.get<u64>(), alive.get<uint8_t>(), n,
                                            kmer_filter.get<unsigned long long>(),
                                            filter_words);
  SBWT_CUDA(cudaGetLastError());
  view.kmer_table = kmer_table.get<u64>();
  view.kmer_table_mask = slots - 1;
  view.kmer_filter = kmer_filter.get<u64>();
  view.filter_words = filter_words;
  table_kmers = n_kmers;
  return true;
}

void IndexImpl::drop_kmer_table() {
  DeviceGuard g(device);
  kmer_table.release();
  kmer_filter.release();
  view.kmer_table = nullptr;
  view.kmer_table_mask = 0;
  view.kmer_filter = nullptr;
  view.filter_words = 0;
  table_kmers = 0;
}

}  // namespace sbwt
