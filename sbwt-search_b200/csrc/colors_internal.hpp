// Internal C++ view of the color index handle (behind sbwt_colors_t).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.hpp"
#include "device_layout.hpp"
#include "formats.hpp"

namespace sbwt {

constexpr u64 kNodeTableMaxBytes = 16ULL << 30;  // per-node record table cap

// Packed set record: start (42 bits) | len (21 bits) | dense (1 bit).  len is
// row words for a dense set, ids for a sparse one; start indexes the dense
// words or the sparse ids.
constexpr uint64_t kRecNone = ~0ULL;
constexpr int kRecLenBits = 21;
__host__ __device__ __forceinline__ uint64_t make_rec(uint64_t start, uint64_t len, bool dense) {
  return (start << (kRecLenBits + 1)) | (len << 1) | (dense ? 1ULL : 0ULL);
}

// Host images of the color set arrays the device keeps: one record per color
// set, the dense rows (each on its own alignment, gaps zero) and the sparse
// ids as u32.
struct HostColorSets {
  std::vector<u64> recs;
  std::vector<u64> dense_words;
  std::vector<uint32_t> sparse;
  bool sparse_sorted = true;  // every sparse list strictly ascending
};
// Checks and lays out the color sets of t (host threads); throws Error
// (SBWT_E_FORMAT) on malformed intervals or ids.
HostColorSets prepare_color_sets(const TColorsFile &t);

// Device view of the color index.
struct ColorsView {
  const Block *key_blocks;  // rank blocks of the key k-mer marks
  const uint64_t *key_l0;
  uint64_t key_bits;
  const uint32_t *csi;      // color set id per key k-mer
  uint64_t n_keys;
  const uint64_t *recs;     // per set: start << 22 | len << 1 | dense
  uint64_t n_sets;
  const uint64_t *node_rec; // per SBWT node: the record of its color set, or nullptr
  const uint64_t *dense;    // word-aligned dense rows
  const uint32_t *sparse;   // sparse color ids
  uint32_t num_colors;
  uint32_t row_words;       // ceil(num_colors / 64)
  uint32_t words_per_lane;  // row words per lane in one color tile (<= 4)
  uint32_t tiles;           // color tiles per read: ceil(row_words / (32 * words_per_lane))
  uint32_t sparse_sorted;   // 1 when every sparse list is strictly ascending
};

struct ColorsImpl {
  ColorsImpl(const TColorsFile &t, int device);
  // Per-read counts (n_reads x num_colors u32).
  void counts(const u64 *vals, const u64 *offs, u64 n_reads, uint32_t *out, u32 flags,
              cudaStream_t st) const;
  // Threshold + sorted ids.
  void pseudoalign(const u64 *vals, const u64 *offs, const u64 *nf, const u64 *inv,
                   u64 n_reads, double tau, u32 flags, uint32_t *ids, u64 capacity,
                   u64 *ids_offsets, cudaStream_t st) const;
  void launch(const u64 *d_vals, const u64 *d_offs, const u64 *d_nf, const u64 *d_inv,
              u64 n_reads, u64 max_kmers, double tau, u32 flags, int mode,
              u64 *d_pass_bits, uint32_t *d_pass_count, uint32_t *d_counts,
              uint32_t *d_err, cudaStream_t st) const;

  void enqueue_pseudoalign(const u64 *d_vals, const u64 *d_offs, u64 n_reads, u64 max_kmers,
                           double tau, u32 flags, u64 *d_pass_bits, uint32_t *d_pass_count,
                           u64 *d_ids_off, uint32_t *d_ids, u64 ids_capacity,
                           uint32_t *d_err, cudaStream_t st) const;
  // sets the shared-memory attribute for batches of up to max_kmers k-mers per
  // read (must precede a stream capture)
  void prepare_launch(u64 max_kmers) const;
  // builds (or drops) the per-node set record table; false when not built
  bool set_node_table(bool enable);
  u64 device_footprint() const;

  int device = 0;
  u64 num_colors = 0;
  u64 device_bytes = 0;
  DeviceBuffer key_blocks, key_l0, csi_buf, recs_buf, dense_buf, sparse_buf, node_buf;
  ColorsView view{};
};

}  // namespace sbwt

struct sbwt_colors {
  sbwt::ColorsImpl *impl;
};
