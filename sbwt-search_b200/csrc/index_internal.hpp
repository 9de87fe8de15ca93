// Internal C++ view of the index handle (behind the sbwt_index_t C type).
#pragma once

#include <cuda_runtime.h>

#include "common.hpp"
#include "device_layout.hpp"

namespace sbwt {

// Launch parameters chosen by the autotuner (0 = built-in default).
// Deepest presearch table (4^14 entries: 2 GiB at 8 bytes per entry, 2.9 GB
// with the shallower levels); the reference fixes 12.
constexpr uint32_t kPresearchMaxLetters = 14;
// Largest k-mer table an index builds (16 bytes per slot, <= 2 slots per k-mer).
constexpr u64 kKmerTableMaxBytes = 32ULL << 30;
// Bits per k-mer of the k-mer filter built with the table.
constexpr u64 kFilterBitsPerKmer = 10;

// Read search kernel of an index with a k-mer table by default
// (LaunchConfig::table_kernel): automatic (the k-mers kernel for small
// tables, else the table kernel).
constexpr uint32_t kDefaultTableKernel = 7;

struct LaunchConfig {
  uint32_t presearch_letters = 0;  // <= the handle's pyramid depth
  uint32_t blocks_per_sm = 8;      // blocks per SM in the grid
  uint32_t block_threads = 256;    // threads per block of the read search (128 or 256)
  uint64_t tile = 0;               // k-mer slots per work tile
  uint64_t chunk_chars = 0;        // host-pointer path: chars per chunk (when set, also
                                   // the piece size of device-pointer batches)
  uint32_t probe_len = 0;          // absent-prefix probe length (0 = auto, ~0u = off)
  uint32_t l2_window = 0;          // persisting L2 window over the index's hot data
  uint32_t table_kernel = kDefaultTableKernel;  // read search kernel with a k-mer table
                                               // (0 general, 1 table, 2-4 walks)
};

struct IndexImpl {
  IndexImpl(const u64 *const acgt[4], u64 num_bits, u32 k, const u64 *sg,
            const u64 *key_marks, int device, unsigned presearch_letters);

  SbwtView view_for(u32 p) const;
  // k-mer -> node hash table (k <= 31) and its k-mer filter: false when not
  // built
  bool build_kmer_table();
  void drop_kmer_table();

  void search_positions(const u64 *bit_seqs, u64 n_words, const u64 *positions,
                        u64 n, u64 *results, u32 flags, cudaStream_t st,
                        const LaunchConfig &cfg) const;
  void search_reads(const char *chars, u64 n_chars, const u64 *read_ends,
                    u64 n_reads, u64 *results, u64 capacity, u64 *n_results,
                    u32 flags, cudaStream_t st, const LaunchConfig &cfg) const;

  // Device-pointer read search of 2^32 or more chars: pieces of at most 2^31
  // chars (whole reads), each on the 32-bit kernels.
  void search_reads_device_pieces(const char *chars, u64 n_chars, const u64 *read_ends,
                                  u64 n_reads, u64 *results, u64 capacity, u64 *n_results,
                                  u32 flags, cudaStream_t st, const LaunchConfig &cfg) const;

  // Bytes per k-mer result that a host-pointer sbwt_search_reads moves from
  // the device with default flags: 4 on the walks kernel, else 8.
  u32 host_result_bytes(const LaunchConfig &cfg) const;

  void search_reads_noalloc(const char *d_chars, u64 n_chars, const u64 *d_ends,
                            u64 n_reads, u64 *d_results, u64 capacity, u64 *n_results,
                            u32 flags, cudaStream_t st, const LaunchConfig &cfg) const;

  int device = 0;
  u64 num_bits = 0;
  u32 k = 0;
  u32 p_max = 12;
  u32 wide = 0;
  u64 c_map[5] = {0, 0, 0, 0, 0};
  u64 device_bytes = 0;
  SbwtView view{};
  DeviceBuffer hot;  // rank blocks of A/C/G/T + suffix-group words, contiguous
  DeviceBuffer l0_all, presearch, key_buf, kmer_table, kmer_filter;
  u64 table_kmers = 0;
  u64 window_bytes = 0;   // L2 access-policy window over `hot`
};

u64 count_kmers_host(const u64 *ends, u64 n_reads, u32 k, u64 base);

// Device scratch of one read batch: scan outputs, packed chars, invalid
// bits, the tile table, the error word and the work-queue counter.
struct ReadsScratch {
  u64 *kmer_off;      // n_reads + 1
  u64 *packed;        // n_words + 2
  uint32_t *invalid;  // n_words + 2
  u64 *block_sums;    // ceil(n_reads / 4096) + 1
  u64 *total;         // 1
  u64 *tile_read;     // n_tiles + 2
  uint32_t *err;      // 1
  unsigned long long *queue;  // 1
};

void enqueue_index_step(const IndexImpl &ix, const char *d_chars, u64 n_chars,
                        const u64 *d_ends, u64 n_reads, const ReadsScratch &sc, u64 *d_out,
                        u64 out_capacity, u64 max_kmers, u32 flags, const LaunchConfig &cfg,
                        cudaStream_t st);
u64 index_tile_size(const IndexImpl &ix, u64 max_kmers, const LaunchConfig &cfg);
LaunchConfig &default_launch_config();

}  // namespace sbwt

struct sbwt_index {
  sbwt::IndexImpl *impl;
};
