// C ABI entry points (include/sbwt_b200.h): argument checks, status codes,
// thread-local last-error message.  No exception crosses this boundary.
#include <cstring>
#include <memory>
#include <string>

#include "common.hpp"
#include "formats.hpp"
#include "colors_internal.hpp"
#include "index_internal.hpp"

namespace sbwt {
static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }
LaunchConfig &default_launch_config() {
  static LaunchConfig cfg;
  return cfg;
}
}  // namespace sbwt
namespace sbwt {
}  // namespace sbwt

using namespace sbwt;

extern "C" {

const char *sbwt_last_error(void) { return g_last_error.c_str(); }
const char *sbwt_version(void) { return "sbwt-b200 0.1 (sm_100a)"; }

int sbwt_index_from_arrays(const uint64_t *const acgt[4], uint64_t num_bits,
                           uint32_t k, const uint64_t *suffix_group_starts,
                           const uint64_t *key_kmer_marks, int device,
                           unsigned presearch_letters, sbwt_index_t **out) {
  if (!acgt || !out) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  *out = nullptr;
  return guarded([&] {
    for (int c = 0; c < 4; ++c)
      if (!acgt[c]) throw Error(SBWT_E_INVALID, "null bitvector");
    auto impl = std::make_unique<IndexImpl>(acgt, num_bits, k, suffix_group_starts,
                                            key_kmer_marks, device, presearch_letters);
    *out = new sbwt_index{impl.release()};
  });
}

int sbwt_index_open(const char *sbwt_path, const char *colors_path, int device,
                    unsigned presearch_letters, sbwt_index_t **out) {
  if (!sbwt_path || !out) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  *out = nullptr;
  return guarded([&] {
    SbwtFile f;
    try {
      f = read_sbwt(sbwt_path);
    } catch (const std::runtime_error &e) {
      std::string m = e.what();
      throw Error(m.rfind("Unable to open", 0) == 0 ? SBWT_E_IO : SBWT_E_FORMAT, m);
    }
    BitVector keys;
    if (colors_path) {
      try {
        keys = read_key_kmer_marks(colors_path);
      } catch (const std::runtime_error &e) {
        std::string m = e.what();
        throw Error(m.rfind("Unable to open", 0) == 0 ? SBWT_E_IO : SBWT_E_FORMAT, m);
      }
      if (keys.num_bits < f.acgt[0].num_bits)
        throw Error(SBWT_E_FORMAT, "key k-mer marks shorter than the SBWT");
    }
    const u64 *acgt[4] = {f.acgt[0].words.data(), f.acgt[1].words.data(),
                          f.acgt[2].words.data(), f.acgt[3].words.data()};
    const u64 *sg = f.suffix_group_starts.num_bits == f.acgt[0].num_bits
                        ? f.suffix_group_starts.words.data()
                        : nullptr;
    auto impl = std::make_unique<IndexImpl>(
        acgt, f.acgt[0].num_bits, (u32)f.k, sg,
        colors_path ? keys.words.data() : nullptr, device, presearch_letters);
    *out = new sbwt_index{impl.release()};
  });
}

void sbwt_index_free(sbwt_index_t *index) {
  if (!index) return;
  delete index->impl;
  delete index;
}

int sbwt_index_get_info(const sbwt_index_t *index, sbwt_index_info_t *info) {
  if (!index || !info) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  const IndexImpl &x = *index->impl;
  info->num_bits = x.num_bits;
  info->k = x.k;
  info->presearch_letters = x.p_max;
  for (int c = 0; c < 5; ++c) info->c_map[c] = x.c_map[c];
  info->device_bytes = x.device_bytes;
  info->device = x.device;
  info->has_key_kmer_marks = x.view.key_marks != nullptr;
  info->kmer_table_bytes = x.kmer_table.size();
  info->kmer_filter_bytes = x.kmer_filter.size();
  info->host_result_bytes = x.host_result_bytes(default_launch_config());
  info->reserved = 0;
  return SBWT_OK;
}

int sbwt_search_positions(const sbwt_index_t *index, const uint64_t *bit_seqs,
                          uint64_t n_words, const uint64_t *positions,
                          uint64_t n_positions, uint64_t *results, uint32_t flags,
                          void *stream) {
  if (!index || (n_positions && (!bit_seqs || !positions || !results))) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    if (!(flags & SBWT_DEVICE_POINTERS)) {
      const u64 cap = n_words * 32;
      for (u64 i = 0; i < n_positions; ++i)
        if (positions[i] > cap || cap - positions[i] < index->impl->k)
          throw Error(SBWT_E_INVALID, "a k-mer position lies past the end of bit_seqs");
    }
    index->impl->search_positions(bit_seqs, n_words, positions, n_positions, results,
                                  flags, static_cast<cudaStream_t>(stream),
                                  default_launch_config());
  });
}

uint64_t sbwt_count_kmers(const uint64_t *read_ends, uint64_t n_reads, uint32_t k) {
  if (!read_ends || k == 0) return 0;
  uint64_t n = 0;
  if (guarded([&] { n = count_kmers_host(read_ends, n_reads, k, 0); }) != SBWT_OK)
    return 0;
  return n;
}

int sbwt_search_reads(const sbwt_index_t *index, const char *chars, uint64_t n_chars,
                      const uint64_t *read_ends, uint64_t n_reads, uint64_t *results,
                      uint64_t results_capacity, uint64_t *n_results, uint32_t flags,
                      void *stream) {
  if (!index || (n_reads && (!read_ends || !results)) || (n_chars && !chars)) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    if ((flags & SBWT_MOVE_TO_KEY_KMER) && !index->impl->view.key_marks)
      throw Error(SBWT_E_INVALID, "SBWT_MOVE_TO_KEY_KMER needs key k-mer marks");
    if (!(flags & SBWT_DEVICE_POINTERS) && n_reads && read_ends[n_reads - 1] > n_chars)
      throw Error(SBWT_E_INVALID, "read_ends exceed n_chars");
    index->impl->search_reads(chars, n_chars, read_ends, n_reads, results,
                              results_capacity, n_results, flags,
                              static_cast<cudaStream_t>(stream),
                              default_launch_config());
  });
}

int sbwt_colors_open(const char *tcolors_path, int device, sbwt_colors_t **out) {
  if (!tcolors_path || !out) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  *out = nullptr;
  return guarded([&] {
    TColorsFile t;
    try {
      t = read_tcolors(tcolors_path);
    } catch (const std::runtime_error &e) {
      std::string m = e.what();
      throw Error(m.rfind("Unable to open", 0) == 0 ? SBWT_E_IO : SBWT_E_FORMAT, m);
    }
    auto impl = std::make_unique<ColorsImpl>(t, device);
    *out = new sbwt_colors{impl.release()};
  });
}

void sbwt_colors_free(sbwt_colors_t *colors) {
  if (!colors) return;
  delete colors->impl;
  delete colors;
}

uint64_t sbwt_colors_num_colors(const sbwt_colors_t *colors) {
  return colors ? colors->impl->num_colors : 0;
}

int sbwt_index_set_kmer_table(sbwt_index_t *index, int enable, uint64_t *table_bytes) {
  if (!index) {
    set_last_error("null index");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    IndexImpl &x = *index->impl;
    if (!enable) {
      x.drop_kmer_table();
    } else if (!x.view.kmer_table) {
      x.build_kmer_table();
    }
    x.device_bytes = x.presearch.size() + x.hot.size() + x.key_buf.size() + x.l0_all.size() +
                     x.kmer_table.size() + x.kmer_filter.size();
    if (table_bytes) *table_bytes = x.kmer_table.size();
  });
}

int sbwt_colors_set_node_table(sbwt_colors_t *colors, int enable, int *built) {
  if (!colors) {
    set_last_error("null color index");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    const bool b = colors->impl->set_node_table(enable != 0);
    if (built) *built = b ? 1 : 0;
  });
}

int sbwt_color_counts(const sbwt_colors_t *colors, const uint64_t *sbwt_idxs,
                      const uint64_t *idx_offsets, uint64_t n_reads, uint32_t *counts,
                      uint32_t flags, void *stream) {
  if (!colors || (n_reads && (!idx_offsets || !counts))) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    colors->impl->counts(sbwt_idxs, idx_offsets, n_reads, counts, flags,
                         static_cast<cudaStream_t>(stream));
  });
}

int sbwt_pseudoalign(const sbwt_colors_t *colors, const uint64_t *sbwt_idxs,
                     const uint64_t *idx_offsets, const uint64_t *not_found,
                     const uint64_t *invalid, uint64_t n_reads, double tau, uint32_t flags,
                     uint32_t *ids, uint64_t ids_capacity, uint64_t *ids_offsets,
                     void *stream) {
  if (!colors || !ids_offsets || (n_reads && !idx_offsets) ||
      ((flags & SBWT_INCLUDE_NOT_FOUND) && n_reads && !not_found) ||
      ((flags & SBWT_INCLUDE_INVALID) && n_reads && !invalid)) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  if (!(tau >= 0.0) || tau > 1.0e300) {
    set_last_error("tau must be a finite non-negative number");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    colors->impl->pseudoalign(sbwt_idxs, idx_offsets, not_found, invalid, n_reads, tau,
                              flags, ids, ids_capacity, ids_offsets,
                              static_cast<cudaStream_t>(stream));
  });
}

int sbwt_search_reads_noalloc(const sbwt_index_t *index, const char *d_chars,
                              uint64_t n_chars, const uint64_t *d_read_ends,
                              uint64_t n_reads, uint64_t *d_results,
                              uint64_t results_capacity, uint64_t *n_results,
                              uint32_t flags, void *stream) {
  if (!index || (n_reads && (!d_read_ends || !d_results)) || (n_chars && !d_chars)) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    if ((flags & SBWT_MOVE_TO_KEY_KMER) && !index->impl->view.key_marks)
      throw Error(SBWT_E_INVALID, "SBWT_MOVE_TO_KEY_KMER needs key k-mer marks");
    index->impl->search_reads_noalloc(d_chars, n_chars, d_read_ends, n_reads, d_results,
                                      results_capacity, n_results, flags,
                                      static_cast<cudaStream_t>(stream),
                                      default_launch_config());
  });
}

// Tuning hook used by the autotuner and the benchmark (not part of the
// reference-facing surface): sets the process-wide launch configuration.
int sbwt_set_launch_config(uint32_t presearch_letters, uint32_t blocks_per_sm,
                           uint64_t tile, uint64_t chunk_chars) {
  LaunchConfig &c = default_launch_config();
  const uint32_t probe = c.probe_len, l2w = c.l2_window, tk = c.table_kernel,
                 bt = c.block_threads;
  c.presearch_letters = presearch_letters;
  c.blocks_per_sm = blocks_per_sm ? blocks_per_sm : 8;
  c.tile = tile;
  c.chunk_chars = chunk_chars;
  c.probe_len = probe;
  c.l2_window = l2w;
  c.table_kernel = tk;
  c.block_threads = bt;
  return SBWT_OK;
}

// Tuning hook: threads per block of the read search kernels (128 or 256,
// the default; 0 = the default).  Results do not depend on it.
int sbwt_set_block_threads(uint32_t threads) {
  if (threads != 0 && threads != 128 && threads != 256) {
    set_last_error("block threads must be 128 or 256");
    return SBWT_E_INVALID;
  }
  default_launch_config().block_threads = threads ? threads : 256;
  return SBWT_OK;
}

// The process-wide launch configuration (what sbwt_set_launch_config,
// sbwt_set_table_kernel and sbwt_autotune set); any pointer may be NULL.
int sbwt_get_launch_config(uint32_t *presearch_letters, uint32_t *blocks_per_sm,
                           uint64_t *tile, uint64_t *chunk_chars, int *table_kernel,
                           uint32_t *block_threads) {
  const LaunchConfig &c = default_launch_config();
  if (block_threads) *block_threads = c.block_threads;
  if (presearch_letters) *presearch_letters = c.presearch_letters;
  if (blocks_per_sm) *blocks_per_sm = c.blocks_per_sm;
  if (tile) *tile = c.tile;
  if (chunk_chars) *chunk_chars = c.chunk_chars;
  if (table_kernel) *table_kernel = (int)c.table_kernel;
  return SBWT_OK;
}

// Tuning hook: persisting-L2 access-policy window over the index's rank
// blocks on the search launches (0 = off, the default; 1 = on).
int sbwt_set_l2_window(int enabled) {
  default_launch_config().l2_window = enabled ? 1u : 0u;
  return SBWT_OK;
}

// Tuning hook: length of the absent-prefix probe of the read search
// (0 = automatic, 0xFFFFFFFF = off).  Results do not depend on it.
int sbwt_set_probe_length(uint32_t probe_len) {
  default_launch_config().probe_len = probe_len;
  return SBWT_OK;
}

// Tuning hook: the read search kernel of an index with a k-mer table (see
// launch_search_kernel in index.cu): 0 general, 1 table, 2..5 walks kernel
// variants, 6 k-mers kernel, 7 automatic, 8/9/10 lean walks kernel, 11/12
// k-mers kernel with 2/8 k-mers per lane, 13/14 lean walks kernel with staged
// stores, 15 k-mers kernel with consecutive slots per lane, 16/17 lean walks
// kernel staging 8/16 slots, 18 the same with the filter and 16 slots,
// negative = the library default.  Results do not depend on it.
int sbwt_set_table_kernel(int mode) {
  if (mode > 19) {
    set_last_error("table kernel mode must be 0..19 (or negative for the default)");
    return SBWT_E_INVALID;
  }
  default_launch_config().table_kernel = mode < 0 ? kDefaultTableKernel : (uint32_t)mode;
  return SBWT_OK;
}

}  // extern "C"
