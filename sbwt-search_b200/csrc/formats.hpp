// File formats of SBWT-Search kept byte-compatible by this library:
//   * .sbwt / .tdbg  -- plain-matrix SBWT (SbwtBuilder.cpp:58-104 of the
//     reference reads it);
//   * .tcolors       -- Themisto "sdsl-hybrid-v4" color index
//     (ColorIndexBuilder.cpp:23-86 of the reference reads it);
//   * length-prefixed strings (Tools/IOUtils.cpp:44-57 of the reference).
// The serialized layouts of sdsl's bit_vector / int_vector<> / rank blobs are
// restated here from the published sdsl format: bit_vector = u64 length in bits
// + ceil(bits/64) u64 words; int_vector<> = u64 length in bits + u8 width +
// ceil(bits/64) words; rank_support_v5 = an int_vector<64> blob.
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <utility>
#include <vector>

namespace sbwt {

using u64 = uint64_t;
using u32 = uint32_t;
using u8 = uint8_t;

// A vector whose resize leaves new elements uninitialised (they are all
// written next), so multi-GB arrays read from files are not cleared first.
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
  template <class U>
  void construct(U *p) noexcept {
    ::new (static_cast<void *>(p)) U;
  }
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
  }
};
using U64Array = std::vector<u64, NoInitAlloc<u64>>;

struct BitVector {
  u64 num_bits = 0;
  U64Array words;  // ceil(num_bits / 64) words, LSB-first bits
  bool get(u64 i) const { return (words[i / 64] >> (i % 64)) & 1ULL; }
  void set(u64 i) { words[i / 64] |= 1ULL << (i % 64); }
  void resize(u64 bits) {
    num_bits = bits;
    words.assign((bits + 63) / 64, 0);
  }
};

struct IntVector {  // sdsl int_vector<> (variable width), LSB-first packing
  u64 num_bits = 0;
  u8 width = 64;
  U64Array words;
  u64 size() const { return width ? num_bits / width : 0; }
  u64 get(u64 idx) const;
  void assign(const std::vector<u64> &values, u8 width);
};

// The plain-matrix SBWT: 4 bitvectors, the suffix-group-start bitvector and
// the scalars of the file.  Rank blobs / C-map / prefix table are not kept.
struct SbwtFile {
  BitVector acgt[4];
  BitVector suffix_group_starts;
  u64 precalc_k = 0, n_nodes = 0, n_kmers = 0, k = 0;
};

// Reads a .sbwt or .tdbg file.  Throws std::runtime_error with the
// reference's messages on bad magic ("Error input is not a plain-matrix
// SBWT", "Error: wrong SBWT version").
SbwtFile read_sbwt(const std::string &path);
// Writes a plain-matrix .sbwt (rank blobs in sdsl rank_support_v5 layout,
// C-map, an empty prefix table with precalc_k = 0).
void write_sbwt(const std::string &path, const SbwtFile &s);

// Themisto sdsl-hybrid-v4 color index.
struct TColorsFile {
  BitVector dense_arrays;
  IntVector dense_arrays_intervals;
  IntVector sparse_arrays;
  IntVector sparse_arrays_intervals;
  BitVector is_dense_marks;
  BitVector key_kmer_marks;
  IntVector color_set_idxs;
  u64 max_color_set_idx = 0;  // first trailing u64
  u64 largest_color = 0;      // second trailing u64 (num_colors = this + 1)
  u64 sum_color_set_sizes = 0;  // third trailing u64
  u64 num_colors() const { return largest_color + 1; }
};

TColorsFile read_tcolors(const std::string &path);
void write_tcolors(const std::string &path, const TColorsFile &t);
// Only the key-k-mer marks (for the index step's -k option).
BitVector read_key_kmer_marks(const std::string &path);

// sdsl rank_support_v5 blob for bv (restated from the published sdsl layout).
std::vector<u64> rank_v5_blob(const BitVector &bv);

}  // namespace sbwt
