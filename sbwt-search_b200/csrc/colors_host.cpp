// Host layout of a .tcolors color index for the device: one packed record per
// color set, the dense rows copied word by word onto their alignment, the
// sparse ids widened to u32.  The set loop that places the rows is serial
// (a few loads per set); the copies run on host threads.
//
// File layout restated: ColorIndexBuilder/ColorIndexBuilder.cpp:23-86 of the
// reference (dense rows are bit ranges of one bitvector delimited by
// dense_arrays_intervals, sparse lists are ranges of an int vector delimited
// by sparse_arrays_intervals, is_dense_marks tells which kind set s is).
#include <algorithm>
#include <atomic>
#include <vector>

#include "colors_internal.hpp"
#include "host_threads.hpp"

namespace sbwt {

HostColorSets prepare_color_sets(const TColorsFile &t) {
  const u64 num_colors = t.num_colors();
  const u64 n_sets = t.is_dense_marks.num_bits;
  const u64 n_ids = t.sparse_arrays.size();
  HostColorSets h;
  h.recs.resize(std::max<u64>(n_sets, 1));
  h.sparse.resize(std::max<u64>(n_ids, 1));
  std::atomic<bool> bad_id{false};
  run_parts(n_ids, host_threads(n_ids, 1 << 20, 32), [&](u64 lo, u64 hi) {
    bool bad = false;
    for (u64 i = lo; i < hi; ++i) {
      const u64 v = t.sparse_arrays.get(i);
      bad |= v >= num_colors;
      h.sparse[i] = (uint32_t)v;
    }
    if (bad) bad_id = true;
  });
  if (bad_id) throw Error(SBWT_E_FORMAT, "sparse color id out of range");

  // Places the sets: a dense row starts on a 64-byte boundary (on its own
  // size when smaller), so it spans the fewest sectors and DRAM bursts.
  struct Row {
    u64 src_bit, at, nbits;
  };
  std::vector<Row> rows;
  std::vector<u64> lists;  // start, end of each sparse list
  u64 n_dense = 0, n_sparse = 0, n_words = 0;
  const u64 n_dense_iv = t.dense_arrays_intervals.size();
  const u64 n_sparse_iv = t.sparse_arrays_intervals.size();
  for (u64 s = 0; s < n_sets; ++s) {
    if (t.is_dense_marks.get(s)) {
      if (n_dense + 1 >= n_dense_iv) throw Error(SBWT_E_FORMAT, "dense intervals too short");
      const u64 st = t.dense_arrays_intervals.get(n_dense);
      const u64 en = t.dense_arrays_intervals.get(n_dense + 1);
      if (en < st || en > t.dense_arrays.num_bits || en - st > num_colors)
        throw Error(SBWT_E_FORMAT, "dense interval out of range");
      const u64 nbits = en - st, nw = (nbits + 63) / 64;
      const u64 align = nw >= 8 ? 8 : nw >= 4 ? 4 : nw >= 2 ? 2 : 1;
      const u64 at = (n_words + align - 1) / align * align;
      rows.push_back({st, at, nbits});
      n_words = at + nw;
      h.recs[s] = make_rec(at, nw, true);
      ++n_dense;
    } else {
      if (n_sparse + 1 >= n_sparse_iv) throw Error(SBWT_E_FORMAT, "sparse intervals too short");
      const u64 st = t.sparse_arrays_intervals.get(n_sparse);
      const u64 en = t.sparse_arrays_intervals.get(n_sparse + 1);
      if (en < st || en > n_ids) throw Error(SBWT_E_FORMAT, "sparse interval out of range");
      if (en - st >= (1ULL << kRecLenBits)) throw Error(SBWT_E_FORMAT, "sparse color set too long");
      lists.push_back(st);
      lists.push_back(en);
      h.recs[s] = make_rec(st, en - st, false);
      ++n_sparse;
    }
  }
  if (std::max<u64>(n_words, n_ids) >= (1ULL << (63 - kRecLenBits)))
    throw Error(SBWT_E_FORMAT, "color arrays too large");

  // Dense rows: 64 source bits per output word (two words shifted together),
  // the last word masked; alignment gaps stay zero.
  h.dense_words.assign(std::max<u64>(n_words, 1), 0);
  const u64 *src = t.dense_arrays.words.data();
  const u64 src_words = t.dense_arrays.words.size();
  run_parts(rows.size(), host_threads(rows.size(), 1 << 14, 32), [&](u64 lo, u64 hi) {
    for (u64 r = lo; r < hi; ++r) {
      const Row &row = rows[r];
      u64 *out = h.dense_words.data() + row.at;
      for (u64 j = 0; j * 64 < row.nbits; ++j) {
        const u64 bit = row.src_bit + j * 64, w = bit / 64, o = bit % 64;
        u64 v = src[w] >> o;
        if (o && w + 1 < src_words) v |= src[w + 1] << (64 - o);
        const u64 rem = row.nbits - j * 64;
        out[j] = rem >= 64 ? v : v & ((1ULL << rem) - 1);
      }
    }
  });

  // Every sparse list strictly ascending?
  std::atomic<bool> unsorted{false};
  run_parts(lists.size() / 2, host_threads(lists.size() / 2, 1 << 14, 32), [&](u64 lo, u64 hi) {
    for (u64 l = lo; l < hi && !unsorted.load(std::memory_order_relaxed); ++l)
      for (u64 i = lists[2 * l] + 1; i < lists[2 * l + 1]; ++i)
        if (h.sparse[i - 1] >= h.sparse[i]) {
          unsorted = true;
          break;
        }
  });
  h.sparse_sorted = !unsorted;
  return h;
}

}  // namespace sbwt
