/*
 * sbwt_oracle.c -- CPU restatement of SBWT-Search's index and colors steps.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it.  The product library never links or calls it.
 *
 * Parity pinning: tests/test_oracle_golden.py checks these functions against
 * the reference's own end-to-end fixtures (test_objects/full_pipeline/
 * index_search/expected, copied into tests/golden/) and against the
 * reference's own index kernels compiled for the host (oracle/_ref).  The
 * colors step has no reference fixture that can run here (its .tcolors input is
 * not shipped with the reference), so it is pinned only by this restatement.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the SBWT-Search source tree).  Code is written from the algorithm, not
 * copied.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef uint32_t u32;
typedef uint8_t u8;

#define HYPER_BITS (1ULL << 32) /* src/Global/GlobalDefinitions.h.in:14 */
#define SUPER_BITS 1024ULL      /* src/Global/GlobalDefinitions.h.in:15 */
#define BASIC_BITS 256ULL       /* src/Global/GlobalDefinitions.h.in:16 */

static inline u64 popc(u64 x) { return (u64)__builtin_popcountll(x); }

/* ------------------------------------------------------------------------ */
/* Poppy rank index (src/PoppyBuilder/PoppyBuilder.cpp:20-70,              */
/* src/Poppy/Poppy.h:19-27).                                                */
/* layer_0[h]  = ones before hyperblock h (2^32 bits).                      */
/* layer_1_2[s] = (ones since hyperblock start before superblock s) << 32   */
/*              | b0 << 20 | b1 << 10 | b2, b_i = popcount of basic block i */
/* of the superblock (the 4th basic block count is implicit).               */
/* ------------------------------------------------------------------------ */
/* One entry more than the reference keeps in each layer, so that rank(v, N)
 * (reached by a step from an interval ending at the last node) reads a defined
 * sentinel equal to the total; the reference reads one past its layer_1_2
 * array when N is a multiple of 1024. */
void oracle_poppy_sizes(u64 num_bits, u64 *n_layer0, u64 *n_layer12) {
  *n_layer0 = num_bits / HYPER_BITS + 1;
  *n_layer12 = num_bits / SUPER_BITS + 1;
}

u64 oracle_poppy_build(const u64 *bits, u64 num_bits, u64 *layer0,
                       u64 *layer12) {
  u64 n_words = (num_bits + 63) / 64;
  u64 n_super = num_bits / SUPER_BITS + 1;
  u64 total = 0, since_hyper = 0;
  for (u64 s = 0; s < n_super; ++s) {
    u64 bit0 = s * SUPER_BITS;
    if (bit0 % HYPER_BITS == 0) {
      layer0[bit0 / HYPER_BITS] = total;
      since_hyper = 0;
    }
    u64 bb[4] = {0, 0, 0, 0};
    for (u64 w = 0; w < SUPER_BITS / 64; ++w) {
      u64 wi = bit0 / 64 + w;
      if (wi < n_words) bb[w / 4] += popc(bits[wi]);
    }
    layer12[s] = (since_hyper << 32) | (bb[0] << 20) | (bb[1] << 10) | bb[2];
    u64 sum = bb[0] + bb[1] + bb[2] + bb[3];
    since_hyper += sum;
    total += sum;
  }
  return total;
}

/* rank1(v, i) = number of set bits in positions [0, i), bits LSB-first in
 * each u64 word (src/UtilityKernels/Rank.cuh:26-65). */
u64 oracle_rank(const u64 *bits, const u64 *layer0, const u64 *layer12,
                u64 i) {
  u64 e12 = layer12[i / SUPER_BITS];
  u64 q = (i % SUPER_BITS) / BASIC_BITS; /* basic block within superblock */
  u64 b[3] = {(e12 >> 20) & 1023, (e12 >> 10) & 1023, e12 & 1023};
  u64 r = layer0[i / HYPER_BITS] + (e12 >> 32);
  for (u64 t = 0; t < q; ++t) r += b[t];
  u64 w0 = (i / BASIC_BITS) * (BASIC_BITS / 64);
  for (u64 w = w0; w < i / 64; ++w) r += popc(bits[w]);
  if (i % 64) r += popc(bits[i / 64] & ((1ULL << (i % 64)) - 1));
  return r;
}

/* Single bit test (src/UtilityKernels/GetBoolFromBitVector.cuh:19-24). */
static inline int get_bit(const u64 *bits, u64 i) {
  return (int)((bits[i / 64] >> (i % 64)) & 1ULL);
}

/* sdsl int_vector<> element read, LSB-first across word boundaries
 * (src/UtilityKernels/VariableLengthIntegerIndex.cuh:23-36). */
u64 oracle_varint(const u64 *words, u32 width, u64 idx) {
  u64 bit = idx * width, w = bit / 64, off = bit % 64;
  u64 v = words[w] >> off;
  if (off + width > 64) v |= words[w + 1] << (64 - off);
  return width == 64 ? v : (v & ((1ULL << width) - 1));
}

/* ------------------------------------------------------------------------ */
/* The SBWT handle for the oracle: 4 bitvectors with their Poppy layers and  */
/* the C-map (src/SbwtBuilder/SbwtBuilder.cpp:106-132).                      */
/* ------------------------------------------------------------------------ */
typedef struct {
  const u64 *acgt[4];
  const u64 *l0[4];
  const u64 *l12[4];
  u64 c_map[5];
} oracle_sbwt;

static inline void sbwt_step(const oracle_sbwt *s, u32 c, u64 *l, u64 *r) {
  /* One backward-search step (src/IndexSearcher/IndexSearcher.cuh:52-54). */
  *l = s->c_map[c] + oracle_rank(s->acgt[c], s->l0[c], s->l12[c], *l);
  *r = s->c_map[c] + oracle_rank(s->acgt[c], s->l0[c], s->l12[c], *r + 1) - 1;
}

static void make_sbwt(oracle_sbwt *s, const u64 *const *acgt,
                      const u64 *const *l0, const u64 *const *l12,
                      const u64 *c_map) {
  for (int c = 0; c < 4; ++c) {
    s->acgt[c] = acgt[c];
    s->l0[c] = l0[c];
    s->l12[c] = l12[c];
  }
  for (int c = 0; c < 5; ++c) s->c_map[c] = c_map[c];
}

/* C-map: c_map[0] = 1 (node 0 is the root), c_map[c+1] = c_map[c] + ones of
 * vector c (src/SbwtBuilder/SbwtBuilder.cpp:126-131). */
void oracle_c_map(const u64 totals[4], u64 c_map[5]) {
  c_map[0] = 1;
  for (int c = 0; c < 4; ++c) c_map[c + 1] = c_map[c] + totals[c];
}

/* Presearch table over all 4^p p-mers, first char in the top bits
 * (src/Presearcher/Presearcher.cuh:19-41).  The reference fixes p = 12. */
void oracle_presearch(const u64 *const *acgt, const u64 *const *l0,
                      const u64 *const *l12, const u64 *c_map, u32 p,
                      u64 *left, u64 *right) {
  oracle_sbwt s;
  make_sbwt(&s, acgt, l0, l12, c_map);
  u64 n = 1ULL << (2 * p);
  for (u64 x = 0; x < n; ++x) {
    u32 c = (u32)((x >> (2 * p - 2)) & 3);
    u64 l = s.c_map[c], r = s.c_map[c + 1] - 1;
    for (int sh = (int)(2 * p) - 4; sh >= 0; sh -= 2)
      sbwt_step(&s, (u32)((x >> sh) & 3), &l, &r);
    left[x] = l;
    right[x] = r;
  }
}

/* 2-bit code of char i of an MSB-first packed sequence, 32 chars per word
 * (src/IndexSearcher/IndexSearcher.cuh:51). */
static inline u32 packed_char(const u64 *bit_seqs, u64 i) {
  return (u32)((bit_seqs[i / 32] >> (62 - (i % 32) * 2)) & 3);
}

/* Per-k-mer search over packed sequences and k-mer start positions
 * (src/IndexSearcher/IndexSearcher.cuh:22-72): presearch lookup of the first p
 * chars, then one step per remaining char; empty interval -> UINT64_MAX.  With
 * key_marks != NULL the found node is moved forward to the next key k-mer
 * (:60-70).  Walks are independent, so no early exit changes the answer
 * (emptiness is preserved by every step because rank is monotone). */
void oracle_search(u32 k, const u64 *const *acgt, const u64 *const *l0,
                   const u64 *const *l12, const u64 *c_map, u32 p,
                   const u64 *pre_left, const u64 *pre_right,
                   const u64 *bit_seqs, const u64 *positions, u64 n,
                   const u64 *key_marks, u64 *out) {
  oracle_sbwt s;
  make_sbwt(&s, acgt, l0, l12, c_map);
  for (u64 t = 0; t < n; ++t) {
    u64 pos = positions[t];
    u64 x = 0;
    for (u32 j = 0; j < p; ++j) x = (x << 2) | packed_char(bit_seqs, pos + j);
    u64 l = pre_left[x], r = pre_right[x];
    for (u64 i = pos + p; i < pos + k; ++i) {
      if (l > r) break;
      sbwt_step(&s, packed_char(bit_seqs, i), &l, &r);
    }
    if (l > r) {
      out[t] = UINT64_MAX;
      continue;
    }
    if (key_marks) {
      while (!get_bit(key_marks, l)) {
        for (u32 c = 0; c < 4; ++c) {
          if (get_bit(acgt[c], l)) {
            l = c_map[c] + oracle_rank(acgt[c], l0[c], l12[c], l);
            break;
          }
        }
      }
    }
    out[t] = l;
  }
}

/* ASCII -> 2-bit codes A0 C1 G2 T3 (either case), MSB-first, 32 chars per
 * word; any other byte packs as 0 and is flagged in invalid[i]
 * (src/SeqToBitsConverter/CharToBits.h:33-40,
 *  src/SeqToBitsConverter/ContinuousSeqToBitsConverter.cpp:91-107). */
void oracle_seq_to_bits(const char *chars, u64 n, u64 *bit_seqs, u8 *invalid) {
  u64 n_words = (n + 31) / 32;
  memset(bit_seqs, 0, n_words * 8);
  for (u64 i = 0; i < n; ++i) {
    u64 code;
    switch (chars[i]) {
      case 'A': case 'a': code = 0; break;
      case 'C': case 'c': code = 1; break;
      case 'G': case 'g': code = 2; break;
      case 'T': case 't': code = 3; break;
      default: code = 99;
    }
    invalid[i] = (u8)(code == 99);
    if (code != 99) bit_seqs[i / 32] |= code << (62 - (i % 32) * 2);
  }
}

/* Start offset of every full k-mer of every read, in read order; reads
 * shorter than k contribute none (src/PositionsBuilder/PositionsBuilder.cpp:
 * 15-47).  read_ends[r] is the exclusive end of read r in the concatenated
 * char buffer (reads are contiguous, read 0 starts at 0).  Returns the count;
 * positions may be NULL to only count. */
u64 oracle_positions(const u64 *read_ends, u64 n_reads, u32 k,
                     u64 *positions) {
  u64 n = 0, start = 0;
  for (u64 r = 0; r < n_reads; ++r) {
    u64 end = read_ends[r];
    if (end >= start + k)
      for (u64 i = start; i + k <= end; ++i) {
        if (positions) positions[n] = i;
        ++n;
      }
    start = end;
  }
  return n;
}

/* Printer-side result mapping (src/IndexResultsPrinter/
 * ContinuousIndexResultsPrinter.hpp:196-205,266-308): a k-mer with any
 * invalid char prints -2 (UINT64_MAX-1), a not-found k-mer -1 (UINT64_MAX),
 * else its index. */
void oracle_mask_invalid(const u8 *invalid, const u64 *positions, u64 n,
                         u32 k, u64 *results) {
  for (u64 t = 0; t < n; ++t) {
    for (u32 j = 0; j < k; ++j)
      if (invalid[positions[t] + j]) {
        results[t] = UINT64_MAX - 1;
        break;
      }
  }
}

/* ------------------------------------------------------------------------ */
/* Colors step.                                                              */
/* ------------------------------------------------------------------------ */
typedef struct {
  const u64 *dense_arrays;           /* bit_vector */
  const u64 *dense_intervals;        /* int_vector<> */
  u32 dense_intervals_width;
  const u64 *sparse_arrays;          /* int_vector<> */
  u32 sparse_arrays_width;
  const u64 *sparse_intervals;       /* int_vector<> */
  u32 sparse_intervals_width;
  const u64 *is_dense;               /* bit_vector */
  const u64 *is_dense_l0, *is_dense_l12;
  const u64 *key_marks;              /* bit_vector */
  const u64 *key_l0, *key_l12;
  const u64 *color_set_idxs;         /* int_vector<> */
  u32 color_set_idxs_width;
  u64 num_colors;
} oracle_colors_index;

/* Adds the color set of one found SBWT index into counts[num_colors]
 * (src/ColorSearcher/ColorSearcher.cuh:99-111 set lookup, :208-237 dense
 * interval, :262-290 sparse interval; the per-warp ballot/popc of :174-205
 * and the per-read sum of src/ColorSearcher/ColorPostProcessor.cuh:28-42 add
 * up to one count per (found k-mer, member color)). */
static void add_color_set(const oracle_colors_index *ci, u64 sbwt_idx,
                          u64 *counts) {
  u64 j = oracle_rank(ci->key_marks, ci->key_l0, ci->key_l12, sbwt_idx);
  u64 csi = oracle_varint(ci->color_set_idxs, ci->color_set_idxs_width, j);
  u64 dense_rank = oracle_rank(ci->is_dense, ci->is_dense_l0,
                               ci->is_dense_l12, csi);
  if (get_bit(ci->is_dense, csi)) {
    u64 st = oracle_varint(ci->dense_intervals, ci->dense_intervals_width,
                           dense_rank);
    u64 en = oracle_varint(ci->dense_intervals, ci->dense_intervals_width,
                           dense_rank + 1);
    for (u64 c = 0; c < en - st; ++c)
      if (get_bit(ci->dense_arrays, st + c)) counts[c] += 1;
  } else {
    u64 q = csi - dense_rank;
    u64 st = oracle_varint(ci->sparse_intervals, ci->sparse_intervals_width, q);
    u64 en = oracle_varint(ci->sparse_intervals, ci->sparse_intervals_width,
                           q + 1);
    for (u64 t = st; t < en; ++t)
      counts[oracle_varint(ci->sparse_arrays, ci->sparse_arrays_width, t)] += 1;
  }
}

/* Per-read counts then the tau threshold
 * (src/ColorResultsPrinter/ContinuousColorResultsPrinter.hpp:235-263):
 *   seq_size = found + include_not_found*not_found + include_invalid*invalid
 *   minimum  = (u64)ceil((double)seq_size * tau)
 *   emit every color c (ascending) with count[c] >= minimum, none if 0.
 * Input per read r: the found SBWT indexes idx[idx_offsets[r] ..
 * idx_offsets[r+1]) (the colors step never sees -1/-2 entries, they are only
 * counted: src/IndexFileParser/AsciiIndexFileParser.cpp:50-64).  Output ids
 * into ids[ids_offsets[r] ..], ids_offsets has n_reads+1 entries; pass ids ==
 * NULL to size the output first.  counts_out (n_reads*num_colors) optional. */
u64 oracle_pseudoalign(const oracle_colors_index *ci, const u64 *idx,
                       const u64 *idx_offsets, const u64 *not_found,
                       const u64 *invalid, u64 n_reads, double tau,
                       int include_not_found, int include_invalid, u32 *ids,
                       u64 *ids_offsets, u64 *counts_out) {
  u64 *counts = (u64 *)malloc(ci->num_colors * sizeof(u64));
  u64 n_ids = 0;
  for (u64 r = 0; r < n_reads; ++r) {
    memset(counts, 0, ci->num_colors * sizeof(u64));
    u64 found = idx_offsets[r + 1] - idx_offsets[r];
    for (u64 t = idx_offsets[r]; t < idx_offsets[r + 1]; ++t)
      add_color_set(ci, idx[t], counts);
    if (counts_out)
      memcpy(counts_out + r * ci->num_colors, counts,
             ci->num_colors * sizeof(u64));
    u64 seq_size = found + (include_not_found ? not_found[r] : 0) +
                   (include_invalid ? invalid[r] : 0);
    u64 minimum = (u64)ceil((double)seq_size * tau);
    ids_offsets[r] = n_ids;
    for (u64 c = 0; minimum > 0 && c < ci->num_colors; ++c)
      if (counts[c] >= minimum) {
        if (ids) ids[n_ids] = (u32)c;
        ++n_ids;
      }
  }
  ids_offsets[n_reads] = n_ids;
  free(counts);
  return n_ids;
}

/* oracle_pseudoalign over reads on `threads` host threads (OpenMP), for the
 * colors CPU baseline: per read only the number of passing colors and a
 * checksum of their ids (sum over passing c of (c + 1) * (index in the read's
 * list + 1)), so that no R x C count matrix is kept.  Returns the total. */
u64 oracle_pseudoalign_mt(const oracle_colors_index *ci, const u64 *idx,
                          const u64 *idx_offsets, const u64 *not_found,
                          const u64 *invalid, u64 n_reads, double tau,
                          int include_not_found, int include_invalid,
                          u64 *n_ids_out, u64 *checksum_out, int threads) {
  u64 total = 0;
#pragma omp parallel num_threads(threads) reduction(+ : total)
  {
    u64 *counts = (u64 *)malloc(ci->num_colors * sizeof(u64));
#pragma omp for schedule(dynamic, 256)
    for (long rr = 0; rr < (long)n_reads; ++rr) {
      const u64 r = (u64)rr;
      memset(counts, 0, ci->num_colors * sizeof(u64));
      u64 found = idx_offsets[r + 1] - idx_offsets[r];
      for (u64 t = idx_offsets[r]; t < idx_offsets[r + 1]; ++t)
        add_color_set(ci, idx[t], counts);
      u64 seq_size = found + (include_not_found ? not_found[r] : 0) +
                     (include_invalid ? invalid[r] : 0);
      u64 minimum = (u64)ceil((double)seq_size * tau);
      u64 n = 0, h = 0;
      for (u64 c = 0; minimum > 0 && c < ci->num_colors; ++c)
        if (counts[c] >= minimum) {
          ++n;
          h += (c + 1) * n;
        }
      n_ids_out[r] = n;
      checksum_out[r] = h;
      total += n;
    }
    free(counts);
  }
  return total;
}

/* Sectors-touched instrumentation for the index walk: counts, per k-mer, the
 * distinct 32-byte sectors of the A/C/G/T bitvectors that the reference walk
 * (steps p..k-1, stopping at the first empty interval) reads.  Used only to
 * state the algorithmic bytes of the roofline. */
u64 oracle_walk_sectors(u32 k, const u64 *const *acgt, const u64 *const *l0,
                        const u64 *const *l12, const u64 *c_map, u32 p,
                        const u64 *pre_left, const u64 *pre_right,
                        const u64 *bit_seqs, const u64 *positions, u64 n) {
  oracle_sbwt s;
  make_sbwt(&s, acgt, l0, l12, c_map);
  u64 sectors = 0;
  for (u64 t = 0; t < n; ++t) {
    u64 pos = positions[t], x = 0;
    for (u32 j = 0; j < p; ++j) x = (x << 2) | packed_char(bit_seqs, pos + j);
    u64 l = pre_left[x], r = pre_right[x];
    for (u64 i = pos + p; i < pos + k && l <= r; ++i) {
      u32 c = packed_char(bit_seqs, i);
      u64 sa = l / 256, sb = (r + 1) / 256;
      sectors += (sa == sb) ? 1 : 2;
      sbwt_step(&s, c, &l, &r);
    }
  }
  return sectors;
}
