// Project tool: builds a plain-matrix SBWT (and optionally a Themisto-layout
// .tcolors color index) from DNA sequences, plus seeded synthetic genomes and
// reads.  SBWT-Search does not build indexes itself (Themisto does), so these
// tools exist to produce test and benchmark inputs in the reference's formats.
//
// SBWT definition used (Alanko et al., "Small searchable k-spectra via subset
// rank queries on the spectral Burrows-Wheeler transform"):
//   nodes  = the k-mers, plus for every k-mer x without a predecessor the
//            dummy nodes $^(k-i) x[0..i) for i = 0..k-1 ($ sorts first);
//   order  = colexicographic (compare last char first);
//   edges  = node u -> w labelled w[k-1] iff u[1..k) == w[0..k-1); the label
//            bit is stored only at the first node of u's suffix group (nodes
//            sharing u[1..k)), so every non-root node has exactly one marked
//            incoming edge and the C-map search of the reference works.
// Node encoding: key = sum code(label[t]) << 2t with $ and A both coded 0,
// plus len = number of non-$ chars; (key, len) ascending is the colex order.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../formats.hpp"

namespace sbwt {
namespace tools {

// Phase timing on stderr when SBWT_TOOLS_VERBOSE is set.
static double wall() { return omp_get_wtime(); }
static void phase(const char *name, double &t) {
  if (std::getenv("SBWT_TOOLS_VERBOSE")) std::fprintf(stderr, "[tools] %-28s %.2f s\n", name, wall() - t);
  t = wall();
}

static inline int code_of(char c) {
  switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return -1;
  }
}

// Parallel sort + unique of u64 keys: bucket by the top bits, sort buckets.
static void sort_unique(std::vector<u64> &v) {
  const int B = 4096;
  const int shift = 64 - 12;
  int T = omp_get_max_threads();
  std::vector<std::vector<u64>> cnt(T, std::vector<u64>(B, 0));
  u64 n = v.size();
#pragma omp parallel
  {
    int t = omp_get_thread_num();
#pragma omp for schedule(static)
    for (u64 i = 0; i < n; ++i) cnt[t][v[i] >> shift]++;
  }
  std::vector<u64> start(B + 1, 0);
  std::vector<std::vector<u64>> off(T, std::vector<u64>(B, 0));
  u64 acc = 0;
  for (int b = 0; b < B; ++b) {
    start[b] = acc;
    for (int t = 0; t < T; ++t) {
      off[t][b] = acc;
      acc += cnt[t][b];
    }
  }
  start[B] = acc;
  std::vector<u64> out(n);
#pragma omp parallel
  {
    int t = omp_get_thread_num();
#pragma omp for schedule(static)
    for (u64 i = 0; i < n; ++i) out[off[t][v[i] >> shift]++] = v[i];
  }
  std::vector<u64> uniq_cnt(B, 0);
#pragma omp parallel for schedule(dynamic, 8)
  for (int b = 0; b < B; ++b) {
    auto first = out.begin() + start[b], last = out.begin() + start[b + 1];
    std::sort(first, last);
    uniq_cnt[b] = std::unique(first, last) - first;
  }
  std::vector<u64> dst(B + 1, 0);
  for (int b = 0; b < B; ++b) dst[b + 1] = dst[b] + uniq_cnt[b];
  v.resize(dst[B]);
#pragma omp parallel for schedule(dynamic, 8)
  for (int b = 0; b < B; ++b)
    std::copy(out.begin() + start[b], out.begin() + start[b] + uniq_cnt[b],
              v.begin() + dst[b]);
}

// All k-mers (and reverse complements if rc) of the sequences, as colex keys.
static std::vector<u64> extract_kmers(const std::vector<const char *> &seqs,
                                      const std::vector<u64> &lens, int k,
                                      bool rc) {
  u64 total = 0;
  std::vector<u64> base(seqs.size() + 1, 0);
  for (size_t i = 0; i < seqs.size(); ++i) {
    u64 m = lens[i] >= (u64)k ? lens[i] - k + 1 : 0;
    base[i + 1] = base[i] + m * (rc ? 2 : 1);
  }
  total = base.back();
  std::vector<u64> keys(total);
  std::vector<u8> valid(total, 0);
  const u64 top = 2ULL * (k - 1);
  const u64 mask = (k == 32) ? ~0ULL : ((1ULL << (2 * k)) - 1);
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t s = 0; s < seqs.size(); ++s) {
    const char *p = seqs[s];
    u64 n = lens[s];
    if (n < (u64)k) continue;
    u64 fwd = 0, rev = 0;
    int run = 0;  // valid chars in the current window
    u64 o = base[s];
    for (u64 i = 0; i < n; ++i) {
      int c = code_of(p[i]);
      if (c < 0) {
        run = 0;
        fwd = rev = 0;
      } else {
        // colex key: newest char (last) at the top bits
        fwd = (fwd >> 2) | ((u64)c << top);
        // reverse complement: its last char is complement of the first of x
        rev = ((rev << 2) | (u64)(3 - c)) & mask;
        ++run;
      }
      if (i + 1 >= (u64)k) {
        u64 slot = i + 1 - k;
        if (run >= k) {
          keys[o + slot * (rc ? 2 : 1)] = fwd;
          valid[o + slot * (rc ? 2 : 1)] = 1;
          if (rc) {
            keys[o + slot * 2 + 1] = rev;
            valid[o + slot * 2 + 1] = 1;
          }
        }
      }
    }
  }
  u64 w = 0;
  for (u64 i = 0; i < total; ++i)
    if (valid[i]) keys[w++] = keys[i];
  keys.resize(w);
  return keys;
}

struct Node {
  u64 key;
  u32 len;
  bool operator<(const Node &o) const {
    return key < o.key || (key == o.key && len < o.len);
  }
  bool operator==(const Node &o) const { return key == o.key && len == o.len; }
};

struct Built {
  SbwtFile sbwt;
  std::vector<u64> kmers;       // sorted colex keys of the real k-mers
  std::vector<u64> kmer_node;   // node index of each real k-mer
};

// Builds the SBWT of a sorted unique k-mer key set.
static Built build_from_keys(std::vector<u64> &&K, int k) {
  Built out;
  const u64 n = K.size();
  const int top = 2 * (k - 1);
  const u64 mask = (k - 1 == 32) ? ~0ULL : ((1ULL << (2 * (k - 1))) - 1);
  // 1. k-mers with a predecessor: targets of groups K' = key >> 2.
  std::vector<u8> has_pred(n, 0);
  {
    int T = omp_get_max_threads();
#pragma omp parallel num_threads(T)
    {
      int t = omp_get_thread_num();
      u64 lo = n * t / T, hi = n * (t + 1) / T;
      // cursors for each last char c: targets K' | c << top increase with K'
      for (int c = 0; c < 4; ++c) {
        u64 cur = 0;
        bool init = false;
        u64 prevg = ~0ULL;
        for (u64 i = lo; i < hi; ++i) {
          u64 g = K[i] >> 2;
          if (g == prevg) continue;
          prevg = g;
          u64 target = g | ((u64)c << top);
          if (!init) {
            cur = std::lower_bound(K.begin(), K.end(), target) - K.begin();
            init = true;
          }
          while (cur < n && K[cur] < target) ++cur;
          if (cur < n && K[cur] == target) has_pred[cur] = 1;
        }
      }
    }
  }
  // 2. dummies $^(k-i) x[0..i) of the sources.
  std::vector<Node> D;
  D.push_back({0, 0});  // root $^k, always present
  for (u64 i = 0; i < n; ++i) {
    if (has_pred[i]) continue;
    u64 x = K[i];
    for (int len = 1; len < k; ++len) {
      u64 pref = x & ((1ULL << (2 * len)) - 1);  // x[0..len)
      D.push_back({pref << (2 * (k - len)), (u32)len});
    }
  }
  std::sort(D.begin(), D.end());
  D.erase(std::unique(D.begin(), D.end()), D.end());
  // 3. merged node order: k-mers carry len = k.
  const u64 N = n + D.size();
  std::vector<u64> nkey(N);
  std::vector<u8> nlen(N);
  out.kmer_node.resize(n);
  {
    u64 a = 0, b = 0, o = 0;
    while (a < n || b < D.size()) {
      bool take_d = (a == n) || (b < D.size() && (D[b].key < K[a] ||
                                                   (D[b].key == K[a])));
      if (take_d) {
        nkey[o] = D[b].key;
        nlen[o] = (u8)D[b].len;
        ++b;
      } else {
        nkey[o] = K[a];
        nlen[o] = (u8)k;
        out.kmer_node[a] = o;
        ++a;
      }
      ++o;
    }
  }
  // 4. edge bits at suffix-group starts, and the group-start bitvector.
  SbwtFile &s = out.sbwt;
  for (auto &b : s.acgt) b.resize(N);
  s.suffix_group_starts.resize(N);
  auto gkey = [&](u64 i) { return nkey[i] >> 2; };
  auto glen = [&](u64 i) { return std::min<u32>(nlen[i], (u32)k - 1); };
  {
    int T = omp_get_max_threads();
    // word-aligned chunks so that threads never share an output word
    u64 words = (N + 63) / 64;
#pragma omp parallel num_threads(T)
    {
      int t = omp_get_thread_num();
      u64 lo = std::min(N, 64 * (words * t / T));
      u64 hi = std::min(N, 64 * (words * (t + 1) / T));
      u64 cur[4] = {0, 0, 0, 0};
      bool init = false;
      for (u64 i = lo; i < hi; ++i) {
        bool start = (i == 0) || gkey(i) != gkey(i - 1) || glen(i) != glen(i - 1);
        if (!start) continue;
        s.suffix_group_starts.set(i);
        u64 g = gkey(i);
        u32 gl = glen(i);
        if (gl == (u32)k - 1) {
          for (int c = 0; c < 4; ++c) {
            u64 target = g | ((u64)c << top);
            if (!init)
              cur[c] = std::lower_bound(K.begin(), K.end(), target) - K.begin();
            while (cur[c] < n && K[cur[c]] < target) ++cur[c];
            if (cur[c] < n && K[cur[c]] == target) s.acgt[c].set(i);
          }
          init = true;
        } else {
          for (int c = 0; c < 4; ++c) {
            Node target{g | ((u64)c << top), gl + 1};
            if (std::binary_search(D.begin(), D.end(), target)) s.acgt[c].set(i);
          }
        }
      }
    }
  }
  (void)mask;
  s.n_nodes = N;
  s.n_kmers = n;
  s.k = (u64)k;
  s.precalc_k = 0;
  out.kmers = std::move(K);
  return out;
}

// --------------------------------------------------------------------------
// Synthetic data (seeded, reproducible)
// --------------------------------------------------------------------------
static const char kACGT[4] = {'A', 'C', 'G', 'T'};

// i.i.d. uniform ACGT genome
static void random_genome(std::mt19937_64 &rng, char *dst, u64 n) {
  for (u64 i = 0; i < n; i += 32) {
    u64 r = rng();
    for (u64 j = 0; j < 32 && i + j < n; ++j) dst[i + j] = kACGT[(r >> (2 * j)) & 3];
  }
}

// Mutates src into dst: each position substituted with probability sub (to a
// different base), and an indel with probability indel (half insertions of a
// random base, half deletions).  Returns the length written.
static u64 mutate(std::mt19937_64 &rng, const char *src, u64 n, double sub,
                  double indel, char *dst, u64 cap) {
  std::uniform_real_distribution<double> U(0.0, 1.0);
  u64 o = 0;
  for (u64 i = 0; i < n && o < cap; ++i) {
    double u = U(rng);
    if (u < indel / 2) continue;  // deletion
    if (u < indel) {              // insertion before this base
      dst[o++] = kACGT[rng() & 3];
      if (o >= cap) break;
    }
    char c = src[i];
    if (U(rng) < sub) {
      int cc = code_of(c);
      c = kACGT[(cc + 1 + (int)(rng() % 3)) & 3];
    }
    dst[o++] = c;
  }
  return o;
}

}  // namespace tools
}  // namespace sbwt

using namespace sbwt;
using namespace sbwt::tools;

extern "C" {

// Error string of the last failing call on this thread.
static thread_local std::string g_tools_err;
const char *sbwt_tools_last_error(void) { return g_tools_err.c_str(); }

// Builds a plain-matrix SBWT of all k-mers of the n_seqs sequences (k-mers
// with non-ACGT chars skipped; reverse complements added when add_rc) and
// writes it to out_path.  Returns the node count, 0 on error.
u64 sbwt_tools_build_sbwt(const char *const *seqs, const u64 *lens, u64 n_seqs,
                          int k, int add_rc, const char *out_path) {
  try {
    if (k < 1 || k > 31) throw std::runtime_error("builder supports 1 <= k <= 31");
    std::vector<const char *> sv(seqs, seqs + n_seqs);
    std::vector<u64> lv(lens, lens + n_seqs);
    auto keys = extract_kmers(sv, lv, k, add_rc != 0);
    sort_unique(keys);
    Built b = build_from_keys(std::move(keys), k);
    write_sbwt(out_path, b.sbwt);
    return b.sbwt.n_nodes;
  } catch (const std::exception &e) {
    g_tools_err = e.what();
    return 0;
  }
}

// Builds the SBWT of genomes[0..n_genomes) and a Themisto sdsl-hybrid-v4
// color index where the color set of a k-mer is the set of genomes that
// contain it (either strand when add_rc) and every real k-mer node is a key
// k-mer (d = 1).  Color sets are deduplicated; a set is dense iff its size is
// greater than num_colors / 64.  Returns the node count, 0 on error.
u64 sbwt_tools_build_colored(const char *const *genomes, const u64 *lens,
                             u64 n_genomes, int k, int add_rc,
                             const char *sbwt_path, const char *tcolors_path) {
  try {
    if (k < 1 || k > 31) throw std::runtime_error("builder supports 1 <= k <= 31");
    double tt = wall();
    // (k-mer, genome) pairs of every genome (both strands), sorted by k-mer
    // then genome: the runs give the k-mer set and each k-mer's color list.
    struct KG {
      u64 key;
      u64 g;
      bool operator<(const KG &o) const { return key < o.key || (key == o.key && g < o.g); }
    };
    std::vector<u64> gbase(n_genomes + 1, 0);
    for (u64 g = 0; g < n_genomes; ++g) {
      const u64 m = lens[g] >= (u64)k ? lens[g] - k + 1 : 0;
      gbase[g + 1] = gbase[g] + m * (add_rc ? 2 : 1);
    }
    std::vector<KG> pairs(gbase[n_genomes]);
    std::vector<u8> pvalid(gbase[n_genomes], 0);
    {
      const u64 top = 2ULL * (k - 1);
      const u64 kmask = (1ULL << (2 * k)) - 1;
#pragma omp parallel for schedule(dynamic, 1)
      for (u64 g = 0; g < n_genomes; ++g) {
        const char *p = genomes[g];
        u64 fwd = 0, rev = 0, o = gbase[g];
        int run = 0;
        for (u64 i = 0; i < lens[g]; ++i) {
          const int c = code_of(p[i]);
          if (c < 0) {
            run = 0;
            fwd = rev = 0;
          } else {
            fwd = (fwd >> 2) | ((u64)c << top);
            rev = ((rev << 2) | (u64)(3 - c)) & kmask;
            ++run;
          }
          if (i + 1 >= (u64)k && run >= k) {
            const u64 slot = (i + 1 - k) * (add_rc ? 2 : 1);
            pairs[o + slot] = KG{fwd, g};
            pvalid[o + slot] = 1;
            if (add_rc) {
              pairs[o + slot + 1] = KG{rev, g};
              pvalid[o + slot + 1] = 1;
            }
          }
        }
      }
    }
    phase("extract pairs", tt);
    {  // bucket by the top 12 key bits, sort each bucket
      const int B = 4096, shift = 2 * k - 12 > 0 ? 2 * k - 12 : 0;
      const u64 np = pairs.size();
      std::vector<u64> bstart(B + 2, 0);
      for (u64 i = 0; i < np; ++i)
        if (pvalid[i]) bstart[std::min<u64>(pairs[i].key >> shift, B - 1) + 1]++;
      for (int x = 0; x < B; ++x) bstart[x + 1] += bstart[x];
      std::vector<KG> out(bstart[B]);
      std::vector<u64> cur(bstart.begin(), bstart.begin() + B);
      for (u64 i = 0; i < np; ++i)
        if (pvalid[i]) out[cur[std::min<u64>(pairs[i].key >> shift, B - 1)]++] = pairs[i];
      pairs.swap(out);
      std::vector<u8>().swap(pvalid);
#pragma omp parallel for schedule(dynamic, 8)
      for (int x = 0; x < B; ++x) std::sort(pairs.begin() + bstart[x], pairs.begin() + bstart[x + 1]);
    }
    phase("sort pairs", tt);
    // unique k-mers + CSR of unique (k-mer, genome) colors
    std::vector<u64> keys;
    std::vector<u64> cnt;
    std::vector<u32> colors;
    keys.reserve(pairs.size() / 2);
    cnt.reserve(pairs.size() / 2 + 1);
    colors.reserve(pairs.size() / 2);
    cnt.push_back(0);
    for (u64 i = 0; i < pairs.size(); ++i) {
      if (i == 0 || pairs[i].key != pairs[i - 1].key) {
        if (i) cnt.push_back(colors.size());
        keys.push_back(pairs[i].key);
        colors.push_back((u32)pairs[i].g);
      } else if (pairs[i].g != pairs[i - 1].g) {
        colors.push_back((u32)pairs[i].g);
      }
    }
    cnt.push_back(colors.size());
    std::vector<KG>().swap(pairs);
    phase("k-mer set + colors", tt);
    Built b = build_from_keys(std::move(keys), k);
    phase("build_from_keys", tt);
    write_sbwt(sbwt_path, b.sbwt);
    phase("write_sbwt", tt);
    const u64 n = b.kmers.size();
    // dedupe color sets: singletons by color, the rest by hash
    std::vector<u64> set_of_kmer(n);
    std::vector<u64> set_first;  // k-mer rank whose list defines the set
    {
      std::vector<u64> single_first(n_genomes, ~0ULL);
      for (u64 r = 0; r < n; ++r)
        if (cnt[r + 1] - cnt[r] == 1 && single_first[colors[cnt[r]]] == ~0ULL)
          single_first[colors[cnt[r]]] = r;
      std::vector<u64> single_id(n_genomes, ~0ULL);
      for (u64 g = 0; g < n_genomes; ++g)
        if (single_first[g] != ~0ULL) {
          single_id[g] = set_first.size();
          set_first.push_back(single_first[g]);
        }
      auto hash_of = [&](u64 r) {
        u64 h = 1469598103934665603ULL ^ (cnt[r + 1] - cnt[r]);
        for (u64 t = cnt[r]; t < cnt[r + 1]; ++t) h = (h ^ colors[t]) * 1099511628211ULL;
        h ^= h >> 29;
        return h * 0xBF58476D1CE4E5B9ULL;
      };
      auto same = [&](u64 a, u64 bb) {
        u64 la = cnt[a + 1] - cnt[a], lb = cnt[bb + 1] - cnt[bb];
        return la == lb && std::equal(colors.begin() + cnt[a], colors.begin() + cnt[a + 1],
                                      colors.begin() + cnt[bb]);
      };
      std::vector<std::pair<u64, u64>> multi;  // (hash, rank)
      for (u64 r = 0; r < n; ++r) {
        if (cnt[r + 1] - cnt[r] == 1)
          set_of_kmer[r] = single_id[colors[cnt[r]]];
        else
          multi.push_back({0, r});
      }
#pragma omp parallel for schedule(static)
      for (u64 i = 0; i < multi.size(); ++i) multi[i].first = hash_of(multi[i].second);
      std::sort(multi.begin(), multi.end());
      for (u64 i = 0; i < multi.size();) {
        u64 j = i;
        while (j < multi.size() && multi[j].first == multi[i].first) ++j;
        std::vector<u64> local;
        for (u64 q = i; q < j; ++q) {
          const u64 r = multi[q].second;
          u64 id = ~0ULL;
          for (u64 f : local)
            if (same(set_first[f], r)) {
              id = f;
              break;
            }
          if (id == ~0ULL) {
            id = set_first.size();
            set_first.push_back(r);
            local.push_back(id);
          }
          set_of_kmer[r] = id;
        }
        i = j;
      }
    }
    phase("csr + dedupe", tt);
    const u64 C = n_genomes;
    const u64 S = set_first.size();
    // dense iff |set| > C/64 (the rule Themisto's hybrid storage uses)
    std::vector<u8> dense(S);
    for (u64 s = 0; s < S; ++s) {
      u64 r = set_first[s];
      dense[s] = (double)(cnt[r + 1] - cnt[r]) > (double)C / 64.0;
    }
    // color set ids: renumber so ids follow first appearance (any order is
    // valid for the format); dense/sparse payloads in id order.
    double t0 = tt;
    TColorsFile t;
    t.is_dense_marks.resize(S);
    std::vector<u64> dense_iv{0}, sparse_iv{0}, sparse_vals;
    u64 dense_bits = 0;
    for (u64 s = 0; s < S; ++s) {
      u64 r = set_first[s];
      if (dense[s]) {
        t.is_dense_marks.set(s);
        u64 maxc = colors[cnt[r + 1] - 1];
        dense_bits += maxc + 1;
        dense_iv.push_back(dense_bits);
      } else {
        for (u64 q = cnt[r]; q < cnt[r + 1]; ++q) sparse_vals.push_back(colors[q]);
        sparse_iv.push_back(sparse_vals.size());
      }
    }
    t.dense_arrays.resize(dense_bits);
    {
      u64 pos = 0;
      for (u64 s = 0; s < S; ++s) {
        if (!dense[s]) continue;
        u64 r = set_first[s];
        u64 maxc = colors[cnt[r + 1] - 1];
        for (u64 q = cnt[r]; q < cnt[r + 1]; ++q) t.dense_arrays.set(pos + colors[q]);
        pos += maxc + 1;
      }
    }
    auto width_for = [](u64 maxv) {
      u8 w = 1;
      while (w < 64 && (maxv >> w)) ++w;
      return w;
    };
    t.dense_arrays_intervals.assign(dense_iv, width_for(dense_iv.back()));
    t.sparse_arrays.assign(sparse_vals, width_for(C ? C - 1 : 0));
    t.sparse_arrays_intervals.assign(sparse_iv, width_for(sparse_iv.back()));
    // key k-mer marks: every real k-mer node; color_set_idxs in node order
    t.key_kmer_marks.resize(b.sbwt.n_nodes);
    std::vector<u64> csi(n);
    for (u64 r = 0; r < n; ++r) {
      t.key_kmer_marks.set(b.kmer_node[r]);
      csi[r] = set_of_kmer[r];  // node order == k-mer rank order among k-mers
    }
    t.color_set_idxs.assign(csi, width_for(S ? S - 1 : 0));
    t.max_color_set_idx = S ? S - 1 : 0;
    t.largest_color = C ? C - 1 : 0;
    t.sum_color_set_sizes = 0;
    for (u64 s = 0; s < S; ++s)
      t.sum_color_set_sizes += cnt[set_first[s] + 1] - cnt[set_first[s]];
    phase("payloads", t0);
    write_tcolors(tcolors_path, t);
    phase("write_tcolors", t0);
    return b.sbwt.n_nodes;
  } catch (const std::exception &e) {
    g_tools_err = e.what();
    return 0;
  }
}

// Seeded random genome(s): n_founders i.i.d. founders of length len; genome g
// derives from founder g % n_founders by per-base substitution rate
// sub_lo + (sub_hi - sub_lo) * u_g (u_g uniform per genome) and indel rate
// indel.  With n_founders == 0 the genomes are themselves i.i.d.  Writes all
// genomes back to back into dst (capacity cap) and their lengths into
// lens_out; returns the total length.
u64 sbwt_tools_gen_genomes(u64 seed, u64 n_genomes, u64 len, u64 n_founders,
                           double sub_lo, double sub_hi, double indel, char *dst,
                           u64 cap, u64 *lens_out) {
  std::mt19937_64 rng(seed);
  std::vector<std::string> founders(n_founders);
  for (auto &f : founders) {
    f.resize(len);
    random_genome(rng, f.data(), len);
  }
  std::vector<u64> seeds(n_genomes);
  std::vector<double> subs(n_genomes);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  for (u64 g = 0; g < n_genomes; ++g) {
    seeds[g] = rng();
    subs[g] = sub_lo + (sub_hi - sub_lo) * U(rng);
  }
  u64 per_cap = len + len / 8 + 64;
  std::vector<u64> glen(n_genomes);
  std::vector<std::string> tmp(n_genomes);
#pragma omp parallel for schedule(dynamic, 1)
  for (u64 g = 0; g < n_genomes; ++g) {
    std::mt19937_64 r(seeds[g]);
    tmp[g].resize(per_cap);
    if (n_founders == 0) {
      random_genome(r, tmp[g].data(), len);
      glen[g] = len;
    } else {
      const std::string &f = founders[g % n_founders];
      glen[g] = mutate(r, f.data(), len, subs[g], indel, tmp[g].data(), per_cap);
    }
  }
  u64 o = 0;
  for (u64 g = 0; g < n_genomes; ++g) {
    u64 m = std::min(glen[g], cap - o);
    memcpy(dst + o, tmp[g].data(), m);
    lens_out[g] = m;
    o += m;
  }
  return o;
}

// Seeded reads.  For each read: with probability frac_from_genome it is a
// substring of a random genome (random strand) of the drawn length, else
// i.i.d. ACGT; then each base is substituted with probability sub and set to
// 'N' with probability n_rate.  Lengths: if len_sigma == 0 all reads have
// length len_median, else log-normal(ln(len_median), len_sigma) clipped to
// [len_min, len_max].  genome_choice_weights selects which genome (NULL =
// uniform over genomes).  Writes chars back to back into dst and cumulative
// read ends into read_ends; returns total chars, 0 on overflow.
u64 sbwt_tools_gen_reads(u64 seed, const char *genomes, const u64 *glens,
                         u64 n_genomes, u64 n_reads, double frac_from_genome,
                         u64 len_median, double len_sigma, u64 len_min,
                         u64 len_max, double sub, double n_rate, char *dst,
                         u64 cap, u64 *read_ends) {
  std::mt19937_64 rng(seed);
  std::vector<u64> gstart(n_genomes + 1, 0);
  for (u64 g = 0; g < n_genomes; ++g) gstart[g + 1] = gstart[g] + glens[g];
  // per-read lengths first (sequential, deterministic)
  std::vector<u64> lens(n_reads);
  std::lognormal_distribution<double> LN(std::log((double)len_median),
                                         len_sigma > 0 ? len_sigma : 1.0);
  for (u64 r = 0; r < n_reads; ++r) {
    if (len_sigma <= 0) {
      lens[r] = len_median;
    } else {
      double x = LN(rng);
      u64 L = (u64)std::llround(x);
      lens[r] = std::min(std::max(L, len_min), len_max);
    }
  }
  std::vector<u64> ends(n_reads);
  u64 acc = 0;
  for (u64 r = 0; r < n_reads; ++r) {
    acc += lens[r];
    ends[r] = acc;
  }
  if (acc > cap) return 0;
  std::vector<u64> seeds(n_reads);
  for (u64 r = 0; r < n_reads; ++r) seeds[r] = rng();
#pragma omp parallel for schedule(dynamic, 4096)
  for (u64 r = 0; r < n_reads; ++r) {
    std::mt19937_64 g(seeds[r]);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    u64 L = lens[r];
    char *p = dst + (r ? ends[r - 1] : 0);
    bool from = n_genomes > 0 && U(g) < frac_from_genome;
    if (from) {
      u64 gi = g() % n_genomes;
      u64 gl = glens[gi];
      if (gl >= L) {
        u64 st = gl == L ? 0 : g() % (gl - L + 1);
        const char *src = genomes + gstart[gi] + st;
        bool rev = g() & 1;
        for (u64 i = 0; i < L; ++i) {
          if (!rev) {
            p[i] = src[i];
          } else {
            int c = code_of(src[L - 1 - i]);
            p[i] = c < 0 ? 'N' : kACGT[3 - c];
          }
        }
      } else {
        from = false;
      }
    }
    if (!from) random_genome(g, p, L);
    for (u64 i = 0; i < L; ++i) {
      double u = U(g);
      if (u < n_rate) {
        p[i] = 'N';
      } else if (u < n_rate + sub) {
        int c = code_of(p[i]);
        if (c >= 0) p[i] = kACGT[(c + 1 + (int)(g() % 3)) & 3];
      }
    }
  }
  memcpy(read_ends, ends.data(), n_reads * 8);
  return acc;
}

}  // extern "C"
