// SBWT construction on the GPU: the same index as the project's host builder
// (csrc/tools/sbwt_build.cpp; SBWT-Search itself loads indexes that Themisto
// builds), written with the same .sbwt writer.
//
// SBWT (Alanko et al., "Small searchable k-spectra via subset rank queries on
// the spectral Burrows-Wheeler transform"): the nodes are the k-mers plus, for
// every k-mer x without a predecessor, the dummy nodes $^(k-i) x[0..i)
// (i = 0..k-1, $ sorts first); they are in colexicographic order; node u has
// an edge labelled c to the node u[1..k) c, and the edge bit is kept only at
// the first node of u's suffix group (the nodes sharing u[1..k)).
//
// A node is (key, len): key = sum of code(char t) << 2t over its k chars ($
// and A both 0), len = its non-$ chars; (key, len) ascending is colex order.
// Steps (k <= 31, so keys fit in 62 bits and ~0 marks "no k-mer"):
//   1. one thread per position: the forward and reverse-complement keys of
//      the k-mer starting there (~0 when it holds a non-ACGT char or crosses
//      a sequence end);
//   2. radix sort + unique of the keys;
//   3. per k-mer: mark its successors x[1..k) c that are k-mers (binary
//      search); unmarked k-mers are sources;
//   4. per source, its k - 1 dummy prefixes; radix sort by len then (stable)
//      by key, unique;
//   5. merged node order: each k-mer / dummy finds its rank in the other list
//      by binary search (dummies precede k-mers of the same key);
//   6. one thread per 64 nodes: suffix-group starts and, at each start, the
//      four edge bits (binary search of the target k-mer or dummy).
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <string>
#include <vector>

#include "common.hpp"
#include "formats.hpp"

namespace sbwt {

namespace {

constexpr uint64_t kNoKey = ~0ULL;

__device__ __forceinline__ int dev_code(uint8_t c) {
  switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return -1;
  }
}

// keys[2i] / keys[2i + 1]: the k-mer at position i and its reverse
// complement (or kNoKey); without rc, keys[i].
__global__ void kmer_keys_kernel(const uint8_t *chars, uint64_t n_chars, const uint64_t *ends,
                                 uint64_t n_seqs, uint32_t k, int rc, uint64_t *keys) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_chars; i += step) {
    uint64_t fwd = kNoKey, rev = kNoKey;
    if (i + k <= n_chars) {
      // the sequence holding position i: first end > i
      uint64_t lo = 0, hi = n_seqs;
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (ends[mid] > i) hi = mid; else lo = mid + 1;
      }
      if (lo < n_seqs && i + k <= ends[lo]) {
        uint64_t f = 0, r = 0;
        bool ok = true;
        for (uint32_t t = 0; t < k; ++t) {
          const int c = dev_code(chars[i + t]);
          if (c < 0) {
            ok = false;
            break;
          }
          f |= (uint64_t)c << (2 * t);
          r |= (uint64_t)(3 - c) << (2 * (k - 1 - t));
        }
        if (ok) {
          fwd = f;
          rev = r;
        }
      }
    }
    if (rc) {
      keys[2 * i] = fwd;
      keys[2 * i + 1] = rev;
    } else {
      keys[i] = fwd;
    }
  }
}

__device__ __forceinline__ uint64_t lower_bound_u64(const uint64_t *a, uint64_t n, uint64_t x) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint64_t upper_bound_u64(const uint64_t *a, uint64_t n, uint64_t x) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// has_pred[j] = 1 for every k-mer j that follows some k-mer (idempotent
// stores); K sorted, unique.
__global__ void successors_kernel(const uint64_t *K, uint64_t n, uint32_t k, uint8_t *has_pred) {
  const uint32_t top = 2 * (k - 1);
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += step) {
    const uint64_t g = K[i] >> 2;
    for (uint32_t c = 0; c < 4; ++c) {
      const uint64_t t = g | ((uint64_t)c << top);
      const uint64_t j = lower_bound_u64(K, n, t);
      if (j < n && K[j] == t) has_pred[j] = 1;
    }
  }
}

__global__ void sources_kernel(const uint8_t *has_pred, uint64_t n, uint64_t *is_src) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += step)
    is_src[i] = has_pred[i] ? 0 : 1;
}

// Dummies of source i at src_off[i] * (k - 1): (x[0..len) << 2 (k - len), len)
// for len = 1..k-1; the root ($^k, 0) goes last.
__global__ void dummies_kernel(const uint64_t *K, uint64_t n, uint32_t k, const uint8_t *has_pred,
                               const uint64_t *src_off, uint64_t *dkey, uint32_t *dlen,
                               uint64_t n_dummies) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += step) {
    if (has_pred[i]) continue;
    const uint64_t x = K[i], o = src_off[i] * (k - 1);
    for (uint32_t len = 1; len < k; ++len) {
      dkey[o + len - 1] = (x & ((1ULL << (2 * len)) - 1)) << (2 * (k - len));
      dlen[o + len - 1] = len;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    dkey[n_dummies - 1] = 0;
    dlen[n_dummies - 1] = 0;
  }
}

// flag[j] = 1 where (key, len) differs from the previous pair (sorted).
__global__ void pair_unique_flags_kernel(const uint64_t *key, const uint32_t *len, uint64_t n,
                                         uint64_t *flag) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += step)
    flag[j] = (j == 0 || key[j] != key[j - 1] || len[j] != len[j - 1]) ? 1 : 0;
}

__global__ void pair_compact_kernel(const uint64_t *key, const uint32_t *len, uint64_t n,
                                    const uint64_t *flag, const uint64_t *off, uint64_t *okey,
                                    uint32_t *olen) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += step)
    if (flag[j]) {
      okey[off[j]] = key[j];
      olen[off[j]] = len[j];
    }
}

// Merged order: node position of every k-mer and every dummy.
__global__ void merge_kernel(const uint64_t *K, uint64_t n, const uint64_t *dkey,
                             const uint32_t *dlen, uint64_t nd, uint32_t k, uint64_t *nkey,
                             uint8_t *nlen, uint64_t *kmer_node) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n + nd; i += step) {
    if (i < n) {  // k-mer: after every dummy of key <= its key
      const uint64_t p = i + upper_bound_u64(dkey, nd, K[i]);
      nkey[p] = K[i];
      nlen[p] = (uint8_t)k;
      if (kmer_node) kmer_node[i] = p;
    } else {  // dummy: after every k-mer of a smaller key
      const uint64_t b = i - n;
      const uint64_t p = b + lower_bound_u64(K, n, dkey[b]);
      nkey[p] = dkey[b];
      nlen[p] = (uint8_t)dlen[b];
    }
  }
}

// One thread per 64 nodes: suffix-group starts and the edge bits there.
__global__ void edges_kernel(const uint64_t *nkey, const uint8_t *nlen, uint64_t N,
                             const uint64_t *K, uint64_t n, const uint64_t *dkey,
                             const uint32_t *dlen, uint64_t nd, uint32_t k, uint64_t *acgt0,
                             uint64_t words, uint64_t *sg) {
  const uint32_t top = 2 * (k - 1);
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < words; w += step) {
    uint64_t bits[4] = {0, 0, 0, 0}, s = 0;
    const uint64_t i0 = 64 * w, i1 = min(N, i0 + 64);
    for (uint64_t i = i0; i < i1; ++i) {
      const uint64_t g = nkey[i] >> 2;
      const uint32_t gl = min((uint32_t)nlen[i], k - 1);
      if (i > 0 && (nkey[i - 1] >> 2) == g && min((uint32_t)nlen[i - 1], k - 1) == gl) continue;
      s |= 1ULL << (i - i0);
      for (uint32_t c = 0; c < 4; ++c) {
        const uint64_t t = g | ((uint64_t)c << top);
        bool has = false;
        if (gl == k - 1) {
          const uint64_t j = lower_bound_u64(K, n, t);
          has = j < n && K[j] == t;
        } else {  // target dummy (t, gl + 1)
          for (uint64_t j = lower_bound_u64(dkey, nd, t); j < nd && dkey[j] == t; ++j)
            if (dlen[j] == gl + 1) {
              has = true;
              break;
            }
        }
        if (has) bits[c] |= 1ULL << (i - i0);
      }
    }
    for (uint32_t c = 0; c < 4; ++c) acgt0[c * words + w] = bits[c];
    sg[w] = s;
  }
}

unsigned grid_for(uint64_t n) {
  return (unsigned)std::max<uint64_t>(std::min<uint64_t>((n + 255) / 256, 148 * 64), 1);
}

// cub temporary storage held across calls
struct CubTemp {
  DeviceBuffer buf;
  void *get(size_t bytes) {
    buf.ensure(std::max<size_t>(bytes, 1));
    return buf.get();
  }
};

}  // namespace

SbwtFile build_from_sorted_keys(const u64 *K, u64 n, uint32_t k, u64 *kmer_node);

// Builds the SBWT of the sequences (chars back to back, ends cumulative) on
// `device`; returns it in host form.
SbwtFile build_sbwt_device(const char *chars, u64 n_chars, const u64 *seq_ends, u64 n_seqs,
                           uint32_t k, bool rc, int device) {
  if (k < 2 || k > 31) throw Error(SBWT_E_INVALID, "the GPU builder supports 2 <= k <= 31");
  for (u64 s = 1; s < n_seqs; ++s)
    if (seq_ends[s] < seq_ends[s - 1]) throw Error(SBWT_E_INVALID, "sequence ends must not decrease");
  if (n_seqs && seq_ends[n_seqs - 1] > n_chars) throw Error(SBWT_E_INVALID, "sequence end past the chars");
  DeviceGuard g(device);
  cudaStream_t st = nullptr;
  CubTemp tmp;
  size_t tb = 0;
  // 1. keys
  const u64 n_keys = (rc ? 2 : 1) * n_chars;
  DeviceBuffer d_chars(std::max<u64>(n_chars, 1)), d_ends(std::max<u64>(n_seqs, 1) * 8);
  DeviceBuffer keys(std::max<u64>(n_keys, 1) * 8), keys2(std::max<u64>(n_keys, 1) * 8);
  if (n_chars) SBWT_CUDA(cudaMemcpy(d_chars.get(), chars, n_chars, cudaMemcpyHostToDevice));
  if (n_seqs) SBWT_CUDA(cudaMemcpy(d_ends.get(), seq_ends, n_seqs * 8, cudaMemcpyHostToDevice));
  if (n_chars)
    kmer_keys_kernel<<<grid_for(n_chars), 256, 0, st>>>(d_chars.get<uint8_t>(), n_chars,
                                                        d_ends.get<u64>(), n_seqs, k, rc ? 1 : 0,
                                                        keys.get<u64>());
  SBWT_CUDA(cudaGetLastError());
  d_chars.release();
  // 2. sort + unique (kNoKey sorts last)
  u64 n = 0;
  DeviceBuffer d_count(8);
  if (n_keys) {
    SBWT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys.get<u64>(), keys2.get<u64>(),
                                             (int64_t)n_keys, 0, 64, st));
    SBWT_CUDA(cub::DeviceRadixSort::SortKeys(tmp.get(tb), tb, keys.get<u64>(), keys2.get<u64>(),
                                             (int64_t)n_keys, 0, 64, st));
    SBWT_CUDA(cub::DeviceSelect::Unique(nullptr, tb, keys2.get<u64>(), keys.get<u64>(),
                                        d_count.get<u64>(), (int64_t)n_keys, st));
    SBWT_CUDA(cub::DeviceSelect::Unique(tmp.get(tb), tb, keys2.get<u64>(), keys.get<u64>(),
                                        d_count.get<u64>(), (int64_t)n_keys, st));
    SBWT_CUDA(cudaMemcpy(&n, d_count.get(), 8, cudaMemcpyDeviceToHost));
    if (n) {
      u64 last = 0;
      SBWT_CUDA(cudaMemcpy(&last, keys.get<u64>() + n - 1, 8, cudaMemcpyDeviceToHost));
      if (last == kNoKey) --n;
    }
  }
  keys2.release();
  return build_from_sorted_keys(keys.get<u64>(), n, k, nullptr);
}

// Steps 3-6 from the sorted unique k-mer keys K[0..n) (device); kmer_node
// (device, optional) receives the node of every k-mer.
SbwtFile build_from_sorted_keys(const u64 *K, u64 n, uint32_t k, u64 *kmer_node) {
  cudaStream_t st = nullptr;
  CubTemp tmp;
  size_t tb = 0;
  // 3. sources
  DeviceBuffer has_pred(std::max<u64>(n, 1)), src_off(std::max<u64>(n, 1) * 8 + 8);
  SBWT_CUDA(cudaMemset(has_pred.get(), 0, std::max<u64>(n, 1)));
  u64 n_src = 0;
  if (n) {
    successors_kernel<<<grid_for(n), 256, 0, st>>>(K, n, k, has_pred.get<uint8_t>());
    sources_kernel<<<grid_for(n), 256, 0, st>>>(has_pred.get<uint8_t>(), n, src_off.get<u64>());
    SBWT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, src_off.get<u64>(), src_off.get<u64>(),
                                            (int64_t)n, st));
    // last entry is_src before the scan overwrites it
    u64 last_src = 0;
    SBWT_CUDA(cudaMemcpy(&last_src, src_off.get<u64>() + n - 1, 8, cudaMemcpyDeviceToHost));
    SBWT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, src_off.get<u64>(),
                                            src_off.get<u64>(), (int64_t)n, st));
    u64 before_last = 0;
    SBWT_CUDA(cudaMemcpy(&before_last, src_off.get<u64>() + n - 1, 8, cudaMemcpyDeviceToHost));
    n_src = before_last + last_src;
  }
  // 4. dummies
  const u64 nd_all = n_src * (k - 1) + 1;
  DeviceBuffer dkey(nd_all * 8), dlen(nd_all * 4), dkey2(nd_all * 8), dlen2(nd_all * 4);
  dummies_kernel<<<grid_for(std::max<u64>(n, 1)), 256, 0, st>>>(
      K, n, k, has_pred.get<uint8_t>(), src_off.get<u64>(), dkey.get<u64>(), dlen.get<uint32_t>(),
      nd_all);
  SBWT_CUDA(cudaGetLastError());
  // by len, then stably by key
  SBWT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, dlen.get<uint32_t>(), dlen2.get<uint32_t>(),
                                            dkey.get<u64>(), dkey2.get<u64>(), (int64_t)nd_all, 0, 8,
                                            st));
  SBWT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, dlen.get<uint32_t>(),
                                            dlen2.get<uint32_t>(), dkey.get<u64>(), dkey2.get<u64>(),
                                            (int64_t)nd_all, 0, 8, st));
  SBWT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, dkey2.get<u64>(), dkey.get<u64>(),
                                            dlen2.get<uint32_t>(), dlen.get<uint32_t>(),
                                            (int64_t)nd_all, 0, 2 * k, st));
  SBWT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, dkey2.get<u64>(), dkey.get<u64>(),
                                            dlen2.get<uint32_t>(), dlen.get<uint32_t>(),
                                            (int64_t)nd_all, 0, 2 * k, st));
  // unique pairs
  DeviceBuffer flag(nd_all * 8 + 8), off(nd_all * 8 + 8);
  pair_unique_flags_kernel<<<grid_for(nd_all), 256, 0, st>>>(dkey.get<u64>(), dlen.get<uint32_t>(),
                                                             nd_all, flag.get<u64>());
  SBWT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.get<u64>(), off.get<u64>(),
                                          (int64_t)nd_all, st));
  SBWT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, flag.get<u64>(), off.get<u64>(),
                                          (int64_t)nd_all, st));
  u64 lf = 0, lo = 0;
  SBWT_CUDA(cudaMemcpy(&lf, flag.get<u64>() + nd_all - 1, 8, cudaMemcpyDeviceToHost));
  SBWT_CUDA(cudaMemcpy(&lo, off.get<u64>() + nd_all - 1, 8, cudaMemcpyDeviceToHost));
  const u64 nd = lo + lf;
  pair_compact_kernel<<<grid_for(nd_all), 256, 0, st>>>(dkey.get<u64>(), dlen.get<uint32_t>(),
                                                        nd_all, flag.get<u64>(), off.get<u64>(),
                                                        dkey2.get<u64>(), dlen2.get<uint32_t>());
  SBWT_CUDA(cudaGetLastError());
  dkey.release();
  dlen.release();
  flag.release();
  off.release();
  const u64 *D = dkey2.get<u64>();
  const uint32_t *DL = dlen2.get<uint32_t>();
  // 5. merged order
  const u64 N = n + nd;
  DeviceBuffer nkey(N * 8), nlen(N);
  merge_kernel<<<grid_for(N), 256, 0, st>>>(K, n, D, DL, nd, k, nkey.get<u64>(),
                                            nlen.get<uint8_t>(), kmer_node);
  // 6. edge bits and suffix-group starts
  const u64 words = (N + 63) / 64;
  DeviceBuffer bits(words * 5 * 8);
  edges_kernel<<<grid_for(words), 256, 0, st>>>(nkey.get<u64>(), nlen.get<uint8_t>(), N, K, n, D,
                                                DL, nd, k, bits.get<u64>(), words,
                                                bits.get<u64>() + 4 * words);
  SBWT_CUDA(cudaGetLastError());
  std::vector<u64> h(words * 5);
  SBWT_CUDA(cudaMemcpy(h.data(), bits.get(), words * 5 * 8, cudaMemcpyDeviceToHost));
  SbwtFile s;
  for (int c = 0; c < 4; ++c) {
    s.acgt[c].num_bits = N;
    s.acgt[c].words.assign(h.begin() + c * words, h.begin() + (c + 1) * words);
  }
  s.suffix_group_starts.num_bits = N;
  s.suffix_group_starts.words.assign(h.begin() + 4 * words, h.end());
  s.n_nodes = N;
  s.n_kmers = n;
  s.k = k;
  s.precalc_k = 0;
  return s;
}

}  // namespace sbwt

using namespace sbwt;

// Builds a plain-matrix SBWT of every k-mer of the sequences on the GPU and
// writes it to out_path (see the header).
extern "C" int sbwt_build_index(const char *chars, uint64_t n_chars, const uint64_t *seq_ends,
                                uint64_t n_seqs, uint32_t k, int add_rc, const char *out_path,
                                int device, uint64_t *n_nodes) {
  if ((n_chars && !chars) || (n_seqs && !seq_ends) || !out_path) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    const SbwtFile s = build_sbwt_device(chars, n_chars, seq_ends, n_seqs, k, add_rc != 0, device);
    write_sbwt(out_path, s);
    if (n_nodes) *n_nodes = s.n_nodes;
  });
}

// ---------------------------------------------------------------------------
// Colored index (.tcolors, Themisto's sdsl-hybrid-v4 layout): the color set of
// a k-mer is the set of genomes that contain it (either strand when rc), every
// k-mer is a key k-mer (d = 1), color sets are deduplicated and numbered as
// the project's host builder numbers them (singleton sets first, by genome;
// then the other sets in (hash of the color list, first k-mer) order), a set
// is dense iff its size > num_colors / 64.
// ---------------------------------------------------------------------------
namespace sbwt {

namespace {

// keys as kmer_keys_kernel, plus the genome of each key slot
__global__ void kmer_pairs_kernel(const uint8_t *chars, uint64_t n_chars, const uint64_t *ends,
                                  uint64_t n_seqs, uint32_t k, int rc, uint64_t *keys,
                                  uint32_t *gen) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_chars; i += step) {
    uint64_t fwd = kNoKey, rev = kNoKey, lo = 0, hi = n_seqs;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (ends[mid] > i) hi = mid; else lo = mid + 1;
    }
    if (i + k <= n_chars && lo < n_seqs && i + k <= ends[lo]) {
      uint64_t f = 0, r = 0;
      bool ok = true;
      for (uint32_t t = 0; t < k && ok; ++t) {
        const int c = dev_code(chars[i + t]);
        ok = c >= 0;
        f |= (uint64_t)(c & 3) << (2 * t);
        r |= (uint64_t)(3 - (c & 3)) << (2 * (k - 1 - t));
      }
      if (ok) {
        fwd = f;
        rev = r;
      }
    }
    const uint32_t g = (uint32_t)min(lo, n_seqs ? n_seqs - 1 : 0);
    if (rc) {
      keys[2 * i] = fwd;
      keys[2 * i + 1] = rev;
      gen[2 * i] = gen[2 * i + 1] = g;
    } else {
      keys[i] = fwd;
      gen[i] = g;
    }
  }
}

// 1 where (key, genome) starts a new distinct valid pair (sorted input)
__global__ void pair_new_kernel(const uint64_t *key, const uint32_t *gen, uint64_t n,
                                uint64_t *flag) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += step)
    flag[i] = key[i] != kNoKey && (i == 0 || key[i] != key[i - 1] || gen[i] != gen[i - 1]);
}

template <class T>
__global__ void compact_kernel(const T *in, const uint64_t *flag, const uint64_t *off, uint64_t n,
                               T *out) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += step)
    if (flag[i]) out[off[i]] = in[i];
}

// 1 where the (distinct) pair starts a new k-mer
__global__ void kmer_new_kernel(const uint64_t *pk, uint64_t n, uint64_t *flag) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += step)
    flag[i] = i == 0 || pk[i] != pk[i - 1];
}

// k-mer r: K[r] and the first pair cnt[r]
__global__ void kmer_csr_kernel(const uint64_t *pk, const uint64_t *flag, const uint64_t *off,
                                uint64_t n, uint64_t *K, uint64_t *cnt) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += step)
    if (flag[i]) {
      K[off[i]] = pk[i];
      cnt[off[i]] = i;
    }
}

// singleton sets: the first k-mer holding exactly {g}; multi-color k-mers
// flagged for the hash pass
__global__ void classify_kernel(const uint64_t *cnt, const uint32_t *colors, uint64_t n,
                                unsigned long long *single_first, uint64_t *is_multi) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += step) {
    const uint64_t size = cnt[r + 1] - cnt[r];
    is_multi[r] = size > 1;
    if (size == 1) atomicMin(single_first + colors[cnt[r]], (unsigned long long)r);
  }
}

__global__ void has_single_kernel(const unsigned long long *single_first, uint64_t C,
                                  uint64_t *has) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < C; g += step)
    has[g] = single_first[g] != ~0ULL;
}

// hash of a color list (the host builder's: FNV-1a over the ids, seeded with
// the length, then a xorshift-multiply finish)
__device__ __forceinline__ uint64_t list_hash(const uint32_t *colors, uint64_t a, uint64_t b) {
  uint64_t h = 1469598103934665603ULL ^ (b - a);
  for (uint64_t t = a; t < b; ++t) h = (h ^ colors[t]) * 1099511628211ULL;
  h ^= h >> 29;
  return h * 0xBF58476D1CE4E5B9ULL;
}

__global__ void multi_hash_kernel(const uint64_t *cnt, const uint32_t *colors,
                                  const uint64_t *is_multi, const uint64_t *off, uint64_t n,
                                  uint64_t *mh, uint64_t *mr) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += step)
    if (is_multi[r]) {
      mh[off[r]] = list_hash(colors, cnt[r], cnt[r + 1]);
      mr[off[r]] = r;
    }
}

__global__ void group_start_kernel(const uint64_t *mh, uint64_t m, uint64_t *flag) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < m; q += step)
    flag[q] = q == 0 || mh[q] != mh[q - 1];
}

__device__ __forceinline__ bool same_list(const uint64_t *cnt, const uint32_t *colors,
                                          uint64_t a, uint64_t b) {
  const uint64_t la = cnt[a + 1] - cnt[a], lb = cnt[b + 1] - cnt[b];
  if (la != lb) return false;
  for (uint64_t t = 0; t < la; ++t)
    if (colors[cnt[a] + t] != colors[cnt[b] + t]) return false;
  return true;
}

// member q of group grp[q] (first member gfirst[grp]): complex[grp] = 1 when
// some member's list differs from the first member's (a hash collision)
__global__ void group_check_kernel(const uint64_t *cnt, const uint32_t *colors,
                                   const uint64_t *mr, const uint64_t *grp, const uint64_t *gfirst,
                                   uint64_t m, uint32_t *complex_) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < m; q += step) {
    const uint64_t f = gfirst[grp[q]];
    if (q != f && !same_list(cnt, colors, mr[q], mr[f])) complex_[grp[q]] = 1;
  }
}

// set ids: singles by genome, multi members by group base + local index; the
// creating k-mer of every id goes to set_first
__global__ void assign_multi_kernel(const uint64_t *mr, const uint64_t *grp, const uint64_t *base,
                                    const uint32_t *local, const uint8_t *creator, uint64_t m,
                                    uint64_t n_single, uint64_t *set_of, uint64_t *set_first) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < m; q += step) {
    const uint64_t id = n_single + base[grp[q]] + local[q];
    set_of[mr[q]] = id;
    if (creator[q]) set_first[id] = mr[q];
  }
}

__global__ void assign_single_kernel(const uint64_t *cnt, const uint32_t *colors, uint64_t n,
                                     const uint64_t *single_id, uint64_t *set_of) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += step)
    if (cnt[r + 1] - cnt[r] == 1) set_of[r] = single_id[colors[cnt[r]]];
}

__global__ void single_first_kernel(const unsigned long long *single_first, const uint64_t *has,
                                    const uint64_t *single_id, uint64_t C, uint64_t *set_first) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < C; g += step)
    if (has[g]) set_first[single_id[g]] = single_first[g];
}

// per set s: dense flag, dense bits (max color + 1) and sparse size
__global__ void set_shape_kernel(const uint64_t *cnt, const uint32_t *colors,
                                 const uint64_t *set_first, uint64_t S, uint64_t C,
                                 uint8_t *dense, uint64_t *dbits, uint64_t *ssize,
                                 unsigned long long *sum_sizes) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < S; s += step) {
    const uint64_t r = set_first[s], size = cnt[r + 1] - cnt[r];
    const bool d = (double)size > (double)C / 64.0;
    dense[s] = d;
    dbits[s] = d ? (uint64_t)colors[cnt[r + 1] - 1] + 1 : 0;
    ssize[s] = d ? 0 : size;
    atomicAdd(sum_sizes, (unsigned long long)size);
  }
}

__global__ void payload_kernel(const uint64_t *cnt, const uint32_t *colors,
                               const uint64_t *set_first, uint64_t S, const uint8_t *dense,
                               const uint64_t *doff, const uint64_t *soff,
                               unsigned long long *dense_words, uint64_t *sparse_vals) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < S; s += step) {
    const uint64_t r = set_first[s];
    for (uint64_t t = cnt[r]; t < cnt[r + 1]; ++t) {
      if (dense[s]) {
        const uint64_t bit = doff[s] + colors[t];
        atomicOr(dense_words + bit / 64, 1ULL << (bit % 64));
      } else {
        sparse_vals[soff[s] + (t - cnt[r])] = colors[t];
      }
    }
  }
}

// Exclusive scan in place over n u64 (total returned).
u64 scan_u64(DeviceBuffer &v, u64 n, CubTemp &tmp) {
  if (n == 0) return 0;
  u64 last = 0, ex_last = 0;
  size_t tb = 0;
  SBWT_CUDA(cudaMemcpy(&last, v.get<u64>() + n - 1, 8, cudaMemcpyDeviceToHost));
  SBWT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, v.get<u64>(), v.get<u64>(), (int64_t)n));
  SBWT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, v.get<u64>(), v.get<u64>(),
                                          (int64_t)n));
  SBWT_CUDA(cudaMemcpy(&ex_last, v.get<u64>() + n - 1, 8, cudaMemcpyDeviceToHost));
  return ex_last + last;
}

template <class T>
std::vector<T> to_host(const DeviceBuffer &b, u64 n) {
  std::vector<T> h(n);
  if (n) SBWT_CUDA(cudaMemcpy(h.data(), b.get(), n * sizeof(T), cudaMemcpyDeviceToHost));
  return h;
}

u8 width_for(u64 maxv) {
  u8 w = 1;
  while (w < 64 && (maxv >> w)) ++w;
  return w;
}

}  // namespace

// SBWT + .tcolors of genomes[0..n_genomes) on `device`.
void build_colored_device(const char *chars, u64 n_chars, const u64 *ends, u64 C, uint32_t k,
                          bool rc, int device, SbwtFile &sbwt, TColorsFile &t) {
  if (k < 2 || k > 31) throw Error(SBWT_E_INVALID, "the GPU builder supports 2 <= k <= 31");
  if (C == 0 || C > (1ULL << 32)) throw Error(SBWT_E_INVALID, "number of genomes out of range");
  for (u64 s = 1; s < C; ++s)
    if (ends[s] < ends[s - 1]) throw Error(SBWT_E_INVALID, "sequence ends must not decrease");
  if (ends[C - 1] > n_chars) throw Error(SBWT_E_INVALID, "sequence end past the chars");
  DeviceGuard dg(device);
  CubTemp tmp;
  size_t tb = 0;
  // (k-mer, genome) pairs, sorted by k-mer (stable: genomes ascend)
  const u64 np = (rc ? 2 : 1) * n_chars;
  DeviceBuffer d_chars(std::max<u64>(n_chars, 1)), d_ends(C * 8);
  DeviceBuffer keys(std::max<u64>(np, 1) * 8), keys2(std::max<u64>(np, 1) * 8);
  DeviceBuffer gen(std::max<u64>(np, 1) * 4), gen2(std::max<u64>(np, 1) * 4);
  if (n_chars) SBWT_CUDA(cudaMemcpy(d_chars.get(), chars, n_chars, cudaMemcpyHostToDevice));
  SBWT_CUDA(cudaMemcpy(d_ends.get(), ends, C * 8, cudaMemcpyHostToDevice));
  if (n_chars)
    kmer_pairs_kernel<<<grid_for(n_chars), 256>>>(d_chars.get<uint8_t>(), n_chars,
                                                  d_ends.get<u64>(), C, k, rc ? 1 : 0,
                                                  keys.get<u64>(), gen.get<uint32_t>());
  SBWT_CUDA(cudaGetLastError());
  d_chars.release();
  if (np) {
    SBWT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get<u64>(), keys2.get<u64>(),
                                              gen.get<uint32_t>(), gen2.get<uint32_t>(),
                                              (int64_t)np, 0, 64));
    SBWT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, keys.get<u64>(),
                                              keys2.get<u64>(), gen.get<uint32_t>(),
                                              gen2.get<uint32_t>(), (int64_t)np, 0, 64));
  }
  // distinct pairs
  DeviceBuffer flag(std::max<u64>(np, 1) * 8), off(std::max<u64>(np, 1) * 8);
  if (np) pair_new_kernel<<<grid_for(np), 256>>>(keys2.get<u64>(), gen2.get<uint32_t>(), np,
                                                 flag.get<u64>());
  SBWT_CUDA(cudaMemcpy(off.get(), flag.get(), np * 8, cudaMemcpyDeviceToDevice));
  const u64 npu = scan_u64(off, np, tmp);
  DeviceBuffer pk(std::max<u64>(npu, 1) * 8), colors(std::max<u64>(npu, 1) * 4);
  if (np) {
    compact_kernel<u64><<<grid_for(np), 256>>>(keys2.get<u64>(), flag.get<u64>(), off.get<u64>(),
                                               np, pk.get<u64>());
    compact_kernel<uint32_t><<<grid_for(np), 256>>>(gen2.get<uint32_t>(), flag.get<u64>(),
                                                    off.get<u64>(), np, colors.get<uint32_t>());
  }
  keys.release(); keys2.release(); gen.release(); gen2.release();
  // k-mers and their color lists (CSR)
  DeviceBuffer kflag(std::max<u64>(npu, 1) * 8), koff(std::max<u64>(npu, 1) * 8);
  if (npu) kmer_new_kernel<<<grid_for(npu), 256>>>(pk.get<u64>(), npu, kflag.get<u64>());
  SBWT_CUDA(cudaMemcpy(koff.get(), kflag.get(), npu * 8, cudaMemcpyDeviceToDevice));
  const u64 n = scan_u64(koff, npu, tmp);
  DeviceBuffer K(std::max<u64>(n, 1) * 8), cnt((n + 1) * 8);
  if (npu) kmer_csr_kernel<<<grid_for(npu), 256>>>(pk.get<u64>(), kflag.get<u64>(),
                                                   koff.get<u64>(), npu, K.get<u64>(),
                                                   cnt.get<u64>());
  SBWT_CUDA(cudaMemcpy(cnt.get<u64>() + n, &npu, 8, cudaMemcpyHostToDevice));
  pk.release(); kflag.release(); koff.release(); flag.release(); off.release();
  // the SBWT of the k-mers, with every k-mer's node
  DeviceBuffer kmer_node(std::max<u64>(n, 1) * 8);
  sbwt = build_from_sorted_keys(K.get<u64>(), n, k, kmer_node.get<u64>());
  K.release();
  const u64 *dcnt = cnt.get<u64>();
  const uint32_t *dcol = colors.get<uint32_t>();
  // singleton sets
  DeviceBuffer single_first(C * 8), has(C * 8), is_multi(std::max<u64>(n, 1) * 8);
  SBWT_CUDA(cudaMemset(single_first.get(), 0xFF, C * 8));
  if (n) classify_kernel<<<grid_for(n), 256>>>(dcnt, dcol, n,
                                               single_first.get<unsigned long long>(),
                                               is_multi.get<u64>());
  has_single_kernel<<<grid_for(C), 256>>>(single_first.get<unsigned long long>(), C,
                                          has.get<u64>());
  DeviceBuffer single_id(C * 8);
  SBWT_CUDA(cudaMemcpy(single_id.get(), has.get(), C * 8, cudaMemcpyDeviceToDevice));
  const u64 n_single = scan_u64(single_id, C, tmp);
  // multi-color k-mers by (hash, rank)
  DeviceBuffer moff(std::max<u64>(n, 1) * 8);
  SBWT_CUDA(cudaMemcpy(moff.get(), is_multi.get(), n * 8, cudaMemcpyDeviceToDevice));
  const u64 m = scan_u64(moff, n, tmp);
  DeviceBuffer mh(std::max<u64>(m, 1) * 8), mr(std::max<u64>(m, 1) * 8);
  DeviceBuffer mh2(std::max<u64>(m, 1) * 8), mr2(std::max<u64>(m, 1) * 8);
  if (n) multi_hash_kernel<<<grid_for(n), 256>>>(dcnt, dcol, is_multi.get<u64>(), moff.get<u64>(),
                                                 n, mh.get<u64>(), mr.get<u64>());
  if (m) {
    SBWT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, mh.get<u64>(), mh2.get<u64>(),
                                              mr.get<u64>(), mr2.get<u64>(), (int64_t)m, 0, 64));
    SBWT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, mh.get<u64>(), mh2.get<u64>(),
                                              mr.get<u64>(), mr2.get<u64>(), (int64_t)m, 0, 64));
  }
  mh.release(); mr.release(); moff.release(); is_multi.release();
  // groups of equal hashes
  DeviceBuffer gflag(std::max<u64>(m, 1) * 8), grp(std::max<u64>(m, 1) * 8);
  if (m) group_start_kernel<<<grid_for(m), 256>>>(mh2.get<u64>(), m, gflag.get<u64>());
  SBWT_CUDA(cudaMemcpy(grp.get(), gflag.get(), m * 8, cudaMemcpyDeviceToDevice));
  const u64 n_groups = scan_u64(grp, m, tmp);  // exclusive: grp[q] + flag = group of q
  // group of q = (exclusive count of starts before q) + flag(q) - 1
  std::vector<u64> h_gflag = to_host<u64>(gflag, m), h_grp = to_host<u64>(grp, m);
  std::vector<u64> h_mr = to_host<u64>(mr2, m);
  std::vector<u64> gfirst(std::max<u64>(n_groups, 1));
  for (u64 q = 0; q < m; ++q) {
    h_grp[q] = h_grp[q] + h_gflag[q] - 1;
    if (h_gflag[q]) gfirst[h_grp[q]] = q;
  }
  SBWT_CUDA(cudaMemcpy(grp.get(), h_grp.data(), m * 8, cudaMemcpyHostToDevice));
  DeviceBuffer d_gfirst(std::max<u64>(n_groups, 1) * 8), complex_(std::max<u64>(n_groups, 1) * 4);
  SBWT_CUDA(cudaMemcpy(d_gfirst.get(), gfirst.data(), n_groups * 8, cudaMemcpyHostToDevice));
  SBWT_CUDA(cudaMemset(complex_.get(), 0, std::max<u64>(n_groups, 1) * 4));
  if (m) group_check_kernel<<<grid_for(m), 256>>>(dcnt, dcol, mr2.get<u64>(), grp.get<u64>(),
                                                  d_gfirst.get<u64>(), m,
                                                  complex_.get<uint32_t>());
  SBWT_CUDA(cudaGetLastError());
  // ids inside each group: one per distinct list, in first-appearance order
  // (a simple group has one; collision groups are resolved here on the host)
  std::vector<uint32_t> h_complex = to_host<uint32_t>(complex_, n_groups);
  std::vector<u64> distinct(std::max<u64>(n_groups, 1), 1);
  std::vector<uint32_t> local(std::max<u64>(m, 1), 0);
  std::vector<uint8_t> creator(std::max<u64>(m, 1), 0);
  std::vector<u64> h_cnt, h_colors_v;
  std::vector<uint32_t> h_colors;
  bool have_lists = false;
  for (u64 gi = 0; gi < n_groups; ++gi) {
    const u64 q0 = gfirst[gi];
    creator[q0] = 1;
    if (!h_complex[gi]) continue;
    if (!have_lists) {
      h_cnt = to_host<u64>(cnt, n + 1);
      h_colors = to_host<uint32_t>(colors, npu);
      have_lists = true;
    }
    auto same = [&](u64 a, u64 b) {
      const u64 la = h_cnt[a + 1] - h_cnt[a], lb = h_cnt[b + 1] - h_cnt[b];
      return la == lb && std::equal(h_colors.begin() + h_cnt[a], h_colors.begin() + h_cnt[a + 1],
                                    h_colors.begin() + h_cnt[b]);
    };
    std::vector<u64> firsts;  // creating member of each local id
    for (u64 q = q0; q < m && h_grp[q] == gi; ++q) {
      u64 id = firsts.size();
      for (u64 f = 0; f < firsts.size(); ++f)
        if (same(h_mr[firsts[f]], h_mr[q])) {
          id = f;
          break;
        }
      if (id == firsts.size()) {
        firsts.push_back(q);
        creator[q] = 1;
      }
      local[q] = (uint32_t)id;
    }
    distinct[gi] = firsts.size();
  }
  std::vector<u64> base(std::max<u64>(n_groups, 1), 0);
  u64 n_multi_sets = 0;
  for (u64 gi = 0; gi < n_groups; ++gi) {
    base[gi] = n_multi_sets;
    n_multi_sets += distinct[gi];
  }
  const u64 S = n_single + n_multi_sets;
  DeviceBuffer d_base(std::max<u64>(n_groups, 1) * 8), d_local(std::max<u64>(m, 1) * 4),
      d_creator(std::max<u64>(m, 1)), set_of(std::max<u64>(n, 1) * 8),
      set_first(std::max<u64>(S, 1) * 8);
  SBWT_CUDA(cudaMemcpy(d_base.get(), base.data(), n_groups * 8, cudaMemcpyHostToDevice));
  SBWT_CUDA(cudaMemcpy(d_local.get(), local.data(), m * 4, cudaMemcpyHostToDevice));
  SBWT_CUDA(cudaMemcpy(d_creator.get(), creator.data(), m, cudaMemcpyHostToDevice));
  if (m) assign_multi_kernel<<<grid_for(m), 256>>>(mr2.get<u64>(), grp.get<u64>(),
                                                   d_base.get<u64>(), d_local.get<uint32_t>(),
                                                   d_creator.get<uint8_t>(), m, n_single,
                                                   set_of.get<u64>(), set_first.get<u64>());
  if (n) assign_single_kernel<<<grid_for(n), 256>>>(dcnt, dcol, n, single_id.get<u64>(),
                                                    set_of.get<u64>());
  single_first_kernel<<<grid_for(C), 256>>>(single_first.get<unsigned long long>(),
                                            has.get<u64>(), single_id.get<u64>(), C,
                                            set_first.get<u64>());
  SBWT_CUDA(cudaGetLastError());
  // set shapes and payloads in id order
  DeviceBuffer dense(std::max<u64>(S, 1)), dbits(std::max<u64>(S, 1) * 8),
      ssize(std::max<u64>(S, 1) * 8), d_sum(8);
  SBWT_CUDA(cudaMemset(d_sum.get(), 0, 8));
  if (S) set_shape_kernel<<<grid_for(S), 256>>>(dcnt, dcol, set_first.get<u64>(), S, C,
                                                dense.get<uint8_t>(), dbits.get<u64>(),
                                                ssize.get<u64>(),
                                                d_sum.get<unsigned long long>());
  std::vector<uint8_t> h_dense = to_host<uint8_t>(dense, S);
  std::vector<u64> h_dbits = to_host<u64>(dbits, S), h_ssize = to_host<u64>(ssize, S);
  const u64 dense_total = scan_u64(dbits, S, tmp);
  const u64 sparse_total = scan_u64(ssize, S, tmp);
  DeviceBuffer dense_words(((dense_total + 63) / 64 + 1) * 8),
      sparse_vals(std::max<u64>(sparse_total, 1) * 8);
  SBWT_CUDA(cudaMemset(dense_words.get(), 0, ((dense_total + 63) / 64 + 1) * 8));
  if (S) payload_kernel<<<grid_for(S), 256>>>(dcnt, dcol, set_first.get<u64>(), S,
                                              dense.get<uint8_t>(), dbits.get<u64>(),
                                              ssize.get<u64>(),
                                              dense_words.get<unsigned long long>(),
                                              sparse_vals.get<u64>());
  SBWT_CUDA(cudaGetLastError());
  // host layout
  t = TColorsFile{};
  t.is_dense_marks.resize(S);
  std::vector<u64> dense_iv{0}, sparse_iv{0};
  u64 dacc = 0, sacc = 0;
  for (u64 s = 0; s < S; ++s) {
    if (h_dense[s]) {
      t.is_dense_marks.set(s);
      dacc += h_dbits[s];
      dense_iv.push_back(dacc);
    } else {
      sacc += h_ssize[s];
      sparse_iv.push_back(sacc);
    }
  }
  t.dense_arrays.num_bits = dense_total;
  {
    const std::vector<u64> w = to_host<u64>(dense_words, (dense_total + 63) / 64);
    t.dense_arrays.words.assign(w.begin(), w.end());
  }
  t.dense_arrays_intervals.assign(dense_iv, width_for(dense_iv.back()));
  t.sparse_arrays.assign(to_host<u64>(sparse_vals, sparse_total), width_for(C - 1));
  t.sparse_arrays_intervals.assign(sparse_iv, width_for(sparse_iv.back()));
  t.key_kmer_marks.resize(sbwt.n_nodes);
  for (u64 v : to_host<u64>(kmer_node, n)) t.key_kmer_marks.set(v);
  t.color_set_idxs.assign(to_host<u64>(set_of, n), width_for(S ? S - 1 : 0));
  t.max_color_set_idx = S ? S - 1 : 0;
  t.largest_color = C - 1;
  SBWT_CUDA(cudaMemcpy(&t.sum_color_set_sizes, d_sum.get(), 8, cudaMemcpyDeviceToHost));
}

}  // namespace sbwt

extern "C" int sbwt_build_colored_index(const char *chars, uint64_t n_chars,
                                        const uint64_t *genome_ends, uint64_t n_genomes,
                                        uint32_t k, int add_rc, const char *sbwt_path,
                                        const char *tcolors_path, int device,
                                        uint64_t *n_nodes) {
  if ((n_chars && !chars) || !genome_ends || !sbwt_path || !tcolors_path) {
    sbwt::set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return sbwt::guarded([&] {
    sbwt::SbwtFile s;
    sbwt::TColorsFile t;
    sbwt::build_colored_device(chars, n_chars, genome_ends, n_genomes, k, add_rc != 0, device, s,
                               t);
    sbwt::write_sbwt(sbwt_path, s);
    sbwt::write_tcolors(tcolors_path, t);
    if (n_nodes) *n_nodes = s.n_nodes;
  });
}
