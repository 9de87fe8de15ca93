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
                             uint8_t *nlen) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n + nd; i += step) {
    if (i < n) {  // k-mer: after every dummy of key <= its key
      const uint64_t p = i + upper_bound_u64(dkey, nd, K[i]);
      nkey[p] = K[i];
      nlen[p] = (uint8_t)k;
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
  const u64 *K = keys.get<u64>();
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
                                            nlen.get<uint8_t>());
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
