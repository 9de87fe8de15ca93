// Colors step on the B200: per-read color counting and the tau threshold.
//
// Reference behaviour restated (SBWT-Search, paths in its src/):
//   d_color_search   ColorSearcher/ColorSearcher.cuh:68-206 (+ helpers :208-318)
//   d_post_process   ColorSearcher/ColorPostProcessor.cuh:21-43
//   threshold        ColorResultsPrinter/ContinuousColorResultsPrinter.hpp:235-263
//   .tcolors layout  ColorIndexBuilder/ColorIndexBuilder.cpp:23-86
//
// Semantics: count[r][c] = number of found k-mers of read r whose color set
// holds c.  The reference gets there with one thread per k-mer, a warp-wide
// loop over the color span and u8 per-(warp, color) partial counts summed by
// a second kernel into an R x C u64 matrix copied to the host.  Here one warp
// owns one read: lane i owns colors [64 i, 64 i + 64) (and i + 32, ... for
// more than 2048 colors) as bit-sliced counters in shared memory (plane j
// holds bit j of 64 counters), a dense color row is added with a ripple-carry
// over the planes (no atomics, no conflicts), a sparse list is turned into the
// same per-lane row words with warp shuffles, and the threshold is a
// bit-sliced comparison; only the passing color bitmask leaves the kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "colors_internal.hpp"
#include "common.hpp"
#include "formats.hpp"
#include "rank_blocks.cuh"

namespace sbwt {

constexpr int kColorWarps = 4;  // warps (reads in flight) per block

struct ColorsJob {
  const uint64_t *vals;     // SBWT indexes (markers allowed when counted)
  const uint64_t *offs;     // n_reads + 1
  const uint64_t *not_found;  // per read or nullptr
  const uint64_t *invalid;    // per read or nullptr
  uint64_t n_reads;
  double tau;
  uint32_t include_not_found, include_invalid;
  uint32_t planes;          // bit planes of the counters
  uint64_t *pass_bits;      // n_reads x row_words (mode 0)
  uint32_t *pass_count;     // n_reads (mode 0)
  uint32_t *counts;         // n_reads x num_colors (mode 1)
};

__device__ __forceinline__ uint64_t rank_key(const ColorsView &cv, uint64_t i) {
  const uint64_t b = i / kBlockBits;
  const Block B = load_block(cv.key_blocks + b);
  return cv.key_l0[b >> kSuperchunkShift] + block_rank(B, (uint32_t)(i - b * kBlockBits));
}

// Adds one row word x (64 colors, one bit each) into the bit-sliced counters
// planes[j * stride] (j = 0..P-1): ripple carry, stops when the carry dies.
__device__ __forceinline__ void add_word(uint64_t *planes, uint32_t stride, uint32_t P,
                                         uint64_t x) {
  for (uint32_t j = 0; j < P && x; ++j) {
    const uint64_t p = planes[j * stride];
    planes[j * stride] = p ^ x;
    x &= p;
  }
}

// mode 0: pass bitmask + count per read; mode 1: full counts.
template <int MODE>
__global__ void __launch_bounds__(32 * kColorWarps) colors_kernel(ColorsView cv,
                                                                  ColorsJob job,
                                                                  uint32_t *err) {
  extern __shared__ uint64_t smem[];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t WL = cv.words_per_lane, P = job.planes;
  // per warp: P planes x (32 * WL) words, plane-major so lanes are contiguous
  const uint32_t stride = 32 * WL;
  uint64_t *planes = smem + (uint64_t)wid * P * stride;
  const uint64_t warps = (uint64_t)gridDim.x * kColorWarps;
  for (uint64_t r = blockIdx.x * (uint64_t)kColorWarps + wid; r < job.n_reads; r += warps) {
    for (uint32_t q = lane; q < P * stride; q += 32) planes[q] = 0;
    __syncwarp();
    const uint64_t o0 = job.offs[r], o1 = job.offs[r + 1];
    uint32_t found = 0, not_found = 0, invalid = 0;
    for (uint64_t base = o0; base < o1; base += 32) {
      // lookup phase: lane t resolves the color set of k-mer base + t
      const uint64_t t = base + lane;
      bool have = false;
      ulonglong2 d = make_ulonglong2(0, 0);
      if (t < o1) {
        const uint64_t v = job.vals[t];
        if (v == SBWT_NOT_FOUND) {
          ++not_found;
        } else if (v == SBWT_INVALID) {
          ++invalid;
        } else if (v >= cv.key_bits) {
          atomicOr(err, 1u);
        } else {
          ++found;
          const uint64_t j = rank_key(cv, v);
          if (j >= cv.n_keys) {
            atomicOr(err, 1u);
          } else {
            const uint32_t s = __ldg(cv.csi + j);
            if (s >= cv.n_sets) {
              atomicOr(err, 1u);
            } else {
              d = __ldg(cv.desc + s);
              have = true;
            }
          }
        }
      }
      // add phase: the warp adds the (up to 32) sets one after the other
      uint32_t todo = __ballot_sync(0xFFFFFFFFu, have);
      while (todo) {
        const int src = __ffs(todo) - 1;
        todo &= todo - 1;
        const uint64_t start = __shfl_sync(0xFFFFFFFFu, d.x, src);
        const uint64_t meta = __shfl_sync(0xFFFFFFFFu, d.y, src);
        const uint32_t len = (uint32_t)(meta >> 1);
        if (meta & 1ULL) {  // dense: len = words of the row
          for (uint32_t w = 0; w < WL; ++w) {
            const uint32_t word = lane + 32 * w;
            if (word < len) add_word(planes + word, stride, P, __ldg(cv.dense + start + word));
          }
        } else {  // sparse: len ids, turned into per-lane row words
          for (uint32_t c0 = 0; c0 < len; c0 += 32) {
            const uint32_t id = (c0 + lane < len) ? __ldg(cv.sparse + start + c0 + lane) : 0xFFFFFFFFu;
            const uint32_t m = min(32u, len - c0);
            uint64_t x[4] = {0, 0, 0, 0};  // up to WL <= 4 words per lane in registers
            for (uint32_t q = 0; q < m; ++q) {
              const uint32_t c = __shfl_sync(0xFFFFFFFFu, id, q);
              const uint32_t word = c >> 6;
              if ((word & 31) == lane && (word >> 5) < WL) x[(word >> 5) & 3] |= 1ULL << (c & 63);
            }
            for (uint32_t w = 0; w < WL && w < 4; ++w)
              if (x[w]) add_word(planes + lane + 32 * w, stride, P, x[w]);
          }
        }
      }
    }
    __syncwarp();
    // per-read sizes
    for (int o = 16; o; o >>= 1) {
      found += __shfl_xor_sync(0xFFFFFFFFu, found, o);
      not_found += __shfl_xor_sync(0xFFFFFFFFu, not_found, o);
      invalid += __shfl_xor_sync(0xFFFFFFFFu, invalid, o);
    }
    if (job.not_found) not_found += (uint32_t)job.not_found[r];
    if (job.invalid) invalid += (uint32_t)job.invalid[r];
    if (MODE == 0) {
      const uint64_t size = (uint64_t)found + (job.include_not_found ? not_found : 0) +
                            (job.include_invalid ? invalid : 0);
      const uint64_t minimum = (uint64_t)ceil((double)size * job.tau);
      uint32_t passing = 0;
      for (uint32_t w = 0; w < WL; ++w) {
        const uint32_t word = lane + 32 * w;
        uint64_t ge = 0;
        if (minimum > 0 && word < cv.row_words && (P >= 64 || (minimum >> P) == 0)) {
          uint64_t gt = 0, eq = ~0ULL;
          for (int j = (int)P - 1; j >= 0; --j) {
            const uint64_t pl = planes[(uint32_t)j * stride + word];
            if ((minimum >> j) & 1ULL) {
              eq &= pl;
            } else {
              gt |= eq & pl;
              eq &= ~pl;
            }
          }
          ge = gt | eq;
          const uint32_t rem = cv.num_colors - word * 64;
          if (rem < 64) ge &= (1ULL << rem) - 1ULL;
        }
        if (word < cv.row_words) job.pass_bits[r * cv.row_words + word] = ge;
        passing += __popcll(ge);
      }
      for (int o = 16; o; o >>= 1) passing += __shfl_xor_sync(0xFFFFFFFFu, passing, o);
      if (lane == 0) job.pass_count[r] = passing;
    } else {
      for (uint32_t w = 0; w < WL; ++w) {
        const uint32_t word = lane + 32 * w;
        if (word >= cv.row_words) continue;
        for (uint32_t b = 0; b < 64; ++b) {
          const uint32_t c = word * 64 + b;
          if (c >= cv.num_colors) break;
          uint32_t cnt = 0;
          for (uint32_t j = 0; j < P; ++j)
            cnt |= (uint32_t)((planes[j * stride + word] >> b) & 1ULL) << j;
          job.counts[r * cv.num_colors + c] = cnt;
        }
      }
    }
    __syncwarp();
  }
}

// Expands each read's pass bitmask into ascending color ids at ids_off[r].
__global__ void emit_ids_kernel(const uint64_t *pass_bits, uint32_t row_words,
                                const uint64_t *ids_off, uint64_t n_reads,
                                uint32_t *ids, uint64_t capacity) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warp0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = warp0; r < n_reads; r += warps) {
    uint64_t out = ids_off[r];
    for (uint32_t w0 = 0; w0 < row_words; w0 += 32) {
      const uint32_t word = w0 + lane;
      uint64_t m = word < row_words ? pass_bits[r * row_words + word] : 0;
      const uint32_t cnt = __popcll(m);
      uint32_t incl = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      uint64_t pos = out + incl - cnt;
      while (m) {
        const uint32_t b = __ffsll(m) - 1;
        m &= m - 1;
        if (pos < capacity) ids[pos] = word * 64 + b;
        ++pos;
      }
      out += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
  }
}

// Exclusive scan of u32 counts into u64 offsets (one block; small inputs are
// the common case, large ones loop).
__global__ void scan_counts_kernel(const uint32_t *cnt, uint64_t n, uint64_t *off) {
  __shared__ uint64_t carry;
  __shared__ uint64_t wsum[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint64_t b0 = 0; b0 < n; b0 += blockDim.x) {
    const uint64_t i = b0 + threadIdx.x;
    uint64_t v = i < n ? cnt[i] : 0, x = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint64_t s = lane < blockDim.x / 32 ? wsum[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
        if (lane >= (uint32_t)o) s += y;
      }
      wsum[lane] = s;
    }
    __syncthreads();
    const uint64_t ex = carry + (wid ? wsum[wid - 1] : 0) + x - v;
    if (i < n) off[i] = ex;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = ex + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) off[n] = carry;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
void build_rank_blocks_host(const u64 *words, u64 num_bits, std::vector<Block> &blocks,
                            std::vector<u64> &l0, u64 &total);

ColorsImpl::ColorsImpl(const TColorsFile &t, int device_) {
  device = device_;
  DeviceGuard g(device);
  num_colors = t.num_colors();
  if (num_colors == 0 || num_colors > (1u << 20))
    throw Error(SBWT_E_FORMAT, "number of colors out of range");
  const u64 n_sets = t.is_dense_marks.num_bits;
  const u64 n_keys = t.color_set_idxs.size();
  // per-set descriptors + word-aligned dense rows + u32 sparse ids
  std::vector<ulonglong2> desc(std::max<u64>(n_sets, 1));
  std::vector<u64> dense_words;
  std::vector<uint32_t> sparse(std::max<u64>(t.sparse_arrays.size(), 1));
  for (u64 i = 0; i < t.sparse_arrays.size(); ++i) {
    const u64 v = t.sparse_arrays.get(i);
    if (v >= num_colors) throw Error(SBWT_E_FORMAT, "sparse color id out of range");
    sparse[i] = (uint32_t)v;
  }
  u64 n_dense = 0, n_sparse = 0;
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
      const u64 at = dense_words.size();
      dense_words.resize(at + nw, 0);
      for (u64 c = 0; c < nbits; ++c)
        if (t.dense_arrays.get(st + c)) dense_words[at + c / 64] |= 1ULL << (c % 64);
      desc[s] = make_ulonglong2(at, (nw << 1) | 1ULL);
      ++n_dense;
    } else {
      if (n_sparse + 1 >= n_sparse_iv) throw Error(SBWT_E_FORMAT, "sparse intervals too short");
      const u64 st = t.sparse_arrays_intervals.get(n_sparse);
      const u64 en = t.sparse_arrays_intervals.get(n_sparse + 1);
      if (en < st || en > t.sparse_arrays.size())
        throw Error(SBWT_E_FORMAT, "sparse interval out of range");
      desc[s] = make_ulonglong2(st, (en - st) << 1);
      ++n_sparse;
    }
  }
  if (dense_words.empty()) dense_words.push_back(0);
  std::vector<uint32_t> csi(std::max<u64>(n_keys, 1));
  for (u64 j = 0; j < n_keys; ++j) {
    const u64 v = t.color_set_idxs.get(j);
    if (v >= n_sets) throw Error(SBWT_E_FORMAT, "color set index out of range");
    csi[j] = (uint32_t)v;
  }
  std::vector<Block> kb;
  std::vector<u64> kl0;
  u64 total_keys = 0;
  build_rank_blocks_host(t.key_kmer_marks.words.data(), t.key_kmer_marks.num_bits, kb, kl0,
                         total_keys);
  if (total_keys > n_keys)
    throw Error(SBWT_E_FORMAT, "more key k-mers than color set indexes");
  auto up = [&](DeviceBuffer &b, const void *src, size_t bytes) {
    b.resize(bytes);
    SBWT_CUDA(cudaMemcpy(b.get(), src, bytes, cudaMemcpyHostToDevice));
  };
  up(key_blocks, kb.data(), kb.size() * sizeof(Block));
  up(key_l0, kl0.data(), kl0.size() * 8);
  up(csi_buf, csi.data(), csi.size() * 4);
  up(desc_buf, desc.data(), desc.size() * sizeof(ulonglong2));
  up(dense_buf, dense_words.data(), dense_words.size() * 8);
  up(sparse_buf, sparse.data(), sparse.size() * 4);
  view = ColorsView{};
  view.key_blocks = key_blocks.get<Block>();
  view.key_l0 = key_l0.get<u64>();
  view.key_bits = t.key_kmer_marks.num_bits;
  view.csi = csi_buf.get<uint32_t>();
  view.n_keys = n_keys;
  view.desc = desc_buf.get<ulonglong2>();
  view.n_sets = n_sets;
  view.dense = dense_buf.get<u64>();
  view.sparse = sparse_buf.get<uint32_t>();
  view.num_colors = (uint32_t)num_colors;
  view.row_words = (uint32_t)((num_colors + 63) / 64);
  view.words_per_lane = (view.row_words + 31) / 32;
  if (view.words_per_lane > 4)
    throw Error(SBWT_E_FORMAT, "more than 8192 colors are not supported");
  device_bytes = key_blocks.size() + key_l0.size() + csi_buf.size() + desc_buf.size() +
                 dense_buf.size() + sparse_buf.size();
}

struct ColorsWorkspace {
  int device = -1;
  DeviceBuffer vals, offs, nf, inv, pass_bits, pass_count, ids_off, ids, counts, err;
  cudaStream_t stream = nullptr;
  ~ColorsWorkspace() {
    if (stream) cudaStreamDestroy(stream);
  }
};

static ColorsWorkspace &colors_workspace(int device) {
  thread_local std::unique_ptr<ColorsWorkspace> ws[16];
  if (device < 0 || device >= 16) throw Error(SBWT_E_INVALID, "device id out of range");
  auto &p = ws[device];
  if (!p) {
    p = std::make_unique<ColorsWorkspace>();
    p->device = device;
    SBWT_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    p->err.resize(4);
    SBWT_CUDA(cudaMemset(p->err.get(), 0, 4));
  }
  return *p;
}

static uint32_t planes_for(u64 max_kmers) {
  uint32_t P = 1;
  while (P < 40 && (max_kmers >> P)) ++P;
  return P;
}

// Runs the colors kernel on device-resident arrays.  mode 0 -> pass bits +
// counts; mode 1 -> counts.  max_kmers bounds the per-read k-mer count.
void ColorsImpl::launch(const u64 *d_vals, const u64 *d_offs, const u64 *d_nf,
                        const u64 *d_inv, u64 n_reads, u64 max_kmers, double tau,
                        u32 flags, int mode, u64 *d_pass_bits, uint32_t *d_pass_count,
                        uint32_t *d_counts, uint32_t *d_err, cudaStream_t st) const {
  if (n_reads == 0) return;
  ColorsJob job{};
  job.vals = d_vals;
  job.offs = d_offs;
  job.not_found = d_nf;
  job.invalid = d_inv;
  job.n_reads = n_reads;
  job.tau = tau;
  job.include_not_found = (flags & SBWT_INCLUDE_NOT_FOUND) ? 1 : 0;
  job.include_invalid = (flags & SBWT_INCLUDE_INVALID) ? 1 : 0;
  job.planes = planes_for(max_kmers);
  job.pass_bits = d_pass_bits;
  job.pass_count = d_pass_count;
  job.counts = d_counts;
  const size_t smem = (size_t)kColorWarps * job.planes * 32 * view.words_per_lane * 8;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const u64 blocks = std::min<u64>((n_reads + kColorWarps - 1) / kColorWarps, (u64)sms * 32);
  if (mode == 0) {
    SBWT_CUDA(cudaFuncSetAttribute(colors_kernel<0>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    colors_kernel<0><<<(unsigned)blocks, 32 * kColorWarps, smem, st>>>(view, job, d_err);
  } else {
    SBWT_CUDA(cudaFuncSetAttribute(colors_kernel<1>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    colors_kernel<1><<<(unsigned)blocks, 32 * kColorWarps, smem, st>>>(view, job, d_err);
  }
  SBWT_CUDA(cudaGetLastError());
}

// The colors step of one device-resident batch without host synchronisation
// (capturable): per-read counting over `vals` (index-step results, -1/-2
// markers counted, not looked up) + threshold, scan of the per-read pass
// counts into d_ids_off (n_reads + 1), ids into d_ids (capacity bound checked
// on the device; d_ids_off[n_reads] is the required size).
void ColorsImpl::enqueue_pseudoalign(const u64 *d_vals, const u64 *d_offs, u64 n_reads,
                                     u64 max_kmers, double tau, u32 flags, u64 *d_pass_bits,
                                     uint32_t *d_pass_count, u64 *d_ids_off, uint32_t *d_ids,
                                     u64 ids_capacity, uint32_t *d_err,
                                     cudaStream_t st) const {
  if (n_reads == 0) {
    SBWT_CUDA(cudaMemsetAsync(d_ids_off, 0, 8, st));
    return;
  }
  launch(d_vals, d_offs, nullptr, nullptr, n_reads, max_kmers, tau, flags, 0, d_pass_bits,
         d_pass_count, nullptr, d_err, st);
  scan_counts_kernel<<<1, 1024, 0, st>>>(d_pass_count, n_reads, d_ids_off);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const u64 blocks = std::min<u64>((n_reads + 7) / 8, (u64)sms * 16);
  emit_ids_kernel<<<(unsigned)std::max<u64>(blocks, 1), 256, 0, st>>>(
      d_pass_bits, view.row_words, d_ids_off, n_reads, d_ids, ids_capacity);
  SBWT_CUDA(cudaGetLastError());
}

void ColorsImpl::prepare_launch(u64 max_kmers) const {
  const uint32_t P = planes_for(max_kmers);
  const size_t smem = (size_t)kColorWarps * P * 32 * view.words_per_lane * 8;
  SBWT_CUDA(cudaFuncSetAttribute(colors_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  SBWT_CUDA(cudaFuncSetAttribute(colors_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
}

static u64 max_span(const u64 *offs, u64 n_reads) {
  u64 m = 0;
  for (u64 r = 0; r < n_reads; ++r) {
    if (offs[r + 1] < offs[r]) throw Error(SBWT_E_INVALID, "offsets must be non-decreasing");
    m = std::max(m, offs[r + 1] - offs[r]);
  }
  return m;
}

static void check_colors_err(ColorsWorkspace &ws, cudaStream_t st) {
  uint32_t e = 0;
  SBWT_CUDA(cudaMemcpyAsync(&e, ws.err.get(), 4, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaStreamSynchronize(st));
  if (e) {
    SBWT_CUDA(cudaMemset(ws.err.get(), 0, 4));
    throw Error(SBWT_E_INVALID, "an SBWT index is not a key k-mer of this color index");
  }
}

void ColorsImpl::counts(const u64 *vals, const u64 *offs, u64 n_reads, uint32_t *out,
                        u32 flags, cudaStream_t user_stream) const {
  DeviceGuard g(device);
  ColorsWorkspace &ws = colors_workspace(device);
  if (n_reads == 0) return;
  if (flags & SBWT_DEVICE_POINTERS) {
    std::vector<u64> h(n_reads + 1);
    SBWT_CUDA(cudaMemcpyAsync(h.data(), offs, (n_reads + 1) * 8, cudaMemcpyDeviceToHost,
                              user_stream));
    SBWT_CUDA(cudaStreamSynchronize(user_stream));
    launch(vals, offs, nullptr, nullptr, n_reads, max_span(h.data(), n_reads), 0.0, 0, 1,
           nullptr, nullptr, out, ws.err.get<uint32_t>(), user_stream);
    check_colors_err(ws, user_stream);
    return;
  }
  const u64 mk = max_span(offs, n_reads);
  const u64 n_vals = offs[n_reads] - offs[0];
  cudaStream_t st = ws.stream;
  ws.vals.ensure(std::max<u64>(n_vals, 1) * 8);
  ws.offs.ensure((n_reads + 1) * 8);
  ws.counts.ensure(n_reads * num_colors * 4);
  // offsets are rebased to the first value
  std::vector<u64> ro(n_reads + 1);
  for (u64 r = 0; r <= n_reads; ++r) ro[r] = offs[r] - offs[0];
  if (n_vals)
    SBWT_CUDA(cudaMemcpyAsync(ws.vals.get(), vals + offs[0], n_vals * 8,
                              cudaMemcpyHostToDevice, st));
  SBWT_CUDA(cudaMemcpyAsync(ws.offs.get(), ro.data(), (n_reads + 1) * 8,
                            cudaMemcpyHostToDevice, st));
  launch(ws.vals.get<u64>(), ws.offs.get<u64>(), nullptr, nullptr, n_reads, mk, 0.0, 0, 1,
         nullptr, nullptr, ws.counts.get<uint32_t>(), ws.err.get<uint32_t>(), st);
  SBWT_CUDA(cudaMemcpyAsync(out, ws.counts.get(), n_reads * num_colors * 4,
                            cudaMemcpyDeviceToHost, st));
  check_colors_err(ws, st);
}

void ColorsImpl::pseudoalign(const u64 *vals, const u64 *offs, const u64 *nf,
                             const u64 *inv, u64 n_reads, double tau, u32 flags,
                             uint32_t *ids, u64 capacity, u64 *ids_offsets,
                             cudaStream_t user_stream) const {
  DeviceGuard g(device);
  ColorsWorkspace &ws = colors_workspace(device);
  const u32 rw = view.row_words;
  const bool dev = flags & SBWT_DEVICE_POINTERS;
  cudaStream_t st = dev ? user_stream : ws.stream;
  if (n_reads == 0) {
    if (dev) {
      SBWT_CUDA(cudaMemsetAsync(ids_offsets, 0, 8, st));
    } else {
      ids_offsets[0] = 0;
    }
    return;
  }
  const u64 *d_vals = vals, *d_offs = offs, *d_nf = nf, *d_inv = inv;
  u64 mk = 0;
  if (dev) {
    std::vector<u64> h(n_reads + 1);
    SBWT_CUDA(cudaMemcpyAsync(h.data(), offs, (n_reads + 1) * 8, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
    mk = max_span(h.data(), n_reads);
  } else {
    mk = max_span(offs, n_reads);
    const u64 n_vals = offs[n_reads] - offs[0];
    ws.vals.ensure(std::max<u64>(n_vals, 1) * 8);
    ws.offs.ensure((n_reads + 1) * 8);
    std::vector<u64> ro(n_reads + 1);
    for (u64 r = 0; r <= n_reads; ++r) ro[r] = offs[r] - offs[0];
    if (n_vals)
      SBWT_CUDA(cudaMemcpyAsync(ws.vals.get(), vals + offs[0], n_vals * 8,
                                cudaMemcpyHostToDevice, st));
    SBWT_CUDA(cudaMemcpyAsync(ws.offs.get(), ro.data(), (n_reads + 1) * 8,
                              cudaMemcpyHostToDevice, st));
    d_vals = ws.vals.get<u64>();
    d_offs = ws.offs.get<u64>();
    d_nf = d_inv = nullptr;
    if (nf && (flags & SBWT_INCLUDE_NOT_FOUND)) {
      ws.nf.ensure(n_reads * 8);
      SBWT_CUDA(cudaMemcpyAsync(ws.nf.get(), nf, n_reads * 8, cudaMemcpyHostToDevice, st));
      d_nf = ws.nf.get<u64>();
    }
    if (inv && (flags & SBWT_INCLUDE_INVALID)) {
      ws.inv.ensure(n_reads * 8);
      SBWT_CUDA(cudaMemcpyAsync(ws.inv.get(), inv, n_reads * 8, cudaMemcpyHostToDevice, st));
      d_inv = ws.inv.get<u64>();
    }
  }
  if (!(flags & SBWT_INCLUDE_NOT_FOUND)) d_nf = nullptr;
  if (!(flags & SBWT_INCLUDE_INVALID)) d_inv = nullptr;
  ws.pass_bits.ensure(n_reads * rw * 8);
  ws.pass_count.ensure(n_reads * 4);
  ws.ids_off.ensure((n_reads + 1) * 8);
  launch(d_vals, d_offs, d_nf, d_inv, n_reads, mk, tau, flags, 0, ws.pass_bits.get<u64>(),
         ws.pass_count.get<uint32_t>(), nullptr, ws.err.get<uint32_t>(), st);
  u64 *d_ids_off = dev ? ids_offsets : ws.ids_off.get<u64>();
  scan_counts_kernel<<<1, 1024, 0, st>>>(ws.pass_count.get<uint32_t>(), n_reads, d_ids_off);
  SBWT_CUDA(cudaGetLastError());
  u64 total = 0;
  SBWT_CUDA(cudaMemcpyAsync(&total, d_ids_off + n_reads, 8, cudaMemcpyDeviceToHost, st));
  check_colors_err(ws, st);
  if (!dev) {
    SBWT_CUDA(cudaMemcpyAsync(ids_offsets, ws.ids_off.get(), (n_reads + 1) * 8,
                              cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
  }
  if (total > capacity) throw Error(SBWT_E_CAPACITY, "ids_capacity too small");
  uint32_t *d_ids = ids;
  if (!dev) {
    ws.ids.ensure(std::max<u64>(total, 1) * 4);
    d_ids = ws.ids.get<uint32_t>();
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const u64 blocks = std::min<u64>((n_reads + 7) / 8, (u64)sms * 16);
  emit_ids_kernel<<<(unsigned)std::max<u64>(blocks, 1), 256, 0, st>>>(
      ws.pass_bits.get<u64>(), rw, d_ids_off, n_reads, d_ids, capacity);
  SBWT_CUDA(cudaGetLastError());
  if (!dev) {
    if (total)
      SBWT_CUDA(cudaMemcpyAsync(ids, d_ids, total * 4, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
  }
}

}  // namespace sbwt
