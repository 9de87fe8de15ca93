// Result formatting on the GPU: the bytes the reference's printers write,
// produced on the device so that the device->host copy carries final output.
//
// Index results (src/IndexResultsPrinter/: AsciiContinuousIndexResultsPrinter
// .cpp:50-55, BinaryContinuousIndexResultsPrinter, BoolContinuousIndexResults
// Printer): per read, ascii = decimal tokens ("-1" not found, "-2" invalid)
// separated by ' ' and ended by '\n'; binary = one u64 per k-mer then u64 -3;
// bool = '0' found / '1' not found / '2' invalid per k-mer then '\n'.
// Color results (src/ColorResultsPrinter/: AsciiContinuousColorResultsPrinter
// .cpp:74-79, Binary..., Csv...): per read, ascii = ids separated by ' ' and
// ended by '\n'; binary = one u64 per id then u64 -1; csv = one "0/1" per
// color separated by ',' and ended by '\n'.  Headers (and the csv title row)
// are written once per file by the host writers, not here.
//
// Ascii needs the byte length of every read before anything is written: one
// warp per read sums its token lengths, a multi-block scan turns the lengths
// into offsets, and one warp per read writes its tokens at warp-scanned
// positions.  The other formats have closed-form offsets.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <memory>

#include "common.hpp"

namespace sbwt {

namespace {

constexpr uint32_t FULL = 0xFFFFFFFFu;
constexpr uint32_t kScanThreads = 1024, kScanPer = 4, kScanSpan = kScanThreads * kScanPer;

__device__ __forceinline__ uint32_t dec_len(uint64_t v) {
  uint32_t n = 1;
  uint64_t p = 10;
  while (n < 20 && v >= p) {
    ++n;
    p *= 10;
  }
  return n;
}

__device__ __forceinline__ void put_dec(uint8_t *out, uint64_t v, uint32_t n) {
  if (v < (1ULL << 32)) {
    uint32_t x = (uint32_t)v;
    for (uint32_t i = n; i-- > 0;) {
      out[i] = (uint8_t)('0' + x % 10);
      x /= 10;
    }
  } else {
    for (uint32_t i = n; i-- > 0;) {
      out[i] = (uint8_t)('0' + v % 10);
      v /= 10;
    }
  }
}

// Ascii token of one index result: its length and its bytes.
__device__ __forceinline__ uint32_t index_token_len(uint64_t v) {
  return (v == SBWT_NOT_FOUND || v == SBWT_INVALID) ? 2 : dec_len(v);
}
__device__ __forceinline__ void index_token(uint8_t *out, uint64_t v, uint32_t n) {
  if (v == SBWT_NOT_FOUND) {
    out[0] = '-';
    out[1] = '1';
  } else if (v == SBWT_INVALID) {
    out[0] = '-';
    out[1] = '2';
  } else {
    put_dec(out, v, n);
  }
}

// k-mers of read r (reads shorter than k have none), from the read ends.
__device__ __forceinline__ uint64_t kmers_of(const uint64_t *ends, uint64_t r, uint32_t k) {
  const uint64_t len = ends[r] - (r ? ends[r - 1] : 0);
  return len >= k ? len - k + 1 : 0;
}

__device__ __forceinline__ uint64_t warp_sum(uint64_t x) {
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
  return x;
}

// Exclusive warp scan; *total = warp sum.
__device__ __forceinline__ uint64_t warp_exclusive(uint64_t v, uint64_t *total) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  *total = __shfl_sync(FULL, x, 31);
  return x - v;
}

// Per read (one warp each): k-mers -> kmers[r], ascii bytes -> bytes[r].
__global__ void index_lengths_kernel(const uint64_t *res, const uint64_t *ends, uint64_t n_reads,
                                     uint32_t k, const uint64_t *kmer_off, uint64_t *bytes) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < n_reads;
       r += warps) {
    const uint64_t m = kmers_of(ends, r, k), t0 = kmer_off[r];
    uint64_t s = 0;
    for (uint64_t j = lane; j < m; j += 32) s += index_token_len(res[t0 + j]);
    s = warp_sum(s);
    if (lane == 0) bytes[r] = s + (m ? m : 1);  // separators + '\n'
  }
}

__global__ void kmer_counts_kernel(const uint64_t *ends, uint64_t n_reads, uint32_t k,
                                   uint64_t *kmers) {
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n_reads; r += step)
    kmers[r] = kmers_of(ends, r, k);
}

__global__ void index_ascii_kernel(const uint64_t *res, const uint64_t *ends, uint64_t n_reads,
                                   uint32_t k, const uint64_t *kmer_off,
                                   const uint64_t *byte_off, uint8_t *out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < n_reads;
       r += warps) {
    const uint64_t m = kmers_of(ends, r, k), t0 = kmer_off[r];
    uint64_t at = byte_off[r];
    if (m == 0) {
      if (lane == 0) out[at] = '\n';
      continue;
    }
    for (uint64_t j0 = 0; j0 < m; j0 += 32) {
      const uint64_t j = j0 + lane;
      uint64_t v = 0;
      uint32_t n = 0;
      if (j < m) {
        v = res[t0 + j];
        n = index_token_len(v);
      }
      uint64_t total;
      const uint64_t pos = at + warp_exclusive(n ? n + 1 : 0, &total);
      if (j < m) {
        index_token(out + pos, v, n);
        out[pos + n] = j + 1 == m ? '\n' : ' ';
      }
      at += total;
    }
  }
}

__global__ void index_fixed_kernel(const uint64_t *res, const uint64_t *ends, uint64_t n_reads,
                                   uint32_t k, const uint64_t *kmer_off, int format,
                                   uint8_t *out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < n_reads;
       r += warps) {
    const uint64_t m = kmers_of(ends, r, k), t0 = kmer_off[r];
    if (format == 1) {  // binary: u64 per k-mer, then -3
      uint64_t *o = reinterpret_cast<uint64_t *>(out) + t0 + r;
      for (uint64_t j = lane; j < m; j += 32) o[j] = res[t0 + j];
      if (lane == 0) o[m] = (uint64_t)-3;
    } else {  // bool
      uint8_t *o = out + t0 + r;
      for (uint64_t j = lane; j < m; j += 32) {
        const uint64_t v = res[t0 + j];
        o[j] = v == SBWT_NOT_FOUND ? '1' : (v == SBWT_INVALID ? '2' : '0');
      }
      if (lane == 0) o[m] = '\n';
    }
  }
}

__global__ void color_lengths_kernel(const uint32_t *ids, const uint64_t *ids_off,
                                     uint64_t n_reads, uint64_t *bytes) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < n_reads;
       r += warps) {
    const uint64_t a = ids_off[r], b = ids_off[r + 1];
    uint64_t s = 0;
    for (uint64_t t = a + lane; t < b; t += 32) s += dec_len(ids[t]);
    s = warp_sum(s);
    if (lane == 0) bytes[r] = s + (b > a ? b - a : 1);
  }
}

__global__ void color_ascii_kernel(const uint32_t *ids, const uint64_t *ids_off,
                                   uint64_t n_reads, const uint64_t *byte_off, uint8_t *out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < n_reads;
       r += warps) {
    const uint64_t a = ids_off[r], b = ids_off[r + 1];
    uint64_t at = byte_off[r];
    if (b == a) {
      if (lane == 0) out[at] = '\n';
      continue;
    }
    for (uint64_t t0 = a; t0 < b; t0 += 32) {
      const uint64_t t = t0 + lane;
      uint32_t v = 0, n = 0;
      if (t < b) {
        v = ids[t];
        n = dec_len(v);
      }
      uint64_t total;
      const uint64_t pos = at + warp_exclusive(n ? n + 1 : 0, &total);
      if (t < b) {
        put_dec(out + pos, v, n);
        out[pos + n] = t + 1 == b ? '\n' : ' ';
      }
      at += total;
    }
  }
}

__global__ void color_binary_kernel(const uint32_t *ids, const uint64_t *ids_off,
                                    uint64_t n_reads, uint64_t *out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < n_reads;
       r += warps) {
    const uint64_t a = ids_off[r], b = ids_off[r + 1];
    uint64_t *o = out + a + r;
    for (uint64_t t = a + lane; t < b; t += 32) o[t - a] = ids[t];
    if (lane == 0) o[b - a] = ~0ULL;
  }
}

// csv: row r at r * 2C; '0' / ',' everywhere, then '1' at the ids.
__global__ void color_csv_kernel(const uint32_t *ids, const uint64_t *ids_off, uint64_t n_reads,
                                 uint64_t num_colors, uint8_t *out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t row = 2 * num_colors;
  for (uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; r < n_reads;
       r += warps) {
    uint8_t *o = out + r * row;
    for (uint64_t i = lane; i < row; i += 32)
      o[i] = (i & 1) ? (i + 1 == row ? '\n' : ',') : '0';
    __syncwarp();
    for (uint64_t t = ids_off[r] + lane; t < ids_off[r + 1]; t += 32) {
      const uint32_t c = ids[t];
      if (c < num_colors) o[2 * (uint64_t)c] = '1';
    }
  }
}

// Multi-block exclusive scan of u64 values in place (v[n] = total): block
// totals into tops[], one block scans tops, the last launch writes.
__device__ __forceinline__ uint64_t block_exclusive(uint64_t v, uint64_t *total) {
  __shared__ uint64_t wsum[32];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint64_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint64_t s = lane < blockDim.x / 32 ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(FULL, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    wsum[lane] = s;
  }
  __syncthreads();
  const uint64_t ex = (wid ? wsum[wid - 1] : 0) + x - v;
  *total = wsum[blockDim.x / 32 - 1];
  __syncthreads();
  return ex;
}

__global__ void __launch_bounds__(kScanThreads) scan_tops_of_kernel(const uint64_t *v, uint64_t n,
                                                                    uint64_t *tops) {
  const uint64_t b0 = blockIdx.x * (uint64_t)kScanSpan;
  uint64_t s = 0;
  for (uint32_t q = 0; q < kScanPer; ++q) {
    const uint64_t i = b0 + q * kScanThreads + threadIdx.x;
    if (i < n) s += v[i];
  }
  uint64_t total;
  block_exclusive(s, &total);
  if (threadIdx.x == 0) tops[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) scan_tops_kernel(uint64_t *tops, uint64_t nb) {
  uint64_t carry = 0;
  for (uint64_t b = 0; b < nb; b += kScanThreads) {
    const uint64_t i = b + threadIdx.x;
    const uint64_t x = i < nb ? tops[i] : 0;
    uint64_t total;
    const uint64_t ex = block_exclusive(x, &total);
    if (i < nb) tops[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) tops[nb] = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(uint64_t *v, uint64_t n,
                                                                  const uint64_t *tops) {
  const uint64_t i0 = blockIdx.x * (uint64_t)kScanSpan + (uint64_t)threadIdx.x * kScanPer;
  uint64_t c[kScanPer], s = 0;
#pragma unroll
  for (uint32_t q = 0; q < kScanPer; ++q) {
    c[q] = i0 + q < n ? v[i0 + q] : 0;
    s += c[q];
  }
  uint64_t total;
  uint64_t at = tops[blockIdx.x] + block_exclusive(s, &total);
#pragma unroll
  for (uint32_t q = 0; q < kScanPer; ++q) {
    if (i0 + q < n) v[i0 + q] = at;
    at += c[q];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) v[n] = tops[gridDim.x];
}

struct FormatWorkspace {
  DeviceBuffer kmer_off, byte_off, tops, in_a, in_b, out;
  cudaStream_t stream = nullptr;
  ~FormatWorkspace() {
    if (stream) cudaStreamDestroy(stream);
  }
};

FormatWorkspace &format_workspace(int device) {
  thread_local std::unique_ptr<FormatWorkspace> ws[16];
  if (device < 0 || device >= 16) throw Error(SBWT_E_INVALID, "device id out of range");
  auto &p = ws[device];
  if (!p) {
    p = std::make_unique<FormatWorkspace>();
    SBWT_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  }
  return *p;
}

// v[0..n) (n + 1 entries) -> exclusive offsets, v[n] = total (returned).
u64 scan_inplace(uint64_t *v, u64 n, FormatWorkspace &ws, cudaStream_t st) {
  const u64 nb = std::max<u64>((n + kScanSpan - 1) / kScanSpan, 1);
  ws.tops.ensure((nb + 1) * 8);
  uint64_t *tops = ws.tops.get<uint64_t>();
  scan_tops_of_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(v, n, tops);
  scan_tops_kernel<<<1, kScanThreads, 0, st>>>(tops, nb);
  scan_apply_kernel<<<(unsigned)nb, kScanThreads, 0, st>>>(v, n, tops);
  SBWT_CUDA(cudaGetLastError());
  u64 total = 0;
  SBWT_CUDA(cudaMemcpyAsync(&total, v + n, 8, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaStreamSynchronize(st));
  return total;
}

unsigned warp_grid(u64 items) {
  return (unsigned)std::min<u64>(std::max<u64>((items + 7) / 8, 1), 148 * 64);
}

// Device-resident index results -> formatted bytes (returns the byte count;
// SBWT_E_CAPACITY with *need set when out_cap is too small).
u64 format_index_device(const uint64_t *res, const uint64_t *ends, u64 n_reads, uint32_t k,
                        int format, uint8_t *out, u64 out_cap, u64 *need, FormatWorkspace &ws,
                        cudaStream_t st) {
  if (n_reads == 0) return 0;
  ws.kmer_off.ensure((n_reads + 1) * 8);
  uint64_t *koff = ws.kmer_off.get<uint64_t>();
  kmer_counts_kernel<<<(unsigned)std::min<u64>((n_reads + 255) / 256, 148 * 16), 256, 0, st>>>(
      ends, n_reads, k, koff);
  const u64 n_kmers = scan_inplace(koff, n_reads, ws, st);
  u64 bytes = 0;
  if (format == 0) {
    ws.byte_off.ensure((n_reads + 1) * 8);
    uint64_t *boff = ws.byte_off.get<uint64_t>();
    index_lengths_kernel<<<warp_grid(n_reads), 256, 0, st>>>(res, ends, n_reads, k, koff, boff);
    bytes = scan_inplace(boff, n_reads, ws, st);
    if (need) *need = bytes;
    if (bytes > out_cap) throw Error(SBWT_E_CAPACITY, "output capacity too small");
    index_ascii_kernel<<<warp_grid(n_reads), 256, 0, st>>>(res, ends, n_reads, k, koff, boff,
                                                            out);
  } else {
    bytes = format == 1 ? 8 * (n_kmers + n_reads) : n_kmers + n_reads;
    if (need) *need = bytes;
    if (bytes > out_cap) throw Error(SBWT_E_CAPACITY, "output capacity too small");
    index_fixed_kernel<<<warp_grid(n_reads), 256, 0, st>>>(res, ends, n_reads, k, koff, format,
                                                            out);
  }
  SBWT_CUDA(cudaGetLastError());
  return bytes;
}

u64 format_colors_device(const uint32_t *ids, const uint64_t *ids_off, u64 n_reads,
                         u64 num_colors, int format, uint8_t *out, u64 out_cap, u64 *need,
                         FormatWorkspace &ws, cudaStream_t st) {
  if (n_reads == 0) return 0;
  u64 bytes = 0;
  if (format == 0) {
    ws.byte_off.ensure((n_reads + 1) * 8);
    uint64_t *boff = ws.byte_off.get<uint64_t>();
    color_lengths_kernel<<<warp_grid(n_reads), 256, 0, st>>>(ids, ids_off, n_reads, boff);
    bytes = scan_inplace(boff, n_reads, ws, st);
    if (need) *need = bytes;
    if (bytes > out_cap) throw Error(SBWT_E_CAPACITY, "output capacity too small");
    color_ascii_kernel<<<warp_grid(n_reads), 256, 0, st>>>(ids, ids_off, n_reads, boff, out);
  } else if (format == 1) {
    u64 n_ids = 0;
    SBWT_CUDA(cudaMemcpyAsync(&n_ids, ids_off + n_reads, 8, cudaMemcpyDeviceToHost, st));
    u64 first = 0;
    SBWT_CUDA(cudaMemcpyAsync(&first, ids_off, 8, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
    if (first != 0) throw Error(SBWT_E_INVALID, "ids offsets must start at 0");
    bytes = 8 * (n_ids + n_reads);
    if (need) *need = bytes;
    if (bytes > out_cap) throw Error(SBWT_E_CAPACITY, "output capacity too small");
    color_binary_kernel<<<warp_grid(n_reads), 256, 0, st>>>(ids, ids_off, n_reads,
                                                             reinterpret_cast<uint64_t *>(out));
  } else {
    bytes = n_reads * 2 * num_colors;
    if (need) *need = bytes;
    if (bytes > out_cap) throw Error(SBWT_E_CAPACITY, "output capacity too small");
    color_csv_kernel<<<warp_grid(n_reads), 256, 0, st>>>(ids, ids_off, n_reads, num_colors, out);
  }
  SBWT_CUDA(cudaGetLastError());
  return bytes;
}

}  // namespace

}  // namespace sbwt

using namespace sbwt;

extern "C" int sbwt_format_index_results(const uint64_t *results, const uint64_t *read_ends,
                                         uint64_t n_reads, uint32_t k, int format, char *out,
                                         uint64_t out_capacity, uint64_t *out_bytes,
                                         uint32_t flags, int device, void *stream) {
  if (!out_bytes || (n_reads && !read_ends) || format < 0 || format > 2 || k == 0) {
    set_last_error("invalid argument");
    return SBWT_E_INVALID;
  }
  *out_bytes = 0;
  return guarded([&] {
    DeviceGuard g(device);
    FormatWorkspace &ws = format_workspace(device);
    const bool dev = flags & SBWT_DEVICE_POINTERS;
    cudaStream_t st = dev && stream ? (cudaStream_t)stream : ws.stream;
    if (dev) {
      if (format == 1 && ((uintptr_t)out & 7))
        throw Error(SBWT_E_INVALID, "binary output must be 8-byte aligned");
      *out_bytes = format_index_device(results, read_ends, n_reads, k, format, (uint8_t *)out,
                                       out_capacity, out_bytes, ws, st);
      SBWT_CUDA(cudaStreamSynchronize(st));
      return;
    }
    if (n_reads == 0) return;
    // host buffers: the k-mer count comes from the read ends
    u64 n_kmers = 0, prev = 0;
    for (u64 r = 0; r < n_reads; ++r) {
      if (read_ends[r] < prev) throw Error(SBWT_E_INVALID, "read ends must not decrease");
      const u64 len = read_ends[r] - prev;
      prev = read_ends[r];
      n_kmers += len >= k ? len - k + 1 : 0;
    }
    if (n_kmers && !results) throw Error(SBWT_E_INVALID, "null results");
    ws.in_a.ensure(std::max<u64>(n_kmers, 1) * 8);
    ws.in_b.ensure(n_reads * 8);
    if (n_kmers)
      SBWT_CUDA(cudaMemcpyAsync(ws.in_a.get(), results, n_kmers * 8, cudaMemcpyHostToDevice, st));
    SBWT_CUDA(cudaMemcpyAsync(ws.in_b.get(), read_ends, n_reads * 8, cudaMemcpyHostToDevice, st));
    const u64 cap = format == 0 ? n_kmers * 21 + n_reads
                                : (format == 1 ? 8 * (n_kmers + n_reads) : n_kmers + n_reads);
    ws.out.ensure(std::max<u64>(cap, 1));
    const u64 bytes = format_index_device(ws.in_a.get<uint64_t>(), ws.in_b.get<uint64_t>(),
                                          n_reads, k, format, ws.out.get<uint8_t>(), cap, nullptr,
                                          ws, st);
    *out_bytes = bytes;
    if (bytes > out_capacity) throw Error(SBWT_E_CAPACITY, "output capacity too small");
    if (!out) throw Error(SBWT_E_INVALID, "null output");
    SBWT_CUDA(cudaMemcpyAsync(out, ws.out.get(), bytes, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
  });
}

extern "C" int sbwt_format_color_results(const uint32_t *ids, const uint64_t *ids_offsets,
                                         uint64_t n_reads, uint64_t num_colors, int format,
                                         char *out, uint64_t out_capacity, uint64_t *out_bytes,
                                         uint32_t flags, int device, void *stream) {
  if (!out_bytes || (n_reads && !ids_offsets) || format < 0 || format > 2 ||
      (format == 2 && num_colors == 0)) {
    set_last_error("invalid argument");
    return SBWT_E_INVALID;
  }
  *out_bytes = 0;
  return guarded([&] {
    DeviceGuard g(device);
    FormatWorkspace &ws = format_workspace(device);
    const bool dev = flags & SBWT_DEVICE_POINTERS;
    cudaStream_t st = dev && stream ? (cudaStream_t)stream : ws.stream;
    if (dev) {
      if (format == 1 && ((uintptr_t)out & 7))
        throw Error(SBWT_E_INVALID, "binary output must be 8-byte aligned");
      *out_bytes = format_colors_device(ids, ids_offsets, n_reads, num_colors, format,
                                        (uint8_t *)out, out_capacity, out_bytes, ws, st);
      SBWT_CUDA(cudaStreamSynchronize(st));
      return;
    }
    if (n_reads == 0) return;
    if (ids_offsets[0] != 0) throw Error(SBWT_E_INVALID, "ids offsets must start at 0");
    for (u64 r = 0; r < n_reads; ++r)
      if (ids_offsets[r + 1] < ids_offsets[r])
        throw Error(SBWT_E_INVALID, "ids offsets must not decrease");
    const u64 n_ids = ids_offsets[n_reads];
    if (n_ids && !ids) throw Error(SBWT_E_INVALID, "null ids");
    ws.in_a.ensure(std::max<u64>(n_ids, 1) * 4);
    ws.in_b.ensure((n_reads + 1) * 8);
    if (n_ids)
      SBWT_CUDA(cudaMemcpyAsync(ws.in_a.get(), ids, n_ids * 4, cudaMemcpyHostToDevice, st));
    SBWT_CUDA(cudaMemcpyAsync(ws.in_b.get(), ids_offsets, (n_reads + 1) * 8,
                              cudaMemcpyHostToDevice, st));
    const u64 cap = format == 0 ? n_ids * 11 + n_reads
                                : (format == 1 ? 8 * (n_ids + n_reads) : n_reads * 2 * num_colors);
    ws.out.ensure(std::max<u64>(cap, 1));
    const u64 bytes =
        format_colors_device(ws.in_a.get<uint32_t>(), ws.in_b.get<uint64_t>(), n_reads,
                             num_colors, format, ws.out.get<uint8_t>(), cap, nullptr, ws, st);
    *out_bytes = bytes;
    if (bytes > out_capacity) throw Error(SBWT_E_CAPACITY, "output capacity too small");
    if (!out) throw Error(SBWT_E_INVALID, "null output");
    SBWT_CUDA(cudaMemcpyAsync(out, ws.out.get(), bytes, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaStreamSynchronize(st));
  });
}
