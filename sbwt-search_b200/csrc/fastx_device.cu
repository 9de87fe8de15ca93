// FASTA/FASTQ text -> concatenated sequence chars + read ends, on the GPU.
//
// Record rules are the host reader's (fastx.cpp, itself kseq's as the
// reference uses them: src/SequenceFileParser/ContinuousSequenceFileParser.cpp
// :148-156): lines end at '\n' (one trailing '\r' is dropped when a '\n'
// follows it); lines before the first header ('>' or '@') are skipped; every
// header starts one read; the lines after it are sequence up to the next
// header or a '+' line; after '+', lines are quality until their lengths reach
// the sequence length; then lines are skipped up to the next header.
//
// The per-line state (searching | sequence of n chars | quality with r chars
// still due) is sequential, so the lines are cut into chunks of kChunkLines:
//   1. newline positions (ballot per 32 bytes, per-warp counts, scan, write);
//   2. every chunk's line roles, speculatively from the "searching" state
//      (one warp per chunk, lines broadcast by shuffles), with the summaries
//      the fix-up needs: the first line that starts with '>' '@' or '+', the
//      sequence length before it, the first kPrefixLines lines, the end state;
//   3. one warp walks the chunks in order with the true entering state: a
//      chunk entered "searching" is right as it is; one entered inside a
//      sequence whose first special line is a header (or that has none) only
//      turns its leading lines into sequence lines (a per-chunk count);
//      anything else (a '+' first, or quality still due) is re-run line by
//      line until the re-run and the speculation both see a header on the same
//      line, after which both states are equal;
//   4. per-chunk chars and headers, a scan, and one warp per chunk writes the
//      chars of its sequence lines and the read ends of its headers.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "common.hpp"

namespace sbwt {

namespace {

constexpr uint32_t FULL = 0xFFFFFFFFu;
constexpr uint32_t kWarpBytes = 4096;  // text bytes per warp in the newline pass
constexpr uint32_t kChunkLines = 1024;
constexpr int kPrefixLines = 8;

enum : uint8_t { R_SKIP = 0, R_HEADER = 1, R_SEQ = 2, R_PLUS = 3, R_QUAL = 4 };
enum : uint32_t { S_SEARCH = 0, S_SEQ = 1, S_QUAL = 2 };

struct Lines {
  const uint8_t *text;
  uint64_t n_bytes;
  const uint64_t *nl;  // positions of the '\n' bytes
  uint64_t n_nl;
  uint64_t n_lines;    // n_nl, + 1 when the text does not end with '\n'
};

// Line i: its first byte, its length (without the '\r' before its '\n') and
// its first char ('\n' for an empty line).
__device__ __forceinline__ void line_at(const Lines &L, uint64_t i, uint64_t &start,
                                        uint32_t &len, uint8_t &c0) {
  start = i ? L.nl[i - 1] + 1 : 0;
  const uint64_t end = i < L.n_nl ? L.nl[i] : L.n_bytes;
  uint64_t n = end - start;
  if (i < L.n_nl && n > 0 && L.text[end - 1] == '\r') --n;
  len = (uint32_t)min(n, (uint64_t)0xFFFFFFFFu);
  c0 = n ? L.text[start] : (uint8_t)'\n';
}

// One line through the record state machine; returns its role.
__device__ __forceinline__ uint8_t step(uint32_t &mode, uint64_t &a, uint32_t len, uint8_t c0) {
  const bool hdr = len > 0 && (c0 == '>' || c0 == '@');
  if (mode == S_SEARCH) {
    if (!hdr) return R_SKIP;
    mode = S_SEQ;
    a = 0;
    return R_HEADER;
  }
  if (mode == S_SEQ) {
    if (hdr) {
      a = 0;
      return R_HEADER;
    }
    if (len > 0 && c0 == '+') {
      mode = a ? S_QUAL : S_SEARCH;  // a: the sequence length, now quality due
      return R_PLUS;
    }
    a += len;
    return R_SEQ;
  }
  a = a > len ? a - len : 0;  // quality
  if (a == 0) mode = S_SEARCH;
  return R_QUAL;
}

__device__ __forceinline__ bool is_special(uint32_t len, uint8_t c0) {
  return len > 0 && (c0 == '>' || c0 == '@' || c0 == '+');
}

struct ChunkInfo {
  uint64_t end_a;          // speculative end state
  uint64_t pre_len;        // sequence chars before the first special line
  uint64_t prefix[kPrefixLines];  // (len << 8) | c0 of the first lines
  uint32_t end_mode;
  uint32_t first_special;  // index in the chunk, n_in_chunk when none
  uint32_t n_in_chunk;
  uint32_t special_c0;     // first char of that line
  uint32_t seq_prefix;     // set by the fix-up: leading lines that are sequence
  uint32_t pad;
};

__global__ void nl_count_kernel(const uint8_t *text, uint64_t n, uint64_t *warp_counts,
                                uint64_t n_warps) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  if (w >= n_warps) return;
  const uint64_t b0 = w * kWarpBytes;
  uint64_t cnt = 0;
  for (uint32_t i = 0; i < kWarpBytes; i += 32) {
    const uint64_t p = b0 + i + lane;
    cnt += __popc(__ballot_sync(FULL, p < n && text[p] == '\n'));
  }
  if (lane == 0) warp_counts[w] = cnt;
}

__global__ void nl_write_kernel(const uint8_t *text, uint64_t n, const uint64_t *warp_off,
                                uint64_t n_warps, uint64_t *nl) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  if (w >= n_warps) return;
  const uint64_t b0 = w * kWarpBytes;
  uint64_t at = warp_off[w];
  for (uint32_t i = 0; i < kWarpBytes; i += 32) {
    const uint64_t p = b0 + i + lane;
    const bool is_nl = p < n && text[p] == '\n';
    const uint32_t m = __ballot_sync(FULL, is_nl);
    if (is_nl) nl[at + __popc(m & ((1u << lane) - 1))] = p;
    at += __popc(m);
  }
}

// In-place exclusive scan of v[0..n) by one block; v[n] = total.
__global__ void scan_small_kernel(uint64_t *v, uint64_t n) {
  __shared__ uint64_t wsum[32];
  __shared__ uint64_t carry;
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint64_t b = 0; b < n; b += blockDim.x) {
    const uint64_t i = b + threadIdx.x;
    const uint64_t x0 = i < n ? v[i] : 0;
    uint64_t x = x0;
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
    const uint64_t ex = carry + (wid ? wsum[wid - 1] : 0) + x - x0;
    if (i < n) v[i] = ex;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = ex + x0;
    __syncthreads();
  }
  if (threadIdx.x == 0) v[n] = carry;
}

// One warp per chunk: speculative roles (from "searching") + summaries.
__global__ void roles_kernel(Lines L, uint8_t *roles, ChunkInfo *ci, uint64_t n_chunks) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  if (c >= n_chunks) return;
  const uint64_t l0 = c * kChunkLines;
  const uint32_t n_in = (uint32_t)min((uint64_t)kChunkLines, L.n_lines - l0);
  uint32_t mode = S_SEARCH, first_special = n_in, special_c0 = 0;
  uint64_t a = 0, pre_len = 0;
  for (uint32_t r0 = 0; r0 < n_in; r0 += 32) {
    uint64_t start = 0;
    uint32_t len = 0;
    uint8_t c0 = '\n';
    if (r0 + lane < n_in) line_at(L, l0 + r0 + lane, start, len, c0);
    if (r0 == 0 && lane < kPrefixLines)
      ci[c].prefix[lane] = ((uint64_t)len << 8) | c0;
    // first special line and the chars before it
    if (first_special == n_in) {
      const uint32_t sp = __ballot_sync(FULL, r0 + lane < n_in && is_special(len, c0));
      const uint32_t upto = sp ? (1u << (__ffs(sp) - 1)) - 1 : FULL;
      uint64_t part = (upto >> lane) & 1u ? len : 0;
      for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(FULL, part, o);
      pre_len += part;
      if (sp) {
        first_special = r0 + __ffs(sp) - 1;
        special_c0 = __shfl_sync(FULL, (uint32_t)c0, __ffs(sp) - 1);
      }
    }
    uint8_t my_role = R_SKIP;
    const uint32_t m = min(32u, n_in - r0);
    for (uint32_t q = 0; q < m; ++q) {
      const uint32_t lq = __shfl_sync(FULL, len, q);
      const uint8_t cq = (uint8_t)__shfl_sync(FULL, (uint32_t)c0, q);
      const uint8_t role = step(mode, a, lq, cq);
      if (lane == q) my_role = role;
    }
    if (r0 + lane < n_in) roles[l0 + r0 + lane] = my_role;
  }
  if (lane == 0) {
    ci[c].end_a = a;
    ci[c].end_mode = mode;
    ci[c].pre_len = pre_len;
    ci[c].first_special = first_special;
    ci[c].special_c0 = special_c0;
    ci[c].n_in_chunk = n_in;
    ci[c].seq_prefix = 0;
  }
}

// Re-runs chunk c line by line from the true entering state until the re-run
// and the speculation both see a header on the same line (then their states
// are equal and the speculative end state holds); corrects the roles on the
// way.  All lanes compute the same; lane 0 writes.  Returns the lines run.
__device__ uint32_t rerun_chunk(const Lines &L, uint8_t *roles, const ChunkInfo &k, uint64_t c,
                                uint32_t &mode, uint64_t &a, uint32_t lane) {
  const uint64_t l0 = c * kChunkLines;
  for (uint32_t j = 0; j < k.n_in_chunk; ++j) {
    uint32_t len;
    uint8_t c0;
    if (j < kPrefixLines) {
      const uint64_t e = k.prefix[j];
      len = (uint32_t)(e >> 8);
      c0 = (uint8_t)e;
    } else {
      uint64_t start;
      line_at(L, l0 + j, start, len, c0);
    }
    const uint8_t role = step(mode, a, len, c0);
    const uint8_t spec = roles[l0 + j];
    if (role == R_HEADER && spec == R_HEADER) {
      mode = k.end_mode;
      a = k.end_a;
      return j + 1;
    }
    __syncwarp();
    if (lane == 0 && role != spec) roles[l0 + j] = role;
    __syncwarp();
  }
  return k.n_in_chunk;
}

// One warp walks the chunks in order with the true entering state; lanes
// fetch the summaries of 32 chunks at a time, the state steps through them by
// shuffles.  stats[0] = lines re-run one by one.
__global__ void fixup_kernel(Lines L, uint8_t *roles, ChunkInfo *ci, uint64_t n_chunks,
                             uint64_t *stats) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t mode = S_SEARCH;
  uint64_t a = 0, rerun = 0;
  for (uint64_t c0 = 0; c0 < n_chunks; c0 += 32) {
    const uint64_t c = c0 + lane;
    uint32_t em = 0, fs = 0, nin = 0, sc = 0;
    uint64_t ea = 0, pl = 0;
    if (c < n_chunks) {
      em = ci[c].end_mode;
      ea = ci[c].end_a;
      fs = ci[c].first_special;
      nin = ci[c].n_in_chunk;
      sc = ci[c].special_c0;
      pl = ci[c].pre_len;
    }
    const uint32_t m = (uint32_t)min((uint64_t)32, n_chunks - c0);
    for (uint32_t q = 0; q < m; ++q) {
      const uint32_t q_em = __shfl_sync(FULL, em, q), q_fs = __shfl_sync(FULL, fs, q);
      const uint32_t q_nin = __shfl_sync(FULL, nin, q), q_sc = __shfl_sync(FULL, sc, q);
      const uint64_t q_ea = __shfl_sync(FULL, ea, q), q_pl = __shfl_sync(FULL, pl, q);
      if (mode == S_SEARCH) {  // the speculation was right
        mode = q_em;
        a = q_ea;
      } else if (mode == S_SEQ && (q_fs == q_nin || q_sc != '+')) {
        // the leading lines continue the open sequence, then as speculated
        if (lane == 0) ci[c0 + q].seq_prefix = q_fs;
        if (q_fs == q_nin) {
          a += q_pl;
        } else {
          mode = q_em;
          a = q_ea;
        }
      } else {
        rerun += rerun_chunk(L, roles, ci[c0 + q], c0 + q, mode, a, lane);
      }
    }
  }
  if (lane == 0) stats[0] = rerun;
}

__device__ __forceinline__ uint8_t final_role(const uint8_t *roles, const ChunkInfo &k,
                                              uint64_t l0, uint32_t j) {
  return j < k.seq_prefix ? R_SEQ : roles[l0 + j];
}

// Per chunk: sequence chars -> tot[c], headers -> tot[n_chunks + 1 + c].
__global__ void chunk_totals_kernel(Lines L, const uint8_t *roles, const ChunkInfo *ci,
                                    uint64_t n_chunks, uint64_t *chars_tot,
                                    uint64_t *hdr_tot) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  if (c >= n_chunks) return;
  const ChunkInfo &k = ci[c];
  const uint64_t l0 = c * kChunkLines;
  uint64_t chars = 0, hdrs = 0;
  for (uint32_t j = lane; j < k.n_in_chunk; j += 32) {
    const uint8_t role = final_role(roles, k, l0, j);
    if (role == R_SEQ) {
      uint64_t start;
      uint32_t len;
      uint8_t c0;
      line_at(L, l0 + j, start, len, c0);
      chars += len;
    }
    hdrs += role == R_HEADER;
  }
  for (int o = 16; o; o >>= 1) {
    chars += __shfl_xor_sync(FULL, chars, o);
    hdrs += __shfl_xor_sync(FULL, hdrs, o);
  }
  if (lane == 0) {
    chars_tot[c] = chars;
    hdr_tot[c] = hdrs;
  }
}

// One warp per chunk: sequence chars to out at their offsets; for the read
// opened by header h > 0, the end of read h - 1.
__global__ void emit_kernel(Lines L, const uint8_t *roles, const ChunkInfo *ci,
                            uint64_t n_chunks, const uint64_t *chars_off,
                            const uint64_t *hdr_off, uint8_t *out, uint64_t *ends) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  if (c >= n_chunks) return;
  const ChunkInfo &k = ci[c];
  const uint64_t l0 = c * kChunkLines;
  uint64_t at = chars_off[c], h = hdr_off[c];
  for (uint32_t r0 = 0; r0 < k.n_in_chunk; r0 += 32) {
    const uint32_t j = r0 + lane;
    uint8_t role = R_SKIP;
    uint64_t start = 0;
    uint32_t len = 0;
    uint8_t c0;
    if (j < k.n_in_chunk) {
      role = final_role(roles, k, l0, j);
      line_at(L, l0 + j, start, len, c0);
    }
    const uint64_t my_chars = role == R_SEQ ? len : 0;
    uint64_t x = my_chars;
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(FULL, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    const uint64_t my_at = at + x - my_chars;
    const uint32_t hm = __ballot_sync(FULL, role == R_HEADER);
    const uint64_t my_h = h + __popc(hm & ((1u << lane) - 1));
    if (role == R_HEADER && my_h > 0) ends[my_h - 1] = my_at;
    const uint32_t sm = __ballot_sync(FULL, role == R_SEQ && len > 0);
    for (uint32_t m = sm; m; m &= m - 1) {
      const int q = __ffs(m) - 1;
      const uint64_t s = __shfl_sync(FULL, start, q);
      const uint64_t d = __shfl_sync(FULL, my_at, q);
      const uint32_t n = __shfl_sync(FULL, len, q);
      for (uint32_t i = lane; i < n; i += 32) out[d + i] = L.text[s + i];
    }
    at = __shfl_sync(FULL, my_at + my_chars, 31);
    h += __popc(hm);
  }
}

__global__ void set_u64_kernel(uint64_t *p, const uint64_t *value) { *p = *value; }

struct FastxWorkspace {
  DeviceBuffer text, warp_counts, nl, roles, chunks, chars_tot, hdr_tot, stats, chars, ends;
  cudaStream_t stream = nullptr;
  ~FastxWorkspace() {
    if (stream) cudaStreamDestroy(stream);
  }
};

FastxWorkspace &fastx_workspace(int device) {
  thread_local std::unique_ptr<FastxWorkspace> ws[16];
  if (device < 0 || device >= 16) throw Error(SBWT_E_INVALID, "device id out of range");
  auto &p = ws[device];
  if (!p) {
    p = std::make_unique<FastxWorkspace>();
    SBWT_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  }
  return *p;
}

unsigned grid_for_warps(uint64_t warps) {
  return (unsigned)std::max<uint64_t>((warps + 7) / 8, 1);  // 256 threads per block
}

}  // namespace

// Device-resident text through newline positions, roles, the fix-up and the
// per-chunk totals (fastx_count), then the chars and read ends (fastx_emit).
struct ParsePlan {
  Lines L{};
  u64 n_chunks = 0, n_chars = 0, n_reads = 0, rerun = 0;
};

ParsePlan fastx_count(const uint8_t *d_text, u64 n_bytes, cudaStream_t st, FastxWorkspace &ws) {
  ParsePlan P;
  if (n_bytes == 0) return P;
  const u64 n_warps = (n_bytes + kWarpBytes - 1) / kWarpBytes;
  ws.warp_counts.ensure((n_warps + 1) * 8);
  u64 *wc = ws.warp_counts.get<u64>();
  nl_count_kernel<<<grid_for_warps(n_warps), 256, 0, st>>>(d_text, n_bytes, wc, n_warps);
  scan_small_kernel<<<1, 1024, 0, st>>>(wc, n_warps);
  SBWT_CUDA(cudaGetLastError());
  u64 n_nl = 0;
  uint8_t last = 0;
  SBWT_CUDA(cudaMemcpyAsync(&n_nl, wc + n_warps, 8, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaMemcpyAsync(&last, d_text + n_bytes - 1, 1, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaStreamSynchronize(st));
  ws.nl.ensure(std::max<u64>(n_nl, 1) * 8);
  nl_write_kernel<<<grid_for_warps(n_warps), 256, 0, st>>>(d_text, n_bytes, wc, n_warps,
                                                            ws.nl.get<u64>());
  P.L = Lines{d_text, n_bytes, ws.nl.get<u64>(), n_nl, n_nl + (last != '\n' ? 1 : 0)};
  P.n_chunks = (P.L.n_lines + kChunkLines - 1) / kChunkLines;
  ws.roles.ensure(std::max<u64>(P.L.n_lines, 1));
  ws.chunks.ensure(std::max<u64>(P.n_chunks, 1) * sizeof(ChunkInfo));
  ws.chars_tot.ensure((P.n_chunks + 1) * 8);
  ws.hdr_tot.ensure((P.n_chunks + 1) * 8);
  ws.stats.ensure(8);
  uint8_t *roles = ws.roles.get<uint8_t>();
  ChunkInfo *ci = ws.chunks.get<ChunkInfo>();
  u64 *ct = ws.chars_tot.get<u64>(), *ht = ws.hdr_tot.get<u64>();
  roles_kernel<<<grid_for_warps(P.n_chunks), 256, 0, st>>>(P.L, roles, ci, P.n_chunks);
  fixup_kernel<<<1, 32, 0, st>>>(P.L, roles, ci, P.n_chunks, ws.stats.get<u64>());
  chunk_totals_kernel<<<grid_for_warps(P.n_chunks), 256, 0, st>>>(P.L, roles, ci, P.n_chunks,
                                                                    ct, ht);
  scan_small_kernel<<<1, 1024, 0, st>>>(ct, P.n_chunks);
  scan_small_kernel<<<1, 1024, 0, st>>>(ht, P.n_chunks);
  SBWT_CUDA(cudaGetLastError());
  u64 tot[3] = {0, 0, 0};
  SBWT_CUDA(cudaMemcpyAsync(&tot[0], ct + P.n_chunks, 8, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaMemcpyAsync(&tot[1], ht + P.n_chunks, 8, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaMemcpyAsync(&tot[2], ws.stats.get(), 8, cudaMemcpyDeviceToHost, st));
  SBWT_CUDA(cudaStreamSynchronize(st));
  P.n_chars = tot[0];
  P.n_reads = tot[1];
  P.rerun = tot[2];
  return P;
}

void fastx_emit(const ParsePlan &P, uint8_t *d_chars, u64 *d_ends, cudaStream_t st,
                FastxWorkspace &ws) {
  if (P.n_chunks == 0) return;
  u64 *ct = ws.chars_tot.get<u64>(), *ht = ws.hdr_tot.get<u64>();
  emit_kernel<<<grid_for_warps(P.n_chunks), 256, 0, st>>>(
      P.L, ws.roles.get<uint8_t>(), ws.chunks.get<ChunkInfo>(), P.n_chunks, ct, ht, d_chars,
      d_ends);
  if (P.n_reads) set_u64_kernel<<<1, 1, 0, st>>>(d_ends + P.n_reads - 1, ct + P.n_chunks);
  SBWT_CUDA(cudaGetLastError());
}

}  // namespace sbwt

using namespace sbwt;

extern "C" int sbwt_fastx_parse(const char *text, uint64_t n_bytes, char *chars,
                                uint64_t chars_capacity, uint64_t *read_ends,
                                uint64_t ends_capacity, uint64_t *n_chars, uint64_t *n_reads,
                                uint32_t flags, int device, void *stream) {
  if (!n_chars || !n_reads || (n_bytes && !text)) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    DeviceGuard g(device);
    FastxWorkspace &ws = fastx_workspace(device);
    const bool dev = flags & SBWT_DEVICE_POINTERS;
    cudaStream_t st = dev && stream ? (cudaStream_t)stream : ws.stream;
    const uint8_t *d_text = (const uint8_t *)text;
    if (!dev) {
      ws.text.ensure(std::max<u64>(n_bytes, 1));
      if (n_bytes)
        SBWT_CUDA(cudaMemcpyAsync(ws.text.get(), text, n_bytes, cudaMemcpyHostToDevice, st));
      d_text = ws.text.get<uint8_t>();
    }
    const ParsePlan P = fastx_count(d_text, n_bytes, st, ws);
    *n_chars = P.n_chars;
    *n_reads = P.n_reads;
    if (P.n_chars > chars_capacity || P.n_reads > ends_capacity)
      throw Error(SBWT_E_CAPACITY, "chars or read ends capacity too small");
    if ((P.n_chars && !chars) || (P.n_reads && !read_ends))
      throw Error(SBWT_E_INVALID, "null output buffer");
    if (dev) {
      fastx_emit(P, (uint8_t *)chars, read_ends, st, ws);
    } else {
      ws.chars.ensure(std::max<u64>(P.n_chars, 1));
      ws.ends.ensure(std::max<u64>(P.n_reads, 1) * 8);
      fastx_emit(P, ws.chars.get<uint8_t>(), ws.ends.get<u64>(), st, ws);
      if (P.n_chars)
        SBWT_CUDA(cudaMemcpyAsync(chars, ws.chars.get(), P.n_chars, cudaMemcpyDeviceToHost, st));
      if (P.n_reads)
        SBWT_CUDA(cudaMemcpyAsync(read_ends, ws.ends.get(), P.n_reads * 8,
                                  cudaMemcpyDeviceToHost, st));
    }
    SBWT_CUDA(cudaStreamSynchronize(st));
  });
}
