#include <algorithm>
#include <charconv>
#include <cstring>
#include <fstream>
#include <emmintrin.h>
#include <unistd.h>

#include <atomic>
#include <stdexcept>

#include "../../include/sbwt_b200.h"
#include "host_io.hpp"
#include "host_threads.hpp"

namespace sbwt {

namespace {

FILE *open_out(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("Unable to open file for writing " + path);
  std::setvbuf(f, nullptr, _IOFBF, 1 << 22);
  return f;
}

void put_string(FILE *f, const std::string &s) {  // length-prefixed
  const u64 n = s.size();
  std::fwrite(&n, 8, 1, f);
  std::fwrite(s.data(), 1, n, f);
}

void flush_buf(FILE *f, std::vector<char> &b) {
  if (!b.empty() && std::fwrite(b.data(), 1, b.size(), f) != b.size())
    throw std::runtime_error("write failed");
  b.clear();
}

inline void put_u64(std::vector<char> &b, u64 v) {
  char tmp[8];
  std::memcpy(tmp, &v, 8);
  b.insert(b.end(), tmp, tmp + 8);
}

inline void put_dec(std::vector<char> &b, u64 v) {
  char tmp[24];
  auto r = std::to_chars(tmp, tmp + sizeof(tmp), v);
  b.insert(b.end(), tmp, r.ptr);
}

}  // namespace

IndexResultsWriter::IndexResultsWriter(const std::string &prefix, IndexFormat fmt,
                                       bool headers)
    : fmt_(fmt) {
  const char *ext = fmt == IndexFormat::Ascii ? ".txt" : fmt == IndexFormat::Binary ? ".bin" : ".bool";
  f_ = open_out(prefix + ext);
  if (headers) {
    put_string(f_, fmt == IndexFormat::Ascii ? "ascii" : fmt == IndexFormat::Binary ? "binary" : "bool");
    put_string(f_, fmt == IndexFormat::Bool ? "v2.0" : "v1.0");
  }
}

IndexResultsWriter::~IndexResultsWriter() {
  if (f_) {
    flush_buf(f_, buf_);
    std::fclose(f_);
  }
}

void IndexResultsWriter::write(const u64 *res, const u64 *ends, u64 n_reads, u32 k) {
  u64 prev = 0, t = 0;
  for (u64 r = 0; r < n_reads; ++r) {
    const u64 len = ends[r] - prev;
    prev = ends[r];
    const u64 m = len >= k ? len - k + 1 : 0;
    for (u64 j = 0; j < m; ++j, ++t) {
      const u64 v = res[t];
      switch (fmt_) {
        case IndexFormat::Ascii:
          if (j) buf_.push_back(' ');
          if (v == SBWT_NOT_FOUND) {
            buf_.push_back('-');
            buf_.push_back('1');
          } else if (v == SBWT_INVALID) {
            buf_.push_back('-');
            buf_.push_back('2');
          } else {
            put_dec(buf_, v);
          }
          break;
        case IndexFormat::Binary:
          put_u64(buf_, v);  // -1 and -2 are the same bit patterns
          break;
        case IndexFormat::Bool:
          buf_.push_back(v == SBWT_NOT_FOUND ? '1' : (v == SBWT_INVALID ? '2' : '0'));
          break;
      }
    }
    if (fmt_ == IndexFormat::Binary)
      put_u64(buf_, (u64)-3);
    else
      buf_.push_back('\n');
    if (buf_.size() > (1u << 22)) flush_buf(f_, buf_);
  }
  flush_buf(f_, buf_);
}

void IndexResultsWriter::write_raw(const char *bytes, u64 n) {
  flush_buf(f_, buf_);
  if (n && std::fwrite(bytes, 1, n, f_) != n) throw std::runtime_error("write failed");
}

ColorResultsWriter::ColorResultsWriter(const std::string &prefix, ColorFormat fmt,
                                       bool headers, u64 num_colors)
    : fmt_(fmt), num_colors_(num_colors) {
  const char *ext = fmt == ColorFormat::Ascii ? ".txt" : fmt == ColorFormat::Binary ? ".bin" : ".csv";
  f_ = open_out(prefix + ext);
  if (fmt == ColorFormat::Csv) {  // the csv header row is always written
    for (u64 i = 1; i <= num_colors; ++i) {
      put_dec(buf_, i);
      buf_.push_back(i == num_colors ? '\n' : ',');
    }
    flush_buf(f_, buf_);
  } else if (headers) {
    put_string(f_, fmt == ColorFormat::Ascii ? "ascii" : "binary");
    put_string(f_, "v1.0");
  }
}

ColorResultsWriter::~ColorResultsWriter() {
  if (f_) {
    flush_buf(f_, buf_);
    std::fclose(f_);
  }
}

void ColorResultsWriter::write(const uint32_t *ids, const u64 *offs, u64 n_reads) {
  std::vector<char> row;
  if (fmt_ == ColorFormat::Csv) {
    row.resize(num_colors_ * 2);
    for (u64 i = 0; i < num_colors_; ++i) {
      row[2 * i] = '0';
      row[2 * i + 1] = (i + 1 == num_colors_) ? '\n' : ',';
    }
  }
  for (u64 r = 0; r < n_reads; ++r) {
    switch (fmt_) {
      case ColorFormat::Ascii:
        for (u64 t = offs[r]; t < offs[r + 1]; ++t) {
          if (t != offs[r]) buf_.push_back(' ');
          put_dec(buf_, ids[t]);
        }
        buf_.push_back('\n');
        break;
      case ColorFormat::Binary:
        for (u64 t = offs[r]; t < offs[r + 1]; ++t) put_u64(buf_, ids[t]);
        put_u64(buf_, (u64)-1);
        break;
      case ColorFormat::Csv: {
        const size_t at = buf_.size();
        buf_.insert(buf_.end(), row.begin(), row.end());
        for (u64 t = offs[r]; t < offs[r + 1]; ++t) buf_[at + 2 * (u64)ids[t]] = '1';
        break;
      }
    }
    if (buf_.size() > (1u << 22)) flush_buf(f_, buf_);
  }
  flush_buf(f_, buf_);
}

void ColorResultsWriter::write_raw(const char *bytes, u64 n) {
  flush_buf(f_, buf_);
  if (n && std::fwrite(bytes, 1, n, f_) != n) throw std::runtime_error("write failed");
}

// Length (0..8) of the run of decimal digits at the start of the 8 bytes x
// (first char in the low byte).  Per byte, without carries between bytes:
// the byte's low 7 bits compared with '0' and ':' by adding to the high
// bit, and the high bit itself clear.
static inline unsigned digit_run8(u64 x) {
  constexpr u64 kHigh = 0x8080808080808080ULL, kLow7 = 0x7F7F7F7F7F7F7F7FULL;
  const u64 low = x & kLow7;
  const u64 ge0 = (low + 0x5050505050505050ULL) & kHigh;    // low >= 0x30
  const u64 gt9 = (low + 0x4646464646464646ULL) & kHigh;    // low >= 0x3A
  const u64 digit = ge0 & ~gt9 & ~x & kHigh;
  const u64 other = ~digit & kHigh;
  return other ? (unsigned)__builtin_ctzll(other) / 8 : 8u;
}

// Value of the first len (0..8) digit chars of x: the digits moved to the
// top bytes (zeros below are leading zeros), then pairs, quads and the
// eight combined by multiply-and-shift (the published SWAR eight-digit
// conversion).
static inline u64 digits_value8(u64 x, unsigned len) {
  u64 d = (x & 0x0F0F0F0F0F0F0F0FULL) << ((8 * (8 - len)) & 63);
  d = (d * 10 + (d >> 8)) & 0x00FF00FF00FF00FFULL;
  d = (d * 100 + (d >> 16)) & 0x0000FFFF0000FFFFULL;
  d = (d * 10000 + (d >> 32)) & 0x00000000FFFFFFFFULL;
  return len ? d : 0;
}

// The decimal number whose digits start at data[i] (i < b), modulo 2^64;
// i moves past its digits.  Up to 8 digits from one 8-byte load, the rest
// one by one.  (Two loads for up to 16 digits without a branch on the
// length were slower on the index workload's 8-9 digit numbers.)
static inline u64 parse_digits(const char *data, size_t &i, size_t b) {
  u64 v = 0;
  if (i + 8 <= b) {
    u64 x;
    std::memcpy(&x, data + i, 8);
    const unsigned len = digit_run8(x);
    v = digits_value8(x, len);
    i += len;
  }
  while (i < b && data[i] >= '0' && data[i] <= '9') v = v * 10 + (u64)(data[i++] - '0');
  return v;
}

// The ascii body of an index results file, bytes [a, b) (whole lines, or the
// file's unterminated tail), token by token: value(v) for a found index,
// nf() / inv() for a -1 / -2, end() at each read's end ('\n', and an
// unterminated tail with tokens is one more read).
template <class V, class NF, class INV, class END>
static void scan_ascii(const char *data, size_t a, size_t b, V &&value, NF &&nf, INV &&inv,
                       END &&end) {
  bool open_read = false;
  size_t i = a;
  while (i < b) {
    const char c = data[i];
    if (c == '\n') {
      end();
      open_read = false;
      ++i;
    } else if (c == '-') {  // -1 / -2 (other negatives are skipped)
      if (i + 1 < b && data[i + 1] == '1') nf();
      else if (i + 1 < b && data[i + 1] == '2') inv();
      ++i;
      while (i < b && data[i] >= '0') ++i;
      open_read = true;
    } else if (c >= '0' && c <= '9') {
      value(parse_digits(data, i, b));
      open_read = true;
    } else {
      ++i;
    }
  }
  if (open_read) end();  // only the file's last part can end inside a read
}

// Bytes [i, i + 64) of an ascii body that ends at b, one bit per byte and
// class (bytes at b and past it read as spaces); bad = none of digit,
// space, newline, '-'.
struct Block64 {
  u64 digit, sep, nl, minus, one, two, bad;
};
static inline Block64 classify64(const char *data, size_t i, size_t b) {
  alignas(16) char tmp[64];
  const char *p = data + i;
  if (b - i < 64) {
    std::memcpy(tmp, p, b - i);
    std::memset(tmp + (b - i), ' ', 64 - (b - i));
    p = tmp;
  }
  const __m128i k0 = _mm_set1_epi8('0'), k9 = _mm_set1_epi8(9), ksp = _mm_set1_epi8(' '),
                knl = _mm_set1_epi8('\n'), kmi = _mm_set1_epi8('-'), k1 = _mm_set1_epi8('1'),
                k2 = _mm_set1_epi8('2');
  Block64 c{0, 0, 0, 0, 0, 0, 0};
  for (int q = 0; q < 4; ++q) {
    const __m128i x = _mm_loadu_si128(reinterpret_cast<const __m128i *>(p + 16 * q));
    const __m128i d = _mm_sub_epi8(x, k0);
    auto bits = [q](__m128i m) { return (u64)(unsigned)_mm_movemask_epi8(m) << (16 * q); };
    const __m128i nl = _mm_cmpeq_epi8(x, knl);
    c.digit |= bits(_mm_cmpeq_epi8(_mm_min_epu8(d, k9), d));  // x - '0' <= 9 unsigned
    c.nl |= bits(nl);
    c.sep |= bits(_mm_or_si128(_mm_cmpeq_epi8(x, ksp), nl));
    c.minus |= bits(_mm_cmpeq_epi8(x, kmi));
    c.one |= bits(_mm_cmpeq_epi8(x, k1));
    c.two |= bits(_mm_cmpeq_epi8(x, k2));
  }
  c.bad = ~(c.digit | c.sep | c.minus);
  return c;
}

// Whether a read is open (a token since the last newline) after block c.
static inline bool open_after(const Block64 &c, bool open) {
  const u64 tok = c.digit | c.minus;
  if (!c.nl) return open || tok != 0;
  const int last = 63 - __builtin_clzll(c.nl);
  return last < 63 && (tok >> (last + 1)) != 0;
}

// On a body of digits, spaces, newlines and '-' only, scan_ascii's tokens
// follow from byte classes 64 bytes at a time: a number starts at a digit
// after a space or newline (or at a, a line start), -1 / -2 are a '-'
// followed by '1' / '2' (its digits never start a number), a read ends at
// each newline and at b when a token came after the last one.
// count_plain_ascii gives scan_ascii's counts of values and reads, or false
// (counts unset) when [a, b) holds another byte; scan_plain_ascii then makes
// scan_ascii's calls in the same order.
static bool count_plain_ascii(const char *data, size_t a, size_t b, u64 &values, u64 &reads) {
  u64 nv = 0, nr = 0, carry = 1;
  bool open = false;
  for (size_t i = a; i < b; i += 64) {
    const Block64 c = classify64(data, i, b);
    if (c.bad) return false;
    nv += (u64)__builtin_popcountll(c.digit & ((c.sep << 1) | carry));
    carry = c.sep >> 63;
    nr += (u64)__builtin_popcountll(c.nl);
    open = open_after(c, open);
  }
  values = nv;
  reads = nr + (open ? 1 : 0);
  return true;
}

template <class V, class NF, class INV, class END>
static void scan_plain_ascii(const char *data, size_t a, size_t b, V &&value, NF &&nf, INV &&inv,
                             END &&end) {
  u64 carry = 1;
  bool open = false;
  for (size_t i = a; i < b; i += 64) {
    const Block64 c = classify64(data, i, b);
    const u64 start = c.digit & ((c.sep << 1) | carry);
    carry = c.sep >> 63;
    const char next = i + 64 < b ? data[i + 64] : ' ';  // the byte after the block
    const u64 m1 = c.minus & ((c.one >> 1) | (next == '1' ? 1ULL << 63 : 0));
    const u64 m2 = c.minus & ((c.two >> 1) | (next == '2' ? 1ULL << 63 : 0));
    for (u64 ev = start | c.nl | m1 | m2; ev; ev &= ev - 1) {
      const int bit = __builtin_ctzll(ev);
      const u64 mb = 1ULL << bit;
      if (start & mb) {
        size_t j = i + (size_t)bit;
        value(parse_digits(data, j, b));
      } else if (c.nl & mb) {
        end();
      } else if (m1 & mb) {
        nf();
      } else {
        inv();
      }
    }
    open = open_after(c, open);
  }
  if (open) end();
}

// The binary body of an index results file, words [a, b) (whole reads, or
// the file's unterminated tail), with the callbacks of scan_ascii: a read
// ends at each -3 word, -1 / -2 are not-found / invalid.
template <class V, class NF, class INV, class END>
static void scan_binary(const char *data, size_t a, size_t b, V &&value, NF &&nf, INV &&inv,
                        END &&end) {
  bool open_read = false;
  for (size_t w = a; w < b; ++w) {
    u64 v;
    std::memcpy(&v, data + 8 * w, 8);
    if (v == (u64)-3) {
      end();
      open_read = false;
      continue;
    }
    if (v == (u64)-1) nf();
    else if (v == (u64)-2) inv();
    else value(v);
    open_read = true;
  }
  if (open_read) end();  // only the file's last part can end inside a read
}

// Output arrays of read_index_results_into: found values, n_reads + 1
// offsets, per-read not-found and invalid counts.
struct ResultArrays {
  u64 *found, *offsets, *not_found, *invalid;
};

// Reads an index results file; alloc(total_found, total_reads) provides the
// output arrays once their sizes are known (between the counting and the
// writing pass), so callers choose their own storage.
template <class Alloc>
static void read_index_results_into(const std::string &path, Alloc &&alloc) {
  FILE *in = std::fopen(path.c_str(), "rb");
  if (!in) throw std::runtime_error("Unable to open file " + path);
  std::unique_ptr<FILE, int (*)(FILE *)> closer(in, std::fclose);
  auto get_str = [&]() {
    u64 n = 0;
    if (std::fread(&n, 8, 1, in) != 1 || n > 64)
      throw std::runtime_error("The file has an incompatible format");
    std::string s(n, '\0');
    if (n && std::fread(s.data(), 1, n, in) != n)
      throw std::runtime_error("The file has an incompatible format");
    return s;
  };
  const std::string fmt = get_str();
  if (fmt != "ascii" && fmt != "binary")
    throw std::runtime_error("Unknown index file format '" + fmt + "'");
  if (get_str() != "v1.0") throw std::runtime_error("The file has an incompatible version number");
  // the body in one read (its size from the file's end), not cleared first
  const long body = std::ftell(in);
  std::fseek(in, 0, SEEK_END);
  const long end_pos = std::ftell(in);
  std::fseek(in, body, SEEK_SET);
  const size_t nbody = end_pos > body ? (size_t)(end_pos - body) : 0;
  std::unique_ptr<char[]> buf(new char[std::max<size_t>(nbody, 1)]);
  {  // in pieces of 64 MiB on host threads (the page-cache copies and the
     // buffer's first touches run in parallel)
    const int fd = fileno(in);
    const size_t piece = 64ULL << 20, n_pieces = (nbody + piece - 1) / piece;
    std::atomic<size_t> next{0};
    std::atomic<bool> failed{false};
    run_threads(host_threads(n_pieces, 1, 16), [&](size_t) {
      for (size_t p; (p = next.fetch_add(1)) < n_pieces;) {
        const size_t off = p * piece, len = std::min(piece, nbody - off);
        size_t got = 0;
        while (got < len) {
          const ssize_t r = ::pread(fd, buf.get() + off + got, len - got, body + (off_t)(off + got));
          if (r <= 0) {
            failed = true;
            return;
          }
          got += (size_t)r;
        }
      }
    });
    if (failed) throw std::runtime_error("read error in index results file");
  }
  const char *data = buf.get();
  // Parts of whole reads on host threads (cut just past a newline, or a -3
  // word): one pass counts each part's reads and found values, the second
  // writes them straight to their places in the output.
  const bool ascii = fmt == "ascii";
  const size_t n = ascii ? nbody : nbody / 8;  // bytes or words (a partial word is ignored)
  auto word = [&](size_t w) {
    u64 v;
    std::memcpy(&v, data + 8 * w, 8);
    return v;
  };
  auto scan = [&](size_t a, size_t b, auto &&value, auto &&nf, auto &&inv, auto &&end) {
    if (ascii) scan_ascii(data, a, b, value, nf, inv, end);
    else scan_binary(data, a, b, value, nf, inv, end);
  };
  const size_t T = host_threads(nbody, 1 << 22, 32);
  std::vector<size_t> cut(T + 1, n);
  cut[0] = 0;
  for (size_t t = 1; t < T; ++t) {  // just past a read's end at or after n * t / T
    size_t c = std::max(cut[t - 1], n * t / T);
    if (ascii)
      while (c < n && data[c] != '\n') ++c;
    else
      while (c < n && word(c) != (u64)-3) ++c;
    cut[t] = c < n ? c + 1 : n;
  }
  std::vector<u64> part_found(T + 1, 0), part_reads(T + 1, 0);
  auto run = [&](auto &&work) { run_threads(T, work); };
  std::vector<char> plain(T, 0);  // part t holds only digits, spaces, newlines, '-'
  run([&](size_t t) {
    u64 nv = 0, nr = 0;
    if (ascii && count_plain_ascii(data, cut[t], cut[t + 1], nv, nr))
      plain[t] = 1;
    else
      scan(cut[t], cut[t + 1], [&](u64) { ++nv; }, [] {}, [] {}, [&] { ++nr; });
    part_found[t] = nv;
    part_reads[t] = nr;
  });
  u64 total_found = 0, total_reads = 0;
  for (size_t t = 0; t < T; ++t) {  // exclusive prefix sums
    const u64 f = part_found[t], r = part_reads[t];
    part_found[t] = total_found;
    part_reads[t] = total_reads;
    total_found += f;
    total_reads += r;
  }
  const ResultArrays out = alloc(total_found, total_reads);
  out.offsets[0] = 0;
  run([&](size_t t) {
    u64 fv = part_found[t], r = part_reads[t], pnf = 0, pinv = 0;
    u64 *found = out.found, *offs = out.offsets;
    u64 *onf = out.not_found, *oinv = out.invalid;
    auto value = [&](u64 v) { found[fv++] = v; };
    auto nf = [&] { ++pnf; };
    auto inv = [&] { ++pinv; };
    auto end = [&] {
      offs[r + 1] = fv;
      onf[r] = pnf;
      oinv[r] = pinv;
      ++r;
      pnf = pinv = 0;
    };
    if (plain[t])
      scan_plain_ascii(data, cut[t], cut[t + 1], value, nf, inv, end);
    else
      scan(cut[t], cut[t + 1], value, nf, inv, end);
  });
}

IndexResults read_index_results(const std::string &path) {
  IndexResults out;
  read_index_results_into(path, [&](u64 n_found, u64 n_reads) {
    out.found.resize(n_found);
    out.offsets.resize(n_reads + 1);
    out.not_found.resize(n_reads);
    out.invalid.resize(n_reads);
    return ResultArrays{out.found.data(), out.offsets.data(), out.not_found.data(),
                        out.invalid.data()};
  });
  return out;
}

}  // namespace sbwt

// ---------------------------------------------------------------------------
// C ABI of the host I/O (no GPU involved)
// ---------------------------------------------------------------------------
#include <cstdlib>
#include <memory>

#include "common.hpp"

using namespace sbwt;

extern "C" {

void sbwt_free(void *p) { std::free(p); }

int sbwt_fastx_read(const char *path, char **chars, uint64_t *n_chars, uint64_t **read_ends,
                    uint64_t *n_reads) {
  if (!path || !chars || !n_chars || !read_ends || !n_reads) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    ReadBatch b;
    FastxReader r(path);
    while (r.next_batch(b, ~0ULL, ~0ULL)) {
    }
    *chars = static_cast<char *>(std::malloc(std::max<size_t>(b.chars.size(), 1)));
    *read_ends = static_cast<uint64_t *>(std::malloc(std::max<size_t>(b.ends.size(), 1) * 8));
    if (!*chars || !*read_ends) throw std::bad_alloc();
    std::memcpy(*chars, b.chars.data(), b.chars.size());
    std::memcpy(*read_ends, b.ends.data(), b.ends.size() * 8);
    *n_chars = b.chars.size();
    *n_reads = b.ends.size();
  });
}

int sbwt_write_index_results(const char *out_prefix, int format, int write_headers,
                             const uint64_t *results, const uint64_t *read_ends,
                             uint64_t n_reads, uint32_t k) {
  if (!out_prefix || (n_reads && !read_ends) || format < 0 || format > 2) {
    set_last_error("bad argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    IndexResultsWriter w(out_prefix, static_cast<IndexFormat>(format), write_headers != 0);
    w.write(results, read_ends, n_reads, k);
  });
}

int sbwt_write_color_results(const char *out_prefix, int format, int write_headers,
                             const uint32_t *ids, const uint64_t *ids_offsets,
                             uint64_t n_reads, uint64_t num_colors) {
  if (!out_prefix || !ids_offsets || format < 0 || format > 2) {
    set_last_error("bad argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    ColorResultsWriter w(out_prefix, static_cast<ColorFormat>(format), write_headers != 0,
                         num_colors);
    w.write(ids, ids_offsets, n_reads);
  });
}

int sbwt_read_index_results(const char *path, uint64_t **found, uint64_t **offsets,
                            uint64_t **not_found, uint64_t **invalid, uint64_t *n_reads) {
  if (!path || !found || !offsets || !not_found || !invalid || !n_reads) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    // the arrays are written in place by the reader (no copies), and freed
    // here if it fails after allocating them
    using Owned = std::unique_ptr<uint64_t, void (*)(void *)>;
    Owned a(nullptr, std::free), b(nullptr, std::free), c(nullptr, std::free),
        d(nullptr, std::free);
    u64 reads = 0;
    read_index_results_into(path, [&](u64 n_found, u64 n) {
      auto get = [](Owned &o, u64 count) {
        o.reset(static_cast<uint64_t *>(std::malloc(std::max<u64>(count, 1) * 8)));
        if (!o) throw std::bad_alloc();
        return o.get();
      };
      reads = n;
      return ResultArrays{get(a, n_found), get(b, n + 1), get(c, n), get(d, n)};
    });
    *found = a.release();
    *offsets = b.release();
    *not_found = c.release();
    *invalid = d.release();
    *n_reads = reads;
  });
}

}  // extern "C"
