#include "formats.hpp"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "host_threads.hpp"

namespace sbwt {

namespace {

// Sequential reader over a file descriptor; arrays above 32 MiB are
// read in parallel pieces (pread on host threads).
class Reader {
 public:
  explicit Reader(const std::string &path) : fd_(::open(path.c_str(), O_RDONLY)) {
    if (fd_ < 0) throw std::runtime_error("Unable to open file " + path);
    struct stat st {};
    size_ = ::fstat(fd_, &st) == 0 ? (u64)st.st_size : 0;
  }
  ~Reader() { ::close(fd_); }
  Reader(const Reader &) = delete;
  Reader &operator=(const Reader &) = delete;
  u64 u64v() {
    u64 v = 0;
    read(&v, 8);
    return v;
  }
  u8 u8v() {
    u8 v = 0;
    read(&v, 1);
    return v;
  }
  std::string str() {  // u64 length + bytes (IOUtils.cpp:50-57)
    u64 n = u64v();
    if (n > (1ULL << 20)) throw std::runtime_error("corrupt string length");
    std::string s(n, '\0');
    read(s.data(), n);
    return s;
  }
  void read(void *dst, u64 n) {
    if (n > size_ || pos_ > size_ - n) throw std::runtime_error("unexpected end of file");
    char *out = static_cast<char *>(dst);
    std::atomic<bool> ok{true};
    run_parts(n, host_threads(n + (32ULL << 20) - 1, 32ULL << 20, 16), [&](u64 a, u64 b) {
      while (a < b) {
        const ssize_t got = ::pread(fd_, out + a, b - a, (off_t)(pos_ + a));
        if (got <= 0) {
          ok = false;
          return;
        }
        a += (u64)got;
      }
    });
    if (!ok) throw std::runtime_error("unexpected end of file");
    pos_ += n;
  }
  void skip(u64 n) {
    if (n > size_ || pos_ > size_ - n) throw std::runtime_error("unexpected end of file");
    pos_ += n;
  }
  // words of a vector of `bits` bits, checked against the rest of the file
  // before anything is allocated for them
  u64 words_for(u64 bits) const {
    const u64 nw = bits / 64 + (bits % 64 ? 1 : 0);
    if (nw > (size_ - pos_) / 8) throw std::runtime_error("unexpected end of file");
    return nw;
  }
  BitVector bitvector() {
    BitVector b;
    b.num_bits = u64v();
    b.words.resize(words_for(b.num_bits));
    read(b.words.data(), b.words.size() * 8);
    return b;
  }
  void skip_bitvector() { skip(words_for(u64v()) * 8); }
  IntVector intvector() {
    IntVector v;
    v.num_bits = u64v();
    v.width = u8v();
    if (v.width > 64) throw std::runtime_error("corrupt int vector width");
    v.words.resize(words_for(v.num_bits));
    read(v.words.data(), v.words.size() * 8);
    return v;
  }
  void skip_intvector() {
    const u64 bits = u64v();
    u8v();
    skip(words_for(bits) * 8);
  }

 private:
  int fd_;
  u64 size_ = 0, pos_ = 0;
};

class Writer {
 public:
  explicit Writer(const std::string &path) : f_(path, std::ios::binary) {
    if (!f_) throw std::runtime_error("Unable to open file for writing " + path);
  }
  void u64v(u64 v) { write(&v, 8); }
  void u8v(u8 v) { write(&v, 1); }
  void str(const std::string &s) {
    u64v(s.size());
    write(s.data(), s.size());
  }
  void write(const void *p, u64 n) {
    f_.write(static_cast<const char *>(p), static_cast<std::streamsize>(n));
    if (!f_) throw std::runtime_error("write failed");
  }
  void bitvector(const BitVector &b) {
    u64v(b.num_bits);
    write(b.words.data(), ((b.num_bits + 63) / 64) * 8);
  }
  void intvector(const IntVector &v) {
    u64v(v.num_bits);
    u8v(v.width);
    write(v.words.data(), ((v.num_bits + 63) / 64) * 8);
  }
  void words_blob(const std::vector<u64> &w) {  // int_vector<64>
    u64v(w.size() * 64);
    write(w.data(), w.size() * 8);
  }

 private:
  std::ofstream f_;
};

}  // namespace

u64 IntVector::get(u64 idx) const {
  if (width == 0) return 0;
  u64 bit = idx * width, w = bit / 64, off = bit % 64;
  u64 v = words[w] >> off;
  if (off + width > 64) v |= words[w + 1] << (64 - off);
  return width == 64 ? v : (v & ((1ULL << width) - 1));
}

void IntVector::assign(const std::vector<u64> &values, u8 w) {
  width = w;
  num_bits = values.size() * static_cast<u64>(w);
  words.assign((num_bits + 63) / 64, 0);
  // chunks of 64 values start on word boundaries, so chunks never share words
  const long chunks = (long)((values.size() + 63) / 64);
#pragma omp parallel for schedule(static)
  for (long ch = 0; ch < chunks; ++ch)
  for (u64 i = (u64)ch * 64; i < std::min<u64>(values.size(), (u64)ch * 64 + 64); ++i) {
    u64 bit = i * w, wi = bit / 64, off = bit % 64;
    u64 v = w == 64 ? values[i] : (values[i] & ((1ULL << w) - 1));
    words[wi] |= v << off;
    if (off + w > 64) words[wi + 1] |= v >> (64 - off);
  }
}

SbwtFile read_sbwt(const std::string &path) {
  Reader r(path);
  SbwtFile s;
  std::string variant = r.str();
  if (variant != "v0.1") {  // .tdbg files start with the version string
    if (variant != "plain-matrix")
      throw std::runtime_error("Error input is not a plain-matrix SBWT");
    if (r.str() != "v0.1") throw std::runtime_error("Error: wrong SBWT version");
  }
  for (auto &b : s.acgt) b = r.bitvector();
  for (int i = 1; i < 4; ++i)
    if (s.acgt[i].num_bits != s.acgt[0].num_bits)
      throw std::runtime_error("SBWT bitvectors differ in length");
  for (int i = 0; i < 4; ++i) r.skip_bitvector();  // rank blobs
  s.suffix_group_starts = r.bitvector();
  for (int i = 0; i < 2; ++i) r.skip(r.u64v());  // C-map, prefix table
  s.precalc_k = r.u64v();
  s.n_nodes = r.u64v();
  s.n_kmers = r.u64v();
  s.k = r.u64v();
  if (s.k == 0 || s.k > 256) throw std::runtime_error("SBWT k out of range");
  return s;
}

std::vector<u64> rank_v5_blob(const BitVector &bv) {
  // rank_support_v5: superblocks of 2048 bits; per superblock two u64: the
  // cumulative count, then five 12-bit counts of the 6-word steps packed at
  // shifts 60-12*(j/6).  Restated from the published sdsl layout.
  u64 cap_words = (bv.num_bits + 63) / 64;
  u64 cap_bits = cap_words * 64;
  std::vector<u64> blk(((cap_bits >> 11) + 1) << 1, 0);
  if (cap_words == 0) return blk;
  u64 j = 0, sum = __builtin_popcountll(bv.words[0]), second = 0, cnt = 1;
  for (u64 i = 1; i < cap_words; ++i, ++cnt) {
    if (cnt == 32) {
      j += 2;
      blk[j - 1] = second;
      blk[j] = blk[j - 2] + sum;
      second = sum = cnt = 0;
    } else if (cnt % 6 == 0) {
      second |= sum << (60 - 12 * (cnt / 6));
    }
    sum += __builtin_popcountll(bv.words[i]);
  }
  if (cnt % 6 == 0) second |= sum << (60 - 12 * (cnt / 6));
  if (cnt == 32) {
    j += 2;
    blk[j - 1] = second;
    blk[j] = blk[j - 2] + sum;
    blk[j + 1] = 0;
  } else {
    blk[j + 1] = second;
  }
  return blk;
}

void write_sbwt(const std::string &path, const SbwtFile &s) {
  Writer w(path);
  w.str("plain-matrix");
  w.str("v0.1");
  for (const auto &b : s.acgt) w.bitvector(b);
  for (const auto &b : s.acgt) w.words_blob(rank_v5_blob(b));
  w.bitvector(s.suffix_group_starts);
  // C array of the SBWT (4 signed 64-bit entries) as a byte vector.
  int64_t c[4];
  int64_t acc = 1;
  for (int i = 0; i < 4; ++i) {
    c[i] = acc;
    u64 ones = 0;
    for (u64 x : s.acgt[i].words) ones += __builtin_popcountll(x);
    acc += static_cast<int64_t>(ones);
  }
  w.u64v(sizeof(c));
  w.write(c, sizeof(c));
  w.u64v(0);  // empty k-mer prefix precalc table
  w.u64v(0);  // precalc_k
  w.u64v(s.n_nodes);
  w.u64v(s.n_kmers);
  w.u64v(s.k);
}

TColorsFile read_tcolors(const std::string &path) {
  Reader r(path);
  if (r.str() != "sdsl-hybrid-v4")
    throw std::runtime_error(
        "The colors file has an incorrect format. Expected 'sdsl-hybrid-v4'");
  TColorsFile t;
  t.dense_arrays = r.bitvector();
  t.dense_arrays_intervals = r.intvector();
  t.sparse_arrays = r.intvector();
  t.sparse_arrays_intervals = r.intvector();
  t.is_dense_marks = r.bitvector();
  r.skip_bitvector();  // rank_support_v5 of is_dense_marks
  t.key_kmer_marks = r.bitvector();
  r.skip_bitvector();  // rank_support_v5 of key_kmer_marks
  t.color_set_idxs = r.intvector();
  t.max_color_set_idx = r.u64v();
  t.largest_color = r.u64v();
  t.sum_color_set_sizes = r.u64v();
  return t;
}

BitVector read_key_kmer_marks(const std::string &path) {
  Reader r(path);
  if (r.str() != "sdsl-hybrid-v4")
    throw std::runtime_error(
        "The colors file has an incorrect format. Expected 'sdsl-hybrid-v4'");
  r.skip_bitvector();
  r.skip_intvector();
  r.skip_intvector();
  r.skip_intvector();
  r.skip_bitvector();
  r.skip_bitvector();
  return r.bitvector();
}

void write_tcolors(const std::string &path, const TColorsFile &t) {
  Writer w(path);
  w.str("sdsl-hybrid-v4");
  w.bitvector(t.dense_arrays);
  w.intvector(t.dense_arrays_intervals);
  w.intvector(t.sparse_arrays);
  w.intvector(t.sparse_arrays_intervals);
  w.bitvector(t.is_dense_marks);
  w.words_blob(rank_v5_blob(t.is_dense_marks));
  w.bitvector(t.key_kmer_marks);
  w.words_blob(rank_v5_blob(t.key_kmer_marks));
  w.intvector(t.color_set_idxs);
  w.u64v(t.max_color_set_idx);
  w.u64v(t.largest_color);
  w.u64v(t.sum_color_set_sizes);
}

}  // namespace sbwt
