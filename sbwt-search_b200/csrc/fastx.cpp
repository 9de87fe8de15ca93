#include <cstring>
#include <fstream>
#include <stdexcept>

#include "host_io.hpp"

namespace sbwt {

FastxReader::FastxReader(const std::string &path) {
  f_ = gzopen(path.c_str(), "rb");
  if (!f_) throw std::runtime_error("Unable to open file " + path);
  gzbuffer(f_, 1 << 20);
  buf_.resize(1 << 22);
}

FastxReader::~FastxReader() {
  if (f_) gzclose(f_);
}

bool FastxReader::getline(std::string &line) {
  line.clear();
  while (true) {
    if (pos_ == len_) {
      if (eof_) return !line.empty();
      const int n = gzread(f_, buf_.data(), (unsigned)buf_.size());
      if (n < 0) throw std::runtime_error("read error in sequence file");
      if (n == 0) {
        eof_ = true;
        return !line.empty();
      }
      pos_ = 0;
      len_ = (size_t)n;
    }
    const char *s = buf_.data() + pos_;
    const void *nl = memchr(s, '\n', len_ - pos_);
    if (nl) {
      const size_t m = (const char *)nl - s;
      line.append(s, m);
      pos_ += m + 1;
      if (!line.empty() && line.back() == '\r') line.pop_back();
      return true;
    }
    line.append(s, len_ - pos_);
    pos_ = len_;
  }
}

bool FastxReader::next_batch(ReadBatch &b, u64 max_chars, u64 max_reads) {
  bool any = false;
  while (b.chars.size() < max_chars && b.ends.size() < max_reads) {
    if (!have_header_) {  // find the next header line
      bool found = false;
      while (getline(line_)) {
        if (!line_.empty() && (line_[0] == '>' || line_[0] == '@')) {
          found = true;
          break;
        }
      }
      if (!found) return any;
      have_header_ = true;
    }
    // sequence lines
    have_header_ = false;
    u64 seq_len = 0;
    bool plus = false;
    while (getline(line_)) {
      const char c0 = line_.empty() ? '\n' : line_[0];
      if (c0 == '>' || c0 == '@') {
        have_header_ = true;
        break;
      }
      if (c0 == '+') {
        plus = true;
        break;
      }
      b.chars.insert(b.chars.end(), line_.begin(), line_.end());
      seq_len += line_.size();
    }
    if (plus) {  // quality: at least as long as the sequence
      u64 q = 0;
      while (q < seq_len && getline(line_)) q += line_.size();
    }
    b.ends.push_back(b.chars.size());
    any = true;
  }
  return true;
}

bool read_whole_file(const std::string &path, u64 max_bytes, std::vector<char> &out) {
  gzFile f = gzopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("Unable to open file " + path);
  gzbuffer(f, 1 << 20);
  out.clear();
  const size_t step = 64 << 20;
  while (true) {
    const size_t at = out.size();
    if (at > max_bytes) {
      gzclose(f);
      return false;
    }
    out.resize(at + step);
    const int n = gzread(f, out.data() + at, (unsigned)step);
    if (n < 0) {
      gzclose(f);
      throw std::runtime_error("read error in sequence file");
    }
    out.resize(at + (size_t)n);
    if (n == 0) break;
  }
  gzclose(f);
  return out.size() <= max_bytes;
}

void paired_file_lists(const std::string &query, const std::string &output,
                       std::vector<std::string> &ins, std::vector<std::string> &outs) {
  auto lines = [](const std::string &name) {
    std::ifstream in(name);
    if (!in) throw std::runtime_error("Unable to open file " + name);
    std::vector<std::string> v;
    std::string ln;
    while (std::getline(in, ln)) v.push_back(ln);
    return v;
  };
  const std::string ext = ".list";
  if (query.size() >= ext.size() &&
      query.compare(query.size() - ext.size(), ext.size(), ext) == 0) {
    ins = lines(query);
    outs = lines(output);
  } else {
    ins = {query};
    outs = {output};
  }
  if (ins.size() != outs.size()) throw std::runtime_error("Input and output file sizes differ");
}

}  // namespace sbwt
