// sbwt_search -- the reference's command line (src/main.cpp:24-34), on the
// B200 library:
//   sbwt_search index  -i <.sbwt|.tdbg> -q <query|.list> -o <prefix|.list>
//                      [-p ascii|binary|bool] [-k <.tcolors>] [--no-headers]
//   sbwt_search colors -k <.tcolors> -q <indexes|.list> -o <prefix|.list>
//                      [-p ascii|binary|csv] [-t <tau>] [--include-not-found]
//                      [--include-invalid] [--no-headers]
// Flags and defaults follow src/ArgumentParser/IndexSearchArgumentParser.cpp
// :29-241 and ColorSearchArgumentParser.cpp:29-177.  The memory / stream flags
// (-u -m -c -g -r -s) are accepted; this build sizes its batches from free
// device memory itself, but -c, -g and -t outside [0, 1] exit 1 with the
// reference's messages.  A missing required flag prints the help and exits 1
// (src/ArgumentParser/ArgumentParser.cpp:20-22); an unreadable input file is
// reported and skipped (src/SequenceFileParser/
// ContinuousSequenceFileParser.cpp:114-133).
//
// A query file whose text fits the device (with its results) is handled on
// the GPU end to end: its bytes are copied once, parsed, searched and
// formatted there, and only the formatted output comes back.  Larger files
// stream through the host reader in batches of 256 M chars.
#include <cuda_runtime.h>

#include <sys/stat.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sbwt_b200.h"
#include "host_io.hpp"

using namespace sbwt;

namespace {

struct Args {
  std::map<std::string, std::string> kv;
  std::map<std::string, bool> flags;
  bool has(const std::string &k) const { return kv.count(k) != 0; }
  std::string get(const std::string &k, const std::string &d = "") const {
    auto it = kv.find(k);
    return it == kv.end() ? d : it->second;
  }
};

const char *kIndexHelp =
    "Usage: sbwt_search index [OPTION...]\n"
    "  -q, --query-file arg            query FASTA/FASTQ file (.gz ok) or .list of files\n"
    "  -i, --index-file arg            .sbwt or .tdbg index\n"
    "  -o, --output-prefix arg         output prefix or .list of prefixes\n"
    "  -p, --print-mode arg            ascii | binary | bool (default: ascii)\n"
    "  -k, --colors-file arg           .tcolors file: report the next key k-mer (d > 1)\n"
    "      --no-headers                do not write the format/version header\n"
    "  -u, -m, -c, -r, -g, -s          memory / stream sizing (unused; -c, -g in [0, 1])\n"
    "  -h, --help                      print this help\n";
const char *kColorsHelp =
    "Usage: sbwt_search colors [OPTION...]\n"
    "  -q, --query-file arg            index results (.txt/.bin) or .list of files\n"
    "  -k, --colors-file arg           .tcolors file\n"
    "  -o, --output-prefix arg         output prefix or .list of prefixes\n"
    "  -p, --print-mode arg            ascii | binary | csv (default: ascii)\n"
    "  -t, --threshold arg             fraction of k-mers a color needs (default: 1)\n"
    "      --include-not-found         count not-found k-mers in the read size\n"
    "      --include-invalid           count invalid k-mers in the read size\n"
    "      --no-headers                do not write the format/version header\n"
    "  -u, -m, -c, -r, -g, -s          memory / stream sizing (unused; -c, -g in [0, 1])\n"
    "  -h, --help                      print this help\n";

Args parse(int argc, char **argv, int first) {
  static const std::map<std::string, std::string> shorts = {
      {"q", "query-file"},    {"i", "index-file"},   {"o", "output-prefix"},
      {"p", "print-mode"},    {"k", "colors-file"},  {"u", "unavailable-main-memory"},
      {"m", "max-main-memory"}, {"c", "cpu-memory-percentage"},
      {"r", "base-pairs-per-seq"}, {"g", "gpu-memory-percentage"}, {"s", "streams"},
      {"t", "threshold"},     {"h", "help"}};
  static const std::vector<std::string> bools = {"no-headers", "include-not-found",
                                                 "include-invalid", "help"};
  Args a;
  for (int i = first; i < argc; ++i) {
    std::string t = argv[i];
    std::string name;
    if (t.rfind("--", 0) == 0) {
      name = t.substr(2);
    } else if (t.size() >= 2 && t[0] == '-') {
      auto it = shorts.find(t.substr(1));
      name = it == shorts.end() ? t.substr(1) : it->second;
    } else {
      continue;
    }
    auto eq = name.find('=');
    if (eq != std::string::npos) {
      a.kv[name.substr(0, eq)] = name.substr(eq + 1);
      continue;
    }
    bool is_bool = false;
    for (auto &b : bools) is_bool |= (b == name);
    if (is_bool) {
      a.flags[name] = true;
    } else if (i + 1 < argc) {
      a.kv[name] = argv[++i];
    }
  }
  return a;
}

int missing(const Args &a, const std::vector<std::string> &req, const char *help) {
  for (auto &r : req)
    if (!a.has(r)) {
      std::printf("Missing option: %s\n%s", r.c_str(), help);
      return 1;
    }
  return 0;
}

// A fraction flag outside [0, 1] (or not a number): the reference prints
// `message` to stderr and exits 1 before any work
// (IndexSearchArgumentParser.cpp:203-222, ColorSearchArgumentParser.cpp:202-235).
int bad_fraction(const Args &a, const std::string &name, const char *message) {
  if (!a.has(name)) return 0;
  const std::string v = a.get(name);
  char *end = nullptr;
  const double x = std::strtod(v.c_str(), &end);
  if (end != v.c_str() && *end == '\0' && x >= 0 && x <= 1) return 0;
  std::fprintf(stderr, "%s\n", message);
  return 1;
}

int bad_sizing(const Args &a) {
  return bad_fraction(a, "cpu-memory-percentage",
                      "Invalid value for cpu-memory-percentage. Must be between 0 and 1.") ||
         bad_fraction(a, "gpu-memory-percentage",
                      "Invalid value for gpu-memory-percentage. Must be between 0 and 1.");
}

void check(int rc) {
  if (rc != SBWT_OK) throw std::runtime_error(sbwt_last_error());
}

void check_cuda(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}

// Device / pinned host memory owned by the command line tool.
struct DevMem {
  void *p = nullptr;
  explicit DevMem(size_t n) { check_cuda(cudaMalloc(&p, n ? n : 1)); }
  ~DevMem() { cudaFree(p); }
  template <class T>
  T *get() const {
    return static_cast<T *>(p);
  }
};
struct HostMem {
  void *p = nullptr;
  explicit HostMem(size_t n) { check_cuda(cudaMallocHost(&p, n ? n : 1)); }
  ~HostMem() { cudaFreeHost(p); }
};

struct Stream {
  cudaStream_t s = nullptr;
  Stream() { check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~Stream() { cudaStreamDestroy(s); }
};

// Largest query text handled on the device in one piece: per char of text at
// most 33 bytes stay within 80 % of the free device memory (text and chars
// 1 each, read ends 8 per read and a read takes at least 4 chars of text,
// one u64 result per k-mer, at most 21 formatted bytes per k-mer).
// SBWT_CLI_DEVICE_PIECE_BYTES (environment) lowers it, e.g. to test the
// batched path on small files.
u64 device_text_budget(int device) {
  size_t free_b = 0, total_b = 0;
  check_cuda(cudaSetDevice(device));
  check_cuda(cudaMemGetInfo(&free_b, &total_b));
  u64 b = (u64)(0.8 * (double)free_b / 33.0);
  if (const char *e = std::getenv("SBWT_CLI_DEVICE_PIECE_BYTES"))
    b = std::min<u64>(b, std::strtoull(e, nullptr, 10));
  return b;
}

// A device buffer that grows to the largest size asked for.
struct GrowMem {
  void *p = nullptr;
  u64 cap = 0;
  ~GrowMem() { cudaFree(p); }
  template <class T>
  T *get(u64 n) {
    if (n > cap || !p) {
      cudaFree(p);
      p = nullptr;
      check_cuda(cudaMalloc(&p, n ? n : 1));
      cap = n;
    }
    return static_cast<T *>(p);
  }
};

struct Event {
  cudaEvent_t e = nullptr;
  Event() { check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)); }
  ~Event() { cudaEventDestroy(e); }
};

// Host <-> device streaming through two pinned buffers of kStageBytes: one is
// filled (or written out) by the host while the other's copy runs, so no
// pinned buffer of the whole file or output is allocated.
constexpr u64 kStageBytes = 64ULL << 20;
struct Staging {
  HostMem buf[2]{HostMem(kStageBytes), HostMem(kStageBytes)};
  Event done[2];
};

// The size of a plain (not gzip) file, or -1 (gzip, unreadable).
long long plain_file_size(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return -1;
  unsigned char m[2] = {0, 0};
  const size_t got = std::fread(m, 1, 2, f);
  std::fclose(f);
  if (got == 2 && m[0] == 0x1f && m[1] == 0x8b) return -1;
  struct stat st{};
  if (::stat(path.c_str(), &st) != 0) return -1;
  return (long long)st.st_size;
}

// Reads a plain file of n bytes into d_text (device), chunk by chunk.
void read_file_to_device(const std::string &path, u64 n, char *d_text, Staging &sg,
                         cudaStream_t st) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("Unable to open file " + path);
  u64 off = 0;
  for (int i = 0; off < n; ++i) {
    const int b = i & 1;
    if (i >= 2) check_cuda(cudaEventSynchronize(sg.done[b].e));  // its last copy is done
    const u64 len = std::min<u64>(kStageBytes, n - off);
    if (std::fread(sg.buf[b].p, 1, len, f) != len) {
      std::fclose(f);
      throw std::runtime_error("read error in sequence file");
    }
    check_cuda(cudaMemcpyAsync(d_text + off, sg.buf[b].p, len, cudaMemcpyHostToDevice, st));
    check_cuda(cudaEventRecord(sg.done[b].e, st));
    off += len;
  }
  std::fclose(f);
}

// Writes nb device bytes to w, chunk by chunk (the copy of chunk i runs
// while chunk i - 1 is written).
void write_device_bytes(const char *d_bytes, u64 nb, IndexResultsWriter &w, Staging &sg,
                        cudaStream_t st) {
  u64 prev_len = 0;
  int prev = -1;
  for (u64 off = 0, i = 0; off < nb; ++i) {
    const int b = (int)(i & 1);
    const u64 len = std::min<u64>(kStageBytes, nb - off);
    check_cuda(cudaMemcpyAsync(sg.buf[b].p, d_bytes + off, len, cudaMemcpyDeviceToHost, st));
    check_cuda(cudaEventRecord(sg.done[b].e, st));
    if (prev >= 0) {
      check_cuda(cudaEventSynchronize(sg.done[prev].e));
      w.write_raw(static_cast<const char *>(sg.buf[prev].p), prev_len);
    }
    prev = b;
    prev_len = len;
    off += len;
  }
  if (prev >= 0) {
    check_cuda(cudaEventSynchronize(sg.done[prev].e));
    w.write_raw(static_cast<const char *>(sg.buf[prev].p), prev_len);
  }
}

// One whole query text through the GPU: parse, search, format; the formatted
// bytes are appended to w.  The text is either in host memory (`text`) or
// read from the plain file `path` of n bytes.
void index_text_on_device(sbwt_index_t *ix, const sbwt_index_info_t &info, uint32_t flags,
                          const std::vector<char> *text, const std::string &path, u64 n,
                          int format, IndexResultsWriter &w) {
  if (n == 0) return;
  Stream st;
  Staging sg;
  const uint32_t dp = SBWT_DEVICE_POINTERS;
  DevMem d_text(n), d_chars(n);
  if (text)
    check_cuda(cudaMemcpyAsync(d_text.p, text->data(), n, cudaMemcpyHostToDevice, st.s));
  else
    read_file_to_device(path, n, d_text.get<char>(), sg, st.s);
  u64 nc = 0, nr = 0;
  int rc = sbwt_fastx_parse(d_text.get<char>(), n, d_chars.get<char>(), n, nullptr, 0, &nc,
                            &nr, dp, info.device, st.s);
  if (rc != SBWT_E_CAPACITY) check(rc);
  if (nr == 0) return;
  DevMem d_ends(nr * 8);
  check(sbwt_fastx_parse(d_text.get<char>(), n, d_chars.get<char>(), n, d_ends.get<u64>(), nr,
                         &nc, &nr, dp, info.device, st.s));
  DevMem d_res(std::max<u64>(nc, 1) * 8);
  u64 nk = 0;
  check(sbwt_search_reads(ix, d_chars.get<char>(), nc, d_ends.get<u64>(), nr, d_res.get<u64>(),
                          std::max<u64>(nc, 1), &nk, flags | dp, st.s));
  u64 nb = 0;
  rc = sbwt_format_index_results(d_res.get<u64>(), d_ends.get<u64>(), nr, info.k, format,
                                 nullptr, 0, &nb, dp, info.device, st.s);
  if (rc != SBWT_E_CAPACITY) check(rc);
  DevMem d_out(nb);
  check(sbwt_format_index_results(d_res.get<u64>(), d_ends.get<u64>(), nr, info.k, format,
                                  d_out.get<char>(), nb, &nb, dp, info.device, st.s));
  write_device_bytes(d_out.get<char>(), nb, w, sg, st.s);
}

// One host-parsed batch (chars and cumulative read ends) through the GPU:
// search, format, and the formatted bytes appended to w.
struct DeviceBatch {
  GrowMem chars, ends, res, out;
};
void index_batch_on_device(sbwt_index_t *ix, const sbwt_index_info_t &info, uint32_t flags,
                           const ReadBatch &b, int format, IndexResultsWriter &w,
                           DeviceBatch &db, Staging &sg, cudaStream_t st) {
  const u64 nc = b.chars.size(), nr = b.ends.size();
  if (nr == 0) return;
  const uint32_t dp = SBWT_DEVICE_POINTERS;
  char *d_chars = db.chars.get<char>(nc + 16);
  u64 *d_ends = db.ends.get<u64>(nr * 8);
  check_cuda(cudaMemcpyAsync(d_chars, b.chars.data(), nc, cudaMemcpyHostToDevice, st));
  check_cuda(cudaMemcpyAsync(d_ends, b.ends.data(), nr * 8, cudaMemcpyHostToDevice, st));
  const u64 cap = std::max<u64>(nc, 1);
  u64 *d_res = db.res.get<u64>(cap * 8);
  u64 nk = 0;
  check(sbwt_search_reads(ix, d_chars, nc, d_ends, nr, d_res, cap, &nk, flags | dp, st));
  u64 nb = 0;
  const int rc = sbwt_format_index_results(d_res, d_ends, nr, info.k, format, nullptr, 0, &nb,
                                           dp, info.device, st);
  if (rc != SBWT_E_CAPACITY) check(rc);
  char *d_out = db.out.get<char>(nb);
  check(sbwt_format_index_results(d_res, d_ends, nr, info.k, format, d_out, nb, &nb, dp,
                                  info.device, st));
  write_device_bytes(d_out, nb, w, sg, st);
}

int run_index(const Args &a) {
  if (a.flags.count("help")) {
    std::printf("%s", kIndexHelp);
    return 1;
  }
  if (missing(a, {"query-file", "index-file", "output-prefix"}, kIndexHelp)) return 1;
  if (bad_sizing(a)) return 1;
  const std::string mode = a.get("print-mode", "ascii");
  IndexFormat fmt = mode == "binary" ? IndexFormat::Binary
                    : mode == "bool" ? IndexFormat::Bool
                                     : IndexFormat::Ascii;
  if (mode != "ascii" && mode != "binary" && mode != "bool")
    throw std::runtime_error("Invalid value passed by user for argument print_mode");
  const bool headers = !a.flags.count("no-headers");
  std::vector<std::string> ins, outs;
  paired_file_lists(a.get("query-file"), a.get("output-prefix"), ins, outs);
  const std::string colors = a.get("colors-file");
  sbwt_index_t *ix = nullptr;
  check(sbwt_index_open(a.get("index-file").c_str(), colors.empty() ? nullptr : colors.c_str(),
                        0, 0, &ix));
  sbwt_index_info_t info{};
  check(sbwt_index_get_info(ix, &info));
  const uint32_t flags = colors.empty() ? 0 : SBWT_MOVE_TO_KEY_KMER;
  const u64 batch_chars = 256ULL << 20;
  const int format = fmt == IndexFormat::Ascii ? 0 : fmt == IndexFormat::Binary ? 1 : 2;
  const u64 budget = device_text_budget(info.device);
  std::vector<char> text;
  for (size_t f = 0; f < ins.size(); ++f) {
    // a plain file that fits goes to the device as it is read; a gzip file
    // that fits is inflated on the host first
    const long long plain = plain_file_size(ins[f]);
    if (plain >= 0 && (u64)plain <= budget) {
      IndexResultsWriter w(outs[f], fmt, headers);
      index_text_on_device(ix, info, flags, nullptr, ins[f], (u64)plain, format, w);
      continue;
    }
    bool whole = false;
    try {
      whole = read_whole_file(ins[f], budget, text);
    } catch (const std::exception &e) {
      std::fprintf(stderr, "[error] %s\n", e.what());
      continue;
    }
    if (whole) {
      IndexResultsWriter w(outs[f], fmt, headers);
      index_text_on_device(ix, info, flags, &text, std::string(), text.size(), format, w);
      continue;
    }
    // larger than one device piece: parsed on the host batch by batch, each
    // batch searched and formatted on the device
    text = std::vector<char>();
    std::unique_ptr<FastxReader> rd = std::make_unique<FastxReader>(ins[f]);
    IndexResultsWriter w(outs[f], fmt, headers);
    Stream st;
    Staging sg;
    DeviceBatch db;
    ReadBatch b;
    while (true) {
      b.clear();
      if (!rd->next_batch(b, batch_chars, ~0ULL)) break;
      index_batch_on_device(ix, info, flags, b, format, w, db, sg, st.s);
    }
  }
  sbwt_index_free(ix);
  return 0;
}

int run_colors(const Args &a) {
  if (a.flags.count("help")) {
    std::printf("%s", kColorsHelp);
    return 1;
  }
  if (missing(a, {"query-file", "colors-file", "output-prefix"}, kColorsHelp)) return 1;
  if (bad_sizing(a) ||
      bad_fraction(a, "threshold",
                   "Invalid value for threshold, must be between 1 and 0 (both included)"))
    return 1;
  const std::string mode = a.get("print-mode", "ascii");
  if (mode != "ascii" && mode != "binary" && mode != "csv")
    throw std::runtime_error("Invalid value passed by user for argument print_mode");
  ColorFormat fmt = mode == "binary" ? ColorFormat::Binary
                    : mode == "csv"  ? ColorFormat::Csv
                                     : ColorFormat::Ascii;
  const bool headers = !a.flags.count("no-headers");
  const double tau = std::stod(a.get("threshold", "1"));
  uint32_t flags = 0;
  if (a.flags.count("include-not-found")) flags |= SBWT_INCLUDE_NOT_FOUND;
  if (a.flags.count("include-invalid")) flags |= SBWT_INCLUDE_INVALID;
  std::vector<std::string> ins, outs;
  paired_file_lists(a.get("query-file"), a.get("output-prefix"), ins, outs);
  sbwt_colors_t *ci = nullptr;
  check(sbwt_colors_open(a.get("colors-file").c_str(), 0, &ci));
  const u64 C = sbwt_colors_num_colors(ci);
  for (size_t f = 0; f < ins.size(); ++f) {
    IndexResults r;
    try {
      r = read_index_results(ins[f]);
    } catch (const std::exception &e) {
      std::fprintf(stderr, "[error] %s\n", e.what());
      continue;
    }
    const u64 n = r.not_found.size();
    U64Array offs(n + 1);
    std::vector<uint32_t, NoInitAlloc<uint32_t>> ids(std::max<u64>(r.found.size(), 1));
    int rc = sbwt_pseudoalign(ci, r.found.data(), r.offsets.data(), r.not_found.data(),
                              r.invalid.data(), n, tau, flags, ids.data(), ids.size(),
                              offs.data(), nullptr);
    if (rc == SBWT_E_CAPACITY) {
      ids.resize(offs[n] + 1);
      rc = sbwt_pseudoalign(ci, r.found.data(), r.offsets.data(), r.not_found.data(),
                            r.invalid.data(), n, tau, flags, ids.data(), ids.size(),
                            offs.data(), nullptr);
    }
    check(rc);
    ColorResultsWriter w(outs[f], fmt, headers, C);
    // ids formatted on the GPU (the same bytes as the host writer)
    const int format = fmt == ColorFormat::Ascii ? 0 : fmt == ColorFormat::Binary ? 1 : 2;
    u64 nb = 0;
    rc = sbwt_format_color_results(ids.data(), offs.data(), n, C, format, nullptr, 0, &nb, 0, 0,
                                   nullptr);
    if (rc != SBWT_E_CAPACITY) check(rc);
    std::vector<char> bytes(std::max<u64>(nb, 1));
    check(sbwt_format_color_results(ids.data(), offs.data(), n, C, format, bytes.data(), nb, &nb,
                                    0, 0, nullptr));
    w.write_raw(bytes.data(), nb);
  }
  sbwt_colors_free(ci);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  const char *usage = "Usage: sbwt_search [index|colors] [OPTIONS]\n";
  if (argc < 2) {
    std::printf("%s", usage);
    return 1;
  }
  const std::string cmd = argv[1];
  try {
    Args a = parse(argc, argv, 2);
    if (cmd == "index") return run_index(a);
    if (cmd == "colors") return run_colors(a);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "[error] %s\n", e.what());
    return 2;
  }
  std::printf("%s", usage);
  return 1;
}
