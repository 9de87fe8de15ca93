// Host-side I/O of the drop-in boundary: FASTA/FASTQ batches in, the
// reference's index / color result formats out, index result files back in.
#pragma once

#include <zlib.h>

#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "formats.hpp"

namespace sbwt {

using u64 = uint64_t;
using u32 = uint32_t;

// Reads of a batch: chars back to back, cumulative exclusive ends.
struct ReadBatch {
  std::vector<char> chars;
  std::vector<u64> ends;
  void clear() {
    chars.clear();
    ends.clear();
  }
};

// FASTA / FASTQ reader with kseq record semantics (the reference parses with
// kseqpp_REad v1.6.0, src/SequenceFileParser/ContinuousSequenceFileParser.cpp
// :148-156): a record starts at '>' or '@'; its sequence is the concatenation
// of the following lines up to a line starting with '>', '+' or '@'; after a
// '+' line, quality lines are consumed until they are as long as the
// sequence; empty records are kept (they print an empty line); trailing '\r'
// is dropped.  gzip input is read transparently.
class FastxReader {
 public:
  explicit FastxReader(const std::string &path);
  ~FastxReader();
  // Appends whole records to `b` until it holds >= max_chars chars or
  // max_reads reads (a record is never split).  Returns false at end of file
  // when nothing was appended.
  bool next_batch(ReadBatch &b, u64 max_chars, u64 max_reads);

 private:
  bool getline(std::string &line);
  gzFile f_ = nullptr;
  std::vector<char> buf_;
  size_t pos_ = 0, len_ = 0;
  bool eof_ = false;
  bool have_header_ = false;  // the next record's header line was consumed
  std::string line_;
};

enum class IndexFormat { Ascii, Binary, Bool };
enum class ColorFormat { Ascii, Binary, Csv };

// Writers of the reference's index-step outputs
// (src/IndexResultsPrinter/*ContinuousIndexResultsPrinter.cpp): extension
// .txt / .bin / .bool, optional header = length-prefixed format and version
// strings ("ascii" "v1.0", "binary" "v1.0", "bool" "v2.0").
class IndexResultsWriter {
 public:
  IndexResultsWriter(const std::string &prefix, IndexFormat fmt, bool headers);
  ~IndexResultsWriter();
  // results: one u64 per k-mer of every read (SBWT_NOT_FOUND / SBWT_INVALID
  // markers), read_ends as passed to the search; k gives k-mers per read.
  void write(const u64 *results, const u64 *read_ends, u64 n_reads, u32 k);
  // Appends bytes that are already in this format (formatted on the GPU).
  void write_raw(const char *bytes, u64 n);

 private:
  FILE *f_ = nullptr;
  IndexFormat fmt_;
  std::vector<char> buf_;
};

// Writers of the colors-step outputs
// (src/ColorResultsPrinter/*ContinuousColorResultsPrinter.cpp): .txt (ids
// separated by spaces, '\n' per read), .bin (u64 ids, u64 -1 per read end),
// .csv (header row 1..N always, then a 0/1 row per read).
class ColorResultsWriter {
 public:
  ColorResultsWriter(const std::string &prefix, ColorFormat fmt, bool headers,
                     u64 num_colors);
  ~ColorResultsWriter();
  void write(const uint32_t *ids, const u64 *ids_offsets, u64 n_reads);
  void write_raw(const char *bytes, u64 n);

 private:
  FILE *f_ = nullptr;
  ColorFormat fmt_;
  u64 num_colors_;
  std::vector<char> buf_;
};

// Index-step result files read back for the colors step
// (src/IndexFileParser/AsciiIndexFileParser.cpp:33-98,
//  BinaryIndexFileParser.cpp:33-69): per read the found indexes, and the
// counts of -1 and -2 tokens.
struct IndexResults {
  U64Array found;    // all reads back to back
  U64Array offsets;  // n_reads + 1
  U64Array not_found, invalid;
};
IndexResults read_index_results(const std::string &path);

// The whole (gzip-transparent) file, or false when it holds more than
// max_bytes bytes.
bool read_whole_file(const std::string &path, u64 max_bytes, std::vector<char> &out);

// The query and output names of one command line, paired as the reference
// pairs them (src/FilenamesParser/FilenamesParser.cpp:19-46): when the query
// name ends in ".list", the query file and the output file are both read as
// one name per line; otherwise each is one name.  Lists of different lengths
// throw "Input and output file sizes differ" (src/Main/IndexSearchMain.cpp:
// 405-407, ColorSearchMain.cpp:224-226).
void paired_file_lists(const std::string &query, const std::string &output,
                       std::vector<std::string> &ins, std::vector<std::string> &outs);

}  // namespace sbwt
