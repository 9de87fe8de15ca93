/*
 * sbwt_b200.h -- C ABI of the B200 (sm_100a) SBWT k-mer search library.
 *
 * Drop-in for the two search steps of SBWT-Search.  Plain pointers and sizes
 * only; every call returns a status code and never aborts the process; the
 * message of the last failing call on the calling thread is kept in
 * sbwt_last_error().  Index and color handles are immutable after they are
 * opened and may be shared by threads; each call uses its own internal
 * scratch keyed by the calling thread and device.
 *
 * Pointer arguments are host pointers unless SBWT_DEVICE_POINTERS is set in
 * flags, in which case every array argument (inputs and outputs) is a device
 * pointer on the handle's device and the call is asynchronous on `stream`
 * (a cudaStream_t, NULL = legacy default stream) except where noted.
 */
#ifndef SBWT_B200_H
#define SBWT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Replace the reference's exceptions
 * (GPU_CHECK: src/Tools/GpuUtils.h:20-29; loader magic checks:
 * src/SbwtBuilder/SbwtBuilder.cpp:61-68, src/ColorIndexBuilder/
 * ColorIndexBuilder.cpp:15-20). */
#define SBWT_OK 0
#define SBWT_E_IO 1        /* file missing / unreadable */
#define SBWT_E_FORMAT 2    /* bad magic, version or corrupt file */
#define SBWT_E_OOM 3       /* device or host allocation failed */
#define SBWT_E_CUDA 4      /* CUDA runtime error */
#define SBWT_E_TIMEOUT 5   /* a bounded device wait ran out */
#define SBWT_E_INVALID 6   /* bad argument */
#define SBWT_E_CAPACITY 7  /* output buffer too small (required size reported) */

/* flags */
#define SBWT_DEVICE_POINTERS 0x1u  /* arrays are device pointers, async */
#define SBWT_MOVE_TO_KEY_KMER 0x2u /* index step: walk found k-mers forward to
                                      the next key k-mer (reference -k / d>1) */
#define SBWT_PER_KMER_WALK 0x4u    /* index step over reads: search every
                                      k-mer independently (no streaming reuse
                                      of the previous k-mer's node) */
#define SBWT_INCLUDE_NOT_FOUND 0x8u /* colors: count -1 k-mers in the read size */
#define SBWT_INCLUDE_INVALID 0x10u  /* colors: count -2 k-mers in the read size */

/* Result markers of the index step (as printed: -1 and -2). */
#define SBWT_NOT_FOUND UINT64_MAX
#define SBWT_INVALID (UINT64_MAX - 1)

const char *sbwt_last_error(void);
const char *sbwt_version(void);

/* ------------------------------------------------------------------------ */
/* Index step                                                               */
/* ------------------------------------------------------------------------ */
typedef struct sbwt_index sbwt_index_t;

typedef struct {
  uint64_t num_bits;          /* nodes of the SBWT (bits per A/C/G/T vector) */
  uint32_t k;                 /* k-mer size */
  uint32_t presearch_letters; /* depth of the presearch table */
  uint64_t c_map[5];          /* c_map[0] = 1, c_map[c+1] = c_map[c] + |c| */
  uint64_t device_bytes;      /* device memory held by the handle */
  int device;
  int has_key_kmer_marks;
  uint64_t kmer_table_bytes;  /* k-mer -> node table (0 when absent) */
  uint64_t kmer_filter_bytes; /* k-mer filter in front of the table (0 when absent) */
  uint32_t host_result_bytes; /* bytes per k-mer a host-pointer sbwt_search_reads moves
                                 device -> host into a pageable results buffer with
                                 default flags: 4 (32-bit codes widened on host
                                 threads) or 8; a pinned buffer always takes 8 */
  uint32_t reserved;
} sbwt_index_info_t;

/* Loads a .sbwt / .tdbg file (and, when colors_path is not NULL, the key
 * k-mer marks of a .tcolors file for SBWT_MOVE_TO_KEY_KMER) onto `device`
 * and builds the rank blocks and the presearch table there.
 * presearch_letters: 0 = default (14 for SBWTs of 2^26 or more nodes, else
 * the reference's 12), else 1..14 (deeper tables replace more search steps;
 * results are the same; the depth-14 pyramid takes 2.9 GB, 5.7 GB for 2^32
 * or more nodes).
 * SBWT_E_IO when a file cannot be opened; SBWT_E_FORMAT for a bad magic or
 * version string, a truncated file or a length the file cannot hold.
 * Replaces SbwtBuilder::get_cpu_sbwt + CpuSbwtContainer::to_gpu +
 * Presearcher::presearch (src/SbwtBuilder/SbwtBuilder.cpp:41-56,
 * src/SbwtContainer/CpuSbwtContainer.cpp:23-35,
 * src/Presearcher/Presearcher.cpp:18-30, src/Main/IndexSearchMain.cpp:87-103).
 */
int sbwt_index_open(const char *sbwt_path, const char *colors_path, int device,
                    unsigned presearch_letters, sbwt_index_t **out);

/* Same from host arrays: acgt[c] has ceil(num_bits/64) words (LSB-first bits).
 * suffix_group_starts (same size) enables the streaming read search; NULL
 * makes sbwt_search_reads fall back to independent per-k-mer walks.
 * key_kmer_marks may be NULL. */
int sbwt_index_from_arrays(const uint64_t *const acgt[4], uint64_t num_bits,
                           uint32_t k, const uint64_t *suffix_group_starts,
                           const uint64_t *key_kmer_marks, int device,
                           unsigned presearch_letters, sbwt_index_t **out);
void sbwt_index_free(sbwt_index_t *index);
int sbwt_index_get_info(const sbwt_index_t *index, sbwt_index_info_t *info);

/* The reference's in-process index seam, IndexSearcher::search
 * (src/IndexSearcher/IndexSearcher.h:41-46, IndexSearcher.cpp:26-51,
 * kernel d_search src/IndexSearcher/IndexSearcher.cuh:22-72):
 *   bit_seqs   -- 2-bit MSB-first packed chars, 32 per word (A0 C1 G2 T3);
 *   positions  -- start char of each k-mer;
 *   results    -- one u64 per position: SBWT node index, or SBWT_NOT_FOUND.
 * Invalid chars are whatever their 2-bit code says (the reference packs them
 * as A); no -2 masking is applied here, as in the reference kernel.
 * bit_seqs must be readable up to word (max position + k - 1) / 32.
 * With host pointers the call is synchronous like the reference's. */
int sbwt_search_positions(const sbwt_index_t *index, const uint64_t *bit_seqs,
                          uint64_t n_words, const uint64_t *positions,
                          uint64_t n_positions, uint64_t *results,
                          uint32_t flags, void *stream);

/* Number of k-mer results of reads whose cumulative exclusive ends are
 * read_ends[0..n_reads): sum over reads of max(0, length - k + 1). */
uint64_t sbwt_count_kmers(const uint64_t *read_ends, uint64_t n_reads,
                          uint32_t k);

/* Fused index step over raw reads (SeqToBits + PositionsBuilder + search +
 * the printer's -1/-2 mapping in one device pipeline; reference
 * src/SeqToBitsConverter/ContinuousSeqToBitsConverter.cpp:65-107,
 * src/PositionsBuilder/PositionsBuilder.cpp:15-47,
 * src/IndexSearcher/IndexSearcher.cuh:22-72,
 * src/IndexResultsPrinter/ContinuousIndexResultsPrinter.hpp:196-205):
 *   chars      -- all reads back to back, ASCII (ACGT/acgt valid);
 *   read_ends  -- cumulative exclusive end of each read in chars;
 *   results    -- for every read in order, for every k-mer start in it:
 *                 node index, SBWT_NOT_FOUND, or SBWT_INVALID when the k-mer
 *                 holds a char other than ACGTacgt.
 * results_capacity must be >= sbwt_count_kmers(...); *n_results receives the
 * count (with device pointers it is computed on the host from read_ends only
 * when read_ends is host-visible; pass n_results = NULL otherwise).
 * Host-pointer calls are synchronous and pipeline copies and compute over
 * chunks of reads. */
int sbwt_search_reads(const sbwt_index_t *index, const char *chars,
                      uint64_t n_chars, const uint64_t *read_ends,
                      uint64_t n_reads, uint64_t *results,
                      uint64_t results_capacity, uint64_t *n_results,
                      uint32_t flags, void *stream);

/* The fused read search with NO device allocation, for callers that may not
 * allocate device memory: code running while another framework owns the
 * device allocator, serving loops where a cudaMalloc / cudaFree would stall
 * or implicitly synchronize the device, hosts with a fixed memory budget.
 * This entry point has no counterpart in the reference.
 *   - All arrays are device pointers on the index's device (SBWT_DEVICE_POINTERS
 *     is implied); the caller allocates inputs and outputs.  n_results (host,
 *     may be NULL) receives the k-mer count; the call returns when the results
 *     are written (it synchronizes `stream`).
 *   - Scratch is one fixed array of about 9 MiB in the library's device
 *     memory, present on every GPU that loads the library until the process
 *     exits.  At most 8 Mi chars (8388608) and 256 Ki reads (262144) per call;
 *     larger calls fail with SBWT_E_INVALID.
 *   - The first call on a device looks up the array's device address; make
 *     that first call before any stream capture on that device.
 *   - Every call shares the array: calls that overlap on the GPU (several host
 *     threads or streams at once) race and must be serialized by the caller.
 * Results are identical to sbwt_search_reads; the call runs the same read
 * search kernel (the one sbwt_set_table_kernel selects). */
int sbwt_search_reads_noalloc(const sbwt_index_t *index, const char *d_chars,
                              uint64_t n_chars, const uint64_t *d_read_ends,
                              uint64_t n_reads, uint64_t *d_results,
                              uint64_t results_capacity, uint64_t *n_results,
                              uint32_t flags, void *stream);

/* Builds a plain-matrix SBWT of every k-mer of the sequences on `device`
 * (chars back to back, seq_ends cumulative; k-mers with a non-ACGT char are
 * skipped; reverse complements added when add_rc; 2 <= k <= 31) and writes
 * it to out_path in the format sbwt_index_open reads; *n_nodes (optional)
 * receives the node count.  The reference loads indexes built elsewhere
 * (Themisto); this is the project's own builder, on the GPU. */
int sbwt_build_index(const char *chars, uint64_t n_chars, const uint64_t *seq_ends,
                     uint64_t n_seqs, uint32_t k, int add_rc, const char *out_path,
                     int device, uint64_t *n_nodes);

/* Builds a plain-matrix SBWT of every k-mer of the genomes and a Themisto
 * "sdsl-hybrid-v4" .tcolors color index on `device`: the color set of a k-mer
 * is the set of genomes holding it (either strand when add_rc), every k-mer is
 * a key k-mer (d = 1), sets are deduplicated and a set is dense iff its size
 * exceeds n_genomes / 64.  Both files are byte-identical to the project's
 * host builder's.  The reference loads these files (built by Themisto). */
int sbwt_build_colored_index(const char *chars, uint64_t n_chars, const uint64_t *genome_ends,
                             uint64_t n_genomes, uint32_t k, int add_rc, const char *sbwt_path,
                             const char *tcolors_path, int device, uint64_t *n_nodes);
/* Builds (enable != 0; kept when already built) or drops the index's k-mer
 * table: every k-mer of the SBWT (k <= 31) -> its node in an open-addressing
 * hash table (16 bytes per slot, at most half full).  With it, a read k-mer
 * that is not reached by a stream step from the previous k-mer costs one
 * table lookup instead of the presearch lookup and the remaining search steps
 * (src/IndexSearcher/IndexSearcher.cuh:43-59); results are identical.
 * sbwt_index_open builds it when it fits (<= 32 GiB and a quarter of the
 * free device memory).  *table_bytes (optional) receives its size, 0 when
 * absent.  No counterpart in the reference. */
int sbwt_index_set_kmer_table(sbwt_index_t *index, int enable, uint64_t *table_bytes);

/* ------------------------------------------------------------------------ */
/* Colors step                                                               */
/* ------------------------------------------------------------------------ */
typedef struct sbwt_colors sbwt_colors_t;

/* Loads a Themisto "sdsl-hybrid-v4" .tcolors file onto `device`
 * (src/ColorIndexBuilder/ColorIndexBuilder.cpp:23-86,
 *  src/ColorIndexContainer/GpuColorIndexContainer.cpp:13-86).
 * SBWT_E_IO when the file cannot be opened; SBWT_E_FORMAT for a bad magic
 * string, a truncated file, a length the file cannot hold (checked before
 * anything is allocated for it), an int vector wider than 64 bits, or a
 * color set index, sparse color id or dense interval past its array. */
int sbwt_colors_open(const char *tcolors_path, int device, sbwt_colors_t **out);
void sbwt_colors_free(sbwt_colors_t *colors);
uint64_t sbwt_colors_num_colors(const sbwt_colors_t *colors);

/* Builds (enable != 0) or drops the per-node color set table: 8 bytes per
 * SBWT node that resolve an index to its color set in one load instead of the
 * rank over the key k-mer marks, the color set index and the set descriptor
 * that the reference reads (src/ColorSearcher/ColorSearcher.cuh:68-206).
 * Results are identical either way.  sbwt_colors_open builds it when it fits
 * (at most 16 GiB and half the free device memory).  *built (optional)
 * receives 1 when the table is in use.  No counterpart in the reference. */
int sbwt_colors_set_node_table(sbwt_colors_t *colors, int enable, int *built);

/* Per-read color counts, the reference's ColorSearcher::search seam
 * (src/ColorSearcher/ColorSearcher.h:43-48, kernels
 * src/ColorSearcher/ColorSearcher.cuh:68-206 and
 * src/ColorSearcher/ColorPostProcessor.cuh:21-43):
 *   sbwt_idxs   -- found SBWT indexes of all reads back to back;
 *   idx_offsets -- n_reads + 1 offsets into sbwt_idxs;
 *   counts      -- n_reads x num_colors u32: k-mers of the read whose color
 *                  set holds the color. */
int sbwt_color_counts(const sbwt_colors_t *colors, const uint64_t *sbwt_idxs,
                      const uint64_t *idx_offsets, uint64_t n_reads,
                      uint32_t *counts, uint32_t flags, void *stream);

/* Pseudoalignment: counts + the tau threshold of the reference's printer
 * (src/ColorResultsPrinter/ContinuousColorResultsPrinter.hpp:235-263):
 *   size = found + [SBWT_INCLUDE_NOT_FOUND] not_found + [SBWT_INCLUDE_INVALID]
 *          invalid;  minimum = (u64)ceil((double)size * tau);
 *   a read lists every color (ascending) whose count >= minimum, none when
 *   minimum == 0.
 * not_found / invalid: per-read counts (may be NULL when the matching flag is
 * off).  Output: ids[ids_offsets[r] .. ids_offsets[r+1]) (u32 color ids).
 * If ids_capacity is too small the call returns SBWT_E_CAPACITY with the
 * offsets filled in (ids_offsets[n_reads] = required size). */
int sbwt_pseudoalign(const sbwt_colors_t *colors, const uint64_t *sbwt_idxs,
                     const uint64_t *idx_offsets, const uint64_t *not_found,
                     const uint64_t *invalid, uint64_t n_reads, double tau,
                     uint32_t flags, uint32_t *ids, uint64_t ids_capacity,
                     uint64_t *ids_offsets, void *stream);

/* ------------------------------------------------------------------------ */
/* Batched pipelines and the serving loop (no counterpart in the reference:  */
/* the reference runs one synchronous copy-kernel-copy per batch per stream,  */
/* src/IndexSearcher/IndexSearcher.cpp:26-51)                                */
/* ------------------------------------------------------------------------ */
typedef struct sbwt_pipeline sbwt_pipeline_t;
typedef struct sbwt_server sbwt_server_t;

/* A reusable device pipeline for batches of up to max_chars chars and
 * max_reads reads: its own device buffers, pinned staging and stream.  Each
 * batch (H2D -> index step -> colors step when `colors` is not NULL -> D2H)
 * runs as one CUDA graph with no host synchronisation inside, captured per
 * batch and applied to the instantiated graph with cudaGraphExecUpdate.  The
 * search kernel is a persistent launch fed by a device work queue. */
int sbwt_pipeline_create(const sbwt_index_t *index, const sbwt_colors_t *colors,
                         uint64_t max_chars, uint64_t max_reads, uint32_t flags,
                         double tau, sbwt_pipeline_t **out);
void sbwt_pipeline_free(sbwt_pipeline_t *p);
/* Runs one batch (host pointers; synchronous).  Without colors: results per
 * k-mer as sbwt_search_reads.  With colors: ids / ids_offsets as
 * sbwt_pseudoalign (tau and flags from sbwt_pipeline_create). */
int sbwt_pipeline_run(sbwt_pipeline_t *p, const char *chars, uint64_t n_chars,
                      const uint64_t *read_ends, uint64_t n_reads,
                      uint64_t *results, uint64_t results_capacity,
                      uint64_t *n_results, uint32_t *ids, uint64_t ids_capacity,
                      uint64_t *ids_offsets);

/* A serving loop over resident indexes: up to `slots` pipelines of
 * batch_chars / batch_reads (shrunk at creation until one fits in half of the
 * free device memory).  Requests of any size are accepted from any thread; a
 * background thread keeps every open slot busy with the pending requests in
 * arrival order (continuous batching: a request arriving while batches run
 * joins the next free slot and runs concurrently with them; a large request
 * is split over several batches).  Admission by free device memory: a slot
 * opens only while the device keeps a slot's bytes free above a reserve of an
 * eighth of its memory (so other tenants of the GPU keep their headroom):
 * at creation the first slot and as many more as fit; later, when batches
 * wait, every open slot is busy and memory has freed up, one more at a time
 * (built on a helper thread); otherwise the batch waits for a running slot.
 * Results are identical to the single calls. */
int sbwt_server_create(const sbwt_index_t *index, const sbwt_colors_t *colors,
                       uint64_t batch_chars, uint64_t batch_reads, int slots,
                       uint32_t flags, double tau, sbwt_server_t **out);
void sbwt_server_free(sbwt_server_t *s);
int sbwt_server_submit(sbwt_server_t *s, const char *chars, uint64_t n_chars,
                       const uint64_t *read_ends, uint64_t n_reads,
                       uint64_t *request_id);
/* Waits up to timeout_ms (< 0: forever; SBWT_E_TIMEOUT if not done) for a
 * request and hands its results over (malloc'ed; sbwt_free):
 *   index mode:  *values (n_values k-mer results), *offsets per read;
 *   colors mode: *ids (n_ids color ids), *offsets per read. */
int sbwt_server_wait(sbwt_server_t *s, uint64_t request_id, double timeout_ms,
                     uint64_t **values, uint64_t *n_values, uint32_t **ids,
                     uint64_t *n_ids, uint64_t **offsets, uint64_t *n_reads);
/* Latency percentiles (seconds, submit -> results ready) of the requests
 * finished since the last reset, their count, reads and batches done and the
 * elapsed time; reset != 0 starts a new window. */
int sbwt_server_stats(sbwt_server_t *s, double *p50_s, double *p99_s,
                      uint64_t *requests_done, uint64_t *reads_done,
                      uint64_t *batches, double *elapsed_s, int reset);
/* Slots open now, the device bytes one slot holds, and how many times a
 * waiting batch found too little free device memory to open a slot. */
int sbwt_server_slots(sbwt_server_t *s, int *open_slots, uint64_t *slot_bytes,
                      uint64_t *denied);

/* ------------------------------------------------------------------------ */
/* Host I/O in the reference's file formats (no GPU involved)               */
/* ------------------------------------------------------------------------ */
/* Reads every record of a FASTA/FASTQ file (.gz ok) with the reference's
 * record rules (kseq: src/SequenceFileParser/ContinuousSequenceFileParser.cpp
 * :148-156): *chars / *read_ends are malloc'ed, release with sbwt_free. */
int sbwt_fastx_read(const char *path, char **chars, uint64_t *n_chars,
                    uint64_t **read_ends, uint64_t *n_reads);
void sbwt_free(void *p);
/* Parses FASTA/FASTQ text (uncompressed, the bytes of a whole file) on
 * `device` with the same record rules as sbwt_fastx_read (kseq's, as the
 * reference uses them: src/SequenceFileParser/ContinuousSequenceFileParser.cpp
 * :148-156; the reference parses on the host).  Writes the sequence chars of
 * every record back to back into `chars` and each record's end offset into
 * `read_ends`; *n_chars / *n_reads receive the totals, also when the
 * capacities are too small (SBWT_E_CAPACITY; nothing written).  flags:
 * SBWT_DEVICE_POINTERS when text / chars / read_ends are device memory (then
 * `stream` orders the work; the call still returns after it ends), else host
 * memory.  The chars need no more than n_bytes. */
int sbwt_fastx_parse(const char *text, uint64_t n_bytes, char *chars,
                     uint64_t chars_capacity, uint64_t *read_ends,
                     uint64_t ends_capacity, uint64_t *n_chars, uint64_t *n_reads,
                     uint32_t flags, int device, void *stream);
/* Formats index results on `device` into the bytes the reference's printers
 * write for one batch, without the file header: format 0 ascii, 1 binary,
 * 2 bool (src/IndexResultsPrinter/AsciiContinuousIndexResultsPrinter.cpp
 * :50-55 and its binary / bool siblings; the reference formats on the host).
 * results: one u64 per k-mer (SBWT_NOT_FOUND / SBWT_INVALID markers) in read
 * order; read_ends: cumulative read lengths (k-mers per read = len - k + 1).
 * *out_bytes receives the size, also on SBWT_E_CAPACITY.  flags:
 * SBWT_DEVICE_POINTERS for device buffers (a binary `out` 8-byte aligned). */
int sbwt_format_index_results(const uint64_t *results, const uint64_t *read_ends,
                              uint64_t n_reads, uint32_t k, int format, char *out,
                              uint64_t out_capacity, uint64_t *out_bytes,
                              uint32_t flags, int device, void *stream);
/* Formats pseudoalignment results (ids + ids_offsets as sbwt_pseudoalign
 * writes them, offsets starting at 0) on `device`: format 0 ascii, 1 binary,
 * 2 csv rows of num_colors (src/ColorResultsPrinter/
 * AsciiContinuousColorResultsPrinter.cpp:74-79 and its binary / csv siblings;
 * no header or csv title row).  Same conventions as above. */
int sbwt_format_color_results(const uint32_t *ids, const uint64_t *ids_offsets,
                              uint64_t n_reads, uint64_t num_colors, int format,
                              char *out, uint64_t out_capacity, uint64_t *out_bytes,
                              uint32_t flags, int device, void *stream);
/* Writes index results as the reference's printers do
 * (src/IndexResultsPrinter/ printers: format 0 ascii .txt, 1 binary .bin, 2 bool
 * .bool; optional length-prefixed format/version header). */
int sbwt_write_index_results(const char *out_prefix, int format,
                             int write_headers, const uint64_t *results,
                             const uint64_t *read_ends, uint64_t n_reads,
                             uint32_t k);
/* Reads an ascii or binary index-results file back (the colors step's input,
 * src/IndexFileParser/AsciiIndexFileParser.cpp:33-98,
 * BinaryIndexFileParser.cpp:33-69): found indexes per read + -1 / -2 counts.
 * Arrays are malloc'ed (sbwt_free).  SBWT_E_IO when the file cannot be
 * opened, SBWT_E_FORMAT for a bad header.  No GPU involved. */
int sbwt_read_index_results(const char *path, uint64_t **found,
                            uint64_t **offsets, uint64_t **not_found,
                            uint64_t **invalid, uint64_t *n_reads);
/* Writes color results as the reference's printers do
 * (src/ColorResultsPrinter/ printers: format 0 ascii .txt, 1 binary .bin, 2 csv). */
int sbwt_write_color_results(const char *out_prefix, int format,
                             int write_headers, const uint32_t *ids,
                             const uint64_t *ids_offsets, uint64_t n_reads,
                             uint64_t num_colors);

/* ------------------------------------------------------------------------ */
/* Tuning and instrumentation (no counterpart in the reference)              */
/* ------------------------------------------------------------------------ */
/* Process-wide launch configuration used by the search calls (0 = default):
 * presearch depth (<= the handle's), 256-thread blocks per SM, k-mer slots
 * per work tile, chars per chunk of the host-pointer pipeline. */
int sbwt_set_launch_config(uint32_t presearch_letters, uint32_t blocks_per_sm,
                           uint64_t tile, uint64_t chunk_chars);
/* Length of the read search's absent-prefix probe (0 = automatic,
 * 0xFFFFFFFF = off).  Results never depend on it. */
int sbwt_set_probe_length(uint32_t probe_len);
/* Read search kernel of an index with a k-mer table (k <= 31, fewer than
 * 192 * 2^24 nodes, no SBWT_MOVE_TO_KEY_KMER):
 *   0 = the general kernel (table lookups plus presearch walks and
 *       absent-prefix probes);
 *   1 = the table kernel (stream steps, group scans and table lookups only,
 *       with L2 eviction priorities on its loads);
 *   2..5 = the walks kernel (the table kernel's steps, plus the k-mer
 *       filter in front of the table, several tiles per lane with their
 *       loads in flight together, and 32-byte result stores) with
 *       (walks per lane, 256-thread blocks per SM) = (1, 5), (2, 4),
 *       (2, 3), (4, 2);
 *   6 = the k-mers kernel (every k-mer on its own: filter, then table; no
 *       stream steps, all loads of a lane independent);
 *   7 = automatic, the default: 11 when the table and filter take at most
 *       256 MiB, else 17;
 *   8, 9 = the walks kernel without the filter and the staged stores, 1 or 2
 *       walks per lane; 10 = the same with 1 walk and the filter in front of
 *       the table, one k-mer at a time; 11, 12 = the k-mers kernel with 2 or
 *       8 k-mers per lane (6 has 4); 13, 14 = 8 and 10 with the staged
 *       32-byte result stores; 15 = the k-mers kernel with 4 consecutive
 *       k-mer slots per lane (one char window, one 32-byte result store);
 *       16, 17 = 13 with 8 or 16 slots staged per store group; 18 = 14 with
 *       16 slots; 19 = 6 without the filter (every valid k-mer to the
 *       table);
 *   negative = the default.
 * Results never depend on it.  Returns SBWT_E_INVALID above 19. */
int sbwt_set_table_kernel(int mode);
/* The process-wide launch configuration (set by sbwt_set_launch_config,
 * sbwt_set_table_kernel, sbwt_autotune); any pointer may be NULL. */
int sbwt_get_launch_config(uint32_t *presearch_letters, uint32_t *blocks_per_sm,
                           uint64_t *tile, uint64_t *chunk_chars, int *table_kernel,
                           uint32_t *block_threads);
/* Threads per block of the read search kernels: 128 or 256 (the default;
 * 0 = the default).  Results never depend on it. */
int sbwt_set_block_threads(uint32_t threads);
/* Persisting-L2 access-policy window over the index's rank blocks on the
 * search launches (0 = off, the default; 1 = on: sets this context's
 * persisting-L2 size). */
int sbwt_set_l2_window(int enabled);
/* Off by default.  When enabled, every search-kernel launch is timed with
 * CUDA events on its own stream and this library's kernel launches are
 * counted; count_work also counts full searches / streaming steps / rank
 * block sectors of the read search kernel. */
int sbwt_profile_enable(int enabled, int count_work);
/* Random 32-byte-sector gather throughput of `device` over a `bytes` buffer
 * (allocated inside the call), `chains` independent dependent-load chains
 * per thread (1, 2, 4 or 8): the roofline denominator of the search kernels. */
int sbwt_measure_random_sectors(int device, uint64_t bytes, int chains,
                                double *gbs, double *sectors_per_s);
/* Autotuner: times the read search on the first sample_chars chars of a
 * device-resident batch over a first axis, tile size (k-mers per walk work
 * unit) {auto, 64, 256}, blocks per SM in the grid {2, 4, 6, 8} and threads
 * per block {128, 256}, checks that every configuration gives the same results,
 * and makes the fastest the process-wide launch configuration.  The first
 * axis is the read search kernel (sbwt_set_table_kernel 1..6: the table
 * kernel, the walks kernel with 1, 2 or 4 walks per lane, the k-mers
 * kernel) when the index has its k-mer table, else the presearch depth (8 up
 * to the index's); the block size (128 or 256 threads) is swept too.
 * sbwt_get_launch_config reads the choice back. */
int sbwt_autotune(const sbwt_index_t *index, const char *d_chars,
                  uint64_t n_chars, const uint64_t *d_read_ends,
                  uint64_t n_reads, uint64_t sample_chars,
                  uint32_t *best_presearch, uint32_t *best_blocks_per_sm,
                  uint64_t *best_tile, double *best_ms);
/* Reads and resets the totals (any pointer may be NULL).  counters (count
 * mode): presearch lookups, rank-block sectors, suffix-group words, probe
 * iterations, warp iterations, lane load steps, k-mers written without a
 * search, k-mers searched, lane steps of each search path (stream step,
 * presearch of a new k-mer, walk, group scan, k-mer table lookup, probe),
 * distinct paths per warp iteration (summed), and one unused entry. */
int sbwt_profile_read(double *search_ms, uint64_t *search_launches,
                      uint64_t *launches, uint64_t counters[16]);

#ifdef __cplusplus
}
#endif
#endif /* SBWT_B200_H */
