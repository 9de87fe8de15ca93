/*
 * ref_driver.cpp -- drives SBWT-Search's own index-step kernels, compiled for
 * the host from the reference's unmodified sources through the CPU shim in
 * oracle/ref_shim, one kernel "thread" per loop iteration (OpenMP across
 * iterations).  Built by oracle/Makefile into oracle/_ref/libsbwt_ref.so.
 * TEST INFRASTRUCTURE ONLY: used by tests/ as a second checker and by
 * bench.py as the reference CPU arm.
 *
 * Functions driven:
 *   PoppyBuilder::get_poppy      src/PoppyBuilder/PoppyBuilder.cpp:20-40
 *   d_presearch                  src/Presearcher/Presearcher.cuh:19-41
 *   d_search<move_to_key_kmer>   src/IndexSearcher/IndexSearcher.cuh:22-72
 */
#include <omp.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "IndexSearcher/IndexSearcher.cuh"
#include "PoppyBuilder/PoppyBuilder.h"
#include "Presearcher/Presearcher.cuh"

thread_local shim_dim3 blockIdx = {0, 0, 0};
thread_local shim_dim3 blockDim = {1, 1, 1};
thread_local shim_dim3 threadIdx = {0, 0, 0};

// u64 comes from the reference's Tools/TypeDefinitions.h (global namespace).

extern "C" {

/* Sizes of the Poppy layers for num_bits bits, each with one sentinel entry
 * appended (the reference kernel reads layer_1_2[N / 1024] for rank(N)). */
void ref_poppy_sizes(u64 num_bits, u64 *n_layer0, u64 *n_layer12) {
  *n_layer0 = num_bits / sbwt_search::hyperblock_bits + 1;
  *n_layer12 = num_bits / sbwt_search::superblock_bits + 1;
}

/* Runs the reference PoppyBuilder; writes both layers (plus the sentinel
 * entries) and returns total_1s. */
u64 ref_poppy_build(u64 *bits, u64 num_bits, u64 *layer0, u64 *layer12) {
  u64 n_words = (num_bits + 63) / 64;
  sbwt_search::PoppyBuilder builder({bits, n_words}, num_bits);
  sbwt_search::Poppy poppy = builder.get_poppy();
  u64 n0 = 0, n12 = 0;
  ref_poppy_sizes(num_bits, &n0, &n12);
  for (u64 i = 0; i < n0; ++i)
    layer0[i] = i < poppy.layer_0.size() ? poppy.layer_0[i] : poppy.total_1s;
  for (u64 i = 0; i < n12; ++i) {
    if (i < poppy.layer_1_2.size()) {
      layer12[i] = poppy.layer_1_2[i];
    } else {
      /* rank(N) sentinel: ones since the hyperblock start, no basic blocks */
      u64 before_hyper = layer0[(i * 1024) / sbwt_search::hyperblock_bits];
      layer12[i] = (poppy.total_1s - before_hyper) << 32;
    }
  }
  return poppy.total_1s;
}

/* d_presearch over all 4^12 12-mers (the reference's compile-time depth). */
void ref_presearch(const u64 *c_map, const u64 *const *acgt,
                   const u64 *const *l0, const u64 *const *l12, u64 *left,
                   u64 *right, int threads) {
  const long n = 1L << (sbwt_search::presearch_letters * 2);
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long i = 0; i < n; ++i) {
    blockIdx.x = 0;
    blockDim.x = 1;
    threadIdx.x = (unsigned)i;
    sbwt_search::d_presearch(c_map, acgt, l0, l12, left, right);
  }
}

/* d_search over n k-mer positions.  bit_seqs must hold one word past the
 * last packed char (the kernel reads the following word of every window). */
void ref_search(unsigned kmer_size, const u64 *c_map, const u64 *const *acgt,
                const u64 *const *l0, const u64 *const *l12,
                const u64 *pre_left, const u64 *pre_right,
                const u64 *positions, const u64 *bit_seqs,
                const u64 *key_kmer_marks, u64 n, u64 *out, int threads) {
#pragma omp parallel for schedule(dynamic, 4096) num_threads(threads)
  for (long i = 0; i < (long)n; ++i) {
    /* every launch sets the whole index: OpenMP threads are shared with the
     * colors driver, which launches with other block shapes */
    blockIdx.x = 0;
    blockDim.x = 1;
    threadIdx.x = (unsigned)i;
    if (key_kmer_marks)
      sbwt_search::d_search<true>(kmer_size, c_map, acgt, l0, l12, pre_left,
                                  pre_right, positions, bit_seqs,
                                  key_kmer_marks, out);
    else
      sbwt_search::d_search<false>(kmer_size, c_map, acgt, l0, l12, pre_left,
                                   pre_right, positions, bit_seqs,
                                   key_kmer_marks, out);
  }
}

int ref_max_threads(void) { return omp_get_max_threads(); }
}
