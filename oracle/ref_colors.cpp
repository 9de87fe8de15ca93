/*
 * ref_colors.cpp -- drives SBWT-Search's own colors-step kernels, compiled
 * for the host from the reference's unmodified sources through the CPU shim
 * in oracle/ref_shim.  Built by oracle/Makefile into oracle/_ref/libsbwt_ref.so
 * next to ref_driver.cpp.  TEST INFRASTRUCTURE ONLY: tests/ use it to pin the
 * colors oracle (oracle/sbwt_oracle.c) and the CUDA colors path to the
 * reference's own code.
 *
 * Functions driven:
 *   d_color_search   src/ColorSearcher/ColorSearcher.cuh:68-206 (+ helpers :208-318)
 *   d_post_process   src/ColorSearcher/ColorPostProcessor.cuh:21-43
 *
 * d_color_search is warp-synchronous: a warp reduces its min and max color
 * with __shfl_xor_sync and counts every color with __ballot_sync, all with a
 * full mask.  Here the 32 lanes of one warp are fibers (ucontext) on one host
 * thread.  A lane runs until its next collective, posts its operand and
 * yields; the scheduler runs lanes 0..31 in turn, so once lane 31 has yielded
 * every lane has posted, and each lane then reads all 32 operands when it
 * resumes.  Collectives alternate between two operand buffers, so a lane that
 * runs ahead to the next collective never overwrites operands that a later
 * lane has yet to read.  OpenMP runs different warps on different threads.
 *
 * Inputs must hold no padding lanes: every index of every warp is a found
 * index.  The reference lets a lane whose index is -1 return before the
 * full-mask collectives (ColorSearcher.cuh:98), which is undefined in CUDA;
 * the driver reports a warp where some lanes finish while others wait in a
 * collective as an error instead of guessing a value.
 */
#include <omp.h>
#include <ucontext.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "ColorSearcher/ColorPostProcessor.cuh"
#include "ColorSearcher/ColorSearcher.cuh"

namespace {

struct ColorArgs {
  const u64 *sbwt_idxs;
  const u64 *key_marks, *key_l0, *key_l12;
  const u64 *color_set_idxs;
  u32 color_set_idxs_width;
  const u64 *is_dense, *is_dense_l0, *is_dense_l12;
  const u64 *dense_arrays;
  const u64 *dense_intervals;
  u32 dense_intervals_width;
  const u64 *sparse_arrays;
  u32 sparse_arrays_width;
  const u64 *sparse_intervals;
  u32 sparse_intervals_width;
  u64 num_colors;
  u8 *fat;
};

u64 low_bits(u32 width) { return width >= 64 ? ~0ULL : ((1ULL << width) - 1ULL); }

constexpr size_t kStack = 256 * 1024;

struct Warp {
  ucontext_t sched;
  ucontext_t lane[32];
  std::vector<char> stacks;
  unsigned long long ops[2][32];
  unsigned gen[32];
  bool finished[32];
  unsigned cur = 0;
  unsigned warp = 0;
  const ColorArgs *args = nullptr;
  Warp() : stacks(kStack * 32) {}
};

thread_local Warp *tw = nullptr;

void lane_entry() {
  Warp *w = tw;
  const ColorArgs &a = *w->args;
  sbwt_search::d_color_search(
      a.sbwt_idxs, a.key_marks, a.key_l0, a.key_l12, a.color_set_idxs,
      a.color_set_idxs_width, low_bits(a.color_set_idxs_width), a.is_dense,
      a.is_dense_l0, a.is_dense_l12, a.dense_arrays, a.dense_intervals,
      a.dense_intervals_width, low_bits(a.dense_intervals_width), a.sparse_arrays,
      a.sparse_arrays_width, low_bits(a.sparse_arrays_width), a.sparse_intervals,
      a.sparse_intervals_width, low_bits(a.sparse_intervals_width), a.num_colors,
      a.fat);
  w->finished[w->cur] = true;
  /* returning resumes uc_link (the scheduler) */
}

/* Runs warp `warp` of the launch to completion; false if its lanes did not
 * all take the same collectives (padding lanes, undefined in CUDA). */
bool run_warp(Warp &w, unsigned warp) {
  w.warp = warp;
  for (unsigned l = 0; l < 32; ++l) {
    w.gen[l] = 0;
    w.finished[l] = false;
    getcontext(&w.lane[l]);
    w.lane[l].uc_stack.ss_sp = w.stacks.data() + l * kStack;
    w.lane[l].uc_stack.ss_size = kStack;
    w.lane[l].uc_link = &w.sched;
    makecontext(&w.lane[l], lane_entry, 0);
  }
  while (true) {
    for (unsigned l = 0; l < 32; ++l) {
      if (w.finished[l]) continue;
      w.cur = l;
      blockDim.x = 32;
      blockIdx.x = warp;
      threadIdx.x = l;
      swapcontext(&w.sched, &w.lane[l]);
    }
    unsigned n_fin = 0;
    for (unsigned l = 0; l < 32; ++l) n_fin += w.finished[l];
    if (n_fin == 32) return true;
    if (n_fin != 0) return false;  /* some lanes left, others wait */
    for (unsigned l = 1; l < 32; ++l)
      if (w.gen[l] != w.gen[0]) return false;
  }
}

}  // namespace

const unsigned long long *shim_warp_exchange(unsigned long long v) {
  Warp *w = tw;
  const unsigned l = w->cur;
  const unsigned b = w->gen[l]++ & 1u;
  w->ops[b][l] = v;
  swapcontext(&w->lane[l], &w->sched);
  return w->ops[b];
}

unsigned shim_lane_id() { return tw->cur; }

extern "C" {

/* The reference colors step over one batch: d_color_search over n_idxs
 * warped indexes (n_idxs a multiple of 32, no -1 padding), fat results
 * zeroed first as ColorSearcher.cu:27-29 does, then d_post_process over
 * n_reads reads with warp_intervals[n_reads + 1] (warps before each read).
 * counts receives n_reads * num_colors u64.  Bit vectors need their Poppy
 * layers from ref_poppy_build and one 256-bit basic block of zero padding;
 * variable-width arrays one word of padding.  Returns 0, or -1 when a warp
 * held lanes that left before a collective. */
int ref_color_counts(const u64 *sbwt_idxs, u64 n_idxs, const u64 *key_marks,
                     const u64 *key_l0, const u64 *key_l12, const u64 *color_set_idxs,
                     u32 color_set_idxs_width, const u64 *is_dense, const u64 *is_dense_l0,
                     const u64 *is_dense_l12, const u64 *dense_arrays,
                     const u64 *dense_intervals, u32 dense_intervals_width,
                     const u64 *sparse_arrays, u32 sparse_arrays_width,
                     const u64 *sparse_intervals, u32 sparse_intervals_width,
                     u64 num_colors, const u64 *warp_intervals, u64 n_reads, u64 *counts,
                     int threads) {
  if (n_idxs % 32 != 0) return -1;
  const u64 n_warps = n_idxs / 32;
  std::vector<u8> fat(n_warps * num_colors + 1, 0);
  ColorArgs a{sbwt_idxs,        key_marks,       key_l0,
              key_l12,          color_set_idxs,  color_set_idxs_width,
              is_dense,         is_dense_l0,     is_dense_l12,
              dense_arrays,     dense_intervals, dense_intervals_width,
              sparse_arrays,    sparse_arrays_width, sparse_intervals,
              sparse_intervals_width, num_colors, fat.data()};
  int bad = 0;
#pragma omp parallel num_threads(threads) reduction(| : bad)
  {
    Warp *w = new Warp();
    w->args = &a;
    tw = w;
#pragma omp for schedule(dynamic, 1)
    for (long wi = 0; wi < (long)n_warps; ++wi)
      if (!run_warp(*w, (unsigned)wi)) bad = 1;
    tw = nullptr;
    delete w;
  }
  if (bad) return -1;
  const u64 n = n_reads * num_colors;
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long t = 0; t < (long)n; ++t) {
    blockDim.x = 1024;
    blockIdx.x = (unsigned)(t / 1024);
    threadIdx.x = (unsigned)(t % 1024);
    sbwt_search::d_post_process(fat.data(), warp_intervals, n_reads, num_colors, counts);
  }
  return 0;
}
}
