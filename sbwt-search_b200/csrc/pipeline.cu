// Batched pipelines and the serving loop.
//
// A Pipeline owns device buffers for batches of up to max_chars chars and
// max_reads reads, pinned host staging, a stream and a CUDA graph.  One batch
// = H2D copies -> index step (scan, pack, tile table, persistent search
// kernel with a device work queue) -> optional colors step (per-read
// counting, threshold, ids) -> D2H copies, enqueued without any host
// synchronisation and captured as a CUDA graph; the executable graph is
// updated in place for the next batch (cudaGraphExecUpdate) and re-made only
// when its shape changes.
//
// The Server keeps an index (and a color index) resident, accepts requests
// of any size from any thread, and keeps `slots` pipelines busy: whenever a
// pipeline is free it takes the pending requests in arrival order (splitting
// a request that does not fit) and launches them as one batch, so requests
// that arrive while others run are admitted as soon as a slot frees and run
// concurrently on the device with the batches already in flight.  Per-request
// latency (submit -> results ready) is recorded for p50 / p99.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "colors_internal.hpp"
#include "common.hpp"
#include "index_internal.hpp"

namespace sbwt {

struct PipelineImpl {
  const IndexImpl *ix;
  const ColorsImpl *ci;
  u64 max_chars, max_reads, ids_capacity;
  u32 flags;
  double tau;
  LaunchConfig cfg;
  int device;
  DeviceBuffer d_chars, d_ends, d_results, kmer_off, packed, invalid, block_sums, total,
      tile_read, err, queue, pass_bits, pass_count, ids_off, ids;
  char *h_chars = nullptr;
  u64 *h_ends = nullptr, *h_results = nullptr, *h_ids_off = nullptr, *h_total = nullptr;
  uint32_t *h_ids = nullptr, *h_err = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaGraphExec_t exec = nullptr;
  // current batch
  u64 n_chars = 0, n_reads = 0, n_kmers = 0, max_read_kmers = 0;

  PipelineImpl(const IndexImpl *ix_, const ColorsImpl *ci_, u64 max_chars_, u64 max_reads_,
               u32 flags_, double tau_)
      : ix(ix_), ci(ci_), max_chars(max_chars_), max_reads(max_reads_), flags(flags_),
        tau(tau_), cfg(default_launch_config()), device(ix_->device) {
    if (max_chars == 0 || max_reads == 0) throw Error(SBWT_E_INVALID, "empty pipeline");
    DeviceGuard g(device);
    const u64 n_words = (max_chars + 31) / 32;
    d_chars.resize(max_chars + 16);
    d_ends.resize(max_reads * 8);
    d_results.resize(max_chars * 8);
    kmer_off.resize((max_reads + 1) * 8);
    packed.resize((n_words + 2) * 8);
    invalid.resize((n_words + 2) * 4);
    block_sums.resize(((max_reads + 4095) / 4096 + 1) * 8);
    total.resize(8);
    tile_read.resize((max_chars / index_tile_size(*ix, max_chars, cfg) + 2) * 8);
    err.resize(8);
    queue.resize(8);
    SBWT_CUDA(cudaMallocHost(&h_chars, max_chars + 16));
    SBWT_CUDA(cudaMallocHost(&h_ends, max_reads * 8));
    SBWT_CUDA(cudaMallocHost(&h_total, 8));
    SBWT_CUDA(cudaMallocHost(&h_err, 8));
    if (ci) {
      const u64 rw = (ci->num_colors + 63) / 64;
      ids_capacity = max_reads * 64;
      pass_bits.resize(max_reads * rw * 8);
      pass_count.resize(max_reads * 4);
      ids_off.resize((max_reads + 1) * 8);
      ids.resize(ids_capacity * 4);
      SBWT_CUDA(cudaMallocHost(&h_ids_off, (max_reads + 1) * 8));
      SBWT_CUDA(cudaMallocHost(&h_ids, ids_capacity * 4));
    } else {
      ids_capacity = 0;
      SBWT_CUDA(cudaMallocHost(&h_results, max_chars * 8));
    }
    SBWT_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    SBWT_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
  }

  ~PipelineImpl() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (done) cudaEventDestroy(done);
    if (stream) cudaStreamDestroy(stream);
    for (void *p : {(void *)h_chars, (void *)h_ends, (void *)h_results, (void *)h_ids_off,
                    (void *)h_total, (void *)h_ids, (void *)h_err})
      if (p) cudaFreeHost(p);
    cudaSetDevice(prev);
  }

  // Host side of a batch: the staged chars / ends are already in h_chars /
  // h_ends (ends relative to the batch); computes the k-mer counts.
  void set_batch(u64 nc, u64 nr) {
    if (nc > max_chars || nr > max_reads) throw Error(SBWT_E_INVALID, "batch exceeds pipeline");
    n_chars = nc;
    n_reads = nr;
    n_kmers = 0;
    max_read_kmers = 0;
    u64 prev = 0;
    for (u64 r = 0; r < nr; ++r) {
      if (h_ends[r] < prev || h_ends[r] > nc)
        throw Error(SBWT_E_INVALID, "read_ends must be non-decreasing within n_chars");
      const u64 len = h_ends[r] - prev;
      const u64 m = len >= ix->k ? len - ix->k + 1 : 0;
      n_kmers += m;
      max_read_kmers = std::max(max_read_kmers, m);
      prev = h_ends[r];
    }
  }

  void enqueue() {
    cudaStream_t st = stream;
    if (n_chars) SBWT_CUDA(cudaMemcpyAsync(d_chars.get(), h_chars, n_chars, cudaMemcpyHostToDevice, st));
    if (n_reads) SBWT_CUDA(cudaMemcpyAsync(d_ends.get(), h_ends, n_reads * 8, cudaMemcpyHostToDevice, st));
    ReadsScratch sc{kmer_off.get<u64>(), packed.get<u64>(), invalid.get<uint32_t>(),
                    block_sums.get<u64>(), total.get<u64>(), tile_read.get<u64>(),
                    err.get<uint32_t>(), queue.get<unsigned long long>()};
    enqueue_index_step(*ix, d_chars.get<char>(), n_chars, d_ends.get<u64>(), n_reads, sc,
                       d_results.get<u64>(), max_chars, max_chars, flags, cfg, st);
    if (ci) {
      ci->enqueue_pseudoalign(d_results.get<u64>(), kmer_off.get<u64>(), n_reads, max_read_kmers,
                              tau, flags, pass_bits.get<u64>(), pass_count.get<uint32_t>(),
                              ids_off.get<u64>(), ids.get<uint32_t>(), ids_capacity,
                              err.get<uint32_t>(), st);
      SBWT_CUDA(cudaMemcpyAsync(h_ids_off, ids_off.get(), (n_reads + 1) * 8,
                                cudaMemcpyDeviceToHost, st));
    } else if (n_kmers) {
      SBWT_CUDA(cudaMemcpyAsync(h_results, d_results.get(), n_kmers * 8,
                                cudaMemcpyDeviceToHost, st));
    }
    SBWT_CUDA(cudaMemcpyAsync(h_total, total.get(), 8, cudaMemcpyDeviceToHost, st));
    SBWT_CUDA(cudaMemcpyAsync(h_err, err.get(), 4, cudaMemcpyDeviceToHost, st));
  }

  // Captures the batch as a graph, updates (or makes) the executable graph and
  // launches it; completion is signalled by `done`.
  void launch() {
    DeviceGuard g(device);
    if (ci) ci->prepare_launch(std::max<u64>(max_read_kmers, 1));
    SBWT_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
    try {
      enqueue();
    } catch (...) {
      cudaGraph_t gph = nullptr;
      cudaStreamEndCapture(stream, &gph);
      if (gph) cudaGraphDestroy(gph);
      throw;
    }
    cudaGraph_t graph = nullptr;
    SBWT_CUDA(cudaStreamEndCapture(stream, &graph));
    bool updated = false;
    if (exec) {
      cudaGraphExecUpdateResultInfo info{};
      updated = cudaGraphExecUpdate(exec, graph, &info) == cudaSuccess;
      if (!updated) {
        cudaGetLastError();
        cudaGraphExecDestroy(exec);
        exec = nullptr;
      }
    }
    if (!updated) {
      const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        throw Error(SBWT_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      }
    }
    cudaGraphDestroy(graph);
    SBWT_CUDA(cudaGraphLaunch(exec, stream));
    SBWT_CUDA(cudaEventRecord(done, stream));
  }

  bool ready() const { return cudaEventQuery(done) == cudaSuccess; }

  // Waits for the batch; copies the ids when the colors step ran.
  void finish() {
    DeviceGuard g(device);
    SBWT_CUDA(cudaEventSynchronize(done));
    if (*h_err & 4u) throw Error(SBWT_E_INVALID, "read_ends are not non-decreasing within n_chars");
    if (*h_err & 1u && !ci)
      throw Error(SBWT_E_TIMEOUT, "key k-mer walk did not reach a key k-mer");
    if (ci && *h_err)
      throw Error(SBWT_E_INVALID, "an SBWT index is not a key k-mer of this color index");
    if (*h_total != n_kmers) throw Error(SBWT_E_CUDA, "k-mer count mismatch");
    if (ci) {
      const u64 n_ids = h_ids_off[n_reads];
      if (n_ids > ids_capacity) {  // rare: more ids than the staging holds
        std::vector<uint32_t> tmp;
        expand_from_bits(tmp);
        return;
      }
      if (n_ids)
        SBWT_CUDA(cudaMemcpyAsync(h_ids, ids.get(), n_ids * 4, cudaMemcpyDeviceToHost, stream));
      SBWT_CUDA(cudaStreamSynchronize(stream));
    }
  }

  // Fallback when a batch passes more ids than ids_capacity: the ids are
  // expanded on the host from the per-read pass bitmasks.
  std::vector<uint32_t> big_ids;
  void expand_from_bits(std::vector<uint32_t> &) {
    const u64 rw = (ci->num_colors + 63) / 64;
    std::vector<u64> bits(n_reads * rw);
    SBWT_CUDA(cudaMemcpy(bits.data(), pass_bits.get(), bits.size() * 8, cudaMemcpyDeviceToHost));
    big_ids.clear();
    h_ids_off[0] = 0;
    for (u64 r = 0; r < n_reads; ++r) {
      for (u64 w = 0; w < rw; ++w) {
        u64 m = bits[r * rw + w];
        while (m) {
          big_ids.push_back((uint32_t)(w * 64 + __builtin_ctzll(m)));
          m &= m - 1;
        }
      }
      h_ids_off[r + 1] = big_ids.size();
    }
  }
  const uint32_t *ids_data() const { return big_ids.empty() ? h_ids : big_ids.data(); }
};

// ---------------------------------------------------------------------------
// Server
// ---------------------------------------------------------------------------
using Clock = std::chrono::steady_clock;

struct Request {
  u64 id;
  std::vector<char> chars;
  std::vector<u64> ends;     // relative to the request
  u64 next_read = 0;         // first read not yet given to a batch
  u64 reads_done = 0;
  std::vector<u64> offs;     // per read output offsets (n_reads + 1), built at the end
  std::vector<u64> out64;    // index mode: results per k-mer
  std::vector<uint32_t> out32;  // colors mode: ids
  // pieces may finish out of order (different slots): results per piece,
  // keyed by its first read, with per-read sizes; assembled when complete
  struct Part {
    std::vector<u64> v64;
    std::vector<uint32_t> v32;
    std::vector<u64> sizes;
  };
  std::map<u64, Part> parts;
  void assemble() {
    offs.assign(ends.size() + 1, 0);
    u64 r = 0;
    for (auto &kv : parts) {
      Part &pt = kv.second;
      out64.insert(out64.end(), pt.v64.begin(), pt.v64.end());
      out32.insert(out32.end(), pt.v32.begin(), pt.v32.end());
      for (u64 sz : pt.sizes) {
        offs[r + 1] = offs[r] + sz;
        ++r;
      }
    }
    parts.clear();
  }
  Clock::time_point t_submit;
  bool complete = false;
  int error = SBWT_OK;
  std::string error_msg;
};

struct Piece {  // reads [r0, r1) of a request inside a batch, from batch read b0
  Request *req;
  u64 r0, r1, b0;
};

struct ServerImpl {
  const IndexImpl *ix;
  const ColorsImpl *ci;
  std::vector<std::unique_ptr<PipelineImpl>> slots;
  std::vector<std::vector<Piece>> slot_pieces;
  std::vector<bool> busy;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> pending;
  std::map<u64, std::unique_ptr<Request>> requests;
  std::vector<double> latencies;
  u64 next_id = 1, reads_done = 0, batches = 0;
  std::atomic<bool> stop{false};
  std::thread worker;
  Clock::time_point t0 = Clock::now();

  // Admission by free device memory.  A slot (one pipeline: its device
  // buffers and CUDA graph) holds about slot_bytes.  The server opens its
  // first slot at creation (shrunk until it fits in half of the free
  // memory) and opens more, up to max_slots, only while batches are waiting
  // and the device still has slot_bytes free above a reserve of an eighth of
  // its memory; otherwise waiting batches queue for a running slot.
  u64 slot_chars_ = 0, slot_reads_ = 0, slot_bytes = 0;
  u32 flags_ = 0;
  double tau_ = 0;
  int max_slots = 1;
  u64 denied = 0;  // times a waiting batch found no free memory for a slot (under mu)
  // A slot is built on a helper thread (device buffers, pinned buffers: a
  // few milliseconds) while the open slots keep serving; the worker adopts
  // it once built.
  std::thread creator;
  bool creating = false;                 // under mu
  std::unique_ptr<PipelineImpl> fresh;  // built, not yet adopted (under mu)

  static double slot_size(const ColorsImpl *ci, u64 chars, u64 reads) {
    const double per_char = 1 + 8 + 0.375 + 1.0 / 16 + 1;  // chars, results, packing, tiles
    const double per_read = 8 * 2 + (ci ? (ci->num_colors / 8.0 + 4 + 8 + 64 * 4) : 0);
    return chars * per_char + reads * per_read;
  }

  ServerImpl(const IndexImpl *ix_, const ColorsImpl *ci_, u64 slot_chars, u64 slot_reads,
             int n_slots, u32 flags, double tau)
      : ix(ix_), ci(ci_) {
    if (n_slots < 1 || n_slots > 8) throw Error(SBWT_E_INVALID, "slots must be 1..8");
    DeviceGuard g(ix->device);
    size_t free_b = 0, total_b = 0;
    SBWT_CUDA(cudaMemGetInfo(&free_b, &total_b));
    while (slot_size(ci, slot_chars, slot_reads) > 0.5 * (double)free_b &&
           slot_chars > (1u << 20)) {
      slot_chars /= 2;
      slot_reads = std::max<u64>(slot_reads / 2, 1024);
    }
    slot_chars_ = slot_chars;
    slot_reads_ = slot_reads;
    slot_bytes = (u64)slot_size(ci, slot_chars, slot_reads);
    flags_ = flags;
    tau_ = tau;
    max_slots = n_slots;
    slots.emplace_back(std::make_unique<PipelineImpl>(ix, ci, slot_chars, slot_reads, flags, tau));
    // more slots now while each leaves the reserve free (building one while
    // batches run stalls them for milliseconds, so slots that fit are built
    // up front; later ones only when memory was short here)
    while ((int)slots.size() < n_slots) {
      SBWT_CUDA(cudaMemGetInfo(&free_b, &total_b));
      if ((double)free_b < (double)slot_bytes + (double)total_b / 8) break;
      slots.emplace_back(
          std::make_unique<PipelineImpl>(ix, ci, slot_chars, slot_reads, flags, tau));
    }
    slot_pieces.resize(slots.size());
    busy.assign(slots.size(), false);
    worker = std::thread([this] { run(); });
  }

  // Starts building one more slot when batches wait, every slot is busy and
  // the device has room for it; called by the worker thread only.
  void admit_slot() {
    {
      std::lock_guard<std::mutex> lk(mu);
      if (creating || fresh || (int)slots.size() >= max_slots) return;
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    std::lock_guard<std::mutex> lk(mu);
    if ((double)free_b < (double)slot_bytes + (double)total_b / 8) {
      ++denied;
      return;
    }
    creating = true;
    if (creator.joinable()) creator.join();  // the previous build has finished
    creator = std::thread([this] {
      std::unique_ptr<PipelineImpl> p;
      try {
        DeviceGuard g(ix->device);
        p = std::make_unique<PipelineImpl>(ix, ci, slot_chars_, slot_reads_, flags_, tau_);
      } catch (const Error &) {
        p.reset();  // the allocation failed after all: keep serving on the open slots
      }
      std::lock_guard<std::mutex> lk2(mu);
      if (p)
        fresh = std::move(p);
      else
        ++denied;
      creating = false;
      cv_work.notify_all();
    });
  }

  // Adopts a slot the helper thread has built; worker thread only.
  void adopt_slot() {
    std::lock_guard<std::mutex> lk(mu);
    if (!fresh) return;
    slots.push_back(std::move(fresh));
    slot_pieces.emplace_back();
    busy.push_back(false);
  }

  ~ServerImpl() {
    stop = true;
    cv_work.notify_all();
    if (worker.joinable()) worker.join();
    if (creator.joinable()) creator.join();
  }

  u64 submit(const char *chars, u64 n_chars, const u64 *ends, u64 n_reads) {
    auto r = std::make_unique<Request>();
    r->chars.assign(chars, chars + n_chars);
    r->ends.assign(ends, ends + n_reads);
    u64 prev = 0;
    for (u64 e : r->ends) {
      if (e < prev || e > n_chars) throw Error(SBWT_E_INVALID, "read_ends must be non-decreasing within n_chars");
      prev = e;
    }
    r->offs.assign(n_reads + 1, 0);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> g(mu);
    r->id = next_id++;
    const u64 id = r->id;
    if (n_reads == 0) {
      r->complete = true;
      latencies.push_back(0.0);
    } else {
      pending.push_back(r.get());
    }
    requests[id] = std::move(r);
    cv_work.notify_one();
    return id;
  }

  // Fills slot s from the pending requests; returns false when there is nothing.
  bool fill(int s) {
    PipelineImpl &p = *slots[s];
    auto &pieces = slot_pieces[s];
    pieces.clear();
    u64 nc = 0, nr = 0;
    while (!pending.empty()) {
      Request *q = pending.front();
      const u64 base = q->next_read ? q->ends[q->next_read - 1] : 0;
      u64 r1 = q->next_read;
      // as many whole reads of q as fit
      while (r1 < q->ends.size() && nr + (r1 - q->next_read) < p.max_reads &&
             nc + (q->ends[r1] - base) <= p.max_chars)
        ++r1;
      if (r1 == q->next_read) {
        if (nr == 0) {  // a single read larger than a slot
          q->error = SBWT_E_INVALID;
          q->error_msg = "a read is longer than the server's batch size";
          q->complete = true;
          pending.pop_front();
          continue;
        }
        break;
      }
      const u64 nchars_q = q->ends[r1 - 1] - base;
      std::memcpy(p.h_chars + nc, q->chars.data() + base, nchars_q);
      for (u64 r = q->next_read; r < r1; ++r) p.h_ends[nr + (r - q->next_read)] = nc + (q->ends[r] - base);
      pieces.push_back(Piece{q, q->next_read, r1, nr});
      nc += nchars_q;
      nr += r1 - q->next_read;
      q->next_read = r1;
      if (r1 == q->ends.size()) pending.pop_front();
      if (nr >= p.max_reads || nc >= p.max_chars) break;
    }
    if (pieces.empty()) return false;
    p.set_batch(nc, nr);
    return true;
  }

  void deliver(int s) {
    PipelineImpl &p = *slots[s];
    int err = SBWT_OK;
    std::string msg;
    try {
      p.finish();
    } catch (const Error &e) {
      err = e.code;
      msg = e.what();
    }
    std::lock_guard<std::mutex> g(mu);
    const auto now = Clock::now();
    for (const Piece &pc : slot_pieces[s]) {
      Request *q = pc.req;
      if (err != SBWT_OK) {
        q->error = err;
        q->error_msg = msg;
      } else if (ci) {
        Request::Part &pt = q->parts[pc.r0];
        const uint32_t *ids = p.ids_data();
        for (u64 r = pc.r0; r < pc.r1; ++r) {
          const u64 b = pc.b0 + (r - pc.r0);
          pt.v32.insert(pt.v32.end(), ids + p.h_ids_off[b], ids + p.h_ids_off[b + 1]);
          pt.sizes.push_back(p.h_ids_off[b + 1] - p.h_ids_off[b]);
        }
      } else {
        Request::Part &pt = q->parts[pc.r0];
        // k-mer results of batch reads [b0, b0 + (r1 - r0))
        u64 kofs = 0;
        for (u64 b = 0; b < pc.b0; ++b) {
          const u64 len = p.h_ends[b] - (b ? p.h_ends[b - 1] : 0);
          kofs += len >= ix->k ? len - ix->k + 1 : 0;
        }
        for (u64 r = pc.r0; r < pc.r1; ++r) {
          const u64 b = pc.b0 + (r - pc.r0);
          const u64 len = p.h_ends[b] - (b ? p.h_ends[b - 1] : 0);
          const u64 m = len >= ix->k ? len - ix->k + 1 : 0;
          pt.v64.insert(pt.v64.end(), p.h_results + kofs, p.h_results + kofs + m);
          pt.sizes.push_back(m);
          kofs += m;
        }
      }
      q->reads_done += pc.r1 - pc.r0;
      reads_done += pc.r1 - pc.r0;
      if (q->reads_done == q->ends.size() || q->error != SBWT_OK) {
        if (!q->complete) {
          if (q->error == SBWT_OK) q->assemble();
          q->complete = true;
          latencies.push_back(std::chrono::duration<double>(now - q->t_submit).count());
        }
      }
    }
    slot_pieces[s].clear();
    busy[s] = false;
    ++batches;
    cv_done.notify_all();
  }

  void run() {
    DeviceGuard g(ix->device);
    while (!stop) {
      bool progressed = false;
      for (size_t s = 0; s < slots.size(); ++s)
        if (busy[s] && slots[s]->ready()) {
          deliver((int)s);
          progressed = true;
        }
      adopt_slot();
      {
        bool all_busy = true, waiting = false;
        for (bool b : busy) all_busy &= b;
        {
          std::lock_guard<std::mutex> lk(mu);
          waiting = !pending.empty();
        }
        if (all_busy && waiting) admit_slot();
      }
      for (size_t s = 0; s < slots.size(); ++s) {
        if (busy[s]) continue;
        bool filled = false;
        {
          std::lock_guard<std::mutex> lk(mu);
          try {
            filled = fill((int)s);
          } catch (const Error &e) {
            for (const Piece &pc : slot_pieces[s]) {
              pc.req->error = e.code;
              pc.req->error_msg = e.what();
              pc.req->complete = true;
            }
            slot_pieces[s].clear();
            cv_done.notify_all();
          }
        }
        if (!filled) break;
        try {
          slots[s]->launch();
          busy[s] = true;
        } catch (const Error &e) {
          std::lock_guard<std::mutex> lk(mu);
          for (const Piece &pc : slot_pieces[s]) {
            pc.req->error = e.code;
            pc.req->error_msg = e.what();
            pc.req->complete = true;
          }
          slot_pieces[s].clear();
          cv_done.notify_all();
        }
        progressed = true;
      }
      if (!progressed) {
        std::unique_lock<std::mutex> lk(mu);
        bool any_busy = false;
        for (bool b : busy) any_busy |= b;
        if (any_busy)
          cv_work.wait_for(lk, std::chrono::microseconds(50));
        else
          cv_work.wait_for(lk, std::chrono::milliseconds(5),
                           [&] { return stop.load() || !pending.empty(); });
      }
    }
    for (size_t s = 0; s < slots.size(); ++s)
      if (busy[s]) deliver((int)s);
  }

  // Waits for request `id` (timeout_ms < 0: forever); moves its results out.
  int wait(u64 id, double timeout_ms, std::unique_ptr<Request> &out) {
    std::unique_lock<std::mutex> lk(mu);
    auto it = requests.find(id);
    if (it == requests.end()) throw Error(SBWT_E_INVALID, "unknown request id");
    Request *q = it->second.get();
    auto pred = [&] { return q->complete; };
    if (timeout_ms < 0) {
      cv_done.wait(lk, pred);
    } else if (!cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred)) {
      return SBWT_E_TIMEOUT;
    }
    out = std::move(it->second);
    requests.erase(it);
    return SBWT_OK;
  }

  void stats(double *p50, double *p99, u64 *n_done, u64 *reads, u64 *n_batches, double *elapsed) {
    std::lock_guard<std::mutex> g(mu);
    std::vector<double> v = latencies;
    std::sort(v.begin(), v.end());
    auto q = [&](double f) {
      if (v.empty()) return 0.0;
      size_t i = (size_t)std::min<double>(v.size() - 1, std::ceil(f * v.size()) - 1);
      return v[i];
    };
    if (p50) *p50 = q(0.50);
    if (p99) *p99 = q(0.99);
    if (n_done) *n_done = v.size();
    if (reads) *reads = reads_done;
    if (n_batches) *n_batches = batches;
    if (elapsed) *elapsed = std::chrono::duration<double>(Clock::now() - t0).count();
  }

  void reset_stats() {
    std::lock_guard<std::mutex> g(mu);
    latencies.clear();
    reads_done = 0;
    batches = 0;
    t0 = Clock::now();
  }
};

}  // namespace sbwt

struct sbwt_pipeline {
  sbwt::PipelineImpl *impl;
};
struct sbwt_server {
  sbwt::ServerImpl *impl;
};

using namespace sbwt;

extern "C" {

int sbwt_pipeline_create(const sbwt_index_t *index, const sbwt_colors_t *colors,
                         uint64_t max_chars, uint64_t max_reads, uint32_t flags, double tau,
                         sbwt_pipeline_t **out) {
  if (!index || !out) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  *out = nullptr;
  return guarded([&] {
    if (colors && colors->impl->device != index->impl->device)
      throw Error(SBWT_E_INVALID, "index and colors live on different devices");
    auto p = std::make_unique<PipelineImpl>(index->impl, colors ? colors->impl : nullptr,
                                            max_chars, max_reads, flags, tau);
    *out = new sbwt_pipeline{p.release()};
  });
}

void sbwt_pipeline_free(sbwt_pipeline_t *p) {
  if (!p) return;
  delete p->impl;
  delete p;
}

int sbwt_pipeline_run(sbwt_pipeline_t *p, const char *chars, uint64_t n_chars,
                      const uint64_t *read_ends, uint64_t n_reads, uint64_t *results,
                      uint64_t results_capacity, uint64_t *n_results, uint32_t *ids,
                      uint64_t ids_capacity, uint64_t *ids_offsets) {
  if (!p || (n_reads && !read_ends) || (n_chars && !chars)) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    PipelineImpl &x = *p->impl;
    if (n_chars > x.max_chars || n_reads > x.max_reads)
      throw Error(SBWT_E_INVALID, "batch larger than the pipeline");
    std::memcpy(x.h_chars, chars, n_chars);
    std::memcpy(x.h_ends, read_ends, n_reads * 8);
    x.set_batch(n_chars, n_reads);
    x.launch();
    x.finish();
    if (n_results) *n_results = x.n_kmers;
    if (x.ci) {
      if (!ids_offsets) throw Error(SBWT_E_INVALID, "ids_offsets needed with a color index");
      std::memcpy(ids_offsets, x.h_ids_off, (n_reads + 1) * 8);
      const u64 n_ids = x.h_ids_off[n_reads];
      if (n_ids > ids_capacity) throw Error(SBWT_E_CAPACITY, "ids_capacity too small");
      if (n_ids) std::memcpy(ids, x.ids_data(), n_ids * 4);
    } else {
      if (x.n_kmers > results_capacity)
        throw Error(SBWT_E_CAPACITY, "results_capacity smaller than the k-mer count");
      if (x.n_kmers) std::memcpy(results, x.h_results, x.n_kmers * 8);
    }
  });
}

int sbwt_server_create(const sbwt_index_t *index, const sbwt_colors_t *colors,
                       uint64_t batch_chars, uint64_t batch_reads, int slots, uint32_t flags,
                       double tau, sbwt_server_t **out) {
  if (!index || !out) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  *out = nullptr;
  return guarded([&] {
    auto s = std::make_unique<ServerImpl>(index->impl, colors ? colors->impl : nullptr,
                                          batch_chars, batch_reads, slots, flags, tau);
    *out = new sbwt_server{s.release()};
  });
}

void sbwt_server_free(sbwt_server_t *s) {
  if (!s) return;
  delete s->impl;
  delete s;
}

int sbwt_server_submit(sbwt_server_t *s, const char *chars, uint64_t n_chars,
                       const uint64_t *read_ends, uint64_t n_reads, uint64_t *request_id) {
  if (!s || !request_id || (n_reads && !read_ends) || (n_chars && !chars)) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] { *request_id = s->impl->submit(chars, n_chars, read_ends, n_reads); });
}

int sbwt_server_wait(sbwt_server_t *s, uint64_t request_id, double timeout_ms,
                     uint64_t **values, uint64_t *n_values, uint32_t **ids, uint64_t *n_ids,
                     uint64_t **offsets, uint64_t *n_reads) {
  if (!s || !offsets || !n_reads) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  int rc = SBWT_OK;
  int g = guarded([&] {
    std::unique_ptr<Request> q;
    rc = s->impl->wait(request_id, timeout_ms, q);
    if (rc != SBWT_OK) return;
    if (q->error != SBWT_OK) {
      rc = q->error;
      set_last_error(q->error_msg);
      return;
    }
    auto dup = [](const void *src, size_t bytes) {
      void *p = std::malloc(std::max<size_t>(bytes, 1));
      if (!p) throw std::bad_alloc();
      if (bytes) std::memcpy(p, src, bytes);
      return p;
    };
    *offsets = static_cast<uint64_t *>(dup(q->offs.data(), q->offs.size() * 8));
    *n_reads = q->ends.size();
    if (values) *values = static_cast<uint64_t *>(dup(q->out64.data(), q->out64.size() * 8));
    if (n_values) *n_values = q->out64.size();
    if (ids) *ids = static_cast<uint32_t *>(dup(q->out32.data(), q->out32.size() * 4));
    if (n_ids) *n_ids = q->out32.size();
  });
  if (g != SBWT_OK) return g;
  if (rc == SBWT_E_TIMEOUT) set_last_error("request not finished before the timeout");
  return rc;
}

int sbwt_server_stats(sbwt_server_t *s, double *p50_s, double *p99_s, uint64_t *requests_done,
                      uint64_t *reads_done, uint64_t *batches, double *elapsed_s, int reset) {
  if (!s) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  s->impl->stats(p50_s, p99_s, requests_done, reads_done, batches, elapsed_s);
  if (reset) s->impl->reset_stats();
  return SBWT_OK;
}

int sbwt_server_slots(sbwt_server_t *s, int *open_slots, uint64_t *slot_bytes,
                      uint64_t *denied) {
  if (!s) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  std::lock_guard<std::mutex> g(s->impl->mu);
  if (open_slots) *open_slots = (int)s->impl->slots.size();
  if (slot_bytes) *slot_bytes = s->impl->slot_bytes;
  if (denied) *denied = s->impl->denied;
  return SBWT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner
// ---------------------------------------------------------------------------
extern "C" {
// Times the read search (device-resident inputs, the first reads of the given
// batch up to sample_chars chars) over presearch depths 8..12 (not above the
// index's), tile sizes {64, 256, 1024, auto} and 256-thread blocks per SM
// {2, 3, 4, 6, 8}; every configuration must reproduce the first run's
// results.  The fastest becomes the process-wide launch configuration and is
// written to *best (presearch, blocks_per_sm, tile) with its time in ms.
int sbwt_autotune(const sbwt_index_t *index, const char *d_chars, uint64_t n_chars,
                  const uint64_t *d_read_ends, uint64_t n_reads, uint64_t sample_chars,
                  uint32_t *best_presearch, uint32_t *best_blocks_per_sm,
                  uint64_t *best_tile, double *best_ms) {
  if (!index || !d_chars || !d_read_ends || !n_reads) {
    set_last_error("null argument");
    return SBWT_E_INVALID;
  }
  return guarded([&] {
    const IndexImpl &ix = *index->impl;
    DeviceGuard g(ix.device);
    // sample: the reads whose ends are within sample_chars
    std::vector<u64> ends(n_reads);
    SBWT_CUDA(cudaMemcpy(ends.data(), d_read_ends, n_reads * 8, cudaMemcpyDeviceToHost));
    u64 nr = 0;
    while (nr < n_reads && ends[nr] <= std::min<u64>(sample_chars, n_chars)) ++nr;
    if (nr == 0) nr = 1;
    const u64 nc = ends[nr - 1];
    const u64 nk = count_kmers_host(ends.data(), nr, ix.k, 0);
    DeviceBuffer out(std::max<u64>(nk, 1) * 8), ref(std::max<u64>(nk, 1) * 8);
    cudaStream_t st;
    SBWT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    SBWT_CUDA(cudaEventCreate(&e0));
    SBWT_CUDA(cudaEventCreate(&e1));
    LaunchConfig saved = default_launch_config();
    double best = 1e30;
    LaunchConfig best_cfg = saved;
    bool have_ref = false;
    std::vector<u64> h_ref, h_out;
    // With the k-mer table (k <= 31, suffix groups, fewer than 192 * 2^24
    // nodes) the read search never reads the presearch table: the first axis
    // is then the kernel (table kernel, walks kernel with the filter, k-mers
    // kernel with 4 and 2 k-mers per lane, lean 16-slot walks kernel without
    // and with the filter), else
    // the presearch depth.
    const bool table_axis = ix.view.kmer_table && ix.view.suffix_group_starts && ix.k <= 31 &&
                            ix.num_bits < (192ULL << 24);
    std::vector<std::pair<u32, u32>> first;  // (presearch, kernel mode)
    if (table_axis) {
      for (u32 m : {1u, 2u, 6u, 11u, 17u, 18u}) first.emplace_back(ix.p_max, m);
    } else {
      for (u32 p = ix.p_max; p >= std::min<u32>(8, ix.p_max); --p) {
        first.emplace_back(p, saved.table_kernel);
        if (p == 0) break;
      }
    }
    for (const auto &pm : first) {
      for (u64 tile : {0ULL, 64ULL, 256ULL}) {
        for (u32 bps : {2u, 4u, 6u, 8u}) {
         for (u32 bt : {128u, 256u}) {
          LaunchConfig c = saved;
          c.presearch_letters = pm.first;
          c.table_kernel = pm.second;
          c.tile = tile;
          c.blocks_per_sm = bt == 128 ? 2 * bps : bps;  // the same threads per SM
          c.block_threads = bt;
          default_launch_config() = c;
          u64 n = 0;
          ix.search_reads(d_chars, nc, d_read_ends, nr, out.get<u64>(), nk, &n,
                          SBWT_DEVICE_POINTERS, st, c);  // warm
          SBWT_CUDA(cudaEventRecord(e0, st));
          for (int rep = 0; rep < 3; ++rep)
            ix.search_reads(d_chars, nc, d_read_ends, nr, out.get<u64>(), nk, &n,
                            SBWT_DEVICE_POINTERS, st, c);
          SBWT_CUDA(cudaEventRecord(e1, st));
          SBWT_CUDA(cudaEventSynchronize(e1));
          float ms = 0;
          SBWT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          h_out.resize(nk);
          SBWT_CUDA(cudaMemcpy(h_out.data(), out.get(), nk * 8, cudaMemcpyDeviceToHost));
          if (!have_ref) {
            h_ref = h_out;
            have_ref = true;
          } else if (h_out != h_ref) {
            default_launch_config() = saved;
            throw Error(SBWT_E_CUDA, "autotune: a configuration changed the results");
          }
          if (ms / 3 < best) {
            best = ms / 3;
            best_cfg = c;
          }
         }
        }
      }
    }
    default_launch_config() = best_cfg;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (best_presearch) *best_presearch = best_cfg.presearch_letters;
    if (best_blocks_per_sm) *best_blocks_per_sm = best_cfg.blocks_per_sm;
    if (best_tile) *best_tile = best_cfg.tile;
    if (best_ms) *best_ms = best;
  });
}
}
