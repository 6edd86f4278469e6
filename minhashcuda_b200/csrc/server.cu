// Continuous-batching hash server (mhcuda_server_*).
//
// The reference has no server: every mhcuda_calc call is one synchronous
// launch per device (minhashcuda.cc:583-642).  Here several "lanes" share one
// device.  Each lane is a host thread with two CUDA streams (high and low
// priority), device buffers for one batch (CSR in, hashes out, chunk
// scratch) and pinned host staging.  Active requests wait in a pool.  A free
// lane forms a batch shortest-remaining-work first: it takes the request with
// the least work left, then the next smallest of the same generator, each
// whole while the batch budget (max_batch_evals nnz*samples) lasts; the
// request that does not fit whole gives a row block and ends the batch.  The
// batch is gathered into one CSR and copy-in, the plan/hash/finalize kernels
// and copy-out run on one of the lane's streams; the lane waits for its own
// event and hands the hashes back.  Requests that arrive while batches are on
// the GPU join the pool at once and go into the next batch any lane forms.
// A batch that finishes all of its requests within max_unit_evals is small:
// it runs on the high-priority stream and uses no copy engine -- the kernels
// read its CSR from the lane's mapped page-locked staging and write the
// hashes into mapped host memory, so it never queues behind a large batch's
// copies.  Large batches launch one chunk per warp (non-persistent), so the
// blocks of a small batch's kernels are scheduled as soon as blocks of a
// large one retire instead of after its whole launch, and at most
// lanes - 2 large batches are out at once, so two lanes are always free for
// small requests.  Lanes overlap each other's copies and kernels.  Device
// memory is bounded by the budget given at start: the lanes are sized from
// it once and nothing grows afterwards.
//
// Per-request guarantees: the hashes equal a lone mhcuda_calc of the same
// request bit for bit (same kernels, same per-row arithmetic; the batch only
// changes which warp walks which positions).  A batch whose device status
// reports invalid CSR is re-run unit by unit so that only the offending
// request fails.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/minhashcuda.h"
#include "../../include/minhashcuda_b200.h"
#include "wmh_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  const MinhashCudaGenerator_ *gen = nullptr;
  mhb::GeneratorView g{};
  const float *weights = nullptr;
  const uint32_t *cols = nullptr;
  const uint32_t *rows = nullptr;
  uint32_t length = 0;
  uint32_t *output = nullptr;
  Clock::time_point submitted, finished;
  // Stage times for tracing (MHCUDA_B200_SERVER_TRACE): first row taken by a
  // lane, last unit's launches enqueued, last unit's device work done.
  Clock::time_point taken, launched, gpu_done;
  bool was_taken = false;
  uint32_t next_row = 0;        // first row not yet handed to a lane
  uint32_t inflight = 0;        // units handed out and not yet complete
  bool in_pinned = false;       // weights and cols are page-locked: large units copy directly
  bool out_pinned = false;      // output is page-locked: large units copy hashes directly
  MHCUDAResult result = mhcudaSuccess;
  bool cancelled = false;
  bool done = false;
};

struct Unit {
  Request *req;
  uint32_t r0, r1;  // rows of the request
};

struct Lane {
  cudaStream_t stream = nullptr;     // low priority
  cudaStream_t hi = nullptr;         // high priority
  bool high = false;                 // the current batch runs on `hi`
  cudaEvent_t done_ev = nullptr;
  // device
  float *w = nullptr;
  uint32_t *c = nullptr, *ip = nullptr, *out = nullptr, *chunk_row = nullptr, *status = nullptr;
  float *part_ln = nullptr;
  uint2 *part_kt = nullptr;
  // pinned host, mapped into the device's address space
  float *hw = nullptr;
  uint32_t *hc = nullptr, *hip = nullptr, *hout = nullptr, *hstatus = nullptr;
  // device addresses of the mapped staging (zero-copy batches)
  float *mw = nullptr;
  uint32_t *mc = nullptr, *mip = nullptr, *mout = nullptr, *mstatus = nullptr;
  bool zero_copy = false;
  std::vector<Unit> units;
  std::vector<uint64_t> unit_rows;  // row offset of each unit inside the batch
  std::vector<uint8_t> unit_direct; // hashes already copied straight to the caller
  std::thread thread;
};

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

uint64_t env_u64(const char *name, uint64_t fallback) {
  const char *v = getenv(name);
  if (!v || !*v) return fallback;
  const unsigned long long x = strtoull(v, nullptr, 10);
  return x ? x : fallback;
}

}  // namespace

struct MinhashCudaServer_ {
  int device = 0;
  int verbosity = 0;
  int sm_count = 148;
  // Per-lane capacities (bytes).
  size_t in_cap = 0, out_cap = 0, scratch_cap = 0;
  size_t scratch_unit = 0;  // scratch = chunk_row (1 unit) | part_ln (4) | part_kt (8)
  uint64_t max_unit_evals = 128ull << 20;   // nnz*samples: high-priority batch limit
  uint64_t max_batch_evals = 512ull << 20;  // nnz*samples of one lane batch
  // Warp items per resident warp a batch is cut into at least (small ones:
  // `min_items_high`, large ones: `min_items_low`).  Finer items for large
  // batches retire their blocks sooner, so a small batch's blocks find SMs
  // sooner.
  uint32_t min_items_high = 2, min_items_low = 2;
  uint32_t max_low_inflight = 6;            // low-priority batches out at once (lanes - 2)
  uint64_t zero_copy_max_bytes = ~0ull;     // CSR bytes of a batch read from mapped memory
  uint32_t low_inflight = 0;
  std::vector<Lane> lanes;

  std::mutex mu;
  std::condition_variable work;      // lanes: a request joined the pool (or stop)
  std::condition_variable finished;  // waiters: a request completed
  std::deque<Request *> ring;        // requests with rows not yet handed out
  std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
  std::vector<double> latencies_ms;  // completed requests, for mhcuda_server_stats
  // Per-request stage trace, written as CSV at stop when
  // MHCUDA_B200_SERVER_TRACE names a file.
  std::string trace_path;
  std::vector<std::string> trace;
  uint64_t next_ticket = 1;
  uint64_t evals_done = 0;
  Clock::time_point stats_since = Clock::now();
  bool stop = false;

  ~MinhashCudaServer_();
  void lane_loop(Lane &lane);
  bool take(Lane &lane);
  void complete(Lane &lane, MHCUDAResult launch_result);
  MHCUDAResult run_units(Lane &lane, const std::vector<Unit> &units, bool solo);
  void finish_locked(Request *r, Clock::time_point now);
  size_t unit_in_bytes(const Unit &u) const {
    const uint64_t n = static_cast<uint64_t>(u.req->rows[u.r1]) - u.req->rows[u.r0];
    return n * 8 + (static_cast<size_t>(u.r1 - u.r0) + 1) * 4;
  }
  size_t unit_out_bytes(const Unit &u) const {
    return static_cast<size_t>(u.r1 - u.r0) * u.req->g.samples * 8;
  }
};

namespace {

bool is_pinned(const void *p) {
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeHost;
}

// Units at least this large move between page-locked caller memory and the
// device with their own copies instead of through the lane's staging.
constexpr size_t kDirectCopyBytes = static_cast<size_t>(1) << 20;

// Copies the batch's device status word to the lane's mapped host word and
// clears it for the next batch (no copy engine involved).
__global__ void publish_status(uint32_t *d_status, uint32_t *h_status) {
  *h_status = *d_status;
  *d_status = 0;
}

void par_copy(void *dst, const void *src, size_t bytes) {
  const size_t kSplit = static_cast<size_t>(16) << 20;
  if (bytes < kSplit) {
    memcpy(dst, src, bytes);
    return;
  }
  const unsigned n = 4;
  const size_t part = (((bytes + n - 1) / n) + 4095) & ~static_cast<size_t>(4095);
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < n; ++t) {
    const size_t off = t * part;
    if (off >= bytes) break;
    const size_t len = std::min(part, bytes - off);
    pool.emplace_back([=]() {
      memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off, len);
    });
  }
  for (auto &th : pool) th.join();
}

}  // namespace

MinhashCudaServer_::~MinhashCudaServer_() {
  {
    std::lock_guard<std::mutex> lock(mu);
    stop = true;
  }
  work.notify_all();
  for (Lane &l : lanes)
    if (l.thread.joinable()) l.thread.join();
  if (!trace_path.empty()) {
    if (FILE *f = fopen(trace_path.c_str(), "w")) {
      fprintf(f, "ticket,samples,rows,nnz,queued_ms,gather_launch_ms,device_ms,complete_ms,"
                 "total_ms\n");
      for (const std::string &line : trace) fprintf(f, "%s\n", line.c_str());
      fclose(f);
    }
  }
  mhb::DeviceGuard on_device(device);
  for (Lane &l : lanes) {
    if (l.stream) cudaStreamSynchronize(l.stream);
    cudaFree(l.w);
    cudaFree(l.c);
    cudaFree(l.ip);
    cudaFree(l.out);
    cudaFree(l.chunk_row);  // base of the scratch that also holds part_ln / part_kt
    cudaFree(l.status);
    cudaFreeHost(l.hw);
    cudaFreeHost(l.hc);
    cudaFreeHost(l.hip);
    cudaFreeHost(l.hout);
    cudaFreeHost(l.hstatus);
    if (l.hi) cudaStreamSynchronize(l.hi);
    if (l.done_ev) cudaEventDestroy(l.done_ev);
    if (l.stream) cudaStreamDestroy(l.stream);
    if (l.hi) cudaStreamDestroy(l.hi);
  }
}

// Gathers `units` into the lane's staging and enqueues copy-in, kernels and
// copy-out on the lane's stream.  With `solo` the call waits for the result
// (used to attribute an invalid-CSR status to single units).
MHCUDAResult MinhashCudaServer_::run_units(Lane &lane, const std::vector<Unit> &units, bool solo) {
  const mhb::GeneratorView &g = units.front().req->g;
  uint64_t R = 0, N = 0;
  lane.unit_rows.assign(units.size() + 1, 0);
  std::vector<uint64_t> pos(units.size() + 1, 0);
  for (size_t k = 0; k < units.size(); ++k) {
    const Unit &u = units[k];
    R += u.r1 - u.r0;
    N += static_cast<uint64_t>(u.req->rows[u.r1]) - u.req->rows[u.r0];
    lane.unit_rows[k + 1] = R;
    pos[k + 1] = N;
  }
  const bool high = lane.high && !solo;
  const cudaStream_t st = high ? lane.hi : lane.stream;
  cudaError_t e = cudaSuccess;
  // Staged units are gathered into contiguous runs of the staging buffers;
  // each run goes over in one copy.  Large page-locked units copy directly.
  uint64_t run_begin = 0, run_end = 0;
  auto flush_run = [&]() {
    if (run_end > run_begin && e == cudaSuccess) {
      e = cudaMemcpyAsync(lane.w + run_begin, lane.hw + run_begin, (run_end - run_begin) * 4,
                          cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(lane.c + run_begin, lane.hc + run_begin, (run_end - run_begin) * 4,
                            cudaMemcpyHostToDevice, st);
    }
    run_begin = run_end;
  };
  // High-priority batches of a lane with mapped staging use no copy engine:
  // the kernels read the CSR from the staging and write the hashes into
  // mapped host memory, so they never queue behind large batches' copies.
  const bool zc = high && lane.zero_copy && N * 8 + R * 4 <= zero_copy_max_bytes;
  for (size_t k = 0; k < units.size(); ++k) {
    const Unit &u = units[k];
    const uint32_t b = u.req->rows[u.r0];
    const uint64_t n = pos[k + 1] - pos[k];
    if (!zc && u.req->in_pinned && n * 4 >= kDirectCopyBytes) {
      flush_run();
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(lane.w + pos[k], u.req->weights + b, n * 4, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(lane.c + pos[k], u.req->cols + b, n * 4, cudaMemcpyHostToDevice, st);
      run_begin = run_end = pos[k + 1];
    } else {
      par_copy(lane.hw + pos[k], u.req->weights + b, n * 4);
      par_copy(lane.hc + pos[k], u.req->cols + b, n * 4);
      run_end = pos[k + 1];
    }
    uint32_t *ip = lane.hip + lane.unit_rows[k];
    for (uint32_t x = u.r0; x < u.r1; ++x) ip[x - u.r0] = static_cast<uint32_t>(pos[k] + (u.req->rows[x] - b));
  }
  if (!zc) flush_run();
  lane.hip[R] = static_cast<uint32_t>(N);
  const uint32_t s_pad = g.s_pad;
  // Batches are small next to a plain call: at least two waves of warp items
  // even when rows are long (the plain plan keeps a few rows per chunk);
  // several lanes' launches overlap, so two are enough.
  mhb::HashPlan plan = mhb::plan_for_generator(units.front().req->gen, N, R,
                                               high ? min_items_high : min_items_low);
  const int bps = mhb::hash_blocks_per_sm(plan.spl, plan.minb, s_pad);
  // Keep the chunk table and partials inside the lane's fixed scratch:
  // nchunks*4 <= unit, 2*nchunks*s_pad*4 <= 4*unit, 2*nchunks*s_pad*8 <= 8*unit.
  const uint64_t max_chunks = std::max<uint64_t>(
      1, std::min<uint64_t>(scratch_unit / 4, scratch_unit / (2 * static_cast<uint64_t>(s_pad))));
  if (N > static_cast<uint64_t>(plan.chunk) * max_chunks) {
    uint64_t chunk = (N + max_chunks - 1) / max_chunks;
    chunk = (chunk + 31) & ~31ull;
    plan.chunk = static_cast<uint32_t>(chunk);
    plan.nchunks = static_cast<uint32_t>((N + chunk - 1) / chunk);
  }
  // High priority: a persistent grid.  Low priority: one item per warp, so
  // blocks retire often and high-priority blocks get their SMs.
  {
    const uint64_t items = static_cast<uint64_t>(plan.nchunks) * plan.ntiles;
    const uint64_t blocks = (items + 7) / 8;
    const uint64_t resident = static_cast<uint64_t>(sm_count) * bps;
    plan.grid = static_cast<uint32_t>(std::max<uint64_t>(
        1, high ? std::min(blocks, resident) : std::min<uint64_t>(blocks, 1u << 30)));
  }
  mhb::HashArgs a{};
  a.params = g.params;
  a.dim = g.dim;
  a.samples = g.samples;
  a.s_pad = s_pad;
  a.weights = zc ? lane.mw : lane.w;
  a.cols = zc ? lane.mc : lane.c;
  a.indptr = zc ? lane.mip : lane.ip;
  a.host_csr = zc ? 1u : 0u;
  a.rows = static_cast<uint32_t>(R);
  a.nnz = static_cast<uint32_t>(N);
  a.chunk = plan.chunk;
  a.nchunks = plan.nchunks;
  a.ntiles = plan.ntiles;
  a.chunk_row = lane.chunk_row;
  a.part_ln = lane.part_ln;
  a.part_kt = lane.part_kt;
  a.out = zc ? lane.mout : lane.out;
  a.status = lane.status;  // zero between batches: publish_status clears it
  if (e == cudaSuccess && !zc)
    e = cudaMemcpyAsync(lane.ip, lane.hip, (R + 1) * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = mhb::launch_plan(a, st);
  if (e == cudaSuccess) e = mhb::launch_hash(a, plan, st);
  if (e == cudaSuccess && plan.nchunks > 1) e = mhb::launch_finalize(a, st);
  if (e == cudaSuccess) {
    publish_status<<<1, 1, 0, st>>>(lane.status, lane.mstatus);
    e = cudaGetLastError();
  }
  // Hashes: large units into page-locked outputs directly, the rest through
  // the lane's staging (copied out by complete()); zero-copy batches have
  // theirs in the staging already.
  lane.unit_direct.assign(units.size(), 0);
  for (size_t k = 0; k < units.size() && e == cudaSuccess && !zc; ++k) {
    const Unit &u = units[k];
    const size_t bytes = unit_out_bytes(u);
    const size_t off = lane.unit_rows[k] * g.samples * 2;
    if (!solo && u.req->out_pinned && bytes >= kDirectCopyBytes) {
      e = cudaMemcpyAsync(u.req->output + static_cast<size_t>(u.r0) * g.samples * 2, lane.out + off,
                          bytes, cudaMemcpyDeviceToHost, st);
      lane.unit_direct[k] = 1;
    } else {
      e = cudaMemcpyAsync(lane.hout + off, lane.out + off, bytes, cudaMemcpyDeviceToHost, st);
    }
  }
  if (e == cudaSuccess) e = cudaEventRecord(lane.done_ev, st);
  if (e == cudaSuccess && solo) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return mhcudaRuntimeError;
  }
  return mhcudaSuccess;
}

// Under `mu`.
void MinhashCudaServer_::finish_locked(Request *r, Clock::time_point now) {
  r->done = true;
  r->finished = now;
  if (!r->cancelled)
    latencies_ms.push_back(std::chrono::duration<double, std::milli>(now - r->submitted).count());
  if (!trace_path.empty() && !r->cancelled && r->was_taken) {
    auto ms = [](Clock::time_point a, Clock::time_point b) {
      return std::chrono::duration<double, std::milli>(b - a).count();
    };
    char line[256];
    snprintf(line, sizeof(line), "%llu,%u,%u,%llu,%.4f,%.4f,%.4f,%.4f,%.4f",
             static_cast<unsigned long long>(r->ticket), r->g.samples, r->length,
             static_cast<unsigned long long>(r->rows[r->length] - r->rows[0]),
             ms(r->submitted, r->taken), ms(r->taken, r->launched), ms(r->launched, r->gpu_done),
             ms(r->gpu_done, now), ms(r->submitted, now));
    trace.emplace_back(line);
  }
}

// Under `mu`: fills lane.units shortest-remaining-work first.  Requests are
// ordered by the nnz*samples they have left; the smallest fixes the batch's
// generator; requests of that generator join whole while the batch budget and
// the lane's capacities last, and the first that does not fit whole gives its
// next row block (at least one row) and ends the batch.  Cancelled requests
// leave the pool.  Returns false if nothing was taken.
bool MinhashCudaServer_::take(Lane &lane) {
  auto remaining = [](const Request *r) {
    return (static_cast<uint64_t>(r->rows[r->length]) - r->rows[r->next_row]) * r->g.samples;
  };
  std::vector<std::pair<uint64_t, Request *>> order;
  order.reserve(ring.size());
  for (auto it = ring.begin(); it != ring.end();) {
    Request *r = *it;
    if (r->cancelled) {
      if (r->inflight == 0 && !r->done) finish_locked(r, Clock::now());
      it = ring.erase(it);
      continue;
    }
    order.emplace_back(remaining(r), r);
    ++it;
  }
  // With max_low_inflight low-priority batches out, only requests that fit a
  // high-priority batch whole are taken: the other lanes stay free for small
  // requests, whose copies then do not queue behind large ones.
  const bool allow_low = low_inflight < max_low_inflight;
  if (!allow_low)
    order.erase(std::remove_if(order.begin(), order.end(),
                               [&](const auto &x) { return x.first > max_unit_evals; }),
                order.end());
  if (order.empty()) return false;
  const uint64_t budget = allow_low ? max_batch_evals : max_unit_evals;
  std::sort(order.begin(), order.end(), [](const auto &x, const auto &y) {
    return x.first != y.first ? x.first < y.first : x.second->ticket < y.second->ticket;
  });
  const MinhashCudaGenerator_ *gen = order.front().second->gen;
  std::vector<Unit> batch;
  size_t in = 0, out = 0;
  uint64_t evals = 0;
  bool whole = true;
  for (const auto &entry : order) {
    Request *r = entry.second;
    if (r->gen != gen) continue;
    if (evals >= budget) break;
    const uint64_t S = r->g.samples;
    const size_t row_out = S * 8;
    uint32_t r1 = r->next_row;
    uint64_t ue = 0;
    size_t ui = 4, uo = 0;
    while (r1 < r->length) {
      const uint64_t nz = static_cast<uint64_t>(r->rows[r1 + 1]) - r->rows[r1];
      const size_t add_in = nz * 8 + 4;
      if (in + ui + add_in > in_cap || out + uo + row_out > out_cap) break;
      if (r1 != r->next_row && evals + ue + nz * S > budget) break;
      ui += add_in;
      uo += row_out;
      ue += nz * S;
      ++r1;
    }
    if (r1 == r->next_row) continue;  // not even one row fits what is left
    if (!allow_low && r1 < r->length) break;  // would not finish in this batch
    if (!r->was_taken) {
      r->was_taken = true;
      r->taken = Clock::now();
    }
    batch.push_back(Unit{r, r->next_row, r1});
    r->next_row = r1;
    ++r->inflight;
    in += ui;
    out += uo;
    evals += ue;
    if (r->next_row < r->length) {
      whole = false;
      break;
    }
  }
  if (batch.empty()) return false;
  for (auto it = ring.begin(); it != ring.end();)
    it = ((*it)->next_row == (*it)->length) ? ring.erase(it) : std::next(it);
  lane.high = whole && evals <= max_unit_evals;
  if (!lane.high) ++low_inflight;
  lane.units = std::move(batch);
  return true;
}

void MinhashCudaServer_::complete(Lane &lane, MHCUDAResult launch_result) {
  std::vector<Unit> units = std::move(lane.units);
  std::vector<MHCUDAResult> unit_result(units.size(), launch_result);
  if (launch_result == mhcudaSuccess && *lane.hstatus != 0) {
    // Attribute the invalid input: run every unit of the batch on its own.
    for (size_t k = 0; k < units.size(); ++k) {
      std::vector<Unit> one{units[k]};
      unit_result[k] = run_units(lane, one, true);
      if (unit_result[k] == mhcudaSuccess && *lane.hstatus != 0)
        unit_result[k] = mhcudaInvalidArguments;
      if (unit_result[k] == mhcudaSuccess) {
        const Unit &u = units[k];
        par_copy(u.req->output + static_cast<size_t>(u.r0) * u.req->g.samples * 2, lane.hout,
                 unit_out_bytes(u));
      }
    }
  } else if (launch_result == mhcudaSuccess) {
    for (size_t k = 0; k < units.size(); ++k) {
      const Unit &u = units[k];
      if (lane.unit_direct[k]) continue;
      par_copy(u.req->output + static_cast<size_t>(u.r0) * u.req->g.samples * 2,
               lane.hout + lane.unit_rows[k] * u.req->g.samples * 2, unit_out_bytes(u));
    }
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!lane.high) {
    --low_inflight;
    work.notify_all();
  }
  const Clock::time_point now = Clock::now();
  for (size_t k = 0; k < units.size(); ++k) {
    Request *r = units[k].req;
    evals_done += (static_cast<uint64_t>(r->rows[units[k].r1]) - r->rows[units[k].r0]) * r->g.samples;
    if (unit_result[k] != mhcudaSuccess) r->result = unit_result[k];
    --r->inflight;
    if (r->inflight == 0 && (r->next_row == r->length || r->cancelled) && !r->done)
      finish_locked(r, now);
  }
  finished.notify_all();
}

void MinhashCudaServer_::lane_loop(Lane &lane) {
  cudaSetDevice(device);
  for (;;) {
    {
      // Woken by a submit, a low-priority batch finishing, or stop.
      std::unique_lock<std::mutex> lock(mu);
      for (;;) {
        if (stop && ring.empty()) return;  // stop requested and nothing left
        if (take(lane)) break;
        work.wait(lock);
      }
    }
    MHCUDAResult r = run_units(lane, lane.units, false);
    const Clock::time_point launched = Clock::now();
    if (r == mhcudaSuccess && cudaEventSynchronize(lane.done_ev) != cudaSuccess) {
      cudaGetLastError();
      r = mhcudaRuntimeError;
    }
    if (!trace_path.empty()) {
      const Clock::time_point done = Clock::now();
      std::lock_guard<std::mutex> lock(mu);
      for (const Unit &u : lane.units) {
        u.req->launched = launched;
        u.req->gpu_done = done;
      }
    }
    complete(lane, r);
  }
}

extern "C" {

MinhashCudaServer *mhcuda_server_start(uint32_t devices, uint64_t hbm_budget_bytes, uint32_t lanes,
                                       int verbosity, enum MHCUDAResult *status) {
  auto set = [&](MHCUDAResult r) {
    if (status) *status = r;
  };
  if (lanes == 0 || lanes > 16 || hbm_budget_bytes < (static_cast<uint64_t>(64) << 20)) {
    set(mhcudaInvalidArguments);
    return nullptr;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    set(mhcudaNoSuchDevice);
    return nullptr;
  }
  int dev = -1;
  if (devices == 0) dev = 0;
  for (int d = 0; d < 32 && d < count && dev < 0; ++d)
    if (devices & (1u << d)) dev = d;
  if (dev < 0) {
    set(mhcudaNoSuchDevice);
    return nullptr;
  }
  mhb::DeviceGuard on_device(dev);
  if (!on_device.ok()) {
    set(mhcudaNoSuchDevice);
    return nullptr;
  }
  std::unique_ptr<MinhashCudaServer_> srv(new MinhashCudaServer_());
  srv->device = dev;
  srv->verbosity = verbosity;
  srv->max_unit_evals = env_u64("MHCUDA_B200_SERVER_UNIT_EVALS", srv->max_unit_evals);
  srv->max_batch_evals = env_u64("MHCUDA_B200_SERVER_BATCH_EVALS", srv->max_batch_evals);
  srv->zero_copy_max_bytes = env_u64("MHCUDA_B200_SERVER_ZERO_COPY_MAX_BYTES", ~0ull);
  if (const char *tp = getenv("MHCUDA_B200_SERVER_TRACE")) srv->trace_path = tp;
  srv->min_items_high =
      static_cast<uint32_t>(env_u64("MHCUDA_B200_SERVER_MIN_ITEMS_HIGH", srv->min_items_high));
  srv->min_items_low =
      static_cast<uint32_t>(env_u64("MHCUDA_B200_SERVER_MIN_ITEMS_LOW", srv->min_items_low));
  srv->max_low_inflight = static_cast<uint32_t>(std::min<uint64_t>(
      lanes, env_u64("MHCUDA_B200_SERVER_LOW_INFLIGHT", lanes > 2 ? lanes - 2 : 1)));
  cudaDeviceGetAttribute(&srv->sm_count, cudaDevAttrMultiProcessorCount, dev);
  const size_t per_lane = hbm_budget_bytes / lanes;
  srv->in_cap = align256(per_lane * 4 / 10);
  srv->out_cap = align256(per_lane * 4 / 10);
  srv->scratch_cap = align256(per_lane - srv->in_cap - srv->out_cap);
  srv->scratch_unit = (srv->scratch_cap / 13) & ~static_cast<size_t>(255);
  srv->lanes.resize(lanes);
  constexpr unsigned kMapped = cudaHostAllocMapped;
  int can_map = 0;
  cudaDeviceGetAttribute(&can_map, cudaDevAttrCanMapHostMemory, dev);
  const bool zero_copy_ok =
      can_map != 0 && env_u64("MHCUDA_B200_SERVER_NO_ZERO_COPY", 0) == 0;
  int prio_low = 0, prio_high = 0;  // numerically lower is higher priority
  if (cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess) {
    cudaGetLastError();
    prio_low = prio_high = 0;
  }
  for (Lane &l : srv->lanes) {
    const size_t max_nnz = srv->in_cap / 8;
    bool ok = cudaStreamCreateWithPriority(&l.stream, cudaStreamNonBlocking, prio_low) ==
                  cudaSuccess &&
              cudaStreamCreateWithPriority(&l.hi, cudaStreamNonBlocking, prio_high) == cudaSuccess &&
              cudaEventCreateWithFlags(&l.done_ev, cudaEventDisableTiming) == cudaSuccess &&
              cudaMalloc(&l.w, max_nnz * 4 + 16) == cudaSuccess &&
              cudaMalloc(&l.c, max_nnz * 4 + 16) == cudaSuccess &&
              cudaMalloc(&l.ip, srv->in_cap + 256) == cudaSuccess &&
              cudaMalloc(&l.out, srv->out_cap) == cudaSuccess &&
              cudaMalloc(&l.status, 256) == cudaSuccess &&
              cudaHostAlloc(reinterpret_cast<void **>(&l.hw), max_nnz * 4 + 16, kMapped) ==
                  cudaSuccess &&
              cudaHostAlloc(reinterpret_cast<void **>(&l.hc), max_nnz * 4 + 16, kMapped) ==
                  cudaSuccess &&
              cudaHostAlloc(reinterpret_cast<void **>(&l.hip), srv->in_cap + 256, kMapped) ==
                  cudaSuccess &&
              cudaHostAlloc(reinterpret_cast<void **>(&l.hout), srv->out_cap, kMapped) ==
                  cudaSuccess &&
              cudaHostAlloc(reinterpret_cast<void **>(&l.hstatus), 256, kMapped) == cudaSuccess &&
              cudaMemset(l.status, 0, 256) == cudaSuccess &&
              cudaHostGetDevicePointer(reinterpret_cast<void **>(&l.mstatus), l.hstatus, 0) ==
                  cudaSuccess;
    // Device addresses of the staging for zero-copy batches; without them a
    // lane copies every batch.
    l.zero_copy =
        ok && zero_copy_ok &&
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&l.mw), l.hw, 0) == cudaSuccess &&
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&l.mc), l.hc, 0) == cudaSuccess &&
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&l.mip), l.hip, 0) == cudaSuccess &&
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&l.mout), l.hout, 0) == cudaSuccess;
    if (ok && !l.zero_copy) cudaGetLastError();
    // Scratch: chunk table then partial minima, carved from one allocation.
    char *scratch = nullptr;
    ok = ok && cudaMalloc(&scratch, srv->scratch_cap) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      if (scratch) cudaFree(scratch);
      set(mhcudaMemoryAllocationFailure);
      return nullptr;
    }
    const size_t unit = srv->scratch_unit;
    l.chunk_row = reinterpret_cast<uint32_t *>(scratch);
    l.part_ln = reinterpret_cast<float *>(scratch + unit);
    l.part_kt = reinterpret_cast<uint2 *>(scratch + 5 * unit);
  }
  for (Lane &l : srv->lanes) {
    MinhashCudaServer_ *s = srv.get();
    l.thread = std::thread([s, &l]() { s->lane_loop(l); });
  }
  set(mhcudaSuccess);
  return srv.release();
}

enum MHCUDAResult mhcuda_server_submit(MinhashCudaServer *srv, const MinhashCudaGenerator *gen,
                                       const float *weights, const uint32_t *cols,
                                       const uint32_t *rows, uint32_t length, uint32_t *output,
                                       uint64_t *ticket) {
  if (!srv || !gen || !weights || !cols || !rows || !output || !ticket || length == 0)
    return mhcudaInvalidArguments;
  std::unique_ptr<Request> r(new Request());
  if (!mhb::generator_view(gen, &r->g)) return mhcudaInvalidArguments;
  if (r->g.device != srv->device) return mhcudaNoSuchDevice;
  if (rows[length] < rows[0]) return mhcudaInvalidArguments;
  // A single row (and one chunk's partials) must fit a lane on its own.
  const size_t row_out = static_cast<size_t>(r->g.samples) * 8;
  if (row_out > srv->out_cap || srv->scratch_unit < 2 * static_cast<size_t>(r->g.s_pad))
    return mhcudaMemoryAllocationFailure;
  for (uint32_t i = 0; i < length; ++i) {
    if (rows[i + 1] < rows[i]) return mhcudaInvalidArguments;
    if ((static_cast<size_t>(rows[i + 1]) - rows[i]) * 8 + 8 > srv->in_cap)
      return mhcudaMemoryAllocationFailure;
  }
  r->in_pinned = is_pinned(weights) && is_pinned(cols);
  r->out_pinned = is_pinned(output);
  r->gen = gen;
  r->weights = weights;
  r->cols = cols;
  r->rows = rows;
  r->length = length;
  r->output = output;
  r->submitted = Clock::now();
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    if (srv->stop) return mhcudaRuntimeError;
    r->ticket = srv->next_ticket++;
    *ticket = r->ticket;
    srv->ring.push_back(r.get());
    srv->requests.emplace(r->ticket, std::move(r));
  }
  srv->work.notify_one();
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_server_poll(MinhashCudaServer *srv, uint64_t ticket, int *done) {
  if (!srv || !done) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(srv->mu);
  auto it = srv->requests.find(ticket);
  if (it == srv->requests.end()) return mhcudaInvalidArguments;
  *done = it->second->done ? 1 : 0;
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_server_wait(MinhashCudaServer *srv, uint64_t ticket, double timeout_s,
                                     double *latency_ms) {
  if (!srv) return mhcudaInvalidArguments;
  std::unique_lock<std::mutex> lock(srv->mu);
  auto it = srv->requests.find(ticket);
  if (it == srv->requests.end()) return mhcudaInvalidArguments;
  Request *r = it->second.get();
  const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                           std::chrono::duration<double>(timeout_s));
  while (!r->done) {
    if (srv->finished.wait_until(lock, deadline) == std::cv_status::timeout && !r->done)
      return mhcudaRuntimeError;
  }
  const MHCUDAResult res = r->result;
  if (latency_ms)
    *latency_ms = std::chrono::duration<double, std::milli>(r->finished - r->submitted).count();
  srv->requests.erase(it);
  return res;
}

enum MHCUDAResult mhcuda_server_cancel(MinhashCudaServer *srv, uint64_t ticket) {
  if (!srv) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(srv->mu);
  auto it = srv->requests.find(ticket);
  if (it == srv->requests.end()) return mhcudaInvalidArguments;
  Request *r = it->second.get();
  if (r->done) return mhcudaInvalidArguments;
  r->cancelled = true;
  r->result = mhcudaRuntimeError;  // its hashes are not (all) computed
  if (r->inflight == 0) {
    auto q = std::find(srv->ring.begin(), srv->ring.end(), r);
    if (q != srv->ring.end()) srv->ring.erase(q);
    srv->finish_locked(r, Clock::now());
    srv->finished.notify_all();
  }
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_server_stats(MinhashCudaServer *srv, int reset, uint64_t *completed,
                                      double *p50_ms, double *p99_ms, double *p999_ms,
                                      double *evals_per_s) {
  if (!srv) return mhcudaInvalidArguments;
  std::lock_guard<std::mutex> lock(srv->mu);
  std::vector<double> v = srv->latencies_ms;
  std::sort(v.begin(), v.end());
  auto q = [&](double p) {
    if (v.empty()) return 0.0;
    const size_t i = std::min(v.size() - 1, static_cast<size_t>(p * (v.size() - 1) + 0.5));
    return v[i];
  };
  if (completed) *completed = v.size();
  if (p50_ms) *p50_ms = q(0.50);
  if (p99_ms) *p99_ms = q(0.99);
  if (p999_ms) *p999_ms = q(0.999);
  const double secs = std::chrono::duration<double>(Clock::now() - srv->stats_since).count();
  if (evals_per_s) *evals_per_s = secs > 0 ? static_cast<double>(srv->evals_done) / secs : 0.0;
  if (reset) {
    srv->latencies_ms.clear();
    srv->evals_done = 0;
    srv->stats_since = Clock::now();
  }
  return mhcudaSuccess;
}

enum MHCUDAResult mhcuda_server_stop(MinhashCudaServer *srv) {
  delete srv;
  return mhcudaSuccess;
}

}  // extern "C"
