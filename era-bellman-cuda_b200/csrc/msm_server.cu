// MSM request server (no counterpart in the reference): continuous batching of
// commitment requests over one resident base table.
//
// Requests (scalars of any length up to the table, device or host memory) are
// submitted from any thread and queue in arrival order.  A scheduler thread
// admits them into groups: a group takes requests from the head of the queue
// while its scratch footprint (sort keys and values, buckets, heads,
// reduction trees, staged host scalars and results) fits in the largest free
// block of a fixed device arena (the HBM budget) and a device stream slot is
// free.  Each group runs as one batched kernel chain (msm_batch.cu) on its
// slot's stream, so groups admitted while others are still on the GPU overlap
// with them on the device.  A group's completion (a host function enqueued
// after its last kernel) frees its arena block and its slot, which admits the
// next requests.  Every request records submit, start and completion times on
// one host clock.
#include "bellman-cuda-b200.h"
#include "device_arena.h"
#include "msm_batch.cuh"

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace msm_b200 {

namespace {

using clock_type = std::chrono::steady_clock;

struct request {
  unsigned long long ticket = 0;
  const void *scalars = nullptr;
  void *results = nullptr;
  unsigned count = 0;
  bool host_scalars = false, host_results = false;
  double submit_us = 0, start_us = 0, done_us = 0;
  unsigned group_size = 0;
  bool done = false;
  cudaError_t status = cudaSuccess;
};

struct server_impl;

struct slot {
  server_impl *server = nullptr;
  cudaStream_t stream = nullptr;
  uint8_t *staging = nullptr; // pinned host copy of the group's descriptors
  size_t staging_bytes = 0;
  bool busy = false;
  // Set by the completion host function, which must never wait for the
  // server lock: the scheduler makes CUDA calls while holding it, and some of
  // them wait for all device work, the host function included.
  std::atomic<bool> finished{false};
  std::vector<request *> members;
  size_t arena_offset = 0, arena_bytes = 0;
};

struct server_impl {
  int device = 0, sms = 0;
  const base_table_impl *table = nullptr;
  unsigned max_group = 16;
  uint8_t *arena_base = nullptr;
  device_arena arena;
  std::vector<std::unique_ptr<slot>> slots;
  std::mutex lock;
  std::condition_variable wake;    // scheduler: submissions, completions, stop
  std::condition_variable settled; // waiters: a request finished
  std::deque<request *> pending;
  std::unordered_map<unsigned long long, std::unique_ptr<request>> requests;
  unsigned long long next_ticket = 1;
  bool stop = false;
  std::thread scheduler;
  clock_type::time_point t0 = clock_type::now();
  unsigned long long groups_run = 0, requests_run = 0, max_inflight = 0;

  double now_us() const { return std::chrono::duration<double, std::micro>(clock_type::now() - t0).count(); }
  ~server_impl();
  void run();
  bool admit_one(slot &s); // called with lock held
};

static bool is_host(const void *ptr, cudaError_t &err) {
  cudaPointerAttributes attr{};
  err = cudaPointerGetAttributes(&attr, ptr);
  return err == cudaSuccess && (attr.type == cudaMemoryTypeUnregistered || attr.type == cudaMemoryTypeHost);
}

static void CUDART_CB group_finished(void *data) {
  slot *s = static_cast<slot *>(data);
  s->finished.store(true, std::memory_order_release);
  s->server->wake.notify_all(); // a wake-up lost to the race is recovered by the scheduler's poll interval
}

// Scratch of a group beyond its batch plan: host scalars are staged into the
// arena, host results are gathered there and copied back.
static size_t staged_bytes(const std::vector<request *> &members) {
  size_t bytes = 0;
  for (const request *r : members) {
    if (r->host_scalars)
      bytes += device_arena::round_up((size_t)r->count * sizeof(fe));
    if (r->host_results)
      bytes += device_arena::round_up(RESULT_BITS * sizeof(jacobian));
  }
  return bytes;
}

bool server_impl::admit_one(slot &s) {
  if (pending.empty())
    return false;
  // grow the group from the head of the queue while its footprint fits
  std::vector<request *> group;
  batch_plan best;
  size_t best_bytes = 0;
  const size_t room = arena.largest_free();
  for (request *r : pending) {
    if (group.size() >= max_group)
      break;
    group.push_back(r);
    std::vector<unsigned> counts;
    for (request *m : group)
      counts.push_back(m->count);
    batch_plan p;
    const cudaError_t e = make_batch_plan(p, table, counts.data(), (unsigned)counts.size(), nullptr, sms);
    const size_t bytes = e == cudaSuccess ? p.bytes + staged_bytes(group) : (size_t)-1;
    if (e != cudaSuccess || bytes > room) {
      group.pop_back();
      break;
    }
    best = std::move(p);
    best_bytes = bytes;
  }
  if (group.empty()) {
    // the head request alone does not fit now; if it never can, fail it
    request *head = pending.front();
    batch_plan p;
    const unsigned cnt = head->count;
    const cudaError_t e = make_batch_plan(p, table, &cnt, 1, nullptr, sms);
    if (e != cudaSuccess || p.bytes + staged_bytes({head}) > arena.size()) {
      pending.pop_front();
      head->status = e != cudaSuccess ? e : cudaErrorMemoryAllocation;
      head->done = true;
      head->done_us = now_us();
      settled.notify_all();
      return true;
    }
    return false;
  }
  size_t offset = 0;
  if (!arena.allocate(best_bytes, offset))
    return false;
  for (size_t k = 0; k < group.size(); k++)
    pending.pop_front();
  s.busy = true;
  s.finished = false;
  s.members = group;
  s.arena_offset = offset;
  s.arena_bytes = best_bytes;
  const double start = now_us();
  for (request *r : group) {
    r->start_us = start;
    r->group_size = (unsigned)group.size();
  }
  groups_run++;
  requests_run += group.size();

  // enqueue: descriptors, staged inputs, the chain, staged outputs, completion
  uint8_t *scratch = arena_base + offset;
  const std::vector<uint8_t> img = descriptor_image(best);
  cudaError_t e = cudaSuccess;
  if (s.staging_bytes < img.size()) {
    if (s.staging)
      cudaFreeHost(s.staging);
    s.staging = nullptr;
    s.staging_bytes = 0;
    e = cudaMallocHost(&s.staging, img.size());
    if (e == cudaSuccess)
      s.staging_bytes = img.size();
  }
  std::vector<const void *> scalars(group.size());
  std::vector<void *> results(group.size());
  size_t extra = best.bytes;
  for (size_t k = 0; k < group.size() && e == cudaSuccess; k++) {
    request *r = group[k];
    scalars[k] = r->scalars;
    results[k] = r->results;
    if (r->host_scalars) {
      const size_t bytes = (size_t)r->count * sizeof(fe);
      e = cudaMemcpyAsync(scratch + extra, r->scalars, bytes, cudaMemcpyHostToDevice, s.stream);
      scalars[k] = scratch + extra;
      extra += device_arena::round_up(bytes);
    }
    if (r->host_results) {
      results[k] = scratch + extra;
      extra += device_arena::round_up(RESULT_BITS * sizeof(jacobian));
    }
  }
  if (e == cudaSuccess) {
    std::memcpy(s.staging, img.data(), img.size());
    e = cudaMemcpyAsync(scratch + best.descriptors, s.staging, img.size(), cudaMemcpyHostToDevice, s.stream);
  }
  if (e == cudaSuccess)
    e = enqueue_io(reinterpret_cast<batch_io *>(scratch + best.io), best.instances, scalars.data(), results.data(), s.stream);
  if (e == cudaSuccess)
    e = enqueue_batch(best, scratch, s.stream, nullptr, nullptr, nullptr);
  for (size_t k = 0; k < group.size() && e == cudaSuccess; k++)
    if (group[k]->host_results)
      e = cudaMemcpyAsync(group[k]->results, results[k], RESULT_BITS * sizeof(jacobian), cudaMemcpyDeviceToHost, s.stream);
  if (e == cudaSuccess)
    e = cudaLaunchHostFunc(s.stream, group_finished, &s);
  if (e != cudaSuccess) {
    // nothing more is enqueued for this group: wait for what was, then fail it
    cudaStreamSynchronize(s.stream);
    for (request *r : group)
      r->status = e;
    s.finished = true;
  }
  unsigned long long inflight = 0;
  for (auto &sl : slots)
    inflight += sl->busy;
  max_inflight = std::max(max_inflight, inflight);
  return true;
}

void server_impl::run() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> g(lock);
  while (true) {
    bool progress = false;
    // completions
    for (auto &sp : slots) {
      slot &s = *sp;
      if (!s.busy || !s.finished.load(std::memory_order_acquire))
        continue;
      const double t = now_us();
      for (request *r : s.members) {
        r->done_us = t;
        r->done = true;
      }
      arena.release(s.arena_offset, s.arena_bytes);
      s.members.clear();
      s.busy = false;
      s.finished = false;
      progress = true;
      settled.notify_all();
    }
    // admissions, oldest request first
    for (auto &sp : slots)
      if (!sp->busy && admit_one(*sp))
        progress = true;
    bool busy = false;
    for (auto &sp : slots)
      busy |= sp->busy;
    if (stop && pending.empty() && !busy)
      break;
    if (!progress)
      wake.wait_for(g, std::chrono::microseconds(200));
  }
}

server_impl::~server_impl() {
  {
    std::lock_guard<std::mutex> g(lock);
    stop = true;
  }
  wake.notify_all();
  if (scheduler.joinable())
    scheduler.join();
  for (auto &sp : slots) {
    if (sp->stream) {
      cudaStreamSynchronize(sp->stream);
      cudaStreamDestroy(sp->stream);
    }
    if (sp->staging)
      cudaFreeHost(sp->staging);
  }
  if (arena_base)
    cudaFree(arena_base);
}

} // namespace

cudaError_t server_create(server_impl **out, const base_table_impl *table, size_t scratch_budget, unsigned streams, unsigned max_group) {
  if (!out || !table || scratch_budget < (1u << 20) || streams == 0 || streams > 64 || max_group == 0 || max_group > MAX_BATCH)
    return cudaErrorInvalidValue;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess)
    return cudaErrorInvalidDevice;
  if (device != table->device)
    return cudaErrorInvalidDevice;
  std::unique_ptr<server_impl> srv(new (std::nothrow) server_impl);
  if (!srv)
    return cudaErrorMemoryAllocation;
  srv->device = device;
  srv->table = table;
  srv->max_group = max_group;
  cudaError_t e = cudaDeviceGetAttribute(&srv->sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess)
    e = batch_set_up();
  if (e == cudaSuccess)
    e = cudaMalloc(&srv->arena_base, scratch_budget);
  if (e != cudaSuccess)
    return e;
  srv->arena.reset(scratch_budget);
  for (unsigned k = 0; k < streams; k++) {
    std::unique_ptr<slot> s(new (std::nothrow) slot);
    if (!s)
      return cudaErrorMemoryAllocation;
    s->server = srv.get();
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
      return e;
    srv->slots.push_back(std::move(s));
  }
  srv->scheduler = std::thread([p = srv.get()] { p->run(); });
  *out = srv.release();
  return cudaSuccess;
}

cudaError_t server_submit(server_impl *srv, const void *scalars, unsigned count, void *results, unsigned long long *ticket) {
  if (!srv || !scalars || !results || !ticket || count == 0)
    return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(scalars) & 15) || (reinterpret_cast<uintptr_t>(results) & 15))
    return cudaErrorInvalidValue;
  std::unique_ptr<request> r(new (std::nothrow) request);
  if (!r)
    return cudaErrorMemoryAllocation;
  cudaError_t e;
  r->host_scalars = is_host(scalars, e);
  if (e != cudaSuccess)
    return e;
  r->host_results = is_host(results, e);
  if (e != cudaSuccess)
    return e;
  r->scalars = scalars;
  r->results = results;
  r->count = count;
  {
    std::lock_guard<std::mutex> g(srv->lock);
    if (srv->stop)
      return cudaErrorInvalidValue;
    r->ticket = srv->next_ticket++;
    r->submit_us = srv->now_us();
    *ticket = r->ticket;
    srv->pending.push_back(r.get());
    srv->requests.emplace(r->ticket, std::move(r));
  }
  srv->wake.notify_all();
  return cudaSuccess;
}

cudaError_t server_wait(server_impl *srv, unsigned long long ticket, msm_b200_request_times *times) {
  if (!srv)
    return cudaErrorInvalidValue;
  std::unique_lock<std::mutex> g(srv->lock);
  auto it = srv->requests.find(ticket);
  if (it == srv->requests.end())
    return cudaErrorInvalidValue;
  request *r = it->second.get();
  srv->settled.wait(g, [&] { return r->done; });
  if (times) {
    times->submit_us = r->submit_us;
    times->start_us = r->start_us;
    times->done_us = r->done_us;
    times->group_size = r->group_size;
  }
  const cudaError_t status = r->status;
  srv->requests.erase(it);
  return status;
}

cudaError_t server_stats(server_impl *srv, msm_b200_server_stats *stats) {
  if (!srv || !stats)
    return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> g(srv->lock);
  stats->groups = srv->groups_run;
  stats->requests = srv->requests_run;
  stats->max_inflight_groups = srv->max_inflight;
  stats->arena_bytes = srv->arena.size();
  stats->arena_used = srv->arena.used();
  stats->pending = srv->pending.size();
  return cudaSuccess;
}

} // namespace msm_b200

extern "C" {

bc_error msm_b200_server_create(msm_b200_server *server, msm_b200_base_table table, size_t scratch_budget, unsigned streams, unsigned max_group) {
  if (!server)
    return bc_error_invalid_value;
  msm_b200::server_impl *s = nullptr;
  const cudaError_t e =
      msm_b200::server_create(&s, reinterpret_cast<const msm_b200::base_table_impl *>(table), scratch_budget, streams, max_group);
  *server = reinterpret_cast<msm_b200_server>(s);
  return static_cast<bc_error>(e);
}

bc_error msm_b200_server_submit(msm_b200_server server, const void *scalars, unsigned count, void *results, unsigned long long *ticket) {
  return static_cast<bc_error>(msm_b200::server_submit(reinterpret_cast<msm_b200::server_impl *>(server), scalars, count, results, ticket));
}

bc_error msm_b200_server_wait(msm_b200_server server, unsigned long long ticket, msm_b200_request_times *times) {
  return static_cast<bc_error>(msm_b200::server_wait(reinterpret_cast<msm_b200::server_impl *>(server), ticket, times));
}

bc_error msm_b200_server_get_stats(msm_b200_server server, msm_b200_server_stats *stats) {
  return static_cast<bc_error>(msm_b200::server_stats(reinterpret_cast<msm_b200::server_impl *>(server), stats));
}

bc_error msm_b200_server_destroy(msm_b200_server server) {
  delete reinterpret_cast<msm_b200::server_impl *>(server);
  return bc_success;
}

} // extern "C"
