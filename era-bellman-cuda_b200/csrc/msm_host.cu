// Host orchestration of the MSM pipeline: planning, scratch layout, launch
// sequence and the msm_* C ABI.  Mirrors the reference's msm::execute_async
// (src/msm.cu:419-460) and schedule_execution (src/msm.cu:85-417): one call
// enqueues the whole pipeline on the caller's stream, all temporaries come
// from the caller's memory pool in stream order, and host-resident scalars,
// bases and results are copied in / out with the optional events and
// callbacks fired after the copies.
#include "bellman-cuda.h"
#include "bellman-cuda-b200.h"
#include "msm_host.cuh"

#include <cuda.h> // driver types of the context lookup (no driver calls are linked)
#include "msm_kernels.cuh"
#include "plain_tuning.h"
#include "pointer_access.h"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <vector>

namespace msm_b200 {

#define CHECK(statement)                                                                                                                       \
  do {                                                                                                                                         \
    cudaError_t check_result_ = (statement);                                                                                                   \
    if (check_result_ != cudaSuccess)                                                                                                          \
      return check_result_;                                                                                                                    \
  } while (0)

static unsigned ceil_log2(unsigned long long v) {
  unsigned r = 0;
  while ((1ull << r) < v)
    r++;
  return r;
}

// Window width by problem size: the checked-in table measured by the
// autotuner (era-bellman-cuda_b200/autotune.py --plain).  Keys take c - 1
// bits, so every width up to 17 sorts in two 8-bit passes.
unsigned default_window_bits(unsigned long long n) {
  const unsigned lg = ceil_log2(n);
  for (const tuning_row &row : PLAIN_TUNING)
    if (lg <= row.max_log_n)
      return row.window_bits;
  return PLAIN_TUNING[sizeof(PLAIN_TUNING) / sizeof(PLAIN_TUNING[0]) - 1].window_bits;
}

// Affine pairing levels ahead of the XYZZ accumulation (msm_affine.cuh).
static std::atomic<int> affine_levels_override{-1};

// None by default: measured on a B200 (uniform scalars, kernel times from a
// launch list), a level's additions cost more than the XYZZ madds they
// replace.  At 2^22 (c = 17) the first level's forward and apply kernels took
// 1.72 + 3.73 ms for 31.0 M pair sums (176 ps each: two random gathers of
// every base, one in each pass), the second level's 0.53 + 1.50 ms for 15.5 M
// (131 ps), the third's 0.28 + 0.79 ms for 7.7 M, each level's inversion
// kernel 0.11 ms, against 150 ps per XYZZ += affine addition of the plain
// accumulation (9.24 ms for 61.8 M); accumulation stage 9.24 ms without
// levels, 10.28 / 10.08 / 10.12 / 10.21 ms with 1 / 2 / 3 / 4.  At 2^20 (bases
// in L2) 2.80 ms without, 2.81 / 2.88 / 3.00 / 3.13 ms with 1-4.  The apply
// kernels run the multiply pipe at 61-74 % (ncu) against the accumulation's
// 84 %, and every level streams its list through DRAM twice.
unsigned default_affine_levels(unsigned long long) { return 0; }

void set_affine_levels_override(int levels) { affine_levels_override.store(levels); }

// Upper bound of a level's output elements for m input elements and `slots`
// buckets: each pair yields one element, or two when its elements belong to
// different buckets, which happens at most once per bucket boundary.
static unsigned long long level_output_bound(unsigned long long m, unsigned long long slots) { return std::min(m, (m + 1) / 2 + slots); }

void set_affine_levels(plan &p, unsigned levels) {
  const unsigned long long entries = (unsigned long long)p.windows * p.n;
  if (entries >= (1ull << 31))
    levels = 0; // the XYZZ pass takes list positions as 31-bit entry values
  p.affine_levels = std::min(levels, MAX_AFFINE_LEVELS);
  if (!p.affine_levels) {
    p.level_warps = 0;
    p.tail_threads = p.acc_threads;
    p.tail_ranges = p.acc_ranges;
    return;
  }
  const unsigned long long slots = (unsigned long long)p.windows << p.log_b;
  unsigned long long left = entries;
  for (unsigned level = 0; level < p.affine_levels; level++)
    left = level_output_bound(left, slots);
  const unsigned long long full = (unsigned long long)p.sms * 4 * ACC_THREADS;
  p.tail_threads = (unsigned)std::max(1ull, std::min(full, (left + 7) / 8));
  p.tail_ranges = accumulation_ranges(p.tail_threads, left, ACC_RANGES_PER_THREAD);
  // one resident apply warp per scheduler slot (AFFINE_APPLY_MIN_BLOCKS blocks
  // per SM), fewer when a lane would have under 16 pairs of the first level
  const unsigned long long pairs = (entries + 1) / 2;
  const unsigned long long most = (unsigned long long)p.sms * AFFINE_APPLY_MIN_BLOCKS * (AFFINE_APPLY_THREADS / 32);
  p.level_warps = (unsigned)std::max(1ull, std::min(most, (pairs + 32 * 16 - 1) / (32 * 16)));
}

struct device_info {
  int sms = 0;
};

static device_info get_device_info(int device) {
  static std::mutex lock;
  static device_info cache[64];
  std::lock_guard<std::mutex> guard(lock);
  if (device < 0 || device >= 64)
    return device_info{148};
  if (cache[device].sms == 0) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
      sms = 148;
    cache[device].sms = sms;
  }
  return cache[device];
}

// Accumulation ranges: a whole number k <= per_thread of ranges per thread,
// as large as keeps ACC_MIN_RANGE entries per range (a range's start-up --
// cursor search, first gather, head -- costs about as much as a few hundred
// additions: 2^21 points ran 3 % slower with 205-entry ranges than with 410).
// Whole multiples keep every warp at the same number of rounds.  Measured at
// the 3.5M-point second chunk of a host-input 2^22 MSM (52 M entries): two
// ranges of 346 entries per thread beat one of 692 by 0.48 ms (end to end
// 12.90 -> 12.40 ms), hence 300 rather than 400.
unsigned accumulation_ranges(unsigned threads, unsigned long long entries, unsigned per_thread) {
  const unsigned long long fit = entries / ((unsigned long long)threads * ACC_MIN_RANGE);
  const unsigned long long k = std::max(1ull, std::min((unsigned long long)per_thread, fit));
  return (unsigned)(threads * k);
}

// log2 of the running-sum group of the reduction per window width.  A group
// thread's 2 (m - 1) additions are one dependent chain, so few buckets want
// small groups (the chain is the stage's latency), many buckets larger ones
// (fewer tree levels).  Measured on a B200, reduction stage with m = 8 / 4 / 2:
// c = 5 (2^12 points) 0.110 / 0.079 / 0.067 ms, c = 11 (2^14) 0.198 / 0.159 /
// 0.145, c = 13 (2^16) 0.226 / 0.198 / 0.194, c = 15 (2^18) 0.290 / 0.312 /
// 0.319, c = 16 (2^20) 0.445 / 0.433 / 0.435, c = 17 (2^22) 0.664 / 0.637 /
// 0.656.
static unsigned reduction_log_m(unsigned c) { return c <= 14 ? 1 : c == 15 ? 3 : 2; }

// Groups of 2^log_m slots (at most the window's slots); the reduction's tree
// and stream buffers hold G = 2^(log_b - log_m) entries per window.
void set_reduction_groups(plan &p, unsigned log_m) {
  p.log_m = std::min(log_m, p.log_b);
  p.log_g = p.log_b - p.log_m;
  p.groups = 1u << p.log_g;
}

plan make_plan(unsigned n, unsigned window_bits, int sms) {
  plan p{};
  p.n = n;
  p.sms = (unsigned)sms;
  p.c = window_bits ? window_bits : default_window_bits(n);
  p.windows = (RESULT_BITS + p.c - 1) / p.c;
  p.log_b = p.c - 1;
  p.key_bits = p.c - 1; // keys are |d| - 1 for |d| in [1, 2^(c-1)]
  p.sort_passes = (p.key_bits + SORT_RADIX_BITS - 1) / SORT_RADIX_BITS;
  p.tiles = (n + SORT_TILE - 1) / SORT_TILE;
  p.lookback_tiles = (n + LOOKBACK_TILE - 1) / LOOKBACK_TILE;
  // One accumulation range per resident thread (4 blocks of ACC_THREADS per
  // SM), fewer for small inputs so that every range has work.
  const unsigned long long entries = (unsigned long long)p.windows * n;
  const unsigned long long full = (unsigned long long)sms * 4 * ACC_THREADS;
  p.acc_threads = (unsigned)std::max(1ull, std::min(full, (entries + 7) / 8));
  p.acc_ranges = accumulation_ranges(p.acc_threads, entries, ACC_RANGES_PER_THREAD);
  set_reduction_groups(p, reduction_log_m(p.c));
  const int forced = affine_levels_override.load();
  set_affine_levels(p, forced >= 0 ? (unsigned)forced : default_affine_levels(n));
  return p;
}

// Host-resident inputs are processed in chunks of points: the copy of chunk
// j + 1 runs on a helper stream while chunk j is sorted and accumulated, and
// every chunk after the first accumulates into its own buckets, which are then
// folded into the MSM's.  Chunk sizes grow by CHUNK_GROWTH (a chunk's pipeline
// takes about five times as long per point as the host-to-device copy, so
// chunk j + 1's copy ends about when chunk j's work does), and only the first
// chunk's copy is exposed; the chunk count trades that copy against one bucket
// fold and one more pipeline start per extra chunk (cost model below, in
// microseconds, fitted to B200 measurements).  Measured at 2^22 end to end:
// two chunks 1:5 12.94 ms, 1:6 13.11 ms (chunk 1's copy outlasts chunk 0's
// work), 1:4 level with 1:5, 1:3 slower; three chunks 1:4:16 13.13 ms.  With
// the later accumulation-range and segment-alignment fixes, three chunks 1:5:25
// still lose to two: 12.30 against 12.27 ms; with the warp-scan head merge
// and the current sort, 11.964 against 11.954 ms.
// Folding by continuing the earlier chunks' buckets inside the accumulation
// (no second bucket set, no fold kernel) measured slower: 13.02 against
// 12.85 ms at 2^22, 25.2 against 23.4 ms at 2^23.  Reference counterpart: the
// chunked copy/compute overlap of schedule_execution (src/msm.cu:160-334).
constexpr unsigned MAX_CHUNKS = 4;
constexpr unsigned CHUNK_GROWTH = 5;
constexpr double COPY_US_PER_POINT = 0.58e-3; // 32 B scalar over PCIe
constexpr double EXTRA_CHUNK_US = 360.0;      // one bucket fold + one more pipeline start
constexpr unsigned MIN_FIRST_CHUNK = 1u << 16;
// Smallest chunk the out-of-memory fit goes down to (the reference stops at
// get_log_min_inputs_count, src/msm.cu:39-57, e.g. 2^19 points at 2^22).
constexpr unsigned MIN_FIT_CHUNK = 1u << 16;
// Largest chunk: the radix passes' look-back words hold counts below 2^30.
constexpr unsigned MAX_CHUNK_POINTS = 1u << 29;

// Chunk boundaries: chunk j holds points [beg[j], beg[j + 1]).  `slots` = 0:
// copies of host-resident inputs go to a copy area of all n points (chunk j at
// offset beg[j]); slots = 2: to two chunk-sized slots used in turn (chunk j in
// slot j & 1), which the out-of-memory fit uses so that the copy area shrinks
// with the chunks.
struct chunking {
  unsigned count = 1;
  unsigned slots = 0;
  std::vector<unsigned> beg;
  unsigned size(unsigned j) const { return beg[j + 1] - beg[j]; }
  unsigned largest() const {
    unsigned m = 0;
    for (unsigned j = 0; j < count; j++)
      m = std::max(m, size(j));
    return m;
  }
  // offset of chunk j in a copy area
  size_t slot_offset(unsigned j) const { return slots ? (size_t)(j % slots) * largest() : beg[j]; }
};

static chunking make_chunks(unsigned n, bool copy_inputs) {
  chunking ch;
  unsigned k = 1;
  if (copy_inputs) {
    // the k <= MAX_CHUNKS of least modelled cost whose first chunk keeps MIN_FIRST_CHUNK points
    double best = n * COPY_US_PER_POINT;
    unsigned long long weight = 1, total = 1;
    for (unsigned cand = 2; cand <= MAX_CHUNKS; cand++) {
      weight *= CHUNK_GROWTH;
      total += weight;
      if ((unsigned long long)n < MIN_FIRST_CHUNK * total)
        break;
      const double cost = (double)n / total * COPY_US_PER_POINT + (cand - 1) * EXTRA_CHUNK_US;
      if (cost < best) {
        best = cost;
        k = cand;
      }
    }
  }
  ch.count = k;
  ch.beg.resize(k + 1);
  unsigned long long total = 0, weight = 1;
  for (unsigned j = 0; j < k; j++, weight *= CHUNK_GROWTH)
    total += weight;
  unsigned long long acc = 0;
  weight = 1;
  for (unsigned j = 0; j < k; j++, weight *= CHUNK_GROWTH) {
    ch.beg[j] = (unsigned)((unsigned long long)n * acc / total);
    acc += weight;
  }
  ch.beg[k] = n;
  return ch;
}

// Equal chunks of at most max_chunk points (the out-of-memory fit); host
// inputs then go through two chunk-sized copy slots.
static chunking equal_chunks(unsigned n, unsigned max_chunk, bool copy_inputs) {
  chunking ch;
  ch.count = (unsigned)(((unsigned long long)n + max_chunk - 1) / max_chunk);
  ch.slots = copy_inputs && ch.count > 1 ? 2 : 0;
  ch.beg.resize(ch.count + 1);
  for (unsigned j = 0; j <= ch.count; j++)
    ch.beg[j] = (unsigned)((unsigned long long)n * j / ch.count);
  return ch;
}

// Scratch layout inside one pool allocation.  `p` is the plan of the largest
// chunk (keys, values and heads are reused chunk after chunk); copies of
// host-resident inputs are sized for `copy_n` points (all of them, or two
// chunk slots); a chunked MSM holds a second bucket set for the chunks after
// the first.
struct layout {
  size_t keys[2], vals[2], counts, totals, zeros, sort_ctrs, sort_error, lookback_words, sort_clear_bytes, buckets, flags,
      chunk_buckets, chunk_flags, hb[2], hp[2], work, tree[2], streams[2], results, scalars, bases, total;
  // affine pairing levels: two output lists (level L writes list (L - 1) & 1),
  // the per-pair prefix products, the per-lane and per-warp arrays, and each
  // level's output count
  size_t level_buckets[2], level_points[2], level_pre, level_others, level_total, level_inverse, level_outputs, level_base, level_counts;
};

static size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

static layout make_layout(const plan &p, bool copy_scalars, bool copy_bases, bool copy_results, unsigned copy_n = 0, bool chunked = false) {
  layout l{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += align_up(bytes);
    return at;
  };
  if (!copy_n)
    copy_n = p.n;
  const size_t entries = (size_t)p.windows * window_stride(p.n);
  for (int i = 0; i < 2; i++) {
    l.keys[i] = take(entries * 4);
    l.vals[i] = take(entries * 4);
  }
  // the first pass's digit counts per (window, digit, tile); then one region
  // cleared per chunk: digit totals per (pass, window, digit), zero digits
  // per window, a tile counter per pass, the look-back error word, and the
  // look-back words of the passes after the first, per (window, look-back
  // tile, digit)
  const size_t lookback_words = (size_t)p.windows * p.lookback_tiles * SORT_RADIX;
  l.counts = take((size_t)p.windows * SORT_RADIX * p.tiles * 4);
  l.sort_clear_bytes = ((size_t)p.sort_passes * p.windows * SORT_RADIX + p.windows + p.sort_passes + 1 + (p.sort_passes - 1) * lookback_words) * 4;
  l.totals = take(l.sort_clear_bytes);
  l.zeros = l.totals + (size_t)p.sort_passes * p.windows * SORT_RADIX * 4;
  l.sort_ctrs = l.zeros + (size_t)p.windows * 4;
  l.sort_error = l.sort_ctrs + (size_t)p.sort_passes * 4;
  l.lookback_words = l.sort_error + 4;
  const size_t slots = (size_t)p.windows << p.log_b;
  l.buckets = take(slots * sizeof(xyzz));
  l.flags = take(slots);
  if (chunked) {
    l.chunk_buckets = take(slots * sizeof(xyzz));
    l.chunk_flags = take(slots);
  }
  const size_t heads = std::max(p.acc_ranges, p.tail_ranges);
  for (int i = 0; i < 2; i++) {
    l.hb[i] = take(heads * 4);
    l.hp[i] = take(heads * sizeof(xyzz));
  }
  if (p.affine_levels) {
    const unsigned long long entries = (unsigned long long)p.windows * p.n, slots = (unsigned long long)p.windows << p.log_b;
    const unsigned long long first = level_output_bound(entries, slots), second = level_output_bound(first, slots);
    // later levels shrink: level L's bound is at most that of level L - 2
    for (int i = 0; i < (p.affine_levels > 1 ? 2 : 1); i++) {
      const unsigned long long bound = i ? second : first;
      l.level_buckets[i] = take(bound * 4);
      l.level_points[i] = take(bound * sizeof(affine));
    }
    const size_t warps = p.level_warps;
    l.level_pre = take((entries + 1) / 2 * sizeof(fe));
    l.level_others = take(warps * 32 * sizeof(fe));
    l.level_total = take(warps * sizeof(fe));
    l.level_inverse = take(warps * sizeof(fe));
    l.level_outputs = take(warps * 4);
    l.level_base = take(warps * 8);
    l.level_counts = take((MAX_AFFINE_LEVELS + 1) * 8);
  }
  l.work = take(sizeof(unsigned));
  for (int i = 0; i < 2; i++) {
    l.tree[i] = take(((size_t)p.windows << p.log_g) * sizeof(xyzz));
    l.streams[i] = take((size_t)p.windows * stream_stride(p.log_g) * sizeof(xyzz));
  }
  l.results = copy_results ? take(RESULT_BITS * sizeof(jacobian)) : 0;
  l.scalars = copy_scalars ? take((size_t)copy_n * sizeof(fe)) : 0;
  l.bases = copy_bases ? take((size_t)copy_n * sizeof(affine)) : 0;
  l.total = off;
  return l;
}

// Plan of the largest chunk of an n-point MSM split as `ch`, at the window
// width of the whole MSM.
static plan largest_chunk_plan(unsigned n, unsigned window_bits, int sms, const chunking &ch) {
  const unsigned c = window_bits ? window_bits : default_window_bits(n);
  return make_plan(ch.largest(), c, sms);
}

// Layout of an MSM split as `ch`.
static layout chunked_layout(unsigned n, unsigned window_bits, int sms, const chunking &ch, bool copy_scalars, bool copy_bases, bool copy_results) {
  const plan p = largest_chunk_plan(n, window_bits, sms, ch);
  const unsigned copy_n = ch.slots ? ch.slots * ch.largest() : n;
  return make_layout(p, copy_scalars, copy_bases, copy_results, copy_n, ch.count > 1);
}

size_t scratch_bytes(unsigned n, unsigned window_bits, bool copy_scalars, bool copy_bases, bool copy_results) {
  int device = 0;
  cudaGetDevice(&device);
  const chunking ch = make_chunks(n, copy_scalars || copy_bases);
  return chunked_layout(n, window_bits, get_device_info(device).sms, ch, copy_scalars, copy_bases, copy_results).total;
}

// Where one of the caller's buffers lives: host memory (pinned or pageable,
// copied in or out by the call: *host = true) or memory the kernels use in
// place.  Device memory of another device is refused unless the current
// device has peer access to it (pointer_access.h): a kernel would fault on it.
static cudaError_t locate(const void *ptr, int device, bool *host) {
  cudaPointerAttributes attr{};
  CHECK(cudaPointerGetAttributes(&attr, ptr));
  *host = attr.type == cudaMemoryTypeUnregistered || attr.type == cudaMemoryTypeHost;
  if (*host)
    return cudaSuccess;
  void *view = nullptr;
  const bool peer = attr.type == cudaMemoryTypeDevice && attr.device != device && peer_access_recorded(device, attr.device);
  return kernel_view(ptr, attr, device, peer, host_memory::refuse, &view);
}

// Dynamic shared memory of digits_histogram_kernel: a counter per (pass,
// window, digit) and one per window for zero digits.
static size_t digit_histogram_smem(unsigned windows, unsigned passes) { return ((size_t)passes * windows * SORT_RADIX + windows) * 4; }

// The largest of those over the window widths that use the kernel.
static size_t max_digit_histogram_smem() {
  size_t most = 0;
  for (unsigned c = 2; c <= 24; c++) {
    const unsigned windows = (RESULT_BITS + c - 1) / c, passes = (c - 1 + SORT_RADIX_BITS - 1) / SORT_RADIX_BITS;
    if (windows <= MAX_FUSED_HISTOGRAM_WINDOWS)
      most = std::max(most, digit_histogram_smem(windows, passes));
  }
  return most;
}

// Stage boundaries: optional caller events recorded before the first stage and
// after each of the PROFILE_STAGES stages, and a count of kernels enqueued.
struct stage_marks {
  cudaEvent_t *events = nullptr;
  unsigned next = 0;
  unsigned launched = 0;
  cudaError_t mark(cudaStream_t stream) { return events ? cudaEventRecord(events[next++], stream) : cudaSuccess; }
};

// Stages 1-5 for the points of one plan: digits, sort, zero counts,
// accumulation and head merge into (buckets, flags).  Flags must be zero for
// buckets that hold nothing yet.
static cudaError_t enqueue_accumulation(const plan &p, const fe *scalars, const affine *bases, xyzz *buckets, uint8_t *flags, uint8_t *scratch,
                                        const layout &l, cudaStream_t stream, stage_marks &m) {
  uint32_t *keys[2] = {reinterpret_cast<uint32_t *>(scratch + l.keys[0]), reinterpret_cast<uint32_t *>(scratch + l.keys[1])};
  uint32_t *vals[2] = {reinterpret_cast<uint32_t *>(scratch + l.vals[0]), reinterpret_cast<uint32_t *>(scratch + l.vals[1])};
  uint32_t *counts = reinterpret_cast<uint32_t *>(scratch + l.counts);
  uint32_t *totals = reinterpret_cast<uint32_t *>(scratch + l.totals);
  uint32_t *zeros = reinterpret_cast<uint32_t *>(scratch + l.zeros);
  uint32_t *hb[2] = {reinterpret_cast<uint32_t *>(scratch + l.hb[0]), reinterpret_cast<uint32_t *>(scratch + l.hb[1])};
  xyzz *hp[2] = {reinterpret_cast<xyzz *>(scratch + l.hp[0]), reinterpret_cast<xyzz *>(scratch + l.hp[1])};
  const unsigned n = p.n;

  unsigned *sort_ctrs = reinterpret_cast<unsigned *>(scratch + l.sort_ctrs);
  unsigned *sort_error = reinterpret_cast<unsigned *>(scratch + l.sort_error);
  CHECK(cudaMemsetAsync(totals, 0, l.sort_clear_bytes, stream));
  int cur = 0;
  if (p.windows <= MAX_FUSED_HISTOGRAM_WINDOWS && p.tiles >= FUSED_DIGITS_MIN_TILES) {
    // 1. digits, with every pass's digit counts per tile
    digits_histogram_kernel<<<p.tiles, SORT_THREADS, digit_histogram_smem(p.windows, p.sort_passes), stream>>>(
        scalars, n, p.c, p.windows, p.sort_passes, p.tiles, keys[0], vals[0], counts, totals, zeros);
    CHECK(cudaGetLastError());
    m.launched++;
    CHECK(m.mark(stream));
    // 2. sort: one scan for the first pass's tile offsets and digit totals,
    // the first pass (drops zero digits), then one look-back kernel per later
    // 8-bit pass (their digit totals come from the digit kernel)
    const unsigned prefix_rows = p.windows * SORT_RADIX;
    sort_scan_kernel<<<(prefix_rows * 32 + 255) / 256, 256, 0, stream>>>(counts, p.tiles, prefix_rows, totals);
    CHECK(cudaGetLastError());
    const dim3 grid(p.tiles, p.windows);
    sort_scatter_first_kernel<<<grid, SORT_THREADS, 0, stream>>>(keys[0], vals[0], keys[1], vals[1], n, p.tiles, 0, counts, totals, zeros);
    CHECK(cudaGetLastError());
    m.launched += 2;
    cur = 1;
    uint32_t *words = reinterpret_cast<uint32_t *>(scratch + l.lookback_words);
    for (unsigned pass = 1; pass < p.sort_passes; pass++) {
      lookback_stable_kernel<<<p.windows * p.lookback_tiles, LOOKBACK_THREADS, lookback_smem_bytes<LOOKBACK_THREADS, LOOKBACK_ITEMS>(), stream>>>(
          keys[cur], vals[cur], keys[cur ^ 1], vals[cur ^ 1], n, p.windows, p.lookback_tiles, pass * SORT_RADIX_BITS,
          words + (size_t)(pass - 1) * p.windows * p.lookback_tiles * SORT_RADIX, totals + (size_t)pass * prefix_rows, zeros, sort_ctrs + pass,
          sort_error);
      CHECK(cudaGetLastError());
      m.launched++;
      cur ^= 1;
    }
  } else {
    // 1. digits (c <= 5: more windows than the digit kernel can count)
    digits_kernel<<<(n + 255) / 256, 256, 0, stream>>>(scalars, n, p.c, p.windows, keys[0], vals[0]);
    CHECK(cudaGetLastError());
    m.launched++;
    CHECK(m.mark(stream));
    // 2. sort, 8 bits per pass: histogram, scan and scatter kernels
    const unsigned rows = p.windows * SORT_RADIX;
    for (unsigned pass = 0; pass < p.sort_passes; pass++) {
      const unsigned shift = pass * SORT_RADIX_BITS;
      const dim3 grid(p.tiles, p.windows);
      if (pass == 0)
        sort_histogram_first_kernel<<<grid, SORT_THREADS, 0, stream>>>(keys[cur], n, p.tiles, shift, counts, zeros);
      else
        sort_histogram_kernel<<<grid, SORT_THREADS, 0, stream>>>(keys[cur], n, p.tiles, shift, counts, zeros);
      CHECK(cudaGetLastError());
      sort_scan_kernel<<<(rows * 32 + 255) / 256, 256, 0, stream>>>(counts, p.tiles, rows, totals);
      CHECK(cudaGetLastError());
      if (pass == 0)
        sort_scatter_first_kernel<<<grid, SORT_THREADS, 0, stream>>>(keys[cur], vals[cur], keys[cur ^ 1], vals[cur ^ 1], n, p.tiles, shift, counts,
                                                                     totals, zeros);
      else
        sort_scatter_stable_kernel<<<grid, SORT_THREADS, 0, stream>>>(keys[cur], vals[cur], keys[cur ^ 1], vals[cur ^ 1], n, p.tiles, shift, counts,
                                                                      totals, zeros);
      CHECK(cudaGetLastError());
      m.launched += 3;
      cur ^= 1;
    }
  }
  CHECK(m.mark(stream));

  // 3. zero digits: counted by the first sort pass (the stage is empty)
  CHECK(m.mark(stream));

  // 4. accumulation: the affine pairing levels, if any, then the XYZZ pass
  unsigned *work = reinterpret_cast<unsigned *>(scratch + l.work);
  CHECK(cudaMemsetAsync(work, 0, sizeof(unsigned), stream));
  if (p.affine_levels) {
    uint32_t *list_buckets[2] = {reinterpret_cast<uint32_t *>(scratch + l.level_buckets[0]),
                                 reinterpret_cast<uint32_t *>(scratch + l.level_buckets[1])};
    affine *list_points[2] = {reinterpret_cast<affine *>(scratch + l.level_points[0]), reinterpret_cast<affine *>(scratch + l.level_points[1])};
    unsigned long long *counts_out = reinterpret_cast<unsigned long long *>(scratch + l.level_counts);
    level_arrays a{};
    a.pre = reinterpret_cast<fe *>(scratch + l.level_pre);
    a.others = reinterpret_cast<fe *>(scratch + l.level_others);
    a.warp_total = reinterpret_cast<fe *>(scratch + l.level_total);
    a.warp_inverse = reinterpret_cast<fe *>(scratch + l.level_inverse);
    a.warp_outputs = reinterpret_cast<uint32_t *>(scratch + l.level_outputs);
    a.warp_base = reinterpret_cast<unsigned long long *>(scratch + l.level_base);
    const unsigned warps = p.level_warps;
    const unsigned forward_blocks = (warps * 32 + AFFINE_FORWARD_THREADS - 1) / AFFINE_FORWARD_THREADS;
    const unsigned apply_blocks = (warps * 32 + AFFINE_APPLY_THREADS - 1) / AFFINE_APPLY_THREADS;
    for (unsigned level = 1; level <= p.affine_levels; level++) {
      const int out = (level - 1) & 1, in = level & 1;
      a.count_out = counts_out + level;
      a.out_buckets = list_buckets[out];
      a.out_points = list_points[out];
      if (level == 1)
        affine_forward_first_kernel<<<forward_blocks, AFFINE_FORWARD_THREADS, 0, stream>>>(keys[cur], vals[cur], bases, n, p.windows, p.log_b, zeros,
                                                                                           a, warps);
      else
        affine_forward_list_kernel<<<forward_blocks, AFFINE_FORWARD_THREADS, 0, stream>>>(list_buckets[in], list_points[in], counts_out + level - 1,
                                                                                          a, warps);
      CHECK(cudaGetLastError());
      affine_invert_kernel<<<1, AFFINE_INVERT_THREADS, 0, stream>>>(a.warp_total, a.warp_outputs, warps, a.warp_inverse, a.warp_base, a.count_out);
      CHECK(cudaGetLastError());
      if (level == 1)
        affine_apply_first_kernel<<<apply_blocks, AFFINE_APPLY_THREADS, 0, stream>>>(keys[cur], vals[cur], bases, n, p.windows, p.log_b, zeros, a,
                                                                                       warps);
      else
        affine_apply_list_kernel<<<apply_blocks, AFFINE_APPLY_THREADS, 0, stream>>>(list_buckets[in], list_points[in], counts_out + level - 1, a,
                                                                                     warps);
      CHECK(cudaGetLastError());
      m.launched += 3;
    }
    const int last = (p.affine_levels - 1) & 1;
    accumulate_list_kernel<<<(p.tail_threads + ACC_THREADS - 1) / ACC_THREADS, ACC_THREADS, 0, stream>>>(
        list_buckets[last], list_points[last], counts_out + p.affine_levels, p.tail_ranges, work, buckets, flags, hb[0], hp[0]);
  } else {
    accumulate_kernel<<<(p.acc_threads + ACC_THREADS - 1) / ACC_THREADS, ACC_THREADS, 0, stream>>>(
        keys[cur], vals[cur], bases, n, p.windows, p.log_b, zeros, p.acc_ranges, work, buckets, flags, hb[0], hp[0]);
  }
  CHECK(cudaGetLastError());
  m.launched++;
  CHECK(m.mark(stream));

  // 5. heads
  CHECK(enqueue_merge_heads(hb, hp, p.tail_ranges, buckets, p.sms, stream, m.launched));
  CHECK(m.mark(stream));
  return cudaSuccess;
}

// Levels of at most this many heads per SM (a few warps per SM either way:
// the launch's time is one chain of dependent additions) take the 4-lane
// merge, 8 heads per warp with each addition in rounds of independent
// products.  Every level that way measured slower (2^12: 0.089 -> 0.123 ms,
// 2^22: 0.081 -> 0.136 ms: more levels); with this threshold the head-merge
// stage at 2^14 0.136 -> 0.118 ms, at 2^16 0.157 -> 0.146 ms, at 2^22
// 0.081 -> 0.089 ms.  A choice per level by modelled costs (about 25 us per
// 32-head level, 14 us per 4-lane level) measured no better overall
// (0.134 ms at 2^14, 0.084 at 2^22).
constexpr unsigned MERGE_GROUP4_HEADS_PER_SM = 32;

cudaError_t enqueue_merge_heads(uint32_t *const hb[2], xyzz *const hp[2], unsigned heads, xyzz *buckets, unsigned sms, cudaStream_t stream,
                                unsigned &launched) {
  int h = 0;
  while (heads > 1) {
    const bool small = heads <= (unsigned long long)sms * MERGE_GROUP4_HEADS_PER_SM;
    const unsigned per_warp = small ? MERGE_HEADS_PER_WARP_GROUP4 : MERGE_HEADS_PER_WARP;
    const unsigned out = (heads + per_warp - 1) / per_warp;
    const unsigned blocks = (unsigned)(((unsigned long long)out * 32 + ACC_THREADS - 1) / ACC_THREADS);
    if (small)
      merge_heads_group4_kernel<<<blocks, ACC_THREADS, 0, stream>>>(hb[h], hp[h], heads, buckets, hb[h ^ 1], hp[h ^ 1]);
    else
      merge_heads_kernel<<<blocks, ACC_THREADS, 0, stream>>>(hb[h], hp[h], heads, buckets, hb[h ^ 1], hp[h ^ 1]);
    CHECK(cudaGetLastError());
    launched++;
    heads = out;
    h ^= 1;
  }
  return cudaSuccess;
}

// Stage 6: bucket reduction of (buckets, flags) into the 254 results.  Blocks
// of ACC_THREADS: at 2^22, blocks of 64 threads measured the same and blocks
// of 96 slower (reduction 0.695 -> 0.815 ms).
cudaError_t enqueue_window_sums(const plan &p, const xyzz *buckets, const uint8_t *flags, xyzz *const tree[2], xyzz *const streams[2],
                                cudaStream_t stream, unsigned &launched) {
  // Launches with fewer jobs than one block of ACC_THREADS per SM run a group
  // of four lanes per job (msm_group4.cuh): there each job's chain of
  // additions is the launch's latency, and four times the threads still fit.
  const unsigned small = p.sms * ACC_THREADS;
  auto blocks = [](unsigned long long threads) { return (unsigned)((threads + ACC_THREADS - 1) / ACC_THREADS); };
  const unsigned group_threads = p.windows << p.log_g;
  if (group_threads <= small)
    reduce_groups_group4_kernel<<<blocks(4ull * group_threads), ACC_THREADS, 0, stream>>>(buckets, flags, p.windows, p.log_b, p.log_m, tree[0],
                                                                                          streams[0]);
  else
    reduce_groups_kernel<<<blocks(group_threads), ACC_THREADS, 0, stream>>>(buckets, flags, p.windows, p.log_b, p.log_m, tree[0], streams[0]);
  CHECK(cudaGetLastError());
  launched++;
  for (unsigned level = 0; level < p.log_g; level++) {
    const unsigned threads = p.windows * (level + 2) * ((1u << p.log_g) >> (level + 1));
    const int in = level & 1;
    if (threads <= small)
      reduce_level_group4_kernel<<<blocks(4ull * threads), ACC_THREADS, 0, stream>>>(tree[in], tree[in ^ 1], streams[in], streams[in ^ 1],
                                                                                      p.windows, p.log_g, level);
    else
      reduce_level_kernel<<<blocks(threads), ACC_THREADS, 0, stream>>>(tree[in], tree[in ^ 1], streams[in], streams[in ^ 1], p.windows, p.log_g,
                                                                       level);
    CHECK(cudaGetLastError());
    launched++;
  }
  return cudaSuccess;
}

static cudaError_t enqueue_reduction(const plan &p, const xyzz *buckets, const uint8_t *flags, jacobian *results, uint8_t *scratch, const layout &l,
                                     cudaStream_t stream, stage_marks &m) {
  xyzz *const tree[2] = {reinterpret_cast<xyzz *>(scratch + l.tree[0]), reinterpret_cast<xyzz *>(scratch + l.tree[1])};
  xyzz *const streams[2] = {reinterpret_cast<xyzz *>(scratch + l.streams[0]), reinterpret_cast<xyzz *>(scratch + l.streams[1])};
  CHECK(enqueue_window_sums(p, buckets, flags, tree, streams, stream, m.launched));
  gather_results_kernel<<<(RESULT_BITS + 127) / 128, 128, 0, stream>>>(streams[p.log_g & 1], buckets, flags, p.windows, p.c, p.log_m, p.log_g,
                                                                       results);
  CHECK(cudaGetLastError());
  m.launched++;
  CHECK(m.mark(stream));
  return cudaSuccess;
}

// Enqueue the kernels of one MSM whose inputs are on the device.
// stage_events (optional): PROFILE_STAGES + 1 events recorded before the first
// stage and after each stage.  launches (optional): kernels enqueued.
cudaError_t enqueue_pipeline(const plan &p, const fe *scalars, const affine *bases, jacobian *results, uint8_t *scratch, const layout &l,
                             cudaStream_t stream, cudaEvent_t *stage_events = nullptr, unsigned *launches = nullptr) {
  stage_marks m;
  m.events = stage_events;
  xyzz *buckets = reinterpret_cast<xyzz *>(scratch + l.buckets);
  uint8_t *flags = scratch + l.flags;
  CHECK(cudaMemsetAsync(flags, 0, (size_t)p.windows << p.log_b, stream));
  CHECK(m.mark(stream));
  CHECK(enqueue_accumulation(p, scalars, bases, buckets, flags, scratch, l, stream, m));
  CHECK(enqueue_reduction(p, buckets, flags, results, scratch, l, stream, m));
  if (launches)
    *launches = m.launched;
  return cudaSuccess;
}

// Synchronises the stream, then reads the stage times and the work counts
// that the scratch buffers still hold.
static cudaError_t collect_profile(const plan &p, const layout &l, const uint8_t *scratch, cudaStream_t stream, const cudaEvent_t *events,
                                   unsigned launches, msm_b200_profile *out) {
  CHECK(cudaStreamSynchronize(stream));
  *out = msm_b200_profile{};
  for (unsigned s = 0; s < PROFILE_STAGES; s++)
    CHECK(cudaEventElapsedTime(&out->stage_ms[s], events[s], events[s + 1]));
  std::vector<uint32_t> zeros(p.windows);
  CHECK(cudaMemcpy(zeros.data(), scratch + l.zeros, zeros.size() * 4, cudaMemcpyDeviceToHost));
  uint32_t sort_error = 0;
  CHECK(cudaMemcpy(&sort_error, scratch + l.sort_error, 4, cudaMemcpyDeviceToHost));
  std::vector<uint8_t> flags((size_t)p.windows << p.log_b);
  CHECK(cudaMemcpy(flags.data(), scratch + l.flags, flags.size(), cudaMemcpyDeviceToHost));
  std::vector<uint32_t> heads(p.tail_ranges);
  CHECK(cudaMemcpy(heads.data(), scratch + l.hb[0], heads.size() * 4, cudaMemcpyDeviceToHost));
  unsigned long long left = 0; // elements the affine levels left for the XYZZ pass
  if (p.affine_levels)
    CHECK(cudaMemcpy(&left, scratch + l.level_counts + p.affine_levels * 8, 8, cudaMemcpyDeviceToHost));
  unsigned long long nonzero = 0, nonempty = 0, continued = 0;
  for (uint32_t z : zeros)
    nonzero += p.n - z;
  for (uint8_t f : flags)
    nonempty += f != 0;
  for (uint32_t h : heads)
    continued += h != INVALID_BUCKET;
  out->nonzero_entries = nonzero;
  out->nonempty_buckets = nonempty;
  out->heads = continued;
  out->window_bits = p.c;
  out->windows = p.windows;
  out->acc_threads = p.tail_ranges;
  out->launches = launches;
  out->sort_wait_timeouts = sort_error;
  out->affine_levels = p.affine_levels;
  out->affine_additions = p.affine_levels ? nonzero - left : 0;
  return cudaSuccess;
}

// Events and the helper stream of a chunked MSM, released when the call ends
// (the CUDA runtime defers the release of a stream or event until its pending
// work completes).
struct chunk_resources {
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ready = nullptr, copies_done = nullptr;
  std::vector<cudaEvent_t> copied, consumed;
  ~chunk_resources() {
    for (const std::vector<cudaEvent_t> *v : {&copied, &consumed})
      for (cudaEvent_t e : *v)
        if (e)
          cudaEventDestroy(e);
    if (ready)
      cudaEventDestroy(ready);
    if (copies_done)
      cudaEventDestroy(copies_done);
    if (copy_stream)
      cudaStreamDestroy(copy_stream);
  }
};

// A chunked MSM: host-resident inputs (see make_chunks), or any inputs whose
// whole-size scratch did not fit (the out-of-memory fit in execute).  Chunk 0
// accumulates into the MSM's buckets, every later chunk into a second bucket
// set that is folded in; the reduction runs once.  With host inputs, copy j + 1
// runs on a helper stream while chunk j computes; with two copy slots
// (ch.slots), the copy into a slot also waits until the chunk that used the
// slot before has finished reading it.
static cudaError_t enqueue_chunked(const execution &e, const chunking &ch, const plan &full, unsigned sms, bool copy_scalars, bool copy_bases,
                                   jacobian *device_results, uint8_t *scratch, const layout &l) {
  cudaStream_t stream = e.stream;
  const bool copying = copy_scalars || copy_bases;
  chunk_resources r;
  fe *scalars = reinterpret_cast<fe *>(scratch + l.scalars);
  affine *bases = reinterpret_cast<affine *>(scratch + l.bases);
  if (copying) {
    CHECK(cudaStreamCreateWithFlags(&r.copy_stream, cudaStreamNonBlocking));
    CHECK(cudaEventCreateWithFlags(&r.ready, cudaEventDisableTiming));
    CHECK(cudaEventCreateWithFlags(&r.copies_done, cudaEventDisableTiming));
    r.copied.assign(ch.count, nullptr);
    r.consumed.assign(ch.count, nullptr);
    for (unsigned j = 0; j < ch.count; j++) {
      CHECK(cudaEventCreateWithFlags(&r.copied[j], cudaEventDisableTiming));
      if (ch.slots)
        CHECK(cudaEventCreateWithFlags(&r.consumed[j], cudaEventDisableTiming));
    }
    // the copies go into scratch allocated in the caller's stream order
    CHECK(cudaEventRecord(r.ready, stream));
    CHECK(cudaStreamWaitEvent(r.copy_stream, r.ready, 0));
  }
  auto enqueue_copy = [&](unsigned j) -> cudaError_t {
    const unsigned b = ch.beg[j], cnt = ch.size(j);
    const size_t at = ch.slot_offset(j);
    if (ch.slots && j >= ch.slots) // the slot's previous chunk must be done with it
      CHECK(cudaStreamWaitEvent(r.copy_stream, r.consumed[j - ch.slots], 0));
    if (copy_scalars)
      CHECK(cudaMemcpyAsync(scalars + at, static_cast<const fe *>(e.scalars) + b, (size_t)cnt * sizeof(fe), cudaMemcpyHostToDevice, r.copy_stream));
    if (copy_bases)
      CHECK(cudaMemcpyAsync(bases + at, static_cast<const affine *>(e.bases) + b, (size_t)cnt * sizeof(affine), cudaMemcpyHostToDevice,
                            r.copy_stream));
    CHECK(cudaEventRecord(r.copied[j], r.copy_stream));
    if (j + 1 == ch.count) {
      if (e.h2d_event)
        CHECK(cudaEventRecord(e.h2d_event, r.copy_stream));
      if (e.h2d_callback)
        CHECK(cudaLaunchHostFunc(r.copy_stream, e.h2d_callback, e.h2d_callback_data));
      CHECK(cudaEventRecord(r.copies_done, r.copy_stream));
    }
    return cudaSuccess;
  };

  xyzz *buckets = reinterpret_cast<xyzz *>(scratch + l.buckets);
  uint8_t *flags = scratch + l.flags;
  xyzz *chunk_buckets = reinterpret_cast<xyzz *>(scratch + l.chunk_buckets);
  uint8_t *chunk_flags = scratch + l.chunk_flags;
  const size_t slots = (size_t)full.windows << full.log_b;
  stage_marks m;
  CHECK(cudaMemsetAsync(flags, 0, slots, stream));
  // copy j + 1 is enqueued before chunk j's kernels, so that the host thread
  // (which stages pageable copies itself) never holds back enqueued work
  if (copying)
    CHECK(enqueue_copy(0));
  for (unsigned j = 0; j < ch.count; j++) {
    if (copying && j + 1 < ch.count)
      CHECK(enqueue_copy(j + 1));
    const unsigned b = ch.beg[j];
    const plan p = make_plan(ch.size(j), full.c, sms);
    const fe *src_scalars = copy_scalars ? scalars + ch.slot_offset(j) : static_cast<const fe *>(e.scalars) + b;
    const affine *src_bases = copy_bases ? bases + ch.slot_offset(j) : static_cast<const affine *>(e.bases) + b;
    if (copying)
      CHECK(cudaStreamWaitEvent(stream, r.copied[j], 0));
    if (j == 0) {
      CHECK(enqueue_accumulation(p, src_scalars, src_bases, buckets, flags, scratch, l, stream, m));
    } else {
      CHECK(cudaMemsetAsync(chunk_flags, 0, slots, stream));
      CHECK(enqueue_accumulation(p, src_scalars, src_bases, chunk_buckets, chunk_flags, scratch, l, stream, m));
      merge_chunk_buckets_kernel<<<(unsigned)((slots + ACC_THREADS - 1) / ACC_THREADS), ACC_THREADS, 0, stream>>>(buckets, flags, chunk_buckets,
                                                                                                                 chunk_flags, (unsigned)slots);
      CHECK(cudaGetLastError());
    }
    if (copying && ch.slots)
      CHECK(cudaEventRecord(r.consumed[j], stream));
  }
  CHECK(enqueue_reduction(full, buckets, flags, device_results, scratch, l, stream, m));
  // the call's stream completes after the copies and the h2d callback
  if (copying)
    CHECK(cudaStreamWaitEvent(stream, r.copies_done, 0));
  return cudaSuccess;
}

// One pool allocation of `bytes` on the call's stream; false with no error
// when the pool (or the device) cannot hold it, so that the caller can try
// smaller chunks.  The failed allocation leaves nothing behind; its error is
// cleared from the runtime's last-error state, as the reference's fit loop
// does (src/msm.cu:442-446).
static cudaError_t allocate_scratch(const execution &e, size_t bytes, void **raw, bool *fits) {
  const cudaError_t err = e.pool ? cudaMallocFromPoolAsync(raw, bytes, e.pool, e.stream) : cudaMallocAsync(raw, bytes, e.stream);
  *fits = err == cudaSuccess;
  if (err == cudaErrorMemoryAllocation) {
    const cudaError_t last = cudaGetLastError();
    return last == cudaErrorMemoryAllocation ? cudaSuccess : last;
  }
  return err;
}

cudaError_t execute(const execution &e) {
  if (e.count == 0 || e.count > (1u << 31) || !e.scalars || !e.bases || !e.results)
    return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(e.bases) & 15) || (reinterpret_cast<uintptr_t>(e.scalars) & 15))
    return cudaErrorInvalidValue;
  if (e.window_bits && (e.window_bits < 2 || e.window_bits > 24))
    return cudaErrorInvalidValue;
  int device = 0;
  CHECK(cudaGetDevice(&device));
  bool copy_scalars = false, copy_bases = false, copy_results = false;
  CHECK(locate(e.scalars, device, &copy_scalars));
  CHECK(locate(e.bases, device, &copy_bases));
  CHECK(locate(e.results, device, &copy_results));
  const int sms = get_device_info(device).sms;
  const bool instrumented = e.profile || e.stage_events;
  const plan p = make_plan(e.count, e.window_bits, sms);
  if (p.windows > 128)
    return cudaErrorInvalidValue;
  // Memory fit (reference: the dry-run loop of msm::execute_async,
  // src/msm.cu:431-459): when the pool cannot hold the scratch of the chosen
  // chunking, the largest chunk is halved -- equal chunks, host inputs through
  // two chunk-sized copy slots -- down to MIN_FIT_CHUNK points, after which
  // the call fails with cudaErrorMemoryAllocation.  Device-resident inputs
  // start as one chunk.  The instrumented entry points run unchunked.
  chunking ch = make_chunks(e.count, (copy_scalars || copy_bases) && !instrumented);
  if (ch.largest() > MAX_CHUNK_POINTS) {
    if (instrumented)
      return cudaErrorInvalidValue;
    ch = equal_chunks(e.count, MAX_CHUNK_POINTS, copy_scalars || copy_bases);
  }
  layout l{};
  void *raw = nullptr;
  for (;;) {
    l = chunked_layout(e.count, p.c, sms, ch, copy_scalars, copy_bases, copy_results);
    bool fits = false;
    CHECK(allocate_scratch(e, l.total, &raw, &fits));
    if (fits)
      break;
    const unsigned largest = ch.largest();
    if (instrumented || largest <= MIN_FIT_CHUNK)
      return cudaErrorMemoryAllocation;
    ch = equal_chunks(e.count, std::max(MIN_FIT_CHUNK, (largest + 1) / 2), copy_scalars || copy_bases);
  }
  cudaStream_t stream = e.stream;
  uint8_t *scratch = static_cast<uint8_t *>(raw);
  cudaError_t status = cudaSuccess;
  do {
    const fe *scalars = static_cast<const fe *>(e.scalars);
    const affine *bases = static_cast<const affine *>(e.bases);
    jacobian *results = static_cast<jacobian *>(e.results);
    jacobian *device_results = copy_results ? reinterpret_cast<jacobian *>(scratch + l.results) : results;
    if (ch.count > 1) {
      if ((status = enqueue_chunked(e, ch, p, sms, copy_scalars, copy_bases, device_results, scratch, l)) != cudaSuccess)
        break;
    } else {
      if (copy_scalars) {
        if ((status = cudaMemcpyAsync(scratch + l.scalars, e.scalars, (size_t)p.n * sizeof(fe), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
          break;
        scalars = reinterpret_cast<const fe *>(scratch + l.scalars);
      }
      if (copy_bases) {
        if ((status = cudaMemcpyAsync(scratch + l.bases, e.bases, (size_t)p.n * sizeof(affine), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
          break;
        bases = reinterpret_cast<const affine *>(scratch + l.bases);
      }
      if (copy_scalars || copy_bases) {
        if (e.h2d_event && (status = cudaEventRecord(e.h2d_event, stream)) != cudaSuccess)
          break;
        if (e.h2d_callback && (status = cudaLaunchHostFunc(stream, e.h2d_callback, e.h2d_callback_data)) != cudaSuccess)
          break;
      }
      cudaEvent_t events[PROFILE_STAGES + 1] = {};
      const cudaEvent_t *stage_events = e.stage_events;
      if (e.profile) {
        for (auto &ev : events)
          if ((status = cudaEventCreate(&ev)) != cudaSuccess)
            break;
        if (status != cudaSuccess)
          break;
      }
      unsigned launches = 0;
      if (e.profile)
        stage_events = events;
      if ((status = enqueue_pipeline(p, scalars, bases, device_results, scratch, l, stream, const_cast<cudaEvent_t *>(stage_events), &launches)) !=
          cudaSuccess)
        break;
      if (e.launches)
        *e.launches = launches;
      if (e.profile) {
        status = collect_profile(p, l, scratch, stream, events, launches, e.profile);
        for (auto &ev : events)
          cudaEventDestroy(ev);
        if (status != cudaSuccess)
          break;
      }
    }
    if (copy_results) {
      if ((status = cudaMemcpyAsync(e.results, device_results, RESULT_BITS * sizeof(jacobian), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        break;
      if (e.d2h_event && (status = cudaEventRecord(e.d2h_event, stream)) != cudaSuccess)
        break;
      if (e.d2h_callback && (status = cudaLaunchHostFunc(stream, e.d2h_callback, e.d2h_callback_data)) != cudaSuccess)
        break;
    }
  } while (false);
  const cudaError_t free_status = cudaFreeAsync(raw, stream);
  return status != cudaSuccess ? status : free_status;
}

#ifndef ACC_CARVEOUT
#define ACC_CARVEOUT 40
#endif

// Shared-memory carveout preference (percent of the maximum): as much L1 as
// still lets the kernel reach its full occupancy.
template <class F> static cudaError_t set_carveout(F *func, int percent) {
  CHECK(cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, percent));
  return cudaSuccess;
}

cudaError_t set_up() {
  CHECK(cudaFuncSetAttribute(digits_histogram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_digit_histogram_smem()));
  CHECK(set_carveout(accumulate_kernel, ACC_CARVEOUT)); // 4 blocks x 19 KB of base-point slots and window bounds
  CHECK(set_carveout(lookback_stable_kernel, cudaSharedmemCarveoutMaxShared)); // 4 blocks x 42 KB
  CHECK(set_carveout(merge_heads_kernel, cudaSharedmemCarveoutMaxL1));
  CHECK(set_carveout(reduce_groups_kernel, cudaSharedmemCarveoutMaxL1));
  CHECK(set_carveout(reduce_level_kernel, cudaSharedmemCarveoutMaxL1));
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// MSM without allocation: scratch in a fixed block of device memory that is
// part of the library image, for callers that cannot allocate at call time.
// ---------------------------------------------------------------------------
static_assert(MSM_B200_NO_ALLOC_SCRATCH_BYTES % 256 == 0, "scratch block size");
static __device__ __align__(256) uint8_t no_alloc_scratch[MSM_B200_NO_ALLOC_SCRATCH_BYTES];

// Unique id of the calling thread's current CUDA context (cuCtxGetCurrent,
// cuCtxGetId, reached through the runtime's driver entry points so that the
// library keeps no link-time dependency on the driver library).
static cudaError_t current_context_id(unsigned long long *id) {
  using get_current_fn = CUresult (*)(CUcontext *);
  using get_id_fn = CUresult (*)(CUcontext, unsigned long long *);
  static std::once_flag once;
  static get_current_fn get_current = nullptr;
  static get_id_fn get_id = nullptr;
  static cudaError_t resolved = cudaSuccess;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSuccess;
    void *fn = nullptr;
    resolved = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &found);
    if (resolved == cudaSuccess && found != cudaDriverEntryPointSuccess)
      resolved = cudaErrorNotSupported;
    get_current = reinterpret_cast<get_current_fn>(fn);
    if (resolved == cudaSuccess) {
      resolved = cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &found);
      if (resolved == cudaSuccess && found != cudaDriverEntryPointSuccess)
        resolved = cudaErrorNotSupported;
      get_id = reinterpret_cast<get_id_fn>(fn);
    }
  });
  CHECK(resolved);
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx)
    return cudaErrorIncompatibleDriverContext;
  if (get_id(ctx, id) != CUDA_SUCCESS)
    return cudaErrorIncompatibleDriverContext;
  return cudaSuccess;
}

// Device address of no_alloc_scratch in the current context.  In host code
// the symbol is only a host-side handle; the address comes from
// cudaGetSymbolAddress, looked up once per context (each context loads the
// library's module, and with it the block, at its own address) and cached by
// the context's unique id, so a reset device or a caller's own context gets
// its own lookup.
static cudaError_t no_alloc_scratch_address(uint8_t **address) {
  static context_cache<uint8_t *> cache;
  unsigned long long id = 0;
  CHECK(current_context_id(&id));
  return cache.get(id, address, [](uint8_t *&ptr) {
    void *raw = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&raw, no_alloc_scratch);
    ptr = static_cast<uint8_t *>(raw);
    return err;
  });
}

cudaError_t execute_no_alloc(cudaStream_t stream, const void *bases, const void *scalars, void *results, unsigned count) {
  if (count == 0 || count > MSM_B200_NO_ALLOC_MAX_COUNT || !bases || !scalars || !results)
    return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(bases) & 15) || (reinterpret_cast<uintptr_t>(scalars) & 15) || (reinterpret_cast<uintptr_t>(results) & 15))
    return cudaErrorInvalidValue;
  int device = 0;
  CHECK(cudaGetDevice(&device));
  for (const void *ptr : {bases, scalars, static_cast<const void *>(results)}) {
    bool host = false;
    CHECK(locate(ptr, device, &host));
    if (host)
      return cudaErrorInvalidValue;
  }
  plan p = make_plan(count, 0, get_device_info(device).sms);
  set_affine_levels(p, 0);   // the fixed scratch holds no level lists
  set_reduction_groups(p, 3); // and the reduction's smallest tree (G = B / 8)
  const layout l = make_layout(p, false, false, false);
  if (l.total > MSM_B200_NO_ALLOC_SCRATCH_BYTES) // only on GPUs far larger than a B200 (heads grow with the SM count)
    return cudaErrorInvalidValue;
  uint8_t *scratch = nullptr;
  CHECK(no_alloc_scratch_address(&scratch));
  return enqueue_pipeline(p, static_cast<const fe *>(scalars), static_cast<const affine *>(bases), static_cast<jacobian *>(results), scratch, l,
                          stream);
}

} // namespace msm_b200

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

bc_error msm_set_up() { return static_cast<bc_error>(msm_b200::set_up()); }

bc_error msm_execute_async(const msm_configuration configuration) {
  if (configuration.log_scalars_count > 31)
    return bc_error_invalid_value;
  msm_b200::execution e{};
  e.pool = static_cast<cudaMemPool_t>(configuration.mem_pool.handle);
  e.stream = static_cast<cudaStream_t>(configuration.stream.handle);
  e.bases = configuration.bases;
  e.scalars = configuration.scalars;
  e.results = configuration.results;
  e.count = 1u << configuration.log_scalars_count;
  e.window_bits = 0;
  e.h2d_event = static_cast<cudaEvent_t>(configuration.h2d_copy_finished.handle);
  e.h2d_callback = configuration.h2d_copy_finished_callback;
  e.h2d_callback_data = configuration.h2d_copy_finished_callback_data;
  e.d2h_event = static_cast<cudaEvent_t>(configuration.d2h_copy_finished.handle);
  e.d2h_callback = configuration.d2h_copy_finished_callback;
  e.d2h_callback_data = configuration.d2h_copy_finished_callback_data;
  return static_cast<bc_error>(msm_b200::execute(e));
}

bc_error msm_tear_down() { return bc_success; }

bc_error msm_b200_execute_async(const msm_b200_configuration *configuration) {
  if (!configuration)
    return bc_error_invalid_value;
  msm_b200::execution e{};
  e.pool = static_cast<cudaMemPool_t>(configuration->mem_pool.handle);
  e.stream = static_cast<cudaStream_t>(configuration->stream.handle);
  e.bases = configuration->bases;
  e.scalars = configuration->scalars;
  e.results = configuration->results;
  e.count = configuration->count;
  e.window_bits = configuration->window_bits;
  return static_cast<bc_error>(msm_b200::execute(e));
}

bc_error msm_b200_execute_profiled(const msm_b200_configuration *configuration, msm_b200_profile *profile) {
  if (!configuration || !profile)
    return bc_error_invalid_value;
  msm_b200::execution e{};
  e.pool = static_cast<cudaMemPool_t>(configuration->mem_pool.handle);
  e.stream = static_cast<cudaStream_t>(configuration->stream.handle);
  e.bases = configuration->bases;
  e.scalars = configuration->scalars;
  e.results = configuration->results;
  e.count = configuration->count;
  e.window_bits = configuration->window_bits;
  e.profile = profile;
  return static_cast<bc_error>(msm_b200::execute(e));
}

bc_error msm_b200_execute_staged_async(const msm_b200_configuration *configuration, const bc_event *stage_events, unsigned *launches) {
  if (!configuration || !stage_events)
    return bc_error_invalid_value;
  cudaEvent_t events[msm_b200::PROFILE_STAGES + 1];
  for (unsigned i = 0; i <= msm_b200::PROFILE_STAGES; i++)
    events[i] = static_cast<cudaEvent_t>(stage_events[i].handle);
  msm_b200::execution e{};
  e.pool = static_cast<cudaMemPool_t>(configuration->mem_pool.handle);
  e.stream = static_cast<cudaStream_t>(configuration->stream.handle);
  e.bases = configuration->bases;
  e.scalars = configuration->scalars;
  e.results = configuration->results;
  e.count = configuration->count;
  e.window_bits = configuration->window_bits;
  e.stage_events = events;
  e.launches = launches;
  return static_cast<bc_error>(msm_b200::execute(e));
}

bc_error msm_b200_scratch_bytes(unsigned count, unsigned window_bits, size_t *bytes) {
  if (!bytes || count == 0)
    return bc_error_invalid_value;
  *bytes = msm_b200::scratch_bytes(count, window_bits, false, false, false);
  return bc_success;
}

bc_error msm_b200_default_window_bits(unsigned count, unsigned *window_bits) {
  if (!window_bits || count == 0)
    return bc_error_invalid_value;
  *window_bits = msm_b200::default_window_bits(count);
  return bc_success;
}

bc_error msm_b200_set_affine_levels(int levels) {
  if (levels > (int)msm_b200::MAX_AFFINE_LEVELS)
    return bc_error_invalid_value;
  msm_b200::set_affine_levels_override(levels < 0 ? -1 : levels);
  return bc_success;
}

bc_error msm_b200_execute_no_alloc_async(bc_stream stream, const void *bases, const void *scalars, void *results, unsigned count) {
  return static_cast<bc_error>(msm_b200::execute_no_alloc(static_cast<cudaStream_t>(stream.handle), bases, scalars, results, count));
}

} // extern "C"
