// Batched MSM over one resident base table (no counterpart in the reference).
//
// A base table holds N affine points on the device and, for every window
// width c it is built for, the precomputed multiples
//     M_c[j][i] = 2^(c j) * P_i,   j < W(c) = ceil(254 / c),
// so that an MSM over a prefix of the table needs ONE set of 2^(c-1) buckets
// instead of W(c): the digit of window j of scalar i selects M_c[j][i].
//
// A batch is a fixed list of instance sizes n_k (any lengths, prefixes of the
// table).  All instances run as one kernel chain:
//   digits       every point of every instance, W(c_k) signed digits each, into
//                its instance's segment of W(c_k) windows of n_k rounded up
//                to whole sort tiles (the padding holds zero digits), with the
//                first radix pass's tile counts and every later pass's digit
//                totals per segment
//   sort         segmented LSD radix sort, tile list over all segments; the
//                first pass (scan + scatter) drops zero digits (counted per
//                segment), every later pass is one look-back kernel whose
//                tiles are handed out interleaved over the segments
//   accumulate   the nonzero entries of all segments split into equal ranges,
//                one per thread: the (instance, bucket-range) work list
//   merge heads  as in the plain pipeline
//   reduction    per group of instances with the same c (one "window" each),
//                the plain pipeline's reduction kernels on the group's buckets,
//                then a gather into each instance's 254 results
// The chain is captured once in a CUDA graph; every execution only writes the
// instances' scalar and result pointers and replays the graph.
#include "batch_tuning.h"
#include "bellman-cuda-b200.h"
#include "msm_device.cuh"
#include "msm_batch.cuh"
#include "msm_host.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <vector>

namespace msm_b200 {

#define CHECK(statement)                                                                                                                       \
  do {                                                                                                                                         \
    cudaError_t check_result_ = (statement);                                                                                                   \
    if (check_result_ != cudaSuccess)                                                                                                          \
      return check_result_;                                                                                                                    \
  } while (0)

constexpr unsigned IO_CHUNK = 64; // instances per descriptor-update launch

static unsigned ceil_log2_u(unsigned long long v) {
  unsigned r = 0;
  while ((1ull << r) < v)
    r++;
  return r;
}

static unsigned windows_for(unsigned c) { return (RESULT_BITS + c - 1) / c; }

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

unsigned batch_window_bits(unsigned n) {
  const unsigned lg = ceil_log2_u(n);
  for (const tuning_row &row : BATCH_TUNING)
    if (lg <= row.max_log_n)
      return row.window_bits;
  return BATCH_TUNING[sizeof(BATCH_TUNING) / sizeof(BATCH_TUNING[0]) - 1].window_bits;
}

// ---------------------------------------------------------------------------
// device descriptors
// ---------------------------------------------------------------------------


struct batch_io_update {
  batch_io io[IO_CHUNK];
  unsigned first, count;
};

__global__ void batch_set_io_kernel(batch_io *__restrict__ dst, batch_io_update u) {
  const unsigned k = threadIdx.x;
  if (k < u.count)
    dst[u.first + k] = u.io[k];
}

// 2^c * prev[i] for the points of one window multiple (one thread per point).
__global__ void __launch_bounds__(128) window_multiples_kernel(const affine *__restrict__ prev, affine *__restrict__ next, unsigned count,
                                                               unsigned c) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count)
    return;
  const affine a = prev[i];
  xyzz p = curve::dbl_affine(a);
  for (unsigned k = 1; k < c; k++)
    p = curve::dbl(p);
  next[i] = curve::to_affine(p); // 2^(cj) P is never infinity: the group order r is an odd prime
}

// One block per point tile (SORT_TILE consecutive points of one instance;
// the padding points n <= i < seg_stride hold zero digits): every window's
// signed digit of each point into the instance's segment (entry w *
// seg_stride + i, value = table index w * stride + i with the sign), and, in
// shared memory (windows x 256 counters), the tile's nonzero keys per window
// and low radix digit.  Since seg_stride is a whole number of sort tiles,
// the entries of window w of this point tile are exactly sort tile w *
// point_tiles + p of the segment, so these are the first radix pass's tile
// counts, written for batch_sort_scan_kernel (no histogram kernel for that
// pass).  Zero digits (padding included) are added to zeros[k].  The block
// also counts its nonzero keys per radix digit of every later pass and adds
// them to the instance's digit totals of that pass, later_totals[(pass - 1)
// * instances + k][digit], which the look-back passes need up front.
__global__ void __launch_bounds__(SORT_THREADS) batch_digits_histogram_kernel(const batch_instance *__restrict__ inst,
                                                                              const unsigned *__restrict__ ptile_seg, const batch_io *__restrict__ io,
                                                                              uint32_t *__restrict__ keys, uint32_t *__restrict__ vals,
                                                                              uint32_t *__restrict__ counts, uint32_t *__restrict__ zeros,
                                                                              unsigned instances, unsigned later_passes,
                                                                              uint32_t *__restrict__ later_totals) {
  // [windows][SORT_RADIX] first-pass counters, [later_passes][SORT_RADIX], then the zero-digit count
  extern __shared__ uint32_t s_hist[];
  const unsigned k = ptile_seg[blockIdx.x];
  const batch_instance d = inst[k];
  const unsigned tile = blockIdx.x - d.ptile_base, windows = d.windows;
  const unsigned counters = windows * SORT_RADIX, later = later_passes * SORT_RADIX;
  uint32_t *s_later = s_hist + counters;
  uint32_t *zero_digits = s_later + later;
  for (unsigned q = threadIdx.x; q <= counters + later; q += blockDim.x)
    s_hist[q] = 0;
  __syncthreads();
  const fe *scalars = io[k].scalars;
  const size_t S = d.seg_stride;
  const unsigned first = tile * SORT_TILE + threadIdx.x;
  uint32_t zero_count = 0;
  auto tile_digits = [&](auto width) {
    constexpr unsigned C = decltype(width)::value;
    // the next scalar is loaded before this one is decomposed
    fe next = fr::zero();
    if (first < d.n)
      next = load_fe_streaming(scalars + first);
    for (unsigned q = 0; q < SORT_ITEMS; q++) {
      const unsigned i = first + q * SORT_THREADS; // < seg_stride
      const fe scalar = next;
      if (q + 1 < SORT_ITEMS && i + SORT_THREADS < d.n)
        next = load_fe_streaming(scalars + i + SORT_THREADS);
      if (i < d.n) {
        scalar_digits_fixed<C>(scalar, d.c, windows, [&](unsigned w, uint32_t magnitude, uint32_t negative) {
          const size_t out = d.entry_offset + w * S + i;
          const uint32_t key = digit_key(magnitude);
          keys[out] = key;
          vals[out] = (w * d.stride + i) | (negative << 31);
          if (magnitude) {
            atomicAdd(&s_hist[w * SORT_RADIX + (key & (SORT_RADIX - 1))], 1u);
            for (unsigned p = 0; p < later_passes; p++)
              atomicAdd(&s_later[p * SORT_RADIX + ((key >> ((p + 1) * SORT_RADIX_BITS)) & (SORT_RADIX - 1))], 1u);
          } else {
            zero_count++;
          }
        });
      } else {
        for (unsigned w = 0; w < windows; w++) {
          keys[d.entry_offset + w * S + i] = ZERO_KEY;
          vals[d.entry_offset + w * S + i] = 0;
        }
        zero_count += windows;
      }
    }
  };
  // the widths the batch table picks for its large instances get unrolled code
  switch (d.c) {
  case 16: tile_digits(width_constant<16>{}); break;
  case 17: tile_digits(width_constant<17>{}); break;
  case 20: tile_digits(width_constant<20>{}); break;
  case 22: tile_digits(width_constant<22>{}); break;
  default: tile_digits(width_constant<0>{}); break;
  }
  if (zero_count)
    atomicAdd(zero_digits, zero_count);
  __syncthreads();
  for (unsigned q = threadIdx.x; q < counters; q += blockDim.x) { // q = w * 256 + digit
    const unsigned w = q / SORT_RADIX, dg = q % SORT_RADIX;
    counts[(size_t)d.tile_base * SORT_RADIX + (size_t)dg * d.tiles + w * d.point_tiles + tile] = s_hist[q];
  }
  for (unsigned q = threadIdx.x; q < later; q += blockDim.x) // q = (pass - 1) * 256 + digit
    if (s_later[q])
      atomicAdd(&later_totals[((size_t)(q / SORT_RADIX) * instances + k) * SORT_RADIX + q % SORT_RADIX], s_later[q]);
  if (threadIdx.x == 0 && *zero_digits)
    atomicAdd(&zeros[k], *zero_digits);
}

// Dynamic shared memory of batch_digits_histogram_kernel for an instance of
// window width c: a counter per (window, digit), per (later pass, digit) and
// the zero-digit count.
static size_t batch_digit_smem(unsigned c, unsigned later_passes) {
  return ((size_t)(windows_for(c) + later_passes) * SORT_RADIX + 1) * 4;
}

// one warp per (segment, digit) row
__global__ void __launch_bounds__(256) batch_sort_scan_kernel(uint32_t *counts, const batch_instance *__restrict__ inst, unsigned rows,
                                                              uint32_t *__restrict__ totals) {
  const unsigned row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= rows)
    return;
  const batch_instance d = inst[row / SORT_RADIX];
  sort_scan_row(counts + (size_t)d.tile_base * SORT_RADIX + (size_t)(row % SORT_RADIX) * d.tiles, d.tiles, totals + row);
}

// The first radix pass (drops zero digits; tile offsets from the scan).
__global__ void __launch_bounds__(SORT_THREADS, SORT_SCATTER_MIN_BLOCKS) batch_sort_scatter_first_kernel(
    const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out,
    const batch_instance *__restrict__ inst, const unsigned *__restrict__ tile_seg, const uint32_t *__restrict__ counts,
    const uint32_t *__restrict__ totals, const uint32_t *__restrict__ zeros) {
  const unsigned t = blockIdx.x;
  const unsigned k = tile_seg[t];
  const batch_instance d = inst[k];
  const unsigned local = t - d.tile_base, base = local * SORT_TILE;
  const unsigned skip = zeros[k];
  const uint32_t *tile_counts = counts + (size_t)d.tile_base * SORT_RADIX + local;
  sort_scatter_tile<false, true>(keys_in, vals_in, keys_out, vals_out, d.entry_offset, d.entry_offset + skip, base,
                                 min(SORT_TILE, d.entries - base), 0, tile_counts, d.tiles, totals + (size_t)k * SORT_RADIX);
}

// A later radix pass in one kernel, positions by decoupled look-back
// (lookback_tile) over the tiles of each instance's segment.  Blocks take
// tickets from *tile_ctr, and ticket q sorts tile tile_order[q]: the
// instances' tiles interleaved (every instance's local tile j before any
// instance's tile j + 1), so the tiles in flight spread over the instances
// and a tile's look-back walks over few aggregates of its own segment; its
// predecessors took their tickets earlier and are resident.  words: 256 per
// global tile (this pass's, zero at launch); totals: the instances' digit
// totals of this pass.  Dynamic shared memory lookback_smem_bytes<SORT_THREADS,
// SORT_ITEMS>().
__global__ void __launch_bounds__(SORT_THREADS, SORT_SCATTER_MIN_BLOCKS) batch_lookback_kernel(
    const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out,
    const batch_instance *__restrict__ inst, const unsigned *__restrict__ tile_seg, const unsigned *__restrict__ tile_order, unsigned shift,
    uint32_t *words, const uint32_t *__restrict__ totals, const uint32_t *__restrict__ zeros, unsigned *tile_ctr, unsigned *error) {
  __shared__ unsigned s_ticket;
  if (threadIdx.x == 0)
    s_ticket = atomicAdd(tile_ctr, 1u);
  __syncthreads();
  const unsigned t = tile_order[s_ticket];
  const unsigned k = tile_seg[t];
  const batch_instance d = inst[k];
  const unsigned local = t - d.tile_base, base = local * SORT_TILE;
  const unsigned skip = zeros[k], live = d.entries - skip;
  if (base >= live) // no later tile of this segment holds entries either, so none waits for this one
    return;
  lookback_tile<SORT_THREADS, SORT_ITEMS>(keys_in, vals_in, keys_out, vals_out, d.entry_offset + skip, local, min(SORT_TILE, live - base), shift,
                                          words + (size_t)d.tile_base * SORT_RADIX, totals + (size_t)k * SORT_RADIX, error);
}

// The batch's segments for accumulate_ranges: one per instance.
struct table_segments {
  static constexpr bool POINT_LIST = false;
  const unsigned long long *s_first, *s_end, *s_prefix;
  const uint32_t *s_bucket, *s_mask;
  const affine *const *s_table;
  unsigned segments;
  __device__ __forceinline__ unsigned count() const { return segments; }
  __device__ __forceinline__ unsigned long long prefix(unsigned s) const { return s_prefix[s]; }
  __device__ __forceinline__ size_t first(unsigned s) const { return s_first[s]; }
  __device__ __forceinline__ size_t end(unsigned s) const { return s_end[s]; }
  __device__ __forceinline__ bool empty(unsigned s) const { return s_first[s] == s_end[s]; }
  __device__ __forceinline__ unsigned bucket(unsigned s, uint32_t key) const { return s_bucket[s] + key_slot(key, s_mask[s]); }
  __device__ __forceinline__ const affine *base(unsigned s, uint32_t val) const { return s_table[s] + (val & 0x7fffffffu); }
};

__global__ void __launch_bounds__(ACC_THREADS, ACC_MIN_BLOCKS) batch_accumulate_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, const batch_instance *__restrict__ inst, unsigned instances,
    const uint32_t *__restrict__ zeros, unsigned ranges, unsigned *__restrict__ work, xyzz *__restrict__ buckets, uint8_t *__restrict__ flags,
    uint32_t *__restrict__ head_bucket, xyzz *__restrict__ head_point) {
  __shared__ unsigned long long s_first[MAX_BATCH], s_end[MAX_BATCH], s_prefix[MAX_BATCH + 1];
  __shared__ uint32_t s_bucket[MAX_BATCH], s_mask[MAX_BATCH];
  __shared__ const affine *s_table[MAX_BATCH];
  __shared__ uint4 s_base[2][4][ACC_THREADS];
  for (unsigned k = threadIdx.x; k < instances; k += blockDim.x) {
    const batch_instance d = inst[k];
    s_first[k] = d.entry_offset + zeros[k];
    s_end[k] = d.entry_offset + d.entries;
    s_bucket[k] = d.bucket_base;
    s_mask[k] = (1u << (d.c - 1)) - 1;
    s_table[k] = d.table;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long acc = 0;
    for (unsigned k = 0; k < instances; k++) {
      s_prefix[k] = acc;
      acc += s_end[k] - s_first[k];
    }
    s_prefix[instances] = acc;
  }
  __syncthreads();
  const table_segments seg{s_first, s_end, s_prefix, s_bucket, s_mask, s_table, instances};
  accumulate_ranges(seg, keys, vals, ranges, work, buckets, flags, head_bucket, head_point, s_base);
}

// Results of the instances of one reduction group (all of window width c):
// instance members[w] is window w of the group's reduction.  Bit i < c comes
// from the group's streams exactly as gather_results_kernel places window 0
// of a plain MSM; bits >= c are infinity.
__global__ void batch_gather_kernel(const xyzz *__restrict__ streams, const xyzz *__restrict__ buckets, const uint8_t *__restrict__ flags,
                                    const unsigned *__restrict__ members, unsigned windows, unsigned c, unsigned log_m, unsigned log_g,
                                    const batch_io *__restrict__ io) {
  const unsigned gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= windows * RESULT_BITS)
    return;
  const unsigned w = gid / RESULT_BITS, i = gid % RESULT_BITS;
  xyzz p = curve::infinity();
  if (i < c) {
    const size_t base = (size_t)w * stream_stride(log_g);
    if (i == 0) {
      p = load_xyzz(streams + base);
    } else if (i == c - 1) {
      const size_t slot0 = (size_t)w << (c - 1);
      if (flags[slot0])
        p = load_xyzz(buckets + slot0);
    } else if (i >= log_m && i - log_m < log_g) {
      p = load_xyzz(streams + base + stream_offset(log_g, i - log_m + 1));
    }
  }
  store_jacobian(io[members[w]].results + i, curve::to_jacobian(p));
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// Builds M_c for the first `prefix` points of `bases` (device memory).
static cudaError_t build_multiples(base_table_impl &t, unsigned c, unsigned prefix, const affine *bases, cudaStream_t stream) {
  const unsigned W = windows_for(c);
  affine *m = nullptr;
  const size_t bytes = (size_t)W * prefix * sizeof(affine);
  CHECK(cudaMalloc(&m, bytes));
  t.mult[c] = m;
  t.prefix[c] = prefix;
  t.bytes += bytes;
  CHECK(cudaMemcpyAsync(m, bases, (size_t)prefix * sizeof(affine), cudaMemcpyDeviceToDevice, stream));
  for (unsigned j = 1; j < W; j++) {
    window_multiples_kernel<<<(prefix + 127) / 128, 128, 0, stream>>>(m + (size_t)(j - 1) * prefix, m + (size_t)j * prefix, prefix, c);
    CHECK(cudaGetLastError());
  }
  return cudaSuccess;
}

cudaError_t base_table_create(base_table_impl **out, const void *bases, unsigned count, const unsigned *window_bits, unsigned widths,
                              cudaStream_t stream) {
  if (!out || !bases || count == 0 || (reinterpret_cast<uintptr_t>(bases) & 15))
    return cudaErrorInvalidValue;
  // window widths and, per width, the longest prefix an instance of that width can use
  std::map<unsigned, unsigned> want;
  if (widths) {
    for (unsigned k = 0; k < widths; k++) {
      if (window_bits[k] < 2 || window_bits[k] > MAX_TABLE_BITS)
        return cudaErrorInvalidValue;
      want[window_bits[k]] = count;
    }
  } else {
    for (unsigned lg = 0; (1ull << lg) < 2ull * count && lg <= 31; lg++) {
      const unsigned n = (unsigned)std::min<unsigned long long>(count, 1ull << lg);
      unsigned &p = want[batch_window_bits(n)];
      p = std::max(p, n);
    }
  }
  base_table_impl *t = new (std::nothrow) base_table_impl;
  if (!t)
    return cudaErrorMemoryAllocation;
  cudaError_t status = cudaGetDevice(&t->device);
  t->count = count;
  affine *staged = nullptr;
  cudaPointerAttributes attr{};
  if (status == cudaSuccess)
    status = cudaPointerGetAttributes(&attr, bases);
  const bool host = attr.type == cudaMemoryTypeUnregistered || attr.type == cudaMemoryTypeHost;
  const affine *src = static_cast<const affine *>(bases);
  if (status == cudaSuccess && host) {
    status = cudaMalloc(&staged, (size_t)count * sizeof(affine));
    if (status == cudaSuccess)
      status = cudaMemcpyAsync(staged, bases, (size_t)count * sizeof(affine), cudaMemcpyHostToDevice, stream);
    src = staged;
  }
  for (auto it = want.begin(); status == cudaSuccess && it != want.end(); ++it)
    status = build_multiples(*t, it->first, it->second, src, stream);
  if (status == cudaSuccess)
    status = cudaStreamSynchronize(stream);
  if (staged)
    cudaFree(staged);
  if (status != cudaSuccess) {
    delete t;
    return status;
  }
  *out = t;
  return cudaSuccess;
}

// Serialised table: a little-endian header (magic, version, point count,
// number of widths, then per width: c, prefix, windows) followed, width by
// width in increasing c, by the W(c) x prefix affine points (Montgomery form,
// 64 B each) of M_c.  Importing it skips the precomputation.
constexpr uint32_t TABLE_MAGIC0 = 0x34354e42; // "BN54"
constexpr uint32_t TABLE_MAGIC1 = 0x4c424154; // "TABL"
constexpr uint32_t TABLE_VERSION = 1;

static size_t table_header_bytes(unsigned widths) { return (size_t)(5 + 3 * widths) * sizeof(uint32_t); }

size_t base_table_serialized_bytes(const base_table_impl &t) {
  unsigned widths = 0;
  size_t bytes = 0;
  for (unsigned c = 2; c <= MAX_TABLE_BITS; c++)
    if (t.mult[c]) {
      widths++;
      bytes += (size_t)windows_for(c) * t.prefix[c] * sizeof(affine);
    }
  return table_header_bytes(widths) + bytes;
}

cudaError_t base_table_export(const base_table_impl &t, void *out, size_t bytes) {
  if (!out || bytes < base_table_serialized_bytes(t))
    return cudaErrorInvalidValue;
  std::vector<uint32_t> header = {TABLE_MAGIC0, TABLE_MAGIC1, TABLE_VERSION, t.count};
  std::vector<unsigned> widths;
  for (unsigned c = 2; c <= MAX_TABLE_BITS; c++)
    if (t.mult[c])
      widths.push_back(c);
  header.push_back((uint32_t)widths.size());
  for (unsigned c : widths) {
    header.push_back(c);
    header.push_back(t.prefix[c]);
    header.push_back(windows_for(c));
  }
  uint8_t *dst = static_cast<uint8_t *>(out);
  // the header: magic (2 words), version, count, widths, then the per-width triples
  std::memcpy(dst, header.data(), header.size() * sizeof(uint32_t));
  dst += header.size() * sizeof(uint32_t);
  for (unsigned c : widths) {
    const size_t n = (size_t)windows_for(c) * t.prefix[c] * sizeof(affine);
    CHECK(cudaMemcpy(dst, t.mult[c], n, cudaMemcpyDeviceToHost));
    dst += n;
  }
  return cudaSuccess;
}

cudaError_t base_table_import(base_table_impl **out, const void *image, size_t bytes, cudaStream_t stream) {
  if (!out || !image || bytes < 5 * sizeof(uint32_t))
    return cudaErrorInvalidValue;
  const uint32_t *h = static_cast<const uint32_t *>(image);
  if (h[0] != TABLE_MAGIC0 || h[1] != TABLE_MAGIC1 || h[2] != TABLE_VERSION || h[3] == 0)
    return cudaErrorInvalidValue;
  const unsigned count = h[3], widths = h[4];
  if (widths == 0 || widths > MAX_TABLE_BITS || bytes < table_header_bytes(widths))
    return cudaErrorInvalidValue;
  const uint32_t *w = h + 5; // per-width triples
  size_t need = table_header_bytes(widths);
  unsigned last_c = 1;
  for (unsigned k = 0; k < widths; k++) {
    const unsigned c = w[3 * k], prefix = w[3 * k + 1], windows = w[3 * k + 2];
    if (c <= last_c || c > MAX_TABLE_BITS || prefix == 0 || prefix > count || windows != windows_for(c))
      return cudaErrorInvalidValue;
    last_c = c;
    need += (size_t)windows * prefix * sizeof(affine);
  }
  if (bytes < need)
    return cudaErrorInvalidValue;
  std::unique_ptr<base_table_impl> t(new (std::nothrow) base_table_impl);
  if (!t)
    return cudaErrorMemoryAllocation;
  CHECK(cudaGetDevice(&t->device));
  t->count = count;
  const uint8_t *src = reinterpret_cast<const uint8_t *>(w + 3 * widths);
  for (unsigned k = 0; k < widths; k++) {
    const unsigned c = w[3 * k], prefix = w[3 * k + 1];
    const size_t n = (size_t)windows_for(c) * prefix * sizeof(affine);
    affine *m = nullptr;
    CHECK(cudaMalloc(&m, n));
    t->mult[c] = m;
    t->prefix[c] = prefix;
    t->bytes += n;
    CHECK(cudaMemcpyAsync(m, src, n, cudaMemcpyHostToDevice, stream));
    src += n;
  }
  CHECK(cudaStreamSynchronize(stream));
  *out = t.release();
  return cudaSuccess;
}

cudaError_t make_batch_plan(batch_plan &b, const base_table_impl *table, const unsigned *counts, unsigned instances, const unsigned *window_bits,
                            int sms) {
  if (!table || !counts || instances == 0 || instances > MAX_BATCH)
    return cudaErrorInvalidValue;
  b = batch_plan{};
  b.instances = instances;
  b.sms = (unsigned)sms;
  b.inst.resize(instances);
  // instance geometry; reduction groups by window width (buckets of a group contiguous)
  std::map<unsigned, std::vector<unsigned>> by_c;
  unsigned max_c = 0;
  unsigned long long points = 0;
  for (unsigned k = 0; k < instances; k++) {
    const unsigned n = counts[k];
    const unsigned c = window_bits && window_bits[k] ? window_bits[k] : batch_window_bits(n);
    if (n == 0 || c < 2 || c > MAX_TABLE_BITS || !table->mult[c] || n > table->prefix[c])
      return cudaErrorInvalidValue;
    batch_instance &d = b.inst[k];
    d.n = n;
    d.c = c;
    d.windows = windows_for(c);
    d.stride = table->prefix[c];
    d.table = table->mult[c];
    const unsigned long long seg_stride = ((unsigned long long)n + SORT_TILE - 1) / SORT_TILE * SORT_TILE;
    if (d.windows * seg_stride >= (1ull << 31) || d.windows * (unsigned long long)d.stride >= (1ull << 31))
      return cudaErrorInvalidValue;
    // every window of the segment is a whole number of sort tiles, so the
    // digit kernel's point tiles count exactly the first pass's sort tiles
    d.seg_stride = (unsigned)seg_stride;
    d.point_tiles = d.seg_stride / SORT_TILE;
    d.entries = d.windows * d.seg_stride;
    d.entry_offset = b.total_entries;
    d.tiles = d.windows * d.point_tiles;
    d.tile_base = b.total_tiles;
    d.ptile_base = b.total_point_tiles;
    b.total_entries += d.entries;
    b.total_tiles += d.tiles;
    b.total_point_tiles += d.point_tiles;
    points += n;
    max_c = std::max(max_c, c);
    by_c[c].push_back(k);
  }
  if (points >= (1ull << 32) || b.total_tiles >= (1u << 31))
    return cudaErrorInvalidValue;
  b.total_points = (unsigned)points;
  b.sort_passes = (max_c - 1 + SORT_RADIX_BITS - 1) / SORT_RADIX_BITS; // keys take c - 1 bits
  for (const batch_instance &d : b.inst)
    b.digit_smem = std::max(b.digit_smem, batch_digit_smem(d.c, b.sort_passes - 1));
  for (auto &kv : by_c) {
    batch_group g;
    g.c = kv.first;
    g.members = kv.second;
    g.bucket_base = b.slots;
    g.p = make_plan(1, g.c, sms);
    // Groups of 8 slots at every width: the batch's reductions run on forked
    // streams beside each other, and the config-3 batch took the same time
    // with the plain path's per-width groups (70.77 against 70.90 ms) but
    // 1.0 GiB more scratch (their trees and streams are larger).
    set_reduction_groups(g.p, 3);
    g.p.windows = (unsigned)g.members.size();
    for (unsigned w = 0; w < g.members.size(); w++)
      b.inst[g.members[w]].bucket_base = b.slots + (w << (g.c - 1));
    b.slots += (unsigned)g.members.size() << (g.c - 1);
    b.groups.push_back(g);
  }
  const unsigned long long full = (unsigned long long)sms * ACC_MIN_BLOCKS * ACC_THREADS;
  b.acc_threads = (unsigned)std::max(1ull, std::min(full, (b.total_entries + 7) / 8));
  b.acc_ranges = accumulation_ranges(b.acc_threads, b.total_entries, BATCH_ACC_RANGES_PER_THREAD);
  // scratch layout
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += align256(bytes);
    return at;
  };
  for (int i = 0; i < 2; i++) {
    b.keys[i] = take(b.total_entries * 4);
    b.vals[i] = take(b.total_entries * 4);
  }
  // the first pass's tile counts, then (cleared after that pass) the first
  // later pass's look-back words, 256 per tile; the second later pass's
  // look-back words (cleared before that pass)
  static_assert((MAX_TABLE_BITS - 1 + SORT_RADIX_BITS - 1) / SORT_RADIX_BITS <= 3, "two look-back word arrays: at most three radix passes");
  b.counts = take((size_t)b.total_tiles * SORT_RADIX * 4);
  b.words2 = b.sort_passes > 2 ? take((size_t)b.total_tiles * SORT_RADIX * 4) : 0;
  b.totals = take((size_t)instances * SORT_RADIX * 4);
  // cleared every execution: zero digits per instance, the later passes'
  // digit totals per instance, a tile ticket counter per later pass and the
  // look-back error word
  const unsigned later = b.sort_passes - 1;
  b.zeros = take(((size_t)instances + (size_t)later * instances * SORT_RADIX + later + 1) * 4);
  b.later_totals = b.zeros + (size_t)instances * 4;
  b.sort_ctrs = b.later_totals + (size_t)later * instances * SORT_RADIX * 4;
  b.sort_error = b.sort_ctrs + (size_t)later * 4;
  b.sort_clear_bytes = b.sort_error + 4 - b.zeros;
  b.buckets = take((size_t)b.slots * sizeof(xyzz));
  b.flags = take(b.slots);
  for (int i = 0; i < 2; i++) {
    b.hb[i] = take((size_t)b.acc_ranges * 4);
    b.hp[i] = take((size_t)b.acc_ranges * sizeof(xyzz));
  }
  b.work = take(sizeof(unsigned));
  for (batch_group &g : b.groups)
    for (int i = 0; i < 2; i++) {
      g.tree[i] = take(((size_t)g.p.windows << g.p.log_g) * sizeof(xyzz));
      g.streams[i] = take((size_t)g.p.windows * stream_stride(g.p.log_g) * sizeof(xyzz));
    }
  b.io = take(instances * sizeof(batch_io));
  // constant descriptors last, in one contiguous range (one upload)
  b.descriptors = off;
  b.inst_dev = take(instances * sizeof(batch_instance));
  b.tile_seg_dev = take((size_t)b.total_tiles * 4);
  b.tile_order_dev = take((size_t)b.total_tiles * 4);
  b.ptile_seg_dev = take((size_t)b.total_point_tiles * 4);
  for (batch_group &g : b.groups)
    g.members_dev = take(g.members.size() * 4);
  b.bytes = off;
  return cudaSuccess;
}

// The constant descriptors as they lie in scratch from b.descriptors on.
std::vector<uint8_t> descriptor_image(const batch_plan &b) {
  std::vector<uint8_t> img(b.bytes - b.descriptors, 0);
  auto put = [&](size_t off, const void *src, size_t bytes) { std::memcpy(img.data() + (off - b.descriptors), src, bytes); };
  put(b.inst_dev, b.inst.data(), b.instances * sizeof(batch_instance));
  unsigned *tile_seg = reinterpret_cast<unsigned *>(img.data() + (b.tile_seg_dev - b.descriptors));
  unsigned *ptile_seg = reinterpret_cast<unsigned *>(img.data() + (b.ptile_seg_dev - b.descriptors));
  unsigned most = 0;
  for (unsigned k = 0; k < b.instances; k++) {
    std::fill(tile_seg + b.inst[k].tile_base, tile_seg + b.inst[k].tile_base + b.inst[k].tiles, k);
    std::fill(ptile_seg + b.inst[k].ptile_base, ptile_seg + b.inst[k].ptile_base + b.inst[k].point_tiles, k);
    most = std::max(most, b.inst[k].tiles);
  }
  // the look-back passes' ticket order: local tile j of every instance before local tile j + 1 of any
  unsigned *tile_order = reinterpret_cast<unsigned *>(img.data() + (b.tile_order_dev - b.descriptors));
  unsigned q = 0;
  for (unsigned j = 0; j < most; j++)
    for (unsigned k = 0; k < b.instances; k++)
      if (j < b.inst[k].tiles)
        tile_order[q++] = b.inst[k].tile_base + j;
  for (const batch_group &g : b.groups)
    put(g.members_dev, g.members.data(), g.members.size() * 4);
  return img;
}

// Enqueues the chain of plan b over `scratch` on stream s.  With forks (one
// stream and one event per reduction group, plus one event), the per-width
// reductions run concurrently; otherwise one after another on s.
cudaError_t enqueue_batch(const batch_plan &b, uint8_t *scratch, cudaStream_t s, const cudaStream_t *forks, const cudaEvent_t *fork_events,
                                 unsigned *launches) {
  auto at = [&](size_t off) { return scratch + off; };
  unsigned launched = 0;
  uint32_t *keys[2] = {reinterpret_cast<uint32_t *>(at(b.keys[0])), reinterpret_cast<uint32_t *>(at(b.keys[1]))};
  uint32_t *vals[2] = {reinterpret_cast<uint32_t *>(at(b.vals[0])), reinterpret_cast<uint32_t *>(at(b.vals[1]))};
  const batch_instance *inst = reinterpret_cast<const batch_instance *>(at(b.inst_dev));
  const batch_io *io = reinterpret_cast<const batch_io *>(at(b.io));
  uint32_t *counts = reinterpret_cast<uint32_t *>(at(b.counts)), *totals = reinterpret_cast<uint32_t *>(at(b.totals)),
           *zeros = reinterpret_cast<uint32_t *>(at(b.zeros));
  const unsigned *tile_seg = reinterpret_cast<const unsigned *>(at(b.tile_seg_dev));
  xyzz *buckets = reinterpret_cast<xyzz *>(at(b.buckets));
  uint8_t *flags = at(b.flags);
  uint32_t *hb[2] = {reinterpret_cast<uint32_t *>(at(b.hb[0])), reinterpret_cast<uint32_t *>(at(b.hb[1]))};
  xyzz *hp[2] = {reinterpret_cast<xyzz *>(at(b.hp[0])), reinterpret_cast<xyzz *>(at(b.hp[1]))};

  CHECK(cudaMemsetAsync(flags, 0, b.slots, s));
  CHECK(cudaMemsetAsync(zeros, 0, b.sort_clear_bytes, s));
  const unsigned later = b.sort_passes - 1;
  uint32_t *later_totals = reinterpret_cast<uint32_t *>(at(b.later_totals));
  // digits, with the first pass's counts per sort tile and the later passes' digit totals
  batch_digits_histogram_kernel<<<b.total_point_tiles, SORT_THREADS, b.digit_smem, s>>>(
      inst, reinterpret_cast<const unsigned *>(at(b.ptile_seg_dev)), io, keys[0], vals[0], counts, zeros, b.instances, later, later_totals);
  CHECK(cudaGetLastError());
  launched++;
  // the first pass: tile offsets and digit totals by one scan, then the scatter (drops zero digits)
  const unsigned rows = b.instances * SORT_RADIX;
  batch_sort_scan_kernel<<<(rows * 32 + 255) / 256, 256, 0, s>>>(counts, inst, rows, totals);
  CHECK(cudaGetLastError());
  batch_sort_scatter_first_kernel<<<b.total_tiles, SORT_THREADS, 0, s>>>(keys[0], vals[0], keys[1], vals[1], inst, tile_seg, counts, totals, zeros);
  CHECK(cudaGetLastError());
  launched += 2;
  int cur = 1;
  // later passes: one look-back kernel each, on words cleared before it
  const unsigned *tile_order = reinterpret_cast<const unsigned *>(at(b.tile_order_dev));
  unsigned *sort_ctrs = reinterpret_cast<unsigned *>(at(b.sort_ctrs)), *sort_error = reinterpret_cast<unsigned *>(at(b.sort_error));
  const size_t word_bytes = (size_t)b.total_tiles * SORT_RADIX * 4;
  for (unsigned pass = 1; pass < b.sort_passes; pass++) {
    uint32_t *words = pass == 1 ? counts : reinterpret_cast<uint32_t *>(at(b.words2));
    CHECK(cudaMemsetAsync(words, 0, word_bytes, s));
    batch_lookback_kernel<<<b.total_tiles, SORT_THREADS, lookback_smem_bytes<SORT_THREADS, SORT_ITEMS>(), s>>>(
        keys[cur], vals[cur], keys[cur ^ 1], vals[cur ^ 1], inst, tile_seg, tile_order, pass * SORT_RADIX_BITS, words,
        later_totals + (size_t)(pass - 1) * b.instances * SORT_RADIX, zeros, sort_ctrs + pass - 1, sort_error);
    CHECK(cudaGetLastError());
    launched++;
    cur ^= 1;
  }
  unsigned *work = reinterpret_cast<unsigned *>(at(b.work));
  CHECK(cudaMemsetAsync(work, 0, sizeof(unsigned), s));
  batch_accumulate_kernel<<<(b.acc_threads + ACC_THREADS - 1) / ACC_THREADS, ACC_THREADS, 0, s>>>(
      keys[cur], vals[cur], inst, b.instances, zeros, b.acc_ranges, work, buckets, flags, hb[0], hp[0]);
  CHECK(cudaGetLastError());
  launched++;
  CHECK(enqueue_merge_heads(hb, hp, b.acc_ranges, buckets, b.sms, s, launched));
  if (forks)
    CHECK(cudaEventRecord(fork_events[0], s));
  for (size_t g = 0; g < b.groups.size(); g++) {
    const batch_group &grp = b.groups[g];
    const plan &p = grp.p;
    cudaStream_t fs = forks ? forks[g] : s;
    if (forks)
      CHECK(cudaStreamWaitEvent(fs, fork_events[0], 0));
    xyzz *gb = buckets + grp.bucket_base;
    const uint8_t *gf = flags + grp.bucket_base;
    xyzz *const tree[2] = {reinterpret_cast<xyzz *>(at(grp.tree[0])), reinterpret_cast<xyzz *>(at(grp.tree[1]))};
    xyzz *const streams[2] = {reinterpret_cast<xyzz *>(at(grp.streams[0])), reinterpret_cast<xyzz *>(at(grp.streams[1]))};
    CHECK(enqueue_window_sums(p, gb, gf, tree, streams, fs, launched));
    const int si = p.log_g & 1;
    const unsigned gather_threads = p.windows * RESULT_BITS;
    batch_gather_kernel<<<(gather_threads + 127) / 128, 128, 0, fs>>>(streams[si], gb, gf, reinterpret_cast<const unsigned *>(at(grp.members_dev)),
                                                                      p.windows, p.c, p.log_m, p.log_g, io);
    CHECK(cudaGetLastError());
    launched++;
    if (forks) {
      CHECK(cudaEventRecord(fork_events[g + 1], fs));
      CHECK(cudaStreamWaitEvent(s, fork_events[g + 1], 0));
    }
  }
  if (launches)
    *launches = launched;
  return cudaSuccess;
}

// Writes the instances' scalar and result pointers into the batch's io table.
cudaError_t enqueue_io(batch_io *io, unsigned instances, const void *const *scalars, void *const *results, cudaStream_t stream) {
  for (unsigned first = 0; first < instances; first += IO_CHUNK) {
    batch_io_update u{};
    u.first = first;
    u.count = std::min(IO_CHUNK, instances - first);
    for (unsigned k = 0; k < u.count; k++) {
      u.io[k].scalars = static_cast<const fe *>(scalars[first + k]);
      u.io[k].results = static_cast<jacobian *>(results[first + k]);
    }
    batch_set_io_kernel<<<1, IO_CHUNK, 0, stream>>>(io, u);
    CHECK(cudaGetLastError());
  }
  return cudaSuccess;
}

// A planned batch with its own scratch and captured graph.
struct batch_impl {
  int device = 0;
  batch_plan b;
  uint8_t *scratch = nullptr;
  cudaStream_t capture = nullptr;
  std::vector<cudaStream_t> forks;
  std::vector<cudaEvent_t> fork_events;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned launches = 0;
  ~batch_impl() {
    if (exec)
      cudaGraphExecDestroy(exec);
    if (graph)
      cudaGraphDestroy(graph);
    for (cudaEvent_t e : fork_events)
      cudaEventDestroy(e);
    for (cudaStream_t s : forks)
      cudaStreamDestroy(s);
    if (capture)
      cudaStreamDestroy(capture);
    if (scratch)
      cudaFree(scratch);
  }
};

static cudaError_t device_sms(int device, int *sms) { return cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, device); }

cudaError_t batch_create(batch_impl **out, const base_table_impl *table, const unsigned *counts, unsigned instances, const unsigned *window_bits) {
  if (!out || !table)
    return cudaErrorInvalidValue;
  int device = 0, sms = 0;
  CHECK(cudaGetDevice(&device));
  if (device != table->device)
    return cudaErrorInvalidDevice;
  CHECK(device_sms(device, &sms));
  std::unique_ptr<batch_impl> owner(new (std::nothrow) batch_impl);
  if (!owner)
    return cudaErrorMemoryAllocation;
  batch_impl &bi = *owner;
  bi.device = device;
  CHECK(make_batch_plan(bi.b, table, counts, instances, window_bits, sms));
  const batch_plan &b = bi.b;
  CHECK(cudaMalloc(&bi.scratch, b.bytes));
  const std::vector<uint8_t> img = descriptor_image(b);
  CHECK(cudaMemcpy(bi.scratch + b.descriptors, img.data(), img.size(), cudaMemcpyHostToDevice));
  CHECK(cudaMemset(bi.scratch + b.io, 0, instances * sizeof(batch_io)));
  // capture the chain
  CHECK(cudaStreamCreateWithFlags(&bi.capture, cudaStreamNonBlocking));
  bi.forks.resize(b.groups.size());
  bi.fork_events.resize(b.groups.size() + 1);
  for (auto &fs : bi.forks)
    CHECK(cudaStreamCreateWithFlags(&fs, cudaStreamNonBlocking));
  for (auto &e : bi.fork_events)
    CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CHECK(cudaStreamBeginCapture(bi.capture, cudaStreamCaptureModeThreadLocal));
  const cudaError_t enq = enqueue_batch(b, bi.scratch, bi.capture, bi.forks.data(), bi.fork_events.data(), &bi.launches);
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(bi.capture, &graph);
  bi.graph = graph;
  CHECK(enq);
  CHECK(end);
  CHECK(cudaGraphInstantiate(&bi.exec, bi.graph, 0));
  *out = owner.release();
  return cudaSuccess;
}

static cudaError_t check_io(unsigned instances, const void *const *scalars, void *const *results) {
  if (!scalars || !results)
    return cudaErrorInvalidValue;
  for (unsigned k = 0; k < instances; k++)
    if (!scalars[k] || !results[k] || (reinterpret_cast<uintptr_t>(scalars[k]) & 15) || (reinterpret_cast<uintptr_t>(results[k]) & 15))
      return cudaErrorInvalidValue;
  return cudaSuccess;
}

cudaError_t batch_execute(batch_impl *bi, const void *const *scalars, void *const *results, cudaStream_t stream) {
  if (!bi)
    return cudaErrorInvalidValue;
  int device = 0;
  CHECK(cudaGetDevice(&device));
  if (device != bi->device)
    return cudaErrorInvalidDevice;
  CHECK(check_io(bi->b.instances, scalars, results));
  CHECK(enqueue_io(reinterpret_cast<batch_io *>(bi->scratch + bi->b.io), bi->b.instances, scalars, results, stream));
  return cudaGraphLaunch(bi->exec, stream);
}

cudaError_t batch_set_up() {
  CHECK(cudaFuncSetAttribute(batch_accumulate_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 50));
  size_t digit_smem = 0; // the widest instance any batch can hold, with the most later passes
  const unsigned most_later = (MAX_TABLE_BITS - 1 + SORT_RADIX_BITS - 1) / SORT_RADIX_BITS - 1;
  for (unsigned c = 2; c <= MAX_TABLE_BITS; c++)
    digit_smem = std::max(digit_smem, batch_digit_smem(c, most_later));
  CHECK(cudaFuncSetAttribute(batch_digits_histogram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)digit_smem));
  return cudaSuccess;
}

} // namespace msm_b200

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

bc_error msm_b200_base_table_create(msm_b200_base_table *table, const void *bases, unsigned count, const unsigned *window_bits, unsigned widths,
                                    bc_stream stream) {
  if (!table)
    return bc_error_invalid_value;
  msm_b200::base_table_impl *t = nullptr;
  const cudaError_t e = msm_b200::base_table_create(&t, bases, count, window_bits, widths, static_cast<cudaStream_t>(stream.handle));
  *table = reinterpret_cast<msm_b200_base_table>(t);
  return static_cast<bc_error>(e);
}

bc_error msm_b200_base_table_bytes(msm_b200_base_table table, size_t *bytes) {
  if (!table || !bytes)
    return bc_error_invalid_value;
  *bytes = reinterpret_cast<msm_b200::base_table_impl *>(table)->bytes;
  return bc_success;
}

bc_error msm_b200_base_table_serialized_bytes(msm_b200_base_table table, size_t *bytes) {
  if (!table || !bytes)
    return bc_error_invalid_value;
  *bytes = msm_b200::base_table_serialized_bytes(*reinterpret_cast<msm_b200::base_table_impl *>(table));
  return bc_success;
}

bc_error msm_b200_base_table_export(msm_b200_base_table table, void *image, size_t bytes) {
  if (!table)
    return bc_error_invalid_value;
  return static_cast<bc_error>(msm_b200::base_table_export(*reinterpret_cast<msm_b200::base_table_impl *>(table), image, bytes));
}

bc_error msm_b200_base_table_import(msm_b200_base_table *table, const void *image, size_t bytes, bc_stream stream) {
  if (!table)
    return bc_error_invalid_value;
  msm_b200::base_table_impl *t = nullptr;
  const cudaError_t e = msm_b200::base_table_import(&t, image, bytes, static_cast<cudaStream_t>(stream.handle));
  *table = reinterpret_cast<msm_b200_base_table>(t);
  return static_cast<bc_error>(e);
}

bc_error msm_b200_base_table_destroy(msm_b200_base_table table) {
  delete reinterpret_cast<msm_b200::base_table_impl *>(table);
  return bc_success;
}

bc_error msm_b200_batch_window_bits(unsigned count, unsigned *window_bits) {
  if (!window_bits || count == 0)
    return bc_error_invalid_value;
  *window_bits = msm_b200::batch_window_bits(count);
  return bc_success;
}

bc_error msm_b200_batch_create(msm_b200_batch *batch, msm_b200_base_table table, const unsigned *counts, unsigned instances,
                               const unsigned *window_bits) {
  if (!batch)
    return bc_error_invalid_value;
  msm_b200::batch_impl *b = nullptr;
  cudaError_t e = msm_b200::batch_set_up();
  if (e == cudaSuccess)
    e = msm_b200::batch_create(&b, reinterpret_cast<const msm_b200::base_table_impl *>(table), counts, instances, window_bits);
  *batch = reinterpret_cast<msm_b200_batch>(b);
  return static_cast<bc_error>(e);
}

bc_error msm_b200_batch_execute_async(msm_b200_batch batch, const void *const *scalars, void *const *results, bc_stream stream) {
  return static_cast<bc_error>(
      msm_b200::batch_execute(reinterpret_cast<msm_b200::batch_impl *>(batch), scalars, results, static_cast<cudaStream_t>(stream.handle)));
}

bc_error msm_b200_batch_info(msm_b200_batch batch, size_t *scratch_bytes, unsigned *kernels, unsigned long long *entries) {
  if (!batch)
    return bc_error_invalid_value;
  const msm_b200::batch_impl *b = reinterpret_cast<const msm_b200::batch_impl *>(batch);
  if (scratch_bytes)
    *scratch_bytes = b->b.bytes;
  if (kernels)
    *kernels = b->launches;
  if (entries)
    *entries = b->b.total_entries;
  return bc_success;
}

bc_error msm_b200_batch_destroy(msm_b200_batch batch) {
  delete reinterpret_cast<msm_b200::batch_impl *>(batch);
  return bc_success;
}

} // extern "C"
