// Internal interface of the batched MSM (msm_batch.cu), shared with the
// request server (msm_server.cu).
#pragma once

#include "bellman-cuda-b200.h"
#include "msm_host.cuh"
#include "msm_kernels.cuh"

#include <vector>

namespace msm_b200 {

constexpr unsigned MAX_BATCH = MSM_B200_MAX_BATCH;
constexpr unsigned MAX_TABLE_BITS = 24;

// Per-instance descriptor read by the batch kernels.
struct batch_instance {
  unsigned long long entry_offset; // first entry of the instance's segment
  const affine *table;             // M_c: table[j * stride + i] = 2^(c j) P_i
  unsigned n, c, windows, stride;
  unsigned seg_stride;  // entries per window in the segment: n rounded up to whole sort tiles (the padding holds zero digits)
  unsigned entries;     // windows * seg_stride
  unsigned tiles;       // sort tiles of the segment (windows * point_tiles)
  unsigned tile_base;   // first global sort tile of the segment
  unsigned point_tiles; // sort tiles per window: seg_stride / SORT_TILE
  unsigned ptile_base;  // first global point tile (digit-kernel block) of the instance
  unsigned bucket_base; // first bucket slot (slot 0 holds |d| = 2^(c-1))
};

// Per-execution pointers of one instance.
struct batch_io {
  const fe *scalars; // n Montgomery-form scalars (device)
  jacobian *results; // 254 Jacobian points (device)
};

// A resident base table with its precomputed window multiples.
struct base_table_impl {
  int device = 0;
  unsigned count = 0;
  affine *mult[MAX_TABLE_BITS + 1] = {}; // mult[c]: windows_for(c) * prefix[c] points, or null
  unsigned prefix[MAX_TABLE_BITS + 1] = {};
  size_t bytes = 0;
  ~base_table_impl() {
    for (affine *m : mult)
      if (m)
        cudaFree(m);
  }
};

struct batch_group {
  unsigned c;
  std::vector<unsigned> members; // instances, in bucket order
  plan p;                        // reduction geometry (windows = members)
  unsigned bucket_base;
  size_t tree[2], streams[2], members_dev;
};

// Geometry, scratch layout (offsets from the scratch base) and constant
// descriptors of one batch of instance lengths.  Allocates nothing.
struct batch_plan {
  unsigned instances = 0;
  unsigned long long total_entries = 0;
  unsigned total_points = 0, total_tiles = 0, total_point_tiles = 0, slots = 0, sort_passes = 0, acc_threads = 0, acc_ranges = 0;
  unsigned sms = 0; // SMs of the device the plan is for
  std::vector<batch_instance> inst;
  std::vector<batch_group> groups;
  size_t keys[2], vals[2], counts, totals, zeros, buckets, flags, hb[2], hp[2], work, inst_dev, tile_seg_dev, ptile_seg_dev, io;
  // the look-back passes (all offsets; the zeros .. sort_error range is cleared every execution)
  size_t words2 = 0, later_totals = 0, sort_ctrs = 0, sort_error = 0, sort_clear_bytes = 0, tile_order_dev = 0;
  size_t digit_smem = 0; // dynamic shared memory of the digit kernel (its widest instance)
  size_t bytes = 0;       // scratch bytes
  size_t descriptors = 0; // offset of the constant descriptors (inst_dev .. end of members)
};

unsigned batch_window_bits(unsigned n);
cudaError_t make_batch_plan(batch_plan &b, const base_table_impl *table, const unsigned *counts, unsigned instances, const unsigned *window_bits,
                            int sms);
// the constant descriptors as they lie in scratch from b.descriptors on
std::vector<uint8_t> descriptor_image(const batch_plan &b);
// the chain of plan b over `scratch`; forks (optional): one stream per
// reduction group and groups + 1 events, for concurrent reductions
cudaError_t enqueue_batch(const batch_plan &b, uint8_t *scratch, cudaStream_t s, const cudaStream_t *forks, const cudaEvent_t *fork_events,
                          unsigned *launches);
// writes the instances' scalar and result pointers into the io table
cudaError_t enqueue_io(batch_io *io, unsigned instances, const void *const *scalars, void *const *results, cudaStream_t stream);
cudaError_t batch_set_up();

} // namespace msm_b200
