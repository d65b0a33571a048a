// First-fit allocator over one fixed range of device memory (offsets only; it
// never touches the memory).  Used by the MSM server to admit requests by
// their scratch footprint against a fixed budget.  Plain C++ so that its
// bookkeeping is tested on the host (tests/native/arena_check.cpp).
#pragma once

#include <cstddef>
#include <iterator>
#include <map>

namespace msm_b200 {

class device_arena {
public:
  static constexpr size_t ALIGN = 256;

  explicit device_arena(size_t bytes = 0) { reset(bytes); }

  void reset(size_t bytes) {
    free_.clear();
    size_ = bytes & ~(ALIGN - 1);
    used_ = 0;
    if (size_)
      free_[0] = size_;
  }

  static size_t round_up(size_t bytes) { return (bytes + ALIGN - 1) & ~(ALIGN - 1); }

  // Offset of a block of at least `bytes`, or false when no free block is large enough.
  bool allocate(size_t bytes, size_t &offset) {
    const size_t need = round_up(bytes ? bytes : 1);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < need)
        continue;
      offset = it->first;
      const size_t rest = it->second - need;
      free_.erase(it);
      if (rest)
        free_[offset + need] = rest;
      used_ += need;
      return true;
    }
    return false;
  }

  // Returns a block; neighbouring free blocks are merged.
  void release(size_t offset, size_t bytes) {
    size_t size = round_up(bytes ? bytes : 1);
    used_ -= size;
    auto next = free_.lower_bound(offset);
    if (next != free_.end() && offset + size == next->first) {
      size += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == offset) {
        prev->second += size;
        return;
      }
    }
    free_[offset] = size;
  }

  size_t largest_free() const {
    size_t best = 0;
    for (const auto &kv : free_)
      best = kv.second > best ? kv.second : best;
    return best;
  }
  size_t used() const { return used_; }
  size_t size() const { return size_; }
  size_t free_blocks() const { return free_.size(); }

private:
  std::map<size_t, size_t> free_; // offset -> bytes, disjoint and non-adjacent
  size_t size_ = 0, used_ = 0;
};

} // namespace msm_b200
