// Frontier arena of the serving loop: first-fit sub-allocation of one device range, with free
// ranges kept by offset and merged with their neighbours when released.  RangeAllocator is the
// host-only bookkeeping (offsets in bytes), so it can be tested without a GPU.
#pragma once

#include <stdint.h>

#include <algorithm>
#include <iterator>
#include <map>

namespace csm {

constexpr uint64_t kGranule = 256;

class RangeAllocator {
  public:
    void reset(uint64_t size) {
        size_ = size / kGranule * kGranule;
        used_ = 0;
        free_.clear();
        if (size_) free_[0] = size_;
    }
    // Grants min(want, largest free range) bytes, rounded up to the granule, if that is at
    // least `least`; returns the granted size (0: nothing granted) and its offset.
    uint64_t take(uint64_t want, uint64_t least, uint64_t *offset) {
        want = (want + kGranule - 1) / kGranule * kGranule;
        auto best = free_.end();
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (best == free_.end() || it->second > best->second) best = it;
        if (best == free_.end()) return 0;
        const uint64_t got = std::min(want, best->second);
        if (got == 0 || got < least) return 0;
        const uint64_t off = best->first, len = best->second;
        free_.erase(best);
        if (len > got) free_[off + got] = len - got;
        used_ += got;
        *offset = off;
        return got;
    }
    void give(uint64_t off, uint64_t bytes) {
        if (!bytes) return;
        used_ -= bytes;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && next->first == off + bytes) {
            bytes += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
    uint64_t used() const { return used_; }
    uint64_t size() const { return size_; }
    size_t free_ranges() const { return free_.size(); }
    uint64_t largest_free() const {
        uint64_t m = 0;
        for (auto &f : free_) m = std::max(m, f.second);
        return m;
    }

  private:
    uint64_t size_ = 0, used_ = 0;
    std::map<uint64_t, uint64_t> free_;
};

}  // namespace csm
