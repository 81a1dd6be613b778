// gsc_pool.hpp -- first-fit sub-allocation of one address range (host-side
// bookkeeping only; no CUDA calls).  The batched instances and the serving
// loop place every device buffer of a problem inside a few large regions
// through it, so admitting or retiring a query costs no cudaMalloc/cudaFree
// and the device-memory budget is a hard cap.
#pragma once

#include <cstdint>
#include <iterator>
#include <map>

namespace gsc_b200 {

class RangePool {
public:
    static constexpr uint64_t kAlign = 256;
    static constexpr uint64_t kNone = ~0ull;

    explicit RangePool(uint64_t capacity = 0) { reset(capacity); }

    void reset(uint64_t capacity) {
        free_.clear();
        cap_ = capacity & ~(kAlign - 1);
        used_ = 0;
        if (cap_) free_[0] = cap_;
    }

    static uint64_t rounded(uint64_t bytes) { return ((bytes ? bytes : 1) + kAlign - 1) & ~(kAlign - 1); }

    // Offset of a free range of `bytes` (rounded up to kAlign), lowest first;
    // kNone when no free range is large enough.
    uint64_t alloc(uint64_t bytes) {
        const uint64_t need = rounded(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < need) continue;
            const uint64_t off = it->first, rest = it->second - need;
            free_.erase(it);
            if (rest) free_[off + need] = rest;
            used_ += need;
            return off;
        }
        return kNone;
    }

    // Returns a range from alloc(); neighbouring free ranges are merged.
    void release(uint64_t off, uint64_t bytes) {
        uint64_t n = rounded(bytes);
        used_ -= n;
        auto next = free_.lower_bound(off);
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                off = prev->first;
                n += prev->second;
                free_.erase(prev);
            }
        }
        if (next != free_.end() && off + n == next->first) {
            n += next->second;
            free_.erase(next);
        }
        free_[off] = n;
    }

    uint64_t capacity() const { return cap_; }
    uint64_t used() const { return used_; }
    uint64_t largest_free() const {
        uint64_t m = 0;
        for (const auto& kv : free_) m = kv.second > m ? kv.second : m;
        return m;
    }
    size_t free_ranges() const { return free_.size(); }

private:
    std::map<uint64_t, uint64_t> free_;   // offset -> length, disjoint and not adjacent
    uint64_t cap_ = 0;
    uint64_t used_ = 0;
};

}  // namespace gsc_b200
