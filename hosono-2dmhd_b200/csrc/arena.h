// arena.h -- first-fit sub-allocator over one fixed range of bytes.
//
// The server takes its memory budget from the device in one allocation at
// start-up and places every admitted solve's buffers inside it, so admission
// and retirement never call cudaMalloc/cudaFree (both may synchronise the
// device) and "does this request fit" is an exact question about free ranges.
// Offsets are aligned to 256 bytes; freed ranges merge with free neighbours.
// Pure host code (no CUDA), so it is unit-tested on the CPU.
#pragma once

#include <cstddef>
#include <iterator>
#include <map>

namespace hosono {

class Arena {
  public:
    static constexpr size_t kAlign = 256;

    void reset(size_t bytes) {
        free_.clear();
        used_.clear();
        cap_ = bytes / kAlign * kAlign;
        inUse_ = 0;
        if (cap_) free_[0] = cap_;
    }

    static size_t round_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

    // first free range that holds `bytes`; false when none does
    bool alloc(size_t bytes, size_t* off) {
        const size_t n = round_up(bytes ? bytes : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const size_t o = it->first, rest = it->second - n;
            free_.erase(it);
            if (rest) free_[o + n] = rest;
            used_[o] = n;
            inUse_ += n;
            *off = o;
            return true;
        }
        return false;
    }

    // returns false if `off` is not the start of a live block
    bool release(size_t off) {
        auto u = used_.find(off);
        if (u == used_.end()) return false;
        size_t o = off, n = u->second;
        used_.erase(u);
        inUse_ -= n;
        auto next = free_.lower_bound(o);
        if (next != free_.end() && o + n == next->first) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == o) {
                o = prev->first;
                n += prev->second;
                free_.erase(prev);
            }
        }
        free_[o] = n;
        return true;
    }

    // whether a block of `bytes` could be placed now
    bool fits(size_t bytes) const {
        const size_t n = round_up(bytes ? bytes : 1);
        for (const auto& f : free_)
            if (f.second >= n) return true;
        return false;
    }
    size_t capacity() const { return cap_; }
    size_t used() const { return inUse_; }
    size_t largest_free() const {
        size_t m = 0;
        for (const auto& f : free_) m = f.second > m ? f.second : m;
        return m;
    }
    size_t blocks() const { return used_.size(); }

    // invariants: free and used ranges tile [0, cap) without overlap, no two
    // free ranges touch, every offset is aligned
    bool check() const {
        std::map<size_t, std::pair<size_t, bool>> all;
        for (const auto& f : free_) all[f.first] = {f.second, true};
        for (const auto& u : used_) {
            if (all.count(u.first)) return false;
            all[u.first] = {u.second, false};
        }
        size_t at = 0, sumUsed = 0;
        bool prevFree = false;
        for (const auto& a : all) {
            if (a.first != at || a.first % kAlign || a.second.first == 0 || a.second.first % kAlign) return false;
            if (a.second.second && prevFree) return false;
            prevFree = a.second.second;
            if (!a.second.second) sumUsed += a.second.first;
            at += a.second.first;
        }
        return at == cap_ && sumUsed == inUse_;
    }

  private:
    std::map<size_t, size_t> free_, used_;  // offset -> bytes
    size_t cap_ = 0, inUse_ = 0;
};

}  // namespace hosono
