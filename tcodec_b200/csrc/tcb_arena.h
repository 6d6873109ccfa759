// tcb_arena.h — device-memory arena for the served form.
//
// One cudaMalloc of the whole HBM budget at server creation; every admitted
// session's frames, MV grids, decision records and flags are carved out of
// it (first fit over an offset-ordered free list, 256-byte granules,
// neighbours coalesced on free).  Admission is therefore an exact
// accounting question — does the session's footprint fit in what is free —
// and sessions come and go without cudaMalloc / cudaFree (which would
// synchronise the device) while other sessions' kernels run.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <unordered_map>

#include <cuda_runtime.h>

#include "tcb_alloc.h"

namespace tcb {

class DeviceArena {
public:
    static constexpr size_t GRANULE = 256;
    static size_t round_up(size_t n) { return (n + GRANULE - 1) & ~(GRANULE - 1); }

    cudaError_t init(size_t bytes) {
        cap_ = round_up(bytes);
        cudaError_t e = dev_alloc(&base_, cap_);
        if (e != cudaSuccess) { base_ = nullptr; cap_ = 0; return e; }
        free_.clear();
        live_.clear();
        free_[0] = cap_;
        used_ = 0;
        return cudaSuccess;
    }
    void destroy() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
        cap_ = used_ = 0;
        free_.clear();
        live_.clear();
    }
    void *alloc(size_t n) {
        n = round_up(n ? n : 1);
        std::lock_guard<std::mutex> lk(mu_);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const size_t off = it->first, rest = it->second - n;
            free_.erase(it);
            if (rest) free_[off + n] = rest;
            live_[off] = n;
            used_ += n;
            return base_ + off;
        }
        return nullptr;
    }
    // Returns false for a pointer this arena did not hand out.
    bool release(void *p) {
        if (!p) return true;
        std::lock_guard<std::mutex> lk(mu_);
        const size_t off = (size_t)((uint8_t *)p - base_);
        auto lv = live_.find(off);
        if ((uint8_t *)p < base_ || lv == live_.end()) return false;
        size_t start = off, len = lv->second;
        live_.erase(lv);
        used_ -= len;
        auto nx = free_.lower_bound(start);
        if (nx != free_.end() && nx->first == start + len) { len += nx->second; nx = free_.erase(nx); }
        if (nx != free_.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == start) { start = pv->first; len += pv->second; free_.erase(pv); }
        }
        free_[start] = len;
        return true;
    }
    bool owns(const void *p) const { return base_ && (const uint8_t *)p >= base_ && (const uint8_t *)p < base_ + cap_; }
    size_t capacity() const { return cap_; }
    size_t used() const { return used_; }
    // Largest single block that alloc() could return right now.
    size_t largest_free() {
        std::lock_guard<std::mutex> lk(mu_);
        size_t m = 0;
        for (auto &f : free_) m = f.second > m ? f.second : m;
        return m;
    }

private:
    uint8_t *base_ = nullptr;
    size_t cap_ = 0, used_ = 0;
    std::map<size_t, size_t> free_;              // offset -> bytes, no two adjacent
    std::unordered_map<size_t, size_t> live_;    // offset -> bytes
    std::mutex mu_;
};

}  // namespace tcb
