// device_util.hpp -- small RAII and error helpers for the engine's host code.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <map>
#include <string>
#include <utility>

#include "rtm_b200.h"

namespace rtmb {

// Status-returning CUDA check used inside Engine methods (sets error_).
#define RTMB_CUDA(expr)                                                                      \
    do {                                                                                     \
        cudaError_t e__ = (expr);                                                            \
        if (e__ != cudaSuccess) return fail(RTM_B200_ECUDA, std::string(#expr) + ": " +     \
                                            cudaGetErrorString(e__));                        \
    } while (0)

#define RTMB_TRY(expr)                 \
    do {                               \
        int rc__ = (expr);             \
        if (rc__ != RTM_B200_OK) return rc__; \
    } while (0)

// Device allocation owned by one object.
class DevMem {
public:
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    DevMem(DevMem&& o) noexcept : p_(o.p_), bytes_(o.bytes_) { o.p_ = nullptr; o.bytes_ = 0; }
    DevMem& operator=(DevMem&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; bytes_ = o.bytes_; o.p_ = nullptr; o.bytes_ = 0; }
        return *this;
    }
    ~DevMem() { release(); }
    cudaError_t alloc(size_t bytes) {
        release();
        if (bytes == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p_, bytes);
        if (e != cudaSuccess) { p_ = nullptr; return e; }
        bytes_ = bytes;
        return cudaSuccess;
    }
    // Grow-only: keeps the buffer when it is already large enough.
    cudaError_t reserve(size_t bytes) { return bytes <= bytes_ ? cudaSuccess : alloc(bytes); }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        bytes_ = 0;
    }
    template <typename T = void>
    T* get() const { return static_cast<T*>(p_); }
    size_t bytes() const { return bytes_; }

private:
    void* p_ = nullptr;
    size_t bytes_ = 0;
};

// Page-locked host staging buffer.
class PinnedMem {
public:
    PinnedMem() = default;
    PinnedMem(const PinnedMem&) = delete;
    PinnedMem& operator=(const PinnedMem&) = delete;
    PinnedMem(PinnedMem&& o) noexcept : p_(o.p_), bytes_(o.bytes_) { o.p_ = nullptr; o.bytes_ = 0; }
    PinnedMem& operator=(PinnedMem&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; bytes_ = o.bytes_; o.p_ = nullptr; o.bytes_ = 0; }
        return *this;
    }
    ~PinnedMem() { release(); }
    cudaError_t reserve(size_t bytes) {
        if (bytes <= bytes_) return cudaSuccess;
        release();
        cudaError_t e = cudaMallocHost(&p_, bytes);
        if (e != cudaSuccess) { p_ = nullptr; return e; }
        bytes_ = bytes;
        return cudaSuccess;
    }
    void release() {
        if (p_) cudaFreeHost(p_);
        p_ = nullptr;
        bytes_ = 0;
    }
    template <typename T = void>
    T* get() const { return static_cast<T*>(p_); }
    size_t bytes() const { return bytes_; }

private:
    void* p_ = nullptr;
    size_t bytes_ = 0;
};

// First-fit allocator of byte ranges inside one device arena (snapshot store).
class RangeAllocator {
public:
    void reset(size_t capacity) {
        free_.clear();
        capacity_ = capacity;
        if (capacity) free_[0] = capacity;
    }
    // Returns true and the offset of a 256-byte aligned range.
    bool allocate(size_t bytes, size_t* off) {
        bytes = (bytes + 255) & ~(size_t)255;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                const size_t rest = it->second - bytes;
                const size_t noff = it->first + bytes;
                free_.erase(it);
                if (rest) free_[noff] = rest;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = (bytes + 255) & ~(size_t)255;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t capacity() const { return capacity_; }
    size_t largest_free() const {
        size_t m = 0;
        for (auto& kv : free_) m = kv.second > m ? kv.second : m;
        return m;
    }

private:
    std::map<size_t, size_t> free_;
    size_t capacity_ = 0;
};

}  // namespace rtmb
