// Shared host/device infrastructure of the B200 pressure-solve library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "voluma_b200.h"

namespace vlm {

// Error carried from the internals to the C ABI, which turns it into a vlm_status.
struct Error : std::runtime_error {
    vlm_status status;
    Error(vlm_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define VLM_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            throw ::vlm::Error(e_ == cudaErrorMemoryAllocation ? VLM_ERR_OOM : VLM_ERR_CUDA,        \
                               std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

#define VLM_REQUIRE(cond, status, msg)                  \
    do {                                                \
        if (!(cond)) throw ::vlm::Error(status, (msg)); \
    } while (0)

// Owning device allocation (cudaMalloc; freed on destruction).
template <class T> class DBuf {
public:
    DBuf() = default;
    explicit DBuf(size_t n) { resize(n); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    ~DBuf() { release(); }
    void resize(size_t n) {
        if (n == n_) return;
        release();
        if (n) VLM_CUDA(cudaMalloc(&p_, n * sizeof(T)));
        n_ = n;
    }
    void upload(const T* h, size_t n, cudaStream_t s) {
        resize(n);
        if (n) VLM_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
    void zero(cudaStream_t s) { if (n_) VLM_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s)); }
    T* get() const { return p_; }
    size_t size() const { return n_; }
    size_t bytes() const { return n_ * sizeof(T); }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }

private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

// Records the message vlm_last_error(NULL) returns on this thread.
void setThreadError(const std::string& msg);

// Row chunk handed to one CTA of a row kernel: rows [start, start+count), count <= 256.
// sys/slot are used by reduction kernels (system index; partial-sum slot).
struct Chunk {
    int32_t start, count, sys, slot;
};

constexpr int kRowsPerCta = 256;
// Level-0 Krylov kernels give each CTA up to this many rows (4 per thread): fewer partial sums.
constexpr int kWideRows = 1024;
// Rows of one block-hybrid Gauss-Seidel block (one CTA of that many threads).
constexpr int kBlockRows = 512;
constexpr int kSlice = 32;  // SELL slice height (one warp)

}  // namespace vlm
