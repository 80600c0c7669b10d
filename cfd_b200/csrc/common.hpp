// Shared host-side utilities of the cfdb library: error propagation to the C ABI, device
// buffers and the host sparse-matrix type used for patterns and AMG hierarchies.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace cfdb {

// Error carrying a cfdb_status code; the C ABI converts it into a return value + message.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
#define CFDB_CUDA(call) ::cfdb::check_cuda((call), #call)

// Fails with status 4 (CFDB_ERR_NO_DEVICE of include/cfdb.h) when no CUDA device is visible:
// the library has no host path to fall back to.
inline void require_cuda_device() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        fail(4, "no CUDA device: this library has no host fallback");
    }
}

// Host CSR matrix (int32 indices, FP64 values).
struct HostCsr {
    int n_rows = 0;
    int n_cols = 0;
    std::vector<int> rp{0};
    std::vector<int> ci;
    std::vector<double> va;
    [[nodiscard]] int nnz() const { return rp.empty() ? 0 : rp.back(); }
    [[nodiscard]] bool empty() const { return n_rows == 0; }
};

// Owning device allocation (256-byte aligned), from the library's stream-ordered memory pool of
// the current device: the pool keeps freed memory for reuse, so a plan rebuild, which frees
// one plan and allocates the next, neither returns memory to the driver nor waits for the
// device to go idle as cudaFree does.
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t bytes) { allocate(bytes, false); }
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) {
        o.ptr_ = nullptr;
        o.bytes_ = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            release();
            ptr_ = o.ptr_;
            bytes_ = o.bytes_;
            o.ptr_ = nullptr;
            o.bytes_ = 0;
        }
        return *this;
    }
    // transient: from the pool of short-lived setup scratch
    void allocate(size_t bytes, bool transient = false);
    void release();
    [[nodiscard]] void* get() const { return ptr_; }
    template <class T> [[nodiscard]] T* as() const { return static_cast<T*>(ptr_); }
    [[nodiscard]] size_t bytes() const { return bytes_; }

private:
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
    int device_ = 0;
};

// Returns the freed blocks of the library's device pools on `device` to the driver.
void trim_device_pools(int device);

// Grow-only page-locked host buffer (staging of device-to-host reads).
class PinnedBuffer {
public:
    PinnedBuffer() = default;
    ~PinnedBuffer();
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    // at least `bytes` bytes (contents not kept when it grows)
    void* get(size_t bytes);
    [[nodiscard]] size_t bytes() const { return bytes_; }

private:
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
};

// Copies between pageable host arrays and device arrays through two page-locked chunks:
// all host threads copy one chunk between the caller's array and page-locked memory while
// the DMA of the other chunk runs, so a large copy moves at the DMA rate instead of the
// driver's single-threaded staging rate. Copies below kDirect bytes go straight through
// cudaMemcpyAsync, and so do copies from or to page-locked host memory. The chunks are
// reused after their last DMA has completed (events).
class StagedCopier {
public:
    StagedCopier() = default;
    ~StagedCopier();
    StagedCopier(const StagedCopier&) = delete;
    StagedCopier& operator=(const StagedCopier&) = delete;
    // enqueues the copy on st; src may be reused when this returns
    void to_device(void* dst, const void* src, size_t bytes, cudaStream_t st);
    // waits for the work already on st, then copies; returns when dst holds the data
    void to_host(void* dst, const void* src, size_t bytes, cudaStream_t st);

    static constexpr size_t kChunk = size_t(8) << 20;
    static constexpr size_t kDirect = size_t(4) << 20;

private:
    static bool page_locked(const void* p);
    void ready(int b);
    PinnedBuffer buf_[2];
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    bool pending_[2] = {false, false};
};

// Device arrays are grouped in an arena per engine so their footprint can be reported.
class DeviceArena {
public:
    template <class T> T* alloc(size_t count) {
        bufs_.emplace_back(sizeof(T) * (count > 0 ? count : 1));
        total_ += bufs_.back().bytes();
        return bufs_.back().as<T>();
    }
    template <class T> T* upload(const std::vector<T>& h, cudaStream_t s) {
        T* d = alloc<T>(h.size());
        if (!h.empty()) {
            CFDB_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
        }
        return d;
    }
    [[nodiscard]] size_t bytes() const { return total_; }
    void clear() {
        bufs_.clear();
        total_ = 0;
    }

private:
    std::vector<DeviceBuffer> bufs_;
    size_t total_ = 0;
};

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }
inline int ceil_div(int v, int m) { return (v + m - 1) / m; }

} // namespace cfdb
