#include "common.hpp"

#include <algorithm>
#include <cstring>
#include <cstdint>
#include <map>
#include <mutex>

namespace cfdb {

void fail(int code, const std::string& msg) { throw Error(code, msg); }

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int code = e == cudaErrorMemoryAllocation ? 3 : e == cudaErrorNoDevice ? 4 : 2;
        throw Error(code, std::string("CUDA ") + what + ": " + cudaGetErrorString(e));
    }
}

namespace {

// Two pools per device, created on first use: one for long-lived plan arrays and one for
// transient setup scratch, so that the scratch of one setup finds the blocks of the previous
// setup free instead of interleaved with arrays that stay. Freed blocks stay in their pool (no
// release threshold) and are reused by later allocations of any thread.
cudaMemPool_t device_pool(int device, bool transient) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    const int key = 2 * device + (transient ? 1 : 0);
    auto it = pools.find(key);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    check_cuda(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
    uint64_t keep = UINT64_MAX;
    check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    pools[key] = pool;
    return pool;
}

} // namespace

void trim_device_pools(int device) {
    for (const bool transient : {false, true}) {
        check_cuda(cudaMemPoolTrimTo(device_pool(device, transient), 0), "cudaMemPoolTrimTo");
    }
}

void DeviceBuffer::allocate(size_t bytes, bool transient) {
    release();
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    void* p = nullptr;
    // allocated in the order of this thread's default stream, then completed, so the block
    // can be used from any stream
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, device_pool(dev, transient), cudaStreamPerThread);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(3, "CUDA malloc of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
    }
    ptr_ = p;
    bytes_ = bytes;
    device_ = dev;
}

PinnedBuffer::~PinnedBuffer() {
    if (ptr_ != nullptr) cudaFreeHost(ptr_);
}

void* PinnedBuffer::get(size_t bytes) {
    if (bytes <= bytes_ && ptr_ != nullptr) return ptr_;
    if (ptr_ != nullptr) {
        cudaFreeHost(ptr_);
        ptr_ = nullptr;
        bytes_ = 0;
    }
    const size_t want = std::max(bytes, static_cast<size_t>(1) << 20);
    void* p = nullptr;
    const cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(3, "CUDA host allocation of " + std::to_string(want) + " bytes: " + cudaGetErrorString(e));
    }
    ptr_ = p;
    bytes_ = want;
    return ptr_;
}

void DeviceBuffer::release() {
    // callers release a buffer only once the work that used it has completed
    if (ptr_ != nullptr) {
        int cur = 0;
        cudaGetDevice(&cur);
        if (cur != device_) cudaSetDevice(device_);
        cudaFreeAsync(ptr_, cudaStreamPerThread);
        if (cur != device_) cudaSetDevice(cur);
        ptr_ = nullptr;
        bytes_ = 0;
    }
}


namespace {

// host memcpy by all OpenMP threads, in blocks of at least 256 KB
void parallel_copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kBlock = size_t(256) << 10;
    const long long nblk = static_cast<long long>((bytes + kBlock - 1) / kBlock);
    auto* d = static_cast<char*>(dst);
    const auto* s = static_cast<const char*>(src);
#pragma omp parallel for schedule(static) if (nblk > 1)
    for (long long b = 0; b < nblk; ++b) {
        const size_t off = static_cast<size_t>(b) * kBlock;
        std::memcpy(d + off, s + off, std::min(kBlock, bytes - off));
    }
}

} // namespace

StagedCopier::~StagedCopier() {
    for (int b = 0; b < 2; ++b) {
        if (ev_[b] != nullptr) {
            cudaEventSynchronize(ev_[b]);
            cudaEventDestroy(ev_[b]);
        }
    }
}

void StagedCopier::ready(int b) {
    if (ev_[b] == nullptr) CFDB_CUDA(cudaEventCreateWithFlags(&ev_[b], cudaEventDisableTiming));
    if (pending_[b]) {
        CFDB_CUDA(cudaEventSynchronize(ev_[b]));
        pending_[b] = false;
    }
}

bool StagedCopier::page_locked(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

void StagedCopier::to_device(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    if (bytes < kDirect || page_locked(src)) {
        CFDB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        return;
    }
    auto* d = static_cast<char*>(dst);
    const auto* s = static_cast<const char*>(src);
    for (size_t off = 0, k = 0; off < bytes; off += kChunk, ++k) {
        const int b = static_cast<int>(k & 1);
        const size_t len = std::min(kChunk, bytes - off);
        ready(b);
        void* pin = buf_[b].get(kChunk);
        parallel_copy(pin, s + off, len);
        CFDB_CUDA(cudaMemcpyAsync(d + off, pin, len, cudaMemcpyHostToDevice, st));
        CFDB_CUDA(cudaEventRecord(ev_[b], st));
        pending_[b] = true;
    }
}

void StagedCopier::to_host(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    if (bytes < kDirect || page_locked(dst)) {
        CFDB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
        CFDB_CUDA(cudaStreamSynchronize(st));
        return;
    }
    auto* d = static_cast<char*>(dst);
    const auto* s = static_cast<const char*>(src);
    const size_t nchunks = (bytes + kChunk - 1) / kChunk;
    auto issue = [&](size_t k) {
        const int b = static_cast<int>(k & 1);
        const size_t off = k * kChunk;
        ready(b);
        CFDB_CUDA(cudaMemcpyAsync(buf_[b].get(kChunk), s + off, std::min(kChunk, bytes - off),
                                  cudaMemcpyDeviceToHost, st));
        CFDB_CUDA(cudaEventRecord(ev_[b], st));
        pending_[b] = true;
    };
    issue(0);
    if (nchunks > 1) issue(1);
    for (size_t k = 0; k < nchunks; ++k) {
        const int b = static_cast<int>(k & 1);
        ready(b); // chunk k has arrived
        const size_t off = k * kChunk;
        parallel_copy(d + off, buf_[b].get(kChunk), std::min(kChunk, bytes - off));
        if (k + 2 < nchunks) issue(k + 2);
    }
}

} // namespace cfdb
