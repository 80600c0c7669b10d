#include "common.hpp"

#include <algorithm>
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

} // namespace cfdb
