#include "common.hpp"

namespace cfdb {

void fail(int code, const std::string& msg) { throw Error(code, msg); }

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int code = e == cudaErrorMemoryAllocation ? 3 : e == cudaErrorNoDevice ? 4 : 2;
        throw Error(code, std::string("CUDA ") + what + ": " + cudaGetErrorString(e));
    }
}

void DeviceBuffer::allocate(size_t bytes) {
    release();
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(3, "CUDA malloc of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
    }
    ptr_ = p;
    bytes_ = bytes;
}

void DeviceBuffer::release() {
    if (ptr_ != nullptr) {
        cudaFree(ptr_);
        ptr_ = nullptr;
        bytes_ = 0;
    }
}

} // namespace cfdb
