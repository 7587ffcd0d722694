// Status codes and the thread-local error message of the C ABI. The reference
// exits on a CUDA error (src/ising_gpu.cuh:44-52); the library reports it.
#include <cstdio>
#include <mutex>
#include <string>

#include "qb_internal.hpp"

namespace qb {

namespace {
thread_local std::string g_last_error;
thread_local bool g_async_on = false;
thread_local bool g_free_legacy = false;
thread_local cudaStream_t g_async_stream = nullptr;
constexpr int kMaxPoolDevices = 64;
}

AsyncAllocScope::AsyncAllocScope(cudaStream_t st, bool free_on_legacy)
    : prev(g_async_stream), prev_on(g_async_on), prev_legacy(g_free_legacy) {
    g_async_on = true;
    g_async_stream = st;
    g_free_legacy = free_on_legacy;
}

AsyncAllocScope::~AsyncAllocScope() {
    g_async_on = prev_on;
    g_async_stream = prev;
    g_free_legacy = prev_legacy;
}

cudaMemPool_t library_pool(int dev) {
    static std::mutex mu;
    static cudaMemPool_t pools[kMaxPoolDevices] = {};
    if (dev < 0 || dev >= kMaxPoolDevices) return nullptr;
    std::lock_guard<std::mutex> g(mu);
    if (!pools[dev]) {
        cudaMemPoolProps pr{};
        pr.allocType = cudaMemAllocationTypePinned;
        pr.location.type = cudaMemLocationTypeDevice;
        pr.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &pr) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = ~uint64_t(0);   // freed memory stays in the pool
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = p;
    }
    return pools[dev];
}

void set_error(const std::string& msg) { g_last_error = msg; }

qb_status fail(qb_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

qb_status cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e),
                  what, file, line);
    g_last_error = buf;
    return e == cudaErrorMemoryAllocation ? QB_ENOMEM : QB_ECUDA;
}

qb_status DevBuf::alloc(size_t n) {
    release();
    if (n == 0) return QB_OK;
    cudaError_t e;
    if (g_async_on) {
        int dev = 0;
        cudaMemPool_t pool = cudaGetDevice(&dev) == cudaSuccess ? library_pool(dev) : nullptr;
        e = pool ? cudaMallocFromPoolAsync(&p, n, pool, g_async_stream) : cudaMallocAsync(&p, n, g_async_stream);
        pooled = e == cudaSuccess;
        sync_free = pooled && g_free_legacy;
        pool_stream = g_free_legacy ? nullptr : g_async_stream;
    } else {
        e = cudaMalloc(&p, n);
    }
    if (e != cudaSuccess) {
        p = nullptr;
        return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    }
    bytes = n;
    return QB_OK;
}

qb_status upload(DevBuf& dst, const void* src, size_t bytes, cudaStream_t st) {
    qb_status s = dst.alloc(bytes);
    if (s != QB_OK) return s;
    if (bytes) QB_CUDA(cudaMemcpyAsync(dst.p, src, bytes, cudaMemcpyHostToDevice, st));
    return QB_OK;
}

}  // namespace qb

extern "C" const char* qb_status_string(qb_status s) {
    switch (s) {
        case QB_OK: return "ok";
        case QB_EINVAL: return "invalid argument";
        case QB_ENOMEM: return "out of memory";
        case QB_EREFUSED: return "refused by the planner";
        case QB_ETIMEDOUT: return "timed out";
        case QB_ECUDA: return "CUDA error";
        case QB_ENOTSUP: return "not supported";
        case QB_ECANCELLED: return "cancelled";
        case QB_EBUSY: return "busy";
    }
    return "unknown status";
}

extern "C" const char* qb_last_error(void) { return qb::g_last_error.c_str(); }

extern "C" int32_t qb_abi_version(void) { return QUBLAR_ABI_VERSION; }

extern "C" int32_t qb_device_count(void) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        qb::cuda_fail(e, "cudaGetDeviceCount", __FILE__, __LINE__);
        return -1;
    }
    return n;
}
