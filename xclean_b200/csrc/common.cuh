// common.cuh -- shared helpers of the sm_100a kernels (xclean B200 hot path).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <mutex>
#include "xcb200.h"

typedef unsigned char u8;
typedef long long i64;
typedef unsigned long long u64;

#define XCB_REFL(i, n) ((i) < 0 ? -(i) : ((i) >= (n) ? 2 * (n) - 2 - (i) : (i)))

#define CUDART_INF_F __int_as_float(0x7f800000)
#define XCB_INF __longlong_as_double(0x7ff0000000000000LL)
#define XCB_NAN __longlong_as_double(0x7ff8000000000000LL)

// number of SMs on a B200; grids of persistent kernels are multiples of it
#define XCB_B200_SMS 148

// float -> order-preserving unsigned (numpy ranks -0.0 equal to +0.0)
__device__ __forceinline__ unsigned int xcb_ord_f(float v)
{
    unsigned int u = __float_as_uint(v);
    if (u == 0x80000000u) u = 0u;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// candidate rank key: response descending, then y ascending, then x ascending (np.lexsort((xs, ys, -resp)))
__device__ __forceinline__ u64 xcb_key(float v, int y, int x)
{
    return ((u64)xcb_ord_f(v) << 32) | ((u64)(0xFFFF - y) << 16) | (u64)(0xFFFF - x);
}
__device__ __forceinline__ int xcb_key_x(u64 k) { return 0xFFFF - (int)(k & 0xFFFFull); }
__device__ __forceinline__ int xcb_key_y(u64 k) { return 0xFFFF - (int)((k >> 16) & 0xFFFFull); }

#define XCB_CHECK_LAUNCH() (cudaGetLastError())

// A kernel's dynamic shared-memory opt-in applies to the device that is current when it is set, so it is raised once
// per device ordinal (one XcbAttrOnce per call site; thread-safe).  The first call on a device sets it: make that
// call outside any stream capture.
struct XcbAttrOnce {
    std::mutex mu;
    int bytes[XCB_NOALLOC_MAX_DEVICES] = {};
};
static inline cudaError_t xcb_smem_attr_once(XcbAttrOnce& s, const void* func, int bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= XCB_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(s.mu);
    if (s.bytes[dev] >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) s.bytes[dev] = bytes;
    return e;
}
