// ba_api.cu -- C ABI of the bundle-adjustment kernels (include/xcb200.h).
#include <string>

#include "ba_kernels.h"
#include "common.cuh"

extern "C" size_t xcb_ba_scratch_bytes(int nw, int Lt)
{
    (void)nw;
    return ((size_t)(Lt > 0 ? Lt : 1) * 3 * sizeof(double) + 255) / 256 * 256 + 256;
}

static int ba_fail(int code, const char* msg);

extern "C" int xcb_ba_solve_windows_dev(const xcb_ba_windows* w, int max_slots, int iters, double lam0, int mode,
                                        double* stats, double* dx0, int dx0_stride, void* scratch,
                                        size_t scratch_bytes, int grid, void* stream)
{
    if (!w || !stats || !scratch) return ba_fail(XCB_ERR_ARG, "ba_solve_windows: null argument");
    if (w->nw <= 0) return XCB_OK;
    if (max_slots < 1 || max_slots > xcb_ba_max_slots())
        return ba_fail(XCB_ERR_CAPACITY, "ba_solve_windows: max_slots out of range (1..20)");
    if (mode != XCB_BA_FP64 && mode != XCB_BA_MIXED) return ba_fail(XCB_ERR_ARG, "ba_solve_windows: bad mode");
    if (dx0 && dx0_stride < 6 * max_slots) return ba_fail(XCB_ERR_ARG, "ba_solve_windows: dx0 stride too small");
    cudaStream_t st = (cudaStream_t)stream;
    // scratch: [counter (256 B)][trial landmark states]
    int* counter = (int*)scratch;
    double* trial = (double*)((char*)scratch + 256);
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    if (grid <= 0) {
        int dev = 0, sms = XCB_B200_SMS;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        grid = sms;
    }
    if (grid > w->nw) grid = w->nw;
    (void)scratch_bytes;
    e = xcb_launch_ba_windows(*w, max_slots, iters, lam0, mode, stats, dx0, dx0_stride, trial, counter, grid, st);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    return XCB_OK;
}

extern void xcb_set_last_error(const std::string& m);

static int ba_fail(int code, const char* msg)
{
    xcb_set_last_error(std::string(msg));
    return code;
}
