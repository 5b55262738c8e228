// ba_api.cu -- C ABI of the bundle-adjustment kernels (include/xcb200.h).
#include <mutex>
#include <string>

#include "ba_kernels.h"
#include "common.cuh"

// scratch: [counter (256 B)][3 doubles per landmark: trial states, rounded to 32 doubles][118 doubles per landmark:
// the float64 back-substitution records]
extern "C" size_t xcb_ba_scratch_bytes(int nw, int Lt)
{
    (void)nw;
    const size_t L = (size_t)(Lt > 0 ? Lt : 1);
    return ((3 * L + 31) / 32 * 32 + 118 * L) * sizeof(double) + 256;
}

static int ba_fail(int code, const char* msg);
static int ba_grid(int grid, int nw);

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
    if (scratch_bytes < 256) return ba_fail(XCB_ERR_CAPACITY, "ba_solve_windows: scratch smaller than 256 bytes");
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
    e = xcb_launch_ba_windows(*w, max_slots, iters, lam0, mode, stats, dx0, dx0_stride, trial, counter, grid, st,
                              nullptr, scratch_bytes > 256 ? (scratch_bytes - 256) / sizeof(double) : 0);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    return XCB_OK;
}

extern "C" int xcb_ba_linearise_windows_dev(const xcb_ba_windows* w, int max_slots, double* out, int out_stride,
                                            double* stats, void* scratch, size_t scratch_bytes, int grid, void* stream)
{
    if (!w || !out || !stats || !scratch) return ba_fail(XCB_ERR_ARG, "ba_linearise_windows: null argument");
    if (w->nw <= 0) return XCB_OK;
    if (max_slots < 1 || max_slots > xcb_ba_max_slots())
        return ba_fail(XCB_ERR_CAPACITY, "ba_linearise_windows: max_slots out of range (1..20)");
    const long long nm = 6LL * max_slots;
    if (out_stride < nm * nm + nm) return ba_fail(XCB_ERR_ARG, "ba_linearise_windows: out stride too small");
    if (scratch_bytes < 256) return ba_fail(XCB_ERR_CAPACITY, "ba_linearise_windows: scratch smaller than 256 bytes");
    cudaStream_t st = (cudaStream_t)stream;
    int* counter = (int*)scratch;
    double* trial = (double*)((char*)scratch + 256);
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    e = xcb_launch_ba_windows(*w, max_slots, 1, 0.0, XCB_BA_LINEARISE, stats, out, out_stride, trial, counter,
                              ba_grid(grid, w->nw), st, nullptr,
                              scratch_bytes > 256 ? (scratch_bytes - 256) / sizeof(double) : 0);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    return XCB_OK;
}

extern void xcb_set_last_error(const std::string& m);

static int ba_fail(int code, const char* msg)
{
    xcb_set_last_error(std::string(msg));
    return code;
}

// Newton / adjoint scratch: [counter (256 B)][19 doubles per landmark][3 doubles per landmark: trial states of the
// constant-landmark window solve][the polish's copies of the reduced systems: 4 per window, one per CTA of its
// cluster]
extern "C" size_t xcb_ba_newton_scratch_bytes(int nw, int Lt)
{
    return ((size_t)(Lt > 0 ? Lt : 1) * 22 * sizeof(double) + 255) / 256 * 256 + 256 +
           xcb_ba_newton_copy_doubles(nw) * sizeof(double);
}

static int ba_grid(int grid, int nw)
{
    if (grid <= 0) {
        int dev = 0, sms = XCB_B200_SMS;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        grid = sms;
    }
    return grid > nw ? nw : grid;
}

extern "C" int xcb_ba_solve_windows_free_dev(const xcb_ba_windows* w, int Lt, int max_slots, int iters, double lam0,
                                             double* stats, void* scratch, size_t scratch_bytes, int grid,
                                             void* stream)
{
    if (!w || !stats || !scratch) return ba_fail(XCB_ERR_ARG, "ba_solve_windows_free: null argument");
    if (w->nw <= 0) return XCB_OK;
    if (max_slots < 1 || max_slots > xcb_ba_max_slots())
        return ba_fail(XCB_ERR_CAPACITY, "ba_solve_windows_free: max_slots out of range (1..20)");
    if (Lt < 0 || scratch_bytes < xcb_ba_newton_scratch_bytes(w->nw, Lt))
        return ba_fail(XCB_ERR_CAPACITY, "ba_solve_windows_free: scratch smaller than xcb_ba_newton_scratch_bytes");
    cudaStream_t st = (cudaStream_t)stream;
    int* counter = (int*)scratch;
    double* lsc = (double*)((char*)scratch + 256);
    double* trial = lsc + (size_t)(Lt > 0 ? Lt : 1) * 19;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    e = xcb_launch_ba_windows(*w, max_slots, iters, lam0, XCB_BA_FP64, stats, nullptr, 0, trial, counter,
                              ba_grid(grid, w->nw), st, lsc, (size_t)(Lt > 0 ? Lt : 1) * 3);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    return XCB_OK;
}

extern "C" int xcb_ba_newton_windows_dev(const xcb_ba_windows* w, int max_slots, int mode, int steps, int maxit,
                                         double tol, const double* gpose, double* gtheta, double* gisig, double* gz,
                                         double* stats, void* scratch, size_t scratch_bytes, int grid, void* stream)
{
    if (!w || !stats || !scratch) return ba_fail(XCB_ERR_ARG, "ba_newton: null argument");
    if (w->nw <= 0) return XCB_OK;
    if (max_slots < 1 || max_slots > xcb_ba_max_slots())
        return ba_fail(XCB_ERR_CAPACITY, "ba_newton: max_slots out of range (1..20)");
    if (mode != XCB_BA_NEWTON_POLISH && mode != XCB_BA_NEWTON_ADJOINT && mode != XCB_BA_NEWTON_POLISH_FIXED)
        return ba_fail(XCB_ERR_ARG, "ba_newton: mode");
    if (mode == XCB_BA_NEWTON_ADJOINT && (!gpose || !gtheta)) return ba_fail(XCB_ERR_ARG, "ba_newton: adjoint outputs");
    if (steps < 0 || maxit < 1) return ba_fail(XCB_ERR_ARG, "ba_newton: steps / maxit");
    cudaStream_t st = (cudaStream_t)stream;
    // scratch: [counter (256 B)][19 doubles per landmark ...][the reduced-system copies at the end]; the kernel
    // checks the batch's landmarks against the part before the copies
    const size_t ncopy = xcb_ba_newton_copy_doubles(w->nw);
    if (scratch_bytes < 256 + ncopy * sizeof(double))
        return ba_fail(XCB_ERR_CAPACITY, "ba_newton: scratch smaller than xcb_ba_newton_scratch_bytes(nw, 0)");
    int* counter = (int*)scratch;
    double* lsc = (double*)((char*)scratch + 256);
    const size_t lsc_doubles = (scratch_bytes - 256) / sizeof(double) - ncopy;
    double* scopy = lsc + lsc_doubles;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    if (grid <= 0) {
        int dev = 0, sms = XCB_B200_SMS;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        grid = sms;
    }
    // at most `grid` CTAs in all, up to 4 per window (a thread-block cluster) when there are fewer windows than CTAs
    e = xcb_launch_ba_newton(*w, max_slots, mode, steps, maxit, tol, gpose, gtheta, gisig, gz, stats, lsc, counter,
                             grid, st, lsc_doubles, scopy);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    return XCB_OK;
}

// ------------------------------------------------------------------------------------------------------------------
// Allocation-free batched window solve.
//
// Some callers cannot call cudaMalloc once they are running: a real-time frame loop, whose latency budget does not
// allow an allocation that may synchronise the device and take unbounded time, and a plugin whose host application
// owns the device memory budget through its own allocator.  xcb_ba_solve_windows_dev needs a scratch buffer from the
// caller; this variant needs none.  Its scratch (the work counter and the trial landmark states) lives in the
// file-scope device array below, XCB_BA_NOALLOC_SCRATCH_BYTES (4 MiB) that every GPU which loads libxcb200.so holds
// until the process exits.  That bounds one call to xcb_ba_noalloc_max_landmarks() landmarks in total.
//
// In host code g_ba_noalloc_scratch is only a host-side stand-in for the device array, not a device address: its
// device address is looked up once per device (cudaGetSymbolAddress, with that device current) by the first call on
// that device, so that first call should come before any stream capture.  All calls share the one array and it keeps
// the last call's contents: the work counter is cleared at the start of every call (the trial states are written
// before they are read), and calls that overlap on the GPU (two streams, or two threads) race on it.
// ------------------------------------------------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_ba_noalloc_scratch[XCB_BA_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[XCB_NOALLOC_MAX_DEVICES];

extern "C" int xcb_ba_noalloc_max_landmarks(void)
{
    return (int)((XCB_BA_NOALLOC_SCRATCH_BYTES - 256) / (3 * sizeof(double)));
}

extern "C" int xcb_ba_solve_windows_noalloc(const xcb_ba_windows* w, int Lt, int max_slots, int iters, double lam0,
                                            int mode, double* stats, double* dx0, int dx0_stride, int grid,
                                            void* stream)
{
    if (!w || !stats) return ba_fail(XCB_ERR_ARG, "ba_solve_windows_noalloc: null argument");
    if (Lt < 0) return ba_fail(XCB_ERR_ARG, "ba_solve_windows_noalloc: negative landmark count");
    if (Lt > xcb_ba_noalloc_max_landmarks())
        return ba_fail(XCB_ERR_CAPACITY, ("ba_solve_windows_noalloc: " + std::to_string(Lt) + " landmarks exceed the "
                                          "static scratch (at most " + std::to_string(xcb_ba_noalloc_max_landmarks()) +
                                          " per call); split the batch or use xcb_ba_solve_windows_dev").c_str());
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= XCB_NOALLOC_MAX_DEVICES) return ba_fail(XCB_ERR_ARG, "ba_solve_windows_noalloc: device ordinal");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_ba_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return ba_fail(XCB_ERR_CUDA, (std::string("ba_solve_windows_noalloc: cudaGetSymbolAddress: ") +
                                              cudaGetErrorString(e)).c_str());
            g_noalloc_addr[dev] = p;
        }
        base = g_noalloc_addr[dev];
    }
    return xcb_ba_solve_windows_dev(w, max_slots, iters, lam0, mode, stats, dx0, dx0_stride, base,
                                    XCB_BA_NOALLOC_SCRATCH_BYTES, grid, stream);
}

// ------------------------------------------------------------------------------------------------------------------
// Large-window path: every window's landmark passes spread over all SMs in chunks (see ba_window.cu).
extern "C" size_t xcb_ba_large_scratch_bytes(int nw, int slots, int Lt)
{
    return xcb_ba_large_scratch_bytes_impl(nw, slots, Lt);
}

extern "C" int xcb_ba_solve_windows_large_dev(const xcb_ba_windows* w, int slots, int Lt, const int32_t* chunks,
                                              int nchunks, int max_slots, int iters, double lam0, int mode,
                                              double* stats, double* dx0, int dx0_stride, void* scratch,
                                              size_t scratch_bytes, void* stream)
{
    if (!w || !stats || !scratch || (!chunks && nchunks > 0)) return ba_fail(XCB_ERR_ARG, "ba_solve_large: null argument");
    if (w->nw <= 0) return XCB_OK;
    if (max_slots < 1 || max_slots > xcb_ba_max_slots())
        return ba_fail(XCB_ERR_CAPACITY, "ba_solve_large: max_slots out of range (1..20)");
    if (mode != XCB_BA_FP64 && mode != XCB_BA_MIXED && mode != XCB_BA_MIXED_NOTC)
        return ba_fail(XCB_ERR_ARG, "ba_solve_large: bad mode");
    if (dx0 && dx0_stride < 6 * max_slots) return ba_fail(XCB_ERR_ARG, "ba_solve_large: dx0 stride too small");
    if (w->pr_m) return ba_fail(XCB_ERR_ARG, "ba_solve_large: windows with a marginal prior take xcb_ba_solve_windows_dev");
    if (slots < 0 || Lt < 0 || nchunks < 0 || iters < 0) return ba_fail(XCB_ERR_ARG, "ba_solve_large: negative size");
    if (scratch_bytes < xcb_ba_large_scratch_bytes_impl(w->nw, slots, Lt))
        return ba_fail(XCB_ERR_CAPACITY, "ba_solve_large: scratch smaller than xcb_ba_large_scratch_bytes");
    cudaError_t e = xcb_launch_ba_large(*w, slots, Lt, chunks, nchunks, max_slots, iters, lam0, mode, stats, dx0,
                                        dx0_stride, scratch, scratch_bytes, (cudaStream_t)stream);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    return XCB_OK;
}

extern "C" int xcb_ba_solve_windows_large_free_dev(const xcb_ba_windows* w, int slots, int Lt, const int32_t* chunks,
                                                   int nchunks, int max_slots, int iters, double lam0, double* stats,
                                                   void* scratch, size_t scratch_bytes, const void* newton_scratch,
                                                   size_t newton_scratch_bytes, void* stream)
{
    if (!w || !stats || !scratch || !newton_scratch || (!chunks && nchunks > 0))
        return ba_fail(XCB_ERR_ARG, "ba_solve_large_free: null argument");
    if (w->nw <= 0) return XCB_OK;
    if (max_slots < 1 || max_slots > xcb_ba_max_slots())
        return ba_fail(XCB_ERR_CAPACITY, "ba_solve_large_free: max_slots out of range (1..20)");
    if (w->pr_m) return ba_fail(XCB_ERR_ARG, "ba_solve_large_free: windows with a marginal prior take xcb_ba_solve_windows_free_dev");
    if (slots < 0 || Lt < 0 || nchunks < 0 || iters < 0) return ba_fail(XCB_ERR_ARG, "ba_solve_large_free: negative size");
    if (scratch_bytes < xcb_ba_large_scratch_bytes_impl(w->nw, slots, Lt))
        return ba_fail(XCB_ERR_CAPACITY, "ba_solve_large_free: scratch smaller than xcb_ba_large_scratch_bytes");
    // the flags: 19 doubles per landmark after the Newton scratch's first 256 bytes
    if (newton_scratch_bytes < 256 + (size_t)19 * (size_t)(Lt > 0 ? Lt : 1) * sizeof(double))
        return ba_fail(XCB_ERR_CAPACITY, "ba_solve_large_free: Newton scratch smaller than 19 doubles per landmark");
    const double* frz = (const double*)((const char*)newton_scratch + 256);
    cudaError_t e = xcb_launch_ba_large(*w, slots, Lt, chunks, nchunks, max_slots, iters, lam0, XCB_BA_FP64, stats,
                                        nullptr, 0, scratch, scratch_bytes, (cudaStream_t)stream, frz);
    if (e != cudaSuccess) return ba_fail(XCB_ERR_CUDA, cudaGetErrorString(e));
    return XCB_OK;
}
