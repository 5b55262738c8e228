// ba_kernels.h -- host-side launchers of the bundle-adjustment kernels (ba_*.cu), used by ba_api.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "xcb200.h"

typedef xcb_ba_windows XcbBaWindows;

size_t xcb_ba_smem_bytes(int maxP);
int xcb_ba_max_slots();
// frz (optional): the Newton scratch's per-landmark flags (19 doubles per landmark, entry 18); flagged landmarks are
// held constant
// trial_doubles: doubles available from lmp_trial on; when they also hold 118 per landmark after the trial states
// (rounded to 32), the float64 mode keeps each landmark's back-substitution record there instead of re-linearising
cudaError_t xcb_launch_ba_windows(const XcbBaWindows& d, int max_slots, int iters, double lam0, int mode,
                                  double* stats, double* dx0, int dx0_stride, double* lmp_trial, int* counter,
                                  int grid, cudaStream_t st, const double* frz = nullptr, size_t trial_doubles = 0);
size_t xcb_ba_newton_smem_bytes(int maxP);
// the Newton polish keeps a copy of each window's reduced system in global memory (scopy: this many doubles)
size_t xcb_ba_newton_copy_doubles(int nw);
cudaError_t xcb_launch_ba_newton(const XcbBaWindows& d, int max_slots, int mode, int steps, int maxit, double tol,
                                 const double* gpose, double* gtheta, double* gisig, double* gz, double* stats,
                                 double* lsc, int* counter, int grid, cudaStream_t st, size_t lsc_doubles,
                                 double* scopy);

// the large-window path: the same LM iterations as xcb_launch_ba_windows, the landmark passes over chunks of every
// window on all SMs (chunks: [nchunks][3] int32 on the device: window, first landmark, end), the per-window steps one
// CTA per window
size_t xcb_ba_large_scratch_bytes_impl(int nw, int slots, int Lt);
// frz (optional): constant-landmark flags as xcb_launch_ba_windows takes them
cudaError_t xcb_launch_ba_large(const XcbBaWindows& d, int slots, int Lt, const int* chunks, int nchunks,
                                int max_slots, int iters, double lam0, int mode, double* stats, double* dx0,
                                int dx0_stride, void* scratch, size_t scratch_bytes, cudaStream_t st,
                                const double* frz = nullptr);
