// front_kernels.h -- host-side launchers of the frontend kernels (defined in front_*.cu, used by front_api.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

struct XcbDetectGeom {
    // greedy cells (features.Frontend._detect: s = max(4, sqrt(WH/n)), cell = floor(y/s) * ncx + floor(x/s))
    double s, r2;
    int ncx, gh, ncell;
    // threshold cells (features.Frontend._response: c = max(4, round(s)), c x c blocks of the zero-padded response)
    int c, gwc, ghc;
    int border;
    // device: ybeg [gh+1], xbeg [ncx+1] pixel ranges of the cell rows / columns; coff [ncell+1] list offsets
    const int* ybeg;
    const int* xbeg;
    const int* coff;
    int max_cell_px;
};

struct XcbNoiseTree {
    int nleaf, nnode, nlvl, root;
    const long long* lstart;   // [nleaf]
    const int* llen;           // [nleaf]
    const int* left;           // [nnode]
    const int* right;          // [nnode]
    const int* lvl;            // [nlvl + 1]
};

cudaError_t xcb_launch_response(const uint8_t* img, int F, int H, int W, int dy_vend, int dx_vend, float* R,
                                int* anypos, cudaStream_t st);
cudaError_t xcb_launch_noise(const uint8_t* img, int F, int H, int W, const XcbNoiseTree& t, float* nodeval,
                             double K, double Q, double* floor_d, float* floor_f, cudaStream_t st);
cudaError_t xcb_launch_candidates(const float* R, int F, int H, int W, const XcbDetectGeom& g, const float* floor_f,
                                  const int* anypos, float* thr, unsigned long long* raw, unsigned long long* sorted,
                                  int* ccount, cudaStream_t st);
cudaError_t xcb_launch_greedy(const float* R, int F, int H, int W, const XcbDetectGeom& g,
                              const unsigned long long* sorted, const int* ccount, int budget, int cap, float* kp,
                              int* counts, int* rounds, unsigned int* err, cudaStream_t st);
size_t xcb_greedy_smem(int ncell);
int xcb_greedy_smem_limit();
cudaError_t xcb_greedy_init_attrs();
cudaError_t xcb_stereo_init_attrs();

cudaError_t xcb_launch_blur(const uint8_t* img, int F, int H, int W, const float* kf, int vr, int vc, uint8_t* out,
                            cudaStream_t st);
cudaError_t xcb_launch_orb(const uint8_t* blur, int F, int Hp, int Wp, const float* kp, const int* counts, int cap,
                           const int8_t* pat, uint8_t* desc, cudaStream_t st);

cudaError_t xcb_launch_shift(const uint8_t* R, int F, int H, int W, double dy, float* Rs, cudaStream_t st);
// stereo over points: mode A (kpd != NULL): n points of frame 0, per-point dlo/dhi; mode B: F x cap float32 keypoints
// with counts, scalar dlo/dhi
cudaError_t xcb_launch_stereo(const uint8_t* L, const uint8_t* R8, const float* Rs, int F, int H, int W,
                              const double* kpd, const long long* dlo_a, const long long* dhi_a, int n,
                              const float* kpf, const int* counts, int cap, int dlo, int dhi, int band, int half,
                              double* od, double* osig, uint8_t* ook, double* ozn, double* ody, unsigned int* err,
                              void* jobs, int warps, int grp, cudaStream_t st);
// the search kernel appends the points that pass to a job list for the LK kernel: xcb_stereo_jobs_bytes(points) of
// device scratch per launch (one launch at a time per buffer)
size_t xcb_stereo_jobs_bytes(long long npts);
cudaError_t xcb_launch_lkcheck(const double* As, const double* gs, int n, double* X, double* Inv, cudaStream_t st);

// Hamming over frame pairs: pair p matches A_p (LA[p] rows at A + p * strideA) with B_p.  Lengths are read on the
// device (pointers to counts), so the launch needs no host sync.
struct XcbHamPairs {
    const uint8_t* A;
    const uint8_t* B;
    long long strideA, strideB;   // bytes between consecutive pairs' descriptor arrays
    const int* LA;                // [npair] query counts
    const int* NB;                // [npair] train counts
    int npair, maxL, maxN;
};
// rows: b1 / b2 / bi [npair x maxL] (best, second, first index of the best); columns: ci [npair x maxN] holds
// (distance << 16 | first-minimum query) as unsigned, all ones where the pair has no query (set by this call)
cudaError_t xcb_launch_hamming(const XcbHamPairs& p, int* b1, int* b2, int* bi, int* ci, cudaStream_t st);
cudaError_t xcb_launch_match_epilogue(const XcbHamPairs& p, const int* b1, const int* b2, const int* bi,
                                      const int* ci, int ham_max, double ratio, long long* i0, long long* i1,
                                      long long out_stride, int* nmatch, cudaStream_t st);
