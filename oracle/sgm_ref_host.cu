// sgm_ref_host.cu -- the launches of the reference's SGM32.compute_gpu (src/xclean/stereo/sgm32.py:278-360), restated
// in C++ around the reference's own kernels (oracle/_ref/sgm32_kernels.cu, read out of sgm32.py by
// oracle/build_ref_sgm.py).  Test infrastructure only: the GPU tests run it as the checker of the device SGM.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "sgm32_kernels.cu"

namespace {

// sgm32.directions(): the 4 axis paths, then every sign combination of the 7 oblique families
void directions(std::vector<int>& dx, std::vector<int>& dy, std::vector<int>& num, std::vector<int>& den)
{
    const int ax[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
    for (auto& a : ax) { dx.push_back(a[0]); dy.push_back(a[1]); num.push_back(1); den.push_back(1); }
    const int fam[7][4] = {{1, 1, 1, 1}, {1, 2, 9, 4}, {2, 1, 9, 4}, {1, 3, 19, 6},
                           {3, 1, 19, 6}, {2, 3, 18, 5}, {3, 2, 18, 5}};
    for (auto& f : fam)
        for (int sx : {1, -1})
            for (int sy : {1, -1}) {
                dx.push_back(sx * f[0]); dy.push_back(sy * f[1]); num.push_back(f[2]); den.push_back(f[3]);
            }
}

}  // namespace

#define RCK(x)                                 \
    do {                                       \
        if ((x) != cudaSuccess) return -2;     \
    } while (0)

// the reference's buffers and launch tables for one image size (sgm32.SGM32.__init__'s allocations)
struct XrSgm {
    int H = 0, W = 0, npaths = 0;
    unsigned long long *L0 = nullptr, *R0 = nullptr;
    unsigned short *L1 = nullptr, *R1 = nullptr, *S = nullptr;
    unsigned char* C = nullptr;
    float* dr = nullptr;
    int *d_sx = nullptr, *d_sy = nullptr, *d_sd = nullptr, *d_dx = nullptr, *d_dy = nullptr, *d_p1 = nullptr,
        *d_p2 = nullptr;
    ~XrSgm()
    {
        cudaFree(L0); cudaFree(R0); cudaFree(L1); cudaFree(R1); cudaFree(C); cudaFree(S); cudaFree(dr);
        cudaFree(d_sx); cudaFree(d_sy); cudaFree(d_sd); cudaFree(d_dx); cudaFree(d_dy); cudaFree(d_p1); cudaFree(d_p2);
    }
    int init(int H_, int W_, int p1, int p2)
    {
        H = H_; W = W_;
        std::vector<int> dx, dy, num, den;
        directions(dx, dy, num, den);
        std::vector<int> p1s, p2s, sx, sy, sd;
        for (size_t k = 0; k < dx.size(); ++k) {
            p1s.push_back(p1 * num[k] / den[k]);
            p2s.push_back(p2 * num[k] / den[k]);
            // sgm32.path_starts: pixels whose predecessor p - (dx, dy) lies outside the image, in row-major order
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x) {
                    const int px = x - dx[k], py = y - dy[k];
                    if (px < 0 || px >= W || py < 0 || py >= H) { sx.push_back(x); sy.push_back(y); sd.push_back((int)k); }
                }
        }
        npaths = (int)sx.size();
        const size_t n = (size_t)H * W;
        RCK(cudaMalloc(&L0, n * 8)); RCK(cudaMalloc(&R0, n * 8)); RCK(cudaMalloc(&L1, n * 2)); RCK(cudaMalloc(&R1, n * 2));
        RCK(cudaMalloc(&C, n * 128)); RCK(cudaMalloc(&S, n * 128 * 2)); RCK(cudaMalloc(&dr, n * 4));
        RCK(cudaMalloc(&d_sx, npaths * 4)); RCK(cudaMalloc(&d_sy, npaths * 4)); RCK(cudaMalloc(&d_sd, npaths * 4));
        RCK(cudaMalloc(&d_dx, 32 * 4)); RCK(cudaMalloc(&d_dy, 32 * 4)); RCK(cudaMalloc(&d_p1, 32 * 4));
        RCK(cudaMalloc(&d_p2, 32 * 4));
        RCK(cudaMemcpy(d_sx, sx.data(), npaths * 4, cudaMemcpyHostToDevice));
        RCK(cudaMemcpy(d_sy, sy.data(), npaths * 4, cudaMemcpyHostToDevice));
        RCK(cudaMemcpy(d_sd, sd.data(), npaths * 4, cudaMemcpyHostToDevice));
        RCK(cudaMemcpy(d_dx, dx.data(), 32 * 4, cudaMemcpyHostToDevice));
        RCK(cudaMemcpy(d_dy, dy.data(), 32 * 4, cudaMemcpyHostToDevice));
        RCK(cudaMemcpy(d_p1, p1s.data(), 32 * 4, cudaMemcpyHostToDevice));
        RCK(cudaMemcpy(d_p2, p2s.data(), 32 * 4, cudaMemcpyHostToDevice));
        return 0;
    }
    // sgm32.SGM32.compute_gpu's launches (sgm32.py:333-360) for one pair
    int run(const uint8_t* l, const uint8_t* r, float uniq, float lr_thr, float dmin, float* disp, float* conf)
    {
        const size_t n = (size_t)H * W;
        const dim3 b2(16, 16), g2((W + 15) / 16, (H + 15) / 16);
        census9<<<g2, b2>>>(l, L0, L1, H, W);
        census9<<<g2, b2>>>(r, R0, R1, H, W);
        const long nc = (long)n * 128;
        cost_volume<<<(unsigned)((nc + 255) / 256), 256>>>(L0, L1, R0, R1, C, H, W);
        RCK(cudaMemsetAsync(S, 0, n * 128 * 2));
        aggregate32<<<(unsigned)(((long)npaths * 32 + 127) / 128), 128>>>(C, (unsigned int*)S, d_sx, d_sy, d_sd, d_dx,
                                                                          d_dy, d_p1, d_p2, npaths, H, W);
        select_left<<<g2, b2>>>(S, disp, conf, H, W, uniq, dmin);
        select_right<<<g2, b2>>>(S, dr, H, W);
        lr_check<<<g2, b2>>>(disp, dr, conf, H, W, lr_thr);
        RCK(cudaGetLastError());
        return 0;
    }
};

// one pair in device memory -> disp / conf (device, H x W float32); S_out (device, may be null): the aggregated volume
extern "C" int xr_sgm(const uint8_t* l, const uint8_t* r, int H, int W, int p1, int p2, float uniq, float lr_thr,
                      float dmin, float* disp, float* conf, uint16_t* S_out)
{
    XrSgm g;
    int rc = g.init(H, W, p1, p2);
    if (rc) return rc;
    rc = g.run(l, r, uniq, lr_thr, dmin, disp, conf);
    if (rc) return rc;
    if (S_out) RCK(cudaMemcpy(S_out, g.S, (size_t)H * W * 128 * 2, cudaMemcpyDeviceToDevice));
    RCK(cudaDeviceSynchronize());
    return 0;
}

// the reference's kernels timed on F pairs already in device memory (frame f at l + f H W), buffers allocated once as
// SGM32 does: one untimed pass, then `passes` passes between two events on the default stream -> ms per frame
extern "C" int xr_sgm_time(const uint8_t* l, const uint8_t* r, int F, int H, int W, int p1, int p2, float uniq,
                           float lr_thr, float dmin, float* disp, float* conf, int passes, float* ms_per_frame)
{
    XrSgm g;
    int rc = g.init(H, W, p1, p2);
    if (rc) return rc;
    const size_t n = (size_t)H * W;
    for (int f = 0; f < F; ++f)
        if ((rc = g.run(l + f * n, r + f * n, uniq, lr_thr, dmin, disp, conf))) return rc;
    cudaEvent_t e0, e1;
    RCK(cudaEventCreate(&e0));
    RCK(cudaEventCreate(&e1));
    RCK(cudaDeviceSynchronize());
    RCK(cudaEventRecord(e0));
    for (int p = 0; p < passes; ++p)
        for (int f = 0; f < F; ++f)
            if ((rc = g.run(l + f * n, r + f * n, uniq, lr_thr, dmin, disp, conf))) return rc;
    RCK(cudaEventRecord(e1));
    RCK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    RCK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms_per_frame = ms / (float)(F * (passes > 0 ? passes : 1));
    return 0;
}
