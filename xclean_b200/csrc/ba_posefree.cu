// ba_posefree.cu -- the pose-free landmark block of the window solve on the device: window.posefree_cost and
// window.posefree_step (src/xclean/vio/window.py:683-765, with _pf_block_fast :550-680 and _cam_poses :109-122).
//
// Pose-free landmarks are seen only in their host keyframe's left image; their observation has no pose coupling, so
// each one is an independent 3x3 problem (the host observation and the inverse-depth prior).  The batched window
// solve carries them as ordinary landmarks; these kernels give the block's own cost, its damped step and, at lam = 0,
// final_linearisation's marginals (window.py:1003-1006).  One thread per landmark; the cost terms are then added in
// landmark order by one thread, as the reference adds them.  Built with --fmad=false: every product and sum is a
// separate round-to-nearest operation in the reference's order, so the results are the reference's bits.
#include <cmath>
#include <string>

#include "common.cuh"

extern void xcb_set_last_error(const std::string& m);

struct PfArgs {
    const double* Rwb;        // [P][3][3]
    const double* pwb;        // [P][3]
    double Rbc[9], pbc[3];
    int P, n;
    const double* lmp;        // [n][3]
    const i64* host;          // [n]
    const double* rmeas;      // [n]
    const double* ris;        // [n]
    const double* z;          // [n][2]
    double isg, fx, fy, cx, cy, huber_k, lam;
    int behind;
    double* terms;            // [n][2] cost terms (observation, prior), 0 where the reference adds nothing
    double* lmp_out;          // [n][3] or NULL
    double* Hinv_out;         // [n][3][3] (written where ok)
    u8* ok_out;               // [n]
};

// _cam_poses for one slot: Rwc = Rwb Rbc, pwc = pwb + Rwb pbc, sums from 0.0 (from pwb) in k order
__device__ __forceinline__ void pf_cam(const PfArgs& a, int s, double* R, double* p)
{
    const double* Rw = a.Rwb + 9 * (size_t)s;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += Rw[3 * i + k] * a.Rbc[3 * k + j];
            R[3 * i + j] = acc;
        }
        double acc = a.pwb[3 * (size_t)s + i];
#pragma unroll
        for (int k = 0; k < 3; ++k) acc += Rw[3 * i + k] * a.pbc[k];
        p[i] = acc;
    }
}

__device__ __forceinline__ double pf_huber_cost(double en, double k)
{
    return en <= k ? 0.5 * en * en : k * (en - 0.5 * k);
}

__global__ void __launch_bounds__(128) k_pf_block(PfArgs a)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= a.n) return;
    const int h = (int)a.host[l];
    double R[9], p[3];
    pf_cam(a, h, R, p);
    const double la = a.lmp[3 * l], lb = a.lmp[3 * l + 1], rho = a.lmp[3 * l + 2];
    const double z0 = a.z[2 * l], z1 = a.z[2 * l + 1], ris = a.ris[l], rmeas = a.rmeas[l];
    const double d0 = p[0] - p[0], d1 = p[1] - p[1], d2 = p[2] - p[2];
    const double Y0 = R[0] * la + R[1] * lb + R[2] + rho * d0;
    const double Y1 = R[3] * la + R[4] * lb + R[5] + rho * d1;
    const double Y2 = R[6] * la + R[7] * lb + R[8] + rho * d2;
    const double q0 = R[0] * Y0 + R[3] * Y1 + R[6] * Y2;
    const double q1 = R[1] * Y0 + R[4] * Y1 + R[7] * Y2;
    const double q2 = R[2] * Y0 + R[5] * Y1 + R[8] * Y2;
    // posefree_cost's terms (window.py:694-709): the observation as obs_residual + the whitening, then the prior
    // (a NaN depth skips the step's observation, q2 > 1e-9, but not the cost's, q2 <= 1e-9: as in the reference)
    double t_obs = 0.0, t_pri = 0.0, e0 = 0.0, e1 = 0.0, en = 0.0;
    const bool front = q2 > 1e-9;
    if (!(q2 <= 1e-9)) {
        e0 = a.fx * q0 / q2 + a.cx - z0;
        e1 = a.fy * q1 / q2 + a.cy - z1;
        double en2 = 0.0;
        e0 *= a.isg;
        en2 += e0 * e0;
        e1 *= a.isg;
        en2 += e1 * e1;
        en = sqrt(en2);
        t_obs = pf_huber_cost(en, a.huber_k);
    } else if (a.behind) {
        t_obs = 1e6;
    }
    double rr = 0.0;
    if (ris > 0.0) {
        rr = (rho - rmeas) * ris;
        t_pri = pf_huber_cost(fabs(rr), a.huber_k);
    }
    a.terms[2 * l] = t_obs;
    a.terms[2 * l + 1] = t_pri;
    if (!a.lmp_out) return;
    // _pf_block_fast (window.py:550-680) and posefree_step's update (:740-765)
    double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, bl[3] = {0, 0, 0};
    int nobs = 0;
    if (front) {
        const double w = en <= a.huber_k ? 1.0 : a.huber_k / en;
        const double iq = 1.0 / q2;
        const double D[6] = {a.fx * iq, 0.0, -a.fx * q0 * iq * iq, 0.0, a.fy * iq, -a.fy * q1 * iq * iq};
        // RcR = Rwc^T Rwc (_mtm)
        double RcR[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) RcR[3 * i + j] = R[i] * R[j] + R[3 + i] * R[3 + j] + R[6 + i] * R[6 + j];
        const double r0 = R[0] * d0 + R[3] * d1 + R[6] * d2;
        const double r1 = R[1] * d0 + R[4] * d1 + R[7] * d2;
        const double r2 = R[2] * d0 + R[5] * d1 + R[8] * d2;
        double J[2][3];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            J[r][0] = D[3 * r] * RcR[0] + D[3 * r + 1] * RcR[3] + D[3 * r + 2] * RcR[6];
            J[r][1] = D[3 * r] * RcR[1] + D[3 * r + 1] * RcR[4] + D[3 * r + 2] * RcR[7];
            J[r][2] = D[3 * r] * r0 + D[3 * r + 1] * r1 + D[3 * r + 2] * r2;
        }
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int j = 0; j < 3; ++j) J[r][j] *= a.isg;
        nobs = 1;
        const double e[2] = {e0, e1};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double acc = 0.0;
                acc += J[0][i] * J[0][j];
                acc += J[1][i] * J[1][j];
                H[3 * i + j] += w * acc;
            }
            double acc = 0.0;
            acc += J[0][i] * e[0];
            acc += J[1][i] * e[1];
            bl[i] += w * acc;
        }
    }
    if (ris > 0.0) {
        const double ar = fabs(rr), wp = ar <= a.huber_k ? 1.0 : a.huber_k / ar;
        H[8] += wp * ris * ris;
        bl[2] += wp * ris * rr;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) H[4 * i] += a.lam * H[4 * i] + 1e-12;
    const double det = H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6])
                       + H[2] * (H[3] * H[7] - H[4] * H[6]);
    const double tr = H[0] + H[4] + H[8];
    double* lo = a.lmp_out + 3 * (size_t)l;
    lo[0] = la;
    lo[1] = lb;
    lo[2] = rho;
    const bool ok = nobs != 0 && det > 1e-18 * tr * tr * tr && isfinite(det);
    a.ok_out[l] = ok;
    if (!ok) return;
    const double idet = 1.0 / det;
    double Hi[9];
    Hi[0] = (H[4] * H[8] - H[5] * H[7]) * idet;
    Hi[1] = (H[2] * H[7] - H[1] * H[8]) * idet;
    Hi[2] = (H[1] * H[5] - H[2] * H[4]) * idet;
    Hi[3] = (H[5] * H[6] - H[3] * H[8]) * idet;
    Hi[4] = (H[0] * H[8] - H[2] * H[6]) * idet;
    Hi[5] = (H[2] * H[3] - H[0] * H[5]) * idet;
    Hi[6] = (H[3] * H[7] - H[4] * H[6]) * idet;
    Hi[7] = (H[1] * H[6] - H[0] * H[7]) * idet;
    Hi[8] = (H[0] * H[4] - H[1] * H[3]) * idet;
#pragma unroll
    for (int i = 0; i < 9; ++i) a.Hinv_out[9 * (size_t)l + i] = Hi[i];
    double v[3], dd[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = bl[i] + 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double acc = 0.0;
        acc += Hi[3 * i] * v[0];
        acc += Hi[3 * i + 1] * v[1];
        acc += Hi[3 * i + 2] * v[2];
        dd[i] = -acc;
    }
    const double r = rho + dd[2];
    if (r > 1e-9 && isfinite(r)) {
        lo[0] = la + dd[0];
        lo[1] = lb + dd[1];
        lo[2] = r;
    }
}

// the terms in landmark order, observation before prior, from 0.0 (posefree_cost's `cost +=` sequence)
__global__ void k_pf_sum(const double* terms, int n, double* cost)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double c = 0.0;
    for (int i = 0; i < 2 * n; ++i) c += terms[i];
    *cost = c;
}

#define PCK(call, where)                                                                                    \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) {                                                                            \
            rc = XCB_ERR_CUDA;                                                                              \
            xcb_set_last_error(std::string(where) + ": " + cudaGetErrorString(e_));                         \
            goto done;                                                                                      \
        }                                                                                                   \
    } while (0)

extern "C" int xcb_ba_posefree_host(int P, const double* Rwb, const double* pwb, const double* Rbc, const double* pbc,
                                    int n, const double* lmp, const int64_t* host, const double* rmeas,
                                    const double* ris, const double* z, double isg, double fx, double fy, double cx,
                                    double cy, double huber_k, int behind, double lam, double* cost_out,
                                    double* lmp_out, double* Hinv_out, uint8_t* ok_out, void* stream)
{
    if (P < 1 || n < 0 || !Rwb || !pwb || !Rbc || !pbc) {
        xcb_set_last_error("ba_posefree_host: bad window");
        return XCB_ERR_ARG;
    }
    const bool want_step = lmp_out || Hinv_out || ok_out;
    if (want_step && !(lmp_out && Hinv_out && ok_out)) {
        xcb_set_last_error("ba_posefree_host: lmp_out, Hinv_out and ok_out go together");
        return XCB_ERR_ARG;
    }
    if (n > 0 && (!lmp || !host || !rmeas || !ris || !z)) {
        xcb_set_last_error("ba_posefree_host: null landmark argument");
        return XCB_ERR_ARG;
    }
    for (int l = 0; l < n; ++l)
        if (host[l] < 0 || host[l] >= P) {
            xcb_set_last_error("ba_posefree_host: a host slot is outside the window");
            return XCB_ERR_ARG;
        }
    if (n == 0) {
        if (cost_out) *cost_out = 0.0;
        return XCB_OK;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int rc = XCB_OK;
    // device block: Rwb 9P, pwb 3P, lmp 3n, host n, rmeas n, ris n, z 2n, terms 2n, cost 1, lmp_out 3n, Hinv 9n, ok n
    const size_t nd = 9 * (size_t)P + 3 * (size_t)P + 3 * (size_t)n + (size_t)n + 2 * (size_t)n + 2 * (size_t)n + 2 * (size_t)n + 1
                      + 3 * (size_t)n + 9 * (size_t)n + (size_t)n;
    double* d = nullptr;
    PfArgs a = {};
    double* o_terms = nullptr;
    cudaError_t e_put = cudaSuccess;
    PCK(cudaMallocAsync((void**)&d, nd * sizeof(double), st), "ba_posefree_host: device memory");
    {
        double* q = d;
        auto put = [&](const void* src, size_t count) -> double* {
            double* at = q;
            q += count;
            const cudaError_t e = cudaMemcpyAsync(at, src, count * sizeof(double), cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) e_put = e;
            return at;
        };
        a.Rwb = put(Rwb, 9 * (size_t)P);
        a.pwb = put(pwb, 3 * (size_t)P);
        a.lmp = put(lmp, 3 * (size_t)n);
        a.host = (const i64*)put(host, (size_t)n);
        a.rmeas = put(rmeas, (size_t)n);
        a.ris = put(ris, (size_t)n);
        a.z = put(z, 2 * (size_t)n);
        o_terms = q;
        q += 2 * (size_t)n + 1;
        a.terms = o_terms;
        if (want_step) {
            a.lmp_out = q;
            a.Hinv_out = q + 3 * (size_t)n;
            a.ok_out = (u8*)(q + 12 * (size_t)n);
        }
    }
    PCK(e_put, "ba_posefree_host: H2D");
    for (int i = 0; i < 9; ++i) a.Rbc[i] = Rbc[i];
    for (int i = 0; i < 3; ++i) a.pbc[i] = pbc[i];
    a.P = P;
    a.n = n;
    a.isg = isg;
    a.fx = fx;
    a.fy = fy;
    a.cx = cx;
    a.cy = cy;
    a.huber_k = huber_k;
    a.lam = lam;
    a.behind = behind != 0;
    if (want_step) PCK(cudaMemcpyAsync(a.Hinv_out, Hinv_out, 9 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st),
                       "ba_posefree_host: H2D");
    k_pf_block<<<(n + 127) / 128, 128, 0, st>>>(a);
    PCK(cudaGetLastError(), "ba_posefree_host: launch");
    if (cost_out) {
        k_pf_sum<<<1, 32, 0, st>>>(o_terms, n, o_terms + 2 * (size_t)n);
        PCK(cudaGetLastError(), "ba_posefree_host: launch");
        PCK(cudaMemcpyAsync(cost_out, o_terms + 2 * (size_t)n, sizeof(double), cudaMemcpyDeviceToHost, st),
            "ba_posefree_host: D2H");
    }
    if (want_step) {
        PCK(cudaMemcpyAsync(lmp_out, a.lmp_out, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st),
            "ba_posefree_host: D2H");
        PCK(cudaMemcpyAsync(Hinv_out, a.Hinv_out, 9 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st),
            "ba_posefree_host: D2H");
        PCK(cudaMemcpyAsync(ok_out, a.ok_out, (size_t)n, cudaMemcpyDeviceToHost, st), "ba_posefree_host: D2H");
    }
    PCK(cudaStreamSynchronize(st), "ba_posefree_host: kernels");
done:
    if (d) cudaFreeAsync(d, st);
    return rc;
}
