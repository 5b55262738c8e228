// front_api.cu -- the frontend's C ABI (include/xcb200.h): buffers, geometry, calibration, launch sequences, CUDA
// graph replay of the batched per-frame pipeline.
//
// The reference's GpuFront (src/xclean/front/gpu_front.py:1073-1420) allocates once per image size and issues one
// H2D, ~20 launches and one D2H per frame.  Here one handle serves batches of up to max_frames frames; every buffer is
// allocated at creation (nothing per call on the device path), and the batched pipeline's ~13 launches are captured
// once into a CUDA graph and replayed.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "front_kernels.h"

static thread_local std::string g_last_error;

extern "C" const char* xcb_last_error(void) { return g_last_error.c_str(); }
void xcb_set_last_error(const std::string& m) { g_last_error = m; }
extern "C" int xcb_version(void) { return 1; }

struct xcb_front {
    int W, H, cap, maxF, Hp, Wp;
    cudaStream_t stream;
    // xcb_front_pipeline_host_batches (made on first use): a copy stream and a second input buffer pair for the
    // uploads; a read-back stream and two device staging blocks that each batch's results are copied into, so the
    // read-back of batch b overlaps batch b+1's compute
    cudaStream_t cstream, rstream;
    cudaEvent_t ev_loaded[2], ev_free[2], ev_staged[2], ev_read[2];
    u8* d_in2[2];
    char* d_stage[2];
    std::string err;
    size_t dev_bytes;
    std::vector<void*> allocs;
    // calibration
    bool calibrated;
    int dy_vend, dx_vend, blur_vr, blur_vc;
    double Q;
    float* d_kf;
    int8_t* d_pat;
    // noise floor tree
    XcbNoiseTree tree;
    float* d_nodeval;
    double K;
    // detection geometry, per budget
    int geom_budget;
    XcbDetectGeom geom;
    int *d_ybeg, *d_xbeg, *d_coff;
    int ncell_max, gh_max, ncx_max, thr_max;
    // frame buffers (frame-major)
    u8 *d_left, *d_right;
    float *d_R, *d_Rs;
    int* d_anypos;
    double* d_floor;
    float* d_floorf;
    float* d_thr;
    u64 *d_raw, *d_sorted;
    int* d_ccount;
    int* d_counts_chain;   // [maxF + 1]: slot 0 = the previous call's last frame
    float* d_kp;
    u8* d_blur;
    u8* d_desc_chain;      // [maxF + 1][cap][32]
    int* d_rounds;
    double *d_d, *d_sig, *d_zn, *d_dy;
    u8* d_ok;
    int *d_b1, *d_b2, *d_bi, *d_ci;
    long long *d_m0, *d_m1;
    int* d_nmatch;
    unsigned int* d_err;
    // host-API point buffers (grow on demand)
    int pts_cap;
    double* d_kpd;
    long long *d_lo, *d_hi;
    double *d_pd, *d_psig, *d_pzn, *d_pdy;
    u8* d_pok;
    u8* d_pjobs;           // the stereo's job list for the host-API points (xcb_stereo_jobs_bytes(pts_cap))
    u8* d_jobs;            // the stereo's job list for the batched pipeline (max_frames x cap points)
    // Hamming host-API buffers
    int ham_capL, ham_capN;
    u8 *d_hA, *d_hB;
    int *d_hL, *d_hN;
    int *d_hb1, *d_hb2, *d_hbi, *d_hci, *d_hnm;
    long long *d_hi0, *d_hi1;
    // pinned staging
    u8* h_stage;
    size_t h_stage_bytes;
    // graph cache of the batched pipeline: one executable graph per (inputs, sizes, options, stream)
    struct GraphEntry {
        cudaGraphExec_t exec;
        const void *left, *right;
        int F, budget, half, dlo, dhi, match_prev;
        cudaStream_t stream;
        unsigned long long used;
        bool timed, fresh;
        cudaEvent_t ev[XCB_FRONT_STAGES + 1];   // stage boundaries, recorded inside the graph when timed
    };
    std::vector<GraphEntry> graphs;
    unsigned long long graph_clock;
    // launch shapes chosen by the tuner (xcb_front_set_tuning; 0 = the built-in default)
    int tune[XCB_TUNE_KNOBS];
    bool stage_timing;
    int last_launches;
};

static void drop_graph(xcb_front::GraphEntry& g)
{
    cudaGraphExecDestroy(g.exec);
    if (g.timed)
        for (int i = 0; i <= XCB_FRONT_STAGES; ++i) cudaEventDestroy(g.ev[i]);
}

static void drop_graphs(xcb_front* f)
{
    for (auto& g : f->graphs) drop_graph(g);
    f->graphs.clear();
}

// an event-record node of the graph being captured (External: replayed with the graph, readable by the host)
static inline cudaError_t mark(const cudaEvent_t* ev, int i, cudaStream_t st)
{
    return ev ? cudaEventRecordWithFlags(ev[i], st, cudaEventRecordExternal) : cudaSuccess;
}

static int fail(xcb_front* f, int code, const std::string& msg)
{
    if (f) f->err = msg;
    g_last_error = msg;
    return code;
}

static int cuda_fail(xcb_front* f, cudaError_t e, const char* where)
{
    return fail(f, XCB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call, where)                                \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return cuda_fail(f, e_, where); \
    } while (0)

template <typename T>
static cudaError_t dalloc(xcb_front* f, T** p, size_t count)
{
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e == cudaSuccess) { f->allocs.push_back((void*)*p); f->dev_bytes += bytes; }
    return e;
}

// numpy floor_divide on float64 (npy_divmod): the cell rows / columns of features.Frontend._detect
static double npy_floordiv(double a, double b)
{
    double mod = std::fmod(a, b);
    double div = (a - mod) / b;
    if (mod != 0.0) {
        if ((b < 0) != (mod < 0)) { mod += b; div -= 1.0; }
    }
    double fd;
    if (div != 0.0) {
        fd = std::floor(div);
        if (div - fd > 0.5) fd += 1.0;
    } else {
        fd = std::copysign(0.0, a / b);
    }
    return fd;
}

static double cell_size(int W, int H, int n) { double s = std::sqrt((double)W * H / (double)(n > 1 ? n : 1)); return s > 4.0 ? s : 4.0; }
static double min_dist(int W, int H, int n)
{
    double r = std::sqrt((double)W * H / (2.0 * std::sqrt(3.0) * (double)(n > 1 ? n : 1)));
    return r > 2.0 ? r : 2.0;
}

struct HostGeom {
    double s, r;
    int c, ncx, gh, ncell, gwc, ghc, max_px;
    std::vector<int> ybeg, xbeg, coff;
};

static HostGeom host_geom(int W, int H, int budget)
{
    HostGeom g;
    g.s = cell_size(W, H, budget);
    g.r = min_dist(W, H, budget);
    g.c = (int)std::nearbyint(g.s);
    if (g.c < 4) g.c = 4;
    g.ncx = (int)std::ceil(W / g.s);
    int maxcy = (int)npy_floordiv((double)(H - 1), g.s);
    g.gh = maxcy + 1;
    g.ybeg.assign(g.gh + 1, H);
    g.xbeg.assign(g.ncx + 1, W);
    for (int y = H - 1; y >= 0; --y) g.ybeg[(int)npy_floordiv((double)y, g.s)] = y;
    for (int x = W - 1; x >= 0; --x) {
        int cx = (int)npy_floordiv((double)x, g.s);
        if (cx < g.ncx) g.xbeg[cx] = x;
    }
    // empty trailing columns/rows keep the next start (monotone)
    for (int k = g.gh - 1; k >= 0; --k) if (g.ybeg[k] > g.ybeg[k + 1]) g.ybeg[k] = g.ybeg[k + 1];
    for (int k = g.ncx - 1; k >= 0; --k) if (g.xbeg[k] > g.xbeg[k + 1]) g.xbeg[k] = g.xbeg[k + 1];
    g.ncell = g.ncx * g.gh;
    g.coff.assign(g.ncell + 1, 0);
    g.max_px = 0;
    for (int c = 0; c < g.ncell; ++c) {
        int cy = c / g.ncx, cx = c % g.ncx;
        int px = (g.ybeg[cy + 1] - g.ybeg[cy]) * (g.xbeg[cx + 1] - g.xbeg[cx]);
        g.coff[c + 1] = g.coff[c] + px;
        if (px > g.max_px) g.max_px = px;
    }
    g.gwc = (W + g.c - 1) / g.c;
    g.ghc = (H + g.c - 1) / g.c;
    return g;
}

// numpy's pairwise float32 sum over n elements as leaves (<= 128 elements) and a combine tree by height
struct TreeBuild {
    std::vector<long long> ls;
    std::vector<int> ll;
    struct Inner { int a, b, h; };   // children: >= 0 leaf id, < 0 -> inner id ~x
    std::vector<Inner> inner;
    int rec(long long st, long long m, int* h)
    {
        if (m <= 128) {
            ls.push_back(st);
            ll.push_back((int)m);
            *h = 0;
            return (int)ls.size() - 1;
        }
        long long n2 = m / 2;
        n2 -= n2 % 8;
        int ha, hb;
        int a = rec(st, n2, &ha);
        int b = rec(st + n2, m - n2, &hb);
        int hh = (ha > hb ? ha : hb) + 1;
        inner.push_back({a, b, hh});
        *h = hh;
        return ~((int)inner.size() - 1);
    }
};

static int build_tree(xcb_front* f)
{
    long long n = (long long)(f->H - 2) * (f->W - 2);
    TreeBuild tb;
    int hroot;
    int root = tb.rec(0, n, &hroot);
    int nl = (int)tb.ls.size(), ni = (int)tb.inner.size();
    // node ids: leaves 0..nl-1, then inner nodes ordered by (height, creation)
    std::vector<int> order(ni);
    for (int i = 0; i < ni; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return tb.inner[x].h < tb.inner[y].h; });
    std::vector<int> nid(ni);
    for (int p = 0; p < ni; ++p) nid[order[p]] = nl + p;
    auto ref = [&](int x) { return x >= 0 ? x : nid[~x]; };
    int nnode = nl + ni;
    std::vector<int> left(nnode, 0), right(nnode, 0);
    int maxh = 0;
    for (int i = 0; i < ni; ++i) {
        left[nid[i]] = ref(tb.inner[i].a);
        right[nid[i]] = ref(tb.inner[i].b);
        if (tb.inner[i].h > maxh) maxh = tb.inner[i].h;
    }
    std::vector<int> lvl(1, nl);
    for (int h = 1; h <= maxh; ++h) {
        int cnt = 0;
        for (int i = 0; i < ni; ++i) cnt += tb.inner[i].h == h;
        lvl.push_back(lvl.back() + cnt);
    }
    long long* d_ls;
    int *d_ll, *d_left, *d_right, *d_lvl;
    CK(dalloc(f, &d_ls, nl), "alloc tree");
    CK(dalloc(f, &d_ll, nl), "alloc tree");
    CK(dalloc(f, &d_left, nnode), "alloc tree");
    CK(dalloc(f, &d_right, nnode), "alloc tree");
    CK(dalloc(f, &d_lvl, lvl.size()), "alloc tree");
    CK(cudaMemcpy(d_ls, tb.ls.data(), nl * sizeof(long long), cudaMemcpyHostToDevice), "upload tree");
    CK(cudaMemcpy(d_ll, tb.ll.data(), nl * sizeof(int), cudaMemcpyHostToDevice), "upload tree");
    CK(cudaMemcpy(d_left, left.data(), nnode * sizeof(int), cudaMemcpyHostToDevice), "upload tree");
    CK(cudaMemcpy(d_right, right.data(), nnode * sizeof(int), cudaMemcpyHostToDevice), "upload tree");
    CK(cudaMemcpy(d_lvl, lvl.data(), lvl.size() * sizeof(int), cudaMemcpyHostToDevice), "upload tree");
    f->tree.nleaf = nl;
    f->tree.nnode = nnode;
    f->tree.nlvl = (int)lvl.size() - 1;
    f->tree.root = ref(root);
    f->tree.lstart = d_ls;
    f->tree.llen = d_ll;
    f->tree.left = d_left;
    f->tree.right = d_right;
    f->tree.lvl = d_lvl;
    f->K = std::sqrt(M_PI / 2.0) / (6.0 * (f->W - 2) * (f->H - 2));
    return XCB_OK;
}

static int set_geometry(xcb_front* f, int budget)
{
    if (f->geom_budget == budget) return XCB_OK;
    HostGeom g = host_geom(f->W, f->H, budget);
    if (g.ncell > f->ncell_max || g.gh + 1 > f->gh_max + 1 || g.ncx + 1 > f->ncx_max + 1 || g.gwc * g.ghc > f->thr_max)
        return fail(f, XCB_ERR_CAPACITY, "detect: budget " + std::to_string(budget) + " needs more cells than the front was created for");
    if (xcb_greedy_smem(g.ncell) > (size_t)xcb_greedy_smem_limit())
        return fail(f, XCB_ERR_CAPACITY, "detect: " + std::to_string(g.ncell) + " cells exceed the greedy kernel's shared memory");
    CK(cudaDeviceSynchronize(), "geometry sync");
    CK(cudaMemcpy(f->d_ybeg, g.ybeg.data(), g.ybeg.size() * sizeof(int), cudaMemcpyHostToDevice), "upload geometry");
    CK(cudaMemcpy(f->d_xbeg, g.xbeg.data(), g.xbeg.size() * sizeof(int), cudaMemcpyHostToDevice), "upload geometry");
    CK(cudaMemcpy(f->d_coff, g.coff.data(), g.coff.size() * sizeof(int), cudaMemcpyHostToDevice), "upload geometry");
    f->geom.s = g.s;
    f->geom.r2 = g.r * g.r;
    f->geom.ncx = g.ncx;
    f->geom.gh = g.gh;
    f->geom.ncell = g.ncell;
    f->geom.c = g.c;
    f->geom.gwc = g.gwc;
    f->geom.ghc = g.ghc;
    f->geom.border = 21 / 2 + 1;
    f->geom.ybeg = f->d_ybeg;
    f->geom.xbeg = f->d_xbeg;
    f->geom.coff = f->d_coff;
    f->geom.max_cell_px = g.max_px;
    f->geom_budget = budget;
    drop_graphs(f);
    return XCB_OK;
}

extern "C" int xcb_front_create(int width, int height, int cap, int max_frames, xcb_front** out)
{
    if (!out) return fail(nullptr, XCB_ERR_ARG, "create: out is NULL");
    *out = nullptr;
    if (width < 48 || height < 48 || width > 8192 || height > 0xFFFF || cap < 1 || cap > 65536 || max_frames < 1)
        return fail(nullptr, XCB_ERR_ARG, "create: bad size (48 <= width <= 8192, 48 <= height <= 65535)");
    xcb_front* f = new xcb_front();
    f->W = width; f->H = height; f->cap = cap; f->maxF = max_frames;
    f->Hp = height + 64; f->Wp = width + 64;
    f->dev_bytes = 0;
    f->calibrated = false;
    f->geom_budget = -1;
    f->graph_clock = 0;
    f->stage_timing = false;
    f->pts_cap = 0;
    f->ham_capL = f->ham_capN = 0;
    f->h_stage = nullptr;
    f->h_stage_bytes = 0;
    f->last_launches = 0;
    int rc = XCB_OK;
    auto bail = [&](int code) { xcb_front_destroy(f); return code; };
    cudaError_t e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { rc = cuda_fail(f, e, "stream"); g_last_error = f->err; return bail(rc); }
    e = xcb_greedy_init_attrs();
    if (e == cudaSuccess) e = xcb_stereo_init_attrs();
    if (e != cudaSuccess) { rc = cuda_fail(f, e, "kernel attributes"); return bail(rc); }
    const size_t W = width, H = height, F = max_frames, npx = W * H;
    // the largest cell grid: the smallest cell, at budget = cap
    HostGeom gmax = host_geom(width, height, cap);
    f->ncell_max = gmax.ncell;
    f->gh_max = gmax.gh;
    f->ncx_max = gmax.ncx;
    f->thr_max = gmax.gwc * gmax.ghc;
#define AL(ptr, n)                                                                  \
    do {                                                                            \
        cudaError_t e_ = dalloc(f, &(ptr), (size_t)(n));                            \
        if (e_ != cudaSuccess) { cuda_fail(f, e_, "cudaMalloc"); g_last_error = f->err; return bail(XCB_ERR_CUDA); } \
    } while (0)
    AL(f->d_kf, 8);
    AL(f->d_pat, 1024);
    AL(f->d_ybeg, f->gh_max + 2);
    AL(f->d_xbeg, f->ncx_max + 2);
    AL(f->d_coff, f->ncell_max + 1);
    AL(f->d_left, F * npx);
    AL(f->d_right, F * npx);
    AL(f->d_R, F * npx);
    AL(f->d_Rs, F * npx);
    AL(f->d_anypos, F);
    AL(f->d_floor, F);
    AL(f->d_floorf, F);
    AL(f->d_thr, F * f->thr_max);
    AL(f->d_raw, F * npx);
    AL(f->d_sorted, F * npx);
    AL(f->d_ccount, F * f->ncell_max);
    AL(f->d_counts_chain, F + 1);
    AL(f->d_kp, F * cap * 2);
    AL(f->d_blur, F * (size_t)f->Hp * f->Wp);
    AL(f->d_desc_chain, (F + 1) * cap * 32);
    AL(f->d_rounds, F);
    AL(f->d_d, F * cap);
    AL(f->d_sig, F * cap);
    AL(f->d_zn, F * cap);
    AL(f->d_dy, F * cap);
    AL(f->d_ok, F * cap);
    AL(f->d_b1, F * cap);
    AL(f->d_b2, F * cap);
    AL(f->d_bi, F * cap);
    AL(f->d_ci, F * cap);
    AL(f->d_m0, F * cap);
    AL(f->d_m1, F * cap);
    AL(f->d_nmatch, F);
    AL(f->d_err, 1);
    AL(f->d_jobs, xcb_stereo_jobs_bytes((long long)F * cap));
#undef AL
    cudaMemset(f->d_counts_chain, 0, (F + 1) * sizeof(int));
    cudaMemset(f->d_err, 0, sizeof(unsigned int));
    rc = build_tree(f);
    if (rc != XCB_OK) { g_last_error = f->err; return bail(rc); }
    e = dalloc(f, &f->d_nodeval, F * (size_t)f->tree.nnode);
    if (e != cudaSuccess) { cuda_fail(f, e, "cudaMalloc"); return bail(XCB_ERR_CUDA); }
    size_t stage = 2 * F * npx + 64;
    e = cudaMallocHost((void**)&f->h_stage, stage);
    if (e != cudaSuccess) { cuda_fail(f, e, "cudaMallocHost"); return bail(XCB_ERR_CUDA); }
    f->h_stage_bytes = stage;
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { cuda_fail(f, e, "create sync"); return bail(XCB_ERR_CUDA); }
    *out = f;
    return XCB_OK;
}

extern "C" void xcb_front_destroy(xcb_front* f)
{
    if (!f) return;
    if (f->stream) cudaStreamSynchronize(f->stream);
    drop_graphs(f);
    for (void* p : f->allocs) cudaFree(p);
    if (f->h_stage) cudaFreeHost(f->h_stage);
    if (f->cstream) {
        cudaStreamSynchronize(f->cstream);
        cudaStreamSynchronize(f->rstream);
        for (int k = 0; k < 2; ++k) {
            cudaEventDestroy(f->ev_loaded[k]);
            cudaEventDestroy(f->ev_free[k]);
            cudaEventDestroy(f->ev_staged[k]);
            cudaEventDestroy(f->ev_read[k]);
        }
        cudaStreamDestroy(f->cstream);
        cudaStreamDestroy(f->rstream);
    }
    if (f->stream) cudaStreamDestroy(f->stream);
    delete f;
}

extern "C" const char* xcb_front_last_error(const xcb_front* f) { return f ? f->err.c_str() : g_last_error.c_str(); }
extern "C" size_t xcb_front_device_bytes(const xcb_front* f) { return f ? f->dev_bytes : 0; }
extern "C" int xcb_front_last_launches(const xcb_front* f) { return f ? f->last_launches : 0; }

extern "C" int xcb_front_set_calibration(xcb_front* f, int dy_vend, int dx_vend, int blur_vr, int blur_vc,
                                         const float* kf7, const int8_t* pattern, double noise_q99)
{
    if (!f || !kf7 || !pattern) return fail(f, XCB_ERR_ARG, "set_calibration: null argument");
    for (int i = 0; i < 1024; ++i)
        if (pattern[i] < -15 || pattern[i] > 15) return fail(f, XCB_ERR_ARG, "set_calibration: ORB pattern out of the 31-px patch");
    CK(cudaDeviceSynchronize(), "calibration sync");
    CK(cudaMemcpy(f->d_kf, kf7, 7 * sizeof(float), cudaMemcpyHostToDevice), "upload kf");
    CK(cudaMemcpy(f->d_pat, pattern, 1024, cudaMemcpyHostToDevice), "upload pattern");
    f->dy_vend = dy_vend; f->dx_vend = dx_vend; f->blur_vr = blur_vr; f->blur_vc = blur_vc;
    f->Q = noise_q99;
    f->calibrated = true;
    drop_graphs(f);
    return XCB_OK;
}

static int check_dev_err(xcb_front* f)
{
    unsigned int e = 0;
    CK(cudaMemcpy(&e, f->d_err, sizeof(e), cudaMemcpyDeviceToHost), "read error word");
    if (e) {
        cudaMemset(f->d_err, 0, sizeof(unsigned int));
        std::string m = "device error word 0x" + std::to_string(e);
        if (e & XCB_DEVERR_GREEDY_ROUNDS) m += " (greedy selection did not converge within its round bound)";
        return fail(f, XCB_ERR_DEVICE, m);
    }
    return XCB_OK;
}

static int upload(xcb_front* f, u8* dst, const uint8_t* src, size_t bytes)
{
    if (bytes > f->h_stage_bytes) return fail(f, XCB_ERR_CAPACITY, "upload larger than the staging buffer");
    std::memcpy(f->h_stage, src, bytes);
    CK(cudaMemcpyAsync(dst, f->h_stage, bytes, cudaMemcpyHostToDevice, f->stream), "H2D");
    CK(cudaStreamSynchronize(f->stream), "H2D sync");
    return XCB_OK;
}

extern "C" int xcb_front_response_host(xcb_front* f, const uint8_t* gray, int dy_vend, int dx_vend, float* R)
{
    if (!f || !gray || !R) return fail(f, XCB_ERR_ARG, "response: null argument");
    size_t npx = (size_t)f->W * f->H;
    int rc = upload(f, f->d_left, gray, npx);
    if (rc) return rc;
    CK(cudaMemsetAsync(f->d_anypos, 0, sizeof(int), f->stream), "memset");
    CK(xcb_launch_response(f->d_left, 1, f->H, f->W, dy_vend, dx_vend, f->d_R, f->d_anypos, f->stream), "response");
    CK(cudaMemcpyAsync(R, f->d_R, npx * sizeof(float), cudaMemcpyDeviceToHost, f->stream), "D2H");
    CK(cudaStreamSynchronize(f->stream), "response sync");
    return XCB_OK;
}

extern "C" int xcb_front_noise_floor_host(xcb_front* f, const uint8_t* gray, double* floor_out)
{
    if (!f || !gray || !floor_out) return fail(f, XCB_ERR_ARG, "noise_floor: null argument");
    if (!f->calibrated) return fail(f, XCB_ERR_NOT_CALIBRATED, "noise_floor: front not calibrated");
    int rc = upload(f, f->d_left, gray, (size_t)f->W * f->H);
    if (rc) return rc;
    CK(xcb_launch_noise(f->d_left, 1, f->H, f->W, f->tree, f->d_nodeval, f->K, f->Q, f->d_floor, f->d_floorf, f->stream), "noise");
    CK(cudaMemcpyAsync(floor_out, f->d_floor, sizeof(double), cudaMemcpyDeviceToHost, f->stream), "D2H");
    CK(cudaStreamSynchronize(f->stream), "noise sync");
    return XCB_OK;
}

extern "C" int xcb_front_blur_host(xcb_front* f, const uint8_t* gray, int blur_vr, int blur_vc, uint8_t* out)
{
    if (!f || !gray || !out) return fail(f, XCB_ERR_ARG, "blur: null argument");
    if (!f->calibrated) return fail(f, XCB_ERR_NOT_CALIBRATED, "blur: the Gaussian taps are set by the calibration");
    int rc = upload(f, f->d_left, gray, (size_t)f->W * f->H);
    if (rc) return rc;
    CK(xcb_launch_blur(f->d_left, 1, f->H, f->W, f->d_kf, blur_vr, blur_vc, f->d_blur, f->stream), "blur");
    CK(cudaMemcpyAsync(out, f->d_blur, (size_t)f->Hp * f->Wp, cudaMemcpyDeviceToHost, f->stream), "D2H");
    CK(cudaStreamSynchronize(f->stream), "blur sync");
    return XCB_OK;
}

// detection + description of F frames already in d_left (results in slots 1..F of the chains); -> launches issued
static int enqueue_detect(xcb_front* f, const u8* left, int F, int budget, cudaStream_t st, int* nl,
                          const cudaEvent_t* ev = nullptr)
{
    const int H = f->H, W = f->W;
    int* counts = f->d_counts_chain + 1;
    u8* desc = f->d_desc_chain + (size_t)f->cap * 32;
    CK(cudaMemsetAsync(f->d_anypos, 0, F * sizeof(int), st), "memset");
    CK(mark(ev, 0, st), "event");
    CK(xcb_launch_response(left, F, H, W, f->dy_vend, f->dx_vend, f->d_R, f->d_anypos, st), "response");
    CK(mark(ev, 1, st), "event");
    CK(xcb_launch_noise(left, F, H, W, f->tree, f->d_nodeval, f->K, f->Q, f->d_floor, f->d_floorf, st), "noise");
    CK(mark(ev, 2, st), "event");
    CK(xcb_launch_candidates(f->d_R, F, H, W, f->geom, f->d_floorf, f->d_anypos, f->d_thr, f->d_raw, f->d_sorted,
                             f->d_ccount, st), "candidates");
    CK(mark(ev, 3, st), "event");
    CK(xcb_launch_greedy(f->d_R, F, H, W, f->geom, f->d_sorted, f->d_ccount, budget, f->cap, f->d_kp, counts,
                         f->d_rounds, f->d_err, st), "greedy");
    CK(mark(ev, 4, st), "event");
    CK(xcb_launch_blur(left, F, H, W, f->d_kf, f->blur_vr, f->blur_vc, f->d_blur, st), "blur");
    CK(xcb_launch_orb(f->d_blur, F, f->Hp, f->Wp, f->d_kp, counts, f->cap, f->d_pat, desc, st), "orb");
    CK(mark(ev, 5, st), "event");
    *nl += 9;
    return XCB_OK;
}

extern "C" int xcb_front_detect_host(xcb_front* f, const uint8_t* gray, int nframes, int budget, int32_t* counts,
                                     float* kp, uint8_t* desc, double* floor_out, int32_t* anypos)
{
    if (!f || !gray || !counts || !kp || !desc) return fail(f, XCB_ERR_ARG, "detect: null argument");
    if (!f->calibrated) return fail(f, XCB_ERR_NOT_CALIBRATED, "detect: front not calibrated");
    if (nframes < 1 || nframes > f->maxF) return fail(f, XCB_ERR_CAPACITY, "detect: frame count out of range");
    if (budget < 1 || budget > f->cap) return fail(f, XCB_ERR_CAPACITY, "detect: budget " + std::to_string(budget) + " > cap " + std::to_string(f->cap));
    int rc = set_geometry(f, budget);
    if (rc) return rc;
    size_t npx = (size_t)f->W * f->H;
    rc = upload(f, f->d_left, gray, npx * nframes);
    if (rc) return rc;
    int nl = 0;
    rc = enqueue_detect(f, f->d_left, nframes, budget, f->stream, &nl);
    if (rc) return rc;
    const size_t F = nframes, cap = f->cap;
    CK(cudaMemcpyAsync(counts, f->d_counts_chain + 1, F * sizeof(int), cudaMemcpyDeviceToHost, f->stream), "D2H");
    CK(cudaMemcpyAsync(kp, f->d_kp, F * cap * 2 * sizeof(float), cudaMemcpyDeviceToHost, f->stream), "D2H");
    CK(cudaMemcpyAsync(desc, f->d_desc_chain + cap * 32, F * cap * 32, cudaMemcpyDeviceToHost, f->stream), "D2H");
    if (floor_out) CK(cudaMemcpyAsync(floor_out, f->d_floor, F * sizeof(double), cudaMemcpyDeviceToHost, f->stream), "D2H");
    if (anypos) CK(cudaMemcpyAsync(anypos, f->d_anypos, F * sizeof(int), cudaMemcpyDeviceToHost, f->stream), "D2H");
    CK(cudaStreamSynchronize(f->stream), "detect sync");
    f->last_launches = nl;
    return check_dev_err(f);
}

extern "C" int xcb_front_describe_host(xcb_front* f, const uint8_t* gray, const float* kp, int n, uint8_t* desc)
{
    if (!f || !gray || (!kp && n) || (!desc && n)) return fail(f, XCB_ERR_ARG, "describe: null argument");
    if (!f->calibrated) return fail(f, XCB_ERR_NOT_CALIBRATED, "describe: front not calibrated");
    if (n < 0 || n > f->cap) return fail(f, XCB_ERR_CAPACITY, "describe: more keypoints than cap");
    if (n == 0) return XCB_OK;
    // the 31-px test pattern around rint(kp + 32) must stay inside the padded image
    for (int i = 0; i < n; ++i) {
        float x = kp[2 * i], y = kp[2 * i + 1];
        if (!(x >= -16.0f && x <= f->W + 15.0f && y >= -16.0f && y <= f->H + 15.0f))
            return fail(f, XCB_ERR_ARG, "describe: keypoint " + std::to_string(i) + " outside the padded image");
    }
    int rc = upload(f, f->d_left, gray, (size_t)f->W * f->H);
    if (rc) return rc;
    int* counts = f->d_counts_chain + 1;
    u8* d_desc = f->d_desc_chain + (size_t)f->cap * 32;
    CK(cudaMemcpyAsync(f->d_kp, kp, (size_t)n * 2 * sizeof(float), cudaMemcpyHostToDevice, f->stream), "H2D");
    CK(cudaMemcpyAsync(counts, &n, sizeof(int), cudaMemcpyHostToDevice, f->stream), "H2D");
    CK(xcb_launch_blur(f->d_left, 1, f->H, f->W, f->d_kf, f->blur_vr, f->blur_vc, f->d_blur, f->stream), "blur");
    CK(xcb_launch_orb(f->d_blur, 1, f->Hp, f->Wp, f->d_kp, counts, f->cap, f->d_pat, d_desc, f->stream), "orb");
    CK(cudaMemcpyAsync(desc, d_desc, (size_t)n * 32, cudaMemcpyDeviceToHost, f->stream), "D2H");
    CK(cudaStreamSynchronize(f->stream), "describe sync");
    return XCB_OK;
}

static int grow_points(xcb_front* f, int n)
{
    if (n <= f->pts_cap) return XCB_OK;
    int c = n < 4096 ? 4096 : n;
    CK(dalloc(f, &f->d_kpd, (size_t)c * 2), "alloc points");
    CK(dalloc(f, &f->d_lo, (size_t)c), "alloc points");
    CK(dalloc(f, &f->d_hi, (size_t)c), "alloc points");
    CK(dalloc(f, &f->d_pd, (size_t)c), "alloc points");
    CK(dalloc(f, &f->d_psig, (size_t)c), "alloc points");
    CK(dalloc(f, &f->d_pzn, (size_t)c), "alloc points");
    CK(dalloc(f, &f->d_pdy, (size_t)c), "alloc points");
    CK(dalloc(f, &f->d_pok, (size_t)c), "alloc points");
    CK(dalloc(f, &f->d_pjobs, xcb_stereo_jobs_bytes(c)), "alloc points");
    f->pts_cap = c;
    return XCB_OK;
}

extern "C" int xcb_front_stereo_host(xcb_front* f, const uint8_t* left, const uint8_t* right, const double* kp,
                                     const int64_t* dlo, const int64_t* dhi, int n, double dy, int band, int half,
                                     double* d, double* sig, uint8_t* ok, double* zn, double* ody)
{
    if (!f || !left || !right) return fail(f, XCB_ERR_ARG, "stereo: null argument");
    if (n < 0) return fail(f, XCB_ERR_ARG, "stereo: negative point count");
    if (half < 3 || half > 5) return fail(f, XCB_ERR_ARG, "stereo: half must be 3, 4 or 5");
    if (band < 0 || band > 16) return fail(f, XCB_ERR_ARG, "stereo: band must be in [0, 16]");
    if (n == 0) return XCB_OK;
    if (!kp || !dlo || !dhi || !d || !sig || !ok || !zn || !ody) return fail(f, XCB_ERR_ARG, "stereo: null argument");
    for (int i = 0; i < 2 * n; ++i)
        if (!std::isfinite(kp[i]) || std::fabs(kp[i]) > 1e9)
            return fail(f, XCB_ERR_ARG, "stereo: non-finite or huge keypoint coordinate (sanitise on the host first)");
    int rc = grow_points(f, n);
    if (rc) return rc;
    size_t npx = (size_t)f->W * f->H;
    rc = upload(f, f->d_left, left, npx);
    if (rc) return rc;
    rc = upload(f, f->d_right, right, npx);
    if (rc) return rc;
    cudaStream_t st = f->stream;
    CK(cudaMemcpyAsync(f->d_kpd, kp, (size_t)n * 2 * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
    CK(cudaMemcpyAsync(f->d_lo, dlo, (size_t)n * sizeof(long long), cudaMemcpyHostToDevice, st), "H2D");
    CK(cudaMemcpyAsync(f->d_hi, dhi, (size_t)n * sizeof(long long), cudaMemcpyHostToDevice, st), "H2D");
    const float* Rs = nullptr;
    if (dy != 0.0) {
        CK(xcb_launch_shift(f->d_right, 1, f->H, f->W, dy, f->d_Rs, st), "shift");
        Rs = f->d_Rs;
    }
    CK(xcb_launch_stereo(f->d_left, f->d_right, Rs, 1, f->H, f->W, f->d_kpd, (const long long*)f->d_lo,
                         (const long long*)f->d_hi, n, nullptr, nullptr, 0, 0, 0, band, half, f->d_pd, f->d_psig,
                         f->d_pok, f->d_pzn, f->d_pdy, f->d_err, f->d_pjobs, f->tune[XCB_TUNE_STEREO_WARPS],
                         f->tune[XCB_TUNE_STEREO_GROUP], st), "stereo");
    CK(cudaMemcpyAsync(d, f->d_pd, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaMemcpyAsync(sig, f->d_psig, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaMemcpyAsync(ok, f->d_pok, (size_t)n, cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaMemcpyAsync(zn, f->d_pzn, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaMemcpyAsync(ody, f->d_pdy, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaStreamSynchronize(st), "stereo sync");
    return check_dev_err(f);
}

static int grow_ham(xcb_front* f, int L, int N)
{
    if (L > f->ham_capL) {
        int c = L < 4096 ? 4096 : L;
        CK(dalloc(f, &f->d_hA, (size_t)c * 32), "alloc hamming");
        CK(dalloc(f, &f->d_hb1, (size_t)c), "alloc hamming");
        CK(dalloc(f, &f->d_hb2, (size_t)c), "alloc hamming");
        CK(dalloc(f, &f->d_hbi, (size_t)c), "alloc hamming");
        CK(dalloc(f, &f->d_hi0, (size_t)c), "alloc hamming");
        CK(dalloc(f, &f->d_hi1, (size_t)c), "alloc hamming");
        if (!f->d_hL) {
            CK(dalloc(f, &f->d_hL, 2), "alloc hamming");
            CK(dalloc(f, &f->d_hN, 2), "alloc hamming");
            CK(dalloc(f, &f->d_hnm, 2), "alloc hamming");
        }
        f->ham_capL = c;
    }
    if (N > f->ham_capN) {
        int c = N < 4096 ? 4096 : N;
        CK(dalloc(f, &f->d_hB, (size_t)c * 32), "alloc hamming");
        CK(dalloc(f, &f->d_hci, (size_t)c), "alloc hamming");
        f->ham_capN = c;
    }
    return XCB_OK;
}

static int ham_upload(xcb_front* f, const uint8_t* A, int L, const uint8_t* B, int N, XcbHamPairs* p)
{
    int rc = grow_ham(f, L > 0 ? L : 1, N > 0 ? N : 1);
    if (rc) return rc;
    cudaStream_t st = f->stream;
    if (L) CK(cudaMemcpyAsync(f->d_hA, A, (size_t)L * 32, cudaMemcpyHostToDevice, st), "H2D");
    if (N) CK(cudaMemcpyAsync(f->d_hB, B, (size_t)N * 32, cudaMemcpyHostToDevice, st), "H2D");
    CK(cudaMemcpyAsync(f->d_hL, &L, sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    CK(cudaMemcpyAsync(f->d_hN, &N, sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    p->A = f->d_hA; p->B = f->d_hB; p->strideA = 0; p->strideB = 0;
    p->LA = f->d_hL; p->NB = f->d_hN; p->npair = 1; p->maxL = L; p->maxN = N;
    return XCB_OK;
}

extern "C" int xcb_front_hamming_host(xcb_front* f, const uint8_t* A, int L, const uint8_t* B, int N, int32_t* b1,
                                      int32_t* b2, int32_t* bi, int32_t* ci)
{
    if (!f || L < 0 || N < 0) return fail(f, XCB_ERR_ARG, "hamming: bad argument");
    if ((L && (!A || !b1 || !b2 || !bi)) || (N && (!B || !ci))) return fail(f, XCB_ERR_ARG, "hamming: null argument");
    if (L == 0 && N == 0) return XCB_OK;
    XcbHamPairs p;
    int rc = ham_upload(f, A, L, B, N, &p);
    if (rc) return rc;
    cudaStream_t st = f->stream;
    CK(xcb_launch_hamming(p, f->d_hb1, f->d_hb2, f->d_hbi, f->d_hci, st), "hamming");
    if (L) {
        CK(cudaMemcpyAsync(b1, f->d_hb1, (size_t)L * 4, cudaMemcpyDeviceToHost, st), "D2H");
        CK(cudaMemcpyAsync(b2, f->d_hb2, (size_t)L * 4, cudaMemcpyDeviceToHost, st), "D2H");
        CK(cudaMemcpyAsync(bi, f->d_hbi, (size_t)L * 4, cudaMemcpyDeviceToHost, st), "D2H");
    }
    if (N) CK(cudaMemcpyAsync(ci, f->d_hci, (size_t)N * 4, cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaStreamSynchronize(st), "hamming sync");
    for (int j = 0; j < N; ++j) {          // device: (distance << 16 | query) column minima, all ones if no query
        const uint32_t v = (uint32_t)ci[j];
        ci[j] = v == 0xffffffffu ? -1 : (int32_t)(v & 0xffffu);
    }
    return XCB_OK;
}

extern "C" int xcb_front_match_host(xcb_front* f, const uint8_t* A, int L, const uint8_t* B, int N, int ham_max,
                                    double ratio, int64_t* i0, int64_t* i1, int32_t* nmatch)
{
    if (!f || L < 0 || N < 0 || !nmatch) return fail(f, XCB_ERR_ARG, "match: bad argument");
    *nmatch = 0;
    if (L < 2 || N < 2) return XCB_OK;
    if (!A || !B || !i0 || !i1) return fail(f, XCB_ERR_ARG, "match: null argument");
    XcbHamPairs p;
    int rc = ham_upload(f, A, L, B, N, &p);
    if (rc) return rc;
    cudaStream_t st = f->stream;
    CK(xcb_launch_hamming(p, f->d_hb1, f->d_hb2, f->d_hbi, f->d_hci, st), "hamming");
    CK(xcb_launch_match_epilogue(p, f->d_hb1, f->d_hb2, f->d_hbi, f->d_hci, ham_max, ratio, f->d_hi0, f->d_hi1, 0,
                                 f->d_hnm, st), "match");
    int m = 0;
    CK(cudaMemcpyAsync(&m, f->d_hnm, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaStreamSynchronize(st), "match sync");
    if (m) {
        CK(cudaMemcpyAsync(i0, f->d_hi0, (size_t)m * 8, cudaMemcpyDeviceToHost, st), "D2H");
        CK(cudaMemcpyAsync(i1, f->d_hi1, (size_t)m * 8, cudaMemcpyDeviceToHost, st), "D2H");
        CK(cudaStreamSynchronize(st), "match sync");
    }
    *nmatch = m;
    return XCB_OK;
}

extern "C" int xcb_front_lk_check_host(xcb_front* f, const double* As, const double* gs, int n, double* X, double* Inv)
{
    if (!f || n < 0 || (n && (!As || !gs || !X || !Inv))) return fail(f, XCB_ERR_ARG, "lk_check: bad argument");
    if (n == 0) return XCB_OK;
    double *dA, *dg, *dX, *dI;
    cudaStream_t st = f->stream;
    CK(cudaMallocAsync((void**)&dA, (size_t)n * 9 * 8, st), "alloc");
    CK(cudaMallocAsync((void**)&dg, (size_t)n * 3 * 8, st), "alloc");
    CK(cudaMallocAsync((void**)&dX, (size_t)n * 3 * 8, st), "alloc");
    CK(cudaMallocAsync((void**)&dI, (size_t)n * 9 * 8, st), "alloc");
    CK(cudaMemcpyAsync(dA, As, (size_t)n * 9 * 8, cudaMemcpyHostToDevice, st), "H2D");
    CK(cudaMemcpyAsync(dg, gs, (size_t)n * 3 * 8, cudaMemcpyHostToDevice, st), "H2D");
    CK(xcb_launch_lkcheck(dA, dg, n, dX, dI, st), "lkcheck");
    CK(cudaMemcpyAsync(X, dX, (size_t)n * 3 * 8, cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaMemcpyAsync(Inv, dI, (size_t)n * 9 * 8, cudaMemcpyDeviceToHost, st), "D2H");
    cudaFreeAsync(dA, st); cudaFreeAsync(dg, st); cudaFreeAsync(dX, st); cudaFreeAsync(dI, st);
    CK(cudaStreamSynchronize(st), "lkcheck sync");
    return XCB_OK;
}

// ----------------------------------------------------------------------------------------------- batched pipeline
static int enqueue_pipeline(xcb_front* f, const u8* left, const u8* right, int F, int budget, int half, int dlo,
                            int dhi, int match_prev, cudaStream_t st, int* nl, const cudaEvent_t* ev)
{
    int rc = enqueue_detect(f, left, F, budget, st, nl, ev);
    if (rc) return rc;
    int* counts = f->d_counts_chain + 1;
    CK(xcb_launch_stereo(left, right, nullptr, F, f->H, f->W, nullptr, nullptr, nullptr, F, f->d_kp, counts, f->cap,
                         dlo, dhi, 0, half, f->d_d, f->d_sig, f->d_ok, f->d_zn, f->d_dy, f->d_err, f->d_jobs,
                         f->tune[XCB_TUNE_STEREO_WARPS], f->tune[XCB_TUNE_STEREO_GROUP], st), "stereo");
    CK(mark(ev, 6, st), "event");
    if (!match_prev) CK(cudaMemsetAsync(f->d_counts_chain, 0, sizeof(int), st), "memset");
    XcbHamPairs p;
    p.A = f->d_desc_chain;
    p.B = f->d_desc_chain + (size_t)f->cap * 32;
    p.strideA = p.strideB = (long long)f->cap * 32;
    p.LA = f->d_counts_chain;
    p.NB = f->d_counts_chain + 1;
    p.npair = F;
    p.maxL = p.maxN = f->cap;
    CK(xcb_launch_hamming(p, f->d_b1, f->d_b2, f->d_bi, f->d_ci, st), "hamming");
    CK(xcb_launch_match_epilogue(p, f->d_b1, f->d_b2, f->d_bi, f->d_ci, 104, 0.8, f->d_m0, f->d_m1, f->cap,
                                 f->d_nmatch, st), "match");
    CK(mark(ev, 7, st), "event");
    // carry the last frame's descriptors to slot 0 for the next call
    CK(cudaMemcpyAsync(f->d_desc_chain, f->d_desc_chain + (size_t)F * f->cap * 32, (size_t)f->cap * 32,
                       cudaMemcpyDeviceToDevice, st), "carry desc");
    CK(cudaMemcpyAsync(f->d_counts_chain, f->d_counts_chain + F, sizeof(int), cudaMemcpyDeviceToDevice, st), "carry count");
    *nl += 5;                        // stereo search + LK, hamming, match epilogue (+ the carry copies)
    return XCB_OK;
}

extern "C" int xcb_front_pipeline_dev(xcb_front* f, const uint8_t* left, const uint8_t* right, int nframes, int budget,
                                      int half, int dlo, int dhi, int match_prev, void* stream)
{
    if (!f || !left || !right) return fail(f, XCB_ERR_ARG, "pipeline: null argument");
    if (!f->calibrated) return fail(f, XCB_ERR_NOT_CALIBRATED, "pipeline: front not calibrated");
    if (nframes < 1 || nframes > f->maxF) return fail(f, XCB_ERR_CAPACITY, "pipeline: frame count out of range");
    if (budget < 1 || budget > f->cap) return fail(f, XCB_ERR_CAPACITY, "pipeline: budget > cap");
    if (half < 3 || half > 5) return fail(f, XCB_ERR_ARG, "pipeline: half must be 3, 4 or 5");
    int rc = set_geometry(f, budget);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : f->stream;
    xcb_front::GraphEntry* hit = nullptr;
    for (auto& g : f->graphs)
        if (g.left == left && g.right == right && g.F == nframes && g.budget == budget && g.half == half &&
            g.dlo == dlo && g.dhi == dhi && g.match_prev == match_prev && g.stream == st) { hit = &g; break; }
    if (!hit) {
        if (f->graphs.size() >= 16) {   // evict the least recently used graph
            size_t lru = 0;
            for (size_t i = 1; i < f->graphs.size(); ++i) if (f->graphs[i].used < f->graphs[lru].used) lru = i;
            drop_graph(f->graphs[lru]);
            f->graphs.erase(f->graphs.begin() + lru);
        }
        int nl = 0;
        cudaGraph_t g;
        xcb_front::GraphEntry e;
        e.timed = f->stage_timing;
        if (e.timed)
            for (int i = 0; i <= XCB_FRONT_STAGES; ++i) CK(cudaEventCreate(&e.ev[i]), "event create");
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
        rc = enqueue_pipeline(f, left, right, nframes, budget, half, dlo, dhi, match_prev, st, &nl,
                              e.timed ? e.ev : nullptr);
        cudaError_t ec = cudaStreamEndCapture(st, &g);
        if (rc || ec != cudaSuccess) {
            if (e.timed)
                for (int i = 0; i <= XCB_FRONT_STAGES; ++i) cudaEventDestroy(e.ev[i]);
            if (rc) return rc;
            return cuda_fail(f, ec, "end capture");
        }
        ec = cudaGraphInstantiate(&e.exec, g, 0);
        cudaGraphDestroy(g);
        if (ec != cudaSuccess) return cuda_fail(f, ec, "graph instantiate");
        e.left = left; e.right = right; e.F = nframes; e.budget = budget; e.half = half; e.dlo = dlo; e.dhi = dhi;
        e.match_prev = match_prev; e.stream = st; e.used = 0;
        f->graphs.push_back(e);
        hit = &f->graphs.back();
        f->last_launches = nl;
    }
    hit->used = ++f->graph_clock;
    hit->fresh = true;
    CK(cudaGraphLaunch(hit->exec, st), "graph launch");
    return XCB_OK;
}

extern "C" int xcb_front_set_stage_timing(xcb_front* f, int on)
{
    if (!f) return fail(f, XCB_ERR_ARG, "set_stage_timing: null handle");
    CK(cudaDeviceSynchronize(), "sync");
    if ((bool)on != f->stage_timing) drop_graphs(f);
    f->stage_timing = on != 0;
    return XCB_OK;
}

extern "C" int xcb_front_set_tuning(xcb_front* f, int knob, int value)
{
    if (!f) return fail(nullptr, XCB_ERR_ARG, "set_tuning: null front");
    if (knob == XCB_TUNE_STEREO_WARPS) {
        if (value < 0 || value > 8) return fail(f, XCB_ERR_ARG, "set_tuning: stereo warps per block in 0..8");
    } else if (knob == XCB_TUNE_STEREO_GROUP) {
        if (value < 0 || value > 32) return fail(f, XCB_ERR_ARG, "set_tuning: stereo points per warp in 0..32");
    } else {
        return fail(f, XCB_ERR_ARG, "set_tuning: not a front knob");
    }
    if (f->tune[knob] != value) {
        f->tune[knob] = value;
        drop_graphs(f);            // the captured pipelines hold the old launch shapes
    }
    return XCB_OK;
}

extern "C" int xcb_front_stage_times(xcb_front* f, float* ms, int* ngraphs)
{
    if (!f || !ms) return fail(f, XCB_ERR_ARG, "stage_times: null argument");
    for (int i = 0; i < XCB_FRONT_STAGES; ++i) ms[i] = 0.0f;
    int n = 0;
    for (auto& g : f->graphs) {
        if (!g.timed || !g.fresh) continue;
        for (int i = 0; i < XCB_FRONT_STAGES; ++i) {
            float t = 0.0f;
            CK(cudaEventElapsedTime(&t, g.ev[i], g.ev[i + 1]), "elapsed");
            ms[i] += t;
        }
        g.fresh = false;
        ++n;
    }
    if (ngraphs) *ngraphs = n;
    return XCB_OK;
}

extern "C" int xcb_front_sync_check(xcb_front* f, void* stream)
{
    if (!f) return fail(f, XCB_ERR_ARG, "sync_check: null handle");
    CK(cudaStreamSynchronize(stream ? (cudaStream_t)stream : f->stream), "sync");
    return check_dev_err(f);
}

extern "C" int xcb_front_buffers(xcb_front* f, xcb_front_bufs* o)
{
    if (!f || !o) return fail(f, XCB_ERR_ARG, "buffers: null argument");
    o->counts = f->d_counts_chain + 1;
    o->kp = f->d_kp;
    o->desc = f->d_desc_chain + (size_t)f->cap * 32;
    o->d = f->d_d; o->sig = f->d_sig; o->ok = f->d_ok; o->zn = f->d_zn; o->dy = f->d_dy;
    o->m0 = (int64_t*)f->d_m0; o->m1 = (int64_t*)f->d_m1; o->nmatch = f->d_nmatch;
    o->floor = f->d_floor; o->anypos = f->d_anypos;
    return XCB_OK;
}

// D2H of every non-NULL result array of `out` for the frames [f0, f0 + nframes) of a host result set
// the result fields of xcb_front_bufs with their bytes per frame, in one table for the staging copies
struct ResField {
    size_t off;      // offset of the field in xcb_front_bufs (a pointer member)
    size_t per;      // bytes per frame
};

static int result_fields(const xcb_front* f, ResField* rf)
{
    const size_t cap = f->cap;
    int n = 0;
#define RF(field, per_frame) rf[n++] = ResField{offsetof(xcb_front_bufs, field), (per_frame)};
    RF(counts, 4) RF(kp, cap * 8) RF(desc, cap * 32) RF(d, cap * 8) RF(sig, cap * 8) RF(ok, cap) RF(zn, cap * 8)
    RF(dy, cap * 8) RF(m0, cap * 8) RF(m1, cap * 8) RF(nmatch, 4) RF(floor, 8) RF(anypos, 4)
#undef RF
    return n;
}

static void* field_ptr(const xcb_front_bufs* b, size_t off) { return *(void* const*)((const char*)b + off); }

// device results of the last batch (fn frames) -> staging block `stage` (fields at maxF-frame strides), on st
static int stage_results(xcb_front* f, const xcb_front_bufs* out, char* stage, size_t fn, cudaStream_t st)
{
    xcb_front_bufs d;
    xcb_front_buffers(f, &d);
    ResField rf[16];
    const int n = result_fields(f, rf);
    size_t base = 0;
    for (int i = 0; i < n; ++i) {
        if (field_ptr(out, rf[i].off))
            CK(cudaMemcpyAsync(stage + base, field_ptr(&d, rf[i].off), fn * rf[i].per, cudaMemcpyDeviceToDevice, st),
               "stage results");
        base += (size_t)f->maxF * rf[i].per;
    }
    return XCB_OK;
}

// staging block -> the host rows f0.. of `out`, on rs
static int read_stage(xcb_front* f, const xcb_front_bufs* out, const char* stage, size_t f0, size_t fn, cudaStream_t rs)
{
    ResField rf[16];
    const int n = result_fields(f, rf);
    size_t base = 0;
    for (int i = 0; i < n; ++i) {
        char* h = (char*)field_ptr(out, rf[i].off);
        if (h) CK(cudaMemcpyAsync(h + f0 * rf[i].per, stage + base, fn * rf[i].per, cudaMemcpyDeviceToHost, rs), "D2H");
        base += (size_t)f->maxF * rf[i].per;
    }
    return XCB_OK;
}

extern "C" int xcb_front_pipeline_host_batches(xcb_front* f, const uint8_t* left, const uint8_t* right, int nframes,
                                               int batch, int budget, int half, int dlo, int dhi, int match_prev,
                                               const xcb_front_bufs* out, void* stream)
{
    if (!f || !left || !right || !out) return fail(f, XCB_ERR_ARG, "pipeline_host_batches: null argument");
    if (nframes < 1 || batch < 1 || batch > f->maxF)
        return fail(f, XCB_ERR_CAPACITY, "pipeline_host_batches: frame or batch count out of range");
    const size_t npx = (size_t)f->W * f->H;
    cudaStream_t st = stream ? (cudaStream_t)stream : f->stream;
    if (!f->cstream) {
        CK(cudaStreamCreateWithFlags(&f->cstream, cudaStreamNonBlocking), "copy stream");
        CK(cudaStreamCreateWithFlags(&f->rstream, cudaStreamNonBlocking), "read-back stream");
        for (int k = 0; k < 2; ++k) {
            CK(cudaEventCreateWithFlags(&f->ev_loaded[k], cudaEventDisableTiming), "event");
            CK(cudaEventCreateWithFlags(&f->ev_free[k], cudaEventDisableTiming), "event");
            CK(cudaEventCreateWithFlags(&f->ev_staged[k], cudaEventDisableTiming), "event");
            CK(cudaEventCreateWithFlags(&f->ev_read[k], cudaEventDisableTiming), "event");
        }
        CK(dalloc(f, &f->d_in2[0], (size_t)f->maxF * npx), "alloc inputs");
        CK(dalloc(f, &f->d_in2[1], (size_t)f->maxF * npx), "alloc inputs");
        ResField rf[16];
        const int nf = result_fields(f, rf);
        size_t per = 0;
        for (int i = 0; i < nf; ++i) per += rf[i].per;
        CK(dalloc(f, &f->d_stage[0], (size_t)f->maxF * per), "alloc staging");
        CK(dalloc(f, &f->d_stage[1], (size_t)f->maxF * per), "alloc staging");
        for (int k = 0; k < 2; ++k) {
            CK(cudaEventRecord(f->ev_free[k], st), "event");
            CK(cudaEventRecord(f->ev_read[k], st), "event");
        }
    }
    // input pairs: buffer 0 = the front's own (d_left, d_right), buffer 1 = d_in2
    u8* inL[2] = {f->d_left, f->d_in2[0]};
    u8* inR[2] = {f->d_right, f->d_in2[1]};
    const int nb = (nframes + batch - 1) / batch;
    auto load = [&](int b) -> int {
        const int k = b & 1;
        const size_t f0 = (size_t)b * batch, fn = (size_t)std::min(batch, nframes - b * batch);
        CK(cudaStreamWaitEvent(f->cstream, f->ev_free[k], 0), "wait free");
        CK(cudaMemcpyAsync(inL[k], left + f0 * npx, fn * npx, cudaMemcpyHostToDevice, f->cstream), "H2D left");
        CK(cudaMemcpyAsync(inR[k], right + f0 * npx, fn * npx, cudaMemcpyHostToDevice, f->cstream), "H2D right");
        CK(cudaEventRecord(f->ev_loaded[k], f->cstream), "loaded");
        return XCB_OK;
    };
    auto read = [&](int b) -> int {
        const int k = b & 1;
        const size_t f0 = (size_t)b * batch, fn = (size_t)std::min(batch, nframes - b * batch);
        CK(cudaStreamWaitEvent(f->rstream, f->ev_staged[k], 0), "wait staged");
        const int r = read_stage(f, out, f->d_stage[k], f0, fn, f->rstream);
        if (r) return r;
        CK(cudaEventRecord(f->ev_read[k], f->rstream), "read");
        return XCB_OK;
    };
    int rc = load(0);
    if (!rc && nb > 1) rc = load(1);
    for (int b = 0; b < nb && !rc; ++b) {
        const int k = b & 1;
        const int fn = std::min(batch, nframes - b * batch);
        CK(cudaStreamWaitEvent(st, f->ev_loaded[k], 0), "wait loaded");
        rc = xcb_front_pipeline_dev(f, inL[k], inR[k], fn, budget, half, dlo, dhi, match_prev || b > 0, st);
        if (rc) break;
        CK(cudaEventRecord(f->ev_free[k], st), "free");
        // the next upload into this buffer pair, then this batch's results into staging block k once batch b-2's
        // read-back from it has finished
        if (b + 2 < nb && (rc = load(b + 2))) break;
        CK(cudaStreamWaitEvent(st, f->ev_read[k], 0), "wait read");
        if ((rc = stage_results(f, out, f->d_stage[k], (size_t)fn, st))) break;
        CK(cudaEventRecord(f->ev_staged[k], st), "staged");
        // the previous batch's read-back is queued only now, so that a read into pageable host memory (which returns
        // only when done) leaves this batch's work already queued on the device
        if (b > 0 && (rc = read(b - 1))) break;
    }
    if (!rc) rc = read(nb - 1);
    if (rc) {
        cudaStreamSynchronize(f->cstream);
        cudaStreamSynchronize(f->rstream);
        cudaStreamSynchronize(st);
        return rc;
    }
    CK(cudaStreamSynchronize(f->rstream), "read-back sync");
    CK(cudaStreamSynchronize(st), "pipeline sync");
    return check_dev_err(f);
}

extern "C" int xcb_front_pipeline_host(xcb_front* f, const uint8_t* left, const uint8_t* right, int nframes,
                                       int budget, int half, int dlo, int dhi, int match_prev, const xcb_front_bufs* out,
                                       void* stream)
{
    if (!f || !left || !right || !out) return fail(f, XCB_ERR_ARG, "pipeline_host: null argument");
    if (nframes < 1 || nframes > f->maxF) return fail(f, XCB_ERR_CAPACITY, "pipeline_host: frame count out of range");
    size_t bytes = (size_t)nframes * f->W * f->H;
    cudaStream_t st = stream ? (cudaStream_t)stream : f->stream;
    // host -> device straight from the caller's (ideally pinned) buffers
    CK(cudaMemcpyAsync(f->d_left, left, bytes, cudaMemcpyHostToDevice, st), "H2D left");
    CK(cudaMemcpyAsync(f->d_right, right, bytes, cudaMemcpyHostToDevice, st), "H2D right");
    int rc = xcb_front_pipeline_dev(f, f->d_left, f->d_right, nframes, budget, half, dlo, dhi, match_prev, st);
    if (rc) return rc;
    const size_t F = nframes, cap = f->cap;
    xcb_front_bufs d;
    xcb_front_buffers(f, &d);
#define DL(field, bytes_)                                                                                   \
    if (out->field) CK(cudaMemcpyAsync(out->field, d.field, (bytes_), cudaMemcpyDeviceToHost, st), "D2H " #field);
    DL(counts, F * 4)
    DL(kp, F * cap * 8)
    DL(desc, F * cap * 32)
    DL(d, F * cap * 8)
    DL(sig, F * cap * 8)
    DL(ok, F * cap)
    DL(zn, F * cap * 8)
    DL(dy, F * cap * 8)
    DL(m0, F * cap * 8)
    DL(m1, F * cap * 8)
    DL(nmatch, F * 4)
    DL(floor, F * 8)
    DL(anypos, F * 4)
#undef DL
    CK(cudaStreamSynchronize(st), "pipeline sync");
    return check_dev_err(f);
}
