// Chi-square reduction over caller-owned device images that performs no
// device allocation (shape_chi2_frames_noalloc in include/shape_b200.h).
//
// Who needs this: callers that cannot call cudaMalloc. A host program that
// hands all of its device memory to another allocator (a PyTorch process
// under a hard memory cap, a pool that pre-plans every byte of a serving
// loop) must not have a library grab memory behind its back, and a caller on
// a latency-critical path cannot afford cudaMalloc/cudaFree, which can
// synchronize the whole device. Such a caller already holds its observed
// images, variances and fit images in device memory; this entry point reads
// them and returns the per-frame sums to host memory.
//
// The per-block partial sums, the frame table and the per-frame results live
// in one file-scope device array, g_noalloc_scratch, sized for at most
// MAX_FRAMES (4096) frames and MAX_ITEMS (65536) blocks of CHI2_BLOCK (2048)
// elements (about 3.5 MB, held by every device that loads the library until
// the process exits). Host code never passes the symbol itself to a kernel
// (on the host it is only a stand-in for the device array): the first call
// on each device, with that device current, resolves the array's device
// address with cudaGetSymbolAddress and caches it. Calls share the array and
// keep the last call's contents; calls that overlap on the GPU (two host
// threads, or two streams) race on it.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "shape_b200.h"

namespace shape {
int report_error(int code, const std::string &msg);   // engine.cu
namespace noalloc {

constexpr int CHI2_BLOCK = 2048;            // elements per partial block
constexpr int THREADS = 256;
constexpr int MAX_FRAMES = 4096;
constexpr int MAX_ITEMS = 65536;            // MAX_ITEMS * CHI2_BLOCK = 134M elements
constexpr int MAX_DEVICES = 64;

// Layout of the scratch array, in doubles:
//   [0, 6*MAX_ITEMS)                 partials: o2, m2, om (each sum + compensation)
//   then MAX_FRAMES+1 long longs     frame offsets (element index of each frame)
//   then MAX_FRAMES+1 ints           first block of each frame (prefix), padded
//   then 3*MAX_FRAMES doubles        weight, cal_floating, cal
//   then 5*MAX_FRAMES doubles        results: o2, m2, om, cal, chi2
constexpr size_t OFF_PARTIALS = 0;
constexpr size_t OFF_OFFSETS = OFF_PARTIALS + 6 * (size_t)MAX_ITEMS;
constexpr size_t OFF_PREFIX = OFF_OFFSETS + (MAX_FRAMES + 1);
constexpr size_t OFF_PARAMS = OFF_PREFIX + (MAX_FRAMES + 2) / 2;
constexpr size_t OFF_RESULTS = OFF_PARAMS + 3 * (size_t)MAX_FRAMES;
constexpr size_t SCRATCH_DOUBLES = OFF_RESULTS + 5 * (size_t)MAX_FRAMES;

static __device__ __align__(256) double g_noalloc_scratch[SCRATCH_DOUBLES];

struct Scratch {
    double *partials;
    long long *offsets;
    int *prefix;
    double *params;
    double *results;
};

__device__ inline void kadd(double &s, double &c, double x)
{
    double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
}

// First block of every frame (prefix over ceil(size / CHI2_BLOCK)).
__global__ void k_plan(Scratch S, int nframes)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int acc = 0;
    for (int f = 0; f < nframes; f++) {
        S.prefix[f] = acc;
        long long n = S.offsets[f + 1] - S.offsets[f];
        acc += (int)((n + CHI2_BLOCK - 1) / CHI2_BLOCK);
    }
    S.prefix[nframes] = acc;
}

// Compensated partial sums of chi2_deldop's o2 / m2 / om
// (src/shape/chi2.c:436-441) for one block of one frame.
__global__ void k_partials(Scratch S, int nframes, int nitems, const double *__restrict__ obs,
                           const double *__restrict__ oov, const double *__restrict__ fit)
{
    __shared__ double red[THREADS / 32][6];
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        int lo = 0, hi = nframes - 1;
        while (lo < hi) {                    // frame of block `it`
            int mid = (lo + hi + 1) / 2;
            if (S.prefix[mid] <= it) lo = mid; else hi = mid - 1;
        }
        const int f = lo;
        const long long start = S.offsets[f] + (long long)(it - S.prefix[f]) * CHI2_BLOCK;
        const long long end = min(start + CHI2_BLOCK, S.offsets[f + 1]);
        double s[3] = {0, 0, 0}, c[3] = {0, 0, 0};
        for (long long k = start + threadIdx.x; k < end; k += blockDim.x) {
            double ob = obs[k], w = oov[k], ft = fit[k];
            kadd(s[0], c[0], ob * ob * w);
            kadd(s[1], c[1], ft * ft * w);
            kadd(s[2], c[2], ft * ob * w);
        }
        for (int off = 16; off > 0; off >>= 1)
            for (int q = 0; q < 3; q++) {
                double os = __shfl_down_sync(0xffffffffu, s[q], off);
                double oc = __shfl_down_sync(0xffffffffu, c[q], off);
                kadd(s[q], c[q], os);
                c[q] += oc;
            }
        if ((threadIdx.x & 31) == 0)
            for (int q = 0; q < 3; q++) {
                red[threadIdx.x >> 5][2 * q] = s[q];
                red[threadIdx.x >> 5][2 * q + 1] = c[q];
            }
        __syncthreads();
        if (threadIdx.x == 0) {
            double rs[3] = {0, 0, 0}, rc[3] = {0, 0, 0};
            for (int w = 0; w < THREADS / 32; w++)
                for (int q = 0; q < 3; q++) {
                    kadd(rs[q], rc[q], red[w][2 * q]);
                    rc[q] += red[w][2 * q + 1];
                }
            for (int q = 0; q < 3; q++) {
                S.partials[(size_t)it * 6 + 2 * q] = rs[q];
                S.partials[(size_t)it * 6 + 2 * q + 1] = rc[q];
            }
        }
        __syncthreads();
    }
}

// Calibration and chi-square per frame (src/shape/chi2.c:447-460).
__global__ void k_frames(Scratch S, int nframes)
{
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nframes) return;
    double s[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    for (int it = S.prefix[f]; it < S.prefix[f + 1]; it++)
        for (int q = 0; q < 3; q++) {
            kadd(s[q], c[q], S.partials[(size_t)it * 6 + 2 * q]);
            c[q] += S.partials[(size_t)it * 6 + 2 * q + 1];
        }
    double o2 = s[0] + c[0], m2 = s[1] + c[1], om = s[2] + c[2];
    double weight = S.params[f], cal = S.params[2 * MAX_FRAMES + f];
    if (S.params[MAX_FRAMES + f] != 0.0)
        cal = (om > 0.0) ? om / m2 : SHAPE_TINYCALFACT;
    double *r = S.results + 5 * (size_t)f;
    r[0] = o2; r[1] = m2; r[2] = om; r[3] = cal;
    r[4] = weight * (o2 - 2 * cal * om + cal * cal * m2);
}

static std::mutex g_mu;
static double *g_addr[MAX_DEVICES];          // device address of g_noalloc_scratch, per device

// Errors go to the message shape_last_error() returns (engine.cu).
static int fail(int code, const std::string &m) { return shape::report_error(code, m); }

// Makes `device` current for the call and gives the caller's current device
// back on every return path.
struct DeviceGuard {
    int prev = -1;
    cudaError_t set(int device)
    {
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) { prev = -1; return e; }
        return prev == device ? cudaSuccess : cudaSetDevice(device);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace noalloc
}  // namespace shape

using namespace shape::noalloc;

extern "C" int shape_chi2_frames_noalloc(int device, int nframes, const long long *frame_offsets,
                                         const double *d_obs, const double *d_oneovervar,
                                         const double *d_fit, const double *weight,
                                         const int *cal_floating, const double *cal, double *out)
{
    if (nframes < 1 || !frame_offsets || !d_obs || !d_oneovervar || !d_fit || !weight ||
        !cal_floating || !cal || !out)
        return fail(SHAPE_E_ARG, "shape_chi2_frames_noalloc: null argument or nframes < 1");
    if (nframes > MAX_FRAMES)
        return fail(SHAPE_E_ARG, "shape_chi2_frames_noalloc: " + std::to_string(nframes) +
                                     " frames exceed the maximum of " + std::to_string(MAX_FRAMES));
    long long nitems = 0;
    for (int f = 0; f < nframes; f++) {
        long long n = frame_offsets[f + 1] - frame_offsets[f];
        if (n < 0) return fail(SHAPE_E_ARG, "shape_chi2_frames_noalloc: frame offsets must not decrease");
        nitems += (n + CHI2_BLOCK - 1) / CHI2_BLOCK;
    }
    if (nitems > MAX_ITEMS)
        return fail(SHAPE_E_ARG, "shape_chi2_frames_noalloc: " + std::to_string(nitems * (long long)CHI2_BLOCK) +
                                     " elements exceed the maximum of " +
                                     std::to_string((long long)MAX_ITEMS * CHI2_BLOCK));
    if (device < 0 || device >= MAX_DEVICES) return fail(SHAPE_E_ARG, "shape_chi2_frames_noalloc: bad device");
    DeviceGuard dg;
    cudaError_t e = dg.set(device);
    if (e != cudaSuccess) return fail(SHAPE_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    double *base;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[device]) {
            // once per device, with that device current
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return fail(SHAPE_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_addr[device] = static_cast<double *>(p);
        }
        base = g_addr[device];
    }
    Scratch S;
    S.partials = base + OFF_PARTIALS;
    S.offsets = reinterpret_cast<long long *>(base + OFF_OFFSETS);
    S.prefix = reinterpret_cast<int *>(base + OFF_PREFIX);
    S.params = base + OFF_PARAMS;
    S.results = base + OFF_RESULTS;
    // frame table into the scratch array (the previous call's contents are
    // overwritten; every partial and result slot read below is written first)
    double fl[2048];
    e = cudaMemcpy(S.offsets, frame_offsets, sizeof(long long) * (nframes + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(S.params, weight, sizeof(double) * nframes, cudaMemcpyHostToDevice);
    for (int f0 = 0; e == cudaSuccess && f0 < nframes; f0 += 2048) {
        int n = nframes - f0 < 2048 ? nframes - f0 : 2048;
        for (int k = 0; k < n; k++) fl[k] = cal_floating[f0 + k] ? 1.0 : 0.0;
        e = cudaMemcpy(S.params + MAX_FRAMES + f0, fl, sizeof(double) * n, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(S.params + 2 * MAX_FRAMES, cal, sizeof(double) * nframes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(S.results, 0, sizeof(double) * 5 * nframes);
    if (e != cudaSuccess) return fail(SHAPE_E_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    k_plan<<<1, 32>>>(S, nframes);
    int blocks = nitems < 4 * 148 ? (int)nitems : 4 * 148;
    if (blocks > 0) k_partials<<<blocks, THREADS>>>(S, nframes, (int)nitems, d_obs, d_oneovervar, d_fit);
    k_frames<<<(nframes + 127) / 128, 128>>>(S, nframes);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, S.results, sizeof(double) * 5 * nframes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(SHAPE_E_CUDA, std::string("chi2 kernels: ") + cudaGetErrorString(e));
    return SHAPE_OK;
}
