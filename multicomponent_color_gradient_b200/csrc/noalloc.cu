// noalloc.cu - float64 population sums that allocate no device memory.
//
// Who needs this: callers that own every byte of device memory themselves and
// allow no allocation once their time loop runs - for example a driver built
// like the reference's main.cu that keeps its populations in its own
// LbmDevice-style buffers and runs with HBM nearly full.  For them a
// cudaMalloc inside a diagnostic can fail outright, and a cudaFree would
// synchronise the whole device in the middle of the step sequence.
// mcg_conservation_sums needs a handle, whose creation allocates; this entry
// point works on the caller's buffers and keeps its scratch (per-plane
// partial sums) in a fixed file-scope device array instead.
//
// The array is sized for MCG_STATIC_SCRATCH_PLANES z-planes (5 doubles each,
// 160 KiB) and lives on every GPU that loads this library until the process
// exits.  All calls share it: two calls whose kernels overlap on the GPU
// (different streams, or several host threads) race on it and must be
// serialised by the caller.  Each call overwrites every slot it reads, so the
// previous call's contents never leak into a result.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "internal.hpp"
#include "lattice.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_static_partials[MCG_STATIC_SCRATCH_PLANES * 5];

__constant__ int c_ncx[mcg::kQ] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
__constant__ int c_ncy[mcg::kQ] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
__constant__ int c_ncz[mcg::kQ] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < kThreads / 32; ++k) r += sh[k];
    return r;
}

// One block per interior z-plane: sums of fr, fb and (fr+fb) c over the
// plane's interior nodes, written (not accumulated) to the plane's slot.
__global__ void __launch_bounds__(kThreads) k_plane_sums(const float *__restrict__ fr, const float *__restrict__ fb,
                                                         int NX, int NY, size_t N, double *partials) {
    __shared__ double sh[kThreads / 32];
    const int z = 1 + int(blockIdx.x);
    double acc[5] = {0, 0, 0, 0, 0};
    const int nxi = NX - 2, nyi = NY - 2;
    for (int k = threadIdx.x; k < nxi * nyi; k += blockDim.x) {
        const int x = 1 + k % nxi, y = 1 + k / nxi;
        const size_t id = size_t(x) + size_t(NX) * (size_t(y) + size_t(NY) * size_t(z));
        for (int i = 0; i < mcg::kQ; ++i) {
            const double a = fr[size_t(i) * N + id], b = fb[size_t(i) * N + id];
            acc[0] += a;
            acc[1] += b;
            acc[2] += (a + b) * c_ncx[i];
            acc[3] += (a + b) * c_ncy[i];
            acc[4] += (a + b) * c_ncz[i];
        }
    }
    for (int q = 0; q < 5; ++q) {
        const double r = block_sum(acc[q], sh);
        if (threadIdx.x == 0) partials[size_t(blockIdx.x) * 5 + q] = r;
    }
}

// One block folds the plane partials in plane order (deterministic).
__global__ void __launch_bounds__(kThreads) k_fold_planes(const double *partials, int nplanes, double *out5) {
    __shared__ double sh[kThreads / 32];
    for (int q = 0; q < 5; ++q) {
        double acc = 0.0;
        for (int p = threadIdx.x; p < nplanes; p += blockDim.x) acc += partials[size_t(p) * 5 + q];
        const double r = block_sum(acc, sh);
        if (threadIdx.x == 0) out5[q] = r;
    }
}

std::mutex g_setup_mutex;
struct ScratchAddr {
    void *ctx = nullptr;  // the context the address belongs to
    double *ptr = nullptr;
};
ScratchAddr g_partials_addr[kMaxDevices];

// cuCtxGetCurrent through the runtime's driver entry point table (the library
// does not link libcuda itself, so that it loads on machines without a GPU).
using CtxGetCurrent = int (*)(void **);
CtxGetCurrent ctx_get_current() {
    static CtxGetCurrent fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return CtxGetCurrent(nullptr);
        }
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    return fn;
}

void *current_context() {
    void *ctx = nullptr;
    if (CtxGetCurrent f = ctx_get_current()) f(&ctx);
    return ctx;
}

// Device address of g_static_partials on the current device.  The host-side
// name is only a stand-in for the symbol; the address comes from
// cudaGetSymbolAddress with that device current, once per device and
// context: a cudaDeviceReset tears the context and its module down, and the
// next context may load the array elsewhere, so a change of the current
// context looks the address up again.
mcg_status scratch_on_current_device(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mcg::cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return mcg::fail(MCG_ERR_UNSUPPORTED, "device index beyond 64");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    ScratchAddr &a = g_partials_addr[dev];
    void *ctx = current_context();
    if (!a.ptr || !ctx || ctx != a.ctx) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_partials);  // initialises the context if needed
        if (e != cudaSuccess) {
            a = ScratchAddr{};
            return mcg::cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
        }
        a.ptr = static_cast<double *>(p);
        a.ctx = current_context();
    }
    *out = a.ptr;
    return MCG_OK;
}

void forget_scratch_on_current_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    g_partials_addr[dev] = ScratchAddr{};
}

}  // namespace

extern "C" mcg_status mcg_conservation_sums_static(const float *fr, const float *fb, int32_t NX, int32_t NY,
                                                   int32_t NZ, double *out5, void *stream) {
    return mcg::guarded([&]() -> mcg_status {
        if (!fr || !fb || !out5) return mcg::fail(MCG_ERR_INVALID_ARG, "fr, fb and out5 must be device pointers");
        if (NX < 3 || NY < 3 || NZ < 3) return mcg::fail(MCG_ERR_INVALID_ARG, "NX, NY, NZ must be >= 3");
        const int planes = NZ - 2;
        if (planes > MCG_STATIC_SCRATCH_PLANES)
            return mcg::fail(MCG_ERR_INVALID_ARG, "NZ - 2 = " + std::to_string(planes) +
                                                      " interior planes exceed the static scratch of " +
                                                      std::to_string(MCG_STATIC_SCRATCH_PLANES) + " planes");
        const double n = double(NX) * NY * NZ;
        if (n >= 2147483647.0) return mcg::fail(MCG_ERR_INVALID_ARG, "NX*NY*NZ must be < 2^31");
        double *partials = nullptr;
        if (mcg_status s = scratch_on_current_device(&partials)) return s;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        k_plane_sums<<<planes, kThreads, 0, st>>>(fr, fb, NX, NY, size_t(n), partials);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) {
            k_fold_planes<<<1, kThreads, 0, st>>>(partials, planes, out5);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) {
            forget_scratch_on_current_device();  // looked up again by the next call
            return mcg::cuda_fail(e, "conservation sums kernels");
        }
        return MCG_OK;
    });
}
