// dot_noalloc.cu -- the dot product of DOT_PRODUCT_PAR for callers that cannot
// allocate device memory.
//
// Some hosts own every byte of device memory through their own pool or run
// under a hard device-memory budget, so a library may not call cudaMalloc
// behind their back; others run timing-critical loops in which the implicit
// device synchronization of cudaMalloc/cudaFree is not acceptable.
// mfixgpu_dot_product_par_noalloc serves them: the scratch it needs (one
// partial sum per block and an arrival counter) is a fixed file-scope
// __device__ array of this library, so the call allocates nothing.  The caller
// passes the inputs and a device pointer for the result.
//
// The array exists once per device that loads the library and is kept until the
// process exits.  Every call on a device shares it and it keeps the last call's
// contents: each call clears the arrival counter before its kernel runs (the
// partial sums are always written before they are read).  Two calls whose work
// overlaps on the GPU, for example on two streams, race on the array.
//
// The first call on each device looks up the array's device address with
// cudaGetSymbolAddress (that device current) and caches it together with the
// device's current context; make that first call before any stream capture.  A
// call that finds another context current (the host reset the device, which
// loads the library's module again at a new address) looks the address up anew.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda.h>  // CUcontext and the cuCtxGetCurrent signature only: the driver is reached through the runtime
#include <cuda_runtime.h>

#include "../../include/mfixgpu.h"

namespace mfixgpu {
void set_last_error(const std::string &msg);  // capi.cu: the text mfixgpu_last_error() returns
}

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr int64_t NOALLOC_CHUNK = int64_t(1) << 17;  // elements each block reduces
constexpr int NOALLOC_MAX_BLOCKS = 2048;            // partial sums the scratch holds
static_assert(NOALLOC_CHUNK * NOALLOC_MAX_BLOCKS == MFIXGPU_NOALLOC_MAX_N, "limit mismatch");

// [0, 8*NOALLOC_MAX_BLOCKS): partial sums; then the arrival counter.
constexpr size_t NOALLOC_COUNTER_OFFSET = sizeof(double) * NOALLOC_MAX_BLOCKS;
static __device__ __align__(256) unsigned char noalloc_scratch[NOALLOC_COUNTER_OFFSET + 256];

__device__ __forceinline__ double block_total(double v)
{
    __shared__ double red[NOALLOC_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    v = 0.0;
    if (warp == 0) {
        v = lane < NOALLOC_THREADS / 32 ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;  // thread 0 holds the block total
}

// Block b sums r1*r2 over its fixed chunk in a fixed order; the last block to
// finish adds the partial sums in block order, so the result does not depend on
// scheduling.
__global__ void __launch_bounds__(NOALLOC_THREADS) k_dot_noalloc(const double *__restrict__ r1,
                                                                const double *__restrict__ r2, int64_t n,
                                                                double *__restrict__ out)
{
    double *partials = reinterpret_cast<double *>(noalloc_scratch);
    unsigned int *counter = reinterpret_cast<unsigned int *>(noalloc_scratch + NOALLOC_COUNTER_OFFSET);
    __shared__ int last;
    const int64_t c0 = (int64_t)blockIdx.x * NOALLOC_CHUNK;
    const int64_t c1 = min(n, c0 + NOALLOC_CHUNK);
    double v = 0.0;
    for (int64_t c = c0 + threadIdx.x; c < c1; c += NOALLOC_THREADS) v += r1[c] * r2[c];
    v = block_total(v);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v;
        __threadfence();
        last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += NOALLOC_THREADS) acc += __ldcg(partials + b);
    acc = block_total(acc);
    if (threadIdx.x == 0) {
        *out = acc;
        *counter = 0u;
    }
}

std::mutex g_mu;
void *g_scratch[64] = {};      // device address of noalloc_scratch, per device ordinal
CUcontext g_scratch_ctx[64] = {};  // the context that address belongs to

// The current context (nullptr when the driver's entry point is unavailable, in
// which case the cached address is trusted as it stands).
CUcontext current_context()
{
    using Fn = CUresult (*)(CUcontext *);
    static Fn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<Fn>(p);
        else
            cudaGetLastError();
    }
    CUcontext c = nullptr;
    if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return c;
}

int fail(const std::string &msg, int code)
{
    mfixgpu::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int mfixgpu_dot_product_par_noalloc(const double *r1_dev, const double *r2_dev, int64_t n,
                                               double *out_dev, void *stream)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!r1_dev || !r2_dev || !out_dev || n < 0) return fail("null pointer or negative length", MFIXGPU_ERR_ARGS);
    if (n > MFIXGPU_NOALLOC_MAX_N)
        return fail("n = " + std::to_string(n) + " exceeds MFIXGPU_NOALLOC_MAX_N = " +
                        std::to_string((long long)MFIXGPU_NOALLOC_MAX_N) + " (the fixed scratch holds " +
                        std::to_string(NOALLOC_MAX_BLOCKS) + " partial sums of " + std::to_string(NOALLOC_CHUNK) +
                        " elements each)",
                    MFIXGPU_ERR_ARGS);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return fail("no usable CUDA device", MFIXGPU_ERR_CUDA);
    }
    if (!g_scratch[dev] || current_context() != g_scratch_ctx[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);  // makes the device's context current
        if (e != cudaSuccess || !p) return fail(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e), MFIXGPU_ERR_CUDA);
        g_scratch[dev] = p;
        g_scratch_ctx[dev] = current_context();
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e =
        cudaMemsetAsync(static_cast<unsigned char *>(g_scratch[dev]) + NOALLOC_COUNTER_OFFSET, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) {
        if (n == 0) {
            e = cudaMemsetAsync(out_dev, 0, sizeof(double), s);
        } else {
            const int grid = (int)((n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK);
            k_dot_noalloc<<<grid, NOALLOC_THREADS, 0, s>>>(r1_dev, r2_dev, n, out_dev);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess) return fail(cudaGetErrorString(e), MFIXGPU_ERR_CUDA);
    return 0;
}
