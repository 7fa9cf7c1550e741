// noalloc.cu -- FP64 sums of a caller-owned moment field without allocating.
//
// mrlbm_reduce_fp64_ref_layout_noalloc reduces an FP32 moment field that the
// caller holds on the device in the reference's idxMom layout (the fMom array
// of the reference's host loop, src/arrayIndex.h:8-17).  Its block partials
// live in a file-scope __device__ array, so the call performs no allocation:
// no cudaMalloc, no cudaFree and no allocating library routine.
//
// Limits and rules (also stated at the declaration in include/mrlbm.h):
//   * scratch: NOALLOC_SCRATCH doubles (37,952 bytes) per device: 592 block
//     partials of 8 sums plus the 8 results.  The call always launches 592
//     blocks of 256 threads and strides over larger fields, so every field
//     size fits the array (checked at compile time).
//   * nothing in the scratch has to start at zero: each call writes every
//     partial before the finishing kernel reads it, and writes all 8 results.
//   * the array's device address is looked up with cudaGetSymbolAddress, with
//     the device current, on the first call in each CUDA context of a device
//     (again after a cudaDeviceReset, which replaces the context and may move
//     the array).
//   * every call synchronises `stream` to return the sums on the host, so no
//     call can be made while `stream` is being captured into a graph.
//   * calls share the one array per device: calls whose executions overlap on
//     a device (two host threads, or two streams with no ordering between
//     them) race on it and return wrong sums.  Serialise them.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "domain.h"

namespace {

constexpr int NOALLOC_THREADS = 256;
// The same partial count and node traversal as the domain reduction
// (mrlbm_reduce_fp64), so a field reduced both ways gives the same sums.
constexpr int NOALLOC_BLOCKS = 148 * 4;
constexpr int NOALLOC_SCRATCH = NOALLOC_BLOCKS * 8 + 8;
constexpr int NOALLOC_MAX_DEVICES = 64;
static_assert(NOALLOC_BLOCKS * 8 + 8 <= NOALLOC_SCRATCH, "the static scratch holds every block partial");

// FP64 block partials over all nodes of an FP32 idxMom field:
//   [0] rho, [1..3] rho u, [4] rho |u|^2 / 2, [5] nodes, [6] max |u|,
//   [7] non-finite moments (src/reduction.cu:100-155 in double).
__global__ void __launch_bounds__(NOALLOC_THREADS)
    noalloc_reduce_kernel(const float* __restrict__ fmom, int nx, int ny, int nz, int nm, float rho0, double* partial)
{
    __shared__ double sh[NOALLOC_THREADS / 32][8];
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long long n = (long long)nx * ny * nz;
    const int nbx = nx / 8, nby = ny / 8;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(g % nx);
        const int y = (int)((g / nx) % ny);
        const int z = (int)(g / ((long long)nx * ny));
        // idxMom: tx + 8*(ty + 8*(tz + 8*(mom + NM*(bx + NBX*(by + NBY*bz)))))
        const long long blk = (x >> 3) + (long long)nbx * ((y >> 3) + (long long)nby * (z >> 3));
        const long long base = (x & 7) + 8 * ((y & 7) + 8 * ((z & 7) + 8 * (long long)nm * blk));
        float v[4];
        bool finite = true;
        for (int k = 0; k < 4; k++) {
            v[k] = fmom[base + 512LL * k];
            finite = finite && isfinite(v[k]);
        }
        const double rho = (double)rho0 + (double)v[0];
        const double ux = v[1] / 3.0, uy = v[2] / 3.0, uz = v[3] / 3.0;
        const double u2 = ux * ux + uy * uy + uz * uz;
        acc[0] += rho;
        acc[1] += rho * ux; acc[2] += rho * uy; acc[3] += rho * uz;
        acc[4] += 0.5 * rho * u2;
        acc[5] += 1.0;
        acc[6] = fmax(acc[6], finite ? sqrt(u2) : INFINITY);
        acc[7] += finite ? 0.0 : 1.0;
    }
    // warp then block reduction, fixed order
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 8; k++) {
        double v = acc[k];
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, off);
            v = (k == 6) ? fmax(v, o) : v + o;
        }
        if (lane == 0) sh[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int k = threadIdx.x;
        double v = sh[0][k];
        for (int i = 1; i < NOALLOC_THREADS / 32; i++) v = (k == 6) ? fmax(v, sh[i][k]) : v + sh[i][k];
        partial[blockIdx.x * 8 + k] = v;
    }
}

__global__ void noalloc_reduce_finish(const double* partial, int nblocks, double* out)
{
    const int k = threadIdx.x;
    if (k >= 8) return;
    double v = 0.0;
    for (int b = 0; b < nblocks; b++) v = (k == 6) ? fmax(v, partial[b * 8 + k]) : v + partial[b * 8 + k];
    out[k] = v;
}

std::mutex g_setup_mutex;
double* g_scratch_ptr[NOALLOC_MAX_DEVICES] = {};
void* g_scratch_ctx[NOALLOC_MAX_DEVICES] = {};  // the CUDA context the address belongs to

// cuCtxGetCurrent through the runtime's driver entry point (no libcuda link)
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current()
{
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (CtxGetCurrentFn)p;
    }
    return fn;
}

}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH];

using mrlbm::fail;

extern "C" mrlbm_status mrlbm_reduce_fp64_ref_layout_noalloc(const float* fmom, int nx, int ny, int nz,
                                                            int num_moments, double rho0, void* stream,
                                                            mrlbm_sums* out)
{
    if (!fmom || !out) return fail(MRLBM_EINVAL, "null argument");
    if (nx <= 0 || ny <= 0 || nz <= 0 || nx % 8 || ny % 8 || nz % 8)
        return fail(MRLBM_EINVAL, "grid %d x %d x %d: the idxMom layout needs positive multiples of 8", nx, ny, nz);
    if (num_moments < 4) return fail(MRLBM_EINVAL, "num_moments %d: need at least rho and u (4)", num_moments);
    const int blocks = NOALLOC_BLOCKS;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(MRLBM_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(MRLBM_EINVAL, "device %d beyond %d", dev, NOALLOC_MAX_DEVICES);
    // the field must be device memory of the current device, or managed
    // memory (which every device can read, wherever it was allocated)
    cudaPointerAttributes pa{};
    e = cudaPointerGetAttributes(&pa, fmom);
    if (e != cudaSuccess) return fail(MRLBM_EINVAL, "cudaPointerGetAttributes: %s", cudaGetErrorString(e));
    if (pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged)
        return fail(MRLBM_EINVAL, "fmom is not device memory (the field must be resident on the current device)");
    if (pa.type == cudaMemoryTypeDevice && pa.device != dev)
        return fail(MRLBM_EINVAL, "fmom is on device %d, the current device is %d", pa.device, dev);
    double* scratch = nullptr;
    {
        // the array's address, looked up once per device and CUDA context
        // (the pointer query above has made the device's context current)
        CtxGetCurrentFn gc = ctx_get_current();
        if (!gc) return fail(MRLBM_ECUDA, "cuCtxGetCurrent unavailable");
        void* ctx = nullptr;
        if (gc(&ctx) != 0) ctx = nullptr;
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev] || !ctx || g_scratch_ctx[dev] != ctx) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return fail(MRLBM_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
            if (gc(&ctx) != 0) ctx = nullptr;
            g_scratch_ptr[dev] = static_cast<double*>(p);
            g_scratch_ctx[dev] = ctx;
        }
        scratch = g_scratch_ptr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* partial = scratch;
    double* res = scratch + (size_t)blocks * 8;
    noalloc_reduce_kernel<<<blocks, NOALLOC_THREADS, 0, s>>>(fmom, nx, ny, nz, num_moments, (float)rho0, partial);
    noalloc_reduce_finish<<<1, 32, 0, s>>>(partial, blocks, res);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MRLBM_ECUDA, "reduction launch: %s", cudaGetErrorString(e));
    double h[8];
    e = cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MRLBM_ECUDA, "reduction result: %s", cudaGetErrorString(e));
    out->mass = h[0];
    out->momentum[0] = h[1]; out->momentum[1] = h[2]; out->momentum[2] = h[3];
    out->kinetic_energy = h[4];
    out->fluid_nodes = h[5];
    out->max_speed = h[6];
    out->nonfinite = h[7];
    return MRLBM_OK;
}
