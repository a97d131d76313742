// Allocation-free incremental potential: vbd_ip_energy_noalloc (declared in include/vbd_b200.h).
//
// Who it is for: code that embeds the solver in a framework owning all device memory (a PyTorch
// caching-allocator pool, a game engine's fixed arena) or in a fixed-latency simulation loop.
// Such callers cannot let a library call cudaMalloc / cudaFree behind their back: those calls
// synchronise the whole device and fail once the framework's pool holds the free memory.  This
// entry point therefore takes only caller-owned buffers and keeps its own scratch -- the FP64
// partial sums of the two-pass reduction -- in a fixed file-scope __device__ array.
//
// Scratch rules:
//   * g_noalloc_scratch holds kMaxBlocks block partials plus one error flag; every GPU that loads
//     this library holds it (4,097 doubles, 32 KiB) until the process exits.
//   * The host never names the array as an address: at the first call on each device, with that
//     device current, cudaGetSymbolAddress gives the device pointer, which is cached per device
//     and passed to the kernels.  That first call therefore has to come before any stream
//     capture on that device.  Later calls look the address up again whenever their stream is not
//     capturing (a lookup allocates nothing), so a cudaDeviceReset between two calls, after which
//     the array lives in a new context, is picked up by the next call.
//   * Calls share the array and it keeps the last call's contents.  The error flag must start at
//     zero and is cleared at the start of every call; each partial slot read in a call is written
//     earlier in the same call.  Two calls whose work overlaps on the GPU (different streams, or
//     different host threads on one device) race on the array.
#include <cuda_runtime.h>

#include <mutex>

#include "vbd_b200.h"
#include "vbd_internal.h"

namespace {

constexpr int kBlock = 256;
constexpr int kPerThread = 16;
constexpr int kPerBlock = kBlock * kPerThread;  // elements (vertices + tets) per block
constexpr int kMaxBlocks = 4096;
constexpr long long kMaxElements = (long long)kMaxBlocks * kPerBlock;  // 16,777,216
constexpr int kFlagSlot = kMaxBlocks;                                  // non-zero: bad tet id seen
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kMaxBlocks + 1];

std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// One element per (block, k, thread): vertices [0, N) contribute m/(2h^2)|x - y|^2, tets [N, N+T)
// contribute V0 psi(F) with psi = mu/2(|F|^2 - 3) - mu(J - 1) + lambda/2 (J - 1)^2 (the energy of
// the reference's force, Energy.cpp:97).  Tets holding an id outside [0, N) are skipped and raise
// the flag.
__global__ void __launch_bounds__(kBlock) k_ip_partials(int n, int t, const float* __restrict__ x,
                                                        const float* __restrict__ y, const float* __restrict__ mass,
                                                        const int* __restrict__ tets, const float* __restrict__ dminv,
                                                        const float* __restrict__ vol, const float* __restrict__ mu,
                                                        const float* __restrict__ lam, double inv_h2,
                                                        double* __restrict__ scratch) {
    double acc = 0.0;
    const long long total = (long long)n + t;
    for (int k = 0; k < kPerThread; ++k) {
        const long long e = (long long)blockIdx.x * kPerBlock + (long long)k * kBlock + threadIdx.x;
        if (e >= total) break;
        if (e < n) {
            const long long i = e;
            const double dx = (double)x[3 * i] - y[3 * i];
            const double dy = (double)x[3 * i + 1] - y[3 * i + 1];
            const double dz = (double)x[3 * i + 2] - y[3 * i + 2];
            acc += 0.5 * (double)mass[i] * inv_h2 * (dx * dx + dy * dy + dz * dz);
        } else {
            const long long q = e - n;
            const int i0 = tets[4 * q], i1 = tets[4 * q + 1], i2 = tets[4 * q + 2], i3 = tets[4 * q + 3];
            if ((unsigned)i0 >= (unsigned)n || (unsigned)i1 >= (unsigned)n || (unsigned)i2 >= (unsigned)n ||
                (unsigned)i3 >= (unsigned)n) {
                scratch[kFlagSlot] = 1.0;
                continue;
            }
            double Ds[3][3];
            for (int r = 0; r < 3; ++r) {
                const double o = x[3LL * i0 + r];
                Ds[r][0] = (double)x[3LL * i1 + r] - o;
                Ds[r][1] = (double)x[3LL * i2 + r] - o;
                Ds[r][2] = (double)x[3LL * i3 + r] - o;
            }
            const float* D = dminv + 9 * q;
            double F[3][3];
            double tr = 0.0;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    F[r][c] = Ds[r][0] * D[c] + Ds[r][1] * D[3 + c] + Ds[r][2] * D[6 + c];
                    tr += F[r][c] * F[r][c];
                }
            const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                             F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                             F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
            const double m = mu[q], l = lam[q];
            acc += (double)vol[q] * (0.5 * m * (tr - 3.0) - m * (J - 1.0) + 0.5 * l * (J - 1.0) * (J - 1.0));
        }
    }
    __shared__ double red[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < kBlock / 32 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) scratch[blockIdx.x] = w;
    }
}

// out[0] = sum of scratch[0..nblocks), in a fixed order.
__global__ void __launch_bounds__(1024) k_ip_total(const double* __restrict__ scratch, int nblocks,
                                                   double* __restrict__ out) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) s += scratch[i];
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) out[0] = w;
    }
}

// Device address of the scratch array on the current device: looked up at the first call on the
// device (set-up), and again at later calls whose stream is not capturing.
int scratch_address(int device, cudaStream_t stream, double** out) {
    if (device < 0 || device >= kMaxDevices) VBD_FAIL(VBD_ERR_NO_DEVICE, "device ordinal %d not supported", device);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    bool lookup = g_scratch_addr[device] == nullptr;
    if (!lookup) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(stream, &cs) == cudaSuccess)
            lookup = cs == cudaStreamCaptureStatusNone;
        else
            cudaGetLastError();  // the failed query's own error is not left for the caller to find
    }
    if (lookup) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            VBD_FAIL(VBD_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
        g_scratch_addr[device] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[device];
    return VBD_OK;
}

}  // namespace

extern "C" int vbd_ip_energy_noalloc(int32_t num_verts, int32_t num_tets, const float* positions, const float* inertia,
                                     const float* vertex_mass, const int32_t* tets, const float* dm_inv,
                                     const float* rest_vol, const float* tet_mu, const float* tet_lambda, float h,
                                     double* out, void* cuda_stream) {
    vbd::clear_error();
    if (num_verts < 0 || num_tets < 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "negative mesh size");
    const long long total = (long long)num_verts + num_tets;
    if (total > kMaxElements)
        VBD_FAIL(VBD_ERR_INVALID_ARG,
                 "num_verts + num_tets = %lld exceeds the no-alloc maximum of %lld (its fixed scratch holds %d "
                 "block partials of %d elements)",
                 total, kMaxElements, kMaxBlocks, kPerBlock);
    if (!out) VBD_FAIL(VBD_ERR_INVALID_ARG, "out is null");
    if (num_verts > 0 && (!positions || !inertia || !vertex_mass))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "positions, inertia and vertex_mass are required");
    if (num_tets > 0 && (!tets || !dm_inv || !rest_vol || !tet_mu || !tet_lambda))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "tets, dm_inv, rest_vol, tet_mu and tet_lambda are required");
    if (!(h > 0.f) || !(h < 3.0e38f)) VBD_FAIL(VBD_ERR_INVALID_ARG, "h must be positive and finite");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) VBD_FAIL(VBD_ERR_NO_DEVICE, "no current CUDA device: %s", cudaGetErrorString(e));
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    double* scratch = nullptr;
    if (int rc = scratch_address(device, stream, &scratch)) return rc;
    const int nblocks = total > 0 ? (int)((total + kPerBlock - 1) / kPerBlock) : 1;
    e = cudaMemsetAsync(scratch + kFlagSlot, 0, sizeof(double), stream);
    if (e != cudaSuccess) VBD_FAIL(VBD_ERR_CUDA, "clearing the scratch flag failed: %s", cudaGetErrorString(e));
    const double inv_h2 = 1.0 / ((double)h * (double)h);
    k_ip_partials<<<nblocks, kBlock, 0, stream>>>(num_verts, num_tets, positions, inertia, vertex_mass, tets, dm_inv,
                                                  rest_vol, tet_mu, tet_lambda, inv_h2, scratch);
    k_ip_total<<<1, 1024, 0, stream>>>(scratch, nblocks, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) VBD_FAIL(VBD_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    double flag = 0.0;
    e = cudaMemcpyAsync(&flag, scratch + kFlagSlot, sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) VBD_FAIL(VBD_ERR_CUDA, "no-alloc energy failed: %s", cudaGetErrorString(e));
    if (flag != 0.0) VBD_FAIL(VBD_ERR_INVALID_ARG, "tets hold vertex ids outside [0, %d); those tets were skipped", num_verts);
    return VBD_OK;
}
