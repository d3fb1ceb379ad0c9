// Electron count and band energy of a packed density matrix without any
// device allocation (ptbgpu_density_traces_noalloc).
//
// Some callers cannot allocate device memory at the point where they want this
// check: a Fortran SCF driver that owns every device buffer through its own
// memory pool, or code that runs while the device is fully committed to the
// matrices of a large box, or inside a latency-critical sequence where the
// implicit device synchronisation of cudaMalloc / cudaFree is not acceptable.
// This entry point needs no library context (creating one allocates) and takes
// device pointers; its only working memory is the fixed array below.
//
// Scratch: kNoAllocMaxDim column partial pairs plus the two results, 1 MB per
// device that loads this code, held until the process exits.  Every call
// writes all slots it later reads, so nothing has to start at zero; calls on
// the same device share the array, so calls whose kernels overlap on the GPU
// (different streams or host threads without ordering) race and must be
// serialised by the caller.
//
// When the array comes into being: the CUDA runtime loads a library's device
// code lazily (CUDA_MODULE_LOADING=LAZY is the default since CUDA 12.2), so
// this file's kernels and the 1 MB array are placed on a device by the first
// call on that device, which looks up the array's address.  A caller that will
// later run with the device full makes its first call early (or runs with
// CUDA_MODULE_LOADING=EAGER, which loads the code when the context is
// created), and makes it before any stream capture.  The address is kept per
// device for the life of the process; a caller that resets a device
// (cudaDeviceReset) discards the loaded code, and later calls on that device
// would use a stale address, so such a caller must not call this entry point
// on that device again.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int64_t kNoAllocMaxDim = 65536;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_traces_scratch[2 * kNoAllocMaxDim + 2];

std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Per packed column j (rows 0..j): sum_i w_ij P_ij S_ij and sum_i w_ij P_ij H_ij,
// w = 1 on the diagonal and 2 off it (the symmetric matrices' two triangles).
__global__ void k_traces_cols(int64_t n, const double* __restrict__ P, const double* __restrict__ S,
                              const double* __restrict__ H, double* __restrict__ part) {
    __shared__ double sh[2][256];
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        const int64_t off = j * (j + 1) / 2;
        double a = 0.0, b = 0.0;
        for (int64_t i = threadIdx.x; i <= j; i += blockDim.x) {
            const double w = (i == j) ? 1.0 : 2.0;
            const double p = P[off + i];
            a += w * p * S[off + i];
            if (H) b += w * p * H[off + i];
        }
        sh[0][threadIdx.x] = a;
        sh[1][threadIdx.x] = b;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) {
                sh[0][threadIdx.x] += sh[0][threadIdx.x + s];
                sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            part[2 * j] = sh[0][0];
            part[2 * j + 1] = sh[1][0];
        }
        __syncthreads();
    }
}

// One block: fixed-order reduction of the n column pairs into part[2n], part[2n+1].
__global__ void k_traces_finish(int64_t n, double* __restrict__ part) {
    __shared__ double sh[2][1024];
    double a = 0.0, b = 0.0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        a += part[2 * j];
        b += part[2 * j + 1];
    }
    sh[0][threadIdx.x] = a;
    sh[1][threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + s];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * n] = sh[0][0];
        part[2 * n + 1] = sh[1][0];
    }
}

void set_msg(char* err, size_t len, const char* fmt, ...) {
    if (!err || len == 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
}

}  // namespace

namespace {

// Makes `device` current for the call and gives the caller's current device
// back on every return path.
struct CurrentDevice {
    int saved = -1;
    cudaError_t set(int device) {
        cudaError_t e = cudaGetDevice(&saved);
        if (e != cudaSuccess) {
            saved = -1;
            return e;
        }
        return saved == device ? cudaSuccess : cudaSetDevice(device);
    }
    ~CurrentDevice() {
        int now = -1;
        if (saved >= 0 && cudaGetDevice(&now) == cudaSuccess && now != saved) cudaSetDevice(saved);
    }
};

}  // namespace

extern "C" int ptbgpu_density_traces_noalloc(int device, int64_t ndim, const double* dPpk, const double* dSpk,
                                             const double* dHpk, double* out, void* stream, char* err,
                                             size_t errlen) {
    set_msg(err, errlen, "%s", "");
    if (!dPpk || !dSpk || !out) {
        set_msg(err, errlen, "null pointer argument");
        return PTBGPU_EINVAL;
    }
    if (ndim <= 0 || ndim > kNoAllocMaxDim) {
        set_msg(err, errlen, "ndim %lld outside 1..%lld, the size of this entry point's fixed scratch array",
                (long long)ndim, (long long)kNoAllocMaxDim);
        return PTBGPU_EINVAL;
    }
    if (device < 0 || device >= kMaxDevices) {
        set_msg(err, errlen, "device %d out of range", device);
        return PTBGPU_EINVAL;
    }
    CurrentDevice cur;
    cudaError_t e = cur.set(device);
    if (e != cudaSuccess) {
        set_msg(err, errlen, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
        return PTBGPU_ECUDA;
    }
    double* scratch = nullptr;
    {
        // first call on a device: the device address of the scratch array (host
        // code only holds a stand-in for the symbol, never a device address)
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch_addr[device]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_traces_scratch);
            if (e != cudaSuccess || p == nullptr) {
                set_msg(err, errlen, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return PTBGPU_ECUDA;
            }
            g_scratch_addr[device] = static_cast<double*>(p);
        }
        scratch = g_scratch_addr[device];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int grid = (int)(ndim < 148 * 8 ? ndim : 148 * 8);
    k_traces_cols<<<grid, 256, 0, s>>>(ndim, dPpk, dSpk, dHpk, scratch);
    k_traces_finish<<<1, 1024, 0, s>>>(ndim, scratch);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch + 2 * ndim, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_msg(err, errlen, "%s", cudaGetErrorString(e));
        return PTBGPU_ECUDA;
    }
    if (!dHpk) out[1] = 0.0;
    return PTBGPU_OK;
}
