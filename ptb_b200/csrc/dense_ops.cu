// Dense FP64 utilities: packed <-> full, filtering, reductions, elementwise
// updates and the library wrappers of the FP64 paths.
//
// Full matrices are column-major (Fortran order, like the reference) with a
// leading dimension ld: element (row i, col j) lives at a[i + j*ld].
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "sm_eig.cuh"

namespace ptb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum; every thread gets the result.
__device__ double block_sum(double v) {
    __shared__ double sh[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
    if (w == 0) v = warp_sum(v);
    if (threadIdx.x == 0) sh[0] = v;
    __syncthreads();
    v = sh[0];
    __syncthreads();
    return v;
}
__device__ double block_max(double v) {
    __shared__ double sh[32];
    v = warp_max(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : -INFINITY;
    if (w == 0) v = warp_max(v);
    if (threadIdx.x == 0) sh[0] = v;
    __syncthreads();
    v = sh[0];
    __syncthreads();
    return v;
}

// Packed column j holds rows 0..j at offset j(j+1)/2.  One 32x32 tile pair per
// block (upper tiles only): the packed reads and the direct upper writes are
// coalesced along rows; the mirrored lower writes go through a shared-memory
// transpose so they are coalesced too.  blockDim = (32, 8).
__global__ void k_unpack(int64_t n, int64_t ld, const double* __restrict__ pk, double* __restrict__ a,
                         double filter) {
    __shared__ double t[32][33];
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = bi * 32, j0 = bj * 32;
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        int64_t i = i0 + tx, j = j0 + ty + k;
        double v = 0.0;
        if (i < n && j < n && i <= j) {
            v = pk[j * (j + 1) / 2 + i];
            if (fabs(v) < filter) v = 0.0;
            a[i + j * ld] = v;
        }
        t[ty + k][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        int64_t j = j0 + tx, i = i0 + ty + k;
        if (i < n && j < n && i < j) a[j + i * ld] = t[tx][ty + k];
    }
}

__global__ void k_pack(int64_t n, int64_t ld, const double* __restrict__ a, double* __restrict__ pk) {
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        double* col = pk + j * (j + 1) / 2;
        for (int64_t i = threadIdx.x; i <= j; i += blockDim.x) col[i] = a[i + j * ld];
    }
}

__global__ void k_filter(int64_t count, double* __restrict__ pk, double filter) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x)
        if (fabs(pk[k]) < filter) pk[k] = 0.0;
}

__global__ void k_set_identity(int64_t n, int64_t ld, double* a, double diag) {
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x)
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) a[i + j * ld] = (i == j) ? diag : 0.0;
}

// Per column j of a symmetric matrix: centre a_jj and radius sum_{i!=j}|a_ij|.
__global__ void k_gershgorin(int64_t n, int64_t ld, const double* __restrict__ a, double* out_lo,
                             double* out_hi) {
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        double r = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) r += fabs(a[i + j * ld]);
        r = block_sum(r);
        double c = a[j + j * ld];
        r -= fabs(c);
        lo = fmin(lo, c - r);
        hi = fmax(hi, c + r);
    }
    if (threadIdx.x == 0) {
        out_lo[blockIdx.x] = lo;
        out_hi[blockIdx.x] = hi;
    }
}

__global__ void k_colabs(int64_t n, int64_t ld, const double* __restrict__ a, double* out) {
    double m = 0.0;
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        double r = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) r += fabs(a[i + j * ld]);
        m = fmax(m, block_sum(r));
    }
    if (threadIdx.x == 0) out[blockIdx.x] = m;
}

// Row abs-sums: thread per row, loop over columns (coalesced across threads).
__global__ void k_rowabs(int64_t n, int64_t ld, const double* __restrict__ a, double* out) {
    double m = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double r = 0.0;
        for (int64_t j = 0; j < n; ++j) r += fabs(a[i + j * ld]);
        m = fmax(m, r);
    }
    m = block_max(m);
    if (threadIdx.x == 0) out[blockIdx.x] = m;
}

// Partial sums of f(x_k) over a strided 2-D block (n x n, leading dim ld).
template <int OP>
__global__ void k_reduce2d(int64_t n, int64_t ld, const double* __restrict__ a,
                           const double* __restrict__ b, double* out) {
    double s = 0.0;
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            double x = a[i + j * ld];
            if (OP == 0) s += x * x;                  // sum of squares
            else if (OP == 1) s += x * b[j + i * ld]; // tr(AB) = sum a_ij b_ji
        }
    }
    s = block_sum(s);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// Partial sums over a flat array: OP 0 sum, 1 dot(a,b), 2 NaN count
template <int OP>
__global__ void k_reduce1d(int64_t count, const double* __restrict__ a, const double* __restrict__ b,
                           double* out) {
    double s = 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x) {
        double x = a[k];
        if (OP == 0) s += x;
        else if (OP == 1) s += x * b[k];
        else if (OP == 2) s += (x != x) ? 1.0 : 0.0;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__global__ void k_trace(int64_t n, int64_t ld, const double* __restrict__ a, double* out) {
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        s += a[i + i * ld];
    s = block_sum(s);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__global__ void k_axpby_diag(int64_t n, int64_t ld, double alpha, const double* __restrict__ x,
                             double beta, double* __restrict__ y, double gamma) {
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x)
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            double v = alpha * (x ? x[i + j * ld] : 0.0) + beta * y[i + j * ld];
            if (i == j) v += gamma;
            y[i + j * ld] = v;
        }
}

// Copy the upper triangle (row i < col j) onto the lower one, 32x32 tiles
// through shared memory so reads and writes are both coalesced.  blockDim = (32, 8).
__global__ void k_symmetrize(int64_t n, int64_t ld, double* a) {
    __shared__ double t[32][33];
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = bi * 32, j0 = bj * 32;
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        int64_t i = i0 + tx, j = j0 + ty + k;
        t[ty + k][tx] = (i < n && j < n && i < j) ? a[i + j * ld] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        int64_t j = j0 + tx, i = i0 + ty + k;
        if (i < n && j < n && i < j) a[j + i * ld] = t[tx][ty + k];
    }
}

__global__ void k_copy(int64_t n, int64_t lds, const double* __restrict__ s, int64_t ldd,
                       double* __restrict__ d) {
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x)
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) d[i + j * ldd] = s[i + j * lds];
}

// FP64 -> FP32 copy plus the bf16 hi/lo split (hi = bf16(x), lo = bf16(x - hi)),
// written into a zero-padded ldp x ldp layout.
__global__ void k_d2f_split(int64_t n, int64_t ldp, const double* __restrict__ x, float* __restrict__ xf,
                            __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
    for (int64_t j = blockIdx.x; j < ldp; j += gridDim.x)
        for (int64_t i = threadIdx.x; i < ldp; i += blockDim.x) {
            float v = (i < n && j < n) ? (float)x[i + j * n] : 0.0f;
            int64_t k = i + j * ldp;
            if (xf) xf[k] = v;
            __nv_bfloat16 h = __float2bfloat16_rn(v);
            hi[k] = h;
            if (lo) lo[k] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
}

// Third split plane: mid = bf16(x - hi), lo = bf16(x - hi - mid) from the FP32 copy.
__global__ void k_split3(int64_t count, const float* __restrict__ xf, const __nv_bfloat16* __restrict__ hi,
                         __nv_bfloat16* __restrict__ mid, __nv_bfloat16* __restrict__ lo) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count;
         k += (int64_t)gridDim.x * blockDim.x) {
        const float r = xf[k] - __bfloat162float(hi[k]);
        const __nv_bfloat16 m = __float2bfloat16_rn(r);
        mid[k] = m;
        lo[k] = __float2bfloat16_rn(r - __bfloat162float(m));
    }
}

int grid_for(int64_t work, int per = kThreads) {
    int64_t g = (work + per - 1) / per;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

double host_reduce(ptbgpu_ctx* c, const double* dpart, int nb, bool is_max) {
    std::vector<double> h(nb);
    PTB_CUDA(cudaMemcpyAsync(h.data(), dpart, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PTB_CUDA(cudaStreamSynchronize(c->stream));
    double r = is_max ? -INFINITY : 0.0;
    for (double v : h) r = is_max ? std::max(r, v) : r + v;
    return r;
}

double* partials(ptbgpu_ctx* c, int nb) {
    DevBuf& b = c->buf(B_MISC3);
    b.reserve(2 * sizeof(double) * (size_t)nb);
    return b.as<double>();
}

}  // namespace

void unpack_sym(cudaStream_t s, int64_t n, int64_t ld, const double* pk, double* full, double filter) {
    unsigned nb = (unsigned)((n + 31) / 32);
    k_unpack<<<dim3(nb, nb), dim3(32, 8), 0, s>>>(n, ld, pk, full, filter);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

void pack_cols(cudaStream_t s, int64_t n, int64_t ld, const double* full, double* pk) {
    k_pack<<<grid_for(n, 1), kThreads, 0, s>>>(n, ld, full, pk);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

void filter_packed(cudaStream_t s, int64_t n, double* pk, double filter) {
    int64_t cnt = npacked(n);
    k_filter<<<grid_for(cnt), kThreads, 0, s>>>(cnt, pk, filter);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

void set_identity(cudaStream_t s, int64_t n, int64_t ld, double* a, double diag) {
    k_set_identity<<<grid_for(n, 1), kThreads, 0, s>>>(n, ld, a, diag);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

void gershgorin_bounds(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a, double* emin, double* emax) {
    int nb = grid_for(n, 1);
    double* p = partials(c, nb);
    k_gershgorin<<<nb, kThreads, 0, c->stream>>>(n, ld, a, p, p + nb);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    std::vector<double> h(2 * nb);
    PTB_CUDA(cudaMemcpyAsync(h.data(), p, 2 * nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PTB_CUDA(cudaStreamSynchronize(c->stream));
    double lo = INFINITY, hi = -INFINITY;
    for (int b = 0; b < nb; ++b) {
        lo = std::min(lo, h[b]);
        hi = std::max(hi, h[nb + b]);
    }
    *emin = lo;
    *emax = hi;
}

double trace_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a) {
    int nb = std::min(grid_for(n), 64);
    double* p = partials(c, nb);
    k_trace<<<nb, kThreads, 0, c->stream>>>(n, ld, a, p);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return host_reduce(c, p, nb, false);
}

double frob_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a) {
    int nb = grid_for(n, 1);
    double* p = partials(c, nb);
    k_reduce2d<0><<<nb, kThreads, 0, c->stream>>>(n, ld, a, nullptr, p);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return std::sqrt(host_reduce(c, p, nb, false));
}

// Sum of nb partials in index order (as host_reduce), optionally its square
// root, into a device scalar; or the OR of "sum > 0" into a device flag.
__global__ void k_sum_partials(const double* __restrict__ p, int nb, double* __restrict__ out, int mode) {
    double r = 0.0;
    for (int i = 0; i < nb; ++i) r = r + p[i];
    if (mode == 0) *out = sqrt(r);
    else if (mode == 1) *out = r;
    else if (r > 0.0) *reinterpret_cast<int*>(out) = 1;
}

void frob_to_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a, double* out) {
    int nb = grid_for(n, 1);
    double* p = partials(c, nb);
    k_reduce2d<0><<<nb, kThreads, 0, c->stream>>>(n, ld, a, nullptr, p);
    k_sum_partials<<<1, 1, 0, c->stream>>>(p, nb, out, 0);
    count_launch(2);
    PTB_CUDA(cudaGetLastError());
}

void nan_flag_dev(ptbgpu_ctx* c, int64_t count, const double* a, int* flag) {
    int nb = grid_for(count);
    double* p = partials(c, nb);
    k_reduce1d<2><<<nb, kThreads, 0, c->stream>>>(count, a, nullptr, p);
    k_sum_partials<<<1, 1, 0, c->stream>>>(p, nb, reinterpret_cast<double*>(flag), 2);
    count_launch(2);
    PTB_CUDA(cudaGetLastError());
}

double trace_prod_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a, const double* b) {
    int nb = grid_for(n, 1);
    double* p = partials(c, nb);
    k_reduce2d<1><<<nb, kThreads, 0, c->stream>>>(n, ld, a, b, p);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return host_reduce(c, p, nb, false);
}

double dot_dev(ptbgpu_ctx* c, int64_t count, const double* a, const double* b) {
    int nb = grid_for(count);
    double* p = partials(c, nb);
    k_reduce1d<1><<<nb, kThreads, 0, c->stream>>>(count, a, b, p);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return host_reduce(c, p, nb, false);
}

double sum_dev(ptbgpu_ctx* c, int64_t count, const double* a) {
    int nb = grid_for(count);
    double* p = partials(c, nb);
    k_reduce1d<0><<<nb, kThreads, 0, c->stream>>>(count, a, nullptr, p);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return host_reduce(c, p, nb, false);
}

bool has_nan_dev(ptbgpu_ctx* c, int64_t count, const double* a) {
    int nb = grid_for(count);
    double* p = partials(c, nb);
    k_reduce1d<2><<<nb, kThreads, 0, c->stream>>>(count, a, nullptr, p);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return host_reduce(c, p, nb, false) > 0.0;
}

double colabs_max_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a) {
    int nb = grid_for(n, 1);
    double* p = partials(c, nb);
    k_colabs<<<nb, kThreads, 0, c->stream>>>(n, ld, a, p);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return host_reduce(c, p, nb, true);
}

double rowabs_max_dev(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* a) {
    int nb = grid_for(n);
    double* p = partials(c, nb);
    k_rowabs<<<nb, kThreads, 0, c->stream>>>(n, ld, a, p);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    return host_reduce(c, p, nb, true);
}

void axpby_diag(cudaStream_t s, int64_t n, int64_t ld, double alpha, const double* x, double beta,
                double* y, double gamma) {
    k_axpby_diag<<<grid_for(n, 1), kThreads, 0, s>>>(n, ld, alpha, x, beta, y, gamma);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

void symmetrize_upper(cudaStream_t s, int64_t n, int64_t ld, double* a) {
    unsigned nb = (unsigned)((n + 31) / 32);
    k_symmetrize<<<dim3(nb, nb), dim3(32, 8), 0, s>>>(n, ld, a);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

void copy_mat(cudaStream_t s, int64_t n, int64_t lds, const double* src, int64_t ldd, double* dst) {
    k_copy<<<grid_for(n, 1), kThreads, 0, s>>>(n, lds, src, ldd, dst);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

void d2f_split(cudaStream_t s, int64_t n, int64_t ldp, const double* x, float* xf, void* hi, void* lo) {
    k_d2f_split<<<grid_for(ldp, 1), kThreads, 0, s>>>(n, ldp, x, xf, (__nv_bfloat16*)hi,
                                                     (__nv_bfloat16*)lo);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

void d2f_split3(cudaStream_t s, int64_t ldp, const float* xf, const void* hi, void* mid, void* lo) {
    const int64_t cnt = ldp * ldp;
    k_split3<<<grid_for(cnt), kThreads, 0, s>>>(cnt, xf, (const __nv_bfloat16*)hi, (__nv_bfloat16*)mid,
                                                (__nv_bfloat16*)lo);
    count_launch();
    PTB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// library wrappers (column-major)
// ---------------------------------------------------------------------------
void dgemm_nn(ptbgpu_ctx* c, int64_t n, int64_t ld, double alpha, const double* A, const double* B,
              double beta, double* C) {
    PTB_CUBLAS(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)n, (int)n, &alpha, A, (int)ld,
                           B, (int)ld, &beta, C, (int)ld));
}

void dsyrk_sq(ptbgpu_ctx* c, int64_t n, int64_t ld, const double* X, double* C) {
    const double one = 1.0, zero = 0.0;
    // C(upper) = X X^T = X X for symmetric X; then mirror to the lower triangle.
    PTB_CUBLAS(cublasDsyrk(c->blas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, (int)n, (int)n, &one, X, (int)ld,
                           &zero, C, (int)ld));
    symmetrize_upper(c->stream, n, ld, C);
}

int dpotrf_lower(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A) {
    int lwork = 0;
    PTB_CUSOLVER(cusolverDnDpotrf_bufferSize(c->solver, CUBLAS_FILL_MODE_LOWER, (int)n, A, (int)ld, &lwork));
    DevBuf& ws = c->buf(B_SOLVER_WS);
    ws.reserve(sizeof(double) * (size_t)std::max(lwork, 1));
    PTB_CUSOLVER(cusolverDnDpotrf(c->solver, CUBLAS_FILL_MODE_LOWER, (int)n, A, (int)ld, ws.as<double>(),
                                  lwork, c->info_dev));
    int info = 0;
    PTB_CUDA(cudaMemcpyAsync(&info, c->info_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PTB_CUDA(cudaStreamSynchronize(c->stream));
    return info;
}

namespace {
// cuSOLVER trtri on one diagonal block (lower, in place).
void trtri_block(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A) {
    size_t wd = 0, wh = 0;
    PTB_CUSOLVER(cusolverDnXtrtri_bufferSize(c->solver, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_NON_UNIT, n, CUDA_R_64F,
                                             A, ld, &wd, &wh));
    DevBuf& ws = c->buf(B_SOLVER_WS);
    ws.reserve(std::max<size_t>(wd, 8));
    std::vector<char> hw(std::max<size_t>(wh, 8));
    PTB_CUSOLVER(cusolverDnXtrtri(c->solver, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_NON_UNIT, n, CUDA_R_64F, A, ld,
                                  ws.ptr, wd, hw.data(), wh, c->info_dev));
    int info = 0;
    PTB_CUDA(cudaMemcpyAsync(&info, c->info_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PTB_CUDA(cudaStreamSynchronize(c->stream));
    PTB_CHECK(info == 0, PTBGPU_ENOTSPD, "triangular inverse failed (trtri info=%d)", info);
}

// Recursive halving: for L = [L11 0; L21 L22], L^-1 = [L11^-1 0; -L22^-1 L21 L11^-1  L22^-1].
// The off-diagonal block takes two triangular products (cuBLAS trmm, in place),
// so the n^3/3 flops run at product speed; blocks of <= 512 go to cuSOLVER.
void trtri_rec(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A) {
    if (n <= 512) {
        trtri_block(c, n, ld, A);
        return;
    }
    const int64_t n1 = (n / 2 + 127) / 128 * 128, n2 = n - n1;
    double* L11 = A;
    double* L21 = A + n1;
    double* L22 = A + n1 + n1 * ld;
    trtri_rec(c, n1, ld, L11);
    trtri_rec(c, n2, ld, L22);
    const double one = 1.0, mone = -1.0;
    PTB_CUBLAS(cublasDtrmm(c->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                           (int)n2, (int)n1, &one, L11, (int)ld, L21, (int)ld, L21, (int)ld));
    PTB_CUBLAS(cublasDtrmm(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                           (int)n2, (int)n1, &mone, L22, (int)ld, L21, (int)ld, L21, (int)ld));
}
}  // namespace

// In-place inverse of the lower triangle of A (column-major); the strict upper
// triangle is not referenced.
void dtrtri_lower(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A) { trtri_rec(c, n, ld, A); }

// All eigenpairs of a symmetric matrix (upper triangle read, eigenvectors over
// A, w ascending): the library's eigensolver up to order kEigLargeMax, cuSOLVER
// above it.
void dsyevd(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A, double* w) {
    if (n <= kEigLargeMax && ld == n) {
        eig_full_upper(c, n, A, nullptr, w);
        return;
    }
    int lwork = 0;
    PTB_CUSOLVER(cusolverDnDsyevd_bufferSize(c->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER,
                                             (int)n, A, (int)ld, w, &lwork));
    DevBuf& ws = c->buf(B_SOLVER_WS);
    ws.reserve(sizeof(double) * (size_t)std::max(lwork, 1));
    PTB_CUSOLVER(cusolverDnDsyevd(c->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, (int)n, A,
                                  (int)ld, w, ws.as<double>(), lwork, c->info_dev));
    int info = 0;
    PTB_CUDA(cudaMemcpyAsync(&info, c->info_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PTB_CUDA(cudaStreamSynchronize(c->stream));
    PTB_CHECK(info == 0, PTBGPU_ECUDA, "dsyevd info=%d", info);
}

// H U = S U diag(w) (upper triangles read, U over A with U^T S U = I, w
// ascending): the library's eigensolver up to order kEigLargeMax, cuSOLVER above
// it.  Returns 0, or n + the order of S's first non-positive leading minor.
int dsygvd(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A, double* B, double* w) {
    if (n <= kEigLargeMax && ld == n) {
        try {
            eig_full_upper(c, n, A, B, w);
        } catch (const Error& e) {
            if (e.code != PTBGPU_ENOTSPD) throw;
            return (int)n + 1;
        }
        return 0;
    }
    int lwork = 0;
    PTB_CUSOLVER(cusolverDnDsygvd_bufferSize(c->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                             CUBLAS_FILL_MODE_UPPER, (int)n, A, (int)ld, B, (int)ld, w,
                                             &lwork));
    DevBuf& ws = c->buf(B_SOLVER_WS);
    ws.reserve(sizeof(double) * (size_t)std::max(lwork, 1));
    PTB_CUSOLVER(cusolverDnDsygvd(c->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                  CUBLAS_FILL_MODE_UPPER, (int)n, A, (int)ld, B, (int)ld, w,
                                  ws.as<double>(), lwork, c->info_dev));
    int info = 0;
    PTB_CUDA(cudaMemcpyAsync(&info, c->info_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PTB_CUDA(cudaStreamSynchronize(c->stream));
    return info;
}

EventTimer::EventTimer(cudaStream_t st) : s(st) {
    PTB_CUDA(cudaEventCreate(&a));
    PTB_CUDA(cudaEventCreate(&b));
}
EventTimer::~EventTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
}
void EventTimer::start() { PTB_CUDA(cudaEventRecord(a, s)); }
float EventTimer::stop_ms() {
    PTB_CUDA(cudaEventRecord(b, s));
    PTB_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    PTB_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

}  // namespace ptb
