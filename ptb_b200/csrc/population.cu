// Mixed Mulliken/Loewdin population analysis on the density matrix the
// density step produced (source/mlpop.f): mlpop14 (S^(1-x), S^x from an FP32
// eigen-decomposition of S, once per geometry) and mlpop2 (atomic and shell
// populations diag(S^x P S^(1-x)) per SCF iteration).
//
// The reference evaluates mlpop2 in REAL*4 (ssymm + sgemm on nao x nao).  Here
// only the diagonal is formed: C = P S^(1-x) is one int8-sliced product with 6
// slices (42 bits of each row maximum, exact int32 sums: more accurate than the
// REAL*4 original), and X_ii = sum_j s2(i,j) C(j,i) is an HBM-bound tiled dot
// product in FP64.  The per-atom and per-shell sums run on the host in the
// reference's AO order.
#include <cmath>

#include "common.cuh"
#include "oz_gemm.cuh"

namespace ptb {

namespace {

__global__ void k_d2f(int64_t count, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}
__global__ void k_f2d_all(int64_t count, const float* __restrict__ a, double* __restrict__ b) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

// cc(i,m) = X(i,m) * f(m) with f(m) = REAL*4(e(m) ** p) (REAL*4 base promoted, REAL(8) exponent).
__global__ void k_scale_cols(int64_t n, const float* __restrict__ X, const float* __restrict__ w, double p,
                             float* __restrict__ cc) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n * n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = k / n;
        cc[k] = X[k] * (float)pow((double)w[m], p);
    }
}

// xd[i] = sum_j s2(i,j) C(j,i), s2 FP32 and C FP64 column-major (ld n); one
// block per 32 consecutive i, 32 x 32 tiles through shared memory, a fixed
// reduction order.  blockDim = (32, 8).
__global__ void k_diag_s2c(int64_t n, const float* __restrict__ s2, const double* __restrict__ C,
                           double* __restrict__ xd) {
    __shared__ float ts[32][33];    // ts[jj][ii] = s2(i0+ii, j0+jj)
    __shared__ double tc[32][33];   // tc[ii][jj] = C(j0+jj, i0+ii)
    __shared__ double part[8][32];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = (int64_t)blockIdx.x * 32;
    double acc = 0.0;
    for (int64_t j0 = 0; j0 < n; j0 += 32) {
#pragma unroll
        for (int r = 0; r < 32; r += 8) {
            const int64_t i = i0 + tx, j = j0 + ty + r;
            ts[ty + r][tx] = (i < n && j < n) ? s2[i + j * n] : 0.f;
            const int64_t jj = j0 + tx, ii = i0 + ty + r;
            tc[ty + r][tx] = (ii < n && jj < n) ? C[jj + ii * n] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int jj = ty * 4 + q;
            acc += (double)ts[jj][tx] * tc[tx][jj];
        }
        __syncthreads();
    }
    part[ty][tx] = acc;
    __syncthreads();
    if (ty == 0) {
        double s = 0.0;
        for (int r = 0; r < 8; ++r) s += part[r][tx];
        if (i0 + tx < n) xd[i0 + tx] = s;
    }
}

int grid_for(int64_t count) { return (int)std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, 148 * 32)); }

}  // namespace

// s34 = S^(1-x), s14 = S^x (REAL*4, column-major nao x nao) from packed FP64 S, source/mlpop.f:142-190.
void mlpop14_device(ptbgpu_ctx* c, int64_t n, const double* dSpk, double x, float* s34, float* s14) {
    cudaStream_t s = c->stream;
    DevBuf& bd = c->buf(B_W0);
    DevBuf& bx = c->buf(B_MISC0);
    DevBuf& bc = c->buf(B_MISC1);
    DevBuf& bw = c->buf(B_MISC2);
    bd.reserve(sizeof(double) * n * n);
    bx.reserve(sizeof(float) * n * n);
    bc.reserve(sizeof(float) * n * n);
    bw.reserve(sizeof(float) * n);
    float* X = bx.as<float>();
    float* cc = bc.as<float>();
    float* w = bw.as<float>();
    unpack_sym(s, n, n, dSpk, bd.as<double>(), 0.0);   // blowsym84: full symmetric, then REAL*4
    k_d2f<<<grid_for(n * n), 256, 0, s>>>(n * n, bd.as<double>(), X);
    count_launch();
    int lwork = 0;
    PTB_CUSOLVER(cusolverDnSsyevd_bufferSize(c->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, (int)n, X,
                                             (int)n, w, &lwork));
    DevBuf& ws = c->buf(B_SOLVER_WS);
    ws.reserve(sizeof(float) * (size_t)std::max(lwork, 1));
    PTB_CUSOLVER(cusolverDnSsyevd(c->solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, (int)n, X, (int)n, w,
                                  ws.as<float>(), lwork, c->info_dev));
    int info = 0;
    PTB_CUDA(cudaMemcpyAsync(&info, c->info_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    PTB_CHECK(info == 0, PTBGPU_ENOTSPD, "ssyevd of the overlap matrix failed (info=%d)", info);
    const float one = 1.f, zero = 0.f;
    float* outs[2] = {s34, s14};
    const double pw[2] = {1.0 - x, x};
    for (int t = 0; t < 2; ++t) {
        k_scale_cols<<<grid_for(n * n), 256, 0, s>>>(n, X, w, pw[t], cc);
        count_launch();
        PTB_CUBLAS(cublasSgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)n, (int)n, (int)n, &one, X, (int)n, cc, (int)n,
                               &zero, outs[t], (int)n));
    }
    PTB_CUDA(cudaGetLastError());
}

// Populations, source/mlpop.f:198-235: xd(i) = (s2 P s1)(i,i) for packed FP64 P
// and REAL*4 s1 = S^(1-x), s2 = S^x (column-major); xd is a host array of n.
void mlpop2_diag_device(ptbgpu_ctx* c, int64_t n, const double* dPpk, const float* s1, const float* s2, double* xd) {
    cudaStream_t s = c->stream;
    // 4 slices (28 bits of the row maxima) gave errors of ~5e-7 on q after the K
    // and diagonal sums, no better than REAL*4; 6 slices keep them near 1e-10
    constexpr int S = 6;
    PTB_CHECK(oz::padded(n) <= oz::max_k(S), PTBGPU_EINVAL, "nao = %lld too large for exact int32 sums",
              (long long)n);
    DevBuf& bp = c->buf(B_W0);
    DevBuf& b1 = c->buf(B_W1);
    DevBuf& bcm = c->buf(B_W2);
    DevBuf& bxd = c->buf(B_MISC2);
    bp.reserve(sizeof(double) * n * n);
    b1.reserve(sizeof(double) * n * n);
    bcm.reserve(sizeof(double) * n * n);
    bxd.reserve(sizeof(double) * n);
    double* P = bp.as<double>();
    double* S1 = b1.as<double>();
    double* Cm = bcm.as<double>();
    unpack_sym(s, n, n, dPpk, P, 0.0);
    k_f2d_all<<<grid_for(n * n), 256, 0, s>>>(n * n, s1, S1);
    count_launch();
    // C = P s1: rows of P (symmetric) times columns of s1 (row j of the B operand = s1(:, j))
    const int64_t ldp = oz::padded(n);
    DevBuf& bpa = c->buf(B_OZ0);
    DevBuf& bpb = c->buf(B_OZ1);
    DevBuf& bea = c->buf(B_OZE0);
    DevBuf& beb = c->buf(B_OZE1);
    DevBuf& brm = c->buf(B_OZR);
    bpa.reserve((size_t)S * ldp * ldp);
    bpb.reserve((size_t)S * ldp * ldp);
    bea.reserve(sizeof(int) * (size_t)ldp);
    beb.reserve(sizeof(int) * (size_t)ldp);
    brm.reserve(sizeof(unsigned long long) * (size_t)ldp);
    oz::Operand oa, ob;
    oa.planes = bpa.as<int8_t>();
    oa.exps = bea.as<int>();
    ob.planes = bpb.as<int8_t>();
    ob.exps = beb.as<int>();
    oa.ldp = ob.ldp = ldp;
    oa.S = ob.S = S;
    oz::slice(s, P, 1, n, n, oz::TRI_NONE, oa, brm.as<unsigned long long>());
    oz::slice(s, S1, n, 1, n, oz::TRI_NONE, ob, brm.as<unsigned long long>());
    const int variant = oz::resolve_variant(oz::V_DEFAULT, S, 0);
    const std::vector<int4> t = oz::build_tiles(ldp, false, oz::TRI_NONE, oz::TRI_NONE, S, variant);
    DevBuf& bt = c->buf(B_OZT);
    bt.reserve(sizeof(int4) * t.size());
    PTB_CUDA(cudaMemcpyAsync(bt.ptr, t.data(), sizeof(int4) * t.size(), cudaMemcpyHostToDevice, s));
    oz::OzEpi ep;
    ep.err = &c->flags->timeout;
    ep.n = n;
    ep.ldp = ldp;
    ep.out = Cm;   // column-major
    ep.ors = 1;
    ep.ocs = n;
    PTB_CUDA(cudaMemsetAsync(&c->flags->timeout, 0, sizeof(int), s));
    cudaEvent_t e0 = c->take_event(), e1 = c->take_event();
    PTB_CUDA(cudaEventRecord(e0, s));
    oz::product(s, oz::OZ_OUT, oa, ob, bt.as<int4>(), (int)t.size(), ep, 0, variant);
    PTB_CUDA(cudaEventRecord(e1, s));
    c->timed.push_back({2, e0, e1});
    c->oz_ops += oz::tile_ops(t, S, variant);
    k_diag_s2c<<<(unsigned)((n + 31) / 32), dim3(32, 8), 0, s>>>(n, s2, Cm, bxd.as<double>());
    count_launch();
    PTB_CUDA(cudaGetLastError());
    PTB_CUDA(cudaMemcpyAsync(xd, bxd.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    int tmo = 0;
    PTB_CUDA(cudaMemcpyAsync(&tmo, &c->flags->timeout, sizeof(int), cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    PTB_CHECK(tmo == 0, PTBGPU_ETIMEOUT, "int8 product gave up waiting (site %d)", tmo);
}

}  // namespace ptb
