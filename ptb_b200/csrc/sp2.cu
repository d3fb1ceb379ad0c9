// Trace-correcting (SP2) purification of the dense density-matrix step.
//
// Both precisions share the orthogonalisation: S = L L^T (Cholesky),
// A = L^-1 H L^-T, Gershgorin bounds [e_min, e_max] of A,
// X_0 = (e_max I - A) / (e_max - e_min), and at the end P = 2 L^-T X L^-1.
// Each SP2 step maps X -> X^2 or X -> 2X - X^2, whichever lands tr X closer
// to N = nel/2 (tr X^2 = ||X||_F^2 for symmetric X is known before the
// product, so the branch is decided first).
//
// PTBGPU_PREC_FP64: every product is an FP64 SYRK (the comparator path).
//
// PTBGPU_PREC_MIXED:
//   pass 1   SP2 products on the tcgen05 kernel with bf16x3 operands and FP32
//            accumulation; the epilogue applies the branch, writes the next
//            iterate (FP32 + bf16 hi/lo planes, kept for every step: the
//            trajectory) and per-tile trace / sum-of-squares partials; a
//            one-block kernel reduces them and decides the next branch and
//            convergence on the device.
//   cleanup  a few FP64 SP2 steps make the pass-1 result P~ idempotent to
//            rounding (its subspace still carries the bf16x3 error).
//   refine   first-order density-matrix perturbation theory around P~: with
//            C = [A, P~] (one FP64 product) the off-diagonal part of A in the
//            P~ basis is A1 = [C, P~] (small, so a bf16x3 product suffices);
//            its response is propagated through the recorded branch sequence
//            over the stored trajectory, X1 <- X0_k X1 + X1 X0_k (or
//            2 X1 - (...)), again with bf16x3 products; P = P~ + X1.
//            The error left is second order in the pass-1 error.
//
// The FP64 products of the mixed path (A = L^-1 H L^-T through the explicit
// triangular inverse, the cleanup squares, the commutator and the
// back-transform) run on the int8 tensor cores with 7-bit operand slices and
// exact int32 sums (oz_gemm.cu) when opts->fp64_slices is 6..8; with 0 they are
// cuBLAS/cuSOLVER FP64 calls, as in the FP64 path.
#include <cuda_bf16.h>

#include <algorithm>
#include <map>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "oz_gemm.cuh"
#include "sp2_state.cuh"
#include "tc_gemm.cuh"

namespace ptb {

namespace {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// X_0 = (e_max I - A)/(e_max - e_min) from column-major FP64 A (n x n), into
// zero-padded FP32 / bf16 hi / bf16 lo planes (ldp x ldp); per-block partials
// of tr X_0 and ||X_0||^2 into stats[2*block].
__global__ void k_x0_init(int64_t n, int64_t ldp, const double* __restrict__ A, double emax, double scale,
                          float* __restrict__ xf, __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ mid,
                          __nv_bfloat16* __restrict__ lo, double* __restrict__ stats) {
    double tr = 0.0, ss = 0.0;
    for (int64_t j = blockIdx.x; j < ldp; j += gridDim.x) {
        for (int64_t i = threadIdx.x; i < ldp; i += blockDim.x) {
            float v = 0.0f;
            if (i < n && j < n) {
                double d = ((i == j) ? emax : 0.0) - A[i + j * n];
                v = (float)(d * scale);
            }
            const int64_t k = i + j * ldp;
            xf[k] = v;
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            const float r = v - __bfloat162float(h);
            const __nv_bfloat16 m = __float2bfloat16_rn(r);
            hi[k] = h;
            mid[k] = m;
            if (lo) lo[k] = __float2bfloat16_rn(r - __bfloat162float(m));
            const double dv = v;
            if (i == j) tr += dv;
            ss += dv * dv;
        }
    }
    __shared__ double sh[2][32];
    tr = warp_sum(tr);
    ss = warp_sum(ss);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[0][w] = tr;
        sh[1][w] = ss;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
            a += sh[0][q];
            b += sh[1][q];
        }
        stats[2 * blockIdx.x] = a;
        stats[2 * blockIdx.x + 1] = b;
    }
}

// Reduce the partials of iterate k in a fixed order and decide the next step.
__global__ void k_decide(SP2State* st, const double* __restrict__ stats, int nparts, double N, double tol_abs,
                         double e_asym, double e_stag, int maxit) {
    if (!st->active) return;
    __shared__ double sh[2][256];
    double a = 0.0, b = 0.0;
    for (int p = threadIdx.x; p < nparts; p += blockDim.x) {
        a += stats[2 * p];
        b += stats[2 * p + 1];
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
    if (threadIdx.x != 0) return;
    sp2_decide(st, sh[0][0], sh[1][0], N, tol_abs, e_asym, e_stag, maxit);
}

// out(i,j) = alpha (W_ij + W_ji) + beta X_ij over the ldp x ldp FP32 planes
// (row-major W), 32x32 tile pairs through shared memory; also writes the bf16
// hi/lo planes of the result.  blockDim = (32, 8).
__global__ void k_sym_update(int64_t ldp, const float* __restrict__ W, const float* __restrict__ X, float alpha,
                             float beta, float* __restrict__ out, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo) {
    __shared__ float t[32][33];
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = bi * 32, j0 = bj * 32;
    // stage W(j-block rows, i-block cols) transposed: t[c][r] = W[j0 + r][i0 + c]
#pragma unroll
    for (int k = 0; k < 32; k += 8) t[tx][ty + k] = W[(j0 + ty + k) * ldp + i0 + tx];
    __syncthreads();
    // element (i, j) = (i0 + ty + k, j0 + tx): W[i][j] + W[j][i]; on a diagonal
    // tile only the upper triangle is computed here and mirrored below, so the
    // result is exactly symmetric even when X is not
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int64_t i = i0 + ty + k, j = j0 + tx;
        const float s = W[i * ldp + j] + t[ty + k][tx];
        const float v = alpha * s + (beta != 0.0f ? beta * X[i * ldp + j] : 0.0f);
        if (bi != bj || i <= j) {
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
            out[i * ldp + j] = v;
            hi[i * ldp + j] = h;
            lo[i * ldp + j] = l;
        }
        t[ty + k][tx] = v;   // each thread rewrites only the slot it read
    }
    __syncthreads();
    // mirrored tile: element (j, i) with j = j0 + ty + k, i = i0 + tx (strictly
    // below the diagonal on a diagonal tile)
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int64_t j = j0 + ty + k, i = i0 + tx;
        if (bi == bj && j <= i) continue;
        const float v = t[tx][ty + k];
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        out[j * ldp + i] = v;
        hi[j * ldp + i] = h;
        lo[j * ldp + i] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// FP32 plane (ldp) -> FP64 column-major n x n, optionally added to y: y = a*x + b*y
__global__ void k_f2d(int64_t n, int64_t ldp, const float* __restrict__ x, double a, double b,
                      double* __restrict__ y) {
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x)
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const double v = a * (double)x[i + j * ldp];
            y[i + j * n] = (b == 0.0) ? v : v + b * y[i + j * n];
        }
}

// bf16 hi/lo planes of an FP32 plane.
__global__ void k_split2(int64_t count, const float* __restrict__ x, __nv_bfloat16* __restrict__ hi,
                         __nv_bfloat16* __restrict__ lo) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
        const __nv_bfloat16 h = __float2bfloat16_rn(x[k]);
        hi[k] = h;
        lo[k] = __float2bfloat16_rn(x[k] - __bfloat162float(h));
    }
}

// y += x over FP32 planes.
__global__ void k_add_f32(int64_t count, const float* __restrict__ x, float* __restrict__ y) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x)
        y[k] += x[k];
}

// Per-block partials of the trace and of max |x_ij| over the leading n x n
// block of a row-major FP32 ldp x ldp matrix: out[2b] = trace, out[2b+1] = max.
__global__ void k_trace_maxabs_f32(int64_t n, int64_t ldp, const float* __restrict__ x, double* __restrict__ out) {
    __shared__ double st[256], sm[256];
    double t = 0.0;
    float m = 0.0f;
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const float* row = x + i * ldp;
        for (int64_t j = threadIdx.x; j < n; j += blockDim.x) m = fmaxf(m, fabsf(row[j]));
        if (threadIdx.x == 0) t += (double)row[i];
    }
    st[threadIdx.x] = t;
    sm[threadIdx.x] = (double)m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            st[threadIdx.x] += st[threadIdx.x + w];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[2 * blockIdx.x] = st[0];
        out[2 * blockIdx.x + 1] = sm[0];
    }
}

// C = W - W^T (column-major FP64), 32x32 tiles.  blockDim = (32, 8).
__global__ void k_antisym(int64_t n, const double* __restrict__ W, double* __restrict__ C) {
    __shared__ double t[32][33];
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = bi * 32, j0 = bj * 32;
    // t[c][r] = W(j0 + c, i0 + r)  (i.e. W^T entries)
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int64_t row = j0 + tx, col = i0 + ty + k;
        t[tx][ty + k] = (row < n && col < n) ? W[row + col * n] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int64_t row = i0 + tx, col = j0 + ty + k;
        if (row < n && col < n) C[row + col * n] = W[row + col * n] - t[ty + k][tx];
    }
}

int grid1(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(n, 148 * 16)); }

// A tensor-core product bracketed by CUDA events on the launching stream; the
// C-ABI layer sums the elapsed times per kind into the call's stats.
// Returns the number of per-CTA stats partials the launch wrote.
int timed_product(ptbgpu_ctx* c, int epi, int np, int64_t ldp, const void* const* pa, const void* const* pb,
                  const tc::ProdList& prods, const int2* tiles, int ntiles, const tc::EpiParams& ep, int kblock = 0,
                  const int2* pairs = nullptr, int npairs = 0) {
    cudaEvent_t a = c->take_event(), b = c->take_event();
    PTB_CUDA(cudaEventRecord(a, c->stream));
    const int parts = tc::launch_product(c->stream, epi, np, ldp, pa, pb, prods, tiles, ntiles, ep, kblock, pairs,
                                         npairs);
    PTB_CUDA(cudaEventRecord(b, c->stream));
    c->timed.push_back({epi == tc::EPI_SP2 ? 0 : 1, a, b});
    return parts;
}

// Device-time phase log of one purification call (print level >= 2): CUDA
// events on the context stream between phases, reported when the call ends.
struct PhaseLog {
    ptbgpu_ctx* c = nullptr;
    std::vector<std::pair<const char*, cudaEvent_t>> marks;
    void add(const char* what) {
        cudaEvent_t e = c->take_event();
        PTB_CUDA(cudaEventRecord(e, c->stream));
        marks.push_back({what, e});
    }
    void report(int prl) {
        if (marks.size() < 2) return;
        PTB_CUDA(cudaEventSynchronize(marks.back().second));
        for (size_t i = 1; i < marks.size(); ++i) {
            float ms = 0.f;
            PTB_CUDA(cudaEventElapsedTime(&ms, marks[i - 1].second, marks[i].second));
            log_line(prl, 2, " * purification %-34s %9.3f ms", marks[i].first, ms);
        }
    }
};
thread_local PhaseLog* t_phases = nullptr;   // set for the duration of a call at print level >= 2
void phase(const char* what) {
    if (t_phases) t_phases->add(what);
}

// ---------------------------------------------------------------------------
// FP64 products on the int8 tensor cores (oz_gemm.cu): context-held operands
// ---------------------------------------------------------------------------
oz::Operand oz_operand(ptbgpu_ctx* c, int slot, int64_t n, int S) {
    const int64_t ldp = oz::padded(n);
    DevBuf& bp = c->buf(B_OZ0 + slot);
    DevBuf& be = c->buf(B_OZE0 + slot);
    bp.reserve((size_t)S * ldp * ldp);
    be.reserve(sizeof(int) * (size_t)ldp);
    oz::Operand op;
    op.planes = bp.as<int8_t>();
    op.exps = be.as<int>();
    op.ldp = ldp;
    op.S = S;
    return op;
}

void oz_slice(ptbgpu_ctx* c, const double* M, int64_t rs, int64_t cs, int64_t n, int tri, const oz::Operand& op) {
    DevBuf& br = c->buf(B_OZR);
    br.reserve(sizeof(unsigned long long) * (size_t)op.ldp);
    oz::slice(c->stream, M, rs, cs, n, tri, op, br.as<unsigned long long>());
}

// One product over a freshly uploaded tile list, bracketed by CUDA events.
// Returns the CTA count (the number of per-CTA stats of OZ_SYM).
int oz_product(ptbgpu_ctx* c, int epi, const oz::Operand& a, const oz::Operand& b, bool upper, int tri_a,
               int tri_b, oz::OzEpi ep, int rb = 0, int variant = oz::V_DEFAULT) {
    variant = oz::resolve_variant(variant, a.S, rb);
    const std::vector<int4> t = oz::build_tiles(a.ldp, upper, tri_a, tri_b, a.S, variant);
    DevBuf& bt = c->buf(B_OZT);
    bt.reserve(sizeof(int4) * t.size());
    PTB_CUDA(cudaMemcpyAsync(bt.ptr, t.data(), sizeof(int4) * t.size(), cudaMemcpyHostToDevice, c->stream));
    ep.ldp = a.ldp;
    if (!ep.err) ep.err = &c->flags->timeout;
    c->oz_ops += oz::tile_ops(t, a.S, variant);
    cudaEvent_t e0 = c->take_event(), e1 = c->take_event();
    PTB_CUDA(cudaEventRecord(e0, c->stream));
    oz::product(c->stream, epi, a, b, bt.as<int4>(), (int)t.size(), ep, rb, variant);
    PTB_CUDA(cudaEventRecord(e1, c->stream));
    c->timed.push_back({2, e0, e1});
    return oz::grid_ctas((int)t.size(), variant);
}

// Slices of the orthogonalisation products: one fewer than the cleanup squares
// (whose errors the SP2 map feeds back and which set the idempotency floor) and
// the back-transform (which sets tr(PS) directly); an error of A moves the
// problem, not the electron count, and 7 slices keep ~2^-49 of the row maxima.
int slices_once(int S) { return std::max(6, S - 1); }

void check_timeout(ptbgpu_ctx* c, const char* what) {
    int tmo = 0;
    PTB_CUDA(cudaMemcpyAsync(&tmo, &c->flags->timeout, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PTB_CUDA(cudaStreamSynchronize(c->stream));
    PTB_CHECK(tmo == 0, PTBGPU_ETIMEOUT, "%s gave up waiting (site %d)", what, tmo);
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
struct Prologue {
    double emin, emax;
};

// H (packed) -> A = L^-1 H L^-T in B_H; S (packed) -> L in B_S.  Both column-major, ld = n.
Prologue orthogonalise(ptbgpu_ctx* c, int64_t n, const double* dHpk, const double* dSpk, double filter) {
    DevBuf& bh = c->buf(B_H);
    DevBuf& bs = c->buf(B_S);
    bh.reserve(sizeof(double) * n * n);
    bs.reserve(sizeof(double) * n * n);
    double* H = bh.as<double>();
    double* S = bs.as<double>();
    unpack_sym(c->stream, n, n, dHpk, H, filter);
    unpack_sym(c->stream, n, n, dSpk, S, filter);
    phase("unpack H, S");
    const int info = dpotrf_lower(c, n, n, S);
    PTB_CHECK(info == 0, PTBGPU_ENOTSPD, "overlap matrix not positive definite (potrf info=%d)", info);
    phase("potrf");
    const double one = 1.0;
    PTB_CUBLAS(cublasDtrsm(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                           (int)n, (int)n, &one, S, (int)n, H, (int)n));
    PTB_CUBLAS(cublasDtrsm(c->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                           (int)n, (int)n, &one, S, (int)n, H, (int)n));
    symmetrize_upper(c->stream, n, n, H);
    phase("2 trsm (A = L^-1 H L^-T)");
    Prologue p;
    gershgorin_bounds(c, n, n, H, &p.emin, &p.emax);
    PTB_CHECK(std::isfinite(p.emin) && std::isfinite(p.emax) && p.emax > p.emin, PTBGPU_ENAN,
              "invalid spectral bounds [%g, %g]", p.emin, p.emax);
    return p;
}

// L^-1 in place (lower triangle, column-major, leading dimension ld) by
// recursive halving, L^-1 = [L11^-1 0; -L22^-1 L21 L11^-1  L22^-1]: where the
// halves are equal and at least 2048, the two products of the off-diagonal
// block run on the int8 tensor cores (S slices, triangular operands masked and
// their zero K blocks skipped, written in place); smaller or uneven blocks go
// to the FP64 routine (cuBLAS trmm, cuSOLVER trtri leaves).
void trtri_oz(ptbgpu_ctx* c, int64_t n, int64_t ld, double* A, int S) {
    const int64_t n1 = (n / 2 + 127) / 128 * 128, n2 = n - n1;
    if (n < 4096 || n1 != n2 || !oz::supported(n1, S)) {
        dtrtri_lower(c, n, ld, A);
        return;
    }
    double* L11 = A;
    double* L21 = A + n1;
    double* L22 = A + n1 + n1 * ld;
    trtri_oz(c, n1, ld, L11, S);
    trtri_oz(c, n2, ld, L22, S);
    const oz::Operand opA = oz_operand(c, 0, n1, S), opB = oz_operand(c, 1, n1, S);
    oz::OzEpi ep;
    ep.n = n1;
    ep.out = L21;
    ep.ors = 1;
    ep.ocs = ld;
    // T = L21 L11^-1: rows of L21 times rows of L11^-T (upper triangular)
    oz_slice(c, L21, 1, ld, n1, oz::TRI_NONE, opA);
    oz_slice(c, L11, ld, 1, n1, oz::TRI_UPPER, opB);
    oz_product(c, oz::OZ_OUT, opA, opB, false, oz::TRI_NONE, oz::TRI_UPPER, ep);
    // L21 <- -L22^-1 T: rows of L22^-1 (lower triangular) times rows of T^T
    oz_slice(c, L22, 1, ld, n1, oz::TRI_LOWER, opA);
    oz_slice(c, L21, ld, 1, n1, oz::TRI_NONE, opB);
    ep.alpha = -1.0;
    oz_product(c, oz::OZ_OUT, opA, opB, false, oz::TRI_LOWER, oz::TRI_NONE, ep);
}

// The same on the int8 tensor cores: L^-1 by cuSOLVER trtri (in place in B_S,
// lower triangle), T = L^-1 H (lower-triangular A operand: K blocks past the
// diagonal are skipped), A = T L^-T (symmetric: upper tiles, mirrored).
Prologue orthogonalise_oz(ptbgpu_ctx* c, int64_t n, const double* dHpk, const double* dSpk, double filter, int S) {
    DevBuf& bh = c->buf(B_H);
    DevBuf& bs = c->buf(B_S);
    DevBuf& bt = c->buf(B_W1);
    bh.reserve(sizeof(double) * n * n);
    bs.reserve(sizeof(double) * n * n);
    bt.reserve(sizeof(double) * n * n);
    double* H = bh.as<double>();
    double* L = bs.as<double>();
    double* T = bt.as<double>();
    unpack_sym(c->stream, n, n, dHpk, H, filter);
    unpack_sym(c->stream, n, n, dSpk, L, filter);
    phase("unpack H, S");
    const int info = dpotrf_lower(c, n, n, L);
    PTB_CHECK(info == 0, PTBGPU_ENOTSPD, "overlap matrix not positive definite (potrf info=%d)", info);
    phase("potrf");
    trtri_oz(c, n, n, L, S);
    phase("trtri");
    const oz::Operand opL = oz_operand(c, 0, n, S), op1 = oz_operand(c, 1, n, S);
    oz_slice(c, L, 1, n, n, oz::TRI_LOWER, opL);   // rows of L^-1 (column-major storage)
    oz_slice(c, H, 1, n, n, oz::TRI_NONE, op1);    // rows of H (symmetric)
    phase("slice L^-1, H");
    oz::OzEpi ep;
    ep.n = n;
    ep.out = T;   // T column-major
    ep.ors = 1;
    ep.ocs = n;
    oz_product(c, oz::OZ_OUT, opL, op1, false, oz::TRI_LOWER, oz::TRI_NONE, ep);
    phase("int8 T = L^-1 H");
    oz_slice(c, T, 1, n, n, oz::TRI_NONE, op1);    // rows of T
    phase("slice T");
    oz::OzEpi es;
    es.n = n;
    es.out = H;   // A overwrites H (its slices are no longer read)
    es.ors = n;
    oz_product(c, oz::OZ_SYM, op1, opL, true, oz::TRI_NONE, oz::TRI_LOWER, es);
    phase("int8 A = T L^-T");
    check_timeout(c, "int8 product (orthogonalisation)");
    Prologue p;
    gershgorin_bounds(c, n, n, H, &p.emin, &p.emax);
    PTB_CHECK(std::isfinite(p.emin) && std::isfinite(p.emax) && p.emax > p.emin, PTBGPU_ENAN,
              "invalid spectral bounds [%g, %g]", p.emin, p.emax);
    return p;
}

// P = 2 L^-T X L^-1 on the int8 tensor cores with L^-1 from orthogonalise_oz:
// T2 = X L^-1 (B operand = rows of L^-T, upper triangular), then
// P = 2 L^-T T2 (A operand = rows of L^-T; symmetric result), packed into dPpk.
// X (column-major, symmetric) is overwritten; W is n x n scratch.
void back_transform_oz(ptbgpu_ctx* c, int64_t n, double* X, double* W, double* dPpk, int S) {
    const double* Linv = c->buf(B_S).as<double>();
    const oz::Operand opLt = oz_operand(c, 0, n, S), op1 = oz_operand(c, 1, n, S);
    oz_slice(c, Linv, n, 1, n, oz::TRI_UPPER, opLt);   // row j of L^-T = column j of L^-1
    oz_slice(c, X, 1, n, n, oz::TRI_NONE, op1);
    phase("slice L^-T, X");
    oz::OzEpi ep;
    ep.n = n;
    ep.out = W;   // T2 column-major
    ep.ors = 1;
    ep.ocs = n;
    oz_product(c, oz::OZ_OUT, op1, opLt, false, oz::TRI_NONE, oz::TRI_UPPER, ep);
    phase("int8 T2 = X L^-1");
    oz_slice(c, W, n, 1, n, oz::TRI_NONE, op1);        // rows of T2^T = columns of T2
    phase("slice T2^T");
    oz::OzEpi es;
    es.n = n;
    es.alpha = 2.0;
    es.out = X;
    es.ors = n;
    oz_product(c, oz::OZ_SYM, opLt, op1, true, oz::TRI_UPPER, oz::TRI_NONE, es);
    phase("int8 P = 2 L^-T T2");
    check_timeout(c, "int8 product (back-transform)");
    pack_cols(c->stream, n, n, X, dPpk);
}

// P = 2 L^-T X L^-1 (X in place, column-major n x n), then packed into dPpk.
void back_transform(ptbgpu_ctx* c, int64_t n, double* X, double* dPpk) {
    const double* L = c->buf(B_S).as<double>();
    const double two = 2.0, one = 1.0;
    PTB_CUBLAS(cublasDtrsm(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                           (int)n, (int)n, &two, L, (int)n, X, (int)n));
    PTB_CUBLAS(cublasDtrsm(c->blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                           (int)n, (int)n, &one, L, (int)n, X, (int)n));
    pack_cols(c->stream, n, n, X, dPpk);
}

// One FP64 SP2 step on X (column-major n x n, symmetric) using W as scratch;
// returns the idempotency error tr X - tr X^2 of the input and whether it squared.
struct StepInfo {
    double trX, trX2, err;
    bool sq;
};
StepInfo fp64_step(ptbgpu_ctx* c, int64_t n, double N, double*& X, double*& W) {
    StepInfo s;
    s.trX = trace_dev(c, n, n, X);
    const double f = frob_dev(c, n, n, X);
    s.trX2 = f * f;
    s.err = s.trX - s.trX2;
    PTB_CHECK(std::isfinite(s.err), PTBGPU_ENAN, "NaN during purification");
    s.sq = std::fabs(s.trX2 - N) <= std::fabs(2.0 * s.trX - s.trX2 - N);
    dsyrk_sq(c, n, n, X, W);                         // W = X^2
    if (!s.sq) axpby_diag(c->stream, n, n, 2.0, X, -1.0, W, 0.0);   // W = 2X - X^2
    std::swap(X, W);
    return s;
}

// FP64 trace-correcting purification of A (B_H, overwritten); the back-transform
// uses L from the cuBLAS prologue (S == 0) or L^-1 from the int8 one (S slices).
void sp2_fp64(ptbgpu_ctx* c, int64_t n, int64_t nel, const Prologue& pro, int maxit, int S, double* dPpk,
              ptbgpu_stats* st, int prl) {
    double* X = c->buf(B_H).as<double>();
    DevBuf& bw = c->buf(B_W0);
    bw.reserve(sizeof(double) * n * n);
    double* W = bw.as<double>();
    const double scale = 1.0 / (pro.emax - pro.emin);
    axpby_diag(c->stream, n, n, 0.0, nullptr, -scale, X, pro.emax * scale);
    const double N = 0.5 * (double)nel;
    std::vector<double> hist;
    int it = 0;
    bool done = false;
    for (it = 1; it <= maxit; ++it) {
        StepInfo s = fp64_step(c, n, N, X, W);
        const double e = std::fabs(s.err);
        hist.push_back(e);
        log_line(prl, 2, " SP2 (fp64) iter %3d  trX %.10f  err %.3e  %s", it, s.trX, s.err, s.sq ? "X^2" : "2X-X^2");
        if (e < 1e-13 * (double)n || (hist.size() > 2 && e < 1e-2 && e >= hist[hist.size() - 3])) {
            done = true;
            break;
        }
    }
    PTB_CHECK(done, PTBGPU_EITER, "trace-correcting purification did not converge in %d iterations", maxit);
    phase("SP2 iterations (FP64 syrk)");
    if (S > 0) back_transform_oz(c, n, X, W, dPpk, S);
    else back_transform(c, n, X, dPpk);
    phase("back-transform and pack");
    if (st) {
        st->iterations = it;
        st->flops += (double)it * (double)n * n * n;   // SYRK-equivalent products
    }
}

bool sp2_mixed(ptbgpu_ctx* c, int64_t n, int64_t nel, const Prologue& pro, int maxit, bool refine,
               int refine_rounds, double refine_tol, int64_t split3_iters, int S, double* dPpk, ptbgpu_stats* st,
               int prl) {
    cudaStream_t s = c->stream;
    const int64_t ldp = round_up(n, tc::tile_n());
    const size_t plane = sizeof(__nv_bfloat16) * (size_t)ldp * ldp;
    const size_t fplane = sizeof(float) * (size_t)ldp * ldp;

    // trajectory slots, bounded by free memory: hi and mid planes per iterate (the
    // bf16x3 products and the replay read these), plus the lo plane only when
    // three-plane products run
    const int tp = split3_iters >= 0 ? 3 : 2;
    size_t free_b = 0, total_b = 0;
    PTB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t other = 6 * fplane + 4 * plane + (size_t)(64 << 20);
    int slots = (int)std::min<int64_t>(maxit + 1, kMaxIt + 1);
    if (free_b > other) slots = (int)std::min<size_t>(slots, (free_b - other) * 6 / 10 / (tp * plane));
    PTB_CHECK(slots >= std::min(8, maxit + 1), PTBGPU_ENOMEM,
              "not enough device memory for the purification trajectory");
    DevBuf& btraj = c->buf(B_TRAJ);
    btraj.reserve(tp * plane * (size_t)slots);
    auto traj = [&](int k, int j) {
        return j < tp ? (__nv_bfloat16*)((char*)btraj.ptr + plane * (tp * (size_t)k + j)) : nullptr;
    };
    auto traj_hi = [&](int k) { return traj(k, 0); };
    auto traj_lo = [&](int k) { return traj(k, 1); };
    c->buf(B_XF0).reserve(fplane);
    c->buf(B_XF1).reserve(fplane);
    float* xf[2] = {c->buf(B_XF0).as<float>(), c->buf(B_XF1).as<float>()};

    // tiles and per-tile stats
    std::vector<int2> up = tc::make_tiles(ldp, true, 256);
    std::vector<int2> up3 = tc::make_tiles(ldp, true, 128);
    std::vector<int2> all = tc::make_tiles(ldp, false, 256);
    std::vector<int2> pup = tc::make_pair_tiles(ldp, true);     // CTA-pair kernel tiles
    std::vector<int2> pall = tc::make_pair_tiles(ldp, false);
    DevBuf& bt = c->buf(B_TILES);
    bt.reserve(sizeof(int2) * (up.size() + up3.size() + all.size() + pup.size() + pall.size()));
    int2* tiles_up = bt.as<int2>();
    int2* tiles_up3 = tiles_up + up.size();
    int2* tiles_all = tiles_up3 + up3.size();
    int2* pairs_up = tiles_all + all.size();
    int2* pairs_all = pairs_up + pup.size();
    PTB_CUDA(cudaMemcpyAsync(tiles_up, up.data(), sizeof(int2) * up.size(), cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(tiles_up3, up3.data(), sizeof(int2) * up3.size(), cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(tiles_all, all.data(), sizeof(int2) * all.size(), cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(pairs_up, pup.data(), sizeof(int2) * pup.size(), cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(pairs_all, pall.data(), sizeof(int2) * pall.size(), cudaMemcpyHostToDevice, s));
    const int npup = (int)pup.size(), npall = (int)pall.size();
    const int x0_blocks = grid1(ldp);
    DevBuf& bstats = c->buf(B_STATS);
    bstats.reserve(sizeof(double) * 2 * std::max({up.size(), up3.size(), 2 * pup.size(), (size_t)x0_blocks}));
    double* stats = bstats.as<double>();
    if (!c->sp2_state) PTB_CUDA(cudaMalloc(&c->sp2_state, sizeof(SP2State)));
    SP2State* state = (SP2State*)c->sp2_state;
    PTB_CUDA(cudaMemsetAsync(state, 0, sizeof(SP2State), s));
    const int one = 1;
    PTB_CUDA(cudaMemcpyAsync(&state->active, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(&c->flags->timeout, 0, sizeof(int), s));

    const double* A = c->buf(B_H).as<double>();
    const double scale = 1.0 / (pro.emax - pro.emin);
    const double N = 0.5 * (double)nel;
    // pass 1 runs to its rounding floor: the two-step non-decrease rule ends it
    const double tol_abs = 1e-12 * (double)n;
    const double e_asym = 0.1, e_stag = 0.01 * (double)n;
    k_x0_init<<<x0_blocks, 256, 0, s>>>(n, ldp, A, pro.emax, scale, xf[0], traj(0, 0), traj(0, 1), traj(0, 2),
                                        stats);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    const int cap = std::min(maxit, slots - 1);
    const int n6 = (int)up3.size(), n3 = (int)up.size();
    k_decide<<<1, 256, 0, s>>>(state, stats, x0_blocks, N, tol_abs, e_asym, e_stag, cap);
    count_launch();
    PTB_CUDA(cudaGetLastError());

    tc::ProdList split3{3, {0, 0, 1}, {0, 1, 0}};
    tc::ProdList split6{6, {0, 0, 1, 0, 2, 1}, {0, 1, 0, 2, 0, 1}};
    tc::EpiParams ep{};
    ep.active = &state->active;
    ep.sq_flag = &state->sq_cur;
    ep.err = &c->flags->timeout;
    ep.ld = ldp;
    ep.stats = stats;
    // three-plane products for the leading steps (0 = all, -1 = none)
    auto three_planes = [&](int k) { return split3_iters < 0 ? false : (split3_iters == 0 || k < split3_iters); };
    int launched = 0;
    const size_t timed0 = c->timed.size();   // pass-1 step timings start here
    SP2State* hs = (SP2State*)c->pinned;   // only the 8-int header is read back while iterating
    for (int k = 0; k < cap; ++k) {
        ep.xcur = xf[k & 1];
        ep.out = xf[(k + 1) & 1];
        ep.hi = traj(k + 1, 0);
        ep.lo = traj(k + 1, 1);
        ep.lo2 = traj(k + 1, 2);   // null with two planes
        const void* pl[3] = {traj(k, 0), traj(k, 1), traj(k, 2)};
        const bool three = three_planes(k);
        const int ntl = three ? timed_product(c, tc::EPI_SP2, 3, ldp, pl, pl, split6, tiles_up3, n6, ep)
                              : timed_product(c, tc::EPI_SP2, 2, ldp, pl, pl, split3, tiles_up, n3, ep, 0, pairs_up,
                                              npup);
        k_decide<<<1, 256, 0, s>>>(state, stats, ntl, N, tol_abs, e_asym, e_stag, cap);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        ++launched;
        if ((k & 3) == 3 || k + 1 == cap) {
            PTB_CUDA(cudaMemcpyAsync(hs, state, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
            PTB_CUDA(cudaStreamSynchronize(s));
            if (!hs->active) break;
        }
    }
    std::vector<SP2State> hstate(1);
    PTB_CUDA(cudaMemcpyAsync(hstate.data(), state, sizeof(SP2State), cudaMemcpyDeviceToHost, s));
    int tmo = 0;
    PTB_CUDA(cudaMemcpyAsync(&tmo, &c->flags->timeout, sizeof(int), cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    const SP2State& H = hstate[0];
    phase("pass 1 (tcgen05 bf16 SP2)");
    PTB_CHECK(tmo == 0, PTBGPU_ETIMEOUT, "tensor-core product gave up waiting (site %d)", tmo);
    PTB_CHECK(H.status == 0, H.status, "pass-1 purification failed (status %d at iterate %d)", H.status, H.next);
    PTB_CHECK(H.converged, PTBGPU_EITER, "pass-1 purification did not converge in %d iterations", cap);
    const int K = H.next;   // index of the final pass-1 iterate
    // steps launched after the decision that ended pass 1 did nothing: drop their timings
    if (timed0 + (size_t)K < c->timed.size()) c->timed.resize(timed0 + (size_t)K);
    // executed tcgen05 flops (all tiles of every launch that ran, every product of the split)
    double tc_exec = 0.0;
    for (int k = 0; k < K; ++k)
        tc_exec += three_planes(k) ? 2.0 * 6 * 128 * 128 * (double)ldp * n6 : 2.0 * 3 * 128 * 256 * (double)ldp * n3;
    const double tc_exec_full = 2.0 * 3 * (double)ldp * ldp * ldp;   // one general bf16x3 product
    for (int k = 0; k <= K && prl >= 2; ++k)
        log_line(prl, 2, " SP2 (bf16x3) iter %3d  trX %.10f  err %.3e  %s", k, H.trX[k], H.err[k],
                 k < K ? (H.sq[k] ? "X^2" : "2X-X^2") : "final");

    // FP64 cleanup of the pass-1 result
    DevBuf& bw0 = c->buf(B_W0);
    DevBuf& bw1 = c->buf(B_W1);
    bw0.reserve(sizeof(double) * n * n);
    bw1.reserve(sizeof(double) * n * n);
    double* X = bw0.as<double>();
    double* W = bw1.as<double>();
    k_f2d<<<grid1(n), 256, 0, s>>>(n, ldp, xf[K & 1], 1.0, 0.0, X);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    // SP2 steps in FP64 precision until the idempotency error reaches FP64
    // rounding or stops falling over two steps (at most 8); returns the steps
    auto cleanup = [&]() -> int {
        std::vector<double> hist;
        int nclean = 0;
        if (S > 0) {
            // int8-sliced squares, X updated in place (the epilogue reads X(r,c), c >= r,
            // before writing it; the mirrored lower triangle is never read); the error
            // of each iterate is checked before its square is taken
            DevBuf& bst = c->buf(B_OZS);
            // per-CTA partials: at most (rows / 128 + 1) x ceil(cols / 48) CTAs for any kernel variant
            bst.reserve(sizeof(double) * 2 * (size_t)(oz::padded(n) / oz::BM + 1) *
                        (size_t)((oz::padded(n) + 47) / 48));
            std::vector<double> hst;
            double trX = trace_dev(c, n, n, X);
            const double f0 = frob_dev(c, n, n, X);
            double trX2 = f0 * f0;
            for (;;) {
                const double err = trX - trX2, e = std::fabs(err);
                PTB_CHECK(std::isfinite(err), PTBGPU_ENAN, "NaN during purification");
                hist.push_back(e);
                log_line(prl, 2, " SP2 (int8 FP64 cleanup) %d  err %.3e", nclean, err);
                if (e < 1e-13 * (double)n || (hist.size() > 2 && e >= hist[hist.size() - 3]) || nclean >= 8) break;
                const bool sq = std::fabs(trX2 - N) <= std::fabs(2.0 * trX - trX2 - N);
                // while the iterate is still far from idempotent its square needs no
                // more than 6 slices (42 bits): the last digits only matter in the
                // final squares, which take the full slice count
                const oz::Operand opX = oz_operand(c, 1, n, e > 1e-4 ? std::min(S, 6) : S);
                oz_slice(c, X, 1, n, n, oz::TRI_NONE, opX);
                oz::OzEpi es;
                es.n = n;
                es.out = X;
                es.ors = n;
                es.xin = X;
                es.square = sq ? 1 : 0;
                es.stats = bst.as<double>();
                const int nt = oz_product(c, oz::OZ_SYM, opX, opX, true, oz::TRI_NONE, oz::TRI_NONE, es);
                hst.resize(2 * (size_t)nt);
                PTB_CUDA(cudaMemcpyAsync(hst.data(), es.stats, sizeof(double) * hst.size(), cudaMemcpyDeviceToHost, s));
                check_timeout(c, "int8 product (cleanup)");
                trX = 0.0;
                trX2 = 0.0;
                for (int t = 0; t < nt; ++t) {
                    trX += hst[2 * t];
                    trX2 += hst[2 * t + 1];
                }
                ++nclean;
            }
        } else {
            for (nclean = 1; nclean <= 8; ++nclean) {
                StepInfo si = fp64_step(c, n, N, X, W);
                const double e = std::fabs(si.err);
                hist.push_back(e);
                log_line(prl, 2, " SP2 (fp64 cleanup) %d  err %.3e", nclean, si.err);
                // until the error reaches FP64 rounding or stops falling over two steps: a
                // single SP2 step squares the deviation on one side of the spectrum but
                // doubles it on the other, so a small error on entry is not enough
                if (e < 1e-13 * (double)n || (hist.size() > 2 && e >= hist[hist.size() - 3])) break;
            }
            nclean = std::min(nclean, 8);
        }
        return nclean;
    };
    int nclean = cleanup();
    phase(S > 0 ? "cleanup (int8 FP64 squares)" : "cleanup (FP64 syrk)");
    // algorithmic: every SP2 step is one symmetric square (n^3), pass 1 and cleanup alike
    double flops = (double)K * (double)n * n * n + (double)nclean * (double)n * n * n;

    // Refinement rounds: each one is a Newton step on the occupied subspace (the
    // first-order response to the part of A that couples the occupied and
    // virtual spaces of P~); the error left is second order in the correction.
    // The replay linearises along the bf16x3 pass-1 trajectory, which is exact
    // for a Hamiltonian a rounding away from A; near the gap that relative error
    // grows like range / gap, so the rounds contract the error linearly with a
    // factor that grows with the first round's response gain g1 = max|X1| /
    // max|X1_0|.  Measured on water clusters, an alkane chain and cubic-lattice
    // systems (range/gap 25 to 1e4): the next correction stays below kRho1 * g1
    // of the first one and below max(kRho2 * g1, last ratio) of a later one.
    // Another round, after an FP64 cleanup of the corrected X, runs while that
    // predicted error exceeds refine_tol, up to refine_rounds.  If the rounds
    // cannot get there (contraction above 1/2, or the cap reached with the
    // prediction above 10 refine_tol) the caller redoes the purification in FP64.
    int rounds = 0;
    double g1 = 0.0, prev_x1max = 0.0, resid = 0.0, rho = 0.0;
    while (refine) {
        // C = A P~ - P~ A (FP64)
        DevBuf& bw2 = c->buf(B_W2);
        bw2.reserve(sizeof(double) * n * n);
        double* Wc = bw2.as<double>();
        if (S > 0) {
            // C is ~1e-6 of |A||P~|: 6 slices (42 bits of the row maxima) leave it
            // with ~1e-7 relative error, far below what its first-order use needs
            const int Sc = 6;
            const oz::Operand opA = oz_operand(c, 0, n, Sc), opP = oz_operand(c, 1, n, Sc);
            oz_slice(c, A, 1, n, n, oz::TRI_NONE, opA);
            oz_slice(c, X, 1, n, n, oz::TRI_NONE, opP);
            oz::OzEpi ep;
            ep.n = n;
            ep.out = W;   // W = A P~, column-major
            ep.ors = 1;
            ep.ocs = n;
            oz_product(c, oz::OZ_OUT, opA, opP, false, oz::TRI_NONE, oz::TRI_NONE, ep);
            phase("int8 W = A P~ (incl. slices)");
        } else {
            dgemm_nn(c, n, n, 1.0, A, X, 0.0, W);
            phase("dgemm W = A P~");
        }
        const unsigned nb = (unsigned)((n + 31) / 32);
        k_antisym<<<dim3(nb, nb), dim3(32, 8), 0, s>>>(n, W, Wc);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        // bf16x3 planes of C and P~ (padded), V = C^T P~ = -C P~ on the tensor cores
        c->buf(B_X1HI).reserve(2 * plane);
        c->buf(B_X1LO).reserve(2 * plane);
        c->buf(B_MISC0).reserve(fplane);   // W (FP32, row-major)
        c->buf(B_X1F0).reserve(fplane);
        c->buf(B_X1F1).reserve(fplane);
        DevBuf& bp = c->buf(B_MISC1);
        bp.reserve(2 * plane);
        __nv_bfloat16* chi = (__nv_bfloat16*)c->buf(B_X1HI).ptr;
        __nv_bfloat16* clo = chi + (size_t)ldp * ldp;
        __nv_bfloat16* phi = (__nv_bfloat16*)bp.ptr;
        __nv_bfloat16* plo = phi + (size_t)ldp * ldp;
        float* wf = c->buf(B_MISC0).as<float>();
        float* x1f[2] = {c->buf(B_X1F0).as<float>(), c->buf(B_X1F1).as<float>()};
        // X1 hi planes live in B_X1LO; its lo planes take over the C planes once
        // the product V below has consumed them (stream order).
        __nv_bfloat16* x1hi[2] = {(__nv_bfloat16*)c->buf(B_X1LO).ptr,
                                  (__nv_bfloat16*)c->buf(B_X1LO).ptr + (size_t)ldp * ldp};
        __nv_bfloat16* x1lo[2] = {chi, clo};
        d2f_split(s, n, ldp, Wc, nullptr, chi, clo);
        d2f_split(s, n, ldp, X, nullptr, phi, plo);
        tc::EpiParams epf{};
        epf.err = &c->flags->timeout;
        epf.ld = ldp;
        epf.out = wf;
        const void* pc[2] = {chi, clo};
        const void* pp[2] = {phi, plo};
        timed_product(c, tc::EPI_FULL, 2, ldp, pc, pp, split3, tiles_all, (int)all.size(), epf, 0, pairs_all, npall);
        // The planes hold C^T (column-major C read row-major), so wf = C^T P~ = -C P~.
        // A1 = C P~ - P~ C = -(wf + wf^T) and X1_0 = -A1 / (e_max - e_min) = (wf + wf^T) * scale.
        const unsigned nbp = (unsigned)(ldp / 32);
        k_sym_update<<<dim3(nbp, nbp), dim3(32, 8), 0, s>>>(ldp, wf, nullptr, (float)scale, 0.0f, x1f[0], x1hi[0],
                                                            x1lo[0]);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        // max |X1_0| (second half of the partials buffer, read with the final ones)
        constexpr int kParts = 296;
        DevBuf& btau = c->buf(B_MISC2);
        btau.reserve(sizeof(double) * 4 * kParts);
        k_trace_maxabs_f32<<<kParts, 256, 0, s>>>(n, ldp, x1f[0], btau.as<double>() + 2 * kParts);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        phase("commutator, planes, A1 product");
        // replay the branch sequence over the stored trajectory
        for (int k = 0; k < K; ++k) {
            const int a = k & 1, b = a ^ 1;
            const void* p0[2] = {traj_hi(k), traj_lo(k)};
            const void* p1[2] = {x1hi[a], x1lo[a]};
            timed_product(c, tc::EPI_FULL, 2, ldp, p0, p1, split3, tiles_all, (int)all.size(), epf, 0, pairs_all, npall);
            const bool sq = H.sq[k] != 0;
            k_sym_update<<<dim3(nbp, nbp), dim3(32, 8), 0, s>>>(ldp, wf, x1f[a], sq ? 1.0f : -1.0f,
                                                                sq ? 0.0f : 2.0f, x1f[b], x1hi[b], x1lo[b]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
        }
        phase("DMPT replay (tcgen05 bf16x3)");
        // Keep only the blocks of X1 that couple occupied and virtual states of
        // P~: X1_od = P~ X1 + X1 P~ - 2 P~ X1 P~ = W + W^T - 2 W P~ with W = P~ X1.
        // The diagonal blocks of the computed X1 are rounding noise of the
        // products; they would shift the energy at first order, X1_od only at
        // second.  Both products are of a small quantity, so bf16x3 suffices.
        {
            const int a = K & 1, b = a ^ 1;
            const void* pp2[2] = {phi, plo};
            const void* px[2] = {x1hi[a], x1lo[a]};
            timed_product(c, tc::EPI_FULL, 2, ldp, pp2, px, split3, tiles_all, (int)all.size(), epf, 0, pairs_all, npall);   // W
            k_split2<<<grid1(ldp * ldp / 256), 256, 0, s>>>(ldp * ldp, wf, x1hi[b], x1lo[b]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            tc::EpiParams epv = epf;
            epv.out = x1f[b];
            const void* pw[2] = {x1hi[b], x1lo[b]};
            timed_product(c, tc::EPI_FULL, 2, ldp, pw, pp2, split3, tiles_all, (int)all.size(), epv, 0, pairs_all, npall);  // W P~
            k_sym_update<<<dim3(nbp, nbp), dim3(32, 8), 0, s>>>(ldp, wf, x1f[b], 1.0f, -2.0f, x1f[a], x1hi[a],
                                                                x1lo[a]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            // Second-order idempotency term of the expansion: for a purely
            // off-diagonal first-order part X1, (P~ + X1)^2 - (P~ + X1) = Y = X1^2
            // (block diagonal, positive semi-definite), which lowers the energy at
            // second order summed over all occupied states.  P2 = -(P~ Y + Y P~ - Y)
            // removes it: X1 <- X1 + Y - (W2 + W2^T), W2 = P~ Y (traceless, small).
            const void* px1[2] = {x1hi[a], x1lo[a]};
            tc::EpiParams epy = epf;
            epy.out = x1f[b];
            timed_product(c, tc::EPI_FULL, 2, ldp, px1, px1, split3, tiles_all, (int)all.size(), epy, 0, pairs_all, npall);   // Y
            k_split2<<<grid1(ldp * ldp / 256), 256, 0, s>>>(ldp * ldp, x1f[b], x1hi[b], x1lo[b]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            const void* py[2] = {x1hi[b], x1lo[b]};
            timed_product(c, tc::EPI_FULL, 2, ldp, pp2, py, split3, tiles_all, (int)all.size(), epf, 0, pairs_all, npall);    // W2
            k_add_f32<<<grid1(ldp * ldp / 256), 256, 0, s>>>(ldp * ldp, x1f[a], x1f[b]);              // Y + X1
            count_launch();
            PTB_CUDA(cudaGetLastError());
            k_sym_update<<<dim3(nbp, nbp), dim3(32, 8), 0, s>>>(ldp, wf, x1f[b], -1.0f, 1.0f, x1f[a], x1hi[a],
                                                                x1lo[a]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
        }
        phase("projection, idempotency term");
        // P_o = P~ (1 - tau/N) + X1_K with tau = tr X1_K: the exact first-order
        // response is traceless; its bf16x3 rounding noise is removed from the
        // trace in FP64 along P~ (a uniform shift of the occupied eigenvalues by
        // tau/N), so tr P_o = N to FP64 rounding.
        k_trace_maxabs_f32<<<kParts, 256, 0, s>>>(n, ldp, x1f[K & 1], btau.as<double>());
        count_launch();
        PTB_CUDA(cudaGetLastError());
        double tparts[4 * kParts];
        PTB_CUDA(cudaMemcpyAsync(tparts, btau.ptr, sizeof(tparts), cudaMemcpyDeviceToHost, s));
        PTB_CUDA(cudaStreamSynchronize(s));
        double tau = 0.0, x1max = 0.0, x10max = 0.0;
        for (int p = 0; p < kParts; ++p) {
            tau += tparts[2 * p];
            x1max = std::max(x1max, tparts[2 * p + 1]);
            x10max = std::max(x10max, tparts[2 * kParts + 2 * p + 1]);
        }
        k_f2d<<<grid1(n), 256, 0, s>>>(n, ldp, x1f[K & 1], 1.0, 1.0 - tau / N, X);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        // algorithmic: FP64 commutator 2n^3, then K + 5 general products of 2n^3
        flops += 2.0 * (double)n * n * n + (double)(K + 5) * 2.0 * (double)n * n * n;
        phase("trace correction");
        PTB_CUDA(cudaMemcpyAsync(&tmo, &c->flags->timeout, sizeof(int), cudaMemcpyDeviceToHost, s));
        PTB_CUDA(cudaStreamSynchronize(s));
        PTB_CHECK(tmo == 0, PTBGPU_ETIMEOUT, "tensor-core product gave up waiting (site %d)", tmo);
        ++rounds;
        // error left after this round, predicted from the size of its correction
        const double gain = x10max > 0.0 ? x1max / x10max : 0.0;
        if (rounds == 1) {
            g1 = gain;
            rho = x10max > 0.0 ? std::min(1.0, kRho1 * g1) : 1.0;
        } else {
            rho = std::min(1.0, std::max(kRho2 * g1, prev_x1max > 0.0 ? x1max / prev_x1max : 1.0));
        }
        prev_x1max = x1max;
        resid = x1max * rho;
        log_line(prl, 2, " refinement round %d  max|X1| %.3e  max|X1_0| %.3e  gain %.3e  predicted %.3e  tau %.3e",
                 rounds, x1max, x10max, gain, resid, tau);
        if (!(resid > refine_tol)) break;
        if (rounds >= refine_rounds || std::min(1.0, kRho2 * g1) > 0.5) {
            if (resid > 10.0 * refine_tol) {
                log_line(prl, 1, " refinement cannot reach %.1e (predicted %.2e after %d rounds): FP64 purification",
                         refine_tol, resid, rounds);
                if (st) st->refine_rounds = rounds;
                return false;
            }
            break;
        }
        const int more = cleanup();
        nclean += more;
        flops += (double)more * (double)n * n * n;
        phase(S > 0 ? "cleanup (int8 FP64 squares)" : "cleanup (FP64 syrk)");
    }
    if (S > 0) back_transform_oz(c, n, X, W, dPpk, S);   // sets tr(PS) directly: full slice count
    else back_transform(c, n, X, dPpk);
    phase("back-transform and pack");
    if (st) {
        st->iterations = K + nclean;
        st->refine_rounds = rounds;
        st->tc_flops += tc_exec + (double)rounds * (double)(K + 5) * tc_exec_full;
        st->flops += flops;
    }
    return true;
}

void tc_purify_device(ptbgpu_ctx* c, int64_t n, int64_t nel, const double* dH, const double* dS, double* dP,
                      const ptbgpu_opts* o, ptbgpu_stats* st) {
    PTB_CHECK(n > 0 && nel > 0 && nel <= 2 * n, PTBGPU_EINVAL, "bad sizes ndim=%lld nel=%lld", (long long)n,
              (long long)nel);
    PTB_CHECK(nel % 2 == 0, PTBGPU_EINVAL, "trace-correcting purification needs an even electron count");
    ptbgpu_opts def;
    ptbgpu_default_opts(&def);
    if (!o) o = &def;
    const int maxit = o->max_iter > 0 ? (int)std::min<int64_t>(o->max_iter, kMaxIt) : 100;
    const int prl = (int)o->print_level;
    // int8-sliced FP64 products on the mixed path, when the dimension keeps the int32 sums exact
    const int S = (o->precision != PTBGPU_PREC_FP64 && o->fp64_slices != 0) ? (int)o->fp64_slices : 0;
    PTB_CHECK(S == 0 || (S >= 6 && S <= 8), PTBGPU_EINVAL, "fp64_slices must be 0 or 6..8 (got %d)", S);
    const int Suse = (S > 0 && oz::supported(n, S)) ? S : 0;
    PTB_CHECK(o->refine_rounds >= 0 && o->refine_rounds <= 16 && o->refine_tol >= 0.0, PTBGPU_EINVAL,
              "refine_rounds must be 0..16 and refine_tol >= 0");
    const int rounds = o->refine_rounds > 0 ? (int)o->refine_rounds : 4;
    const double rtol = o->refine_tol > 0.0 ? o->refine_tol : 1e-7;
    PhaseLog plog;
    plog.c = c;
    struct Scope {
        PhaseLog* p;
        explicit Scope(PhaseLog* q) : p(q) { t_phases = q; }
        ~Scope() { t_phases = nullptr; }
    } scope(prl >= 2 ? &plog : nullptr);
    phase("start");
    Prologue pro = Suse > 0 ? orthogonalise_oz(c, n, dH, dS, o->filter, slices_once(Suse))
                            : orthogonalise(c, n, dH, dS, o->filter);
    phase("Gershgorin bounds");
    if (st) st->flops += (1.0 / 3.0 + 4.0) * (double)n * n * n;   // potrf + 4 trsm
    if (o->precision == PTBGPU_PREC_FP64) {
        sp2_fp64(c, n, nel, pro, maxit, 0, dP, st, prl);
    } else if (!sp2_mixed(c, n, nel, pro, maxit, o->precision != 2, rounds, rtol, o->split3_iters, Suse, dP, st,
                          prl)) {
        // A (B_H) is still intact: the mixed path only reads it
        sp2_fp64(c, n, nel, pro, maxit, Suse, dP, st, prl);
        if (st) st->fp64_fallback = 1;
    }
    if (prl >= 2) plog.report(prl);
}

}  // namespace

void tc_purify_entry(ptbgpu_ctx* c, int64_t n, int64_t nel, const double* dH, const double* dS, double* dP,
                     const ptbgpu_opts* o, ptbgpu_stats* st) {
    tc_purify_device(c, n, nel, dH, dS, dP, o, st);
}

// C = X X with the split-bf16 kernel (every tile, EPI_FULL) for kernel-level
// tests: np = 2 planes (bf16x3 products) or 3 planes (bf16x6 products).
void symsq_entry(ptbgpu_ctx* c, int64_t n, int np, int kblock, const double* hX, float* hC) {
    cudaStream_t s = c->stream;
    const int64_t ldp = round_up(n, tc::tile_n());
    const size_t plane = sizeof(__nv_bfloat16) * (size_t)ldp * ldp;
    DevBuf& bx = c->buf(B_W0);
    bx.reserve(sizeof(double) * n * n);
    PTB_CUDA(cudaMemcpyAsync(bx.ptr, hX, sizeof(double) * n * n, cudaMemcpyHostToDevice, s));
    DevBuf& bp = c->buf(B_MISC1);
    bp.reserve(3 * plane);
    __nv_bfloat16* hi = (__nv_bfloat16*)bp.ptr;
    __nv_bfloat16* mid = hi + (size_t)ldp * ldp;
    __nv_bfloat16* lo = mid + (size_t)ldp * ldp;
    DevBuf& bc = c->buf(B_MISC0);
    bc.reserve(sizeof(float) * (size_t)ldp * ldp);
    float* xf = bc.as<float>();
    // planes of the FP32-rounded X: hi, mid = bf16(x - hi), lo = bf16(x - hi - mid)
    d2f_split(s, n, ldp, bx.as<double>(), xf, hi, mid);
    d2f_split3(s, ldp, xf, hi, mid, lo);
    std::vector<int2> all = tc::make_tiles(ldp, false, np == 2 ? 256 : 128);
    std::vector<int2> pall = np == 2 ? tc::make_pair_tiles(ldp, false) : std::vector<int2>();
    DevBuf& bt = c->buf(B_TILES);
    bt.reserve(sizeof(int2) * (all.size() + pall.size()));
    PTB_CUDA(cudaMemcpyAsync(bt.ptr, all.data(), sizeof(int2) * all.size(), cudaMemcpyHostToDevice, s));
    int2* pairs = pall.empty() ? nullptr : bt.as<int2>() + all.size();
    if (pairs)
        PTB_CUDA(cudaMemcpyAsync(pairs, pall.data(), sizeof(int2) * pall.size(), cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(&c->flags->timeout, 0, sizeof(int), s));
    tc::ProdList split3{3, {0, 0, 1}, {0, 1, 0}};
    tc::ProdList split6{6, {0, 0, 1, 0, 2, 1}, {0, 1, 0, 2, 0, 1}};
    tc::EpiParams ep{};
    ep.err = &c->flags->timeout;
    ep.ld = ldp;
    ep.out = xf;   // the FP32 copy is consumed by the split above (stream order)
    const void* pl[3] = {hi, mid, lo};
    timed_product(c, tc::EPI_FULL, np, ldp, pl, pl, np == 2 ? split3 : split6, bt.as<int2>(), (int)all.size(), ep,
                  kblock, pairs, (int)pall.size());
    PTB_CUDA(cudaMemcpy2DAsync(hC, sizeof(float) * n, xf, sizeof(float) * ldp, sizeof(float) * n, n,
                               cudaMemcpyDeviceToHost, s));
    int tmo = 0;
    PTB_CUDA(cudaMemcpyAsync(&tmo, &c->flags->timeout, sizeof(int), cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    PTB_CHECK(tmo == 0, PTBGPU_ETIMEOUT, "tensor-core product gave up waiting (site %d)", tmo);
}

// C = A B (n x n, row-major host FP64) with the int8-sliced kernel, for
// kernel-level tests.  tri_a / tri_b describe A and B as matrices (1 lower,
// 2 upper); sym: only the upper triangle of C is computed and mirrored.
void oz_gemm_entry(ptbgpu_ctx* c, int64_t n, int S, int kblock, int variant, int tri_a, int tri_b, bool sym,
                   const double* hA, const double* hB, double* hC) {
    PTB_CHECK(oz::supported(n, S), PTBGPU_EINVAL, "n = %lld is too large for exact int32 sums with %d slices",
              (long long)n, S);
    cudaStream_t s = c->stream;
    DevBuf& ba = c->buf(B_W0);
    DevBuf& bb = c->buf(B_W1);
    DevBuf& bc = c->buf(B_W2);
    ba.reserve(sizeof(double) * n * n);
    bb.reserve(sizeof(double) * n * n);
    bc.reserve(sizeof(double) * n * n);
    PTB_CUDA(cudaMemcpyAsync(ba.ptr, hA, sizeof(double) * n * n, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(bb.ptr, hB, sizeof(double) * n * n, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemsetAsync(&c->flags->timeout, 0, sizeof(int), s));
    const oz::Operand opA = oz_operand(c, 0, n, S), opB = oz_operand(c, 1, n, S);
    // rows of A: A(i,k) = A[i n + k]; rows of B^T: B^T(j,k) = B(k,j) = B[j + k n]
    const int ta = tri_a, tb = tri_b == 1 ? oz::TRI_UPPER : tri_b == 2 ? oz::TRI_LOWER : oz::TRI_NONE;
    oz_slice(c, ba.as<double>(), n, 1, n, ta, opA);
    oz_slice(c, bb.as<double>(), 1, n, n, tb, opB);
    oz::OzEpi ep;
    ep.n = n;
    ep.out = bc.as<double>();
    ep.ors = n;
    ep.ocs = 1;
    oz_product(c, sym ? oz::OZ_SYM : oz::OZ_OUT, opA, opB, sym, ta, tb, ep, kblock, variant);
    PTB_CUDA(cudaMemcpyAsync(hC, bc.ptr, sizeof(double) * n * n, cudaMemcpyDeviceToHost, s));
    check_timeout(c, "int8 product");
}

// ---------------------------------------------------------------------------
// General FP64-class products on the int8 tensor cores for the module code
// (purification module, metrics): C = alpha op(A) op(B) for column-major
// n x n device matrices, S slices (8: about 53 bits relative to the row and
// column maxima).  The device tile list of each (n, S) is kept on the context,
// so a product is two slicings and one launch with no host round trip.
namespace {
struct OzTiles {
    DevBuf buf;
    int count = 0;
    double ops = 0.0;
};
struct OzTileCache {
    std::map<std::pair<int64_t, int>, OzTiles> lists;
    ~OzTileCache() {
        for (auto& kv : lists) kv.second.buf.release();
    }
};
}  // namespace

void oz_dgemm(ptbgpu_ctx* c, int64_t n, double alpha, const double* A, bool ta, const double* B, bool tb,
              double* C, int S) {
    PTB_CHECK(oz::supported(n, S), PTBGPU_EINVAL, "n = %lld is too large for exact int32 sums with %d slices",
              (long long)n, S);
    if (!c->oz_tile_cache) c->oz_tile_cache = std::make_shared<OzTileCache>();
    OzTileCache& tc = *static_cast<OzTileCache*>(c->oz_tile_cache.get());
    const oz::Operand opA = oz_operand(c, 0, n, S), opB = oz_operand(c, 1, n, S);
    const int variant = oz::resolve_variant(oz::V_DEFAULT, S, 0);
    auto key = std::make_pair(n, S);
    auto it = tc.lists.find(key);
    if (it == tc.lists.end()) {
        const std::vector<int4> t = oz::build_tiles(opA.ldp, false, oz::TRI_NONE, oz::TRI_NONE, S, variant);
        OzTiles e;
        e.buf.reserve(sizeof(int4) * t.size());
        e.count = (int)t.size();
        e.ops = oz::tile_ops(t, S, variant);
        PTB_CUDA(cudaMemcpy(e.buf.ptr, t.data(), sizeof(int4) * t.size(), cudaMemcpyHostToDevice));
        it = tc.lists.emplace(key, e).first;
    }
    c->oz_ops += it->second.ops;
    // rows i of op(A): A(i,k) = A[i + k n], A^T(i,k) = A[k + i n]
    oz_slice(c, A, ta ? n : 1, ta ? 1 : n, n, oz::TRI_NONE, opA);
    // rows j of op(B)^T, i.e. op(B)(k, j): B[k + j n], or B^T: B[j + k n]
    oz_slice(c, B, tb ? 1 : n, tb ? n : 1, n, oz::TRI_NONE, opB);
    oz::OzEpi ep;
    ep.n = n;
    ep.alpha = alpha;
    ep.out = C;
    ep.ors = 1;
    ep.ocs = n;
    ep.ldp = opA.ldp;
    ep.err = &c->flags->timeout;
    oz::product(c->stream, oz::OZ_OUT, opA, opB, it->second.buf.as<int4>(), it->second.count, ep, 0, variant);
    count_launch();
}

void oz_check(ptbgpu_ctx* c, const char* what) { check_timeout(c, what); }

}  // namespace ptb
