// Grouped trace-correcting purification of many independent systems.
//
// The systems are bucketed by their dimension rounded up to 256 (B).  Within a
// bucket every system is padded to B x B: S gets a unit diagonal and the
// orthogonalised A the system's upper spectral bound on the padded diagonal,
// which X_0 maps to exactly 0, a fixed point of both SP2 branches, so the
// padding stays decoupled and contributes nothing to any trace.  The padded
// systems are stacked along the rows of one set of planes, and every step of
// the purification is one launch over all systems of the chunk:
//   - FP64 prologue / cleanup / commutator / back-transform: cuSOLVER potrf per
//     system, cuBLAS trsmBatched and DgemmStridedBatched;
//   - pass 1 and the refinement products: the tcgen05 split-bf16 kernel over the
//     stacked planes (tiles carry global row blocks, the epilogue works in the
//     tile's system; per-system branch and stop flags on the device);
//   - per-system decisions (branch, stop at the rounding floor) in one kernel
//     with a block per system, the same rule as the single-system path.
// Systems that finish pass 1 earlier are skipped by the product kernel (their
// tiles exit at once); in the replay the systems are ordered by their
// pass-1 length, so the tiles still active at step k are a prefix of the list.
// Each refinement round runs for every system of the chunk that still needs
// one; a system whose rounds cannot reach the tolerance (or that does not
// converge) is redone by the single-system FP64 path afterwards.
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "sp2_state.cuh"
#include "tc_gemm.cuh"

namespace ptb {

namespace {

using bf16 = __nv_bfloat16;
constexpr int kThr = 256;

__device__ __forceinline__ void block_sum2(double& a, double& b) {
    __shared__ double sh[2][32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) {
        sh[0][w] = a;
        sh[1][w] = b;
    }
    __syncthreads();
    a = 0.0;
    b = 0.0;
    for (int q = 0; q < nw; ++q) {   // every thread, fixed order
        a += sh[0][q];
        b += sh[1][q];
    }
}

__device__ __forceinline__ void split3(float v, bf16& h, bf16& m, bf16& l) {
    h = __float2bfloat16_rn(v);
    const float r = v - __bfloat162float(h);
    m = __float2bfloat16_rn(r);
    l = __float2bfloat16_rn(r - __bfloat162float(m));
}

// M(i,i) = val[s] (or v) for n_s <= i < B.  grid (x, nb).
__global__ void k_pad_diag(int64_t B, const int* __restrict__ nsys, double* __restrict__ M,
                           const double* __restrict__ val, double v) {
    const int s = blockIdx.y;
    double* m = M + (int64_t)s * B * B;
    const double d = val ? val[s] : v;
    for (int64_t i = nsys[s] + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < B; i += (int64_t)gridDim.x * blockDim.x)
        m[i + i * B] = d;
}

// Exact symmetry: M(j,i) := M(i,j) for i < j (column-major).  grid (B/32, B/32, nb), block (32, 8).
__global__ void k_sym_lower(int64_t B, double* __restrict__ M) {
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    __shared__ double t[32][33];
    double* m = M + (int64_t)blockIdx.z * B * B;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = bi * 32, j0 = bj * 32;
#pragma unroll
    for (int k = 0; k < 32; k += 8) t[ty + k][tx] = m[(i0 + tx) + (j0 + ty + k) * B];   // t[c][r] = M(i0+r, j0+c)
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int r = ty + k, cc = tx;
        if (i0 + r < j0 + cc) m[(j0 + cc) + (i0 + r) * B] = t[cc][r];
    }
}

// C = W - W^T per system (column-major).  grid (B/32, B/32, nb), block (32, 8).
__global__ void k_antisym_g(int64_t B, const double* __restrict__ W, double* __restrict__ Cm) {
    __shared__ double t[32][33];
    const int64_t off = (int64_t)blockIdx.z * B * B;
    const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int k = 0; k < 32; k += 8) t[tx][ty + k] = W[off + (j0 + tx) + (i0 + ty + k) * B];   // W(j0+tx, i0+ty+k)
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int64_t row = i0 + tx, col = j0 + ty + k;
        Cm[off + row + col * B] = W[off + row + col * B] - t[ty + k][tx];   // W(row,col) - W(col,row)
    }
}

// Gershgorin bounds over the first n_s columns of every system (column i:
// a_ii -+ sum_{j != i} |a_ji|, symmetric A); per-block min / max partials.
// grid (nchunk, nb).
__global__ void k_gersh(int64_t B, const int* __restrict__ nsys, const double* __restrict__ A,
                        double* __restrict__ plo, double* __restrict__ phi) {
    const int s = blockIdx.y;
    const int64_t n = nsys[s];
    const double* a = A + (int64_t)s * B * B;
    double lo = INFINITY, hi = -INFINITY;
    for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
        double r = 0.0, d = 0.0;
        for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
            const double v = a[j + i * B];
            if (j == i) d = v;
            else r += fabs(v);
        }
        block_sum2(r, d);
        lo = fmin(lo, d - r);
        hi = fmax(hi, d + r);
    }
    if (threadIdx.x == 0) {
        plo[(int64_t)s * gridDim.x + blockIdx.x] = lo;
        phi[(int64_t)s * gridDim.x + blockIdx.x] = hi;
    }
}

// X_0 = (e_max I - A) * scale (per system) into the stacked FP32 / bf16 planes
// (linear copy: the systems are symmetric), with per-block partials of tr X_0
// and ||X_0||^2.  grid (nchunk, nb).
__global__ void k_x0(int64_t B, const double* __restrict__ A, const double* __restrict__ emax,
                     const double* __restrict__ scale, float* __restrict__ xf, bf16* __restrict__ hi,
                     bf16* __restrict__ mid, bf16* __restrict__ lo, double* __restrict__ stats) {
    const int s = blockIdx.y;
    const int64_t base = (int64_t)s * B * B, nn = B * B;
    double tr = 0.0, ss = 0.0;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nn; l += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = l % B, j = l / B;
        const float v = (float)((((i == j) ? emax[s] : 0.0) - A[base + l]) * scale[s]);
        bf16 h, m, q;
        split3(v, h, m, q);
        xf[base + l] = v;
        hi[base + l] = h;
        mid[base + l] = m;
        if (lo) lo[base + l] = q;
        if (i == j) tr += v;
        ss += (double)v * v;
    }
    block_sum2(tr, ss);
    if (threadIdx.x == 0) {
        stats[2 * ((int64_t)s * gridDim.x + blockIdx.x)] = tr;
        stats[2 * ((int64_t)s * gridDim.x + blockIdx.x) + 1] = ss;
    }
}

// FP64 X_0 (the FP64 path).  grid (x, nb).
__global__ void k_x0d(int64_t B, const double* __restrict__ A, const double* __restrict__ emax,
                      const double* __restrict__ scale, double* __restrict__ X) {
    const int s = blockIdx.y;
    const int64_t base = (int64_t)s * B * B, nn = B * B;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nn; l += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = l % B, j = l / B;
        X[base + l] = (((i == j) ? emax[s] : 0.0) - A[base + l]) * scale[s];
    }
}

// Block s: reduce its `per` partials in a fixed order and run the decision.
__global__ void k_decide_g(SP2State* __restrict__ st, const double* __restrict__ stats, int per,
                           const double* __restrict__ N, const double* __restrict__ tol, double e_asym,
                           const double* __restrict__ e_stag, int maxit, int* __restrict__ active,
                           int* __restrict__ sq) {
    const int s = blockIdx.x;
    if (!st[s].active) return;
    double a = 0.0, b = 0.0;
    for (int p = threadIdx.x; p < per; p += blockDim.x) {
        a += stats[2 * ((int64_t)s * per + p)];
        b += stats[2 * ((int64_t)s * per + p) + 1];
    }
    block_sum2(a, b);
    if (threadIdx.x != 0) return;
    sp2_decide(&st[s], a, b, N[s], tol[s], e_asym, e_stag[s], maxit);
    active[s] = st[s].active;
    sq[s] = st[s].sq_cur;
}

// X (FP64) = the FP32 plane of the system's final pass-1 iterate (parity par[s]).  grid (x, nb).
__global__ void k_f2d_par(int64_t B, const float* __restrict__ x0, const float* __restrict__ x1,
                          const int* __restrict__ par, double* __restrict__ X) {
    const int s = blockIdx.y;
    const int64_t base = (int64_t)s * B * B, nn = B * B;
    const float* x = par[s] ? x1 : x0;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nn; l += (int64_t)gridDim.x * blockDim.x)
        X[base + l] = (double)x[base + l];
}

// Per-block partials of tr X and ||X||^2 (FP64).  grid (nchunk, nb).
__global__ void k_trfrob(int64_t B, const double* __restrict__ X, double* __restrict__ parts) {
    const int s = blockIdx.y;
    const int64_t base = (int64_t)s * B * B, nn = B * B;
    double tr = 0.0, ss = 0.0;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nn; l += (int64_t)gridDim.x * blockDim.x) {
        const double v = X[base + l];
        if (l % B == l / B) tr += v;
        ss += v * v;
    }
    block_sum2(tr, ss);
    if (threadIdx.x == 0) {
        parts[2 * ((int64_t)s * gridDim.x + blockIdx.x)] = tr;
        parts[2 * ((int64_t)s * gridDim.x + blockIdx.x) + 1] = ss;
    }
}

// SP2 update in FP64: mode 1 X = W, 2 X = 2X - W, 0 unchanged.  grid (x, nb).
__global__ void k_sp2_update(int64_t B, const int* __restrict__ mode, const double* __restrict__ W,
                             double* __restrict__ X) {
    const int s = blockIdx.y, md = mode[s];
    if (md == 0) return;
    const int64_t base = (int64_t)s * B * B, nn = B * B;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nn; l += (int64_t)gridDim.x * blockDim.x)
        X[base + l] = md == 1 ? W[base + l] : 2.0 * X[base + l] - W[base + l];
}

// bf16 hi/lo planes of an FP64 array (linear).
__global__ void k_split_d(int64_t count, const double* __restrict__ x, bf16* __restrict__ hi, bf16* __restrict__ lo) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
        const float v = (float)x[k];
        const bf16 h = __float2bfloat16_rn(v);
        hi[k] = h;
        lo[k] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// bf16 hi/lo planes of an FP32 array (linear).
__global__ void k_split_f(int64_t count, const float* __restrict__ x, bf16* __restrict__ hi, bf16* __restrict__ lo) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
        const bf16 h = __float2bfloat16_rn(x[k]);
        hi[k] = h;
        lo[k] = __float2bfloat16_rn(x[k] - __bfloat162float(h));
    }
}

// y += x (FP32, linear).
__global__ void k_add_f(int64_t count, const float* __restrict__ x, float* __restrict__ y) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x)
        y[k] += x[k];
}

// out = alpha_s (W + W^T) + beta_s X per system (stacked row-major FP32 B x B
// blocks), exactly symmetric, with its bf16 hi/lo planes; alpha_s = 0 copies X
// without reading W.  grid (B/32, B/32, nb), block (32, 8).
__global__ void k_sym_update_g(int64_t B, const float* __restrict__ W, const float* __restrict__ X,
                               const float* __restrict__ alpha, const float* __restrict__ beta,
                               float* __restrict__ out, bf16* __restrict__ hi, bf16* __restrict__ lo) {
    __shared__ float t[32][33];
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    const int s = blockIdx.z;
    const int64_t off = (int64_t)s * B * B;
    const float al = alpha[s], be = beta[s];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t i0 = bi * 32, j0 = bj * 32;
#pragma unroll
    for (int k = 0; k < 32; k += 8) t[tx][ty + k] = al != 0.0f ? W[off + (j0 + ty + k) * B + i0 + tx] : 0.0f;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int64_t i = i0 + ty + k, j = j0 + tx;
        const float sw = al != 0.0f ? W[off + i * B + j] + t[ty + k][tx] : 0.0f;
        const float v = al * sw + (be != 0.0f ? be * X[off + i * B + j] : 0.0f);
        if (bi != bj || i <= j) {
            const bf16 h = __float2bfloat16_rn(v);
            out[off + i * B + j] = v;
            hi[off + i * B + j] = h;
            lo[off + i * B + j] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
        t[ty + k][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int64_t j = j0 + ty + k, i = i0 + tx;
        if (bi == bj && j <= i) continue;
        const float v = t[tx][ty + k];
        const bf16 h = __float2bfloat16_rn(v);
        out[off + j * B + i] = v;
        hi[off + j * B + i] = h;
        lo[off + j * B + i] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// Per-block partials of the trace and max |x| of every system's FP32 block.  grid (nchunk, nb).
__global__ void k_trmax(int64_t B, const float* __restrict__ x, double* __restrict__ parts) {
    const int s = blockIdx.y;
    const int64_t base = (int64_t)s * B * B, nn = B * B;
    double tr = 0.0, mx = 0.0;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nn; l += (int64_t)gridDim.x * blockDim.x) {
        const float v = x[base + l];
        if (l % B == l / B) tr += v;
        mx = fmax(mx, (double)fabsf(v));
    }
    __shared__ double sh[2][kThr];
    sh[0][threadIdx.x] = tr;
    sh[1][threadIdx.x] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
            sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        parts[2 * ((int64_t)s * gridDim.x + blockIdx.x)] = sh[0][0];
        parts[2 * ((int64_t)s * gridDim.x + blockIdx.x) + 1] = sh[1][0];
    }
}

// X = X * fac[s] + x1 for the systems with upd[s] (linear; symmetric blocks).  grid (x, nb).
__global__ void k_apply(int64_t B, const float* __restrict__ x1, const double* __restrict__ fac,
                        const int* __restrict__ upd, double* __restrict__ X) {
    const int s = blockIdx.y;
    if (!upd[s]) return;
    const int64_t base = (int64_t)s * B * B, nn = B * B;
    const double f = fac[s];
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < nn; l += (int64_t)gridDim.x * blockDim.x)
        X[base + l] = X[base + l] * f + (double)x1[base + l];
}

// ---- host side --------------------------------------------------------------

// Stacked tile lists: per-system tiles in `unit` x `unit2` blocks, shifted to
// the system's rows, concatenated in the order of `order`.
std::vector<int2> stack(const std::vector<int2>& t, const std::vector<int>& order, int64_t B, int unit_r, int unit_c) {
    std::vector<int2> out;
    out.reserve(t.size() * order.size());
    for (int s : order)
        for (const int2& x : t)
            out.push_back(make_int2((int)(s * B / unit_r) + x.x, (int)(s * B / unit_c) + x.y));
    return out;
}

template <class T>
T* upload(ptbgpu_ctx* c, DevBuf& b, const std::vector<T>& v) {
    b.reserve(sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty())
        PTB_CUDA(cudaMemcpyAsync(b.ptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, c->stream));
    return b.as<T>();
}

unsigned gx(int64_t work, int per_block, int cap) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + per_block - 1) / per_block, cap));
}

struct Chunk {
    int64_t B;
    std::vector<int64_t> ids;   // caller's system indices
};

// One chunk of equal-B systems, all on the device.  dHpk / dSpk: per-system
// device packed inputs; dPpk: per-system device packed outputs.  Marks the
// systems that need the single-system FP64 path in `redo`.
void run_chunk(ptbgpu_ctx* c, const Chunk& ch, const int64_t* ndim, const int64_t* nel,
               const std::vector<const double*>& dHpk, const std::vector<const double*>& dSpk,
               const std::vector<double*>& dPpk, const ptbgpu_opts* o, ptbgpu_stats* st, std::vector<int>& redo,
               int slots) {
    cudaStream_t s = c->stream;
    const int64_t B = ch.B, BB = B * B;
    const int nb = (int)ch.ids.size();
    const int64_t rows = (int64_t)nb * B;
    const bool mixed = o->precision != PTBGPU_PREC_FP64;
    const int maxit = o->max_iter > 0 ? (int)std::min<int64_t>(o->max_iter, kMaxIt) : 100;
    const int refine_rounds = o->refine_rounds > 0 ? (int)o->refine_rounds : 4;
    const double refine_tol = o->refine_tol > 0.0 ? o->refine_tol : 1e-7;
    const int prl = (int)o->print_level;
    const int tp = o->split3_iters >= 0 ? 3 : 2;   // bf16 planes per trajectory iterate
    // phase times of the chunk (print level >= 2; host clock after a stream synchronisation)
    auto tclock = std::chrono::steady_clock::now();
    std::vector<std::pair<const char*, double>> tph;
    auto tmark = [&](const char* what) {
        if (prl < 2) return;
        PTB_CUDA(cudaStreamSynchronize(c->stream));
        const auto now = std::chrono::steady_clock::now();
        tph.push_back({what, std::chrono::duration<double, std::milli>(now - tclock).count()});
        tclock = now;
    };

    // ---- device buffers (grouped slots) ----
    DevBuf& bA = c->buf(B_G0);     // A (FP64), later also P
    DevBuf& bL = c->buf(B_G1);     // Cholesky factors
    DevBuf& bX = c->buf(B_G2);     // X (FP64)
    DevBuf& bW = c->buf(B_G3);     // W (FP64)
    DevBuf& bC = c->buf(B_G4);     // C (FP64)
    DevBuf& bF = c->buf(B_G5);     // FP32 planes: xf0, xf1, x1f0, x1f1, wf
    DevBuf& bP = c->buf(B_G6);     // bf16 planes: x1 hi/lo (x2), C hi/lo, P hi/lo
    DevBuf& bT = c->buf(B_G7);     // bf16 trajectory
    DevBuf& bM = c->buf(B_G8);     // small per-system arrays, tiles, partials
    bA.reserve(8 * (size_t)nb * BB);
    bL.reserve(8 * (size_t)nb * BB);
    bX.reserve(8 * (size_t)nb * BB);
    bW.reserve(8 * (size_t)nb * BB);
    if (mixed) {
        bC.reserve(8 * (size_t)nb * BB);
        bF.reserve(4 * 5 * (size_t)nb * BB);
        bP.reserve(2 * 8 * (size_t)nb * BB);
        bT.reserve(2 * (size_t)tp * slots * nb * BB);
    }
    double* A = bA.as<double>();
    double* L = bL.as<double>();
    double* X = bX.as<double>();
    double* W = bW.as<double>();
    double* Cm = bC.as<double>();
    float* xf[2] = {bF.as<float>(), bF.as<float>() + (size_t)nb * BB};
    float* x1f[2] = {bF.as<float>() + 2 * (size_t)nb * BB, bF.as<float>() + 3 * (size_t)nb * BB};
    float* wf = bF.as<float>() + 4 * (size_t)nb * BB;
    bf16* pl = bP.as<bf16>();
    auto plane = [&](int k) { return pl + (size_t)k * nb * BB; };
    bf16* x1hi[2] = {plane(0), plane(1)};
    bf16* x1lo[2] = {plane(2), plane(3)};
    bf16* chi = plane(4);
    bf16* clo = plane(5);
    bf16* phi = plane(6);
    bf16* plo = plane(7);
    auto traj = [&](int k, int j) { return j < tp ? bT.as<bf16>() + (size_t)(tp * k + j) * nb * BB : nullptr; };

    // ---- unpack, pad, Cholesky, A = L^-1 H L^-T ----
    PTB_CUDA(cudaMemsetAsync(A, 0, 8 * (size_t)nb * BB, s));
    PTB_CUDA(cudaMemsetAsync(L, 0, 8 * (size_t)nb * BB, s));
    std::vector<int> nsys(nb);
    for (int q = 0; q < nb; ++q) {
        const int64_t i = ch.ids[q];
        nsys[q] = (int)ndim[i];
        unpack_sym(s, ndim[i], B, dHpk[q], A + q * BB, o->filter);
        unpack_sym(s, ndim[i], B, dSpk[q], L + q * BB, o->filter);
    }
    // small per-system device arrays in one buffer
    enum { M_NSYS = 0, M_EMAX, M_SCALE, M_N, M_TOL, M_ESTAG, M_ACTIVE, M_SQ, M_PAR, M_MODE, M_FAC, M_UPD, M_INFO,
           M_COUNT };
    bM.reserve(64 * (size_t)M_COUNT * (nb + 1) + 16 * (size_t)nb * sizeof(void*));
    auto marr = [&](int k) { return (char*)bM.ptr + (size_t)k * 8 * (nb + 1); };
    int* d_nsys = (int*)marr(M_NSYS);
    double* d_emax = (double*)marr(M_EMAX);
    double* d_scale = (double*)marr(M_SCALE);
    double* d_N = (double*)marr(M_N);
    double* d_tol = (double*)marr(M_TOL);
    double* d_estag = (double*)marr(M_ESTAG);
    int* d_active = (int*)marr(M_ACTIVE);
    int* d_sq = (int*)marr(M_SQ);
    int* d_par = (int*)marr(M_PAR);
    int* d_mode = (int*)marr(M_MODE);
    double* d_fac = (double*)marr(M_FAC);
    int* d_upd = (int*)marr(M_UPD);
    int* d_info = (int*)marr(M_INFO);
    const double** d_ptrA = (const double**)marr(M_COUNT);
    double** d_ptrB = (double**)(d_ptrA + nb);
    PTB_CUDA(cudaMemcpyAsync(d_nsys, nsys.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
    const dim3 gpad(gx(B, kThr, 64), nb);
    k_pad_diag<<<gpad, kThr, 0, s>>>(B, d_nsys, L, nullptr, 1.0);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    {
        int lwork = 0;
        PTB_CUSOLVER(cusolverDnDpotrf_bufferSize(c->solver, CUBLAS_FILL_MODE_LOWER, (int)B, L, (int)B, &lwork));
        DevBuf& ws = c->buf(B_SOLVER_WS);
        ws.reserve(sizeof(double) * (size_t)std::max(lwork, 1));
        for (int q = 0; q < nb; ++q)
            PTB_CUSOLVER(cusolverDnDpotrf(c->solver, CUBLAS_FILL_MODE_LOWER, (int)B, L + q * BB, (int)B,
                                          ws.as<double>(), lwork, d_info + q));
    }
    std::vector<int> info(nb);
    PTB_CUDA(cudaMemcpyAsync(info.data(), d_info, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nb; ++q)
        PTB_CHECK(info[q] == 0, PTBGPU_ENOTSPD, "system %lld: overlap matrix not positive definite (potrf info=%d)",
                  (long long)ch.ids[q], info[q]);
    std::vector<const double*> hpa(nb);
    std::vector<double*> hpb(nb);
    for (int q = 0; q < nb; ++q) {
        hpa[q] = L + q * BB;
        hpb[q] = A + q * BB;
    }
    PTB_CUDA(cudaMemcpyAsync(d_ptrA, hpa.data(), sizeof(void*) * nb, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(d_ptrB, hpb.data(), sizeof(void*) * nb, cudaMemcpyHostToDevice, s));
    const double one = 1.0, two = 2.0, zero = 0.0;
    // triangular solves with every system's L: one batched call for small systems,
    // one call per system from B = 1024 on (where the batched routine is slower)
    auto trsm_all = [&](cublasSideMode_t side, cublasOperation_t op, double alpha) {
        if (B < 1024) {
            PTB_CUBLAS(cublasDtrsmBatched(c->blas, side, CUBLAS_FILL_MODE_LOWER, op, CUBLAS_DIAG_NON_UNIT, (int)B,
                                          (int)B, &alpha, d_ptrA, (int)B, d_ptrB, (int)B, nb));
        } else {
            for (int q = 0; q < nb; ++q)
                PTB_CUBLAS(cublasDtrsm(c->blas, side, CUBLAS_FILL_MODE_LOWER, op, CUBLAS_DIAG_NON_UNIT, (int)B,
                                       (int)B, &alpha, hpa[q], (int)B, hpb[q], (int)B));
        }
    };
    trsm_all(CUBLAS_SIDE_LEFT, CUBLAS_OP_N, one);
    trsm_all(CUBLAS_SIDE_RIGHT, CUBLAS_OP_T, one);
    const dim3 g32((unsigned)(B / 32), (unsigned)(B / 32), (unsigned)nb), b32(32, 8);
    k_sym_lower<<<g32, b32, 0, s>>>(B, A);
    count_launch();
    PTB_CUDA(cudaGetLastError());

    // ---- per-system spectral bounds; padded diagonal at e_max ----
    const int ng = (int)std::min<int64_t>(B, 64);
    DevBuf& bparts = c->buf(B_STATS);
    const int nchunk = (int)std::max<int64_t>(1, std::min<int64_t>(B * B / (kThr * 16), 64));
    const std::vector<int2> up = tc::make_tiles(B, true, 256), up3 = tc::make_tiles(B, true, 128),
                            all = tc::make_tiles(B, false, 256), pup = tc::make_pair_tiles(B, true),
                            pall = tc::make_pair_tiles(B, false);
    const int T1 = (int)up.size(), T3 = (int)up3.size(), TF = (int)all.size();
    bparts.reserve(sizeof(double) * 2 * (size_t)nb * std::max({T1, T3, TF, ng, nchunk}));
    double* parts = bparts.as<double>();
    k_gersh<<<dim3(ng, nb), kThr, 0, s>>>(B, d_nsys, A, parts, parts + (size_t)nb * ng);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    std::vector<double> hg(2 * (size_t)nb * ng);
    PTB_CUDA(cudaMemcpyAsync(hg.data(), parts, sizeof(double) * hg.size(), cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    std::vector<double> emin(nb), emax(nb), scale(nb), Nv(nb), tol(nb), estag(nb);
    for (int q = 0; q < nb; ++q) {
        double lo = INFINITY, hi = -INFINITY;
        for (int b = 0; b < ng; ++b) {
            lo = std::min(lo, hg[(size_t)q * ng + b]);
            hi = std::max(hi, hg[(size_t)nb * ng + (size_t)q * ng + b]);
        }
        PTB_CHECK(std::isfinite(lo) && std::isfinite(hi) && hi > lo, PTBGPU_ENAN,
                  "system %lld: invalid spectral bounds [%g, %g]", (long long)ch.ids[q], lo, hi);
        emin[q] = lo;
        emax[q] = hi;
        scale[q] = 1.0 / (hi - lo);
        Nv[q] = 0.5 * (double)nel[ch.ids[q]];
        tol[q] = 1e-12 * (double)nsys[q];
        estag[q] = 0.01 * (double)nsys[q];
    }
    PTB_CUDA(cudaMemcpyAsync(d_emax, emax.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(d_scale, scale.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(d_N, Nv.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(d_tol, tol.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(d_estag, estag.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
    k_pad_diag<<<gpad, kThr, 0, s>>>(B, d_nsys, A, d_emax, 0.0);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    tmark("prologue");

    const int gel = (int)std::min<int64_t>(148 * 4, std::max<int64_t>(1, B * B / 4096));   // x-blocks of elementwise kernels
    const dim3 gE(gel, nb);
    std::vector<int> kfin(nb, 0), conv(nb, 0);
    std::vector<SP2State> hst(nb);
    std::vector<int> rounds(nb, 0), nclean(nb, 0);

    // FP64 cleanup / FP64 purification on X: SP2 steps with per-system stop rules.
    // fp64_path: the whole purification (stop e < 1e-13 n, or e < 1e-2 not falling over two
    // steps, up to maxit); otherwise the cleanup rule (e < 1e-13 n, not falling over two steps,
    // at most 8 steps).  Only systems with sel[q] take part.
    auto fp64_steps = [&](const std::vector<int>& sel, bool fp64_path) {
        std::vector<std::vector<double>> hist(nb);
        std::vector<int> done(nb, 0), steps(nb, 0), mode(nb, 0);
        std::vector<double> hp(2 * (size_t)nb * nchunk);
        const int cap = fp64_path ? maxit : 8;
        for (int it = 0;; ++it) {
            k_trfrob<<<dim3(nchunk, nb), kThr, 0, s>>>(B, X, parts);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            PTB_CUDA(cudaMemcpyAsync(hp.data(), parts, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s));
            PTB_CUDA(cudaStreamSynchronize(s));
            bool any = false;
            for (int q = 0; q < nb; ++q) {
                mode[q] = 0;
                if (!sel[q] || done[q]) continue;
                double trX = 0.0, trX2 = 0.0;
                for (int b = 0; b < nchunk; ++b) {
                    trX += hp[2 * ((size_t)q * nchunk + b)];
                    trX2 += hp[2 * ((size_t)q * nchunk + b) + 1];
                }
                const double err = trX - trX2, e = std::fabs(err);
                if (!std::isfinite(err)) {   // left to the single-system path
                    done[q] = 1;
                    conv[q] = 0;
                    redo[ch.ids[q]] = 1;
                    continue;
                }
                hist[q].push_back(e);
                const auto& h = hist[q];
                const bool flat = h.size() > 2 && e >= h[h.size() - 3] && (!fp64_path || e < 1e-2);
                if (e < 1e-13 * (double)nsys[q] || flat || steps[q] >= cap) {
                    done[q] = 1;
                    if (fp64_path && !(e < 1e-13 * (double)nsys[q] || flat)) conv[q] = 0;
                    continue;
                }
                mode[q] = std::fabs(trX2 - Nv[q]) <= std::fabs(2.0 * trX - trX2 - Nv[q]) ? 1 : 2;
                ++steps[q];
                any = true;
            }
            if (!any) break;
            PTB_CUDA(cudaMemcpyAsync(d_mode, mode.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
            if (B < 1024) {
                PTB_CUBLAS(cublasDgemmStridedBatched(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)B, (int)B, (int)B, &one,
                                                     X, (int)B, BB, X, (int)B, BB, &zero, W, (int)B, BB, nb));
            } else {
                // symmetric squares of the systems that step (half the flops of a GEMM)
                for (int q = 0; q < nb; ++q)
                    if (mode[q]) dsyrk_sq(c, B, B, X + q * BB, W + q * BB);
            }
            k_sp2_update<<<gE, kThr, 0, s>>>(B, d_mode, W, X);
            count_launch();
            PTB_CUDA(cudaGetLastError());
        }
        for (int q = 0; q < nb; ++q) nclean[q] += steps[q];
    };

    if (!mixed) {
        k_x0d<<<gE, kThr, 0, s>>>(B, A, d_emax, d_scale, X);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        std::fill(conv.begin(), conv.end(), 1);
        fp64_steps(std::vector<int>(nb, 1), true);
        for (int q = 0; q < nb; ++q)
            if (!conv[q]) redo[ch.ids[q]] = 1;
    } else {
        // ---- pass 1: stacked tcgen05 SP2 ----
        const int cap = std::min(maxit, slots - 1);
        std::vector<int> order(nb);
        std::iota(order.begin(), order.end(), 0);
        const std::vector<int2> t_up = stack(up, order, B, 128, 256), t_up3 = stack(up3, order, B, 128, 128),
                                t_pup = stack(pup, order, B, 256, 256);
        DevBuf& btl = c->buf(B_TILES);
        btl.reserve(sizeof(int2) * (t_up.size() + t_up3.size() + t_pup.size() + 2 * (size_t)nb * (TF + TF)));
        int2* d_up = btl.as<int2>();
        int2* d_up3 = d_up + t_up.size();
        int2* d_pup = d_up3 + t_up3.size();
        int2* d_all = d_pup + t_pup.size();
        int2* d_pall = d_all + (size_t)nb * TF;
        PTB_CUDA(cudaMemcpyAsync(d_up, t_up.data(), sizeof(int2) * t_up.size(), cudaMemcpyHostToDevice, s));
        PTB_CUDA(cudaMemcpyAsync(d_up3, t_up3.data(), sizeof(int2) * t_up3.size(), cudaMemcpyHostToDevice, s));
        PTB_CUDA(cudaMemcpyAsync(d_pup, t_pup.data(), sizeof(int2) * t_pup.size(), cudaMemcpyHostToDevice, s));
        DevBuf& bstate = c->buf(B_G9);
        bstate.reserve(sizeof(SP2State) * nb);
        SP2State* d_state = bstate.as<SP2State>();
        std::vector<SP2State> init(nb);
        for (auto& x : init) {
            memset(&x, 0, sizeof(x));
            x.active = 1;
        }
        PTB_CUDA(cudaMemcpyAsync(d_state, init.data(), sizeof(SP2State) * nb, cudaMemcpyHostToDevice, s));
        PTB_CUDA(cudaMemsetAsync(&c->flags->timeout, 0, sizeof(int), s));
        k_x0<<<dim3(nchunk, nb), kThr, 0, s>>>(B, A, d_emax, d_scale, xf[0], traj(0, 0), traj(0, 1), traj(0, 2),
                                               parts);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        const double e_asym = 0.1;
        k_decide_g<<<nb, kThr, 0, s>>>(d_state, parts, nchunk, d_N, d_tol, e_asym, d_estag, cap, d_active, d_sq);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        tc::ProdList split3{3, {0, 0, 1}, {0, 1, 0}};
        tc::ProdList split6{6, {0, 0, 1, 0, 2, 1}, {0, 1, 0, 2, 0, 1}};
        tc::EpiParams ep{};
        ep.active = d_active;
        ep.sq_flag = d_sq;
        ep.stacked = 1;
        ep.err = &c->flags->timeout;
        ep.ld = B;
        ep.stats = parts;
        const int64_t split3_iters = o->split3_iters;
        auto three_planes = [&](int k) { return split3_iters < 0 ? false : (split3_iters == 0 || k < split3_iters); };
        std::vector<int> hact(nb);
        for (int k = 0; k < cap; ++k) {
            ep.xcur = xf[k & 1];
            ep.out = xf[(k + 1) & 1];
            ep.hi = traj(k + 1, 0);
            ep.lo = traj(k + 1, 1);
            ep.lo2 = traj(k + 1, 2);
            const void* pk[3] = {traj(k, 0), traj(k, 1), traj(k, 2)};
            int per;
            if (three_planes(k)) {
                const int n = tc::launch_product(s, tc::EPI_SP2, 3, B, pk, pk, split6, d_up3, nb * T3, ep, 0, nullptr,
                                                 0, rows);
                PTB_CHECK(n == nb * T3, PTBGPU_ECUDA, "unexpected partial count");
                per = T3;
            } else {
                const int n = tc::launch_product(s, tc::EPI_SP2, 2, B, pk, pk, split3, d_up, nb * T1, ep, 0, d_pup,
                                                 (int)t_pup.size(), rows);
                PTB_CHECK(n == nb * T1, PTBGPU_ECUDA, "unexpected partial count");
                per = T1;
            }
            PTB_CUDA(cudaGetLastError());
            k_decide_g<<<nb, kThr, 0, s>>>(d_state, parts, per, d_N, d_tol, e_asym, d_estag, cap, d_active, d_sq);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            if ((k & 3) == 3 || k + 1 == cap) {
                PTB_CUDA(cudaMemcpyAsync(hact.data(), d_active, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
                PTB_CUDA(cudaStreamSynchronize(s));
                if (std::all_of(hact.begin(), hact.end(), [](int v) { return v == 0; })) break;
            }
        }
        int tmo = 0;
        PTB_CUDA(cudaMemcpyAsync(hst.data(), d_state, sizeof(SP2State) * nb, cudaMemcpyDeviceToHost, s));
        PTB_CUDA(cudaMemcpyAsync(&tmo, &c->flags->timeout, sizeof(int), cudaMemcpyDeviceToHost, s));
        PTB_CUDA(cudaStreamSynchronize(s));
        PTB_CHECK(tmo == 0, PTBGPU_ETIMEOUT, "tensor-core product gave up waiting (site %d)", tmo);
        std::vector<int> par(nb), sel(nb);
        int Kmax = 0;
        for (int q = 0; q < nb; ++q) {
            conv[q] = hst[q].converged && hst[q].status == 0;
            kfin[q] = conv[q] ? hst[q].next : 0;
            par[q] = kfin[q] & 1;
            sel[q] = conv[q];
            if (!conv[q]) redo[ch.ids[q]] = 1;
            Kmax = std::max(Kmax, kfin[q]);
            log_line(prl, 2, " grouped SP2: system %lld  iterations %d  final err %.3e%s", (long long)ch.ids[q],
                     kfin[q], conv[q] ? hst[q].err[kfin[q]] : 0.0, conv[q] ? "" : "  (not converged)");
        }
        tmark("pass 1");
        PTB_CUDA(cudaMemcpyAsync(d_par, par.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
        k_f2d_par<<<gE, kThr, 0, s>>>(B, xf[0], xf[1], d_par, X);
        count_launch();
        PTB_CUDA(cudaGetLastError());
        fp64_steps(sel, false);
        tmark("cleanup");

        // ---- refinement rounds (stacked) ----
        // replay order: longest pass 1 first, so the systems still replaying at step k are a prefix
        // (each round's tile lists hold only the systems that take part in it)
        std::vector<int> rorder;
        const int TP = (int)pall.size();
        tc::EpiParams epf{};
        epf.err = &c->flags->timeout;
        epf.ld = B;
        epf.stacked = 1;
        epf.out = wf;
        auto full_product = [&](const void* const* a, const void* const* b, int nsys_active, float* out) {
            tc::EpiParams e = epf;
            e.out = out;
            tc::launch_product(s, tc::EPI_FULL, 2, B, a, b, split3, d_all, nsys_active * TF, e, 0, d_pall,
                               nsys_active * TP, rows);
            PTB_CUDA(cudaGetLastError());
        };
        // coefficient table of the symmetric updates, uploaded once: row 0 X1_0 = scale (W + W^T),
        // rows 1..Kmax the replay's branches (identity once a system's pass 1 has ended),
        // row Kmax+1 the projection, row Kmax+2 the idempotency term
        const int ncoef = Kmax + 3;
        std::vector<float> coef(2 * (size_t)ncoef * nb);
        auto set_coef = [&](int row, int q, float al, float be) {
            coef[2 * (size_t)row * nb + q] = al;
            coef[2 * (size_t)row * nb + nb + q] = be;
        };
        for (int q = 0; q < nb; ++q) {
            set_coef(0, q, (float)scale[q], 0.0f);
            for (int k = 0; k < Kmax; ++k) {
                if (k < kfin[q]) {
                    const bool sq = hst[q].sq[k] != 0;
                    set_coef(1 + k, q, sq ? 1.0f : -1.0f, sq ? 0.0f : 2.0f);
                } else {
                    set_coef(1 + k, q, 0.0f, 1.0f);
                }
            }
            set_coef(Kmax + 1, q, 1.0f, -2.0f);
            set_coef(Kmax + 2, q, -1.0f, 1.0f);
        }
        DevBuf& bcoef = c->buf(B_G10);
        float* d_coef = upload(c, bcoef, coef);
        auto calpha = [&](int row) { return d_coef + 2 * (size_t)row * nb; };
        auto cbeta = [&](int row) { return d_coef + 2 * (size_t)row * nb + nb; };
        std::vector<double> g1(nb, 0.0), prevmax(nb, 0.0), resid(nb, 0.0), fac(nb, 1.0);
        std::vector<int> need(nb), upd(nb);
        for (int q = 0; q < nb; ++q) need[q] = conv[q];
        std::vector<double> hp(2 * (size_t)nb * nchunk), hp0(2 * (size_t)nb * nchunk);
        const int64_t cnt = (int64_t)nb * BB;
        const unsigned gl = gx(cnt, kThr, 148 * 16);
        while (std::any_of(need.begin(), need.end(), [](int v) { return v != 0; })) {
            rorder.clear();
            for (int q = 0; q < nb; ++q)
                if (need[q]) rorder.push_back(q);
            std::stable_sort(rorder.begin(), rorder.end(), [&](int x, int y) { return kfin[x] > kfin[y]; });
            const int na = (int)rorder.size();
            const std::vector<int2> t_all = stack(all, rorder, B, 128, 256), t_pall = stack(pall, rorder, B, 256, 256);
            PTB_CUDA(cudaMemcpyAsync(d_all, t_all.data(), sizeof(int2) * t_all.size(), cudaMemcpyHostToDevice, s));
            PTB_CUDA(cudaMemcpyAsync(d_pall, t_pall.data(), sizeof(int2) * t_pall.size(), cudaMemcpyHostToDevice, s));
            int kmax_r = 0;
            for (int q : rorder) kmax_r = std::max(kmax_r, kfin[q]);
            // C = A X - X A; planes of C (as C^T) and X
            PTB_CUBLAS(cublasDgemmStridedBatched(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)B, (int)B, (int)B, &one, A,
                                                 (int)B, BB, X, (int)B, BB, &zero, W, (int)B, BB, nb));
            k_antisym_g<<<g32, b32, 0, s>>>(B, W, Cm);
            count_launch();
            k_split_d<<<gl, kThr, 0, s>>>(cnt, Cm, chi, clo);
            count_launch();
            k_split_d<<<gl, kThr, 0, s>>>(cnt, X, phi, plo);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            const void* pc[2] = {chi, clo};
            const void* pp[2] = {phi, plo};
            full_product(pc, pp, na, wf);   // wf = C^T P = -C P
            k_sym_update_g<<<g32, b32, 0, s>>>(B, wf, x1f[1], calpha(0), cbeta(0), x1f[0], x1hi[0], x1lo[0]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            k_trmax<<<dim3(nchunk, nb), kThr, 0, s>>>(B, x1f[0], parts);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            PTB_CUDA(cudaMemcpyAsync(hp0.data(), parts, sizeof(double) * hp0.size(), cudaMemcpyDeviceToHost, s));
            // replay over the recorded branches
            // (up to the longest pass 1 of this round's systems; shorter ones carry X1 over)
            for (int k = 0; k < kmax_r; ++k) {
                const int a = k & 1, b = a ^ 1;
                int m = 0;
                while (m < na && kfin[rorder[m]] > k) ++m;
                const void* p0[2] = {traj(k, 0), traj(k, 1)};
                const void* p1[2] = {x1hi[a], x1lo[a]};
                if (m > 0) full_product(p0, p1, m, wf);
                k_sym_update_g<<<g32, b32, 0, s>>>(B, wf, x1f[a], calpha(1 + k), cbeta(1 + k), x1f[b], x1hi[b],
                                                   x1lo[b]);
                count_launch();
                PTB_CUDA(cudaGetLastError());
            }
            // projection onto the occupied-virtual blocks and the second-order idempotency term
            const int a = kmax_r & 1, b = a ^ 1;
            const void* ppx[2] = {x1hi[a], x1lo[a]};
            full_product(pp, ppx, na, wf);                                  // W = P X1
            k_split_f<<<gl, kThr, 0, s>>>(cnt, wf, x1hi[b], x1lo[b]);
            count_launch();
            const void* pw[2] = {x1hi[b], x1lo[b]};
            full_product(pw, pp, na, x1f[b]);                               // W P
            k_sym_update_g<<<g32, b32, 0, s>>>(B, wf, x1f[b], calpha(Kmax + 1), cbeta(Kmax + 1), x1f[a], x1hi[a],
                                               x1lo[a]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            const void* px1[2] = {x1hi[a], x1lo[a]};
            full_product(px1, px1, na, x1f[b]);                             // Y = X1^2
            k_split_f<<<gl, kThr, 0, s>>>(cnt, x1f[b], x1hi[b], x1lo[b]);
            count_launch();
            const void* py[2] = {x1hi[b], x1lo[b]};
            full_product(pp, py, na, wf);                                   // W2 = P Y
            k_add_f<<<gl, kThr, 0, s>>>(cnt, x1f[a], x1f[b]);                // Y + X1
            count_launch();
            k_sym_update_g<<<g32, b32, 0, s>>>(B, wf, x1f[b], calpha(Kmax + 2), cbeta(Kmax + 2), x1f[a], x1hi[a],
                                               x1lo[a]);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            // trace correction and the size of the correction, per system
            k_trmax<<<dim3(nchunk, nb), kThr, 0, s>>>(B, x1f[a], parts);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            PTB_CUDA(cudaMemcpyAsync(hp.data(), parts, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s));
            PTB_CUDA(cudaMemcpyAsync(&tmo, &c->flags->timeout, sizeof(int), cudaMemcpyDeviceToHost, s));
            PTB_CUDA(cudaStreamSynchronize(s));
            PTB_CHECK(tmo == 0, PTBGPU_ETIMEOUT, "tensor-core product gave up waiting (site %d)", tmo);
            std::vector<int> next(nb, 0);
            for (int q = 0; q < nb; ++q) {
                upd[q] = need[q];
                if (!need[q]) continue;
                double tau = 0.0, x1max = 0.0, x10max = 0.0;
                for (int bb = 0; bb < nchunk; ++bb) {
                    tau += hp[2 * ((size_t)q * nchunk + bb)];
                    x1max = std::max(x1max, hp[2 * ((size_t)q * nchunk + bb) + 1]);
                    x10max = std::max(x10max, hp0[2 * ((size_t)q * nchunk + bb) + 1]);
                }
                fac[q] = 1.0 - tau / Nv[q];
                ++rounds[q];
                const double gain = x10max > 0.0 ? x1max / x10max : 0.0;
                double rho;
                if (rounds[q] == 1) {
                    g1[q] = gain;
                    rho = x10max > 0.0 ? std::min(1.0, kRho1 * g1[q]) : 1.0;
                } else {
                    rho = std::min(1.0, std::max(kRho2 * g1[q], prevmax[q] > 0.0 ? x1max / prevmax[q] : 1.0));
                }
                prevmax[q] = x1max;
                resid[q] = x1max * rho;
                log_line(prl, 2, " grouped refinement: system %lld round %d  max|X1| %.3e  gain %.3e  predicted %.3e",
                         (long long)ch.ids[q], rounds[q], x1max, gain, resid[q]);
                if (!(resid[q] > refine_tol)) continue;
                if (rounds[q] >= refine_rounds || std::min(1.0, kRho2 * g1[q]) > 0.5) {
                    if (resid[q] > 10.0 * refine_tol) {
                        redo[ch.ids[q]] = 1;
                        upd[q] = 0;
                    }
                    continue;
                }
                next[q] = 1;
            }
            PTB_CUDA(cudaMemcpyAsync(d_fac, fac.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
            PTB_CUDA(cudaMemcpyAsync(d_upd, upd.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
            k_apply<<<gE, kThr, 0, s>>>(B, x1f[a], d_fac, d_upd, X);
            count_launch();
            PTB_CUDA(cudaGetLastError());
            PTB_CUDA(cudaStreamSynchronize(s));
            need = next;
            tmark("refinement round");
            if (std::any_of(need.begin(), need.end(), [](int v) { return v != 0; })) {
                fp64_steps(need, false);
                tmark("cleanup");
            }
        }
    }

    // ---- P = 2 L^-T X L^-1, packed per system ----
    for (int q = 0; q < nb; ++q) hpb[q] = X + q * BB;
    PTB_CUDA(cudaMemcpyAsync(d_ptrB, hpb.data(), sizeof(void*) * nb, cudaMemcpyHostToDevice, s));
    trsm_all(CUBLAS_SIDE_LEFT, CUBLAS_OP_T, two);
    trsm_all(CUBLAS_SIDE_RIGHT, CUBLAS_OP_N, one);
    for (int q = 0; q < nb; ++q) pack_cols(s, nsys[q], B, X + q * BB, dPpk[q]);
    PTB_CUDA(cudaStreamSynchronize(s));
    tmark("back-transform");
    if (prl >= 2) {
        std::string line;
        char buf[96];
        for (const auto& x : tph) {
            snprintf(buf, sizeof(buf), "  %s %.1f", x.first, x.second);
            line += buf;
        }
        log_line(prl, 2, " grouped chunk B=%lld systems=%d (ms):%s", (long long)B, nb, line.c_str());
    }
    for (int q = 0; q < nb; ++q) {
        ptbgpu_stats* t = st ? &st[ch.ids[q]] : nullptr;
        if (!t) continue;
        const double n3 = (double)nsys[q] * nsys[q] * nsys[q];
        t->iterations = kfin[q] + nclean[q];
        t->refine_rounds = rounds[q];
        t->flops = (1.0 / 3.0 + 4.0) * n3 + (double)(kfin[q] + nclean[q]) * n3 +
                   (double)rounds[q] * (2.0 + 2.0 * (kfin[q] + 5)) * n3;
    }
}

}  // namespace

// Grouped trace-correcting purification of ninst independent systems (host
// packed arrays in and out).  Systems the grouped path cannot finish (pass 1
// not converged, refinement rounds short of refine_tol) are redone one by one
// by the single-system path in FP64.
void tc_purify_grouped(ptbgpu_ctx* c, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                       const double* const* Hpk, const double* const* Spk, double* const* Ppk, const ptbgpu_opts* o,
                       ptbgpu_stats* st, std::vector<int>& redo) {
    redo.assign((size_t)ninst, 0);
    for (int64_t i = 0; i < ninst; ++i) {
        PTB_CHECK(ndim[i] > 0 && nel[i] > 0 && nel[i] <= 2 * ndim[i] && nel[i] % 2 == 0 && Hpk[i] && Spk[i] && Ppk[i],
                  PTBGPU_EINVAL, "system %lld: bad sizes ndim=%lld nel=%lld (nel must be even)", (long long)i,
                  (long long)ndim[i], (long long)nel[i]);
    }
    PTB_CHECK(o->refine_rounds >= 0 && o->refine_rounds <= 16 && o->refine_tol >= 0.0, PTBGPU_EINVAL,
              "refine_rounds must be 0..16 and refine_tol >= 0");
    cudaStream_t s = c->stream;
    const bool mixed = o->precision != PTBGPU_PREC_FP64;
    const int maxit = o->max_iter > 0 ? (int)std::min<int64_t>(o->max_iter, kMaxIt) : 100;
    const int slots = std::min(maxit, 90) + 1;
    // buckets of equal padded dimension, chunks bounded by device memory
    std::vector<int64_t> idx((size_t)ninst);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return ndim[a] > ndim[b]; });
    size_t free_b = 0, total_b = 0;
    PTB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const double budget = 0.6 * (double)free_b;
    std::vector<Chunk> chunks;
    for (size_t p = 0; p < idx.size();) {
        const int64_t B = round_up(ndim[idx[p]], 256);
        const double per = (double)B * B * (mixed ? 88.0 + 2.0 * (o->split3_iters >= 0 ? 3 : 2) * slots : 40.0) +
                           24.0 * (double)B * B;
        Chunk ch{B, {}};
        while (p < idx.size() && round_up(ndim[idx[p]], 256) == B &&
               (ch.ids.empty() || (double)(ch.ids.size() + 1) * per <= budget)) {
            ch.ids.push_back(idx[p]);
            ++p;
        }
        chunks.push_back(ch);
    }
    DevBuf& bin = c->buf(B_PK0);
    DevBuf& bout = c->buf(B_PK1);
    for (const Chunk& ch : chunks) {
        size_t tot = 0;
        for (int64_t i : ch.ids) tot += (size_t)npacked(ndim[i]);
        bin.reserve(sizeof(double) * 2 * tot);
        bout.reserve(sizeof(double) * tot);
        std::vector<const double*> dH, dS;
        std::vector<double*> dP;
        size_t off = 0;
        for (int64_t i : ch.ids) {
            const size_t np = (size_t)npacked(ndim[i]);
            double* h = bin.as<double>() + 2 * off;
            double* sm = h + np;
            PTB_CUDA(cudaMemcpyAsync(h, Hpk[i], sizeof(double) * np, cudaMemcpyHostToDevice, s));
            PTB_CUDA(cudaMemcpyAsync(sm, Spk[i], sizeof(double) * np, cudaMemcpyHostToDevice, s));
            dH.push_back(h);
            dS.push_back(sm);
            dP.push_back(bout.as<double>() + off);
            off += np;
        }
        run_chunk(c, ch, ndim, nel, dH, dS, dP, o, st, redo, slots);
        for (size_t q = 0; q < ch.ids.size(); ++q) {
            const int64_t i = ch.ids[q];
            if (!redo[i])
                PTB_CUDA(cudaMemcpyAsync(Ppk[i], dP[q], sizeof(double) * (size_t)npacked(ndim[i]),
                                         cudaMemcpyDeviceToHost, s));
        }
        PTB_CUDA(cudaStreamSynchronize(s));
    }
    // the grouped working set is large: give it back
    for (int b = B_G0; b <= B_G10; ++b) c->buf(b).release();
}

}  // namespace ptb
