// Long-range damping of the exchange-correlation term in the second SCF
// iteration of PTB (source/pgtb.f90:482-513): the first consumer of the density
// matrix the density step returns.  With the special radius rad(a) of atom a,
// the per-AO scale hao(i) = shell_cnf2(shell, element) * gq(atom) and the
// per-AO diagonal factor xdiag(i) = shell_xi(8, element) (both formed by the
// caller from the parameter tables, as the reference's loops do inline):
//
//   xab(lin(a,b)) = (1 + erf(-1.8 (rab(lin(a,b)) - r) / r)) / 2,  r = rad(a) + rad(b)
//   H(k) += P(k) (hao(i) + hao(j)) xab(lin(aoat(j), aoat(i)))      k = lin(j,i), j < i
//   H(k) += 2 P(k) xdiag(i) hao(i) xab(lin(aoat(i), aoat(i)))      k = lin(i,i)
//
// on the packed arrays (lin(j,i) = i(i-1)/2 + j, 1-based).  The atom-pair table
// is small (9 MB at 1536 atoms) and stays in L2; the AO-pair update streams
// P and H once: 24 bytes of HBM traffic per packed element.  Products and sums
// are rounded one by one in the reference's order (no fused multiply-add), so
// the update equals a straightforward FP64 evaluation up to the last bit of erf
// and of r (the reference adds the second atom's two radius terms to rad(a)
// one at a time).
#include <cmath>

#include "common.cuh"

namespace ptb {

namespace {

// One block per atom column a (rows b <= a of the packed atom-pair arrays).
__global__ void k_xab(int64_t nat, const double* __restrict__ rab, const double* __restrict__ rad,
                      double* __restrict__ xab) {
    for (int64_t a = blockIdx.x; a < nat; a += gridDim.x) {
        const int64_t base = a * (a + 1) / 2;
        const double ra = rad[a];
        for (int64_t b = threadIdx.x; b <= a; b += blockDim.x) {
            const double r = __dadd_rn(ra, rad[b]);
            const double t8 = __ddiv_rn(__dsub_rn(rab[base + b], r), r);
            xab[base + b] = __dmul_rn(0.5, __dadd_rn(1.0, erf(__dmul_rn(-1.8, t8))));
        }
    }
}

// AO-pair update of one packed element k in column i, row j (0-based).
__device__ __forceinline__ double xc_add(int64_t i, int64_t j, double p, const int64_t* __restrict__ aoat,
                                         const double* __restrict__ hao, const double* __restrict__ xdiag,
                                         const double* __restrict__ xab) {
    const int64_t ia = aoat[i] - 1, ib = aoat[j] - 1;
    const int64_t hi = ia > ib ? ia : ib, lo = ia > ib ? ib : ia;
    const double x = xab[hi * (hi + 1) / 2 + lo];
    if (j < i) return __dmul_rn(__dmul_rn(p, __dadd_rn(hao[i], hao[j])), x);
    return __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, p), xdiag[i]), hao[i]), x);
}

// Column of packed element k (0-based): an FP64 square root, corrected by integer steps.
__device__ __forceinline__ int64_t packed_col(int64_t k) {
    int64_t i = (int64_t)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
    while (i > 0 && i * (i + 1) / 2 > k) --i;
    while ((i + 1) * (i + 2) / 2 <= k) ++i;
    return i;
}

// Two consecutive packed elements per thread and step (16-byte loads and
// stores of P and H; the arrays start 16-byte aligned), the second one's
// column found from the first's; an odd last element is done by thread 0.
__global__ void k_xc_update(int64_t ndim, const int64_t* __restrict__ aoat, const double* __restrict__ hao,
                            const double* __restrict__ xdiag, const double* __restrict__ xab,
                            const double* __restrict__ P, double* __restrict__ H) {
    const int64_t np = ndim * (ndim + 1) / 2, npairs = np / 2;
    const double2* P2 = reinterpret_cast<const double2*>(P);
    double2* H2 = reinterpret_cast<double2*>(H);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < npairs;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = 2 * q;
        const int64_t i0 = packed_col(k), j0 = k - i0 * (i0 + 1) / 2;
        const int64_t i1 = j0 + 1 > i0 ? i0 + 1 : i0, j1 = j0 + 1 > i0 ? 0 : j0 + 1;
        const double2 p = P2[q];
        double2 h = H2[q];
        h.x = __dadd_rn(h.x, xc_add(i0, j0, p.x, aoat, hao, xdiag, xab));
        h.y = __dadd_rn(h.y, xc_add(i1, j1, p.y, aoat, hao, xdiag, xab));
        H2[q] = h;
    }
    if ((np & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const int64_t k = np - 1, i = packed_col(k);
        H[k] = __dadd_rn(H[k], xc_add(i, k - i * (i + 1) / 2, P[k], aoat, hao, xdiag, xab));
    }
}

}  // namespace

// dP, dH: device packed (ndim); the remaining arrays are host arrays, copied in.
// Returns the device time of the AO-pair update kernel in milliseconds.
float xc_damping_device(ptbgpu_ctx* c, int64_t nat, int64_t ndim, const int64_t* aoat, const double* rab,
                        const double* rad, const double* hao, const double* xdiag, const double* dP, double* dH) {
    PTB_CHECK(nat > 0 && ndim > 0 && aoat && rab && rad && hao && xdiag && dP && dH, PTBGPU_EINVAL,
              "bad arguments");
    for (int64_t i = 0; i < ndim; ++i)
        PTB_CHECK(aoat[i] >= 1 && aoat[i] <= nat, PTBGPU_EINVAL, "aoat(%lld) = %lld outside 1..%lld",
                  (long long)(i + 1), (long long)aoat[i], (long long)nat);
    const int64_t npat = nat * (nat + 1) / 2;
    DevBuf& bsmall = c->buf(B_MISC0);
    DevBuf& brab = c->buf(B_MISC1);
    DevBuf& bxab = c->buf(B_MISC2);
    bsmall.reserve(sizeof(double) * (size_t)(3 * ndim + nat));
    brab.reserve(sizeof(double) * (size_t)npat);
    bxab.reserve(sizeof(double) * (size_t)npat);
    int64_t* d_aoat = bsmall.as<int64_t>();
    double* d_hao = reinterpret_cast<double*>(d_aoat + ndim);
    double* d_xdiag = d_hao + ndim;
    double* d_rad = d_xdiag + ndim;
    cudaStream_t s = c->stream;
    PTB_CUDA(cudaMemcpyAsync(d_aoat, aoat, sizeof(int64_t) * ndim, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(d_hao, hao, sizeof(double) * ndim, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(d_xdiag, xdiag, sizeof(double) * ndim, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(d_rad, rad, sizeof(double) * nat, cudaMemcpyHostToDevice, s));
    PTB_CUDA(cudaMemcpyAsync(brab.ptr, rab, sizeof(double) * npat, cudaMemcpyHostToDevice, s));
    k_xab<<<(unsigned)std::min<int64_t>(nat, 148 * 8), 256, 0, s>>>(nat, brab.as<double>(), d_rad,
                                                                   bxab.as<double>());
    count_launch();
    PTB_CUDA(cudaGetLastError());
    const int64_t np = ndim * (ndim + 1) / 2;
    PTB_CHECK(((uintptr_t)dP & 15) == 0 && ((uintptr_t)dH & 15) == 0, PTBGPU_EINVAL,
              "P and H must start on a 16-byte boundary");
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((np / 2 + 255) / 256, 148 * 16));
    cudaEvent_t e0 = c->take_event(), e1 = c->take_event();
    PTB_CUDA(cudaEventRecord(e0, s));
    k_xc_update<<<grid, 256, 0, s>>>(ndim, d_aoat, d_hao, d_xdiag, bxab.as<double>(), dP, dH);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    PTB_CUDA(cudaEventRecord(e1, s));
    PTB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PTB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    return ms;
}

}  // namespace ptb
