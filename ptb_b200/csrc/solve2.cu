// Dense FP64 density step (the reference's check-mode oracle, solve2) and the
// density checks of source/metrics.f90, on the device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "oz_gemm.cuh"

namespace ptb {

namespace {

__global__ void k_scale_cols2(int64_t n, const double* __restrict__ V, const double* __restrict__ d,
                              double* __restrict__ out) {
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        const double s = d[j];
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) out[i + j * n] = V[i + j * n] * s;
    }
}

// occu, source/fermi.f:71-124: restricted occupations -> alpha / beta.
void occu(int64_t ndim, int64_t nel, int64_t nopen, int64_t& ihomoa, int64_t& ihomob, std::vector<double>& fa,
          std::vector<double>& fb) {
    std::vector<int64_t> focc(ndim, 0);
    if (nel % 2 == 0) {
        int64_t ihomo = nel / 2;
        for (int64_t i = 0; i < ihomo && i < ndim; ++i) focc[i] = 2;
        if (nopen > 1) {
            for (int64_t i = 1; i <= nopen / 2; ++i) {
                focc[ihomo - i] -= 1;
                focc[ihomo + i - 1] += 1;
            }
        }
    } else {
        const int64_t na = nel / 2 + (nopen - 1) / 2 + 1, nb = nel / 2 - (nopen - 1) / 2;
        for (int64_t i = 0; i < na && i < ndim; ++i) focc[i] += 1;
        for (int64_t i = 0; i < nb && i < ndim; ++i) focc[i] += 1;
    }
    fa.assign(ndim, 0.0);
    fb.assign(ndim, 0.0);
    ihomoa = ihomob = 0;
    for (int64_t i = 0; i < ndim; ++i) {
        if (focc[i] == 2) fa[i] = fb[i] = 1.0;
        if (focc[i] == 1) fa[i] = 1.0;
        if (fa[i] > 0.99) ihomoa = i + 1;
        if (fb[i] > 0.99) ihomob = i + 1;
    }
    PTB_CHECK(ihomoa >= 1, PTBGPU_EINVAL, "internal error in occu");
}

// FERMISMEAR, source/fermi.f:5-67 (BOLTZ is a REAL(4) literal in the reference).
void fermismear(int64_t norbs, int64_t nel, double t, const std::vector<double>& eig, std::vector<double>& occ) {
    const double boltz = (double)3.166808578545117e-06f;
    const double bkt = boltz * t;
    double ef = 0.5 * (eig[nel - 1] + eig[nel]);
    const double occt = (double)nel;
    occ.assign(norbs, 0.0);
    for (int ncycle = 1;; ++ncycle) {
        double tot = 0.0, totd = 0.0;
        for (int64_t i = 0; i < norbs; ++i) {
            const double x = (eig[i] - ef) / bkt;
            double ff = 0.0, df = 0.0;
            if (x < 50) {
                const double ex = std::exp(x);
                ff = 1.0 / (ex + 1.0);
                df = ex / (bkt * (ex + 1.0) * (ex + 1.0));
            }
            occ[i] = ff;
            tot += ff;
            totd += df;
        }
        ef += (occt - tot) / (totd + 1e-14);
        if (!(std::fabs(occt - tot) > 1e-9 && ncycle < 200)) break;
    }
}

int g1(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(n, 148 * 16)); }

}  // namespace

// solve2, source/pgtb.f90:1066-1170.
void solve2_device(ptbgpu_ctx* c, int64_t mode, int64_t n, int64_t nel, int64_t nopen, const double* dH,
                   const double* dS, double* dP, double* he, double* hfocc, const ptbgpu_opts* o, ptbgpu_stats* st) {
    PTB_CHECK(n > 0 && nel >= 0 && nel <= 2 * n, PTBGPU_EINVAL, "bad sizes");
    const double filter = o ? o->filter : 0.0;
    const double et = (o && o->electronic_temp > 0) ? o->electronic_temp : 300.0;
    cudaStream_t s = c->stream;
    DevBuf& bh = c->buf(B_H);
    DevBuf& bs = c->buf(B_S);
    DevBuf& bw = c->buf(B_W0);
    for (DevBuf* b : {&bh, &bs, &bw}) b->reserve(sizeof(double) * n * n);
    DevBuf& bv = c->buf(B_MISC2);
    bv.reserve(sizeof(double) * n);
    double* U = bh.as<double>();
    double* B = bs.as<double>();
    using clk = std::chrono::steady_clock;
    const int prl = o ? (int)o->print_level : 0;
    PTB_CUDA(cudaStreamSynchronize(s));
    const auto t0 = clk::now();
    unpack_sym(s, n, n, dH, U, filter);
    unpack_sym(s, n, n, dS, B, filter);
    PTB_CUDA(cudaStreamSynchronize(s));
    const auto t1 = clk::now();
    const int info = dsygvd(c, n, n, U, B, bv.as<double>());
    const auto t2 = clk::now();
    std::vector<double> e(n);
    PTB_CUDA(cudaMemcpy(e.data(), bv.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (mode >= 2) {
        const double g15 = o ? o->glob_par15 : 0.0, g17 = o ? o->glob_par17 : 0.0;
        for (auto& v : e) v = v + g15 + g17 * v;
    }
    std::vector<double> fa(n, 0.0), fb(n, 0.0);
    int64_t ia = 0, ib = 0;
    if (nel > 0) occu(n, nel, nopen, ia, ib, fa, fb);
    if (ia + 1 <= n) fermismear(n, ia, et, e, fa);
    if (ib + 1 <= n && nel > 1) fermismear(n, ib, et, e, fb);
    std::vector<double> focc(n);
    for (int64_t i = 0; i < n; ++i) focc[i] = fa[i] + fb[i];
    PTB_CUDA(cudaMemcpy(bv.ptr, focc.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    double* Ptmp = bw.as<double>();
    k_scale_cols2<<<g1(n), 256, 0, s>>>(n, U, bv.as<double>(), Ptmp);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    // P = C diag(focc) C^T (dmat, source/solve.f:263-283): FP64-class product on
    // the int8 tensor cores; beyond its exact range (n > 16643) cuBLAS DGEMM
    if (oz::supported(n, 8)) {
        oz_dgemm(c, n, 1.0, U, false, Ptmp, true, B, 8);
        oz_check(c, "int8 product (density matrix)");
    } else {
        const double one = 1.0, zero = 0.0;
        PTB_CUBLAS(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, (int)n, (int)n, (int)n, &one, U, (int)n, Ptmp,
                               (int)n, &zero, B, (int)n));
    }
    pack_cols(s, n, n, B, dP);
    PTB_CUDA(cudaStreamSynchronize(s));
    // the reference's closing timer block of solve2 (source/pgtb.f90:1108-1168)
    log_timer_block(prl, "Total solve2", std::chrono::duration<double>(clk::now() - t0).count(),
                    {{"sygvd solver", std::chrono::duration<double>(t2 - t1).count()}});
    if (he) std::copy(e.begin(), e.end(), he);
    if (hfocc) std::copy(focc.begin(), focc.end(), hfocc);
    if (st) {
        st->info = info;
        st->flops += 9.0 * (double)n * n * n;
    }
    PTB_CHECK(info == 0, PTBGPU_ENOTSPD, "dsygvd failed (info=%d)", info);
}

// check_density (source/metrics.f90:144-179) with get_nel (:202-230),
// band_structure (:253-277) and idempotent_packed (:316-360) on packed input.
void check_density_device(ptbgpu_ctx* c, int64_t n, const double* dP, const double* dS, const double* dH,
                          ptbgpu_stats* st) {
    cudaStream_t s = c->stream;
    DevBuf& bp = c->buf(B_W0);
    DevBuf& bs = c->buf(B_W1);
    DevBuf& bm = c->buf(B_W2);
    DevBuf& bq = c->buf(B_W3);
    for (DevBuf* b : {&bp, &bs, &bm, &bq}) b->reserve(sizeof(double) * n * n);
    double* P = bp.as<double>();
    double* S = bs.as<double>();
    double* M = bm.as<double>();
    double* Q = bq.as<double>();
    unpack_sym(s, n, n, dP, P, 0.0);
    unpack_sym(s, n, n, dS, S, 0.0);
    st->nel = trace_prod_dev(c, n, n, P, S);
    if (dH) {
        unpack_sym(s, n, n, dH, M, 0.0);
        st->band_energy = trace_prod_dev(c, n, n, P, M);
    }
    // 1/2 P S P: FP64-class products on the int8 tensor cores (beyond their
    // exact range, n > 16643, cuBLAS)
    if (oz::supported(n, 8)) {
        oz_dgemm(c, n, 1.0, P, false, S, false, M, 8);                 // P S
        oz_dgemm(c, n, 0.5, M, false, P, false, Q, 8);                 // 1/2 P S P
        oz_check(c, "int8 product (idempotency)");
    } else {
        const double one = 1.0, half = 0.5, zero = 0.0;
        PTB_CUBLAS(cublasDsymm(c->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, (int)n, (int)n, &one, P, (int)n,
                               S, (int)n, &zero, M, (int)n));
        PTB_CUBLAS(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)n, (int)n, &half, M, (int)n, P,
                               (int)n, &zero, Q, (int)n));
    }
    axpby_diag(s, n, n, -1.0, P, 1.0, Q, 0.0);                         // mm2 - P
    st->idempotency_ref = std::fabs(sum_dev(c, n * n, Q));
    st->idempotency_frob = frob_dev(c, n, n, Q);
}

}  // namespace ptb
