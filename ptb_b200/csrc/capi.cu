// extern "C" entry points: argument checks, host <-> device copies of the
// packed arrays, CUDA-event timing, and translation of internal errors into
// status codes plus a message readable through ptbgpu_last_error().
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "common.cuh"
#include "sm_eig.cuh"
#include "oz_gemm.cuh"
#include "tc_gemm.cuh"

namespace ptb {
void tc_purify_entry(ptbgpu_ctx* c, int64_t n, int64_t nel, const double* dH, const double* dS, double* dP,
                     const ptbgpu_opts* o, ptbgpu_stats* st);
void symsq_entry(ptbgpu_ctx* c, int64_t n, int np, int kblock, const double* hX, float* hC);
std::vector<int64_t> kmeans_partition(ptbgpu_ctx* c, int64_t n, const double* dH, const double* dS, int64_t nat,
                                      const double* xyz, const int64_t* aoat, uint64_t seed, int* nsm_out,
                                      double* effort_out);
void sm_plan_entry(ptbgpu_ctx* c, int64_t n, const double* dH, const double* dS, int64_t nat, const double* xyz,
                   const int64_t* aoat, int64_t columns, int64_t mode, const int64_t* partition, const ptbgpu_opts* o,
                   int64_t* nsm, int64_t* dims);
void sm_prepare_entry(ptbgpu_ctx* c, int64_t nlocal, const int64_t* ids, ptbgpu_stats* st);
double sm_nel_entry(ptbgpu_ctx* c, double mu);
void sm_finish_entry(ptbgpu_ctx* c, double mu, double* dP);
void mlpop14_device(ptbgpu_ctx* c, int64_t n, const double* dSpk, double x, float* s34, float* s14);
void mlpop2_diag_device(ptbgpu_ctx* c, int64_t n, const double* dPpk, const float* s1, const float* s2, double* xd);
float xc_damping_device(ptbgpu_ctx* c, int64_t nat, int64_t ndim, const int64_t* aoat, const double* rab,
                        const double* rad, const double* hao, const double* xdiag, const double* dP, double* dH);
void tc_purify_grouped(ptbgpu_ctx* c, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                       const double* const* Hpk, const double* const* Spk, double* const* Ppk, const ptbgpu_opts* o,
                       ptbgpu_stats* st, std::vector<int>& redo);
void oz_gemm_entry(ptbgpu_ctx* c, int64_t n, int S, int kblock, int variant, int tri_a, int tri_b, bool sym,
                   const double* hA,
                   const double* hB, double* hC);
void purify_ref_device(ptbgpu_ctx* c, const ptbgpu_pur_settings& pur, int64_t n, const double* dH,
                       const double* dS, double* dP, const ptbgpu_opts* o, ptbgpu_stats* st);
void solve2_device(ptbgpu_ctx* c, int64_t mode, int64_t n, int64_t nel, int64_t nopen, const double* dH,
                   const double* dS, double* dP, double* he, double* hfocc, const ptbgpu_opts* o, ptbgpu_stats* st);
void check_density_device(ptbgpu_ctx* c, int64_t n, const double* dP, const double* dS, const double* dH,
                          ptbgpu_stats* st);
void sm_density_device(ptbgpu_ctx* c, int64_t ndim, int64_t nelref, const double* dH, const double* dS, double* dP,
                       int64_t nat, const double* xyz, const int64_t* aoat, int64_t columns, int64_t mode,
                       const int64_t* partition, const ptbgpu_opts* o, ptbgpu_stats* st);
}  // namespace ptb

namespace {

using namespace ptb;

template <class F>
int guarded(ptbgpu_ctx* c, F&& f) {
    if (!c) return PTBGPU_EINVAL;
    try {
        PTB_CUDA(cudaSetDevice(c->device));
        launch_counter() = 0;
        c->evused = 0;
        c->timed.clear();
        c->oz_ops = 0.0;
        f();
        c->last_error.clear();
        return PTBGPU_OK;
    } catch (const Error& e) {
        c->last_error = e.msg;
        // report a pending or sticky device error too: library status codes such
        // as cuSOLVER's internal error can be the echo of an earlier kernel fault
        cudaError_t pend = c->stream ? cudaStreamSynchronize(c->stream) : cudaSuccess;
        cudaError_t last = cudaGetLastError();
        if (pend != cudaSuccess || last != cudaSuccess)
            c->last_error += std::string(" [device: ") + cudaGetErrorString(pend != cudaSuccess ? pend : last) + "]";
        return e.code;
    } catch (const std::exception& e) {
        c->last_error = e.what();
        return PTBGPU_ECUDA;
    }
}

// Device copies of up to three packed inputs and one packed output.
struct PackedIO {
    ptbgpu_ctx* c;
    int64_t n;
    double* d[3] = {nullptr, nullptr, nullptr};
    PackedIO(ptbgpu_ctx* cc, int64_t nn) : c(cc), n(nn) {
        for (int k = 0; k < 3; ++k) {
            DevBuf& b = c->buf(B_PK0 + k);
            b.reserve(sizeof(double) * (size_t)npacked(n));
            d[k] = b.as<double>();
        }
    }
    void in(int k, const double* h) {
        PTB_CUDA(cudaMemcpyAsync(d[k], h, sizeof(double) * (size_t)npacked(n), cudaMemcpyHostToDevice, c->stream));
    }
    void out(int k, double* h) {
        PTB_CUDA(cudaMemcpyAsync(h, d[k], sizeof(double) * (size_t)npacked(n), cudaMemcpyDeviceToHost, c->stream));
    }
};

// Records ms_h2d / ms_solve / ms_d2h / ms_total with CUDA events on the context stream.
struct PhaseTimer {
    ptbgpu_ctx* c;
    explicit PhaseTimer(ptbgpu_ctx* cc) : c(cc) { PTB_CUDA(cudaEventRecord(c->ev[0], c->stream)); }
    void mark(int k) { PTB_CUDA(cudaEventRecord(c->ev[k], c->stream)); }
    void finish(ptbgpu_stats* st) {
        PTB_CUDA(cudaEventRecord(c->ev[3], c->stream));
        PTB_CUDA(cudaEventSynchronize(c->ev[3]));
        if (!st) return;
        float a = 0, b = 0, d = 0;
        PTB_CUDA(cudaEventElapsedTime(&a, c->ev[0], c->ev[1]));
        PTB_CUDA(cudaEventElapsedTime(&b, c->ev[1], c->ev[2]));
        PTB_CUDA(cudaEventElapsedTime(&d, c->ev[2], c->ev[3]));
        st->ms_h2d = a;
        st->ms_solve = b;
        st->ms_d2h = d;
        st->ms_total = a + b + d;
        for (const auto& t : c->timed) {
            float ms = 0.f;
            PTB_CUDA(cudaEventElapsedTime(&ms, t.a, t.b));
            if (t.kind == 0) {
                st->ms_tc_sp2 += ms;
                st->n_tc_sp2 += 1;
            } else if (t.kind == 2) {
                st->ms_oz += ms;
                st->n_oz += 1;
            } else {
                st->ms_tc_full += ms;
                st->n_tc_full += 1;
            }
        }
        st->kernel_launches = launch_counter();
        st->oz_ops = c->oz_ops;
    }
};

void clear_stats(ptbgpu_stats* st) {
    if (st) memset(st, 0, sizeof(*st));
}

// q(aoat(i)) += xd(i), qsh(shell2ao(i), aoat(i)) += xd(i) in AO order, as
// source/mlpop.f:225-233 (1-based maps; qsh is Fortran qsh(10, n)).
void accumulate_pops(int64_t nat, int64_t nao, const double* xd, const int64_t* aoat, const int64_t* shell2ao,
                     double* q, double* qsh) {
    for (int64_t a = 0; a < nat; ++a) q[a] = 0.0;
    for (int64_t k = 0; k < 10 * nat; ++k) qsh[k] = 0.0;
    for (int64_t i = 0; i < nao; ++i) {
        const int64_t ia = aoat[i] - 1, ish = shell2ao[i] - 1;
        PTB_CHECK(ia >= 0 && ia < nat && ish >= 0 && ish < 10, PTBGPU_EINVAL,
                  "aoat(%lld) = %lld or shell2ao = %lld out of range", (long long)(i + 1), (long long)aoat[i],
                  (long long)shell2ao[i]);
        q[ia] += xd[i];
        qsh[ia * 10 + ish] += xd[i];
    }
}

}  // namespace

extern "C" {

int ptbgpu_filter_packed(ptbgpu_ctx* c, int64_t n, double* Apk, double filter) {
    return guarded(c, [&] {
        PTB_CHECK(n > 0 && Apk, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, n);
        io.in(0, Apk);
        filter_packed(c->stream, n, io.d[0], filter);
        io.out(0, Apk);
        PTB_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int ptbgpu_check_density(ptbgpu_ctx* c, int64_t ndim, const double* Ppk, const double* Spk, const double* Hpk,
                         ptbgpu_stats* st) {
    return guarded(c, [&] {
        PTB_CHECK(ndim > 0 && Ppk && Spk && st, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        io.in(0, Ppk);
        io.in(1, Spk);
        if (Hpk) io.in(2, Hpk);
        check_density_device(c, ndim, io.d[0], io.d[1], Hpk ? io.d[2] : nullptr, st);
        PTB_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int ptbgpu_sm_density(ptbgpu_ctx* c, int64_t ndim, int64_t nelref, const double* Hpk, const double* Spk,
                      double* Ppk, int64_t nat, const double* xyz, const int64_t* aoat, int64_t columns,
                      int64_t mode, const int64_t* partition, const ptbgpu_opts* opts, ptbgpu_stats* st) {
    clear_stats(st);
    return guarded(c, [&] {
        PTB_CHECK(ndim > 0 && Hpk && Spk && Ppk && aoat, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        PhaseTimer t(c);
        io.in(0, Hpk);
        io.in(1, Spk);
        t.mark(1);
        sm_density_device(c, ndim, nelref, io.d[0], io.d[1], io.d[2], nat, xyz, aoat, columns, mode, partition,
                          opts, st);
        t.mark(2);
        io.out(2, Ppk);
        t.finish(st);
    });
}

int ptbgpu_purify(ptbgpu_ctx* c, const ptbgpu_pur_settings* pur, int64_t ndim, const double* Hpk,
                  const double* Spk, double* Ppk, const ptbgpu_opts* opts, ptbgpu_stats* st) {
    clear_stats(st);
    return guarded(c, [&] {
        PTB_CHECK(pur && ndim > 0 && Hpk && Spk && Ppk, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        PhaseTimer t(c);
        io.in(0, Hpk);
        io.in(1, Spk);
        t.mark(1);
        purify_ref_device(c, *pur, ndim, io.d[0], io.d[1], io.d[2], opts, st);
        t.mark(2);
        io.out(2, Ppk);
        t.finish(st);
    });
}

int ptbgpu_tc_purify(ptbgpu_ctx* c, int64_t ndim, int64_t nel, const double* Hpk, const double* Spk, double* Ppk,
                     const ptbgpu_opts* opts, ptbgpu_stats* st) {
    clear_stats(st);
    return guarded(c, [&] {
        PTB_CHECK(ndim > 0 && Hpk && Spk && Ppk, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        PhaseTimer t(c);
        io.in(0, Hpk);
        io.in(1, Spk);
        t.mark(1);
        tc_purify_entry(c, ndim, nel, io.d[0], io.d[1], io.d[2], opts, st);
        t.mark(2);
        io.out(2, Ppk);
        t.finish(st);
    });
}

int ptbgpu_tc_purify_device(ptbgpu_ctx* c, int64_t ndim, int64_t nel, const double* dH, const double* dS,
                            double* dP, const ptbgpu_opts* opts, ptbgpu_stats* st) {
    clear_stats(st);
    return guarded(c, [&] {
        PTB_CHECK(ndim > 0 && dH && dS && dP, PTBGPU_EINVAL, "bad arguments");
        PhaseTimer t(c);
        t.mark(1);
        tc_purify_entry(c, ndim, nel, dH, dS, dP, opts, st);
        t.mark(2);
        t.finish(st);
    });
}

int ptbgpu_eig_density_batch(ptbgpu_ctx* c, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                             const double* const* Hpk, const double* const* Spk, double* const* Ppk,
                             const ptbgpu_opts* opts, ptbgpu_stats* st, double* wall_ms) {
    if (st)
        for (int64_t i = 0; i < ninst; ++i) clear_stats(&st[i]);
    return guarded(c, [&] {
        PTB_CHECK(ninst >= 0 && (ninst == 0 || (ndim && nel && Hpk && Spk && Ppk)), PTBGPU_EINVAL, "bad arguments");
        const auto t0 = std::chrono::steady_clock::now();
        eig_density_batch(c, ninst, ndim, nel, Hpk, Spk, Ppk, opts ? opts->filter : 0.0,
                          opts ? (int)opts->print_level : 0, st);
        if (st && ninst > 0) st[0].kernel_launches = launch_counter();   // the whole call's launches
        if (wall_ms)
            *wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
}

int ptbgpu_tc_purify_batch(ptbgpu_ctx* c, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                           const double* const* Hpk, const double* const* Spk, double* const* Ppk, int64_t workers,
                           const ptbgpu_opts* opts, ptbgpu_stats* st, double* wall_ms) {
    if (!c) return PTBGPU_EINVAL;
    if (ninst < 0 || (ninst > 0 && (!ndim || !nel || !Hpk || !Spk || !Ppk)) || workers < 0) {
        c->last_error = "bad arguments";
        return PTBGPU_EINVAL;
    }
    const int64_t want = workers == 0 ? 4 : workers;
    const int nw = (int)std::max<int64_t>(1, std::min<int64_t>(want, std::max<int64_t>(ninst, 1)));
    // worker contexts: created once per main context, reused by later batches
    while ((int)c->workers.size() < nw) {
        ptbgpu_ctx* w = nullptr;
        const int rc = ptbgpu_init(c->device, &w);
        if (rc != PTBGPU_OK) {
            c->last_error = "could not create a worker context";
            return rc;
        }
        c->workers.push_back(w);
    }
    // largest systems first, so that the small ones fill in around them
    std::vector<int64_t> order((size_t)ninst);
    for (int64_t i = 0; i < ninst; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return ndim[a] > ndim[b]; });
    std::atomic<int64_t> next{0};
    std::atomic<int> first_rc{PTBGPU_OK};
    std::mutex err_mu;
    std::string err_msg;
    auto run = [&](ptbgpu_ctx* w) {
        for (int64_t q = next++; q < ninst && first_rc.load() == PTBGPU_OK; q = next++) {
            const int64_t i = order[q];
            const int rc = ptbgpu_tc_purify(w, ndim[i], nel[i], Hpk[i], Spk[i], Ppk[i], opts, st ? &st[i] : nullptr);
            if (rc != PTBGPU_OK) {
                int expect = PTBGPU_OK;
                if (first_rc.compare_exchange_strong(expect, rc)) {
                    std::lock_guard<std::mutex> lock(err_mu);
                    err_msg = "system " + std::to_string(i) + ": " + w->last_error;
                }
            }
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < nw; ++t) pool.emplace_back(run, c->workers[t]);
    for (auto& t : pool) t.join();
    if (wall_ms) *wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const int rc = first_rc.load();
    c->last_error = rc == PTBGPU_OK ? std::string() : err_msg;
    return rc;
}

int ptbgpu_tc_purify_grouped(ptbgpu_ctx* c, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                             const double* const* Hpk, const double* const* Spk, double* const* Ppk,
                             const ptbgpu_opts* opts, ptbgpu_stats* st, double* wall_ms) {
    if (!c) return PTBGPU_EINVAL;
    if (ninst < 0 || (ninst > 0 && (!ndim || !nel || !Hpk || !Spk || !Ppk))) {
        c->last_error = "bad arguments";
        return PTBGPU_EINVAL;
    }
    ptbgpu_opts def;
    ptbgpu_default_opts(&def);
    const ptbgpu_opts* o = opts ? opts : &def;
    if (st)
        for (int64_t i = 0; i < ninst; ++i) clear_stats(&st[i]);
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<int> redo;
    int rc = guarded(c, [&] { tc_purify_grouped(c, ninst, ndim, nel, Hpk, Spk, Ppk, o, st, redo); });
    // systems the grouped path left (pass 1 not converged, refinement short of its
    // tolerance, NaN): the single-system path in FP64, the same as its own fallback
    for (int64_t i = 0; rc == PTBGPU_OK && i < ninst; ++i) {
        if (!redo[i]) continue;
        ptbgpu_opts o64 = *o;
        o64.precision = PTBGPU_PREC_FP64;
        rc = ptbgpu_tc_purify(c, ndim[i], nel[i], Hpk[i], Spk[i], Ppk[i], &o64, st ? &st[i] : nullptr);
        if (rc != PTBGPU_OK) c->last_error = "system " + std::to_string(i) + ": " + c->last_error;
        else if (st && o->precision != PTBGPU_PREC_FP64) st[i].fp64_fallback = 1;
    }
    if (wall_ms) *wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int ptbgpu_solve2(ptbgpu_ctx* c, int64_t mode, int64_t ndim, int64_t nel, int64_t nopen, const double* Hpk,
                  const double* Spk, double* Ppk, double* e, double* focc, const ptbgpu_opts* opts,
                  ptbgpu_stats* st) {
    clear_stats(st);
    return guarded(c, [&] {
        PTB_CHECK(ndim > 0 && Hpk && Spk && Ppk, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        PhaseTimer t(c);
        io.in(0, Hpk);
        io.in(1, Spk);
        t.mark(1);
        solve2_device(c, mode, ndim, nel, nopen, io.d[0], io.d[1], io.d[2], e, focc, opts, st);
        t.mark(2);
        io.out(2, Ppk);
        t.finish(st);
    });
}

int ptbgpu_symsq_bf16x3(ptbgpu_ctx* c, int64_t n, const double* X, float* C) {
    return guarded(c, [&] {
        PTB_CHECK(n > 0 && X && C, PTBGPU_EINVAL, "bad arguments");
        symsq_entry(c, n, 2, 0, X, C);
    });
}

int ptbgpu_symsq_bf16x6(ptbgpu_ctx* c, int64_t n, const double* X, float* C) {
    return guarded(c, [&] {
        PTB_CHECK(n > 0 && X && C, PTBGPU_EINVAL, "bad arguments");
        symsq_entry(c, n, 3, 0, X, C);
    });
}

int ptbgpu_symsq_split(ptbgpu_ctx* c, int64_t n, int64_t planes, int64_t kblock, const double* X, float* C,
                       double* ms) {
    return guarded(c, [&] {
        // kblock: 0 tuned, 32 / 64 one CTA, 1032 / 1064 CTA pair (two planes only)
        const bool pair = kblock == tc::kPairKernel + 32 || kblock == tc::kPairKernel + 64;
        PTB_CHECK(n > 0 && X && C && (planes == 2 || planes == 3) &&
                      (kblock == 0 || kblock == 32 || kblock == 64 || (pair && planes == 2)),
                  PTBGPU_EINVAL, "bad arguments");
        symsq_entry(c, n, (int)planes, (int)kblock, X, C);
        if (ms) {
            *ms = 0.0;
            for (const auto& t : c->timed) {
                float x = 0.f;
                PTB_CUDA(cudaEventElapsedTime(&x, t.a, t.b));
                *ms += x;
            }
        }
    });
}

int ptbgpu_sm_plan(ptbgpu_ctx* c, int64_t ndim, const double* Hpk, const double* Spk, int64_t nat,
                   const double* xyz, const int64_t* aoat, int64_t columns, int64_t mode, const int64_t* partition,
                   const ptbgpu_opts* opts, int64_t* nsm, int64_t* dims) {
    return guarded(c, [&] {
        PTB_CHECK(ndim > 0 && Hpk && Spk && aoat && nsm && dims, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        io.in(0, Hpk);
        io.in(1, Spk);
        sm_plan_entry(c, ndim, io.d[0], io.d[1], nat, xyz, aoat, columns, mode, partition, opts, nsm, dims);
    });
}

int ptbgpu_sm_prepare(ptbgpu_ctx* c, int64_t nlocal, const int64_t* ids, ptbgpu_stats* st) {
    clear_stats(st);
    return guarded(c, [&] {
        PTB_CHECK(nlocal >= 0 && (ids || nlocal == 0), PTBGPU_EINVAL, "bad arguments");
        sm_prepare_entry(c, nlocal, ids, st);
    });
}

int ptbgpu_sm_nel(ptbgpu_ctx* c, double mu, double* nel) {
    return guarded(c, [&] {
        PTB_CHECK(nel != nullptr, PTBGPU_EINVAL, "bad arguments");
        *nel = sm_nel_entry(c, mu);
    });
}

int ptbgpu_sm_finish(ptbgpu_ctx* c, int64_t ndim, double mu, double* Ppk) {
    return guarded(c, [&] {
        PTB_CHECK(ndim > 0 && Ppk, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        sm_finish_entry(c, mu, io.d[2]);
        io.out(2, Ppk);
        PTB_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int ptbgpu_kmeans_partition(ptbgpu_ctx* c, int64_t ndim, const double* Hpk, const double* Spk, int64_t nat,
                            const double* xyz, const int64_t* aoat, uint64_t seed, const ptbgpu_opts* opts,
                            int64_t* partition, int64_t* nsm, double* effort) {
    return guarded(c, [&] {
        PTB_CHECK(ndim > 0 && Hpk && Spk && nat > 0 && xyz && aoat && partition, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        io.in(0, Hpk);
        io.in(1, Spk);
        DevBuf& bh = c->buf(B_H);
        DevBuf& bs = c->buf(B_S);
        bh.reserve(sizeof(double) * ndim * ndim);
        bs.reserve(sizeof(double) * ndim * ndim);
        const double filter = opts ? opts->filter : 0.0;
        unpack_sym(c->stream, ndim, ndim, io.d[0], bh.as<double>(), filter);
        unpack_sym(c->stream, ndim, ndim, io.d[1], bs.as<double>(), filter);
        int k = 0;
        double e = 0.0;
        const std::vector<int64_t> p =
            kmeans_partition(c, ndim, bh.as<double>(), bs.as<double>(), nat, xyz, aoat, seed, &k, &e);
        std::copy(p.begin(), p.end(), partition);
        if (nsm) *nsm = k;
        if (effort) *effort = e;
    });
}

int ptbgpu_mlpop14(ptbgpu_ctx* c, int64_t nao, const double* Spk, double x, float* s34, float* s14) {
    return guarded(c, [&] {
        PTB_CHECK(nao > 0 && Spk && s34 && s14, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, nao);
        io.in(0, Spk);
        DevBuf& b3 = c->buf(B_X1F0);
        DevBuf& b1 = c->buf(B_X1F1);
        b3.reserve(sizeof(float) * nao * nao);
        b1.reserve(sizeof(float) * nao * nao);
        mlpop14_device(c, nao, io.d[0], x, b3.as<float>(), b1.as<float>());
        PTB_CUDA(cudaMemcpyAsync(s34, b3.ptr, sizeof(float) * nao * nao, cudaMemcpyDeviceToHost, c->stream));
        PTB_CUDA(cudaMemcpyAsync(s14, b1.ptr, sizeof(float) * nao * nao, cudaMemcpyDeviceToHost, c->stream));
        PTB_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int ptbgpu_mlpop14_device(ptbgpu_ctx* c, int64_t nao, const double* dSpk, double x, float* d_s34, float* d_s14) {
    return guarded(c, [&] {
        PTB_CHECK(nao > 0 && dSpk && d_s34 && d_s14, PTBGPU_EINVAL, "bad arguments");
        mlpop14_device(c, nao, dSpk, x, d_s34, d_s14);
        PTB_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int ptbgpu_mlpop2(ptbgpu_ctx* c, int64_t n, int64_t nao, const double* Ppk, const float* s1, const float* s2,
                  const int64_t* aoat, const int64_t* shell2ao, double* q, double* qsh, ptbgpu_stats* st) {
    clear_stats(st);
    return guarded(c, [&] {
        PTB_CHECK(n > 0 && nao > 0 && Ppk && s1 && s2 && aoat && shell2ao && q && qsh, PTBGPU_EINVAL,
                  "bad arguments");
        PackedIO io(c, nao);
        DevBuf& b1 = c->buf(B_MISC0);
        DevBuf& b2 = c->buf(B_MISC1);
        b1.reserve(sizeof(float) * nao * nao);
        b2.reserve(sizeof(float) * nao * nao);
        PhaseTimer t(c);
        io.in(0, Ppk);
        PTB_CUDA(cudaMemcpyAsync(b1.ptr, s1, sizeof(float) * nao * nao, cudaMemcpyHostToDevice, c->stream));
        PTB_CUDA(cudaMemcpyAsync(b2.ptr, s2, sizeof(float) * nao * nao, cudaMemcpyHostToDevice, c->stream));
        t.mark(1);
        std::vector<double> xd((size_t)nao);
        mlpop2_diag_device(c, nao, io.d[0], b1.as<float>(), b2.as<float>(), xd.data());
        t.mark(2);
        t.finish(st);
        accumulate_pops(n, nao, xd.data(), aoat, shell2ao, q, qsh);
    });
}

int ptbgpu_mlpop2_device(ptbgpu_ctx* c, int64_t n, int64_t nao, const double* dPpk, const float* d_s1,
                         const float* d_s2, const int64_t* aoat, const int64_t* shell2ao, double* q, double* qsh,
                         ptbgpu_stats* st) {
    clear_stats(st);
    return guarded(c, [&] {
        PTB_CHECK(n > 0 && nao > 0 && dPpk && d_s1 && d_s2 && aoat && shell2ao && q && qsh, PTBGPU_EINVAL,
                  "bad arguments");
        PhaseTimer t(c);
        t.mark(1);
        std::vector<double> xd((size_t)nao);
        mlpop2_diag_device(c, nao, dPpk, d_s1, d_s2, xd.data());
        t.mark(2);
        t.finish(st);
        accumulate_pops(n, nao, xd.data(), aoat, shell2ao, q, qsh);
    });
}

int ptbgpu_xc_damping(ptbgpu_ctx* c, int64_t nat, int64_t ndim, const int64_t* aoat, const double* rab,
                      const double* rad, const double* hao, const double* xdiag, const double* Ppk, double* Hpk,
                      double* ms_update) {
    return guarded(c, [&] {
        PTB_CHECK(nat > 0 && ndim > 0 && Ppk && Hpk, PTBGPU_EINVAL, "bad arguments");
        PackedIO io(c, ndim);
        io.in(0, Ppk);
        io.in(1, Hpk);
        const float ms = xc_damping_device(c, nat, ndim, aoat, rab, rad, hao, xdiag, io.d[0], io.d[1]);
        io.out(1, Hpk);
        PTB_CUDA(cudaStreamSynchronize(c->stream));
        if (ms_update) *ms_update = ms;
    });
}

int ptbgpu_xc_damping_device(ptbgpu_ctx* c, int64_t nat, int64_t ndim, const int64_t* aoat, const double* rab,
                             const double* rad, const double* hao, const double* xdiag, const double* dPpk,
                             double* dHpk, double* ms_update) {
    return guarded(c, [&] {
        const float ms = xc_damping_device(c, nat, ndim, aoat, rab, rad, hao, xdiag, dPpk, dHpk);
        if (ms_update) *ms_update = ms;
    });
}

int ptbgpu_oz_tiles(int64_t n, int64_t slices, int64_t kblock, int64_t variant, int64_t a_tri, int64_t b_tri,
                    int64_t symmetric, int32_t* tiles, int64_t cap, int64_t* ntiles, int64_t* info) {
    if (n <= 0 || !(slices == 4 || (slices >= 6 && slices <= 8)) || !(kblock == 0 || kblock == 32 || kblock == 64) ||
        variant < 0 || variant > 5 || a_tri < 0 || a_tri > 2 || b_tri < 0 || b_tri > 2 || cap < 0 ||
        (cap > 0 && !tiles) || !ntiles || !info)
        return PTBGPU_EINVAL;
    try {
        const int S = (int)slices;
        const int v = oz::resolve_variant((int)variant, S, (int)kblock);
        PTB_CHECK(!((v == oz::V_WIDE || v == oz::V_WPAIR) && kblock == 64), PTBGPU_EINVAL,
                  "the 128-column kernels take 32-byte K blocks");
        const std::vector<int4> t =
            oz::build_tiles(oz::padded(n), symmetric != 0, (int)a_tri, (int)b_tri, S, v);
        *ntiles = (int64_t)t.size();
        for (int64_t i = 0; i < std::min<int64_t>(cap, (int64_t)t.size()); ++i) {
            tiles[4 * i] = t[i].x;
            tiles[4 * i + 1] = t[i].y;
            tiles[4 * i + 2] = t[i].z;
            tiles[4 * i + 3] = t[i].w;
        }
        info[0] = v;
        info[1] = oz::tile_n(S, v);
        info[2] = oz::grid_ctas((int)t.size(), v);
        info[3] = (v == oz::V_PAIR || v == oz::V_WPAIR) ? 2 * oz::BM : oz::BM;
        return PTBGPU_OK;
    } catch (const Error& e) {
        return e.code;
    } catch (const std::exception&) {
        return PTBGPU_EINVAL;
    }
}

int ptbgpu_oz_gemm(ptbgpu_ctx* c, int64_t n, int64_t slices, int64_t kblock, int64_t variant, int64_t tri_a,
                   int64_t tri_b, int64_t symmetric, const double* A, const double* B, double* Cout, double* ms) {
    return guarded(c, [&] {
        PTB_CHECK(n > 0 && A && B && Cout && (slices == 4 || (slices >= 6 && slices <= 8)) &&
                      (kblock == 0 || kblock == 32 || kblock == 64) && variant >= 0 && variant <= 5 &&
                      tri_a >= 0 && tri_a <= 2 && tri_b >= 0 && tri_b <= 2,
                  PTBGPU_EINVAL, "bad arguments");
        oz_gemm_entry(c, n, (int)slices, (int)kblock, (int)variant, (int)tri_a, (int)tri_b, symmetric != 0, A, B,
                      Cout);
        if (ms) {
            *ms = 0.0;
            for (const auto& t : c->timed) {
                float x = 0.f;
                PTB_CUDA(cudaEventElapsedTime(&x, t.a, t.b));
                *ms += x;
            }
        }
    });
}

int ptbgpu_sygv_batched(ptbgpu_ctx* c, int64_t nprob, const int64_t* dims, const double* H, const double* S,
                        const int64_t* nown, const int64_t* owned, double mu, double* e, double* fe,
                        double* Pcols) {
    return guarded(c, [&] {
        PTB_CHECK(nprob > 0 && dims && H && S && nown && owned && e && fe, PTBGPU_EINVAL, "bad arguments");
        sygv_batched_entry(c, nprob, dims, H, S, nown, owned, mu, e, fe, Pcols);
    });
}

}  // extern "C"
