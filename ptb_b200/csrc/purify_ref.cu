// The reference's purification module in FP64 on the device
// (source/purification.f90, source/purification_settings.f90):
// metric X = S^-1 or S^-1/2 (eigendecomposition or Newton-Schulz), the guess,
// McWeeny / Pade / Newton-Schulz sign / eigen-sign solvers and the outer
// chemical-potential search, with the reference's thresholds, stop rules and
// quirks (documented beside each routine).  Dense column-major matrices; the
// products run on the int8 tensor cores as FP64-class sliced products
// (oz_dgemm), the eigendecompositions of the metric and of the eigen-sign
// solver on the library's FP64 eigensolver (dsyevd: one thread-block cluster
// up to order 4096, a cooperative grid up to 12032, cuSOLVER DSYEVD above).
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "oz_gemm.cuh"

namespace ptb {

namespace {

struct Thr {
    double high, normal, low;
};

// adjust_thresholds_dp, source/metrics.f90:82-113 (REAL(4) literals promoted to REAL(8)).
Thr thresholds(int64_t n) {
    float h, m, l;
    if (n < 300) {
        h = 1e-10f; m = 1e-9f; l = 1e-8f;
    } else if (n < 2000) {
        h = 1e-7f; m = 1e-6f; l = 1e-5f;
    } else if (n < 15000) {
        h = 1e-5f; m = 1e-4f; l = 1e-3f;
    } else {
        h = 1e-3f; m = 1e-2f; l = 1e-1f;
    }
    return Thr{(double)h, (double)m, (double)l};
}

__global__ void k_scale_cols(int64_t n, const double* __restrict__ V, const double* __restrict__ d,
                             double* __restrict__ out) {
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        const double s = d[j];
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) out[i + j * n] = V[i + j * n] * s;
    }
}

__global__ void k_colsq(int64_t n, const double* __restrict__ V, double* __restrict__ out) {
    __shared__ double sh[256];
    for (int64_t j = blockIdx.x; j < n; j += gridDim.x) {
        double s = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += V[i + j * n] * V[i + j * n];
        sh[threadIdx.x] = s;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[j] = sh[0];
        __syncthreads();
    }
}

int g1(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(n, 148 * 16)); }

// ---------------------------------------------------------------------------
// Iteration loops as CUDA graphs: after one eager iteration (which sizes every
// buffer and tile list the body touches and gives the host its first stop
// decision), the body of one iteration is captured into the body graph of a
// conditional WHILE node, and a one-thread kernel at its end applies the
// loop's stop rule on the device (cudaGraphSetConditional), so the remaining
// iterations run as one graph launch without a host round trip each.  The
// norms are summed in the same order as on the host, so the iteration counts
// and results equal those of the eager loop.
struct LoopDev {
    double norm0, norm1;   // the norm the stop rule compares against, the new one
    long long iters;       // iterations done (the eager one included)
    int nan;               // a NaN was met in the body
    int pad;
};

// sign_iterative's rule (source/purification.f90:587): stop when
// | ||X||_F - ||X_prev||_F | < thrs%normal, at the cycle cap, or on a NaN.
// McWeeny's rule (source/purification.f90:496) is the same with the norm
// carried over to the next iteration.
__global__ void k_loop_decide(cudaGraphConditionalHandle h, LoopDev* d, double thr, long long cycles, int carry) {
    d->iters += 1;
    const bool stop = d->nan != 0 || std::fabs(d->norm1 - d->norm0) < thr || d->iters >= cycles;
    if (!stop && carry) d->norm0 = d->norm1;
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

struct LoopGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle handle{};
    int64_t body_launches = 0;
    double body_flops = 0.0;
    bool failed = false;
    ~LoopGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// PTBGPU_GRAPH_LOOPS=0 runs every iteration eagerly instead.
bool graph_loops() {
    static const bool on = [] {
        const char* v = getenv("PTBGPU_GRAPH_LOOPS");
        return !(v && v[0] == '0');
    }();
    return on;
}

struct Ctx {
    ptbgpu_ctx* c;
    int64_t n;
    Thr thr;
    int prl;
    DevBuf scratch[8];
    double* m[8];
    double gemm_flops = 0.0;   // 2n^3 per DGEMM issued (eigensolves not counted)
    Ctx(ptbgpu_ctx* cc, int64_t nn, int p) : c(cc), n(nn), thr(thresholds(nn)), prl(p) {
        for (int k = 0; k < 8; ++k) {
            scratch[k].reserve(sizeof(double) * nn * nn);
            m[k] = scratch[k].as<double>();
        }
    }
    ~Ctx() {
        for (auto& b : scratch) b.release();
    }
    // The module's products on the int8 tensor cores (8 slices, FP64 class);
    // beyond the exact int32 range of the slice sums (n > 16643) cuBLAS DGEMM.
    void gemm(const double* A, const double* B, double* C, double alpha = 1.0, bool transb = false) {
        if (oz::supported(n, kSlices)) {
            oz_dgemm(c, n, alpha, A, false, B, transb, C, kSlices);
        } else {
            const double beta = 0.0;
            PTB_CUBLAS(cublasDgemm(c->blas, CUBLAS_OP_N, transb ? CUBLAS_OP_T : CUBLAS_OP_N, (int)n, (int)n,
                                   (int)n, &alpha, A, (int)n, B, (int)n, &beta, C, (int)n));
        }
        gemm_flops += 2.0 * (double)n * (double)n * (double)n;
    }
    static constexpr int kSlices = 8;
    DevBuf loopdev;
    LoopGraph sign_loop, mcw_loop;
    LoopDev* ld() {
        loopdev.reserve(sizeof(LoopDev));
        return loopdev.as<LoopDev>();
    }
    // Captures body() into a WHILE node's body graph followed by the decision
    // kernel; false if the stream could not be captured (then the loop runs
    // eagerly).
    template <class Body>
    bool build_loop(LoopGraph& lg, Body body, double thr, long long cycles, int carry) {
        if (lg.exec) return true;
        if (lg.failed) return false;
        cudaStream_t s = c->stream;
        LoopDev* d = ld();
        bool ok = cudaGraphCreate(&lg.graph, 0) == cudaSuccess &&
                  cudaGraphConditionalHandleCreate(&lg.handle, lg.graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraphNode_t node;
        cudaGraphNodeParams cp = {};
        cudaGraph_t bodyg = nullptr;
        if (ok) {
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = lg.handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            ok = cudaGraphAddNode(&node, lg.graph, nullptr, 0, &cp) == cudaSuccess;
            if (ok) bodyg = cp.conditional.phGraph_out[0];
        }
        if (ok) ok = cudaStreamBeginCaptureToGraph(s, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
                     cudaSuccess;
        if (ok) {
            const int64_t l0 = launch_counter();
            const double f0 = gemm_flops;
            try {
                body();
                k_loop_decide<<<1, 1, 0, s>>>(lg.handle, d, thr, cycles, carry);
                count_launch();
            } catch (...) {
                ok = false;
            }
            cudaGraph_t out = nullptr;
            const cudaError_t e = cudaStreamEndCapture(s, &out);
            ok = ok && e == cudaSuccess;
            lg.body_launches = launch_counter() - l0;
            lg.body_flops = gemm_flops - f0;
            launch_counter() = l0;   // counted per executed iteration after the launch
            gemm_flops = f0;
        }
        if (ok) ok = cudaGraphInstantiate(&lg.exec, lg.graph, 0) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            if (lg.exec) cudaGraphExecDestroy(lg.exec);
            if (lg.graph) cudaGraphDestroy(lg.graph);
            lg.exec = nullptr;
            lg.graph = nullptr;
            lg.failed = true;
            log_line(prl, 2, " purification loop: CUDA graph capture failed, running eagerly");
        }
        return ok;
    }
    // One launch of a built loop from the state `init` (iterations done so far
    // and the norm to compare against); returns the loop's final device state.
    LoopDev run_loop(LoopGraph& lg, LoopDev init) {
        cudaStream_t s = c->stream;
        LoopDev* d = ld();
        PTB_CUDA(cudaMemcpyAsync(d, &init, sizeof(LoopDev), cudaMemcpyHostToDevice, s));
        PTB_CUDA(cudaGraphLaunch(lg.exec, s));
        LoopDev out;
        PTB_CUDA(cudaMemcpyAsync(&out, d, sizeof(LoopDev), cudaMemcpyDeviceToHost, s));
        PTB_CUDA(cudaStreamSynchronize(s));
        const long long ran = out.iters - init.iters;
        count_launch((int)(ran * lg.body_launches));
        gemm_flops += (double)ran * lg.body_flops;
        return out;
    }
    double frob(const double* a) { return frob_dev(c, n, n, a); }
    void nan_check(const double* a, const char* msg) {
        PTB_CHECK(!has_nan_dev(c, n * n, a), PTBGPU_ENAN, "%s", msg);
    }
};

// get_transformation_matrix, source/purification.f90:83-229.  X into m[0]; S in Sm.
void transformation(Ctx& x, const ptbgpu_pur_settings& pur, const double* S, double* X) {
    const int64_t n = x.n;
    cudaStream_t s = x.c->stream;
    double* atmp = x.m[4];
    double* XsX = x.m[5];
    double* atmp2 = x.m[6];
    if (pur.metric_iterative) {
        if (pur.metric_type == PTBGPU_METRIC_INV) {
            const double inf = rowabs_max_dev(x.c, n, n, S);
            copy_mat(s, n, n, S, n, X);
            axpby_diag(s, n, n, 0.0, nullptr, 1.0 / (inf * inf), X, 0.0);
            for (int64_t i = 0; i < pur.metric_cycles; ++i) {
                x.gemm(S, X, atmp);
                x.gemm(X, atmp, XsX);
                axpby_diag(s, n, n, 2.0, X, 0.0, X, 0.0);           // X = 2X
                axpby_diag(s, n, n, -1.0, XsX, 1.0, X, 0.0);        // X = 2X - XsX
                x.gemm(X, S, atmp2);                                // check = X S
                axpby_diag(s, n, n, 0.0, nullptr, -1.0, atmp2, 1.0);   // I - check
                if (x.frob(atmp2) < x.thr.low) break;
            }
        } else if (pur.metric_type == PTBGPU_METRIC_INV_SQRT) {
            const double fr = x.frob(S);
            copy_mat(s, n, n, S, n, X);
            axpby_diag(s, n, n, 0.0, nullptr, 1.0 / (fr * fr), X, 0.0);
            for (int64_t i = 0; i < pur.metric_cycles; ++i) {
                x.gemm(X, X, atmp);
                x.gemm(atmp, S, XsX);
                x.gemm(X, XsX, atmp2);
                axpby_diag(s, n, n, -0.5, atmp2, 1.5, X, 0.0);      // X = 0.5 (3X - atmp2)
                copy_mat(s, n, n, XsX, n, atmp);
                axpby_diag(s, n, n, 0.0, nullptr, -1.0, atmp, 1.0);   // I - XsX
                if (x.frob(atmp) < x.thr.low) break;
                x.nan_check(XsX, "Error, NaN encountered");
            }
        } else {
            set_identity(s, n, n, X, 0.0);
        }
        return;
    }
    // eigendecomposition of S: X = V D V^T with D = 1/w or 1/sqrt(w)
    double* V = x.m[4];
    copy_mat(s, n, n, S, n, V);
    DevBuf w;
    w.reserve(sizeof(double) * n);
    dsyevd(x.c, n, n, V, w.as<double>());
    std::vector<double> hw(n);
    PTB_CUDA(cudaMemcpy(hw.data(), w.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost));
    for (auto& v : hw) {
        if (pur.metric_type == PTBGPU_METRIC_INV) v = 1.0 / v;
        else if (pur.metric_type == PTBGPU_METRIC_INV_SQRT) v = 1.0 / std::sqrt(v);
        else v = 0.0;
    }
    PTB_CUDA(cudaMemcpy(w.ptr, hw.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    k_scale_cols<<<g1(n), 256, 0, s>>>(n, V, w.as<double>(), atmp2);
    count_launch();
    PTB_CUDA(cudaGetLastError());
    x.gemm(atmp2, V, X, 1.0, true);
    w.release();
}

// build_guess, source/purification.f90:355-436.
void build_guess(Ctx& x, const ptbgpu_pur_settings& pur, const double* H, const double* X, double chempot,
                 double* guess) {
    const int64_t n = x.n;
    cudaStream_t s = x.c->stream;
    double* t2 = x.m[4];
    double* t3 = x.m[5];
    if (pur.type == PTBGPU_TYPE_MCWEENY) {
        x.gemm(H, X, t2);
        x.gemm(X, t2, t3);
        axpby_diag(s, n, n, chempot, X, -1.0, t3, 0.0);   // term4 = mu X - X H X
        const double a = 1.0 / std::min(x.frob(t3), colabs_max_dev(x.c, n, n, t3));
        copy_mat(s, n, n, X, n, guess);
        axpby_diag(s, n, n, 0.5 * a, t3, 0.5, guess, 0.0);   // 0.5 (a term4 + X)
        return;
    }
    if (pur.metric_type == PTBGPU_METRIC_INV_SQRT) {
        x.gemm(H, X, t2);
        x.gemm(X, t2, t3);
        axpby_diag(s, n, n, 0.0, nullptr, 1.0, t3, -chempot);   // X H X - mu I
    } else if (pur.metric_type == PTBGPU_METRIC_INV) {
        x.gemm(X, H, t3);
        axpby_diag(s, n, n, 0.0, nullptr, 1.0, t3, -chempot);   // X H - mu I
    } else {
        set_identity(s, n, n, guess, 0.0);
        return;
    }
    const double a = 1.0 / std::min(x.frob(t3), colabs_max_dev(x.c, n, n, t3));
    copy_mat(s, n, n, t3, n, guess);
    axpby_diag(s, n, n, 0.0, nullptr, a, guess, 0.0);
}

// mcweeny_, source/purification.f90:438-510: P <- 3PSP - 2PSPSP, stop on
// | ||P||_F - ||P_prev||_F | < thrs%normal, then P*2.
void mcweeny(Ctx& x, const ptbgpu_pur_settings& pur, const double* guess, const double* S, double* P) {
    const int64_t n = x.n;
    cudaStream_t s = x.c->stream;
    double* g = x.m[4];
    double* t1 = x.m[5];
    double* t2 = x.m[6];
    double* t3 = x.m[7];
    copy_mat(s, n, n, guess, n, g);
    double norm = x.frob(g);
    copy_mat(s, n, n, guess, n, P);
    auto step = [&] {
        x.gemm(S, g, t1);
        x.gemm(g, t1, t2);
        x.gemm(t2, t1, t3);
        copy_mat(s, n, n, t2, n, P);
        axpby_diag(s, n, n, -2.0, t3, 3.0, P, 0.0);
    };
    for (int64_t i = 0; i < pur.cycles; ++i) {
        step();
        x.nan_check(P, "Error: NaN is encountered during purification");
        const double np = x.frob(P);
        if (std::fabs(np - norm) < x.thr.normal) break;
        copy_mat(s, n, n, P, n, g);
        norm = np;
        // the remaining iterations as one graph launch (the stop rule on the device)
        if (i + 1 < pur.cycles && graph_loops()) {
            LoopDev* d = x.ld();
            auto body = [&] {
                step();
                nan_flag_dev(x.c, n * n, P, &d->nan);
                frob_to_dev(x.c, n, n, P, &d->norm1);
                copy_mat(s, n, n, P, n, g);   // the next iteration's input (unused after the last)
            };
            if (x.build_loop(x.mcw_loop, body, x.thr.normal, (long long)pur.cycles, 1)) {
                const LoopDev r = x.run_loop(x.mcw_loop, LoopDev{norm, 0.0, (long long)(i + 1), 0, 0});
                PTB_CHECK(r.nan == 0, PTBGPU_ENAN, "%s", "Error: NaN is encountered during purification");
                break;
            }
        }
    }
    axpby_diag(s, n, n, 0.0, nullptr, 2.0, P, 0.0);
}

// sign_to_density_matrix, source/purification.f90:603-647 (without the caller's *2).
void sign_to_density(Ctx& x, const ptbgpu_pur_settings& pur, const double* sign, const double* X, double* P) {
    const int64_t n = x.n;
    cudaStream_t s = x.c->stream;
    double* ims = x.m[6];
    double* tmp = x.m[7];
    copy_mat(s, n, n, sign, n, ims);
    axpby_diag(s, n, n, 0.0, nullptr, -1.0, ims, 1.0);   // I - sign
    if (pur.metric_type == PTBGPU_METRIC_INV_SQRT) {
        x.gemm(ims, X, tmp);
        x.gemm(X, tmp, P, 0.5);
    } else if (pur.metric_type == PTBGPU_METRIC_INV) {
        x.gemm(ims, X, P, 0.5);
    } else {
        set_identity(s, n, n, P, 0.0);
    }
    x.nan_check(P, "Error: NaN is encountered during purification");
}

// sign_iterative, source/purification.f90:512-601.
void sign_iterative(Ctx& x, const ptbgpu_pur_settings& pur, const double* guess, const double* X, double* P,
                    int64_t* iters) {
    const int64_t n = x.n;
    cudaStream_t s = x.c->stream;
    double* Y = x.m[4];
    double* t1 = x.m[5];
    double* t2 = x.m[6];
    double* t3 = x.m[7];
    copy_mat(s, n, n, guess, n, Y);
    auto step = [&] {
        if (pur.type == PTBGPU_TYPE_PADE) {
            x.gemm(Y, Y, t1);
            x.gemm(t1, t1, t2);
            copy_mat(s, n, n, t2, n, t3);
            axpby_diag(s, n, n, -10.0, t1, 3.0, t3, 15.0);   // 15 I - 10 X^2 + 3 X^4
            x.gemm(Y, t3, t1, 0.125);
            copy_mat(s, n, n, t1, n, Y);
        } else {
            x.gemm(Y, Y, t1);
            x.gemm(Y, t1, t2);
            axpby_diag(s, n, n, -0.5, t2, 1.5, Y, 0.0);      // 0.5 (3X - X^3)
        }
    };
    for (int64_t i = 0; i < pur.cycles; ++i) {
        const double norm = x.frob(Y);
        ++*iters;
        step();
        x.nan_check(Y, "Error: NaN is encountered during purification");
        if (std::fabs(x.frob(Y) - norm) < x.thr.normal) break;
        // the remaining iterations as one graph launch (the stop rule on the device)
        if (i + 1 < pur.cycles && graph_loops()) {
            LoopDev* d = x.ld();
            auto body = [&] {
                frob_to_dev(x.c, n, n, Y, &d->norm0);
                step();
                nan_flag_dev(x.c, n * n, Y, &d->nan);
                frob_to_dev(x.c, n, n, Y, &d->norm1);
            };
            if (x.build_loop(x.sign_loop, body, x.thr.normal, (long long)pur.cycles, 0)) {
                const LoopDev r = x.run_loop(x.sign_loop, LoopDev{0.0, 0.0, (long long)(i + 1), 0, 0});
                *iters += r.iters - (i + 1);
                PTB_CHECK(r.nan == 0, PTBGPU_ENAN, "%s", "Error: NaN is encountered during purification");
                break;
            }
        }
    }
    // sign_to_density uses m[6], m[7]; keep Y in m[4]
    sign_to_density(x, pur, Y, X, P);
    axpby_diag(s, n, n, 0.0, nullptr, 2.0, P, 0.0);
}

// sign_diagonalization_, source/purification.f90:650-782.  chempot is updated
// in place like the reference's intent(inout) argument.
void sign_diag(Ctx& x, const ptbgpu_pur_settings& pur, double& chempot, const double* guess, const double* X,
               double* P) {
    const int64_t n = x.n;
    cudaStream_t s = x.c->stream;
    double* V = x.m[4];
    double* tmp = x.m[5];
    copy_mat(s, n, n, guess, n, V);
    DevBuf w, cs;
    w.reserve(sizeof(double) * n);
    cs.reserve(sizeof(double) * n);
    dsyevd(x.c, n, n, V, w.as<double>());
    k_colsq<<<g1(n), 256, 0, s>>>(n, V, cs.as<double>());
    count_launch();
    PTB_CUDA(cudaGetLastError());
    std::vector<double> hw(n), hcs(n), sgn(n, 0.0);
    PTB_CUDA(cudaMemcpyAsync(hw.data(), w.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaMemcpyAsync(hcs.data(), cs.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    PTB_CUDA(cudaStreamSynchronize(s));
    const double nel = (double)(float)pur.nel;
    double incr = pur.chempot_increment, lower = 0.0, upper = 0.0;
    bool is_lower = false, is_upper = false;
    for (int64_t k = 0; k < pur.chempot_cycles; ++k) {
        double nelcalc = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            const double eg = hw[i] - chempot;
            sgn[i] = (std::fabs(eg) < x.thr.normal) ? 0.0 : (eg > 0.0 ? 1.0 : -1.0);
            nelcalc += 1.0 - hcs[i] * sgn[i];
        }
        if (std::fabs(nelcalc - nel) < x.thr.normal) break;
        if (nelcalc < nel) {
            is_lower = true;
            lower = chempot;
            chempot += incr;
        } else {
            is_upper = true;
            upper = chempot;
            chempot -= incr;
        }
        incr *= 2.0;
        if (is_lower && is_upper) {
            chempot = 0.5 * (lower + upper);
            if (std::fabs(upper - lower) < x.thr.high) break;
        }
    }
    PTB_CUDA(cudaMemcpyAsync(w.ptr, sgn.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
    k_scale_cols<<<g1(n), 256, 0, s>>>(n, V, w.as<double>(), tmp);   // V diag(sgn)
    PTB_CUDA(cudaGetLastError());
    count_launch();
    double* sign = x.m[6];
    x.gemm(tmp, V, sign, 1.0, true);                                  // Q sgn Q^T
    copy_mat(s, n, n, sign, n, x.m[5]);
    sign_to_density(x, pur, x.m[5], X, P);
    axpby_diag(s, n, n, 0.0, nullptr, 2.0, P, 0.0);
    PTB_CUDA(cudaStreamSynchronize(s));
    w.release();
    cs.release();
}

}  // namespace

// purification_wrapper + purification_search, source/purification.f90:28-80, 232-353.
void purify_ref_device(ptbgpu_ctx* c, const ptbgpu_pur_settings& pur, int64_t n, const double* dH,
                       const double* dS, double* dP, const ptbgpu_opts* o, ptbgpu_stats* st) {
    PTB_CHECK(n > 0, PTBGPU_EINVAL, "ndim must be positive");
    PTB_CHECK(pur.type >= 1 && pur.type <= 4, PTBGPU_EINVAL, "invalid purification type %lld",
              (long long)pur.type);
    const int prl = o ? (int)o->print_level : 0;
    const double filter = o ? o->filter : 0.0;
    cudaStream_t s = c->stream;
    DevBuf& bh = c->buf(B_H);
    DevBuf& bs = c->buf(B_S);
    DevBuf& bp = c->buf(B_W0);
    DevBuf& bx = c->buf(B_W1);
    DevBuf& bg = c->buf(B_W2);
    for (DevBuf* b : {&bh, &bs, &bp, &bx, &bg}) b->reserve(sizeof(double) * n * n);
    double* H = bh.as<double>();
    double* S = bs.as<double>();
    double* P = bp.as<double>();
    double* X = bx.as<double>();
    double* guess = bg.as<double>();
    unpack_sym(s, n, n, dH, H, filter);
    unpack_sym(s, n, n, dS, S, filter);
    Ctx x(c, n, prl);
    transformation(x, pur, S, X);

    double chempot = pur.chempot_guess, incr = pur.chempot_increment, lower = 0.0, upper = 0.0;
    bool is_lower = false, is_upper = false, bisection = false;
    int64_t steps = 0, iters = 0;
    const double nel = (double)pur.nel;
    for (int64_t i = 0; i < pur.chempot_cycles; ++i) {
        if (bisection) {
            chempot = 0.5 * (lower + upper);
            if (std::fabs(upper - lower) < x.thr.high) {
                log_line(prl, 1, "Chemical potential search. Too short/big interval to bisect. %lld cycles",
                         (long long)(i + 1));
                break;
            }
        }
        build_guess(x, pur, H, X, chempot, guess);
        if (pur.type == PTBGPU_TYPE_MCWEENY)
            mcweeny(x, pur, guess, S, P);
        else if (pur.type == PTBGPU_TYPE_PADE || pur.type == PTBGPU_TYPE_NEWTON)
            sign_iterative(x, pur, guess, X, P, &iters);
        else
            sign_diag(x, pur, chempot, guess, X, P);
        ++steps;
        const double nel_calc = trace_prod_dev(c, n, n, P, S);
        if (pur.type != PTBGPU_TYPE_DIAG)
            log_line(prl, 1, "Search number: %lld  chemical potential: %.8f  electrons: %.8f", (long long)(i + 1),
                     chempot, nel_calc);
        if (std::fabs(nel_calc - (double)(float)pur.nel) < x.thr.normal) break;
        if (nel_calc < nel) {
            is_lower = true;
            lower = chempot;
            chempot += incr;
        } else {
            is_upper = true;
            upper = chempot;
            chempot -= incr;
        }
        bisection = is_lower && is_upper;
        incr *= 2.0;
    }
    oz_check(c, "int8 product (purification module)");
    pack_cols(s, n, n, P, dP);
    if (st) {
        st->mu = chempot;
        st->mu_iterations = steps;
        st->iterations = iters;
        st->flops = x.gemm_flops;
    }
}

}  // namespace ptb
