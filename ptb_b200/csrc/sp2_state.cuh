// State and stopping rule of the trace-correcting (SP2) purification on the
// device, shared by the single-system path (sp2.cu) and the grouped one
// (sp2_batch.cu).
#pragma once

#include <cmath>

#include "ptbgpu.h"

namespace ptb {

constexpr int kMaxIt = 255;
// Contraction of the refinement rounds per unit response gain g of the first
// round (measured bounds, see sp2_mixed): the first round leaves at most
// kRho1 * g of its correction, every later one at most kRho2 * g of its own.
constexpr double kRho1 = 6.5e-5;
constexpr double kRho2 = 2.6e-4;

struct SP2State {
    int active;      // 1 while pass 1 runs; product/decision launches are no-ops at 0
    int next;        // index of the iterate the next decision evaluates
    int converged;
    int status;      // 0 or a PTBGPU_E* code
    int sq_cur;      // branch for the step about to run
    int pad[3];
    double trX[kMaxIt + 1];
    double trX2[kMaxIt + 1];
    double err[kMaxIt + 1];
    int sq[kMaxIt + 1];
};

// Record iterate k's traces and decide the next step (one thread): the branch
// by the trace (Niklasson's trace correction), the stop at the rounding floor,
// the iteration cap.
__device__ __forceinline__ void sp2_decide(SP2State* st, double trX, double trX2, double N, double tol_abs,
                                           double e_asym, double e_stag, int maxit) {
    const int k = st->next;
    const double e = trX - trX2;
    st->trX[k] = trX;
    st->trX2[k] = trX2;
    st->err[k] = e;
    if (!(e == e)) {
        st->status = PTBGPU_ENAN;
        st->active = 0;
        return;
    }
    const int sq = fabs(trX2 - N) <= fabs(2.0 * trX - trX2 - N) ? 1 : 0;
    st->sq[k] = sq;
    st->sq_cur = sq;
    const double ae = fabs(e);
    // Rounding floor: in the asymptotic regime (every eigenvalue within ~0.1 of
    // 0 or 1, which e < e_asym implies) two exact steps always lower e, so no
    // decrease over two steps means rounding; above e_asym states near a small
    // gap can hold e level for a step or two, so there only six steps that all
    // stay above the best error before them count (for floors above e_asym).
    bool conv = ae < tol_abs || (k >= 2 && ae < e_asym && ae >= fabs(st->err[k - 2]));
    if (!conv && k >= 8 && ae < e_stag) {
        double before = fabs(st->err[0]), window = ae;
        for (int j = 1; j <= k - 6; ++j) before = fmin(before, fabs(st->err[j]));
        for (int j = k - 5; j < k; ++j) window = fmin(window, fabs(st->err[j]));
        conv = window >= before;
    }
    if (conv) {
        st->converged = 1;
        st->active = 0;
    } else if (k >= maxit || k >= kMaxIt) {
        st->status = PTBGPU_EITER;
        st->active = 0;
    } else {
        st->next = k + 1;
    }
}

}  // namespace ptb
