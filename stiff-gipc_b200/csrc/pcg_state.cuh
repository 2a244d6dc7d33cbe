// pcg_state.cuh -- device-side PCG state transition shared by the kernels
// that end an iteration.
#pragma once
#include "ctx.hpp"

// PCG state transition at the end of an iteration (PCGSolver::pcg :251-299);
// kind 1 = after the initial apply, 2 = regular iteration, 3 = profiling replay.
__device__ __forceinline__ void pcg_end_iteration(PcgState* st, double rz_new, double rr, int kind, int set_cond,
                                  unsigned long long cond) {
    if (kind == 3) {  // profiling replay: reduce, leave the loop state alone
        st->rz_new = rz_new;
        return;
    }
    if (kind == 1) {
        st->rz = rz_new;
        st->rz0 = rz_new;
        st->rr0 = st->warm ? st->w_bb : rr;  // a start guess: convergence relative to ||b||
        st->rr = rr;
        st->k = 1;
        st->beta = 0.0;
        st->done = st->max_iter <= 1;
        st->iters = 1;
    } else {
        const int k = st->k;
        st->rz_new = rz_new;
        bool conv = false;
        if (k % st->check_every == 0) {
            st->rr = rr;
            conv = st->use_prec_norm ? (rz_new <= st->rel2 * st->rz0 || rz_new <= st->abs2)
                                     : (rr <= st->rel2 * st->rr0 || rr <= st->abs2);
            if (!(rz_new == rz_new) || !(rr == rr)) conv = true;  // non-finite: stop, host reports it
        }
        if (conv) {
            st->done = 1;
            st->iters = k;
            st->converged = (rz_new == rz_new) && (rr == rr);
        } else {
            st->beta = rz_new / st->rz;
            st->rz = rz_new;
            st->k = k + 1;
            if (k + 1 >= st->max_iter) { st->done = 1; st->iters = k + 1; }
        }
    }
    if (set_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, st->done ? 0u : 1u);
}

