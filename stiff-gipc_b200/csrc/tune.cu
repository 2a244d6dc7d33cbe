// tune.cu -- the autotuner of the PCG loop's launch shape.
//
// The persistent form (pcg_persistent.cu) runs on any grid from the fewest
// CTAs whose level-0 subdomains fit one slot per thread up to one CTA per SM;
// the graph form (pcg.cu) always fits and uses the whole GPU.  Which is best
// depends on the system and on what else shares the GPU: alone, the fastest
// loop wins (latency); beside other solves, the one with the least SM-time
// per iteration does (throughput), since the SMs it leaves free run other
// scenes.  The tuner times short trial solves of each candidate on the real
// system and keeps the best on the context.  The reference has no such step
// (its solve always launches the same kernels); this is the project's own.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/sgmas.h"
#include "ctx.hpp"

using namespace sgmas;

extern "C" {

int sgmas_autotune_pcg(sgmas_context* c, const sgmas_bcoo* A, const double* d_b, const sgmas_pcg_config* cfg,
                       int objective, int concurrency, int trial_iters, int reps, sgmas_tune_report* report) {
    if (!c || !A || !d_b || !cfg) return SGMAS_ERR_ARG;
    if (objective != SGMAS_TUNE_LATENCY && objective != SGMAS_TUNE_THROUGHPUT)
        return ctx_fail(c, SGMAS_ERR_ARG, "objective must be SGMAS_TUNE_LATENCY or SGMAS_TUNE_THROUGHPUT");
    if (trial_iters < 2 || reps < 1 || concurrency < 1)
        return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_autotune_pcg: trial_iters >= 2, reps >= 1, concurrency >= 1 required");
    if (A->n_block_rows < 1) return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_autotune_pcg: bad matrix");
    SG_CUDA(c, cudaSetDevice(c->device));
    int sms = 0;
    SG_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));

    // candidates: persistent grids from the fewest CTAs that can hold every
    // level-0 subdomain (one slot per thread: 512 / bank subdomains per CTA)
    // up to every SM, about x1.4 apart; then the graph form (ctas = 0)
    std::vector<int> grids;
    const int per_cta = 512 / c->bank;
    int g = 1;
    if (cfg->preconditioner == 1 && c->mas_init) g = std::max(1, (c->Mm / c->bank + per_cta - 1) / per_cta);
    g = std::min(g, sms);
    while (g < sms && (int)grids.size() < SGMAS_TUNE_MAX_CANDIDATES - 2) {
        grids.push_back(g);
        g = std::max(g + 1, (int)std::ceil(g * 1.4));
    }
    grids.push_back(sms);

    // scratch solution (kept on the context: the last solve's vectors stay valid for sgmas_pcg_profile)
    if (ctx_alloc_grow(c, &c->d_tune_x, &c->tune_cap, 3 * A->n_block_rows)) return SGMAS_ERR_CUDA;
    double* x = c->d_tune_x;
    sgmas_pcg_config tc = *cfg;
    tc.max_iter = trial_iters;
    tc.initial_guess = 0;
    const bool was_persistent = c->persistent;
    const int was_ctas = c->pcg_ctas;

    sgmas_tune_report r = {};
    r.sms = sms;
    int rc = SGMAS_OK;
    auto trial = [&](int ctas, bool persistent) -> int {
        c->persistent = persistent;
        c->pcg_ctas = ctas;
        double best = INFINITY;
        int ran_persistent = 0;
        for (int k = 0; k < reps; ++k) {
            sgmas_pcg_report pr = {};
            const int e = sgmas_pcg_solve(c, A, d_b, x, &tc, &pr);
            if (e) return e;
            if (pr.iterations < 1) continue;
            best = std::min(best, 1e3 * (double)pr.solve_ms / pr.iterations);
            ran_persistent = pr.kernel_launches == 1;
        }
        const int i = r.n_candidates++;
        r.ctas[i] = persistent ? (ran_persistent ? ctas : 0) : 0;
        r.persistent[i] = ran_persistent;
        r.us_per_iter[i] = best;
        // SM-time, each solve charged at least its share of the GPU: with
        // `concurrency` solves in flight, SMs a smaller grid leaves free idle
        const double used = std::max((double)(ran_persistent ? std::min(ctas, sms) : sms), (double)sms / concurrency);
        r.cost[i] = objective == SGMAS_TUNE_LATENCY ? best : best * used;
        return 0;
    };
    // largest grid first: a grid too small for the system ran the graph form,
    // and every smaller grid would too (more subdomains per CTA), so stop there
    for (int q = (int)grids.size() - 1; q >= 0; --q) {
        if ((rc = trial(grids[q], true))) break;
        if (!r.persistent[r.n_candidates - 1]) { r.n_candidates--; break; }
    }
    if (!rc) {  // persistent candidates in ascending grid order, then the graph form
        std::reverse(r.ctas, r.ctas + r.n_candidates);
        std::reverse(r.persistent, r.persistent + r.n_candidates);
        std::reverse(r.us_per_iter, r.us_per_iter + r.n_candidates);
        std::reverse(r.cost, r.cost + r.n_candidates);
        rc = trial(0, false);
    }
    if (rc) {
        c->persistent = was_persistent;
        c->pcg_ctas = was_ctas;
        return rc;
    }
    int best = 0;
    for (int i = 1; i < r.n_candidates; ++i)
        if (r.cost[i] < r.cost[best]) best = i;
    r.chosen = best;
    c->persistent = r.persistent[best] != 0;
    c->pcg_ctas = r.persistent[best] ? r.ctas[best] : 0;
    if (report) *report = r;
    return SGMAS_OK;
}

}  // extern "C"
