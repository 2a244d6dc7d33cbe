// pcg_persistent.cu -- the whole PCG solve (PCGSolver::pcg,
// SG/linear_system/solver/pcg_solver.cu:171-304) with the MAS preconditioner
// (MASPreconditioner::preconditioning, SG/MASPreconditioner.cu:2173-2196) as
// one cooperative, persistent kernel: one CTA per SM for the whole loop.
//
// Ownership.  Level-1 nodes of the MAS hierarchy are numbered in level-0 bank
// order (component ids are an exclusive scan over the banks), so a range of
// level-1 banks is fed by a range of level-0 banks.  CTA c owns a contiguous
// range of level-1 banks (chosen on the host so that the largest number of
// level-0 banks any CTA processes is as small as possible) and processes
// every level-0 bank whose components fall in them (a bank split between two CTAs is processed by both; each vertex
// belongs to the CTA that owns its level-1 node).  Level 0, level 1 and the
// push of level-1 residuals into level 2 then need no grid-wide step; the few
// nodes of levels >= 2 are processed redundantly by every CTA in shared
// memory.  An iteration is three phases with a grid barrier after each:
//   A  p = z + beta p_old, Ap = A p, p.Ap partials            (SpMV)
//   B  x += alpha p, r -= alpha Ap, level-0 and level-1 Schwarz, R2 push
//   C  levels >= 2 (redundant per CTA) + CollectFinalZ, r.z / r.r partials
// (B and C fuse when the hierarchy has at most two levels.)  Every 10th
// iteration adds x += alpha p | r = b - A x (the reference's true residual).
//
//  * Each thread keeps its level-0 slot's x, r and level-0 Schwarz result in
//    registers across the phases; x and r reach global memory only for the
//    residual refresh and at the end.
//  * The CTA partials of p.Ap, r.z, r.r go to a small array; every CTA sums
//    all partials in CTA order itself (same values everywhere, deterministic).
//  * Subdomain inverse tiles (levels 0, 1 and, when they fit, >= 2) are
//    copied into shared memory once per solve (one bulk copy) and stay there.
//  * Data written by other CTAs in an earlier phase is read with plain weak
//    loads: the grid barrier is a release (red.release) / acquire
//    (ld.acquire) pair, after which weak loads see every write before it.
//  * Sums keep the order of the graph-form kernels (component sums and group
//    sums in lane order, Schwarz columns ascending, collect in level order),
//    so z is bit-identical to sgmas_mas_apply.
#include <algorithm>
#include <vector>

#include "../../include/sgmas.h"
#include "ctx.hpp"
#include "mas_dev.cuh"
#include "spmv_dev.cuh"
#include "extra_dev.cuh"
#include "patch_dev.cuh"

using namespace sgmas;

namespace {

constexpr int kPT = 512;  // threads per CTA

struct PArgs {
    BsrView A;
    const double* b;
    double *x, *r, *z, *p0, *p1, *Ap;
    int nrows;
    // SpMV plan (k_spmv_plan): per CTA {units, halo offset, halo size, first unit}
    const int4* cinfo;
    const int4* udesc_c;  // work-unit descriptors of every CTA, [first unit + u][lane group]
    const int* lcols;     // halo-local column index of every stored block
    const int* halo;      // vertex of each halo index (per CTA from its halo offset)
    int hcap;             // halo entries staged in shared memory (the largest halo)
    // MAS
    int N, Mm, L, total;
    int lvl_count[kMaxLevels + 2], lvl_begin[kMaxLevels + 2];
    const int *part_map, *going_next, *coarse_table;
    const unsigned* fine_mask;
    const int* l1_bank;  // level-0 bank of each level-1 node
    const int* own1;     // [grid + 1]: CTA c owns level-1 banks [own1[c], own1[c + 1])
    const void* inv;
    void* R;             // level-2 residual pushes (Acc, global node ids)
    int k0, k1, nb0, nb1;  // level-0 banks per CTA (max), level-1 banks per CTA, bank counts
    int nc;                // nodes of levels >= 2 (a multiple of B)
    int capc;              // tiles of levels >= 2 a CTA holds in shared memory (<= kPT / B)
    int t0g, t1g;          // level-0 / level-1 tiles read from global memory (they did not fit)
    int upw;               // SpMV unit descriptors cached per warp in shared memory
    ExtraRows ex;          // rows outside the MAS range (bodies, other rows); MAS vertex v is row ex.fem_off + v
    PatchView pv;          // body patches (pv.bodies = 0: none)
    // block-Jacobi
    const double* dinv;
    int abd_rows, precond;
    // control
    int max_iter, check_every, use_prec_norm;
    int warm;          // x holds a start guess (scaled, rejected when it raises ||r0||)
    double rel2, abs2;
    double* partials;  // [4][grid]
    unsigned* sync;    // [0] barrier arrivals (monotonic)
    int spin_limit;    // polls of each grid barrier / mbarrier wait before it gives up
    int phantom;       // arrivals each grid barrier expects beyond the grid (fault injection; 0 normally)
    PcgState* st;
    int* err;
    // optional phase stamps (clock64 of CTA 0): [0] start, [1] end, [2] loop
    // passes, then 8 per iteration k = 1..stamp_iters at 8 * (k + 1): loop
    // top, after the SpMV barrier, after the refresh, after the level 0-1
    // barrier (0 when fused), -, after the last barrier.  From
    // 8 * (stamp_iters + 2) on, 16 per CTA: per barrier slot (0 SpMV, 1 x
    // refresh, 2 r refresh, 3 levels 0-1, 5 end of iteration) the cycles of
    // work before it and of waiting in it, summed over the loop.
    unsigned long long* stamps;
    int stamp_iters;
};

__device__ __forceinline__ void stamp(const PArgs& a, int k, int slot) {
    if (a.stamps && blockIdx.x == 0 && threadIdx.x == 0 && k <= a.stamp_iters)
        a.stamps[8 * (size_t)(k + 1) + slot] = clock64();
}

// ---- grid barrier: monotonic arrival counter, release add / acquire poll ---
// Barrier number `epoch` (1, 2, ...) completes when the counter reaches
// epoch * (gridDim.x + phantom).  At most `limit` polls; a timeout sets the
// error flag.  (phantom > 0 makes every barrier wait for arrivals that never
// come: the host's fault injection for the timeout path.)
// acc (thread 0 of each CTA, profiling only): += work and wait cycles of this
// barrier slot; t_rel carries the previous release time.
// The split form: grid_arrive by one thread, after a CTA or named barrier that
// orders the CTA's writes before it; grid_barrier(..., arrive = false) then
// completes the next barrier without arriving again.
__device__ __forceinline__ void grid_arrive(unsigned* count) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(count) : "memory");
}

__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned& epoch, int* err, int limit, int phantom,
                                             unsigned long long* acc = nullptr, long long* t_rel = nullptr,
                                             bool arrive = true) {
    __shared__ int ok_sh;
    __syncthreads();
    if (threadIdx.x == 0) {
        const long long t_arrive = acc ? clock64() : 0;
        epoch += 1u;
        const unsigned target = epoch * (gridDim.x + (unsigned)phantom);
        if (arrive) grid_arrive(count);
        int ok = 0;
        for (int it = 0; it < limit; ++it) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if ((int)(v - target) >= 0) { ok = 1; break; }
        }
        if (!ok) set_error(err, kDevWaitTimeout);
        ok_sh = ok;
        if (acc) {
            const long long t = clock64();
            acc[0] += (unsigned long long)(t_arrive - *t_rel);
            acc[1] += (unsigned long long)(t - t_arrive);
            *t_rel = t;
        }
    }
    __syncthreads();
    return ok_sh != 0;
}

// sum of the grid's partials (every thread of every CTA gets the same value):
// warp 0 reads them lane-strided and folds them with an xor butterfly, whose
// additions pair the same operands in every lane and every CTA; one warp per
// CTA keeps the L2 requests to the shared partial lines few
__device__ __forceinline__ double sum_partials(const double* part) {
    __shared__ double out;
    if (threadIdx.x < 32) {
        double s = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) s += __ldcg(part + i);
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) out = s;
    }
    __syncthreads();
    const double v = out;
    __syncthreads();
    return v;
}

// both sums of the end of an iteration in one pass
__device__ __forceinline__ void sum_partials2(const double* pa, const double* pb, double& va, double& vb) {
    __shared__ double out2[2];
    if (threadIdx.x < 32) {
        double s0 = 0.0, s1 = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) { s0 += __ldcg(pa + i); s1 += __ldcg(pb + i); }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        }
        if (threadIdx.x == 0) { out2[0] = s0; out2[1] = s1; }
    }
    __syncthreads();
    va = out2[0];
    vb = out2[1];
    __syncthreads();
}

// two block sums in one pass (valid in thread 0)
__device__ __forceinline__ void block_sum2(double& a, double& b, double* sh) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sh[w] = a; sh[16 + w] = b; }
    __syncthreads();
    if (threadIdx.x < 32) {
        a = threadIdx.x < kPT / 32 ? sh[threadIdx.x] : 0.0;
        b = threadIdx.x < kPT / 32 ? sh[16 + threadIdx.x] : 0.0;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
    __syncthreads();
}

// ---- block-Jacobi tail (z = D^-1 r with 3x3 inverses) ----------------------
__device__ void phase_jacobi(const PArgs& a, int mode, double alpha, const double* pcur, double* part_rz,
                             double* part_rr, double* sh) {
    double rz = 0.0, rr = 0.0;
    // body rows first: 12x12 block-Jacobi per affine body (a.ex lists the bodies)
    extra_rows_work(a.ex, 0, mode, alpha, a.x, a.r, pcur, a.Ap, a.z, blockIdx.x * (kPT / 32) + threadIdx.x / 32,
                    gridDim.x * (kPT / 32), threadIdx.x & 31, rz, rr);
    for (int i = a.abd_rows + blockIdx.x * kPT + threadIdx.x; i < a.nrows; i += gridDim.x * kPT) {
        double rv[3], xv[3], pv[3], qv[3], D[9];
        #pragma unroll
        for (int d = 0; d < 3; ++d) rv[d] = a.r[3 * (size_t)i + d];
        #pragma unroll
        for (int q = 0; q < 9; ++q) D[q] = a.dinv[9 * (size_t)i + q];
        if (mode == 1) {  // every load before the first store (the pointers may alias)
            #pragma unroll
            for (int d = 0; d < 3; ++d) {
                xv[d] = a.x[3 * (size_t)i + d];
                pv[d] = pcur[3 * (size_t)i + d];
                qv[d] = a.Ap[3 * (size_t)i + d];
            }
            #pragma unroll
            for (int d = 0; d < 3; ++d) {
                rv[d] = rv[d] - alpha * qv[d];
                a.x[3 * (size_t)i + d] = xv[d] + alpha * pv[d];
                a.r[3 * (size_t)i + d] = rv[d];
            }
        }
        rr += rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
        double zv[3];
        #pragma unroll
        for (int d = 0; d < 3; ++d) zv[d] = D[3 * d] * rv[0] + D[3 * d + 1] * rv[1] + D[3 * d + 2] * rv[2];
        #pragma unroll
        for (int d = 0; d < 3; ++d) a.z[3 * (size_t)i + d] = zv[d];
        rz += rv[0] * zv[0] + rv[1] * zv[1] + rv[2] * zv[2];
    }
    block_sum2(rz, rr, sh);
    if (threadIdx.x == 0) { part_rz[blockIdx.x] = rz; part_rr[blockIdx.x] = rr; }
}

// per-CTA ranges of the MAS ownership
struct Own {
    int lo, nbk0;  // level-0 banks [lo, lo + nbk0)
    int j0, nbk1;  // level-1 banks [j0, j0 + nbk1) (bank index within level 1)
};

template <int B>
__device__ __forceinline__ Own own_ranges(const PArgs& a) {
    Own o;
    if (a.L >= 2) {
        const int cnt1 = a.lvl_count[1];
        o.j0 = a.own1[blockIdx.x];
        const int j1 = a.own1[blockIdx.x + 1];
        o.nbk1 = max(0, j1 - o.j0);
        const int n_lo = o.j0 * B, n_hi = min(j1 * B, cnt1) - 1;
        if (n_lo <= n_hi) {
            o.lo = a.l1_bank[n_lo];
            o.nbk0 = a.l1_bank[n_hi] - o.lo + 1;
        } else {
            o.lo = 0;
            o.nbk0 = 0;
        }
    } else {
        o.j0 = 0;
        o.nbk1 = 0;
        o.lo = blockIdx.x * a.k0;
        o.nbk0 = max(0, min(a.k0, a.nb0 - o.lo));
    }
    return o;
}

// Schwarz of `nbk` banks whose residuals are in shared memory (rs, node-local
// index) with tiles at `tiles`; results to zs.  Warps whose half-warps are all
// idle skip (the shuffles need whole warps).
template <int B, typename S, typename Acc>
__device__ __forceinline__ void smem_banks(const S* tiles, const Acc* rs, Acc* zs, int nbk, Acc* xch) {
    constexpr int bs = bsym_of(B);
    constexpr int HPW = 32 / B;
    const int lane = threadIdx.x % B;
    for (int q0 = 0; q0 < nbk; q0 += kPT / B) {
        const int hw = q0 + threadIdx.x / B;
        if ((hw / HPW) * HPW >= nbk) continue;  // whole warp idle
        const bool valid = hw < nbk;
        const int i = hw * B + lane;
        const Acc v0 = valid ? rs[3 * i] : (Acc)0, v1 = valid ? rs[3 * i + 1] : (Acc)0,
                  v2 = valid ? rs[3 * i + 2] : (Acc)0;
        Acc* xb = bank_slot<B>(xch);
        xch_put(xb, lane, v0, v1, v2);
        Acc z0, z1, z2;
        schwarz_rows<B, S, Acc>(tiles + (size_t)(valid ? hw : 0) * bs * 9, lane, xb, z0, z1, z2);
        if (valid) { zs[3 * i] = z0; zs[3 * i + 1] = z1; zs[3 * i + 2] = z2; }
    }
}

// Ancestor banks of this CTA's vertices at levels >= 2: node ids of every
// level are assigned in bank order, so each level's ancestors form one
// contiguous range of banks.  anc_lo[l] = first global bank, anc_nb[l] =
// banks at level l; the tiles of all of them, level after level, fill the
// first anc_total tiles of tilesC when anc_total <= capc.
struct Anc {
    int lo[kMaxLevels + 2], nb[kMaxLevels + 2];
    int total;
};

// levels >= 2, redundantly in every CTA: level-2 residuals from global memory,
// levels >= 3 by group sums in shared memory, then the Schwarz products of
// this CTA's ancestor banks (cached tiles, or staged per level).
template <int B, typename S, typename Acc>
__device__ __forceinline__ bool levels_c(const PArgs& a, const Anc& anc, S* tilesC, Acc* Rc, Acc* Zc,
                                         const int* parc, uint64_t* mbar, unsigned& mphase, Acc* xch) {
    constexpr int bs = bsym_of(B);
    constexpr int HPW = 32 / B;
    const int base = a.lvl_begin[2];
    const Acc* Rg = (const Acc*)a.R;
    for (int i = threadIdx.x; i < a.lvl_count[2]; i += kPT) {
        Rc[3 * i] = Rg[3 * (size_t)(base + i)];
        Rc[3 * i + 1] = Rg[3 * (size_t)(base + i) + 1];
        Rc[3 * i + 2] = Rg[3 * (size_t)(base + i) + 2];
    }
    __syncthreads();
    const int lane = threadIdx.x % B;
    for (int lvl = 3; lvl < a.L; ++lvl) {
        const int off = a.lvl_begin[lvl - 1] - base, cnt = a.lvl_count[lvl - 1];
        const int nb = (cnt + B - 1) / B;
        for (int q0 = 0; q0 < nb; q0 += kPT / B) {
            const int k = q0 + threadIdx.x / B;
            if ((k / HPW) * HPW >= nb) continue;
            const bool valid = k < nb && k * B + lane < cnt;
            const int i = off + k * B + lane;
            const Acc v0 = valid ? Rc[3 * i] : (Acc)0, v1 = valid ? Rc[3 * i + 1] : (Acc)0,
                      v2 = valid ? Rc[3 * i + 2] : (Acc)0;
            const int par = valid ? parc[i] : -1;
            Acc* xb = bank_slot<B>(xch);
            xch_put(xb, lane, v0, v1, v2);
            Acc s0, s1, s2;
            bool lead;
            group_sum<B, Acc>(par, xb, lane, s0, s1, s2, lead);
            if (lead) { Rc[3 * par] = s0; Rc[3 * par + 1] = s1; Rc[3 * par + 2] = s2; }
        }
        __syncthreads();
    }
    const int bbase = base / B;  // global bank index of the first level-2 bank
    if (anc.total <= a.capc) {   // one pass over all ancestor banks, tiles resident
        const int hw = threadIdx.x / B;
        if ((hw / HPW) * HPW < anc.total) {
            const bool valid = hw < anc.total;
            int l = 2, first = 0;  // level of entry hw
            while (l + 1 < a.L && hw >= first + anc.nb[l]) { first += anc.nb[l]; ++l; }
            const int i = valid ? (anc.lo[l] + hw - first - bbase) * B + lane : 0;
            const Acc v0 = valid ? Rc[3 * i] : (Acc)0, v1 = valid ? Rc[3 * i + 1] : (Acc)0,
                      v2 = valid ? Rc[3 * i + 2] : (Acc)0;
            Acc* xb = bank_slot<B>(xch);
            xch_put(xb, lane, v0, v1, v2);
            Acc z0, z1, z2;
            schwarz_rows<B, S, Acc>(tilesC + (size_t)(valid ? hw : 0) * bs * 9, lane, xb, z0, z1, z2);
            if (valid) { Zc[3 * i] = z0; Zc[3 * i + 1] = z1; Zc[3 * i + 2] = z2; }
        }
    } else {  // staged: each level's range in chunks of capc tiles
        for (int l = 2; l < a.L; ++l) {
            for (int c0 = 0; c0 < anc.nb[l]; c0 += a.capc) {
                const int ncb = min(a.capc, anc.nb[l] - c0);
                __syncthreads();  // the previous chunk's tiles are no longer read
                if (threadIdx.x == 0) {
                    const unsigned bytes = (unsigned)(ncb * bs * 9 * sizeof(S));
                    mbar_expect_tx(mbar, bytes);
                    bulk_g2s(tilesC, (const S*)a.inv + (size_t)(anc.lo[l] + c0) * bs * 9, bytes, mbar);
                }
                if (!mbar_wait(mbar, mphase, a.err, a.spin_limit)) return false;
                mphase ^= 1u;
                const int off = (anc.lo[l] + c0 - bbase) * B;
                smem_banks<B, S, Acc>(tilesC, Rc + 3 * (size_t)off, Zc + 3 * (size_t)off, ncb, xch);
            }
        }
    }
    __syncthreads();
    return true;
}

// One SpMV over this CTA's row range: stage the halo (MODE 1: p_new = z +
// beta p_old from src = z and pold; MODE 2: src = x; MODE 3: x + beta p from
// src = x and pold = p, y = rhs - A (x + beta p)) in shared memory, then
// the CTA's work units round-robin over its warps (descriptors cached in
// shared memory, ud_sm, the first a.upw per warp).
template <int MODE>
__device__ __forceinline__ double spmv_cta(const PArgs& a, int4 ci, const int4* ud_sm, double* hv,
                                           const int* hidx, const double* src, const double* pold, double beta,
                                           double* pnew, double* y, const double* rhs) {
    // two halo vertices per thread and pass: all their loads in flight at once
    for (int h = threadIdx.x; h < ci.z; h += 2 * kPT) {
        const int h2 = h + kPT;
        const bool two = h2 < ci.z;
        const int v = hidx[h], v2 = two ? hidx[h2] : v;
        double s0[6], q[6];
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            s0[d] = ldv<true>(src + 3 * (size_t)v + d);
            s0[3 + d] = ldv<true>(src + 3 * (size_t)v2 + d);
            if (MODE == 1 || MODE == 3) {
                q[d] = ldv<true>(pold + 3 * (size_t)v + d);
                q[3 + d] = ldv<true>(pold + 3 * (size_t)v2 + d);
            }
        }
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (MODE == 1 && a.pv.bodies) {  // z = MAS part + the patches' parts
                s0[d] += patch_z(a.pv, v, d);
                s0[3 + d] += patch_z(a.pv, v2, d);
            }
            hv[3 * h + d] = MODE != 2 ? __fma_rn(beta, q[d], s0[d]) : s0[d];
            if (two) hv[3 * h2 + d] = MODE != 2 ? __fma_rn(beta, q[3 + d], s0[3 + d]) : s0[3 + d];
        }
    }
    __syncthreads();
    double dot = 0.0;
    const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
    const int4* ud = ud_sm + w * a.upw * kRowGroups + lane / kRowLanes;
    for (int u = w, i = 0; u < ci.x; u += kPT / 32, ++i) {
        const int4 d = i < a.upw ? ud[kRowGroups * i] : a.udesc_c[(size_t)(ci.w + u) * kRowGroups + lane / kRowLanes];
        dot += spmv_unit_h<MODE == 3 ? 2 : MODE>(a.A, d, lane, a.lcols, hv, pnew, y, rhs);
    }
    return dot;
}

// storage of the body patches for each MAS storage: factored W in FP32, or
// in FP64 with the FP64 MAS (BF16 rounding of W loses the stiff contact
// directions the patches exist for: measured, it did not converge)
template <typename S> struct PatchS { using T = Fact<float>; };
template <> struct PatchS<double> { using T = double; };

// TG: some level-0 / level-1 tiles are read from global memory (a.t0g, a.t1g)
template <int B, typename S, typename Acc, bool TG>
__global__ void __launch_bounds__(kPT, 1) k_pcg_persistent(PArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t mbar;
    __shared__ double sh[32];
    __shared__ __align__(16) Acc xch[(kPT / 32) * kXchPerWarp];
    constexpr int bs = bsym_of(B);
    constexpr int HPW = 32 / B;
    const size_t tb = (size_t)bs * 9;  // elements per tile
    const bool mas = a.precond == 1;
    // shared memory: tiles0 [k0] | tiles1 [k1] | tilesC [capc] | R1s, Z1s [k1 B 3] | Rc, Zc [nc 3] | parc [nc]
    S* tiles0 = reinterpret_cast<S*>(smem_raw);
    S* tiles1 = tiles0 + (size_t)(a.t0g ? 0 : a.k0) * tb;
    S* tilesC = tiles1 + (size_t)(a.t1g ? 0 : a.k1) * tb;
    Acc* R1s = reinterpret_cast<Acc*>(tilesC + (size_t)a.capc * tb);
    __shared__ Anc anc;
    __shared__ int rng[2];
    __shared__ unsigned short ctab[(kMaxLevels - 2) * kPT];  // a.nc <= 65535 (host check)
    Acc* Z1s = R1s + 3 * (size_t)a.k1 * B;
    Acc* Rc = Z1s + 3 * (size_t)a.k1 * B;
    Acc* Zc = Rc + 3 * (size_t)a.nc;
    int* parc = reinterpret_cast<int*>(Zc + 3 * (size_t)a.nc);
    // SpMV unit descriptors: [warp][unit of the warp][lane group of 8]
    int4* udesc = reinterpret_cast<int4*>(smem_raw + (((size_t)(reinterpret_cast<unsigned char*>(parc + a.nc) -
                                                                smem_raw) + 15) & ~(size_t)15));
    // staged halo of the SpMV: 3 doubles per halo vertex
    double* hv = reinterpret_cast<double*>(udesc + (size_t)(kPT / 32) * a.upw * kRowGroups);
    // the halo's vertex ids (fixed for the solve)
    int* hidx = reinterpret_cast<int*>(hv + 3 * (size_t)a.hcap);
    // body-patch scratch: the patch's r and y (12 + 3 kPatchMax each)
    Acc* prl = reinterpret_cast<Acc*>(reinterpret_cast<unsigned char*>(hidx) + ((4 * (size_t)a.hcap + 15) & ~(size_t)15));
    Acc* pyl = prl + 12 + 3 * kPatchMax;
    const int4 ci = a.cinfo[blockIdx.x];
    if (a.stamps && blockIdx.x == 0 && threadIdx.x == 0) a.stamps[0] = clock64();
    unsigned epoch = 0u, mphase = 0u;
    double* part_pap = a.partials;
    double* part_rz = a.partials + gridDim.x;
    double* part_rr = a.partials + 2 * gridDim.x;
    const int lane = threadIdx.x % B, hw = threadIdx.x / B;
    bool ok = true;

    // ---- ownership, per-thread constants, cached tiles ----------------------
    Own o = {0, 0, 0, 0};
    int v = -1, n1loc = -1, par1 = -1;
    // level-1 bank of this half-warp: the level-1 banks go to the CTA's last
    // warps (hw1 = hw - base1), which have no level-0 bank unless the CTA has
    // nearly 32 of them, so the level-1 products run beside the level-0 ones
    int hw1 = -1;
    int vo = 0;  // 3 * (global row of vertex v)
    unsigned msk = 0u;
    bool own = false;
    if (mas) {
        o = own_ranges<B>(a);
        const int b1 = a.lvl_begin[1] / B;
        if (threadIdx.x == 0) { mbar_init(&mbar, 1); fence_mbar_init(); }
        for (int i = threadIdx.x; i < 3 * a.k1 * B; i += kPT) { R1s[i] = (Acc)0; Z1s[i] = (Acc)0; }
        for (int i = threadIdx.x; i < 3 * a.nc; i += kPT) { Rc[i] = (Acc)0; Zc[i] = (Acc)0; }
        for (int i = threadIdx.x; i < a.nc; i += kPT) {  // parents of the nodes of levels 2 .. L-2
            const int node = a.lvl_begin[2] + i;
            int par = -1;
            for (int l = 2; l + 1 < a.L; ++l)
                if (node >= a.lvl_begin[l] && node < a.lvl_begin[l] + a.lvl_count[l])
                    par = a.going_next[node] - a.lvl_begin[2];
            parc[i] = par;
        }
        // ancestor bank ranges, level by level (parents of the previous range)
        if (threadIdx.x == 0) {
            anc.total = 0;
            for (int l = 0; l < kMaxLevels + 2; ++l) { anc.lo[l] = 0; anc.nb[l] = 0; }
        }
        int lo_n = a.lvl_begin[1] + o.j0 * B, hi_n = min(a.lvl_begin[1] + (o.j0 + o.nbk1) * B,
                                                         a.lvl_begin[1] + a.lvl_count[1]) - 1;
        for (int l = 2; l < a.L && lo_n <= hi_n; ++l) {
            if (threadIdx.x == 0) { rng[0] = 0x7fffffff; rng[1] = -1; }
            __syncthreads();
            int mn = 0x7fffffff, mx = -1;
            for (int n = lo_n + (int)threadIdx.x; n <= hi_n; n += kPT) {
                const int par = a.going_next[n];
                mn = min(mn, par);
                mx = max(mx, par);
            }
            if (mx >= 0) { atomicMin(&rng[0], mn); atomicMax(&rng[1], mx); }
            __syncthreads();
            lo_n = rng[0];
            hi_n = rng[1];
            if (threadIdx.x == 0 && lo_n <= hi_n) {
                anc.lo[l] = lo_n / B;
                anc.nb[l] = hi_n / B - lo_n / B + 1;
                anc.total += anc.nb[l];
            }
            __syncthreads();
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned by0 = a.t0g ? 0u : (unsigned)(o.nbk0 * tb * sizeof(S));
            const unsigned by1 = a.t1g ? 0u : (unsigned)(o.nbk1 * tb * sizeof(S));
            const bool cache_c = anc.total <= a.capc;
            const unsigned byc = cache_c ? (unsigned)(anc.total * tb * sizeof(S)) : 0u;
            mbar_expect_tx(&mbar, by0 + by1 + byc);
            if (by0) bulk_g2s(tiles0, (const S*)a.inv + (size_t)o.lo * tb, by0, &mbar);
            if (by1) bulk_g2s(tiles1, (const S*)a.inv + (size_t)(b1 + o.j0) * tb, by1, &mbar);
            if (byc) {
                int t = 0;
                for (int l = 2; l < a.L; ++l) {
                    if (anc.nb[l] == 0) continue;
                    bulk_g2s(tilesC + (size_t)t * tb, (const S*)a.inv + (size_t)anc.lo[l] * tb,
                             (unsigned)(anc.nb[l] * tb * sizeof(S)), &mbar);
                    t += anc.nb[l];
                }
            }
        }
        if (hw < o.nbk0) v = a.part_map[(o.lo + hw) * B + lane];
        if (v >= 0) {
            vo = 3 * (a.ex.fem_off + v);
            msk = a.fine_mask[v];
            if (a.L >= 2) {
                const int n1 = a.going_next[v] - a.lvl_begin[1];
                n1loc = n1 - o.j0 * B;
                own = n1loc >= 0 && n1loc < o.nbk1 * B;
            } else {
                own = true;
            }
        }
        if (own)  // coarse nodes of the slot's vertex at levels >= 2 (fixed for the solve)
            for (int l = 2; l < a.L; ++l)
                ctab[(l - 2) * kPT + threadIdx.x] =
                    (unsigned short)(a.coarse_table[(size_t)kMaxLevels * v + l - 1] - a.lvl_begin[2]);
        hw1 = TG ? hw : hw - (kPT / B - ((o.nbk1 + HPW - 1) / HPW) * HPW);
        if (a.L > 2 && hw1 >= 0 && hw1 < o.nbk1) {
            const int i1 = (o.j0 + hw1) * B + lane;
            if (i1 < a.lvl_count[1]) par1 = a.going_next[a.lvl_begin[1] + i1] - a.lvl_begin[2];
        }
        ok = mbar_wait(&mbar, mphase, a.err, a.spin_limit);
        mphase ^= 1u;
    }
    const bool act0 = (hw / HPW) * HPW < o.nbk0;  // this warp has level-0 work
    // level-1 work: the last warps, or (tiles in global memory, where the
    // level-0 products are memory-bound) the first warps after the level-0 products
    const bool act1 = TG ? (hw / HPW) * HPW < o.nbk1
                         : o.nbk1 > 0 && (hw / HPW) * HPW >= kPT / B - ((o.nbk1 + HPW - 1) / HPW) * HPW;

    // ---- MAS pieces on the registers of this thread's slot ----------------
    // the slot's x lives in shared memory (touched once per iteration), which
    // leaves its registers to the SpMV (measured: FP64 tiles 44.4 -> 42.3 us
    // per iteration, BF16 28.1 -> 28.0 on the contact benchmark)
    __shared__ double xsh[3 * kPT];
    double& x0 = xsh[3 * threadIdx.x];
    double& x1 = xsh[3 * threadIdx.x + 1];
    double& x2 = xsh[3 * threadIdx.x + 2];
    x0 = 0.0; x1 = 0.0; x2 = 0.0;
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    Acc zl0 = 0, zl1 = 0, zl2 = 0;  // level-0 Schwarz of the slot
    // level-1 warps of this CTA (act1): the first of them and their count
    const int n1w = min(kPT / 32, (o.nbk1 + HPW - 1) / HPW);
    const int w1first = TG ? 0 : kPT / 32 - n1w;
    // level-0 (+ level-1) part of the apply on r (registers).  arrive: this
    // CTA arrives at the next grid barrier as soon as what other CTAs read
    // after it is written (the level-2 residual pushes, or r for the body
    // patches), so the Schwarz products run while the other CTAs catch up
    auto apply_b = [&](bool arrive) {
        // level-0 tiles: shared memory, or global memory when they did not fit
        const S* t0 = TG && a.t0g ? (const S*)a.inv + (size_t)o.lo * tb : tiles0;
        if (act0) {  // the slot's r into the bank exchange, level-0 component sums -> level-1 residuals
            Acc* xb = bank_slot<B>(xch);
            xch_put(xb, lane, (Acc)r0, (Acc)r1, (Acc)r2);
            Acc s0, s1, s2;
            mask_sum<B, Acc>(msk, xb, s0, s1, s2);
            if (own && a.L >= 2 && __popc(msk & lanemask_lt(lane)) == 0) {
                R1s[3 * n1loc] = s0; R1s[3 * n1loc + 1] = s1; R1s[3 * n1loc + 2] = s2;
            }
        }
        if (TG || a.L < 2) {
            if (act0) schwarz_rows<B, S, Acc>(t0 + (size_t)(hw < o.nbk0 ? hw : 0) * tb, lane, bank_slot<B>(xch), zl0, zl1, zl2);
            if (a.L < 2) {
                if (arrive) {
                    __syncthreads();
                    if (threadIdx.x == 0) grid_arrive(a.sync);
                }
                return;
            }
        }
        __syncthreads();  // level-1 residuals complete
        const bool push_arrive = arrive && a.L > 2 && n1w > 0;  // else thread 0 arrives here
        if (arrive && !push_arrive && threadIdx.x == 0) grid_arrive(a.sync);
        if (!TG && act0)  // level-0 Schwarz on r (still in the bank exchange)
            schwarz_rows<B, S, Acc>(t0 + (size_t)(hw < o.nbk0 ? hw : 0) * tb, lane, bank_slot<B>(xch), zl0, zl1, zl2);
        if (act1) {  // level-1 banks of this CTA: push to level 2, Schwarz
            const bool valid = hw1 >= 0 && hw1 < o.nbk1;
            const int i = (valid ? hw1 : 0) * B + lane;
            const Acc v0 = valid ? R1s[3 * i] : (Acc)0, v1 = valid ? R1s[3 * i + 1] : (Acc)0,
                      v2 = valid ? R1s[3 * i + 2] : (Acc)0;
            Acc* xb = bank_slot<B>(xch);
            xch_put(xb, lane, v0, v1, v2);
            if (a.L > 2) {
                Acc s0, s1, s2;
                bool lead;
                group_sum<B, Acc>(par1, xb, lane, s0, s1, s2, lead);
                if (lead) {
                    Acc* Rg = (Acc*)a.R + 3 * (size_t)(a.lvl_begin[2] + par1);
                    Rg[0] = s0; Rg[1] = s1; Rg[2] = s2;
                }
            }
            if (push_arrive) {  // the level-1 warps' pushes are complete: arrive
                asm volatile("bar.sync 1, %0;" ::"r"(32 * n1w) : "memory");
                if (threadIdx.x == 32 * w1first) grid_arrive(a.sync);
            }
            Acc z0, z1, z2;
            const S* t1 = TG && a.t1g ? (const S*)a.inv + (size_t)(a.lvl_begin[1] / B + o.j0) * tb : tiles1;
            schwarz_rows<B, S, Acc>(t1 + (size_t)(valid ? hw1 : 0) * tb, lane, xb, z0, z1, z2);
            if (valid) { Z1s[3 * i] = z0; Z1s[3 * i + 1] = z1; Z1s[3 * i + 2] = z2; }
        }
        __syncthreads();
    };
    // CollectFinalZ for the owned slot + r.z, r.r partials
    auto collect = [&](int mode, double alpha, const double* pcur, bool write_x) {
        double rz = 0.0, rr = 0.0;
        extra_rows_work(a.ex, a.N, mode, alpha, a.x, a.r, pcur, a.Ap, a.z, blockIdx.x * (kPT / 32) + threadIdx.x / 32,
                        gridDim.x * (kPT / 32), threadIdx.x & 31, rz, rr);
        if (own) {
            Acc c0 = zl0, c1 = zl1, c2 = zl2;
            if (a.L >= 2) { c0 += Z1s[3 * n1loc]; c1 += Z1s[3 * n1loc + 1]; c2 += Z1s[3 * n1loc + 2]; }
            for (int l = 2; l < a.L; ++l) {
                const int n = ctab[(l - 2) * kPT + threadIdx.x];
                c0 += Zc[3 * n]; c1 += Zc[3 * n + 1]; c2 += Zc[3 * n + 2];
            }
            const double z0 = (double)c0, z1 = (double)c1, z2 = (double)c2;
            a.z[vo] = z0; a.z[vo + 1] = z1; a.z[vo + 2] = z2;
            if (write_x) { a.x[vo] = x0; a.x[vo + 1] = x1; a.x[vo + 2] = x2; }  // the next refresh stages it
            rz += r0 * z0 + r1 * z1 + r2 * z2;
            rr += r0 * r0 + r1 * r1 + r2 * r2;
        }
        // body patches (r complete in global memory: stored in phase B, a grid barrier since)
        for (int pb = blockIdx.x; pb < a.pv.bodies; pb += gridDim.x)
            patch_apply_cta<typename PatchS<S>::T, Acc>(a.pv, pb, a.ex.fem_off, a.r, a.z, prl, pyl, rz, rr);
        block_sum2(rz, rr, sh);
        if (threadIdx.x == 0) { part_rz[blockIdx.x] = rz; part_rr[blockIdx.x] = rr; }
    };

    // ---- SpMV unit descriptors of this CTA's warps (fixed for the solve)
    {
        const int w = threadIdx.x / 32, lane32 = threadIdx.x & 31;
        for (int i = 0; i < a.upw; ++i) {
            const int u = w + i * (kPT / 32);
            int4 d = {-1, 0, 0, 0};
            if (u < ci.x) d = a.udesc_c[(size_t)(ci.w + u) * kRowGroups + lane32 / kRowLanes];
            if (lane32 % kRowLanes == 0) udesc[(w * a.upw + i) * kRowGroups + lane32 / kRowLanes] = d;
        }
        for (int h = threadIdx.x; h < ci.z; h += kPT) hidx[h] = a.halo[ci.y + h];
        __syncthreads();
    }
    // ---- prologue: x = 0, r = b, p_old = 0, z = M^-1 r, r.z, r.r
    for (int i = blockIdx.x * kPT + threadIdx.x; i < 3 * a.nrows; i += gridDim.x * kPT) {
        a.p0[i] = 0.0;
        if (!a.warm && (!mas || a.ex.n_units > 0)) { a.x[i] = 0.0; a.r[i] = a.b[i]; }
    }
    // start guess x0 (in x): Ap = A x0 with x0.A x0 (the SpMV with p = x0,
    // beta = 0, p written to p1 as scratch), x0.b, b.b; then alpha = x0.b /
    // x0.A x0 (0 unless positive), r = b - alpha A x0, x = alpha x0, r.r; a
    // guess that raises ||r|| above ||b|| is rejected (x = 0, r = b).  All
    // CTAs sum the same partials, so all take the same branch.
    double w_bb = 0.0;
    if (a.warm) {
        double w_alpha = 0.0, w_rr = 0.0;
        double* part_w = a.partials + 3 * gridDim.x;
        double xax = 0.0, xb = 0.0, bb = 0.0;
        __syncthreads();  // the descriptor cache is complete
        xax = spmv_cta<1>(a, ci, udesc, hv, hidx, a.x, a.x, 0.0, a.p1, a.Ap, nullptr);  // p = x0 (beta 0)
        for (int i = blockIdx.x * kPT + threadIdx.x; i < 3 * a.nrows; i += gridDim.x * kPT) {
            const double bi = a.b[i];
            xb += a.x[i] * bi;
            bb += bi * bi;
        }
        xax = block_sum<kPT>(xax, sh);
        xb = block_sum<kPT>(xb, sh);
        bb = block_sum<kPT>(bb, sh);
        if (threadIdx.x == 0) { part_pap[blockIdx.x] = xax; part_rz[blockIdx.x] = xb; part_rr[blockIdx.x] = bb; }
        ok = ok && grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom);
        if (ok) {
            xax = sum_partials(part_pap);
            sum_partials2(part_rz, part_rr, xb, bb);
            w_bb = bb;
            w_alpha = (xax > 0.0 && xb > 0.0) ? xb / xax : 0.0;
            double rr = 0.0;
            for (int i = blockIdx.x * kPT + threadIdx.x; i < 3 * a.nrows; i += gridDim.x * kPT) {
                const double ri = a.b[i] - w_alpha * a.Ap[i];
                a.r[i] = ri;
                a.x[i] = w_alpha * a.x[i];
                rr += ri * ri;
            }
            rr = block_sum<kPT>(rr, sh);
            if (threadIdx.x == 0) part_w[blockIdx.x] = rr;
        }
        ok = ok && grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom);
        if (ok) {
            w_rr = sum_partials(part_w);
            const int w_rej = !(w_rr <= w_bb) || w_alpha == 0.0;
            if (blockIdx.x == 0 && threadIdx.x == 0) {  // read back by the same thread at the end
                a.st->w_alpha = w_alpha; a.st->w_rr = w_rr; a.st->w_reject = w_rej;
            }
            if (w_rej) {
                for (int i = blockIdx.x * kPT + threadIdx.x; i < 3 * a.nrows; i += gridDim.x * kPT) {
                    a.r[i] = a.b[i];
                    a.x[i] = 0.0;
                }
                ok = grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom);
            }
        }
    }
    if (mas) {
        if (v >= 0) {
            const double* r_in = a.warm ? a.r : a.b;
            r0 = r_in[vo]; r1 = r_in[vo + 1]; r2 = r_in[vo + 2];
            if (a.warm && own) { x0 = a.x[vo]; x1 = a.x[vo + 1]; x2 = a.x[vo + 2]; }
        }
        const bool need = a.L > 2 || a.pv.bodies;  // (the patches read r of other CTAs' rows)
        if (ok) apply_b(need);
        if (need) {
            ok = ok && grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom, nullptr, nullptr, false);
            if (ok && a.L > 2) ok = levels_c<B, S, Acc>(a, anc, tilesC, Rc, Zc, parc, &mbar, mphase, xch);
        }
        if (ok) collect(0, 0.0, a.p1, false);
    } else {
        ok = ok && grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom);
        if (ok) phase_jacobi(a, 0, 0.0, a.p1, part_rz, part_rr, sh);
    }
    ok = ok && grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom);
    double rz = ok ? sum_partials(part_rz) : 0.0;
    const double rz0 = rz;
    const double rr0_r = ok ? sum_partials(part_rr) : 0.0;
    const double rr0 = a.warm ? w_bb : rr0_r;  // a start guess: convergence relative to ||b||
    double rr_last = rr0_r, beta = 0.0;
    int k = 1, iters = 1, converged = 0, breakdown = 0;
    bool done = !ok || a.max_iter <= 1;
    double* pold = a.p0;
    double* pnew = a.p1;
    unsigned long long* acc = a.stamps ? a.stamps + 8 * (size_t)(a.stamp_iters + 2) + 16 * (size_t)blockIdx.x : nullptr;
    long long t_rel = clock64();
#define SLOT(i) (acc ? acc + 2 * (i) : nullptr), &t_rel
    int passes = 0;
    while (!done) {
        ++passes;
        // A: p_new = z + beta p_old, Ap = A p_new, p.Ap
        stamp(a, k, 0);
        double dot = spmv_cta<1>(a, ci, udesc, hv, hidx, a.z, pold, beta, pnew, a.Ap, nullptr);
        dot = block_sum<kPT>(dot, sh);
        if (threadIdx.x == 0) part_pap[blockIdx.x] = dot;
        if (!grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom, SLOT(0))) { ok = false; break; }
        stamp(a, k, 1);
        const bool refresh = k % 10 == 0;  // true residual (pcg_solver.cu:240-244)
        // B: the slot's p and Ap are loaded before the partials are summed
        double p0v = 0.0, p1v = 0.0, p2v = 0.0, q0 = 0.0, q1 = 0.0, q2 = 0.0;
        if (mas && v >= 0) {
            if (own) { p0v = pnew[vo]; p1v = pnew[vo + 1]; p2v = pnew[vo + 2]; }
            if (!refresh) { q0 = a.Ap[vo]; q1 = a.Ap[vo + 1]; q2 = a.Ap[vo + 2]; }
        }
        const double pap = sum_partials(part_pap);
        if (!(pap > 0.0)) {  // same value in every CTA: all stop here
            // finite p.Ap <= 0: CG breakdown (r = 0 exactly is a solution); NaN: reported as non-finite
            const bool finite = pap == pap && rz == rz;
            breakdown = finite && rz != 0.0;
            converged = finite && rz == 0.0;
            iters = k;
            break;
        }
        const double alpha = rz / pap;
        if (refresh) {
            // r = b - A x_new with x_new = x + alpha p formed in the halo staging from x in global
            // memory (the previous iteration's, written by the collect), so no grid barrier is
            // needed between the x update and the SpMV; the slot's own x is updated with the same
            // fused multiply-add
            if (mas && own) {
                x0 = __fma_rn(alpha, p0v, x0); x1 = __fma_rn(alpha, p1v, x1); x2 = __fma_rn(alpha, p2v, x2);
            }
            spmv_cta<3>(a, ci, udesc, hv, hidx, a.x, pnew, alpha, nullptr, a.r, a.b);
            if (!grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom, SLOT(2))) { ok = false; break; }
            // rows kept in global memory only (outside the MAS range; every row without MAS): x +=
            // alpha p once every CTA's staging has read the old x
            if (mas) {
                const int lo_n = 3 * a.ex.fem_off, hi_n = 3 * (a.ex.fem_off + a.N);
                for (int i = blockIdx.x * kPT + threadIdx.x; i < 3 * a.nrows - (hi_n - lo_n); i += gridDim.x * kPT) {
                    const int e = i < lo_n ? i : i + (hi_n - lo_n);
                    a.x[e] = __fma_rn(alpha, pnew[e], a.x[e]);
                }
            } else {
                for (int i = blockIdx.x * kPT + threadIdx.x; i < 3 * a.nrows; i += gridDim.x * kPT)
                    a.x[i] = __fma_rn(alpha, pnew[i], a.x[i]);
            }
            if (mas && v >= 0) { r0 = a.r[vo]; r1 = a.r[vo + 1]; r2 = a.r[vo + 2]; }
        } else {
            if (mas && v >= 0) {
                r0 = r0 - alpha * q0; r1 = r1 - alpha * q1; r2 = r2 - alpha * q2;
                if (own) {
                    x0 = __fma_rn(alpha, p0v, x0); x1 = __fma_rn(alpha, p1v, x1); x2 = __fma_rn(alpha, p2v, x2);
                }
                if (own && a.pv.bodies) { a.r[vo] = r0; a.r[vo + 1] = r1; a.r[vo + 2] = r2; }
            }
            // body rows with patches: updated here, before the patches read them in phase C
            for (int i = blockIdx.x * kPT + threadIdx.x; i < 12 * a.pv.bodies; i += gridDim.x * kPT) {
                a.x[i] = a.x[i] + alpha * pnew[i];
                a.r[i] = a.r[i] - alpha * a.Ap[i];
            }
        }
        stamp(a, k, 2);
        if (mas) {
            apply_b(a.L > 2 || a.pv.bodies);
            if (a.L > 2 || a.pv.bodies) {
                if (!grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom, SLOT(3), false)) { ok = false; break; }
                stamp(a, k, 3);
                if (a.L > 2 && !levels_c<B, S, Acc>(a, anc, tilesC, Rc, Zc, parc, &mbar, mphase, xch)) ok = false;
            }
            collect(refresh ? 0 : 1, alpha, pnew, k % 10 == 9);
        } else {
            phase_jacobi(a, refresh ? 0 : 1, alpha, pnew, part_rz, part_rr, sh);
        }
        if (!grid_barrier(a.sync, epoch, a.err, a.spin_limit, a.phantom, SLOT(5)) || !ok) { ok = false; break; }
        stamp(a, k, 5);
        double rz_new, rr;
        sum_partials2(part_rz, part_rr, rz_new, rr);
        bool conv = false;
        if (k % a.check_every == 0) {
            rr_last = rr;
            conv = a.use_prec_norm ? (rz_new <= a.rel2 * rz0 || rz_new <= a.abs2)
                                   : (rr <= a.rel2 * rr0 || rr <= a.abs2);
            if (!(rz_new == rz_new) || !(rr == rr)) { conv = true; ok = false; }
        }
        if (conv) {
            iters = k;
            converged = ok ? 1 : 0;
            done = true;
        } else {
            beta = rz_new / rz;
            rz = rz_new;
            ++k;
            iters = k;
            if (k >= a.max_iter) done = true;
            double* t = pold; pold = pnew; pnew = t;
        }
    }
#undef SLOT
    if (mas && own) {
        a.x[vo] = x0; a.x[vo + 1] = x1; a.x[vo + 2] = x2;
        a.r[vo] = r0; a.r[vo + 1] = r1; a.r[vo + 2] = r2;
        if (a.pv.bodies)  // the last z with its patch part (the loop ended after a grid barrier)
            for (int d = 0; d < 3; ++d) a.z[vo + d] += patch_z(a.pv, vo / 3, d);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        PcgState s = {};
        s.rz = rz; s.rz0 = rz0; s.rr0 = rr0; s.rr = rr_last; s.k = k; s.iters = iters; s.done = 1;
        s.converged = converged;
        s.breakdown = breakdown;
        s.max_iter = a.max_iter;
        s.check_every = a.check_every;
        s.warm = a.warm;
        if (a.warm) { s.w_alpha = a.st->w_alpha; s.w_rr = a.st->w_rr; s.w_reject = a.st->w_reject; s.w_bb = rr0; }
        *a.st = s;
        if (a.stamps) {
            a.stamps[1] = clock64();
            a.stamps[2] = (unsigned long long)passes;
        }
    }
}

// ---- SpMV plan of the persistent loop (once per solve) ----------------------
// CTA c takes a contiguous range of block rows in partition order (the MAS
// rows in slot order, so a range is a compact piece of the mesh), balanced by
// stored blocks plus a per-row cost.  Its halo is every column its rows touch;
// the rows' column indices are rewritten as halo indices (lcols), so the SpMV
// gathers from shared memory.  Work units inside the range as the graph form
// makes them: a long row (more than kLongRowP blocks) per warp, else four
// short rows of 8 lanes each.
constexpr int kLongRowP = 32;
constexpr int kRowCost = 4;

// row order (one CTA of 1024 threads): rows [0, fem_off) and [fem_off + N,
// nrows) in place, the MAS rows by slot
__global__ void __launch_bounds__(1024) k_row_order(int nrows, int mas, int fem_off, int N, int Mm,
                                                    const int* __restrict__ part_map, int* row_order) {
    __shared__ int sh[64];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    if (!mas) {
        for (int i = threadIdx.x; i < nrows; i += 1024) row_order[i] = i;
        return;
    }
    for (int i = threadIdx.x; i < fem_off; i += 1024) row_order[i] = i;
    for (int i = fem_off + N + threadIdx.x; i < nrows; i += 1024) row_order[i] = i;
    for (int base = 0; base < Mm; base += 1024) {
        const int s = base + threadIdx.x;
        const int v = s < Mm ? part_map[s] : -1;
        int tot;
        const int pre = block_scan1024(v >= 0, sh, &tot);
        if (v >= 0) row_order[fem_off + carry + pre] = fem_off + v;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

// stored blocks of the row at each position of the order (into cpre, scratch)
__global__ void k_order_len(int nrows, const int* __restrict__ row_order, const int* __restrict__ row_ptr,
                            int* len_at) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const int r = row_order[i];
    len_at[i] = row_ptr[r + 1] - row_ptr[r];
}

// prefix sums along the order (one CTA of 1024 threads, a contiguous chunk
// per thread): cpre of the balance cost (blocks + kRowCost per row), epre of
// max(blocks, 1) (room in the halo lists: a row is in its own halo); cpre
// holds the row lengths on entry, each thread reads its chunk before writing it
__global__ void __launch_bounds__(1024) k_order_prefix(int nrows, int* cpre, int* epre) {
    __shared__ int sh[64];
    const int chunk = (nrows + 1023) / 1024;
    const int b0 = min(nrows, (int)threadIdx.x * chunk), b1 = min(nrows, b0 + chunk);
    int cs = 0, es = 0;
    for (int i = b0; i < b1; ++i) {
        const int len = cpre[i];
        cs += len + kRowCost;
        es += max(len, 1);
    }
    int ct, et;
    const int cp = block_scan1024(cs, sh, &ct);
    const int ep = block_scan1024(es, sh, &et);
    cs = cp;
    es = ep;
    for (int i = b0; i < b1; ++i) {
        const int len = cpre[i];
        cpre[i] = cs;
        epre[i] = es;
        cs += len + kRowCost;
        es += max(len, 1);
    }
    if (threadIdx.x == 0) { cpre[nrows] = ct; epre[nrows] = et; }
}

__device__ __forceinline__ int range_begin(const int* cpre, int nrows, int c, int G) {
    const long long target = ((long long)cpre[nrows] * c + G - 1) / G;  // first i with cpre[i] >= c T / G
    int lo = 0, hi = nrows;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((long long)cpre[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    return c == 0 ? 0 : lo;
}

// one CTA (512 threads) per CTA of the persistent launch: its row range, halo
// (bitmap over all rows in shared memory, nrows bits + a word prefix),
// lcols, work units.  cinfo[c] = {units, halo offset, halo size, first unit};
// stats[0] = largest halo, stats[1] = most units of a CTA (atomicMax).
__global__ void __launch_bounds__(512) k_spmv_plan(int nrows, const int* __restrict__ row_order,
                                                   const int* __restrict__ cpre, const int* __restrict__ epre,
                                                   const int* __restrict__ row_ptr, const int* __restrict__ cols,
                                                   int* lcols, int* halo, int4* cinfo, int4* udesc, int* stats) {
    extern __shared__ unsigned bm[];  // [nw] bitmap, then [nw] exclusive word prefix (as int)
    __shared__ int sh[64];
    __shared__ int rng[2];
    __shared__ int nlong_sh, carry_l, carry_s;
    const int G = gridDim.x, c = blockIdx.x;
    const int nw = (nrows + 31) >> 5;
    int* wpre = reinterpret_cast<int*>(bm + nw);
    if (threadIdx.x == 0) {
        rng[0] = range_begin(cpre, nrows, c, G);
        rng[1] = c + 1 == G ? nrows : range_begin(cpre, nrows, c + 1, G);
        carry_l = 0;
        carry_s = 0;
    }
    for (int w = threadIdx.x; w < nw; w += 512) bm[w] = 0u;
    __syncthreads();
    const int lo = rng[0], hi = rng[1];
    const int hoff = epre[lo];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = lo + warp; i < hi; i += 16) {  // mark the range's rows and the columns they touch
        const int r = row_order[i];
        if (lane == 0) atomicOr(bm + (r >> 5), 1u << (r & 31));
        for (int p = row_ptr[r] + lane; p < row_ptr[r + 1]; p += 32) {
            const int col = cols[p];
            atomicOr(bm + (col >> 5), 1u << (col & 31));
        }
    }
    __syncthreads();
    // word prefix of the bit counts: a contiguous chunk of words per thread
    const int chunk = (nw + 511) / 512;
    const int w0 = min(nw, (int)threadIdx.x * chunk), w1 = min(nw, w0 + chunk);
    int cnt = 0;
    for (int w = w0; w < w1; ++w) cnt += __popc(bm[w]);
    // block scan of 512 values with the 1024-thread helper's pattern
    int x = cnt;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int y = lane < 16 ? sh[lane] : 0;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += t;
        }
        sh[32 + lane] = y;
    }
    __syncthreads();
    int pre = (warp ? sh[32 + warp - 1] : 0) + x - cnt;
    const int H = sh[32 + 15];
    for (int w = w0; w < w1; ++w) {
        wpre[w] = pre;
        pre += __popc(bm[w]);
    }
    __syncthreads();
    // halo list: vertex of each halo index
    for (int w = threadIdx.x; w < nw; w += 512) {
        unsigned m = bm[w];
        int k = wpre[w];
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1u;
            halo[hoff + k++] = 32 * w + b;
        }
    }
    auto local = [&](int col) { return wpre[col >> 5] + __popc(bm[col >> 5] & ((1u << (col & 31)) - 1u)); };
    for (int i = lo + warp; i < hi; i += 16) {  // halo-local column indices
        const int r = row_order[i];
        for (int p = row_ptr[r] + lane; p < row_ptr[r + 1]; p += 32) lcols[p] = local(cols[p]);
    }
    // work units: the range's long rows first (one unit each), then its short rows, four per unit
    if (threadIdx.x == 0) nlong_sh = 0;
    __syncthreads();
    {
        int nl = 0;
        for (int i = lo + (int)threadIdx.x; i < hi; i += 512) {
            const int r = row_order[i];
            nl += (row_ptr[r + 1] - row_ptr[r]) > kLongRowP;
        }
        if (nl) atomicAdd(&nlong_sh, nl);
    }
    __syncthreads();
    const int nl = nlong_sh;
    for (int base = lo; base < hi; base += 512) {
        const int i = base + threadIdx.x;
        int r = -1, len = 0;
        if (i < hi) {
            r = row_order[i];
            len = row_ptr[r + 1] - row_ptr[r];
        }
        const bool isl = i < hi && len > kLongRowP, iss = i < hi && !isl;
        const unsigned bl = __ballot_sync(0xffffffffu, isl), bs = __ballot_sync(0xffffffffu, iss);
        if (lane == 0) { sh[warp] = __popc(bl); sh[16 + warp] = __popc(bs); }
        __syncthreads();
        int offl = carry_l, offs = carry_s;
        for (int k = 0; k < warp; ++k) { offl += sh[k]; offs += sh[16 + k]; }
        const unsigned lt = (1u << lane) - 1u;
        if (isl) {
            const int u = offl + __popc(bl & lt);
            const int4 d = make_int4(r, row_ptr[r], row_ptr[r + 1], 1 | (local(r) << 1));
            #pragma unroll
            for (int g = 0; g < kRowGroups; ++g) udesc[(size_t)(lo + u) * kRowGroups + g] = d;
        } else if (iss) {
            const int sidx = offs + __popc(bs & lt);
            const int u = nl + sidx / kRowGroups, g = sidx % kRowGroups;
            udesc[(size_t)(lo + u) * kRowGroups + g] = make_int4(r, row_ptr[r], row_ptr[r + 1], local(r) << 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 0; k < 16; ++k) { carry_l += sh[k]; carry_s += sh[16 + k]; }
        }
        __syncthreads();
    }
    const int ns = carry_s;
    const int units = nl + (ns + kRowGroups - 1) / kRowGroups;
    if (threadIdx.x < kRowGroups && ns % kRowGroups && threadIdx.x >= ns % kRowGroups)  // empty groups of the last unit
        udesc[(size_t)(lo + units - 1) * kRowGroups + threadIdx.x] = make_int4(-1, 0, 0, 0);
    if (threadIdx.x == 0) {
        cinfo[c] = make_int4(units, hoff, H, lo);
        atomicMax(stats, H);
        atomicMax(stats + 1, units);
    }
}

// level-0 bank of every level-1 node (all slots of a component agree)
template <int B>
__global__ void k_l1_bank(int Mm, int l1_begin, const int* __restrict__ part_map, const int* __restrict__ going_next,
                          int* l1_bank) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= Mm) return;
    const int v = part_map[s];
    if (v >= 0) l1_bank[going_next[v] - l1_begin] = s / B;
}

template <int B, typename S, typename Acc>
int launch_t(sgmas_context* c, PArgs& a, float* ms) {
    int dev_sms = 0;
    SG_CUDA(c, cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device));
    constexpr int bs = bsym_of(B);
    const size_t tb = (size_t)bs * 9 * sizeof(S);
    int max_smem = 0;
    SG_CUDA(c, cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    cudaFuncAttributes fa;  // both instantiations have the same static shared memory
    SG_CUDA(c, cudaFuncGetAttributes(&fa, k_pcg_persistent<B, S, Acc, false>));
    const size_t budget = (size_t)max_smem - fa.sharedSizeBytes - 256;  // minus the kernel's static shared memory
    const int G = c->pcg_ctas > 0 ? std::min(dev_sms, c->pcg_ctas) : dev_sms;  // CTAs of this solve
    // SpMV plan: row order, CTA row ranges, halos, halo-local columns, work units
    int max_units = 0;
    {
        cudaStream_t s = c->stream;
        const int nrows = a.nrows;
        const long long cap = c->bsr.cap;
        if (ctx_alloc_grow(c, &c->d_row_order, &c->row_order_cap, nrows) ||
            ctx_alloc_grow(c, &c->d_cpre, &c->cpre_cap, 2 * (nrows + 1)) ||
            ctx_alloc_grow(c, &c->d_udesc_c, &c->udesc_c_cap, nrows * kRowGroups) ||
            ctx_alloc_grow(c, &c->d_lcols, &c->lcols_cap, (int)cap) ||
            ctx_alloc_grow(c, &c->d_halo, &c->halo_cap, (int)cap + nrows) ||
            ctx_alloc_grow(c, &c->d_cinfo, &c->cinfo_cap, G) ||
            ctx_alloc_grow(c, &c->d_plan_stats, &c->plan_stats_cap, 2))
            return SGMAS_ERR_CUDA;
        int* cpre = c->d_cpre;
        int* epre = c->d_cpre + nrows + 1;
        k_row_order<<<1, 1024, 0, s>>>(nrows, a.precond == 1, a.precond == 1 ? a.ex.fem_off : 0, a.N, a.Mm,
                                       a.part_map, c->d_row_order);
        k_order_len<<<(nrows + 255) / 256, 256, 0, s>>>(nrows, c->d_row_order, a.A.row_ptr, cpre);
        k_order_prefix<<<1, 1024, 0, s>>>(nrows, cpre, epre);
        SG_CUDA(c, cudaMemsetAsync(c->d_plan_stats, 0, 2 * sizeof(int), s));
        const size_t plan_smem = 2 * (size_t)((nrows + 31) / 32) * sizeof(unsigned);
        if (plan_smem + 1024 > (size_t)max_smem) return 1;  // (the kernel's static shared memory is < 1 KB)
        if (plan_smem > 48 * 1024)
            SG_CUDA(c, cudaFuncSetAttribute(k_spmv_plan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan_smem));
        k_spmv_plan<<<G, 512, plan_smem, s>>>(nrows, c->d_row_order, cpre, epre, a.A.row_ptr, a.A.cols, c->d_lcols,
                                              c->d_halo, c->d_cinfo, c->d_udesc_c, c->d_plan_stats);
        c->build_launches += 4;
        SG_CUDA(c, cudaGetLastError());
        int st[2] = {0, 0};  // largest halo, most units of a CTA
        SG_CUDA(c, cudaMemcpyAsync(st, c->d_plan_stats, sizeof(st), cudaMemcpyDeviceToHost, s));
        SG_CUDA(c, cudaStreamSynchronize(s));
        a.hcap = st[0];
        max_units = st[1];
        a.cinfo = c->d_cinfo;
        a.udesc_c = c->d_udesc_c;
        a.lcols = c->d_lcols;
        a.halo = c->d_halo;
    }
    // the staged halo comes first; the subdomain tiles share what is left
    const size_t hbytes = ((3 * sizeof(double) * (size_t)a.hcap + 15) & ~(size_t)15) +  // halo values, ids
                          ((4 * (size_t)a.hcap + 15) & ~(size_t)15);
    const size_t pbytes = a.pv.bodies ? 2 * (12 + 3 * kPatchMax) * sizeof(Acc) : 0;  // body-patch scratch
    if (hbytes + pbytes + 256 > budget) return 1;
    const size_t tbudget = budget - hbytes - pbytes;
    size_t smem = 0;
    if (a.precond == 1) {
        a.nb0 = a.Mm / B;
        if (a.L >= 2) {
            a.nb1 = (a.lvl_count[1] + B - 1) / B;
            if (ctx_alloc_grow(c, &c->d_l1_bank, &c->l1_bank_cap, a.lvl_count[1])) return SGMAS_ERR_CUDA;
            if (ctx_alloc_grow(c, &c->d_own1, &c->own1_cap, G + 1)) return SGMAS_ERR_CUDA;
            a.l1_bank = c->d_l1_bank;
            a.own1 = c->d_own1;
            k_l1_bank<B><<<(a.Mm + 255) / 256, 256, 0, c->stream>>>(a.Mm, a.lvl_begin[1], a.part_map, a.going_next,
                                                                 c->d_l1_bank);
            c->build_launches += 1;
            // level-0 span of every level-1 bank, then contiguous CTA ranges of level-1 banks whose
            // largest level-0 span is minimal (binary search on that span, greedy fill)
            std::vector<int> l1b(a.lvl_count[1]);
            SG_CUDA(c, cudaMemcpyAsync(l1b.data(), c->d_l1_bank, sizeof(int) * l1b.size(), cudaMemcpyDeviceToHost,
                                       c->stream));
            SG_CUDA(c, cudaStreamSynchronize(c->stream));
            const int cnt1 = a.lvl_count[1], nb1 = a.nb1;
            auto first0 = [&](int j) { return l1b[(size_t)j * B]; };
            auto last0 = [&](int j) { return l1b[std::min((size_t)j * B + B - 1, (size_t)cnt1 - 1)]; };
            auto groups_for = [&](int M, std::vector<int>* starts) {  // CTAs needed with span <= M
                int n = 0, j = 0;
                while (j < nb1) {
                    if (starts) starts->push_back(j);
                    const int lo = first0(j);
                    int e = j + 1;
                    while (e < nb1 && e - j < kPT / B && last0(e) - lo + 1 <= M) ++e;
                    j = e;
                    ++n;
                }
                return n;
            };
            int lo_m = 1, hi_m = std::max(1, last0(nb1 - 1) - first0(0) + 1);
            for (int j = 0; j < nb1; ++j) lo_m = std::max(lo_m, last0(j) - first0(j) + 1);
            while (lo_m < hi_m) {
                const int mid = (lo_m + hi_m) / 2;
                if (groups_for(mid, nullptr) <= G) hi_m = mid;
                else lo_m = mid + 1;
            }
            std::vector<int> starts;
            groups_for(lo_m, &starts);
            std::vector<int> own(G + 1, nb1);
            for (size_t g = 0; g < starts.size() && g < (size_t)G; ++g) own[g] = starts[g];
            a.k0 = 0;
            a.k1 = 0;
            for (int g = 0; g < G; ++g) {
                const int j0 = own[g], j1 = own[g + 1];
                if (j1 <= j0) continue;
                a.k1 = std::max(a.k1, j1 - j0);
                a.k0 = std::max(a.k0, last0(j1 - 1) - first0(j0) + 1);
            }
            SG_CUDA(c, cudaMemcpyAsync(c->d_own1, own.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice,
                                       c->stream));
            SG_CUDA(c, cudaStreamSynchronize(c->stream));  // own is a host temporary
        } else {
            a.nb1 = 0;
            a.k1 = 0;
            a.k0 = (a.nb0 + G - 1) / G;
        }
        a.nc = a.L > 2 ? a.total - a.lvl_begin[2] : 0;
        if (a.k0 > kPT / B || a.k1 > kPT / B) return 1;  // one slot per thread: use the graph form
        if (a.nc > 65535) return 1;                         // coarse indices are cached as 16 bits
        const size_t small = 2 * 3 * (size_t)a.k1 * B * sizeof(Acc) + 2 * 3 * (size_t)a.nc * sizeof(Acc) +
                             (size_t)a.nc * sizeof(int);
        // level-0 tiles stay in shared memory if anything does; level-1 tiles next
        a.t0g = a.t1g = 0;
        if (small + (size_t)(a.k0 + a.k1) * tb + (a.L > 2 ? tb : 0) > tbudget) a.t1g = 1;
        if (small + (size_t)a.k0 * tb + (a.L > 2 ? tb : 0) > tbudget) a.t0g = 1;
        const size_t fixed = small + (size_t)((a.t0g ? 0 : a.k0) + (a.t1g ? 0 : a.k1)) * tb;
        if (a.L > 2) {
            if (fixed + tb > tbudget) return 1;
            a.capc = (int)std::min<size_t>({(size_t)(a.nc / B), (size_t)(kPT / B), (tbudget - fixed) / tb});
        } else {
            if (fixed > tbudget) return 1;
            a.capc = 0;
        }
        smem = fixed + (size_t)a.capc * tb;
    } else {
        a.k0 = a.k1 = a.nb0 = a.nb1 = a.nc = a.capc = a.t0g = a.t1g = 0;
    }
    // the staged halo (3 doubles per vertex), then as many cached unit descriptors (16 B per warp,
    // unit and lane group) as fit, at most 16 units per warp
    {
        smem = (smem + 15) & ~(size_t)15;
        if (smem + hbytes > budget) return 1;
        const int per_warp = (max_units + kPT / 32 - 1) / (kPT / 32);
        const size_t per_unit = (size_t)(kPT / 32) * kRowGroups * sizeof(int4);
        if (smem + hbytes + pbytes > budget) return 1;
        const size_t room = (budget - smem - hbytes - pbytes) / per_unit;
        a.upw = (int)std::min<size_t>({(size_t)per_warp, (size_t)16, room});
        smem += (size_t)a.upw * per_unit + hbytes + pbytes;
    }
    auto kern = (a.t0g || a.t1g) ? k_pcg_persistent<B, S, Acc, true> : k_pcg_persistent<B, S, Acc, false>;
    // the attribute is per function, shared by every context and host thread: always the full
    // budget, so that a concurrent launch never finds it below its own request
    SG_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
    int per_sm = 0;
    SG_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPT, smem));
    if (per_sm < 1) return 1;
    SG_CUDA(c, cudaMemsetAsync(a.sync, 0, sizeof(unsigned), c->stream));
    void* params[] = {&a};
    SG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    SG_CUDA(c, cudaLaunchCooperativeKernel((const void*)kern, dim3(G), dim3(kPT), params, smem, c->stream));
    SG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    SG_CUDA(c, cudaEventSynchronize(c->ev1));
    SG_CUDA(c, cudaEventElapsedTime(ms, c->ev0, c->ev1));
    return 0;
}

}  // namespace

// Returns 0 when solved, 1 when the system does not fit this kernel (the
// caller then uses the graph path), negative on error.
int pcg_run_persistent(sgmas_context* c, const double* b, double* x, const PcgRunCfg& cfg, float* solve_ms,
                       int* launches, unsigned long long* stamps, int stamp_iters) {
    const BsrMatrix& M = c->bsr;

    PArgs a = {};
    a.A = BsrView{M.row_ptr, M.cols, M.vals, M.cap, M.row_list, M.nrows, M.n_long, nullptr};
    a.b = b; a.x = x; a.r = c->d_r; a.z = c->d_z; a.p0 = c->d_p0; a.p1 = c->d_p1; a.Ap = c->d_Ap;
    a.nrows = M.nrows;
    a.precond = cfg.precond;
    a.dinv = c->d_diag_inv;
    a.abd_rows = cfg.precond == 0 ? 4 * cfg.abd_bodies : 0;
    if (cfg.precond == 0)  // block-Jacobi: the bodies are the only extra units
        a.ex = ExtraRows{4 * cfg.abd_bodies, cfg.abd_bodies, M.nrows, cfg.abd_bodies, c->d_abd_inv};
    a.max_iter = cfg.max_iter == 0 ? 3 * M.nrows : cfg.max_iter;
    a.check_every = cfg.check_every;
    a.use_prec_norm = cfg.use_prec_norm;
    a.warm = cfg.warm;
    a.rel2 = cfg.rel_tol * cfg.rel_tol;
    a.abs2 = cfg.abs_tol * cfg.abs_tol;
    a.err = c->d_err;
    a.stamps = stamps;
    a.stamp_iters = stamp_iters;
    if (!c->d_psync) {
        if (ctx_alloc(c, &c->d_psync, 8)) return SGMAS_ERR_CUDA;
    }
    a.sync = c->d_psync;
    a.spin_limit = c->wait_limit;
    a.phantom = c->phantom_arrivals;
    int dev_sms = 0;
    SG_CUDA(c, cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, c->device));
    if (2 * c->partial_cap < 4 * dev_sms) {  // partials of p.Ap, r.z, r.r (+ start guess) per CTA (2 * partial_cap doubles)
        const int cap = 2 * dev_sms;
        if (ctx_alloc(c, &c->d_partials, 2 * (size_t)cap)) return SGMAS_ERR_CUDA;
        c->partial_cap = cap;
    }
    if (!c->d_state && ctx_alloc(c, &c->d_state, 1)) return SGMAS_ERR_CUDA;
    a.st = c->d_state;
    a.partials = c->d_partials;
    if (cfg.precond == 1) {
        a.N = c->N; a.Mm = c->Mm; a.L = c->L; a.total = c->total;
        for (int l = 0; l <= c->L; ++l) { a.lvl_count[l] = c->h_level_size[2 * l]; a.lvl_begin[l] = c->h_level_size[2 * l + 1]; }
        a.part_map = c->d_part_map; a.going_next = c->d_going_next;
        a.coarse_table = c->d_coarse_table; a.fine_mask = c->d_fine_mask;
        a.inv = c->d_inv; a.R = c->d_R;
        a.ex = extra_rows_of(c, cfg);
        if (cfg.patches) {
            if (c->patch_bodies != cfg.abd_bodies || !c->d_patch_info) return SGMAS_ERR_STATE;
            if (ctx_alloc_grow(c, &c->d_patch_zs, &c->patch_zs_cap, 3 * kPatchMax * cfg.abd_bodies))
                return SGMAS_ERR_CUDA;
            a.pv = PatchView{cfg.abd_bodies, c->d_patch_list, c->d_patch_info, c->d_patch_wcol, c->d_patch_wrow,
                             c->d_patch_zs, c->d_patch_owner + M.nrows, c->d_patch_ent};
            a.ex.patch = 1;
        }
    }
    int rc;
    switch ((c->bank == 16 ? 0 : 4) + c->precision) {
        case 0 + SGMAS_MAS_FP32: rc = launch_t<16, float, float>(c, a, solve_ms); break;
        case 0 + SGMAS_MAS_BF16: rc = launch_t<16, Fact<__nv_bfloat16>, float>(c, a, solve_ms); break;
        case 0 + SGMAS_MAS_FP64: rc = launch_t<16, double, double>(c, a, solve_ms); break;
        case 0 + SGMAS_MAS_FP32_FACTORED: rc = launch_t<16, Fact<float>, float>(c, a, solve_ms); break;
        case 4 + SGMAS_MAS_FP32: rc = launch_t<32, float, float>(c, a, solve_ms); break;
        case 4 + SGMAS_MAS_BF16: rc = launch_t<32, Fact<__nv_bfloat16>, float>(c, a, solve_ms); break;
        case 4 + SGMAS_MAS_FP64: rc = launch_t<32, double, double>(c, a, solve_ms); break;
        default: rc = launch_t<32, Fact<float>, float>(c, a, solve_ms); break;
    }
    if (rc) return rc;
    if (launches) *launches = 1;
    c->last_persistent = true;
    c->last_run = cfg;
    c->last_cfg = {cfg.precond, cfg.abd_bodies, 1};
    c->last_b = b;
    c->last_x = x;
    c->solved = true;
    return 0;
}
