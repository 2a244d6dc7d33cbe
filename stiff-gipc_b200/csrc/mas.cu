// mas.cu -- MAS preconditioner on sm_100a: hierarchy build, Hessian scatter,
// dense subdomain inverses and the apply.
//
// Restates SG/MASPreconditioner.cu (StiffGIPC) with a B200 layout:
//  * a subdomain ("bank") of B=16 slots is a half-warp; bank-local masks,
//    closures, cluster counts and ids use shuffles and ballots instead of the
//    reference's racy shared-memory patterns;
//  * every level count stays on the device (grids are sized by upper bounds),
//    so the build has one host read (the total cluster count) per rebuild;
//  * the apply stages each bank's packed inverse tile into shared memory with
//    one cp.async.bulk per CTA and fuses the PCG update, the level-0 Schwarz
//    product and the component sums of the residual into one kernel.
#include <stdio.h>

#include <algorithm>

#include "../../include/sgmas.h"
#include "ctx.hpp"
#include "pcg_state.cuh"
#include "mas_dev.cuh"
#include "extra_dev.cuh"

using namespace sgmas;

namespace {

constexpr int kThreads = 256;
constexpr int kCollectThreads = 128;


template <int B>
__device__ __forceinline__ unsigned seg_ballot(bool pred) {
    unsigned bal = __ballot_sync(0xffffffffu, pred);
    if (B == 32) return bal;
    const int base = (threadIdx.x & 31) & ~(B - 1);
    return (bal >> base) & ((1u << (B & 31)) - 1u);
}

// ---------------------------------------------------------------------------
// Hierarchy build (MASPreconditioner::ReorderRealtime, :1768-1807)
// ---------------------------------------------------------------------------

// _buildCML0_new (:63-103): same-bank neighbour mask; out-of-bank neighbours
// compacted into the working list (read from the initial copy, so no reset).
template <int B>
__global__ void k_l0_masks(int Mm, int N, const int* __restrict__ part_map, const int* __restrict__ real_map,
                           const unsigned* __restrict__ nb_start, const unsigned* __restrict__ nb_num0,
                           const unsigned* __restrict__ nb_list0, unsigned* nb_num, unsigned* nb_list,
                           unsigned* fine_mask, int* err) {
    const int tdx = blockIdx.x * blockDim.x + threadIdx.x;
    if (tdx >= Mm) return;
    const int idx = part_map[tdx];
    if (idx < 0) return;
    if (idx >= N) { set_error(err, kDevBadIndex); return; }
    const int w = tdx / B, lane = tdx % B;
    unsigned msk = 1u << lane, nk = 0;
    const unsigned st = nb_start[idx], cnt = nb_num0[idx];
    for (unsigned i = 0; i < cnt; ++i) {
        const unsigned v = nb_list0[st + i];
        if (v >= (unsigned)N) { set_error(err, kDevBadIndex); continue; }
        const int s = real_map[v];
        if (s / B == w) msk |= 1u << (s % B);
        else nb_list[st + nk++] = v;
    }
    nb_num[idx] = nk;
    fine_mask[idx] = msk;
}

// _buildCollisionConnection_new (:1126-1538): decode the int4 contact and OR
// same-bank bits between its nodes; level 0 ORs into mask[vertex] through the
// slot map, level >= 1 into mask[coarse id].
template <int B>
__global__ void k_collision(int cp, const int4* __restrict__ pairs, int level, int node_offset, int N,
                           const int* __restrict__ real_map, const int* __restrict__ coarse_space,
                           unsigned* mask) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= cp) return;
    int v[4], id[4];
    const int nv = decode_contact(pairs[q], v);
    unsigned cm[4] = {0u, 0u, 0u, 0u};
    for (int i = 0; i < nv; ++i) {
        v[i] -= node_offset;
        if (v[i] >= 0 && v[i] < N) id[i] = level >= 1 ? coarse_space[(size_t)(level - 1) * N + v[i]] : real_map[v[i]];
        else id[i] = -1;
    }
    for (int i = 0; i < nv; ++i)
        for (int j = i + 1; j < nv; ++j) {
            if (id[i] == id[j] || id[i] < 0 || id[j] < 0) continue;
            if (id[i] / B == id[j] / B) {
                cm[i] |= 1u << (id[j] % B);
                cm[j] |= 1u << (id[i] % B);
            }
        }
    for (int i = 0; i < nv; ++i) {
        if (!cm[i]) continue;
        if (level >= 1) { if (id[i] >= 0) atomicOr(mask + id[i], cm[i]); }
        else if (v[i] >= 0 && v[i] < N) atomicOr(mask + v[i], cm[i]);
    }
}

// Bank-local transitive closure (the BFS of _preparePrefixSumL0_new :157-214
// and _nextLevelCluster :480-528) with a fixed trip count so every lane
// takes part in every shuffle.  Returns the closure; *leader = lowest lane.
template <int B>
__device__ __forceinline__ unsigned bank_closure(unsigned orig, bool valid, int lane, bool* leader) {
    unsigned msk = orig, visited = 1u << lane;
    #pragma unroll 1
    for (int it = 0; it < B; ++it) {
        const unsigned todo = valid ? (visited ^ msk) : 0u;
        const int nv = todo ? (__ffs(todo) - 1) : lane;
        const unsigned other = __shfl_sync(0xffffffffu, orig, nv, B);
        if (todo) { visited |= 1u << nv; msk |= other; }
    }
    *leader = valid && __popc(msk & lanemask_lt(lane)) == 0;
    return msk;
}

template <int B>
__global__ void k_l0_closure(int Mm, const int* __restrict__ part_map, unsigned* fine_mask, int* prefix_orig) {
    const int tdx = blockIdx.x * blockDim.x + threadIdx.x;  // all threads stay for the shuffles
    const int lane = tdx % B;
    const int idx = tdx < Mm ? part_map[tdx] : -1;
    const unsigned orig = idx >= 0 ? fine_mask[idx] : 0u;
    bool leader;
    const unsigned msk = bank_closure<B>(orig, idx >= 0, lane, &leader);
    const unsigned el = seg_ballot<B>(leader);
    if (tdx < Mm && lane == 0) prefix_orig[tdx / B] = __popc(el);  // all-padding bank -> 0
    if (idx >= 0) fine_mask[idx] = msk;
}

// Exclusive scan of per-bank cluster counts in one CTA (thrust::exclusive_scan
// at :1604-1606 / :1698-1700) and the level size bookkeeping of
// _buildLevel1_new (:305-309) / _prefixSumLx (:553-557).
// from_level == 0: n = Mm/B banks, next begin = round(Mm);
// from_level >= 1: n = ceil(count/B), next begin = begin + round(count).
template <int B>
__global__ void k_level_scan(const int* __restrict__ cnt, int* pre, int Mm, int from_level, int* level_size) {
    __shared__ int sh[1024];
    __shared__ int carry;
    int n, next_begin;
    if (from_level == 0) {
        n = Mm / B;
        next_begin = round_up(Mm, B);
    } else {
        const int count = level_size[2 * from_level], begin = level_size[2 * from_level + 1];
        n = (count + B - 1) / B;
        next_begin = begin + round_up(count, B);
    }
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < n ? cnt[i] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < n) pre[i] = carry + sh[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += sh[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        level_size[2 * (from_level + 1)] = carry;
        level_size[2 * (from_level + 1) + 1] = next_begin;
    }
}

// _buildLevel1_new (:271-328): level-1 id = bank prefix + rank of the
// component's lowest lane among the bank's leaders.
template <int B>
__global__ void k_l1_ids(int Mm, const int* __restrict__ part_map, const unsigned* __restrict__ fine_mask,
                         const int* __restrict__ pre, int* coarse_space, int* going_next) {
    const int tdx = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = tdx % B;
    const int idx = tdx < Mm ? part_map[tdx] : -1;
    const unsigned msk = idx >= 0 ? fine_mask[idx] : 0u;
    const bool leader = idx >= 0 && __popc(msk & lanemask_lt(lane)) == 0;
    const unsigned el = seg_ballot<B>(leader);
    if (idx < 0) return;
    const int id = __popc(el & lanemask_lt(__ffs(msk) - 1)) + pre[tdx / B];
    coarse_space[idx] = id;
    going_next[idx] = id + round_up(Mm, B);
}

// _buildConnectMaskLx_new (:401-477): neighbours whose level-`level` node
// shares this vertex's coarse bank set bits of its coarse mask; the others
// stay in the compacted list.  (The reference's per-component OR equals this
// per-vertex OR: all members of a level-0 component share every coarse id.)
template <int B>
__global__ void k_lx_connect(int Mm, int N, int level, const int* __restrict__ part_map,
                             const unsigned* __restrict__ nb_start, unsigned* nb_num, unsigned* nb_list,
                             const int* __restrict__ coarse_space, unsigned* next_mask) {
    const int tdx = blockIdx.x * blockDim.x + threadIdx.x;
    if (tdx >= Mm) return;
    const int idx = part_map[tdx];
    if (idx < 0) return;
    const int* cs = coarse_space + (size_t)(level - 1) * N;
    const int ci = cs[idx];
    unsigned conn = 0u, nk = 0u;
    const unsigned st = nb_start[idx], cnt = nb_num[idx];
    for (unsigned i = 0; i < cnt; ++i) {
        const unsigned v = nb_list[st + i];
        const int cc = cs[v];
        if (ci / B == cc / B) conn |= 1u << (cc % B);
        else nb_list[st + nk++] = v;
    }
    nb_num[idx] = nk;
    if (conn) atomicOr(next_mask + ci, conn);
}

// _nextLevelCluster (:480-528): closure over the coarse banks at `level`.
template <int B>
__global__ void k_lx_closure(int level, const int* __restrict__ level_size, unsigned* next_mask, int* cnt) {
    const int count = level_size[2 * level];
    if ((int)(blockIdx.x * blockDim.x) >= round_up(count, B)) return;  // whole CTA beyond the level
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = idx % B;
    const bool valid = idx < count;
    const unsigned orig = valid ? ((1u << lane) | next_mask[idx]) : 0u;
    bool leader;
    const unsigned msk = bank_closure<B>(orig, valid, lane, &leader);
    const unsigned el = seg_ballot<B>(leader);
    if (lane == 0 && idx < count) cnt[idx / B] = __popc(el);
    if (valid) next_mask[idx] = msk;
}

// _prefixSumLx (:530-577): ids for level+1 and goingNext of level `level`.
template <int B>
__global__ void k_lx_ids(int level, const int* __restrict__ level_size, unsigned* next_mask,
                         const int* __restrict__ pre, int* going_next, int gn_cap, int* err) {
    const int count = level_size[2 * level];
    const int begin = level_size[2 * level + 1];
    if ((int)(blockIdx.x * blockDim.x) >= round_up(count, B)) return;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = idx % B;
    const bool valid = idx < count;
    const unsigned msk = valid ? next_mask[idx] : 0u;
    const bool leader = valid && __popc(msk & lanemask_lt(lane)) == 0;
    const unsigned el = seg_ballot<B>(leader);
    if (!valid) return;
    const int id = __popc(el & lanemask_lt(__ffs(msk) - 1)) + pre[idx / B];
    next_mask[idx] = (unsigned)id;
    const int g = idx + begin;
    if (g < gn_cap) going_next[g] = id + begin + round_up(count, B);
    else set_error(err, kDevCapacity);
}

// _computeNextLevel (:579-590)
__global__ void k_next_table(int N, int level, int* coarse_space, const unsigned* __restrict__ next_mask) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int nx = coarse_space[(size_t)(level - 1) * N + v];
    coarse_space[(size_t)level * N + v] = (int)next_mask[nx];
}

// _aggregationKernel (:592-625)
__global__ void k_aggregate(int N, int L, const int* __restrict__ going_next, int gn_cap, int* coarse_table,
                            int* err) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    int cur = v;
    int t[kMaxLevels] = {0, 0, 0, 0, 0, 0};
    for (int l = 0; l < L - 1; ++l) {
        if (cur < 0 || cur >= gn_cap) { set_error(err, kDevBadIndex); break; }
        cur = going_next[cur];
        t[l] = cur;
    }
    #pragma unroll
    for (int l = 0; l < kMaxLevels; ++l) coarse_table[(size_t)kMaxLevels * v + l] = t[l];
}

// ---------------------------------------------------------------------------
// Hessian scatter (PrepareHessian_bcoo, :1810-2054)
// ---------------------------------------------------------------------------
template <int B>
__device__ __forceinline__ double* blk_ptr(double* hess, int r, int c) {
    return hess + ((size_t)(c / B) * bsym_of(B) + sym_index(B, r % B, c % B)) * 9;
}

// Add 9 values into the block of the warp's group of lanes that share `key`
// (one set of atomics per group instead of per lane).
__device__ __forceinline__ void warp_grouped_add(long long key, const double (&m)[9], double* hess) {
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    double s[9];
    if (peers == 0xffffffffu) {  // whole warp on one target: butterfly sum
        #pragma unroll
        for (int q = 0; q < 9; ++q) {
            double v = m[q];
            #pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            s[q] = v;
        }
    } else {
        #pragma unroll
        for (int q = 0; q < 9; ++q) s[q] = 0.0;
        for (int j = 0; j < 32; ++j) {
            const bool mine = (peers >> j) & 1u;
            #pragma unroll
            for (int q = 0; q < 9; ++q) {
                const double v = __shfl_sync(0xffffffffu, m[q], j);
                if (mine) s[q] += v;
            }
        }
    }
    if (key >= 0 && (peers & lanemask_lt(lane)) == 0) {
        double* D = hess + key * 9;
        #pragma unroll
        for (int q = 0; q < 9; ++q) atomicAdd(D + q, s[q]);
    }
}

// phase 1: every FEM block.  Same-bank blocks are stored (transposed when the
// column slot precedes the row slot -- the reference drops that case, which
// its own slot maps never produce); other blocks climb goingNext and add into
// each level where both ends share a bank, summed per warp per target block.
template <int B>
__global__ void __launch_bounds__(256) k_scatter1(int n, const double* __restrict__ vals, const int* __restrict__ rows,
                                                  const int* __restrict__ cols, const uint32_t* __restrict__ indices,
                                                  int offset, int N, int L, const int* __restrict__ real_map,
                                                  const int* __restrict__ going_next, double* hess,
                                                  const int* __restrict__ level_size, int* err) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = I < n;  // every lane stays for the warp-level sums
    int rr = 0, cc = 0;
    double H[9];
    if (live) {
        const int k = indices ? (int)indices[I] : I;
        rr = rows[k] - offset;
        cc = cols[k] - offset;
        live = rr >= 0 && rr < N && cc >= 0 && cc < N;
        #pragma unroll
        for (int q = 0; q < 9; ++q) H[q] = live ? vals[(size_t)9 * k + q] : 0.0;
    } else {
        #pragma unroll
        for (int q = 0; q < 9; ++q) H[q] = 0.0;
    }
    const int total = level_size[2 * L + 1];
    int sr = 0, sc = 0;
    if (live) {
        sr = real_map[rr];
        sc = real_map[cc];
        if (sr / B == sc / B) {
            if (sc >= sr) {
                double* D = blk_ptr<B>(hess, sr, sc);
                #pragma unroll
                for (int q = 0; q < 9; ++q) D[q] = H[q];
            } else {
                double* D = blk_ptr<B>(hess, sc, sr);
                #pragma unroll
                for (int i = 0; i < 3; ++i)
                    #pragma unroll
                    for (int j = 0; j < 3; ++j) D[i + 3 * j] = H[j + 3 * i];
            }
            live = false;
        }
    }
    if (__ballot_sync(0xffffffffu, live) == 0u) return;
    int vr = rr, vc = cc;
    for (int level = 1; level < L; ++level) {
        long long key = -1;
        double m[9];
        if (live) {
            vr = going_next[vr];
            vc = going_next[vc];
            if (vr >= total || vc >= total || vr < 0 || vc < 0) {
                set_error(err, kDevBadIndex);
                live = false;
            }
        }
        if (live && vr / B == vc / B) {
            if (vc >= vr) {
                key = ((long long)(vc / B) * bsym_of(B) + sym_index(B, vr % B, vc % B));
                #pragma unroll
                for (int i = 0; i < 3; ++i)
                    #pragma unroll
                    for (int j = 0; j < 3; ++j)
                        m[i + 3 * j] = H[i + 3 * j] + (vc == vr ? H[j + 3 * i] : 0.0);
            } else {
                key = ((long long)(vr / B) * bsym_of(B) + sym_index(B, vc % B, vr % B));
                #pragma unroll
                for (int i = 0; i < 3; ++i)
                    #pragma unroll
                    for (int j = 0; j < 3; ++j) m[i + 3 * j] = H[j + 3 * i];
            }
        } else {
            #pragma unroll
            for (int q = 0; q < 9; ++q) m[q] = 0.0;
        }
        warp_grouped_add(key, m, hess);
    }
}

// phase 2: one CTA of B*B threads per level-0 bank; thread (r, c).  A bank's
// vertices share one coarse node per level-0 component, so the bank's blocks
// are first summed per component pair in shared memory and each component
// pair climbs goingNext once (same sums as the reference's per-pair climb).
template <int B>
__global__ void k_scatter2(int nbank0, int L, const int* __restrict__ part_map, const unsigned* __restrict__ fine_mask,
                           const int* __restrict__ going_next, double* hess) {
    extern __shared__ double S[];  // [B][B][9] component-pair sums
    __shared__ int comp_of[B], lead_vertex[B], ncomp;
    const int h = blockIdx.x;
    const int r = threadIdx.x / B, c = threadIdx.x % B;
    if (threadIdx.x < 32) {
        const int t = threadIdx.x;
        const int idx = t < B ? part_map[h * B + t] : -1;
        const unsigned msk = idx >= 0 ? fine_mask[idx] : 0u;
        const bool leader = idx >= 0 && __popc(msk & lanemask_lt(t)) == 0;
        const unsigned lb = __ballot_sync(0xffffffffu, leader);
        if (t < B) {
            comp_of[t] = idx >= 0 ? __popc(lb & lanemask_lt(__ffs(msk) - 1)) : -1;
            if (leader) lead_vertex[__popc(lb & lanemask_lt(t))] = idx;
        }
        if (t == 0) ncomp = __popc(lb);
    }
    for (int q = threadIdx.x; q < B * B * 9; q += blockDim.x) S[q] = 0.0;
    __syncthreads();
    const int cr = comp_of[r], ccp = comp_of[c];
    if (cr >= 0 && ccp >= 0) {
        const double* T = hess + ((size_t)h * bsym_of(B) + sym_index(B, c >= r ? r : c, c >= r ? c : r)) * 9;
        double* D = S + (cr * B + ccp) * 9;
        #pragma unroll
        for (int i = 0; i < 3; ++i)
            #pragma unroll
            for (int j = 0; j < 3; ++j) atomicAdd(D + i + 3 * j, c >= r ? T[i + 3 * j] : T[j + 3 * i]);
    }
    __syncthreads();
    const int nc = ncomp;
    if ((int)threadIdx.x >= nc * nc) return;
    const int a = threadIdx.x / nc, b = threadIdx.x % nc;
    const double* M = S + (a * B + b) * 9;
    int vr = lead_vertex[a], vc = lead_vertex[b];
    for (int level = 1; level < L; ++level) {
        vr = going_next[vr];
        vc = going_next[vc];
        if (vr / B == vc / B && vc >= vr) {
            double* D = blk_ptr<B>(hess, vr, vc);
            #pragma unroll
            for (int q = 0; q < 9; ++q) atomicAdd(D + q, M[q]);
        }
    }
}

// ---------------------------------------------------------------------------
// Dense subdomain inverse (__inverse6_P96x96, :626-724): Gauss-Jordan without
// pivoting, zero diagonal -> 1, partial symmetrisation of the diagonal 3x3
// blocks.  One warp per matrix, the matrix in shared memory, lane-owned
// columns; each element sees the reference's exact operation sequence
// (IEEE divide, fused multiply-add), so the FP64 result is reproducible.
// ---------------------------------------------------------------------------
template <int B>
__host__ __device__ constexpr int inv_warps() { return B == 16 ? 4 : 1; }

template <int B, typename S>
__global__ void __launch_bounds__(32 * inv_warps<B>()) k_invert(int nblk, const double* __restrict__ hess, S* inv,
                                                               double* inv64, const int* __restrict__ level_size,
                                                               int L) {
    constexpr int n = 3 * B;
    constexpr int bs = bsym_of(B);
    extern __shared__ double smem_inv[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mat = blockIdx.x * inv_warps<B>() + w;
    const int limit = level_size ? level_size[2 * L + 1] / B : nblk;
    if (mat >= nblk || mat >= limit) return;
    double* A = smem_inv + (size_t)w * (n * n + n);
    double* col = A + n * n;
    const double* P = hess + (size_t)mat * bs * 9;
    for (int e = lane; e < n * n; e += 32) {
        const int j = e / n, i = e % n;
        const int rb = j / 3, cb = i / 3;
        double v = cb >= rb ? P[sym_index(B, rb, cb) * 9 + (j % 3) + 3 * (i % 3)]
                            : P[sym_index(B, cb, rb) * 9 + (i % 3) + 3 * (j % 3)];
        if (i == j && v == 0.0) v = 1.0;
        A[e] = v;
    }
    __syncwarp();
    for (int j = 0; j < n; ++j) {
        const double rt = A[j * n + j];
        for (int k = lane; k < n; k += 32) col[k] = A[k * n + j];
        __syncwarp();
        for (int i = lane; i < n; i += 32) {
            const double piv = (i == j ? 1.0 : A[j * n + i]) / rt;
            A[j * n + i] = piv;
            for (int k = 0; k < n; ++k) {
                if (k == j) continue;
                const double base = (i == j) ? 0.0 : A[k * n + i];
                A[k * n + i] = __fma_rn(-col[k], piv, base);
            }
        }
        __syncwarp();
    }
    for (int i = lane; i < n; i += 32) {
        if (i % 3 < 2) A[(i + 1) * n + i] = A[i * n + i + 1];
        else A[i * n + i - 2] = A[(i - 2) * n + i];
    }
    __syncwarp();
    S* out = inv + (size_t)mat * bs * 9;
    for (int e = lane; e < bs * 9; e += 32) {
        const int b = e / 9, q = e % 9;
        int rb = 0, off = 0;
        while (off + (B - rb) <= b) { off += B - rb; ++rb; }
        const int cb = rb + (b - off);
        const int a = q % 3, cc = q / 3;
        const double v = A[(rb * 3 + a) * n + cb * 3 + cc];
        out[e] = Store<S>::from_double(v);
        if (inv64) inv64[(size_t)mat * bs * 9 + e] = v;
    }
}

// Factored inverse of one subdomain matrix per warp (storage Fact<T>): lower
// Cholesky M = L L^T in FP64 (right-looking; a pivot that is not positive
// becomes 1), then W = L^-1; the tile slot (rb, cb), rb <= cb, receives block
// (cb, rb) of W.  Every element's operations run in one fixed order (fma for
// each update; W_ij = acc / L_ii with acc = fma(-L_ik, W_kj, acc) over
// k = j .. i-1 ascending), restated by the oracle.  The padding rows of a bank
// (zero diagonal) become identity, as the reference's inverse does
// (:628-724).  The matrix sits in shared memory with a padded row stride
// (n + 1 doubles) so that lanes walking down a column hit distinct banks;
// W = L^-1 is formed row by row (step k finishes row k of W, then every later
// row takes its term k: independent updates across lanes), L in the lower
// triangle, W^T accumulating in the upper.
template <int B>
__host__ __device__ constexpr int chol_ld() { return 3 * B + 1; }
// shared memory per warp (doubles) of k_chol_inv / k_invert
template <int B>
constexpr size_t inv_smem_doubles(bool fact) {
    return fact ? (size_t)3 * B * chol_ld<B>() + 3 * B : (size_t)9 * B * B + 3 * B;
}

template <int B, typename S>
__global__ void __launch_bounds__(32 * inv_warps<B>()) k_chol_inv(int nblk, const double* __restrict__ hess, S* inv,
                                                                 double* inv64, const int* __restrict__ level_size,
                                                                 int L) {
    constexpr int n = 3 * B;
    constexpr int ld = chol_ld<B>();
    constexpr int bs = bsym_of(B);
    extern __shared__ double smem_inv[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mat = blockIdx.x * inv_warps<B>() + w;
    const int limit = level_size ? level_size[2 * L + 1] / B : nblk;
    if (mat >= nblk || mat >= limit) return;
    double* A = smem_inv + (size_t)w * (n * ld + n);  // row-major, stride ld; L lower, W^T upper
    double* dW = A + n * ld;                         // diagonal of W
    const double* P = hess + (size_t)mat * bs * 9;
    for (int e = lane; e < n * n; e += 32) {  // lower triangle of M; the upper accumulates W^T from 0
        const int i = e / n, j = e % n;
        if (j > i) { A[i * ld + j] = 0.0; continue; }
        const int rb = j / 3, cb = i / 3;
        double v = rb == cb ? P[sym_index(B, rb, rb) * 9 + (i % 3) + 3 * (j % 3)]
                            : P[sym_index(B, rb, cb) * 9 + (j % 3) + 3 * (i % 3)];
        if (i == j && v == 0.0) v = 1.0;
        A[i * ld + j] = v;
    }
    __syncwarp();
    for (int k = 0; k < n; ++k) {
        double d = A[k * ld + k];
        if (!(d > 0.0)) d = 1.0;
        const double lkk = sqrt(d);
        for (int i = k + 1 + lane; i < n; i += 32) A[i * ld + k] = A[i * ld + k] / lkk;
        __syncwarp();
        if (lane == 0) A[k * ld + k] = lkk;
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double lik = A[i * ld + k];
            for (int j = k + 1; j <= i; ++j) A[i * ld + j] = __fma_rn(-lik, A[j * ld + k], A[i * ld + j]);
        }
        __syncwarp();
    }
    for (int j = lane; j < n; j += 32) dW[j] = 1.0 / A[j * ld + j];
    __syncwarp();
    for (int k = 0; k < n; ++k) {
        // row k of W is complete: W_kj = acc_kj / L_kk (stored at A[j][k])
        for (int j = lane; j < k; j += 32) A[j * ld + k] = A[j * ld + k] / A[k * ld + k];
        __syncwarp();
        // every later row i takes its term k: acc_ij = fma(-L_ik, W_kj, acc_ij), j <= k
        for (int i = k + 1 + lane; i < n; i += 32) {
            const double lik = A[i * ld + k];
            for (int j = 0; j < k; ++j) A[j * ld + i] = __fma_rn(-lik, A[j * ld + k], A[j * ld + i]);
            A[k * ld + i] = __fma_rn(-lik, dW[k], A[k * ld + i]);
        }
        __syncwarp();
    }
    S* out = inv + (size_t)mat * bs * 9;
    for (int e = lane; e < bs * 9; e += 32) {
        const int b = e / 9, q = e % 9;
        int rb = 0, off = 0;
        while (off + (B - rb) <= b) { off += B - rb; ++rb; }
        const int cb = rb + (b - off);
        const int i = 3 * cb + q % 3, j = 3 * rb + q / 3;  // element (i, j) of W
        const double v = i > j ? A[j * ld + i] : (i == j ? dW[i] : 0.0);
        out[e] = Store<S>::from_double(v);
        if (inv64) inv64[(size_t)mat * bs * 9 + e] = v;
    }
}

// ---------------------------------------------------------------------------
// Apply (preconditioning, :2210-2251)
// ---------------------------------------------------------------------------


// Start staging `nb` consecutive bank tiles into shared memory with one bulk
// copy; the caller waits on `bar` (phase 0) before it reads them.
template <typename S>
__device__ __forceinline__ void stage_tiles_issue(S* tile, const S* src, int nb, int bs, uint64_t* bar) {
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const unsigned bytes = (unsigned)(nb * bs * 9 * sizeof(S));
    if (threadIdx.x == 0) {
        mbar_expect_tx(bar, bytes);
        bulk_g2s(tile, src, bytes, bar);
    }
}

constexpr int kL0Banks = 4;         // level-0 banks per CTA of the level-0 kernel
constexpr int kCoarseThreads = 256;  // threads per CTA of the coarse kernel
constexpr int kCoarseSmem = 80 * 1024;

template <int B>
__host__ __device__ constexpr int coarse_bpc() { return kCoarseThreads / B; }


// Level-0 kernel (BuildMultiLevelR :727-845 + the level-0 part of
// _schwarzLocalXSym6 :954-1024): mode 1 first applies the PCG update
// x += alpha p, r -= alpha Ap for the bank's vertices; then r -> Acc, the
// level-0 Schwarz product from the staged tile, and each level-0 component's
// residual sum stored into its level-1 node (a level-1 node has exactly one
// level-0 component, so plain stores suffice -- no atomics).
template <int B, typename S, typename Acc>
__global__ void __launch_bounds__(kL0Banks * B) k_apply_l0(int Mm, int L, const int* __restrict__ part_map,
                                                          const unsigned* __restrict__ fine_mask,
                                                          const int* __restrict__ going_next, const S* __restrict__ inv,
                                                          double* r, Acc* R, Acc* Z, int mode, double* x,
                                                          const double* __restrict__ p, const double* __restrict__ Ap,
                                                          const PcgState* st, int* err) {
    if (st && st->done) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    __shared__ __align__(16) Acc xch[(kL0Banks * B / 32) * kXchPerWarp];
    constexpr int bs = bsym_of(B);
    S* tile = reinterpret_cast<S*>(smem_raw);
    const int bank0 = blockIdx.x * kL0Banks;
    const int nb = min(kL0Banks, Mm / B - bank0);
    // the tiles arrive while the slot's vectors are read and updated
    stage_tiles_issue<S>(tile, inv + (size_t)bank0 * bs * 9, nb, bs, &bar);

    const int tdx = blockIdx.x * (kL0Banks * B) + threadIdx.x;
    const int lane = threadIdx.x % B;
    const int idx = tdx < Mm ? part_map[tdx] : -1;
    double rv0 = 0.0, rv1 = 0.0, rv2 = 0.0;
    unsigned msk = 0u;
    if (idx >= 0) {
        msk = fine_mask[idx];
        double* rp = r + 3 * (size_t)idx;
        rv0 = rp[0]; rv1 = rp[1]; rv2 = rp[2];
        if (mode == 1) {
            const double a = st->alpha;
            double* xp = x + 3 * (size_t)idx;
            const double* pp = p + 3 * (size_t)idx;
            const double* ap = Ap + 3 * (size_t)idx;
            xp[0] = xp[0] + a * pp[0]; xp[1] = xp[1] + a * pp[1]; xp[2] = xp[2] + a * pp[2];
            rv0 = rv0 - a * ap[0]; rv1 = rv1 - a * ap[1]; rv2 = rv2 - a * ap[2];
            rp[0] = rv0; rp[1] = rv1; rp[2] = rv2;
        }
    }
    Acc* xb = bank_slot<B>(xch);
    xch_put(xb, lane, (Acc)rv0, (Acc)rv1, (Acc)rv2);
    Acc s0, s1, s2;
    mask_sum<B, Acc>(msk, xb, s0, s1, s2);
    if (idx >= 0 && L > 1 && __popc(msk & lanemask_lt(lane)) == 0) {
        const int nx = going_next[idx];
        R[3 * (size_t)nx] = s0; R[3 * (size_t)nx + 1] = s1; R[3 * (size_t)nx + 2] = s2;
    }
    if (!mbar_wait(&bar, 0, err)) return;
    Acc z0, z1, z2;
    schwarz_rows<B, S, Acc>(tile + (size_t)(threadIdx.x / B) * bs * 9, lane, xb, z0, z1, z2);
    if (tdx < Mm) {
        Z[3 * (size_t)tdx] = z0; Z[3 * (size_t)tdx + 1] = z1; Z[3 * (size_t)tdx + 2] = z2;
    }
}

// Schwarz products for `nbk` consecutive banks starting at `bank0`, staged in
// chunks of at most `chunk` tiles.  With PUSH, each bank's residuals are
// also summed per parent node (the children of a node of the next level
// all lie in one bank) and stored into the parent.
template <int B, typename S, typename Acc, bool PUSH>
__device__ __forceinline__ bool schwarz_banks(const S* __restrict__ inv, Acc* R, Acc* Z,
                                              const int* __restrict__ going_next, int node_end, int bank0, int nbk,
                                              int chunk, S* tile, uint64_t* bar, unsigned& phase, int* err,
                                              Acc* xch) {
    constexpr int bs = bsym_of(B);
    const int per_pass = blockDim.x / B;
    const int lane = threadIdx.x % B;
    for (int c0 = 0; c0 < nbk; c0 += chunk) {
        const int nc = min(chunk, nbk - c0);
        __syncthreads();  // the previous chunk's tiles are no longer read
        if (threadIdx.x == 0) {
            const unsigned bytes = (unsigned)(nc * bs * 9 * sizeof(S));
            mbar_expect_tx(bar, bytes);
            bulk_g2s(tile, inv + (size_t)(bank0 + c0) * bs * 9, bytes, bar);
        }
        bool staged = false;  // the first pass reads its residuals while the tiles arrive
        for (int q = threadIdx.x / B; q < ((nc + per_pass - 1) / per_pass) * per_pass; q += per_pass) {
            const bool valid = q < nc;
            const int node = (bank0 + c0 + q) * B + lane;
            const Acc v0 = valid ? __ldcg(R + 3 * (size_t)node) : (Acc)0;
            const Acc v1 = valid ? __ldcg(R + 3 * (size_t)node + 1) : (Acc)0;
            const Acc v2 = valid ? __ldcg(R + 3 * (size_t)node + 2) : (Acc)0;
            Acc* xb = bank_slot<B>(xch);
            xch_put(xb, lane, v0, v1, v2);
            if (PUSH) {
                const int par = (valid && node < node_end) ? going_next[node] : -1;
                Acc s0, s1, s2;
                bool lead;
                group_sum<B, Acc>(par, xb, lane, s0, s1, s2, lead);
                if (lead) { R[3 * (size_t)par] = s0; R[3 * (size_t)par + 1] = s1; R[3 * (size_t)par + 2] = s2; }
            }
            if (!staged) {  // same trip count on every thread: all wait here once per chunk
                if (!mbar_wait(bar, phase, err)) return false;
                phase ^= 1u;
                staged = true;
            }
            Acc z0, z1, z2;
            schwarz_rows<B, S, Acc>(tile + (size_t)(valid ? q : 0) * bs * 9, lane, xb, z0, z1, z2);
            if (valid) { Z[3 * (size_t)node] = z0; Z[3 * (size_t)node + 1] = z1; Z[3 * (size_t)node + 2] = z2; }
        }
    }
    return true;
}

// Coarse levels (_schwarzLocalXSym6 for levels >= 1).  Each CTA applies a
// run of level-1 banks and sums their residuals into the level-2 nodes; the
// CTA that finishes last (a ticket, nothing waits) then builds levels >= 3
// the same way, bank by bank, and applies the banks of levels >= 2 -- unless
// k_apply_coarse_hi follows (hi_kernel = 1) and they are more than two rounds
// of one CTA (large systems: a hundred or more banks), which it then spreads
// over CTAs.  Both read the level sizes on the device, so a recorded graph
// stays right when the hierarchy of a later solve changes size.
template <int B, typename S, typename Acc>
__global__ void __launch_bounds__(kCoarseThreads) k_apply_coarse(int L, const int* __restrict__ level_size,
                                                                 const int* __restrict__ going_next,
                                                                 const S* __restrict__ inv, Acc* R, Acc* Z,
                                                                 const PcgState* st, unsigned* ticket, int hi_kernel,
                                                                 int* err) {
    if (st && st->done) return;
    if (L < 2) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    __shared__ bool am_last;
    __shared__ __align__(16) Acc xch[(kCoarseThreads / 32) * kXchPerWarp];
    constexpr int bs = bsym_of(B);
    constexpr int BPC = coarse_bpc<B>();
    S* tile = reinterpret_cast<S*>(smem_raw);
    const int chunk = max(1, min(BPC, (int)(kCoarseSmem / (bs * 9 * sizeof(S)))));
    const int total = level_size[2 * L + 1];
    const int beg1 = level_size[3], cnt1 = level_size[2];
    const int b1 = beg1 / B;                                    // first level-1 bank
    const int b2 = (L > 2 ? level_size[5] : total) / B;         // first level-2 bank
    const int active = (b2 - b1 + BPC - 1) / BPC;               // CTAs with level-1 work
    if ((int)blockIdx.x >= active) return;
    const int bank0 = b1 + blockIdx.x * BPC;
    unsigned phase = 0u;
    if (threadIdx.x == 0) { mbar_init(&bar, 1); fence_mbar_init(); }
    bool ok;
    if (L > 2)
        ok = schwarz_banks<B, S, Acc, true>(inv, R, Z, going_next, beg1 + cnt1, bank0, min(BPC, b2 - bank0), chunk,
                                            tile, &bar, phase, err, xch);
    else
        ok = schwarz_banks<B, S, Acc, false>(inv, R, Z, going_next, 0, bank0, min(BPC, b2 - bank0), chunk, tile,
                                             &bar, phase, err, xch);
    if (!ok || L <= 2) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        am_last = atomicAdd(ticket, 1u) == (unsigned)(active - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    // levels >= 3 from level 2, bank by bank (uniform trip counts per warp)
    const int lane = threadIdx.x % B;
    const int warp = threadIdx.x / 32, nwarp = blockDim.x / 32;
    constexpr int HPW = 32 / B;
    for (int lvl = 3; lvl < L; ++lvl) {
        const int beg = level_size[2 * (lvl - 1) + 1], cnt = level_size[2 * (lvl - 1)];
        const int nbk = (cnt + B - 1) / B;
        for (int kk = warp * HPW; kk < nbk; kk += nwarp * HPW) {
            const int k = kk + (threadIdx.x % 32) / B;
            const bool valid = k < nbk && k * B + lane < cnt;
            const int node = beg + k * B + lane;
            const Acc v0 = valid ? __ldcg(R + 3 * (size_t)node) : (Acc)0;
            const Acc v1 = valid ? __ldcg(R + 3 * (size_t)node + 1) : (Acc)0;
            const Acc v2 = valid ? __ldcg(R + 3 * (size_t)node + 2) : (Acc)0;
            const int par = valid ? going_next[node] : -1;
            Acc* xb = bank_slot<B>(xch);
            xch_put(xb, lane, v0, v1, v2);
            Acc s0, s1, s2;
            bool lead;
            group_sum<B, Acc>(par, xb, lane, s0, s1, s2, lead);
            if (lead) { R[3 * (size_t)par] = s0; R[3 * (size_t)par + 1] = s1; R[3 * (size_t)par + 2] = s2; }
        }
        __syncthreads();
    }
    if (!(hi_kernel && total / B - b2 > 2 * BPC))
        schwarz_banks<B, S, Acc, false>(inv, R, Z, going_next, 0, b2, total / B - b2, chunk, tile, &bar, phase, err,
                                        xch);
    if (threadIdx.x == 0) *ticket = 0u;
}

// The Schwarz products of the banks of levels >= 2 (residuals complete: the
// previous kernel built them) when there are more than two rounds of one CTA
// of them: coarse_bpc banks per CTA, grid-stride.
template <int B, typename S, typename Acc>
__global__ void __launch_bounds__(kCoarseThreads) k_apply_coarse_hi(int L, const int* __restrict__ level_size,
                                                                    const int* __restrict__ going_next,
                                                                    const S* __restrict__ inv, Acc* R, Acc* Z,
                                                                    const PcgState* st, int* err) {
    if (st && st->done) return;
    if (L < 3) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint64_t bar;
    __shared__ __align__(16) Acc xch[(kCoarseThreads / 32) * kXchPerWarp];
    constexpr int bs = bsym_of(B);
    constexpr int BPC = coarse_bpc<B>();
    S* tile = reinterpret_cast<S*>(smem_raw);
    const int chunk = max(1, min(BPC, (int)(kCoarseSmem / (bs * 9 * sizeof(S)))));
    const int b2 = level_size[5] / B, bend = level_size[2 * L + 1] / B;
    if (bend - b2 <= 2 * BPC || b2 + (int)blockIdx.x * BPC >= bend) return;  // k_apply_coarse took them
    unsigned phase = 0u;
    if (threadIdx.x == 0) { mbar_init(&bar, 1); fence_mbar_init(); }
    for (int bank0 = b2 + blockIdx.x * BPC; bank0 < bend; bank0 += gridDim.x * BPC)
        if (!schwarz_banks<B, S, Acc, false>(inv, R, Z, going_next, 0, bank0, min(BPC, bend - bank0), chunk, tile,
                                             &bar, phase, err, xch))
            return;
}

}  // namespace

namespace {

// CollectFinalZ (:848-877) + r.z and r.r (kind >= 1).
template <typename Acc>
__global__ void __launch_bounds__(kCollectThreads) k_collect(int N, int L, int Mm, const int* __restrict__ level_size,
                                                      const int* __restrict__ real_map,
                                                      const int* __restrict__ coarse_table, const Acc* __restrict__ Z,
                                                      Acc* R, double* r, double* z, ExtraRows ex, int mode, double* x,
                                                      const double* p, const double* Ap, int kind,
                                                      PcgState* st, double* partials, unsigned* ticket,
                                                      int set_cond, unsigned long long cond) {
    if (st && st->done) {
        // the last kernel of a WHILE body must always leave the condition set
        if (set_cond && blockIdx.x == 0 && threadIdx.x == 0)
            cudaGraphSetConditional((cudaGraphConditionalHandle)cond, 0u);
        return;
    }
    __shared__ double sh[32];
    const int v = blockIdx.x * blockDim.x + threadIdx.x;  // MAS vertex v is row ex.fem_off + v of r, z
    double rz = 0.0, rr = 0.0;
    if (v < N) {
        const int rd = real_map[v];
        const size_t o = 3 * (size_t)(ex.fem_off + v);
        Acc c0 = Z[3 * (size_t)rd], c1 = Z[3 * (size_t)rd + 1], c2 = Z[3 * (size_t)rd + 2];
        for (int i = 1; i < L; ++i) {
            const int now = coarse_table[(size_t)kMaxLevels * v + i - 1];
            c0 += Z[3 * (size_t)now]; c1 += Z[3 * (size_t)now + 1]; c2 += Z[3 * (size_t)now + 2];
        }
        const double z0 = (double)c0, z1 = (double)c1, z2 = (double)c2;
        z[o] = z0; z[o + 1] = z1; z[o + 2] = z2;
        if (kind >= 1) {
            const double r0 = r[o], r1 = r[o + 1], r2 = r[o + 2];
            rz = r0 * z0 + r1 * z1 + r2 * z2;
            rr = r0 * r0 + r1 * r1 + r2 * r2;
        }
    }
    const int npad = (N + 31) & ~31;  // warps from npad on take the rows outside the MAS range
    if (kind >= 1 && ex.n_units > 0 && v >= npad) {
        const int wid = (v - npad) >> 5, nw = (gridDim.x * blockDim.x - npad) >> 5;
        extra_rows_work(ex, N, mode, mode == 1 ? st->alpha : 0.0, x, r, p, Ap, z, wid, nw, threadIdx.x & 31, rz,
                        rr);
    }
    if (kind < 1) return;
    const double brz = block_sum<kCollectThreads>(rz, sh);
    const double brr = block_sum<kCollectThreads>(rr, sh);
    __shared__ bool am_last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = brz;
        partials[gridDim.x + blockIdx.x] = brr;
        __threadfence();
        am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double s1 = 0.0, s2 = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kCollectThreads) {
        s1 += ((volatile double*)partials)[i];
        s2 += ((volatile double*)partials)[gridDim.x + i];
    }
    s1 = block_sum<kCollectThreads>(s1, sh);
    s2 = block_sum<kCollectThreads>(s2, sh);
    if (threadIdx.x == 0) {
        *ticket = 0u;
        pcg_end_iteration(st, s1, s2, kind, set_cond, cond);
    }
}

template <int B>
int build_hierarchy_t(sgmas_context* c) {
    cudaStream_t s = c->stream;
    const int Mm = c->Mm, N = c->N, L = c->L;
    const int gM = (Mm + kThreads - 1) / kThreads, gN = (N + kThreads - 1) / kThreads;
    SG_CUDA(c, cudaMemsetAsync(c->d_level_size, 0, sizeof(int) * 2 * (kMaxLevels + 2), s));
    k_l0_masks<B><<<gM, kThreads, 0, s>>>(Mm, N, c->d_part_map, c->d_real_map, c->d_nb_start, c->d_nb_num0,
                                          c->d_nb_list0, c->d_nb_num, c->d_nb_list, c->d_fine_mask, c->d_err);
    if (c->cp_num > 0)
        k_collision<B><<<(c->cp_num + kThreads - 1) / kThreads, kThreads, 0, s>>>(
            c->cp_num, (const int4*)c->d_pairs, 0, c->node_offset, N, c->d_real_map, c->d_coarse_space,
            c->d_fine_mask);
    k_l0_closure<B><<<gM, kThreads, 0, s>>>(Mm, c->d_part_map, c->d_fine_mask, c->d_prefix_orig);
    k_level_scan<B><<<1, 1024, 0, s>>>(c->d_prefix_orig, c->d_bank_pre, Mm, 0, c->d_level_size);
    k_l1_ids<B><<<gM, kThreads, 0, s>>>(Mm, c->d_part_map, c->d_fine_mask, c->d_bank_pre, c->d_coarse_space,
                                        c->d_going_next);
    for (int level = 1; level < L; ++level) {
        SG_CUDA(c, cudaMemsetAsync(c->d_next_mask, 0, sizeof(unsigned) * N, s));
        k_lx_connect<B><<<gM, kThreads, 0, s>>>(Mm, N, level, c->d_part_map, c->d_nb_start, c->d_nb_num,
                                                c->d_nb_list, c->d_coarse_space, c->d_next_mask);
        if (c->cp_num > 0)
            k_collision<B><<<(c->cp_num + kThreads - 1) / kThreads, kThreads, 0, s>>>(
                c->cp_num, (const int4*)c->d_pairs, level, c->node_offset, N, c->d_real_map, c->d_coarse_space,
                c->d_next_mask);
        const int gC = (round_up(N, B) + kThreads - 1) / kThreads;
        k_lx_closure<B><<<gC, kThreads, 0, s>>>(level, c->d_level_size, c->d_next_mask, c->d_bank_cnt);
        k_level_scan<B><<<1, 1024, 0, s>>>(c->d_bank_cnt, c->d_bank_pre, Mm, level, c->d_level_size);
        k_lx_ids<B><<<gC, kThreads, 0, s>>>(level, c->d_level_size, c->d_next_mask, c->d_bank_pre,
                                            c->d_going_next, c->gn_cap, c->d_err);
        k_next_table<<<gN, kThreads, 0, s>>>(N, level, c->d_coarse_space, c->d_next_mask);
    }
    k_aggregate<<<gN, kThreads, 0, s>>>(N, L, c->d_going_next, c->gn_cap, c->d_coarse_table, c->d_err);
    // kernels launched above: 4 at level 0 (+ contacts), 5 per coarser level (+ contacts), aggregate
    c->build_launches += 5 + (L - 1) * 5 + L * (c->cp_num > 0 ? 1 : 0);
    SG_CUDA(c, cudaGetLastError());
    SG_CUDA(c, cudaMemcpyAsync(c->h_level_size, c->d_level_size, sizeof(int) * 2 * (kMaxLevels + 2),
                               cudaMemcpyDeviceToHost, s));
    SG_CUDA(c, cudaStreamSynchronize(s));
    int herr = 0;
    SG_CUDA(c, cudaMemcpy(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) return ctx_fail(c, SGMAS_ERR_DEVICE, "MAS hierarchy build: device error %d", herr);
    c->total = c->h_level_size[2 * L + 1];
    return 0;
}

template <int B, typename S, typename Acc>
int scatter_invert_t(sgmas_context* c, const double* vals, const int* rows, const int* cols, const uint32_t* indices,
                     int offset, int n) {
    cudaStream_t s = c->stream;
    const int nblk = c->total / B;
    const size_t bs = bsym_of(B);
    SG_CUDA(c, cudaMemsetAsync(c->d_hess, 0, sizeof(double) * nblk * bs * 9, s));
    if (n > 0)
        k_scatter1<B><<<(n + 255) / 256, 256, 0, s>>>(
            n, vals, rows, cols, indices, offset, c->N, c->L, c->d_real_map, c->d_going_next, c->d_hess,
            c->d_level_size, c->d_err);
    {
        const size_t smem2 = (size_t)B * B * 9 * sizeof(double);
        SG_CUDA(c, cudaFuncSetAttribute(k_scatter2<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
        k_scatter2<B><<<c->Mm / B, B * B, smem2, s>>>(c->Mm / B, c->L, c->d_part_map, c->d_fine_mask, c->d_going_next,
                                                     c->d_hess);
    }
    constexpr int W = inv_warps<B>();
    const size_t smem = (size_t)W * inv_smem_doubles<B>(is_fact<S>::value) * sizeof(double);
    auto kern = is_fact<S>::value ? k_chol_inv<B, S> : k_invert<B, S>;
    SG_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(nblk + W - 1) / W, 32 * W, smem, s>>>(nblk, c->d_hess, (S*)c->d_inv, nullptr, c->d_level_size, c->L);
    c->build_launches += (n > 0 ? 1 : 0) + 2;  // scatter1, scatter2, invert
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

template <int B, typename S, typename Acc>
int apply_t(sgmas_context* c, const double* r, double* z, int mode, const PcgState* st, double* x, const double* p,
            const double* Ap, double* partials, unsigned* ticket, int kind, unsigned long long cond, int* launches,
            const ExtraRows& ex) {
    // r, z, x, p, Ap are whole-system vectors; the MAS kernels see the FEM range
    const size_t fo = 3 * (size_t)ex.fem_off;
    cudaStream_t s = c->stream;
    constexpr int bs = bsym_of(B);
    const size_t smem0 = (size_t)kL0Banks * bs * 9 * sizeof(S);
    const int chunk = std::max(1, std::min(coarse_bpc<B>(), (int)(kCoarseSmem / (bs * 9 * sizeof(S)))));
    const size_t smem1 = (size_t)chunk * bs * 9 * sizeof(S);
    auto k0 = k_apply_l0<B, S, Acc>;
    auto k1 = k_apply_coarse<B, S, Acc>;
    SG_CUDA(c, cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem0));
    SG_CUDA(c, cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
    const int nbank0 = c->Mm / B;
    const int parts = c->apply_parts;
    if (parts & 1)
        k0<<<(nbank0 + kL0Banks - 1) / kL0Banks, kL0Banks * B, smem0, s>>>(
            c->Mm, c->L, c->d_part_map, c->d_fine_mask, c->d_going_next, (const S*)c->d_inv, (double*)r + fo,
            (Acc*)c->d_R, (Acc*)c->d_Z, mode, x ? x + fo : nullptr, p ? p + fo : nullptr, Ap ? Ap + fo : nullptr,
            st, c->d_err);
    // level-1 banks are bounded by the vertex count (extra CTAs return at once)
    const int l1_cap = (c->N + B - 1) / B + 1;
    // banks of levels >= 2: more than two rounds of one CTA go to their own
    // kernel (the kernels decide again from the device's level sizes)
    const int nb_hi = c->L > 2 ? (c->h_level_size[2 * c->L + 1] - c->h_level_size[5]) / B : 0;
    const int hi_apart = nb_hi > 2 * coarse_bpc<B>();
    if (parts & 2) {
        k1<<<(l1_cap + coarse_bpc<B>() - 1) / coarse_bpc<B>(), kCoarseThreads, smem1, s>>>(
            c->L, c->d_level_size, c->d_going_next, (const S*)c->d_inv, (Acc*)c->d_R, (Acc*)c->d_Z, st,
            c->d_coarse_ticket, hi_apart, c->d_err);
        if (hi_apart) {
            auto k2 = k_apply_coarse_hi<B, S, Acc>;
            SG_CUDA(c, cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
            k2<<<(nb_hi + coarse_bpc<B>() - 1) / coarse_bpc<B>(), kCoarseThreads, smem1, s>>>(
                c->L, c->d_level_size, c->d_going_next, (const S*)c->d_inv, (Acc*)c->d_R, (Acc*)c->d_Z, st, c->d_err);
        }
    }
    // threads past the MAS vertices (padded to a warp): 16 per body, then one per other row
    const int n_extra = kind >= 1 && ex.n_units > 0 ? 16 * ex.abd_bodies + (ex.n_units - ex.abd_bodies) : 0;
    const int gN = (((c->N + 31) & ~31) + n_extra + kCollectThreads - 1) / kCollectThreads;
    if (parts & 4)
        k_collect<Acc><<<gN, kCollectThreads, 0, s>>>(
            c->N, c->L, c->Mm, c->d_level_size, c->d_real_map, c->d_coarse_table, (const Acc*)c->d_Z, (Acc*)c->d_R,
            (double*)r, z, ex, mode, x, p, Ap, kind, (PcgState*)st, partials, ticket, cond != 0ull, cond);
    SG_CUDA(c, cudaGetLastError());
    if (launches) *launches += 3 + hi_apart;
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// internal entry points
// ---------------------------------------------------------------------------
int mas_build_hierarchy(sgmas_context* c) {
    if (c->bank == 16) return build_hierarchy_t<16>(c);
    return build_hierarchy_t<32>(c);
}

int mas_scatter_and_invert(sgmas_context* c, const double* vals, const int* rows, const int* cols,
                           const uint32_t* indices, int offset, int n) {
#define SG_DISPATCH(B)                                                                                   \
    switch (c->precision) {                                                                              \
        case SGMAS_MAS_FP32: return scatter_invert_t<B, float, float>(c, vals, rows, cols, indices, offset, n); \
        case SGMAS_MAS_BF16:                                                                             \
            return scatter_invert_t<B, Fact<__nv_bfloat16>, float>(c, vals, rows, cols, indices, offset, n); \
        case SGMAS_MAS_FP32_FACTORED:                                                                    \
            return scatter_invert_t<B, Fact<float>, float>(c, vals, rows, cols, indices, offset, n);     \
        default: return scatter_invert_t<B, double, double>(c, vals, rows, cols, indices, offset, n);   \
    }
    if (c->bank == 16) { SG_DISPATCH(16) }
    SG_DISPATCH(32)
#undef SG_DISPATCH
}

int mas_launch_apply(sgmas_context* c, const double* r, double* z, int mode, const PcgState* st, double* x,
                     const double* p, const double* Ap, double* partials, unsigned* ticket, int iter_kind,
                     unsigned long long cond_handle, int* launches, const ExtraRows& ex) {
#define SG_DISPATCH(B)                                                                                          \
    switch (c->precision) {                                                                                     \
        case SGMAS_MAS_FP32:                                                                                    \
            return apply_t<B, float, float>(c, r, z, mode, st, x, p, Ap, partials, ticket, iter_kind, cond_handle, \
                                            launches, ex);                                                          \
        case SGMAS_MAS_BF16:                                                                                    \
            return apply_t<B, Fact<__nv_bfloat16>, float>(c, r, z, mode, st, x, p, Ap, partials, ticket,        \
                                                          iter_kind, cond_handle, launches, ex);                \
        case SGMAS_MAS_FP32_FACTORED:                                                                           \
            return apply_t<B, Fact<float>, float>(c, r, z, mode, st, x, p, Ap, partials, ticket, iter_kind,     \
                                                  cond_handle, launches, ex);                                   \
        default:                                                                                                \
            return apply_t<B, double, double>(c, r, z, mode, st, x, p, Ap, partials, ticket, iter_kind,         \
                                              cond_handle, launches, ex);                                       \
    }
    if (c->bank == 16) { SG_DISPATCH(16) }
    SG_DISPATCH(32)
#undef SG_DISPATCH
}

int mas_invert_blocks_dev(sgmas_context* c, const double* hess, int nblk, double* out64) {
    cudaStream_t s = c->stream;
    float* tmp = nullptr;
    const size_t bs = (size_t)c->bank * (c->bank + 1) / 2;
    SG_CUDA(c, cudaMallocAsync((void**)&tmp, sizeof(float) * nblk * bs * 9, s));
    const bool fact = c->precision == SGMAS_MAS_BF16 || c->precision == SGMAS_MAS_FP32_FACTORED;
    if (c->bank == 16) {
        const size_t smem = (size_t)inv_warps<16>() * inv_smem_doubles<16>(fact) * sizeof(double);
        auto kern = fact ? k_chol_inv<16, float> : k_invert<16, float>;
        SG_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<(nblk + 3) / 4, 128, smem, s>>>(nblk, hess, tmp, out64, nullptr, 0);
    } else {
        const size_t smem = inv_smem_doubles<32>(fact) * sizeof(double);
        auto kern = fact ? k_chol_inv<32, float> : k_invert<32, float>;
        SG_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<nblk, 32, smem, s>>>(nblk, hess, tmp, out64, nullptr, 0);
    }
    SG_CUDA(c, cudaGetLastError());
    SG_CUDA(c, cudaFreeAsync(tmp, s));
    return 0;
}
