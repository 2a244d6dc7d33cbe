// patch.cu -- body patches: an overlapping Schwarz block around each affine
// body, added to the MAS on the FEM range.
//
// The reference preconditions a hybrid scene with the 12x12 block-Jacobi of
// each affine body (SG/abd_system/abd_system_function/
// setup_abd_system_gradient_and_hessian.cu:603-645) beside the MAS on the FEM
// vertices (SG/linear_system/linear_system/global_linear_system.cu:509-522).
// Neither piece sees the barrier couplings between a body and the FEM
// vertices it touches; with the contact stiffness of a resting body (kappa
// 1e5, distances down to 1e-3 dhat) those couplings dominate the matrix and
// PCG stalls.  A body patch is the body's 4 block rows plus the FEM vertices
// coupled to it (at most kPatchMax, the lowest ids; patches of neighbouring
// bodies overlap): its dense (12 + 3k) square block of A, factored in FP64
// (Cholesky, non-positive pivots replaced by 1 as the MAS's factored inverse
// does), stored as W = L^-1 in FP32 (FP64 beside the FP64 MAS).  The apply adds
// z += R^T W^T W R r per patch (R = restriction to the patch); the MAS still
// covers every FEM vertex.  An FEM vertex's patch parts are summed in body
// order through a per-row list of (body, local vertex) entries.  The
// library's own addition: the reference has no such block.
//
// W is stored twice, packed: row-major (row i holds W[i][0..i]) for y = W r
// with a warp per row, column-major (column j holds W[j..n-1][j]) for
// z = W^T y with a warp per column, so both passes read W coalesced.
#include <algorithm>

#include "../../include/sgmas.h"
#include "ctx.hpp"
#include "patch_dev.cuh"

using namespace sgmas;

namespace {

constexpr int kPT = 512;
constexpr int kCand = 1024;  // candidate FEM vertices gathered per body

// per-row lists of the patch entries e = b kPatchMax + i that cover the row:
// counts, an exclusive scan (one CTA), entries in claim order, then each
// row's list sorted (so the sums run in body order)
__global__ void k_patch_count(int nbodies, int fem_off, const int* __restrict__ plist, const int2* __restrict__ info,
                              int* cnt) {
    const int b = blockIdx.x;
    for (int i = threadIdx.x; i < info[b].x; i += blockDim.x) atomicAdd(cnt + fem_off + plist[(size_t)b * kPatchMax + i], 1);
}
__global__ void __launch_bounds__(1024) k_patch_scan(int nrows, const int* __restrict__ cnt, int* off) {
    __shared__ int sh[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nrows; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < nrows ? cnt[i] : 0;
        int x = v;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane == 31) sh[w] = x;
        __syncthreads();
        if (w == 0) {
            int y = sh[lane];
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += t;
            }
            sh[lane] = y;
        }
        __syncthreads();
        const int pre = carry + (w ? sh[w - 1] : 0) + x - v;
        if (i < nrows) off[i] = pre;
        __syncthreads();
        if (threadIdx.x == 1023) carry = pre + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) off[nrows] = carry;
}
__global__ void k_patch_fill(int nbodies, int fem_off, const int* __restrict__ plist, const int2* __restrict__ info,
                             const int* __restrict__ off, int* fill, int* ent) {
    const int b = blockIdx.x;
    for (int i = threadIdx.x; i < info[b].x; i += blockDim.x) {
        const int row = fem_off + plist[(size_t)b * kPatchMax + i];
        ent[off[row] + atomicAdd(fill + row, 1)] = b * kPatchMax + i;
    }
}
__global__ void k_patch_sort(int nrows, const int* __restrict__ off, int* ent) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    for (int a = off[row] + 1; a < off[row + 1]; ++a) {  // insertion sort (lists of a few entries)
        const int e = ent[a];
        int q = a - 1;
        while (q >= off[row] && ent[q] > e) { ent[q + 1] = ent[q]; --q; }
        ent[q + 1] = e;
    }
}

// one CTA per body: patch list, dense block in shared memory (packed lower,
// FP64), Cholesky, W = L^-1 into w64 (packed row-major, FP64 scratch), then
// both stored layouts in S.  info[b] = {k, truncated}.
template <typename S>
__global__ void __launch_bounds__(kPT) k_patch_build(int nbodies, int fem_off, int N, const int* __restrict__ row_ptr,
                                                     const int* __restrict__ cols, const uint32_t* __restrict__ src,
                                                     const double* __restrict__ vals, long long cap,
                                                     int* plist, int2* info,
                                                     double* w64, S* wcol, S* wrow, int* err) {
    extern __shared__ double Ash[];  // packed lower, patch_packed(kPatchMax) doubles
    __shared__ int cand[kCand];
    __shared__ int pl[kPatchMax];
    __shared__ int nc, kk, trunc;
    const int b = blockIdx.x;
    if (threadIdx.x == 0) { nc = 0; trunc = 0; }
    __syncthreads();
    for (int i = threadIdx.x; i < kCand; i += kPT) cand[i] = 0x7fffffff;
    __syncthreads();
    for (int r = 4 * b; r < 4 * b + 4; ++r)
        for (int p = row_ptr[r] + threadIdx.x; p < row_ptr[r + 1]; p += kPT) {
            const int c = cols[p] - fem_off;
            if (c >= 0 && c < N) {
                const int q = atomicAdd(&nc, 1);
                if (q < kCand) cand[q] = c;
                else trunc = 1;
            }
        }
    __syncthreads();
    // bitonic sort of the candidates (ascending)
    for (int size = 2; size <= kCand; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < kCand / 2; t += kPT) {
                const int lo = 2 * t - (t & (stride - 1)), hi = lo + stride;
                const bool up = (lo & size) == 0;
                const int x = cand[lo], y = cand[hi];
                if ((x > y) == up) { cand[lo] = y; cand[hi] = x; }
            }
            __syncthreads();
        }
    if (threadIdx.x == 0) {  // distinct vertices, at most kPatchMax (the lowest ids)
        int k = 0;
        for (int i = 0; i < kCand && cand[i] != 0x7fffffff; ++i)
            if (i == 0 || cand[i] != cand[i - 1]) {
                if (k < kPatchMax) pl[k++] = cand[i];
                else trunc = 1;
            }
        kk = k;
    }
    __syncthreads();
    const int k = kk, nb = 4 + k, n = 3 * nb;
    for (int i = threadIdx.x; i < k; i += kPT) plist[(size_t)b * kPatchMax + i] = pl[i];
    for (int i = threadIdx.x; i < n * (n + 1) / 2; i += kPT) Ash[i] = 0.0;
    __syncthreads();
    // the lower blocks of the patch's rows: local block row L (body rows 0-3,
    // then the patch vertices), local column from the CSR column
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int L = warp; L < nb; L += kPT / 32) {
        const int gr = L < 4 ? 4 * b + L : fem_off + pl[L - 4];
        for (int p = row_ptr[gr] + lane; p < row_ptr[gr + 1]; p += 32) {
            if (src[p] == 0xffffffffu) continue;  // row padding
            const int gc = cols[p];
            int Lc = -1;
            if (gc >= 4 * b && gc < 4 * b + 4) {
                Lc = gc - 4 * b;
            } else if (gc >= fem_off && gc < fem_off + N) {
                const int v = gc - fem_off;
                int lo = 0, hi = k;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (pl[mid] < v) lo = mid + 1;
                    else hi = mid;
                }
                if (lo < k && pl[lo] == v) Lc = 4 + lo;
            }
            if (Lc < 0 || Lc > L) continue;
            #pragma unroll
            for (int a = 0; a < 3; ++a)
                #pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    const int i = 3 * L + a, j = 3 * Lc + cc;
                    if (j <= i) Ash[packed_lower(i, j)] = vals[(3 * a + cc) * cap + p];  // row-major component
                }
        }
    }
    __syncthreads();
    // Cholesky (right-looking), packed lower, in place
    __shared__ double piv;
    for (int c = 0; c < n; ++c) {
        if (threadIdx.x == 0) {
            double d = Ash[packed_lower(c, c)];
            if (!(d > 0.0)) d = 1.0;
            piv = sqrt(d);
            Ash[packed_lower(c, c)] = piv;
        }
        __syncthreads();
        for (int i = c + 1 + threadIdx.x; i < n; i += kPT) Ash[packed_lower(i, c)] = Ash[packed_lower(i, c)] / piv;
        __syncthreads();
        const int m = n - c - 1;  // trailing size: element (c + 1 + t / m, c + 1 + t % m), lower part
        for (int t = threadIdx.x; t < m * m; t += kPT) {
            const int gi = c + 1 + t / m, gj = c + 1 + t % m;
            if (gj <= gi)
                Ash[packed_lower(gi, gj)] = __fma_rn(-Ash[packed_lower(gi, c)], Ash[packed_lower(gj, c)], Ash[packed_lower(gi, gj)]);
        }
        __syncthreads();
    }
    // W = L^-1, one column per thread: W_jj = 1 / L_jj, W_ij = -(sum_{t=j}^{i-1} L_it W_tj) / L_ii,
    // t ascending; the column lives in w64 (row-major packed), read back as it grows
    double* W = w64 + (size_t)b * patch_packed(kPatchMax);
    for (int j = threadIdx.x; j < n; j += kPT) {
        W[packed_lower(j, j)] = 1.0 / Ash[packed_lower(j, j)];
        for (int i = j + 1; i < n; ++i) {
            double s = 0.0;
            for (int t = j; t < i; ++t) s = __fma_rn(Ash[packed_lower(i, t)], W[packed_lower(t, j)], s);
            W[packed_lower(i, j)] = -s / Ash[packed_lower(i, i)];
        }
    }
    __syncthreads();
    S* wc = wcol + (size_t)b * patch_packed(kPatchMax);
    S* wr = wrow + (size_t)b * patch_packed(kPatchMax);
    for (int e = threadIdx.x; e < n * (n + 1) / 2; e += kPT) {
        // row-major packed index e -> (i, j)
        int i = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
        while (i * (i + 1) / 2 > e) --i;
        while ((i + 1) * (i + 2) / 2 <= e) ++i;
        const int j = e - i * (i + 1) / 2;
        const S v = Store<S>::from_double(W[e]);
        wr[e] = v;
        wc[packed_col(n, i, j)] = v;
    }
    if (threadIdx.x == 0) info[b] = make_int2(k, trunc);  // a truncated patch is still SPD: reported, not an error
}

template <typename S>
int build_t(sgmas_context* c, int nbodies, int fem_off) {
    cudaStream_t s = c->stream;
    const BsrMatrix& B = c->bsr;
    const size_t per = patch_packed(kPatchMax);
    const int nrows = B.nrows;
    if (ctx_alloc_grow(c, &c->d_patch_owner, &c->patch_owner_cap, 2 * nrows + 1) ||  // counts / fill, row offsets
        ctx_alloc_grow(c, &c->d_patch_ent, &c->patch_ent_cap, nbodies * kPatchMax) ||
        ctx_alloc_grow(c, &c->d_patch_list, &c->patch_list_cap, nbodies * kPatchMax) ||
        ctx_alloc_grow(c, &c->d_patch_info, &c->patch_info_cap, nbodies) ||
        ctx_alloc_grow(c, &c->d_patch_w64, &c->patch_w64_cap, (int)(nbodies * per)))
        return SGMAS_ERR_CUDA;
    const size_t wbytes = nbodies * per * sizeof(S);
    if (wbytes > c->patch_w_bytes) {
        if (c->d_patch_wcol) cudaFree(c->d_patch_wcol);
        if (c->d_patch_wrow) cudaFree(c->d_patch_wrow);
        c->d_patch_wcol = c->d_patch_wrow = nullptr;
        SG_CUDA(c, cudaMalloc(&c->d_patch_wcol, wbytes));
        SG_CUDA(c, cudaMalloc(&c->d_patch_wrow, wbytes));
        c->patch_w_bytes = wbytes;
    }
    const size_t smem = per * sizeof(double);
    SG_CUDA(c, cudaFuncSetAttribute(k_patch_build<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_patch_build<S><<<nbodies, kPT, smem, s>>>(nbodies, fem_off, c->N, B.row_ptr, B.cols, B.src, B.vals, B.cap,
                                                c->d_patch_list, c->d_patch_info, c->d_patch_w64,
                                                (S*)c->d_patch_wcol, (S*)c->d_patch_wrow, c->d_err);
    int* cnt = c->d_patch_owner;          // [nrows]: counts, then the fill cursor
    int* off = c->d_patch_owner + nrows;  // [nrows + 1] row offsets into the entries
    SG_CUDA(c, cudaMemsetAsync(cnt, 0, sizeof(int) * nrows, s));
    k_patch_count<<<nbodies, 64, 0, s>>>(nbodies, fem_off, c->d_patch_list, c->d_patch_info, cnt);
    k_patch_scan<<<1, 1024, 0, s>>>(nrows, cnt, off);
    SG_CUDA(c, cudaMemsetAsync(cnt, 0, sizeof(int) * nrows, s));
    k_patch_fill<<<nbodies, 64, 0, s>>>(nbodies, fem_off, c->d_patch_list, c->d_patch_info, off, cnt, c->d_patch_ent);
    k_patch_sort<<<(nrows + 255) / 256, 256, 0, s>>>(nrows, off, c->d_patch_ent);
    c->build_launches += 6;
    SG_CUDA(c, cudaGetLastError());
    c->patch_bodies = nbodies;
    return 0;
}

}  // namespace

// Build the body patches of a hybrid solve (bodies 0 .. nbodies-1 in block
// rows 0 .. 4 nbodies - 1, the MAS's FEM vertices from fem_off) on the block
// CSR of the current solve, in the context's MAS storage precision.
int patch_build(sgmas_context* c, int nbodies, int fem_off) {
    if (c->precision == SGMAS_MAS_FP64) return build_t<double>(c, nbodies, fem_off);
    return build_t<Fact<float>>(c, nbodies, fem_off);  // FP32 W beside the BF16 / FP32 MAS
}
