// convert.cu -- Hessian scatter-assembly into the BCOO layout and the Morton
// codes, on sm_100a.
//
//  * write_upper_blocks: element matrices -> upper 3x3 triplets
//    (write_triplet_fem SG/femEnergy.cu:14-62, write_triplet<12,12> with
//    SymGH SG/GIPC.cu:82-139);
//  * convert_triplets: raw triplets -> merged sorted BCOO
//    (Converter::convert SG/linear_system/utils/converter.cu:23-189) with a
//    project radix sort (LSD, 8-bit digits, stable) on compacted keys and a
//    segmented sum that walks each key's run in sorted order, so the merged
//    values are deterministic;
//  * element_plan / element_assemble: element matrices of fixed groups
//    straight into the planned merged structure (the sum of
//    write_upper_blocks + convert_triplets, bit for bit, without the raw
//    triplet array);
//  * morton_codes: _calcVertMChash / hash_code(type -1) (SG/GIPC.cu:142-201,
//    412-461).
#include <climits>

#include "../../include/sgmas.h"
#include "ctx.hpp"

using namespace sgmas;

namespace {

constexpr int kT = 256;
constexpr int kTile = 2048;  // keys per radix tile (256 threads x 8)

__global__ void k_radix_hist(const uint64_t* __restrict__ keys, int n, int shift, int ntiles, int* hist) {
    __shared__ int cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kTile;
    #pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int i = base + j * kT + threadIdx.x;
        if (i < n) atomicAdd(cnt + (int)((keys[i] >> shift) & 255u), 1);
    }
    __syncthreads();
    hist[threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// stable scatter: within a tile keys are ranked in index order (rounds of
// 256, warps in order, lanes in order) with __match_any_sync per digit
__global__ void k_radix_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, int n, int shift,
                                int ntiles, const int* __restrict__ offs, uint64_t* kout, uint32_t* vout) {
    __shared__ int run[256];
    __shared__ int wc[8][256];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    run[t] = offs[t * ntiles + blockIdx.x];
    #pragma unroll
    for (int q = 0; q < 8; ++q) wc[q][t] = 0;
    __syncthreads();
    const int base = blockIdx.x * kTile;
    for (int j = 0; j < 8; ++j) {
        const int i = base + j * kT + t;
        const bool valid = i < n;
        const uint64_t key = valid ? kin[i] : 0ull;
        const uint32_t val = (valid && vin) ? vin[i] : 0u;
        const int d = valid ? (int)((key >> shift) & 255u) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lanemask_lt(lane));
        if (valid && rank == 0) wc[w][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int off = run[d] + rank;
            for (int q = 0; q < w; ++q) off += wc[q][d];
            kout[off] = key;
            if (vout) vout[off] = val;
        }
        __syncthreads();
        int add = 0;
        #pragma unroll
        for (int q = 0; q < 8; ++q) { add += wc[q][t]; wc[q][t] = 0; }
        run[t] += add;
        __syncthreads();
    }
}

// exclusive scan of ints, two levels: per-CTA scan of 1024 items + block sums
__global__ void k_scan_local(const int* __restrict__ in, int* out, int n, int* sums) {
    __shared__ int sh[1024];
    const int i = blockIdx.x * 1024 + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) out[i] = sh[threadIdx.x] - v;
    if (threadIdx.x == 1023) sums[blockIdx.x] = sh[1023];
}
__global__ void k_scan_top(int* sums, int n, int* total) {
    __shared__ int sh[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < n ? sums[i] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < n) sums[i] = carry + sh[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += sh[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}
__global__ void k_scan_add(int* out, int n, const int* __restrict__ sums) {
    const int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

__global__ void k_make_keys(int n, const int* __restrict__ rows, const int* __restrict__ cols, int cb, uint64_t* keys,
                            uint32_t* idx, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = rows[i], c = cols[i];
    if (r < 0 || c < 0) set_error(err, kDevBadIndex);
    keys[i] = ((uint64_t)(uint32_t)r << cb) | (uint64_t)(uint32_t)c;
    idx[i] = (uint32_t)i;
}
__global__ void k_max_index(int n, const int* __restrict__ rows, const int* __restrict__ cols, int* mx) {
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = max(m, max(rows[i], cols[i]));
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(mx, m);
}
__global__ void k_heads(int n, const uint64_t* __restrict__ keys, int* head) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}
__global__ void k_seg_starts(int n, const uint64_t* __restrict__ keys, const int* __restrict__ head,
                             const int* __restrict__ seg, int cb, int* start, int* out_rows, int* out_cols) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !head[i]) return;
    const int u = seg[i];
    start[u] = i;
    out_rows[u] = (int)(keys[i] >> cb);
    out_cols[u] = (int)(keys[i] & ((1ull << cb) - 1ull));
}
// nine threads per merged block, one per component: each sums its component
// over the block's run in sorted (stable) order -- the order, and so the
// result, of a per-block sum -- while the nine read one block's 72 bytes
// together.  The run is read kSegBatch triplets at a time, all their loads in
// flight before the additions, which stay in run order.
constexpr int kSegBatch = 8;

__global__ void k_seg_sum(int nu, int n, const int* __restrict__ start, const uint32_t* __restrict__ idx,
                          const double* __restrict__ vals, double* out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 9LL * nu) return;
    const int u = (int)(t / 9), q = (int)(t % 9);
    const int b = start[u], e = (u + 1 < nu) ? start[u + 1] : n;
    double s = 0.0;
    for (int i0 = b; i0 < e; i0 += kSegBatch) {
        uint32_t ix[kSegBatch];
        double v[kSegBatch];
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j) ix[j] = i0 + j < e ? idx[i0 + j] : 0u;
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j) v[j] = i0 + j < e ? vals[9 * (size_t)ix[j] + q] : 0.0;
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j)
            if (i0 + j < e) s = (i0 + j == b) ? v[j] : s + v[j];  // the first value as is (keeps -0.0)
    }
    out[9 * (size_t)u + q] = s;
}

// upper block pair q (0 .. k(k+1)/2 - 1) of a k-node element: (ii, jj), ii <= jj, row-major
__device__ __forceinline__ void upper_pair(int k, int q, int& ii, int& jj) {
    int off = 0;
    ii = 0;
    while (off + (k - ii) <= q) { off += k - ii; ++ii; }
    jj = ii + (q - off);
}

// ---- element groups in a planned structure ----------------------------------
constexpr int kMaxElemGroups = 4;
struct ElemTab {
    const double* H[kMaxElemGroups];
    const int* nodes[kMaxElemGroups];
    long long off[kMaxElemGroups + 1];  // first raw triplet of each group
    int k[kMaxElemGroups];
    int ng;
};

// group g's matrices and row stride, selected with constant indices (a
// computed index into the kernel's parameter struct would copy it to local memory)
__device__ __forceinline__ const double* elem_H(const ElemTab& T, int g, int& w) {
    const double* h = T.H[0];
    w = 3 * T.k[0];
    if (g == 1) { h = T.H[1]; w = 3 * T.k[1]; }
    if (g == 2) { h = T.H[2]; w = 3 * T.k[2]; }
    if (g == 3) { h = T.H[3]; w = 3 * T.k[3]; }
    return h;
}

__device__ __forceinline__ int elem_group_of(const ElemTab& T, long long o) {
    int g = 0;
    while (g + 1 < T.ng && o >= T.off[g + 1]) ++g;
    return g;
}

// raw rows / cols of the groups in write order (k_upper_blocks' indices)
__global__ void k_elem_struct(ElemTab T, int* rows, int* cols) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= T.off[T.ng]) return;
    const int g = elem_group_of(T, o), k = T.k[g], np = k * (k + 1) / 2;
    const long long lo = o - T.off[g];
    const long long e = lo / np;
    int ii, jj;
    upper_pair(k, (int)(lo % np), ii, jj);
    const int row = T.nodes[g][e * k + ii], col = T.nodes[g][e * k + jj];
    rows[o] = min(row, col);
    cols[o] = max(row, col);
}

// for each sorted triplet: the first element of its block in the group's
// matrices (the transposed block, as k_upper_blocks writes it, when row > col)
__global__ void k_elem_src(int n, ElemTab T, const uint32_t* __restrict__ idx, long long* src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long o = idx[i];
    const int g = elem_group_of(T, o), k = T.k[g], np = k * (k + 1) / 2, w = 3 * k;
    const long long lo = o - T.off[g];
    const long long e = lo / np;
    int ii, jj;
    upper_pair(k, (int)(lo % np), ii, jj);
    const bool swap = T.nodes[g][e * k + ii] > T.nodes[g][e * k + jj];
    const long long base = e * w * w + (swap ? (long long)jj * 3 * w + ii * 3 : (long long)ii * 3 * w + jj * 3);
    src[i] = ((long long)g << 56) | base;
}

// k_seg_sum with the values read from the element matrices: three threads
// per merged block, one per block row a, each summing its row's three
// components (a, c) -- column-major index a + 3 c, as k_upper_blocks writes
// them -- = H[base + a w + c] (3 contiguous doubles) over the run in order,
// kSegBatch triplets' loads in flight before their additions.
__global__ void k_elem_seg_sum(int nu, int n, const int* __restrict__ start, const long long* __restrict__ src,
                               ElemTab T, double* out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3LL * nu) return;
    const int u = (int)(t / 3), a = (int)(t % 3);
    const int b = start[u], e = (u + 1 < nu) ? start[u + 1] : n;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int i0 = b; i0 < e; i0 += kSegBatch) {
        long long sv[kSegBatch];
        double v[kSegBatch][3];
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j) sv[j] = i0 + j < e ? src[i0 + j] : 0ll;
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j) {
            int w;
            const double* h0 = elem_H(T, (int)(sv[j] >> 56) & 3, w);
            const double* h = h0 + (sv[j] & ((1ll << 56) - 1)) + a * w;
            const bool in = i0 + j < e;
            v[j][0] = in ? __ldg(h) : 0.0;
            v[j][1] = in ? __ldg(h + 1) : 0.0;
            v[j][2] = in ? __ldg(h + 2) : 0.0;
        }
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j)
            if (i0 + j < e) {
                const bool f = i0 + j == b;  // the first value as is (keeps -0.0)
                s0 = f ? v[j][0] : s0 + v[j][0];
                s1 = f ? v[j][1] : s1 + v[j][1];
                s2 = f ? v[j][2] : s2 + v[j][2];
            }
    }
    out[9 * (size_t)u + a] = s0;
    out[9 * (size_t)u + a + 3] = s1;
    out[9 * (size_t)u + a + 6] = s2;
}

// ---- sorted append: raw triplets into a merged, sorted structure ----------
__device__ __forceinline__ bool key_less(int r0, int c0, int r1, int c1) {
    return r0 < r1 || (r0 == r1 && c0 < c1);
}

// for each distinct appended key u: lb[u] = its insertion point among the base
// blocks (first base block not below it), nw[u] = 1 when no base block has it
__global__ void k_append_locate(int nu, const int* __restrict__ urow, const int* __restrict__ ucol,
                                const int* __restrict__ brow, const int* __restrict__ bcol, int nb, int* lb, int* nw) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu) return;
    const int r = urow[u], c = ucol[u];
    int lo = 0, hi = nb;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key_less(brow[mid], bcol[mid], r, c)) lo = mid + 1;
        else hi = mid;
    }
    lb[u] = lo;
    nw[u] = !(lo < nb && brow[lo] == r && bcol[lo] == c);
}

// insertion points of the new keys, in order (non-decreasing)
__global__ void k_append_compact(int nu, const int* __restrict__ lb, const int* __restrict__ nw,
                                 const int* __restrict__ rank, int* nlb) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < nu && nw[u]) nlb[rank[u]] = lb[u];
}

// output place of base block j: j + the new keys inserted at or before it
__device__ __forceinline__ int base_place(int j, const int* __restrict__ nlb, int nnew) {
    int lo = 0, hi = nnew;  // upper bound of j in nlb
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (nlb[mid] <= j) lo = mid + 1;
        else hi = mid;
    }
    return j + lo;
}

// every base block to its output place (nine threads per block, one per component)
__global__ void k_append_base(int nb, const double* __restrict__ bval, const int* __restrict__ brow,
                              const int* __restrict__ bcol, const int* __restrict__ nlb, int nnew, double* oval,
                              int* orow, int* ocol) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 9LL * nb) return;
    const int j = (int)(t / 9), q = (int)(t % 9);
    const int o = base_place(j, nlb, nnew);
    oval[9 * (size_t)o + q] = bval[9 * (size_t)j + q];
    if (q == 0) { orow[o] = brow[j]; ocol[o] = bcol[j]; }
}

// every distinct appended key: the base block's value (when the base has the
// key) followed by the key's run in sorted (stable) order, summed in that
// order -- the order of a convert of the base's triplets followed by these
__global__ void k_append_sum(int nu, int n, const int* __restrict__ start, const uint32_t* __restrict__ idx,
                             const double* __restrict__ vals, const int* __restrict__ urow,
                             const int* __restrict__ ucol, const int* __restrict__ lb, const int* __restrict__ nw,
                             const int* __restrict__ rank, const int* __restrict__ nlb, int nnew,
                             const double* __restrict__ bval, double* oval, int* orow, int* ocol) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 9LL * nu) return;
    const int u = (int)(t / 9), q = (int)(t % 9);
    const int b = start[u], e = (u + 1 < nu) ? start[u + 1] : n;
    const bool fresh = nw[u] != 0;
    const int o = fresh ? lb[u] + rank[u] : base_place(lb[u], nlb, nnew);
    double s = fresh ? 0.0 : bval[9 * (size_t)lb[u] + q];
    for (int i0 = b; i0 < e; i0 += kSegBatch) {
        uint32_t ix[kSegBatch];
        double v[kSegBatch];
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j) ix[j] = i0 + j < e ? idx[i0 + j] : 0u;
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j) v[j] = i0 + j < e ? vals[9 * (size_t)ix[j] + q] : 0.0;
        #pragma unroll
        for (int j = 0; j < kSegBatch; ++j)
            if (i0 + j < e) s = (fresh && i0 + j == b) ? v[j] : s + v[j];
    }
    oval[9 * (size_t)o + q] = s;
    if (q == 0 && fresh) { orow[o] = urow[u]; ocol[o] = ucol[u]; }
}

// upper triplets of element matrices: one thread per (element, block pair)
__global__ void k_upper_blocks(int n_elem, int k, const double* __restrict__ H, const int* __restrict__ nodes,
                               double* vals, int* rows, int* cols) {
    const int np = k * (k + 1) / 2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n_elem * np) return;
    const int e = (int)(t / np), q = (int)(t % np);
    int ii, jj;
    upper_pair(k, q, ii, jj);
    const int row = nodes[(size_t)e * k + ii], col = nodes[(size_t)e * k + jj];
    const bool swap = row > col;
    const int w = 3 * k;
    const double* He = H + (size_t)e * w * w;
    const size_t o = (size_t)e * np + q;
    rows[o] = swap ? col : row;
    cols[o] = swap ? row : col;
    #pragma unroll
    for (int a = 0; a < 3; ++a)
        #pragma unroll
        for (int c = 0; c < 3; ++c)
            vals[9 * o + a + 3 * c] = swap ? He[(jj * 3 + a) * w + ii * 3 + c] : He[(ii * 3 + a) * w + jj * 3 + c];
}

// ---- Morton codes ----------------------------------------------------------
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
// std::min(std::max(x, lo), hi) with the std:: argument semantics (NaN passes through)
__device__ __forceinline__ double clamp_std(double x, double lo, double hi) {
    const double t = (x < lo) ? lo : x;
    return (hi < t) ? hi : t;
}
__device__ __forceinline__ uint32_t hash_code(double x, double y, double z, double res) {
    x = clamp_std(x * res, 0.0, res - 1.0);
    y = clamp_std(y * res, 0.0, res - 1.0);
    z = clamp_std(z * res, 0.0, res - 1.0);
    const uint32_t xx = expand_bits(__double2uint_rz(x));
    const uint32_t yy = expand_bits(__double2uint_rz(y));
    const uint32_t zz = expand_bits(__double2uint_rz(z));
    return (xx << 2) + (yy << 1) + zz;
}

__global__ void k_aabb(int n, const double* __restrict__ pos, double* part, unsigned* ticket, double* box) {
    __shared__ double sh[6][kT];
    double lo[3] = {1e308, 1e308, 1e308}, hi[3] = {-1e308, -1e308, -1e308};
    for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT)
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double v = pos[3 * (size_t)i + d];
            lo[d] = v < lo[d] ? v : lo[d];
            hi[d] = v > hi[d] ? v : hi[d];
        }
    #pragma unroll
    for (int d = 0; d < 3; ++d) { sh[d][threadIdx.x] = lo[d]; sh[3 + d][threadIdx.x] = hi[d]; }
    __syncthreads();
    for (int o = kT / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            #pragma unroll
            for (int d = 0; d < 3; ++d) {
                sh[d][threadIdx.x] = fmin(sh[d][threadIdx.x], sh[d][threadIdx.x + o]);
                sh[3 + d][threadIdx.x] = fmax(sh[3 + d][threadIdx.x], sh[3 + d][threadIdx.x + o]);
            }
        __syncthreads();
    }
    __shared__ bool last;
    if (threadIdx.x == 0) {
        for (int d = 0; d < 6; ++d) part[6 * blockIdx.x + d] = sh[d][0];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double b[6] = {1e308, 1e308, 1e308, -1e308, -1e308, -1e308};
    for (unsigned g = 0; g < gridDim.x; ++g)
        for (int d = 0; d < 3; ++d) {
            b[d] = fmin(b[d], ((volatile double*)part)[6 * g + d]);
            b[3 + d] = fmax(b[3 + d], ((volatile double*)part)[6 * g + 3 + d]);
        }
    for (int d = 0; d < 6; ++d) box[d] = b[d];
    *ticket = 0u;
}

__global__ void k_morton(int n, const double* __restrict__ pos, const double* __restrict__ box, uint64_t* codes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double sx = box[3] - box[0], sy = box[4] - box[1], sz = box[5] - box[2];
    const uint64_t mc = hash_code((pos[3 * (size_t)i] - box[0]) / sx, (pos[3 * (size_t)i + 1] - box[1]) / sy,
                                  (pos[3 * (size_t)i + 2] - box[2]) / sz, 1024.0);
    codes[i] = (mc << 32) | (uint64_t)(uint32_t)i;
}

struct Scratch {
    unsigned char* p;
    size_t off;
    template <typename T>
    T* take(size_t count) {
        off = (off + 255) & ~(size_t)255;
        T* r = reinterpret_cast<T*>(p + off);
        off += count * sizeof(T);
        return r;
    }
};

int ensure_scratch(sgmas_context* c, size_t bytes) {
    if (bytes <= c->sort_scratch_bytes) return 0;
    if (c->d_sort_scratch) cudaFree(c->d_sort_scratch);
    c->d_sort_scratch = nullptr;
    c->sort_scratch_bytes = 0;
    SG_CUDA(c, cudaMalloc(&c->d_sort_scratch, bytes));
    c->sort_scratch_bytes = bytes;
    return 0;
}

int scan_ints(sgmas_context* c, const int* in, int* out, int n, int* sums, int* total) {
    const int nb = (n + 1023) / 1024;
    k_scan_local<<<nb, 1024, 0, c->stream>>>(in, out, n, sums);
    k_scan_top<<<1, 1024, 0, c->stream>>>(sums, nb, total);
    k_scan_add<<<nb, 1024, 0, c->stream>>>(out, n, sums);
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

size_t sort_scratch_size(int n) {
    const size_t ntiles = (n + kTile - 1) / kTile;
    return (size_t)n * 12 + 2 * 256 * ntiles * 4 + ((256 * ntiles + 1023) / 1024 + 1) * 4 + 4096;
}

// LSD radix sort of (key, value) pairs in place; values may be null
int sort_pairs_impl(sgmas_context* c, uint64_t* keys, uint32_t* vals, int n, int key_bits, Scratch& S) {
    if (n <= 1) return 0;
    const int ntiles = (n + kTile - 1) / kTile;
    uint64_t* k2 = S.take<uint64_t>(n);
    uint32_t* v2 = vals ? S.take<uint32_t>(n) : nullptr;
    int* hist = S.take<int>((size_t)256 * ntiles);
    int* offs = S.take<int>((size_t)256 * ntiles);
    int* sums = S.take<int>(((size_t)256 * ntiles + 1023) / 1024 + 1);
    uint64_t *ka = keys, *kb = k2;
    uint32_t *va = vals, *vb = v2;
    const int passes = (key_bits + 7) / 8;
    for (int p = 0; p < passes; ++p) {
        k_radix_hist<<<ntiles, kT, 0, c->stream>>>(ka, n, 8 * p, ntiles, hist);
        if (scan_ints(c, hist, offs, 256 * ntiles, sums, nullptr)) return SGMAS_ERR_CUDA;
        k_radix_scatter<<<ntiles, kT, 0, c->stream>>>(ka, va, n, 8 * p, ntiles, offs, kb, vb);
        uint64_t* tk = ka; ka = kb; kb = tk;
        uint32_t* tv = va; va = vb; vb = tv;
    }
    if (ka != keys) {
        SG_CUDA(c, cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, c->stream));
        if (vals) SG_CUDA(c, cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, c->stream));
    }
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

}  // namespace

int sort_u64_pairs(sgmas_context* c, uint64_t* keys, uint32_t* vals, int n, int key_bits) {
    if (ensure_scratch(c, sort_scratch_size(n))) return SGMAS_ERR_CUDA;
    Scratch S{(unsigned char*)c->d_sort_scratch, 0};
    return sort_pairs_impl(c, keys, vals, n, key_bits, S);
}

int convert_triplets(sgmas_context* c, const double* vals, const int* rows, const int* cols, int n, double* out_vals,
                     int* out_rows, int* out_cols, int* n_unique) {
    *n_unique = 0;
    if (n == 0) return 0;
    cudaStream_t s = c->stream;
    const size_t need = (size_t)n * (8 + 4 + 4 + 4 + 4) + sort_scratch_size(n) + 8192;
    if (ensure_scratch(c, need)) return SGMAS_ERR_CUDA;
    Scratch S{(unsigned char*)c->d_sort_scratch, 0};
    uint64_t* keys = S.take<uint64_t>(n);
    uint32_t* idx = S.take<uint32_t>(n);
    int* head = S.take<int>(n);
    int* seg = S.take<int>(n);
    int* start = S.take<int>(n);
    int* misc = S.take<int>(4);
    int* sums = S.take<int>((n + 1023) / 1024 + 1);
    SG_CUDA(c, cudaMemsetAsync(misc, 0, sizeof(int) * 4, s));
    k_max_index<<<min(1024, (n + kT - 1) / kT), kT, 0, s>>>(n, rows, cols, misc);
    int mx = 0;
    SG_CUDA(c, cudaMemcpyAsync(&mx, misc, sizeof(int), cudaMemcpyDeviceToHost, s));
    SG_CUDA(c, cudaStreamSynchronize(s));
    int cb = 1;
    while ((1ll << cb) <= (long long)mx) ++cb;
    const int g = (n + kT - 1) / kT;
    k_make_keys<<<g, kT, 0, s>>>(n, rows, cols, cb, keys, idx, c->d_err);
    int rc = sort_pairs_impl(c, keys, idx, n, 2 * cb, S);
    if (rc) return rc;
    k_heads<<<g, kT, 0, s>>>(n, keys, head);
    rc = scan_ints(c, head, seg, n, sums, misc + 1);
    if (rc) return rc;
    int h2[2];
    SG_CUDA(c, cudaMemcpyAsync(h2, misc, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
    SG_CUDA(c, cudaStreamSynchronize(s));
    const int nu = h2[1];
    k_seg_starts<<<g, kT, 0, s>>>(n, keys, head, seg, cb, start, out_rows, out_cols);
    k_seg_sum<<<(int)((9LL * nu + kT - 1) / kT), kT, 0, s>>>(nu, n, start, idx, vals, out_vals);
    SG_CUDA(c, cudaGetLastError());
    *n_unique = nu;
    return 0;
}

// Sorted append: the n raw triplets are sorted and merged on their own (the
// steps of convert_triplets up to the segment starts), each distinct key is
// located among the n_base sorted base blocks, and the union is written in
// order: base blocks shifted by the new keys before them, then every appended
// key's sum (base value first when the base has the key).
int append_triplets(sgmas_context* c, const double* bval, const int* brow, const int* bcol, int nb,
                    const double* vals, const int* rows, const int* cols, int n, double* oval, int* orow, int* ocol,
                    int* n_out) {
    *n_out = 0;
    cudaStream_t s = c->stream;
    const int nn = std::max(n, 1);
    const size_t need = (size_t)nn * (8 + 4 * 11) + sort_scratch_size(nn) + 16384;
    if (ensure_scratch(c, need)) return SGMAS_ERR_CUDA;
    Scratch S{(unsigned char*)c->d_sort_scratch, 0};
    uint64_t* keys = S.take<uint64_t>(nn);
    uint32_t* idx = S.take<uint32_t>(nn);
    int* head = S.take<int>(nn);
    int* seg = S.take<int>(nn);
    int* start = S.take<int>(nn);
    int* urow = S.take<int>(nn);
    int* ucol = S.take<int>(nn);
    int* lb = S.take<int>(nn);
    int* nw = S.take<int>(nn);
    int* rank = S.take<int>(nn);
    int* nlb = S.take<int>(nn);
    int* misc = S.take<int>(4);
    int* sums = S.take<int>((nn + 1023) / 1024 + 1);
    int nu = 0, nnew = 0;
    if (n > 0) {
        SG_CUDA(c, cudaMemsetAsync(misc, 0, sizeof(int) * 4, s));
        k_max_index<<<min(1024, (n + kT - 1) / kT), kT, 0, s>>>(n, rows, cols, misc);
        int mx = 0;
        SG_CUDA(c, cudaMemcpyAsync(&mx, misc, sizeof(int), cudaMemcpyDeviceToHost, s));
        SG_CUDA(c, cudaStreamSynchronize(s));
        int cb = 1;
        while ((1ll << cb) <= (long long)mx) ++cb;
        const int g = (n + kT - 1) / kT;
        k_make_keys<<<g, kT, 0, s>>>(n, rows, cols, cb, keys, idx, c->d_err);
        int rc = sort_pairs_impl(c, keys, idx, n, 2 * cb, S);
        if (rc) return rc;
        k_heads<<<g, kT, 0, s>>>(n, keys, head);
        if ((rc = scan_ints(c, head, seg, n, sums, misc + 1))) return rc;
        int h2[2];
        SG_CUDA(c, cudaMemcpyAsync(h2, misc, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
        SG_CUDA(c, cudaStreamSynchronize(s));
        nu = h2[1];
        k_seg_starts<<<g, kT, 0, s>>>(n, keys, head, seg, cb, start, urow, ucol);
        const int gu = (nu + kT - 1) / kT;
        k_append_locate<<<gu, kT, 0, s>>>(nu, urow, ucol, brow, bcol, nb, lb, nw);
        if ((rc = scan_ints(c, nw, rank, nu, sums, misc + 2))) return rc;
        SG_CUDA(c, cudaMemcpyAsync(&nnew, misc + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
        SG_CUDA(c, cudaStreamSynchronize(s));
        k_append_compact<<<gu, kT, 0, s>>>(nu, lb, nw, rank, nlb);
    }
    if (nb > 0)
        k_append_base<<<(int)((9LL * nb + kT - 1) / kT), kT, 0, s>>>(nb, bval, brow, bcol, nlb, nnew, oval, orow,
                                                                      ocol);
    if (nu > 0)  // after the base copy: the shared keys' blocks are rewritten with their sums
        k_append_sum<<<(int)((9LL * nu + kT - 1) / kT), kT, 0, s>>>(nu, n, start, idx, vals, urow, ucol, lb, nw, rank,
                                                                     nlb, nnew, bval, oval, orow, ocol);
    SG_CUDA(c, cudaGetLastError());
    *n_out = nb + nnew;
    return 0;
}

// Assembly plan: the key sort and merge of convert_triplets for a fixed
// triplet structure, once.  The stable sorted order (idx) and the segment
// starts stay on the context; assemble_planned then runs only k_seg_sum, so
// its sums are convert_triplets' to the bit.
int assembly_plan(sgmas_context* c, const int* rows, const int* cols, int n, int* out_rows, int* out_cols,
                  int* n_unique) {
    *n_unique = 0;
    c->plan_n = -1;
    c->elem_ng = 0;  // element_plan sets it again after this call
    if (n == 0) {
        c->plan_n = 0;
        c->plan_nu = 0;
        return 0;
    }
    if (ctx_alloc_grow(c, &c->d_plan_idx, &c->plan_idx_cap, n) || ctx_alloc_grow(c, &c->d_plan_start, &c->plan_start_cap, n))
        return SGMAS_ERR_CUDA;
    cudaStream_t s = c->stream;
    const size_t need = (size_t)n * (8 + 4 + 4) + sort_scratch_size(n) + 8192;
    if (ensure_scratch(c, need)) return SGMAS_ERR_CUDA;
    Scratch S{(unsigned char*)c->d_sort_scratch, 0};
    uint64_t* keys = S.take<uint64_t>(n);
    int* head = S.take<int>(n);
    int* seg = S.take<int>(n);
    int* misc = S.take<int>(4);
    int* sums = S.take<int>((n + 1023) / 1024 + 1);
    uint32_t* idx = reinterpret_cast<uint32_t*>(c->d_plan_idx);
    SG_CUDA(c, cudaMemsetAsync(misc, 0, sizeof(int) * 4, s));
    k_max_index<<<min(1024, (n + kT - 1) / kT), kT, 0, s>>>(n, rows, cols, misc);
    int mx = 0;
    SG_CUDA(c, cudaMemcpyAsync(&mx, misc, sizeof(int), cudaMemcpyDeviceToHost, s));
    SG_CUDA(c, cudaStreamSynchronize(s));
    int cb = 1;
    while ((1ll << cb) <= (long long)mx) ++cb;
    const int g = (n + kT - 1) / kT;
    k_make_keys<<<g, kT, 0, s>>>(n, rows, cols, cb, keys, idx, c->d_err);
    int rc = sort_pairs_impl(c, keys, idx, n, 2 * cb, S);
    if (rc) return rc;
    k_heads<<<g, kT, 0, s>>>(n, keys, head);
    rc = scan_ints(c, head, seg, n, sums, misc + 1);
    if (rc) return rc;
    int h2[2];
    SG_CUDA(c, cudaMemcpyAsync(h2, misc, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
    SG_CUDA(c, cudaStreamSynchronize(s));
    k_seg_starts<<<g, kT, 0, s>>>(n, keys, head, seg, cb, c->d_plan_start, out_rows, out_cols);
    SG_CUDA(c, cudaGetLastError());
    c->plan_n = n;
    c->plan_nu = h2[1];
    *n_unique = h2[1];
    return 0;
}

int assemble_planned(sgmas_context* c, const double* vals, int n, double* out_vals) {
    if (c->plan_n < 0) return ctx_fail(c, SGMAS_ERR_STATE, "sgmas_assemble before sgmas_assembly_plan");
    if (n != c->plan_n)
        return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_assemble: %d triplets, the plan has %d", n, c->plan_n);
    const int nu = c->plan_nu;
    if (nu == 0) return 0;
    k_seg_sum<<<(int)((9LL * nu + kT - 1) / kT), kT, 0, c->stream>>>(nu, n, c->d_plan_start,
                                                        reinterpret_cast<const uint32_t*>(c->d_plan_idx), vals,
                                                        out_vals);
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

namespace {
// the group table of a call (an error status for bad groups)
int elem_tab(sgmas_context* c, const sgmas_element_group* groups, int ng, bool need_nodes, bool need_H, ElemTab& T,
             const char* fn) {
    T = ElemTab{};
    T.ng = ng;
    for (int g = 0; g < ng; ++g) {
        const sgmas_element_group& G = groups[g];
        if (G.n_elem < 0 || G.nodes_per_elem < 1 || G.nodes_per_elem > 4)
            return ctx_fail(c, SGMAS_ERR_ARG, "%s: group %d has n_elem %d, nodes_per_elem %d (1..4)", fn, g,
                            G.n_elem, G.nodes_per_elem);
        if (G.n_elem > 0 && ((need_nodes && !G.d_nodes) || (need_H && !G.d_H)))
            return ctx_fail(c, SGMAS_ERR_ARG, "%s: group %d has a NULL %s", fn, g, need_H ? "d_H" : "d_nodes");
        T.H[g] = G.d_H;
        T.nodes[g] = G.d_nodes;
        T.k[g] = G.nodes_per_elem;
        T.off[g + 1] = T.off[g] + (long long)G.n_elem * (G.nodes_per_elem * (G.nodes_per_elem + 1) / 2);
    }
    if (T.off[ng] > INT_MAX / 2) return ctx_fail(c, SGMAS_ERR_ARG, "%s: more than 2^30 - 1 triplets", fn);
    return 0;
}
}  // namespace

int element_plan(sgmas_context* c, const sgmas_element_group* groups, int ng, int* out_rows, int* out_cols,
                 int* n_unique) {
    *n_unique = 0;
    c->elem_ng = 0;
    ElemTab T;
    int rc = elem_tab(c, groups, ng, true, false, T, "sgmas_element_plan");
    if (rc) return rc;
    const int n = (int)T.off[ng];
    if (n > 0 && (!out_rows || !out_cols)) return SGMAS_ERR_ARG;
    if (n > 0) {
        if (ctx_alloc_grow(c, &c->d_elem_rc, &c->elem_rc_cap, 2 * n) ||
            ctx_alloc_grow(c, &c->d_elem_src, &c->elem_src_cap, n))
            return SGMAS_ERR_CUDA;
        k_elem_struct<<<(n + kT - 1) / kT, kT, 0, c->stream>>>(T, c->d_elem_rc, c->d_elem_rc + n);
        SG_CUDA(c, cudaGetLastError());
    }
    rc = assembly_plan(c, c->d_elem_rc, c->d_elem_rc + n, n, out_rows, out_cols, n_unique);
    if (rc) return rc;
    if (n > 0) {
        k_elem_src<<<(n + kT - 1) / kT, kT, 0, c->stream>>>(n, T, reinterpret_cast<const uint32_t*>(c->d_plan_idx),
                                                              c->d_elem_src);
        SG_CUDA(c, cudaGetLastError());
    }
    c->elem_ng = ng;
    for (int g = 0; g < ng; ++g) { c->elem_n[g] = groups[g].n_elem; c->elem_k[g] = groups[g].nodes_per_elem; }
    return 0;
}

int element_assemble(sgmas_context* c, const sgmas_element_group* groups, int ng, double* out_vals) {
    if (c->elem_ng == 0 || c->plan_n < 0)
        return ctx_fail(c, SGMAS_ERR_STATE, "sgmas_element_assemble before sgmas_element_plan");
    if (ng != c->elem_ng)
        return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_element_assemble: %d groups, the plan has %d", ng, c->elem_ng);
    for (int g = 0; g < ng; ++g)
        if (groups[g].n_elem != c->elem_n[g] || groups[g].nodes_per_elem != c->elem_k[g])
            return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_element_assemble: group %d is %d x %d nodes, planned %d x %d", g,
                            groups[g].n_elem, groups[g].nodes_per_elem, c->elem_n[g], c->elem_k[g]);
    ElemTab T;
    int rc = elem_tab(c, groups, ng, false, true, T, "sgmas_element_assemble");
    if (rc) return rc;
    const int nu = c->plan_nu;
    if (nu == 0) return 0;
    if (!out_vals) return SGMAS_ERR_ARG;
    k_elem_seg_sum<<<(int)((3LL * nu + kT - 1) / kT), kT, 0, c->stream>>>(nu, c->plan_n, c->d_plan_start,
                                                                          c->d_elem_src, T, out_vals);
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

int write_upper_blocks(sgmas_context* c, const double* H, int n_elem, int k, const int* nodes, double* vals, int* rows,
                       int* cols) {
    const long long total = (long long)n_elem * (k * (k + 1) / 2);
    if (total == 0) return 0;
    k_upper_blocks<<<(int)((total + kT - 1) / kT), kT, 0, c->stream>>>(n_elem, k, H, nodes, vals, rows, cols);
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

int morton_codes(sgmas_context* c, const double* pos, int n, const double* aabb, uint64_t* codes) {
    if (n == 0) return 0;
    const int g = min(296, (n + kT - 1) / kT);
    if (ensure_scratch(c, 6 * 8 * (size_t)(g + 2) + 512)) return SGMAS_ERR_CUDA;
    Scratch S{(unsigned char*)c->d_sort_scratch, 0};
    double* part = S.take<double>(6 * (size_t)g);
    double* box = S.take<double>(6);
    unsigned* ticket = S.take<unsigned>(1);
    if (aabb) {
        SG_CUDA(c, cudaMemcpyAsync(box, aabb, sizeof(double) * 6, cudaMemcpyHostToDevice, c->stream));
    } else {
        SG_CUDA(c, cudaMemsetAsync(ticket, 0, sizeof(unsigned), c->stream));
        k_aabb<<<g, kT, 0, c->stream>>>(n, pos, part, ticket, box);
    }
    k_morton<<<(n + kT - 1) / kT, kT, 0, c->stream>>>(n, pos, box, codes);
    SG_CUDA(c, cudaGetLastError());
    // the box is read from scratch by the kernel above; keep it alive until done
    SG_CUDA(c, cudaStreamSynchronize(c->stream));
    return 0;
}
