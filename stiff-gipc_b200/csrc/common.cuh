// common.cuh -- shared device helpers for the sm_100a MAS-PCG kernels.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace sgmas {

constexpr int kMaxLevels = 6;          // levelnum cap (SG/MASPreconditioner.cu:1735-1736)
constexpr int kSpinLimit = 1 << 22;    // default bound on every device-side wait (polls)

// device error flags (ctx->d_err[0]); kernels never trap
enum DeviceError : int {
    kDevOk = 0,
    kDevWaitTimeout = 1,
    kDevBadIndex = 2,
    kDevCapacity = 3,
};

__device__ __forceinline__ unsigned lanemask_lt(int lane) {
    return lane >= 32 ? 0xffffffffu : ((1u << lane) - 1u);
}

__device__ __forceinline__ void set_error(int* err, int code) {
    if (err) atomicCAS(err, 0, code);
}

// ---- mbarrier + 1D bulk copy (TMA) -------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// one bulk global->shared copy; dst/src 16-byte aligned, bytes multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// bounded wait on phase `parity` (at most `limit` polls); returns false (and
// flags) if it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err, int limit = kSpinLimit) {
    uint32_t addr = smem_u32(bar);
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    set_error(err, kDevWaitTimeout);
    return false;
}

// Vertices of one contact in the reference's int4 encoding (the decoding of
// _buildCollisionConnection_new, SG/MASPreconditioner.cu:1140-1537): point-
// triangle / edge-edge and their degenerate point-point / point-edge forms,
// told apart by the signs of the entries.  Returns the vertex count (2-4).
__device__ __forceinline__ int decode_contact(int4 P, int v[4]) {
    int nv = 4;
    if (P.x >= 0) {
        if (P.w < 0) P.w = -P.w - 1;
        v[0] = P.x; v[1] = P.y; v[2] = P.z; v[3] = P.w;
    } else {
        const int x = -P.x - 1;
        if (P.z < 0) {
            if (P.y < 0) { v[0] = x; v[1] = -P.y - 1; v[2] = -P.z - 1; v[3] = -P.w - 1; }
            else { v[0] = x; v[1] = P.y; nv = 2; }
        } else if (P.w < 0) {
            if (P.y < 0) { v[0] = x; v[1] = -P.y - 1; v[2] = P.z; v[3] = -P.w - 1; }
            else { v[0] = x; v[1] = P.y; v[2] = P.z; nv = 3; }
        } else { v[0] = x; v[1] = P.y; v[2] = P.z; v[3] = P.w; }
    }
    return nv;
}

// ---- precision helpers ---------------------------------------------------
template <typename T> struct Store;
template <> struct Store<float> {
    __device__ __forceinline__ static float to_acc(float v) { return v; }
    __device__ __forceinline__ static float from_double(double v) { return __double2float_rn(v); }
};
template <> struct Store<__nv_bfloat16> {
    __device__ __forceinline__ static float to_acc(__nv_bfloat16 v) { return __bfloat162float(v); }
    // double -> float (RN) -> bf16 (RN): two explicit steps, mirrored by the oracle
    __device__ __forceinline__ static __nv_bfloat16 from_double(double v) {
        return __float2bfloat16_rn(__double2float_rn(v));
    }
};
template <> struct Store<double> {
    __device__ __forceinline__ static double to_acc(double v) { return v; }
    __device__ __forceinline__ static double from_double(double v) { return v; }
};

// Storage tag of the factored subdomain inverse: the tile holds W = L^-1 of
// the subdomain's Cholesky factor (M^-1 = W^T W, SPD for any rounding of W)
// in T; same tile size and slots as the explicit symmetric inverse.
template <typename T> struct Fact {
    T v;
};
template <typename T> struct Store<Fact<T>> {
    __device__ __forceinline__ static float to_acc(Fact<T> x) { return Store<T>::to_acc(x.v); }
    __device__ __forceinline__ static Fact<T> from_double(double v) { return Fact<T>{Store<T>::from_double(v)}; }
};
template <typename S> struct is_fact { static constexpr bool value = false; };
template <typename T> struct is_fact<Fact<T>> { static constexpr bool value = true; };

__device__ __forceinline__ float fma_acc(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_acc(double a, double b, double c) { return __fma_rn(a, b, c); }

// ---- deterministic block + grid reductions ----------------------------------
// Sum `v` over the CTA (fixed tree); result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = (threadIdx.x < NT / 32) ? sh[threadIdx.x] : 0.0;
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

// exclusive block-wide scan of one int per thread (1024 threads); returns the
// prefix, *total receives the sum
__device__ __forceinline__ int block_scan1024(int v, int* sh, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
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
        sh[32 + lane] = y;
    }
    __syncthreads();
    const int pre = (w ? sh[32 + w - 1] : 0) + x - v;
    *total = sh[63];
    __syncthreads();
    return pre;
}

// Last-CTA-done grid reduction (no waiting): every CTA writes its partial,
// the CTA that takes the last ticket sums all partials in blockIdx order.
// Returns true in thread 0 of the last CTA, with *out = total.
template <int NT>
__device__ __forceinline__ bool grid_sum_last(double partial, double* partials, unsigned* ticket,
                                              double* sh, double* out) {
    __shared__ bool am_last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = partial;
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += NT) s += ((volatile double*)partials)[i];
    s = block_sum<NT>(s, sh);
    if (threadIdx.x == 0) {
        *out = s;
        *ticket = 0u;
    }
    return threadIdx.x == 0;
}

}  // namespace sgmas
