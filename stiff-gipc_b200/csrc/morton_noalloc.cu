// morton_noalloc.cu -- Morton codes for callers that cannot allocate device
// memory.
//
// sgmas_morton_codes needs a context (whose creation allocates) and a scratch
// buffer for the bounding-box reduction (allocated on first use).  Some
// callers cannot do either: a host application whose device memory is handed
// out by its own pool or fixed at start-up, which must not grow behind its
// back, or a simulation loop that has a rule against allocating once it runs.
// For them this file offers sgmas_morton_codes_noalloc: the same codes
// (hash_code type -1 of SG/GIPC.cu:142-168, packed as in _calcVertMChash
// SG/GIPC.cu:412-461), with the reduction scratch in a fixed static device
// array instead of an allocation.
//
// The scratch (g_noalloc_scratch below) holds one partial bounding box per
// CTA; each CTA covers kTile vertices, so the array bounds the input size:
// at most kMaxCtas * kTile = 2,097,152 vertices.  Every GPU that loads the
// library holds the 49,216-byte array until the process exits.  All calls
// share it: two calls whose kernels overlap on the GPU race on it, so calls
// must be ordered (same stream, or synchronised).
//
// The first call on a device looks the array's device address up and loads
// both kernels; the address is kept per device for the life of the process,
// which assumes the device's primary context (the runtime's) is never reset
// (cudaDeviceReset) while the library is loaded.
#include <mutex>

#include "../../include/sgmas.h"
#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kTile = 2048;      // vertices per CTA (8 per thread)
constexpr int kMaxCtas = 1024;   // partial boxes the scratch holds
constexpr int kBoxOff = 6 * kMaxCtas;
constexpr int kTicketOff = kBoxOff + 6;
constexpr int kScratchDoubles = kTicketOff + 2;

// [0, kBoxOff): partial boxes (lo.xyz, hi.xyz per CTA); [kBoxOff, +6): the
// box; then the CTA ticket (an unsigned in the next slot)
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// the device address of g_noalloc_scratch, looked up once per device
constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ double clamp_std(double x, double lo, double hi) {
    const double t = (x < lo) ? lo : x;  // std::max(x, lo): NaN passes through
    return (hi < t) ? hi : t;            // std::min(t, hi)
}
__device__ __forceinline__ uint32_t hash_code(double x, double y, double z, double res) {
    x = clamp_std(x * res, 0.0, res - 1.0);
    y = clamp_std(y * res, 0.0, res - 1.0);
    z = clamp_std(z * res, 0.0, res - 1.0);
    return (expand_bits(__double2uint_rz(x)) << 2) + (expand_bits(__double2uint_rz(y)) << 1) +
           expand_bits(__double2uint_rz(z));
}

// bounding box: each CTA reduces its tile into its partial slot; the CTA that
// takes the last ticket reduces the partials in CTA order into the box
__global__ void k_box_tiles(int n, const double* __restrict__ pos, double* scratch) {
    __shared__ double sh[6][kThreads];
    double lo[3] = {1e308, 1e308, 1e308}, hi[3] = {-1e308, -1e308, -1e308};
    const int base = blockIdx.x * kTile;
    for (int i = base + threadIdx.x; i < min(n, base + kTile); i += kThreads)
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double v = pos[3 * (size_t)i + d];
            lo[d] = v < lo[d] ? v : lo[d];
            hi[d] = v > hi[d] ? v : hi[d];
        }
    #pragma unroll
    for (int d = 0; d < 3; ++d) { sh[d][threadIdx.x] = lo[d]; sh[3 + d][threadIdx.x] = hi[d]; }
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            #pragma unroll
            for (int d = 0; d < 3; ++d) {
                sh[d][threadIdx.x] = fmin(sh[d][threadIdx.x], sh[d][threadIdx.x + o]);
                sh[3 + d][threadIdx.x] = fmax(sh[3 + d][threadIdx.x], sh[3 + d][threadIdx.x + o]);
            }
        __syncthreads();
    }
    __shared__ bool last;
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kTicketOff);
    if (threadIdx.x == 0) {
        for (int d = 0; d < 6; ++d) scratch[6 * blockIdx.x + d] = sh[d][0];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double b[6] = {1e308, 1e308, 1e308, -1e308, -1e308, -1e308};
    for (unsigned g = 0; g < gridDim.x; ++g)
        for (int d = 0; d < 3; ++d) {
            b[d] = fmin(b[d], ((volatile double*)scratch)[6 * g + d]);
            b[3 + d] = fmax(b[3 + d], ((volatile double*)scratch)[6 * g + 3 + d]);
        }
    for (int d = 0; d < 6; ++d) scratch[kBoxOff + d] = b[d];
    *ticket = 0u;
}

__global__ void k_codes(int n, const double* __restrict__ pos, const double* __restrict__ scratch, int given,
                        double l0, double l1, double l2, double h0, double h1, double h2, uint64_t* codes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double lo[3], hi[3];
    if (given) {
        lo[0] = l0; lo[1] = l1; lo[2] = l2; hi[0] = h0; hi[1] = h1; hi[2] = h2;
    } else {
        #pragma unroll
        for (int d = 0; d < 3; ++d) { lo[d] = scratch[kBoxOff + d]; hi[d] = scratch[kBoxOff + 3 + d]; }
    }
    const uint64_t mc = hash_code((pos[3 * (size_t)i] - lo[0]) / (hi[0] - lo[0]),
                                  (pos[3 * (size_t)i + 1] - lo[1]) / (hi[1] - lo[1]),
                                  (pos[3 * (size_t)i + 2] - lo[2]) / (hi[2] - lo[2]), 1024.0);
    codes[i] = (mc << 32) | (uint64_t)(uint32_t)i;
}

// Look the scratch array up on the current device (first call per device)
// and load both kernels there, so that no later call is the first to touch
// them (under lazy module loading a kernel loads on its first use).
int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SGMAS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return SGMAS_ERR_CUDA;
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k_box_tiles) != cudaSuccess) return SGMAS_ERR_CUDA;
        if (cudaFuncGetAttributes(&fa, k_codes) != cudaSuccess) return SGMAS_ERR_CUDA;
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return SGMAS_OK;
}

}  // namespace

extern "C" int sgmas_morton_codes_noalloc(const double* d_pos, int n, const double* aabb, uint64_t* d_codes,
                                          void* stream) {
    if (n < 0 || (n > 0 && (!d_pos || !d_codes))) return SGMAS_ERR_ARG;
    if (n > SGMAS_MORTON_NOALLOC_MAX_VERTS) return SGMAS_ERR_CAPACITY;
    if (n == 0) return SGMAS_OK;
    // an error left pending by the caller's own earlier work is theirs: report it
    // without clearing it, and queue nothing
    if (cudaPeekAtLastError() != cudaSuccess) return SGMAS_ERR_CUDA;
    double* scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != SGMAS_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (!aabb) {
        // the ticket must start at zero (a failed earlier call may have left it set)
        if (cudaMemsetAsync(scratch + kTicketOff, 0, sizeof(unsigned), s) != cudaSuccess) return SGMAS_ERR_CUDA;
        k_box_tiles<<<(n + kTile - 1) / kTile, kThreads, 0, s>>>(n, d_pos, scratch);
        if (cudaGetLastError() != cudaSuccess) return SGMAS_ERR_CUDA;
    }
    const double z = 0.0;
    k_codes<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
        n, d_pos, scratch, aabb != nullptr, aabb ? aabb[0] : z, aabb ? aabb[1] : z, aabb ? aabb[2] : z,
        aabb ? aabb[3] : z, aabb ? aabb[4] : z, aabb ? aabb[5] : z, d_codes);
    return cudaGetLastError() == cudaSuccess ? SGMAS_OK : SGMAS_ERR_CUDA;
}

static_assert(SGMAS_MORTON_NOALLOC_MAX_VERTS == kMaxCtas * kTile, "header and scratch size disagree");
