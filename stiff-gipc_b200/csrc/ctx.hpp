// ctx.hpp -- the opaque context behind the sgmas C-ABI (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/sgmas.h"
#include "common.cuh"

struct PcgState {
    double rz, rz0, rr0, rr, pAp, alpha, beta, rz_new;
    int k, done, iters, converged;
    int max_iter, check_every;
    double rel2, abs2;
    int use_prec_norm, pad;
    // start guess (initial_guess = 1): x0.b, b.b, scale, ||b - alpha A x0||^2
    double w_xb, w_bb, w_alpha, w_rr;
    int warm, w_reject;
    int breakdown;  // p.Ap <= 0 with r != 0: A (or the preconditioner) is not SPD
};

// Rows of a solve outside the MAS range (the reference's hybrid scenes:
// affine bodies first, 4 block rows each, then the FEM vertices the MAS
// covers at fem_off .. fem_off + N, then any further rows).  Each unit is a
// body (12x12 block-Jacobi) or one other row (identity: z = r).
struct ExtraRows {
    int fem_off, abd_bodies, nrows, n_units;
    const double* abd_inv;  // 144 per body, row-major inverse
    int patch;              // 1: the bodies are preconditioned by their patches (patch.cu), not here
};

struct PcgRunCfgLite {
    int precond, abd_bodies, valid;
};

struct PcgRunCfg {
    int max_iter;
    double rel_tol, abs_tol;
    int use_prec_norm;
    int precond;       // 0 Jacobi, 1 MAS
    int abd_bodies;
    int fem_offset;
    int check_every;
    int warm;          // 1: x holds a start guess (scaled, rejected when it raises ||r0||)
    int patches;       // 1: body patches (patch.cu) on the body rows and the FEM vertices they touch
};

struct BsrMatrix {
    int nrows = 0, nblocks = 0;       // upper blocks in
    long long nnz_pad = 0, cap = 0;   // full (both triangles), rows padded to even length
    int* row_ptr = nullptr;           // [nrows + 1]
    int* cols = nullptr;              // [cap]
    uint32_t* src = nullptr;          // [cap] source block | transposed bit
    double* vals = nullptr;           // 9 * cap, SoA: vals[q * cap + p], row-major component q
    int* cnt = nullptr;               // [nrows] entries per row
    int* cnt_lower = nullptr;         // [nrows]
    int* fill = nullptr;              // [nrows]
    int* first = nullptr;             // [nrows] first upper block of each row
    int* tcols = nullptr;             // [cap] lower entries in claim order (scratch)
    uint32_t* tsrc = nullptr;         // [cap]
    int* row_list = nullptr;          // [nrows] long rows first, then short rows (row order)
    int4* udesc = nullptr;            // [nrows * 4] SpMV work-unit descriptors (unit, lane group)
    int* d_nlong = nullptr;           // [1]
    int n_long = 0;                   // rows handled by a whole warp
    int rows_cap = 0;
};

// kernel-argument view of a BsrMatrix
struct BsrView {
    const int* row_ptr;
    const int* cols;
    const double* vals;
    long long cap;
    const int* row_list;
    int nrows;
    int n_long;
    const int4* udesc;  // precomputed unit descriptors (NULL: computed from row_list / row_ptr)
};

struct sgmas_context {
    int device = 0;
    cudaStream_t stream = nullptr;      // stream all work is ordered on
    cudaStream_t cap_stream = nullptr;  // the context's own stream (default)
    cudaStream_t rec_stream = nullptr;  // graph recording
    std::string err;
    int bank = 16;
    int precision = 0;
    int* d_err = nullptr;             // device error flag

    // ---- MAS setup ----
    bool mas_init = false, mas_assembled = false;
    int N = 0, Mm = 0, L = 0, node_offset = 0, nb_size = 0;
    unsigned *d_nb_list0 = nullptr, *d_nb_num0 = nullptr, *d_nb_start = nullptr;
    unsigned *d_nb_list = nullptr, *d_nb_num = nullptr;
    int *d_part_map = nullptr, *d_real_map = nullptr;
    unsigned *d_fine_mask = nullptr, *d_next_mask = nullptr;
    int *d_prefix_orig = nullptr;     // level-0 clusters per bank
    int *d_bank_cnt = nullptr, *d_bank_pre = nullptr;  // per-level scratch
    int *d_coarse_space = nullptr, *d_going_next = nullptr;
    int gn_cap = 0;
    int *d_level_size = nullptr;      // 2 * (kMaxLevels + 2)
    int h_level_size[2 * (sgmas::kMaxLevels + 2)] = {0};
    int *d_coarse_table = nullptr;    // 6 * N
    int total = 0, cap_total = 0;     // clusters (nodes over all levels)
    double* d_hess = nullptr;         // [cap_total / bank][bsym][9]
    void* d_inv = nullptr;            // same shape in the storage precision
    void* d_R = nullptr;              // 3 * cap_total accumulators
    void* d_Z = nullptr;
    const int* d_pairs = nullptr;
    int cp_num = 0;
    int mas_launches = 0;             // kernels per apply
    int build_launches = 0;           // kernels launched by the set-up of the current solve
    int apply_parts = 7;              // which apply kernels to launch (profiling)

    // ---- PCG ----
    BsrMatrix bsr;
    double *d_r = nullptr, *d_z = nullptr, *d_p0 = nullptr, *d_p1 = nullptr, *d_Ap = nullptr;
    double* d_diag_inv = nullptr;     // 9 * nrows (3x3 block-Jacobi)
    double* d_abd_inv = nullptr;      // 144 * bodies
    int vec_cap = 0, diag_cap = 0, abd_cap = 0;
    double* d_partials = nullptr;     // reduction partials
    unsigned* d_ticket = nullptr;
    unsigned* d_coarse_ticket = nullptr;  // last-CTA ticket of the coarse MAS kernel
    unsigned* d_psync = nullptr;          // grid barrier + ticket of the persistent PCG kernel
    bool persistent = true;               // solve with the persistent kernel when the system fits
    int wait_limit = sgmas::kSpinLimit;   // polls of each device-side wait of the persistent kernel
    int phantom_arrivals = 0;             // fault injection: arrivals each grid barrier waits for beyond the grid
    int pcg_ctas = 0;                     // CTAs of the persistent kernel (0: one per SM)
    bool last_persistent = false;         // the last solve ran the persistent kernel
    PcgRunCfg last_run = {};
    unsigned long long* d_stamps = nullptr;  // phase clock stamps of a profiled persistent solve
    size_t stamps_cap = 0;
    int* d_l1_bank = nullptr;             // level-0 bank of each level-1 node (persistent ownership)
    int l1_bank_cap = 0;
    int* d_own1 = nullptr;                // first level-1 bank of each CTA of the persistent kernel
    int own1_cap = 0;
    // body patches (patch.cu): owner body of each FEM vertex, patch lists, {k, truncated}, FP64 scratch,
    // W packed by columns and by rows (storage precision), the patches' part of z
    int* d_patch_owner = nullptr;          // per-row entry counts and offsets of the patch lists
    int* d_patch_ent = nullptr;            // patch entries (b kPatchMax + i) covering each row, body order
    int* d_patch_list = nullptr;
    int2* d_patch_info = nullptr;
    double* d_patch_w64 = nullptr;
    void* d_patch_wcol = nullptr;
    void* d_patch_wrow = nullptr;
    double* d_patch_zs = nullptr;          // [bodies][3 kPatchMax] each patch's part of z on its FEM rows
    int patch_owner_cap = 0, patch_ent_cap = 0, patch_list_cap = 0, patch_info_cap = 0, patch_w64_cap = 0, patch_zs_cap = 0;
    size_t patch_w_bytes = 0;
    int patch_bodies = 0;
    // SpMV plan of the persistent kernel (per solve): row order, cost prefixes, CTA work units,
    // halo-local column indices, halo vertex lists, per-CTA info, largest halo / unit count
    int* d_row_order = nullptr;
    int* d_cpre = nullptr;
    int4* d_udesc_c = nullptr;
    int* d_lcols = nullptr;
    int* d_halo = nullptr;
    int4* d_cinfo = nullptr;
    int* d_plan_stats = nullptr;
    int row_order_cap = 0, cpre_cap = 0, udesc_c_cap = 0, lcols_cap = 0, halo_cap = 0, cinfo_cap = 0,
        plan_stats_cap = 0;
    int partial_cap = 0;
    double* d_tune_x = nullptr;           // scratch solution of the autotuner's trial solves
    int spmv_resident = 0;                // resident CTAs of the graph-form SpMV (0: not yet queried)
    // assembly plan (sgmas_assembly_plan): stable sorted order of the raw triplets, segment starts
    int* d_plan_idx = nullptr;
    int* d_plan_start = nullptr;
    int plan_idx_cap = 0, plan_start_cap = 0;
    int plan_n = -1, plan_nu = 0;         // raw triplets and merged blocks of the plan (-1: none)
    // element plan (sgmas_element_plan): the plan above built from element groups, plus each sorted
    // triplet's source block in its group's element matrices (group << 56 | offset in doubles)
    long long* d_elem_src = nullptr;
    int* d_elem_rc = nullptr;             // raw rows, cols of the planned groups (the plan's input)
    int elem_src_cap = 0, elem_rc_cap = 0;
    int elem_ng = 0;                      // groups of the element plan (0: the plan is not an element plan)
    int elem_n[4] = {0, 0, 0, 0}, elem_k[4] = {0, 0, 0, 0};
    int tune_cap = 0;
    PcgState* d_state = nullptr;
    // uploaded host systems (sgmas_pcg_solve_host)
    double *d_hvals = nullptr, *d_hb = nullptr, *d_hx = nullptr;
    int *d_hrows = nullptr, *d_hcols = nullptr;
    long long hcap_blocks = 0, hcap_vec = 0;
    // graph cache
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraph_t graph = nullptr;
    unsigned long long graph_key[10] = {0};
    int graph_kernels_prologue = 0, graph_kernels_body = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    PcgRunCfgLite last_cfg = {0, 0, 0};
    const double* last_b = nullptr;
    double* last_x = nullptr;
    bool solved = false;
    // converter scratch
    void* d_sort_scratch = nullptr;
    size_t sort_scratch_bytes = 0;
    // learned start guess (csrc/mlp.cu)
    struct MlpState* mlp = nullptr;
    // the block CSR was built for these arrays by the learned start guess and
    // not used since: the next solve on the same arrays reuses it
    const void* bsr_src[3] = {nullptr, nullptr, nullptr};
    int bsr_src_nb = 0, bsr_src_nrows = 0;
    bool bsr_fresh = false;
};

// error helpers
int ctx_fail(sgmas_context* c, int code, const char* fmt, ...);
void mlp_free(sgmas_context* c);  // the learned start guess's buffers
#define SG_CUDA(c, expr)                                                                      \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess)                                                                \
            return ctx_fail((c), SGMAS_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr, \
                            cudaGetErrorString(_e));                                          \
    } while (0)

template <typename T>
int ctx_alloc(sgmas_context* c, T** p, size_t count) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return ctx_fail(c, -2, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
    return 0;
}

// (re)allocate only when `count` exceeds the capacity `*cap`
template <typename T>
int ctx_alloc_grow(sgmas_context* c, T** p, int* cap, int count) {
    if (*p && count <= *cap) return 0;
    if (ctx_alloc(c, p, (size_t)count)) return -2;
    *cap = count;
    return 0;
}

// internal entry points across translation units
int mas_build_hierarchy(sgmas_context* c);   // ReorderRealtime on the device
int mas_scatter_and_invert(sgmas_context* c, const double* vals, const int* rows, const int* cols,
                           const uint32_t* indices, int offset, int n);
int mas_launch_apply(sgmas_context* c, const double* r, double* z, int mode, const PcgState* st,
                     double* x, const double* p, const double* Ap, double* partials, unsigned* ticket,
                     int iter_kind, unsigned long long cond_handle, int* launches, const ExtraRows& ex);
// the extra rows of a MAS solve with configuration cfg (n_units = 0 when the MAS covers every row)
ExtraRows extra_rows_of(const sgmas_context* c, const PcgRunCfg& cfg);
int bsr_build(sgmas_context* c, const double* vals, const int* rows, const int* cols, int nblocks,
              int nrows);
int assembly_plan(sgmas_context* c, const int* rows, const int* cols, int n, int* out_rows, int* out_cols,
                  int* n_unique);
int assemble_planned(sgmas_context* c, const double* vals, int n, double* out_vals);
int append_triplets(sgmas_context* c, const double* bval, const int* brow, const int* bcol, int nb,
                    const double* vals, const int* rows, const int* cols, int n, double* oval, int* orow, int* ocol,
                    int* n_out);
int element_plan(sgmas_context* c, const sgmas_element_group* groups, int ng, int* out_rows, int* out_cols,
                 int* n_unique);
int element_assemble(sgmas_context* c, const sgmas_element_group* groups, int ng, double* out_vals);
void bsr_mark_fresh(sgmas_context* c, const sgmas_bcoo* A);  // the CSR just built is A's
bool bsr_reuse(sgmas_context* c, const sgmas_bcoo* A);       // true (once) when the fresh CSR is A's
int bsr_spmv_plain(sgmas_context* c, double a, const double* x, double b, double* y);
int bcoo_spmv_ref(sgmas_context* c, double a, const double* vals, const int* rows, const int* cols,
                  int nblocks, int nrows, const double* x, double b, double* y);
int pcg_run(sgmas_context* c, const double* b, double* x, const PcgRunCfg& cfg,
            float* solve_ms, int* launches);
int convert_triplets(sgmas_context* c, const double* vals, const int* rows, const int* cols, int n,
                     double* out_vals, int* out_rows, int* out_cols, int* n_unique);
int write_upper_blocks(sgmas_context* c, const double* H, int n_elem, int k, const int* nodes,
                       double* vals, int* rows, int* cols);
int morton_codes(sgmas_context* c, const double* pos, int n, const double* aabb, uint64_t* codes);
int sort_u64_pairs(sgmas_context* c, uint64_t* keys, uint32_t* vals, int n, int key_bits);
int mas_invert_blocks_dev(sgmas_context* c, const double* hess, int nblk, double* out64);
int pcg_profile(sgmas_context* c, int reps, float* ms, int n_ms);
int patch_build(sgmas_context* c, int nbodies, int fem_off);  // body patches of the current block CSR
int pcg_run_persistent(sgmas_context* c, const double* b, double* x, const PcgRunCfg& cfg, float* solve_ms,
                       int* launches, unsigned long long* stamps = nullptr, int stamp_iters = 0);

