// capi.cu -- the extern "C" boundary (include/sgmas.h).  Every entry point
// validates its arguments, returns a status and never aborts.
#include <climits>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/sgmas.h"
#include "ctx.hpp"

using namespace sgmas;

// message of the last failed call of this thread that had no context
static thread_local std::string g_host_err = "no error";

int ctx_fail(sgmas_context* c, int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    else g_host_err = buf;
    return code;
}

namespace {

int round_up(int v, int b) { return (v + b - 1) / b * b; }

// computeNumLevels (SG/MASPreconditioner.cu:1720-1739)
int num_levels(int max_nodes, int bank) {
    int n = 1, sz = round_up(max_nodes, bank);
    while (sz > bank) {
        sz /= bank;
        ++n;
        sz = round_up(sz, bank);
    }
    n += 1;
    return n > kMaxLevels ? kMaxLevels : n;
}

size_t store_size(int precision) {
    return precision == SGMAS_MAS_BF16 ? 2 : precision == SGMAS_MAS_FP64 ? 8 : 4;
}
size_t acc_size(int precision) { return precision == SGMAS_MAS_FP64 ? 8 : 4; }

int check_device_error(sgmas_context* c, const char* where) {
    int herr = 0;
    SG_CUDA(c, cudaMemcpyAsync(&herr, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (herr) {
        cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
        return ctx_fail(c, SGMAS_ERR_DEVICE, "%s: device error %d (%s)", where, herr,
                        herr == kDevWaitTimeout ? "bounded wait expired"
                        : herr == kDevBadIndex  ? "index out of range"
                                                : "capacity exceeded");
    }
    return 0;
}

int alloc_mas_matrices(sgmas_context* c, int total) {
    const int B = c->bank;
    int cap = round_up((int)(total * 1.05) + 1, B);
    if (cap < total) cap = round_up(total, B);
    const size_t nblk = cap / B, bs = (size_t)B * (B + 1) / 2;
    if (ctx_alloc(c, &c->d_hess, nblk * bs * 9)) return SGMAS_ERR_CUDA;
    if (ctx_alloc(c, (unsigned char**)&c->d_inv, nblk * bs * 9 * store_size(c->precision))) return SGMAS_ERR_CUDA;
    if (ctx_alloc(c, (unsigned char**)&c->d_R, 3 * (size_t)cap * acc_size(c->precision))) return SGMAS_ERR_CUDA;
    if (ctx_alloc(c, (unsigned char**)&c->d_Z, 3 * (size_t)cap * acc_size(c->precision))) return SGMAS_ERR_CUDA;
    SG_CUDA(c, cudaMemsetAsync(c->d_R, 0, 3 * (size_t)cap * acc_size(c->precision), c->stream));
    SG_CUDA(c, cudaMemsetAsync(c->d_inv, 0, nblk * bs * 9 * store_size(c->precision), c->stream));
    c->cap_total = cap;
    return 0;
}

void free_all(sgmas_context* c) {
    void* ptrs[] = {c->d_err, c->d_nb_list0, c->d_nb_num0, c->d_nb_start, c->d_nb_list, c->d_nb_num,
                    c->d_part_map, c->d_real_map, c->d_fine_mask, c->d_next_mask, c->d_prefix_orig,
                    c->d_bank_cnt, c->d_bank_pre, c->d_coarse_space, c->d_going_next, c->d_level_size,
                    c->d_coarse_table, c->d_hess, c->d_inv, c->d_R, c->d_Z, c->bsr.row_ptr, c->bsr.cols,
                    c->bsr.src, c->bsr.vals, c->bsr.cnt, c->bsr.cnt_lower, c->bsr.fill, c->bsr.first, c->d_r,
                    c->d_z, c->d_p0, c->d_p1, c->d_Ap, c->d_diag_inv, c->d_abd_inv, c->d_partials, c->d_ticket,
                    c->d_state, c->d_hvals, c->d_hb, c->d_hx, c->d_hrows, c->d_hcols, c->d_sort_scratch,
                    c->d_coarse_ticket, c->bsr.row_list, c->bsr.d_nlong, c->bsr.tcols, c->bsr.tsrc,
                    c->d_psync, c->d_stamps, c->d_l1_bank, c->d_own1, c->d_tune_x, c->bsr.udesc, c->d_plan_idx, c->d_elem_src, c->d_elem_rc,
                    c->d_plan_start, c->d_row_order, c->d_cpre, c->d_udesc_c, c->d_lcols, c->d_halo,
                    c->d_cinfo, c->d_plan_stats, c->d_patch_owner, c->d_patch_ent, c->d_patch_list, c->d_patch_info,
                    c->d_patch_w64, c->d_patch_wcol, c->d_patch_wrow, c->d_patch_zs};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

}  // namespace

int pcg_prepare(sgmas_context* c, const sgmas_bcoo* A, const PcgRunCfg& cfg);
int pcg_read_state(sgmas_context* c, PcgState* h);

extern "C" {

int sgmas_create(const sgmas_config* cfg, sgmas_context** out) {
    if (!out) return SGMAS_ERR_ARG;
    *out = nullptr;
    sgmas_config def = {0, 16, SGMAS_MAS_FP32};
    if (!cfg) cfg = &def;
    if (cfg->bank_size != 16 && cfg->bank_size != 32) return SGMAS_ERR_ARG;
    if (cfg->mas_precision < 0 || cfg->mas_precision > 3) return SGMAS_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SGMAS_ERR_CUDA;
    if (cfg->device < 0 || cfg->device >= ndev) return SGMAS_ERR_ARG;
    sgmas_context* c = new sgmas_context();
    c->device = cfg->device;
    c->bank = cfg->bank_size;
    c->precision = cfg->mas_precision;
    if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess || cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) {
        delete c;
        return SGMAS_ERR_CUDA;
    }
    c->stream = c->cap_stream;
    *out = c;
    return SGMAS_OK;
}

void sgmas_destroy(sgmas_context* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev2) cudaEventDestroy(c->ev2);
    free_all(c);
    mlp_free(c);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    if (c->rec_stream) cudaStreamDestroy(c->rec_stream);
    delete c;
}

const char* sgmas_last_error(const sgmas_context* c) { return c ? c->err.c_str() : g_host_err.c_str(); }

int sgmas_set_stream(sgmas_context* c, void* stream) {
    if (!c) return SGMAS_ERR_ARG;
    c->stream = (cudaStream_t)stream;  // NULL is the legacy default stream, as in the CUDA runtime
    return SGMAS_OK;
}

int sgmas_synchronize(sgmas_context* c) {
    if (!c) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_device_error(c, "synchronize");
}

int sgmas_mas_init(sgmas_context* c, int vert_num, int collision_node_offset, int nb_size, const unsigned* nb_list,
                   const unsigned* nb_start, const unsigned* nb_num, const int* part_map, int part_map_size,
                   const int* real_map) {
    if (!c) return SGMAS_ERR_ARG;
    if (vert_num < 1 || part_map_size < vert_num || part_map_size % c->bank || nb_size < 0 || !nb_start || !nb_num ||
        !part_map || !real_map || (nb_size > 0 && !nb_list))
        return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_mas_init: bad sizes (vert_num %d, part_map_size %d, bank %d)",
                        vert_num, part_map_size, c->bank);
    // host-side validation of the slot maps and the CSR
    for (int s = 0; s < part_map_size; ++s)
        if (part_map[s] >= vert_num || part_map[s] < -1)
            return ctx_fail(c, SGMAS_ERR_ARG, "part_map[%d] = %d out of range", s, part_map[s]);
    for (int v = 0; v < vert_num; ++v) {
        if (real_map[v] < 0 || real_map[v] >= part_map_size || part_map[real_map[v]] != v)
            return ctx_fail(c, SGMAS_ERR_ARG, "real_map[%d] = %d is not the inverse of part_map", v, real_map[v]);
        if ((long long)nb_start[v] + nb_num[v] > nb_size)
            return ctx_fail(c, SGMAS_ERR_ARG, "neighbour CSR row %d exceeds the list", v);
    }
    for (int i = 0; i < nb_size; ++i)
        if (nb_list[i] >= (unsigned)vert_num) return ctx_fail(c, SGMAS_ERR_ARG, "neighbour %d out of range", i);
    SG_CUDA(c, cudaSetDevice(c->device));
    c->N = vert_num;
    c->Mm = part_map_size;
    c->node_offset = collision_node_offset;
    c->nb_size = nb_size;
    c->L = num_levels(part_map_size > vert_num ? part_map_size : vert_num, c->bank);
    const int N = vert_num, B = c->bank;
    c->gn_cap = round_up(part_map_size, B) + (c->L + 1) * (N + B);
    if (ctx_alloc(c, &c->d_nb_list0, nb_size) || ctx_alloc(c, &c->d_nb_list, nb_size) ||
        ctx_alloc(c, &c->d_nb_num0, N) || ctx_alloc(c, &c->d_nb_num, N) || ctx_alloc(c, &c->d_nb_start, N) ||
        ctx_alloc(c, &c->d_part_map, part_map_size) || ctx_alloc(c, &c->d_real_map, N) ||
        ctx_alloc(c, &c->d_fine_mask, N) || ctx_alloc(c, &c->d_next_mask, N) ||
        ctx_alloc(c, &c->d_prefix_orig, part_map_size / B) || ctx_alloc(c, &c->d_bank_cnt, part_map_size / B + N / B + 2) ||
        ctx_alloc(c, &c->d_bank_pre, part_map_size / B + N / B + 2) || ctx_alloc(c, &c->d_coarse_space, (size_t)N * c->L) ||
        ctx_alloc(c, &c->d_going_next, c->gn_cap) || ctx_alloc(c, &c->d_level_size, 2 * (kMaxLevels + 2)) ||
        ctx_alloc(c, &c->d_coarse_table, (size_t)kMaxLevels * N) || ctx_alloc(c, &c->d_coarse_ticket, 1))
        return SGMAS_ERR_CUDA;
    SG_CUDA(c, cudaMemsetAsync(c->d_coarse_ticket, 0, sizeof(unsigned), c->stream));
    cudaStream_t s = c->stream;
    if (nb_size > 0) SG_CUDA(c, cudaMemcpyAsync(c->d_nb_list0, nb_list, sizeof(unsigned) * nb_size, cudaMemcpyHostToDevice, s));
    SG_CUDA(c, cudaMemcpyAsync(c->d_nb_num0, nb_num, sizeof(unsigned) * N, cudaMemcpyHostToDevice, s));
    SG_CUDA(c, cudaMemcpyAsync(c->d_nb_start, nb_start, sizeof(unsigned) * N, cudaMemcpyHostToDevice, s));
    SG_CUDA(c, cudaMemcpyAsync(c->d_part_map, part_map, sizeof(int) * part_map_size, cudaMemcpyHostToDevice, s));
    SG_CUDA(c, cudaMemcpyAsync(c->d_real_map, real_map, sizeof(int) * N, cudaMemcpyHostToDevice, s));
    SG_CUDA(c, cudaMemsetAsync(c->d_going_next, 0, sizeof(int) * c->gn_cap, s));
    SG_CUDA(c, cudaMemsetAsync(c->d_coarse_space, 0, sizeof(int) * (size_t)N * c->L, s));
    // initPreconditioner_Matrix: ReorderRealtime(0) sizes the matrices (x1.05)
    const int saved_cp = c->cp_num;
    c->cp_num = 0;
    int rc = mas_build_hierarchy(c);
    c->cp_num = saved_cp;
    if (rc) return rc;
    rc = alloc_mas_matrices(c, c->total);
    if (rc) return rc;
    c->mas_init = true;
    c->mas_assembled = false;
    return SGMAS_OK;
}

int sgmas_mas_set_contacts(sgmas_context* c, const int* d_pairs, int cp_num) {
    if (!c || cp_num < 0 || (cp_num > 0 && !d_pairs)) return SGMAS_ERR_ARG;
    c->d_pairs = d_pairs;
    c->cp_num = cp_num;
    return SGMAS_OK;
}

static int mas_assemble_impl(sgmas_context* c, const double* vals, const int* rows, const int* cols,
                             const uint32_t* indices, int offset, int n, int cp_num) {
    if (!c->mas_init) return ctx_fail(c, SGMAS_ERR_STATE, "MAS used before sgmas_mas_init");
    if (n < 0 || (n > 0 && (!vals || !rows || !cols))) return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_mas_assemble: bad matrix");
    if (cp_num < 0 || (cp_num > 0 && !c->d_pairs))
        return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_mas_assemble: %d contacts but no pair buffer", cp_num);
    c->cp_num = cp_num;
    int rc = mas_build_hierarchy(c);
    if (rc) return rc;
    if (c->total > c->cap_total) {
        rc = alloc_mas_matrices(c, c->total);
        if (rc) return rc;
    } else {
        // padding nodes of a rebuilt hierarchy must hold finite values: they
        // meet exact zeros of the inverses in the Schwarz products
        SG_CUDA(c, cudaMemsetAsync(c->d_R, 0, 3 * (size_t)c->total * acc_size(c->precision), c->stream));
    }
    rc = mas_scatter_and_invert(c, vals, rows, cols, indices, offset, n);
    if (rc) return rc;
    c->mas_assembled = true;
    return SGMAS_OK;
}

int sgmas_mas_assemble(sgmas_context* c, const double* d_values, const int* d_rows, const int* d_cols,
                       const uint32_t* d_indices, int offset, int triplet_num, int cp_num) {
    if (!c) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    int rc = mas_assemble_impl(c, d_values, d_rows, d_cols, d_indices, offset, triplet_num, cp_num);
    if (rc) return rc;
    return check_device_error(c, "sgmas_mas_assemble");
}

int sgmas_mas_apply(sgmas_context* c, const double* d_r, double* d_z) {
    if (!c || !d_r || !d_z) return SGMAS_ERR_ARG;
    if (!c->mas_assembled) return ctx_fail(c, SGMAS_ERR_STATE, "sgmas_mas_apply before sgmas_mas_assemble");
    SG_CUDA(c, cudaSetDevice(c->device));
    const ExtraRows none = {0, 0, c->N, 0, nullptr};
    return mas_launch_apply(c, d_r, d_z, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, 0ull, nullptr,
                            none);
}

int sgmas_mas_info(sgmas_context* c, int* levelnum, int* total_clusters, int* n_mas_blocks) {
    if (!c) return SGMAS_ERR_ARG;
    if (levelnum) *levelnum = c->L;
    if (total_clusters) *total_clusters = c->total;
    if (n_mas_blocks) *n_mas_blocks = c->total / c->bank;
    return SGMAS_OK;
}

int sgmas_mas_download_tables(sgmas_context* c, unsigned* fine_mask, int* coarse_space, int* going_next,
                              int going_next_cap, int* level_size, int* prefix_orig, int* coarse_table) {
    if (!c) return SGMAS_ERR_ARG;
    if (!c->mas_init) return ctx_fail(c, SGMAS_ERR_STATE, "no MAS");
    SG_CUDA(c, cudaStreamSynchronize(c->stream));
    const int N = c->N;
    if (fine_mask) SG_CUDA(c, cudaMemcpy(fine_mask, c->d_fine_mask, sizeof(unsigned) * N, cudaMemcpyDeviceToHost));
    if (coarse_space) SG_CUDA(c, cudaMemcpy(coarse_space, c->d_coarse_space, sizeof(int) * (size_t)N * c->L, cudaMemcpyDeviceToHost));
    if (going_next) {
        const int n = going_next_cap < c->gn_cap ? going_next_cap : c->gn_cap;
        SG_CUDA(c, cudaMemcpy(going_next, c->d_going_next, sizeof(int) * n, cudaMemcpyDeviceToHost));
    }
    if (level_size) SG_CUDA(c, cudaMemcpy(level_size, c->d_level_size, sizeof(int) * 2 * (c->L + 1), cudaMemcpyDeviceToHost));
    if (prefix_orig) SG_CUDA(c, cudaMemcpy(prefix_orig, c->d_prefix_orig, sizeof(int) * (c->Mm / c->bank), cudaMemcpyDeviceToHost));
    if (coarse_table) SG_CUDA(c, cudaMemcpy(coarse_table, c->d_coarse_table, sizeof(int) * (size_t)kMaxLevels * N, cudaMemcpyDeviceToHost));
    return SGMAS_OK;
}

int sgmas_mas_download_matrices(sgmas_context* c, double* hess64, double* inv_as_double) {
    if (!c) return SGMAS_ERR_ARG;
    if (!c->mas_assembled) return ctx_fail(c, SGMAS_ERR_STATE, "no assembled MAS");
    SG_CUDA(c, cudaStreamSynchronize(c->stream));
    const size_t bs = (size_t)c->bank * (c->bank + 1) / 2;
    const size_t nval = (size_t)(c->total / c->bank) * bs * 9;
    if (hess64) SG_CUDA(c, cudaMemcpy(hess64, c->d_hess, sizeof(double) * nval, cudaMemcpyDeviceToHost));
    if (inv_as_double) {
        const size_t es = store_size(c->precision);
        std::vector<unsigned char> raw(nval * es);
        SG_CUDA(c, cudaMemcpy(raw.data(), c->d_inv, nval * es, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < nval; ++i) {
            if (es == 8) { double v; memcpy(&v, &raw[i * 8], 8); inv_as_double[i] = v; }
            else if (es == 4) { float v; memcpy(&v, &raw[i * 4], 4); inv_as_double[i] = v; }
            else {
                uint16_t h; memcpy(&h, &raw[i * 2], 2);
                uint32_t u = (uint32_t)h << 16; float v; memcpy(&v, &u, 4); inv_as_double[i] = v;
            }
        }
    }
    return SGMAS_OK;
}

int sgmas_mas_invert_host(sgmas_context* c, const double* hess64, int nblocks, double* inv64) {
    if (!c || !hess64 || !inv64 || nblocks < 1) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    const size_t bs = (size_t)c->bank * (c->bank + 1) / 2;
    const size_t nval = (size_t)nblocks * bs * 9;
    double *d_in = nullptr, *d_out = nullptr;
    SG_CUDA(c, cudaMalloc(&d_in, nval * 8));
    SG_CUDA(c, cudaMalloc(&d_out, nval * 8));
    cudaMemcpy(d_in, hess64, nval * 8, cudaMemcpyHostToDevice);
    int rc = mas_invert_blocks_dev(c, d_in, nblocks, d_out);
    if (rc == 0) {
        cudaStreamSynchronize(c->stream);
        if (cudaMemcpy(inv64, d_out, nval * 8, cudaMemcpyDeviceToHost) != cudaSuccess) rc = SGMAS_ERR_CUDA;
    }
    cudaFree(d_in);
    cudaFree(d_out);
    return rc;
}

int sgmas_pcg_solve(sgmas_context* c, const sgmas_bcoo* A, const double* d_b, double* d_x,
                    const sgmas_pcg_config* cfg, sgmas_pcg_report* report) {
    if (!c || !A || !d_b || !d_x || !cfg) return SGMAS_ERR_ARG;
    if (A->n_block_rows < 1 || A->n_blocks < 0 || (A->n_blocks > 0 && (!A->d_values || !A->d_rows || !A->d_cols)))
        return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_pcg_solve: bad matrix");
    if (cfg->preconditioner != 0 && cfg->preconditioner != 1)
        return ctx_fail(c, SGMAS_ERR_ARG, "preconditioner must be 0 (block-Jacobi) or 1 (MAS)");
    if (cfg->rel_tol < 0 || cfg->abs_tol < 0 || cfg->max_iter < 0 || cfg->abd_bodies < 0 ||
        4LL * cfg->abd_bodies > A->n_block_rows)
        return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_pcg_solve: bad configuration");
    if (cfg->preconditioner == 1) {
        if (!c->mas_init) return ctx_fail(c, SGMAS_ERR_STATE, "MAS preconditioner requested before sgmas_mas_init");
        // bodies first (rows 0 .. 4 bodies), the MAS's N vertices at fem_offset (global_linear_system.cu:509-522)
        if (cfg->fem_offset < 4 * cfg->abd_bodies || cfg->fem_offset + c->N > A->n_block_rows)
            return ctx_fail(c, SGMAS_ERR_ARG,
                            "MAS range [fem_offset, fem_offset + N) must follow the body rows and fit the system "
                            "(N=%d, rows=%d, offset=%d, bodies=%d)",
                            c->N, A->n_block_rows, cfg->fem_offset, cfg->abd_bodies);
    }
    SG_CUDA(c, cudaSetDevice(c->device));
    PcgRunCfg rc_cfg = {};
    rc_cfg.max_iter = cfg->max_iter;
    rc_cfg.rel_tol = cfg->rel_tol;
    rc_cfg.abs_tol = cfg->abs_tol;
    rc_cfg.use_prec_norm = cfg->use_preconditioned_norm;
    rc_cfg.precond = cfg->preconditioner;
    rc_cfg.abd_bodies = cfg->abd_bodies;
    rc_cfg.fem_offset = cfg->fem_offset;
    rc_cfg.check_every = cfg->check_every > 0 ? cfg->check_every : 10;
    if (cfg->initial_guess != 0 && cfg->initial_guess != 1)
        return ctx_fail(c, SGMAS_ERR_ARG, "initial_guess must be 0 (x0 = 0) or 1 (x holds the start guess)");
    rc_cfg.warm = cfg->initial_guess;
    if (cfg->body_patches != 0 && cfg->body_patches != 1)
        return ctx_fail(c, SGMAS_ERR_ARG, "body_patches must be 0 or 1");
    if (cfg->body_patches && (cfg->preconditioner != 1 || cfg->abd_bodies < 1))
        return ctx_fail(c, SGMAS_ERR_ARG, "body_patches needs the MAS preconditioner and abd_bodies > 0");
    rc_cfg.patches = cfg->body_patches;
    if (!c->ev0) {
        SG_CUDA(c, cudaEventCreate(&c->ev0));
        SG_CUDA(c, cudaEventCreate(&c->ev1));
        SG_CUDA(c, cudaEventCreate(&c->ev2));
    }
    SG_CUDA(c, cudaEventRecord(c->ev2, c->stream));
    c->build_launches = 0;
    int rc = pcg_prepare(c, A, rc_cfg);
    if (rc) return rc;
    if (rc_cfg.precond == 1) {
        rc = mas_assemble_impl(c, A->d_values, A->d_rows, A->d_cols, nullptr, rc_cfg.fem_offset, A->n_blocks,
                               c->cp_num);
        if (rc) return rc;
    }
    float solve_ms = 0.f;
    int launches = 0;
    SG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    float prep_ms = 0.f;
    rc = c->persistent ? pcg_run_persistent(c, d_b, d_x, rc_cfg, &solve_ms, &launches) : 1;
    if (rc == 1 && rc_cfg.patches)
        return ctx_fail(c, SGMAS_ERR_STATE, "body patches run in the persistent form only, which %s",
                        c->persistent ? "does not fit this system" : "is switched off (sgmas_set_pcg_mode)");
    if (rc == 1) rc = pcg_run(c, d_b, d_x, rc_cfg, &solve_ms, &launches);  // graph path
    if (rc) return rc;
    cudaEventElapsedTime(&prep_ms, c->ev2, c->ev0);
    rc = check_device_error(c, "sgmas_pcg_solve");
    if (rc) return rc;
    PcgState h;
    rc = pcg_read_state(c, &h);
    if (rc) return rc;
    if (report) {
        report->iterations = h.iters;
        report->converged = h.converged;
        report->rz0 = h.rz0;
        report->rr0 = h.rr0;
        report->rr_last = h.rr;
        report->solve_ms = solve_ms;
        report->precond_ms = prep_ms;
        report->kernel_launches = launches;
        report->build_launches = c->build_launches;
        report->x0_rejected = rc_cfg.warm ? h.w_reject : 0;
        report->x0_scale = rc_cfg.warm ? h.w_alpha : 0.0;
        report->rr_x0 = rc_cfg.warm ? h.w_rr : 0.0;
        report->bb = rc_cfg.warm ? h.w_bb : h.rr0;
    }
    if (h.breakdown)
        return ctx_fail(c, SGMAS_ERR_NUMERIC,
                        "CG breakdown at iteration %d: p.A p <= 0 with r != 0 (the matrix or the preconditioner "
                        "is not positive definite)", h.iters);
    if (!(h.rz == h.rz) || !(h.rr == h.rr)) return ctx_fail(c, SGMAS_ERR_NUMERIC, "non-finite residual in PCG");
    return SGMAS_OK;
}

int sgmas_set_wait_limit(sgmas_context* c, int spin_limit, int phantom_arrivals) {
    if (!c) return SGMAS_ERR_ARG;
    if (spin_limit < 0 || phantom_arrivals < 0)
        return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_set_wait_limit: spin_limit and phantom_arrivals must be >= 0");
    c->wait_limit = spin_limit > 0 ? spin_limit : kSpinLimit;
    c->phantom_arrivals = phantom_arrivals;
    return SGMAS_OK;
}

int sgmas_pcg_solve_host(sgmas_context* c, const double* values, const int* rows, const int* cols, int n_blocks,
                         int n_block_rows, const double* b, double* x, const sgmas_pcg_config* cfg,
                         sgmas_pcg_report* report) {
    if (!c || !values || !rows || !cols || !b || !x || n_blocks < 1 || n_block_rows < 1) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    if (n_blocks > c->hcap_blocks) {
        if (ctx_alloc(c, &c->d_hvals, 9 * (size_t)n_blocks) || ctx_alloc(c, &c->d_hrows, n_blocks) ||
            ctx_alloc(c, &c->d_hcols, n_blocks))
            return SGMAS_ERR_CUDA;
        c->hcap_blocks = n_blocks;
    }
    if (n_block_rows > c->hcap_vec) {
        if (ctx_alloc(c, &c->d_hb, 3 * (size_t)n_block_rows) || ctx_alloc(c, &c->d_hx, 3 * (size_t)n_block_rows))
            return SGMAS_ERR_CUDA;
        c->hcap_vec = n_block_rows;
    }
    cudaStream_t s = c->stream;
    SG_CUDA(c, cudaMemcpyAsync(c->d_hvals, values, sizeof(double) * 9 * n_blocks, cudaMemcpyHostToDevice, s));
    SG_CUDA(c, cudaMemcpyAsync(c->d_hrows, rows, sizeof(int) * n_blocks, cudaMemcpyHostToDevice, s));
    SG_CUDA(c, cudaMemcpyAsync(c->d_hcols, cols, sizeof(int) * n_blocks, cudaMemcpyHostToDevice, s));
    SG_CUDA(c, cudaMemcpyAsync(c->d_hb, b, sizeof(double) * 3 * n_block_rows, cudaMemcpyHostToDevice, s));
    if (cfg && cfg->initial_guess == 1)  // x carries the start guess in
        SG_CUDA(c, cudaMemcpyAsync(c->d_hx, x, sizeof(double) * 3 * n_block_rows, cudaMemcpyHostToDevice, s));
    sgmas_bcoo A = {c->d_hvals, c->d_hrows, c->d_hcols, n_blocks, n_block_rows};
    int rc = sgmas_pcg_solve(c, &A, c->d_hb, c->d_hx, cfg, report);
    if (rc) return rc;
    SG_CUDA(c, cudaMemcpyAsync(x, c->d_hx, sizeof(double) * 3 * n_block_rows, cudaMemcpyDeviceToHost, s));
    SG_CUDA(c, cudaStreamSynchronize(s));
    return SGMAS_OK;
}

int sgmas_spmv(sgmas_context* c, double a, const sgmas_bcoo* A, const double* d_x, double b, double* d_y) {
    if (!c || !A || !d_x || !d_y || A->n_block_rows < 1) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    return bcoo_spmv_ref(c, a, A->d_values, A->d_rows, A->d_cols, A->n_blocks, A->n_block_rows, d_x, b, d_y);
}

int sgmas_convert(sgmas_context* c, const double* d_values, const int* d_rows, const int* d_cols, int n,
                  double* d_out_values, int* d_out_rows, int* d_out_cols, int* n_unique) {
    if (!c || n < 0 || !n_unique || (n > 0 && (!d_values || !d_rows || !d_cols || !d_out_values || !d_out_rows || !d_out_cols)))
        return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    int rc = convert_triplets(c, d_values, d_rows, d_cols, n, d_out_values, d_out_rows, d_out_cols, n_unique);
    if (rc) return rc;
    return check_device_error(c, "sgmas_convert");
}

int sgmas_assembly_plan(sgmas_context* c, const int* d_rows, const int* d_cols, int n, int* d_out_rows,
                        int* d_out_cols, int* n_unique) {
    if (!c || n < 0 || !n_unique || (n > 0 && (!d_rows || !d_cols || !d_out_rows || !d_out_cols)))
        return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    int rc = assembly_plan(c, d_rows, d_cols, n, d_out_rows, d_out_cols, n_unique);
    if (rc) return rc;
    return check_device_error(c, "sgmas_assembly_plan");
}

int sgmas_assemble(sgmas_context* c, const double* d_values, int n, double* d_out_values) {
    if (!c || n < 0 || (n > 0 && (!d_values || !d_out_values))) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    return assemble_planned(c, d_values, n, d_out_values);
}

int sgmas_append_triplets(sgmas_context* c, const double* d_base_values, const int* d_base_rows,
                          const int* d_base_cols, int n_base, const double* d_values, const int* d_rows,
                          const int* d_cols, int n, double* d_out_values, int* d_out_rows, int* d_out_cols,
                          int* n_out) {
    if (!c || !n_out || n_base < 0 || n < 0) return SGMAS_ERR_ARG;
    if ((n_base > 0 && (!d_base_values || !d_base_rows || !d_base_cols)) || (n > 0 && (!d_values || !d_rows || !d_cols)) ||
        (n_base + n > 0 && (!d_out_values || !d_out_rows || !d_out_cols)))
        return SGMAS_ERR_ARG;
    if ((long long)n_base + n > INT_MAX) return ctx_fail(c, SGMAS_ERR_ARG, "sgmas_append_triplets: more than 2^31 - 1 blocks");
    SG_CUDA(c, cudaSetDevice(c->device));
    int rc = append_triplets(c, d_base_values, d_base_rows, d_base_cols, n_base, d_values, d_rows, d_cols, n,
                             d_out_values, d_out_rows, d_out_cols, n_out);
    if (rc) return rc;
    return check_device_error(c, "sgmas_append_triplets");
}

int sgmas_element_plan(sgmas_context* c, const sgmas_element_group* groups, int n_groups, int* d_out_rows,
                       int* d_out_cols, int* n_unique) {
    if (!c || !n_unique || n_groups < 1 || n_groups > 4 || !groups) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    int rc = element_plan(c, groups, n_groups, d_out_rows, d_out_cols, n_unique);
    if (rc) return rc;
    return check_device_error(c, "sgmas_element_plan");
}

int sgmas_element_assemble(sgmas_context* c, const sgmas_element_group* groups, int n_groups,
                           double* d_out_values) {
    if (!c || n_groups < 1 || n_groups > 4 || !groups) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    return element_assemble(c, groups, n_groups, d_out_values);
}

int sgmas_write_upper_blocks(sgmas_context* c, const double* d_H, int n_elem, int k, const int* d_nodes,
                             double* d_values, int* d_rows, int* d_cols) {
    if (!c || n_elem < 0 || k < 1 || k > 4 || (n_elem > 0 && (!d_H || !d_nodes || !d_values || !d_rows || !d_cols)))
        return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    return write_upper_blocks(c, d_H, n_elem, k, d_nodes, d_values, d_rows, d_cols);
}

int sgmas_morton_codes(sgmas_context* c, const double* d_pos, int n, const double* aabb, uint64_t* d_codes) {
    if (!c || n < 0 || (n > 0 && (!d_pos || !d_codes))) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    return morton_codes(c, d_pos, n, aabb, d_codes);
}

int sgmas_morton_partition(sgmas_context* c, const double* d_pos, int n, int* part_map, int part_map_cap,
                           int* part_map_size, int* real_map) {
    if (!c || n < 1 || !d_pos || !part_map || !part_map_size || !real_map) return SGMAS_ERR_ARG;
    const int B = c->bank;
    const int size = round_up(n, B);
    if (part_map_cap < size) return ctx_fail(c, SGMAS_ERR_CAPACITY, "part_map needs %d entries", size);
    SG_CUDA(c, cudaSetDevice(c->device));
    uint64_t* d_codes = nullptr;
    SG_CUDA(c, cudaMalloc(&d_codes, sizeof(uint64_t) * n));
    // the low 32 bits of each code are the vertex index, so the sorted codes
    // are the Morton order (ties broken by index, as a stable sort would)
    int rc = morton_codes(c, d_pos, n, nullptr, d_codes);
    if (!rc) rc = sort_u64_pairs(c, d_codes, nullptr, n, 64);
    std::vector<uint64_t> sorted(n);
    std::vector<uint32_t> order(n);
    if (!rc) {
        cudaStreamSynchronize(c->stream);
        if (cudaMemcpy(sorted.data(), d_codes, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost) != cudaSuccess) rc = SGMAS_ERR_CUDA;
        for (int s = 0; s < n; ++s) order[s] = (uint32_t)(sorted[s] & 0xffffffffu);
    }
    cudaFree(d_codes);
    if (rc) return rc;
    for (int s = 0; s < size; ++s) part_map[s] = s < n ? (int)order[s] : -1;
    for (int s = 0; s < n; ++s) real_map[order[s]] = s;
    *part_map_size = size;
    return SGMAS_OK;
}

int sgmas_pcg_last_vectors(sgmas_context* c, double* d_r, double* d_z) {
    if (!c) return SGMAS_ERR_ARG;
    if (!c->last_cfg.valid) return ctx_fail(c, SGMAS_ERR_STATE, "sgmas_pcg_last_vectors needs a completed solve");
    SG_CUDA(c, cudaSetDevice(c->device));
    const size_t bytes = sizeof(double) * 3 * (size_t)c->bsr.nrows;
    if (d_r) SG_CUDA(c, cudaMemcpyAsync(d_r, c->d_r, bytes, cudaMemcpyDeviceToDevice, c->stream));
    if (d_z) SG_CUDA(c, cudaMemcpyAsync(d_z, c->d_z, bytes, cudaMemcpyDeviceToDevice, c->stream));
    return SGMAS_OK;
}

int sgmas_set_pcg_mode(sgmas_context* c, int mode) {
    if (!c || (mode != SGMAS_PCG_GRAPH && mode != SGMAS_PCG_PERSISTENT)) return SGMAS_ERR_ARG;
    c->persistent = mode == SGMAS_PCG_PERSISTENT;
    return SGMAS_OK;
}

int sgmas_set_pcg_ctas(sgmas_context* c, int max_ctas) {
    if (!c) return SGMAS_ERR_ARG;
    if (max_ctas < 0) return ctx_fail(c, SGMAS_ERR_ARG, "max_ctas must be >= 0 (0: one CTA per SM)");
    c->pcg_ctas = max_ctas;
    return SGMAS_OK;
}

int sgmas_pcg_profile(sgmas_context* c, int reps, float* ms, int n_ms) {
    if (!c || reps < 1 || !ms || n_ms < 1) return SGMAS_ERR_ARG;
    SG_CUDA(c, cudaSetDevice(c->device));
    return pcg_profile(c, reps, ms, n_ms);
}

// getVertNeighbors (SG/load_mesh.cpp:894-999): the first-inserted orientation
// of every undirected edge, iterated in (first, second) order.
int sgmas_vert_neighbors(const int* tets, int n_tets, const int* tris, int n_tris, int n_verts, int abd_vert_offset,
                         unsigned* nb_start, unsigned* nb_num, unsigned* nb_list, int nb_cap) {
    if (n_verts < 1 || n_tets < 0 || n_tris < 0 || (n_tets > 0 && !tets) || (n_tris > 0 && !tris) || !nb_start ||
        !nb_num || (nb_cap > 0 && !nb_list))
        return SGMAS_ERR_ARG;
    struct E { uint64_t a, b; int64_t seq; };
    std::vector<E> e;
    e.reserve(6 * (size_t)n_tets + 9 * (size_t)n_tris);
    static const int tp[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    for (int t = 0; t < n_tets; ++t)
        for (int k = 0; k < 6; ++k)
            e.push_back({(uint64_t)(uint32_t)tets[4 * t + tp[k][0]], (uint64_t)(uint32_t)tets[4 * t + tp[k][1]],
                         (int64_t)e.size()});
    for (int t = 0; t < n_tris; ++t)
        for (int rep = 0; rep < 3; ++rep) {  // the reference repeats the same three edges three times
            const uint64_t x = (uint32_t)tris[3 * t], y = (uint32_t)tris[3 * t + 1], z = (uint32_t)tris[3 * t + 2];
            e.push_back({x, y, (int64_t)e.size()});
            e.push_back({y, z, (int64_t)e.size()});
            e.push_back({z, x, (int64_t)e.size()});
        }
    auto lo = [](const E& q) { return q.a < q.b ? q.a : q.b; };
    auto hi = [](const E& q) { return q.a < q.b ? q.b : q.a; };
    std::sort(e.begin(), e.end(), [&](const E& p, const E& q) {
        if (lo(p) != lo(q)) return lo(p) < lo(q);
        if (hi(p) != hi(q)) return hi(p) < hi(q);
        return p.seq < q.seq;
    });
    std::vector<E> u;
    u.reserve(e.size());
    for (size_t i = 0; i < e.size(); ++i)
        if (u.empty() || lo(u.back()) != lo(e[i]) || hi(u.back()) != hi(e[i])) u.push_back(e[i]);
    std::sort(u.begin(), u.end(), [](const E& p, const E& q) { return p.a != q.a ? p.a < q.a : p.b < q.b; });
    for (int i = 0; i < n_verts; ++i) nb_num[i] = 0;
    for (const E& q : u) {
        const int64_t f = (int64_t)q.a - abd_vert_offset, s = (int64_t)q.b - abd_vert_offset;
        if (f < 0 || f >= n_verts || s < 0 || s >= n_verts) return SGMAS_ERR_ARG;
        nb_num[f]++;
        nb_num[s]++;
    }
    unsigned off = 0;
    for (int i = 0; i < n_verts; ++i) {
        nb_start[i] = off;
        off += nb_num[i];
    }
    if ((long long)off > nb_cap) return SGMAS_ERR_CAPACITY;
    std::vector<unsigned> fill(n_verts, 0u);
    for (const E& q : u) {
        const int64_t f = (int64_t)q.a - abd_vert_offset, s = (int64_t)q.b - abd_vert_offset;
        nb_list[nb_start[f] + fill[f]++] = (unsigned)s;
        nb_list[nb_start[s] + fill[s]++] = (unsigned)f;
    }
    return (int)off;
}

// setMAS_partition (SG/main.cu:47-75); part_offset = last part id + 1 as
// load_parts sets it.  Where the reference would write past a bank or leave
// real_map entries unset, this returns SGMAS_ERR_ARG instead.
int sgmas_part_maps(const int* part_id, int n, int bank, int* part_map, int part_map_cap, int* part_map_size,
                    int* real_map) {
    if (!part_id || n < 1 || (bank != 16 && bank != 32) || !part_map || !part_map_size || !real_map)
        return SGMAS_ERR_ARG;
    const int part_offset = part_id[n - 1] + 1;
    const long long size = (long long)part_offset * bank;
    if (part_offset < 1) return SGMAS_ERR_ARG;
    if (size > part_map_cap) return SGMAS_ERR_CAPACITY;
    for (long long i = 0; i < size; ++i) part_map[i] = -1;
    int index = 0;
    for (int i = 0; i < n; ++i) {
        if (part_id[i] < 0 || part_id[i] >= part_offset || index >= bank) return SGMAS_ERR_ARG;
        part_map[(long long)bank * part_id[i] + index] = i;
        ++index;
        if (i <= n - 2 && part_id[i + 1] != part_id[i]) index = 0;
    }
    index = 0;
    for (long long i = 0; i < size; ++i)
        if (part_map[i] == index) real_map[index++] = (int)i;
    if (index != n) return SGMAS_ERR_ARG;
    *part_map_size = (int)size;
    return SGMAS_OK;
}

}  // extern "C"
