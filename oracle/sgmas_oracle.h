/*
 * sgmas_oracle.h -- CPU restatement of StiffGIPC's Newton-step linear solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in stiff-gipc_b200/: only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference legs load it.  The product
 * path never calls it and has no CPU fallback.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the StiffGIPC project root, "SG/" = StiffGIPC/).
 *
 * Parity status: the integer stages (slot maps, neighbour CSR, level masks,
 * cluster ids, goingNext, coarse tables, Morton codes, BCOO key order) are
 * defined exactly as the reference computes them.  The reference ships no
 * golden A/b/x vectors and its GPU code cannot be built here (it needs Eigen
 * in device code), so the floating-point stages are pinned by an FP64 direct
 * solve in the tests, not by reference outputs.
 */
#ifndef SGMAS_ORACLE_H
#define SGMAS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- setup: SG/main.cu:47-75, SG/load_mesh.cpp:449-480, 894-999 ---- */
int or_mas_partition(const int* part_id, int n, int bank, int* part_offset_out,
                     int* part_map, int part_map_cap, int* real_map);
int or_vert_neighbors(const int* tets, int ntet, const int* tris, int ntri,
                      int n_verts, int abd_vert_offset, unsigned* nb_start,
                      unsigned* nb_num, unsigned* nb_list, int nb_cap);
int or_num_levels(int max_nodes, int bank);

/* ---- Morton codes: SG/GIPC.cu:142-201, 412-461 ---- */
uint32_t or_hash_code(double x, double y, double z, double resolution);
void or_vert_morton(const double* pos, int n, uint64_t* out);

/* ---- symmetric BCOO SpMV, dots, block-Jacobi, converter ---- */
void or_spmv_sym(double a, const double* vals, const int* rows, const int* cols,
                 int nb, const double* x, double b, double* y, int ndof);
double or_dot(const double* a, const double* b, int n);
int or_convert(const double* vals, const int* rows, const int* cols, int n,
               double* out_vals, int* out_rows, int* out_cols);
void or_write_upper_blocks(const double* H, int nnode, const int* nodes,
                           double* vals, int* rows, int* cols);

/* ---- MAS preconditioner: SG/MASPreconditioner.cu ---- */
typedef struct or_mas or_mas;
or_mas* or_mas_create(int bank, int n_verts, int collision_node_offset,
                      const unsigned* nb_list, int nb_size,
                      const unsigned* nb_start, const unsigned* nb_num,
                      const int* part_map, int part_map_size,
                      const int* real_map);
void or_mas_destroy(or_mas* m);
int or_mas_reorder(or_mas* m, const int* pairs4, int cp_num);
int or_mas_levelnum(const or_mas* m);
int or_mas_total_clusters(const or_mas* m);
int or_mas_get_tables(const or_mas* m, unsigned* fine_mask, int* coarse_space,
                      int* going_next, int going_next_cap, int* level_size,
                      int* prefix_orig, int* coarse_table);
/* precision: 0 = FP32 inverses (reference), 1 = BF16 inverses / FP32 apply,
 *            2 = FP64 inverses / FP64 apply */
int or_mas_assemble(or_mas* m, const double* vals, const int* rows,
                    const int* cols, const uint32_t* indices, int offset,
                    int n, int precision);
int or_mas_get_matrices(const or_mas* m, double* hess64, double* inv64,
                        float* inv32);
int or_mas_set_hess(or_mas* m, const double* hess, int precision);
void or_mas_invert_blocks(const double* in, int nblocks, int bank, double* out64);
/* factored inverse W = L^-1 per subdomain (the library's BF16 / FP32-factored storage) */
int or_mas_factor_blocks(const double* in, int nblocks, int bank, double* out64);
int or_mas_apply(or_mas* m, const double* r, double* z);

/* ---- PCG: SG/linear_system/solver/pcg_solver.cu:155-304 ---- */
typedef struct {
    int max_iter;          /* 0 -> ndof */
    double rel_tol;
    double abs_tol;
    int use_preconditioned_norm;
    int precond;           /* 0 identity, 1 3x3 block-Jacobi, 2 MAS */
    int abd_bodies;        /* bodies whose 12x12 diagonal blocks are inverted */
    int fem_offset;        /* first FEM block row (MAS sub-range) */
    int nthreads;          /* OpenMP threads for the timed CPU arm (0 = all) */
    int initial_guess;     /* 1: x holds x0; scaled by x0.b / x0.A x0, rejected when it raises ||r||,
                              convergence against ||b|| (the library's start-guess rule) */
} or_pcg_cfg;

typedef struct {
    int iterations;
    double rel_residual;   /* ||b - Ax|| / ||b|| at exit, recomputed */
    double rz0, rr0;
    double ms;
    double x0_scale;       /* initial_guess: the scale applied to x0 */
    int x0_rejected;       /* initial_guess: 1 when x0 was rejected */
} or_pcg_report;

int or_pcg(const double* vals, const int* rows, const int* cols, int nb,
           int nrows, const double* b, double* x, const or_pcg_cfg* cfg,
           or_mas* mas, or_pcg_report* rep);

/* ---- helpers for tests ---- */
int or_bf16_round(const double* in, int n, float* out);
int or_omp_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
