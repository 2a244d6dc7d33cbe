/*
 * sgmas.h -- C-ABI of the B200-native MAS-PCG Newton-step solve.
 *
 * Drop-in boundary for StiffGIPC's linear solve (paths below are relative to
 * the StiffGIPC project; "SG/" = StiffGIPC/).  Every entry point returns
 * SGMAS_OK (0) or a negative status and never aborts; sgmas_last_error()
 * gives the message.  Device pointers ("d_") are borrowed for the duration of
 * the call (or until replaced, for contact pairs); the context owns its
 * internal arrays.  Calls on one context are stream-ordered on the context's
 * stream and are not re-entrant.
 *
 * Matrix layout (GIPCTripletMatrix, SG/linear_system/linear_system/
 * global_matrix.h:18-203): merged upper-triangular 3x3 block COO, sorted by
 * (row, col), row <= col, values 9 doubles column-major per block
 * (Eigen::Matrix3d), rows/cols int32 block indices.  Vectors are double[3n].
 */
#ifndef SGMAS_H
#define SGMAS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SGMAS_OK 0
#define SGMAS_ERR_ARG -1      /* invalid argument */
#define SGMAS_ERR_CUDA -2     /* CUDA runtime error */
#define SGMAS_ERR_STATE -3    /* call out of order (e.g. apply before assemble) */
#define SGMAS_ERR_CAPACITY -4 /* a size exceeds an allocated or stated maximum */
#define SGMAS_ERR_DEVICE -5   /* a kernel reported an error (bounded wait expired, bad index) */
#define SGMAS_ERR_NUMERIC -6  /* non-finite value in the solve */

typedef struct sgmas_context sgmas_context;

/* precision of the stored subdomain inverses and of the MAS apply */
#define SGMAS_MAS_FP32 0 /* reference parity: FP64 build, FP32 inverses and apply */
#define SGMAS_MAS_BF16 1 /* BF16 factored inverses (W = L^-1 of each subdomain's FP64 Cholesky
                            factor, z = W^T W r), FP32 accumulate: SPD for any rounding of W */
#define SGMAS_MAS_FP64 2 /* FP64 inverses and apply (plain FP64 MAS-PCG) */
#define SGMAS_MAS_FP32_FACTORED 3 /* FP32 factored inverses, FP32 accumulate */

typedef struct {
    int device;        /* CUDA device ordinal */
    int bank_size;     /* subdomain size; 16 = BANKSIZE (SG/eigen_data.h:17) */
    int mas_precision; /* SGMAS_MAS_* */
} sgmas_config;

/* gipc::PCGSolverConfig (SG/linear_system/solver/pcg_solver.h:6-15) plus the
 * preconditioner selection of GIPC::create_LinearSystem (SG/gipc/gipc.cu:42-73). */
typedef struct {
    int max_iter;                /* 0 -> number of DOF, as the reference */
    double rel_tol;
    double abs_tol;
    int use_preconditioned_norm; /* 1: r.z <= rel^2 r0.z0; 0: ||r||^2 <= rel^2 ||r0||^2 */
    int preconditioner;          /* 0: 3x3 block-Jacobi (P_type 0); 1: MAS (P_type 1) */
    int abd_bodies;              /* 12x12 block-Jacobi on block rows [0, 4*abd_bodies) */
    int fem_offset;              /* first FEM block row (MAS sub-range) */
    int check_every;             /* convergence-test cadence; 10 = reference (pcg_solver.cu:240,260) */
    int initial_guess;           /* 0: x0 = 0, r0 = b (reference, pcg_solver.cu:175).  1: d_x holds a start
                                    guess x0 (e.g. a learned warm start, sgmas_mlp_warm_start): the solve
                                    scales it by alpha = x0.b / x0.A x0 (0 unless positive), rejects it
                                    (x0 = 0) when ||b - alpha A x0|| > ||b||, and tests convergence
                                    against ||b|| instead of ||r0|| */
    int body_patches;            /* 0: the reference's composition (12x12 block-Jacobi on the bodies, MAS on the
                                    FEM range).  1 (needs preconditioner 1 and abd_bodies > 0, persistent form):
                                    each body's block is widened to a patch -- the body's 4 block rows plus the
                                    FEM vertices coupled to it (at most 64, the lowest ids; neighbouring patches
                                    overlap) -- factored densely in FP64 and stored as W = L^-1 in FP32 (FP64
                                    with the FP64 MAS); z = MAS(r) + sum of the patches' W^T W r.  For bodies
                                    resting on FEM surfaces with stiff barrier contact, where the body-FEM
                                    couplings dominate.  The library's own; no reference counterpart */
} sgmas_pcg_config;

typedef struct {
    int iterations;      /* value returned by PCGSolver::pcg (pcg_solver.cu:303) */
    int converged;
    double rz0, rr0;     /* initial r.z and r.r */
    double rr_last;      /* r.r at the last convergence test */
    float solve_ms;      /* device time of the PCG loop (CUDA events) */
    float precond_ms;    /* device time of the preconditioner build */
    int kernel_launches; /* kernels of the PCG loop (1 for the persistent form, graph nodes executed otherwise) */
    int build_launches;  /* kernels of the solve's set-up: block CSR, MAS hierarchy, scatter, inverses */
    int x0_rejected;     /* initial_guess = 1: 1 when the start guess was rejected (the solve began at 0) */
    double x0_scale;     /* initial_guess = 1: the scale alpha applied to the start guess */
    double rr_x0;        /* initial_guess = 1: ||b - alpha A x0||^2 before the rejection test */
    double bb;           /* initial_guess = 1: ||b||^2, the reference of the convergence test */
} sgmas_pcg_report;

/* One BCOO matrix on the device (borrowed). */
typedef struct {
    const double* d_values; /* [n_blocks][9], column-major 3x3 */
    const int* d_rows;
    const int* d_cols;
    int n_blocks;
    int n_block_rows;       /* block rows = DOF / 3 */
} sgmas_bcoo;

/* ---- MatrixMarket boundary (host only, no context, no GPU) --------------
 * The files GlobalLinearSystem::export_matrix_market_files writes
 * (SG/linear_system/linear_system/global_linear_system.cu:98-261): A as a
 * general coordinate real matrix with every stored block expanded to both
 * triangles ("%d %d %.17g", 1-based), b as an M x 1 real array.
 * sgmas_mtx_write writes exactly that from a host BCOO (values 9 doubles
 * column-major per upper block); path_b may be NULL.
 * sgmas_mtx_read reads such files (or symmetric ones) back into an upper,
 * (row, col)-sorted BCOO with duplicates summed in file order, as
 * read_mm_coordinate_real + to_upper_triangle_block_triplets do
 * (SG/main.cu:398-646); a missing diagonal block is an error.  It sets
 * *n_blocks / *n_block_rows first and returns SGMAS_ERR_CAPACITY (nothing
 * copied) when the arrays are NULL or too small: call once to size, once to
 * read.  path_b may be NULL.  Failures: sgmas_last_error(NULL). */
int sgmas_mtx_write(const char* path_A, const char* path_b, const double* values, const int* rows,
                    const int* cols, int n_blocks, int n_block_rows, const double* b);
int sgmas_mtx_read(const char* path_A, const char* path_b, double* values, int* rows, int* cols,
                   int cap_blocks, double* b, int cap_b, int* n_blocks, int* n_block_rows);

/* ---- context ---------------------------------------------------------- */
int sgmas_create(const sgmas_config* cfg, sgmas_context** out);
/* MASPreconditioner::FreeMAS (SG/MASPreconditioner.cu:2321-2350) + release */
void sgmas_destroy(sgmas_context* ctx);
const char* sgmas_last_error(const sgmas_context* ctx);  /* NULL: this thread's last context-free call */
/* the reference runs on the per-thread default stream (CMakeLists.txt:101);
 * a new context uses a stream of its own; NULL selects the legacy default
 * stream, as everywhere in the CUDA runtime */
int sgmas_set_stream(sgmas_context* ctx, void* cuda_stream);
int sgmas_synchronize(sgmas_context* ctx);

/* ---- MASPreconditioner (SG/MASPreconditioner.cuh:14-102) --------------- */
/* initPreconditioner_Neighbor (:2253-2290) + the uploads of the public
 * neighbour / slot-map arrays done by the caller at SG/main.cu:998-1027 +
 * initPreconditioner_Matrix (:2292-2319).  Host arrays; neighbour CSR as
 * tetrahedra_obj::getVertNeighbors (SG/load_mesh.cpp:894-999); slot maps as
 * setMAS_partition (SG/main.cu:47-75). */
int sgmas_mas_init(sgmas_context* ctx, int vert_num, int collision_node_offset,
                   int neighbor_list_size, const unsigned* neighbor_list,
                   const unsigned* neighbor_start, const unsigned* neighbor_num,
                   const int* part_map, int part_map_size, const int* real_map);
/* the int4 contact pairs the reference keeps as _collisonPairs (device, borrowed) */
int sgmas_mas_set_contacts(sgmas_context* ctx, const int* d_pairs_int4, int cp_num);
/* setPreconditioner_bcoo (:2169-2207): hierarchy rebuild + Hessian scatter +
 * dense subdomain inverses.  d_indices selects the FEM blocks: triplet_num
 * block indices into d_values / d_rows / d_cols, each below the BCOO's block
 * count (what calculate_subsystem_bcoo_indices, i_preconditioner.cu:32-72,
 * returns with its count).  NULL = every one of the triplet_num blocks whose
 * row and column lie in [offset, offset + vert_num). */
int sgmas_mas_assemble(sgmas_context* ctx, const double* d_values, const int* d_rows,
                       const int* d_cols, const uint32_t* d_indices, int offset,
                       int triplet_num, int cp_num);
/* preconditioning (:2210-2251): d_z = MAS(d_r) over the FEM range */
int sgmas_mas_apply(sgmas_context* ctx, const double* d_r, double* d_z);
int sgmas_mas_info(sgmas_context* ctx, int* levelnum, int* total_clusters, int* n_mas_blocks);
/* copies of the hierarchy tables (host arrays, any may be NULL): fine_mask[N],
 * coarse_space[levelnum*N], going_next[cap], level_size[2*(levelnum+1)],
 * prefix_orig[part_map_size/bank], coarse_table[6*N] */
int sgmas_mas_download_tables(sgmas_context* ctx, unsigned* fine_mask, int* coarse_space,
                              int* going_next, int going_next_cap, int* level_size,
                              int* prefix_orig, int* coarse_table);
/* assembled FP64 subdomain matrices and their inverses as stored
 * (float for FP32 / BF16 widened to float, double for FP64); host arrays of
 * n_mas_blocks * bank*(bank+1)/2 * 9 entries */
int sgmas_mas_download_matrices(sgmas_context* ctx, double* hess64, double* inv_as_double);
/* invert host FP64 packed subdomain matrices with the device kernel (tests) */
int sgmas_mas_invert_host(sgmas_context* ctx, const double* hess64, int nblocks, double* inv64);

/* ---- PCGSolver (SG/linear_system/solver/pcg_solver.cu:155-304) -------- */
/* x = 0 (or the start guess in d_x, cfg->initial_guess), then PCG on the device with device-side scalars; the whole loop is
 * one CUDA graph (conditional WHILE node).  Requires sgmas_mas_init (and
 * assembles the MAS itself) when cfg->preconditioner == 1. */
int sgmas_pcg_solve(sgmas_context* ctx, const sgmas_bcoo* A, const double* d_b, double* d_x,
                    const sgmas_pcg_config* cfg, sgmas_pcg_report* report);
/* How sgmas_pcg_solve runs the loop: SGMAS_PCG_PERSISTENT (default) = one
 * cooperative kernel, one CTA per SM, grid barriers between phases (falls
 * back to the graph form when the system's subdomain tiles do not fit in
 * shared memory); SGMAS_PCG_GRAPH = one kernel per phase in a CUDA graph with
 * a conditional WHILE node. */
/* Copy the residual r and the preconditioned residual z = M^-1 r of the last
 * iteration of the last sgmas_pcg_solve (PCGSolver's members r and z,
 * SG/linear_system/solver/pcg_solver.h:29-30) into d_r / d_z (3 * n_block_rows
 * doubles each; either may be NULL).  After a solve stopped by max_iter = 1, z
 * is M^-1 b.  sgmas_pcg_profile overwrites both. */
int sgmas_pcg_last_vectors(sgmas_context* ctx, double* d_r, double* d_z);
#define SGMAS_PCG_GRAPH 0
#define SGMAS_PCG_PERSISTENT 1
int sgmas_set_pcg_mode(sgmas_context* ctx, int mode);
/* At most max_ctas CTAs (one per SM) for the persistent form; 0 (default) =
 * every SM.  A small system solved on a few SMs leaves the rest to solves of
 * other contexts on other streams (batched serving of many scenes): the
 * cooperative launches of such solves run side by side.  A system needing
 * more than 32 level-0 subdomains per CTA falls back to the graph form. */
int sgmas_set_pcg_ctas(sgmas_context* ctx, int max_ctas);
/* Bound on each device-side wait of the persistent form (the grid barriers
 * between its phases and the waits for its bulk tile copies): at most
 * spin_limit polls (0 = the default, 4,194,304), after which the kernel sets
 * its error flag, leaves the loop and returns; sgmas_pcg_solve then reports
 * SGMAS_ERR_DEVICE ("bounded wait expired") and the context stays usable.
 * phantom_arrivals > 0 is fault injection for tests: every grid barrier then
 * waits for that many arrivals beyond the grid's CTAs, which never come, so
 * the first wait runs out (0 = normal operation).  No reference counterpart:
 * the reference's loop is host-driven and has no device-side waits. */
int sgmas_set_wait_limit(sgmas_context* ctx, int spin_limit, int phantom_arrivals);
/* Autotuner of the loop's launch shape: the persistent form on candidate grid
 * sizes (from the fewest CTAs the system fits on up to every SM, about x1.4
 * apart; tried from the largest down, until one does not fit) and the
 * graph form, each timed by `reps` trial solves of
 * trial_iters iterations (cfg as given, x0 = 0, into a scratch vector;
 * builds included, the loop's time per iteration compared).  Objective
 * SGMAS_TUNE_LATENCY picks the least time per iteration, SGMAS_TUNE_THROUGHPUT
 * the least SM-time per iteration for `concurrency` solves sharing the GPU
 * (time x max(CTAs, SMs / concurrency); the graph form counts every SM): a
 * grid below its share of the SMs gains nothing, the SMs it leaves idle.  The
 * choice stays set on the context (sgmas_set_pcg_mode / sgmas_set_pcg_ctas).
 * The project's own: the reference has no autotuner. */
#define SGMAS_TUNE_LATENCY 0
#define SGMAS_TUNE_THROUGHPUT 1
#define SGMAS_TUNE_MAX_CANDIDATES 16
typedef struct {
    int n_candidates;
    int ctas[SGMAS_TUNE_MAX_CANDIDATES];        /* grid tried (the graph form: 0) */
    int persistent[SGMAS_TUNE_MAX_CANDIDATES];  /* 1: the trial ran the persistent form */
    double us_per_iter[SGMAS_TUNE_MAX_CANDIDATES];  /* least over the reps */
    double cost[SGMAS_TUNE_MAX_CANDIDATES];     /* the objective's figure (us, or SM-us) */
    int chosen;                                 /* index of the choice */
    int sms;                                    /* SMs of the device */
} sgmas_tune_report;
int sgmas_autotune_pcg(sgmas_context* ctx, const sgmas_bcoo* A, const double* d_b, const sgmas_pcg_config* cfg,
                       int objective, int concurrency, int trial_iters, int reps, sgmas_tune_report* report);
/* the same with host arrays: uploads A and b, solves, downloads x */
int sgmas_pcg_solve_host(sgmas_context* ctx, const double* values, const int* rows,
                         const int* cols, int n_blocks, int n_block_rows, const double* b,
                         double* x, const sgmas_pcg_config* cfg, sgmas_pcg_report* report);

/* Device time of each phase of one PCG iteration on the buffers of the last
 * sgmas_pcg_solve (which it overwrites): ms[0] SpMV with the fused p update
 * and p.Ap, ms[1] update + level-0 MAS (or the block-Jacobi tail), ms[2]
 * coarse Schwarz, ms[3] CollectFinalZ + r.z.  After a graph-form solve each
 * kernel is replayed `reps` times between events.  After a persistent solve
 * the solve is run once more with clock stamps at every grid barrier: ms[0]
 * SpMV phase, ms[1] update + levels 0-1 (+ collect when the hierarchy has at
 * most two levels), ms[2] levels >= 2 + collect, ms[3] 0, ms[4] that solve's
 * loop time, ms[5] iterations averaged, and for each barrier slot (0 SpMV,
 * 1 x refresh, 2 r refresh, 3 levels 0-1, 4 unused, 5 end of iteration)
 * ms[6 + 3 * slot + 0..2] = the CTAs' mean and maximum work before it and
 * their mean wait in it, per occurrence (`reps` unused). */
int sgmas_pcg_profile(sgmas_context* ctx, int reps, float* ms, int n_ms);

/* ---- MAS set-up data on the host (no GPU needed) ----------------------- */
/* tetrahedra_obj::getVertNeighbors (SG/load_mesh.cpp:894-999): undirected
 * edges of the tets and triangles (global ids, FEM vertices from
 * abd_vert_offset) -> neighbour CSR; returns the list size or a negative
 * status.  nb_start/nb_num have n_verts entries, nb_list nb_cap. */
int sgmas_vert_neighbors(const int* tets, int n_tets, const int* tris, int n_tris, int n_verts,
                         int abd_vert_offset, unsigned* nb_start, unsigned* nb_num, unsigned* nb_list,
                         int nb_cap);
/* setMAS_partition (SG/main.cu:47-75) after load_parts (SG/load_mesh.cpp:449-480):
 * part ids (sorted-mesh order) -> part_map[part_offset*bank], real_map[n] */
int sgmas_part_maps(const int* part_id, int n, int bank, int* part_map, int part_map_cap,
                    int* part_map_size, int* real_map);

/* ---- kernels of the path, callable on their own ------------------------ */
/* Spmv::warp_reduce_sym_spmv (SG/linear_system/utils/spmv.cu:8-133): y = a A x + b y */
int sgmas_spmv(sgmas_context* ctx, double a, const sgmas_bcoo* A, const double* d_x, double b,
               double* d_y);
/* Converter::convert (SG/linear_system/utils/converter.cu:23-189): raw
 * triplets -> merged sorted BCOO; *n_unique receives the merged count
 * (h_unique_key_number, global_matrix.h:197).  Outputs need n entries. */
int sgmas_convert(sgmas_context* ctx, const double* d_values, const int* d_rows, const int* d_cols,
                  int n, double* d_out_values, int* d_out_rows, int* d_out_cols, int* n_unique);
/* The same merge for a triplet structure that stays fixed across Newton steps
 * (elastic terms of a mesh: same rows and cols in the same order every step).
 * sgmas_assembly_plan sorts and merges d_rows / d_cols of n raw triplets once:
 * the merged structure goes to d_out_rows / d_out_cols (*n_unique entries,
 * room for n), the sorted order stays on the context.  sgmas_assemble then
 * merges that step's n raw values (d_values [n][9]) into d_out_values
 * [n_unique][9] with one kernel and no sort, bit-identical to what
 * sgmas_convert returns for the same triplets.  The project's own: the
 * reference sorts every step. */
int sgmas_assembly_plan(sgmas_context* ctx, const int* d_rows, const int* d_cols, int n, int* d_out_rows,
                        int* d_out_cols, int* n_unique);
int sgmas_assemble(sgmas_context* ctx, const double* d_values, int n, double* d_out_values);

/* Element matrices straight into the planned structure: no raw triplet array.
 * A group is one element type (write_triplet_fem SG/femEnergy.cu:14-62 and
 * the barrier writers of SG/GIPC.cu:82-139 write one each): d_H [n_elem]
 * [3k][3k] row-major element matrices, d_nodes [n_elem][k] vertex ids,
 * k = nodes_per_elem in 1..4.  sgmas_element_plan takes 1..4 groups, lays out
 * their upper triplets in the order sgmas_write_upper_blocks writes them
 * (group after group; at most 2^30 - 1 of them), sorts and merges them as
 * sgmas_assembly_plan does (d_out_rows / d_out_cols need room for all raw
 * triplets), and keeps, for
 * each sorted triplet, where its 3x3 block sits in its group's matrices
 * (d_H is not read).  sgmas_element_assemble then reads that step's element
 * matrices (same groups, counts and nodes as planned; d_nodes is not read)
 * and writes the merged values with one kernel, bit-identical to
 * sgmas_write_upper_blocks of each group followed by sgmas_convert.  A later
 * sgmas_assembly_plan replaces the element plan.  The project's own (the
 * reference writes triplets and sorts them every step). */
/* The contact terms of a step into an assembled system: a sorted append.
 * d_base_* is a merged block list sorted by (row, col) with n_base blocks
 * (what sgmas_convert, sgmas_assemble or sgmas_element_assemble return); the
 * n raw triplets d_values / d_rows / d_cols (this step's contact blocks, e.g.
 * from sgmas_write_upper_blocks) are sorted on their own, each (row, col) run
 * is added to the base block with that key or becomes a new block, and the
 * union goes to d_out_* sorted (room for n_base + n blocks; the outputs must
 * not overlap the inputs), *n_out blocks.  Bit-identical to sgmas_convert of
 * the base's own raw triplets followed by these n.  The project's own (the
 * reference converts all triplets every step). */
int sgmas_append_triplets(sgmas_context* ctx, const double* d_base_values, const int* d_base_rows,
                          const int* d_base_cols, int n_base, const double* d_values, const int* d_rows,
                          const int* d_cols, int n, double* d_out_values, int* d_out_rows, int* d_out_cols,
                          int* n_out);

typedef struct sgmas_element_group {
    const double* d_H;
    const int* d_nodes;
    int n_elem;
    int nodes_per_elem;
} sgmas_element_group;
int sgmas_element_plan(sgmas_context* ctx, const sgmas_element_group* groups, int n_groups, int* d_out_rows,
                       int* d_out_cols, int* n_unique);
int sgmas_element_assemble(sgmas_context* ctx, const sgmas_element_group* groups, int n_groups,
                           double* d_out_values);

/* Affine-body coupling (ABDSystem::_setup_abd_system_hessian,
 * SG/abd_system/abd_system_function/setup_abd_system_gradient_and_hessian.cu:419-601):
 * vertex-level 3x3 blocks into the 3x3 triplets of the 12-DOF body rows (body b
 * owns block rows 4b .. 4b + 3).  A body vertex moves as x = J(xb) q with
 * J = [I | e1 xb^T | e2 xb^T | e3 xb^T] of its rest position xb (d_xbar [3 per
 * vertex]); d_body_of gives each body vertex's body, d_fixed[b] != 0 marks a
 * fixed body (BodyBoundaryType::Fixed).  Blocks are 9 doubles column-major.
 * sgmas_abd_body_blocks: each body's 12x12 Hessian (144 doubles, column-major)
 *   -> its 10 upper blocks (write_abd_body_hessian :127-136).
 * sgmas_abd_pair_blocks: n merged body-body vertex-pair blocks (row, col =
 *   vertex ids) -> 16 blocks each of J_i^T H J_j at [16 t, 16 t + 16), blocks
 *   below the diagonal written as zero with swapped indices (write_barrier_hessian
 *   :84-124); zero when either body is fixed.
 * sgmas_abd_fem_blocks: n body-vertex / FEM-vertex blocks (col = global point
 *   id, FEM point = col - fem_point_offset) -> 4 blocks each of J^T H at rows
 *   4 body + k, column 4 n_bodies + FEM point (:505-560); zero when the FEM
 *   point's boundary type (d_fem_boundary) is nonzero or the body is fixed. */
int sgmas_abd_body_blocks(sgmas_context* ctx, const double* d_H12, int n_bodies, double* d_vals, int* d_rows,
                          int* d_cols);
int sgmas_abd_pair_blocks(sgmas_context* ctx, const double* d_in_vals, const int* d_in_rows, const int* d_in_cols,
                          int n, const double* d_xbar, const int* d_body_of, const int* d_fixed, double* d_vals,
                          int* d_rows, int* d_cols);
int sgmas_abd_fem_blocks(sgmas_context* ctx, const double* d_in_vals, const int* d_in_rows, const int* d_in_cols,
                         int n, const double* d_xbar, const int* d_body_of, const int* d_fixed,
                         const int* d_fem_boundary, int fem_point_offset, int n_bodies, double* d_vals, int* d_rows,
                         int* d_cols);
/* write_triplet_fem / write_triplet<12,12> with SymGH (SG/femEnergy.cu:14-62,
 * SG/GIPC.cu:82-139): element matrices [n_elem][3k][3k] row-major with node
 * lists [n_elem][k] -> k(k+1)/2 upper triplets per element */
int sgmas_write_upper_blocks(sgmas_context* ctx, const double* d_H, int n_elem, int nodes_per_elem,
                             const int* d_nodes, double* d_values, int* d_rows, int* d_cols);
/* _calcVertMChash (SG/GIPC.cu:412-461, hash_code type -1 at :142-168):
 * (morton30 << 32) | vertex index; aabb = {lo.xyz, hi.xyz} or NULL for the
 * vertices' own bounding box */
int sgmas_morton_codes(sgmas_context* ctx, const double* d_pos, int n, const double* aabb,
                       uint64_t* d_codes);
/* Morton codes exactly as sgmas_morton_codes, for callers that cannot
 * allocate device memory: hosts whose device memory comes from their own pool
 * or is fixed at start-up, and loops that must not allocate once they run.
 * No reference counterpart: this entry point exists only in this library.
 * It needs no context and calls no allocating routine; the bounding-box
 * reduction uses a fixed 49,216-byte static device array that every GPU
 * loading the library holds until exit.  n must not exceed
 * SGMAS_MORTON_NOALLOC_MAX_VERTS (SGMAS_ERR_CAPACITY otherwise, before any
 * work is queued).  Runs on the current device and `stream` (NULL = legacy
 * default stream).  The first call on a device looks the array up
 * (cudaGetSymbolAddress) and loads the kernels: make that first call before
 * any stream capture.  The address is kept for the life of the process, so
 * the device's primary context must not be reset while the library is loaded.
 * An error already pending in the CUDA runtime when the call begins is
 * returned as SGMAS_ERR_CUDA and left pending, with no work queued.  All
 * calls share the array: calls that overlap on the GPU race, so order them
 * (same stream or synchronised). */
#define SGMAS_MORTON_NOALLOC_MAX_VERTS 2097152
int sgmas_morton_codes_noalloc(const double* d_pos, int n, const double* aabb, uint64_t* d_codes,
                               void* stream);
/* Morton order cut into bank-size subdomains: slot maps in the layout of
 * setMAS_partition (part_map[part_map_size], real_map[n]; host arrays) */
int sgmas_morton_partition(sgmas_context* ctx, const double* d_pos, int n, int* part_map,
                           int part_map_cap, int* part_map_size, int* real_map);

/* ---- learned start guess (no reference counterpart) ----------------------
 * A per-vertex MLP, 16 -> 128 -> 128 -> 6 with GELU, over features of the
 * Newton system.  For vertex v (row = fem_offset + v), with D its diagonal
 * 3x3 block, S_v = sum_j A_vj its 3x3 block row sum, u_v = S_v^-1 b_v (the
 * lumped step, exact for a rigid translation; D^-1 b_v where S_v has no
 * positive trace and determinant), t = trace(D) / 3 and s, s_b the RMS over
 * the MAS vertices of |u_v| and |b_v|, the features are: u_v / s (3), the
 * previous Newton step / s (3), D^-1 b_v / s (3), D_ii / t - 1 (3), D_01,
 * D_02, D_12 / t (3), min(contacts of v, 32) / 8 (1).  The network predicts
 * the correction (dx - u) / s: outputs 0-2 per vertex, outputs 3-5 a coarse
 * term averaged over the vertex's 16-slot MAS subdomain.  Rows are in the
 * MAS slot order of sgmas_mas_init (16 per subdomain, padding slots masked).
 * Parameters (FP32, SGMAS_MLP_PARAMS floats): W1 [16][128] (input-major),
 * b1 [128], W2 [128][128], b2 [128], W3 [128][6], b3 [6].  Training is FP32
 * (forward, backward, Adam with beta 0.9 / 0.999, eps 1e-8); the start guess
 * runs the network in BF16 with FP32 accumulation on the tensor cores. */
#define SGMAS_MLP_PARAMS 19462
/* set the FP32 parameters (host array) and reset the Adam state */
int sgmas_mlp_set_params(sgmas_context* ctx, const float* params, int n);
int sgmas_mlp_get_params(sgmas_context* ctx, float* params, int n);
/* features in slot order: d_X [Mm][16], d_mask [Mm] (1 = vertex, 0 = padding);
 * with d_dx (a solved step, 3 * n_block_rows doubles) also the training
 * target d_T [Mm][3] = (dx - u) / s.  d_prev: the previous Newton step or
 * NULL.  scales (host, may be NULL) receives (s, s_b).  Needs sgmas_mas_init and,
 * for the contact counts, sgmas_mas_set_contacts. */
int sgmas_mlp_features(sgmas_context* ctx, const sgmas_bcoo* A, const double* d_b, const double* d_prev,
                       const double* d_dx, int fem_offset, float* d_X, float* d_mask, float* d_T,
                       double* scales);
/* Loss on n_rows slot rows (a multiple of 16): inv_n * sum over valid rows of
 * |step + subdomain mean of the coarse term - T|^2.  sgmas_mlp_gradient writes
 * the gradient (SGMAS_MLP_PARAMS floats, device) without changing the
 * parameters; sgmas_mlp_train_step takes one Adam step with learning rate lr.
 * *loss (host, may be NULL) receives the loss before the step. */
int sgmas_mlp_gradient(sgmas_context* ctx, const float* d_X, const float* d_T, const float* d_mask, int n_rows,
                       float inv_n, float* d_grad, float* loss);
int sgmas_mlp_train_step(sgmas_context* ctx, const float* d_X, const float* d_T, const float* d_mask, int n_rows,
                         float inv_n, float lr, float* loss);
/* raw network outputs d_Y [n_rows][6]: bf16 = 0 the FP32 training network,
 * bf16 = 1 the BF16 tensor-core inference (tcgen05; d_X 16-byte aligned) */
int sgmas_mlp_forward(sgmas_context* ctx, const float* d_X, int n_rows, int bf16, float* d_Y);
/* The start guess of system (A, b), written to d_x0 (3 * n_block_rows
 * doubles): features + BF16 inference give the candidates v1 = u (the lumped
 * step S^-1 b, S = 3x3 block row sums of A), v2 = s * network step, v3 = s *
 * subdomain mean of the network's coarse term (MAS rows only), and v0 =
 * d_prev (the previous Newton step, when given); x0 = sum c_k v_k with
 * (V^T A V) c = V^T b, the A-norm-best combination (a candidate that is zero
 * or linearly dependent on earlier ones gets c_k = 0).  coef (host, may be
 * NULL) receives c_0..c_3.  Pass d_x0 as d_x of sgmas_pcg_solve with
 * initial_guess = 1, which rejects it if it raises the residual.  The block
 * CSR of A built here is reused by the next sgmas_pcg_solve on the same
 * arrays (they must not change in between). */
int sgmas_mlp_warm_start(sgmas_context* ctx, const sgmas_bcoo* A, const double* d_b, const double* d_prev,
                         int fem_offset, double* d_x0, double* coef);

#ifdef __cplusplus
}
#endif
#endif
