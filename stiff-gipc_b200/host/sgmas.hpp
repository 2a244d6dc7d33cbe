// sgmas.hpp -- C++ host mirror of the reference's MASPreconditioner and
// PCGSolver over the sgmas C-ABI (include/sgmas.h).
//
// The classes keep the reference's names, argument meaning and call order
// (SG/MASPreconditioner.cuh:14-102, SG/linear_system/solver/pcg_solver.h:6-40)
// so a caller of the reference can switch with minimal edits; errors are
// thrown as sgmas::Error instead of aborting (the reference's CUDA_SAFE_CALL,
// SG/cuda_tools/cuda_tools.h:35-46).
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sgmas.h"

namespace sgmas {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(sgmas_context* ctx, int rc, const char* what) {
    if (rc != SGMAS_OK) throw Error(rc, std::string(what) + ": " + sgmas_last_error(ctx));
}

// One context per device; the MAS state lives in it.
class Context {
  public:
    explicit Context(int device = 0, int bank = 16, int precision = SGMAS_MAS_FP32) {
        sgmas_config cfg = {device, bank, precision};
        const int rc = sgmas_create(&cfg, &ctx_);
        if (rc != SGMAS_OK) throw Error(rc, "sgmas_create failed");
    }
    ~Context() { sgmas_destroy(ctx_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    sgmas_context* get() const { return ctx_; }
    void set_stream(void* s) { check(ctx_, sgmas_set_stream(ctx_, s), "sgmas_set_stream"); }
    // SGMAS_PCG_PERSISTENT (default) or SGMAS_PCG_GRAPH
    void set_pcg_mode(int mode) { check(ctx_, sgmas_set_pcg_mode(ctx_, mode), "sgmas_set_pcg_mode"); }
    // at most max_ctas CTAs for the persistent form (0: every SM); for solves of many contexts side by side
    void set_pcg_ctas(int max_ctas) { check(ctx_, sgmas_set_pcg_ctas(ctx_, max_ctas), "sgmas_set_pcg_ctas"); }
    // launch shape by timed trial solves on A (kept on the context); see sgmas_autotune_pcg
    sgmas_tune_report autotune(const sgmas_bcoo& A, const double* d_b, const sgmas_pcg_config& cfg,
                               int objective = SGMAS_TUNE_THROUGHPUT, int concurrency = 1, int trial_iters = 30,
                               int reps = 2) {
        sgmas_tune_report r{};
        check(ctx_, sgmas_autotune_pcg(ctx_, &A, d_b, &cfg, objective, concurrency, trial_iters, reps, &r),
              "sgmas_autotune_pcg");
        return r;
    }
    // fixed triplet structure: sort and merge once, then merge each step's values without a sort
    int assembly_plan(const int* d_rows, const int* d_cols, int n, int* d_out_rows, int* d_out_cols) {
        int nu = 0;
        check(ctx_, sgmas_assembly_plan(ctx_, d_rows, d_cols, n, d_out_rows, d_out_cols, &nu), "sgmas_assembly_plan");
        return nu;
    }
    void assemble(const double* d_values, int n, double* d_out_values) {
        check(ctx_, sgmas_assemble(ctx_, d_values, n, d_out_values), "sgmas_assemble");
    }

  private:
    sgmas_context* ctx_ = nullptr;
};

// MASPreconditioner (SG/MASPreconditioner.cuh:14-102).  The reference fills
// public device arrays between initPreconditioner_Neighbor and
// initPreconditioner_Matrix (SG/main.cu:998-1027); here the host arrays are
// handed over in one call.
class MASPreconditioner {
  public:
    explicit MASPreconditioner(Context& ctx) : ctx_(ctx.get()) {}

    void initPreconditioner_Neighbor(int vertNum, int mCollision_node_offset, const std::vector<unsigned>& neighborList,
                                     const std::vector<unsigned>& neighborStart,
                                     const std::vector<unsigned>& neighborNum, const std::vector<int>& partId_map_real,
                                     const std::vector<int>& real_map_partId) {
        check(ctx_,
              sgmas_mas_init(ctx_, vertNum, mCollision_node_offset, (int)neighborList.size(), neighborList.data(),
                             neighborStart.data(), neighborNum.data(), partId_map_real.data(),
                             (int)partId_map_real.size(), real_map_partId.data()),
              "initPreconditioner_Neighbor");
    }
    // the initial ReorderRealtime(0) and allocation happen inside
    // initPreconditioner_Neighbor; kept for call-site compatibility
    void initPreconditioner_Matrix() {}

    // _collisonPairs (device int4 array) for the next setPreconditioner_bcoo
    void setCollisionPairs(const int* d_pairs_int4, int capacity) {
        check(ctx_, sgmas_mas_set_contacts(ctx_, d_pairs_int4, capacity), "setCollisionPairs");
    }

    void setPreconditioner_bcoo(const double* triplet_values, const int* row_ids, const int* col_ids,
                                const uint32_t* indices, int offset, int triplet_num, int cpNum) {
        check(ctx_, sgmas_mas_assemble(ctx_, triplet_values, row_ids, col_ids, indices, offset, triplet_num, cpNum),
              "setPreconditioner_bcoo");
    }

    void preconditioning(const double* R, double* Z) {
        check(ctx_, sgmas_mas_apply(ctx_, R, Z), "preconditioning");
    }

    void FreeMAS() {}  // the context owns and frees the arrays

  private:
    sgmas_context* ctx_;
};

// gipc::PCGSolverConfig (pcg_solver.h:6-15) + the preconditioner choice.
struct PCGSolverConfig {
    int max_iter = 0;
    double rel_tol = 1e-2;
    double abs_tol = 0.0;
    bool use_preconditioned_residual_norm = true;
    int preconditioner = 1;  // 0: block-Jacobi (P_type 0), 1: MAS (P_type 1)
    int abd_bodies = 0;      // affine bodies first, 4 block rows each (12x12 block-Jacobi)
    int fem_offset = 0;      // first block row of the MAS range (the FEM vertices)
    bool initial_guess = false;  // d_x holds a start guess (scaled; rejected when it raises ||r0||)
};

// gipc::PCGSolver::solve (pcg_solver.cu:155-168): x = 0 (or the start guess
// in d_x with initial_guess), PCG, returns the iteration count.
class PCGSolver {
  public:
    PCGSolver(Context& ctx, const PCGSolverConfig& cfg) : ctx_(ctx.get()), cfg_(cfg) {}
    int solve(const sgmas_bcoo& A, double* d_x, const double* d_b, sgmas_pcg_report* report = nullptr) {
        sgmas_pcg_config c = {cfg_.max_iter,       cfg_.rel_tol,    cfg_.abs_tol, cfg_.use_preconditioned_residual_norm,
                              cfg_.preconditioner, cfg_.abd_bodies, cfg_.fem_offset, 10,
                              cfg_.initial_guess ? 1 : 0};
        sgmas_pcg_report rep = {};
        check(ctx_, sgmas_pcg_solve(ctx_, &A, d_b, d_x, &c, &rep), "PCGSolver::solve");
        if (report) *report = rep;
        return rep.iterations;
    }
    // the solver's members r and z after the last solve (pcg_solver.h:29-30), device arrays
    void last_vectors(double* d_r, double* d_z) {
        check(ctx_, sgmas_pcg_last_vectors(ctx_, d_r, d_z), "PCGSolver::last_vectors");
    }

  private:
    sgmas_context* ctx_;
    PCGSolverConfig cfg_;
};

// A host BCOO system: the reference's export / import files
// (GlobalLinearSystem::export_matrix_market_files; SG/main.cu:398-646).
struct HostSystem {
    std::vector<double> values;  // 9 per block, column-major
    std::vector<int> rows, cols;
    int n_block_rows = 0;
    std::vector<double> b;
};

inline void mtx_write(const std::string& path_A, const std::string& path_b, const HostSystem& s) {
    check(nullptr,
          sgmas_mtx_write(path_A.c_str(), path_b.empty() ? nullptr : path_b.c_str(), s.values.data(), s.rows.data(),
                          s.cols.data(), (int)s.rows.size(), s.n_block_rows, s.b.empty() ? nullptr : s.b.data()),
          "mtx_write");
}

inline HostSystem mtx_read(const std::string& path_A, const std::string& path_b = "") {
    HostSystem s;
    int nb = 0, nr = 0;
    const char* pb = path_b.empty() ? nullptr : path_b.c_str();
    int rc = sgmas_mtx_read(path_A.c_str(), pb, nullptr, nullptr, nullptr, 0, nullptr, 0, &nb, &nr);
    if (rc != SGMAS_OK && rc != SGMAS_ERR_CAPACITY) check(nullptr, rc, "mtx_read");
    s.values.resize(9 * (size_t)nb);
    s.rows.resize(nb);
    s.cols.resize(nb);
    s.n_block_rows = nr;
    if (pb) s.b.resize(3 * (size_t)nr);
    check(nullptr,
          sgmas_mtx_read(path_A.c_str(), pb, s.values.data(), s.rows.data(), s.cols.data(), nb,
                         pb ? s.b.data() : nullptr, (int)s.b.size(), &nb, &nr),
          "mtx_read");
    return s;
}

}  // namespace sgmas
