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
    int abd_bodies = 0;
};

// gipc::PCGSolver::solve (pcg_solver.cu:155-168): x = 0, PCG, returns the
// iteration count.
class PCGSolver {
  public:
    PCGSolver(Context& ctx, const PCGSolverConfig& cfg) : ctx_(ctx.get()), cfg_(cfg) {}
    int solve(const sgmas_bcoo& A, double* d_x, const double* d_b, sgmas_pcg_report* report = nullptr) {
        sgmas_pcg_config c = {cfg_.max_iter, cfg_.rel_tol,    cfg_.abs_tol, cfg_.use_preconditioned_residual_norm,
                              cfg_.preconditioner, cfg_.abd_bodies, 0,  10};
        sgmas_pcg_report rep = {};
        check(ctx_, sgmas_pcg_solve(ctx_, &A, d_b, d_x, &c, &rep), "PCGSolver::solve");
        if (report) *report = rep;
        return rep.iterations;
    }

  private:
    sgmas_context* ctx_;
    PCGSolverConfig cfg_;
};

}  // namespace sgmas
