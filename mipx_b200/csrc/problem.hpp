// Host-side LP model and scaling pipeline of the engine.
//
// The LP is kept in ranged form (row_lb <= A x <= row_ub, col_lb <= x <= col_ub)
// exactly like mipx::LpProblem (include/mipx/lp_problem.h:14-64).  Scaling
// follows PdlpSolver::buildScaledProblem (src/lp/pdlp.cpp:469-669) step for step
// in FP64 so that the scaled problem the device iterates on is the one the
// reference iterates on: sense normalisation, optional zero filter, Ruiz
// equilibration, Pock-Chambolle step preconditioner, bound/objective rescaling,
// row classification.  The explicit transpose follows buildTransposeCSR
// (pdlp.cpp:671-707): entries of each A^T row are in ascending row order.
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "pdlpx.h"

namespace pdlpx {

struct Csr {
    int32_t rows = 0, cols = 0;
    std::vector<int32_t> ptr{0};
    std::vector<int32_t> idx;
    std::vector<double> val;
    int32_t nnz() const { return static_cast<int32_t>(val.size()); }
};

struct HostLp {
    int32_t m = 0, n = 0;
    bool maximize = false;
    Csr a;
    std::vector<double> obj, cl, cu, rl, ru;
    double offset = 0.0;
};

// Row classes of the dual proximal step (pdlp.cpp:652-666).
enum RowType : int8_t { kRowEq = 0, kRowUpper = 1, kRowLower = 2, kRowRanged = 3 };

struct ScaledLp {
    double obj_sign = 1.0;
    double obj_scale = 1.0;  // objective_scale_
    double con_scale = 1.0;  // constraint_scale_
    Csr a;                   // scaled A (m x n)
    Csr at;                  // scaled A^T (n x m)
    std::vector<double> c, cl, cu, rl, ru;
    std::vector<double> row_scale, col_scale;
    std::vector<double> sigma, tau;  // Pock-Chambolle sigma_base / tau_base
    std::vector<int8_t> row_type;
    double precond_pw = 1.0;
};

// Canonical CSR with mipx::SparseMatrix triplet semantics (sparse_matrix.cpp:12-73):
// columns sorted within rows, duplicates summed, exact zeros dropped.
// Returns false on out-of-range indices or a non-monotone row pointer.
bool canonicalCsr(int32_t m, int32_t n, int32_t nnz, const int32_t* rp, const int32_t* ci,
                  const double* v, Csr& out);

void transposeCsr(const Csr& a, Csr& at);

// Ruiz equilibration done elsewhere (the device): scales the matrix values and
// multiplies the factors into row_scale / col_scale exactly as the host loop
// would; returns false to leave the work to the host loop.
using RuizFn = std::function<bool(Csr& a, std::vector<double>& row_scale, std::vector<double>& col_scale, int passes)>;

void buildScaled(const HostLp& lp, const pdlpx_options& o, ScaledLp& s, const RuizFn& ruiz = {});

// Ruiz passes on `device` (scaling.cu); bit-identical to the host loop.
// verbose prints the time of its phases.
bool ruizOnDevice(Csr& a, std::vector<double>& row_scale, std::vector<double>& col_scale, int passes, int device,
                  std::string& err, bool verbose = false);

// The Ruiz hook the options ask for: the device for scale_on_device = 1, or for
// -1 (auto) from 200k nonzeros; none (host loop) otherwise.  When the device
// passes fail (the host loop then does the work, with identical results) the
// reason goes to *fallback_note if given.
RuizFn ruizFor(const pdlpx_options& o, int64_t nnz, std::string* fallback_note = nullptr);

// Recompute sigma/tau from the scaled matrix (pdlp.cpp:713-742).
void pockChambolle(const ScaledLp& s, std::vector<double>& sigma, std::vector<double>& tau);

// Norms of the original objective and finite row bounds used by the relative
// termination criteria (pdlp.cpp:53-81).
void terminationNorms(const HostLp& lp, int32_t norm, double& c_norm, double& b_norm);

// y = A x / y = A^T x in FP64 on the host (used for reduced costs of the
// original problem after a solve, pdlp.cpp:2808-2819).
void csrMultiplyTranspose(const Csr& a, const double* x, double* y);

}  // namespace pdlpx
