// Host interface of the packed batch engine (batch.cu), used by the batched
// solve and by the request server (server.cpp).
//
// An LP is first prepared on the host (copied, scaled like
// PdlpSolver::buildScaledProblem, its launch shapes and storage chosen); then
// any number of prepared LPs are solved together as one pack on their own CUDA
// stream.  Each LP is reported through a callback as soon as the restart
// cycle that finishes it returns, so results stream out of a pack while its
// other LPs keep iterating.
#pragma once

#include <atomic>
#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "pdlpx.h"

namespace pdlpx {

// Result of one LP: the pdlpx_result plus x and y in original space.
struct LpOutcome {
    pdlpx_result r{};
    std::vector<double> x, y;
};

// Called with the LP's index in the pack and its outcome.
using LpDone = std::function<void(int, LpOutcome&&)>;

struct PreparedLp;  // opaque: copy of the LP, scaled problem, pack layout choices
struct PreparedLpDeleter {
    void operator()(PreparedLp* p) const;
};
using PreparedPtr = std::unique_ptr<PreparedLp, PreparedLpDeleter>;

// Copy, validate and scale one LP (the caller's buffers may be freed afterwards).
int32_t prepareLp(const pdlpx_lp& lp, const pdlpx_options& o, PreparedPtr& out, std::string& err);
// An LP with no rows or no columns: closed form on the host, no device.
bool preparedTrivial(const PreparedLp& p);
int32_t solvePreparedTrivial(const PreparedLp& p, const pdlpx_options& o, LpOutcome& out, std::string& err);
// Device bytes the LP adds to a pack.
size_t preparedBytes(const PreparedLp& p);
int32_t preparedRows(const PreparedLp& p);
int32_t preparedCols(const PreparedLp& p);

// Solve non-trivial prepared LPs as one pack on the current device.  `stop`
// (may be null) ends the pack between restart cycles; unfinished LPs are then
// reported with status TimeLimit (or Optimal when their main loop had
// converged, as a time limit inside polish).  Returns PDLPX_* codes.
int32_t solvePrepared(const std::vector<PreparedLp*>& lps, const pdlpx_options& o, const std::atomic<int>* stop,
                      const LpDone& done, std::string& err);

}  // namespace pdlpx
