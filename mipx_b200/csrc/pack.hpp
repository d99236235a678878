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

// ---- families: node LPs of one base LP ---------------------------------------
// Branch-and-bound node LPs keep the base LP's constraint rows (bounds,
// objective and row bounds may change) and may append rows after them.  Up to
// kFamilyLanes such LPs are solved as one family pack: the base rows stored
// once, one lane per LP (family.cuh).
constexpr int kFamilyLanes = 32;

struct FamilyBase {
    int32_t m = 0, n = 0;           // base rows, columns
    std::vector<int32_t> ptr, idx;  // canonical CSR of the base rows, original values
    std::vector<double> val;
};
using FamilyPtr = std::shared_ptr<const FamilyBase>;

// Canonical copy of an LP's rows as a family base (null for an invalid LP or one without rows).
FamilyPtr makeFamilyBase(const pdlpx_lp& base);
// Whether a prepared LP is a member: same columns, the base rows first and
// unchanged, options that keep the original matrix (no zero filter).
bool familyMember(const PreparedLp& p, const FamilyBase& f, const pdlpx_options& o);
// Device bytes a member adds to a family pack (its lane plus its share of the base rows).
size_t familyMemberBytes(const PreparedLp& p, const FamilyBase& f);
// Offered between restart cycles while a family pack has a free lane: return a
// prepared member of the same family for which fits(lp) holds (its appended
// rows fit the room the pack reserved) and an id under which the pack reports
// it through `done`, or false when no member is waiting.  The caller keeps the
// returned LP alive until it is reported.
using FamilyAdmit =
    std::function<bool(const std::function<bool(const PreparedLp&)>& fits, PreparedLp*& lp, int& id)>;

// Solve up to kFamilyLanes members of one family as one pack on the current
// device (FP64 iterates, per-LP scaling and state); `done` as for solvePrepared
// (ids 0..lps.size()-1 for the initial members).  With `admit`, members that
// arrive while the pack runs take the lanes of finished ones (or unused lanes)
// between restart cycles, and the pack runs until no lane is busy.
int32_t solveFamily(const FamilyBase& f, const std::vector<PreparedLp*>& lps, const pdlpx_options& o,
                    const std::atomic<int>* stop, const LpDone& done, std::string& err,
                    const FamilyAdmit& admit = {});

}  // namespace pdlpx
