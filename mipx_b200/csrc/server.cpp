// Request server over the packed batch engine (pdlpx_server_* in pdlpx.h).
//
// Three kinds of host threads:
//   * preparation workers copy nothing (submit already copied the LP) but scale
//     it and choose its pack layout (prepareLp), in parallel;
//   * one dispatcher forms a pack from every prepared request that is waiting,
//     up to max_pack_lps and within the device budget left by the packs in
//     flight, whenever fewer than max_packs packs run;
//   * one worker per pack runs it on its own CUDA stream (solvePrepared) and
//     completes each request as soon as the restart cycle that finishes it
//     returns.
// A request submitted with a warm-start ticket whose constraint rows start with
// the ticket's rows unchanged (a branch-and-bound node of that LP: new bounds,
// appended cut rows) joins the ticket's family; the dispatcher packs members
// of one family together and runs them as a family pack (solveFamily: the
// base rows stored once, one lane per LP).
// So requests that arrive while packs run are admitted as soon as a stream and
// memory free up, and the packs' kernels overlap on the device.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "engine.hpp"
#include "pack.hpp"
#include "pdlpx.h"

namespace pdlpx {
namespace {

using Clock = std::chrono::steady_clock;

// Owned copy of a caller's pdlpx_lp.
struct OwnedLp {
    int32_t m = 0, n = 0, nnz = 0, sense = PDLPX_MINIMIZE;
    double offset = 0.0;
    std::vector<int32_t> ptr, idx;
    std::vector<double> val, obj, cl, cu, rl, ru, wx, wy;

    bool copy(const pdlpx_lp& in) {
        if (in.m < 0 || in.n < 0 || in.nnz < 0 || (in.m > 0 && in.row_ptr == nullptr) ||
            (in.nnz > 0 && (in.col_idx == nullptr || in.val == nullptr)) ||
            (in.n > 0 && (in.obj == nullptr || in.col_lb == nullptr || in.col_ub == nullptr)) ||
            (in.m > 0 && (in.row_lb == nullptr || in.row_ub == nullptr)))
            return false;
        m = in.m;
        n = in.n;
        nnz = in.nnz;
        sense = in.sense;
        offset = in.obj_offset;
        ptr.assign(in.row_ptr ? in.row_ptr : nullptr, in.row_ptr ? in.row_ptr + m + 1 : nullptr);
        if (ptr.empty()) ptr.assign(1, 0);
        idx.assign(in.col_idx, in.col_idx + nnz);
        val.assign(in.val, in.val + nnz);
        obj.assign(in.obj, in.obj + n);
        cl.assign(in.col_lb, in.col_lb + n);
        cu.assign(in.col_ub, in.col_ub + n);
        rl.assign(in.row_lb, in.row_lb + m);
        ru.assign(in.row_ub, in.row_ub + m);
        if (in.warm_x != nullptr && in.warm_y != nullptr) {
            wx.assign(in.warm_x, in.warm_x + n);
            wy.assign(in.warm_y, in.warm_y + m);
        }
        return true;
    }

    pdlpx_lp view() const {
        pdlpx_lp v{};
        v.m = m;
        v.n = n;
        v.nnz = nnz;
        v.row_ptr = ptr.data();
        v.col_idx = idx.data();
        v.val = val.data();
        v.obj = obj.data();
        v.col_lb = cl.data();
        v.col_ub = cu.data();
        v.row_lb = rl.data();
        v.row_ub = ru.data();
        v.sense = sense;
        v.obj_offset = offset;
        v.warm_x = wx.empty() ? nullptr : wx.data();
        v.warm_y = wy.empty() ? nullptr : wy.data();
        return v;
    }
};

enum ReqState { kQueued = 0, kPrepared = 1, kRunning = 2, kDone = 3 };

struct Request {
    int64_t ticket = 0;
    OwnedLp raw;
    PreparedPtr prep;
    size_t bytes = 0;
    Clock::time_point submitted, ready, finished;
    int state = kQueued;
    int32_t code = PDLPX_OK;
    std::string err;
    LpOutcome out;
    FamilyPtr fam_self;  // this LP as a family base (built when a node first links to it)
    FamilyPtr family;    // base of the family this request belongs to, or null
};

double quantile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * static_cast<double>(v.size() - 1);
    const size_t lo = static_cast<size_t>(pos);
    const size_t hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (pos - static_cast<double>(lo)) * (v[hi] - v[lo]);
}

}  // namespace

class Server {
public:
    // devices[k] is a CUDA ordinal, budget[k] its device-byte budget for packs in flight.
    Server(const pdlpx_options& o, const pdlpx_server_config& c, std::vector<int> devices, std::vector<size_t> budget)
        : opt_(o), cfg_(c), devices_(std::move(devices)), budget_(std::move(budget)),
          bytes_in_flight_(devices_.size(), 0), packs_on_(devices_.size(), 0) {}

    ~Server() { shutdown(); }

    void start() {
        const int prep = cfg_.prep_threads > 0
                             ? cfg_.prep_threads
                             : std::max(1, static_cast<int>(std::thread::hardware_concurrency()) - 1);
        for (int k = 0; k < prep; ++k) prep_threads_.emplace_back([this] { prepLoop(); });
        dispatcher_ = std::thread([this] { dispatchLoop(); });
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> g(mu_);
            if (closed_) return;
            closed_ = true;
            stop_.store(1);
        }
        cv_prep_.notify_all();
        cv_dispatch_.notify_all();
        for (auto& t : prep_threads_) t.join();
        if (dispatcher_.joinable()) dispatcher_.join();
        std::unique_lock<std::mutex> lk(mu_);
        cv_packs_.wait(lk, [this] { return packs_running_ == 0; });
        // requests that never reached a pack
        for (auto& kv : reqs_) {
            Request& r = *kv.second;
            if (r.state != kDone) {
                r.state = kDone;
                r.code = PDLPX_E_INVALID;
                r.err = "server shut down before the request was solved";
                r.finished = Clock::now();
            }
        }
        cv_done_.notify_all();
    }

    int32_t submit(const pdlpx_lp& lp, int64_t warm_ticket, int64_t* ticket, std::string& err) {
        auto req = std::make_unique<Request>();
        if (!req->raw.copy(lp)) {
            err = "invalid LP (sizes or missing arrays)";
            return PDLPX_E_INVALID;
        }
        std::lock_guard<std::mutex> g(mu_);
        if (closed_) {
            err = "server is shut down";
            return PDLPX_E_INVALID;
        }
        if (submitted_ - completed_ >= static_cast<int64_t>(cfg_.queue_limit)) {
            err = "request queue is full";
            return PDLPX_E_BUSY;
        }
        if (warm_ticket >= 0) {
            auto it = reqs_.find(warm_ticket);
            if (it == reqs_.end() || it->second->state != kDone || it->second->code != PDLPX_OK) {
                err = "warm-start ticket is unknown, unfinished or failed";
                return PDLPX_E_UNKNOWN_TICKET;
            }
            Request& base = *it->second;
            if (cfg_.families && base.raw.m > 0 && base.raw.n == req->raw.n && base.raw.m <= req->raw.m) {
                if (!base.fam_self) base.fam_self = makeFamilyBase(base.raw.view());
                req->family = base.fam_self;  // confirmed against the prepared LP
            }
            const LpOutcome& w = base.out;
            if (static_cast<int32_t>(w.x.size()) == req->raw.n && !w.x.empty()) {
                req->raw.wx = w.x;
                req->raw.wy.assign(req->raw.m, 0.0);
                const size_t k = std::min(w.y.size(), req->raw.wy.size());
                std::copy(w.y.begin(), w.y.begin() + static_cast<std::ptrdiff_t>(k), req->raw.wy.begin());
            }
        }
        const int64_t t = next_ticket_++;
        req->ticket = t;
        req->submitted = Clock::now();
        if (submitted_ == 0) first_submit_ = req->submitted;
        ++submitted_;
        *ticket = t;
        prep_q_.push_back(t);
        reqs_.emplace(t, std::move(req));
        cv_prep_.notify_one();
        return PDLPX_OK;
    }

    int32_t poll(int64_t ticket, int32_t* done) const {
        std::lock_guard<std::mutex> g(mu_);
        auto it = reqs_.find(ticket);
        if (it == reqs_.end()) return PDLPX_E_UNKNOWN_TICKET;
        *done = it->second->state == kDone ? 1 : 0;
        return PDLPX_OK;
    }

    int32_t wait(int64_t ticket, double timeout, pdlpx_result* out, std::string& err) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = reqs_.find(ticket);
        if (it == reqs_.end()) return PDLPX_E_UNKNOWN_TICKET;
        Request* r = it->second.get();
        auto ready = [r] { return r->state == kDone; };
        if (timeout < 0.0) {
            cv_done_.wait(lk, ready);
        } else if (!cv_done_.wait_for(lk, std::chrono::duration<double>(timeout), ready)) {
            err = "request still running";
            return PDLPX_E_TIMEOUT;
        }
        if (r->code != PDLPX_OK) {
            err = r->err;
            return r->code;
        }
        if (out) *out = r->out.r;
        return PDLPX_OK;
    }

    int32_t solution(int64_t ticket, double* x, int32_t n, double* y, int32_t m, std::string& err) const {
        std::lock_guard<std::mutex> g(mu_);
        auto it = reqs_.find(ticket);
        if (it == reqs_.end()) return PDLPX_E_UNKNOWN_TICKET;
        const Request& r = *it->second;
        if (r.state != kDone || r.code != PDLPX_OK) {
            err = "request unfinished or failed";
            return PDLPX_E_INVALID;
        }
        if ((x && n != static_cast<int32_t>(r.out.x.size())) || (y && m != static_cast<int32_t>(r.out.y.size()))) {
            err = "solution sizes do not match the LP";
            return PDLPX_E_INVALID;
        }
        if (x && n > 0) std::memcpy(x, r.out.x.data(), 8 * static_cast<size_t>(n));
        if (y && m > 0) std::memcpy(y, r.out.y.data(), 8 * static_cast<size_t>(m));
        return PDLPX_OK;
    }

    int32_t release(int64_t ticket) {
        std::lock_guard<std::mutex> g(mu_);
        auto it = reqs_.find(ticket);
        if (it == reqs_.end()) return PDLPX_E_UNKNOWN_TICKET;
        if (it->second->state != kDone) return PDLPX_E_BUSY;
        reqs_.erase(it);
        return PDLPX_OK;
    }

    void stats(pdlpx_server_stats* s) const {
        std::lock_guard<std::mutex> g(mu_);
        std::memset(s, 0, sizeof(*s));
        s->submitted = submitted_;
        s->completed = completed_;
        int64_t waiting = 0, running = 0;
        for (const auto& kv : reqs_) {
            const int st = kv.second->state;
            waiting += st == kQueued || st == kPrepared;
            running += st == kRunning;
        }
        s->waiting = waiting;
        s->running = running;
        s->packs_running = packs_running_;
        size_t inflight = 0;
        for (size_t b : bytes_in_flight_) inflight += b;
        s->p50_latency_s = quantile(latencies_, 0.50);
        s->p99_latency_s = quantile(latencies_, 0.99);
        double sum = 0.0, mx = 0.0;
        for (double v : latencies_) {
            sum += v;
            mx = std::max(mx, v);
        }
        s->mean_latency_s = latencies_.empty() ? 0.0 : sum / static_cast<double>(latencies_.size());
        s->max_latency_s = mx;
        const double span = completed_ > 0 ? std::chrono::duration<double>(last_complete_ - first_submit_).count() : 0.0;
        s->lps_per_sec = span > 0.0 ? static_cast<double>(completed_) / span : 0.0;
        s->bytes_in_flight = static_cast<double>(inflight);
        s->admitted = admitted_;
    }

private:
    // Completion of one request (mu_ held).
    void finishLocked(Request& r) {
        r.state = kDone;
        r.finished = Clock::now();
        ++completed_;
        last_complete_ = r.finished;
        latencies_.push_back(std::chrono::duration<double>(r.finished - r.submitted).count());
    }

    void prepLoop() {
        while (true) {
            Request* r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_prep_.wait(lk, [this] { return closed_ || !prep_q_.empty(); });
                if (closed_) return;
                r = reqs_.at(prep_q_.front()).get();
                prep_q_.pop_front();
            }
            // r stays valid: a request is only erased once done
            std::string err;
            PreparedPtr p;
            int32_t rc = prepareLp(r->raw.view(), opt_, p, err);
            LpOutcome trivial;
            if (rc == PDLPX_OK && preparedTrivial(*p)) rc = solvePreparedTrivial(*p, opt_, trivial, err);
            std::lock_guard<std::mutex> g(mu_);
            if (rc != PDLPX_OK) {
                r->code = rc;
                r->err = err;
                finishLocked(*r);
                cv_done_.notify_all();
            } else if (preparedTrivial(*p)) {
                r->out = std::move(trivial);
                finishLocked(*r);
                cv_done_.notify_all();
            } else {
                if (r->family && !familyMember(*p, *r->family, opt_)) r->family = nullptr;
                r->bytes = r->family ? familyMemberBytes(*p, *r->family) : preparedBytes(*p);
                r->prep = std::move(p);
                r->state = kPrepared;
                r->ready = Clock::now();
                ready_q_.push_back(r->ticket);
                cv_dispatch_.notify_one();
            }
        }
    }

    // The device a pack of `head` would start on now (mu_ held): among the
    // devices with a free stream whose budget admits the head request (or that
    // run nothing), the one with the fewest bytes in flight, ties to the lower
    // index; -1 when none.
    int pickDevice(const Request& head, int max_packs) const {
        int best = -1;
        for (size_t d = 0; d < devices_.size(); ++d) {
            if (packs_on_[d] >= max_packs) continue;
            if (bytes_in_flight_[d] != 0 && bytes_in_flight_[d] + head.bytes > budget_[d]) continue;
            if (best < 0 || bytes_in_flight_[d] < bytes_in_flight_[static_cast<size_t>(best)]) best = static_cast<int>(d);
        }
        return best;
    }

    void dispatchLoop() {
        const int max_packs = std::max(1, cfg_.max_packs);
        const size_t max_lps = static_cast<size_t>(std::max(1, cfg_.max_pack_lps));
        while (true) {
            std::vector<Request*> pack;
            size_t bytes = 0;
            int dev = -1;
            {
                std::unique_lock<std::mutex> lk(mu_);
                // A pack starts when a stream and memory are free on some device and
                // either a full pack is ready or the oldest ready request has waited
                // the batching window (a pack runs for many restart cycles, so a
                // short wait that fills it costs less latency than it saves).
                const auto window = std::chrono::milliseconds(std::max(0, cfg_.batch_window_ms));
                while (true) {
                    if (closed_) return;
                    bool can = !ready_q_.empty();
                    if (can) {
                        const Request& head = *reqs_.at(ready_q_.front());
                        dev = pickDevice(head, max_packs);
                        can = dev >= 0;
                        if (can && ready_q_.size() < max_lps) {
                            const auto due = head.ready + window;
                            if (Clock::now() < due) {
                                cv_dispatch_.wait_until(lk, due);
                                continue;
                            }
                        }
                    }
                    if (can) break;
                    cv_dispatch_.wait(lk);
                }
                // the head request's family (or the requests outside any family),
                // in arrival order
                const FamilyPtr fam = reqs_.at(ready_q_.front())->family;
                const size_t cap = fam ? std::min<size_t>(max_lps, kFamilyLanes) : max_lps;
                const size_t du = static_cast<size_t>(dev);
                std::deque<int64_t> rest;
                while (!ready_q_.empty()) {
                    Request* r = reqs_.at(ready_q_.front()).get();
                    const bool take = r->family == fam && pack.size() < cap &&
                                      (pack.empty() || bytes_in_flight_[du] + bytes + r->bytes <= budget_[du]);
                    if (take) {
                        bytes += r->bytes;
                        r->state = kRunning;
                        pack.push_back(r);
                    } else {
                        rest.push_back(ready_q_.front());
                    }
                    ready_q_.pop_front();
                }
                ready_q_.swap(rest);
                bytes_in_flight_[du] += bytes;
                ++packs_on_[du];
                ++packs_running_;
            }
            std::thread([this, pack, bytes, dev] { runPack(pack, bytes, dev); }).detach();
            pack.clear();
        }
    }

    // The pack owns its prepared LPs until it returns (the engine reads every
    // LP of the pack until the last one finishes), and a finished request may be
    // released by its client at once, so completion is tracked here, never by
    // reading a request after it was completed.
    void runPack(std::vector<Request*> pack, size_t bytes, int dev) {
        std::vector<PreparedPtr> preps;
        std::vector<PreparedLp*> lps;
        FamilyPtr fam;
        {
            std::lock_guard<std::mutex> g(mu_);
            fam = pack.front()->family;
            for (Request* r : pack) {
                preps.push_back(std::move(r->prep));
                lps.push_back(preps.back().get());
            }
        }
        std::vector<char> finished(pack.size(), 0);
        std::string err;
        auto done = [&](int l, LpOutcome&& out) {
            std::lock_guard<std::mutex> g(mu_);
            finished[l] = 1;
            Request& r = *pack[l];
            r.out = std::move(out);
            finishLocked(r);
            cv_done_.notify_all();
        };
        pdlpx_options o = opt_;
        o.device = devices_[static_cast<size_t>(dev)];
        const size_t du = static_cast<size_t>(dev);
        // Continuous admission into a family pack: between restart cycles the pack
        // offers its free lanes, and a waiting member of its family whose
        // appended rows fit takes one (within this device's budget) instead of
        // waiting for a new pack.
        FamilyAdmit admit;
        if (fam && cfg_.lane_admission) {
            admit = [&](const std::function<bool(const PreparedLp&)>& fits, PreparedLp*& lp, int& id) -> bool {
                std::lock_guard<std::mutex> g(mu_);
                if (closed_) return false;
                for (auto it = ready_q_.begin(); it != ready_q_.end(); ++it) {
                    Request* r = reqs_.at(*it).get();
                    if (r->family != fam || !fits(*r->prep)) continue;
                    if (bytes_in_flight_[du] + r->bytes > budget_[du]) return false;
                    r->state = kRunning;
                    bytes += r->bytes;
                    bytes_in_flight_[du] += r->bytes;
                    pack.push_back(r);
                    finished.push_back(0);
                    preps.push_back(std::move(r->prep));
                    lp = preps.back().get();
                    id = static_cast<int>(pack.size()) - 1;
                    ready_q_.erase(it);
                    ++admitted_;
                    return true;
                }
                return false;
            };
        }
        const int32_t rc =
            fam ? solveFamily(*fam, lps, o, &stop_, done, err, admit) : solvePrepared(lps, o, &stop_, done, err);
        std::lock_guard<std::mutex> g(mu_);
        for (size_t k = 0; k < pack.size(); ++k) {
            if (finished[k]) continue;
            Request* r = pack[k];
            r->code = rc != PDLPX_OK ? rc : PDLPX_E_CUDA;
            r->err = rc != PDLPX_OK ? err : "pack ended without a result";
            finishLocked(*r);
        }
        bytes_in_flight_[static_cast<size_t>(dev)] -= bytes;
        --packs_on_[static_cast<size_t>(dev)];
        --packs_running_;
        cv_done_.notify_all();
        cv_dispatch_.notify_all();
        cv_packs_.notify_all();
    }

    const pdlpx_options opt_;
    const pdlpx_server_config cfg_;
    const std::vector<int> devices_;     // CUDA ordinals the packs run on
    const std::vector<size_t> budget_;   // per device
    mutable std::mutex mu_;
    std::condition_variable cv_prep_, cv_dispatch_, cv_done_, cv_packs_;
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs_;
    std::deque<int64_t> prep_q_, ready_q_;
    std::vector<std::thread> prep_threads_;
    std::thread dispatcher_;
    std::atomic<int> stop_{0};
    bool closed_ = false;
    int packs_running_ = 0;               // all devices
    std::vector<size_t> bytes_in_flight_;  // per device
    std::vector<int> packs_on_;            // per device
    int64_t next_ticket_ = 1, submitted_ = 0, completed_ = 0;
    int64_t admitted_ = 0;  // requests that joined a running family pack
    Clock::time_point first_submit_, last_complete_;
    std::vector<double> latencies_;
};

}  // namespace pdlpx

struct pdlpx_server {
    std::unique_ptr<pdlpx::Server> impl;
    mutable std::mutex err_mu;
    std::string last_error;
    void setError(const std::string& e) {
        std::lock_guard<std::mutex> g(err_mu);
        last_error = e;
    }
};

extern "C" {

void pdlpx_server_config_default(pdlpx_server_config* c) {
    if (c == nullptr) return;
    std::memset(c, 0, sizeof(*c));
    c->budget_bytes = 0.0;
    c->max_packs = 4;
    c->max_pack_lps = 32;
    c->prep_threads = 0;
    c->queue_limit = 100000;
    c->batch_window_ms = 50;
    c->families = 1;
    c->lane_admission = 1;
}

int32_t pdlpx_server_create(const pdlpx_options* opts, const pdlpx_server_config* cfg, pdlpx_server** out) {
    if (out == nullptr) return PDLPX_E_INVALID;
    *out = nullptr;
    try {
        pdlpx_options o;
        pdlpx_options_default(&o);
        if (opts) o = *opts;
        pdlpx_server_config c;
        pdlpx_server_config_default(&c);
        if (cfg) c = *cfg;
        if (c.queue_limit <= 0) c.queue_limit = 100000;
        int devcount = 0;
        if (cudaGetDeviceCount(&devcount) != cudaSuccess || devcount <= 0) {
            cudaGetLastError();
            pdlpx::setGlobalError("no CUDA device visible");
            return PDLPX_E_NO_DEVICE;
        }
        std::vector<int> devices;
        if (c.num_devices > 1) {
            if (c.num_devices > static_cast<int32_t>(sizeof(c.devices) / sizeof(c.devices[0]))) {
                pdlpx::setGlobalError("num_devices exceeds the devices array");
                return PDLPX_E_INVALID;
            }
            for (int32_t k = 0; k < c.num_devices; ++k) {
                if (c.devices[k] < 0 || c.devices[k] >= devcount) {
                    pdlpx::setGlobalError("device ordinal " + std::to_string(c.devices[k]) + " out of range");
                    return PDLPX_E_INVALID;
                }
                devices.push_back(c.devices[k]);
            }
        } else {
            devices.push_back((o.device >= 0 && o.device < devcount) ? o.device : 0);
        }
        std::vector<size_t> budget;
        for (int dev : devices) {
            size_t b = static_cast<size_t>(c.budget_bytes > 0.0 ? c.budget_bytes : 0.0);
            if (b == 0) {
                size_t free_b = 0, total_b = 0;
                if (cudaSetDevice(dev) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
                    cudaGetLastError();
                    pdlpx::setGlobalError("cudaMemGetInfo failed");
                    return PDLPX_E_CUDA;
                }
                // a device listed twice shares its memory between its entries
                const auto copies = std::count(devices.begin(), devices.end(), dev);
                b = static_cast<size_t>(0.85 * static_cast<double>(free_b) / static_cast<double>(copies));
            }
            budget.push_back(b);
        }
        cudaSetDevice(devices.front());
        auto* s = new pdlpx_server();
        s->impl = std::make_unique<pdlpx::Server>(o, c, devices, budget);
        s->impl->start();
        *out = s;
        return PDLPX_OK;
    } catch (const std::bad_alloc&) {
        return PDLPX_E_NOMEM;
    } catch (...) {
        return PDLPX_E_INVALID;
    }
}

int32_t pdlpx_server_destroy(pdlpx_server* s) {
    if (s == nullptr) return PDLPX_E_INVALID;
    s->impl->shutdown();
    delete s;
    return PDLPX_OK;
}

static int32_t submitCommon(pdlpx_server* s, const pdlpx_lp* lp, int64_t warm, int64_t* ticket) {
    if (s == nullptr || lp == nullptr || ticket == nullptr) return PDLPX_E_INVALID;
    try {
        std::string err;
        const int32_t rc = s->impl->submit(*lp, warm, ticket, err);
        if (rc != PDLPX_OK) s->setError(err);
        return rc;
    } catch (const std::bad_alloc&) {
        s->setError("host allocation failed");
        return PDLPX_E_NOMEM;
    }
}

int32_t pdlpx_server_submit(pdlpx_server* s, const pdlpx_lp* lp, int64_t* ticket) {
    return submitCommon(s, lp, -1, ticket);
}

int32_t pdlpx_server_submit_warm(pdlpx_server* s, const pdlpx_lp* lp, int64_t warm_ticket, int64_t* ticket) {
    if (warm_ticket < 0) return PDLPX_E_INVALID;
    return submitCommon(s, lp, warm_ticket, ticket);
}

int32_t pdlpx_server_poll(pdlpx_server* s, int64_t ticket, int32_t* done) {
    if (s == nullptr || done == nullptr) return PDLPX_E_INVALID;
    return s->impl->poll(ticket, done);
}

int32_t pdlpx_server_wait(pdlpx_server* s, int64_t ticket, double timeout_seconds, pdlpx_result* out) {
    if (s == nullptr) return PDLPX_E_INVALID;
    std::string err;
    const int32_t rc = s->impl->wait(ticket, timeout_seconds, out, err);
    if (rc != PDLPX_OK) s->setError(err);
    return rc;
}

int32_t pdlpx_server_get_solution(const pdlpx_server* s, int64_t ticket, double* x, int32_t n, double* y,
                                  int32_t m) {
    if (s == nullptr) return PDLPX_E_INVALID;
    std::string err;
    const int32_t rc = s->impl->solution(ticket, x, n, y, m, err);
    if (rc != PDLPX_OK) const_cast<pdlpx_server*>(s)->setError(err);
    return rc;
}

int32_t pdlpx_server_release(pdlpx_server* s, int64_t ticket) {
    if (s == nullptr) return PDLPX_E_INVALID;
    return s->impl->release(ticket);
}

int32_t pdlpx_server_get_stats(const pdlpx_server* s, pdlpx_server_stats* out) {
    if (s == nullptr || out == nullptr) return PDLPX_E_INVALID;
    s->impl->stats(out);
    return PDLPX_OK;
}

const char* pdlpx_server_last_error(const pdlpx_server* s) {
    if (s == nullptr) return "";
    return s->last_error.c_str();
}

}  // extern "C"
