// Serving loop implementation (see server.h).
#include "server.h"
#include "nvtx.h"

#include <cuda_runtime.h>

#include <string.h>

#include <algorithm>

namespace uf {

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    if (thread_.joinable()) thread_.join();
    launches_.clear();
    keys_.release();
}

int Server::start(const ServerConfig& cfg) {
    if (started_) return be_->set_error(kErrBadInput, "server already started");
    if (!be_->ready()) return be_->set_error(kErrGpuDevice, "context not ready");
    cfg_ = cfg;
    if (cfg_.slots == 0 || cfg_.slots > 64) return be_->set_error(kErrBadInput, "slots must be 1..64");
    if (cfg_.max_launch_items == 0 || cfg_.max_launch_items > BatchSlot::kGraphMaxItems)
        return be_->set_error(kErrBadInput, "max_launch_items must be 1..65536");
    // every slot holds pinned + device staging for its largest graph bucket
    const QueueLayout maxl(BatchSlot::kGraphMaxItems, BatchSlot::kGraphMaxItems);
    const uint64_t slot_bytes = (uint64_t)maxl.host_bytes + maxl.total;
    if (cfg_.key_cache_log2 != 0 &&
        (cfg_.key_cache_log2 < KeyTable::kMinLog2 || cfg_.key_cache_log2 > KeyTable::kMaxLog2))
        return be_->set_error(kErrBadInput, "key_cache_log2 must be 0 or 8..24");
    const uint64_t cache_bytes =
        cfg_.key_cache_log2 ? (kPubCacheSlotBytes << cfg_.key_cache_log2) + 256 : 0;
    if (cfg_.memory_budget_bytes < slot_bytes + cache_bytes)
        return be_->set_error(kErrBadInput, "memory budget below one slot and the key cache");
    cfg_.slots = (uint32_t)std::min<uint64_t>(
        cfg_.slots, std::max<uint64_t>(1, (cfg_.memory_budget_bytes - cache_bytes) / slot_bytes));
    if (cfg_.key_cache_log2) {
        const int rc = keys_.create(be_, cfg_.key_cache_log2);
        if (rc != kOk) return rc;
    }
    launches_.resize(cfg_.slots);
    for (auto& L : launches_) {
        L.slot.reset(new BatchSlot());
        const int rc = L.slot->init(be_);
        if (rc != kOk) {
            launches_.clear();
            return rc;
        }
        if (keys_.on()) L.slot->set_cache(keys_.slots(), keys_.mask(), keys_.counters());
        // instantiate every launch shape now, not on a request's critical path
        const int pw = L.slot->prewarm(cfg_.max_launch_items);
        if (pw != kOk) {
            launches_.clear();
            return pw;
        }
    }
    reserved_ = slot_bytes * launches_.size() + cache_bytes;
    budget_used_ = reserved_;
    peak_budget_ = reserved_;
    started_ = true;
    thread_ = std::thread([this] { loop(); });
    return kOk;
}

int Server::submit(const VerifyJob* jobs, size_t n_jobs, const ufsecp_cancel_token* cancel, uint64_t* id) {
    std::unique_ptr<Request> r(new Request());
    if (cancel && cancel->is_cancelled) {
        r->has_token = true;
        r->token = *cancel;
    }
    r->jobs.reserve(n_jobs);
    for (size_t j = 0; j < n_jobs; ++j) {
        if (jobs[j].count == 0) continue;
        r->jobs.push_back(jobs[j]);
        r->items += jobs[j].count;
    }
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(mu_);
    if (!started_ || stop_) return kErrGpuQueue;
    r->id = next_id_++;
    *id = r->id;
    if (!have_first_) {
        have_first_ = true;
        t_first_submit_ = r->t_submit;
    }
    Request* raw = r.get();
    reqs_.emplace(raw->id, std::move(r));
    if (raw->items == 0) {
        raw->all_launched = raw->done = true;
        lat_us_.push_back(0.0);
        cv_done_.notify_all();
        return kOk;
    }
    pending_.push_back(raw);
    cv_work_.notify_one();
    return kOk;
}

namespace {
bool token_cancelled(const ufsecp_cancel_token& t) {
    try {
        return t.is_cancelled(t.user) != 0;
    } catch (...) {
        return true;   // a predicate that throws counts as a cancellation (fail closed)
    }
}
}  // namespace

void Server::drop_pending(Request* r) {
    if (r->all_launched) return;
    r->all_launched = true;
    auto it = std::find(pending_.begin(), pending_.end(), r);
    if (it != pending_.end()) pending_.erase(it);
}

void Server::finalize(Request* r) {
    r->done = true;
    if (r->status != kOk) {
        // fail closed: a failed or cancelled request reports no verdict as valid
        for (const VerifyJob& J : r->jobs) memset(J.out, 0, J.count);
        return;
    }
    lat_us_.push_back(std::chrono::duration<double, std::micro>(Clock::now() - r->t_submit).count());
    items_done_ += r->items;
    t_last_done_ = Clock::now();
}

int Server::cancel(uint64_t id, uint32_t timeout_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return kErrBadInput;
    Request* r = it->second.get();
    if (!r->done) {
        r->abandoned = true;
        drop_pending(r);
        if (!cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), [r] { return r->pieces_in_flight == 0; }))
            return kErrGpuQueue;
        if (!r->done) {
            r->status = kErrCancelled;
            finalize(r);
        }
    }
    reqs_.erase(it);
    return kOk;
}

int Server::wait(uint64_t id, uint32_t timeout_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return kErrBadInput;
    Request* r = it->second.get();
    if (!cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), [r] { return r->done; })) return kErrGpuQueue;
    const int st = r->status;
    reqs_.erase(it);
    return st;
}

bool Server::admit(Launch& L) {
    NvtxRange range("server: admit");
    L.jobs.clear();
    L.owners.clear();
    size_t items = 0, bytes = 0;
    const size_t cap = cfg_.max_launch_items;
    bool budget_stop = false;
    while (!pending_.empty() && items < cap && !budget_stop) {
        Request* r = pending_.front();
        if (r->has_token && token_cancelled(r->token)) {
            // the caller's token asks to stop: no further piece of r is launched
            r->status = kErrCancelled;
            drop_pending(r);
            if (r->pieces_in_flight == 0) finalize(r);
            cv_done_.notify_all();
            continue;
        }
        while (r->next_job < r->jobs.size() && items < cap) {
            const VerifyJob& J = r->jobs[r->next_job];
            const size_t take = std::min(J.count - r->next_item, cap - items);
            const size_t b = take * bytes_per_item(J.kind);
            // with nothing in flight the first piece is always admitted (no deadlock)
            if (budget_used_ + bytes + b > cfg_.memory_budget_bytes && (items > 0 || in_flight_ > 0)) {
                budget_stop = true;
                break;
            }
            const size_t o = r->next_item;
            const size_t ps = J.kind == 0 ? 33 : 32;
            L.jobs.push_back(VerifyJob{J.kind, take, J.msgs + 32 * o, J.pubs + ps * o, J.sigs + 64 * o, J.out + o});
            L.owners.push_back(r);
            r->pieces_in_flight++;
            items += take;
            bytes += b;
            r->next_item += take;
            if (r->next_item == J.count) {
                r->next_job++;
                r->next_item = 0;
            }
        }
        if (r->next_job == r->jobs.size()) {
            r->all_launched = true;
            pending_.pop_front();
        } else {
            break;   // partly launched; the rest waits for the next free slot
        }
    }
    if (L.jobs.empty()) return false;
    L.busy = true;
    L.bytes = bytes;
    budget_used_ += bytes;
    peak_budget_ = std::max<uint64_t>(peak_budget_, budget_used_);
    if (in_flight_++ == 0) t_busy_since_ = Clock::now();
    peak_in_flight_ = std::max(peak_in_flight_, in_flight_);
    n_launches_++;
    return true;
}

void Server::complete(Launch& L, int rc) {
    const Clock::time_point now = Clock::now();
    for (Request* r : L.owners) {
        r->pieces_in_flight--;
        if (rc != kOk && r->status == kOk) r->status = rc;
        if (rc != kOk) drop_pending(r);    // the rest of a failed request is not launched
        if (r->abandoned && r->status == kOk) r->status = kErrCancelled;
        if (r->all_launched && r->pieces_in_flight == 0 && !r->done) finalize(r);
    }
    budget_used_ -= L.bytes;
    if (--in_flight_ == 0) busy_s_ += std::chrono::duration<double>(now - t_busy_since_).count();
    L.busy = false;
    L.bytes = 0;
    L.jobs.clear();
    L.owners.clear();
    cv_done_.notify_all();
}

void Server::loop() {
    cudaSetDevice(be_->device());
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        bool progressed = false;
        for (Launch& L : launches_) {
            if (!L.busy) continue;
            lk.unlock();
            const bool done = L.slot->ready();
            int rc = kOk;
            if (done) rc = L.slot->finish(L.jobs.data(), L.jobs.size());
            lk.lock();
            if (done) {
                complete(L, rc);
                progressed = true;
            }
        }
        if (stop_ && pending_.empty() && in_flight_ == 0) break;
        for (Launch& L : launches_) {
            if (L.busy || pending_.empty()) continue;
            if (cfg_.batch_window_us && in_flight_ > 0) {
                // let a small batch grow while the device is busy anyway
                size_t queued = 0;
                for (const Request* r : pending_) queued += r->items;
                const double age_us =
                    std::chrono::duration<double, std::micro>(Clock::now() - pending_.front()->t_submit).count();
                if (queued < cfg_.max_launch_items / 4 && age_us < cfg_.batch_window_us) break;
            }
            if (!admit(L)) break;
            lk.unlock();
            const int rc = L.slot->enqueue(L.jobs.data(), L.jobs.size());
            lk.lock();
            if (rc != kOk) complete(L, rc);
            progressed = true;
        }
        if (!progressed) {
            if (in_flight_ > 0) cv_work_.wait_for(lk, std::chrono::microseconds(20));
            else cv_work_.wait_for(lk, std::chrono::milliseconds(2));
        }
    }
}

void Server::stats(ServerStats* out, bool reset) {
    std::lock_guard<std::mutex> lk(mu_);
    ServerStats s;
    s.requests_done = lat_us_.size();
    s.items_done = items_done_;
    s.launches = n_launches_;
    s.peak_budget_bytes = peak_budget_;
    s.reserved_bytes = reserved_;
    if (keys_.on()) (void)keys_.read_counters(&s.cache_lookups, &s.cache_hits);
    s.peak_slots_in_flight = peak_in_flight_;
    s.pending_requests = pending_.size();
    s.busy_s = busy_s_;
    if (in_flight_ > 0) s.busy_s += std::chrono::duration<double>(Clock::now() - t_busy_since_).count();
    if (have_first_ && items_done_) s.span_s = std::chrono::duration<double>(t_last_done_ - t_first_submit_).count();
    if (!lat_us_.empty()) {
        std::vector<double> v(lat_us_);
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) { return v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
        s.p50_us = pct(0.50);
        s.p99_us = pct(0.99);
        s.max_us = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        s.mean_us = sum / v.size();
    }
    *out = s;
    if (reset) {
        lat_us_.clear();
        items_done_ = 0;
        n_launches_ = 0;
        peak_budget_ = budget_used_;
        peak_in_flight_ = in_flight_;
        busy_s_ = 0;
        if (in_flight_ > 0) t_busy_since_ = Clock::now();
        have_first_ = false;
    }
}

}  // namespace uf
