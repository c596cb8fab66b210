// Host thread pool for staging copies (see pack_pool.h).
#include "pack_pool.h"

namespace uf {

PackPool::PackPool(int threads) {
    for (int i = 1; i < threads; ++i) helpers_.emplace_back([this] { helper(); });
}

PackPool::~PackPool() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    work_cv_.notify_all();
    for (auto& t : helpers_) t.join();
}

void PackPool::helper() {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
        work_cv_.wait(lk, [this] { return stop_ || (fn_ && next_ < parts_); });
        if (stop_) return;
        const int p = next_++;
        const std::function<void(int)>* f = fn_;
        lk.unlock();
        (*f)(p);
        lk.lock();
        if (--remaining_ == 0) done_cv_.notify_all();
    }
}

void PackPool::run(int parts, const std::function<void(int)>& fn) {
    if (parts <= 0) return;
    if (helpers_.empty() || parts == 1) {
        for (int p = 0; p < parts; ++p) fn(p);
        return;
    }
    std::unique_lock<std::mutex> lk(mu_);
    fn_ = &fn;
    parts_ = parts;
    next_ = 0;
    remaining_ = parts;
    lk.unlock();
    work_cv_.notify_all();
    lk.lock();
    while (next_ < parts_) {
        const int p = next_++;
        lk.unlock();
        fn(p);
        lk.lock();
        --remaining_;
    }
    done_cv_.wait(lk, [this] { return remaining_ == 0; });
    fn_ = nullptr;
    parts_ = 0;
}

}  // namespace uf
