// A small persistent thread pool for the host side's staging copies.
//
// A host-buffer verify call copies the caller's arrays into pinned staging
// (about 128 bytes per signature) while the device verifies earlier chunks.
// At tens of millions of signatures per second that copy needs several GB/s,
// near one core's memcpy rate, so a chunk's copy is split into parts run by
// the calling thread and the pool's helpers.  Parts are claimed under the
// pool's mutex; run() returns when every part has finished, so the function
// it is given (and what that function refers to) only has to outlive the call.
#pragma once
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace uf {

class PackPool {
public:
    // threads: total threads working on a run() (the caller included); 1 = no helpers.
    explicit PackPool(int threads);
    ~PackPool();
    PackPool(const PackPool&) = delete;
    PackPool& operator=(const PackPool&) = delete;

    int threads() const { return (int)helpers_.size() + 1; }
    // fn(part) for every part in [0, parts), on the caller and the helpers.
    void run(int parts, const std::function<void(int)>& fn);

private:
    void helper();

    std::vector<std::thread> helpers_;
    std::mutex mu_;
    std::condition_variable work_cv_, done_cv_;
    const std::function<void(int)>* fn_ = nullptr;
    int parts_ = 0, next_ = 0, remaining_ = 0;
    bool stop_ = false;
};

}  // namespace uf
