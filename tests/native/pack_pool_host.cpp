// Test harness: the host pack pool (csrc/pack_pool.cpp) driven from Python.
#include <atomic>
#include <vector>

#include "../../ultrafastsecp256k1_b200/csrc/pack_pool.cpp"

extern "C" {

// `runs` rounds of run(parts) on a pool of `threads`; each part fills its own
// slice of a buffer and counts its calls.  Returns 0 when every part ran
// exactly once per round and every slice was written before run() returned,
// else the first failing round + 1.
int pp_check(int threads, int parts, int runs) {
    uf::PackPool pool(threads);
    if (pool.threads() != (threads < 1 ? 1 : threads)) return -1;
    std::vector<int> buf(parts * 64);
    std::vector<std::atomic<int>> calls(parts);
    for (int r = 0; r < runs; ++r) {
        for (auto& c : calls) c.store(0);
        const std::function<void(int)> fn = [&](int p) {
            calls[p].fetch_add(1);
            for (int i = 0; i < 64; ++i) buf[p * 64 + i] = r * 1000 + p;
        };
        pool.run(parts, fn);
        for (int p = 0; p < parts; ++p) {
            if (calls[p].load() != 1) return r + 1;
            for (int i = 0; i < 64; ++i)
                if (buf[p * 64 + i] != r * 1000 + p) return r + 1;
        }
    }
    return 0;
}

}
