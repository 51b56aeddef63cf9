// Host test of lbm_b200/csrc/alloc_set.hpp with a fake allocator that fails
// on its k-th call: after a failure every slot is still null and every buffer
// that was obtained has been released; after a success every slot is set.
// Exit code 0 on success.
#include <cstdio>
#include <cstdlib>
#include <set>

#include "../../lbm_b200/csrc/alloc_set.hpp"

int main()
{
    constexpr int n = 8;
    for (int fail_at = 0; fail_at <= n; ++fail_at) {
        void* slots[n] = {};
        lbm::AllocSlot set[n];
        for (int i = 0; i < n; ++i) set[i] = {&slots[i], 64u * (i + 1), i % 2};
        int calls = 0;
        std::set<void*> live;
        auto alloc = [&](int, void** p, std::size_t bytes) {
            if (calls++ == fail_at) return false;
            *p = std::malloc(bytes);
            live.insert(*p);
            return true;
        };
        auto release = [&](int, void* p) {
            if (!live.erase(p)) std::exit(10);   // released twice or never allocated
            std::free(p);
        };
        const bool ok = lbm::alloc_set(set, n, alloc, release);
        if (fail_at < n) {
            if (ok) return 11;
            for (void* s : slots)
                if (s) return 12;                // a slot was written on failure
            if (!live.empty()) return 13;        // a buffer leaked
        } else {
            if (!ok) return 14;
            for (void* s : slots)
                if (!s || !live.count(s)) return 15;
            for (void* s : slots) std::free(s);
        }
    }
    std::puts("alloc_set ok");
    return 0;
}
