// alloc_set.hpp -- all-or-nothing allocation of a set of buffers.
//
// A handle allocates some buffer sets lazily, the first time an option needs
// them (the Krylov work vectors, the Anderson history), and tests "is the set
// there" by its first pointer.  If one allocation of the set failed after
// others had succeeded, a retried call would take the set as present and use
// null pointers.  alloc_set() allocates every buffer of a set into locals and
// stores them into their slots only when all succeeded; on a failure it
// releases what it got and leaves every slot untouched (null).
//
// Header-only and free of CUDA types, so the host tests can drive it with a
// failing allocator (tests/cpp/alloc_set_test.cpp).
#pragma once

#include <cstddef>

namespace lbm {

struct AllocSlot {
    void** slot;       // where the pointer goes on success
    std::size_t bytes;
    int kind;          // passed through to the allocator (e.g. device or pinned host)
};

// alloc(kind, void** out, bytes) -> bool; release(kind, void* p).
template <class Alloc, class Release>
bool alloc_set(const AllocSlot* slots, int n, Alloc alloc, Release release)
{
    constexpr int kMax = 16;
    if (n < 0 || n > kMax) return false;
    void* got[kMax] = {};
    for (int i = 0; i < n; ++i) {
        if (!alloc(slots[i].kind, &got[i], slots[i].bytes) || !got[i]) {
            for (int j = 0; j < i; ++j) release(slots[j].kind, got[j]);
            return false;
        }
    }
    for (int i = 0; i < n; ++i) *slots[i].slot = got[i];
    return true;
}

}  // namespace lbm
