// Binomial checkpointing (host code): the order of forward steps, stored states and reversed
// steps that reverses an n-step run with a fixed number of state slots and the fewest forward
// steps, the strategy of Griewank and Walther's "revolve" (ACM TOMS 26, 2000), restated here as
// a recursion with a closed-form cost.
//
// Model: the run's initial state is held in slot 0; `slots` more states fit.  Reversing step j
// needs the state before it (state j) to be current.  To reverse steps [a, b) with the state a
// held and s free slots: one step is reversed at once; with no free slot, each step j = b-1 .. a
// is reached again from state a; otherwise advance a -> m, store state m, reverse [m, b) with one
// slot fewer, release it and reverse [a, m).  The number of forward steps F(l, s) for l = b - a
// then satisfies F(1, s) = 0, F(l, 0) = l(l-1)/2 and F(l, s) = min_m m + F(l-m, s-1) + F(m, s),
// whose minimum has the closed form
//     F(l, s) = t l - C(s+t+1, t-1),  t the least integer with C(s+1+t, t) >= l,
// (with s+1 the snapshot count of the revolve papers); the split m is chosen by evaluating it.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace dasha {

struct CkptAction {
    enum Kind : int { Restore = 0, Advance = 1, Store = 2, Release = 3, Reverse = 4 };
    int kind;
    int a;      // Restore: slot; Advance: from step; Store / Release: slot; Reverse: step
    int b;      // Advance: to step; Store: the step whose state is stored
};

// C(n, k), saturating at `cap` (the callers only compare it with step counts)
inline long long binom_capped(long long n, long long k, long long cap) {
    if (k < 0 || n < 0 || k > n) return 0;
    k = std::min(k, n - k);
    long long r = 1;
    for (long long i = 1; i <= k; ++i) {
        const long long f = n - k + i;
        if (r > cap / f) return cap;   // r * f would pass the cap
        r = r * f / i;                 // exact: r * f = C(n-k+i, i) * i
    }
    return std::min(r, cap);
}

// F(l, s): the fewest forward steps that reverse l steps with s free slots
inline long long binomial_cost(long long l, long long s) {
    if (l <= 1) return 0;
    if (s <= 0) return l * (l - 1) / 2;
    const long long cap = (long long)1 << 62;
    long long t = 0;
    while (binom_capped(s + 1 + t, t, cap) < l) ++t;
    return t * l - binom_capped(s + t + 1, t - 1, cap);
}

inline int binomial_split(int l, int s) {
    int best = 1;
    long long bc = -1;
    for (int m = 1; m < l; ++m) {
        const long long c = m + binomial_cost(l - m, s - 1) + binomial_cost(m, s);
        if (bc < 0 || c < bc) { bc = c; best = m; }
    }
    return best;
}

namespace detail {
inline void reverse_range(int a, int b, int base_slot, std::vector<int>& free_slots, int& current,
                          std::vector<CkptAction>& out) {
    auto reach = [&](int j) {   // make state j current, starting from the held state a
        if (current != a) { out.push_back({CkptAction::Restore, base_slot, a}); current = a; }
        if (j > current) { out.push_back({CkptAction::Advance, current, j}); current = j; }
    };
    if (b - a == 1) {
        reach(a);
        out.push_back({CkptAction::Reverse, a, 0});
        current = -1;
        return;
    }
    if (free_slots.empty()) {
        for (int j = b - 1; j >= a; --j) {
            reach(j);
            out.push_back({CkptAction::Reverse, j, 0});
            current = -1;
        }
        return;
    }
    const int m = a + binomial_split(b - a, (int)free_slots.size());
    reach(m);
    const int slot = free_slots.back();
    free_slots.pop_back();
    out.push_back({CkptAction::Store, slot, m});
    reverse_range(m, b, slot, free_slots, current, out);
    out.push_back({CkptAction::Release, slot, m});
    free_slots.push_back(slot);
    reverse_range(a, m, base_slot, free_slots, current, out);
}
}  // namespace detail

// The actions that reverse steps n-1 .. 0 with slots 1..`slots` free (slot 0 holds state 0 and
// is current at the start).  The Advance actions add up to binomial_cost(n, slots) steps.
inline std::vector<CkptAction> binomial_schedule(int n, int slots) {
    std::vector<CkptAction> out;
    if (n <= 0) return out;
    std::vector<int> free_slots;
    for (int q = std::max(slots, 0); q >= 1; --q) free_slots.push_back(q);
    int current = 0;
    detail::reverse_range(0, n, 0, free_slots, current, out);
    return out;
}

}  // namespace dasha
