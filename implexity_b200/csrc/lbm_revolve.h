// lbm_revolve.h -- the binomial checkpoint schedule ("revolve") of the
// horizon adjoint, built on the host.
//
// Restates BinomialSchedule::new and its builder (implexity-ad/src/
// revolve.rs:128-283): a chain of `length` steps starting at state a, whose
// start is held in slot `own`, with `slots` slots available, is advanced to
// the optimal split point m, the state there is stored in a fresh slot, the
// tail chain (length - m steps, one slot fewer) is reversed recursively, the
// slot is released, and the loop continues with the head chain of m steps.
// The split is the largest m allowed by the binomial bounds of revolve.rs:
// 230-245 (beta(s, r) = C(s + r, s), r = repetitions).  The first reverse
// step is preceded by the advance of the last step (T-1 -> T), which
// produces the final state that seeds the adjoint.  The total of advanced
// steps is optimal_forward_steps (revolve.rs:90-125); revolve_plan checks it
// and replays the action list against a model of the slots before returning.
#pragma once

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace lbm {

struct RevolveAction {
    enum Kind { ADVANCE, SNAPSHOT, RESTORE, REVERSE, RELEASE };
    Kind kind;
    int64_t a;  // ADVANCE: from; SNAPSHOT, RESTORE: state index; REVERSE: step k (state k-1 -> k); RELEASE: slot
    int64_t b;  // ADVANCE: to; SNAPSHOT, RESTORE: slot
};

struct RevolvePlan {
    std::vector<RevolveAction> actions;
    size_t reverse_start = 0;   // index of the first action after the forward sweep
    int64_t forward_steps = 0;  // steps advanced in all, forward sweep included
    int64_t peak = 0;           // most slots held at once
};

namespace revolve_detail {

using u128 = unsigned __int128;
constexpr u128 kSaturated = (u128)1 << 100;

// C(s + r, s), saturating at kSaturated; 0 for r < 0.
inline u128 beta(int64_t s, int64_t r) {
    if (r < 0) return 0;
    u128 v = 1;
    for (int64_t i = 1; i <= r; ++i) {
        v = v * (u128)(s + i) / (u128)i;
        if (v >= kSaturated) return kSaturated;
    }
    return v;
}

// The smallest r with C(s + r, r) >= steps (0 for steps <= 1).
inline int64_t repetitions(int64_t steps, int64_t s) {
    if (steps <= 1) return 0;
    int64_t r = 0;
    u128 v = 1;
    while (v < (u128)steps) {
        ++r;
        v = v * (u128)(s + r) / (u128)r;
    }
    return r;
}

// Steps advanced to reverse a chain of `length` steps with `s` slots.
inline u128 chain_advances(int64_t length, int64_t s) {
    if (length <= 1) return 0;
    const int64_t r = repetitions(length, s);
    const u128 v = beta(s, r);
    return (u128)r * (u128)length - v * (u128)r / (u128)(s + 1);
}

inline int64_t split(int64_t length, int64_t slots) {
    if (slots < 1) throw std::invalid_argument("a chain of more than one step needs a snapshot slot");
    if (slots == 1) return length - 1;
    const int64_t r = repetitions(length, slots);
    const u128 l = (u128)length;
    auto sub = [](u128 x, u128 y) { return x > y ? x - y : (u128)0; };
    const u128 lo = std::max({(u128)1, beta(slots, r - 2), sub(l, beta(slots - 1, r))});
    const u128 hi = std::min({l - 1, beta(slots, r - 1), sub(l, beta(slots - 1, r - 1))});
    if (lo > hi)
        throw std::invalid_argument("no optimal split for a chain of " + std::to_string(length) + " steps with " +
                                    std::to_string(slots) + " slots");
    return (int64_t)hi;
}

class Builder {
public:
    Builder(int64_t steps, int64_t slots) : steps_(steps) {
        for (int64_t s = slots - 1; s >= 0; --s) free_.push_back(s);  // back() = lowest slot
    }
    RevolvePlan run(int64_t slots) {
        const int64_t own = take();
        plan_.actions.push_back({RevolveAction::SNAPSHOT, 0, own});
        cursor_ = 0;
        chain(0, steps_, own, slots);
        plan_.forward_steps = advanced_;
        plan_.peak = peak_;
        return std::move(plan_);
    }

private:
    int64_t take() {
        if (free_.empty()) throw std::invalid_argument("checkpoint schedule ran out of snapshot slots");
        const int64_t s = free_.back();
        free_.pop_back();
        peak_ = std::max(peak_, ++in_use_);
        return s;
    }
    void release(int64_t s) {
        plan_.actions.push_back({RevolveAction::RELEASE, s, 0});
        --in_use_;
        free_.push_back(s);
        std::sort(free_.begin(), free_.end(), [](int64_t x, int64_t y) { return x > y; });
    }
    void advance(int64_t from, int64_t to) {
        if (to <= from) return;
        plan_.actions.push_back({RevolveAction::ADVANCE, from, to});
        advanced_ += to - from;
        cursor_ = to;
    }
    void at(int64_t position, int64_t slot) {
        if (cursor_ != position) {
            plan_.actions.push_back({RevolveAction::RESTORE, position, slot});
            cursor_ = position;
        }
    }
    void reverse(int64_t k) {
        if (!started_) {
            plan_.actions.push_back({RevolveAction::ADVANCE, steps_ - 1, steps_});
            ++advanced_;
            started_ = true;
            plan_.reverse_start = plan_.actions.size();
        }
        plan_.actions.push_back({RevolveAction::REVERSE, k, 0});
        cursor_ = -1;
    }
    void chain(int64_t a, int64_t length, int64_t own, int64_t slots) {
        while (true) {
            if (length == 0) return;
            if (length == 1) {
                at(a, own);
                reverse(a + 1);
                return;
            }
            const int64_t m = split(length, slots);
            at(a, own);
            advance(a, a + m);
            if (length - m > 1) {
                const int64_t s = take();
                plan_.actions.push_back({RevolveAction::SNAPSHOT, a + m, s});
                chain(a + m, length - m, s, slots - 1);
                release(s);
            } else {
                reverse(a + length);
            }
            length = m;
        }
    }

    int64_t steps_;
    RevolvePlan plan_;
    std::vector<int64_t> free_;
    int64_t in_use_ = 0, peak_ = 0, advanced_ = 0, cursor_ = -1;
    bool started_ = false;
};

}  // namespace revolve_detail

// optimal_forward_steps (revolve.rs:117-125): the fewest steps any schedule
// with `snapshots` states advances for `steps` steps.
inline int64_t revolve_optimal_forward(int64_t steps, int64_t snapshots) {
    if (steps <= 0) return 0;
    if (steps == 1) return 1;
    const revolve_detail::u128 v = revolve_detail::chain_advances(steps, snapshots) + 1;
    return v > (revolve_detail::u128)INT64_MAX ? INT64_MAX : (int64_t)v;
}

// The schedule for `steps` >= 1 and `snapshots` >= 1 slots.  Throws
// std::invalid_argument on bad sizes, std::logic_error if the replay of the
// action list finds an inconsistency.
inline RevolvePlan revolve_plan(int64_t steps, int64_t snapshots) {
    if (steps < 1) throw std::invalid_argument("a checkpoint schedule needs at least one step");
    if (snapshots < 1) throw std::invalid_argument("binomial checkpointing needs at least one snapshot");
    RevolvePlan p = revolve_detail::Builder(steps, snapshots).run(snapshots);
    if (p.forward_steps != revolve_optimal_forward(steps, snapshots))
        throw std::logic_error("binomial schedule is not optimal");
    // replay: every state reached, stored and restored where the plan says;
    // every step reversed once, in decreasing order
    std::vector<int64_t> slot(snapshots, -1);
    int64_t cursor = 0, next_reverse = steps;
    bool forward = true;
    for (size_t i = 0; i < p.actions.size(); ++i) {
        const RevolveAction& x = p.actions[i];
        if (i == p.reverse_start) {
            if (cursor != steps) throw std::logic_error("forward sweep does not end at the final state");
            cursor = steps - 1;  // the state before the last step is still held
            forward = false;
        }
        switch (x.kind) {
            case RevolveAction::ADVANCE:
                if (cursor != x.a || x.b <= x.a) throw std::logic_error("advance from a state not held");
                cursor = x.b;
                break;
            case RevolveAction::SNAPSHOT:
                if (cursor != x.a || x.b < 0 || x.b >= snapshots || slot[x.b] != -1)
                    throw std::logic_error("snapshot of a state not held or into a used slot");
                slot[x.b] = x.a;
                break;
            case RevolveAction::RESTORE:
                if (forward || x.b < 0 || x.b >= snapshots || slot[x.b] != x.a)
                    throw std::logic_error("restore of a state the slot does not hold");
                cursor = x.a;
                break;
            case RevolveAction::REVERSE:
                if (forward || x.a != next_reverse || cursor != x.a - 1)
                    throw std::logic_error("reverse of a step whose state is not held");
                --next_reverse;
                cursor = -1;
                break;
            case RevolveAction::RELEASE:
                if (x.a < 0 || x.a >= snapshots || slot[x.a] == -1) throw std::logic_error("release of a free slot");
                slot[x.a] = -1;
                break;
        }
    }
    if (next_reverse != 0) throw std::logic_error("not every step was reversed");
    return p;
}

}  // namespace lbm
