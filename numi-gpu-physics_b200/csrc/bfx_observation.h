// Observation slots of the macroscopic fields: the reference's field
// publication protocol (BirdFlowSimulation.swift:456-478 state,
// 1148-1171 acquireLatestGPUFieldFrame, 1806-1918 selectCaptureSlot /
// publishFieldSlot / abandonFieldSlot / releaseFieldSlot /
// currentPublishedFieldSlot).
//
// Each slot holds one density + velocity volume and its metadata and moves
// through free -> writing -> published -> leased -> free.  A capture takes a
// free slot, else the oldest-index published one; a required capture waits
// for a release when every slot is leased or being written, a best-effort
// capture drops the frame instead.  Publishing a slot frees the previously
// published, unleased one; acquiring leases only the newest published slot.
//
// Host-only C++ (no CUDA): the advancing thread and consumer threads share
// one mutex and condition variable, and a release may come from a CUDA host
// callback once a consumer's reads have completed.
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <vector>

namespace bfx {

enum class CaptureMode : int { Required = 0, BestEffort = 1, Disabled = 2 };

// select() results besides a slot index
constexpr int kNoSlot = -1;         // disabled, or best-effort with no slot available (dropped)
constexpr int kSlotWaitTimeout = -2;  // required, and no slot came free within the wait limit

template <class Meta>
class FieldSlots {
public:
    enum State { Free, Writing, Published, Leased };

    explicit FieldSlots(int count) : state_(count, Free), meta_(count), lease_(count, 0) {}

    int count() const { return (int)state_.size(); }

    // selectCaptureSlot.  timeout_ms <= 0 waits without limit, as the
    // reference does; a positive limit bounds the wait of a required capture.
    int select(CaptureMode mode, int64_t timeout_ms) {
        if (mode == CaptureMode::Disabled) return kNoSlot;
        std::unique_lock<std::mutex> lk(mu_);
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
        for (;;) {
            int index = first(Free);
            if (index < 0) index = first(Published);
            if (index >= 0) {
                if (latest_ == index) latest_ = -1;
                state_[index] = Writing;
                return index;
            }
            if (mode == CaptureMode::BestEffort) {
                ++dropped_;
                return kNoSlot;
            }
            ++waits_;
            if (timeout_ms <= 0) {
                cv_.wait(lk);
            } else if (cv_.wait_until(lk, deadline) == std::cv_status::timeout) {
                int again = first(Free);
                if (again < 0) again = first(Published);
                if (again < 0) return kSlotWaitTimeout;
            }
        }
    }

    // publishFieldSlot: index must be Writing.
    void publish(int index, const Meta& meta) {
        std::lock_guard<std::mutex> lk(mu_);
        if (latest_ >= 0 && latest_ != index && state_[latest_] == Published) state_[latest_] = Free;
        meta_[index] = meta;
        state_[index] = Published;
        latest_ = index;
        cv_.notify_all();
    }

    // abandonFieldSlot: a capture that failed gives its slot back.
    void abandon(int index) {
        std::lock_guard<std::mutex> lk(mu_);
        if (index >= 0 && index < count() && state_[index] == Writing) state_[index] = Free;
        cv_.notify_all();
    }

    // acquireLatestGPUFieldFrame: the lease id (0: nothing newer to lease).
    uint64_t acquire(bool has_after, uint64_t after_step, Meta* out, int* slot) {
        std::lock_guard<std::mutex> lk(mu_);
        if (latest_ < 0 || state_[latest_] != Published) return 0;
        if (has_after && !(step_of(meta_[latest_]) > after_step)) return 0;
        const int index = latest_;
        state_[index] = Leased;
        latest_ = -1;
        lease_[index] = ++next_lease_;
        if (out) *out = meta_[index];
        if (slot) *slot = index;
        return lease_[index];
    }

    // The slot a live lease holds (-1 when the lease was released or never issued).
    int leased_slot(uint64_t lease) {
        std::lock_guard<std::mutex> lk(mu_);
        return find_lease(lease);
    }

    // releaseFieldSlot: releasing twice, or a lease that is no longer live, is a no-op.
    bool release(uint64_t lease) {
        std::lock_guard<std::mutex> lk(mu_);
        const int index = find_lease(lease);
        if (index < 0) return false;
        state_[index] = Free;
        lease_[index] = 0;
        cv_.notify_all();
        return true;
    }

    // currentPublishedFieldSlot: the newest published slot, else slot 0.
    int current() {
        std::lock_guard<std::mutex> lk(mu_);
        return latest_ >= 0 ? latest_ : 0;
    }

    // Initialisation and restore: every slot free, then slot 0 published.
    // Live leases are forfeited (their release becomes a no-op).
    void reset(const Meta& meta) {
        std::lock_guard<std::mutex> lk(mu_);
        for (int i = 0; i < count(); ++i) {
            state_[i] = Free;
            lease_[i] = 0;
        }
        meta_[0] = meta;
        state_[0] = Published;
        latest_ = 0;
        cv_.notify_all();
    }

    // No slot is leased or being written.
    bool idle() {
        std::lock_guard<std::mutex> lk(mu_);
        for (State s : state_)
            if (s == Leased || s == Writing) return false;
        return true;
    }

    State state(int index) {
        std::lock_guard<std::mutex> lk(mu_);
        return state_[index];
    }
    uint64_t dropped() {
        std::lock_guard<std::mutex> lk(mu_);
        return dropped_;
    }
    uint64_t waits() {
        std::lock_guard<std::mutex> lk(mu_);
        return waits_;
    }
    // a replacement slot set keeps counting from its predecessor's totals
    void add_counters(uint64_t dropped, uint64_t waits) {
        std::lock_guard<std::mutex> lk(mu_);
        dropped_ += dropped;
        waits_ += waits;
    }

private:
    static uint64_t step_of(const Meta& m) { return m.snapshot.step; }
    int first(State s) const {
        for (int i = 0; i < count(); ++i)
            if (state_[i] == s) return i;
        return -1;
    }
    int find_lease(uint64_t lease) const {
        if (lease == 0) return -1;
        for (int i = 0; i < count(); ++i)
            if (state_[i] == Leased && lease_[i] == lease) return i;
        return -1;
    }

    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<State> state_;
    std::vector<Meta> meta_;
    std::vector<uint64_t> lease_;
    int latest_ = -1;
    uint64_t next_lease_ = 0;
    uint64_t dropped_ = 0;
    uint64_t waits_ = 0;
};

}  // namespace bfx
