"""Field observation slot protocol on the CPU: the host-only header
numi-gpu-physics_b200/csrc/bfx_observation.h (selectCaptureSlot,
publishFieldSlot, abandonFieldSlot, acquireLatestGPUFieldFrame,
releaseFieldSlot and currentPublishedFieldSlot of
BirdFlowSimulation.swift:1148-1171, 1806-1918) compiled with g++ into a small
driver.  The scenarios follow ObservationAndCheckpointTests.swift:62-87
(exhausted viewer slots drop without waiting) and the wait / release rules of
the reference's NSCondition protocol."""
from __future__ import annotations

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "numi-gpu-physics_b200", "csrc")

DRIVER = r'''
#include <cstdio>
#include <thread>
#include "bfx_observation.h"
using namespace bfx;
struct Snap { unsigned long long step; };
struct Meta { Snap snapshot; int tag; };
static Meta at(unsigned long long step) { Meta m; m.snapshot.step = step; m.tag = (int)step; return m; }
#define CHECK(c) do { if (!(c)) { std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); return 1; } } while (0)
typedef FieldSlots<Meta> Slots;

static int exhausted_viewer_slots_drop_without_waiting() {
    Slots s(3);
    s.reset(at(0));                                   // initial frame in slot 0
    Meta m; int slot = -1;
    uint64_t first = s.acquire(false, 0, &m, &slot);
    CHECK(first != 0 && slot == 0 && m.snapshot.step == 0);
    int w = s.select(CaptureMode::BestEffort, 0);
    CHECK(w == 1);
    s.publish(w, at(1));
    uint64_t second = s.acquire(false, 0, &m, &slot);
    CHECK(second != 0 && slot == 1 && m.snapshot.step == 1);
    w = s.select(CaptureMode::BestEffort, 0);
    CHECK(w == 2);
    s.publish(w, at(2));
    uint64_t third = s.acquire(false, 0, &m, &slot);
    CHECK(third != 0 && slot == 2);
    CHECK(s.select(CaptureMode::BestEffort, 0) == kNoSlot);
    CHECK(s.dropped() == 1 && s.waits() == 0);
    CHECK(s.release(first) && s.release(second) && s.release(third));
    CHECK(!s.release(third));                         // releasing twice is a no-op
    CHECK(s.idle());
    return 0;
}

static int publication_supersedes_and_after_step() {
    Slots s(3);
    s.reset(at(0));
    int a = s.select(CaptureMode::Required, 0);       // a free slot before a published one
    CHECK(a == 1);
    s.publish(a, at(5));
    CHECK(s.state(0) == Slots::Free);                 // the unleased older frame is freed
    CHECK(s.current() == 1);
    Meta m; int slot = -1;
    CHECK(s.acquire(true, 5, &m, &slot) == 0);        // not newer than step 5
    uint64_t l = s.acquire(true, 4, &m, &slot);
    CHECK(l != 0 && slot == 1 && m.tag == 5);
    CHECK(s.acquire(false, 0, &m, &slot) == 0);       // only the newest frame is leased, once
    CHECK(s.current() == 0);                          // no published frame: slot 0
    CHECK(s.leased_slot(l) == 1);
    int b = s.select(CaptureMode::Disabled, 0);
    CHECK(b == kNoSlot && s.dropped() == 0);
    b = s.select(CaptureMode::Required, 0);
    CHECK(b == 0);
    s.abandon(b);                                     // a failed capture gives the slot back
    CHECK(s.state(0) == Slots::Free);
    CHECK(s.release(l) && s.leased_slot(l) == -1);
    return 0;
}

static int published_slot_is_reused_when_none_is_free() {
    Slots s(2);
    s.reset(at(0));
    Meta m; int slot = -1;
    uint64_t l = s.acquire(false, 0, &m, &slot);     // slot 0 leased
    int w = s.select(CaptureMode::Required, 0);
    CHECK(w == 1);
    s.publish(w, at(1));
    w = s.select(CaptureMode::BestEffort, 0);        // slot 1 published, not leased: overwritten
    CHECK(w == 1 && s.current() == 0);
    s.publish(w, at(2));
    CHECK(s.current() == 1 && s.dropped() == 0);
    s.release(l);
    return 0;
}

static int required_capture_waits_for_a_release() {
    Slots s(1);
    s.reset(at(0));
    Meta m; int slot = -1;
    uint64_t l = s.acquire(false, 0, &m, &slot);
    std::thread consumer([&] {
        std::this_thread::sleep_for(std::chrono::milliseconds(100));
        s.release(l);
    });
    int w = s.select(CaptureMode::Required, 5000);
    consumer.join();
    CHECK(w == 0);
    CHECK(s.waits() >= 1 && s.dropped() == 0);
    s.publish(w, at(1));
    return 0;
}

static int required_capture_wait_limit() {
    Slots s(1);
    s.reset(at(0));
    Meta m; int slot = -1;
    uint64_t l = s.acquire(false, 0, &m, &slot);
    CHECK(s.select(CaptureMode::Required, 50) == kSlotWaitTimeout);
    CHECK(s.waits() >= 1);
    CHECK(s.state(0) == Slots::Leased);               // nothing changed
    s.release(l);
    CHECK(s.select(CaptureMode::Required, 50) == 0);
    return 0;
}

static int reset_forfeits_leases() {
    Slots s(2);
    s.reset(at(0));
    Meta m; int slot = -1;
    uint64_t l = s.acquire(false, 0, &m, &slot);
    s.reset(at(7));                                   // restore
    CHECK(s.leased_slot(l) == -1 && !s.release(l));
    uint64_t l2 = s.acquire(false, 0, &m, &slot);
    CHECK(l2 != 0 && l2 != l && m.tag == 7 && slot == 0);
    return 0;
}

int main() {
    int rc = 0;
    rc |= exhausted_viewer_slots_drop_without_waiting();
    rc |= publication_supersedes_and_after_step();
    rc |= published_slot_is_reused_when_none_is_free();
    rc |= required_capture_waits_for_a_release();
    rc |= required_capture_wait_limit();
    rc |= reset_forfeits_leases();
    if (rc == 0) std::printf("OK\n");
    return rc;
}
'''


def test_observation_slot_protocol(tmp_path):
    src = tmp_path / "slots.cpp"
    exe = tmp_path / "slots"
    src.write_text(DRIVER)
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "OK", out.stdout + out.stderr


def test_capture_mode_names():
    from bfx.simulation import _capture_mode
    import bfx._lib as L
    assert _capture_mode("required") == L.FIELD_CAPTURE_REQUIRED
    assert _capture_mode("bestEffort") == L.FIELD_CAPTURE_BEST_EFFORT
    assert _capture_mode("disabled") == L.FIELD_CAPTURE_DISABLED
    assert _capture_mode(True) == L.FIELD_CAPTURE_REQUIRED and _capture_mode(False) == L.FIELD_CAPTURE_DISABLED
    with pytest.raises(ValueError):
        _capture_mode("latest")


STRESS = r'''
#include <atomic>
#include <cstdio>
#include <set>
#include <thread>
#include <vector>
#include "bfx_observation.h"
using namespace bfx;
struct Snap { unsigned long long step; };
struct Meta { Snap snapshot; };
int main() {
    FieldSlots<Meta> s(3);
    Meta m0; m0.snapshot.step = 0;
    s.reset(m0);
    std::atomic<bool> done(false);
    std::atomic<long> leased(0), bad(0);
    std::vector<std::thread> consumers;
    std::vector<std::vector<uint64_t>> ids(3);
    for (int c = 0; c < 3; ++c) {
        consumers.emplace_back([&, c] {
            unsigned long long last = 0;
            while (!done.load()) {
                Meta m; int slot = -1;
                uint64_t l = s.acquire(false, 0, &m, &slot);
                if (l) {
                    ++leased;
                    ids[c].push_back(l);
                    if (slot < 0 || slot > 2 || s.leased_slot(l) != slot) ++bad;
                    if (m.snapshot.step < last) ++bad;   // newest frames only move forward per consumer
                    last = m.snapshot.step;
                    std::this_thread::yield();
                    if (!s.release(l)) ++bad;
                    if (s.release(l)) ++bad;             // a second release is a no-op
                }
            }
        });
    }
    unsigned long long step = 0;
    for (int i = 0; i < 20000; ++i) {
        const CaptureMode mode = (i % 3 == 0) ? CaptureMode::Required : CaptureMode::BestEffort;
        const int w = s.select(mode, 1000);
        if (w == kSlotWaitTimeout) { ++bad; continue; }
        if (w < 0) continue;
        Meta m; m.snapshot.step = ++step;
        if (i % 97 == 0) s.abandon(w);
        else s.publish(w, m);
    }
    done = true;
    for (auto& t : consumers) t.join();
    std::set<uint64_t> all;
    size_t n = 0;
    for (auto& v : ids) { n += v.size(); all.insert(v.begin(), v.end()); }
    if (all.size() != n) ++bad;                       // lease ids are never reused
    if (!s.idle()) ++bad;
    std::printf("%s leased=%ld dropped=%llu waits=%llu\n", bad.load() ? "BAD" : "OK", leased.load(),
                (unsigned long long)s.dropped(), (unsigned long long)s.waits());
    return bad.load() ? 1 : 0;
}
'''


def test_observation_slots_under_concurrent_consumers(tmp_path):
    """Three consumer threads lease and release the newest frame while the
    advancing thread captures (best-effort and required with a wait limit),
    publishes and abandons 20,000 frames; built with ThreadSanitizer when the
    compiler has it.  Leases stay unique, each consumer's frames move forward,
    double releases are no-ops and every slot ends free."""
    src = tmp_path / "stress.cpp"
    src.write_text(STRESS)
    exe = tmp_path / "stress"
    base = ["g++", "-std=c++17", "-O1", "-pthread", "-I", CSRC, str(src), "-o", str(exe)]
    tsan = subprocess.run(base[:2] + ["-fsanitize=thread", "-g"] + base[2:], capture_output=True, text=True)
    if tsan.returncode != 0:
        subprocess.run(base, check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK"), out.stdout
    assert "WARNING: ThreadSanitizer" not in out.stderr, out.stderr[:2000]
