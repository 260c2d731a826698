// Host model of the lap-tagged MPMC ring protocol (gtap_b200/csrc/gtap_ring.h),
// compiled with g++ by tests/test_ring_model_cpu.py.  It uses the same
// encoding functions as the device code and replays the protocol of
// ring_push_warp / ring_push_one / ring_pop_warp (gtap_device.cuh) and of the
// launch reset (head moved to tail) as interleaved steps of simulated
// producers and consumers, then checks that a consumer only ever accepts the
// word written for its own position.  Exit status 0 = every check passed;
// each failed check prints one line.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include "../gtap_b200/csrc/gtap_ring.h"

using gtap::ring_tag_of;
using gtap::ring_word_of;
using gtap::ring_word_ready;
using gtap::ring_word_value;

static int g_failures = 0;
#define CHECK(cond, ...)                                  \
    do {                                                  \
        if (!(cond)) {                                    \
            ++g_failures;                                 \
            std::printf("FAIL line %d: ", __LINE__);      \
            std::printf(__VA_ARGS__);                     \
            std::printf("\n");                            \
        }                                                 \
    } while (0)

struct Ring {
    std::vector<uint64_t> slots;
    uint32_t head = 0, tail = 0, cap_log2;
    explicit Ring(uint32_t lg) : slots(size_t(1) << lg, 0), cap_log2(lg) {}
    uint32_t mask() const { return (1u << cap_log2) - 1u; }
    uint32_t reserve(uint32_t n) { uint32_t p = tail; tail += n; return p; }   // atomicAdd on tail
    void write(uint32_t p, int32_t v) { slots[p & mask()] = ring_word_of(p, cap_log2, v); }
    void reset() { head = tail; }                                           // launch reset
    bool ready(uint32_t p) const { return ring_word_ready(slots[p & mask()], p, cap_log2); }
    int32_t value(uint32_t p) const { return ring_word_value(slots[p & mask()]); }
};

// The encoding used before: a 16-bit launch epoch and a 16-bit lap, cursors
// reset to 0 at every launch.
static uint64_t old_word(uint32_t epoch, uint32_t pos, uint32_t cap_log2, int32_t v) {
    uint32_t tag = ((epoch & 0xFFFFu) << 16) | ((pos >> cap_log2) & 0xFFFFu);
    return (uint64_t(tag) << 32) | uint32_t(v + 1);
}
static bool old_ready(uint64_t w, uint32_t epoch, uint32_t pos, uint32_t cap_log2) {
    return uint32_t(w >> 32) == (((epoch & 0xFFFFu) << 16) | ((pos >> cap_log2) & 0xFFFFu));
}

// 1. A never-written slot never matches (tags start at 1).
static void fresh_ring() {
    for (uint32_t lg : {8u, 12u, 20u, 27u}) {
        Ring r(lg);
        for (uint32_t p = 0; p < 64; ++p) CHECK(!r.ready(p), "fresh slot of position %u matched (cap 2^%u)", p, lg);
        CHECK(!r.ready(0xFFFFFFFFu), "fresh slot of the last position matched (cap 2^%u)", lg);
        CHECK(ring_tag_of(0, lg) == 1u, "tag of position 0 must be 1");
    }
}

// 2. A slot written for any other position with the same index is refused:
//    every earlier lap, and the laps on both sides of the 2^32 wrap.
static void stale_laps() {
    for (uint32_t lg : {8u, 10u, 20u, 27u}) {
        const uint32_t cap = 1u << lg;
        const uint32_t laps = 1u << (32 - lg);
        std::mt19937 rng(lg);
        for (int t = 0; t < 4000; ++t) {
            uint32_t p = rng();
            uint32_t k = 1 + rng() % (laps - 1);   // any other lap of the same slot
            uint32_t q = p - k * cap;              // mod 2^32
            uint64_t w = ring_word_of(q, lg, 7);
            CHECK(!ring_word_ready(w, p, lg), "stale word of position %u accepted for %u (cap 2^%u)", q, p, lg);
            CHECK(ring_word_ready(ring_word_of(p, lg, 7), p, lg), "own word refused");
        }
        // across the wrap: the last lap before 2^32 and the first after it
        uint32_t last = 0u - cap;          // first position of the last lap
        for (uint32_t i = 0; i < cap && i < 4096; ++i) {
            uint64_t w = ring_word_of(last + i, lg, 1);
            CHECK(!ring_word_ready(w, i, lg), "wrap: lap 2^%u-1 slot accepted for lap 0 (i=%u)", 32 - lg, i);
            CHECK(!ring_word_ready(ring_word_of(i, lg, 1), last + i, lg), "wrap: lap 0 slot accepted for the last lap");
        }
    }
}

// 3. The scenario of the old encoding's failure: a slot left by a launch
//    65,536 launches earlier at the next position, never overwritten since.
//    The old tags match it; the new ones do not.
static void launch_65536_ago() {
    const uint32_t lg = 20;
    // old scheme: launch e wants position 5 (lap 0); launch e - 65536 wrote
    // position 5 and no launch since reached it
    const uint32_t e = 70000, pos = 5;
    uint64_t planted = old_word(e - 65536, pos, lg, 1234);
    CHECK(old_ready(planted, e, pos, lg), "the old encoding should accept the planted slot (this check models the bug)");
    // new scheme, same history: 65,536 launches, each pushing 3 items of a
    // ring whose positions continue across launches.  The slot of the next
    // position still holds a word from long ago; the consumer must wait.
    Ring r(lg);
    const uint32_t target = 5;                 // the planted slot index
    r.write(target, 1234);                     // launch 0 wrote position 5
    for (uint32_t launch = 1; launch <= 65536; ++launch) {
        r.reset();
        uint32_t p = r.reserve(3);
        for (uint32_t i = 0; i < 3; ++i)
            if (((p + i) & r.mask()) != target) r.write(p + i, (int32_t)launch);   // the planted slot stays
        r.head += 3;
    }
    r.reset();
    // advance to the next position that maps onto the planted slot
    uint32_t next = (r.tail & ~r.mask()) + target;
    if (next < r.tail) next += 1u << lg;
    CHECK(!r.ready(next), "a slot from an old launch was taken for position %u", next);
    r.write(next, 99);
    CHECK(r.ready(next) && r.value(next) == 99, "the written slot must be taken once written");
}

// 4. Randomised protocol replay: several producers reserve batches and write
//    their slots in random order, consumers claim positions and poll; some
//    launches end early with reservations never written; launches reset by
//    moving head to tail.  Cursors start just below the 2^32 wrap.  A consumer
//    may only accept the word its position's producer wrote.
static void replay(uint32_t lg, uint32_t start, uint64_t seed) {
    Ring r(lg);
    r.head = r.tail = start;
    std::mt19937_64 rng(seed);
    const uint32_t cap = 1u << lg;
    int64_t accepted = 0, waits = 0;
    for (int launch = 0; launch < 400; ++launch) {
        r.reset();
        struct Pending { uint32_t pos; int32_t val; };
        std::vector<Pending> unwritten;          // reserved, not yet written
        std::vector<uint32_t> claimed;            // claimed by consumers, not yet read
        std::vector<int32_t> expect((size_t)1 << 16, -1);
        auto key = [](uint32_t p) { return p & 0xFFFFu; };
        const bool aborts = (rng() % 5) == 0;
        int steps = 200 + (int)(rng() % 800);
        for (int s = 0; s < steps; ++s) {
            const int op = (int)(rng() % 3);
            // the device sizes each ring for every task id of the arena, so
            // the positions between the oldest one not yet read and tail
            // never exceed the capacity: no producer laps an unread slot
            uint32_t span = r.tail - r.head;
            for (uint32_t c : claimed) span = std::max(span, r.tail - c);
            if (op == 0 && span + 32 <= cap) {
                const uint32_t n = 1 + (uint32_t)(rng() % 32);
                const uint32_t p = r.reserve(n);
                for (uint32_t i = 0; i < n; ++i) {
                    const int32_t v = (int32_t)(rng() % (1u << 27));
                    unwritten.push_back({p + i, v});
                    expect[key(p + i)] = v;
                }
            } else if (op == 1 && !unwritten.empty()) {
                const size_t j = rng() % unwritten.size();
                r.write(unwritten[j].pos, unwritten[j].val);
                unwritten[j] = unwritten.back();
                unwritten.pop_back();
            } else if (r.tail != r.head) {
                claimed.push_back(r.head++);   // CAS on head succeeded
            }
            // every claimed position polls once
            for (size_t j = 0; j < claimed.size();) {
                const uint32_t p = claimed[j];
                bool written = true;
                for (const Pending& u : unwritten)
                    if (u.pos == p) { written = false; break; }
                if (r.ready(p)) {
                    CHECK(written, "position %u accepted before its producer wrote it (launch %d)", p, launch);
                    CHECK(r.value(p) == expect[key(p)], "position %u read %d, producer wrote %d", p, r.value(p),
                          expect[key(p)]);
                    ++accepted;
                    claimed[j] = claimed.back();
                    claimed.pop_back();
                } else {
                    CHECK(!written, "position %u refused after its producer wrote it", p);
                    ++waits;
                    ++j;
                }
            }
        }
        if (!aborts) {
            // a launch that completes: every reservation is written and read
            for (const Pending& u : unwritten) r.write(u.pos, u.val);
            unwritten.clear();
            while (r.tail != r.head) claimed.push_back(r.head++);
            for (uint32_t p : claimed) {
                CHECK(r.ready(p) && r.value(p) == expect[key(p)], "drain: position %u not as written", p);
                ++accepted;
            }
        }
        // an aborted launch leaves reservations unwritten and claims unread:
        // the next launch's reset drops them
    }
    CHECK(accepted > 0 && waits > 0, "replay exercised nothing (accepted %lld, waits %lld)", (long long)accepted,
          (long long)waits);
    CHECK(uint32_t(r.tail - start) > 0, "cursor did not move");
}

// 5. The recycled-id pool's claims (pool_claim in gtap_device.cuh): while
//    the pool looked long enough, a consumer claims `want` positions with an
//    add on head instead of a compare-and-swap; positions past the producer
//    cursor at that moment are given up.  Consumers read (head, tail) in one
//    step and add in a later one, so other claims interleave and some adds
//    overshoot (the margin here is small to make that happen).  Checked: no
//    consumer accepts a word that is not its position's, every produced
//    value is either accepted once or lies in a given-up position, and no
//    given-up position is ever read.
static void pool_claims(uint32_t lg, uint32_t start, uint64_t seed, uint32_t margin) {
    Ring r(lg);
    r.head = r.tail = start;
    std::mt19937_64 rng(seed);
    const uint32_t cap = 1u << lg;
    struct Pending { uint32_t pos; int32_t val; };
    struct Claimer { uint32_t h, t; bool armed; };
    std::vector<Pending> unwritten;
    std::vector<uint32_t> claimed;           // positions to read
    std::vector<Claimer> claimers(16, Claimer{0, 0, false});
    std::vector<uint8_t> state((size_t)1 << 20, 0);   // by position offset: 1 produced, 2 read, 3 given up
    std::vector<int32_t> expect((size_t)1 << 20, -1);
    auto off = [&](uint32_t p) { return (size_t)(uint32_t)(p - start); };
    int64_t read = 0, given_up = 0, faa = 0;
    for (int step = 0; step < 40000; ++step) {
        const int op = (int)(rng() % 4);
        uint32_t span = r.tail - r.head;
        for (uint32_t c : claimed) span = std::max(span, r.tail - c);
        if (op == 0 && span + 32 <= cap && off(r.tail) + 64 < state.size()) {   // push
            const uint32_t n = 1 + (uint32_t)(rng() % 32);
            const uint32_t p = r.reserve(n);
            for (uint32_t i = 0; i < n; ++i) {
                const int32_t v = (int32_t)(rng() % (1u << 27));
                unwritten.push_back({p + i, v});
                expect[off(p + i)] = v;
            }
        } else if (op == 1 && !unwritten.empty()) {                              // a producer writes
            const size_t j = rng() % unwritten.size();
            r.write(unwritten[j].pos, unwritten[j].val);
            state[off(unwritten[j].pos)] = state[off(unwritten[j].pos)] == 3 ? 3 : 1;
            unwritten[j] = unwritten.back();
            unwritten.pop_back();
        } else if (op == 2) {                                                    // a claimer acts
            Claimer& c = claimers[rng() % claimers.size()];
            const uint32_t want = 1 + (uint32_t)(rng() % 32);
            if (!c.armed) {                       // first step: read head, then tail
                c.h = r.head;
                c.t = r.tail;
                c.armed = true;
            } else {                              // second step: claim
                c.armed = false;
                const uint32_t avail = c.t - c.h;
                if (avail == 0 || avail > cap) continue;
                uint32_t p, got;
                if (avail >= want + margin) {
                    p = r.head;
                    r.head += want;               // the add cannot fail
                    const int produced = (int)(r.tail - p);
                    got = produced <= 0 ? 0u : std::min((uint32_t)produced, want);
                    ++faa;
                    for (uint32_t i = got; i < want; ++i) {
                        state[off(p + i)] = 3;
                        ++given_up;
                    }
                } else {
                    if (r.head != c.h) continue;  // the compare-and-swap fails
                    got = std::min(avail, want);
                    p = c.h;
                    r.head += got;
                }
                for (uint32_t i = 0; i < got; ++i) claimed.push_back(p + i);
            }
        }
        for (size_t j = 0; j < claimed.size();) {                                 // claimed positions poll
            const uint32_t p = claimed[j];
            CHECK(state[off(p)] != 3, "a given-up position %u was claimed for reading", p);
            if (r.ready(p)) {
                CHECK(r.value(p) == expect[off(p)], "position %u read %d, producer wrote %d", p, r.value(p),
                      expect[off(p)]);
                CHECK(state[off(p)] == 1, "position %u read before it was written or twice", p);
                state[off(p)] = 2;
                ++read;
                claimed[j] = claimed.back();
                claimed.pop_back();
            } else {
                ++j;
            }
        }
        if (off(r.tail) + 64 >= state.size()) break;
    }
    CHECK(read > 1000 && faa > 100, "pool replay exercised too little (read %lld, adds %lld)", (long long)read,
          (long long)faa);
    CHECK(given_up > 0, "the small margin should make some adds overshoot");
}

int main() {
    fresh_ring();
    stale_laps();
    launch_65536_ago();
    replay(8, 0xFFFFFFFFu - 3000u, 1);    // tiny ring: many laps, wraps 2^32
    replay(10, 0xFFFFFF00u, 2);
    replay(20, 0xFFFFF000u, 3);
    replay(12, 0, 4);
    pool_claims(12, 0xFFFFF000u, 5, 8);
    pool_claims(16, 7, 6, 40);
    if (g_failures) {
        std::printf("%d failures\n", g_failures);
        return 1;
    }
    std::printf("ring model: all checks passed\n");
    return 0;
}
