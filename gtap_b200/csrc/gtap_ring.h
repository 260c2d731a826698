// gtap_ring.h -- slot encoding of the lap-tagged MPMC rings (the global
// overflow queue and the recycled task-id pool).  Plain C++ with no CUDA
// dependency, so the host-side model of the ring protocol in the CPU tests
// compiles the very functions the device uses.
//
// A ring has 2^cap_log2 64-bit slots and two 32-bit cursors, head (consumer)
// and tail (producer).  A producer reserves position p with an atomic add on
// tail and writes slot p mod 2^cap_log2 as
//
//     word = (tag(p) << 32) | (value + 1),   tag(p) = (p >> cap_log2) + 1
//
// i.e. the lap number of p plus one.  A consumer that claimed position p
// (a CAS on head) spins until the slot's tag equals tag(p), so it never takes
// an unwritten slot or one left over from an earlier lap.
//
// Properties the device relies on:
//   * never-written slots hold 0 and tag(p) >= 1, so a fresh ring never
//     matches;
//   * the cursors are never reset while the ring exists.  Between launches the
//     reset kernel drops whatever is queued by moving head to tail, so the
//     positions of one launch continue the previous launch's: every position
//     is used once per 2^32, and tag(p) repeats only for positions 2^32 apart.
//     A slot is rewritten on every lap (each reserved position is written by
//     its producer), so a stale slot is at most a lap or two old -- never
//     2^(32 - cap_log2) laps, the distance at which the tag would repeat;
//   * the 32-bit cursors may wrap: p mod 2^cap_log2 and the unsigned
//     difference tail - head stay exact across the wrap, and the lap number
//     restarts at 0 with tag 1, which differs from the last lap's tag.
//     Whatever moves the cursors other than by use (a test that jumps them
//     close to the wrap) must clear the slots, or a word written before the
//     jump may carry the tag of a position 2^32 further on.
//
// An earlier encoding kept a per-launch epoch in the tag and reset the
// cursors to 0 at every launch; a 16-bit epoch repeats after 65,536
// launches, at which point a slot from an old launch at the same position
// could be taken for the current one.  Continuing positions need no epoch.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GTAP_RING_HD __host__ __device__ __forceinline__
#else
#define GTAP_RING_HD inline
#endif

namespace gtap {

GTAP_RING_HD uint32_t ring_tag_of(uint32_t pos, uint32_t cap_log2) { return (pos >> cap_log2) + 1u; }

GTAP_RING_HD uint64_t ring_word_of(uint32_t pos, uint32_t cap_log2, int32_t value) {
    return ((uint64_t)ring_tag_of(pos, cap_log2) << 32) | (uint32_t)(value + 1);
}

// The slot written for position pos holds this word; anything else means
// "not written yet" to the consumer of pos.
GTAP_RING_HD bool ring_word_ready(uint64_t word, uint32_t pos, uint32_t cap_log2) {
    return (uint32_t)(word >> 32) == ring_tag_of(pos, cap_log2);
}

GTAP_RING_HD int32_t ring_word_value(uint64_t word) { return (int32_t)(uint32_t)(word & 0xFFFFFFFFu) - 1; }

}  // namespace gtap
