// gtap_selftest.cuh -- exactly-once stress test of the scheduler's queue
// primitives on the device: the per-worker deque (publish_src / pop_own /
// steal) and the global overflow ring (ring_push_warp / ring_pop_warp).
//
// Every warp produces unique tokens (worker * 16384 + sequence, below the
// 2^27 task-id range) through the
// same publish path the scheduler uses, and consumes tokens by popping its own
// deque, stealing from others and draining the overflow ring.  Each consumed
// token increments seen[token]; the host checks that every produced token was
// consumed exactly once.  Tokens are only counted, never dereferenced, so a
// duplicate or a loss shows up as a count, not as a fault.
#pragma once
#include "gtap_thread_sched.cuh"

namespace gtap {

struct SelftestCounters {
    unsigned produced;
    unsigned consumed;
    unsigned producers_done;
    unsigned bad_tokens;
};

// mode bits select the consumers active while tokens are produced:
// 1 = own-deque pops, 2 = steals, 4 = overflow-queue reads (all run in the drain)
static __global__ void selftest_queue_kernel(const __grid_constant__ Arena A, int rounds, int per_round_max, unsigned* seen,
                                      SelftestCounters* c, int mode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int wib = threadIdx.x >> 5;
    const unsigned lane = lane_id();
    WarpShared* ws = reinterpret_cast<WarpShared*>(smem_raw);
    int* sb_base = reinterpret_cast<int*>(smem_raw + sizeof(WarpShared) * A.warps_per_block);
    WarpShared& S = ws[wib];
    const int worker = blockIdx.x * A.warps_per_block + wib;
    if (lane == 0) {
        S.worker = worker;
        S.sbuf = sb_base + (size_t)wib * A.num_queues * A.spawn_cap;
        for (int k = 0; k < kMaxQueues; ++k) {
            S.cnt[k] = 0;
        }
        for (int i = 0; i < GTAP_STAT_COUNT; ++i) S.st[i] = 0;
    }
    __syncwarp();
    QueuePos<kMaxQueues> P;
    queue_pos_init(P);
    unsigned rng = 0x2545F491u ^ (unsigned)(worker * 2654435761u) ^ (lane * 0x9E3779B9u);
    if (rng == 0) rng = 1;
    int last_victim = -1;
    unsigned seq = 0;
    unsigned my_consumed = 0;
    const unsigned ntok = (unsigned)A.num_workers * 16384u;
    auto consume = [&](int got, int tok) {
        if ((int)lane < got) {
            if ((unsigned)tok < ntok) atomicAdd(&seen[tok], 1u);
            else atomicAdd(&c->bad_tokens, 1u);
        }
        my_consumed += __popc(__ballot_sync(0xffffffffu, (int)lane < got));
    };
    for (int r = 0; r < rounds; ++r) {
        unsigned draw = __shfl_sync(0xffffffffu, xorshift32(rng), 0);
        int m = (int)(draw % (unsigned)(per_round_max + 1));
        m = min(m, A.spawn_cap);
        if (seq + (unsigned)m > 16383u) m = 0;
        for (int e = (int)lane; e < m; e += 32) S.sbuf[e] = (int)((unsigned)worker * 16384u + seq + (unsigned)e);
        __syncwarp();
        seq += (unsigned)m;
        if (m > 0) publish_src(A, S, P, 0, S.sbuf, 0, 0xFFFFFFFFu, m);
        int tok = -1;
        int got = 0;
        if (mode & 1) {
            got = pop_own(A, S, P, 0, tok);
            consume(got, tok);
        }
        if ((mode & 2) && ((draw >> 8) & 1u)) {
            got = steal(A, S, 0, rng, last_victim, tok);
            consume(got, tok);
        }
        if ((mode & 4) && ((draw >> 9) & 1u)) {
            got = ring_pop_warp(A, A.overflow, 32, &tok);
            consume(got, tok);
        }
    }
    if (lane == 0) {
        atomicAdd(&c->produced, seq);
        __threadfence();
        atomicAdd(&c->producers_done, 1u);
    }
    // drain: pop, steal and read the ring until every token is accounted for
    for (int spin = 0; spin < (1 << 20); ++spin) {
        int tok = -1;
        int g1 = pop_own(A, S, P, 0, tok);
        consume(g1, tok);
        int g2 = steal(A, S, 0, rng, last_victim, tok);
        consume(g2, tok);
        int g3 = ring_pop_warp(A, A.overflow, 32, &tok);
        consume(g3, tok);
        if (g1 == 0 && g2 == 0 && g3 == 0) {
            int stop = 0;
            if (lane == 0) {
                if (my_consumed) atomicAdd(&c->consumed, my_consumed);
                __threadfence();
                if (ld_relaxed(&c->producers_done) == (unsigned)A.num_workers &&
                    ld_relaxed(&c->consumed) >= ld_relaxed(&c->produced))
                    stop = 1;
            }
            my_consumed = 0;
            if (__shfl_sync(0xffffffffu, stop, 0)) return;
            __nanosleep(256);
        }
    }
    if (lane == 0 && my_consumed) atomicAdd(&c->consumed, my_consumed);
}

}  // namespace gtap
