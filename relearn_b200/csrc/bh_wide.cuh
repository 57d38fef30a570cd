// One Barnes-Hut search per warp: the parts shared by the FP64 search
// (bh_search.cu) and the FP32 form (fp32.cu).
//
// For search lists whose sources lie far apart (a network whose elements grow
// slowly searches for a few thousand of its million neurons per update), a
// packet of 32 sources walks the union of 32 unrelated walks, and one lane per
// search leaves the device nearly idle.  Here a whole warp runs ONE search:
//   * Candidates are collected in rounds, one tree level at a time: the lanes
//     evaluate a round's nodes side by side (acceptance test and weight do not
//     depend on the walk), and the children of expanded nodes, appended in
//     visiting order (descending octant) behind each other by a warp scan,
//     form the next round.  Every round lies in the reference's visiting order
//     (BarnesHutBase::get_nodes_to_consider, BarnesHutBase.h:129-206: a LIFO
//     stack with the children pushed 0..7).
//   * The position of every accepted candidate in that depth-first visiting
//     order follows from the rounds: bottom-up, each expanded node counts the
//     candidates below it; top-down, a node's position is its parent's plus
//     the counts of its earlier siblings.  The weights are scattered into that
//     order.
//   * The running sum is one sequential chain in that order (all lanes add,
//     each keeps the sum at its own element), so every partial sum has the
//     bits of the per-lane sequential sum of the packet kernels
//     (ProbabilityPicker::pick_target, ProbabilityPicker.h:46-112); the pick
//     is the first partial sum that reaches r.
// Deeper descents run the same way from the picked node.  A warp's scratch
// holds `cap` walk entries; a search that does not fit is left to the packet
// kernel (target kRedo).
#pragma once

#include "rl_context.cuh"

namespace rl {

constexpr int32_t kRedo = -2;
constexpr int kWideRounds = kMaxLevels + 2;

// The scratch of one warp: `cap` entries per array.
struct WideSlot {
    uint32_t* node;      // node of a walk entry
    uint32_t* info;      // status | children << 2
    uint32_t* child;     // first entry of an expanded node's children
    uint32_t* cnt;       // candidates in the entry's subtree
    uint32_t* pos;       // position of the entry's first candidate in visiting order
    uint32_t* ord_node;  // candidates in visiting order
    double* w;           // weight of an accepted entry
    double* ord_w;       // weights in visiting order, then the running sums
};

// Status of a node for the walk: 0 discard, 1 expand, 2 accept (the packet
// kernels' ST_* / S_* values).
struct WideEval {
    int status;
    double w;
    uint32_t nch;    // children of an expanded node
    uint32_t first;  // its first child
    bool bad;        // node index out of range
};

// Warp inclusive prefix sum of v.
__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) {
            v += t;
        }
    }
    return v;
}

// L1 prefetch of a global address (no data is returned, nothing waits for it).
__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// The candidates of the subtree whose root has k0 children from `first0` on,
// in visiting order (P.ord_node, weights in P.ord_w): returns their number
// F, or -1 when a walk entry did not fit, -2 when the walk left the node range
// or went deeper than any octree.  eval(node) evaluates one node; pre(node)
// prefetches what eval will read of it.  Each pass over a round's entries, 32
// at a time, loads the entries of its next 32 while it works on the current
// ones (a round's entries are all written before the round starts), so that a
// step of the walk waits on one memory round trip instead of two.
template <class Eval, class Pre>
__device__ int64_t wide_collect(const WideSlot& P, uint32_t cap, uint32_t first0, uint32_t k0, uint32_t* s_round, uint32_t& touched, Eval&& eval,
                                Pre&& pre) {
    const int lane = threadIdx.x & 31;
    if ((uint32_t)lane < k0) {
        P.node[lane] = first0 + k0 - 1u - (uint32_t)lane;  // children in visiting order: last octant first
    }
    s_round[0] = 0;
    s_round[1] = k0;
    int rounds = 0;
    bool bad = false;
    __syncwarp();
    // forward: evaluate round after round
    for (;;) {
        const uint32_t rb = s_round[rounds], re = s_round[rounds + 1];
        if (rb == re) {
            break;
        }
        if (rounds + 2 >= kWideRounds) {
            return -2;
        }
        uint32_t next = re;
        uint32_t nd_cur = rb + (uint32_t)lane < re ? P.node[rb + (uint32_t)lane] : 0u;
        for (uint32_t base = rb; base < re; base += 32) {
            const uint32_t e = base + (uint32_t)lane;
            // the next 32 entries lie below re: this round writes only behind re
            const uint32_t nd_next = e + 32u < re ? P.node[e + 32u] : 0u;
            WideEval ev{ 0, 0.0, 0u, 0u, false };
            if (e < re) {
                ev = eval(nd_cur);
                bad = bad || ev.bad;
                ++touched;
            }
            if (e + 32u < re) {
                pre(nd_next);
            }
            nd_cur = nd_next;
            const uint32_t nch = ev.status == 1 ? ev.nch : 0u;
            const uint32_t inc = warp_inclusive(nch);
            const uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
            if (next + total > cap) {
                return -1;
            }
            const uint32_t cs = next + inc - nch;
            if (e < re) {
                P.info[e] = (uint32_t)ev.status | (nch << 2);
                P.child[e] = cs;
                P.w[e] = ev.w;
            }
            for (uint32_t c = 0; c < nch; ++c) {
                P.node[cs + c] = ev.first + nch - 1u - c;
            }
            next += total;
        }
        if (__any_sync(0xFFFFFFFFu, bad)) {
            return -2;
        }
        ++rounds;
        if (lane == 0) {
            s_round[rounds + 1] = next;
        }
        __syncwarp();
    }
    // bottom-up: candidates below every entry
    for (int r = rounds - 1; r >= 0; --r) {
        const uint32_t rb = s_round[r], re = s_round[r + 1];
        uint32_t inf_n = 0u, c0_n = 0u;
        if (rb + (uint32_t)lane < re) {
            inf_n = P.info[rb + (uint32_t)lane];
            c0_n = P.child[rb + (uint32_t)lane];
        }
        for (uint32_t e = rb + (uint32_t)lane; e < re; e += 32) {
            const uint32_t inf = inf_n;
            const uint32_t c0 = c0_n;
            if (e + 32u < re) {
                inf_n = P.info[e + 32u];
                c0_n = P.child[e + 32u];
            }
            const int st = (int)(inf & 3u);
            uint32_t n = st == 2 ? 1u : 0u;
            if (st == 1) {
                for (uint32_t c = 0; c < (inf >> 2); ++c) {
                    n += P.cnt[c0 + c];
                }
            }
            P.cnt[e] = n;
        }
        __syncwarp();
    }
    // top-down: positions in visiting order; the candidates go to their place
    uint32_t carry = 0;
    for (uint32_t base = 0; base < k0; base += 32) {
        const uint32_t e = base + (uint32_t)lane;
        const uint32_t n = e < k0 ? P.cnt[e] : 0u;
        const uint32_t inc = warp_inclusive(n);
        if (e < k0) {
            P.pos[e] = carry + inc - n;
        }
        carry += __shfl_sync(0xFFFFFFFFu, inc, 31);
    }
    __syncwarp();
    for (int r = 0; r < rounds; ++r) {
        const uint32_t rb = s_round[r], re = s_round[r + 1];
        uint32_t inf_n = rb + (uint32_t)lane < re ? P.info[rb + (uint32_t)lane] : 0u;
        for (uint32_t e = rb + (uint32_t)lane; e < re; e += 32) {
            const uint32_t inf = inf_n;
            if (e + 32u < re) {
                inf_n = P.info[e + 32u];
            }
            const int st = (int)(inf & 3u);
            const uint32_t p = P.pos[e];
            if (st == 2) {
                P.ord_node[p] = P.node[e];
                P.ord_w[p] = P.w[e];
            } else if (st == 1) {
                const uint32_t c0 = P.child[e];
                uint32_t acc = p;
                for (uint32_t c = 0; c < (inf >> 2); ++c) {
                    P.pos[c0 + c] = acc;
                    acc += P.cnt[c0 + c];
                }
            }
        }
        __syncwarp();
    }
    return (int64_t)carry;
}

// The running sum of ord_w[0, F) in order, one FP64 addition after the other
// (the per-lane sum of the packet kernels); ord_w[i] becomes the sum up to
// and including i.  Returns the total.
__device__ __forceinline__ double wide_running_sum64(double* ord_w, uint32_t F) {
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (uint32_t base = 0; base < F; base += 32) {
        const uint32_t i = base + (uint32_t)lane;
        const double v = i < F ? ord_w[i] : 0.0;
        double mine = 0.0;
        if (F - base >= 32) {
#pragma unroll
            for (int q = 0; q < 32; ++q) {
                s = s + __shfl_sync(0xFFFFFFFFu, v, q);
                mine = q == lane ? s : mine;
            }
        } else {
            const uint32_t lim = F - base;
            for (uint32_t q = 0; q < lim; ++q) {
                s = s + __shfl_sync(0xFFFFFFFFu, v, (int)q);
                mine = q == (uint32_t)lane ? s : mine;
            }
        }
        if (i < F) {
            ord_w[i] = mine;
        }
    }
    __syncwarp();
    return s;
}

// The same in FP32 with Kahan compensation, as the FP32 form's packet kernels
// add (s, c): ord_w holds FP32 weights and becomes the running s.
__device__ __forceinline__ float wide_running_sum32(double* ord_w, uint32_t F) {
    const int lane = threadIdx.x & 31;
    float s = 0.0f, c = 0.0f;
    for (uint32_t base = 0; base < F; base += 32) {
        const uint32_t i = base + (uint32_t)lane;
        const float v = i < F ? (float)ord_w[i] : 0.0f;
        float mine = 0.0f;
        const uint32_t lim = F - base >= 32 ? 32u : F - base;
        for (uint32_t q = 0; q < lim; ++q) {
            const float x = __shfl_sync(0xFFFFFFFFu, v, (int)q);
            const float y = x - c;
            const float t = s + y;
            c = (t - s) - y;
            s = t;
            mine = q == (uint32_t)lane ? s : mine;
        }
        if (i < F) {
            ord_w[i] = (double)mine;
        }
    }
    __syncwarp();
    return s;
}

// The first candidate whose running sum reaches r, -1 if none does.
__device__ __forceinline__ int64_t wide_pick(const double* ord_w, const uint32_t* ord_node, uint32_t F, double r) {
    for (uint32_t base = 0; base < F; base += 32) {
        const uint32_t i = base + (threadIdx.x & 31);
        const uint32_t hit = __ballot_sync(0xFFFFFFFFu, i < F && ord_w[i] >= r);
        if (hit) {
            return ord_node[base + (uint32_t)(__ffs((int)hit) - 1)];
        }
    }
    return -1;
}

// The list entry of wide task `task` (32 tasks per warp task of the packet
// kernels' segment layout): its segment, or false for a padding slot.
__device__ __forceinline__ bool wide_task_entry(uint32_t task, const uint32_t* seg_warp, const uint64_t* seg_begin, const uint64_t* seg_end,
                                                uint32_t num_segs, uint32_t& seg, uint64_t& idx) {
    const uint32_t wg = task >> 5;
    uint32_t lo = 0, hi = num_segs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (seg_warp[mid] <= wg) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    seg = lo;
    idx = seg_begin[lo] + (uint64_t)(wg - seg_warp[lo]) * 32 + (task & 31u);
    return idx < seg_end[lo];
}

}  // namespace rl
