// Acceptance test and attraction weight of one octree node in the FP64
// search: BarnesHutBase::test_acceptance_criterion (BarnesHutBase.h:72-114)
// and Kernel::calculate_attractiveness_to_connect (Kernel/Kernel.h:61-75).
// Shared by the production search (bh_search.cu) and the candidate diagnostic
// (fp32.cu, rl_candidate_weights), so the diagnostic reports the weights the
// search itself computes.
#pragma once

#include "rl_context.cuh"
#include "rl_math.cuh"

namespace rl {

enum : int { ST_DISCARD = 0, ST_EXPAND = 1, ST_ACCEPT = 2 };

__device__ __forceinline__ uint32_t rcount(const double4& r) {
    return (uint32_t)__double_as_longlong(r.w);
}

struct Eval {
    int status;
    double w;
};

// Status and weight of one node for a source at (sx, sy, sz): discard an
// empty cell or one at distance 0, accept a leaf or a cell with
// maxdim < theta * d, expand otherwise.
__device__ __forceinline__ Eval evaluate(const double4& r, uint2 t, double md, double sx, double sy, double sz, uint32_t source, double theta, double mu,
                                         double scale, bool fallback, const KernelParams& K) {
    Eval e{ ST_DISCARD, 0.0 };
    const uint32_t cnt = rcount(r);
    if (cnt == 0) {
        return e;
    }
    const double d = rl_hypot3(r.x - sx, r.y - sy, r.z - sz);
    if (d == 0.0) {
        return e;
    }
    const bool leaf = topo_leaf(t.y);
    if (!leaf && !(md < theta * d)) {
        e.status = ST_EXPAND;
        return e;
    }
    e.status = ST_ACCEPT;
    if (leaf && t.x == source) {
        e.w = 0.0;  // a neuron never connects to itself
    } else if (!fallback) {
        e.w = (rl_kernel_prob(K.type, d, mu, scale, K.k_minus_1, K.a, K.b, K.cutoff, K.cutoff_inf) * 1.0) * (double)cnt;
    } else {
        e.w = (double)cnt / d;
    }
    return e;
}

}  // namespace rl
