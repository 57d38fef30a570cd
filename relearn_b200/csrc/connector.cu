// Connector and synapse graph.
//
// Reference semantics: ForwardConnector::process_requests / process_responses
// (relearn/source/algorithm/Connector.cpp:33-197).  Requests are processed
// in a random order; a request is accepted while its target still has a
// vacant dendrite of the needed type (the searching neuron's signal type);
// an accepted request connects one dendrite of the target and one axon of the
// source and adds a synapse of weight +1 (excitatory) or -1 (inhibitory).
// A request whose target is its source fails without consuming anything.
//
// The random order is a sort on a 64-bit Philox key per (step, source, j)
// with ties broken by (source, j).  Within each (target, type) group the
// processing order is therefore the key order, so the first `vacant` requests
// of a group are the accepted ones.  Two stable radix sorts give that order:
// first on the key, then on the group.
#include "rl_context.cuh"
#include "rl_math.cuh"

namespace rl {
namespace {

__global__ void k_conn_keys(uint64_t m, uint32_t n, const uint32_t* __restrict__ tgt, const uint32_t* __restrict__ src, const uint32_t* __restrict__ jj,
                            const uint32_t* __restrict__ sig, uint64_t seed, uint32_t step, uint64_t* __restrict__ key, uint32_t* __restrict__ idx,
                            uint32_t* __restrict__ gkey) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) {
        return;
    }
    const u32x4 w = draw(seed, step, src[i], jj[i], STREAM_CONNECTOR, 0u);
    key[i] = bits64(w);
    idx[i] = (uint32_t)i;
    // autapses go to a group past all real ones and are rejected there
    gkey[i] = tgt[i] == src[i] ? 2u * n : 2u * tgt[i] + sig[i];
}

__global__ void k_gather_u32(uint64_t m, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        out[i] = in[perm[i]];
    }
}

__global__ void k_group_heads(uint64_t m, const uint32_t* __restrict__ g, uint32_t* __restrict__ start) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < m && (p == 0 || g[p] != g[p - 1])) {
        start[g[p]] = (uint32_t)p;
    }
}

struct AcceptArgs {
    uint64_t m;
    uint32_t n;
    const uint32_t* g;      // group of sorted position
    const uint32_t* perm;   // request index of sorted position
    const uint32_t* start;  // first sorted position of each group
    const uint32_t* tgt;
    const uint32_t* src;
    const uint32_t* sig;
    uint32_t* vac_exc;
    uint32_t* vac_inh;
    uint32_t* con_exc;
    uint32_t* con_inh;
    uint32_t* vac_axon;
    uint32_t* con_axon;
    const uint32_t* vac_exc_before;  // vacant dendrites when the connector starts
    const uint32_t* vac_inh_before;
    uint32_t* accepted;  // per sorted position
    uint32_t* err;
};

__global__ void k_accept(AcceptArgs A) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.m) {
        return;
    }
    const uint32_t g = A.g[p];
    uint32_t acc = 0;
    if (g < 2u * A.n) {
        const uint32_t rank = (uint32_t)p - A.start[g];
        const uint32_t i = A.perm[p];
        const uint32_t t = A.tgt[i];
        const bool inh = A.sig[i] != 0;
        const uint32_t vac = inh ? A.vac_inh_before[t] : A.vac_exc_before[t];
        if (rank < vac) {
            acc = 1;
            atomicAdd(inh ? &A.con_inh[t] : &A.con_exc[t], 1u);
            atomicSub(inh ? &A.vac_inh[t] : &A.vac_exc[t], 1u);
            const uint32_t s = A.src[i];
            const uint32_t old = atomicSub(&A.vac_axon[s], 1u);
            if (old == 0) {
                atomicOr(A.err, (uint32_t)DERR_CONNECT);
            }
            atomicAdd(&A.con_axon[s], 1u);
        }
    }
    A.accepted[p] = acc;
}

__global__ void k_emit_edges(uint64_t m, const uint32_t* __restrict__ accepted, const uint32_t* __restrict__ pos, const uint32_t* __restrict__ perm,
                             const uint32_t* __restrict__ tgt, const uint32_t* __restrict__ src, const uint32_t* __restrict__ sig, uint64_t base,
                             uint32_t* __restrict__ et, uint32_t* __restrict__ es, int32_t* __restrict__ ew) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m || !accepted[p]) {
        return;
    }
    const uint32_t i = perm[p];
    const uint64_t o = base + pos[p];
    et[o] = tgt[i];
    es[o] = src[i];
    ew[o] = sig[i] ? -1 : 1;
}

// ---- graph rebuild
__global__ void k_csr_expand(uint32_t n, const uint32_t* __restrict__ off, uint32_t* __restrict__ tgt) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) {
        return;
    }
    for (uint32_t e = off[t]; e < off[t + 1]; ++e) {
        tgt[e] = t;
    }
}

__global__ void k_iota(uint64_t m, uint32_t* __restrict__ p) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        p[i] = (uint32_t)i;
    }
}

__global__ void k_count_targets(uint64_t m, const uint32_t* __restrict__ tgt, uint32_t* __restrict__ cnt) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        atomicAdd(&cnt[tgt[i]], 1u);
    }
}

__global__ void k_gather_edges(uint64_t m, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ s_in, const int32_t* __restrict__ w_in,
                               uint32_t* __restrict__ s_out, int32_t* __restrict__ w_out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        s_out[i] = s_in[perm[i]];
        w_out[i] = w_in[perm[i]];
    }
}

}  // namespace

uint64_t run_connector(Ctx& c, uint32_t step) {
    const uint64_t m = c.search.num_requests;
    Search& S = c.search;
    Graph& G = c.graph;
    cudaStream_t st = c.stream;
    const uint32_t n = c.n;
    if (m == 0) {
        return 0;
    }
    S.ckey.ensure(m);
    S.cidx.ensure(m);
    S.gkey.ensure(m);
    S.accepted.ensure(m);
    S.rank.ensure(m);
    S.flags.ensure(2 * (size_t)n + 2);
    k_conn_keys<<<blocks_for(m, 256), 256, 0, st>>>(m, n, S.req_tgt.p, S.req_src.p, S.req_j.p, S.req_sig.p, c.cfg.seed, step, S.ckey.p, S.cidx.p,
                                                    S.gkey.p);
    RL_LAUNCH_CHECK();
    radix_sort_u64(S.ckey.p, S.cidx.p, m, 64, c.prim, st);
    // group key in key order, then a stable sort on it
    k_gather_u32<<<blocks_for(m, 256), 256, 0, st>>>(m, S.cidx.p, S.gkey.p, S.rank.p);
    RL_LAUNCH_CHECK();
    int gbits = 1;
    while (gbits < 32 && ((uint64_t)1 << gbits) <= 2ull * n) {
        ++gbits;
    }
    radix_sort_u32(S.rank.p, S.cidx.p, m, gbits, c.prim, st);
    // S.rank now holds the sorted group keys, S.cidx the request index
    k_group_heads<<<blocks_for(m, 256), 256, 0, st>>>(m, S.rank.p, S.flags.p);
    RL_LAUNCH_CHECK();
    // vacant dendrite counts before the connector
    DBuf<uint32_t> before;
    before.alloc(2 * (size_t)n);
    RL_CUDA_TRY(cudaMemcpyAsync(before.p, c.nr.vacant[1].p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    RL_CUDA_TRY(cudaMemcpyAsync(before.p + n, c.nr.vacant[2].p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    AcceptArgs A;
    A.m = m;
    A.n = n;
    A.g = S.rank.p;
    A.perm = S.cidx.p;
    A.start = S.flags.p;
    A.tgt = S.req_tgt.p;
    A.src = S.req_src.p;
    A.sig = S.req_sig.p;
    A.vac_exc = c.nr.vacant[1].p;
    A.vac_inh = c.nr.vacant[2].p;
    A.con_exc = c.nr.connected[1].p;
    A.con_inh = c.nr.connected[2].p;
    A.vac_axon = c.nr.vacant[0].p;
    A.con_axon = c.nr.connected[0].p;
    A.vac_exc_before = before.p;
    A.vac_inh_before = before.p + n;
    A.accepted = S.accepted.p;
    A.err = c.err.p;
    k_accept<<<blocks_for(m, 256), 256, 0, st>>>(A);
    RL_LAUNCH_CHECK();
    // compact accepted into the new-edge buffer (sorted-position order)
    DBuf<uint32_t> pos;
    pos.alloc(m);
    const uint64_t created = exclusive_scan_u32(S.accepted.p, pos.p, m, c.prim, st);
    const uint64_t need = G.num_new + created;
    if (need > G.new_tgt.n) {
        // grow, keeping what is already there
        DBuf<uint32_t> t2, s2;
        DBuf<int32_t> w2;
        t2.alloc(need * 2);
        s2.alloc(need * 2);
        w2.alloc(need * 2);
        if (G.num_new) {
            RL_CUDA_TRY(cudaMemcpyAsync(t2.p, G.new_tgt.p, G.num_new * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
            RL_CUDA_TRY(cudaMemcpyAsync(s2.p, G.new_src.p, G.num_new * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
            RL_CUDA_TRY(cudaMemcpyAsync(w2.p, G.new_w.p, G.num_new * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
        }
        RL_CUDA_TRY(cudaStreamSynchronize(st));
        std::swap(G.new_tgt.p, t2.p);
        std::swap(G.new_tgt.n, t2.n);
        std::swap(G.new_src.p, s2.p);
        std::swap(G.new_src.n, s2.n);
        std::swap(G.new_w.p, w2.p);
        std::swap(G.new_w.n, w2.n);
    }
    k_emit_edges<<<blocks_for(m, 256), 256, 0, st>>>(m, S.accepted.p, pos.p, S.cidx.p, S.req_tgt.p, S.req_src.p, S.req_sig.p, G.num_new, G.new_tgt.p,
                                                     G.new_src.p, G.new_w.p);
    RL_LAUNCH_CHECK();
    G.num_new += created;
    check_device_error(c, "connector");
    c.stats.synapses_created += created;
    return created;
}

void rebuild_graph(Ctx& c) {
    Graph& G = c.graph;
    if (G.num_new == 0) {
        return;
    }
    cudaStream_t st = c.stream;
    const uint32_t n = c.n;
    const uint64_t old = G.num_edges;
    const uint64_t m = old + G.num_new;
    RL_CHECK(m < 0xFFFFFFFFull, RL_ERR_OVERFLOW, "synapse count exceeds 2^32");
    DBuf<uint32_t> tgt, perm, srcs, cnt;
    DBuf<int32_t> ws;
    tgt.alloc(m);
    perm.alloc(m);
    srcs.alloc(m);
    ws.alloc(m);
    cnt.alloc((size_t)n + 1);
    if (old) {
        k_csr_expand<<<blocks_for(n, 256), 256, 0, st>>>(n, G.offsets.p, tgt.p);
        RL_LAUNCH_CHECK();
        RL_CUDA_TRY(cudaMemcpyAsync(srcs.p, G.src.p, old * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        RL_CUDA_TRY(cudaMemcpyAsync(ws.p, G.weight.p, old * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    }
    RL_CUDA_TRY(cudaMemcpyAsync(tgt.p + old, G.new_tgt.p, G.num_new * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    RL_CUDA_TRY(cudaMemcpyAsync(srcs.p + old, G.new_src.p, G.num_new * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    RL_CUDA_TRY(cudaMemcpyAsync(ws.p + old, G.new_w.p, G.num_new * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    RL_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, ((size_t)n + 1) * sizeof(uint32_t), st));
    k_count_targets<<<blocks_for(m, 256), 256, 0, st>>>(m, tgt.p, cnt.p);
    RL_LAUNCH_CHECK();
    G.offsets.ensure((size_t)n + 1);
    exclusive_scan_u32(cnt.p, G.offsets.p, (uint64_t)n + 1, c.prim, st);
    k_iota<<<blocks_for(m, 256), 256, 0, st>>>(m, perm.p);
    RL_LAUNCH_CHECK();
    int bits = 1;
    while (bits < 32 && ((uint64_t)1 << bits) <= n) {
        ++bits;
    }
    radix_sort_u32(tgt.p, perm.p, m, bits, c.prim, st);
    G.src.ensure(m);
    G.weight.ensure(m);
    k_gather_edges<<<blocks_for(m, 256), 256, 0, st>>>(m, perm.p, srcs.p, ws.p, G.src.p, G.weight.p);
    RL_LAUNCH_CHECK();
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    G.num_edges = m;
    G.num_new = 0;
}

void add_edges_host(Ctx& c, uint64_t m, const uint32_t* t, const uint32_t* s, const int32_t* w) {
    if (m == 0) {
        return;
    }
    Graph& G = c.graph;
    cudaStream_t st = c.stream;
    for (uint64_t k = 0; k < m; ++k) {
        RL_CHECK(t[k] < c.n && s[k] < c.n, RL_ERR_INVALID, "edge endpoint out of range");
    }
    const uint64_t need = G.num_new + m;
    DBuf<uint32_t> t2, s2;
    DBuf<int32_t> w2;
    t2.alloc(need);
    s2.alloc(need);
    w2.alloc(need);
    if (G.num_new) {
        RL_CUDA_TRY(cudaMemcpyAsync(t2.p, G.new_tgt.p, G.num_new * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        RL_CUDA_TRY(cudaMemcpyAsync(s2.p, G.new_src.p, G.num_new * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        RL_CUDA_TRY(cudaMemcpyAsync(w2.p, G.new_w.p, G.num_new * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    }
    RL_CUDA_TRY(cudaMemcpyAsync(t2.p + G.num_new, t, m * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    RL_CUDA_TRY(cudaMemcpyAsync(s2.p + G.num_new, s, m * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    RL_CUDA_TRY(cudaMemcpyAsync(w2.p + G.num_new, w, m * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    std::swap(G.new_tgt.p, t2.p);
    std::swap(G.new_tgt.n, t2.n);
    std::swap(G.new_src.p, s2.p);
    std::swap(G.new_src.n, s2.n);
    std::swap(G.new_w.p, w2.p);
    std::swap(G.new_w.n, w2.n);
    G.num_new = need;
    rebuild_graph(c);
}

}  // namespace rl
