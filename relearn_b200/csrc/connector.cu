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
                            const uint32_t* __restrict__ sig, const NetInfo* __restrict__ nets, const uint16_t* __restrict__ net_of, uint32_t step,
                            uint64_t* __restrict__ key, uint32_t* __restrict__ idx, uint32_t* __restrict__ gkey) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) {
        return;
    }
    const NetInfo& N = nets[net_of[src[i]]];
    const u32x4 w = draw(N.seed, step, src[i] - N.first, jj[i], STREAM_CONNECTOR, 0u);
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
            if (A.vac_axon) {  // null: the sources live on other ranks (process_requests only)
                const uint32_t s = A.src[i];
                const uint32_t old = atomicSub(&A.vac_axon[s], 1u);
                if (old == 0) {
                    atomicOr(A.err, (uint32_t)DERR_CONNECT);
                }
                atomicAdd(&A.con_axon[s], 1u);
            }
        }
    }
    A.accepted[p] = acc;
}

// ForwardConnector::process_responses (Connector.cpp:119-197): one vacant
// axon of the source bound per accepted request; a source without one is an
// error (the reference throws).
__global__ void k_bind_axons(uint64_t m, const uint32_t* __restrict__ src, uint32_t* __restrict__ vac_axon, uint32_t* __restrict__ con_axon,
                             uint32_t* __restrict__ err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) {
        return;
    }
    const uint32_t s = src[i];
    const uint32_t old = atomicSub(&vac_axon[s], 1u);
    if (old == 0) {
        atomicAdd(&vac_axon[s], 1u);  // leave the count as it was
        atomicOr(err, (uint32_t)DERR_CONNECT);
        return;
    }
    atomicAdd(&con_axon[s], 1u);
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

// ---- graph
__global__ void k_keep_flags(uint64_t m, const int32_t* __restrict__ w, uint32_t* __restrict__ keep) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        keep[i] = w[i] != 0 ? 1u : 0u;
    }
}

__global__ void k_compact_edges(uint64_t m, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos, const uint32_t* __restrict__ t_in,
                                const uint32_t* __restrict__ s_in, const int32_t* __restrict__ w_in, uint32_t* __restrict__ t_out,
                                uint32_t* __restrict__ s_out, int32_t* __restrict__ w_out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && keep[i]) {
        const uint32_t o = pos[i];
        t_out[o] = t_in[i];
        s_out[o] = s_in[i];
        w_out[o] = w_in[i];
    }
}

// ---- incremental graph update
// The edge list stays sorted by (target, source) and the out-CSR permutation
// by (source, target), equal pairs in insertion order.  A plasticity update
// adds a few thousand synapses to a list of millions, so the new ones are
// sorted alone and merged in: an old entry moves up by the number of new keys
// below its own, a new entry lands after every old entry with a key at or
// below its own (old entries first among equals, as a stable sort of the
// concatenation orders them).

__device__ __forceinline__ uint64_t pair_key(uint32_t hi, uint32_t lo, int bn) {
    return ((uint64_t)hi << bn) | lo;
}

// Number of keys in the sorted array k[0, n) below x (or at or below it).
__device__ __forceinline__ uint64_t count_below(const uint64_t* __restrict__ k, uint64_t n, uint64_t x, bool or_equal) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        const bool below = or_equal ? k[mid] <= x : k[mid] < x;
        if (below) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// Keys of the new entries and their indices, for the small sort.
__global__ void k_new_keys(uint64_t m, const uint32_t* __restrict__ hi, const uint32_t* __restrict__ lo, const uint32_t* __restrict__ map, int bn,
                           uint64_t* __restrict__ key, uint32_t* __restrict__ val) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        key[i] = pair_key(hi[i], lo[i], bn);
        val[i] = map ? map[i] : (uint32_t)i;
    }
}

// Old entries (sorted by (target, source)) into the merged list.
__global__ void k_merge_old(uint64_t m, const uint32_t* __restrict__ t, const uint32_t* __restrict__ src, const int32_t* __restrict__ w,
                            const uint64_t* __restrict__ nkey, uint64_t mn, int bn, uint32_t* __restrict__ pos, uint32_t* __restrict__ t_out,
                            uint32_t* __restrict__ s_out, int32_t* __restrict__ w_out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) {
        const uint64_t o = i + count_below(nkey, mn, pair_key(t[i], src[i], bn), false);
        pos[i] = (uint32_t)o;
        t_out[o] = t[i];
        s_out[o] = src[i];
        w_out[o] = w[i];
    }
}

// Number of old entries with a key at or below x (keys made from the sorted
// old arrays on the fly).
__device__ __forceinline__ uint64_t count_old_at_or_below(const uint32_t* __restrict__ hi, const uint32_t* __restrict__ lo,
                                                          const uint32_t* __restrict__ perm, uint64_t n, uint64_t x, int bn) {
    uint64_t a = 0, b = n;
    while (a < b) {
        const uint64_t mid = (a + b) >> 1;
        const uint32_t e = perm ? perm[mid] : (uint32_t)mid;
        if (pair_key(hi[e], lo[e], bn) <= x) {
            a = mid + 1;
        } else {
            b = mid;
        }
    }
    return a;
}

// New entries (sorted; val = index among the new ones) into the merged list;
// newpos[val] receives each one's place.
__global__ void k_merge_new(uint64_t mn, const uint64_t* __restrict__ nkey, const uint32_t* __restrict__ nval, const uint32_t* __restrict__ nt,
                            const uint32_t* __restrict__ ns, const int32_t* __restrict__ nw, const uint32_t* __restrict__ t, const uint32_t* __restrict__ src,
                            uint64_t m, int bn, uint32_t* __restrict__ newpos, uint32_t* __restrict__ t_out, uint32_t* __restrict__ s_out,
                            int32_t* __restrict__ w_out) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < mn) {
        const uint64_t o = j + count_old_at_or_below(t, src, nullptr, m, nkey[j], bn);
        const uint32_t v = nval[j];
        newpos[v] = (uint32_t)o;
        t_out[o] = nt[v];
        s_out[o] = ns[v];
        w_out[o] = nw[v];
    }
}

// The out-CSR permutation: old entries (in (source, target) order, as edge
// indices of the old list) moved to their merged indices and places.
__global__ void k_merge_out_old(uint64_t m, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ t, const uint32_t* __restrict__ src,
                                const uint32_t* __restrict__ pos, const uint64_t* __restrict__ nkey, uint64_t mn, int bn, uint32_t* __restrict__ out) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) {
        const uint32_t e = perm[k];
        out[k + count_below(nkey, mn, pair_key(src[e], t[e], bn), false)] = pos[e];
    }
}

__global__ void k_merge_out_new(uint64_t mn, const uint64_t* __restrict__ nkey, const uint32_t* __restrict__ nval, const uint32_t* __restrict__ perm,
                                const uint32_t* __restrict__ t, const uint32_t* __restrict__ src, uint64_t m, int bn, uint32_t* __restrict__ out) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < mn) {
        out[j + count_old_at_or_below(src, t, perm, m, nkey[j], bn)] = nval[j];
    }
}

// Row offsets of a list sorted by row: off[r] = the first entry whose row is
// r or more, for r = 0..n (entries e in [0, m]; `perm` maps list order to
// edge indices, or null).
__global__ void k_row_offsets(uint64_t m, const uint32_t* __restrict__ row, const uint32_t* __restrict__ perm, uint32_t n, uint32_t* __restrict__ off) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e > m) {
        return;
    }
    const uint32_t lo = e == 0 ? 0u : row[perm ? perm[e - 1] : (uint32_t)(e - 1)] + 1u;
    const uint32_t hi = e == m ? n : row[perm ? perm[e] : (uint32_t)e];
    for (uint32_t r = lo; r <= hi; ++r) {
        off[r] = (uint32_t)e;
    }
}

// Out-CSR entries that survive the zero compaction, renumbered.
__global__ void k_keep_out(uint64_t m, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ keep, uint32_t* __restrict__ keep_out) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) {
        keep_out[k] = keep[perm[k]];
    }
}

__global__ void k_compact_out(uint64_t m, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ keep_out, const uint32_t* __restrict__ opos,
                              const uint32_t* __restrict__ epos, uint32_t* __restrict__ out) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m && keep_out[k]) {
        out[opos[k]] = epos[perm[k]];
    }
}

struct DeleteArgs {
    uint32_t n;
    int type;  // 0 axon, 1 excitatory dendrite, 2 inhibitory dendrite
    uint32_t step;
    const NetInfo* nets;
    const uint16_t* net_of;
    const uint32_t* to_delete;
    const uint8_t* signal;
    const uint8_t* enabled;
    const uint32_t* in_off;
    const uint32_t* out_off;
    const uint32_t* out_perm;
    const uint32_t* etgt;
    const uint32_t* esrc;
    int32_t* ew;
    uint32_t* connected[3];
    uint32_t* vacant[3];
    unsigned long long* deleted;
    uint32_t* err;
};

constexpr uint32_t kMaxDeletePerNeuron = 64;

// Random synapse deletion for one element type (SynapseDeletionFinderCPU
// find_synapses_to_delete + commit_deletions, neurons/helper/
// SynapseDeletionFinderCPU.cpp:93-237; RandomSynapseDeletionFinder
// SynapseDeletionFinder.cpp:52-68).  A neuron's synapse list holds every
// partner |weight| times, ordered by partner id; d distinct indices are drawn
// (redrawing duplicates, util/Random.h:99-115).  Every synapse belongs to the
// list of exactly one neuron in a pass, so the weight updates need no atomics;
// the partners' elements are disconnected with atomics (integer, order free).
__global__ void k_delete(DeleteArgs A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) {
        return;
    }
    const uint32_t d = A.to_delete[i];
    if (d == 0 || !A.enabled[i]) {
        return;
    }
    const bool axon = A.type == 0;
    const int signal = axon ? (int)A.signal[i] : A.type - 1;
    const uint32_t r0 = axon ? A.out_off[i] : A.in_off[i];
    const uint32_t r1 = axon ? A.out_off[i + 1] : A.in_off[i + 1];
    auto edge_at = [&](uint32_t r) { return axon ? A.out_perm[r] : r; };
    auto matches = [&](int32_t w) { return axon || (signal == 0 ? w > 0 : w < 0); };
    uint32_t total = 0;
    for (uint32_t r = r0; r < r1; ++r) {
        const int32_t w = A.ew[edge_at(r)];
        if (matches(w)) {
            total += (uint32_t)(w < 0 ? -w : w);
        }
    }
    if (d > total || d > kMaxDeletePerNeuron) {
        atomicOr(A.err, (uint32_t)DERR_CONNECT);
        return;
    }
    uint32_t chosen[kMaxDeletePerNeuron];
    const NetInfo& N = A.nets[A.net_of[i]];
    for (uint32_t k = 0; k < d; ++k) {
        uint32_t idx = 0;
        bool ok = false;
        for (uint32_t attempt = 0; attempt < (1u << 20) && !ok; ++attempt) {
            const u32x4 w = draw(N.seed, A.step, i - N.first, ((uint32_t)A.type << 24) | k, STREAM_DELETION, attempt);
            idx = (uint32_t)__umul64hi(bits64(w), (uint64_t)total);
            ok = true;
            for (uint32_t q = 0; q < k; ++q) {
                if (chosen[q] == idx) {
                    ok = false;
                    break;
                }
            }
        }
        if (!ok) {
            atomicOr(A.err, (uint32_t)DERR_TIMEOUT);
            return;
        }
        chosen[k] = idx;
    }
    // sort the chosen list indices, then walk the row once over the original
    // multiplicities: entry e covers list indices [acc, acc + |w_e|)
    for (uint32_t a = 1; a < d; ++a) {
        const uint32_t v = chosen[a];
        uint32_t b = a;
        while (b > 0 && chosen[b - 1] > v) {
            chosen[b] = chosen[b - 1];
            --b;
        }
        chosen[b] = v;
    }
    uint32_t acc = 0;
    uint32_t q = 0;
    for (uint32_t r = r0; r < r1 && q < d; ++r) {
        const uint32_t e = edge_at(r);
        const int32_t w = A.ew[e];
        if (!matches(w)) {
            continue;
        }
        const uint32_t mult = (uint32_t)(w < 0 ? -w : w);
        uint32_t hits = 0;
        while (q < d && chosen[q] < acc + mult) {
            ++hits;
            ++q;
        }
        acc += mult;
        if (hits == 0) {
            continue;
        }
        A.ew[e] = w < 0 ? w + (int32_t)hits : w - (int32_t)hits;
        const uint32_t partner = axon ? A.etgt[e] : A.esrc[e];
        // ElementBaseBase::disconnect_elements (ElementBaseBase.h:311-319) on the partner
        const int pt = axon ? 1 + signal : 0;
        atomicSub(&A.connected[pt][partner], hits);
        atomicAdd(&A.vacant[pt][partner], hits);
    }
    atomicAdd(A.deleted, (unsigned long long)d);
}

}  // namespace

uint64_t run_connector(Ctx& c, uint32_t step, bool bind_axons) {
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
    k_conn_keys<<<blocks_for(m, 256), 256, 0, st>>>(m, n, S.req_tgt.p, S.req_src.p, S.req_j.p, S.req_sig.p, c.d_nets.p, c.net_of.p, step, S.ckey.p,
                                                    S.cidx.p, S.gkey.p);
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
    DBuf<uint32_t>& before = S.vac_before;
    before.fit(2 * (size_t)n);
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
    A.vac_axon = bind_axons ? c.nr.vacant[0].p : nullptr;
    A.con_axon = bind_axons ? c.nr.connected[0].p : nullptr;
    A.vac_exc_before = before.p;
    A.vac_inh_before = before.p + n;
    A.accepted = S.accepted.p;
    A.err = c.err.p;
    k_accept<<<blocks_for(m, 256), 256, 0, st>>>(A);
    RL_LAUNCH_CHECK();
    // compact accepted into the new-edge buffer (sorted-position order)
    DBuf<uint32_t>& pos = S.accept_pos;
    pos.fit(m);
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
        G.new_tgt.swap(t2);
        G.new_src.swap(s2);
        G.new_w.swap(w2);
    }
    k_emit_edges<<<blocks_for(m, 256), 256, 0, st>>>(m, S.accepted.p, pos.p, S.cidx.p, S.req_tgt.p, S.req_src.p, S.req_sig.p, G.num_new, G.new_tgt.p,
                                                     G.new_src.p, G.new_w.p);
    RL_LAUNCH_CHECK();
    G.num_new += created;
    check_device_error(c, "connector");
    c.stats.synapses_created += created;
    return created;
}

namespace {

int bits_for(uint64_t v) {
    int b = 1;
    while (b < 32 && ((uint64_t)1 << b) <= v) {
        ++b;
    }
    return b;
}

// The new entries' keys sorted with their values (insertion order among
// equal keys): one block for a plasticity update's few thousand, the radix
// sort beyond that.
// Stable sort of the new entries' keys (values: insertion index, or merged
// positions increasing with it among equal keys, so equal keys keep their
// insertion order); up to 4,096 entries in one launch.
void sort_new(Ctx& c, uint64_t* key, uint32_t* val, uint64_t m, int bits) {
    radix_sort_u64(key, val, m, bits, c.prim, c.stream);
}

}  // namespace

// Merges the new synapses into the sorted list and the out-CSR, drops the
// entries deletions left at weight 0 once they may be an eighth of the list,
// and rebuilds both row-offset arrays.
void rebuild_graph(Ctx& c) {
    Graph& G = c.graph;
    const bool compact = G.zeros && G.zero_bound * 8 >= G.num_edges + G.num_new;
    if (G.num_new == 0 && !compact) {
        return;
    }
    cudaStream_t st = c.stream;
    const uint32_t n = c.n;
    const uint64_t mo = G.num_edges;
    const uint64_t mn = G.num_new;
    uint64_t m = mo + mn;
    RL_CHECK(m < 0xFFFFFFFFull, RL_ERR_OVERFLOW, "synapse count exceeds 2^32");
    const int bn = bits_for(n);
    // the working arrays persist in the graph, so that a rebuild allocates
    // only when the list outgrows them; T, S, W and out become the graph's
    // lists below, and the lists they replace are the next rebuild's arrays
    DBuf<uint32_t>& T = G.m_tgt;
    DBuf<uint32_t>& S = G.m_src;
    DBuf<int32_t>& W = G.m_w;
    DBuf<uint32_t>& out = G.m_out;
    DBuf<uint32_t>& pos = G.m_pos;
    DBuf<uint32_t>& newpos = G.m_newpos;
    DBuf<uint64_t>& nk = G.m_nk;
    DBuf<uint32_t>& nv = G.m_nv;
    T.fit(m ? m : 1);
    S.fit(m ? m : 1);
    W.fit(m ? m : 1);
    out.fit(m ? m : 1);
    pos.fit(mo ? mo : 1);
    newpos.fit(mn ? mn : 1);
    nk.fit(mn ? mn : 1);
    nv.fit(mn ? mn : 1);
    // list order: new entries by (target, source), merged behind equal old ones
    if (mn) {
        k_new_keys<<<blocks_for(mn, 256), 256, 0, st>>>(mn, G.new_tgt.p, G.new_src.p, nullptr, bn, nk.p, nv.p);
        RL_LAUNCH_CHECK();
        sort_new(c, nk.p, nv.p, mn, 2 * bn);
    }
    if (mo) {
        k_merge_old<<<blocks_for(mo, 256), 256, 0, st>>>(mo, G.tgt.p, G.src.p, G.weight.p, nk.p, mn, bn, pos.p, T.p, S.p, W.p);
        RL_LAUNCH_CHECK();
    }
    if (mn) {
        k_merge_new<<<blocks_for(mn, 256), 256, 0, st>>>(mn, nk.p, nv.p, G.new_tgt.p, G.new_src.p, G.new_w.p, G.tgt.p, G.src.p, mo, bn, newpos.p, T.p,
                                                        S.p, W.p);
        RL_LAUNCH_CHECK();
        // out order: new entries by (source, target), valued by their merged index
        k_new_keys<<<blocks_for(mn, 256), 256, 0, st>>>(mn, G.new_src.p, G.new_tgt.p, newpos.p, bn, nk.p, nv.p);
        RL_LAUNCH_CHECK();
        sort_new(c, nk.p, nv.p, mn, 2 * bn);
    }
    if (mo) {
        k_merge_out_old<<<blocks_for(mo, 256), 256, 0, st>>>(mo, G.out_perm.p, G.tgt.p, G.src.p, pos.p, nk.p, mn, bn, out.p);
        RL_LAUNCH_CHECK();
    }
    if (mn) {
        k_merge_out_new<<<blocks_for(mn, 256), 256, 0, st>>>(mn, nk.p, nv.p, G.out_perm.p, G.tgt.p, G.src.p, mo, bn, out.p);
        RL_LAUNCH_CHECK();
    }
    if (compact && m) {
        // the entries deletions left at weight 0 go; the order stays
        DBuf<uint32_t> keep, epos, keep_out, opos, T2, S2, out2;
        DBuf<int32_t> W2;
        keep.alloc(m);
        epos.alloc(m);
        keep_out.alloc(m);
        opos.alloc(m);
        k_keep_flags<<<blocks_for(m, 256), 256, 0, st>>>(m, W.p, keep.p);
        RL_LAUNCH_CHECK();
        const uint64_t kept = exclusive_scan_u32(keep.p, epos.p, m, c.prim, st);
        k_keep_out<<<blocks_for(m, 256), 256, 0, st>>>(m, out.p, keep.p, keep_out.p);
        RL_LAUNCH_CHECK();
        exclusive_scan_u32_async(keep_out.p, opos.p, m, c.prim, st);
        T2.alloc(kept ? kept : 1);
        S2.alloc(kept ? kept : 1);
        W2.alloc(kept ? kept : 1);
        out2.alloc(kept ? kept : 1);
        k_compact_edges<<<blocks_for(m, 256), 256, 0, st>>>(m, keep.p, epos.p, T.p, S.p, W.p, T2.p, S2.p, W2.p);
        RL_LAUNCH_CHECK();
        k_compact_out<<<blocks_for(m, 256), 256, 0, st>>>(m, out.p, keep_out.p, opos.p, epos.p, out2.p);
        RL_LAUNCH_CHECK();
        T.swap(T2);
        S.swap(S2);
        W.swap(W2);
        out.swap(out2);
        m = kept;
    }
    G.tgt.swap(T);
    G.src.swap(S);
    G.weight.swap(W);
    G.out_perm.swap(out);
    G.num_edges = m;
    G.num_new = 0;
    if (compact) {
        G.zeros = false;
        G.zero_bound = 0;
    }
    G.offsets.ensure((size_t)n + 1);
    G.out_off.ensure((size_t)n + 1);
    k_row_offsets<<<blocks_for(m + 1, 256), 256, 0, st>>>(m, G.tgt.p, nullptr, n, G.offsets.p);
    RL_LAUNCH_CHECK();
    k_row_offsets<<<blocks_for(m + 1, 256), 256, 0, st>>>(m, G.src.p, G.out_perm.p, n, G.out_off.p);
    RL_LAUNCH_CHECK();
}

uint64_t run_deletion(Ctx& c, uint32_t step, int type) {
    Graph& G = c.graph;
    cudaStream_t st = c.stream;
    rebuild_graph(c);
    if (G.num_edges == 0) {
        // nothing to delete: the elements say otherwise only if the state was set inconsistently
        RL_CUDA_TRY(cudaMemsetAsync(c.err.p, 0, sizeof(uint32_t), st));
    }
    unsigned long long* d_cnt = reinterpret_cast<unsigned long long*>(c.counters.p) + 2;
    RL_CUDA_TRY(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st));
    DeleteArgs A;
    A.n = c.n;
    A.type = type;
    A.step = step;
    A.nets = c.d_nets.p;
    A.net_of = c.net_of.p;
    A.to_delete = c.to_delete.p;
    A.signal = c.nr.signal.p;
    A.enabled = c.nr.enabled.p;
    A.in_off = G.offsets.p;
    A.out_off = G.out_off.p;
    A.out_perm = G.out_perm.p;
    A.etgt = G.tgt.p;
    A.esrc = G.src.p;
    A.ew = G.weight.p;
    for (int t = 0; t < 3; ++t) {
        A.connected[t] = c.nr.connected[t].p;
        A.vacant[t] = c.nr.vacant[t].p;
    }
    A.deleted = d_cnt;
    A.err = c.err.p;
    k_delete<<<blocks_for(c.n, 128), 128, 0, st>>>(A);
    RL_LAUNCH_CHECK();
    check_device_error(c, "synapse deletion");
    unsigned long long deleted = 0;
    RL_CUDA_TRY(cudaMemcpyAsync(&deleted, d_cnt, sizeof(deleted), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    // Entries whose weight reached zero stay until a rebuild drops them (once
    // they may be an eighth of the list): a zero entry adds nothing to a
    // neuron's input and is no synapse to a later deletion (a partner appears
    // |weight| times), and the edge order and both CSRs stay valid meanwhile;
    // rl_get_edges aggregates pairs and leaves zero weights out.
    if (deleted) {
        G.zeros = true;
        G.zero_bound += deleted;
    }
    return deleted;
}

void bind_axons_host(Ctx& c, uint64_t m, const uint32_t* src) {
    if (m == 0) {
        return;
    }
    for (uint64_t k = 0; k < m; ++k) {
        RL_CHECK(src[k] < c.n, RL_ERR_INVALID, "source out of range");
    }
    DBuf<uint32_t> d;
    d.alloc(m);
    RL_CUDA_TRY(cudaMemcpyAsync(d.p, src, m * sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
    k_bind_axons<<<blocks_for(m, 256), 256, 0, c.stream>>>(m, d.p, c.nr.vacant[0].p, c.nr.connected[0].p, c.err.p);
    RL_LAUNCH_CHECK();
    check_device_error(c, "process_responses");
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
    G.new_tgt.swap(t2);
    G.new_src.swap(s2);
    G.new_w.swap(w2);
    G.num_new = need;
    rebuild_graph(c);
}

}  // namespace rl
