// Barnes-Hut target search: one search per vacant axon element.
//
// Reference semantics (relearn/source/algorithm):
//   BarnesHut::find_target_neurons (BarnesHutInternal/BarnesHut.cpp:36-94),
//   BarnesHutBase::find_target_neurons / find_target_neuron /
//   get_nodes_to_consider / test_acceptance_criterion (BarnesHutBase.h:72-298),
//   Kernel::pick_target / create_probability_interval (Kernel/Kernel.h:61-173),
//   GaussianDistributionKernel::get_probability (Kernel/Gaussian.h:62-68),
//   ProbabilityPicker::pick_target (util/ProbabilityPicker.h:46-112).
//
// A descent collects candidates by a depth-first walk that visits the
// children of every expanded node in descending octant order (the
// reference's LIFO stack), sums their weights in that order, draws
// r in [0, nextafter(total)) and picks the first candidate whose running sum
// reaches r.  Bit-exactness needs the same candidate order and the same
// sequential FP64 additions, so every sum here is a per-lane sequential sum in
// that order.
//
// Work split on the GPU:
//   * The descent from the root (about 3,000 candidates per search at 1M
//     neurons) runs as a warp packet: the 32 lanes are 32 searches whose
//     sources are adjacent in Morton order; the warp walks the tree once, a
//     node is expanded when any lane expands it, and each lane evaluates and
//     sums only the nodes it would visit itself.  Node records are loaded once
//     per warp (broadcast).  The running sum at the start of every child
//     subtree of the root is kept as a checkpoint, so the pick re-walks a
//     single root-child subtree per lane instead of the whole candidate list.
//   * Deeper descents (a handful of candidates) run per lane: a sum pass and a
//     pick pass over the chosen node's subtree.
//   * Walks carry no stack: they follow per-node escape links.
//   * A persistent form keeps the top levels of the octree in shared memory.
//   * For sparse search lists, one search per warp (k_search_wide): the lanes
//     evaluate a tree level of candidates side by side and the sum runs in
//     the reference's order over the collected candidates.
#include "bh_eval.cuh"
#include "bh_wide.cuh"
#include "rl_context.cuh"
#include "rl_math.cuh"

namespace rl {
namespace {



struct SearchArgs {
    const double4* rec;  // records of the searched dendrite type
    const double* maxdim;
    const uint4* meta;     // topo, escape link, FP32 cell length (k_meta)
    const uint32_t* first_key;  // Morton rank of the first neuron under a node
    const uint32_t* leaf_of;    // neuron -> leaf node
    uint32_t* tasks;       // persistent form: warp tasks handed out so far
    uint32_t num_nodes;
    const double *px, *py, *pz;
    const uint32_t* list_src;
    const uint32_t* list_j;
    // segments of the search list, one per network with searches: warps
    // [seg_warp[s], seg_warp[s+1]) handle list entries [seg_begin[s], seg_end[s])
    const uint32_t* seg_warp;
    const uint64_t* seg_begin;
    const uint64_t* seg_end;
    const uint32_t* seg_net;
    uint32_t num_segs;
    const NetInfo* nets;
    int32_t* target;
    double mu;
    uint32_t step;
    uint32_t* err;
    unsigned long long* touched;
    KernelParams kernel;
};

// Parameters of the network a warp searches in.
struct WarpNet {
    double theta;
    double scale;
    uint64_t seed;
    uint32_t root;
    uint32_t first;
};

// Random number of ProbabilityPicker::pick_target(values, key) for a total.
__device__ __forceinline__ double pick_threshold(double total, uint64_t seed, uint32_t step, uint32_t source, uint32_t j, uint32_t depth) {
    const double next = next_up_eps(total);
    const u32x4 w = draw(seed, step, source, j, STREAM_BH_PICK, depth);
    double r = uniform01(w) * next;
    if (r >= next) {
        r = total;
    }
    if (!(r > 0.0)) {
        r = 4.9406564584124654e-324;  // r == 0 picks the first positive weight
    }
    return r;
}

// The shared-memory copy of the first nodes of the node array (the top
// levels of the octree, breadth-first) in the persistent form; n = 0 elsewhere.
struct Hot64 {
    const double4* rec;
    const uint4* meta;
    const double* maxdim;
    uint32_t n;
};

template <bool HOT>
__device__ __forceinline__ void load_node(const SearchArgs& A, const Hot64& H, uint32_t i, double4& r, uint4& m, double& md) {
    if (HOT && i < H.n) {
        r = H.rec[i];
        m = H.meta[i];
        md = H.maxdim[i];
    } else {
        r = ldg4(&A.rec[i]);
        m = __ldg(&A.meta[i]);
        md = __ldg(&A.maxdim[i]);
    }
}

// Walks follow the reference's depth-first order without a stack: after a
// node that is not expanded the walk continues at the node's escape link
// (meta.z, k_meta), after an expanded node at its last child (children are
// visited 7..0, the LIFO order of BarnesHutBase::get_nodes_to_consider), so a
// walk keeps one node index.  Every walk visits a node at most once; a walk
// that leaves the node range or runs longer than the node count reports
// DERR_WALK instead of looping.
__device__ __forceinline__ uint32_t last_child(uint2 t) {
    return t.x + (uint32_t)__popc(topo_mask(t.y)) - 1u;
}

struct WalkResult {
    double sum;
    int32_t picked;  // node index in pick mode, -1 otherwise
    uint32_t touched;
};

// Per-lane walk of the subtree of `sub` (evaluating `sub` itself when
// `include_root`).  Sum mode adds all weights; pick mode stops at the first
// candidate whose running sum reaches r and returns it.
template <bool HOT>
__device__ WalkResult lane_walk(const SearchArgs& A, const Hot64& H, const WarpNet& W, uint32_t sub, bool include_root, double start_sum,
                                bool pick_mode, double r, double sx, double sy, double sz, uint32_t source, bool fallback, bool& bad) {
    WalkResult res{ start_sum, -1, 0 };
    double4 rs;
    uint4 ms;
    double mds;
    load_node<HOT>(A, H, sub, rs, ms, mds);
    const uint2 ts = make_uint2(ms.x, ms.y);
    if (include_root) {
        const Eval e = evaluate(rs, ts, mds, sx, sy, sz, source, W.theta, A.mu, W.scale, fallback, A.kernel);
        ++res.touched;
        if (e.status == ST_ACCEPT) {
            res.sum += e.w;
            if (pick_mode && res.sum >= r) {
                res.picked = (int32_t)sub;
            }
            return res;
        }
        if (e.status == ST_DISCARD) {
            return res;
        }
    }
    const uint32_t end = ms.z;
    uint32_t node = last_child(ts);
    for (uint32_t guard = 0; node != end; ++guard) {
        if (node >= A.num_nodes || guard >= A.num_nodes) {
            bad = true;
            return res;
        }
        double4 rr;
        uint4 mm;
        double md;
        load_node<HOT>(A, H, node, rr, mm, md);
        const uint2 tt = make_uint2(mm.x, mm.y);
        const Eval e = evaluate(rr, tt, md, sx, sy, sz, source, W.theta, A.mu, W.scale, fallback, A.kernel);
        ++res.touched;
        if (e.status == ST_ACCEPT) {
            res.sum += e.w;
            if (pick_mode && res.sum >= r) {
                res.picked = (int32_t)node;
                return res;
            }
        }
        node = e.status == ST_EXPAND ? last_child(tt) : mm.z;
    }
    return res;
}

// Checkpoints of a packet walk, per lane: the running sum before each child
// of the root, and, where the lane expanded them, before each child of its own
// level-1 and level-2 ancestors (the cells that contain its source; every
// walk expands them for theta < 1/sqrt(3)).  The pick re-walks only the
// smallest of these subtrees that holds the crossing.  Kept in local memory
// (written at the top three levels only).
constexpr int kCpPerLevel = 8;
struct Ancestry {
    uint32_t a1 = kNoNode, a1_first = 0, a1_n = 0;  // level-1 ancestor and its children
    uint32_t a2 = kNoNode, a2_first = 0, a2_n = 0;  // level-2 ancestor and its children
    bool valid2 = false, valid3 = false;            // checkpoints below a1 / a2 recorded
};

__device__ __forceinline__ uint32_t inner_children(const uint4& m) {
    return topo_leaf(m.y) ? 0u : (uint32_t)__popc(topo_mask(m.y));
}

// Packet walk over the whole tree: the lanes of packet mask `pm` (a warp or
// an aligned part of it) walk together; `lanes` are the packet's active lanes.
// A node is expanded when any lane expands it; a lane that does not expand a
// node the packet expands sits out the node's subtree (it keeps the node's
// escape link and joins again there), so each lane evaluates exactly the nodes
// of its own walk and returns its own sequential sum.  `my_rank` is the Morton
// rank of the lane's source; `cp` receives its checkpoints.
template <bool HOT>
__device__ double packet_walk(const SearchArgs& A, const Hot64& H, const WarpNet& W, uint32_t pm, uint32_t lanes, double sx, double sy, double sz,
                              uint32_t source, uint32_t my_rank, bool fallback, double* cp, Ancestry& an, uint32_t& touched, bool& bad) {
    const int lane = threadIdx.x & 31;
    const bool me = (lanes >> lane) & 1u;
    double sum = 0.0;
    an = Ancestry{};
    const uint4 rm = __ldg(&A.meta[W.root]);
    const uint32_t first0 = rm.x;
    const uint32_t root_level = topo_level(rm.y);
    uint32_t node = last_child(make_uint2(rm.x, rm.y));
    bool act = me;
    uint32_t resume = kNoNode;
    for (uint32_t guard = 0; node != kNoNode; ++guard) {
        if (node >= A.num_nodes || guard >= A.num_nodes) {
            bad = true;
            break;
        }
        if (!act && node == resume) {
            act = true;
            resume = kNoNode;
        }
        double4 rr;
        uint4 mm;
        double md;
        load_node<HOT>(A, H, node, rr, mm, md);
        const uint2 tt = make_uint2(mm.x, mm.y);
        const uint32_t lvl = topo_level(mm.y) - root_level;
        if (lvl <= 3u) {  // the top of the tree: checkpoints (the branch is uniform)
            if (lvl == 1u) {
                if (me) {
                    cp[node - first0] = sum;
                    if (an.a1 == kNoNode && __ldg(&A.first_key[node]) <= my_rank) {
                        an.a1 = node;
                        an.a1_first = mm.x;
                        an.a1_n = inner_children(mm);
                    }
                }
            } else if (lvl == 2u) {
                if (act && node - an.a1_first < an.a1_n) {
                    cp[kCpPerLevel + (node - an.a1_first)] = sum;
                    an.valid2 = true;
                    if (an.a2 == kNoNode && __ldg(&A.first_key[node]) <= my_rank) {
                        an.a2 = node;
                        an.a2_first = mm.x;
                        an.a2_n = inner_children(mm);
                    }
                }
            } else if (lvl == 3u) {
                if (act && node - an.a2_first < an.a2_n) {
                    cp[2 * kCpPerLevel + (node - an.a2_first)] = sum;
                    an.valid3 = true;
                }
            }
        }
        int status = ST_DISCARD;
        if (act) {
            const Eval e = evaluate(rr, tt, md, sx, sy, sz, source, W.theta, A.mu, W.scale, fallback, A.kernel);
            status = e.status;
            ++touched;
            if (e.status == ST_ACCEPT) {
                sum += e.w;
            }
        }
        const uint32_t expand = __ballot_sync(pm, status == ST_EXPAND);
        if (expand) {
            if (act && status != ST_EXPAND) {
                act = false;
                resume = mm.z;
            }
            node = last_child(tt);
        } else {
            node = mm.z;
        }
    }
    __syncwarp(pm);
    return sum;
}

// The child (first + k) of a checkpointed level that holds the crossing of r:
// the last child in walking order (children are walked in descending rank)
// whose checkpoint lies below r; -1 if none does.
__device__ __forceinline__ int crossing_child(const double* cp, uint32_t n, double r) {
    int k = -1;
    for (int q = (int)n - 1; q >= 0; --q) {
        if (cp[q] < r) {
            k = q;
        } else {
            break;
        }
    }
    return k;
}

// The searches of one warp task: 32 consecutive entries of the search list
// (Morton-adjacent sources) as 32/PW packets of PW lanes.
template <int PW, bool HOT>
__device__ __forceinline__ void search_task(const SearchArgs& A, const Hot64& H, uint32_t warp_global) {
    const int lane = threadIdx.x & 31;
    const int pk = lane / PW;
    const uint32_t pm = PW == 32 ? 0xFFFFFFFFu : (((1u << PW) - 1u) << (pk * PW));
    if (warp_global >= A.seg_warp[A.num_segs]) {
        return;  // whole warp idle
    }
    // segment (network) of this warp
    uint32_t lo = 0, hi = A.num_segs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (A.seg_warp[mid] <= warp_global) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    const NetInfo& N = A.nets[A.seg_net[lo]];
    const WarpNet W{ N.theta, N.scale, N.seed, A.seg_net[lo], N.first };
    const uint64_t idx = A.seg_begin[lo] + (uint64_t)(warp_global - A.seg_warp[lo]) * 32 + lane;
    const bool active = idx < A.seg_end[lo];
    if (N.root_leaf) {
        // a network of one neuron: its only candidate is itself
        if (active) {
            A.target[idx] = -1;
        }
        return;
    }
    const uint32_t source = active ? A.list_src[idx] : 0u;
    const uint32_t j = active ? A.list_j[idx] : 0u;
    const double sx = active ? A.px[source] : 0.0;
    const double sy = active ? A.py[source] : 0.0;
    const double sz = active ? A.pz[source] : 0.0;
    const uint32_t my_rank = active ? __ldg(&A.first_key[__ldg(&A.leaf_of[source])]) : 0u;
    double cp[3 * kCpPerLevel];
    Ancestry an;
    uint32_t touched = 0;
    bool overflow = false;
    bool bad = false;
    const uint32_t lanes = __ballot_sync(pm, active);
    int32_t result = -1;
    bool done = !active;
    uint32_t sub = 0;
    if (lanes) {
        // ---- descent 0: packet walk over the whole tree
        double total = packet_walk<HOT>(A, H, W, pm, lanes, sx, sy, sz, source, my_rank, false, cp, an, touched, bad);
        bool fallback = false;
        const uint32_t need_fb = __ballot_sync(pm, active && total == 0.0);
        if (need_fb) {
            uint32_t t2 = 0;
            Ancestry an_fb;
            const double fb = packet_walk<HOT>(A, H, W, pm, need_fb, sx, sy, sz, source, my_rank, true, cp, an_fb, t2, bad);
            if ((need_fb >> lane) & 1u) {
                total = fb;
                fallback = true;
                an = an_fb;
            }
        }
        if (active && total == 0.0) {
            done = true;  // no candidate: the search fails
        }
        if (!done) {
            const double r = pick_threshold(total, W.seed, A.step, source - W.first, j, 0);
            // the crossing lies in the last root child (walking order) whose
            // checkpoint is below r; inside the lane's own ancestors, in the
            // last of their checkpointed children below r
            const uint4 rm = __ldg(&A.meta[W.root]);
            const int k1 = crossing_child(cp, inner_children(rm), r);
            if (k1 < 0) {
                atomicOr(A.err, (uint32_t)DERR_NO_CROSSING);
                done = true;
            } else {
                uint32_t c0 = rm.x + (uint32_t)k1;
                double start = cp[k1];
                if (an.valid2 && c0 == an.a1) {
                    const int k2 = crossing_child(cp + kCpPerLevel, an.a1_n, r);
                    if (k2 >= 0) {
                        c0 = an.a1_first + (uint32_t)k2;
                        start = cp[kCpPerLevel + k2];
                        if (an.valid3 && c0 == an.a2) {
                            const int k3 = crossing_child(cp + 2 * kCpPerLevel, an.a2_n, r);
                            if (k3 >= 0) {
                                c0 = an.a2_first + (uint32_t)k3;
                                start = cp[2 * kCpPerLevel + k3];
                            }
                        }
                    }
                }
                const WalkResult wr = lane_walk<HOT>(A, H, W, c0, true, start, true, r, sx, sy, sz, source, fallback, bad);
                if (wr.picked < 0) {
                    atomicOr(A.err, (uint32_t)DERR_NO_CROSSING);
                    done = true;
                } else {
                    sub = (uint32_t)wr.picked;
                }
            }
        }
    }
    // ---- deeper descents, per lane
    for (uint32_t depth = 1; !done; ++depth) {
        if (depth > (uint32_t)kMaxLevels + 2u) {
            overflow = true;  // a descent always moves one level down; cannot recur this often
            break;
        }
        const uint4 sm = __ldg(&A.meta[sub]);
        if (topo_leaf(sm.y)) {
            result = (int32_t)sm.x;
            done = true;
            break;
        }
        WalkResult s1 = lane_walk<HOT>(A, H, W, sub, false, 0.0, false, 0.0, sx, sy, sz, source, false, bad);
        touched += s1.touched;
        bool fb = false;
        if (s1.sum == 0.0) {
            s1 = lane_walk<HOT>(A, H, W, sub, false, 0.0, false, 0.0, sx, sy, sz, source, true, bad);
            fb = true;
        }
        if (s1.sum == 0.0 || bad) {
            done = true;
            break;
        }
        const double r = pick_threshold(s1.sum, W.seed, A.step, source - W.first, j, depth);
        const WalkResult s2 = lane_walk<HOT>(A, H, W, sub, false, 0.0, true, r, sx, sy, sz, source, fb, bad);
        if (s2.picked < 0) {
            atomicOr(A.err, (uint32_t)DERR_NO_CROSSING);
            done = true;
            break;
        }
        sub = (uint32_t)s2.picked;
    }
    if (overflow) {
        atomicOr(A.err, (uint32_t)DERR_STACK);
        result = -1;
    }
    if (bad) {
        atomicOr(A.err, (uint32_t)DERR_WALK);
        result = -1;
    }
    if (active) {
        A.target[idx] = result;
    }
    // touched-node counter (reference-equivalent acceptance tests)
    unsigned long long t = touched;
    for (int o = 16; o > 0; o >>= 1) {
        t += __shfl_down_sync(0xFFFFFFFFu, t, o);
    }
    if (lane == 0) {
        atomicAdd(A.touched, t);
    }
}

// One warp task per warp.  WPB warps per block; CAP = 1 caps the registers at
// 64 (a resident block count of 32 / WPB), for more warps in flight.
template <int WPB, int PW, int CAP>
__global__ void __launch_bounds__(WPB * 32, CAP ? 32 / WPB : 1) k_search(SearchArgs A) {
    const int wib = threadIdx.x >> 5;
    search_task<PW, false>(A, Hot64{ nullptr, nullptr, nullptr, 0u }, blockIdx.x * WPB + wib);
}

// Persistent form: one block of 32 warps per SM.  The block first copies the
// first `hot` nodes (the top levels of the octree) into shared memory, then
// its warps take warp tasks until none are left: one each by block and warp
// index, then the next free one from the task counter.
template <int PW>
__global__ void __launch_bounds__(1024, 1) k_search_hot(SearchArgs A, uint32_t hot) {
    extern __shared__ __align__(16) unsigned char smem[];
    double4* hrec = reinterpret_cast<double4*>(smem);
    uint4* hmeta = reinterpret_cast<uint4*>(hrec + hot);
    double* hmd = reinterpret_cast<double*>(hmeta + hot);
    for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) {
        hrec[i] = ldg4(&A.rec[i]);
        hmeta[i] = __ldg(&A.meta[i]);
        hmd[i] = __ldg(&A.maxdim[i]);
    }
    __syncthreads();
    const Hot64 H{ hrec, hmeta, hmd, hot };
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t total = A.seg_warp[A.num_segs];
    uint32_t w = blockIdx.x * 32 + wib;
    while (w < total) {
        search_task<PW, true>(A, H, w);
        uint32_t next = 0;
        if (lane == 0) {
            next = atomicAdd(A.tasks, 1u) + gridDim.x * 32;
        }
        w = __shfl_sync(0xFFFFFFFFu, next, 0);
    }
}

// ------------------------------------------------- one search per warp
// (bh_wide.cuh): the FP64 evaluation, search and kernel.
// Both signal types' search lists in one launch: the tasks of S[0] (the
// excitatory list) first, then those of S[1]; a type without searches has no
// tasks.  Every search waits on memory round after round, so the lists of the
// two types share the device instead of running one launch after the other.
struct WideArgs {
    SearchArgs S[2];
    uint32_t num_tasks[2];
    WideSlot all;        // scratch of every warp slot, `cap` entries each
    uint32_t cap;
    uint32_t slots;
    uint32_t* tasks;     // task counter over both lists
    uint32_t* overflow;  // per type: searches left to the packet kernel
    unsigned long long* touched;
};

__device__ __forceinline__ WideSlot wide_slot(const WideSlot& all, uint64_t off) {
    return WideSlot{ all.node + off, all.info + off, all.child + off, all.cnt + off, all.pos + off, all.ord_node + off, all.w + off, all.ord_w + off };
}

// The FP64 candidates of the subtree of `sub` in visiting order.
__device__ __forceinline__ int64_t wide_collect64(const SearchArgs& S, uint32_t cap, const WideSlot& P, const WarpNet& W, uint32_t sub, double sx,
                                                  double sy, double sz, uint32_t source, uint32_t* s_round, uint32_t& touched) {
    const uint4 sm = __ldg(&S.meta[sub]);
    return wide_collect(P, cap, sm.x, inner_children(sm), s_round, touched, [&](uint32_t nd) {
        WideEval r{ ST_DISCARD, 0.0, 0u, 0u, false };
        if (nd >= S.num_nodes) {
            r.bad = true;
            return r;
        }
        const uint4 mm = __ldg(&S.meta[nd]);
        const Eval ev = evaluate(ldg4(&S.rec[nd]), make_uint2(mm.x, mm.y), __ldg(&S.maxdim[nd]), sx, sy, sz, source, W.theta, S.mu, W.scale, false,
                                 S.kernel);
        r.status = ev.status;
        r.w = ev.w;
        if (ev.status == ST_EXPAND) {
            r.nch = (uint32_t)__popc(topo_mask(mm.y));
            r.first = mm.x;
        }
        return r;
    }, [&](uint32_t nd) {
        if (nd < S.num_nodes) {
            prefetch_l1(&S.meta[nd]);
            prefetch_l1(&S.rec[nd]);
            prefetch_l1(&S.maxdim[nd]);
        }
    });
}

// One search (one vacant axon element j of `source`) by the whole warp:
// the target neuron, -1 when the search fails, kRedo when it did not fit.
__device__ int32_t wide_search(const SearchArgs& S, uint32_t cap, const WideSlot& P, const WarpNet& W, uint32_t source, uint32_t j, uint32_t* s_round,
                               uint32_t& touched) {
    const double sx = S.px[source], sy = S.py[source], sz = S.pz[source];
    uint32_t sub = W.root;
    for (uint32_t depth = 0; depth <= (uint32_t)kMaxLevels + 2u; ++depth) {
        const uint4 sm = __ldg(&S.meta[sub]);
        if (topo_leaf(sm.y)) {
            return depth == 0 ? -1 : (int32_t)sm.x;
        }
        const int64_t got = wide_collect64(S, cap, P, W, sub, sx, sy, sz, source, s_round, touched);
        if (got == -1) {
            return kRedo;
        }
        if (got < 0) {
            atomicOr(S.err, (uint32_t)DERR_WALK);
            return -1;
        }
        const uint32_t F = (uint32_t)got;
        double total = wide_running_sum64(P.ord_w, F);
        if (total == 0.0) {
            // every weight underflowed: count / distance weights over the same candidates
            for (uint32_t i = threadIdx.x & 31; i < F; i += 32) {
                const uint32_t nd = P.ord_node[i];
                const uint4 mm = __ldg(&S.meta[nd]);
                const Eval ev = evaluate(ldg4(&S.rec[nd]), make_uint2(mm.x, mm.y), __ldg(&S.maxdim[nd]), sx, sy, sz, source, W.theta, S.mu, W.scale,
                                         true, S.kernel);
                P.ord_w[i] = ev.w;
            }
            __syncwarp();
            total = wide_running_sum64(P.ord_w, F);
        }
        if (total == 0.0) {
            return -1;  // no candidate: the search fails
        }
        const double r = pick_threshold(total, W.seed, S.step, source - W.first, j, depth);
        const int64_t pick = wide_pick(P.ord_w, P.ord_node, F, r);
        if (pick < 0) {
            atomicOr(S.err, (uint32_t)DERR_NO_CROSSING);
            return -1;
        }
        sub = (uint32_t)pick;
        __syncwarp();  // the next descent overwrites the scratch this one read
    }
    atomicOr(S.err, (uint32_t)DERR_STACK);
    return -1;
}

// Persistent warps, one search per task: the task counter hands out list
// entries (32 per warp task of the packet kernels' segment layout).
template <int WPB>
__global__ void __launch_bounds__(WPB * 32, 2) k_search_wide(WideArgs A) {
    __shared__ uint32_t s_round_all[WPB][kWideRounds + 1];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * WPB + (uint32_t)wib;
    if (slot >= A.slots) {
        return;  // whole warp
    }
    uint32_t* s_round = s_round_all[wib];
    const WideSlot P = wide_slot(A.all, (uint64_t)slot * A.cap);
    const uint32_t total0 = A.num_tasks[0];
    const uint32_t total_tasks = total0 + A.num_tasks[1];
    uint32_t touched = 0;
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) {
            task = atomicAdd(A.tasks, 1u);
        }
        task = __shfl_sync(0xFFFFFFFFu, task, 0);
        if (task >= total_tasks) {
            break;
        }
        const int t = task < total0 ? 0 : 1;
        const SearchArgs& S = A.S[t];
        uint32_t lo = 0;
        uint64_t idx = 0;
        if (!wide_task_entry(task - (t ? total0 : 0u), S.seg_warp, S.seg_begin, S.seg_end, S.num_segs, lo, idx)) {
            continue;
        }
        const NetInfo& N = S.nets[S.seg_net[lo]];
        const WarpNet W{ N.theta, N.scale, N.seed, S.seg_net[lo], N.first };
        int32_t result = -1;
        if (!N.root_leaf) {
            result = wide_search(S, A.cap, P, W, S.list_src[idx], S.list_j[idx], s_round, touched);
        }
        if (lane == 0) {
            S.target[idx] = result;
            if (result == kRedo) {
                atomicAdd(A.overflow + t, 1u);
            }
        }
        __syncwarp();
    }
    unsigned long long sum = touched;
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xFFFFFFFFu, sum, o);
    }
    if (lane == 0) {
        atomicAdd(A.touched, sum);
    }
}

using SearchKernel = void (*)(SearchArgs);
using HotKernel = void (*)(SearchArgs, uint32_t);

// The search variants the tuner chooses from, indexed by SearchVariant.
SearchKernel fp64_search_kernel(const SearchVariant& v) {
#define RL_SV(w, p, c)                                            \
    if (v.hot == 0 && v.warps == w && v.packet == p && v.cap == c) { \
        return &k_search<w, p, c>;                                \
    }
#define RL_SV2(w, p) RL_SV(w, p, 0) RL_SV(w, p, 1)
    RL_SV2(2, 32) RL_SV2(4, 32) RL_SV2(8, 32) RL_SV2(2, 16) RL_SV2(4, 16) RL_SV2(8, 16)
    RL_SV2(2, 4) RL_SV2(4, 4) RL_SV2(8, 4) RL_SV2(2, 1) RL_SV2(4, 1) RL_SV2(8, 1)
#undef RL_SV2
#undef RL_SV
    return nullptr;
}

HotKernel fp64_hot_kernel(const SearchVariant& v) {
    if (v.hot == 0) {
        return nullptr;
    }
    return v.packet == 16 ? &k_search_hot<16> : &k_search_hot<32>;
}

// ---------------------------------------------------------- search list
__global__ void k_search_counts(uint32_t n, const uint32_t* __restrict__ morton, const uint8_t* __restrict__ enabled, const uint8_t* __restrict__ signal,
                                const uint32_t* __restrict__ vacant, uint32_t* __restrict__ cnt_exc, uint32_t* __restrict__ cnt_inh) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) {
        return;
    }
    const uint32_t nid = morton[r];
    const uint32_t v = enabled[nid] ? vacant[nid] : 0u;
    const bool inh = signal[nid] != 0;
    cnt_exc[r] = inh ? 0u : v;
    cnt_inh[r] = inh ? v : 0u;
}

__global__ void k_search_fill(uint32_t n, const uint32_t* __restrict__ morton, const uint8_t* __restrict__ enabled, const uint8_t* __restrict__ signal,
                              const uint32_t* __restrict__ vacant, const uint32_t* __restrict__ off_exc, const uint32_t* __restrict__ off_inh,
                              uint64_t num_exc, uint32_t* __restrict__ list_src, uint32_t* __restrict__ list_j) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) {
        return;
    }
    const uint32_t nid = morton[r];
    const uint32_t v = enabled[nid] ? vacant[nid] : 0u;
    const bool inh = signal[nid] != 0;
    const uint64_t base = inh ? num_exc + off_inh[r] : off_exc[r];
    for (uint32_t j = 0; j < v; ++j) {
        list_src[base + j] = nid;
        list_j[base + j] = j;
    }
}

// Start of every network's searches in the exclusive scans of both types.
__global__ void k_net_starts(uint32_t K, const NetInfo* __restrict__ nets, const uint32_t* __restrict__ off_exc, const uint32_t* __restrict__ off_inh,
                             uint32_t n, uint32_t* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) {
        const uint32_t f = nets[k].first;
        out[k] = off_exc[f];
        out[K + k] = off_inh[f];
    }
}

__global__ void k_fill_u32(uint32_t* p, uint64_t n, uint32_t v) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        p[i] = v;
    }
}

// BarnesHutBase::find_target_neurons stops a neuron's loop at its first
// failed search: record the smallest failing j per source.
__global__ void k_first_fail(uint64_t m, const uint32_t* __restrict__ list_src, const uint32_t* __restrict__ list_j, const int32_t* __restrict__ target,
                             uint32_t* __restrict__ first_fail) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m && target[i] < 0) {
        atomicMin(&first_fail[list_src[i]], list_j[i]);
    }
}

__global__ void k_req_count(uint32_t n, const uint32_t* __restrict__ first_fail, const uint32_t* __restrict__ vacant, const uint8_t* __restrict__ enabled,
                            uint32_t* __restrict__ cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const uint32_t v = enabled[i] ? vacant[i] : 0u;
    const uint32_t f = first_fail[i];
    cnt[i] = f < v ? f : v;
}

__global__ void k_req_scatter(uint64_t m, const uint32_t* __restrict__ list_src, const uint32_t* __restrict__ list_j, const int32_t* __restrict__ target,
                              const uint32_t* __restrict__ first_fail, const uint32_t* __restrict__ off, const uint8_t* __restrict__ signal,
                              uint32_t* __restrict__ rt, uint32_t* __restrict__ rs, uint32_t* __restrict__ rj, uint32_t* __restrict__ rg) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) {
        return;
    }
    const uint32_t s = list_src[i];
    const uint32_t j = list_j[i];
    if (j >= first_fail[s] || target[i] < 0) {
        return;
    }
    const uint32_t o = off[s] + j;
    rt[o] = (uint32_t)target[i];
    rs[o] = s;
    rj[o] = j;
    rg[o] = signal[s];
}

}  // namespace

// Walk entries per warp of the one-search-per-warp form: a descent evaluates
// every node at most once, so a small tree never overflows.
uint32_t wide_cap(const Ctx& c) {
    return (uint32_t)std::min<uint64_t>(kWideCap, (c.tree.num_nodes + 31) / 32 * 32);
}

// The scratch of `slots` warps of `cap` entries each (grown as needed).
WideSlot wide_scratch(Ctx& c, uint32_t slots, uint32_t cap) {
    Search& S = c.search;
    const size_t cells = (size_t)slots * cap;
    S.w_node.ensure(cells);
    S.w_info.ensure(cells);
    S.w_child.ensure(cells);
    S.w_cnt.ensure(cells);
    S.w_pos.ensure(cells);
    S.w_ord_node.ensure(cells);
    S.w_w.ensure(cells);
    S.w_ord_w.ensure(cells);
    return WideSlot{ S.w_node.p, S.w_info.p, S.w_child.p, S.w_cnt.p, S.w_pos.p, S.w_ord_node.p, S.w_w.p, S.w_ord_w.p };
}

// Whether the tuner times a candidate shape on this context's search list:
// the one-search-per-warp form pays off on large networks with sparse lists
// only (on a dense list its scratch would hold a warp slot per resident warp
// for nothing: packets of Morton neighbours are several times faster there).
bool search_variant_applies(const Ctx& c, const SearchVariant& v) {
    return v.packet != 0 || (c.n >= kWideMinNeurons && search_density_class(c.n, c.search.num_searches) != 0);
}

namespace {

// The one-search-per-warp kernel on both signal types' lists (warps[t]
// packet-layout warps of type t, 0 for a type without searches); a type with
// searches that did not fit their warp's scratch is redone by the packet
// kernel (which writes every target of its list again).
void launch_wide(Ctx& c, const SearchArgs (&a)[2], const uint32_t (&warps)[2]) {
    constexpr int WPB = 4;
    Search& S = c.search;
    cudaStream_t st = c.stream;
    const uint32_t tasks = (warps[0] + warps[1]) * 32u;
    const uint32_t cap = wide_cap(c);
    const uint32_t slots = std::min<uint32_t>(tasks, (uint32_t)c.num_sms * kWideWarpsPerSM);
    S.w_overflow.ensure(2);
    RL_CUDA_TRY(cudaMemsetAsync(S.tasks.p, 0, sizeof(uint32_t), st));
    RL_CUDA_TRY(cudaMemsetAsync(S.w_overflow.p, 0, 2 * sizeof(uint32_t), st));
    WideArgs A;
    for (int t = 0; t < 2; ++t) {
        A.S[t] = a[t];
        A.num_tasks[t] = warps[t] * 32u;
    }
    A.all = wide_scratch(c, slots, cap);
    A.cap = cap;
    A.slots = slots;
    A.tasks = S.tasks.p;
    A.overflow = S.w_overflow.p;
    A.touched = reinterpret_cast<unsigned long long*>(c.counters.p);
    k_search_wide<WPB><<<(slots + WPB - 1) / WPB, WPB * 32, 0, st>>>(A);
    RL_LAUNCH_CHECK();
    uint32_t over[2] = { 0, 0 };
    RL_CUDA_TRY(cudaMemcpyAsync(over, S.w_overflow.p, sizeof(over), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    for (int t = 0; t < 2; ++t) {
        if (over[t]) {
            k_search<2, 32, 1><<<(warps[t] + 1) / 2, 64, 0, st>>>(a[t]);
            RL_LAUNCH_CHECK();
        }
    }
}

}  // namespace

// Times every search variant that fits the octree on the current search list
// and keeps the fastest.  Each variant runs twice (the second run is timed);
// the searches are deterministic, so the variants leave the same targets, and
// the touched-node counter is restored afterwards.
template <typename F>
void tune_search(Ctx& c, F&& launch_all) {
    cudaStream_t st = c.stream;
    std::vector<uint64_t> saved(4);
    RL_CUDA_TRY(cudaMemcpyAsync(saved.data(), c.counters.p, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    cudaEvent_t e0, e1;
    RL_CUDA_TRY(cudaEventCreate(&e0));
    RL_CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    SearchVariant pick = c.tune.search;
    for (const SearchVariant& v : search_variants()) {
        if (!search_variant_applies(c, v)) {
            c.tune.search_ms.push_back(0.0f);  // keeps the times in candidate order
            continue;
        }
        launch_all(v);
        RL_CUDA_TRY(cudaEventRecord(e0, st));
        launch_all(v);
        RL_CUDA_TRY(cudaEventRecord(e1, st));
        RL_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.0f;
        RL_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        c.tune.search_ms.push_back(ms);
        if (ms < best) {
            best = ms;
            pick = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    RL_CUDA_TRY(cudaMemcpyAsync(c.counters.p, saved.data(), 4 * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    c.tune.search = pick;
}

const std::vector<SearchVariant>& search_variants() {
    static const std::vector<SearchVariant> v = [] {
        std::vector<SearchVariant> out;
        // packets of 32 or 16 Morton-adjacent searches suit dense search lists;
        // on sparse ones the sources of a packet lie far apart and the packet
        // walks the union of their walks, so packets of 4 and single-lane walks
        // are candidates too
        for (int cap : { 0, 1 }) {
            for (int p : { 32, 16, 4, 1 }) {
                for (int w : { 2, 4, 8 }) {
                    out.push_back(SearchVariant{ w, p, cap, 0 });
                }
            }
        }
        for (int hot : { 1024, 4096 }) {
            for (int p : { 32, 16 }) {
                out.push_back(SearchVariant{ 32, p, 1, hot });
            }
        }
        // one search per warp (packet 0; FP64 form, large networks): for
        // search lists whose sources lie far apart
        out.push_back(SearchVariant{ 4, 0, 0, 0 });
        return out;
    }();
    return v;
}

// Nodes of the persistent form's shared-memory copy: the shape's cap, no more
// than the octree has and than fit in a block's shared memory.
uint32_t hot_nodes(const Ctx& c, const SearchVariant& v, size_t node_bytes) {
    if (v.hot <= 0) {
        return 0;
    }
    const size_t room = (size_t)c.smem_optin / node_bytes;
    size_t h = std::min<size_t>((size_t)v.hot, room);
    h = std::min<size_t>(h, c.tree.num_nodes);
    return (uint32_t)(h & ~(size_t)1);  // even: keeps the last array of the copy 16-byte aligned
}

void run_search(Ctx& c, uint32_t step) {
    const uint32_t n = c.n;
    cudaStream_t st = c.stream;
    Search& S = c.search;
    S.counts.ensure(2 * (size_t)n + 2);
    uint32_t* cnt_exc = S.counts.p;
    uint32_t* cnt_inh = S.counts.p + n;
    k_search_counts<<<blocks_for(n, 256), 256, 0, st>>>(n, c.tree.morton.p, c.nr.enabled.p, c.nr.signal.p, c.nr.search_vacant.p, cnt_exc, cnt_inh);
    RL_LAUNCH_CHECK();
    // one scan over both halves: excitatory offsets, then inhibitory offsets
    // counted on from the last excitatory search
    const uint32_t* dtot = exclusive_scan_u32_async(S.counts.p, S.counts.p, 2 * (uint64_t)n, c.prim, st);
    uint32_t h[2] = { 0, 0 };
    RL_CUDA_TRY(cudaMemcpyAsync(&h[0], cnt_inh, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaMemcpyAsync(&h[1], dtot, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    const uint64_t num_exc = h[0];
    const uint64_t m = h[1];
    const uint64_t num_inh = m - num_exc;
    S.num_searches = m;
    S.num_exc = num_exc;
    if (m == 0) {
        S.num_requests = 0;  // nothing searches: no requests, nothing else to run
        return;
    }
    S.first_fail.ensure(n);
    S.tasks.ensure(2);
    S.req_count.ensure(n);
    S.req_off.ensure(n);
    k_fill_u32<<<blocks_for(n, 256), 256, 0, st>>>(S.first_fail.p, n, 0xFFFFFFFFu);
    RL_LAUNCH_CHECK();
    if (m > 0) {
        S.src.ensure(m);
        S.jj.ensure(m);
        S.target.ensure(m);
        k_search_fill<<<blocks_for(n, 256), 256, 0, st>>>(n, c.tree.morton.p, c.nr.enabled.p, c.nr.signal.p, c.nr.search_vacant.p, cnt_exc, cnt_inh,
                                                          0, S.src.p, S.jj.p);
        RL_LAUNCH_CHECK();
        // segments: one per (type, network) with searches, so a warp never mixes networks
        const uint32_t K = (uint32_t)c.nets.size();
        std::vector<uint32_t> starts(2 * (size_t)K, 0u);
        if (K > 1) {
            S.seg_starts.ensure(2 * (size_t)K);
            k_net_starts<<<blocks_for(K, 128), 128, 0, st>>>(K, c.d_nets.p, cnt_exc, cnt_inh, n, S.seg_starts.p);
            RL_LAUNCH_CHECK();
            RL_CUDA_TRY(cudaMemcpyAsync(starts.data(), S.seg_starts.p, 2 * (size_t)K * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            RL_CUDA_TRY(cudaStreamSynchronize(st));
            for (uint32_t k = 0; k < K; ++k) {
                starts[K + k] -= (uint32_t)num_exc;  // inhibitory starts relative to the first inhibitory search
            }
        }
        if (is_fp32(c)) {
            pack_tree_f32(c);
        }
        struct SearchLaunch {
            bool on = false;
            uint32_t warps = 0;
            uint32_t segs = 0;
        };
        SearchLaunch launches[2];
        SearchArgs args[2] = {};
        for (int t = 0; t < 2; ++t) {
            const uint64_t base = t == 0 ? 0 : num_exc;
            const uint64_t total = t == 0 ? num_exc : num_inh;
            std::vector<uint32_t> warp{ 0u }, net;
            std::vector<uint64_t> begin, endv;
            for (uint32_t k = 0; k < K; ++k) {
                const uint64_t b = starts[(size_t)t * K + k];
                const uint64_t e = k + 1 < K ? starts[(size_t)t * K + k + 1] : total;
                if (e > b) {
                    begin.push_back(base + b);
                    endv.push_back(base + e);
                    net.push_back(k);
                    warp.push_back(warp.back() + (uint32_t)((e - b + 31) / 32));
                }
            }
            if (net.empty()) {
                continue;
            }
            const uint32_t segs = (uint32_t)net.size();
            S.seg_warp[t].ensure(segs + 1);
            S.seg_begin[t].ensure(segs);
            S.seg_end[t].ensure(segs);
            S.seg_net[t].ensure(segs);
            RL_CUDA_TRY(cudaMemcpyAsync(S.seg_warp[t].p, warp.data(), (segs + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
            RL_CUDA_TRY(cudaMemcpyAsync(S.seg_begin[t].p, begin.data(), segs * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
            RL_CUDA_TRY(cudaMemcpyAsync(S.seg_end[t].p, endv.data(), segs * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
            RL_CUDA_TRY(cudaMemcpyAsync(S.seg_net[t].p, net.data(), segs * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
            const uint32_t warps = warp.back();
            SearchLaunch& L = launches[t];
            L.on = true;
            L.warps = warps;
            L.segs = segs;
            if (is_fp32(c)) {
                continue;
            }
            SearchArgs& A = args[t];
            A.rec = c.tree.rec[t].p;
            A.maxdim = c.tree.maxdim.p;
            A.tasks = S.tasks.p + t;
            A.first_key = c.tree.first_key.p;
            A.leaf_of = c.tree.leaf_of.p;
            A.meta = c.tree.meta.p;
            A.num_nodes = c.tree.num_nodes;
            A.px = c.nr.px.p;
            A.py = c.nr.py.p;
            A.pz = c.nr.pz.p;
            A.list_src = S.src.p;
            A.list_j = S.jj.p;
            A.seg_warp = S.seg_warp[t].p;
            A.seg_begin = S.seg_begin[t].p;
            A.seg_end = S.seg_end[t].p;
            A.seg_net = S.seg_net[t].p;
            A.num_segs = segs;
            A.nets = c.d_nets.p;
            A.target = S.target.p;
            A.mu = c.cfg.mu;
            A.step = step;
            A.err = c.err.p;
            A.touched = reinterpret_cast<unsigned long long*>(c.counters.p);
            A.kernel = c.kernel;
        }
        auto launch_all = [&](const SearchVariant& v) {
            if (v.packet == 0) {
                // one search per warp: both types in one launch
                const uint32_t w[2] = { launches[0].on ? launches[0].warps : 0u, launches[1].on ? launches[1].warps : 0u };
                if (is_fp32(c)) {
                    launch_search_wide_f32(c, w, launches[0].segs, launches[1].segs, step);
                } else {
                    launch_wide(c, args, w);
                }
                return;
            }
            for (int t = 0; t < 2; ++t) {
                if (!launches[t].on) {
                    continue;
                }
                if (v.hot > 0) {
                    RL_CUDA_TRY(cudaMemsetAsync(S.tasks.p + t, 0, sizeof(uint32_t), st));
                }
                if (is_fp32(c)) {
                    launch_search_f32(c, t, S.seg_warp[t].p, S.seg_begin[t].p, S.seg_end[t].p, S.seg_net[t].p, launches[t].segs, launches[t].warps, step, v,
                                      S.tasks.p + t);
                } else if (v.hot > 0) {
                    const HotKernel kern = fp64_hot_kernel(v);
                    const uint32_t hot = hot_nodes(c, v, sizeof(double4) + sizeof(uint4) + sizeof(double));
                    const size_t smem = (size_t)hot * (sizeof(double4) + sizeof(uint4) + sizeof(double));
                    RL_CUDA_TRY(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                    const unsigned blocks = std::min<unsigned>((unsigned)c.num_sms, (launches[t].warps + 31) / 32);
                    kern<<<blocks, 1024, smem, st>>>(args[t], hot);
                    RL_LAUNCH_CHECK();
                } else {
                    const SearchKernel kern = fp64_search_kernel(v);
                    RL_CHECK(kern != nullptr, RL_ERR_INVALID, "no such search variant");
                    const unsigned blocks = (launches[t].warps + v.warps - 1) / v.warps;
                    kern<<<blocks, v.warps * 32, 0, st>>>(args[t]);
                    RL_LAUNCH_CHECK();
                }
            }
        };
        if (c.tune.search_state != TUNE_OFF) {
            // automatic shapes: one per density class of the search list
            const int dc = search_density_class(c.n, m);
            auto known = c.tune.search_by_class.find(dc);
            if (known != c.tune.search_by_class.end()) {
                c.tune.search = known->second;
            } else {
                if (c.tune.force || !recall_search_tuning(c, dc)) {
                    tune_search(c, launch_all);
                    remember_search_tuning(c, dc);
                }
                c.tune.search_by_class[dc] = c.tune.search;
            }
            c.tune.search_state = TUNE_DONE;
        }
        {
            PhaseScope ps(c, PH_SEARCH_KERNEL);
            launch_all(c.tune.search);
        }
        k_first_fail<<<blocks_for(m, 256), 256, 0, st>>>(m, S.src.p, S.jj.p, S.target.p, S.first_fail.p);
        RL_LAUNCH_CHECK();
    }
    k_req_count<<<blocks_for(n, 256), 256, 0, st>>>(n, S.first_fail.p, c.nr.search_vacant.p, c.nr.enabled.p, S.req_count.p);
    RL_LAUNCH_CHECK();
    const uint64_t nreq = exclusive_scan_u32(S.req_count.p, S.req_off.p, n, c.prim, st);
    S.num_requests = nreq;
    S.req_tgt.ensure(nreq);
    S.req_src.ensure(nreq);
    S.req_j.ensure(nreq);
    S.req_sig.ensure(nreq);
    if (m > 0) {
        k_req_scatter<<<blocks_for(m, 256), 256, 0, st>>>(m, S.src.p, S.jj.p, S.target.p, S.first_fail.p, S.req_off.p, c.nr.signal.p, S.req_tgt.p,
                                                          S.req_src.p, S.req_j.p, S.req_sig.p);
        RL_LAUNCH_CHECK();
    }
    check_device_error(c, "barnes-hut search");
    c.stats.searches += m;
    c.stats.requests += nreq;
}

}  // namespace rl
