// Device-resident state of one network (one rl_ctx).
#pragma once

#include <map>

#include "rl_internal.cuh"

namespace rl {

// Octree levels encoded in the two key words (3 bits per level, 21 per word).
constexpr int kLevelsPerWord = 21;
constexpr int kMaxLevels = 2 * kLevelsPerWord;  // deepest leaf level + 1 representable

// Node topology word y: child mask (bits 0-7), leaf flag (bit 8), level (bits 16-31).
__host__ __device__ __forceinline__ uint32_t topo_mask(uint32_t y) { return y & 0xFFu; }
__host__ __device__ __forceinline__ bool topo_leaf(uint32_t y) { return (y >> 8) & 1u; }
__host__ __device__ __forceinline__ uint32_t topo_level(uint32_t y) { return y >> 16; }
// Escape link past the last node of a tree.
constexpr uint32_t kNoNode = 0xFFFFFFFFu;

#if defined(__CUDACC__)
// Read-only 32-byte record load through the non-coherent path.
__device__ __forceinline__ double4 ldg4(const double4* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
#endif

// The octree in breadth-first order (root first; within a level, Morton order).
struct Tree {
    uint32_t num_nodes = 0;
    uint32_t max_level = 0;
    bool root_is_leaf = false;
    uint32_t root_neuron = 0;
    DBuf<double4> rec[2];     // per dendrite type: centroid (x, y, z), w = count bits (low 32)
    DBuf<uint2> topo;         // x: first child (inner) or neuron id (leaf); y: see topo_*
    // what a walk reads of a node besides its record, in one 16-byte load:
    // topo.x, topo.y, the escape link (the node a depth-first walk visits after
    // this node's subtree; kNoNode after the last) and maxdim as FP32 bits
    DBuf<uint4> meta;
    DBuf<double> maxdim;      // BoundingBox::get_maximum_difference of the cell
    DBuf<double> bmin[3], bmax[3];
    DBuf<int32_t> parent;
    DBuf<uint32_t> first_key;  // Morton rank of the first neuron under the node
    DBuf<uint32_t> leaf_of;    // neuron -> node
    DBuf<uint32_t> morton;     // Morton rank -> neuron
    std::vector<uint32_t> level_off;  // host copy: nodes of level l are [level_off[l], level_off[l+1])
    DBuf<uint32_t> dirty;       // nodes to recompute in the running update
    DBuf<uint32_t> level_dirty; // per level: nodes of the level marked so far (entries of `work`)
    DBuf<uint32_t> work;        // marked nodes of level l at [level_off[l], level_off[l] + level_dirty[l])
    DBuf<uint32_t> level_lo;    // device copy of level_off
    DBuf<unsigned long long> level_runs;  // level launches the captured update ran (counted on the device)
    unsigned long long level_runs_seen = 0;  // of those, already added to the launch count
    DBuf<uint2> last_counts;    // per neuron: leaf counts (exc, inh) of the last update
    bool force_full = true;     // next update takes every leaf as changed
    bool recq_valid = false;    // fixed-point records match the FP64 records
    bool graph_keeps_q = false; // the captured update also maintains them
    cudaGraphExec_t update_graph = nullptr;  // the bottom-up update of this octree, captured once
    void drop_graph() {
        if (update_graph) {
            cudaGraphExecDestroy(update_graph);
            update_graph = nullptr;
        }
    }
    ~Tree() { drop_graph(); }
    // FP32 form: records (centroid, count bits in w); cell lengths are in meta
    DBuf<uint4> recq[2];  // centroid in fixed point (QFrame), w = count
};

struct Neurons {
    DBuf<double> px, py, pz;    // positions (SoA)
    DBuf<uint8_t> signal;       // 0 excitatory, 1 inhibitory
    DBuf<uint8_t> enabled;      // NeuronsExtraInfo disable flags (1 = enabled)
    DBuf<uint8_t> update;       // takes part in plasticity
    DBuf<double> x, u, calcium, target, input;
    DBuf<uint8_t> fired[2];     // double-buffered fired flags
    int cur = 0;                // fired[cur] holds the last step's flags
    DBuf<double> grown[3], delta[3];
    DBuf<uint32_t> connected[3], vacant[3];
    DBuf<uint32_t> search_vacant;  // vacant axons handed to the next search
    // FP32 form: authoritative membrane / growth state in FP32
    DBuf<float> x32, u32, input32, delta32[3];
    DBuf<float> target32;  // per-neuron target calcium (allocated when the targets differ)
};

// Synapse list: one entry per (target, source) synapse group with an integer
// weight (+1 per excitatory, -1 per inhibitory synapse), sorted by
// (target, source); in-CSR over targets and out-CSR (a permutation sorted by
// (source, target)) over sources.  New synapses of a plasticity update are
// appended to the new_* buffers and merged by rebuild_graph.
struct Graph {
    uint64_t num_edges = 0;
    DBuf<uint32_t> offsets;  // in-CSR, n + 1
    DBuf<uint32_t> tgt, src;
    DBuf<int32_t> weight;
    DBuf<uint32_t> out_off;   // out-CSR, n + 1
    DBuf<uint32_t> out_perm;  // edge indices in (source, target) order
    DBuf<uint32_t> new_tgt, new_src;
    DBuf<int32_t> new_w;
    uint64_t num_new = 0;
    bool zeros = false;  // deletions left entries of weight 0
    // Deletions since the zero entries were last dropped (at least the number
    // of zero entries).  A zero entry adds nothing to a pulled or pushed sum
    // and is no partner to a deletion, so the rebuild drops them only once
    // they may be an eighth of the list.
    uint64_t zero_bound = 0;
    // working arrays of the rebuild, kept between rebuilds (grown, never
    // shrunk): the merged lists before they swap with the ones above, merge
    // positions, and the keys and values of the new entries
    DBuf<uint32_t> m_tgt, m_src, m_out, m_pos, m_newpos, m_nv;
    DBuf<int32_t> m_w;
    DBuf<uint64_t> m_nk;
};

struct Search {
    DBuf<uint32_t> counts;   // per Morton rank, per type
    DBuf<uint32_t> src, jj;  // search list: exc segment then inh segment
    DBuf<int32_t> target;    // result per search (-1 failure)
    DBuf<uint32_t> first_fail;   // per neuron: smallest failing j
    DBuf<uint32_t> req_count;    // per neuron: valid requests
    DBuf<uint32_t> req_off;      // per neuron: output offset
    DBuf<uint32_t> req_tgt, req_src, req_j, req_sig;  // requests in (source, j) order
    DBuf<uint32_t> vac_before;   // connector: vacant dendrite counts before it (exc, then inh)
    DBuf<uint32_t> accept_pos;   // connector: output position of each accepted request
    DBuf<uint32_t> seg_starts;
    DBuf<uint32_t> tasks;    // persistent search form: task counter per signal type
    DBuf<uint32_t> seg_warp[2], seg_net[2];
    DBuf<uint64_t> seg_begin[2], seg_end[2];
    // one-search-per-warp form: walk entries of every warp slot
    DBuf<uint32_t> w_node, w_info, w_child, w_cnt, w_pos, w_ord_node, w_overflow;
    DBuf<double> w_w, w_ord_w;
    uint64_t num_searches = 0;
    uint64_t num_exc = 0;
    uint64_t num_requests = 0;
    // connector
    DBuf<uint64_t> ckey;
    DBuf<uint32_t> cidx;
    DBuf<uint32_t> gkey;
    DBuf<uint32_t> accepted;
    DBuf<uint32_t> rank;
    DBuf<uint32_t> flags;
};

// Per-phase device time, measured with CUDA events on the context's stream.
enum Phase : int {
    PH_ACTIVITY_KERNEL = RL_PHASE_ACTIVITY_KERNEL,
    PH_COMMIT = RL_PHASE_COMMIT,
    PH_TREE_UPDATE = RL_PHASE_TREE_UPDATE,
    PH_SEARCH_KERNEL = RL_PHASE_SEARCH_KERNEL,
    PH_SEARCH = RL_PHASE_SEARCH,
    PH_CONNECTOR = RL_PHASE_CONNECTOR,
    PH_GRAPH = RL_PHASE_GRAPH,
    PH_COUNT = RL_NUM_PHASES,
};

struct PendingTimer {
    cudaEvent_t start;
    cudaEvent_t end;
    uint32_t weight;  // kernel launches the interval stands for
};

struct PhaseTimer {
    bool on = false;
    std::vector<cudaEvent_t> free_events;
    std::vector<PendingTimer> pending[PH_COUNT];
    double ms[PH_COUNT] = {};
    uint64_t count[PH_COUNT] = {};
};

// One network of a context.  A context holds one or more networks in one set
// of arrays: network k owns neurons [first, first + count); the octree is a
// forest whose root of network k is node k; every random draw of a neuron is
// keyed on the network's seed and the neuron's index inside its network, so a
// network evolves exactly as it would alone.
// Fixed-point frame of a network for the FP32 search: a coordinate x is stored
// as the integer round((x - origin) / quantum) in [0, 2^30], origin = the
// network's box_min, quantum = the smallest power of two that maps the box's
// longest edge into 2^30 steps.  The difference of two stored coordinates
// converts to micrometres exactly up to the float rounding of the difference
// itself (distances keep their relative precision however far from the origin
// the cells lie), and each network's frame depends on its own box only.
struct QFrame {
    double origin[3] = { 0.0, 0.0, 0.0 };
    double inv_quantum = 1.0;  // 1 / quantum
    float quantum = 1.0f;
};

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t quantize(double x, double origin, double inv_quantum) {
    const double q = (x - origin) * inv_quantum;
    return q > 0.0 ? (uint32_t)__double2uint_rn(q) : 0u;  // also 0 for the NaN centroid of an empty cell
}

__device__ __forceinline__ uint4 quantize_record(const double4& r, const QFrame& f) {
    return make_uint4(quantize(r.x, f.origin[0], f.inv_quantum), quantize(r.y, f.origin[1], f.inv_quantum), quantize(r.z, f.origin[2], f.inv_quantum),
                      (uint32_t)__double_as_longlong(r.w));
}
#endif

struct NetInfo {
    uint64_t seed;
    uint32_t first;
    uint32_t count;
    double theta;
    double scale;  // -1 / sigma^2
    double sigma;
    double nu[3];
    double box_min[3];
    double box_max[3];
    float theta32;
    float inv_sigma2_32;
    float nu32[3];
    uint32_t root_leaf;  // the network has a single neuron
    QFrame frame;
};

// Rows of the spike history of one launch per step (row k % kHistSteps holds
// the flags of the block's step k); calcium and growth are computed per chunk
// of kGrowthChunk steps, the chunk before the last one beside the next
// chunk's steps (their rows differ).  A row holds one byte per neuron and is
// padded to a multiple of 16 bytes, so that a thread's vector store of its V
// flags (V = 1, 2, 4 from a multiple of V) is aligned in every row.
constexpr uint32_t kHistSteps = 128;
constexpr uint32_t kGrowthChunk = 64;
inline size_t hist_stride(uint32_t n) {
    return ((size_t)n + 15) / 16 * 16;
}

// A block of at most kNetBlock neurons of one network: [first, first + count).
constexpr uint32_t kNetBlock = 128;
struct NetBlock {
    uint32_t first;
    uint16_t net;
    uint16_t count;
};

// Probability kernel of the search: `type` is an RL_KERNEL_* value; a and b
// are the kernel's constants (gamma: 1/(Gamma(k) theta^k) and -1/theta;
// Weibull: b k and b); k_minus_1 the exponent of d; the linear cut-off.
struct KernelParams {
    int type = RL_KERNEL_GAUSSIAN;
    int cutoff_inf = 1;
    double k_minus_1 = 0.0;
    double a = 0.0;
    double b = 0.0;
    double cutoff = 0.0;
};

struct Ctx;
// Records an event pair around a scope when profiling is on.
struct PhaseScope {
    Ctx* c;
    int phase;
    cudaEvent_t end = nullptr;
    PhaseScope(Ctx& ctx, int ph, uint32_t weight = 1);
    ~PhaseScope();
};

// Per-block values of the activity kernels, read from device memory so that a
// captured 100-step graph stays valid when the synapse graph is rebuilt.
struct ActDesc {
    uint32_t base_step;
    uint32_t has_edges;
    const uint32_t* off;  // in-CSR
    const uint32_t* src;
    const int32_t* w;
    // Steps of the block.  Its first step pulls each neuron's synaptic sum
    // over the in-CSR; a neuron whose spike flag is set at a step before the
    // block's last adds its out-edges' weights (out-CSR: out_off, out_perm into
    // tgt and w) to its targets' sums of the next step, which that step reads
    // and clears.  Integer sums: the same values in any order.
    uint32_t block_len;
    const uint32_t* out_off;
    const uint32_t* out_perm;
    const uint32_t* tgt;
};

// Launch shape of the Barnes-Hut search kernels.
struct SearchVariant {
    int warps = 2;    // warps per block
    int packet = 32;  // lanes (sources) that walk the descent from the root together
    int cap = 1;      // 1: registers capped at 64 for more resident warps
    int hot = 0;      // > 0: persistent form, one block of 32 warps per SM with up
                      // to `hot` top octree nodes in shared memory
};


// Launch shape of the activity kernel.
struct ActVariant {
    int block = 256;     // threads per block
    int persistent = 0;  // 1: one resident wave of blocks looping over the neurons
    int vec = 1;         // neurons per thread (vector loads and stores; FP32 form)
};

enum : int { TUNE_OFF = 0, TUNE_REQUESTED = 1, TUNE_DONE = 2 };

// Launch shapes in use and the tuner's state.
struct Tuning {
    SearchVariant search;
    ActVariant act;
    int search_state = TUNE_OFF;
    int act_state = TUNE_OFF;
    bool force = false;            // time again even when the process has a result for this shape
    // automatic search shapes per density class of the search list (search_density_class)
    std::map<int, SearchVariant> search_by_class;
    std::vector<float> search_ms;  // per variant tried, in search_variants() order
    std::vector<float> act_ms;     // per variant tried, in act_variants() order
};

const std::vector<SearchVariant>& search_variants();
bool search_variant_applies(const Ctx& c, const SearchVariant& v);
struct WideSlot;
uint32_t wide_cap(const Ctx& c);
WideSlot wide_scratch(Ctx& c, uint32_t slots, uint32_t cap);
// one-search-per-warp form: walk entries per warp, warps per SM, smallest network
constexpr uint32_t kWideCap = 6144;
constexpr uint32_t kWideWarpsPerSM = 16;
constexpr uint32_t kWideMinNeurons = 65536;
uint32_t hot_nodes(const Ctx& c, const SearchVariant& v, size_t node_bytes);
const std::vector<ActVariant>& act_variants();

struct Ctx {
    rl_config cfg{};
    uint32_t n = 0;
    int device = 0;
    int num_sms = 148;          // streaming multiprocessors of the device
    int smem_optin = 232448;    // shared memory a block may opt in to (bytes)
    cudaStream_t stream = nullptr;      // stream all work is issued on
    cudaStream_t own_stream = nullptr;  // the context's own stream
    PhaseTimer timer;
    DBuf<ActDesc> act_desc;
    // synaptic sums pushed by the spikes of a step, by step parity (FP64 form:
    // syn_in64, FP32 form: syn_in32); zero at every block boundary
    DBuf<long long> syn_in64[2];
    DBuf<int32_t> syn_in32[2];
    // one launch per step: the spike flags of up to kHistSteps steps (row k:
    // step k of the chunk, one byte per neuron), from which calcium and the
    // growth deltas of the chunk are computed at its end
    DBuf<uint8_t> spike_hist;
    cudaGraphExec_t act_graph[2] = { nullptr, nullptr };  // per fired-buffer parity
    uint32_t act_graph_len = 0;
    uint32_t act_block_len = 0;  // steps of the activity block being issued: only its last step stores the input
    bool use_graphs = true;
    bool step_fusion = true;  // blocks of steps of a network without synapses in one launch
    bool capturing = false;
    std::vector<NetInfo> nets;  // host copy
    DBuf<NetInfo> d_nets;
    DBuf<uint16_t> net_of;      // network of each neuron
    // The neurons of a batched context in blocks of kNetBlock that never span
    // two networks (a network's last block may be short), for the kernels that
    // run a block of steps per launch: a thread block holds one network, so its
    // seed is the same in every thread and lane pairs hold neuron pairs.
    DBuf<NetBlock> net_blocks;
    uint32_t num_net_blocks = 0;
    bool multi() const { return nets.size() > 1; }
    std::string last_error;
    bool positions_set = false;
    Tree tree;
    Neurons nr;
    Graph graph;
    Search search;
    PrimScratch prim;
    DBuf<uint32_t> to_delete;  // per neuron, bound elements to delete in the current pass
    DBuf<uint32_t> err;       // device error word
    DBuf<uint64_t> counters;  // device counters
    DBuf<unsigned long long> commit_cnt;  // bound elements to delete per element type of an update, then vacant axons
    unsigned long long* h_commit = nullptr;  // pinned host copy of commit_cnt (read without blocking the enqueue)
    bool target_uniform = true;  // every neuron has cfg.target_calcium as its target
    // Host transfers that overlap the work on the context's stream: uploads
    // of enabled flags and snapshots of calcium and fired flags go through
    // device staging buffers and copy streams of their own (one per
    // direction, so that an upload never queues behind a snapshot).
    cudaStream_t copy_stream = nullptr;    // snapshots (device -> host)
    cudaStream_t upload_stream = nullptr;  // enabled flags (host -> device)
    // calcium and growth of a chunk of one launch per step run here while the
    // context's stream runs the next chunk's steps (fork and join events)
    cudaStream_t growth_stream = nullptr;
    cudaEvent_t growth_fork = nullptr;
    cudaEvent_t growth_join = nullptr;
    DBuf<uint8_t> enabled_stage;
    cudaEvent_t upload_done = nullptr;   // the last upload reached the staging buffer
    cudaEvent_t stage_free = nullptr;    // the context's stream has consumed it
    bool stage_used = false;
    struct SnapSlot {
        DBuf<double> calcium;
        DBuf<uint8_t> fired;
        cudaEvent_t staged = nullptr;  // state copied into the slot (context's stream)
        cudaEvent_t landed = nullptr;  // slot copied to the host (copy stream)
        double* host_calcium = nullptr;
        uint8_t* host_fired = nullptr;
        bool pending = false;  // not waited for yet
        bool issued = false;   // the copy to the host is on the copy stream
    };
    SnapSlot snap[2];
    int snap_next = 0;
    // order between the context's stream and a caller stream handed to
    // rl_prepare_update_connectivity_noalloc (created by its first call on this context)
    cudaEvent_t noalloc_before = nullptr;
    cudaEvent_t noalloc_after = nullptr;
    bool no_searches = false;             // the update's commit left no vacant axon: the search has nothing to do
    bool deleted_last = false;            // the last plasticity update deleted synapses
    rl_stats stats{};
    uint64_t launches = 0;     // kernels launched for this context
    int64_t device_bytes = 0;  // device memory held now
    int64_t device_peak = 0;   // and at most so far
    bool counted = false;      // counted among the device's live contexts
    Tuning tune;
    KernelParams kernel;
};

// Tuning results shared by the contexts of a process, keyed by precision,
// batched or not, and the neuron count's power of two.
void remember_search_tuning(const Ctx& c, int density_class);
bool recall_search_tuning(Ctx& c, int density_class);
// Density class of a search list of m searches over n neurons: 0 when more
// than a quarter of the neurons search, 1 above 1/32, 2 above 1/256, else 3.
inline int search_density_class(uint64_t n, uint64_t m) {
    if (4 * m > n) return 0;
    if (32 * m > n) return 1;
    if (256 * m > n) return 2;
    return 3;
}
void remember_act_tuning(const Ctx& c);
bool recall_act_tuning(Ctx& c);
// Releases the captured activity intervals (they are captured again on use).
void drop_activity_graphs(Ctx& c);
// The pushed synaptic sums (ActDesc): allocated (zero) before the first block
// with synapses; cleared after steps that are undone.
void ensure_syn_in(Ctx& c);
void clear_syn_in(Ctx& c);
// The spike history of one launch per step (allocated before the first such
// block), and calcium and growth of the last m steps from it.
void ensure_spike_hist(Ctx& c);
void launch_calcium_growth(Ctx& c, uint32_t row0, uint32_t m, cudaStream_t st);
void launch_calcium_growth64(Ctx& c, uint32_t row0, uint32_t m, cudaStream_t st);
void launch_calcium_growth32(Ctx& c, uint32_t row0, uint32_t m, cudaStream_t st);
// Blocks of an activity launch of variant v of `kernel`.
unsigned act_grid(Ctx& c, const ActVariant& v, const void* kernel);

// octree.cu
void build_octree(Ctx& c, const double* h_xyz);
void update_tree(Ctx& c);  // leaf counts from nr.vacant[1..2] and nr.update, then the reduction
// Leaf update + reduction with caller-given device vacancy arrays and an
// external arrival-counter buffer of at least tree.num_nodes words.
void launch_tree_update_scratch(Ctx& c, const uint32_t* d_vac_exc, const uint32_t* d_vac_inh, const uint8_t* d_update, uint32_t* arrive,
                                cudaStream_t st);
void dump_tree(Ctx& c, int32_t* level, int32_t* neuron, uint8_t* child_mask, int32_t* first_child, double* bmin, double* bmax, uint32_t* cnt_exc,
               uint32_t* cnt_inh, double* pos_exc, double* pos_inh);

// bh_search.cu
void run_search(Ctx& c, uint32_t step);  // fills search.req_* (requests in (source, j) order)

// connector.cu
// accepts requests, updates elements, appends new edges; bind_axons false:
// the target side only (the sources' axons are bound by bind_axons_host)
uint64_t run_connector(Ctx& c, uint32_t step, bool bind_axons = true);
void bind_axons_host(Ctx& c, uint64_t m, const uint32_t* src);  // one vacant axon per listed source
void rebuild_graph(Ctx& c);                     // merge new edges into the CSR
uint64_t run_deletion(Ctx& c, uint32_t step, int type);  // delete to_delete[] synapses per neuron for one element type
void add_edges_host(Ctx& c, uint64_t m, const uint32_t* t, const uint32_t* s, const int32_t* w);

// fp32.cu (precision form)
bool is_fp32(const Ctx& c);
void alloc_fp32(Ctx& c);
void f32_from_f64(Ctx& c);  // state arrays FP64 -> FP32 (after a host upload)
void target_f32_from_f64(Ctx& c);  // per-neuron target calcium FP64 -> FP32
void f64_from_f32(Ctx& c);  // state arrays FP32 -> FP64 (before a host download)
void launch_activity_f32(Ctx& c, uint32_t k, const uint8_t* fired_prev, uint8_t* fired_cur, const ActVariant& v);
void launch_activity_fp64(Ctx& c, uint32_t k, const uint8_t* fired_prev, uint8_t* fired_cur, const ActVariant& v);
// A block of nsteps steps in one launch; only for a network without synapses.
void launch_activity_f32_steps(Ctx& c, uint32_t nsteps);
void launch_activity_fp64_steps(Ctx& c, uint32_t nsteps);
uint64_t run_commit_f32(Ctx& c, int type);
void pack_tree_f32(Ctx& c);
void launch_search_f32(Ctx& c, int type, const uint32_t* seg_warp, const uint64_t* seg_begin, const uint64_t* seg_end, const uint32_t* seg_net,
                       uint32_t num_segs, uint32_t warps, uint32_t step, const SearchVariant& v, uint32_t* tasks);
// One search per warp over both signal types' lists at once.
void launch_search_wide_f32(Ctx& c, const uint32_t (&warps)[2], uint32_t segs0, uint32_t segs1, uint32_t step);
void candidate_weights(Ctx& c, uint32_t source, int precision, std::vector<uint32_t>& nodes, std::vector<double>& w);

// activity.cu
// Activity steps first..first+nsteps-1 (one fused kernel per step; a full
// plasticity interval runs as a captured CUDA graph).
void run_activity_block(Ctx& c, uint32_t first_step, uint32_t nsteps);
// Frees a context and everything it holds (after its stream has drained).
void discard(Ctx* c);
void ensure_copy_stream(Ctx& c);
// Puts the host copies of staged snapshots on the copy stream.  Called after
// the next work has been queued on the context's stream, so that the copies
// overlap it (and do not hold up an upload issued in between).
void issue_snapshots(Ctx& c);
uint64_t run_commit(Ctx& c, int type);
// Commit of `type` that does nothing when an earlier type of the same update
// (its count in commit_cnt) left bound elements to delete; counts into
// commit_cnt[type].  The three are launched back to back and read once.
void launch_commit_guarded(Ctx& c, int type);
// All three commits and the vacant-axon count in one cooperative launch, with
// the same skip rule; false when a cooperative launch is not available.
bool launch_commit_all(Ctx& c);
// Adds the vacant axons of the enabled neurons to *out.
void launch_vacant_axon_count(Ctx& c, unsigned long long* out);
void launch_commit_f32(Ctx& c, int type, unsigned long long* total, const unsigned long long* guard, int guard_n);  // commit one element type; to_delete[] per neuron, returns the sum

void check_device_error(Ctx& c, const char* phase);

}  // namespace rl
