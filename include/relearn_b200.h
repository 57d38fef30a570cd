/*
 * relearn_b200 — C ABI of the B200 structural-plasticity hot path.
 *
 * One context holds one network on one GPU: neuron positions and signal
 * types, the linear octree over them, the Izhikevich / calcium / synaptic
 * element state, the synapse list and the scratch the kernels need.  All
 * arrays crossing this boundary are caller-owned HOST buffers with plain
 * pointers and sizes; the context owns all device memory.  No C++ types and
 * no exceptions cross the boundary: every entry point returns an rl_status,
 * and rl_last_error() gives a message for the last failing call.
 *
 * Threading: a context is used by one host thread at a time (not
 * re-entrant); several contexts may share a device.
 *
 * The entry points replace the following reference interfaces (paths relative
 * to relearn/source in tuda-hpclab/relearn):
 *   Algorithm (algorithm/Algorithm.h:48-197) selected by --algorithm barnes-hut
 *     init(n)                        -> rl_set_positions
 *     prepare_update_connectivity    -> rl_prepare_update_connectivity
 *     update_connectivity(n)         -> rl_update_connectivity
 *   NeuronModel (neurons/models/NeuronModelBase.h) selected by
 *   --neuron-model izhikevich, with CalciumCalculator and SynapticElements
 *   as driven by Neurons (neurons/Neurons.cpp:351-384)
 *     update_electrical_activity + update_calcium + update_number_elements
 *                                    -> rl_activity_block
 *   Neurons::update_connectivity (neurons/Neurons.cpp:588-608)
 *                                    -> rl_plasticity_update
 *   Simulation::simulate (sim/Simulation.cpp:388-480) -> rl_simulate
 */
#ifndef RELEARN_B200_H
#define RELEARN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RL_ABI_VERSION 4

#if defined(__GNUC__)
#define RL_API __attribute__((visibility("default")))
#else
#define RL_API
#endif

typedef enum rl_status {
    RL_OK = 0,
    RL_ERR_INVALID = 1,   /* bad argument, size or state (RelearnException::check) */
    RL_ERR_OOM = 2,       /* device allocation failed */
    RL_ERR_DEVICE = 3,    /* CUDA runtime error, or no usable device */
    RL_ERR_TIMEOUT = 4,   /* a bounded device wait ran out */
    RL_ERR_OVERFLOW = 5,  /* a fixed-capacity device structure overflowed */
    RL_ERR_UNSUPPORTED = 6 /* configuration outside what this build implements */
} rl_status;

/* Element types, in the reference's order (SynapticElementType). */
enum { RL_AXON = 0, RL_DENDRITE_EXC = 1, RL_DENDRITE_INH = 2 };

/* Signal types (SignalType): 0 excitatory, 1 inhibitory. */
enum { RL_EXCITATORY = 0, RL_INHIBITORY = 1 };

/* Parameters of one network.  Defaults of the reference are given in
 * brackets; rl_config_default() fills them. */
typedef struct rl_config {
    uint32_t num_neurons;
    uint32_t plasticity_interval; /* [100] Config::plasticity_update_step */
    uint32_t h_model;             /* [10] Euler substeps of the neuron model */
    uint32_t h_calcium;           /* [10] Euler substeps of the calcium */
    uint64_t seed;                /* key of the Philox stream */
    double box_min[3];            /* simulation box (root cell) */
    double box_max[3];
    double theta;                 /* [0.3] Barnes-Hut acceptance criterion, (0, 0.5] */
    double sigma;                 /* [750] Gaussian kernel sigma (um) */
    double mu;                    /* [0] Gaussian kernel offset */
    double iz_a, iz_b, iz_c, iz_d, iz_v_spike, iz_k1, iz_k2, iz_k3;
    double beta;                  /* [0.001] calcium increase per spike */
    double tau_c;                 /* [10000] calcium decay time */
    double target_calcium;        /* [0.7] */
    double initial_calcium;       /* [0] */
    double growth_rate[3];        /* [1e-4] nu per element type */
    double min_calcium[3];        /* eta per element type [0.4, 0.1, 0.0] */
    double retract_ratio[3];      /* [0] vacant retract ratio per element type */
    double conductance;           /* synaptic_equally_weighted conductance */
    double noise_mean;            /* normal background input mean */
    double noise_stddev;          /* normal background input stddev */
    int32_t device;               /* CUDA device ordinal */
    int32_t precision;            /* RL_PRECISION_FP64 (drop-in, bit-exact) or RL_PRECISION_FP32 */
    int32_t kernel_type;          /* [RL_KERNEL_GAUSSIAN] probability kernel (--kernel-type) */
    int32_t reserved;
    double kernel_k;              /* [1] shape of the gamma / Weibull kernel (--gamma-k, --weibull-k) */
    double kernel_scale;          /* [1] gamma theta / Weibull b (--gamma-theta, --weibull-b) */
    double linear_cutoff;         /* [+inf] cut-off of the linear kernel (--linear-cutoff) */
    int32_t neuron_model;         /* [RL_MODEL_IZHIKEVICH] --neuron-model */
    uint32_t poisson_refractory;  /* [4] Poisson: steps without spiking after a spike */
    double poisson_x0;            /* [0.05] Poisson: resting potential */
    double poisson_tau_x;         /* [5] Poisson: decay of the potential */
    double fhn_a, fhn_b, fhn_phi; /* [0.7, 0.8, 0.08] FitzHugh-Nagumo */
    double fhn_init_x, fhn_init_w;  /* [-1.2, -0.6] FitzHugh-Nagumo initial x and w */
    double aeif_C, aeif_g_L, aeif_E_L, aeif_V_T, aeif_d_T;  /* [281, 30, -70.6, -50.4, 2] AEIF */
    double aeif_tau_w, aeif_a, aeif_b, aeif_V_spike;          /* [144, 4, 0.0805, 20] AEIF */
} rl_config;

/* Neuron models (--neuron-model; the classes under neurons/models), defaults of their
 * Parameters.h.  The second state variable (rl_get_neurons' u) is the
 * Izhikevich recovery u, the FitzHugh-Nagumo and AEIF adaptation w, or the
 * Poisson model's refractory steps left.  Both precision forms run all four. */
enum { RL_MODEL_IZHIKEVICH = 0, RL_MODEL_POISSON = 1, RL_MODEL_FITZHUGH_NAGUMO = 2, RL_MODEL_AEIF = 3 };

/* Probability kernels of the search (algorithm/Kernel/KernelType.h): the
 * attraction of a cell at distance d, times its vacant count, is
 *   Gaussian: exp((d - mu)^2 * (-1 / sigma^2))              (Gaussian.h:62-68)
 *   gamma:    1 / (Gamma(k) theta^k) * d^(k-1) * exp(-d / theta) (Gamma.h)
 *   linear:   1 - d / cutoff for d <= cutoff, else 0; 1 for an infinite cutoff (Linear.h)
 *   Weibull:  b k * d^(k-1) * exp(-b d^(k-1) d)             (Weibull.h)
 * sigma is per network in a batched context; the other parameters are shared. */
enum { RL_KERNEL_GAUSSIAN = 0, RL_KERNEL_GAMMA = 1, RL_KERNEL_LINEAR = 2, RL_KERNEL_WEIBULL = 3 };

/* Precision forms.  FP64: the drop-in; every FP64 operation in the reference's
 * order, bit-exact against the oracle.  FP32: membrane, input, growth and
 * attraction arithmetic in FP32 with Kahan-compensated attraction sums; calcium
 * integrated in FP64; octree centroids reduced in FP64 and read by the search
 * in 32-bit fixed point. */
enum { RL_PRECISION_FP64 = 0, RL_PRECISION_FP32 = 1 };

/* One synapse creation request (SynapseCreationRequest,
 * neurons/helper/SynapseCreationRequests.h) plus the vacant-axon index j. */
typedef struct rl_request {
    uint32_t target;
    uint32_t source;
    uint32_t j;
    uint32_t signal;
} rl_request;

/* One synapse: target (dendrite side), source (axon side), weight +1/-1. */
typedef struct rl_synapse {
    uint32_t target;
    uint32_t source;
    int32_t weight;
    uint32_t reserved;
} rl_synapse;

/* Counters accumulated by a context. */
typedef struct rl_stats {
    uint64_t searches;           /* single-element Barnes-Hut searches run */
    uint64_t requests;           /* requests emitted by the searches */
    uint64_t synapses_created;   /* requests accepted by the connector */
    uint64_t bound_to_delete;    /* bound elements the commits asked to delete */
    uint64_t synapses_deleted;   /* synapses removed by the deletion passes */
    uint64_t activity_steps;     /* activity steps run */
    uint64_t plasticity_updates; /* plasticity updates run */
    uint64_t gpu_launches;       /* kernels this library launched */
    uint64_t num_nodes;          /* octree nodes */
    uint32_t max_level;          /* deepest octree level */
    uint32_t reserved;
    uint64_t nodes_touched;      /* acceptance tests the searches ran (nodes visited, as the reference's walk visits them) */
} rl_stats;

/* Phases timed with CUDA events when profiling is on (rl_set_profiling). */
enum {
    RL_PHASE_ACTIVITY_KERNEL = 0, /* the fused activity kernel */
    RL_PHASE_COMMIT = 1,          /* commit of the synaptic elements */
    RL_PHASE_TREE_UPDATE = 2,     /* leaf update + bottom-up reduction */
    RL_PHASE_SEARCH_KERNEL = 3,   /* the Barnes-Hut search kernels */
    RL_PHASE_SEARCH = 4,          /* search including list building and request compaction */
    RL_PHASE_CONNECTOR = 5,       /* connector */
    RL_PHASE_GRAPH = 6,           /* synapse graph rebuild */
    RL_NUM_PHASES = 7
};

/* One network of an ensemble (rl_ensemble_create): its own size, seed, cube,
 * acceptance criterion, kernel width and growth rates; everything else comes
 * from the ensemble's base rl_config. */
typedef struct rl_network {
    uint32_t num_neurons;
    uint32_t reserved;
    uint64_t seed;
    double box_min[3];
    double box_max[3];
    double theta;
    double sigma;
    double growth_rate[3];
} rl_network;

/* Fill *cfg with the reference defaults for n neurons in the given cube. */
RL_API void rl_config_default(rl_config* cfg, uint32_t num_neurons, double side);

/* Create a context for cfg->num_neurons neurons on cfg->device. */
RL_API rl_status rl_ctx_create(const rl_config* cfg, void** ctx);

/* Create one context holding `num_networks` independent networks (the batched
 * form): their neurons are concatenated in network order in every array of
 * the other entry points, each activity step is one launch over all networks,
 * and each network evolves exactly as it would in a context of its own with
 * the same parameters.  base->num_neurons is ignored. */
RL_API rl_status rl_ensemble_create(const rl_config* base, const rl_network* networks, uint32_t num_networks, void** ctx);
RL_API rl_status rl_ctx_destroy(void* ctx);
RL_API const char* rl_last_error(void* ctx);
RL_API const char* rl_status_string(rl_status s);
RL_API int32_t rl_abi_version(void);

/* Algorithm::init / OctreeAlgorithm::init (algorithm/Internal/OctreeAlgorithm.h:58-67):
 * positions (N x 3 doubles, row-major) and signal types (N bytes); builds the
 * octree on the device (Morton keys, radix sort, PR-octree).  Positions must
 * lie in the configured box and be pairwise distinct. */
RL_API rl_status rl_set_positions(void* ctx, const double* xyz, const uint8_t* signal);

/* Octree size after rl_set_positions. */
RL_API rl_status rl_tree_info(void* ctx, uint64_t* num_nodes, uint32_t* max_level);

/* Canonical dump of the octree in breadth-first order (root, then level by
 * level, children in octant order): level, neuron id (-1 for inner nodes),
 * child mask, index of the first child (-1 for leaves), cell box (x3),
 * vacant dendrite counts and their positions (x3, NaN when absent).
 * Every pointer may be NULL to skip that field. */
RL_API rl_status rl_dump_tree(void* ctx, int32_t* level, int32_t* neuron, uint8_t* child_mask, int32_t* first_child, double* bmin, double* bmax,
                       uint32_t* cnt_exc, uint32_t* cnt_inh, double* pos_exc, double* pos_inh);

/* Algorithm::prepare_update_connectivity (algorithm/Algorithm.h) ->
 * OctreeAlgorithm::update_tree (algorithm/Internal/OctreeAlgorithm.h:100-238):
 * stores the vacant axon counts for the next search, writes the vacant
 * dendrite counts into the leaves and reduces counts and centroids bottom-up.
 * `update` (nullable) marks neurons that take part in plasticity. */
RL_API rl_status rl_prepare_update_connectivity(void* ctx, const uint8_t* signal, const uint32_t* vacant_axons, const uint32_t* vacant_exc,
                                         const uint32_t* vacant_inh, const uint8_t* update);

/* The search half of Algorithm::update_connectivity
 * (BarnesHut::find_target_neurons, algorithm/BarnesHutInternal/BarnesHut.cpp:36-94):
 * one Barnes-Hut search per vacant axon element; returns the requests in
 * (source, j) order.  *count receives the number of requests; at most
 * `capacity` are copied to out (out may be NULL). */
RL_API rl_status rl_find_targets(void* ctx, uint32_t step, rl_request* out, uint64_t capacity, uint64_t* count);

/* Algorithm::update_connectivity (algorithm/Internal/ExchangingAlgorithm.h:58-87):
 * search, then the connector (algorithm/Connector.cpp:33-197).  Connects
 * elements in the context's own element state, appends the synapses to the
 * context's synapse list and returns them (accepted requests, in connector
 * order).  *created receives their number. */
RL_API rl_status rl_update_connectivity(void* ctx, uint32_t step, rl_synapse* out, uint64_t capacity, uint64_t* created);

/* Synaptic-element state per type (RL_AXON, RL_DENDRITE_EXC, RL_DENDRITE_INH):
 * grown (double), delta since the last commit (double), connected and vacant
 * counts (uint32).  NULL pointers are skipped. */
/* ForwardConnector::process_requests + process_responses
 * (algorithm/Connector.cpp:33-197) over a caller-given list of `count`
 * requests, the form the reference's connector tests drive: requests are
 * processed in the keyed random order of rl_update_connectivity; a request
 * whose target is its source fails, and so does one whose target has no
 * vacant dendrite of the request's type left; an accepted request binds one
 * vacant dendrite of the target and one vacant axon of the source and adds a
 * synapse of weight +1 (excitatory) or -1 (inhibitory).  A source needs a
 * vacant axon per accepted request (else RL_ERR_DEVICE).  `accepted` (may be
 * NULL) receives one flag per request in the caller's order; *created the
 * number of synapses formed. */
RL_API rl_status rl_connect(void* ctx, uint32_t step, const rl_request* requests, uint64_t count, uint8_t* accepted, uint64_t* created);

/* The two halves of the connector for a network split over ranks, each rank
 * a context over every neuron's position (the octree is replicated) that owns
 * a share of the neurons; neuron ids are global, so every draw is the one a
 * single context makes.
 *
 * ForwardConnector::process_requests (algorithm/Connector.cpp:33-117) on the
 * rank that owns the requests' targets: the requests of all ranks, processed
 * in the keyed random order of rl_connect; a request whose target is its
 * source fails, and so does one whose target has no vacant dendrite of the
 * request's type left; an accepted request binds one vacant dendrite of the
 * target and adds the synapse to the context's synapse list.  The sources'
 * axons are not touched.  `accepted` (may be NULL) receives one flag per
 * request in the caller's order (the responses); *created the number of
 * synapses formed. */
RL_API rl_status rl_process_requests(void* ctx, uint32_t step, const rl_request* requests, uint64_t count, uint8_t* accepted, uint64_t* created);

/* ForwardConnector::process_responses (algorithm/Connector.cpp:119-197) on the
 * rank that owns the requests' sources: one vacant axon of the source is bound
 * per accepted request (a source without one gives RL_ERR_DEVICE, the
 * reference's exception); requests with `append` set (may be NULL: none) add
 * their synapse to the context's synapse list — those whose target lives on
 * another rank, whose synapse rl_process_requests did not add here.
 * *bound (may be NULL) receives the number of axons bound. */
RL_API rl_status rl_process_responses(void* ctx, const rl_request* requests, const uint8_t* accepted, const uint8_t* append, uint64_t count,
                                      uint64_t* bound);

RL_API rl_status rl_set_elements(void* ctx, int type, const double* grown, const double* delta, const uint32_t* connected, const uint32_t* vacant);
RL_API rl_status rl_get_elements(void* ctx, int type, double* grown, double* delta, uint32_t* connected, uint32_t* vacant);

/* Neuron state: membrane potential x, recovery u, calcium, fired flag of the
 * last step, and the input of the last step.  NULL pointers are skipped. */
RL_API rl_status rl_set_neurons(void* ctx, const double* x, const double* u, const double* calcium, const uint8_t* fired);
RL_API rl_status rl_get_neurons(void* ctx, double* x, double* u, double* calcium, uint8_t* fired, double* input);

/* Asynchronous read of calcium and fired flags (either may be NULL), for
 * monitoring a running simulation without stalling it: the state is copied to
 * a device staging buffer in order with the context's work, and from there to
 * the caller's buffers on a copy stream of the context, so the copy overlaps
 * whatever the context runs next.  The buffers receive the values as of the
 * call (after the work issued before it) and must stay valid until
 * rl_snapshot_wait returns; pinned host memory makes the copy asynchronous.
 * Two snapshots may be in flight.  Serves what the reference's NeuronMonitor
 * records between steps (sim/Simulation.cpp:428-430) without a host stall. */
RL_API rl_status rl_snapshot_neurons(void* ctx, double* calcium, uint8_t* fired);
/* Waits until every snapshot issued so far has landed in host memory. */
RL_API rl_status rl_snapshot_wait(void* ctx);

/* Target calcium per neuron (the target function CalciumIO builds from a
 * --file-calcium, io/CalciumIO.cpp:27-130; otherwise every neuron has
 * rl_config.target_calcium), in either precision form (the FP32 form keeps an
 * FP32 copy and evaluates each neuron's growth curves in FP32). */
RL_API rl_status rl_set_target_calcium(void* ctx, const double* target);
RL_API rl_status rl_get_target_calcium(void* ctx, double* target);

/* Enable flags (NeuronsExtraInfo disable flags): 1 enabled, 0 disabled. */
RL_API rl_status rl_set_enabled(void* ctx, const uint8_t* enabled);

/* Synapse list (NetworkGraph plastic edges).  rl_get_edges aggregates equal
 * (target, source) pairs, drops zero weights and sorts by (target, source);
 * *count receives the number of aggregated edges. */
RL_API rl_status rl_add_edges(void* ctx, uint64_t m, const uint32_t* target, const uint32_t* source, const int32_t* weight);
RL_API rl_status rl_get_edges(void* ctx, uint32_t* target, uint32_t* source, int32_t* weight, uint64_t capacity, uint64_t* count);

/* Activity steps first_step .. first_step+nsteps-1 without plasticity:
 * input (synaptic_equally_weighted + normal), Izhikevich, calcium, growth
 * deltas — one fused kernel per step (NeuronModelCPU::update_electrical_activity,
 * CalciumCalculatorCPU::update_calcium, SynapticElementsCPU::update_number_elements). */
RL_API rl_status rl_activity_block(void* ctx, uint32_t first_step, uint32_t nsteps);

/* One plasticity update at `step` (Neurons::update_connectivity): commit of
 * the three element types, tree update, search, connector, graph rebuild. */
RL_API rl_status rl_plasticity_update(void* ctx, uint32_t step);

/* Simulation::simulate over steps first_step .. first_step+nsteps-1: one
 * activity step each, a plasticity update when step % interval == 0. */
RL_API rl_status rl_simulate(void* ctx, uint32_t first_step, uint32_t nsteps);

/* Block until all work of the context has finished. */
RL_API rl_status rl_synchronize(void* ctx);

RL_API rl_status rl_get_stats(void* ctx, rl_stats* out);

/* Issue all work of the context on `cuda_stream` (a cudaStream_t of the
 * context's device), or on the context's own stream when NULL. */
RL_API rl_status rl_set_stream(void* ctx, void* cuda_stream);

/* Allocation-free form of the tree part of rl_prepare_update_connectivity
 * (leaf counts + bottom-up reduction).  No counterpart in the reference: it
 * exists for callers that cannot allocate device memory when they update the
 * octree (a runtime that hands out all device memory from its own pool or
 * budget, or a host that must not touch the allocator once set-up is done).
 * Inputs are DEVICE arrays of n entries (vacant excitatory and inhibitory
 * dendrites, optional plasticity flags, NULL = the enabled flags); the result
 * goes to the context's octree, and the dendrite counts and flags are copied
 * into the context's own arrays, which the connector of the next
 * rl_update_connectivity accepts against.  The vacant AXON counts (the search
 * sources) are not an input here: they stay as the last commit or
 * rl_prepare_update_connectivity left them.
 * The call allocates nothing: its scratch (one counter per octree node) is a
 * file-scope device array of 2,097,152 counters (8 MiB) that every GPU
 * loading the library holds until exit; larger trees are rejected with
 * RL_ERR_OVERFLOW.  All calls share that array, so calls that overlap on the
 * GPU race.  The first call on a device looks up the array's device address,
 * and the first call on a context creates two events that order a caller
 * stream against the context's stream; both should come before any stream
 * capture.  Work is enqueued on cuda_stream (NULL: the context's stream)
 * after the context's earlier work, and the context's later work waits for
 * it; the caller synchronizes that stream before reading results on the
 * host.  Device errors of this call are reported by the next call that
 * checks for them (rl_synchronize does).  The caller's current device is
 * left as it was. */
RL_API rl_status rl_prepare_update_connectivity_noalloc(void* ctx, const uint32_t* d_vacant_exc, const uint32_t* d_vacant_inh,
                                                        const uint8_t* d_update, void* cuda_stream);

/* Diagnostic: the candidates of the first descent (from the root) of a search
 * by `source`, in visiting order, with their unnormalised attraction weights
 * evaluated in `precision` (RL_PRECISION_FP64 or RL_PRECISION_FP32) on the
 * current octree (after rl_prepare_update_connectivity).  *count receives the
 * number of candidates; at most `capacity` are copied. */
RL_API rl_status rl_candidate_weights(void* ctx, uint32_t source, int precision, uint32_t* nodes, double* weights, uint64_t capacity,
                                      uint64_t* count);

/* Run each full plasticity interval of activity steps as one captured CUDA
 * graph (1, the default) or as separate launches (0).  Graphs are used only on
 * a stream other than the legacy default stream. */
RL_API rl_status rl_set_graphs(void* ctx, int enable);

/* While the network has no synapses (no in-edges anywhere: the start of a
 * simulation, before the first connections), a neuron's step reads nothing of
 * the other neurons, so a block of activity steps runs as one launch with each
 * neuron's state kept in registers for the whole block (1, the default); 0
 * runs one launch per step.  The results are the same bits either way.  No
 * counterpart in the reference (its CPU loops run step by step). */
RL_API rl_status rl_set_step_fusion(void* ctx, int enable);

/* Turn per-phase CUDA-event timing on (1) or off (0). */
RL_API rl_status rl_set_profiling(void* ctx, int enable);

/* Accumulated device milliseconds and invocation counts per phase since the
 * last call (arrays of RL_NUM_PHASES entries); resets the accumulators. */
RL_API rl_status rl_get_phase_times(void* ctx, double* ms, uint64_t* counts);

/* Launch shapes of the hot kernels.  The search kernels walk the octree
 * without a stack (through per-node escape links) with `search_warps` warps per
 * block and `search_packet` lanes (sources) walking the descent from the root
 * together; `search_hot` > 0 selects the persistent form (one block of 32 warps
 * per SM taking warp tasks from a counter) that first copies up to
 * `search_hot` nodes of the top octree levels into shared memory;
 * the activity kernel runs `act_block` threads per block with `act_vec`
 * neurons per thread (FP32: vector loads and stores; FP64: 1, or 2 whose
 * steps the compiler interleaves), and with
 * `act_persistent` one resident wave of blocks strides over the neurons.  No
 * counterpart in the reference (its CPU loops have no launch shape). */
typedef struct rl_tuning {
    int32_t search_warps;    /* 2, 4 or 8 */
    int32_t search_hot;      /* 0, or 1024 / 4096 top octree nodes in shared memory (search_warps 32) */
    int32_t search_packet;   /* 32, 16, 4 or 1 searches of Morton-adjacent sources walking the first descent together;
                                0: one search per warp (search_warps 4; the tuner times it on networks of 65,536 neurons or more) */
    int32_t search_cap;      /* 1: registers capped at 64 (more resident warps), 0: as compiled */
    int32_t act_block;       /* 128, 256 or 512 */
    int32_t act_persistent;  /* 0 or 1 */
    int32_t act_vec;         /* 1, 2 or 4 (FP64: 1 or 2) */
    int32_t tuned;           /* bit 0: search shape timed or recalled, bit 1: activity shape */
} rl_tuning;

/* Candidates the tuner times, in the order of the times rl_get_tuning returns:
 * search: cap 0 then 1, packet 32, 16, 4, 1, warps 2, 4, 8 (24 shapes), then the
 * persistent form with 1024 and 4096 nodes in shared memory, packet 32 then 16
 * (4 shapes, 32 warps, registers capped at 64), then one search per warp
 * (packet 0, 4 warps per block; timed on networks of 65,536 neurons or more, 0 ms
 * elsewhere); the search shape is tuned per
 * density class of the search list (searches per neuron above 1/4, 1/32,
 * 1/256, or below), since sparse lists favour narrow packets;
 * activity: persistent 0 then 1, block 128, 256, 512, vec 1, 2, 4 (18 shapes). */
#define RL_NUM_SEARCH_SHAPES 29
#define RL_NUM_ACT_SHAPES 18

/* Autotuning: 0 keeps the current shapes; 1 times the candidates on the
 * context's own data at the next activity block and the next search and keeps the fastest,
 * reusing a result the process already has for the same precision, form, size
 * class (power of two of the neuron count), neuron model and kernel; 2 times them
 * again even then.
 * Timing runs the kernels on the current state and restores it, so results do
 * not depend on tuning. */
RL_API rl_status rl_autotune(void* ctx, int mode);

/* Shapes in use; search_ms / act_ms (NULL to skip) receive the timed
 * milliseconds per candidate (0 for a candidate not timed). */
RL_API rl_status rl_get_tuning(void* ctx, rl_tuning* out, float* search_ms, float* act_ms);

/* Set the shapes by hand (`tuned` is ignored); RL_ERR_INVALID for a shape that
 * is not a candidate. */
RL_API rl_status rl_set_tuning(void* ctx, const rl_tuning* t);

/* Device memory the context holds now and at most since creation (bytes). */
RL_API rl_status rl_ctx_memory(void* ctx, uint64_t* current, uint64_t* peak);

/* ------------------------------------------------------------------ serving
 * A request loop for sweep runs.  No counterpart in the reference, whose
 * Simulation (sim/Simulation.cpp) runs one network per process; a sweep there
 * is one mpirun per parameter set.  Here one process serves a stream of runs
 * on one GPU: each request is one network (rl_network: its size, seed, box,
 * theta, sigma and growth rates; the model parameters come from the server's
 * base rl_config) simulated for steps 1..steps exactly as rl_simulate does in a
 * context of its own.
 *
 * Admission is continuous: `slots` worker threads each run one context on a
 * stream of their own, so the work of running requests overlaps on the GPU,
 * and a pending request is admitted as soon as a slot is free and its device
 * footprint (rl_serve_footprint) fits into what is left of the HBM budget.
 * Pending requests are taken in arrival order; a request that does not fit
 * lets later ones pass at most 2*slots times before admission waits for it.
 * When several small requests are pending, one slot takes up to
 * `pack_networks` of them (each of at most `pack_max_neurons` neurons, all with
 * the same number of steps) into one batched context (rl_ensemble_create), so
 * they share every launch.  Results do not depend on how requests were
 * grouped or overlapped: each network evolves bit for bit as in a context of
 * its own. */
typedef struct rl_serve_config {
    uint64_t hbm_budget_bytes;  /* device bytes that admitted requests may hold together */
    uint64_t pack_max_neurons;  /* requests up to this size may share a batched context */
    int32_t slots;              /* runs on the GPU at a time (worker threads, one stream each) */
    int32_t pack_networks;      /* most requests in one batched context (1 = never pack) */
    int32_t use_graphs;         /* capture activity intervals as CUDA graphs (rl_set_graphs) */
    int32_t autotune;           /* rl_autotune mode of every context (shapes reused per size class) */
} rl_serve_config;

typedef struct rl_serve_request {
    rl_network net;             /* the network; net.num_neurons > 0 */
    const double* xyz;          /* 3*num_neurons positions, copied at submission */
    const uint8_t* signal;      /* num_neurons signal types (1 = inhibitory), copied */
    const double* grown[3];     /* initial grown elements per type, or NULL for 0; copied */
    uint32_t steps;             /* simulate steps 1..steps */
    uint32_t keep_state;        /* 1: keep the final state for rl_serve_fetch */
} rl_serve_request;

typedef struct rl_serve_done {
    uint64_t id;
    int32_t status;             /* rl_status of the run */
    uint32_t pack_size;         /* requests that shared its context */
    double t_submit;            /* seconds since the server was created */
    double t_admit;
    double t_finish;
    uint64_t num_neurons;
    uint64_t num_synapses;      /* synapses of this network after the last step */
    uint64_t footprint_bytes;   /* what admission reserved for it */
    uint64_t device_peak_bytes; /* peak bytes of the context it ran in */
    uint64_t neuron_steps;      /* num_neurons * steps */
} rl_serve_done;

/* Device bytes admission reserves for a request: an upper bound on what its
 * context holds at any time, from its size, the initial axons and the most
 * the axons can grow in `steps` steps (growth_rate[0] per step). */
RL_API rl_status rl_serve_footprint(const rl_config* base, const rl_network* net, double initial_axons, uint32_t steps, uint64_t* bytes);

RL_API rl_status rl_serve_create(const rl_config* base, const rl_serve_config* sc, void** server);

/* Queue a request; *id receives its number.  Requests whose footprint exceeds
 * the whole budget are refused with RL_ERR_OOM. */
RL_API rl_status rl_serve_submit(void* server, const rl_serve_request* req, uint64_t* id);

/* Finished requests in completion order: up to `capacity` records, waiting up
 * to wait_ms milliseconds for the first one (0: do not wait). */
RL_API rl_status rl_serve_poll(void* server, rl_serve_done* out, uint64_t capacity, uint64_t* count, int32_t wait_ms);

/* The kept final state of a finished request (keep_state = 1): x, u, calcium
 * (num_neurons each), connected elements (3*num_neurons, type-major) and its
 * synapses (network-local ids, sorted by target then source); NULL pointers
 * are skipped.  The record is released afterwards. */
RL_API rl_status rl_serve_fetch(void* server, uint64_t id, double* x, double* u, double* calcium, uint32_t* connected,
                                rl_synapse* synapses, uint64_t capacity);

/* Requests queued, running, and device bytes reserved now. */
RL_API rl_status rl_serve_load(void* server, uint64_t* pending, uint64_t* running, uint64_t* reserved_bytes);

/* Let every queued and running request finish, then stop the workers and free
 * the server with the results nobody fetched. */
RL_API rl_status rl_serve_destroy(void* server);

#ifdef __cplusplus
}
#endif

#endif /* RELEARN_B200_H */
