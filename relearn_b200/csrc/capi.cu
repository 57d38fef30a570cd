// C ABI of librelearn_b200 (declared in include/relearn_b200.h).
#include <atomic>
#include <tuple>
#include <mutex>
#include <map>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

#include "rl_context.cuh"

namespace rl {

namespace {
constexpr int kMaxDevices = 64;
std::atomic<int> g_live[kMaxDevices];  // contexts alive per device
}  // namespace

PhaseScope::PhaseScope(Ctx& ctx, int ph, uint32_t weight) : c(&ctx), phase(ph) {
    if (!c->timer.on || c->capturing) {
        c = nullptr;
        return;
    }
    auto take = [&]() {
        cudaEvent_t e;
        if (!c->timer.free_events.empty()) {
            e = c->timer.free_events.back();
            c->timer.free_events.pop_back();
        } else {
            RL_CUDA_TRY(cudaEventCreate(&e));
        }
        return e;
    };
    cudaEvent_t start = take();
    end = take();
    RL_CUDA_TRY(cudaEventRecord(start, c->stream));
    c->timer.pending[phase].push_back(PendingTimer{ start, end, weight });
}

PhaseScope::~PhaseScope() {
    if (c) {
        cudaEventRecord(end, c->stream);
    }
}

static void resolve_timers(Ctx& c) {
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    for (int p = 0; p < PH_COUNT; ++p) {
        for (auto& pr : c.timer.pending[p]) {
            float ms = 0.f;
            RL_CUDA_TRY(cudaEventElapsedTime(&ms, pr.start, pr.end));
            c.timer.ms[p] += ms;
            c.timer.count[p] += pr.weight;
            c.timer.free_events.push_back(pr.start);
            c.timer.free_events.push_back(pr.end);
        }
        c.timer.pending[p].clear();
    }
}

void check_device_error(Ctx& c, const char* phase) {
    uint32_t h = 0;
    RL_CUDA_TRY(cudaMemcpyAsync(&h, c.err.p, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    if (h == 0) {
        return;
    }
    RL_CUDA_TRY(cudaMemsetAsync(c.err.p, 0, sizeof(uint32_t), c.stream));
    std::string msg = std::string(phase) + ": device error";
    rl_status st = RL_ERR_DEVICE;
    if (h & DERR_OUT_OF_BOX) {
        msg += " [position outside the simulation box]";
        st = RL_ERR_INVALID;
    }
    if (h & DERR_DUPLICATE) {
        msg += " [two positions coincide within 42 octree levels]";
        st = RL_ERR_INVALID;
    }
    if (h & DERR_STACK) {
        msg += " [octree walk deeper than its bound]";
        st = RL_ERR_OVERFLOW;
    }
    if (h & DERR_WALK) {
        msg += " [octree walk left the node range]";
    }
    if (h & DERR_NO_CROSSING) {
        msg += " [pick found no crossing]";
    }
    if (h & DERR_CAPACITY) {
        msg += " [buffer capacity]";
        st = RL_ERR_OVERFLOW;
    }
    if (h & DERR_CONNECT) {
        msg += " [connector element underflow]";
    }
    if (h & DERR_TIMEOUT) {
        msg += " [bounded wait ran out]";
        st = RL_ERR_TIMEOUT;
    }
    throw Error{ st, msg };
}

namespace {

template <typename T>
void upload(DBuf<T>& d, const T* h, size_t n, cudaStream_t st) {
    RL_CUDA_TRY(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

template <typename T>
void download(T* h, const DBuf<T>& d, size_t n, cudaStream_t st) {
    RL_CUDA_TRY(cudaMemcpyAsync(h, d.p, n * sizeof(T), cudaMemcpyDeviceToHost, st));
}

__global__ void k_fill_f64(double* p, uint64_t n, double v) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        p[i] = v;
    }
}

void fill(DBuf<double>& d, size_t n, double v, cudaStream_t st) {
    k_fill_f64<<<blocks_for(n, 256), 256, 0, st>>>(d.p, n, v);
    RL_LAUNCH_CHECK();
}

void validate(const rl_config& k) {
    RL_CHECK(k.num_neurons > 0, RL_ERR_INVALID, "num_neurons must be positive");
    RL_CHECK(k.num_neurons < (1u << 30), RL_ERR_UNSUPPORTED, "num_neurons must be below 2^30");
    RL_CHECK(k.theta > 0.0 && k.theta <= 0.5, RL_ERR_INVALID, "theta must lie in (0, 0.5] (Constants::bh_max_theta)");
    RL_CHECK(k.sigma > 0.0, RL_ERR_INVALID, "sigma must be positive");
    RL_CHECK(k.h_model >= 1 && k.h_model <= 1000, RL_ERR_INVALID, "h_model must lie in [1, 1000]");
    RL_CHECK(k.h_calcium >= 1 && k.h_calcium <= 1000, RL_ERR_INVALID, "h_calcium must lie in [1, 1000]");
    RL_CHECK(k.noise_stddev > 0.0, RL_ERR_INVALID, "noise_stddev must be positive");
    RL_CHECK(k.precision == RL_PRECISION_FP64 || k.precision == RL_PRECISION_FP32, RL_ERR_INVALID, "precision must be FP64 or FP32");
    RL_CHECK(k.kernel_type >= RL_KERNEL_GAUSSIAN && k.kernel_type <= RL_KERNEL_WEIBULL, RL_ERR_INVALID, "unknown kernel type");
    RL_CHECK(k.neuron_model >= RL_MODEL_IZHIKEVICH && k.neuron_model <= RL_MODEL_AEIF, RL_ERR_INVALID, "unknown neuron model");
    RL_CHECK(k.neuron_model != RL_MODEL_POISSON || k.poisson_tau_x > 0.0, RL_ERR_INVALID, "Poisson tau_x must be positive");
    RL_CHECK(k.neuron_model != RL_MODEL_AEIF || (k.aeif_C > 0.0 && k.aeif_d_T > 0.0 && k.aeif_tau_w > 0.0), RL_ERR_INVALID,
             "AEIF C, d_T and tau_w must be positive");
    // GammaDistributionKernel / WeibullDistributionKernel / LinearDistributionKernel constructors
    RL_CHECK(k.kernel_type != RL_KERNEL_GAMMA || (k.kernel_k > 0.0 && k.kernel_scale > 0.0), RL_ERR_INVALID, "gamma k and theta must be positive");
    RL_CHECK(k.kernel_type != RL_KERNEL_WEIBULL || (k.kernel_k > 0.0 && k.kernel_scale > 0.0), RL_ERR_INVALID, "Weibull k and b must be positive");
    RL_CHECK(k.kernel_type != RL_KERNEL_LINEAR || k.linear_cutoff >= 0.0, RL_ERR_INVALID, "the linear cut-off must not be negative");
    for (int a = 0; a < 3; ++a) {
        RL_CHECK(k.box_min[a] <= k.box_max[a], RL_ERR_INVALID, "box_min must not exceed box_max");
        RL_CHECK(k.retract_ratio[a] >= 0.0 && k.retract_ratio[a] <= 1.0, RL_ERR_INVALID, "retract ratio must lie in [0, 1]");
    }
}

// Constants of the probability kernel, as the kernels' constructors compute
// them (algorithm/Kernel/Gamma.h, Weibull.h, Linear.h).
KernelParams make_kernel(const rl_config& k) {
    KernelParams p;
    p.type = k.kernel_type;
    p.k_minus_1 = k.kernel_k - 1.0;
    if (k.kernel_type == RL_KERNEL_GAMMA) {
        p.a = 1.0 / (std::tgamma(k.kernel_k) * std::pow(k.kernel_scale, k.kernel_k));  // gamma_divisor_inv
        p.b = -1.0 / k.kernel_scale;                                                   // theta_divisor
    } else if (k.kernel_type == RL_KERNEL_WEIBULL) {
        p.a = k.kernel_scale * k.kernel_k;  // factor_1 = b * k
        p.b = k.kernel_scale;               // b
    }
    p.cutoff = k.linear_cutoff;
    p.cutoff_inf = std::isinf(k.linear_cutoff) ? 1 : 0;
    return p;
}

// The network table: one network from the config, or the ensemble's list.
void setup_nets(Ctx& c, const rl_network* nets, uint32_t num) {
    c.nets.clear();
    uint32_t first = 0;
    for (uint32_t k = 0; k < (nets ? num : 1u); ++k) {
        NetInfo N{};
        if (nets) {
            const rl_network& r = nets[k];
            RL_CHECK(r.num_neurons > 0, RL_ERR_INVALID, "every network needs at least one neuron");
            RL_CHECK(r.theta > 0.0 && r.theta <= 0.5, RL_ERR_INVALID, "theta must lie in (0, 0.5] (Constants::bh_max_theta)");
            RL_CHECK(r.sigma > 0.0, RL_ERR_INVALID, "sigma must be positive");
            N.seed = r.seed;
            N.count = r.num_neurons;
            N.theta = r.theta;
            N.sigma = r.sigma;
            for (int a = 0; a < 3; ++a) {
                RL_CHECK(r.box_min[a] <= r.box_max[a], RL_ERR_INVALID, "box_min must not exceed box_max");
                N.box_min[a] = r.box_min[a];
                N.box_max[a] = r.box_max[a];
                N.nu[a] = r.growth_rate[a];
            }
        } else {
            const rl_config& cf = c.cfg;
            N.seed = cf.seed;
            N.count = cf.num_neurons;
            N.theta = cf.theta;
            N.sigma = cf.sigma;
            for (int a = 0; a < 3; ++a) {
                N.box_min[a] = cf.box_min[a];
                N.box_max[a] = cf.box_max[a];
                N.nu[a] = cf.growth_rate[a];
            }
        }
        N.first = first;
        first += N.count;
        N.scale = -1.0 / (N.sigma * N.sigma);
        N.theta32 = (float)N.theta;
        N.inv_sigma2_32 = (float)(1.0 / (N.sigma * N.sigma));
        for (int a = 0; a < 3; ++a) {
            N.nu32[a] = (float)N.nu[a];
        }
        N.root_leaf = 0;
        // fixed-point frame of the FP32 search
        const double extent = std::max(N.box_max[0] - N.box_min[0], std::max(N.box_max[1] - N.box_min[1], N.box_max[2] - N.box_min[2]));
        double quantum = 1.0;
        while (quantum * 1073741824.0 < extent) {
            quantum *= 2.0;
        }
        while (quantum * 0.5 * 1073741824.0 >= extent && quantum > 1e-30) {
            quantum *= 0.5;
        }
        for (int a = 0; a < 3; ++a) {
            N.frame.origin[a] = N.box_min[a];
        }
        N.frame.quantum = (float)quantum;
        N.frame.inv_quantum = 1.0 / quantum;
        c.nets.push_back(N);
    }
    RL_CHECK(first == c.n, RL_ERR_INVALID, "network sizes do not add up to num_neurons");

    RL_CHECK(c.nets.size() <= 65535, RL_ERR_UNSUPPORTED, "at most 65535 networks per context");
    c.d_nets.alloc(c.nets.size());
    RL_CUDA_TRY(cudaMemcpyAsync(c.d_nets.p, c.nets.data(), c.nets.size() * sizeof(NetInfo), cudaMemcpyHostToDevice, c.stream));
    std::vector<uint16_t> net_of(c.n);
    for (size_t k = 0; k < c.nets.size(); ++k) {
        std::fill(net_of.begin() + c.nets[k].first, net_of.begin() + c.nets[k].first + c.nets[k].count, (uint16_t)k);
    }
    c.net_of.alloc(c.n);
    RL_CUDA_TRY(cudaMemcpyAsync(c.net_of.p, net_of.data(), c.n * sizeof(uint16_t), cudaMemcpyHostToDevice, c.stream));
    std::vector<NetBlock> blocks;
    for (size_t k = 0; k < c.nets.size(); ++k) {
        for (uint32_t b = 0; b < c.nets[k].count; b += kNetBlock) {
            const uint32_t left = c.nets[k].count - b;
            blocks.push_back(NetBlock{ c.nets[k].first + b, (uint16_t)k, (uint16_t)(left < kNetBlock ? left : kNetBlock) });
        }
    }
    c.num_net_blocks = (uint32_t)blocks.size();
    c.net_blocks.alloc(blocks.size());
    RL_CUDA_TRY(cudaMemcpyAsync(c.net_blocks.p, blocks.data(), blocks.size() * sizeof(NetBlock), cudaMemcpyHostToDevice, c.stream));
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
}

// Small pinned host slots (four counters each) for the contexts' count reads.
// Pinned memory is taken from the driver a page at a time and never given
// back: cudaMallocHost and cudaFreeHost are slow and cudaFreeHost waits for the
// whole device, which a serving loop that creates and destroys contexts while
// others run must not do.
std::mutex g_pinned_mu;
std::vector<unsigned long long*> g_pinned_free;

unsigned long long* pinned_slot_take() {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    if (g_pinned_free.empty()) {
        constexpr size_t kSlot = 4, kSlots = 512;  // 16 KiB per page
        unsigned long long* page = nullptr;
        RL_CUDA_TRY(cudaMallocHost(&page, kSlot * kSlots * sizeof(unsigned long long)));
        for (size_t k = 0; k < kSlots; ++k) {
            g_pinned_free.push_back(page + k * kSlot);
        }
    }
    unsigned long long* s = g_pinned_free.back();
    g_pinned_free.pop_back();
    return s;
}

void pinned_slot_give(unsigned long long* s) {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    g_pinned_free.push_back(s);
}

void create(Ctx& c, const rl_config& k, const rl_network* nets = nullptr, uint32_t num_nets = 0) {
    validate(k);
    c.cfg = k;
    c.kernel = make_kernel(k);
    c.n = k.num_neurons;
    c.device = k.device;
    int count = 0;
    RL_CUDA_TRY(cudaGetDeviceCount(&count));
    RL_CHECK(k.device >= 0 && k.device < count, RL_ERR_DEVICE, "no such CUDA device");
    RL_CUDA_TRY(cudaSetDevice(k.device));
    RL_CUDA_TRY(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, k.device));
    RL_CUDA_TRY(cudaDeviceGetAttribute(&c.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, k.device));
    RL_CUDA_TRY(cudaStreamCreateWithFlags(&c.own_stream, cudaStreamNonBlocking));
    c.stream = c.own_stream;
    g_bind = Binding{ c.stream, &c.launches, &c.device_bytes, &c.device_peak };
    RL_CHECK(k.device < kMaxDevices, RL_ERR_DEVICE, "device ordinal above what this build tracks");
    {
        // keep freed device memory in the pool for the next context or buffer
        cudaMemPool_t pool;
        RL_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, k.device));
        uint64_t keep = UINT64_MAX;
        RL_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    g_live[k.device].fetch_add(1);
    c.counted = true;
    const size_t n = c.n;
    Neurons& N = c.nr;
    N.px.alloc(n);
    N.py.alloc(n);
    N.pz.alloc(n);
    N.signal.alloc(n);
    N.enabled.alloc(n);
    N.update.alloc(n);
    N.x.alloc(n);
    N.u.alloc(n);
    N.calcium.alloc(n);
    N.target.alloc(n);
    N.input.alloc(n);
    N.fired[0].alloc(n);
    N.fired[1].alloc(n);
    for (int t = 0; t < 3; ++t) {
        N.grown[t].alloc(n);
        N.delta[t].alloc(n);
        N.connected[t].alloc(n);
        N.vacant[t].alloc(n);
        RL_CUDA_TRY(cudaMemsetAsync(N.grown[t].p, 0, n * sizeof(double), c.stream));
        RL_CUDA_TRY(cudaMemsetAsync(N.delta[t].p, 0, n * sizeof(double), c.stream));
        RL_CUDA_TRY(cudaMemsetAsync(N.connected[t].p, 0, n * sizeof(uint32_t), c.stream));
        RL_CUDA_TRY(cudaMemsetAsync(N.vacant[t].p, 0, n * sizeof(uint32_t), c.stream));
    }
    N.search_vacant.alloc(n);
    RL_CUDA_TRY(cudaMemsetAsync(N.search_vacant.p, 0, n * sizeof(uint32_t), c.stream));
    RL_CUDA_TRY(cudaMemsetAsync(N.signal.p, 0, n, c.stream));
    RL_CUDA_TRY(cudaMemsetAsync(N.enabled.p, 1, n, c.stream));
    RL_CUDA_TRY(cudaMemsetAsync(N.update.p, 1, n, c.stream));
    RL_CUDA_TRY(cudaMemsetAsync(N.fired[0].p, 0, n, c.stream));
    RL_CUDA_TRY(cudaMemsetAsync(N.fired[1].p, 0, n, c.stream));
    // initial x and second state variable per model: init_neurons of
    // IzhikevichModelBase (models/izhikevich/IzhikevichModelBase.cpp:59-66),
    // FitzHughNagumoModelBase and AEIFModelBase; NeuronModel::init and
    // PoissonModelBase::init: x = 0, no refractory steps
    double x0 = k.iz_c, u0 = 0.0;
    if (k.neuron_model == RL_MODEL_POISSON) {
        x0 = 0.0;
    } else if (k.neuron_model == RL_MODEL_FITZHUGH_NAGUMO) {
        x0 = k.fhn_init_x;
        u0 = k.fhn_init_w;
    } else if (k.neuron_model == RL_MODEL_AEIF) {
        x0 = k.aeif_E_L;
    }
    fill(N.x, n, x0, c.stream);
    fill(N.u, n, u0, c.stream);
    fill(N.calcium, n, k.initial_calcium, c.stream);
    fill(N.target, n, k.target_calcium, c.stream);
    fill(N.input, n, 0.0, c.stream);
    c.graph.offsets.alloc(n + 1);
    RL_CUDA_TRY(cudaMemsetAsync(c.graph.offsets.p, 0, (n + 1) * sizeof(uint32_t), c.stream));
    c.to_delete.alloc(n);
    c.act_desc.alloc(1);
    c.err.alloc(1);
    RL_CUDA_TRY(cudaMemsetAsync(c.err.p, 0, sizeof(uint32_t), c.stream));
    c.commit_cnt.alloc(4);
    c.h_commit = pinned_slot_take();
    c.counters.alloc(4);
    RL_CUDA_TRY(cudaMemsetAsync(c.counters.p, 0, 4 * sizeof(uint64_t), c.stream));
    setup_nets(c, nets, num_nets);
    if (is_fp32(c)) {
        alloc_fp32(c);
    }
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
}

void require_tree(Ctx& c) {
    RL_CHECK(c.positions_set, RL_ERR_INVALID, "rl_set_positions has not been called");
}

void plasticity_update(Ctx& c, uint32_t step) {
    require_tree(c);
    // SynapseDeletionFinderCPU::delete_synapses: commit the three element types
    {
        // SynapseDeletionFinderCPU::delete_synapses (neurons/helper/SynapseDeletionFinderCPU.cpp:27-92):
        // commit axons, delete; commit excitatory dendrites, delete; commit inhibitory dendrites, delete
        // The commit of a type reads the connected counts that the deletion
        // of an earlier type changes, so types are committed in order with the
        // deletions between them.  Usually nothing is deleted: the three
        // commits go out at once, each skipping itself on the device when an
        // earlier one left deletions, and a single read says where the
        // sequential path has to take over.
        {
            PhaseScope ps(c, PH_COMMIT);
            RL_CUDA_TRY(cudaMemsetAsync(c.commit_cnt.p, 0, 4 * sizeof(unsigned long long), c.stream));
            if (!launch_commit_all(c)) {
                for (int t = 0; t < 3; ++t) {
                    launch_commit_guarded(c, t);
                }
                // the same read says whether the search will have anything to do
                launch_vacant_axon_count(c, c.commit_cnt.p + 3);
            }
            RL_CUDA_TRY(cudaMemcpyAsync(c.h_commit, c.commit_cnt.p, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.stream));
        }
        // The octree update goes out before the host reads the counts, so that
        // the GPU works while the host waits; it is correct unless deletions
        // follow, which change vacant dendrites: then it runs again below
        // (incrementally: only the leaves the deletions changed).  A network
        // whose last update deleted synapses will most likely delete again
        // (once synapses exist, every update deletes some), so there the
        // update waits for the deletions and runs once.  Either way every
        // changed leaf is reduced before the search, so the octree is the same.
        RL_CUDA_TRY(cudaMemcpyAsync(c.nr.update.p, c.nr.enabled.p, c.n, cudaMemcpyDeviceToDevice, c.stream));
        const bool speculate = !c.deleted_last;
        if (speculate) {
            PhaseScope ps(c, PH_TREE_UPDATE);
            update_tree(c);
        }
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
        const unsigned long long* h = c.h_commit;
        c.stats.bound_to_delete += h[0] + h[1] + h[2];
        const int first = h[0] ? 0 : (h[1] ? 1 : (h[2] ? 2 : 3));
        // deletions change vacant axons: then the search counts them itself
        c.no_searches = first == 3 && h[3] == 0;
        if (first < 3) {
            PhaseScope ps(c, PH_COMMIT);
            c.stats.synapses_deleted += run_deletion(c, step, first);
            for (int t = first + 1; t < 3; ++t) {
                if (run_commit(c, t) > 0) {
                    c.stats.synapses_deleted += run_deletion(c, step, t);
                }
            }
        }
        if (first < 3 || !speculate) {
            PhaseScope ps(c, PH_TREE_UPDATE);
            update_tree(c);
        }
        c.deleted_last = first < 3;
    }
    // Neurons::create_synapses: search from the committed vacant axons
    RL_CUDA_TRY(cudaMemcpyAsync(c.nr.search_vacant.p, c.nr.vacant[0].p, c.n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c.stream));
    {
        // phases without work record no timing events (they would only add
        // host calls while the device waits)
        if (c.no_searches) {
            c.search.num_searches = 0;  // no enabled neuron has a vacant axon
            c.search.num_requests = 0;
        } else {
            PhaseScope ps(c, PH_SEARCH);
            run_search(c, step);
        }
        c.no_searches = false;
    }
    if (c.search.num_requests > 0) {
        PhaseScope ps(c, PH_CONNECTOR);
        run_connector(c, step);
    }
    if (c.graph.num_new > 0 || c.graph.zeros) {
        PhaseScope ps(c, PH_GRAPH);
        rebuild_graph(c);
    }
    c.stats.plasticity_updates += 1;
}

}  // namespace

// ------------------------------------------------------------ tuning cache
namespace {
std::mutex g_tune_mu;
using TuneKey = std::tuple<int, int, int, int, int>;
std::map<std::pair<TuneKey, int>, SearchVariant> g_search_shapes;  // with the search list's density class
std::map<TuneKey, ActVariant> g_act_shapes;

// precision, batched or not, power of two of the neuron count, neuron model, kernel
TuneKey tune_key(const Ctx& c) {
    int lg = 0;
    while (lg < 40 && (1ull << (lg + 1)) <= (uint64_t)c.n) {
        ++lg;
    }
    // networks with synapses read in-edges every step: a class of their own
    return std::make_tuple(c.cfg.precision, (c.multi() ? 1 : 0) | (c.graph.num_edges > 0 ? 2 : 0), lg, c.cfg.neuron_model, c.cfg.kernel_type);
}
}  // namespace

void remember_search_tuning(const Ctx& c, int density_class) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_search_shapes[std::make_pair(tune_key(c), density_class)] = c.tune.search;
}

bool recall_search_tuning(Ctx& c, int density_class) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_search_shapes.find(std::make_pair(tune_key(c), density_class));
    if (it == g_search_shapes.end()) {
        return false;
    }
    c.tune.search = it->second;
    return true;
}

void remember_act_tuning(const Ctx& c) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_act_shapes[tune_key(c)] = c.tune.act;
}

bool recall_act_tuning(Ctx& c) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_act_shapes.find(tune_key(c));
    if (it == g_act_shapes.end()) {
        return false;
    }
    c.tune.act = it->second;
    return true;
}

namespace {

Ctx* as_ctx(void* p) {
    return static_cast<Ctx*>(p);
}

// Binds a context to the calling thread for one entry point.
struct Bind {
    explicit Bind(Ctx& c) { g_bind = Binding{ c.stream, &c.launches, &c.device_bytes, &c.device_peak }; }
    ~Bind() { g_bind = Binding{}; }
    Bind(const Bind&) = delete;
    Bind& operator=(const Bind&) = delete;
};

template <typename F>
rl_status guarded(void* ctx, F&& f) {
    if (!ctx) {
        return RL_ERR_INVALID;
    }
    Ctx& c = *as_ctx(ctx);
    Bind bind(c);
    try {
        RL_CUDA_TRY(cudaSetDevice(c.device));
        f(c);
        return RL_OK;
    } catch (const Error& e) {
        c.last_error = e.message;
        return e.status;
    } catch (const std::bad_alloc&) {
        c.last_error = "host allocation failed";
        return RL_ERR_OOM;
    } catch (...) {
        c.last_error = "unexpected host exception";
        return RL_ERR_INVALID;
    }
}

}  // namespace
}  // namespace rl

using rl::Ctx;

extern "C" {

int32_t rl_abi_version(void) {
    return RL_ABI_VERSION;
}

const char* rl_status_string(rl_status s) {
    switch (s) {
        case RL_OK: return "ok";
        case RL_ERR_INVALID: return "invalid argument or state";
        case RL_ERR_OOM: return "device allocation failed";
        case RL_ERR_DEVICE: return "CUDA device error";
        case RL_ERR_TIMEOUT: return "bounded device wait ran out";
        case RL_ERR_OVERFLOW: return "device buffer overflow";
        case RL_ERR_UNSUPPORTED: return "unsupported configuration";
    }
    return "unknown status";
}

void rl_config_default(rl_config* k, uint32_t num_neurons, double side) {
    std::memset(k, 0, sizeof(*k));
    k->num_neurons = num_neurons;
    k->plasticity_interval = 100;
    k->h_model = 10;
    k->h_calcium = 10;
    k->seed = 1;
    for (int a = 0; a < 3; ++a) {
        k->box_min[a] = 0.0;
        k->box_max[a] = side;
        k->growth_rate[a] = 1e-4;
        k->retract_ratio[a] = 0.0;
    }
    k->theta = 0.3;
    k->sigma = 750.0;
    k->mu = 0.0;
    k->iz_a = 0.1;
    k->iz_b = 0.2;
    k->iz_c = -65.0;
    k->iz_d = 2.0;
    k->iz_v_spike = 30.0;
    k->iz_k1 = 0.04;
    k->iz_k2 = 5.0;
    k->iz_k3 = 140.0;
    k->beta = 0.001;
    k->tau_c = 10000.0;
    k->target_calcium = 0.7;
    k->initial_calcium = 0.0;
    k->min_calcium[0] = 0.4;
    k->min_calcium[1] = 0.1;
    k->min_calcium[2] = 0.0;
    k->conductance = 1.0;
    k->noise_mean = 5.0;
    k->noise_stddev = 2.0;
    k->device = 0;
    k->kernel_type = RL_KERNEL_GAUSSIAN;
    k->kernel_k = 1.0;
    k->kernel_scale = 1.0;
    k->linear_cutoff = INFINITY;
    // neurons/models/*/Parameters.h defaults
    k->neuron_model = RL_MODEL_IZHIKEVICH;
    k->poisson_refractory = 4;
    k->poisson_x0 = 0.05;
    k->poisson_tau_x = 5.0;
    k->fhn_a = 0.7;
    k->fhn_b = 0.8;
    k->fhn_phi = 0.08;
    k->fhn_init_x = -1.2;
    k->fhn_init_w = -0.6;
    k->aeif_C = 281.0;
    k->aeif_g_L = 30.0;
    k->aeif_E_L = -70.6;
    k->aeif_V_T = -50.4;
    k->aeif_d_T = 2.0;
    k->aeif_tau_w = 144.0;
    k->aeif_a = 4.0;
    k->aeif_b = 0.0805;
    k->aeif_V_spike = 20.0;
}

rl_status rl_ctx_create(const rl_config* cfg, void** out) {
    if (!cfg || !out) {
        return RL_ERR_INVALID;
    }
    *out = nullptr;
    Ctx* c = new (std::nothrow) Ctx();
    if (!c) {
        return RL_ERR_OOM;
    }
    try {
        rl::create(*c, *cfg);
    } catch (const rl::Error& e) {
        std::fprintf(stderr, "rl_ctx_create: %s\n", e.message.c_str());
        rl::discard(c);
        return e.status;
    }
    rl::g_bind = rl::Binding{};
    *out = c;
    return RL_OK;
}

rl_status rl_ensemble_create(const rl_config* base, const rl_network* networks, uint32_t num_networks, void** out) {
    if (!base || !networks || !out || num_networks == 0) {
        return RL_ERR_INVALID;
    }
    *out = nullptr;
    rl_config cfg = *base;
    uint64_t total = 0;
    for (uint32_t k = 0; k < num_networks; ++k) {
        total += networks[k].num_neurons;
    }
    if (total == 0 || total >= (1ull << 30)) {
        return RL_ERR_INVALID;
    }
    cfg.num_neurons = (uint32_t)total;
    // the base box and theta only need to pass validation; each network brings its own
    for (int a = 0; a < 3; ++a) {
        cfg.box_min[a] = 0.0;
        cfg.box_max[a] = 1.0;
    }
    Ctx* c = new (std::nothrow) Ctx();
    if (!c) {
        return RL_ERR_OOM;
    }
    try {
        rl::create(*c, cfg, networks, num_networks);
    } catch (const rl::Error& e) {
        std::fprintf(stderr, "rl_ensemble_create: %s\n", e.message.c_str());
        rl::discard(c);
        return e.status;
    }
    rl::g_bind = rl::Binding{};
    *out = c;
    return RL_OK;
}

rl_status rl_ctx_destroy(void* ctx) {
    if (!ctx) {
        return RL_ERR_INVALID;
    }
    rl::discard(static_cast<Ctx*>(ctx));
    return RL_OK;
}

}  // extern "C"

namespace rl {

void ensure_copy_stream(Ctx& c) {
    if (c.copy_stream) {
        return;
    }
    RL_CUDA_TRY(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
    RL_CUDA_TRY(cudaStreamCreateWithFlags(&c.upload_stream, cudaStreamNonBlocking));
    RL_CUDA_TRY(cudaEventCreateWithFlags(&c.upload_done, cudaEventDisableTiming));
    RL_CUDA_TRY(cudaEventCreateWithFlags(&c.stage_free, cudaEventDisableTiming));
    for (auto& s : c.snap) {
        RL_CUDA_TRY(cudaEventCreateWithFlags(&s.staged, cudaEventDisableTiming));
        RL_CUDA_TRY(cudaEventCreateWithFlags(&s.landed, cudaEventDisableTiming));
    }
}

void issue_snapshots(Ctx& c) {
    for (int k = 0; k < 2; ++k) {
        // the older slot first, so the host copies land in call order
        Ctx::SnapSlot& s = c.snap[(c.snap_next + k) & 1];
        if (!s.pending || s.issued) {
            continue;
        }
        RL_CUDA_TRY(cudaStreamWaitEvent(c.copy_stream, s.staged, 0));
        if (s.host_calcium) {
            RL_CUDA_TRY(cudaMemcpyAsync(s.host_calcium, s.calcium.p, c.n * sizeof(double), cudaMemcpyDeviceToHost, c.copy_stream));
        }
        if (s.host_fired) {
            RL_CUDA_TRY(cudaMemcpyAsync(s.host_fired, s.fired.p, c.n, cudaMemcpyDeviceToHost, c.copy_stream));
        }
        RL_CUDA_TRY(cudaEventRecord(s.landed, c.copy_stream));
        s.issued = true;
    }
}

void discard(Ctx* c) {
    cudaSetDevice(c->device);
    if (c->copy_stream) {
        try {
            issue_snapshots(*c);  // buffers handed over must still be written
        } catch (...) {
        }
    }
    g_bind = Binding{ c->stream, &c->launches, &c->device_bytes, &c->device_peak };
    if (c->copy_stream) {
        // snapshots in flight read the staging buffers: let them land first
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamSynchronize(c->upload_stream);
        cudaStreamDestroy(c->copy_stream);
        cudaStreamDestroy(c->upload_stream);
        c->copy_stream = nullptr;
        c->upload_stream = nullptr;
        for (cudaEvent_t e : { c->upload_done, c->stage_free, c->snap[0].staged, c->snap[0].landed, c->snap[1].staged, c->snap[1].landed }) {
            if (e) {
                cudaEventDestroy(e);
            }
        }
    }
    if (c->stream) {
        cudaStreamSynchronize(c->stream);
    }
    if (c->growth_stream) {
        cudaStreamSynchronize(c->growth_stream);
        cudaStreamDestroy(c->growth_stream);
        cudaEventDestroy(c->growth_fork);
        cudaEventDestroy(c->growth_join);
        c->growth_stream = nullptr;
    }
    for (cudaEvent_t e : { c->noalloc_before, c->noalloc_after }) {
        if (e) {
            cudaEventSynchronize(e);
            cudaEventDestroy(e);
        }
    }
    for (int p = 0; p < rl::PH_COUNT; ++p) {
        for (auto& pr : c->timer.pending[p]) {
            cudaEventDestroy(pr.start);
            cudaEventDestroy(pr.end);
        }
    }
    for (auto e : c->timer.free_events) {
        cudaEventDestroy(e);
    }
    for (auto& g : c->act_graph) {
        if (g) {
            cudaGraphExecDestroy(g);
        }
    }
    if (c->h_commit) {
        pinned_slot_give(c->h_commit);
        c->h_commit = nullptr;
    }
    // device buffers are freed on their streams; the context's own stream
    // goes last
    cudaStream_t own = c->own_stream;
    cudaStream_t last = c->stream;
    const int dev = c->device;
    const bool counted = c->counted;
    delete c;
    g_bind = Binding{};
    if (last) {
        cudaStreamSynchronize(last);
    }
    if (own) {
        cudaStreamDestroy(own);
    }
    // the pool keeps freed memory for the next context; give it back to the
    // device when the last context of the device is gone
    if (counted && dev >= 0 && dev < kMaxDevices && g_live[dev].fetch_sub(1) == 1) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            cudaMemPoolTrimTo(pool, 0);
        }
    }
}

}  // namespace rl

extern "C" {

const char* rl_last_error(void* ctx) {
    return ctx ? static_cast<Ctx*>(ctx)->last_error.c_str() : "null context";
}

rl_status rl_set_positions(void* ctx, const double* xyz, const uint8_t* signal) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(xyz != nullptr && signal != nullptr, RL_ERR_INVALID, "positions and signal types are required");
        for (uint32_t i = 0; i < c.n; ++i) {
            RL_CHECK(signal[i] <= 1, RL_ERR_INVALID, "signal type must be 0 or 1");
        }
        rl::upload(c.nr.signal, signal, c.n, c.stream);
        rl::build_octree(c, xyz);
        c.positions_set = true;
        c.stats.num_nodes = c.tree.num_nodes;
        c.stats.max_level = c.tree.max_level;
    });
}

rl_status rl_tree_info(void* ctx, uint64_t* num_nodes, uint32_t* max_level) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::require_tree(c);
        if (num_nodes) *num_nodes = c.tree.num_nodes;
        if (max_level) *max_level = c.tree.max_level;
    });
}

rl_status rl_dump_tree(void* ctx, int32_t* level, int32_t* neuron, uint8_t* child_mask, int32_t* first_child, double* bmin, double* bmax,
                       uint32_t* cnt_exc, uint32_t* cnt_inh, double* pos_exc, double* pos_inh) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::require_tree(c);
        rl::dump_tree(c, level, neuron, child_mask, first_child, bmin, bmax, cnt_exc, cnt_inh, pos_exc, pos_inh);
    });
}

rl_status rl_prepare_update_connectivity(void* ctx, const uint8_t* signal, const uint32_t* vacant_axons, const uint32_t* vacant_exc,
                                         const uint32_t* vacant_inh, const uint8_t* update) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::require_tree(c);
        RL_CHECK(vacant_axons && vacant_exc && vacant_inh, RL_ERR_INVALID, "vacant element arrays are required");
        if (signal) {
            rl::upload(c.nr.signal, signal, c.n, c.stream);
        }
        rl::upload(c.nr.search_vacant, vacant_axons, c.n, c.stream);
        rl::upload(c.nr.vacant[0], vacant_axons, c.n, c.stream);
        rl::upload(c.nr.vacant[1], vacant_exc, c.n, c.stream);
        rl::upload(c.nr.vacant[2], vacant_inh, c.n, c.stream);
        if (update) {
            rl::upload(c.nr.update, update, c.n, c.stream);
        } else {
            RL_CUDA_TRY(cudaMemcpyAsync(c.nr.update.p, c.nr.enabled.p, c.n, cudaMemcpyDeviceToDevice, c.stream));
        }
        rl::update_tree(c);
        rl::check_device_error(c, "prepare_update_connectivity");
    });
}

rl_status rl_find_targets(void* ctx, uint32_t step, rl_request* out, uint64_t capacity, uint64_t* count) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::require_tree(c);
        rl::run_search(c, step);
        const uint64_t m = c.search.num_requests;
        if (count) *count = m;
        const uint64_t k = m < capacity ? m : capacity;
        if (out && k) {
            std::vector<uint32_t> t(k), s(k), j(k), g(k);
            RL_CUDA_TRY(cudaMemcpyAsync(t.data(), c.search.req_tgt.p, k * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaMemcpyAsync(s.data(), c.search.req_src.p, k * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaMemcpyAsync(j.data(), c.search.req_j.p, k * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaMemcpyAsync(g.data(), c.search.req_sig.p, k * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
            for (uint64_t i = 0; i < k; ++i) {
                out[i] = rl_request{ t[i], s[i], j[i], g[i] };
            }
        }
    });
}

rl_status rl_update_connectivity(void* ctx, uint32_t step, rl_synapse* out, uint64_t capacity, uint64_t* created) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::require_tree(c);
        rl::run_search(c, step);
        const uint64_t before = c.graph.num_new;
        const uint64_t m = rl::run_connector(c, step);
        if (created) *created = m;
        const uint64_t k = m < capacity ? m : capacity;
        if (out && k) {
            std::vector<uint32_t> t(k), s(k);
            std::vector<int32_t> w(k);
            RL_CUDA_TRY(cudaMemcpyAsync(t.data(), c.graph.new_tgt.p + before, k * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaMemcpyAsync(s.data(), c.graph.new_src.p + before, k * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaMemcpyAsync(w.data(), c.graph.new_w.p + before, k * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
            for (uint64_t i = 0; i < k; ++i) {
                out[i] = rl_synapse{ t[i], s[i], w[i], 0u };
            }
        }
        rl::rebuild_graph(c);
    });
}

namespace {

// The connector over caller-given requests; bind_axons false leaves the
// sources' axons alone (process_requests on the rank owning the targets).
rl_status connect_given(void* ctx, uint32_t step, const rl_request* requests, uint64_t count, uint8_t* accepted, uint64_t* created,
                        bool bind_axons) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(count == 0 || requests != nullptr, RL_ERR_INVALID, "requests are required");
        RL_CHECK(count < ((uint64_t)1 << 32), RL_ERR_INVALID, "at most 2^32 - 1 requests per call");
        std::vector<uint32_t> t(count), s(count), j(count), g(count);
        for (uint64_t i = 0; i < count; ++i) {
            const rl_request& r = requests[i];
            RL_CHECK(r.target < c.n && r.source < c.n, RL_ERR_INVALID, "request " + std::to_string(i) + ": neuron id out of range");
            RL_CHECK(r.signal <= 1, RL_ERR_INVALID, "request " + std::to_string(i) + ": signal must be 0 or 1");
            t[i] = r.target;
            s[i] = r.source;
            j[i] = r.j;
            g[i] = r.signal;
        }
        rl::Search& S = c.search;
        if (count) {
            S.req_tgt.ensure(count);
            S.req_src.ensure(count);
            S.req_j.ensure(count);
            S.req_sig.ensure(count);
            rl::upload(S.req_tgt, t.data(), count, c.stream);
            rl::upload(S.req_src, s.data(), count, c.stream);
            rl::upload(S.req_j, j.data(), count, c.stream);
            rl::upload(S.req_sig, g.data(), count, c.stream);
        }
        S.num_requests = count;
        const uint64_t m = rl::run_connector(c, step, bind_axons);
        if (created) *created = m;
        if (accepted && count) {
            // the connector keeps its flags in processing order; cidx maps back to the request
            std::vector<uint32_t> flag(count), perm(count);
            RL_CUDA_TRY(cudaMemcpyAsync(flag.data(), S.accepted.p, count * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaMemcpyAsync(perm.data(), S.cidx.p, count * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
            for (uint64_t p = 0; p < count; ++p) {
                accepted[perm[p]] = flag[p] ? 1 : 0;
            }
        }
        S.num_requests = 0;
        rl::rebuild_graph(c);
    });
}

}  // namespace

rl_status rl_connect(void* ctx, uint32_t step, const rl_request* requests, uint64_t count, uint8_t* accepted, uint64_t* created) {
    return connect_given(ctx, step, requests, count, accepted, created, true);
}

rl_status rl_process_requests(void* ctx, uint32_t step, const rl_request* requests, uint64_t count, uint8_t* accepted, uint64_t* created) {
    return connect_given(ctx, step, requests, count, accepted, created, false);
}

rl_status rl_process_responses(void* ctx, const rl_request* requests, const uint8_t* accepted, const uint8_t* append, uint64_t count,
                               uint64_t* bound) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(count == 0 || (requests != nullptr && accepted != nullptr), RL_ERR_INVALID, "requests and accepted flags are required");
        std::vector<uint32_t> src;
        std::vector<uint32_t> et, es;
        std::vector<int32_t> ew;
        for (uint64_t i = 0; i < count; ++i) {
            const rl_request& r = requests[i];
            RL_CHECK(r.target < c.n && r.source < c.n, RL_ERR_INVALID, "request " + std::to_string(i) + ": neuron id out of range");
            RL_CHECK(r.signal <= 1, RL_ERR_INVALID, "request " + std::to_string(i) + ": signal must be 0 or 1");
            if (!accepted[i]) {
                continue;
            }
            src.push_back(r.source);
            if (append && append[i]) {
                et.push_back(r.target);
                es.push_back(r.source);
                ew.push_back(r.signal ? -1 : 1);
            }
        }
        if (bound) *bound = src.size();
        rl::bind_axons_host(c, src.size(), src.data());
        rl::add_edges_host(c, et.size(), et.data(), es.data(), ew.data());
    });
}

rl_status rl_set_elements(void* ctx, int type, const double* grown, const double* delta, const uint32_t* connected, const uint32_t* vacant) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(type >= 0 && type < 3, RL_ERR_INVALID, "element type must be 0, 1 or 2");
        if (rl::is_fp32(c)) {
            rl::f64_from_f32(c);
        }
        if (grown) rl::upload(c.nr.grown[type], grown, c.n, c.stream);
        if (delta) rl::upload(c.nr.delta[type], delta, c.n, c.stream);
        if (connected) rl::upload(c.nr.connected[type], connected, c.n, c.stream);
        if (vacant) rl::upload(c.nr.vacant[type], vacant, c.n, c.stream);
        if (rl::is_fp32(c)) {
            rl::f32_from_f64(c);
        }
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    });
}

rl_status rl_get_elements(void* ctx, int type, double* grown, double* delta, uint32_t* connected, uint32_t* vacant) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(type >= 0 && type < 3, RL_ERR_INVALID, "element type must be 0, 1 or 2");
        if (rl::is_fp32(c)) {
            rl::f64_from_f32(c);
        }
        if (grown) rl::download(grown, c.nr.grown[type], c.n, c.stream);
        if (delta) rl::download(delta, c.nr.delta[type], c.n, c.stream);
        if (connected) rl::download(connected, c.nr.connected[type], c.n, c.stream);
        if (vacant) rl::download(vacant, c.nr.vacant[type], c.n, c.stream);
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    });
}

rl_status rl_set_neurons(void* ctx, const double* x, const double* u, const double* calcium, const uint8_t* fired) {
    return rl::guarded(ctx, [&](Ctx& c) {
        if (rl::is_fp32(c)) {
            rl::f64_from_f32(c);
        }
        if (x) rl::upload(c.nr.x, x, c.n, c.stream);
        if (u) rl::upload(c.nr.u, u, c.n, c.stream);
        if (calcium) rl::upload(c.nr.calcium, calcium, c.n, c.stream);
        if (fired) rl::upload(c.nr.fired[c.nr.cur], fired, c.n, c.stream);
        if (rl::is_fp32(c)) {
            rl::f32_from_f64(c);
        }
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    });
}

rl_status rl_set_target_calcium(void* ctx, const double* target) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(target != nullptr, RL_ERR_INVALID, "null target");
        bool same = true;
        for (uint32_t i = 1; i < c.n && same; ++i) {
            same = target[i] == target[0];
        }
        c.target_uniform = same;
        if (same && c.n > 0) {
            c.cfg.target_calcium = target[0];
        }
        rl::drop_activity_graphs(c);  // captured intervals hold the growth-curve constants
        rl::upload(c.nr.target, target, c.n, c.stream);
        if (rl::is_fp32(c) && !same) {
            rl::target_f32_from_f64(c);  // the FP32 kernels read an FP32 copy
        }
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    });
}

rl_status rl_get_target_calcium(void* ctx, double* target) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(target != nullptr, RL_ERR_INVALID, "null target");
        rl::download(target, c.nr.target, c.n, c.stream);
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    });
}

rl_status rl_get_neurons(void* ctx, double* x, double* u, double* calcium, uint8_t* fired, double* input) {
    return rl::guarded(ctx, [&](Ctx& c) {
        if (rl::is_fp32(c)) {
            rl::f64_from_f32(c);
        }
        if (x) rl::download(x, c.nr.x, c.n, c.stream);
        if (u) rl::download(u, c.nr.u, c.n, c.stream);
        if (calcium) rl::download(calcium, c.nr.calcium, c.n, c.stream);
        if (fired) rl::download(fired, c.nr.fired[c.nr.cur], c.n, c.stream);
        if (input) rl::download(input, c.nr.input, c.n, c.stream);
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    });
}

rl_status rl_set_enabled(void* ctx, const uint8_t* enabled) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(enabled != nullptr, RL_ERR_INVALID, "enabled flags are required");
        // host -> staging on the upload stream (the caller's buffer is free when
        // that copy has landed), staging -> state in order on the context's
        // stream: the upload overlaps the work already queued there
        rl::ensure_copy_stream(c);
        if (c.enabled_stage.n < c.n) {
            c.enabled_stage.ensure(c.n);
            RL_CUDA_TRY(cudaStreamSynchronize(c.stream));  // the allocation is stream-ordered
        }
        if (c.stage_used) {
            RL_CUDA_TRY(cudaStreamWaitEvent(c.upload_stream, c.stage_free, 0));
        }
        RL_CUDA_TRY(cudaMemcpyAsync(c.enabled_stage.p, enabled, c.n, cudaMemcpyHostToDevice, c.upload_stream));
        RL_CUDA_TRY(cudaEventRecord(c.upload_done, c.upload_stream));
        RL_CUDA_TRY(cudaEventSynchronize(c.upload_done));
        RL_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.upload_done, 0));
        RL_CUDA_TRY(cudaMemcpyAsync(c.nr.enabled.p, c.enabled_stage.p, c.n, cudaMemcpyDeviceToDevice, c.stream));
        RL_CUDA_TRY(cudaEventRecord(c.stage_free, c.stream));
        c.stage_used = true;
    });
}

rl_status rl_snapshot_neurons(void* ctx, double* calcium, uint8_t* fired) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(calcium != nullptr || fired != nullptr, RL_ERR_INVALID, "no output buffer");
        rl::ensure_copy_stream(c);
        Ctx::SnapSlot& s = c.snap[c.snap_next];
        c.snap_next ^= 1;
        if (s.calcium.n < c.n) {
            s.calcium.ensure(c.n);
            s.fired.ensure(c.n);
            RL_CUDA_TRY(cudaStreamSynchronize(c.stream));  // the allocation is stream-ordered
        }
        if (s.pending) {
            rl::issue_snapshots(c);
            RL_CUDA_TRY(cudaStreamWaitEvent(c.stream, s.landed, 0));  // the slot's last copy has left it
        }
        if (calcium) {
            RL_CUDA_TRY(cudaMemcpyAsync(s.calcium.p, c.nr.calcium.p, c.n * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
        }
        if (fired) {
            RL_CUDA_TRY(cudaMemcpyAsync(s.fired.p, c.nr.fired[c.nr.cur].p, c.n, cudaMemcpyDeviceToDevice, c.stream));
        }
        RL_CUDA_TRY(cudaEventRecord(s.staged, c.stream));
        s.host_calcium = calcium;
        s.host_fired = fired;
        s.pending = true;
        s.issued = false;  // the host copy goes out with the next work
    });
}

rl_status rl_snapshot_wait(void* ctx) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::issue_snapshots(c);
        for (auto& s : c.snap) {
            if (s.pending) {
                RL_CUDA_TRY(cudaEventSynchronize(s.landed));
                s.pending = false;
            }
        }
    });
}

rl_status rl_add_edges(void* ctx, uint64_t m, const uint32_t* target, const uint32_t* source, const int32_t* weight) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(m == 0 || (target && source && weight), RL_ERR_INVALID, "edge arrays are required");
        rl::add_edges_host(c, m, target, source, weight);
    });
}

rl_status rl_get_edges(void* ctx, uint32_t* target, uint32_t* source, int32_t* weight, uint64_t capacity, uint64_t* count) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::rebuild_graph(c);
        const uint64_t m = c.graph.num_edges;
        std::vector<uint32_t> off(c.n + 1), s(m);
        std::vector<int32_t> w(m);
        RL_CUDA_TRY(cudaMemcpyAsync(off.data(), c.graph.offsets.p, (c.n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream));
        if (m) {
            RL_CUDA_TRY(cudaMemcpyAsync(s.data(), c.graph.src.p, m * 4, cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaMemcpyAsync(w.data(), c.graph.weight.p, m * 4, cudaMemcpyDeviceToHost, c.stream));
        }
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
        // aggregate (target, source) pairs, drop zero weights (NetworkGraph::add_edge)
        uint64_t k = 0;
        std::vector<std::pair<uint32_t, int32_t>> row;
        for (uint32_t t = 0; t < c.n; ++t) {
            row.clear();
            for (uint32_t e = off[t]; e < off[t + 1]; ++e) {
                row.emplace_back(s[e], w[e]);
            }
            std::sort(row.begin(), row.end());
            for (size_t a = 0; a < row.size();) {
                size_t b = a;
                int64_t sum = 0;
                while (b < row.size() && row[b].first == row[a].first) {
                    sum += row[b].second;
                    ++b;
                }
                if (sum != 0) {
                    if (k < capacity) {
                        if (target) target[k] = t;
                        if (source) source[k] = row[a].first;
                        if (weight) weight[k] = (int32_t)sum;
                    }
                    ++k;
                }
                a = b;
            }
        }
        if (count) *count = k;
    });
}

rl_status rl_activity_block(void* ctx, uint32_t first_step, uint32_t nsteps) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::rebuild_graph(c);
        rl::run_activity_block(c, first_step, nsteps);
    });
}

rl_status rl_plasticity_update(void* ctx, uint32_t step) {
    return rl::guarded(ctx, [&](Ctx& c) { rl::plasticity_update(c, step); });
}

rl_status rl_simulate(void* ctx, uint32_t first_step, uint32_t nsteps) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::require_tree(c);
        rl::rebuild_graph(c);
        const uint32_t interval = c.cfg.plasticity_interval;
        const uint64_t end = (uint64_t)first_step + nsteps;  // exclusive
        uint64_t step = first_step;
        while (step < end) {
            // activity up to and including the next plasticity step, then the update
            uint64_t stop = end;
            if (interval > 0) {
                const uint64_t next = ((step + interval - 1) / interval) * interval;  // first multiple >= step
                if (next < end) {
                    stop = next + 1;
                }
            }
            rl::run_activity_block(c, (uint32_t)step, (uint32_t)(stop - step));
            if (interval > 0 && (stop - 1) % interval == 0 && stop - 1 >= step) {
                rl::plasticity_update(c, (uint32_t)(stop - 1));
            }
            step = stop;
        }
    });
}

rl_status rl_synchronize(void* ctx) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
        rl::check_device_error(c, "synchronize");
    });
}

rl_status rl_candidate_weights(void* ctx, uint32_t source, int precision, uint32_t* nodes, double* weights, uint64_t capacity, uint64_t* count) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::require_tree(c);
        RL_CHECK(precision == RL_PRECISION_FP64 || precision == RL_PRECISION_FP32, RL_ERR_INVALID, "precision must be FP64 or FP32");
        std::vector<uint32_t> nd;
        std::vector<double> w;
        rl::candidate_weights(c, source, precision, nd, w);
        if (count) *count = nd.size();
        const uint64_t k = nd.size() < capacity ? nd.size() : capacity;
        for (uint64_t i = 0; i < k; ++i) {
            if (nodes) nodes[i] = nd[i];
            if (weights) weights[i] = w[i];
        }
    });
}

rl_status rl_set_stream(void* ctx, void* cuda_stream) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
        c.stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : c.own_stream;
    });
}

rl_status rl_set_graphs(void* ctx, int enable) {
    return rl::guarded(ctx, [&](Ctx& c) { c.use_graphs = enable != 0; });
}

rl_status rl_set_step_fusion(void* ctx, int enable) {
    return rl::guarded(ctx, [&](Ctx& c) { c.step_fusion = enable != 0; });
}

rl_status rl_set_profiling(void* ctx, int enable) {
    return rl::guarded(ctx, [&](Ctx& c) { c.timer.on = enable != 0; });
}

rl_status rl_get_phase_times(void* ctx, double* ms, uint64_t* counts) {
    return rl::guarded(ctx, [&](Ctx& c) {
        rl::resolve_timers(c);
        for (int p = 0; p < rl::PH_COUNT; ++p) {
            if (ms) ms[p] = c.timer.ms[p];
            if (counts) counts[p] = c.timer.count[p];
            c.timer.ms[p] = 0.0;
            c.timer.count[p] = 0;
        }
    });
}

rl_status rl_autotune(void* ctx, int mode) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(mode >= 0 && mode <= 2, RL_ERR_INVALID, "autotune mode must be 0, 1 or 2");
        c.tune.force = mode == 2;
        const int st = mode == 0 ? rl::TUNE_OFF : rl::TUNE_REQUESTED;
        c.tune.search_state = st;
        c.tune.act_state = st;
        if (mode != 0) {
            c.tune.search_ms.clear();
            c.tune.act_ms.clear();
            c.tune.search_by_class.clear();
        }
    });
}

rl_status rl_get_tuning(void* ctx, rl_tuning* out, float* search_ms, float* act_ms) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(out != nullptr, RL_ERR_INVALID, "null output");
        out->search_warps = c.tune.search.warps;
        out->search_hot = c.tune.search.hot;
        out->search_packet = c.tune.search.packet;
        out->search_cap = c.tune.search.cap;
        out->act_block = c.tune.act.block;
        out->act_persistent = c.tune.act.persistent;
        out->act_vec = c.tune.act.vec;
        out->tuned = (c.tune.search_state == rl::TUNE_DONE ? 1 : 0) | (c.tune.act_state == rl::TUNE_DONE ? 2 : 0);
        // times in candidate order (0 where none was taken)
        if (search_ms) {
            for (size_t v = 0; v < rl::search_variants().size(); ++v) {
                search_ms[v] = v < c.tune.search_ms.size() ? c.tune.search_ms[v] : 0.0f;
            }
        }
        if (act_ms) {
            for (size_t v = 0; v < rl::act_variants().size(); ++v) {
                act_ms[v] = v < c.tune.act_ms.size() ? c.tune.act_ms[v] : 0.0f;
            }
        }
    });
}

rl_status rl_set_tuning(void* ctx, const rl_tuning* t) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(t != nullptr, RL_ERR_INVALID, "null tuning");
        bool s_ok = false, a_ok = false;
        for (const auto& v : rl::search_variants()) {
            s_ok = s_ok || (v.warps == t->search_warps && v.hot == t->search_hot && v.packet == t->search_packet && v.cap == t->search_cap);
        }
        for (const auto& v : rl::act_variants()) {
            a_ok = a_ok || (v.block == t->act_block && v.persistent == t->act_persistent && v.vec == t->act_vec);
        }
        RL_CHECK(s_ok && a_ok, RL_ERR_INVALID, "not a candidate shape");
        RL_CHECK(rl::is_fp32(c) || t->act_vec <= 2, RL_ERR_INVALID, "the FP64 activity kernel runs one or two neurons per thread");
        c.tune.search = rl::SearchVariant{ t->search_warps, t->search_packet, t->search_cap, t->search_hot };
        c.tune.act = rl::ActVariant{ t->act_block, t->act_persistent, t->act_vec };
        c.tune.search_state = rl::TUNE_OFF;
        c.tune.act_state = rl::TUNE_OFF;
        rl::drop_activity_graphs(c);
    });
}

rl_status rl_ctx_memory(void* ctx, uint64_t* current, uint64_t* peak) {
    return rl::guarded(ctx, [&](Ctx& c) {
        if (current) *current = (uint64_t)c.device_bytes;
        if (peak) *peak = (uint64_t)c.device_peak;
    });
}

rl_status rl_get_stats(void* ctx, rl_stats* out) {
    return rl::guarded(ctx, [&](Ctx& c) {
        RL_CHECK(out != nullptr, RL_ERR_INVALID, "null output");
        *out = c.stats;
        if (c.tree.level_runs.p) {
            // level reductions the captured octree updates ran (conditional graph node)
            unsigned long long runs = 0;
            RL_CUDA_TRY(cudaMemcpyAsync(&runs, c.tree.level_runs.p, sizeof(runs), cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
            c.launches += runs - c.tree.level_runs_seen;
            c.tree.level_runs_seen = runs;
        }
        out->gpu_launches = c.launches;
        {
            unsigned long long touched = 0;
            RL_CUDA_TRY(cudaMemcpyAsync(&touched, c.counters.p, sizeof(touched), cudaMemcpyDeviceToHost, c.stream));
            RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
            out->nodes_touched = touched;
        }
        out->num_nodes = c.tree.num_nodes;
        out->max_level = c.tree.max_level;
    });
}

}  // extern "C"
