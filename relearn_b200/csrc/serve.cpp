// Serving form: a request loop that admits sweep runs against an HBM budget and
// runs them side by side on one GPU.
//
// The reference has no counterpart: its Simulation (sim/Simulation.cpp) runs
// one network per process.  Each request here is one network simulated for
// steps 1..steps through the same entry points a single-network caller uses
// (rl_ensemble_create, rl_set_positions, rl_set_elements, rl_simulate), so a
// request's result is the same whether it ran alone, beside other requests on
// the GPU, or packed with other small requests into one batched context (a
// network of a batched context evolves bit for bit as in a context of its
// own).
//
// Threads: `slots` workers, each running one context at a time on the stream
// the context owns.  The lock guards the queues and the budget only; every
// device call happens outside it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/relearn_b200.h"

namespace rl_serve {

using Clock = std::chrono::steady_clock;

// Device bytes a context holds, as an upper bound: a constant for the memory
// pool's granularity and the captured graphs; per neuron the state (positions,
// flags, x, u, calcium, target, input, two fired buffers, grown / delta /
// connected / vacant of three element types: 145 B, 28 B more in the FP32
// form), the octree at up to 2 nodes per neuron (140 B per node, 36 B more in
// the FP32 form) and the per-neuron search, connector and sort tables; per
// axon that can exist (the initial ones plus growth_rate[0] per neuron and
// step) the synapse it can form (synapse list, rebuild and sort scratch,
// out-edge permutation) and its search and connector entries.  Measured peaks
// (rl_ctx_memory) over uniform and clustered networks of 2,000 to 4,000,000
// neurons: 454-555 B per neuron (FP64) and 478-655 B (FP32) at 1.48 octree
// nodes per neuron, 55-100 B per axon of the bound; one launch per step adds
// the spike history (128 steps of one byte, rows padded to 16 bytes) and the
// two pushed-sum arrays (16 B FP64, 8 B FP32) per neuron.  The constants below
// leave headroom for trees of up to 2 nodes per neuron.
constexpr double kBaseBytes = 32.0 * 1024 * 1024;
constexpr double kNeuronBytes[2] = { 760.0, 830.0 };
constexpr double kAxonBytes[2] = { 120.0, 160.0 };

uint64_t footprint(const rl_config& base, const rl_network& net, double initial_axons, uint32_t steps) {
    const double n = net.num_neurons;
    const double axons = std::max(0.0, initial_axons) + n * std::max(0.0, net.growth_rate[0]) * steps;
    const int p = base.precision == RL_PRECISION_FP32 ? 1 : 0;
    return (uint64_t)(kBaseBytes + n * kNeuronBytes[p] + axons * kAxonBytes[p]);
}

struct Request {
    uint64_t id = 0;
    rl_network net{};
    std::vector<double> xyz;
    std::vector<uint8_t> signal;
    std::vector<double> grown[3];
    uint32_t steps = 0;
    bool keep = false;
    uint32_t bypassed = 0;
    rl_serve_done done{};
    // kept final state
    std::vector<double> x, u, calcium;
    std::vector<uint32_t> connected;
    std::vector<rl_synapse> synapses;
};

using ReqPtr = std::shared_ptr<Request>;

struct Server {
    rl_config base{};
    rl_serve_config sc{};
    Clock::time_point t0;
    std::mutex m;
    std::condition_variable cv_work;
    std::condition_variable cv_done;
    std::deque<ReqPtr> pending;
    std::deque<ReqPtr> finished;                   // not yet polled
    std::unordered_map<uint64_t, ReqPtr> kept;     // finished with keep_state
    uint64_t reserved = 0;
    uint64_t running = 0;
    uint64_t next_id = 1;
    bool stopping = false;
    std::vector<std::thread> workers;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    // Under the lock: the requests the next free slot takes, or none.
    std::vector<ReqPtr> take() {
        std::vector<ReqPtr> pack;
        const uint64_t budget = sc.hbm_budget_bytes;
        const uint32_t max_bypass = 2u * (uint32_t)sc.slots;
        size_t first = pending.size();
        for (size_t i = 0; i < pending.size(); ++i) {
            if (reserved + pending[i]->done.footprint_bytes <= budget) {
                first = i;
                break;
            }
            if (i == 0 && pending[0]->bypassed >= max_bypass) {
                return pack;  // the head has waited long enough: hold the rest back
            }
        }
        if (first == pending.size()) {
            return pack;
        }
        if (first > 0) {
            pending[0]->bypassed += 1;
        }
        ReqPtr lead = pending[first];
        pending.erase(pending.begin() + (std::ptrdiff_t)first);
        uint64_t fp = lead->done.footprint_bytes;
        pack.push_back(lead);
        if (sc.pack_networks > 1 && lead->net.num_neurons <= sc.pack_max_neurons) {
            for (size_t i = 0; i < pending.size() && (int)pack.size() < sc.pack_networks;) {
                const ReqPtr& q = pending[i];
                if (q->net.num_neurons <= sc.pack_max_neurons && q->steps == lead->steps && reserved + fp + q->done.footprint_bytes <= budget) {
                    fp += q->done.footprint_bytes;
                    pack.push_back(q);
                    pending.erase(pending.begin() + (std::ptrdiff_t)i);
                } else {
                    ++i;
                }
            }
        }
        reserved += fp;
        running += pack.size();
        return pack;
    }

    void worker() {
        for (;;) {
            std::vector<ReqPtr> pack;
            {
                std::unique_lock<std::mutex> lk(m);
                for (;;) {
                    if (!pending.empty()) {
                        pack = take();
                        if (!pack.empty()) {
                            break;
                        }
                    } else if (stopping) {
                        return;
                    }
                    cv_work.wait(lk);
                }
                const double t = now();
                for (auto& r : pack) {
                    r->done.t_admit = t;
                    r->done.pack_size = (uint32_t)pack.size();
                }
            }
            run(pack);
            {
                std::lock_guard<std::mutex> lk(m);
                for (auto& r : pack) {
                    reserved -= r->done.footprint_bytes;
                    running -= 1;
                    finished.push_back(r);
                    if (r->keep && r->done.status == RL_OK) {
                        kept[r->id] = r;
                    }
                }
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }

    void run(std::vector<ReqPtr>& pack) {
        std::vector<rl_network> nets;
        uint64_t total = 0;
        for (auto& r : pack) {
            nets.push_back(r->net);
            total += r->net.num_neurons;
        }
        void* ctx = nullptr;
        rl_status st = rl_ensemble_create(&base, nets.data(), (uint32_t)nets.size(), &ctx);
        auto fail = [&](rl_status s, const char* what) {
            std::fprintf(stderr, "relearn_b200 serve: %s failed: %s\n", what, ctx ? rl_last_error(ctx) : rl_status_string(s));
            for (auto& r : pack) {
                r->done.status = s;
                r->done.t_finish = now();
            }
            if (ctx) {
                rl_ctx_destroy(ctx);
            }
        };
        if (st != RL_OK) {
            ctx = nullptr;
            fail(st, "rl_ensemble_create");
            return;
        }
        {
            std::vector<double> xyz;
            std::vector<uint8_t> sig;
            xyz.reserve(3 * total);
            sig.reserve(total);
            for (auto& r : pack) {
                xyz.insert(xyz.end(), r->xyz.begin(), r->xyz.end());
                sig.insert(sig.end(), r->signal.begin(), r->signal.end());
            }
            if ((st = rl_set_positions(ctx, xyz.data(), sig.data())) != RL_OK) {
                return fail(st, "rl_set_positions");
            }
        }
        for (int t = 0; t < 3; ++t) {
            bool any = false;
            for (auto& r : pack) {
                any = any || !r->grown[t].empty();
            }
            if (!any) {
                continue;
            }
            std::vector<double> g(total, 0.0);
            uint64_t off = 0;
            for (auto& r : pack) {
                if (!r->grown[t].empty()) {
                    std::copy(r->grown[t].begin(), r->grown[t].end(), g.begin() + (std::ptrdiff_t)off);
                }
                off += r->net.num_neurons;
            }
            if ((st = rl_set_elements(ctx, t, g.data(), nullptr, nullptr, nullptr)) != RL_OK) {
                return fail(st, "rl_set_elements");
            }
        }
        if ((st = rl_set_graphs(ctx, sc.use_graphs)) != RL_OK) {
            return fail(st, "rl_set_graphs");
        }
        // One launch per activity step: a fused block of steps keeps its SMs
        // for the whole block (about a millisecond for a large network), which
        // holds back the kernels of the requests running beside it.
        if ((st = rl_set_step_fusion(ctx, 0)) != RL_OK) {
            return fail(st, "rl_set_step_fusion");
        }
        if ((st = rl_autotune(ctx, sc.autotune)) != RL_OK) {
            return fail(st, "rl_autotune");
        }
        if ((st = rl_simulate(ctx, 1, pack[0]->steps)) != RL_OK) {
            return fail(st, "rl_simulate");
        }
        bool keep_any = false;
        for (auto& r : pack) {
            keep_any = keep_any || r->keep;
        }
        // synapses, sorted by (target, source): each network's are one run
        uint64_t ne = 0;
        if ((st = rl_get_edges(ctx, nullptr, nullptr, nullptr, 0, &ne)) != RL_OK) {
            return fail(st, "rl_get_edges");
        }
        std::vector<uint32_t> tgt, src;
        std::vector<int32_t> w;
        if (keep_any || pack.size() > 1) {
            tgt.resize(ne ? ne : 1);
            src.resize(ne ? ne : 1);
            w.resize(ne ? ne : 1);
            if ((st = rl_get_edges(ctx, tgt.data(), src.data(), w.data(), ne, &ne)) != RL_OK) {
                return fail(st, "rl_get_edges");
            }
        } else {
            tgt.assign(ne ? ne : 1, 0u);  // one network: every synapse is its own
        }
        std::vector<double> x, u, ca;
        std::vector<uint32_t> con[3];
        if (keep_any) {
            x.resize(total);
            u.resize(total);
            ca.resize(total);
            if ((st = rl_get_neurons(ctx, x.data(), u.data(), ca.data(), nullptr, nullptr)) != RL_OK) {
                return fail(st, "rl_get_neurons");
            }
            for (int t = 0; t < 3; ++t) {
                con[t].resize(total);
                if ((st = rl_get_elements(ctx, t, nullptr, nullptr, con[t].data(), nullptr)) != RL_OK) {
                    return fail(st, "rl_get_elements");
                }
            }
        }
        uint64_t cur = 0, peak = 0;
        rl_ctx_memory(ctx, &cur, &peak);
        const double t_end = now();
        uint64_t first = 0;
        for (auto& r : pack) {
            const uint64_t n = r->net.num_neurons;
            const auto lo = std::lower_bound(tgt.begin(), tgt.begin() + (std::ptrdiff_t)ne, (uint32_t)first) - tgt.begin();
            const auto hi = std::lower_bound(tgt.begin(), tgt.begin() + (std::ptrdiff_t)ne, (uint32_t)(first + n)) - tgt.begin();
            r->done.num_synapses = (uint64_t)(hi - lo);
            r->done.device_peak_bytes = peak;
            r->done.status = RL_OK;
            r->done.t_finish = t_end;
            if (r->keep) {
                r->x.assign(x.begin() + (std::ptrdiff_t)first, x.begin() + (std::ptrdiff_t)(first + n));
                r->u.assign(u.begin() + (std::ptrdiff_t)first, u.begin() + (std::ptrdiff_t)(first + n));
                r->calcium.assign(ca.begin() + (std::ptrdiff_t)first, ca.begin() + (std::ptrdiff_t)(first + n));
                r->connected.resize(3 * n);
                for (int t = 0; t < 3; ++t) {
                    std::copy(con[t].begin() + (std::ptrdiff_t)first, con[t].begin() + (std::ptrdiff_t)(first + n), r->connected.begin() + (std::ptrdiff_t)(t * n));
                }
                r->synapses.resize((size_t)(hi - lo));
                for (auto k = lo; k < hi; ++k) {
                    r->synapses[(size_t)(k - lo)] = rl_synapse{ tgt[(size_t)k] - (uint32_t)first, src[(size_t)k] - (uint32_t)first, w[(size_t)k], 0u };
                }
            }
            first += n;
        }
        rl_ctx_destroy(ctx);
    }
};

}  // namespace rl_serve

extern "C" {

RL_API rl_status rl_serve_footprint(const rl_config* base, const rl_network* net, double initial_axons, uint32_t steps, uint64_t* bytes) {
    if (!base || !net || !bytes) {
        return RL_ERR_INVALID;
    }
    *bytes = rl_serve::footprint(*base, *net, initial_axons, steps);
    return RL_OK;
}

RL_API rl_status rl_serve_create(const rl_config* base, const rl_serve_config* sc, void** server) {
    if (!base || !sc || !server || sc->slots < 1 || sc->slots > 256 || sc->pack_networks < 1 || sc->hbm_budget_bytes == 0 || sc->autotune < 0 ||
        sc->autotune > 2) {
        return RL_ERR_INVALID;
    }
    *server = nullptr;
    auto* s = new (std::nothrow) rl_serve::Server();
    if (!s) {
        return RL_ERR_OOM;
    }
    s->base = *base;
    s->sc = *sc;
    s->t0 = rl_serve::Clock::now();
    try {
        for (int k = 0; k < sc->slots; ++k) {
            s->workers.emplace_back([s] { s->worker(); });
        }
    } catch (...) {
        {
            std::lock_guard<std::mutex> lk(s->m);
            s->stopping = true;
        }
        s->cv_work.notify_all();
        for (auto& t : s->workers) {
            t.join();
        }
        delete s;
        return RL_ERR_INVALID;
    }
    *server = s;
    return RL_OK;
}

RL_API rl_status rl_serve_submit(void* server, const rl_serve_request* req, uint64_t* id) {
    auto* s = static_cast<rl_serve::Server*>(server);
    if (!s || !req || !id || req->net.num_neurons == 0 || !req->xyz || !req->signal || req->steps == 0) {
        return RL_ERR_INVALID;
    }
    try {
        auto r = std::make_shared<rl_serve::Request>();
        const size_t n = req->net.num_neurons;
        r->net = req->net;
        r->xyz.assign(req->xyz, req->xyz + 3 * n);
        r->signal.assign(req->signal, req->signal + n);
        double axons = 0.0;
        for (int t = 0; t < 3; ++t) {
            if (req->grown[t]) {
                r->grown[t].assign(req->grown[t], req->grown[t] + n);
            }
        }
        for (double g : r->grown[0]) {
            axons += g;
        }
        r->steps = req->steps;
        r->keep = req->keep_state != 0;
        r->done.num_neurons = n;
        r->done.neuron_steps = (uint64_t)n * req->steps;
        r->done.footprint_bytes = rl_serve::footprint(s->base, req->net, axons, req->steps);
        if (r->done.footprint_bytes > s->sc.hbm_budget_bytes) {
            return RL_ERR_OOM;
        }
        {
            std::lock_guard<std::mutex> lk(s->m);
            if (s->stopping) {
                return RL_ERR_INVALID;
            }
            r->id = s->next_id++;
            r->done.id = r->id;
            r->done.t_submit = s->now();
            s->pending.push_back(r);
            *id = r->id;
        }
        s->cv_work.notify_one();
        return RL_OK;
    } catch (const std::bad_alloc&) {
        return RL_ERR_OOM;
    }
}

RL_API rl_status rl_serve_poll(void* server, rl_serve_done* out, uint64_t capacity, uint64_t* count, int32_t wait_ms) {
    auto* s = static_cast<rl_serve::Server*>(server);
    if (!s || !count || (capacity > 0 && !out)) {
        return RL_ERR_INVALID;
    }
    std::unique_lock<std::mutex> lk(s->m);
    if (s->finished.empty() && wait_ms > 0) {
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [s] { return !s->finished.empty(); });
    }
    uint64_t k = 0;
    while (k < capacity && !s->finished.empty()) {
        out[k++] = s->finished.front()->done;
        s->finished.pop_front();
    }
    *count = k;
    return RL_OK;
}

RL_API rl_status rl_serve_fetch(void* server, uint64_t id, double* x, double* u, double* calcium, uint32_t* connected, rl_synapse* synapses,
                                uint64_t capacity) {
    auto* s = static_cast<rl_serve::Server*>(server);
    if (!s) {
        return RL_ERR_INVALID;
    }
    rl_serve::ReqPtr r;
    {
        std::lock_guard<std::mutex> lk(s->m);
        auto it = s->kept.find(id);
        if (it == s->kept.end()) {
            return RL_ERR_INVALID;
        }
        r = it->second;
        s->kept.erase(it);
    }
    const size_t n = r->net.num_neurons;
    if (x) std::memcpy(x, r->x.data(), n * sizeof(double));
    if (u) std::memcpy(u, r->u.data(), n * sizeof(double));
    if (calcium) std::memcpy(calcium, r->calcium.data(), n * sizeof(double));
    if (connected) std::memcpy(connected, r->connected.data(), 3 * n * sizeof(uint32_t));
    if (synapses) {
        std::memcpy(synapses, r->synapses.data(), std::min<uint64_t>(capacity, r->synapses.size()) * sizeof(rl_synapse));
    }
    return RL_OK;
}

RL_API rl_status rl_serve_load(void* server, uint64_t* pending, uint64_t* running, uint64_t* reserved_bytes) {
    auto* s = static_cast<rl_serve::Server*>(server);
    if (!s) {
        return RL_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(s->m);
    if (pending) *pending = s->pending.size();
    if (running) *running = s->running;
    if (reserved_bytes) *reserved_bytes = s->reserved;
    return RL_OK;
}

RL_API rl_status rl_serve_destroy(void* server) {
    auto* s = static_cast<rl_serve::Server*>(server);
    if (!s) {
        return RL_ERR_INVALID;
    }
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) {
        t.join();
    }
    delete s;
    return RL_OK;
}

}  // extern "C"
