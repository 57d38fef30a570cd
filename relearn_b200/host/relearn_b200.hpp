// C++ host side of relearn-b200: the reference's plugin interfaces for the
// structural-plasticity path, implemented over the C ABI of
// include/relearn_b200.h (every call goes to the sm_100a kernels of
// librelearn_b200.so; there is no CPU fallback).
//
// Names, argument meaning and error behaviour follow the reference (paths
// relative to relearn/source of tuda-hpclab/relearn):
//   * Algorithm (algorithm/Algorithm.h:48-197): init, prepare_update_connectivity
//     with spans of signal types and vacant element counts, update_connectivity
//     returning a ConnectivityUpdateResult, get_algorithm_type; BarnesHut is the
//     --algorithm barnes-hut implementation.
//   * NeuronModel (neurons/models/NeuronModelBase.h): update_electrical_activity
//     per step and the per-neuron getters; ActivityModel runs the --neuron-model
//     of the context (izhikevich, poisson, fitzhughnagumo, aeif) with the
//     calcium and synaptic-element updates Neurons drives every step
//     (neurons/Neurons.cpp:351-384).
//   * Simulation::simulate (sim/Simulation.cpp:388-480): steps 1 .. number_steps + 1,
//     plasticity every plasticity_update_step steps.
//   * RelearnException::check / fail (util/RelearnException.h): every non-OK
//     status becomes a RelearnException carrying the library's message.
#pragma once

#include <cstdint>
#include <fstream>
#include <memory>
#include <span>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/relearn_b200.h"

namespace relearn_b200 {

class RelearnException : public std::runtime_error {
public:
    explicit RelearnException(const std::string& what, rl_status status = RL_ERR_INVALID)
        : std::runtime_error(what), status_(status) { }

    static void check(bool condition, const std::string& message) {
        if (!condition) {
            throw RelearnException(message);
        }
    }

    [[noreturn]] static void fail(const std::string& message) { throw RelearnException(message); }

    rl_status status() const { return status_; }

private:
    rl_status status_;
};

enum class SignalType : uint8_t { Excitatory = RL_EXCITATORY, Inhibitory = RL_INHIBITORY };
enum class ElementType : int { Axon = RL_AXON, DendriteExcitatory = RL_DENDRITE_EXC, DendriteInhibitory = RL_DENDRITE_INH };
enum class AlgorithmEnum { BarnesHut };
enum class NeuronModelEnum : int {
    Izhikevich = RL_MODEL_IZHIKEVICH,
    Poisson = RL_MODEL_POISSON,
    FitzHughNagumo = RL_MODEL_FITZHUGH_NAGUMO,
    AEIF = RL_MODEL_AEIF
};

using number_neurons_type = uint64_t;
using counter_type = uint32_t;  // RelearnTypes::counter_type
using step_type = uint32_t;

namespace detail {
inline void check_status(rl_status s, void* ctx, const char* what) {
    if (s != RL_OK) {
        std::string msg = std::string(what) + ": " + rl_status_string(s);
        if (ctx) {
            msg += " (" + std::string(rl_last_error(ctx)) + ")";
        }
        throw RelearnException(msg, s);
    }
}
}  // namespace detail

// Model parameters of one network; the reference defaults come from
// rl_config_default.
struct Parameters {
    rl_config cfg{};

    static Parameters defaults(uint32_t number_neurons, double side) {
        Parameters p;
        rl_config_default(&p.cfg, number_neurons, side);
        return p;
    }
};

// One network on one GPU: owns the library context.
class Context {
public:
    explicit Context(const Parameters& p) {
        void* h = nullptr;
        detail::check_status(rl_ctx_create(&p.cfg, &h), nullptr, "rl_ctx_create");
        ctx_ = h;
        n_ = p.cfg.num_neurons;
        interval_ = p.cfg.plasticity_interval;
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    Context(Context&& o) noexcept : ctx_(std::exchange(o.ctx_, nullptr)), n_(o.n_), interval_(o.interval_) { }
    ~Context() {
        if (ctx_) {
            rl_ctx_destroy(ctx_);
        }
    }

    void* handle() const { return ctx_; }
    number_neurons_type size() const { return n_; }
    uint32_t plasticity_interval() const { return interval_; }
    void check(rl_status s, const char* what) const { detail::check_status(s, ctx_, what); }

    rl_stats stats() const {
        rl_stats st{};
        check(rl_get_stats(ctx_, &st), "rl_get_stats");
        return st;
    }

private:
    void* ctx_ = nullptr;
    number_neurons_type n_ = 0;
    uint32_t interval_ = 100;
};

struct SynapseCreationRequest {
    uint32_t target;
    uint32_t source;
    SignalType signal_type;
};

struct PlasticLocalSynapse {
    uint32_t target;
    uint32_t source;
    int32_t weight;
};

struct ConnectivityUpdateResult {
    uint64_t number_synapses_created = 0;
    std::vector<PlasticLocalSynapse> local_synapses;
};

// Algorithm: the connectivity update of the structural-plasticity model.
class Algorithm {
public:
    virtual ~Algorithm() = default;
    virtual void init(number_neurons_type number_neurons) = 0;
    virtual void prepare_update_connectivity(std::span<const SignalType> signal_types, std::span<const counter_type> vacant_axons,
                                             std::span<const counter_type> vacant_excitatory_dendrites,
                                             std::span<const counter_type> vacant_inhibitory_dendrites) = 0;
    [[nodiscard]] virtual ConnectivityUpdateResult update_connectivity(number_neurons_type number_neurons) = 0;
    [[nodiscard]] virtual AlgorithmEnum get_algorithm_type() const = 0;
};

// --algorithm barnes-hut on the GPU.
class BarnesHut final : public Algorithm {
public:
    // positions: 3 * n coordinates (x, y, z per neuron) in the simulation box.
    BarnesHut(Context& ctx, std::span<const double> positions, std::span<const SignalType> signal_types)
        : ctx_(ctx), positions_(positions.begin(), positions.end()), signal_(signal_types.size()) {
        for (size_t i = 0; i < signal_types.size(); ++i) {
            signal_[i] = static_cast<uint8_t>(signal_types[i]);
        }
    }

    void init(number_neurons_type number_neurons) override {
        RelearnException::check(number_neurons == ctx_.size(), "BarnesHut::init: number of neurons does not match the context");
        RelearnException::check(positions_.size() == 3 * number_neurons && signal_.size() == number_neurons,
                                "BarnesHut::init: positions or signal types have the wrong size");
        ctx_.check(rl_set_positions(ctx_.handle(), positions_.data(), signal_.data()), "rl_set_positions");
    }

    void prepare_update_connectivity(std::span<const SignalType> signal_types, std::span<const counter_type> vacant_axons,
                                     std::span<const counter_type> vacant_excitatory_dendrites,
                                     std::span<const counter_type> vacant_inhibitory_dendrites) override {
        const size_t n = ctx_.size();
        RelearnException::check(signal_types.size() == n && vacant_axons.size() == n && vacant_excitatory_dendrites.size() == n &&
                                    vacant_inhibitory_dendrites.size() == n,
                                "BarnesHut::prepare_update_connectivity: spans must have one entry per neuron");
        std::vector<uint8_t> sig(n);
        for (size_t i = 0; i < n; ++i) {
            sig[i] = static_cast<uint8_t>(signal_types[i]);
        }
        ctx_.check(rl_prepare_update_connectivity(ctx_.handle(), sig.data(), vacant_axons.data(), vacant_excitatory_dendrites.data(),
                                                  vacant_inhibitory_dendrites.data(), nullptr),
                   "rl_prepare_update_connectivity");
        pending_axons_ = 0;
        for (counter_type v : vacant_axons) {
            pending_axons_ += v;
        }
    }

    // Searches for every vacant axon of the last prepare_update_connectivity
    // and connects the accepted requests (the caller's step number keys the
    // random stream).
    ConnectivityUpdateResult update_connectivity_at(step_type step) {
        std::vector<rl_synapse> out(pending_axons_ ? pending_axons_ : 1);
        uint64_t created = 0;
        ctx_.check(rl_update_connectivity(ctx_.handle(), step, out.data(), out.size(), &created), "rl_update_connectivity");
        ConnectivityUpdateResult r;
        r.number_synapses_created = created;
        r.local_synapses.reserve(created);
        for (uint64_t k = 0; k < created && k < out.size(); ++k) {
            r.local_synapses.push_back({ out[k].target, out[k].source, out[k].weight });
        }
        return r;
    }

    ConnectivityUpdateResult update_connectivity(number_neurons_type number_neurons) override {
        RelearnException::check(number_neurons == ctx_.size(), "BarnesHut::update_connectivity: number of neurons does not match the context");
        return update_connectivity_at(step_);
    }

    // The requests of one search pass without connecting them
    // (BarnesHut::find_target_neurons).
    std::vector<SynapseCreationRequest> find_target_neurons(step_type step) {
        std::vector<rl_request> out(pending_axons_ ? pending_axons_ : 1);
        uint64_t count = 0;
        ctx_.check(rl_find_targets(ctx_.handle(), step, out.data(), out.size(), &count), "rl_find_targets");
        std::vector<SynapseCreationRequest> r;
        r.reserve(count);
        for (uint64_t k = 0; k < count && k < out.size(); ++k) {
            r.push_back({ out[k].target, out[k].source, out[k].signal ? SignalType::Inhibitory : SignalType::Excitatory });
        }
        return r;
    }

    void set_step(step_type step) { step_ = step; }

    AlgorithmEnum get_algorithm_type() const override { return AlgorithmEnum::BarnesHut; }

private:
    Context& ctx_;
    std::vector<double> positions_;
    std::vector<uint8_t> signal_;
    uint64_t pending_axons_ = 0;
    step_type step_ = 0;
};

// NeuronModel: the electrical activity between plasticity updates.
class NeuronModel {
public:
    virtual ~NeuronModel() = default;
    virtual void update_electrical_activity(step_type step) = 0;
    [[nodiscard]] virtual std::vector<double> get_x() const = 0;
    [[nodiscard]] virtual std::vector<uint8_t> get_fired() const = 0;
    [[nodiscard]] virtual NeuronModelEnum get_model_type() const = 0;
};

// The --neuron-model chosen for the context (izhikevich, poisson,
// fitzhughnagumo or aeif) with the calcium and growth updates of each step.
class ActivityModel final : public NeuronModel {
public:
    ActivityModel(Context& ctx, NeuronModelEnum type) : ctx_(ctx), type_(type) { }

    void update_electrical_activity(step_type step) override {
        ctx_.check(rl_activity_block(ctx_.handle(), step, 1), "rl_activity_block");
    }

    // Steps first .. first + count - 1 at once (one launch each, or one CUDA
    // graph per full plasticity interval).
    void update_electrical_activity_block(step_type first, uint32_t count) {
        ctx_.check(rl_activity_block(ctx_.handle(), first, count), "rl_activity_block");
    }

    std::vector<double> get_x() const override { return neurons().x; }
    std::vector<uint8_t> get_fired() const override { return neurons().fired; }
    std::vector<double> get_calcium() const { return neurons().calcium; }
    NeuronModelEnum get_model_type() const override { return type_; }

    struct State {
        std::vector<double> x, u, calcium, input;
        std::vector<uint8_t> fired;
    };

    State neurons() const {
        const size_t n = ctx_.size();
        State s{ std::vector<double>(n), std::vector<double>(n), std::vector<double>(n), std::vector<double>(n), std::vector<uint8_t>(n) };
        ctx_.check(rl_get_neurons(ctx_.handle(), s.x.data(), s.u.data(), s.calcium.data(), s.fired.data(), s.input.data()), "rl_get_neurons");
        return s;
    }

private:
    Context& ctx_;
    NeuronModelEnum type_;
};

// Simulation::simulate on one GPU.
class Simulation {
public:
    Simulation(const Parameters& params, std::span<const double> positions, std::span<const SignalType> signal_types,
               const std::string& algorithm = "barnes-hut", const std::string& neuron_model = "izhikevich")
        : ctx_(checked(params, algorithm, neuron_model)), algorithm_(ctx_, positions, signal_types),
          model_(ctx_, static_cast<NeuronModelEnum>(checked(params, algorithm, neuron_model).cfg.neuron_model)) {
        algorithm_.init(ctx_.size());
    }

    // Initial grown elements of one type (--synaptic-elements-lower-bound /
    // --synaptic-elements-upper-bound draw these); vacant = floor(grown).
    void set_initial_elements(ElementType type, std::span<const double> grown) {
        const size_t n = ctx_.size();
        RelearnException::check(grown.size() == n, "Simulation::set_initial_elements: one value per neuron");
        std::vector<double> delta(n, 0.0);
        std::vector<uint32_t> connected(n, 0u), vacant(n);
        for (size_t i = 0; i < n; ++i) {
            vacant[i] = static_cast<uint32_t>(grown[i]);
        }
        ctx_.check(rl_set_elements(ctx_.handle(), static_cast<int>(type), grown.data(), delta.data(), connected.data(), vacant.data()),
                   "rl_set_elements");
    }

    // Runs number_steps + 1 steps, as the reference does.
    void simulate(step_type number_steps) {
        const uint32_t count = number_steps + 1;
        ctx_.check(rl_simulate(ctx_.handle(), step_, count), "rl_simulate");
        step_ += count;
    }

    struct Synapses {
        std::vector<uint32_t> target, source;
        std::vector<int32_t> weight;
    };

    Synapses synapses() const {
        uint64_t m = 0;
        ctx_.check(rl_get_edges(ctx_.handle(), nullptr, nullptr, nullptr, 0, &m), "rl_get_edges");
        Synapses s{ std::vector<uint32_t>(m), std::vector<uint32_t>(m), std::vector<int32_t>(m) };
        ctx_.check(rl_get_edges(ctx_.handle(), s.target.data(), s.source.data(), s.weight.data(), m, &m), "rl_get_edges");
        return s;
    }

    std::vector<uint32_t> connected(ElementType type) const {
        std::vector<uint32_t> c(ctx_.size());
        ctx_.check(rl_get_elements(ctx_.handle(), static_cast<int>(type), nullptr, nullptr, c.data(), nullptr), "rl_get_elements");
        return c;
    }

    Context& context() { return ctx_; }
    BarnesHut& algorithm() { return algorithm_; }
    ActivityModel& neuron_model() { return model_; }
    step_type current_step() const { return step_; }

private:
    // The parameters with the --neuron-model chosen by name (relearn.cpp:326-333).
    static Parameters checked(const Parameters& p, const std::string& algorithm, const std::string& neuron_model) {
        if (algorithm != "barnes-hut") {
            throw RelearnException("algorithm '" + algorithm + "' is not built here (have barnes-hut)", RL_ERR_UNSUPPORTED);
        }
        Parameters q = p;
        if (neuron_model == "izhikevich") {
            q.cfg.neuron_model = RL_MODEL_IZHIKEVICH;
        } else if (neuron_model == "poisson") {
            q.cfg.neuron_model = RL_MODEL_POISSON;
        } else if (neuron_model == "fitzhughnagumo") {
            q.cfg.neuron_model = RL_MODEL_FITZHUGH_NAGUMO;
        } else if (neuron_model == "aeif") {
            q.cfg.neuron_model = RL_MODEL_AEIF;
        } else {
            throw RelearnException("neuron model '" + neuron_model + "' is not built here (have aeif, fitzhughnagumo, izhikevich, poisson)",
                                   RL_ERR_UNSUPPORTED);
        }
        return q;
    }

    Context ctx_;
    BarnesHut algorithm_;
    ActivityModel model_;
    step_type step_ = 1;
};

}  // namespace relearn_b200

namespace relearn_b200 {

// A positions file in the reference's format (NeuronIO::read_neuron_positions_and_signals,
// io/NeuronIO.cpp:229-300): '#' comment lines, then one neuron per line as
// "id x y z signal" with ids 1, 2, ... in order, non-negative coordinates and
// signal "in" for inhibitory (anything else excitatory).
struct LoadedNeurons {
    std::vector<double> positions;  // x, y, z per neuron
    std::vector<SignalType> signal_types;
    double maximum[3] = { 0.0, 0.0, 0.0 };
    // simulation box from the "# Minimum x:" .. "# Maximum z:" comment lines
    // (NeuronIO::parse_additional_position_information, io/NeuronIO.cpp:107-148;
    // MultipleSubdomainsFromFile sets the box from them), when all six are present
    bool has_box = false;
    double box_min[3] = { 0.0, 0.0, 0.0 };
    double box_max[3] = { 0.0, 0.0, 0.0 };
};

inline LoadedNeurons read_neuron_positions_and_signals(const std::string& path) {
    std::ifstream file(path);
    RelearnException::check(file.good(), "read_neuron_positions_and_signals: cannot open '" + path + "'");
    LoadedNeurons out;
    uint64_t expected = 0;
    std::string line;
    static const char* const box_keys[6] = { "# Minimum x:", "# Minimum y:", "# Minimum z:", "# Maximum x:", "# Maximum y:", "# Maximum z:" };
    bool box_seen[6] = { false, false, false, false, false, false };
    double box[6] = { 0.0, 0.0, 0.0, 0.0, 0.0, 0.0 };
    while (std::getline(file, line)) {
        if (line.empty()) {
            continue;
        }
        if (line[0] == '#') {
            for (int k = 0; k < 6; ++k) {
                const std::string key = box_keys[k];
                if (!box_seen[k] && line.compare(0, key.size(), key) == 0) {
                    box[k] = std::stod(line.substr(key.size()));  // the first matching comment counts
                    box_seen[k] = true;
                }
            }
            continue;
        }
        std::istringstream ss(line);
        uint64_t id = 0;
        double x = 0, y = 0, z = 0;
        std::string signal;
        if (!(ss >> id >> x >> y >> z >> signal)) {
            continue;  // the reference skips lines it cannot parse
        }
        RelearnException::check(x >= 0 && y >= 0 && z >= 0, "read_neuron_positions_and_signals: negative position of neuron " + std::to_string(id));
        RelearnException::check(id >= 1, "read_neuron_positions_and_signals: neuron id is too small");
        RelearnException::check(id - 1 == expected, "read_neuron_positions_and_signals: loaded neuron " + std::to_string(id - 1) + " but expected " +
                                                        std::to_string(expected));
        ++expected;
        out.positions.insert(out.positions.end(), { x, y, z });
        out.signal_types.push_back(signal == "in" ? SignalType::Inhibitory : SignalType::Excitatory);
        out.maximum[0] = x > out.maximum[0] ? x : out.maximum[0];
        out.maximum[1] = y > out.maximum[1] ? y : out.maximum[1];
        out.maximum[2] = z > out.maximum[2] ? z : out.maximum[2];
    }
    out.has_box = box_seen[0] && box_seen[1] && box_seen[2] && box_seen[3] && box_seen[4] && box_seen[5];
    if (out.has_box) {
        for (int a = 0; a < 3; ++a) {
            out.box_min[a] = box[a];
            out.box_max[a] = box[3 + a];
        }
    }
    return out;
}

}  // namespace relearn_b200

#include <algorithm>
#include <numeric>
#include <tuple>

namespace relearn_b200 {

// Plastic synapses of one rank in the reference's network files
// (NeuronIO::read_in_synapses / write_in_synapses, io/NeuronIO.cpp:793-860 and
// 935-1030): '#' comment lines, then "target_rank target_id source_rank
// source_id weight plastic" with ids from 1.  This path runs one rank and
// plastic synapses only: other ranks and static synapses are refused.
struct NetworkSynapses {
    std::vector<uint32_t> target, source;
    std::vector<int32_t> weight;
};

inline NetworkSynapses read_in_network(const std::string& path, number_neurons_type number_neurons) {
    std::ifstream file(path);
    RelearnException::check(file.good(), "read_in_network: cannot open '" + path + "'");
    NetworkSynapses out;
    std::string line;
    while (std::getline(file, line)) {
        if (line.empty() || line[0] == '#') {
            continue;
        }
        std::istringstream ss(line);
        int64_t target_rank = 0, source_rank = 0, weight = 0;
        uint64_t target_id = 0, source_id = 0;
        int plastic = 0;
        if (!(ss >> target_rank >> target_id >> source_rank >> source_id >> weight >> plastic)) {
            continue;  // the reference skips lines it cannot parse
        }
        RelearnException::check(target_rank == 0 && source_rank == 0, "read_in_network: synapses of other ranks are not supported on one GPU");
        RelearnException::check(target_id >= 1 && target_id <= number_neurons && source_id >= 1 && source_id <= number_neurons,
                                "read_in_network: neuron id out of range in '" + line + "'");
        RelearnException::check(weight != 0, "read_in_network: weight was 0");
        if (!plastic) {
            throw RelearnException("read_in_network: static synapses are not supported by this path", RL_ERR_UNSUPPORTED);
        }
        out.target.push_back((uint32_t)(target_id - 1));
        out.source.push_back((uint32_t)(source_id - 1));
        out.weight.push_back((int32_t)weight);
    }
    return out;
}

// rank_0_in_network.txt (sorted by target, then source) and
// rank_0_out_network.txt (sorted by source, then target) in `directory`.
inline void write_network_files(const std::string& directory, number_neurons_type number_neurons, const NetworkSynapses& s) {
    std::vector<size_t> order(s.target.size());
    std::iota(order.begin(), order.end(), size_t{ 0 });
    for (int side = 0; side < 2; ++side) {
        const bool in = side == 0;
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            return in ? std::tie(s.target[a], s.source[a]) < std::tie(s.target[b], s.source[b])
                      : std::tie(s.source[a], s.target[a]) < std::tie(s.source[b], s.target[b]);
        });
        const std::string path = directory + (in ? "/rank_0_in_network.txt" : "/rank_0_out_network.txt");
        std::ofstream f(path);
        RelearnException::check(f.good(), "write_network_files: cannot write '" + path + "'");
        f << "# " << number_neurons << "\n# <target rank> <target neuron id>\t<source rank> <source neuron id>\t<weight>\t<plastic>\n";
        for (size_t k : order) {
            f << "0 " << s.target[k] + 1 << "\t0 " << s.source[k] + 1 << "\t" << s.weight[k] << "\t1\n";
        }
    }
}

// Loads synapses into a simulation as Neurons::init_synaptic_elements does
// (neurons/Neurons.cpp:105-127): every synapse adds |weight| connected and
// grown elements to its source's axons and to its target's excitatory or
// inhibitory dendrites (by the weight's sign).
inline void load_network(Simulation& sim, const NetworkSynapses& s) {
    Context& ctx = sim.context();
    const size_t n = ctx.size();
    const size_t m = s.target.size();
    ctx.check(rl_add_edges(ctx.handle(), m, s.target.data(), s.source.data(), s.weight.data()), "rl_add_edges");
    std::vector<uint32_t> add[3] = { std::vector<uint32_t>(n, 0u), std::vector<uint32_t>(n, 0u), std::vector<uint32_t>(n, 0u) };
    for (size_t k = 0; k < m; ++k) {
        const uint32_t a = (uint32_t)(s.weight[k] < 0 ? -s.weight[k] : s.weight[k]);
        add[RL_AXON][s.source[k]] += a;
        add[s.weight[k] < 0 ? RL_DENDRITE_INH : RL_DENDRITE_EXC][s.target[k]] += a;
    }
    for (int t = 0; t < 3; ++t) {
        std::vector<double> grown(n), delta(n);
        std::vector<uint32_t> connected(n), vacant(n);
        ctx.check(rl_get_elements(ctx.handle(), t, grown.data(), delta.data(), connected.data(), vacant.data()), "rl_get_elements");
        for (size_t i = 0; i < n; ++i) {
            connected[i] += add[t][i];
            grown[i] += (double)add[t][i];
        }
        ctx.check(rl_set_elements(ctx.handle(), t, grown.data(), delta.data(), connected.data(), vacant.data()), "rl_set_elements");
    }
}

}  // namespace relearn_b200

namespace relearn_b200 {

// Initial and target calcium per neuron from a calcium file of the reference
// (CalciumIO::load_initial_and_target_function, io/CalciumIO.cpp:27-130):
// lines "<description> <initial> <target>", the description "default" (at most
// once) or ';'-separated "<rank>:<neuron id>" with 1-based ids (rank -1 = this
// rank; one rank here).  A neuron gets at most one pair; the others take the
// default.  Neuron groups are not supported.
struct CalciumValues {
    std::vector<double> initial, target;
};

inline CalciumValues read_calcium_file(const std::string& path, number_neurons_type number_neurons) {
    std::ifstream file(path);
    RelearnException::check(file.good(), "read_calcium_file: cannot open '" + path + "'");
    CalciumValues v{ std::vector<double>(number_neurons, 0.0), std::vector<double>(number_neurons, 0.0) };
    std::vector<uint8_t> seen(number_neurons, 0);
    bool has_default = false;
    double def_initial = 0.0, def_target = 0.0;
    std::string line;
    while (std::getline(file, line)) {
        if (!line.empty() && line[0] == '#') {
            continue;
        }
        std::istringstream ss(line);
        std::string description;
        double initial = 0.0, target = 0.0;
        if (!(ss >> description >> initial >> target)) {
            continue;
        }
        if (description == "default") {
            RelearnException::check(!has_default, "read_calcium_file: more than one default");
            has_default = true;
            def_initial = initial;
            def_target = target;
            continue;
        }
        std::istringstream items(description);
        std::string item;
        while (std::getline(items, item, ';')) {
            const auto colon = item.find(':');
            RelearnException::check(colon != std::string::npos, "read_calcium_file: neuron groups are not supported: " + item);
            const long rank = std::stol(item.substr(0, colon));
            const long long id = std::stoll(item.substr(colon + 1));
            RelearnException::check(rank == 0 || rank == -1, "read_calcium_file: one rank only: " + item);
            RelearnException::check(id >= 1 && (uint64_t)id <= number_neurons, "read_calcium_file: neuron id out of range (ids are 1-based): " + item);
            RelearnException::check(!seen[id - 1], "read_calcium_file: neuron " + std::to_string(id) + " assigned twice");
            seen[id - 1] = 1;
            v.initial[id - 1] = initial;
            v.target[id - 1] = target;
        }
    }
    for (size_t i = 0; i < number_neurons; ++i) {
        if (!seen[i]) {
            RelearnException::check(has_default, "read_calcium_file: neurons without values and no default");
            v.initial[i] = def_initial;
            v.target[i] = def_target;
        }
    }
    return v;
}

// Applies a calcium file's values: the calcium state starts at `initial`, the
// growth curves use `target`.
inline void set_calcium(Simulation& sim, const CalciumValues& v) {
    Context& ctx = sim.context();
    ctx.check(rl_set_neurons(ctx.handle(), nullptr, nullptr, v.initial.data(), nullptr), "rl_set_neurons");
    ctx.check(rl_set_target_calcium(ctx.handle(), v.target.data()), "rl_set_target_calcium");
}

}  // namespace relearn_b200
