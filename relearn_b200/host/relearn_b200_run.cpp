// relearn_b200_run: runs Simulation::simulate for one network on the GPU
// through the C++ host classes, with the reference's command-line names for
// the options of this path (relearn.cpp:380-660) and defaults of the library
// (rl_config_default, the reference's defaults).  Prints one JSON line with the
// run's counters; --output-prefix writes the final calcium (one value per
// line, %.17g) and the synapses ("target source weight").
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "relearn_b200.hpp"

using namespace relearn_b200;

namespace {

// SplitMix64 (Steele, Lea and Flood, OOPSLA 2014): the driver's generator for
// positions without --file and for the initial elements, simple enough to be
// reproduced exactly by other tools (the tests do).
struct SplitMix64 {
    uint64_t x;
    uint64_t next() {
        x += 0x9E3779B97F4A7C15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0, 1)
};

struct Options {
    uint32_t num_neurons = 2000;
    std::string file;
    uint32_t steps = 20000;
    std::string algorithm = "barnes-hut";
    std::string neuron_model = "izhikevich";
    double side = 0.0;
    double lower = 0.0, upper = 0.0;
    std::string precision = "fp64";
    std::string output_prefix;
    std::string graph;           // directory with rank_0_in_network.txt
    std::string file_calcium;    // initial and target calcium per neuron
    std::string output_network;  // directory for the final network files
    rl_config cfg{};
};

void usage() {
    std::printf(
        "usage: relearn_b200_run [--num-neurons N | --file POSITIONS] -s STEPS [options]\n"
        "  reference options: --algorithm barnes-hut, --neuron-model izhikevich, -t/--theta, --gaussian-sigma,\n"
        "    --gaussian-mu, --kernel-type gaussian|gamma|linear|weibull, --gamma-k, --gamma-theta, --linear-cutoff,\n"
        "    --weibull-k, --weibull-b,\n"
        "    -r/--random-seed, --plasticity-update-step, --synapse-conductance, --background-activity-mean,\n"
        "    --background-activity-stddev, --beta, --calcium-decay, --target-ca, --initial-ca,\n"
        "    --growth-rate-axon, --growth-rate-dendrite-exc, --growth-rate-dendrite-inh, --min-calcium-axons,\n"
        "    --min-calcium-excitatory-dendrites, --min-calcium-inhibitory-dendrites, --retract-ratio,\n"
        "    --synaptic-elements-lower-bound, --synaptic-elements-upper-bound\n"
        "    -g/--graph DIR (rank_0_in_network.txt with plastic synapses), --file-calcium FILE\n"
        "  added here: --izhikevich-a/-b/-c/-d, --side UM (cube edge; default: the box of the positions file's\n"
        "    '# Minimum/Maximum' header lines, else the largest coordinate),\n"
        "    --precision fp64|fp32, --output-prefix P (final calcium and synapses as text),\n"
        "    --output-network DIR (final rank_0_in_network.txt and rank_0_out_network.txt)\n");
}

bool parse(int argc, char** argv, Options& o) {
    rl_config_default(&o.cfg, 1, 1.0);
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) {
                throw RelearnException("missing value for " + a);
            }
            return argv[++i];
        };
        auto num = [&]() { return std::stod(next()); };
        rl_config& c = o.cfg;
        if (a == "--help" || a == "-h") {
            usage();
            return false;
        } else if (a == "--num-neurons") {
            o.num_neurons = (uint32_t)std::stoul(next());
        } else if (a == "--file" || a == "-f") {
            o.file = next();
        } else if (a == "--steps" || a == "-s") {
            o.steps = (uint32_t)std::stoul(next());
        } else if (a == "--algorithm" || a == "-a") {
            o.algorithm = next();
        } else if (a == "--neuron-model") {
            o.neuron_model = next();
        } else if (a == "--theta" || a == "-t") {
            c.theta = num();
        } else if (a == "--gaussian-sigma") {
            c.sigma = num();
        } else if (a == "--gaussian-mu") {
            c.mu = num();
        } else if (a == "--kernel-type") {
            const std::string t = next();
            if (t == "gaussian") {
                c.kernel_type = RL_KERNEL_GAUSSIAN;
            } else if (t == "gamma") {
                c.kernel_type = RL_KERNEL_GAMMA;
            } else if (t == "linear") {
                c.kernel_type = RL_KERNEL_LINEAR;
            } else if (t == "weibull") {
                c.kernel_type = RL_KERNEL_WEIBULL;
            } else {
                throw RelearnException("unknown kernel type " + t + " (gaussian, gamma, linear, weibull)");
            }
        } else if (a == "--gamma-k" || a == "--weibull-k") {
            c.kernel_k = num();
        } else if (a == "--gamma-theta" || a == "--weibull-b") {
            c.kernel_scale = num();
        } else if (a == "--linear-cutoff") {
            c.linear_cutoff = num();
        } else if (a == "--random-seed" || a == "-r") {
            c.seed = std::stoull(next());
        } else if (a == "--plasticity-update-step") {
            c.plasticity_interval = (uint32_t)std::stoul(next());
        } else if (a == "--synapse-conductance") {
            c.conductance = num();
        } else if (a == "--background-activity-mean") {
            c.noise_mean = num();
        } else if (a == "--background-activity-stddev") {
            c.noise_stddev = num();
        } else if (a == "--beta") {
            c.beta = num();
        } else if (a == "--calcium-decay") {
            c.tau_c = num();
        } else if (a == "--target-ca") {
            c.target_calcium = num();
        } else if (a == "--initial-ca") {
            c.initial_calcium = num();
        } else if (a == "--growth-rate-axon") {
            c.growth_rate[RL_AXON] = num();
        } else if (a == "--growth-rate-dendrite-exc") {
            c.growth_rate[RL_DENDRITE_EXC] = num();
        } else if (a == "--growth-rate-dendrite-inh") {
            c.growth_rate[RL_DENDRITE_INH] = num();
        } else if (a == "--min-calcium-axons") {
            c.min_calcium[RL_AXON] = num();
        } else if (a == "--min-calcium-excitatory-dendrites") {
            c.min_calcium[RL_DENDRITE_EXC] = num();
        } else if (a == "--min-calcium-inhibitory-dendrites") {
            c.min_calcium[RL_DENDRITE_INH] = num();
        } else if (a == "--retract-ratio") {
            const double r = num();
            c.retract_ratio[0] = c.retract_ratio[1] = c.retract_ratio[2] = r;
        } else if (a == "--synaptic-elements-lower-bound") {
            o.lower = num();
        } else if (a == "--synaptic-elements-upper-bound") {
            o.upper = num();
        } else if (a == "--izhikevich-a") {
            c.iz_a = num();
        } else if (a == "--izhikevich-b") {
            c.iz_b = num();
        } else if (a == "--izhikevich-c") {
            c.iz_c = num();
        } else if (a == "--izhikevich-d") {
            c.iz_d = num();
        } else if (a == "--side") {
            o.side = num();
        } else if (a == "--precision") {
            o.precision = next();
        } else if (a == "--output-prefix") {
            o.output_prefix = next();
        } else if (a == "--graph" || a == "-g") {
            o.graph = next();
        } else if (a == "--file-calcium") {
            o.file_calcium = next();
        } else if (a == "--output-network") {
            o.output_network = next();
        } else {
            throw RelearnException("unknown option " + a);
        }
    }
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        Options o;
        if (!parse(argc, argv, o)) {
            return 0;
        }
        LoadedNeurons neurons;
        if (!o.file.empty()) {
            neurons = read_neuron_positions_and_signals(o.file);
            o.num_neurons = (uint32_t)neurons.signal_types.size();
        } else {
            // uniform in a cube at one neuron per 1000 um^3, 20 % inhibitory
            const double side = o.side > 0 ? o.side : std::cbrt(1000.0 * o.num_neurons);
            SplitMix64 gen{ o.cfg.seed };
            for (uint32_t i = 0; i < o.num_neurons; ++i) {
                const double x = side * gen.uniform(), y = side * gen.uniform(), z = side * gen.uniform();
                neurons.positions.insert(neurons.positions.end(), { x, y, z });
                neurons.signal_types.push_back(i % 5 == 4 ? SignalType::Inhibitory : SignalType::Excitatory);
            }
            neurons.maximum[0] = neurons.maximum[1] = neurons.maximum[2] = side;
        }
        RelearnException::check(o.num_neurons > 0, "no neurons");
        Parameters p;
        p.cfg = o.cfg;
        p.cfg.num_neurons = o.num_neurons;
        if (o.side <= 0 && neurons.has_box) {
            // the box of the file's header, as MultipleSubdomainsFromFile::read_neurons_from_file
            // (sim/file/MultipleSubdomainsFromFile.cpp:60-90) sets it
            for (int a = 0; a < 3; ++a) {
                p.cfg.box_min[a] = neurons.box_min[a];
                p.cfg.box_max[a] = neurons.box_max[a];
            }
        } else {
            double side = o.side;
            if (side <= 0) {
                side = std::max(neurons.maximum[0], std::max(neurons.maximum[1], neurons.maximum[2]));
                side = std::nextafter(side, 2 * side + 1);  // the box must contain the largest coordinate
            }
            for (int a = 0; a < 3; ++a) {
                p.cfg.box_min[a] = 0.0;
                p.cfg.box_max[a] = side;
            }
        }
        RelearnException::check(o.precision == "fp64" || o.precision == "fp32", "--precision must be fp64 or fp32");
        p.cfg.precision = o.precision == "fp32" ? RL_PRECISION_FP32 : RL_PRECISION_FP64;

        Simulation sim(p, neurons.positions, neurons.signal_types, o.algorithm, o.neuron_model);
        if (o.upper > 0.0) {
            // grown elements lower + (upper - lower) * u per type and neuron, in that order
            RelearnException::check(o.lower <= o.upper, "--synaptic-elements-lower-bound must not exceed the upper bound");
            SplitMix64 gen{ o.cfg.seed + 17 };
            for (int t = 0; t < 3; ++t) {
                std::vector<double> grown(o.num_neurons);
                for (auto& g : grown) {
                    g = o.lower + (o.upper - o.lower) * gen.uniform();
                }
                sim.set_initial_elements(static_cast<ElementType>(t), grown);
            }
        }
        if (!o.graph.empty()) {
            load_network(sim, read_in_network(o.graph + "/rank_0_in_network.txt", o.num_neurons));
        }
        if (!o.file_calcium.empty()) {
            set_calcium(sim, read_calcium_file(o.file_calcium, o.num_neurons));
        }
        const auto t0 = std::chrono::steady_clock::now();
        sim.simulate(o.steps);
        const auto calcium = sim.neuron_model().get_calcium();
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const auto syn = sim.synapses();
        const rl_stats st = sim.context().stats();
        double mean_ca = 0.0;
        for (double c : calcium) {
            mean_ca += c;
        }
        mean_ca /= (double)calcium.size();
        std::printf(
            "{\"neurons\": %u, \"steps\": %u, \"seconds\": %.6f, \"neuron_steps_per_s\": %.6e, \"mean_calcium\": %.17g, \"synapses\": %zu, "
            "\"synapses_created\": %llu, \"synapses_deleted\": %llu, \"searches\": %llu, \"plasticity_updates\": %llu}\n",
            o.num_neurons, o.steps + 1, secs, (double)o.num_neurons * (o.steps + 1) / secs, mean_ca, syn.target.size(),
            (unsigned long long)st.synapses_created, (unsigned long long)st.synapses_deleted, (unsigned long long)st.searches,
            (unsigned long long)st.plasticity_updates);
        if (!o.output_network.empty()) {
            write_network_files(o.output_network, o.num_neurons, NetworkSynapses{ syn.target, syn.source, syn.weight });
        }
        if (!o.output_prefix.empty()) {
            FILE* f = std::fopen((o.output_prefix + "_calcium.txt").c_str(), "w");
            RelearnException::check(f != nullptr, "cannot write " + o.output_prefix + "_calcium.txt");
            for (double c : calcium) {
                std::fprintf(f, "%.17g\n", c);
            }
            std::fclose(f);
            f = std::fopen((o.output_prefix + "_synapses.txt").c_str(), "w");
            RelearnException::check(f != nullptr, "cannot write " + o.output_prefix + "_synapses.txt");
            for (size_t k = 0; k < syn.target.size(); ++k) {
                std::fprintf(f, "%u %u %d\n", syn.target[k], syn.source[k], syn.weight[k]);
            }
            std::fclose(f);
        }
        return 0;
    } catch (const RelearnException& e) {
        std::fprintf(stderr, "relearn_b200_run: %s\n", e.what());
        return 2;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "relearn_b200_run: %s\n", e.what());
        return 2;
    }
}
