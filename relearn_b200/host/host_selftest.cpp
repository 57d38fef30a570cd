// Host-side checks of the C++ layer that need no GPU: the positions-file
// reader (the reference's format and its error cases) and the translation of
// status codes into RelearnException.  Prints "ok" and exits 0 on success.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>

#include "relearn_b200.hpp"

using namespace relearn_b200;

#define EXPECT(cond)                                                        \
    do {                                                                    \
        if (!(cond)) {                                                      \
            std::fprintf(stderr, "%s:%d: failed: %s\n", __FILE__, __LINE__, #cond); \
            std::exit(1);                                                   \
        }                                                                   \
    } while (0)

template <typename F>
rl_status throws(F&& f) {
    try {
        f();
    } catch (const RelearnException& e) {
        return e.status();
    }
    return RL_OK;
}

int main(int argc, char** argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    const std::string good = dir + "/positions_good.txt";
    {
        std::ofstream f(good);
        f << "# comment line\n"
          << "# another\n"
          << "1 10.5 20.25 30.125 ex\n"
          << "\n"
          << "2 1 2 3 in\n"
          << "this line is skipped\n"
          << "3 0.1 0.2 0.3 ex\n";
    }
    const LoadedNeurons n = read_neuron_positions_and_signals(good);
    EXPECT(n.signal_types.size() == 3);
    EXPECT(n.positions.size() == 9);
    EXPECT(n.positions[0] == 10.5 && n.positions[1] == 20.25 && n.positions[2] == 30.125);
    EXPECT(n.signal_types[0] == SignalType::Excitatory && n.signal_types[1] == SignalType::Inhibitory);
    EXPECT(n.maximum[0] == 10.5 && n.maximum[1] == 20.25 && n.maximum[2] == 30.125);

    const std::string gap = dir + "/positions_gap.txt";
    {
        std::ofstream f(gap);
        f << "1 1 1 1 ex\n3 2 2 2 ex\n";
    }
    EXPECT(throws([&] { read_neuron_positions_and_signals(gap); }) == RL_ERR_INVALID);
    const std::string neg = dir + "/positions_negative.txt";
    {
        std::ofstream f(neg);
        f << "1 -1 1 1 ex\n";
    }
    EXPECT(throws([&] { read_neuron_positions_and_signals(neg); }) == RL_ERR_INVALID);
    EXPECT(throws([&] { read_neuron_positions_and_signals(dir + "/does_not_exist.txt"); }) == RL_ERR_INVALID);

    // network files: write, read back, refuse what one GPU does not run
    {
        NetworkSynapses s{ { 2, 0, 1, 2 }, { 1, 2, 2, 0 }, { 1, -1, 2, 1 } };
        write_network_files(dir, 3, s);
        const NetworkSynapses r = read_in_network(dir + "/rank_0_in_network.txt", 3);
        EXPECT(r.target.size() == 4);
        // sorted by (target, source)
        EXPECT(r.target[0] == 0 && r.source[0] == 2 && r.weight[0] == -1);
        EXPECT(r.target[1] == 1 && r.source[1] == 2 && r.weight[1] == 2);
        EXPECT(r.target[3] == 2 && r.source[3] == 1 && r.weight[3] == 1);
        const NetworkSynapses o = read_in_network(dir + "/rank_0_out_network.txt", 3);
        EXPECT(o.target.size() == 4 && o.source[0] == 0 && o.target[0] == 2);
        std::ofstream(dir + "/static.txt") << "0 1 0 2 1 0\n";
        EXPECT(throws([&] { read_in_network(dir + "/static.txt", 3); }) == RL_ERR_UNSUPPORTED);
        std::ofstream(dir + "/rank1.txt") << "1 1 0 2 1 1\n";
        EXPECT(throws([&] { read_in_network(dir + "/rank1.txt", 3); }) == RL_ERR_INVALID);
        std::ofstream(dir + "/range.txt") << "0 4 0 2 1 1\n";
        EXPECT(throws([&] { read_in_network(dir + "/range.txt", 3); }) == RL_ERR_INVALID);
    }

    // calcium files
    {
        std::ofstream(dir + "/calcium.txt") << "# comment\ndefault 0.1 0.7\n0:2;-1:4 0.3 0.9\n0:1 0.0 0.5\n";
        const CalciumValues v = read_calcium_file(dir + "/calcium.txt", 5);
        EXPECT(v.initial[0] == 0.0 && v.target[0] == 0.5);
        EXPECT(v.initial[1] == 0.3 && v.target[1] == 0.9 && v.initial[3] == 0.3 && v.target[3] == 0.9);
        EXPECT(v.initial[2] == 0.1 && v.target[2] == 0.7 && v.initial[4] == 0.1);
        std::ofstream(dir + "/calcium_twice.txt") << "default 0 0.7\n0:1 0 1\n0:1 0 1\n";
        EXPECT(throws([&] { read_calcium_file(dir + "/calcium_twice.txt", 5); }) == RL_ERR_INVALID);
        std::ofstream(dir + "/calcium_nodefault.txt") << "0:1 0 1\n";
        EXPECT(throws([&] { read_calcium_file(dir + "/calcium_nodefault.txt", 5); }) == RL_ERR_INVALID);
        std::ofstream(dir + "/calcium_group.txt") << "default 0 0.7\nexcitatory 0 1\n";
        EXPECT(throws([&] { read_calcium_file(dir + "/calcium_group.txt", 5); }) == RL_ERR_INVALID);
    }

    // plugin names the reference offers but this path does not build
    Parameters p = Parameters::defaults(3, 100.0);
    EXPECT(p.cfg.plasticity_interval == 100 && p.cfg.theta == 0.3 && p.cfg.sigma == 750.0);
    EXPECT(throws([&] { Simulation s(p, n.positions, n.signal_types, "naive"); }) == RL_ERR_UNSUPPORTED);
    EXPECT(throws([&] { Simulation s(p, n.positions, n.signal_types, "barnes-hut", "hodgkin-huxley"); }) == RL_ERR_UNSUPPORTED);

    // without a device the context cannot be created: the status comes back as an exception
    if (argc > 2 && std::string(argv[2]) == "--no-device") {
        EXPECT(throws([&] { Context c(p); }) == RL_ERR_DEVICE);
    }
    std::printf("ok\n");
    return 0;
}
