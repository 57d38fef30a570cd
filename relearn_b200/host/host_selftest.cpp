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

    // plugin names the reference offers but this path does not build
    Parameters p = Parameters::defaults(3, 100.0);
    EXPECT(p.cfg.plasticity_interval == 100 && p.cfg.theta == 0.3 && p.cfg.sigma == 750.0);
    EXPECT(throws([&] { Simulation s(p, n.positions, n.signal_types, "naive"); }) == RL_ERR_UNSUPPORTED);
    EXPECT(throws([&] { Simulation s(p, n.positions, n.signal_types, "barnes-hut", "poisson"); }) == RL_ERR_UNSUPPORTED);

    // without a device the context cannot be created: the status comes back as an exception
    if (argc > 2 && std::string(argv[2]) == "--no-device") {
        EXPECT(throws([&] { Context c(p); }) == RL_ERR_DEVICE);
    }
    std::printf("ok\n");
    return 0;
}
