// Host build of the product's shared arithmetic header, for the agreement
// test against the oracle (compiled with g++ -ffp-contract=off).
#include <cmath>
#include "../../relearn_b200/csrc/rl_math.cuh"

extern "C" {
double probe_exp(double x) { return rl::rl_exp(x); }
double probe_exp_flat(double x) { return rl::rl_exp_flat(x); }
double probe_exp_flat_nonpos(double x) { return rl::rl_exp_flat_nonpos(x); }
double probe_log(double x) { return rl::rl_log(x); }
double probe_hypot3(double x, double y, double z) { return rl::rl_hypot3(x, y, z); }
// libstdc++'s own three-argument std::hypot, which the reference calls
double probe_std_hypot3(double x, double y, double z) { return std::hypot(x, y, z); }
// rl_hypot3 against libstdc++'s std::hypot(x, y, z) on n vectors drawn by
// xorshift from `seed`: coordinate differences of cells and neurons in boxes
// up to 20,000 um, small and mixed magnitudes, equal components; returns the
// number of vectors whose results differ in any bit.
long probe_hypot_sweep(long n, unsigned long long seed) {
    unsigned long long st = seed * 0x9E3779B97F4A7C15ull + 1;
    auto next = [&]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return st;
    };
    auto u01 = [&]() { return (double)(next() >> 11) * 0x1p-53; };
    long bad = 0;
    for (long i = 0; i < n; ++i) {
        double v[3];
        for (int k = 0; k < 3; ++k) {
            switch ((i + k) % 4) {
                case 0: v[k] = (u01() - 0.5) * 40000.0; break;
                case 1: v[k] = (u01() - 0.5) * 2.0; break;
                case 2: v[k] = std::ldexp(1.0 + u01(), (int)(next() % 120) - 60); break;
                default: v[k] = (double)(int64_t)(next() % 2001) - 1000.0; break;
            }
        }
        if (i % 7 == 0) {
            v[1] = v[0];  // equal magnitudes
        }
        const double a = rl::rl_hypot3(v[0], v[1], v[2]);
        const double b = std::hypot(v[0], v[1], v[2]);
        if (a != b) {
            ++bad;
        }
    }
    return bad;
}
double probe_quantile(double p) { return rl::normal_quantile(p); }
double probe_normal(unsigned long long seed, unsigned step, unsigned neuron, double mean, double sd) {
    return rl::background_normal(seed, step, neuron, mean, sd);
}
void probe_philox(unsigned c0, unsigned c1, unsigned c2, unsigned c3, unsigned k0, unsigned k1, unsigned* out) {
    const rl::u32x4 r = rl::philox4x32_10(rl::u32x4{ c0, c1, c2, c3 }, k0, k1);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    out[3] = r.w;
}
double probe_next_up(double t) { return rl::next_up_eps(t); }
double probe_kernel_prob(int type, double d, double mu, double scale, double km1, double a, double b, double cutoff, int inf) {
    return rl::rl_kernel_prob(type, d, mu, scale, km1, a, b, cutoff, inf);
}
}
