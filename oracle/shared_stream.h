// ORACLE — test infrastructure only.  Not part of the product; only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
//
// Oracle-side statement of the injected random stream and of the arithmetic
// that both sides must evaluate identically:
//   * Philox4x32-10 (Salmon et al., SC'11) keyed on
//     (seed, step, neuron, sub-index, stream, depth); replaces RandomHolder
//     (relearn/source/util/Random.h:70-284) at ProbabilityPicker.h:108-109,
//     Connector.cpp:71 and NormalActivityInputCPU.cpp:35.
//   * exp / log written from the mathematics (Tang's table-driven exp, atanh
//     series for log) standing in for glibc's std::exp (Gaussian.h:66,
//     GrowthCurves.h:51); set use_libm to evaluate std::exp / std::log instead.
//   * hypot of three arguments as libstdc++ evaluates it
//     (Vec3.hpp:549-551 -> std::hypot(x, y, z)).
//   * Wichura AS241 normal quantile for the background input.
// Build with -ffp-contract=off: no multiply-add contraction.  The polynomials of
// exp, log and the quantile use explicit std::fma (one rounding, as on the
// device); the reference's own formulas never do.  Built with -mfma so that
// std::fma is a single instruction.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle {

inline uint64_t bits_of(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
}
inline double from_bits(uint64_t u) {
    double x;
    std::memcpy(&x, &u, 8);
    return x;
}

struct Words {
    uint32_t w[4];
};

inline Words philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    uint32_t c[4] = { c0, c1, c2, c3 };
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c[0] = n0;
        c[1] = n1;
        c[2] = n2;
        c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return Words{ { c[0], c[1], c[2], c[3] } };
}

enum : uint32_t { S_BH = 1, S_CONNECT = 2, S_NOISE = 3, S_DELETE = 4, S_POISSON = 5 };

inline Words stream_draw(uint64_t seed, uint32_t step, uint32_t neuron, uint32_t sub, uint32_t stream, uint32_t depth) {
    return philox(step, neuron, sub, (stream << 24) | (depth & 0xFFFFFFu), (uint32_t)seed, (uint32_t)(seed >> 32));
}

inline uint64_t take53(const Words& r) {
    return ((uint64_t)r.w[0] << 21) | (uint64_t)(r.w[1] >> 11);
}
inline double unit_closed_open(const Words& r) {
    return (double)take53(r) * 0x1.0p-53;
}
inline double unit_open(const Words& r) {
    return ((double)take53(r) + 0.5) * 0x1.0p-53;
}
// Background input: one block per neuron pair (2m, 2m + 1) and step, words
// 0-1 for the even neuron and 2-3 for the odd one.
inline double noise_unit_open(uint64_t seed, uint32_t step, uint32_t neuron) {
    const Words r = stream_draw(seed, step, neuron >> 1, 0, S_NOISE, 0);
    const int o = (neuron & 1u) ? 2 : 0;
    const uint64_t b = ((uint64_t)r.w[o] << 21) | (uint64_t)(r.w[o + 1] >> 11);
    return ((double)b + 0.5) * 0x1.0p-53;
}
inline uint64_t take64(const Words& r) {
    return ((uint64_t)r.w[0] << 32) | (uint64_t)r.w[1];
}

// ---- exp
inline double times_pow2(double y, int k) {
    if (k > 1023) {
        y *= from_bits((uint64_t)(2046) << 52);
        k -= 1023;
        if (k > 1023) {
            k = 1023;
        }
        return y * from_bits((uint64_t)(k + 1023) << 52);
    }
    if (k < -1021) {
        const double t = y * from_bits((uint64_t)(k + 54 + 1023) << 52);
        return t * from_bits((uint64_t)(1023 - 54) << 52);
    }
    return y * from_bits((uint64_t)(k + 1023) << 52);
}

// 2^(j/64) for j = 0..63 as (nearest double, nearest double of the rest);
// the same 128 numbers as the product's table (relearn_b200/csrc/exp_table.py).
inline constexpr double kPow2Sixtyfourths[64][2] = {
    { 0x1.0000000000000p+0, 0x0.0p+0 },
    { 0x1.02c9a3e778061p+0, -0x1.19083535b085dp-56 },
    { 0x1.059b0d3158574p+0, 0x1.d73e2a475b465p-55 },
    { 0x1.0874518759bc8p+0, 0x1.186be4bb284ffp-57 },
    { 0x1.0b5586cf9890fp+0, 0x1.8a62e4adc610bp-54 },
    { 0x1.0e3ec32d3d1a2p+0, 0x1.03a1727c57b53p-59 },
    { 0x1.11301d0125b51p+0, -0x1.6c51039449b3ap-54 },
    { 0x1.1429aaea92de0p+0, -0x1.32fbf9af1369ep-54 },
    { 0x1.172b83c7d517bp+0, -0x1.19041b9d78a76p-55 },
    { 0x1.1a35beb6fcb75p+0, 0x1.e5b4c7b4968e4p-55 },
    { 0x1.1d4873168b9aap+0, 0x1.e016e00a2643cp-54 },
    { 0x1.2063b88628cd6p+0, 0x1.dc775814a8495p-55 },
    { 0x1.2387a6e756238p+0, 0x1.9b07eb6c70573p-54 },
    { 0x1.26b4565e27cddp+0, 0x1.2bd339940e9d9p-55 },
    { 0x1.29e9df51fdee1p+0, 0x1.612e8afad1255p-55 },
    { 0x1.2d285a6e4030bp+0, 0x1.0024754db41d5p-54 },
    { 0x1.306fe0a31b715p+0, 0x1.6f46ad23182e4p-55 },
    { 0x1.33c08b26416ffp+0, 0x1.32721843659a6p-54 },
    { 0x1.371a7373aa9cbp+0, -0x1.63aeabf42eae2p-54 },
    { 0x1.3a7db34e59ff7p+0, -0x1.5e436d661f5e3p-56 },
    { 0x1.3dea64c123422p+0, 0x1.ada0911f09ebcp-55 },
    { 0x1.4160a21f72e2ap+0, -0x1.ef3691c309278p-58 },
    { 0x1.44e086061892dp+0, 0x1.89b7a04ef80d0p-59 },
    { 0x1.486a2b5c13cd0p+0, 0x1.3c1a3b69062f0p-56 },
    { 0x1.4bfdad5362a27p+0, 0x1.d4397afec42e2p-56 },
    { 0x1.4f9b2769d2ca7p+0, -0x1.4b309d25957e3p-54 },
    { 0x1.5342b569d4f82p+0, -0x1.07abe1db13cadp-55 },
    { 0x1.56f4736b527dap+0, 0x1.9bb2c011d93adp-54 },
    { 0x1.5ab07dd485429p+0, 0x1.6324c054647adp-54 },
    { 0x1.5e76f15ad2148p+0, 0x1.ba6f93080e65ep-54 },
    { 0x1.6247eb03a5585p+0, -0x1.383c17e40b497p-54 },
    { 0x1.6623882552225p+0, -0x1.bb60987591c34p-54 },
    { 0x1.6a09e667f3bcdp+0, -0x1.bdd3413b26456p-54 },
    { 0x1.6dfb23c651a2fp+0, -0x1.bbe3a683c88abp-57 },
    { 0x1.71f75e8ec5f74p+0, -0x1.16e4786887a99p-55 },
    { 0x1.75feb564267c9p+0, -0x1.0245957316dd3p-54 },
    { 0x1.7a11473eb0187p+0, -0x1.41577ee04992fp-55 },
    { 0x1.7e2f336cf4e62p+0, 0x1.05d02ba15797ep-56 },
    { 0x1.82589994cce13p+0, -0x1.d4c1dd41532d8p-54 },
    { 0x1.868d99b4492edp+0, -0x1.fc6f89bd4f6bap-54 },
    { 0x1.8ace5422aa0dbp+0, 0x1.6e9f156864b27p-54 },
    { 0x1.8f1ae99157736p+0, 0x1.5cc13a2e3976cp-55 },
    { 0x1.93737b0cdc5e5p+0, -0x1.75fc781b57ebcp-57 },
    { 0x1.97d829fde4e50p+0, -0x1.d185b7c1b85d1p-54 },
    { 0x1.9c49182a3f090p+0, 0x1.c7c46b071f2bep-56 },
    { 0x1.a0c667b5de565p+0, -0x1.359495d1cd533p-54 },
    { 0x1.a5503b23e255dp+0, -0x1.d2f6edb8d41e1p-54 },
    { 0x1.a9e6b5579fdbfp+0, 0x1.0fac90ef7fd31p-54 },
    { 0x1.ae89f995ad3adp+0, 0x1.7a1cd345dcc81p-54 },
    { 0x1.b33a2b84f15fbp+0, -0x1.2805e3084d708p-57 },
    { 0x1.b7f76f2fb5e47p+0, -0x1.5584f7e54ac3bp-56 },
    { 0x1.bcc1e904bc1d2p+0, 0x1.23dd07a2d9e84p-55 },
    { 0x1.c199bdd85529cp+0, 0x1.11065895048ddp-55 },
    { 0x1.c67f12e57d14bp+0, 0x1.2884dff483cadp-54 },
    { 0x1.cb720dcef9069p+0, 0x1.503cbd1e949dbp-56 },
    { 0x1.d072d4a07897cp+0, -0x1.cbc3743797a9cp-54 },
    { 0x1.d5818dcfba487p+0, 0x1.2ed02d75b3707p-55 },
    { 0x1.da9e603db3285p+0, 0x1.c2300696db532p-54 },
    { 0x1.dfc97337b9b5fp+0, -0x1.1a5cd4f184b5cp-54 },
    { 0x1.e502ee78b3ff6p+0, 0x1.39e8980a9cc8fp-55 },
    { 0x1.ea4afa2a490dap+0, -0x1.e9c23179c2893p-54 },
    { 0x1.efa1bee615a27p+0, 0x1.dc7f486a4b6b0p-54 },
    { 0x1.f50765b6e4540p+0, 0x1.9d3e12dd8a18bp-54 },
    { 0x1.fa7c1819e90d8p+0, 0x1.74853f3a5931ep-55 },
};

// exp by Tang's table method (ACM TOMS 15(2), 1989): k = nearest integer to
// x * 64/ln2, r = x - k ln2/64 in two parts, exp(r) - 1 by the Taylor
// polynomial of degree 6, 2^(k mod 64 / 64) from the table, times 2^floor(k/64).
inline double own_exp(double x) {
    if (std::isnan(x)) {
        return x;
    }
    if (x > 709.782712893384) {
        return HUGE_VAL;
    }
    if (x < -745.1332191019412) {
        return 0.0;
    }
    const double ln2_hi = 0.6931467056274414;      // ln 2, low 32 mantissa bits cleared
    const double ln2_lo = 4.7493250390316726e-07;  // ln 2 - ln2_hi
    const double k = std::floor(x * 92.332482616893656768 + 0.5);
    const double r = std::fma(-k, ln2_lo / 64.0, x - k * (ln2_hi / 64.0));
    const int ki = static_cast<int>(k);
    const double* t = kPow2Sixtyfourths[ki & 63];
    // Horner from 1/720 down to 1/2, then r + r^2 * (...)
    static const double coef[5] = { 1.3888888888888889e-03, 8.3333333333333332e-03, 4.1666666666666664e-02, 1.6666666666666666e-01, 0.5 };
    double p = coef[0];
    for (int i = 1; i < 5; ++i) {
        p = std::fma(p, r, coef[i]);
    }
    p = std::fma(r * r, p, r);
    return times_pow2(t[0] + std::fma(t[0], p, t[1]), ki >> 6);
}

inline double own_log(double x) {
    const uint64_t b = bits_of(x);
    int e = (int)((b >> 52) & 0x7FF) - 1023;
    double m = from_bits((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
    if (m > 1.4142135623730951) {
        m *= 0.5;
        e += 1;
    }
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    double R = 1.0 / 23.0;
    for (int d = 21; d >= 3; d -= 2) {
        R = std::fma(R, z, 1.0 / (double)d);
    }
    R = R * z;
    const double two_s = 2.0 * s;
    const double logm = std::fma(two_s, R, two_s);
    const double ed = (double)e;
    return ed * 0.6931467056274414 + std::fma(ed, 4.7493250390316726e-07, logm);
}

// libstdc++ <cmath> three-argument hypot: a = max(|x|,|y|,|z|),
// a * sqrt((x/a)^2 + (y/a)^2 + (z/a)^2).
inline double hypot3(double x, double y, double z) {
    x = std::fabs(x);
    y = std::fabs(y);
    z = std::fabs(z);
    const double a = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (a == 0.0) {
        return 0.0;
    }
    return a * std::sqrt((x / a) * (x / a) + (y / a) * (y / a) + (z / a) * (z / a));
}

// AS241 (Wichura 1988) normal quantile; `lg` is the log to use.
template <typename Log>
inline double as241(double p, Log lg) {
    const double q = p - 0.5;
    if (std::fabs(q) <= 0.425) {
        const double r = 0.180625 - q * q;
        static const double A[8] = { 2.5090809287301226727e+3, 3.3430575583588128105e+4, 6.7265770927008700853e+4, 4.5921953931549871457e+4,
                                     1.3731693765509461125e+4, 1.9715909503065514427e+3, 1.3314166789178437745e+2, 3.3871328727963666080e+0 };
        static const double B[8] = { 5.2264952788528545610e+3, 2.8729085735721942674e+4, 3.9307895800092710610e+4, 2.1213794301586595867e+4,
                                     5.3941960214247511077e+3, 6.8718700749205790830e+2, 4.2313330701600911252e+1, 1.0 };
        double num = A[0];
        double den = B[0];
        for (int i = 1; i < 8; ++i) {
            num = std::fma(num, r, A[i]);
        }
        for (int i = 1; i < 8; ++i) {
            den = std::fma(den, r, B[i]);
        }
        return (num * q) / den;
    }
    double r = q < 0.0 ? p : 1.0 - p;
    r = std::sqrt(-lg(r));
    double num;
    double den;
    if (r <= 5.0) {
        r = r - 1.6;
        static const double C[8] = { 7.7454501427834140764e-4, 2.2723844989269184583e-2, 2.4178072517745061177e-1, 1.2704582524523683826e+0,
                                     3.6478483247632046050e+0, 5.7694972214606914055e+0, 4.6303378461565452959e+0, 1.4234371107496835773e+0 };
        static const double D[8] = { 1.0507500716444168432e-9, 5.4759380849953449460e-4, 1.5198666563616457197e-2, 1.4810397642748007459e-1,
                                     6.8976733498510000455e-1, 1.6763848301838038494e+0, 2.0531916266377588219e+0, 1.0 };
        num = C[0];
        den = D[0];
        for (int i = 1; i < 8; ++i) {
            num = std::fma(num, r, C[i]);
        }
        for (int i = 1; i < 8; ++i) {
            den = std::fma(den, r, D[i]);
        }
    } else {
        r = r - 5.0;
        static const double E[8] = { 2.0103343992922881327e-7, 2.7115555687434875782e-5, 1.2426609473880784386e-3, 2.6532189526576123093e-2,
                                     2.9656057182850489123e-1, 1.7848265399172913358e+0, 5.4637849111641143699e+0, 6.6579046435011037772e+0 };
        static const double F[8] = { 2.0442631033899397856e-15, 1.4215117583164458887e-7, 1.8463183175100546818e-5, 7.8686913114561325910e-4,
                                     1.4875361290850614853e-2, 1.3692988092273580531e-1, 5.9983220655588793769e-1, 1.0 };
        num = E[0];
        den = F[0];
        for (int i = 1; i < 8; ++i) {
            num = std::fma(num, r, E[i]);
        }
        for (int i = 1; i < 8; ++i) {
            den = std::fma(den, r, F[i]);
        }
    }
    const double x = num / den;
    return q < 0.0 ? -x : x;
}

}  // namespace oracle
