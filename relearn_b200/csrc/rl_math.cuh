// Shared arithmetic for the structural-plasticity hot path.
//
// Every function here is __host__ __device__ and uses only IEEE-754 binary64
// additions, multiplications, divisions, square roots and explicit fused
// multiply-adds (each correctly rounded on both sides) plus integer bit
// manipulation.  The translation units that include this header are compiled
// without multiply-add contraction (nvcc -fmad=false, g++ -ffp-contract=off),
// so host and device produce the same bits for the same inputs.  That is what
// makes the FP64 path bit-exact against the CPU oracle.  The fused
// multiply-adds are only in the functions written here (the polynomials of
// exp, log and the normal quantile), never in the reference's own formulas.
//
// Contents
//   * rl_philox4x32_10 : Philox4x32-10 counter-based generator (Salmon, Moraes,
//     Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).  It
//     replaces the reference's thread_local std::mt19937 draws
//     (relearn/source/util/Random.h:245-283) by a stream keyed on
//     (seed, step, neuron, sub-index, stream/depth).
//   * rl_exp, rl_log   : exponential (Tang's table-driven method) and natural
//     log (atanh series) written from the mathematics.
//     They stand in for std::exp in GaussianDistributionKernel::get_probability
//     (relearn/source/algorithm/Kernel/Gaussian.h:62-68) and
//     gaussian_growth_curve (relearn/source/neurons/synaptic_elements/GrowthCurves.h:30-53).
//   * rl_hypot3        : the three-argument hypot of libstdc++ (scale by the
//     largest magnitude, then sqrt of the sum of scaled squares), which the
//     reference reaches through Vec3::calculate_2_norm
//     (relearn/external/cpp-utility/data-structure/Vec3.hpp:549-551).
//   * rl_normal_quantile: Wichura's AS241 (PPND16) rational approximation of
//     the standard normal quantile (Applied Statistics 37 (1988) 477-484); one
//     uniform per normal draw, replacing boost::random::normal_distribution
//     (relearn/source/util/Random.h:128-140).
#pragma once

#include <stdint.h>
#include <math.h>


#if defined(__CUDACC__)
#define RL_HD __host__ __device__ __forceinline__
#else
#define RL_HD inline
#endif

namespace rl {

// ---------------------------------------------------------------- bit casts
RL_HD uint64_t as_u64(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    __builtin_memcpy(&u, &x, sizeof(u));
    return u;
#endif
}

RL_HD double as_f64(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double x;
    __builtin_memcpy(&x, &u, sizeof(x));
    return x;
#endif
}

// ------------------------------------------------------------------ Philox
struct u32x4 {
    uint32_t x, y, z, w;
};

RL_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

// Philox4x32 with 10 rounds.  Round function and constants as published:
// multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key increments 0x9E3779B9 /
// 0xBB67AE85.
RL_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c.x, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
        c = u32x4{ hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0 };
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// The same generator with the round keys given (k0 + r W0, k1 + r W1 for
// r = 0..9), for kernels whose key is the same in every thread.
RL_HD u32x4 philox4x32_10_rk(u32x4 c, const uint32_t* rk0, const uint32_t* rk1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c.x, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
        c = u32x4{ hi1 ^ c.y ^ rk0[round], lo1, hi0 ^ c.w ^ rk1[round], lo0 };
    }
    return c;
}

// Stream identifiers (upper byte of the fourth counter word).
enum Stream : uint32_t {
    STREAM_BH_PICK = 1,    // Barnes-Hut weighted pick (per descent)
    STREAM_CONNECTOR = 2,  // connector shuffle key (per request)
    STREAM_NOISE = 3,      // normal background input (per neuron pair and step)
    STREAM_DELETION = 4,   // synapse deletion picks
    STREAM_POISSON = 5,    // Poisson model spike thresholds (per neuron-step)
};

// Draw the four words keyed on (seed, step, neuron, sub, stream, depth).
RL_HD u32x4 draw(uint64_t seed, uint32_t step, uint32_t neuron, uint32_t sub, uint32_t stream, uint32_t depth) {
    const u32x4 ctr{ step, neuron, sub, (stream << 24) | (depth & 0xFFFFFFu) };
    return philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// 53 random bits from two words.
RL_HD uint64_t bits53(const u32x4& r) {
    return ((uint64_t)r.x << 21) | (uint64_t)(r.y >> 11);
}

// Uniform double in [0, 1).
RL_HD double uniform01(const u32x4& r) {
    return (double)bits53(r) * 1.1102230246251565404e-16;  // 2^-53
}

// Uniform double in the open interval (0, 1).
RL_HD double uniform_open01(const u32x4& r) {
    return ((double)bits53(r) + 0.5) * 1.1102230246251565404e-16;
}

// 64-bit key (connector shuffle).
RL_HD uint64_t bits64(const u32x4& r) {
    return ((uint64_t)r.x << 32) | (uint64_t)r.y;
}

// a * b + c with one rounding (fma on both sides).
RL_HD double rl_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return __builtin_fma(a, b, c);
#endif
}

// -------------------------------------------------------------- exp / log
// ln 2 split so that k * LN2_HI is exact for |k| < 2^20.
#define RL_LN2_HI 0.6931467056274414
#define RL_LN2_LO 4.7493250390316726e-07
#define RL_INV_LN2 1.4426950408889634

// y * 2^k for y in [0.5, 2) and k in [-1080, 1030]; one rounding at most.
RL_HD double scale_pow2(double y, int k) {
    if (k > 1023) {
        y = y * as_f64((uint64_t)(1023 + 1023) << 52);
        k -= 1023;
        if (k > 1023) {
            k = 1023;
        }
        return y * as_f64((uint64_t)(k + 1023) << 52);
    }
    if (k < -1021) {
        // exact move into the normal range, then a single rounding into the subnormals
        const double t = y * as_f64((uint64_t)(k + 54 + 1023) << 52);
        return t * as_f64((uint64_t)(-54 + 1023) << 52);
    }
    return y * as_f64((uint64_t)(k + 1023) << 52);
}

// 2^(j/64), j = 0..63, as hi + lo (hi rounded to nearest, lo the rounded
// remainder), from 60-digit decimal arithmetic (exp_table.py beside this file).
#define RL_EXP_TABLE_INIT \
    { 0x1.0000000000000p+0, 0x0.0p+0 }, \
    { 0x1.02c9a3e778061p+0, -0x1.19083535b085dp-56 }, \
    { 0x1.059b0d3158574p+0, 0x1.d73e2a475b465p-55 }, \
    { 0x1.0874518759bc8p+0, 0x1.186be4bb284ffp-57 }, \
    { 0x1.0b5586cf9890fp+0, 0x1.8a62e4adc610bp-54 }, \
    { 0x1.0e3ec32d3d1a2p+0, 0x1.03a1727c57b53p-59 }, \
    { 0x1.11301d0125b51p+0, -0x1.6c51039449b3ap-54 }, \
    { 0x1.1429aaea92de0p+0, -0x1.32fbf9af1369ep-54 }, \
    { 0x1.172b83c7d517bp+0, -0x1.19041b9d78a76p-55 }, \
    { 0x1.1a35beb6fcb75p+0, 0x1.e5b4c7b4968e4p-55 }, \
    { 0x1.1d4873168b9aap+0, 0x1.e016e00a2643cp-54 }, \
    { 0x1.2063b88628cd6p+0, 0x1.dc775814a8495p-55 }, \
    { 0x1.2387a6e756238p+0, 0x1.9b07eb6c70573p-54 }, \
    { 0x1.26b4565e27cddp+0, 0x1.2bd339940e9d9p-55 }, \
    { 0x1.29e9df51fdee1p+0, 0x1.612e8afad1255p-55 }, \
    { 0x1.2d285a6e4030bp+0, 0x1.0024754db41d5p-54 }, \
    { 0x1.306fe0a31b715p+0, 0x1.6f46ad23182e4p-55 }, \
    { 0x1.33c08b26416ffp+0, 0x1.32721843659a6p-54 }, \
    { 0x1.371a7373aa9cbp+0, -0x1.63aeabf42eae2p-54 }, \
    { 0x1.3a7db34e59ff7p+0, -0x1.5e436d661f5e3p-56 }, \
    { 0x1.3dea64c123422p+0, 0x1.ada0911f09ebcp-55 }, \
    { 0x1.4160a21f72e2ap+0, -0x1.ef3691c309278p-58 }, \
    { 0x1.44e086061892dp+0, 0x1.89b7a04ef80d0p-59 }, \
    { 0x1.486a2b5c13cd0p+0, 0x1.3c1a3b69062f0p-56 }, \
    { 0x1.4bfdad5362a27p+0, 0x1.d4397afec42e2p-56 }, \
    { 0x1.4f9b2769d2ca7p+0, -0x1.4b309d25957e3p-54 }, \
    { 0x1.5342b569d4f82p+0, -0x1.07abe1db13cadp-55 }, \
    { 0x1.56f4736b527dap+0, 0x1.9bb2c011d93adp-54 }, \
    { 0x1.5ab07dd485429p+0, 0x1.6324c054647adp-54 }, \
    { 0x1.5e76f15ad2148p+0, 0x1.ba6f93080e65ep-54 }, \
    { 0x1.6247eb03a5585p+0, -0x1.383c17e40b497p-54 }, \
    { 0x1.6623882552225p+0, -0x1.bb60987591c34p-54 }, \
    { 0x1.6a09e667f3bcdp+0, -0x1.bdd3413b26456p-54 }, \
    { 0x1.6dfb23c651a2fp+0, -0x1.bbe3a683c88abp-57 }, \
    { 0x1.71f75e8ec5f74p+0, -0x1.16e4786887a99p-55 }, \
    { 0x1.75feb564267c9p+0, -0x1.0245957316dd3p-54 }, \
    { 0x1.7a11473eb0187p+0, -0x1.41577ee04992fp-55 }, \
    { 0x1.7e2f336cf4e62p+0, 0x1.05d02ba15797ep-56 }, \
    { 0x1.82589994cce13p+0, -0x1.d4c1dd41532d8p-54 }, \
    { 0x1.868d99b4492edp+0, -0x1.fc6f89bd4f6bap-54 }, \
    { 0x1.8ace5422aa0dbp+0, 0x1.6e9f156864b27p-54 }, \
    { 0x1.8f1ae99157736p+0, 0x1.5cc13a2e3976cp-55 }, \
    { 0x1.93737b0cdc5e5p+0, -0x1.75fc781b57ebcp-57 }, \
    { 0x1.97d829fde4e50p+0, -0x1.d185b7c1b85d1p-54 }, \
    { 0x1.9c49182a3f090p+0, 0x1.c7c46b071f2bep-56 }, \
    { 0x1.a0c667b5de565p+0, -0x1.359495d1cd533p-54 }, \
    { 0x1.a5503b23e255dp+0, -0x1.d2f6edb8d41e1p-54 }, \
    { 0x1.a9e6b5579fdbfp+0, 0x1.0fac90ef7fd31p-54 }, \
    { 0x1.ae89f995ad3adp+0, 0x1.7a1cd345dcc81p-54 }, \
    { 0x1.b33a2b84f15fbp+0, -0x1.2805e3084d708p-57 }, \
    { 0x1.b7f76f2fb5e47p+0, -0x1.5584f7e54ac3bp-56 }, \
    { 0x1.bcc1e904bc1d2p+0, 0x1.23dd07a2d9e84p-55 }, \
    { 0x1.c199bdd85529cp+0, 0x1.11065895048ddp-55 }, \
    { 0x1.c67f12e57d14bp+0, 0x1.2884dff483cadp-54 }, \
    { 0x1.cb720dcef9069p+0, 0x1.503cbd1e949dbp-56 }, \
    { 0x1.d072d4a07897cp+0, -0x1.cbc3743797a9cp-54 }, \
    { 0x1.d5818dcfba487p+0, 0x1.2ed02d75b3707p-55 }, \
    { 0x1.da9e603db3285p+0, 0x1.c2300696db532p-54 }, \
    { 0x1.dfc97337b9b5fp+0, -0x1.1a5cd4f184b5cp-54 }, \
    { 0x1.e502ee78b3ff6p+0, 0x1.39e8980a9cc8fp-55 }, \
    { 0x1.ea4afa2a490dap+0, -0x1.e9c23179c2893p-54 }, \
    { 0x1.efa1bee615a27p+0, 0x1.dc7f486a4b6b0p-54 }, \
    { 0x1.f50765b6e4540p+0, 0x1.9d3e12dd8a18bp-54 }, \
    { 0x1.fa7c1819e90d8p+0, 0x1.74853f3a5931ep-55 },

#if defined(__CUDACC__)
static __device__ const double2 rl_exp_table_dev[64] = { RL_EXP_TABLE_INIT };
#endif
static const double rl_exp_table_host[64][2] = { RL_EXP_TABLE_INIT };

// exp's constants: the Taylor coefficients 1/720, 1/120, 1/24, 1/6, 1/2,
// 64 / ln 2 and ln 2 / 64 as hi + lo (device: constant memory, as the normal
// quantile's coefficients).
#define RL_EXP_CONST_INIT \
    { 1.3888888888888889e-03, 8.3333333333333332e-03, 4.1666666666666664e-02, 1.6666666666666666e-01, 0.5, 92.332482616893656768, \
      RL_LN2_HI / 64.0, RL_LN2_LO / 64.0 }
#if defined(__CUDACC__)
static __constant__ double rl_exp_const_dev[8] = RL_EXP_CONST_INIT;
#endif
static const double rl_exp_const_host[8] = RL_EXP_CONST_INIT;
#if defined(__CUDA_ARCH__)
#define RL_EXPC(k) rl_exp_const_dev[k]
#else
#define RL_EXPC(k) rl_exp_const_host[k]
#endif

// exp(x) by Tang's table-driven method (P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15(2), 1989, 144-157): x = (64 m + j) ln2/64 + r with
// |r| <= ln2/128 (up to the rounding of k), exp(x) = 2^m 2^(j/64) exp(r),
// exp(r) - 1 by its Taylor polynomial of degree 6 (truncation error below
// 1e-19), 2^(j/64) from the table as hi + lo.  12 FP64 operations and one
// table load; differs from glibc's exp in 0.2 % of arguments, by one ulp.
RL_HD double rl_exp(double x) {
    if (x != x) {
        return x;
    }
    if (x > 709.782712893384) {
        return as_f64(0x7FF0000000000000ull);
    }
    if (x < -745.1332191019412) {
        return 0.0;
    }
    const double kd = floor(x * RL_EXPC(5) + 0.5);  // 64 / ln 2
    // kd * (RL_LN2_HI / 64) is exact; so is the subtraction (Sterbenz, or kd = 0)
    const double r = rl_fma(-kd, RL_EXPC(7), x - kd * RL_EXPC(6));
    const int ki = (int)kd;
    const int j = ki & 63;
    const int m = ki >> 6;  // floor(ki / 64)
    // exp(r) - 1 = r + r^2 (1/2 + r/6 + r^2/24 + r^3/120 + r^4/720)
    double p = rl_fma(RL_EXPC(0), r, RL_EXPC(1));  // 1/720, 1/120
    p = rl_fma(p, r, RL_EXPC(2));  // 1/24
    p = rl_fma(p, r, RL_EXPC(3));  // 1/6
    p = rl_fma(p, r, RL_EXPC(4));
    p = rl_fma(r * r, p, r);
#if defined(__CUDA_ARCH__)
    const double2 t = __ldg(&rl_exp_table_dev[j]);
    const double t_hi = t.x, t_lo = t.y;
#else
    const double t_hi = rl_exp_table_host[j][0], t_lo = rl_exp_table_host[j][1];
#endif
    // 2^(j/64) (1 + p) = hi + (hi p + lo), dropping lo p (below 1e-18 of the result)
    return scale_pow2(t_hi + rl_fma(t_hi, p, t_lo), m);
}

// rl_exp without branches, for kernels that interleave independent chains of
// arithmetic (a branch ends the stretch of code the compiler schedules as
// one): the main path always runs, the scaling by 2^m is always two
// multiplications by powers of two — 2^m and 1 in the normal range,
// 2^1023 and 2^(m-1023) above it, 2^(m+54) and 2^-54 into the subnormals, as
// scale_pow2 does — and NaN, overflow and underflow are selected at the end.
// The same bits as rl_exp for every argument: in range every operation is
// the same, and every product by a power of two is exact except the one
// rounding both forms make.  Out of range the main path's value is discarded
// (the host clamps the argument first, so that its int conversion is
// defined; on the device the conversion saturates).
RL_HD double rl_exp_flat(double x) {
#if defined(__CUDA_ARCH__)
    const double xc = x;
#else
    const double xc = x != x ? 0.0 : fmin(fmax(x, -746.0), 710.0);
#endif
    const double kd = floor(xc * RL_EXPC(5) + 0.5);  // 64 / ln 2
    const double r = rl_fma(-kd, RL_EXPC(7), xc - kd * RL_EXPC(6));
    const int ki = (int)kd;
    const int j = ki & 63;
    const int m = ki >> 6;
    double p = rl_fma(RL_EXPC(0), r, RL_EXPC(1));
    p = rl_fma(p, r, RL_EXPC(2));
    p = rl_fma(p, r, RL_EXPC(3));
    p = rl_fma(p, r, RL_EXPC(4));
    p = rl_fma(r * r, p, r);
#if defined(__CUDA_ARCH__)
    const double2 t = __ldg(&rl_exp_table_dev[j]);
    const double t_hi = t.x, t_lo = t.y;
#else
    const double t_hi = rl_exp_table_host[j][0], t_lo = rl_exp_table_host[j][1];
#endif
    const double y = t_hi + rl_fma(t_hi, p, t_lo);
    const bool low = m < -1021;
    const bool high = m > 1023;
    int a = low ? m + 54 : (high ? 1023 : m);
    int b = low ? -54 : (high ? m - 1023 : 0);
    a = a < -1022 ? -1022 : (a > 1023 ? 1023 : a);  // only out-of-range arguments reach the clamps
    b = b < -1022 ? -1022 : (b > 1023 ? 1023 : b);
    const double v = (y * as_f64((uint64_t)(a + 1023) << 52)) * as_f64((uint64_t)(b + 1023) << 52);
    return x != x ? x : (x > 709.782712893384 ? as_f64(0x7FF0000000000000ull) : (x < -745.1332191019412 ? 0.0 : v));
}

// rl_exp_flat for x <= 0 and NaN (the growth curves' exp(-q^2)): the same
// bits as rl_exp there, without the overflow case (m <= 0 for x <= 0).
RL_HD double rl_exp_flat_nonpos(double x) {
#if defined(__CUDA_ARCH__)
    const double xc = x;
#else
    const double xc = x != x ? 0.0 : fmin(fmax(x, -746.0), 0.0);
#endif
    const double kd = floor(xc * RL_EXPC(5) + 0.5);  // 64 / ln 2
    const double r = rl_fma(-kd, RL_EXPC(7), xc - kd * RL_EXPC(6));
    const int ki = (int)kd;
    const int j = ki & 63;
    const int m = ki >> 6;
    double p = rl_fma(RL_EXPC(0), r, RL_EXPC(1));
    p = rl_fma(p, r, RL_EXPC(2));
    p = rl_fma(p, r, RL_EXPC(3));
    p = rl_fma(p, r, RL_EXPC(4));
    p = rl_fma(r * r, p, r);
#if defined(__CUDA_ARCH__)
    const double2 t = __ldg(&rl_exp_table_dev[j]);
    const double t_hi = t.x, t_lo = t.y;
#else
    const double t_hi = rl_exp_table_host[j][0], t_lo = rl_exp_table_host[j][1];
#endif
    const double y = t_hi + rl_fma(t_hi, p, t_lo);
    const bool low = m < -1021;
    int a = low ? m + 54 : m;
    a = a < -1022 ? -1022 : a;  // only arguments below the underflow reach the clamp
    const double v = (y * as_f64((uint64_t)(a + 1023) << 52)) * as_f64((uint64_t)((low ? -54 : 0) + 1023) << 52);
    return x != x ? x : (x < -745.1332191019412 ? 0.0 : v);
}

// log(x) for finite x > 0 (normal range): x = m 2^e with m in
// [sqrt(2)/2, sqrt(2)), log(m) = 2 atanh(s), s = (m-1)/(m+1), odd series in s.
RL_HD double rl_log(double x) {
    uint64_t b = as_u64(x);
    int e = (int)((b >> 52) & 0x7FF) - 1023;
    double m = as_f64((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        e += 1;
    }
    const double f = m - 1.0;
    const double s = f / (2.0 + f);
    const double z = s * s;
    double R = 1.0 / 23.0;
    R = rl_fma(R, z, 1.0 / 21.0);
    R = rl_fma(R, z, 1.0 / 19.0);
    R = rl_fma(R, z, 1.0 / 17.0);
    R = rl_fma(R, z, 1.0 / 15.0);
    R = rl_fma(R, z, 1.0 / 13.0);
    R = rl_fma(R, z, 1.0 / 11.0);
    R = rl_fma(R, z, 1.0 / 9.0);
    R = rl_fma(R, z, 1.0 / 7.0);
    R = rl_fma(R, z, 1.0 / 5.0);
    R = rl_fma(R, z, 1.0 / 3.0);
    R = R * z;
    const double two_s = 2.0 * s;
    const double logm = rl_fma(two_s, R, two_s);
    const double ed = (double)e;
    return ed * RL_LN2_HI + rl_fma(ed, RL_LN2_LO, logm);
}

// ----------------------------------------------------------------- hypot3
// The correctly rounded reciprocal 1/a (both sides round to nearest).
RL_HD double rl_recip(double a) {
#if defined(__CUDA_ARCH__)
    return __drcp_rn(a);
#else
    return 1.0 / a;
#endif
}

// p / a rounded once, from the correctly rounded reciprocal ra = 1/a:
// q0 = p ra, r = p - a q0 (exact with an FMA), q0 + r ra rounded once is the
// correctly rounded quotient (Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34 (1990)), as
// long as nothing under- or overflows.
RL_HD double quotient_from_recip(double p, double a, double ra) {
    const double q0 = p * ra;
    const double r = rl_fma(-a, q0, p);
    return rl_fma(r, ra, q0);
}

// Whether quotient_from_recip is exact for p / a: a in [2^-900, 2^901) and p
// zero, or normal, at least 2^-963 and at most 2^900 below a.
RL_HD bool recip_quotient_safe(double p, double a) {
    const int ea = (int)((as_u64(a) >> 52) & 0x7FF);
    const int ep = (int)((as_u64(p) >> 52) & 0x7FF);
    return ea >= 123 && ea <= 1923 && (p == 0.0 || (ep >= 60 && ep >= ea - 900));
}

RL_HD double rl_hypot3(double x, double y, double z) {
    x = fabs(x);
    y = fabs(y);
    z = fabs(z);
    const double a = x < y ? (y < z ? z : y) : (x < z ? z : x);
    if (a == 0.0) {
        return 0.0;
    }
    // The largest component divided by a is exactly 1, so only the other two
    // are divided (an FP64 division is a long sequence on the GPU); the terms
    // are still added in x, y, z order, so the result is the same bits.
    const bool zmax = a == z;
    const bool ymax = !zmax && a == y;
    const double p = zmax || ymax ? x : y;  // first component that is not the maximum
    const double q = zmax ? y : z;          // second one
    // p / a and q / a from one reciprocal (the same bits as the two
    // divisions wherever that is exact, which covers every realistic distance)
    double ps, qs;
    if (recip_quotient_safe(p, a) && recip_quotient_safe(q, a)) {
        const double ra = rl_recip(a);
        ps = quotient_from_recip(p, a, ra);
        qs = quotient_from_recip(q, a, ra);
    } else {
        ps = p / a;
        qs = q / a;
    }
    const double p2 = ps * ps, q2 = qs * qs;
    const double t0 = zmax || ymax ? p2 : 1.0;
    const double t1 = zmax ? q2 : (ymax ? 1.0 : p2);
    const double t2 = zmax ? 1.0 : q2;
    return a * sqrt(t0 + t1 + t2);
}

// d^y for d > 0 (the std::pow(distance, k - 1) of the gamma and Weibull
// kernels): exact for y = 0 and y = 1, exp(y log d) with the shared exp / log
// otherwise, so that host and device agree bit for bit.
RL_HD double rl_pow_pos(double d, double y) {
    if (y == 0.0) {
        return 1.0;
    }
    if (y == 1.0) {
        return d;
    }
    return rl_exp(y * rl_log(d));
}

// Attraction of a cell at distance d > 0 for the kernel `type`
// (KernelBase::get_probability(distance)): Gaussian scale = -1/sigma^2 and mu;
// gamma a = 1/(Gamma(k) theta^k), b = -1/theta; Weibull a = b k, b = b;
// linear cut-off.  Operation order as in the reference's kernels.
RL_HD double rl_kernel_prob(int type, double d, double mu, double scale, double k_minus_1, double a, double b, double cutoff, int cutoff_inf) {
    if (type == 1) {  // gamma (Gamma.h)
        const double f1 = rl_pow_pos(d, k_minus_1);
        const double f2 = rl_exp(d * b);
        return a * f1 * f2;
    }
    if (type == 2) {  // linear (Linear.h)
        if (cutoff_inf) {
            return 1.0;
        }
        if (d > cutoff) {
            return 0.0;
        }
        return 1 - d / cutoff;
    }
    if (type == 3) {  // Weibull (Weibull.h)
        const double f2 = rl_pow_pos(d, k_minus_1);
        const double exponent = -b * f2 * d;
        const double f3 = rl_exp(exponent);
        return a * f2 * f3;
    }
    const double num = (d - mu) * (d - mu);  // Gaussian (Gaussian.h:62-68)
    return rl_exp(num * scale);
}

// std::nextafter(total, total + 1e-5) for finite total > 0
// (ProbabilityPicker.h:108 of the reference).
RL_HD double next_up_eps(double total) {
    const double toward = total + 1e-5;
    if (toward > total) {
        return as_f64(as_u64(total) + 1);
    }
    return total;
}

// ------------------------------------------------------ normal quantile
// AS241 / PPND16: standard normal quantile for p in (0, 1), in two pieces:
// the central rational function for |p - 0.5| <= 0.425 and the tails.  A
// kernel that draws for many neurons runs the tail piece for the few that need
// it together (it holds a log, a square root and two divisions).
RL_HD bool normal_in_tail(double p) {
    return !(fabs(p - 0.5) <= 0.425);
}

// The central piece's coefficients, highest power first (numerator, then
// denominator).  On the device they sit in constant memory, where a fused
// multiply-add reads them as an operand (no instructions to materialise the
// 64-bit literals in registers); the host reads the same values.
#define RL_AS241_CENTRAL_INIT                                                                                                 \
    { 2.5090809287301226727e+3, 3.3430575583588128105e+4, 6.7265770927008700853e+4, 4.5921953931549871457e+4,              \
      1.3731693765509461125e+4, 1.9715909503065514427e+3, 1.3314166789178437745e+2, 3.3871328727963666080e+0,              \
      5.2264952788528545610e+3, 2.8729085735721942674e+4, 3.9307895800092710610e+4, 2.1213794301586595867e+4,              \
      5.3941960214247511077e+3, 6.8718700749205790830e+2, 4.2313330701600911252e+1, 1.0 }
#if defined(__CUDACC__)
static __constant__ double rl_as241_central_dev[16] = RL_AS241_CENTRAL_INIT;
#endif
static const double rl_as241_central_host[16] = RL_AS241_CENTRAL_INIT;
#if defined(__CUDA_ARCH__)
#define RL_AS241_C(k) rl_as241_central_dev[k]
#else
#define RL_AS241_C(k) rl_as241_central_host[k]
#endif

RL_HD double normal_quantile_central(double p) {
    const double q = p - 0.5;
    const double r = 0.180625 - q * q;
    double num = RL_AS241_C(0);
#pragma unroll
    for (int k = 1; k < 8; ++k) {
        num = rl_fma(num, r, RL_AS241_C(k));
    }
    double den = RL_AS241_C(8);
#pragma unroll
    for (int k = 9; k < 16; ++k) {
        den = rl_fma(den, r, RL_AS241_C(k));
    }
    return (num * q) / den;
}

RL_HD double normal_quantile_tail(double p) {
    const double q = p - 0.5;
    double r = q < 0.0 ? p : 1.0 - p;
    r = sqrt(-rl_log(r));
    double num;
    double den;
    if (r <= 5.0) {
        r = r - 1.6;
        num = 7.7454501427834140764e-4;
        num = rl_fma(num, r, 2.2723844989269184583e-2);
        num = rl_fma(num, r, 2.4178072517745061177e-1);
        num = rl_fma(num, r, 1.2704582524523683826e+0);
        num = rl_fma(num, r, 3.6478483247632046050e+0);
        num = rl_fma(num, r, 5.7694972214606914055e+0);
        num = rl_fma(num, r, 4.6303378461565452959e+0);
        num = rl_fma(num, r, 1.4234371107496835773e+0);
        den = 1.0507500716444168432e-9;
        den = rl_fma(den, r, 5.4759380849953449460e-4);
        den = rl_fma(den, r, 1.5198666563616457197e-2);
        den = rl_fma(den, r, 1.4810397642748007459e-1);
        den = rl_fma(den, r, 6.8976733498510000455e-1);
        den = rl_fma(den, r, 1.6763848301838038494e+0);
        den = rl_fma(den, r, 2.0531916266377588219e+0);
        den = rl_fma(den, r, 1.0);
    } else {
        r = r - 5.0;
        num = 2.0103343992922881327e-7;
        num = rl_fma(num, r, 2.7115555687434875782e-5);
        num = rl_fma(num, r, 1.2426609473880784386e-3);
        num = rl_fma(num, r, 2.6532189526576123093e-2);
        num = rl_fma(num, r, 2.9656057182850489123e-1);
        num = rl_fma(num, r, 1.7848265399172913358e+0);
        num = rl_fma(num, r, 5.4637849111641143699e+0);
        num = rl_fma(num, r, 6.6579046435011037772e+0);
        den = 2.0442631033899397856e-15;
        den = rl_fma(den, r, 1.4215117583164458887e-7);
        den = rl_fma(den, r, 1.8463183175100546818e-5);
        den = rl_fma(den, r, 7.8686913114561325910e-4);
        den = rl_fma(den, r, 1.4875361290850614853e-2);
        den = rl_fma(den, r, 1.3692988092273580531e-1);
        den = rl_fma(den, r, 5.9983220655588793769e-1);
        den = rl_fma(den, r, 1.0);
    }
    const double x = num / den;
    return q < 0.0 ? -x : x;
}

RL_HD double normal_quantile(double p) {
    return normal_in_tail(p) ? normal_quantile_tail(p) : normal_quantile_central(p);
}

// Normal(mean, stddev) background draw for (seed, step, neuron).
// One Philox block serves the background draws of the neuron pair (2m, 2m + 1)
// of a network at a step: words (x, y) for the even neuron, (z, w) for the odd
// one, so that a thread updating a pair draws once.
RL_HD u32x4 noise_block(uint64_t seed, uint32_t step, uint32_t neuron) {
    return draw(seed, step, neuron >> 1, 0u, STREAM_NOISE, 0u);
}
RL_HD u32x4 noise_block_rk(const uint32_t* rk0, const uint32_t* rk1, uint32_t step, uint32_t neuron) {
    return philox4x32_10_rk(u32x4{ step, neuron >> 1, 0u, (uint32_t)STREAM_NOISE << 24 }, rk0, rk1);
}
RL_HD uint64_t noise_bits53(const u32x4& r, uint32_t neuron) {
    return (neuron & 1u) ? (((uint64_t)r.z << 21) | (uint64_t)(r.w >> 11)) : (((uint64_t)r.x << 21) | (uint64_t)(r.y >> 11));
}

// The open-interval uniform of a neuron's background draw.
RL_HD double noise_uniform(uint64_t seed, uint32_t step, uint32_t neuron) {
    const u32x4 r = noise_block(seed, step, neuron);
    return ((double)noise_bits53(r, neuron) + 0.5) * 1.1102230246251565404e-16;  // open (0, 1)
}

RL_HD double noise_uniform_rk(const uint32_t* rk0, const uint32_t* rk1, uint32_t step, uint32_t neuron) {
    const u32x4 r = noise_block_rk(rk0, rk1, step, neuron);
    return ((double)noise_bits53(r, neuron) + 0.5) * 1.1102230246251565404e-16;  // open (0, 1)
}

RL_HD double background_normal(uint64_t seed, uint32_t step, uint32_t neuron, double mean, double stddev) {
    return mean + stddev * normal_quantile(noise_uniform(seed, step, neuron));
}

}  // namespace rl
