// FP32 precision form of the activity update and of the Barnes-Hut search.
//
// Same algorithms as the FP64 drop-in (activity.cu, bh_search.cu) with
// different arithmetic, as the precision form specifies:
//   * membrane (Izhikevich), input (normal background, the same Philox draw
//     as the FP64 form mapped through an FP32 erfinv) and growth-curve
//     arithmetic in FP32, state x, u, growth deltas stored as FP32;
//   * calcium integrated in FP64.  The h Euler substeps of
//     CalciumCalculatorCPU::update_current_calcium (calcium/CalciumCalculatorCPU.cpp:61-68)
//     form the linear recurrence c <- c*A + s*beta*fired with A = 1 + s/(-tau);
//     h substeps are applied at once as c*A^h + s*beta*fired*(A^(h-1)+...+1)
//     with both factors precomputed in FP64;
//   * octree counts and centroids reduced in FP64 (octree.cu), then read by
//     the search as 16-byte records with the centroid in 32-bit fixed point
//     (QFrame): a coordinate difference is exact in the integers and rounds
//     once when it becomes a float, so distances keep FP32 relative precision
//     even between cells far from the origin (FP32 coordinates would round
//     each coordinate to its own magnitude);
//   * attraction weights exp(-(d-mu)^2/sigma^2)*count in FP32, summed per lane in
//     visiting order with Kahan compensation; the pick compares the
//     compensated running sum with r.
// Errors against the FP64 form are measured, not assumed (bench.py
// --precision-report): selection probabilities, calcium drift, distances of
// formed synapses.
#include "bh_eval.cuh"
#include "bh_wide.cuh"
#include "rl_context.cuh"
#include "rl_math.cuh"

namespace rl {

bool is_fp32(const Ctx& c) {
    return c.cfg.precision == RL_PRECISION_FP32;
}

namespace {

__global__ void k_d2f(uint32_t n, const double* __restrict__ a, float* __restrict__ b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        b[i] = (float)a[i];
    }
}

__global__ void k_f2d(uint32_t n, const float* __restrict__ a, double* __restrict__ b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        b[i] = (double)a[i];
    }
}

// ----------------------------------------------------------- activity
struct Act32 {
    uint32_t n;
    const uint8_t* enabled;
    const uint8_t* fired_prev;
    uint8_t* fired_cur;
    float* x;
    float* u;
    float* input;
    double* calcium;
    float* delta[3];
    float conductance, noise_mean, noise_stddev;
    uint32_t h_model;
    // one Euler substep with s = 1/h, each increment rounded at its own (small)
    // magnitude before it meets the state:
    //   x' = x + [x (s k1 x + s k2) + (s k3 + s I) - s u]      (3 FMA + 1 add)
    //   u' = u + s a (b x - u)                                  (2 FMA)
    // Folding the 1 into the factor, x' = x (1 + s k2 + s k1 x) + ..., saves an
    // operation but rounds at the magnitude of x twice per substep, which
    // shifts the resting point and biased the firing rate by +2.4e-5 against
    // FP64 in a 200,000-neuron, 1,000-step check; this form: +2.1e-6.
    float c, d, v_spike, s, sk1, sk2, sk3, sa, b;
    double ca_mul, ca_add;  // calcium: c <- c*ca_mul + fired*ca_add
    float xi[3], inv_zeta[3];
    int flat[3];            // eta == epsilon corner case of gaussian_growth_curve
    float eta[3];
    // per-neuron target calcium (null: one target, folded into xi / inv_zeta);
    // kz / (eta - epsilon) is a neuron's inv_zeta
    const float* target;
    float kz;
    const NetInfo* nets;
    const uint16_t* net_of;
    const NetBlock* blocks;  // a batched context's neurons in blocks of one network
    uint32_t num_blocks;
    int32_t* syn_in[2];  // pushed synaptic sums by step parity (ActDesc)
    uint8_t* hist;       // spike history (kHistSteps rows of hist_stride bytes)
    size_t hist_stride;
    // a context with one network: its seed and growth rates, so that the
    // kernel reads no network table
    uint64_t seed1;
    float nu1[3];
    uint32_t rk0[10], rk1[10];  // that network's Philox round keys
    // the other neuron models (neurons/models/*), their constants in FP32
    float p_x0, p_tau_inv, p_refractory;                                   // Poisson
    float f_a, f_b, f_phi;                                                 // FitzHugh-Nagumo
    float e_g_L, e_E_L, e_V_T, e_g_L_d_T, e_d_T_inv, e_tau_w_inv, e_C_inv, e_a, e_b, e_V_spike;  // AEIF
};

// Standard normal quantile of u = (k + 0.5) 2^-24 in FP32 as sqrt(2) erfinv(2u - 1),
// with the single-precision erfinv approximation of M. Giles ("Approximating
// the erfinv function", GPU Computing Gems Jade Edition, 2011): the central
// branch covers 99.7 % of the draws, so warps rarely diverge.
__device__ __forceinline__ float normal_from_bits24(uint32_t k24) {
    const float x = (float)((int)(2u * k24 + 1u) - (1 << 24)) * 5.9604644775390625e-8f;  // 2u - 1, exact
    float w = -__logf((1.0f - x) * (1.0f + x));
    float p;
    if (w < 5.0f) {
        w -= 2.5f;
        p = 2.81022636e-08f;
        p = fmaf(p, w, 3.43273939e-07f);
        p = fmaf(p, w, -3.5233877e-06f);
        p = fmaf(p, w, -4.39150654e-06f);
        p = fmaf(p, w, 0.00021858087f);
        p = fmaf(p, w, -0.00125372503f);
        p = fmaf(p, w, -0.00417768164f);
        p = fmaf(p, w, 0.246640727f);
        p = fmaf(p, w, 1.50140941f);
    } else {
        w = sqrtf(w) - 3.0f;
        p = -0.000200214257f;
        p = fmaf(p, w, 0.000100950558f);
        p = fmaf(p, w, 0.00134934322f);
        p = fmaf(p, w, -0.00367342844f);
        p = fmaf(p, w, 0.00573950773f);
        p = fmaf(p, w, -0.0076224613f);
        p = fmaf(p, w, 0.00943887047f);
        p = fmaf(p, w, 1.00167406f);
        p = fmaf(p, w, 2.83297682f);
    }
    return 1.41421356237f * (p * x);
}

// One neuron's activity step on registers: `x`, `u`, `ca` and the three
// deltas are read and updated in place; `input` and `fired` are outputs.
// 2^x with the special-function unit (ex2.approx, relative error ~2^-22).
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// A neuron's growth-curve constants per element type (gaussian_growth_curve
// with epsilon = max(target, eta)): xi, the scaled 1 / zeta, and the eta ==
// epsilon case as a bit; from the context's constants when every neuron has
// the same target, else from the neuron's own target.  Made once per neuron
// and launch, not per step.
struct Grow32 {
    float xi[3], iz[3];
    uint32_t flat;
};

__device__ __forceinline__ Grow32 grow32_of(const Act32& A, float tgt) {
    Grow32 G;
    G.flat = 0;
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (A.target) {
            const float eta = A.eta[t];
            const float eps = fmaxf(tgt, eta);
            const bool flat = eta == eps;
            G.xi[t] = 0.5f * (eta + eps);
            G.iz[t] = flat ? 0.0f : __fdividef(A.kz, eta - eps);
            G.flat |= (flat ? 1u : 0u) << t;
        } else {
            G.xi[t] = A.xi[t];
            G.iz[t] = A.inv_zeta[t];
            G.flat |= (A.flat[t] ? 1u : 0u) << t;
        }
    }
    return G;
}

// One step of calcium (FP64: the h substeps' closed form) and of the three
// growth deltas after the spike flag `spiked`.
__device__ __forceinline__ void calcium_growth_f32(const Act32& A, uint8_t spiked, const float (&nu)[3], const Grow32& G, double& ca,
                                                   float (&delta)[3]) {
    ca = fma(ca, A.ca_mul, spiked ? A.ca_add : 0.0);
    const float caf = (float)ca;
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const float q = (caf - G.xi[t]) * G.iz[t];
        const float curve = fmaf(2.0f, ex2_approx(-q * q), -1.0f);
        const float dz = ((G.flat >> t) & 1u) ? (caf == A.eta[t] ? 0.0f : -1.0f) : curve;
        delta[t] = fmaf(dz, nu[t], delta[t]);
    }
}

// `k24`: the neuron's 24 random bits of this step's background draw;
// `k24p`: 24 bits of its Poisson-threshold draw (Poisson model only).  The
// synaptic sum is pulled over the in-edges (`pull`, a block's first step) or
// is `pushed`, what the sources that fired at the step before pushed.  GROW
// false: calcium and growth are left to k_calcium_growth_f32 at the end of the
// chunk (ca, delta, nu and G are not used).
template <int H, int MODEL, bool EDGES = true, bool GROW = true>
__device__ __forceinline__ void neuron_f32(const Act32& A, const ActDesc* __restrict__ D, uint32_t i, bool enabled, uint8_t fired_prev, uint32_t k24,
                                           uint32_t k24p, const float (&nu)[3], const Grow32& G, float& x, float& u, double& ca, float (&delta)[3],
                                           float& input, uint8_t& fired, bool pull = true, int pushed = 0) {
    if (!enabled) {
        input = 0.0f;
        fired = fired_prev;
        return;
    }
    int isum = 0;
    if (EDGES && D->has_edges) {  // EDGES false: a network without synapses (the block kernel)
        if (pull) {
            const uint32_t* __restrict__ off = D->off;
            const uint32_t* __restrict__ src = D->src;
            const int32_t* __restrict__ wt = D->w;
            const uint32_t e0 = off[i], e1 = off[i + 1];
            for (uint32_t e = e0; e < e1; ++e) {
                if (A.fired_prev[src[e]]) {
                    isum += wt[e];
                }
            }
        } else {
            isum = pushed;
        }
    }
    input = fmaf((float)isum, A.conductance, fmaf(A.noise_stddev, normal_from_bits24(k24), A.noise_mean));

    float xv = x;
    float uv = u;
    uint8_t spiked = 0;
    const uint32_t h = H > 0 ? (uint32_t)H : A.h_model;
    if (MODEL == RL_MODEL_IZHIKEVICH) {
        const float sc = fmaf(A.s, input, A.sk3);
        const float ms = -A.s;
#pragma unroll
        for (uint32_t it = 0; it < h; ++it) {
            const float inc = fmaf(xv, fmaf(A.sk1, xv, A.sk2), fmaf(ms, uv, sc));
            uv = fmaf(A.sa, fmaf(A.b, xv, -uv), uv);
            xv = xv + inc;
            if (xv >= A.v_spike) {
                xv = A.c;
                uv += A.d;
                spiked = 1;
                break;
            }
        }
    } else if (MODEL == RL_MODEL_POISSON) {
        // PoissonModelCPU::update_activity; u counts the refractory steps left
        for (uint32_t it = 0; it < h; ++it) {
            xv = fmaf(fmaf(A.p_x0 - xv, A.p_tau_inv, input), A.s, xv);
        }
        if (uv == 0.0f) {
            const float threshold = (float)k24p * 5.9604644775390625e-8f;  // the FP64 form's uniform, 24 bits of it
            if (xv >= threshold) {
                spiked = 1;
                uv = A.p_refractory;
            }
        } else {
            uv -= 1.0f;
        }
    } else if (MODEL == RL_MODEL_FITZHUGH_NAGUMO) {
        // FitzHughNagumoModelCPU::update_activity: no reset, spike test after the substeps
        const float third = 1.0f / 3.0f;
        for (uint32_t it = 0; it < h; ++it) {
            const float x3 = xv * xv * xv;
            const float x_inc = fmaf(-x3, third, xv) - uv + input;
            const float w_inc = A.f_phi * fmaf(-A.f_b, uv, xv + A.f_a);
            xv = fmaf(x_inc, A.s, xv);
            uv = fmaf(w_inc, A.s, uv);
        }
        spiked = (uv > fmaf(-xv * xv * xv, third, xv) && xv > 1.0f) ? 1 : 0;
    } else {
        // AEIFModelCPU::update_activity
        for (uint32_t it = 0; it < h; ++it) {
            const float lin = -A.e_g_L * (xv - A.e_E_L);
            const float ex = A.e_g_L_d_T * __expf((xv - A.e_V_T) * A.e_d_T_inv);
            const float x_inc = (lin + ex - uv + input) * A.e_C_inv;
            const float w_inc = fmaf(A.e_a, xv - A.e_E_L, -uv) * A.e_tau_w_inv;
            xv = fmaf(x_inc, A.s, xv);
            uv = fmaf(w_inc, A.s, uv);
            if (xv >= A.e_V_spike) {
                xv = A.e_E_L;
                uv += A.e_b;
                spiked = 1;
                break;
            }
        }
    }
    x = xv;
    u = uv;
    fired = spiked;
    if (GROW) {
        calcium_growth_f32(A, spiked, nu, G, ca, delta);
    }
}

// Vector loads and stores of V consecutive entries (V = 1, 2, 4); the
// caller's index is a multiple of V, so every access is aligned to its width.
template <int V>
__device__ __forceinline__ void ld_f(const float* p, float (&v)[V]) {
    if constexpr (V == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
    } else if constexpr (V == 2) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        v[0] = t.x, v[1] = t.y;
    } else {
        v[0] = *p;
    }
}
template <int V>
__device__ __forceinline__ void st_f(float* p, const float (&v)[V]) {
    if constexpr (V == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (V == 2) {
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    } else {
        *p = v[0];
    }
}
template <int V>
__device__ __forceinline__ void ld_d(const double* p, double (&v)[V]) {
    if constexpr (V >= 2) {
#pragma unroll
        for (int k = 0; k < V; k += 2) {
            const double2 t = *reinterpret_cast<const double2*>(p + k);
            v[k] = t.x, v[k + 1] = t.y;
        }
    } else {
        v[0] = *p;
    }
}
template <int V>
__device__ __forceinline__ void st_d(double* p, const double (&v)[V]) {
    if constexpr (V >= 2) {
#pragma unroll
        for (int k = 0; k < V; k += 2) {
            *reinterpret_cast<double2*>(p + k) = make_double2(v[k], v[k + 1]);
        }
    } else {
        *p = v[0];
    }
}
template <int V>
__device__ __forceinline__ void ld_b(const uint8_t* p, uint8_t (&v)[V]) {
    if constexpr (V == 4) {
        const uint32_t t = *reinterpret_cast<const uint32_t*>(p);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = (uint8_t)(t >> (8 * k));
        }
    } else if constexpr (V == 2) {
        const uint16_t t = *reinterpret_cast<const uint16_t*>(p);
        v[0] = (uint8_t)t, v[1] = (uint8_t)(t >> 8);
    } else {
        v[0] = *p;
    }
}
template <int V>
__device__ __forceinline__ void st_b(uint8_t* p, const uint8_t (&v)[V]) {
    if constexpr (V == 4) {
        *reinterpret_cast<uint32_t*>(p) = (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
    } else if constexpr (V == 2) {
        *reinterpret_cast<uint16_t*>(p) = (uint16_t)(v[0] | (v[1] << 8));
    } else {
        *p = v[0];
    }
}
template <int V>
__device__ __forceinline__ void ld_h(const uint16_t* p, uint16_t (&v)[V]) {
    if constexpr (V == 4) {
        const uint2 t = *reinterpret_cast<const uint2*>(p);
        v[0] = (uint16_t)t.x, v[1] = (uint16_t)(t.x >> 16), v[2] = (uint16_t)t.y, v[3] = (uint16_t)(t.y >> 16);
    } else if constexpr (V == 2) {
        const uint32_t t = *reinterpret_cast<const uint32_t*>(p);
        v[0] = (uint16_t)t, v[1] = (uint16_t)(t >> 16);
    } else {
        v[0] = *p;
    }
}

// A set spike flag of neuron i at step k of the block: its out-edges' weights
// go to their targets' sums of the next step (none after the block's last).
__device__ __forceinline__ void push_spike32(const Act32& A, const ActDesc* __restrict__ D, uint32_t k, uint32_t step, uint32_t i) {
    if (!D->has_edges || k + 1 >= D->block_len) {
        return;
    }
    int32_t* next = A.syn_in[(step + 1u) & 1u];
    const uint32_t e0 = D->out_off[i], e1 = D->out_off[i + 1];
    for (uint32_t j = e0; j < e1; ++j) {
        const uint32_t e = D->out_perm[j];
        atomicAdd(next + D->tgt[e], D->w[e]);
    }
}

// V consecutive neurons from index i (a multiple of V) at step kstep of the block:
// all loads first, so that each thread keeps its whole footprint in flight,
// then the updates, then the stores; the spikes' pushes last.
template <int H, int V, bool MULTI, int MODEL>
__device__ __forceinline__ void neurons_f32(const Act32& A, const ActDesc* __restrict__ D, uint32_t kstep, uint32_t step, uint32_t i) {
    uint8_t en[V], fp[V], fired[V];
    uint16_t net[V];
    float x[V], u[V], input[V];
    ld_b<V>(A.enabled + i, en);
    ld_b<V>(A.fired_prev + i, fp);
    if (MULTI) {
        ld_h<V>(A.net_of + i, net);
    }
    ld_f<V>(A.x + i, x);
    ld_f<V>(A.u + i, u);
    // the sums pushed at the step before (read and cleared; a block's first
    // step pulls instead)
    const bool pull = kstep == 0;
    int pushed[V] = {};
    if (D->has_edges && !pull) {
        int32_t* in = A.syn_in[step & 1u];
        ld_f<V>(reinterpret_cast<const float*>(in + i), reinterpret_cast<float(&)[V]>(pushed));
#pragma unroll
        for (int v = 0; v < V; ++v) {
            if (pushed[v] != 0) {
                in[i + v] = 0;
            }
        }
    }
    // Background draws: the same Philox blocks as the FP64 form, 24 bits of
    // each neuron's words; one block serves an even-odd pair of a network, so
    // a thread with two neurons of a pair draws once.  Draws are keyed on the
    // network's seed and the neuron's index in its network.
    uint32_t k24[V];
    uint32_t k24p[V] = {};
    u32x4 blk{ 0u, 0u, 0u, 0u };
    bool have = false;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const uint64_t seed = MULTI ? A.nets[net[k]].seed : A.seed1;
        const uint32_t local = MULTI ? i + k - A.nets[net[k]].first : i + k;
        const bool reuse = have && (local & 1u) && (!MULTI || net[k] == net[k - 1 < 0 ? 0 : k - 1]);
        if (!reuse) {
            blk = MULTI ? noise_block(seed, step, local) : noise_block_rk(A.rk0, A.rk1, step, local);
        }
        have = (local & 1u) == 0u;
        k24[k] = ((local & 1u) ? blk.z : blk.x) >> 8;
        if (MODEL == RL_MODEL_POISSON) {
            // the threshold draw of PoissonModelCPU, keyed as in the FP64 form
            const u32x4 w = MULTI ? draw(seed, step, local, 0u, STREAM_POISSON, 0u)
                                  : philox4x32_10_rk(u32x4{ step, local, 0u, (uint32_t)STREAM_POISSON << 24 }, A.rk0, A.rk1);
            k24p[k] = w.x >> 8;
        }
    }
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const float nu[3] = { 0.0f, 0.0f, 0.0f };  // calcium and growth: k_calcium_growth_f32
        double ca = 0.0;
        float d[3] = { 0.0f, 0.0f, 0.0f };
        const Grow32 G{};
        neuron_f32<H, MODEL, true, false>(A, D, i + k, en[k] != 0, fp[k], k24[k], k24p[k], nu, G, x[k], u[k], ca, d, input[k], fired[k], pull,
                                          pushed[k]);
    }
    if (A.input) {
        st_f<V>(A.input + i, input);
    }
    st_b<V>(A.fired_cur + i, fired);
    st_f<V>(A.x + i, x);
    st_f<V>(A.u + i, u);
    st_b<V>(A.hist + (kstep % kHistSteps) * A.hist_stride + i, fired);  // a disabled neuron's entry is not read
#pragma unroll
    for (int v = 0; v < V; ++v) {
        if (fired[v]) {
            push_spike32(A, D, kstep, step, i + v);
        }
    }
}

// H > 0: h_model fixed at compile time (the loop unrolls); BLOCK threads per
// block, V neurons per thread, striding over the neurons when the grid is one
// resident wave.  The last n % V neurons go one per thread.  Registers are
// capped for 1,536 resident threads per SM: the step waits on its loads, and
// more resident warps hide them (1M neurons with synapses: 15.1 -> 14.4 us per
// step with the calcium-and-growth replay).
template <int H, int BLOCK, int V, bool MULTI, int MODEL>
__global__ void __launch_bounds__(BLOCK, 1536 / BLOCK) k_activity_f32(Act32 A, const ActDesc* __restrict__ D, uint32_t k) {
    pdl_wait_then_release();  // every input is the previous step's output
    const uint32_t step = D->base_step + k;
    const uint32_t groups = A.n / V;
    const uint32_t tid = blockIdx.x * BLOCK + threadIdx.x;
    const uint32_t stride = gridDim.x * BLOCK;
    for (uint32_t g = tid; g < groups; g += stride) {
        neurons_f32<H, V, MULTI, MODEL>(A, D, k, step, g * V);
    }
    if (V > 1 && tid < A.n - groups * V) {
        neurons_f32<H, 1, MULTI, MODEL>(A, D, k, step, groups * V + tid);
    }
}

// One neuron's block of `nsteps` steps on registers (k_activity_f32_steps):
// neuron i of the context, `local` its index in its network, whose growth
// rates are nu and whose Philox round keys are rk0 / rk1.  A lane with `in`
// false holds no neuron but still draws for its lane pair.  With `share`, lanes
// 2m and 2m + 1 hold the even and odd member of one neuron pair (or the even
// member and an idle lane), whose background draws of a step are one Philox
// block (words x and z): the even lane computes the block of step k, the odd
// lane that of step k + 1, and each hands the other the word it needs, one
// block per lane for two steps.  The trip count is the same for the whole
// warp (the pair draws exchange words between lanes).
template <int H, bool MULTI, int MODEL>
__device__ __forceinline__ void neuron_steps_f32(const Act32& A, const ActDesc* __restrict__ D, uint32_t nsteps, uint8_t* __restrict__ fired_before_last,
                                                 uint32_t i, bool in, uint32_t local, bool share, const float (&nu)[3], const uint32_t (&rk0)[10],
                                                 const uint32_t (&rk1)[10]) {
    const uint32_t step0 = D->base_step;
    const bool en = in && A.enabled[i] != 0;
    uint8_t f = 0;
    float x = 0.0f, u = 0.0f;
    double ca = 0.0;
    float d[3] = { 0.0f, 0.0f, 0.0f };
    float tg = 0.0f;
    if (in) {
        if (A.target) {
            tg = A.target[i];
        }
        f = A.fired_prev[i];
        x = A.x[i];
        u = A.u[i];
        ca = A.calcium[i];
        d[0] = A.delta[0][i];
        d[1] = A.delta[1][i];
        d[2] = A.delta[2][i];
    }
    uint8_t f_before = f;
    float input = 0.0f;
    const Grow32 G = grow32_of(A, tg);
    auto one_step = [&](uint32_t step, uint32_t word) {
        uint32_t k24p = 0;
        if (MODEL == RL_MODEL_POISSON && en) {
            // the threshold draw of PoissonModelCPU, keyed as in the FP64 form
            k24p = philox4x32_10_rk(u32x4{ step, local, 0u, (uint32_t)STREAM_POISSON << 24 }, rk0, rk1).x >> 8;
        }
        uint8_t fired;
        neuron_f32<H, MODEL, false>(A, D, i, en, f, word >> 8, k24p, nu, G, x, u, ca, d, input, fired);
        f_before = f;
        f = fired;
    };
    uint32_t k = 0;
    if (share) {
        const bool odd = (threadIdx.x & 1u) != 0;
        for (; k + 1 < nsteps; k += 2) {
            const uint32_t st = step0 + k + (odd ? 1u : 0u);
            const u32x4 blk = noise_block_rk(rk0, rk1, st, local);
            const uint32_t got = __shfl_xor_sync(0xFFFFFFFFu, odd ? blk.x : blk.z, 1);
            const uint32_t own = odd ? blk.z : blk.x;
            one_step(step0 + k, odd ? got : own);
            one_step(step0 + k + 1, odd ? own : got);
        }
    }
    for (; k < nsteps; ++k) {
        const uint32_t step = step0 + k;
        const u32x4 blk = noise_block_rk(rk0, rk1, step, local);
        one_step(step, (local & 1u) ? blk.z : blk.x);
    }
    if (in) {
        A.x[i] = x;
        A.u[i] = u;
        A.calcium[i] = ca;
        A.delta[0][i] = d[0];
        A.delta[1][i] = d[1];
        A.delta[2][i] = d[2];
        if (A.input) {
            A.input[i] = input;
        }
        A.fired_cur[i] = f;
        fired_before_last[i] = f_before;
    }
}

// A block of `nsteps` steps in one launch, for a network without synapses: a
// neuron's step then reads nothing of the other neurons, so each thread
// carries its neuron's state through the block in registers.  The same
// per-step function and draws as k_activity_f32, so the same bits; the spike
// flags of the last step go to A.fired_cur and those of the step before to
// fired_before_last, the input of the last step to A.input.  A batched context
// (MULTI) runs its neurons in the blocks of A.blocks, each of one network and
// starting at an even index of it (a multiple of kNetBlock), so that its seed,
// round keys and growth rates are the block's and every lane pair holds a
// neuron pair.
template <int H, int BLOCK, bool MULTI, int MODEL>
__global__ void __launch_bounds__(BLOCK) k_activity_f32_steps(Act32 A, const ActDesc* __restrict__ D, uint32_t nsteps,
                                                              uint8_t* __restrict__ fired_before_last) {
    pdl_wait_then_release();  // every input is the previous launch's output
    if constexpr (MULTI) {
        static_assert(BLOCK == (int)kNetBlock, "a thread block is a block of A.blocks");
        for (uint32_t b = blockIdx.x; b < A.num_blocks; b += gridDim.x) {
            const NetBlock B = A.blocks[b];
            const NetInfo& N = A.nets[B.net];
            const uint64_t seed = N.seed;
            uint32_t rk0[10], rk1[10];
#pragma unroll
            for (int r = 0; r < 10; ++r) {
                rk0[r] = (uint32_t)seed + (uint32_t)r * 0x9E3779B9u;
                rk1[r] = (uint32_t)(seed >> 32) + (uint32_t)r * 0xBB67AE85u;
            }
            const float nu[3] = { N.nu32[0], N.nu32[1], N.nu32[2] };
            neuron_steps_f32<H, true, MODEL>(A, D, nsteps, fired_before_last, B.first + threadIdx.x, threadIdx.x < B.count,
                                             B.first - N.first + threadIdx.x, true, nu, rk0, rk1);
        }
    } else {
        const uint32_t stride = gridDim.x * BLOCK;
        for (uint32_t base = blockIdx.x * BLOCK; base < A.n; base += stride) {
            const uint32_t i = base + threadIdx.x;
            neuron_steps_f32<H, false, MODEL>(A, D, nsteps, fired_before_last, i, i < A.n, i, true, A.nu1, A.rk0, A.rk1);
        }
    }
}

// Calcium and the growth deltas of the last m steps of one launch per step
// from the spike history (row j: the chunk's step j), with the state in
// registers: the same function and order as step by step, so the same bits.
// A disabled neuron keeps its calcium and deltas.
template <bool MULTI>
__global__ void __launch_bounds__(256) k_calcium_growth_f32(Act32 A, uint32_t row0, uint32_t m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n || !A.enabled[i]) {
        return;
    }
    float nu[3] = { A.nu1[0], A.nu1[1], A.nu1[2] };
    if (MULTI) {
        const NetInfo& N = A.nets[A.net_of[i]];
        nu[0] = N.nu32[0];
        nu[1] = N.nu32[1];
        nu[2] = N.nu32[2];
    }
    const Grow32 G = grow32_of(A, A.target ? A.target[i] : 0.0f);
    double ca = A.calcium[i];
    float d[3] = { A.delta[0][i], A.delta[1][i], A.delta[2][i] };
    const uint8_t* __restrict__ h = A.hist + row0 * A.hist_stride + i;
#pragma unroll 4
    for (uint32_t j = 0; j < m; ++j) {
        calcium_growth_f32(A, h[j * A.hist_stride], nu, G, ca, d);
    }
    A.calcium[i] = ca;
    A.delta[0][i] = d[0];
    A.delta[1][i] = d[1];
    A.delta[2][i] = d[2];
}

// ElementBaseBase::update with an FP32 delta.
__global__ void k_commit_f32(uint32_t n, const uint8_t* __restrict__ enabled, double* grown, float* delta, uint32_t* connected, uint32_t* vacant,
                             double retract, uint32_t* to_delete, unsigned long long* total, const unsigned long long* guard, int guard_n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    unsigned long long g = 0;
    for (int t = 0; t < guard_n; ++t) {
        g += guard[t];
    }
    if (g != 0) {
        return;  // an earlier type of this update left synapses to delete first
    }
    if (!enabled[i]) {
        to_delete[i] = 0u;
        return;
    }
    const double current_count = grown[i];
    const double current_delta = (double)delta[i];
    const uint32_t conn_int = connected[i];
    const double conn = (double)conn_int;
    const double new_vacant = (current_count - conn) + current_delta;
    const double keep = 1.0 - retract;
    uint32_t del = 0;
    if (new_vacant >= 0.0) {
        const double after = keep * new_vacant;
        grown[i] = after + conn;
        vacant[i] = (uint32_t)after;
    } else if (current_count + current_delta <= 0.0) {
        grown[i] = 0.0;
        vacant[i] = 0u;
        connected[i] = 0u;
        del = conn_int;
    } else {
        const double new_count = current_count + current_delta;
        const double new_conn = floor(new_count);
        grown[i] = keep * (new_count - new_conn) + new_conn;
        vacant[i] = 0u;
        connected[i] = (uint32_t)new_conn;
        del = (uint32_t)(conn - new_conn);
    }
    delta[i] = 0.0f;
    to_delete[i] = del;
    if (del) {
        atomicAdd(total, (unsigned long long)del);
    }
}

// FP64 records -> fixed-point records (in the frame of the node's network,
// found through the first neuron under the node) and FP32 cell lengths.
__global__ void k_pack(uint32_t m, const double4* __restrict__ r0, const double4* __restrict__ r1, const double* __restrict__ md, uint4* __restrict__ o0,
                       uint4* __restrict__ o1, const uint32_t* __restrict__ first_key, const uint32_t* __restrict__ morton,
                       const uint16_t* __restrict__ net_of, const NetInfo* __restrict__ nets) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) {
        return;
    }
    const QFrame& f = nets[net_of[morton[first_key[i]]]].frame;
    o0[i] = quantize_record(r0[i], f);
    o1[i] = quantize_record(r1[i], f);
}

// ----------------------------------------------------------- search
constexpr int kStack = kMaxLevels + 4;  // the diagnostic walk
enum : int { S_DISCARD = 0, S_EXPAND = 1, S_ACCEPT = 2 };

// The probability kernel's constants in FP32 (KernelParams).
struct Kernel32 {
    int type;
    int cutoff_inf;
    float k_minus_1, a, b, cutoff;
};

__device__ __forceinline__ float pow_pos32(float d, float y) {
    return y == 0.0f ? 1.0f : (y == 1.0f ? d : exp2f(y * __log2f(d)));
}

// Attraction of a cell at distance d (FP32) for the non-Gaussian kernels.
__device__ __forceinline__ float kernel_prob32(const Kernel32& K, float d) {
    if (K.type == RL_KERNEL_GAMMA) {
        return K.a * pow_pos32(d, K.k_minus_1) * __expf(d * K.b);
    }
    if (K.type == RL_KERNEL_LINEAR) {
        return K.cutoff_inf ? 1.0f : (d > K.cutoff ? 0.0f : 1.0f - __fdividef(d, K.cutoff));
    }
    const float f2 = pow_pos32(d, K.k_minus_1);  // Weibull
    return K.a * f2 * __expf(-K.b * f2 * d);
}

struct Search32 {
    const uint4* rec;
    const uint4* meta;  // topo, escape link, FP32 cell length (k_meta)
    uint32_t num_nodes;
    const uint32_t* first_key;  // Morton rank of the first neuron under a node
    const uint32_t* leaf_of;    // neuron -> leaf node
    uint32_t* tasks;    // persistent form: warp tasks handed out so far
    const double *px, *py, *pz;
    const uint32_t* list_src;
    const uint32_t* list_j;
    const uint32_t* seg_warp;
    const uint64_t* seg_begin;
    const uint64_t* seg_end;
    const uint32_t* seg_net;
    uint32_t num_segs;
    const NetInfo* nets;
    int32_t* target;
    float mu;
    uint32_t step;
    uint32_t* err;
    Kernel32 kernel;
};

// Parameters of the network a warp searches in.
struct Net32 {
    float theta;
    float inv_sigma2;
    uint64_t seed;
    uint32_t root;
    uint32_t first;
    float quantum;
};

struct KSum {
    float s, c;
    __device__ __forceinline__ void add(float x) {
        const float y = x - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

struct E32 {
    int status;
    float w;
};

// A node's topology and FP32 cell length from its meta entry.
__device__ __forceinline__ uint2 mtopo(const uint4& m) {
    return make_uint2(m.x, m.y);
}
__device__ __forceinline__ float mmaxdim(const uint4& m) {
    return __uint_as_float(m.w);
}

// Euclidean length in FP32 as d2 * rsqrt(d2) (MUFU.RSQ, relative error below
// 2e-7); 0 for a zero vector.  The precision form's error budget (1e-5 on
// selection probabilities) leaves room for it.
__device__ __forceinline__ float dist32(float dx, float dy, float dz) {
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    return d2 > 0.0f ? d2 * rsqrtf(d2) : 0.0f;
}

// Source position in the fixed-point frame.
struct QPos {
    uint32_t x, y, z;
};

__device__ __forceinline__ float qdiff(uint32_t a, uint32_t b, float quantum) {
    return (float)(int32_t)(a - b) * quantum;
}

__device__ __forceinline__ E32 eval32(const uint4& r, uint2 t, float md, const QPos& s, uint32_t source, const Search32& A, const Net32& W, bool fb) {
    E32 e{ S_DISCARD, 0.0f };
    const uint32_t cnt = r.w;
    if (cnt == 0) {
        return e;
    }
    const float q = W.quantum;
    const float dx = qdiff(r.x, s.x, q), dy = qdiff(r.y, s.y, q), dz = qdiff(r.z, s.z, q);
    const float d = dist32(dx, dy, dz);
    if (d == 0.0f) {
        return e;
    }
    const bool leaf = topo_leaf(t.y);
    if (!leaf && !(md < W.theta * d)) {
        e.status = S_EXPAND;
        return e;
    }
    e.status = S_ACCEPT;
    if (leaf && t.x == source) {
        e.w = 0.0f;
    } else if (!fb) {
        if (A.kernel.type == RL_KERNEL_GAUSSIAN) {
            const float dm = d - A.mu;
            e.w = __expf(-(dm * dm) * W.inv_sigma2) * (float)cnt;
        } else {
            e.w = kernel_prob32(A.kernel, d) * (float)cnt;
        }
    } else {
        e.w = __fdividef((float)cnt, d);
    }
    return e;
}

__device__ __forceinline__ uint32_t child_of(uint2 t, int oct) {
    return t.x + (uint32_t)__popc(topo_mask(t.y) & ((1u << oct) - 1u));
}

__device__ __forceinline__ float threshold32(float total, const Search32& A, const Net32& W, uint32_t source, uint32_t j, uint32_t depth) {
    const u32x4 w = draw(W.seed, A.step, source - W.first, j, STREAM_BH_PICK, depth);
    float r = (float)(w.x >> 8) * 5.9604644775390625e-8f * total;  // [0, total)
    return r > 0.0f ? r : 1.0e-38f;
}

struct Walk32 {
    KSum sum;
    int32_t picked;
};

// Shared-memory copy of the first nodes (the top octree levels) in the
// persistent form; n = 0 elsewhere.
struct Hot32 {
    const uint4* rec;
    const uint4* meta;
    uint32_t n;
};

template <bool HOT>
__device__ __forceinline__ void load_node32(const Search32& A, const Hot32& H, uint32_t i, uint4& r, uint4& m) {
    if (HOT && i < H.n) {
        r = H.rec[i];
        m = H.meta[i];
    } else {
        r = A.rec[i];
        m = A.meta[i];
    }
}

// Walks without a stack through the escape links, in the reference's
// depth-first order (see the FP64 search).
__device__ __forceinline__ uint32_t last_child32(uint2 t) {
    return t.x + (uint32_t)__popc(topo_mask(t.y)) - 1u;
}

template <bool HOT>
__device__ Walk32 lane_walk32(const Search32& A, const Hot32& H, const Net32& W, uint32_t sub, bool include_root, KSum start, bool pick, float r,
                              const QPos& sp, uint32_t source, bool fb, bool& bad) {
    Walk32 res{ start, -1 };
    uint4 rs, ms;
    load_node32<HOT>(A, H, sub, rs, ms);
    const uint2 ts = mtopo(ms);
    if (include_root) {
        const E32 e = eval32(rs, ts, mmaxdim(ms), sp, source, A, W, fb);
        if (e.status == S_ACCEPT) {
            res.sum.add(e.w);
            if (pick && res.sum.s >= r) {
                res.picked = (int32_t)sub;
            }
            return res;
        }
        if (e.status == S_DISCARD) {
            return res;
        }
    }
    const uint32_t end = ms.z;
    uint32_t node = last_child32(ts);
    for (uint32_t guard = 0; node != end; ++guard) {
        if (node >= A.num_nodes || guard >= A.num_nodes) {
            bad = true;
            return res;
        }
        uint4 rr, mm;
        load_node32<HOT>(A, H, node, rr, mm);
        const uint2 tt = mtopo(mm);
        const E32 e = eval32(rr, tt, mmaxdim(mm), sp, source, A, W, fb);
        if (e.status == S_ACCEPT) {
            res.sum.add(e.w);
            if (pick && res.sum.s >= r) {
                res.picked = (int32_t)node;
                return res;
            }
        }
        node = e.status == S_EXPAND ? last_child32(tt) : mm.z;
    }
    return res;
}

// Checkpoints of a packet walk (see the FP64 search): the running sum before
// each root child and, where the lane expanded them, before each child of its
// level-1 and level-2 ancestors.
constexpr int kCp32PerLevel = 8;
struct Ancestry32 {
    uint32_t a1 = kNoNode, a1_first = 0, a1_n = 0;
    uint32_t a2 = kNoNode, a2_first = 0, a2_n = 0;
    bool valid2 = false, valid3 = false;
};

__device__ __forceinline__ uint32_t inner_children32(const uint4& m) {
    return topo_leaf(m.y) ? 0u : (uint32_t)__popc(topo_mask(m.y));
}

// Packet walk of the lanes in packet mask `pm` (see the FP64 search).
template <bool HOT>
__device__ KSum packet32(const Search32& A, const Hot32& H, const Net32& W, uint32_t pm, uint32_t lanes, const QPos& sp, uint32_t source,
                         uint32_t my_rank, bool fb, float2* cp, Ancestry32& an, bool& bad) {
    const int lane = threadIdx.x & 31;
    const bool me = (lanes >> lane) & 1u;
    KSum sum{ 0.0f, 0.0f };
    an = Ancestry32{};
    const uint4 rm = A.meta[W.root];
    const uint32_t first0 = rm.x;
    const uint32_t root_level = topo_level(rm.y);
    uint32_t node = last_child32(mtopo(rm));
    bool act = me;
    uint32_t resume = kNoNode;
    for (uint32_t guard = 0; node != kNoNode; ++guard) {
        if (node >= A.num_nodes || guard >= A.num_nodes) {
            bad = true;
            break;
        }
        if (!act && node == resume) {
            act = true;
            resume = kNoNode;
        }
        uint4 rr, mm;
        load_node32<HOT>(A, H, node, rr, mm);
        const uint2 tt = mtopo(mm);
        const uint32_t lvl = topo_level(mm.y) - root_level;
        if (lvl <= 3u) {  // the top of the tree: checkpoints (the branch is uniform)
            const float2 now = make_float2(sum.s, sum.c);
            if (lvl == 1u) {
                if (me) {
                    cp[node - first0] = now;
                    if (an.a1 == kNoNode && A.first_key[node] <= my_rank) {
                        an.a1 = node;
                        an.a1_first = mm.x;
                        an.a1_n = inner_children32(mm);
                    }
                }
            } else if (lvl == 2u) {
                if (act && node - an.a1_first < an.a1_n) {
                    cp[kCp32PerLevel + (node - an.a1_first)] = now;
                    an.valid2 = true;
                    if (an.a2 == kNoNode && A.first_key[node] <= my_rank) {
                        an.a2 = node;
                        an.a2_first = mm.x;
                        an.a2_n = inner_children32(mm);
                    }
                }
            } else if (lvl == 3u) {
                if (act && node - an.a2_first < an.a2_n) {
                    cp[2 * kCp32PerLevel + (node - an.a2_first)] = now;
                    an.valid3 = true;
                }
            }
        }
        int status = S_DISCARD;
        if (act) {
            const E32 e = eval32(rr, tt, mmaxdim(mm), sp, source, A, W, fb);
            status = e.status;
            if (e.status == S_ACCEPT) {
                sum.add(e.w);
            }
        }
        const uint32_t expand = __ballot_sync(pm, status == S_EXPAND);
        if (expand) {
            if (act && status != S_EXPAND) {
                act = false;
                resume = mm.z;
            }
            node = last_child32(tt);
        } else {
            node = mm.z;
        }
    }
    __syncwarp(pm);
    return sum;
}

__device__ __forceinline__ int crossing_child32(const float2* cp, uint32_t n, float r) {
    int k = -1;
    for (int q = (int)n - 1; q >= 0; --q) {
        if (cp[q].x < r) {
            k = q;
        } else {
            break;
        }
    }
    return k;
}

// The searches of one warp task (see the FP64 search).
template <int PW, bool HOT>
__device__ __forceinline__ void search_task32(const Search32& A, const Hot32& H, uint32_t warp_global) {
    const int lane = threadIdx.x & 31;
    const int pk = lane / PW;
    const uint32_t pm = PW == 32 ? 0xFFFFFFFFu : (((1u << PW) - 1u) << (pk * PW));
    if (warp_global >= A.seg_warp[A.num_segs]) {
        return;
    }
    uint32_t lo = 0, hi = A.num_segs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (A.seg_warp[mid] <= warp_global) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    const NetInfo& N = A.nets[A.seg_net[lo]];
    const Net32 W{ N.theta32, N.inv_sigma2_32, N.seed, A.seg_net[lo], N.first, N.frame.quantum };
    const uint64_t idx = A.seg_begin[lo] + (uint64_t)(warp_global - A.seg_warp[lo]) * 32 + lane;
    const bool active = idx < A.seg_end[lo];
    if (N.root_leaf) {
        if (active) {
            A.target[idx] = -1;
        }
        return;
    }
    const uint32_t source = active ? A.list_src[idx] : 0u;
    const uint32_t j = active ? A.list_j[idx] : 0u;
    const QFrame& F = N.frame;
    const QPos sp = active ? QPos{ quantize(A.px[source], F.origin[0], F.inv_quantum), quantize(A.py[source], F.origin[1], F.inv_quantum),
                                   quantize(A.pz[source], F.origin[2], F.inv_quantum) }
                           : QPos{ 0u, 0u, 0u };
    const uint32_t my_rank = active ? A.first_key[A.leaf_of[source]] : 0u;
    float2 cp[3 * kCp32PerLevel];
    Ancestry32 an;
    bool overflow = false;
    bool bad = false;
    const uint32_t lanes = __ballot_sync(pm, active);
    int32_t result = -1;
    bool done = !active;
    uint32_t sub = 0;
    if (lanes) {
        KSum total = packet32<HOT>(A, H, W, pm, lanes, sp, source, my_rank, false, cp, an, bad);
        bool fb = false;
        const uint32_t need_fb = __ballot_sync(pm, active && total.s == 0.0f);
        if (need_fb) {
            Ancestry32 an_fb;
            const KSum t2 = packet32<HOT>(A, H, W, pm, need_fb, sp, source, my_rank, true, cp, an_fb, bad);
            if ((need_fb >> lane) & 1u) {
                total = t2;
                fb = true;
                an = an_fb;
            }
        }
        done = done || total.s == 0.0f;
        if (!done) {
            const float r = threshold32(total.s, A, W, source, j, 0);
            const uint4 rm = A.meta[W.root];
            const int k1 = crossing_child32(cp, inner_children32(rm), r);
            if (k1 < 0) {
                done = true;
            } else {
                uint32_t c0 = rm.x + (uint32_t)k1;
                float2 start = cp[k1];
                if (an.valid2 && c0 == an.a1) {
                    const int k2 = crossing_child32(cp + kCp32PerLevel, an.a1_n, r);
                    if (k2 >= 0) {
                        c0 = an.a1_first + (uint32_t)k2;
                        start = cp[kCp32PerLevel + k2];
                        if (an.valid3 && c0 == an.a2) {
                            const int k3 = crossing_child32(cp + 2 * kCp32PerLevel, an.a2_n, r);
                            if (k3 >= 0) {
                                c0 = an.a2_first + (uint32_t)k3;
                                start = cp[2 * kCp32PerLevel + k3];
                            }
                        }
                    }
                }
                const Walk32 wr = lane_walk32<HOT>(A, H, W, c0, true, KSum{ start.x, start.y }, true, r, sp, source, fb, bad);
                if (wr.picked < 0) {
                    done = true;  // rounding left the crossing past the last candidate: no pick
                } else {
                    sub = (uint32_t)wr.picked;
                }
            }
        }
    }
    for (uint32_t depth = 1; !done; ++depth) {
        if (depth > (uint32_t)kMaxLevels + 2u) {
            overflow = true;
            break;
        }
        const uint2 st = mtopo(A.meta[sub]);
        if (topo_leaf(st.y)) {
            result = (int32_t)st.x;
            break;
        }
        Walk32 s1 = lane_walk32<HOT>(A, H, W, sub, false, KSum{ 0.0f, 0.0f }, false, 0.0f, sp, source, false, bad);
        bool f = false;
        if (s1.sum.s == 0.0f) {
            s1 = lane_walk32<HOT>(A, H, W, sub, false, KSum{ 0.0f, 0.0f }, false, 0.0f, sp, source, true, bad);
            f = true;
        }
        if (s1.sum.s == 0.0f || bad) {
            break;
        }
        const float r = threshold32(s1.sum.s, A, W, source, j, depth);
        const Walk32 s2 = lane_walk32<HOT>(A, H, W, sub, false, KSum{ 0.0f, 0.0f }, true, r, sp, source, f, bad);
        if (s2.picked < 0) {
            break;
        }
        sub = (uint32_t)s2.picked;
    }
    if (overflow) {
        atomicOr(A.err, (uint32_t)DERR_STACK);
        result = -1;
    }
    if (bad) {
        atomicOr(A.err, (uint32_t)DERR_WALK);
        result = -1;
    }
    if (active) {
        A.target[idx] = result;
    }
}

template <int WPB, int PW, int CAP>
__global__ void __launch_bounds__(WPB * 32, CAP ? 32 / WPB : 1) k_search_f32(Search32 A) {
    const int wib = threadIdx.x >> 5;
    search_task32<PW, false>(A, Hot32{ nullptr, nullptr, 0u }, blockIdx.x * WPB + wib);
}

// Persistent form with the top octree nodes in shared memory (see the FP64
// search).
template <int PW>
__global__ void __launch_bounds__(1024, 1) k_search_f32_hot(Search32 A, uint32_t hot) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint4* hrec = reinterpret_cast<uint4*>(smem);
    uint4* hmeta = hrec + hot;
    for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) {
        hrec[i] = A.rec[i];
        hmeta[i] = A.meta[i];
    }
    __syncthreads();
    const Hot32 H{ hrec, hmeta, hot };
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t total = A.seg_warp[A.num_segs];
    uint32_t w = blockIdx.x * 32 + wib;
    while (w < total) {
        search_task32<PW, true>(A, H, w);
        uint32_t next = 0;
        if (lane == 0) {
            next = atomicAdd(A.tasks, 1u) + gridDim.x * 32;
        }
        w = __shfl_sync(0xFFFFFFFFu, next, 0);
    }
}

// One search per warp (bh_wide.cuh) in the FP32 form: the same visiting
// order and the same Kahan sums as the packet kernels, so the same targets.
// Both signal types' lists in one launch (the FP64 form's WideArgs).
struct WideArgs32 {
    Search32 S[2];
    uint32_t num_tasks[2];
    WideSlot all;
    uint32_t cap;
    uint32_t slots;
    uint32_t* tasks;
    uint32_t* overflow;  // per type
};

__device__ int32_t wide_search32(const Search32& S, uint32_t cap, const WideSlot& P, const Net32& W, const QPos& sp, uint32_t source, uint32_t j,
                                 uint32_t* s_round) {
    uint32_t touched = 0;
    uint32_t sub = W.root;
    for (uint32_t depth = 0; depth <= (uint32_t)kMaxLevels + 2u; ++depth) {
        const uint4 sm = S.meta[sub];
        if (topo_leaf(sm.y)) {
            return depth == 0 ? -1 : (int32_t)sm.x;
        }
        auto collect = [&](bool fb) {
            return wide_collect(P, cap, sm.x, inner_children32(sm), s_round, touched, [&](uint32_t nd) {
                WideEval r{ S_DISCARD, 0.0, 0u, 0u, false };
                if (nd >= S.num_nodes) {
                    r.bad = true;
                    return r;
                }
                const uint4 mm = S.meta[nd];
                const E32 e = eval32(S.rec[nd], mtopo(mm), mmaxdim(mm), sp, source, S, W, fb);
                r.status = e.status;
                r.w = (double)e.w;
                if (e.status == S_EXPAND) {
                    r.nch = (uint32_t)__popc(topo_mask(mm.y));
                    r.first = mm.x;
                }
                return r;
            }, [&](uint32_t nd) {
                if (nd < S.num_nodes) {
                    prefetch_l1(&S.meta[nd]);
                    prefetch_l1(&S.rec[nd]);
                }
            });
        };
        int64_t got = collect(false);
        if (got == -1) {
            return kRedo;
        }
        if (got < 0) {
            atomicOr(S.err, (uint32_t)DERR_WALK);
            return -1;
        }
        float total = wide_running_sum32(P.ord_w, (uint32_t)got);
        if (total == 0.0f) {
            // every weight underflowed: count / distance weights (the same walk)
            __syncwarp();
            got = collect(true);
            if (got < 0) {
                return got == -1 ? kRedo : -1;
            }
            total = wide_running_sum32(P.ord_w, (uint32_t)got);
        }
        if (total == 0.0f) {
            return -1;
        }
        const float r = threshold32(total, S, W, source, j, depth);
        const int64_t pick = wide_pick(P.ord_w, P.ord_node, (uint32_t)got, (double)r);
        if (pick < 0) {
            return -1;  // rounding left the crossing past the last candidate: no pick
        }
        sub = (uint32_t)pick;
        __syncwarp();
    }
    atomicOr(S.err, (uint32_t)DERR_STACK);
    return -1;
}

template <int WPB>
__global__ void __launch_bounds__(WPB * 32, 2) k_search_wide32(WideArgs32 A) {
    __shared__ uint32_t s_round_all[WPB][kWideRounds + 1];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * WPB + (uint32_t)wib;
    if (slot >= A.slots) {
        return;  // whole warp
    }
    const uint64_t off = (uint64_t)slot * A.cap;
    const WideSlot P{ A.all.node + off, A.all.info + off, A.all.child + off, A.all.cnt + off, A.all.pos + off, A.all.ord_node + off, A.all.w + off,
                      A.all.ord_w + off };
    const uint32_t total0 = A.num_tasks[0];
    const uint32_t total_tasks = total0 + A.num_tasks[1];
    for (;;) {
        uint32_t task = 0;
        if (lane == 0) {
            task = atomicAdd(A.tasks, 1u);
        }
        task = __shfl_sync(0xFFFFFFFFu, task, 0);
        if (task >= total_tasks) {
            break;
        }
        const int t = task < total0 ? 0 : 1;
        const Search32& S = A.S[t];
        uint32_t seg = 0;
        uint64_t idx = 0;
        if (!wide_task_entry(task - (t ? total0 : 0u), S.seg_warp, S.seg_begin, S.seg_end, S.num_segs, seg, idx)) {
            continue;
        }
        const NetInfo& N = S.nets[S.seg_net[seg]];
        const Net32 W{ N.theta32, N.inv_sigma2_32, N.seed, S.seg_net[seg], N.first, N.frame.quantum };
        int32_t result = -1;
        if (!N.root_leaf) {
            const uint32_t source = S.list_src[idx];
            const QFrame& F = N.frame;
            const QPos sp{ quantize(S.px[source], F.origin[0], F.inv_quantum), quantize(S.py[source], F.origin[1], F.inv_quantum),
                           quantize(S.pz[source], F.origin[2], F.inv_quantum) };
            result = wide_search32(S, A.cap, P, W, sp, source, S.list_j[idx], s_round_all[wib]);
        }
        if (lane == 0) {
            S.target[idx] = result;
            if (result == kRedo) {
                atomicAdd(A.overflow + t, 1u);
            }
        }
        __syncwarp();
    }
}

using Search32Kernel = void (*)(Search32);

Search32Kernel fp32_search_kernel(const SearchVariant& v) {
#define RL_SV(w, p, c)                                            \
    if (v.hot == 0 && v.warps == w && v.packet == p && v.cap == c) { \
        return &k_search_f32<w, p, c>;                            \
    }
#define RL_SV2(w, p) RL_SV(w, p, 0) RL_SV(w, p, 1)
    RL_SV2(2, 32) RL_SV2(4, 32) RL_SV2(8, 32) RL_SV2(2, 16) RL_SV2(4, 16) RL_SV2(8, 16)
    RL_SV2(2, 4) RL_SV2(4, 4) RL_SV2(8, 4) RL_SV2(2, 1) RL_SV2(4, 1) RL_SV2(8, 1)
#undef RL_SV2
#undef RL_SV
    return nullptr;
}

// ----------------------------------------------------------- diagnostic
// The weights come from the functions the production searches evaluate every
// node with: evaluate (FP64, k_search) and eval32 (FP32, k_search_f32), on
// the searches' own parameters (A32: mu and kernel; W32: the network's theta,
// 1/sigma^2 and frame).
__global__ void k_candidates(const double4* rec64, const uint4* recq, const uint2* topo, const double* md64, const uint4* meta, double sx, double sy,
                             double sz, uint32_t source, uint32_t root, int precision, double theta, double mu, double sigma, uint32_t* nodes, double* w,
                             uint64_t capacity, unsigned long long* count, uint32_t* err, QFrame f, KernelParams K, Search32 A32, Net32 W32) {
    const QPos sp{ quantize(sx, f.origin[0], f.inv_quantum), quantize(sy, f.origin[1], f.inv_quantum), quantize(sz, f.origin[2], f.inv_quantum) };
    uint32_t fnode[kStack];
    uint32_t frem[kStack];
    int depth = 1;
    fnode[0] = root;
    frem[0] = topo_mask(topo[root].y);
    uint64_t k = 0;
    const double scale = -1.0 / (sigma * sigma);
    while (depth > 0) {
        const int top = depth - 1;
        const uint32_t rem = frem[top];
        if (rem == 0) {
            --depth;
            continue;
        }
        const int oct = 31 - __clz(rem);
        frem[top] = rem & ~(1u << oct);
        const uint32_t child = child_of(topo[fnode[top]], oct);
        const uint2 tt = topo[child];
        int status = S_DISCARD;
        double weight = 0.0;
        if (precision == RL_PRECISION_FP64) {
            const Eval e = evaluate(rec64[child], tt, md64[child], sx, sy, sz, source, theta, mu, scale, false, K);
            status = e.status == ST_ACCEPT ? S_ACCEPT : (e.status == ST_EXPAND ? S_EXPAND : S_DISCARD);
            weight = e.w;
        } else {
            const uint4 m = meta[child];
            const E32 e = eval32(recq[child], mtopo(m), mmaxdim(m), sp, source, A32, W32, false);
            status = e.status;
            weight = (double)e.w;
        }
        if (status == S_ACCEPT) {
            if (k < capacity) {
                nodes[k] = child;
                w[k] = weight;
            }
            ++k;
        } else if (status == S_EXPAND) {
            if (depth >= kStack) {
                atomicOr(err, (uint32_t)DERR_STACK);
                break;
            }
            fnode[depth] = child;
            frem[depth] = topo_mask(tt.y);
            ++depth;
        }
    }
    *count = k;
}

}  // namespace

void alloc_fp32(Ctx& c) {
    const size_t n = c.n;
    c.nr.x32.alloc(n);
    c.nr.u32.alloc(n);
    c.nr.input32.alloc(n);
    for (int t = 0; t < 3; ++t) {
        c.nr.delta32[t].alloc(n);
    }
    f32_from_f64(c);
}

void f32_from_f64(Ctx& c) {
    const uint32_t n = c.n;
    const unsigned b = blocks_for(n, 256);
    k_d2f<<<b, 256, 0, c.stream>>>(n, c.nr.x.p, c.nr.x32.p);
    RL_LAUNCH_CHECK();
    k_d2f<<<b, 256, 0, c.stream>>>(n, c.nr.u.p, c.nr.u32.p);
    RL_LAUNCH_CHECK();
    k_d2f<<<b, 256, 0, c.stream>>>(n, c.nr.input.p, c.nr.input32.p);
    RL_LAUNCH_CHECK();
    for (int t = 0; t < 3; ++t) {
        k_d2f<<<b, 256, 0, c.stream>>>(n, c.nr.delta[t].p, c.nr.delta32[t].p);
        RL_LAUNCH_CHECK();
    }
}

void target_f32_from_f64(Ctx& c) {
    c.nr.target32.ensure(c.n);
    k_d2f<<<blocks_for(c.n, 256), 256, 0, c.stream>>>(c.n, c.nr.target.p, c.nr.target32.p);
    RL_LAUNCH_CHECK();
}

void f64_from_f32(Ctx& c) {
    const uint32_t n = c.n;
    const unsigned b = blocks_for(n, 256);
    k_f2d<<<b, 256, 0, c.stream>>>(n, c.nr.x32.p, c.nr.x.p);
    RL_LAUNCH_CHECK();
    k_f2d<<<b, 256, 0, c.stream>>>(n, c.nr.u32.p, c.nr.u.p);
    RL_LAUNCH_CHECK();
    k_f2d<<<b, 256, 0, c.stream>>>(n, c.nr.input32.p, c.nr.input.p);
    RL_LAUNCH_CHECK();
    for (int t = 0; t < 3; ++t) {
        k_f2d<<<b, 256, 0, c.stream>>>(n, c.nr.delta32[t].p, c.nr.delta[t].p);
        RL_LAUNCH_CHECK();
    }
}

template <int H, int BLOCK, int V, int MODEL>
void launch_act32(Ctx& c, const ActVariant& v, const Act32& A, uint32_t kstep) {
    if (c.multi()) {
        launch_pdl(&k_activity_f32<H, BLOCK, V, true, MODEL>, act_grid(c, v, (const void*)&k_activity_f32<H, BLOCK, V, true, MODEL>), BLOCK, c.stream,
                   A, (const ActDesc*)c.act_desc.p, kstep);
    } else {
        launch_pdl(&k_activity_f32<H, BLOCK, V, false, MODEL>, act_grid(c, v, (const void*)&k_activity_f32<H, BLOCK, V, false, MODEL>), BLOCK,
                   c.stream, A, (const ActDesc*)c.act_desc.p, kstep);
    }
}

template <int H, int BLOCK, int MODEL>
void launch_act32_b(Ctx& c, const ActVariant& v, const Act32& A, uint32_t kstep) {
    switch (v.vec) {
        case 4:
            launch_act32<H, BLOCK, 4, MODEL>(c, v, A, kstep);
            break;
        case 2:
            launch_act32<H, BLOCK, 2, MODEL>(c, v, A, kstep);
            break;
        default:
            launch_act32<H, BLOCK, 1, MODEL>(c, v, A, kstep);
            break;
    }
}

template <int H, int MODEL = RL_MODEL_IZHIKEVICH>
void launch_act32_h(Ctx& c, const ActVariant& v, const Act32& A, uint32_t kstep) {
    switch (v.block) {
        case 128:
            launch_act32_b<H, 128, MODEL>(c, v, A, kstep);
            break;
        case 512:
            launch_act32_b<H, 512, MODEL>(c, v, A, kstep);
            break;
        default:
            launch_act32_b<H, 256, MODEL>(c, v, A, kstep);
            break;
    }
}

template <int H, int MODEL = RL_MODEL_IZHIKEVICH>
void launch_steps32(Ctx& c, const Act32& A, uint32_t nsteps, uint8_t* fired_before_last) {
    if (c.multi()) {
        launch_pdl(&k_activity_f32_steps<H, kNetBlock, true, MODEL>, c.num_net_blocks, kNetBlock, c.stream, A, (const ActDesc*)c.act_desc.p,
                   nsteps, fired_before_last);
    } else {
        launch_pdl(&k_activity_f32_steps<H, 128, false, MODEL>, blocks_for(c.n, 128), 128, c.stream, A, (const ActDesc*)c.act_desc.p, nsteps,
                   fired_before_last);
    }
}

Act32 act32_args(Ctx& c, uint32_t kstep, const uint8_t* fired_prev, uint8_t* fired_cur) {
    const rl_config& k = c.cfg;
    Act32 A;
    A.n = c.n;
    A.enabled = c.nr.enabled.p;
    A.fired_prev = fired_prev;
    A.fired_cur = fired_cur;
    A.x = c.nr.x32.p;
    A.u = c.nr.u32.p;
    A.input = kstep + 1 >= c.act_block_len ? c.nr.input32.p : nullptr;  // the block's last step stores the input
    A.calcium = c.nr.calcium.p;
    for (int t = 0; t < 3; ++t) {
        A.delta[t] = c.nr.delta32[t].p;
    }
    A.conductance = (float)k.conductance;
    A.noise_mean = (float)k.noise_mean;
    A.noise_stddev = (float)k.noise_stddev;
    A.h_model = k.h_model;
    const double sm = 1.0 / (double)k.h_model;
    A.s = (float)sm;
    A.sk1 = (float)(sm * k.iz_k1);
    A.sk2 = (float)(sm * k.iz_k2);
    A.sk3 = (float)(sm * k.iz_k3);
    A.sa = (float)(sm * k.iz_a);
    A.b = (float)k.iz_b;
    A.c = (float)k.iz_c;
    A.d = (float)k.iz_d;
    A.v_spike = (float)k.iz_v_spike;
    // h calcium substeps c <- c*a + b at once
    const long double s = 1.0L / (long double)k.h_calcium;
    const long double a = 1.0L + s * (-1.0L / (long double)k.tau_c);
    long double an = 1.0L, geo = 0.0L;
    for (uint32_t it = 0; it < k.h_calcium; ++it) {
        geo += an;
        an *= a;
    }
    A.ca_mul = (double)an;
    A.ca_add = (double)(s * (long double)k.beta * geo);
    const double factor_inv = 1.0 / 1.6651092223153955127063292897904020952611777045288814583336582344;
    for (int t = 0; t < 3; ++t) {
        const double eta = k.min_calcium[t];
        const double eps = k.target_calcium < eta ? eta : k.target_calcium;
        A.flat[t] = eta == eps;
        A.eta[t] = (float)eta;
        A.xi[t] = (float)((eta + eps) * 0.5);
        // scaled by sqrt(log2 e), so that exp(-q^2) is one exp2 of -(q')^2
        A.inv_zeta[t] = A.flat[t] ? 0.0f : (float)(1.2011224087864498 / ((eta - eps) * factor_inv));
    }
    A.target = c.target_uniform ? nullptr : c.nr.target32.p;
    A.kz = (float)(1.2011224087864498 / factor_inv);
    A.nets = c.d_nets.p;
    A.net_of = c.net_of.p;
    A.blocks = c.net_blocks.p;
    A.num_blocks = c.num_net_blocks;
    A.syn_in[0] = c.syn_in32[0].p;
    A.syn_in[1] = c.syn_in32[1].p;
    A.hist = c.spike_hist.p;
    A.hist_stride = hist_stride(c.n);
    A.seed1 = c.nets[0].seed;
    for (int r = 0; r < 10; ++r) {
        A.rk0[r] = (uint32_t)A.seed1 + (uint32_t)r * 0x9E3779B9u;
        A.rk1[r] = (uint32_t)(A.seed1 >> 32) + (uint32_t)r * 0xBB67AE85u;
    }
    for (int t = 0; t < 3; ++t) {
        A.nu1[t] = c.nets[0].nu32[t];
    }
    A.p_x0 = (float)k.poisson_x0;
    A.p_tau_inv = (float)(1.0 / k.poisson_tau_x);
    A.p_refractory = (float)k.poisson_refractory;
    A.f_a = (float)k.fhn_a;
    A.f_b = (float)k.fhn_b;
    A.f_phi = (float)k.fhn_phi;
    A.e_g_L = (float)k.aeif_g_L;
    A.e_E_L = (float)k.aeif_E_L;
    A.e_V_T = (float)k.aeif_V_T;
    A.e_g_L_d_T = (float)(k.aeif_g_L * k.aeif_d_T);
    A.e_d_T_inv = (float)(1.0 / k.aeif_d_T);
    A.e_tau_w_inv = (float)(1.0 / k.aeif_tau_w);
    A.e_C_inv = (float)(1.0 / k.aeif_C);
    A.e_a = (float)k.aeif_a;
    A.e_b = (float)k.aeif_b;
    A.e_V_spike = (float)k.aeif_V_spike;
    return A;
}

void launch_activity_f32(Ctx& c, uint32_t kstep, const uint8_t* fired_prev, uint8_t* fired_cur, const ActVariant& v) {
    const rl_config& k = c.cfg;
    const Act32 A = act32_args(c, kstep, fired_prev, fired_cur);
    if (k.neuron_model == RL_MODEL_POISSON) {
        launch_act32_h<0, RL_MODEL_POISSON>(c, v, A, kstep);
    } else if (k.neuron_model == RL_MODEL_FITZHUGH_NAGUMO) {
        launch_act32_h<0, RL_MODEL_FITZHUGH_NAGUMO>(c, v, A, kstep);
    } else if (k.neuron_model == RL_MODEL_AEIF) {
        launch_act32_h<0, RL_MODEL_AEIF>(c, v, A, kstep);
    } else if (k.h_model == 10) {
        launch_act32_h<10>(c, v, A, kstep);
    } else {
        launch_act32_h<0>(c, v, A, kstep);
    }
}

// The whole block of nsteps steps in one launch (a network without synapses).
void launch_activity_f32_steps(Ctx& c, uint32_t nsteps) {
    const rl_config& k = c.cfg;
    const int p0 = c.nr.cur & 1;
    const Act32 A = act32_args(c, nsteps - 1, c.nr.fired[p0].p, c.nr.fired[(p0 + (int)nsteps) & 1].p);
    uint8_t* before_last = c.nr.fired[(p0 + (int)nsteps - 1) & 1].p;
    if (k.neuron_model == RL_MODEL_POISSON) {
        launch_steps32<0, RL_MODEL_POISSON>(c, A, nsteps, before_last);
    } else if (k.neuron_model == RL_MODEL_FITZHUGH_NAGUMO) {
        launch_steps32<0, RL_MODEL_FITZHUGH_NAGUMO>(c, A, nsteps, before_last);
    } else if (k.neuron_model == RL_MODEL_AEIF) {
        launch_steps32<0, RL_MODEL_AEIF>(c, A, nsteps, before_last);
    } else if (k.h_model == 10) {
        launch_steps32<10>(c, A, nsteps, before_last);
    } else {
        launch_steps32<0>(c, A, nsteps, before_last);
    }
}

void launch_calcium_growth32(Ctx& c, uint32_t row0, uint32_t m, cudaStream_t st) {
    const Act32 A = act32_args(c, 0, nullptr, nullptr);
    const unsigned grid = blocks_for(c.n, 256);
    if (c.multi()) {
        k_calcium_growth_f32<true><<<grid, 256, 0, st>>>(A, row0, m);
    } else {
        k_calcium_growth_f32<false><<<grid, 256, 0, st>>>(A, row0, m);
    }
    RL_LAUNCH_CHECK();
}

void launch_commit_f32(Ctx& c, int type, unsigned long long* total, const unsigned long long* guard, int guard_n) {
    k_commit_f32<<<blocks_for(c.n, 256), 256, 0, c.stream>>>(c.n, c.nr.enabled.p, c.nr.grown[type].p, c.nr.delta32[type].p, c.nr.connected[type].p,
                                                             c.nr.vacant[type].p, c.cfg.retract_ratio[type], c.to_delete.p, total, guard, guard_n);
    RL_LAUNCH_CHECK();
}

uint64_t run_commit_f32(Ctx& c, int type) {
    unsigned long long* d_del = reinterpret_cast<unsigned long long*>(c.counters.p) + 1;
    RL_CUDA_TRY(cudaMemsetAsync(d_del, 0, sizeof(unsigned long long), c.stream));
    k_commit_f32<<<blocks_for(c.n, 256), 256, 0, c.stream>>>(c.n, c.nr.enabled.p, c.nr.grown[type].p, c.nr.delta32[type].p, c.nr.connected[type].p,
                                                             c.nr.vacant[type].p, c.cfg.retract_ratio[type], c.to_delete.p, d_del, nullptr, 0);
    RL_LAUNCH_CHECK();
    unsigned long long h = 0;
    RL_CUDA_TRY(cudaMemcpyAsync(&h, d_del, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    c.stats.bound_to_delete += h;
    return h;
}

void pack_tree_f32(Ctx& c) {
    Tree& T = c.tree;
    if (T.recq_valid) {
        return;  // kept in step by the incremental octree update
    }
    const uint32_t m = T.num_nodes;
    T.recq[0].ensure(m);
    T.recq[1].ensure(m);
    k_pack<<<blocks_for(m, 256), 256, 0, c.stream>>>(m, T.rec[0].p, T.rec[1].p, T.maxdim.p, T.recq[0].p, T.recq[1].p, T.first_key.p,
                                                     T.morton.p, c.net_of.p, c.d_nets.p);
    RL_LAUNCH_CHECK();
    T.recq_valid = true;
}

namespace {

// The FP32 search arguments of signal type `type`'s list.
Search32 search32_args(Ctx& c, int type, const uint32_t* seg_warp, const uint64_t* seg_begin, const uint64_t* seg_end, const uint32_t* seg_net,
                       uint32_t num_segs, uint32_t step, uint32_t* tasks) {
    Search32 A;
    A.rec = c.tree.recq[type].p;
    A.meta = c.tree.meta.p;
    A.num_nodes = c.tree.num_nodes;
    A.tasks = tasks;
    A.first_key = c.tree.first_key.p;
    A.leaf_of = c.tree.leaf_of.p;
    A.px = c.nr.px.p;
    A.py = c.nr.py.p;
    A.pz = c.nr.pz.p;
    A.list_src = c.search.src.p;
    A.list_j = c.search.jj.p;
    A.seg_warp = seg_warp;
    A.seg_begin = seg_begin;
    A.seg_end = seg_end;
    A.seg_net = seg_net;
    A.num_segs = num_segs;
    A.nets = c.d_nets.p;
    A.target = c.search.target.p;
    A.mu = (float)c.cfg.mu;
    A.step = step;
    A.err = c.err.p;
    A.kernel = Kernel32{ c.kernel.type, c.kernel.cutoff_inf, (float)c.kernel.k_minus_1, (float)c.kernel.a, (float)c.kernel.b, (float)c.kernel.cutoff };
    return A;
}

}  // namespace

void launch_search_f32(Ctx& c, int type, const uint32_t* seg_warp, const uint64_t* seg_begin, const uint64_t* seg_end, const uint32_t* seg_net,
                       uint32_t num_segs, uint32_t warps, uint32_t step, const SearchVariant& v, uint32_t* tasks) {
    const Search32 A = search32_args(c, type, seg_warp, seg_begin, seg_end, seg_net, num_segs, step, tasks);
    if (v.hot > 0) {
        const auto kern = v.packet == 16 ? &k_search_f32_hot<16> : &k_search_f32_hot<32>;
        const uint32_t hot = hot_nodes(c, v, 2 * sizeof(uint4));
        const size_t smem = (size_t)hot * 2 * sizeof(uint4);
        RL_CUDA_TRY(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const unsigned blocks = std::min<unsigned>((unsigned)c.num_sms, (warps + 31) / 32);
        kern<<<blocks, 1024, smem, c.stream>>>(A, hot);
        RL_LAUNCH_CHECK();
        return;
    }
    RL_CHECK(v.packet != 0, RL_ERR_INVALID, "one search per warp runs both types at once (launch_search_wide_f32)");
    const Search32Kernel kern = fp32_search_kernel(v);
    RL_CHECK(kern != nullptr, RL_ERR_INVALID, "no such search variant");
    const unsigned blocks = (warps + v.warps - 1) / v.warps;
    kern<<<blocks, v.warps * 32, 0, c.stream>>>(A);
    RL_LAUNCH_CHECK();
}

// One search per warp over both signal types' lists (warps[t] packet-layout
// warps of type t, 0 for a type without searches, num_segs[t] segments in
// c.search.seg_*[t]); a type with searches that did not fit their warp's
// scratch is redone by the packet kernel.
void launch_search_wide_f32(Ctx& c, const uint32_t (&warps)[2], uint32_t segs0, uint32_t segs1, uint32_t step) {
    constexpr int WPB = 4;
    Search& S = c.search;
    const uint32_t segs[2] = { segs0, segs1 };
    WideArgs32 W;
    for (int t = 0; t < 2; ++t) {
        W.S[t] = warps[t] ? search32_args(c, t, S.seg_warp[t].p, S.seg_begin[t].p, S.seg_end[t].p, S.seg_net[t].p, segs[t], step, S.tasks.p + t)
                          : Search32{};
        W.num_tasks[t] = warps[t] * 32u;
    }
    const uint32_t cap = wide_cap(c);
    const uint32_t slots = std::min<uint32_t>((warps[0] + warps[1]) * 32u, (uint32_t)c.num_sms * kWideWarpsPerSM);
    S.w_overflow.ensure(2);
    RL_CUDA_TRY(cudaMemsetAsync(S.tasks.p, 0, sizeof(uint32_t), c.stream));
    RL_CUDA_TRY(cudaMemsetAsync(S.w_overflow.p, 0, 2 * sizeof(uint32_t), c.stream));
    W.all = wide_scratch(c, slots, cap);
    W.cap = cap;
    W.slots = slots;
    W.tasks = S.tasks.p;
    W.overflow = S.w_overflow.p;
    k_search_wide32<WPB><<<(slots + WPB - 1) / WPB, WPB * 32, 0, c.stream>>>(W);
    RL_LAUNCH_CHECK();
    uint32_t over[2] = { 0, 0 };
    RL_CUDA_TRY(cudaMemcpyAsync(over, S.w_overflow.p, sizeof(over), cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    for (int t = 0; t < 2; ++t) {
        if (over[t]) {
            k_search_f32<2, 32, 1><<<(warps[t] + 1) / 2, 64, 0, c.stream>>>(W.S[t]);
            RL_LAUNCH_CHECK();
        }
    }
}

void candidate_weights(Ctx& c, uint32_t source, int precision, std::vector<uint32_t>& nodes, std::vector<double>& w) {
    RL_CHECK(source < c.n, RL_ERR_INVALID, "source out of range");
    uint16_t net = 0;
    RL_CUDA_TRY(cudaMemcpy(&net, c.net_of.p + source, sizeof(net), cudaMemcpyDeviceToHost));
    const NetInfo& N = c.nets[net];
    RL_CHECK(!N.root_leaf, RL_ERR_INVALID, "the network has a single neuron");
    if (precision == RL_PRECISION_FP32) {
        pack_tree_f32(c);
    }
    uint8_t sig = 0;
    double pos[3];
    RL_CUDA_TRY(cudaMemcpyAsync(&sig, c.nr.signal.p + source, 1, cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaMemcpyAsync(&pos[0], c.nr.px.p + source, 8, cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaMemcpyAsync(&pos[1], c.nr.py.p + source, 8, cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaMemcpyAsync(&pos[2], c.nr.pz.p + source, 8, cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    const uint64_t cap = 1u << 16;
    DBuf<uint32_t> dn;
    DBuf<double> dw;
    DBuf<unsigned long long> dc;
    dn.alloc(cap);
    dw.alloc(cap);
    dc.alloc(1);
    Search32 A32{};
    A32.mu = (float)c.cfg.mu;
    A32.kernel = Kernel32{ c.kernel.type, c.kernel.cutoff_inf, (float)c.kernel.k_minus_1, (float)c.kernel.a, (float)c.kernel.b, (float)c.kernel.cutoff };
    const Net32 W32{ N.theta32, N.inv_sigma2_32, N.seed, net, N.first, N.frame.quantum };
    k_candidates<<<1, 1, 0, c.stream>>>(c.tree.rec[sig].p, precision == RL_PRECISION_FP32 ? c.tree.recq[sig].p : nullptr, c.tree.topo.p, c.tree.maxdim.p,
                                        c.tree.meta.p, pos[0], pos[1], pos[2], source, net, precision,
                                        N.theta, c.cfg.mu, N.sigma, dn.p, dw.p, cap, dc.p, c.err.p, N.frame, c.kernel, A32, W32);
    RL_LAUNCH_CHECK();
    unsigned long long k = 0;
    RL_CUDA_TRY(cudaMemcpyAsync(&k, dc.p, sizeof(k), cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    check_device_error(c, "candidate weights");
    RL_CHECK(k <= cap, RL_ERR_OVERFLOW, "more than 65536 candidates");
    nodes.resize(k);
    w.resize(k);
    if (k) {
        RL_CUDA_TRY(cudaMemcpyAsync(nodes.data(), dn.p, k * 4, cudaMemcpyDeviceToHost, c.stream));
        RL_CUDA_TRY(cudaMemcpyAsync(w.data(), dw.p, k * 8, cudaMemcpyDeviceToHost, c.stream));
        RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    }
}

}  // namespace rl
