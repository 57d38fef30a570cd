// Fused activity step (input + Izhikevich + calcium + growth) and the commit
// of the synaptic elements at a plasticity update.
//
// Reference semantics (relearn/source/neurons), one rank, in the order of
// Simulation::simulate (sim/Simulation.cpp:443-453):
//   * CombinedActivityInputCPU::update_input_range: input = 0; += synaptic; += normal
//     - SynapticEquallyWeightedActivityInputCPU::update_local_input
//       (input/SynapticEquallyWeightedActivityInputCPU.cpp:21-48):
//       conductance * sum of the weights of in-edges whose source fired in the
//       previous step (an integer sum, exact in any order)
//     - NormalActivityInputCPU::update_input_range (input/NormalActivityInputCPU.cpp:21-39)
//   * IzhikevichModelCPU::update_activity (models/izhikevich/IzhikevichModelCPU.cpp:75-125)
//   * CalciumCalculatorCPU::update_current_calcium (calcium/CalciumCalculatorCPU.cpp:40-103)
//   * update_number_elements_openmp + gaussian_growth_curve
//     (synaptic_elements/SynapticElementsCPU.cpp:25-49, GrowthCurves.h:30-53)
//   * ElementBaseBase::update (synaptic_elements/ElementBaseBase.h:420-481) at a
//     plasticity update.
// All state is structure-of-arrays in HBM; one thread per neuron reads and
// writes each of its words once per step.
#include <memory>

#include <cooperative_groups.h>

#include "rl_context.cuh"
#include "rl_math.cuh"

namespace rl {
namespace {

struct ActArgs {
    uint32_t n;
    const uint8_t* enabled;
    const uint8_t* fired_prev;
    uint8_t* fired_cur;
    double* x;
    double* u;
    double* calcium;
    const double* target;
    double* input;
    double* delta0;
    double* delta1;
    double* delta2;
    double conductance, noise_mean, noise_stddev;
    double syn0;  // the synaptic input without in-edges: 0.0 + 0.0 * conductance
    uint32_t h_model, h_calcium;
    double a, ab, c, d, v_spike, k1, k2, k3, scale_m;
    double beta, tau_inv, scale_c;
    double eta[3];
    const NetInfo* nets;
    const uint16_t* net_of;
    const NetBlock* blocks;  // a batched context's neurons in blocks of one network
    uint32_t num_blocks;
    long long* syn_in[2];  // pushed synaptic sums by step parity (ActDesc)
    uint8_t* hist;         // spike history (kHistSteps rows of hist_stride bytes)
    size_t hist_stride;
    // a context with one network: its seed and growth rates (the kernel then
    // reads no network table)
    uint64_t seed1;
    double nu1[3];
    uint32_t rk0[10], rk1[10];  // that network's Philox round keys
    // one target calcium for every neuron: the growth curves' constants,
    // computed on the host with the same operations as growth_curve
    int uniform_target;
    int flat_u[3];
    double xi_u[3], zeta_u[3], zeta_inv_u[3];
    // other neuron models (neurons/models/*)
    double p_x0, p_tau_inv;  // Poisson
    uint32_t p_refractory;
    double f_a, f_b, f_phi;  // FitzHugh-Nagumo
    double e_g_L, e_E_L, e_V_T, e_d_T, e_d_T_inv, e_tau_w_inv, e_C_inv, e_a, e_b, e_V_spike;  // AEIF
};

__device__ __forceinline__ double growth_curve(double current, double eta, double eps) {
    if (eta == eps) {
        return current == eta ? 0.0 : -1.0;
    }
    const double factor_inv = 1.0 / 1.6651092223153955127063292897904020952611777045288814583336582344;
    const double xi = (eta + eps) * 0.5;
    const double zeta = (eta - eps) * factor_inv;
    const double diff = current - xi;
    const double quot = diff / zeta;
    const double prod = quot * quot;
    return rl_fma(2.0, rl_exp(-prod), -1.0);  // (2 e) - 1: 2 e is exact, so one rounding either way
}

// gaussian_growth_curve with xi and zeta of a uniform target (growth_curve's
// own operations, done once on the host).  The division by the constant zeta
// goes through its reciprocal y = RN(1/zeta), also from the host: q0 = diff*y,
// r = diff - zeta*q0 (exact with an FMA), q = q0 + r*y rounded once is the
// correctly rounded diff/zeta (Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34 (1990); it
// needs y correctly rounded and no overflow or underflow, which the growth
// curve's operands keep far from).  The same bits as the division, at three
// FP64 operations; 8.6e9 random quotients on a B200 showed no difference.
__device__ __forceinline__ double growth_curve_pre(double current, double eta, int flat, double xi, double zeta, double zeta_inv) {
    if (flat) {
        return current == eta ? 0.0 : -1.0;
    }
    const double diff = current - xi;
    const double q0 = diff * zeta_inv;
    const double r = rl_fma(-zeta, q0, diff);
    const double quot = rl_fma(r, zeta_inv, q0);  // == diff / zeta
    const double prod = quot * quot;
    return rl_fma(2.0, rl_exp(-prod), -1.0);  // (2 e) - 1, as in growth_curve
}

// growth_curve_pre without branches (rl_exp_flat; the eta == epsilon case
// selected), for the software-pipelined block kernel.
__device__ __forceinline__ double growth_curve_flat(double current, double eta, int flat, double xi, double zeta, double zeta_inv) {
    const double diff = current - xi;
    const double q0 = diff * zeta_inv;
    const double r = rl_fma(-zeta, q0, diff);
    const double quot = rl_fma(r, zeta_inv, q0);
    const double prod = quot * quot;
    const double g = rl_fma(2.0, rl_exp_flat_nonpos(-prod), -1.0);
    return flat ? (current == eta ? 0.0 : -1.0) : g;
}

// The network of neuron i: draws are keyed on the network's seed and the
// neuron's index in its network.
// A neuron's growth rates per element type, held in registers (read once per
// neuron, not per use).
struct Nu {
    double v[3];
};

template <bool MULTI>
__device__ __forceinline__ void neuron_net(const ActArgs& A, uint32_t i, uint64_t& seed, uint32_t& local, Nu& nu) {
    seed = A.seed1;
    local = i;
    nu = Nu{ { A.nu1[0], A.nu1[1], A.nu1[2] } };
    if (MULTI) {
        const NetInfo& N = A.nets[A.net_of[i]];
        seed = N.seed;
        local = i - N.first;
        nu = Nu{ { N.nu[0], N.nu[1], N.nu[2] } };
    }
}

// This step's input: the synaptic sum (an integer, exact in any order) times
// the conductance, then NormalActivityInputCPU's draw z.
__device__ __forceinline__ double step_input(const ActArgs& A, long long isum, double z) {
    double input = 0.0;
    input += (double)isum * A.conductance;
    input += A.noise_mean + A.noise_stddev * z;
    return input;
}

// The neuron model's h substeps on (x, u); returns the spike flag.  H > 0:
// h_model is H, fixed at compile time.  MODEL is the neuron model (RL_MODEL_*).
template <int H, int MODEL>
__device__ __forceinline__ uint8_t model_step(const ActArgs& A, uint32_t step, uint64_t seed, uint32_t local, double input, double& x,
                                              double& u) {
    double xv = x;
    double uv = u;
    uint8_t spiked = 0;
    const uint32_t hm = H > 0 ? (uint32_t)H : A.h_model;
    if (MODEL == RL_MODEL_IZHIKEVICH) {
        // IzhikevichModelCPU::update_activity (IzhikevichModelCPU.cpp:75-125)
#pragma unroll
        for (uint32_t it = 0; it < hm; ++it) {
            const double x_inc = (A.k1 * xv * xv) + (A.k2 * xv) + A.k3 - uv + input;
            const double u_inc = (A.ab * xv) - (A.a * uv);
            xv += x_inc * A.scale_m;
            uv += u_inc * A.scale_m;
            if (xv >= A.v_spike) {
                xv = A.c;
                uv += A.d;
                spiked = 1;
                break;
            }
        }
    } else if (MODEL == RL_MODEL_POISSON) {
        // PoissonModelCPU::update_activity (models/poisson/PoissonModelCPU.cpp):
        // u holds the refractory steps left
        for (uint32_t it = 0; it < hm; ++it) {
            xv += ((A.p_x0 - xv) * A.p_tau_inv + input) * A.scale_m;
        }
        if (uv == 0.0) {
            const double threshold = uniform01(draw(seed, step, local, 0u, STREAM_POISSON, 0u));
            if (xv >= threshold) {
                spiked = 1;
                uv = (double)A.p_refractory;
            }
        } else {
            uv -= 1.0;
        }
    } else if (MODEL == RL_MODEL_FITZHUGH_NAGUMO) {
        // FitzHughNagumoModelCPU::update_activity (models/fitzhughnagumo/FitzHughNagumoModelCPU.cpp):
        // no reset; the spike test follows the h substeps
        const double third = 1.0 / 3.0;
        for (uint32_t it = 0; it < hm; ++it) {
            const double x_inc = xv - (xv * xv * xv * third) - uv + input;
            const double w_inc = A.f_phi * (xv + A.f_a - A.f_b * uv);
            xv += x_inc * A.scale_m;
            uv += w_inc * A.scale_m;
        }
        spiked = (uv > xv - xv * xv * xv * third && xv > 1.0) ? 1 : 0;
    } else {
        // AEIFModelCPU::update_activity (models/aeif/AEIFModelCPU.cpp)
        for (uint32_t it = 0; it < hm; ++it) {
            const double linear_part = -A.e_g_L * (xv - A.e_E_L);
            const double exp_part = A.e_g_L * A.e_d_T * rl_exp((xv - A.e_V_T) * A.e_d_T_inv);
            const double x_inc = (linear_part + exp_part - uv + input) * A.e_C_inv;
            const double w_inc = (A.e_a * (xv - A.e_E_L) - uv) * A.e_tau_w_inv;
            xv += x_inc * A.scale_m;
            uv += w_inc * A.scale_m;
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
    return spiked;
}

// CalciumCalculatorCPU::update_current_calcium: h substeps of
// ca += (ca * (-1/tau) + beta * fired) / h.
template <int H>
__device__ __forceinline__ double calcium_step(const ActArgs& A, uint8_t spiked, double ca) {
    const uint32_t hc = H > 0 ? (uint32_t)H : A.h_calcium;
    if (spiked) {
        const double local_beta = A.beta * 1.0;
#pragma unroll
        for (uint32_t it = 0; it < hc; ++it) {
            ca += A.scale_c * (ca * A.tau_inv + local_beta);
        }
    } else {
        // local_beta is +0: x + 0 = x for x != 0, and where ca * tau_inv is a
        // signed zero the sign is lost again when the scaled term is added to ca
#pragma unroll
        for (uint32_t it = 0; it < hc; ++it) {
            ca += A.scale_c * (ca * A.tau_inv);
        }
    }
    return ca;
}

// The growth of element type t this step (update_number_elements_openmp with
// gaussian_growth_curve); tgt is the neuron's target calcium when the targets
// are not uniform.
__device__ __forceinline__ double growth_step(const ActArgs& A, int t, double ca, double tgt, const Nu& nu) {
    if (A.uniform_target) {
        return growth_curve_pre(ca, A.eta[t], A.flat_u[t], A.xi_u[t], A.zeta_u[t], A.zeta_inv_u[t]) * nu.v[t];
    }
    const double eta = A.eta[t];
    const double eps = tgt < eta ? eta : tgt;  // std::max(target, eta)
    return growth_curve(ca, eta, eps) * nu.v[t];
}

// The Izhikevich model's H substeps without the reference's break: the
// substeps run on, and the state at the first crossing is what the function
// returns — x = c and u = u(crossing) + d, as model_step leaves them — so the
// bits are model_step's.  The substeps after a crossing compute values that
// are discarded (they may grow to infinity; nothing traps).  The function has
// no branch (a branch ends the stretch of code the compiler schedules
// together), and a substep costs one select (the u of a first crossing) on
// top of the model's arithmetic.
template <int H>
__device__ __forceinline__ uint8_t izhikevich_frozen(const ActArgs& A, double input, double& x, double& u) {
    double xv = x;
    double uv = u;
    double u_cross = 0.0;
    bool done = false;
#pragma unroll
    for (int it = 0; it < H; ++it) {
        const double x_inc = (A.k1 * xv * xv) + (A.k2 * xv) + A.k3 - uv + input;
        const double u_inc = (A.ab * xv) - (A.a * uv);
        xv = xv + x_inc * A.scale_m;
        uv = uv + u_inc * A.scale_m;
        const bool first = !done && xv >= A.v_spike;
        u_cross = first ? uv : u_cross;
        done = done || first;
    }
    x = done ? A.c : xv;
    u = done ? u_cross + A.d : uv;
    return done ? 1 : 0;
}

// calcium_step without the branch on the spike: beta * fired is added in
// every substep, as the reference writes it (beta * 0 = +0 leaves every value
// as it was, the sign of a zero included).
template <int H>
__device__ __forceinline__ double calcium_flat(const ActArgs& A, uint8_t spiked, double ca) {
    const double local_beta = A.beta * (spiked ? 1.0 : 0.0);
#pragma unroll
    for (int it = 0; it < H; ++it) {
        ca += A.scale_c * (ca * A.tau_inv + local_beta);
    }
    return ca;
}

// Calcium and growth of one step (one target calcium for all neurons).
// MULTI false: the context's one network, whose growth rates the kernel
// reads from its parameters (nu is not used).
template <int H, bool MULTI>
__device__ __forceinline__ void calcium_growth_flat(const ActArgs& A, uint8_t spiked, const Nu& nu, double& ca, double& d0, double& d1,
                                                    double& d2) {
    ca = calcium_flat<H>(A, spiked, ca);
    d0 = d0 + growth_curve_flat(ca, A.eta[0], A.flat_u[0], A.xi_u[0], A.zeta_u[0], A.zeta_inv_u[0]) * (MULTI ? nu.v[0] : A.nu1[0]);
    d1 = d1 + growth_curve_flat(ca, A.eta[1], A.flat_u[1], A.xi_u[1], A.zeta_u[1], A.zeta_inv_u[1]) * (MULTI ? nu.v[1] : A.nu1[1]);
    d2 = d2 + growth_curve_flat(ca, A.eta[2], A.flat_u[2], A.xi_u[2], A.zeta_u[2], A.zeta_inv_u[2]) * (MULTI ? nu.v[2] : A.nu1[2]);
}

// m consecutive steps of an Izhikevich neuron without synaptic input (one
// target calcium for all neurons), software-pipelined: the model of step
// k + 1 reads only x and u, not the calcium and growth of step k, so each
// loop iteration computes both, and with every function in it free of
// branches the compiler interleaves the two chains of dependent FP64
// operations.  The operations and values are those of the step-by-step
// order, so the bits are too.  zs[k * stride] is step k's standard normal
// draw; `input` receives the last step's input, f and f_before the last two
// spike flags.
template <int H, bool MULTI>
__device__ __forceinline__ void izhikevich_chunk(const ActArgs& A, const double* zs, uint32_t stride, uint32_t m, const Nu& nu, double& xv,
                                                 double& uv, double& ca, double& d0, double& d1, double& d2, double& input, uint8_t& f,
                                                 uint8_t& f_before) {
    double in_k = A.syn0 + (A.noise_mean + A.noise_stddev * zs[0]);
    uint8_t sp = izhikevich_frozen<H>(A, in_k, xv, uv);
    for (uint32_t k = 0; k + 1 < m; ++k) {
        const double in_n = A.syn0 + (A.noise_mean + A.noise_stddev * zs[(k + 1) * stride]);
        const uint8_t sp_n = izhikevich_frozen<H>(A, in_n, xv, uv);
        calcium_growth_flat<H, MULTI>(A, sp, nu, ca, d0, d1, d2);
        f_before = f;
        f = sp;
        sp = sp_n;
        in_k = in_n;
    }
    calcium_growth_flat<H, MULTI>(A, sp, nu, ca, d0, d1, d2);
    f_before = f;
    f = sp;
    input = in_k;
}

// The synaptic input's integer sum: the weights of in-edges whose source
// fired in the previous step (exact in any order).
__device__ __forceinline__ long long synaptic_sum(const ActArgs& A, const ActDesc* __restrict__ D, uint32_t i) {
    long long isum = 0;
    if (D->has_edges) {
        const uint32_t* __restrict__ off = D->off;
        const uint32_t* __restrict__ src = D->src;
        const int32_t* __restrict__ wt = D->w;
        const uint32_t e0 = off[i], e1 = off[i + 1];
        for (uint32_t e = e0; e < e1; ++e) {
            if (A.fired_prev[src[e]]) {
                isum += wt[e];
            }
        }
    }
    return isum;
}

// Neuron i's synaptic sum at step k of the block: pulled over its in-edges at
// the block's first step, else the sum its sources pushed at the step before
// (read and cleared; every neuron clears its own entry, enabled or not).
__device__ __forceinline__ long long synaptic_sum_k(const ActArgs& A, const ActDesc* __restrict__ D, uint32_t k, uint32_t step, uint32_t i,
                                                    bool on) {
    if (!D->has_edges) {
        return 0;
    }
    if (k == 0) {
        return on ? synaptic_sum(A, D, i) : 0;
    }
    long long* in = A.syn_in[step & 1u];
    const long long s = in[i];
    if (s != 0) {
        in[i] = 0;
    }
    return on ? s : 0;
}

// A set spike flag of neuron i at step k of the block: its out-edges' weights
// go to their targets' sums of the next step (none after the block's last).
__device__ __forceinline__ void push_spike(const ActArgs& A, const ActDesc* __restrict__ D, uint32_t k, uint32_t step, uint32_t i) {
    if (!D->has_edges || k + 1 >= D->block_len) {
        return;
    }
    unsigned long long* next = reinterpret_cast<unsigned long long*>(A.syn_in[(step + 1u) & 1u]);
    const uint32_t e0 = D->out_off[i], e1 = D->out_off[i + 1];
    for (uint32_t j = e0; j < e1; ++j) {
        const uint32_t e = D->out_perm[j];
        atomicAdd(next + D->tgt[e], (unsigned long long)(long long)D->w[e]);  // two's complement: the signed sum
    }
}

// One enabled neuron's input and model step on state already in registers
// (loaded before the kernel's draw phase); `z` is the neuron's standard normal
// draw of this step.  Calcium and growth follow from the spike history at the
// end of the chunk (k_calcium_growth).
template <int H, int MODEL>
__device__ __forceinline__ uint8_t activity_neuron_regs(const ActArgs& A, uint32_t step, uint32_t i, uint64_t seed, uint32_t local, double z,
                                                        long long isum, double xv, double uv) {
    const double input = step_input(A, isum, z);
    if (A.input) {
        A.input[i] = input;
    }
    const uint8_t spiked = model_step<H, MODEL>(A, step, seed, local, input, xv, uv);
    A.x[i] = xv;
    A.u[i] = uv;
    A.fired_cur[i] = spiked;
    return spiked;
}

// One thread per neuron; with fewer blocks than neurons / BLOCK (the
// persistent shape) each thread strides over the neurons.  A neuron's state
// and synaptic sum are loaded first, so that their memory latency overlaps
// the draw and its tail queue.
// The background draw's tail piece (about 15 % of the draws, but some lane
// of nearly every warp) is run for the whole block together: lanes whose
// uniform falls in the tails queue it in shared memory, the first warps of the
// block evaluate the queue at full width, and each lane takes its value back.
// The same function as the per-lane evaluation, so the same bits.  The loop
// over a block's neurons has the same trip count in every thread (the block
// synchronises inside it).
template <int BLOCK, int H, int MODEL, bool MULTI, int V>
__global__ void __launch_bounds__(BLOCK) k_activity(ActArgs A, const ActDesc* __restrict__ D, uint32_t k) {
    __shared__ double s_p[V * BLOCK];
    __shared__ double s_z[V * BLOCK];
    __shared__ uint16_t s_who[V * BLOCK];
    __shared__ uint32_t s_cnt[2];
    pdl_wait_then_release();  // every input is the previous step's output
    const uint32_t step = D->base_step + k;
    const uint32_t lane = threadIdx.x & 31u;
    if (threadIdx.x < 2) {
        s_cnt[threadIdx.x] = 0u;
    }
    __syncthreads();
    const uint32_t stride = gridDim.x * V * BLOCK;
    // V = 2 in a context with one network: a thread's two neurons are the
    // even-odd pair 2t, 2t + 1 of its block's 2 BLOCK neurons, whose
    // background draws of a step are one Philox block (words x, y and z, w)
    constexpr bool PAIR = V == 2 && !MULTI;
    uint32_t parity = 0;
    for (uint32_t base = blockIdx.x * V * BLOCK; base < A.n; base += stride, parity ^= 1u) {
        uint32_t i[V];
        bool on[V], tail[V];
        uint64_t seed[V];
        uint32_t local[V];
        Nu nu[V];
        double p[V], z[V], xv[V], uv[V];
        long long isum[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            i[v] = base + (PAIR ? 2u * threadIdx.x + (uint32_t)v : (uint32_t)v * BLOCK + threadIdx.x);
            on[v] = i[v] < A.n && A.enabled[i[v]];
            seed[v] = 0;
            local[v] = 0;
            nu[v] = Nu{ { 0.0, 0.0, 0.0 } };
            p[v] = 0.5;
            xv[v] = uv[v] = 0.0;
            isum[v] = 0;
            if (i[v] < A.n) {
                isum[v] = synaptic_sum_k(A, D, k, step, i[v], on[v]);
            }
            if (on[v]) {
                xv[v] = A.x[i[v]];
                uv[v] = A.u[i[v]];
                neuron_net<MULTI>(A, i[v], seed[v], local[v], nu[v]);
                if (!PAIR) {
                    p[v] = MULTI ? noise_uniform(seed[v], step, local[v]) : noise_uniform_rk(A.rk0, A.rk1, step, local[v]);
                }
            }
        }
        if constexpr (PAIR) {
            if (on[0] || on[1]) {
                const u32x4 r = noise_block_rk(A.rk0, A.rk1, step, i[0]);
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    if (on[v]) {
                        p[v] = ((double)noise_bits53(r, i[v]) + 0.5) * 1.1102230246251565404e-16;  // noise_uniform_rk's open (0, 1)
                    }
                }
            }
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            tail[v] = on[v] && normal_in_tail(p[v]);
            const uint32_t mask = __ballot_sync(0xFFFFFFFFu, tail[v]);
            uint32_t first = 0;
            if (lane == 0 && mask) {
                first = atomicAdd(&s_cnt[parity], (uint32_t)__popc(mask));
            }
            first = __shfl_sync(0xFFFFFFFFu, first, 0);
            if (tail[v]) {
                const uint32_t slot = first + (uint32_t)__popc(mask & ((1u << lane) - 1u));
                s_p[slot] = p[v];
                s_who[slot] = (uint16_t)(v * BLOCK + threadIdx.x);
            }
            z[v] = on[v] && !tail[v] ? normal_quantile_central(p[v]) : 0.0;
        }
        __syncthreads();
        const uint32_t cnt = s_cnt[parity];
        for (uint32_t q = threadIdx.x; q < cnt; q += BLOCK) {
            s_z[s_who[q]] = normal_quantile_tail(s_p[q]);
        }
        if (threadIdx.x == 0) {
            s_cnt[parity ^ 1u] = 0u;  // the next round's counter; nobody reads it before the barrier below
        }
        __syncthreads();
#pragma unroll
        for (int v = 0; v < V; ++v) {
            if (tail[v]) {
                z[v] = s_z[v * BLOCK + threadIdx.x];
            }
        }
        bool done = false;
        uint8_t spike[V];
#pragma unroll
        for (int v = 0; v < V; ++v) {
            spike[v] = 0;
        }
        if constexpr (V == 2 && MODEL == RL_MODEL_IZHIKEVICH && H > 0) {
            // both neurons' steps in one stretch without branches, so that
            // the compiler interleaves their chains of FP64 operations
            double in[V];
            uint8_t sp[V];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                in[v] = step_input(A, isum[v], z[v]);
                sp[v] = izhikevich_frozen<H>(A, in[v], xv[v], uv[v]);
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                if (on[v]) {
                    if (A.input) {
                        A.input[i[v]] = in[v];
                    }
                    A.x[i[v]] = xv[v];
                    A.u[i[v]] = uv[v];
                    A.fired_cur[i[v]] = sp[v];
                    spike[v] = sp[v];
                }
            }
            done = true;
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
            if (on[v] && !done) {
                spike[v] = activity_neuron_regs<H, MODEL>(A, step, i[v], seed[v], local[v], z[v], isum[v], xv[v], uv[v]);
            } else if (!on[v] && i[v] < A.n) {
                if (A.input) {
                    A.input[i[v]] = 0.0;
                }
                spike[v] = A.fired_prev[i[v]];  // a disabled neuron keeps its flag (and its targets still read it)
                A.fired_cur[i[v]] = spike[v];
            }
            if (on[v]) {
                A.hist[(k % kHistSteps) * A.hist_stride + i[v]] = spike[v];
            }
        }
        // the spikes' pushes last, with the neurons' state already stored
#pragma unroll
        for (int v = 0; v < V; ++v) {
            if (spike[v]) {
                push_spike(A, D, k, step, i[v]);
            }
        }
    }
}

// Calcium and the growth deltas of m steps (a chunk of one launch per step)
// from the spike history: row row0 + j holds the spike flags of the chunk's
// step j.  A neuron's calcium and growth read nothing but its own spike flags,
// so they run here once per chunk with the state in registers instead of in
// every step's launch; the operations and their order are those of one step
// after the other, so the bits are the same.  A disabled neuron keeps its
// calcium, and its deltas become d + 0 (as at each of its steps).
template <int H, bool MULTI>
__global__ void __launch_bounds__(256) k_calcium_growth(ActArgs A, uint32_t row0, uint32_t m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) {
        return;
    }
    double d0 = A.delta0[i], d1 = A.delta1[i], d2 = A.delta2[i];
    if (A.enabled[i]) {
        uint64_t seed;
        uint32_t local;
        Nu nu;
        neuron_net<MULTI>(A, i, seed, local, nu);
        double ca = A.calcium[i];
        const uint8_t* __restrict__ h = A.hist + row0 * A.hist_stride + i;
        bool flat = false;
        if constexpr (H > 0) {
            if (A.uniform_target) {
#pragma unroll 4
                for (uint32_t j = 0; j < m; ++j) {
                    calcium_growth_flat<H, MULTI>(A, h[j * A.hist_stride], nu, ca, d0, d1, d2);
                }
                flat = true;
            }
        }
        if (!flat) {
            const double tgt = A.uniform_target ? 0.0 : A.target[i];
            for (uint32_t j = 0; j < m; ++j) {
                ca = calcium_step<H>(A, h[j * A.hist_stride], ca);
                d0 = d0 + growth_step(A, 0, ca, tgt, nu);
                d1 = d1 + growth_step(A, 1, ca, tgt, nu);
                d2 = d2 + growth_step(A, 2, ca, tgt, nu);
            }
        }
        A.calcium[i] = ca;
        A.delta0[i] = d0;
        A.delta1[i] = d1;
        A.delta2[i] = d2;
    } else {
        A.delta0[i] = d0 + 0.0;
        A.delta1[i] = d1 + 0.0;
        A.delta2[i] = d2 + 0.0;
    }
}

// Background draws a block-of-steps launch prepares per barrier round.
constexpr int kDrawChunk = 10;

// One neuron's block of `nsteps` steps on registers (k_activity_steps): neuron
// i of the context, `local` its index in its network, whose seed is `seed`
// (its round keys rk0 / rk1 in a context with one network) and whose growth
// rates are nu.  A lane with `in` false holds no
// neuron but still draws for its lane pair.  Lanes 2j and 2j + 1 hold a neuron
// pair (or its even member and an idle lane), whose draws of a step come from
// one Philox block: the even lane computes step k's block, the odd lane step
// k + 1's, and each hands the other the two words it needs (the same words as
// a block per lane).  `parity` selects the shared tail-queue counter of the
// next chunk.
template <int BLOCK, int H, int MODEL, bool MULTI>
__device__ __forceinline__ void neuron_steps64(const ActArgs& A, const ActDesc* __restrict__ D, uint32_t nsteps,
                                               uint8_t* __restrict__ fired_before_last, uint32_t i, bool in, uint64_t seed, uint32_t local,
                                               const Nu& nu, const uint32_t (&rk0)[10], const uint32_t (&rk1)[10], uint32_t& parity, double* s_z,
                                               uint16_t* s_who, uint32_t* s_cnt) {
    constexpr int S = kDrawChunk;
    const uint32_t step0 = D->base_step;
    const uint32_t lane = threadIdx.x & 31u;
    const bool on = in && A.enabled[i];
    double xv = 0.0, uv = 0.0, ca = 0.0, tgt = 0.0, d0 = 0.0, d1 = 0.0, d2 = 0.0, input = 0.0;
    uint8_t f = 0;
    if (in) {
        f = A.fired_prev[i];
        d0 = A.delta0[i];
        d1 = A.delta1[i];
        d2 = A.delta2[i];
    }
    if (on) {
        xv = A.x[i];
        uv = A.u[i];
        ca = A.calcium[i];
        tgt = A.uniform_target ? 0.0 : A.target[i];
    }
    uint8_t f_before = f;
    for (uint32_t k0 = 0; k0 < nsteps; k0 += S, parity ^= 1u) {
        const uint32_t m = nsteps - k0 < (uint32_t)S ? nsteps - k0 : (uint32_t)S;
        const uint32_t stepc = step0 + k0;
#pragma unroll
        for (int k = 0; k < S; k += 2) {
            uint64_t b[2];
            const uint32_t odd = lane & 1u;
            // a batched context derives the round keys from the seed as it goes
            // (twenty more registers would spill)
            const u32x4 r = MULTI ? noise_block(seed, stepc + (uint32_t)k + odd, local) : noise_block_rk(rk0, rk1, stepc + (uint32_t)k + odd, local);
            const uint32_t g0 = __shfl_xor_sync(0xFFFFFFFFu, odd ? r.x : r.z, 1);
            const uint32_t g1 = __shfl_xor_sync(0xFFFFFFFFu, odd ? r.y : r.w, 1);
            const uint64_t got = ((uint64_t)g0 << 21) | (uint64_t)(g1 >> 11);
            b[0] = odd ? got : (((uint64_t)r.x << 21) | (uint64_t)(r.y >> 11));
            b[1] = odd ? (((uint64_t)r.z << 21) | (uint64_t)(r.w >> 11)) : got;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const bool use = on && (uint32_t)(k + h) < m;
                const double p = ((double)b[h] + 0.5) * 1.1102230246251565404e-16;  // open (0, 1)
                const bool tail = use && normal_in_tail(p);
                const uint32_t mask = __ballot_sync(0xFFFFFFFFu, tail);
                uint32_t first = 0;
                if (lane == 0 && mask) {
                    first = atomicAdd(&s_cnt[parity], (uint32_t)__popc(mask));
                }
                first = __shfl_sync(0xFFFFFFFFu, first, 0);
                const uint32_t slot = (uint32_t)(k + h) * BLOCK + threadIdx.x;
                if (tail) {
                    s_who[first + (uint32_t)__popc(mask & ((1u << lane) - 1u))] = (uint16_t)slot;
                }
                s_z[slot] = tail ? p : (use ? normal_quantile_central(p) : 0.0);
            }
        }
        __syncthreads();
        const uint32_t cnt = s_cnt[parity];
        for (uint32_t q = threadIdx.x; q < cnt; q += BLOCK) {
            const uint32_t slot = s_who[q];
            s_z[slot] = normal_quantile_tail(s_z[slot]);
        }
        if (threadIdx.x == 0) {
            s_cnt[parity ^ 1u] = 0u;  // the next chunk's counter; nobody reads it before the barrier below
        }
        __syncthreads();
        bool piped = false;
        if constexpr (MODEL == RL_MODEL_IZHIKEVICH && H > 0) {
            if (on && A.uniform_target) {
                izhikevich_chunk<H, MULTI>(A, s_z + threadIdx.x, BLOCK, m, nu, xv, uv, ca, d0, d1, d2, input, f, f_before);
                piped = true;
            }
        }
        if (on && !piped) {
            for (uint32_t k = 0; k < m; ++k) {
                const uint32_t step = stepc + k;
                input = step_input(A, 0, s_z[k * BLOCK + threadIdx.x]);
                f_before = f;
                f = model_step<H, MODEL>(A, step, seed, local, input, xv, uv);
                ca = calcium_step<H>(A, f, ca);
                d0 = d0 + growth_step(A, 0, ca, tgt, nu);
                d1 = d1 + growth_step(A, 1, ca, tgt, nu);
                d2 = d2 + growth_step(A, 2, ca, tgt, nu);
            }
        }
    }
    if (on) {
        A.x[i] = xv;
        A.u[i] = uv;
        A.calcium[i] = ca;
        A.delta0[i] = d0;
        A.delta1[i] = d1;
        A.delta2[i] = d2;
    } else if (in) {
        A.delta0[i] = d0 + 0.0;
        A.delta1[i] = d1 + 0.0;
        A.delta2[i] = d2 + 0.0;
    }
    if (in) {
        if (A.input) {
            A.input[i] = on ? input : 0.0;
        }
        A.fired_cur[i] = f;
        fired_before_last[i] = f_before;
    }
}

// A block of `nsteps` steps in one launch, for a network without synapses:
// then a neuron's step reads nothing of the other neurons (its input is its
// own background draw), so each thread carries its neuron's state through the
// block in registers and touches memory once at each end.  The operations and
// their order are those of k_activity step by step, so the state is the same
// bits; so are both spike-flag buffers (the last step's flags in
// A.fired_cur, the step before's in fired_before_last) and the input (last
// step).  A disabled neuron keeps x, u, calcium and its spike flag; its
// deltas become d + 0 as in every step of k_activity.
//
// The draws do not depend on the state, so they are made kDrawChunk steps at a
// time: every thread evaluates its central-piece draws of those steps
// (independent of one another), queues its tail-piece ones in shared memory,
// the whole block evaluates the queue after one barrier, and after a second
// barrier each thread runs its steps on the draws.  Two barriers per chunk
// instead of two per step, and the tail queue of a chunk spreads over every
// warp of the block.  A batched context (MULTI) runs its neurons in the blocks
// of A.blocks, each of one network and starting at an even index of it (a
// multiple of kNetBlock), so that the seed and growth rates are the block's
// and every lane pair holds a neuron pair.
template <int BLOCK, int H, int MODEL, bool MULTI>
__global__ void __launch_bounds__(BLOCK, (MULTI ? 640 : 768) / BLOCK) k_activity_steps(ActArgs A, const ActDesc* __restrict__ D, uint32_t nsteps,
                                                                          uint8_t* __restrict__ fired_before_last) {
    __shared__ double s_z[kDrawChunk * BLOCK];      // draw of step k0 + k of thread t at k * BLOCK + t
    __shared__ uint16_t s_who[kDrawChunk * BLOCK];  // tail queue: slots of s_z holding a uniform to map
    __shared__ uint32_t s_cnt[2];
    pdl_wait_then_release();  // every input is the previous launch's output
    if (threadIdx.x < 2) {
        s_cnt[threadIdx.x] = 0u;
    }
    __syncthreads();
    uint32_t parity = 0;
    if constexpr (MULTI) {
        static_assert(BLOCK == (int)kNetBlock, "a thread block is a block of A.blocks");
        for (uint32_t b = blockIdx.x; b < A.num_blocks; b += gridDim.x) {
            const NetBlock B = A.blocks[b];
            const NetInfo& N = A.nets[B.net];
            const Nu nu{ { N.nu[0], N.nu[1], N.nu[2] } };
            neuron_steps64<BLOCK, H, MODEL, true>(A, D, nsteps, fired_before_last, B.first + threadIdx.x, threadIdx.x < B.count, N.seed,
                                                  B.first - N.first + threadIdx.x, nu, A.rk0, A.rk1, parity, s_z, s_who, s_cnt);
        }
    } else {
        const uint32_t stride = gridDim.x * BLOCK;
        const Nu nu{ { A.nu1[0], A.nu1[1], A.nu1[2] } };
        for (uint32_t base = blockIdx.x * BLOCK; base < A.n; base += stride) {
            const uint32_t i = base + threadIdx.x;
            neuron_steps64<BLOCK, H, MODEL, false>(A, D, nsteps, fired_before_last, i, i < A.n, A.seed1, i, nu, A.rk0, A.rk1, parity, s_z,
                                                   s_who, s_cnt);
        }
    }
}

struct CommitArgs {
    uint32_t n;
    const uint8_t* enabled;
    double* grown;
    double* delta;
    uint32_t* connected;
    uint32_t* vacant;
    double retract;
    uint32_t* to_delete;
    unsigned long long* total;
    const unsigned long long* guard;  // counts of the earlier types of this update
    int guard_n;                      // how many of them; any nonzero count skips the commit
};

__device__ __forceinline__ bool commit_guarded(const unsigned long long* guard, int guard_n) {
    unsigned long long g = 0;
    for (int t = 0; t < guard_n; ++t) {
        g += guard[t];
    }
    return g != 0;
}

// ElementBaseBase::update for one element type.
__global__ void k_commit(CommitArgs A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n || commit_guarded(A.guard, A.guard_n)) {
        return;
    }
    if (!A.enabled[i]) {
        A.to_delete[i] = 0u;
        return;
    }
    const double current_count = A.grown[i];
    const double current_delta = A.delta[i];
    const uint32_t conn_int = A.connected[i];
    const double conn = (double)conn_int;
    const double current_vacant = current_count - conn;
    const double new_vacant = current_vacant + current_delta;
    const double keep = 1.0 - A.retract;
    uint32_t del = 0;
    if (new_vacant >= 0.0) {
        const double after = keep * new_vacant;
        A.grown[i] = after + conn;
        A.delta[i] = 0.0;
        A.vacant[i] = (uint32_t)after;
    } else if (current_count + current_delta <= 0.0) {
        A.grown[i] = 0.0;
        A.delta[i] = 0.0;
        A.vacant[i] = 0u;
        A.connected[i] = 0u;
        del = conn_int;
    } else {
        const double new_count = current_count + current_delta;
        const double new_conn = floor(new_count);
        const double num_vacant = new_count - new_conn;
        A.grown[i] = (keep * num_vacant) + new_conn;
        A.delta[i] = 0.0;
        A.vacant[i] = 0u;
        A.connected[i] = (uint32_t)new_conn;
        del = (uint32_t)(conn - new_conn);
    }
    A.to_delete[i] = del;
    if (del) {
        atomicAdd(A.total, (unsigned long long)del);
    }
}

// Sum of v[i] over enabled neurons (the vacant axons the next search will
// start from), one atomic per block.
__global__ void k_sum_enabled(uint32_t n, const uint8_t* __restrict__ enabled, const uint32_t* __restrict__ v, unsigned long long* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t x = (i < n && enabled[i]) ? v[i] : 0u;
    for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_down_sync(0xFFFFFFFFu, x, o);
    }
    __shared__ uint32_t part[32];
    if ((threadIdx.x & 31) == 0) {
        part[threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long y = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0u;
        for (int o = 16; o > 0; o >>= 1) {
            y += __shfl_down_sync(0xFFFFFFFFu, y, o);
        }
        if (threadIdx.x == 0 && y) {
            atomicAdd(out, y);
        }
    }
}

}  // namespace

void launch_vacant_axon_count(Ctx& c, unsigned long long* out) {
    k_sum_enabled<<<blocks_for(c.n, 256), 256, 0, c.stream>>>(c.n, c.nr.enabled.p, c.nr.vacant[0].p, out);
    RL_LAUNCH_CHECK();
}

template <int BLOCK, int H, int MODEL, int V>
void launch_act64_v(Ctx& c, const ActVariant& v, const ActArgs& A, uint32_t kstep) {
    if (c.multi()) {
        launch_pdl(&k_activity<BLOCK, H, MODEL, true, V>, act_grid(c, v, (const void*)&k_activity<BLOCK, H, MODEL, true, V>), BLOCK, c.stream, A,
                   (const ActDesc*)c.act_desc.p, kstep);
    } else {
        launch_pdl(&k_activity<BLOCK, H, MODEL, false, V>, act_grid(c, v, (const void*)&k_activity<BLOCK, H, MODEL, false, V>), BLOCK, c.stream, A,
                   (const ActDesc*)c.act_desc.p, kstep);
    }
}

// One or two neurons per thread (rows i and i + BLOCK of a block's range).
template <int BLOCK, int H, int MODEL>
void launch_act64_b(Ctx& c, const ActVariant& v, const ActArgs& A, uint32_t kstep) {
    if (v.vec == 2) {
        launch_act64_v<BLOCK, H, MODEL, 2>(c, v, A, kstep);
    } else {
        launch_act64_v<BLOCK, H, MODEL, 1>(c, v, A, kstep);
    }
}

template <int H, int MODEL>
void launch_act64_m(Ctx& c, const ActVariant& v, const ActArgs& A, uint32_t kstep) {
    switch (v.block) {
        case 128:
            launch_act64_b<128, H, MODEL>(c, v, A, kstep);
            break;
        case 512:
            launch_act64_b<512, H, MODEL>(c, v, A, kstep);
            break;
        default:
            launch_act64_b<256, H, MODEL>(c, v, A, kstep);
            break;
    }
}

template <int H>
void launch_act64(Ctx& c, const ActVariant& v, const ActArgs& A, uint32_t kstep) {
    switch (c.cfg.neuron_model) {
        case RL_MODEL_POISSON:
            launch_act64_m<H, RL_MODEL_POISSON>(c, v, A, kstep);
            break;
        case RL_MODEL_FITZHUGH_NAGUMO:
            launch_act64_m<H, RL_MODEL_FITZHUGH_NAGUMO>(c, v, A, kstep);
            break;
        case RL_MODEL_AEIF:
            launch_act64_m<H, RL_MODEL_AEIF>(c, v, A, kstep);
            break;
        default:
            launch_act64_m<H, RL_MODEL_IZHIKEVICH>(c, v, A, kstep);
            break;
    }
}

namespace {

ActArgs act64_args(Ctx& c, uint32_t kstep, const uint8_t* fired_prev, uint8_t* fired_cur) {
    const rl_config& k = c.cfg;
    ActArgs A;
    A.n = c.n;
    A.enabled = c.nr.enabled.p;
    A.fired_prev = fired_prev;
    A.fired_cur = fired_cur;
    A.x = c.nr.x.p;
    A.u = c.nr.u.p;
    A.calcium = c.nr.calcium.p;
    A.target = c.nr.target.p;
    // the input is state a caller can read only between blocks: the block's
    // last step stores it, the others skip the store
    A.input = kstep + 1 >= c.act_block_len ? c.nr.input.p : nullptr;
    A.delta0 = c.nr.delta[0].p;
    A.delta1 = c.nr.delta[1].p;
    A.delta2 = c.nr.delta[2].p;
    A.conductance = k.conductance;
    A.noise_mean = k.noise_mean;
    A.noise_stddev = k.noise_stddev;
    {
        volatile double zero = 0.0;  // evaluated at run time, as the kernels' step_input does
        A.syn0 = zero + zero * k.conductance;
    }
    A.h_model = k.h_model;
    A.h_calcium = k.h_calcium;
    A.a = k.iz_a;
    A.ab = k.iz_a * k.iz_b;
    A.c = k.iz_c;
    A.d = k.iz_d;
    A.v_spike = k.iz_v_spike;
    A.k1 = k.iz_k1;
    A.k2 = k.iz_k2;
    A.k3 = k.iz_k3;
    A.scale_m = 1.0 / (double)k.h_model;
    A.beta = k.beta;
    A.tau_inv = -1.0 / k.tau_c;
    A.scale_c = 1.0 / (double)k.h_calcium;
    for (int t = 0; t < 3; ++t) {
        A.eta[t] = k.min_calcium[t];
    }
    A.nets = c.d_nets.p;
    A.net_of = c.net_of.p;
    A.blocks = c.net_blocks.p;
    A.num_blocks = c.num_net_blocks;
    A.syn_in[0] = c.syn_in64[0].p;
    A.syn_in[1] = c.syn_in64[1].p;
    A.hist = c.spike_hist.p;
    A.hist_stride = hist_stride(c.n);
    A.seed1 = c.nets[0].seed;
    for (int r = 0; r < 10; ++r) {
        A.rk0[r] = (uint32_t)A.seed1 + (uint32_t)r * 0x9E3779B9u;
        A.rk1[r] = (uint32_t)(A.seed1 >> 32) + (uint32_t)r * 0xBB67AE85u;
    }
    A.uniform_target = c.target_uniform ? 1 : 0;
    const double factor_inv = 1.0 / 1.6651092223153955127063292897904020952611777045288814583336582344;
    for (int t = 0; t < 3; ++t) {
        A.nu1[t] = c.nets[0].nu[t];
        // gaussian_growth_curve's constants for the one target, in its operation order
        const double eta = k.min_calcium[t];
        const double tgt = k.target_calcium;
        const double eps = tgt < eta ? eta : tgt;
        A.flat_u[t] = eta == eps ? 1 : 0;
        A.xi_u[t] = (eta + eps) * 0.5;
        A.zeta_u[t] = (eta - eps) * factor_inv;
        A.zeta_inv_u[t] = A.flat_u[t] ? 0.0 : 1.0 / A.zeta_u[t];
    }
    A.p_x0 = k.poisson_x0;
    A.p_tau_inv = 1.0 / k.poisson_tau_x;
    A.p_refractory = k.poisson_refractory;
    A.f_a = k.fhn_a;
    A.f_b = k.fhn_b;
    A.f_phi = k.fhn_phi;
    A.e_g_L = k.aeif_g_L;
    A.e_E_L = k.aeif_E_L;
    A.e_V_T = k.aeif_V_T;
    A.e_d_T = k.aeif_d_T;
    A.e_d_T_inv = 1.0 / k.aeif_d_T;
    A.e_tau_w_inv = 1.0 / k.aeif_tau_w;
    A.e_C_inv = 1.0 / k.aeif_C;
    A.e_a = k.aeif_a;
    A.e_b = k.aeif_b;
    A.e_V_spike = k.aeif_V_spike;
    return A;
}

template <int BLOCK, int H, int MODEL>
void launch_steps64_m(Ctx& c, const ActArgs& A, uint32_t nsteps, uint8_t* fired_before_last) {
    if (c.multi()) {
        launch_pdl(&k_activity_steps<BLOCK, H, MODEL, true>, c.num_net_blocks, BLOCK, c.stream, A, (const ActDesc*)c.act_desc.p, nsteps,
                   fired_before_last);
    } else {
        launch_pdl(&k_activity_steps<BLOCK, H, MODEL, false>, blocks_for(c.n, BLOCK), BLOCK, c.stream, A, (const ActDesc*)c.act_desc.p, nsteps,
                   fired_before_last);
    }
}

template <int H>
void launch_steps64(Ctx& c, const ActArgs& A, uint32_t nsteps, uint8_t* fired_before_last) {
    switch (c.cfg.neuron_model) {
        case RL_MODEL_POISSON:
            launch_steps64_m<128, H, RL_MODEL_POISSON>(c, A, nsteps, fired_before_last);
            break;
        case RL_MODEL_FITZHUGH_NAGUMO:
            launch_steps64_m<128, H, RL_MODEL_FITZHUGH_NAGUMO>(c, A, nsteps, fired_before_last);
            break;
        case RL_MODEL_AEIF:
            launch_steps64_m<128, H, RL_MODEL_AEIF>(c, A, nsteps, fired_before_last);
            break;
        default:
            launch_steps64_m<128, H, RL_MODEL_IZHIKEVICH>(c, A, nsteps, fired_before_last);
            break;
    }
}

}  // namespace

void launch_activity_fp64(Ctx& c, uint32_t kstep, const uint8_t* fired_prev, uint8_t* fired_cur, const ActVariant& v) {
    const ActArgs A = act64_args(c, kstep, fired_prev, fired_cur);
    if (c.cfg.h_model == 10 && c.cfg.h_calcium == 10) {
        launch_act64<10>(c, v, A, kstep);
    } else {
        launch_act64<0>(c, v, A, kstep);
    }
}

// Calcium and growth of m steps of one launch per step (history rows row0 on).
void launch_calcium_growth64(Ctx& c, uint32_t row0, uint32_t m, cudaStream_t st) {
    const ActArgs A = act64_args(c, 0, nullptr, nullptr);
    const unsigned grid = blocks_for(c.n, 256);
    const bool h10 = c.cfg.h_model == 10 && c.cfg.h_calcium == 10;
    if (c.multi()) {
        (h10 ? k_calcium_growth<10, true> : k_calcium_growth<0, true>)<<<grid, 256, 0, st>>>(A, row0, m);
    } else {
        (h10 ? k_calcium_growth<10, false> : k_calcium_growth<0, false>)<<<grid, 256, 0, st>>>(A, row0, m);
    }
    RL_LAUNCH_CHECK();
}

// The whole block of nsteps steps in one launch (a network without synapses).
void launch_activity_fp64_steps(Ctx& c, uint32_t nsteps) {
    const int p0 = c.nr.cur & 1;
    ActArgs A = act64_args(c, nsteps - 1, c.nr.fired[p0].p, c.nr.fired[(p0 + (int)nsteps) & 1].p);
    uint8_t* before_last = c.nr.fired[(p0 + (int)nsteps - 1) & 1].p;
    if (c.cfg.h_model == 10 && c.cfg.h_calcium == 10) {
        launch_steps64<10>(c, A, nsteps, before_last);
    } else {
        launch_steps64<0>(c, A, nsteps, before_last);
    }
}

namespace {

__global__ void k_set_desc(ActDesc* D, ActDesc v) {
    *D = v;
}

void launch_step(Ctx& c, uint32_t kstep, const ActVariant& v) {
    const int p = (c.nr.cur + (int)kstep) & 1;
    if (is_fp32(c)) {
        launch_activity_f32(c, kstep, c.nr.fired[p].p, c.nr.fired[p ^ 1].p, v);
    } else {
        launch_activity_fp64(c, kstep, c.nr.fired[p].p, c.nr.fired[p ^ 1].p, v);
    }
}

void launch_step(Ctx& c, uint32_t kstep) {
    launch_step(c, kstep, c.tune.act);
}

// Copies of the state one activity step writes, so that the tuner can run
// steps and put everything back.
struct ActSnapshot {
    std::vector<std::pair<void*, size_t>> bufs;
    std::vector<std::unique_ptr<DBuf<uint8_t>>> copies;
    explicit ActSnapshot(Ctx& c) {
        Neurons& N = c.nr;
        const size_t n = c.n;
        if (is_fp32(c)) {
            bufs = { { N.x32.p, 4 * n }, { N.u32.p, 4 * n }, { N.input32.p, 4 * n }, { N.calcium.p, 8 * n } };
            for (int t = 0; t < 3; ++t) {
                bufs.push_back({ N.delta32[t].p, 4 * n });
            }
        } else {
            bufs = { { N.x.p, 8 * n }, { N.u.p, 8 * n }, { N.input.p, 8 * n }, { N.calcium.p, 8 * n } };
            for (int t = 0; t < 3; ++t) {
                bufs.push_back({ N.delta[t].p, 8 * n });
            }
        }
        bufs.push_back({ N.fired[0].p, n });
        bufs.push_back({ N.fired[1].p, n });
        for (size_t b = 0; b < bufs.size(); ++b) {
            copies.push_back(std::make_unique<DBuf<uint8_t>>());
            copies[b]->alloc(bufs[b].second);
            RL_CUDA_TRY(cudaMemcpyAsync(copies[b]->p, bufs[b].first, bufs[b].second, cudaMemcpyDeviceToDevice, c.stream));
        }
    }
    void restore(Ctx& c) {
        for (size_t b = 0; b < bufs.size(); ++b) {
            RL_CUDA_TRY(cudaMemcpyAsync(bufs[b].first, copies[b]->p, bufs[b].second, cudaMemcpyDeviceToDevice, c.stream));
        }
        clear_syn_in(c);  // the timed steps left sums pushed for a step that will not run
    }
};

// Times every activity variant on four steps from the current state (the
// last three are timed) and keeps the fastest; the state is restored after
// each.
void tune_activity(Ctx& c) {
    ActSnapshot snap(c);
    cudaEvent_t e0, e1;
    RL_CUDA_TRY(cudaEventCreate(&e0));
    RL_CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    ActVariant pick = c.tune.act;
    for (const ActVariant& v : act_variants()) {
        if (!is_fp32(c) && v.vec > 2) {
            c.tune.act_ms.push_back(0.0f);  // the FP64 kernel runs one or two neurons per thread
            continue;
        }
        launch_step(c, 0, v);
        RL_CUDA_TRY(cudaEventRecord(e0, c.stream));
        for (uint32_t k = 1; k <= 3; ++k) {
            launch_step(c, k, v);
        }
        RL_CUDA_TRY(cudaEventRecord(e1, c.stream));
        RL_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.0f;
        RL_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        c.tune.act_ms.push_back(ms);
        if (ms < best) {
            best = ms;
            pick = v;
        }
        snap.restore(c);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    c.tune.act = pick;
}

}  // namespace

const std::vector<ActVariant>& act_variants() {
    static const std::vector<ActVariant> v = [] {
        std::vector<ActVariant> out;
        for (int p : { 0, 1 }) {
            for (int b : { 128, 256, 512 }) {
                for (int v : { 1, 2, 4 }) {
                    out.push_back(ActVariant{ b, p, v });
                }
            }
        }
        return out;
    }();
    return v;
}

unsigned act_grid(Ctx& c, const ActVariant& v, const void* kernel) {
    const uint32_t groups = c.n / (uint32_t)v.vec;
    const uint32_t tail = c.n - groups * (uint32_t)v.vec;
    const unsigned full = blocks_for(groups > tail ? groups : tail, (unsigned)v.block);
    if (!v.persistent) {
        return full;
    }
    int per_sm = 0;
    RL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, v.block, 0));
    int sms = 0;
    RL_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device));
    const unsigned wave = (unsigned)(per_sm > 0 ? per_sm : 1) * (unsigned)sms;
    return full < wave ? full : wave;
}

void ensure_syn_in(Ctx& c) {
    if (is_fp32(c) ? c.syn_in32[0].p != nullptr : c.syn_in64[0].p != nullptr) {
        return;
    }
    for (int p = 0; p < 2; ++p) {
        if (is_fp32(c)) {
            c.syn_in32[p].alloc(c.n);
        } else {
            c.syn_in64[p].alloc(c.n);
        }
    }
    drop_activity_graphs(c);  // captured launches hold the kernel arguments
    clear_syn_in(c);
}

void ensure_spike_hist(Ctx& c) {
    const size_t need = hist_stride(c.n) * kHistSteps;
    if (c.spike_hist.p == nullptr || c.spike_hist.n < need) {
        c.spike_hist.alloc(need);
        drop_activity_graphs(c);  // captured launches hold the kernel arguments
    }
}

void launch_calcium_growth(Ctx& c, uint32_t row0, uint32_t m, cudaStream_t st) {
    if (is_fp32(c)) {
        launch_calcium_growth32(c, row0, m, st);
    } else {
        launch_calcium_growth64(c, row0, m, st);
    }
}

void clear_syn_in(Ctx& c) {
    for (int p = 0; p < 2; ++p) {
        if (c.syn_in64[p].p) {
            RL_CUDA_TRY(cudaMemsetAsync(c.syn_in64[p].p, 0, c.syn_in64[p].n * sizeof(long long), c.stream));
        }
        if (c.syn_in32[p].p) {
            RL_CUDA_TRY(cudaMemsetAsync(c.syn_in32[p].p, 0, c.syn_in32[p].n * sizeof(int32_t), c.stream));
        }
    }
}

void drop_activity_graphs(Ctx& c) {
    for (auto& g : c.act_graph) {
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    }
}

void run_activity_block(Ctx& c, uint32_t first_step, uint32_t nsteps) {
    if (nsteps == 0) {
        return;
    }
    c.act_block_len = nsteps;
    const bool edges = c.graph.num_edges > 0;
    if (edges) {
        ensure_syn_in(c);
    }
    const ActDesc v{ first_step, edges ? 1u : 0u, c.graph.offsets.p, c.graph.src.p, c.graph.weight.p, nsteps, c.graph.out_off.p, c.graph.out_perm.p,
                     c.graph.tgt.p };
    k_set_desc<<<1, 1, 0, c.stream>>>(c.act_desc.p, v);
    RL_LAUNCH_CHECK();
    const bool fused = c.step_fusion && c.graph.num_edges == 0 && nsteps > 1;
    if (!fused) {
        ensure_spike_hist(c);
        if (nsteps > kGrowthChunk && c.growth_stream == nullptr) {
            RL_CUDA_TRY(cudaStreamCreateWithFlags(&c.growth_stream, cudaStreamNonBlocking));
            RL_CUDA_TRY(cudaEventCreateWithFlags(&c.growth_fork, cudaEventDisableTiming));
            RL_CUDA_TRY(cudaEventCreateWithFlags(&c.growth_join, cudaEventDisableTiming));
        }
    }
    // the launch shape is a shape of the per-step kernel: it is timed at the
    // first block that runs one launch per step (with the synapses it will
    // read), not while blocks run as one fused launch
    if (c.tune.act_state == TUNE_REQUESTED && !fused) {
        if (c.tune.force || !recall_act_tuning(c)) {
            tune_activity(c);
            remember_act_tuning(c);
        }
        c.tune.act_state = TUNE_DONE;
        drop_activity_graphs(c);
    }
    const bool graph = !fused && c.use_graphs && c.stream != nullptr && nsteps > 1 && nsteps == c.cfg.plasticity_interval;
    // One launch per step; calcium and growth of each chunk of kGrowthChunk
    // steps from the spike history.  A chunk's calcium and growth go to the
    // growth stream, after the chunk's steps, and run beside the next chunk's
    // steps; the context's stream waits for them at the next chunk's end
    // (the chunk after next reuses their history rows, and each chunk's
    // calcium and growth continue the one before).  The last chunk's run on
    // the context's stream after the growth stream's.
    bool forked = false;
    auto step_and_growth = [&](uint32_t k) {
        launch_step(c, k);
        if ((k + 1) % kGrowthChunk != 0 && k + 1 != nsteps) {
            return;
        }
        const uint32_t row0 = (k - k % kGrowthChunk) % kHistSteps;
        const uint32_t m = k % kGrowthChunk + 1;
        if (forked) {
            RL_CUDA_TRY(cudaEventRecord(c.growth_join, c.growth_stream));
            RL_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.growth_join, 0));
        }
        if (k + 1 == nsteps) {
            launch_calcium_growth(c, row0, m, c.stream);
            forked = false;
        } else {
            RL_CUDA_TRY(cudaEventRecord(c.growth_fork, c.stream));
            RL_CUDA_TRY(cudaStreamWaitEvent(c.growth_stream, c.growth_fork, 0));
            launch_calcium_growth(c, row0, m, c.growth_stream);
            forked = true;
        }
    };
    if (fused) {
        // no synapses: every neuron's steps are independent of the others'
        PhaseScope ps(c, PH_ACTIVITY_KERNEL, nsteps);
        if (is_fp32(c)) {
            launch_activity_f32_steps(c, nsteps);
        } else {
            launch_activity_fp64_steps(c, nsteps);
        }
    } else if (graph) {
        const int p = c.nr.cur & 1;
        if (c.act_graph[p] == nullptr || c.act_graph_len != nsteps) {
            for (auto& g : c.act_graph) {
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
            }
            // capture one interval of activity kernels for this parity
            cudaGraph_t gr = nullptr;
            const bool timer = c.timer.on;
            c.timer.on = false;
            const uint64_t launches = c.launches;
            RL_CUDA_TRY(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
            c.capturing = true;
            try {
                for (uint32_t k = 0; k < nsteps; ++k) {
                    step_and_growth(k);
                }
            } catch (...) {
                c.capturing = false;
                cudaStreamEndCapture(c.stream, &gr);
                if (gr) {
                    cudaGraphDestroy(gr);
                }
                c.timer.on = timer;
                throw;
            }
            c.capturing = false;
            RL_CUDA_TRY(cudaStreamEndCapture(c.stream, &gr));
            c.timer.on = timer;
            c.launches = launches;
            cudaGraphExec_t ex = nullptr;
            const cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
            cudaGraphDestroy(gr);
            RL_CUDA_TRY(e);
            c.act_graph[p] = ex;
            c.act_graph_len = nsteps;
        }
        PhaseScope ps(c, PH_ACTIVITY_KERNEL, nsteps);
        RL_CUDA_TRY(cudaGraphLaunch(c.act_graph[p], c.stream));
        c.launches += nsteps;
    } else {
        for (uint32_t k = 0; k < nsteps; ++k) {
            PhaseScope ps(c, PH_ACTIVITY_KERNEL);
            step_and_growth(k);
        }
    }
    c.nr.cur ^= (int)(nsteps & 1u);
    c.stats.activity_steps += nsteps;
    if (c.copy_stream) {
        issue_snapshots(c);  // the block is queued: snapshot copies now overlap it
    }
}

namespace {

// The three commits of a plasticity update in one cooperative launch
// (SynapseDeletionFinderCPU::delete_synapses order: axons, excitatory,
// inhibitory dendrites).  A type whose commit leaves bound elements to delete
// ends the launch after a grid-wide barrier, so the later types wait for the
// deletions exactly as with one launch per type; the axon pass also sums the
// vacant axons of enabled neurons (counts in cnt[0..2], cnt[3]).  D is the
// delta type of the precision form.
template <typename D>
struct CommitAll {
    uint32_t n;
    const uint8_t* enabled;
    double* grown[3];
    D* delta[3];
    uint32_t* connected[3];
    uint32_t* vacant[3];
    double retract[3];
    uint32_t* to_delete;
    unsigned long long* cnt;
};

// ElementBaseBase::update for one neuron and type (the arithmetic of k_commit
// and k_commit_f32); returns the bound elements to delete.
template <typename D>
__device__ __forceinline__ uint32_t commit_one(const CommitAll<D>& A, int t, uint32_t i) {
    if (!A.enabled[i]) {
        A.to_delete[i] = 0u;
        return 0u;
    }
    const double current_count = A.grown[t][i];
    const double current_delta = (double)A.delta[t][i];
    const uint32_t conn_int = A.connected[t][i];
    const double conn = (double)conn_int;
    const double current_vacant = current_count - conn;
    const double new_vacant = current_vacant + current_delta;
    const double keep = 1.0 - A.retract[t];
    uint32_t del = 0;
    if (new_vacant >= 0.0) {
        const double after = keep * new_vacant;
        A.grown[t][i] = after + conn;
        A.vacant[t][i] = (uint32_t)after;
    } else if (current_count + current_delta <= 0.0) {
        A.grown[t][i] = 0.0;
        A.vacant[t][i] = 0u;
        A.connected[t][i] = 0u;
        del = conn_int;
    } else {
        const double new_count = current_count + current_delta;
        const double new_conn = floor(new_count);
        const double num_vacant = new_count - new_conn;
        A.grown[t][i] = (keep * num_vacant) + new_conn;
        A.vacant[t][i] = 0u;
        A.connected[t][i] = (uint32_t)new_conn;
        del = (uint32_t)(conn - new_conn);
    }
    A.delta[t][i] = (D)0;
    A.to_delete[i] = del;
    return del;
}

__device__ __forceinline__ void block_add(unsigned long long v, unsigned long long* out, unsigned long long* part) {
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        part[threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long w = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0ull;
        for (int o = 16; o > 0; o >>= 1) {
            w += __shfl_down_sync(0xFFFFFFFFu, w, o);
        }
        if (threadIdx.x == 0 && w) {
            atomicAdd(out, w);
        }
    }
    __syncthreads();
}

template <typename D>
__global__ void __launch_bounds__(256) k_commit_all(CommitAll<D> A) {
    __shared__ unsigned long long part[8];
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const uint32_t stride = gridDim.x * blockDim.x;
    for (int t = 0; t < 3; ++t) {
        if (t > 0) {
            grid.sync();
            if (A.cnt[t - 1] != 0ull) {
                return;  // the same decision in every thread: deletions first
            }
        }
        unsigned long long del = 0, vac = 0;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride) {
            del += commit_one<D>(A, t, i);
            if (t == 0 && A.enabled[i]) {
                vac += A.vacant[0][i];
            }
        }
        block_add(del, &A.cnt[t], part);
        if (t == 0) {
            block_add(vac, &A.cnt[3], part);
        }
    }
}

template <typename D>
bool launch_commit_all_t(Ctx& c, D* const* delta) {
    CommitAll<D> A;
    A.n = c.n;
    A.enabled = c.nr.enabled.p;
    for (int t = 0; t < 3; ++t) {
        A.grown[t] = c.nr.grown[t].p;
        A.delta[t] = delta[t];
        A.connected[t] = c.nr.connected[t].p;
        A.vacant[t] = c.nr.vacant[t].p;
        A.retract[t] = c.cfg.retract_ratio[t];
    }
    A.to_delete = c.to_delete.p;
    A.cnt = c.commit_cnt.p;
    int per_sm = 0;
    RL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)&k_commit_all<D>, 256, 0));
    if (per_sm <= 0) {
        return false;
    }
    unsigned blocks = (unsigned)per_sm * (unsigned)c.num_sms;
    const unsigned need = blocks_for(c.n, 256);
    if (need < blocks) {
        blocks = need;
    }
    void* args[] = { &A };
    const cudaError_t e = cudaLaunchCooperativeKernel((const void*)&k_commit_all<D>, dim3(blocks), dim3(256), args, 0, c.stream);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();  // cooperative launch unavailable: the caller takes the per-type launches
        return false;
    }
    if (g_bind.launches) {
        ++*g_bind.launches;
    }
    return true;
}

}  // namespace

bool launch_commit_all(Ctx& c) {
    if (is_fp32(c)) {
        float* d[3] = { c.nr.delta32[0].p, c.nr.delta32[1].p, c.nr.delta32[2].p };
        return launch_commit_all_t<float>(c, d);
    }
    double* d[3] = { c.nr.delta[0].p, c.nr.delta[1].p, c.nr.delta[2].p };
    return launch_commit_all_t<double>(c, d);
}

void launch_commit_guarded(Ctx& c, int type) {
    unsigned long long* cnt = c.commit_cnt.p;
    if (is_fp32(c)) {
        launch_commit_f32(c, type, cnt + type, cnt, type);
        return;
    }
    CommitArgs A;
    A.n = c.n;
    A.enabled = c.nr.enabled.p;
    A.grown = c.nr.grown[type].p;
    A.delta = c.nr.delta[type].p;
    A.connected = c.nr.connected[type].p;
    A.vacant = c.nr.vacant[type].p;
    A.retract = c.cfg.retract_ratio[type];
    A.to_delete = c.to_delete.p;
    A.total = cnt + type;
    A.guard = cnt;
    A.guard_n = type;
    k_commit<<<blocks_for(c.n, 256), 256, 0, c.stream>>>(A);
    RL_LAUNCH_CHECK();
}

uint64_t run_commit(Ctx& c, int type) {
    if (is_fp32(c)) {
        return run_commit_f32(c, type);
    }
    CommitArgs A;
    A.n = c.n;
    A.enabled = c.nr.enabled.p;
    A.grown = c.nr.grown[type].p;
    A.delta = c.nr.delta[type].p;
    A.connected = c.nr.connected[type].p;
    A.vacant = c.nr.vacant[type].p;
    A.retract = c.cfg.retract_ratio[type];
    A.to_delete = c.to_delete.p;
    unsigned long long* d_del = reinterpret_cast<unsigned long long*>(c.counters.p) + 1;
    RL_CUDA_TRY(cudaMemsetAsync(d_del, 0, sizeof(unsigned long long), c.stream));
    A.total = d_del;
    A.guard = nullptr;
    A.guard_n = 0;
    k_commit<<<blocks_for(c.n, 256), 256, 0, c.stream>>>(A);
    RL_LAUNCH_CHECK();
    unsigned long long h = 0;
    RL_CUDA_TRY(cudaMemcpyAsync(&h, d_del, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    RL_CUDA_TRY(cudaStreamSynchronize(c.stream));
    c.stats.bound_to_delete += h;
    return h;
}

}  // namespace rl
