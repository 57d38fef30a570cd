// ORACLE — test infrastructure only.
//
// A CPU restatement of RELeARN's single-rank `barnes-hut` + `izhikevich` hot
// path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// may load it; the product never links it.  Each function cites the
// reference file:line it follows (paths relative to relearn/source unless
// noted).  The reference's random draws are replaced by the injected Philox
// stream of shared_stream.h; everything else follows the reference's
// arithmetic operation by operation (compile with -ffp-contract=off).
//
// Deviation, stated once: the connector shuffle (Connector.cpp:71, a
// Fisher-Yates pass over boost uniform_int draws) is replaced by a sort of the
// requests on a 64-bit Philox key drawn per (step, source, j), ties broken by
// (source, j).  Both yield a uniformly random processing order; the keyed form
// is independent of request-list order and can be evaluated in parallel.
#include "shared_stream.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Parameters of one network; mirrors rl_config of the product header.
typedef struct orc_config {
    uint32_t num_neurons;
    uint32_t plasticity_interval;  // Config::plasticity_update_step = 100
    uint32_t h_model;              // NeuronModelBase.h:241 default_h = 10
    uint32_t h_calcium;            // CalciumCalculatorBase.h:210 default_h = 10
    uint64_t seed;
    double box_min[3];
    double box_max[3];
    double theta;  // BarnesHut acceptance criterion
    double sigma;  // GaussianDistributionKernel sigma
    double mu;     // GaussianDistributionKernel mu
    double iz_a, iz_b, iz_c, iz_d, iz_v_spike, iz_k1, iz_k2, iz_k3;
    double beta, tau_c, target_calcium, initial_calcium;
    double growth_rate[3];    // axon, excitatory dendrite, inhibitory dendrite
    double min_calcium[3];    // eta per element type
    double retract_ratio[3];  // vacant retract ratio per element type
    double conductance;       // synaptic_equally_weighted conductance
    double noise_mean, noise_stddev;
    int32_t use_libm;  // 1: std::exp/std::log instead of the shared exp/log
    int32_t kernel_type;    // 0 Gaussian, 1 gamma, 2 linear, 3 Weibull (KernelType.h)
    double kernel_k;        // gamma / Weibull shape
    double kernel_scale;    // gamma theta / Weibull b
    double linear_cutoff;   // linear cut-off (+inf: constant 1)
    int32_t neuron_model;   // 0 Izhikevich, 1 Poisson, 2 FitzHugh-Nagumo, 3 AEIF
    uint32_t poisson_refractory;
    double poisson_x0, poisson_tau_x;
    double fhn_a, fhn_b, fhn_phi, fhn_init_x, fhn_init_w;
    double aeif_C, aeif_g_L, aeif_E_L, aeif_V_T, aeif_d_T, aeif_tau_w, aeif_a, aeif_b, aeif_V_spike;
} orc_config;

typedef struct orc_request {
    uint32_t target;
    uint32_t source;
    uint32_t j;       // index of the vacant axon element of the source
    uint32_t signal;  // 0 excitatory, 1 inhibitory (dendrite type searched)
} orc_request;

}  // extern "C"

namespace {

using oracle::hypot3;

constexpr int32_t kVirtual = -1;
constexpr int kMaxLevel = 1000;

struct V3 {
    double x, y, z;
};

// One node of the pointer octree (OctreeNode<BarnesHutCell>, OctreeNode.h;
// Cell.h; BaseCell.h).  Children are indices into the node pool.
struct Node {
    int32_t child[8];
    int32_t neuron;  // actual neuron id, or kVirtual
    bool parent;
    int level;
    V3 bmin, bmax;
    V3 npos;  // neuron position set by set_cell_neuron_position
    uint32_t cnt[2];       // vacant excitatory / inhibitory dendrites
    bool has_dpos[2];      // dendrite position present
    V3 dpos[2];            // dendrite position per signal type
};

// Cell::get_octant_for_position (Cell.h:104-137).
inline int octant_of(const Node& n, const V3& p) {
    int idx = 0;
    idx |= (p.x < (n.bmin.x + n.bmax.x) / 2.0) ? 0 : 1;
    idx |= (p.y < (n.bmin.y + n.bmax.y) / 2.0) ? 0 : 2;
    idx |= (p.z < (n.bmin.z + n.bmax.z) / 2.0) ? 0 : 4;
    return idx;
}

// Cell::get_size_for_octant (Cell.h:145-178).  std::midpoint(a, b) equals
// (a + b) / 2 for finite |a|, |b| <= DBL_MAX / 2 (libstdc++ <numeric>).
inline void box_for_octant(const Node& n, int oct, V3& lo, V3& hi) {
    lo = n.bmin;
    hi = n.bmax;
    const V3 mid{ (n.bmin.x + n.bmax.x) / 2.0, (n.bmin.y + n.bmax.y) / 2.0, (n.bmin.z + n.bmax.z) / 2.0 };
    if (oct & 1) {
        lo.x = mid.x;
    } else {
        hi.x = mid.x;
    }
    if (oct & 2) {
        lo.y = mid.y;
    } else {
        hi.y = mid.y;
    }
    if (oct & 4) {
        lo.z = mid.z;
    } else {
        hi.z = mid.z;
    }
}

inline bool in_box(const V3& p, const V3& lo, const V3& hi) {
    return lo.x <= p.x && p.x <= hi.x && lo.y <= p.y && p.y <= hi.y && lo.z <= p.z && p.z <= hi.z;
}

// std::clamp as used by Vec3::clip_to_box (Vec3.hpp:760-768).
inline double clamp_to(double v, double lo, double hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

struct Octree {
    std::vector<Node> pool;
    std::vector<int32_t> leaf_of;  // neuron id -> node index (Octree.h:230-270)
    int error = 0;

    Node make_node() const {
        Node n{};
        for (int i = 0; i < 8; ++i) {
            n.child[i] = -1;
        }
        n.neuron = kVirtual;
        n.parent = false;
        n.level = 0;
        return n;
    }

    // Octree ctor root + construct_global_tree_part on one rank (Octree.h:331-396):
    // the root is a virtual leaf covering the simulation box at level 0.
    void init_root(const V3& lo, const V3& hi) {
        pool.clear();
        Node root = make_node();
        root.bmin = lo;
        root.bmax = hi;
        const V3 centre{ ((hi.x - lo.x) / 1.0) / 2.0 + lo.x, ((hi.y - lo.y) / 1.0) / 2.0 + lo.y, ((hi.z - lo.z) / 1.0) / 2.0 + lo.z };
        root.npos = centre;
        root.has_dpos[0] = root.has_dpos[1] = true;
        root.dpos[0] = root.dpos[1] = centre;
        pool.push_back(root);
    }

    void set_neuron_position(Node& n, const V3& p) {
        n.npos = p;
        n.has_dpos[0] = n.has_dpos[1] = true;
        n.dpos[0] = n.dpos[1] = p;
    }

    // OctreeNode::insert (OctreeNode.h:153-250).
    int insert(const V3& pos, int32_t id) {
        if (!in_box(pos, pool[0].bmin, pool[0].bmax)) {
            return 1;
        }
        int parent = -1;
        for (int cur = 0; cur != -1;) {
            const int oct = octant_of(pool[cur], pos);
            parent = cur;
            cur = pool[cur].child[oct];
        }
        if (!pool[parent].parent) {
            if (pool[parent].neuron == kVirtual && id != pool[parent].neuron) {
                pool[parent].neuron = id;
                set_neuron_position(pool[parent], pos);
                return 0;
            }
            while (true) {
                const V3 ppos = pool[parent].npos;
                const int own = octant_of(pool[parent], ppos);
                V3 lo, hi;
                box_for_octant(pool[parent], own, lo, hi);
                Node nn = make_node();
                nn.bmin = lo;
                nn.bmax = hi;
                set_neuron_position(nn, ppos);
                nn.level = pool[parent].level + 1;
                nn.neuron = pool[parent].neuron;
                if (nn.level > kMaxLevel) {
                    return 2;  // coincident positions: the reference would never terminate
                }
                pool.push_back(nn);
                const int nidx = (int)pool.size() - 1;
                pool[parent].child[own] = nidx;
                pool[parent].parent = true;
                pool[parent].neuron = kVirtual;
                if (octant_of(pool[parent], pos) == own) {
                    parent = nidx;
                } else {
                    break;
                }
            }
        }
        const int oct = octant_of(pool[parent], pos);
        V3 lo, hi;
        box_for_octant(pool[parent], oct, lo, hi);
        Node nn = make_node();
        nn.bmin = lo;
        nn.bmax = hi;
        set_neuron_position(nn, pos);
        nn.neuron = id;
        nn.level = pool[parent].level + 1;
        pool.push_back(nn);
        pool[parent].child[oct] = (int)pool.size() - 1;
        pool[parent].parent = true;
        return 0;
    }

    // Octree::initializes_leaf_nodes (Octree.h:230-270).
    void index_leaves(uint32_t n) {
        leaf_of.assign(n, -1);
        for (int i = 0; i < (int)pool.size(); ++i) {
            if (!pool[i].parent && pool[i].neuron >= 0 && (uint32_t)pool[i].neuron < n) {
                leaf_of[pool[i].neuron] = i;
            }
        }
    }

    // OctreeNodeUpdater::update_node (OctreeNodeHelper.h:43-152), both dendrite types.
    void update_node(Node& node) {
        for (int t = 0; t < 2; ++t) {
            V3 acc{ 0.0, 0.0, 0.0 };
            uint32_t total = 0;
            for (int c = 0; c < 8; ++c) {
                if (node.child[c] < 0) {
                    continue;
                }
                const Node& ch = pool[node.child[c]];
                const uint32_t k = ch.cnt[t];
                total += k;
                if (ch.has_dpos[t]) {
                    const double kd = (double)k;
                    acc.x += ch.dpos[t].x * kd;
                    acc.y += ch.dpos[t].y * kd;
                    acc.z += ch.dpos[t].z * kd;
                }
            }
            node.cnt[t] = total;
            if (total == 0) {
                node.has_dpos[t] = false;
            } else {
                const double td = (double)total;
                V3 p{ acc.x / td, acc.y / td, acc.z / td };
                p.x = clamp_to(p.x, node.bmin.x, node.bmax.x);
                p.y = clamp_to(p.y, node.bmin.y, node.bmax.y);
                p.z = clamp_to(p.z, node.bmin.z, node.bmax.z);
                node.has_dpos[t] = true;
                node.dpos[t] = p;
            }
        }
    }

    // OctreeNodeUpdater::update_tree (OctreeNodeHelper.h:266-355): post-order.
    // Children always have larger pool indices than their parent, so a reverse
    // sweep over the pool visits every child before its parent.
    void update_all() {
        for (int i = (int)pool.size() - 1; i >= 0; --i) {
            if (pool[i].parent) {
                update_node(pool[i]);
            }
        }
    }

    // BFS order: root, then level by level, children in octant order.
    std::vector<int32_t> bfs_order() const {
        std::vector<int32_t> order;
        order.reserve(pool.size());
        order.push_back(0);
        for (size_t h = 0; h < order.size(); ++h) {
            const Node& n = pool[order[h]];
            for (int c = 0; c < 8; ++c) {
                if (n.child[c] >= 0) {
                    order.push_back(n.child[c]);
                }
            }
        }
        return order;
    }
};

struct Elements {
    // ElementBaseBase state (ElementBaseBase.h): grown, delta, connected, vacant.
    std::vector<double> grown, delta;
    std::vector<uint32_t> connected, vacant;
    void resize(uint32_t n) {
        grown.assign(n, 0.0);
        delta.assign(n, 0.0);
        connected.assign(n, 0);
        vacant.assign(n, 0);
    }
};

struct Sim {
    orc_config cfg{};
    uint32_t n = 0;
    std::vector<V3> pos;
    std::vector<uint8_t> signal;  // 0 excitatory, 1 inhibitory
    std::vector<uint8_t> enabled;
    Octree tree;
    // neuron model
    std::vector<double> x, u, input, calcium, target;
    std::vector<uint8_t> fired, fired_prev;
    Elements el[3];  // 0 axon, 1 excitatory dendrite, 2 inhibitory dendrite
    // network graph: in-edges per target, (source -> weight)
    std::vector<std::map<uint32_t, int32_t>> in_edges;
    // last plasticity update
    std::vector<orc_request> last_requests;
    std::vector<uint8_t> last_accepted;
    uint64_t total_created = 0;
    uint64_t total_deleted_requests = 0;
    uint64_t total_deleted = 0;
    uint64_t searches = 0;
    uint64_t nodes_touched = 0;
    uint64_t descents = 0;
    int threads = 1;
    int error = 0;

    double ex(double v) const {
        return cfg.use_libm ? std::exp(v) : oracle::own_exp(v);
    }
    double lg(double v) const {
        return cfg.use_libm ? std::log(v) : oracle::own_log(v);
    }
};

// ------------------------------------------------------------- BH search
struct SearchStats {
    uint64_t touched = 0;
    uint64_t descents = 0;
};

enum class Status { Discard, Expand, Accept };

// BarnesHutBase::test_acceptance_criterion (BarnesHutBase.h:72-114).
inline Status acceptance(const Node& node, const V3& src, int t, double theta, double& dist_out) {
    if (node.cnt[t] == 0) {
        return Status::Discard;
    }
    const V3& tp = node.dpos[t];
    const double d = hypot3(tp.x - src.x, tp.y - src.y, tp.z - src.z);
    dist_out = d;
    if (d == 0.0) {
        return Status::Discard;
    }
    if (!node.parent) {
        return Status::Accept;
    }
    const double lx = node.bmax.x - node.bmin.x;
    const double ly = node.bmax.y - node.bmin.y;
    const double lz = node.bmax.z - node.bmin.z;
    const double length = std::max({ lx, ly, lz });  // BoundingBox::get_maximum_difference
    return length < (theta * d) ? Status::Accept : Status::Expand;
}

// BarnesHutBase::get_nodes_to_consider (BarnesHutBase.h:129-206): LIFO stack,
// children pushed in octant order 0..7, so octants are visited descending.
void nodes_to_consider(const Octree& tr, const V3& src, int root, int t, double theta, std::vector<int>& out, SearchStats& st) {
    out.clear();
    const Node& r = tr.pool[root];
    if (r.cnt[t] == 0) {
        return;
    }
    double d;
    if (!r.parent) {
        ++st.touched;
        if (acceptance(r, src, t, theta, d) != Status::Discard) {
            out.push_back(root);
        }
        return;
    }
    std::vector<int> stack;
    stack.reserve(256);
    for (int c = 0; c < 8; ++c) {
        if (r.child[c] >= 0) {
            stack.push_back(r.child[c]);
        }
    }
    while (!stack.empty()) {
        const int idx = stack.back();
        stack.pop_back();
        const Node& nd = tr.pool[idx];
        ++st.touched;
        const Status s = acceptance(nd, src, t, theta, d);
        if (s == Status::Discard) {
            continue;
        }
        if (s == Status::Accept) {
            out.push_back(idx);
            continue;
        }
        for (int c = 0; c < 8; ++c) {
            if (nd.child[c] >= 0) {
                stack.push_back(nd.child[c]);
            }
        }
    }
}

// ProbabilityPicker::pick_target(values, random_number) (ProbabilityPicker.h:46-87).
long pick_index(const double* p, long size, double r) {
    if (!(0.0 < r)) {
        for (long i = 0; i < size; ++i) {
            if (p[i] > 0.0) {
                return i;
            }
        }
        return -1;
    }
    long counter = 0;
    double sum = 0.0;
    for (; counter < size && sum < r; counter++) {
        sum += p[counter];
    }
    if (!(sum > 0.0)) {
        return -1;
    }
    while (p[counter - 1] <= 0.0) {
        counter--;
    }
    return counter - 1;
}

// KernelBase::get_probability(distance) of the configured kernel:
// GaussianDistributionKernel (Gaussian.h:62-68), GammaDistributionKernel
// (Gamma.h: gamma_divisor_inv * pow(d, k - 1) * exp(d * theta_divisor)),
// LinearDistributionKernel (Linear.h) and WeibullDistributionKernel (Weibull.h:
// b k * pow(d, k - 1) * exp(-b * pow(d, k - 1) * d)); pow(d, y) is exact for
// y = 0 and 1 and exp(y log d) otherwise.
double kernel_probability(const Sim& s, double d, double scale) {
    const orc_config& c = s.cfg;
    auto pw = [&](double y) { return y == 0.0 ? 1.0 : (y == 1.0 ? d : s.ex(y * s.lg(d))); };
    if (c.kernel_type == 1) {
        const double gamma_divisor_inv = 1.0 / (std::tgamma(c.kernel_k) * std::pow(c.kernel_scale, c.kernel_k));
        const double theta_divisor = -1.0 / c.kernel_scale;
        const double f1 = pw(c.kernel_k - 1.0);
        const double f2 = s.ex(d * theta_divisor);
        return gamma_divisor_inv * f1 * f2;
    }
    if (c.kernel_type == 2) {
        if (std::isinf(c.linear_cutoff)) {
            return 1.0;
        }
        if (d > c.linear_cutoff) {
            return 0.0;
        }
        const double factor = d / c.linear_cutoff;
        return 1 - factor;
    }
    if (c.kernel_type == 3) {
        const double f1 = c.kernel_scale * c.kernel_k;
        const double f2 = pw(c.kernel_k - 1.0);
        const double exponent = -c.kernel_scale * f2 * d;
        const double f3 = s.ex(exponent);
        return f1 * f2 * f3;
    }
    const double num = (d - s.cfg.mu) * (d - s.cfg.mu);
    return s.ex(num * scale);
}

// Kernel::pick_target + create_probability_interval (Kernel.h:90-173) with
// the kernel's get_probability and ProbabilityPicker::pick_target(values, key)
// (ProbabilityPicker.h:97-112).
int pick_candidate(const Sim& s, const std::vector<int>& cand, uint32_t source, const V3& src, int t, uint32_t step, uint32_t j, uint32_t depth, std::vector<double>& w) {
    if (cand.empty()) {
        return -1;
    }
    const double scale = -1.0 / (s.cfg.sigma * s.cfg.sigma);
    w.assign(cand.size(), 0.0);
    double sum = 0.0;
    for (size_t i = 0; i < cand.size(); ++i) {
        const Node& nd = s.tree.pool[cand[i]];
        double prob = 0.0;
        if (!(!nd.parent && nd.neuron == (int32_t)source)) {
            const V3& tp = nd.dpos[t];
            const double d = hypot3(tp.x - src.x, tp.y - src.y, tp.z - src.z);
            const double e = kernel_probability(s, d, scale);
            prob = (e * 1.0) * (double)nd.cnt[t];
        }
        w[i] = prob;
        sum += prob;
    }
    if (sum == 0.0) {
        for (size_t i = 0; i < cand.size(); ++i) {
            const Node& nd = s.tree.pool[cand[i]];
            double prob = 0.0;
            if (!(!nd.parent && nd.neuron == (int32_t)source)) {
                const V3& tp = nd.dpos[t];
                prob = (double)nd.cnt[t] / hypot3(tp.x - src.x, tp.y - src.y, tp.z - src.z);
            }
            w[i] = prob;
            sum += prob;
        }
    }
    if (sum == 0.0) {
        return -1;
    }
    double total = 0.0;
    for (double v : w) {
        total += v;
    }
    const double next = std::nextafter(total, total + 1e-5);
    const oracle::Words r = oracle::stream_draw(s.cfg.seed, step, source, j, oracle::S_BH, depth);
    double rnd = oracle::unit_closed_open(r) * next;
    if (rnd >= next) {
        rnd = total;
    }
    const long idx = pick_index(w.data(), (long)w.size(), rnd);
    return idx < 0 ? -1 : cand[idx];
}

// BarnesHutBase::find_target_neuron (BarnesHutBase.h:223-255).
int find_target(const Sim& s, uint32_t source, const V3& src, int t, uint32_t step, uint32_t j, std::vector<int>& cand, std::vector<double>& w, SearchStats& st) {
    const Node& root = s.tree.pool[0];
    if (!root.parent) {
        if (root.neuron == (int32_t)source) {
            return -1;
        }
        return root.neuron;
    }
    int sub = 0;
    for (uint32_t depth = 0;; ++depth) {
        nodes_to_consider(s.tree, src, sub, t, s.cfg.theta, cand, st);
        ++st.descents;
        const int sel = pick_candidate(s, cand, source, src, t, step, j, depth, w);
        if (sel < 0) {
            return -1;
        }
        if (!s.tree.pool[sel].parent) {
            return s.tree.pool[sel].neuron;
        }
        sub = sel;
    }
}

// BarnesHut::find_target_neurons (BarnesHut.cpp:36-94) +
// BarnesHutBase::find_target_neurons (BarnesHutBase.h:272-298).  Requests are
// produced per neuron into private slots and concatenated in neuron order, so
// the result does not depend on the thread count.
std::vector<orc_request> find_target_neurons(Sim& s, uint32_t step) {
    const uint32_t n = s.n;
    std::vector<std::vector<orc_request>> per(n);
    uint64_t touched = 0, descents = 0, searches = 0;
#pragma omp parallel num_threads(s.threads) reduction(+ : touched, descents, searches)
    {
        std::vector<int> cand;
        std::vector<double> w;
        SearchStats st;
#pragma omp for schedule(dynamic, 64)
        for (long nid = 0; nid < (long)n; ++nid) {
            if (!s.enabled[nid]) {
                continue;
            }
            const uint32_t v = s.el[0].vacant[nid];
            if (v == 0) {
                continue;
            }
            const int t = s.signal[nid];
            const V3 src = s.pos[nid];
            for (uint32_t j = 0; j < v; ++j) {
                ++searches;
                const int tgt = find_target(s, (uint32_t)nid, src, t, step, j, cand, w, st);
                if (tgt < 0) {
                    break;
                }
                per[nid].push_back(orc_request{ (uint32_t)tgt, (uint32_t)nid, j, (uint32_t)t });
            }
        }
        touched += st.touched;
        descents += st.descents;
    }
    s.nodes_touched += touched;
    s.descents += descents;
    s.searches += searches;
    std::vector<orc_request> out;
    for (auto& v : per) {
        out.insert(out.end(), v.begin(), v.end());
    }
    return out;
}

// ForwardConnector::process_requests (Connector.cpp:33-117) with the keyed
// shuffle stated at the top of this file: the target side (dendrites and the
// synapse list) of every accepted request.
uint64_t process_requests(Sim& s, uint32_t step, const std::vector<orc_request>& req, std::vector<uint8_t>& accepted) {
    const size_t m = req.size();
    std::vector<std::pair<uint64_t, size_t>> order(m);
    for (size_t i = 0; i < m; ++i) {
        const oracle::Words r = oracle::stream_draw(s.cfg.seed, step, req[i].source, req[i].j, oracle::S_CONNECT, 0);
        order[i] = { oracle::take64(r), i };
    }
    std::sort(order.begin(), order.end(), [&](const auto& a, const auto& b) {
        if (a.first != b.first) {
            return a.first < b.first;
        }
        const orc_request& ra = req[a.second];
        const orc_request& rb = req[b.second];
        if (ra.source != rb.source) {
            return ra.source < rb.source;
        }
        return ra.j < rb.j;
    });
    accepted.assign(m, 0);
    uint64_t created = 0;
    for (const auto& [key, i] : order) {
        const orc_request& r = req[i];
        if (r.target == r.source) {
            continue;
        }
        Elements& den = s.el[1 + r.signal];
        if (den.vacant[r.target] == 0) {
            continue;
        }
        den.connected[r.target] += 1;  // ElementBaseBase::connect_elements (ElementBaseBase.h:274-283)
        den.vacant[r.target] -= 1;
        accepted[i] = 1;
        ++created;
        const int32_t weight = r.signal == 1 ? -1 : 1;
        auto& edges = s.in_edges[r.target];
        auto it = edges.find(r.source);
        if (it == edges.end()) {
            edges.emplace(r.source, weight);
        } else {
            it->second += weight;
            if (it->second == 0) {
                edges.erase(it);
            }
        }
    }
    return created;
}

// ForwardConnector::process_responses (Connector.cpp:119-197): the axon side of
// every accepted request.  Returns false when a source has no vacant axon left
// (the reference throws).
bool process_responses(Sim& s, const std::vector<orc_request>& req, const std::vector<uint8_t>& accepted) {
    for (size_t i = 0; i < req.size(); ++i) {
        if (accepted[i]) {
            if (s.el[0].vacant[req[i].source] == 0) {
                return false;
            }
            s.el[0].connected[req[i].source] += 1;
            s.el[0].vacant[req[i].source] -= 1;
        }
    }
    return true;
}

// Both halves on one rank.
uint64_t connect(Sim& s, uint32_t step, const std::vector<orc_request>& req, std::vector<uint8_t>& accepted) {
    const uint64_t created = process_requests(s, step, req, accepted);
    process_responses(s, req, accepted);
    return created;
}

// ElementBaseBase::update (ElementBaseBase.h:420-481); returns the number of
// bound elements to delete.
uint32_t commit_element(Elements& e, uint32_t i, double retract) {
    const double current_count = e.grown[i];
    const double current_delta = e.delta[i];
    const uint32_t conn_int = e.connected[i];
    const double conn = (double)conn_int;
    const double current_vacant = current_count - conn;
    const double new_vacant = current_vacant + current_delta;
    if (new_vacant >= 0.0) {
        const double after = (1 - retract) * new_vacant;
        e.grown[i] = after + conn;
        e.delta[i] = 0.0;
        e.vacant[i] = (uint32_t)after;
        return 0;
    }
    if (current_count + current_delta <= 0.0) {
        e.grown[i] = 0.0;
        e.delta[i] = 0.0;
        e.vacant[i] = 0;
        e.connected[i] = 0;
        return conn_int;
    }
    const double new_count = current_count + current_delta;
    const double new_conn = std::floor(new_count);
    const double num_vacant = new_count - new_conn;
    e.grown[i] = ((1 - retract) * num_vacant) + new_conn;
    e.delta[i] = 0.0;
    e.vacant[i] = 0;
    e.connected[i] = (uint32_t)new_conn;
    return (uint32_t)(conn - new_conn);
}

// RandomHolder::get_random_uniform_indices (util/Random.h:99-115): `count`
// distinct uniform indices below `total`, redrawing duplicates; the draws come
// from the injected stream keyed on (step, neuron, pass, k, attempt).
std::vector<uint32_t> draw_indices(uint64_t seed, uint32_t step, uint32_t neuron, uint32_t pass, uint32_t count, uint32_t total) {
    std::vector<uint32_t> chosen;
    chosen.reserve(count);
    for (uint32_t k = 0; k < count; ++k) {
        for (uint32_t attempt = 0;; ++attempt) {
            const oracle::Words r = oracle::stream_draw(seed, step, neuron, (pass << 24) | k, oracle::S_DELETE, attempt);
            const uint32_t idx = (uint32_t)(((unsigned __int128)oracle::take64(r) * total) >> 64);
            if (std::find(chosen.begin(), chosen.end(), idx) == chosen.end()) {
                chosen.push_back(idx);
                break;
            }
        }
    }
    return chosen;
}

void add_weight(Sim& s, uint32_t target, uint32_t source, int32_t w) {
    auto& edges = s.in_edges[target];
    auto it = edges.find(source);
    if (it == edges.end()) {
        edges.emplace(source, w);
    } else {
        it->second += w;
        if (it->second == 0) {
            edges.erase(it);
        }
    }
}

// SynapseDeletionFinderCPU::find_synapses_to_delete + commit_deletions
// (neurons/helper/SynapseDeletionFinderCPU.cpp:93-237) with the random
// finder (SynapseDeletionFinder.cpp:52-68, register_synapses
// SynapseDeletionFinderBase.cpp:52-110) for one element type.  The synapse
// list of a neuron holds each partner |weight| times; here it is ordered by
// partner id (the reference's order is the insertion order of its edge
// vectors, which only relabels the uniform choice).
uint64_t delete_synapses(Sim& s, uint32_t step, int pass, const std::vector<uint32_t>& to_delete) {
    const uint32_t n = s.n;
    std::vector<std::vector<std::pair<uint32_t, int32_t>>> out_edges;
    if (pass == 0) {
        out_edges.assign(n, {});
        for (uint32_t t = 0; t < n; ++t) {
            for (const auto& [src, w] : s.in_edges[t]) {
                out_edges[src].emplace_back(t, w);
            }
        }
    }
    std::vector<std::pair<uint32_t, uint32_t>> requests;  // (initiator, partner)
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t d = to_delete[i];
        if (d == 0 || !s.enabled[i]) {
            continue;
        }
        std::vector<uint32_t> partners;
        if (pass == 0) {
            for (const auto& [tg, w] : out_edges[i]) {
                for (int32_t k = 0; k < std::abs(w); ++k) {
                    partners.push_back(tg);
                }
            }
        } else {
            const bool exc = pass == 1;
            for (const auto& [src, w] : s.in_edges[i]) {
                if ((exc && w < 0) || (!exc && w > 0)) {
                    continue;
                }
                for (int32_t k = 0; k < std::abs(w); ++k) {
                    partners.push_back(src);
                }
            }
        }
        if (d > partners.size()) {
            s.error = 3;  // the reference throws: more deletions than synapses
            continue;
        }
        for (uint32_t idx : draw_indices(s.cfg.seed, step, i, (uint32_t)pass, d, (uint32_t)partners.size())) {
            requests.emplace_back(i, partners[idx]);
        }
    }
    for (const auto& [i, p] : requests) {
        const int signal = pass == 0 ? s.signal[i] : pass - 1;
        const int32_t weight = signal == 0 ? -1 : 1;
        if (pass == 0) {
            add_weight(s, p, i, weight);
            Elements& den = s.el[1 + signal];  // ElementBaseBase::disconnect_elements (ElementBaseBase.h:311-319)
            den.connected[p] -= 1;
            den.vacant[p] += 1;
        } else {
            add_weight(s, i, p, weight);
            s.el[0].connected[p] -= 1;
            s.el[0].vacant[p] += 1;
        }
    }
    return requests.size();
}

// One neuron's update_activity for the configured model, on x and the second
// state variable u (Izhikevich u, FitzHugh-Nagumo / AEIF w, Poisson refractory
// steps left); returns the fired flag.
uint8_t model_step(const Sim& s, double& xv, double& uv, double input, uint32_t step, uint32_t neuron) {
    const orc_config& c = s.cfg;
    const double scale_m = 1.0 / (double)c.h_model;
    const double ab = c.iz_a * c.iz_b;
    uint8_t spiked = 0;
    if (c.neuron_model == 1) {
        // PoissonModelCPU::update_activity (models/poisson/PoissonModelCPU.cpp):
        // u counts the refractory steps left; the threshold is
        // RandomHolder::get_random_uniform_double(PoissonModel, 0, 1) from the shared stream
        const double tau_x_inverse = 1.0 / c.poisson_tau_x;
        for (uint32_t it = 0; it < c.h_model; ++it) {
            xv += ((c.poisson_x0 - xv) * tau_x_inverse + input) * scale_m;
        }
        if (uv == 0.0) {
            const double threshold = oracle::unit_closed_open(oracle::stream_draw(c.seed, step, neuron, 0, oracle::S_POISSON, 0));
            if (xv >= threshold) {
                spiked = 1;
                uv = (double)c.poisson_refractory;
            }
        } else {
            uv -= 1.0;
        }
    } else if (c.neuron_model == 2) {
        // FitzHughNagumoModelCPU::update_activity (models/fitzhughnagumo/FitzHughNagumoModelCPU.cpp)
        const double third = 1.0 / 3.0;
        for (uint32_t it = 0; it < c.h_model; ++it) {
            const double x_increase = xv - (xv * xv * xv * third) - uv + input;
            const double w_increase = c.fhn_phi * (xv + c.fhn_a - c.fhn_b * uv);
            xv += x_increase * scale_m;
            uv += w_increase * scale_m;
        }
        spiked = (uv > xv - xv * xv * xv * third && xv > 1.0) ? 1 : 0;
    } else if (c.neuron_model == 3) {
        // AEIFModelCPU::update_activity (models/aeif/AEIFModelCPU.cpp)
        const double d_T_inverse = 1.0 / c.aeif_d_T;
        const double tau_w_inverse = 1.0 / c.aeif_tau_w;
        const double C_inverse = 1.0 / c.aeif_C;
        for (uint32_t it = 0; it < c.h_model; ++it) {
            const double linear_part = -c.aeif_g_L * (xv - c.aeif_E_L);
            const double exp_part = c.aeif_g_L * c.aeif_d_T * s.ex((xv - c.aeif_V_T) * d_T_inverse);
            const double x_increase = (linear_part + exp_part - uv + input) * C_inverse;
            const double w_increase = (c.aeif_a * (xv - c.aeif_E_L) - uv) * tau_w_inverse;
            xv += x_increase * scale_m;
            uv += w_increase * scale_m;
            if (xv >= c.aeif_V_spike) {
                xv = c.aeif_E_L;
                uv += c.aeif_b;
                spiked = 1;
                break;
            }
        }
    } else {
        // IzhikevichModelCPU::update_activity (IzhikevichModelCPU.cpp:75-125)
        for (uint32_t it = 0; it < c.h_model; ++it) {
            const double x_inc = (c.iz_k1 * xv * xv) + (c.iz_k2 * xv) + c.iz_k3 - uv + input;
            const double u_inc = (ab * xv) - (c.iz_a * uv);
            xv += x_inc * scale_m;
            uv += u_inc * scale_m;
            if (xv >= c.iz_v_spike) {
                xv = c.iz_c;
                uv += c.iz_d;
                spiked = 1;
                break;
            }
        }
    }
    return spiked;
}

// One activity step, in the order of Simulation::simulate
// (sim/Simulation.cpp:443-453): input, the neuron model, calcium, growth deltas.
void activity_step(Sim& s, uint32_t step) {
    const orc_config& c = s.cfg;
    const uint32_t n = s.n;
    s.fired_prev = s.fired;
    const double scale_c = 1.0 / (double)c.h_calcium;
    const double tau_inv = -1.0 / c.tau_c;
    const double factor_inv = 1.0 / 1.6651092223153955127063292897904020952611777045288814583336582344;
#pragma omp parallel for num_threads(s.threads) schedule(static)
    for (long i = 0; i < (long)n; ++i) {
        if (!s.enabled[i]) {
            s.input[i] = 0.0;
            for (int t = 0; t < 3; ++t) {
                s.el[t].delta[i] += 0.0;
            }
            continue;
        }
        // CombinedActivityInputCPU::update_input_range (CombinedActivityInputCPU.h):
        // input = 0; input += synaptic; input += normal.
        // SynapticEquallyWeightedActivityInputCPU::update_local_input (…CPU.cpp:21-48)
        double inp = 0.0;
        for (const auto& [src, wgt] : s.in_edges[i]) {
            if (s.fired_prev[src]) {
                inp += (double)wgt;
            }
        }
        double input = 0.0;
        input += inp * c.conductance;
        // NormalActivityInputCPU::update_input_range (NormalActivityInputCPU.cpp:21-39)
        const double z = oracle::as241(oracle::noise_unit_open(c.seed, step, (uint32_t)i), [&](double v) { return s.lg(v); });
        input += c.noise_mean + c.noise_stddev * z;
        s.input[i] = input;
        double xv = s.x[i];
        double uv = s.u[i];
        const uint8_t spiked = model_step(s, xv, uv, input, step, (uint32_t)i);
        s.x[i] = xv;
        s.u[i] = uv;
        s.fired[i] = spiked;
        // CalciumCalculatorCPU::update_current_calcium (CalciumCalculatorCPU.cpp:40-103)
        double ca = s.calcium[i];
        const double local_beta = c.beta * (double)(spiked ? 1 : 0);
        for (uint32_t it = 0; it < c.h_calcium; ++it) {
            ca += scale_c * (ca * tau_inv + local_beta);
        }
        s.calcium[i] = ca;
        // update_number_elements_openmp (SynapticElementsCPU.cpp:25-49) with
        // gaussian_growth_curve (GrowthCurves.h:30-53)
        for (int t = 0; t < 3; ++t) {
            const double eta = c.min_calcium[t];
            const double eps = std::max(s.target[i], eta);
            double dz;
            if (eta == eps) {
                dz = (ca == eta) ? 0.0 : -1.0;
            } else {
                const double xi = (eta + eps) * 0.5;
                const double zeta = (eta - eps) * factor_inv;
                const double diff = ca - xi;
                const double quot = diff / zeta;
                const double prod = quot * quot;
                dz = (2.0 * s.ex(-prod)) - 1.0;
            }
            const double inc = dz * c.growth_rate[t];
            s.el[t].delta[i] += inc;
        }
    }
}

// Neurons::update_connectivity (neurons/Neurons.cpp:588-608) on one rank:
// commit (SynapseDeletionFinderCPU.cpp:64-85), tree update
// (OctreeAlgorithm.h:100-238), search, connector, edge insertion.
void plasticity_step(Sim& s, uint32_t step) {
    const uint32_t n = s.n;
    // SynapseDeletionFinderCPU::delete_synapses (SynapseDeletionFinderCPU.cpp:27-92):
    // per element type (axon, excitatory, inhibitory dendrite) commit, then delete
    std::vector<uint32_t> to_delete(n);
    for (int t = 0; t < 3; ++t) {
        uint64_t sum = 0;
        for (uint32_t i = 0; i < n; ++i) {
            to_delete[i] = s.enabled[i] ? commit_element(s.el[t], i, s.cfg.retract_ratio[t]) : 0u;
            sum += to_delete[i];
        }
        s.total_deleted_requests += sum;
        if (sum) {
            s.total_deleted += delete_synapses(s, step, t, to_delete);
        }
    }
    // update_leaf_nodes (OctreeAlgorithm.h:154-238)
    for (uint32_t i = 0; i < n; ++i) {
        Node& leaf = s.tree.pool[s.tree.leaf_of[i]];
        if (!s.enabled[i]) {
            leaf.cnt[0] = leaf.cnt[1] = 0;
            continue;
        }
        leaf.cnt[0] = s.el[1].vacant[i];
        leaf.cnt[1] = s.el[2].vacant[i];
    }
    s.tree.update_all();
    s.last_requests = find_target_neurons(s, step);
    s.total_created += connect(s, step, s.last_requests, s.last_accepted);
}

}  // namespace

// =================================================================== C API
extern "C" {

void* orc_create(const orc_config* cfg, const double* pos_xyz, const uint8_t* signal, int threads) {
    auto* s = new Sim();
    s->cfg = *cfg;
    s->n = cfg->num_neurons;
    s->threads = threads > 0 ? threads : 1;
    const uint32_t n = s->n;
    s->pos.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        s->pos[i] = V3{ pos_xyz[3 * i], pos_xyz[3 * i + 1], pos_xyz[3 * i + 2] };
    }
    s->signal.assign(signal, signal + n);
    s->enabled.assign(n, 1);
    // OctreeAlgorithm::init (OctreeAlgorithm.h:58-67): insert in id order.
    s->tree.init_root(V3{ cfg->box_min[0], cfg->box_min[1], cfg->box_min[2] }, V3{ cfg->box_max[0], cfg->box_max[1], cfg->box_max[2] });
    for (uint32_t i = 0; i < n; ++i) {
        const int rc = s->tree.insert(s->pos[i], (int32_t)i);
        if (rc != 0) {
            s->error = rc;
            break;
        }
    }
    s->tree.index_leaves(n);
    // IzhikevichModelBase::init_neurons (IzhikevichModelBase.cpp:59-66)
    // init_neurons of the model (IzhikevichModelBase, FitzHughNagumoModelBase,
    // AEIFModelBase); NeuronModel::init and PoissonModelBase::init: x = 0, no
    // refractory steps
    double x0 = cfg->iz_c, u0 = 0.0;
    if (cfg->neuron_model == 1) {
        x0 = 0.0;
    } else if (cfg->neuron_model == 2) {
        x0 = cfg->fhn_init_x;
        u0 = cfg->fhn_init_w;
    } else if (cfg->neuron_model == 3) {
        x0 = cfg->aeif_E_L;
    }
    s->x.assign(n, x0);
    s->u.assign(n, u0);
    s->input.assign(n, 0.0);
    s->fired.assign(n, 0);
    s->fired_prev.assign(n, 0);
    s->calcium.assign(n, cfg->initial_calcium);
    s->target.assign(n, cfg->target_calcium);
    for (auto& e : s->el) {
        e.resize(n);
    }
    s->in_edges.assign(n, {});
    return s;
}

int orc_error(void* h) {
    return static_cast<Sim*>(h)->error;
}

void orc_destroy(void* h) {
    delete static_cast<Sim*>(h);
}

void orc_set_threads(void* h, int threads) {
    static_cast<Sim*>(h)->threads = threads > 0 ? threads : 1;
}

uint64_t orc_num_nodes(void* h) {
    return static_cast<Sim*>(h)->tree.pool.size();
}

// Canonical dump of the tree in BFS order (root, then level by level, children
// in octant order).  Arrays have num_nodes entries (x3 for vectors).
void orc_dump_tree(void* h, int32_t* level, int32_t* neuron, uint8_t* child_mask, int32_t* first_child, double* bmin, double* bmax,
                   uint32_t* cnt_exc, uint32_t* cnt_inh, double* pos_exc, double* pos_inh) {
    const Sim* s = static_cast<Sim*>(h);
    const auto order = s->tree.bfs_order();
    std::vector<int32_t> bfs_index(s->tree.pool.size(), -1);
    for (size_t i = 0; i < order.size(); ++i) {
        bfs_index[order[i]] = (int32_t)i;
    }
    const double nan = std::nan("");
    for (size_t i = 0; i < order.size(); ++i) {
        const Node& nd = s->tree.pool[order[i]];
        level[i] = nd.level;
        neuron[i] = nd.parent ? -1 : nd.neuron;
        uint8_t mask = 0;
        int32_t first = -1;
        for (int c = 0; c < 8; ++c) {
            if (nd.child[c] >= 0) {
                mask |= (uint8_t)(1u << c);
                if (first < 0) {
                    first = bfs_index[nd.child[c]];
                }
            }
        }
        child_mask[i] = mask;
        first_child[i] = first;
        bmin[3 * i] = nd.bmin.x;
        bmin[3 * i + 1] = nd.bmin.y;
        bmin[3 * i + 2] = nd.bmin.z;
        bmax[3 * i] = nd.bmax.x;
        bmax[3 * i + 1] = nd.bmax.y;
        bmax[3 * i + 2] = nd.bmax.z;
        cnt_exc[i] = nd.cnt[0];
        cnt_inh[i] = nd.cnt[1];
        // an inner node without vacant elements has no position
        // (OctreeNodeHelper.h:89-90); before the first update it still holds
        // the split neuron's position, which is reported as absent too
        const bool he = nd.has_dpos[0] && !(nd.parent && nd.cnt[0] == 0);
        const bool hi = nd.has_dpos[1] && !(nd.parent && nd.cnt[1] == 0);
        const V3 pe = he ? nd.dpos[0] : V3{ nan, nan, nan };
        const V3 pi = hi ? nd.dpos[1] : V3{ nan, nan, nan };
        pos_exc[3 * i] = pe.x;
        pos_exc[3 * i + 1] = pe.y;
        pos_exc[3 * i + 2] = pe.z;
        pos_inh[3 * i] = pi.x;
        pos_inh[3 * i + 1] = pi.y;
        pos_inh[3 * i + 2] = pi.z;
    }
}

// Set the synaptic-element state of every neuron (type 0 axon, 1 exc, 2 inh).
void orc_set_elements(void* h, int type, const double* grown, const double* delta, const uint32_t* connected, const uint32_t* vacant) {
    Sim* s = static_cast<Sim*>(h);
    Elements& e = s->el[type];
    std::copy(grown, grown + s->n, e.grown.begin());
    std::copy(delta, delta + s->n, e.delta.begin());
    std::copy(connected, connected + s->n, e.connected.begin());
    std::copy(vacant, vacant + s->n, e.vacant.begin());
}

void orc_get_elements(void* h, int type, double* grown, double* delta, uint32_t* connected, uint32_t* vacant) {
    const Sim* s = static_cast<Sim*>(h);
    const Elements& e = s->el[type];
    std::copy(e.grown.begin(), e.grown.end(), grown);
    std::copy(e.delta.begin(), e.delta.end(), delta);
    std::copy(e.connected.begin(), e.connected.end(), connected);
    std::copy(e.vacant.begin(), e.vacant.end(), vacant);
}

void orc_set_enabled(void* h, const uint8_t* enabled) {
    Sim* s = static_cast<Sim*>(h);
    std::copy(enabled, enabled + s->n, s->enabled.begin());
}

// prepare_update_connectivity: leaf update + bottom-up reduction with the
// given vacant dendrite counts (OctreeAlgorithm::update_tree).
void orc_update_tree(void* h, const uint32_t* vac_exc, const uint32_t* vac_inh) {
    Sim* s = static_cast<Sim*>(h);
    for (uint32_t i = 0; i < s->n; ++i) {
        Node& leaf = s->tree.pool[s->tree.leaf_of[i]];
        leaf.cnt[0] = s->enabled[i] ? vac_exc[i] : 0;
        leaf.cnt[1] = s->enabled[i] ? vac_inh[i] : 0;
    }
    s->tree.update_all();
}

// Barnes-Hut search for every neuron with vacant axons (from the current
// axon element state).  Returns the number of requests; copies at most
// `capacity` of them, in (source, j) order.
uint64_t orc_find_targets(void* h, uint32_t step, orc_request* out, uint64_t capacity) {
    Sim* s = static_cast<Sim*>(h);
    s->last_requests = find_target_neurons(*s, step);
    const uint64_t m = s->last_requests.size();
    for (uint64_t i = 0; i < m && i < capacity; ++i) {
        out[i] = s->last_requests[i];
    }
    return m;
}

// Connector over the requests of the last orc_find_targets call.
uint64_t orc_connect(void* h, uint32_t step, uint8_t* accepted_out) {
    Sim* s = static_cast<Sim*>(h);
    const uint64_t created = connect(*s, step, s->last_requests, s->last_accepted);
    s->total_created += created;
    if (accepted_out) {
        std::copy(s->last_accepted.begin(), s->last_accepted.end(), accepted_out);
    }
    return created;
}

// Connector over a caller-given request list (ForwardConnector::process_requests
// + process_responses, Connector.cpp:33-197), as the reference's connector
// tests drive it.  accepted_out gets one flag per request.
uint64_t orc_connect_requests(void* h, uint32_t step, const orc_request* req, uint64_t m, uint8_t* accepted_out) {
    Sim* s = static_cast<Sim*>(h);
    std::vector<orc_request> list(req, req + m);
    std::vector<uint8_t> accepted;
    const uint64_t created = connect(*s, step, list, accepted);
    s->total_created += created;
    if (accepted_out) {
        std::copy(accepted.begin(), accepted.end(), accepted_out);
    }
    return created;
}

// The target half of the connector over a caller-given request list (the
// requests that reach the rank owning their targets).
uint64_t orc_process_requests(void* h, uint32_t step, const orc_request* req, uint64_t m, uint8_t* accepted_out) {
    Sim* s = static_cast<Sim*>(h);
    std::vector<orc_request> list(req, req + m);
    std::vector<uint8_t> accepted;
    const uint64_t created = process_requests(*s, step, list, accepted);
    s->total_created += created;
    if (accepted_out) {
        std::copy(accepted.begin(), accepted.end(), accepted_out);
    }
    return created;
}

// The axon half over the responses to this rank's requests; requests flagged
// in `append` (may be null) add their synapse to the synapse list (their
// target lives on another rank).  Returns -1 when a source has no vacant axon.
int orc_process_responses(void* h, const orc_request* req, const uint8_t* accepted, const uint8_t* append, uint64_t m) {
    Sim* s = static_cast<Sim*>(h);
    std::vector<orc_request> list(req, req + m);
    std::vector<uint8_t> acc(accepted, accepted + m);
    if (!process_responses(*s, list, acc)) {
        return -1;
    }
    for (uint64_t i = 0; i < m; ++i) {
        if (acc[i] && append && append[i]) {
            const int32_t weight = list[i].signal == 1 ? -1 : 1;
            auto& edges = s->in_edges[list[i].target];
            auto it = edges.find(list[i].source);
            if (it == edges.end()) {
                edges.emplace(list[i].source, weight);
            } else {
                it->second += weight;
                if (it->second == 0) {
                    edges.erase(it);
                }
            }
        }
    }
    return 0;
}

// Cell::get_octant_for_position (Cell.h:104-137) of one cell box; -1 when
// the position lies outside the box (the reference throws).
int orc_octant_of(const double* bmin, const double* bmax, const double* pos) {
    Node n{};
    n.bmin = V3{ bmin[0], bmin[1], bmin[2] };
    n.bmax = V3{ bmax[0], bmax[1], bmax[2] };
    const V3 p{ pos[0], pos[1], pos[2] };
    if (!in_box(p, n.bmin, n.bmax)) {
        return -1;
    }
    return octant_of(n, p);
}

// Cell::get_size_for_octant (Cell.h:145-178) of one cell box.
void orc_box_for_octant(const double* bmin, const double* bmax, int oct, double* lo, double* hi) {
    Node n{};
    n.bmin = V3{ bmin[0], bmin[1], bmin[2] };
    n.bmax = V3{ bmax[0], bmax[1], bmax[2] };
    V3 a, b;
    box_for_octant(n, oct, a, b);
    lo[0] = a.x;
    lo[1] = a.y;
    lo[2] = a.z;
    hi[0] = b.x;
    hi[1] = b.y;
    hi[2] = b.z;
}

// BarnesHutBase::test_acceptance_criterion (BarnesHutBase.h:72-114) of one
// node: a leaf (parent = 0) or an inner node with the given cell box, vacant
// dendrite count and dendrite position.  Returns 0 discard, 1 expand,
// 2 accept, -1 for theta outside (0, 0.5] (the reference throws).
int orc_acceptance(int parent, const double* bmin, const double* bmax, uint32_t count, const double* dpos, const double* src, double theta) {
    if (!(theta > 0.0) || theta > 0.5) {
        return -1;
    }
    Node n{};
    n.parent = parent != 0;
    n.bmin = V3{ bmin[0], bmin[1], bmin[2] };
    n.bmax = V3{ bmax[0], bmax[1], bmax[2] };
    n.cnt[0] = count;
    n.has_dpos[0] = true;
    n.dpos[0] = V3{ dpos[0], dpos[1], dpos[2] };
    double d = 0.0;
    const Status st = acceptance(n, V3{ src[0], src[1], src[2] }, 0, theta, d);
    return st == Status::Discard ? 0 : (st == Status::Expand ? 1 : 2);
}

// BarnesHutBase::get_nodes_to_consider (BarnesHutBase.h:129-206) from the
// root for a source position and dendrite type (0 exc, 1 inh) on the current
// tree, with the simulation's theta.  Nodes are reported by their index in
// orc_dump_tree's breadth-first order, in the walk's visiting order.
uint64_t orc_nodes_to_consider(void* h, const double* src, int type, int32_t* out, uint64_t capacity) {
    const Sim* s = static_cast<Sim*>(h);
    const auto order = s->tree.bfs_order();
    std::vector<int32_t> bfs_index(s->tree.pool.size(), -1);
    for (size_t i = 0; i < order.size(); ++i) {
        bfs_index[order[i]] = (int32_t)i;
    }
    std::vector<int> cand;
    SearchStats st;
    nodes_to_consider(s->tree, V3{ src[0], src[1], src[2] }, 0, type, s->cfg.theta, cand, st);
    for (size_t i = 0; i < cand.size() && i < capacity; ++i) {
        out[i] = bfs_index[cand[i]];
    }
    return cand.size();
}

// BarnesHutBase::find_target_neuron (BarnesHutBase.h:223-255) for one source
// id at a given position, dendrite type and vacant-axon index j: the target
// neuron, or -1 when the search fails.
int64_t orc_find_target(void* h, uint32_t source, const double* src, int type, uint32_t step, uint32_t j) {
    const Sim* s = static_cast<Sim*>(h);
    std::vector<int> cand;
    std::vector<double> w;
    SearchStats st;
    return find_target(*s, source, V3{ src[0], src[1], src[2] }, type, step, j, cand, w, st);
}

// Run steps first..first+count-1 of Simulation::simulate: every step one
// activity update, every plasticity_interval-th step a plasticity update.
void orc_simulate(void* h, uint32_t first_step, uint32_t count) {
    Sim* s = static_cast<Sim*>(h);
    for (uint32_t st = first_step; st < first_step + count; ++st) {
        activity_step(*s, st);
        if (s->cfg.plasticity_interval > 0 && st % s->cfg.plasticity_interval == 0) {
            plasticity_step(*s, st);
        }
    }
}

void orc_activity_step(void* h, uint32_t step) {
    activity_step(*static_cast<Sim*>(h), step);
}

void orc_plasticity_step(void* h, uint32_t step) {
    plasticity_step(*static_cast<Sim*>(h), step);
}

void orc_get_neurons(void* h, double* x, double* u, double* calcium, uint8_t* fired, double* input) {
    const Sim* s = static_cast<Sim*>(h);
    if (x) std::copy(s->x.begin(), s->x.end(), x);
    if (u) std::copy(s->u.begin(), s->u.end(), u);
    if (calcium) std::copy(s->calcium.begin(), s->calcium.end(), calcium);
    if (fired) std::copy(s->fired.begin(), s->fired.end(), fired);
    if (input) std::copy(s->input.begin(), s->input.end(), input);
}

void orc_set_neurons(void* h, const double* x, const double* u, const double* calcium, const uint8_t* fired) {
    Sim* s = static_cast<Sim*>(h);
    if (x) std::copy(x, x + s->n, s->x.begin());
    if (u) std::copy(u, u + s->n, s->u.begin());
    if (calcium) std::copy(calcium, calcium + s->n, s->calcium.begin());
    if (fired) std::copy(fired, fired + s->n, s->fired.begin());
}

// The kernel probability of distance d (for the agreement test of the shared
// formula): a Gaussian / gamma / linear / Weibull kernel with the shared exp / log.
double orc_kernel_prob(int type, double d, double mu, double sigma, double k, double scale, double cutoff) {
    Sim s{};
    s.cfg.kernel_type = type;
    s.cfg.mu = mu;
    s.cfg.sigma = sigma;
    s.cfg.kernel_k = k;
    s.cfg.kernel_scale = scale;
    s.cfg.linear_cutoff = cutoff;
    s.cfg.use_libm = 0;
    return kernel_probability(s, d, -1.0 / (sigma * sigma));
}

// One model update (h substeps) of a single neuron for the pins of the neuron
// models: *x, *u in and out, returns the fired flag.
int orc_model_step(const orc_config* cfg, double* x, double* u, double input, uint32_t step, uint32_t neuron) {
    Sim s{};
    s.cfg = *cfg;
    return model_step(s, *x, *u, input, step, neuron);
}

// Per-neuron target calcium (CalciumIO's target function, io/CalciumIO.cpp:27-130).
void orc_set_targets(void* h, const double* target) {
    Sim* s = static_cast<Sim*>(h);
    std::copy(target, target + s->n, s->target.begin());
}

// Number of distinct (target, source) pairs with non-zero weight.
uint64_t orc_num_edges(void* h) {
    const Sim* s = static_cast<Sim*>(h);
    uint64_t m = 0;
    for (const auto& e : s->in_edges) {
        m += e.size();
    }
    return m;
}

// Edges sorted by (target, source).
void orc_get_edges(void* h, uint32_t* target, uint32_t* source, int32_t* weight) {
    const Sim* s = static_cast<Sim*>(h);
    uint64_t k = 0;
    for (uint32_t t = 0; t < s->n; ++t) {
        for (const auto& [src, w] : s->in_edges[t]) {
            target[k] = t;
            source[k] = src;
            weight[k] = w;
            ++k;
        }
    }
}

void orc_add_edges(void* h, uint64_t m, const uint32_t* target, const uint32_t* source, const int32_t* weight) {
    Sim* s = static_cast<Sim*>(h);
    for (uint64_t k = 0; k < m; ++k) {
        auto& edges = s->in_edges[target[k]];
        auto it = edges.find(source[k]);
        if (it == edges.end()) {
            edges.emplace(source[k], weight[k]);
        } else {
            it->second += weight[k];
            if (it->second == 0) {
                edges.erase(it);
            }
        }
    }
}

void orc_stats(void* h, uint64_t* out) {
    const Sim* s = static_cast<Sim*>(h);
    out[0] = s->total_created;
    out[1] = s->total_deleted_requests;
    out[2] = s->searches;
    out[3] = s->nodes_touched;
    out[4] = s->descents;
    out[5] = s->total_deleted;
}

// ---- element-level functions for known-answer tests -------------------

// ProbabilityPicker::pick_target(values, random_number)
long orc_pick_index(const double* p, long size, double r) {
    return pick_index(p, size, r);
}

// izhikevich update of one neuron (IzhikevichModelCPU.cpp:97-122)
int orc_izhikevich(double* x, double* u, double input, uint32_t h, double a, double b, double c, double d, double v_spike, double k1, double k2,
                   double k3) {
    const double scale = 1.0 / (double)h;
    const double ab = a * b;
    double xv = *x;
    double uv = *u;
    int spiked = 0;
    for (uint32_t it = 0; it < h; ++it) {
        const double x_inc = (k1 * xv * xv) + (k2 * xv) + k3 - uv + input;
        const double u_inc = (ab * xv) - (a * uv);
        xv += x_inc * scale;
        uv += u_inc * scale;
        if (xv >= v_spike) {
            xv = c;
            uv += d;
            spiked = 1;
            break;
        }
    }
    *x = xv;
    *u = uv;
    return spiked;
}

// gaussian_growth_curve (GrowthCurves.h:30-53)
double orc_growth_curve(double current, double eta, double epsilon, int use_libm) {
    if (eta == epsilon) {
        return current == eta ? 0.0 : -1.0;
    }
    const double factor_inv = 1.0 / 1.6651092223153955127063292897904020952611777045288814583336582344;
    const double xi = (eta + epsilon) * 0.5;
    const double zeta = (eta - epsilon) * factor_inv;
    const double q = (current - xi) / zeta;
    const double e = use_libm ? std::exp(-(q * q)) : oracle::own_exp(-(q * q));
    return (2.0 * e) - 1.0;
}

// calcium update of one neuron (CalciumCalculatorCPU.cpp:61-68)
double orc_calcium(double c, int fired, double beta, double tau, uint32_t h) {
    const double scale = 1.0 / (double)h;
    const double tau_inv = -1.0 / tau;
    const double lb = beta * (double)(fired ? 1 : 0);
    for (uint32_t i = 0; i < h; ++i) {
        c += scale * (c * tau_inv + lb);
    }
    return c;
}

// ElementBaseBase::update on one element; state in/out.
uint32_t orc_commit_element(double* grown, double* delta, uint32_t* connected, uint32_t* vacant, double retract) {
    Elements e;
    e.resize(1);
    e.grown[0] = *grown;
    e.delta[0] = *delta;
    e.connected[0] = *connected;
    e.vacant[0] = *vacant;
    const uint32_t del = commit_element(e, 0, retract);
    *grown = e.grown[0];
    *delta = e.delta[0];
    *connected = e.connected[0];
    *vacant = e.vacant[0];
    return del;
}

// Shared math entry points (for agreement tests against the product header).
double orc_exp(double x) {
    return oracle::own_exp(x);
}
double orc_log(double x) {
    return oracle::own_log(x);
}
double orc_hypot3(double x, double y, double z) {
    return oracle::hypot3(x, y, z);
}
double orc_normal(uint64_t seed, uint32_t step, uint32_t neuron, double mean, double stddev) {
    return mean + stddev * oracle::as241(oracle::noise_unit_open(seed, step, neuron), [](double v) { return oracle::own_log(v); });
}
double orc_quantile(double p) {
    return oracle::as241(p, [](double v) { return oracle::own_log(v); });
}
void orc_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t* out) {
    const oracle::Words w = oracle::philox(c0, c1, c2, c3, k0, k1);
    std::memcpy(out, w.w, 16);
}

}  // extern "C"
