// Linear octree over the neuron positions, built on the device, and the
// bottom-up aggregation of vacant dendrites.
//
// Reference semantics (relearn/source):
//   * Octree::insert / OctreeNode::insert (algorithm/Internal/octree/Octree.h:201-209,
//     OctreeNode.h:153-250) build the point-region octree: one neuron per leaf,
//     a cell splits until its two neurons fall into different octants.  The
//     result does not depend on insertion order.
//   * Cell::get_octant_for_position (Cell.h:104-137): bit = !(x < (min+max)/2);
//     Cell::get_size_for_octant (Cell.h:145-178): child box via the midpoint.
//   * OctreeNodeUpdater::update_node (OctreeNodeHelper.h:43-152): per dendrite
//     type, count = sum of child counts; position = (sum over children in
//     octant order of child_position * count) / count, clipped to the cell.
//
// Construction here: each neuron computes its octant digits level by level
// with exactly the reference's midpoint comparisons (two 63-bit words, 42
// levels), the keys are radix sorted, and the octree nodes are the distinct
// digit prefixes shared by at least two neurons (inner nodes) plus one leaf per
// neuron at the first level where its prefix is unique.  Nodes are laid out
// breadth-first (level, then Morton order), so the children of a node are
// contiguous and in octant order.
#include "rl_context.cuh"
#include "rl_math.cuh"

#include <cooperative_groups.h>

#include <algorithm>

namespace cg = cooperative_groups;

namespace rl {
namespace {

__device__ __forceinline__ int octant_step(double p, double& lo, double& hi) {
    const double mid = (lo + hi) / 2.0;
    if (p < mid) {
        hi = mid;
        return 0;
    }
    lo = mid;
    return 1;
}

__global__ void k_keys(uint32_t n, const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
                       const NetInfo* __restrict__ nets, const uint16_t* __restrict__ net_of, uint64_t* __restrict__ key0, uint64_t* __restrict__ key1,
                       uint32_t* __restrict__ idx, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const double x = px[i], y = py[i], z = pz[i];
    const NetInfo& N = nets[net_of[i]];
    const double3 bmin = make_double3(N.box_min[0], N.box_min[1], N.box_min[2]);
    const double3 bmax = make_double3(N.box_max[0], N.box_max[1], N.box_max[2]);
    idx[i] = i;
    if (!(bmin.x <= x && x <= bmax.x && bmin.y <= y && y <= bmax.y && bmin.z <= z && z <= bmax.z)) {
        atomicOr(err, (uint32_t)DERR_OUT_OF_BOX);
        key0[i] = 0;
        key1[i] = 0;
        return;
    }
    double lx = bmin.x, hx = bmax.x, ly = bmin.y, hy = bmax.y, lz = bmin.z, hz = bmax.z;
    uint64_t k0 = 0, k1 = 0;
    for (int l = 0; l < kLevelsPerWord; ++l) {
        const int bx = octant_step(x, lx, hx);
        const int by = octant_step(y, ly, hy);
        const int bz = octant_step(z, lz, hz);
        k0 = (k0 << 3) | (uint64_t)(bx | (by << 1) | (bz << 2));
    }
    for (int l = 0; l < kLevelsPerWord; ++l) {
        const int bx = octant_step(x, lx, hx);
        const int by = octant_step(y, ly, hy);
        const int bz = octant_step(z, lz, hz);
        k1 = (k1 << 3) | (uint64_t)(bx | (by << 1) | (bz << 2));
    }
    key0[i] = k0;
    key1[i] = k1;
}

// Neurons whose first words agree are ordered by the second word (runs are
// tiny: the cell of a 21-level prefix is 2^-21 of the box).
__global__ void k_fix_runs(uint32_t n, uint64_t* __restrict__ k0s, uint32_t* __restrict__ idx, const uint64_t* __restrict__ key1,
                           const uint16_t* __restrict__ net_of, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + 1 >= n) {
        return;
    }
    auto same = [&](uint32_t a, uint32_t b) { return k0s[a] == k0s[b] && net_of[idx[a]] == net_of[idx[b]]; };
    if (!same(i, i + 1) || (i > 0 && same(i - 1, i))) {
        return;
    }
    uint32_t end = i + 1;
    while (end + 1 < n && same(end + 1, i)) {
        ++end;
    }
    for (uint32_t a = i + 1; a <= end; ++a) {
        const uint32_t v = idx[a];
        const uint64_t kv = key1[v];
        uint32_t b = a;
        while (b > i && key1[idx[b - 1]] > kv) {
            idx[b] = idx[b - 1];
            --b;
        }
        idx[b] = v;
    }
    for (uint32_t a = i; a < end; ++a) {
        if (key1[idx[a]] == key1[idx[a + 1]]) {
            atomicOr(err, (uint32_t)DERR_DUPLICATE);
        }
    }
}

__device__ __forceinline__ int common_levels(uint64_t a0, uint64_t a1, uint64_t b0, uint64_t b1) {
    const uint64_t x = a0 ^ b0;
    if (x) {
        return (__clzll((long long)x) - 1) / 3;
    }
    const uint64_t y = a1 ^ b1;
    if (y) {
        return kLevelsPerWord + (__clzll((long long)y) - 1) / 3;
    }
    return kMaxLevels;  // identical keys (flagged as duplicate elsewhere)
}

// lcp[i] = common levels of sorted neighbours i and i+1, for i < n-1.
__global__ void k_lcp(uint32_t n, const uint64_t* __restrict__ k0s, const uint32_t* __restrict__ idx, const uint64_t* __restrict__ key1,
                      const uint16_t* __restrict__ net_of, int32_t* __restrict__ lcp, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i + 1 >= n) {
        return;
    }
    if (net_of[idx[i]] != net_of[idx[i + 1]]) {
        lcp[i] = -1;  // different networks share no node
        return;
    }
    const int c = common_levels(k0s[i], key1[idx[i]], k0s[i + 1], key1[idx[i + 1]]);
    if (c >= kMaxLevels) {
        atomicOr(err, (uint32_t)DERR_DUPLICATE);
    }
    lcp[i] = c;
}

__device__ __forceinline__ int lcp_at(const int32_t* lcp, int64_t i, uint32_t n) {
    return (i < 0 || i >= (int64_t)n - 1) ? -1 : lcp[i];
}

// Nodes starting at sorted position i occupy levels [s_i, e_i]:
// s_i = lcp(i-1) + 1, e_i = max(lcp(i-1), lcp(i)) + 1; the last is the leaf.
__global__ void k_node_counts(uint32_t n, const int32_t* __restrict__ lcp, uint32_t* __restrict__ cnt, uint32_t* __restrict__ maxlev) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const int a = lcp_at(lcp, (int64_t)i - 1, n);
    const int b = lcp_at(lcp, i, n);
    const int s = a + 1;
    const int e = (a > b ? a : b) + 1;
    cnt[i] = (uint32_t)(e - s + 1);
    atomicMax(maxlev, (uint32_t)e);
}

__global__ void k_node_keys(uint32_t n, const int32_t* __restrict__ lcp, const uint32_t* __restrict__ base, uint32_t* __restrict__ skey,
                            uint32_t* __restrict__ sval) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const int a = lcp_at(lcp, (int64_t)i - 1, n);
    const int b = lcp_at(lcp, i, n);
    const int s = a + 1;
    const int e = (a > b ? a : b) + 1;
    uint32_t m = base[i];
    for (int l = s; l <= e; ++l, ++m) {
        skey[m] = (uint32_t)l * n + i;
        sval[m] = m;
    }
}

__global__ void k_invert(uint32_t m, const uint32_t* __restrict__ sval, uint32_t* __restrict__ bfs_of) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < m) {
        bfs_of[sval[b]] = b;
    }
}

__device__ __forceinline__ int digit_at(uint64_t k0, uint64_t k1, int level) {
    // level 1..42
    if (level <= kLevelsPerWord) {
        return (int)((k0 >> (3 * (kLevelsPerWord - level))) & 7u);
    }
    return (int)((k1 >> (3 * (2 * kLevelsPerWord - level))) & 7u);
}

__global__ void k_net_keys(uint32_t n, const uint32_t* __restrict__ idx, const uint16_t* __restrict__ net_of, uint32_t* __restrict__ netk,
                           uint32_t* __restrict__ perm) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        netk[i] = net_of[idx[i]];
        perm[i] = i;
    }
}

__global__ void k_permute_keys(uint32_t n, const uint32_t* __restrict__ perm, const uint64_t* __restrict__ k0s, const uint32_t* __restrict__ idx,
                               uint64_t* __restrict__ k0o, uint32_t* __restrict__ idxo) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        k0o[i] = k0s[perm[i]];
        idxo[i] = idx[perm[i]];
    }
}

struct FillArgs {
    uint32_t n, m;
    const uint32_t* skey;
    const uint32_t* sval;
    const uint32_t* bfs_of;
    const int32_t* lcp;
    const uint64_t* k0s;
    const uint64_t* key1;
    const uint32_t* idx;
    const double *px, *py, *pz;
    const NetInfo* nets;
    const uint16_t* net_of;
    double4* rec0;
    double4* rec1;
    uint2* topo;
    double* maxdim;
    double *bx0, *by0, *bz0, *bx1, *by1, *bz1;
    uint32_t* first_key;
    uint32_t* leaf_of;
    int32_t* parent;
    uint32_t* level_count;
};

__global__ void k_fill(FillArgs A) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= A.m) {
        return;
    }
    const uint32_t key = A.skey[b];
    const uint32_t l = key / A.n;
    const uint32_t i = key - l * A.n;
    const uint32_t mi = A.sval[b];
    const int a = lcp_at(A.lcp, (int64_t)i - 1, A.n);
    const int bb = lcp_at(A.lcp, i, A.n);
    const int s = a + 1;
    const int e = (a > bb ? a : bb) + 1;
    const bool leaf = (int)l == e;
    const uint32_t neuron = A.idx[i];
    const uint64_t k0 = A.k0s[i];
    const uint64_t k1 = A.key1[neuron];
    const NetInfo& N = A.nets[A.net_of[neuron]];
    // cell box: descend l levels along the digits of the first neuron
    double lx = N.box_min[0], hx = N.box_max[0], ly = N.box_min[1], hy = N.box_max[1], lz = N.box_min[2], hz = N.box_max[2];
    for (int lev = 1; lev <= (int)l; ++lev) {
        const int d = digit_at(k0, k1, lev);
        const double mx = (lx + hx) / 2.0, my = (ly + hy) / 2.0, mz = (lz + hz) / 2.0;
        if (d & 1) lx = mx; else hx = mx;
        if (d & 2) ly = my; else hy = my;
        if (d & 4) lz = mz; else hz = mz;
    }
    A.bx0[b] = lx;
    A.by0[b] = ly;
    A.bz0[b] = lz;
    A.bx1[b] = hx;
    A.by1[b] = hy;
    A.bz1[b] = hz;
    const double dx = hx - lx, dy = hy - ly, dz = hz - lz;
    // std::max({x, y, z}) of Vec3::get_maximum
    double md = dx;
    if (md < dy) md = dy;
    if (md < dz) md = dz;
    A.maxdim[b] = md;
    A.first_key[b] = i;
    const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
    if (leaf) {
        const double4 p = make_double4(A.px[neuron], A.py[neuron], A.pz[neuron], 0.0);
        A.rec0[b] = p;
        A.rec1[b] = p;
        A.topo[b] = make_uint2(neuron, (1u << 8) | (l << 16));
        A.leaf_of[neuron] = b;
    } else {
        A.rec0[b] = zero;
        A.rec1[b] = zero;
        A.topo[b] = make_uint2(A.bfs_of[mi + 1], (l << 16));
    }
    if (l == 0) {
        A.parent[b] = -1;
    } else if ((int)l > s) {
        A.parent[b] = (int32_t)A.bfs_of[mi - 1];
    } else {
        A.parent[b] = -2;  // resolved by k_parent_search
    }
    atomicAdd(&A.level_count[l], 1u);
}

// For a node that is the first node of its start position, the parent is the
// last node of the previous level that starts at or before it.
__global__ void k_parent_search(uint32_t m, const uint32_t* __restrict__ level_off, const uint32_t* __restrict__ first_key, const uint2* topo_in,
                                int32_t* __restrict__ parent) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m || parent[b] != -2) {
        return;
    }
    const uint32_t l = topo_level(topo_in[b].y);
    const uint32_t i = first_key[b];
    uint32_t lo = level_off[l - 1], hi = level_off[l];  // search [lo, hi)
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (first_key[mid] <= i) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    parent[b] = (int32_t)lo;
}

__global__ void k_child_mask(uint32_t m, const int32_t* __restrict__ parent, const uint32_t* __restrict__ first_key, const uint64_t* __restrict__ k0s,
                             const uint32_t* __restrict__ idx, const uint64_t* __restrict__ key1, uint2* topo) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m) {
        return;
    }
    const int32_t p = parent[b];
    if (p < 0) {
        return;
    }
    const uint32_t i = first_key[b];
    const uint32_t l = topo_level(topo[b].y);
    const int d = digit_at(k0s[i], key1[idx[i]], (int)l);
    atomicOr(&topo[p].y, 1u << d);
}

// Escape link of every node for walks without a stack.  The reference's walk
// (BarnesHutBase::get_nodes_to_consider, BarnesHutBase.h:129-206) pushes the
// children of an expanded node in octant order 0..7 onto a LIFO stack, so it
// visits them 7..0; children are contiguous in octant order here, so after the
// subtree of node v the walk continues at v - 1 unless v is its parent's first
// child, in which case it continues wherever the parent's subtree is left.
// kNoNode after the last node of a tree (the roots have no parent).  Written
// into the node's meta entry with its topology and FP32 cell length.
__global__ void k_meta(uint32_t m, const int32_t* __restrict__ parent, const uint2* __restrict__ topo, const double* __restrict__ maxdim,
                       uint4* __restrict__ meta, uint32_t* __restrict__ err) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m) {
        return;
    }
    uint32_t skip = kNoNode;
    uint32_t v = b;
    int up = 0;
    for (; up <= kMaxLevels; ++up) {
        const int32_t p = parent[v];
        if (p < 0) {
            break;
        }
        if (v != topo[p].x) {
            skip = v - 1;
            break;
        }
        v = (uint32_t)p;
    }
    if (up > kMaxLevels) {
        atomicOr(err, (uint32_t)DERR_WALK);  // deeper than any octree built here
    }
    const uint2 t = topo[b];
    meta[b] = make_uint4(t.x, t.y, skip, __float_as_uint((float)maxdim[b]));
}

// ------------------------------------------------------------ aggregation
__global__ void k_leaf_counts(uint32_t n, const uint32_t* __restrict__ leaf_of, const uint8_t* __restrict__ enabled, const uint8_t* __restrict__ update,
                              const uint32_t* __restrict__ vac_exc, const uint32_t* __restrict__ vac_inh, double4* rec0, double4* rec1) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const uint32_t leaf = leaf_of[i];
    const bool on = enabled[i] && update[i];
    const uint32_t ce = on ? vac_exc[i] : 0u;
    const uint32_t ci = on ? vac_inh[i] : 0u;
    reinterpret_cast<long long*>(&rec0[leaf])[3] = (long long)ce;
    reinterpret_cast<long long*>(&rec1[leaf])[3] = (long long)ci;
}

__device__ __forceinline__ uint32_t rec_count(const double4& r) {
    return (uint32_t)__double_as_longlong(r.w);
}

__device__ __forceinline__ double4 ldcg4(const double4* p) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ void stcg4(double4* p, const double4& v) {
    __stcg(reinterpret_cast<double2*>(p), make_double2(v.x, v.y));
    __stcg(reinterpret_cast<double2*>(p) + 1, make_double2(v.z, v.w));
}

// Centroid = count-weighted sum / total count, clipped to the cell; NaN
// centroid and count 0 for a cell without vacant elements.
__device__ __forceinline__ double4 finish_centroid(double ax, double ay, double az, uint32_t total, double lx, double ly, double lz, double hx, double hy,
                                                   double hz) {
    if (total == 0) {
        const double nan = __longlong_as_double(0x7FF8000000000000ll);
        return make_double4(nan, nan, nan, 0.0);
    }
    const double td = (double)total;
    double x = ax / td, y = ay / td, z = az / td;
    x = x < lx ? lx : (hx < x ? hx : x);
    y = y < ly ? ly : (hy < y ? hy : y);
    z = z < lz ? lz : (hz < z ? hz : z);
    return make_double4(x, y, z, __longlong_as_double((long long)total));
}

// OctreeNodeUpdater::update_node for one dendrite type.
__device__ __forceinline__ double4 update_type(const double4* rec, const uint2* topo, uint32_t base, uint32_t mask, double lx, double ly, double lz,
                                               double hx, double hy, double hz) {
    double ax = 0.0, ay = 0.0, az = 0.0;
    uint32_t total = 0;
    uint32_t k = 0;
    for (int c = 0; c < 8; ++c) {
        if (!((mask >> c) & 1u)) {
            continue;
        }
        const uint32_t child = base + k++;
        const double4 r = ldcg4(&rec[child]);
        const uint32_t cnt = rec_count(r);
        total += cnt;
        const bool has = topo_leaf(__ldg(&topo[child].y)) || cnt > 0;
        if (has) {
            const double kd = (double)cnt;
            ax = ax + r.x * kd;
            ay = ay + r.y * kd;
            az = az + r.z * kd;
        }
    }
    return finish_centroid(ax, ay, az, total, lx, ly, lz, hx, hy, hz);
}

struct ReduceArgs {
    uint32_t n;
    const uint32_t* leaf_of;
    const int32_t* parent;
    const uint2* topo;
    const double *bx0, *by0, *bz0, *bx1, *by1, *bz1;
    double4* rec0;
    double4* rec1;
    uint32_t* arrive;
    // incremental update: nodes to recompute (a per-level list of the marked
    // nodes: level l's at work[level_lo[l] ...], level_dirty[l] of them), and
    // the leaf counts of the last update
    uint32_t* dirty;
    uint32_t* level_dirty;
    uint32_t* work;
    const uint32_t* level_lo;
    uint2* last;
    // leaf counts: vacant dendrites of the neurons that take part
    const uint8_t* enabled;
    const uint8_t* update;
    const uint32_t* vac_exc;
    const uint32_t* vac_inh;
    int force;  // every leaf counts as changed
    // FP32 form: fixed-point records kept in step (null otherwise)
    uint4* recq0;
    uint4* recq1;
    const uint32_t* first_key;
    const uint32_t* morton;
    const uint16_t* net_of;
    const NetInfo* nets;
    // captured update: the leaf pass switches the level reductions on
    // (conditional graph node) and each level launch counts itself
    int has_cond;
    cudaGraphConditionalHandle cond;
    unsigned long long* level_runs;
};

// Marks node p for recomputation: the first mark of the update appends it to
// its level's list (a node is on it at most once).  The lanes of a warp that
// append to the same level take their slots with one atomic between them: in
// an update that changes most leaves, every node of a level is appended, and
// one counter per level would otherwise take an atomic per node.
__device__ __forceinline__ void mark_node(const ReduceArgs& A, int32_t p) {
    if (atomicExch(&A.dirty[p], 1u) == 0u) {
        const uint32_t l = topo_level(A.topo[p].y);
        const cg::coalesced_group appending = cg::coalesced_threads();
        const cg::coalesced_group same_level = cg::labeled_partition(appending, l);
        uint32_t base = 0;
        if (same_level.thread_rank() == 0) {
            base = atomicAdd(&A.level_dirty[l], same_level.size());
        }
        base = same_level.shfl(base, 0);
        A.work[A.level_lo[l] + base + same_level.thread_rank()] = (uint32_t)p;
    }
}

// Leaf pass of the incremental update (OctreeAlgorithm::update_leaf_nodes):
// one thread per neuron; a leaf whose vacant counts differ from the last
// update gets the new counts and marks its parent for recomputation.
__global__ void k_leaf_update(ReduceArgs A) {
    pdl_wait_then_release();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) {
        return;
    }
    const bool on = A.enabled[i] && A.update[i];
    const uint2 now = make_uint2(on ? A.vac_exc[i] : 0u, on ? A.vac_inh[i] : 0u);
    const uint2 was = A.last[i];
    if (!A.force && now.x == was.x && now.y == was.y) {
        return;
    }
    A.last[i] = now;
    const uint32_t leaf = A.leaf_of[i];
    reinterpret_cast<long long*>(&A.rec0[leaf])[3] = (long long)now.x;
    reinterpret_cast<long long*>(&A.rec1[leaf])[3] = (long long)now.y;
    if (A.recq0) {
        A.recq0[leaf].w = now.x;
        A.recq1[leaf].w = now.y;
    }
    const int32_t p = A.parent[leaf];
    if (p >= 0) {
        mark_node(A, p);
        if (A.has_cond) {
            cudaGraphSetConditional(A.cond, 1u);  // some level has work: run the reductions
        }
    }
}

// One level of the bottom-up reduction: one thread per marked node of the
// level (the level's list, filled by the launch one level deeper or by the
// leaf pass); a marked node is recomputed from its children (leaves refreshed
// by the leaf pass, inner children by the previous launch, one level deeper),
// read in octant order as the reference sums them
// (OctreeNodeUpdater::update_node), and marks its parent.  Recomputing only
// the nodes above changed leaves gives the same records as recomputing all,
// and a node's record does not depend on the order of the list.  A level with
// no marked node (most levels, most updates) returns at once; the grid strides
// over the list, capped at a few blocks per SM.
__device__ __forceinline__ void reduce_node(const ReduceArgs& A, uint32_t node);

__global__ void k_reduce_level(ReduceArgs A, uint32_t lo, uint32_t hi, uint32_t level) {
    pdl_wait_then_release();
    if (A.level_runs && blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd(A.level_runs, 1ull);
    }
    const uint32_t marked = A.level_dirty[level];  // at most hi - lo: each node is listed once
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < marked; t += gridDim.x * blockDim.x) {
        reduce_node(A, A.work[lo + t]);
    }
}

__device__ __forceinline__ void reduce_node(const ReduceArgs& A, uint32_t node) {
    A.dirty[node] = 0;
    const uint2 t = A.topo[node];
    const uint32_t mask = topo_mask(t.y);
    double ax0 = 0.0, ay0 = 0.0, az0 = 0.0, ax1 = 0.0, ay1 = 0.0, az1 = 0.0;
    uint32_t tot0 = 0, tot1 = 0;
    uint32_t k = 0;
    for (int oct = 0; oct < 8; ++oct) {
        if (!((mask >> oct) & 1u)) {
            continue;
        }
        const uint32_t child = t.x + k++;
        const bool leaf = topo_leaf(A.topo[child].y);
        const double4 r0 = ldcg4(&A.rec0[child]);
        const double4 r1 = ldcg4(&A.rec1[child]);
        const uint32_t c0 = rec_count(r0), c1 = rec_count(r1);
        tot0 += c0;
        tot1 += c1;
        if (leaf || c0 > 0) {
            const double kd = (double)c0;
            ax0 = ax0 + r0.x * kd;
            ay0 = ay0 + r0.y * kd;
            az0 = az0 + r0.z * kd;
        }
        if (leaf || c1 > 0) {
            const double kd = (double)c1;
            ax1 = ax1 + r1.x * kd;
            ay1 = ay1 + r1.y * kd;
            az1 = az1 + r1.z * kd;
        }
    }
    const double lx = A.bx0[node], ly = A.by0[node], lz = A.bz0[node];
    const double hx = A.bx1[node], hy = A.by1[node], hz = A.bz1[node];
    const double4 n0 = finish_centroid(ax0, ay0, az0, tot0, lx, ly, lz, hx, hy, hz);
    const double4 n1 = finish_centroid(ax1, ay1, az1, tot1, lx, ly, lz, hx, hy, hz);
    stcg4(&A.rec0[node], n0);
    stcg4(&A.rec1[node], n1);
    if (A.recq0) {
        const QFrame& f = A.nets[A.net_of[A.morton[A.first_key[node]]]].frame;
        A.recq0[node] = quantize_record(n0, f);
        A.recq1[node] = quantize_record(n1, f);
    }
    const int32_t p = A.parent[node];
    if (p >= 0) {
        mark_node(A, p);
    }
}

// One thread per leaf walks up; the last child to arrive at a node computes
// it (reading all children in octant order), so every node is computed once
// and in the reference's summation order.  Used by the allocation-free entry
// point, whose only scratch is the arrival counters.
__global__ void k_reduce(ReduceArgs A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n) {
        return;
    }
    int32_t node = A.parent[A.leaf_of[i]];
    while (node >= 0) {
        __threadfence();
        const uint2 t = A.topo[node];
        const uint32_t mask = topo_mask(t.y);
        const uint32_t old = atomicAdd(&A.arrive[node], 1u);
        if (old + 1 != (uint32_t)__popc(mask)) {
            return;
        }
        __threadfence();
        const double lx = A.bx0[node], ly = A.by0[node], lz = A.bz0[node];
        const double hx = A.bx1[node], hy = A.by1[node], hz = A.bz1[node];
        const double4 r0 = update_type(A.rec0, A.topo, t.x, mask, lx, ly, lz, hx, hy, hz);
        const double4 r1 = update_type(A.rec1, A.topo, t.x, mask, lx, ly, lz, hx, hy, hz);
        stcg4(&A.rec0[node], r0);
        stcg4(&A.rec1[node], r1);
        node = A.parent[node];
    }
}

}  // namespace

void build_octree(Ctx& c, const double* h_xyz) {
    const uint32_t n = c.n;
    cudaStream_t st = c.stream;
    Tree& T = c.tree;
    T.drop_graph();
    T.force_full = true;
    T.recq_valid = false;
    // positions to SoA on the host side of the copy
    std::vector<double> hx(n), hy(n), hz(n);
    for (uint32_t i = 0; i < n; ++i) {
        hx[i] = h_xyz[3 * (size_t)i];
        hy[i] = h_xyz[3 * (size_t)i + 1];
        hz[i] = h_xyz[3 * (size_t)i + 2];
    }
    RL_CUDA_TRY(cudaMemcpyAsync(c.nr.px.p, hx.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    RL_CUDA_TRY(cudaMemcpyAsync(c.nr.py.p, hy.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    RL_CUDA_TRY(cudaMemcpyAsync(c.nr.pz.p, hz.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    RL_CUDA_TRY(cudaMemsetAsync(c.err.p, 0, sizeof(uint32_t), st));

    DBuf<uint64_t> key0, key1;
    DBuf<uint32_t> idx;
    key0.alloc(n);
    key1.alloc(n);
    idx.alloc(n);
    k_keys<<<blocks_for(n, 256), 256, 0, st>>>(n, c.nr.px.p, c.nr.py.p, c.nr.pz.p, c.d_nets.p, c.net_of.p, key0.p, key1.p, idx.p, c.err.p);
    RL_LAUNCH_CHECK();
    check_device_error(c, "octree keys");
    // sort on the first word (63 bits), then stably by network; order ties by the second word
    DBuf<uint64_t> k0s;
    k0s.alloc(n);
    RL_CUDA_TRY(cudaMemcpyAsync(k0s.p, key0.p, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    radix_sort_u64(k0s.p, idx.p, n, 63, c.prim, st);
    if (c.multi()) {
        DBuf<uint32_t> netk, perm, idx2;
        DBuf<uint64_t> k02;
        netk.alloc(n);
        perm.alloc(n);
        idx2.alloc(n);
        k02.alloc(n);
        k_net_keys<<<blocks_for(n, 256), 256, 0, st>>>(n, idx.p, c.net_of.p, netk.p, perm.p);
        RL_LAUNCH_CHECK();
        int nb = 1;
        while (nb < 16 && ((uint64_t)1 << nb) < c.nets.size()) {
            ++nb;
        }
        radix_sort_u32(netk.p, perm.p, n, nb, c.prim, st);
        k_permute_keys<<<blocks_for(n, 256), 256, 0, st>>>(n, perm.p, k0s.p, idx.p, k02.p, idx2.p);
        RL_LAUNCH_CHECK();
        RL_CUDA_TRY(cudaMemcpyAsync(k0s.p, k02.p, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
        RL_CUDA_TRY(cudaMemcpyAsync(idx.p, idx2.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        RL_CUDA_TRY(cudaStreamSynchronize(st));
    }
    k_fix_runs<<<blocks_for(n, 256), 256, 0, st>>>(n, k0s.p, idx.p, key1.p, c.net_of.p, c.err.p);
    RL_LAUNCH_CHECK();
    DBuf<int32_t> lcp;
    lcp.alloc(n);
    k_lcp<<<blocks_for(n, 256), 256, 0, st>>>(n, k0s.p, idx.p, key1.p, c.net_of.p, lcp.p, c.err.p);
    RL_LAUNCH_CHECK();
    check_device_error(c, "octree keys");

    DBuf<uint32_t> cnt, base, maxlev;
    cnt.alloc(n);
    base.alloc(n);
    maxlev.alloc(1);
    RL_CUDA_TRY(cudaMemsetAsync(maxlev.p, 0, sizeof(uint32_t), st));
    k_node_counts<<<blocks_for(n, 256), 256, 0, st>>>(n, lcp.p, cnt.p, maxlev.p);
    RL_LAUNCH_CHECK();
    const uint32_t m = exclusive_scan_u32(cnt.p, base.p, n, c.prim, st);
    uint32_t max_level = 0;
    RL_CUDA_TRY(cudaMemcpyAsync(&max_level, maxlev.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    RL_CHECK((uint64_t)(max_level + 1) * n < 0xFFFFFFFFull, RL_ERR_UNSUPPORTED, "octree too deep for the node key");

    DBuf<uint32_t> skey, sval, bfs_of;
    skey.alloc(m);
    sval.alloc(m);
    bfs_of.alloc(m);
    k_node_keys<<<blocks_for(n, 256), 256, 0, st>>>(n, lcp.p, base.p, skey.p, sval.p);
    RL_LAUNCH_CHECK();
    int bits = 1;
    while (bits < 32 && ((uint64_t)1 << bits) <= (uint64_t)(max_level + 1) * n) {
        ++bits;
    }
    radix_sort_u32(skey.p, sval.p, m, bits, c.prim, st);
    k_invert<<<blocks_for(m, 256), 256, 0, st>>>(m, sval.p, bfs_of.p);
    RL_LAUNCH_CHECK();

    T.num_nodes = m;
    T.max_level = max_level;
    for (int t = 0; t < 2; ++t) {
        T.rec[t].alloc(m);
    }
    T.topo.alloc(m);
    T.maxdim.alloc(m);
    for (int a = 0; a < 3; ++a) {
        T.bmin[a].alloc(m);
        T.bmax[a].alloc(m);
    }
    T.parent.alloc(m);
    T.meta.alloc(m);
    T.dirty.alloc(m);
    RL_CUDA_TRY(cudaMemsetAsync(T.dirty.p, 0, m * sizeof(uint32_t), st));
    T.work.alloc(m);
    T.level_dirty.alloc(kMaxLevels + 2);
    T.level_runs.alloc(1);
    RL_CUDA_TRY(cudaMemsetAsync(T.level_runs.p, 0, sizeof(unsigned long long), st));
    T.level_runs_seen = 0;
    T.last_counts.alloc(n);
    T.first_key.alloc(m);
    T.leaf_of.alloc(n);
    T.morton.alloc(n);
    RL_CUDA_TRY(cudaMemcpyAsync(T.morton.p, idx.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));

    DBuf<uint32_t> level_count;
    level_count.alloc(kMaxLevels + 2);
    RL_CUDA_TRY(cudaMemsetAsync(level_count.p, 0, (kMaxLevels + 2) * sizeof(uint32_t), st));
    FillArgs A;
    A.n = n;
    A.m = m;
    A.skey = skey.p;
    A.sval = sval.p;
    A.bfs_of = bfs_of.p;
    A.lcp = lcp.p;
    A.k0s = k0s.p;
    A.key1 = key1.p;
    A.idx = idx.p;
    A.px = c.nr.px.p;
    A.py = c.nr.py.p;
    A.pz = c.nr.pz.p;
    A.nets = c.d_nets.p;
    A.net_of = c.net_of.p;
    A.rec0 = T.rec[0].p;
    A.rec1 = T.rec[1].p;
    A.topo = T.topo.p;
    A.maxdim = T.maxdim.p;
    A.bx0 = T.bmin[0].p;
    A.by0 = T.bmin[1].p;
    A.bz0 = T.bmin[2].p;
    A.bx1 = T.bmax[0].p;
    A.by1 = T.bmax[1].p;
    A.bz1 = T.bmax[2].p;
    A.first_key = T.first_key.p;
    A.leaf_of = T.leaf_of.p;
    A.parent = T.parent.p;
    A.level_count = level_count.p;
    k_fill<<<blocks_for(m, 256), 256, 0, st>>>(A);
    RL_LAUNCH_CHECK();
    std::vector<uint32_t> hcount(kMaxLevels + 2, 0);
    RL_CUDA_TRY(cudaMemcpyAsync(hcount.data(), level_count.p, hcount.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<uint32_t> hoff(kMaxLevels + 3, 0);
    for (int l = 0; l < kMaxLevels + 2; ++l) {
        hoff[l + 1] = hoff[l] + hcount[l];
    }
    T.level_off = hoff;
    T.level_lo.alloc(hoff.size());
    RL_CUDA_TRY(cudaMemcpyAsync(T.level_lo.p, T.level_off.data(), hoff.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    DBuf<uint32_t> level_off;
    level_off.alloc(hoff.size());
    RL_CUDA_TRY(cudaMemcpyAsync(level_off.p, hoff.data(), hoff.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    k_parent_search<<<blocks_for(m, 256), 256, 0, st>>>(m, level_off.p, T.first_key.p, T.topo.p, T.parent.p);
    RL_LAUNCH_CHECK();
    k_child_mask<<<blocks_for(m, 256), 256, 0, st>>>(m, T.parent.p, T.first_key.p, k0s.p, idx.p, key1.p, T.topo.p);
    RL_LAUNCH_CHECK();
    k_meta<<<blocks_for(m, 256), 256, 0, st>>>(m, T.parent.p, T.topo.p, T.maxdim.p, T.meta.p, c.err.p);
    RL_LAUNCH_CHECK();
    // the roots: level 0 holds one node per network, in network order
    const size_t K = c.nets.size();
    RL_CHECK(hcount[0] == K, RL_ERR_INVALID, "every network needs at least one neuron");
    std::vector<uint2> roots(K);
    RL_CUDA_TRY(cudaMemcpyAsync(roots.data(), T.topo.p, K * sizeof(uint2), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t k = 0; k < K; ++k) {
        c.nets[k].root_leaf = topo_leaf(roots[k].y) ? 1u : 0u;
    }
    RL_CUDA_TRY(cudaMemcpyAsync(c.d_nets.p, c.nets.data(), K * sizeof(NetInfo), cudaMemcpyHostToDevice, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    T.root_is_leaf = K == 1 && topo_leaf(roots[0].y);
    T.root_neuron = roots[0].x;
    check_device_error(c, "octree build");
}

void update_tree(Ctx& c) {
    const uint32_t n = c.n;
    Tree& T = c.tree;
    ReduceArgs A;
    A.n = n;
    A.leaf_of = T.leaf_of.p;
    A.parent = T.parent.p;
    A.topo = T.topo.p;
    A.bx0 = T.bmin[0].p;
    A.by0 = T.bmin[1].p;
    A.bz0 = T.bmin[2].p;
    A.bx1 = T.bmax[0].p;
    A.by1 = T.bmax[1].p;
    A.bz1 = T.bmax[2].p;
    A.rec0 = T.rec[0].p;
    A.rec1 = T.rec[1].p;
    A.arrive = nullptr;
    A.dirty = T.dirty.p;
    A.level_dirty = T.level_dirty.p;
    A.work = T.work.p;
    A.level_lo = T.level_lo.p;
    A.last = T.last_counts.p;
    A.enabled = c.nr.enabled.p;
    A.update = c.nr.update.p;
    A.vac_exc = c.nr.vacant[1].p;
    A.vac_inh = c.nr.vacant[2].p;
    // the FP32 form's fixed-point records follow the update once they exist
    const bool keep_q = is_fp32(c) && T.recq_valid;
    if (!keep_q) {
        T.recq_valid = false;
    }
    A.recq0 = keep_q ? T.recq[0].p : nullptr;
    A.recq1 = keep_q ? T.recq[1].p : nullptr;
    A.first_key = T.first_key.p;
    A.morton = T.morton.p;
    A.net_of = c.net_of.p;
    A.nets = c.d_nets.p;
    // bottom-up, one launch per level from the deepest level with inner nodes
    int deepest = (int)T.level_off.size() - 2;
    while (deepest > 0 && T.level_off[deepest + 1] == T.level_off[deepest]) {
        --deepest;
    }
    A.has_cond = 0;
    A.cond = 0;
    A.level_runs = nullptr;
    auto enqueue_leaves = [&](cudaStream_t st, const ReduceArgs& a) {
        RL_CUDA_TRY(cudaMemsetAsync(T.level_dirty.p, 0, T.level_dirty.n * sizeof(uint32_t), st));
        launch_pdl(&k_leaf_update, blocks_for(n, 256), 256, st, a);
    };
    auto enqueue_levels = [&](cudaStream_t st, const ReduceArgs& a) {
        uint32_t kernels = 0;
        const unsigned cap = 4u * (unsigned)c.num_sms;
        for (int l = deepest - 1; l >= 0; --l) {
            const uint32_t lo = T.level_off[l], hi = T.level_off[l + 1];
            if (hi > lo) {
                const unsigned blocks = blocks_for(hi - lo, 128);
                launch_pdl(&k_reduce_level, blocks < cap ? blocks : cap, 128, st, a, lo, hi, (uint32_t)l);
                ++kernels;
            }
        }
        return kernels;
    };
    // the first update after a build (or after an update outside this path)
    // takes every leaf as changed
    const int force = T.force_full ? 1 : 0;
    T.force_full = false;
    if (force || !c.use_graphs || c.stream == nullptr || c.capturing) {
        ReduceArgs a = A;
        a.force = force;
        enqueue_leaves(c.stream, a);
        enqueue_levels(c.stream, a);
        return;
    }
    if (T.update_graph != nullptr && keep_q != T.graph_keeps_q) {
        T.drop_graph();
    }
    // The launches depend only on the octree's shape: captured once per build,
    // as the leaf pass followed by a conditional node whose body holds the
    // level reductions.  The leaf pass sets the condition when it changes a
    // leaf, so an update that changes none (most of them in a long run) ends
    // after one kernel.  The level launches count themselves on the device.
    if (T.update_graph == nullptr) {
        T.graph_keeps_q = keep_q;
        const uint64_t launches = c.launches;
        cudaGraph_t gr = nullptr;
        RL_CUDA_TRY(cudaGraphCreate(&gr, 0));
        cudaGraphConditionalHandle cond = 0;
        ReduceArgs a = A;
        a.force = 0;
        bool capturing = false;
        try {
            RL_CUDA_TRY(cudaGraphConditionalHandleCreate(&cond, gr, 0u, cudaGraphCondAssignDefault));
            a.has_cond = 1;
            a.cond = cond;
            a.level_runs = T.level_runs.p;
            RL_CUDA_TRY(cudaStreamBeginCaptureToGraph(c.stream, gr, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            capturing = c.capturing = true;
            enqueue_leaves(c.stream, a);
            cudaStreamCaptureStatus status;
            const cudaGraphNode_t* deps = nullptr;
            size_t ndeps = 0;
            RL_CUDA_TRY(cudaStreamGetCaptureInfo(c.stream, &status, nullptr, nullptr, &deps, &ndeps));
            cudaGraphNodeParams cp{};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeIf;
            cp.conditional.size = 1;
            cudaGraphNode_t cnode = nullptr;
            RL_CUDA_TRY(cudaGraphAddNode(&cnode, gr, deps, ndeps, &cp));
            RL_CUDA_TRY(cudaStreamUpdateCaptureDependencies(c.stream, &cnode, 1, cudaStreamSetCaptureDependencies));
            RL_CUDA_TRY(cudaStreamEndCapture(c.stream, &gr));
            capturing = c.capturing = false;
            // the body: the level reductions
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            RL_CUDA_TRY(cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            capturing = c.capturing = true;
            enqueue_levels(c.stream, a);
            RL_CUDA_TRY(cudaStreamEndCapture(c.stream, &body));
            capturing = c.capturing = false;
        } catch (...) {
            if (capturing) {
                cudaGraph_t g2 = nullptr;
                cudaStreamEndCapture(c.stream, &g2);
            }
            c.capturing = false;
            cudaGraphDestroy(gr);
            c.launches = launches;
            throw;
        }
        c.launches = launches;
        cudaGraphExec_t ex = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
        cudaGraphDestroy(gr);
        RL_CUDA_TRY(e);
        T.update_graph = ex;
    }
    RL_CUDA_TRY(cudaGraphLaunch(T.update_graph, c.stream));
    c.launches += 1;  // the leaf pass; the level launches are counted on the device
}

void launch_tree_update_scratch(Ctx& c, const uint32_t* d_vac_exc, const uint32_t* d_vac_inh, const uint8_t* d_update, uint32_t* arrive,
                                cudaStream_t st) {
    const uint32_t n = c.n;
    Tree& T = c.tree;
    // this update bypasses the incremental bookkeeping: the next regular one is complete
    T.force_full = true;
    T.recq_valid = false;
    k_leaf_counts<<<blocks_for(n, 256), 256, 0, st>>>(n, T.leaf_of.p, c.nr.enabled.p, d_update ? d_update : c.nr.enabled.p, d_vac_exc, d_vac_inh,
                                                      T.rec[0].p, T.rec[1].p);
    RL_LAUNCH_CHECK();
    if (T.root_is_leaf) {
        return;
    }
    RL_CUDA_TRY(cudaMemsetAsync(arrive, 0, T.num_nodes * sizeof(uint32_t), st));
    ReduceArgs A;
    A.n = n;
    A.leaf_of = T.leaf_of.p;
    A.parent = T.parent.p;
    A.topo = T.topo.p;
    A.bx0 = T.bmin[0].p;
    A.by0 = T.bmin[1].p;
    A.bz0 = T.bmin[2].p;
    A.bx1 = T.bmax[0].p;
    A.by1 = T.bmax[1].p;
    A.bz1 = T.bmax[2].p;
    A.rec0 = T.rec[0].p;
    A.rec1 = T.rec[1].p;
    A.arrive = arrive;
    k_reduce<<<blocks_for(n, 128), 128, 0, st>>>(A);
    RL_LAUNCH_CHECK();
}

void dump_tree(Ctx& c, int32_t* level, int32_t* neuron, uint8_t* child_mask, int32_t* first_child, double* bmin, double* bmax, uint32_t* cnt_exc,
               uint32_t* cnt_inh, double* pos_exc, double* pos_inh) {
    const uint32_t m = c.tree.num_nodes;
    cudaStream_t st = c.stream;
    std::vector<uint2> topo(m);
    std::vector<double4> r0(m), r1(m);
    std::vector<double> b[6];
    RL_CUDA_TRY(cudaMemcpyAsync(topo.data(), c.tree.topo.p, m * sizeof(uint2), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaMemcpyAsync(r0.data(), c.tree.rec[0].p, m * sizeof(double4), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaMemcpyAsync(r1.data(), c.tree.rec[1].p, m * sizeof(double4), cudaMemcpyDeviceToHost, st));
    for (int a = 0; a < 3; ++a) {
        b[a].resize(m);
        b[3 + a].resize(m);
        RL_CUDA_TRY(cudaMemcpyAsync(b[a].data(), c.tree.bmin[a].p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
        RL_CUDA_TRY(cudaMemcpyAsync(b[3 + a].data(), c.tree.bmax[a].p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    const double nan = __builtin_nan("");
    for (uint32_t i = 0; i < m; ++i) {
        const bool leaf = topo_leaf(topo[i].y);
        if (level) level[i] = (int32_t)topo_level(topo[i].y);
        if (neuron) neuron[i] = leaf ? (int32_t)topo[i].x : -1;
        if (child_mask) child_mask[i] = (uint8_t)topo_mask(topo[i].y);
        if (first_child) first_child[i] = leaf ? -1 : (int32_t)topo[i].x;
        for (int a = 0; a < 3; ++a) {
            if (bmin) bmin[3 * (size_t)i + a] = b[a][i];
            if (bmax) bmax[3 * (size_t)i + a] = b[3 + a][i];
        }
        uint64_t ce, ci;
        __builtin_memcpy(&ce, &r0[i].w, 8);
        __builtin_memcpy(&ci, &r1[i].w, 8);
        if (cnt_exc) cnt_exc[i] = (uint32_t)ce;
        if (cnt_inh) cnt_inh[i] = (uint32_t)ci;
        const bool he = leaf || (uint32_t)ce > 0;
        const bool hi = leaf || (uint32_t)ci > 0;
        if (pos_exc) {
            pos_exc[3 * (size_t)i] = he ? r0[i].x : nan;
            pos_exc[3 * (size_t)i + 1] = he ? r0[i].y : nan;
            pos_exc[3 * (size_t)i + 2] = he ? r0[i].z : nan;
        }
        if (pos_inh) {
            pos_inh[3 * (size_t)i] = hi ? r1[i].x : nan;
            pos_inh[3 * (size_t)i + 1] = hi ? r1[i].y : nan;
            pos_inh[3 * (size_t)i + 2] = hi ? r1[i].z : nan;
        }
    }
}

}  // namespace rl
