// Device-wide primitives written for this library: exclusive scan of u32 and
// a stable LSD radix sort (8-bit digits) of (key, u32 value) pairs.
//
// Radix sort layout: a tile is 2048 keys handled by 256 threads in 8 rounds
// of 256 consecutive keys (striped), so processing order equals input order
// and the scatter is stable.  Per pass: digit histogram per tile (digit-major
// counts), one device scan over the counts, then the scatter ranks every key
// inside its tile with __match_any_sync (peers with the same digit in the
// warp) plus per-warp digit counts in shared memory.
#include "rl_internal.cuh"

namespace rl {

thread_local Binding g_bind;


namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) {
            v += t;
        }
    }
    return v;
}

// Exclusive block scan of one value per thread (blockDim a multiple of 32);
// the block total is returned in *total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[33];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const uint32_t inc = warp_inclusive_scan(v);
    if (lane == 31) {
        warp_sums[warp] = inc;
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < nwarps ? warp_sums[lane] : 0u;
        const uint32_t wi = warp_inclusive_scan(w);
        warp_sums[lane] = wi - w;
        if (lane == 31) {
            warp_sums[32] = wi;
        }
    }
    __syncthreads();
    const uint32_t res = warp_sums[warp] + inc - v;
    *total = warp_sums[32];
    __syncthreads();
    return res;
}

__global__ void scan_tile_sums(const uint32_t* __restrict__ in, uint64_t n, uint32_t* __restrict__ sums) {
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) {
            s += in[base + k];
        }
    }
    uint32_t total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) {
        sums[blockIdx.x] = total;
    }
}

// Single block: exclusive scan of sums[0..m), grand total to sums[m].
__global__ void scan_sums_single(uint32_t* sums, uint32_t m) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < m; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < m ? sums[i] : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(v, &total);
        if (i < m) {
            sums[i] = carry + ex;
        }
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[m] = carry;
    }
}

// An array of at most one tile in one launch: the exclusive scan and its
// total (in and out may be the same array).
__global__ void scan_one_tile(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* __restrict__ total_out) {
    const uint64_t base = (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) {
            out[base + k] = run;
        }
        run += v[k];
    }
    if (threadIdx.x == 0) {
        *total_out = total;
    }
}

__global__ void scan_apply(const uint32_t* in, uint32_t* out, uint64_t n, const uint32_t* __restrict__ sums) {
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = block_exclusive_scan(s, &total) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) {
            out[base + k] = run;
        }
        run += v[k];
    }
}

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 8;
constexpr int kSortTile = kSortThreads * kSortRounds;

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_hist(const K* __restrict__ keys, uint64_t n, int shift, uint32_t* __restrict__ counts,
                                                           uint32_t num_tiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t i = base + (uint64_t)r * kSortThreads + threadIdx.x;
        if (i < n) {
            atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 255u], 1u);
        }
    }
    __syncthreads();
    counts[(uint64_t)threadIdx.x * num_tiles + blockIdx.x] = h[threadIdx.x];
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_scatter(const K* __restrict__ kin, const uint32_t* __restrict__ vin, K* __restrict__ kout,
                                                              uint32_t* __restrict__ vout, uint64_t n, int shift, const uint32_t* __restrict__ offsets,
                                                              uint32_t num_tiles) {
    __shared__ uint32_t base_off[256];
    __shared__ uint32_t run[256];
    __shared__ uint32_t wc[kSortThreads / 32][256];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    base_off[tid] = offsets[(uint64_t)tid * num_tiles + blockIdx.x];
    run[tid] = 0;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
        wc[w][tid] = 0;
    }
    __syncthreads();
    const uint64_t tile = (uint64_t)blockIdx.x * kSortTile;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int r = 0; r < kSortRounds; ++r) {
        const uint64_t i = tile + (uint64_t)r * kSortThreads + tid;
        const bool valid = i < n;
        K k = 0;
        uint32_t v = 0;
        uint32_t d = 256u;
        if (valid) {
            k = kin[i];
            v = vin[i];
            d = (uint32_t)(k >> shift) & 255u;
        }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        const uint32_t lrank = __popc(peers & lt_mask);
        if (valid && lrank == 0) {
            wc[warp][d] = __popc(peers);
        }
        __syncthreads();
        if (valid) {
            uint32_t off = run[d];
            for (int w = 0; w < warp; ++w) {
                off += wc[w][d];
            }
            const uint32_t pos = base_off[d] + off + lrank;
            kout[pos] = k;
            vout[pos] = v;
        }
        __syncthreads();
        uint32_t tsum = 0;
#pragma unroll
        for (int w = 0; w < kSortThreads / 32; ++w) {
            tsum += wc[w][tid];
            wc[w][tid] = 0;
        }
        run[tid] += tsum;
        __syncthreads();
    }
}

// Up to kSmallRadix pairs are sorted by one block with the pairs in shared
// memory: the same 8-bit passes and the same stable order as the multi-block
// sort (a pass counts the digits, scans the 256 counts, and scatters rounds of
// kSmallThreads consecutive keys, ranking equal digits by their position), so
// the same permutation, in one launch instead of five per pass.
constexpr uint32_t kSmallRadix = 4096;
constexpr int kSmallThreads = 1024;

template <typename K>
__global__ void __launch_bounds__(kSmallThreads) radix_small(K* keys, uint32_t* vals, uint32_t n, int passes) {
    extern __shared__ __align__(16) unsigned char smem[];
    K* ka = reinterpret_cast<K*>(smem);
    K* kb = ka + kSmallRadix;
    uint32_t* va = reinterpret_cast<uint32_t*>(kb + kSmallRadix);
    uint32_t* vb = va + kSmallRadix;
    __shared__ uint32_t run[256];
    __shared__ uint32_t wsum[8];
    __shared__ uint32_t wc[kSmallThreads / 32][256];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    for (uint32_t i = tid; i < n; i += kSmallThreads) {
        ka[i] = keys[i];
        va[i] = vals[i];
    }
    for (int e = tid; e < (kSmallThreads / 32) * 256; e += kSmallThreads) {
        wc[e >> 8][e & 255] = 0u;
    }
    __syncthreads();
    K* kin = ka;
    K* kout = kb;
    uint32_t* vin = va;
    uint32_t* vout = vb;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        if (tid < 256) {
            run[tid] = 0u;
        }
        __syncthreads();
        for (uint32_t i = tid; i < n; i += kSmallThreads) {
            atomicAdd(&run[(uint32_t)(kin[i] >> shift) & 255u], 1u);
        }
        __syncthreads();
        // exclusive scan of the 256 digit counts by the first eight warps
        uint32_t cnt = 0, inc = 0;
        if (tid < 256) {
            cnt = run[tid];
            inc = warp_inclusive_scan(cnt);
            if (lane == 31) {
                wsum[warp] = inc;
            }
        }
        __syncthreads();
        if (tid < 256) {
            uint32_t before = 0;
            for (int w = 0; w < warp; ++w) {
                before += wsum[w];
            }
            run[tid] = before + inc - cnt;
        }
        __syncthreads();
        for (uint32_t base = 0; base < n; base += kSmallThreads) {
            const uint32_t i = base + (uint32_t)tid;
            const bool valid = i < n;
            K k = 0;
            uint32_t v = 0;
            uint32_t d = 256u;
            if (valid) {
                k = kin[i];
                v = vin[i];
                d = (uint32_t)(k >> shift) & 255u;
            }
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
            const uint32_t lrank = __popc(peers & lt_mask);
            if (valid && lrank == 0) {
                wc[warp][d] = __popc(peers);
            }
            __syncthreads();
            if (valid) {
                uint32_t off = run[d];
                for (int w = 0; w < warp; ++w) {
                    off += wc[w][d];
                }
                kout[off + lrank] = k;
                vout[off + lrank] = v;
            }
            __syncthreads();
            if (tid < 256) {
                uint32_t tsum = 0;
#pragma unroll 8
                for (int w = 0; w < kSmallThreads / 32; ++w) {
                    tsum += wc[w][tid];
                    wc[w][tid] = 0u;
                }
                run[tid] += tsum;
            }
            __syncthreads();
        }
        K* tk = kin;
        kin = kout;
        kout = tk;
        uint32_t* tv = vin;
        vin = vout;
        vout = tv;
    }
    for (uint32_t i = tid; i < n; i += kSmallThreads) {
        keys[i] = kin[i];
        vals[i] = vin[i];
    }
}

template <typename K>
void radix_sort_impl(K* keys, uint32_t* vals, uint64_t n, int bits, DBuf<K>& ktmp, PrimScratch& s, cudaStream_t st) {
    if (n <= 1 || bits <= 0) {
        return;
    }
    if (n <= kSmallRadix) {
        const size_t smem = (size_t)kSmallRadix * 2 * (sizeof(K) + sizeof(uint32_t));
        RL_CUDA_TRY(cudaFuncSetAttribute((const void*)&radix_small<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        radix_small<K><<<1, kSmallThreads, smem, st>>>(keys, vals, (uint32_t)n, (bits + 7) / 8);
        RL_LAUNCH_CHECK();
        return;
    }
    const uint32_t num_tiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
    s.a.ensure((size_t)256 * num_tiles + 1);
    ktmp.ensure(n);
    s.v32.ensure(n);
    K* kin = keys;
    K* kout = ktmp.p;
    uint32_t* vin = vals;
    uint32_t* vout = s.v32.p;
    const int passes = (bits + 7) / 8;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        radix_hist<K><<<num_tiles, kSortThreads, 0, st>>>(kin, n, shift, s.a.p, num_tiles);
        RL_LAUNCH_CHECK();
        exclusive_scan_u32_async(s.a.p, s.a.p, (uint64_t)256 * num_tiles, s, st);
        radix_scatter<K><<<num_tiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, shift, s.a.p, num_tiles);
        RL_LAUNCH_CHECK();
        K* tk = kin;
        kin = kout;
        kout = tk;
        uint32_t* tv = vin;
        vin = vout;
        vout = tv;
    }
    if (kin != keys) {
        RL_CUDA_TRY(cudaMemcpyAsync(keys, kin, n * sizeof(K), cudaMemcpyDeviceToDevice, st));
        RL_CUDA_TRY(cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    }
}

}  // namespace

uint32_t* exclusive_scan_u32_async(const uint32_t* in, uint32_t* out, uint64_t n, PrimScratch& s, cudaStream_t st) {
    const uint32_t tiles = (uint32_t)((n + kScanTile - 1) / kScanTile);
    const uint32_t t = tiles ? tiles : 1;
    s.c.ensure((size_t)t + 1);
    if (tiles == 1) {
        scan_one_tile<<<1, kScanThreads, 0, st>>>(in, out, n, s.c.p + 1);
        RL_LAUNCH_CHECK();
        return s.c.p + 1;
    }
    if (n > 0) {
        scan_tile_sums<<<t, kScanThreads, 0, st>>>(in, n, s.c.p);
        RL_LAUNCH_CHECK();
    } else {
        RL_CUDA_TRY(cudaMemsetAsync(s.c.p, 0, sizeof(uint32_t), st));
    }
    scan_sums_single<<<1, 1024, 0, st>>>(s.c.p, n > 0 ? t : 0u);
    RL_LAUNCH_CHECK();
    if (n > 0) {
        scan_apply<<<t, kScanThreads, 0, st>>>(in, out, n, s.c.p);
        RL_LAUNCH_CHECK();
    }
    return s.c.p + (n > 0 ? t : 0u);
}

uint32_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, PrimScratch& s, cudaStream_t st) {
    const uint32_t* dtotal = exclusive_scan_u32_async(in, out, n, s, st);
    uint32_t total = 0;
    RL_CUDA_TRY(cudaMemcpyAsync(&total, dtotal, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    RL_CUDA_TRY(cudaStreamSynchronize(st));
    return total;
}

void radix_sort_u64(uint64_t* keys, uint32_t* vals, uint64_t n, int bits, PrimScratch& s, cudaStream_t st) {
    radix_sort_impl<uint64_t>(keys, vals, n, bits, s.k64, s, st);
}

void radix_sort_u32(uint32_t* keys, uint32_t* vals, uint64_t n, int bits, PrimScratch& s, cudaStream_t st) {
    radix_sort_impl<uint32_t>(keys, vals, n, bits, s.b, s, st);
}

}  // namespace rl
