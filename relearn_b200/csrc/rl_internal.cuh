// Internal declarations shared by the translation units of librelearn_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/relearn_b200.h"

namespace rl {

// ------------------------------------------------------------------ errors
struct Error {
    rl_status status;
    std::string message;
};

#define RL_CUDA_TRY(expr)                                                                              \
    do {                                                                                               \
        cudaError_t _e = (expr);                                                                       \
        if (_e != cudaSuccess) {                                                                       \
            throw ::rl::Error{ _e == cudaErrorMemoryAllocation ? RL_ERR_OOM : RL_ERR_DEVICE,           \
                               std::string(#expr) + ": " + cudaGetErrorString(_e) };                   \
        }                                                                                              \
    } while (0)

#define RL_CHECK(cond, status, msg)                        \
    do {                                                   \
        if (!(cond)) {                                     \
            throw ::rl::Error{ (status), std::string(msg) }; \
        }                                                  \
    } while (0)

// The context an entry point works for, bound to the calling thread for the
// duration of the call: the stream its device memory is ordered on and its
// launch and device-memory counters.  Contexts driven from different host
// threads therefore share no mutable state in the library.
struct Binding {
    cudaStream_t stream = nullptr;
    uint64_t* launches = nullptr;
    int64_t* bytes = nullptr;
    int64_t* peak = nullptr;
};
extern thread_local Binding g_bind;

// Every kernel launch of the library goes through this counter.
#define RL_LAUNCH_CHECK()                          \
    do {                                           \
        if (::rl::g_bind.launches) {               \
            ++*::rl::g_bind.launches;              \
        }                                          \
        RL_CUDA_TRY(cudaPeekAtLastError());        \
    } while (0)

constexpr int kSmCount = 148;

// Programmatic dependent launch: a kernel launched this way may be scheduled
// while its stream predecessor is still draining (its blocks become resident
// as the predecessor's last wave leaves the SMs), which hides the launch gap
// between the short kernels of an activity block.  Such a kernel begins with
// pdl_wait(), which returns once the predecessor grid has completed and its
// memory is visible, and then lets its own successor launch.
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    RL_CUDA_TRY(cudaLaunchKernelEx(&cfg, kernel, args...));
    if (g_bind.launches) {
        ++*g_bind.launches;
    }
}

#if defined(__CUDACC__)
__device__ __forceinline__ void pdl_wait_then_release() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#endif

inline unsigned blocks_for(uint64_t n, unsigned threads) {
    uint64_t b = (n + threads - 1) / threads;
    if (b == 0) {
        b = 1;
    }
    return (unsigned)b;
}

// Device error word bits (written by kernels, read by the host after a phase).
enum DeviceError : uint32_t {
    DERR_NONE = 0,
    DERR_OUT_OF_BOX = 1u << 0,      // a position outside the root cell
    DERR_DUPLICATE = 1u << 1,       // two positions share all key levels
    DERR_STACK = 1u << 2,           // a walk or descent ran past its depth bound
    DERR_NO_CROSSING = 1u << 3,     // pick scan found no crossing
    DERR_CAPACITY = 1u << 4,        // a device buffer was too small
    DERR_CONNECT = 1u << 5,         // connector bookkeeping underflow
    DERR_TIMEOUT = 1u << 6,         // bounded wait ran out
    DERR_WALK = 1u << 7,            // a walk left the node range or its bound
};

// ------------------------------------------------------------- device buffer
// Device memory is stream ordered (cudaMallocAsync / cudaFreeAsync from the
// device's memory pool) on the bound context's stream, so contexts that run
// side by side never synchronise the device by allocating or freeing, and the
// bytes each context holds are counted.
inline void account(int64_t delta) {
    if (g_bind.bytes) {
        *g_bind.bytes += delta;
        if (g_bind.peak && *g_bind.bytes > *g_bind.peak) {
            *g_bind.peak = *g_bind.bytes;
        }
    }
}

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        release();
        if (count == 0) {
            count = 1;
        }
        RL_CUDA_TRY(cudaMallocAsync((void**)&p, count * sizeof(T), g_bind.stream));
        n = count;
        account((int64_t)(n * sizeof(T)));
    }
    void ensure(size_t count) {
        if (count > n || p == nullptr) {
            size_t c = n ? n : 1;
            while (c < count) {
                c *= 2;
            }
            alloc(c);
        }
    }
    // Capacity for `count` with an eighth of headroom, for arrays kept
    // between calls whose size drifts a little from call to call.
    void fit(size_t count) {
        if (count > n || p == nullptr) {
            alloc(count + count / 8);
        }
    }
    void release() {
        if (p) {
            if (g_bind.stream) {
                cudaFreeAsync(p, g_bind.stream);
            } else {
                cudaFree(p);
            }
            account(-(int64_t)(n * sizeof(T)));
        }
        p = nullptr;
        n = 0;
    }
    void swap(DBuf& o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
    ~DBuf() { release(); }
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
};

// ------------------------------------------------------------- primitives
// Scratch for the primitives; grows on demand.
struct PrimScratch {
    DBuf<uint32_t> a, b, c;
    DBuf<uint64_t> k64;
    DBuf<uint32_t> v32;
};

// out[i] = sum_{j<i} in[i]; returns the total (synchronous read of one word).
// in and out may alias.
uint32_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, PrimScratch& s, cudaStream_t st);
// Same without the host read: returns a device pointer to the total.
uint32_t* exclusive_scan_u32_async(const uint32_t* in, uint32_t* out, uint64_t n, PrimScratch& s, cudaStream_t st);

// Stable LSD radix sort of (key, value) pairs on the low `bits` bits of the
// keys.  keys/vals are sorted in place (ping-pong through the scratch).
void radix_sort_u64(uint64_t* keys, uint32_t* vals, uint64_t n, int bits, PrimScratch& s, cudaStream_t st);
void radix_sort_u32(uint32_t* keys, uint32_t* vals, uint64_t n, int bits, PrimScratch& s, cudaStream_t st);

}  // namespace rl
