// Allocation-free tree update.
//
// Some callers cannot allocate device memory at the point where they update
// the octree: runtimes that hand out all device memory from their own fixed
// pool or budget, and hosts that must not touch the CUDA allocator during a
// simulation once set-up has finished.  rl_prepare_update_connectivity_noalloc
// serves them: it takes device arrays for its inputs, writes its results into
// the context's octree and copies the dendrite counts and plasticity flags into
// the context's own arrays (the connector accepts against those), and keeps
// the only scratch it needs — one arrival
// counter per octree node for the bottom-up reduction — in a file-scope device
// array instead of context memory.  It calls no cudaMalloc / cudaFree and no
// allocating library routine.
//
// The scratch array holds kMaxNodes counters (8 MiB) and is part of every GPU
// that loads the library, until the process exits.  All calls share it and it
// keeps the last call's contents: each call clears the counters it uses before
// the reduction, and calls that overlap on the GPU (on different streams, or
// from different contexts on the same device) race on it.
//
// Host code cannot use the array's name as a device address, so its device
// address is looked up once per device with cudaGetSymbolAddress, with that
// device current, on the first call on that device; that first call should
// come before any stream capture.
#include <mutex>

#include "rl_context.cuh"

namespace {

constexpr uint32_t kMaxNodes = 1u << 21;  // 2,097,152 nodes

static __device__ __align__(256) uint32_t g_tree_arrive[kMaxNodes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
uint32_t* g_scratch[kMaxDevices] = {};

// Device address of g_tree_arrive on `device` (looked up on first use).
uint32_t* scratch_on(int device) {
    RL_CHECK(device >= 0 && device < kMaxDevices, RL_ERR_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_scratch[device] == nullptr) {
        void* p = nullptr;
        RL_CUDA_TRY(cudaGetSymbolAddress(&p, g_tree_arrive));
        g_scratch[device] = static_cast<uint32_t*>(p);
    }
    return g_scratch[device];
}

}  // namespace

extern "C" RL_API rl_status rl_prepare_update_connectivity_noalloc(void* ctx, const uint32_t* d_vacant_exc, const uint32_t* d_vacant_inh,
                                                                   const uint8_t* d_update, void* cuda_stream) {
    if (!ctx) {
        return RL_ERR_INVALID;
    }
    rl::Ctx& c = *static_cast<rl::Ctx*>(ctx);
    // the caller's current device comes back on every return path
    int prev_device = -1;
    cudaGetDevice(&prev_device);
    struct RestoreDevice {
        int d;
        ~RestoreDevice() {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{ prev_device };
    const rl::Binding prev_bind = rl::g_bind;
    try {
        RL_CHECK(c.positions_set, RL_ERR_INVALID, "rl_set_positions has not been called");
        RL_CHECK(d_vacant_exc && d_vacant_inh, RL_ERR_INVALID, "device vacancy arrays are required");
        RL_CHECK(c.tree.num_nodes <= kMaxNodes, RL_ERR_OVERFLOW,
                 "the octree has " + std::to_string(c.tree.num_nodes) + " nodes; the allocation-free update supports at most " +
                     std::to_string(kMaxNodes));
        RL_CUDA_TRY(cudaSetDevice(c.device));
        uint32_t* arrive = scratch_on(c.device);
        if (c.noalloc_before == nullptr) {
            // set-up of the first call on this context (not a memory allocation)
            RL_CUDA_TRY(cudaEventCreateWithFlags(&c.noalloc_before, cudaEventDisableTiming));
            RL_CUDA_TRY(cudaEventCreateWithFlags(&c.noalloc_after, cudaEventDisableTiming));
        }
        cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : c.stream;
        rl::g_bind = rl::Binding{ st, &c.launches, &c.device_bytes, &c.device_peak };
        if (st != c.stream) {
            // the octree is rewritten only after the context's earlier work, which may still read it
            RL_CUDA_TRY(cudaEventRecord(c.noalloc_before, c.stream));
            RL_CUDA_TRY(cudaStreamWaitEvent(st, c.noalloc_before, 0));
        }
        // the connector accepts against the context's dendrite counts and plasticity flags:
        // they take the new values too, as rl_prepare_update_connectivity does
        const size_t n = c.n;
        RL_CUDA_TRY(cudaMemcpyAsync(c.nr.vacant[1].p, d_vacant_exc, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        RL_CUDA_TRY(cudaMemcpyAsync(c.nr.vacant[2].p, d_vacant_inh, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        RL_CUDA_TRY(cudaMemcpyAsync(c.nr.update.p, d_update ? d_update : c.nr.enabled.p, n, cudaMemcpyDeviceToDevice, st));
        rl::launch_tree_update_scratch(c, d_vacant_exc, d_vacant_inh, d_update, arrive, st);
        if (st != c.stream) {
            // the context's later work (searches, FP32 record refresh, graphs) reads the new octree
            RL_CUDA_TRY(cudaEventRecord(c.noalloc_after, st));
            RL_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.noalloc_after, 0));
        }
        rl::g_bind = prev_bind;
        return RL_OK;
    } catch (const rl::Error& e) {
        rl::g_bind = prev_bind;
        c.last_error = e.message;
        return e.status;
    } catch (...) {
        rl::g_bind = prev_bind;
        c.last_error = "unexpected host exception";
        return RL_ERR_INVALID;
    }
}
