// bn_noalloc.cu -- Protocol 2 verification that allocates nothing.
//
// bn_flat_verify_noalloc runs the same Freivalds computation as
// bn_flat_verify with the CUDA-core engine, but every byte of scratch it
// needs lives in the file-scope array below.  It exists for callers that
// cannot allocate device memory while they score:
//   - services that pre-reserve their whole device-memory budget at start-up
//     (the reference's VRAM budget model, scorer-gpu-common/src/budget.rs)
//     and must not fail an allocation under memory pressure mid-request;
//   - latency-critical request threads, where cudaMalloc / cudaFree may
//     synchronise the device and stall every stream in flight.
//
// CUDA loads a module lazily, when one of its kernels or symbols is first
// used, and the load itself allocates device memory (this array among it).
// So bn_ctx_create calls bn_internal_noalloc_setup for its device, which
// resolves the array's address and loads every kernel the entry point
// launches; after that the entry point allocates nothing.
//
// Limits: at most BN_NOALLOC_MAX_TRIALS trials and the row chunking below
// (the array holds 16 x 24 chunk-trial pairs of 1024 z partials, ~3 MiB per
// GPU, kept until the process exits; fewer trials leave room for more
// chunks).  With 16 chunks, at N = 1M rows and 20 trials, a call took
// 138 ms on a B200, against 62 ms for the CUDA-core engine's Protocol 2 in
// bn_flat_query (which spreads the rows over ~150 chunks) and about 1.5 ms
// for the fused tensor-core pass.  Every call shares the one array, so
// calls that overlap on the GPU (two streams, or two threads) race and
// corrupt each other's partial sums: serialise them.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "bn_b200.h"
#include "bn_kernels.cuh"

using namespace bn;

namespace {

constexpr uint32_t NOALLOC_CHUNKS = 16;
constexpr uint32_t NOALLOC_TRIALS = BN_NOALLOC_MAX_TRIALS;

// Layout: z partials | u.r partials | rejection flags | segment descriptor.
constexpr size_t Z_WORDS = (size_t)NOALLOC_CHUNKS * NOALLOC_TRIALS * N;
constexpr size_t UR_WORDS = (size_t)NOALLOC_CHUNKS * NOALLOC_TRIALS;
constexpr size_t FLAGS_OFF = (Z_WORDS + UR_WORDS) * 8;
constexpr size_t VSEG_OFF = FLAGS_OFF + 256;
constexpr size_t SCRATCH_BYTES = VSEG_OFF + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

// Clears what must start at zero and writes this call's segment descriptor;
// `plant` sets the draw flag (bn_debug_plant_draw_hit).
__global__ void noalloc_init_kernel(uint32_t rows, uint32_t plant) {
    uint32_t* flags = reinterpret_cast<uint32_t*>(g_noalloc_scratch + FLAGS_OFF);
    VerifySeg* vseg = reinterpret_cast<VerifySeg*>(g_noalloc_scratch + VSEG_OFF);
    *flags = plant ? DRAW_HIT_P : 0u;
    *vseg = VerifySeg{0, 0, rows, 0};
}

// A draw equalled p: the verdict may differ from the reference's, so it is
// replaced by -2 (nothing is read back to the host to report BN_EDRAW).
__global__ void noalloc_flag_kernel(int32_t* failed) {
    if (*reinterpret_cast<const uint32_t*>(g_noalloc_scratch + FLAGS_OFF) & DRAW_HIT_P) *failed = -2;
}

// Empty corpus: every trial compares two empty sums (bn_flat_verify's result).
__global__ void noalloc_empty_kernel(uint32_t trials, int32_t* failed, uint64_t* ur, uint64_t* zv) {
    for (uint32_t t = threadIdx.x; t < trials; t += blockDim.x) ur[t] = zv[t] = 0;
    if (threadIdx.x == 0) *failed = -1;
}

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void* g_scratch_ptr[MAX_DEVICES] = {nullptr};

thread_local char g_msg[512];

}  // namespace

// Defined in bn_capi.cu: records a message for bn_last_error().
extern "C" int bn_internal_set_error(int code, const char* msg);
// Defined in bn_capi.cu: the device, device-resident m_enc, rows, SM count
// and debug flags of a flat handle.
extern "C" int bn_internal_flat_view(const bn_flat* h, int* device, const uint64_t** d_m_enc, uint64_t* rows,
                                     int* num_sms, int* debug_draw_hit);

// Per device, once, with that device current (bn_ctx_create): the array's
// device address and the load of every kernel bn_flat_verify_noalloc
// launches.  Idempotent.
extern "C" int bn_internal_noalloc_setup(int device) {
    if (device < 0 || device >= MAX_DEVICES) return bn_internal_set_error(BN_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> g(g_mu);
    if (g_scratch_ptr[device]) return BN_OK;
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
        snprintf(g_msg, sizeof g_msg, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return bn_internal_set_error(BN_ECUDA, g_msg);
    }
    cudaFuncAttributes a;
    const void* own[] = {reinterpret_cast<const void*>(noalloc_init_kernel),
                         reinterpret_cast<const void*>(noalloc_flag_kernel),
                         reinterpret_cast<const void*>(noalloc_empty_kernel)};
    for (const void* f : own)
        if ((e = cudaFuncGetAttributes(&a, f)) != cudaSuccess) break;
    if (e == cudaSuccess) e = preload_freivalds_kernels();
    if (e != cudaSuccess) {
        snprintf(g_msg, sizeof g_msg, "loading the allocation-free verifier's kernels: %s", cudaGetErrorString(e));
        return bn_internal_set_error(BN_ECUDA, g_msg);
    }
    g_scratch_ptr[device] = ptr;
    return BN_OK;
}

namespace {

// Restores the calling thread's current device on every return path.
struct DeviceGuard {
    int prev = -1;
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" int bn_flat_verify_noalloc(bn_flat* h, const uint64_t* d_r, const uint64_t* d_v_enc,
                                      const uint8_t* d_v_seed, uint32_t trials, int32_t* d_failed_trial,
                                      uint64_t* d_ur, uint64_t* d_zv, void* stream) {
    if (!h || !d_r || !d_v_enc || !d_v_seed || !d_failed_trial || !d_ur || !d_zv)
        return bn_internal_set_error(BN_EINVAL, "bn_flat_verify_noalloc: null argument");
    if (trials == 0 || trials > NOALLOC_TRIALS) {
        snprintf(g_msg, sizeof g_msg, "bn_flat_verify_noalloc: trials = %u is outside 1..=%u (static scratch limit)",
                 trials, NOALLOC_TRIALS);
        return bn_internal_set_error(BN_EINVAL, g_msg);
    }
    int device = 0, sms = 0, plant = 0;
    const uint64_t* m_enc = nullptr;
    uint64_t rows = 0;
    int rc = bn_internal_flat_view(h, &device, &m_enc, &rows, &sms, &plant);
    if (rc != BN_OK) return rc;
    if (rows > 0xffffffffull)
        return bn_internal_set_error(BN_EINVAL, "bn_flat_verify_noalloc: the corpus must have fewer than 2^32 rows");
    if (device < 0 || device >= MAX_DEVICES) return bn_internal_set_error(BN_EINVAL, "device index out of range");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> g(g_mu);
        base = g_scratch_ptr[device];
    }
    if (!base)  // bn_ctx_create sets the device up; a handle implies a context
        return bn_internal_set_error(BN_ECUDA, "bn_flat_verify_noalloc: the device was not set up by bn_ctx_create");

    DeviceGuard guard;
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != device) {
        guard.prev = prev;
        e = cudaSetDevice(device);
    }
    if (e != cudaSuccess) {
        snprintf(g_msg, sizeof g_msg, "cudaSetDevice: %s", cudaGetErrorString(e));
        return bn_internal_set_error(BN_ECUDA, g_msg);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (rows == 0) {
        noalloc_empty_kernel<<<1, 32, 0, s>>>(trials, d_failed_trial, d_ur, d_zv);
    } else {
        // Fit the rows into as many chunks (of 32-row multiples) as the
        // array holds partials for at this trial count: 16 at 24 trials, 19
        // at 20, 128 at 3 (more chunks, more CTAs in flight).
        const uint64_t max_chunks = (uint64_t)NOALLOC_CHUNKS * NOALLOC_TRIALS / trials;
        FreivaldsPlan plan = plan_freivalds(rows, 1, sms);
        if (plan.chunks > max_chunks) {
            uint64_t cr = (rows + max_chunks - 1) / max_chunks;
            cr = (cr + 31) / 32 * 32;
            plan.chunk_rows = (uint32_t)cr;
            plan.chunks = (uint32_t)((rows + cr - 1) / cr);
        }
        unsigned char* sb = static_cast<unsigned char*>(base);
        uint64_t* z_part = reinterpret_cast<uint64_t*>(sb);
        uint64_t* ur_part = z_part + Z_WORDS;
        uint32_t* flags = reinterpret_cast<uint32_t*>(sb + FLAGS_OFF);
        VerifySeg* vseg = reinterpret_cast<VerifySeg*>(sb + VSEG_OFF);
        // The array keeps the previous call's contents: reset the rejection
        // flag and write this call's segment descriptor on the stream.  The z
        // and u.r partials are fully overwritten by the kernels below.
        noalloc_init_kernel<<<1, 1, 0, s>>>((uint32_t)rows, plant ? 1u : 0u);
        launch_freivalds(m_enc, d_r, vseg, 1, reinterpret_cast<const ChaChaKey*>(d_v_seed), trials, plan, z_part,
                         ur_part, flags, s);
        launch_freivalds_finish(z_part, ur_part, d_v_enc, vseg, 1, trials, plan, d_ur, d_zv, d_failed_trial, s);
        noalloc_flag_kernel<<<1, 1, 0, s>>>(d_failed_trial);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_msg, sizeof g_msg, "bn_flat_verify_noalloc launch: %s", cudaGetErrorString(e));
        return bn_internal_set_error(BN_ECUDA, g_msg);
    }
    return BN_OK;
}
