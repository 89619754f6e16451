// bn_route.cu -- IVF routing on the device: the nprobe nearest centroids of
// every query of a batch (ivf-index/src/ivf.rs:150-164 probe_route).
//
// The distance is the reference's scalar l2_f32 (ivf-index/src/distance.rs:
// 30-36): sqrt of the sum over the dimensions, in order, of (x - y)^2, every
// operation rounded on its own (no fused multiply-add), so each distance is
// bit-identical to the host form (bn_host_probe_route, compiled without
// contraction).  Centroids are ranked by (distance, index): total_cmp order
// for the non-negative distances, ties to the lower index.  The reference's
// AVX-512 build sums in 16 lanes with fused multiply-adds instead and may
// rank near-ties differently; its scalar build agrees with this one.

#include "bn_internal.cuh"

namespace bn {
namespace {

constexpr uint32_t RT_THREADS = 256;
constexpr uint32_t RT_SORT_THREADS = 1024;

// dist[q][c] for centroid c = blockIdx.x * 256 + threadIdx.x; centroids are
// stored dimension-major (cent_t[i][c]) so a warp's loads are coalesced.
__global__ void __launch_bounds__(RT_THREADS)
route_dist_kernel(const float* __restrict__ cent_t, uint32_t nlist, uint32_t d, const float* __restrict__ queries,
                  float* __restrict__ dist) {
    extern __shared__ float qs[];
    const uint32_t q = blockIdx.y;
    for (uint32_t i = threadIdx.x; i < d; i += blockDim.x) qs[i] = queries[(uint64_t)q * d + i];
    __syncthreads();
    const uint32_t c = blockIdx.x * RT_THREADS + threadIdx.x;
    if (c >= nlist) return;
    float s = 0.0f;
    for (uint32_t i = 0; i < d; ++i) {
        const float t = __fsub_rn(qs[i], cent_t[(uint64_t)i * nlist + c]);
        s = __fadd_rn(s, __fmul_rn(t, t));
    }
    dist[(uint64_t)q * nlist + c] = __fsqrt_rn(s);
}

// One CTA per query: keys (distance bits << 32 | index) -- the bits of a
// non-negative float order like the float -- bitonic-sorted ascending in
// shared memory; the first np indices are the probes.
__global__ void __launch_bounds__(RT_SORT_THREADS)
route_select_kernel(const float* __restrict__ dist, uint32_t nlist, uint32_t np, uint32_t pow2,
                    uint32_t* __restrict__ probes) {
    extern __shared__ uint64_t keys[];
    const uint32_t q = blockIdx.x;
    for (uint32_t i = threadIdx.x; i < pow2; i += blockDim.x)
        keys[i] = i < nlist ? ((uint64_t)__float_as_uint(dist[(uint64_t)q * nlist + i]) << 32) | i : ~0ull;
    for (uint32_t size = 2; size <= pow2; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < pow2 / 2; i += blockDim.x) {
                const uint32_t lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                const bool up = (lo & size) == 0;
                const uint64_t a = keys[lo], b = keys[hi];
                if ((a > b) == up) {
                    keys[lo] = b;
                    keys[hi] = a;
                }
            }
        }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < np; i += blockDim.x) probes[(uint64_t)q * np + i] = (uint32_t)keys[i];
}

}  // namespace
}  // namespace bn

using namespace bn;
using namespace bn::api;

namespace {
constexpr uint32_t ROUTE_MAX_NLIST = 16384;  // the sort's keys fit in 128 KB of shared memory
constexpr uint32_t ROUTE_MAX_DIM = 8192;
}  // namespace

extern "C" {

int bn_ivf_set_centroids(bn_ivf* v, const float* centroids, uint32_t d) {
    if (!v || !centroids) return fail(BN_EINVAL, "null argument");
    if (d == 0 || d > ROUTE_MAX_DIM) return fail(BN_EINVAL, "centroid dimension %u not in 1..=%u", d, ROUTE_MAX_DIM);
    if (v->nlist > ROUTE_MAX_NLIST) return fail(BN_EINVAL, "%u lists exceed the %u the router ranks", v->nlist, ROUTE_MAX_NLIST);
    std::lock_guard<std::mutex> g(v->e.mu);
    CU(cudaSetDevice(v->e.ctx->device));
    std::vector<float> t((uint64_t)d * v->nlist);
    for (uint32_t c = 0; c < v->nlist; ++c)
        for (uint32_t i = 0; i < d; ++i) t[(uint64_t)i * v->nlist + c] = centroids[(uint64_t)c * d + i];
    TRY(v->cent_t.alloc(v->e.ctx, std::max<uint64_t>(t.size(), 1) * 4));
    CU(cudaMemcpy(v->cent_t.p, t.data(), t.size() * 4, cudaMemcpyHostToDevice));
    v->cent_d = d;
    return BN_OK;
}

int bn_ivf_route(bn_ivf* v, uint32_t B, const float* queries, uint32_t nprobe, uint32_t* probes) {
    if (!v) return fail(BN_EINVAL, "null handle");
    if (B == 0) return BN_OK;
    if (!queries || !probes) return fail(BN_EINVAL, "null argument");
    if (!v->cent_d) return fail(BN_EINVAL, "no centroids: call bn_ivf_set_centroids first");
    if (nprobe == 0) return fail(BN_EINVAL, "nprobe must be positive");
    if (B > 65535) return fail(BN_EINVAL, "B = %u exceeds 65535 queries per call", B);
    const uint32_t nlist = v->nlist, d = v->cent_d, np = std::min(nprobe, nlist);
    if (nlist == 0) return BN_OK;
    std::lock_guard<std::mutex> g(v->e.mu);
    CU(cudaSetDevice(v->e.ctx->device));
    Layout L;
    const uint64_t o_q = L.take<float>((uint64_t)B * d);
    const uint64_t o_d = L.take<float>((uint64_t)B * nlist);
    const uint64_t o_p = L.take<uint32_t>((uint64_t)B * np);
    TRY(v->e.ws.reserve(v->e.ctx, L.off));
    char* dv = v->e.ws.at<char>();
    cudaStream_t s = v->e.stream;
    CU(cudaMemcpyAsync(dv + o_q, queries, (uint64_t)B * d * 4, cudaMemcpyHostToDevice, s));
    route_dist_kernel<<<dim3((nlist + RT_THREADS - 1) / RT_THREADS, B), RT_THREADS, d * 4, s>>>(
        v->cent_t.at<float>(), nlist, d, reinterpret_cast<const float*>(dv + o_q), reinterpret_cast<float*>(dv + o_d));
    uint32_t pow2 = 1;
    while (pow2 < nlist) pow2 <<= 1;
    const int smem = (int)(pow2 * 8);
    CU(cudaFuncSetAttribute(route_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, ROUTE_MAX_NLIST * 8));
    route_select_kernel<<<B, RT_SORT_THREADS, smem, s>>>(reinterpret_cast<const float*>(dv + o_d), nlist, np, pow2,
                                                         reinterpret_cast<uint32_t*>(dv + o_p));
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(probes, dv + o_p, (uint64_t)B * np * 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return BN_OK;
}

}  // extern "C"
