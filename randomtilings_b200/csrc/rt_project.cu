// rt_project.cu -- exact integer Lipschitz projection of a height surface
// (include/rt_b200_project.h) on the GPU.
//
// Step 2 is a monotone min-plus relaxation: every pass lowers each interior
// vertex to min(h(w), h(v) + c(v -> w)) over its in-domain neighbours v,
// in place.  Values only decrease and never drop below the largest
// constraint-satisfying function under the start, so any order of updates
// (a racing read sees an old or a new value, both upper bounds) converges to
// that same unique function; passes repeat until one changes nothing.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rt_b200_project.h"
#include "rt_internal.h"
#include "rt_guard.h"

using rtb::guarded;

namespace rtb {

__constant__ int c_dom_di[4] = {1, -1, 0, 0};
__constant__ int c_dom_dj[4] = {0, 0, 1, -1};
__constant__ int c_loz_di[6] = {0, -1, -1, 0, 1, 1};
__constant__ int c_loz_dj[6] = {1, 1, 0, -1, -1, 0};
__constant__ int c_loz_s[6] = {-1, 1, -1, 1, -1, 1};

// Orientation step s of the edge from vertex (i, j) in direction nb
// (dominoes: DominoTiler.cpp:221-231 checkerboard rule; lozenges: fixed per
// direction, LozengeTiler.h:12-16).
template <bool DOM>
__device__ __forceinline__ int edge_step(int i, int j, int nb) {
    if (DOM) return (nb > 1 ? 1 : -1) * (((i + j) & 1) == 0 ? 1 : -1);
    return c_loz_s[nb];
}

template <bool DOM>
__global__ void project_init(const uint8_t* __restrict__ kind, const int32_t* __restrict__ hmin,
                             const int32_t* __restrict__ hmax, const float* __restrict__ target, int32_t* h, int n) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (int64_t)n * n) return;
    const int k = kind[v];
    if (k == 0) {
        h[v] = INT_MAX;
        return;
    }
    const int32_t lo = hmin[v], hi = hmax[v];
    if (k == 2) {
        h[v] = lo;
        return;
    }
    const double M = DOM ? 4.0 : 3.0;
    const double q = floor(((double)target[v] - (double)lo) / M + 0.5);
    double g = (double)lo + M * q;
    g = g < (double)lo ? (double)lo : g > (double)hi ? (double)hi : g;
    h[v] = (int32_t)g;
}

template <bool DOM>
__global__ void project_relax(const uint8_t* __restrict__ kind, const uint8_t* __restrict__ edges, int32_t* h, int n,
                              unsigned long long* changed) {
    constexpr int NB = DOM ? 4 : 6;
    constexpr int M1 = DOM ? 3 : 2;  // M - 1
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (int64_t)n * n || kind[v] != 1) return;
    const int i = (int)(v / n), j = (int)(v % n);
    const uint32_t e = edges[v];
    int32_t best = *(volatile int32_t*)(h + v);
    const int32_t old = best;
#pragma unroll
    for (int nb = 0; nb < NB; ++nb) {
        if (!(e & (1u << nb))) continue;
        const int i2 = i + (DOM ? c_dom_di[nb] : c_loz_di[nb]), j2 = j + (DOM ? c_dom_dj[nb] : c_loz_dj[nb]);
        const int32_t hv = *(volatile int32_t*)(h + (int64_t)i2 * n + j2);
        // h(w) - h(v) <= 1 along s(v -> w) = +1, i.e. s(w -> v) = -1; <= M-1 otherwise.
        const int32_t cand = hv + (edge_step<DOM>(i, j, nb) == -1 ? 1 : M1);
        best = cand < best ? cand : best;
    }
    if (best < old) {
        h[v] = best;
        atomicAdd(changed, 1ull);
    }
}

__global__ void project_finish(const uint8_t* __restrict__ kind, const int32_t* __restrict__ hmin, int32_t* h, int n,
                               unsigned long long* raised) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (int64_t)n * n || kind[v] == 0) return;
    if (h[v] < hmin[v]) {
        h[v] = hmin[v];
        atomicAdd(raised, 1ull);
    }
}

}  // namespace rtb

using namespace rtb;

namespace {
struct DevMem {
    void* p = nullptr;
    ~DevMem() {
        if (p) cudaFree(p);
    }
    bool alloc(size_t b) { return cudaMalloc(&p, b) == cudaSuccess; }
};
}  // namespace

extern "C" rt_status rt_project_heights(int32_t model, const int32_t* d, int64_t dlen, const int32_t* hmin,
                                        const int32_t* hmax, const float* target, int32_t* out, int64_t hlen,
                                        int32_t device, rt_project_stats* stats) {
    return guarded([&]() -> rt_status {
        if ((model != RT_DOMINO && model != RT_LOZENGE) || !d || !hmin || !hmax || !target || !out) return RT_E_INVAL;
        int n = 0;
        std::vector<uint8_t> kind, edges;
        if (!lipschitz_graph(model, d, dlen, &n, &kind, &edges) || (int64_t)n * n != hlen) return RT_E_INVAL;
        for (int64_t v = 0; v < hlen; ++v)
            if (kind[v] && (hmin[v] == INT_MAX || hmax[v] == INT_MAX || hmin[v] > hmax[v] ||
                            ((int64_t)hmax[v] - hmin[v]) % (model == RT_DOMINO ? 4 : 3) != 0))
                return RT_E_INVAL;  // not a pair of height functions of this domain
        if (cudaSetDevice(device) != cudaSuccess) return RT_E_NODEVICE;
        const size_t N2 = (size_t)hlen;
        DevMem dk, de, dlo, dhi, dt, dh, dc;
        if (!dk.alloc(N2) || !de.alloc(N2) || !dlo.alloc(N2 * 4) || !dhi.alloc(N2 * 4) || !dt.alloc(N2 * 4) ||
            !dh.alloc(N2 * 4) || !dc.alloc(16))
            return RT_E_NOMEM;
        cudaStream_t s;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return RT_E_CUDA;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaMemcpyAsync(dk.p, kind.data(), N2, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(de.p, edges.data(), N2, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(dlo.p, hmin, N2 * 4, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(dhi.p, hmax, N2 * 4, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(dt.p, target, N2 * 4, cudaMemcpyHostToDevice, s);
        const int threads = 256;
        const unsigned blocks = (unsigned)((N2 + threads - 1) / threads);
        const bool dom = model == RT_DOMINO;
        auto* K = static_cast<const uint8_t*>(dk.p);
        auto* E = static_cast<const uint8_t*>(de.p);
        auto* H = static_cast<int32_t*>(dh.p);
        auto* C = static_cast<unsigned long long*>(dc.p);
        cudaEventRecord(e0, s);
        if (dom)
            project_init<true><<<blocks, threads, 0, s>>>(K, (const int32_t*)dlo.p, (const int32_t*)dhi.p,
                                                          (const float*)dt.p, H, n);
        else
            project_init<false><<<blocks, threads, 0, s>>>(K, (const int32_t*)dlo.p, (const int32_t*)dhi.p,
                                                           (const float*)dt.p, H, n);
        int64_t passes = 0, lowered = 0;
        unsigned long long cnt[2] = {0, 0};
        // Passes in chunks of 16 with one readback of the change counter per chunk;
        // every pass is a monotone step, so extra passes after convergence are no-ops.
        const int64_t cap = (int64_t)hlen + 32;  // Bellman-Ford bound: no more passes than vertices
        for (;;) {
            cudaMemsetAsync(C, 0, 8, s);
            for (int k = 0; k < 16; ++k) {
                if (dom)
                    project_relax<true><<<blocks, threads, 0, s>>>(K, E, H, n, C);
                else
                    project_relax<false><<<blocks, threads, 0, s>>>(K, E, H, n, C);
            }
            passes += 16;
            cudaError_t ce = cudaMemcpyAsync(cnt, C, 8, cudaMemcpyDeviceToHost, s);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
            if (ce != cudaSuccess) {
                cudaStreamDestroy(s);
                return RT_E_CUDA;
            }
            lowered += (int64_t)cnt[0];
            if (cnt[0] == 0 || passes > cap) break;
        }
        cudaMemsetAsync(C + 1, 0, 8, s);
        project_finish<<<blocks, threads, 0, s>>>(K, (const int32_t*)dlo.p, H, n, C + 1);
        cudaEventRecord(e1, s);
        cudaMemcpyAsync(out, H, N2 * 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&cnt[1], C + 1, 8, cudaMemcpyDeviceToHost, s);
        cudaError_t ce = cudaStreamSynchronize(s);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(s);
        if (ce != cudaSuccess) return RT_E_CUDA;
        if (stats) {
            stats->passes = passes;
            stats->lowered = lowered;
            stats->raised = (int64_t)cnt[1];
            stats->device_ms = ms;
        }
        return RT_OK;
    });
}
