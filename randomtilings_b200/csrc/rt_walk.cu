// rt_walk.cu -- the persistent walk kernel and its launcher.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "rt_internal.h"
#include "rt_models.cuh"

namespace rtb {

// Blocks until both neighbouring CTAs have completed `need` phases.  One
// thread polls (acquire loads at gpu scope); the others wait at the barrier.
// The wait is bounded: after a.timeout_ns of waiting, or when another CTA has
// already raised an error, every CTA returns early and the host reports
// RT_E_TIMEOUT.
__device__ __forceinline__ bool wait_neighbours(const WalkArgs& a, int cta, unsigned need) {
    __shared__ int s_abort;
    if (threadIdx.x == 0) {
        int abort_flag = 0;
        uint64_t t0 = 0;
        for (int side = 0; side < 2 && !abort_flag; ++side) {
            const int nb = side == 0 ? cta - 1 : cta + 1;
            if (nb < 0 || nb >= (int)gridDim.x) continue;
            unsigned spins = 0;
            while (ld_acquire(a.flags + nb) < need) {
                if ((++spins & 15u) == 0u) {
                    if (*(volatile int*)a.err) {
                        abort_flag = 1;
                        break;
                    }
                    const uint64_t now = global_ns();
                    if (t0 == 0) {
                        t0 = now;
                    } else if (now - t0 > a.timeout_ns) {
                        atomicOr(a.err, ERR_TIMEOUT);
                        abort_flag = 1;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        s_abort = abort_flag;
    }
    __syncthreads();
    return s_abort == 0;
}

__device__ __forceinline__ void publish(const WalkArgs& a, int cta, unsigned done) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release(a.flags + cta, done);
    }
}

template <class Model, int ITEMS, int BLOCK>
__global__ void __launch_bounds__(BLOCK) walk_kernel(const __grid_constant__ WalkArgs a) {
    const int cta = blockIdx.x;
    const int r0 = cta * a.rows_per_cta;
    const int r1 = min(a.rows, r0 + a.rows_per_cta);
    const int npos = max(0, r1 - r0) * a.cols;

    int pr[ITEMS], pc[ITEMS];
    uint32_t sid[ITEMS];
    TinyState st[ITEMS];
    TinyParams tp[ITEMS];
#pragma unroll
    for (int u = 0; u < ITEMS; ++u) {
        const int q = (int)threadIdx.x + u * BLOCK;
        pr[u] = q < npos ? r0 + q / a.cols : -1;
        pc[u] = q < npos ? q % a.cols : 0;
        sid[u] = pr[u] >= 0 ? Model::stream_id(a, pr[u], pc[u]) : 0u;
        if (a.params != nullptr && pr[u] >= 0) {
            const uint4 p = __ldg(a.params + sid[u]);
            tp[u] = TinyParams{p.x, p.y, p.z};
        } else {
            tp[u] = TinyParams{a.mat1, a.mat2, a.tmat};
        }
        st[u] = TinyState{0u, 0u, 0u, 0u};
    }

    int epoch = -1;
    for (int64_t ph = 0; ph < a.nphases; ++ph) {
        if (a.rng_kind == 0) {
            bool reseed = false;
            while (epoch + 1 < a.nepochs && ph == a.epoch_start[epoch + 1]) {
                ++epoch;
                reseed = true;
            }
            if (reseed) {
                const uint32_t seed = a.epoch_seed[epoch];
#pragma unroll
                for (int u = 0; u < ITEMS; ++u)
                    if (pr[u] >= 0) tiny_seed(st[u], tp[u], seed + sid[u]);
            }
        }
        if (ph > 0 && !wait_neighbours(a, cta, (unsigned)ph)) return;
        const uint32_t d = __ldg(a.phases + ph);
        const bool draws = (d & PH_DRAWS) != 0u;
#pragma unroll
        for (int u = 0; u < ITEMS; ++u) {
            if (pr[u] < 0) continue;
            uint32_t k = 0;
            if (draws) {
                k = a.rng_kind == 0 ? tiny_draw23(st[u], tp[u])
                                    : philox_first(sid[u], (uint32_t)ph, (uint32_t)((uint64_t)ph >> 32), a.chain,
                                                   a.key0, a.key1) >> 9;
            }
            Model::apply(a, d, pr[u], pc[u], k);
        }
        publish(a, cta, (unsigned)(ph + 1));
    }
}

// ---------------------------------------------------------------------------
// Launch planning: the smallest per-thread item count whose CTA count fits
// the cooperative co-residency limit.
// ---------------------------------------------------------------------------
constexpr int kBlock = 256;

using KernelFn = void (*)(WalkArgs);

template <class Model>
static KernelFn pick_kernel(int items) {
    switch (items) {
        case 1: return walk_kernel<Model, 1, kBlock>;
        case 2: return walk_kernel<Model, 2, kBlock>;
        case 4: return walk_kernel<Model, 4, kBlock>;
        default: return walk_kernel<Model, 8, kBlock>;
    }
}

static KernelFn kernel_for(int family, int items) {
    switch (family) {
        case FAM_DOMINO: return pick_kernel<DominoRule<false>>(items);
        case FAM_DOMINO_HB: return pick_kernel<DominoRule<true>>(items);
        case FAM_LOZENGE8: return pick_kernel<ThreeColour<int8_t, LozengeRule<int8_t, false>>>(items);
        case FAM_QLOZENGE32: return pick_kernel<ThreeColour<int32_t, LozengeRule<int32_t, true>>>(items);
        case FAM_RECTTRI: return pick_kernel<ThreeColour<int32_t, RectTriRule>>(items);
        default: return nullptr;
    }
}

rt_status plan_walk(int family, int device, int rows, int cols, WalkPlan* plan, std::string* err) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        *err = "cudaDeviceGetAttribute failed";
        return RT_E_CUDA;
    }
    static const int kItems[] = {1, 2, 4, 8};
    for (int items : kItems) {
        const int per_cta = kBlock * items;
        if (cols > per_cta) continue;
        const int rows_per_cta = std::max(1, per_cta / std::max(cols, 1));
        const int ctas = (rows + rows_per_cta - 1) / rows_per_cta;
        KernelFn fn = kernel_for(family, items);
        if (!fn) {
            *err = "unknown kernel family";
            return RT_E_INVAL;
        }
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, kBlock, 0) != cudaSuccess) {
            *err = "cudaOccupancyMaxActiveBlocksPerMultiprocessor failed";
            return RT_E_CUDA;
        }
        if (ctas <= per_sm * sms) {
            plan->items = items;
            plan->block = kBlock;
            plan->rows_per_cta = rows_per_cta;
            plan->ctas = std::max(ctas, 1);
            plan->fn = (const void*)fn;
            return RT_OK;
        }
    }
    *err = "lattice too large for the register-resident walk (" + std::to_string(rows) + " x " + std::to_string(cols) +
           " positions)";
    return RT_E_INVAL;
}

rt_status launch_walk(const WalkPlan& plan, WalkArgs& args, cudaStream_t stream, std::string* err) {
    args.rows_per_cta = plan.rows_per_cta;
    void* kargs[] = {&args};
    cudaError_t e = cudaLaunchCooperativeKernel(plan.fn, dim3(plan.ctas), dim3(plan.block), kargs, 0, stream);
    if (e != cudaSuccess) {
        *err = std::string("cooperative launch failed: ") + cudaGetErrorString(e);
        return RT_E_CUDA;
    }
    return RT_OK;
}

// ---------------------------------------------------------------------------
// Split / merge between the host tiling layout and the colour arrays.
// ---------------------------------------------------------------------------
template <class T>
__global__ void split_kernel(const int32_t* __restrict__ t, int n, int ncol, int kind, T* a0, T* a1, T* a2) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * n) return;
    const int i = (int)(idx / n), j = (int)(idx % n);
    const int w = n / ncol;
    int c, col;
    if (kind == 0) {  // domino: (i+j) even -> array 0
        c = (i + j) & 1;
        col = j / 2;
    } else if (kind == 1) {  // lozenge: ((j-i) mod 3)
        c = ((j - i) % 3 + 3) % 3;
        col = j / 3;
    } else {  // rect-triangle: ((i-j) mod 3)
        c = ((i - j) % 3 + 3) % 3;
        col = j / 3;
    }
    T* dst = c == 0 ? a0 : c == 1 ? a1 : a2;
    dst[(int64_t)i * w + col] = (T)t[idx];
}

template <class T>
__global__ void merge_kernel(int32_t* __restrict__ t, int n, int ncol, int kind, const T* a0, const T* a1,
                             const T* a2) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)n * n) return;
    const int i = (int)(idx / n), j = (int)(idx % n);
    const int w = n / ncol;
    int c, col;
    if (kind == 0) {
        c = (i + j) & 1;
        col = j / 2;
    } else if (kind == 1) {
        c = ((j - i) % 3 + 3) % 3;
        col = j / 3;
    } else {
        c = ((i - j) % 3 + 3) % 3;
        col = j / 3;
    }
    const T* src = c == 0 ? a0 : c == 1 ? a1 : a2;
    t[idx] = (int32_t)src[(int64_t)i * w + col];
}

rt_status launch_split(bool merge, int elem_bytes, int kind, int ncol, int n, int32_t* tiling, void* const* arr,
                       cudaStream_t stream, std::string* err) {
    const int64_t total = (int64_t)n * n;
    const int threads = 256;
    const unsigned blocks = (unsigned)((total + threads - 1) / threads);
    if (elem_bytes == 1) {
        int8_t* a[3] = {(int8_t*)arr[0], (int8_t*)arr[1], ncol > 2 ? (int8_t*)arr[2] : nullptr};
        if (merge)
            merge_kernel<int8_t><<<blocks, threads, 0, stream>>>(tiling, n, ncol, kind, a[0], a[1], a[2]);
        else
            split_kernel<int8_t><<<blocks, threads, 0, stream>>>(tiling, n, ncol, kind, a[0], a[1], a[2]);
    } else {
        int32_t* a[3] = {(int32_t*)arr[0], (int32_t*)arr[1], ncol > 2 ? (int32_t*)arr[2] : nullptr};
        if (merge)
            merge_kernel<int32_t><<<blocks, threads, 0, stream>>>(tiling, n, ncol, kind, a[0], a[1], a[2]);
        else
            split_kernel<int32_t><<<blocks, threads, 0, stream>>>(tiling, n, ncol, kind, a[0], a[1], a[2]);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        *err = std::string("split/merge launch failed: ") + cudaGetErrorString(e);
        return RT_E_CUDA;
    }
    return RT_OK;
}

}  // namespace rtb
