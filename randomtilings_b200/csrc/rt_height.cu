// rt_height.cu -- height functions of device tilings (include/rt_b200_height.h).
//
// Three launches per call:
//   row_scan     one CTA per vertex row: the exclusive prefix sum P_i(j) of the
//                horizontal edge steps over the row's run [lo_i, hi_i];
//   row_offsets  one CTA: the offset R_i of every row, from the vertical edge
//                tying it to the row above (a prefix sum over rows), anchored
//                so that the first boundary vertex has height 0;
//   finish       h = P_i(j) + R_i at every domain vertex, written, added to a
//                running sum, or compared with a reference surface.
// Edge steps (host rules: rt_host.cpp, DominoTiler.cpp:221-231,
// LozengeTiler.cpp:12-16): an edge not crossed by a tile changes the height
// by its orientation step s, a crossed one by -3s (dominoes) or -2s
// (lozenges); the bit of the edge at its first vertex says which.
#include <cuda_runtime.h>

#include <climits>
#include <string>
#include <vector>

#include "../../include/rt_b200_height.h"
#include "rt_internal.h"
#include "rt_guard.h"

using rtb::guarded;

namespace rtb {

constexpr int kScanThreads = 256;

// Step of the horizontal edge (i, j) -> (i, j + 1) given the tiling value at (i, j).
template <bool DOM>
__device__ __forceinline__ int hstep(int i, int j, int32_t t) {
    if (DOM) {
        const int s = ((i + j) & 1) == 0 ? 1 : -1;  // direction j+1: +1 on even vertices
        return (t & 8) ? -3 * s : s;
    }
    return (t & 8) ? 2 : -1;  // direction (0, +1): s = -1
}

// Step of the vertical edge (i - 1, c) -> (i, c) given the tiling value at (i - 1, c).
template <bool DOM>
__device__ __forceinline__ int vstep(int i, int c, int32_t t) {
    if (DOM) {
        const int s = ((i - 1 + c) & 1) == 0 ? -1 : 1;  // direction i+1: -1 on even vertices
        return (t & 2) ? -3 * s : s;
    }
    return (t & 32) ? -2 : 1;  // direction (+1, 0): s = +1
}

// Block-wide exclusive scan of one int per thread (kScanThreads threads).
__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kScanThreads / 32) warp_tot[lane] = w;  // inclusive totals per warp
    }
    __syncthreads();
    const int before = warp > 0 ? warp_tot[warp - 1] : 0;
    const int r = before + x - v;
    __syncthreads();
    return r;
}

template <bool DOM>
__global__ void __launch_bounds__(kScanThreads) row_scan(const int32_t* __restrict__ t, int n,
                                                         const int* __restrict__ lo, const int* __restrict__ hi,
                                                         int32_t* __restrict__ out) {
    __shared__ int warp_tot[kScanThreads / 32];
    const int i = blockIdx.x;
    const int a = lo[i], b = hi[i];
    int32_t* row = out + (size_t)i * n;
    const int32_t* trow = t + (size_t)i * n;
    for (int j = threadIdx.x; j < n; j += kScanThreads)
        if (j < a || j > b) row[j] = INT_MAX;
    if (a > b) return;  // uniform per block: the barriers below are not reached by anyone
    const int len = b - a + 1;
    const int chunk = (len + kScanThreads - 1) / kScanThreads;
    const int j0 = a + threadIdx.x * chunk, j1 = min(b + 1, j0 + chunk);
    int sum = 0;
    for (int j = j0; j < j1 && j < b; ++j) sum += hstep<DOM>(i, j, trow[j]);
    int p = block_exclusive_scan(sum, warp_tot);
    for (int j = j0; j < j1; ++j) {
        row[j] = p;
        if (j < b) p += hstep<DOM>(i, j, trow[j]);
    }
}

// R[i] such that h(i, j) = P_i(j) + R[i]; rows without domain vertices get 0.
template <bool DOM>
__global__ void __launch_bounds__(1024) row_offsets(const int32_t* __restrict__ t, int n, const int* __restrict__ lo,
                                                    const int* __restrict__ hi, const int* __restrict__ conn,
                                                    const int32_t* __restrict__ P, int i0, int j0,
                                                    int32_t* __restrict__ R) {
    __shared__ int warp_tot[32];
    __shared__ int anchor;
    const int chunk = (n + blockDim.x - 1) / blockDim.x;
    const int r0 = threadIdx.x * chunk, r1 = min(n, r0 + chunk);
    auto delta = [&](int i) -> int {
        const int c = conn[i];
        if (c < 0) return 0;
        return P[(size_t)(i - 1) * n + c] + vstep<DOM>(i, c, t[(size_t)(i - 1) * n + c]) - P[(size_t)i * n + c];
    };
    int sum = 0;
    for (int i = r0; i < r1; ++i) sum += delta(i);
    // exclusive scan of the per-thread sums (1024 threads = 32 warps)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_tot[lane] = w;
    }
    __syncthreads();
    int s = (warp > 0 ? warp_tot[warp - 1] : 0) + x - sum;
    for (int i = r0; i < r1; ++i) {
        s += delta(i);
        R[i] = s;  // inclusive sum up to row i
        if (i == i0) anchor = s + P[(size_t)i0 * n + j0];
    }
    __syncthreads();
    for (int i = r0; i < r1; ++i) R[i] -= anchor;
}

enum FinishMode { FIN_WRITE = 0, FIN_SUM = 1, FIN_ERROR = 2 };

template <int MODE>
__global__ void finish(int n, const int* __restrict__ lo, const int* __restrict__ hi, const int32_t* __restrict__ R,
                       int32_t* P, int64_t* __restrict__ sum, const float* __restrict__ ref, double* err) {
    const int i = blockIdx.y;
    const int a = lo[i], b = hi[i];
    double acc = 0.0;
    const int32_t r = R[i];
    for (int j = a + blockIdx.x * blockDim.x + threadIdx.x; j <= b; j += gridDim.x * blockDim.x) {
        const size_t v = (size_t)i * n + j;
        const int32_t h = P[v] + r;
        if (MODE == FIN_WRITE) P[v] = h;
        if (MODE == FIN_SUM) sum[v] += h;
        if (MODE == FIN_ERROR) acc += fabs((double)h - (double)ref[v]);
    }
    if (MODE == FIN_ERROR) {
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(err, acc);
    }
}

}  // namespace rtb

using namespace rtb;

struct rt_hplan {
    int model = 0, device = 0, n = 0, i0 = 0, j0 = 0;
    int64_t vertices = 0;
    int* d_lo = nullptr;
    int* d_hi = nullptr;
    int* d_conn = nullptr;
    int32_t* d_R = nullptr;
    int32_t* d_P = nullptr;  // scratch heights for the sum / error forms
    double* d_err = nullptr;
    std::string err;
    rt_status fail(rt_status s, const std::string& m) {
        err = m;
        return s;
    }
};

namespace {

thread_local std::string g_hplan_create_error;

rt_status create_fail(rt_hplan* p, rt_status s, const std::string& m) {
    g_hplan_create_error = m;
    rt_hplan_destroy(p);
    return s;
}

// Launches the scan and the offsets; P receives the row prefix sums.
rt_status scan_rows(rt_hplan* p, const int32_t* t, int32_t* P, cudaStream_t s) {
    const int n = p->n;
    if (p->model == RT_DOMINO) {
        row_scan<true><<<n, kScanThreads, 0, s>>>(t, n, p->d_lo, p->d_hi, P);
        row_offsets<true><<<1, 1024, 0, s>>>(t, n, p->d_lo, p->d_hi, p->d_conn, P, p->i0, p->j0, p->d_R);
    } else {
        row_scan<false><<<n, kScanThreads, 0, s>>>(t, n, p->d_lo, p->d_hi, P);
        row_offsets<false><<<1, 1024, 0, s>>>(t, n, p->d_lo, p->d_hi, p->d_conn, P, p->i0, p->j0, p->d_R);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return p->fail(RT_E_CUDA, std::string("height scan launch: ") + cudaGetErrorString(e));
    return RT_OK;
}

dim3 finish_grid(int n) { return dim3((unsigned)std::max(1, std::min(16, (n + 255) / 256)), (unsigned)n); }

}  // namespace

extern "C" {

rt_status rt_hplan_create(int32_t model, const int32_t* d, int64_t dlen, int32_t device, rt_hplan** out) {
    return guarded([&]() -> rt_status {
        if (!out) return RT_E_INVAL;
        *out = nullptr;
        if (model != RT_DOMINO && model != RT_LOZENGE) {
            g_hplan_create_error = "height plans exist for dominoes and lozenges";
            return RT_E_INVAL;
        }
        int n = 0;
        std::vector<uint8_t> kind, edges;
        if (!lipschitz_graph(model, d, dlen, &n, &kind, &edges)) {
            g_hplan_create_error = "not a domain of this model";
            return RT_E_INVAL;
        }
        const int right = model == RT_DOMINO ? 2 : 0;  // direction (0, +1)
        const int down = model == RT_DOMINO ? 0 : 5;   // direction (+1, 0)
        std::vector<int> lo(n, n), hi(n, -1), conn(n, -1);
        int64_t verts = 0;
        int first = -1, last = -1, i0 = -1, j0 = -1;
        for (int i = 0; i < n; ++i) {
            for (int j = 0; j < n; ++j) {
                const int k = kind[(size_t)i * n + j];
                if (!k) continue;
                lo[i] = std::min(lo[i], j);
                hi[i] = std::max(hi[i], j);
                ++verts;
                if (k == 2 && i0 < 0) i0 = i, j0 = j;
            }
            if (hi[i] < 0) continue;
            for (int j = lo[i]; j < hi[i]; ++j)
                if (!kind[(size_t)i * n + j] || !(edges[(size_t)i * n + j] & (1u << right))) {
                    g_hplan_create_error = "vertex row " + std::to_string(i) + " is not one run of domain vertices";
                    return RT_E_INVAL;
                }
            if (first < 0) {
                first = i;
            } else {
                if (last != i - 1) {
                    g_hplan_create_error = "rows without domain vertices between domain rows";
                    return RT_E_INVAL;
                }
                for (int c = std::max(lo[i], lo[i - 1]); c <= std::min(hi[i], hi[i - 1]); ++c)
                    if (edges[(size_t)(i - 1) * n + c] & (1u << down)) {
                        conn[i] = c;
                        break;
                    }
                if (conn[i] < 0) {
                    g_hplan_create_error = "vertex rows " + std::to_string(i - 1) + " and " + std::to_string(i) +
                                           " share no in-domain edge";
                    return RT_E_INVAL;
                }
            }
            last = i;
        }
        if (i0 < 0) {
            g_hplan_create_error = "domain has no boundary vertex";
            return RT_E_INVAL;
        }
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
            g_hplan_create_error = "no CUDA device with that ordinal";
            return RT_E_NODEVICE;
        }
        cudaSetDevice(device);
        rt_hplan* p = new rt_hplan();
        p->model = model;
        p->device = device;
        p->n = n;
        p->i0 = i0;
        p->j0 = j0;
        p->vertices = verts;
        bool ok = cudaMalloc(&p->d_lo, n * sizeof(int)) == cudaSuccess &&
                  cudaMalloc(&p->d_hi, n * sizeof(int)) == cudaSuccess &&
                  cudaMalloc(&p->d_conn, n * sizeof(int)) == cudaSuccess &&
                  cudaMalloc(&p->d_R, n * sizeof(int32_t)) == cudaSuccess &&
                  cudaMalloc(&p->d_P, (size_t)n * n * sizeof(int32_t)) == cudaSuccess &&
                  cudaMalloc(&p->d_err, sizeof(double)) == cudaSuccess;
        if (!ok) return create_fail(p, RT_E_NOMEM, "height plan buffers");
        ok = cudaMemcpy(p->d_lo, lo.data(), n * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(p->d_hi, hi.data(), n * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(p->d_conn, conn.data(), n * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
        if (!ok) return create_fail(p, RT_E_CUDA, "height plan upload");
        *out = p;
        return RT_OK;
    });
}

rt_status rt_hplan_destroy(rt_hplan* p) {
    return guarded([&]() -> rt_status {
        if (!p) return RT_E_INVAL;
        cudaSetDevice(p->device);
        cudaFree(p->d_lo);
        cudaFree(p->d_hi);
        cudaFree(p->d_conn);
        cudaFree(p->d_R);
        cudaFree(p->d_P);
        cudaFree(p->d_err);
        delete p;
        return RT_OK;
    });
}

rt_status rt_hplan_info(rt_hplan* p, int32_t* n, int64_t* vertices) {
    return guarded([&]() -> rt_status {
        if (!p) return RT_E_INVAL;
        if (n) *n = p->n;
        if (vertices) *vertices = p->vertices;
        return RT_OK;
    });
}

const char* rt_hplan_last_error(rt_hplan* p) { return p ? p->err.c_str() : g_hplan_create_error.c_str(); }

rt_status rt_hplan_heights(rt_hplan* p, const int32_t* d_tiling, int32_t* d_heights, void* stream) {
    return guarded([&]() -> rt_status {
        if (!p || !d_tiling || !d_heights) return p ? p->fail(RT_E_INVAL, "null pointer") : RT_E_INVAL;
        cudaSetDevice(p->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        rt_status st = scan_rows(p, d_tiling, d_heights, s);
        if (st != RT_OK) return st;
        finish<FIN_WRITE><<<finish_grid(p->n), 256, 0, s>>>(p->n, p->d_lo, p->d_hi, p->d_R, d_heights, nullptr, nullptr,
                                                            nullptr);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? RT_OK : p->fail(RT_E_CUDA, std::string("height launch: ") + cudaGetErrorString(e));
    });
}

rt_status rt_hplan_accumulate(rt_hplan* p, const int32_t* d_tiling, int64_t* d_sum, void* stream) {
    return guarded([&]() -> rt_status {
        if (!p || !d_tiling || !d_sum) return p ? p->fail(RT_E_INVAL, "null pointer") : RT_E_INVAL;
        cudaSetDevice(p->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        rt_status st = scan_rows(p, d_tiling, p->d_P, s);
        if (st != RT_OK) return st;
        finish<FIN_SUM><<<finish_grid(p->n), 256, 0, s>>>(p->n, p->d_lo, p->d_hi, p->d_R, p->d_P, d_sum, nullptr, nullptr);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? RT_OK : p->fail(RT_E_CUDA, std::string("height launch: ") + cudaGetErrorString(e));
    });
}

rt_status rt_hplan_error(rt_hplan* p, const int32_t* d_tiling, const float* d_ref, double* mean_abs, void* stream) {
    return guarded([&]() -> rt_status {
        if (!p || !d_tiling || !d_ref || !mean_abs) return p ? p->fail(RT_E_INVAL, "null pointer") : RT_E_INVAL;
        cudaSetDevice(p->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        cudaError_t e = cudaMemsetAsync(p->d_err, 0, sizeof(double), s);
        if (e != cudaSuccess) return p->fail(RT_E_CUDA, std::string("memset: ") + cudaGetErrorString(e));
        rt_status st = scan_rows(p, d_tiling, p->d_P, s);
        if (st != RT_OK) return st;
        finish<FIN_ERROR><<<finish_grid(p->n), 256, 0, s>>>(p->n, p->d_lo, p->d_hi, p->d_R, p->d_P, nullptr, d_ref,
                                                            p->d_err);
        double sum = 0.0;
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&sum, p->d_err, sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return p->fail(RT_E_CUDA, std::string("height error: ") + cudaGetErrorString(e));
        *mean_abs = p->vertices > 0 ? sum / (double)p->vertices : 0.0;
        return RT_OK;
    });
}

}  // extern "C"
