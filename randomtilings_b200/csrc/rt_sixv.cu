// rt_sixv.cu -- the six-vertex model (square ice) with domain-wall boundary
// conditions (include/rt_b200_sixv.h).
//
// The reference names the model (README.md:3) without code; this is the
// domino height machinery applied to it.  Heights live on the faces as int16.
// A colour step updates one of the four face classes (i mod 2, j mod 2); an
// epoch's steps run in one launch of the band kernel below when the bands
// fit shared memory, else one launch per step on the heights in HBM.  A
// thread owns four faces of its class in one row, (i, 8q + p + 2b) for
// b = 0..3, takes the four output words of one Philox4x32-10 call as their
// draws, and applies the heat bath: a face whose four edge neighbours share
// the height m becomes m+1 when its draw is below the threshold of its
// diagonal pattern, else m-1.  Faces of one class share no neighbour (edge
// or diagonal), so a launch is race-free and the result is independent of the
// order of the threads.  Coupled CFTP chains are two lattices of the same
// launch fed the same draws.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/rt_b200_sixv.h"
#include "rt_device.cuh"
#include "rt_internal.h"
#include "rt_guard.h"

using rtb::guarded;

namespace rtb {

struct SixvArgs {
    int16_t* h[2];  // heights of each lattice, (n+1) x (n+1), row stride n+1
    int nlat;
    int n;
    int pi, pj;     // class: row parity, column parity
    int rows, Q;    // rows of the class, quads per row
    uint32_t s_lo, s_hi, chain, k0, k1;
    uint32_t thr[16];
};

__global__ void __launch_bounds__(256) sixv_step_kernel(const __grid_constant__ SixvArgs a) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.rows * a.Q) return;
    const int r = idx / a.Q, q = idx - r * a.Q;
    const int i = (a.pi == 0 ? 2 : 1) + 2 * r;
    const int S = a.n + 1;
    const uint4 w4 = philox4((uint32_t)(i * a.Q + q), a.s_lo, a.s_hi, a.chain, a.k0, a.k1);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = 8 * q + a.pj + 2 * b;
        if (j < 1 || j > a.n - 1) continue;
        const uint32_t k = quad_word(w4, b) >> 9;
        for (int l = 0; l < a.nlat; ++l) {
            int16_t* f = a.h[l] + (size_t)i * S + j;
            const int m = f[-S];
            if (f[S] != m || f[-1] != m || f[1] != m) continue;
            const int p = (f[-S - 1] > m) | ((f[-S + 1] > m) << 1) | ((f[S - 1] > m) << 2) | ((f[S + 1] > m) << 3);
            *f = (int16_t)(k < a.thr[p] ? m + 1 : m - 1);
        }
    }
}

// ---------------------------------------------------------------------------
// The heights on chip for a whole epoch: CTA c owns face rows [r0, r1) of
// every lattice in shared memory (row stride sp = n + 1 rounded up to even,
// plus the rows r0 - 1 and r1 as halo).  Each colour step updates the band's
// faces of its class exactly as sixv_step_kernel does (same draws, same
// rule).  Steps 2t and 2t + 1 update rows of one parity, so the halo rows
// (the other parity) cannot change between them: after each odd step the
// band's first and last rows go to the neighbours through tagged 64-bit
// global slots (32 bits of heights and the step + 1), double-buffered by
// the parity of the exchange's number, and a CTA reads its halo rows before
// each even step.  A CTA publishes exchange t + 1 only after it read
// exchange t, which each neighbour published after reading exchange t - 1
// from it, so a slot is rewritten only after it was read.  Every wait is
// bounded: past timeout_ns the CTA sets ERR_TIMEOUT in *err and returns, and
// the others see it.  The launch is cooperative, so every CTA is resident.
// ---------------------------------------------------------------------------
struct SixvBandArgs {
    int16_t* h[2];
    int nlat, n, Q;
    uint32_t chain, k0, k1;
    uint32_t thr[16];
    int64_t steps;
    int rows_per_cta, sp, xwords;
    unsigned long long* xbuf;  // [cta][side][parity][lattice][xwords]
    int* err;
    uint64_t timeout_ns;
};

__device__ __forceinline__ unsigned long long* sixv_slot(const SixvBandArgs& a, int cta, int side, int par, int l) {
    return a.xbuf + ((((size_t)cta * 2 + side) * 2 + par) * a.nlat + l) * a.xwords;
}

__device__ __forceinline__ bool sixv_wait(const SixvBandArgs& a, const unsigned long long* p, uint32_t tag,
                                          uint32_t* out) {
    unsigned spins = 0;
    uint64_t t0 = 0;
    for (;;) {
        unsigned long long x;
        asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(x) : "l"(p) : "memory");
        if ((uint32_t)(x >> 32) == tag) {
            *out = (uint32_t)x;
            return true;
        }
        if ((++spins & 63u) == 0u) {
            if (*(volatile int*)a.err) return false;
            const uint64_t now = global_ns();
            if (t0 == 0) {
                t0 = now;
            } else if (now - t0 > a.timeout_ns) {
                atomicOr(a.err, ERR_TIMEOUT);
                return false;
            }
        }
    }
}

template <int NLAT>
__global__ void __launch_bounds__(1024, 1) sixv_band_kernel(const __grid_constant__ SixvBandArgs a) {
    extern __shared__ __align__(16) int16_t sh[];
    const int S = a.n + 1, sp = a.sp, X = a.xwords;
    const int cta = blockIdx.x, nct = gridDim.x, tid = threadIdx.x, BLOCK = blockDim.x;
    const int r0 = min(S, cta * a.rows_per_cta), r1 = min(S, r0 + a.rows_per_cta), nrows = r1 - r0;
    const int plane = (a.rows_per_cta + 2) * sp;  // per lattice; band row i sits at row i - r0 + 1
    for (int l = 0; l < NLAT; ++l)
        for (int e = tid; e < (nrows + 2) * sp; e += BLOCK) {
            const int rr = r0 - 1 + e / sp, j = e % sp;
            sh[l * plane + e] = rr >= 0 && rr < S && j < S ? a.h[l][(size_t)rr * S + j] : (int16_t)0;
        }
    __syncthreads();
    for (int64_t s = 0; s < a.steps; ++s) {
        if (s > 0 && (s & 1) == 0) {
            // halo rows: the neighbours' edge rows after step s - 1 (exchange s / 2)
            bool ok = true;
            const int par = (int)((s >> 1) & 1);
            const uint32_t tag = (uint32_t)s;
            for (int e = tid; e < 2 * NLAT * X && ok; e += BLOCK) {
                const int side = e >= NLAT * X, rem = e - side * NLAT * X, l = rem / X, w = rem - l * X;
                const int from = side == 0 ? cta - 1 : cta + 1;
                if (from < 0 || from >= nct || nrows <= 0) continue;
                uint32_t v;
                ok = sixv_wait(a, sixv_slot(a, from, 1 - side, par, l) + w, tag, &v);
                if (ok)
                    reinterpret_cast<uint32_t*>(sh + l * plane + (side == 0 ? 0 : nrows + 1) * sp)[w] = v;
            }
            if (__syncthreads_or(!ok)) return;
        }
        // this step's class: row parity (s mod 4) / 2, column parity s mod 2
        const int pi = (int)((s & 3) >> 1), pj = (int)(s & 1);
        const int par_row = pi == 0 ? 0 : 1;  // rows 2, 4, .. or 1, 3, .. up to n - 1
        const int lo = max(r0, 1), hi = min(r1, a.n);
        const int first = lo + ((lo & 1) != par_row);
        const int nlive = first < hi ? (hi - first + 1) / 2 : 0;
        const uint32_t s_lo = (uint32_t)s, s_hi = (uint32_t)((uint64_t)s >> 32);
        for (int u = tid; u < nlive * a.Q; u += BLOCK) {
            const int rr = u / a.Q, q = u - rr * a.Q;
            const int i = first + 2 * rr;
            const uint4 w4 = philox4((uint32_t)(i * a.Q + q), s_lo, s_hi, a.chain, a.k0, a.k1);
            const int j0 = 8 * q + pj;  // the faces j0, j0 + 2, j0 + 4, j0 + 6
            // Columns j0 - 1 .. j0 + 7 clamped to the row: a clamped column
            // serves only faces outside 1 .. n - 1, which are skipped.  All
            // reads come before the writes (no face of the class is another's
            // neighbour), so they need not wait on them.
            int col[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) col[t] = min(max(j0 - 1 + t, 0), sp - 1);
#pragma unroll
            for (int l = 0; l < NLAT; ++l) {
                int16_t* row = sh + l * plane + (i - r0 + 1) * sp;
                int up[9], dn[9], md[5];
#pragma unroll
                for (int t = 0; t < 9; ++t) {
                    up[t] = row[col[t] - sp];
                    dn[t] = row[col[t] + sp];
                }
#pragma unroll
                for (int t = 0; t < 5; ++t) md[t] = row[col[2 * t]];
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int j = j0 + 2 * b, m = up[2 * b + 1];
                    if (j < 1 || j > a.n - 1 || dn[2 * b + 1] != m || md[b] != m || md[b + 1] != m) continue;
                    const int p = (up[2 * b] > m) | ((up[2 * b + 2] > m) << 1) | ((dn[2 * b] > m) << 2) |
                                  ((dn[2 * b + 2] > m) << 3);
                    const uint32_t k = quad_word(w4, b) >> 9;
                    row[j] = (int16_t)(k < a.thr[p] ? m + 1 : m - 1);
                }
            }
        }
        __syncthreads();
        if ((s & 1) && s + 1 < a.steps && nrows > 0) {
            // the band's first and last rows, for the neighbours' next two steps
            const int par = (int)(((s + 1) >> 1) & 1);
            const unsigned long long tag = (unsigned long long)(uint32_t)(s + 1) << 32;
            for (int e = tid; e < 2 * NLAT * X; e += BLOCK) {
                const int side = e >= NLAT * X, rem = e - side * NLAT * X, l = rem / X, w = rem - l * X;
                const int to = side == 0 ? cta - 1 : cta + 1;
                if (to < 0 || to >= nct) continue;
                const uint32_t v =
                    reinterpret_cast<const uint32_t*>(sh + l * plane + (side == 0 ? 1 : nrows) * sp)[w];
                unsigned long long* dst = sixv_slot(a, cta, side, par, l) + w;
                asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(dst), "l"(tag | v) : "memory");
            }
        }
    }
    __syncthreads();
    for (int l = 0; l < NLAT; ++l)
        for (int e = tid; e < nrows * S; e += BLOCK) {
            const int rr = e / S, j = e - rr * S;
            a.h[l][(size_t)(r0 + rr) * S + j] = sh[l * plane + (rr + 1) * sp + j];
        }
}

__global__ void sixv_narrow_kernel(const int32_t* __restrict__ src, int16_t* __restrict__ dst, int64_t count) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) dst[k] = (int16_t)src[k];
}

__global__ void sixv_widen_kernel(const int16_t* __restrict__ src, int32_t* __restrict__ dst, int64_t count) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) dst[k] = src[k];
}

// Vertex type of faces NW a, NE b, SW c, SE d (the header's numbering), -1 if none.
static int vertex_type(int a, int b, int c, int d) {
    if (b == a + 1 && c == a - 1 && d == a) return 0;
    if (b == a - 1 && c == a + 1 && d == a) return 1;
    if (b == a + 1 && c == a + 1) return d == a + 2 ? 2 : d == a ? 4 : -1;
    if (b == a - 1 && c == a - 1) return d == a - 2 ? 3 : d == a ? 5 : -1;
    return -1;
}

// Heat-bath thresholds of the 16 diagonal patterns (heights relative to m).
static void sixv_thresholds(const double w[6], uint32_t thr[16], bool* monotone) {
    for (int p = 0; p < 16; ++p) {
        const int d1 = (p & 1) ? 1 : -1, d2 = (p & 2) ? 1 : -1, d3 = (p & 4) ? 1 : -1, d4 = (p & 8) ? 1 : -1;
        double wt[2];
        for (int up = 0; up < 2; ++up) {
            const int h = up ? 1 : -1;
            wt[up] = w[vertex_type(d1, 0, 0, h)] * w[vertex_type(0, d2, h, 0)] * w[vertex_type(0, h, d3, 0)] *
                     w[vertex_type(h, 0, 0, d4)];
        }
        thr[p] = below_threshold(wt[1] / (wt[0] + wt[1]));
    }
    bool mono = true;
    for (int p = 0; p < 16; ++p)
        for (int b = 0; b < 4; ++b)
            if (!(p & (1 << b)) && thr[p | (1 << b)] < thr[p]) mono = false;
    *monotone = mono;
}

}  // namespace rtb

using namespace rtb;

struct rt_sixv {
    int device = 0;
    cudaStream_t stream = nullptr;
    double w[6] = {1, 1, 1, 1, 1, 1};
    uint32_t thr[16] = {};
    bool monotone = true;
    std::string err;
    void* d_h[2] = {nullptr, nullptr};  // int16 lattices
    size_t cap = 0;                     // bytes of each
    int32_t* d_wide = nullptr;          // int32 staging
    size_t wide_cap = 0;
    unsigned long long* d_count = nullptr;
    unsigned long long* d_xbuf = nullptr;  // band kernel: halo slots
    size_t xcap = 0;
    int* d_err = nullptr;                  // band kernel: error word

    rt_status fail(rt_status s, const std::string& m) {
        err = m;
        return s;
    }
    rt_status cuda_fail(cudaError_t e, const char* what) {
        return fail(RT_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
    bool reserve(int n) {
        const size_t bytes = (((size_t)(n + 1) * (n + 1) * 2) + 255) & ~(size_t)255;
        const size_t wide = (size_t)(n + 1) * (n + 1) * 4;
        if (bytes > cap) {
            for (auto& p : d_h) {
                if (p) cudaFree(p);
                p = nullptr;
            }
            cap = 0;
            if (cudaMalloc(&d_h[0], bytes) != cudaSuccess || cudaMalloc(&d_h[1], bytes) != cudaSuccess) return false;
            cap = bytes;
        }
        if (wide > wide_cap) {
            if (d_wide) cudaFree(d_wide);
            d_wide = nullptr;
            wide_cap = 0;
            if (cudaMalloc(&d_wide, wide) != cudaSuccess) return false;
            wide_cap = wide;
        }
        if (!d_count && cudaMalloc(&d_count, sizeof *d_count) != cudaSuccess) return false;
        return true;
    }
    ~rt_sixv() {
        for (auto& p : d_h)
            if (p) cudaFree(p);
        if (d_wide) cudaFree(d_wide);
        if (d_count) cudaFree(d_count);
        if (d_xbuf) cudaFree(d_xbuf);
        if (d_err) cudaFree(d_err);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Host heights -> int16 lattice l (its padding zeroed, so that lattices
// compare word by word).
rt_status upload(rt_sixv* h, const int32_t* heights, int n, int l) {
    const int64_t count = (int64_t)(n + 1) * (n + 1);
    cudaError_t e = cudaMemsetAsync(h->d_h[l], 0, h->cap, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->d_wide, heights, (size_t)count * 4, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) {
        sixv_narrow_kernel<<<(unsigned)((count + 255) / 256), 256, 0, h->stream>>>(
            h->d_wide, static_cast<int16_t*>(h->d_h[l]), count);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? RT_OK : h->cuda_fail(e, "upload");
}

rt_status download(rt_sixv* h, int32_t* heights, int n, int l) {
    const int64_t count = (int64_t)(n + 1) * (n + 1);
    sixv_widen_kernel<<<(unsigned)((count + 255) / 256), 256, 0, h->stream>>>(static_cast<const int16_t*>(h->d_h[l]),
                                                                            h->d_wide, count);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(heights, h->d_wide, (size_t)count * 4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? RT_OK : h->cuda_fail(e, "download");
}

// Colour steps 0 .. 4 sweeps - 1 of one epoch on `nlat` lattices.
rt_status run_epoch(rt_sixv* h, int n, int nlat, int64_t sweeps, uint64_t key, uint32_t chain) {
    SixvArgs a;
    std::memset(&a, 0, sizeof a);
    a.h[0] = static_cast<int16_t*>(h->d_h[0]);
    a.h[1] = static_cast<int16_t*>(h->d_h[1]);
    a.nlat = nlat;
    a.n = n;
    a.Q = (n + 1 + 7) / 8;
    a.chain = chain;
    a.k0 = (uint32_t)key;
    a.k1 = (uint32_t)(key >> 32);
    std::memcpy(a.thr, h->thr, sizeof a.thr);
    if (sweeps <= 0) return RT_OK;
    {
        // The band kernel, when every CTA's rows (and halo) fit shared memory.
        int dev = 0, sms = 0, optin = 0;
        const int S = n + 1, sp = (S + 1) & ~1;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && sms > 0) {
            int ctas = std::min(sms, S);
            const int rpc = (S + ctas - 1) / ctas;
            ctas = (S + rpc - 1) / rpc;
            const size_t smem = (size_t)nlat * (rpc + 2) * sp * sizeof(int16_t);
            const size_t xbytes = (size_t)ctas * 2 * 2 * nlat * (sp / 2) * sizeof(unsigned long long);
            const void* band_fn = nlat == 2 ? (const void*)sixv_band_kernel<2> : (const void*)sixv_band_kernel<1>;
            bool ready = smem <= (size_t)optin &&
                         cudaFuncSetAttribute(band_fn,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess;
            if (ready && xbytes > h->xcap) {
                if (h->d_xbuf) cudaFree(h->d_xbuf);
                h->d_xbuf = nullptr;
                h->xcap = 0;
                ready = cudaMalloc(&h->d_xbuf, xbytes) == cudaSuccess;
                if (ready) h->xcap = xbytes;
            }
            if (ready && !h->d_err) ready = cudaMalloc(&h->d_err, sizeof(int)) == cudaSuccess;
            if (ready) {
                SixvBandArgs b;
                std::memset(&b, 0, sizeof b);
                b.h[0] = a.h[0];
                b.h[1] = a.h[1];
                b.nlat = nlat;
                b.n = n;
                b.Q = a.Q;
                b.chain = a.chain;
                b.k0 = a.k0;
                b.k1 = a.k1;
                std::memcpy(b.thr, a.thr, sizeof b.thr);
                b.steps = 4 * sweeps;
                b.rows_per_cta = rpc;
                b.sp = sp;
                b.xwords = sp / 2;
                b.xbuf = h->d_xbuf;
                b.err = h->d_err;
                b.timeout_ns = 5000000000ull;
                void* args[] = {&b};
                cudaError_t e = cudaMemsetAsync(h->d_xbuf, 0, xbytes, h->stream);
                if (e == cudaSuccess) e = cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream);
                if (e == cudaSuccess)
                    e = cudaLaunchCooperativeKernel(band_fn, dim3((unsigned)ctas), dim3(1024),
                                                    args, smem, h->stream);
                if (e == cudaSuccess) {
                    int flag = 0;
                    e = cudaMemcpyAsync(&flag, h->d_err, sizeof flag, cudaMemcpyDeviceToHost, h->stream);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
                    if (e != cudaSuccess) return h->cuda_fail(e, "six-vertex band walk");
                    if (flag) return h->fail(RT_E_TIMEOUT, "six-vertex band walk: a halo wait timed out");
                    return RT_OK;
                }
                cudaGetLastError();  // not launched: one launch per colour step below
            }
        }
    }
    for (int64_t s = 0; s < 4 * sweeps; ++s) {
        a.pi = (int)((s & 3) >> 1);
        a.pj = (int)(s & 1);
        // rows i = 2, 4, .. or 1, 3, .. up to n - 1
        const int first = a.pi == 0 ? 2 : 1;
        a.rows = n - 1 >= first ? (n - 1 - first) / 2 + 1 : 0;
        if (a.rows <= 0) continue;
        a.s_lo = (uint32_t)s;
        a.s_hi = (uint32_t)((uint64_t)s >> 32);
        const int64_t threads = (int64_t)a.rows * a.Q;
        sixv_step_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, h->stream>>>(a);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RT_OK : h->cuda_fail(e, "six-vertex step launch");
}

bool valid_n(int n) { return n >= 1 && n <= 32000; }

}  // namespace

extern "C" {

rt_status rt_sixv_create(int32_t device, rt_sixv** out) {
    return guarded([&]() -> rt_status {
        if (!out) return RT_E_INVAL;
        *out = nullptr;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return RT_E_NODEVICE;
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return RT_E_NODEVICE;
        cudaSetDevice(device);
        rt_sixv* h = new rt_sixv();
        h->device = device;
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete h;
            return RT_E_CUDA;
        }
        sixv_thresholds(h->w, h->thr, &h->monotone);
        *out = h;
        return RT_OK;
    });
}

rt_status rt_sixv_destroy(rt_sixv* h) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        cudaSetDevice(h->device);
        cudaStreamSynchronize(h->stream);
        delete h;
        return RT_OK;
    });
}

const char* rt_sixv_last_error(rt_sixv* h) { return h ? h->err.c_str() : ""; }

rt_status rt_sixv_set_weights(rt_sixv* h, const double w[6]) {
    return guarded([&]() -> rt_status {
        if (!h || !w) return RT_E_INVAL;
        for (int t = 0; t < 6; ++t)
            if (!(w[t] > 0) || !std::isfinite(w[t])) return h->fail(RT_E_INVAL, "vertex weights must be finite and > 0");
        std::memcpy(h->w, w, sizeof h->w);
        sixv_thresholds(h->w, h->thr, &h->monotone);
        return RT_OK;
    });
}

rt_status rt_sixv_thresholds(rt_sixv* h, uint32_t thr[16], int32_t* monotone) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        if (thr) std::memcpy(thr, h->thr, sizeof h->thr);
        if (monotone) *monotone = h->monotone ? 1 : 0;
        return RT_OK;
    });
}

rt_status rt_sixv_dwbc_heights(int32_t n, int32_t* hmin, int32_t* hmax) {
    return guarded([&]() -> rt_status {
        if (!valid_n(n)) return RT_E_INVAL;
        for (int i = 0; i <= n; ++i)
            for (int j = 0; j <= n; ++j) {
                const size_t at = (size_t)i * (n + 1) + j;
                if (hmin) hmin[at] = std::abs(i - j);
                if (hmax) hmax[at] = std::min(i + j, 2 * n - i - j);
            }
        return RT_OK;
    });
}

rt_status rt_sixv_check(const int32_t* heights, int32_t n) {
    return guarded([&]() -> rt_status {
        if (!heights || !valid_n(n)) return RT_E_INVAL;
        const int S = n + 1;
        auto H = [&](int i, int j) { return heights[(size_t)i * S + j]; };
        for (int k = 0; k <= n; ++k)
            if (H(0, k) != k || H(k, 0) != k || H(n, k) != n - k || H(k, n) != n - k) return RT_E_INVAL;
        // Every edge joins heights that differ by exactly 1: a row at a time,
        // branch-free.  Differences are taken modulo 2^32 (defined for any
        // input; d is +-1 iff d + 1 is 0 or 2).  That accepts exactly what
        // the exact test accepts: every face is within n / 2 edges of the
        // boundary, whose heights are 0..n, so heights that pass every edge
        // stay within [-n, 2n] and no difference wraps.
        for (int i = 0; i <= n; ++i) {
            const uint32_t* r = reinterpret_cast<const uint32_t*>(heights) + (size_t)i * S;
            uint32_t bad = 0;
            for (int j = 0; j < n; ++j) bad |= (r[j + 1] - r[j] + 1u) & ~2u;
            if (i < n)
                for (int j = 0; j <= n; ++j) bad |= (r[j + S] - r[j] + 1u) & ~2u;
            if (bad) return RT_E_INVAL;
        }
        return RT_OK;
    });
}

rt_status rt_sixv_to_asm(const int32_t* heights, int32_t n, int32_t* asm_out) {
    return guarded([&]() -> rt_status {
        if (!asm_out || rt_sixv_check(heights, n) != RT_OK) return RT_E_INVAL;
        const int S = n + 1;
        for (int i = 1; i <= n; ++i)
            for (int j = 1; j <= n; ++j) {
                const int a = heights[(size_t)(i - 1) * S + j - 1], b = heights[(size_t)(i - 1) * S + j];
                const int c = heights[(size_t)i * S + j - 1], d = heights[(size_t)i * S + j];
                asm_out[(size_t)(i - 1) * n + (j - 1)] = (b + c - a - d) / 2;
            }
        return RT_OK;
    });
}

rt_status rt_sixv_vertex_types(const int32_t* heights, int32_t n, int32_t* types) {
    return guarded([&]() -> rt_status {
        if (!types || rt_sixv_check(heights, n) != RT_OK) return RT_E_INVAL;
        const int S = n + 1;
        for (int i = 1; i <= n; ++i)
            for (int j = 1; j <= n; ++j)
                types[(size_t)(i - 1) * n + (j - 1)] =
                    vertex_type(heights[(size_t)(i - 1) * S + j - 1], heights[(size_t)(i - 1) * S + j],
                                heights[(size_t)i * S + j - 1], heights[(size_t)i * S + j]);
        return RT_OK;
    });
}

rt_status rt_sixv_walk(rt_sixv* h, int32_t* heights, int32_t n, int64_t sweeps, uint64_t key, uint32_t chain) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        if (!heights || !valid_n(n) || sweeps < 0) return h->fail(RT_E_INVAL, "bad arguments");
        if (sweeps > kMaxColourSteps / 4) return h->fail(RT_E_INVAL, "more than 2^38 sweeps in one call");
        if (rt_sixv_check(heights, n) != RT_OK)
            return h->fail(RT_E_INVAL, "not a domain-wall height function of this size");
        cudaSetDevice(h->device);
        if (!h->reserve(n)) return h->fail(RT_E_NOMEM, "cudaMalloc six-vertex lattice");
        rt_status s = upload(h, heights, n, 0);
        if (s == RT_OK) s = run_epoch(h, n, 1, sweeps, key, chain);
        if (s == RT_OK) s = download(h, heights, n, 0);
        return s;
    });
}

rt_status rt_sixv_cftp(rt_sixv* h, int32_t n, int64_t first_sweeps, int64_t master_seed, int32_t max_trials,
                       int32_t* out_heights, rt_cftp_stats* stats) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        if (!valid_n(n) || first_sweeps <= 0 || max_trials <= 0) return h->fail(RT_E_INVAL, "bad CFTP arguments");
        if (first_sweeps > kMaxColourSteps / 4) return h->fail(RT_E_INVAL, "more than 2^38 sweeps in one call");
        if (!h->monotone) return h->fail(RT_E_INVAL, "these weights give a heat bath that is not monotone: no CFTP");
        cudaSetDevice(h->device);
        if (!h->reserve(n)) return h->fail(RT_E_NOMEM, "cudaMalloc six-vertex lattices");
        std::vector<int32_t> hmin((size_t)(n + 1) * (n + 1)), hmax(hmin.size());
        rt_sixv_dwbc_heights(n, hmin.data(), hmax.data());
        std::mt19937 mt((std::mt19937::result_type)master_seed);
        std::vector<int64_t> sweeps{first_sweeps};
        std::vector<uint64_t> keys{(uint64_t)mt()};
        rt_cftp_stats st{};
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        rt_status s = RT_OK;
        double ms_total = 0;
        for (int trial = 0; trial < max_trials && s == RT_OK; ++trial) {
            s = upload(h, hmax.data(), n, 0);
            if (s == RT_OK) s = upload(h, hmin.data(), n, 1);
            if (s != RT_OK) break;
            cudaEventRecord(e0, h->stream);
            for (size_t e = 0; e < sweeps.size() && s == RT_OK; ++e) s = run_epoch(h, n, 2, sweeps[e], keys[e], 0);
            if (s != RT_OK) break;
            cudaEventRecord(e1, h->stream);
            s = launch_count_diff(h->d_h[0], h->d_h[1], h->cap, h->d_count, h->stream, &h->err);
            if (s != RT_OK) break;
            unsigned long long diff = 0;
            cudaError_t ce = cudaMemcpyAsync(&diff, h->d_count, sizeof diff, cudaMemcpyDeviceToHost, h->stream);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
            if (ce != cudaSuccess) {
                s = h->cuda_fail(ce, "coalescence readback");
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_total += ms;
            st.trials = trial + 1;
            int64_t total = 0;
            for (int64_t x : sweeps) total += x;
            st.total_steps = 4 * total;
            if (diff == 0) {
                st.coalesced = 1;
                break;
            }
            if (trial + 1 < max_trials && total > kMaxColourSteps / 8) {
                // the next trial would run 2 total sweeps
                s = h->fail(RT_E_INVAL, "CFTP schedule beyond 2^38 sweeps without coalescence");
                break;
            }
            sweeps.insert(sweeps.begin(), total);
            keys.insert(keys.begin(), (uint64_t)mt());
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        st.device_ms = ms_total;
        if (stats) *stats = st;
        if (s != RT_OK) return s;
        if (out_heights) return download(h, out_heights, n, 0);
        return RT_OK;
    });
}

}  // extern "C"
