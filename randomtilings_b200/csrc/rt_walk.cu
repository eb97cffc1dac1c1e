// rt_walk.cu -- the persistent walk kernel and its launcher.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "rt_internal.h"
#include "rt_models.cuh"
#include "rt_exchange.cuh"
#include "rt_tridimer.cuh"

namespace rtb {

// Shared memory of one CTA: in bit-exact mode the generator states of its
// positions (struct of arrays s0[], s1[], s2[], s3[], so consecutive threads
// hit consecutive banks; the fast mode keeps no state), then the lattice
// band(s): for each lattice, NCOL colour planes of (rows + 2 halo rows) x wpad
// elements.
template <class Model, int BLOCK, bool UNIFORM, bool PHILOX>
__global__ void __launch_bounds__(BLOCK, 1) walk_kernel(const __grid_constant__ WalkArgs a) {
    using T = typename Model::Elem;
    constexpr int NC = Model::NCOL;
    extern __shared__ __align__(16) unsigned char smem_raw[];

    const int cta = blockIdx.x;
    const int nct = gridDim.x;
    const int tid = threadIdx.x;
    const int r0 = cta * a.rows_per_cta;
    const int r1 = min(a.rows, r0 + a.rows_per_cta);
    const int a0 = r0 + Model::ROFF, a1 = r1 + Model::ROFF;  // owned colour-array rows
    const int hr = a1 - a0 + 2;                                // + one halo row each side
    const int W = a.wpad;
    const int plane = hr * W;
    const int cols = a.cols;
    const int npos = max(0, r1 - r0) * cols;
    const int spos = PHILOX ? 0 : a.rows_per_cta * cols;  // state slots (same for every CTA)

    uint32_t* s_st = reinterpret_cast<uint32_t*>(smem_raw);
    T* lat = reinterpret_cast<T*>(smem_raw + (size_t)4 * spos * sizeof(uint32_t));
    auto row_ptr = [&](int l, int c, int i) { return lat + ((size_t)l * NC + c) * plane + (size_t)(i - (a0 - 1)) * W; };

    // Band + halo rows from the global colour arrays.
    for (int l = 0; l < a.nlat; ++l)
        for (int c = 0; c < NC; ++c) {
            const T* g = static_cast<const T*>(a.arr[l][c]);
            T* s = lat + ((size_t)l * NC + c) * plane;
            for (int e = tid; e < plane; e += BLOCK) {
                const int rr = a0 - 1 + e / W, j = e % W;
                T v = (T)0;
                if (rr >= 0 && rr < a.arows && j < a.width) v = g[(size_t)rr * a.width + j];
                s[e] = v;
            }
        }

    const TinyParams up{a.mat1, a.mat2, a.tmat};
    auto params_of = [&](uint32_t sid) {
        if (UNIFORM) return up;
        const uint4 p = __ldg(a.params + sid);
        return TinyParams{p.x, p.y, p.z};
    };

    // Positions in the band's first (last) row read the halo row that the CTA
    // above (below) exchanges, so they are updated after the import ("edge"
    // positions, spread over all threads); all other positions are updated
    // before the wait, overlapping the neighbours' progress.
    const bool has_top = cta > 0, has_bot = cta + 1 < nct;
    const bool bot_edge = has_bot && !(has_top && r1 - r0 == 1);  // last row is an edge row of its own
    const int q_lo = has_top ? min(cols, npos) : 0;
    const int q_hi = has_bot ? max(q_lo, npos - cols) : npos;
    const int top_n = has_top ? min(cols, npos) : 0;
    const int bot_n = bot_edge ? cols : 0;
    const int n_edge = top_n + bot_n;
    // Interior positions of this thread: q = q_lo + tid + m * BLOCK, walked
    // with an incremental (row, column) instead of a division per site.
    const int dr = BLOCK / cols, dc = BLOCK % cols;
    const int q_first = q_lo + tid;
    const int r_first = r0 + q_first / cols, c_first = q_first % cols;
    // Fast mode walks quads instead -- the words of four consecutive sites of
    // a colour-array row, one Philox call each: quads qlo..qlo+G-1 of every
    // row cover the positions; interior rows ri_lo..ri_hi-1, the same edge
    // rows.
    const int Gw = (a.width + 3) >> 2;  // quads per colour-array row (counter)
    const int qlo = Model::COFF >> 2;
    const int G = ((Model::COFF + cols - 1) >> 2) - qlo + 1;
    const int ri_lo = r0 + (has_top ? 1 : 0);
    const int ri_hi = max(ri_lo, r1 - (has_bot ? 1 : 0));
    const int nq_in = (ri_hi - ri_lo) * G;
    const int nq_edge = ((has_top ? 1 : 0) + (bot_edge ? 1 : 0)) * G;
    const int dqr = BLOCK / G, dqc = BLOCK % G;

    int epoch = -1;
    int64_t next_epoch = a.nepochs > 0 ? a.epoch_start[0] : INT64_MAX;
    uint32_t key0 = 0, key1 = 0;  // fast mode: Philox key of the epoch
    int64_t dstep = 0;            // fast mode: drawing steps since the epoch started
    uint32_t d = a.nphases > 0 ? __ldg(a.phases) : 0u;
    uint32_t d_prev = 0u;

    __syncthreads();
    for (int64_t ph = 0; ph < a.nphases; ++ph) {
        const uint32_t d_next = ph + 1 < a.nphases ? __ldg(a.phases + ph + 1) : 0u;
        if (ph == next_epoch) {
            while (epoch + 1 < a.nepochs && a.epoch_start[epoch + 1] == ph) ++epoch;
            next_epoch = epoch + 1 < a.nepochs ? a.epoch_start[epoch + 1] : INT64_MAX;
            const uint64_t eseed = a.epoch_seed[epoch];
            if (PHILOX) {
                key0 = (uint32_t)eseed;
                key1 = (uint32_t)(eseed >> 32);
                dstep = 0;
            } else {
                const uint32_t seed = (uint32_t)eseed;
                for (int q = tid; q < npos; q += BLOCK) {
                    const uint32_t sid = Model::stream_id(a, r0 + q / cols, q % cols);
                    TinyState s;
                    tiny_seed(s, params_of(sid), seed + sid);
                    s_st[q] = s.s0;
                    s_st[spos + q] = s.s1;
                    s_st[2 * spos + q] = s.s2;
                    s_st[3 * spos + q] = s.s3;
                }
                __syncthreads();  // positions are drawn by other threads than the ones seeding them
            }
        }
        const bool draws = (d & PH_DRAWS) != 0u;
        const typename Model::Ctx x0 = Model::ctx(a, lat, plane, d, a0 - 1);
        const typename Model::Ctx x1 = Model::ctx(a, lat + (size_t)NC * plane, plane, d, a0 - 1);

        auto site_k = [&](int r, int c, uint32_t k) {
            const int i = r + Model::ROFF, j = c + Model::COFF;
            const int off = (r - r0 + 1) * W + j;
            Model::site(a, x0, off, i, j, k);
            if (a.nlat > 1) Model::site(a, x1, off, i, j, k);
        };
        // Bit-exact mode: one position, its TinyMT state in shared memory.
        auto site = [&](int q, int r, int c) {
            uint32_t k = 0;
            if (draws) {
                const uint32_t sid = UNIFORM ? 0u : Model::stream_id(a, r, c);
                TinyState s{s_st[q], s_st[spos + q], s_st[2 * spos + q], s_st[3 * spos + q]};
                k = tiny_draw23(s, params_of(sid));
                s_st[q] = s.s0;
                s_st[spos + q] = s.s1;
                s_st[2 * spos + q] = s.s2;
                s_st[3 * spos + q] = s.s3;
            }
            site_k(r, c, k);
        };
        // Fast mode: quad qlo + cq of position row r, one Philox call for the
        // (up to) four positions whose sites it holds.
        auto quad = [&](int r, int cq) {
            const int q = qlo + cq;
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (draws)
                w = philox4((uint32_t)((r + Model::ROFF) * Gw + q), (uint32_t)dstep, (uint32_t)((uint64_t)dstep >> 32),
                            a.chain, key0, key1);
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int c = 4 * q + b - Model::COFF;
                if (c >= 0 && c < cols) site_k(r, c, quad_word(w, b) >> 9);
            }
        };

        if (PHILOX) {
            int u = tid, r = ri_lo + tid / G, cq = tid % G;
            while (u < nq_in) {
                quad(r, cq);
                u += BLOCK;
                r += dqr;
                cq += dqc;
                if (cq >= G) {
                    cq -= G;
                    ++r;
                }
            }
        } else {
            int q = q_first, r = r_first, c = c_first;
            while (q < q_hi) {
                site(q, r, c);
                q += BLOCK;
                r += dr;
                c += dc;
                if (c >= cols) {
                    c -= cols;
                    ++r;
                }
            }
        }
        if (ph > 0) {
            // Halo rows of every array the neighbours wrote in the previous phase.
            const uint32_t mask = Model::written(d_prev);
            const int nx = __popc(mask);
            const int par = (int)((ph - 1) & 1);
            const uint32_t tag = (uint32_t)ph;
            bool ok = true;
            const int per_side = a.nlat * nx * a.xwords;
            for (int e = tid; e < 2 * per_side && ok; e += BLOCK) {
                const int side = e / per_side;  // 0: row above (from cta-1), 1: row below (from cta+1)
                const int rem = e % per_side;
                const int l = rem / (nx * a.xwords), kx = (rem / a.xwords) % nx, w = rem % a.xwords;
                const int src = side == 0 ? cta - 1 : cta + 1;
                if (src < 0 || src >= nct) continue;
                uint32_t v;
                ok = wait_word(a, slot(a, src, side == 0 ? 1 : 0, par, l, kx) + w, tag, &v);
                if (ok) unpack_word<T>(row_ptr(l, nth_bit(mask, kx), side == 0 ? a0 - 1 : a1), w, v);
            }
            if (__syncthreads_or(!ok)) return;
        }
        if (PHILOX) {
            for (int e = tid; e < nq_edge; e += BLOCK) {
                const bool top = has_top && e < G;
                quad(top ? r0 : r1 - 1, top ? e : e - (has_top ? G : 0));
            }
        } else {
            for (int e = tid; e < n_edge; e += BLOCK) {
                const bool top = e < top_n;
                const int c = top ? e : e - top_n;
                const int r = top ? r0 : r1 - 1;
                site((r - r0) * cols + c, r, c);
            }
        }
        __syncthreads();
        if (ph + 1 < a.nphases && !(cta == 0 && ph == a.drop_phase)) {
            // Publish the band's first / last row of every array written in this phase.
            const uint32_t mask = Model::written(d);
            const int nx = __popc(mask);
            const int par = (int)(ph & 1);
            const unsigned long long tag = (unsigned long long)(uint32_t)(ph + 1) << 32;
            const int per_side = a.nlat * nx * a.xwords;
            for (int e = tid; e < 2 * per_side; e += BLOCK) {
                const int side = e / per_side;  // 0: first row (read by cta-1), 1: last row (read by cta+1)
                const int rem = e % per_side;
                const int l = rem / (nx * a.xwords), kx = (rem / a.xwords) % nx, w = rem % a.xwords;
                const int dst = side == 0 ? cta - 1 : cta + 1;
                if (dst < 0 || dst >= nct) continue;
                const uint32_t v = pack_word<T>(row_ptr(l, nth_bit(mask, kx), side == 0 ? a0 : a1 - 1), w);
                st_relaxed64(slot(a, cta, side, par, l, kx) + w, tag | v);
            }
        }
        if (PHILOX && draws) ++dstep;
        d_prev = d;
        d = d_next;
    }

    // Owned rows back to the global colour arrays.
    __syncthreads();
    for (int l = 0; l < a.nlat; ++l)
        for (int c = 0; c < NC; ++c) {
            T* g = static_cast<T*>(a.arr[l][c]);
            for (int e = tid; e < (a1 - a0) * a.width; e += BLOCK) {
                const int rr = a0 + e / a.width, j = e % a.width;
                g[(size_t)rr * a.width + j] = row_ptr(l, c, rr)[j];
            }
        }
}

// ---------------------------------------------------------------------------
// Launch planning: the thinnest row bands whose CTAs are all co-resident
// (cooperative launch) with their states and lattice band in shared memory.
// ---------------------------------------------------------------------------
constexpr int kBlock = 1024;

using KernelFn = void (*)(WalkArgs);

template <class Model>
static KernelFn pick_kernel(bool uniform, bool philox) {
    if (philox) return walk_kernel<Model, kBlock, true, true>;
    return uniform ? walk_kernel<Model, kBlock, true, false> : walk_kernel<Model, kBlock, false, false>;
}

static KernelFn kernel_for(int family, bool uniform, bool philox) {
    switch (family) {
        case FAM_DOMINO: return pick_kernel<DominoRule<false>>(uniform, philox);
        case FAM_DOMINO_HB: return pick_kernel<DominoRule<true>>(uniform, philox);
        case FAM_LOZENGE8: return pick_kernel<ThreeColour<int8_t, LozengeRule<false>>>(uniform, philox);
        case FAM_QLOZENGE8: return pick_kernel<ThreeColour<int8_t, LozengeRule<true>>>(uniform, philox);
        case FAM_RECTTRI: return pick_kernel<ThreeColour<int32_t, RectTriRule>>(uniform, philox);
        case FAM_TRIDIMER: return pick_kernel<TriDimerRule>(uniform, philox);
        default: return nullptr;
    }
}

static int family_ncol(int family) { return family <= FAM_DOMINO_HB ? 2 : family == FAM_TRIDIMER ? 8 : 3; }
static int family_elem(int family) { return family <= FAM_QLOZENGE8 ? 1 : 4; }
static int family_xslots(int family) { return family == FAM_TRIDIMER ? 4 : 1; }

size_t walk_smem_bytes(int family, int nlat, int rows_per_cta, int cols, int width, bool philox) {
    const int wpad = (width + 3) & ~3;
    return (philox ? (size_t)0 : (size_t)4 * 4 * rows_per_cta * cols) +
           (size_t)nlat * family_ncol(family) * (rows_per_cta + 2) * wpad * family_elem(family);
}

rt_status plan_walk(int family, int device, int nlat, int rows, int cols, int width, bool uniform, bool philox,
                    WalkPlan* plan, std::string* err) {
    int sms = 0, smem_optin = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) {
        *err = "cudaDeviceGetAttribute failed";
        return RT_E_CUDA;
    }
    KernelFn fn = kernel_for(family, uniform, philox);
    if (!fn) {
        *err = "unknown kernel family";
        return RT_E_INVAL;
    }
    if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin) !=
        cudaSuccess) {
        *err = "cudaFuncSetAttribute failed";
        return RT_E_CUDA;
    }
    const int wpad = (width + 3) & ~3;
    for (int rpc = std::max(1, rows / (2 * sms)); rpc <= rows; ++rpc) {
        const size_t smem = walk_smem_bytes(family, nlat, rpc, cols, width, philox);
        if (smem > (size_t)smem_optin) break;
        const int ctas = (rows + rpc - 1) / rpc;
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, kBlock, smem) != cudaSuccess) {
            *err = "cudaOccupancyMaxActiveBlocksPerMultiprocessor failed";
            return RT_E_CUDA;
        }
        if (ctas <= per_sm * sms) {
            plan->items = (rpc * cols + kBlock - 1) / kBlock;
            plan->block = kBlock;
            plan->rows_per_cta = rpc;
            plan->ctas = std::max(ctas, 1);
            plan->smem = smem;
            plan->wpad = wpad;
            plan->xwords = family_elem(family) == 1 ? wpad / 4 : wpad;
            plan->xslots = family_xslots(family);
            plan->fn = (const void*)fn;
            return RT_OK;
        }
    }
    *err = "lattice too large for the shared-memory-resident walk (" + std::to_string(rows) + " x " +
           std::to_string(cols) + " positions)";
    return RT_E_INVAL;
}

rt_status launch_walk(const WalkPlan& plan, WalkArgs& args, cudaStream_t stream, std::string* err) {
    args.rows_per_cta = plan.rows_per_cta;
    args.wpad = plan.wpad;
    args.xwords = plan.xwords;
    args.xslots = plan.xslots;
    args.depth = plan.depth;
    args.pwords = plan.pwords;
    void* kargs[] = {&args};
    cudaError_t e = cudaLaunchCooperativeKernel(plan.fn, dim3(plan.ctas), dim3(plan.block), kargs, plan.smem, stream);
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
    if (kind == 3) {
        // Triangle dimers: only the lozenge states go back (TriangleDimerTiler.cpp:362-376);
        // (even, even) cells keep the caller's values.
        const int m = n / 2;
        const int64_t at = (int64_t)(i / 2) * m + j / 2;
        if (i % 2 == 0) {
            if (j % 2 == 1) t[idx] = (int32_t)a0[at];
        } else {
            t[idx] = (int32_t)(j % 2 == 0 ? a1[at] : a2[at]);
        }
        return;
    }
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

// Number of differing 32-bit words between two equally sized arrays (CFTP
// coalescence test of the coupled chains, done on the device so that only a
// counter crosses to the host).
__global__ void count_diff_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, size_t words,
                                  unsigned long long* count) {
    unsigned long long local = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x)
        local += __ldg(a + i) != __ldg(b + i);
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

rt_status launch_count_diff(const void* a, const void* b, size_t bytes, unsigned long long* d_count,
                            cudaStream_t stream, std::string* err) {
    const size_t words = bytes / 4;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((words + threads - 1) / threads, 148 * 8);
    cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof *d_count, stream);
    if (e == cudaSuccess && blocks > 0) {
        count_diff_kernel<<<blocks, threads, 0, stream>>>(static_cast<const uint32_t*>(a),
                                                          static_cast<const uint32_t*>(b), words, d_count);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        *err = std::string("coalescence check failed: ") + cudaGetErrorString(e);
        return RT_E_CUDA;
    }
    return RT_OK;
}

}  // namespace rtb
