// rt_word.cu -- the word-parallel walk kernel of the int8 models.
//
// Dominoes (dominokernel.cl, dominokernelCFTP.cl) and uniform lozenges
// (lozengekernel.cl) store one byte per site.  This kernel treats a 32-bit
// word of four consecutive sites of a colour-array row as its unit of work:
// the Update of a colour is a handful of masks and byte shifts on words of
// the flipped colour (neighbours at j +- 1 are funnel shifts of two adjacent
// words), the flip test is a per-byte compare, and each thread keeps the
// TinyMT states of the four positions of each of its words in registers for
// the whole walk (bit-exact mode) or draws them from one Philox call per word
// (fast mode).  Schedule, bands, tagged halo slots and bounded waits are
// those of the generic walk kernel (rt_walk.cu) and it produces the same
// bytes.  With one word per thread, the owners of the band's edge words poll
// their halo words themselves and only their warps meet at the halo barrier,
// so the interior words of the other warps overlap the exchange; a colour
// step then costs the longer of one interior word and (halo wait + one edge
// word) rather than their sum.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "rt_exchange.cuh"
#include "rt_internal.h"
#include "rt_models.cuh"
#include "rt_word.cuh"

namespace rtb {

constexpr int kWordBlockMax = 512;

// bar.red.or on named barrier `id`, which `n` threads (whole warps) execute;
// returns the OR of their `v`.
__device__ __forceinline__ bool bar_red_or_n(int id, int n, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(n)
        : "memory");
    return r != 0u;
}

// Shared memory: 16 bytes of slack, then for each lattice NC colour planes of
// (band rows + 2 halo rows) x wpad bytes, then 16 bytes of slack (the funnel
// shifts read one word beyond a row; those bytes only reach sites outside
// the update / flip masks).
// WT: 0 the uniform rules; 1 periodic weights (a.wper > 0), a per-site
// threshold instead of thr[0]; 2 the lozenges' volume weight q
// (qlozengekernel.cl), add below thr[2], remove in [2^22, thr[3]).  Separate
// instantiations, so that the uniform kernel carries none of it.
template <int FAM, int MAXW, bool PHILOX, int LB, int WT>
__global__ void __launch_bounds__(LB, 1) word_kernel(const __grid_constant__ WalkArgs a) {
    using M = WordModel<FAM>;
    constexpr int NC = M::NC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* lat = smem_raw + 16;

    const int BLOCK = blockDim.x;
    const int cta = blockIdx.x, nct = gridDim.x, tid = threadIdx.x;
    const int r0 = cta * a.rows_per_cta;
    const int r1 = min(a.rows, r0 + a.rows_per_cta);
    const int nrows = r1 - r0;
    const int a0 = r0 + M::ROFF, a1 = r1 + M::ROFF;
    const int W = a.wpad;
    const int plane = (nrows + 2) * W;
    const int Gw = W >> 2;  // words per row (the fast mode's counter stride too)
    const int nwords = nrows * Gw;
    const int N = a.n;

    for (int l = 0; l < a.nlat; ++l)
        for (int c = 0; c < NC; ++c) {
            const int8_t* g = static_cast<const int8_t*>(a.arr[l][c]);
            unsigned char* s = lat + (l * NC + c) * plane;
            for (int e = tid; e < plane; e += BLOCK) {
                const int rr = a0 - 1 + e / W, j = e % W;
                int8_t v = 0;
                if (rr >= 0 && rr < a.arows && j < a.width) v = g[(size_t)rr * a.width + j];
                s[e] = (unsigned char)v;
            }
        }

    const bool has_top = cta > 0, has_bot = cta + 1 < nct;
    const bool bot_edge = has_bot && !(has_top && nrows == 1);
    // Update mask of band row rr / word w: rows 1..N-2, columns 1..width-2;
    // Rotate positions: columns COFF..COFF+cols-1 (all band rows).
    auto info_at = [&](int rr, int w) {
        WordInfo wi;
        wi.off = (rr + 1) * W + 4 * w;
        const int i = a0 + rr;
        wi.cls = M::DOM ? (i & 1) : i % 3;
        const int j0 = 4 * w;
        uint32_t ub = 0, vb = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int j = j0 + b;
            if (j >= 1 && j <= a.width - 2) ub |= 1u << b;
            if (j >= M::COFF && j < M::COFF + a.cols) vb |= 1u << b;
        }
        if (!(i >= 1 && i <= N - 2)) ub = 0;
        wi.um = lane_bytes(ub) * 0xffu;
        wi.vm = lane_bytes(vb);
        return wi;
    };
    auto is_edge = [&](int u) {
        const int rr = u / Gw;
        return (has_top && rr == 0) || (bot_edge && rr == nrows - 1);
    };
    // Lozenge column shifts for each colour t whose Update is applied.
    uint32_t shift_tab[3] = {0u, 0u, 0u};
    if (!M::DOM) {
        shift_tab[0] = lozenge_shift_table(0);
        shift_tab[1] = lozenge_shift_table(1);
        shift_tab[2] = lozenge_shift_table(2);
    }
    // This thread's share of the halo exchange: words e = tid + x * BLOCK of
    // [side][lattice][word] (one array per phase in these models).
    const int per_side = a.nlat * a.xwords;

    // The words u = tid + m * BLOCK (m < MAXW) of this thread, their facts
    // and (bit-exact mode) their positions' TinyMT states, all in registers.
    // MAXW = 0 (fast mode on large bands): words are walked at run time.
    constexpr int NW = MAXW > 0 ? MAXW : 1;
    WordInfo winfo[NW];
    TinyState st[PHILOX ? 1 : NW][4];
    uint32_t wflags = 0;  // bit 2m: word m exists, bit 2m+1: it is an edge word
    if (MAXW > 0) {
#pragma unroll
        for (int m = 0; m < MAXW; ++m) {
            const int u = tid + m * BLOCK;
            if (u < nwords) {
                winfo[m] = info_at(u / Gw, u % Gw);
                wflags |= (1u << (2 * m)) | ((is_edge(u) ? 1u : 0u) << (2 * m + 1));
            } else {
                winfo[m] = WordInfo{0, 0, 0u, 0u};
            }
        }
    }
    const TinyParams tp{a.mat1, a.mat2, a.tmat};

    // One word per thread: the owner of word w of the band's first row polls
    // word w of the row above, the owner of word w of its last row the row
    // below, and only the warps that hold edge words meet at the halo
    // barrier -- the other warps' words overlap the whole exchange.
    bool poll_top = false, poll_bot = false, in_group = false;
    int gthreads = 0;
    if (MAXW == 1) {
        const int rr = tid / Gw;
        poll_top = tid < nwords && has_top && rr == 0;
        poll_bot = tid < nwords && has_bot && rr == nrows - 1;
        in_group = __any_sync(0xffffffffu, poll_top || poll_bot);
        gthreads = 32 * __syncthreads_count((tid & 31) == 0 && in_group);
    }
    // The split only pays when some warps hold no edge word.
    const bool split = MAXW == 1 && gthreads < BLOCK;

    int epoch = -1;
    int64_t next_epoch = a.nepochs > 0 ? a.epoch_start[0] : INT64_MAX;
    uint32_t key0 = 0, key1 = 0;
    int64_t dstep = 0;
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
#pragma unroll
                for (int m = 0; m < NW; ++m) {
                    if (!(wflags & (1u << (2 * m)))) continue;
                    const int rpos = r0 + winfo[m].off / W - 1;  // position row
                    const int jw = winfo[m].off % W;             // 4 * word
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        if (!(winfo[m].vm & (1u << (8 * b)))) continue;
                        const uint32_t sid = (uint32_t)(jw + b - M::COFF) + (uint32_t)a.cols * (uint32_t)rpos;
                        tiny_seed(st[m][b], tp, (uint32_t)eseed + sid);
                    }
                }
            }
        }
        const bool draws = (d & PH_DRAWS) != 0u;
        const WordPhase P = word_phase_of<FAM>(d, lat, plane, shift_tab);
        const int lat1 = NC * plane;  // second lattice (coupled CFTP chains)
        auto apply = [&](const WordInfo& wi, const uint32_t (&k)[4]) {
            uint32_t m0 = 0, m1 = 0;
            if (draws) {
                if (WT == 1 && FAM == FAM_DOMINO_HB) {
                    // weighted heat bath: a threshold per site from its vertex (i, j);
                    // array column c of the rotated array A is vertex column 2 c + ((i + A) & 1)
                    const int i = a0 + wi.off / W - 1, c0 = wi.off % W, par = (i + 1 - (int)ph_a(d)) & 1;
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        m0 |= (uint32_t)(k[b] < weight_thr(a, i, 2 * (c0 + b) + par)) << (8 * b);
                } else if (WT == 1 && FAM == FAM_LOZENGE8) {
                    // weighted lozenges: the add threshold of each site's vertex; array
                    // column c of colour C is vertex column 3 c + (C + i) mod 3
                    const int i = a0 + wi.off / W - 1, c0 = wi.off % W, rem = ((int)ph_a(d) + i) % 3;
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        m0 |= (uint32_t)(k[b] < weight_thr(a, i, 3 * (c0 + b) + rem)) << (8 * b);
                } else if (WT == 2) {
                    m0 = below4(k, a.thr[2]);
                } else {
                    m0 = below4(k, a.thr[0]);
                }
                if (WT == 2)
                    m1 = below4(k, a.thr[3]) & ~below4(k, 1u << 22);
                else if (!M::DOM)
                    m1 = below4(k, a.thr[1]) & ~m0;
            }
            word_phase<FAM>(P, 0, W, wi, m0, m1);
            if (a.nlat > 1) word_phase<FAM>(P, lat1, W, wi, m0, m1);
        };
        // Word m of this thread (u = tid + m * BLOCK of the band).
        auto own_word = [&](int m) {
            uint32_t k[4] = {0u, 0u, 0u, 0u};
            if (draws) {
                if (PHILOX) {
                    const int u = tid + m * BLOCK;
                    const uint4 w4 = philox4((uint32_t)(a0 * Gw + u), (uint32_t)dstep, (uint32_t)((uint64_t)dstep >> 32),
                                             a.chain, key0, key1);
                    k[0] = w4.x >> 9;
                    k[1] = w4.y >> 9;
                    k[2] = w4.z >> 9;
                    k[3] = w4.w >> 9;
                } else {
                    // The four generators advance side by side; a site that is
                    // not a Rotate position keeps its state (and draws nothing).
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        TinyState& sb = st[PHILOX ? 0 : m][b];
                        TinyState nx = sb;
                        tiny_advance(nx, tp);
                        const uint32_t out = tiny_output(nx, tp) >> 9;
                        const bool on = (winfo[m].vm >> (8 * b)) & 1u;
                        k[b] = on ? out : 0u;
                        sb.s0 = on ? nx.s0 : sb.s0;
                        sb.s1 = on ? nx.s1 : sb.s1;
                        sb.s2 = on ? nx.s2 : sb.s2;
                        sb.s3 = on ? nx.s3 : sb.s3;
                    }
                }
            }
            apply(winfo[m], k);
        };
        auto philox_word = [&](int rr, int w) {
            const WordInfo wi = info_at(rr, w);
            uint32_t k[4] = {0u, 0u, 0u, 0u};
            if (draws) {
                const uint4 w4 = philox4((uint32_t)((a0 + rr) * Gw + w), (uint32_t)dstep,
                                         (uint32_t)((uint64_t)dstep >> 32), a.chain, key0, key1);
                k[0] = w4.x >> 9;
                k[1] = w4.y >> 9;
                k[2] = w4.z >> 9;
                k[3] = w4.w >> 9;
            }
            apply(wi, k);
        };
        // Fast mode: words u = lo + tid + x * BLOCK < hi, walked with an
        // incremental (row, word) pair.
        auto philox_range = [&](int lo, int hi) {
            int u = lo + tid;
            if (u >= hi) return;
            int rr = u / Gw, w = u - rr * Gw;
            const int drr = BLOCK / Gw, dw = BLOCK - drr * Gw;
            for (; u < hi; u += BLOCK) {
                philox_word(rr, w);
                rr += drr;
                w += dw;
                if (w >= Gw) {
                    w -= Gw;
                    ++rr;
                }
            }
        };

        if (MAXW == 1 && split) {
            bool fail = false;
            if (!in_group) {
                if (wflags & 1u) own_word(0);
            } else {
                if (ph > 0 && gthreads > 0) {
                    // Halo words of the array the neighbours flipped in the previous phase.
                    const uint32_t mask = M::written(d_prev);
                    bool ok = true;
                    if (mask && (poll_top || poll_bot)) {
                        const int arr = __ffs(mask) - 1;
                        const int par = (int)((ph - 1) & 1);
                        const uint32_t tag = (uint32_t)ph;
                        const int w = tid % Gw;
                        for (int l = 0; l < a.nlat && ok; ++l) {
                            uint32_t v;
                            if (poll_top) {
                                ok = wait_word(a, slot(a, cta - 1, 1, par, l, 0) + w, tag, &v);
                                if (ok) sts(lat + (l * NC + arr) * plane + 4 * w, v);
                            }
                            if (poll_bot && ok) {
                                ok = wait_word(a, slot(a, cta + 1, 0, par, l, 0) + w, tag, &v);
                                if (ok) sts(lat + (l * NC + arr) * plane + (nrows + 1) * W + 4 * w, v);
                            }
                        }
                    }
                    fail = bar_red_or_n(1, gthreads, !ok);
                }
                if (!fail && wflags) own_word(0);  // the edge word, or a word of the row next to it
            }
            if (__syncthreads_or(fail)) return;
        } else {
            // Words away from the band's edge rows first, overlapping the neighbours' progress.
            if (MAXW == 0) {
                const int lo = has_top ? Gw : 0;
                philox_range(lo, max(lo, nwords - (has_bot ? Gw : 0)));
            } else {
#pragma unroll
                for (int m = 0; m < NW; ++m)
                    if ((wflags >> (2 * m) & 3u) == 1u) own_word(m);
            }
            if (ph > 0) {
                // Halo rows of the array the neighbours flipped in the previous phase.
                const uint32_t mask = M::written(d_prev);
                bool ok = true;
                if (mask) {
                    const int arr = __ffs(mask) - 1;
                    const int par = (int)((ph - 1) & 1);
                    const uint32_t tag = (uint32_t)ph;
                    for (int e = tid; e < 2 * per_side && ok; e += BLOCK) {
                        const int side = e >= per_side;  // 0: row above (from cta-1), 1: row below (from cta+1)
                        const int rem = e - side * per_side;
                        const int l = rem >= a.xwords;
                        const int w = rem - l * a.xwords;
                        const int src = side == 0 ? cta - 1 : cta + 1;
                        if (src < 0 || src >= nct) continue;
                        uint32_t v;
                        ok = wait_word(a, slot(a, src, 1 - side, par, l, 0) + w, tag, &v);
                        if (ok) sts(lat + (l * NC + arr) * plane + (side == 0 ? 0 : nrows + 1) * W + 4 * w, v);
                    }
                }
                if (__syncthreads_or(!ok)) return;
            }
            if (MAXW == 0) {
                if (has_top) philox_range(0, Gw);
                if (bot_edge) philox_range(nwords - Gw, nwords);
            } else {
#pragma unroll
                for (int m = 0; m < NW; ++m)
                    if ((wflags >> (2 * m) & 3u) == 3u) own_word(m);
            }
            __syncthreads();
        }
        if (ph + 1 < a.nphases && !(cta == 0 && ph == a.drop_phase)) {
            // Publish the band's first / last row of the array flipped in this phase.
            const uint32_t mask = M::written(d);
            if (mask) {
                const int arr = __ffs(mask) - 1;
                const int par = (int)(ph & 1);
                const unsigned long long tag = (unsigned long long)(uint32_t)(ph + 1) << 32;
                for (int e = tid; e < 2 * per_side; e += BLOCK) {
                    const int side = e >= per_side;  // 0: first row (read by cta-1), 1: last row (read by cta+1)
                    const int rem = e - side * per_side;
                    const int l = rem >= a.xwords;
                    const int w = rem - l * a.xwords;
                    const int dst = side == 0 ? cta - 1 : cta + 1;
                    if (dst < 0 || dst >= nct) continue;
                    const unsigned char* row = lat + (l * NC + arr) * plane + (side == 0 ? 1 : nrows) * W;
                    st_relaxed64(slot(a, cta, side, par, l, 0) + w, tag | lds(row + 4 * w));
                }
            }
        }
        if (PHILOX && draws) ++dstep;
        d_prev = d;
        d = d_next;
    }

    __syncthreads();
    for (int l = 0; l < a.nlat; ++l)
        for (int c = 0; c < NC; ++c) {
            int8_t* g = static_cast<int8_t*>(a.arr[l][c]);
            const unsigned char* s = lat + (l * NC + c) * plane;
            for (int e = tid; e < nrows * a.width; e += BLOCK) {
                const int rr = e / a.width, j = e % a.width;
                g[(size_t)(a0 + rr) * a.width + j] = (int8_t)s[(rr + 1) * W + j];
            }
        }
}

using KernelFn = void (*)(WalkArgs);

template <int FAM, int WT>
static KernelFn word_fn(int maxw, bool philox) {
    if (philox) {
        switch (maxw) {
            case 0: return word_kernel<FAM, 0, true, 1024, WT>;
            case 1: return word_kernel<FAM, 1, true, 1024, WT>;
            case 2: return word_kernel<FAM, 2, true, 1024, WT>;
            case 4: return word_kernel<FAM, 4, true, 1024, WT>;
            default: return nullptr;
        }
    }
    switch (maxw) {
        case 1: return word_kernel<FAM, 1, false, 1024, WT>;
        case 2: return word_kernel<FAM, 2, false, 512, WT>;
        case 4: return word_kernel<FAM, 4, false, 512, WT>;
        default: return nullptr;
    }
}

static KernelFn word_kernel_for(int family, int maxw, bool philox, bool weighted) {
    switch (family) {
        case FAM_DOMINO: return word_fn<FAM_DOMINO, 0>(maxw, philox);
        case FAM_DOMINO_HB:
            return weighted ? word_fn<FAM_DOMINO_HB, 1>(maxw, philox) : word_fn<FAM_DOMINO_HB, 0>(maxw, philox);
        case FAM_LOZENGE8:
            return weighted ? word_fn<FAM_LOZENGE8, 1>(maxw, philox) : word_fn<FAM_LOZENGE8, 0>(maxw, philox);
        case FAM_QLOZENGE8: return weighted ? nullptr : word_fn<FAM_LOZENGE8, 2>(maxw, philox);
        default: return nullptr;
    }
}

bool word_family(int family) { return family == FAM_DOMINO || family == FAM_DOMINO_HB || family == FAM_LOZENGE8; }

rt_status plan_word_walk(int family, int device, int nlat, int rows, int width, bool philox, int ctas_hint,
                         WalkPlan* plan, std::string* err, bool weighted) {
    if (!word_family(family) && family != FAM_QLOZENGE8) {
        *err = "no word kernel for this model";
        return RT_E_INVAL;
    }
    int sms = 0, smem_optin = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) {
        *err = "cudaDeviceGetAttribute failed";
        return RT_E_CUDA;
    }
    const int nc = family == FAM_LOZENGE8 || family == FAM_QLOZENGE8 ? 3 : 2;
    const int wpad = (width + 3) & ~3;
    const int gw = wpad / 4;
    int ctas = std::max(1, std::min(ctas_hint > 0 ? ctas_hint : sms, rows));
    const int rpc = (rows + ctas - 1) / ctas;
    ctas = (rows + rpc - 1) / rpc;
    const int words = rpc * gw;
    // One word per thread up to 1024 threads; bit-exact mode then keeps 2
    // or 4 words' generator states per thread in registers (512 threads).
    int maxw = 1, block = 0;
    if (philox) {
        // Fast mode keeps no generator state: up to 4 words' facts per thread
        // in registers, beyond that words are walked at run time.
        maxw = words <= 1024 ? 1 : words <= 2048 ? 2 : words <= 4096 ? 4 : 0;
        block = maxw == 0 ? 1024 : std::min(1024, ((words + maxw - 1) / maxw + 31) / 32 * 32);
    } else if (words <= 1024) {
        block = (words + 31) / 32 * 32;
    } else {
        for (maxw = 2; maxw <= 4; maxw *= 2)
            if ((words + maxw - 1) / maxw <= kWordBlockMax) break;
        if (maxw > 4) {
            *err = "band too wide for register-resident generator states";
            return RT_E_INVAL;
        }
        block = ((words + maxw - 1) / maxw + 31) / 32 * 32;
    }
    const size_t smem = 32 + (size_t)nlat * nc * (rpc + 2) * wpad;
    if (smem > (size_t)smem_optin) {
        *err = "band does not fit in shared memory";
        return RT_E_INVAL;
    }
    KernelFn fn = word_kernel_for(family, maxw, philox, weighted);
    if (!fn) {
        *err = "no word kernel for this configuration";
        return RT_E_INVAL;
    }
    if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
        *err = "cudaFuncSetAttribute failed";
        return RT_E_CUDA;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, block, smem) != cudaSuccess) {
        *err = "cudaOccupancyMaxActiveBlocksPerMultiprocessor failed";
        return RT_E_CUDA;
    }
    if (per_sm < 1 || ctas > per_sm * sms) {
        *err = "word-kernel grid cannot be co-resident";
        return RT_E_INVAL;
    }
    plan->items = maxw;
    plan->block = block;
    plan->rows_per_cta = rpc;
    plan->ctas = ctas;
    plan->smem = smem;
    plan->wpad = wpad;
    plan->xwords = wpad / 4;
    plan->xslots = 1;
    plan->fn = (const void*)fn;
    return RT_OK;
}

}  // namespace rtb
