// rt_plane.cu -- the bit-plane walk kernel of the int8 models (RT_RNG_PLANES).
//
// Dominoes and uniform lozenges keep 4 / 6 edge bits per site.  Here a
// colour array lives in shared memory as 4 / 6 bit planes, one 32-bit word
// per 32 consecutive sites of a row, so every Update and Rotate of the
// reference kernels (dominokernel.cl, dominokernelCFTP.cl, lozengekernel.cl)
// becomes a few bitwise operations on whole words: an Update copies one
// neighbour plane per refreshed bit (shifted by one column with a funnel
// shift where the neighbour is at j +- 1), a Rotate finds the rotatable
// sites by plane algebra and flips them where the random bits say so.  One
// Philox4x32-10 call gives the bits of 128 sites; the rules (no reference
// counterpart, so each is its own fast dynamics with the same equilibrium):
//   dominoes, heat bath (RT_KERNEL_CFTP): a rotatable site becomes 12
//       (two vertical dominoes) where its bit is 1, else 3;
//   dominoes, toggle (RT_KERNEL_DEFAULT): a rotatable site toggles 3 <-> 12
//       where either of its two bits is 1 (probability 3/4);
//   lozenges (RT_KERNEL_DEFAULT), heat bath: 25 -> 38 (add a cube) where the
//       bit is 1, 38 -> 25 where it is 0.
// The heat-bath rules are monotone under shared bits (CFTP).
//
// Temporal blocking: a CTA holds its band of rows plus H rows of every
// colour array above and below it, and runs H phases between two halo
// exchanges, recomputing the halo rows itself (the draws depend only on the
// site, the step and the key, so every CTA computes the same values for a
// row): after phase k of a block the rows within H - k - 1 of the band are
// current, so after H phases exactly the band is.  Then each CTA publishes
// its first and last H rows of every colour (the tagged-word protocol of
// rt_exchange.cuh, one tag per block) and reads its neighbours' ones.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "rt_exchange.cuh"
#include "rt_internal.h"
#include "rt_models.cuh"
#include "rt_word.cuh"

namespace rtb {

template <int FAM>
struct PlaneModel {
    static constexpr bool DOM = FAM != FAM_LOZENGE8;
    static constexpr int NC = DOM ? 2 : 3;  // colour arrays
    static constexpr int NP = DOM ? 4 : 6;  // bit planes per colour
    static constexpr int ROFF = DOM ? 1 : 0;
    static constexpr int COFF = DOM ? 1 : 0;
};

__device__ __forceinline__ uint32_t col_next(uint32_t cur, uint32_t nxt) { return __funnelshift_r(cur, nxt, 1); }
__device__ __forceinline__ uint32_t col_prev(uint32_t prv, uint32_t cur) { return __funnelshift_l(prv, cur, 1); }

// Bits [lo, hi) of the 32 columns starting at column 32 w.
__device__ __forceinline__ uint32_t col_mask(int w, int lo, int hi) {
    const int a = max(lo - 32 * w, 0), b = min(hi - 32 * w, 32);
    if (b <= a) return 0u;
    const uint32_t upper = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
    return upper & ~((1u << a) - 1u);
}

// Shared memory: planes [lattice][colour][plane][stored row][RS words];
// stored row s is colour-array row a0 - H + s; word 0 and word WW + 1 of a
// row are zero padding for the funnel shifts; then two masks per word.
// WPT: words per work item -- 1 (small bands: the most parallelism; the
// four words of a Philox call each recompute it) or 4 (one call per item).
template <int FAM, int LB, int WPT>
__global__ void __launch_bounds__(LB, 1) plane_kernel(const __grid_constant__ WalkArgs a) {
    using M = PlaneModel<FAM>;
    constexpr int NC = M::NC, NP = M::NP;
    extern __shared__ __align__(16) uint32_t psm[];
    __shared__ uint32_t s_dph[32];  // descriptors of the current block (depth <= 32)
    const int BLOCK = blockDim.x, tid = threadIdx.x;
    const int cta = blockIdx.x, nct = gridDim.x;
    const int H = a.depth, WW = a.pwords, RS = WW + 2;
    const int QPR = (WW + 3) >> 2;  // Philox calls per row
    // balanced bands: every CTA has floor or ceil(rows / nct) rows
    const int r0 = (int)((int64_t)cta * a.rows / nct), r1 = (int)((int64_t)(cta + 1) * a.rows / nct);
    const int nrows = r1 - r0;
    const int R = a.rows_per_cta + 2 * H;  // stored rows (rows_per_cta = ceil(rows / nct))
    const int a0 = r0 + M::ROFF;            // colour-array row of the band's first row
    const int N = a.n;
    const int PLANE = R * RS;  // words per plane (shared memory: fits an int)
    uint32_t* um_col = psm + a.nlat * NC * NP * PLANE;
    uint32_t* vm_col = um_col + WW;
    auto pl = [&](int l, int c, int k) { return psm + ((l * NC + c) * NP + k) * PLANE; };

    for (int w = tid; w < WW; w += BLOCK) {
        um_col[w] = col_mask(w, 1, a.width - 1);
        vm_col[w] = col_mask(w, M::COFF, M::COFF + a.cols);
    }
    // Load: stored rows [0, nrows + 2H) from the byte arrays; rows outside
    // the lattice stay zero.  Padding words are zero.
    for (int l = 0; l < a.nlat; ++l)
        for (int c = 0; c < NC; ++c) {
            const int8_t* g = static_cast<const int8_t*>(a.arr[l][c]);
            for (int e = tid; e < R * RS; e += BLOCK) {
                const int s = e / RS, w = e % RS - 1;
                const int i = a0 - H + s;
                uint32_t bits[NP];
#pragma unroll
                for (int k = 0; k < NP; ++k) bits[k] = 0u;
                if (w >= 0 && w < WW && s < nrows + 2 * H && i >= 0 && i < a.arows) {
                    const int8_t* row = g + (size_t)i * a.width;
                    const int jend = min(32, a.width - 32 * w);
                    for (int b = 0; b < jend; ++b) {
                        const uint32_t v = (uint32_t)(uint8_t)row[32 * w + b];
                        if (v >> NP) atomicOr(a.err, ERR_BADOP);
#pragma unroll
                        for (int k = 0; k < NP; ++k) bits[k] |= ((v >> k) & 1u) << b;
                    }
                }
#pragma unroll
                for (int k = 0; k < NP; ++k) pl(l, c, k)[e] = bits[k];
            }
        }
    const int per_lat = NC * NP * H * WW;  // exchange words per side and lattice
    // lozenge column shifts: 9 bits per pending colour t, 3 per row class
    const uint32_t shifts = M::DOM ? 0u
                                   : lozenge_shift_table(0) | (lozenge_shift_table(1) << 9) |
                                         (lozenge_shift_table(2) << 18);

    int epoch = -1;
    int64_t next_epoch = a.nepochs > 0 ? a.epoch_start[0] : INT64_MAX;
    uint32_t key0 = 0, key1 = 0;
    int64_t dstep = 0;
    __syncthreads();

    int64_t blk = 0;
    for (int64_t b0 = 0; b0 < a.nphases; b0 += H, ++blk) {
        const int K = (int)min((int64_t)H, a.nphases - b0);
        // The block's phase descriptors, loaded before any wait (every thread
        // read the previous block's ones before that block's last barrier).
        if (tid < K) s_dph[tid] = __ldg(a.phases + b0 + tid);
        if (b0 > 0 && nct > 1) {
            // Halo rows of every colour from the neighbours' previous block:
            // four tagged words per thread are loaded at once, and only the
            // ones not yet published are polled one by one (bounded).
            const int par = (int)((blk - 1) & 1);
            const uint32_t tag = (uint32_t)blk;
            const int total = 2 * a.nlat * per_lat;
            bool ok = true;
            for (int base = 0; base < total && ok; base += 4 * BLOCK) {
                unsigned long long v[4];
                const unsigned long long* src_at[4];
#pragma unroll
                for (int x8 = 0; x8 < 4; ++x8) {
                    const int e = base + tid + x8 * BLOCK;
                    src_at[x8] = nullptr;
                    v[x8] = 0ull;
                    if (e >= total) continue;
                    const int side = e >= a.nlat * per_lat;  // 0: rows above (from cta-1), 1: below (cta+1)
                    const int rem = e - side * a.nlat * per_lat;
                    const int l = rem / per_lat;
                    const int x = rem - l * per_lat;
                    const int src = side == 0 ? cta - 1 : cta + 1;
                    if (src < 0 || src >= nct) continue;
                    src_at[x8] = slot(a, src, 1 - side, par, l, 0) + x;
                    v[x8] = ld_relaxed64(src_at[x8]);
                }
#pragma unroll
                for (int x8 = 0; x8 < 4; ++x8) {
                    if (!src_at[x8] || !ok) continue;
                    uint32_t val = (uint32_t)v[x8];
                    if ((uint32_t)(v[x8] >> 32) != tag) ok = wait_word(a, src_at[x8], tag, &val);
                    if (!ok) break;
                    const int e = base + tid + x8 * BLOCK;
                    const int side = e >= a.nlat * per_lat;
                    const int rem = e - side * a.nlat * per_lat;
                    const int l = rem / per_lat;
                    const int x = rem - l * per_lat;
                    const int w = x % WW, j = (x / WW) % H, ck = x / (WW * H);
                    const int s = side == 0 ? j : H + nrows + j;
                    pl(l, ck / NP, ck % NP)[(size_t)s * RS + w + 1] = val;
                }
            }
            if (__syncthreads_or(!ok)) return;
        } else {
            __syncthreads();
        }
        for (int k = 0; k < K; ++k) {
            const int64_t ph = b0 + k;
            if (ph == next_epoch) {
                while (epoch + 1 < a.nepochs && a.epoch_start[epoch + 1] == ph) ++epoch;
                next_epoch = epoch + 1 < a.nepochs ? a.epoch_start[epoch + 1] : INT64_MAX;
                key0 = (uint32_t)a.epoch_seed[epoch];
                key1 = (uint32_t)(a.epoch_seed[epoch] >> 32);
                dstep = 0;
            }
            const uint32_t d = s_dph[k];
            const bool draws = (d & PH_DRAWS) != 0u;
            const int op = (int)ph_op(d), ca = (int)ph_a(d), cb = (int)ph_b(d);
            const bool step = op == (int)OP_STEP;
            const bool upd = step ? (cb != (int)NO_COLOUR && cb != ca) : true;
            const int tt = step ? (upd ? cb : 0) : ca;  // colour whose Update is pending
            // rows computed in this phase (global band-row index g)
            const int g_lo = max(0, r0 - H + k + 1), g_hi = min(a.rows, r1 + H - k - 1);
            const int s_lo = g_lo - (r0 - H);
            const int IPR = WPT == 1 ? WW : QPR;  // work items per row
            const int items = (g_hi - g_lo) * IPR;
            // Plane offsets (32-bit shared-memory word indices) used by this phase,
            // lattice 0; lattice l adds l * LAT.
            const int LAT = NC * NP * PLANE;
            int dst_off = 0, src_off = 0, tt_off = 0, t1_off = 0, t2_off = 0, ca_off = 0;
            if (M::DOM) {
                const int dst = step ? 1 - ca : ca;  // reference colour r flips array 1 - r
                dst_off = dst * NP * PLANE;
                src_off = (1 - dst) * NP * PLANE;
            } else {
                const int t1 = tt == 2 ? 0 : tt + 1, t2 = tt == 0 ? 2 : tt - 1;
                tt_off = tt * NP * PLANE;
                t1_off = t1 * NP * PLANE;
                t2_off = t2 * NP * PLANE;
                ca_off = ca * NP * PLANE;
            }
            const bool ca_is_t1 = !M::DOM && ca == (tt == 2 ? 0 : tt + 1);
            int srow = s_lo + tid / IPR, it = tid - (tid / IPR) * IPR;
            const int dsr = BLOCK / IPR, dit = BLOCK - dsr * IPR;
            for (int u = tid; u < items; u += BLOCK) {
                const int s = srow;
                const int i = a0 - H + s;  // colour-array row
                uint4 r1 = make_uint4(0u, 0u, 0u, 0u), r2 = make_uint4(0u, 0u, 0u, 0u);
                if (draws) {
                    const uint32_t c0 = (uint32_t)((i - M::ROFF) * QPR + (WPT == 1 ? (it >> 2) : it));
                    r1 = philox4(c0, (uint32_t)dstep, (uint32_t)((uint64_t)dstep >> 32), a.chain, key0, key1);
                    if (FAM == FAM_DOMINO)
                        r2 = philox4(c0 | 0x80000000u, (uint32_t)dstep, (uint32_t)((uint64_t)dstep >> 32), a.chain,
                                     key0, key1);
                }
                const bool row_upd = i >= 1 && i <= N - 2;
                const int p = (i ^ tt) & 1;                                                  // dominoes
                const uint32_t sh = M::DOM ? 0u : (shifts >> (9 * tt + 3 * (i % 3))) & 7u;  // lozenges
#pragma unroll
                for (int x4 = 0; x4 < WPT; ++x4) {
                const int w = WPT == 1 ? it : 4 * it + x4;
                if (w >= WW) break;
                const int o = s * RS + w + 1;
                const uint32_t um = row_upd ? um_col[w] : 0u;
                const uint32_t vm = vm_col[w];
                const uint32_t b1 = quad_word(r1, w & 3), b2 = quad_word(r2, w & 3);
                for (int l = 0; l < a.nlat; ++l) {
                    uint32_t* const L = psm + l * LAT;
                    if (M::DOM) {
                        uint32_t* const D = L + dst_off + o;
                        const uint32_t* const S = L + src_off + o;
                        uint32_t v[4];
#pragma unroll
                        for (int q = 0; q < 4; ++q) v[q] = D[q * PLANE];
                        if (upd) {
                            // domino_refresh (dominokernel.cl:22-31): bit 1 <- up's bit 2,
                            // bit 2 <- down's bit 1, bit 4 <- west's bit 8, bit 8 <- east's bit 4;
                            // west / east share the column in rows of one parity.
                            const uint32_t up = S[PLANE - RS], dn = S[RS];
                            const uint32_t* s3 = S + 3 * PLANE;
                            const uint32_t* s2 = S + 2 * PLANE;
                            const uint32_t west = p ? s3[0] : col_prev(s3[-1], s3[0]);
                            const uint32_t east = p ? col_next(s2[0], s2[1]) : s2[0];
                            v[0] = (v[0] & ~um) | (up & um);
                            v[1] = (v[1] & ~um) | (dn & um);
                            v[2] = (v[2] & ~um) | (west & um);
                            v[3] = (v[3] & ~um) | (east & um);
                        }
                        if (step) {
                            const uint32_t rot = ((v[0] & v[1] & ~v[2] & ~v[3]) | (~v[0] & ~v[1] & v[2] & v[3])) & vm;
                            if (FAM == FAM_DOMINO_HB) {
                                // heat bath: 12 (planes 2, 3) where the bit is 1, else 3 (planes 0, 1)
                                v[0] = (v[0] & ~rot) | (~b1 & rot);
                                v[1] = (v[1] & ~rot) | (~b1 & rot);
                                v[2] = (v[2] & ~rot) | (b1 & rot);
                                v[3] = (v[3] & ~rot) | (b1 & rot);
                            } else {
                                const uint32_t tog = rot & (b1 | b2);
#pragma unroll
                                for (int q = 0; q < 4; ++q) v[q] ^= tog;
                            }
                        }
#pragma unroll
                        for (int q = 0; q < 4; ++q) D[q * PLANE] = v[q];
                    } else {
                        uint32_t v[6];
                        uint32_t* const C = L + ca_off + o;
                        if (upd) {
                            // lozenge_refresh (lozengekernel.cl:36-54): colour t+1 takes bits
                            // {2, 4, 32} from the flipped colour t at (i-1, j+sa), (i, j-sw),
                            // (i+1, j); colour t+2 takes {1, 8, 16} from (i-1, j), (i, j+se),
                            // (i+1, j-sa).
                            const uint32_t* const F = L + tt_off + o;
                            const uint32_t* f4 = F + 4 * PLANE - RS;
                            const uint32_t* f3 = F + 3 * PLANE;
                            const uint32_t* f1 = F + PLANE + RS;
                            const uint32_t* f2 = F + 2 * PLANE;
                            const uint32_t n1 = (sh & 1u) ? col_next(f4[0], f4[1]) : f4[0];
                            const uint32_t n2 = (sh & 2u) ? col_prev(f3[-1], f3[0]) : f3[0];
                            const uint32_t n5 = F[RS];
                            const uint32_t m0 = F[5 * PLANE - RS];
                            const uint32_t m3 = (sh & 4u) ? col_next(f2[0], f2[1]) : f2[0];
                            const uint32_t m4 = (sh & 1u) ? col_prev(f1[-1], f1[0]) : f1[0];
                            uint32_t* const A = L + t1_off + o;
                            uint32_t* const B = L + t2_off + o;
                            const uint32_t a1 = (A[PLANE] & ~um) | (n1 & um), a2 = (A[2 * PLANE] & ~um) | (n2 & um),
                                           a5 = (A[5 * PLANE] & ~um) | (n5 & um);
                            const uint32_t c0v = (B[0] & ~um) | (m0 & um), c3 = (B[3 * PLANE] & ~um) | (m3 & um),
                                           c4 = (B[4 * PLANE] & ~um) | (m4 & um);
                            if (!step) {
                                A[PLANE] = a1;
                                A[2 * PLANE] = a2;
                                A[5 * PLANE] = a5;
                                B[0] = c0v;
                                B[3 * PLANE] = c3;
                                B[4 * PLANE] = c4;
                                continue;
                            }
                            // the colour not flipped now keeps its refreshed planes
                            if (ca_is_t1) {
                                B[0] = c0v;
                                B[3 * PLANE] = c3;
                                B[4 * PLANE] = c4;
                                v[1] = a1;
                                v[2] = a2;
                                v[5] = a5;
                                v[0] = C[0];
                                v[3] = C[3 * PLANE];
                                v[4] = C[4 * PLANE];
                            } else {
                                A[PLANE] = a1;
                                A[2 * PLANE] = a2;
                                A[5 * PLANE] = a5;
                                v[0] = c0v;
                                v[3] = c3;
                                v[4] = c4;
                                v[1] = C[PLANE];
                                v[2] = C[2 * PLANE];
                                v[5] = C[5 * PLANE];
                            }
                        } else {
#pragma unroll
                            for (int q = 0; q < 6; ++q) v[q] = C[q * PLANE];
                        }
                        // heat bath: 25 (planes 0, 3, 4) -> 38 (planes 1, 2, 5) where the bit is 1, back where 0
                        const uint32_t e25 = v[0] & ~v[1] & ~v[2] & v[3] & v[4] & ~v[5];
                        const uint32_t e38 = ~v[0] & v[1] & v[2] & ~v[3] & ~v[4] & v[5];
                        const uint32_t tog = ((e25 & b1) | (e38 & ~b1)) & vm;
#pragma unroll
                        for (int q = 0; q < 6; ++q) C[q * PLANE] = v[q] ^ tog;
                    }
                }
                }
                srow += dsr;
                it += dit;
                if (it >= IPR) {
                    it -= IPR;
                    ++srow;
                }
            }
            if (draws) ++dstep;
            __syncthreads();
        }
        if (b0 + K < a.nphases && nct > 1 && !(cta == 0 && blk == a.drop_phase)) {
            // Publish the band's first and last H rows of every colour.
            const int par = (int)(blk & 1);
            const unsigned long long tag = (unsigned long long)(uint32_t)(blk + 1) << 32;
            for (int e = tid; e < 2 * a.nlat * per_lat; e += BLOCK) {
                const int side = e >= a.nlat * per_lat;  // 0: first rows (read by cta-1), 1: last rows (cta+1)
                const int rem = e - side * a.nlat * per_lat;
                const int l = rem / per_lat;
                const int x = rem - l * per_lat;
                const int dst = side == 0 ? cta - 1 : cta + 1;
                if (dst < 0 || dst >= nct) continue;
                const int w = x % WW, j = (x / WW) % H, ck = x / (WW * H);
                const int s = side == 0 ? H + j : nrows + j;
                st_relaxed64(slot(a, cta, side, par, l, 0) + x, tag | pl(l, ck / NP, ck % NP)[(size_t)s * RS + w + 1]);
            }
        }
    }

    __syncthreads();
    // Store the band rows back as bytes.
    for (int l = 0; l < a.nlat; ++l)
        for (int c = 0; c < NC; ++c) {
            int8_t* g = static_cast<int8_t*>(a.arr[l][c]);
            for (int e = tid; e < nrows * a.width; e += BLOCK) {
                const int rr = e / a.width, j = e % a.width;
                const size_t o = (size_t)(H + rr) * RS + (j >> 5) + 1;
                uint32_t v = 0u;
#pragma unroll
                for (int k = 0; k < NP; ++k) v |= ((pl(l, c, k)[o] >> (j & 31)) & 1u) << k;
                g[(size_t)(a0 + rr) * a.width + j] = (int8_t)v;
            }
        }
}

using PlaneFn = void (*)(WalkArgs);

template <int FAM>
static PlaneFn plane_fn_of(int block, int wpt) {
    if (wpt == 4) return block > 512 ? plane_kernel<FAM, 1024, 4> : plane_kernel<FAM, 512, 4>;
    return block > 512 ? plane_kernel<FAM, 1024, 1> : plane_kernel<FAM, 512, 1>;
}

static PlaneFn plane_fn(int family, int block, int wpt) {
    switch (family) {
        case FAM_DOMINO: return plane_fn_of<FAM_DOMINO>(block, wpt);
        case FAM_DOMINO_HB: return plane_fn_of<FAM_DOMINO_HB>(block, wpt);
        case FAM_LOZENGE8: return plane_fn_of<FAM_LOZENGE8>(block, wpt);
        default: return nullptr;
    }
}

rt_status plan_plane_walk(int family, int device, int nlat, int rows, int width, int ctas_hint, int depth_hint,
                          WalkPlan* plan, std::string* err) {
    if (!word_family(family)) {
        *err = "bit-plane walks exist for dominoes and uniform lozenges";
        return RT_E_INVAL;
    }
    int sms = 0, smem_optin = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) {
        *err = "cudaDeviceGetAttribute failed";
        return RT_E_CUDA;
    }
    const int nc = family == FAM_LOZENGE8 ? 3 : 2, np = family == FAM_LOZENGE8 ? 6 : 4;
    const int ww = (width + 31) / 32, rs = ww + 2;
    int ctas = std::max(1, std::min(ctas_hint > 0 ? ctas_hint : sms, rows));
    const int rpc = (rows + ctas - 1) / ctas;
    const int min_rows = rows / ctas;
    int depth = std::max(1, std::min(depth_hint > 0 ? std::min(depth_hint, 32) : 8, min_rows));
    if (ctas == 1) depth = 1;
    size_t smem = 0;
    for (;; --depth) {
        smem = (size_t)nlat * nc * np * (rpc + 2 * depth) * rs * 4 + 2 * (size_t)ww * 4;
        if (smem <= (size_t)smem_optin || depth == 1) break;
    }
    if (smem > (size_t)smem_optin) {
        *err = "band does not fit in shared memory";
        return RT_E_INVAL;
    }
    // Work items of the widest phase (band + 2 (depth - 1) rows): one word
    // each while that keeps 1024 threads busy at most twice, else four words
    // (one Philox call each).  The halo exchange uses every thread, so small
    // bands still launch 512.
    const int words = (rpc + 2 * (depth - 1)) * ww;
    const int wpt = words > 2048 ? 4 : 1;
    const int items = wpt == 4 ? (rpc + 2 * (depth - 1)) * ((ww + 3) / 4) : words;
    const int block = items > 512 ? 1024 : 512;
    PlaneFn fn = plane_fn(family, block, wpt);
    if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        *err = "cudaFuncSetAttribute failed";
        return RT_E_CUDA;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, block, smem) != cudaSuccess) {
        *err = "cudaOccupancyMaxActiveBlocksPerMultiprocessor failed";
        return RT_E_CUDA;
    }
    if (per_sm < 1 || ctas > per_sm * sms) {
        *err = "bit-plane grid cannot be co-resident";
        return RT_E_INVAL;
    }
    plan->items = 0;
    plan->block = block;
    plan->rows_per_cta = rpc;
    plan->ctas = ctas;
    plan->smem = smem;
    plan->wpad = rs;
    plan->xwords = nc * np * depth * ww;
    plan->xslots = 1;
    plan->depth = depth;
    plan->pwords = ww;
    plan->fn = (const void*)fn;
    return RT_OK;
}

}  // namespace rtb
