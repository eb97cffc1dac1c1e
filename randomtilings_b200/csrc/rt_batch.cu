// rt_batch.cu -- batched chains (include/rt_b200_batch.h): kernels, planner,
// autotuner and the CUDA graph that runs them.
//
// One launch per kernel family.  Its grid is a set of thread-block clusters;
// cluster c walks chains c, c + C, c + 2C, ... of the family's list (sorted by
// size, largest first), each chain from its first phase to its last without
// leaving the SMs: the cluster's CTAs split the chain's rows into bands held
// in shared memory, and after every phase each CTA pulls the rows next to its
// band that its neighbours just wrote from their shared memory (distributed
// shared memory, two cluster barriers per phase).  Chains never wait on other
// clusters, so the launch needs no co-residency beyond the cluster itself.
// The per-site arithmetic is that of the single-walk kernels (word_phase for
// the int8 models, Model::site for the int32 ones), and the draws are the
// fast mode's, so every chain equals its single-chain fast-mode walk.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rt_b200_batch.h"
#include "rt_internal.h"
#include "rt_guard.h"
#include "rt_models.cuh"
#include "rt_tdplane.cuh"
#include "rt_tridimer.cuh"
#include "rt_word.cuh"

using rtb::guarded;

namespace cg = cooperative_groups;

namespace rtb {

struct BatchChain {
    void* arr[8];  // colour arrays of the chain
    int n, rows, cols, arows, width, wpad;
    uint32_t chain, pad_;
    uint64_t key;
    uint32_t thr[3];  // lozenges: add below thr[0]; remove in [thr[2], thr[1])
    uint32_t pad2_;
};

struct BatchArgs {
    const BatchChain* chains;
    const int* order;  // chain indices, largest first
    int nchains;
    const uint32_t* phases;
    int64_t nphases;
    const int64_t* step0;  // colour steps the chains have already made (Philox step counter offset)
    int64_t step_add;      // colour steps of this run made by the family's earlier launches in it
    uint32_t thr[4];
    float weights[16];
};

__device__ __forceinline__ void cluster_or_block_sync(cg::cluster_group& cluster, int CL) {
    if (CL > 1)
        cluster.sync();
    else
        __syncthreads();
}

// ---------------------------------------------------------------------------
// int8 models: words of four sites (rt_word.cuh).
// Shared memory: 16 B slack, NC planes of (rpc + 2) x wpad bytes, 16 B
// slack, then per band row its class (i mod 3 or i mod 2) and "row can be
// refreshed" flag, then per word column its update and position masks.
// ---------------------------------------------------------------------------
template <int FAM>
__global__ void __launch_bounds__(1024, 1) batch_word_kernel(const __grid_constant__ BatchArgs b) {
    using M = WordModel<FAM>;
    constexpr int NC = M::NC;
    cg::cluster_group cluster = cg::this_cluster();
    const int CL = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int ncl = gridDim.x / CL;
    const int cid = blockIdx.x / CL;
    const int BLOCK = blockDim.x, tid = threadIdx.x;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* lat = smem_raw + 16;
    uint32_t shift_tab[3] = {0u, 0u, 0u};
    if (!M::DOM) {
        shift_tab[0] = lozenge_shift_table(0);
        shift_tab[1] = lozenge_shift_table(1);
        shift_tab[2] = lozenge_shift_table(2);
    }

    for (int q = cid; q < b.nchains; q += ncl) {
        const BatchChain& ch = b.chains[b.order[q]];
        const int rows = ch.rows, W = ch.wpad, Gw = W >> 2, N = ch.n, width = ch.width, cols = ch.cols;
        const int rpc = (rows + CL - 1) / CL;
        const int r0 = min(rows, rank * rpc), r1 = min(rows, r0 + rpc);
        const int nrows = r1 - r0;
        const int a0 = r0 + M::ROFF;
        const int plane = (rpc + 2) * W;
        unsigned char* row_cls = lat + NC * plane + 16;
        unsigned char* row_ok = row_cls + rpc;
        uint32_t* col_um = reinterpret_cast<uint32_t*>(row_cls + ((2 * rpc + 3) & ~3));
        uint32_t* col_vm = col_um + Gw;

        for (int c = 0; c < NC; ++c) {
            const int8_t* g = static_cast<const int8_t*>(ch.arr[c]);
            unsigned char* s = lat + c * plane;
            for (int e = tid; e < (nrows + 2) * W; e += BLOCK) {
                const int rr = a0 - 1 + e / W, j = e % W;
                int8_t v = 0;
                if (rr >= 0 && rr < ch.arows && j < width) v = g[(size_t)rr * width + j];
                s[e] = (unsigned char)v;
            }
        }
        for (int rr = tid; rr < nrows; rr += BLOCK) {
            const int i = a0 + rr;
            row_cls[rr] = (unsigned char)(M::DOM ? (i & 1) : i % 3);
            row_ok[rr] = (unsigned char)(i >= 1 && i <= N - 2);
        }
        for (int w = tid; w < Gw; w += BLOCK) {
            uint32_t ub = 0, vb = 0;
#pragma unroll
            for (int bb = 0; bb < 4; ++bb) {
                const int j = 4 * w + bb;
                if (j >= 1 && j <= width - 2) ub |= 1u << bb;
                if (j >= M::COFF && j < M::COFF + cols) vb |= 1u << bb;
            }
            col_um[w] = lane_bytes(ub) * 0xffu;
            col_vm[w] = lane_bytes(vb);
        }
        __syncthreads();

        const uint32_t key0 = (uint32_t)ch.key, key1 = (uint32_t)(ch.key >> 32);
        int64_t dstep = *b.step0 + b.step_add;
        const int nwords = nrows * Gw;
        const int drr = BLOCK / Gw, dw = BLOCK - drr * Gw;
        for (int64_t ph = 0; ph < b.nphases; ++ph) {
            const uint32_t d = __ldg(b.phases + ph);
            const bool draws = (d & PH_DRAWS) != 0u;
            const WordPhase P = word_phase_of<FAM>(d, lat, plane, shift_tab);
            int rr = tid / Gw, w = tid - (tid / Gw) * Gw;
            for (int u = tid; u < nwords; u += BLOCK) {
                WordInfo wi;
                wi.off = (rr + 1) * W + 4 * w;
                wi.cls = row_cls[rr];
                wi.um = row_ok[rr] ? col_um[w] : 0u;
                wi.vm = col_vm[w];
                uint32_t m0 = 0, m1 = 0;
                if (draws) {
                    const uint4 w4 = philox4((uint32_t)((a0 + rr) * Gw + w), (uint32_t)dstep,
                                             (uint32_t)((uint64_t)dstep >> 32), ch.chain, key0, key1);
                    const uint32_t k[4] = {w4.x >> 9, w4.y >> 9, w4.z >> 9, w4.w >> 9};
                    if (M::DOM) {
                        m0 = below4(k, b.thr[0]);
                    } else {
                        m0 = below4(k, ch.thr[0]);
                        m1 = below4(k, ch.thr[1]) & ~below4(k, ch.thr[2]);
                    }
                }
                word_phase<FAM>(P, 0, W, wi, m0, m1);
                rr += drr;
                w += dw;
                if (w >= Gw) {
                    w -= Gw;
                    ++rr;
                }
            }
            if (draws) ++dstep;
            if (CL > 1) {
                cluster.sync();
                const uint32_t mask = M::written(d);
                if (mask && nrows > 0) {
                    // Rows next to the band: the upper CTA's last row, the lower CTA's first.
                    const int arr = __ffs(mask) - 1;
                    for (int e = tid; e < 2 * Gw; e += BLOCK) {
                        const int side = e >= Gw, x = e - side * Gw;
                        if ((side == 0 && rank == 0) || (side == 1 && r1 >= rows)) continue;
                        unsigned char* mine = lat + arr * plane + (side == 0 ? 0 : nrows + 1) * W + 4 * x;
                        unsigned char* theirs = lat + arr * plane + (side == 0 ? rpc : 1) * W + 4 * x;
                        sts(mine, lds(cluster.map_shared_rank(theirs, rank + (side == 0 ? -1 : 1))));
                    }
                }
                cluster.sync();
            } else {
                __syncthreads();
            }
        }
        for (int c = 0; c < NC; ++c) {
            int8_t* g = static_cast<int8_t*>(ch.arr[c]);
            const unsigned char* s = lat + c * plane;
            for (int e = tid; e < nrows * width; e += BLOCK) {
                const int rr = e / width, j = e % width;
                g[(size_t)(a0 + rr) * width + j] = (int8_t)s[(rr + 1) * W + j];
            }
        }
        cluster_or_block_sync(cluster, CL);
    }
}

// ---------------------------------------------------------------------------
// int32 models (rectangle-triangles, triangle dimers): the per-site rules of
// the generic walk kernel, positions taken in quads of one Philox call.
// Shared memory: NC planes of (rpc + 2) x wpad int32.
// ---------------------------------------------------------------------------
template <class Model>
__global__ void __launch_bounds__(1024, 1) batch_site_kernel(const __grid_constant__ BatchArgs b) {
    using T = typename Model::Elem;
    constexpr int NC = Model::NCOL;
    cg::cluster_group cluster = cg::this_cluster();
    const int CL = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int ncl = gridDim.x / CL;
    const int cid = blockIdx.x / CL;
    const int BLOCK = blockDim.x, tid = threadIdx.x;
    __shared__ WalkArgs wa;  // the fields the site rules read: n, wpad, thr, weights
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* lat = reinterpret_cast<T*>(smem_raw);

    for (int q = cid; q < b.nchains; q += ncl) {
        const BatchChain& ch = b.chains[b.order[q]];
        const int rows = ch.rows, W = ch.wpad, cols = ch.cols, width = ch.width;
        const int rpc = (rows + CL - 1) / CL;
        const int r0 = min(rows, rank * rpc), r1 = min(rows, r0 + rpc);
        const int nrows = r1 - r0;
        const int a0 = r0 + Model::ROFF;
        const int plane = (rpc + 2) * W;
        if (tid == 0) {
            wa.n = ch.n;
            wa.wpad = W;
            for (int x = 0; x < 4; ++x) wa.thr[x] = b.thr[x];
            for (int x = 0; x < 16; ++x) wa.weights[x] = b.weights[x];
            wa.wper = 0;  // no weighted dominoes in batches
        }
        for (int c = 0; c < NC; ++c) {
            const T* g = static_cast<const T*>(ch.arr[c]);
            T* s = lat + c * plane;
            for (int e = tid; e < (nrows + 2) * W; e += BLOCK) {
                const int rr = a0 - 1 + e / W, j = e % W;
                T v = (T)0;
                if (rr >= 0 && rr < ch.arows && j < width) v = g[(size_t)rr * width + j];
                s[e] = v;
            }
        }
        __syncthreads();

        const uint32_t key0 = (uint32_t)ch.key, key1 = (uint32_t)(ch.key >> 32);
        int64_t dstep = *b.step0 + b.step_add;
        const int Gw = (width + 3) >> 2;
        const int qlo = Model::COFF >> 2;
        const int G = ((Model::COFF + cols - 1) >> 2) - qlo + 1;
        const int nq = nrows * G;
        const int drr = BLOCK / G, dq = BLOCK - drr * G;
        for (int64_t ph = 0; ph < b.nphases; ++ph) {
            const uint32_t d = __ldg(b.phases + ph);
            const bool draws = (d & PH_DRAWS) != 0u;
            const typename Model::Ctx x0 = Model::ctx(wa, lat, plane, d, a0 - 1);
            int rr = tid / G, cq = tid - (tid / G) * G;
            for (int u = tid; u < nq; u += BLOCK) {
                const int qq = qlo + cq, r = r0 + rr;
                uint4 w4 = make_uint4(0u, 0u, 0u, 0u);
                if (draws)
                    w4 = philox4((uint32_t)((r + Model::ROFF) * Gw + qq), (uint32_t)dstep,
                                 (uint32_t)((uint64_t)dstep >> 32), ch.chain, key0, key1);
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    const int c = 4 * qq + bb - Model::COFF;
                    if (c >= 0 && c < cols) {
                        const int i = r + Model::ROFF, j = c + Model::COFF;
                        Model::site(wa, x0, (rr + 1) * W + j, i, j, quad_word(w4, bb) >> 9);
                    }
                }
                rr += drr;
                cq += dq;
                if (cq >= G) {
                    cq -= G;
                    ++rr;
                }
            }
            if (draws) ++dstep;
            if (CL > 1) {
                cluster.sync();
                uint32_t mask = Model::written(d);
                if (nrows > 0) {
                    while (mask) {
                        const int arr = __ffs(mask) - 1;
                        mask &= mask - 1;
                        for (int e = tid; e < 2 * W; e += BLOCK) {
                            const int side = e >= W, x = e - side * W;
                            if ((side == 0 && rank == 0) || (side == 1 && r1 >= rows)) continue;
                            T* mine = lat + arr * plane + (side == 0 ? 0 : nrows + 1) * W + x;
                            T* theirs = lat + arr * plane + (side == 0 ? rpc : 1) * W + x;
                            *mine = *cluster.map_shared_rank(theirs, rank + (side == 0 ? -1 : 1));
                        }
                    }
                }
                cluster.sync();
            } else {
                __syncthreads();
            }
        }
        for (int c = 0; c < NC; ++c) {
            T* g = static_cast<T*>(ch.arr[c]);
            const T* s = lat + c * plane;
            for (int e = tid; e < nrows * width; e += BLOCK) {
                const int rr = e / width, j = e % width;
                g[(size_t)(a0 + rr) * width + j] = s[(rr + 1) * W + j];
            }
        }
        cluster_or_block_sync(cluster, CL);
    }
}

// One phase of op OP over the band rows [r0, r0 + nrows) of a triangle-dimer
// chain held as bit planes: only the rows TriDimerRule::live_rows admits, one
// 32-site word per work item.  Drawing ops take the fast mode's draws: quad
// cq of array row r is Philox4x32-10 of (r Gw + cq, step, chain), and a site
// flips when its output word is below 2^31 (k = word >> 9 below 2^22).
template <uint32_t OP, int T, int B = -1>
__device__ __forceinline__ void tdp_phase(uint32_t* planes, int ps, int rs, int row0, uint32_t a, uint32_t b, int m,
                                          int width, int r0, int nrows, int wb, int tid, int BLOCK, int64_t dstep,
                                          uint32_t chain, uint32_t key0, uint32_t key1) {
    constexpr bool DRAWS = OP == TD_ROT_LOZ || OP == TD_ROT_TRI || OP == TD_ROT_BFLY;
    int S, o;
    TriDimerRule::live_rows<OP>(a, b, &S, &o);
    const int first = r0 + ((o - r0) % S + S) % S;
    if (first >= r0 + nrows) return;
    const int nlive = (r0 + nrows - first + S - 1) / S;
    const int items = nlive * wb;
    const int Gw = (width + 3) >> 2;
    for (int u = tid; u < items; u += BLOCK) {
        const int rr = u / wb, c = u - rr * wb;
        const int r = first + S * rr;
        uint32_t draw = 0u;
        if (DRAWS) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int cq = 8 * c + q;
                if (cq < Gw) {
                    const uint4 w4 = philox4((uint32_t)(r * Gw + cq), (uint32_t)dstep, (uint32_t)((uint64_t)dstep >> 32),
                                             chain, key0, key1);
                    draw |= ((~w4.x >> 31) | ((~w4.y >> 31) << 1) | ((~w4.z >> 31) << 2) | ((~w4.w >> 31) << 3))
                            << (4 * q);
                }
            }
        }
        const tdp::View v{planes, ps, rs, row0, r, c};
        tdp::word_op<OP, T, B>(v, a, b, m, width, draw);
    }
}

// ---------------------------------------------------------------------------
// Triangle dimers: the eight arrays as 51 bit planes (rt_tdplane.cuh), 32
// sites per word.  Shared memory: one zero word, then per plane (rpc + 2)
// rows of wb + 1 words (the last word of a row stays zero), wb = words per
// array row.  Rows move between global int32 arrays and planes one warp per
// 32 columns, with a ballot per bit.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512, 1) batch_td_kernel(const __grid_constant__ BatchArgs b) {
    using R = TriDimerRule;
    cg::cluster_group cluster = cg::this_cluster();
    const int CL = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int ncl = gridDim.x / CL;
    const int cid = blockIdx.x / CL;
    const int BLOCK = blockDim.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = BLOCK >> 5;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* sm = reinterpret_cast<uint32_t*>(smem_raw);

    for (int q = cid; q < b.nchains; q += ncl) {
        const BatchChain& ch = b.chains[b.order[q]];
        const int rows = ch.rows, width = ch.width;
        const int rpc = (rows + CL - 1) / CL;
        const int r0 = min(rows, rank * rpc), r1 = min(rows, r0 + rpc);
        const int nrows = r1 - r0;
        const int wb = (width + 31) >> 5, rs = wb + 1, ps = (rpc + 2) * rs;
        uint32_t* planes = sm + 1;
        for (int e = tid; e < 1 + tdp::kPlanes * ps; e += BLOCK) sm[e] = 0u;
        __syncthreads();
        // global int32 rows r0 - 1 .. r1 -> planes
        for (int it = warp; it < (nrows + 2) * 8 * wb; it += nwarps) {
            const int sr = it / (8 * wb), rem = it - sr * 8 * wb, arr = rem / wb, c = rem - arr * wb;
            const int rr = r0 - 1 + sr, j = 32 * c + lane;
            int32_t v = 0;
            if (rr >= 0 && rr < ch.arows && j < width) v = static_cast<const int32_t*>(ch.arr[arr])[(size_t)rr * width + j];
            for (int k = 0; k < tdp::bits_of(arr); ++k) {
                const uint32_t w = __ballot_sync(0xffffffffu, (v >> k) & 1);
                if (lane == 0) planes[(tdp::plane_of(arr) + k) * ps + sr * rs + c] = w;
            }
        }
        __syncthreads();

        const uint32_t key0 = (uint32_t)ch.key, key1 = (uint32_t)(ch.key >> 32);
        const int m = ch.n / 2, row0 = r0 - 1;
        int64_t dstep = *b.step0 + b.step_add;
        for (int64_t ph = 0; ph < b.nphases; ++ph) {
            const uint32_t d = __ldg(b.phases + ph);
            const bool draws = (d & PH_DRAWS) != 0u;
            const uint32_t op = ph_op(d), pa = ph_a(d), pb = ph_b(d);
#define RT_TDP_ARGS planes, ps, rs, row0, pa, pb, m, width, r0, nrows, wb, tid, BLOCK, dstep, ch.chain, key0, key1
            switch (op) {
#define RT_TD_PHASE(OPC)                           \
    case OPC:                                      \
        if (pa == 0)                               \
            tdp_phase<OPC, 0>(RT_TDP_ARGS);        \
        else if (pa == 1)                          \
            tdp_phase<OPC, 1>(RT_TDP_ARGS);        \
        else                                       \
            tdp_phase<OPC, 2>(RT_TDP_ARGS);        \
        break;
                RT_TD_PHASE(TD_ROT_LOZ)
                RT_TD_PHASE(TD_LOZ_FLIPPED)
                RT_TD_PHASE(TD_LOZ_OTHER)
                RT_TD_PHASE(TD_UP_FROM_LOZ)
                case TD_TRI_OTHER:  // (a, b) in {(0, 7), (0, 0), (1, 0)} in the phase program
                    if (pa == 0 && pb == 7)
                        tdp_phase<TD_TRI_OTHER, 0, 7>(RT_TDP_ARGS);
                    else if (pa == 0 && pb == 0)
                        tdp_phase<TD_TRI_OTHER, 0, 0>(RT_TDP_ARGS);
                    else if (pa == 1 && pb == 0)
                        tdp_phase<TD_TRI_OTHER, 1, 0>(RT_TDP_ARGS);
                    else
                        tdp_phase<TD_TRI_OTHER, -1>(RT_TDP_ARGS);
                    break;
                RT_TD_PHASE(TD_ROT_TRI)
                RT_TD_PHASE(TD_TRI_FLIPPED)
                RT_TD_PHASE(TD_LOZ_FROM_TRI)
                case TD_BFLY_FROM_LOZ:  // (a, b) in {(0, 7), (1, 3), (1, 5), (1, 6)}
                    if (pa == 0 && pb == 7)
                        tdp_phase<TD_BFLY_FROM_LOZ, 0, 7>(RT_TDP_ARGS);
                    else if (pa == 1 && pb == 3)
                        tdp_phase<TD_BFLY_FROM_LOZ, 1, 3>(RT_TDP_ARGS);
                    else if (pa == 1 && pb == 5)
                        tdp_phase<TD_BFLY_FROM_LOZ, 1, 5>(RT_TDP_ARGS);
                    else if (pa == 1 && pb == 6)
                        tdp_phase<TD_BFLY_FROM_LOZ, 1, 6>(RT_TDP_ARGS);
                    else
                        tdp_phase<TD_BFLY_FROM_LOZ, -1>(RT_TDP_ARGS);
                    break;
                RT_TD_PHASE(TD_ROT_BFLY)
                RT_TD_PHASE(TD_BFLY_SAME)
                RT_TD_PHASE(TD_BFLY_21)
                RT_TD_PHASE(TD_BFLY_22)
                RT_TD_PHASE(TD_BFLY_23_LOZ)
#undef RT_TD_PHASE
#undef RT_TDP_ARGS
                default: break;
            }
            if (draws) ++dstep;
            if (CL > 1) {
                cluster.sync();
                uint32_t mask = R::written(d);
                if (nrows > 0) {
                    while (mask) {
                        const int arr = __ffs(mask) - 1;
                        mask &= mask - 1;
                        const int nb = tdp::bits_of(arr), p0 = tdp::plane_of(arr);
                        for (int e = tid; e < 2 * nb * wb; e += BLOCK) {
                            const int side = e >= nb * wb, rem = e - side * nb * wb, k = rem / wb, c = rem - k * wb;
                            if ((side == 0 && rank == 0) || (side == 1 && r1 >= rows)) continue;
                            const int mine = (p0 + k) * ps + (side == 0 ? 0 : nrows + 1) * rs + c;
                            const int theirs = (p0 + k) * ps + (side == 0 ? rpc : 1) * rs + c;
                            planes[mine] = *cluster.map_shared_rank(planes + theirs, rank + (side == 0 ? -1 : 1));
                        }
                    }
                }
                cluster.sync();
            } else {
                __syncthreads();
            }
        }
        // planes -> global int32 rows r0 .. r1 - 1
        for (int it = warp; it < nrows * 8 * wb; it += nwarps) {
            const int sr = 1 + it / (8 * wb), rem = it - (sr - 1) * 8 * wb, arr = rem / wb, c = rem - arr * wb;
            const int j = 32 * c + lane;
            int32_t v = 0;
            for (int k = 0; k < tdp::bits_of(arr); ++k)
                v |= (int32_t)((planes[(tdp::plane_of(arr) + k) * ps + sr * rs + c] >> lane) & 1u) << k;
            if (j < width) static_cast<int32_t*>(ch.arr[arr])[(size_t)(r0 - 1 + sr) * width + j] = v;
        }
        cluster_or_block_sync(cluster, CL);
    }
}

using BatchFn = void (*)(BatchArgs);

static BatchFn batch_fn(int family) {
    switch (family) {
        case FAM_DOMINO: return batch_word_kernel<FAM_DOMINO>;
        case FAM_DOMINO_HB: return batch_word_kernel<FAM_DOMINO_HB>;
        case FAM_LOZENGE8: return batch_word_kernel<FAM_LOZENGE8>;
        case FAM_RECTTRI: return batch_site_kernel<ThreeColour<int32_t, RectTriRule>>;
        case FAM_TRIDIMER: return batch_td_kernel;
        default: return nullptr;
    }
}

}  // namespace rtb

using namespace rtb;

namespace {

constexpr int kFamilies = 6;

struct Chain {
    int fam = 0, kind = 0, n = 0, ncol = 0, elem = 1;
    uint32_t thr[3] = {0u, 0u, 0u};
    int rows = 0, cols = 0, arows = 0, width = 0;
    uint32_t chain = 0;
    uint64_t key = 0;
    size_t off = 0;       // byte offset of its first colour array in the family buffer
    size_t per_arr = 0;   // bytes per colour array (256-aligned)
    std::vector<int32_t> start;  // the tiling as added (cells the arrays do not hold come from here)
};

struct Dev {
    void* p = nullptr;
    size_t cap = 0;
    bool reserve(size_t bytes) {
        if (bytes <= cap) return true;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return false;
        cap = bytes;
        return true;
    }
    ~Dev() {
        if (p) cudaFree(p);
    }
};

struct Plan {
    int cl = 1, block = 256, clusters = 1;
    size_t smem = 0;
    int64_t spl = 0;  // sweeps per launch: a run of S sweeps is S / spl launches (+ one for the rest); 0 = one
};

struct FamilyState {
    std::vector<int> members;  // chain indices
    std::vector<int> order;    // members sorted by lattice size, largest first (as indices into members)
    size_t bytes = 0;
    Dev data, recs, ord, phases, phases2, scratch, scratch_recs, step0;
    int64_t nphases = 0, phases_sweeps = -1;    // phases: one launch's sweeps
    int64_t nphases2 = 0, phases2_sweeps = -1;  // phases2: the last launch's, when shorter
    Plan plan;
    bool planned = false;
    double work = 0;  // relative cost of a sweep of the whole family (launch order)
};

int family_of(int32_t model, int32_t kernel) {
    if (model == RT_DOMINO) return kernel == RT_KERNEL_CFTP ? FAM_DOMINO_HB : kernel == RT_KERNEL_DEFAULT ? FAM_DOMINO : -1;
    if (model == RT_LOZENGE) return kernel == RT_KERNEL_DEFAULT ? FAM_LOZENGE8 : -1;
    if (model == RT_RECTTRI) return kernel == RT_KERNEL_DEFAULT ? FAM_RECTTRI : -1;
    if (model == RT_TRIDIMER) return kernel == RT_KERNEL_DEFAULT ? FAM_TRIDIMER : -1;
    return -1;
}
int kind_of(int fam) { return fam <= FAM_DOMINO_HB ? 0 : fam == FAM_LOZENGE8 ? 1 : fam == FAM_RECTTRI ? 2 : 3; }
int ncol_of(int fam) { return fam <= FAM_DOMINO_HB ? 2 : fam == FAM_TRIDIMER ? 8 : 3; }
int elem_of(int fam) { return fam <= FAM_LOZENGE8 ? 1 : 4; }
int steps_per_sweep(int kind) { return kind == 0 ? 2 : kind == 3 ? 30 : 3; }
bool word_fam(int fam) { return fam <= FAM_LOZENGE8; }

// Shared memory one CTA of a cluster of `cl` needs for chain c.
size_t smem_for(const Chain& c, int cl) {
    const int rpc = (c.rows + cl - 1) / cl;
    const int wpad = (c.width + 3) & ~3;
    if (word_fam(c.fam)) {
        return 16 + (size_t)c.ncol * (rpc + 2) * wpad + 16 + (size_t)((2 * rpc + 3) & ~3) + 2 * 4 * (size_t)(wpad / 4);
    }
    if (c.fam == FAM_TRIDIMER) {  // batch_td_kernel: one zero word, then 51 planes of (rpc + 2) x (wb + 1) words
        const size_t wb = (size_t)(c.width + 31) / 32;
        return 4 * (1 + (size_t)tdp::kPlanes * (rpc + 2) * (wb + 1));
    }
    return (size_t)c.ncol * (rpc + 2) * wpad * 4;
}

}  // namespace

struct rt_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t fam_stream[kFamilies] = {};
    cudaEvent_t fork = nullptr, join[kFamilies] = {}, t0 = nullptr, t1 = nullptr;
    std::string err;
    std::vector<Chain> chains;
    FamilyState fam[kFamilies];
    bool uploaded = false;
    int autotune = 1, force_cl = 0, force_block = 0;
    int64_t force_spl = -1;  // sweeps per launch set by the caller (-1: the autotuner's, or one launch)
    double tune_ms = 0, run_ms = 0;
    int64_t last_attempts = 0, last_bytes = 0;
    int64_t sweeps_done = 0;       // sweeps every chain has made so far
    int64_t* h_step0 = nullptr;    // pinned: per family, colour steps made so far
    cudaGraphExec_t exec = nullptr;
    int64_t exec_sweeps = -1;

    rt_status fail(rt_status s, const std::string& m) {
        err = m;
        return s;
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        exec_sweeps = -1;
    }
};

namespace {

thread_local std::string g_batch_create_error;

// rest: the launch runs the shorter phase list (the last launch of a run
// whose sweeps the plan's sweeps per launch do not divide).
BatchArgs args_for(rt_batch* b, int f, const void* recs, int64_t step_add = 0, bool rest = false) {
    FamilyState& F = b->fam[f];
    BatchArgs a;
    std::memset(&a, 0, sizeof a);
    a.chains = static_cast<const BatchChain*>(recs);
    a.order = static_cast<const int*>(F.ord.p);
    a.nchains = (int)F.members.size();
    a.phases = static_cast<const uint32_t*>(rest ? F.phases2.p : F.phases.p);
    a.nphases = rest ? F.nphases2 : F.nphases;
    a.step0 = static_cast<const int64_t*>(F.step0.p);
    a.step_add = step_add;
    family_thresholds(f, 0.99, RT_QCMP_FLOAT32, a.thr);
    a.weights[0] = 0.0f;  // recttrianglekernel.cl:13
    for (int i = 1; i < 16; ++i) a.weights[i] = 1.0f;
    return a;
}

// priority: a CUDA stream priority (lower = scheduled first); 0 = default.
rt_status launch_family(rt_batch* b, int f, const Plan& p, const void* recs, cudaStream_t s, int priority = 0,
                        int64_t step_add = 0, bool rest = false) {
    BatchFn fn = batch_fn(f);
    BatchArgs a = args_for(b, f, recs, step_add, rest);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(p.clusters * p.cl));
    cfg.blockDim = dim3((unsigned)p.block);
    cfg.dynamicSmemBytes = p.smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)p.cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributePriority;
    attr[1].val.priority = priority;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    cudaError_t e = cudaLaunchKernelEx(&cfg, fn, a);
    if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    return RT_OK;
}

// Completes a plan (clusters that fit at once) for cluster size cl and CTA
// size block; false if it cannot run.
bool fill_plan(rt_batch* b, int f, int cl, int block, Plan* p) {
    FamilyState& F = b->fam[f];
    size_t smem = 0;
    for (int i : F.members) smem = std::max(smem, smem_for(b->chains[i], cl));
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
    BatchFn fn = batch_fn(f);
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, (const void*)fn) != cudaSuccess) return false;
    // A family's kernel may be built for fewer threads than asked for (the
    // bit-plane triangle-dimer kernel: 512); it then runs with its maximum.
    block = std::min(block, fa.maxThreadsPerBlock);
    if (smem + fa.sharedSizeBytes > (size_t)optin) return false;
    if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return false;
    if (cl > 8 && cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cl);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int active = 0;
    if (cudaOccupancyMaxActiveClusters(&active, (const void*)fn, &cfg) != cudaSuccess || active < 1) {
        cudaGetLastError();
        return false;
    }
    p->cl = cl;
    p->block = block;
    p->smem = smem;
    // Every resident cluster slot is used (fewer clusters with full rounds
    // measured slower: the families are bound by instruction issue and lose
    // more from fewer resident warps than they gain from the shorter tail).
    p->clusters = std::min<int>((int)F.members.size(), active);
    return true;
}

// The phase list of a launch of `sweeps` sweeps, into the family's first
// (rest = false) or second list.  Launches compose: each ends with the last
// colour's Update and the next starts with no Update pending, the same
// sequence of site updates as one longer launch.
rt_status stage_phases(rt_batch* b, int f, int64_t sweeps, bool rest = false) {
    FamilyState& F = b->fam[f];
    int64_t& have = rest ? F.phases2_sweeps : F.phases_sweeps;
    if (have == sweeps) return RT_OK;
    std::vector<uint32_t> ph;
    fast_phases(kind_of(f), sweeps * steps_per_sweep(kind_of(f)), ph);
    Dev& buf = rest ? F.phases2 : F.phases;
    if (!buf.reserve(std::max<size_t>(4, ph.size() * 4))) return b->fail(RT_E_NOMEM, "phase list");
    cudaError_t e = cudaMemcpy(buf.p, ph.data(), ph.size() * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("phase upload: ") + cudaGetErrorString(e));
    (rest ? F.nphases2 : F.nphases) = (int64_t)ph.size();
    have = sweeps;
    return RT_OK;
}

// Launches of a run of `sweeps` sweeps under sweeps-per-launch spl:
// (full launches, sweeps each, sweeps of the last shorter launch or 0).
struct LaunchSplit {
    int64_t full, per, rest;
};
LaunchSplit split_run(int64_t sweeps, int64_t spl) {
    if (spl <= 0 || spl >= sweeps) return {1, sweeps, 0};
    return {sweeps / spl, spl, sweeps % spl};
}

// Chain records whose arrays live at `base` (the family buffer or its scratch copy).
std::vector<BatchChain> records(rt_batch* b, int f, char* base) {
    FamilyState& F = b->fam[f];
    std::vector<BatchChain> r(F.members.size());
    for (size_t k = 0; k < F.members.size(); ++k) {
        const Chain& c = b->chains[F.members[k]];
        BatchChain& x = r[k];
        std::memset(&x, 0, sizeof x);
        for (int a = 0; a < c.ncol; ++a) x.arr[a] = base + c.off + a * c.per_arr;
        x.n = c.n;
        x.rows = c.rows;
        x.cols = c.cols;
        x.arows = c.arows;
        x.width = c.width;
        x.wpad = (c.width + 3) & ~3;
        x.chain = c.chain;
        x.key = c.key;
        for (int k = 0; k < 3; ++k) x.thr[k] = c.thr[k];
    }
    return r;
}

rt_status upload(rt_batch* b) {
    if (b->uploaded) return RT_OK;
    cudaSetDevice(b->device);
    Dev tmp;
    for (int f = 0; f < kFamilies; ++f) {
        FamilyState& F = b->fam[f];
        if (F.members.empty()) continue;
        size_t off = 0;
        for (int i : F.members) {
            Chain& c = b->chains[i];
            c.off = off;
            off += c.per_arr * c.ncol;
        }
        F.bytes = std::max<size_t>(off, 256);
        if (!F.data.reserve(F.bytes)) return b->fail(RT_E_NOMEM, "batch lattice buffer");
        cudaMemsetAsync(F.data.p, 0, F.bytes, b->stream);
        for (int i : F.members) {
            Chain& c = b->chains[i];
            char* base = static_cast<char*>(F.data.p) + c.off;
            void* arr[8] = {};
            for (int a = 0; a < c.ncol; ++a) arr[a] = base + a * c.per_arr;
            if (c.kind == 3) {
                std::vector<int32_t> arrays((size_t)8 * c.arows * c.width);
                td_split_host(c.start.data(), c.n, arrays.data());
                // batch_td_kernel keeps array a as tdp::bits_of(a) bit planes
                const size_t per = (size_t)c.arows * c.width;
                for (size_t e = 0; e < 8 * per; ++e) {
                    const int32_t v = arrays[e];
                    if (v < 0 || v >= (1 << tdp::bits_of((int)(e / per))))
                        return b->fail(RT_E_INVAL, "triangle-dimer state out of range for the bit planes");
                }
                for (int a = 0; a < 8; ++a)
                    cudaMemcpyAsync(arr[a], arrays.data() + (size_t)a * c.arows * c.width,
                                    (size_t)c.arows * c.width * 4, cudaMemcpyHostToDevice, b->stream);
                cudaStreamSynchronize(b->stream);
            } else {
                const size_t tb = (size_t)c.n * c.n * 4;
                if (!tmp.reserve(tb)) return b->fail(RT_E_NOMEM, "staging buffer");
                cudaMemcpyAsync(tmp.p, c.start.data(), tb, cudaMemcpyHostToDevice, b->stream);
                std::string e;
                if (launch_split(false, c.elem, c.kind, c.ncol, c.n, static_cast<int32_t*>(tmp.p), arr, b->stream, &e) !=
                    RT_OK)
                    return b->fail(RT_E_CUDA, e);
                cudaStreamSynchronize(b->stream);
            }
        }
        // Largest lattices first, so that round-robin over clusters balances.
        std::vector<int> order(F.members.size());
        for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            const Chain& cx = b->chains[F.members[x]];
            const Chain& cy = b->chains[F.members[y]];
            return (int64_t)cx.rows * cx.width > (int64_t)cy.rows * cy.width;
        });
        F.order = order;
        if (!F.step0.reserve(sizeof(int64_t))) return b->fail(RT_E_NOMEM, "step counter");
        cudaMemset(F.step0.p, 0, sizeof(int64_t));
        if (!F.ord.reserve(order.size() * sizeof(int))) return b->fail(RT_E_NOMEM, "chain order");
        cudaMemcpy(F.ord.p, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice);
        std::vector<BatchChain> r = records(b, f, static_cast<char*>(F.data.p));
        if (!F.recs.reserve(r.size() * sizeof(BatchChain))) return b->fail(RT_E_NOMEM, "chain records");
        cudaMemcpy(F.recs.p, r.data(), r.size() * sizeof(BatchChain), cudaMemcpyHostToDevice);
    }
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("batch upload: ") + cudaGetErrorString(e));
    b->uploaded = true;
    return RT_OK;
}

// Picks cluster and CTA size for family f: every feasible candidate runs a
// few sweeps on a scratch copy of the family's lattices; the fastest wins.
rt_status plan_family(rt_batch* b, int f) {
    FamilyState& F = b->fam[f];
    F.work = 0;
    const int blocks[] = {256, 512, 1024};
    const int cls[] = {1, 2, 4, 8};
    std::vector<Plan> cand;
    if (!b->autotune) {
        Plan p;
        const int cl = b->force_cl > 0 ? b->force_cl : 1;
        const int bl = b->force_block > 0 ? b->force_block : 512;
        if (!fill_plan(b, f, cl, bl, &p)) {
            // The requested cluster size cannot hold the largest chain: take the
            // smallest one that can.
            bool ok = false;
            for (int c : cls)
                if (c >= cl && fill_plan(b, f, c, bl, &p)) {
                    ok = true;
                    break;
                }
            if (!ok) return b->fail(RT_E_INVAL, "no cluster size holds the largest chain of a family in shared memory");
        }
        p.spl = b->force_spl > 0 ? b->force_spl : 0;
        F.plan = p;
        F.planned = true;
        return RT_OK;
    }
    for (int c : cls)
        for (int bl : blocks) {
            Plan p;
            if (!fill_plan(b, f, c, bl, &p)) continue;
            bool seen = false;  // a capped block size can repeat a candidate
            for (const Plan& q : cand) seen = seen || (q.cl == p.cl && q.block == p.block);
            if (!seen) cand.push_back(p);
        }
    if (cand.empty()) return b->fail(RT_E_INVAL, "no cluster size holds the largest chain of a family in shared memory");
    if (cand.size() == 1) {
        F.plan = cand[0];
        F.plan.spl = b->force_spl > 0 ? b->force_spl : 0;
        F.planned = true;
        return RT_OK;
    }
    if (!F.scratch.reserve(F.bytes) || !F.scratch_recs.reserve(F.members.size() * sizeof(BatchChain)))
        return b->fail(RT_E_NOMEM, "autotuner scratch");
    std::vector<BatchChain> r = records(b, f, static_cast<char*>(F.scratch.p));
    cudaMemcpy(F.scratch_recs.p, r.data(), r.size() * sizeof(BatchChain), cudaMemcpyHostToDevice);
    rt_status s = stage_phases(b, f, 4);
    if (s != RT_OK) return s;
    float best = 1e30f;
    for (const Plan& p : cand) {
        // Candidates set different shared-memory limits; this one's applies now.
        cudaFuncSetAttribute((const void*)batch_fn(f), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
        cudaMemcpyAsync(F.scratch.p, F.data.p, F.bytes, cudaMemcpyDeviceToDevice, b->stream);
        // one untimed run, then a timed one
        for (int rep = 0; rep < 2; ++rep) {
            cudaEventRecord(b->t0, b->stream);
            s = launch_family(b, f, p, F.scratch_recs.p, b->stream);
            if (s != RT_OK) return s;
            cudaEventRecord(b->t1, b->stream);
        }
        cudaError_t e = cudaEventSynchronize(b->t1);
        if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("autotuner run: ") + cudaGetErrorString(e));
        float ms = 0;
        cudaEventElapsedTime(&ms, b->t0, b->t1);
        if (ms < best) {
            best = ms;
            F.work = ms;
            F.plan = p;
        }
    }
    // Sweeps per launch at the chosen shape: a run of 32 sweeps as one
    // launch, against four launches of 8 (each reloading the lattices from
    // global memory, with its own tail of uneven chains).
    cudaFuncSetAttribute((const void*)batch_fn(f), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F.plan.smem);
    if ((s = stage_phases(b, f, 32)) != RT_OK || (s = stage_phases(b, f, 8, true)) != RT_OK) return s;
    float best_spl = 1e30f;
    for (const int64_t spl : {(int64_t)0, (int64_t)8}) {
        cudaMemcpyAsync(F.scratch.p, F.data.p, F.bytes, cudaMemcpyDeviceToDevice, b->stream);
        cudaEventRecord(b->t0, b->stream);
        const int nl = spl == 0 ? 1 : 32 / (int)spl;
        for (int k = 0; k < nl && s == RT_OK; ++k)
            s = launch_family(b, f, F.plan, F.scratch_recs.p, b->stream, 0,
                              (int64_t)k * 8 * steps_per_sweep(kind_of(f)), spl != 0);
        if (s != RT_OK) return s;
        cudaEventRecord(b->t1, b->stream);
        cudaError_t e = cudaEventSynchronize(b->t1);
        if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("autotuner run: ") + cudaGetErrorString(e));
        float ms = 0;
        cudaEventElapsedTime(&ms, b->t0, b->t1);
        if (ms < best_spl) {
            best_spl = ms;
            F.plan.spl = spl;
        }
    }
    F.phases_sweeps = F.phases2_sweeps = -1;  // the run stages its own lists
    if (b->force_spl >= 0) F.plan.spl = b->force_spl;
    F.planned = true;
    return RT_OK;
}

}  // namespace

extern "C" {

rt_status rt_batch_create(int32_t device, rt_batch** out) {
    return guarded([&]() -> rt_status {
        if (!out) return RT_E_INVAL;
        *out = nullptr;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
            g_batch_create_error = "no CUDA device with that ordinal";
            return RT_E_NODEVICE;
        }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
            g_batch_create_error = "device is not sm_100";
            return RT_E_NODEVICE;
        }
        cudaSetDevice(device);
        rt_batch* b = new rt_batch();
        b->device = device;
        bool ok = cudaMallocHost(&b->h_step0, kFamilies * sizeof(int64_t)) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
                  cudaEventCreate(&b->t0) == cudaSuccess && cudaEventCreate(&b->t1) == cudaSuccess;
        for (int f = 0; f < kFamilies && ok; ++f)
            ok = cudaStreamCreateWithFlags(&b->fam_stream[f], cudaStreamNonBlocking) == cudaSuccess &&
                 cudaEventCreateWithFlags(&b->join[f], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            rt_batch_destroy(b);
            g_batch_create_error = "stream / event creation failed";
            return RT_E_CUDA;
        }
        *out = b;
        return RT_OK;
    });
}

rt_status rt_batch_destroy(rt_batch* b) {
    return guarded([&]() -> rt_status {
        if (!b) return RT_E_INVAL;
        cudaSetDevice(b->device);
        if (b->stream) cudaStreamSynchronize(b->stream);
        b->drop_graph();
        for (int f = 0; f < kFamilies; ++f) {
            if (b->fam_stream[f]) cudaStreamDestroy(b->fam_stream[f]);
            if (b->join[f]) cudaEventDestroy(b->join[f]);
        }
        if (b->fork) cudaEventDestroy(b->fork);
        if (b->t0) cudaEventDestroy(b->t0);
        if (b->t1) cudaEventDestroy(b->t1);
        if (b->stream) cudaStreamDestroy(b->stream);
        if (b->h_step0) cudaFreeHost(b->h_step0);
        delete b;
        return RT_OK;
    });
}

const char* rt_batch_last_error(rt_batch* b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

rt_status rt_batch_add(rt_batch* b, const rt_chain* c, const int32_t* tiling, int32_t n, int64_t* index) {
    return guarded([&]() -> rt_status {
        if (!b || !c || !tiling) return b ? b->fail(RT_E_INVAL, "null argument") : RT_E_INVAL;
        if (b->sweeps_done > 0) return b->fail(RT_E_STATE, "chains are added before the first run");
        const int f = family_of(c->model, c->kernel);
        if (f < 0) return b->fail(RT_E_INVAL, "unsupported model / kernel in a batch");
        Chain ch;
        ch.fam = f;
        ch.kind = kind_of(f);
        ch.ncol = ncol_of(f);
        ch.elem = elem_of(f);
        ch.n = n;
        if (n > kMaxTilingSide) return b->fail(RT_E_INVAL, "tiling side above 32767");
        if (ch.kind == 0 && (n < 6 || n % 2)) return b->fail(RT_E_INVAL, "domino tiling side must be even and >= 6");
        if ((ch.kind == 1 || ch.kind == 2) && (n < 9 || n % 3))
            return b->fail(RT_E_INVAL, "tiling side must be a multiple of 3 and >= 9");
        if (ch.kind == 3 && (n < 8 || n % 2)) return b->fail(RT_E_INVAL, "triangle-dimer tiling side must be even and >= 8");
        if (ch.kind == 0) {
            ch.rows = n - 2, ch.cols = n / 2 - 2, ch.arows = n, ch.width = n / 2;
        } else if (ch.kind == 3) {
            ch.rows = n / 2, ch.cols = n / 2, ch.arows = n / 2, ch.width = n / 2;
        } else {
            ch.rows = n, ch.cols = n / 3, ch.arows = n, ch.width = n / 3;
        }
        ch.per_arr = ((size_t)ch.arows * ch.width * ch.elem + 255) & ~(size_t)255;
        const double q = c->q == 0.0f ? 1.0 : (double)c->q;
        if (!(q > 0.0 && q <= 1.0) || (ch.kind != 1 && q != 1.0))
            return b->fail(RT_E_INVAL, "q must lie in (0, 1] (lozenges) or be 0");
        if (ch.kind == 1) {
            ch.thr[0] = below_threshold(0.4 * q);
            ch.thr[1] = below_threshold(0.8);
            ch.thr[2] = below_threshold(0.4);
        }
        ch.chain = c->chain;
        ch.key = (uint64_t)c->key;
        ch.start.assign(tiling, tiling + (size_t)n * n);
        if (index) *index = (int64_t)b->chains.size();
        b->fam[f].members.push_back((int)b->chains.size());
        b->fam[f].planned = false;
        b->chains.push_back(std::move(ch));
        b->uploaded = false;
        b->drop_graph();
        for (int x = 0; x < kFamilies; ++x) b->fam[x].phases_sweeps = -1;
        return RT_OK;
    });
}

rt_status rt_batch_set_tuning(rt_batch* b, int32_t autotune, int32_t cluster, int32_t block) {
    return guarded([&]() -> rt_status {
        if (!b) return RT_E_INVAL;
        if (cluster < 0 || cluster > 16 || block < 0 || block > 1024 || block % 32)
            return b->fail(RT_E_INVAL, "cluster size must be 0..16, block a multiple of 32 up to 1024");
        b->autotune = autotune ? 1 : 0;
        b->force_cl = cluster;
        b->force_block = block;
        for (int f = 0; f < kFamilies; ++f) b->fam[f].planned = false;
        b->drop_graph();
        return RT_OK;
    });
}

rt_status rt_batch_set_sweeps_per_launch(rt_batch* b, int64_t sweeps) {
    return guarded([&]() -> rt_status {
        if (!b) return RT_E_INVAL;
        if (sweeps < -1) return b->fail(RT_E_INVAL, "sweeps per launch must be >= -1");
        if (sweeps > kMaxColourSteps / 32) return b->fail(RT_E_INVAL, "more than 2^35 sweeps per launch");
        b->force_spl = sweeps;
        for (int f = 0; f < kFamilies; ++f) b->fam[f].planned = false;
        b->drop_graph();
        return RT_OK;
    });
}

rt_status rt_batch_run(rt_batch* b, int64_t sweeps) {
    return guarded([&]() -> rt_status {
        if (!b) return RT_E_INVAL;
        if (sweeps < 0) return b->fail(RT_E_INVAL, "negative sweep count");
        if (sweeps > kMaxColourSteps / 32) return b->fail(RT_E_INVAL, "more than 2^35 sweeps in one call");
        if (b->chains.empty() || sweeps == 0) return RT_OK;
        cudaSetDevice(b->device);
        rt_status s = upload(b);
        if (s != RT_OK) return s;
        const auto w0 = std::chrono::steady_clock::now();
        bool tuned = false;
        for (int f = 0; f < kFamilies; ++f) {
            if (b->fam[f].members.empty() || b->fam[f].planned) continue;
            s = plan_family(b, f);
            if (s != RT_OK) return s;
            tuned = true;
            b->drop_graph();
        }
        if (tuned)
            b->tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        for (int f = 0; f < kFamilies; ++f) {
            FamilyState& F = b->fam[f];
            if (F.members.empty()) continue;
            const LaunchSplit ls = split_run(sweeps, F.plan.spl);
            if (F.phases_sweeps != ls.per || (ls.rest && F.phases2_sweeps != ls.rest) || b->exec_sweeps != sweeps)
                b->drop_graph();
            s = stage_phases(b, f, ls.per);
            if (s == RT_OK && ls.rest) s = stage_phases(b, f, ls.rest, true);
            if (s != RT_OK) return s;
        }
        if (!b->exec) {
            for (int f = 0; f < kFamilies; ++f)
                if (!b->fam[f].members.empty())
                    cudaFuncSetAttribute((const void*)batch_fn(f), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)b->fam[f].plan.smem);
            // One graph: fork to a stream per family, one launch each, join.  The
            // family with the most work goes first at the highest priority, so its
            // CTAs take the SMs and the smaller families fill the slots its last
            // round leaves idle.
            // Work of a family: the autotuner's time of its best plan when every
            // family has one, else its lattice bytes per sweep.
            int order[kFamilies], nf = 0;
            double est[kFamilies] = {};
            bool timed = true;
            for (int f = 0; f < kFamilies; ++f) {
                if (b->fam[f].members.empty()) continue;
                timed = timed && b->fam[f].work > 0;
                for (int i : b->fam[f].members) {
                    const Chain& c = b->chains[i];
                    est[f] += (double)steps_per_sweep(c.kind) * c.ncol * c.arows * c.width * c.elem;
                }
                order[nf++] = f;
            }
            if (timed)
                for (int k = 0; k < nf; ++k) est[order[k]] = b->fam[order[k]].work;
            std::sort(order, order + nf, [&](int x, int y) { return est[x] > est[y]; });
            int prio_low = 0, prio_high = 0;
            cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            cudaEventRecord(b->fork, b->stream);
            rt_status ls = RT_OK;
            for (int k = 0; k < nf && ls == RT_OK; ++k) {
                const int f = order[k];
                const LaunchSplit sp = split_run(sweeps, b->fam[f].plan.spl);
                const int64_t sps = steps_per_sweep(kind_of(f));
                cudaStreamWaitEvent(b->fam_stream[f], b->fork, 0);
                for (int64_t l = 0; l < sp.full + (sp.rest ? 1 : 0) && ls == RT_OK; ++l)
                    ls = launch_family(b, f, b->fam[f].plan, b->fam[f].recs.p, b->fam_stream[f],
                                       k == 0 ? prio_high : prio_low, l * sp.per * sps, l == sp.full);
                cudaEventRecord(b->join[f], b->fam_stream[f]);
                cudaStreamWaitEvent(b->stream, b->join[f], 0);
            }
            e = cudaStreamEndCapture(b->stream, &g);
            if (ls != RT_OK) {
                if (g) cudaGraphDestroy(g);
                return ls;
            }
            if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&b->exec, g, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                b->exec = nullptr;
                return b->fail(RT_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            }
            b->exec_sweeps = sweeps;
        }
        // Philox step counters continue where the previous run stopped, so two
        // runs of s1 and s2 sweeps equal one run of s1 + s2.
        for (int f = 0; f < kFamilies; ++f) {
            if (b->fam[f].members.empty()) continue;
            b->h_step0[f] = b->sweeps_done * steps_per_sweep(kind_of(f));
            cudaMemcpyAsync(b->fam[f].step0.p, &b->h_step0[f], sizeof(int64_t), cudaMemcpyHostToDevice, b->stream);
        }
        cudaEventRecord(b->t0, b->stream);
        cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
        if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
        cudaEventRecord(b->t1, b->stream);
        e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) return b->fail(RT_E_CUDA, std::string("batch run: ") + cudaGetErrorString(e));
        float ms = 0;
        cudaEventElapsedTime(&ms, b->t0, b->t1);
        b->run_ms = ms;
        b->sweeps_done += sweeps;
        int64_t att = 0, bytes = 0;
        for (const Chain& c : b->chains) {
            const int64_t steps = sweeps * steps_per_sweep(c.kind);
            att += steps * (int64_t)c.rows * c.cols;
            bytes += steps * 2 * (int64_t)c.ncol * c.arows * c.width * c.elem;
        }
        b->last_attempts = att;
        b->last_bytes = bytes;
        return RT_OK;
    });
}

rt_status rt_batch_download(rt_batch* b, int64_t index, int32_t* tiling) {
    return guarded([&]() -> rt_status {
        if (!b || !tiling) return b ? b->fail(RT_E_INVAL, "null tiling") : RT_E_INVAL;
        if (index < 0 || index >= (int64_t)b->chains.size()) return b->fail(RT_E_INVAL, "no chain with that index");
        cudaSetDevice(b->device);
        rt_status s = upload(b);
        if (s != RT_OK) return s;
        const Chain& c = b->chains[(size_t)index];
        FamilyState& F = b->fam[c.fam];
        char* base = static_cast<char*>(F.data.p) + c.off;
        void* arr[8] = {};
        for (int a = 0; a < c.ncol; ++a) arr[a] = base + a * c.per_arr;
        Dev tmp;
        const size_t tb = (size_t)c.n * c.n * 4;
        if (!tmp.reserve(tb)) return b->fail(RT_E_NOMEM, "staging buffer");
        cudaMemcpyAsync(tmp.p, c.start.data(), tb, cudaMemcpyHostToDevice, b->stream);
        void* merge_arr[3] = {arr[0], arr[1], arr[2]};
        std::string e;
        if (launch_split(true, c.elem, c.kind, c.ncol, c.n, static_cast<int32_t*>(tmp.p), merge_arr, b->stream, &e) != RT_OK)
            return b->fail(RT_E_CUDA, e);
        cudaError_t ce = cudaMemcpyAsync(tiling, tmp.p, tb, cudaMemcpyDeviceToHost, b->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(b->stream);
        if (ce != cudaSuccess) return b->fail(RT_E_CUDA, std::string("batch download: ") + cudaGetErrorString(ce));
        return RT_OK;
    });
}

rt_status rt_batch_device_tiling(rt_batch* b, int64_t index, int32_t* d_tiling, void* stream) {
    return guarded([&]() -> rt_status {
        if (!b || !d_tiling) return b ? b->fail(RT_E_INVAL, "null tiling") : RT_E_INVAL;
        if (index < 0 || index >= (int64_t)b->chains.size()) return b->fail(RT_E_INVAL, "no chain with that index");
        cudaSetDevice(b->device);
        rt_status s = upload(b);
        if (s != RT_OK) return s;
        const Chain& c = b->chains[(size_t)index];
        if (c.kind == 3) return b->fail(RT_E_INVAL, "device tilings of triangle-dimer chains are not merged on the device");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        // The merge writes every cell of the colour models' tilings.
        char* base = static_cast<char*>(b->fam[c.fam].data.p) + c.off;
        void* arr[3] = {base, base + c.per_arr, c.ncol > 2 ? base + 2 * c.per_arr : nullptr};
        std::string e;
        if (launch_split(true, c.elem, c.kind, c.ncol, c.n, d_tiling, arr, st, &e) != RT_OK) return b->fail(RT_E_CUDA, e);
        return RT_OK;
    });
}

rt_status rt_batch_get_info(rt_batch* b, rt_batch_info* info) {
    return guarded([&]() -> rt_status {
        if (!b || !info) return RT_E_INVAL;
        std::memset(info, 0, sizeof *info);
        info->chains = (int32_t)b->chains.size();
        for (int f = 0; f < kFamilies; ++f) {
            if (b->fam[f].members.empty() || !b->fam[f].planned) continue;
            info->cluster[f] = b->fam[f].plan.cl;
            info->block[f] = b->fam[f].plan.block;
            info->clusters[f] = b->fam[f].plan.clusters;
            info->sweeps_per_launch[f] = b->fam[f].plan.spl;
        }
        info->tune_ms = b->tune_ms;
        info->run_ms = b->run_ms;
        info->attempts = b->last_attempts;
        info->algorithmic_bytes = b->last_bytes;
        return RT_OK;
    });
}

}  // extern "C"
