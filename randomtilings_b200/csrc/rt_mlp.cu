// rt_mlp.cu -- training and inference kernels of the coordinate MLP
// (include/rt_b200_mlp.h).
//
// Layers 1 and 2 (128 x 128) run on the fifth-generation tensor cores: a CTA
// of four warps computes a 128 x 128 tile of C = A * B with tcgen05.mma
// (BF16 inputs, FP32 accumulator in tensor memory), A and B staged through
// shared memory 64 columns of K at a time; each GEMM names its operands'
// layouts, so one kernel serves the forward product X * W^T, the input
// gradient dZ * W and the weight gradient dZ^T * X (the last split over K,
// reduced with FP32 atomics).  Operands contiguous along K are staged with
// 16-byte asynchronous copies, the others as 8 x 8 core matrices transposed
// in registers.  Epilogues, read from tensor memory with tcgen05.ld and
// turned through shared memory so that global accesses run along rows, fuse
// bias + GELU (forward) and the GELU derivative (backward).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/rt_b200_mlp.h"
#include "rt_device.cuh"
#include "rt_guard.h"

using rtb::guarded;

namespace rtb {
namespace mlp {

constexpr int IN = RT_MLP_IN;
constexpr int H = RT_MLP_WIDTH;
// Offsets into the FP32 parameter vector.
constexpr int OW0 = 0, OB0 = OW0 + H * IN, OW1 = OB0 + H, OB1 = OW1 + H * H, OW2 = OB1 + H, OB2 = OW2 + H * H,
              OW3 = OB2 + H, OB3 = OW3 + H, NPARAM = OB3 + 1;
static_assert(NPARAM == RT_MLP_PARAMS, "parameter layout");

// GELU, tanh form: 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))).
__device__ __forceinline__ float gelu(float z) {
    const float u = 0.7978845608f * (z + 0.044715f * z * z * z);
    return 0.5f * z * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float u = 0.7978845608f * (z + 0.044715f * z * z * z);
    const float t = tanhf(u);
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * 0.7978845608f * (1.0f + 3.0f * 0.044715f * z * z);
}

// ---------------------------------------------------------------------------
// Operand access.  A matrix operand is (ptr, ld, trans): element (r, c) of
// the logical matrix is ptr[r * ld + c], or ptr[c * ld + r] when trans.
// ---------------------------------------------------------------------------
struct Op {
    const __nv_bfloat16* p;
    int ld;
    int trans;
};
__device__ __forceinline__ __nv_bfloat16 op_at(const Op& o, int r, int c) {
    return o.trans ? o.p[(size_t)c * o.ld + r] : o.p[(size_t)r * o.ld + c];
}

enum Epi : int {
    EPI_FWD = 0,     // z = acc + bias[n]; out_f = z; out_h = bf16(gelu(z))
    EPI_DGELU = 1,   // d = acc * gelu'(zin[m][n]); out_f = d; out_h = bf16(d)
    EPI_ATOMIC = 2   // out_f[m][n] += acc (weight gradients, split over K)
};

struct GemmArgs {
    Op A, B;        // C[M][N] = A[M][K] * B[K][N], N = 128
    int M, N, K;
    int ksplit;     // K range per blockIdx.z
    int epi;
    const float* bias;
    const float* zin;   // EPI_DGELU: pre-activation [M][N]
    float* out_f;       // [M][N]
    __nv_bfloat16* out_h;  // [M][N] (EPI_FWD, EPI_DGELU)
    int* err;           // set to 1 when a bounded wait gives up
};

// ---------------------------------------------------------------------------
// tcgen05 GEMM.  A CTA of four warps computes a 128 x 128 tile of C in a
// tensor-memory accumulator (128 lanes = rows, 128 FP32 columns).  K is
// walked in chunks of 64: all threads stage the A chunk (128 x 64) and the B
// chunk (as 128 n-rows x 64 k) into shared memory in the canonical K-major
// layout without swizzle -- core matrices of 8 rows x 16 bytes, the 8 core
// matrices of a row group side by side (leading byte offset 128 B, stride
// byte offset 1 KB) -- then one thread issues the four K = 16 MMAs
// (tcgen05.mma kind::f16, BF16 A and B, FP32 accumulate) and commits them to
// an mbarrier that every thread waits on before the next chunk overwrites
// the operands.  The epilogue reads the accumulator with tcgen05.ld (warp w
// owns lanes 32w..32w+31, i.e. rows) 32 columns at a time.
// ---------------------------------------------------------------------------
constexpr int TBM = 128, TBN = 128, TBK = 64;
constexpr uint32_t kTmemCols = 128;
// Instruction descriptor (PTX ISA, kind::f16): D = F32 (bits 4-5 = 1), A = B =
// BF16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at
// bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TBN >> 3) << 17) | ((uint32_t)(TBM >> 4) << 24);
constexpr unsigned long long kWaitLimit = 1ull << 28;  // mbarrier polls before giving up

// Shared-memory matrix descriptor (K-major, no swizzle): start address,
// leading byte offset 128 B (next core matrix along K), stride byte offset
// 1 KB (next group of 8 rows), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46);
}
// Byte offset of element (row r, k) of a 128 x 64 operand chunk in that layout.
__device__ __forceinline__ uint32_t chunk_off(int r, int k) {
    return (uint32_t)(((r >> 3) * (TBK / 8) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (unsigned long long it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
    // src_bytes 0: the 16 bytes are zero-filled and nothing is read
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

// Stages rows [r0, r0 + 128) x k [k0, k_end) of a logical operand whose
// element (r, k) is p[r * ld + k] into the canonical K-major layout: every
// 16-byte group of 8 consecutive k is one asynchronous copy (zero-filled
// for rows >= rlim), so all of a chunk's loads are in flight together; a
// group cut by k_end is assembled element by element.
__device__ __forceinline__ void stage_kcontig(uint32_t sdst, unsigned char* dst, const __nv_bfloat16* p, int ld,
                                              int r0, int rlim, int k0, int k_end) {
    const uint16_t* q = reinterpret_cast<const uint16_t*>(p);
    for (int e = threadIdx.x; e < TBM * (TBK / 8); e += 128) {
        const int r = e / (TBK / 8), k8 = (e % (TBK / 8)) * 8;
        const int gr = r0 + r, gk = k0 + k8;
        const uint32_t off = chunk_off(r, k8);
        if (gr >= rlim || gk + 8 <= k_end) {
            const bool in = gr < rlim;
            cp_async16(sdst + off, in ? (const void*)(q + (size_t)gr * ld + gk) : (const void*)q, in ? 16u : 0u);
        } else {
            uint32_t w[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const uint32_t lo = gk + 2 * x < k_end ? q[(size_t)gr * ld + gk + 2 * x] : 0u;
                const uint32_t hi = gk + 2 * x + 1 < k_end ? q[(size_t)gr * ld + gk + 2 * x + 1] : 0u;
                w[x] = lo | hi << 16;
            }
            *reinterpret_cast<uint4*>(dst + off) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// The same chunk of an operand stored the other way, element (r, k) at
// p[k * ld + r].  Thread t builds core matrix (t / 8, t % 8) -- rows
// 8 (t / 8) .. +7, k 8 (t % 8) .. +7: eight 16-byte loads along r, an 8 x 8
// transpose of 16-bit values in registers, eight 16-byte stores that fill
// the core matrix's 128 contiguous bytes.
__device__ __forceinline__ void stage_mncontig(unsigned char* dst, const __nv_bfloat16* p, int ld, int r0, int rlim,
                                               int k0, int k_end) {
    const uint16_t* q = reinterpret_cast<const uint16_t*>(p);
    const int rg = threadIdx.x >> 3, kg = threadIdx.x & 7;
    const int gr = r0 + 8 * rg, gkb = k0 + 8 * kg;
    uint32_t w[8][4];  // w[kk]: r = gr .. gr + 7 at k = gkb + kk, two per word
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        const int gk = gkb + kk;
        if (gk < k_end && gr + 8 <= rlim) {
            const uint4 v = *reinterpret_cast<const uint4*>(q + (size_t)gk * ld + gr);
            w[kk][0] = v.x, w[kk][1] = v.y, w[kk][2] = v.z, w[kk][3] = v.w;
        } else {
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const uint32_t lo = (gk < k_end && gr + 2 * x < rlim) ? q[(size_t)gk * ld + gr + 2 * x] : 0u;
                const uint32_t hi = (gk < k_end && gr + 2 * x + 1 < rlim) ? q[(size_t)gk * ld + gr + 2 * x + 1] : 0u;
                w[kk][x] = lo | hi << 16;
            }
        }
    }
#pragma unroll
    for (int rr = 0; rr < 8; ++rr) {
        uint32_t o[4];
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            const uint32_t a = (w[2 * x][rr >> 1] >> (16 * (rr & 1))) & 0xFFFFu;
            const uint32_t b = (w[2 * x + 1][rr >> 1] >> (16 * (rr & 1))) & 0xFFFFu;
            o[x] = a | b << 16;
        }
        *reinterpret_cast<uint4*>(dst + chunk_off(8 * rg + rr, 8 * kg)) = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

__global__ void __launch_bounds__(128, 1) gemm_tc(const __grid_constant__ GemmArgs g) {
    // A and B chunks; after the last MMA the epilogue's per-warp staging
    __shared__ __align__(128) unsigned char sAB[(TBM + TBN) * TBK * 2];
    unsigned char* sA = sAB;
    unsigned char* sB = sAB + TBM * TBK * 2;
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TBM;
    const int k_begin = blockIdx.z * g.ksplit, k_end = min(g.K, k_begin + g.ksplit);
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(sA), sb = (uint32_t)__cvta_generic_to_shared(sB);
    const uint32_t mb = (uint32_t)__cvta_generic_to_shared(&mbar);

    if (warp == 0) {
        const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&tmem_slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    uint32_t parity = 0;
    bool first = true;
    for (int k0 = k_begin; k0 < k_end; k0 += TBK) {
        // Stage A as (m, k) and B as (n, k) = B[k][n]; zero outside the matrices.
        // A(m, k) is contiguous along k unless A is transposed; B(k, n) as (n, k)
        // is contiguous along k when B is transposed.
        if (g.A.trans == 0)
            stage_kcontig(sa, sA, g.A.p, g.A.ld, m0, g.M, k0, k_end);
        else
            stage_mncontig(sA, g.A.p, g.A.ld, m0, g.M, k0, k_end);
        if (g.B.trans != 0)
            stage_kcontig(sb, sB, g.B.p, g.B.ld, 0, g.N, k0, k_end);
        else
            stage_mncontig(sB, g.B.p, g.B.ld, 0, g.N, k0, k_end);
        asm volatile("cp.async.wait_all;" ::: "memory");
        // shared-memory writes -> visible to the tensor core's async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < TBK / 16; ++kk) {
                // K = 16 per MMA: two core matrices along K = 256 bytes
                const uint64_t da = smem_desc(sa + 256u * kk), db = smem_desc(sb + 256u * kk);
                const uint32_t acc = (first && kk == 0) ? 0u : 1u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                         : "memory");
        }
        first = false;
        if (!mbar_wait(mb, parity)) {
            s_fail = 1;  // racy but every writer writes 1
            atomicOr(g.err, 1);
        }
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
        if (s_fail) break;
    }

    if (!s_fail && !first) {
        // Epilogue: this warp's 32 rows (TMEM lanes 32w .. 32w + 31), 32
        // columns per tcgen05.ld (lane = row), turned through shared memory
        // (32 x 33 floats per warp) so that the global loads and stores run
        // along rows: lane = column.
        float* stg = reinterpret_cast<float*>(sAB) + warp * (32 * 33);
        const int mrow = m0 + 32 * warp;
#pragma unroll 1
        for (int c0 = 0; c0 < TBN; c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int x = 0; x < 32; ++x) stg[lane * 33 + x] = __uint_as_float(v[x]);
            __syncwarp();
            const int n = c0 + lane;
            const float b = (g.epi == EPI_FWD && n < g.N) ? g.bias[n] : 0.0f;
#pragma unroll 4
            for (int rr = 0; rr < 32; ++rr) {
                const int m = mrow + rr;
                if (m >= g.M || n >= g.N) continue;
                const float acc = stg[rr * 33 + lane];
                const size_t at = (size_t)m * g.N + n;
                if (g.epi == EPI_FWD) {
                    const float z = acc + b;
                    g.out_f[at] = z;
                    g.out_h[at] = __float2bfloat16(gelu(z));
                } else if (g.epi == EPI_DGELU) {
                    const float dd = acc * gelu_grad(g.zin[at]);
                    g.out_f[at] = dd;
                    g.out_h[at] = __float2bfloat16(dd);
                } else {
                    atomicAdd(g.out_f + at, acc);
                }
            }
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        if (s_fail) {
            // the MMAs may still be running: wait for them (bounded) before freeing their accumulator
            mbar_wait(mb, parity ^ 1u);
        }
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// Layer 0 (IN -> H), FP32: z0 = x W0^T + b0, h1 = bf16(gelu(z0)).
__global__ void layer0_fwd(const float* __restrict__ x, const float* __restrict__ P, int n, float* z0,
                           __nv_bfloat16* h1) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * H) return;
    const int r = (int)(e / H), o = (int)(e % H);
    float z = P[OB0 + o];
#pragma unroll
    for (int k = 0; k < IN; ++k) z += P[OW0 + o * IN + k] * x[(size_t)r * IN + k];
    z0[e] = z;
    h1[e] = __float2bfloat16(gelu(z));
}

// Layer 3 (H -> 1), FP32, one warp per row: y = h3 . W3 + b3; with a target,
// also dy = 2 (y - t) / n and the mean squared error (one atomic per block).
__global__ void layer3_fwd(const __nv_bfloat16* __restrict__ h3, const float* __restrict__ P, int n, float* y,
                           const float* __restrict__ target, float* dy, float* loss) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    __shared__ float part[32];
    float err = 0.0f;
    if (row < n) {
        float s = 0.0f;
        for (int k = lane; k < H; k += 32) s += __bfloat162float(h3[(size_t)row * H + k]) * P[OW3 + k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        const float v = s + P[OB3];
        if (lane == 0) {
            if (y) y[row] = v;
            if (target) {
                const float e = v - target[row];
                dy[row] = 2.0f * e / (float)n;
                err = e * e / (float)n;
            }
        }
    }
    if (!target) return;
    if (lane == 0) part[threadIdx.x >> 5] = err;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        atomicAdd(loss, t);
    }
}

// Backward of layer 3, elementwise: dz2 = dy W3 * gelu'(z2) (FP32 and BF16).
__global__ void layer3_bwd(const float* __restrict__ z2, const float* __restrict__ dy, const float* __restrict__ P,
                           int n, float* dz2, __nv_bfloat16* dz2h) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * H) return;
    const int r = (int)(e / H), k = (int)(e % H);
    const float g = dy[r] * P[OW3 + k] * gelu_grad(z2[e]);
    dz2[e] = g;
    dz2h[e] = __float2bfloat16(g);
}

// Output-layer weights: G[W3][k] = sum_r dy[r] h3[r][k] (block k < H), and
// G[b3] = sum_r dy[r] (block H).
__global__ void layer3_wgrad(const __nv_bfloat16* __restrict__ h3, const float* __restrict__ dy, int n, float* G) {
    const int k = blockIdx.x;
    float s = 0.0f;
    for (int r = threadIdx.x; r < n; r += blockDim.x)
        s += dy[r] * (k < H ? __bfloat162float(h3[(size_t)r * H + k]) : 1.0f);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        G[k < H ? OW3 + k : OB3] += t;
    }
}

// Bias gradient: G[off + c] += sum_r d[r][c].
__global__ void bias_grad(const float* __restrict__ d, int n, float* G, int off) {
    const int c = blockIdx.x;
    float s = 0.0f;
    for (int r = threadIdx.x; r < n; r += blockDim.x) s += d[(size_t)r * H + c];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        G[off + c] += t;
    }
}

// Layer 0 weights: G[W0] += dz0^T x, G[b0] by bias_grad.
__global__ void layer0_wgrad(const float* __restrict__ dz0, const float* __restrict__ x, int n, float* G) {
    const int o = blockIdx.x, k = threadIdx.x & 7, part = threadIdx.x >> 3;  // 256 threads: 32 parts x 8 inputs
    float s = 0.0f;
    for (int r = part; r < n; r += 32) s += dz0[(size_t)r * H + o] * x[(size_t)r * IN + k];
    __shared__ float red[32][IN];
    red[part][k] = s;
    __syncthreads();
    if (part == 0) {
        float t = 0.0f;
        for (int p = 0; p < 32; ++p) t += red[p][k];
        G[OW0 + o * IN + k] += t;
    }
}

// BF16 copies of W1, W2 for the tensor-core GEMMs.
__global__ void to_bf16(const float* __restrict__ P, __nv_bfloat16* w1, __nv_bfloat16* w2) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= H * H) return;
    w1[e] = __float2bfloat16(P[OW1 + e]);
    w2[e] = __float2bfloat16(P[OW2 + e]);
}

__global__ void adam(float* P, const float* __restrict__ G, float* m1, float* m2, int n, float lr, float b1t,
                     float b2t) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float g = G[e];
    const float a = 0.9f * m1[e] + 0.1f * g;
    const float b = 0.999f * m2[e] + 0.001f * g * g;
    m1[e] = a;
    m2[e] = b;
    const float mh = a / (1.0f - b1t), vh = b / (1.0f - b2t);
    P[e] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

// Batch rows drawn with replacement: row = floor(u * rows) with u from
// Philox keyed by (seed, step).
__global__ void gather_batch(const float* __restrict__ X, const float* __restrict__ T, int64_t rows, int batch,
                             uint64_t seed, int64_t step, float* xb, float* tb) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    const uint4 w = philox4((uint32_t)b, (uint32_t)step, (uint32_t)((uint64_t)step >> 32), 0x4d4c50u,
                            (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t r64 = (((uint64_t)w.x << 32) | w.y) % (uint64_t)rows;
#pragma unroll
    for (int k = 0; k < IN; ++k) xb[(size_t)b * IN + k] = X[r64 * IN + k];
    tb[b] = T[r64];
}

}  // namespace mlp
}  // namespace rtb

using namespace rtb::mlp;

struct rt_mlp {
    int device = 0;
    cudaStream_t s = nullptr;
    float *P = nullptr, *G = nullptr, *M1 = nullptr, *M2 = nullptr;
    __nv_bfloat16 *w1 = nullptr, *w2 = nullptr;
    int64_t adam_t = 0;
    // workspace for batches of up to `cap` rows
    int64_t cap = 0;
    float *x = nullptr, *t = nullptr, *y = nullptr, *dy = nullptr, *z0 = nullptr, *z1 = nullptr, *z2 = nullptr,
          *d0 = nullptr, *d1 = nullptr, *d2 = nullptr, *loss = nullptr;
    __nv_bfloat16 *h1 = nullptr, *h2 = nullptr, *h3 = nullptr, *d1h = nullptr, *d2h = nullptr;
    float *X = nullptr, *T = nullptr;
    int64_t rows = 0;
    int* err = nullptr;  // device: set when a GEMM's bounded wait gave up
};

namespace {

void free_ws(rt_mlp* m) {
    void* ps[] = {m->x, m->t, m->y, m->dy, m->z0, m->z1, m->z2, m->d0, m->d1, m->d2, m->h1, m->h2, m->h3, m->d1h, m->d2h};
    for (void* p : ps)
        if (p) cudaFree(p);
    m->x = m->t = m->y = m->dy = m->z0 = m->z1 = m->z2 = m->d0 = m->d1 = m->d2 = nullptr;
    m->h1 = m->h2 = m->h3 = m->d1h = m->d2h = nullptr;
    m->cap = 0;
}

bool reserve(rt_mlp* m, int64_t n) {
    if (n <= m->cap) return true;
    free_ws(m);
    const size_t nh = (size_t)n * H;
    bool ok = cudaMalloc(&m->x, (size_t)n * IN * 4) == cudaSuccess && cudaMalloc(&m->t, (size_t)n * 4) == cudaSuccess &&
              cudaMalloc(&m->y, (size_t)n * 4) == cudaSuccess && cudaMalloc(&m->dy, (size_t)n * 4) == cudaSuccess &&
              cudaMalloc(&m->z0, nh * 4) == cudaSuccess && cudaMalloc(&m->z1, nh * 4) == cudaSuccess &&
              cudaMalloc(&m->z2, nh * 4) == cudaSuccess && cudaMalloc(&m->d0, nh * 4) == cudaSuccess &&
              cudaMalloc(&m->d1, nh * 4) == cudaSuccess && cudaMalloc(&m->d2, nh * 4) == cudaSuccess &&
              cudaMalloc(&m->h1, nh * 2) == cudaSuccess && cudaMalloc(&m->h2, nh * 2) == cudaSuccess &&
              cudaMalloc(&m->h3, nh * 2) == cudaSuccess && cudaMalloc(&m->d1h, nh * 2) == cudaSuccess &&
              cudaMalloc(&m->d2h, nh * 2) == cudaSuccess;
    if (!ok) {
        free_ws(m);
        return false;
    }
    m->cap = n;
    return true;
}

GemmArgs gemm(Op A, Op B, int M, int N, int K, int epi) {
    GemmArgs g;
    std::memset(&g, 0, sizeof g);
    g.A = A;
    g.B = B;
    g.M = M;
    g.N = N;
    g.K = K;
    g.ksplit = K;
    g.epi = epi;
    return g;
}

// N is always the hidden width (128 = one tile); M rows in tiles of 128, K
// split over blockIdx.z for the weight gradients.
void launch_gemm(rt_mlp* m, GemmArgs g, int splits, cudaStream_t s) {
    g.err = m->err;
    dim3 grid(1, (g.M + TBM - 1) / TBM, splits);
    gemm_tc<<<grid, 128, 0, s>>>(g);
}

// Forward pass of the n rows in m->x; with `with_target`, also the loss and
// dy.  Returns y in m->y.
void forward(rt_mlp* m, int n, bool with_target) {
    cudaStream_t s = m->s;
    const int nh = n * H;
    layer0_fwd<<<(nh + 255) / 256, 256, 0, s>>>(m->x, m->P, n, m->z0, m->h1);
    // z1 = h1 W1^T + b1: A = h1 [n][H], B(k, o) = W1[o][k] -> (w1, H, trans)
    GemmArgs g = gemm(Op{m->h1, H, 0}, Op{m->w1, H, 1}, n, H, H, EPI_FWD);
    g.bias = m->P + OB1;
    g.out_f = m->z1;
    g.out_h = m->h2;
    launch_gemm(m, g, 1, s);
    g = gemm(Op{m->h2, H, 0}, Op{m->w2, H, 1}, n, H, H, EPI_FWD);
    g.bias = m->P + OB2;
    g.out_f = m->z2;
    g.out_h = m->h3;
    launch_gemm(m, g, 1, s);
    if (with_target) cudaMemsetAsync(m->loss, 0, 4, s);
    layer3_fwd<<<(n + 7) / 8, 256, 0, s>>>(m->h3, m->P, n, m->y, with_target ? m->t : nullptr, m->dy, m->loss);
}

// Gradient of the loss over the batch in m->x / m->t into m->G (zeroed here).
void backward(rt_mlp* m, int n) {
    cudaStream_t s = m->s;
    const int nh = n * H;
    cudaMemsetAsync(m->G, 0, NPARAM * 4, s);
    layer3_wgrad<<<H + 1, 256, 0, s>>>(m->h3, m->dy, n, m->G);
    layer3_bwd<<<(nh + 255) / 256, 256, 0, s>>>(m->z2, m->dy, m->P, n, m->d2, m->d2h);
    const int splits = (n + 255) / 256;  // weight-gradient GEMMs: K = rows, 256 per CTA
    const int ks = ((n + splits - 1) / splits + TBK - 1) / TBK * TBK;
    // dW2 = dz2^T h2: A(o, r) = dz2[r][o] -> (d2h, H, trans); B(r, k) = h2[r][k]
    GemmArgs g = gemm(Op{m->d2h, H, 1}, Op{m->h2, H, 0}, H, H, n, EPI_ATOMIC);
    g.ksplit = ks;
    g.out_f = m->G + OW2;
    launch_gemm(m, g, splits, s);
    bias_grad<<<H, 256, 0, s>>>(m->d2, n, m->G, OB2);
    // dz1 = (dz2 W2) * gelu'(z1): A = dz2 [n][H], B(o, k) = W2[o][k]
    g = gemm(Op{m->d2h, H, 0}, Op{m->w2, H, 0}, n, H, H, EPI_DGELU);
    g.zin = m->z1;
    g.out_f = m->d1;
    g.out_h = m->d1h;
    launch_gemm(m, g, 1, s);
    g = gemm(Op{m->d1h, H, 1}, Op{m->h1, H, 0}, H, H, n, EPI_ATOMIC);
    g.ksplit = ks;
    g.out_f = m->G + OW1;
    launch_gemm(m, g, splits, s);
    bias_grad<<<H, 256, 0, s>>>(m->d1, n, m->G, OB1);
    g = gemm(Op{m->d1h, H, 0}, Op{m->w1, H, 0}, n, H, H, EPI_DGELU);
    g.zin = m->z0;
    g.out_f = m->d0;
    g.out_h = m->h3;  // scratch: the BF16 copy of dz0 is not needed
    launch_gemm(m, g, 1, s);
    layer0_wgrad<<<H, 256, 0, s>>>(m->d0, m->x, n, m->G);
    bias_grad<<<H, 256, 0, s>>>(m->d0, n, m->G, OB0);
}

rt_status sync(rt_mlp* m) {
    if (cudaStreamSynchronize(m->s) != cudaSuccess) return RT_E_CUDA;
    int e = 0;
    if (cudaMemcpy(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return RT_E_CUDA;
    return e ? RT_E_TIMEOUT : RT_OK;
}

}  // namespace

extern "C" {

rt_status rt_mlp_create(int32_t device, uint64_t seed, rt_mlp** out) {
    return guarded([&]() -> rt_status {
        if (!out) return RT_E_INVAL;
        *out = nullptr;
        if (cudaSetDevice(device) != cudaSuccess) return RT_E_NODEVICE;
        rt_mlp* m = new rt_mlp();
        m->device = device;
        bool ok = cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaMalloc(&m->P, NPARAM * 4) == cudaSuccess && cudaMalloc(&m->G, NPARAM * 4) == cudaSuccess &&
                  cudaMalloc(&m->M1, NPARAM * 4) == cudaSuccess && cudaMalloc(&m->M2, NPARAM * 4) == cudaSuccess &&
                  cudaMalloc(&m->w1, H * H * 2) == cudaSuccess && cudaMalloc(&m->w2, H * H * 2) == cudaSuccess &&
                  cudaMalloc(&m->loss, 4) == cudaSuccess && cudaMalloc(&m->err, sizeof(int)) == cudaSuccess &&
                  cudaMemset(m->err, 0, sizeof(int)) == cudaSuccess;
        if (!ok) {
            rt_mlp_destroy(m);
            return RT_E_NOMEM;
        }
        // Initialisation: weights uniform in +-1/sqrt(fan_in) from Philox(seed), biases 0.
        std::vector<float> p(NPARAM, 0.0f);
        auto fill = [&](int off, int count, int fan_in) {
            const float a = 1.0f / std::sqrt((float)fan_in);
            for (int i = 0; i < count; ++i) {
                const uint4 w = rtb::philox4((uint32_t)(off + i), 0x494e4954u, 0, 0, (uint32_t)seed, (uint32_t)(seed >> 32));
                p[off + i] = a * (2.0f * ((float)(w.x >> 8) * (1.0f / 16777216.0f)) - 1.0f);
            }
        };
        fill(OW0, H * IN, IN);
        fill(OW1, H * H, H);
        fill(OW2, H * H, H);
        fill(OW3, H, H);
        *out = m;
        return rt_mlp_set_params(m, p.data());
    });
}

rt_status rt_mlp_destroy(rt_mlp* m) {
    return guarded([&]() -> rt_status {
        if (!m) return RT_E_INVAL;
        cudaSetDevice(m->device);
        if (m->s) cudaStreamSynchronize(m->s);
        free_ws(m);
        void* ps[] = {m->P, m->G, m->M1, m->M2, m->w1, m->w2, m->loss, m->X, m->T, m->err};
        for (void* p : ps)
            if (p) cudaFree(p);
        if (m->s) cudaStreamDestroy(m->s);
        delete m;
        return RT_OK;
    });
}

rt_status rt_mlp_get_params(rt_mlp* m, float* params) {
    return guarded([&]() -> rt_status {
        if (!m || !params) return RT_E_INVAL;
        cudaSetDevice(m->device);
        if (cudaMemcpyAsync(params, m->P, NPARAM * 4, cudaMemcpyDeviceToHost, m->s) != cudaSuccess) return RT_E_CUDA;
        return sync(m);
    });
}

rt_status rt_mlp_set_params(rt_mlp* m, const float* params) {
    return guarded([&]() -> rt_status {
        if (!m || !params) return RT_E_INVAL;
        cudaSetDevice(m->device);
        cudaMemcpyAsync(m->P, params, NPARAM * 4, cudaMemcpyHostToDevice, m->s);
        cudaMemsetAsync(m->M1, 0, NPARAM * 4, m->s);
        cudaMemsetAsync(m->M2, 0, NPARAM * 4, m->s);
        m->adam_t = 0;
        to_bf16<<<(H * H + 255) / 256, 256, 0, m->s>>>(m->P, m->w1, m->w2);
        return sync(m);
    });
}

rt_status rt_mlp_predict(rt_mlp* m, const float* x, int64_t n, float* y) {
    return guarded([&]() -> rt_status {
        if (!m || !x || !y || n < 0) return RT_E_INVAL;
        cudaSetDevice(m->device);
        const int64_t chunk = 1 << 18;
        for (int64_t r0 = 0; r0 < n; r0 += chunk) {
            const int rn = (int)std::min<int64_t>(chunk, n - r0);
            if (!reserve(m, rn)) return RT_E_NOMEM;
            cudaMemcpyAsync(m->x, x + r0 * IN, (size_t)rn * IN * 4, cudaMemcpyHostToDevice, m->s);
            forward(m, rn, false);
            cudaMemcpyAsync(y + r0, m->y, (size_t)rn * 4, cudaMemcpyDeviceToHost, m->s);
            rt_status st = sync(m);
            if (st != RT_OK) return st;
        }
        return RT_OK;
    });
}

rt_status rt_mlp_loss_grad(rt_mlp* m, const float* x, const float* target, int64_t n, float* loss, float* grad) {
    return guarded([&]() -> rt_status {
        if (!m || !x || !target || n <= 0 || n > (1 << 22)) return RT_E_INVAL;
        cudaSetDevice(m->device);
        if (!reserve(m, n)) return RT_E_NOMEM;
        cudaMemcpyAsync(m->x, x, (size_t)n * IN * 4, cudaMemcpyHostToDevice, m->s);
        cudaMemcpyAsync(m->t, target, (size_t)n * 4, cudaMemcpyHostToDevice, m->s);
        forward(m, (int)n, true);
        backward(m, (int)n);
        if (loss) cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->s);
        if (grad) cudaMemcpyAsync(grad, m->G, NPARAM * 4, cudaMemcpyDeviceToHost, m->s);
        return sync(m);
    });
}

rt_status rt_mlp_set_data(rt_mlp* m, const float* x, const float* target, int64_t n) {
    return guarded([&]() -> rt_status {
        // At most 2^40 rows, so that no byte count below can wrap.
        if (!m || !x || !target || n <= 0 || n > ((int64_t)1 << 40)) return RT_E_INVAL;
        cudaSetDevice(m->device);
        if (m->X) cudaFree(m->X);
        if (m->T) cudaFree(m->T);
        m->X = m->T = nullptr;
        m->rows = 0;
        // Both buffers or neither: training checks for both.
        float *X = nullptr, *T = nullptr;
        const bool okx = cudaMalloc(&X, (size_t)n * IN * 4) == cudaSuccess;
        const bool okt = okx && cudaMalloc(&T, (size_t)n * 4) == cudaSuccess;
        if (!okt) {
            if (okx) cudaFree(X);
            cudaGetLastError();
            return RT_E_NOMEM;
        }
        m->X = X;
        m->T = T;
        cudaMemcpyAsync(m->X, x, (size_t)n * IN * 4, cudaMemcpyHostToDevice, m->s);
        cudaMemcpyAsync(m->T, target, (size_t)n * 4, cudaMemcpyHostToDevice, m->s);
        m->rows = n;
        return sync(m);
    });
}

rt_status rt_mlp_train(rt_mlp* m, int64_t steps, int32_t batch, float lr, uint64_t seed, float* loss) {
    return guarded([&]() -> rt_status {
        if (!m || steps < 0 || batch <= 0 || batch > (1 << 22) || !m->X || !m->T || m->rows <= 0) return RT_E_INVAL;
        cudaSetDevice(m->device);
        if (!reserve(m, batch)) return RT_E_NOMEM;
        for (int64_t k = 0; k < steps; ++k) {
            gather_batch<<<(batch + 255) / 256, 256, 0, m->s>>>(m->X, m->T, m->rows, batch, seed, m->adam_t, m->x, m->t);
            forward(m, batch, true);
            backward(m, batch);
            ++m->adam_t;
            const float b1t = std::pow(0.9f, (float)m->adam_t), b2t = std::pow(0.999f, (float)m->adam_t);
            adam<<<(NPARAM + 255) / 256, 256, 0, m->s>>>(m->P, m->G, m->M1, m->M2, NPARAM, lr, b1t, b2t);
            to_bf16<<<(H * H + 255) / 256, 256, 0, m->s>>>(m->P, m->w1, m->w2);
        }
        if (loss) cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->s);
        return sync(m);
    });
}

}  // extern "C"
