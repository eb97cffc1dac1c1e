// rt_extremal.cu -- extremal tilings and their height functions on the GPU
// (include/rt_b200_extremal.h).
//
// The reference builds MaxTiling / MinTiling by a breadth-first flood on the
// host (DominoTiler.cpp:214-399, LozengeTiler.cpp:140-318): from the boundary
// heights, an interior vertex takes the height of the first vertex that
// reaches it along an edge whose orientation step is +1 (maximal function),
// plus one -- i.e. h(w) = min over such in-neighbours v of h(v) + 1, the
// shortest-path fixpoint -- and symmetrically for the minimal function with
// steps of -1.  Here both fixpoints are reached by a monotone relaxation:
// values start at +-kBig inside, only ever move towards the fixpoint, and a
// read racing a write sees an old or a new value, both bounds, so any update
// order converges to the same unique function.
//
// Layout: vertex kinds (uint8, 0 outside / 1 interior / 2 boundary) and the
// two height arrays (int32) on the n x n vertex grid, row-major.  The
// relaxation runs over 32 x 64-vertex tiles: a CTA loads its tile and a
// one-vertex halo into shared memory, each thread keeps an 8-vertex column
// segment in registers and sweeps it down and up, the CTA iterating until
// nothing changes; then it writes back what changed and marks for the next
// pass the neighbours that read a changed border value.  Tiles not marked
// return at once, so a pass costs in proportion to the moving front.
#include <cuda_runtime.h>

#include <chrono>
#include <climits>
#include <cstring>
#include <vector>

#include "../../include/rt_b200_extremal.h"
#include "rt_internal.h"
#include "rt_guard.h"

using rtb::guarded;

namespace rtb {
namespace {

constexpr int32_t kBig = 0x3FFFFFFF;  // "not reached": +kBig (maximal), -kBig (minimal); kBig + 1 cannot overflow
constexpr int XR = 32, XC = 64;       // tile rows x columns
constexpr int XT = 256;               // 64 columns x 4 groups of 8 rows
constexpr int XPR = XR + 2, XPC = XC + 2;
constexpr int kLocalCap = 4096;       // sweeps of one tile per pass (the tile is marked again if it is cut short)
constexpr int kGroup = 8;             // passes between two reads of the change counters

__constant__ int c_ldi[6] = {0, -1, -1, 0, 1, 1};
__constant__ int c_ldj[6] = {1, 1, 0, -1, -1, 0};
__constant__ int c_lbit[6] = {8, 2, 1, 4, 16, 32};
// (row offset, offset from 2j) of the two triangles beside lozenge edge nb.
__constant__ int c_lface[6][4] = {{0, 0, -1, 1}, {-1, 1, -1, 0}, {-1, 0, -1, -1},
                                  {-1, -1, 0, -2}, {0, -2, 0, -1}, {0, -1, 0, 0}};
__constant__ int c_ddi[4] = {1, -1, 0, 0};
__constant__ int c_ddj[4] = {0, 0, 1, -1};
__constant__ int c_dbit[4] = {2, 1, 8, 4};

__device__ __forceinline__ int dface(const int32_t* __restrict__ d, int m, int i, int j) {
    return (i >= 0 && j >= 0 && i < m && j < m) ? d[(int64_t)i * m + j] : 0;
}
__device__ __forceinline__ int lface(const int32_t* __restrict__ d, int m, int r, int c) {
    return (r >= 0 && c >= 0 && r < m && c < 2 * m) ? d[(int64_t)r * 2 * m + c] : 0;
}

// Vertex kinds (DomainToVertices, DominoTiler.cpp:479-506,
// LozengeTiler.cpp:405-430) and the initial heights.
template <bool DOM>
__global__ void ext_classify(const int32_t* __restrict__ d, int m, uint8_t* kind, int32_t* hx, int32_t* hn) {
    const int n = m + 1;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (int64_t)n * n) return;
    const int i = (int)(v / n), j = (int)(v % n);
    int k;
    if (DOM) {
        if (i == 0 || j == 0 || i == m || j == m) {
            const int i0 = i - (i == m), i1 = i - 1 + (i == 0), j0 = j - (j == m), j1 = j - 1 + (j == 0);
            k = (dface(d, m, i0, j0) || dface(d, m, i1, j0) || dface(d, m, i0, j1) || dface(d, m, i1, j1)) ? 2 : 0;
        } else {
            const int s = (dface(d, m, i - 1, j - 1) != 0) + (dface(d, m, i - 1, j) != 0) +
                          (dface(d, m, i, j - 1) != 0) + (dface(d, m, i, j) != 0);
            k = s == 4 ? 1 : s > 0 ? 2 : 0;
        }
    } else {
        k = 0;
        if (i >= 1 && j >= 1 && i < m && j < m) {
            const int s = (lface(d, m, i, 2 * j) != 0) + (lface(d, m, i, 2 * j - 1) != 0) +
                          (lface(d, m, i, 2 * j - 2) != 0) + (lface(d, m, i - 1, 2 * j) != 0) +
                          (lface(d, m, i - 1, 2 * j + 1) != 0) + (lface(d, m, i - 1, 2 * j - 1) != 0);
            k = s == 6 ? 1 : s > 0 ? 2 : 0;
        }
    }
    kind[v] = (uint8_t)k;
    hx[v] = kBig;
    hn[v] = -kBig;
}

__global__ void ext_seed(const int64_t* __restrict__ idx, const int32_t* __restrict__ h, int64_t cnt, int32_t* hx,
                         int32_t* hn) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cnt) return;
    hx[idx[k]] = h[k];
    hn[idx[k]] = h[k];
}

// One pass over the marked tiles.  Dominoes: an even vertex (i + j even)
// steps +1 along horizontal edges and -1 along vertical ones, an odd vertex
// the reverse (DominoTiler.cpp:221-231), so the maximal function of an even
// vertex comes from its vertical neighbours and the minimal one from its
// horizontal neighbours.  Lozenges: edges (0,+1), (-1,0), (+1,-1) step -1
// from the vertex and (-1,+1), (0,-1), (+1,0) step +1 (LozengeTiler.h:12-16).
template <bool DOM>
__global__ void __launch_bounds__(XT) ext_relax(const uint8_t* __restrict__ kind, int32_t* hx, int32_t* hn, int n,
                                                int tiles_x, int tiles_y, uint8_t* dirty_in, uint8_t* dirty_out,
                                                unsigned* changed_tiles) {
    const int tile = blockIdx.x;
    if (!dirty_in[tile]) return;  // the same answer for the whole block
    __shared__ int32_t sx[XPR][XPC], sn[XPR][XPC];
    __shared__ uint8_t sk[XPR][XPC];
    __shared__ unsigned s_mark;
    const int ty = tile / tiles_x, tx = tile % tiles_x;
    const int r0 = ty * XR, c0 = tx * XC;
    for (int e = threadIdx.x; e < XPR * XPC; e += XT) {
        const int r = e / XPC, c = e % XPC;
        const int gi = r0 + r - 1, gj = c0 + c - 1;
        uint8_t k = 0;
        int32_t a = kBig, b = -kBig;
        if (gi >= 0 && gj >= 0 && gi < n && gj < n) {
            const int64_t g = (int64_t)gi * n + gj;
            k = kind[g];
            a = hx[g];
            b = hn[g];
        }
        sk[r][c] = k;
        sx[r][c] = a;
        sn[r][c] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dirty_in[tile] = 0;  // nothing else writes dirty_in during this pass
        s_mark = 0;          // read after the barriers of the sweep loop
    }

    // Thread: column c, rows 8 grp .. 8 grp + 7 of the tile, kept in registers
    // (x = maximal, y = minimal function).  An iteration reads the values it
    // needs from the neighbouring columns and the rows just outside its
    // segment, sweeps the segment down and then up (vertical neighbours come
    // from registers, already updated), and publishes what changed.
    const int c = threadIdx.x & (XC - 1), grp = threadIdx.x / XC;
    const int cc = c + 1, rb = 8 * grp + 1, gj = c0 + c;
    const int p0 = (r0 + 8 * grp + gj) & 1;  // parity of the segment's first vertex (dominoes)
    int32_t x[8], y[8];
    uint32_t mine = 0;  // bit k: vertex k of the segment is interior
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = sx[rb + k][cc];
        y[k] = sn[rb + k][cc];
        if (sk[rb + k][cc] == 1) mine |= 1u << k;
    }
    uint32_t wrote = 0;  // bit k: x[k] lowered; bit k + 8: y[k] raised
    bool capped = true;
    for (int it = 0; it < kLocalCap; ++it) {
        uint32_t chg = 0;
        if (mine) {
            // candidates from the other columns, fixed for this iteration
            int32_t ax[8], ay[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int r = rb + k;
                if (DOM) {
                    // even vertex: y from left / right; odd vertex: x from left / right
                    if (((p0 ^ k) & 1) == 0) {
                        ay[k] = max(sn[r][cc - 1], sn[r][cc + 1]);
                        ax[k] = kBig;
                    } else {
                        ax[k] = min(sx[r][cc - 1], sx[r][cc + 1]);
                        ay[k] = -kBig;
                    }
                } else {
                    ax[k] = min(sx[r][cc + 1], sx[r + 1][cc - 1]);  // (0,+1), (+1,-1)
                    ay[k] = max(sn[r - 1][cc + 1], sn[r][cc - 1]);  // (-1,+1), (0,-1)
                }
            }
            const int32_t xt = sx[rb - 1][cc], xb = sx[rb + 8][cc], yt = sn[rb - 1][cc], yb = sn[rb + 8][cc];
#pragma unroll
            for (int sweep = 0; sweep < 2; ++sweep) {
#pragma unroll
                for (int kk = 0; kk < 8; ++kk) {
                    const int k = sweep == 0 ? kk : 7 - kk;
                    if (!(mine >> k & 1u)) continue;
                    const int32_t xu = k > 0 ? x[k - 1] : xt, xd = k < 7 ? x[k + 1] : xb;
                    const int32_t yu = k > 0 ? y[k - 1] : yt, yd = k < 7 ? y[k + 1] : yb;
                    int32_t nx, ny;
                    if (DOM) {
                        if (((p0 ^ k) & 1) == 0) {
                            nx = min(xu, xd) + 1;
                            ny = ay[k] - 1;
                        } else {
                            nx = ax[k] + 1;
                            ny = max(yu, yd) - 1;
                        }
                    } else {
                        nx = min(ax[k], xu) + 1;  // (-1,0) is up
                        ny = max(ay[k], yd) - 1;  // (+1,0) is down
                    }
                    if (nx < x[k]) {
                        x[k] = nx;
                        chg |= 1u << k;
                    }
                    if (ny > y[k]) {
                        y[k] = ny;
                        chg |= 1u << (k + 8);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (chg >> k & 1u) sx[rb + k][cc] = x[k];
                if (chg >> (k + 8) & 1u) sn[rb + k][cc] = y[k];
            }
            wrote |= chg;
        }
        if (!__syncthreads_or(chg != 0)) {
            capped = false;
            break;
        }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int64_t g = (int64_t)(r0 + 8 * grp + k) * n + gj;
        if (wrote >> k & 1u) hx[g] = x[k];
        if (wrote >> (k + 8) & 1u) hn[g] = y[k];
    }
    // Which neighbours read a changed value: the tile above reads row 0, the
    // one below row XR-1, the side tiles the outer columns; lozenge rules also
    // read the (-1,+1) and (+1,-1) diagonals, i.e. the corner vertices.  A
    // tile that stopped at its sweep cap is marked again itself.
    enum : unsigned { M_UP = 1, M_DOWN = 2, M_LEFT = 4, M_RIGHT = 8, M_UPRIGHT = 16, M_DOWNLEFT = 32, M_SELF = 64,
                      M_ANY = 128 };
    const uint32_t top = wrote & (1u | 1u << 8), bottom = wrote & (1u << 7 | 1u << 15);
    unsigned mark = 0;
    if (wrote) mark |= M_ANY;
    if (grp == 0 && top) mark |= M_UP;
    if (grp == XR / 8 - 1 && bottom) mark |= M_DOWN;
    if (c == 0 && wrote) mark |= M_LEFT;
    if (c == XC - 1 && wrote) mark |= M_RIGHT;
    if (!DOM && grp == 0 && c == XC - 1 && top) mark |= M_UPRIGHT;
    if (!DOM && grp == XR / 8 - 1 && c == 0 && bottom) mark |= M_DOWNLEFT;
    if (capped && threadIdx.x == 0) mark |= M_SELF;
    if (mark) atomicOr(&s_mark, mark);
    __syncthreads();
    if (threadIdx.x == 0 && s_mark) {
        const unsigned m = s_mark;
        auto set = [&](int y, int x) {
            if (y >= 0 && x >= 0 && y < tiles_y && x < tiles_x) dirty_out[y * tiles_x + x] = 1;
        };
        if (m & M_UP) set(ty - 1, tx);
        if (m & M_DOWN) set(ty + 1, tx);
        if (m & M_LEFT) set(ty, tx - 1);
        if (m & M_RIGHT) set(ty, tx + 1);
        if (m & M_UPRIGHT) set(ty - 1, tx + 1);
        if (m & M_DOWNLEFT) set(ty + 1, tx - 1);
        if (m & M_SELF) set(ty, tx);
        if (m & M_ANY) atomicAdd(changed_tiles, 1u);
    }
}

// The flood's tileability check (a reached interior vertex v whose move
// reaches a boundary vertex w past w's fixed height), then the reference's
// height arrays: INT_MAX outside the domain and wherever the flood did not
// reach.  The check reads both arrays before any is rewritten, so it runs as
// its own kernel.
template <bool DOM>
__global__ void ext_check(const uint8_t* __restrict__ kind, const int32_t* __restrict__ hx,
                          const int32_t* __restrict__ hn, int n, unsigned* bad) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (int64_t)n * n || kind[v] != 1) return;
    const int i = (int)(v / n), j = (int)(v % n);
    const bool even = ((i + j) & 1) == 0;
    const int nbs = DOM ? 4 : 6;
    for (int nb = 0; nb < nbs; ++nb) {
        const int i2 = i + (DOM ? c_ddi[nb] : c_ldi[nb]), j2 = j + (DOM ? c_ddj[nb] : c_ldj[nb]);
        if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n) continue;
        const int64_t w = (int64_t)i2 * n + j2;
        if (kind[w] != 2) continue;
        // step of the edge v -> w
        const int s = DOM ? ((nb > 1) == even ? 1 : -1) : ((nb & 1) ? 1 : -1);
        if (s == 1 && hx[v] < kBig) {
            const int64_t hw = hx[w] < kBig ? (int64_t)hx[w] : (int64_t)INT_MAX;
            if (hw > (int64_t)hx[v] + 1) atomicAdd(bad, 1u);
        }
        if (s == -1 && hn[v] > -kBig) {
            const int64_t hw = hn[w] > -kBig ? (int64_t)hn[w] : (int64_t)INT_MAX;
            if (hw < (int64_t)hn[v] - 1) atomicAdd(bad, 1u);
        }
    }
}

__global__ void ext_finish(const uint8_t* __restrict__ kind, int32_t* hx, int32_t* hn, int64_t nn) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    const bool out = kind[v] == 0;
    if (out || hx[v] >= kBig) hx[v] = INT_MAX;
    if (out || hn[v] <= -kBig) hn[v] = INT_MAX;
}

// HeightfuncToTiling (DominoTiler.cpp:402-421, LozengeTiler.cpp:321-342) of
// both functions at once.
template <bool DOM>
__global__ void ext_tiling(const int32_t* __restrict__ d, int m, const int32_t* __restrict__ h0,
                           const int32_t* __restrict__ h1, int32_t* t0, int32_t* t1) {
    const int n = m + 1;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= (int64_t)n * n) return;
    const int i = (int)(v / n), j = (int)(v % n);
    int32_t a = 0, b = 0;
    if (DOM) {
        for (int nb = 0; nb < 4; ++nb) {
            const int i2 = i + c_ddi[nb], j2 = j + c_ddj[nb];
            if (i2 < 0 || j2 < 0 || i2 >= n || j2 >= n) continue;
            int f0, f1, f2, f3;
            switch (nb) {
                case 0: f0 = i, f1 = j - 1, f2 = i, f3 = j; break;
                case 1: f0 = i - 1, f1 = j - 1, f2 = i - 1, f3 = j; break;
                case 2: f0 = i - 1, f1 = j, f2 = i, f3 = j; break;
                default: f0 = i - 1, f1 = j - 1, f2 = i, f3 = j - 1; break;
            }
            if (!dface(d, m, f0, f1) && !dface(d, m, f2, f3)) continue;
            const int64_t w = (int64_t)i2 * n + j2;
            if (h0[v] != INT_MAX && h0[w] != INT_MAX) {
                const int64_t q = ((int64_t)h0[w] - h0[v]) / 2;
                a += c_dbit[nb] * (int32_t)(q < 0 ? -q : q);
            }
            if (h1[v] != INT_MAX && h1[w] != INT_MAX) {
                const int64_t q = ((int64_t)h1[w] - h1[v]) / 2;
                b += c_dbit[nb] * (int32_t)(q < 0 ? -q : q);
            }
        }
    } else if (i >= 1 && j >= 1 && i < n - 1 && j < n - 1) {
        for (int nb = 0; nb < 6; ++nb) {
            if (!lface(d, m, i + c_lface[nb][0], 2 * j + c_lface[nb][1]) &&
                !lface(d, m, i + c_lface[nb][2], 2 * j + c_lface[nb][3]))
                continue;
            const int64_t w = (int64_t)(i + c_ldi[nb]) * n + (j + c_ldj[nb]);
            const int64_t d0 = (int64_t)h0[w] - h0[v], d1 = (int64_t)h1[w] - h1[v];
            if (d0 == 2 || d0 == -2) a += c_lbit[nb];
            if (d1 == 2 || d1 == -2) b += c_lbit[nb];
        }
    }
    t0[v] = a;
    t1[v] = b;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    bool alloc(size_t b) { return cudaMalloc(&p, b ? b : 1) == cudaSuccess; }
};

struct Stream {
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Stream() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (s) cudaStreamDestroy(s);
    }
};

}  // namespace
}  // namespace rtb

using namespace rtb;

namespace {

// Device memory of `device` (or managed memory), the only kind the kernels may write.
bool device_memory(const void* p, int device) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == device;
}

// Both entry points: outputs in host memory (copied back) or, with dev_out,
// the caller's device buffers (the relaxation and the tilings are written
// there directly).
rt_status extremal_run(int32_t model, const int32_t* d, int64_t dlen, int32_t device, int32_t* tmin, int32_t* tmax,
                       int32_t* hmin, int32_t* hmax, int64_t len, rt_extremal_stats* stats, bool dev_out) {
    if ((model != RT_DOMINO && model != RT_LOZENGE) || !d || dlen <= 0) return RT_E_INVAL;
    const bool dom = model == RT_DOMINO;
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
    auto t0 = clk::now();
    int n = 0;
    std::vector<int64_t> bidx;
    std::vector<int32_t> bh;
    if (!boundary_walk(model, d, dlen, &n, &bidx, &bh)) return RT_E_INVAL;
    const double walk_ms = ms_since(t0);
    const int m = n - 1;
    const int64_t nn = (int64_t)n * n;
    if (len != nn) return RT_E_INVAL;
    if (cudaSetDevice(device) != cudaSuccess) return RT_E_NODEVICE;
    if (dev_out)
        for (const int32_t* o : {tmin, tmax, hmin, hmax})
            if (o && !device_memory(o, device)) return RT_E_INVAL;
    const int tiles_x = (n + XC - 1) / XC, tiles_y = (n + XR - 1) / XR;
    const int64_t tiles = (int64_t)tiles_x * tiles_y;
    if (tiles > INT_MAX) return RT_E_INVAL;
    t0 = clk::now();
    DevBuf dd, dk, dx, dn, dtx, dtn, dbi, dbh, dflag, dcnt;
    // the caller's device buffers serve as the work arrays where given
    const bool own_hx = !(dev_out && hmax), own_hn = !(dev_out && hmin), tilings = tmin || tmax;
    const bool own_tx = tilings && !(dev_out && tmax), own_tn = tilings && !(dev_out && tmin);
    if (!dd.alloc((size_t)dlen * 4) || !dk.alloc((size_t)nn) || (own_hx && !dx.alloc((size_t)nn * 4)) ||
        (own_hn && !dn.alloc((size_t)nn * 4)) || (own_tx && !dtx.alloc((size_t)nn * 4)) ||
        (own_tn && !dtn.alloc((size_t)nn * 4)) || !dbi.alloc(bidx.size() * 8) || !dbh.alloc(bh.size() * 4) ||
        !dflag.alloc((size_t)tiles * 2) || !dcnt.alloc((kGroup + 1) * 4))
        return RT_E_NOMEM;
    Stream st;
    if (cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&st.e0) != cudaSuccess || cudaEventCreate(&st.e1) != cudaSuccess)
        return RT_E_CUDA;
    cudaStream_t s = st.s;
    const double alloc_ms = ms_since(t0);
    t0 = clk::now();
    auto* K = static_cast<uint8_t*>(dk.p);
    auto* HX = own_hx ? static_cast<int32_t*>(dx.p) : hmax;
    auto* HN = own_hn ? static_cast<int32_t*>(dn.p) : hmin;
    auto* F = static_cast<uint8_t*>(dflag.p);
    auto* C = static_cast<unsigned*>(dcnt.p);
    cudaMemcpyAsync(dd.p, d, (size_t)dlen * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dbi.p, bidx.data(), bidx.size() * 8, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dbh.p, bh.data(), bh.size() * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(F, 1, (size_t)tiles, s);
    cudaMemsetAsync(F + tiles, 0, (size_t)tiles, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return RT_E_CUDA;
    const double upload_ms = ms_since(t0);
    cudaEventRecord(st.e0, s);
    const int T = 256;
    const unsigned vb = (unsigned)((nn + T - 1) / T);
    const auto* D = static_cast<const int32_t*>(dd.p);
    if (dom)
        ext_classify<true><<<vb, T, 0, s>>>(D, m, K, HX, HN);
    else
        ext_classify<false><<<vb, T, 0, s>>>(D, m, K, HX, HN);
    const int64_t nb = (int64_t)bidx.size();
    ext_seed<<<(unsigned)((nb + T - 1) / T), T, 0, s>>>(static_cast<const int64_t*>(dbi.p),
                                                       static_cast<const int32_t*>(dbh.p), nb, HX, HN);
    // Passes in groups; the counters of a group are read once.  A pass that
    // changes nothing leaves no tile marked, so the relaxation has converged.
    int64_t passes = 0, updates = 0;
    const int64_t cap = 64 + 4 * ((int64_t)n + tiles);  // far above any domain's need; a guard, not a tuning
    unsigned cnt[kGroup];
    for (;;) {
        cudaMemsetAsync(C, 0, kGroup * 4, s);
        for (int p = 0; p < kGroup; ++p) {
            uint8_t* in = F + (p & 1) * tiles;
            uint8_t* out = F + ((p & 1) ^ 1) * tiles;
            if (dom)
                ext_relax<true><<<(unsigned)tiles, XT, 0, s>>>(K, HX, HN, n, tiles_x, tiles_y, in, out, C + p);
            else
                ext_relax<false><<<(unsigned)tiles, XT, 0, s>>>(K, HX, HN, n, tiles_x, tiles_y, in, out, C + p);
        }
        passes += kGroup;
        cudaError_t ce = cudaMemcpyAsync(cnt, C, sizeof cnt, cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
        if (ce != cudaSuccess) return RT_E_CUDA;
        for (int p = 0; p < kGroup; ++p) updates += cnt[p];
        if (cnt[kGroup - 1] == 0) break;
        if (passes > cap) return RT_E_TIMEOUT;
    }
    cudaMemsetAsync(C + kGroup, 0, 4, s);
    if (dom)
        ext_check<true><<<vb, T, 0, s>>>(K, HX, HN, n, C + kGroup);
    else
        ext_check<false><<<vb, T, 0, s>>>(K, HX, HN, n, C + kGroup);
    ext_finish<<<vb, T, 0, s>>>(K, HX, HN, nn);
    auto* TX = own_tx ? static_cast<int32_t*>(dtx.p) : tmax;
    auto* TN = own_tn ? static_cast<int32_t*>(dtn.p) : tmin;
    if (tilings) {
        if (dom)
            ext_tiling<true><<<vb, T, 0, s>>>(D, m, HN, HX, TN, TX);
        else
            ext_tiling<false><<<vb, T, 0, s>>>(D, m, HN, HX, TN, TX);
    }
    cudaEventRecord(st.e1, s);
    unsigned bad = 0;
    cudaMemcpyAsync(&bad, C + kGroup, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return RT_E_CUDA;
    if (bad) return RT_E_INVAL;  // not tileable: the flood ran past a boundary height
    t0 = clk::now();
    if (!dev_out) {
        if (tmin) cudaMemcpyAsync(tmin, TN, (size_t)nn * 4, cudaMemcpyDeviceToHost, s);
        if (tmax) cudaMemcpyAsync(tmax, TX, (size_t)nn * 4, cudaMemcpyDeviceToHost, s);
        if (hmin) cudaMemcpyAsync(hmin, HN, (size_t)nn * 4, cudaMemcpyDeviceToHost, s);
        if (hmax) cudaMemcpyAsync(hmax, HX, (size_t)nn * 4, cudaMemcpyDeviceToHost, s);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) return RT_E_CUDA;
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, st.e0, st.e1);
        stats->n = n;
        stats->boundary = nb;
        stats->passes = passes;
        stats->tile_updates = updates;
        stats->device_ms = ms;
        stats->walk_ms = walk_ms;
        stats->alloc_ms = alloc_ms;
        stats->upload_ms = upload_ms;
        stats->download_ms = ms_since(t0);
    }
    return RT_OK;
}

}  // namespace

extern "C" rt_status rt_extremal_tilings(int32_t model, const int32_t* d, int64_t dlen, int32_t device, int32_t* tmin,
                                         int32_t* tmax, int32_t* hmin, int32_t* hmax, int64_t len,
                                         rt_extremal_stats* stats) {
    return guarded([&]() -> rt_status {
        return extremal_run(model, d, dlen, device, tmin, tmax, hmin, hmax, len, stats, false);
    });
}

extern "C" rt_status rt_extremal_tilings_device(int32_t model, const int32_t* d, int64_t dlen, int32_t device,
                                                int32_t* d_tmin, int32_t* d_tmax, int32_t* d_hmin, int32_t* d_hmax,
                                                int64_t len, rt_extremal_stats* stats) {
    return guarded([&]() -> rt_status {
        return extremal_run(model, d, dlen, device, d_tmin, d_tmax, d_hmin, d_hmax, len, stats, true);
    });
}
