// rt_capi.cu -- the C ABI (include/rt_b200.h): handles, schedules, transfers.
//
// The host side of a walk follows the reference's Walk methods: the colour
// of every step comes from the same libstdc++ engines the reference uses on
// its host (std::mt19937 for dominoes, DominoTiler.cpp:31-42;
// std::default_random_engine + uniform_int_distribution<int>(0,2) for the
// three-colour models, LozengeTiler.cpp:50-55, RectTriangleTiler.cpp:41-48),
// drawn once per call into a phase list that the device walks in one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "rt_internal.h"
#include "rt_guard.h"
#include "rt_models.cuh"
#include "rt_tridimer.cuh"

using rtb::guarded;

using namespace rtb;

namespace {

constexpr uint32_t kMat1 = 0x8f7011eeu;  // TinyMT32J, src/TinyMT/tinymt32def.h:47-49
constexpr uint32_t kMat2 = 0xfc78ff1fu;
constexpr uint32_t kTmat = 0x3793fdffu;

thread_local std::string g_create_error;

struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
    bool reserve(size_t bytes) {
        if (bytes <= cap) return true;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) return false;
        cap = bytes;
        return true;
    }
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
};

struct DevBuf {
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
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

// Largest K with  K <= x * 2^e  (clamped to [0, 2^32-1]).
uint32_t floor_scaled(double x, int e) {
    const double s = std::floor(std::ldexp(x, e));
    if (s <= 0) return 0;
    if (s >= 4294967295.0) return 0xffffffffu;
    return (uint32_t)s;
}

}  // namespace

namespace rtb {

uint32_t below_threshold(double x) {
    const double s = std::ceil(x * 8388608.0);
    if (s <= 0) return 0;
    if (s >= 4294967295.0) return 0xffffffffu;
    return (uint32_t)s;
}

// Phases of one triangle-dimer step (TriangleDimerTiler.cpp:243-347): the
// flip family `kind` (0 lozenges, 1 triangles, 2 butterflies), orientation /
// class r1, kind or parity r2, and for butterflies the slice p1 and parity p2.
int64_t td_step_phases(uint32_t* ph, int64_t at, uint32_t kind, uint32_t r1, uint32_t r2, uint32_t p1, uint32_t p2) {
    if (kind == 0) {  // lozenge flips, :243-278
        ph[at++] = make_phase(TD_ROT_LOZ, r1, r2, true);
        ph[at++] = make_phase(TD_LOZ_FLIPPED, r1, r2, false);
        ph[at++] = make_phase(TD_LOZ_OTHER, r1, 0, false);
        ph[at++] = make_phase(TD_UP_FROM_LOZ, 0, 0, false);
        ph[at++] = make_phase(TD_TRI_OTHER, 0, 7, false);
    } else if (kind == 1) {  // triangle flips, :279-305
        ph[at++] = make_phase(TD_ROT_TRI, r2, r1, true);
        ph[at++] = make_phase(TD_TRI_FLIPPED, r2, r1, false);
        ph[at++] = make_phase(TD_TRI_OTHER, r2, 0, false);
        ph[at++] = make_phase(TD_LOZ_FROM_TRI, 0, 0, false);
        ph[at++] = make_phase(TD_BFLY_FROM_LOZ, 0, 7, false);
    } else {  // butterfly flips, :306-347
        ph[at++] = make_phase(TD_ROT_BFLY, r1, p1 | (p2 << 2), true);
        ph[at++] = make_phase(TD_BFLY_SAME, r1, p1 | (p2 << 2), false);
        ph[at++] = make_phase(TD_BFLY_21, r1, p1, false);
        ph[at++] = make_phase(TD_BFLY_22, r1, p1, false);
        ph[at++] = make_phase(TD_BFLY_23_LOZ, r1, p1, false);
        ph[at++] = make_phase(TD_BFLY_FROM_LOZ, 1, 7u & ~(1u << r1), false);
        ph[at++] = make_phase(TD_TRI_OTHER, 0, 0, false);
    }
    return at;
}

// Fast-mode step s of an epoch: dominoes flip the black array (0) on even
// steps and the white one on odd steps (reference colour r flips array
// 1 - r); lozenges and rectangle-triangles flip colour s mod 3; triangle
// dimers make move s mod 30 of a sweep over every flip class.
int64_t fast_step_phases(int kind, int64_t s, uint32_t* ph, int64_t at, uint32_t* prev) {
    if (kind == 3) {
        const uint32_t mv = (uint32_t)(s % 30);
        if (mv < 6) return td_step_phases(ph, at, 0, mv / 2, mv % 2, 0, 0);
        if (mv < 12) return td_step_phases(ph, at, 1, (mv - 6) % 3, (mv - 6) / 3, 0, 0);
        return td_step_phases(ph, at, 2, (mv - 12) / 6, 0, ((mv - 12) / 2) % 3, (mv - 12) % 2);
    }
    const uint32_t r = kind == 0 ? (uint32_t)(1 - (s & 1)) : (uint32_t)(s % 3);
    ph[at++] = make_phase(OP_STEP, r, *prev, true);
    *prev = r;
    return at;
}

void fast_phases(int kind, int64_t steps, std::vector<uint32_t>& ph) {
    const size_t base = ph.size();
    ph.resize(base + (size_t)(kind == 3 ? 7 * steps : steps + 1));
    int64_t at = (int64_t)base;
    uint32_t prev = NO_COLOUR;
    for (int64_t s = 0; s < steps; ++s) at = fast_step_phases(kind, s, ph.data(), at, &prev);
    if (kind != 3 && steps > 0) ph[at++] = make_phase(OP_FINAL, prev, NO_COLOUR, false);
    ph.resize((size_t)at);
}

rt_status choose_plan(int family, int device, int nlat, int rows, int cols, int width, bool uniform, bool fast,
                      bool planes, bool weighted, int kernel_choice, int ctas_hint, int depth_hint, WalkPlan* plan,
                      std::string* err) {
    if (planes) return plan_plane_walk(family, device, nlat, rows, width, ctas_hint, depth_hint, plan, err);
    rt_status s = RT_E_INVAL;
    if (kernel_choice != 1 && uniform && (word_family(family) || family == FAM_QLOZENGE8))
        s = plan_word_walk(family, device, nlat, rows, width, fast, ctas_hint, plan, err, weighted);
    if (s == RT_OK || kernel_choice == 2) return s;
    return plan_walk(family, device, nlat, rows, cols, width, uniform, fast, plan, err);
}

void family_thresholds(int family, double q, int qcmp, uint32_t thr[4]) {
    thr[0] = thr[1] = thr[2] = thr[3] = 0;
    switch (family) {
        case FAM_DOMINO: thr[0] = below_threshold(0.8); break;     // dominokernel.cl:13
        case FAM_DOMINO_HB: thr[0] = below_threshold(0.5); break;  // dominokernelCFTP.cl:22
        case FAM_LOZENGE8:                                          // lozengekernel.cl:19-21
            thr[0] = below_threshold(0.4);
            thr[1] = below_threshold(0.8);
            break;
        case FAM_QLOZENGE8:  // qlozengekernel.cl:18-26
            if (qcmp == RT_QCMP_DOUBLE) {
                thr[0] = floor_scaled(q, 22);
                thr[1] = floor_scaled(1.0 / q, 24);
            } else {
                const float qf = (float)q;
                const float inv = 1.0f / qf;
                thr[0] = floor_scaled((double)qf, 22);
                thr[1] = floor_scaled((double)inv, 24);
            }
            // The same rule as bounds on k for the word kernel: add iff
            // k < thr[2] (k < 2^22 and k <= thr[0]); remove iff
            // 2^22 <= k < thr[3] (k - 2^22 <= thr[1]); k < 2^23 always.
            thr[2] = (uint32_t)std::min<uint64_t>(1u << 22, (uint64_t)thr[0] + 1);
            thr[3] = (uint32_t)std::min<uint64_t>(1u << 23, (uint64_t)(1u << 22) + thr[1] + 1);
            break;
        default: break;
    }
}

}  // namespace rtb

struct rt_tiler {
    rt_config cfg{};
    int family = 0;
    int ncol = 0;     // colour arrays
    int kind = 0;     // split layout (0 domino, 1 lozenge, 2 rect-triangle)
    int elem = 1;     // bytes per stored site
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    std::vector<uint32_t> table;  // 3 per id
    bool table_dirty = false;
    DevBuf d_params;
    int64_t d_params_n = 0;

    int n = 0, rows = 0, cols = 0;
    int arows = 0, width = 0;  // shape of one colour array
    int nlat = 1;
    DevBuf d_arr_block;  // all colour arrays of all lattices
    void* d_arr[2][8] = {};
    DevBuf d_tiling, d_tiling2;
    size_t per_arr_al = 0;  // bytes of one colour array (256-aligned)
    DevBuf d_count;
    PinnedBuf h_count;
    bool uploaded = false;

    DevBuf d_phases, d_epoch_start, d_epoch_seed, d_xbuf, d_err;
    PinnedBuf h_phases, h_epoch_start, h_epoch_seed, h_err;
    cudaEvent_t ev_staged = nullptr;

    WalkPlan plan;
    int plan_rows = -1, plan_cols = -1, plan_nlat = -1;
    bool plan_uniform = true;
    bool plan_weighted = false;
    int kernel_choice = 0;  // 0 auto, 1 generic walk kernel only, 2 word kernel only (RT_WALK_KERNEL)
    int ctas_hint = 0;      // word kernel grid (RT_WALK_CTAS; 0 = one CTA per SM)
    int depth_hint = 0;     // bit-plane kernel: phases per halo exchange (RT_PLANE_DEPTH; 0 = up to 8)
    int64_t drop_phase = -1;  // RT_TEST_DROP_PUBLISH: a phase whose rows CTA 0 withholds (bounded-wait tests)
    int64_t last_phases = 0, last_launches = 0;
    uint64_t timeout_ns = 5000000000ull;
    int wper = 0;           // weighted domino heat bath: period (0 = uniform)
    uint32_t wthr[16] = {};

    rt_status fail(rt_status s, const std::string& msg) {
        err = msg;
        return s;
    }
    rt_status cuda_fail(cudaError_t e, const char* what) {
        return fail(RT_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
};

extern "C" {

const char* rt_version(void) { return "randomtilings_b200 0.1 (sm_100a)"; }

void rt_config_default(rt_config* cfg, int32_t model) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof *cfg);
    cfg->model = model;
    cfg->kernel = RT_KERNEL_DEFAULT;
    cfg->rng = RT_RNG_TINYMT;
    cfg->qcmp = RT_QCMP_FLOAT32;
    cfg->q = 0.99;  // qlozengekernel.cl:3
    cfg->weights[0] = 0.0f;  // recttrianglekernel.cl:13
    for (int i = 1; i < 16; ++i) cfg->weights[i] = 1.0f;
    cfg->device = 0;
    cfg->stream = nullptr;
}

rt_status rt_create(const rt_config* cfg, rt_tiler** out) {
    return guarded([&]() -> rt_status {
        if (!cfg || !out) {
            g_create_error = "null argument";
            return RT_E_INVAL;
        }
        *out = nullptr;
        int family = -1, ncol = 0, kind = 0, elem = 1;
        switch (cfg->model) {
            case RT_DOMINO:
                if (cfg->kernel != RT_KERNEL_DEFAULT && cfg->kernel != RT_KERNEL_CFTP) break;
                family = cfg->kernel == RT_KERNEL_CFTP ? FAM_DOMINO_HB : FAM_DOMINO;
                ncol = 2, kind = 0, elem = 1;
                break;
            case RT_LOZENGE:
                if (cfg->kernel == RT_KERNEL_DEFAULT) family = FAM_LOZENGE8, elem = 1;
                else if (cfg->kernel == RT_KERNEL_QWEIGHT) family = FAM_QLOZENGE8, elem = 1;
                ncol = 3, kind = 1;
                break;
            case RT_RECTTRI:
                if (cfg->kernel != RT_KERNEL_DEFAULT) break;
                family = FAM_RECTTRI, ncol = 3, kind = 2, elem = 4;
                break;
            case RT_TRIDIMER:
                if (cfg->kernel != RT_KERNEL_DEFAULT) break;
                family = FAM_TRIDIMER, ncol = 8, kind = 3, elem = 4;
                break;
            default:
                break;
        }
        if (family < 0) {
            g_create_error = "unsupported model/kernel combination";
            return RT_E_INVAL;
        }
        if (cfg->rng != RT_RNG_TINYMT && cfg->rng != RT_RNG_PHILOX && cfg->rng != RT_RNG_PLANES) {
            g_create_error = "unknown rng mode";
            return RT_E_INVAL;
        }
        if (cfg->rng == RT_RNG_PLANES && !word_family(family)) {
            g_create_error = "bit-plane mode exists for dominoes and uniform lozenges";
            return RT_E_INVAL;
        }
        if (family == FAM_QLOZENGE8 && (!(cfg->q >= 0.0) || !std::isfinite(cfg->q))) {
            g_create_error = "q must be a finite non-negative number";
            return RT_E_INVAL;
        }
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
            g_create_error = "no CUDA device with that ordinal";
            return RT_E_NODEVICE;
        }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major != 10) {
            g_create_error = "device is not sm_100 (this library carries sm_100a code only)";
            return RT_E_NODEVICE;
        }
        if (!prop.cooperativeLaunch) {
            g_create_error = "device does not support cooperative launches";
            return RT_E_NODEVICE;
        }
        cudaSetDevice(cfg->device);
        rt_tiler* h = new rt_tiler();
        h->cfg = *cfg;
        h->family = family;
        h->ncol = ncol;
        h->kind = kind;
        h->elem = elem;
        if (cfg->stream) {
            h->stream = static_cast<cudaStream_t>(cfg->stream);
        } else {
            if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
                delete h;
                g_create_error = "cudaStreamCreate failed";
                return RT_E_CUDA;
            }
            h->own_stream = true;
        }
        if (cudaEventCreateWithFlags(&h->ev_staged, cudaEventDisableTiming) != cudaSuccess) {
            if (h->own_stream) cudaStreamDestroy(h->stream);
            delete h;
            g_create_error = "cudaEventCreate failed";
            return RT_E_CUDA;
        }
        if (const char* kc = std::getenv("RT_WALK_KERNEL")) {
            if (std::strcmp(kc, "generic") == 0) h->kernel_choice = 1;
            if (std::strcmp(kc, "word") == 0) h->kernel_choice = 2;
        }
        if (const char* ct = std::getenv("RT_WALK_CTAS")) h->ctas_hint = std::max(0, std::atoi(ct));
        if (const char* dp = std::getenv("RT_PLANE_DEPTH")) h->depth_hint = std::max(0, std::atoi(dp));
        if (const char* dp = std::getenv("RT_TEST_DROP_PUBLISH")) h->drop_phase = std::atoll(dp);
        if (const char* t = std::getenv("RT_WAIT_TIMEOUT_MS")) {
            const long ms = std::atol(t);
            if (ms > 0) h->timeout_ns = (uint64_t)ms * 1000000ull;
        }
        *out = h;
        return RT_OK;
    });
}

rt_status rt_destroy(rt_tiler* h) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        cudaSetDevice(h->cfg.device);
        cudaStreamSynchronize(h->stream);
        if (h->ev_staged) cudaEventDestroy(h->ev_staged);
        if (h->own_stream) cudaStreamDestroy(h->stream);
        delete h;
        return RT_OK;
    });
}

const char* rt_last_error(rt_tiler* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

void* rt_stream(rt_tiler* h) { return h ? static_cast<void*>(h->stream) : nullptr; }

rt_status rt_set_domino_weights(rt_tiler* h, int32_t period, const double* wh, const double* wv) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        if (h->family != FAM_DOMINO_HB) return h->fail(RT_E_INVAL, "weights need the domino heat-bath kernel (RT_KERNEL_CFTP)");
        if (h->cfg.rng == RT_RNG_PLANES) return h->fail(RT_E_INVAL, "the bit-plane mode draws one bit per site: no weights");
        if (period == 0) {
            h->wper = 0;
            return RT_OK;
        }
        if ((period != 1 && period != 2 && period != 4) || !wh || !wv)
            return h->fail(RT_E_INVAL, "weight period must be 1, 2 or 4, with two period x period tables");
        const int P = period;
        for (int k = 0; k < P * P; ++k)
            if (!(wh[k] > 0 && wv[k] > 0) || !std::isfinite(wh[k]) || !std::isfinite(wv[k]))
                return h->fail(RT_E_INVAL, "domino weights must be finite and > 0");
        auto W = [&](const double* w, int r, int c) { return w[(((r % P) + P) % P) * P + (((c % P) + P) % P)]; };
        for (int i = 0; i < P; ++i)
            for (int j = 0; j < P; ++j) {
                // vertex class (i, j): the squares (i-1, j-1), (i-1, j), (i, j-1) around it
                const double w3 = W(wh, i - 1, j - 1) * W(wh, i, j - 1);
                const double w12 = W(wv, i - 1, j - 1) * W(wv, i - 1, j);
                h->wthr[i * P + j] = below_threshold(w12 / (w3 + w12));
            }
        h->wper = P;
        return RT_OK;
    });
}

rt_status rt_set_lozenge_weights(rt_tiler* h, int32_t period, const double* w0, const double* w1, const double* w2) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        if (h->family != FAM_LOZENGE8) return h->fail(RT_E_INVAL, "weights need the uniform lozenge kernel (char storage)");
        if (h->cfg.rng == RT_RNG_PLANES) return h->fail(RT_E_INVAL, "the bit-plane mode draws one bit per site: no weights");
        if (period == 0) {
            h->wper = 0;
            return RT_OK;
        }
        if ((period != 1 && period != 2 && period != 4) || !w0 || !w1 || !w2)
            return h->fail(RT_E_INVAL, "weight period must be 1, 2 or 4, with three period x period tables");
        const int P = period;
        for (int k = 0; k < P * P; ++k)
            for (const double* w : {w0, w1, w2})
                if (!(w[k] > 0) || !std::isfinite(w[k])) return h->fail(RT_E_INVAL, "lozenge weights must be finite and > 0");
        auto W = [&](const double* w, int r, int c) { return w[(((r % P) + P) % P) * P + (((c % P) + P) % P)]; };
        for (int i = 0; i < P; ++i)
            for (int j = 0; j < P; ++j) {
                const double w25 = W(w2, i, j) * W(w0, i, j) * W(w1, i + 1, j - 1);
                const double w38 = W(w1, i, j) * W(w0, i, j - 1) * W(w2, i + 1, j);
                h->wthr[i * P + j] = below_threshold(0.8 * (w38 / (w25 + w38)));
            }
        h->wper = P;
        return RT_OK;
    });
}

rt_status rt_set_rng_params(rt_tiler* h, const uint32_t* table, int64_t n) {
    return guarded([&]() -> rt_status {
        if (!h || (!table && n > 0) || n < 0) return h ? h->fail(RT_E_INVAL, "bad parameter table") : RT_E_INVAL;
        h->table.assign(table, table + 3 * n);
        h->table_dirty = true;
        return RT_OK;
    });
}

// The layout src/TinyMT/file_reader.cpp:51-70,139-166 reads: lines starting
// with '#' are skipped; mat1, mat2 and tmat are the hexadecimal fields after
// the 3rd, 4th and 5th comma.
rt_status rt_load_rng_params(rt_tiler* h, const char* path, int64_t n) {
    return guarded([&]() -> rt_status {
        if (!h || !path || n < 0) return h ? h->fail(RT_E_INVAL, "bad arguments") : RT_E_INVAL;
        std::ifstream in(path);
        if (!in) return h->fail(RT_E_PARAMS, std::string("cannot open parameter file ") + path);
        std::vector<uint32_t> t;
        // The file, not n, bounds the table: reserve at most 2^21 entries ahead.
        t.reserve((size_t)std::min<int64_t>(n, (int64_t)1 << 21) * 3);
        std::string line;
        int64_t got = 0;
        while (got < n && std::getline(in, line)) {
            if (!line.empty() && line[0] == '#') continue;
            size_t pos[5];
            int commas = 0;
            for (size_t i = 0; i < line.size() && commas < 5; ++i)
                if (line[i] == ',') pos[commas++] = i;
            if (commas < 5) return h->fail(RT_E_PARAMS, "parameter line " + std::to_string(got) + ": comma not found");
            for (int f = 2; f < 5; ++f) t.push_back((uint32_t)std::strtoul(line.c_str() + pos[f] + 1, nullptr, 16));
            ++got;
        }
        if (got < n) return h->fail(RT_E_PARAMS, "parameter file has " + std::to_string(got) + " entries, need " + std::to_string(n));
        h->table.swap(t);
        h->table_dirty = true;
        return RT_OK;
    });
}

static rt_status check_size(rt_tiler* h, int n) {
    if (n > kMaxTilingSide) return h->fail(RT_E_INVAL, "tiling side above 32767");
    if (h->kind == 0 && (n < 6 || n % 2 != 0)) return h->fail(RT_E_INVAL, "domino tiling side must be even and >= 6");
    if (h->kind == 3 && (n < 8 || n % 2 != 0))
        return h->fail(RT_E_INVAL, "triangle-dimer tiling side must be even and >= 8");
    if ((h->kind == 1 || h->kind == 2) && (n < 9 || n % 3 != 0))
        return h->fail(RT_E_INVAL, "tiling side must be a multiple of 3 and >= 9");
    return RT_OK;
}

static void grid_of(const rt_tiler* h, int n, int* rows, int* cols) {
    if (h->kind == 0) {  // Rotate NDRange (N-2, N/2-2), DominoTiler.cpp:37
        *rows = n - 2;
        *cols = n / 2 - 2;
    } else if (h->kind == 3) {  // (M, M), TriangleDimerTiler.cpp:246
        *rows = n / 2;
        *cols = n / 2;
    } else {  // (N, N/3), LozengeTiler.cpp:58, RectTriangleTiler.cpp:51
        *rows = n;
        *cols = n / 3;
    }
}

// Shape of one colour array: domino N x N/2, three-colour N x N/3,
// triangle-dimer N/2 x N/2.
static void array_shape(const rt_tiler* h, int n, int* arows, int* width) {
    if (h->kind == 3) {
        *arows = n / 2;
        *width = n / 2;
    } else {
        *arows = n;
        *width = n / h->ncol;
    }
}

rt_status rt_upload(rt_tiler* h, const int32_t* tiling, int32_t n) {
    return guarded([&]() -> rt_status {
        if (!h || !tiling) return h ? h->fail(RT_E_INVAL, "null tiling") : RT_E_INVAL;
        rt_status s = check_size(h, n);
        if (s != RT_OK) return s;
        cudaSetDevice(h->cfg.device);
        int arows, width;
        array_shape(h, n, &arows, &width);
        const size_t per_arr = (size_t)arows * (size_t)width * (size_t)h->elem;
        const size_t per_arr_al = (per_arr + 255) & ~(size_t)255;
        h->per_arr_al = per_arr_al;
        if (!h->d_arr_block.reserve(per_arr_al * h->ncol * 2)) return h->fail(RT_E_NOMEM, "cudaMalloc lattice");
        if (!h->d_tiling.reserve((size_t)n * n * 4)) return h->fail(RT_E_NOMEM, "cudaMalloc tiling");
        for (int l = 0; l < 2; ++l)
            for (int c = 0; c < 8; ++c)
                h->d_arr[l][c] = c < h->ncol ? static_cast<char*>(h->d_arr_block.p) + (l * h->ncol + c) * per_arr_al : nullptr;
        // Alignment padding between the colour arrays is compared by the CFTP
        // coalescence test, so it must hold the same bytes in both lattices.
        cudaError_t e = cudaMemsetAsync(h->d_arr_block.p, 0, per_arr_al * h->ncol * 2, h->stream);
        if (e != cudaSuccess) return h->cuda_fail(e, "memset lattice");
        e = cudaMemcpyAsync(h->d_tiling.p, tiling, (size_t)n * n * 4, cudaMemcpyHostToDevice, h->stream);
        if (e != cudaSuccess) return h->cuda_fail(e, "upload");
        if (h->kind == 3) {
            // The eight triangle-dimer arrays are derived on the host
            // (TriangleDimerTiler.cpp:90-133) and copied up as they are.
            std::vector<int32_t> arrays((size_t)8 * arows * width);
            td_split_host(tiling, n, arrays.data());
            for (int c = 0; c < 8 && e == cudaSuccess; ++c)
                e = cudaMemcpy(h->d_arr[0][c], arrays.data() + (size_t)c * arows * width, per_arr, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return h->cuda_fail(e, "upload of the triangle-dimer arrays");
        } else {
            s = launch_split(false, h->elem, h->kind, h->ncol, n, static_cast<int32_t*>(h->d_tiling.p), h->d_arr[0],
                             h->stream, &h->err);
            if (s != RT_OK) return s;
        }
        if (!h->d_err.reserve(sizeof(int)) || !h->h_err.reserve(sizeof(int))) return h->fail(RT_E_NOMEM, "error word");
        e = cudaMemsetAsync(h->d_err.p, 0, sizeof(int), h->stream);
        if (e != cudaSuccess) return h->cuda_fail(e, "memset");
        h->n = n;
        h->arows = arows;
        h->width = width;
        grid_of(h, n, &h->rows, &h->cols);
        h->uploaded = true;
        return RT_OK;
    });
}

rt_status rt_download(rt_tiler* h, int32_t* tiling) {
    return guarded([&]() -> rt_status {
        if (!h || !tiling) return h ? h->fail(RT_E_INVAL, "null tiling") : RT_E_INVAL;
        if (!h->uploaded) return h->fail(RT_E_STATE, "download before upload");
        cudaSetDevice(h->cfg.device);
        const int n = h->n;
        rt_status s = launch_split(true, h->elem, h->kind, h->ncol, n, static_cast<int32_t*>(h->d_tiling.p), h->d_arr[0],
                                   h->stream, &h->err);
        if (s != RT_OK) return s;
        cudaError_t e = cudaMemcpyAsync(tiling, h->d_tiling.p, (size_t)n * n * 4, cudaMemcpyDeviceToHost, h->stream);
        if (e != cudaSuccess) return h->cuda_fail(e, "download");
        return rt_synchronize(h);
    });
}

rt_status rt_device_tiling(rt_tiler* h, int32_t** d_tiling) {
    return guarded([&]() -> rt_status {
        if (!h || !d_tiling) return h ? h->fail(RT_E_INVAL, "null pointer") : RT_E_INVAL;
        if (!h->uploaded) return h->fail(RT_E_STATE, "device tiling before upload");
        cudaSetDevice(h->cfg.device);
        rt_status s = launch_split(true, h->elem, h->kind, h->ncol, h->n, static_cast<int32_t*>(h->d_tiling.p), h->d_arr[0],
                                   h->stream, &h->err);
        if (s != RT_OK) return s;
        *d_tiling = static_cast<int32_t*>(h->d_tiling.p);
        return RT_OK;
    });
}

rt_status rt_synchronize(rt_tiler* h) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        cudaSetDevice(h->cfg.device);
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return h->cuda_fail(e, "stream synchronize");
        if (h->uploaded) {
            e = cudaMemcpy(h->h_err.p, h->d_err.p, sizeof(int), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) return h->cuda_fail(e, "error word readback");
            const int code = *static_cast<int*>(h->h_err.p);
            if (code & ERR_TIMEOUT) return h->fail(RT_E_TIMEOUT, "a bounded wait between CTAs timed out; walk aborted");
            if (code) return h->fail(RT_E_CUDA, "device error word " + std::to_string(code));
        }
        return RT_OK;
    });
}

// Stages the TinyMT parameter table on the device (all ids the walk uses).
static rt_status stage_params(rt_tiler* h, int64_t needed) {
    if (h->table.empty()) return RT_OK;  // uniform TinyMT32J parameters
    const int64_t have = (int64_t)h->table.size() / 3;
    if (have < needed)
        return h->fail(RT_E_PARAMS, "parameter table has " + std::to_string(have) + " entries, the walk needs " +
                                         std::to_string(needed));
    if (!h->table_dirty && h->d_params_n >= needed) return RT_OK;
    std::vector<uint4> p((size_t)needed);
    for (int64_t i = 0; i < needed; ++i) p[i] = make_uint4(h->table[3 * i], h->table[3 * i + 1], h->table[3 * i + 2], 0u);
    if (!h->d_params.reserve((size_t)needed * sizeof(uint4))) return h->fail(RT_E_NOMEM, "cudaMalloc params");
    cudaError_t e = cudaMemcpy(h->d_params.p, p.data(), (size_t)needed * sizeof(uint4), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return h->cuda_fail(e, "params upload");
    h->d_params_n = needed;
    h->table_dirty = false;
    return RT_OK;
}

// Builds the phase list of `k` epochs and launches the walk.
//
// Bit-exact mode draws the colours as the reference's host loops do.  Fast
// mode (RT_RNG_PHILOX) has no host generator: step s of an epoch flips
// colour s mod NCOL in a fixed cycle (dominoes: the black array, then the
// white; lozenges and rectangle-triangles: 0, 1, 2; triangle dimers: move
// s mod 30 of a sweep over every flip class), and each epoch's seed is its
// 64-bit Philox key.
static rt_status run_schedule(rt_tiler* h, const int64_t* steps, const int64_t* seeds, int k, bool single_walk) {
    if (!h->uploaded) return h->fail(RT_E_STATE, "run before upload");
    cudaSetDevice(h->cfg.device);
    const bool planes = h->cfg.rng == RT_RNG_PLANES;
    const bool fast = h->cfg.rng == RT_RNG_PHILOX || planes;  // counter-based draws, cyclic colours
    int64_t total = 0;
    for (int e = 0; e < k; ++e) {
        if (steps[e] < 0) return h->fail(RT_E_INVAL, "negative step count");
        if (steps[e] > kMaxColourSteps - total) return h->fail(RT_E_INVAL, "more than 2^40 steps in one call");
        total += steps[e];
    }
    h->last_phases = 0;
    h->last_launches = 0;
    if (total == 0) return RT_OK;
    // At most 7 phases per triangle-dimer step; one per step + the final
    // Update for the colour models.
    const int64_t cap_ph = h->kind == 3 ? 7 * total : total + 1;
    // The staging buffers may still feed the previous run's copies.
    cudaEventSynchronize(h->ev_staged);
    if (!h->h_phases.reserve((size_t)cap_ph * 4) || !h->d_phases.reserve((size_t)cap_ph * 4) ||
        !h->h_epoch_start.reserve((size_t)k * 8) || !h->d_epoch_start.reserve((size_t)k * 8) ||
        !h->h_epoch_seed.reserve((size_t)k * 8) || !h->d_epoch_seed.reserve((size_t)k * 8))
        return h->fail(RT_E_NOMEM, "schedule buffers");
    uint32_t* ph = static_cast<uint32_t*>(h->h_phases.p);
    int64_t* es = static_cast<int64_t*>(h->h_epoch_start.p);
    uint64_t* sd = static_cast<uint64_t*>(h->h_epoch_seed.p);
    int64_t at = 0;
    uint32_t prev = NO_COLOUR;
    for (int e = 0; e < k; ++e) {
        es[e] = at;
        if (fast) {
            sd[e] = (uint64_t)seeds[e];
            for (int64_t s = 0; s < steps[e]; ++s) at = fast_step_phases(h->kind, s, ph, at, &prev);
        } else if (h->kind == 0) {
            std::mt19937 mt_rand(seeds[e]);
            sd[e] = single_walk ? (uint32_t)mt_rand() : (uint32_t)seeds[e];  // DominoTiler.cpp:31-32 vs :81-82
            for (int64_t s = 0; s < steps[e]; ++s) {
                const uint32_t r = (uint32_t)(mt_rand() % 2);
                ph[at++] = make_phase(OP_STEP, r, prev, true);
                prev = r;
            }
        } else if (h->kind == 3) {
            // TriangleDimerTiler.cpp:230-348: per step the flip family, the
            // orientation / class and the kind (or parity), and for butterflies
            // the slice and parity, all from one default_random_engine.
            std::default_random_engine generator;
            std::uniform_int_distribution<int> d1(0, 2), d2(0, 1);
            generator.seed(seeds[e]);
            sd[e] = (uint32_t)seeds[e];
            for (int64_t s = 0; s < steps[e]; ++s) {
                const uint32_t kind = (uint32_t)d1(generator), r1 = (uint32_t)d1(generator),
                               r2 = (uint32_t)d2(generator);
                uint32_t p1 = 0, p2 = 0;
                if (kind == 2) {
                    p1 = (uint32_t)d1(generator);
                    p2 = (uint32_t)d2(generator);
                }
                at = td_step_phases(ph, at, kind, r1, r2, p1, p2);
            }
        } else {
            std::default_random_engine generator;
            std::uniform_int_distribution<int> distribution(0, 2);
            generator.seed(seeds[e]);
            sd[e] = (uint32_t)seeds[e];  // Walk passes `seed` to InitTinyMT's uint argument
            for (int64_t s = 0; s < steps[e]; ++s) {
                const uint32_t r = (uint32_t)distribution(generator);
                ph[at++] = make_phase(OP_STEP, r, prev, true);
                prev = r;
            }
        }
    }
    if (h->kind != 3) ph[at++] = make_phase(OP_FINAL, prev, NO_COLOUR, false);
    const int64_t nph = at;

    const int width = h->width;
    const bool uniform = fast || h->table.empty();
    const bool weighted = h->wper > 0;
    if (h->plan_rows != h->rows || h->plan_cols != h->cols || h->plan_nlat != h->nlat || h->plan_uniform != uniform ||
        h->plan_weighted != weighted) {
        rt_status s = choose_plan(h->family, h->cfg.device, h->nlat, h->rows, h->cols, width, uniform, fast, planes,
                                  weighted, h->kernel_choice, h->ctas_hint, h->depth_hint, &h->plan, &h->err);
        if (s != RT_OK) return s;
        h->plan_rows = h->rows;
        h->plan_cols = h->cols;
        h->plan_nlat = h->nlat;
        h->plan_uniform = uniform;
        h->plan_weighted = weighted;
    }
    const int64_t ids = (int64_t)h->rows * h->cols;
    rt_status s = fast ? RT_OK : stage_params(h, ids);
    if (s != RT_OK) return s;
    const size_t xbytes =
        (size_t)h->plan.ctas * 2 * 2 * h->nlat * h->plan.xslots * h->plan.xwords * sizeof(unsigned long long);
    if (!h->d_xbuf.reserve(xbytes)) return h->fail(RT_E_NOMEM, "halo exchange buffer");

    cudaError_t e;
    if ((e = cudaMemcpyAsync(h->d_phases.p, ph, (size_t)nph * 4, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_epoch_start.p, es, (size_t)k * 8, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(h->d_epoch_seed.p, sd, (size_t)k * 8, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
        (e = cudaEventRecord(h->ev_staged, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->d_xbuf.p, 0, xbytes, h->stream)) != cudaSuccess)
        return h->cuda_fail(e, "schedule staging");

    WalkArgs a;
    std::memset(&a, 0, sizeof a);
    for (int l = 0; l < 2; ++l)
        for (int c = 0; c < 8; ++c) a.arr[l][c] = h->d_arr[l][c];
    a.nlat = h->nlat;
    a.n = h->n;
    a.rows = h->rows;
    a.cols = h->cols;
    a.arows = h->arows;
    a.width = width;
    a.rng_kind = fast ? 1 : 0;
    a.chain = h->cfg.chain;
    a.params = uniform ? nullptr : static_cast<const uint4*>(h->d_params.p);
    a.mat1 = kMat1;
    a.mat2 = kMat2;
    a.tmat = kTmat;
    a.phases = static_cast<const uint32_t*>(h->d_phases.p);
    a.nphases = nph;
    a.epoch_start = static_cast<const int64_t*>(h->d_epoch_start.p);
    a.epoch_seed = static_cast<const uint64_t*>(h->d_epoch_seed.p);
    a.nepochs = k;
    family_thresholds(h->family, h->cfg.q, h->cfg.qcmp, a.thr);
    std::memcpy(a.weights, h->cfg.weights, sizeof a.weights);
    a.wper = h->wper;
    std::memcpy(a.wthr, h->wthr, sizeof a.wthr);
    a.xbuf = static_cast<unsigned long long*>(h->d_xbuf.p);
    a.err = static_cast<int*>(h->d_err.p);
    a.timeout_ns = h->timeout_ns;
    a.drop_phase = h->drop_phase;
    s = launch_walk(h->plan, a, h->stream, &h->err);
    if (s != RT_OK) return s;
    h->last_phases = nph;
    h->last_launches = 1;
    return RT_OK;
}

rt_status rt_run(rt_tiler* h, int64_t steps, int64_t seed) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        return run_schedule(h, &steps, &seed, 1, true);
    });
}

rt_status rt_walk(rt_tiler* h, int32_t* tiling, int32_t n, int64_t steps, int64_t seed) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        rt_status s = rt_upload(h, tiling, n);
        if (s == RT_OK) s = run_schedule(h, &steps, &seed, 1, true);
        if (s == RT_OK) s = rt_download(h, tiling);
        return s;
    });
}

rt_status rt_walk_epochs(rt_tiler* h, int32_t* tiling, int32_t n, const int64_t* steps, const int64_t* seeds,
                         int32_t k) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        if (h->kind != 0) return h->fail(RT_E_INVAL, "epoch walks exist for dominoes only (DominoTiler.h:76)");
        if (k < 0 || (k > 0 && (!steps || !seeds))) return h->fail(RT_E_INVAL, "bad epoch arrays");
        rt_status s = rt_upload(h, tiling, n);
        if (s == RT_OK && k > 0) s = run_schedule(h, steps, seeds, k, false);
        if (s == RT_OK) s = rt_download(h, tiling);
        return s;
    });
}

rt_status rt_last_run_info(rt_tiler* h, int64_t* phases, int64_t* launches) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        if (phases) *phases = h->last_phases;
        if (launches) *launches = h->last_launches;
        return RT_OK;
    });
}

// Coupling from the past: the reference's Examples/AztecDiamondCftpEx.cpp:42-68
// built on DominoTiler::Walk(tiling&, vector<long>, vector<long>)
// (DominoTiler.cpp:58-107).  Each trial runs the chains from the maximal and
// the minimal tiling through the same epochs (same seeds, so the same draws)
// -- here as two coupled lattices of one launch -- and compares them on the
// device.  Epoch seeds are successive outputs of std::mt19937(master_seed),
// the newest epoch first, exactly as the example draws them.  Any kernel whose
// update is monotone under shared draws qualifies: the domino heat bath
// (dominokernelCFTP.cl) and both lozenge kernels (a draw either raises the
// site, lowers it, or leaves it, whatever its state; lozengekernel.cl:19-31,
// qlozengekernel.cl:18-29).  Lozenge epochs restart the colour engine and the
// draws from the epoch seed as the domino epoch Walk does.  In fast mode the
// epoch seeds are the epochs' Philox keys.
rt_status rt_cftp(rt_tiler* h, const int32_t* tmax, const int32_t* tmin, int32_t n, int64_t first_steps,
                  int32_t schedule, int64_t master_seed, int32_t max_trials, int32_t* out_tiling,
                  rt_cftp_stats* stats) {
    return guarded([&]() -> rt_status {
        if (!h) return RT_E_INVAL;
        if (h->family != FAM_DOMINO_HB && h->family != FAM_LOZENGE8 && h->family != FAM_QLOZENGE8)
            return h->fail(RT_E_INVAL,
                           "CFTP needs a monotone kernel: the domino heat bath (RT_KERNEL_CFTP, dominokernelCFTP.cl) "
                           "or a lozenge kernel");
        // (bit-plane mode: both admitted families use heat-bath rules, monotone under shared bits)
        if (!tmax || !tmin || first_steps <= 0 || max_trials <= 0 ||
            (schedule != RT_CFTP_DOUBLING && schedule != RT_CFTP_REFERENCE))
            return h->fail(RT_E_INVAL, "bad CFTP arguments");
        rt_status s = rt_upload(h, tmax, n);
        if (s != RT_OK) return s;
        const size_t tb = (size_t)n * n * 4;
        if (!h->d_tiling2.reserve(tb) || !h->d_count.reserve(8) || !h->h_count.reserve(8))
            return h->fail(RT_E_NOMEM, "CFTP buffers");
        cudaError_t e = cudaMemcpyAsync(h->d_tiling2.p, tmin, tb, cudaMemcpyHostToDevice, h->stream);
        if (e != cudaSuccess) return h->cuda_fail(e, "upload of the minimal tiling");
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        std::mt19937 mt(master_seed);
        std::vector<int64_t> steps{first_steps}, seeds{(int64_t)mt()};
        rt_cftp_stats st{};
        double ms_total = 0;
        h->nlat = 2;
        for (int trial = 0; trial < max_trials; ++trial) {
            // Restart both chains at the far end of the current schedule.
            s = launch_split(false, h->elem, h->kind, h->ncol, n, static_cast<int32_t*>(h->d_tiling.p), h->d_arr[0],
                             h->stream, &h->err);
            if (s == RT_OK)
                s = launch_split(false, h->elem, h->kind, h->ncol, n, static_cast<int32_t*>(h->d_tiling2.p), h->d_arr[1],
                                 h->stream, &h->err);
            if (s != RT_OK) break;
            cudaEventRecord(e0, h->stream);
            s = run_schedule(h, steps.data(), seeds.data(), (int)steps.size(), false);
            if (s != RT_OK) break;
            cudaEventRecord(e1, h->stream);
            s = launch_count_diff(h->d_arr[0][0], h->d_arr[1][0], h->per_arr_al * h->ncol,
                                  static_cast<unsigned long long*>(h->d_count.p), h->stream, &h->err);
            if (s != RT_OK) break;
            e = cudaMemcpyAsync(h->h_count.p, h->d_count.p, 8, cudaMemcpyDeviceToHost, h->stream);
            if (e != cudaSuccess) {
                s = h->cuda_fail(e, "coalescence readback");
                break;
            }
            s = rt_synchronize(h);
            if (s != RT_OK) break;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_total += ms;
            st.trials = trial + 1;
            st.total_steps = 0;
            for (int64_t x : steps) st.total_steps += x;
            if (*static_cast<unsigned long long*>(h->h_count.p) == 0) {
                st.coalesced = 1;
                break;
            }
            // Extend further into the past: the reference example prepends
            // 2 * steps[last] (Examples/AztecDiamondCftpEx.cpp:67); the doubling
            // schedule prepends the current total.
            const int64_t add = schedule == RT_CFTP_REFERENCE ? 2 * steps.back() : st.total_steps;
            steps.insert(steps.begin(), add);
            seeds.insert(seeds.begin(), (int64_t)mt());
        }
        h->nlat = 1;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        st.device_ms = ms_total;
        if (stats) *stats = st;
        if (s != RT_OK) return s;
        if (out_tiling) {
            s = rt_download(h, out_tiling);  // lattice 0 = the chain started from the maximal tiling
            if (s != RT_OK) return s;
        }
        return RT_OK;
    });
}

}  // extern "C"
