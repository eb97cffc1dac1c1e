// rt_noalloc.cu -- a walk entry point that allocates no memory of its own.
//
// Some programs that embed this library own every byte of GPU memory
// themselves: they carve a fixed budget out of the device up front and hand
// it out through their own pool, so a library that calls cudaMalloc /
// cudaFree behind their back breaks their accounting (and those calls also
// synchronise the whole device, stalling the host program's other streams).
// rt_walk_device_noalloc serves such callers.  The caller passes the tiling
// as device memory (its input and output); everything else the walk needs --
// the colour arrays, the phase schedule, the halo exchange slots and the
// error word -- lives in one file-scope __device__ array of fixed size
// (kScratchBytes) that every GPU loading the library keeps until the process
// exits.  No cudaMalloc, cudaFree or cudaMallocHost is called here.
//
// The array's name is only a host-side stand-in in host code, so its device
// address is looked up once per device with cudaGetSymbolAddress (with that
// device current) on the first call that uses the device; make that first
// call before any stream capture.  All calls share the one array, so two
// calls whose work overlaps on the same GPU race: serialise them (one stream,
// or one call at a time).  The array keeps whatever the last call left in it;
// the parts that must start at zero are cleared at the start of every call.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <string>

#include "rt_internal.h"
#include "rt_guard.h"
#include "rt_models.cuh"

using rtb::guarded;

using namespace rtb;

namespace {

constexpr size_t kScratchBytes = (size_t)16 << 20;  // 16 MiB per GPU
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_rt_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

void say(char* buf, size_t cap, const char* fmt, ...) {
    if (!buf || cap == 0) return;
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, cap, fmt, ap);
    va_end(ap);
}

// Device address of the scratch array on `dev` (the current device).
rt_status scratch_on(int dev, unsigned char** out, char* eb, size_t ec) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_rt_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            say(eb, ec, "cudaGetSymbolAddress of the scratch array failed: %s", cudaGetErrorString(e));
            return RT_E_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
    return RT_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" rt_status rt_walk_device_noalloc(const rt_config* cfg, int32_t* d_tiling, int32_t n, int64_t steps,
                                            int64_t seed, char* errbuf, size_t errcap) {
    return guarded([&]() -> rt_status {
        if (errbuf && errcap) errbuf[0] = '\0';
        if (!cfg || !d_tiling || steps < 0) {
            say(errbuf, errcap, "null configuration or tiling, or negative step count");
            return RT_E_INVAL;
        }
        // One 4-byte phase per step lives in the array: larger step counts can
        // never fit, and bounding them first keeps the size arithmetic below exact.
        if (steps > (int64_t)(kScratchBytes / 4) - 1) {
            say(errbuf, errcap, "%lld steps do not fit the built-in %zu-byte scratch array", (long long)steps,
                kScratchBytes);
            return RT_E_INVAL;
        }
        int family = -1, ncol = 0, kind = 0, elem = 1;
        if (cfg->model == RT_DOMINO && (cfg->kernel == RT_KERNEL_DEFAULT || cfg->kernel == RT_KERNEL_CFTP)) {
            family = cfg->kernel == RT_KERNEL_CFTP ? FAM_DOMINO_HB : FAM_DOMINO, ncol = 2, kind = 0, elem = 1;
        } else if (cfg->model == RT_LOZENGE && cfg->kernel == RT_KERNEL_DEFAULT) {
            family = FAM_LOZENGE8, ncol = 3, kind = 1, elem = 1;
        } else if (cfg->model == RT_LOZENGE && cfg->kernel == RT_KERNEL_QWEIGHT) {
            family = FAM_QLOZENGE8, ncol = 3, kind = 1, elem = 1;
        } else if (cfg->model == RT_RECTTRI && cfg->kernel == RT_KERNEL_DEFAULT) {
            family = FAM_RECTTRI, ncol = 3, kind = 2, elem = 4;
        }
        if (family < 0 || cfg->rng != RT_RNG_TINYMT) {
            say(errbuf, errcap, "unsupported model / kernel / rng combination");
            return RT_E_INVAL;
        }
        if (family == FAM_QLOZENGE8 && !(cfg->q >= 0.0 && std::isfinite(cfg->q))) {
            say(errbuf, errcap, "q must be a finite non-negative number");
            return RT_E_INVAL;
        }
        if ((kind == 0 && (n < 6 || n % 2 != 0)) || (kind != 0 && (n < 9 || n % 3 != 0))) {
            say(errbuf, errcap, "tiling side %d not allowed for this model", (int)n);
            return RT_E_INVAL;
        }
        // The colour arrays alone (n x n bytes at least) must fit the array.
        if ((int64_t)n * n > (int64_t)kScratchBytes) {
            say(errbuf, errcap, "tiling side %d does not fit the built-in %zu-byte scratch array", (int)n, kScratchBytes);
            return RT_E_INVAL;
        }
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev ||
            cfg->device >= kMaxDevices) {
            say(errbuf, errcap, "no CUDA device with ordinal %d", (int)cfg->device);
            return RT_E_NODEVICE;
        }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major != 10 || !prop.cooperativeLaunch) {
            say(errbuf, errcap, "device %d is not an sm_100 device with cooperative launches", (int)cfg->device);
            return RT_E_NODEVICE;
        }
        cudaError_t e = cudaSetDevice(cfg->device);
        if (e != cudaSuccess) {
            say(errbuf, errcap, "cudaSetDevice: %s", cudaGetErrorString(e));
            return RT_E_CUDA;
        }
        unsigned char* base = nullptr;
        rt_status s = scratch_on(cfg->device, &base, errbuf, errcap);
        if (s != RT_OK) return s;
        cudaStream_t stream = static_cast<cudaStream_t>(cfg->stream);

        const int width = n / ncol;
        int rows, cols;
        if (kind == 0) {
            rows = n - 2, cols = n / 2 - 2;
        } else {
            rows = n, cols = n / 3;
        }
        std::string perr;  // filled only on a failure path
        WalkPlan plan;
        // The kernel rt_walk would run for this walk (word kernel for the int8
        // models, the generic walk kernel otherwise).
        s = choose_plan(family, cfg->device, 1, rows, cols, width, true, false, false, false, 0, 0, 0, &plan, &perr);
        if (s != RT_OK) {
            say(errbuf, errcap, "%s", perr.c_str());
            return s;
        }

        // Scratch layout: colour arrays | phases | epoch start + seed | exchange slots | error word.
        const size_t per_arr = align256((size_t)n * width * elem);
        const int64_t nph = steps > 0 ? steps + 1 : 0;
        const size_t off_ph = per_arr * ncol;
        const size_t off_ep = off_ph + align256((size_t)nph * 4);
        const size_t off_x = off_ep + 256;
        const size_t xbytes = (size_t)plan.ctas * 2 * 2 * plan.xslots * plan.xwords * sizeof(unsigned long long);
        const size_t off_err = off_x + align256(xbytes);
        const size_t need = off_err + 256;
        if (need > kScratchBytes) {
            say(errbuf, errcap,
                "walk needs %zu bytes of scratch (tiling side %d, %lld steps); the built-in array holds %zu",
                need, (int)n, (long long)steps, kScratchBytes);
            return RT_E_INVAL;
        }
        void* arr[3] = {base, base + per_arr, ncol > 2 ? base + 2 * per_arr : nullptr};

        s = launch_split(false, elem, kind, ncol, n, d_tiling, arr, stream, &perr);
        if (s != RT_OK) {
            say(errbuf, errcap, "%s", perr.c_str());
            return s;
        }
        if (nph > 0) {
            // Colour schedule, drawn as the reference's Walk draws it (std::mt19937
            // for dominoes, DominoTiler.cpp:31-42; default_random_engine +
            // uniform_int_distribution<int>(0,2) otherwise, LozengeTiler.cpp:50-55),
            // staged through a small stack buffer.
            uint32_t chunk[2048];
            int64_t done = 0;
            int fill = 0;
            uint32_t prev = NO_COLOUR;
            uint64_t tseed;
            std::mt19937 mt(seed);
            std::default_random_engine lcg;
            std::uniform_int_distribution<int> dist(0, 2);
            if (kind == 0) {
                tseed = (uint32_t)mt();
            } else {
                lcg.seed(seed);
                tseed = (uint32_t)seed;
            }
            auto flush = [&]() -> cudaError_t {
                if (fill == 0) return cudaSuccess;
                const cudaError_t ce = cudaMemcpyAsync(base + off_ph + (size_t)done * 4, chunk, (size_t)fill * 4,
                                                       cudaMemcpyHostToDevice, stream);
                done += fill;
                fill = 0;
                return ce;
            };
            for (int64_t st = 0; st < steps; ++st) {
                const uint32_t r = kind == 0 ? (uint32_t)(mt() % 2) : (uint32_t)dist(lcg);
                chunk[fill++] = make_phase(OP_STEP, r, prev, true);
                prev = r;
                if (fill == 2048 && (e = flush()) != cudaSuccess) break;
            }
            if (e == cudaSuccess) {
                chunk[fill++] = make_phase(OP_FINAL, prev, NO_COLOUR, false);
                e = flush();
            }
            const int64_t ep_start = 0;
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(base + off_ep, &ep_start, 8, cudaMemcpyHostToDevice, stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(base + off_ep + 8, &tseed, 8, cudaMemcpyHostToDevice, stream);
            // The exchange slots and the error word must start at zero on every call.
            if (e == cudaSuccess) e = cudaMemsetAsync(base + off_x, 0, xbytes, stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(base + off_err, 0, sizeof(int), stream);
            if (e != cudaSuccess) {
                say(errbuf, errcap, "staging the schedule: %s", cudaGetErrorString(e));
                return RT_E_CUDA;
            }
            // Both pageable copies above are from stack memory; they complete
            // before the kernel runs on the same stream.
            e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) {
                say(errbuf, errcap, "synchronize: %s", cudaGetErrorString(e));
                return RT_E_CUDA;
            }

            WalkArgs a;
            std::memset(&a, 0, sizeof a);
            a.arr[0][0] = arr[0];
            a.arr[0][1] = arr[1];
            a.arr[0][2] = arr[2];
            a.nlat = 1;
            a.n = n;
            a.rows = rows;
            a.cols = cols;
            a.arows = n;
            a.width = width;
            a.rng_kind = 0;
            a.params = nullptr;
            a.mat1 = 0x8f7011eeu;  // TinyMT32J, src/TinyMT/tinymt32def.h:47-49
            a.mat2 = 0xfc78ff1fu;
            a.tmat = 0x3793fdffu;
            a.phases = reinterpret_cast<const uint32_t*>(base + off_ph);
            a.nphases = nph;
            a.epoch_start = reinterpret_cast<const int64_t*>(base + off_ep);
            a.epoch_seed = reinterpret_cast<const uint64_t*>(base + off_ep + 8);
            a.nepochs = 1;
            family_thresholds(family, cfg->q, cfg->qcmp, a.thr);
            std::memcpy(a.weights, cfg->weights, sizeof a.weights);
            a.xbuf = reinterpret_cast<unsigned long long*>(base + off_x);
            a.err = reinterpret_cast<int*>(base + off_err);
            a.timeout_ns = 5000000000ull;
            a.drop_phase = -1;
            s = launch_walk(plan, a, stream, &perr);
            if (s != RT_OK) {
                say(errbuf, errcap, "%s", perr.c_str());
                return s;
            }
            e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) {
                say(errbuf, errcap, "walk failed: %s", cudaGetErrorString(e));
                return RT_E_CUDA;
            }
            // The caller's tiling is written back only after a walk that finished:
            // a walk stopped by a timed-out wait leaves it as it was.
            int code = 0;
            e = cudaMemcpy(&code, base + off_err, sizeof code, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                say(errbuf, errcap, "error word readback: %s", cudaGetErrorString(e));
                return RT_E_CUDA;
            }
            if (code & ERR_TIMEOUT) {
                say(errbuf, errcap, "a bounded wait between CTAs timed out; walk aborted");
                return RT_E_TIMEOUT;
            }
            if (code) {
                say(errbuf, errcap, "device error word %d", code);
                return RT_E_CUDA;
            }
        }
        s = launch_split(true, elem, kind, ncol, n, d_tiling, arr, stream, &perr);
        if (s != RT_OK) {
            say(errbuf, errcap, "%s", perr.c_str());
            return s;
        }
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) {
            say(errbuf, errcap, "merge failed: %s", cudaGetErrorString(e));
            return RT_E_CUDA;
        }
        return RT_OK;
    });
}
