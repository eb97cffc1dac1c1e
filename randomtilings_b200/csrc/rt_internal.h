// rt_internal.h -- declarations shared by the C-ABI layer and the kernels.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/rt_b200.h"

namespace rtb {

struct WalkArgs;

enum Family : int {
    FAM_DOMINO = 0,      // dominokernel.cl, int8
    FAM_DOMINO_HB = 1,   // dominokernelCFTP.cl, int8
    FAM_LOZENGE8 = 2,    // lozengekernel.cl, int8
    FAM_QLOZENGE8 = 3,   // qlozengekernel.cl; int8 (the reference's int states are below 64)
    FAM_RECTTRI = 4,     // recttrianglekernel.cl, int32
    FAM_TRIDIMER = 5     // triangledimerkernel.cl, 8 int32 arrays
};

// The most colour steps one call may ask for, about 1.1e12: weeks of device
// time even on small lattices.  Every entry point that sizes a schedule or a
// phase list from a step or sweep count refuses larger counts first, so no
// size computed from a count can wrap.
constexpr int64_t kMaxColourSteps = int64_t(1) << 40;

// The largest tiling side a walk accepts: the kernels index a lattice with
// 32-bit integers, and a side of 32,767 keeps every index below 2^31.
constexpr int kMaxTilingSide = 32767;

struct WalkPlan {
    int items = 0;
    int block = 0;
    int rows_per_cta = 0;
    int ctas = 0;
    size_t smem = 0;
    int wpad = 0;    // shared-memory row stride (elements)
    int xwords = 0;  // exchange words per halo row
    int xslots = 1;  // arrays exchanged per phase
    int depth = 1;   // bit-plane kernel: phases per halo exchange
    int pwords = 0;  // bit-plane kernel: words per row
    const void* fn = nullptr;
};

rt_status plan_walk(int family, int device, int nlat, int rows, int cols, int width, bool uniform, bool philox,
                    WalkPlan* plan, std::string* err);
rt_status launch_walk(const WalkPlan& plan, WalkArgs& args, cudaStream_t stream, std::string* err);
// Word-parallel kernel of the int8 models (rt_word.cu): uniform TinyMT32J
// parameters or fast mode.  ctas_hint <= 0: one CTA per SM.
bool word_family(int family);
// weighted: the instantiation that reads per-site thresholds (WalkArgs::wper > 0).
rt_status plan_word_walk(int family, int device, int nlat, int rows, int width, bool philox, int ctas_hint,
                         WalkPlan* plan, std::string* err, bool weighted = false);
// Bit-plane kernel of the int8 models (rt_plane.cu, RT_RNG_PLANES).
// ctas_hint / depth_hint <= 0: one CTA per SM / the largest depth up to 8.
rt_status plan_plane_walk(int family, int device, int nlat, int rows, int width, int ctas_hint, int depth_hint,
                          WalkPlan* plan, std::string* err);
// The kernel a walk runs on, as every walk entry point chooses it: the
// bit-plane kernel in RT_RNG_PLANES mode; otherwise the word kernel for the
// int8 models with uniform generator parameters (unless kernel_choice = 1),
// falling back to the generic walk kernel for every other case and for any
// band the word kernel cannot hold (kernel_choice = 2 forbids the fallback).
rt_status choose_plan(int family, int device, int nlat, int rows, int cols, int width, bool uniform, bool fast,
                      bool planes, bool weighted, int kernel_choice, int ctas_hint, int depth_hint, WalkPlan* plan,
                      std::string* err);
// kind: 0 domino, 1 lozenge, 2 rect-triangle, 3 triangle-dimer (merge only).
rt_status launch_split(bool merge, int elem_bytes, int kind, int ncol, int n, int32_t* tiling, void* const* arr,
                       cudaStream_t stream, std::string* err);

// Fast-mode schedules (rt_capi.cu).  kind: 0 domino, 1 lozenge,
// 2 rect-triangle, 3 triangle dimer.  fast_step_phases appends the phases of
// step s of an epoch; fast_phases appends a whole walk of `steps` steps
// (with the final Update of the colour models).
int64_t fast_step_phases(int kind, int64_t s, uint32_t* ph, int64_t at, uint32_t* prev);
void fast_phases(int kind, int64_t steps, std::vector<uint32_t>& ph);
// Integer threshold K with (k * 2^-23 < x) <=> (k < K) for k in [0, 2^23).
uint32_t below_threshold(double x);
// Integer acceptance thresholds of a kernel family on the 23-bit draw.
void family_thresholds(int family, double q, int qcmp, uint32_t thr[4]);

// Vertex kinds and in-domain edge bits of a domino / lozenge domain
// (rt_host.cpp), the graph of the height-function projection.
bool lipschitz_graph(int model, const int32_t* d, int64_t dlen, int* n_out, std::vector<uint8_t>* kind,
                     std::vector<uint8_t>* edges);

// Boundary heights of a domino / lozenge domain (rt_host.cpp): the vertex
// indices reachable from the first boundary vertex along boundary edges and
// their heights (0 at the start), in visiting order; vertex side in *n_out.
bool boundary_walk(int model, const int32_t* d, int64_t dlen, int* n_out, std::vector<int64_t>* idx,
                   std::vector<int32_t>* h);

// Host split of a triangle-dimer tiling into its eight M x M arrays
// (H, L, R, U, D, BH, BL, BR), rt_host.cpp.
void td_split_host(const int32_t* t, int n, int32_t* arrays);

// Counts differing 32-bit words of a and b (bytes must be a multiple of 4).
rt_status launch_count_diff(const void* a, const void* b, size_t bytes, unsigned long long* d_count,
                            cudaStream_t stream, std::string* err);

}  // namespace rtb
