// C entry points over the reference's own host classes, for ctypes.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref).  This file is compiled together with
// the reference's unmodified src/*/*Tiler.cpp, src/common/common.cpp and
// src/TinyMT/file_reader.cpp, and with its kernels (src/*/*.cl) compiled as
// C++ through oracle/shim.  It lets the tests and the CPU baseline call the
// reference's Walk, builders, height functions and SVG writers directly.
//
// The only algorithmic code here is QLozengeLoop::Walk: the reference ships
// the q-weighted kernel (src/Lozenge/qlozengekernel.cl, int* tiling) but its
// LozengeTiler::Walk (src/Lozenge/LozengeTiler.cpp:18-88) uploads char
// arrays, so no reference host loop drives that kernel correctly.  The loop
// below is LozengeTiler.cpp:18-88 with int arrays, nothing else changed.
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "src/Domino/DominoTiler.h"
#include "src/Lozenge/LozengeTiler.h"
#include "src/RectTriangle/RectTriangleTiler.h"
#include "src/TinyMT/file_reader.h"
#include "src/TriangleDimer/TriangleDimerTiler.h"

namespace {

class QLozengeLoop {
    cl::Context context;
    cl::CommandQueue queue;
    cl::Program program;
    cl::make_kernel<cl::Buffer, const int> InitTinyMT;
    cl::make_kernel<cl::Buffer, cl::Buffer, const int> RotateTiles;
    cl::make_kernel<cl::Buffer, cl::Buffer, cl::Buffer, const int, const int> UpdateTiles;
    cl::Buffer tinymtparams;

public:
    QLozengeLoop(cl::Context c, cl::CommandQueue q, std::vector<cl::Device> devices, std::string source)
        : context(c),
          queue(q),
          program(LoadCLProgram(context, devices, source)),
          InitTinyMT(program, "InitTinyMT"),
          RotateTiles(program, "RotateTiles"),
          UpdateTiles(program, "UpdateTiles") {}

    void LoadTinyMT(std::string params, int size) { tinymtparams = get_params_buffer(params, context, queue, size); }

    void Walk(tiling& t, int steps, long seed) {
        int N = std::sqrt(t.size());
        int M = N / 3;
        std::vector<int> h_vR(N * M, 0), h_vB(N * M, 0), h_vG(N * M, 0);
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                const int c = ((j - i) % 3 + 3) % 3;
                (c == 0 ? h_vR : c == 1 ? h_vB : h_vG)[i * M + j / 3] = t[i * N + j];
            }
        cl::Buffer d_vR(context, h_vR.begin(), h_vR.end(), CL_FALSE);
        cl::Buffer d_vB(context, h_vB.begin(), h_vB.end(), CL_FALSE);
        cl::Buffer d_vG(context, h_vG.begin(), h_vG.end(), CL_FALSE);
        InitTinyMT(cl::EnqueueArgs(queue, cl::NDRange(N * (N / 3))), tinymtparams, seed);
        std::default_random_engine generator;
        std::uniform_int_distribution<int> distribution(0, 2);
        generator.seed(seed);
        for (int i = 0; i < steps; ++i) {
            int r = distribution(generator);
            if (r == 0) {
                RotateTiles(cl::EnqueueArgs(queue, cl::NDRange(N, N / 3)), tinymtparams, d_vR, N);
                UpdateTiles(cl::EnqueueArgs(queue, cl::NDRange(N, N / 3)), d_vR, d_vB, d_vG, N, 0);
            } else if (r == 1) {
                RotateTiles(cl::EnqueueArgs(queue, cl::NDRange(N, N / 3)), tinymtparams, d_vB, N);
                UpdateTiles(cl::EnqueueArgs(queue, cl::NDRange(N, N / 3)), d_vB, d_vG, d_vR, N, 1);
            } else {
                RotateTiles(cl::EnqueueArgs(queue, cl::NDRange(N, N / 3)), tinymtparams, d_vG, N);
                UpdateTiles(cl::EnqueueArgs(queue, cl::NDRange(N, N / 3)), d_vG, d_vR, d_vB, N, 2);
            }
        }
        cl::copy(queue, d_vR, h_vR.begin(), h_vR.end());
        cl::copy(queue, d_vB, h_vB.begin(), h_vB.end());
        cl::copy(queue, d_vG, h_vG.begin(), h_vG.end());
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) {
                const int c = ((j - i) % 3 + 3) % 3;
                t[i * N + j] = (c == 0 ? h_vR : c == 1 ? h_vB : h_vG)[i * M + j / 3];
            }
    }
};

// M_QLOZENGE_F32: the same loop over qlozengekernel.cl compiled with single-precision
// arithmetic (k_qlozenge_f32.cpp), the comparison of an fp32-only OpenCL device.
enum Model {
    M_DOMINO = 0,
    M_DOMINO_CFTP = 1,
    M_LOZENGE = 2,
    M_QLOZENGE = 3,
    M_RECTTRI = 4,
    M_TRIDIMER = 5,
    M_QLOZENGE_F32 = 6
};

struct Handle {
    int model;
    cl::Context context;
    cl::CommandQueue queue;
    std::vector<cl::Device> devices;
    DominoTiler* domino = nullptr;
    LozengeTiler* lozenge = nullptr;
    QLozengeLoop* qlozenge = nullptr;
    RectTriangleTiler* recttri = nullptr;
    TriangleDimerTiler* tridimer = nullptr;
    ~Handle() {
        delete domino;
        delete lozenge;
        delete qlozenge;
        delete recttri;
        delete tridimer;
    }
};

const char* kProgramIds[] = {"domino", "domino_cftp", "lozenge", "qlozenge", "recttri", "tridimer", "qlozenge_f32"};

long emit(const std::vector<int>& v, int* out, long cap) {
    const long n = static_cast<long>(v.size());
    if (out && cap >= n) std::copy(v.begin(), v.end(), out);
    return n;
}

}  // namespace

extern "C" {

int ref_set_threads(int n) {
    clshim::set_num_threads(n);
    return clshim::num_threads();
}

// Writes `count` parameter lines in the layout src/TinyMT/file_reader.cpp:139-166
// parses (mat1, mat2, tmat after the 3rd, 4th and 5th comma, hexadecimal).
int ref_write_params(const char* path, long count, unsigned mat1, unsigned mat2, unsigned tmat) {
    FILE* f = std::fopen(path, "w");
    if (!f) return -1;
    std::fprintf(f, "# tinymt32 parameter table written for the oracle\n");
    for (long i = 0; i < count; ++i) std::fprintf(f, "tinymt32,%ld,127,%08x,%08x,%08x,0\n", i, mat1, mat2, tmat);
    std::fclose(f);
    return 0;
}

void* ref_tiler_create(int model, const char* params_path, long n_params) {
    if (model < 0 || model > 6) return nullptr;
    try {
        Handle* h = new Handle();
        h->model = model;
        h->devices.assign(1, cl::Device());
        cl_int err = 0;
        clshim::set_next_program(kProgramIds[model]);
        const std::string src = "/dev/null";  // the fake runtime binds kernels by program id
        switch (model) {
            case M_DOMINO:
            case M_DOMINO_CFTP:
                h->domino = new DominoTiler(h->context, h->queue, h->devices, src, err);
                h->domino->LoadTinyMT(params_path, static_cast<int>(n_params));
                break;
            case M_LOZENGE:
                h->lozenge = new LozengeTiler(h->context, h->queue, h->devices, src, err);
                h->lozenge->LoadTinyMT(params_path, static_cast<int>(n_params));
                break;
            case M_QLOZENGE:
            case M_QLOZENGE_F32:
                h->qlozenge = new QLozengeLoop(h->context, h->queue, h->devices, src);
                h->qlozenge->LoadTinyMT(params_path, static_cast<int>(n_params));
                break;
            case M_RECTTRI:
                h->recttri = new RectTriangleTiler(h->context, h->queue, h->devices, src, err);
                h->recttri->LoadTinyMT(params_path, static_cast<int>(n_params));
                break;
            case M_TRIDIMER:
                h->tridimer = new TriangleDimerTiler(h->context, h->queue, h->devices, src, err);
                h->tridimer->LoadTinyMT(params_path, static_cast<int>(n_params));
                break;
        }
        return h;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_tiler_create: %s\n", e.what());
        return nullptr;
    }
}

void ref_tiler_destroy(void* p) { delete static_cast<Handle*>(p); }

int ref_tiler_walk(void* p, int* t, long tlen, long steps, long seed) {
    Handle* h = static_cast<Handle*>(p);
    if (!h) return -1;
    try {
        tiling T(t, t + tlen);
        switch (h->model) {
            case M_DOMINO:
            case M_DOMINO_CFTP:
                h->domino->Walk(T, steps, seed);
                break;
            case M_LOZENGE:
                h->lozenge->Walk(T, static_cast<int>(steps), seed);
                break;
            case M_QLOZENGE:
            case M_QLOZENGE_F32:
                h->qlozenge->Walk(T, static_cast<int>(steps), seed);
                break;
            case M_RECTTRI:
                h->recttri->Walk(T, static_cast<int>(steps), seed);
                break;
            case M_TRIDIMER:
                h->tridimer->Walk(T, static_cast<int>(steps), seed);
                break;
        }
        std::copy(T.begin(), T.end(), t);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_tiler_walk: %s\n", e.what());
        return -2;
    }
}

// DominoTiler::Walk(tiling&, vector<long> steps, vector<long> seeds)
// (src/Domino/DominoTiler.cpp:58-107).
int ref_tiler_walk_epochs(void* p, int* t, long tlen, const long* steps, const long* seeds, int k) {
    Handle* h = static_cast<Handle*>(p);
    if (!h || !h->domino) return -1;
    try {
        tiling T(t, t + tlen);
        std::vector<long> st(steps, steps + k), se(seeds, seeds + k);
        h->domino->Walk(T, st, se);
        std::copy(T.begin(), T.end(), t);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_tiler_walk_epochs: %s\n", e.what());
        return -2;
    }
}

// Static builders, height functions and conversions.  Returns the result
// length; the result is written when out != NULL and cap is large enough.
long ref_build(int what, const int* a, long alen, const int* b, long blen, int p0, int p1, int* out, long cap) {
    std::vector<int> A(a ? a : nullptr, a ? a + alen : nullptr), B(b ? b : nullptr, b ? b + blen : nullptr);
    switch (what) {
        case 0: return emit(DominoTiler::Rectangle(p0, p1), out, cap);
        case 1: return emit(DominoTiler::AztecDiamond(p0), out, cap);
        case 2: return emit(DominoTiler::AztecRectangle(p0, A), out, cap);
        case 3: return emit(DominoTiler::MaxTiling(A), out, cap);
        case 4: return emit(DominoTiler::MinTiling(A), out, cap);
        case 5: return emit(DominoTiler::DomainToVertices(A), out, cap);
        case 6: return emit(DominoTiler::TilingToDomain(A), out, cap);
        case 7: return emit(DominoTiler::HeightfuncToTiling(A, B), out, cap);
        case 8: return emit(DominoTiler::TilingToHeightfunc(A, B), out, cap);
        case 10: return emit(LozengeTiler::AlmostHexDomain(p0, p1), out, cap);
        case 11: return emit(LozengeTiler::MaxTiling(A), out, cap);
        case 12: return emit(LozengeTiler::MinTiling(A), out, cap);
        case 13: return emit(LozengeTiler::DomainToVertices(A), out, cap);
        case 14: return emit(LozengeTiler::TilingToDomain(A), out, cap);
        case 15: return emit(LozengeTiler::HeightfuncToTiling(A, B), out, cap);
        case 16: return emit(LozengeTiler::TilingToHeightfunc(A, B), out, cap);
        case 20: return emit(RectTriangleTiler::maxHex(p0), out, cap);
        case 21: return emit(RectTriangleTiler::minHex(p0), out, cap);
        case 22: return emit(RectTriangleTiler::slopeHex(p0), out, cap);
        case 23: return emit(RectTriangleTiler::LozengeToRectTriangle(A, B), out, cap);
        case 30: return emit(TriangleDimerTiler::IceCreamCone(p0, p1), out, cap);
        case 31: return emit(TriangleDimerTiler::TestButterfly(p0), out, cap);
        case 32: return emit(TriangleDimerTiler::TilingToTriangleFlips(A), out, cap);
        case 33: return emit(TriangleDimerTiler::TilingToButterflyFlips(A), out, cap);
        case 34: return emit(TriangleDimerTiler::TilingToVertices(A), out, cap);
        case 35: return emit(TriangleDimerTiler::TilingToDomain(A), out, cap);
        case 36: return emit(TriangleDimerTiler::DimerIndicator(A, p0), out, cap);
        default: return -1;
    }
}

// SVG and text writers.
int ref_write(int what, const int* a, long alen, const int* b, long blen, const char* filename) {
    std::vector<int> A(a ? a : nullptr, a ? a + alen : nullptr), B(b ? b : nullptr, b ? b + blen : nullptr);
    const std::string f(filename);
    switch (what) {
        case 0: DominoTiler::DomainToSVG(A, f); return 0;
        case 1: DominoTiler::TilingToSVG(A, f); return 0;
        case 2: DominoTiler::MayaToSVG(A, f); return 0;
        case 3: DominoTiler::DimerToSVG(A, f); return 0;
        case 4: DominoTiler::DimerToSVG(A, B, f); return 0;
        case 10: LozengeTiler::DomainToSVG(A, f); return 0;
        case 11: LozengeTiler::TilingToSVG(A, f); return 0;
        case 12: LozengeTiler::DimerToSVG(A, f); return 0;
        case 13: LozengeTiler::DimerToSVG(A, B, f); return 0;
        case 14: LozengeTiler::PrintDomain(A, f); return 0;
        case 20: RectTriangleTiler::TilingToSVG(A, f); return 0;
        case 30: TriangleDimerTiler::DomainToSVG(A, f); return 0;
        case 31: TriangleDimerTiler::TilingToSVG(A, f); return 0;
        case 32: TriangleDimerTiler::DimerToSVG(A, f); return 0;
        case 33: TriangleDimerTiler::DimerToSVG(A, B, f); return 0;
        case 40: SaveMatrix(A, f); return 0;
        default: return -1;
    }
}

}  // extern "C"
