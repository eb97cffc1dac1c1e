// Tilers.hpp -- header-only C++ layer with the reference's class and method
// names over the C ABI of librt_b200.so.
//
// A caller of GPUTilings/RandomTilings keeps its code: `tiling`, `domain` and
// `heightfunc` are std::vector<int> (src/common/common.h:43-45), Walk mutates
// the tiling in place, builders return vectors by value.  The only change is
// the constructor: the reference takes (cl::Context, cl::CommandQueue,
// std::vector<cl::Device>, std::string kernelFile, cl_int&) and compiles an
// OpenCL program; here it takes a device ordinal and the kernel variant.
// Failures throw rt::Error (the reference throws cl::Error or exits).
#pragma once

#include <climits>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../rt_b200.h"
#include "../rt_b200_host.h"
#include "../rt_b200_sixv.h"
#include "../rt_b200_svg.h"

namespace rt {

typedef std::vector<int> domain;
typedef std::vector<int> heightfunc;
typedef std::vector<int> tiling;

class Error : public std::runtime_error {
public:
    Error(rt_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    rt_status status;
};

namespace detail {
inline void check(rt_status s, rt_tiler* h) {
    if (s != RT_OK) throw Error(s, rt_last_error(h));
}
inline int side(const std::vector<int>& v) {
    int n = 0;
    while ((long long)(n + 1) * (n + 1) <= (long long)v.size()) ++n;
    if ((long long)n * n != (long long)v.size()) throw Error(RT_E_INVAL, "array is not square");
    return n;
}
// Calls a builder of rt_b200_host.h twice: size query, then fill.
template <class F>
std::vector<int> build(F f) {
    int64_t len = 0;
    check(f(nullptr, 0, &len), nullptr);
    std::vector<int> out((size_t)len);
    check(f(reinterpret_cast<int32_t*>(out.data()), len, &len), nullptr);
    return out;
}
inline const int32_t* p(const std::vector<int>& v) { return reinterpret_cast<const int32_t*>(v.data()); }
}  // namespace detail

class TilerBase {
protected:
    rt_tiler* h_ = nullptr;
    explicit TilerBase(int32_t model, int device, int32_t kernel) {
        rt_config cfg;
        rt_config_default(&cfg, model);
        cfg.device = device;
        cfg.kernel = kernel;
        detail::check(rt_create(&cfg, &h_), nullptr);
    }
    explicit TilerBase(const rt_config& cfg) { detail::check(rt_create(&cfg, &h_), nullptr); }

public:
    TilerBase(const TilerBase&) = delete;
    TilerBase& operator=(const TilerBase&) = delete;
    ~TilerBase() {
        if (h_) rt_destroy(h_);
    }
    // LoadTinyMT(std::string params, int size): the tinymt32dc parameter table.
    void LoadTinyMT(const std::string& params, int size) {
        detail::check(rt_load_rng_params(h_, params.c_str(), size), h_);
    }
    // Walk(tiling&, steps, seed).
    void Walk(tiling& t, long steps, long seed) {
        detail::check(rt_walk(h_, reinterpret_cast<int32_t*>(t.data()), detail::side(t), steps, seed), h_);
    }
    rt_tiler* handle() { return h_; }
    // Coupling from the past (Examples/AztecDiamondCftpEx.cpp:42-68) on a
    // monotone kernel; returns the coalesced tiling, stats in *st.
    tiling CFTP(const tiling& tmax, const tiling& tmin, long first_steps, long master_seed,
                int32_t schedule = RT_CFTP_DOUBLING, int max_trials = 30, rt_cftp_stats* st = nullptr) {
        if (tmax.size() != tmin.size()) throw Error(RT_E_INVAL, "tmax and tmin differ in size");
        tiling out(tmax.size());
        rt_cftp_stats local{};
        detail::check(rt_cftp(h_, detail::p(tmax), detail::p(tmin), detail::side(tmax), first_steps, schedule,
                              master_seed, max_trials, reinterpret_cast<int32_t*>(out.data()), st ? st : &local),
                      h_);
        return out;
    }
    // src/common/common.h:50-69
    static void SaveMatrix(const std::vector<int>& a, const std::string& f) {
        detail::check(rt_save_matrix(detail::p(a), a.size(), f.c_str()), nullptr);
    }
    static std::vector<int> LoadMatrix(const std::string& f) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) { return rt_load_matrix(f.c_str(), o, c, l); });
    }
};

// src/Domino/DominoTiler.h:43-115
class DominoTiler : public TilerBase {
public:
    // cftp = true selects dominokernelCFTP.cl (monotone heat bath).
    explicit DominoTiler(int device = 0, bool cftp = false)
        : TilerBase(RT_DOMINO, device, cftp ? RT_KERNEL_CFTP : RT_KERNEL_DEFAULT) {}
    explicit DominoTiler(const rt_config& cfg) : TilerBase(cfg) {}
    using TilerBase::Walk;
    // Walk(tiling&, vector<long> steps, vector<long> seeds): epochs, TinyMT re-seeded per epoch.
    void Walk(tiling& t, const std::vector<long>& steps, const std::vector<long>& seeds) {
        if (steps.size() != seeds.size()) throw Error(RT_E_INVAL, "steps and seeds differ in length");
        std::vector<int64_t> st(steps.begin(), steps.end()), se(seeds.begin(), seeds.end());
        detail::check(rt_walk_epochs(h_, reinterpret_cast<int32_t*>(t.data()), detail::side(t), st.data(), se.data(),
                                     (int32_t)st.size()),
                      h_);
    }
    // Periodic domino weights for the heat bath (rt_set_domino_weights): P x P
    // row-major tables, P = 1, 2 or 4; P = 0 returns to uniform weights.
    void SetWeights(int P, const std::vector<double>& wh, const std::vector<double>& wv) {
        if (P != 0 && (wh.size() != (size_t)(P * P) || wv.size() != (size_t)(P * P)))
            throw Error(RT_E_INVAL, "weight tables must hold P x P values");
        detail::check(rt_set_domino_weights(h_, P, P ? wh.data() : nullptr, P ? wv.data() : nullptr), h_);
    }
    static domain Rectangle(int M, int N) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) { return rt_domino_rectangle(M, N, o, c, l); });
    }
    static domain AztecRectangle(int N, const std::vector<int>& remove) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_domino_aztec_rectangle(N, detail::p(remove), (int32_t)remove.size(), o, c, l);
        });
    }
    static domain AztecDiamond(int N) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) { return rt_domino_aztec(N, o, c, l); });
    }
    static tiling MaxTiling(const domain& d) {
        return detail::build(
            [&](int32_t* o, int64_t c, int64_t* l) { return rt_domino_max_tiling(detail::p(d), d.size(), o, c, l); });
    }
    static tiling MinTiling(const domain& d) {
        return detail::build(
            [&](int32_t* o, int64_t c, int64_t* l) { return rt_domino_min_tiling(detail::p(d), d.size(), o, c, l); });
    }
    static std::vector<int> DomainToVertices(const domain& d) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_domino_domain_to_vertices(detail::p(d), d.size(), o, c, l);
        });
    }
    static domain TilingToDomain(const tiling& t) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_domino_tiling_to_domain(detail::p(t), t.size(), o, c, l);
        });
    }
    static tiling HeightfuncToTiling(const heightfunc& hf, const domain& d) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_domino_height_to_tiling(detail::p(hf), hf.size(), detail::p(d), d.size(), o, c, l);
        });
    }
    static heightfunc TilingToHeightfunc(const tiling& t, const domain& d) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_domino_tiling_to_height(detail::p(t), t.size(), detail::p(d), d.size(), o, c, l);
        });
    }
    static void DomainToSVG(const domain& d, const std::string& f) {
        detail::check(rt_domino_domain_svg(detail::p(d), d.size(), f.c_str()), nullptr);
    }
    static void TilingToSVG(const tiling& t, const std::string& f) {
        detail::check(rt_domino_tiling_svg(detail::p(t), t.size(), f.c_str()), nullptr);
    }
    static void MayaToSVG(const tiling& t, const std::string& f) {
        detail::check(rt_domino_maya_svg(detail::p(t), t.size(), f.c_str()), nullptr);
    }
    static void DimerToSVG(const tiling& t, const std::string& f) {
        detail::check(rt_domino_dimer_svg(detail::p(t), t.size(), nullptr, 0, f.c_str()), nullptr);
    }
    static void DimerToSVG(const tiling& t, const domain& d, const std::string& f) {
        detail::check(rt_domino_dimer_svg(detail::p(t), t.size(), detail::p(d), d.size(), f.c_str()), nullptr);
    }
};

// src/Lozenge/LozengeTiler.h:35-79
class LozengeTiler : public TilerBase {
public:
    // qweight = true selects qlozengekernel.cl (volume weight q, int32 storage).
    explicit LozengeTiler(int device = 0, bool qweight = false)
        : TilerBase(RT_LOZENGE, device, qweight ? RT_KERNEL_QWEIGHT : RT_KERNEL_DEFAULT) {}
    explicit LozengeTiler(const rt_config& cfg) : TilerBase(cfg) {}
    // Periodic lozenge weights for the uniform kernel (rt_set_lozenge_weights):
    // P x P row-major tables w0, w1, w2, P = 1, 2 or 4; P = 0 returns to uniform.
    void SetWeights(int P, const std::vector<double>& w0, const std::vector<double>& w1,
                    const std::vector<double>& w2) {
        const size_t nn = (size_t)(P * P);
        if (P != 0 && (w0.size() != nn || w1.size() != nn || w2.size() != nn))
            throw Error(RT_E_INVAL, "weight tables must hold P x P values");
        detail::check(rt_set_lozenge_weights(h_, P, P ? w0.data() : nullptr, P ? w1.data() : nullptr,
                                             P ? w2.data() : nullptr),
                      h_);
    }
    static domain AlmostHexDomain(int N, int M) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) { return rt_lozenge_almost_hex(N, M, o, c, l); });
    }
    static tiling MaxTiling(const domain& d) {
        return detail::build(
            [&](int32_t* o, int64_t c, int64_t* l) { return rt_lozenge_max_tiling(detail::p(d), d.size(), o, c, l); });
    }
    static tiling MinTiling(const domain& d) {
        return detail::build(
            [&](int32_t* o, int64_t c, int64_t* l) { return rt_lozenge_min_tiling(detail::p(d), d.size(), o, c, l); });
    }
    static std::vector<int> DomainToVertices(const domain& d) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_lozenge_domain_to_vertices(detail::p(d), d.size(), o, c, l);
        });
    }
    static domain TilingToDomain(const tiling& t) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_lozenge_tiling_to_domain(detail::p(t), t.size(), o, c, l);
        });
    }
    static tiling HeightfuncToTiling(const heightfunc& hf, const domain& d) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_lozenge_height_to_tiling(detail::p(hf), hf.size(), detail::p(d), d.size(), o, c, l);
        });
    }
    static heightfunc TilingToHeightfunc(const tiling& t, const domain& d) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_lozenge_tiling_to_height(detail::p(t), t.size(), detail::p(d), d.size(), o, c, l);
        });
    }
    static void DomainToSVG(const domain& d, const std::string& f) {
        detail::check(rt_lozenge_domain_svg(detail::p(d), d.size(), f.c_str()), nullptr);
    }
    static void TilingToSVG(const tiling& t, const std::string& f) {
        detail::check(rt_lozenge_tiling_svg(detail::p(t), t.size(), f.c_str()), nullptr);
    }
    static void DimerToSVG(const tiling& t, const std::string& f) {
        detail::check(rt_lozenge_dimer_svg(detail::p(t), t.size(), nullptr, 0, f.c_str()), nullptr);
    }
    static void DimerToSVG(const tiling& t, const domain& d, const std::string& f) {
        detail::check(rt_lozenge_dimer_svg(detail::p(t), t.size(), detail::p(d), d.size(), f.c_str()), nullptr);
    }
    static void PrintDomain(const domain& d, const std::string& f) {
        detail::check(rt_lozenge_print_domain(detail::p(d), d.size(), f.c_str()), nullptr);
    }
};

// src/RectTriangle/RectTriangleTiler.h:30-73
class RectTriangleTiler : public TilerBase {
public:
    explicit RectTriangleTiler(int device = 0) : TilerBase(RT_RECTTRI, device, RT_KERNEL_DEFAULT) {}
    explicit RectTriangleTiler(const rt_config& cfg) : TilerBase(cfg) {}
    static tiling maxHex(int N) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) { return rt_recttri_max_hex(N, o, c, l); });
    }
    static tiling minHex(int N) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) { return rt_recttri_min_hex(N, o, c, l); });
    }
    static tiling LozengeToRectTriangle(const tiling& tL, const domain& dL) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_recttri_from_lozenge(detail::p(tL), tL.size(), detail::p(dL), dL.size(), o, c, l);
        });
    }
    static void TilingToSVG(const tiling& t, const std::string& f) {
        detail::check(rt_recttri_tiling_svg(detail::p(t), t.size(), f.c_str()), nullptr);
    }
};

// src/TriangleDimer/TriangleDimerTiler.h:72-202
class TriangleDimerTiler : public TilerBase {
public:
    explicit TriangleDimerTiler(int device = 0) : TilerBase(RT_TRIDIMER, device, RT_KERNEL_DEFAULT) {}
    explicit TriangleDimerTiler(const rt_config& cfg) : TilerBase(cfg) {}
    static tiling IceCreamCone(int N, int M) {
        return detail::build(
            [&](int32_t* o, int64_t c, int64_t* l) { return rt_tridimer_ice_cream_cone(N, M, o, c, l); });
    }
    static tiling TestButterfly(int type) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) { return rt_tridimer_test_butterfly(type, o, c, l); });
    }
    static std::vector<int> TilingToTriangleFlips(const tiling& t) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_tridimer_triangle_flips(detail::p(t), t.size(), o, c, l);
        });
    }
    static std::vector<int> TilingToButterflyFlips(const tiling& t) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_tridimer_butterfly_flips(detail::p(t), t.size(), o, c, l);
        });
    }
    static std::vector<int> TilingToVertices(const tiling& t) {
        return detail::build(
            [&](int32_t* o, int64_t c, int64_t* l) { return rt_tridimer_vertices(detail::p(t), t.size(), o, c, l); });
    }
    static domain TilingToDomain(const tiling& t) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_tridimer_tiling_to_domain(detail::p(t), t.size(), o, c, l);
        });
    }
    static std::vector<int> DimerIndicator(const tiling& t, int c0) {
        return detail::build([&](int32_t* o, int64_t c, int64_t* l) {
            return rt_tridimer_dimer_indicator(detail::p(t), t.size(), c0, o, c, l);
        });
    }
    static void DomainToSVG(const domain& d, const std::string& f) {
        detail::check(rt_tridimer_domain_svg(detail::p(d), d.size(), f.c_str()), nullptr);
    }
    static void TilingToSVG(const tiling& t, const std::string& f) {
        detail::check(rt_tridimer_tiling_svg(detail::p(t), t.size(), f.c_str()), nullptr);
    }
    static void DimerToSVG(const tiling& t, const std::string& f) {
        detail::check(rt_tridimer_dimer_svg(detail::p(t), t.size(), nullptr, 0, f.c_str()), nullptr);
    }
    static void DimerToSVG(const tiling& t, const domain& d, const std::string& f) {
        detail::check(rt_tridimer_dimer_svg(detail::p(t), t.size(), detail::p(d), d.size(), f.c_str()), nullptr);
    }
};

// The six-vertex model with domain-wall boundary conditions (no reference
// class: the reference's README.md:3 names the model only).  States are
// height functions on the (n+1) x (n+1) faces, as heightfunc vectors.
class SixVertexTiler {
    rt_sixv* h_ = nullptr;
    void check(rt_status s) const {
        if (s != RT_OK) throw Error(s, rt_sixv_last_error(h_));
    }
    static int side1(const heightfunc& v) { return detail::side(v) - 1; }

public:
    explicit SixVertexTiler(int device = 0) {
        if (rt_sixv_create(device, &h_) != RT_OK) throw Error(RT_E_NODEVICE, "rt_sixv_create failed");
    }
    SixVertexTiler(const SixVertexTiler&) = delete;
    SixVertexTiler& operator=(const SixVertexTiler&) = delete;
    ~SixVertexTiler() {
        if (h_) rt_sixv_destroy(h_);
    }
    // Weights of the vertex types a1, a2, b1, b2, c1, c2.
    void SetWeights(const std::vector<double>& w) {
        if (w.size() != 6) throw Error(RT_E_INVAL, "six weights expected");
        check(rt_sixv_set_weights(h_, w.data()));
    }
    static heightfunc MinHeights(int n) {
        heightfunc h((size_t)(n + 1) * (n + 1));
        detail::check(rt_sixv_dwbc_heights(n, reinterpret_cast<int32_t*>(h.data()), nullptr), nullptr);
        return h;
    }
    static heightfunc MaxHeights(int n) {
        heightfunc h((size_t)(n + 1) * (n + 1));
        detail::check(rt_sixv_dwbc_heights(n, nullptr, reinterpret_cast<int32_t*>(h.data())), nullptr);
        return h;
    }
    static std::vector<int> HeightsToASM(const heightfunc& h) {
        const int n = side1(h);
        std::vector<int> a((size_t)n * n);
        detail::check(rt_sixv_to_asm(detail::p(h), n, reinterpret_cast<int32_t*>(a.data())), nullptr);
        return a;
    }
    void Walk(heightfunc& h, long sweeps, long seed) {
        check(rt_sixv_walk(h_, reinterpret_cast<int32_t*>(h.data()), side1(h), sweeps, (uint64_t)seed, 0));
    }
    heightfunc CFTP(int n, long first_sweeps, long master_seed, rt_cftp_stats* stats = nullptr) {
        heightfunc h((size_t)(n + 1) * (n + 1));
        rt_cftp_stats local{};
        check(rt_sixv_cftp(h_, n, first_sweeps, master_seed, 30, reinterpret_cast<int32_t*>(h.data()),
                           stats ? stats : &local));
        return h;
    }
};

}  // namespace rt
