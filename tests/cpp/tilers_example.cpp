// A reference-style caller of the C++ layer (include/randomtilings/Tilers.hpp):
// the flow of the reference's MinimalLozengeEx / AztecDiamond examples with
// the OpenCL set-up replaced by a device ordinal.  Used by the tests:
//   tilers_example builders <out.txt>     host builders only (no GPU)
//   tilers_example walk <out.txt>         + Walk on cuda:0
#include <cstdio>
#include <cstring>
#include <fstream>

#include "randomtilings/Tilers.hpp"

static void save(std::ofstream& f, const char* name, const std::vector<int>& v) {
    f << name << " " << v.size();
    for (int x : v) f << " " << x;
    f << "\n";
}

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const bool walk = std::strcmp(argv[1], "walk") == 0;
    std::ofstream f(argv[2]);
    try {
        rt::domain d = rt::LozengeTiler::AlmostHexDomain(10, 2);
        rt::tiling t = rt::LozengeTiler::MaxTiling(d);
        save(f, "lozenge_max", t);
        save(f, "lozenge_hmax", rt::LozengeTiler::TilingToHeightfunc(t, d));
        rt::tiling cone = rt::TriangleDimerTiler::IceCreamCone(10, 3);
        save(f, "cone", cone);
        if (argc > 3) rt::LozengeTiler::TilingToSVG(t, argv[3]);
        save(f, "sixv_max", rt::SixVertexTiler::MaxHeights(6));
        save(f, "sixv_asm_max", rt::SixVertexTiler::HeightsToASM(rt::SixVertexTiler::MaxHeights(6)));
        rt::domain a = rt::DominoTiler::AztecDiamond(12);
        rt::tiling m = rt::DominoTiler::MinTiling(a);
        save(f, "aztec_min", m);
        if (walk) {
            rt::tiling t2 = t;
            rt::LozengeTiler L(0);
            L.Walk(t, 1000, 42);
            save(f, "lozenge_walk", t);
            rt::LozengeTiler LW(0);
            LW.SetWeights(2, {1.0, 0.4, 1.6, 0.8}, {0.5, 1.2, 2.0, 1.0}, {1.5, 0.7, 0.9, 1.1});
            LW.Walk(t2, 1000, 42);
            save(f, "lozenge_weighted", t2);
            rt::DominoTiler D(0, /*cftp=*/true);
            std::vector<long> steps{256, 128}, seeds{2718281, 345903};
            rt::tiling m2 = m;
            D.Walk(m, steps, seeds);
            save(f, "aztec_epochs", m);
            rt::DominoTiler W(0, /*cftp=*/true);
            W.SetWeights(2, {1.0, 0.3, 0.5, 2.0}, {0.7, 1.5, 1.0, 0.2});
            W.Walk(m2, steps, seeds);
            save(f, "aztec_weighted", m2);
            rt::SixVertexTiler S(0);
            rt::heightfunc sh = rt::SixVertexTiler::MinHeights(20);
            S.Walk(sh, 300, 5);
            save(f, "sixv_walk", sh);
            save(f, "sixv_cftp", S.CFTP(8, 8, 3));
            rt::TriangleDimerTiler T(0);
            T.Walk(cone, 800, 9);
            save(f, "cone_walk", cone);
        }
    } catch (const rt::Error& e) {
        std::fprintf(stderr, "rt::Error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
    return 0;
}
