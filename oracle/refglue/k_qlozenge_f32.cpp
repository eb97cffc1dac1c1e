// Registers the reference's src/Lozenge/qlozengekernel.cl a second time,
// compiled with single-precision arithmetic.  TEST INFRASTRUCTURE ONLY (oracle).
//
// The kernel compares `q >= rd` with `#define q 0.99` (a double literal) and
// a float draw (qlozengekernel.cl:3,19-28).  Compiled as C++ (k_qlozenge.cpp)
// the comparison runs in double, as on an OpenCL device with fp64.  On an
// fp32-only device the literals are single precision, and the two differ at
// exactly one draw.  This translation unit reproduces the fp32-only device:
// the kernel's `float` variables become `f32`, whose arithmetic and
// comparisons with a double operand first round that operand to float, so
// `q >= rd` compares float(0.99) with the draw and `rd /= .5`, `(rd-.5)*.5`
// run in single precision.  The kernel source itself is included unchanged.
#include "clc_shim.h"
namespace ref_k_qlozenge_f32 {
// The generator header comes first, so that its own floats stay float (its
// include guard then skips the kernel file's #include of it).
#include "src/TinyMT/tinymt32.clh"

struct f32 {
    float v;
    f32(float x) : v(x) {}
    f32& operator/=(double d) {
        v = v / static_cast<float>(d);
        return *this;
    }
};
inline f32 operator-(f32 a, double b) { return f32(a.v - static_cast<float>(b)); }
inline f32 operator*(f32 a, double b) { return f32(a.v * static_cast<float>(b)); }
inline bool operator<(f32 a, double b) { return a.v < static_cast<float>(b); }
inline bool operator>=(double a, f32 b) { return static_cast<float>(a) >= b.v; }

#define float f32
#include "src/Lozenge/qlozengekernel.cl"
#undef float
}  // namespace ref_k_qlozenge_f32
#undef q
#include "cl_registry.h"
static const bool registered = clshim::register_program(
    "qlozenge_f32", {{"InitTinyMT", clshim::make_launcher(&ref_k_qlozenge_f32::InitTinyMT)},
                     {"RotateTiles", clshim::make_launcher(&ref_k_qlozenge_f32::RotateTiles)},
                     {"UpdateTiles", clshim::make_launcher(&ref_k_qlozenge_f32::UpdateTiles)}});
