// Registers the reference's src/TriangleDimer/triangledimerkernel.cl with the
// fake OpenCL runtime.  TEST INFRASTRUCTURE ONLY (oracle).
#include "clc_shim.h"
namespace ref_k_tridimer {
#include "src/TriangleDimer/triangledimerkernel.cl"
}
#include "cl_registry.h"
static const bool registered = clshim::register_program(
    "tridimer", {
                 {"RotateLozenges", clshim::make_launcher(&ref_k_tridimer::RotateLozenges)},
                 {"UpdateLozengesFlipped", clshim::make_launcher(&ref_k_tridimer::UpdateLozengesFlipped)},
                 {"UpdateLozenges0", clshim::make_launcher(&ref_k_tridimer::UpdateLozenges0)},
                 {"UpdateLozenges1", clshim::make_launcher(&ref_k_tridimer::UpdateLozenges1)},
                 {"UpdateLozenges2", clshim::make_launcher(&ref_k_tridimer::UpdateLozenges2)},
                 {"UpdateLozenges", clshim::make_launcher(&ref_k_tridimer::UpdateLozenges)},
                 {"UpdateTriangleUFromLozenges", clshim::make_launcher(&ref_k_tridimer::UpdateTriangleUFromLozenges)},
                 {"UpdateButterflysHFromLozenge", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysHFromLozenge)},
                 {"UpdateButterflysLFromLozenge", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysLFromLozenge)},
                 {"UpdateButterflysRFromLozenge", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysRFromLozenge)},
                 {"RotateTriangles", clshim::make_launcher(&ref_k_tridimer::RotateTriangles)},
                 {"UpdateTrianglesFlipped0", clshim::make_launcher(&ref_k_tridimer::UpdateTrianglesFlipped0)},
                 {"UpdateTrianglesFlipped1", clshim::make_launcher(&ref_k_tridimer::UpdateTrianglesFlipped1)},
                 {"UpdateTriangles", clshim::make_launcher(&ref_k_tridimer::UpdateTriangles)},
                 {"UpdateLozengeHFromTriangles", clshim::make_launcher(&ref_k_tridimer::UpdateLozengeHFromTriangles)},
                 {"UpdateLozengeLFromTriangles", clshim::make_launcher(&ref_k_tridimer::UpdateLozengeLFromTriangles)},
                 {"UpdateLozengeRFromTriangles", clshim::make_launcher(&ref_k_tridimer::UpdateLozengeRFromTriangles)},
                 {"RotateButterflys", clshim::make_launcher(&ref_k_tridimer::RotateButterflys)},
                 {"UpdateButterflysFlippedH1", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedH1)},
                 {"UpdateButterflysFlippedH21", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedH21)},
                 {"UpdateButterflysFlippedH22", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedH22)},
                 {"UpdateButterflysFlippedH23", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedH23)},
                 {"UpdateButterflysFlippedL1", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedL1)},
                 {"UpdateButterflysFlippedL21", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedL21)},
                 {"UpdateButterflysFlippedL22", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedL22)},
                 {"UpdateButterflysFlippedL23", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedL23)},
                 {"UpdateButterflysFlippedR1", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedR1)},
                 {"UpdateButterflysFlippedR21", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedR21)},
                 {"UpdateButterflysFlippedR22", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedR22)},
                 {"UpdateButterflysFlippedR23", clshim::make_launcher(&ref_k_tridimer::UpdateButterflysFlippedR23)},
                 {"UpdateLozengeFromButterflysH", clshim::make_launcher(&ref_k_tridimer::UpdateLozengeFromButterflysH)},
                 {"UpdateLozengeFromButterflysL", clshim::make_launcher(&ref_k_tridimer::UpdateLozengeFromButterflysL)},
                 {"UpdateLozengeFromButterflysR", clshim::make_launcher(&ref_k_tridimer::UpdateLozengeFromButterflysR)},
                 {"InitTinyMT", clshim::make_launcher(&ref_k_tridimer::InitTinyMT)}});
