// Registers the reference's src/Lozenge/qlozengekernel.cl with the fake OpenCL
// runtime.  TEST INFRASTRUCTURE ONLY (oracle).  The file defines the macro q;
// it is removed again after the include.
#include "clc_shim.h"
namespace ref_k_qlozenge {
#include "src/Lozenge/qlozengekernel.cl"
}
#undef q
#include "cl_registry.h"
static const bool registered = clshim::register_program(
    "qlozenge", {{"InitTinyMT", clshim::make_launcher(&ref_k_qlozenge::InitTinyMT)},
                 {"RotateTiles", clshim::make_launcher(&ref_k_qlozenge::RotateTiles)},
                 {"UpdateTiles", clshim::make_launcher(&ref_k_qlozenge::UpdateTiles)}});
