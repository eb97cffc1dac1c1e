// Registers the reference's src/Lozenge/lozengekernel.cl with the fake OpenCL
// runtime.  TEST INFRASTRUCTURE ONLY (oracle).
#include "clc_shim.h"
namespace ref_k_lozenge {
#include "src/Lozenge/lozengekernel.cl"
}
#include "cl_registry.h"
static const bool registered = clshim::register_program(
    "lozenge", {{"InitTinyMT", clshim::make_launcher(&ref_k_lozenge::InitTinyMT)},
                {"RotateTiles", clshim::make_launcher(&ref_k_lozenge::RotateTiles)},
                {"UpdateTiles", clshim::make_launcher(&ref_k_lozenge::UpdateTiles)}});
