// Registers the reference's src/RectTriangle/recttrianglekernel.cl with the
// fake OpenCL runtime.  TEST INFRASTRUCTURE ONLY (oracle).
#include "clc_shim.h"
namespace ref_k_recttri {
#include "src/RectTriangle/recttrianglekernel.cl"
}
#include "cl_registry.h"
static const bool registered = clshim::register_program(
    "recttri", {{"InitTinyMT", clshim::make_launcher(&ref_k_recttri::InitTinyMT)},
                {"flipTiles", clshim::make_launcher(&ref_k_recttri::flipTiles)},
                {"updateTiles1", clshim::make_launcher(&ref_k_recttri::updateTiles1)},
                {"updateTiles2", clshim::make_launcher(&ref_k_recttri::updateTiles2)}});
