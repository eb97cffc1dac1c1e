// Registers the reference's src/Domino/dominokernel.cl with the fake OpenCL
// runtime.  TEST INFRASTRUCTURE ONLY (oracle).
#include "clc_shim.h"
namespace ref_k_domino {
#include "src/Domino/dominokernel.cl"
}
#include "cl_registry.h"
static const bool registered = clshim::register_program(
    "domino", {{"InitTinyMT", clshim::make_launcher(&ref_k_domino::InitTinyMT)},
               {"RotateTiles", clshim::make_launcher(&ref_k_domino::RotateTiles)},
               {"UpdateTiles", clshim::make_launcher(&ref_k_domino::UpdateTiles)}});
