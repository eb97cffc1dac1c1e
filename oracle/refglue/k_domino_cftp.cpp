// Registers the reference's src/Domino/dominokernelCFTP.cl with the fake
// OpenCL runtime.  TEST INFRASTRUCTURE ONLY (oracle).
#include "clc_shim.h"
namespace ref_k_domino_cftp {
#include "src/Domino/dominokernelCFTP.cl"
}
#include "cl_registry.h"
static const bool registered = clshim::register_program(
    "domino_cftp", {{"InitTinyMT", clshim::make_launcher(&ref_k_domino_cftp::InitTinyMT)},
                    {"RotateTiles", clshim::make_launcher(&ref_k_domino_cftp::RotateTiles)},
                    {"UpdateTiles", clshim::make_launcher(&ref_k_domino_cftp::UpdateTiles)}});
