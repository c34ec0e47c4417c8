// dipole.cuh -- transition moments between two sets of vib-rot states (the reference's DIPOLE3).
#pragma once

#include <string>

#include "../../include/dvr3d_b200.h"
#include "pipeline.cuh"

namespace dvr3d {

// DIPOLE3 on two wavefunction files (see dvr3d_b200_dipole3). Fills res (capacities from the
// caller) and the printed text; throws HostError / CudaFail.
void dipole3_run(dvr3d_ctx *ctx, const char *deck_text, const char *ket_path, const char *bra_path,
                 dvr3d_dipd_fn dipd, dvr3d_dipsa_fn dipsa, void *user, const char *tra_path,
                 dvr3d_dipole_result &res, std::string &text);

}  // namespace dvr3d
