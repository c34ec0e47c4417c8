// rotlev.cuh -- the second variational step (ROTLEV3B) on the device.
#pragma once

#include <string>
#include <vector>

#include "pipeline.cuh"

namespace dvr3d {

struct RotInfo {
    int nbass = 0, nblk = 0, neval = 0;
    std::vector<int> mvib;       // vibrational functions used per k block
    double offdiag_flops = 0.0;  // algorithmic flops of the Coriolis blocks (two GEMMs each)
};

// ROTLEV3B for one parity: reads its deck (namelist PRT, nvib/neval/kmin/ibass/neval2/npnt card,
// title, optional EZERO) and the first step's wavefunction file; returns the lowest levels (Eh)
// and the printed level table. With a kvec_path (ZTRAN) the eigenvectors are transformed back to
// the first step's basis and written there as dstore does. Throws HostError / CudaFail.
// KMIN = 2 (both sets from a KMIN = 2 file) needs levels_f: the e levels go to levels, the f
// levels of the second pass to levels_f, their vectors (ZTRAN) to kvec_path and kvec2_path.
void rotlev3b_solve(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, std::vector<double> &levels,
                    std::string &table, RotInfo &info, const char *kvec_path = nullptr,
                    std::vector<double> *levels_f = nullptr, const char *kvec2_path = nullptr);

}  // namespace dvr3d
