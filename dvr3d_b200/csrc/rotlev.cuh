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

// ROTLEV3 (z along r1 or r2; Jacobi and unsymmetrised Radau files): reads its deck (namelist
// PRT, NVIB/NEVAL/KMIN/IBASS/NEVAL2 card, title, optional EZERO) and the first step's file.
// levels: the e set (KMIN = 1, 2) or the f set (KMIN = 0); levels_f: the f set of KMIN = 2;
// text: the printed level lists. With kvec_path / kvec2_path (ZTRAN) the vectors of the first /
// second set are written as dstore does; J = 1 f (KMIN = 0) writes its set to kvec2_path, as the
// reference does. Throws HostError / CudaFail.
void rotlev3_solve(dvr3d_ctx *ctx, const char *deck_text, const char *wave_path, std::vector<double> &levels,
                   std::vector<double> &levels_f, std::string &text, RotInfo &info, const char *kvec_path,
                   const char *kvec2_path);

}  // namespace dvr3d
