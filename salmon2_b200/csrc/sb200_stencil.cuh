// sb200_stencil.cuh -- argument block of the tiled hpsi kernel.
#pragma once
#include <cuda_runtime.h>

namespace sb200 {

struct TiledArgs {
  int nx, ny, nz, periodic, nspin, nspin_no, nlma, nent, phase_per_k, zchunk;
  long npts;
  double lapt[12], nab[12];  // coef_lap, coef_nab (k+A applied in the kernel)
  const double* kcoef;
  const double* vloc;
  const float* vloc32;
  const int *pmap, *ent_lma;
  const double2* ent_zk;
  const double2* proj;
  // (point, atom) pair form of the scatter (use_pairs = 1: pmap holds pair ranges)
  int use_pairs, npair;
  const int* pair_lma;
  const double* pair_uv;
  const double2* pair_ph;
  double2 zc;
};


}  // namespace sb200

struct sb200_ctx;
namespace sb200 {
// coefficient / table block of one context for the tiled kernel (z chunk = nz)
TiledArgs make_tiled_args(const sb200_ctx* c, double2 zc);
}  // namespace sb200
