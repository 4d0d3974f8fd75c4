// sb200_orbital.cuh -- argument block of the orbital-resident Taylor-term kernel.
#pragma once
#include <cuda_runtime.h>

namespace sb200 {

constexpr int ORB_MAX_NLMA = 1024;  // projections held in shared memory

struct OrbArgs {
  long npts;
  int nspin, nspin_no, nlma, natom, nps, totpts, nent;
  double lapt[12], nab[12], off[3];
  const double* kcoef;
  const double* vloc;
  const int *pmap, *ent_lma;
  const double2* ent_zk;
  const double2* phase;
  const int *atom_start, *mps, *lma_start, *nproj, *pt_lin;
  const int* lma_atom;
  const double *pt_r, *uv, *rinv;
  double2 zc;
  double* obs;  // [norb][OBS_NQ] or null
  double* jw;   // [norb][3] or null
};

// KB (point, atom) pair tables the fused step stages in shared memory
struct StageArgs {
  int npair;
  const double2* pair_ph;  // [nk][npair] exp(i (k+A).r)
  const double* pair_uv;   // [npair][4] uV of the atom's projectors
  const int* pair_lma;     // [npair] lma0 | nproj << 24
  const int* pair_pt;      // [npair] grid point
  const int* apj;          // [totpts] flat sphere point -> pair
  const int* pmap2;        // [npts] (first pair << 8) | count, or -1
};

constexpr int STEP_MAX_NTERM = 8;  // Taylor terms of the fused step kernel
struct StepZC {
  double2 v[STEP_MAX_NTERM];  // zc(1..n_hamil)
};

}  // namespace sb200
