// sb200_orbital.cuh -- argument block of the orbital-resident Taylor-term kernel.
#pragma once
#include <cuda_runtime.h>

#include <vector>

struct sb200_ctx;

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

// extra arguments of the register-blocked fused step (sb200_orbital_blk.cu)
struct BlkArgs {
  double mhl[12];      // -coef_lap / 2
  int npair;           // (point, atom) pairs
  const int* pmap2;    // [npts] (first pair << 8) | count, or -1
  int tpad;            // flat sphere points rounded up to a multiple of 4
  const double* uv4;   // [4][tpad] uV of each sphere point's atom projectors
  const double* r3;    // [3][tpad] sphere-point coordinates
  const int* sap;      // [tpad] (pair index << 12) | shared-memory grid index
  int* err;            // device error flag (a bounded wait expired)
  int kbcache;         // 1: each atom's uV and phases kept in TMEM by its warp
  int prefetch_ahead;  // CTA o prefetches the orbital of CTA o + prefetch_ahead into L2 (0: none)
};

// The register-blocked fused step; SB200_ERR_UNSUPPORTED (no error recorded)
// when its shared-memory tables do not fit or the KB tables have no pair form.
// Host-side tables of the blocked fused step (called by sb200_set_pp).
int blk_build_tables(sb200_ctx* c, const std::vector<int>& pt_lin, const std::vector<int>& apj,
                     const std::vector<double>& uv_lma, const std::vector<double>& pt_r,
                     const std::vector<int>& atom_start, const std::vector<int>& mps,
                     const std::vector<int>& lma_start, const std::vector<int>& nproj);
int launch_step_blk(sb200_ctx* c, const double2* in, double2* out, const OrbArgs& a, const StepZC& z, int n_hamil,
                    bool with_obs);

}  // namespace sb200
