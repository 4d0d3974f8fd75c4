// sb200_internal.cuh -- shared declarations of the B200 RT-TDDFT library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/salmon_b200.h"

namespace sb200 {

constexpr int ND = 4;            // stencil half-width (Nd of the reference)
constexpr int KC = 20;           // doubles per k-point coefficient record: kAc(3), k_lap0, k_nabt(12), B kAc(3), pad
constexpr int OBS_NQ = 7;        // per-orbital local observables (see k_observables)
constexpr int OBS_THREADS = 256;
constexpr int OBS_PTS_PER_THREAD = 8;

// Per-k coefficient record written by k_prep_k (hamiltonian.f90:146-155):
//   [0..2] kAc, [3] k_lap0, [4..15] k_nabt(4,3) column-major.

struct GridInfo {
  bool set = false;
  int nx = 0, ny = 0, nz = 0;
  long npts = 0;
  int periodic = 0;
  int is[3], ie[3], is_array[3], ie_array[3], lg_num[3];
  double hgs[3], hvol = 0, coef_lap0 = 0, coef_lap[12], coef_nab[12];
  // non-orthogonal lattice (sb200_set_lattice): rmatrix_B (3,3) column-major, coef_F(6)
  int nonorth = 0;
  double rB[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double coefF[6] = {1, 1, 1, 0, 0, 0};
  long vol_array() const {
    return (long)(ie_array[0] - is_array[0] + 1) * (ie_array[1] - is_array[1] + 1) *
           (ie_array[2] - is_array[2] + 1);
  }
};

struct OrbInfo {
  bool set = false;
  int nspin = 0, no = 0, nk = 0, norb = 0;
  std::vector<double> vec_k;   // (3,nk)
  std::vector<double> weight;  // per orbital rocc*wtk, orbital order
  std::vector<double> rocc;    // (no,nk,nspin) as given
  std::vector<double> wtk;     // (nk)
};

// Kleinman-Bylander tables, re-indexed for the device.
struct PPInfo {
  int natom = 0, nps = 0, nlma = 0, totpts = 0, nprojmax = 0;
  int nvi = 0, nent = 0;
  // per atom
  int* d_atom_start = nullptr;  // first flat sphere point of the atom
  int* d_mps = nullptr;
  int* d_lma_start = nullptr;   // first (0-based) ilma of the atom
  int* d_lma_atom = nullptr;    // atom (0-based) of each ilma
  int* d_nproj = nullptr;       // projectors of the atom
  // per flat sphere point
  int* d_pt_lin = nullptr;      // linear resident-layout point index
  double* d_pt_r = nullptr;     // rxyz, 3 per point
  // per projector
  double* d_uv = nullptr;       // uv(j, ilma) at [ilma*nps + j]
  double* d_rinv = nullptr;     // rinv_uvu
  // scatter inverse map: point -> entries (ilma, flat point, uv), ilma ascending
  int* d_map = nullptr;         // [npts] -> vi or -1
  int* d_vi_start = nullptr;    // [nvi+1]
  int* d_ent_lma = nullptr;
  int* d_ent_pt = nullptr;
  double* d_ent_uv = nullptr;
  // projector phases exp(i kAc.r): [nk_phase][totpts]
  double2* d_phase = nullptr;
  int nk_phase = 0;
  // per grid point: (first entry << 8) | entry count, or -1 outside every sphere
  int* d_pmap = nullptr;
  // zekr_uV of every scatter entry for every k: [nk_phase][nent] (k_prep)
  double2* d_ent_zk = nullptr;
  // (point, atom) pairs of the scatter for the tiled / tensor-copy kernels (atoms
  // with at most 4 projectors): per point (first pair << 8) | pair count,
  // per pair lma0 | (nproj << 24), uV of its projectors, flat sphere point,
  // and exp(i (k+A).r) per k (k_prep)
  int npair = 0;
  int* d_pmap2 = nullptr;
  int* d_pair_lma = nullptr;
  double* d_pair_uv = nullptr;  // [npair][4]
  int* d_pair_fp = nullptr;
  double2* d_pair_ph = nullptr; // [nk_phase][npair]
  int* d_pair_pt = nullptr;     // [npair] grid point of the pair
  int* d_apj = nullptr;         // [totpts] pair of each flat sphere point
  // the register-blocked fused step's tables in its shared-memory layout (16^3 grids)
  int blk_tpad = 0;
  double* d_blk_uv = nullptr;   // [4][blk_tpad]
  double* d_blk_r = nullptr;    // [3][blk_tpad]
  int* d_blk_sap = nullptr;     // [blk_tpad]
};

struct RTBuffers {
  int cap_nt = -1;
  double* d_Ac_ext = nullptr;   // (3, 0:nt+1)
  double* d_Ac_ind = nullptr;
  double* d_Ac_tot = nullptr;
  double* d_curr = nullptr;     // (3, nt)
  double* d_rbox = nullptr;     // (4, nt)
  int* d_step = nullptr;        // current itt
  double2* d_zc = nullptr;      // n_hamil coefficients
  // continuation (sb200_rt_set_start, sb200_read_restart): the next loop runs
  // global steps start_mit + 1 .. start_mit + nt, its history entries 0 and 1
  // seeded with Ac_tot / Ac_ind at steps start_mit and start_mit + 1
  int start_mit = 0;
  int loop_mit0 = 0;  // start step of the loop being issued (global itt = local + loop_mit0)
  bool seed_on = false;
  double seed_tot[6] = {0, 0, 0, 0, 0, 0}, seed_ind[6] = {0, 0, 0, 0, 0, 0};
  // the last loop: global step reached and its local step count (-1: none yet)
  int last_mit = 0, last_nt = -1;
};

// ground-state (real orbital) work state, sb200_gs.cu
constexpr int CG_NC = 12;  // per-orbital CG coefficients
enum { CG_XKHXK = 0, CG_GKGK, CG_UK, CG_ZS, CG_SUM, CG_CX, CG_CP, CG_XKXK };
struct GSState {
  long n = 0;         // npts * norb of the buffers below
  int norb = 0, nblk = 0;
  bool have_work = false;
  double* d_proj = nullptr;   // [norb][nlma] real projections
  double* d_part = nullptr;   // [norb][nblk][3] dot partials
  double* d_dots = nullptr;   // [norb][3]
  double* d_coef = nullptr;   // [norb][CG_NC]
  double* d_work = nullptr;   // 7 orbital blocks for the CG
  double* d_gram = nullptr;   // Gram partials
  size_t gram_cap = 0;
  double* d_mat = nullptr;    // small matrices (Gram results, eigenvectors)
  size_t mat_cap = 0;
};

}  // namespace sb200

struct sb200_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  int precision = SB200_PREC_FP64;
  sb200::GridInfo g;
  sb200::OrbInfo orb;
  sb200::PPInfo pp;
  sb200::RTBuffers rt;
  sb200::GSState gs;
  double vec_Ac[3] = {0, 0, 0};
  // device tables
  double* d_vloc = nullptr;     // [nspin][npts]
  float* d_vloc32 = nullptr;    // FP32 copy for the mixed form
  double* d_vec_k = nullptr;    // [nk][3]
  double* d_weight = nullptr;   // [norb]
  double* d_kcoef = nullptr;    // [nk][KC] for the hpsi coefficients in use
  double* d_kcoef_cur = nullptr;// [nk][KC] for calc_current's A
  // scratch
  double2* d_proj = nullptr;    // [norb][nlma] projections of the current input
  double* d_jw = nullptr;       // [norb][natom][3] nonlocal current pieces
  double* d_obs = nullptr;      // [norb][obs_blocks][OBS_NQ] partial sums
  double* d_obs1 = nullptr;     // [norb][OBS_NQ + 3] per-orbital sums (observables, nonlocal current)
  double* d_result = nullptr;   // small result area (8 doubles)
  int* d_err = nullptr;         // device error flag: a bounded wait expired
  int obs_blocks = 0;
  double* d_rho_part = nullptr; // [chunk][nspin][npts] density partial sums (calc_density)
  size_t rho_part_cap = 0;
  void* d_stage = nullptr;      // relayout staging
  size_t stage_bytes = 0;
  bool vloc_set = false;
  int stencil_variant = 1;     // 0: per-point reference kernel, 1: tiled 2.5-D sweep
  int orbital_variant = 4;     // 16^3 periodic grids: 4 fused Taylor step with register blocking (when its
                               // tables fit, else form 2), 2 fused step with the KB tables staged in shared memory
                               // (when they fit), 3 fused without staging, 0 one launch per term, 1 persistent per term
  int project_variant = 1;     // KB projections: 1 tensor cores where a k-point fills a 16-orbital tile, else
                               // a CTA per (orbital, atom) below 1184 pairs, else a warp per pair; 2 tensor
                               // cores always, 0 one warp per (orbital, atom), 3 one CTA per (orbital, atom)
  int blk_depth = 2;           // z depth of the register block of the blocked fused step (2: 512 threads, 4: 256)
  int blk_split = 1;           // blocked fused step: KB projections by two warps per atom, overlapped with the
                               // stencil (1), or one warp per atom between the terms (0)
  int blk_prefetch = 1;        // blocked fused step: each CTA prefetches the orbital one wave ahead into L2
  int tma_variant = 1;         // tiled hpsi fed by tensor copies where it applies (0: register-prefetch sweep)
  // optional per-kernel-class device timing (sb200_set_timing)
  bool timing = false;
  std::vector<cudaEvent_t> ev;  // pairs (start, stop)
  std::vector<int> ev_kind;
  int ev_used = 0;
  double kt_ms[SB200_KIND_COUNT] = {0};
  long kt_count[SB200_KIND_COUNT] = {0};
  // learned preconditioner (sb200_learned.cu)
  bool learned_set = false;
  void* learned = nullptr;
  // per-step potential update (sb200_scf.cu)
  void* scf = nullptr;
  // isolated Hartree potential by CG (sb200_poisson_cg.cu)
  void* pcg = nullptr;
  // non-orthogonal H psi: first-pass H psi and the x / y first derivatives [3][norb][npts]
  double2* d_nonorth = nullptr;
  size_t nonorth_cap = 0;
  // single-scale Maxwell-TDDFT (sb200_set_micro_ac): Ac_micro [npts][3] and div Ac [npts]
  int microac = 0;
  int micro_sym = 0;  // sb200_set_symmetrized_stencil
  // isolated grid driven by a pulse in the length gauge (sb200_set_length_gauge):
  // during a loop (lg_active) V_local = V_base + E_ext(itt).r before each step
  int length_gauge = 0, lg_active = 0;
  double* d_vloc_base = nullptr;  // [nspin][npts]
  size_t vloc_base_cap = 0;
  double* d_eext = nullptr;       // (3, 0:nt+1)
  size_t eext_cap = 0;
  // gram_schmidt_interval >= 1 (sb200_set_gram_schmidt_interval): the loop's
  // Gram-Schmidt of psi(t+dt) every gs_interval steps, its scratch and the
  // stream that captures the body of its conditional node
  int gs_interval = -1;
  double2* d_gs_scratch = nullptr;  // part [no][nb], then coeff [no]
  size_t gs_scratch_cap = 0;
  cudaStream_t gs_side = nullptr;
  // yn_predictor_corrector = 'y' (sb200_set_predictor_corrector): the step's
  // input orbitals and V_local kept across the predictor, and the loop's
  // initial (field-free) V_local for a fixed potential
  int pred_corr = 0;
  double2* d_pc_psi = nullptr;  // [norb][npts]
  size_t pc_psi_cap = 0;
  double* d_pc_v = nullptr;     // [2][nspin][npts]: V_tmp, V0
  size_t pc_v_cap = 0;
  // propagator = 'aetrs' (sb200_set_propagator): the two stored potentials
  int aetrs = 0;
  double* d_vloc_old = nullptr;  // [2][nspin][npts]
  size_t vloc_old_cap = 0;
  // absorbing boundary along z (sb200_set_absorbing_boundary): w(z) per plane
  int cap_on = 0;
  double* d_cap = nullptr;  // [nz]
  double* d_acm = nullptr;
  double* d_divac = nullptr;
  // microscopic current (sb200_calc_microscopic_current): chunk sums and the result
  double* d_mcur = nullptr;
  size_t mcur_cap = 0;
};

namespace sb200 {

// error reporting
int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* where);
#define SB_CUDA(call)                                                  \
  do {                                                                 \
    cudaError_t _e = (call);                                           \
    if (_e != cudaSuccess) return ::sb200::cuda_error(_e, #call);      \
  } while (0)
#define SB_LAUNCH_CHECK(what)                                          \
  do {                                                                 \
    cudaError_t _e = cudaGetLastError();                               \
    if (_e != cudaSuccess) return ::sb200::cuda_error(_e, what);       \
  } while (0)

template <typename T>
int dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return SB200_OK;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return set_error(SB200_ERR_OOM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  return SB200_OK;
}
template <typename T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

// ---- kernel launchers (sb200_kernels.cu) ----
struct HpsiLaunch {
  const void* in;       // double2 (FP64 modes) or float2 (modes 6..8)
  void* hout;           // double2 (modes 0..2) or float2 (modes 5..7); unused otherwise
  double2* out;         // FP64 Taylor accumulator psi_out
  float2* d32 = nullptr;// FP32 correction accumulator of the mixed form
  double2 zc;
  int mode;             // 0: h; 1: h, out = in + zc h; 2: h, out += zc h; 3: out += zc h;
                        // 4: out = in + zc h (no h store); 5..8: mixed form, see sb200_stencil.cu
};
int launch_prep_k(sb200_ctx* c, const double* d_A, int a_mode, int itt_from_device,
                  double* d_kcoef, bool phases);
int launch_project(sb200_ctx* c, const void* in, double2* proj, bool in32 = false);
// KB projections on the FP64 tensor cores; SB200_ERR_UNSUPPORTED (no error
// recorded) when the form does not apply (sb200_project_mma.cu)
int launch_project_dmma(sb200_ctx* c, const void* in, double2* proj, bool in32);
// symmetric eigen-decomposition of the upper triangle of row-major M (n x n)
// on the GPU: w ascending, V[i n + k] = component k of eigenvector i; work
// 2 n^2 doubles; *info = 1 when the QL iterations did not converge (sb200_eigh.cu)
int launch_eigh(sb200_ctx* c, const double* M, int n, double* work, double* V, double* w, int* info);
int launch_hpsi(sb200_ctx* c, const HpsiLaunch& L);
int nonorth_prepare(sb200_ctx* c);  // scratch of the non-orthogonal hpsi, before a graph capture
int launch_hpsi_tiled(sb200_ctx* c, const HpsiLaunch& L);  // sb200_stencil.cu
// tensor-copy-fed tiled kernel; SB200_ERR_UNSUPPORTED when it does not apply (sb200_tma_stencil.cu)
int launch_hpsi_tma(sb200_ctx* c, const HpsiLaunch& L);
bool orbital_kernel_applies(const sb200_ctx* c);             // sb200_orbital.cu
int launch_term_orbital(sb200_ctx* c, const HpsiLaunch& L, bool with_obs);
int launch_hpsi_kinetic(sb200_ctx* c, const double2* in, double2* tt);       // sb200_kernels.cu
int launch_energy_parts(sb200_ctx* c, const double2* psi, const double2* h, const double2* tt, double* part,
                        int nblk);
bool step_orbital_applies(const sb200_ctx* c, int n_hamil);                  // sb200_orbital.cu
int launch_step_orbital(sb200_ctx* c, const double2* in, double2* out, const double2* zc, int n_hamil,
                        bool with_obs);
int launch_observables(sb200_ctx* c, const double2* psi);
struct KickArgs {
  double e, ep[3], h[3], c0[3];  // e_impulse, direction, spacing, coordinate offset per axis
};
int launch_impulse_kick(sb200_ctx* c, double2* psi, double e_impulse, const double epdir[3]);
int launch_project_moments(sb200_ctx* c, const double2* psi);
int launch_finalize(sb200_ctx* c, int itt_host, int nt, int trans_longi, double dt, int spin_filter,
                    bool fused_obs = false);
// kind >= 0: each launch bracketed for sb200_kernel_times (SB200_KIND_*)
int launch_density(sb200_ctx* c, const double2* psi, double* rho, int kind = -1);
// length gauge: V_local = V_base + E_ext(itt).r (itt from the device counter),
// and the field-free V_local back from V_base after the loop
int launch_vbox(sb200_ctx* c, int kind = -1);
int launch_vloc_restore(sb200_ctx* c);
// AETRS: the extrapolated V_local between the half steps
int launch_aetrs_vloc(sb200_ctx* c);
int density_prepare(sb200_ctx* c);
// microscopic current [npts][3] into curr (device); part: micro_current_part_len(c) doubles
size_t micro_current_part_len(const sb200_ctx* c);
int launch_micro_current(sb200_ctx* c, const double2* psi, double* curr, double* part);
int launch_dip(sb200_ctx* c, const double* rho, double* d_out4);
int launch_relayout(sb200_ctx* c, const void* src, void* dst, int norb_chunk, bool to_ref);
// time-loop histories of capacity nt (sb200_api.cu)
int rt_alloc(sb200_ctx* c, int nt);
// per-kernel-class event timing on c->stream when c->timing is set (sb200_api.cu)
int kernel_timing_mark(sb200_ctx* c, int kind, bool start);
int kernel_timing_flush(sb200_ctx* c);
// low-pass preconditioner of the ground-state CG (sb200_gs.cu)
int gs_precond(sb200_ctx* c, const double* g, double* pre, double alpha);
// learned preconditioner: pre = net(g, V_local) for every orbital (sb200_learned.cu)
int learned_precond_apply(sb200_ctx* c, const double* g, const double* x, double* pre);
// Y -= X (X^T Y) hvol: components of n orbitals Y along m orthonormal X removed (sb200_gs.cu)
int gs_project_out(sb200_ctx* c, const double* X, int m, double* Y, int n);
void learned_free(sb200_ctx* c);
void scf_free(sb200_ctx* c);
void pcg_free(sb200_ctx* c);
// isolated Hartree potential by CG with the multipole boundary (sb200_poisson_cg.cu):
// rho, vh host or device (vh: start value in, solution out); rion [natom][3]
// (layout 2); npole_xyz: cells of layout 3 (NULL or zeros: about 8 A each)
int hartree_isolated_cg(sb200_ctx* c, const double* rho, double* vh, int layout, int lmax, const double* rion,
                        int natom, const int npole_xyz[3], double threshold, int maxiter, int* iterations);
void pcg_default_cells(const sb200_ctx* c, int out[3]);
// the same solve in pieces for the self-consistent loop: configure once, then
// issue per step on device arrays (inside a stream capture the iterations
// become a conditional WHILE node); the Vh extrapolation of isolated steps
int pcg_configure(sb200_ctx* c, int layout, int lmax, const double* rion, int natom, const int npole_xyz[3],
                  double threshold, int maxiter);
int pcg_issue(sb200_ctx* c, const double* d_rho, double* d_vh, int* iterations);
int pcg_vh_stock(sb200_ctx* c, const int* d_step, int offset, double* d_vh, double* d_s1, double* d_s2, bool before);
// self-consistent time loop (sb200_scf.cu): buffers sized before a capture, and
// the per-step potential update issued after each Taylor step (no-ops unless
// sb200_set_self_consistent enabled it)
int scf_rt_prepare(sb200_ctx* c);
int scf_rt_issue(sb200_ctx* c, const double2* psi);
// gram_schmidt_col_complex8's launches with caller-given scratch (sb200_gs.cu)
size_t gs_complex_part_len(const sb200_ctx* c);
int gs_complex_issue(sb200_ctx* c, double2* z, double2* part, double2* coeff);
// predictor_corrector (time_evolution_step.f90:374-428): V_local = (V_tmp + V_new) / 2
// with V_new the potential of the predicted orbitals psi (self-consistent) or v0
int scf_pc_potential(sb200_ctx* c, const double2* psi, const double* vtmp, const double* v0);
// initialization_rt.f90:268-283 with yn_restart = 'y' (isolated, CG): Vh from the
// stored potentials, the Hartree solve of psi's density, stock update, V_local
int scf_restart_potential(sb200_ctx* c, const double2* psi);
bool scf_cg_on(const sb200_ctx* c);
// the stored potentials of the CG loop (device), or false when there are none
bool scf_vh_stock(sb200_ctx* c, double** vh, double** s1, double** s2);
// sum of a device density over the k-point shards (no-op without a communicator)
int scf_density_allreduce(sb200_ctx* c, double* d_rho);
// k-point shard communicator (sb200_set_density_comm): set?, and an in-place
// sum of n device doubles over the shards on the context's stream
bool shard_comm_set(const sb200_ctx* c);
int shard_sum(sb200_ctx* c, double* d, size_t n);

}  // namespace sb200
