// sb200_api.cu -- C ABI of the B200 RT-TDDFT library: context, set-up, the
// hpsi / taylor / observable entry points and the CUDA-graph time loop.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sb200_internal.cuh"
#include "sb200_orbital.cuh"

using namespace sb200;

namespace sb200 {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_error(cudaError_t e, const char* where) {
  return set_error(SB200_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

}  // namespace sb200

namespace {

#define CHECK_CTX(c)                                                        \
  do {                                                                      \
    if ((c) == nullptr) return set_error(SB200_ERR_INVALID_ARG, "null ctx"); \
  } while (0)
#define TRY(x)                      \
  do {                              \
    int _r = (x);                   \
    if (_r != SB200_OK) return _r;  \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

bool is_device_ptr(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

int ensure_stage(sb200_ctx* c, size_t bytes) {
  if (c->stage_bytes >= bytes) return SB200_OK;
  if (c->d_stage) cudaFree(c->d_stage);
  c->d_stage = nullptr;
  c->stage_bytes = 0;
  cudaError_t e = cudaMalloc(&c->d_stage, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(SB200_ERR_OOM, "staging buffer allocation failed");
  }
  c->stage_bytes = bytes;
  return SB200_OK;
}

// (re)allocate work buffers that depend on grid x orbitals x projectors
int ensure_work(sb200_ctx* c) {
  if (!c->g.set || !c->orb.set) return SB200_OK;
  dfree(c->d_proj);
  dfree(c->d_jw);
  dfree(c->d_obs);
  const long nblk = (c->g.npts + (long)OBS_THREADS * OBS_PTS_PER_THREAD - 1) / ((long)OBS_THREADS * OBS_PTS_PER_THREAD);
  c->obs_blocks = (int)nblk;
  TRY(dalloc(&c->d_obs, (size_t)c->orb.norb * nblk * OBS_NQ + 4096));
  dfree(c->d_obs1);
  TRY(dalloc(&c->d_obs1, (size_t)c->orb.norb * (OBS_NQ + 3)));
  if (c->pp.nlma > 0) {
    TRY(dalloc(&c->d_proj, (size_t)c->orb.norb * c->pp.nlma));
    TRY(dalloc(&c->d_jw, (size_t)c->orb.norb * c->pp.natom * 3));
  }
  return SB200_OK;
}

int require_ready(sb200_ctx* c, bool need_vloc = true) {
  if (!c->g.set) return set_error(SB200_ERR_STATE, "sb200_set_grid has not been called");
  if (!c->orb.set) return set_error(SB200_ERR_STATE, "sb200_set_orbitals has not been called");
  if (need_vloc && !c->vloc_set) return set_error(SB200_ERR_STATE, "sb200_set_vlocal has not been called");
  return SB200_OK;
}

// after a stream synchronisation: did a kernel give up a bounded wait?
int check_device_flag(sb200_ctx* c) {
  int flag = 0;
  SB_CUDA(cudaMemcpy(&flag, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag != 0) {
    SB_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
    SB_CUDA(cudaDeviceSynchronize());
    return set_error(SB200_ERR_TIMEOUT, "a bounded device wait expired (a bulk copy or a grid barrier did not complete)");
  }
  return SB200_OK;
}

void free_pp(PPInfo& p) {
  dfree(p.d_atom_start);
  dfree(p.d_mps);
  dfree(p.d_lma_start);
  dfree(p.d_lma_atom);
  dfree(p.d_nproj);
  dfree(p.d_pt_lin);
  dfree(p.d_pt_r);
  dfree(p.d_uv);
  dfree(p.d_rinv);
  dfree(p.d_map);
  dfree(p.d_vi_start);
  dfree(p.d_pair_pt);
  dfree(p.d_apj);
  dfree(p.d_ent_lma);
  dfree(p.d_ent_pt);
  dfree(p.d_ent_uv);
  dfree(p.d_phase);
  dfree(p.d_pmap);
  dfree(p.d_ent_zk);
  dfree(p.d_pmap2);
  dfree(p.d_pair_lma);
  dfree(p.d_pair_uv);
  dfree(p.d_pair_fp);
  dfree(p.d_pair_ph);
  dfree(p.d_blk_uv);
  dfree(p.d_blk_r);
  dfree(p.d_blk_sap);
  p = PPInfo();
}

template <typename T>
int upload(T** d, const std::vector<T>& h) {
  TRY(dalloc(d, h.size()));
  if (!h.empty()) SB_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  // a copy from pageable memory may still be landing when cudaMemcpy returns;
  // the context's stream does not wait for the legacy stream
  SB_CUDA(cudaDeviceSynchronize());
  return SB200_OK;
}

// refresh k+A coefficients (and projector phases) for system%vec_Ac
int refresh_k(sb200_ctx* c) {
  if (!c->g.set || !c->orb.set) return SB200_OK;
  SB_CUDA(cudaMemcpyAsync(c->d_result + 8, c->vec_Ac, 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return launch_prep_k(c, c->d_result + 8, 0, 0, c->d_kcoef, true);
}

int alloc_rt(sb200_ctx* c, int nt) {
  RTBuffers& r = c->rt;
  if (r.cap_nt >= nt) return SB200_OK;
  dfree(r.d_Ac_ext);
  dfree(r.d_Ac_ind);
  dfree(r.d_Ac_tot);
  dfree(r.d_curr);
  dfree(r.d_rbox);
  r.cap_nt = -1;
  TRY(dalloc(&r.d_Ac_ext, 3 * (size_t)(nt + 2)));
  TRY(dalloc(&r.d_Ac_ind, 3 * (size_t)(nt + 2)));
  TRY(dalloc(&r.d_Ac_tot, 3 * (size_t)(nt + 2)));
  TRY(dalloc(&r.d_curr, 3 * (size_t)(nt + 1)));
  TRY(dalloc(&r.d_rbox, 4 * (size_t)(nt + 1)));
  r.cap_nt = nt;
  return SB200_OK;
}

// ---- optional per-kernel-class device timing ----
int timing_mark(sb200_ctx* c, int kind, bool start) {
  if (!c->timing) return SB200_OK;
  if (start) {
    if ((size_t)(2 * c->ev_used + 2) > c->ev.size()) {
      for (int i = 0; i < 2; ++i) {
        cudaEvent_t e;
        SB_CUDA(cudaEventCreate(&e));
        c->ev.push_back(e);
      }
      c->ev_kind.push_back(kind);
    }
    c->ev_kind[c->ev_used] = kind;
    SB_CUDA(cudaEventRecord(c->ev[2 * c->ev_used], c->stream));
  } else {
    SB_CUDA(cudaEventRecord(c->ev[2 * c->ev_used + 1], c->stream));
    c->ev_used += 1;
  }
  return SB200_OK;
}

int timing_flush(sb200_ctx* c) {
  if (!c->timing || c->ev_used == 0) return SB200_OK;
  SB_CUDA(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < c->ev_used; ++i) {
    float ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&ms, c->ev[2 * i], c->ev[2 * i + 1]));
    c->kt_ms[c->ev_kind[i]] += ms;
    c->kt_count[c->ev_kind[i]] += 1;
  }
  c->ev_used = 0;
  return SB200_OK;
}

#define TIMED(c, kind, call)                 \
  do {                                       \
    TRY(timing_mark((c), (kind), true));     \
    TRY(call);                               \
    TRY(timing_mark((c), (kind), false));    \
  } while (0)

// One Taylor step tspsi_in -> tspsi_out (taylor.f90:43-119) with the
// projections of each term's input computed first.
int issue_taylor(sb200_ctx* c, double2* tin, double2* tout, double2* work, const double2* zc, int n_hamil,
                 bool last_with_obs = false) {
  if (step_orbital_applies(c, n_hamil)) {  // all terms in one launch, observables fused
    TIMED(c, SB200_KIND_HPSI, launch_step_orbital(c, tin, tout, zc, n_hamil, last_with_obs));
    return SB200_OK;
  }
  const bool orbital = orbital_kernel_applies(c);
  for (int nn = 1; nn <= n_hamil; ++nn) {
    if (orbital) {  // one CTA per orbital: projections and observables in-kernel
      const bool odd = (nn % 2) == 1;
      HpsiLaunch L;
      L.in = odd ? tin : work;
      L.hout = odd ? work : tin;
      L.out = tout;
      L.zc = zc[nn - 1];
      const bool last = nn == n_hamil;
      if (nn == 1) L.mode = last ? 4 : 1;
      else L.mode = last ? 3 : 2;
      TIMED(c, SB200_KIND_HPSI, launch_term_orbital(c, L, last && last_with_obs));
      continue;
    }
    if (c->precision == SB200_PREC_MIXED && n_hamil > 1) {
      // mixed form: term 1 in FP64 (h1 stored as complex64 in the first half
      // of work), terms n >= 2 in FP32 ping-ponging between the two halves of
      // work, their sum in an FP32 correction kept in tspsi_in (free after
      // term 1) and added to psi_out in FP64 by the last term.
      const long n = c->g.npts * c->orb.norb;
      float2* w1 = (float2*)work;
      float2* w2 = (float2*)work + n;
      float2* corr = (float2*)tin;
      const void* src = (nn == 1) ? (const void*)tin : (const void*)((nn % 2) == 0 ? w1 : w2);
      void* dst = (nn % 2) == 1 ? (void*)w1 : (void*)w2;
      TIMED(c, SB200_KIND_PROJECT, launch_project(c, src, c->d_proj, nn > 1));
      HpsiLaunch L;
      L.in = src;
      L.hout = dst;
      L.out = tout;
      L.d32 = corr;
      L.zc = zc[nn - 1];
      const bool last = nn == n_hamil;
      L.mode = (nn == 1) ? 5 : (last ? 8 : (nn == 2 ? 6 : 7));
      TIMED(c, SB200_KIND_HPSI, launch_hpsi(c, L));
      continue;
    }
    const bool odd = (nn % 2) == 1;
    double2* src = odd ? tin : work;
    double2* dst = odd ? work : tin;
    TIMED(c, SB200_KIND_PROJECT, launch_project(c, src, c->d_proj));
    HpsiLaunch L;
    L.in = src;
    L.hout = dst;
    L.out = tout;
    L.zc = zc[nn - 1];
    const bool last = nn == n_hamil;
    if (nn == 1) L.mode = last ? 4 : 1;
    else L.mode = last ? 3 : 2;
    TIMED(c, SB200_KIND_HPSI, launch_hpsi(c, L));
  }
  return SB200_OK;
}

// the condition of the Gram-Schmidt node: mod(itt, interval) == 0 with the
// global step itt (time_evolution_step.f90:149-152)
__global__ void k_gs_condition(cudaGraphConditionalHandle h, const int* step, int offset, int interval) {
  const int itt = *step + offset;
  cudaGraphSetConditional(h, (itt % interval == 0) ? 1u : 0u);
}

// gram_schmidt every gs_interval steps, on psi (the step's result, before its
// density and current): a conditional IF node inside a capture, a host check of
// the step counter otherwise
int issue_rt_gram_schmidt(sb200_ctx* c, double2* psi) {
  double2* part = c->d_gs_scratch;
  double2* coeff = c->d_gs_scratch + gs_complex_part_len(c);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  SB_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &g, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive) {
    int step = 0;
    SB_CUDA(cudaMemcpyAsync(&step, c->rt.d_step, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
    if ((step + c->rt.loop_mit0) % c->gs_interval != 0) return SB200_OK;
    return gs_complex_issue(c, psi, part, coeff);
  }
  cudaGraphConditionalHandle h;
  SB_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0u, cudaGraphCondAssignDefault));
  k_gs_condition<<<1, 1, 0, c->stream>>>(h, c->rt.d_step, c->rt.loop_mit0, c->gs_interval);
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  SB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  SB_CUDA(cudaStreamUpdateCaptureDependencies(c->stream, &node, 1, cudaStreamSetCaptureDependencies));
  SB_CUDA(cudaStreamBeginCaptureToGraph(c->gs_side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  cudaStream_t keep = c->stream;
  c->stream = c->gs_side;  // the launch sequence issues on c->stream
  const int r = gs_complex_issue(c, psi, part, coeff);
  c->stream = keep;
  cudaGraph_t captured = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(c->gs_side, &captured);
  if (r != SB200_OK) return r;
  if (ee != cudaSuccess) return cuda_error(ee, "cudaStreamEndCapture (Gram-Schmidt body)");
  return SB200_OK;
}

// one time_evolution_step on the device (itt from the device counter); with
// AETRS the step's result is back in `in` (out is the half step's scratch)
int issue_rt_step(sb200_ctx* c, double2* in, double2* out, double2* work, const double2* zc, int n_hamil,
                  int trans_longi, double dt) {
  if (c->aetrs) {
    // propagator = 'aetrs' (time_evolution_step.f90:117-147, 430-470; zc of the
    // half step -i dt/2): a half step with A(itt) and V(t), then V extrapolated
    // (3 V - 3 V_old1 + V_old2) and A(itt+1) predicted, the second half step
    if (c->g.periodic) TIMED(c, SB200_KIND_PREP, launch_prep_k(c, c->rt.d_Ac_tot, 2, -1, c->d_kcoef, true));
    if (c->lg_active) TRY(launch_vbox(c, c->timing ? SB200_KIND_POTENTIAL : -1));
    TRY(issue_taylor(c, in, out, work, zc, n_hamil));
    TIMED(c, SB200_KIND_POTENTIAL, launch_aetrs_vloc(c));
    if (c->g.periodic) TIMED(c, SB200_KIND_PREP, launch_prep_k(c, c->rt.d_Ac_ext, 3, -1, c->d_kcoef, true));
    if (orbital_kernel_applies(c) && c->gs_interval < 1) {
      TRY(issue_taylor(c, out, in, work, zc, n_hamil, true));
      TIMED(c, SB200_KIND_FINAL, launch_finalize(c, -1, 0, trans_longi, dt, -1, true));
      return scf_rt_issue(c, in);
    }
    TRY(issue_taylor(c, out, in, work, zc, n_hamil));
    if (c->gs_interval >= 1) TRY(issue_rt_gram_schmidt(c, in));
    TIMED(c, SB200_KIND_OBS, launch_observables(c, in));
    if (c->g.periodic) TIMED(c, SB200_KIND_MOMENTS, launch_project_moments(c, in));
    TIMED(c, SB200_KIND_FINAL, launch_finalize(c, -1, 0, trans_longi, dt, -1));
    return scf_rt_issue(c, in);
  }
  if (c->g.periodic) TIMED(c, SB200_KIND_PREP, launch_prep_k(c, c->rt.d_Ac_tot, 1, -1, c->d_kcoef, true));
  if (c->lg_active) TRY(launch_vbox(c, c->timing ? SB200_KIND_POTENTIAL : -1));
  if (c->pred_corr) {  // predictor_corrector, time_evolution_step.f90:139-143, 374-428
    const size_t nv = (size_t)c->g.npts * c->orb.nspin, nb = (size_t)c->g.npts * c->orb.norb;
    SB_CUDA(cudaMemcpyAsync(c->d_pc_v, c->d_vloc, nv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    SB_CUDA(cudaMemcpyAsync(c->d_pc_psi, in, nb * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
    TRY(issue_taylor(c, in, out, work, zc, n_hamil));
    TRY(scf_pc_potential(c, out, c->d_pc_v, c->d_pc_v + nv));
    SB_CUDA(cudaMemcpyAsync(in, c->d_pc_psi, nb * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
  }
  if (orbital_kernel_applies(c) && c->gs_interval < 1) {  // observables fused into the last Taylor term
    TRY(issue_taylor(c, in, out, work, zc, n_hamil, true));
    TIMED(c, SB200_KIND_FINAL, launch_finalize(c, -1, 0, trans_longi, dt, -1, true));
    return scf_rt_issue(c, out);
  }
  TRY(issue_taylor(c, in, out, work, zc, n_hamil));
  if (c->gs_interval >= 1) TRY(issue_rt_gram_schmidt(c, out));
  TIMED(c, SB200_KIND_OBS, launch_observables(c, out));
  if (c->g.periodic) TIMED(c, SB200_KIND_MOMENTS, launch_project_moments(c, out));
  TIMED(c, SB200_KIND_FINAL, launch_finalize(c, -1, 0, trans_longi, dt, -1));
  // self-consistent path: V_local of the next step from rho(t+dt)
  return scf_rt_issue(c, out);
}

}  // namespace

namespace sb200 {
int rt_alloc(sb200_ctx* c, int nt) { return alloc_rt(c, nt); }
int kernel_timing_mark(sb200_ctx* c, int kind, bool start) { return timing_mark(c, kind, start); }
int kernel_timing_flush(sb200_ctx* c) { return timing_flush(c); }
}  // namespace sb200

extern "C" {

const char* sb200_last_error(void) { return g_last_error.c_str(); }
const char* sb200_version(void) { return "salmon_b200 0.1.0 (sm_100a)"; }

int sb200_ctx_create(int device, sb200_ctx** out) {
  if (!out) return set_error(SB200_ERR_INVALID_ARG, "null out pointer");
  *out = nullptr;
  int n = 0;
  SB_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return set_error(SB200_ERR_INVALID_ARG, "device index out of range");
  DeviceGuard dg(device);
  sb200_ctx* c = new sb200_ctx();
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return cuda_error(e, "cudaStreamCreate");
  }
  c->stream = c->own_stream;
  if (const char* v = getenv("SB200_STENCIL")) c->stencil_variant = (v[0] == 'n') ? 0 : 1;
  if (const char* v = getenv("SB200_ORBITAL"))
    c->orbital_variant = (v[0] == 'p') ? 1 : (v[0] == 't') ? 0 : (v[0] == 'u') ? 3 : (v[0] == 's') ? 2 : 4;
  if (const char* v = getenv("SB200_PROJECT")) c->project_variant = (v[0] == 'w') ? 0 : (v[0] == 'd') ? 2 : (v[0] == 's') ? 3 : 1;
  if (const char* v = getenv("SB200_BLK_DEPTH")) c->blk_depth = (v[0] == '4') ? 4 : 2;
  if (const char* v = getenv("SB200_BLK_SPLIT")) c->blk_split = (v[0] == '0') ? 0 : 1;
  if (const char* v = getenv("SB200_BLK_PREFETCH")) c->blk_prefetch = (v[0] == '0') ? 0 : 1;
  if (const char* v = getenv("SB200_TMA")) c->tma_variant = (v[0] == 'o' && v[1] == 'f') ? 0 : 1;
  int r = dalloc(&c->d_result, 24);  // results [0, 8), staged A [8, 11), shard sums [16, 23)
  if (r == SB200_OK) r = dalloc(&c->rt.d_step, 1);
  if (r == SB200_OK) r = dalloc(&c->d_err, 1);
  if (r == SB200_OK && cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) r = cuda_error(cudaGetLastError(), "cudaMemset");
  if (r != SB200_OK) {
    sb200_ctx_destroy(c);
    return r;
  }
  cudaMemset(c->d_result, 0, 16 * sizeof(double));
  cudaDeviceSynchronize();  // the legacy-stream fills land before the context's non-blocking stream runs
  *out = c;
  return SB200_OK;
}

int sb200_ctx_destroy(sb200_ctx* c) {
  if (!c) return SB200_OK;
  DeviceGuard dg(c->device);
  cudaStreamSynchronize(c->stream);
  free_pp(c->pp);
  dfree(c->d_vloc);
  dfree(c->d_vloc32);
  dfree(c->d_vec_k);
  dfree(c->d_weight);
  dfree(c->d_kcoef);
  dfree(c->d_kcoef_cur);
  dfree(c->d_proj);
  dfree(c->d_jw);
  dfree(c->d_obs);
  dfree(c->d_obs1);
  dfree(c->d_rho_part);
  dfree(c->d_result);
  dfree(c->rt.d_Ac_ext);
  dfree(c->rt.d_Ac_ind);
  dfree(c->rt.d_Ac_tot);
  dfree(c->rt.d_curr);
  dfree(c->rt.d_rbox);
  dfree(c->rt.d_step);
  dfree(c->d_err);
  dfree(c->rt.d_zc);
  if (c->d_stage) cudaFree(c->d_stage);
  dfree(c->gs.d_proj);
  dfree(c->gs.d_part);
  dfree(c->gs.d_dots);
  dfree(c->gs.d_coef);
  dfree(c->gs.d_work);
  dfree(c->gs.d_gram);
  dfree(c->gs.d_mat);
  learned_free(c);
  scf_free(c);
  pcg_free(c);
  dfree(c->d_nonorth);
  dfree(c->d_acm);
  dfree(c->d_divac);
  dfree(c->d_mcur);
  dfree(c->d_cap);
  dfree(c->d_vloc_base);
  dfree(c->d_eext);
  dfree(c->d_vloc_old);
  dfree(c->d_pc_psi);
  dfree(c->d_pc_v);
  dfree(c->d_gs_scratch);
  if (c->gs_side) cudaStreamDestroy(c->gs_side);
  for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return SB200_OK;
}

int sb200_set_timing(sb200_ctx* c, int enable) {
  CHECK_CTX(c);
  DeviceGuard dg(c->device);
  TRY(timing_flush(c));
  c->timing = enable != 0;
  return SB200_OK;
}

int sb200_kernel_times(sb200_ctx* c, double ms[SB200_KIND_COUNT], long count[SB200_KIND_COUNT], int reset) {
  CHECK_CTX(c);
  if (!ms || !count) return set_error(SB200_ERR_INVALID_ARG, "null output");
  DeviceGuard dg(c->device);
  TRY(timing_flush(c));
  for (int i = 0; i < SB200_KIND_COUNT; ++i) {
    ms[i] = c->kt_ms[i];
    count[i] = c->kt_count[i];
    if (reset) {
      c->kt_ms[i] = 0.0;
      c->kt_count[i] = 0;
    }
  }
  return SB200_OK;
}

int sb200_ctx_set_stream(sb200_ctx* c, void* stream) {
  CHECK_CTX(c);
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return SB200_OK;
}

int sb200_ctx_sync(sb200_ctx* c) {
  CHECK_CTX(c);
  DeviceGuard dg(c->device);
  SB_CUDA(cudaStreamSynchronize(c->stream));
  SB_CUDA(cudaGetLastError());
  return check_device_flag(c);
}

int sb200_set_grid(sb200_ctx* c, const int is[3], const int ie[3], const int is_array[3], const int ie_array[3],
                   const int* idx, const int* idy, const int* idz, const int lg_num[3], const double hgs[3],
                   double hvol, double coef_lap0, const double coef_lap[12], const double coef_nab[12]) {
  CHECK_CTX(c);
  if (!is || !ie || !is_array || !ie_array || !idx || !idy || !idz || !lg_num || !hgs || !coef_lap || !coef_nab)
    return set_error(SB200_ERR_INVALID_ARG, "sb200_set_grid: null argument");
  DeviceGuard dg(c->device);
  GridInfo g;
  const int* maps[3] = {idx, idy, idz};
  int periodic = -1;
  for (int d = 0; d < 3; ++d) {
    const int n = ie[d] - is[d] + 1;
    if (n < ND) return set_error(SB200_ERR_BAD_SHAPE, "grid extent smaller than the stencil half-width 4");
    if (is_array[d] > is[d] || ie_array[d] < ie[d])
      return set_error(SB200_ERR_BAD_SHAPE, "array bounds do not contain the interior");
    bool ident = true, modular = true;
    for (int j = is[d] - ND; j <= ie[d] + ND; ++j) {
      const int v = maps[d][j - (is[d] - ND)];
      if (v != j) ident = false;
      const int m = ((j - is[d]) % n + n) % n + is[d];
      if (v != m) modular = false;
    }
    const int p = modular ? 1 : (ident ? 0 : -1);
    if (p < 0)
      return set_error(SB200_ERR_UNSUPPORTED, "idx/idy/idz must be the identity (halo) or the periodic modular map");
    if (p == 0 && (is_array[d] > is[d] - ND || ie_array[d] < ie[d] + ND))
      return set_error(SB200_ERR_BAD_SHAPE, "identity neighbour map needs a 4-deep halo in the array bounds");
    if (periodic < 0) periodic = p;
    else if (periodic != p) return set_error(SB200_ERR_UNSUPPORTED, "mixed periodic / isolated axes");
    g.is[d] = is[d];
    g.ie[d] = ie[d];
    g.is_array[d] = is_array[d];
    g.ie_array[d] = ie_array[d];
    g.lg_num[d] = lg_num[d];
    g.hgs[d] = hgs[d];
  }
  g.periodic = periodic;
  g.nx = ie[0] - is[0] + 1;
  g.ny = ie[1] - is[1] + 1;
  g.nz = ie[2] - is[2] + 1;
  g.npts = (long)g.nx * g.ny * g.nz;
  g.hvol = hvol;
  g.coef_lap0 = coef_lap0;
  for (int i = 0; i < 12; ++i) {
    g.coef_lap[i] = coef_lap[i];
    g.coef_nab[i] = coef_nab[i];
  }
  g.set = true;
  const bool changed = !c->g.set || c->g.npts != g.npts || c->g.periodic != g.periodic;
  c->g = g;
  if (changed) {
    // tables that depend on the grid must be provided again
    free_pp(c->pp);
    dfree(c->d_vloc);
    dfree(c->d_vloc32);
    c->vloc_set = false;
  }
  TRY(ensure_work(c));
  TRY(refresh_k(c));
  return SB200_OK;
}

int sb200_set_orbitals(sb200_ctx* c, int nspin, int no, int nk, const double* vec_k, const double* rocc,
                       const double* wtk) {
  CHECK_CTX(c);
  if (nspin < 1 || nspin > 2 || no < 1 || nk < 1 || !vec_k || !rocc || !wtk)
    return set_error(SB200_ERR_INVALID_ARG, "sb200_set_orbitals: bad sizes or null pointer");
  DeviceGuard dg(c->device);
  OrbInfo& o = c->orb;
  const bool nk_changed = o.nk != nk;
  o.nspin = nspin;
  o.no = no;
  o.nk = nk;
  o.norb = nspin * no * nk;
  o.vec_k.assign(vec_k, vec_k + 3 * nk);
  o.rocc.assign(rocc, rocc + (size_t)no * nk * nspin);
  o.wtk.assign(wtk, wtk + nk);
  o.weight.assign(o.norb, 0.0);
  for (int ik = 0; ik < nk; ++ik)
    for (int io = 0; io < no; ++io)
      for (int is = 0; is < nspin; ++is)
        o.weight[is + nspin * (io + no * ik)] = rocc[io + (long)no * (ik + (long)nk * is)] * wtk[ik];
  o.set = true;
  dfree(c->d_vec_k);
  dfree(c->d_weight);
  dfree(c->d_kcoef);
  dfree(c->d_kcoef_cur);
  TRY(upload(&c->d_vec_k, o.vec_k));
  TRY(upload(&c->d_weight, o.weight));
  TRY(dalloc(&c->d_kcoef, (size_t)KC * nk));
  TRY(dalloc(&c->d_kcoef_cur, (size_t)KC * nk));
  if (nk_changed && c->pp.totpts > 0 && c->g.periodic) {
    dfree(c->pp.d_phase);
    dfree(c->pp.d_ent_zk);
    c->pp.nk_phase = nk;
    TRY(dalloc(&c->pp.d_phase, (size_t)nk * c->pp.totpts));
    TRY(dalloc(&c->pp.d_ent_zk, (size_t)nk * (c->pp.nent > 0 ? c->pp.nent : 1)));
  }
  TRY(ensure_work(c));
  TRY(refresh_k(c));
  return SB200_OK;
}

int sb200_set_vlocal(sb200_ctx* c, const double* V_local) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  if (!V_local) return set_error(SB200_ERR_INVALID_ARG, "null V_local");
  DeviceGuard dg(c->device);
  const size_t n = (size_t)c->g.npts * c->orb.nspin;
  if (!c->d_vloc) TRY(dalloc(&c->d_vloc, n));
  SB_CUDA(cudaMemcpy(c->d_vloc, V_local, n * sizeof(double), cudaMemcpyDefault));
  if (!c->d_vloc32) TRY(dalloc(&c->d_vloc32, n));
  std::vector<float> v32(n);
  std::vector<double> tmp(n);
  SB_CUDA(cudaMemcpy(tmp.data(), c->d_vloc, n * sizeof(double), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < n; ++i) v32[i] = (float)tmp[i];
  SB_CUDA(cudaMemcpy(c->d_vloc32, v32.data(), n * sizeof(float), cudaMemcpyHostToDevice));
  SB_CUDA(cudaDeviceSynchronize());  // landed before the context's (non-blocking) stream reads it
  c->vloc_set = true;
  return SB200_OK;
}

int sb200_set_pp(sb200_ctx* c, int natom, int nps, int nlma, const int* mps, const int* jxyz, const double* rxyz,
                 const double* uv, const int* ia_tbl, const double* rinv_uvu) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  DeviceGuard dg(c->device);
  free_pp(c->pp);
  if (natom <= 0 || nlma <= 0) {
    TRY(ensure_work(c));
    return SB200_OK;
  }
  if (nps < 0 || !mps || !jxyz || !rxyz || !uv || !ia_tbl || !rinv_uvu)
    return set_error(SB200_ERR_INVALID_ARG, "sb200_set_pp: null table");
  const GridInfo& g = c->g;
  // projectors of one atom must be contiguous in ilma (set_lma, prep_pp.f90:374-420)
  std::vector<int> lma_start(natom, 0), nproj(natom, 0), atom_start(natom, 0), hmps(mps, mps + natom);
  int prev = 0;
  for (int l = 0; l < nlma; ++l) {
    const int a = ia_tbl[l];
    if (a < 1 || a > natom) return set_error(SB200_ERR_INVALID_ARG, "ia_tbl entry out of range");
    if (a < prev) return set_error(SB200_ERR_UNSUPPORTED, "projectors of an atom must be contiguous in ilma");
    if (a != prev) {
      if (nproj[a - 1] != 0) return set_error(SB200_ERR_UNSUPPORTED, "projectors of an atom must be contiguous");
      lma_start[a - 1] = l;
    }
    nproj[a - 1] += 1;
    prev = a;
  }
  int tot = 0, npmax = 0;
  for (int a = 0; a < natom; ++a) {
    if (hmps[a] < 0 || hmps[a] > nps) return set_error(SB200_ERR_INVALID_ARG, "mps entry out of range");
    atom_start[a] = tot;
    tot += hmps[a];
    if (nproj[a] > npmax) npmax = nproj[a];
  }
  std::vector<int> pt_lin(tot);
  std::vector<double> pt_r(3 * (size_t)tot);
  for (int a = 0; a < natom; ++a)
    for (int j = 0; j < hmps[a]; ++j) {
      int ic[3];
      for (int d = 0; d < 3; ++d) {
        ic[d] = jxyz[d + 3L * (j + (long)nps * a)];
        if (ic[d] < g.is[d] || ic[d] > g.ie[d])  // host-side bounds check of every table index
          return set_error(SB200_ERR_BAD_SHAPE, "jxyz point outside the grid interior");
        pt_r[3L * (atom_start[a] + j) + d] = rxyz[d + 3L * (j + (long)nps * a)];
      }
      pt_lin[atom_start[a] + j] =
          (ic[0] - g.is[0]) + g.nx * ((ic[1] - g.is[1]) + (long)g.ny * (ic[2] - g.is[2]));
    }
  // inverse map: point -> (ilma, flat point, uv) entries in ilma order
  std::vector<std::vector<int>> ent_of_point;
  std::vector<int> map(g.npts, -1), vi_pt;
  std::vector<int> cnt;
  for (int l = 0; l < nlma; ++l) {
    const int a = ia_tbl[l] - 1;
    for (int j = 0; j < hmps[a]; ++j) {
      const int p = pt_lin[atom_start[a] + j];
      if (map[p] < 0) {
        map[p] = (int)vi_pt.size();
        vi_pt.push_back(p);
        cnt.push_back(0);
      }
      cnt[map[p]] += 1;
    }
  }
  const int nvi = (int)vi_pt.size();
  std::vector<int> vi_start(nvi + 1, 0);
  for (int v = 0; v < nvi; ++v) vi_start[v + 1] = vi_start[v] + cnt[v];
  const int nent = vi_start[nvi];
  std::vector<int> ent_lma(nent), ent_pt(nent), fill(vi_start.begin(), vi_start.end() - 1);
  std::vector<double> ent_uv(nent);
  for (int l = 0; l < nlma; ++l) {
    const int a = ia_tbl[l] - 1;
    for (int j = 0; j < hmps[a]; ++j) {
      const int fp = atom_start[a] + j;
      const int v = map[pt_lin[fp]];
      const int e = fill[v]++;
      ent_lma[e] = l;
      ent_pt[e] = fp;
      ent_uv[e] = uv[j + (long)nps * l];
    }
  }
  std::vector<double> huv((size_t)nlma * (nps > 0 ? nps : 1), 0.0);
  for (int l = 0; l < nlma; ++l)
    for (int j = 0; j < nps; ++j) huv[(size_t)l * nps + j] = uv[j + (long)nps * l];
  std::vector<double> hrinv(rinv_uvu, rinv_uvu + nlma);
  PPInfo& p = c->pp;
  p.natom = natom;
  p.nps = nps;
  p.nlma = nlma;
  p.totpts = tot;
  p.nprojmax = npmax;
  p.nvi = nvi;
  p.nent = nent;
  TRY(upload(&p.d_atom_start, atom_start));
  TRY(upload(&p.d_mps, hmps));
  TRY(upload(&p.d_lma_start, lma_start));
  {
    std::vector<int> lma_atom(nlma);
    for (int l = 0; l < nlma; ++l) lma_atom[l] = ia_tbl[l] - 1;
    TRY(upload(&p.d_lma_atom, lma_atom));
  }
  TRY(upload(&p.d_nproj, nproj));
  TRY(upload(&p.d_pt_lin, pt_lin));
  TRY(upload(&p.d_pt_r, pt_r));
  TRY(upload(&p.d_uv, huv));
  TRY(upload(&p.d_rinv, hrinv));
  TRY(upload(&p.d_map, map));
  TRY(upload(&p.d_vi_start, vi_start));
  TRY(upload(&p.d_ent_lma, ent_lma));
  TRY(upload(&p.d_ent_pt, ent_pt));
  TRY(upload(&p.d_ent_uv, ent_uv));
  p.nk_phase = g.periodic ? c->orb.nk : 1;
  TRY(dalloc(&p.d_phase, (size_t)p.nk_phase * (tot > 0 ? tot : 1)));
  // packed point map: (first entry << 8) | count
  std::vector<int> pmap(g.npts, -1);
  for (int v = 0; v < nvi; ++v) {
    const int cnt = vi_start[v + 1] - vi_start[v];
    if (cnt > 255 || vi_start[v] >= (1 << 23))
      return set_error(SB200_ERR_UNSUPPORTED, "more than 255 projector entries on one grid point");
    pmap[vi_pt[v]] = (vi_start[v] << 8) | cnt;
  }
  TRY(upload(&p.d_pmap, pmap));
  // (point, atom) pairs: the entries of a point grouped by atom (ilma
  // ascending).  A sphere that reaches the same grid point twice (through two
  // periodic images) has no pair form.
  bool pair_form = npmax <= 4;
  for (int v = 0; v < nvi && pair_form; ++v) {
    int prev_atom = -1, run = 0;
    for (int e = vi_start[v]; e < vi_start[v + 1]; ++e) {
      const int at = ia_tbl[ent_lma[e]] - 1;
      run = (at == prev_atom) ? run + 1 : 1;
      prev_atom = at;
      if (run > nproj[at]) pair_form = false;
    }
  }
  if (pair_form) {
    std::vector<int> pmap2(g.npts, -1), pair_lma, pair_fp;
    std::vector<double> pair_uv;
    std::vector<int> apj(tot > 0 ? tot : 1, -1);
    for (int v = 0; v < nvi; ++v) {
      const int first = (int)pair_lma.size();
      int prev_atom = -1;
      for (int e = vi_start[v]; e < vi_start[v + 1]; ++e) {
        const int at = ia_tbl[ent_lma[e]] - 1;
        if (at == prev_atom) continue;
        prev_atom = at;
        apj[ent_pt[e]] = (int)pair_lma.size();
        const int fp = ent_pt[e];
        const int j = fp - atom_start[at];
        pair_lma.push_back(lma_start[at] | (nproj[at] << 24));
        pair_fp.push_back(fp);
        for (int q = 0; q < 4; ++q)
          pair_uv.push_back(q < nproj[at] ? huv[(size_t)(lma_start[at] + q) * nps + j] : 0.0);
      }
      const int cnt = (int)pair_lma.size() - first;
      if (cnt > 255) return set_error(SB200_ERR_UNSUPPORTED, "more than 255 atoms on one grid point");
      pmap2[vi_pt[v]] = (first << 8) | cnt;
    }
    p.npair = (int)pair_lma.size();
    std::vector<int> pair_pt(pair_fp.size());
    for (size_t i = 0; i < pair_fp.size(); ++i) pair_pt[i] = pt_lin[pair_fp[i]];
    TRY(upload(&p.d_pair_pt, pair_pt));
    TRY(upload(&p.d_apj, apj));
    TRY(upload(&p.d_pmap2, pmap2));
    TRY(upload(&p.d_pair_lma, pair_lma));
    TRY(upload(&p.d_pair_uv, pair_uv));
    TRY(upload(&p.d_pair_fp, pair_fp));
    TRY(blk_build_tables(c, pt_lin, apj, huv, pt_r, atom_start, hmps, lma_start, nproj));
    TRY(dalloc(&p.d_pair_ph, (size_t)p.nk_phase * (p.npair > 0 ? p.npair : 1)));
    if (!g.periodic) {  // isolated: exp(i 0.r) = 1
      std::vector<double2> one(p.npair > 0 ? p.npair : 1, make_double2(1.0, 0.0));
      SB_CUDA(cudaMemcpy(p.d_pair_ph, one.data(), one.size() * sizeof(double2), cudaMemcpyHostToDevice));
      SB_CUDA(cudaDeviceSynchronize());
    }
  }
  TRY(dalloc(&p.d_ent_zk, (size_t)p.nk_phase * (nent > 0 ? nent : 1)));
  if (!g.periodic) {  // isolated: zekr_uV = uV (prep_pp.f90:618-619)
    std::vector<double2> one(tot > 0 ? tot : 1, make_double2(1.0, 0.0));
    TRY(upload(&p.d_phase, one));
    std::vector<double2> zk(nent > 0 ? nent : 1, make_double2(0.0, 0.0));
    for (int e = 0; e < nent; ++e) zk[e] = make_double2(ent_uv[e], 0.0);
    SB_CUDA(cudaMemcpy(p.d_ent_zk, zk.data(), zk.size() * sizeof(double2), cudaMemcpyHostToDevice));
    SB_CUDA(cudaDeviceSynchronize());
  }
  TRY(ensure_work(c));
  TRY(refresh_k(c));
  return SB200_OK;
}

int sb200_impulse_kick(sb200_ctx* c, void* psi, double e_impulse, const double epdir[3]) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  if (!psi || !epdir) return set_error(SB200_ERR_INVALID_ARG, "sb200_impulse_kick: null pointer");
  DeviceGuard dg(c->device);
  TRY(launch_impulse_kick(c, (double2*)psi, e_impulse, epdir));
  return SB200_OK;
}

int sb200_set_vec_Ac(sb200_ctx* c, const double vec_Ac[3]) {
  CHECK_CTX(c);
  if (!vec_Ac) return set_error(SB200_ERR_INVALID_ARG, "null vec_Ac");
  DeviceGuard dg(c->device);
  for (int d = 0; d < 3; ++d) c->vec_Ac[d] = vec_Ac[d];
  TRY(refresh_k(c));
  return SB200_OK;
}

int sb200_set_lattice(sb200_ctx* c, const double rmatrix_B[9], const double coef_F[6]) {
  CHECK_CTX(c);
  if (!c->g.set) return set_error(SB200_ERR_STATE, "sb200_set_grid has not been called");
  DeviceGuard dg(c->device);
  if (!rmatrix_B || !coef_F) {  // back to the orthogonal branch
    c->g.nonorth = 0;
    for (int i = 0; i < 9; ++i) c->g.rB[i] = (i % 4 == 0) ? 1.0 : 0.0;
    for (int i = 0; i < 6; ++i) c->g.coefF[i] = i < 3 ? 1.0 : 0.0;
  } else {
    if (!c->g.periodic) return set_error(SB200_ERR_UNSUPPORTED, "a non-orthogonal lattice needs a periodic grid");
    if (c->cap_on)
      return set_error(SB200_ERR_UNSUPPORTED, "the absorbing boundary is for orthogonal cells (inputoutput.f90:2789-2795)");
    for (int i = 0; i < 9; ++i) c->g.rB[i] = rmatrix_B[i];
    for (int i = 0; i < 6; ++i) c->g.coefF[i] = coef_F[i];
    c->g.nonorth = 1;
  }
  if (c->orb.set) {
    TRY(refresh_k(c));
    TRY(nonorth_prepare(c));  // the two-pass scratch at set-up, not inside a later capture
  }
  return SB200_OK;
}

int sb200_set_micro_ac(sb200_ctx* c, const double* Ac_micro, const double* div_Ac) {
  CHECK_CTX(c);
  if (!c->g.set) return set_error(SB200_ERR_STATE, "sb200_set_grid has not been called");
  DeviceGuard dg(c->device);
  if (!Ac_micro) {
    c->microac = 0;
    return SB200_OK;
  }
  if (c->g.nonorth)
    return set_error(SB200_ERR_UNSUPPORTED, "a microscopic vector potential needs an orthogonal lattice");
  const size_t n = (size_t)c->g.npts;
  if (!c->d_acm) TRY(dalloc(&c->d_acm, 3 * n));
  if (!c->d_divac) TRY(dalloc(&c->d_divac, n));
  SB_CUDA(cudaMemcpyAsync(c->d_acm, Ac_micro, 3 * n * sizeof(double), cudaMemcpyDefault, c->stream));
  if (div_Ac)
    SB_CUDA(cudaMemcpyAsync(c->d_divac, div_Ac, n * sizeof(double), cudaMemcpyDefault, c->stream));
  else
    SB_CUDA(cudaMemsetAsync(c->d_divac, 0, n * sizeof(double), c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  c->microac = 1;
  return SB200_OK;
}

int sb200_set_gram_schmidt_interval(sb200_ctx* c, int gram_schmidt_interval) {
  CHECK_CTX(c);
  c->gs_interval = gram_schmidt_interval;
  return SB200_OK;
}

int sb200_set_predictor_corrector(sb200_ctx* c, int yn) {
  CHECK_CTX(c);
  if (yn != 0 && yn != 1) return set_error(SB200_ERR_INVALID_ARG, "yn_predictor_corrector is 0 or 1");
  c->pred_corr = yn;
  return SB200_OK;
}

int sb200_set_propagator(sb200_ctx* c, int aetrs) {
  CHECK_CTX(c);
  if (aetrs != 0 && aetrs != 1) return set_error(SB200_ERR_INVALID_ARG, "propagator: 0 = middlepoint, 1 = aetrs");
  c->aetrs = aetrs;
  return SB200_OK;
}

int sb200_set_length_gauge(sb200_ctx* c, int on) {
  CHECK_CTX(c);
  if (!c->g.set) return set_error(SB200_ERR_STATE, "sb200_set_grid has not been called");
  if (on && c->g.periodic)
    return set_error(SB200_ERR_UNSUPPORTED, "the length gauge is for isolated grids (periodic ones take A(t))");
  c->length_gauge = on ? 1 : 0;
  return SB200_OK;
}

int sb200_set_absorbing_boundary(sb200_ctx* c, int yn_z, double w0, double dr, double al_z) {
  CHECK_CTX(c);
  if (!c->g.set) return set_error(SB200_ERR_STATE, "sb200_set_grid has not been called");
  if (!yn_z) {
    c->cap_on = 0;
    return SB200_OK;
  }
  if (c->g.nonorth)
    return set_error(SB200_ERR_UNSUPPORTED, "the absorbing boundary is for orthogonal cells (inputoutput.f90:2789-2795)");
  if (!(dr > 0.0) || !(al_z > 0.0)) return set_error(SB200_ERR_INVALID_ARG, "imagnary_potential_dr and al(3) must be > 0");
  DeviceGuard dg(c->device);
  // add_imaginary_potential_for_absorbing_boundary_z (hamiltonian.f90:760-807):
  // z = iz hgs(3); -i w0 (z1 - z) / dr below z1 = dr, -i w0 (z - z2) / dr above
  // z2 = al(3) - dr, nothing between; the table holds the w of each plane
  const int nz = c->g.nz;
  std::vector<double> w(nz, 0.0);
  const double z1 = dr, z2 = al_z - dr;
  for (int k = 0; k < nz; ++k) {
    const double z = (double)(c->g.is[2] + k) * c->g.hgs[2];
    if (z <= z1) w[k] = w0 * (z1 - z) / dr;
    else if (z >= z2) w[k] = w0 * (z - z2) / dr;
  }
  dfree(c->d_cap);
  TRY(upload(&c->d_cap, w));
  c->cap_on = 1;
  return SB200_OK;
}

int sb200_set_symmetrized_stencil(sb200_ctx* c, int yn) {
  CHECK_CTX(c);
  if (yn != 0 && yn != 1) return set_error(SB200_ERR_INVALID_ARG, "yn_symmetrized_stencil is 0 or 1");
  c->micro_sym = yn;
  return SB200_OK;
}

int sb200_calc_microscopic_current(sb200_ctx* c, const double* psi, double* curr) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  if (!psi || !curr) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  DeviceGuard dg(c->device);
  const size_t n3 = 3 * (size_t)c->g.npts;
  const size_t need = n3 + micro_current_part_len(c);
  if (c->mcur_cap < need) {
    dfree(c->d_mcur);
    c->mcur_cap = 0;
    TRY(dalloc(&c->d_mcur, need));
    c->mcur_cap = need;
  }
  double* out = is_device_ptr(curr) ? curr : c->d_mcur;
  TRY(launch_micro_current(c, (const double2*)psi, out, c->d_mcur + n3));
  TRY(shard_sum(c, out, n3));  // comm_summation over icomm_ko
  if (out != curr) SB_CUDA(cudaMemcpyAsync(curr, out, n3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

int sb200_set_precision(sb200_ctx* c, int mode) {
  CHECK_CTX(c);
  if (mode != SB200_PREC_FP64 && mode != SB200_PREC_MIXED)
    return set_error(SB200_ERR_INVALID_ARG, "unknown precision mode");
  c->precision = mode;
  return SB200_OK;
}

size_t sb200_orbital_block_bytes(const sb200_ctx* c) {
  if (!c || !c->g.set || !c->orb.set) return 0;
  return (size_t)c->g.npts * c->orb.norb * 2 * sizeof(double);
}

static int relayout_all(sb200_ctx* c, const double* src_ref, double* dst_dev, double* dst_ref, const double* src_dev,
                        bool to_ref) {
  const size_t blk = (size_t)c->g.vol_array() * 2 * sizeof(double);
  const int norb = c->orb.norb;
  int chunk = (int)((size_t)(256u << 20) / blk);
  if (chunk < 1) chunk = 1;
  if (chunk > norb) chunk = norb;
  TRY(ensure_stage(c, blk * chunk));
  for (int o0 = 0; o0 < norb; o0 += chunk) {
    const int n = (o0 + chunk <= norb) ? chunk : norb - o0;
    if (!to_ref) {
      SB_CUDA(cudaMemcpyAsync(c->d_stage, (const char*)src_ref + blk * o0, blk * n, cudaMemcpyDefault, c->stream));
      TRY(launch_relayout(c, c->d_stage, dst_dev + 2 * c->g.npts * o0, n, false));
    } else {
      SB_CUDA(cudaMemsetAsync(c->d_stage, 0, blk * n, c->stream));
      TRY(launch_relayout(c, src_dev + 2 * c->g.npts * o0, c->d_stage, n, true));
      SB_CUDA(cudaMemcpyAsync((char*)dst_ref + blk * o0, c->d_stage, blk * n, cudaMemcpyDefault, c->stream));
    }
    SB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return SB200_OK;
}

int sb200_orbitals_from_ref(sb200_ctx* c, const double* zwf_ref, double* psi_dev) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  if (!zwf_ref || !psi_dev) return set_error(SB200_ERR_INVALID_ARG, "null orbital pointer");
  DeviceGuard dg(c->device);
  return relayout_all(c, zwf_ref, psi_dev, nullptr, nullptr, false);
}

int sb200_orbitals_to_ref(sb200_ctx* c, const double* psi_dev, double* zwf_ref) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  if (!zwf_ref || !psi_dev) return set_error(SB200_ERR_INVALID_ARG, "null orbital pointer");
  DeviceGuard dg(c->device);
  return relayout_all(c, nullptr, nullptr, zwf_ref, psi_dev, true);
}

int sb200_hpsi(sb200_ctx* c, const double* tpsi, double* htpsi) {
  CHECK_CTX(c);
  TRY(require_ready(c));
  if (!tpsi || !htpsi || tpsi == htpsi) return set_error(SB200_ERR_INVALID_ARG, "tpsi/htpsi null or aliased");
  DeviceGuard dg(c->device);
  TIMED(c, SB200_KIND_PROJECT, launch_project(c, (const double2*)tpsi, c->d_proj));
  HpsiLaunch L;
  L.in = (const double2*)tpsi;
  L.hout = (double2*)htpsi;
  L.out = nullptr;
  L.zc = make_double2(0.0, 0.0);
  L.mode = 0;
  TIMED(c, SB200_KIND_HPSI, launch_hpsi(c, L));
  return SB200_OK;
}

int sb200_hpsi_tt(sb200_ctx* c, const double* tpsi, double* htpsi, double* ttpsi) {
  CHECK_CTX(c);
  TRY(require_ready(c));
  if (!tpsi || !htpsi || !ttpsi || tpsi == htpsi || tpsi == ttpsi || htpsi == ttpsi)
    return set_error(SB200_ERR_INVALID_ARG, "tpsi/htpsi/ttpsi null or aliased");
  TRY(sb200_hpsi(c, tpsi, htpsi));
  DeviceGuard dg(c->device);
  TIMED(c, SB200_KIND_HPSI, launch_hpsi_kinetic(c, (const double2*)tpsi, (double2*)ttpsi));
  return SB200_OK;
}

int sb200_calc_eigen_energy(sb200_ctx* c, const double* psi, double* htpsi, double* ttpsi, double* esp,
                            double* e_kin, double* e_nloc) {
  CHECK_CTX(c);
  if (!esp || !e_kin || !e_nloc) return set_error(SB200_ERR_INVALID_ARG, "null output pointer");
  TRY(sb200_hpsi_tt(c, psi, htpsi, ttpsi));
  DeviceGuard dg(c->device);
  const int nblk = 32;
  const int norb = c->orb.norb;
  double* part = nullptr;
  TRY(dalloc(&part, (size_t)norb * nblk * 3));
  int r = launch_energy_parts(c, (const double2*)psi, (const double2*)htpsi, (const double2*)ttpsi, part, nblk);
  std::vector<double> h((size_t)norb * nblk * 3);
  if (r == SB200_OK) {
    cudaError_t e = cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) r = cuda_error(e, "energy partial sums");
  }
  dfree(part);
  TRY(r);
  TRY(check_device_flag(c));
  // calc_eigen_energy (total_energy.f90:505-775): per-orbital sums in block
  // order, then the weighted totals in the reference's (ispin, ik, io) order
  const int nspin = c->orb.nspin, no = c->orb.no, nk = c->orb.nk;
  const double hv = c->g.hvol;
  double ek = 0.0, en = 0.0;
  for (int is = 0; is < nspin; ++is)
    for (int ik = 0; ik < nk; ++ik)
      for (int io = 0; io < no; ++io) {
        const long o = is + (long)nspin * (io + (long)no * ik);
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int b = 0; b < nblk; ++b) {
          s0 += h[(o * nblk + b) * 3 + 0];
          s1 += h[(o * nblk + b) * 3 + 1];
          s2 += h[(o * nblk + b) * 3 + 2];
        }
        esp[io + (long)no * (ik + (long)nk * is)] = s0 * hv;
        const double w = c->orb.weight[o];
        ek += w * s1 * hv;
        en += w * hv * s2;
      }
  *e_kin = ek;
  *e_nloc = en;
  return SB200_OK;
}

int sb200_taylor(sb200_ctx* c, double* tspsi_in, double* tspsi_out, double* sshtpsi, const double* zc, int n_hamil) {
  CHECK_CTX(c);
  TRY(require_ready(c));
  if (!tspsi_in || !tspsi_out || !sshtpsi || !zc) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  if (tspsi_in == tspsi_out || tspsi_in == sshtpsi || tspsi_out == sshtpsi)
    return set_error(SB200_ERR_INVALID_ARG, "taylor buffers must be distinct");
  if (n_hamil < 1 || n_hamil > 16) return set_error(SB200_ERR_INVALID_ARG, "n_hamil out of range");
  DeviceGuard dg(c->device);
  std::vector<double2> z(n_hamil);
  for (int i = 0; i < n_hamil; ++i) z[i] = make_double2(zc[2 * i], zc[2 * i + 1]);
  return issue_taylor(c, (double2*)tspsi_in, (double2*)tspsi_out, (double2*)sshtpsi, z.data(), n_hamil);
}

int sb200_calc_density(sb200_ctx* c, const double* psi, double* rho) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  if (!psi || !rho) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  DeviceGuard dg(c->device);
  const size_t n = (size_t)c->g.npts * c->orb.nspin;
  if (is_device_ptr(rho)) {
    TRY(launch_density(c, (const double2*)psi, rho));
    TRY(scf_density_allreduce(c, rho));
  } else {
    TRY(ensure_stage(c, n * sizeof(double)));
    TRY(launch_density(c, (const double2*)psi, (double*)c->d_stage));
    TRY(scf_density_allreduce(c, (double*)c->d_stage));
    SB_CUDA(cudaMemcpyAsync(rho, c->d_stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  }
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

int sb200_calc_current(sb200_ctx* c, const double* psi, const double vec_Ac[3], double* curr) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  if (!psi || !vec_Ac || !curr) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  if (!c->g.periodic) return set_error(SB200_ERR_UNSUPPORTED, "calc_current needs a periodic grid");
  DeviceGuard dg(c->device);
  TRY(launch_observables(c, (const double2*)psi));
  TRY(launch_project_moments(c, (const double2*)psi));
  SB_CUDA(cudaMemcpyAsync(c->d_result + 8, vec_Ac, 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  for (int is = 0; is < c->orb.nspin; ++is) {
    TRY(launch_finalize(c, 0, 0, SB200_TRANS_TR, 0.0, c->orb.nspin > 1 ? is : -1));
    double res[8];
    SB_CUDA(cudaMemcpyAsync(res, c->d_result, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    SB_CUDA(cudaStreamSynchronize(c->stream));
    for (int d = 0; d < 3; ++d) curr[3 * is + d] = res[d];
  }
  return SB200_OK;
}

int sb200_calc_dip(sb200_ctx* c, const double* rho, double rbox[4]) {
  CHECK_CTX(c);
  TRY(require_ready(c, false));
  if (!rho || !rbox) return set_error(SB200_ERR_INVALID_ARG, "null argument");
  DeviceGuard dg(c->device);
  const size_t n = (size_t)c->g.npts * c->orb.nspin;
  const double* src = rho;
  if (!is_device_ptr(rho)) {
    TRY(ensure_stage(c, n * sizeof(double)));
    SB_CUDA(cudaMemcpyAsync(c->d_stage, rho, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    src = (const double*)c->d_stage;
  }
  TRY(launch_dip(c, src, c->d_result));
  SB_CUDA(cudaMemcpyAsync(rbox, c->d_result, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

int sb200_rt_propagate(sb200_ctx* c, double* psi_a, double* psi_b, double* work, int nt, double dt, const double* zc,
                       int n_hamil, const double* Ac_ext, int trans_longi, double* curr_out, double* rbox_out,
                       double* Ac_tot_out, double** psi_final) {
  CHECK_CTX(c);
  TRY(require_ready(c));
  if (!psi_a || !psi_b || !work || !zc || nt < 0 || n_hamil < 1 || n_hamil > 16)
    return set_error(SB200_ERR_INVALID_ARG, "sb200_rt_propagate: bad argument");
  if (psi_a == psi_b || psi_a == work || psi_b == work)
    return set_error(SB200_ERR_INVALID_ARG, "orbital buffers must be distinct");
  if (trans_longi != SB200_TRANS_TR && trans_longi != SB200_TRANS_LO)
    return set_error(SB200_ERR_INVALID_ARG, "trans_longi must be SB200_TRANS_TR or SB200_TRANS_LO");
  DeviceGuard dg(c->device);
  TRY(alloc_rt(c, nt));
  RTBuffers& r = c->rt;
  const size_t na = 3 * (size_t)(nt + 2);
  if (Ac_ext) SB_CUDA(cudaMemcpyAsync(r.d_Ac_ext, Ac_ext, na * sizeof(double), cudaMemcpyDefault, c->stream));
  else SB_CUDA(cudaMemsetAsync(r.d_Ac_ext, 0, na * sizeof(double), c->stream));
  SB_CUDA(cudaMemsetAsync(r.d_Ac_ind, 0, na * sizeof(double), c->stream));
  SB_CUDA(cudaMemcpyAsync(r.d_Ac_tot, r.d_Ac_ext, na * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  // a continued loop (sb200_rt_set_start / sb200_read_restart): local entries 0
  // and 1 are the steps start_mit and start_mit + 1 (main_tddft.f90:89, itt =
  // Mit + 1 .. nt; read_rtdata, checkpoint_restart.f90:1959-1993)
  if (r.seed_on) {
    SB_CUDA(cudaMemcpyAsync(r.d_Ac_tot, r.seed_tot, 6 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    SB_CUDA(cudaMemcpyAsync(r.d_Ac_ind, r.seed_ind, 6 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  r.loop_mit0 = r.start_mit;
  const int one = 1;
  SB_CUDA(cudaMemcpyAsync(r.d_step, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  if (!c->g.periodic) {
    const double zero[3] = {0.0, 0.0, 0.0};
    SB_CUDA(cudaMemcpyAsync(c->d_result + 8, zero, 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    TRY(launch_prep_k(c, c->d_result + 8, 0, 0, c->d_kcoef, false));
  }
  std::vector<double2> z(n_hamil);
  for (int i = 0; i < n_hamil; ++i) z[i] = make_double2(zc[2 * i], zc[2 * i + 1]);
  double2* A = (double2*)psi_a;
  double2* B = (double2*)psi_b;
  double2* W = (double2*)work;
  TRY(scf_rt_prepare(c));
  TRY(nonorth_prepare(c));
  if (c->length_gauge && !c->g.periodic) {  // E_ext(itt) = -(Ac_ext(itt+1) - Ac_ext(itt)) / dt, initialization_rt.f90:180-183
    std::vector<double> ac(na, 0.0), e(na, 0.0);
    if (Ac_ext) SB_CUDA(cudaMemcpy(ac.data(), Ac_ext, na * sizeof(double), cudaMemcpyDefault));
    for (int itt = 0; itt <= nt; ++itt)
      for (int d = 0; d < 3; ++d) e[3 * itt + d] = -(ac[3 * (itt + 1) + d] - ac[3 * itt + d]) / dt;
    for (int d = 0; d < 3; ++d) e[3 * (nt + 1) + d] = e[3 * nt + d];
    if (c->eext_cap < na) {
      dfree(c->d_eext);
      c->eext_cap = 0;
      TRY(dalloc(&c->d_eext, na));
      c->eext_cap = na;
    }
    const size_t nv = (size_t)c->g.npts * c->orb.nspin;
    if (c->vloc_base_cap < nv) {
      dfree(c->d_vloc_base);
      c->vloc_base_cap = 0;
      TRY(dalloc(&c->d_vloc_base, nv));
      c->vloc_base_cap = nv;
    }
    SB_CUDA(cudaMemcpyAsync(c->d_eext, e.data(), na * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    SB_CUDA(cudaMemcpyAsync(c->d_vloc_base, c->d_vloc, nv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    c->lg_active = 1;
  }
  if (c->gs_interval >= 1) {  // the loop's Gram-Schmidt: scratch and body stream
    const size_t need = gs_complex_part_len(c) + (size_t)c->orb.no;
    if (c->gs_scratch_cap < need) {
      dfree(c->d_gs_scratch);
      c->gs_scratch_cap = 0;
      TRY(dalloc(&c->d_gs_scratch, need));
      c->gs_scratch_cap = need;
    }
    if (!c->gs_side) SB_CUDA(cudaStreamCreateWithFlags(&c->gs_side, cudaStreamNonBlocking));
  }
  if (c->pred_corr && !c->aetrs) {  // the step's saved input, V_tmp and the initial V0
    const size_t nv = (size_t)c->g.npts * c->orb.nspin, nb = (size_t)c->g.npts * c->orb.norb;
    if (c->pc_psi_cap < nb) {
      dfree(c->d_pc_psi);
      c->pc_psi_cap = 0;
      TRY(dalloc(&c->d_pc_psi, nb));
      c->pc_psi_cap = nb;
    }
    if (c->pc_v_cap < 2 * nv) {
      dfree(c->d_pc_v);
      c->pc_v_cap = 0;
      TRY(dalloc(&c->d_pc_v, 2 * nv));
      c->pc_v_cap = 2 * nv;
    }
    SB_CUDA(cudaMemcpyAsync(c->d_pc_v + nv, c->d_vloc, nv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  if (c->aetrs) {  // vloc_old(:,1:2) = V_local (initialization_rt.f90:287-292)
    const size_t nv = (size_t)c->g.npts * c->orb.nspin;
    if (c->vloc_old_cap < 2 * nv) {
      dfree(c->d_vloc_old);
      c->vloc_old_cap = 0;
      TRY(dalloc(&c->d_vloc_old, 2 * nv));
      c->vloc_old_cap = 2 * nv;
    }
    SB_CUDA(cudaMemcpyAsync(c->d_vloc_old, c->d_vloc, nv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    SB_CUDA(cudaMemcpyAsync(c->d_vloc_old + nv, c->d_vloc, nv * sizeof(double), cudaMemcpyDeviceToDevice,
                            c->stream));
  }
  SB_CUDA(cudaStreamSynchronize(c->stream));

  // Two steps (A->B, B->A) captured as one CUDA graph and replayed.
  cudaGraphExec_t exec2 = nullptr;
  const int pairs = c->timing ? 0 : nt / 2;
  int rc = SB200_OK;
  // with AETRS every step maps A -> A (B its half-step scratch)
  double2* A2 = c->aetrs ? A : B;
  double2* B2 = c->aetrs ? B : A;
  if (c->timing) {  // instrumented: every launch bracketed by events, no graph
    for (int i = 0; i + 1 < nt; i += 2) {
      TRY(issue_rt_step(c, A, B, W, z.data(), n_hamil, trans_longi, dt));
      TRY(timing_flush(c));
      TRY(issue_rt_step(c, A2, B2, W, z.data(), n_hamil, trans_longi, dt));
      TRY(timing_flush(c));
    }
  }
  if (pairs > 0) {
    cudaGraph_t graph = nullptr;
    SB_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    rc = issue_rt_step(c, A, B, W, z.data(), n_hamil, trans_longi, dt);
    if (rc == SB200_OK) rc = issue_rt_step(c, A2, B2, W, z.data(), n_hamil, trans_longi, dt);
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc != SB200_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&exec2, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
    for (int i = 0; i < pairs && rc == SB200_OK; ++i) {
      e = cudaGraphLaunch(exec2, c->stream);
      if (e != cudaSuccess) rc = cuda_error(e, "cudaGraphLaunch");
    }
    cudaGraphExecDestroy(exec2);
    if (rc != SB200_OK) return rc;
  }
  double2* final_buf = A;
  if (nt % 2 == 1) {
    TRY(issue_rt_step(c, A, B, W, z.data(), n_hamil, trans_longi, dt));
    final_buf = c->aetrs ? A : B;
  }
  if (curr_out && nt > 0)
    SB_CUDA(cudaMemcpyAsync(curr_out, r.d_curr, 3 * (size_t)nt * sizeof(double), cudaMemcpyDefault, c->stream));
  if (rbox_out && nt > 0)
    SB_CUDA(cudaMemcpyAsync(rbox_out, r.d_rbox, 4 * (size_t)nt * sizeof(double), cudaMemcpyDefault, c->stream));
  if (Ac_tot_out)
    SB_CUDA(cudaMemcpyAsync(Ac_tot_out, r.d_Ac_tot, na * sizeof(double), cudaMemcpyDefault, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  SB_CUDA(cudaGetLastError());
  TRY(check_device_flag(c));
  if (c->lg_active) {  // the field-free V_local the last step's update_vlocal leaves
    c->lg_active = 0;
    TRY(launch_vloc_restore(c));
    SB_CUDA(cudaStreamSynchronize(c->stream));
  }
  r.last_mit = r.loop_mit0 + nt;
  r.last_nt = nt;
  r.start_mit = 0;
  r.loop_mit0 = 0;
  r.seed_on = false;
  if (psi_final) *psi_final = (double*)final_buf;
  // leave hpsi coefficients consistent with system%vec_Ac for later hpsi calls
  TRY(refresh_k(c));
  return SB200_OK;
}

int sb200_rt_set_start(sb200_ctx* c, int mit, const double Ac_tot[6], const double Ac_ind[6]) {
  CHECK_CTX(c);
  if (mit < 0) return set_error(SB200_ERR_INVALID_ARG, "sb200_rt_set_start: Mit < 0");
  if (Ac_ind && !Ac_tot) return set_error(SB200_ERR_INVALID_ARG, "sb200_rt_set_start: Ac_ind without Ac_tot");
  RTBuffers& r = c->rt;
  r.start_mit = mit;
  r.seed_on = Ac_tot != nullptr || Ac_ind != nullptr;
  for (int i = 0; i < 6; ++i) {
    r.seed_tot[i] = Ac_tot ? Ac_tot[i] : 0.0;
    r.seed_ind[i] = Ac_ind ? Ac_ind[i] : 0.0;
  }
  return SB200_OK;
}

int sb200_rt_get_state(sb200_ctx* c, int* mit, double Ac_tot[6], double Ac_ind[6]) {
  CHECK_CTX(c);
  RTBuffers& r = c->rt;
  if (r.last_nt < 0) return set_error(SB200_ERR_STATE, "no sb200_rt_propagate has run on this context");
  DeviceGuard dg(c->device);
  if (mit) *mit = r.last_mit;
  const size_t off = 3 * (size_t)r.last_nt;  // local entries nt and nt + 1
  if (Ac_tot)
    SB_CUDA(cudaMemcpyAsync(Ac_tot, r.d_Ac_tot + off, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (Ac_ind)
    SB_CUDA(cudaMemcpyAsync(Ac_ind, r.d_Ac_ind + off, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  SB_CUDA(cudaStreamSynchronize(c->stream));
  return SB200_OK;
}

}  // extern "C"
