// sb200_tma_body.cuh -- the TMA-fed tiled hpsi sweep as a device function,
// shared by the per-system kernel (sb200_tma_stencil.cu) and the batched
// persistent kernel (sb200_batch.cu).  See sb200_tma_stencil.cu for the design.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "sb200_internal.cuh"
#include "sb200_stencil.cuh"
#include "sb200_tiled_body.cuh"
#include "sb200_tma.cuh"

namespace sb200 {
namespace tmak {


using namespace tiled;

constexpr int TX = 32, TY = 8, NT = TX * TY, HALO = ND;
constexpr int RING = 8;   // input planes resident / in flight
constexpr int ARING = 4;  // accumulator planes in flight
constexpr int TMA_MAX_NLMA = 512;  // projections staged in shared memory (else read from global)

struct TmaMaps {
  CUtensorMap in;    // input planes: (2 SX) x SY box, or (2 TX) x TY for the periodic centre rows
  CUtensorMap inh;   // periodic: (2 TX) x 4 halo rows
  CUtensorMap acc;   // FP64 accumulator tile (2 TX) x TY
  CUtensorMap d32;   // FP32 correction tile (2 TX) x TY
};

template <int MODE, bool PER>
struct Geo {
  using R = typename ModeT<MODE>::R;
  using C2 = typename Cx<R>::T;
  static constexpr int SX = PER ? TX : TX + 2 * HALO;
  static constexpr int SY = TY + 2 * HALO;
  static constexpr int PLANE = SX * SY;  // complex values per ring slot
  static constexpr unsigned PLANE_BYTES = PLANE * sizeof(C2);
  static constexpr bool ACC64 = (MODE == 2 || MODE == 3 || MODE == 8);  // reads psi_out
  static constexpr bool D32 = (MODE == 7 || MODE == 8);                 // reads the FP32 correction
  static constexpr unsigned ACC_BYTES = ACC64 ? NT * 16u : 0u;
  static constexpr unsigned D32_BYTES = D32 ? NT * 8u : 0u;
  static constexpr size_t RING_OFF = 0;
  static constexpr size_t ACC_OFF = RING_OFF + (size_t)RING * PLANE_BYTES;
  static constexpr size_t D32_OFF = ACC_OFF + (size_t)ARING * ACC_BYTES;
  static constexpr size_t BAR_OFF = D32_OFF + (size_t)ARING * D32_BYTES;
  static constexpr size_t PS_OFF = BAR_OFF + 128;  // projections of the item's orbital
  static constexpr size_t SMEM = PS_OFF + (size_t)TMA_MAX_NLMA * 16 + 128;  // + alignment slack
};

template <int MODE, bool PER>
__device__ __forceinline__ void issue_plane(const TmaMaps& m, unsigned char* base, uint64_t* pbar, int r, int q,
                                            int x0, int y0, int o, int nz, int ny) {
  using G = Geo<MODE, PER>;
  const int slot = r & (RING - 1);
  unsigned char* dst = base + G::RING_OFF + (size_t)slot * G::PLANE_BYTES;
  tma::mbar_arrive_expect_tx(&pbar[slot], G::PLANE_BYTES);
  if (!PER) {
    tma::tensor_load_4d(dst, &m.in, 2 * (x0 - HALO), y0 - HALO, q, o, &pbar[slot]);
  } else {
    int qz = q % nz;
    if (qz < 0) qz += nz;
    const int ya = y0 - HALO < 0 ? y0 - HALO + ny : y0 - HALO;
    const int yb = y0 + TY >= ny ? y0 + TY - ny : y0 + TY;
    constexpr size_t ROW = (size_t)TX * sizeof(typename G::C2);
    tma::tensor_load_4d(dst, &m.inh, 0, ya, qz, o, &pbar[slot]);
    tma::tensor_load_4d(dst + HALO * ROW, &m.in, 0, y0, qz, o, &pbar[slot]);
    tma::tensor_load_4d(dst + (HALO + TY) * ROW, &m.inh, 0, yb, qz, o, &pbar[slot]);
  }
}

template <int MODE, bool PER>
__device__ __forceinline__ void issue_acc(const TmaMaps& m, unsigned char* base, uint64_t* abar, int k, int z,
                                          int x0, int y0, int o) {
  using G = Geo<MODE, PER>;
  const int slot = k & (ARING - 1);
  tma::mbar_arrive_expect_tx(&abar[slot], G::ACC_BYTES + G::D32_BYTES);
  if (G::ACC64) tma::tensor_load_4d(base + G::ACC_OFF + (size_t)slot * G::ACC_BYTES, &m.acc, 2 * x0, y0, z, o, &abar[slot]);
  if (G::D32) tma::tensor_load_4d(base + G::D32_OFF + (size_t)slot * G::D32_BYTES, &m.d32, 2 * x0, y0, z, o, &abar[slot]);
}

// f(integral_constant<J>, k0 + J) for J = J0 .. N-1 while k0 + J < nsteps;
// false as soon as one call returns false
template <int J, int N, typename F>
__device__ __forceinline__ bool run_steps(F& f, int k0, int nsteps) {
  if constexpr (J < N) {
    if (k0 + J >= nsteps) return true;
    if (!f(std::integral_constant<int, J>{}, k0 + J)) return false;
    return run_steps<J + 1, N>(f, k0, nsteps);
  } else {
    return true;
  }
}

// One work item: tile bx, z chunk by, orbital bz.  `base` is the 128-byte
// aligned shared-memory area of Geo<MODE, PER>; its barriers are initialised
// by the caller and keep their phases across items in pmask / amask (bit s =
// parity of the next completion of slot s).  Returns false when a copy did
// not arrive in time (err is set and the CTA's other copies are drained).
template <int MODE, bool PER>
__device__ __forceinline__ bool tma_body(const TmaMaps& maps, void* __restrict__ hout, double2* __restrict__ acc,
                                         float2* __restrict__ d32, const TiledArgs& a, int* __restrict__ err,
                                         int bx, int by, int bz, unsigned char* base, uint32_t& pmask,
                                         uint32_t& amask) {
  using G = Geo<MODE, PER>;
  using R = typename G::R;
  using C2 = typename G::C2;
  constexpr int SX = G::SX;
  const C2* ring = (const C2*)(base + G::RING_OFF);
  const double2* accr = (const double2*)(base + G::ACC_OFF);
  const float2* d32r = (const float2*)(base + G::D32_OFF);
  uint64_t* pbar = (uint64_t*)(base + G::BAR_OFF);
  double2* psm = (double2*)(base + G::PS_OFF);
  uint64_t* abar = pbar + RING;

  const int t = threadIdx.x;
  const int tx = t & (TX - 1), ty = t / TX;
  const int ntx = (a.nx + TX - 1) / TX;
  const int x0 = (bx % ntx) * TX, y0 = (bx / ntx) * TY;
  const int x = x0 + tx, y = y0 + ty;
  const bool active = (x < a.nx) && (y < a.ny);
  const int zc0 = by * a.zchunk;
  const int zc1 = min(a.nz, zc0 + a.zchunk);
  const int nsteps = zc1 - zc0;
  const int ntot = nsteps + 2 * HALO;  // input planes zc0-4 .. zc1+3
  const int o = bz;
  const int ik = o / a.nspin_no;
  const int ispin = o % a.nspin;
  const double* kc = a.kcoef + (long)KC * ik;
  const R kx = (R)kc[0], ky = (R)kc[1], kz = (R)kc[2], lap0 = (R)kc[3];
  const int ctr = (ty + HALO) * SX + (PER ? tx : tx + HALO);
  const long sz = (long)a.nx * a.ny;
  const long pxy = (long)y * a.nx + x;
  constexpr bool GRAD = PER;

  // copies issued / waited, tracked identically by every thread
  int p_issued = 0, p_waited = 0, a_issued = 0, a_waited = 0;
  const int pro = ntot < RING ? ntot : RING;
  if (t == 0) {
    tma::fence_proxy_async_smem();  // the previous item's reads of the rings come first
    for (int r = 0; r < pro; ++r)
      issue_plane<MODE, PER>(maps, base, pbar, r, zc0 - HALO + r, x0, y0, o, a.nz, a.ny);
    if (G::ACC64 || G::D32)
      for (int k = 0; k < ARING && k < nsteps; ++k) issue_acc<MODE, PER>(maps, base, abar, k, zc0 + k, x0, y0, o);
  }
  p_issued = pro;
  if (G::ACC64 || G::D32) a_issued = nsteps < ARING ? nsteps : ARING;

  // projections of this orbital into shared memory (read before the first
  // barrier below; the previous item's readers have all passed its last barrier)
  const bool ps_smem = a.nlma > 0 && a.nlma <= TMA_MAX_NLMA;
  if (ps_smem)
    for (int i = t; i < a.nlma; i += NT) psm[i] = a.proj[(long)o * a.nlma + i];
  bool ok = true;
  C2 w[2 * HALO + 1];
  // window planes zc0-4 .. zc0+3
#pragma unroll
  for (int r = 0; r < 2 * HALO; ++r) {
    ok = tma::mbar_wait(&pbar[r], (pmask >> r) & 1u) && ok;
    pmask ^= 1u << r;
    w[r] = ring[(size_t)r * G::PLANE + ctr];
  }
  p_waited = 2 * HALO;
  bool all_ok = __syncthreads_and(ok);  // the same in every thread
  if (all_ok) {
    if (t == 0) {  // the four pre-window slots take planes zc0+4 .. zc0+7
      tma::fence_proxy_async_smem();
      for (int r = RING; r < RING + HALO && r < ntot; ++r)
        issue_plane<MODE, PER>(maps, base, pbar, r, zc0 - HALO + r, x0, y0, o, a.nz, a.ny);
    }
    p_issued = ntot < RING + HALO ? ntot : RING + HALO;

    const C2 czc = Cx<R>::make((R)a.zc.x, (R)a.zc.y);
    const R* vsrc;
    if (sizeof(R) == 8) vsrc = (const R*)(a.vloc + (long)ispin * a.npts);
    else vsrc = (const R*)(a.vloc32 + (long)ispin * a.npts);
    R vl_n = active ? __ldg(vsrc + (long)zc0 * sz + pxy) : (R)0;
    int pm_n = (active && a.nlma > 0) ? __ldg(a.pmap + (long)zc0 * sz + pxy) : -1;
    // pair form of the KB scatter: the first pair of the next plane's point
    // is loaded at the end of each step, from pm_n (loaded at its start); in
    // the inner FP64 terms and the FP32 terms, and in the first FP64 term of
    // periodic grids (where it spills a little but still gains; measured)
    constexpr bool AHEAD = (MODE == 2 || MODE == 3 || MODE >= 6 || (MODE == 1 && PER));
    const bool pairs = AHEAD && a.nlma > 0 && a.use_pairs;
    const double2* pair_ph = pairs ? a.pair_ph + (a.phase_per_k ? (long)ik * a.npair : 0L) : nullptr;
    Pair1<R> f1;
    f1.lm = 0;
    if (pairs) load_pair1<R>(f1, pm_n, a, pair_ph);
    // FP64 stencils: the window rotates through the registers -- in step j of
    // a group of nine, plane z - 4 + i sits in w[(j + i) % 9] (constant
    // indices, no moves); FP32 stencils (issue-bound, code-size sensitive)
    // shift the window after each step instead (j = 0 throughout)
    constexpr int NWIN = 2 * HALO + 1;
    constexpr bool ROTATE = (MODE < 6);
    auto step = [&](auto jc, const int k) -> bool {
      constexpr int j = decltype(jc)::value;
      const int z = zc0 + k;
      const int rf = k + 2 * HALO;  // plane z+4 feeds the window
      ok = tma::mbar_wait(&pbar[rf & (RING - 1)], (pmask >> (rf & (RING - 1))) & 1u) && ok;
      pmask ^= 1u << (rf & (RING - 1));
      w[(j + 2 * HALO) % NWIN] = ring[(size_t)(rf & (RING - 1)) * G::PLANE + ctr];
      p_waited = rf + 1;
      if (G::ACC64 || G::D32) {
        ok = tma::mbar_wait(&abar[k & (ARING - 1)], (amask >> (k & (ARING - 1))) & 1u) && ok;
        amask ^= 1u << (k & (ARING - 1));
        a_waited = k + 1;
      }
      const R vl = vl_n;
      const int pm = pm_n;
      if (k + 1 < nsteps && active) {
        vl_n = __ldg(vsrc + (long)(z + 1) * sz + pxy);
        if (a.nlma > 0) pm_n = __ldg(a.pmap + (long)(z + 1) * sz + pxy);
      }
      if (active) {
        const C2* P = ring + (size_t)((k + HALO) & (RING - 1)) * G::PLANE;
        C2 vx = Cx<R>::make(0, 0), wx = vx, vy = vx, wy = vx, vz = vx, wz = vx;
#pragma unroll
        for (int s = 1; s <= HALO; ++s) {
          C2 tp, tm;
          if (PER) {
            tp = P[(ty + HALO) * SX + ((tx + s) & (TX - 1))];
            tm = P[(ty + HALO) * SX + ((tx - s) & (TX - 1))];
          } else {
            tp = P[ctr + s];
            tm = P[ctr - s];
          }
          vx = cfma((R)a.lapt[s - 1], cadd(tp, tm), vx);
          if (GRAD) wx = cfma((R)a.nab[s - 1], csub(tp, tm), wx);
        }
#pragma unroll
        for (int s = 1; s <= HALO; ++s) {
          const C2 tp = P[ctr + s * SX], tm = P[ctr - s * SX];
          vy = cfma((R)a.lapt[4 + s - 1], cadd(tp, tm), vy);
          if (GRAD) wy = cfma((R)a.nab[4 + s - 1], csub(tp, tm), wy);
        }
#pragma unroll
        for (int s = 0; s < HALO; ++s) {
          const C2 tp = w[(j + HALO + 1 + s) % NWIN], tm = w[(j + HALO - 1 - s) % NWIN];
          vz = cfma((R)a.lapt[8 + s], cadd(tp, tm), vz);
          if (GRAD) wz = cfma((R)a.nab[8 + s], csub(tp, tm), wz);
        }
        const C2 v = cadd(vz, cadd(vy, vx));
        const C2 c = w[(j + HALO) % NWIN];
        C2 h;  // stencil value, then + KB term
        h = hcore(vl, lap0, c, v);
        if (GRAD) {
          const C2 ww = cfma(kz, wz, cfma(ky, wy, cscal(kx, wx)));
          h.x += ww.y;
          h.y -= ww.x;
        }
        if (a.nlma > 0 && pm >= 0 && a.use_pairs) {
          if (AHEAD) h = kb_pairs_ahead<R>(h, pm, ps_smem ? psm : a.proj + (long)o * a.nlma, a, ik, f1);
          else h = kb_pairs<R>(h, pm, ps_smem ? psm : a.proj + (long)o * a.nlma, a, ik);
        } else if (a.nlma > 0 && pm >= 0) {
          const double2* pj = ps_smem ? psm : a.proj + (long)o * a.nlma;
          const double2* zk = a.ent_zk + (a.phase_per_k ? (long)ik * a.nent : 0L);
          const int e0 = pm >> 8, e1 = e0 + (pm & 255);
          for (int e = e0; e < e1; e += 8) {  // entries eight at a time, summed in entry order
            int l[8];
            double2 zv[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const int ee = min(e + i, e1 - 1);
              l[i] = __ldg(a.ent_lma + ee);
              zv[i] = __ldg(zk + ee);
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
              if (e + i < e1) {
                const double2 pv = pj[l[i]];
                h = cadd(h, cmul(Cx<R>::make((R)pv.x, (R)pv.y), Cx<R>::make((R)zv[i].x, (R)zv[i].y)));
              }
          }
        }
        const long gi = (long)o * a.npts + (long)z * sz + pxy;
        const int ti = (k & (ARING - 1)) * NT + t;
        if (ModeT<MODE>::store_h) {
          if (ModeT<MODE>::h32) ((float2*)hout)[gi] = make_float2((float)h.x, (float)h.y);
          else ((double2*)hout)[gi] = make_double2((double)h.x, (double)h.y);
        }
        if (MODE == 1 || MODE == 4 || MODE == 5) {
          const double2 cd = make_double2((double)c.x, (double)c.y);
          const double2 hd = make_double2((double)h.x, (double)h.y);
          acc[gi] = cadd(cd, cmul(a.zc, hd));
        } else if (MODE == 2 || MODE == 3) {
          const double2 hd = make_double2((double)h.x, (double)h.y);
          acc[gi] = cadd(accr[ti], cmul(a.zc, hd));
        } else if (MODE == 6) {
          const C2 tt = cmul(czc, h);
          d32[gi] = make_float2((float)tt.x, (float)tt.y);
        } else if (MODE == 7) {
          const float2 dd = d32r[ti];
          const C2 tt = cadd(Cx<R>::make((R)dd.x, (R)dd.y), cmul(czc, h));
          d32[gi] = make_float2((float)tt.x, (float)tt.y);
        } else if (MODE == 8) {
          const float2 dd = d32r[ti];
          const C2 tt = cadd(Cx<R>::make((R)dd.x, (R)dd.y), cmul(czc, h));
          acc[gi] = cadd(accr[ti], make_double2((double)tt.x, (double)tt.y));
        }
        if (pairs && k + 1 < nsteps) load_pair1<R>(f1, pm_n, a, pair_ph);
      }
      // warp 0 waits for the next step's copies before the step barrier, so the
      // other warps find them complete at their own (first) try-wait and
      // block in the barrier instead of polling
      if (t < 32 && k + 1 < nsteps) {
        const int rf1 = k + 1 + 2 * HALO;
        ok = tma::mbar_wait(&pbar[rf1 & (RING - 1)], (pmask >> (rf1 & (RING - 1))) & 1u) && ok;
        if (G::ACC64 || G::D32)
          ok = tma::mbar_wait(&abar[(k + 1) & (ARING - 1)], (amask >> ((k + 1) & (ARING - 1))) & 1u) && ok;
      }
      all_ok = __syncthreads_and(ok);
      if (!all_ok) return false;
      if (t == 0) {  // refill the slots of plane z and of accumulator step k
        tma::fence_proxy_async_smem();
        const int rn = k + RING + HALO;  // plane z+8
        if (rn < ntot) issue_plane<MODE, PER>(maps, base, pbar, rn, zc0 - HALO + rn, x0, y0, o, a.nz, a.ny);
        if ((G::ACC64 || G::D32) && k + ARING < nsteps)
          issue_acc<MODE, PER>(maps, base, abar, k + ARING, z + ARING, x0, y0, o);
      }
      if (k + RING + HALO < ntot) p_issued = k + RING + HALO + 1;
      if ((G::ACC64 || G::D32) && k + ARING < nsteps) a_issued = k + ARING + 1;
      return true;
    };
    if (ROTATE) {
      for (int k0 = 0; k0 < nsteps; k0 += NWIN)
        if (!run_steps<0, NWIN>(step, k0, nsteps)) break;
    } else {
      for (int k = 0; k < nsteps; ++k) {
        if (!step(std::integral_constant<int, 0>{}, k)) break;
#pragma unroll
        for (int i = 0; i < 2 * HALO; ++i) w[i] = w[i + 1];
      }
    }
  }
  if (!all_ok) {
    // a copy did not arrive in time: flag it, wait (bounded) for the copies
    // still in flight into this CTA's shared memory, and leave
    if (t == 0) {
      atomicExch(err, 1);
      for (int r = p_waited; r < p_issued; ++r) {
        tma::mbar_wait(&pbar[r & (RING - 1)], (pmask >> (r & (RING - 1))) & 1u);
        pmask ^= 1u << (r & (RING - 1));
      }
      for (int k = a_waited; k < a_issued; ++k) {
        tma::mbar_wait(&abar[k & (ARING - 1)], (amask >> (k & (ARING - 1))) & 1u);
        amask ^= 1u << (k & (ARING - 1));
      }
    }
    __syncthreads();
  }
  return all_ok;
}


// barriers of a Geo<MODE, PER> area, initialised once per CTA
template <int MODE, bool PER>
__device__ __forceinline__ void tma_init_barriers(unsigned char* base) {
  using G = Geo<MODE, PER>;
  if (threadIdx.x == 0) {
    uint64_t* bar = (uint64_t*)(base + G::BAR_OFF);
    for (int i = 0; i < RING + ARING; ++i) tma::mbar_init(&bar[i], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
}

__device__ __forceinline__ unsigned char* tma_area(unsigned char* raw) {
  return (unsigned char*)(((uintptr_t)raw + 127) & ~(uintptr_t)127);
}

}  // namespace tmak

// 4-D map over an orbital block [norb][nz][ny][2 nx] of FP64 or FP32 reals
// with the given box; false when the copy engine cannot address it.
bool make_tma_map(CUtensorMap* m, const void* base, bool f32, const GridInfo& g, int norb, int box0, int box1);

}  // namespace sb200
