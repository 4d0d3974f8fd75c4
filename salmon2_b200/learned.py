"""Training and evaluation driver of the learned CG preconditioner.

The network and its kernels live in ``libsalmon_b200.so`` (sb200_learned_*);
this module only orchestrates them:

* ``converge``: the ground-state eigensolver loop the reference runs in its SCF
  (``scf_iteration_step``, ``src/gs/scf_iteration.f90:22-138``, with a fixed
  potential): ``gscg_rwf`` iterations, Gram-Schmidt and subspace
  diagonalisation, until the eigenvalues stop changing.
* ``collect_samples``: residual -> correction pairs from the plain (low-pass
  preconditioned) solver's own runs: for each iterate x and residual
  g = Hx - <x|H|x> x, the network input is [g/rms(g), V_local], the offset is
  lowpass(g)/rms(g) and the target direction is minus the part of x outside
  the converged occupied subspace span(x*) -- the error that no rotation
  within the subspace (Gram-Schmidt, subspace diagonalisation) removes.
* ``train``: Adam steps through ``sb200_learned_train_step`` on the GPU.

Array preparation uses torch tensors on the device; all network arithmetic
(forward, backward, optimiser) is the library's.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from ._lib import check, lib


def _lowpass(torch, g, shape, hgs, alpha=0.6):
    """preconditioning.f90:25-77 on [B, n] tensors, zero (Dirichlet) boundary."""
    nx, ny, nz = shape
    B = g.shape[0]
    G = g.reshape(B, nz, ny, nx)
    P = torch.nn.functional.pad(G, (1, 1, 1, 1, 1, 1))
    lap = ((P[:, 1:-1, 1:-1, 2:] - 2 * G + P[:, 1:-1, 1:-1, :-2]) / hgs[0] ** 2 +
           (P[:, 1:-1, 2:, 1:-1] - 2 * G + P[:, 1:-1, :-2, 1:-1]) / hgs[1] ** 2 +
           (P[:, 2:, 1:-1, 1:-1] - 2 * G + P[:, :-2, 1:-1, 1:-1]) / hgs[2] ** 2)
    omega = 2.0 * (1.0 - alpha)
    d = -0.5 * sum(-2.0 / h ** 2 for h in hgs)
    return (omega / d * (2.0 * G - omega / d * (-0.5 * lap))).reshape(B, -1)


def converge(ctx, psi, tol=1e-8, max_outer=400, precondition="lowpass", ncg=4, record=None, ref=None):
    """Outer loop gscg + Gram-Schmidt + subspace diagonalisation.  Stops when
    max_i |eps_i - ref_i| <= tol (Hartree) if reference eigenvalues ``ref`` are
    given, else when max_i |eps_i - eps_i(previous outer iteration)| <= tol.
    Returns a dict with the eigenvalues, outer iterations, CG iterations, wall
    time and whether the criterion was met."""
    torch = ctx.torch
    prev = None
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    it = 0
    ev = None
    done = False
    for it in range(1, max_outer + 1):
        if record is not None:
            record(psi)
        ctx.gscg(psi, ncg=ncg, precondition=precondition)
        ctx.gram_schmidt_real(psi)
        ev = ctx.subspace_diag_real(psi)
        if ref is not None:
            if np.max(np.abs(ev - ref)) <= tol:
                done = True
                break
        elif prev is not None and np.max(np.abs(ev - prev)) <= tol:
            done = True
            break
        prev = ev
    torch.cuda.synchronize()
    return dict(evals=ev, outer=it, cg_iters=it * ncg, seconds=time.perf_counter() - t0, converged=done)


def collect_samples(ctx, psi0, n_outer=12, ncg=4, tol=1e-10):
    """Residual -> correction samples from a plain low-pass CG run."""
    torch = ctx.torch
    s = ctx.sys
    ref = psi0.clone()
    converge(ctx, ref, tol=tol, max_outer=600, precondition="lowpass", ncg=ncg)
    xstar = ref.reshape(s.no, -1)
    hvol = float(s.grid.hvol)
    shape = s.grid.shape
    V = torch.from_numpy(np.ascontiguousarray(s.V_local[..., 0].ravel(order="F"))).to(xstar)
    x0s, offs, tgts = [], [], []
    h = ctx.gs_empty()

    def record(psi):
        ctx.hpsi_real(psi, h)
        torch.cuda.synchronize()
        X = psi.reshape(s.no, -1)
        HX = h.reshape(s.no, -1)
        eps = (X * HX).sum(1, keepdim=True) / (X * X).sum(1, keepdim=True)
        g = HX - eps * X
        # error of the iterate against the converged subspace: minus its part
        # outside span(x*), which no rotation inside the subspace removes
        # (orthonormal x* in the hvol metric: the projector needs hvol)
        e = -(X - (X @ xstar.T) @ xstar * hvol)
        rms = torch.sqrt((g * g).mean(1, keepdim=True)).clamp_min(1e-300)
        gn = g / rms
        x0 = torch.stack([gn, V.expand_as(gn)], dim=1)
        x0s.append(x0.float())
        offs.append((_lowpass(torch, g, shape, s.grid.hgs) / rms).float())
        tgts.append(e.float())

    psi = psi0.clone()
    converge(ctx, psi, tol=0.0, max_outer=n_outer, precondition="lowpass", ncg=ncg, record=record)
    return torch.cat(x0s), torch.cat(offs), torch.cat(tgts)


def initial_params(seed=0, channels=None):
    """Training start: He-normal hidden layers, zero biases and a zero output
    layer (so the starting network is the low-pass preconditioner and every
    layer receives gradient).  Layout [W1, b1, W2, b2, W3, b3] with W1
    (C, 2, 27), W2 (C, C, 27), W3 (1, C, 27) as in sb200_learned.cu."""
    C_ = _lib.LEARNED_CHANNELS if channels is None else channels
    rng = np.random.default_rng(seed)
    w1 = rng.standard_normal(C_ * 2 * 27) * np.sqrt(2.0 / (2 * 27))
    w2 = rng.standard_normal(C_ * C_ * 27) * np.sqrt(2.0 / (C_ * 27))
    p = np.concatenate([w1, np.zeros(C_), w2, np.zeros(C_), np.zeros(C_ * 27), np.zeros(1)]).astype(np.float32)
    assert p.size == _lib.LEARNED_NPARAM
    return p


def init(ctx, batch, params=None):
    """Load parameters (None: all zero, the network that adds nothing to the
    low-pass preconditioner)."""
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
    check(lib().sb200_learned_init(ctx.h, None if p is None else C.c_void_p(p.ctypes.data), _lib.LEARNED_NPARAM,
                                   int(batch)))


def get_params(ctx):
    out = np.zeros(_lib.LEARNED_NPARAM, np.float32)
    check(lib().sb200_learned_get_params(ctx.h, C.c_void_p(out.ctypes.data), _lib.LEARNED_NPARAM))
    return out


def train(ctx, x0, off, tgt, steps=300, batch=8, lr=1e-3, seed=0, log_every=0):
    """Adam on random mini-batches of the device-resident samples."""
    torch = ctx.torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = x0.shape[0]
    losses = []
    lv = C.c_double(0.0)
    for step in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g).to(x0.device)
        xb, ob, tb = x0[idx].contiguous(), off[idx].contiguous(), tgt[idx].contiguous()
        check(lib().sb200_learned_train_step(ctx.h, C.c_void_p(xb.data_ptr()), C.c_void_p(ob.data_ptr()),
                                             C.c_void_p(tb.data_ptr()), batch, float(lr), C.byref(lv)))
        losses.append(lv.value / batch)
        if log_every and step % log_every == 0:
            print(f"step {step} loss {losses[-1]:.4f}", flush=True)
    return np.array(losses)


def eval_loss(ctx, x0, off, tgt, batch=8):
    lv = C.c_double(0.0)
    tot = 0.0
    n = x0.shape[0]
    for i in range(0, n - batch + 1, batch):
        check(lib().sb200_learned_loss_grad(ctx.h, C.c_void_p(x0[i:i + batch].data_ptr()),
                                            C.c_void_p(off[i:i + batch].data_ptr()),
                                            C.c_void_p(tgt[i:i + batch].data_ptr()), batch, C.byref(lv), None))
        tot += lv.value
    return tot / max(1, (n // batch) * batch)


def evaluate(ctx, psi_ref_layout, tol=1e-8, max_outer=600, ncg=4, restart_batch=None):
    """Outer iterations and wall time for the low-pass, learned and
    unpreconditioned CG to reach the converged eigenvalues (tightly converged
    low-pass CG, 1e-12 Ha, as the reference values) within `tol` Hartree.
    With ``restart_batch`` (the network's batch) also "lowpass_restart": the
    learned hook with an all-zero network, i.e. the low-pass direction with the
    conjugation restarted at every CG iteration as the hook does; the trained
    weights are restored afterwards."""
    psi = ctx.gs_upload(psi_ref_layout)
    ctx.gram_schmidt_real(psi)
    ref = converge(ctx, psi, tol=1e-12, max_outer=3 * max_outer, precondition="lowpass", ncg=ncg)["evals"]
    out = {}
    for pre in ("lowpass", "learned", "none"):
        psi = ctx.gs_upload(psi_ref_layout)
        ctx.gram_schmidt_real(psi)
        r = converge(ctx, psi, tol=tol, max_outer=max_outer, precondition=pre, ncg=ncg, ref=ref)
        out[pre] = dict(outer=r["outer"], seconds=r["seconds"], converged=r["converged"],
                        max_err=float(np.max(np.abs(r["evals"] - ref))))
    if restart_batch is not None:
        params = get_params(ctx)
        init(ctx, restart_batch, None)
        psi = ctx.gs_upload(psi_ref_layout)
        ctx.gram_schmidt_real(psi)
        r = converge(ctx, psi, tol=tol, max_outer=max_outer, precondition="learned", ncg=ncg, ref=ref)
        out["lowpass_restart"] = dict(outer=r["outer"], seconds=r["seconds"], converged=r["converged"],
                                      max_err=float(np.max(np.abs(r["evals"] - ref))))
        init(ctx, restart_batch, params)
    return out
