"""Learned preconditioner: the forward pass and the loss gradients of the
hand-written GPU kernels against a float64 numpy restatement of the same
network on a tiny grid (weights rounded to BF16 on both sides)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NCH = 16
K3 = 27


def bf16_round(a):
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def unpack(params):
    o = 0
    sizes = [(NCH, 2, K3), (NCH,), (NCH, NCH, K3), (NCH,), (1, NCH, K3), (1,)]
    out = []
    for sh in sizes:
        n = int(np.prod(sh))
        out.append(params[o:o + n].reshape(sh))
        o += n
    return out


def conv(x, W, b, shape):
    """x: (cin, n) -> (cout, n); 3x3x3, zero padding; grid index x fastest."""
    nx, ny, nz = shape
    cin = x.shape[0]
    cout = W.shape[0]
    xg = x.reshape(cin, nz, ny, nx)
    pad = np.zeros((cin, nz + 2, ny + 2, nx + 2))
    pad[:, 1:-1, 1:-1, 1:-1] = xg
    out = np.zeros((cout, nz, ny, nx))
    for k in range(K3):
        dx, dy, dz = k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1
        sl = pad[:, 1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx]
        out += np.einsum("oc,czyx->ozyx", W[:, :, k], sl)
    out += b[:, None, None, None]
    return out.reshape(cout, -1)


def forward(params, x0, shape):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    a1 = conv(x0, W1, b1, shape)
    x1 = np.maximum(a1, 0)
    a2 = conv(x1, W2, b2, shape)
    x2 = np.maximum(a2, 0)
    return conv(x2, W3, b3, shape)[0]


def loss(params, x0s, offs, ts, shape):
    L = 0.0
    for x0, off, t in zip(x0s, offs, ts):
        y = forward(params, x0, shape) + off
        L += 1.0 - np.dot(y, t) ** 2 / (np.dot(y, y) * np.dot(t, t))
    return L


def test_forward_and_gradients_match_numpy():
    import torch
    from salmon2_b200 import _lib, synth
    from salmon2_b200.rt import Context

    s = synth.isolated_system(num=8, no=1, natom=1, seed=51, real=True, name="net8")
    ctx = Context(s)
    shape = s.grid.shape
    n = int(np.prod(shape))
    rng = np.random.default_rng(3)
    params = bf16_round(rng.normal(0, 0.15, _lib.LEARNED_NPARAM)).astype(np.float64)
    # biases are FP32 in both implementations; keep them small
    B = 2
    x0 = rng.normal(size=(B, 2, n)).astype(np.float32)
    t = rng.normal(size=(B, n)).astype(np.float32)
    off = rng.normal(size=(B, n)).astype(np.float32)
    p32 = np.ascontiguousarray(params, dtype=np.float32)
    L = _lib.lib()
    _lib.check(L.sb200_learned_init(ctx.h, C.c_void_p(p32.ctypes.data), _lib.LEARNED_NPARAM, B))
    y = np.zeros((B, n), np.float32)
    _lib.check(L.sb200_learned_forward(ctx.h, C.c_void_p(x0.ctypes.data), C.c_void_p(y.ctypes.data), B))
    for b in range(B):
        ref = forward(params, x0[b].astype(np.float64), shape)
        assert np.max(np.abs(y[b] - ref)) <= 1e-4 * np.max(np.abs(ref))
    lval = C.c_double(0)
    g = np.zeros(_lib.LEARNED_NPARAM, np.float32)
    _lib.check(L.sb200_learned_loss_grad(ctx.h, C.c_void_p(x0.ctypes.data), C.c_void_p(off.ctypes.data),
                                         C.c_void_p(t.ctypes.data), B, C.byref(lval), C.c_void_p(g.ctypes.data)))
    X, O, T = x0.astype(np.float64), off.astype(np.float64), t.astype(np.float64)
    lref = loss(params, X, O, T, shape)
    assert abs(lval.value - lref) <= 1e-5 * abs(lref)
    # central differences on a sample of parameters of every layer
    sel = list(range(0, 864, 97)) + [864 + 3] + list(range(880, 7792, 811)) + [7792 + 5] + list(range(7808, 8240, 61)) + [8240]
    h = 1e-3
    for i in sel:
        pp, pm = params.copy(), params.copy()
        pp[i] += h
        pm[i] -= h
        fd = (loss(pp, X, O, T, shape) - loss(pm, X, O, T, shape)) / (2 * h)
        assert abs(g[i] - fd) <= 2e-3 * max(1.0, abs(fd)) + 1e-3, (i, g[i], fd)
    ctx.close()


def test_untrained_network_is_lowpass_cg():
    """With zero weights the learned preconditioner is the low-pass one (one CG
    iteration: with the network the conjugation restarts every iteration)."""
    from salmon2_b200 import _lib, synth
    from salmon2_b200.rt import Context
    from oracle import Oracle

    s = synth.isolated_system(num=20, no=4, natom=2, seed=52, real=True, name="net20")
    O = Oracle(s)
    psi0 = O.gram_schmidt_real(s.psi)
    ctx = Context(s)
    _lib.check(_lib.lib().sb200_learned_init(ctx.h, None, _lib.LEARNED_NPARAM, 4))
    a = ctx.gs_upload(psi0)
    esp_l = ctx.gscg(a, ncg=1, precondition="learned")
    b = ctx.gs_upload(psi0)
    esp_p = ctx.gscg(b, ncg=1, precondition="lowpass")
    np.testing.assert_allclose(esp_l, esp_p, rtol=1e-12, atol=1e-14)


def test_learned_cg_iteration_matches_torch_restatement():
    """One CG iteration with the network direction (hook inside sb200_gscg)
    against the same iteration written out with torch: g = Hx - eps x, the
    network input [g/rms(g), V], p = lowpass(g) + rms(g) y with the sign rule,
    the direction orthogonalised to x and normalised, the 2x2 Rayleigh-Ritz."""
    import torch
    from salmon2_b200 import _lib, learned, synth
    from salmon2_b200.rt import Context
    from oracle import Oracle

    s = synth.isolated_system(num=(14, 12, 16), no=3, natom=2, seed=53, real=True, name="net_cg")
    psi0 = Oracle(s).gram_schmidt_real(s.psi)
    ctx = Context(s)
    params = learned.initial_params(7)
    rng = np.random.default_rng(9)
    i3 = params.size - 1 - 16 * 27
    params[i3:-1] = rng.normal(0, 0.2, 16 * 27).astype(np.float32)  # a non-zero output layer
    learned.init(ctx, batch=s.no, params=params)
    a = ctx.gs_upload(psi0)
    ctx.gscg(a, ncg=1, precondition="learned")
    got = ctx.gs_download(a)

    hv = s.grid.hvol
    x = ctx.gs_upload(psi0).reshape(s.no, -1)
    h = ctx.gs_empty()
    ctx.hpsi_real(x.reshape(ctx.gs_empty().shape), h)
    hx = h.reshape(s.no, -1)
    eps = (x * hx).sum(1, keepdim=True) * hv
    g = hx - eps * x
    rms = torch.sqrt((g * g).mean(1, keepdim=True))
    V = torch.from_numpy(np.ascontiguousarray(s.V_local[..., 0].ravel(order="F"))).to(g)
    x0 = torch.stack([g / rms, V.expand_as(g)], dim=1).float().contiguous()
    y = torch.empty((s.no, g.shape[1]), dtype=torch.float32, device=g.device)
    _lib.check(_lib.lib().sb200_learned_forward(ctx.h, C.c_void_p(x0.data_ptr()), C.c_void_p(y.data_ptr()), s.no))
    torch.cuda.synchronize()
    lp = learned._lowpass(torch, g, s.grid.shape, s.grid.hgs)
    corr = rms * y.double()
    corr = corr - (corr @ x.T * hv) @ x  # components along the current orbitals removed
    d0 = (lp * g).sum(1, keepdim=True)
    D = d0 + (corr * g).sum(1, keepdim=True)
    sign = torch.where(D >= 0.2 * d0, 1.0, torch.where(D <= -0.2 * d0, -1.0, 0.0))
    pre = torch.where(sign == 0, lp, sign * (lp + corr))
    zs = (x * pre).sum(1, keepdim=True) * hv
    pko = pre - zs * x
    pko = pko / torch.sqrt((pko * pko).sum(1, keepdim=True) * hv)
    ctx.hpsi_real(pko.reshape(ctx.gs_empty().shape).contiguous(), h)
    hw = h.reshape(s.no, -1)
    xhx = eps
    xhp = (x * hw).sum(1, keepdim=True) * hv
    php = (pko * hw).sum(1, keepdim=True) * hv
    ev = 0.5 * ((xhx + php) - torch.sqrt((xhx - php) ** 2 + 4.0 * xhp.abs() ** 2))
    cx = xhp / (ev - xhx)
    cp = 1.0 / torch.sqrt(1.0 + cx.abs() ** 2)
    cx = cx * cp
    xn = cx * x + cp * pko
    xn = xn / torch.sqrt((xn * xn).sum(1, keepdim=True) * hv)
    want = ctx.gs_download(xn.reshape(ctx.gs_empty().shape).contiguous())
    # the network input and its scale rms(g) pass through FP32 in the library
    err = np.max(np.abs(got - want)) / np.max(np.abs(want))
    assert err < 1e-7, err


def test_trained_network_gain_is_measured():
    """Train on residual -> correction pairs of plain low-pass CG runs on two
    seeded systems, then measure on a held-out system: the network's direction
    is better aligned with the target than the low-pass one (held-out loss),
    and the CG with it is timed against the plain CG on the same system.  The
    learned CG must still reach the plain CG's eigenvalues (1e-8 Ha); the
    iteration counts and times are printed, not asserted in its favour, next
    to the low-pass CG restarted at every iteration (the hook's conjugation
    without a network), which separates the network's effect from the cost of
    the restart."""
    import torch
    from salmon2_b200 import learned, synth
    from salmon2_b200.rt import Context

    X, O, T = [], [], []
    for seed in (61, 62):
        s = synth.isolated_system(num=20, no=6, natom=2, seed=seed, real=True, h_aa=0.3)
        c = Context(s)
        psi = c.gs_upload(s.psi)
        c.gram_schmidt_real(psi)
        x0, off, tgt = learned.collect_samples(c, psi, n_outer=8)
        X.append(x0); O.append(off); T.append(tgt)
        c.close()
    x0, off, tgt = torch.cat(X), torch.cat(O), torch.cat(T)
    s = synth.isolated_system(num=20, no=6, natom=2, seed=63, real=True, h_aa=0.3)
    c = Context(s)
    learned.init(c, batch=8, params=learned.initial_params(0))
    learned.train(c, x0, off, tgt, steps=600, batch=8, lr=2e-3)
    params = learned.get_params(c)
    psi = c.gs_upload(s.psi)
    c.gram_schmidt_real(psi)
    xh, oh, th = learned.collect_samples(c, psi, n_outer=8)
    learned.init(c, batch=8, params=np.zeros_like(params))
    loss_lowpass = learned.eval_loss(c, xh, oh, th)
    learned.init(c, batch=8, params=params)
    loss_trained = learned.eval_loss(c, xh, oh, th)
    assert loss_trained < loss_lowpass, (loss_trained, loss_lowpass)
    learned.init(c, batch=s.no, params=params)
    res = learned.evaluate(c, s.psi, tol=1e-8, max_outer=1200, restart_batch=s.no)
    print("held-out loss: low-pass direction %.3f, trained %.3f" % (loss_lowpass, loss_trained))
    print("CG to 1e-8 Ha:", {k: (v["outer"], round(v["seconds"], 3)) for k, v in res.items()})
    assert res["lowpass"]["converged"] and res["learned"]["converged"], res
