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
    """With zero weights the learned preconditioner is the low-pass one."""
    from salmon2_b200 import _lib, synth
    from salmon2_b200.rt import Context
    from oracle import Oracle

    s = synth.isolated_system(num=20, no=4, natom=2, seed=52, real=True, name="net20")
    O = Oracle(s)
    psi0 = O.gram_schmidt_real(s.psi)
    ctx = Context(s)
    _lib.check(_lib.lib().sb200_learned_init(ctx.h, None, _lib.LEARNED_NPARAM, 4))
    a = ctx.gs_upload(psi0)
    esp_l = ctx.gscg(a, ncg=3, precondition="learned")
    b = ctx.gs_upload(psi0)
    esp_p = ctx.gscg(b, ncg=3, precondition="lowpass")
    np.testing.assert_allclose(esp_l, esp_p, rtol=1e-12, atol=1e-14)
