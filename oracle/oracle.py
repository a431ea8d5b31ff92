"""ctypes front end of the CPU oracle (oracle/nps_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, always as the checker.  The product library
(nprush_b200) never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libnps_oracle.so"
SOURCES = [HERE / "nps_oracle.cpp", HERE / "nps_oracle_gs.cpp", HERE / "nps_oracle_mlp.cpp"]
HEADERS = [HERE / "gs_model.h"]


def build(force: bool = False) -> Path:
    newest = max(s.stat().st_mtime for s in SOURCES + HEADERS if s.exists())
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest:
        return LIB
    tmp = f"{LIB}.{os.getpid()}.tmp"  # concurrent builders each write their own file
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
           "-shared", "-o", tmp] + [str(s) for s in SOURCES if s.exists()]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr[-4000:])
    os.replace(tmp, LIB)
    return LIB


_lib = None
F = ctypes.POINTER(ctypes.c_float)
I = ctypes.POINTER(ctypes.c_int32)
U = ctypes.POINTER(ctypes.c_uint32)
D = ctypes.POINTER(ctypes.c_double)


def lib():
    global _lib
    if _lib is None:
        build()  # no-op unless a source or header is newer than the library
        _lib = ctypes.CDLL(str(LIB))
    return _lib


def _p(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------- compat splats
def splat_backward(splats, vp, vpinv, tgt_rgba, tgt_depth, grads_q=None, want_float=True, want_image=True,
                   terms=None):
    """One view of splat_backward.wgsl. Returns dict(grads_q, grads_f, image, tile_count, terms): terms[i]
    counts the (pixel, splat) backward terms (alpha >= 0.001) splat i's gradient sums (added to `terms`
    when given)."""
    splats = _f32(splats)
    n = splats.shape[0]
    h, w = tgt_depth.shape
    gq = np.zeros((n, 16), np.int32) if grads_q is None else grads_q
    gf = np.zeros((n, 16), np.float32) if want_float else None
    img = np.zeros((h, w, 4), np.float32) if want_image else None
    tc = np.zeros(((h + 15) // 16, (w + 15) // 16), np.uint32)
    tm = np.zeros(n, np.uint32) if terms is None else terms
    lib().orc_splat_backward(_p(splats, F), n, _p(_f32(vp), F), _p(_f32(vpinv), F), _p(_f32(tgt_rgba), F),
                             _p(_f32(tgt_depth), F), w, h, _p(gq, I), _p(gf, F), _p(img, F), _p(tc, U), _p(tm, U))
    return dict(grads_q=gq, grads_f=gf, image=img, tile_count=tc, terms=tm)


def splat_step(splats, grads, m, v, adam_t, grad_accum):
    """In place: splats, grads (zeroed), m, v, grad_accum. Returns new t."""
    t = np.array([adam_t], np.float32)
    lib().orc_splat_step(_p(splats, F), _p(grads, I), _p(m, F), _p(v, F), _p(t, F), _p(grad_accum, F),
                         splats.shape[0])
    return float(t[0])


def splat_adc(splats, m, v, adam_t, grad_accum):
    lib().orc_splat_adc(_p(splats, F), _p(m, F), _p(v, F), ctypes.c_float(adam_t), _p(grad_accum, F),
                        splats.shape[0])


# ------------------------------------------------------------ compat beziers
def bezier_backward(beziers, vp, uni, tgt_rgba, tgt_depth, bg_rgba, bg_depth, normal_rgba,
                    grads_q=None, loss_accum=None, pixel_loss=None, want_float=True, want_image=True, terms=None):
    beziers = _f32(beziers)
    n = beziers.shape[0]
    h, w = tgt_depth.shape
    gq = np.zeros((n, 18), np.int32) if grads_q is None else grads_q
    gf = np.zeros((n, 18), np.float32) if want_float else None
    la = np.zeros(n, np.float32) if loss_accum is None else loss_accum
    pl = np.zeros(512 * 512, np.int32) if pixel_loss is None else pixel_loss
    img = np.zeros((h, w, 4), np.float32) if want_image else None
    tc = np.zeros(((h + 15) // 16, (w + 15) // 16), np.uint32)
    tm = np.zeros(n, np.uint32) if terms is None else terms
    lib().orc_bezier_backward(_p(beziers, F), n, _p(_f32(vp), F), _p(_f32(uni), F), _p(_f32(tgt_rgba), F),
                              _p(_f32(tgt_depth), F), _p(_f32(bg_rgba), F), _p(_f32(bg_depth), F),
                              _p(_f32(normal_rgba), F), w, h, _p(gq, I), _p(gf, F), _p(la, F), _p(pl, I),
                              _p(img, F), _p(tc, U), _p(tm, U))
    return dict(grads_q=gq, grads_f=gf, loss_accum=la, pixel_loss=pl, image=img, tile_count=tc, terms=tm)


def bezier_step(beziers, grads, m, v, adam_t, pixel_count, no_kill, grad_accum, vp, uni):
    t = np.array([adam_t], np.float32)
    lib().orc_bezier_step(_p(beziers, F), _p(grads, I), _p(m, F), _p(v, F), _p(t, F), ctypes.c_float(pixel_count),
                          ctypes.c_float(no_kill), _p(grad_accum, F), _p(_f32(vp), F), _p(_f32(uni), F),
                          beziers.shape[0])
    return float(t[0])


def bezier_adc(beziers, m, v, adam_t, no_kill, grad_accum, loss_accum, pixel_loss, vp, vpinv):
    lib().orc_bezier_adc(_p(beziers, F), _p(m, F), _p(v, F), ctypes.c_float(adam_t), ctypes.c_float(no_kill),
                         _p(grad_accum, F), _p(loss_accum, F), _p(pixel_loss, I), _p(_f32(vp), F),
                         _p(_f32(vpinv), F), beziers.shape[0])


# ------------------------------------------------------------- Gaussians
def _setup_gs():
    L = lib()
    L.orc_gs_loss_f64.restype = ctypes.c_double
    return L


def gs_forward(params, deg, views48, w, h, bg=(0.0, 0.0, 0.0)):
    params = _f32(params)
    views48 = _f32(views48)
    nv = views48.shape[0]
    img = np.zeros((nv, h, w, 4), np.float32)
    nc = np.zeros((nv, h, w), np.uint32)
    bgv = _f32(bg)
    lib().orc_gs_forward(_p(params, F), params.shape[0], deg, _p(views48, F), nv, w, h, _p(bgv, F), _p(img, F),
                         _p(nc, U))
    return img, nc


LOSS_KINDS = {"l1_dssim": 0, "l1": 1, "l2": 2}


def gs_loss(img, targets, tids, lam=0.2, loss="l1_dssim"):
    """fp32 loss and dL/dimage.  loss: "l1_dssim" ((1 - lam) L1 + lam D-SSIM;
    l3 = loss, mean L1, mean SSIM), "l1" or "l2" (l3 = loss, mean L1, mean
    squared error)."""
    img = _f32(img)
    nv, h, w, _ = img.shape
    targets = _f32(targets)
    tids = np.ascontiguousarray(tids, np.uint32)
    l3 = np.zeros(3, np.float32)
    dimg = np.zeros_like(img)
    lib().orc_gs_loss(_p(img, F), _p(targets, F), _p(tids, U), nv, w, h, ctypes.c_float(lam), LOSS_KINDS[loss],
                      _p(l3, F), _p(dimg, F))
    return l3, dimg


def gs_backward(params, deg, views48, w, h, img, ncontrib, dimg, bg=(0.0, 0.0, 0.0), with_adc=False):
    """Parameter gradients; with_adc also returns the ADC statistic
    (n x 2: summed NDC-space view-loss gradient norms, views seen)."""
    params = _f32(params)
    views48 = _f32(views48)
    grads = np.zeros_like(params)
    bgv = _f32(bg)
    adc2 = np.zeros((params.shape[0], 2), np.float32)
    lib().orc_gs_backward(_p(params, F), params.shape[0], deg, _p(views48, F), views48.shape[0], w, h, _p(bgv, F),
                          _p(_f32(img), F), _p(np.ascontiguousarray(ncontrib, np.uint32), U), _p(_f32(dimg), F),
                          _p(grads, F), _p(adc2, F), ctypes.c_float(views48.shape[0]))
    return (grads, adc2) if with_adc else grads


def gs_adam(params, grads, m, v, step, lr6):
    lr = _f32(lr6)
    lib().orc_gs_adam(_p(params, F), _p(_f32(grads), F), _p(m, F), _p(v, F), params.shape[0], step, _p(lr, F))


def gs_adc(params, m, v, adc_grad, adc_denom, cap, seed, thresh=2e-4, split_scale=0.01, prune_op=0.005):
    """Plain threshold ADC; returns (params, m, v, counts[before, after, densified, pruned])."""
    params, m, v = _f32(params), _f32(m), _f32(v)
    n = params.shape[0]
    op, om, ov = (np.zeros((cap, params.shape[1]), np.float32) for _ in range(3))
    c = np.zeros(4, np.uint32)
    lib().orc_gs_adc(_p(params, F), _p(m, F), _p(v, F), _p(_f32(adc_grad), F), _p(_f32(adc_denom), F), n, cap,
                     ctypes.c_float(thresh), ctypes.c_float(split_scale), ctypes.c_float(prune_op), seed, _p(op, F),
                     _p(om, F), _p(ov, F), _p(c, U))
    k = int(c[1])
    return op[:k], om[:k], ov[:k], c


def gs_loss_f64(params, deg, views48, w, h, targets, tids, lam=0.2, bg=(0.0, 0.0, 0.0), loss="l1_dssim"):
    L = _setup_gs()
    params = _f32(params)
    views48 = _f32(views48)
    tids = np.ascontiguousarray(tids, np.uint32)
    return L.orc_gs_loss_f64(_p(params, F), params.shape[0], deg, _p(views48, F), views48.shape[0], w, h,
                             _p(_f32(bg), F), _p(_f32(targets), F), _p(tids, U), ctypes.c_double(lam),
                             LOSS_KINDS[loss])


def gs_loss_cd(params, deg, views48, w, h, targets, tids, pidx, h_rel=1e-4, lam=0.2, bg=(0.0, 0.0, 0.0),
               loss="l1_dssim"):
    """FP64 central differences of the loss w.r.t. flat parameter indices."""
    params = _f32(params)
    views48 = _f32(views48)
    tids = np.ascontiguousarray(tids, np.uint32)
    pidx = np.ascontiguousarray(pidx, np.uint32)
    out = np.zeros(len(pidx), np.float64)
    lib().orc_gs_loss_cd(_p(params, F), params.shape[0], deg, _p(views48, F), views48.shape[0], w, h,
                         _p(_f32(bg), F), _p(_f32(targets), F), _p(tids, U), ctypes.c_double(lam), LOSS_KINDS[loss],
                         _p(pidx, U), len(pidx), ctypes.c_double(h_rel), _p(out, D))
    return out


def gs_sh(dirs):
    """FP64 degree-3 SH basis and its x / y / z partials at dirs (n x 3): four n x 16 arrays."""
    dirs = np.ascontiguousarray(dirs, np.float64).reshape(-1, 3)
    out = [np.zeros((len(dirs), 16), np.float64) for _ in range(4)]
    lib().orc_gs_sh(_p(dirs, D), len(dirs), *(_p(o, D) for o in out))
    return out


def gs_rot(q, G):
    """FP64 rotation matrix of the unit quaternion q and dq = sum G * dR/dq."""
    q = np.ascontiguousarray(q, np.float64)
    G = np.ascontiguousarray(G, np.float64).reshape(9)
    R, dq = np.zeros(9, np.float64), np.zeros(4, np.float64)
    lib().orc_gs_rot(_p(q, D), _p(G, D), _p(R, D), _p(dq, D))
    return R.reshape(3, 3), dq


# ------------------------------------------------------------ display forwards
def splat_render(splats, vp, w, h):
    splats = _f32(splats)
    rgba = np.zeros((h, w, 4), np.float32)
    dep = np.zeros((h, w, 4), np.float32)
    lib().orc_splat_render(_p(splats, F), splats.shape[0], _p(_f32(vp), F), w, h, _p(rgba, F), _p(dep, F))
    return rgba, dep


def splat_render_blend(splats, vp, w, h, rgba, depth=None):
    """The splat forward pass blended fragment by fragment in draw order over
    the given starting images (H x W x 4, copied); returns (rgba, depth)."""
    splats = _f32(splats)
    rgba = np.array(rgba, np.float32, copy=True, order="C")
    dep = None if depth is None else np.array(depth, np.float32, copy=True, order="C")
    lib().orc_splat_render_blend(_p(splats, F), splats.shape[0], _p(_f32(vp), F), w, h, _p(rgba, F), _p(dep, F))
    return rgba, dep


def bezier_render(beziers, vp, w, h, bg=None, brush=None):
    beziers = _f32(beziers)
    bg = np.zeros((h, w, 4), np.float32) if bg is None else _f32(bg)
    out = np.zeros((h, w, 4), np.float32)
    bb = None if brush is None else _f32(brush)
    bh, bw = (0, 0) if brush is None else brush.shape
    lib().orc_bezier_render(_p(beziers, F), beziers.shape[0], _p(_f32(vp), F), w, h, _p(bg, F), _p(bb, F), bw, bh,
                            _p(out, F))
    return out


# ------------------------------------------------------------ learned-ADC MLP
def mlp_grads(params, X, labels, class_w=(1.0, 1.0, 1.0, 1.0), round_bf16=True):
    """(grads, mean loss, logits [n, 3]) of the policy network on one batch."""
    L = lib()
    params, X = _f32(params), _f32(X)
    n = X.shape[0]
    g = np.zeros(L.orc_mlp_num_params(), np.float32)
    loss = np.zeros(1, np.float32)
    logits = np.zeros((n, 3), np.float32)
    lab = None if labels is None else np.ascontiguousarray(labels, np.uint8)
    L.orc_mlp_grads(_p(params, F), _p(X, F), None if lab is None else lab.ctypes.data, n, _p(_f32(class_w), F),
                    int(round_bf16), _p(g, F), _p(loss, F), _p(logits, F))
    return g, float(loss[0]), logits


def mlp_loss_f64(params, X, labels, class_w=(1.0, 1.0, 1.0, 1.0), with_grads=False):
    L = lib()
    L.orc_mlp_loss_f64.restype = ctypes.c_double
    params, X = _f32(params), _f32(X)
    lab = np.ascontiguousarray(labels, np.uint8)
    g = np.zeros(L.orc_mlp_num_params(), np.float64)
    loss = L.orc_mlp_loss_f64(_p(params, F), _p(X, F), lab.ctypes.data, X.shape[0], _p(_f32(class_w), F),
                              _p(g, D) if with_grads else None)
    return (loss, g) if with_grads else loss
