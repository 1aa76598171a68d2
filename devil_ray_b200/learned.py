"""Learned initial guess for the Newton inversion (no reference counterpart).

A small MLP (the candidate hex element's control-point coordinates + the 3
point coordinates -> 128 -> 128 -> 3, GELU, BF16 weights, FP32
accumulation; 84 inputs at order 2, 195 at order 3) predicts the
reference-space coordinates of a point in the element.
It is trained on Newton solutions the method itself produces, by the
library's own tcgen05 forward/backward kernels (drb_mlp_train_step, Adam in
drb_mlp_adam), and used only as the first guess of the first candidate
element: plain Newton from the element centre remains the fallback whenever
the guessed solve does not converge.

Pipeline per batch of queries (LearnedLocator.locate):
  drb_query_order       Morton order of the queries (the points are then
                        gathered into that order, and the results scattered
                        back at the end)
  drb_first_candidates  first candidate leaf of every query (traversal only)
  drb_mlp_guess         fused tensor-core inference on (query, element) pairs
  drb_locate_hinted     persistent locate starting at the hinted candidate
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np
import torch

from . import _lib as L
from .api import BatchedLocator, UnstructuredMesh, _dev, _ptr, _stream

N_HID, N_OUT = 128, 3


class Layout:
    """Offsets of the network's parameters in its fp32 vector for order-P
    hex elements: W1 [128 x n_in], b1, W2 [128 x 128], b2, W3 [3 x 128], b3."""

    def __init__(self, order: int):
        self.order = order
        self.n_in = 3 * (order + 1) ** 3 + 3
        self.n_in_pad = (self.n_in + 15) // 16 * 16
        self.W1 = 0
        self.B1 = self.W1 + N_HID * self.n_in
        self.W2 = self.B1 + N_HID
        self.B2 = self.W2 + N_HID * N_HID
        self.W3 = self.B2 + N_HID
        self.B3 = self.W3 + N_OUT * N_HID
        self.n_params = self.B3 + N_OUT


# the order-2 network of the learned-guess workload
_L2 = Layout(2)
N_IN, N_IN_PAD = _L2.n_in, _L2.n_in_pad
W1, B1, W2, B2, W3, B3, N_PARAMS = _L2.W1, _L2.B1, _L2.W2, _L2.B2, _L2.W3, _L2.B3, _L2.n_params

_configured = False


def _lib():
    global _configured
    lib = L.lib()
    if not _configured:
        vp, ci, cf = C.c_void_p, C.c_int, C.c_float
        sig = {
            "drb_mlp_param_count": (ci, [ci]),
            "drb_mlp_bf16_count": (ci, [ci]),
            "drb_mlp_input_width": (ci, [ci]),
            "drb_mlp_workspace_bytes": (C.c_longlong, [ci, ci]),
            "drb_mlp_prepare": (ci, [ci, vp, vp, vp]),
            "drb_mlp_features": (ci, [C.POINTER(L.DrbMesh), vp, vp, ci, ci, vp, vp]),
            "drb_mlp_forward": (ci, [ci, vp, vp, vp, ci, ci, vp, vp, vp, vp]),
            "drb_mlp_train_step": (ci, [ci, vp, vp, vp, vp, vp, ci, ci, vp, vp, vp, vp, vp]),
            "drb_mlp_adam": (ci, [ci, vp, vp, vp, vp, cf, cf, cf, cf, ci, vp]),
            "drb_mlp_guess": (ci, [vp, vp, C.POINTER(L.DrbMesh), vp, vp, vp, ci, vp, vp, vp]),
            "drb_map_points": (ci, [C.POINTER(L.DrbMesh), vp, vp, ci, vp, vp]),
            "drb_newton_pairs": (ci, [C.POINTER(L.DrbMesh), vp, vp, ci, cf, ci, vp, vp, vp, vp,
                                      vp]),
            "drb_first_candidates": (ci, [C.POINTER(L.DrbBvh), vp, ci, vp, vp, vp, vp]),
            "drb_locate_hinted": (ci, [C.POINTER(L.DrbMesh), C.POINTER(L.DrbBvh), vp, ci, vp, vp,
                                       C.POINTER(L.DrbNewtonOpts), vp, vp, vp, L.DrbQueryStats,
                                       vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        _configured = True
    return lib


def map_points(mesh: UnstructuredMesh, elem: torch.Tensor, ref: torch.Tensor, stream=None):
    pts = torch.empty_like(ref)
    L.check(_lib().drb_map_points(C.byref(mesh.desc()), _ptr(elem), _ptr(ref), elem.numel(),
                                  _ptr(pts), _stream(stream)), "drb_map_points")
    return pts


def newton_pairs(mesh: UnstructuredMesh, elem, pts, tol=1e-5, max_steps=20, guess=None,
                 stream=None):
    n = elem.numel()
    ref = torch.empty((n, 3), dtype=torch.float32, device=mesh.device)
    found = torch.empty(n, dtype=torch.int32, device=mesh.device)
    iters = torch.empty(n, dtype=torch.int32, device=mesh.device)
    L.check(_lib().drb_newton_pairs(C.byref(mesh.desc()), _ptr(elem), _ptr(pts), n, tol,
                                    max_steps, _ptr(guess), _ptr(ref), _ptr(found), _ptr(iters),
                                    _stream(stream)), "drb_newton_pairs")
    return ref, found.bool(), iters


class GuessMLP:
    """Parameters (fp32 masters on the device) and the library calls."""

    def __init__(self, device="cuda", seed=0, order: int = 2):
        lib = _lib()
        self.order = order
        self.layout = lay = Layout(order)
        assert lib.drb_mlp_param_count(order) == lay.n_params
        assert lib.drb_mlp_input_width(order) == lay.n_in_pad
        self.device = torch.device(device)
        g = torch.Generator().manual_seed(seed)
        p = torch.zeros(lay.n_params, dtype=torch.float32)

        def init(off, fan_out, fan_in):
            bound = math.sqrt(6.0 / (fan_in + fan_out))
            p[off:off + fan_out * fan_in] = (torch.rand(fan_out * fan_in, generator=g) * 2 - 1) * bound

        init(lay.W1, N_HID, lay.n_in)
        init(lay.W2, N_HID, N_HID)
        init(lay.W3, N_OUT, N_HID)
        p[lay.B3:lay.B3 + 3] = 0.5  # centre of the reference element
        self.params = p.to(self.device)
        self.wbf16 = torch.empty(lib.drb_mlp_bf16_count(order), dtype=torch.bfloat16,
                                 device=self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.prepare()

    def prepare(self, stream=None):
        L.check(_lib().drb_mlp_prepare(self.order, _ptr(self.params), _ptr(self.wbf16),
                                       _stream(stream)), "drb_mlp_prepare")

    def check_err(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core kernel's bounded mbarrier wait ran out")

    @staticmethod
    def pad(n):
        return ((n + 127) // 128) * 128

    def features(self, mesh, elem, pts, n_pad=None, stream=None):
        n = elem.numel()
        n_pad = n_pad or self.pad(n)
        if mesh.order != self.order:
            raise ValueError(f"network of order {self.order}, mesh of order {mesh.order}")
        X = torch.empty((n_pad, self.layout.n_in_pad), dtype=torch.bfloat16, device=self.device)
        L.check(_lib().drb_mlp_features(C.byref(mesh.desc()), _ptr(elem), _ptr(pts), n, n_pad,
                                        _ptr(X), _stream(stream)), "drb_mlp_features")
        return X

    def workspace(self, n_pad):
        nb = _lib().drb_mlp_workspace_bytes(self.order, n_pad)
        return torch.empty(nb, dtype=torch.uint8, device=self.device)

    def forward(self, X, n, ws=None, stream=None):
        n_pad = X.shape[0]
        ws = ws if ws is not None else self.workspace(n_pad)
        y = torch.empty((max(n, 1), 3), dtype=torch.float32, device=self.device)
        L.check(_lib().drb_mlp_forward(self.order, _ptr(self.params), _ptr(self.wbf16), _ptr(X), n,
                                       n_pad,
                                       _ptr(y), _ptr(ws), _ptr(self.err), _stream(stream)),
                "drb_mlp_forward")
        return y[:n]

    def grad(self, X, target, n, weight=None, ws=None, stream=None):
        n_pad = X.shape[0]
        ws = ws if ws is not None else self.workspace(n_pad)
        g = torch.empty_like(self.params)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        L.check(_lib().drb_mlp_train_step(self.order, _ptr(self.params), _ptr(self.wbf16), _ptr(X),
                                          _ptr(target), _ptr(weight), n, n_pad, _ptr(g),
                                          _ptr(loss), _ptr(ws), _ptr(self.err), _stream(stream)),
                "drb_mlp_train_step")
        return g, loss

    def adam(self, g, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        L.check(_lib().drb_mlp_adam(self.order, _ptr(self.params), _ptr(g), _ptr(self.m),
                                    _ptr(self.v), lr,
                                    b1, b2, eps, self.step_count, _stream(stream)), "drb_mlp_adam")
        self.prepare(stream)

    def guess(self, mesh, elem, pts, order=None, stream=None):
        if mesh.order != self.order:
            raise ValueError(f"network of order {self.order}, mesh of order {mesh.order}")
        n = elem.numel()
        out = torch.empty((max(n, 1), 3), dtype=torch.float32, device=self.device)
        L.check(_lib().drb_mlp_guess(_ptr(self.params), _ptr(self.wbf16), C.byref(mesh.desc()),
                                     _ptr(elem), _ptr(pts), _ptr(order), n, _ptr(out),
                                     _ptr(self.err), _stream(stream)), "drb_mlp_guess")
        return out[:n]

    # -- checkpoint of weights and optimiser state --
    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy(), m=self.m.cpu().numpy(),
                 v=self.v.cpu().numpy(), step=self.step_count)

    def load(self, path):
        d = np.load(path)
        self.params.copy_(torch.as_tensor(d["params"]))
        self.m.copy_(torch.as_tensor(d["m"]))
        self.v.copy_(torch.as_tensor(d["v"]))
        self.step_count = int(d["step"])
        self.prepare()


def training_set(mesh: UnstructuredMesh, count: int, seed: int, tol=1e-5, max_steps=20):
    """(element, point, label, weight): uniform reference points in uniform
    elements mapped forward; labels are the method's own Newton solutions
    from the element centre; pairs whose solve fails get weight 0."""
    g = torch.Generator(device=mesh.device).manual_seed(seed)
    elem = torch.randint(0, mesh.n_elem, (count,), generator=g, device=mesh.device,
                         dtype=torch.int32)
    r = torch.rand((count, 3), generator=g, device=mesh.device)
    pts = map_points(mesh, elem, r)
    label, found, _ = newton_pairs(mesh, elem, pts, tol, max_steps)
    return elem, pts, label, found.float()


def train(model: GuessMLP, mesh: UnstructuredMesh, samples=1 << 22, batch=16384, epochs=2,
          lr=2e-3, seed=1, log=None):
    elem, pts, label, w = training_set(mesh, samples, seed)
    ws = model.workspace(batch)
    steps = 0
    losses = []
    gen = torch.Generator(device=mesh.device).manual_seed(seed + 1)
    for ep in range(epochs):
        perm = torch.randperm(samples, generator=gen, device=mesh.device)
        for b0 in range(0, samples - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            e, p, t, ww = elem[idx].contiguous(), pts[idx].contiguous(), label[idx].contiguous(), \
                w[idx].contiguous()
            X = model.features(mesh, e, p, batch)
            frac = steps / max(1, epochs * (samples // batch))
            g, loss = model.grad(X, t, batch, ww, ws)
            model.adam(g, lr=lr * 0.5 * (1 + math.cos(math.pi * frac)))
            steps += 1
            if steps == 1 or steps % 50 == 0:
                losses.append(float(loss.item()))
                if log:
                    log(f"step {steps} loss {losses[-1]:.3e}")
    model.check_err()
    return losses


class LearnedLocator:
    """Batched point location with the learned first guess.

    bvh: None for the mesh's own BVH.  A BVH with grid lists
    (BVH.build_grid) takes the first candidates from the query's cell and
    solves through drb_locate_batched with the given guesses; otherwise the
    hinted locate resumes the tree walk after the first candidate.  Both
    equal drb_locate with DRB_GUESS_GIVEN."""

    def __init__(self, mesh: UnstructuredMesh, model: GuessMLP, tol=1e-5, max_steps=20,
                 config: L.DrbLocateConfig | None = None, bvh=None):
        self.mesh, self.model = mesh, model
        self.tol, self.max_steps = tol, max_steps
        self.config = config
        self.bvh = bvh
        self._order = BatchedLocator(mesh, tol, max_steps)

    def locate(self, points, order=None, stats=False, out=None, stream=None):
        pts = _dev(points, torch.float32, self.mesh.device).reshape(-1, 3)
        n = pts.shape[0]
        dev = self.mesh.device
        bvh = self.bvh if self.bvh is not None else self.mesh.get_bvh()
        if order is None:
            order = self._order.order(pts, stream)
        # Work on a Morton-ordered copy of the points: the first-candidate
        # traversal, the guess network and the hinted locate then read and
        # write contiguous arrays, and one scatter puts the results back in
        # input order (each query's result does not depend on the order).
        ol = order.long()
        pts_s = pts.index_select(0, ol)
        first_leaf = torch.empty(n, dtype=torch.int32, device=dev)
        first_elem = torch.empty(n, dtype=torch.int32, device=dev)
        L.check(_lib().drb_first_candidates(C.byref(bvh.desc()), _ptr(pts_s), n, None,
                                            _ptr(first_leaf), _ptr(first_elem), _stream(stream)),
                "drb_first_candidates")
        guess = self.model.guess(self.mesh, first_elem, pts_s, None, stream)
        if out is None:
            cell = torch.empty(n, dtype=torch.int32, device=dev)
            ref = torch.empty((n, 3), dtype=torch.float32, device=dev)
        else:
            cell, ref = out
        cell_s = torch.empty(n, dtype=torch.int32, device=dev)
        ref_s = torch.empty((n, 3), dtype=torch.float32, device=dev)
        st = [torch.empty(n, dtype=torch.int32, device=dev) for _ in range(3)] if stats else None
        qs = L.DrbQueryStats(*(t.data_ptr() for t in st)) if stats else L.DrbQueryStats()
        opts = L.DrbNewtonOpts(self.tol, self.max_steps, L.GUESS_GIVEN, guess.data_ptr())
        if bvh.grid_start is not None:
            # the points are in Morton order already: solve them in index order
            cfg = L.DrbLocateConfig(128, 0, 64, 1, 0) if self.config is None else \
                L.DrbLocateConfig(*(getattr(self.config, f) for f, _ in L.DrbLocateConfig._fields_))
            cfg.sort_queries = 0
            bd = bvh.desc()
            L.check(_lib().drb_locate_batched(C.byref(self.mesh.desc()), C.byref(bd), _ptr(pts_s),
                                              n, C.byref(opts), C.byref(cfg), _ptr(cell_s),
                                              _ptr(ref_s), qs, _stream(stream)),
                    "drb_locate_batched")
        else:
            cfg = None if self.config is None else C.byref(self.config)
            L.check(_lib().drb_locate_hinted(C.byref(self.mesh.desc()), C.byref(bvh.desc()),
                                             _ptr(pts_s), n, None, _ptr(first_leaf),
                                             C.byref(opts), cfg, _ptr(cell_s), _ptr(ref_s), qs,
                                             _stream(stream)), "drb_locate_hinted")
        cell.index_copy_(0, ol, cell_s)
        ref.index_copy_(0, ol, ref_s)
        if stats:
            st = [torch.empty_like(t).index_copy_(0, ol, t) for t in st]
            return cell, ref, st[0], st[1], st[2]
        return cell, ref
