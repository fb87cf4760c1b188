"""Learned right preconditioner for flexible GMRES: training data, training
and evaluation on the GPU.

The network (a message-passing net over the octree's leaf boxes, 3 layers of
width 64, bfloat16 weights, gains predicted from static geometric and
material features) corrects the near-field preconditioner's output
z = P_near v by a fixed linear map per body, y = (I + L) z; its forward
pass, backward pass and Adam step are the library's own CUDA kernels
(``mlfma_lp_*`` in include/mlfma_pmchwt.h). This module only moves data: it
builds (v, z) pairs, loops over them, and evaluates the result. PyTorch
provides the device buffers.

Pairs:
  random_directions  v complex white noise (with the residual loss
                     |A M v - v|^2 this is the Frobenius-norm objective of a
                     sparse approximate inverse; the default);
  krylov_directions  the first flexible GMRES cycle's basis vectors;
  harvest            residual / error pairs from the method's own solves:
                     x* = an FGMRES solve to a tight tolerance, x_0 = 0,
                     x_(k+1) = x_k + one short FGMRES cycle; per iterate
                     v = r / |r|, e = (x* - x_k) / |r|, z = P_near v.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import MLFMM, lp_adam_device, lp_param_count, plane_wave

# parameter blocks in storage order (the layout of include/mlfma_pmchwt.h)
_F, _H, _NG, _LAYERS = 16, 64, 32, 3


def layout():
    out = [("We", (_H, _F)), ("be", (_H,))]
    for l in range(_LAYERS):
        out += [(f"Ws{l}", (_H, _H)), (f"Wn{l}", (_H, _H)), (f"Wg{l}", (_H, _H)), (f"c{l}", (_H,))]
    out += [("Wd1", (_H, 2 * _H)), ("d1", (_H,)), ("Wd2", (_NG, _H)), ("d2", (_NG,))]
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-scaled weights (halved in the message-passing layers), zero biases
    and a zero output layer: the untrained network returns y = z."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in layout():
        if len(shape) == 1 or name == "Wd2":
            parts.append(np.zeros(shape))
        else:
            mp = name.startswith(("Ws", "Wn", "Wg"))
            fan_in = shape[1] * (2 if mp else 1)
            parts.append(rng.normal(0.0, math.sqrt(2.0 / fan_in) * (0.5 if mp else 1.0), size=shape))
    theta = np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)
    assert theta.size == lp_param_count()
    return theta


def incidences(count: int, phi_deg: float = 0.0):
    """count plane waves with theta uniformly spaced over 0-180 deg and
    alternating theta / phi polarisation (pol 0 / 90)."""
    out = []
    for j in range(count):
        th = 180.0 * j / max(count - 1, 1)
        out.append(plane_wave(90.0 * (j % 2), th, phi_deg))
    return out


def harvest(op: MLFMM, rhs_rows, inner_its: int = 8, cycle: int = 3, tol: float = 1e-3, tight: float = 1e-7,
            max_cycles: int = 12):
    """(v, z, e) triples on the device (torch complex128 [k, 2N] each) from
    the FGMRES solves of the given right-hand sides."""
    import torch
    vs, es = [], []
    for b in rhs_rows:
        b = np.asarray(b, dtype=np.complex128)
        xs, st = op.matrix_solver(b, tol_rel=tight, tol_abs=0.0, mr=50, itr_max=600, inner_its=inner_its)
        bn = np.linalg.norm(b)
        x = np.zeros_like(b)
        for _ in range(max_cycles + 1):
            r = b - op.apply_ax(x)
            rn = np.linalg.norm(r)
            vs.append(r / rn)
            es.append((xs - x) / rn)
            if rn < tol * bn:
                break
            x, _ = op.matrix_solver(b, x0=x, itr_max=cycle, mr=cycle, tol_rel=tol, tol_abs=0.0, inner_its=inner_its)
    dev = torch.device("cuda", op.device)
    V = torch.from_numpy(np.stack(vs)).to(dev)
    E = torch.from_numpy(np.stack(es)).to(dev)
    Z = torch.empty_like(V)
    torch.cuda.synchronize(dev)  # the plan's stream reads V next
    for k in range(V.shape[0]):
        op.near_precondition_device(inner_its, V[k].data_ptr(), Z[k].data_ptr())
    return dict(v=V, z=Z, e=E)


def krylov_directions(op: MLFMM, rhs_rows, inner_its: int = 8, steps: int = 24):
    """(v, z) pairs on the device: the basis vectors of the first flexible
    GMRES cycle of each right-hand side, v_1 = b / |b|, v_(j+1) = A z_j
    orthonormalised against v_1..v_j (two Gram-Schmidt passes), z_j = P_near v_j
    -- the inputs the preconditioner meets inside the solve."""
    import torch
    dev = torch.device("cuda", op.device)
    ts = torch.cuda.Stream(dev)
    ts.wait_stream(torch.cuda.current_stream(dev))
    vs, zs = [], []
    with torch.cuda.stream(ts):
        for b in rhs_rows:
            Vb = torch.empty((steps, op.n), dtype=torch.complex128, device=dev)
            Zb = torch.empty_like(Vb)
            w = torch.empty(op.n, dtype=torch.complex128, device=dev)
            bt = torch.from_numpy(np.asarray(b, dtype=np.complex128)).to(dev)
            Vb[0] = bt / torch.linalg.vector_norm(bt)
            for j in range(steps):
                op.near_precondition_device(inner_its, Vb[j].data_ptr(), Zb[j].data_ptr(), ts.cuda_stream)
                if j + 1 == steps:
                    break
                op.apply_device(Zb[j].data_ptr(), w.data_ptr(), ts.cuda_stream)
                for _ in range(2):
                    h = torch.mv(Vb[:j + 1].conj(), w)
                    w -= torch.mv(Vb[:j + 1].transpose(0, 1), h)
                Vb[j + 1] = w / torch.linalg.vector_norm(w)
            vs.append(Vb)
            zs.append(Zb)
    ts.synchronize()
    return dict(v=torch.cat(vs), z=torch.cat(zs))


def random_directions(op: MLFMM, count: int, inner_its: int = 8, seed: int = 0):
    """(v, z) pairs on the device with v complex white noise of unit norm and
    z = P_near v: with the residual loss |A M v - v|^2 they give the
    Frobenius-norm objective |A M - I|_F^2 of sparse approximate inverses."""
    import torch
    dev = torch.device("cuda", op.device)
    g = torch.Generator(device="cpu").manual_seed(seed)
    V = torch.complex(torch.randn(count, op.n, generator=g, dtype=torch.float64),
                      torch.randn(count, op.n, generator=g, dtype=torch.float64)).to(dev)
    V /= torch.linalg.vector_norm(V, dim=1, keepdim=True)
    Z = torch.empty_like(V)
    torch.cuda.synchronize(dev)
    for k in range(count):
        op.near_precondition_device(inner_its, V[k].data_ptr(), Z[k].data_ptr())
    return dict(v=V, z=Z)


def merge(*datasets):
    """One dataset of (v, z) pairs from several (e dropped unless all have it)."""
    import torch
    out = dict(v=torch.cat([d["v"] for d in datasets]), z=torch.cat([d["z"] for d in datasets]))
    if all("e" in d for d in datasets):
        out["e"] = torch.cat([d["e"] for d in datasets])
    return out


def solve_gain(op: MLFMM, params, rhs_rows, inner_its: int = 8, tol: float = 1e-3, mr: int = 50,
               itr_max: int = 400) -> dict:
    """FGMRES iterations and seconds per right-hand side with the near-field
    preconditioner alone and with the network attached after it."""
    out = {}
    for tag, p in (("near_field", None), ("learned", params)):
        op.attach_learned(p)
        its, secs, conv = [], 0.0, 0
        for b in rhs_rows:
            _, st = op.matrix_solver(b, tol_rel=tol, tol_abs=0.0, mr=mr, itr_max=itr_max, inner_its=inner_its)
            its.append(int(st["iterations"]))
            secs += st["seconds"]
            conv += int(st["converged"])
        out[tag] = dict(iterations=its, iterations_mean=float(np.mean(its)), s_per_rhs=secs / len(rhs_rows),
                        converged=conv)
    op.attach_learned(None)
    return out


class Trainer:
    """Adam on the network's parameters over the triples of several bodies
    (each body: an operator and its harvested triples)."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0, device: int = 0, loss: str = "residual"):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        if loss not in ("residual", "aligned", "error"):
            raise ValueError("loss must be 'residual' (|A y - v|^2 / |v|^2), 'aligned' "
                             "(min_a |a A y - v|^2 / |v|^2) or 'error' (|y - e|^2 / |e|^2)")
        self.loss_kind = loss
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float32)
        self.theta = torch.from_numpy(p.copy()).to(self.dev)
        self.grad = torch.zeros_like(self.theta)
        self.m = torch.zeros_like(self.theta)
        self.s = torch.zeros_like(self.theta)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self.step = 0
        # a stream of its own: handle 0 (torch's legacy default stream) would
        # mean the plan's stream to the library, unordered with torch's work
        self.tstream = torch.cuda.Stream(self.dev)
        self.tstream.wait_stream(torch.cuda.current_stream(self.dev))
        self.stream = self.tstream.cuda_stream

    def params(self) -> np.ndarray:
        self.tstream.synchronize()
        return self.theta.cpu().numpy()

    def _loss_grad(self, op: MLFMM, data: dict, k: int, buf, grad: bool = True):
        """Adds pair k's loss to self.loss and (grad, or always for the error
        loss) its parameter gradient to self.grad. Error loss: |y - e|^2 / |e|^2. Residual loss:
        |A y - v|^2 / |v|^2. Aligned loss: the part of v that the direction
        A y leaves unexplained, min over complex a of |a A y - v|^2 / |v|^2
        (what one flexible GMRES step gains from y). With r = a A y - v
        (a = 1 for the residual loss, a = (A y)^H v / |A y|^2 for the aligned
        one) the gradient with respect to y is 2 conj(a) A^H r / |v|^2;
        A^H r = conj(D A D conj(r)) with D = diag(I, -I), because the PMCHWT
        blocks are symmetric (A^T = D A D)."""
        v, z = data["v"][k], data["z"][k]
        y = buf[0]
        if self.loss_kind == "error":
            op.lp_loss_grad_device(self.theta.data_ptr(), v.data_ptr(), z.data_ptr(), data["e"][k].data_ptr(),
                                   y.data_ptr(), self.grad.data_ptr(), self.loss.data_ptr(), self.stream)
            return
        w, a = buf[1], buf[2]
        N = op.N
        op.lp_forward_device(self.theta.data_ptr(), v.data_ptr(), z.data_ptr(), y.data_ptr(), self.stream)
        op.apply_device(y.data_ptr(), w.data_ptr(), self.stream)
        vn2 = torch_sq(self.torch, v)
        if self.loss_kind == "aligned":
            alpha = self.torch.vdot(w, v) / torch_sq(self.torch, w)
            w.mul_(alpha)
        else:
            alpha = self.torch.ones((), dtype=w.dtype, device=w.device)
        w.sub_(v)
        self.loss.add_((torch_sq(self.torch, w) / vn2).float())
        if not grad:
            return
        a.copy_(w.conj())
        a[N:].neg_()
        op.apply_device(a.data_ptr(), y.data_ptr(), self.stream)
        y[N:].neg_()
        a.copy_(y.conj())
        a.mul_(2.0 * alpha.conj() / vn2)
        op.lp_backward_device(self.theta.data_ptr(), a.data_ptr(), self.grad.data_ptr(), self.stream)

    def _buffers(self, d):
        return [self.torch.empty_like(d["v"][0]) for _ in range(3)]

    def epoch(self, bodies, lr: float = 1e-3, batch: int = 8, rng=None) -> float:
        """One pass over every triple in random order, an Adam step per batch;
        returns the mean loss seen during the pass."""
        torch = self.torch
        rng = rng or np.random.default_rng(self.step)
        items = [(i, k) for i, (_, d) in enumerate(bodies) for k in range(d["v"].shape[0])]
        order = rng.permutation(len(items))
        with torch.cuda.stream(self.tstream):
            return self._epoch(bodies, items, order, lr, batch)

    def _epoch(self, bodies, items, order, lr, batch) -> float:
        torch = self.torch
        ys = [self._buffers(d) for _, d in bodies]
        total = torch.zeros(1, dtype=torch.float32, device=self.dev)
        for start in range(0, len(order), batch):
            chunk = order[start:start + batch]
            self.grad.zero_()
            self.loss.zero_()
            for j in chunk:
                i, k = items[j]
                self._loss_grad(bodies[i][0], bodies[i][1], k, ys[i])
            self.step += 1
            lp_adam_device(self.theta.numel(), self.theta.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                           self.s.data_ptr(), lr, self.step, grad_scale=1.0 / len(chunk), stream=self.stream)
            total += self.loss
        return float(total.item()) / max(len(items), 1)

    def evaluate(self, bodies) -> dict:
        """Mean loss of the network and of the near-field preconditioner alone
        (y = z) over the triples, without training."""
        with self.torch.cuda.stream(self.tstream):
            return self._evaluate(bodies)

    def _evaluate(self, bodies) -> dict:
        torch = self.torch
        g_keep = self.grad.clone()
        net = base = 0.0
        count = 0
        for op, d in bodies:
            buf = self._buffers(d)
            for k in range(d["v"].shape[0]):
                self.loss.zero_()
                self._loss_grad(op, d, k, buf, grad=False)
                net += float(self.loss.item())
                v, z = d["v"][k], d["z"][k]
                if self.loss_kind == "error":
                    e = d["e"][k]
                    base += float((torch_sq(torch, z - e) / torch_sq(torch, e)).item())
                else:
                    w = buf[1]
                    op.apply_device(z.data_ptr(), w.data_ptr(), self.stream)
                    alpha = torch.vdot(w, v) / torch_sq(torch, w) if self.loss_kind == "aligned" else 1.0
                    base += float((torch_sq(torch, alpha * w - v) / torch_sq(torch, v)).item())
                count += 1
        self.grad.copy_(g_keep)
        return dict(network=net / max(count, 1), near_only=base / max(count, 1), triples=count)


def torch_sq(torch, x):
    return torch.linalg.vector_norm(x) ** 2


def train(bodies, epochs: int = 15, lr: float = 1e-3, batch: int = 8, seed: int = 0, params=None,
          lr_final: float | None = None, log=None, loss: str = "residual"):
    """Trains from init_params(seed) (or params) over the bodies' triples;
    cosine decay of the learning rate to lr_final (default lr / 10). Returns
    (parameters as float32 numpy, per-epoch mean losses, seconds)."""
    t0 = time.perf_counter()
    tr = Trainer(params, seed, loss=loss)
    lr_final = lr / 10 if lr_final is None else lr_final
    hist = []
    rng = np.random.default_rng(seed)
    for ep in range(epochs):
        lr_ep = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * ep / max(epochs - 1, 1)))
        hist.append(tr.epoch(bodies, lr=lr_ep, batch=batch, rng=rng))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f} (lr {lr_ep:.2e})")
    tr.torch.cuda.synchronize()
    return tr.params(), hist, time.perf_counter() - t0
