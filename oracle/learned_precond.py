"""Test infrastructure: the CPU oracle of the learned leaf-box preconditioner.

The preconditioner has no counterpart in the reference (whose solvers are
unpreconditioned, Code/GMRES.h:65-217); this module is the float64 numpy
statement of the network that ``csrc/learned.cu`` runs on the GPU, used by
the tests to check the GPU forward pass, loss and parameter gradients, and
itself checked by finite differences.

Preconditioner: given a Krylov vector v (complex [2N], J then M) and the
near-field preconditioner's output z = P_near v, it returns

    y_c[i] = z_c[i] + sum_t G[i, c, t] * u_t[i]        c in {J, M}, t < 8

with the linear terms (all linear in z)

    u = (z_J, z_M, d_i . Z2_J[box], d_i . Z2_M[box],
         d_i . Zb_J[box], d_i . Zb_M[box], d_i . Zn_J[box], d_i . Zn_M[box])

where d_i is RWG i's normalised dipole vector l_i (c+ - c-), Zb_c[b] the mean
of z_c[j] d_j over the RWGs j of box b, Zn_c[b] the mean of Zb_c over b and its
near-field neighbour boxes, and Z2_c[b] the same mean of Zn_c (two rings). The
complex gains G are predicted per RWG by a message-passing network over the
octree's leaf boxes from static geometric and material features only, so the
preconditioner is linear: y = (I + L) P_near v with a fixed L per body.

Network (weights stored in bfloat16, arithmetic in float32 on the GPU):
  encoder   a_i = relu(We f_i + be)                      f_i: 16 static features
  pooling   h0_b = mean_{i in b} a_i
  3 layers  h_{l+1,b} = h_l,b + relu(Ws h_l,b + Wn m_l,b + Wg g_l + c_l)
            m_l,b = mean over {b} + near(b) of h_l ; g_l = mean over boxes
  decoder   q_i = relu(Wd1 [h3_box(i); a_i] + d1) ;  G_i = Wd2 q_i + d2
Losses: of a (v, z, e) triple, e the exact solution A^-1 v,
  L = sum |y - e|^2 / sum |e|^2 ;
or any L(y) through its gradient gy = dL/dRe(y) + j dL/dIm(y), such as the
residual-space loss min_a |a A y - v|^2 / |v|^2.
"""
from __future__ import annotations

import numpy as np

F, H, T, NG, LAYERS = 16, 64, 8, 32, 3


def layout():
    """(name, shape) of each parameter block, in storage order."""
    out = [("We", (H, F)), ("be", (H,))]
    for l in range(LAYERS):
        out += [(f"Ws{l}", (H, H)), (f"Wn{l}", (H, H)), (f"Wg{l}", (H, H)), (f"c{l}", (H,))]
    out += [("Wd1", (H, 2 * H)), ("d1", (H,)), ("Wd2", (NG, H)), ("d2", (NG,))]
    return out


def param_count() -> int:
    return sum(int(np.prod(s)) for _, s in layout())


def unpack(theta: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in layout():
        k = int(np.prod(shape))
        out[name] = theta[o:o + k].reshape(shape)
        o += k
    return out


def pack(blocks: dict) -> np.ndarray:
    return np.concatenate([np.asarray(blocks[name], dtype=np.float64).reshape(-1) for name, _ in layout()])


def init_params(seed: int = 0) -> np.ndarray:
    """He-scaled weights, zero biases, and a zero output layer, so that the
    untrained network returns y = z (the near-field preconditioner)."""
    rng = np.random.default_rng(seed)
    b = {}
    for name, shape in layout():
        if len(shape) == 1 or name == "Wd2":
            b[name] = np.zeros(shape)
        else:
            fan_in = shape[1] * (2 if name.startswith(("Ws", "Wn", "Wg")) else 1)
            scale = np.sqrt(2.0 / fan_in) * (0.5 if name.startswith(("Ws", "Wn", "Wg")) else 1.0)
            b[name] = rng.normal(0.0, scale, size=shape)
    return pack(b).astype(np.float32)


def bf16_round(x) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


class Graph:
    """Static tables of one body: leaf boxes, their RWGs, neighbourhoods and
    the RWG dipoles.

    leaf_ptr/leaf_rwg: RWG ids per leaf box (the plan's leaf order);
    near_ptr/near_idx: near-field neighbour boxes at the leaf level;
    points/faces: the mesh; face_pos/face_neg/length: the RWGs."""

    def __init__(self, leaf_ptr, leaf_rwg, near_ptr, near_idx, points, faces, face_pos, face_neg, length, eps_r):
        self.leaf_ptr = np.asarray(leaf_ptr, dtype=np.int64)
        self.leaf_rwg = np.asarray(leaf_rwg, dtype=np.int64)
        self.B = len(self.leaf_ptr) - 1
        self.N = len(self.leaf_rwg)
        self.box_of_pos = np.repeat(np.arange(self.B), np.diff(self.leaf_ptr))
        self.nbr = []
        for b in range(self.B):
            s = set(int(j) for j in near_idx[near_ptr[b]:near_ptr[b + 1]])
            s.add(b)
            self.nbr.append(np.array(sorted(s), dtype=np.int64))
        pts = np.asarray(points, dtype=np.float64)
        tri = pts[np.asarray(faces)]
        cen = tri.mean(axis=1)
        cr = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
        area = 0.5 * np.linalg.norm(cr, axis=1)
        nrm = cr / np.linalg.norm(cr, axis=1)[:, None]
        fp, fn, length = np.asarray(face_pos), np.asarray(face_neg), np.asarray(length, dtype=np.float64)
        d = length[:, None] * (cen[fp] - cen[fn])
        self.dip = d / np.mean(np.linalg.norm(d, axis=1))
        eps_r = complex(eps_r)
        # static features per RWG id (leaf-order copies are taken in forward)
        n_b = np.diff(self.leaf_ptr).astype(np.float64)
        box_of_rwg = np.empty(self.N, dtype=np.int64)
        box_of_rwg[self.leaf_rwg] = self.box_of_pos
        dsum = np.zeros((self.B, 3))
        np.add.at(dsum, self.box_of_pos, self.dip[self.leaf_rwg])
        coh = np.linalg.norm(dsum, axis=1) / n_b
        nnb = np.array([len(x) for x in self.nbr], dtype=np.float64)
        f = np.zeros((self.N, F))
        f[:, 0] = length / length.mean()
        f[:, 1] = area[fp] / area.mean()
        f[:, 2] = area[fn] / area.mean()
        f[:, 3] = np.einsum("ij,ij->i", nrm[fp], nrm[fn])
        f[:, 4] = np.linalg.norm(self.dip, axis=1)
        f[:, 5] = n_b[box_of_rwg] / 16.0
        f[:, 6] = nnb[box_of_rwg] / 27.0
        f[:, 7] = coh[box_of_rwg]
        f[:, 8] = np.log(eps_r.real)
        f[:, 9] = abs(eps_r.imag) / eps_r.real
        f[:, 10] = np.sqrt(eps_r.real) / 2.0
        self.feat = f


def forward(theta, g: Graph, v, z, keep: bool = False, bf16: bool = True):
    """y for one vector (complex [2N]; v enters through z = P_near v only);
    with keep, also the intermediates the backward pass needs. bf16=False takes the parameters as they are
    (float64), for finite-difference checks of the gradient."""
    if bf16:
        W = {k: bf16_round(a) for k, a in unpack(np.asarray(theta, dtype=np.float32)).items()}
    else:
        W = unpack(np.asarray(theta, dtype=np.float64))
    N, B = g.N, g.B
    z = np.asarray(z, dtype=np.complex128)
    ids = g.leaf_rwg                                        # leaf order -> RWG id
    zJ, zM = z[:N][ids], z[N:][ids]
    dip = g.dip[ids]
    zb = np.zeros((B, 2, 3), dtype=np.complex128)
    for b in range(B):
        s = slice(g.leaf_ptr[b], g.leaf_ptr[b + 1])
        n_b = s.stop - s.start
        zb[b, 0] = (zJ[s, None] * dip[s]).sum(axis=0) / n_b
        zb[b, 1] = (zM[s, None] * dip[s]).sum(axis=0) / n_b
    zn = np.stack([zb[g.nbr[b]].mean(axis=0) for b in range(B)])
    z2 = np.stack([zn[g.nbr[b]].mean(axis=0) for b in range(B)])
    box = g.box_of_pos
    dot = lambda zz, c: np.einsum("ik,ik->i", dip, zz[box, c])
    u = np.stack([zJ, zM, dot(z2, 0), dot(z2, 1), dot(zb, 0), dot(zb, 1), dot(zn, 0), dot(zn, 1)], axis=1)
    f = g.feat[ids]
    pre_e = f @ W["We"].T + W["be"]
    a = np.maximum(pre_e, 0.0)
    n_b = np.diff(g.leaf_ptr).astype(np.float64)
    h = [np.add.reduceat(a, g.leaf_ptr[:-1], axis=0) / n_b[:, None]]
    ms, Ps, gs = [], [], []
    for l in range(LAYERS):
        hl = h[-1]
        m = np.stack([hl[g.nbr[b]].mean(axis=0) for b in range(B)])
        gl = hl.mean(axis=0)
        P = hl @ W[f"Ws{l}"].T + m @ W[f"Wn{l}"].T + gl @ W[f"Wg{l}"].T + W[f"c{l}"]
        h.append(hl + np.maximum(P, 0.0))
        ms.append(m)
        Ps.append(P)
        gs.append(gl)
    x = np.concatenate([h[-1][box], a], axis=1)
    pre_q = x @ W["Wd1"].T + W["d1"]
    qh = np.maximum(pre_q, 0.0)
    Gr = qh @ W["Wd2"].T + W["d2"]                          # [N][32]
    Gc = (Gr[:, 0::2] + 1j * Gr[:, 1::2]).reshape(N, 2, T)  # [N][c][t]
    yl = np.stack([zJ, zM], axis=1) + np.einsum("ict,it->ic", Gc, u)
    y = np.empty(2 * N, dtype=np.complex128)
    y[ids], y[N + ids] = yl[:, 0], yl[:, 1]
    if not keep:
        return y
    cache = dict(W=W, f=f, pre_e=pre_e, a=a, h=h, ms=ms, Ps=Ps, gs=gs, x=x, pre_q=pre_q, qh=qh, u=u, yl=yl,
                 ids=ids, box=box, n_b=n_b)
    return y, cache


def loss_grad(theta, g: Graph, v, z, e, bf16: bool = True):
    """Loss and its gradient with respect to the parameters; the gradient is
    taken at the bf16-rounded weights the forward pass uses (bf16=False: at
    the parameters themselves)."""
    y, c = forward(theta, g, v, z, keep=True, bf16=bf16)
    e = np.asarray(e, dtype=np.complex128)
    E = np.sum(np.abs(e) ** 2)
    loss = np.sum(np.abs(y - e) ** 2) / E
    return loss, _backward(c, g, 2.0 * (y - e) / E), y


def grad_from_gy(theta, g: Graph, v, z, gy, bf16: bool = True):
    """Parameter gradient of a loss L(y) given gy = dL/dRe(y) + j dL/dIm(y)
    (complex [2N]), e.g. gy = 2 A^H (A y - v) / |v|^2 for the residual-space
    loss |A y - v|^2 / |v|^2."""
    y, c = forward(theta, g, v, z, keep=True, bf16=bf16)
    return _backward(c, g, np.asarray(gy, dtype=np.complex128)), y


def _backward(c, g: Graph, gy):
    W, N, B = c["W"], g.N, g.B
    ids = c["ids"]
    gl = np.stack([gy[:N][ids], gy[N:][ids]], axis=1)      # [N][2]
    # dL/dG: gain (c, t) multiplies u_t in output c
    cu = np.conj(gl)[:, :, None] * c["u"][:, None, :]       # [N][2][T]
    dG = np.empty((N, NG))
    dG[:, 0::2] = cu.real.reshape(N, 2 * T)
    dG[:, 1::2] = -cu.imag.reshape(N, 2 * T)
    grad = {}
    grad["Wd2"] = dG.T @ c["qh"]
    grad["d2"] = dG.sum(axis=0)
    dq = (dG @ W["Wd2"]) * (c["pre_q"] > 0)
    grad["Wd1"] = dq.T @ c["x"]
    grad["d1"] = dq.sum(axis=0)
    dx = dq @ W["Wd1"]
    da = dx[:, H:].copy()
    dh = np.zeros((B, H))
    np.add.at(dh, c["box"], dx[:, :H])
    for l in reversed(range(LAYERS)):
        dP = dh * (c["Ps"][l] > 0)
        S = dP.sum(axis=0)
        grad[f"Ws{l}"] = dP.T @ c["h"][l]
        grad[f"Wn{l}"] = dP.T @ c["ms"][l]
        grad[f"Wg{l}"] = np.outer(S, c["gs"][l])
        grad[f"c{l}"] = S
        dm = dP @ W[f"Wn{l}"]
        dh_new = dh + dP @ W[f"Ws{l}"] + (S @ W[f"Wg{l}"]) / B
        for b in range(B):
            nb = g.nbr[b]
            dh_new[nb] += dm[b] / len(nb)
        dh = dh_new
    da += dh[c["box"]] / c["n_b"][c["box"]][:, None]
    dpre = da * (c["pre_e"] > 0)
    grad["We"] = dpre.T @ c["f"]
    grad["be"] = dpre.sum(axis=0)
    return pack(grad)


def adam(theta, grad, m, s, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (float32 state), as the GPU kernel takes it."""
    theta, grad, m, s = (np.asarray(a, dtype=np.float32) for a in (theta, grad, m, s))
    m = b1 * m + (1 - b1) * grad
    s = b2 * s + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    sh = s / (1 - b2 ** step)
    return (theta - lr * mh / (np.sqrt(sh) + eps)).astype(np.float32), m.astype(np.float32), s.astype(np.float32)
