"""Block-Krylov study (host only, not collected by pytest): does a block
flexible GMRES over many incidences need fewer operator applications per
right-hand side than flexible GMRES one incidence at a time? Both use the
near-field preconditioner (8 GMRES steps on Z_near, as mlfma_fgmres), on the
reference's dense MoM matrix (Code/Zmartix.h:467-539) of the sphere of radius
1 m, icosphere sub 3 (3,840 unknowns), eps_r 4, with R plane waves theta_i =
i * 180 / (R - 1), phi = 0, polarisation alternating, to 1e-3 relative
residual per right-hand side. The block method restarts every 20 blocks and
stops a block once all its columns meet the tolerance.

    python tests/study_block_krylov.py [R]       # about 3 minutes for R = 32

Result for R = 32: 40.8 applications per right-hand side one at a time,
against 52.9 / 52.5 / 49.0 for blocks of 4 / 8 / 16.
"""
import os
import sys
import tempfile
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import numpy as np, scipy.sparse as sp, scipy.sparse.linalg as spla
from oracle import oracle as O
from mlfma_pmchwt_b200 import mesh as M
O.set_threads(os.cpu_count())
FREQ = 3e8
m = M.icosphere(3, 1.0)
d = tempfile.mkdtemp(); p = M.write_nas(m, os.path.join(d, 's3.nas'))
t=time.time(); ref = O.RefOperator(p, freq=FREQ, eps_r=4.0, leaf_coeff=0.25); print('ref', time.time()-t)
A = ref.mom_matrix(); n = A.shape[0]
ptr, ids, vals = ref.znear(); Zn = sp.csr_matrix((vals, ids, ptr), shape=(n, n))
lu = spla.splu(Zn.tocsc())
R = int(sys.argv[1]) if len(sys.argv) > 1 else 32
th = np.array([180.0 * i / (R - 1) for i in range(R)])
B = np.stack([ref.rhs(90.0 * (i % 2), th[i], 0.0)[0] for i in range(R)], axis=1)
inner = 8
def prec(v):  # inner GMRES steps on Zn from zero
    beta = np.linalg.norm(v); Q = [v / beta]; H = np.zeros((inner + 1, inner), complex)
    for j in range(inner):
        u = Zn @ Q[j]
        for _ in range(2):
            for i in range(j + 1):
                h = np.vdot(Q[i], u); H[i, j] += h; u = u - h * Q[i]
        H[j + 1, j] = np.linalg.norm(u)
        if H[j + 1, j] < 1e-14 * beta: 
            k = j + 1; break
        Q.append(u / H[j + 1, j]); k = j + 1
    e = np.zeros(k + 1, complex); e[0] = beta
    y = np.linalg.lstsq(H[:k + 1, :k], e, rcond=None)[0]
    return sum(y[i] * Q[i] for i in range(k))
def fgmres(b, mr=50, tol=1e-3):
    x = np.zeros(n, complex); mv = 0; bn = np.linalg.norm(b)
    while True:
        r = b - A @ x; mv += 1
        beta = np.linalg.norm(r)
        if beta / bn < tol: return x, mv
        V = [r / beta]; Z = []; H = np.zeros((mr + 1, mr), complex)
        for j in range(mr):
            z = prec(V[j]); Z.append(z); w = A @ z; mv += 1
            for _ in range(2):
                for i in range(j + 1):
                    h = np.vdot(V[i], w); H[i, j] += h; w = w - h * V[i]
            H[j + 1, j] = np.linalg.norm(w); V.append(w / H[j + 1, j])
            e = np.zeros(j + 2, complex); e[0] = beta
            y, res, *_ = np.linalg.lstsq(H[:j + 2, :j + 1], e, rcond=None)
            if np.linalg.norm(e - H[:j + 2, :j + 1] @ y) / bn < tol: break
        x = x + sum(y[i] * Z[i] for i in range(len(y)))
def block_fgmres(Bm, mr=20, tol=1e-3):
    p = Bm.shape[1]; X = np.zeros_like(Bm); mv = 0; bn = np.linalg.norm(Bm, axis=0)
    while True:
        Rm = Bm - A @ X; mv += p
        rn = np.linalg.norm(Rm, axis=0)
        if np.all(rn / bn < tol): return X, mv
        V0, S = np.linalg.qr(Rm)
        V = [V0]; Zs = []; H = np.zeros(((mr + 1) * p, mr * p), complex)
        for j in range(mr):
            Zj = np.stack([prec(V[j][:, c]) for c in range(p)], axis=1); Zs.append(Zj)
            W = A @ Zj; mv += p
            for _ in range(2):
                for i in range(j + 1):
                    Hij = V[i].conj().T @ W; H[i*p:(i+1)*p, j*p:(j+1)*p] += Hij; W = W - V[i] @ Hij
            Vn, Hn = np.linalg.qr(W); H[(j+1)*p:(j+2)*p, j*p:(j+1)*p] = Hn; V.append(Vn)
            E = np.zeros(((j + 2) * p, p), complex); E[:p] = S
            Hm = H[:(j + 2) * p, :(j + 1) * p]
            Y = np.linalg.lstsq(Hm, E, rcond=None)[0]
            res = np.linalg.norm(E - Hm @ Y, axis=0) / bn
            if np.all(res < tol): break
        Zall = np.concatenate(Zs, axis=1)
        X = X + Zall @ Y
tot = 0
t = time.time()
for c in range(R):
    _, mv = fgmres(B[:, c]); tot += mv
print('per-RHS FGMRES: matvecs/RHS', tot / R, 'precond/RHS (same)', round(time.time() - t, 1), 's')
for p in (4, 8, 16):
    tot = 0; t = time.time()
    for c0 in range(0, R, p):
        _, mv = block_fgmres(B[:, c0:c0 + p]); tot += mv
    print('block p', p, 'matvecs/RHS', tot / R, round(time.time() - t, 1), 's')
