"""Learned initial density for RHF: a small MLP over atom-pair features.

The reference starts every SCF from P = I (src/scf.rs:757-764).  This module
predicts the converged density block by block instead:

* every unordered atom pair (A, B), A == B included, gets a local frame F
  (orthonormal rows e1, e2, e3).  Off the diagonal e1 points from A to B and
  the origin O is the bond midpoint; on the diagonal O = R_A and e1 points to
  the nearest atom of another element (the nearest atom if there is none).
  e2 lies in the plane of e1 and the nearest third atom that is not on the
  e1 axis, pointing towards it; e3 = e1 x e2.
* features: the pair type (one-hot over element pairs and diagonal
  elements), r_AB, exp(-r_AB / 2), and for each element and each radial
  Gaussian g_k the sums over the other atoms j of g_k(|d_j|) [1, d_j/|d_j|],
  with d_j = F (R_j - O).  They are invariant under rotation and translation
  of the molecule.
* target: the block rotated into the frame, P_loc = A_A(F)^T P_AB A_B(F),
  with A(Q) the matrix that carries cartesian GTOs through the rotation Q
  (libcint cartesian order), stored in an nmax x nmax grid with a mask.

Prediction inverts the rotation, P_AB = A_A(F^T)^T P_loc A_B(F^T), fills the
lower triangle from the upper one and scales P so that tr(P S) = N_elec.
The network (FP32, SiLU hidden layers, linear output) runs and trains on the
GPU through this library's own kernels (lrb_mlp_forward / lrb_mlp_backward /
lrb_mse / lrb_adam); torch only holds the device memory.  The guess is tied
to one basis per element; ``LearnedGuess.applies`` says whether a molecule
matches and the SCF falls back to the core-Hamiltonian guess when it does not.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from .basis import Molecule, ncart

RADIAL_CENTRES = np.array([1.0, 2.5, 4.0, 5.5, 7.0, 8.5, 10.0])   # bohr
RADIAL_WIDTH = 1.2


# ----------------------------------------------------------------- rotations
def cart_exponents(l: int):
    """libcint cartesian order: x power descending, then y descending."""
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


# d monomials xx, xy, xz, yy, yz, zz as axis pairs (libcint order)
_D_PAIRS = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))


def cart_rotation(l: int, Q: np.ndarray) -> np.ndarray:
    """A with phi_mu(Q^T v) = sum_nu A[mu, nu] phi_nu(v) for the cartesian
    monomials of degree l; A(Q1 Q2) = A(Q2) A(Q1)."""
    if l == 0:
        return np.ones((1, 1))
    if l == 1:
        return np.ascontiguousarray(Q.T)
    if l == 2:
        # (Q^T v)_i (Q^T v)_j = sum_kl Q[k,i] Q[l,j] v_k v_l
        A = np.empty((6, 6))
        for mu, (i, j) in enumerate(_D_PAIRS):
            for nu, (k, m) in enumerate(_D_PAIRS):
                A[mu, nu] = Q[k, i] * Q[m, j] + (Q[m, i] * Q[k, j] if k != m else 0.0)
        return A
    exps = cart_exponents(l)
    index = {e: i for i, e in enumerate(exps)}
    A = np.zeros((len(exps), len(exps)))
    for mu, e in enumerate(exps):
        poly = {(0, 0, 0): 1.0}
        for axis, power in enumerate(e):
            for _ in range(power):
                nxt = {}
                for mono, c in poly.items():
                    for j in range(3):
                        q = Q[j, axis]          # (Q^T v)_axis = sum_j Q[j, axis] v_j
                        if q == 0.0:
                            continue
                        m2 = list(mono)
                        m2[j] += 1
                        m2 = tuple(m2)
                        nxt[m2] = nxt.get(m2, 0.0) + c * q
                poly = nxt
        for mono, c in poly.items():
            A[mu, index[mono]] += c
    return A


def _atom_layout(m: Molecule):
    """Per atom: (ao offset, [l of each shell], ncart total)."""
    bas = np.asarray(m.bas).reshape(-1, 8)
    off = 0
    atoms = {}
    for b in bas:
        a, l = int(b[0]), int(b[1])
        nc = ncart(l) * int(b[3])
        atoms.setdefault(a, [None, [], 0])
        if atoms[a][0] is None:
            atoms[a][0] = off
        if off != atoms[a][0] + atoms[a][2]:
            raise ValueError("shells of one atom must be contiguous")
        atoms[a][1].append(l)
        atoms[a][2] += nc
        off += nc
    return [tuple(atoms[a]) for a in range(len(atoms))]


def _atom_prims(m: Molecule):
    """Per atom: its shells' exponents and coefficients, concatenated."""
    bas = np.asarray(m.bas).reshape(-1, 8)
    env = np.asarray(m.env)
    out = {}
    for b in bas:
        k = int(b[2]) * 1
        v = np.concatenate([env[b[5]:b[5] + k], env[b[6]:b[6] + k * int(b[3])]])
        out.setdefault(int(b[0]), []).append(v)
    return [np.concatenate(out[a]) for a in range(len(out))]


def atom_rotation(ls, Q):
    n = sum(ncart(l) for l in ls)
    A = np.zeros((n, n))
    o = 0
    for l in ls:
        k = ncart(l)
        A[o:o + k, o:o + k] = cart_rotation(l, Q)
        o += k
    return A


def cart_rotation_batch(l: int, Q: np.ndarray) -> np.ndarray:
    """cart_rotation for a stack of matrices Q (m, 3, 3), l <= 2."""
    m = Q.shape[0]
    if l == 0:
        return np.ones((m, 1, 1))
    if l == 1:
        return np.ascontiguousarray(np.transpose(Q, (0, 2, 1)))
    if l == 2:
        A = np.empty((m, 6, 6))
        for mu, (i, j) in enumerate(_D_PAIRS):
            for nu, (k, q) in enumerate(_D_PAIRS):
                v = Q[:, k, i] * Q[:, q, j]
                if k != q:
                    v = v + Q[:, q, i] * Q[:, k, j]
                A[:, mu, nu] = v
        return A
    return np.stack([cart_rotation(l, q) for q in Q])


def atom_rotation_batch(ls, Q):
    """atom_rotation for a stack of matrices Q (m, 3, 3)."""
    n = sum(ncart(l) for l in ls)
    A = np.zeros((Q.shape[0], n, n))
    o = 0
    for l in ls:
        k = ncart(l)
        A[:, o:o + k, o:o + k] = cart_rotation_batch(l, Q)
        o += k
    return A


# ------------------------------------------------------------------ features
def molecule_geometry(m: Molecule):
    atm = np.asarray(m.atm).reshape(-1, 6)
    env = np.asarray(m.env)
    z = atm[:, 0].astype(int)
    xyz = np.stack([env[p:p + 3] for p in atm[:, 1]])
    return z, xyz


def _frames(xyz, z, A, B):
    """Origins (m, 3) and frames (m, 3, 3) of the pairs (A[i], B[i]) -- the
    rules of _frame, for all pairs at once."""
    m = len(A)
    idx = np.arange(m)
    diag = A == B
    O = np.where(diag[:, None], xyz[A], 0.5 * (xyz[A] + xyz[B]))
    D = np.linalg.norm(xyz[None, :, :] - xyz[:, None, :], axis=2)
    np.fill_diagonal(D, np.inf)
    other = np.where(z[None, :] != z[:, None], D, np.inf)
    near = np.where(np.isfinite(other).any(1), np.argmin(other, 1), np.argmin(D, 1))
    e1 = np.where(diag[:, None], xyz[near[A]] - xyz[A], xyz[B] - xyz[A])
    e1 = e1 / np.linalg.norm(e1, axis=1)[:, None]
    T = xyz[None, :, :] - O[:, None, :]                          # (m, n, 3)
    perp = T - np.einsum("mnk,mk->mn", T, e1)[..., None] * e1[:, None, :]
    pn = np.linalg.norm(perp, axis=2)
    key = np.where(pn > 0.1, np.linalg.norm(T, axis=2), np.inf)
    key[idx, A] = np.inf
    key[idx, B] = np.inf
    j2 = np.argmin(key, axis=1)                                   # first among ties
    has = np.isfinite(key[idx, j2])
    e2 = perp[idx, j2] / np.where(has, pn[idx, j2], 1.0)[:, None]
    if not has.all():                                             # linear: any perpendicular
        t = np.where((np.abs(e1[:, 0]) < 0.9)[:, None], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0])
        t = t - np.sum(t * e1, axis=1)[:, None] * e1
        t = t / np.linalg.norm(t, axis=1)[:, None]
        e2 = np.where(has[:, None], e2, t)
    e3 = np.cross(e1, e2)
    return O, np.stack([e1, e2, e3], axis=1)


def _frame(xyz, z, a, b):
    n = len(xyz)
    if a != b:
        o = 0.5 * (xyz[a] + xyz[b])
        e1 = xyz[b] - xyz[a]
    else:
        o = xyz[a]
        d = np.linalg.norm(xyz - o, axis=1)
        d[a] = np.inf
        other = np.where(z != z[a], d, np.inf)
        j = int(np.argmin(other)) if np.isfinite(other).any() else int(np.argmin(d))
        e1 = xyz[j] - o
    e1 = e1 / np.linalg.norm(e1)
    d = np.linalg.norm(xyz - o, axis=1)
    order = np.argsort(d, kind="stable")
    e2 = None
    for j in order:
        if j in (a, b):
            continue
        t = xyz[j] - o
        perp = t - (t @ e1) * e1
        if np.linalg.norm(perp) > 0.1:
            e2 = perp / np.linalg.norm(perp)
            break
    if e2 is None:                       # linear molecule: any perpendicular
        t = np.array([1.0, 0.0, 0.0]) if abs(e1[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        e2 = t - (t @ e1) * e1
        e2 /= np.linalg.norm(e2)
    e3 = np.cross(e1, e2)
    return o, np.stack([e1, e2, e3])


@dataclass
class PairSet:
    pairs: np.ndarray        # (np, 2) atom indices, a <= b after type ordering
    types: np.ndarray        # (np,) type index
    frames: np.ndarray       # (np, 3, 3)
    X: np.ndarray            # (np, nfeat) float64


class PairModel:
    """Element set and per-element AO layout a network is built for."""

    def __init__(self, elements, layouts, prims=None):
        self.elements = tuple(sorted(elements, reverse=True))
        self.layouts = {int(k): tuple(v) for k, v in layouts.items()}   # Z -> shell ls
        # Z -> concatenated (exponents, coefficients) of its shells, or None
        self.prims = {int(k): np.asarray(v) for k, v in (prims or {}).items()}
        self.nao = {zz: sum(ncart(l) for l in self.layouts[zz]) for zz in self.elements}
        self.nmax = max(self.nao.values())
        pt = [(p, q) for i, p in enumerate(self.elements) for q in self.elements[i:]]
        self.type_names = [f"{p}-{q}" for p, q in pt] + [f"{p}" for p in self.elements]
        self.type_index = {pq: i for i, pq in enumerate(pt)}
        for i, p in enumerate(self.elements):
            self.type_index[(p,)] = len(pt) + i
        self.ntypes = len(self.type_names)
        self.nfeat = self.ntypes + 2 + len(self.elements) * len(RADIAL_CENTRES) * 4
        self.nout = self.nmax * self.nmax

    @staticmethod
    def from_molecule(m: Molecule) -> "PairModel":
        z, _ = molecule_geometry(m)
        lay, prims = {}, {}
        ap = _atom_prims(m)
        for a, (_, ls, _) in enumerate(_atom_layout(m)):
            zz = int(z[a])
            if zz in lay and (tuple(lay[zz]) != tuple(ls) or not np.array_equal(prims[zz], ap[a])):
                raise ValueError("atoms of one element carry different shells")
            lay[zz] = tuple(ls)
            prims[zz] = ap[a]
        return PairModel(sorted(set(int(v) for v in z)), lay, prims)

    def applies(self, m: Molecule) -> bool:
        """Same elements (a subset), the same shells per element and (when the
        model records them) the same exponents and coefficients."""
        z, _ = molecule_geometry(m)
        try:
            lay = _atom_layout(m)
        except ValueError:
            return False
        bas = np.asarray(m.bas).reshape(-1, 8)
        if not (bas[:, 3] == 1).all():
            return False
        ap = _atom_prims(m)
        for a, (_, ls, _) in enumerate(lay):
            zz = int(z[a])
            if zz not in self.layouts or tuple(ls) != self.layouts[zz]:
                return False
            ref = self.prims.get(zz)
            if ref is not None and (ref.shape != ap[a].shape or
                                    not np.allclose(ref, ap[a], rtol=1e-12, atol=0.0)):
                return False
        return True

    def pairs(self, m: Molecule) -> PairSet:
        """All unordered atom pairs (heavier element first, diagonal
        included) with their frames and features."""
        z, xyz = molecule_geometry(m)
        n = len(z)
        a, b = np.triu_indices(n)
        swap = z[b] > z[a]
        A = np.where(swap, b, a)
        B = np.where(swap, a, b)
        T = np.array([self.type_index[(int(z[p]),)] if p == q else
                      self.type_index[(int(z[p]), int(z[q]))] for p, q in zip(A, B)], dtype=np.int64)
        O, F = _frames(xyz, z, A, B)
        X = np.zeros((len(A), self.nfeat))
        X[np.arange(len(A)), T] = 1.0
        off = A != B
        r = np.linalg.norm(xyz[B] - xyz[A], axis=1)
        X[:, self.ntypes] = np.where(off, r, 0.0)
        X[:, self.ntypes + 1] = np.where(off, np.exp(-0.5 * r), 0.0)
        d = np.einsum("mij,mnj->mni", F, xyz[None, :, :] - O[:, None, :])   # frame coordinates
        rj = np.linalg.norm(d, axis=2)
        u = d / np.maximum(rj, 1e-12)[..., None]
        g = np.exp(-((rj[..., None] - RADIAL_CENTRES) / RADIAL_WIDTH) ** 2)  # (m, n, nk)
        keep = np.ones((len(A), n))
        keep[np.arange(len(A)), A] = 0.0
        keep[np.arange(len(A)), B] = 0.0
        g = g * keep[..., None]
        nk = len(RADIAL_CENTRES)
        base = self.ntypes + 2
        for e, ze in enumerate(self.elements):
            sel = z == ze
            if not sel.any():
                continue
            ge, ue = g[:, sel], u[:, sel]
            blk = base + e * nk * 4
            X[:, blk:blk + nk] = ge.sum(1)
            for c in range(3):
                X[:, blk + (c + 1) * nk:blk + (c + 2) * nk] = (ge * ue[:, :, c, None]).sum(1)
        return PairSet(np.stack([A, B], 1).astype(np.int64), T, F, X)

    def _rots(self, z, ps: PairSet, frames):
        """Rotation matrices of the A and B atoms of every pair for the given
        frames, batched per element."""
        RA = [None] * len(ps.pairs)
        RB = [None] * len(ps.pairs)
        for side, R in ((0, RA), (1, RB)):
            zs = z[ps.pairs[:, side]]
            for ze in np.unique(zs):
                sel = np.nonzero(zs == ze)[0]
                rot = atom_rotation_batch(self.layouts[int(ze)], frames[sel])
                for k, i in enumerate(sel):
                    R[i] = rot[k]
        return RA, RB

    def _rot(self, zz, F):
        return atom_rotation(self.layouts[zz], F)

    def to_local(self, m: Molecule, P: np.ndarray, ps: PairSet):
        """(np, nmax*nmax) targets and masks from a density."""
        z, _ = molecule_geometry(m)
        lay = _atom_layout(m)
        Y = np.zeros((len(ps.pairs), self.nmax, self.nmax))
        M = np.zeros_like(Y)
        RA, RB = self._rots(z, ps, ps.frames)
        for i, (a, b) in enumerate(ps.pairs):
            oa, _, na = lay[a]
            ob, _, nb = lay[b]
            Y[i, :na, :nb] = RA[i].T @ P[oa:oa + na, ob:ob + nb] @ RB[i]
            M[i, :na, :nb] = 1.0
        return Y.reshape(len(ps.pairs), -1), M.reshape(len(ps.pairs), -1)

    def to_density(self, m: Molecule, Yloc: np.ndarray, ps: PairSet):
        z, _ = molecule_geometry(m)
        lay = _atom_layout(m)
        n = lay[-1][0] + lay[-1][2]
        P = np.zeros((n, n))
        Y = Yloc.reshape(len(ps.pairs), self.nmax, self.nmax)
        RA, RB = self._rots(z, ps, np.transpose(ps.frames, (0, 2, 1)))
        for i, (a, b) in enumerate(ps.pairs):
            oa, _, na = lay[a]
            ob, _, nb = lay[b]
            blk = RA[i].T @ Y[i, :na, :nb] @ RB[i]
            if a == b:
                blk = 0.5 * (blk + blk.T)
            P[oa:oa + na, ob:ob + nb] = blk
            P[ob:ob + nb, oa:oa + na] = blk.T
        return P


# ------------------------------------------------------------------- network
class MLP:
    """Fully connected network; FP32 parameters on the GPU, this library's
    kernels for forward, backward, loss and Adam."""

    def __init__(self, sizes, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.sizes = list(sizes)
        g = np.random.default_rng(seed)
        self.W, self.b = [], []
        for k, n in zip(self.sizes[:-1], self.sizes[1:]):
            w = g.normal(0.0, math.sqrt(1.0 / k), size=(n, k)).astype(np.float32)
            self.W.append(torch.tensor(w, device=device))
            self.b.append(torch.zeros(n, dtype=torch.float32, device=device))
        self.device = device

    @property
    def params(self):
        return [p for pair in zip(self.W, self.b) for p in pair]

    def state(self):
        return {f"p{i}": p.detach().cpu().numpy() for i, p in enumerate(self.params)}

    def load(self, st):
        ps = self.params
        for i, p in enumerate(ps):
            p.copy_(self.torch.tensor(st[f"p{i}"], device=self.device))

    def forward(self, X, keep=False):
        from . import _bindings as B
        torch = self.torch
        lib = B.lib()
        stream = torch.cuda.current_stream().cuda_stream
        h = X.contiguous()
        acts, zs = [h], []
        L = len(self.W)
        for i, (W, b) in enumerate(zip(self.W, self.b)):
            n = W.shape[0]
            y = torch.empty((h.shape[0], n), dtype=torch.float32, device=self.device)
            z = torch.empty_like(y) if keep else None
            act = 1 if i < L - 1 else 0
            rc = lib.lrb_mlp_forward(_fp(h), h.shape[0], h.shape[1], _fp(W), _fp(b), n, act,
                                     _fp(z) if z is not None else None, _fp(y),
                                     ctypes.c_void_p(stream))
            B.check(rc, "lrb_mlp_forward")
            acts.append(y)
            zs.append(z)
            h = y
        return (h, acts, zs) if keep else h

    def backward(self, acts, zs, dY):
        """Gradients of every parameter from dLoss/dOutput."""
        from . import _bindings as B
        torch = self.torch
        lib = B.lib()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        grads = [None] * (2 * len(self.W))
        g = dY
        L = len(self.W)
        for i in range(L - 1, -1, -1):
            W = self.W[i]
            n, k = W.shape
            X = acts[i]
            M = X.shape[0]
            dZ = torch.empty((M, n), dtype=torch.float32, device=self.device)
            dW = torch.empty_like(W)
            db = torch.empty_like(self.b[i])
            dX = torch.empty((M, k), dtype=torch.float32, device=self.device) if i > 0 else None
            act = 1 if i < L - 1 else 0
            z = zs[i]
            rc = lib.lrb_mlp_backward(_fp(X), M, k, _fp(W), n, act, _fp(z), _fp(g), _fp(dZ),
                                      _fp(dW), _fp(db), _fp(dX) if dX is not None else None, stream)
            B.check(rc, "lrb_mlp_backward")
            grads[2 * i] = dW
            grads[2 * i + 1] = db
            g = dX
        return grads


def _fp(t):
    return ctypes.c_void_p(t.data_ptr())


class Adam:
    def __init__(self, params, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        import torch
        self.params = params
        self.m = [torch.zeros_like(p) for p in params]
        self.v = [torch.zeros_like(p) for p in params]
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps
        self.t = 0

    def step(self, grads, lr=None):
        from . import _bindings as B
        import torch
        self.t += 1
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        for p, g, m, v in zip(self.params, grads, self.m, self.v):
            rc = B.lib().lrb_adam(_fp(p), _fp(g), _fp(m), _fp(v), p.numel(),
                                  self.lr if lr is None else lr, self.b1, self.b2, self.eps,
                                  self.t, stream)
            B.check(rc, "lrb_adam")


def mse(Y, T, Wt, loss, inv_count=None):
    """Weighted squared error sum(w (y - t)^2) * inv_count (default 1/numel);
    returns dY and accumulates the loss into the device scalar ``loss``."""
    from . import _bindings as B
    import torch
    dY = torch.empty_like(Y)
    inv = 1.0 / Y.numel() if inv_count is None else inv_count
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = B.lib().lrb_mse(_fp(Y), _fp(T), _fp(Wt) if Wt is not None else None, Y.numel(),
                         inv, _fp(dY), _fp(loss), stream)
    B.check(rc, "lrb_mse")
    return dY


# -------------------------------------------------------------- the guess
def lowdin(S):
    """S^(1/2) and S^(-1/2) of a positive definite overlap matrix."""
    w, U = np.linalg.eigh(S)
    return (U * np.sqrt(w)) @ U.T, (U / np.sqrt(w)) @ U.T


def fractional_occupations(w, nocc, iters=200):
    """Occupations f_i = clip(w_i + mu, 0, 2) of eigenvalues w with the shift
    mu (bisection) that makes sum f = 2 nocc: the order of the eigenvalues
    is kept and every occupation lies in [0, 2]."""
    lo, hi = -float(w.max()) - 2.0, 2.0 - float(w.min())
    for _ in range(iters):
        mu = 0.5 * (lo + hi)
        if np.clip(w + mu, 0.0, 2.0).sum() > 2.0 * nocc:
            hi = mu
        else:
            lo = mu
    return np.clip(w + 0.5 * (lo + hi), 0.0, 2.0)


def density_from_lowdin(Pt, S, nocc, fractional=False):
    """Closed-shell AO density from an approximate Loewdin density.  By
    default the N/2 largest eigenvectors C of sym(Pt) give
    S^(-1/2) (2 C C^T) S^(-1/2), idempotent in the S metric (P S P = 2 P)
    with tr(P S) = 2 nocc.  With ``fractional`` the eigenvectors keep
    occupations in [0, 2] from their eigenvalues (fractional_occupations),
    so orbitals the prediction leaves near the occupation cut enter the
    first Fock build partly filled instead of being dropped; tr(P S) is
    still 2 nocc."""
    w, V = np.linalg.eigh(0.5 * (Pt + Pt.T))
    _, Sih = lowdin(S)
    if fractional:
        f = fractional_occupations(w, nocc)
        return Sih @ ((V * f) @ V.T) @ Sih
    C = V[:, len(w) - nocc:]
    return Sih @ (2.0 * C @ C.T) @ Sih


class LearnedGuess:
    """Pair model + network + normalisation; ``predict(m, S)`` gives P0.

    The network learns blocks of the Loewdin-transformed density
    P~ = S^(1/2) P S^(1/2) (eigenvalues 0 and 2).  In the raw AO basis the
    density has large, nearly unobservable components along near-null
    overlap directions (diffuse shells on neighbouring atoms) that change a
    lot between nearby geometries; P~ varies about four times less and is
    what a Fock build actually responds to.  The prediction is projected on
    the N/2 largest eigenvectors of P~ (an idempotent density with the right
    electron count) and transformed back with S^(-1/2)."""

    def __init__(self, model: PairModel, hidden=(256, 256, 256), seed=0, device="cuda"):
        self.model = model
        self.hidden = tuple(hidden)
        self.net = MLP([model.nfeat, *hidden, model.nout], seed=seed, device=device)
        self.xmu = np.zeros(model.nfeat)
        self.xsd = np.ones(model.nfeat)
        self.ymu = np.zeros((model.ntypes, model.nout))
        self.ysd = np.ones((model.ntypes, model.nout))
        self.device = device

    def applies(self, m: Molecule) -> bool:
        return self.model.applies(m)

    # data ------------------------------------------------------------
    def dataset(self, mols, dens):
        """Training arrays from molecules and their Loewdin densities P~."""
        X, Y, M, T = [], [], [], []
        for m, P in zip(mols, dens):
            ps = self.model.pairs(m)
            y, mk = self.model.to_local(m, P, ps)
            X.append(ps.X)
            Y.append(y)
            M.append(mk)
            T.append(ps.types)
        return np.concatenate(X), np.concatenate(Y), np.concatenate(M), np.concatenate(T)

    def fit_normalisation(self, X, Y, M, T):
        self.xmu = X.mean(0)
        sd = X.std(0)
        self.xsd = np.where(sd > 1e-6, sd, 1.0)
        for t in range(self.model.ntypes):
            sel = T == t
            if not sel.any():
                continue
            self.ymu[t] = Y[sel].mean(0)
            sd = Y[sel].std(0)
            self.ysd[t] = np.where(sd > 1e-8, sd, 1e-8) * M[sel][0]

    def _scaled(self, X, Y, M, T):
        xs = (X - self.xmu) / self.xsd
        ysd = self.ysd[T]
        ys = np.where(ysd > 1e-8, (Y - self.ymu[T]) / np.maximum(ysd, 1e-8), 0.0)
        w = M * (ysd > 1e-8)
        return xs, ys, w

    def train(self, X, Y, M, T, epochs=200, batch=2048, lr=1e-3, seed=0, log=None):
        """Adam on the weighted MSE of the standardised targets, all on the
        GPU; returns the per-epoch mean loss."""
        import torch
        xs, ys, w = self._scaled(X, Y, M, T)
        dev = self.device
        Xd = torch.tensor(xs, dtype=torch.float32, device=dev)
        Yd = torch.tensor(ys, dtype=torch.float32, device=dev)
        Wd = torch.tensor(w, dtype=torch.float32, device=dev)
        opt = Adam(self.net.params, lr=lr)
        n = len(xs)
        g = torch.Generator(device="cpu").manual_seed(seed)
        loss = torch.zeros(1, dtype=torch.float32, device=dev)
        hist = []
        total = epochs * ((n + batch - 1) // batch)
        step = 0
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(dev)
            loss.zero_()
            nb = 0
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                xb, yb, wb = Xd[idx].contiguous(), Yd[idx].contiguous(), Wd[idx].contiguous()
                out, acts, zs = self.net.forward(xb, keep=True)
                dY = mse(out, yb, wb, loss)
                grads = self.net.backward(acts, zs, dY)
                cur = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(total, 1)))
                opt.step(grads, lr=max(cur, lr * 0.02))
                step += 1
                nb += 1
            hist.append(float(loss.item()) / nb)
            if log and (ep % max(1, epochs // 10) == 0 or ep == epochs - 1):
                log(f"epoch {ep}: loss {hist[-1]:.4e}")
        return hist

    def predict_local(self, X, T):
        import torch
        xs = (X - self.xmu) / self.xsd
        out = self.net.forward(torch.tensor(xs, dtype=torch.float32, device=self.device))
        y = out.double().cpu().numpy()
        return self.ymu[T] + self.ysd[T] * y

    def predict(self, m: Molecule, S: np.ndarray, nelec=None, fractional=False):
        """P0 in the AO basis from the overlap matrix S of ``m`` (projected on
        the N/2 most occupied predicted orbitals, or with fractional
        occupations: density_from_lowdin)."""
        ps = self.model.pairs(m)
        Pt = self.model.to_density(m, self.predict_local(ps.X, ps.types), ps)
        return density_from_lowdin(Pt, S, (m.nelec if nelec is None else nelec) // 2,
                                   fractional=fractional)

    # persistence -----------------------------------------------------
    def save(self, path):
        st = self.net.state()
        lay = {f"layout_{z}": np.array(v, dtype=np.int64) for z, v in self.model.layouts.items()}
        lay.update({f"prims_{z}": v for z, v in self.model.prims.items()})
        np.savez_compressed(path, sizes=np.array(self.net.sizes), xmu=self.xmu, xsd=self.xsd,
                            ymu=self.ymu, ysd=self.ysd, elements=np.array(self.model.elements),
                            **lay, **st)

    @staticmethod
    def load(path, device="cuda") -> "LearnedGuess":
        f = np.load(path)
        el = [int(v) for v in f["elements"]]
        model = PairModel(el, {z: tuple(int(v) for v in f[f"layout_{z}"]) for z in el},
                          {z: f[f"prims_{z}"] for z in el if f"prims_{z}" in f.files})
        sizes = [int(v) for v in f["sizes"]]
        g = LearnedGuess(model, hidden=sizes[1:-1], device=device)
        g.xmu, g.xsd, g.ymu, g.ysd = f["xmu"], f["xsd"], f["ymu"], f["ysd"]
        g.net.load({k: f[k] for k in f.files if k.startswith("p")})
        return g
