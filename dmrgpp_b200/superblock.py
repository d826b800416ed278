"""Superblock sector descriptions and seeded synthetic generators.

A sector of the superblock Hamiltonian is described the way the GPU plugin of
DMRG++ receives it (dmrg/GPUPlugin/BatchedGemm.h:11-56,
dmrg/Engine/MatrixVectorKron/BatchedGemmPluginSc.h:50-125):

* ``npatches`` patches; patch ``p`` pairs a left symmetry group of size
  ``l[p]`` with a right group of size ``r[p]``;
* ``noperator`` Kronecker terms; term ``k`` has a block table whose entry
  ``(i, j)`` is ``A_k(i,j)`` (``l[i] x l[j]``) and ``B_k(i,j)``
  (``r[i] x r[j]``), column-major, or absent;
* the sector vector is the concatenation over patches of column-major
  ``r[p] x l[p]`` blocks (``InitKronBase.h:277-310``).

``H*x`` is ``Y_i = sum_{j,k} B_k(i,j) X_j A_k(i,j)^T``.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Optional, Tuple

import numpy as np

Block = Tuple[int, int, int]  # (i = output patch, j = input patch, k = term)


@dataclasses.dataclass
class KronProblem:
    """Block tables of one superblock sector (plugin convention)."""

    lsz: np.ndarray  # (np,) int64 left patch sizes
    rsz: np.ndarray  # (np,) int64 right patch sizes
    noperator: int
    A: Dict[Block, np.ndarray]  # (i,j,k) -> Fortran-ordered float64 l_i x l_j
    B: Dict[Block, np.ndarray]  # (i,j,k) -> Fortran-ordered float64 r_i x r_j
    name: str = "sector"

    @property
    def npatches(self) -> int:
        return int(len(self.lsz))

    @property
    def xy_start(self) -> np.ndarray:
        s = np.zeros(self.npatches + 1, dtype=np.int64)
        np.cumsum(self.lsz * self.rsz, out=s[1:])
        return s

    @property
    def dim(self) -> int:
        return int(np.sum(self.lsz * self.rsz))

    def triples(self):
        """Contributing (i,j,k): both blocks present and not all-zero
        (``setup_nC.cpp:67-121``)."""
        out = []
        for (i, j, k), a in self.A.items():
            b = self.B.get((i, j, k))
            if b is None:
                continue
            if np.any(a != 0) and np.any(b != 0):
                out.append((i, j, k))
        return sorted(out, key=lambda t: (t[0], t[1], t[2]))

    def flops(self) -> float:
        """F_alg = sum 2 r_i l_j (r_j + l_i) over contributing triples."""
        f = 0.0
        for i, j, _ in self.triples():
            f += 2.0 * self.rsz[i] * self.lsz[j] * (self.rsz[j] + self.lsz[i])
        return f

    def operator_bytes(self) -> int:
        b = 0
        for i, j, _ in self.triples():
            b += 8 * (self.lsz[i] * self.lsz[j] + self.rsz[i] * self.rsz[j])
        return int(b)

    def tables(self):
        """Flat plugin tables: lists of (array or None) and leading dims,
        indexed ``i + j*np + k*np*np``."""
        n = self.npatches
        tot = n * n * self.noperator
        A = [None] * tot
        B = [None] * tot
        ldA = np.zeros(tot, dtype=np.uint64)
        ldB = np.zeros(tot, dtype=np.uint64)
        for (i, j, k), a in self.A.items():
            b = self.B.get((i, j, k))
            if b is None:
                continue
            t = i + j * n + k * n * n
            A[t] = a
            B[t] = b
            ldA[t] = a.shape[0]
            ldB[t] = b.shape[0]
        return A, ldA, B, ldB

    def dense(self) -> np.ndarray:
        """Explicit sector matrix (small cases only): row/column order is
        the patch order of the sector vector."""
        s = self.xy_start
        D = self.dim
        H = np.zeros((D, D))
        for i, j, k in self.triples():
            a, b = self.A[(i, j, k)], self.B[(i, j, k)]
            # vec(B X A^T) = (A kron B) vec(X) for column-major vec
            H[s[i]:s[i + 1], s[j]:s[j + 1]] += np.kron(a, b)
        return H


def _sym(rng, n):
    m = rng.standard_normal((n, n))
    return np.asfortranarray(0.5 * (m + m.T))


def gaussian_sector_sizes(total: int = 1024, nsec: int = 21, sigma: float = 4.0):
    """Discretised Gaussian histogram of symmetry-sector sizes, remainder on
    the centre sector."""
    s = np.arange(nsec) - nsec // 2
    w = np.exp(-(s.astype(np.float64) ** 2) / (2.0 * sigma * sigma))
    n = np.floor(total * w / w.sum()).astype(np.int64)
    n[nsec // 2] += total - int(n.sum())
    return n


def spin_chain_like(sizes_left, sizes_right=None, seed: int = 20261203,
                    name: str = "spin-chain-like") -> KronProblem:
    """Sz-conserving superblock sector with the five Kronecker terms of a
    spin-1/2 link: H_L x I, I x H_R, Sz x Sz (block diagonal) and
    1/2 S+ x S-, 1/2 S- x S+ (nearest patches).  Patch p pairs left Sz group
    p with the right group of opposite Sz, so every patch is in the Sz=0
    superblock sector.  Entries are N(0,1) (H_L, H_R, SzSz symmetrised,
    S- blocks the transposes of S+ blocks, so H is symmetric)."""
    rng = np.random.default_rng(seed)
    l = np.asarray(sizes_left, dtype=np.int64)
    # right group of patch p has Sz = -Sz_left(p); with a symmetric histogram
    # its size equals the left one unless given explicitly
    r = l.copy() if sizes_right is None else np.asarray(sizes_right, dtype=np.int64)
    n = len(l)
    A, B = {}, {}
    for p in range(n):
        A[(p, p, 0)] = _sym(rng, l[p])
        B[(p, p, 0)] = np.asfortranarray(np.eye(r[p]))
        A[(p, p, 1)] = np.asfortranarray(np.eye(l[p]))
        B[(p, p, 1)] = _sym(rng, r[p])
        A[(p, p, 2)] = _sym(rng, l[p])
        B[(p, p, 2)] = _sym(rng, r[p])
    for p in range(n - 1):
        q = p + 1
        sp = rng.standard_normal((l[q], l[p]))  # S+ on the left: group p -> p+1
        sm = rng.standard_normal((r[q], r[p]))  # S- on the right
        A[(q, p, 3)] = np.asfortranarray(0.5 * sp)
        B[(q, p, 3)] = np.asfortranarray(sm)
        A[(p, q, 4)] = np.asfortranarray(0.5 * sp.T)
        B[(p, q, 4)] = np.asfortranarray(sm.T)
    return KronProblem(l, r, 5, A, B, name=name)


def spin_chain_dominant(sizes, seed: int = 20261203, mixing: float = 0.15,
                        name: str = "spin-chain-diagonal-dominant") -> KronProblem:
    """Like spin_chain_like, but with block Hamiltonians close to diagonal in
    their own basis (sorted level energies plus weak N(0, mixing^2) mixing)
    and weaker boundary couplings, as for blocks expressed in bases close to
    their energy eigenstates; the diagonal of H then carries the spectrum."""
    p = spin_chain_like(sizes, seed=seed, name=name)
    rng = np.random.default_rng(seed + 1)
    for (i, j, k), a in list(p.A.items()):
        if k == 0:   # H_L (x) I
            n = a.shape[0]
            h = np.diag(np.sort(rng.uniform(-4.0, 4.0, n))) + mixing * _sym(rng, n)
            p.A[(i, j, k)] = np.asfortranarray(h)
        elif k == 1:  # I (x) H_R
            n = p.B[(i, j, k)].shape[0]
            h = np.diag(np.sort(rng.uniform(-4.0, 4.0, n))) + mixing * _sym(rng, n)
            p.B[(i, j, k)] = np.asfortranarray(h)
        else:        # S.S couplings across the boundary
            p.A[(i, j, k)] = np.asfortranarray(0.3 * a)
    # keep S- = (S+)^T after the rescaling
    for (i, j, k) in list(p.A):
        if k == 4:
            p.A[(i, j, 4)] = np.asfortranarray(p.A[(j, i, 3)].T)
    return p


def c2_problem(seed: int = 20261203) -> KronProblem:
    """Synthetic Kronecker-matvec microbench: left = right = 1024 states in 21
    Sz groups (discretised Gaussian, sigma = 4 groups), K = 5 terms,
    D = 76,406, 103 contributing (i,j,k) triples, F_alg = 0.130 GFLOP."""
    sizes = gaussian_sector_sizes(1024, 21, 4.0)
    return spin_chain_like(sizes, seed=seed, name="kron-microbench-1024x1024-21sec-K5")


def random_problem(npatches: int, noperator: int, max_size: int = 12, seed: int = 0,
                   density: float = 0.5, zero_block_rate: float = 0.1,
                   symmetric: bool = False, min_size: int = 1,
                   name: str = "random") -> KronProblem:
    """Ragged random sector for parity tests: uneven patch sizes (including 1),
    missing blocks, present-but-all-zero blocks (which must not contribute),
    and different left/right sizes."""
    rng = np.random.default_rng(seed)
    l = rng.integers(min_size, max_size + 1, size=npatches).astype(np.int64)
    r = rng.integers(min_size, max_size + 1, size=npatches).astype(np.int64)
    A, B = {}, {}
    for k in range(noperator):
        for i in range(npatches):
            for j in range(npatches):
                if symmetric and j > i:
                    continue
                if i != j and rng.random() > density:
                    continue
                a = rng.standard_normal((l[i], l[j]))
                b = rng.standard_normal((r[i], r[j]))
                z = rng.random()
                if z < zero_block_rate / 2:
                    a[:] = 0.0
                elif z < zero_block_rate:
                    b[:] = 0.0
                if symmetric and i == j:
                    a = 0.5 * (a + a.T)
                    b = 0.5 * (b + b.T)
                A[(i, j, k)] = np.asfortranarray(a)
                B[(i, j, k)] = np.asfortranarray(b)
                if symmetric and i != j:
                    A[(j, i, k)] = np.asfortranarray(a.T)
                    B[(j, i, k)] = np.asfortranarray(b.T)
    return KronProblem(l, r, noperator, A, B, name=name)


def random_unit_vector(dim: int, seed: int = 1) -> np.ndarray:
    v = np.random.default_rng(seed).standard_normal(dim)
    return v / np.linalg.norm(v)


def ladder_problem(total_states: int = 16000, sigma: float = 2.5, seed: int = 20261203,
                   min_group: int = 1, name: str = "", legs: int = 2) -> KronProblem:
    """Sector shaped like a two-leg Hubbard ladder superblock at m ~ 4000
    (left and right blocks of `total_states` states each, 4 states per site).
    Left groups are (N_up, N_down) pairs whose sizes follow a 2-D discretised
    Gaussian (width sigma in particle number); patch p pairs left group
    (nu, nd) with the right group that completes the target (N_up, N_down),
    whose size follows the same histogram.  K = 10 terms: H_L x I, I x H_R and
    8 hopping terms c^dag_{s,leg} x c_{s,leg} (2 spins x 2 legs x 2
    directions), each moving one particle of one spin across the boundary,
    so it couples patches whose (nu, nd) differ by one.  Blocks are dense
    N(0,1) (H_L, H_R symmetrised; the two directions are transposes), the
    synthetic stand-in for operators of a real sweep.  legs=1 gives the
    Hubbard-chain shape (K = 6: 4 hopping terms)."""
    rng = np.random.default_rng(seed)
    R = int(np.ceil(4 * sigma))
    qs = [(a, b) for a in range(-R, R + 1) for b in range(-R, R + 1)]
    w = np.array([np.exp(-(a * a + b * b) / (2 * sigma * sigma)) for a, b in qs])
    n = np.floor(total_states * w / w.sum()).astype(np.int64)
    n[np.argmax(w)] += total_states - int(n.sum())
    keep = [i for i in range(len(qs)) if n[i] >= min_group]
    qs = [qs[i] for i in keep]
    n = n[keep]
    index = {q: p for p, q in enumerate(qs)}
    l = n.copy()
    r = np.array([n[index[(-a, -b)]] for a, b in qs], dtype=np.int64)
    A, B = {}, {}
    for p in range(len(qs)):
        A[(p, p, 0)] = _sym(rng, l[p])
        B[(p, p, 0)] = np.asfortranarray(np.eye(r[p]))
        A[(p, p, 1)] = np.asfortranarray(np.eye(l[p]))
        B[(p, p, 1)] = _sym(rng, r[p])
    k = 2
    for spin in range(2):
        for leg in range(legs):
            for p, (a, b) in enumerate(qs):
                q_to = (a + 1, b) if spin == 0 else (a, b + 1)
                if q_to not in index:
                    continue
                q = index[q_to]
                cd = rng.standard_normal((l[q], l[p]))  # c^dag on the left: p -> q
                c = rng.standard_normal((r[q], r[p]))   # c on the right
                A[(q, p, k)] = np.asfortranarray(cd)
                B[(q, p, k)] = np.asfortranarray(c)
                A[(p, q, k + 1)] = np.asfortranarray(cd.T)
                B[(p, q, k + 1)] = np.asfortranarray(c.T)
            k += 2
    K = 2 + 4 * legs
    shape = "ladder" if legs == 2 else ("chain" if legs == 1 else f"{legs}leg")
    return KronProblem(l, r, K, A, B,
                       name=name or f"hubbard-{shape}-like-{total_states}x{total_states}-"
                                    f"{len(qs)}sec-K{K}")


def serving_batch(nproblems: int = 256, seed: int = 20261203):
    """Independent superblock sectors shaped like a serving-style batch of
    ground-state problems: Heisenberg and Hubbard chains (half each, seeded
    coin) with L uniform in [16, 48], U uniform in [0, 8] for Hubbard and m
    drawn from {64, 128, 256, 512}.  Heisenberg: left and right blocks of 2m
    states in 2 round(sqrt(L/2)) + 1 Sz groups (discretised Gaussian), K = 5
    (spin_chain_like).  Hubbard: blocks of 4m states in (N_up, N_down)
    groups of width 1 + L/32, K = 6 (ladder_problem with one leg), with U
    times a seeded double-occupancy count added to the diagonal of H_L and
    H_R.  Seeded N(0,1) blocks stand in for the operators of real sweeps.
    Returns the list of KronProblem and a list of dicts describing them."""
    rng = np.random.default_rng(seed)
    probs, meta = [], []
    for q in range(nproblems):
        L = int(rng.integers(16, 49))
        m = int(rng.choice([64, 128, 256, 512]))
        sub = int(rng.integers(0, 2**31 - 1))
        if rng.random() < 0.5:
            nsec = 2 * int(round(np.sqrt(L / 2))) + 1
            sizes = gaussian_sector_sizes(2 * m, nsec, nsec / 5.0)
            sizes = sizes[sizes > 0]
            p = spin_chain_like(sizes, seed=sub, name=f"heisenberg-L{L}-m{m}")
            meta.append({"model": "heisenberg", "L": L, "m": m})
        else:
            U = float(rng.uniform(0.0, 8.0))
            p = ladder_problem(total_states=4 * m, sigma=1.0 + L / 32.0, seed=sub, legs=1,
                               name=f"hubbard-L{L}-m{m}-U{U:.2f}")
            r2 = np.random.default_rng(sub + 1)
            for pi in range(p.npatches):
                a = p.A[(pi, pi, 0)]
                p.A[(pi, pi, 0)] = np.asfortranarray(
                    a + U * np.diag(r2.integers(0, max(2, L // 4), a.shape[0]).astype(float)))
                b = p.B[(pi, pi, 1)]
                p.B[(pi, pi, 1)] = np.asfortranarray(
                    b + U * np.diag(r2.integers(0, max(2, L // 4), b.shape[0]).astype(float)))
            meta.append({"model": "hubbard", "L": L, "m": m, "U": U})
        probs.append(p)
    return probs, meta
