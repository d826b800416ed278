"""Minimal two-site DMRG driver (spin-1/2 Heisenberg and Fermi-Hubbard chains)
that produces real superblock sectors in the plugin's table format and hands
each sector eigensolve to a pluggable solver.

TEST INFRASTRUCTURE (oracle): used by tests/ to run whole DMRG calculations
with the compiled reference solver (oracle.RefKron: the reference's
PsimagLite::LanczosSolver over Dmrg::BatchedGemmCpu) or with the CUDA
library, and to compare energies with the reference's own published results
(dmrg/CMakeLists.txt:343-344, input3100: Heisenberg L=32 OBC, -13.9973 within
2e-5; dmrg/CMakeLists.txt:180-181, input2_batchedgemm: Hubbard L=8 U=0,
-9.51754).  Nothing in dmrgpp_b200/ imports it.

The algorithm restates the reference's two-site scheme: blocks grow by one
site (Basis::setToProduct, dmrg/Engine/Basis.h:162-...), states are grouped
by conserved quantum numbers (Sz, or (N_up, N_down)), the superblock sector
pairs every left group with the right group that completes the target
(GenIjPatch.h:104-118), H = H_L x I + I x H_R + sum over the central link
(InitKronHamiltonian.h:242-283; fermion signs as in
InitKronBase::calculateAhat, InitKronBase.h:393-413: the left operator of a
link carries the left block's parity), and blocks are truncated to the m
eigenvectors of the reduced density matrix with the largest weights
(DensityMatrixSvd.h:285-391, Truncation.h:245-256): infinite-system growth to
L sites, then finite sweeps.

Operators are block-sparse by quantum number: {(out_group, in_group): dense}.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from dmrgpp_b200.superblock import KronProblem

BlockOp = Dict[Tuple[int, int], np.ndarray]


class KeptBasis(dict):
    """{group: U_g (group size x kept)}: the kept eigenvectors of a block's
    reduced density matrix chosen outside the driver (DMRG.truncator)."""


@dataclass
class Block:
    """A block of sites: quantum-number groups (sorted), their sizes, and
    block-sparse operators (H, the edge-site operators, the parity)."""
    qns: List[tuple]
    sizes: List[int]
    ops: Dict[str, BlockOp] = field(default_factory=dict)
    length: int = 1

    def index(self):
        return {q: g for g, q in enumerate(self.qns)}


def _add(a, b):
    return tuple(x + y for x, y in zip(a, b))


def _sub(a, b):
    return tuple(x - y for x, y in zip(a, b))


# ------------------------------------------------------------------ models
class Heisenberg:
    """Spin-1/2 Heisenberg chain, H = J sum S_i.S_{i+1}, open boundaries;
    quantum number (2 Sz,)."""

    def __init__(self, J: float = 1.0):
        self.J = J

    def site(self) -> Block:
        # groups: (-1,): down, (+1,): up
        sz = {(0, 0): np.array([[-0.5]]), (1, 1): np.array([[0.5]])}
        sp = {(1, 0): np.array([[1.0]])}          # S+ |down> = |up>
        return Block([(-1,), (1,)], [1, 1], {"H": {}, "Sz": sz, "Sp": sp}, 1)

    def edge_names(self):
        return ["Sz", "Sp"]

    def links(self, left_edge, right_edge, left_parity):
        """(coefficient, left operator, right operator) of the central link:
        J [Sz Sz + 1/2 (S+ S- + S- S+)]."""
        sm_l = transpose(left_edge["Sp"])
        sm_r = transpose(right_edge["Sp"])
        return [(self.J, left_edge["Sz"], right_edge["Sz"]),
                (0.5 * self.J, left_edge["Sp"], sm_r),
                (0.5 * self.J, sm_l, right_edge["Sp"])]

    def target(self, L: int):
        return (0,)


class Hubbard:
    """Fermi-Hubbard chain, H = -t sum_{i,s} (c+_{i,s} c_{i+1,s} + h.c.)
    + U sum_i n_{i,up} n_{i,down}, open boundaries; quantum number
    (N_up, N_down); Jordan-Wigner order: sites left to right, up before down
    on a site."""

    def __init__(self, t: float = 1.0, U: float = 0.0, n_up: int = None, n_dn: int = None):
        self.t, self.U, self.n_up, self.n_dn = t, U, n_up, n_dn

    def site(self) -> Block:
        # groups (states): (0,0): |0>, (0,1): |dn>, (1,0): |up>, (1,1): |up dn>
        qns = [(0, 0), (0, 1), (1, 0), (1, 1)]
        g = {q: i for i, q in enumerate(qns)}
        one = np.array([[1.0]])
        # c_up: |up> -> |0>, |up dn> -> |dn>  (up is first in the site's order)
        cu = {(g[(0, 0)], g[(1, 0)]): one.copy(), (g[(0, 1)], g[(1, 1)]): one.copy()}
        # c_dn: |dn> -> |0>, |up dn> -> -|up> (passes the up fermion)
        cd = {(g[(0, 0)], g[(0, 1)]): one.copy(), (g[(1, 0)], g[(1, 1)]): -one.copy()}
        par = {(i, i): np.array([[(-1.0) ** (q[0] + q[1])]]) for i, q in enumerate(qns)}
        H = {(g[(1, 1)], g[(1, 1)]): np.array([[self.U]])} if self.U != 0.0 else {}
        return Block(qns, [1, 1, 1, 1], {"H": H, "Cu": cu, "Cd": cd, "P": par}, 1)

    def edge_names(self):
        return ["Cu", "Cd"]

    def links(self, left_edge, right_edge, left_parity):
        """-t sum_s (c+_l c_r + c+_r c_l) with the left block's parity on the
        left operator: c+_l c_r = (c+_l P_L) x c_r, c+_r c_l = (P_L c_l) x c+_r."""
        out = []
        for name in ("Cu", "Cd"):
            cl, cr = left_edge[name], right_edge[name]
            out.append((-self.t, matmul(transpose(cl), left_parity), cr))
            out.append((-self.t, matmul(left_parity, cl), transpose(cr)))
        return out

    def target(self, L: int):
        nu = self.n_up if self.n_up is not None else L // 2
        nd = self.n_dn if self.n_dn is not None else L // 2
        return (nu, nd)


class HubbardLadder(Hubbard):
    """Two-leg Fermi-Hubbard ladder, H = -t_leg sum_leg - t_rung sum_rung
    sum_s (c+_i,s c_j,s + h.c.) + U sum_i n_i,up n_i,down, open boundaries,
    in the reference's site order (PsimagLite/src/PsimagLite/Geometry/
    Ladder.h:87-292, LadderLeg=2): site i sits on rung i // 2 and leg i % 2;
    sites on one rung (i, i+1 with i even) and on one leg two apart (i, i+2)
    are connected.  Blocks grow one site at a time along that order, so each
    block carries the operators of its last two sites (depth 2).  Quantum
    number (N_up, N_down); the target of an N-site stage is the full
    system's filling scaled to N sites (rounded)."""

    depth = 2

    def __init__(self, Lx: int, t_leg: float = 1.0, t_rung: float = 1.0, U: float = 0.0,
                 n_up: int = None, n_dn: int = None):
        super().__init__(t=t_leg, U=U, n_up=n_up, n_dn=n_dn)
        self.Lx, self.t_leg, self.t_rung = Lx, t_leg, t_rung

    @staticmethod
    def connected(i: int, j: int) -> bool:
        ci, cj, ri, rj = i // 2, j // 2, i % 2, j % 2
        if ci == cj:
            return abs(ri - rj) == 1
        return ri == rj and abs(ci - cj) == 1

    def link_terms(self, left_edge, right_edge, left_parity, i: int, j: int):
        t = self.t_rung if i // 2 == j // 2 else self.t_leg
        out = []
        for name in ("Cu", "Cd"):
            cl, cr = left_edge[name], right_edge[name]
            out.append((-t, matmul(transpose(cl), left_parity), cr))
            out.append((-t, matmul(left_parity, cl), transpose(cr)))
        return out

    def bonds(self):
        """(i, j, t) of every connected pair, i < j (for exact checks)."""
        L = 2 * self.Lx
        return [(i, j, self.t_rung if i // 2 == j // 2 else self.t_leg)
                for i in range(L) for j in range(i + 1, L) if self.connected(i, j)]

    def target(self, N: int):
        L = 2 * self.Lx
        nu = self.n_up if self.n_up is not None else L // 2
        nd = self.n_dn if self.n_dn is not None else L // 2
        return (int(np.floor(nu * N / L + 0.5)), int(np.floor(nd * N / L + 0.5)))


# ---------------------------------------------------- block-sparse algebra
def transpose(a: BlockOp) -> BlockOp:
    return {(j, i): m.T.copy() for (i, j), m in a.items()}


def matmul(a: BlockOp, b: BlockOp) -> BlockOp:
    out: BlockOp = {}
    by_row = {}
    for (k, j), m in b.items():
        by_row.setdefault(k, []).append((j, m))
    for (i, k), ma in a.items():
        for j, mb in by_row.get(k, []):
            p = ma @ mb
            out[(i, j)] = out[(i, j)] + p if (i, j) in out else p
    return out


def scale(a: BlockOp, c: float) -> BlockOp:
    return {k: c * m for k, m in a.items()}


def add_into(acc: BlockOp, a: BlockOp, c: float = 1.0) -> None:
    for k, m in a.items():
        acc[k] = acc[k] + c * m if k in acc else c * m


def identity(blk: Block) -> BlockOp:
    return {(g, g): np.eye(n) for g, n in enumerate(blk.sizes)}


def product_basis(first: Block, second: Block):
    """Groups of first (x) second: for every new quantum number, the list of
    (group of first, group of second, offset) segments, first-group major;
    a state (a, b) of segment (g1, g2) sits at offset + a * size(g2) + b."""
    segs: Dict[tuple, list] = {}
    for g1, q1 in enumerate(first.qns):
        for g2, q2 in enumerate(second.qns):
            segs.setdefault(_add(q1, q2), []).append((g1, g2))
    qns = sorted(segs)
    layout, sizes = [], []
    for q in qns:
        off, lst = 0, []
        for g1, g2 in segs[q]:
            lst.append((g1, g2, off))
            off += first.sizes[g1] * second.sizes[g2]
        layout.append(lst)
        sizes.append(off)
    return qns, sizes, layout


def kron_op(a: BlockOp, b: BlockOp, qns, sizes, layout) -> BlockOp:
    """(a x b) in the product basis: element [(a', b'), (a, b)] = a[a', a] b[b', b]."""
    where = {}
    for g, lst in enumerate(layout):
        for g1, g2, off in lst:
            where[(g1, g2)] = (g, off)
    out: BlockOp = {}
    for (i1, j1), ma in a.items():
        for (i2, j2), mb in b.items():
            if (i1, i2) not in where or (j1, j2) not in where:
                continue
            go, oo = where[(i1, i2)]
            gi, oi = where[(j1, j2)]
            blk = out.get((go, gi))
            if blk is None:
                blk = np.zeros((sizes[go], sizes[gi]))
                out[(go, gi)] = blk
            k = np.kron(ma, mb)
            blk[oo:oo + k.shape[0], oi:oi + k.shape[1]] += k
    return out


# ------------------------------------------------------------ DMRG pieces
class DMRG:
    """Two-site DMRG with a pluggable sector solver.

    solver(problem: KronProblem, init: ndarray) -> (energy, vector, steps)
    """

    def __init__(self, model, L: int, m: int, solver: Callable, seed: int = 7):
        self.model, self.L, self.m, self.solver = model, L, m, solver
        self.rng = np.random.default_rng(seed)
        self.site = model.site()
        self.energies: List[float] = []
        self.sectors: List[KronProblem] = []
        self.keep_sectors = False
        # optional (prob, patches, psi, side, enlarged block, m) -> KeptBasis
        # (side 0: the left block, 1: the right block) in place of the
        # driver's own density-matrix truncation
        self.truncator: Optional[Callable] = None

    # boundary sites: chains couple nearest neighbours only (one boundary site
    # per block); the two-leg ladder also couples sites two apart, so its
    # blocks carry the operators of their last two sites (slot 0: the
    # outermost site, slot 1: the one before it, names suffixed "~1")
    def _depth(self) -> int:
        return getattr(self.model, "depth", 1)

    def _connected(self, i: int, j: int) -> bool:
        f = getattr(self.model, "connected", None)
        return f(i, j) if f is not None else abs(i - j) == 1

    def _link_terms(self, lops, rops, parity, i: int, j: int):
        f = getattr(self.model, "link_terms", None)
        return f(lops, rops, parity, i, j) if f is not None else self.model.links(lops, rops, parity)

    def _slot(self, blk: Block, d: int):
        if d == 0:
            return blk.ops
        return {n: blk.ops[f"{n}~{d}"] for n in self.model.edge_names()}

    # enlarge a left block (sites 0 .. k-1) by site k on its right
    def grow_left(self, b: Block) -> Block:
        s = self.site
        k = b.length
        qns, sizes, layout = product_basis(b, s)
        H = kron_op(b.ops["H"], identity(s), qns, sizes, layout)
        add_into(H, kron_op(identity(b), s.ops["H"], qns, sizes, layout))
        parity = b.ops.get("P")
        for d in range(min(self._depth(), b.length)):
            if self._connected(k - 1 - d, k):
                for c, lo, ro in self._link_terms(self._slot(b, d), s.ops, parity, k - 1 - d, k):
                    add_into(H, kron_op(lo, ro, qns, sizes, layout), c)
        ops = {"H": H}
        for name in self.model.edge_names():   # the new site is the edge
            left = parity if parity is not None else identity(b)
            ops[name] = kron_op(left, s.ops[name], qns, sizes, layout)
            for d in range(1, min(self._depth(), b.length + 1)):
                ops[f"{name}~{d}"] = kron_op(self._slot(b, d - 1)[name], identity(s), qns, sizes,
                                             layout)
        if parity is not None:
            ops["P"] = kron_op(parity, s.ops["P"], qns, sizes, layout)
        return Block(qns, sizes, ops, b.length + 1)

    # enlarge a right block (the last sites of an N-site system) by the site
    # on its left
    def grow_right(self, b: Block, N: int = 0) -> Block:
        s = self.site
        k = N - b.length - 1                    # the new site's index
        qns, sizes, layout = product_basis(s, b)
        H = kron_op(identity(s), b.ops["H"], qns, sizes, layout)
        add_into(H, kron_op(s.ops["H"], identity(b), qns, sizes, layout))
        sp = s.ops.get("P")
        for d in range(min(self._depth(), b.length)):
            if self._connected(k, k + 1 + d):
                for c, lo, ro in self._link_terms(s.ops, self._slot(b, d), sp, k, k + 1 + d):
                    add_into(H, kron_op(lo, ro, qns, sizes, layout), c)
        ops = {"H": H}
        for name in self.model.edge_names():   # the new site is the edge
            ops[name] = kron_op(s.ops[name], identity(b), qns, sizes, layout)
            for d in range(1, min(self._depth(), b.length + 1)):
                left = sp if sp is not None else identity(s)
                ops[f"{name}~{d}"] = kron_op(left, self._slot(b, d - 1)[name], qns, sizes, layout)
        if sp is not None:
            ops["P"] = kron_op(sp, b.ops["P"], qns, sizes, layout)
        return Block(qns, sizes, ops, b.length + 1)

    def superblock(self, left: Block, right: Block, target, N: int = 0) -> Tuple[KronProblem, list]:
        """Sector `target` of left (x) right (an N-site system) as plugin tables."""
        ridx = right.index()
        patches = []
        for gl, ql in enumerate(left.qns):
            qr = _sub(target, ql)
            if qr in ridx:
                patches.append((gl, ridx[qr]))
        pidx_l = {gl: p for p, (gl, _) in enumerate(patches)}
        lsz = np.array([left.sizes[gl] for gl, _ in patches], dtype=np.int64)
        rsz = np.array([right.sizes[gr] for _, gr in patches], dtype=np.int64)
        terms = [(1.0, left.ops["H"], identity(right)), (1.0, identity(left), right.ops["H"])]
        N = N or (left.length + right.length)
        for d in range(min(self._depth(), left.length)):
            for e in range(min(self._depth(), right.length)):
                i, j = left.length - 1 - d, N - right.length + e
                if self._connected(i, j):
                    terms += self._link_terms(self._slot(left, d), self._slot(right, e),
                                              left.ops.get("P"), i, j)
        A, B = {}, {}
        for k, (c, lo, ro) in enumerate(terms):
            for (gi, gj), a in lo.items():
                if gi not in pidx_l or gj not in pidx_l:
                    continue
                pi, pj = pidx_l[gi], pidx_l[gj]
                b = ro.get((patches[pi][1], patches[pj][1]))
                if b is None:
                    continue
                A[(pi, pj, k)] = np.asfortranarray(c * a)
                B[(pi, pj, k)] = np.asfortranarray(b)
        prob = KronProblem(lsz, rsz, len(terms), A, B,
                           name=f"dmrg-superblock-{left.length}+{right.length}")
        return prob, patches

    def truncate(self, blk: Block, rho) -> Block:
        """Keep the m largest-weight eigenvectors of the block-diagonal
        reduced density matrix (DensityMatrixSvd.h:285-391); rho is either
        {group: rho_g} or a KeptBasis chosen by an external truncation."""
        if isinstance(rho, KeptBasis):
            U = {g: u for g, u in rho.items() if u.shape[1] > 0}
        else:
            evals, evecs = [], {}
            for g, r in rho.items():
                w, v = np.linalg.eigh(0.5 * (r + r.T))
                evecs[g] = (w, v)
                evals += [(wi, g, i) for i, wi in enumerate(w)]
            evals.sort(key=lambda t: -t[0])
            kept: Dict[int, List[int]] = {}
            for wi, g, i in evals[:self.m]:
                kept.setdefault(g, []).append(i)
            U = {g: evecs[g][1][:, sorted(kept[g])] for g in sorted(kept)}
        groups = sorted(U)
        newi = {g: n for n, g in enumerate(groups)}
        ops = {}
        for name, op in blk.ops.items():
            t: BlockOp = {}
            for (i, j), mtx in op.items():
                if i in newi and j in newi:
                    t[(newi[i], newi[j])] = U[i].T @ mtx @ U[j]
            ops[name] = t
        return Block([blk.qns[g] for g in groups], [U[g].shape[1] for g in groups], ops,
                     blk.length)

    def step(self, left: Block, right: Block, sites: int):
        """One superblock solve: enlarge both, solve the target sector,
        return (energy, enlarged left, enlarged right, rho_L, rho_R)."""
        lp, rp = self.grow_left(left), self.grow_right(right, sites)
        target = self.model.target(sites)
        prob, patches = self.superblock(lp, rp, target, sites)
        init = self.rng.standard_normal(prob.dim)
        e, psi, _ = self.solver(prob, init)
        psi = np.asarray(psi)
        self.energies.append(float(e))
        if self.keep_sectors:
            self.sectors.append(prob)
        if self.truncator is not None:
            return (float(e), lp, rp, self.truncator(prob, patches, psi, 0, lp, self.m),
                    self.truncator(prob, patches, psi, 1, rp, self.m))
        rho_l, rho_r = {}, {}
        xs = prob.xy_start
        for p, (gl, gr) in enumerate(patches):
            X = psi[xs[p]:xs[p + 1]].reshape(int(prob.lsz[p]), int(prob.rsz[p])).T  # r x l
            rho_l[gl] = rho_l.get(gl, 0.0) + X.T @ X
            rho_r[gr] = rho_r.get(gr, 0.0) + X @ X.T
        return float(e), lp, rp, rho_l, rho_r

    def run(self, sweeps: int = 2) -> float:
        """Infinite-system growth to L sites, then `sweeps` finite sweeps
        (each left-to-right then right-to-left); returns the last energy."""
        L = self.L
        left = {1: self.site}
        right = {1: self.site}
        b_l, b_r = self.site, self.site
        n = 1
        while 2 * (n + 1) <= L:
            e, lp, rp, rl, rr = self.step(b_l, b_r, 2 * (n + 1))
            b_l, b_r = self.truncate(lp, rl), self.truncate(rp, rr)
            n += 1
            left[n], right[n] = b_l, b_r
        for _ in range(sweeps):
            # left to right: the left block grows, the right block shrinks
            for nl in range(L // 2, L - 2):
                e, lp, rp, rl, rr = self.step(left[nl], right[L - nl - 2], L)
                left[nl + 1] = self.truncate(lp, rl)
            # right to left
            for nr in range(1, L - 2):
                e, lp, rp, rl, rr = self.step(left[L - nr - 2], right[nr], L)
                right[nr + 1] = self.truncate(rp, rr)
            # back to the middle
            for nl in range(1, L // 2):
                e, lp, rp, rl, rr = self.step(left[nl], right[L - nl - 2], L)
                left[nl + 1] = self.truncate(lp, rl)
        return self.energies[-1]


# ----------------------------------------------------------------- solvers
def reference_solver(tolerance: float = 1e-12, steps: int = 200):
    """Sector solve by the reference's own LanczosSolver over BatchedGemmCpu
    (compiled into oracle/_ref)."""
    import oracle

    def solve(prob, init):
        rk = oracle.RefKron(prob)
        return rk.lanczos(init, steps=steps, min_steps=4, tolerance=tolerance, reortho=True)
    return solve


def dense_solver():
    """Exact lowest eigenpair of the sector by dense diagonalisation (small
    superblocks only)."""
    def solve(prob, init):
        w, v = np.linalg.eigh(prob.dense())
        return float(w[0]), v[:, 0], 0
    return solve


def free_fermion_energy(L: int, n_up: int, n_dn: int, t: float = 1.0) -> float:
    """Exact U=0 open-chain energy: fill the lowest single-particle levels
    -2t cos(k pi / (L+1))."""
    lev = np.sort(-2.0 * t * np.cos(np.arange(1, L + 1) * np.pi / (L + 1)))
    return float(lev[:n_up].sum() + lev[:n_dn].sum())


def hubbard_ed(L: int, U: float, n_up: int, n_dn: int, t: float = 1.0, bonds=None) -> float:
    """Lowest energy of the open Hubbard chain (or of the lattice given by
    bonds, (i, j, t) per connected pair) by diagonalising H in the
    fixed-(N_up, N_down) Fock space built directly from creation and
    annihilation operators (modes site-major, up before down), independent
    of the block construction above (small L only)."""
    modes = 2 * L
    up_mask = sum(1 << (2 * s) for s in range(L))
    dn_mask = sum(1 << (2 * s + 1) for s in range(L))
    states = [s for s in range(1 << modes)
              if bin(s & up_mask).count("1") == n_up and bin(s & dn_mask).count("1") == n_dn]
    idx = {s: i for i, s in enumerate(states)}
    H = np.zeros((len(states), len(states)))

    def hop(s, i, j):  # c+_i c_j |s>
        if not (s >> j) & 1:
            return None, 0
        sign = (-1) ** bin(s & ((1 << j) - 1)).count("1")
        s2 = s ^ (1 << j)
        if (s2 >> i) & 1:
            return None, 0
        sign *= (-1) ** bin(s2 & ((1 << i) - 1)).count("1")
        return s2 | (1 << i), sign

    for s in states:
        for site in range(L):
            if (s >> (2 * site)) & 1 and (s >> (2 * site + 1)) & 1:
                H[idx[s], idx[s]] += U
        for si, sj, tb in (bonds if bonds is not None else [(q, q + 1, t) for q in range(L - 1)]):
            for sp in range(2):
                a, b = 2 * si + sp, 2 * sj + sp
                for i, j in ((a, b), (b, a)):
                    s2, sg = hop(s, i, j)
                    if s2 is not None:
                        H[idx[s2], idx[s]] += -tb * sg
    return float(np.linalg.eigvalsh(H)[0])
