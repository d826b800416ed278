"""Superblock sectors of real DMRG steps with their super-basis permutation,
for the sector gather index (dmrgpp_kron_gather_index) tests.

The enlarged left and right blocks come from the oracle's two-site DMRG driver
(Heisenberg and Hubbard chains, quantum-number groups), the patches are the
driver's GenIjPatch pairs for the target, and the permutation is the
superblock product of Basis::setToProduct (oracle/superbasis.py)."""
import numpy as np

from oracle import dmrg_driver as dd
from oracle import superbasis


def sector_case(model: str, L: int, m: int, steps: int):
    """Runs `steps` infinite-growth steps and returns the next step's sector:
    dict(prob, patch_left, patch_right, left_partition, right_partition,
    perm_inverse, offset, size)."""
    mdl = dd.Heisenberg() if model == "heisenberg" else dd.Hubbard(U=4.0)
    solver = dd.dense_solver()
    drv = dd.DMRG(mdl, L, m, solver)
    b_l = b_r = drv.site
    for n in range(1, steps + 1):
        e, lp, rp, rl, rr = drv.step(b_l, b_r, 2 * (n + 1))
        b_l, b_r = drv.truncate(lp, rl), drv.truncate(rp, rr)
    lp, rp = drv.grow_left(b_l), drv.grow_right(b_r)
    target = mdl.target(2 * (steps + 2))
    prob, patches = drv.superblock(lp, rp, target)
    perm, sectors = superbasis.product_permutation(lp.qns, lp.sizes, rp.qns, rp.sizes)
    offset, size = sectors[target]
    assert size == prob.dim
    return dict(prob=prob, left_qns=lp.qns, right_qns=rp.qns, target=target,
                patch_left=[gl for gl, _ in patches],
                patch_right=[gr for _, gr in patches],
                left_partition=np.concatenate([[0], np.cumsum(lp.sizes)]).astype(np.uint64),
                right_partition=np.concatenate([[0], np.cumsum(rp.sizes)]).astype(np.uint64),
                perm_inverse=perm, offset=offset, size=size)


CASES = [("heisenberg", 12, 16, 3), ("heisenberg", 16, 24, 5), ("hubbard", 8, 24, 2),
         ("hubbard", 10, 32, 3)]
