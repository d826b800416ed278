"""dmrgpp_kron_create_crs on the GPU: a sector built on the device from its
CRS operators is the handle dmrgpp_kron_create builds from the same blocks as
dense tables (H*x bitwise equal, FP64 and TF32x3), within 1e-12 of the
oracle, and the same holds for real superblock sectors of a DMRG run."""
import numpy as np
import pytest

from crs_cases import random_crs_case
from oracle import crs_oracle

pytestmark = pytest.mark.gpu


def _pair(c, precision):
    from dmrgpp_b200 import plugin
    prob = crs_oracle.problem_from_crs(c["loff"], c["lsz"], c["roff"], c["rsz"], c["A"], c["B"],
                                       c["value"], c["fermion"], c["parity"])
    dense = plugin.BatchedGemm.from_problem(prob, precision=precision)
    crs = plugin.BatchedGemm.from_crs(c["loff"], c["lsz"], c["roff"], c["rsz"], c["A"], c["B"],
                                      value=c["value"], fermion=c["fermion"],
                                      left_parity=c["parity"], precision=precision)
    return prob, dense, crs


@pytest.mark.parametrize("seed,ngroups,maxg,K", [(1, 5, 30, 5), (2, 7, 70, 6), (3, 3, 150, 4),
                                                 (4, 9, 12, 7), (6, 2, 1, 3)])
def test_crs_handle_equals_dense_handle(cuda_lib, cuda_device, oracle_built, seed, ngroups, maxg, K):
    import torch
    from dmrgpp_b200 import plugin
    c = random_crs_case(seed, ngroups=ngroups, maxg=maxg, K=K)
    for precision in (plugin.FP64, plugin.TF32X3):
        prob, dense, crs = _pair(c, precision)
        assert crs.dim == dense.dim == prob.dim and crs.f_alg == dense.f_alg
        x = torch.from_numpy(np.random.default_rng(seed).standard_normal(prob.dim)).cuda()
        y1, y2 = torch.empty_like(x), torch.empty_like(x)
        dense.apply_Htarget(x, y1)
        crs.apply_Htarget(x, y2)
        torch.cuda.synchronize()
        assert torch.equal(y1, y2), precision
        if precision == plugin.FP64:
            ref = oracle_built.kron_apply(prob, x.cpu().numpy())
            err = np.abs(y2.cpu().numpy() - ref).max() / max(np.abs(ref).max(), 1e-300)
            assert err < 1e-12
            assert torch.equal(dense.diagonal(), crs.diagonal())
        dense.close()
        crs.close()


def test_crs_handle_of_real_superblocks(cuda_lib, cuda_device):
    """Heisenberg and Hubbard superblock sectors of the oracle DMRG driver,
    their block operators written as CRS over the block bases: bitwise the
    handle of the driver's own tables."""
    import torch
    from oracle import dmrg_driver as dd
    from dmrgpp_b200 import plugin

    def crs_of(blockop, sizes):
        off = np.concatenate([[0], np.cumsum(sizes)])
        n = int(off[-1])
        M = np.zeros((n, n))
        for (g, h), a in blockop.items():
            M[off[g]:off[g + 1], off[h]:off[h + 1]] = a
        ip, ix, dv = [0], [], []
        for r in range(n):
            nz = np.nonzero(M[r])[0]
            ix.extend(int(b) for b in nz)
            dv.extend(float(M[r, b]) for b in nz)
            ip.append(len(ix))
        return np.array(ip, np.int32), np.array(ix, np.int32), np.array(dv)

    for model, L, m in ((dd.Heisenberg(), 12, 32), (dd.Hubbard(U=4.0), 6, 48)):
        d = dd.DMRG(model, L=L, m=m, solver=dd.dense_solver())
        left, right = d.site, d.site
        for _ in range(3):
            left, right = d.grow_left(left), d.grow_right(right)
        lp, rp = d.grow_left(left), d.grow_right(right)
        target = model.target(2 * lp.length)
        prob, patches = d.superblock(lp, rp, target)
        terms = [(1.0, lp.ops["H"], dd.identity(rp)), (1.0, dd.identity(lp), rp.ops["H"])]
        terms += model.links(lp.ops, rp.ops, lp.ops.get("P"))
        loff = np.concatenate([[0], np.cumsum(lp.sizes)])
        roff = np.concatenate([[0], np.cumsum(rp.sizes)])
        A = [crs_of(lo, lp.sizes) for _, lo, _ in terms]
        B = [crs_of(ro, rp.sizes) for _, _, ro in terms]
        vals = [c for c, _, _ in terms]
        crs = plugin.BatchedGemm.from_crs([int(loff[gl]) for gl, _ in patches], prob.lsz,
                                          [int(roff[gr]) for _, gr in patches], prob.rsz, A, B,
                                          value=vals)
        dense = plugin.BatchedGemm.from_problem(prob)
        x = torch.from_numpy(np.random.default_rng(L).standard_normal(prob.dim)).cuda()
        y1, y2 = torch.empty_like(x), torch.empty_like(x)
        dense.apply_Htarget(x, y1)
        crs.apply_Htarget(x, y2)
        torch.cuda.synchronize()
        assert torch.equal(y1, y2), model
        dense.close()
        crs.close()
