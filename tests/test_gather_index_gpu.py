"""Device sector gather / scatter (dmrgpp_gather, dmrgpp_scatter) with the
library's copyIn / copyOut index (dmrgpp_kron_gather_index) on real DMRG
superblock sectors, bit for bit against the oracle's restatement of the
reference loops (oracle_gather_index, InitKronHamiltonian.h:158-221 and
InitKronBase.h:315-360), and one whole KronMatrix step: copyIn, H*x in patch
order, copyOut (KronMatrix.h:137-171) against the oracle."""
import numpy as np
import pytest

from dmrgpp_b200 import plugin

from gather_cases import CASES, sector_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("model,L,m,steps", CASES)
def test_gather_scatter_bitwise_against_oracle_index(cuda_lib, cuda_device, oracle_built, model,
                                                     L, m, steps):
    import torch
    c = sector_case(model, L, m, steps)
    idx = plugin.sector_gather_index(c["patch_left"], c["patch_right"], c["left_partition"],
                                     c["right_partition"], c["perm_inverse"], c["offset"],
                                     c["size"])
    nl = int(c["left_partition"][-1])
    ref_idx = oracle_built.gather_index(len(c["patch_left"]), c["left_partition"],
                                        c["right_partition"], c["patch_left"], c["patch_right"], nl,
                                        c["perm_inverse"], c["offset"], c["size"])
    n = c["size"]
    vin = np.random.default_rng(5).standard_normal(n)        # the sector in super-basis order
    s = torch.cuda.current_stream().cuda_stream
    src = torch.from_numpy(vin).to(cuda_device)
    di = torch.from_numpy(idx).to(cuda_device)
    yin = torch.full_like(src, float("nan"))
    assert cuda_lib.dmrgpp_gather(src.data_ptr(), di.data_ptr(), yin.data_ptr(), n, s) == 0
    back = torch.full_like(src, float("nan"))
    assert cuda_lib.dmrgpp_scatter(yin.data_ptr(), di.data_ptr(), back.data_ptr(), n, s) == 0
    torch.cuda.synchronize()
    assert np.array_equal(yin.cpu().numpy(), vin[ref_idx])    # copyIn
    out = np.full(n, np.nan)
    out[ref_idx] = yin.cpu().numpy()                           # copyOut
    assert np.array_equal(back.cpu().numpy(), out)
    assert np.array_equal(back.cpu().numpy(), vin)


def test_kron_matrix_step_in_super_basis_order(cuda_lib, cuda_device, oracle_built):
    """x_out = P^T H P x_in: gather to patch order, H*x on the device,
    scatter back, against the oracle's H*x on the gathered vector."""
    import torch
    c = sector_case("hubbard", 10, 32, 3)
    prob = c["prob"]
    idx = plugin.sector_gather_index(c["patch_left"], c["patch_right"], c["left_partition"],
                                     c["right_partition"], c["perm_inverse"], c["offset"],
                                     c["size"])
    n = c["size"]
    vin = np.random.default_rng(7).standard_normal(n)
    s = torch.cuda.current_stream().cuda_stream
    bg = plugin.BatchedGemm.from_problem(prob, stream=s)
    src = torch.from_numpy(vin).to(cuda_device)
    di = torch.from_numpy(idx).to(cuda_device)
    yin = torch.empty_like(src)
    xout = torch.empty_like(src)
    vout = torch.empty_like(src)
    assert cuda_lib.dmrgpp_gather(src.data_ptr(), di.data_ptr(), yin.data_ptr(), n, s) == 0
    bg.apply_Htarget(yin, xout)
    assert cuda_lib.dmrgpp_scatter(xout.data_ptr(), di.data_ptr(), vout.data_ptr(), n, s) == 0
    torch.cuda.synchronize()
    bg.close()
    ref = np.empty(n)
    ref[idx] = oracle_built.kron_apply(prob, vin[idx])
    got = vout.cpu().numpy()
    assert float(np.abs(got - ref).max() / np.abs(ref).max()) < 1e-12
