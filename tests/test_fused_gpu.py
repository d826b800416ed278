"""Parity of the fused FP64 H*x form (kron_fused.cu: both passes of an output
tile in one CTA, the parts of a tile summed through the distributed shared
memory of a thread-block cluster) with the oracle, through the C ABI.

FP64 tolerance as for the two-pass form: max |y - y_oracle| <= 1e-12 *
max |y_oracle| (test_BatchedGemm.cpp:232-257); results are bitwise
reproducible from call to call, and the group solver's sector mask, device
step records (graph replay) and the tuner's choice work as with the two-pass
form."""
import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

pytestmark = pytest.mark.gpu
RTOL = 1e-12
FUSED0 = 6          # first fused configuration (include/dmrgpp_kron.h)
NFUSED = 2


def rel_err(y, ref):
    return float(np.abs(y - ref).max() / max(np.abs(ref).max(), 1e-300))


@pytest.mark.parametrize("f", list(range(NFUSED)))
@pytest.mark.parametrize("parts", [1, 4])
def test_every_fused_configuration(cuda_lib, cuda_device, oracle_built, f, parts):
    """Ragged patches (1..150: several row and column tiles, chunks of X_j
    narrower than 32), missing and all-zero blocks, an output patch with no
    terms at all."""
    from dmrgpp_b200 import plugin
    prob = sb.random_problem(npatches=12, noperator=4, max_size=150, seed=70 + f,
                             density=0.6, zero_block_rate=0.1)
    x = np.random.default_rng(f).standard_normal(prob.dim)
    bg = plugin.BatchedGemm.from_problem(prob)
    bg.set_config(FUSED0 + f, parts)
    assert bg.get_config() == (FUSED0 + f, parts)
    y = bg(x)
    assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL
    assert np.array_equal(bg(x), y)
    bg.close()


def test_fused_output_patch_without_terms_is_zeroed(cuda_lib, cuda_device, oracle_built):
    """Overwrite semantics: an output patch no triple reaches is written as 0
    even when y held data before."""
    import torch
    from dmrgpp_b200 import plugin
    l, r = np.array([5, 7, 3]), np.array([4, 6, 2])
    rng = np.random.default_rng(3)
    A = {(0, 1, 0): np.asfortranarray(rng.standard_normal((5, 7))),
         (1, 1, 0): np.asfortranarray(rng.standard_normal((7, 7)))}
    B = {(0, 1, 0): np.asfortranarray(rng.standard_normal((4, 6))),
         (1, 1, 0): np.asfortranarray(rng.standard_normal((6, 6)))}
    prob = sb.KronProblem(l, r, 1, A, B)
    x = rng.standard_normal(prob.dim)
    bg = plugin.BatchedGemm.from_problem(prob)
    for f in (0, 1):
        bg.set_config(FUSED0 + f, 2)
        xd = torch.from_numpy(x).cuda()
        yd = torch.full_like(xd, float("nan"))
        bg.apply_Htarget(xd, yd)
        y = yd.cpu().numpy()
        assert not np.isnan(y).any()
        assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL
        assert np.all(y[prob.xy_start[2]:] == 0.0)
    bg.close()


@pytest.mark.parametrize("f", [0, 1])
def test_fused_microbench_sector(cuda_lib, cuda_device, oracle_built, f):
    from dmrgpp_b200 import plugin
    prob = sb.c2_problem()
    x = sb.random_unit_vector(prob.dim, seed=12)
    bg = plugin.BatchedGemm.from_problem(prob)
    bg.set_config(FUSED0 + f, 2)
    y = bg(x)
    assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL
    bg.set_config(0, 2)                      # the two-pass form agrees to round-off
    assert rel_err(bg(x), y) < 1e-14
    bg.close()


def test_fused_group_with_sector_mask_and_lanczos(cuda_lib, cuda_device, oracle_built):
    """A group handle (independent sectors in one launch) in the fused form:
    H*x per sector against the oracle, and the lockstep group Lanczos (which
    masks stopped sectors) against the two-pass form's energies."""
    from dmrgpp_b200 import plugin
    probs = [sb.random_problem(npatches=5, noperator=3, max_size=40, seed=1, symmetric=True),
             sb.c2_problem(seed=5),
             sb.random_problem(npatches=1, noperator=1, max_size=1, seed=2, symmetric=True),
             sb.spin_chain_like(sb.gaussian_sector_sizes(128, 7, 1.4), seed=6)]
    bg = plugin.BatchedGemm.from_problems(probs)
    offs = bg.sector_offsets()
    init = np.random.default_rng(11).standard_normal(bg.dim)
    e_ref, _, steps_ref = bg.lanczos_lowest_group(init, steps=200, tolerance=1e-12)
    bg.set_config(FUSED0 + 1, 2)
    y = bg(init)
    for s, p in enumerate(probs):
        assert rel_err(y[offs[s]:offs[s + 1]], oracle_built.kron_apply(p, init[offs[s]:offs[s + 1]])) < RTOL
    e, _, steps = bg.lanczos_lowest_group(init, steps=200, tolerance=1e-12)
    for s in range(len(probs)):
        assert abs(e[s] - e_ref[s]) <= 1e-11 * max(1.0, abs(e_ref[s])), (s, e[s], e_ref[s])
    bg.close()


def test_fused_graph_replayed_lanczos_is_bitwise_identical(cuda_lib, cuda_device):
    """The captured solver steps read x and y from the device step record;
    the fused launch (a cluster launch) is captured and replayed like the
    persistent one."""
    import torch
    from dmrgpp_b200 import plugin
    prob = sb.c2_problem(seed=21)
    bg = plugin.BatchedGemm.from_problem(prob)
    bg.set_config(FUSED0 + 1, 2)
    init = torch.from_numpy(np.random.default_rng(4).standard_normal(prob.dim)).cuda()
    e0, z0, n0 = bg.lanczos_lowest(init, steps=77, use_graph=False)
    e1, z1, n1 = bg.lanczos_lowest(init, steps=77, use_graph=True)
    assert e0 == e1 and n0 == n1
    assert torch.equal(z0, z1)
    bg.close()


def test_tuner_considers_the_fused_form(cuda_lib, cuda_device, oracle_built, tmp_path):
    """On the microbench sector every configuration is timed; whichever wins
    gives the oracle's result."""
    from dmrgpp_b200 import plugin
    prob = sb.c2_problem()
    x = sb.random_unit_vector(prob.dim, seed=3)
    bg = plugin.BatchedGemm.from_problem(prob)
    cfg, us = bg.autotune(str(tmp_path / "tune.txt"), reps=3)
    assert 0 <= cfg < FUSED0 + NFUSED and us > 0
    assert rel_err(bg(x), oracle_built.kron_apply(prob, x)) < RTOL
    bg.close()
