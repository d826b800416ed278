"""The sector gather index of the reference's copyIn / copyOut
(InitKronHamiltonian.h:158-221, InitKronBase.h:315-360), built by the library
on the host cores (dmrgpp_kron_gather_index, no GPU), against the oracle's
restatement (oracle_gather_index in oracle/kron_oracle.c) on real DMRG
superblock sectors, bit for bit, and the reference's own checks turned into
errors."""
import numpy as np
import pytest

import oracle
from dmrgpp_b200 import _capi, plugin

from gather_cases import CASES, sector_case


def _product(c):
    return plugin.sector_gather_index(c["patch_left"], c["patch_right"], c["left_partition"],
                                      c["right_partition"], c["perm_inverse"], c["offset"],
                                      c["size"])


@pytest.mark.parametrize("model,L,m,steps", CASES)
def test_index_matches_oracle_on_dmrg_sectors(oracle_built, model, L, m, steps):
    c = sector_case(model, L, m, steps)
    idx = _product(c)
    nl = int(c["left_partition"][-1])
    ref = oracle_built.gather_index(len(c["patch_left"]), c["left_partition"],
                                    c["right_partition"], c["patch_left"], c["patch_right"], nl,
                                    c["perm_inverse"], c["offset"], c["size"])
    assert np.array_equal(idx, ref)
    assert np.array_equal(np.sort(idx), np.arange(c["size"]))
    # the copyIn loops themselves, element by element, on a random super-vector
    rng = np.random.default_rng(3)
    v = rng.standard_normal(len(c["perm_inverse"]))
    vin = v[c["offset"]:c["offset"] + c["size"]]
    yin = np.empty(c["size"])
    lp, rp = c["left_partition"].astype(np.int64), c["right_partition"].astype(np.int64)
    ip = 0
    for gl, gr in zip(c["patch_left"], c["patch_right"]):
        sl, sr = lp[gl + 1] - lp[gl], rp[gr + 1] - rp[gr]
        for il in range(sl):
            for ir in range(sr):
                r = int(c["perm_inverse"][(il + lp[gl]) + (ir + rp[gr]) * nl])
                yin[ip + ir + il * sr] = vin[r - c["offset"]]
        ip += sl * sr
    assert np.array_equal(vin[idx], yin)


def test_reference_assertions_become_errors():
    c = sector_case("heisenberg", 12, 16, 3)
    bad = dict(c)
    perm = c["perm_inverse"].copy()
    nl = int(c["left_partition"][-1])
    gl, gr = c["patch_left"][0], c["patch_right"][0]
    q = int(c["left_partition"][gl]) + int(c["right_partition"][gr]) * nl
    perm[q] = c["offset"] + c["size"]                    # outside the sector
    bad["perm_inverse"] = perm
    with pytest.raises(_capi.DmrgppError) as e:
        _product(bad)
    assert e.value.status == _capi.INVALID_ARG and "outside the sector" in str(e.value)
    lp = c["left_partition"]
    p2 = next(p for p, g in enumerate(c["patch_left"]) if lp[g + 1] - lp[g] >= 2)
    q2 = int(lp[c["patch_left"][p2]]) + int(c["right_partition"][c["patch_right"][p2]]) * nl
    perm = c["perm_inverse"].copy()
    perm[q2] = perm[q2 + 1]                              # two states of one patch on one position
    bad["perm_inverse"] = perm
    with pytest.raises(_capi.DmrgppError) as e:
        _product(bad)
    assert "two patch-order elements" in str(e.value)
    bad = dict(c, patch_left=[len(c["left_partition"])] + list(c["patch_left"][1:]))
    with pytest.raises(_capi.DmrgppError) as e:
        _product(bad)
    assert "out of range" in str(e.value)
    bad = dict(c, size=c["size"] + 1)
    with pytest.raises(_capi.DmrgppError) as e:
        _product(bad)
    assert "patches hold" in str(e.value)


@pytest.mark.parametrize("model,L,m,steps", CASES)
def test_patch_list_matches_the_drivers_genijpatch(model, L, m, steps):
    """dmrgpp_kron_patch_list against the DMRG driver's restatement of
    GenIjPatch (GenIjPatch.h:104-118) on real superblocks: same pairs, same
    order."""
    c = sector_case(model, L, m, steps)
    pl, pr = plugin.sector_patches(c["left_qns"], c["right_qns"], c["target"])
    assert list(pl) == list(c["patch_left"]) and list(pr) == list(c["patch_right"])


def test_patch_list_capacity_and_multi_component_numbers():
    lq = [(0, 0), (1, 0), (0, 1), (1, 1)]
    rq = [(1, 1), (0, 1), (1, 0), (0, 0), (1, 1)]     # a repeated right number too
    pl, pr = plugin.sector_patches(lq, rq, (1, 1))
    direct = [(i, j) for i, a in enumerate(lq) for j, b in enumerate(rq)
              if (a[0] + b[0], a[1] + b[1]) == (1, 1)]
    assert list(zip(pl, pr)) == direct
    import ctypes
    n = ctypes.c_size_t()
    i64 = ctypes.POINTER(ctypes.c_int64)
    a = np.array(lq, dtype=np.int64)
    b = np.array(rq, dtype=np.int64)
    t = np.array([1, 1], dtype=np.int64)
    rc = _capi.lib().dmrgpp_kron_patch_list(4, a.ctypes.data_as(i64), 5, b.ctypes.data_as(i64), 2,
                                            t.ctypes.data_as(i64), 0, None, None, ctypes.byref(n))
    assert rc == _capi.INVALID_ARG and n.value == len(direct)
