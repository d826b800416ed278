"""The CRS set-up without a GPU: the oracle's slicing against dense slicing
of the same matrices, and dmrgpp_kron_create_crs's checks of its input,
which run before any device work."""
import numpy as np
import pytest

from crs_cases import random_crs_case
from oracle import crs_oracle


def _dense(ip, ix, dv, n):
    M = np.zeros((n, n))
    for a in range(n):
        for e in range(ip[a], ip[a + 1]):
            M[a, ix[e]] = dv[e]
    return M


def test_oracle_blocks_are_the_dense_slices():
    c = random_crs_case(3)
    prob = crs_oracle.problem_from_crs(c["loff"], c["lsz"], c["roff"], c["rsz"], c["A"], c["B"],
                                       c["value"], c["fermion"], c["parity"])
    sign = np.where(c["parity"] == 1, -1.0, 1.0)
    for (i, j, k), a in prob.A.items():
        A = _dense(*c["A"][k], c["nL"])
        if c["fermion"][k]:
            A = A * sign[:, None]
        A = A * c["value"][k]
        li, lj = c["loff"][i], c["loff"][j]
        assert np.array_equal(a, A[li:li + c["lsz"][i], lj:lj + c["lsz"][j]])
        B = _dense(*c["B"][k], c["nR"])
        ri, rj = c["roff"][i], c["roff"][j]
        assert np.array_equal(prob.B[(i, j, k)], B[ri:ri + c["rsz"][i], rj:rj + c["rsz"][j]])
    assert len(prob.A) > 0


def _create(c, **over):
    from dmrgpp_b200 import plugin
    args = dict(left_offset=c["loff"], left_size=c["lsz"], right_offset=c["roff"],
                right_size=c["rsz"], A=c["A"], B=c["B"], value=c["value"], fermion=c["fermion"],
                left_parity=c["parity"])
    args.update(over)
    return plugin.BatchedGemm.from_crs(**args)


@pytest.mark.parametrize("what", ["column", "repeat", "overlap", "parity", "rows", "past"])
def test_malformed_input_is_rejected_before_device_work(cuda_lib, what):
    from dmrgpp_b200 import _capi
    c = random_crs_case(5)
    over = {}
    if what == "column":
        ip, ix, dv = c["A"][0]
        ix = ix.copy()
        ix[0] = c["nL"] + 3
        over["A"] = [(ip, ix, dv)] + c["A"][1:]
    elif what == "repeat":
        ip, ix, dv = c["A"][0]
        row = next(a for a in range(len(ip) - 1) if ip[a + 1] - ip[a] >= 2)
        ix = ix.copy()
        ix[ip[row] + 1] = ix[ip[row]]
        over["A"] = [(ip, ix, dv)] + c["A"][1:]
    elif what == "overlap":
        lo = list(c["loff"])
        lo[1] = lo[0]
        ls = list(c["lsz"])
        ls[1] = ls[0]
        over["left_offset"], over["left_size"] = lo, ls
    elif what == "parity":
        over["left_parity"] = None
    elif what == "rows":
        ip, ix, dv = c["B"][1]
        over["B"] = c["B"][:1] + [(ip[:-1], ix[:ip[-2]], dv[:ip[-2]])] + c["B"][2:]
    elif what == "past":
        ls = list(c["lsz"])
        ls[-1] = c["nL"]
        over["left_size"] = ls
    with pytest.raises(_capi.DmrgppError) as ei:
        _create(c, **over)
    assert ei.value.status == _capi.INVALID_ARG, str(ei.value)
