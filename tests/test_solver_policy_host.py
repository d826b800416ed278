"""Host logic of the library's sector solves (BatchedGemm.solve_lowest and
solve_lowest_group), without a GPU: the handle's device calls are replaced
by fakes that record what was asked, so the tests check which method runs,
that the handle's precision and correction preconditioner come back as they
were, and which sectors the group fallback solves and from which start."""
import numpy as np
import pytest
import torch

from dmrgpp_b200 import _capi, plugin


class FakeHandle(plugin.BatchedGemm):
    """BatchedGemm with every library call replaced (no C library needed)."""

    def __init__(self, precision, tuned=(-1.0, -1.0), refine_converges=True, offsets=None):
        self.precision = precision
        self.precond = _capi.PRECOND_NONE
        self.tuned = tuned
        self.refine_converges = refine_converges
        self.calls = []
        self.offsets = offsets if offsets is not None else [0, 4]
        self.dim = self.offsets[-1]

    # --- the device calls solve_lowest / solve_lowest_group make
    def tuned_times(self):
        return self.tuned

    def get_precision(self):
        return self.precision

    def set_precision(self, p):
        self.precision = p

    def set_correction_preconditioner(self, m):
        self.precond = m

    def lanczos_lowest(self, init, steps=200, tolerance=1e-12, reortho=True, **kw):
        self.calls.append(("lanczos", self.precision, reortho, steps))
        return -1.0, init.clone(), 10

    def refine_lowest(self, z, **kw):
        self.calls.append(("refine", self.precision, self.precond))
        return -1.0, {"converged": int(self.refine_converges), "outer_iterations": 3,
                      "inner_matvecs": 40, "fp64_matvecs": 4, "residual_norm": 0.0}

    def sector_offsets(self):
        return np.array(self.offsets)

    def lanczos_lowest_group(self, init, steps=200, tolerance=1e-12, reortho=True, mask=None, **kw):
        self.calls.append(("lanczos_group", self.precision, reortho,
                           None if mask is None else np.asarray(mask).copy(), init.clone()))
        n = len(self.offsets) - 1
        e = np.full(n, -2.0) if mask is None else np.where(mask, -3.0, np.nan)
        return e, init.clone() + 1.0, np.full(n, 7)

    def refine_lowest_group(self, z, **kw):
        self.calls.append(("refine_group", self.precision, self.precond))
        n = len(self.offsets) - 1
        conv = np.ones(n, dtype=bool) if self.refine_converges is True else np.asarray(self.refine_converges)
        return np.full(n, -1.0), conv, {"outer_iterations": 2, "inner_matvecs": 10,
                                        "fp64_matvecs": 3, "residual_norm": 0.0, "converged": 1}


def test_auto_picks_fp64_where_tf32x3_is_not_faster():
    h = FakeHandle(plugin.TF32X3, tuned=(30.0, 38.0))        # TF32x3 slower: 0.8x
    e, z, st = h.solve_lowest(torch.ones(4))
    assert st["method"] == "fp64"
    assert h.calls == [("lanczos", plugin.FP64, True, 400)]
    assert h.precision == plugin.TF32X3


def test_auto_picks_mixed_where_tf32x3_pays_and_restores_settings():
    h = FakeHandle(plugin.TF32X3, tuned=(300.0, 100.0))      # 3x
    e, z, st = h.solve_lowest(torch.ones(4))
    assert st["method"] == "mixed" and st["fallback"] == 0
    assert h.calls[0] == ("lanczos", plugin.TF32X3, False, 150)
    assert h.calls[1] == ("refine", plugin.TF32X3, _capi.PRECOND_JACOBI)
    assert h.precision == plugin.TF32X3 and h.precond == _capi.PRECOND_NONE


def test_mixed_falls_back_to_fp64_lanczos_from_a_perturbed_state():
    h = FakeHandle(plugin.TF32X3, tuned=(300.0, 100.0), refine_converges=False)
    e, z, st = h.solve_lowest(torch.ones(4), correction="none")
    assert st["fallback"] == 1 and st["converged"] == 1
    assert h.calls[1] == ("refine", plugin.TF32X3, _capi.PRECOND_NONE)
    assert h.calls[2][:2] == ("lanczos", plugin.FP64)
    assert h.precision == plugin.TF32X3


def test_fp64_handle_never_runs_mixed():
    h = FakeHandle(plugin.FP64)
    e, z, st = h.solve_lowest(torch.ones(4))
    assert st["method"] == "fp64" and h.precision == plugin.FP64


def test_unknown_options_are_rejected():
    h = FakeHandle(plugin.TF32X3)
    with pytest.raises(ValueError):
        h.solve_lowest(torch.ones(4), method="fast")
    with pytest.raises(ValueError):
        h.solve_lowest(torch.ones(4), correction="ilu")


def test_group_solve_finishes_only_the_unconverged_sectors():
    conv = np.array([True, False, True, False])
    h = FakeHandle(plugin.TF32X3, refine_converges=conv, offsets=[0, 3, 5, 9, 12])
    init = torch.arange(12, dtype=torch.float64)
    e, z, st = h.solve_lowest_group(init)
    assert st["fallbacks"] == 2
    kinds = [c[0] for c in h.calls]
    assert kinds == ["lanczos_group", "refine_group", "lanczos_group"]
    assert h.calls[1] == ("refine_group", plugin.TF32X3, _capi.PRECOND_JACOBI)
    _, prec, _, mask, start = h.calls[2]
    assert prec == plugin.FP64 and list(mask) == [False, True, False, True]
    # converged sectors keep the refined energies; the others take the fallback's
    assert list(e) == [-1.0, -3.0, -1.0, -3.0]
    # the fallback starts from the refined vectors, perturbed only where it solves
    refined = init + 1.0                     # the fake group Lanczos returns init + 1
    assert torch.equal(start[0:3], refined[0:3]) and torch.equal(start[5:9], refined[5:9])
    for a, b in ((3, 5), (9, 12)):
        d = float(torch.linalg.vector_norm(start[a:b] - refined[a:b]))
        assert 0.9e-3 < d < 1.1e-3
    assert h.precision == plugin.TF32X3 and h.precond == _capi.PRECOND_NONE


def test_group_solve_without_failures_has_no_fallback():
    h = FakeHandle(plugin.TF32X3, offsets=[0, 3, 5])
    e, z, st = h.solve_lowest_group(torch.ones(5), correction="none")
    assert st["fallbacks"] == 0 and st["fallback_seconds"] == 0.0
    assert [c[0] for c in h.calls] == ["lanczos_group", "refine_group"]
    assert h.calls[1][2] == _capi.PRECOND_NONE
