"""The benchmark's DMRG configurations through the CUDA solver (the sweep
engine is the oracle's two-site driver; tests/dmrg_runs.py holds the runs,
here at reduced length: one finite sweep of the Hubbard chain, one ladder
sector).

* Hubbard chain, t=1, U=4, open BC, half filling, L=64, m=1000 (the
  configuration's size) over the infinite growth and one finite sweep: the
  mixed-precision solve (TF32x3 Lanczos, FP64 refinement, a counted FP64
  fallback when the refinement reports no convergence) against the plain
  FP64 Lanczos on the same sector from the same start at every step, and the
  final energies of the two trajectories: |dE|/site <= 1e-9.
* Two-leg Hubbard ladder (t_leg = t_rung = 1, U=8, filling 0.875): the last
  infinite-growth sector of an 8-rung ladder at m=400 solved every way the
  ladder measurement does; every form converges to the plain FP64 energy
  within 1e-9 per site.
"""
import pytest

from dmrg_runs import c3, ladder_infinite, ladder_step_measurement

pytestmark = pytest.mark.gpu


def test_c3_hubbard_L64_m1000_one_sweep_mixed_matches_fp64(cuda_lib, cuda_device):
    out = c3(L=64, U=4.0, m=1000, sweeps=1, fp64_run=True, log=lambda *a: None)
    assert out["steps"] == 31 + 122
    assert out["all_converged"]
    assert out["max_abs_dE_per_site_same_input"] <= 1e-9, out["max_abs_dE_per_site_same_input"]
    assert out["final_abs_dE_per_site"] <= 1e-9, out["final_abs_dE_per_site"]


def test_ladder_sector_every_solver_agrees(cuda_lib, cuda_device):
    recs = ladder_infinite(Lx=8, m=400, measure_last=1, log=lambda *a: None,
                           on_sector=lambda prob, init, q: ladder_step_measurement(
                               prob, init, 16, mlp=None))
    assert len(recs) == 1
    r = recs[0]
    # H_L, H_R and 2 leg bonds across the centre (between two rungs) x 4 hoppings
    assert r["noperator"] == 2 + 2 * 4
    e64 = r["fp64_lanczos"]["energy"]
    assert r["fp64_jacobi_davidson"]["converged"]
    assert abs(r["fp64_jacobi_davidson"]["energy"] - e64) / 16 <= 1e-9
    assert r["mixed_lanczos_refined"]["converged"]
    assert r["mixed_lanczos_refined"]["abs_dE_per_site"] <= 1e-9
    for k in ("mixed_davidson_none", "mixed_davidson_jacobi"):
        assert r[k]["converged"], k
        assert r[k]["abs_dE_per_site"] <= 1e-9, k
