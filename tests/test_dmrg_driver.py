"""The two-site DMRG driver of the oracle (oracle/dmrg_driver.py) pinned on
the CPU: exact small cases and the reference's own published energies with
the reference's own sector solver.  These runs make the driver a trusted
harness for the GPU runs in test_dmrg_gpu.py."""
import json
import os

import pytest

from oracle import dmrg_driver as dd

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_heisenberg_L8_exact():
    d = dd.DMRG(dd.Heisenberg(), L=8, m=64, solver=dd.dense_solver())
    assert abs(d.run(sweeps=1) - (-3.374932598687897)) < 1e-12


@pytest.mark.parametrize("U", [0.0, 4.0])
def test_hubbard_L4_exact(U):
    d = dd.DMRG(dd.Hubbard(U=U), L=4, m=64, solver=dd.dense_solver())
    e = d.run(sweeps=1)
    assert abs(e - dd.hubbard_ed(4, U, 2, 2)) < 1e-12
    if U == 0.0:
        assert abs(e - dd.free_fermion_energy(4, 2, 2)) < 1e-12


def test_hubbard_L8_U0_reference_solver(oracle_built):
    """dmrg/CMakeLists.txt:180-181 (input2_batchedgemm): Hubbard L=8, U=0,
    half filling, -9.51754; exact free-fermion value -9.517540966..."""
    d = dd.DMRG(dd.Hubbard(U=0.0), L=8, m=256, solver=dd.reference_solver())
    e = d.run(sweeps=1)
    assert abs(e - (-9.51754)) < 1e-5
    assert abs(e - dd.free_fermion_energy(8, 4, 4)) < 1e-9


def test_heisenberg_L32_golden_is_the_reference_value():
    g = json.load(open(os.path.join(GOLDEN, "dmrg_heisenberg_L32_m128.json")))
    assert abs(g["energy"] - g["reference_test_energy"]) < g["reference_test_tolerance"]
    assert len(g["energies"]) == 131


@pytest.mark.parametrize("Lx,U,n", [(2, 4.0, 2), (3, 8.0, 3), (4, 8.0, 3)])
def test_hubbard_ladder_matches_exact_diagonalisation(Lx, U, n):
    """Two-leg ladder in the reference's site order (Ladder.h:87-292: rungs
    (2c, 2c+1), legs (i, i+2)): blocks carry their last two sites'
    operators; with every state kept the DMRG energy is the Fock-space exact
    energy of the same bond list."""
    mdl = dd.HubbardLadder(Lx, U=U, n_up=n, n_dn=n)
    exact = dd.hubbard_ed(2 * Lx, U, n, n, bonds=mdl.bonds())
    d = dd.DMRG(mdl, L=2 * Lx, m=400, solver=dd.dense_solver())
    assert abs(d.run(sweeps=1) - exact) < 1e-11


def test_ladder_bonds_follow_the_reference_geometry():
    mdl = dd.HubbardLadder(3)
    assert mdl.bonds() == [(0, 1, 1.0), (0, 2, 1.0), (1, 3, 1.0), (2, 3, 1.0), (2, 4, 1.0),
                           (3, 5, 1.0), (4, 5, 1.0)]
