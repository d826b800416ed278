"""KronLogger files (dmrg/Engine/MatrixVectorKron/KronLogger.hh:112-174):
write plugin tables in the reference's dump format and read them back."""
import numpy as np
import pytest

from dmrgpp_b200 import kronlog
from dmrgpp_b200 import superblock as sb


@pytest.mark.parametrize("make", [lambda: sb.c2_problem(seed=4),
                                  lambda: sb.random_problem(5, 3, max_size=9, seed=2,
                                                            zero_block_rate=0.0),
                                  lambda: sb.ladder_problem(total_states=300, sigma=1.2, seed=1,
                                                            legs=1)])
def test_round_trip(tmp_path, oracle_built, make):
    prob = make()
    v = np.random.default_rng(1).standard_normal(prob.dim)
    path = str(tmp_path / "kron.txt")
    kronlog.write_kronlog(prob, v, path)
    back, v2 = kronlog.read_kronlog(path)
    assert np.array_equal(v, v2)
    assert list(back.lsz) == list(prob.lsz) and list(back.rsz) == list(prob.rsz)
    np.testing.assert_array_equal(oracle_built.kron_apply(back, v), oracle_built.kron_apply(prob, v))


def test_reader_rejects_inconsistent_offsets(tmp_path):
    prob = sb.random_problem(3, 1, max_size=4, seed=5, zero_block_rate=0.0)
    v = np.ones(prob.dim)
    path = tmp_path / "bad.txt"
    kronlog.write_kronlog(prob, v, str(path))
    text = path.read_text().splitlines()
    i = next(k for k, ln in enumerate(text) if ln.startswith("# nc")) + 1
    f = text[i].split()
    f[-1] = str(int(f[-1]) + 1)             # offsetY off by one
    text[i] = " ".join(f)
    path.write_text("\n".join(text) + "\n")
    with pytest.raises(ValueError):
        kronlog.read_kronlog(str(path))
