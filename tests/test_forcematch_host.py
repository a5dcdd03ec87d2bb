"""Host side of force matching: parameter tables, their derivatives and the
seeded 2-type configuration (no GPU)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from lammps_b200.forcematch import force_matching_case, lj_tables, pair_matrix  # noqa: E402


def test_pair_matrix_is_symmetric_and_differentiable():
    v = torch.tensor([1.0, 2.0, 3.0], dtype=torch.float64, requires_grad=True)
    m = pair_matrix(v, 2)
    assert m.shape == (3, 3)
    assert torch.equal(m, m.T)
    assert m[1, 1] == 1.0 and m[1, 2] == 2.0 and m[2, 2] == 3.0 and m[0].abs().sum() == 0
    m.sum().backward()
    assert v.grad.tolist() == [1.0, 2.0, 1.0]  # off-diagonal value appears twice
    with pytest.raises(ValueError):
        pair_matrix(torch.zeros(2), 2)


def test_lj_tables_match_init_one():
    eps = pair_matrix(torch.tensor([1.0, 0.8, 1.2], dtype=torch.float64), 2)
    sig = pair_matrix(torch.tensor([1.0, 1.05, 0.95], dtype=torch.float64), 2)
    lj1, lj2, cutsq = lj_tables(eps, sig, 2.5)
    w = 3
    # PairLJCut::init_one (src/pair_lj_cut.cpp:560-563)
    assert lj1[1 * w + 2].item() == pytest.approx(48 * 0.8 * 1.05 ** 12, rel=1e-15)
    assert lj2[2 * w + 2].item() == pytest.approx(24 * 1.2 * 0.95 ** 6, rel=1e-15)
    assert cutsq[2 * w + 1] == pytest.approx((2.5 * 1.05) ** 2, rel=1e-15)
    assert cutsq[0] == 0.0


def test_lj_table_chain_rule():
    ev = torch.tensor([1.0, 0.8, 1.2], dtype=torch.float64, requires_grad=True)
    sv = torch.tensor([1.0, 1.05, 0.95], dtype=torch.float64, requires_grad=True)
    lj1, lj2, _ = lj_tables(pair_matrix(ev, 2), pair_matrix(sv, 2))
    (lj1[4] + lj2[4]).backward()  # entry (1,1)
    assert ev.grad[0].item() == pytest.approx(48 + 24)
    assert sv.grad[0].item() == pytest.approx(48 * 12 + 24 * 6)


def test_force_matching_case_is_seeded():
    a = force_matching_case()
    b = force_matching_case()
    assert a["x"].shape == (8000, 3)
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["types"], b["types"])
    assert (a["types"] == 1).sum() == 4000 and (a["types"] == 2).sum() == 4000
    assert np.all((a["eps"] >= 0.5) & (a["eps"] <= 1.5))
    assert np.all((a["sigma"] >= 0.9) & (a["sigma"] <= 1.1))
    assert np.all(a["x"] >= 0) and np.all(a["x"] < a["hi"])
    # non-cubic box: 10 x 10 x 20 cells at rho* 0.85
    assert a["hi"][2] == pytest.approx(2 * a["hi"][0])
    assert 8000 / np.prod(a["hi"]) == pytest.approx(0.85)
