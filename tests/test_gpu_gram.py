"""mz_gram_device (Powell's normal equations on the device) against FP64
products on the host: the square form (gamma^T gamma, symmetric tiles
only), the general tiled form and the vector form (gamma^T e and the
updated column), exact symmetry and bit-reproducibility."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-13  # vs the host product, relative to sum_k |a_k b_k|


@pytest.fixture(scope="module")
def ev():
    from meamzilla_b200 import synth
    from meamzilla_b200.potential import Database, Evaluator, PotentialFile
    spec, cells = synth.make_workload("eam54", seed=3, ncells=2)
    pot = PotentialFile.from_spec(spec)
    return Evaluator(Database.from_cells(cells, pot), pot, 1.0, 1.0, 0)


def _gram(ev, A, B):
    import torch
    dA = torch.tensor(A, device="cuda")
    dB = dA if B is A else torch.tensor(B, device="cuda")
    out = torch.empty((A.shape[0], B.shape[0]), dtype=torch.float64, device="cuda")
    ev.gram_device(dA, dB, out)
    ev.sync()
    return out.cpu().numpy()


def _close(got, A, B):
    ref = A @ B.T
    scale = np.abs(A) @ np.abs(B).T
    assert np.all(np.abs(got - ref) <= REL * scale + 1e-300)


@pytest.mark.parametrize("na,nb,n", [(136, 136, 400_000), (5, 5, 7), (200, 200, 33), (1, 1, 1)])
def test_square_symmetric(ev, na, nb, n):
    A = np.random.default_rng(na + n).normal(size=(na, n))
    got = _gram(ev, A, A)
    _close(got, A, A)
    assert np.array_equal(got, got.T)
    assert np.array_equal(got, _gram(ev, A, A))


@pytest.mark.parametrize("na,nb,n", [(70, 130, 3000), (136, 5, 100_003), (136, 1, 1_230_000), (136, 2, 12345),
                                     (3, 4, 2049)])
def test_general_and_vector(ev, na, nb, n):
    rng = np.random.default_rng(na * nb + n)
    A = rng.normal(size=(na, n))
    B = rng.normal(size=(nb, n))
    got = _gram(ev, A, B)
    _close(got, A, B)
    assert np.array_equal(got, _gram(ev, A, B))


def test_strided_rows(ev):
    """Rows of a wider array (lda > n): the update's gamma[max_col] view."""
    import torch
    rng = np.random.default_rng(5)
    W = rng.normal(size=(12, 1000))
    dW = torch.tensor(W, device="cuda")
    A, B = dW[:, :777], dW[3:5, 100:877]
    out = torch.empty((12, 2), dtype=torch.float64, device="cuda")
    ev.gram_device(A, B, out)
    ev.sync()
    _close(out.cpu().numpy(), W[:, :777], W[3:5, 100:877])


def test_rejects_bad_shapes(ev):
    import torch
    a = torch.zeros((3, 10), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        ev.gram_device(a, torch.zeros((2, 9), dtype=torch.float64, device="cuda"),
                       torch.zeros((3, 2), dtype=torch.float64, device="cuda"))
    with pytest.raises(TypeError):
        ev.gram_device(a.float(), a.float(), torch.zeros((3, 3), dtype=torch.float64, device="cuda"))
