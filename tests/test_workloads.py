"""The oracle's own generators of the synthetic workloads (used by the CPU
baseline, which must not load the product library) against the product's
generators: identical CSR, right-hand side and exact solution, bit for bit."""
import numpy as np
import pytest


def _same(A, S):
    rp, ci, v = A.csr()
    assert A.n == S.n
    assert np.array_equal(rp, S.rp) and np.array_equal(ci, S.ci)
    assert np.array_equal(v.view(np.uint64), S.v.view(np.uint64))
    assert np.array_equal(A.b().view(np.uint64), S.b.view(np.uint64))


@pytest.mark.parametrize("N", [1, 2, 17, 256])
def test_poisson2d_matches_product(mf, O, N):
    _same(mf.Matrix.poisson2d(N), O.gen_poisson2d(N))


@pytest.mark.parametrize("N,v,seed", [(1, (1.0, 0.5, 0.25), 0), (9, (1.0, 0.5, 0.25), 0), (64, (1.0, 0.5, 0.25), 0),
                                      (7, (-0.7, 0.0, 2.5), 11)])
def test_convdiff3d_matches_product(mf, O, N, v, seed):
    _same(mf.Matrix.convdiff3d(N, v=v, seed=seed), O.gen_convdiff3d(N, v=v, seed=seed))


@pytest.mark.parametrize("N,klo,khi,seed", [(1, 1e-3, 1e3, 1), (13, 1e-3, 1e3, 1), (32, 1e-4, 1e4, 5),
                                            (128, 1e-3, 1e3, 1)])
def test_varpoisson3d_matches_product(mf, O, N, klo, khi, seed):
    A = mf.Matrix.varpoisson3d(N, klo=klo, khi=khi, seed=seed)
    S = O.gen_varpoisson3d(N, klo=klo, khi=khi, seed=seed)
    _same(A, S)
    assert np.array_equal(A.xstar().view(np.uint64), S.xstar.view(np.uint64))


def test_generator_sizes_of_the_measured_configurations(O):
    assert O.gen_poisson2d(256).ci.size == 326656
    assert O.gen_convdiff3d(64).ci.size == 1810432
    assert O.gen_varpoisson3d(128).ci.size == 14581760


def test_bad_arguments_raise(O):
    with pytest.raises(ValueError):
        O.gen_poisson2d(0)
    with pytest.raises(ValueError):
        O.gen_varpoisson3d(4, klo=0.0)
