"""GPU parity for SYS_TYPE 9 (asymmetric top + symmetric top) with the oracle's literal
case-9 restatements: the expansion build (1e-12 of the largest element), the direct
quadrature (FP64 1e-12, BF16x3 1e-4) and the projection (case 0's, 1e-12 max|V| 16 pi^2)."""
import numpy as np
import pytest

from test_oracle_type9 import CHANS, CM, LABELS, systems

pytestmark = pytest.mark.gpu


def test_type9_expansion_matches_oracle(mq, oracle, gpu_available):
    s, o9, _ = systems(mq, oracle)
    R = mq.r_grid(24, 3.0, 20.0)
    T = np.random.default_rng(21).normal(size=(len(R), len(LABELS))) * np.exp(-R)[:, None] * 1e4
    m, _, sk = mq.build_matrix_expansion(s, R, LABELS, T, mij_cutoff=0.0)
    mo = oracle.expansion_matrix_type0(o9, o9.states(), s.ind_mat, LABELS, T, CM)
    assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()
    assert not sk.any()


@pytest.mark.parametrize("prec,tol", [("PREC_FP64", 1e-12), ("PREC_BF16X3", 1e-4)])
def test_type9_direct_build_matches_oracle(mq, oracle, gpu_available, prec, tol):
    s, o9, _ = systems(mq, oracle, CHANS[:6])
    R = mq.r_grid(3, 5.0, 9.0)
    shape = (4, 6, 6, 4, 4)     # alpha2, beta1, beta2, gamma1, gamma2
    V = np.random.default_rng(22).normal(size=(len(R),) + shape) * 200.0 + 30.0
    n2, n3, n4, n5, n6 = shape
    g = (n3, n5, 0, n4, n2, n6, 1)
    pes = dict(kind=mq._abi.PES_TABLE, n_terms=0, params=np.zeros(1), table=V.reshape(-1))
    m, _, _ = mq.build_matrix(s, R, g, pes, precision=getattr(mq, prec), mij_cutoff=0.0)
    opes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
    mo, _, _ = oracle.build_matrix(o9, o9.states(), s.ind_mat, R, g, opes, mij_cut=0.0)
    assert np.max(np.abs(m - mo)) <= tol * np.abs(mo).max()


def test_type9_projection_matches_oracle(mq, oracle, gpu_available):
    V = np.random.default_rng(23).normal(size=(2, 4, 6, 5, 6, 4)) * 300.0
    T, Ti = mq.project_terms(9, LABELS, V)
    To, Tio = oracle.project_terms(0, LABELS, V)
    bound = 1e-12 * np.abs(V).max() * 16 * np.pi ** 2
    assert np.max(np.abs(T - To.T)) <= bound and np.max(np.abs(Ti - Tio.T)) <= bound
