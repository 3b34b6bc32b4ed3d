"""GPU parity of the rotor + atom expansion build (SYS_TYPE 1 and 4,
mqct_build_matrix_expansion) with the oracle restatement, and the cross-path check of
tests/test_oracle_expansion_atom.py through the GPU's direct build (FP64) and expansion
build: both within 1e-10 of the largest element."""
import numpy as np
import pytest

from mqct_b200 import synthetic as syn
from test_oracle_expansion_atom import CASES, CM, oracle_system, term_table

pytestmark = pytest.mark.gpu


def test_type4_expansion_matches_oracle(mq, oracle, gpu_available):
    chans = [c for c in syn.config_c2()["channels"] if c[0] <= 6]
    s = mq.CollisionSystem(4, chans, A=27.9, B=14.5, C=9.3)
    ch = s.channels
    osys = oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=s.e_ch,
                               vec1=s.vec1.reshape(-1), ldv=s.ldv)
    labels = [(l, nu) for l in range(7) for nu in range(l + 1)]
    R = mq.r_grid(40, 3.0, 20.0)
    rng = np.random.default_rng(8)
    T = rng.normal(size=(len(R), len(labels))) * np.exp(-R)[:, None] * 1e4
    m, y2, sk = mq.build_matrix_expansion(s, R, labels, T, mij_cutoff=0.0)
    mo = oracle.expansion_matrix_atom(osys, osys.states(), s.ind_mat, labels, T, CM)
    assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()
    assert not sk.any()


def test_type1_expansion_matches_oracle(mq, oracle, gpu_available):
    c1 = syn.config_c1()
    s = mq.CollisionSystem(1, c1["channels"], BE=c1["BE"])
    osys = oracle.OracleSystem(1, s.channels[:, 0], e_ch=s.e_ch)
    labels = [(l,) for l in range(9)]
    R = mq.r_grid(60, 3.0, 20.0)
    T = np.random.default_rng(1).normal(size=(len(R), len(labels))) * 100.0
    m, _, _ = mq.build_matrix_expansion(s, R, labels, T, mij_cutoff=0.0)
    mo = oracle.expansion_matrix_atom(osys, osys.states(), s.ind_mat, labels, T, CM)
    assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()


@pytest.mark.parametrize("sys_type", [4, 1])
def test_direct_and_expansion_builds_agree_on_gpu(mq, oracle, gpu_available, sys_type):
    case = CASES[sys_type]
    s, _ = oracle_system(mq, oracle, sys_type, case)
    W = term_table(oracle, case["labels"], case["grid"], sys_type)
    R = np.array([5.0, 6.0, 7.0])
    v = np.random.default_rng(2).normal(size=(len(case["labels"]), len(R))) * 100
    V = np.einsum("tr,t...->r...", v, W)
    nb, ng = case["grid"]
    grid = (nb, ng, 0, 0, 0, 0, 1) if sys_type == 4 else (nb, 0, 0, 0, 0, 0, 1)
    pes = dict(kind=mq._abi.PES_TABLE, n_terms=0, params=np.zeros(1), table=V.reshape(-1))
    direct, _, _ = mq.build_matrix(s, R, grid, pes, precision=mq.PREC_FP64, mij_cutoff=0.0)
    expan, _, _ = mq.build_matrix_expansion(s, R, case["labels"], v.T, mij_cutoff=0.0)
    assert np.max(np.abs(direct - expan)) <= 1e-10 * np.abs(direct).max()


@pytest.mark.parametrize("sys_type,shape,eq", [(4, (3, 20, 16), True), (4, (2, 12, 9), False),
                                               (1, (4, 30), True)])
def test_atom_projection_matches_oracle(mq, oracle, gpu_available, sys_type, shape, eq):
    labels = CASES[sys_type]["labels"]
    V = np.random.default_rng(9).normal(size=shape) * 1e3 + 20.0
    T, Ti = mq.project_terms(sys_type, labels, V, eq_gamma=eq)
    To, Tio = oracle.project_terms_atom(sys_type, labels, V, eq_gamma=eq)
    bound = 1e-12 * np.abs(V).max() * 4 * np.pi
    assert np.max(np.abs(T - To.T)) <= bound and np.max(np.abs(Ti - Tio.T)) <= bound


@pytest.mark.parametrize("sys_type", [4, 1])
def test_atom_projection_to_matrix_pipeline(mq, oracle, gpu_available, sys_type):
    """PES table -> projected terms -> expansion matrix, all on the GPU, against the
    direct build of the same table: equal for type 1; for type 4 after reversing the
    sign of the odd-nju terms (the projection's (-1)^nju, see the oracle tests)."""
    case = CASES[sys_type]
    s, _ = oracle_system(mq, oracle, sys_type, case)
    W = term_table(oracle, case["labels"], case["grid"], sys_type)
    R = np.array([5.0, 7.0])
    v = np.random.default_rng(2).normal(size=(len(case["labels"]), len(R))) * 100
    V = np.einsum("tr,t...->r...", v, W)
    T, _ = mq.project_terms(sys_type, case["labels"], V)
    if sys_type == 4:
        T = T * np.array([(-1.0) ** lab[1] for lab in case["labels"]])[None, :]
    assert np.allclose(T, v.T, rtol=0, atol=1e-10 * np.abs(v).max())
    nb, ng = case["grid"]
    grid = (nb, ng, 0, 0, 0, 0, 1) if sys_type == 4 else (nb, 0, 0, 0, 0, 0, 1)
    pes = dict(kind=mq._abi.PES_TABLE, n_terms=0, params=np.zeros(1), table=V.reshape(-1))
    direct, _, _ = mq.build_matrix(s, R, grid, pes, precision=mq.PREC_FP64, mij_cutoff=0.0)
    expan, _, _ = mq.build_matrix_expansion(s, R, case["labels"], T, mij_cutoff=0.0)
    assert np.max(np.abs(direct - expan)) <= 1e-10 * np.abs(direct).max()


def test_type5_expansion_matches_oracle(mq, oracle, gpu_available):
    from test_oracle_type5 import LABS, type5_oracle
    s, o8, _ = type5_oracle(mq, oracle)
    R = mq.r_grid(30, 4.0, 15.0)
    T = np.random.default_rng(5).normal(size=(len(R), len(LABS))) * np.exp(-R)[:, None] * 1e4
    m, _, _ = mq.build_matrix_expansion(s, R, LABS, T, mij_cutoff=0.0)
    mo = oracle.expansion_matrix_type8(o8, o8.states(), s.ind_mat,
                                       [(a, 0, b, c) for a, b, c in LABS], T)
    assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()


def test_type3_expansion_matches_oracle(mq, oracle, gpu_available):
    """SYS_TYPE 3 (symmetric top + atom): the GPU build against the oracle's case-3
    formula, with the -nju branch factor the reference writes for it."""
    from test_oracle_type3 import LABELS, systems

    s, o3, _ = systems(mq, oracle)
    R = mq.r_grid(30, 3.0, 20.0)
    T = np.random.default_rng(12).normal(size=(len(R), len(LABELS))) * np.exp(-R)[:, None] * 1e4
    m, _, sk = mq.build_matrix_expansion(s, R, LABELS, T, mij_cutoff=0.0)
    mo = oracle.expansion_matrix_atom(o3, o3.states(), s.ind_mat, LABELS, T, CM)
    assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()
    assert not sk.any()


def test_type3_projection_matches_oracle(mq, oracle, gpu_available):
    from test_oracle_type3 import LABELS

    V = np.random.default_rng(13).normal(size=(3, 16, 12)) * 1e3 + 20.0
    T, Ti = mq.project_terms(3, LABELS, V)
    To, Tio = oracle.project_terms_atom(3, LABELS, V)
    bound = 1e-12 * np.abs(V).max() * 4 * np.pi
    assert np.max(np.abs(T - To.T)) <= bound and np.max(np.abs(Ti - Tio.T)) <= bound


@pytest.mark.parametrize("prec,tol", [("PREC_FP64", 1e-12), ("PREC_BF16X3", 1e-4)])
def test_type3_direct_build_matches_oracle(mq, oracle, gpu_available, prec, tol):
    """INTEGRATOR_TEMP case 3 on the GPU (run as case 4 on the parity-adapted vectors)
    against the oracle's WF_SYM_TOP quadrature, on a seeded table PES."""
    from test_oracle_type3 import systems

    s, o3, _ = systems(mq, oracle)
    R = mq.r_grid(6, 4.0, 12.0)
    grid = (16, 14)
    V = np.random.default_rng(14).normal(size=(len(R),) + grid) * 300.0 + 50.0
    g = grid + (0, 0, 0, 0, 1)
    pes = dict(kind=mq._abi.PES_TABLE, n_terms=0, params=np.zeros(1), table=V.reshape(-1))
    m, _, _ = mq.build_matrix(s, R, g, pes, precision=getattr(mq, prec), mij_cutoff=0.0)
    opes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
    mo, _, _ = oracle.build_matrix(o3, o3.states(), s.ind_mat, R, g, opes, mij_cut=0.0)
    assert np.max(np.abs(m - mo)) <= tol * np.abs(mo).max()
