"""EXPANSION_MATRIX_ELEMENT for a rotor and an atom (SYS_TYPE 1 and 4,
MQCT_SOURCE_CODES/pot_comp.f:6551-6622, 6955-7075).  No reference example builds these
matrices from expansion terms (its SYS_TYPE 1 and 4 examples integrate the PES directly),
so the restatement is pinned by a cross-path check: for a PES built from the terms'
functions on the grid, V = sum_t v_t (Y_{l nju} + Y_{l nju}^*) with Y = WF_DIAT_TOP
(one Y for nju = 0), the direct quadrature (INTEGRATOR_TEMP, MQCT_SOURCE_CODES/pot_comp.f:
1919-1953, 2503-2560) and the expansion formula with the coefficients v_t give the same
matrix.  (The reference's projection EXPANSION_TERM, :3776-3780, multiplies the type-4
function by (-1)^nju, so a projected type-4 PES enters this formula with the sign of its
odd-nju terms reversed; both are restated as written.)"""
import ctypes as C

import numpy as np
import pytest

CM = 1.0 / 8065.5448 / 27.21113845

CASES = {
    4: dict(channels=[(0, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0), (2, 0, 2), (2, 1, 2), (2, 1, 1),
                      (2, 2, 1), (2, 2, 0), (3, 0, 3), (3, 1, 3)],
            labels=[(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 1), (3, 2), (4, 3), (3, 0),
                    (5, 4)],
            kw=dict(A=27.9, B=14.5, C=9.3), grid=(24, 24)),
    1: dict(channels=[(0,), (1,), (2,), (3,), (4,)], labels=[(0,), (1,), (2,), (3,), (4,), (6,)],
            kw=dict(BE=1.93), grid=(24, 1)),
}


def oracle_system(mq, oracle, sys_type, case):
    s = mq.CollisionSystem(sys_type, case["channels"], **case["kw"])
    ch = s.channels
    if sys_type == 4:
        osys = oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=s.e_ch,
                                   vec1=s.vec1.reshape(-1), ldv=s.ldv)
    else:
        osys = oracle.OracleSystem(1, ch[:, 0], e_ch=s.e_ch)
    return s, osys


def term_table(oracle, labels, grid, sys_type):
    """W_t on the (beta, gamma) grid: Y_{l nju} + Y_{l nju}^* (Y for nju = 0)."""
    nb, ng = grid
    x, _ = np.polynomial.legendre.leggauss(nb)
    beta = np.pi / 2 + np.pi / 2 * x
    gam = (np.arange(ng) + 0.5) * 2 * np.pi / ng
    W = np.zeros((len(labels), nb, ng))
    re, im = C.c_double(), C.c_double()
    for t, lab in enumerate(labels):
        l, nu = lab[0], (lab[1] if len(lab) > 1 else 0)
        for i in range(nb):
            for j in range(ng):
                oracle.lib().orc_wf_diat(l, nu, beta[i], gam[j], C.byref(re), C.byref(im))
                W[t, i, j] = re.value * (1.0 if nu == 0 else 2.0)
    return W if sys_type == 4 else W[..., 0]


@pytest.mark.parametrize("sys_type", [4, 1])
def test_expansion_equals_direct_quadrature(mq, oracle, sys_type):
    case = CASES[sys_type]
    s, osys = oracle_system(mq, oracle, sys_type, case)
    W = term_table(oracle, case["labels"], case["grid"], sys_type)
    R = np.array([5.0, 7.0])
    v = np.random.default_rng(2).normal(size=(len(case["labels"]), len(R))) * 100
    V = np.einsum("tr,t...->r...", v, W)
    pes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
    nb, ng = case["grid"]
    grid = (nb, ng, 0, 0, 0, 0, 1) if sys_type == 4 else (nb, 0, 0, 0, 0, 0, 1)
    st = osys.states()
    direct, _, _ = oracle.build_matrix(osys, st, s.ind_mat, R, grid, pes, mij_cut=0.0)
    expan = oracle.expansion_matrix_atom(osys, st, s.ind_mat, case["labels"],
                                         np.ascontiguousarray(v.T), CM)
    assert np.max(np.abs(direct - expan)) <= 1e-10 * np.abs(direct).max()


def test_type1_term_is_the_gaunt_coefficient(mq, oracle):
    """A single Legendre term v P_l-like: M = v sqrt((2l+1)/4pi) sqrt((2j'+1)/(2j''+1))
    <j' m l 0|j'' m> <j' 0 l 0|j'' 0> (the closed form of case 1)."""
    case = CASES[1]
    s, osys = oracle_system(mq, oracle, 1, case)
    st = osys.states()
    ic, j12, m12, _ = st
    T = np.zeros((1, len(case["labels"])))
    T[0, 2] = 1.0 / CM   # l = 2, one Hartree
    m = oracle.expansion_matrix_atom(osys, st, s.ind_mat, case["labels"], T, CM)
    for k, (a, b) in enumerate(s.ind_mat):
        jp, jpp, mm = j12[a - 1], j12[b - 1], m12[a - 1]
        want = (np.sqrt(5 / (4 * np.pi)) * np.sqrt((2 * jp + 1) / (2 * jpp + 1)) *
                oracle.cg(jp, 2, jpp, mm, 0, mm) * oracle.cg(jp, 2, jpp, 0, 0, 0))
        assert abs(m[k, 0] - want) < 1e-14


@pytest.mark.parametrize("sys_type", [4, 1])
def test_projection_recovers_the_coefficients(oracle, sys_type):
    """CALC_EXPANSION_TERMS cases 1 and 4: a PES built from the projection's own functions,
    V = sum_t v_t W'_t with W'_t = Re((-1)^nju Y), doubled for nju != 0 (type 4), or Y
    (type 1), projects back onto v_t: the functions are orthonormal on the sphere (case 1
    supplies the azimuthal 2 pi of its beta-only grid)."""
    case = CASES[sys_type]
    W = term_table(oracle, case["labels"], case["grid"], sys_type)
    if sys_type == 4:
        sg = np.array([(-1.0) ** lab[1] for lab in case["labels"]])
        W = W * sg[:, None, None]
    v = np.random.default_rng(4).normal(size=(len(case["labels"]), 2)) * 50
    V = np.einsum("tr,t...->r...", v, W)
    T, _ = oracle.project_terms_atom(sys_type, case["labels"], V)
    assert np.max(np.abs(T - v)) <= 1e-10 * np.abs(v).max()
