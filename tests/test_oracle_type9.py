"""SYS_TYPE 9, an asymmetric top + a symmetric top: channels (j1, ka1, kc1, j2, k2, eps2)
with levels EIGEN_VAL(A, B, C) + A2 j2(j2+1) - (A2-C2) k2^2
(MQCT_SOURCE_CODES/iotest.f:9445-9498), states j12 = |j1-j2|..j1+j2 as for two rotors,
MTRX.DAT columns J1 K1A K1C J2 K2 EPS written i3 (matrix_ini.f:4821-4832), the
expansion matrix of pot_comp.f:8059-8256 and the direct quadrature of
WF_ASYM_TOP_SYM_TOP (basis_wave_functions.f:42-82, pot_comp.f:3350-3538).

The reference ships no SYS_TYPE 9 example, so the case-9 formula, restated literally
(the four Clebsch-Gordan terms CG_1a..CG_4a of the second rotor with coef_parity), is
tied to the pinned case-0 formula: with the second rotor's parity-adapted vector
(|j k> + (-1)^eps |j -k>) / sqrt(2 (1 + delta_k0)) as its "asymmetric-top" vector, case 0
gives the same matrix, and so does the direct quadrature."""
import numpy as np
import pytest

CM = 1.0 / 8065.5448 / 27.21113845
ABC = dict(A=27.9, B=14.5, C=9.3, A2=9.94, C2=6.23)
CHANS = [(0, 0, 0, 0, 0, 0), (0, 0, 0, 1, 0, 0), (0, 0, 0, 1, 1, 0), (0, 0, 0, 1, 1, 1),
         (1, 0, 1, 0, 0, 0), (1, 0, 1, 1, 1, 1), (1, 1, 1, 1, 0, 0), (1, 1, 0, 2, 1, 0),
         (1, 1, 0, 2, 2, 1), (2, 1, 2, 1, 1, 0)]
LABELS = [(0, 0, 0, 0, 0), (1, 0, 1, 0, 0), (1, 0, 1, 0, 2), (2, 0, 0, 0, 2), (2, 2, 0, 0, 2),
          (0, 0, 2, 2, 2), (2, 1, 1, 1, 2), (1, 1, 1, -1, 2), (2, 2, 2, -2, 4), (2, 0, 2, 0, 0),
          (1, 0, 0, 0, 1), (2, 1, 1, 0, 3), (3, 3, 2, 2, 3), (1, 0, 2, 1, 3)]


def systems(mq, oracle, chans=CHANS):
    s = mq.CollisionSystem(9, chans, **ABC)
    ch = s.channels
    o9 = oracle.OracleSystem(9, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                             e_ch=s.e_ch, vec1=s.vec1.reshape(-1), ldv=s.ldv)
    o0 = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                             e_ch=s.e_ch, vec1=s.vec1.reshape(-1), vec2=s.vec2.reshape(-1),
                             ldv=s.ldv)
    return s, o9, o0


def test_type9_levels_states_and_records(mq, oracle):
    s = mq.CollisionSystem(9, CHANS, **ABC)
    for i, c in enumerate(CHANS):
        e1, _ = mq.asym_top_level(ABC["A"], ABC["B"], ABC["C"], *c[:3])
        j, k = c[3], c[4]
        assert abs(s.e_ch[i] - (e1 + ABC["A2"] * j * (j + 1) - (ABC["A2"] - ABC["C2"]) * k * k)) < 1e-12
    assert s.n_states == sum(2 * js + 1 for c in CHANS for js in range(abs(c[0] - c[3]), c[0] + c[3] + 1))
    rec = s.state_records()
    assert rec.shape[1] == 10 and np.array_equal(rec[:, 4:], s.channels[s.indx_chann - 1])
    ic, j12, m12, _ = systems(mq, oracle)[1].states()
    assert np.array_equal(ic, s.indx_chann) and np.array_equal(j12, s.j12)
    assert np.array_equal(m12, s.m12)
    with pytest.raises(ValueError):
        mq.CollisionSystem(9, [(0, 0, 0, 1, 0, 1)], **ABC)


def test_type9_mtrx_dat_columns(mq, tmp_path):
    s = mq.CollisionSystem(9, CHANS[:3], **ABC)
    R = np.array([4.0, 5.0])
    mat = np.arange(s.P * 2, dtype=float).reshape(s.P, 2)
    path = str(tmp_path / "MTRX.DAT")
    mq.write_mtrx_dat(path, s, R, mat)
    lines = open(path).read().split("\n")
    assert lines[5] == "  #STATE #CHANNEL J12 M12  J1 K1A K1C  J2  K2 EPS"
    assert lines[6] == "       1        1   0   0   0   0   0   0   0   0"
    d = mq.read_mtrx_dat(path)
    assert np.array_equal(d["mat"], mat)


def test_type9_expansion_equals_type0_of_the_parity_vectors(mq, oracle):
    s, o9, o0 = systems(mq, oracle)
    R = np.array([5.0, 7.0, 9.0])
    T = np.random.default_rng(9).normal(size=(len(R), len(LABELS))) * 100
    m9 = oracle.expansion_matrix_type0(o9, o9.states(), s.ind_mat, LABELS, T, CM)
    m0 = oracle.expansion_matrix_type0(o0, o0.states(), s.ind_mat, LABELS, T, CM)
    assert np.abs(m9).max() > 0
    assert np.max(np.abs(m9 - m0)) <= 1e-13 * np.abs(m0).max()


def test_type9_direct_quadrature_and_expansion(mq, oracle):
    """Direct quadrature of WF_ASYM_TOP_SYM_TOP (case 9) against case 0 with the parity
    vectors, and against the case-9 expansion for V = sum_t v_t W_t."""
    from test_oracle_projection import _basis

    s, o9, o0 = systems(mq, oracle, CHANS[:5])
    shape = (6, 14, 14, 6, 6)
    W = _basis(oracle, 0, LABELS[:10], shape)
    R = np.array([5.0, 8.0])
    v = np.random.default_rng(4).normal(size=(10, len(R))) * 100.0
    V = np.einsum("tr,t...->r...", v, W)
    pes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
    n2, n3, n4, n5, n6 = shape
    g = (n3, n5, 0, n4, n2, n6, 1)
    d9, _, _ = oracle.build_matrix(o9, o9.states(), s.ind_mat, R, g, pes, mij_cut=0.0)
    d0, _, _ = oracle.build_matrix(o0, o0.states(), s.ind_mat, R, g, pes, mij_cut=0.0)
    assert np.max(np.abs(d9 - d0)) <= 1e-13 * np.abs(d0).max()
    e9 = oracle.expansion_matrix_type0(o9, o9.states(), s.ind_mat, LABELS[:10],
                                       np.ascontiguousarray(v.T), CM)
    assert np.max(np.abs(d9 - e9)) <= 1e-10 * np.abs(d9).max()


def test_type9_second_top_constants_follow_the_reference(mq):
    """A2 = B2 of the symmetric top: given as B2 alone (the reference's input form) it
    gives the same levels as A2; neither, or no C2, is an error (iotest.f:9414-9416)."""
    base = dict(A=27.9, B=14.5, C=9.3)
    s_a = mq.CollisionSystem(9, CHANS, A2=9.94, C2=6.23, **base)
    s_b = mq.CollisionSystem(9, CHANS, B2=9.94, C2=6.23, **base)
    assert np.array_equal(s_a.e_ch, s_b.e_ch)
    # distinct constants for the two molecules change the symmetric-top part only
    s_c = mq.CollisionSystem(9, CHANS, B2=5.0, C2=3.0, **base)
    for i, c in enumerate(CHANS):
        e1, _ = mq.asym_top_level(27.9, 14.5, 9.3, *c[:3])
        j, k = c[3], c[4]
        assert abs(s_c.e_ch[i] - (e1 + 5.0 * j * (j + 1) - (5.0 - 3.0) * k * k)) < 1e-12
    with pytest.raises(ValueError):
        mq.CollisionSystem(9, CHANS, C2=6.23, **base)
    with pytest.raises(ValueError):
        mq.CollisionSystem(9, CHANS, A2=9.94, **base)
