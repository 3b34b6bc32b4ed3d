"""Two diatoms (SYS_TYPE 5, distinguishable partners): states (MQCT_SOURCE_CODES/
matrix_ini.f:323-336), energies BE1 j1(j1+1) - DE1 (j1(j1+1))^2 + BE2 j2(j2+1) - ..., and
the expansion matrix of EXPANSION_MATRIX_ELEMENT case 5 (pot_comp.f:7076-7386), which is
case 8 with a diatom for the first rotor.  No reference example prints a SYS_TYPE 5
matrix; the restatement is tied to the pinned SYS_TYPE 0 formula (G1, G5c): for two
linear rotors (one K = 0 component each) the type-0 element equals the type-5 one divided
by 2 pi (the terms' 8 pi^2 and 4 pi normalisations)."""
import numpy as np

CM = 1.0 / 8065.5448 / 27.21113845
CHANS = [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (0, 2), (2, 1), (1, 2), (2, 2)]
LABS = [(0, 0, 0), (1, 0, 1), (0, 1, 1), (1, 1, 0), (1, 1, 2), (2, 0, 2), (2, 2, 4), (2, 1, 3),
        (2, 2, 0)]


def type5_oracle(mq, oracle):
    s = mq.CollisionSystem(5, CHANS, BE=1.92, DE=6e-6)
    ch = s.channels
    j1, j2 = ch[:, 0], ch[:, 1]
    n = len(ch)
    unit1 = np.zeros((n, s.ldv))
    unit1[np.arange(n), j1] = 1.0
    o8 = oracle.OracleSystem(8, j1, np.zeros(n, np.int32), j1, j2, e_ch=s.e_ch,
                             vec1=unit1.reshape(-1), ldv=s.ldv)
    return s, o8, unit1


def test_type5_states_and_levels(mq):
    s = mq.CollisionSystem(5, CHANS, BE=1.92, DE=6e-6, BE2=2.0, DE2=0.0)
    want = sum(2 * js + 1 for j1, j2 in CHANS for js in range(abs(j1 - j2), j1 + j2 + 1))
    assert s.n_states == want
    jj1 = np.array([a * (a + 1.0) for a, _ in CHANS])
    jj2 = np.array([b * (b + 1.0) for _, b in CHANS])
    assert np.allclose(s.e_ch, 1.92 * jj1 - 6e-6 * jj1 ** 2 + 2.0 * jj2)
    rec = s.state_records()
    assert rec.shape[1] == 6 and np.array_equal(rec[:, 4:], s.channels[s.indx_chann - 1])


def test_type5_matches_the_type0_formula_for_linear_rotors(mq, oracle):
    s, o8, unit1 = type5_oracle(mq, oracle)
    ch = s.channels
    n = len(ch)
    unit2 = np.zeros_like(unit1)
    unit2[np.arange(n), ch[:, 1]] = 1.0
    R = np.array([5.0, 7.0, 9.0])
    T = np.random.default_rng(3).normal(size=(len(R), len(LABS))) * 100
    m5 = oracle.expansion_matrix_type8(o8, o8.states(), s.ind_mat, [(a, 0, b, c) for a, b, c in LABS], T)
    o0 = oracle.OracleSystem(0, ch[:, 0], np.zeros(n, np.int32), ch[:, 0], ch[:, 1],
                             np.zeros(n, np.int32), ch[:, 1], e_ch=s.e_ch, vec1=unit1.reshape(-1),
                             vec2=unit2.reshape(-1), ldv=s.ldv)
    m0 = oracle.expansion_matrix_type0(o0, o0.states(), s.ind_mat,
                                       [(a, 0, b, 0, c) for a, b, c in LABS], T, CM)
    assert np.max(np.abs(m0 * 2 * np.pi - m5)) <= 1e-13 * np.abs(m5).max()
