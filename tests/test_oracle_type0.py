"""Known answer for the two-rotor (SYS_TYPE 0) integration of the oracle: with a
constant surface V = 1 cm^-1 the matrix is the overlap of the coupled basis,
M_ij = delta_ij (in Hartree), once the 5-D grid resolves the products of the
basis functions (GL in both beta; midpoint alpha2, gamma1, gamma2 with more
points than the largest K or m difference)."""
import numpy as np

from mqct_b200 import synthetic as syn


def _type0_system(mq, oracle, jmax=1):
    chans = [a + b for a in syn.asym_channels(jmax) for b in syn.asym_channels(jmax)]
    s = mq.CollisionSystem(0, chans, A=27.9, B=14.5, C=9.3)
    ch = s.channels
    osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                               e_ch=s.e_ch, vec1=s.vec1.reshape(-1), vec2=s.vec2.reshape(-1),
                               ldv=s.ldv)
    return s, osys


def test_type0_states_match_product(mq, oracle):
    s, osys = _type0_system(mq, oracle)
    ic, j12, m12, _ = osys.states()
    assert s.n_states == 100 and np.array_equal(ic, s.indx_chann)
    assert np.array_equal(j12, s.j12) and np.array_equal(m12, s.m12)


def test_type0_constant_surface_gives_identity(mq, oracle):
    s, osys = _type0_system(mq, oracle)
    grid = (12, 4, 0, 12, 4, 4, 1)
    R = np.array([5.0, 6.0, 7.0, 8.0])
    G = 12 * 4 * 12 * 4 * 4
    pes = oracle.OraclePes(0, 0, np.zeros(1), table=np.ones(len(R) * G))
    m, _, _ = oracle.build_matrix(osys, osys.states(), s.ind_mat, R, grid, pes, mij_cut=0.0)
    diag = s.ind_mat[:, 0] == s.ind_mat[:, 1]
    m = m / syn.CM_TO_HARTREE
    assert np.max(np.abs(m[diag] - 1.0)) < 1e-12
    assert np.max(np.abs(m[~diag])) < 1e-12
