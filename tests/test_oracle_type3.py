"""SYS_TYPE 3, a rigid symmetric top + an atom: channels (j, k, eps) with levels
A j(j+1) - (A-C) k^2 (MQCT_SOURCE_CODES/iotest.f:6250, 6355), states m = -j..j
(matrix_ini.f:302-310), MTRX.DAT columns J K EPS (matrix_ini.f:4744-4751), and the
expansion matrix of pot_comp.f:6846-6954.

The reference ships no SYS_TYPE 3 matrix (its C6H6+He example has one channel and
integrates the PES directly), so the type-3 formula is tied to the type-4 formula of the
same parity-adapted top vectors (|j k> + (-1)^eps |j -k>) / sqrt(2 (1 + delta_k0)).  The
two differ only in the factor of their -nju branch, as written in the reference: type 4
takes (-1)^nju (-1)^nju = 1, type 3 takes (-1)**(-1)**nju (-1)^nju = -(-1)^nju.  With
the symmetry <j' -K l -nju|j'' -K-nju> = (-1)^(j'+l-j'') <j' K l nju|j'' K+nju> of the
Clebsch-Gordan coefficients, the -nju branch of parity-adapted vectors equals
s = (-1)^(j'+l-j''+eps'+eps'') times the +nju branch, so:
  nju = 0 or odd:    M3 = M4;
  nju even, > 0:     M3 = b (1 - s), M4 = b (1 + s): one of the two vanishes."""
import os

import numpy as np
import pytest

CM = 1.0 / 8065.5448 / 27.21113845
A3, C3 = 0.18960, 0.09480      # C6H6 (cm^-1), the reference's SYS_TYPE 3 example
CHANS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (1, 1, 1), (2, 0, 0), (2, 1, 0), (2, 1, 1),
         (2, 2, 0), (2, 2, 1), (3, 0, 0), (3, 2, 1), (3, 3, 0), (3, 3, 1)]
LABELS = [(0, 0), (1, 0), (2, 0), (1, 1), (2, 1), (3, 1), (2, 2), (3, 2), (4, 2), (3, 3),
          (4, 4), (6, 6), (5, 3)]


def systems(mq, oracle):
    s = mq.CollisionSystem(3, CHANS, A=A3, C=C3)
    ch = s.channels
    o3 = oracle.OracleSystem(3, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=s.e_ch)
    o4 = oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=s.e_ch,
                             vec1=s.vec1.reshape(-1), ldv=s.ldv)
    return s, o3, o4


def test_type3_levels_states_and_records(mq, oracle):
    s = mq.CollisionSystem(3, CHANS, A=A3, C=C3)
    j = np.array([c[0] for c in CHANS], float)
    k = np.array([c[1] for c in CHANS], float)
    assert np.allclose(s.e_ch, A3 * j * (j + 1) - (A3 - C3) * k ** 2, rtol=0, atol=1e-15)
    assert s.n_states == sum(2 * c[0] + 1 for c in CHANS)
    ic, j12, m12, _ = oracle.OracleSystem(3, s.channels[:, 0], s.channels[:, 1],
                                          s.channels[:, 2], e_ch=s.e_ch).states()
    assert np.array_equal(ic, s.indx_chann) and np.array_equal(m12, s.m12)
    assert np.array_equal(j12, s.j12)
    rec = s.state_records()
    assert rec.shape[1] == 7 and np.array_equal(rec[:, 4:], s.channels[s.indx_chann - 1])
    # the parity-adapted vectors are normalised
    assert np.allclose(np.sum(s.vec1 ** 2, axis=1), 1.0)
    with pytest.raises(ValueError):
        mq.CollisionSystem(3, [(1, 0, 1)], A=A3, C=C3)    # k = 0 has eps = 0 only


def test_type3_mtrx_dat_columns(mq, tmp_path):
    s = mq.CollisionSystem(3, CHANS[:4], A=A3, C=C3)
    R = np.array([4.0, 5.0])
    mat = np.arange(s.P * 2, dtype=float).reshape(s.P, 2)
    path = str(tmp_path / "MTRX.DAT")
    mq.write_mtrx_dat(path, s, R, mat)
    text = open(path).read()
    assert "K" in text and "EPS" in text
    d = mq.read_mtrx_dat(path)
    assert np.array_equal(d["mat"], mat)


def test_type3_formula_against_type4_of_the_same_vectors(mq, oracle):
    s, o3, o4 = systems(mq, oracle)
    R = np.array([5.0, 7.0])
    T = np.random.default_rng(6).normal(size=(len(R), len(LABELS))) * 100
    st = o3.states()
    for t, (l, nu) in enumerate(LABELS):
        Tt = np.zeros_like(T)
        Tt[:, t] = T[:, t]
        m3 = oracle.expansion_matrix_atom(o3, st, s.ind_mat, LABELS, Tt, CM)
        m4 = oracle.expansion_matrix_atom(o4, o4.states(), s.ind_mat, LABELS, Tt, CM)
        scale = max(np.abs(m4).max(), np.abs(m3).max(), 1e-300)
        if nu == 0 or nu % 2:
            assert np.max(np.abs(m3 - m4)) <= 1e-13 * scale, (l, nu)
        else:
            assert np.max(np.abs(m3 * m4)) <= 1e-13 * scale ** 2, (l, nu)
            assert np.abs(m3).max() > 0 and np.abs(m4).max() > 0, (l, nu)


def _pes_from_terms(mq, oracle, labels, grid, R, seed):
    """V = sum_t v_t (Y_{l nju} + Y*_{l nju}) on the (beta, gamma) grid (Y for nju = 0)."""
    from test_oracle_expansion_atom import term_table

    W = term_table(oracle, labels, grid, 4)
    v = np.random.default_rng(seed).normal(size=(len(labels), len(R))) * 100
    return v, np.einsum("tr,t...->r...", v, W)


def test_type3_direct_quadrature_agrees_with_type4_of_the_same_vectors(mq, oracle):
    """INTEGRATOR_TEMP case 3 (WF_SYM_TOP, pot_comp.f:2259-2303) equals case 4 with the
    parity-adapted vectors, for a PES with all nju."""
    s, o3, o4 = systems(mq, oracle)
    R = np.array([5.0, 7.0])
    grid = (16, 14)
    _, V = _pes_from_terms(mq, oracle, LABELS, grid, R, 7)
    pes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
    g = grid + (0, 0, 0, 0, 1)
    m3, _, _ = oracle.build_matrix(o3, o3.states(), s.ind_mat, R, g, pes, mij_cut=0.0)
    m4, _, _ = oracle.build_matrix(o4, o4.states(), s.ind_mat, R, g, pes, mij_cut=0.0)
    assert np.max(np.abs(m3 - m4)) <= 1e-13 * np.abs(m4).max()


def test_type3_direct_and_expansion_paths(mq, oracle):
    """The direct quadrature of V = sum_t v_t (Y + Y*) equals the case-3 expansion formula
    for terms with nju = 0 or odd nju, and the case-4 formula of the same vectors for all
    terms: the -nju factor of case 3 breaks the direct/expansion agreement at even nju > 0,
    as written in the reference."""
    s, o3, o4 = systems(mq, oracle)
    R = np.array([5.0, 7.0])
    grid = (20, 24)
    g = grid + (0, 0, 0, 0, 1)
    for labels, ok3 in (([lab for lab in LABELS if lab[1] == 0 or lab[1] % 2], True),
                        (LABELS, False)):
        v, V = _pes_from_terms(mq, oracle, labels, grid, R, 8)
        pes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
        direct, _, _ = oracle.build_matrix(o3, o3.states(), s.ind_mat, R, g, pes, mij_cut=0.0)
        e4 = oracle.expansion_matrix_atom(o4, o4.states(), s.ind_mat, labels,
                                          np.ascontiguousarray(v.T), CM)
        e3 = oracle.expansion_matrix_atom(o3, o3.states(), s.ind_mat, labels,
                                          np.ascontiguousarray(v.T), CM)
        tol = 1e-10 * np.abs(direct).max()
        assert np.max(np.abs(direct - e4)) <= tol
        assert (np.max(np.abs(direct - e3)) <= tol) == ok3


def test_type3_orthonormal_functions(mq, oracle):
    """V = 1: the direct quadrature gives the unit matrix in Hartree per cm^-1 (Gauss-Legendre
    in beta itself integrates the trigonometric integrand to 1e-12 from 30 points)."""
    s, o3, _ = systems(mq, oracle)
    R = np.array([5.0, 6.0])
    grid = (30, 14)
    V = np.ones((len(R),) + grid)
    pes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
    m, _, _ = oracle.build_matrix(o3, o3.states(), s.ind_mat, R, grid + (0, 0, 0, 0, 1), pes,
                                  mij_cut=0.0)
    diag = s.ind_mat[:, 0] == s.ind_mat[:, 1]
    assert np.allclose(m[diag], CM, rtol=1e-12, atol=0)
    assert np.max(np.abs(m[~diag])) <= 1e-13 * CM
