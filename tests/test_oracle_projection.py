"""CALC_EXPANSION_TERMS (MQCT_SOURCE_CODES/pot_comp.f:4695-6274): the oracle's
projection of a tabulated PES onto the expansion terms, and the PES_EXPAN_TERMS.DAT
writer.

The reference's examples of the projection evaluate user PES routines written in Fortran,
so no printed projection can be replayed here.  The projection is pinned instead by
(a) a known answer: the angular functions of EXPANSION_TERM are orthonormal on the
reference's grids, so a PES built from them projects back onto its coefficients, with
the factor 1/2 of the real part for terms with nju != 0; and (b) a cross-path check:
for such a PES the state-to-state matrix of the direct quadrature (INTEGRATOR_TEMP,
pinned by the reference's MTRX.DAT files) equals the matrix built from the projected
terms by EXPANSION_MATRIX_ELEMENT (pinned by the H2O+H2O example), so the projection
uses the convention the reference's matrix formula reads its terms in.  The writer is
pinned byte for byte by the two PES_EXPAN_TERMS.DAT files of
EXAMPLES_IO/SYS_TYPE_7/NH3_H2_IR_BGN_FIN (fixture tests/golden/g7_expan_terms_files.npz)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CM = 1.0 / 8065.5448 / 27.21113845


def _gl(n):
    x, _ = np.polynomial.legendre.leggauss(n)
    return np.pi / 2 + np.pi / 2 * x


def _eq(n):
    return (np.arange(n) + 0.5) * 2 * np.pi / n


def _basis(oracle, sys_type, labels, shape):
    """W_t on the grid: Re EXPANSION_TERM_t, doubled when nju1 or nju2 != 0, so that the
    PES sum_t v_t W_t has the coefficients v_t."""
    n2, n3, n4, n5 = shape[:4]
    n6 = shape[4] if sys_type == 0 else 1
    b1, b2, g1, a2, g2 = _gl(n3), _gl(n4), _eq(n5), _eq(n2), _eq(n6)
    W = np.zeros((len(labels), n2, n3, n4, n5, n6))
    for t, lab in enumerate(labels):
        if sys_type == 0:
            l1, nu1, l2, nu2, l = lab
        else:
            (l1, nu1, l2, l), nu2 = lab, 0
        f = 1.0 if nu1 == 0 and nu2 == 0 else 2.0
        for i2 in range(n2):
            for i3 in range(n3):
                for i4 in range(n4):
                    for i5 in range(n5):
                        for i6 in range(n6):
                            r, _ = oracle.expansion_term(sys_type, l, l1, l2, nu1, nu2, b1[i3],
                                                         g1[i5], a2[i2], b2[i4],
                                                         g2[i6] if sys_type == 0 else 0.0)
                            W[t, i2, i3, i4, i5, i6] = f * r
    return W if sys_type == 0 else W[..., 0]


LAB8 = [(0, 0, 0, 0), (1, 0, 0, 1), (1, 1, 0, 1), (2, 2, 2, 4), (2, 1, 1, 2), (3, 3, 2, 1),
        (2, 0, 2, 2), (2, 0, 2, 0)]
LAB0 = [(0, 0, 0, 0, 0), (1, 0, 1, 0, 0), (1, 0, 1, 0, 2), (2, 0, 0, 0, 2), (2, 2, 0, 0, 2),
        (0, 0, 2, 2, 2), (2, 1, 1, 1, 2), (1, 1, 1, -1, 2), (2, 2, 2, -2, 4), (2, 0, 2, 0, 0),
        (1, 0, 0, 0, 1), (2, 1, 1, 0, 3)]


@pytest.mark.parametrize("sys_type,labels,shape", [(8, LAB8, (8, 14, 14, 8)),
                                                   (7, LAB8, (8, 14, 14, 8)),
                                                   (0, LAB0, (6, 14, 14, 6, 6))])
def test_projection_recovers_the_coefficients(oracle, sys_type, labels, shape):
    W = _basis(oracle, sys_type, labels, shape)
    rng = np.random.default_rng(5)
    v = rng.normal(size=(len(labels), 3)) * 100.0
    V = np.einsum("tr,t...->r...", v, W)
    T, Ti = oracle.project_terms(sys_type, labels, V)
    assert np.max(np.abs(T - v)) <= 1e-11 * np.abs(v).max()
    assert np.max(np.abs(Ti)) <= 1e-11 * np.abs(v).max()


def test_projection_of_one_term_is_one_or_one_half(oracle):
    """Re Y_s projects onto s alone, with 1 for nju = 0 and 1/2 otherwise (the conjugate
    partner -nju is not in a valid term list); odd l1 + l2 + l with nju = 0 has Re Y = 0."""
    labels = LAB8
    W = _basis(oracle, 8, labels, (8, 14, 14, 8))
    for s, lab in enumerate(labels):
        re_y = W[s] if lab[1] == 0 else 0.5 * W[s]
        T, _ = oracle.project_terms(8, labels, re_y[None])
        want = np.zeros(len(labels))
        want[s] = 1.0 if lab[1] == 0 else 0.5
        assert np.allclose(T[:, 0], want, atol=1e-11), (lab, T[:, 0])
    r, i = oracle.expansion_term(8, 1, 1, 1, 0, 0, 0.7, 1.1, 0.3, 2.0)  # l1 + l2 + l odd
    assert abs(r) < 1e-15 and abs(i) > 1e-3


def test_projection_agrees_with_the_direct_quadrature(mq, oracle):
    """Type 0, H2O+H2O: for V = sum_t v_t W_t on the 5-D grid, Mat_el of INTEGRATOR_TEMP
    with V tabulated equals EXPANSION_MATRIX_ELEMENT of the projected terms."""
    g = np.load(os.path.join(GOLD, "g1_h2o_h2o_at.npz"))
    s = mq.CollisionSystem(0, g["channels"][:4], A=float(g["A"]), B=float(g["B"]),
                           C=float(g["C"]))
    ch = s.channels
    osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                               e_ch=s.e_ch, vec1=s.vec1.reshape(-1), vec2=s.vec2.reshape(-1),
                               ldv=s.ldv)
    shape = (8, 14, 14, 8, 8)
    W = _basis(oracle, 0, LAB0, shape)
    R = np.array([5.0, 6.5, 8.0])
    v = np.random.default_rng(3).normal(size=(len(LAB0), len(R))) * 100.0
    V = np.einsum("tr,t...->r...", v, W)
    T, _ = oracle.project_terms(0, LAB0, V)
    st = osys.states()
    pes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
    n2, n3, n4, n5, n6 = shape
    direct, _, _ = oracle.build_matrix(osys, st, s.ind_mat, R, (n3, n5, 0, n4, n2, n6, 1), pes,
                                       mij_cut=0.0)
    expan = oracle.expansion_matrix_type0(osys, st, s.ind_mat, LAB0,
                                          np.ascontiguousarray(T.T), CM)
    assert np.max(np.abs(direct - expan)) <= 1e-10 * np.abs(direct).max()


def _rows(lines):
    out = []
    for ln in lines[1:]:
        if ln.strip():
            out.append([float(x) for x in ln.split()])
    return np.array(out)


def test_expansion_terms_file_is_written_as_the_reference_writes_it(mq, tmp_path):
    g = np.load(os.path.join(GOLD, "g7_expan_terms_files.npz"))
    ref = "\n".join(str(x) for x in g["lines_1_20"])
    src = tmp_path / "ref.DAT"
    src.write_text(ref)
    R, T = mq.read_expansion_terms(str(src), 20, len(g["labels"]))
    out = tmp_path / "PES_EXPAN_TERMS.DAT"
    mq.write_expansion_terms(str(out), 7, g["labels"], R, T)
    assert out.read_text() == ref


def test_expansion_terms_file_appends_over_r_ranges(mq, tmp_path):
    """IR_BGN/IR_FIN runs append to one file: the header once, then the rows in order."""
    g = np.load(os.path.join(GOLD, "g7_expan_terms_files.npz"))
    out = tmp_path / "PES_EXPAN_TERMS.DAT"
    for key in ("lines_1_20", "lines_21_40"):
        src = tmp_path / f"{key}.DAT"
        src.write_text("\n".join(str(x) for x in g[key]))
        R, T = mq.read_expansion_terms(str(src), 20, len(g["labels"]))
        mq.write_expansion_terms(str(out), 7, g["labels"], R, T)
    lines = out.read_text().split("\n")
    assert lines[0] == str(g["lines_1_20"][0])
    assert lines[1:21] == [str(x) for x in g["lines_1_20"][1:21]]
    assert lines[21:41] == [str(x) for x in g["lines_21_40"][1:21]]
    assert sum(ln.startswith("R_Bohr") for ln in lines) == 1


def test_type0_header_labels(mq, tmp_path):
    out = tmp_path / "PES_EXPAN_TERMS.DAT"
    mq.write_expansion_terms(str(out), 0, [(1, 0, 1, 0, 0), (12, 11, 10, -9, 20)], [3.0],
                             [[1.5, -2.0e-7]])
    head, row = out.read_text().split("\n")[:2]
    assert head == "R_Bohr " + "v_1_0_1_0_0".rjust(19) + "   " + "v_12_11_10_-9_20".rjust(19) + "   "
    assert row == "  3.00 " + " 0.150000000000E+01   " + "-0.200000000000E-06   "


@pytest.mark.parametrize("sys_type,labels,msg", [
    (8, [(1, 0, 1, 3)], "TRIANGULAR"),
    (8, [(1, 1, 1, 2), (1, -1, 1, 2)], "M1 should be always positive"),
    (0, [(1, 0, 1, -1, 2)], "M2 should be positive only for M1 = 0"),
    (8, [(2, 1, 1, 2), (2, 1, 1, 2)], "two same terms"),
    (7, [(2, 3, 1, 2)], "exceeds its l"),
])
def test_term_list_checks(mq, sys_type, labels, msg):
    shape = (1, 2, 3, 3, 2) + ((2,) if sys_type == 0 else ())
    with pytest.raises(mq.MqctError, match=msg):
        mq.project_terms(sys_type, labels, np.zeros(shape))


def test_identical_term_list_checks(mq):
    V = np.zeros((1, 2, 3, 3, 2, 2))
    with pytest.raises(mq.MqctError, match="L2 should be less or equal to L1"):
        mq.project_terms(0, [(1, 0, 2, 1, 2)], V, identical=True)
    with pytest.raises(mq.MqctError, match=r"greater or equal to abs\(M2\)"):
        mq.project_terms(0, [(2, 0, 2, 1, 2)], V, identical=True)
    with pytest.raises(mq.MqctError, match="SYS_TYPE 0"):
        mq.project_terms(8, [(1, 0, 1, 2)], np.zeros((1, 2, 3, 3, 2)), identical=True)
