"""Formatted matrix and expansion-term files of the library's host side: MTRX.DAT as
PRINT_MIJ writes it and READ_MIJ reads it (SAVE_MTRX / READ_MTRX with UNFORMAT = NO,
MQCT_SOURCE_CODES/matrix_ini.f:4692-4877) and PES_EXPAN_TERMS.DAT as
READ_EXPANSION_TERMS reads it (MQCT_SOURCE_CODES/pot_comp.f:6344-6388).

The reference's own H2O + H2 matrix (G3 fixture, parsed from its MTRX.DAT) written
by the library reproduces the lines of that file; files round-trip bit for bit; the
oracle's independent reader agrees."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _g3_system(mq):
    g = np.load(os.path.join(GOLD, "g3_h2o_h2_type8.npz"))
    s = mq.CollisionSystem(8, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           BE=float(g["BE"]))
    return g, s


def test_mtrx_dat_lines_match_the_reference_file(mq, tmp_path):
    g, s = _g3_system(mq)
    path = str(tmp_path / "MTRX.DAT")
    mq.write_mtrx_dat(path, s, g["R"], g["mat"])
    lines = open(path).read().splitlines()
    # lines of EXAMPLES_IO/SYS_TYPE_8/H2O_H2_Dynamics/MTRX.DAT
    assert lines[:7] == ["COLLISION_TYPE= 8", "NUMBER_OF_CHANLS=   10",
                         "NUMBER_OF_STATES=    104", "MATRIX_SIZE=       891",
                         "R_GRID_SIZE=  101",
                         "  #STATE #CHANNEL      J12      M12       J1      K1A      K1C       J2",
                         "       1        1        0        0        0        0        0        0"]
    assert lines[110:112] == ["       MIJ_INDEX     ST_1     ST_2",
                              "               1        1        1"]
    assert lines[1002:1005] == ["  #iR           R_COM(iR)", "    1  0.300000000000E+01",
                                "    2  0.327000000000E+01"]
    assert lines[1104:1107] == ["        #k_matel      #iR     Mij(iR,k_matel)",
                                "               1        1  0.105476646204E+00",
                                "               1        2  0.658040166253E-01"]
    assert len(lines) == 91096


def test_mtrx_dat_round_trip_and_oracle_reader(mq, oracle, tmp_path):
    g, s = _g3_system(mq)
    path = str(tmp_path / "MTRX.DAT")
    mq.write_mtrx_dat(path, s, g["R"], g["mat"])
    d = mq.read_mtrx_dat(path)
    assert d["coll_type"] == 8 and d["n_channels"] == 10
    assert np.array_equal(d["states"], g["states"]) and np.array_equal(d["ind_mat"], g["ind_mat"])
    # the fixture holds the file's 12-digit values: the round trip is exact
    assert np.array_equal(d["R"], g["R"]) and np.array_equal(d["mat"], g["mat"])
    o = oracle.read_mtrx_dat(path, 8)
    assert np.array_equal(o["mat"], d["mat"]) and np.array_equal(o["ind_mat"], d["ind_mat"])


def test_fortran_e_format_edge_cases(mq, tmp_path):
    s = mq.CollisionSystem(1, [[0], [1]], BE=1.0)
    R = np.array([1.0, 2.0])
    vals = np.array([0.0, -1.0, 0.99999999999995, 9.99999999999951e5, 1.23456789012345e-120,
                     -4.5e150, 5e-324, 1.0 / 3.0])
    mat = np.resize(vals, s.P * 2).reshape(s.P, 2)
    path = str(tmp_path / "m.dat")
    mq.write_mtrx_dat(path, s, R, mat)
    text = open(path).read()
    assert " 0.100000000000E+01" in text           # 0.99999999999995 rounds up a digit
    assert "0.123456789012-119" in text           # three-digit exponent drops the letter
    d = mq.read_mtrx_dat(path)
    expect = np.array([float(f"{v:.11e}") for v in mat.reshape(-1)]).reshape(mat.shape)
    assert np.array_equal(d["mat"], expect)


def test_expansion_terms_reader(mq, tmp_path):
    g5 = np.load(os.path.join(GOLD, "g5_h2o_h2_expansion_terms.npz"))
    R, T, lab = g5["R"], g5["terms"], g5["labels"]
    path = str(tmp_path / "PES_EXPAN_TERMS.DAT")
    with open(path, "w") as f:   # the layout the reference reads: f6.2, then e19.12 values
        f.write("R_Bohr " + " ".join("v_" + "_".join(map(str, l)) for l in lab) + "\n")
        for i in range(len(R)):
            f.write(f"{R[i]:6.2f} " + "   ".join(f"{v: .12E}" for v in T[i]) + "\n")
    R2, T2 = mq.read_expansion_terms(path, len(R), len(lab))
    assert np.array_equal(R2, R) and np.array_equal(T2, T)
    with pytest.raises(mq.MqctError):
        mq.read_expansion_terms(path, len(R) + 1, len(lab))      # one R point too many
    with pytest.raises(mq.MqctError):
        mq.read_expansion_terms(path, len(R), len(lab) + 1)      # one term too many


def test_malformed_mtrx_dat_is_rejected(mq, tmp_path):
    g, s = _g3_system(mq)
    path = str(tmp_path / "MTRX.DAT")
    mq.write_mtrx_dat(path, s, g["R"], g["mat"])
    lines = open(path).read().splitlines()
    bad = str(tmp_path / "bad.dat")
    open(bad, "w").write("\n".join(lines[:-5]) + "\n")            # truncated elements
    with pytest.raises(mq.MqctError):
        mq.read_mtrx_dat(bad)
    open(bad, "w").write("\n".join(["NUMBER_OF_CHANLS=   10"] + lines[1:]) + "\n")
    with pytest.raises(mq.MqctError):
        mq.read_mtrx_dat(bad)


def test_expansion_term_lists_match_the_reference(mq, tmp_path):
    """CALC_EXPANSION's term lists for the two generating examples, and the file layout."""
    g = np.load(os.path.join(GOLD, "g6_expansion_term_lists.npz"))
    t8 = mq.expansion_terms_list(8, 4, 4, nju1_max=4, axl_sym1=2, equ_sym2=2, odd_l1l2l=True)
    assert np.array_equal(t8, g["h2o_h2_type8"])
    t7 = mq.expansion_terms_list(7, 4, 2, nju1_max=3)
    assert np.array_equal(t7, g["nh3_h2_type7"])
    path = str(tmp_path / "EXPANSION_TERMS_LIST.DAT")
    mq.write_expansion_terms_list(path, t7)
    lines = open(path).read().splitlines()
    assert lines[:2] == ["0,0,0,0,", "0,0,1,1,"] and lines[-1] == "4,3,2,6,"
    assert len(lines) == 79
