"""The PES-expansion path of the oracle against the reference's own output: the
H2O + H2 (SYS_TYPE 8) matrix that the reference built from its expansion terms
(EXAMPLES_IO/SYS_TYPE_8/H2O_H2_MTRXCalculation: PES_EXPAN_TERMS.DAT -> MTRX.DAT, the
G3 matrix) is reproduced from the same terms.  The asymmetric-top eigenvector sign
is a free phase of each rotor level (LAPACK's choice in the reference, a fixed rule
here), so elements agree up to s_a s_b with one sign per level; the test finds the
signs, checks that one sign per level explains every element, then compares."""
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def level_gauge(system, mat, ref, tol=1e-9):
    """Per-pair sign s_a s_b (one sign per rotor-1 level) that maps ref onto mat;
    asserts that such signs exist."""
    ch = system.channels
    ic = system.indx_chann
    lev = {}
    for c in range(system.n_channels):
        lev.setdefault(tuple(ch[c, :3]), len(lev))
    clev = np.array([lev[tuple(ch[c, :3])] for c in range(system.n_channels)])
    la = clev[ic[system.ind_mat[:, 0] - 1] - 1]
    lb = clev[ic[system.ind_mat[:, 1] - 1] - 1]
    rowmax = np.abs(ref).max(axis=1)
    sig = rowmax > tol * rowmax.max()
    psign = np.zeros(len(la))
    for k in np.nonzero(sig)[0]:
        i = np.argmax(np.abs(ref[k]))
        psign[k] = np.sign(mat[k, i] / ref[k, i])
    sg = {}
    for root in range(len(lev)):
        if root in sg:
            continue
        sg[root] = 1.0
        changed = True
        while changed:
            changed = False
            for k in np.nonzero(psign)[0]:
                x, y = la[k], lb[k]
                if x in sg and y not in sg:
                    sg[y] = sg[x] * psign[k]
                    changed = True
                if y in sg and x not in sg:
                    sg[x] = sg[y] * psign[k]
                    changed = True
    gauge = np.array([sg[la[k]] * sg[lb[k]] for k in range(len(la))])
    assert np.all(gauge[psign != 0] == psign[psign != 0]), "no per-level sign explains the signs"
    return gauge


def test_expansion_reproduces_reference_matrix(mq, oracle):
    g = np.load(os.path.join(GOLD, "g3_h2o_h2_type8.npz"))
    g5 = np.load(os.path.join(GOLD, "g5_h2o_h2_expansion_terms.npz"))
    assert np.array_equal(g5["R"], g["R"])
    s = mq.CollisionSystem(8, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           BE=float(g["BE"]))
    ch = s.channels
    osys = oracle.OracleSystem(8, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], e_ch=s.e_ch,
                               vec1=s.vec1.reshape(-1), ldv=s.ldv)
    m = oracle.expansion_matrix_type8(osys, osys.states(), s.ind_mat, g5["labels"], g5["terms"])
    ref = g["mat"]
    gauge = level_gauge(s, m, ref)
    assert (gauge < 0).any()  # the phase convention does differ for some levels
    assert np.max(np.abs(m - gauge[:, None] * ref)) <= 1e-10 * np.abs(ref).max()


def _g5b():
    return np.load(os.path.join(GOLD, "g5b_nd3_d2_type7.npz"))


def test_type7_levels_states_and_pairs(mq):
    """SYS_TYPE 7 (ND3 + D2): printed channel energies, the state table and the pair
    order of the reference's MTRX.DAT."""
    g = _g5b()
    s = mq.CollisionSystem(7, g["channels"], A=float(g["A"]), C=float(g["C"]), BE=float(g["BE"]))
    assert np.allclose(s.e_ch, g["e_ch_printed"], atol=1e-9)
    st = g["states"]
    assert s.n_states == 80 and s.P == 461
    assert (s.indx_chann == st[:, 1]).all() and (s.j12 == st[:, 2]).all()
    assert (s.m12 == st[:, 3]).all() and (s.ind_mat == g["ind_mat"]).all()
    assert (s.state_records()[:, 4:] == st[:, 4:]).all()   # J1, K, EPS, J2 columns


def test_type7_expansion_reproduces_reference_matrix(mq, oracle):
    g = _g5b()
    s = mq.CollisionSystem(7, g["channels"], A=float(g["A"]), C=float(g["C"]), BE=float(g["BE"]))
    ch = s.channels
    osys = oracle.OracleSystem(7, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], e_ch=s.e_ch, ldv=1)
    m = oracle.expansion_matrix_type7(osys, osys.states(), s.ind_mat, g["labels"], g["terms"],
                                      mq.E_UNIT["CM-1"])
    ref = g["mat"]
    assert np.max(np.abs(m - ref)) <= 1e-11 * np.abs(ref).max()


def test_type7_equals_type8_form_with_parity_adapted_vector(mq, oracle):
    """The reduction the GPU kernel uses: the four-term symmetric-top bracket of
    case 7 equals the K-sum of case 8 over the parity-adapted vector."""
    g = _g5b()
    s = mq.CollisionSystem(7, g["channels"], A=float(g["A"]), C=float(g["C"]), BE=float(g["BE"]))
    ch = s.channels
    o7 = oracle.OracleSystem(7, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], e_ch=s.e_ch, ldv=1)
    m7 = oracle.expansion_matrix_type7(o7, o7.states(), s.ind_mat, g["labels"], g["terms"], 1.0)
    o8 = oracle.OracleSystem(8, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], e_ch=s.e_ch,
                             vec1=s.vec1.reshape(-1), ldv=s.ldv)
    # the type-8 restatement works in cm^-1 and converts to Hartree itself
    m8 = oracle.expansion_matrix_type8(o8, o8.states(), s.ind_mat, g["labels"], g["terms"])
    assert np.max(np.abs(m8 / mq.E_UNIT["CM-1"] - m7)) <= 1e-12 * np.abs(m7).max()


def _g5c():
    return np.load(os.path.join(GOLD, "g5c_h2o_h2o_identical.npz"))


def identical_gauge(system, mat, ref):
    """Per-pair sign from one sign per rotor level (the eigenvector phase, LAPACK's in the
    reference, a fixed rule here), found over all level-sign choices; returns (gauge,
    max deviation relative to the largest element)."""
    import itertools
    ch = system.channels
    levels = sorted({tuple(c[:3]) for c in ch} | {tuple(c[3:]) for c in ch})
    ic, ind = system.indx_chann, system.ind_mat
    best = None
    for signs in itertools.product((1, -1), repeat=len(levels)):
        sg = dict(zip(levels, signs))
        cs = np.array([sg[tuple(c[:3])] * sg[tuple(c[3:])] for c in ch])
        gauge = cs[ic[ind[:, 0] - 1] - 1] * cs[ic[ind[:, 1] - 1] - 1]
        e = np.max(np.abs(mat - gauge[:, None] * ref)) / np.abs(ref).max()
        if best is None or e < best[1]:
            best = (gauge, e)
    return best


def test_identical_states_and_pairs(mq):
    """IDENTICAL = YES: the 81 parity-adapted states (with their exchange parity) and the
    322 equal-parity pairs of the reference's H2O + H2O MTRX.DAT."""
    g = _g5c()
    s = mq.CollisionSystem(0, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           identical=True)
    st = g["states"]
    assert s.n_states == 81 and s.P == 322
    assert np.array_equal(s.state_records(), st)
    assert np.array_equal(s.ind_mat, g["ind_mat"])


def test_identical_expansion_reproduces_reference_matrix(mq, oracle):
    g = _g5c()
    s = mq.CollisionSystem(0, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           identical=True)
    ch = s.channels
    osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                               e_ch=s.e_ch, vec1=s.vec1.reshape(-1), vec2=s.vec2.reshape(-1),
                               ldv=s.ldv)
    m = oracle.expansion_matrix_type0_identical(osys, (s.indx_chann, s.j12, s.m12, None),
                                                s.parity, s.ind_mat,
                                                g["labels"], g["terms"], mq.E_UNIT["KCAL"])
    gauge, err = identical_gauge(s, m, g["mat"])
    assert (gauge < 0).any()   # LAPACK's phases differ from the fixed rule for some levels
    assert err <= 1e-10


def test_identical_mtrx_dat_layout(mq, tmp_path):
    g = _g5c()
    s = mq.CollisionSystem(0, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           identical=True)
    path = str(tmp_path / "MTRX.DAT")
    mq.write_mtrx_dat(path, s, g["R"], g["mat"])
    lines = open(path).read().splitlines()
    # lines of EXAMPLES_IO/SYS_TYPE_0/H2O_H2O_Identical/MTRX.DAT
    assert lines[:7] == ["COLLISION_TYPE= 0", "NUMBER_OF_CHANLS=    6",
                         "NUMBER_OF_STATES=     81", "MATRIX_SIZE=       322",
                         "R_GRID_SIZE=    2",
                         "  #STATE #CHANNEL      J12      M12       J1      KA1      KC1       J2"
                         "      KA2      KC2  P",
                         "       1        1        0        0        0        0        0        0"
                         "        0        0  1"]
    d = mq.read_mtrx_dat(path)
    assert np.array_equal(d["states"], g["states"]) and np.array_equal(d["mat"], g["mat"])
