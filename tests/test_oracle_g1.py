"""The two-run H2O + H2O AT-MQCT example of the reference (SYS_TYPE 0, PES expansion
terms in kcal/mol), replayed by the oracle and compared with the reference's own
outputs (EXAMPLES_IO/SYS_TYPE_0/H2O_H2O_AT_Approximation, fixture
tests/golden/g1_h2o_h2o_at.npz):

1st run: the one-channel matrix from the expansion terms, MIJ_SHIFT, standard
MQCT of the 14 trajectories l = 9, 28, ..., 256 with SAVE_TRAJECT: the records
equal the reference's AT_APPROX_TRAJS files (count, first, middle and last
records).
2nd run: the 9-channel (81 states, 594 pairs) matrix from the same terms, MIJ_SHIFT
and MIJ_CUTOFF, AT-MQCT along the 1st run's paths: per-trajectory channel
probabilities equal OPACITY_FUNCTIONS_L.out (8 printed digits) and the cross
sections with DL = 19 equal CROSS_SECTIONS.out / M_PROJ_CROSSECTIONS.out (10
printed digits).  The matrix is not printed by that example, so this pins the
SYS_TYPE 0 expansion path through the dynamics it drives."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
AUTOEV, EVTOWN, AMU, ABOHR, KCAL = 27.21113845, 8065.5448, 1822.8885, 0.52917721067, 627.509469


def _g1():
    return np.load(os.path.join(GOLD, "g1_h2o_h2o_at.npz"))


def _systems(mq, oracle, g, chans):
    s = mq.CollisionSystem(0, chans, A=float(g["A"]), B=float(g["B"]), C=float(g["C"]))
    ch = s.channels
    osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                               e_ch=s.e_ch, vec1=s.vec1.reshape(-1), vec2=s.vec2.reshape(-1),
                               ldv=s.ldv)
    return s, osys


def _tables(oracle, s, mat, R, mass):
    """MIJ_SHIFT, MIJ_CUTOFF (1e-12 cm^-1 at the R points nearest 6 and 8 bohr) and the
    clamped spline, as the reference prepares a matrix for propagation."""
    mat = mat - mat[:, -1:]
    ir1, ir2 = np.argmin(np.abs(R - 6.0)), np.argmin(np.abs(R - 8.0))
    keep = np.maximum(np.abs(mat[:, ir1]), np.abs(mat[:, ir2])) >= 1e-12 / EVTOWN / AUTOEV
    mk = mat[keep]
    y2 = np.array([oracle.spline(R, c, (c[1] - c[0]) / (R[1] - R[0]),
                                 (c[-1] - c[-2]) / (R[-1] - R[-2])) for c in mk])
    return oracle.OracleTables(s.j12, s.m12, s.ej_cm / EVTOWN / AUTOEV, s.ind_mat[keep], R, mk,
                               y2, mass)


@pytest.fixture(scope="module")
def g1_run(mq, oracle):
    g = _g1()
    R, lab, T = g["R"], g["labels"], g["terms"]
    mass = float(g["mass_red"]) * AMU
    U = float(g["U"])
    E = U / EVTOWN / AUTOEV
    rmax = float(g["rmax"])
    s1, o1 = _systems(mq, oracle, g, g["channels"][:1])
    m1 = oracle.expansion_matrix_type0(o1, o1.states(), s1.ind_mat, lab, T, 1.0 / KCAL)
    tab1 = _tables(oracle, s1, m1, R, mass)
    dt1 = float(g["time_step1"]) / np.sqrt(U / 300.0)
    paths = []
    for l in g["l"]:
        tr = oracle.make_traj(E, float(l), 1, dt1, rmax, rmax, 1, 1, float(g["time_lim"]))
        paths.append(oracle.dotraject_record(tab1, tr)[3])
    s9, o9 = _systems(mq, oracle, g, g["channels"])
    m9 = oracle.expansion_matrix_type0(o9, o9.states(), s9.ind_mat, lab, T, 1.0 / KCAL)
    tab9 = _tables(oracle, s9, m9, R, mass)
    dt2 = float(g["time_step2"]) / np.sqrt(U / 300.0)
    N = s9.n_states
    prob = np.zeros((len(g["l"]), 9))
    for i, l in enumerate(g["l"]):
        tr = oracle.make_traj(E, float(l), 1, dt2, rmax, rmax, 1, 1, float(g["time_lim"]))
        amp, _ = oracle.dotraject_at(tab9, tr, paths[i])
        p = amp[:N] ** 2 + amp[N:] ** 2
        np.add.at(prob[i], s9.indx_chann - 1, p)
    k = np.sqrt(2 * mass * E)
    return dict(g=g, paths=paths, prob=prob, k=k, s9=s9, m9=m9)


def test_first_run_records_equal_the_saved_paths(g1_run):
    g = g1_run["g"]
    for i, rec in enumerate(g1_run["paths"]):
        assert len(rec) == g["n_rec"][i]
        h = len(rec) // 2
        for mine, ref in ((rec[:4], g["rec_head"][i]), (rec[h - 1:h + 2], g["rec_mid"][i]),
                          (rec[-3:], g["rec_tail"][i])):
            assert np.max(np.abs(mine - ref) / np.maximum(np.abs(ref), 1e-300)) <= 1e-12
    # the closing record is stamped one step past the final time
    r = g1_run["paths"][0]
    assert np.isclose(r[-1, 0] - r[-2, 0], 2 * (r[-2, 0] - r[-3, 0]))


def test_second_run_probabilities(g1_run):
    ref = g1_run["g"]["opacity2"]
    assert np.array_equal(ref[:, 1].astype(int), g1_run["g"]["l"])
    r = ref[:, 2:]
    err = np.abs(g1_run["prob"] - r) / np.abs(r)
    assert np.max(err) < 2e-7, np.max(err)


def test_second_run_cross_sections(oracle, g1_run):
    g = g1_run["g"]
    k = g1_run["k"]
    jmax = int(float(g["b_impct"]) * k)
    assert jmax == 259  # "TOTAL J RANGE: FROM 0 TO 259" in the reference log
    sig = oracle.inelast(9, 0, 0, jmax, 0, g1_run["prob"], k, dl=int(g["dl"])) * ABOHR ** 2
    assert np.allclose(sig[1:], g["sigma2"][1:], rtol=2e-9, atol=0)
    assert np.allclose(sig, g["sigma2_mproj"], rtol=2e-9, atol=0)


def test_type0_expansion_is_hermitian(oracle, g1_run):
    """The potential is a real symmetric operator: the element of (b, a) equals that of
    (a, b), although the formula treats the two states differently."""
    g, s9, m9 = g1_run["g"], g1_run["s9"], g1_run["m9"]
    ch = s9.channels
    osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                               e_ch=s9.e_ch, vec1=s9.vec1.reshape(-1),
                               vec2=s9.vec2.reshape(-1), ldv=s9.ldv)
    swapped = np.ascontiguousarray(s9.ind_mat[:, ::-1])
    m_sw = oracle.expansion_matrix_type0(osys, osys.states(), swapped, g["labels"], g["terms"],
                                         1.0 / KCAL)
    assert np.max(np.abs(m_sw - m9)) <= 1e-12 * np.abs(m9).max()


def test_host_trajectory_set_and_cross_sections_with_dl(mq, oracle, g1_run):
    """The library's host side of the same run: the trajectory l values of DL = 19
    (bin midpoints, the reference's file names) and INELAST_CALC with DL bins."""
    g = g1_run["g"]
    trajs, meta = mq.trajectory_set(float(g["U"]), float(g["b_impct"]), float(g["mass_red"]), 1,
                                    float(g["time_step1"]), float(g["rmax"]), dl=int(g["dl"]))
    assert [t.l_real for t in trajs] == [float(l) for l in g["l"]]
    assert np.isclose(trajs[0].dt, 10.0 / np.sqrt(500.0 / 300.0))
    assert meta["J_up"] == 259 and meta["L_min"] == 0
    sig = mq.cross_sections(g1_run["prob"], 0, 0, meta["J_up"], 0, meta["k"], dl=meta["dl"])
    ref = oracle.inelast(9, 0, 0, meta["J_up"], 0, g1_run["prob"], g1_run["k"], dl=19) * ABOHR ** 2
    assert np.allclose(sig, ref, rtol=1e-13)
    assert np.allclose(sig, g["sigma2_mproj"], rtol=2e-9)


def test_partial_cross_sections_per_j(g1_run):
    """PARTIAL_CROSS_SECTIONS_J.out of the second run: per total J the cross section
    pi/k^2 (2J+1) P_f(traj(J)) (j_ini = 0, l = J) in Angstrom^2, traj(l) = (l - L_MIN)/DL."""
    g, prob, k = g1_run["g"], g1_run["prob"], g1_run["k"]
    ref = g["partial2"]
    J = ref[:, 0].astype(int)
    assert np.array_equal(J, np.arange(260))
    mine = (2 * J + 1.0)[:, None] / k ** 2 * np.pi * prob[J // int(g["dl"])] * ABOHR ** 2
    r = ref[:, 1:]
    assert np.max(np.abs(mine - r) / r) < 2e-7   # 8 printed digits


def test_at_adaptive_step(oracle, g1_run):
    """AT_ADAPT_STP (propagator.f:3034-3049, 3821-3860) on the example's second run:
    steps from the coupling energy along each path, TIME_STEP as the smallest step.
    No reference example runs it.  With the default AT_ADAPTOL = 0.5 the rule takes
    steps of thousands of a.u. on these paths and RK4 diverges, as the restated rule
    does; with AT_ADAPTOL = 5e-4 the run takes about a fifth of the fixed steps and
    stays within 2e-3 of the fixed-step probabilities."""
    g = g1_run["g"]
    mass = float(g["mass_red"]) * AMU
    U = float(g["U"])
    E = U / EVTOWN / AUTOEV
    rmax = float(g["rmax"])
    s9 = g1_run["s9"]
    tab9 = _tables(oracle, s9, g1_run["m9"], g["R"], mass)
    dt2 = float(g["time_step2"]) / np.sqrt(U / 300.0)
    N = s9.n_states
    for i, l in enumerate(g["l"][:4]):
        tr = oracle.make_traj(E, float(l), 1, dt2, rmax, rmax, 1, 1, float(g["time_lim"]),
                              method=2, eps=5e-4, hmin=float(g["time_step2"]))
        amp, diag = oracle.dotraject_at(tab9, tr, g1_run["paths"][i])
        tf = oracle.make_traj(E, float(l), 1, dt2, rmax, rmax, 1, 1, float(g["time_lim"]))
        amp_f, diag_f = oracle.dotraject_at(tab9, tf, g1_run["paths"][i])
        assert diag[1] < 0.5 * diag_f[1]
        assert diag[0] == pytest.approx(diag_f[0], rel=1e-12)   # both end at the path's end
        assert diag[2] < 1e-3
        p = amp[:N] ** 2 + amp[N:] ** 2
        pf = amp_f[:N] ** 2 + amp_f[N:] ** 2
        assert np.max(np.abs(p - pf)) < 2e-3
