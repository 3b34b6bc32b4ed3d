"""Elastic scattering (ELAST_CALC, MQCT_SOURCE_CODES/propagator.f:5581-6137) pinned to the
reference's printed results: the scattering phases (backward trapezoid over the deflection
function), the elastic cross section of CROSS_SECTIONS.out, the differential cross section
of DIFF_CROSS.out and its integral, and the DEFLECTION_FUNCTION.out / DIFF_CROSS.out
layouts.  Inputs are the values the reference printed (8 digits for the deflection
function and the probabilities, 7 for DIFF_CROSS.out): the MF + He CS example (fixture
g4_type4_layout.npz) and the ND3 + D2 DIFF_CROSS example (g8_diff_cross.npz, EXAMPLES_IO/
SYS_TYPE_7/NH3_H2_DIFF_CROSS).  Tolerances follow from the printed digits: phases within
1e-6 rad (sums of up to 100 rounded deflections), cross sections within 1e-7 relative,
the differential cross section within 5e-6 relative."""
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _k(U_cm, mass_red):
    E = U_cm / 8065.5448 / 27.21113845
    return np.sqrt(2 * mass_red * 1822.8885 * E)


def test_phases_and_elastic_cross_section_mf_he(mq):
    g = np.load(os.path.join(GOLD, "g4_type4_layout.npz"))
    d = g["deflection"]
    l = d[:, 0]
    ph = mq.scattering_phases(l, d[:, 2])
    assert ph[-1] == 0.0
    assert np.max(np.abs(ph - d[:, 3])) < 1e-6
    k = _k(float(g["U"]), float(g["mass_red"]))
    p_el = g["opacity"][:, 2]
    sig = mq.elastic_cross_section(l, p_el, ph, k)
    assert abs(sig / g["sigma_U"][0] - 1) < 1e-7          # 0.2827385615E+03 A^2


def test_differential_cross_section_nd3_d2(mq):
    g = np.load(os.path.join(GOLD, "g8_diff_cross.npz"))
    d = g["deflection"]
    ph = mq.scattering_phases(d[:, 0], d[:, 2])
    assert np.max(np.abs(ph - d[:, 3])) < 1e-6
    k = _k(float(g["U"]), float(g["mass_red"]))
    th, dcs, sig = mq.differential_cross_section(g["p_elastic"], ph, int(g["j_ini"]),
                                                 int(g["J_down"]), int(g["J_up"]),
                                                 int(g["L_min"]), k, int(g["n_angles"]),
                                                 dl=int(g["dl"]))
    ref = np.array([[float(x) for x in ln.split()] for ln in str(g["text_diff_cross"]).split("\n")
                    if len(ln.split()) == 2 and ln.split()[0][0] in "0123456789"])
    assert ref.shape == (2000, 2)
    assert np.max(np.abs(th * 180 / np.pi - ref[:, 0])) < 1e-4
    assert np.max(np.abs(dcs - ref[:, 1]) / ref[:, 1]) < 5e-6
    # with DIFF_CROSS the elastic cross section is the integral of dsigma/dOmega
    assert abs(sig / g["sigma_U"][0] - 1) < 1e-7           # 0.1360644281E+03 A^2


def test_deflection_files_byte_for_byte(mq, tmp_path):
    for name in ("g4_type4_layout.npz", "g8_diff_cross.npz"):
        g = np.load(os.path.join(GOLD, name))
        ref = str(g["text_deflection_function"])
        d = g["deflection"]
        U = float(g["U"])
        k = _k(U, float(g["mass_red"]))
        p = tmp_path / ("DEFLECTION_FUNCTION_" + name + ".out")
        mq.write_deflection(str(p), 1, 0, 0, 1, U, d[:, 0].astype(int), k, d[:, 2], d[:, 3],
                            d[:, 4], d[:, 5], d[:, 6], d[:, 7].astype(int), d[:, 8].astype(int))
        got = p.read_text()
        # l / k is recomputed from U and the reduced mass: the B_IMPACT column within its
        # last printed digit, every other character as printed
        got_l, ref_l = got.split("\n"), ref.split("\n")
        assert len(got_l) == len(ref_l)
        for a, b in zip(got_l, ref_l):
            if a != b:
                assert a[:6] == b[:6] and a[21:] == b[21:]
                assert abs(float(a[6:21]) - float(b[6:21])) <= 1.01e-8 * max(1.0, abs(float(b[6:21])))


def test_diff_cross_file_byte_for_byte(mq, tmp_path):
    g = np.load(os.path.join(GOLD, "g8_diff_cross.npz"))
    ref = str(g["text_diff_cross"])
    rows = np.array([[float(x) for x in ln.split()] for ln in ref.split("\n")
                     if len(ln.split()) == 2 and ln.split()[0][0] in "0123456789"])
    n = int(g["n_angles"])
    th = np.arange(n) * np.pi / (n - 1)
    p = tmp_path / "DIFF_CROSS.out"
    mq.write_diff_cross(str(p), 1, 1, 0, 0, th, rows[:, 1])
    assert p.read_text() == ref


def test_deflection_angles_from_final_states(mq, oracle):
    """The deflection function from the final classical states of the oracle's FP64
    propagation of the MF + He example reproduces the printed one (8 digits)."""
    from test_oracle_cs import g4_tables, g4_trajs
    g = np.load(os.path.join(GOLD, "g4_type4_layout.npz"))
    trajs, k, _ = g4_trajs(oracle, g, True)
    _, cls, _ = oracle.propagate_batch(g4_tables(oracle, g), trajs)
    U = float(g["U"])
    init = [mq.Trajectory(U / 8065.5448 / 27.21113845, float(l), 1, 1.0, float(g["rmax"]),
                          float(g["rmax"]), max_steps=1) for l in range(len(trajs))]
    chi = mq.deflection_angles(cls, init, float(g["mass_red"]) * 1822.8885)
    assert np.max(np.abs(chi - g["deflection"][:, 2])) < 2e-7


def test_probability_spline_cross_sections_co_h2(mq, tmp_path):
    """PROB_SPLINE = YES with DL = 3 (CO + H2, fixture g9_prob_spline.npz, EXAMPLES_IO/
    SYS_TYPE_6/CO_H2_Prob_spline): inelastic cross sections from the probabilities splined
    over l (1e-7 relative of the printed ones), the elastic cross section from the splined
    deflection function and elastic probability (1e-7), and the splined table of
    INTERPOLATED_PROBS_DEFLECTION_L.out (the reference's earlier name of
    SPLINED_DEFLECTION_OPACITY_L.out, probabilities splined linearly there) byte for byte."""
    g = np.load(os.path.join(GOLD, "g9_prob_spline.npz"))
    op, d = g["opacity"], g["deflection"]
    lt = op[:, 1]
    assert np.array_equal(lt, np.arange(1, 140, 3)) and np.array_equal(lt, d[:, 0])
    k = _k(float(g["U"]), float(g["mass_red"]))
    L_min, L_max = int(g["L_min"]), int(g["L_max"])
    sig = mq.cross_sections_spline(op[:, 2:], lt, 0, L_min, L_max, k)
    assert np.allclose(sig[1:], g["sigma_U"][1:], rtol=1e-7, atol=0)
    sig_el, ph = mq.elastic_cross_section_spline(lt, op[:, 2], d[:, 2], L_min, L_max, k)
    assert ph[-1] == 0.0 and len(ph) == L_max - L_min + 1
    assert abs(sig_el / g["sigma_U"][0] - 1) < 1e-7        # 0.3243445614E+03 A^2
    ls, chi, p = mq.splined_opacity(lt, op[:, 2:], d[:, 2], L_min, L_max, log_space=False)
    ref = str(g["text_interpolated"])
    rows = np.array([[float(x) for x in ln.split()] for ln in ref.split("\n")[1:]
                     if len(ln.split()) == 7])
    assert np.array_equal(rows[:, 1], ls)
    assert np.max(np.abs(chi - rows[:, 2])) < 5.01e-5        # printed with 4 decimals
    # the elastic column to the inputs' 8 digits; the inelastic ones fall by decades between
    # knots, and a value splined between two of them keeps fewer of the inputs' digits
    assert np.max(np.abs(p[:, 0] - rows[:, 3]) / rows[:, 3]) < 2e-8
    assert np.max(np.abs(p - rows[:, 3:]) / rows[:, 3:]) < 5e-6
    path = tmp_path / "SPLINED_DEFLECTION_OPACITY_L.out"
    mq.write_splined_opacity(str(path), ls, k, rows[:, 2], rows[:, 3:])
    got_l, ref_l = path.read_text().split("\n"), ref.split("\n")
    assert len(got_l) == len(ref_l) and got_l[0] == ref_l[0]
    for a, b in zip(got_l[1:], ref_l[1:]):       # l / k recomputed: within its last digit
        if a != b:
            assert a[15:] == b[15:]
            assert abs(float(a[:15]) - float(b[:15])) <= 1.01e-8 * max(1.0, abs(float(b[:15])))
    # log-space splines (the reference's present ELAST_CALC) give the same probabilities
    # to the printed digits where they are not tiny
    _, _, plog = mq.splined_opacity(lt, op[:, 2:], d[:, 2], L_min, L_max)
    assert np.max(np.abs(plog[:, 0] - rows[:, 3])) < 1e-7


def test_clamped_spline_matches_scipy(mq):
    """The host spline of the PROB_SPLINE branch (Numerical Recipes' clamped spline with
    chord end slopes, as the reference calls it) against scipy's clamped cubic spline on
    a non-uniform grid, inside and outside the knots."""
    from scipy.interpolate import CubicSpline
    rng = np.random.default_rng(5)
    x = np.cumsum(rng.uniform(0.5, 3.0, 25))
    y = np.exp(-0.1 * x) * np.cos(0.7 * x) + 0.01 * rng.standard_normal(25)
    yp1, ypn = (y[1] - y[0]) / (x[1] - x[0]), (y[-1] - y[-2]) / (x[-1] - x[-2])
    ref = CubicSpline(x, y, bc_type=((1, yp1), (1, ypn)))
    y2 = mq._clamped_spline(x, y)
    assert np.allclose(y2, ref(x, 2), rtol=1e-10, atol=1e-12)
    for v in np.concatenate([np.linspace(x[0], x[-1], 101), [x[0] - 1.0, x[-1] + 1.0]]):
        assert abs(mq._splint(x, y, y2, v) - ref(v)) < 1e-12


def test_deflection_and_elastic_standard_mode_h2o_h2(mq, oracle):
    """Standard MQCT (Coriolis coupling on) on the reference's H2O + H2 example (fixture
    g3_h2o_h2_type8.npz, 123 trajectories): the deflection function from the oracle's
    final classical states against the printed one (8 digits), the phases from it, and the
    elastic cross section of CROSS_SECTIONS.out (the probabilities agree with the printed
    ones to ~2e-7, so 1e-6 relative)."""
    g = np.load(os.path.join(GOLD, "g3_h2o_h2_type8.npz"))
    s = mq.CollisionSystem(8, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           BE=float(g["BE"]))
    tab = mq.PropagationTables.from_system(s, g["R"], g["mat"], float(g["mass_red"]))
    otab = oracle.OracleTables(tab.j12, tab.m12, tab.ej, tab.ind_mat, tab.R, tab.mat, tab.y2,
                               tab.mass_au)
    trajs, meta = mq.trajectory_set(float(g["U"]), float(g["b_impct"]), float(g["mass_red"]), 1,
                                    float(g["time_step"]), float(g["rmax"]),
                                    time_lim=float(g["time_lim"]))
    ot = [oracle.make_traj(t.e_coll, t.l_real, t.s_st, t.dt, t.r_start, t.r_fin,
                           t.numb_orb_prds, t.numb_oscl_prds, t.time_lim, t.max_steps)
          for t in trajs]
    amp, cls, _ = oracle.propagate_batch(otab, ot)
    d = g["deflection"]
    chi = mq.deflection_angles(cls, trajs, tab.mass_au)
    assert np.max(np.abs(chi - d[:, 2])) < 2e-7
    l = np.array([t.l_real for t in trajs])
    ph = mq.scattering_phases(l, chi)
    assert np.max(np.abs(ph - d[:, 3])) < 2e-6
    p = mq.channel_probabilities(amp, s.indx_chann, 10)
    sig = mq.elastic_cross_section(l, p[:, 0], ph, meta["k"])
    assert abs(sig / g["sigma_U"][0] - 1) < 1e-6                # 0.9913967495E+02 A^2
