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
