"""The coupled-states approximation (CS_APPROX = YES, MQCT_SOURCE_CODES/mqct_eqtns.f:
208-210, 270, 362, 787, 845): the oracle replays the reference's MF + He example
(EXAMPLES_IO/SYS_TYPE_4/MF_He_CS_MQCT, asymmetric top + atom, 3 channels, 7 states,
12 pairs, 198 R) from the reference's own MTRX.DAT, with MIJ_SHIFT, MIJ_CUTOFF and
the clamped spline, 36 trajectories at U = 50 cm^-1 (fixture
tests/golden/g4_type4_layout.npz), and reproduces its per-trajectory probabilities
(OPACITY_FUNCTIONS_L.out, 8 printed digits), finish times (DEFLECTION_FUNCTION.out) and
inelastic cross sections (CROSS_SECTIONS.out).  The same run without the approximation
misses them by up to 90%, so the example pins the approximation itself."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
AUTOEV, EVTOWN, AMU, ABOHR = 27.21113845, 8065.5448, 1822.8885, 0.52917721067


def g4_tables(po, g):
    ech = np.array([po.asym_top(float(g["A"]), float(g["B"]), float(g["C"]), *map(int, c))[0]
                    for c in g["channels"]])
    st, R = g["states"], g["R"]
    mat = g["mat"] - g["mat"][:, -1:]          # MIJ_SHIFT
    ir1, ir2 = np.argmin(np.abs(R - 6.0)), np.argmin(np.abs(R - 8.0))
    keep = np.maximum(np.abs(mat[:, ir1]), np.abs(mat[:, ir2])) >= 1e-12 / EVTOWN / AUTOEV
    mk = mat[keep]
    y2 = np.array([po.spline(R, c, (c[1] - c[0]) / (R[1] - R[0]), (c[-1] - c[-2]) / (R[-1] - R[-2]))
                   for c in mk])
    ej = ech[st[:, 1] - 1] / EVTOWN / AUTOEV
    return po.OracleTables(st[:, 2], st[:, 3], ej, g["ind_mat"][keep], R, mk, y2,
                           float(g["mass_red"]) * AMU)


def g4_trajs(po, g, cs):
    U = float(g["U"])
    E = U / EVTOWN / AUTOEV
    k = np.sqrt(2 * float(g["mass_red"]) * AMU * E)
    jmax = int(float(g["b_impct"]) * k)
    dt = float(g["time_step"]) / np.sqrt(U / 300.0)
    rmax = float(g["rmax"])
    return [po.make_traj(E, float(l), 1, dt, rmax, rmax, 1, 1, float(g["time_lim"]), cs=cs)
            for l in range(jmax + 1)], k, jmax


def channel_prob(amp, states, n_ch=3):
    N = len(states)
    p = amp[:, :N] ** 2 + amp[:, N:] ** 2
    prob = np.zeros((len(amp), n_ch))
    for s in range(N):
        prob[:, states[s, 1] - 1] += p[:, s]
    return prob


@pytest.fixture(scope="module")
def g4_cs(oracle):
    g = np.load(os.path.join(GOLD, "g4_type4_layout.npz"))
    tab = g4_tables(oracle, g)
    trajs, k, jmax = g4_trajs(oracle, g, True)
    amp, cls, diag = oracle.propagate_batch(tab, trajs)
    return dict(g=g, tab=tab, prob=channel_prob(amp, g["states"]), cls=cls, diag=diag, k=k,
                jmax=jmax)


def test_cs_probabilities_match_reference(g4_cs):
    ref = g4_cs["g"]["opacity"]
    assert ref.shape[0] == 36 and g4_cs["jmax"] == 35      # "TOTAL J RANGE: FROM 0 TO 35"
    assert np.array_equal(ref[:, 1].astype(int), np.arange(36))
    r = ref[:, 2:]
    assert np.max(np.abs(g4_cs["prob"] - r) / r) < 2e-7


def test_cs_finish_times_and_torque(g4_cs):
    assert np.allclose(g4_cs["diag"][:, 0], g4_cs["g"]["deflection"][:, 4], rtol=1e-7)
    # no Coriolis torque: P_phi keeps its initial value (l)
    ls = np.arange(36, dtype=float)
    assert np.allclose(g4_cs["cls"][:, 5], np.sqrt(ls * (ls + 1)), rtol=1e-13, atol=0)


def test_cs_cross_sections_match_reference(oracle, g4_cs):
    sig = oracle.inelast(3, 0, 0, g4_cs["jmax"], 0, g4_cs["prob"], g4_cs["k"]) * ABOHR ** 2
    ref = g4_cs["g"]["sigma_U"]
    assert np.allclose(sig[1:], ref[1:], rtol=2e-7)   # 1 -> 2, 1 -> 3 (1 -> 1 is ELAST_CALC)


def test_without_cs_the_example_is_not_reproduced(oracle, g4_cs):
    g = g4_cs["g"]
    trajs, _, _ = g4_trajs(oracle, g, False)
    amp, _, _ = oracle.propagate_batch(g4_cs["tab"], trajs[::7])
    prob = channel_prob(amp, g["states"])
    r = g["opacity"][::7, 2:]
    assert np.max(np.abs(prob - r) / r) > 0.1
