"""Pin the CPU oracle against the reference's own outputs and closed forms.

Golden fixtures come from the reference's EXAMPLES_IO (tests/golden/make_golden.py):
 - H2O+H2 (SYS_TYPE 8): MTRX.DAT -> per-trajectory channel probabilities
   (OPACITY_FUNCTIONS_L.out), finish times (DEFLECTION_FUNCTION.out) and
   cross sections (CROSS_SECTIONS.out);
 - channel energies printed in USER_INPUT_CHECK.out (asymmetric-top levels);
 - the MF+He (SYS_TYPE 4) state ordering of MTRX.DAT;
 - the AT trajectory record layout of AT_APPROX_TRAJS.
"""
import math
import os
from fractions import Fraction

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
AUTOEV, EVTOWN, AMU, ABOHR = 27.21113845, 8065.5448, 1822.8885, 0.52917721067


def _g3():
    return np.load(os.path.join(GOLD, "g3_h2o_h2_type8.npz"))


def _g3_tables(po, g):
    chan = g["channels"]
    ech = np.array([po.asym_top(float(g["A"]), float(g["B"]), float(g["C"]), *map(int, c[:3]))[0]
                    + float(g["BE"]) * c[3] * (c[3] + 1) for c in chan])
    st = g["states"]
    R = g["R"]
    mat = g["mat"] - g["mat"][:, -1:]          # MIJ_SHIFT (default on)
    ir1, ir2 = np.argmin(np.abs(R - 6.0)), np.argmin(np.abs(R - 8.0))
    keep = np.maximum(np.abs(mat[:, ir1]), np.abs(mat[:, ir2])) >= 1e-12 / EVTOWN / AUTOEV
    mk = mat[keep]
    y2 = np.array([po.spline(R, c, (c[1] - c[0]) / (R[1] - R[0]), (c[-1] - c[-2]) / (R[-1] - R[-2]))
                   for c in mk])
    ej = ech[st[:, 1] - 1] / EVTOWN / AUTOEV
    tab = po.OracleTables(st[:, 2], st[:, 3], ej, g["ind_mat"][keep], R, mk, y2,
                          float(g["mass_red"]) * AMU)
    return tab, ech, keep


def test_asym_top_levels_match_printed_energies(oracle):
    g = _g3()
    for c, e_ref in zip(g["channels"], g["e_ch_printed"]):
        e = oracle.asym_top(float(g["A"]), float(g["B"]), float(g["C"]), *map(int, c[:3]))[0]
        e += float(g["BE"]) * c[3] * (c[3] + 1)
        assert abs(e - e_ref) < 6e-4
    g4 = np.load(os.path.join(GOLD, "g4_type4_layout.npz"))
    for c, e_ref in zip(g4["channels"], g4["e_ch_printed"]):
        e = oracle.asym_top(float(g4["A"]), float(g4["B"]), float(g4["C"]), *map(int, c))[0]
        assert abs(e - e_ref) < 6e-4


def test_asym_top_eigenvectors_are_orthonormal_eigenpairs(oracle):
    A, B, Cc = 27.9, 14.5, 9.3
    for j in range(0, 9):
        vecs, ens = [], []
        ka_list = [0] + [i // 2 for i in range(2, 2 * j + 2)]
        for i in range(2 * j + 1):
            e, v = oracle.asym_top(A, B, Cc, j, ka_list[i], ka_list[::-1][i])
            vecs.append(v)
            ens.append(e)
        V = np.array(vecs)
        assert np.allclose(V @ V.T, np.eye(2 * j + 1), atol=1e-12)
        assert np.all(np.diff(ens) >= -1e-12)
    # closed form for j = 1: levels C+... (A+B, A+C, B+C)
    es = sorted(oracle.asym_top(A, B, Cc, 1, ka, kc)[0] for ka, kc in [(0, 1), (1, 1), (1, 0)])
    assert np.allclose(es, sorted([A + B, A + Cc, B + Cc]), atol=1e-12)


def test_type4_state_ordering_matches_reference_matrix_file(oracle):
    g4 = np.load(os.path.join(GOLD, "g4_type4_layout.npz"))
    ch = g4["channels"]
    osys = oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=np.zeros(len(ch)),
                               vec1=np.zeros(3 * len(ch)), ldv=3)
    ic, j12, m12, _ = osys.states()
    st = g4["states"]
    assert (ic == st[:, 1]).all() and (j12 == st[:, 2]).all() and (m12 == st[:, 3]).all()
    ind = oracle.ind_mat(m12)
    assert (ind == g4["ind_mat"]).all()


def test_type8_state_and_pair_ordering(oracle):
    g = _g3()
    ch = g["channels"]
    osys = oracle.OracleSystem(8, ch[:, 0], ch[:, 1], ch[:, 2], j2=ch[:, 3],
                               e_ch=np.zeros(len(ch)), vec1=np.zeros(7 * len(ch)), ldv=7)
    ic, j12, m12, _ = osys.states()
    st = g["states"]
    assert (ic == st[:, 1]).all() and (j12 == st[:, 2]).all() and (m12 == st[:, 3]).all()
    assert (oracle.ind_mat(m12) == g["ind_mat"]).all()


@pytest.fixture(scope="module")
def g3_run(oracle):
    g = _g3()
    tab, ech, keep = _g3_tables(oracle, g)
    U = float(g["U"])
    E = U / EVTOWN / AUTOEV
    mass = float(g["mass_red"]) * AMU
    k = np.sqrt(2 * mass * E)
    jmax = int(float(g["b_impct"]) * k)
    dt = float(g["time_step"]) / np.sqrt(U / 300.0)
    rmax = float(g["rmax"])
    trajs = [oracle.make_traj(E, float(l), 1, dt, rmax, rmax, 1, 1, float(g["time_lim"]))
             for l in range(jmax + 1)]
    amp, cls, diag = oracle.propagate_batch(tab, trajs)
    st = g["states"]
    N = len(st)
    p = amp[:, :N] ** 2 + amp[:, N:] ** 2
    prob = np.zeros((len(trajs), 10))
    for s in range(N):
        prob[:, st[s, 1] - 1] += p[:, s]
    return dict(g=g, prob=prob, diag=diag, k=k, jmax=jmax, keep=keep)


def test_g3_truncation_count(g3_run):
    # "THE SIZE OF NON_ZERO PART OF Mij = 591" in the reference log
    assert int(g3_run["keep"].sum()) == 591


def test_g3_per_trajectory_probabilities(g3_run):
    ref = g3_run["g"]["opacity"]
    prob = g3_run["prob"]
    assert ref.shape[0] == prob.shape[0] == 123
    assert np.array_equal(ref[:, 1].astype(int), np.arange(123))
    r = ref[:, 2:]
    # the golden file prints 8 significant digits
    err = np.abs(prob - r) / np.maximum(np.abs(r), 1e-30)
    big = r > 1e-25
    assert np.max(err[big]) < 2e-7, np.max(err[big])


def test_g3_finish_times(g3_run):
    ref = g3_run["g"]["deflection"]
    assert np.allclose(g3_run["diag"][:, 0], ref[:, 4], rtol=2e-8)


def test_g3_cross_sections(oracle, g3_run):
    sig = oracle.inelast(10, 0, 0, g3_run["jmax"], 0, g3_run["prob"], g3_run["k"]) * ABOHR ** 2
    ref = g3_run["g"]["sigma_U"]
    # inelastic channels 2-4 (channel 1 is the elastic cross section, ELAST_CALC)
    assert np.allclose(sig[1:4], ref[1:4], rtol=2e-7)
    assert np.all(sig[4:] == 0) and np.all(ref[4:] == 0)


def test_at_trajectory_record_layout():
    g = np.load(os.path.join(GOLD, "g1_at_traj_l9.npz"))
    head = g["head"]
    assert int(g["n_records"]) == int(g["n_file"])
    # first record: t=0, R=RMAX, theta=pi/2, P_phi = sqrt(l(l+1)) for l=9
    assert head[0, 0] == 0.0 and head[0, 1] == 30.0
    assert abs(head[0, 3] - math.pi / 2) < 1e-15
    assert abs(head[0, 6] - math.sqrt(9 * 10)) < 1e-12
    assert np.all(np.diff(head[:, 0]) > 0)


# ---------------------------------------------------------------- closed forms
def _w3j(j1, j2, j3, m1, m2, m3):
    """Wigner 3j by the Racah formula in exact rational arithmetic."""
    if m1 + m2 + m3 != 0 or j3 > j1 + j2 or j3 < abs(j1 - j2):
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    f = math.factorial
    tri = Fraction(f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3), f(j1 + j2 + j3 + 1))
    pre = tri * f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3)
    s = Fraction(0)
    for t in range(0, j1 + j2 + j3 + 1):
        a = [t, j3 - j2 + t + m1, j3 - j1 + t - m2, j1 + j2 - j3 - t, j1 - t - m1, j2 - t + m2]
        if min(a) < 0:
            continue
        den = 1
        for x in a:
            den *= f(x)
        s += Fraction((-1) ** t, den)
    sign = -1 if (j1 - j2 - m3) % 2 else 1
    return float(sign * s) * math.sqrt(float(pre))


def test_w3j_and_cg_against_exact(oracle):
    for (j1, j2, j3, m1, m2) in [(1, 1, 2, 0, 0), (2, 3, 4, 1, -1), (5, 5, 6, 2, -3), (8, 4, 6, -3, 1)]:
        m3 = -(m1 + m2)
        assert abs(oracle.lib().orc_w3js(2 * j1, 2 * j2, 2 * j3, 2 * m1, 2 * m2, 2 * m3)
                   - _w3j(j1, j2, j3, m1, m2, m3)) < 1e-13


def test_diatom_matrix_equals_legendre_projection(oracle):
    """Type 1 with V = sum_l v_l(R) P_l(cos theta): the quadrature equals
    sum_l v_l (-1)^m sqrt((2j+1)(2j'+1)) (j l j'; 0 0 0)(j l j'; -m 0 m) exactly
    (64-point Gauss-Legendre is exact for the polynomial degrees involved)."""
    from mqct_b200 import synthetic as syn
    pes_d = syn.legendre_pes(7, seed=1)
    pes = oracle.OraclePes(pes_d["kind"], pes_d["n_terms"], pes_d["params"])
    js = list(range(6))
    osys = oracle.OracleSystem(1, js, e_ch=np.zeros(len(js)), vec1=np.ones(len(js)), ldv=1)
    states = osys.states()
    ic, j12, m12, _ = states
    ind = oracle.ind_mat(m12)
    R = np.array([3.0, 4.5, 7.0, 12.0])
    mat, y2, sk = oracle.build_matrix(osys, states, ind, R, (64, 0, 0, 0, 0, 0, 1), pes,
                                      mij_cut=0.0)
    p = pes_d["params"]
    n = pes_d["n_terms"]
    for k, (a, b) in enumerate(ind):
        ja, jb, m = j12[a - 1], j12[b - 1], m12[a - 1]
        for i, r in enumerate(R):
            v = 0.0
            for l in range(n):
                vl = p[l] * np.exp(-p[n + l] * r) - p[2 * n + l] / r ** 6
                v += vl * (-1.0) ** m * math.sqrt((2 * ja + 1) * (2 * jb + 1)) * \
                    _w3j(ja, l, jb, 0, 0, 0) * _w3j(ja, l, jb, -m, 0, m)
            v /= EVTOWN * AUTOEV
            assert abs(mat[k, i] - v) <= 1e-12 * max(1.0, abs(v)) + 1e-15


def test_asym_top_isotropic_pes_is_orthonormal(oracle):
    """Type 4 with an isotropic V(R): M = V(R) * identity (orthonormal basis on
    the GL x midpoint grid), which checks the Wigner-D normalisation."""
    A, B, Cc = 27.9, 14.5, 9.3
    chans = [(0, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0), (2, 0, 2), (2, 1, 2), (2, 1, 1),
             (2, 2, 1), (2, 2, 0), (3, 1, 3)]
    vecs = np.zeros((len(chans), 7))
    for i, c in enumerate(chans):
        vecs[i, :2 * c[0] + 1] = oracle.asym_top(A, B, Cc, *c)[1]
    ch = np.array(chans)
    osys = oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=np.zeros(len(ch)),
                               vec1=vecs.reshape(-1), ldv=7)
    states = osys.states()
    ind = oracle.ind_mat(states[2])
    # isotropic: Legendre surface with only l = 0
    pes = oracle.OraclePes(1, 1, np.array([5000.0, 1.7, 3e4]))
    R = np.array([3.0, 6.0, 9.0])
    mat, _, _ = oracle.build_matrix(osys, states, ind, R, (16, 16, 0, 0, 0, 0, 1), pes, mij_cut=0.0)
    v = (5000.0 * np.exp(-1.7 * R) - 3e4 / R ** 6) / (EVTOWN * AUTOEV)
    diag = ind[:, 0] == ind[:, 1]
    assert np.allclose(mat[diag], v[None, :], rtol=1e-12)
    assert np.max(np.abs(mat[~diag])) < 1e-13 * np.max(np.abs(v))


def test_alpha_grid_quadrature_equals_analytic_alpha(oracle):
    """Type 4: the explicit midpoint alpha grid gives the reference's analytic
    2*pi alpha integral (same-m pairs) to rounding."""
    A, B, Cc = 27.9, 14.5, 9.3
    chans = [(0, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0), (2, 1, 2), (2, 2, 0)]
    vecs = np.zeros((len(chans), 5))
    for i, c in enumerate(chans):
        vecs[i, :2 * c[0] + 1] = oracle.asym_top(A, B, Cc, *c)[1]
    ch = np.array(chans)
    osys = oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=np.zeros(len(ch)),
                               vec1=vecs.reshape(-1), ldv=5)
    from mqct_b200 import synthetic as syn
    pd = syn.site_pes(12, seed=2)
    pes = oracle.OraclePes(pd["kind"], pd["n_terms"], pd["params"], sites1=pd["sites1"])
    states = osys.states()
    ind = oracle.ind_mat(states[2])
    R = np.array([4.0, 6.0])
    m2, _, _ = oracle.build_matrix(osys, states, ind, R, (12, 12, 0, 0, 0, 0, 1), pes, mij_cut=0.0)
    m3, _, _ = oracle.build_matrix(osys, states, ind, R, (12, 12, 8, 0, 0, 0, 1), pes, mij_cut=0.0)
    assert np.allclose(m3, m2, rtol=1e-11, atol=1e-13 * np.abs(m2).max())


def test_oracle_mtrx_uf_layout(oracle, tmp_path):
    """Fortran unformatted sequential records with 4-byte markers."""
    import struct
    ind = np.array([1, 1, 2, 1, 2, 2], np.int32)
    R = np.array([3.0, 4.0, 5.0])
    mat = np.arange(9, dtype=np.float64)
    st = np.array([1, 1, 0, 0, 0, 2, 2, 1, 0, 1], np.int32)
    path = str(tmp_path / "MTRX_UF.DAT")
    oracle.lib().orc_write_mtrx_uf(path.encode(), 1, 2, 2, st, 5, 3, ind, 3, R, mat)
    raw = open(path, "rb").read()
    n0, v, n1 = struct.unpack_from("<iii", raw, 0)
    assert (n0, v, n1) == (4, 1, 4)
    # 5 header records, 2 state records (5 ints), 3 pair records, 3 R records, 3 x (k, Mat_el)
    size = 5 * 12 + 2 * (20 + 8) + 3 * (12 + 8) + 3 * (12 + 8) + 3 * (12 + 24 + 8)
    assert len(raw) == size
