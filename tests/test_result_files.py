"""The per-energy result files (OPACITY_FUNCTIONS_L.out, TOTAL_PROBABILITIES_L.out,
PARTIAL_CROSS_SECTIONS_J.out, M_PROJ_CROSSECTIONS.out, CROSS_SECTIONS.out) written from
the values the reference printed in its MF + He CS example
(EXAMPLES_IO/SYS_TYPE_4/MF_He_CS_MQCT, fixture tests/golden/g4_type4_layout.npz) reproduce
those files byte for byte (the sigma(U) column of CROSS_SECTIONS.out, which the writer
forms from sigma_f and E_bill as the reference does, within 1e-7: E_bill is printed with 6
decimals)."""
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _g4():
    return np.load(os.path.join(GOLD, "g4_type4_layout.npz"))


def _rows(text, n):
    out = []
    for ln in text.split("\n"):
        t = ln.split()
        if len(t) == n:
            try:
                out.append([float(x) for x in t])
            except ValueError:
                pass
    return np.array(out)


def test_opacity_and_total_probability_files(mq, tmp_path):
    g = _g4()
    ref = str(g["text_opacity_functions_l"])
    rows = _rows(ref, 5)
    E = float(g["U"]) / 8065.5448 / 27.21113845
    k = np.sqrt(2 * float(g["mass_red"]) * 1822.8885 * E)
    p, pt = tmp_path / "OPACITY_FUNCTIONS_L.out", tmp_path / "TOTAL_PROBABILITIES_L.out"
    mq.write_opacity(str(p), 1, 0, 0, 1, 50.0, rows[:, 1].astype(int), k, rows[:, 2:],
                     path_total=str(pt), chann_ini=1)
    assert p.read_text() == ref
    ref_t = str(g["text_total_probabilities_l"]).split("\n")
    got_t = pt.read_text().split("\n")
    assert got_t[:5] == ref_t[:5] and len(got_t) == len(ref_t)
    a, b = _rows("\n".join(got_t), 4), _rows("\n".join(ref_t), 4)
    assert np.allclose(a, b, rtol=2e-7, atol=0)        # sums of 8-digit probabilities


def test_partial_j_file_byte_for_byte(mq, tmp_path):
    g = _g4()
    ref = str(g["text_partial_cross_sections_j"])
    rows = _rows(ref, 4)
    p = tmp_path / "PARTIAL_CROSS_SECTIONS_J.out"
    mq.write_partial_j(str(p), 1, 0, 0, 1, 50.0, rows[:, 0].astype(int), rows[:, 1:])
    assert p.read_text() == ref


def test_m_proj_file_byte_for_byte(mq, tmp_path):
    g = _g4()
    ref = str(g["text_m_proj_crossections"])
    sig = _rows(ref, 2)[:, 1]
    p = tmp_path / "M_PROJ_CROSSECTIONS.out"
    mq.write_m_proj(str(p), 1, 1, 0, 0, sig)
    assert p.read_text() == ref


def test_cross_sections_file(mq, tmp_path):
    g = _g4()
    ref = str(g["text_cross_sections"])
    rows = _rows(ref, 5)
    p = tmp_path / "CROSS_SECTIONS.out"
    mq.write_cross_sections(str(p), 50.0, 1, rows[:, 4], rows[:, 3], 0.40188e-7,
                            e_err_pct=0.99993e2)
    mq.write_cross_sections_footer(str(p), 36)
    mine, theirs = p.read_text().split("\n"), ref.split("\n")
    assert len(mine) == len(theirs)
    for a, b in zip(mine, theirs):
        ta, tb = a.split(), b.split()
        if len(tb) == 5 and tb[0].isdigit():      # sigma(U) = sigma_f / U * E_bill
            assert a[:15] == b[:15] and a[36:] == b[36:]
            assert abs(float(ta[2]) - float(tb[2])) <= 1e-7 * abs(float(tb[2]))
        else:
            assert a == b
