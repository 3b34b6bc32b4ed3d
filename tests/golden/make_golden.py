"""Regenerate the golden fixtures in tests/golden/ from the reference's own
example outputs (EXAMPLES_IO of MarquetteQuantum/MQCT).

Run where the reference tree is available:
    python tests/golden/make_golden.py /path/to/MQCT
The fixtures are small numpy archives; tests read only the archives, so they
also run where the reference tree is absent.
"""
from __future__ import annotations

import os
import re
import struct
import sys

import numpy as np


def _read_mtrx_dat(path, n_cols):
    with open(path) as f:
        lines = f.read().splitlines()
    hdr = [int(lines[i].split("=")[1]) for i in range(5)]
    coll, nch, ns, P, nR = hdr
    p = 6
    states = np.array([[int(x) for x in lines[p + s].split()[:n_cols]] for s in range(ns)],
                      dtype=np.int32)
    p += ns + 1
    ind = np.array([[int(x) for x in lines[p + k].split()[1:3]] for k in range(P)], dtype=np.int32)
    p += P + 1
    R = np.array([float(lines[p + i].split()[1]) for i in range(nR)])
    p += nR + 1
    mat = np.zeros((P, nR))
    for q in range(P * nR):
        t = lines[p + q].split()
        mat[int(t[0]) - 1, int(t[1]) - 1] = float(t[2])
    return coll, nch, states, ind, R, mat


def _read_table(path, ncols, first_int=True):
    rows = []
    for line in open(path):
        t = line.split()
        if len(t) == ncols and t[0 if not first_int else 1].replace(".", "").isdigit():
            try:
                rows.append([float(x) for x in t])
            except ValueError:
                pass
    return np.array(rows)


def main(ref_root):
    ex = os.path.join(ref_root, "EXAMPLES_IO")
    out = os.path.dirname(os.path.abspath(__file__))

    # G3: asymmetric top + diatom (SYS_TYPE 8), H2O+H2, matrix read -> dynamics.
    d = os.path.join(ex, "SYS_TYPE_8", "H2O_H2_Dynamics")
    coll, nch, states, ind, R, mat = _read_mtrx_dat(os.path.join(d, "MTRX.DAT"), 8)
    opac = _read_table(os.path.join(d, "OPACITY_FUNCTIONS_L.out"), 2 + nch)
    defl = _read_table(os.path.join(d, "DEFLECTION_FUNCTION.out"), 9, first_int=False)
    sig = []
    for line in open(os.path.join(d, "CROSS_SECTIONS.out")):
        t = line.split()
        if len(t) == 5 and t[0].isdigit():
            sig.append(float(t[2]))
    np.savez_compressed(
        os.path.join(out, "g3_h2o_h2_type8.npz"), coll=coll, states=states, ind_mat=ind, R=R,
        mat=mat, opacity=opac, deflection=defl, sigma_U=np.array(sig),
        # $BASIS/$SYSTEM of H2OH2.inp
        A=27.88063134, B=9.277708381, C=14.52176959, BE=60.853, mass_red=1.812773730,
        rmax=30.0, time_step=10.0, U=800.0, b_impct=25.0, time_lim=3.5e6,
        channels=np.array([[0, 0, 0, 0], [1, 1, 1, 0], [2, 0, 2, 0], [2, 1, 1, 0], [1, 0, 1, 1],
                           [1, 1, 0, 1], [2, 1, 2, 1], [2, 2, 1, 1], [3, 1, 2, 1], [3, 2, 1, 1]],
                          dtype=np.int32),
        # CHANNELS ENERGIES, CM-1 printed in USER_INPUT_CHECK.out (3 decimals)
        e_ch_printed=np.array([0.000, 37.158, 70.133, 95.245, 145.505, 164.108, 201.219, 257.028,
                               295.304, 334.334]))

    # G5: the PES expansion terms from which the reference built the G3 matrix
    # (EXAMPLES_IO/SYS_TYPE_8/H2O_H2_MTRXCalculation: PES_EXPAN_TERMS.DAT -> MTRX.DAT,
    # which is identical to the G3 MTRX.DAT).  Header "R_Bohr v_l1_nju1_l2_l ...",
    # then one row per R (f6.2 R, e19.12 values, cm^-1).
    d = os.path.join(ex, "SYS_TYPE_8", "H2O_H2_MTRXCalculation")
    with open(os.path.join(d, "PES_EXPAN_TERMS.DAT")) as f:
        head = f.readline().split()
        rows = [[float(x) for x in ln.split()] for ln in f if ln.strip()]
    labels = np.array([[int(x) for x in h.split("_")[1:]] for h in head[1:]], dtype=np.int32)
    vals = np.array(rows)
    np.savez_compressed(os.path.join(out, "g5_h2o_h2_expansion_terms.npz"), labels=labels,
                        R=vals[:, 0], terms=vals[:, 1:])

    # G5b: symmetric top + diatom (SYS_TYPE 7), ND3+D2
    # (EXAMPLES_IO/SYS_TYPE_7/NH3_H2_MTRX_calculation: PES_EXPAN_TERMS.DAT, 377 terms
    # (l1, nju1, l2, l) in cm^-1 -> MTRX.DAT, 80 states, 461 pairs, 86 R).  Every R
    # point of the expansion is independent of the others, so 12 of the 86 R points
    # are kept: the terms there and all 461 matrix columns.
    d = os.path.join(ex, "SYS_TYPE_7", "NH3_H2_MTRX_calculation")
    coll7, nch7, states7, ind7, R7, mat7 = _read_mtrx_dat(os.path.join(d, "MTRX.DAT"), 8)
    with open(os.path.join(d, "PES_EXPAN_TERMS.DAT")) as f:
        head = f.readline().split()
        rows = np.array([[float(x) for x in ln.split()] for ln in f if ln.strip()])
    labels7 = np.array([[int(x) for x in h.split("_")[1:]] for h in head[1:]], dtype=np.int32)
    keep = np.linspace(0, len(R7) - 1, 12).round().astype(int)
    assert np.allclose(rows[keep, 0], R7[keep], atol=5e-3)
    np.savez_compressed(
        os.path.join(out, "g5b_nd3_d2_type7.npz"), coll=coll7, states=states7, ind_mat=ind7,
        r_index=keep, R=R7[keep], mat=mat7[:, keep], labels=labels7, terms=rows[keep, 1:],
        # $BASIS of NH3H2.inp: A = B, C of the symmetric top, BE of the diatom
        A=5.1432, C=3.1015, BE=30.443,
        channels=np.array([[0, 0, 0, 0], [1, 0, 0, 0], [2, 0, 0, 0], [3, 0, 0, 0], [3, 3, 0, 0],
                           [3, 3, 1, 0], [1, 1, 0, 0], [1, 1, 1, 0], [2, 1, 0, 0], [2, 1, 1, 0],
                           [3, 1, 0, 0], [3, 1, 1, 0], [4, 1, 0, 0], [5, 1, 0, 0]],
                          dtype=np.int32),
        # CHANNELS ENERGIES, CM-1 of USER_INPUT_CHECK.out
        e_ch_printed=np.array([0.0, 10.2864, 30.8592, 61.7184, 43.3431, 43.3431, 8.2447, 8.2447,
                               28.8175, 28.8175, 59.6767, 59.6767, 100.8223, 152.2543]))

    # G5c: two identical asymmetric tops (SYS_TYPE 0, IDENTICAL = YES, IDENTICAL_PES = YES),
    # H2O+H2O (EXAMPLES_IO/SYS_TYPE_0/H2O_H2O_Identical): 152 terms (kcal/mol) at 2 R
    # points -> MTRX.DAT (81 parity-adapted states with their exchange parity P, 322 pairs).
    d = os.path.join(ex, "SYS_TYPE_0", "H2O_H2O_Identical")
    coll0, nch0, states0, ind0, R0, mat0 = _read_mtrx_dat(os.path.join(d, "MTRX.DAT"), 11)
    inp = open(os.path.join(d, "H2O_H2O_Identical.inp")).read()
    tl = re.split(r"(?<![A-Z_])TERMS\s*=", inp)[1].split("$END")[0]
    lab0 = np.array([int(x) for x in tl.replace(",", " ").split()], dtype=np.int32).reshape(-1, 5)
    with open(os.path.join(d, "PES_EXPAN_TERMS.DAT")) as f:
        f.readline()
        rows0 = np.array([[float(x) for x in ln.split()] for ln in f if ln.strip()])
    np.savez_compressed(
        os.path.join(out, "g5c_h2o_h2o_identical.npz"), coll=coll0, states=states0, ind_mat=ind0,
        R=R0, mat=mat0, labels=lab0, terms=rows0[:, 1:], R_terms=rows0[:, 0],
        A=27.87700, B=9.28500, C=14.51200,
        channels=np.array([[0, 0, 0, 0, 0, 0], [0, 0, 0, 1, 1, 1], [0, 0, 0, 2, 0, 2],
                           [1, 1, 1, 1, 1, 1], [1, 1, 1, 2, 0, 2], [2, 0, 2, 2, 0, 2]],
                          dtype=np.int32))

    # G6: the term lists CALC_EXPANSION generated from the $POTENTIAL limits
    # (EXPANSION_TERMS_LIST.DAT of EXAMPLES_IO/SYS_TYPE_8/H2O_H2_GeneratingTerms:
    # L1 0-4, L2 0-4, M1_MAX 4, AXL_SYM1 2, EQU_SYM2 2, ODD_L1L2L YES; and of
    # EXAMPLES_IO/SYS_TYPE_7/NH3_H2_Generation_of_Terms: L1 0-4, L2 0-2, M1_MAX 3).
    lists = {}
    for key, sub in (("h2o_h2_type8", ("SYS_TYPE_8", "H2O_H2_GeneratingTerms")),
                     ("nh3_h2_type7", ("SYS_TYPE_7", "NH3_H2_Generation_of_Terms"))):
        txt = open(os.path.join(ex, *sub, "EXPANSION_TERMS_LIST.DAT")).read().split()
        lists[key] = np.array([[int(x) for x in t.strip(",").split(",")] for t in txt],
                              dtype=np.int32)
    np.savez_compressed(os.path.join(out, "g6_expansion_term_lists.npz"), **lists)

    # G7: PES_EXPAN_TERMS.DAT as CALC_EXPANSION_TERMS wrote it over two R ranges
    # (EXAMPLES_IO/SYS_TYPE_7/NH3_H2_IR_BGN_FIN, IR_BGN/IR_FIN = 1-20 and 21-40; 37 terms,
    # ND3+D2): the exact text lines of both files and the term labels.
    d = os.path.join(ex, "SYS_TYPE_7", "NH3_H2_IR_BGN_FIN")
    texts = {}
    for key, sub in (("lines_1_20", "GRD_R_1_20"), ("lines_21_40", "GRD_R_21_40")):
        with open(os.path.join(d, sub, "PES_EXPAN_TERMS.DAT")) as f:
            texts[key] = np.array(f.read().split("\n"))
    head = str(texts["lines_1_20"][0]).split()
    labels_ir = np.array([[int(x) for x in h.split("_")[1:]] for h in head[1:]], dtype=np.int32)
    np.savez_compressed(os.path.join(out, "g7_expan_terms_files.npz"), labels=labels_ir, **texts)

    # G4: asymmetric top + atom (SYS_TYPE 4), MF_He with CS_APPROX = YES: state ordering,
    # levels, and the coupled-states dynamics on the reference's own matrix
    # (OPACITY_FUNCTIONS_L.out, DEFLECTION_FUNCTION.out finish times, CROSS_SECTIONS.out).
    d = os.path.join(ex, "SYS_TYPE_4", "MF_He_CS_MQCT")
    coll, nch, states4, ind4, R4, mat4 = _read_mtrx_dat(os.path.join(d, "MTRX.DAT"), 7)
    opac4 = _read_table(os.path.join(d, "OPACITY_FUNCTIONS_L.out"), 2 + nch)
    defl4 = _read_table(os.path.join(d, "DEFLECTION_FUNCTION.out"), 9, first_int=False)
    sig4 = []
    for line in open(os.path.join(d, "CROSS_SECTIONS.out")):
        t = line.split()
        if len(t) == 5 and t[0].isdigit():
            sig4.append(float(t[2]))
    np.savez_compressed(os.path.join(out, "g4_type4_layout.npz"), states=states4, ind_mat=ind4,
                        R=R4, mat=mat4, A=0.6666525, B=0.1769383, C=0.2306476,
                        channels=np.array([[0, 0, 0], [1, 0, 1], [1, 1, 1]], dtype=np.int32),
                        e_ch_printed=np.array([0.000, 0.408, 0.844]),
                        opacity=opac4, deflection=defl4, sigma_U=np.array(sig4),
                        # the result files as written (for the writers' byte-for-byte tests)
                        **{"text_" + name.split(".")[0].lower(): np.array(
                            open(os.path.join(d, name)).read())
                           for name in ("OPACITY_FUNCTIONS_L.out", "TOTAL_PROBABILITIES_L.out",
                                        "PARTIAL_CROSS_SECTIONS_J.out", "M_PROJ_CROSSECTIONS.out",
                                        "CROSS_SECTIONS.out", "DEFLECTION_FUNCTION.out")},
                        # $SYSTEM of MF_He_CS_MQCT.inp (R_COM in bohr whatever R_UNITS)
                        mass_red=3.7523705333, rmax=42.40, U=50.0, b_impct=20.0,
                        time_step=10.0, time_lim=3.5e6)

    # G8: elastic scattering with DIFF_CROSS = YES (ND3 + D2, SYS_TYPE 7, U = 800 cm^-1,
    # 101 trajectories l = 0..100, j_ini = 0, 2000 angles): the printed deflection function
    # and phases, the elastic channel's probabilities, the differential cross section and
    # the elastic cross section of CROSS_SECTIONS.out (ELAST_CALC, propagator.f:5581-6137).
    d = os.path.join(ex, "SYS_TYPE_7", "NH3_H2_DIFF_CROSS")
    defl8 = _read_table(os.path.join(d, "DEFLECTION_FUNCTION.out"), 9, first_int=False)
    opac8 = _read_table(os.path.join(d, "OPACITY_FUNCTIONS_L.out"), 16)
    sig8 = []
    for line in open(os.path.join(d, "CROSS_SECTIONS.out")):
        t = line.split()
        if len(t) == 5 and t[0].isdigit():
            sig8.append(float(t[2]))
    np.savez_compressed(os.path.join(out, "g8_diff_cross.npz"), deflection=defl8,
                        p_elastic=opac8[:, 2], sigma_U=np.array(sig8),
                        text_diff_cross=np.array(open(os.path.join(d, "DIFF_CROSS.out")).read()),
                        text_deflection_function=np.array(
                            open(os.path.join(d, "DEFLECTION_FUNCTION.out")).read()),
                        # $SYSTEM of NH3H2.inp
                        mass_red=3.354120939, U=800.0, n_angles=2000, j_ini=0, J_down=0,
                        J_up=100, L_min=0, dl=1)

    # G9: PROB_SPLINE = YES with DL = 3 (CO + H2, SYS_TYPE 6, U = 1000 cm^-1, 47
    # trajectories at l = 1, 4, ..., 139, j_ini = 0): probabilities and deflection function
    # splined over l in INELAST_CALC and ELAST_CALC (propagator.f:4889-4975, 5960-6110).
    d = os.path.join(ex, "SYS_TYPE_6", "CO_H2_Prob_spline")
    opac9 = _read_table(os.path.join(d, "OPACITY_FUNCTIONS_L.out"), 6)
    defl9 = _read_table(os.path.join(d, "DEFLECTION_FUNCTION.out"), 9, first_int=False)
    sig9 = []
    for line in open(os.path.join(d, "CROSS_SECTIONS.out")):
        t = line.split()
        if len(t) == 5 and t[0].isdigit():
            sig9.append(float(t[2]))
    np.savez_compressed(os.path.join(out, "g9_prob_spline.npz"), opacity=opac9, deflection=defl9,
                        sigma_U=np.array(sig9),
                        text_interpolated=np.array(open(os.path.join(
                            d, "INTERPOLATED_PROBS_DEFLECTION_L.out")).read()),
                        # $SYSTEM of CO_H2_Prob_spline.inp; l = 0 .. int(B_IMPCT k)
                        mass_red=1.88027, U=1000.0, dl=3, L_min=0, L_max=139)

    # G1 AT trajectory record layout: Fortran unformatted, 8 float64 per record.
    d = os.path.join(ex, "SYS_TYPE_0", "H2O_H2O_AT_Approximation", "AT_MQCT_2nd_Step",
                     "AT_APPROX_TRAJS", "500.00000", "0", "0")
    raw = open(os.path.join(d, "AT_0_0_9_0"), "rb").read()
    cnt = struct.unpack("<iii", open(os.path.join(d, "n_AT_0_0_9_0"), "rb").read())[1]
    recs = []
    off = 0
    while off < len(raw):
        n = struct.unpack_from("<i", raw, off)[0]
        recs.append(struct.unpack_from("<8d", raw, off + 4))
        off += n + 8
    recs = np.array(recs)
    np.savez_compressed(os.path.join(out, "g1_at_traj_l9.npz"), n_records=cnt,
                        head=recs[:8], tail=recs[-4:], n_file=len(recs),
                        t_span=np.array([recs[0, 0], recs[-1, 0]]))
    # G1: two asymmetric tops (SYS_TYPE 0), H2O+H2O AT-MQCT in two runs
    # (EXAMPLES_IO/SYS_TYPE_0/H2O_H2O_AT_Approximation).  Both runs build their
    # matrix from the same PES_EXPAN_TERMS.DAT (empty header line, then one row per
    # R: f6.2 R and 28 values in kcal/mol); the term labels (l1, nju1, l2, nju2, l)
    # are the TERMS list of the input.  The 1st run (one channel, RK4 step 10)
    # saves the classical paths (AT_APPROX_TRAJS, one file per l = 9, 28, ..., 256);
    # the 2nd run (9 channels, AT_APPROX, step 100) propagates along them.  Kept:
    # per path its record count and its first 4, middle 3 and last 3 records; the
    # 2nd run's opacities, deflection table and cross sections.
    base = os.path.join(ex, "SYS_TYPE_0", "H2O_H2O_AT_Approximation")
    d1 = os.path.join(base, "AT_MQCT_1st_Step")
    d2 = os.path.join(base, "AT_MQCT_2nd_Step")
    inp = open(os.path.join(d2, "H2O_H2O_AT_MQCT_2nd_run.inp")).read()
    tl = re.split(r"(?<![A-Z_])TERMS\s*=", inp)[1].split("$END")[0]
    lab = np.array([int(x) for x in tl.replace(",", " ").split()], dtype=np.int32).reshape(-1, 5)
    with open(os.path.join(d2, "PES_EXPAN_TERMS.DAT")) as f:
        f.readline()
        rows = np.array([[float(x) for x in ln.split()] for ln in f if ln.strip()])
    tdir = os.path.join(d2, "AT_APPROX_TRAJS", "500.00000", "0", "0")
    ls = np.arange(9, 257, 19)
    n_rec, heads, mids, tails = [], [], [], []
    for l in ls:
        raw = open(os.path.join(tdir, f"AT_0_0_{l}_0"), "rb").read()
        recs = []
        off = 0
        while off < len(raw):
            n = struct.unpack_from("<i", raw, off)[0]
            recs.append(struct.unpack_from("<8d", raw, off + 4))
            off += n + 8
        recs = np.array(recs)
        n_rec.append(len(recs))
        heads.append(recs[:4])
        h = len(recs) // 2
        mids.append(recs[h - 1:h + 2])
        tails.append(recs[-3:])
    sig2 = []
    for line in open(os.path.join(d2, "CROSS_SECTIONS.out")):
        t = line.split()
        if len(t) == 5 and t[0].isdigit():
            sig2.append(float(t[2]))
    # M-resolved cross sections (channel 1 there is the probability sum of the
    # initial channel; CROSS_SECTIONS.out reports ELAST_CALC's elastic value instead)
    sig2m = []
    for line in open(os.path.join(d2, "M_PROJ_CROSSECTIONS.out")):
        t = line.split()
        if len(t) == 2 and t[0].isdigit():
            sig2m.append(float(t[1]))
    # J-resolved cross sections (Angstrom^2) of PARTIAL_CROSS_SECTIONS_J.out: J, 9 channels
    part = np.array([[float(x) for x in ln.split()]
                     for ln in open(os.path.join(d2, "PARTIAL_CROSS_SECTIONS_J.out"))
                     if len(ln.split()) == 10 and ln.split()[0].isdigit()])
    np.savez_compressed(
        os.path.join(out, "g1_h2o_h2o_at.npz"), labels=lab, R=rows[:, 0], terms=rows[:, 1:],
        sigma2_mproj=np.array(sig2m), partial2=part,
        l=ls, n_rec=np.array(n_rec), rec_head=np.array(heads), rec_mid=np.array(mids),
        rec_tail=np.array(tails),
        opacity2=_read_table(os.path.join(d2, "OPACITY_FUNCTIONS_L.out"), 11),
        deflection1=_read_table(os.path.join(d1, "DEFLECTION_FUNCTION.out"), 9, first_int=False),
        deflection2=_read_table(os.path.join(d2, "DEFLECTION_FUNCTION.out"), 9, first_int=False),
        sigma2=np.array(sig2),
        # $BASIS/$SYSTEM of the two inputs
        A=27.87700, B=9.28500, C=14.51200, mass_red=9.00764, U=500.0, b_impct=30.0, rmax=30.0,
        dl=19, time_step1=10.0, time_step2=100.0, time_lim=3.5e6,
        channels=np.array([[0, 0, 0, 0, 0, 0], [0, 0, 0, 1, 1, 1], [0, 0, 0, 2, 0, 2],
                           [1, 1, 1, 0, 0, 0], [1, 1, 1, 1, 1, 1], [1, 1, 1, 2, 0, 2],
                           [2, 0, 2, 0, 0, 0], [2, 0, 2, 1, 1, 1], [2, 0, 2, 2, 0, 2]],
                          dtype=np.int32))
    print("fixtures written to", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the MQCT reference checkout>")
    main(sys.argv[1])
