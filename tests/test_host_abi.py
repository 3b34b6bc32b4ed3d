"""CPU checks of the product library: it loads, exports every symbol that
include/mqct_b200.h declares, and its host-side logic (levels, states, pairs,
R grid, matrix files, argument validation) agrees with the oracle.  No
compute entry point is called here (no GPU in this tier)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header_symbols(mq):
    from mqct_b200 import _abi
    L = _abi.lib()
    hdr = open(os.path.join(ROOT, "include", "mqct_b200.h")).read()
    declared = set(re.findall(r"\b(mqct_[a-z0-9_]+)\s*\(", hdr))
    assert declared == set(_abi.EXPORTS), declared ^ set(_abi.EXPORTS)
    for name in declared:
        assert hasattr(L, name), name
    assert L.mqct_version() >= 10000


def test_levels_and_eigenvectors_match_oracle(mq, oracle):
    for (A, B, Cc) in [(27.9, 14.5, 9.3), (27.88063134, 9.277708381, 14.52176959)]:
        for j in range(0, 9):
            ka = [0] + [i // 2 for i in range(2, 2 * j + 2)]
            for i in range(2 * j + 1):
                e1, v1 = mq.asym_top_level(A, B, Cc, j, ka[i], ka[::-1][i])
                e2, v2 = oracle.asym_top(A, B, Cc, j, ka[i], ka[::-1][i])
                assert abs(e1 - e2) <= 1e-11 * max(1.0, abs(e2))
                assert np.max(np.abs(v1 - v2)) < 1e-10


def test_invalid_level_is_an_error(mq):
    with pytest.raises(mq.MqctError):
        mq.asym_top_level(27.9, 14.5, 9.3, 2, 2, 2)


@pytest.mark.parametrize("sys_type,chans", [
    (1, [(j,) for j in range(11)]),
    (4, [(0, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0), (2, 0, 2), (2, 1, 1)]),
    (8, [(0, 0, 0, 0), (1, 1, 1, 0), (1, 0, 1, 1), (2, 1, 2, 1)]),
])
def test_states_and_pairs_match_oracle(mq, oracle, sys_type, chans):
    s = mq.CollisionSystem(sys_type, chans, A=27.9, B=14.5, C=9.3, BE=1.93)
    ch = np.array(chans)
    if sys_type == 1:
        osys = oracle.OracleSystem(1, ch[:, 0], e_ch=s.e_ch, vec1=np.ones(len(ch)), ldv=1)
    elif sys_type == 4:
        osys = oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=s.e_ch, vec1=s.vec1, ldv=s.ldv)
    else:
        osys = oracle.OracleSystem(8, ch[:, 0], ch[:, 1], ch[:, 2], j2=ch[:, 3], e_ch=s.e_ch,
                                   vec1=s.vec1, ldv=s.ldv)
    ic, j12, m12, ej = osys.states()
    assert (ic == s.indx_chann).all() and (j12 == s.j12).all() and (m12 == s.m12).all()
    assert np.allclose(ej, s.ej_cm)
    assert (oracle.ind_mat(m12) == s.ind_mat).all()


def test_c2_basis_counts(mq):
    from mqct_b200 import synthetic as syn
    c2 = syn.config_c2()
    s = mq.CollisionSystem(4, c2["channels"], A=27.9, B=14.5, C=9.3)
    assert (s.n_channels, s.n_states, s.P) == (81, 969, 31977)


def test_r_grids_match_oracle(mq, oracle):
    for eq in (True, False):
        for n in (3, 7, 200, 301):
            assert np.array_equal(mq.r_grid(n, 3.0, 25.0, eq), oracle.rgrid(n, 3.0, 25.0, eq))
    assert np.array_equal(mq.r_grid(2, 3.0, 25.0, True), [3.0, 25.0])
    with pytest.raises(mq.MqctError):
        mq.r_grid(2, 3.0, 25.0, False)


def test_mtrx_uf_roundtrip_and_oracle_layout(mq, oracle, tmp_path):
    s = mq.CollisionSystem(4, [(0, 0, 0), (1, 0, 1), (1, 1, 1), (2, 0, 2)], A=27.9, B=14.5, C=9.3)
    R = np.linspace(3, 20, 17)
    mat = np.random.default_rng(0).normal(size=(s.P, len(R)))
    p1 = str(tmp_path / "a.dat")
    p2 = str(tmp_path / "b.dat")
    mq.write_mtrx_uf(p1, s, R, mat)
    rec = s.state_records()
    oracle.lib().orc_write_mtrx_uf(p2.encode(), 4, s.n_channels, s.n_states,
                                   np.ascontiguousarray(rec.reshape(-1)), rec.shape[1], s.P,
                                   np.ascontiguousarray(s.ind_mat.reshape(-1)), len(R), R,
                                   np.ascontiguousarray(mat.reshape(-1)))
    assert open(p1, "rb").read() == open(p2, "rb").read()
    back = mq.read_mtrx_uf(p1)
    assert back["coll_type"] == 4 and back["n_channels"] == s.n_channels
    assert np.array_equal(back["states"], rec)
    assert np.array_equal(back["ind_mat"], s.ind_mat)
    assert np.array_equal(back["R"], R) and np.array_equal(back["mat"], mat)


def test_malformed_matrix_file_is_rejected(mq, tmp_path):
    s = mq.CollisionSystem(1, [(0,), (1,), (2,)], BE=1.93)
    R = np.linspace(3, 10, 5)
    p = str(tmp_path / "m.dat")
    mq.write_mtrx_uf(p, s, R, np.ones((s.P, 5)))
    raw = bytearray(open(p, "rb").read())
    open(p, "wb").write(raw[: len(raw) - 13])          # truncated
    with pytest.raises(mq.MqctError):
        mq.read_mtrx_uf(p)
    raw2 = bytearray(raw)
    raw2[60] ^= 0x40                                    # corrupt the first state-record marker
    open(p, "wb").write(raw2)
    with pytest.raises(mq.MqctError):
        mq.read_mtrx_uf(p)
    with pytest.raises(mq.MqctError):
        mq.read_mtrx_uf(str(tmp_path / "missing.dat"))


def test_host_spline_matches_oracle(mq, oracle):
    R = np.linspace(3, 25, 41)
    Y = np.stack([np.exp(-R) * np.cos(R), 1 / R ** 6, np.sin(R) * 1e-6])
    y2 = mq.spline_y2(R, Y)
    for k in range(3):
        c = Y[k]
        ref = oracle.spline(R, c, (c[1] - c[0]) / (R[1] - R[0]), (c[-1] - c[-2]) / (R[-1] - R[-2]))
        assert np.allclose(y2[k], ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def test_compute_entry_points_validate_arguments(mq):
    """Argument errors are returned as codes (no device work is started)."""
    from mqct_b200 import _abi
    L = _abi.lib()
    rc = L.mqct_build_matrix(None, np.zeros(2, np.int32), 1, np.zeros(2), 2, None, None, 0, 0.0,
                             6.0, 8.0, np.zeros(2), None, None, None)
    assert rc < 0
    h = _abi.vp()
    rc = L.mqct_prop_plan_create(None, 1, C.byref(h))
    assert rc < 0


def test_synthetic_pes_kinds_match_the_abi(mq):
    """The synthetic module keeps the PES kinds as plain numbers (it loads without the
    CUDA library); they are the C ABI's MQCT_PES_* values."""
    from mqct_b200 import _abi, synthetic as syn
    assert (syn.PES_TABLE, syn.PES_LEGENDRE, syn.PES_SITES1, syn.PES_SITES2) == (
        _abi.PES_TABLE, _abi.PES_LEGENDRE, _abi.PES_SITES1, _abi.PES_SITES2)
