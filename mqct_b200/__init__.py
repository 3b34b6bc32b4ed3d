"""mqct_b200 -- B200-native matrix build and trajectory propagation for MQCT.

Host API mirroring the reference's flow (MarquetteQuantum/MQCT):

    $BASIS    -> CollisionSystem        (channels, levels, INI_ARRAYS states/pairs)
    $POTENTIAL-> build_matrix / MatrixPlan (MATRIX_MAKE direct integration, CUDA)
              -> write_mtrx_uf / read_mtrx_uf (SAVE_MTRX / READ_MTRX, MTRX_UF.DAT)
    $SYSTEM   -> PropagationTables + trajectory_set + propagate (PROPAGATE/DOTRAJECT, CUDA)
              -> cross_sections (INELAST_CALC + the Billing correction)

All compute runs in libmqct_b200.so (include/mqct_b200.h); this module only
prepares host arrays and calls the C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import (ENGINE_AUTO, ENGINE_LOCKSTEP, ENGINE_LOCKSTEP_TAIL, ENGINE_PER_TRAJECTORY,
                   ENGINE_RESIDENT, MODE_AT, MODE_CS, MODE_STD, PREC_BF16X3, PREC_F16X3, PREC_FP64, PROP_FP32, PROP_FP64,
                   MqctError, check, lib, ptr)
from .synthetic import A_BOHR, AMU_TO_AU, AU_TO_EV, CM_TO_HARTREE, EV_TO_WN

__all__ = ["CollisionSystem", "build_matrix", "MatrixPlan", "PropagationTables", "propagate",
           "PropagationPlan", "propagate_record", "trajectory_set", "cross_sections",
           "cross_sections_device", "write_mtrx_uf",
           "read_mtrx_uf", "write_mtrx_dat", "read_mtrx_dat", "read_expansion_terms",
           "spline_y2", "Surrogate", "release_cached_build", "build_matrix_expansion", "ExpansionPlan", "E_UNIT",
           "expansion_terms_list", "write_expansion_terms_list",
           "MqctError",
           "PREC_FP64", "PREC_BF16X3", "PREC_F16X3", "PROP_FP32", "PROP_FP64", "MODE_STD",
           "MODE_AT", "MODE_CS"]


def asym_top_level(A, B, Cc, j, ka, kc):
    """Energy and symmetric-top coefficients (K=-j..j) of level (j, ka, kc)."""
    e = C.c_double()
    v = np.zeros(2 * j + 1)
    check(lib().mqct_asym_top_level(A, B, Cc, j, ka, kc, C.byref(e), v))
    return e.value, v


class CollisionSystem:
    """Collision system after the $BASIS block and INI_ARRAYS.

    sys_type 1: channels (j,), energy BE j(j+1) - DE (j(j+1))^2 (MQCT_SOURCE_CODES/iotest.f:5454);
    sys_type 5: channels (j1, j2) of two diatoms, energy BE j1(j1+1) - DE (j1(j1+1))^2 +
    BE2 j2(j2+1) - DE2 (j2(j2+1))^2 (BE1/DE1/BE2/DE2 of $BASIS; BE2, DE2 default to BE, DE);
    sys_type 3: channels (j, k, eps) of a symmetric top, energy A j(j+1) - (A-C) k^2
    (MQCT_SOURCE_CODES/iotest.f:6250, 6355); k and eps are kept in ka1 and kc1, vec1 as for 7;
    sys_type 4: channels (j, ka, kc), energy EIGEN_VAL(A,B,C) (MQCT_SOURCE_CODES/iotest.f:6611-6618);
    sys_type 7: channels (j1, k, eps, j2), A j1(j1+1) - (A-C) k^2 + BE j2(j2+1) - DE (j2(j2+1))^2
    (MQCT_SOURCE_CODES/iotest.f:8311-8312); k and eps are kept in ka1 and kc1, and vec1 holds
    the parity-adapted top (|j k> + (-1)^eps |j -k>) / sqrt(2 (1 + delta_k0)) over K;
    sys_type 8: channels (j1, ka1, kc1, j2), EIGEN_VAL + BE j2(j2+1) (MQCT_SOURCE_CODES/iotest.f:9069-9079);
    sys_type 9: channels (j1, ka1, kc1, j2, k2, eps2), EIGEN_VAL(A,B,C) + A2 j2(j2+1) -
    (A2-C2) k2^2 (MQCT_SOURCE_CODES/iotest.f:9445-9498, 9670-9677); A2 = B2 of the symmetric
    top, taken from B2 when A2 is not given, C2 required (iotest.f:9414-9416); k2 and eps2
    are kept in ka2 and kc2, vec2 holds the second rotor's parity-adapted vector;
    sys_type 0: channels (j1, ka1, kc1, j2, ka2, kc2), EIGEN_VAL(A1..) + EIGEN_VAL(A2..);
    identical=True (IDENTICAL = YES): parity-adapted states with their exchange parity
    (self.parity), pairs only between equal parities (MQCT_SOURCE_CODES/matrix_ini.f:482-627).
    """

    def __init__(self, sys_type, channels, A=0.0, B=0.0, C=0.0, BE=0.0, DE=0.0, A2=None,
                 B2=None, C2=None, e_ch=None, identical=False, BE2=None, DE2=None):
        ch = np.asarray(channels, dtype=np.int32)
        if ch.ndim == 1:
            ch = ch[:, None]
        self.sys_type = int(sys_type)
        self.channels = ch
        nch = len(ch)
        self.n_channels = nch
        z = np.zeros(nch, np.int32)
        self.j1 = np.ascontiguousarray(ch[:, 0])
        self.ka1 = self.kc1 = self.j2 = self.ka2 = self.kc2 = z
        j2col = 1 if sys_type == 5 else 3
        jmax = (int(ch[:, 0].max()) if sys_type in (1, 3, 4)
                else int(max(ch[:, 0].max(), ch[:, j2col].max())))
        self.ldv = 2 * jmax + 1
        self.vec1 = np.zeros((nch, self.ldv))
        self.vec2 = np.zeros((nch, self.ldv))
        E = np.zeros(nch)
        if sys_type == 1:
            jj = self.j1 * (self.j1 + 1.0)
            E = BE * jj - DE * jj ** 2
            self.vec1[:, 0] = 1.0
        elif sys_type == 5:
            self.j2 = np.ascontiguousarray(ch[:, 1])
            BE2 = BE if BE2 is None else BE2
            DE2 = DE if DE2 is None else DE2
            jj1 = self.j1 * (self.j1 + 1.0)
            jj2 = self.j2 * (self.j2 + 1.0)
            E = BE * jj1 - DE * jj1 ** 2 + BE2 * jj2 - DE2 * jj2 ** 2
            self.vec1[np.arange(nch), self.j1] = 1.0
        elif sys_type in (4, 8):
            self.ka1 = np.ascontiguousarray(ch[:, 1])
            self.kc1 = np.ascontiguousarray(ch[:, 2])
            for i in range(nch):
                e, v = asym_top_level(A, B, C, int(ch[i, 0]), int(ch[i, 1]), int(ch[i, 2]))
                E[i] = e
                self.vec1[i, :len(v)] = v
            if sys_type == 8:
                self.j2 = np.ascontiguousarray(ch[:, 3])
                jj = self.j2 * (self.j2 + 1.0)
                E = E + BE * jj - DE * jj ** 2
        elif sys_type in (3, 7):
            self.ka1 = np.ascontiguousarray(ch[:, 1])
            self.kc1 = np.ascontiguousarray(ch[:, 2])
            j1 = self.j1.astype(np.float64)
            E = A * j1 * (j1 + 1.0) - (A - C) * self.ka1 ** 2.0
            if sys_type == 7:
                self.j2 = np.ascontiguousarray(ch[:, 3])
                jj = self.j2 * (self.j2 + 1.0)
                E = E + BE * jj - DE * jj ** 2
            for i in range(nch):
                j, k, eps = int(ch[i, 0]), int(ch[i, 1]), int(ch[i, 2])
                if not (0 <= k <= j and eps in (0, 1) and not (k == 0 and eps == 1)):
                    raise ValueError(f"bad symmetric-top channel {tuple(ch[i])}")
                a = 1.0 / np.sqrt(2.0 * (1.0 + (k == 0)))
                self.vec1[i, j + k] += a
                self.vec1[i, j - k] += -a if eps else a
        elif sys_type == 9:
            self.ka1, self.kc1 = np.ascontiguousarray(ch[:, 1]), np.ascontiguousarray(ch[:, 2])
            self.j2, self.ka2, self.kc2 = (np.ascontiguousarray(ch[:, 3]),
                                           np.ascontiguousarray(ch[:, 4]),
                                           np.ascontiguousarray(ch[:, 5]))
            # the second (symmetric) top: A2 = B2, taken from B2 when A2 is not given, and
            # C2 required (MQCT_SOURCE_CODES/iotest.f:1675-1677, 9414-9416)
            a2 = 0.0 if A2 is None else float(A2)
            b2 = 0.0 if B2 is None else float(B2)
            if a2 + b2 == 0.0:
                raise ValueError("SYS_TYPE 9: supply A2 or B2 of the symmetric top")
            A2 = a2 if a2 != 0.0 else b2
            if C2 is None or float(C2) == 0.0:
                raise ValueError("SYS_TYPE 9: supply C2 of the symmetric top")
            for i in range(nch):
                e1, v1 = asym_top_level(A, B, C, *map(int, ch[i, 0:3]))
                j, k, eps = map(int, ch[i, 3:6])
                if not (0 <= k <= j and eps in (0, 1) and not (k == 0 and eps == 1)):
                    raise ValueError(f"bad symmetric-top level {tuple(ch[i, 3:6])}")
                E[i] = e1 + A2 * j * (j + 1.0) - (A2 - C2) * k ** 2
                self.vec1[i, :len(v1)] = v1
                a = 1.0 / np.sqrt(2.0 * (1.0 + (k == 0)))
                self.vec2[i, j + k] += a
                self.vec2[i, j - k] += -a if eps else a
        elif sys_type == 0:
            self.ka1, self.kc1 = np.ascontiguousarray(ch[:, 1]), np.ascontiguousarray(ch[:, 2])
            self.j2, self.ka2, self.kc2 = (np.ascontiguousarray(ch[:, 3]),
                                           np.ascontiguousarray(ch[:, 4]),
                                           np.ascontiguousarray(ch[:, 5]))
            A2 = A if A2 is None else A2
            B2 = B if B2 is None else B2
            C2 = C if C2 is None else C2
            for i in range(nch):
                e1, v1 = asym_top_level(A, B, C, *map(int, ch[i, 0:3]))
                e2, v2 = asym_top_level(A2, B2, C2, *map(int, ch[i, 3:6]))
                E[i] = e1 + e2
                self.vec1[i, :len(v1)] = v1
                self.vec2[i, :len(v2)] = v2
        else:
            raise ValueError(f"unsupported SYS_TYPE {sys_type}")
        self.e_ch = np.asarray(E if e_ch is None else e_ch, dtype=np.float64)
        L = lib()
        self.identical = bool(identical)
        self.parity = None
        if self.identical:
            # IDENTICAL = YES: states carry the exchange parity, pairs join equal parities
            if sys_type != 0:
                raise ValueError("identical partners are supported for SYS_TYPE 0")
            rot = [np.ascontiguousarray(x, np.int32) for x in
                   (self.j1, self.ka1, self.kc1, self.j2, self.ka2, self.kc2)]
            n = check(L.mqct_count_states_identical(nch, *rot))
            self.indx_chann = np.zeros(n, np.int32)
            self.j12 = np.zeros(n, np.int32)
            self.m12 = np.zeros(n, np.int32)
            self.parity = np.zeros(n, np.int32)
            check(L.mqct_enumerate_states_identical(nch, *rot, self.indx_chann, self.j12,
                                                    self.m12, self.parity))
            P = check(L.mqct_count_pairs_identical(n, self.m12, self.parity))
            ind = np.zeros(2 * P, np.int32)
            check(L.mqct_fill_ind_mat_identical(n, self.m12, self.parity, ind))
        else:
            j2p = ptr(self.j2) if sys_type in (5, 7, 8, 9, 0) else None
            n = check(L.mqct_count_states(self.sys_type, nch, self.j1, j2p))
            self.indx_chann = np.zeros(n, np.int32)
            self.j12 = np.zeros(n, np.int32)
            self.m12 = np.zeros(n, np.int32)
            check(L.mqct_enumerate_states(self.sys_type, nch, self.j1, j2p, self.indx_chann,
                                          self.j12, self.m12))
            P = check(L.mqct_count_pairs(n, self.m12))
            ind = np.zeros(2 * P, np.int32)
            check(L.mqct_fill_ind_mat(n, self.m12, ind))
        self.n_states = n
        self.ej_cm = self.e_ch[self.indx_chann - 1]
        self.ind_mat = ind.reshape(P, 2)
        self.P = int(P)
        self.vec1 = np.ascontiguousarray(self.vec1)
        self.vec2 = np.ascontiguousarray(self.vec2)

    def c_struct(self):
        return _abi.Sys(self.sys_type, self.n_channels, ptr(self.j1), ptr(self.ka1), ptr(self.kc1),
                        ptr(self.j2), ptr(self.ka2), ptr(self.kc2), ptr(self.vec1),
                        ptr(self.vec2), self.ldv, self.n_states, ptr(self.indx_chann),
                        ptr(self.j12), ptr(self.m12), ptr(self.parity))

    def state_records(self):
        """Per-state records of MTRX_UF.DAT (MQCT_SOURCE_CODES/matrix_ini.f:6666-6757)."""
        st = np.arange(1, self.n_states + 1, dtype=np.int32)
        ic = self.indx_chann
        cols = [st, ic, self.j12, self.m12]
        if self.sys_type == 1:
            cols += [self.j1[ic - 1]]
        elif self.sys_type in (3, 4):                      # matrix_ini.f:4744-4759
            cols += [self.j1[ic - 1], self.ka1[ic - 1], self.kc1[ic - 1]]
        elif self.sys_type == 5:
            cols += [self.j1[ic - 1], self.j2[ic - 1]]    # matrix_ini.f:4760-4767
        elif self.sys_type in (7, 8):
            cols += [self.j1[ic - 1], self.ka1[ic - 1], self.kc1[ic - 1], self.j2[ic - 1]]
        else:
            cols += [self.j1[ic - 1], self.ka1[ic - 1], self.kc1[ic - 1], self.j2[ic - 1],
                     self.ka2[ic - 1], self.kc2[ic - 1]]
            if self.identical:
                cols += [self.parity]       # the P column (matrix_ini.f:4846-4857)
        return np.ascontiguousarray(np.stack(cols, axis=1).astype(np.int32))


class Surrogate:
    """Learned PES surrogate (MLP on (R, cos/sin of the angles)) trained on the GPU
    by the library's own kernels; see mqct_surrogate_* in include/mqct_b200.h."""

    N_FEATURES = 11

    def __init__(self, sys_type, pes, hidden=256, layers=4, seed=1, r_min=4.0, r_max=25.0):
        self._pes = PesSpec.from_dict(pes) if isinstance(pes, dict) else pes
        self._ps = self._pes.c_struct()
        h = C.c_void_p()
        check(lib().mqct_surrogate_create(int(sys_type), C.byref(self._ps), hidden, layers,
                                          seed, r_min, r_max, C.byref(h)))
        self.h = h
        self.sys_type = int(sys_type)

    def train(self, n_samples=2_000_000, epochs=10, batch=4096, lr=1e-3):
        """Returns (last-batch loss per epoch, held-out RMSE), target units."""
        loss = np.zeros(epochs)
        val = C.c_double()
        check(lib().mqct_surrogate_train(self.h, n_samples, epochs, batch, lr, ptr(loss),
                                         C.byref(val)))
        return loss, float(val.value)

    def predict(self, args):
        """V (cm^-1) at rows (R, beta1, gamma1, alpha2, beta2, gamma2)."""
        a = np.ascontiguousarray(args, dtype=np.float64).reshape(-1, 6)
        out = np.zeros(len(a))
        check(lib().mqct_surrogate_predict(self.h, ptr(a), len(a), ptr(out)))
        return out

    def params(self):
        n = lib().mqct_surrogate_n_params(self.h)
        out = np.zeros(n, np.float32)
        check(lib().mqct_surrogate_get_params(self.h, ptr(out)))
        return out

    def loss_grad(self, X, y):
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(lib().mqct_surrogate_n_params(self.h), np.float32)
        loss = C.c_double()
        check(lib().mqct_surrogate_loss_grad(self.h, ptr(X), ptr(y), len(y), C.byref(loss), ptr(g)))
        return float(loss.value), g

    def close(self):
        if self.h:
            lib().mqct_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def r_grid(n, rmin, rmax, equidistant=True):
    R = np.zeros(n)
    check(lib().mqct_r_grid(n, rmin, rmax, 1 if equidistant else 0, R))
    return R


@dataclass
class PesSpec:
    kind: int
    n_terms: int
    params: np.ndarray
    sites1: np.ndarray | None = None
    sites2: np.ndarray | None = None
    table: np.ndarray | None = None

    @staticmethod
    def from_dict(d):
        return PesSpec(d["kind"], d["n_terms"], np.ascontiguousarray(d["params"], np.float64),
                       None if d.get("sites1") is None else np.ascontiguousarray(d["sites1"], np.float64),
                       None if d.get("sites2") is None else np.ascontiguousarray(d["sites2"], np.float64),
                       None if d.get("table") is None else np.ascontiguousarray(d["table"], np.float64))

    def c_struct(self):
        return _abi.Pes(self.kind, self.n_terms, ptr(self.params),
                        0 if self.sites1 is None else len(self.sites1) // 3,
                        0 if self.sites2 is None else len(self.sites2) // 3,
                        ptr(self.sites1), ptr(self.sites2), ptr(self.table))


def _grid_struct(grid):
    if isinstance(grid, _abi.Grid):
        return grid
    g = list(grid) + [0] * (7 - len(grid))
    return _abi.Grid(*g)


def build_matrix(system: CollisionSystem, R, grid, pes, precision=PREC_FP64, mij_cutoff=1e-12,
                 r_cut1=6.0, r_cut2=8.0, out=None):
    """MATRIX_MAKE direct integration on the GPU: returns Mat_el (P x nR, Hartree),
    its spline second derivatives and the MIJ_CUTOFF flags.  out: optional (mat, y2,
    skipped) arrays of shapes (P, nR), (P, nR), (P,) to fill (a host loop that reuses
    its buffers, as the reference's host keeps Mat_el allocated)."""
    R = np.ascontiguousarray(R, np.float64)
    pes = pes if isinstance(pes, PesSpec) else PesSpec.from_dict(pes)
    P, nR = system.P, len(R)
    if out is not None:
        mat, y2, sk = out
        if (mat.shape != (P, nR) or y2.shape != (P, nR) or sk.shape != (P,)
                or mat.dtype != np.float64 or y2.dtype != np.float64 or sk.dtype != np.int32
                or not (mat.flags.c_contiguous and y2.flags.c_contiguous and sk.flags.c_contiguous)):
            raise ValueError("out arrays must be C-contiguous float64 (P, nR) x 2 and int32 (P,)")
    else:
        mat = np.zeros((P, nR))
        y2 = np.zeros((P, nR))
        sk = np.zeros(P, np.int32)
    s = system.c_struct()
    g = _grid_struct(grid)
    ps = pes.c_struct()
    check(lib().mqct_build_matrix(C.byref(s), np.ascontiguousarray(system.ind_mat.reshape(-1)), P,
                                  R, nR, C.byref(g), C.byref(ps), precision, mij_cutoff, r_cut1,
                                  r_cut2, mat.reshape(-1), ptr(y2), ptr(sk), None))
    return mat, y2, sk


def release_cached_build():
    """Free the plan and device buffers that build_matrix keeps from its last call."""
    lib().mqct_release_cached_build()


# Hartree value of the PES_EXPAN_TERMS.DAT energy units (E_UNITS, conv_unit_e of
# MQCT_SOURCE_CODES/matrix_ini.f:918-921 with the constants of iotest.f:20-24)
E_UNIT = {"CM-1": CM_TO_HARTREE, "KCAL": 1.0 / 627.509469, "K": 1.0 / 1.1604519e4 / 27.21113845,
          "AU": 1.0}


def expansion_terms_list(sys_type, l1_max, l2_max, l1_min=0, l2_min=0, nju1_max=-1, l_max=-1,
                         axl_sym1=1, equ_sym1=1, equ_sym2=1, odd_l1l2l=False):
    """The term list CALC_EXPANSION generates for SYS_TYPE 7, 8 and 9 from the $POTENTIAL
    keywords L1_MIN/L1_MAX, L2_MIN/L2_MAX, M1_MAX (nju1_max), L_MAX, AXL_SYM1, EQU_SYM1,
    EQU_SYM2 and ODD_L1L2L (MQCT_SOURCE_CODES/pot_comp.f:4237-4262, 4314-4339): l1 in steps
    of EQU_SYM1, nju1 = 0..min(l1, M1_MAX) in steps of AXL_SYM1, l2 in steps of EQU_SYM2,
    l = |l1-l2|..min(l1+l2, L_MAX), without odd l1+l2+l unless ODD_L1L2L.  Returns an
    (n, 4) array of (l1, nju1, l2, l), the rows of EXPANSION_TERMS_LIST.DAT."""
    if sys_type not in (7, 8, 9):
        raise ValueError("term lists are generated here for SYS_TYPE 7, 8 and 9")
    nju1_max = l1_max if nju1_max < 0 else nju1_max
    l_max = l1_max + l2_max if l_max < 0 else l_max
    out = []
    for l1 in range(l1_min, l1_max + 1, equ_sym1):
        for nju1 in range(0, min(l1, nju1_max) + 1, axl_sym1):
            for l2 in range(l2_min, l2_max + 1, equ_sym2):
                for l in range(abs(l1 - l2), min(l1 + l2, l_max) + 1):
                    if not odd_l1l2l and (l1 + l2 + l) % 2:
                        continue
                    out.append((l1, nju1, l2, l))
    return np.array(out, dtype=np.int32).reshape(-1, 4)


def write_expansion_terms_list(path, labels):
    """EXPANSION_TERMS_LIST.DAT: one term per line, 'l1,nju1,l2,l,' (pot_comp.f:4250)."""
    with open(path, "w") as f:
        for row in np.asarray(labels, np.int32):
            f.write("".join(f"{int(v)}," for v in row) + "\n")


def build_matrix_expansion(system: CollisionSystem, R, labels, terms, e_unit="CM-1",
                           mij_cutoff=1e-12, r_cut1=6.0, r_cut2=8.0):
    """Matrix from PES expansion terms (READ_EXPANSION path; SYS_TYPE 1, 3, 4, 5, 7, 8, 0).

    labels: the TERMS list, one row per term: (l,) for SYS_TYPE 1, (l, nju) for SYS_TYPE
    3 and 4, (l1, l2, l) for SYS_TYPE 5, (l1, nju1, l2, l) for SYS_TYPE 7 and 8, (l1, nju1, l2,
    nju2, l) for SYS_TYPE 0.  terms: nR x n_terms as the rows of
    PES_EXPAN_TERMS.DAT, in the unit e_unit (a key of E_UNIT or the Hartree value of
    one unit).  Returns (Mat_el, y2, skipped) as build_matrix."""
    R = np.ascontiguousarray(R, np.float64)
    lab = np.asarray(labels, np.int32)
    lab = lab.reshape(len(lab), -1)
    a_top = np.zeros((len(lab), 5), np.int32)  # A_TOP(5, nterms)
    a_top[:, :lab.shape[1]] = lab
    # expansion_terms(n_r_coll, nterms): R fastest
    T = np.ascontiguousarray(np.asarray(terms, np.float64).reshape(len(R), len(lab)).T)
    eu = E_UNIT[e_unit.upper()] if isinstance(e_unit, str) else float(e_unit)
    P, nR = system.P, len(R)
    mat = np.zeros(P * nR)
    y2 = np.zeros(P * nR)
    sk = np.zeros(P, np.int32)
    sd = system.c_struct()
    ind = np.ascontiguousarray(system.ind_mat.reshape(-1))
    check(lib().mqct_build_matrix_expansion(C.byref(sd), ind, P, R, nR, len(lab),
                                            a_top.reshape(-1), T.reshape(-1), eu, mij_cutoff,
                                            r_cut1, r_cut2, mat, ptr(y2), ptr(sk)))
    return mat.reshape(P, nR), y2.reshape(P, nR), sk


class ExpansionPlan:
    """The expansion build with the angular coefficients formed once (mqct_expansion_plan_*);
    execute() turns radial terms on the device into Mat_el, y2 and the MIJ_CUTOFF flags in
    device buffers (torch tensors or raw device pointers)."""

    def __init__(self, system: CollisionSystem, R, labels, mij_cutoff=1e-12, r_cut1=6.0,
                 r_cut2=8.0):
        self.R = np.ascontiguousarray(R, np.float64)
        lab = np.asarray(labels, np.int32)
        lab = lab.reshape(len(lab), -1)
        a_top = np.zeros((len(lab), 5), np.int32)
        a_top[:, :lab.shape[1]] = lab
        self.n_terms = len(lab)
        self.P = system.P
        self._sd = system.c_struct()
        h = _abi.vp()
        check(lib().mqct_expansion_plan_create(C.byref(self._sd),
                                               np.ascontiguousarray(system.ind_mat.reshape(-1)),
                                               self.P, self.R, len(self.R), self.n_terms,
                                               a_top.reshape(-1), mij_cutoff, r_cut1, r_cut2,
                                               C.byref(h)))
        self.h = h

    def execute(self, d_terms, d_mat, d_y2, d_skipped, e_unit="CM-1"):
        """d_terms: device terms[t * nR + iR] (a CUDA tensor n_terms x nR, or a pointer);
        outputs P x nR (float64) and P (int32) device buffers."""
        eu = E_UNIT[e_unit.upper()] if isinstance(e_unit, str) else float(e_unit)
        p = [x.data_ptr() if hasattr(x, "data_ptr") else x for x in (d_terms, d_mat, d_y2, d_skipped)]
        check(lib().mqct_expansion_plan_execute(self.h, p[0], eu, p[1], p[2], p[3]))

    def sync(self):
        check(lib().mqct_expansion_plan_sync(self.h))

    def timing(self):
        """(angular set-up ms, last execute ms) on the device."""
        a, e = C.c_float(), C.c_float()
        check(lib().mqct_expansion_plan_timing(self.h, C.byref(a), C.byref(e)))
        return float(a.value), float(e.value)

    def close(self):
        if self.h:
            lib().mqct_expansion_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MatrixPlan:
    """Device-resident matrix build (mqct_matrix_plan_*); outputs in caller device buffers."""

    def __init__(self, system, R, grid, pes, precision=PREC_BF16X3, mij_cutoff=1e-12,
                 r_cut1=6.0, r_cut2=8.0):
        self.R = np.ascontiguousarray(R, np.float64)
        self.pes = pes if isinstance(pes, PesSpec) else PesSpec.from_dict(pes)
        self.system = system
        self._s = system.c_struct()
        self._g = _grid_struct(grid)
        self._p = self.pes.c_struct()
        self._ind = np.ascontiguousarray(system.ind_mat.reshape(-1))
        h = _abi.vp()
        check(lib().mqct_matrix_plan_create(C.byref(self._s), self._ind, system.P, self.R,
                                            len(self.R), C.byref(self._g), C.byref(self._p),
                                            precision, mij_cutoff, r_cut1, r_cut2, C.byref(h)))
        self.h = h
        self.flops = lib().mqct_matrix_plan_flops(h)

    def execute(self, d_mat: int, d_y2: int = 0, d_skipped: int = 0):
        check(lib().mqct_matrix_plan_execute(self.h, d_mat, d_y2 or None, d_skipped or None))

    def sync(self):
        check(lib().mqct_matrix_plan_sync(self.h))

    def set_surrogate(self, sur, rel_bound=1e-2, abs_bound_cm=0.5, n_check=64):
        """Evaluate the PES table with a trained Surrogate (None detaches)."""
        check(lib().mqct_matrix_plan_set_surrogate(self.h, None if sur is None else sur.h,
                                                   rel_bound, abs_bound_cm, n_check))
        self._sur = sur

    def set_drain(self, slices_per_drain):
        """Alpha points accumulated on the tensor cores between two FP64 drains."""
        check(lib().mqct_matrix_plan_set_drain(self.h, int(slices_per_drain)))

    def layout(self):
        """(alpha points per drain, grid-chunk ranges, radial column parts)."""
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().mqct_matrix_plan_layout(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return int(a.value), int(b.value), int(c.value)

    def tune(self, d_mat: int, d_y2: int = 0, d_skipped: int = 0):
        """Time the two epilogue layouts of the tensor-core contraction (four executes each
        into these device outputs, the minimum of the last three) and keep the faster
        (mqct_matrix_plan_tune)."""
        check(lib().mqct_matrix_plan_tune(self.h, d_mat, d_y2 or None, d_skipped or None))

    def set_epilogue(self, warps=0):
        """Force 8 or 16 epilogue warps for the following executes (0: the default rule)."""
        check(lib().mqct_matrix_plan_set_epilogue(self.h, int(warps)))

    def epilogue(self):
        """(epilogue warps of the next execute, contraction ms of the 8- and 16-warp layouts
        after tuning)."""
        w = C.c_int32()
        ms = (C.c_float * 2)()
        check(lib().mqct_matrix_plan_epilogue(self.h, C.byref(w), ms))
        return int(w.value), (float(ms[0]), float(ms[1]))

    def surrogate_stats(self):
        """(radial points re-evaluated exactly, largest checked residual ratio) of the
        last execute."""
        n = C.c_int32()
        r = C.c_double()
        check(lib().mqct_matrix_plan_surrogate_stats(self.h, C.byref(n), C.byref(r)))
        return int(n.value), float(r.value)

    def timing(self):
        """(basis+PES, contraction, finalize) milliseconds of the last execute."""
        t = (C.c_float * 3)()
        check(lib().mqct_matrix_plan_timing(self.h, t))
        return tuple(float(x) for x in t)

    def close(self):
        if self.h:
            lib().mqct_matrix_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spline_y2(R, mat):
    """Clamped cubic-spline second derivatives with finite-difference end slopes for
    every row of mat (READ_MIJ re-splines on read, MQCT_SOURCE_CODES/matrix_ini.f:5746-5753),
    the tridiagonal recurrence of MQCT_SOURCE_CODES/suppl_routines.f:914-965 vectorised
    over elements."""
    R = np.asarray(R, np.float64)
    Y = np.asarray(mat, np.float64)
    P, n = Y.shape
    y2 = np.zeros_like(Y)
    u = np.zeros_like(Y)
    yp1 = (Y[:, 1] - Y[:, 0]) / (R[1] - R[0])
    ypn = (Y[:, -1] - Y[:, -2]) / (R[-1] - R[-2])
    y2[:, 0] = -0.5
    u[:, 0] = (3.0 / (R[1] - R[0])) * ((Y[:, 1] - Y[:, 0]) / (R[1] - R[0]) - yp1)
    for i in range(1, n - 1):
        sig = (R[i] - R[i - 1]) / (R[i + 1] - R[i - 1])
        p = sig * y2[:, i - 1] + 2.0
        y2[:, i] = (sig - 1.0) / p
        u[:, i] = (6.0 * ((Y[:, i + 1] - Y[:, i]) / (R[i + 1] - R[i]) -
                          (Y[:, i] - Y[:, i - 1]) / (R[i] - R[i - 1])) / (R[i + 1] - R[i - 1]) -
                   sig * u[:, i - 1]) / p
    un = (3.0 / (R[-1] - R[-2])) * (ypn - (Y[:, -1] - Y[:, -2]) / (R[-1] - R[-2]))
    y2[:, -1] = (un - 0.5 * u[:, -2]) / (0.5 * y2[:, -2] + 1.0)
    for k in range(n - 2, -1, -1):
        y2[:, k] = y2[:, k] * y2[:, k + 1] + u[:, k]
    return y2


class PropagationTables:
    """Matrix tables as DOTRAJECT sees them: MIJ_SHIFT (M -= M(R_max), default on,
    MQCT_SOURCE_CODES/iotest.f:3754, :matrix_ini.f:5739-5743), MIJ_CUTOFF exclusion of
    elements below mij_cutoff cm^-1 at R~r_cut1 and r_cut2 (MQCT_SOURCE_CODES/matrix_ini.f:4288-4378)
    and re-splined knots."""

    def __init__(self, j12, m12, ej_hartree, ind_mat, R, mat, mass_amu, y2=None, mij_shift=True,
                 mij_cutoff=1e-12, r_cut1=6.0, r_cut2=8.0):
        R = np.ascontiguousarray(R, np.float64)
        mat = np.asarray(mat, np.float64)
        if mij_shift:
            mat = mat - mat[:, -1:]
        ir1 = int(np.argmin(np.abs(R - r_cut1)))
        ir2 = int(np.argmin(np.abs(R - r_cut2)))
        keep = np.maximum(np.abs(mat[:, ir1]), np.abs(mat[:, ir2])) >= mij_cutoff * CM_TO_HARTREE
        self.keep = keep
        self.mat = np.ascontiguousarray(mat[keep])
        self.y2 = np.ascontiguousarray(spline_y2(R, self.mat) if y2 is None else np.asarray(y2)[keep])
        self.ind_mat = np.ascontiguousarray(np.asarray(ind_mat, np.int32)[keep])
        self.R = R
        self.j12 = np.ascontiguousarray(j12, np.int32)
        self.m12 = np.ascontiguousarray(m12, np.int32)
        self.ej = np.ascontiguousarray(ej_hartree, np.float64)
        self.mass_au = float(mass_amu) * AMU_TO_AU
        self.n_states = len(self.j12)
        self.P = len(self.ind_mat)

    @staticmethod
    def from_system(system: CollisionSystem, R, mat, mass_amu, **kw):
        return PropagationTables(system.j12, system.m12, system.ej_cm * CM_TO_HARTREE,
                                 system.ind_mat, R, mat, mass_amu, **kw)

    def c_struct(self):
        self._ind_flat = np.ascontiguousarray(self.ind_mat.reshape(-1))
        return _abi.Tables(self.n_states, ptr(self.j12), ptr(self.m12), ptr(self.ej), self.P,
                           ptr(self._ind_flat), len(self.R), ptr(self.R), ptr(self.mat),
                           ptr(self.y2), self.mass_au)


@dataclass
class Trajectory:
    e_coll: float           # Hartree
    l_real: float
    s_st: int               # 1-based
    dt: float
    r_start: float
    r_fin: float
    numb_orb_prds: int = 1
    numb_oscl_prds: int = 1
    time_lim: float = 0.0
    max_steps: int = 2_000_000

    def c_struct(self):
        return _abi.TrajInit(self.e_coll, self.l_real, self.s_st, self.dt, self.r_start,
                             self.r_fin, self.numb_orb_prds, self.numb_oscl_prds, self.time_lim,
                             self.max_steps)


def trajectory_set(U_cm, b_max, mass_amu, s_st, time_step, rmax, j_max_ini=0, dl=1,
                   time_lim=0.0, max_steps=2_000_000):
    """Integer-l trajectory set of PROPAGATE (MQCT_SOURCE_CODES/propagator.f:419-495):
    k = sqrt(2 mu E), J_max = int(b_max k) - j_max, (L_MAX - L_MIN)/DL + 1 trajectories
    at the midpoints of their l bins, l = int((id - 1/2) DL + L_MIN) capped at L_MAX
    (TRAJ_ORB, MQCT_SOURCE_CODES/propagator.f:5163-5167, 5195-5198; for DL = 1,
    l = L_MIN, L_MIN + 1, ...); dt = TIME_STEP / sqrt(U / 300)
    (MQCT_SOURCE_CODES/propagator.f:2436)."""
    E = U_cm * CM_TO_HARTREE
    mu = mass_amu * AMU_TO_AU
    k = np.sqrt(mu * 2.0 * E)
    J_max = int(b_max * k) - j_max_ini
    L_max = J_max + j_max_ini
    L_min = max(0, 0 if J_max >= j_max_ini else j_max_ini - J_max)
    dt = time_step / np.sqrt(U_cm / 300.0)
    n_traj = (L_max - L_min) // dl + 1
    ls = [min(int((i - 0.5) * dl + L_min), L_max) for i in range(1, n_traj + 1)]
    trajs = [Trajectory(E, float(l), s_st, dt, rmax, rmax, time_lim=time_lim, max_steps=max_steps)
             for l in ls]
    return trajs, dict(k=k, J_down=0, J_up=J_max, L_min=L_min, E=E, dl=dl)


def _traj_array(trajs):
    arr = (_abi.TrajInit * len(trajs))(*[t.c_struct() for t in trajs])
    return arr


def _integrator(integrator):
    """None or "RK4": RK4 with the trajectories' dt; ("ODEINT", eps, hmin): the adaptive
    Cash-Karp scheme (PROPAGATOR = ODEINT) with accuracy eps and minimum step hmin;
    ("AT_ADAPT", tol, time_step): RK4 whose AT-mode steps follow AT_ADAPT_STP with
    AT_ADAPTOL = tol and the unscaled TIME_STEP as the smallest step; ("BK_INT", eps,
    hmin): ODEINT with bikram_int (one adaptive call with per-step stop rules)."""
    if integrator is None or (isinstance(integrator, str) and integrator.upper() == "RK4"):
        return None
    name, eps, hmin = integrator
    kind = {"ODEINT": _abi.INTEG_ODEINT, "AT_ADAPT": _abi.INTEG_AT_ADAPT,
            "BK_INT": _abi.INTEG_BK_INT}.get(name.upper())
    if kind is None:
        raise ValueError(f"unknown integrator {name!r}")
    return _abi.Integrator(kind, float(eps), float(hmin))


def propagate(tables: PropagationTables, trajs, arith=PROP_FP64, mode=MODE_STD, at_paths=None,
              integrator=None, coupled_states=False):
    """Batched DOTRAJECT on the GPU.  Returns (amp [n, 2N], cls [n, 6], diag [n, 8]).
    integrator: None (RK4) or ("ODEINT", eps, hmin); coupled_states: CS_APPROX = YES
    (no Coriolis coupling between m12 blocks, no Coriolis torque)."""
    n = len(trajs)
    N = tables.n_states
    amp = np.zeros(n * 2 * N)
    cls = np.zeros(n * 6)
    diag = np.zeros(n * 8)
    t = tables.c_struct()
    arr = _traj_array(trajs)
    at = None
    if mode & MODE_AT:
        recs = [np.ascontiguousarray(p, np.float64).reshape(-1, 8) for p in at_paths]
        n_rec = np.array([len(r) for r in recs], np.int32)
        off = np.concatenate([[0], np.cumsum(n_rec)[:-1]]).astype(np.int64)
        flat = np.ascontiguousarray(np.concatenate(recs).reshape(-1))
        at_keep = (n_rec, off, flat)
        at = _abi.AtPaths(ptr(off), ptr(n_rec), ptr(flat))
    integ = _integrator(integrator)
    if coupled_states:
        mode = mode | MODE_CS
    if integ is None:
        check(lib().mqct_propagate_batch(C.byref(t), arr, n, mode, C.byref(at) if at else None,
                                         arith, amp, cls, diag))
    else:
        check(lib().mqct_propagate_batch_integ(C.byref(t), arr, n, mode,
                                               C.byref(at) if at else None, arith,
                                               C.byref(integ), amp, cls, diag))
    return amp.reshape(n, 2 * N), cls.reshape(n, 6), diag.reshape(n, 8)


def propagate_record(tables: PropagationTables, trajs, arith=PROP_FP64, max_rec=1 << 15):
    """Standard-mode DOTRAJECT with SAVE_TRAJECT on the GPU: returns (amp, cls, diag,
    paths), paths[t] the (n x 8) records (t, R, P_R, theta, P_theta, phi, P_phi, pot)
    that an AT-MQCT run takes as at_paths."""
    n = len(trajs)
    N = tables.n_states
    amp = np.zeros(n * 2 * N)
    cls = np.zeros(n * 6)
    diag = np.zeros(n * 8)
    rec = np.zeros(n * max_rec * 8)
    n_rec = np.zeros(n, np.int64)
    t = tables.c_struct()
    check(lib().mqct_propagate_batch_rec(C.byref(t), _traj_array(trajs), n, arith, max_rec, amp,
                                         cls, diag, rec, n_rec))
    if (n_rec > max_rec).any():
        raise MqctError(-1, f"{int(n_rec.max())} records exceed max_rec={max_rec}")
    rec = rec.reshape(n, max_rec, 8)
    paths = [rec[i, :n_rec[i]].copy() for i in range(n)]
    return amp.reshape(n, 2 * N), cls.reshape(n, 6), diag.reshape(n, 8), paths


class PropagationPlan:
    """Tables uploaded once (mqct_prop_plan_*); run() per trajectory batch."""

    def __init__(self, tables: PropagationTables, arith=PROP_FP32):
        self.tables = tables
        self._t = tables.c_struct()
        h = _abi.vp()
        check(lib().mqct_prop_plan_create(C.byref(self._t), arith, C.byref(h)))
        self.h = h
        self.bytes_per_step = lib().mqct_prop_plan_bytes_per_step(h)

    def run(self, trajs):
        n = len(trajs)
        N = self.tables.n_states
        amp = np.zeros(n * 2 * N)
        cls = np.zeros(n * 6)
        diag = np.zeros(n * 8)
        check(lib().mqct_prop_plan_run(self.h, _traj_array(trajs), n, amp, cls, diag))
        return amp.reshape(n, 2 * N), cls.reshape(n, 6), diag.reshape(n, 8)

    def run_device(self, d_init: int, n: int, d_amp: int, d_cls: int, d_diag: int):
        check(lib().mqct_prop_plan_run_device(self.h, d_init, n, d_amp, d_cls, d_diag))

    def set_integrator(self, integrator=None):
        """None or "RK4" (default), or ("ODEINT", eps, hmin) for the following runs."""
        integ = _integrator(integrator) or _abi.Integrator(_abi.INTEG_RK4, 0.0, 0.0)
        check(lib().mqct_prop_plan_set_integrator(self.h, C.byref(integ)))

    def set_coupled_states(self, cs=True):
        """CS_APPROX for the following runs."""
        check(lib().mqct_prop_plan_set_coupled_states(self.h, 1 if cs else 0))

    def set_engine(self, engine=ENGINE_AUTO):
        """ENGINE_AUTO, ENGINE_PER_TRAJECTORY, ENGINE_LOCKSTEP, ENGINE_RESIDENT or
        ENGINE_LOCKSTEP_TAIL for the following runs (mqct_prop_plan_set_engine)."""
        check(lib().mqct_prop_plan_set_engine(self.h, int(engine)))

    def set_cluster(self, ctas=0):
        """Cluster size of the resident engine: 0 the smallest that fits, else 2..8
        (mqct_prop_plan_set_cluster)."""
        check(lib().mqct_prop_plan_set_cluster(self.h, int(ctas)))

    def cluster(self):
        """(CTAs per cluster, clusters resident on the device) of the resident engine for
        this plan's tables, (0, 0) where it does not apply (mqct_prop_plan_cluster)."""
        a, b = C.c_int32(), C.c_int32()
        check(lib().mqct_prop_plan_cluster(self.h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def handed(self):
        """Trajectories the last lockstep run handed to the resident engine
        (mqct_prop_plan_handed)."""
        n = C.c_int32()
        check(lib().mqct_prop_plan_handed(self.h, C.byref(n)))
        return int(n.value)

    def engine(self):
        """(engine of the last run, lockstep rounds of the last run or 0)."""
        e, r = C.c_int32(), C.c_int64()
        check(lib().mqct_prop_plan_engine(self.h, C.byref(e), C.byref(r)))
        return int(e.value), int(r.value)

    def tune(self, trajs, mode=MODE_STD):
        """Time the launch shapes on these trajectories (capped) and keep the faster."""
        arr = _traj_array(trajs)
        check(lib().mqct_prop_plan_tune(self.h, C.cast(arr, C.c_void_p), len(arr), mode))

    def shape(self):
        """(threads per CTA, CTAs per SM, probe ms of the 512x1 and 256x2 shapes)."""
        t, c = C.c_int32(), C.c_int32()
        ms = (C.c_float * 2)()
        check(lib().mqct_prop_plan_shape(self.h, C.byref(t), C.byref(c), ms))
        return int(t.value), int(c.value), (float(ms[0]), float(ms[1]))

    def sync(self):
        check(lib().mqct_prop_plan_sync(self.h))

    def timing(self):
        """Kernel milliseconds of the last run."""
        t = C.c_float()
        check(lib().mqct_prop_plan_timing(self.h, C.byref(t)))
        return float(t.value)

    def close(self):
        if self.h:
            lib().mqct_prop_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def channel_probabilities(amp, indx_chann, n_channels):
    """probab(channel) = sum of |a|^2 over the channel's states
    (MQCT_SOURCE_CODES/propagator.f:4364-4380)."""
    N = len(indx_chann)
    p = amp[:, :N] ** 2 + amp[:, N:] ** 2
    out = np.zeros((amp.shape[0], n_channels))
    for c in range(n_channels):
        out[:, c] = p[:, indx_chann == c + 1].sum(axis=1)
    return out


def cross_sections(prob, j_ini, J_down, J_up, L_min, k_vec, U_cm=None, e_ch=None, chann_ini=1,
                   dl=1):
    """INELAST_CALC (MQCT_SOURCE_CODES/propagator.f:4776-4841):
    sigma_f = pi/k^2 sum_J sum_{l=|J-j|}^{J+j} (2J+1)/(2j+1) P_f(traj(l)), in Angstrom^2
    (sigma(U) column of CROSS_SECTIONS.out), traj(l) = (l - L_MIN) / DL the trajectory of
    l's bin (TRAJ_ORB, MQCT_SOURCE_CODES/propagator.f:5127-5134).  With U_cm and e_ch also
    returns the Billing-corrected sigma(E_coll) (MQCT_SOURCE_CODES/propagator.f:1207-1208,
    276-286)."""
    n_traj, nch = prob.shape
    sig = np.zeros(nch)
    for J in range(J_down, J_up + 1):
        for l in range(abs(J - j_ini), J + j_ini + 1):
            i = (l - L_min) // dl
            if 0 <= i < n_traj:
                sig += prob[i] * (2.0 * J + 1.0) / k_vec ** 2 / (2.0 * j_ini + 1) * np.pi
    sig_U = sig * A_BOHR ** 2
    if U_cm is None:
        return sig_U
    dE = np.asarray(e_ch) - e_ch[chann_ini - 1]
    e_bill = U_cm + dE / 2.0 + dE ** 2 / 16.0 / U_cm
    return sig_U, sig_U * U_cm / e_bill, e_bill


def deflection_angles(cls, trajs, mass_au):
    """Deflection angle of each trajectory (rad), the DEFLCT_ANGLE column of
    DEFLECTION_FUNCTION.out (MQCT_SOURCE_CODES/propagator.f:3260-3294, 4485): the angle
    from the final to the initial velocity, signed by the z component of
    v_final x v_initial, its windings past -pi counted (the reference's loop count); pi for
    l = 0 (head-on).  cls: the final classical variables (R, P_R, theta, P_theta, phi, P_phi)
    as the propagation returns them; trajs: the initial conditions (e_coll, l_real,
    r_start).  The motion stays in the plane theta = pi/2, so the velocity's direction
    angle is phi + atan2(v_phi, v_R) with v_phi = P_phi / (m R sin theta) > 0, a continuous
    function of time: its change over the trajectory is the reference's step-by-step
    angle with its loops.  The reference evaluates it at the start of its last loop pass
    (one step before the final state); the difference is below its printed digits."""
    cls = np.asarray(cls, dtype=np.float64)
    out = np.empty(len(trajs))
    for i, t in enumerate(trajs):
        if t.l_real == 0.0:
            out[i] = np.pi
            continue
        k = np.sqrt(2.0 * mass_au * t.e_coll)
        lo = np.sqrt(t.l_real * (t.l_real + 1.0))
        pr0 = -np.sqrt(k * k - lo * lo / (t.r_start * t.r_start))
        psi0 = np.arctan2(lo / (mass_au * t.r_start), pr0 / mass_au)
        R, PR, th, _, phi, Pphi = cls[i]
        psi = phi + np.arctan2(Pphi / (mass_au * R * np.sin(th)), PR / mass_au)
        out[i] = psi0 - psi
    return out


def scattering_phases(l, deflection):
    """Scattering phase of each trajectory (rad), the SCAT_PHASE column of
    DEFLECTION_FUNCTION.out (ELAST_CALC, MQCT_SOURCE_CODES/propagator.f:5694-5715): zero for
    the last trajectory, then backwards phase_i = phase_{i+1} - (chi_i + chi_{i+1}) / 2
    |l_{i+1} - l_i| (trapezoid over the deflection function)."""
    l = np.asarray(l, dtype=np.float64)
    chi = np.asarray(deflection, dtype=np.float64)
    ph = np.zeros(len(chi))
    for i in range(len(chi) - 2, -1, -1):
        ph[i] = ph[i + 1] - (chi[i] + chi[i + 1]) / 2.0 * abs(l[i + 1] - l[i])
    return ph


def elastic_cross_section(l, p_elastic, phase, k_vec, weight=None):
    """Elastic cross section (Angstrom^2), the elastic row of CROSS_SECTIONS.out without
    DIFF_CROSS (ELAST_CALC, MQCT_SOURCE_CODES/propagator.f:5717-5749):
    sigma_el = pi / k^2 sum_i w_i |1 - sqrt(P_el,i) e^{i phase_i}|^2 (2 l_i + 1) |l_{i+1} - l_i|
    over all trajectories but the last; weight: the identical-particle parity weights w_i
    (1 when None)."""
    l = np.asarray(l, dtype=np.float64)
    p = np.asarray(p_elastic, dtype=np.float64)
    ph = np.asarray(phase, dtype=np.float64)
    w = np.ones(len(l)) if weight is None else np.asarray(weight, dtype=np.float64)
    s = 0.0
    for i in range(len(l) - 1):
        amp = 1.0 - np.sqrt(p[i]) * np.exp(1j * ph[i])
        s += w[i] * abs(amp) ** 2 / k_vec ** 2 * np.pi * (2.0 * l[i] + 1.0) * abs(l[i + 1] - l[i])
    return s * A_BOHR ** 2


def differential_cross_section(p_elastic, phase, j_ini, J_down, J_up, L_min, k_vec, n_angles,
                               dl=1):
    """Elastic differential cross section (DIFF_CROSS = YES; ELAST_CALC,
    MQCT_SOURCE_CODES/propagator.f:5755-5830): on the angles theta_k = (k - 1) pi /
    (n_angles - 1),
    f(theta) = i / (2 k (2j + 1)) sum_J (2J + 1) sum_{l=|J-j|}^{J+j} P_l(cos theta)
               (1 - sqrt(P_el(traj(l))) e^{i phase(traj(l))}),
    dsigma/dOmega = |f|^2 (Angstrom^2, the DIFF_CROSS.out column), and the elastic cross
    section 2 pi int dsigma/dOmega sin theta dtheta by the trapezoid rule over the angles,
    which replaces the one above in CROSS_SECTIONS.out.  traj(l) = (l - L_min) / dl as in
    INELAST_CALC.  Returns (theta in rad, dsigma/dOmega, sigma_el).  The reference's
    trapezoid sum starts at k = 1 and so reads the elements before its arrays; it starts at
    the second angle here."""
    p = np.asarray(p_elastic, dtype=np.float64)
    ph = np.asarray(phase, dtype=np.float64)
    n_traj = len(p)
    theta = np.arange(n_angles) * np.pi / (n_angles - 1)
    x = np.cos(theta)
    lmax = J_up + j_ini
    # Legendre polynomials P_l(x) by the three-term recurrence
    P = np.zeros((lmax + 1, n_angles))
    P[0] = 1.0
    if lmax >= 1:
        P[1] = x
    for n in range(2, lmax + 1):
        P[n] = ((2 * n - 1) * x * P[n - 1] - (n - 1) * P[n - 2]) / n
    f = np.zeros(n_angles, dtype=np.complex128)
    for J in range(J_down, J_up + 1):
        for lv in range(abs(J - j_ini), J + j_ini + 1):
            i = (lv - L_min) // dl
            if 0 <= i < n_traj:
                f += (P[lv] * (1.0 - np.sqrt(p[i]) * np.exp(1j * ph[i])) * (2.0 * J + 1.0)
                      * 1j / k_vec / 2.0 / (2.0 * j_ini + 1.0))
    dcs = np.abs(f) ** 2
    sig = float(np.sum((dcs[:-1] * np.sin(theta[:-1]) + dcs[1:] * np.sin(theta[1:]))
                       * np.pi * np.diff(theta)))
    return theta, dcs * A_BOHR ** 2, sig * A_BOHR ** 2


def _clamped_spline(x, y):
    """Second derivatives of the cubic spline through (x, y) with the end slopes of the
    first and last chords (the tridiagonal recurrence of Numerical Recipes' `spline`, as
    the reference calls it with finite-difference end slopes)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = len(x)
    yp1 = (y[1] - y[0]) / (x[1] - x[0])
    ypn = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2])
    y2, u = np.zeros(n), np.zeros(n)
    y2[0] = -0.5
    u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1)
    for i in range(1, n - 1):
        sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1])
        p = sig * y2[i - 1] + 2.0
        y2[i] = (sig - 1.0) / p
        u[i] = (6.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]))
                / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p
    un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]))
    y2[n - 1] = (un - 0.5 * u[n - 2]) / (0.5 * y2[n - 2] + 1.0)
    for k in range(n - 2, -1, -1):
        y2[k] = y2[k] * y2[k + 1] + u[k]
    return y2


def _splint(x, y, y2, v):
    """The spline at v (bisection for the interval; outside the knots the end interval's
    cubic)."""
    klo, khi = 0, len(x) - 1
    while khi - klo > 1:
        k = (khi + klo) // 2
        if x[k] > v:
            khi = k
        else:
            klo = k
    h = x[khi] - x[klo]
    a, b = (x[khi] - v) / h, (v - x[klo]) / h
    return a * y[klo] + b * y[khi] + ((a ** 3 - a) * y2[klo] + (b ** 3 - b) * y2[khi]) * h * h / 6.0


def cross_sections_spline(prob, l_traj, j_ini, J_down, J_up, k_vec):
    """INELAST_CALC with PROB_SPLINE = YES (MQCT_SOURCE_CODES/propagator.f:4889-4975): the
    channel probabilities of the trajectories (run at l_traj, e.g. every DL-th l) are
    splined over l (clamped, chord end slopes) and the J sums take the spline at every
    integer l: sigma_f = pi/k^2 sum_J sum_{l=|J-j|}^{J+j} (2J+1)/(2j+1) P_f(l), Angstrom^2."""
    prob = np.asarray(prob, dtype=np.float64)
    lt = np.asarray(l_traj, dtype=np.float64)
    sig = np.zeros(prob.shape[1])
    for c in range(prob.shape[1]):
        y2 = _clamped_spline(lt, prob[:, c])
        for J in range(J_down, J_up + 1):
            for lv in range(abs(J - j_ini), J + j_ini + 1):
                sig[c] += (_splint(lt, prob[:, c], y2, float(lv)) * (2.0 * J + 1.0) / k_vec ** 2
                           / (2.0 * j_ini + 1) * np.pi)
    return sig * A_BOHR ** 2


def elastic_cross_section_spline(l_traj, p_elastic, deflection, L_min, L_max, k_vec):
    """ELAST_CALC with PROB_SPLINE = YES (MQCT_SOURCE_CODES/propagator.f:5960-6060): the
    deflection function and log10 of the elastic probability (floored at 1e-30) of the
    trajectories at l_traj are splined over l; the phases run backwards on the integer
    grid, phase(L_max) = 0, phase(l) = phase(l + 1) - (chi(l) + chi(l + 1)) / 2, and
    sigma_el = pi/k^2 sum_{l=L_min}^{L_max-1} |1 - sqrt(P_el(l)) e^{i phase(l)}|^2 (2l + 1).
    Returns (sigma_el in Angstrom^2, phases at l = L_min..L_max)."""
    lt = np.asarray(l_traj, dtype=np.float64)
    chi = np.asarray(deflection, dtype=np.float64)
    lp = np.log10(np.maximum(np.asarray(p_elastic, dtype=np.float64), 1e-30))
    y2c, y2p = _clamped_spline(lt, chi), _clamped_spline(lt, lp)
    ph = np.zeros(L_max - L_min + 1)
    s = 0.0
    for lv in range(L_max - 1, L_min - 1, -1):
        c1 = _splint(lt, chi, y2c, float(lv))
        c2 = _splint(lt, chi, y2c, float(lv + 1))
        i = lv - L_min
        ph[i] = ph[i + 1] - (c1 + c2) / 2.0
        p = 10.0 ** _splint(lt, lp, y2p, float(lv))
        s += abs(1.0 - np.sqrt(p) * np.exp(1j * ph[i])) ** 2 / k_vec ** 2 * np.pi * (2.0 * lv + 1)
    return s * A_BOHR ** 2, ph


def splined_opacity(l_traj, prob, deflection, L_min, L_max, log_space=True):
    """The deflection function and channel probabilities splined to every integer l from
    L_min to L_max, as SPLINED_DEFLECTION_OPACITY_L.out lists them
    (MQCT_SOURCE_CODES/propagator.f:6080-6110): probabilities splined in log10 space
    (floored at 1e-30) as the reference does now, or linearly (log_space=False) as its
    earlier INTERPOLATED_PROBS_DEFLECTION_L.out did.  Returns (l, chi, prob [n_l, n_ch])."""
    lt = np.asarray(l_traj, dtype=np.float64)
    prob = np.asarray(prob, dtype=np.float64)
    chi = np.asarray(deflection, dtype=np.float64)
    ls = np.arange(L_min, L_max + 1)
    y2c = _clamped_spline(lt, chi)
    out_chi = np.array([_splint(lt, chi, y2c, float(v)) for v in ls])
    out_p = np.zeros((len(ls), prob.shape[1]))
    for c in range(prob.shape[1]):
        y = np.log10(np.maximum(prob[:, c], 1e-30)) if log_space else prob[:, c]
        y2 = _clamped_spline(lt, y)
        v = np.array([_splint(lt, y, y2, float(q)) for q in ls])
        out_p[:, c] = 10.0 ** v if log_space else v
    return ls, out_chi, out_p


def cross_sections_device(d_amp, system: CollisionSystem, j_ini, J_down, J_up, L_min, k_vec,
                          dl=1):
    """INELAST_CALC on the GPU from device amplitudes (a CUDA float64 torch tensor, n_traj x
    2N, as propagate returns them): returns CUDA tensors (prob [n_traj, n_channels],
    partial [J_up - J_down + 1, n_channels], sigma [n_channels]), cross sections in
    Angstrom^2, computed on torch's current stream."""
    import torch
    amp = d_amp.contiguous()
    if amp.dtype != torch.float64 or not amp.is_cuda or amp.shape[1] != 2 * system.n_states:
        raise ValueError("d_amp must be a CUDA float64 tensor of shape (n_traj, 2 n_states)")
    n_traj, nch = amp.shape[0], system.n_channels
    prob = torch.empty((n_traj, nch), dtype=torch.float64, device=amp.device)
    partial = torch.empty((J_up - J_down + 1, nch), dtype=torch.float64, device=amp.device)
    sigma = torch.empty(nch, dtype=torch.float64, device=amp.device)
    stream = torch.cuda.current_stream(amp.device).cuda_stream
    check(lib().mqct_cross_sections_device(amp.data_ptr(), n_traj, system.n_states,
                                           np.ascontiguousarray(system.indx_chann, np.int32), nch,
                                           j_ini, J_down, J_up, L_min, dl, k_vec,
                                           prob.data_ptr(), partial.data_ptr(), sigma.data_ptr(),
                                           stream))
    return prob, partial, sigma


def write_mtrx_uf(path, system: CollisionSystem, R, mat):
    rec = system.state_records()
    check(lib().mqct_write_mtrx_uf(path.encode(), system.sys_type, system.n_channels,
                                   system.n_states, np.ascontiguousarray(rec.reshape(-1)),
                                   rec.shape[1], system.P,
                                   np.ascontiguousarray(system.ind_mat.reshape(-1)), len(R),
                                   np.ascontiguousarray(R, np.float64),
                                   np.ascontiguousarray(mat, np.float64).reshape(-1)))


def read_mtrx_uf(path):
    L = lib()
    ct, nch, ns, nR, srl = (C.c_int32() for _ in range(5))
    P = C.c_int64()
    check(L.mqct_read_mtrx_uf_header(path.encode(), C.byref(ct), C.byref(nch), C.byref(ns),
                                     C.byref(P), C.byref(nR), C.byref(srl)))
    st = np.zeros(ns.value * srl.value, np.int32)
    ind = np.zeros(2 * P.value, np.int32)
    R = np.zeros(nR.value)
    mat = np.zeros(P.value * nR.value)
    check(L.mqct_read_mtrx_uf(path.encode(), srl.value, st, ind, R, mat))
    return dict(coll_type=ct.value, n_channels=nch.value, states=st.reshape(ns.value, srl.value),
                ind_mat=ind.reshape(P.value, 2), R=R, mat=mat.reshape(P.value, nR.value))


def write_mtrx_dat(path, system: CollisionSystem, R, mat):
    """Formatted MTRX.DAT as PRINT_MIJ writes it (MQCT_SOURCE_CODES/matrix_ini.f:4692-4877)."""
    rec = system.state_records()
    check(lib().mqct_write_mtrx_dat(path.encode(), system.sys_type, system.n_channels,
                                    system.n_states, np.ascontiguousarray(rec.reshape(-1)),
                                    rec.shape[1], system.P,
                                    np.ascontiguousarray(system.ind_mat.reshape(-1)), len(R),
                                    np.ascontiguousarray(R, np.float64),
                                    np.ascontiguousarray(mat, np.float64).reshape(-1)))


def read_mtrx_dat(path):
    """Formatted MTRX.DAT (READ_MTRX with UNFORMAT = NO): coll_type, n_channels, the state
    table, ind_mat, R and Mat_el (P x nR)."""
    L = lib()
    ct, nch, ns, nR, srl = (C.c_int32() for _ in range(5))
    P = C.c_int64()
    check(L.mqct_read_mtrx_dat_header(path.encode(), C.byref(ct), C.byref(nch), C.byref(ns),
                                      C.byref(P), C.byref(nR), C.byref(srl)))
    st = np.zeros(ns.value * srl.value, np.int32)
    ind = np.zeros(2 * P.value, np.int32)
    R = np.zeros(nR.value)
    mat = np.zeros(P.value * nR.value)
    check(L.mqct_read_mtrx_dat(path.encode(), srl.value, st, ind, R, mat))
    return dict(coll_type=ct.value, n_channels=nch.value, states=st.reshape(ns.value, srl.value),
                ind_mat=ind.reshape(P.value, 2), R=R, mat=mat.reshape(P.value, nR.value))


def read_expansion_terms(path, nR, n_terms):
    """PES_EXPAN_TERMS.DAT (READ_EXPANSION_TERMS): returns R (nR) and the terms as the
    file's rows (nR x n_terms), ready for build_matrix_expansion."""
    R = np.zeros(nR)
    T = np.zeros(nR * n_terms)
    check(lib().mqct_read_expansion_terms(path.encode(), nR, n_terms, R, T))
    return R, np.ascontiguousarray(T.reshape(n_terms, nR).T)


def write_expansion_terms(path, sys_type, labels, R, terms):
    """Append R and the terms (nR x n_terms, the rows of the file) to PES_EXPAN_TERMS.DAT
    as CALC_EXPANSION_TERMS writes it, the header first when the file holds at most one
    line."""
    a_top = _a_top(labels)
    R = np.ascontiguousarray(R, np.float64)
    T = np.ascontiguousarray(np.asarray(terms, np.float64).reshape(len(R), len(a_top)).T)
    check(lib().mqct_write_expansion_terms(path.encode(), int(sys_type), len(a_top),
                                           a_top.reshape(-1), len(R), R, T.reshape(-1)))


def _a_top(labels):
    lab = np.asarray(labels, np.int32)
    lab = lab.reshape(len(lab), -1)
    a_top = np.zeros((len(lab), 5), np.int32)  # A_TOP(5, nterms)
    a_top[:, :lab.shape[1]] = lab
    return a_top


def _projection_grid(V, sys_type, eq_gamma):
    if sys_type in (1, 3, 4):
        if V.ndim != (2 if sys_type == 1 else 3):
            raise ValueError("V must be (nR, n_beta) for SYS_TYPE 1, (nR, n_beta, n_gamma) for 4")
        return _abi.Grid(V.shape[1], V.shape[2] if sys_type != 1 else 0, 0, 0, 0, 0,
                         1 if eq_gamma else 0)
    nR, n2, n3, n4, n5 = V.shape[:5]
    n6 = V.shape[5] if sys_type in (0, 9) else 0
    if sys_type in (0, 9) and V.ndim != 6 or sys_type not in (0, 9) and V.ndim != 5:
        raise ValueError("V must be (nR, n_alpha2, n_beta1, n_beta2, n_gamma1[, n_gamma2])")
    return _abi.Grid(n3, n5, 0, n4, n2, n6, 1 if eq_gamma else 0)


def project_terms(sys_type, labels, V, eq_gamma=True, identical=False):
    """CALC_EXPANSION_TERMS on the GPU: project V, tabulated on the angular grid as
    (nR, n_beta) for SYS_TYPE 1, (nR, n_beta, n_gamma) for 4, (nR, n_alpha2, n_beta1,
    n_beta2, n_gamma1) for 7 and 8 or with a trailing n_gamma2 axis for 0, onto the terms
    (rows (l,), (l, nju), (l1, nju1, l2, l) or (l1, nju1, l2, nju2, l)).  Returns (terms, terms_im), nR x n_terms each, the rows of
    PES_EXPAN_TERMS.DAT in the unit of V."""
    a_top = _a_top(labels)
    V = np.ascontiguousarray(V, np.float64)
    g = _projection_grid(V, sys_type, eq_gamma)
    nR, nt = V.shape[0], len(a_top)
    T = np.zeros(nt * nR)
    Ti = np.zeros(nt * nR)
    check(lib().mqct_project_terms(int(sys_type), nt, a_top.reshape(-1), C.byref(g),
                                   1 if identical else 0, nR, V.reshape(-1), T,
                                   Ti.ctypes.data))
    return T.reshape(nt, nR).T.copy(), Ti.reshape(nt, nR).T.copy()


class ProjectionPlan:
    """CALC_EXPANSION_TERMS with the per-term tables formed once (mqct_projection_plan_*);
    execute() projects V on the device into device terms[t * nR + iR] (the layout that
    ExpansionPlan.execute takes)."""

    def __init__(self, sys_type, labels, grid_shape, eq_gamma=True, identical=False):
        """grid_shape: (n_beta,) for SYS_TYPE 1, (n_beta, n_gamma) for 3 and 4, (n_alpha2,
        n_beta1, n_beta2, n_gamma1[, n_gamma2]) for 7, 8 and 0."""
        a_top = _a_top(labels)
        self.n_terms = len(a_top)
        if sys_type in (1, 3, 4):
            gs = tuple(grid_shape) + (0,)
            self.grid = _abi.Grid(gs[0], gs[1] if sys_type != 1 else 0, 0, 0, 0, 0,
                                  1 if eq_gamma else 0)
        else:
            gs = tuple(grid_shape) + ((0,) if len(grid_shape) == 4 else ())
            self.grid = _abi.Grid(gs[1], gs[3], 0, gs[2], gs[0], gs[4], 1 if eq_gamma else 0)
        h = _abi.vp()
        check(lib().mqct_projection_plan_create(int(sys_type), self.n_terms, a_top.reshape(-1),
                                                C.byref(self.grid), 1 if identical else 0,
                                                C.byref(h)))
        self.h = h

    def execute(self, d_V, nR, d_terms, d_terms_im=None):
        p = [x.data_ptr() if hasattr(x, "data_ptr") else x for x in (d_V, d_terms, d_terms_im)]
        check(lib().mqct_projection_plan_execute(self.h, p[0], int(nR), p[1], p[2]))

    def sync(self):
        check(lib().mqct_projection_plan_sync(self.h))

    def timing(self):
        """(gamma, alpha2, beta contraction ms) of the last execute, on the device."""
        a, b, c = C.c_float(), C.c_float(), C.c_float()
        check(lib().mqct_projection_plan_timing(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return float(a.value), float(b.value), float(c.value)

    def close(self):
        if self.h:
            lib().mqct_projection_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_opacity(path, s_st, j12, m12, i_ener, U_cm, l, k_vec, prob, path_total=None,
                  chann_ini=1):
    """Append one block to OPACITY_FUNCTIONS_L.out (and TOTAL_PROBABILITIES_L.out when
    path_total is given): prob is n_traj x n_channels, l the trajectories' l."""
    prob = np.ascontiguousarray(prob, np.float64)
    li = np.ascontiguousarray(l, np.int32)
    check(lib().mqct_write_opacity(path.encode(), path_total.encode() if path_total else None,
                                   int(s_st), int(j12), int(m12), int(i_ener), float(U_cm),
                                   len(li), li, float(k_vec), prob.shape[1], prob.reshape(-1),
                                   int(chann_ini)))


def write_deflection(path, s_st, j12, m12, i_ener, U_cm, l, k_vec, deflection, phase,
                     finish_time, e_err_pct, p_err_pct, periods, oscillations):
    """Append one block to DEFLECTION_FUNCTION.out (per trajectory: l, l / k, deflection
    angle and scattering phase in rad, finish time in a.u., energy and norm errors in
    percent, orbiting periods, oscillations of R)."""
    f64 = lambda a: np.ascontiguousarray(a, np.float64)  # noqa: E731
    li = np.ascontiguousarray(l, np.int32)
    check(lib().mqct_write_deflection(path.encode(), int(s_st), int(j12), int(m12), int(i_ener),
                                      float(U_cm), len(li), li, float(k_vec), f64(deflection),
                                      f64(phase), f64(finish_time), f64(e_err_pct),
                                      f64(p_err_pct), np.ascontiguousarray(periods, np.int32),
                                      np.ascontiguousarray(oscillations, np.int32)))


def write_diff_cross(path, i_ener, s_st, j12, m12, theta, dcs):
    """Append one block to DIFF_CROSS.out (theta in rad, written in degrees; dsigma/dOmega
    in Angstrom^2)."""
    th = np.ascontiguousarray(theta, np.float64)
    check(lib().mqct_write_diff_cross(path.encode(), int(i_ener), int(s_st), int(j12), int(m12),
                                      len(th), th, np.ascontiguousarray(dcs, np.float64)))


def write_splined_opacity(path, l, k_vec, deflection, prob):
    """Append the SPLINED_DEFLECTION_OPACITY_L.out table (per integer l: l / k, l, the splined
    deflection function, the splined channel probabilities prob [n_l, n_channels])."""
    li = np.ascontiguousarray(l, np.int32)
    prob = np.ascontiguousarray(prob, np.float64)
    check(lib().mqct_write_splined_opacity(path.encode(), len(li), li, float(k_vec),
                                           np.ascontiguousarray(deflection, np.float64),
                                           prob.shape[1], prob.reshape(-1)))


def write_partial_j(path, s_st, j12, m12, i_ener, U_cm, J, partial):
    """Append one block to PARTIAL_CROSS_SECTIONS_J.out (partial: n_J x n_channels, A^2)."""
    partial = np.ascontiguousarray(partial, np.float64)
    Ji = np.ascontiguousarray(J, np.int32)
    check(lib().mqct_write_partial_j(path.encode(), int(s_st), int(j12), int(m12), int(i_ener),
                                     float(U_cm), len(Ji), Ji, partial.shape[1],
                                     partial.reshape(-1)))


def write_m_proj(path, s_st, i_ener, j12, m12, sigma):
    """Append one block to M_PROJ_CROSSECTIONS.out (sigma per channel, A^2)."""
    sigma = np.ascontiguousarray(sigma, np.float64)
    check(lib().mqct_write_m_proj(path.encode(), int(s_st), int(i_ener), int(j12), int(m12),
                                  len(sigma), sigma))


def write_cross_sections(path, U_cm, chann_ini, sigma_f, E_bill, p_err_pct, e_err_pct=None,
                         exists=None):
    """Append one energy block to CROSS_SECTIONS.out."""
    sigma_f = np.ascontiguousarray(sigma_f, np.float64)
    E_bill = np.ascontiguousarray(E_bill, np.float64)
    ex = None if exists is None else np.ascontiguousarray(exists, np.int32)
    check(lib().mqct_write_cross_sections(path.encode(), float(U_cm), int(chann_ini),
                                          len(sigma_f), None if ex is None else ex.ctypes.data,
                                          sigma_f, E_bill, float(p_err_pct),
                                          0 if e_err_pct is None else 1,
                                          0.0 if e_err_pct is None else float(e_err_pct)))


def write_cross_sections_footer(path, n_traj_total):
    check(lib().mqct_write_cross_sections_footer(path.encode(), int(n_traj_total)))

