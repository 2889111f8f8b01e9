"""ctypes binding of the CPU parity checkers.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module; the product never does.

* :class:`OracleSim` wraps ``_build/libfnoracle.so`` (fibre_oracle.c, the C
  restatement of kernel.cl and RunSimulationLoop) in REF or MIRROR mode.
* :class:`RefSim` wraps ``_ref/libfnref.so``, the reference's own kernel.cl
  compiled as C (present where the reference tree was available at build
  time; it travels to the GPU box as a built file).

Both take any object with the attributes of ``fibrenet_b200.model.Model``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libfnoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfnref.so")
REF_SRC_ENV = "FIBRENET_REF_SRC"  # the reference's FibreNet folder (holding kernel.cl)

MODE_REF = 0
MODE_MIRROR = 1

FIELD = {"pos": 0, "img": 1, "vel": 2, "force": 3, "vel_old": 4, "force_old": 5}

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class FoModel(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("lam", C.c_double), ("damping", C.c_double),
        ("gravity", C.c_double * 3), ("cutoff", C.c_double), ("box_unit_cell", C.c_double),
        ("box", C.c_double * 3), ("wall_k", C.c_double), ("bc_type", C.c_int),
        ("grid_update_freq", C.c_int), ("skin_ratio", C.c_double), ("n_types", C.c_int),
        ("pair_kind", _I), ("pair_raw", _D),
        ("n_beads", C.c_int), ("type", _I), ("tag", _I), ("loc_id", _I), ("radius", _D),
        ("mass", _D), ("pos", _D), ("vel", _D), ("vel_old", _D), ("force", _D), ("img", _D),
        ("n_springs", C.c_int), ("s_type", _I), ("s_tag", _I), ("s_p1", _I), ("s_p2", _I),
        ("s_rest", _D), ("s_k", _D), ("s_c1", _D), ("s_c2", _D),
        ("n_angles", C.c_int), ("a_type", _I), ("a_b1", _I), ("a_b2", _I), ("a_b3", _I),
        ("a_s1", _I), ("a_s2", _I), ("a_theta0", _D), ("a_k", _D),
        ("periodic_mask", C.c_int),
    ]


def build(ref_src: str | None = None, quiet: bool = True) -> None:
    """Builds the restatement (always) and the reference copy when the
    reference's FibreNet folder is given (``ref_src`` or the FIBRENET_REF_SRC
    environment variable); without it an already built copy is kept."""
    env = dict(os.environ)
    targets = ["oracle"]
    src = ref_src or os.environ.get(REF_SRC_ENV)
    if src:
        if not os.path.isfile(os.path.join(src, "kernel.cl")):
            raise RuntimeError(f"{REF_SRC_ENV}={src}: no kernel.cl there (give the reference's "
                               "FibreNet folder)")
        targets.append("ref")
        env["REF_SRC"] = src
    out = subprocess.run(["make", "-C", HERE, *targets], env=env, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


def ref_available() -> bool:
    return os.path.isfile(REF_SO)


class _Holder:
    """Keeps the numpy buffers alive while a FoModel points into them."""


def make_fo_model(m) -> tuple[FoModel, _Holder]:
    h = _Holder()
    s = m.settings

    def d(name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        setattr(h, name, a)
        return a.ctypes.data_as(_D)

    def i(name, arr):
        a = np.ascontiguousarray(arr, dtype=np.int32).ravel()
        setattr(h, name, a)
        return a.ctypes.data_as(_I)

    fm = FoModel()
    fm.dt, fm.lam, fm.damping = s.dt, s.lam, s.damping
    fm.gravity = (C.c_double * 3)(*s.gravity)
    fm.cutoff, fm.box_unit_cell = s.cutoff, s.box_unit_cell
    fm.box = (C.c_double * 3)(*s.box)
    fm.wall_k, fm.bc_type = s.wall_k, s.bc_type
    fm.grid_update_freq, fm.skin_ratio = s.grid_update_freq, s.skin_ratio
    fm.n_types = len(m.type_names)
    fm.pair_kind = i("pair_kind", m.pair_kind)
    fm.pair_raw = d("pair_raw", m.pair_raw)
    fm.n_beads = int(len(m.type))
    fm.type, fm.tag, fm.loc_id = i("type", m.type), i("tag", m.tag), i("loc_id", m.loc_id)
    fm.radius, fm.mass = d("radius", m.radius), d("mass", m.mass)
    fm.pos, fm.vel, fm.vel_old = d("pos", m.pos), d("vel", m.vel), d("vel_old", m.vel_old)
    fm.force, fm.img = d("force", m.force), d("img", m.img)
    fm.n_springs = int(len(m.s_type))
    fm.s_type, fm.s_tag = i("s_type", m.s_type), i("s_tag", m.s_tag)
    fm.s_p1, fm.s_p2 = i("s_p1", m.s_p1), i("s_p2", m.s_p2)
    fm.s_rest, fm.s_k = d("s_rest", m.s_rest), d("s_k", m.s_k)
    fm.s_c1, fm.s_c2 = d("s_c1", m.s_c1), d("s_c2", m.s_c2)
    fm.n_angles = int(len(m.a_type))
    fm.a_type = i("a_type", m.a_type)
    fm.a_b1, fm.a_b2, fm.a_b3 = i("a_b1", m.a_b1), i("a_b2", m.a_b2), i("a_b3", m.a_b3)
    fm.a_s1, fm.a_s2 = i("a_s1", m.a_s1), i("a_s2", m.a_s2)
    fm.a_theta0, fm.a_k = d("a_theta0", m.a_theta0), d("a_k", m.a_k)
    fm.periodic_mask = int(s.periodic_mask)
    return fm, h


_oracle_lib = None
_ref_lib = None


def _load_oracle():
    global _oracle_lib
    if _oracle_lib is None:
        if not os.path.isfile(ORACLE_SO):
            build()
        lib = C.CDLL(ORACLE_SO)
        lib.fo_create.restype = _P
        lib.fo_create.argtypes = [C.POINTER(FoModel), C.c_int, C.c_int, C.c_int]
        lib.fo_destroy.argtypes = [_P]
        lib.fo_run.argtypes = [_P, C.c_int]
        lib.fo_run.restype = C.c_int
        lib.fo_rebuild.argtypes = [_P]
        lib.fo_reset_energy.argtypes = [_P]
        lib.fo_forces_only.argtypes = [_P, C.c_int, C.c_int, C.c_int]
        lib.fo_get_beads.argtypes = [_P, C.c_int, _D]
        lib.fo_set_beads.argtypes = [_P, C.c_int, _D]
        lib.fo_get_status.argtypes = [_P, _I, _I]
        lib.fo_set_status.argtypes = [_P, _I, _I]
        lib.fo_n_cells.argtypes = [_P]
        lib.fo_n_cells.restype = C.c_int
        lib.fo_list_cap.argtypes = [_P]
        lib.fo_list_cap.restype = C.c_int
        lib.fo_get_cells.argtypes = [_P, _I, _I]
        lib.fo_get_lists.argtypes = [_P, _I, _I, _I]
        lib.fo_overflow.argtypes = [_P, C.POINTER(C.c_long)]
        lib.fo_get_derived.argtypes = [_P, _D]
        lib.fo_get_pairs.argtypes = [_P, _D, _I]
        lib.fo_get_pairs.restype = C.c_int
        _oracle_lib = lib
    return _oracle_lib


def _load_ref():
    global _ref_lib
    if _ref_lib is None:
        if not os.path.isfile(REF_SO):
            raise FileNotFoundError("reference build missing: " + REF_SO)
        lib = C.CDLL(REF_SO)
        lib.ref_create.restype = _P
        lib.ref_create.argtypes = [C.POINTER(FoModel), C.c_int]
        lib.ref_destroy.argtypes = [_P]
        lib.ref_run.argtypes = [_P, C.c_int]
        lib.ref_run.restype = C.c_int
        lib.ref_rebuild.argtypes = [_P]
        lib.ref_reset_energy.argtypes = [_P]
        lib.ref_set_threads.argtypes = [_P, C.c_int]
        lib.ref_forces_only.argtypes = [_P, C.c_int, C.c_int, C.c_int]
        lib.ref_get_beads.argtypes = [_P, C.c_int, _D]
        lib.ref_get_status.argtypes = [_P, _I, _I]
        lib.ref_n_cells.argtypes = [_P]
        lib.ref_n_cells.restype = C.c_int
        lib.ref_get_grid.argtypes = [_P, _I, _I]
        lib.ref_get_lists.argtypes = [_P, _I, _I, _I]
        lib.ref_sizeof.argtypes = [C.c_int]
        lib.ref_sizeof.restype = C.c_int
        _ref_lib = lib
    return _ref_lib


class _Base:
    nb: int
    ns: int
    na: int

    def _vec(self):
        return np.zeros((self.nb, 3), np.float64)


class OracleSim(_Base):
    """The C restatement (fibre_oracle.c)."""

    def __init__(self, model, mode: int = MODE_REF, cell_cap: int = 64, list_cap: int = 256):
        self.lib = _load_oracle()
        fm, self._hold = make_fo_model(model)
        self.nb, self.ns, self.na = fm.n_beads, fm.n_springs, fm.n_angles
        self.h = self.lib.fo_create(C.byref(fm), mode, cell_cap, list_cap)
        self.mode = mode

    def close(self):
        if getattr(self, "h", None):
            self.lib.fo_destroy(self.h)
            self.h = None

    __del__ = close

    def run(self, n: int):
        assert self.lib.fo_run(self.h, n) == 0

    def derived(self) -> np.ndarray:
        """dt, half_dt, half_dt2, lambda_dt, damping, cutoff_sq, wall_k,
        gravity[3], box[3], step[3], half_box_sq, nx, ny, nz."""
        out = np.zeros(20)
        self.lib.fo_get_derived(self.h, out.ctypes.data_as(_D))
        return out

    def pairs(self):
        """Pair table: (coefficients c1..c6 per pair, kind per pair)."""
        n = 64 * 65 // 2
        c6 = np.zeros((n, 6)); k = np.zeros(n, np.int32)
        np_ = self.lib.fo_get_pairs(self.h, c6.ctypes.data_as(_D), k.ctypes.data_as(_I))
        return c6[:np_], k[:np_]

    def rebuild(self):
        self.lib.fo_rebuild(self.h)

    def reset_energy(self):
        self.lib.fo_reset_energy(self.h)

    def forces_only(self, springs=True, angles=True, contacts=True):
        self.lib.fo_forces_only(self.h, int(springs), int(angles), int(contacts))

    def get(self, field: str) -> np.ndarray:
        out = self._vec()
        self.lib.fo_get_beads(self.h, FIELD[field], out.ctypes.data_as(_D))
        return out

    def set(self, field: str, values) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(self.nb, 3)
        self.lib.fo_set_beads(self.h, FIELD[field], a.ctypes.data_as(_D))

    def status(self):
        s = np.zeros(max(self.ns, 1), np.int32)
        a = np.zeros(max(self.na, 1), np.int32)
        self.lib.fo_get_status(self.h, s.ctypes.data_as(_I), a.ctypes.data_as(_I))
        return s[: self.ns], a[: self.na]

    def set_status(self, springs, angles):
        s = np.ascontiguousarray(springs, np.int32)
        a = np.ascontiguousarray(angles, np.int32)
        self.lib.fo_set_status(self.h, s.ctypes.data_as(_I), a.ctypes.data_as(_I))

    def cells(self):
        bc = np.zeros(self.nb, np.int32)
        cc = np.zeros(self.lib.fo_n_cells(self.h), np.int32)
        self.lib.fo_get_cells(self.h, bc.ctypes.data_as(_I), cc.ctypes.data_as(_I))
        return bc, cc

    def lists(self):
        cap = self.lib.fo_list_cap(self.h)
        head = np.zeros(self.nb, np.int32)
        part = np.zeros((self.nb, cap), np.int32)
        pair = np.zeros((self.nb, cap), np.int32)
        self.lib.fo_get_lists(self.h, head.ctypes.data_as(_I), part.ctypes.data_as(_I),
                              pair.ctypes.data_as(_I))
        return head, part, pair

    def overflow(self):
        out = (C.c_long * 2)()
        self.lib.fo_overflow(self.h, out)
        return int(out[0]), int(out[1])


class RefSim(_Base):
    """The reference's own kernels (kernel.cl compiled as C)."""

    def __init__(self, model, threads: int = 1):
        self.lib = _load_ref()
        fm, self._hold = make_fo_model(model)
        self.nb, self.ns, self.na = fm.n_beads, fm.n_springs, fm.n_angles
        self.h = self.lib.ref_create(C.byref(fm), threads)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    __del__ = close

    def set_threads(self, n: int):
        self.lib.ref_set_threads(self.h, n)

    def run(self, n: int):
        assert self.lib.ref_run(self.h, n) == 0

    def rebuild(self):
        self.lib.ref_rebuild(self.h)

    def reset_energy(self):
        self.lib.ref_reset_energy(self.h)

    def forces_only(self, springs=True, angles=True, contacts=True):
        self.lib.ref_forces_only(self.h, int(springs), int(angles), int(contacts))

    def get(self, field: str) -> np.ndarray:
        out = self._vec()
        self.lib.ref_get_beads(self.h, FIELD[field], out.ctypes.data_as(_D))
        return out

    def status(self):
        s = np.zeros(max(self.ns, 1), np.int32)
        a = np.zeros(max(self.na, 1), np.int32)
        self.lib.ref_get_status(self.h, s.ctypes.data_as(_I), a.ctypes.data_as(_I))
        return s[: self.ns], a[: self.na]

    def grid(self):
        n = self.lib.ref_n_cells(self.h)
        head = np.zeros(n, np.int32)
        tail = np.zeros((n, 64), np.int32)
        self.lib.ref_get_grid(self.h, head.ctypes.data_as(_I), tail.ctypes.data_as(_I))
        return head, tail

    def lists(self):
        head = np.zeros(self.nb, np.int32)
        part = np.zeros((self.nb, 256), np.int32)
        pair = np.zeros((self.nb, 256), np.int32)
        self.lib.ref_get_lists(self.h, head.ctypes.data_as(_I), part.ctypes.data_as(_I),
                               pair.ctypes.data_as(_I))
        return head, part, pair


def pair_set(head, partners, pairs=None, cap=None):
    """Unordered (i, j[, pair]) set of a per-bead contact list."""
    out = set()
    nb = head.shape[0]
    cap = cap or partners.shape[1]
    for i in range(nb):
        for k in range(min(int(head[i]), cap)):
            j = int(partners[i, k])
            key = (min(i, j), max(i, j))
            if pairs is not None:
                key = key + (int(pairs[i, k]),)
            out.add(key)
    return out
