"""ctypes binding of libfibrenet.so (the C ABI in include/fibrenet.h).

There is no CPU fallback: if the library or a CUDA device is missing, the
constructor raises.  Arrays cross the boundary as plain host buffers; the
context owns all device memory.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .model import Model

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfibrenet.so")

FN_OK = 0
ERRORS = {1: "bad argument", 2: "CUDA error", 3: "out of device memory", 4: "capacity exceeded",
          5: "call out of order", 6: "non-finite state", 7: "unsupported"}
FIELDS = {"pos": 0, "img": 1, "vel": 2, "force": 3, "vel_old": 4}

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class FnSettings(C.Structure):
    _fields_ = [("dt", C.c_double), ("lam", C.c_double), ("damping", C.c_double),
                ("gravity", C.c_double * 3), ("cutoff", C.c_double),
                ("box_unit_cell", C.c_double), ("box", C.c_double * 3), ("wall_k", C.c_double),
                ("bc_type", C.c_int), ("grid_update_freq", C.c_int), ("skin_ratio", C.c_double),
                ("n_types", C.c_int), ("periodic_mask", C.c_int)]


class FnNetworkDesc(C.Structure):
    _fields_ = [("settings", FnSettings), ("pair_kind", _I), ("pair_raw", _D),
                ("n_beads", C.c_int), ("type", _I), ("tag", _I), ("loc_id", _I),
                ("radius", _D), ("mass", _D), ("pos", _D), ("vel", _D), ("vel_old", _D),
                ("force", _D), ("img", _D),
                ("n_springs", C.c_int), ("s_type", _I), ("s_p1", _I), ("s_p2", _I),
                ("s_rest", _D), ("s_k", _D), ("s_c1", _D), ("s_c2", _D),
                ("n_angles", C.c_int), ("a_type", _I), ("a_b1", _I), ("a_b2", _I), ("a_b3", _I),
                ("a_s1", _I), ("a_s2", _I), ("a_theta0", _D), ("a_k", _D)]


class FnConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("cell_capacity", C.c_int), ("list_capacity", C.c_int),
                ("reorder", C.c_int), ("use_graphs", C.c_int), ("block_size", C.c_int),
                ("chain_mode", C.c_int), ("verlet_skin", C.c_double), ("host_upload", C.c_int)]


class FnStats(C.Structure):
    _fields_ = [("cell_overflow", C.c_longlong), ("list_overflow", C.c_longlong),
                ("rebuilds", C.c_longlong), ("steps", C.c_longlong), ("block_size", C.c_int),
                ("bond_path", C.c_int), ("n_networks", C.c_int), ("n_beads", C.c_longlong),
                ("device_bytes", C.c_longlong), ("graph_launches", C.c_longlong),
                ("nonfinite", C.c_longlong), ("items_per_thread", C.c_int),
                ("stalls", C.c_longlong), ("upload_on_device", C.c_int), ("list_by_bricks", C.c_int),
                ("list_build", C.c_int)]


class FnView(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("n", C.c_longlong), ("elem_bytes", C.c_int),
                ("components", C.c_int)]


class FnObservables(C.Structure):
    _fields_ = [("reaction", C.c_double * 3), ("broken", C.c_longlong),
                ("angles_dead", C.c_longlong)]


class FnEnergy(C.Structure):
    _fields_ = [("kinetic", C.c_double), ("spring", C.c_double), ("angle", C.c_double),
                ("contact", C.c_double), ("wall", C.c_double), ("gravity", C.c_double),
                ("virial", C.c_double * 9), ("contacts", C.c_longlong)]


ENERGY_FIELDS = ["kinetic", "spring", "angle", "contact", "wall", "gravity"]
SERIES_COLUMNS = (["step", "reaction_x", "reaction_y", "reaction_z", "broken", "angles_dead"]
                  + ENERGY_FIELDS + [f"virial_{a}{b}" for a in "xyz" for b in "xyz"] + ["contacts"])


class FnRunInfo(C.Structure):
    _fields_ = [("run_steps", C.c_int), ("output_freq", C.c_int), ("minimize_steps", C.c_int),
                ("minimize_substeps", C.c_int), ("minimize_reset", C.c_int),
                ("export_position", C.c_int), ("export_velocity", C.c_int),
                ("export_force", C.c_int), ("has_skin_override", C.c_int), ("strict", C.c_int)]


# every exported entry point: name -> (restype, argtypes)
SIGNATURES = {
    "fn_create": (C.c_int, [C.POINTER(FnConfig), C.POINTER(C.c_void_p)]),
    "fn_destroy": (None, [C.c_void_p]),
    "fn_last_error": (C.c_char_p, [C.c_void_p]),
    "fn_upload": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(FnNetworkDesc)]),
    "fn_step": (C.c_int, [C.c_void_p, C.c_int]),
    "fn_rebuild_contacts": (C.c_int, [C.c_void_p]),
    "fn_reset_energy": (C.c_int, [C.c_void_p]),
    "fn_sync": (C.c_int, [C.c_void_p]),
    "fn_download": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "fn_set_beads": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "fn_set_mass": (C.c_int, [C.c_void_p, _D]),
    "fn_set_skin": (C.c_int, [C.c_void_p, _D]),
    "fn_set_springs": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "fn_set_angles": (C.c_int, [C.c_void_p, _D, _D]),
    "fn_download_status": (C.c_int, [C.c_void_p, _I, _I]),
    "fn_set_status": (C.c_int, [C.c_void_p, _I, _I]),
    "fn_observe": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(FnObservables)]),
    "fn_get_stats": (C.c_int, [C.c_void_p, C.POINTER(FnStats)]),
    "fn_observe_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "fn_energy_eval": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(FnEnergy)]),
    "fn_device_view": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(FnView)]),
    "fn_adjoint_forward": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _D]),
    "fn_adjoint_backward": (C.c_int, [C.c_void_p, _D, _D, _D, _D, _D, _D]),
    "fn_adjoint_release": (C.c_int, [C.c_void_p]),
    "fn_step_series": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _D]),
    "fn_get_cells": (C.c_int, [C.c_void_p, _I, _I, C.c_longlong]),
    "fn_get_lists": (C.c_int, [C.c_void_p, _I, _I, C.c_int]),
    "fn_n_cells": (C.c_longlong, [C.c_void_p]),
    "fn_get_permutation": (C.c_int, [C.c_void_p, _I]),
    "fn_forces_only": (C.c_int, [C.c_void_p, C.c_int]),
    "fn_autotune": (C.c_int, [C.c_void_p, C.c_int]),
    "fn_set_kernel_shape": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "fn_set_list_build": (C.c_int, [C.c_void_p, C.c_int]),
    "fn_state_save": (C.c_int, [C.c_void_p]),
    "fn_state_restore": (C.c_int, [C.c_void_p]),
    "fn_step_timed": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "fn_enable_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "fn_kernel_time": (C.c_int, [C.c_void_p, _D, C.POINTER(C.c_longlong), _D,
                                 C.POINTER(C.c_longlong)]),
    "fn_place_fibres": (C.c_int, [C.c_ulonglong, C.c_int, C.c_int, _D, C.c_int, C.c_double,
                                  C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                  C.c_int, _D]),
    # include/fibrenet_io.h
    "fn_input_read": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p), C.c_char_p, C.c_int]),
    "fn_input_free": (None, [C.c_void_p]),
    "fn_input_desc": (C.c_int, [C.c_void_p, C.POINTER(FnNetworkDesc)]),
    "fn_input_info": (C.c_int, [C.c_void_p, C.POINTER(FnRunInfo)]),
    "fn_input_skin": (C.POINTER(C.c_double), [C.c_void_p]),
    "fn_input_type_name": (C.c_char_p, [C.c_void_p, C.c_int]),
    "fn_input_output_stem": (C.c_char_p, [C.c_void_p]),
    "fn_run_input": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_int]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Loads the native library (building it first if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class NativeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Keep:
    pass


def network_desc(m: Model, keep: _Keep) -> FnNetworkDesc:
    m = m.normalised()
    keep.__dict__.setdefault("models", []).append(m)
    s = m.settings
    d = FnNetworkDesc()
    st = d.settings
    st.dt, st.lam, st.damping = s.dt, s.lam, s.damping
    st.gravity = (C.c_double * 3)(*s.gravity)
    st.cutoff, st.box_unit_cell = s.cutoff, s.box_unit_cell
    st.box = (C.c_double * 3)(*s.box)
    st.wall_k, st.bc_type, st.grid_update_freq = s.wall_k, s.bc_type, s.grid_update_freq
    st.skin_ratio, st.n_types, st.periodic_mask = s.skin_ratio, m.n_types, s.periodic_mask

    def dp(a):
        return a.ctypes.data_as(_D)

    def ip(a):
        return a.ctypes.data_as(_I)

    d.pair_kind, d.pair_raw = ip(m.pair_kind), dp(m.pair_raw)
    d.n_beads = m.n_beads
    d.type, d.tag, d.loc_id = ip(m.type), ip(m.tag), ip(m.loc_id)
    d.radius, d.mass = dp(m.radius), dp(m.mass)
    d.pos, d.vel, d.vel_old, d.force, d.img = dp(m.pos), dp(m.vel), dp(m.vel_old), dp(m.force), dp(m.img)
    d.n_springs = m.n_springs
    d.s_type, d.s_p1, d.s_p2 = ip(m.s_type), ip(m.s_p1), ip(m.s_p2)
    d.s_rest, d.s_k, d.s_c1, d.s_c2 = dp(m.s_rest), dp(m.s_k), dp(m.s_c1), dp(m.s_c2)
    d.n_angles = m.n_angles
    d.a_type, d.a_b1, d.a_b2, d.a_b3 = ip(m.a_type), ip(m.a_b1), ip(m.a_b2), ip(m.a_b3)
    d.a_s1, d.a_s2, d.a_theta0, d.a_k = ip(m.a_s1), ip(m.a_s2), dp(m.a_theta0), dp(m.a_k)
    return d


class Simulation:
    """One device context holding one network or a batched ensemble."""

    def __init__(self, models, device: int = 0, cell_capacity: int = 64, list_capacity: int = 64,
                 reorder: bool = True, use_graphs: bool = False, block_size: int = 0,
                 chain: bool = True, verlet_skin: float = 0.0, staged: bool = True,
                 host_upload: bool = False):
        self.lib = load()
        self.models = [models] if isinstance(models, Model) else list(models)
        chain_mode = (0 if staged else 1) if chain else 2
        cfg = FnConfig(device, cell_capacity, list_capacity, int(reorder), int(use_graphs),
                       block_size, chain_mode, float(verlet_skin), int(host_upload))
        h = C.c_void_p()
        rc = self.lib.fn_create(C.byref(cfg), C.byref(h))
        if rc != FN_OK:
            raise NativeError(rc, "fn_create failed (no CUDA device or bad config)")
        self.h = h
        self.device = device
        self.list_capacity = list_capacity
        keep = _Keep()
        descs = (FnNetworkDesc * len(self.models))(*[network_desc(m, keep) for m in self.models])
        self._check(self.lib.fn_upload(self.h, len(self.models), descs))
        self.nb = sum(m.n_beads for m in self.models)
        self.ns = sum(m.n_springs for m in self.models)
        self.na = sum(m.n_angles for m in self.models)

    def _check(self, rc):
        if rc != FN_OK:
            msg = self.lib.fn_last_error(self.h).decode() if getattr(self, "h", None) else ""
            raise NativeError(rc, msg)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- stepping
    def step(self, n: int):
        self._check(self.lib.fn_step(self.h, int(n)))

    def step_timed(self, n: int) -> float:
        """fn_step(n) timed with CUDA events on the context's stream; returns
        the device time in ms (waits for the steps)."""
        ms = C.c_double()
        self._check(self.lib.fn_step_timed(self.h, int(n), C.byref(ms)))
        return ms.value

    def save_state(self):
        """Device-side snapshot of the dynamic state (fn_state_save)."""
        self._check(self.lib.fn_state_save(self.h))

    def restore_state(self):
        """Puts the last snapshot back (fn_state_restore)."""
        self._check(self.lib.fn_state_restore(self.h))

    def rebuild(self):
        self._check(self.lib.fn_rebuild_contacts(self.h))

    def reset_energy(self):
        self._check(self.lib.fn_reset_energy(self.h))

    def sync(self):
        self._check(self.lib.fn_sync(self.h))

    def forces_only(self, springs=True, angles=True, contacts=True):
        terms = (1 if springs else 0) | (2 if angles else 0) | (4 if contacts else 0)
        self._check(self.lib.fn_forces_only(self.h, terms))

    # --- state
    def get(self, field: str) -> np.ndarray:
        out = np.empty((self.nb, 3), np.float64)  # every element is written by fn_download
        self._check(self.lib.fn_download(self.h, FIELDS[field], out.ctypes.data_as(_D)))
        return out

    def set(self, field: str, values) -> None:
        a = np.ascontiguousarray(values, np.float64).reshape(self.nb, 3)
        self._check(self.lib.fn_set_beads(self.h, FIELDS[field], a.ctypes.data_as(_D)))

    def set_mass(self, mass) -> None:
        a = np.ascontiguousarray(mass, np.float64).reshape(self.nb)
        self._check(self.lib.fn_set_mass(self.h, a.ctypes.data_as(_D)))

    def set_skin(self, skin) -> None:
        a = np.ascontiguousarray(skin, np.float64).reshape(self.nb)
        self._check(self.lib.fn_set_skin(self.h, a.ctypes.data_as(_D)))

    def set_springs(self, rest=None, k=None, c1=None, c2=None) -> None:
        arrs = [None if x is None else np.ascontiguousarray(x, np.float64).reshape(self.ns)
                for x in (rest, k, c1, c2)]
        ptrs = [None if a is None else a.ctypes.data_as(_D) for a in arrs]
        self._check(self.lib.fn_set_springs(self.h, *ptrs))

    def set_angles(self, theta0=None, k=None) -> None:
        arrs = [None if x is None else np.ascontiguousarray(x, np.float64).reshape(self.na)
                for x in (theta0, k)]
        ptrs = [None if a is None else a.ctypes.data_as(_D) for a in arrs]
        self._check(self.lib.fn_set_angles(self.h, *ptrs))

    def status(self):
        s = np.zeros(max(self.ns, 1), np.int32)
        a = np.zeros(max(self.na, 1), np.int32)
        self._check(self.lib.fn_download_status(self.h, s.ctypes.data_as(_I), a.ctypes.data_as(_I)))
        return s[: self.ns], a[: self.na]

    def set_status(self, springs=None, angles=None):
        s = None if springs is None else np.ascontiguousarray(springs, np.int32)
        a = None if angles is None else np.ascontiguousarray(angles, np.int32)
        self._check(self.lib.fn_set_status(self.h, None if s is None else s.ctypes.data_as(_I),
                                           None if a is None else a.ctypes.data_as(_I)))

    def observe(self, net: int = 0, reaction_type: int = -1) -> dict:
        o = FnObservables()
        self._check(self.lib.fn_observe(self.h, net, reaction_type, C.byref(o)))
        return {"reaction": np.array(o.reaction[:]), "broken": int(o.broken),
                "angles_dead": int(o.angles_dead)}

    def observe_noalloc(self, out_device_ptr: int, net: int = 0, reaction_type: int = -1) -> None:
        """fn_observe without device allocation: writes 5 doubles (reaction
        x, y, z, broken springs, dead angles) to a caller-owned device buffer
        asynchronously; call sync() before reading it."""
        self._check(self.lib.fn_observe_noalloc(self.h, net, reaction_type,
                                                C.c_void_p(out_device_ptr)))

    def energy(self, net: int = 0) -> dict:
        """Energy terms, their sum ("total"), the 3x3 virial and the count of
        acting contact pairs of network ``net`` (fn_energy_eval)."""
        e = FnEnergy()
        self._check(self.lib.fn_energy_eval(self.h, net, C.byref(e)))
        out = {f: float(getattr(e, f)) for f in ENERGY_FIELDS}
        out["total"] = sum(out[f] for f in ENERGY_FIELDS)
        out["virial"] = np.array(e.virial[:]).reshape(3, 3)
        out["contacts"] = int(e.contacts)
        return out

    def step_series(self, nsteps: int, every: int, net: int = 0, reaction_type: int = -1,
                    energy: bool = False) -> np.ndarray:
        """Runs nsteps in chunks of ``every`` and returns one row per chunk
        (columns SERIES_COLUMNS[:6], or all 22 with ``energy``)."""
        width = len(SERIES_COLUMNS) if energy else 6
        rows = -(-nsteps // every)
        out = np.zeros((rows, width), np.float64)
        self._check(self.lib.fn_step_series(self.h, nsteps, every, net, reaction_type, int(energy),
                                            out.ctypes.data_as(_D)))
        return out

    def device_view(self, field: str):
        """The device array of ``field`` as a torch tensor [n, 4] without a
        copy (internal bead order, see permutation()); valid until the next
        step, upload or state restore."""
        import torch
        v = FnView()
        self._check(self.lib.fn_device_view(self.h, FIELDS[field], C.byref(v)))

        class _Iface:
            pass
        it = _Iface()
        it.__cuda_array_interface__ = {
            "shape": (int(v.n), int(v.components)), "typestr": "<f8" if v.elem_bytes == 8 else "<f4",
            "data": (int(v.ptr), False), "version": 3, "strides": None}
        return torch.as_tensor(it, device=f"cuda:{self.device}")

    # --- differentiation
    def adjoint_forward(self, nsamples: int, every: int, checkpoint_every: int,
                        reaction_type: int) -> np.ndarray:
        """nsamples step(every) calls with checkpoints; returns the reaction of
        every network after each call, [nsamples, n_networks, 3]."""
        out = np.zeros((nsamples, len(self.models), 3), np.float64)
        self._check(self.lib.fn_adjoint_forward(self.h, nsamples, every, checkpoint_every,
                                                reaction_type, out.ctypes.data_as(_D)))
        return out

    def adjoint_backward(self, dloss_dreaction) -> dict:
        """Gradients for dL/d reaction ([nsamples, n_networks, 3]): spring_k,
        spring_rest (per spring), angle_k (per angle), pos0 and vel0 (per
        bead, [n, 3]), all in upload order."""
        g = np.ascontiguousarray(dloss_dreaction, np.float64)
        out = {"spring_k": np.zeros(self.ns), "spring_rest": np.zeros(self.ns),
               "angle_k": np.zeros(self.na), "pos0": np.zeros((self.nb, 3)),
               "vel0": np.zeros((self.nb, 3))}
        self._check(self.lib.fn_adjoint_backward(
            self.h, g.ctypes.data_as(_D), *[out[k].ctypes.data_as(_D) for k in
                                            ("spring_k", "spring_rest", "angle_k", "pos0", "vel0")]))
        return out

    def adjoint_release(self) -> None:
        self._check(self.lib.fn_adjoint_release(self.h))

    def stats(self) -> dict:
        s = FnStats()
        self._check(self.lib.fn_get_stats(self.h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in FnStats._fields_}

    def cells(self):
        n = int(self.lib.fn_n_cells(self.h))
        bc = np.zeros(self.nb, np.int32)
        cc = np.zeros(n, np.int32)
        self._check(self.lib.fn_get_cells(self.h, bc.ctypes.data_as(_I), cc.ctypes.data_as(_I), n))
        return bc, cc

    def lists(self):
        cap = self.list_capacity
        cnt = np.zeros(self.nb, np.int32)
        part = np.full((self.nb, cap), -1, np.int32)
        self._check(self.lib.fn_get_lists(self.h, cnt.ctypes.data_as(_I), part.ctypes.data_as(_I), cap))
        return cnt, part

    def permutation(self) -> np.ndarray:
        p = np.zeros(self.nb, np.int32)
        self._check(self.lib.fn_get_permutation(self.h, p.ctypes.data_as(_I)))
        return p

    def enable_timing(self, on: bool = True):
        self._check(self.lib.fn_enable_timing(self.h, int(on)))

    def kernel_time(self):
        ms = C.c_double()
        n = C.c_longlong()
        rms = C.c_double()
        rn = C.c_longlong()
        self._check(self.lib.fn_kernel_time(self.h, C.byref(ms), C.byref(n), C.byref(rms), C.byref(rn)))
        return {"step_ms": ms.value, "launches": n.value, "rebuild_ms": rms.value,
                "rebuilds": rn.value}

    def set_kernel_shape(self, block: int, items_per_thread: int = 0) -> None:
        """Step-kernel shape: block size and, for the staged chain kernel,
        contact items per thread and round (0: no staging)."""
        self._check(self.lib.fn_set_kernel_shape(self.h, int(block), int(items_per_thread)))

    LIST_BUILDS = ("beads", "bricks", "groups")

    def set_list_build(self, mode) -> None:
        """How contact lists are built: "beads" (one thread per bead, the
        default; also False / 0), "bricks" (cells staged in shared memory;
        also True / 1) or "groups" (8 lanes per bead; also 2)."""
        m = self.LIST_BUILDS.index(mode) if isinstance(mode, str) else int(mode)
        self._check(self.lib.fn_set_list_build(self.h, m))

    def autotune(self, steps_per_trial: int = 20) -> int:
        self._check(self.lib.fn_autotune(self.h, steps_per_trial))
        return self.stats()["block_size"]
