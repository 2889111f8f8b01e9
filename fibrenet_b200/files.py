"""The reference's input and model files from Python.

Writers produce files in the formats of README.md:32-606 (model: BEAD /
SPRING / ANGLE lines; input: one command per line).  Reading goes through the
native parser (``fn_input_read``, include/fibrenet_io.h), the same code the
command-line runner uses, so Python and C++ see identical models.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .model import PAIR_HS, PAIR_HSR, PAIR_LJ, PAIR_ST, Model, Settings, pair_index

PAIR_NAMES = {PAIR_LJ: "lj", PAIR_HS: "hs", PAIR_ST: "st", PAIR_HSR: "hsr"}
PAIR_TOKENS = {PAIR_LJ: 3, PAIR_HS: 1, PAIR_ST: 4, PAIR_HSR: 3}


def _g(x) -> str:
    return repr(float(x))


def write_model_file(m: Model, path: str) -> None:
    """Model file with every value written exactly (shortest round-trip
    repr), tab-delimited as README.md:34 describes."""
    m = m.normalised()
    lines = []
    names = m.type_names
    for i in range(m.n_beads):
        f = [names[m.type[i]], str(m.tag[i]), str(m.loc_id[i]), _g(m.radius[i]), _g(m.mass[i]),
             *map(_g, m.pos[i]), *map(_g, m.vel[i]), *map(_g, m.force[i]), *map(_g, m.img[i])]
        lines.append("BEAD\t" + "\t".join(f))
    for s in range(m.n_springs):
        kind = "HR_FL" if m.s_type[s] == 1 else "HR"
        f = [kind, str(m.s_tag[s]), str(m.s_p1[s]), str(m.s_p2[s]), _g(m.s_rest[s]), _g(m.s_k[s])]
        if m.s_type[s] == 1:
            f += [_g(m.s_c1[s]), _g(m.s_c2[s])]
        lines.append("SPRING\t" + "\t".join(f))
    for a in range(m.n_angles):
        kind = "HR_FL" if m.a_type[a] == 1 else "HR"
        f = [kind, str(m.a_tag[a]), str(m.a_b1[a]), str(m.a_b2[a]), str(m.a_b3[a]), str(m.a_s1[a]),
             str(m.a_s2[a]), _g(m.a_theta0[a]), _g(m.a_k[a])]
        lines.append("ANGLE\t" + "\t".join(f))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_input_file(m: Model, path: str, model_path: str, output_stem: str, run: int,
                     output_freq: int, output_data=("position",), output_types=None,
                     minimize=None, extra_lines=()) -> None:
    """Input file for model ``m`` (README.md:123-606).  ``minimize`` =
    (steps, substeps, reset)."""
    s = m.settings
    L = [f"model_file\t{model_path}", f"output_file\t{output_stem}", f"output_freq\t{output_freq}"]
    L += [f"output_data\t{d}" for d in output_data]
    L += [f"output_type\t{t}" for t in (output_types or m.type_names)]
    L += [f"run\t{run}", f"step\t{_g(s.dt)}", f"lambda\t{_g(s.lam)}", f"cutoff\t{_g(s.cutoff)}"]
    if s.damping:
        L.append(f"damping\t{_g(s.damping)}")
    if any(s.gravity):
        L.append("gravity\t" + "\t".join(map(_g, s.gravity)))
    if minimize:
        L += [f"minimize_steps\t{minimize[0]}", f"minimize_substeps\t{minimize[1]}",
              f"minimize_reset\t{'yes' if minimize[2] else 'no'}"]
    L += [f"box_unit_cell\t{_g(s.box_unit_cell)}", "box_size\t" + "\t".join(map(_g, s.box)),
          f"box_type\t{'pbc' if s.bc_type == 0 else 'finite'}", f"box_wall_rep\t{_g(s.wall_k)}",
          f"grid_update_freq\t{s.grid_update_freq}"]
    L += [f"type\t{t}" for t in m.type_names]
    nt = m.n_types
    raw = np.asarray(m.pair_raw).reshape(-1, 4)
    for t1 in range(nt):
        for t2 in range(t1, nt):
            k = pair_index(t1, t2, nt)
            kind = int(m.pair_kind[k])
            vals = "\t".join(_g(v) for v in raw[k][:PAIR_TOKENS[kind]])
            L.append(f"pair\t{PAIR_NAMES[kind]}\t{m.type_names[t1]}\t{m.type_names[t2]}\t{vals}")
    L += list(extra_lines)
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")


def _lib():
    from . import native
    return native.load()


class InputError(ValueError):
    pass


def read_input(path: str, strict: bool = False):
    """Parses an input file (and its model / restart files) with the native
    parser.  Returns (Model, run-info dict, per-bead skin radius or None)."""
    lib = _lib()
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    rc = lib.fn_input_read(os.fsencode(path), int(strict), C.byref(h), err, 512)
    if rc != 0:
        raise InputError(err.value.decode())
    try:
        from .native import FnNetworkDesc
        d = FnNetworkDesc()
        lib.fn_input_desc(h, C.byref(d))
        from .native import FnRunInfo
        info = FnRunInfo()
        lib.fn_input_info(h, C.byref(info))
        n, ns, na = d.n_beads, d.n_springs, d.n_angles
        nt = d.settings.n_types

        def arr(ptr, count, dt):
            if count == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt).copy()

        st = d.settings
        settings = Settings(dt=st.dt, lam=st.lam, damping=st.damping, gravity=tuple(st.gravity),
                            cutoff=st.cutoff, box_unit_cell=st.box_unit_cell, box=tuple(st.box),
                            wall_k=st.wall_k, bc_type=st.bc_type, grid_update_freq=st.grid_update_freq,
                            skin_ratio=st.skin_ratio, periodic_mask=st.periodic_mask)
        names = [lib.fn_input_type_name(h, t).decode() for t in range(nt)]
        npairs = nt * (nt + 1) // 2
        i32, f64 = np.int32, np.float64
        m = Model(
            settings=settings, type_names=names, pair_kind=arr(d.pair_kind, npairs, i32),
            pair_raw=arr(d.pair_raw, 4 * npairs, f64).reshape(-1, 4),
            type=arr(d.type, n, i32), tag=arr(d.tag, n, i32), loc_id=arr(d.loc_id, n, i32),
            radius=arr(d.radius, n, f64), mass=arr(d.mass, n, f64),
            pos=arr(d.pos, 3 * n, f64).reshape(n, 3), vel=arr(d.vel, 3 * n, f64).reshape(n, 3),
            vel_old=arr(d.vel_old, 3 * n, f64).reshape(n, 3),
            force=arr(d.force, 3 * n, f64).reshape(n, 3), img=arr(d.img, 3 * n, f64).reshape(n, 3),
            s_type=arr(d.s_type, ns, i32), s_tag=np.zeros(ns, i32), s_p1=arr(d.s_p1, ns, i32),
            s_p2=arr(d.s_p2, ns, i32), s_rest=arr(d.s_rest, ns, f64), s_k=arr(d.s_k, ns, f64),
            s_c1=arr(d.s_c1, ns, f64), s_c2=arr(d.s_c2, ns, f64),
            a_type=arr(d.a_type, na, i32), a_tag=np.zeros(na, i32), a_b1=arr(d.a_b1, na, i32),
            a_b2=arr(d.a_b2, na, i32), a_b3=arr(d.a_b3, na, i32), a_s1=arr(d.a_s1, na, i32),
            a_s2=arr(d.a_s2, na, i32), a_theta0=arr(d.a_theta0, na, f64), a_k=arr(d.a_k, na, f64),
        )
        skin = arr(lib.fn_input_skin(h), n, f64) if info.has_skin_override else None
        run = {f: getattr(info, f) for f, _ in FnRunInfo._fields_}
        run["output_stem"] = lib.fn_input_output_stem(h).decode()
        return m, run, skin
    finally:
        lib.fn_input_free(h)


def run_input(path: str, device: int = 0, strict: bool = False) -> None:
    """SimulationManager's Initialize + Run + Close on an input file."""
    lib = _lib()
    err = C.create_string_buffer(512)
    rc = lib.fn_run_input(os.fsencode(path), device, int(strict), err, 512)
    if rc != 0:
        raise InputError(f"run failed ({rc}): {err.value.decode()}")


def read_xyz(path: str):
    """Frames of an XYZ output file: list of (step, names, [n, 3] array)."""
    frames = []
    with open(path) as fh:
        lines = fh.read().splitlines()
    i = 0
    while i < len(lines):
        n = int(lines[i])
        head = lines[i + 1].split()
        rows = [ln.split() for ln in lines[i + 2:i + 2 + n]]
        frames.append((int(head[1]), [r[0] for r in rows],
                       np.array([[float(x) for x in r[1:4]] for r in rows])))
        i += 2 + n
    return frames
