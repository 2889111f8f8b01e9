"""In-memory description of one FibreNet simulation (settings + model).

This is the Python-side mirror of what the reference reads from its input
file (``SimulationManager::ReadInputFile``, SimulationManager.cpp:1153-1171)
and its model file (``ReadBeadsData`` / ``ReadSpringData`` /
``ReadAngleData``, SimulationManager.cpp:1372-1661).  Values are kept exactly
as written in those files; derived constants (inverse masses, pair
coefficients, grid geometry) are computed by the native host layer.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import numpy as np

# pair kinds, SimulationManager.cpp:891-932 (type ids written into Pair.type)
PAIR_LJ = 1
PAIR_HS = 2
PAIR_ST = 3
PAIR_HSR = 4  # extension: penalty + soft harmonic repulsion on one type pair

SPRING_HR = 0
SPRING_HR_FL = 1
ANGLE_HR = 0
ANGLE_HR_FL = 1


def pair_index(t1: int, t2: int, n_types: int) -> int:
    """GETADRESS (kernel.cl:9, SimulationManager.cpp:886)."""
    if t1 > t2:
        t1, t2 = t2, t1
    return n_types * t1 + t2 - (t1 * (t1 + 1)) // 2


@dataclass
class Settings:
    """Input-file settings (README.md:123-606)."""

    dt: float = 0.001  # 'step'
    lam: float = 0.5  # 'lambda'
    damping: float = 0.0  # 'damping' as written (the host negates it)
    gravity: tuple = (0.0, 0.0, 0.0)
    cutoff: float = 1.0
    box_unit_cell: float = 1.0
    box: tuple = (10.0, 10.0, 10.0)
    wall_k: float = 0.0  # 'box_wall_rep'
    bc_type: int = 0  # 0 pbc, 1 finite
    grid_update_freq: int = 8
    skin_ratio: float = 0.5
    # extension: bit a set = axis a periodic; -1 = from bc_type (reference)
    periodic_mask: int = -1


@dataclass
class Model:
    settings: Settings
    type_names: list
    pair_kind: np.ndarray  # int32 [n_pairs]
    pair_raw: np.ndarray  # float64 [n_pairs, 4]  raw 'pair' tokens 4..7
    # beads
    type: np.ndarray
    tag: np.ndarray
    loc_id: np.ndarray
    radius: np.ndarray
    mass: np.ndarray
    pos: np.ndarray  # [N, 3] float64, inside the box
    vel: np.ndarray
    vel_old: np.ndarray
    force: np.ndarray
    img: np.ndarray  # unwrapped ('image') positions
    # springs
    s_type: np.ndarray
    s_tag: np.ndarray
    s_p1: np.ndarray
    s_p2: np.ndarray
    s_rest: np.ndarray
    s_k: np.ndarray
    s_c1: np.ndarray
    s_c2: np.ndarray
    # angles
    a_type: np.ndarray
    a_tag: np.ndarray
    a_b1: np.ndarray
    a_b2: np.ndarray
    a_b3: np.ndarray
    a_s1: np.ndarray
    a_s2: np.ndarray
    a_theta0: np.ndarray
    a_k: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n_beads(self) -> int:
        return int(self.type.shape[0])

    @property
    def n_springs(self) -> int:
        return int(self.s_type.shape[0])

    @property
    def n_angles(self) -> int:
        return int(self.a_type.shape[0])

    @property
    def n_types(self) -> int:
        return len(self.type_names)

    def copy(self) -> "Model":
        out = {}
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            if isinstance(v, np.ndarray):
                out[f.name] = v.copy()
            elif isinstance(v, Settings):
                out[f.name] = dataclasses.replace(v)
            elif isinstance(v, (list, dict)):
                out[f.name] = type(v)(v)
            else:
                out[f.name] = v
        return Model(**out)

    def normalised(self) -> "Model":
        """Same model with every array in the dtype and layout the native
        layers expect (contiguous int32 / float64); arrays already in that
        form are shared, not copied."""
        m = dataclasses.replace(self, settings=dataclasses.replace(self.settings),
                                type_names=list(self.type_names), meta=dict(self.meta))
        ints = ["pair_kind", "type", "tag", "loc_id", "s_type", "s_tag", "s_p1", "s_p2",
                "a_type", "a_tag", "a_b1", "a_b2", "a_b3", "a_s1", "a_s2"]
        for name in ints:
            setattr(m, name, np.ascontiguousarray(getattr(m, name), dtype=np.int32))
        for name in ["pair_raw", "radius", "mass", "pos", "vel", "vel_old", "force", "img",
                     "s_rest", "s_k", "s_c1", "s_c2", "a_theta0", "a_k"]:
            setattr(m, name, np.ascontiguousarray(getattr(m, name), dtype=np.float64))
        m.pair_raw = m.pair_raw.reshape(-1, 4)
        for name in ["pos", "vel", "vel_old", "force", "img"]:
            setattr(m, name, getattr(m, name).reshape(-1, 3))
        return m

    def fp32_representable(self) -> "Model":
        """Same model with every per-bead and per-bond real value rounded to
        float32 (the values the B200 path stores), so a float64 checker and
        the device see identical inputs."""
        m = self.normalised()
        for name in ["radius", "vel", "vel_old", "force", "s_rest", "s_k", "s_c1", "s_c2",
                     "a_theta0", "a_k"]:
            setattr(m, name, getattr(m, name).astype(np.float32).astype(np.float64))
        return m


def empty_bonds(m_beads: int):
    z_i = np.zeros(0, np.int32)
    z_d = np.zeros(0, np.float64)
    return z_i, z_d


_ARRAYS = ["pair_kind", "pair_raw", "type", "tag", "loc_id", "radius", "mass", "pos", "vel",
           "vel_old", "force", "img", "s_type", "s_tag", "s_p1", "s_p2", "s_rest", "s_k", "s_c1",
           "s_c2", "a_type", "a_tag", "a_b1", "a_b2", "a_b3", "a_s1", "a_s2", "a_theta0", "a_k"]


def model_to_arrays(m: Model, prefix: str = "m_") -> dict:
    """Flat dict of numpy arrays (for .npz storage)."""
    import json
    out = {prefix + k: np.asarray(getattr(m, k)) for k in _ARRAYS}
    s = dataclasses.asdict(m.settings)
    out[prefix + "settings"] = np.array(json.dumps(s))
    out[prefix + "type_names"] = np.array(json.dumps(list(m.type_names)))
    return out


def model_from_arrays(d, prefix: str = "m_") -> Model:
    import json
    s = json.loads(str(d[prefix + "settings"]))
    s["gravity"] = tuple(s["gravity"])
    s["box"] = tuple(s["box"])
    kw = {k: np.array(d[prefix + k]) for k in _ARRAYS}
    return Model(settings=Settings(**s), type_names=json.loads(str(d[prefix + "type_names"])), **kw)


def permute_model(m: Model, perm) -> Model:
    """Model with beads renumbered: new bead q is old bead perm[q]; bond
    endpoints are remapped, bond order is kept."""
    m = m.normalised()
    perm = np.asarray(perm, np.int64)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    out = m.copy()
    for name in ["type", "tag", "loc_id", "radius", "mass", "pos", "vel", "vel_old", "force", "img"]:
        setattr(out, name, np.ascontiguousarray(getattr(m, name)[perm]))
    for name in ["s_p1", "s_p2", "a_b1", "a_b2", "a_b3"]:
        setattr(out, name, inv[getattr(m, name)].astype(np.int32))
    return out
