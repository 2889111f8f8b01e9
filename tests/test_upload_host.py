"""The model upload's host logic on the CPU: fn_create + fn_upload built
against host stand-ins for the CUDA runtime (tests/host_upload/), so the bead
ordering, the packed bead arrays, the spring ends, the bond path chosen and
the argument checks are checked without a GPU.  The rule the order must
follow is restated here: spring-connected components (fibres) sorted by the
Morton code of their lowest bead (then that bead's index), the beads of each
component in file order."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))
HERE = os.path.join(ROOT, "tests", "host_upload")
LIB = os.path.join(HERE, "_build", "libhostupload.so")
SOURCES = [os.path.join(HERE, "harness.cu"), os.path.join(HERE, "fake_cuda.h")] + [
    os.path.join(ROOT, "fibrenet_b200", "csrc", f)
    for f in ("fn_engine.cu", "fn_engine_internal.h", "fn_kernels.h", "fn_types.h")] + [
    os.path.join(ROOT, "include", "fibrenet.h")]


@pytest.fixture(scope="module")
def hu():
    from fibrenet_b200 import build
    if not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in SOURCES):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        cmd = [build.nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O1",
               "-Xcompiler", "-fPIC", "-include", os.path.join(HERE, "fake_cuda.h"), "-shared",
               "-o", LIB + ".tmp", os.path.join(HERE, "harness.cu")]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            pytest.fail("building the host upload harness failed:\n" + out.stderr[-3000:])
        os.replace(LIB + ".tmp", LIB)
    lib = C.CDLL(LIB)
    lib.hu_error.restype = C.c_char_p
    lib.hu_create.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    for f in ("hu_upload", "hu_permutation", "hu_chain", "hu_beads", "hu_springs", "hu_destroy",
              "hu_error", "hu_tiles", "hu_block", "hu_spring_incidence", "hu_net", "hu_pairs",
              "hu_chain_records", "fn_set_springs", "fn_set_angles", "fn_set_mass",
              "fn_set_status", "fn_download_status"):
        getattr(lib, f).argtypes = None
    return lib


class Upload:
    def __init__(self, lib, models, reorder=True, chain=True):
        from fibrenet_b200 import native
        self.lib = lib
        self.models = models if isinstance(models, list) else [models]
        self.h = C.c_void_p()
        assert lib.hu_create(int(reorder), 0 if chain else 2, C.byref(self.h)) == 0
        keep = native._Keep()
        descs = (native.FnNetworkDesc * len(self.models))(*[native.network_desc(m, keep) for m in self.models])
        self.rc = lib.hu_upload(self.h, len(self.models), descs)
        self.err = lib.hu_error(self.h).decode()
        self.nb = sum(m.n_beads for m in self.models)
        self.ns = sum(m.n_springs for m in self.models)

    def perm(self):
        p = np.zeros(self.nb, np.int32)
        assert self.lib.hu_permutation(self.h, p.ctypes.data_as(C.c_void_p)) == 0
        return p

    def beads(self):
        pos = np.zeros((self.nb, 4)); img = np.zeros((self.nb, 4))
        self.lib.hu_beads(self.h, pos.ctypes.data_as(C.c_void_p), img.ctypes.data_as(C.c_void_p))
        return pos, img

    def springs(self):
        e = np.zeros((max(self.ns, 1), 2), np.int32)
        self.lib.hu_springs(self.h, e.ctypes.data_as(C.c_void_p))
        return e[:self.ns]

    def close(self):
        self.lib.hu_destroy(self.h)


def _spread10(v):
    v = v.astype(np.uint64) & 0x3FF
    v = (v | (v << 16)) & 0x030000FF
    v = (v | (v << 8)) & 0x0300F00F
    v = (v | (v << 4)) & 0x030C30C3
    v = (v | (v << 2)) & 0x09249249
    return v


def expected_order(m):
    """Internal order of one network: components by (Morton code of the
    lowest bead, its index), beads of a component ascending."""
    n = m.n_beads
    parent = np.arange(n)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x
    for a, b in zip(m.s_p1, m.s_p2):
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    root = np.array([find(i) for i in range(n)])
    roots = np.unique(root)
    x = m.pos[roots] / np.asarray(m.settings.box) * 1024.0
    x = np.where(x >= 0.0, x, 0.0)
    q = np.minimum(x, 1023.0).astype(np.uint32)
    code = _spread10(q[:, 0]) | (_spread10(q[:, 1]) << 1) | (_spread10(q[:, 2]) << 2)
    key = {int(r): (int(c), int(r)) for r, c in zip(roots, code)}
    return np.array(sorted(range(n), key=lambda i: (key[int(root[i])], i)), np.int32)


def small_tensile(seed=8):
    from fibrenet_b200 import generate as g
    return g.tensile_network(seed=seed, fibres=40, beads=20, box=(40.0, 30.0, 8.0), z_range=(1.0, 7.0),
                             clamp_lo=2.0, clamp_hi=38.0, cell=2.5)


def test_bead_order_and_staged_beads(hu):
    m = small_tensile().normalised()
    u = Upload(hu, m)
    try:
        assert u.rc == 0, u.err
        perm = u.perm()
        np.testing.assert_array_equal(perm, expected_order(m))
        pos, img = u.beads()
        np.testing.assert_array_equal(pos[:, :3], m.pos[perm])
        np.testing.assert_array_equal(img[:, :3], m.img[perm])
        minv = np.where(m.mass > 0, 1.0 / np.where(m.mass > 0, m.mass, 1.0), 0.0)
        np.testing.assert_array_equal(img[:, 3], minv[perm])
        inv = np.empty_like(perm)
        inv[perm] = np.arange(len(perm))
        np.testing.assert_array_equal(u.springs(), np.stack([inv[m.s_p1], inv[m.s_p2]], 1))
        assert hu.hu_chain(u.h) == 1
    finally:
        u.close()


def test_general_topology_order_and_bond_path(hu):
    from test_gpu_parity import _crosslinked
    m = _crosslinked().normalised()
    u = Upload(hu, m)
    try:
        assert u.rc == 0, u.err
        np.testing.assert_array_equal(u.perm(), expected_order(m))
        assert hu.hu_chain(u.h) == 0  # cross-links: not chain form
    finally:
        u.close()


def test_reversed_and_shuffled_springs(hu):
    from test_gpu_parity import _reversed
    m = _reversed(small_tensile(9))
    u = Upload(hu, m)
    try:
        assert u.rc == 0, u.err
        np.testing.assert_array_equal(u.perm(), expected_order(m))
        assert hu.hu_chain(u.h) == 1
    finally:
        u.close()
    m = small_tensile(10).normalised().copy()
    p = np.random.default_rng(3).permutation(m.n_springs)
    for f in ("s_type", "s_tag", "s_p1", "s_p2", "s_rest", "s_k", "s_c1", "s_c2"):
        setattr(m, f, getattr(m, f)[p].copy())
    u = Upload(hu, m)
    try:
        assert u.rc == 0, u.err
        np.testing.assert_array_equal(u.perm(), expected_order(m))
        assert hu.hu_chain(u.h) == 0  # bonds out of ascending order around a bead
    finally:
        u.close()


def test_file_order_kept_without_reorder(hu):
    m = small_tensile(11).normalised()
    u = Upload(hu, m, reorder=False)
    try:
        assert u.rc == 0, u.err
        np.testing.assert_array_equal(u.perm(), np.arange(m.n_beads))
    finally:
        u.close()


def test_batch_orders_each_network_in_its_range(hu):
    from fibrenet_b200 import generate as g
    models = [m.normalised() for m in g.ensemble_networks(seed=3, n_networks=3, fibres_lo=5, fibres_hi=30)]
    u = Upload(hu, models)
    try:
        assert u.rc == 0, u.err
        perm = u.perm()
        base = 0
        for m in models:
            np.testing.assert_array_equal(perm[base:base + m.n_beads] - base, expected_order(m))
            base += m.n_beads
    finally:
        u.close()


@pytest.mark.parametrize("field,idx,val,msg", [
    ("type", 37, 9, "bead 37 has an undeclared type"),
    ("mass", 40, -1.0, "negative mass"),
    ("s_p2", 55, 10**6, "spring 55 references a missing bead"),
    ("a_b3", 70, -2, "angle 70 references a missing bead"),
])
def test_invalid_models_are_named(hu, field, idx, val, msg):
    m = small_tensile(12).normalised().copy()
    a = getattr(m, field).copy()
    a[idx] = val
    a[idx + 5] = val  # a later offender too: the first one is reported
    setattr(m, field, a)
    u = Upload(hu, m)
    try:
        assert u.rc == 1
        assert msg in u.err, u.err
    finally:
        u.close()


def _tiles(hu, u):
    cap = u.nb + 1
    t = np.zeros((cap, 3), np.int32)
    n = hu.hu_tiles(u.h, t.ctypes.data_as(C.c_void_p), cap)
    return t[:n]


def test_tiles_cover_each_network_without_crossing_it(hu):
    """The tile table drives every launch of a batch: each block's beads lie
    in one network, every bead is in exactly one tile, and a chain tile holds
    block - 4 beads (its two-bead halo on each side fills the block)."""
    from fibrenet_b200 import generate as g
    models = [m.normalised() for m in g.ensemble_networks(seed=4, n_networks=4, fibres_lo=3, fibres_hi=25)]
    u = Upload(hu, models)
    try:
        assert u.rc == 0, u.err
        tiles = _tiles(hu, u)
        block = hu.hu_block(u.h)
        starts = np.cumsum([0] + [m.n_beads for m in models])
        covered = np.zeros(u.nb, np.int32)
        for net, b, e in tiles:
            assert starts[net] <= b < e <= starts[net + 1]
            assert e - b <= block - 4
            covered[b:e] += 1
        np.testing.assert_array_equal(covered, 1)
    finally:
        u.close()


def test_spring_incidence_lists_every_end_in_order(hu):
    """General topology (cross-links): each bead lists its springs in
    ascending index, each spring appears once at each of its two ends."""
    from test_gpu_parity import _crosslinked
    m = _crosslinked().normalised()
    u = Upload(hu, m, chain=False)
    try:
        assert u.rc == 0, u.err
        off = np.zeros(u.nb + 1, np.int32)
        ent = np.zeros(2 * u.ns, np.int32)
        hu.hu_spring_incidence(u.h, off.ctypes.data_as(C.c_void_p), ent.ctypes.data_as(C.c_void_p))
        ends = u.springs()
        seen = np.zeros((u.ns, 2), np.int32)
        for i in range(u.nb):
            row = ent[off[i]:off[i + 1]]
            assert np.all(np.diff(row >> 1) >= 0)
            for x in row:
                s_, end = x >> 1, x & 1
                assert ends[s_, end] == i
                seen[s_, end] += 1
        np.testing.assert_array_equal(seen, 1)
    finally:
        u.close()


@pytest.mark.parametrize("which", ["tensile", "plain", "multitype", "dense"])
def test_derived_settings_and_pair_table_match_the_oracle(hu, oracle_built, which):
    """The engine's host precompute -- time-step constants, damping sign,
    cut-off, grid size and cell step, half box, the pair coefficients (LJ
    force shift, st remap) -- equals the oracle's restatement of
    SimulationManager's, bit for bit."""
    import pyoracle as po
    from fibrenet_b200 import generate as g
    if which == "tensile":
        m = small_tensile(13)
    elif which == "plain":
        m = g.plain_network(seed=1, fibres=20, beads=10, box=(20.0, 20.0, 6.0), z_range=(1.0, 5.0))
    elif which == "dense":
        m = g.dense_mat(seed=2, fibres=40, beads=10, box=(12.0, 12.0, 12.0))
    else:
        m = _multitype()
    m = m.normalised()
    u = Upload(hu, m)
    try:
        assert u.rc == 0, u.err
        mine = np.zeros(20)
        hu.hu_net(u.h, 0, mine.ctypes.data_as(C.c_void_p))
        c6 = np.zeros((m.n_types * (m.n_types + 1) // 2, 6)); kinds = np.zeros(len(c6), np.int32)
        hu.hu_pairs(u.h, 0, c6.ctypes.data_as(C.c_void_p), kinds.ctypes.data_as(C.c_void_p))
    finally:
        u.close()
    o = po.OracleSim(m, po.MODE_REF)
    np.testing.assert_array_equal(mine, o.derived())
    oc6, okinds = o.pairs()
    np.testing.assert_array_equal(kinds, okinds)
    np.testing.assert_array_equal(c6, oc6)


def _multitype():
    """Three bead types with one lj, one hs and one st pair among them."""
    from fibrenet_b200 import generate as g
    from fibrenet_b200.model import PAIR_HS, PAIR_LJ, PAIR_ST
    m = g.plain_network(seed=3, fibres=12, beads=8, box=(16.0, 16.0, 6.0), z_range=(1.0, 5.0)).normalised().copy()
    m.type = (np.arange(m.n_beads) % 3).astype(np.int32)
    m.type_names = ["A", "B", "C"]
    kinds = [PAIR_LJ, PAIR_HS, PAIR_ST, PAIR_LJ, PAIR_HS, PAIR_ST]
    raw = [[1.0, 1.0, 2.5, 0.0], [50.0, 0.0, 0.0, 0.0], [1.0, 20.0, 1.5, 5.0],
           [0.9, 0.5, 2.2, 0.0], [30.0, 0.0, 0.0, 0.0], [0.8, 10.0, 1.2, 3.0]]
    m.pair_kind = np.array(kinds, np.int32)
    m.pair_raw = np.array(raw, np.float64).reshape(-1)
    return m


def test_modifications_reach_the_chain_records(hu):
    """fn_set_springs / fn_set_angles / fn_set_mass (the reference's
    modif_spring and modif_bead, SimulationManager.cpp:189-636): values given
    in file order land on the right beads of the chain records and of the
    image positions' 1/mass."""
    m = small_tensile(14).normalised()
    u = Upload(hu, m)
    try:
        assert u.rc == 0, u.err
        rng = np.random.default_rng(5)
        rest = rng.uniform(0.5, 1.5, m.n_springs)
        k = rng.uniform(10, 200, m.n_springs)
        theta0 = rng.uniform(2.5, 3.1, m.n_angles)
        ka = rng.uniform(1, 20, m.n_angles)
        mass = rng.uniform(0.5, 2.0, m.n_beads)
        mass[::7] = 0.0
        P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        assert hu.fn_set_springs(u.h, P(rest), P(k), None, None) == 0
        assert hu.fn_set_angles(u.h, P(theta0), P(ka)) == 0
        assert hu.fn_set_mass(u.h, P(mass)) == 0
        sp4 = np.zeros((u.nb, 4), np.float32)
        an2 = np.zeros((u.nb, 2), np.float32)
        hu.hu_chain_records(u.h, P(sp4), P(an2))
        perm = u.perm()
        inv = np.empty_like(perm)
        inv[perm] = np.arange(len(perm))
        lower = np.minimum(inv[m.s_p1], inv[m.s_p2])
        np.testing.assert_array_equal(sp4[lower, 0], rest.astype(np.float32))
        np.testing.assert_array_equal(sp4[lower, 1], k.astype(np.float32))
        np.testing.assert_array_equal(sp4[lower, 2], m.s_c1.astype(np.float32))
        centre = inv[m.a_b2]
        np.testing.assert_array_equal(an2[centre, 0], theta0.astype(np.float32))
        np.testing.assert_array_equal(an2[centre, 1], ka.astype(np.float32))
        _, img = u.beads()
        want = np.where(mass > 0, 1.0 / np.where(mass > 0, mass, 1.0), 0.0)
        np.testing.assert_array_equal(img[:, 3], want[perm])
    finally:
        u.close()


@pytest.mark.parametrize("chain", [True, False])
def test_status_round_trip(hu, chain):
    """Spring and angle statuses set in file order come back unchanged, both
    from the chain form's per-bead status bits and from the per-bond arrays
    of the incidence path; every upload starts with all bonds alive."""
    m = small_tensile(15).normalised()
    u = Upload(hu, m, chain=chain)
    try:
        assert u.rc == 0, u.err
        assert hu.hu_chain(u.h) == int(chain)
        P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        s0 = np.zeros(m.n_springs, np.int32); a0 = np.zeros(m.n_angles, np.int32)
        assert hu.fn_download_status(u.h, P(s0), P(a0)) == 0
        assert s0.all() and a0.all()
        rng = np.random.default_rng(6)
        s1 = (rng.random(m.n_springs) < 0.7).astype(np.int32)
        a1 = (rng.random(m.n_angles) < 0.6).astype(np.int32)
        assert hu.fn_set_status(u.h, P(s1), P(a1)) == 0
        s2 = np.zeros_like(s1); a2 = np.zeros_like(a1)
        assert hu.fn_download_status(u.h, P(s2), P(a2)) == 0
        np.testing.assert_array_equal(s2, s1)
        np.testing.assert_array_equal(a2, a1)
    finally:
        u.close()
