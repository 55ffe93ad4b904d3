"""ctypes wrapper of liboracle.so — TEST INFRASTRUCTURE ONLY.

The CPU restatement of the reference's layout step (see oracle.cpp for the
reference file:line each function follows). Imported only by tests/, by
__graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


class Fa2Settings(ctypes.Structure):
    """Fa2BhSettings (fa2_bh.rs:84-119)."""
    _fields_ = [("gravity", ctypes.c_float), ("strong_gravity", ctypes.c_int32),
                ("scaling_ratio", ctypes.c_float), ("edge_weight_influence", ctypes.c_float),
                ("jitter_tolerance", ctypes.c_float), ("lin_log_mode", ctypes.c_int32),
                ("prevent_overlap", ctypes.c_int32), ("time_step", ctypes.c_float),
                ("theta", ctypes.c_float), ("max_displacement", ctypes.c_float)]


FA2_DEFAULTS = dict(gravity=1.0, strong_gravity=False, scaling_ratio=2.0, edge_weight_influence=1.0,
                    jitter_tolerance=1.0, lin_log_mode=False, prevent_overlap=False, time_step=1.0, theta=0.7,
                    max_displacement=10.0)

SGD_DEFAULTS = dict(n_pivots=50, sweeps_per_step=1, eta_max=1.0, eta_min=0.01, n_anneal_steps=30,
                    seed=0x5EEDC0DE12345678)

_SIG = {
    "orc_octree_build": (ctypes.c_uint32, [ctypes.c_uint32, _f32p, _f32p, ctypes.c_uint32, _vp, ctypes.c_uint32,
                                           _u32p]),
    "orc_octree_walk_all": (None, [_vp, ctypes.c_uint32, ctypes.c_uint32, _f32p, _f32p, ctypes.c_float,
                                   ctypes.c_float, _f32p]),
    "orc_fa2_create": (_vp, [ctypes.c_uint32, _u32p, _u32p, _f32p, ctypes.POINTER(Fa2Settings), ctypes.c_int]),
    "orc_fa2_destroy": (None, [_vp]),
    "orc_fa2_set_tree_capacity": (None, [_vp, ctypes.c_uint32]),
    "orc_fa2_step": (None, [_vp, ctypes.c_int]),
    "orc_fa2_force_pass": (None, [_vp, ctypes.c_int]),
    "orc_fa2_get": (None, [_vp, _f32p, _f32p, _f32p, _f32p, _f32p, _u32p]),
    "orc_fa2_counts": (None, [_vp, _u64p]),
    "orc_fa2_set_state": (None, [_vp, _f32p, _f32p, ctypes.c_float, ctypes.c_float]),
    "orc_fa2_attraction": (ctypes.c_uint64, [_vp, _u32p, _u32p]),
    "orc_fa2_attraction_scan": (None, [_vp, ctypes.c_uint32, _f32p]),
    "orc_fa2_exact_forces_f64": (None, [_vp, _f64p]),
    "orc_adaptive_speed_update": (ctypes.c_float, [_f32p, _f32p, ctypes.c_uint32, ctypes.c_float, _f32p,
                                                   ctypes.c_uint64]),
    "orc_bfs": (None, [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p]),
    "orc_sgd_create": (_vp, [ctypes.c_uint32, _u32p, _u32p, _f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                             ctypes.c_float, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int]),
    "orc_sgd_destroy": (None, [_vp]),
    "orc_sgd_pivots": (ctypes.c_uint32, [_vp, _u32p, _u32p]),
    "orc_sgd_step": (None, [_vp, ctypes.c_int]),
    "orc_sgd_positions": (None, [_vp, _f32p]),
    "orc_sgd_set_positions": (None, [_vp, _f32p]),
    "orc_sgd_set_scatter_batches": (None, [_vp, ctypes.c_uint32]),
    "orc_anneal_eta": (ctypes.c_float, [ctypes.c_uint64, ctypes.c_float, ctypes.c_float, ctypes.c_uint32]),
    "orc_scale_normalized_stress": (ctypes.c_float, [_f32p, _u32p, _u32p, _f32p, ctypes.c_uint64]),
    "orc_stress": (ctypes.c_float, [_f32p, _u32p, _u32p, _f32p, ctypes.c_uint64]),
    "orc_edge_length_cv": (ctypes.c_float, [_f32p, _u32p, _u32p, ctypes.c_uint64]),
    "orc_num_threads": (ctypes.c_int, []),
    "orc_mpnn_num_params": (ctypes.c_uint32, []),
    "orc_mpnn_features": (None, [ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p, _u32p, ctypes.c_uint64,
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, _f32p]),
    "orc_mpnn_grad": (None, [ctypes.c_uint32, ctypes.c_uint32, _u32p, _u32p, _u32p, _f32p, _f32p, ctypes.c_int,
                             _f32p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                             ctypes.c_uint32, ctypes.c_int, _f64p, _f64p, _f64p, _f64p]),
    "orc_f32_to_f16": (ctypes.c_uint16, [ctypes.c_float]),
    "orc_f16_to_f32": (ctypes.c_float, [ctypes.c_uint16]),
    "orc_f32_to_f16_array": (None, [ctypes.c_uint64, _f32p, ctypes.POINTER(ctypes.c_uint16)]),
    "orc_frame_encode_f16": (ctypes.c_int, [ctypes.c_uint64, _f32p, _f32p, ctypes.POINTER(ctypes.c_uint16)]),
    "orc_coarsen": (_vp, [ctypes.c_uint32, _u32p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    "orc_cascade_levels": (ctypes.c_uint32, [_vp]),
    "orc_cascade_level": (ctypes.c_uint32, [_vp, ctypes.c_uint32, _u64p]),
    "orc_cascade_get": (None, [_vp, ctypes.c_uint32, _u32p, _u32p]),
    "orc_cascade_free": (None, [_vp]),
    "orc_prolong": (None, [_f32p, _u32p, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32, _f32p]),
    "orc_fold_up": (None, [_vp, _f32p, _f32p]),
    "orc_level_csr": (ctypes.c_uint64, [ctypes.c_uint32, _u32p, ctypes.c_uint64, _u32p, _u32p]),
    "orc_sweeps_for_level": (ctypes.c_uint32, [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32]),
    "orc_gen_rmat_pairs": (ctypes.c_uint64, [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_uint64, _u32p]),
    "orc_csr_from_pairs": (ctypes.c_uint64, [ctypes.c_uint32, _u32p, ctypes.c_uint64, _u32p, _u32p]),
    "orc_seed_uniform": (None, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _f32p]),
}

_LIB = None


def build() -> Path:
    """Compile liboracle.so from oracle.cpp if it is missing or stale."""
    srcs = [HERE / "oracle.cpp", HERE / "mpnn.cpp", HERE / "frames.cpp", HERE / "multilevel.cpp",
            HERE / "graphgen.cpp"]
    if not LIB_PATH.exists() or any(LIB_PATH.stat().st_mtime < s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _LIB
    if _LIB is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIG.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t)


def _u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def fa2_settings(**kw) -> Fa2Settings:
    d = dict(FA2_DEFAULTS)
    d.update(kw)
    return Fa2Settings(d["gravity"], int(d["strong_gravity"]), d["scaling_ratio"], d["edge_weight_influence"],
                       d["jitter_tolerance"], int(d["lin_log_mode"]), int(d["prevent_overlap"]), d["time_step"],
                       d["theta"], d["max_displacement"])


class Fa2:
    """The reference FA2 engine (bh=True: fa2-bh, bh=False: fa2-brute) on the CPU."""

    def __init__(self, csr, positions, bh: bool = True, **settings):
        self.L = lib()
        self.n = csr.n_nodes
        self._off = _u32(csr.offsets)
        self._nb = _u32(csr.neighbors) if len(csr.neighbors) else np.zeros(1, np.uint32)
        pos = _f32(positions).reshape(-1)
        assert len(pos) == 3 * self.n
        self._s = fa2_settings(**settings)
        self.h = self.L.orc_fa2_create(self.n, _p(self._off, _u32p), _p(self._nb, _u32p), _p(pos, _f32p),
                                       ctypes.byref(self._s), 1 if bh else 0)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_fa2_destroy(self.h)
            self.h = None

    def set_tree_capacity(self, cap: int):
        self.L.orc_fa2_set_tree_capacity(self.h, cap)

    def step(self, threads: int = 0):
        self.L.orc_fa2_step(self.h, threads)

    def force_pass(self, threads: int = 0):
        self.L.orc_fa2_force_pass(self.h, threads)

    def get(self) -> dict:
        n = self.n
        pos = np.zeros(3 * n, np.float32)
        f = np.zeros(3 * n, np.float32)
        of = np.zeros(3 * n, np.float32)
        st = np.zeros(2 * n, np.float32)
        sp = np.zeros(2, np.float32)
        info = np.zeros(4, np.uint32)
        self.L.orc_fa2_get(self.h, _p(pos, _f32p), _p(f, _f32p), _p(of, _f32p), _p(st, _f32p), _p(sp, _f32p),
                           _p(info, _u32p))
        cnt = np.zeros(2, np.uint64)
        self.L.orc_fa2_counts(self.h, _p(cnt, _u64p))
        return dict(pos=pos, force=f, old_force=of, stats=st, speed=float(sp[0]), speed_eff=float(sp[1]),
                    n_octree=int(info[0]), n_inserted=int(info[1]), n_inter=int(cnt[0]), n_open=int(cnt[1]))

    def set_state(self, pos=None, old_force=None, speed=1.0, speed_eff=1.0):
        p = _f32(pos) if pos is not None else None
        o = _f32(old_force) if old_force is not None else None
        self.L.orc_fa2_set_state(self.h, _p(p, _f32p) if p is not None else None,
                                 _p(o, _f32p) if o is not None else None, speed, speed_eff)

    def attraction(self):
        m = self.L.orc_fa2_attraction(self.h, None, None)
        off = np.zeros(self.n + 1, np.uint32)
        nb = np.zeros(max(m, 1), np.uint32)
        self.L.orc_fa2_attraction(self.h, _p(off, _u32p), _p(nb, _u32p))
        return off, nb[:m]

    def attraction_scan(self, i: int) -> np.ndarray:
        f = np.zeros(3, np.float32)
        self.L.orc_fa2_attraction_scan(self.h, i, _p(f, _f32p))
        return f

    def exact_forces_f64(self) -> np.ndarray:
        out = np.zeros(3 * self.n, np.float64)
        self.L.orc_fa2_exact_forces_f64(self.h, _p(out, _f64p))
        return out


OCT_DTYPE = np.dtype([("pos_size", "<f4", 4), ("com_mass", "<f4", 4), ("meta", "<u4", 4)])


def octree_build(pos4, mass, max_nodes: int):
    """OctreeBuild::rebuild (fa2_bh.rs:761-827): (nodes, used, inserted)."""
    L = lib()
    p = _f32(pos4).reshape(-1)
    m = _f32(mass)
    n = len(m)
    cap = max_nodes
    nodes = np.zeros(max(cap, 1), dtype=OCT_DTYPE)
    ins = np.zeros(1, np.uint32)
    used = L.orc_octree_build(n, _p(p, _f32p), _p(m, _f32p), max_nodes, nodes.ctypes.data, cap, _p(ins, _u32p))
    return nodes[:used], int(used), int(ins[0])


def octree_walk_all(nodes, pos4, deg_plus1, scaling: float, theta: float) -> np.ndarray:
    L = lib()
    p = _f32(pos4).reshape(-1)
    d = _f32(deg_plus1)
    n = len(d)
    nd = np.ascontiguousarray(nodes)
    out = np.zeros(3 * n, np.float32)
    L.orc_octree_walk_all(nd.ctypes.data, len(nd), n, _p(p, _f32p), _p(d, _f32p), scaling, theta, _p(out, _f32p))
    return out


class AdaptiveSpeed:
    """fa2_speed.rs:24-100."""

    def __init__(self):
        self.speed = np.array([1.0], np.float32)
        self.eff = np.array([1.0], np.float32)

    def update(self, n_nodes: int, jitter_tolerance: float, stats) -> float:
        s = _f32(stats).reshape(-1)
        if len(s) == 0:
            s = np.zeros(2, np.float32)
            n_pairs = 0
        else:
            n_pairs = len(s) // 2
        return float(lib().orc_adaptive_speed_update(_p(self.speed, _f32p), _p(self.eff, _f32p), n_nodes,
                                                     jitter_tolerance, _p(s, _f32p), n_pairs))

    @property
    def speed_efficiency(self) -> float:
        return float(self.eff[0])


def bfs(csr, src: int) -> np.ndarray:
    out = np.zeros(max(csr.n_nodes, 1), np.uint32)
    nb = _u32(csr.neighbors) if len(csr.neighbors) else np.zeros(1, np.uint32)
    lib().orc_bfs(csr.n_nodes, _p(_u32(csr.offsets), _u32p), _p(nb, _u32p), src, _p(out, _u32p))
    return out[:csr.n_nodes]


class Sgd:
    """sgd_stress.rs (mode 0: CPU s_gd2) / sgd_stress_gpu.rs + sgd_stress.wgsl
    (mode 1: Jacobi) / the device "sgd-stress" engine's batched fixed-point
    scatter (mode 2; `scatter_batches` as the engine's setting)."""

    def __init__(self, csr, positions, mode: int = 0, scatter_batches: int = 0, **settings):
        self.L = lib()
        s = dict(SGD_DEFAULTS)
        s.update(settings)
        self.n = csr.n_nodes
        off = _u32(csr.offsets)
        nb = _u32(csr.neighbors) if len(csr.neighbors) else np.zeros(1, np.uint32)
        pos = _f32(positions).reshape(-1)
        self.h = self.L.orc_sgd_create(self.n, _p(off, _u32p), _p(nb, _u32p), _p(pos, _f32p), s["n_pivots"],
                                       s["sweeps_per_step"], s["eta_max"], s["eta_min"], s["n_anneal_steps"],
                                       s["seed"], mode)
        if scatter_batches:
            self.L.orc_sgd_set_scatter_batches(self.h, scatter_batches)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_sgd_destroy(self.h)
            self.h = None

    def pivots(self):
        k = self.L.orc_sgd_pivots(self.h, None, None)
        piv = np.zeros(max(k, 1), np.uint32)
        dist = np.zeros(max(k * self.n, 1), np.uint32)
        self.L.orc_sgd_pivots(self.h, _p(piv, _u32p), _p(dist, _u32p))
        return piv[:k], dist[:k * self.n].reshape(k, self.n)

    def step(self, threads: int = 0) -> np.ndarray:
        self.L.orc_sgd_step(self.h, threads)
        return self.positions()

    def positions(self) -> np.ndarray:
        out = np.zeros(max(3 * self.n, 1), np.float32)
        self.L.orc_sgd_positions(self.h, _p(out, _f32p))
        return out[:3 * self.n]

    def set_positions(self, xyz):
        p = _f32(xyz)
        self.L.orc_sgd_set_positions(self.h, _p(p, _f32p))


def anneal_eta(sweep: int, eta_max: float, eta_min: float, n_anneal: int) -> float:
    return float(lib().orc_anneal_eta(sweep, eta_max, eta_min, n_anneal))


def _terms(terms):
    t = list(terms)
    ti = _u32([a for a, _, _ in t])
    tj = _u32([b for _, b, _ in t])
    td = _f32([d for _, _, d in t])
    return ti, tj, td


def scale_normalized_stress(pos, terms) -> float:
    """metrics.rs:31-59."""
    ti, tj, td = _terms(terms)
    p = _f32(pos)
    if len(ti) == 0:
        return 0.0
    return float(lib().orc_scale_normalized_stress(_p(p, _f32p), _p(ti, _u32p), _p(tj, _u32p), _p(td, _f32p), len(ti)))


def stress(pos, terms) -> float:
    """metrics.rs:64-76."""
    ti, tj, td = _terms(terms)
    p = _f32(pos)
    if len(ti) == 0:
        return 0.0
    return float(lib().orc_stress(_p(p, _f32p), _p(ti, _u32p), _p(tj, _u32p), _p(td, _f32p), len(ti)))


def edge_length_cv(pos, edges) -> float:
    """metrics.rs:150-164."""
    e = np.asarray(list(edges), dtype=np.uint32).reshape(-1, 2)
    if len(e) < 2:
        return 0.0
    ei = _u32(e[:, 0])
    ej = _u32(e[:, 1])
    p = _f32(pos)
    return float(lib().orc_edge_length_cv(_p(p, _f32p), _p(ei, _u32p), _p(ej, _u32p), len(ei)))


def all_pairs_terms(csr):
    """(i, j, d_ij) for every reachable pair i<j (BFS from every node)."""
    out = []
    for i in range(csr.n_nodes):
        d = bfs(csr, i)
        for j in range(i + 1, csr.n_nodes):
            if d[j] != 0xFFFFFFFF and d[j] != 0:
                out.append((i, j, float(d[j])))
    return out


def pivot_terms(pivots, dist):
    """(node, pivot, d) terms of a pivot distance matrix (k x n)."""
    out = []
    k, n = dist.shape
    for t in range(k):
        j = int(pivots[t])
        row = dist[t]
        for i in range(n):
            d = int(row[i])
            if i != j and d != 0xFFFFFFFF and d != 0:
                out.append((i, j, float(d)))
    return out


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ------------------------------------------------------- learned warm start --
class GraphSet:
    """Graphs joined into one global CSR (ids offset by each graph's first node)."""

    def __init__(self, graphs):
        graphs = list(graphs)
        sizes = [g.n_nodes for g in graphs]
        self.G = len(graphs)
        self.go = _u32(np.concatenate([[0], np.cumsum(sizes)]))
        self.n = int(self.go[-1])
        offs, nbs, e0 = [], [], 0
        for g, b in zip(graphs, self.go[:-1]):
            offs.append(np.asarray(g.offsets[:-1], np.int64) + e0)
            nbs.append(np.asarray(g.neighbors, np.int64) + int(b))
            e0 += int(g.offsets[-1])
        self.off = _u32(np.concatenate(offs + [[e0]]))
        self.nbr = _u32(np.concatenate(nbs)) if e0 else np.zeros(1, np.uint32)


def mpnn_num_params() -> int:
    return int(lib().orc_mpnn_num_params())


def mpnn_features(gs: GraphSet, seed: int, smooth_steps: int = 64, cheb_steps: int = 64,
                  cheb_b: float = 0.993) -> np.ndarray:
    """Node features (n x 32, bf16 values) as the device computes them."""
    X = np.zeros((gs.n, 32), np.float32)
    lib().orc_mpnn_features(gs.n, gs.G, _p(gs.go, _u32p), _p(gs.off, _u32p), _p(gs.nbr, _u32p), seed,
                            smooth_steps, cheb_steps, cheb_b, _p(X, _f32p))
    return X


def mpnn_grad(gs: GraphSet, X, T, dim: int, theta, partners: int, seed: int, pair_step: int, g0: int, g1: int,
              emulate: bool = True, upstream=None):
    """f64 forward + loss + backward on graphs [g0, g1): (loss, Y nb x 4, grad).
    T: n x 4 targets; upstream (nb x 4) replaces the stress loss by <upstream, Y>."""
    X = _f32(X).reshape(gs.n, 32)
    T = _f32(T).reshape(gs.n, 4)
    theta = _f32(theta)
    nb = int(gs.go[g1] - gs.go[g0])
    Y = np.zeros((nb, 4), np.float64)
    grad = np.zeros(mpnn_num_params(), np.float64)
    loss = ctypes.c_double()
    up = None if upstream is None else np.ascontiguousarray(np.asarray(upstream, np.float64).reshape(nb, 4))
    lib().orc_mpnn_grad(gs.n, gs.G, _p(gs.go, _u32p), _p(gs.off, _u32p), _p(gs.nbr, _u32p), _p(X, _f32p),
                        _p(T, _f32p), dim, _p(theta, _f32p), partners, seed, pair_step, g0, g1, int(emulate),
                        None if up is None else _p(up, _f64p), ctypes.byref(loss), _p(Y, _f64p), _p(grad, _f64p))
    return loss.value, Y, grad


# ---------------------------------------------------------------- frames --
def f32_to_f16_bits(x) -> np.ndarray:
    """binary16 round-to-nearest-even bits of each f32 (oracle/frames.cpp)."""
    x = _f32(x).reshape(-1)
    out = np.zeros(len(x), np.uint16)
    lib().orc_f32_to_f16_array(len(x), _p(x, _f32p), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)))
    return out


class FrameEncoder:
    """The binary16 delta-frame encoder restated (oracle/frames.cpp)."""

    def __init__(self, n_nodes: int):
        self.rec = np.zeros(3 * n_nodes, np.float32)
        self.started = False

    def encode(self, xyz):
        """Returns ("f32", payload f32 array) or ("f16", payload u16 array)."""
        x = _f32(xyz).reshape(-1)
        if not self.started:
            self.rec[:] = x
            self.started = True
            return "f32", x.copy()
        out = np.zeros(len(x), np.uint16)
        key = lib().orc_frame_encode_f16(len(x), _p(x, _f32p), _p(self.rec, _f32p),
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)))
        return ("f32", x.copy()) if key else ("f16", out)


# ------------------------------------------------------------ multilevel --
def csr_edges(csr) -> np.ndarray:
    """The multilevel wrapper's flat edge list: (v, u) with v < u in CSR order
    (engines/multilevel.rs:372-386)."""
    deg = np.diff(csr.offsets.astype(np.int64))
    src = np.repeat(np.arange(csr.n_nodes, dtype=np.uint32), deg)
    m = src < csr.neighbors
    return np.stack([src[m], csr.neighbors[m]], axis=1).reshape(-1).astype(np.uint32)


class Cascade:
    """coarsen (coarsen.rs:52-90): levels as (n, flat edges, parent_map)."""

    def __init__(self, n: int, edges, max_levels: int = 6, target_size: int = 500):
        e = _u32(edges)
        h = lib().orc_coarsen(n, _p(e, _u32p), len(e), max_levels, target_size)
        self._h = h
        self.levels = []
        for l in range(lib().orc_cascade_levels(h)):
            w = ctypes.c_uint64(0)
            nl = lib().orc_cascade_level(h, l, ctypes.byref(w))
            ed = np.zeros(w.value, np.uint32)
            pm = np.zeros(self.levels[-1][0] if l else 0, np.uint32)
            lib().orc_cascade_get(h, l, _p(ed, _u32p), _p(pm, _u32p))
            self.levels.append((int(nl), ed, pm))

    def fold_up(self, fine_xyz) -> np.ndarray:
        x = _f32(fine_xyz).reshape(-1)
        out = np.zeros(3 * self.levels[-1][0], np.float32)
        lib().orc_fold_up(self._h, _p(x, _f32p), _p(out, _f32p))
        return out

    def __del__(self):
        try:
            lib().orc_cascade_free(self._h)
        except Exception:
            pass


def prolong(parent_xyz, parent_map, n_child: int, jitter: float, seed: int) -> np.ndarray:
    """prolong (coarsen.rs:157-183)."""
    px, pm = _f32(parent_xyz).reshape(-1), _u32(parent_map)
    out = np.zeros(3 * n_child, np.float32)
    lib().orc_prolong(_p(px, _f32p), _p(pm, _u32p), n_child, jitter, seed & 0xFFFFFFFF, _p(out, _f32p))
    return out


def level_csr(n: int, edges):
    """level_csr (multilevel.rs:259-294) as (offsets, neighbors)."""
    e = _u32(edges)
    off = np.zeros(n + 1, np.uint32)
    nb = np.zeros(max(len(e), 1), np.uint32)
    m = lib().orc_level_csr(n, _p(e, _u32p), len(e), _p(off, _u32p), _p(nb, _u32p))
    return off, nb[:m].copy()


def sweeps_for_level(schedule: str, level: int, base: int) -> int:
    return int(lib().orc_sweeps_for_level({"uniform": 0, "linear": 1, "geometric": 2}[schedule], level, base))


class Graph:
    """A CSR graph (offsets[n + 1], neighbors) built on the oracle side."""

    def __init__(self, n_nodes: int, offsets: np.ndarray, neighbors: np.ndarray):
        self.n_nodes = n_nodes
        self.offsets = offsets
        self.neighbors = neighbors


def csr_from_pairs(n: int, pairs) -> Graph:
    """Symmetric CSR, rows sorted and deduplicated (stability.rs:86-110)."""
    pr = _u32(np.asarray(pairs, np.uint32).reshape(-1))
    cnt = len(pr) // 2
    off = np.zeros(n + 1, np.uint32)
    nb = np.zeros(max(2 * cnt, 1), np.uint32)
    m = lib().orc_csr_from_pairs(n, _p(pr, _u32p) if cnt else None, cnt, _p(off, _u32p), _p(nb, _u32p))
    return Graph(n, off, nb[:m].copy())


def gen_rmat(scale: int, n_edges: int, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 1) -> Graph:
    """R-MAT graph of 2^scale nodes and n_edges distinct undirected pairs (graphgen.cpp)."""
    pairs = np.zeros(2 * n_edges, np.uint32)
    got = lib().orc_gen_rmat_pairs(scale, n_edges, a, b, c, seed, _p(pairs, _u32p))
    if got != n_edges:
        raise ValueError("R-MAT arguments out of range")
    return csr_from_pairs(1 << scale, pairs)


def seed_uniform(n: int, dim: int, seed: int) -> np.ndarray:
    """Uniform [-1, 1]^dim seed, 3 floats per node (graphgen.cpp)."""
    out = np.zeros(3 * n, np.float32)
    lib().orc_seed_uniform(n, dim, seed, _p(out, _f32p))
    return out
