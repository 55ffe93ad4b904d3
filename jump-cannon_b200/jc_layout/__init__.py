"""Python bindings for libjc_layout.so (the B200 layout-step engine).

The C ABI (include/jc_layout.h) mirrors the reference's Rust trait
`LayoutEngine` (crates/graph-compute/src/engines/mod.rs:383-444); this module
wraps it with numpy arrays so tests and the benchmark read like the
reference's own engine tests:

    eng = LayoutEngine("fa2-bh")
    eng.set_params({"theta": 0.8})
    eng.init(csr, positions)
    out = eng.step()          # interleaved x, y, z (3 n floats)

Every call goes through the shared library; there is no Python or CPU
fallback. A missing library raises at import of `lib()`.
"""
from __future__ import annotations

import ctypes
import os
import json
import time
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

PKG_DIR = Path(__file__).resolve().parent.parent
# JC_LAYOUT_LIB names another build of the library (A/B measurements).
LIB_PATH = Path(os.environ["JC_LAYOUT_LIB"]) if os.environ.get("JC_LAYOUT_LIB") else PKG_DIR / "libjc_layout.so"

JC_OK = 0
JC_ERR_ARG = 1
JC_ERR_CUDA = 2
JC_ERR_CAPACITY = 3
JC_ERR_DEVICE_TIMEOUT = 4
JC_ERR_NONFINITE = 5
JC_ERR_STATE = 6
JC_ERR_UNKNOWN_ENGINE = 7
JC_ERR_PARAMS = 8
JC_ERR_BOUNDS = 9

JC_WARN_REF_CAPACITY = 1
JC_WARN_DEPTH_CAP = 2
JC_WARN_NONFINITE = 4

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f32p = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


class JcDescriptor(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_char_p),
        ("kind", ctypes.c_int32),
        ("display_name", ctypes.c_char_p),
        ("description", ctypes.c_char_p),
        ("needs_edges", ctypes.c_int32),
        ("needs_cpu_positions", ctypes.c_int32),
        ("needs_gpu_positions_buffer", ctypes.c_int32),
    ]


_SIGNATURES = {
    "jc_engine_count": (ctypes.c_uint32, []),
    "jc_engine_id_at": (ctypes.c_char_p, [ctypes.c_uint32]),
    "jc_engine_create": (ctypes.c_int32, [ctypes.c_char_p, ctypes.POINTER(_vp)]),
    "jc_engine_destroy": (None, [_vp]),
    "jc_engine_descriptor": (ctypes.c_int32, [_vp, ctypes.POINTER(JcDescriptor)]),
    "jc_engine_set_params": (ctypes.c_int32, [_vp, ctypes.c_char_p]),
    "jc_engine_init": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint64, _f32p]),
    "jc_engine_reinit": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint64, _f32p]),
    "jc_engine_step": (ctypes.c_int32, [_vp, _f32p]),
    "jc_engine_step_many": (ctypes.c_int32, [_vp, ctypes.c_uint32, _f32p]),
    "jc_engine_apply_halo": (ctypes.c_int32, [_vp, ctypes.c_uint64, ctypes.c_uint32, _u32p, _f32p, ctypes.c_uint32]),
    "jc_engine_is_halted": (ctypes.c_int32, [_vp]),
    "jc_engine_last_error": (ctypes.c_char_p, [_vp]),
    "jc_engine_save_state": (ctypes.c_int32, [_vp, _vp, ctypes.c_uint64, _u64p]),
    "jc_engine_load_state": (ctypes.c_int32, [_vp, _vp, ctypes.c_uint64]),
    "jc_engine_positions": (ctypes.c_int32, [_vp, _f32p]),
    "jc_engine_forces": (ctypes.c_int32, [_vp, _f32p, _f32p]),
    "jc_engine_speed": (ctypes.c_int32, [_vp, _f32p, _f32p]),
    "jc_engine_status_bits": (ctypes.c_uint32, [_vp]),
    "jc_engine_tree_info": (ctypes.c_int32, [_vp, _u32p]),
    "jc_engine_walk_counts": (ctypes.c_int32, [_vp, _u64p]),
    "jc_engine_time_steps": (ctypes.c_int32, [_vp, ctypes.c_uint32, _f32p, _f32p]),
    "jc_engine_stress": (ctypes.c_int32, [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "jc_engine_pivots": (ctypes.c_int32, [_vp, _u32p, _u32p, _u32p]),
    "jc_engine_init_batch": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _u32p, _u32p, _f32p]),
    "jc_engine_graph_speed": (ctypes.c_int32, [_vp, ctypes.c_uint32, _f32p, _f32p]),
    "jc_engine_autotune": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _f32p]),
    "jc_engine_batch_schedule": (ctypes.c_int32, [_vp, _u32p, _f32p]),
    "jc_engine_launches_per_step": (ctypes.c_uint32, [_vp]),
    "jc_engine_output_nodes": (ctypes.c_uint32, [_vp]),
    "jc_gen_scale_free": (_vp, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]),
    "jc_csr_from_pairs": (_vp, [ctypes.c_uint32, _u32p, ctypes.c_uint64]),
    "jc_gen_path": (_vp, [ctypes.c_uint32]),
    "jc_gen_grid": (_vp, [ctypes.c_uint32, ctypes.c_uint32]),
    "jc_gen_rmat": (_vp, [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                          ctypes.c_uint64]),
    "jc_gen_watts_strogatz": (_vp, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64]),
    "jc_gen_rgg": (_vp, [ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64, _f32p]),
    "jc_csr_n_nodes": (ctypes.c_uint32, [_vp]),
    "jc_csr_n_neighbors": (ctypes.c_uint64, [_vp]),
    "jc_csr_offsets": (_u32p, [_vp]),
    "jc_csr_neighbors": (_u32p, [_vp]),
    "jc_csr_free": (None, [_vp]),
    "jc_seed_ball": (None, [ctypes.c_uint32, ctypes.c_uint64, _f32p]),
    "jc_seed_uniform": (None, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _f32p]),
    "jc_build_info": (ctypes.c_char_p, []),
    "jc_set_device": (ctypes.c_int32, [ctypes.c_int32]),
    "jc_selftest_sort_wait": (ctypes.c_int32, [_u32p, _f32p]),
    "jc_selftest_gemm_wait": (ctypes.c_int32, [_u32p, _f32p]),
}

class Fa2Params(ctypes.Structure):
    """jc_fa2_params (force-law subset of the fa2-bh settings)."""
    _fields_ = [("gravity", ctypes.c_float), ("strong_gravity", ctypes.c_int32), ("scaling_ratio", ctypes.c_float),
                ("edge_weight_influence", ctypes.c_float), ("lin_log_mode", ctypes.c_int32), ("theta", ctypes.c_float)]


_SIGNATURES["jc_fa2_bh_forces_noalloc"] = (ctypes.c_int32, [ctypes.c_uint32, _vp, _vp, _vp, ctypes.POINTER(Fa2Params),
                                                            _vp, _vp])

_SIGNATURES["jc_tc_gemm_bf16"] = (ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp, ctypes.c_int32,
                                                   _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                   _f32p])

_f64p = ctypes.POINTER(ctypes.c_double)
_SIGNATURES.update({
    "jc_batch_create": (ctypes.c_int32, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_vp)]),
    "jc_batch_destroy": (None, [_vp]),
    "jc_batch_last_error": (ctypes.c_char_p, [_vp]),
    "jc_batch_add_graph": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint64, _f32p, _u32p]),
    "jc_batch_bind": (ctypes.c_int32, [_vp]),
    "jc_batch_run": (ctypes.c_int32, [_vp, ctypes.c_uint32]),
    "jc_batch_graph_count": (ctypes.c_uint32, [_vp]),
    "jc_batch_positions": (ctypes.c_int32, [_vp, ctypes.c_uint32, _f32p]),
    "jc_batch_engine": (_vp, [_vp]),
})
_SIGNATURES.update({
    "jc_mpnn_create": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "jc_mpnn_destroy": (None, [_vp]),
    "jc_mpnn_last_error": (ctypes.c_char_p, [_vp]),
    "jc_mpnn_num_params": (ctypes.c_uint32, []),
    "jc_mpnn_set_params": (ctypes.c_int32, [_vp, ctypes.c_char_p]),
    "jc_mpnn_get_weights": (ctypes.c_int32, [_vp, _f32p]),
    "jc_mpnn_set_weights": (ctypes.c_int32, [_vp, _f32p]),
    "jc_mpnn_bind": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _u32p, _u32p, _f32p]),
    "jc_mpnn_batches": (ctypes.c_int32, [_vp, _u32p]),
    "jc_mpnn_features": (ctypes.c_int32, [_vp, _f32p]),
    "jc_mpnn_train": (ctypes.c_int32, [_vp, ctypes.c_uint32, _f32p]),
    "jc_mpnn_eval_loss": (ctypes.c_int32, [_vp, _f64p]),
    "jc_mpnn_grad": (ctypes.c_int32, [_vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _f32p, _f32p, _f32p]),
    "jc_mpnn_predict": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _u32p, _u32p, _f32p, _f32p]),
    "jc_mpnn_predict_stages": (ctypes.c_int32, [_vp, _f32p]),
    "jc_mpnn_warm_start": (ctypes.c_int32, [_vp, _vp, ctypes.c_uint32, _u32p, _u32p, _u32p, _f32p, _f32p,
                                            ctypes.POINTER(ctypes.c_uint8), _f32p]),
    "jc_mpnn_state_size": (ctypes.c_uint64, [_vp]),
    "jc_mpnn_save_state": (ctypes.c_int32, [_vp, _vp]),
    "jc_mpnn_load_state": (ctypes.c_int32, [_vp, _vp, ctypes.c_uint64]),
    "jc_eval_create": (ctypes.c_int32, [ctypes.c_uint32, _u32p, _u32p, _u32p, ctypes.c_uint32, ctypes.c_uint64,
                                        ctypes.POINTER(_vp)]),
    "jc_eval_destroy": (None, [_vp]),
    "jc_eval_last_error": (ctypes.c_char_p, [_vp]),
    "jc_eval_pivots": (ctypes.c_int32, [_vp, _u32p]),
    "jc_eval_layout": (ctypes.c_int32, [_vp, _f32p, _f64p, _f64p, _f64p]),
})

JC_FRAME_F32 = 0
JC_FRAME_F16_DELTA = 1


class JcFrame(ctypes.Structure):
    """jc_frame (one position frame message in library-owned page-locked memory)."""
    _fields_ = [("frame", ctypes.c_uint64), ("n_nodes", ctypes.c_uint32), ("encoding", ctypes.c_uint32),
                ("data", ctypes.c_void_p), ("bytes", ctypes.c_uint64), ("payload", ctypes.c_void_p),
                ("payload_bytes", ctypes.c_uint64)]


_SIGNATURES.update({
    "jc_engine_stream_open": (ctypes.c_int32, [_vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    "jc_engine_stream_step": (ctypes.c_int32, [_vp, ctypes.c_uint32]),
    "jc_engine_stream_next": (ctypes.c_int32, [_vp, ctypes.POINTER(JcFrame)]),
    "jc_engine_stream_close": (ctypes.c_int32, [_vp]),
    "jc_frame_decoder_create": (_vp, [ctypes.c_uint32]),
    "jc_frame_decoder_destroy": (None, [_vp]),
    "jc_frame_decode": (ctypes.c_int32, [_vp, _vp, ctypes.c_uint64, _f32p]),
    "jc_frame_decoder_last_error": (ctypes.c_char_p, [_vp]),
})

class JcPartitionView(ctypes.Structure):
    """jc_partition_view (one partition of a jc_partitions set)."""
    _fields_ = [("partition_id", ctypes.c_uint32), ("n_partitions", ctypes.c_uint32), ("n_local", ctypes.c_uint32),
                ("n_owned", ctypes.c_uint32), ("n_neighbors", ctypes.c_uint64), ("n_boundary", ctypes.c_uint32),
                ("offsets", _u32p), ("neighbors", _u32p), ("global_ids", _u32p), ("boundary", _u32p)]


_SIGNATURES.update({
    "jc_partition_csr": (ctypes.c_int32, [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint64, ctypes.c_uint32,
                                          ctypes.c_int32, ctypes.POINTER(_vp)]),
    "jc_partitions_free": (None, [_vp]),
    "jc_partitions_count": (ctypes.c_uint32, [_vp]),
    "jc_partitions_edge_cut": (ctypes.c_uint64, [_vp]),
    "jc_partitions_owner": (_u32p, [_vp]),
    "jc_partition_get": (ctypes.c_int32, [_vp, ctypes.c_uint32, ctypes.POINTER(JcPartitionView)]),
    "jc_engine_init_partitions": (ctypes.c_int32, [_vp, _vp, _f32p]),
    "jc_engine_partition_positions": (ctypes.c_int32, [_vp, _f32p]),
    "jc_engine_halo_delta": (ctypes.c_int32, [_vp, ctypes.c_uint32, _f32p, _u32p]),
})

_SIGNATURES.update({
    "jc_engine_level_info": (ctypes.c_int32, [_vp, _u32p, _u32p, _u32p]),
    "jc_engine_cascade_level": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _u64p, _u32p, _u32p]),
    "jc_coarsen": (ctypes.c_int32, [ctypes.c_uint32, _u32p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                    ctypes.POINTER(_vp)]),
    "jc_cascade_levels": (ctypes.c_uint32, [_vp]),
    "jc_cascade_get": (ctypes.c_int32, [_vp, ctypes.c_uint32, _u32p, _u64p, _u32p, _u32p]),
    "jc_cascade_free": (None, [_vp]),
})

_LIB: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    """Load libjc_layout.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python jump-cannon_b200/build.py`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


class JcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


# ---------------------------------------------------------------- graphs --
@dataclass
class Csr:
    """CsrGraph (crates/graph-compute/src/sim.rs:20-27)."""
    n_nodes: int
    offsets: np.ndarray
    neighbors: np.ndarray

    def pairs(self) -> np.ndarray:
        """Unique undirected (i<j) pairs as an (m, 2) array."""
        deg = np.diff(self.offsets.astype(np.int64))
        src = np.repeat(np.arange(self.n_nodes, dtype=np.uint32), deg)
        m = src < self.neighbors
        return np.stack([src[m], self.neighbors[m]], axis=1)

    def to_bin(self) -> bytes:
        """Little-endian binary CSR (sim.rs:53-58)."""
        hdr = np.array([self.n_nodes, len(self.neighbors)], dtype="<u4")
        return hdr.tobytes() + self.offsets.astype("<u4").tobytes() + self.neighbors.astype("<u4").tobytes()

    @staticmethod
    def from_bin(data: bytes) -> "Csr":
        if len(data) < 8:
            raise ValueError(f"CSR truncated: {len(data)} bytes < 8-byte header")
        n, m = np.frombuffer(data[:8], dtype="<u4")
        expect = 8 + 4 * (int(n) + 1) + 4 * int(m)
        if len(data) != expect:
            raise ValueError(f"CSR length mismatch: got {len(data)} bytes, expected {expect}")
        off = np.frombuffer(data[8:8 + 4 * (int(n) + 1)], dtype="<u4").astype(np.uint32)
        nb = np.frombuffer(data[8 + 4 * (int(n) + 1):], dtype="<u4").astype(np.uint32)
        return Csr(int(n), off, nb)


def _take_csr(h) -> Csr:
    if not h:
        raise RuntimeError("graph generator failed")
    L = lib()
    try:
        n = L.jc_csr_n_nodes(h)
        m = L.jc_csr_n_neighbors(h)
        off = np.ctypeslib.as_array(L.jc_csr_offsets(h), shape=(n + 1,)).copy()
        nb = np.ctypeslib.as_array(L.jc_csr_neighbors(h), shape=(m,)).copy() if m else np.zeros(0, np.uint32)
        return Csr(int(n), off.astype(np.uint32), nb.astype(np.uint32))
    finally:
        L.jc_csr_free(h)


def gen_scale_free(n: int, m: int, seed: int) -> Csr:
    """stability.rs:56-81 synthetic_scale_free."""
    return _take_csr(lib().jc_gen_scale_free(n, m, seed))


def csr_from_pairs(n: int, pairs) -> Csr:
    p = _u32(pairs).reshape(-1)
    return _take_csr(lib().jc_csr_from_pairs(n, _p(p, _u32p), len(p) // 2))


def gen_path(n: int) -> Csr:
    return _take_csr(lib().jc_gen_path(n))


def gen_grid(w: int, h: Optional[int] = None) -> Csr:
    return _take_csr(lib().jc_gen_grid(w, w if h is None else h))


def gen_rmat(scale: int, n_edges: int, a=0.57, b=0.19, c=0.19, seed: int = 1) -> Csr:
    return _take_csr(lib().jc_gen_rmat(scale, n_edges, a, b, c, seed))


def gen_watts_strogatz(n: int, k: int, p: float, seed: int) -> Csr:
    return _take_csr(lib().jc_gen_watts_strogatz(n, k, p, seed))


def gen_rgg(n: int, radius: float, seed: int, return_points: bool = False):
    pts = np.zeros(2 * n, dtype=np.float32)
    g = _take_csr(lib().jc_gen_rgg(n, radius, seed, _p(pts, _f32p)))
    return (g, pts.reshape(n, 2)) if return_points else g


def seed_ball(n: int, seed: int) -> np.ndarray:
    """stability.rs:30-49 ball_seed."""
    out = np.zeros(3 * n, dtype=np.float32)
    lib().jc_seed_ball(n, seed, _p(out, _f32p))
    return out


def seed_uniform(n: int, dim: int, seed: int) -> np.ndarray:
    out = np.zeros(3 * n, dtype=np.float32)
    lib().jc_seed_uniform(n, dim, seed, _p(out, _f32p))
    return out


def engine_ids() -> list[str]:
    L = lib()
    return [L.jc_engine_id_at(i).decode() for i in range(L.jc_engine_count())]


# ---------------------------------------------------------------- engine --
class LayoutEngine:
    """One engine handle (construct_leaf(id) + the LayoutEngine methods)."""

    def __init__(self, engine_id: str):
        self._L = lib()
        h = _vp()
        rc = self._L.jc_engine_create(engine_id.encode(), ctypes.byref(h))
        if rc != JC_OK:
            raise JcError(rc, f"jc_engine_create({engine_id!r}) failed")
        self._h = h
        self._cap = 0  # nodes of the bound graph: the most a step can write

    @property
    def n(self) -> int:
        """Nodes of the engine's current positions (jc_engine_output_nodes)."""
        return int(self._L.jc_engine_output_nodes(self._h)) if getattr(self, "_h", None) else 0

    @classmethod
    def _borrowed(cls, handle, owner, cap: int) -> "LayoutEngine":
        """A view of an engine handle that `owner` owns and destroys."""
        e = cls.__new__(cls)
        e._L = lib()
        e._h = handle
        e._cap = cap
        e._owner = owner  # keeps the owner (and so the handle) alive
        return e

    # -- lifecycle --
    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owner", None) is None:
                self._L.jc_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != JC_OK:
            raise JcError(rc, self._L.jc_engine_last_error(self._h).decode(errors="replace"))

    # -- trait methods --
    def descriptor(self) -> dict:
        d = JcDescriptor()
        self._check(self._L.jc_engine_descriptor(self._h, ctypes.byref(d)))
        return {
            "id": d.id.decode(), "kind": "Physics" if d.kind == 1 else "Static",
            "display_name": d.display_name.decode(), "description": d.description.decode(),
            "requirements": {"needs_edges": bool(d.needs_edges), "needs_cpu_positions": bool(d.needs_cpu_positions),
                             "needs_gpu_positions_buffer": bool(d.needs_gpu_positions_buffer)},
        }

    def set_params(self, params) -> None:
        text = params if isinstance(params, str) else json.dumps(params)
        self._check(self._L.jc_engine_set_params(self._h, text.encode()))

    def _bind(self, fn, csr: Csr, positions):
        off = _u32(csr.offsets)
        nb = _u32(csr.neighbors)
        pos = _f32(positions).reshape(-1)
        if len(pos) != 3 * csr.n_nodes:
            raise JcError(JC_ERR_ARG, f"initial positions length {len(pos)} != 3 * n_nodes {3 * csr.n_nodes}")
        nb_p = _p(nb, _u32p) if len(nb) else None
        self._check(fn(self._h, csr.n_nodes, _p(off, _u32p), nb_p, len(nb), _p(pos, _f32p)))
        self._cap = csr.n_nodes

    def init(self, csr: Csr, positions) -> None:
        self._bind(self._L.jc_engine_init, csr, positions)

    def reinit(self, csr: Csr, positions) -> None:
        self._bind(self._L.jc_engine_reinit, csr, positions)

    def init_batch(self, graphs, positions) -> None:
        """Bind a list of Csr graphs (each with its own 3*n positions)."""
        graphs = list(graphs)
        nodes = _u32([g.n_nodes for g in graphs])
        off = _u32(np.concatenate([g.offsets for g in graphs]))
        nbs = [g.neighbors for g in graphs if len(g.neighbors)]
        nb = _u32(np.concatenate(nbs)) if nbs else np.zeros(1, np.uint32)
        pos = _f32(np.concatenate([np.asarray(p, np.float32).reshape(-1) for p in positions]))
        if len(pos) != 3 * int(nodes.sum()):
            raise JcError(JC_ERR_ARG, "positions do not match the graphs")
        self._check(self._L.jc_engine_init_batch(self._h, len(graphs), _p(nodes, _u32p), _p(off, _u32p),
                                                 _p(nb, _u32p), _p(pos, _f32p)))
        self._cap = int(nodes.sum())
        self.graph_nodes = nodes.copy()

    def graph_speed(self, g: int):
        a, b = ctypes.c_float(), ctypes.c_float()
        self._check(self._L.jc_engine_graph_speed(self._h, g, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def autotune(self, probe_steps: int = 3):
        """Pick the fastest walk schedule; returns (group, ms per step of groups 1..32)."""
        g = ctypes.c_uint32()
        ms = np.zeros(6, np.float32)
        self._check(self._L.jc_engine_autotune(self._h, probe_steps, ctypes.byref(g), _p(ms, _f32p)))
        return int(g.value), ms

    def batch_schedule(self):
        """(True when one CTA per graph runs the batch, autotuner ms per step of that schedule)."""
        t, ms = ctypes.c_uint32(), ctypes.c_float()
        self._check(self._L.jc_engine_batch_schedule(self._h, ctypes.byref(t), ctypes.byref(ms)))
        return bool(t.value), float(ms.value)

    def step(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """One tick; returns the positions it wrote (3 x jc_engine_output_nodes)."""
        cap = max(self._cap, self.n)
        if out is None:
            out = np.zeros(3 * cap, dtype=np.float32)
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size < 3 * cap:
            raise JcError(JC_ERR_ARG, f"step output needs {3 * cap} contiguous f32")
        self._check(self._L.jc_engine_step(self._h, _p(out, _f32p) if cap else None))
        return out[:3 * self.n]

    def step_many(self, iters: int, readback: bool = True) -> Optional[np.ndarray]:
        cap = max(self._cap, self.n)
        out = np.zeros(3 * cap, dtype=np.float32) if readback else None
        self._check(self._L.jc_engine_step_many(self._h, iters, _p(out, _f32p) if (readback and cap) else None))
        return out[:3 * self.n] if readback else None

    def apply_halo(self, frame: int = 0, owner: int = 0, ids=(), positions=()) -> None:
        i = _u32(ids)
        p = _f32(positions)
        self._check(self._L.jc_engine_apply_halo(self._h, frame, owner, _p(i, _u32p), _p(p, _f32p), len(i)))

    # ---- multilevel wrapper ----
    def level_info(self) -> tuple[int, int, int]:
        """(current level, number of levels, inner steps at this level)."""
        a, b, c = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        self._check(lib().jc_engine_level_info(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return int(a.value), int(b.value), int(c.value)

    def cascade(self) -> list:
        """The engine's cascade: [(n_nodes, flat edges, parent_map), ...], level 0 first."""
        _, nl, _ = self.level_info()
        return _read_cascade(lambda l, *a: lib().jc_engine_cascade_level(self._h, l, *a), nl, self._check)

    # ---- partition-driven batching ----
    def init_partitions(self, parts: "Partitions", global_xyz) -> None:
        """Bind every partition's local graph as one batch (jc_engine_init_partitions)."""
        x = _f32(global_xyz)
        if len(x) != 3 * parts.n_nodes:
            raise JcError(JC_ERR_ARG, "positions do not match the partitioned graph")
        self._check(lib().jc_engine_init_partitions(self._h, parts._h, _p(x, _f32p)))
        self._parts = parts  # keep the set alive while the engine uses it
        self._cap = sum(p.local.n_nodes for p in parts.parts)

    def partition_positions(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Owned positions of every partition at their global ids (into `out` if given)."""
        if out is None:
            out = np.zeros(3 * self._parts.n_nodes, np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.size == 3 * self._parts.n_nodes
        self._check(lib().jc_engine_partition_positions(self._h, _p(out, _f32p)))
        return out

    def halo_delta(self, p: int) -> np.ndarray:
        """Partition p's boundary positions (3 x boundary size, parallel to its boundary ids)."""
        cnt = ctypes.c_uint32(0)
        self._check(lib().jc_engine_halo_delta(self._h, p, None, ctypes.byref(cnt)))
        out = np.zeros(3 * cnt.value, np.float32)
        if cnt.value:
            self._check(lib().jc_engine_halo_delta(self._h, p, _p(out, _f32p), ctypes.byref(cnt)))
        return out

    # ---- position frames (PositionDelta without a host wait per step) ----
    def stream_open(self, encoding: str = "f32", depth: int = 2, keyframe_interval: int = 0) -> None:
        """Open a frame stream: "f32" (raw LE f32 x,y,z) or "f16" (binary16 deltas)."""
        enc = {"f32": JC_FRAME_F32, "f16": JC_FRAME_F16_DELTA}[encoding]
        self._check(lib().jc_engine_stream_open(self._h, enc, depth, keyframe_interval))

    def stream_step(self, iters: int = 1) -> None:
        """Enqueue `iters` steps and their frame; returns without waiting."""
        self._check(lib().jc_engine_stream_step(self._h, iters))

    def stream_next_raw(self) -> JcFrame:
        """The oldest pending frame, pointing into library memory (valid until
        its slot is reused by a later stream_step)."""
        f = JcFrame()
        self._check(lib().jc_engine_stream_next(self._h, ctypes.byref(f)))
        return f

    def stream_next(self) -> "Frame":
        """The oldest pending frame, copied into Python bytes."""
        f = self.stream_next_raw()
        return Frame(int(f.frame), int(f.n_nodes), "f32" if f.encoding == JC_FRAME_F32 else "f16",
                     ctypes.string_at(f.data, f.bytes))

    def stream_close(self) -> None:
        self._check(lib().jc_engine_stream_close(self._h))

    def is_halted(self) -> bool:
        return bool(self._L.jc_engine_is_halted(self._h))

    # -- read-outs --
    def positions(self) -> np.ndarray:
        out = np.zeros(3 * self.n, dtype=np.float32)
        self._check(self._L.jc_engine_positions(self._h, _p(out, _f32p)))
        return out

    def forces(self):
        f = np.zeros(3 * self.n, dtype=np.float32)
        s = np.zeros(2 * self.n, dtype=np.float32)
        self._check(self._L.jc_engine_forces(self._h, _p(f, _f32p), _p(s, _f32p)))
        return f, s

    def speed(self):
        a, b = ctypes.c_float(), ctypes.c_float()
        self._check(self._L.jc_engine_speed(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def status_bits(self) -> int:
        return int(self._L.jc_engine_status_bits(self._h))

    def tree_info(self) -> dict:
        o = np.zeros(4, dtype=np.uint32)
        self._check(self._L.jc_engine_tree_info(self._h, _p(o, _u32p)))
        return {"nodes": int(o[0]), "bodies": int(o[1]), "max_depth": int(o[2]), "dropped": int(o[3])}

    def walk_counts(self) -> tuple[int, int]:
        o = np.zeros(2, dtype=np.uint64)
        self._check(self._L.jc_engine_walk_counts(self._h, _p(o, _u64p)))
        return int(o[0]), int(o[1])

    def time_steps(self, iters: int):
        t = ctypes.c_float()
        ph = np.zeros(4, dtype=np.float32)
        self._check(self._L.jc_engine_time_steps(self._h, iters, ctypes.byref(t), _p(ph, _f32p)))
        return t.value, ph

    def stress(self):
        """(raw, scale-normalized) stress over the engine's pivot terms."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self._L.jc_engine_stress(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def pivots(self):
        """(pivot ids, k x n hop distances) of an SGD engine."""
        k = ctypes.c_uint32()
        self._check(self._L.jc_engine_pivots(self._h, ctypes.byref(k), None, None))
        piv = np.zeros(max(k.value, 1), np.uint32)
        dist = np.zeros(max(k.value * self.n, 1), np.uint32)
        self._check(self._L.jc_engine_pivots(self._h, None, _p(piv, _u32p), _p(dist, _u32p)))
        return piv[:k.value], dist[:k.value * self.n].reshape(k.value, self.n)

    def launches_per_step(self) -> int:
        return int(self._L.jc_engine_launches_per_step(self._h))

    def save_state(self) -> bytes:
        need = ctypes.c_uint64()
        self._check(self._L.jc_engine_save_state(self._h, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value)
        self._check(self._L.jc_engine_save_state(self._h, buf, need.value, ctypes.byref(need)))
        return buf.raw

    def load_state(self, data: bytes) -> None:
        buf = ctypes.create_string_buffer(data, len(data))
        self._check(self._L.jc_engine_load_state(self._h, buf, len(data)))


def _read_cascade(get, n_levels: int, check) -> list:
    out = []
    for l in range(n_levels):
        n, w = ctypes.c_uint32(), ctypes.c_uint64()
        check(get(l, ctypes.byref(n), ctypes.byref(w), None, None))
        ed = np.zeros(max(w.value, 1), np.uint32)
        pm = np.zeros(max(out[-1][0] if out else 0, 1), np.uint32)
        check(get(l, ctypes.byref(n), ctypes.byref(w), _p(ed, _u32p), _p(pm, _u32p)))
        out.append((int(n.value), ed[:w.value].copy(), pm[:out[-1][0] if out else 0].copy()))
    return out


def coarsen(n_nodes: int, edges, max_levels: int = 6, target_size: int = 500) -> list:
    """graph_layouts::coarsen (coarsen.rs:52-90) of a flat edge list, through jc_coarsen."""
    e = _u32(edges)
    h = _vp()
    rc = lib().jc_coarsen(n_nodes, _p(e, _u32p) if len(e) else None, len(e), max_levels, target_size,
                          ctypes.byref(h))
    if rc != 0:
        raise JcError(rc, "jc_coarsen failed")

    def check(rc):
        if rc != 0:
            raise JcError(rc, "jc_cascade_get failed")
    try:
        return _read_cascade(lambda l, *a: lib().jc_cascade_get(h, l, *a), lib().jc_cascade_levels(h), check)
    finally:
        lib().jc_cascade_free(h)


@dataclass
class Partition:
    """One partition (crates/graph-compute/src/partition.rs:54-91)."""
    partition_id: int
    n_partitions: int
    n_owned: int
    local: Csr
    global_ids: np.ndarray
    boundary: np.ndarray

    @property
    def owned_global_ids(self) -> np.ndarray:
        return self.global_ids[:self.n_owned]

    @property
    def ghost_global_ids(self) -> np.ndarray:
        return self.global_ids[self.n_owned:]


class Partitions:
    """partition_csr / partition_csr_refined of one graph (jc_partition_csr)."""

    def __init__(self, csr: Csr, n_partitions: int, refine: bool = False):
        off, nb = _u32(csr.offsets), _u32(csr.neighbors)
        h = _vp()
        rc = lib().jc_partition_csr(csr.n_nodes, _p(off, _u32p), _p(nb, _u32p), len(nb), n_partitions,
                                    1 if refine else 0, ctypes.byref(h))
        if rc != 0:
            raise JcError(rc, "jc_partition_csr failed")
        self._h = h
        self.n_nodes = csr.n_nodes
        L = lib()
        self.edge_cut = int(L.jc_partitions_edge_cut(h))
        own = L.jc_partitions_owner(h)
        self.owner = (np.ctypeslib.as_array(own, shape=(csr.n_nodes,)).copy() if csr.n_nodes
                      else np.zeros(0, np.uint32))
        self.parts = []
        for i in range(L.jc_partitions_count(h)):
            v = JcPartitionView()
            if L.jc_partition_get(h, i, ctypes.byref(v)) != 0:
                raise JcError(JC_ERR_ARG, "jc_partition_get failed")

            def arr(ptr, k):
                return np.ctypeslib.as_array(ptr, shape=(k,)).copy() if k else np.zeros(0, np.uint32)
            local = Csr(int(v.n_local), arr(v.offsets, v.n_local + 1), arr(v.neighbors, v.n_neighbors))
            self.parts.append(Partition(int(v.partition_id), int(v.n_partitions), int(v.n_owned), local,
                                        arr(v.global_ids, v.n_local), arr(v.boundary, v.n_boundary)))

    def close(self):
        if getattr(self, "_h", None):
            lib().jc_partitions_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.parts)

    def __getitem__(self, i) -> Partition:
        return self.parts[i]


def partition_csr(csr: Csr, n_partitions: int, refine: bool = False) -> Partitions:
    """partition.rs:191 partition_csr (refine=True: :510 partition_csr_refined)."""
    return Partitions(csr, n_partitions, refine)


@dataclass
class Frame:
    """One position frame message: 64-byte header + payload (jc_frame)."""
    frame: int
    n_nodes: int
    encoding: str
    data: bytes

    @property
    def payload(self) -> np.ndarray:
        body = self.data[64:]
        return np.frombuffer(body, dtype="<f4" if self.encoding == "f32" else "<u2")


def frame_message(frame: int, n_nodes: int, encoding: str, payload: np.ndarray) -> bytes:
    """Builds the wire form of a frame (header layout of jc_frame)."""
    enc = JC_FRAME_F32 if encoding == "f32" else JC_FRAME_F16_DELTA
    body = np.ascontiguousarray(payload, dtype="<f4" if encoding == "f32" else "<u2").tobytes()
    hdr = np.zeros(16, dtype="<u4")
    hdr[0] = 0x3146434A
    hdr[1] = enc
    hdr[2:4] = np.array([frame], dtype="<u8").view("<u4")
    hdr[4] = n_nodes
    hdr[6:8] = np.array([len(body)], dtype="<u8").view("<u4")
    return hdr.tobytes() + body


class FrameDecoder:
    """A receiver's reconstruction of a frame stream (jc_frame_decode)."""

    def __init__(self, n_nodes: int):
        self.n_nodes = n_nodes
        self._h = lib().jc_frame_decoder_create(n_nodes)
        if not self._h:
            raise MemoryError("jc_frame_decoder_create failed")

    def close(self):
        if self._h:
            lib().jc_frame_decoder_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def decode(self, data) -> np.ndarray:
        buf = bytes(data.data if isinstance(data, Frame) else data)
        out = np.zeros(3 * self.n_nodes, np.float32)
        rc = lib().jc_frame_decode(self._h, ctypes.c_char_p(buf), len(buf), _p(out, _f32p))
        if rc != 0:
            raise JcError(rc, lib().jc_frame_decoder_last_error(self._h).decode())
        return out


def fa2_bh_forces_noalloc(n_nodes: int, d_offsets: int, d_neighbors: int, d_positions_xyz: int, d_forces_xyz: int,
                          theta: float = 0.7, gravity: float = 1.0, scaling_ratio: float = 2.0,
                          edge_weight_influence: float = 1.0, strong_gravity: bool = False,
                          lin_log_mode: bool = False, stream: int = 0) -> None:
    """Barnes-Hut force pass over caller-owned device buffers (raw device
    addresses), with no device allocation (jc_fa2_bh_forces_noalloc)."""
    prm = Fa2Params(gravity, int(strong_gravity), scaling_ratio, edge_weight_influence, int(lin_log_mode), theta)
    rc = lib().jc_fa2_bh_forces_noalloc(n_nodes, d_offsets, d_neighbors, d_positions_xyz, ctypes.byref(prm),
                                        d_forces_xyz, stream or None)
    if rc != JC_OK:
        raise JcError(rc, "jc_fa2_bh_forces_noalloc failed")


def set_device(device: int) -> None:
    rc = lib().jc_set_device(device)
    if rc != JC_OK:
        raise JcError(rc, f"jc_set_device({device}) failed")


def to_bf16_bits(x) -> np.ndarray:
    """Round-to-nearest-even f32 -> bf16 bit patterns (uint16)."""
    u = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


GEMM_STAGING = {"auto": 0, "cp.async": 1, "tma": 2}


def tc_gemm_bf16(a_bits, b_bits, M: int, N: int, K: int, a_kmajor: bool = True, b_kmajor: bool = True,
                 bn: int = 128, splits: int = 1, staging: str = "auto") -> np.ndarray:
    """C = A B on the tcgen05 tensor cores (test entry point). `staging`:
    "auto", "cp.async" or "tma" (the kernel that stages the operands)."""
    a = np.ascontiguousarray(a_bits, np.uint16)
    b = np.ascontiguousarray(b_bits, np.uint16)
    c = np.zeros(M * N, np.float32)
    rc = lib().jc_tc_gemm_bf16(M, N, K, a.ctypes.data, int(a_kmajor), b.ctypes.data, int(b_kmajor), bn, splits,
                               GEMM_STAGING[staging], _p(c, _f32p))
    if rc != JC_OK:
        raise JcError(rc, "jc_tc_gemm_bf16 failed")
    return c.reshape(M, N)


def gen_batch_graphs(n_graphs: int, seed: int = 4096, lo: int = 50, hi: int = 20000):
    """Seeded batch of uneven graphs: node counts floor(exp(U(ln lo, ln hi))),
    generator g mod 3 = Barabasi-Albert (m uniform in 2..4), Watts-Strogatz
    (k = 6, p = 0.1), random geometric (mean degree 6); plus uniform
    [-1,1]^2 seeds (z = 0). Returns (graphs, seeds)."""
    mask = (1 << 64) - 1
    state = seed

    def nxt():
        nonlocal state
        state = (state + 0x9E3779B97F4A7C15) & mask
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        return z ^ (z >> 31)

    graphs, pos = [], []
    a, b = np.log(float(lo)), np.log(float(hi))
    for g in range(n_graphs):
        u = (nxt() >> 11) / float(1 << 53)
        n = int(np.floor(np.exp(a + u * (b - a))))
        kind = g % 3
        if kind == 0:
            graphs.append(gen_scale_free(n, 2 + nxt() % 3, nxt()))
        elif kind == 1:
            graphs.append(gen_watts_strogatz(n, 6, 0.1, nxt()))
        else:
            graphs.append(gen_rgg(n, float(np.sqrt(6.0 / (np.pi * n))), nxt()))
        pos.append(seed_uniform(graphs[-1].n_nodes, 2, nxt()))
    return graphs, pos


def _graph_arrays(graphs):
    """(graph_nodes, concatenated offsets, concatenated neighbours) in the
    jc_engine_init_batch convention."""
    graphs = list(graphs)
    nodes = _u32([g.n_nodes for g in graphs])
    off = _u32(np.concatenate([g.offsets for g in graphs]))
    nbs = [g.neighbors for g in graphs if len(g.neighbors)]
    nb = _u32(np.concatenate(nbs)) if nbs else np.zeros(1, np.uint32)
    return nodes, off, nb


class Batch:
    """Batch builder (jc_batch_*): graphs added one at a time with their own
    CSR and seed positions, bound together on the first run and stepped as
    one fa2-bh batch."""

    def __init__(self, params=None, engine_id: str = "fa2-bh"):
        self._L = lib()
        h = _vp()
        js = None if params is None else (params if isinstance(params, str) else json.dumps(params)).encode()
        rc = self._L.jc_batch_create(engine_id.encode(), js, ctypes.byref(h))
        if rc != JC_OK:
            raise JcError(rc, f"jc_batch_create({engine_id!r}) failed")
        self._h = h
        self.graph_nodes = []

    def close(self):
        if getattr(self, "_h", None):
            self._L.jc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self) -> int:
        return int(self._L.jc_batch_graph_count(self._h))

    def _check(self, rc: int):
        if rc != JC_OK:
            raise JcError(rc, self._L.jc_batch_last_error(self._h).decode(errors="replace"))

    def add_graph(self, g: "Csr", positions) -> int:
        off, nb = _u32(g.offsets), _u32(g.neighbors)
        pos = _f32(np.asarray(positions, np.float32).reshape(-1))
        if len(pos) != 3 * g.n_nodes:
            raise JcError(JC_ERR_ARG, "positions do not match the graph")
        idx = ctypes.c_uint32()
        self._check(self._L.jc_batch_add_graph(self._h, g.n_nodes, _p(off, _u32p),
                                               _p(nb if len(nb) else np.zeros(1, np.uint32), _u32p), len(nb),
                                               _p(pos, _f32p) if len(pos) else None, ctypes.byref(idx)))
        self.graph_nodes.append(g.n_nodes)
        return idx.value

    def bind(self) -> None:
        self._check(self._L.jc_batch_bind(self._h))

    def run(self, iters: int) -> None:
        self._check(self._L.jc_batch_run(self._h, iters))

    def positions(self, graph: int) -> np.ndarray:
        if not 0 <= graph < len(self.graph_nodes):
            raise JcError(JC_ERR_ARG, "graph index out of range")
        out = np.zeros(3 * self.graph_nodes[graph], np.float32)
        self._check(self._L.jc_batch_positions(self._h, graph, _p(out, _f32p)))
        return out

    def engine(self) -> LayoutEngine:
        """The bound engine (owned by this batch): autotune, checkpoints, frame streams."""
        return LayoutEngine._borrowed(self._L.jc_batch_engine(self._h), self, sum(self.graph_nodes))


class Mpnn:
    """Learned warm start: the message-passing network of jc_mpnn_* (train on
    graphs + target layouts, then predict initial coordinates)."""

    def __init__(self, dim: int = 2, seed: int = 0x5EED):
        self._L = lib()
        h = _vp()
        rc = self._L.jc_mpnn_create(dim, seed, ctypes.byref(h))
        if rc != JC_OK:
            raise JcError(rc, f"jc_mpnn_create(dim={dim}) failed")
        self._h = h
        self.dim = dim
        self.n = 0

    def close(self):
        if getattr(self, "_h", None):
            self._L.jc_mpnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != JC_OK:
            raise JcError(rc, self._L.jc_mpnn_last_error(self._h).decode())

    @staticmethod
    def num_params() -> int:
        return int(lib().jc_mpnn_num_params())

    def set_params(self, params) -> None:
        self._check(self._L.jc_mpnn_set_params(self._h, json.dumps(params).encode()))

    def weights(self) -> np.ndarray:
        w = np.zeros(self.num_params(), np.float32)
        self._check(self._L.jc_mpnn_get_weights(self._h, _p(w, _f32p)))
        return w

    def set_weights(self, w) -> None:
        w = _f32(w)
        if len(w) != self.num_params():
            raise JcError(JC_ERR_ARG, "weight vector has the wrong length")
        self._check(self._L.jc_mpnn_set_weights(self._h, _p(w, _f32p)))

    def bind(self, graphs, targets) -> None:
        """Training set: graphs and target layouts (each 3*n floats)."""
        nodes, off, nb = _graph_arrays(graphs)
        t = _f32(np.concatenate([np.asarray(x, np.float32).reshape(-1) for x in targets]))
        if len(t) != 3 * int(nodes.sum()):
            raise JcError(JC_ERR_ARG, "targets do not match the graphs")
        self._check(self._L.jc_mpnn_bind(self._h, len(nodes), _p(nodes, _u32p), _p(off, _u32p), _p(nb, _u32p),
                                         _p(t, _f32p)))
        self.n = int(nodes.sum())
        self.graph_nodes = nodes.copy()

    def batches(self) -> int:
        c = ctypes.c_uint32()
        self._check(self._L.jc_mpnn_batches(self._h, ctypes.byref(c)))
        return c.value

    def features(self) -> np.ndarray:
        x = np.zeros((self.n, 32), np.float32)
        self._check(self._L.jc_mpnn_features(self._h, _p(x, _f32p)))
        return x

    def train(self, steps: int) -> np.ndarray:
        losses = np.zeros(max(steps, 1), np.float32)
        self._check(self._L.jc_mpnn_train(self._h, steps, _p(losses, _f32p)))
        return losses[:steps]

    def eval_loss(self) -> float:
        v = ctypes.c_double()
        self._check(self._L.jc_mpnn_eval_loss(self._h, ctypes.byref(v)))
        return v.value

    def grad(self, g0: int, g1: int, pair_step: int = 0):
        """(loss, Y nb x 4, gradient) on graphs [g0, g1) of the bound set, no update."""
        nb = int(self.graph_nodes[g0:g1].sum())
        y = np.zeros((max(nb, 1), 4), np.float32)
        g = np.zeros(self.num_params(), np.float32)
        loss = ctypes.c_float()
        self._check(self._L.jc_mpnn_grad(self._h, g0, g1, pair_step, ctypes.byref(loss), _p(y, _f32p), _p(g, _f32p)))
        return loss.value, y[:nb], g

    def predict(self, graphs):
        """(xyz list per graph, device ms of features + forward + hand-off scale)."""
        graphs = list(graphs)
        nodes, off, nb = _graph_arrays(graphs)
        out = np.zeros(3 * max(int(nodes.sum()), 1), np.float32)
        ms = ctypes.c_float()
        self._check(self._L.jc_mpnn_predict(self._h, len(nodes), _p(nodes, _u32p), _p(off, _u32p), _p(nb, _u32p),
                                            _p(out, _f32p), ctypes.byref(ms)))
        res, b = [], 0
        for k in nodes:
            res.append(out[3 * b: 3 * (b + int(k))].copy())
            b += int(k)
        return res, ms.value

    def warm_start(self, graphs, seeds, evaluator):
        """Guarded hand-off: each graph starts from the prediction only where
        the prediction's pivot stress (`evaluator`, built on the same graphs)
        is below that of the graph's own seed layout; elsewhere the seed is
        kept, so plain ForceAtlas2 from the seed stays the fallback. Returns
        (xyz per graph, bool per graph: prediction kept, wall ms of the call,
        device ms of the prediction and both evaluations)."""
        graphs = list(graphs)
        nodes, off, nb = _graph_arrays(graphs)
        seed = _f32(np.concatenate([np.asarray(s, np.float32).reshape(-1) for s in seeds]))
        if len(seed) != 3 * int(nodes.sum()):
            raise JcError(JC_ERR_ARG, "seeds do not match the graphs")
        out = np.zeros(max(len(seed), 1), np.float32)
        kept = np.zeros(len(nodes), np.uint8)
        ms = ctypes.c_float()
        t0 = time.perf_counter()
        self._check(self._L.jc_mpnn_warm_start(self._h, evaluator._h, len(nodes), _p(nodes, _u32p), _p(off, _u32p),
                                               _p(nb, _u32p), _p(seed, _f32p), _p(out, _f32p),
                                               kept.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                               ctypes.byref(ms)))
        wall = (time.perf_counter() - t0) * 1e3
        res, b = [], 0
        for k in nodes:
            res.append(out[3 * b: 3 * (b + int(k))].copy())
            b += int(k)
        return res, kept.astype(bool), wall, ms.value

    def predict_stages(self):
        """Device ms of the last predict: (features, network, hand-off scale)."""
        ms = np.zeros(3, np.float32)
        self._check(self._L.jc_mpnn_predict_stages(self._h, _p(ms, _f32p)))
        return tuple(float(x) for x in ms)

    def save_state(self) -> bytes:
        n = int(self._L.jc_mpnn_state_size(self._h))
        buf = ctypes.create_string_buffer(n)
        self._check(self._L.jc_mpnn_save_state(self._h, ctypes.cast(buf, _vp)))
        return buf.raw

    def load_state(self, data: bytes) -> None:
        buf = ctypes.create_string_buffer(data, len(data))
        self._check(self._L.jc_mpnn_load_state(self._h, ctypes.cast(buf, _vp), len(data)))


class Evaluator:
    """Per-graph scale-normalized pivot stress and edge-length CV on the device."""

    def __init__(self, graphs, n_pivots: int = 16, seed: int = 0xE7A1):
        self._L = lib()
        graphs = list(graphs)
        nodes, off, nb = _graph_arrays(graphs)
        h = _vp()
        rc = self._L.jc_eval_create(len(nodes), _p(nodes, _u32p), _p(off, _u32p), _p(nb, _u32p), n_pivots, seed,
                                    ctypes.byref(h))
        if rc != JC_OK:
            raise JcError(rc, "jc_eval_create failed")
        self._h = h
        self.G = len(nodes)
        self.k = n_pivots
        self.n = int(nodes.sum())

    def close(self):
        if getattr(self, "_h", None):
            self._L.jc_eval_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != JC_OK:
            raise JcError(rc, self._L.jc_eval_last_error(self._h).decode())

    def pivots(self) -> np.ndarray:
        p = np.zeros(self.G * self.k, np.uint32)
        self._check(self._L.jc_eval_pivots(self._h, _p(p, _u32p)))
        return p.reshape(self.G, self.k)

    def __call__(self, xyz):
        """(mean stress, mean cv, per-graph stress, per-graph cv) of a layout (3n floats)."""
        x = _f32(np.asarray(xyz, np.float32).reshape(-1))
        if len(x) != 3 * self.n:
            raise JcError(JC_ERR_ARG, "positions do not match the graphs")
        st = np.zeros(self.G, np.float64)
        cv = np.zeros(self.G, np.float64)
        means = np.zeros(2, np.float64)
        self._check(self._L.jc_eval_layout(self._h, _p(x, _f32p), _p(st, _f64p), _p(cv, _f64p), _p(means, _f64p)))
        return float(means[0]), float(means[1]), st, cv


def build_info() -> str:
    return lib().jc_build_info().decode()
