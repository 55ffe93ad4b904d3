"""Runs in a child process with JC_LAYOUT_LIB pointing at the bounds-check
build (libjc_layout_bc.so): the device index checks must never fire on valid
inputs, and the results must be those of the normal build (bit-exact against
the oracle). Used by tests/test_bounds_check.py."""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
for p in (str(ROOT), str(ROOT / "jump-cannon_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import jc_layout as jc  # noqa: E402
import oracle.oracle as orc  # noqa: E402


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def main():
    assert "bounds-check" in jc.build_info(), jc.build_info()
    jc.set_device(0)
    cases = [
        (jc.gen_scale_free(3000, 3, 9), jc.seed_uniform(3000, 3, 1), {"theta": 0.8}),
        (jc.gen_rmat(13, 65536, seed=2), jc.seed_uniform(8192, 3, 3), {"theta": 0.8, "hub_threshold": 1 << 30}),
        (jc.gen_grid(40), jc.seed_uniform(1600, 2, 4), {"theta": 0.6, "use_graph": False}),
    ]
    for g, pos, prm in cases:
        e = jc.LayoutEngine("fa2-bh")
        e.set_params(prm)
        e.init(g, pos)
        e.step_many(3, readback=False)
        f, _ = e.forces()
        o = orc.Fa2(g, pos, bh=True, **{k: v for k, v in prm.items() if k in ("theta",)})
        for _ in range(3):
            o.step()
        assert np.array_equal(bits(f), bits(o.get()["force"]))
        assert e.walk_counts() == (o.get()["n_inter"], o.get()["n_open"])
        e.close()
    # hubs (block reduction) and the warp path
    g = jc.gen_rmat(15, 1 << 19, seed=5)
    pos = jc.seed_uniform(g.n_nodes, 3, 7)
    e = jc.LayoutEngine("fa2-bh")
    e.set_params({"theta": 0.8})
    e.init(g, pos)
    e.step()
    f, _ = e.forces()
    o = orc.Fa2(g, pos, bh=True, theta=0.8)
    o.step()
    ref = o.get()["force"].astype(np.float64)
    assert np.linalg.norm(f - ref) / np.linalg.norm(ref) < 1e-6
    # a batch of graphs (forest keys, per-graph trees)
    graphs, seeds = jc.gen_batch_graphs(64, seed=11, hi=3000)
    b = jc.LayoutEngine("fa2-bh")
    b.set_params({"theta": 0.8})
    b.init_batch(graphs, seeds)
    out = b.step_many(5)
    assert np.all(np.isfinite(out))
    ref_pos = []
    for gg, ss in zip(graphs[:4], seeds[:4]):
        oo = orc.Fa2(gg, ss, bh=True, theta=0.8)
        for _ in range(5):
            oo.step()
        ref_pos.append(oo.get()["pos"])
    got = out[:3 * sum(gg.n_nodes for gg in graphs[:4])]
    assert np.array_equal(bits(got), bits(np.concatenate(ref_pos)))
    print("bounds-check build: no check fired, results bit-exact")


if __name__ == "__main__":
    main()
