"""Golden fixtures (tests/golden/layout_step_golden.json, written by
tests/golden/make_golden.py after the C++ oracle and an independent
float32 pure-Python restatement of the reference agreed on them).

CPU: the oracle and the product's seeded generators reproduce the fixtures.
GPU: the CUDA engines reproduce them through the C ABI.
"""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "layout_step_golden.json").read_text())
FA2_CASES = sorted(k for k in GOLDEN if k.startswith("fa2"))


def f32(bits):
    return np.array(bits, np.uint32).view(np.float32)


def csr(jc, d):
    return jc.Csr(d["n"], np.array(d["offsets"], np.uint32), np.array(d["neighbors"], np.uint32))


def test_generators_reproduce_fixtures(jc):
    g = jc.gen_scale_free(64, 3, 0xC0FFEE)
    d = GOLDEN["gen_scale_free_64_3_c0ffee"]
    assert g.offsets.tolist() == d["offsets"] and g.neighbors.tolist() == d["neighbors"]
    assert jc.seed_ball(16, 0x5EED).view(np.uint32).tolist() == GOLDEN["seed_ball_16_5eed"]
    assert jc.seed_uniform(8, 3, 7).view(np.uint32).tolist() == GOLDEN["seed_uniform_8_3_7"]


@pytest.mark.parametrize("name", FA2_CASES)
def test_oracle_reproduces_fa2_fixture(jc, orc, name):
    rec = GOLDEN[name]
    o = orc.Fa2(csr(jc, rec["csr"]), f32(rec["seed"]), bh=rec["bh"], **rec["settings"])
    for s in rec["steps"]:
        o.step()
        r = o.get()
        assert r["pos"].view(np.uint32).tolist() == s["pos"]
        assert r["force"].view(np.uint32).tolist() == s["force"]


@pytest.mark.parametrize("name", ["sgd_jacobi_grid5", "sgd_cpu_path12"])
def test_oracle_reproduces_sgd_fixture(jc, orc, name):
    rec = GOLDEN[name]
    o = orc.Sgd(csr(jc, rec["csr"]), f32(rec["seed"]), mode=rec["mode"])
    for s in rec["steps"]:
        assert o.step().view(np.uint32).tolist() == s


@pytest.mark.gpu
@pytest.mark.parametrize("name", FA2_CASES)
def test_engine_reproduces_fa2_fixture(jc, name):
    rec = GOLDEN[name]
    e = jc.LayoutEngine("fa2-bh" if rec["bh"] else "fa2-brute")
    e.set_params(rec["settings"])
    e.init(csr(jc, rec["csr"]), f32(rec["seed"]))
    for k, s in enumerate(rec["steps"]):
        out = e.step()
        f, st = e.forces()
        assert f.view(np.uint32).tolist() == s["force"], (name, k)
        assert st.view(np.uint32).tolist() == s["stats"], (name, k)
        assert out.view(np.uint32).tolist() == s["pos"], (name, k)


@pytest.mark.gpu
def test_engine_reproduces_jacobi_fixture(jc):
    rec = GOLDEN["sgd_jacobi_grid5"]
    e = jc.LayoutEngine("sgd-stress-gpu")
    e.init(csr(jc, rec["csr"]), f32(rec["seed"]))
    for s in rec["steps"]:
        assert e.step().view(np.uint32).tolist() == s
