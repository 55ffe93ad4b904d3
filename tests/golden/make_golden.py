"""Generates tests/golden/*.json: small seeded cases of the layout step.

Two independent restatements of the reference must agree before a fixture is
written:
  * the C++ oracle (oracle/oracle.cpp), and
  * the pure-Python restatement below, evaluated with numpy float32 scalars
    one operation at a time, of crates/graph-compute/src/engines/fa2_bh.rs
    (OctreeBuild :761-1045, walk :1096-1147), fa2_barnes_hut.wgsl
    (fa2_force :96-198, fa2_apply :203-226) and fa2_speed.rs (:48-100).
Floats are stored as uint32 bit patterns so the fixtures are exact.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "jump-cannon_b200"), str(ROOT / "tests")]

F = np.float32
END = 0xFFFFFFFF


# ---------------------------------------------------- pure-Python restatement
class PyOctree:
    """fa2_bh.rs:747-1045 with float32 scalar arithmetic."""

    def __init__(self):
        self.ps, self.cm, self.meta, self.ch = [], [], [], []

    def _push(self, c, h, cm, body):
        self.ps.append([c[0], c[1], c[2], h])
        self.cm.append(list(cm))
        self.meta.append([body, END, END, 0])
        self.ch.append([END] * 8)
        return len(self.ps) - 1

    def insert(self, node, p, body, mass, cap):
        for _ in range(32):
            c = self.ps[node]
            o = (1 if p[0] >= c[0] else 0) | (2 if p[1] >= c[1] else 0) | (4 if p[2] >= c[2] else 0)
            child = self.ch[node][o]
            if child == END:
                if len(self.ps) >= cap:
                    return False
                h = F(c[3] * F(0.5))
                cc = [F(c[k] + (h if o & (1 << k) else -h)) for k in range(3)]
                idx = self._push(cc, h, [p[0], p[1], p[2], mass], body)
                self.ch[node][o] = idx
                self.meta[node][3] += 1
                return True
            if self.meta[child][0] == END:
                node = child
                continue
            prev = self.cm[child]
            pb = self.meta[child][0]
            self.cm[child] = [F(0), F(0), F(0), F(0)]
            self.meta[child][0] = END
            self.meta[child][3] = 0
            if not self.insert(child, prev[:3], pb, max(prev[3], F(1e-3)), cap):
                return False
            node = child
        return True

    def build(self, pos, mass, cap):
        n = len(mass)
        mn = [F(np.inf)] * 3
        mx = [F(-np.inf)] * 3
        for i in range(n):
            for k in range(3):
                v = pos[i][k]
                if not np.isfinite(v):
                    continue
                if v < mn[k]:
                    mn[k] = v
                if v > mx[k]:
                    mx[k] = v
        if not np.isfinite(mn[0]):
            mn, mx = [F(-1)] * 3, [F(1)] * 3
        c = [F(F(0.5) * F(mn[k] + mx[k])) for k in range(3)]
        ext = [F(mx[k] - mn[k]) for k in range(3)]
        half = F(max(max(ext[0], ext[1]), ext[2]) * F(0.5))
        if not np.isfinite(half) or half <= 0:
            half = F(1.0)
        half = F(half * F(1.05))
        self._push(c, half, [F(0)] * 4, END)
        for b in range(n):
            p = pos[b]
            if not all(np.isfinite(p)):
                continue
            if not self.insert(0, p, b, max(mass[b], F(1e-3)), cap):
                break
        self._com(0)
        self._ropes()

    def _com(self, idx):
        if self.meta[idx][0] != END:
            return
        for k in range(8):
            if self.ch[idx][k] != END:
                self._com(self.ch[idx][k])
        tot, s = F(0), [F(0), F(0), F(0)]
        for k in range(8):
            c = self.ch[idx][k]
            if c == END:
                continue
            m = self.cm[c][3]
            tot = F(tot + m)
            s = [F(s[j] + F(self.cm[c][j] * m)) for j in range(3)]
        if tot > 0:
            s = [F(s[j] / tot) for j in range(3)]
        self.cm[idx] = [s[0], s[1], s[2], tot]

    def _ropes(self):
        order = []

        def dfs(i, skip):
            order.append(i)
            kids = [c for c in self.ch[i] if c != END] if self.meta[i][0] == END else []
            self.meta[i][1] = kids[0] if kids else END
            self.meta[i][2] = skip
            for a, c in enumerate(kids):
                dfs(c, kids[a + 1] if a + 1 < len(kids) else skip)

        dfs(0, END)

    def walk(self, p, i, deg, scaling, theta):
        f = [F(0), F(0), F(0)]
        th2 = F(F(theta) * F(theta))
        idx = 0
        while idx != END:
            body, nxt, skip, _ = self.meta[idx]
            com, m = self.cm[idx][:3], self.cm[idx][3]
            s = F(self.ps[idx][3] * F(2.0))
            d = [F(p[k] - com[k]) for k in range(3)]
            r2 = F(F(F(d[0] * d[0]) + F(d[1] * d[1])) + F(d[2] * d[2]))
            if body != END:
                if body != i and m > 0:
                    c = F(F(F(F(scaling) * deg) * m) / max(r2, F(1e-4)))
                    f = [F(f[k] + F(d[k] * c)) for k in range(3)]
                idx = skip
                continue
            if m > 0 and r2 > 0 and F(s * s) < F(th2 * r2):
                c = F(F(F(F(scaling) * deg) * m) / max(r2, F(1e-4)))
                f = [F(f[k] + F(d[k] * c)) for k in range(3)]
                idx = skip
            else:
                idx = nxt
        return f


def length(v):
    return F(np.sqrt(F(F(F(v[0] * v[0]) + F(v[1] * v[1])) + F(v[2] * v[2]))))


def py_fa2_step(csr, pos3, old3, speed, eff, theta, scaling=2.0, gravity=1.0, jt_tol=1.0, max_disp=10.0):
    """One fa2-bh step (fa2_bh.rs:546-692) on float32 scalars."""
    n = csr.n_nodes
    pos = [[F(pos3[3 * i + k]) for k in range(3)] for i in range(n)]
    old = [[F(old3[3 * i + k]) for k in range(3)] for i in range(n)]
    deg = [0] * n
    edges = []
    for v in range(n):
        for e in range(csr.offsets[v], csr.offsets[v + 1]):
            u = int(csr.neighbors[e])
            if u == v:
                continue
            deg[v] += 1
            if v < u:
                edges.append((v, u))
    degf = [F(F(d) + F(1.0)) for d in deg]
    t = PyOctree()
    t.build(pos, degf, 2 * n + 8)
    forces, stats = [], []
    for i in range(n):
        f = t.walk(pos[i], i, degf[i], scaling, theta)
        for (a, b) in edges:  # fa2_barnes_hut.wgsl:160-181 (edge weight 1)
            if a == i:
                o = b
            elif b == i:
                o = a
            else:
                continue
            d = [F(pos[o][k] - pos[i][k]) for k in range(3)]
            f = [F(f[k] + F(d[k] * F(1.0))) for k in range(3)]
        r0 = max(length(pos[i]), F(1e-3))
        gd = F(F(gravity) * degf[i])
        f = [F(f[k] - F(F(pos[i][k] / r0) * gd)) for k in range(3)]
        forces.append(f)
        stats.append((F(degf[i] * length([F(old[i][k] - f[k]) for k in range(3)])),
                      F(F(degf[i] * F(0.5)) * length([F(old[i][k] + f[k]) for k in range(3)]))))
    # fa2_speed.rs:48-100
    ts = sum(float(s) for s, tr in stats if np.isfinite(s) and np.isfinite(tr))
    tt = sum(float(tr) for s, tr in stats if np.isfinite(s) and np.isfinite(tr))
    speed, eff = F(speed), F(eff)
    if ts > 0 and tt > 0 and n > 0:
        nn = float(n)
        est = 0.05 * math.sqrt(nn)
        jt = float(jt_tol) * max(math.sqrt(est), min(10.0, est * tt / (nn * nn)))
        if ts / tt > 2.0:
            if eff > F(0.05):
                eff = F(eff * F(0.5))
            jt = max(jt, float(jt_tol))
        target = jt * float(eff) * tt / ts
        if ts > jt * tt:
            if eff > F(0.05):
                eff = F(eff * F(0.7))
        elif speed < F(1000.0):
            eff = F(eff * F(1.3))
        sp = float(speed)
        speed = F(sp + min(target - sp, 0.5 * sp))
    out = []
    for i in range(n):
        f = forces[i]
        sw = F(degf[i] * length([F(old[i][k] - f[k]) for k in range(3)]))
        fac = F(speed / F(F(1.0) + F(np.sqrt(F(speed * sw)))))
        df = length(f)
        if max_disp > 0 and df > F(1e-9):
            fac = min(fac, F(F(max_disp) / df))
        kk = F(fac * F(1.0))
        out.append([F(pos[i][k] + F(f[k] * kk)) for k in range(3)])
    flat = lambda rows: np.array([x for r in rows for x in r], np.float32)
    return flat(out), flat(forces), np.array([x for s in stats for x in s], np.float32), speed, eff


# ------------------------------------------------------------------ fixtures
def hexbits(a):
    return [int(x) for x in np.ascontiguousarray(a, np.float32).view(np.uint32)]


def csr_dict(g):
    return {"n": g.n_nodes, "offsets": [int(x) for x in g.offsets], "neighbors": [int(x) for x in g.neighbors]}


def main():
    import jc_layout as jc
    import oracle.oracle as orc
    from conftest import ring_seed, spiral_seed

    out_dir = Path(__file__).resolve().parent
    fixtures = {}

    # generators (stability.rs fixtures)
    fixtures["gen_scale_free_64_3_c0ffee"] = csr_dict(jc.gen_scale_free(64, 3, 0xC0FFEE))
    fixtures["seed_ball_16_5eed"] = hexbits(jc.seed_ball(16, 0x5EED))
    fixtures["seed_uniform_8_3_7"] = hexbits(jc.seed_uniform(8, 3, 7))

    # FA2 cases: several steps from the oracle, first step cross-checked
    cases = {
        "fa2bh_path24_theta08": (jc.gen_path(24), spiral_seed(24), True, {"theta": 0.8}, 4),
        "fa2bh_path24_theta0": (jc.gen_path(24), spiral_seed(24), True, {"theta": 0.0}, 2),
        "fa2bh_grid6_theta07": (jc.gen_grid(6), spiral_seed(36), True, {"theta": 0.7}, 3),
        "fa2bh_sf200_ball": (jc.gen_scale_free(200, 3, 0xC0FFEE), jc.seed_ball(200, 0x5EED), True, {}, 3),
        "fa2brute_path24": (jc.gen_path(24), spiral_seed(24), False, {}, 2),
    }
    for name, (g, pos, bh, settings, steps) in cases.items():
        o = orc.Fa2(g, pos, bh=bh, **settings)
        rec = {"csr": csr_dict(g), "seed": hexbits(pos), "bh": bh, "settings": settings, "steps": []}
        for s in range(steps):
            o.step()
            r = o.get()
            rec["steps"].append({"pos": hexbits(r["pos"]), "force": hexbits(r["force"]), "stats": hexbits(r["stats"]),
                                 "speed": hexbits([r["speed"]])[0], "speed_eff": hexbits([r["speed_eff"]])[0]})
        if bh:
            p1, f1, s1, sp1, ef1 = py_fa2_step(g, pos, np.zeros(3 * g.n_nodes, np.float32), 1.0, 1.0,
                                               settings.get("theta", 0.7))
            first = rec["steps"][0]
            assert hexbits(f1) == first["force"], f"{name}: python restatement disagrees on forces"
            assert hexbits(s1) == first["stats"], f"{name}: python restatement disagrees on stats"
            assert hexbits([sp1])[0] == first["speed"], f"{name}: speed"
            assert hexbits(p1) == first["pos"], f"{name}: positions"
        fixtures[name] = rec

    # SGD: Jacobi (sgd_stress.wgsl) and CPU s_gd2 (sgd_stress.rs)
    for name, (g, pos, mode, steps) in {
        "sgd_jacobi_grid5": (jc.gen_grid(5), ring_seed(25), 1, 4),
        "sgd_cpu_path12": (jc.gen_path(12), ring_seed(12), 0, 5),
    }.items():
        o = orc.Sgd(g, pos, mode=mode)
        rec = {"csr": csr_dict(g), "seed": hexbits(pos), "mode": mode, "steps": []}
        for _ in range(steps):
            rec["steps"].append(hexbits(o.step()))
        fixtures[name] = rec

    path = out_dir / "layout_step_golden.json"
    path.write_text(json.dumps(fixtures, separators=(",", ":")))
    print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
