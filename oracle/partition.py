"""CPU oracle for edge-cut partitioning — TEST INFRASTRUCTURE ONLY.

A plain-Python restatement of crates/graph-compute/src/partition.rs, used by
tests/ to check the library's partitioner (jump-cannon_b200/csrc/jc_partition.cu)
partition for partition:
  * assign_owners_bfs            partition.rs:244-293
  * build_partition              partition.rs:298-431 (attributes left out)
  * edge_cut / edge_cut_owner    partition.rs:456-477
  * refine_partitions (FM)       partition.rs:550-643 (tolerance 0.10, 8 passes)
Pinned by the reference's own partition tests, restated in
tests/test_partition.py (path(6) split in two, the 8-node graph whose BFS
cut of 3 refines to 1, boundary == owned nodes that are peers' ghosts).
"""
from __future__ import annotations

import math
from collections import deque
from dataclasses import dataclass, field

UNSET = 0xFFFFFFFF


@dataclass
class Part:
    partition_id: int
    n_partitions: int
    n_owned: int
    offsets: list = field(default_factory=lambda: [0])
    neighbors: list = field(default_factory=list)
    global_ids: list = field(default_factory=list)
    boundary: list = field(default_factory=list)


def assign_owners_bfs(n, off, nbr, p):
    target = max(-(-n // p), 1)
    owner = [UNSET] * n
    assigned = 0
    next_seed = 0
    for pid in range(p):
        cap = math.inf if pid + 1 == p else target
        count = 0
        queue = deque()
        while count < cap and assigned < n:
            if not queue:
                while next_seed < n and owner[next_seed] != UNSET:
                    next_seed += 1
                if next_seed >= n:
                    break
                queue.append(next_seed)
                owner[next_seed] = pid
                assigned += 1
                count += 1
            if not queue:
                break
            v = queue.popleft()
            for u in nbr[off[v]:off[v + 1]]:
                if owner[u] == UNSET and count < cap:
                    owner[u] = pid
                    assigned += 1
                    count += 1
                    queue.append(u)
    return [p - 1 if o == UNSET else o for o in owner]


def build_partition(n, off, nbr, owner, pid, p, owned_ids):
    n_owned = len(owned_ids)
    global_ids = list(owned_ids)
    g2l = {g: i for i, g in enumerate(owned_ids)}
    ghosts, boundary = [], []
    for g in owned_ids:
        is_b = False
        for u in nbr[off[g]:off[g + 1]]:
            if owner[u] != pid:
                is_b = True
                if u not in g2l:
                    g2l[u] = n_owned + len(ghosts)
                    ghosts.append(u)
        if is_b:
            boundary.append(g)
    global_ids += ghosts
    offsets, neighbors = [0], []
    for li in range(len(global_ids)):
        if li < n_owned:
            g = global_ids[li]
            for u in nbr[off[g]:off[g + 1]]:
                if u in g2l:
                    neighbors.append(g2l[u])
        offsets.append(len(neighbors))
    return Part(pid, p, n_owned, offsets, neighbors, global_ids, boundary)


def build_from_owner(n, off, nbr, owner, p):
    owned = [[] for _ in range(p)]
    for g, o in enumerate(owner):
        owned[o].append(g)
    return [build_partition(n, off, nbr, owner, pid, p, owned[pid]) for pid in range(p)]


def partition_csr(n, off, nbr, n_partitions):
    p = max(n_partitions, 1)
    if n == 0:
        return [Part(pid, p, 0) for pid in range(p)]
    owner = assign_owners_bfs(n, off, nbr, p)
    return build_from_owner(n, off, nbr, owner, p)


def owner_of(parts, n):
    owner = [0] * n
    for part in parts:
        for g in part.global_ids[:part.n_owned]:
            owner[g] = part.partition_id
    return owner


def edge_cut(parts, n, off, nbr):
    owner = owner_of(parts, n)
    return sum(1 for u in range(n) for v in nbr[off[u]:off[u + 1]] if u < v and owner[u] != owner[v])


def refine_partitions(n, off, nbr, parts):
    if not parts:
        return parts
    p = parts[0].n_partitions
    if n == 0 or p <= 1:
        return parts
    owner = owner_of(parts, n)
    sizes = [0] * p
    for o in owner:
        sizes[o] += 1
    ideal = n / p
    max_size = math.ceil((1.0 + 0.10) * ideal)
    min_size = math.floor((1.0 - 0.10) * ideal)
    for _ in range(8):
        moved = False
        for v in range(n):
            a = owner[v]
            internal = 0
            ext = [0] * p
            for u in nbr[off[v]:off[v + 1]]:
                if u == v:
                    continue
                if owner[u] == a:
                    internal += 1
                else:
                    ext[owner[u]] += 1
            best, best_ext = None, 0
            for b, e in enumerate(ext):
                if b == a or e == 0:
                    continue
                if e > best_ext:
                    best_ext, best = e, b
            if best is None:
                continue
            if best_ext - internal <= 0:
                continue
            if sizes[best] + 1 > max_size:
                continue
            if max(sizes[a] - 1, 0) < min_size:
                continue
            owner[v] = best
            sizes[a] -= 1
            sizes[best] += 1
            moved = True
        if not moved:
            break
    return build_from_owner(n, off, nbr, owner, p)


def partition_csr_refined(n, off, nbr, n_partitions):
    return refine_partitions(n, off, nbr, partition_csr(n, off, nbr, n_partitions))
