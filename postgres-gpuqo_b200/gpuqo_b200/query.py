"""Join-graph description and seeded synthetic generators.

A :class:`Query` holds exactly what the planner glue of the reference puts into
``GpuqoPlannerInfoC`` (src/include/optimizer/gpuqo_planner_info.h:180-189),
with relation ``i`` (0-based) carrying the Postgres relid bit ``i + 1``:

* per base relation: ``rows``, ``tuples``, ``cost = (startup, total)``,
  ``width`` (``BaseRelationC``, gpuqo_planner_info.h:172-178);
* the adjacency ``edges[i]`` (``edge_table``);
* the equivalence classes (``EqClassInfo``, gpuqo_planner_info.h:163-170):
  member relations in increasing index order, one selectivity per unordered
  member pair in ``eqClassIndex`` order (src/include/optimizer/gpuqo_common.h:
  72-79), one foreign-key target set per member and one ``VarInfo`` per member.

The generators follow the shapes of the reference's benchmark databases
(scripts/databases/star-small/star.py, snowflake-small/snowflake.py) with the
row/selectivity distributions of the workloads measured here:

* star: fact rows log-uniform [1e6, 1e8], dimensions [1e2, 1e5], FK-PK edges
  with selectivity 1/rows(dim);
* snowflake: a root with U{4..6} children, every node with U{0..3} children up
  to depth 4, grown or truncated to exactly n nodes; rows log-uniform
  [1e2, 1e8], FK-PK selectivity 1/rows(PK side);
* clique / chain / cycle: rows log-uniform [1e3, 1e6], per-edge selectivity
  log-uniform [1e-4, 1e-1], no foreign keys.

Relation indices are assigned by a seeded random permutation, so the fact
table is not always relation 0.  All numbers are rounded to float32 exactly
once, here, so every consumer sees identical bytes.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

CPU_TUPLE_COST = 0.01
SEQ_PAGE_COST = 1.0
BLCKSZ = 8192


def f32(x: float) -> float:
    return float(np.float32(x))


@dataclass
class VarInfo:
    """Column statistics and index info of one equivalence-class member."""
    stadistinct: float = 0.0
    stanullfrac: float = 0.0
    mcvfreq: float = 0.0
    index_available: bool = False
    index_unique: bool = False
    index_rows: float = 0.0
    index_startup: float = 0.0
    index_total: float = 0.0

    def to_list(self):
        return [self.stadistinct, self.stanullfrac, self.mcvfreq,
                int(self.index_available), int(self.index_unique),
                self.index_rows, self.index_startup, self.index_total]

    @staticmethod
    def from_list(v):
        return VarInfo(float(v[0]), float(v[1]), float(v[2]), bool(v[3]),
                       bool(v[4]), float(v[5]), float(v[6]), float(v[7]))


@dataclass
class EqClass:
    members: List[int]                 # relation indices, increasing
    sels: List[float]                  # len = s*(s-1)/2, eqClassIndex order
    fks: List[List[int]]               # per member: referenced relation indices
    vars: List[VarInfo]                # per member

    def to_dict(self):
        return {"members": self.members, "sels": self.sels, "fks": self.fks,
                "vars": [v.to_list() for v in self.vars]}

    @staticmethod
    def from_dict(d):
        return EqClass(list(d["members"]), [float(x) for x in d["sels"]],
                       [list(x) for x in d["fks"]],
                       [VarInfo.from_list(v) for v in d["vars"]])


@dataclass
class Query:
    n: int
    rows: List[float]
    tuples: List[float]
    startup: List[float]
    total: List[float]
    width: List[int]
    edges: List[List[int]]             # adjacency, relation indices
    eq_classes: List[EqClass]
    name: str = ""

    # ------------------------------------------------------------------
    def edge_masks(self) -> List[int]:
        """Adjacency as Postgres-relid bitmasks (bit j+1 for relation j)."""
        out = []
        for i in range(self.n):
            m = 0
            for j in self.edges[i]:
                m |= 1 << (j + 1)
            out.append(m)
        return out

    def to_dict(self):
        return {"name": self.name, "n": self.n, "rows": self.rows,
                "tuples": self.tuples, "startup": self.startup,
                "total": self.total, "width": self.width,
                "edges": self.edges,
                "eq_classes": [e.to_dict() for e in self.eq_classes]}

    @staticmethod
    def from_dict(d):
        return Query(int(d["n"]), [float(x) for x in d["rows"]],
                     [float(x) for x in d["tuples"]],
                     [float(x) for x in d["startup"]],
                     [float(x) for x in d["total"]],
                     [int(x) for x in d["width"]],
                     [list(x) for x in d["edges"]],
                     [EqClass.from_dict(e) for e in d["eq_classes"]],
                     d.get("name", ""))

    def to_json(self) -> str:
        return json.dumps(self.to_dict(), separators=(",", ":"))

    @staticmethod
    def from_json(s: str) -> "Query":
        return Query.from_dict(json.loads(s))


# ----------------------------------------------------------------------------
# generators
# ----------------------------------------------------------------------------

def _loguniform(rng, lo, hi, size=None):
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size))


def _base_cost(rows: float, width: int):
    pages = math.ceil(rows * width / BLCKSZ)
    return 0.0, f32(rows * CPU_TUPLE_COST + pages * SEQ_PAGE_COST)


def _assemble(name, n_logical, logical_rows, logical_width, logical_edges,
              rng, perm=None, rich=False):
    """Build a Query from logical nodes/edges.

    logical_edges: list of (a, b, sel, fk) with fk in {None, 'a', 'b'}; fk='a'
    means member a holds a foreign key referencing b's primary key.
    perm maps logical node -> relation index.
    rich: fill column statistics and unique indexes on PK sides so the
    index-nested-loop, inner-unique and hash-bucket branches of the cost model
    are exercised.
    """
    n = n_logical
    if perm is None:
        perm = rng.permutation(n)
    rows = [0.0] * n
    width = [0] * n
    for lg in range(n):
        rows[perm[lg]] = f32(round(float(logical_rows[lg])))
        width[perm[lg]] = int(logical_width[lg])
    tuples = list(rows)
    startup, total = [], []
    for i in range(n):
        s, t = _base_cost(rows[i], width[i])
        startup.append(s)
        total.append(t)
    adj = [set() for _ in range(n)]
    ecs = []
    for (a, b, sel, fk) in logical_edges:
        ra, rb = int(perm[a]), int(perm[b])
        adj[ra].add(rb)
        adj[rb].add(ra)
        members = sorted([ra, rb])
        fks = [[], []]
        vars_ = [VarInfo(), VarInfo()]
        if fk is not None:
            holder, target = (ra, rb) if fk == "a" else (rb, ra)
            fks[members.index(holder)] = [target]
            if rich:
                ti = members.index(target)
                hi = members.index(holder)
                vars_[ti] = VarInfo(stadistinct=-1.0, stanullfrac=0.0,
                                    mcvfreq=f32(1.0 / max(1.0, rows[target])),
                                    index_available=True, index_unique=True,
                                    index_rows=1.0,
                                    index_startup=f32(0.29),
                                    index_total=f32(8.31))
                vars_[hi] = VarInfo(stadistinct=f32(max(1.0, rows[target] * 0.5)),
                                    stanullfrac=f32(rng.uniform(0, 0.1)),
                                    mcvfreq=f32(rng.uniform(0.0, 0.05)))
        elif rich:
            for k in range(2):
                vars_[k] = VarInfo(stadistinct=f32(rng.uniform(-1.0, 1000.0)),
                                   stanullfrac=f32(rng.uniform(0, 0.2)),
                                   mcvfreq=f32(rng.uniform(0.0, 0.2)),
                                   index_available=bool(rng.integers(0, 2)),
                                   index_unique=bool(rng.integers(0, 2)),
                                   index_rows=f32(rng.uniform(1, 100)),
                                   index_startup=f32(rng.uniform(0, 1)),
                                   index_total=f32(rng.uniform(1, 50)))
        ecs.append(EqClass(members, [f32(sel)], fks, vars_))
    # deterministic eq-class order: by (first member, second member)
    ecs.sort(key=lambda e: tuple(e.members))
    q = Query(n, rows, tuples, startup, total, width,
              [sorted(a) for a in adj], ecs, name)
    return q


def star(n: int, seed: int, rich: bool = False) -> Query:
    rng = np.random.default_rng([seed, 1, n])
    lrows = [_loguniform(rng, 1e6, 1e8)] + list(_loguniform(rng, 1e2, 1e5, n - 1))
    lwidth = [8] * n
    edges = []
    for d in range(1, n):
        edges.append((0, d, 1.0 / f32(round(float(lrows[d]))), "a"))
    return _assemble(f"star{n}_s{seed}", n, lrows, lwidth, edges, rng, rich=rich)


def snowflake_tree(n: int, rng) -> List[tuple]:
    """Parent links of a snowflake: root 0 with U{4..6} children, others
    U{0..3} children, depth <= 4, exactly n nodes."""
    parent = [-1]
    depth = [0]
    frontier = [0]
    first = True
    while frontier and len(parent) < n:
        nxt = []
        for u in frontier:
            k = int(rng.integers(4, 7)) if first else int(rng.integers(0, 4))
            if depth[u] >= 4:
                k = 0
            for _ in range(k):
                if len(parent) >= n:
                    break
                parent.append(u)
                depth.append(depth[u] + 1)
                nxt.append(len(parent) - 1)
            first = False
        frontier = nxt
    while len(parent) < n:
        cands = [u for u in range(len(parent)) if depth[u] < 4]
        u = cands[int(rng.integers(0, len(cands)))]
        parent.append(u)
        depth.append(depth[u] + 1)
    return parent


def snowflake(n: int, seed: int, rich: bool = False) -> Query:
    rng = np.random.default_rng([seed, 2, n])
    parent = snowflake_tree(n, rng)
    lrows = _loguniform(rng, 1e2, 1e8, n)
    lwidth = [8] * n
    edges = []
    for c in range(1, n):
        p = parent[c]
        # the parent holds the foreign key, the child's primary key is referenced
        edges.append((p, c, 1.0 / f32(round(float(lrows[c]))), "a"))
    return _assemble(f"snowflake{n}_s{seed}", n, lrows, lwidth, edges, rng, rich=rich)


def _plain_edges(pairs, rng):
    return [(a, b, float(_loguniform(rng, 1e-4, 1e-1)), None) for (a, b) in pairs]


def clique(n: int, seed: int, rich: bool = False) -> Query:
    rng = np.random.default_rng([seed, 3, n])
    lrows = _loguniform(rng, 1e3, 1e6, n)
    pairs = [(a, b) for a in range(n) for b in range(a + 1, n)]
    return _assemble(f"clique{n}_s{seed}", n, lrows, [8] * n,
                     _plain_edges(pairs, rng), rng, rich=rich)


def chain(n: int, seed: int, rich: bool = False) -> Query:
    rng = np.random.default_rng([seed, 4, n])
    lrows = _loguniform(rng, 1e3, 1e6, n)
    pairs = [(a, a + 1) for a in range(n - 1)]
    return _assemble(f"chain{n}_s{seed}", n, lrows, [8] * n,
                     _plain_edges(pairs, rng), rng, rich=rich)


def cycle(n: int, seed: int, rich: bool = False) -> Query:
    rng = np.random.default_rng([seed, 5, n])
    lrows = _loguniform(rng, 1e3, 1e6, n)
    pairs = [(a, a + 1) for a in range(n - 1)] + [(0, n - 1)]
    return _assemble(f"cycle{n}_s{seed}", n, lrows, [8] * n,
                     _plain_edges(pairs, rng), rng, rich=rich)


def _key_edges(pairs, lrows):
    """Key joins: in each pair (a, b) a references b's primary key
    (selectivity 1 / rows of b), so a path's row estimate stays that of its
    first relation and long paths do not overflow float32."""
    return [(a, b, 1.0 / f32(round(float(lrows[b]))), "a") for (a, b) in pairs]


def key_chain(n: int, seed: int, rich: bool = False) -> Query:
    """A chain of n relations joined on keys, each referencing the next."""
    rng = np.random.default_rng([seed, 10, n])
    lrows = _loguniform(rng, 1e2, 1e7, n)
    lwidth = [int(w) for w in rng.integers(4, 65, n)]
    pairs = [(a, a + 1) for a in range(n - 1)]
    return _assemble(f"key_chain{n}_s{seed}", n, lrows, lwidth, _key_edges(pairs, lrows), rng, rich=rich)


def key_cycle(n: int, seed: int, rich: bool = False) -> Query:
    """A cycle of n relations joined on keys (one biconnected block)."""
    rng = np.random.default_rng([seed, 11, n])
    lrows = _loguniform(rng, 1e2, 1e7, n)
    lwidth = [int(w) for w in rng.integers(4, 65, n)]
    pairs = [(a, a + 1) for a in range(n - 1)] + [(n - 1, 0)]
    return _assemble(f"key_cycle{n}_s{seed}", n, lrows, lwidth, _key_edges(pairs, lrows), rng, rich=rich)


def ring_path(n: int, seed: int, rich: bool = False) -> Query:
    """Rings of 4 to 6 relations alternating with paths of 4 to 8 relations
    (biconnected blocks that are cycles, joined by bridges), key joins along
    the way."""
    rng = np.random.default_rng([seed, 12, n])
    lrows = _loguniform(rng, 1e2, 1e7, n)
    lwidth = [int(w) for w in rng.integers(4, 65, n)]
    pairs = []
    cur, nxt, ring = 0, 1, True
    while nxt < n:
        m = int(rng.integers(4, 7)) if ring else int(rng.integers(4, 9)) + 1
        seg = list(range(nxt, min(n, nxt + m - 1)))
        nxt += len(seg)
        path = [cur] + seg
        pairs += [(path[i], path[i + 1]) for i in range(len(path) - 1)]
        if ring and len(seg) == m - 1:
            pairs.append((path[-1], cur))
        cur = seg[len(seg) // 2] if ring else seg[-1]
        ring = not ring
    return _assemble(f"ring_path{n}_s{seed}", n, lrows, lwidth, _key_edges(pairs, lrows), rng, rich=rich)


def lollipop(n: int, seed: int, rich: bool = False) -> Query:
    """A cycle of n // 3 relations with a path of the others hanging off it."""
    rng = np.random.default_rng([seed, 13, n])
    lrows = _loguniform(rng, 1e2, 1e7, n)
    lwidth = [int(w) for w in rng.integers(4, 65, n)]
    m = n // 3
    pairs = [(a, a + 1) for a in range(m - 1)] + [(m - 1, 0), (0, m)] + [(a, a + 1) for a in range(m, n - 1)]
    return _assemble(f"lollipop{n}_s{seed}", n, lrows, lwidth, _key_edges(pairs, lrows), rng, rich=rich)


def random_graph(n: int, seed: int, extra_edge_p: float = 0.2,
                 rich: bool = False, equal: bool = False) -> Query:
    """A random connected graph: a random spanning tree plus extra edges with
    probability extra_edge_p.  equal=True makes every relation and edge
    identical, which maximises exact cost ties (tie-breaking tests)."""
    rng = np.random.default_rng([seed, 6, n])
    parent = [-1] + [int(rng.integers(0, i)) for i in range(1, n)]
    pairs = set((parent[i], i) for i in range(1, n))
    for a in range(n):
        for b in range(a + 1, n):
            if (a, b) not in pairs and rng.uniform() < extra_edge_p:
                pairs.add((a, b))
    pairs = sorted(pairs)
    if equal:
        lrows = [1000.0] * n
        edges = [(a, b, 0.01, None) for (a, b) in pairs]
    else:
        lrows = _loguniform(rng, 1e2, 1e6, n)
        edges = []
        for (a, b) in pairs:
            if rng.uniform() < 0.5:
                edges.append((a, b, 1.0 / f32(round(float(lrows[b]))), "a"))
            else:
                edges.append((a, b, float(_loguniform(rng, 1e-4, 1e-1)), None))
    lwidth = [int(w) for w in rng.integers(4, 65, n)]
    return _assemble(f"random{n}_s{seed}", n, lrows, lwidth, edges, rng, rich=rich)


def multi_member_classes(n: int, seed: int) -> Query:
    """A chain whose equivalence classes span three or more relations
    (A.x = B.x = C.x), exercising eqClassIndex, multi-member selectivity
    lookup and multi-member foreign keys."""
    rng = np.random.default_rng([seed, 7, n])
    lrows = _loguniform(rng, 1e2, 1e6, n)
    perm = rng.permutation(n)
    q = _assemble(f"multi{n}_s{seed}", n, lrows, [8] * n,
                  [(a, a + 1, float(_loguniform(rng, 1e-4, 1e-1)), None)
                   for a in range(n - 1)], rng, perm=perm, rich=True)
    # add a few wide classes over consecutive relations
    for start in range(0, n - 2, 3):
        mem_logical = list(range(start, min(n, start + 3 + int(rng.integers(0, 2)))))
        members = sorted(int(perm[m]) for m in mem_logical)
        s = len(members)
        sels = [f32(_loguniform(rng, 1e-4, 1e-1)) for _ in range(s * (s - 1) // 2)]
        fks = [[] for _ in range(s)]
        fks[0] = [members[-1]]
        vars_ = [VarInfo(stadistinct=f32(rng.uniform(1, 500)),
                         stanullfrac=f32(rng.uniform(0, 0.1)),
                         mcvfreq=f32(rng.uniform(0, 0.1)),
                         index_available=bool(rng.integers(0, 2)),
                         index_unique=bool(rng.integers(0, 2)),
                         index_rows=f32(rng.uniform(1, 10)),
                         index_startup=f32(0.3), index_total=f32(rng.uniform(1, 20)))
                 for _ in range(s)]
        for i in range(s):
            for j in range(i + 1, s):
                a, b = members[i], members[j]
                if b not in q.edges[a]:
                    q.edges[a] = sorted(q.edges[a] + [b])
                    q.edges[b] = sorted(q.edges[b] + [a])
        q.eq_classes.append(EqClass(members, sels, fks, vars_))
    return q


SHAPES = {"star": star, "snowflake": snowflake, "clique": clique,
          "chain": chain, "cycle": cycle, "key_chain": key_chain,
          "key_cycle": key_cycle, "ring_path": ring_path,
          "lollipop": lollipop}


def make(shape: str, n: int, seed: int, **kw) -> Query:
    return SHAPES[shape](n, seed, **kw)


def batch_mix(n_queries: int, seed: int, nmin: int = 8, nmax: int = 28) -> List[Query]:
    """The batched workload: relation counts uniform in [nmin, nmax], shapes
    40% star / 40% snowflake / 10% chain / 10% cycle, each query seeded."""
    rng = np.random.default_rng([seed, 8, n_queries, nmin, nmax])
    out = []
    for i in range(n_queries):
        n = int(rng.integers(nmin, nmax + 1))
        u = rng.uniform()
        if u < 0.4:
            q = star(n, seed * 100003 + i)
        elif u < 0.8:
            q = snowflake(n, seed * 100003 + i)
        elif u < 0.9:
            q = chain(max(n, 2), seed * 100003 + i)
        else:
            q = cycle(max(n, 3), seed * 100003 + i)
        out.append(q)
    return out
