"""Seeded synthetic inputs for the fixpoint workloads.

The reference's drivers read TSV edge lists (``u\\tv\\n``; test/tc.cu:17-57)
and, for CSPA, a directory holding ``assign.facts`` and
``dereference.facts`` (test/cspa.cu:109-112).  No public dataset is needed:
every workload here is generated from a seed, with the shapes, sizes and
value distributions of the benchmark configurations:

* ``grid_edges``     – directed R x C grid, edges (r,c)->(r,c+1) and
                       (r,c)->(r+1,c), node id r*C+c (transitive closure).
* ``rmat_edges``     – R-MAT graph (Chakrabarti et al. 2004) with
                       probabilities a,b,c,d, self loops and duplicates
                       dropped, sampled until the requested edge count
                       (same generation).
* ``cspa_facts``     – assign / dereference pairs, source bounded Zipf(s)
                       over the variables, target uniform (CSPA).
* ``layered_dag``    – L layers of width W, every node with two out-edges
                       to uniform nodes of the next layer, duplicates
                       dropped (batched transitive closure).
* ``dag_batch``      – many layered DAGs with L, W log-uniform.

All arrays are ``numpy.uint64`` of shape (n, 2), row-major, which is the
host layout ``load_relation`` takes (src/relation.cu:815-838).
"""
from __future__ import annotations

import os

import numpy as np

U64 = np.uint64


def grid_edges(rows: int = 64, cols: int = 64) -> np.ndarray:
    """Directed grid: (r,c)->(r,c+1) and (r,c)->(r+1,c); id = r*cols + c."""
    r, c = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    node = (r * cols + c).ravel()
    right = (c < cols - 1).ravel()
    down = (r < rows - 1).ravel()
    e_right = np.stack([node[right], node[right] + 1], axis=1)
    e_down = np.stack([node[down], node[down] + cols], axis=1)
    return np.concatenate([e_right, e_down]).astype(U64)


def grid_tc_size(rows: int, cols: int) -> int:
    """Closure size of the directed grid: pairs (u,v), u != v, v reachable."""
    return (rows * (rows + 1) // 2) * (cols * (cols + 1) // 2) - rows * cols


def _dedup_in_order(pairs: np.ndarray) -> np.ndarray:
    """Keep the first occurrence of each row, in first-occurrence order."""
    if len(pairs) == 0:
        return pairs
    key = (pairs[:, 0].astype(np.uint64) << np.uint64(32)) | pairs[:, 1].astype(np.uint64)
    _, first = np.unique(key, return_index=True)
    return pairs[np.sort(first)]


def rmat_edges(scale: int, n_edges: int, a: float = 0.57, b: float = 0.19,
               c: float = 0.19, seed: int = 14) -> np.ndarray:
    """R-MAT edges on 2**scale nodes, no self loops, no duplicates.

    Each edge descends `scale` levels of the adjacency matrix, choosing the
    quadrant (src bit, dst bit) = (0,0),(0,1),(1,0),(1,1) with probability
    a, b, c, d = 1-a-b-c.  Edges are drawn in batches until `n_edges`
    distinct non-self-loop edges exist; the first `n_edges` in draw order
    are kept.
    """
    rng = np.random.default_rng(seed)
    have = np.zeros((0, 2), dtype=np.int64)
    cut_b, cut_c = a + b, a + b + c
    while len(have) < n_edges:
        m = max(2 * (n_edges - len(have)), 1024)
        x = rng.random((m, scale))
        src_bit = (x >= cut_b).astype(np.int64)
        dst_bit = (((x >= a) & (x < cut_b)) | (x >= cut_c)).astype(np.int64)
        weights = (1 << np.arange(scale - 1, -1, -1)).astype(np.int64)
        src = src_bit @ weights
        dst = dst_bit @ weights
        keep = src != dst
        batch = np.stack([src[keep], dst[keep]], axis=1)
        have = _dedup_in_order(np.concatenate([have, batch]))
    return have[:n_edges].astype(U64)


def bounded_zipf(rng: np.random.Generator, n_values: int, s: float, size: int) -> np.ndarray:
    """Draw `size` ranks in [0, n_values) with P(k) proportional to (k+1)^-s."""
    w = np.arange(1, n_values + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    return np.minimum(np.searchsorted(cdf, rng.random(size), side="right"), n_values - 1)


def cspa_facts(n_vars: int = 20000, n_assign: int = 40000, n_deref: int = 15000,
               s: float = 1.1, seed: int = 3) -> tuple[np.ndarray, np.ndarray]:
    """assign and dereference pairs: source ~ bounded Zipf(s), target uniform.

    Duplicates are kept (the engine deduplicates at load, as the reference
    does at src/relation.cu:586-590).
    """
    rng = np.random.default_rng(seed)

    def pairs(n):
        src = bounded_zipf(rng, n_vars, s, n)
        dst = rng.integers(0, n_vars, n)
        return np.stack([src, dst], axis=1).astype(U64)

    assign = pairs(n_assign)
    deref = pairs(n_deref)
    return assign, deref


def layered_dag(n_layers: int, width: int, seed: int) -> np.ndarray:
    """L layers of width W; each node of layer l < L-1 gets two out-edges to
    uniformly chosen nodes of layer l+1 (a collision leaves one edge).  Node
    id = layer * W + i."""
    rng = np.random.default_rng(seed)
    if n_layers < 2:
        return np.zeros((0, 2), dtype=U64)
    src = np.repeat(np.arange((n_layers - 1) * width), 2)
    layer = src // width
    dst = (layer + 1) * width + rng.integers(0, width, len(src))
    e = np.stack([src, dst], axis=1)
    return _dedup_in_order(e).astype(U64)


def log_uniform_int(rng: np.random.Generator, lo: int, hi: int) -> int:
    return int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))


def dag_batch(n_instances: int = 384, seed: int = 2024, l_range=(8, 128),
              w_range=(16, 256)) -> list[tuple[int, int, np.ndarray]]:
    """(L, W, edges) for each instance; L, W log-uniform; instance i's edges
    use seed + 1 + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_instances):
        L = log_uniform_int(rng, *l_range)
        W = log_uniform_int(rng, *w_range)
        out.append((L, W, layered_dag(L, W, seed + 1 + i)))
    return out


def reverse(edges):
    """(u,v) -> (v,u), the host-side reversal the drivers do before loading
    (test/tc.cu:97-101).  Device-resident rows (gdlog_b200.DeviceRows)
    return their reversed twin, also on the device."""
    if hasattr(edges, "reversed"):
        return edges.reversed()
    edges = np.asarray(edges)
    # two column copies: ~4x faster than copying the reversed strided view
    out = np.empty_like(edges, order="C")
    out[:, 0] = edges[:, 1]
    out[:, 1] = edges[:, 0]
    return out


def write_tsv(path: str, rows: np.ndarray) -> None:
    """Write rows as ``u\\tv\\n`` lines, the drivers' input format."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savetxt(path, rows.astype(np.int64), fmt="%d", delimiter="\t")


def read_tsv(path: str) -> np.ndarray:
    """Parse a ``u\\tv`` file the way get_relation_from_file does
    (test/tc.cu:31-57): one row per newline-terminated line."""
    data = np.loadtxt(path, dtype=np.int64, delimiter="\t", ndmin=2)
    return data.astype(U64)
