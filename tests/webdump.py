"""Writer of the reference pageRank app's on-disk input (test helper).

Layout, as the app reads it (pageRank.cpp:53-143): `<base>/web_dump_metadata`
holds three u32 (total pages, max out-links per page, pages per file); page
file `<base>/web/page_<1 + i * pages_per_file>` holds pages i*ppf .. of file i,
each page a u32 out-link count followed by max_outlinks u32 slots whose first
`count` are 1-based target page ids (the rest zero).  Graphs are seeded
synthetic: out-degrees uniform in [0, max_outlinks]; targets 1 + floor(n u^skew)
for uniform u, so skew > 1 concentrates in-links on low page ids (ranks in
the hundreds, which makes a lost subtask contribution visible even to the
app's own |serial - parallel| < 1 comparison).
"""
from __future__ import annotations

import os

import numpy as np


def make_dump(n_pages: int, max_outlinks: int, seed: int, skew: float = 1.0) -> np.ndarray:
    """Padded page records, shape (n_pages, max_outlinks + 1), uint32."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(0, max_outlinks + 1, n_pages, dtype=np.uint32)
    dump = np.zeros((n_pages, max_outlinks + 1), np.uint32)
    dump[:, 0] = counts
    u = rng.random((n_pages, max_outlinks))
    targets = np.minimum(1 + np.floor(n_pages * u ** skew), n_pages).astype(np.uint32)
    mask = np.arange(max_outlinks)[None, :] < counts[:, None]
    dump[:, 1:] = np.where(mask, targets, 0)
    return dump


def write_webdump(base: str, dump: np.ndarray, pages_per_file: int) -> None:
    n_pages, stride = dump.shape
    os.makedirs(os.path.join(base, "web"), exist_ok=True)
    np.array([n_pages, stride - 1, pages_per_file], np.uint32).tofile(os.path.join(base, "web_dump_metadata"))
    for first in range(0, n_pages, pages_per_file):
        dump[first:first + pages_per_file].tofile(os.path.join(base, "web", f"page_{first + 1}"))


def edges_of(dump: np.ndarray):
    """(src, dst) 0-based edge arrays in page order."""
    counts = dump[:, 0].astype(np.int64)
    mask = np.arange(dump.shape[1] - 1)[None, :] < counts[:, None]
    src = np.repeat(np.arange(dump.shape[0], dtype=np.uint32), counts)
    dst = (dump[:, 1:][mask] - 1).astype(np.uint32)
    return src, dst
