"""Writers and readers for the reference's on-disk formats.

* ``_disk.index`` -- DiskANN's page-laid graph file as the reference reads it
  (``Layout::parse_diskann_metadata``, src/layout.cpp:11-69; records read at
  src/impl/pure_mem.cuh:261-292): a 4096-byte first sector holding a
  ``uint32 nr, uint32 nc=1`` metadata block of ``uint64`` values
  ``[n, dim, medoid, max_node_len, nodes_per_sector, num_frozen, frozen_id,
  reorder_exists, file_size]``, then pages of ``nodes_per_sector`` records
  ``[vector dim*elt][uint32 deg][uint32 nbr * R]``.
* ``<prefix>_pq_pivots.bin`` / ``<prefix>_pq_compressed.bin`` -- DiskANN's PQ
  files as read by ``PQSearch::read_data`` (src/pq_search.cu:56-121): an offsets
  block (4 x 1 uint64: pivots, centroid, chunk offsets, file size), the pivots
  ``256 x dim`` float, the centroid ``dim x 1`` float and the chunk offsets
  ``(M+1) x 1`` uint32; codes ``n x M`` uint8.
* pivot graph directory -- ``nav_index`` (DiskANN in-memory graph: uint64 size,
  uint32 max degree, uint32 start, uint64 frozen, then ``uint32 deg, deg x uint32``
  per node), ``nav_index.data`` (``int n, int dim``, vectors) and ``map.txt``
  (one global id per line), as read by ``NavGraph::init`` (src/nav_graph.cu:41-100).
* ``fvecs``/``bvecs``/``ivecs`` query and ground-truth files
  (bin/utils.hpp:24-102).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np

PAGE = 4096


def node_len(dim: int, elt: int, R: int) -> int:
    return dim * elt + (R + 1) * 4


def write_disk_index(path: str, data: np.ndarray, graph: np.ndarray, degrees: np.ndarray,
                     medoid: int, R: int, chunk_nodes: int = 1 << 20) -> dict:
    """Write ``data`` (n x dim, uint8 or float32) with adjacency ``graph``
    (n x >=R int32, rows padded) and ``degrees`` (n) as a DiskANN _disk.index."""
    n, dim = data.shape
    elt = data.dtype.itemsize
    if data.dtype not in (np.uint8, np.float32):
        raise ValueError("data must be uint8 or float32")
    nl = node_len(dim, elt, R)
    npp = PAGE // nl
    if npp < 1:
        raise ValueError("a node does not fit one 4 KB page")
    num_pages = (n + npp - 1) // npp
    file_size = PAGE * (num_pages + 1)
    meta = np.array([n, dim, medoid, nl, npp, 0, 0, 0, file_size], dtype=np.uint64)
    header = np.zeros(PAGE, dtype=np.uint8)
    hb = struct.pack("<II", len(meta), 1) + meta.tobytes()
    header[: len(hb)] = np.frombuffer(hb, dtype=np.uint8)
    with open(path, "wb") as f:
        f.write(header.tobytes())
        step = max(npp, (chunk_nodes // npp) * npp)
        for s in range(0, n, step):
            e = min(n, s + step)
            cnt = e - s
            rec = np.zeros((cnt, nl), dtype=np.uint8)
            rec[:, : dim * elt] = np.ascontiguousarray(data[s:e]).view(np.uint8).reshape(cnt, dim * elt)
            adj = np.zeros((cnt, R + 1), dtype=np.uint32)
            deg = np.asarray(degrees[s:e], dtype=np.int64)
            adj[:, 0] = deg
            g = np.asarray(graph[s:e, :R], dtype=np.int64)
            mask = np.arange(R)[None, :] < deg[:, None]
            adj[:, 1:] = np.where(mask, g, 0).astype(np.uint32)
            rec[:, dim * elt:] = adj.view(np.uint8).reshape(cnt, (R + 1) * 4)
            pages = (cnt + npp - 1) // npp
            buf = np.zeros((pages, PAGE), dtype=np.uint8)
            full = np.zeros((pages * npp, nl), dtype=np.uint8)
            full[:cnt] = rec
            buf[:, : npp * nl] = full.reshape(pages, npp * nl)
            f.write(buf.tobytes())
    return {"n": n, "dim": dim, "node_len": nl, "npp": npp, "num_pages": num_pages, "R": R}


def write_disk_index_torch(path: str, x, graph, degrees, medoid: int, R: int, chunk_nodes: int = 1 << 20) -> dict:
    """write_disk_index for tensors on the GPU: every chunk of pages is laid
    out on the device (vector, degree, neighbour slots, zero padding) and
    written as it is copied back, so no host copy of the whole base is made.
    ``graph`` rows hold their neighbours first (``degrees`` of them)."""
    import torch

    n, dim = x.shape
    if x.dtype not in (torch.uint8, torch.float32):
        raise ValueError("data must be uint8 or float32")
    elt = x.element_size()
    nl = node_len(dim, elt, R)
    npp = PAGE // nl
    if npp < 1:
        raise ValueError("a node does not fit one 4 KB page")
    num_pages = (n + npp - 1) // npp
    file_size = PAGE * (num_pages + 1)
    meta = np.array([n, dim, medoid, nl, npp, 0, 0, 0, file_size], dtype=np.uint64)
    header = np.zeros(PAGE, dtype=np.uint8)
    hb = struct.pack("<II", len(meta), 1) + meta.tobytes()
    header[: len(hb)] = np.frombuffer(hb, dtype=np.uint8)
    dev = x.device
    cols = torch.arange(R, device=dev)
    with open(path, "wb") as f:
        f.write(header.tobytes())
        step = max(npp, (chunk_nodes // npp) * npp)
        for s in range(0, n, step):
            e = min(n, s + step)
            cnt = e - s
            pages = (cnt + npp - 1) // npp
            rec = torch.zeros((pages * npp, nl), dtype=torch.uint8, device=dev)
            rec[:cnt, : dim * elt] = x[s:e].contiguous().view(torch.uint8).view(cnt, dim * elt)
            deg = degrees[s:e].to(device=dev, dtype=torch.int32)
            adj = torch.zeros((cnt, R + 1), dtype=torch.int32, device=dev)
            adj[:, 0] = deg
            adj[:, 1:] = torch.where(cols[None, :] < deg[:, None], graph[s:e, :R].to(device=dev, dtype=torch.int32),
                                     torch.zeros((), dtype=torch.int32, device=dev))
            rec[:cnt, dim * elt:] = adj.view(torch.uint8).view(cnt, (R + 1) * 4)
            pg = torch.zeros((pages, PAGE), dtype=torch.uint8, device=dev)
            pg[:, : npp * nl] = rec.view(pages, npp * nl)
            f.write(pg.cpu().numpy())
    return {"n": n, "dim": dim, "node_len": nl, "npp": npp, "num_pages": num_pages, "R": R}


def _bin_block(arr: np.ndarray) -> bytes:
    rows, cols = arr.shape
    return struct.pack("<ii", rows, cols) + np.ascontiguousarray(arr).tobytes()


def write_pq(prefix: str, pivots: np.ndarray, centroid: np.ndarray, chunk_offsets: np.ndarray,
             codes: np.ndarray, legacy: bool = False) -> None:
    """Write ``<prefix>_pivots.bin`` and ``<prefix>_compressed.bin``. ``legacy``
    writes the 5-entry offsets table (pq_search.cu:78-100 reads the chunk
    offsets from entry 3 then)."""
    pivots = np.asarray(pivots, dtype=np.float32)
    assert pivots.shape[0] == 256
    dim = pivots.shape[1]
    blocks = [
        _bin_block(pivots),
        _bin_block(np.asarray(centroid, dtype=np.float32).reshape(dim, 1)),
        _bin_block(np.asarray(chunk_offsets, dtype=np.uint32).reshape(-1, 1)),
    ]
    if legacy:  # rearrangement block sits at entry 2, chunk offsets at entry 3
        blocks.insert(2, _bin_block(np.arange(dim, dtype=np.uint32).reshape(-1, 1)))
    nr = len(blocks) + 1
    offs = []
    pos = PAGE
    for b in blocks:
        offs.append(pos)
        pos += len(b)
    offs.append(pos)
    with open(prefix + "_pivots.bin", "wb") as f:
        head = _bin_block(np.array(offs, dtype=np.uint64).reshape(nr, 1))
        f.write(head + b"\0" * (PAGE - len(head)))
        for b in blocks:
            f.write(b)
    with open(prefix + "_compressed.bin", "wb") as f:
        f.write(_bin_block(np.asarray(codes, dtype=np.uint8)))


def write_nav(directory: str, data: np.ndarray, graph: np.ndarray, degrees: np.ndarray, start: int,
              mapping: np.ndarray) -> None:
    """Write a pivot graph directory (``nav_index``, ``nav_index.data``, ``map.txt``)."""
    os.makedirs(directory, exist_ok=True)
    n, dim = data.shape
    with open(os.path.join(directory, "nav_index.data"), "wb") as f:
        f.write(struct.pack("<ii", n, dim))
        f.write(np.ascontiguousarray(data).tobytes())
    with open(os.path.join(directory, "map.txt"), "w") as f:
        f.write("\n".join(str(int(x)) for x in mapping) + "\n")
    degrees = np.asarray(degrees, dtype=np.int64)
    max_deg = int(degrees.max()) if n else 0
    graph = np.asarray(graph)
    starts = np.cumsum(degrees + 1) - (degrees + 1)
    body = np.empty(int((degrees + 1).sum()), dtype=np.uint32)
    body[starts] = degrees
    cols = np.arange(graph.shape[1] if graph.ndim == 2 else 0)
    mask = cols[None, :] < degrees[:, None]
    body[(starts[:, None] + 1 + cols[None, :])[mask]] = graph[mask].astype(np.uint32)
    size = 24 + body.nbytes
    with open(os.path.join(directory, "nav_index"), "wb") as f:
        f.write(struct.pack("<QIIQ", size, max_deg, start, 0))
        f.write(body.tobytes())


@dataclass
class DiskIndex:
    n: int
    dim: int
    medoid: int
    node_len: int
    npp: int
    R: int
    data: np.ndarray
    degrees: np.ndarray
    graph: np.ndarray


def read_disk_index(path: str, dtype) -> DiskIndex:
    """Parse a _disk.index back into arrays (tests and tooling)."""
    dtype = np.dtype(dtype)
    raw = np.fromfile(path, dtype=np.uint8)
    nr, nc = struct.unpack_from("<II", raw, 0)
    n, dim, medoid, nl, npp = struct.unpack_from("<5Q", raw, 8)
    elt = dtype.itemsize
    R = (nl - dim * elt) // 4 - 1
    pages = raw[PAGE:].reshape(-1, PAGE)[:, : npp * nl].reshape(-1, nl)[:n]
    data = np.ascontiguousarray(pages[:, : dim * elt]).view(dtype).reshape(n, dim)
    adj = np.ascontiguousarray(pages[:, dim * elt:]).view(np.uint32).reshape(n, R + 1)
    return DiskIndex(n, dim, medoid, nl, npp, R, data, adj[:, 0].astype(np.int32),
                     adj[:, 1:].astype(np.int32))


def read_index_vectors(path: str, dtype, ids: np.ndarray) -> np.ndarray:
    """The vectors of the given node ids from a _disk.index, read through a
    memory map page by page (no full load)."""
    dtype = np.dtype(dtype)
    head = np.fromfile(path, dtype=np.uint8, count=8 + 5 * 8)
    n, dim, medoid, nl, npp = struct.unpack_from("<5Q", head.tobytes(), 8)
    mm = np.memmap(path, dtype=np.uint8, mode="r")
    ids = np.asarray(ids, dtype=np.int64).reshape(-1)
    off = PAGE + (ids // npp) * PAGE + (ids % npp) * nl
    nbytes = dim * dtype.itemsize
    rows = np.stack([np.asarray(mm[o:o + nbytes]) for o in off]) if len(ids) else np.zeros((0, nbytes), np.uint8)
    return np.ascontiguousarray(rows).view(dtype).reshape(len(ids), dim)


def read_pq_pivots(prefix: str):
    """(pivots 256 x dim float32, centroid dim float32, chunk offsets M + 1
    uint32) from <prefix>_pivots.bin, either offsets-table size (4 or the
    legacy 5, PQSearch::read_data, src/pq_search.cu:74-100)."""
    raw = open(prefix + "_pivots.bin", "rb").read()
    nr = struct.unpack_from("<i", raw, 0)[0]
    offs = np.frombuffer(raw, np.uint64, count=nr, offset=8)
    rows, dim = struct.unpack_from("<ii", raw, int(offs[0]))
    piv = np.frombuffer(raw, np.float32, count=256 * dim, offset=int(offs[0]) + 8).reshape(256, dim)
    mu = np.frombuffer(raw, np.float32, count=dim, offset=int(offs[1]) + 8)
    co_off = int(offs[3 if nr == 5 else 2])
    m1 = struct.unpack_from("<i", raw, co_off)[0]
    co = np.frombuffer(raw, np.uint32, count=m1, offset=co_off + 8)
    return piv.copy(), mu.copy(), co.copy()


def write_vecs(path: str, arr: np.ndarray) -> None:
    """fvecs (float32), ivecs (int32) or bvecs (uint8): per row a 4-byte dim then the row."""
    arr = np.ascontiguousarray(arr)
    n, d = arr.shape
    with open(path, "wb") as f:
        hdr = np.full((n, 1), d, dtype=np.int32).view(np.uint8)
        body = arr.view(np.uint8).reshape(n, d * arr.dtype.itemsize)
        f.write(np.concatenate([hdr, body], axis=1).tobytes())


def read_vecs(path: str, dtype) -> np.ndarray:
    """Inverse of write_vecs (fvecs_read / bvecs_read / ivecs_read, bin/utils.hpp:24-95)."""
    dtype = np.dtype(dtype)
    raw = np.fromfile(path, dtype=np.uint8)
    d = int(raw[:4].view(np.int32)[0])
    row = 4 + d * dtype.itemsize
    rows = raw.reshape(-1, row)
    return np.ascontiguousarray(rows[:, 4:]).view(dtype).reshape(-1, d)


def write_bin(path: str, arr: np.ndarray) -> None:
    """DiskANN .bin: int32 n, int32 dim, then the rows."""
    arr = np.ascontiguousarray(arr)
    with open(path, "wb") as f:
        f.write(struct.pack("<ii", arr.shape[0], arr.shape[1]))
        f.write(arr.tobytes())
