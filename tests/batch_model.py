"""CPU model of the batched walk with FP32 tables (test infrastructure).

The batched form's results depend only on the query, L, k and W, never on
warp timing or on what its visited cache holds. This model restates those
semantics without any cache, one step at a time:

* the list starts with the entry node (its ADC key), unexpanded;
* a step picks the first W unexpanded entries; every neighbour of every pick
  is scored by ADC (FP32 table built in the reference's order; for M a multiple
  of 16 four quarter sums in chunk order, combined (q0 + q1) + (q2 + q3),
  otherwise one sequential sum) and survives if the list is not full or its
  key (distance, id) is below the last entry's, and it is not in the list;
* the picks' exact distances (int32 for uint8 vectors with an integral query,
  else FP32 in the reference's lane-strided order) enter the top-k in pick
  order, a new value after equal ones;
* the survivors (each id once) merge into the list by key, which keeps L.

The oracle supplies the entry node, the FP32 table and the FP32 exact distance.
"""
import bisect

import numpy as np


class BatchModel:
    def __init__(self, oracle_mod, meta):
        from gustann_b200.indexing import formats

        self.om = oracle_mod
        self.o = oracle_mod.Oracle(meta["index_file"], meta["pq_prefix"], meta["nav_dir"], meta["dtype"])
        di = formats.read_disk_index(meta["index_file"], np.uint8 if meta["dtype"] == 0 else np.float32)
        self.data, self.deg, self.graph = di.data, di.degrees, di.graph
        self.M = meta["M"]
        self.codes = np.fromfile(meta["pq_prefix"] + "_compressed.bin", np.uint8)[8:].reshape(di.n, self.M)
        self.u8 = meta["dtype"] == 0

    def adc(self, table, vs):
        c = self.codes[vs]
        M = self.M
        if M % 16 == 0:
            qn = M // 4
            parts = []
            for qq in range(4):
                d = np.zeros(len(vs), np.float32)
                for j in range(qq * qn, (qq + 1) * qn):
                    d = (d + table[j, c[:, j]]).astype(np.float32)
                parts.append(d)
            return ((parts[0] + parts[1]).astype(np.float32) + (parts[2] + parts[3]).astype(np.float32)).astype(
                np.float32)
        d = np.zeros(len(vs), np.float32)
        for j in range(M):
            d = (d + table[j, c[:, j]]).astype(np.float32)
        return d

    def exact(self, q, u, int_query):
        v = self.data[u]
        if int_query:
            return np.float32(int(((q.astype(np.int64) - v.astype(np.int64)) ** 2).sum()))
        return np.float32(self.om.exact_dist(q, v, True))

    def search(self, queries, k, L, W, entries=None):
        """entries: the entry node of each query, or None for the pivot-graph
        walk's (the oracle's nav walk)."""
        queries = np.ascontiguousarray(queries, dtype=np.float32)
        ents = self.o.search(queries, 1, 1)[5] if entries is None else np.asarray(entries)
        nq = len(queries)
        ids = np.zeros((nq, k), np.int32)
        dis = np.zeros((nq, k), np.float32)
        fnd = np.zeros(nq, np.int32)
        for qi in range(nq):
            r = self.search_one(queries[qi], int(ents[qi]), k, L, W)
            fnd[qi] = len(r)
            for j, (d, u) in enumerate(r):
                ids[qi, j], dis[qi, j] = u, d
        return ids, dis, fnd

    def search_one(self, q, u0, k, L, W):
        table, _ = self.o.pq_table(q)
        int_query = self.u8 and bool(np.all((q == np.rint(q)) & (q >= 0) & (q <= 255)))
        keys = [(float(self.adc(table, np.array([u0]))[0]), u0)]
        expanded = [False]
        top = []  # (distance, id) in top-k order
        while True:
            picks = [i for i in range(len(keys)) if not expanded[i]][:W]
            if not picks:
                break
            full = len(keys) == L
            tail = keys[-1] if full else None
            surv = {}
            for p in picks:
                u = keys[p][1]
                nb = self.graph[u, :self.deg[u]]
                if len(nb) == 0:
                    continue
                ds = self.adc(table, nb)
                for v, d in zip(nb.tolist(), ds.tolist()):
                    key = (d, v)
                    if full and not key < tail:
                        continue
                    lb = bisect.bisect_left(keys, key)
                    if lb < len(keys) and keys[lb][1] == v:
                        continue
                    surv[v] = key
            for p in picks:
                u = keys[p][1]
                e = float(self.exact(q, u, int_query))
                pos = sum(1 for d, _ in top if d <= e)
                if pos < k:
                    top.insert(pos, (e, u))
                    del top[k:]
                expanded[p] = True
            merged = sorted([(keys[i], expanded[i]) for i in range(len(keys))] + [(s, False) for s in surv.values()])
            merged = merged[:L]
            keys = [m[0] for m in merged]
            expanded = [m[1] for m in merged]
        return top
