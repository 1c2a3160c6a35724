"""Generates the golden fixtures in tests/golden/ by running the reference's
own code, compiled from its sources by oracle/Makefile (target `ref`).

Run in a container that has the reference sources (REF_ROOT, default
/root/reference):

    make -C oracle all ref && python tests/golden/make_golden.py

Fixtures (all small):
  exact_c1.npz     reference utils.h:80 Bruteforce top-100 ids for seeded
                   synthetic data with the config-1 distributions
                   (N=20000, queries with >= 100 passing rows)
  exact_c4.npz     the same with the config-4 distributions (Zipf 1.5 over
                   10,000 labels, log-uniform windows)
  exact_ties.npz   rows repeated three times (exact distance ties), type 0
  dummy_gt.npz     reference ids on the reference's shipped dummy-data.bin /
                   dummy-queries.bin, with the files' SHA-256
  sq8.npz          reference SQ8SymmetricQuantizer alpha + codes digest and
                   bruteforce / bruteforce_subgraph outputs (heap order)
  sq8_kat.json     the known answer of test_simd_distance.cpp:196-203: the
                   two fixed int8 vectors parsed from that file and the
                   reference L2SqrSQ8_sym value
  graph_hnsw.npz   a graph built by the reference HNSW::Build (Graph::save
                   bytes, N=2000, R=24, points in timestamp order) and the
                   reference Searcher's ids (and dists) for all six search
                   forms over seeded queries, time windows and id ranges
Each npz also stores the SHA-256 of the generated inputs so a generator
change is detected instead of silently compared.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "sigmod-2024-contest_b200"))
sys.path.insert(0, os.path.dirname(HERE))
import oracle  # noqa: E402
from fknn import datagen  # noqa: E402
from graph_util import GRAPH_CASES, graph_inputs  # noqa: E402

REF_ROOT = os.environ.get("REF_ROOT", "/root/reference")


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def ref_gt(vecs, labels, ts, q, metas):
    R = oracle.ref_exact()
    rows = datagen.to_rows(vecs, labels, ts)
    qrows = datagen.to_query_rows(q, metas)
    gt = np.empty((q.shape[0], 100), dtype=np.uint32)
    rc = R.ref_exact_bruteforce(rows.ctypes.data, rows.shape[0], qrows.ctypes.data, qrows.shape[0], gt.ctypes.data,
                                None)
    assert rc == 0, "reference Bruteforce threw"
    return gt


def exact_case(name, cfg, n, nq):
    vecs, labels, ts, q, metas = datagen.make_workload(cfg, n=n, nq=nq)
    cnt = oracle.count_matches(labels, ts, metas)
    sel = np.nonzero(cnt >= 100)[0].astype(np.int64)
    gt = ref_gt(vecs, labels, ts, q[sel], metas[sel])
    np.savez_compressed(os.path.join(HERE, name), cfg=cfg, n=n, nq=nq, sel=sel, gt=gt, counts=cnt,
                        sha_inputs=digest(vecs, labels, ts, q, metas))
    print(name, "queries pinned:", len(sel), "of", nq)


def ties_case():
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=400, nq=30)
    v3 = np.repeat(vecs[:400], 3, axis=0)
    l3 = np.repeat(labels, 3)
    t3 = np.repeat(ts, 3)
    q3 = np.concatenate([vecs[:20], q[:10]])
    m3 = np.zeros((30, 4), dtype=np.float32)
    gt = ref_gt(v3, l3, t3, q3, m3)
    np.savez_compressed(os.path.join(HERE, "exact_ties.npz"), gt=gt, sha_inputs=digest(v3, l3, t3, q3, m3))
    print("exact_ties.npz")


def dummy_case():
    dpath = os.path.join(REF_ROOT, "dummy-data.bin")
    qpath = os.path.join(REF_ROOT, "dummy-queries.bin")
    vecs, labels, ts = datagen.read_base(dpath)
    q, metas = datagen.read_queries(qpath)
    gt = ref_gt(vecs, labels, ts, q, metas)
    sha = lambda p: hashlib.sha256(open(p, "rb").read()).hexdigest()  # noqa: E731
    np.savez_compressed(os.path.join(HERE, "dummy_gt.npz"), gt=gt, sha_data=sha(dpath), sha_queries=sha(qpath))
    print("dummy_gt.npz", gt.shape)


def sq8_case():
    R = oracle.ref_sq8()
    vecs, labels, ts, q, metas = datagen.make_workload(1, n=6000, nq=12)
    a = ctypes.c_float()
    codes = np.empty((vecs.shape[0], 112), dtype=np.int8)
    R.ref_sq8_sym_train(vecs.ctypes.data, vecs.shape[0], ctypes.byref(a), codes.ctypes.data)
    alpha = a.value
    qcodes = np.zeros((q.shape[0], 112), dtype=np.int8)
    for i in range(q.shape[0]):
        row = np.ascontiguousarray(q[i])
        R.ref_sq8_sym_encode(row.ctypes.data, ctypes.c_float(alpha), qcodes[i].ctypes.data)
    # slabs: full, a middle slab, k == npoints, and a slab with many ties
    # (every code repeated) where the heap order depends on replacement ties
    tie_codes = np.ascontiguousarray(np.repeat(codes[:700], 4, axis=0))
    cases = [(140, 0, 6000, "codes"), (140, 1234, 2500, "codes"), (100, 500, 100, "codes"), (140, 0, 2800, "ties"),
             (1, 10, 777, "codes")]
    out_ids, out_d = [], []
    for (k, s, npnt, src) in cases:
        slab = np.ascontiguousarray((codes if src == "codes" else tie_codes)[s:s + npnt])
        ids_q, d_q = [], []
        for i in range(q.shape[0]):
            ids = np.empty(k, dtype=np.int32)
            d = np.empty(k, dtype=np.float32)
            R.ref_sq8_bruteforce_subgraph(k, ids.ctypes.data, d.ctypes.data, npnt, slab.ctypes.data,
                                          ctypes.c_float(alpha), qcodes[i].ctypes.data)
            ids2 = np.empty(k, dtype=np.int32)
            R.ref_sq8_bruteforce(k, ids2.ctypes.data, npnt, slab.ctypes.data, ctypes.c_float(alpha),
                                 qcodes[i].ctypes.data)
            assert np.array_equal(ids, ids2)
            ids_q.append(ids)
            d_q.append(d)
        out_ids.append(np.stack(ids_q))
        out_d.append(np.stack(d_q))
    np.savez_compressed(os.path.join(HERE, "sq8.npz"), alpha=np.float32(alpha), codes_sha=digest(codes),
                        qcodes=qcodes, cases=np.array([(c[0], c[1], c[2], 0 if c[3] == "codes" else 1) for c in cases]),
                        **{f"ids{j}": out_ids[j] for j in range(len(cases))},
                        **{f"dists{j}": out_d[j] for j in range(len(cases))},
                        sha_inputs=digest(vecs, q))
    print("sq8.npz alpha", alpha)


def sq8_kat():
    src = open(os.path.join(REF_ROOT, "test_simd_distance.cpp")).read()
    arrs = {}
    for name in ("a0", "a1"):
        m = re.search(r"int8_t\s+%s\[32\]\s*=\s*\{([^}]*)\}" % name, src)
        arrs[name] = [int(x) for x in m.group(1).split(",")]
    x = np.zeros(112, dtype=np.int8)
    y = np.zeros(112, dtype=np.int8)
    x[:32] = arrs["a0"]
    y[:32] = arrs["a1"]
    val = oracle.ref_sq8().ref_l2sqr_sq8_sym(x.ctypes.data, y.ctypes.data)
    with open(os.path.join(HERE, "sq8_kat.json"), "w") as f:
        json.dump({"source": "test_simd_distance.cpp:196-203", "a0": arrs["a0"], "a1": arrs["a1"],
                   "l2sqr_sq8_sym": int(val)}, f, indent=1)
    print("sq8_kat.json", val)


def graph_case():
    vecs, labels, ts, q, bounds, ib = graph_inputs()
    path = "/tmp/fknn_golden_graph.bin"
    gb = oracle.ref_hnsw_graph(vecs, ts, 24, 100, path)
    out = {}
    for j, (mode, k, refine) in enumerate(GRAPH_CASES):
        wd = mode in (2, 4)
        r = oracle.ref_graph_search(path, vecs, labels, ts, q, mode, k, refine, bounds, ib, with_dists=wd)
        out[f"ids{j}"] = r[0] if wd else r
        if wd:
            out[f"dists{j}"] = r[1]
    np.savez_compressed(os.path.join(HERE, "graph_hnsw.npz"), graph=np.frombuffer(gb, dtype=np.uint8),
                        cases=np.array(GRAPH_CASES, dtype=np.int32), bounds=bounds, id_bounds=ib,
                        sha_inputs=digest(vecs, labels, ts, q), **out)
    print("graph_hnsw.npz", len(gb), "graph bytes")


CASES = {"exact": lambda: (exact_case("exact_c1.npz", 1, 20000, 300), exact_case("exact_c4.npz", 4, 20000, 200)),
         "ties": ties_case, "dummy": dummy_case, "sq8": sq8_case, "kat": sq8_kat, "graph": graph_case}

if __name__ == "__main__":
    oracle.build(ref=True)
    for name in (sys.argv[1:] or list(CASES)):
        CASES[name]()
