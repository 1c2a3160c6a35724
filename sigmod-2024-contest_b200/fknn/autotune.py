"""Autotuner for the search plans and kernels (fknn_index_set_tuning) and
the candidate width k' of the reduced-precision forms.

For one index and a sample of its query stream it measures each setting
with the index resident and the sample in device memory, keeps the
fastest setting whose recall@100 against the exact path (same sample) is at
least the target, and records it in a JSON table keyed by device name, base
size and mode.  Index.apply_tuning() looks the table up and sets the index.

The search is coordinate descent: k' first (smallest meeting the recall
target at the current tuning), then each tuning field over its candidate
values, twice around.  Every setting is timed as the median of a few
searches after one warm-up.
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, Optional

import numpy as np

from . import _lib
from .datagen import recall_matrix

DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_table.json")

SPACE = {
    "items_per_sm": [2, 3, 4, 6, 8],
    "pilot_stride": [0, 8, 16, 32, 64],
    "list_slack": [256, 384, 512],
    "min_chunk_blocks": [4, 8, 16],
    "bound_refresh": [0, 2, 8, 32],
}
EXACT_SPACE = {"items_per_sm": [8, 12, 16, 24], "min_chunk_blocks": [8, 16, 32], "pilot_stride": [0, 8, 16, 32]}
KPRIMES = [100, 112, 128, 160, 200, 256, 320, 400, 512, 640, 800, 1024]


def device_name(device: int = 0) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:  # noqa: BLE001
        return "cuda"


def table_key(device: str, n: int, mode: int) -> str:
    """Base sizes bucket by powers of ten (1e5 .. 1e7 share nothing)."""
    return f"{device}|n=1e{int(round(np.log10(max(n, 1))))}|mode={mode}"


def _timed(index, q, m, mode, kprime, reps, graph=False):
    ids = dd = None
    times = []
    for r in range(reps + 1):
        t0 = time.perf_counter()
        ids, dd = index.search(q, m, k=100, mode=mode, kprime=kprime, ids=ids, dists=dd, graph=graph)
        if hasattr(ids, "is_cuda"):
            import torch
            torch.cuda.synchronize()
        if r:
            times.append(time.perf_counter() - t0)
    out = ids.cpu().numpy() if hasattr(ids, "cpu") else ids
    return float(np.median(times)), out.view(np.uint32)


def autotune(index, qvecs, metas, mode: int, recall_target: float = 0.99, reps: int = 3,
             kprimes=None, log=None, graph: bool = True) -> Dict:
    """Tunes `index` for `mode` on the query sample (qvecs, metas: host or
    torch CUDA arrays).  Leaves the index set to the best setting and
    returns it: {"tuning": {...}, "kprime": k', "ms": ..., "recall": ...}.
    graph: time the reduced-precision modes in their captured form (the
    plan built on the device), as the bench and serving use them."""
    graph = graph and mode != _lib.MODE_EXACT_FP32
    exact_ms, gt = _timed(index, qvecs, metas, _lib.MODE_EXACT_FP32, 0, reps)
    space = EXACT_SPACE if mode == _lib.MODE_EXACT_FP32 else SPACE
    cur = index.get_tuning(mode)
    best = {"tuning": dict(cur), "kprime": 0, "ms": float("inf"), "recall": 0.0}

    def run(tuning, kprime):
        index.set_tuning(mode, tuning["list_slack"], tuning["items_per_sm"], tuning["min_chunk_blocks"],
                         tuning["bound_refresh"], tuning["pilot_stride"])
        ms, ids = _timed(index, qvecs, metas, mode, kprime, reps, graph)
        rec = 1.0 if mode == _lib.MODE_EXACT_FP32 else recall_matrix(ids, gt)
        if log:
            log(json.dumps({"tuning": tuning, "kprime": kprime, "ms": ms * 1e3, "recall": rec}))
        return ms, rec

    kp = 0
    if mode != _lib.MODE_EXACT_FP32:
        for k in (kprimes or KPRIMES):
            ms, rec = run(cur, k)
            if rec >= recall_target:
                kp = k
                best = {"tuning": dict(cur), "kprime": k, "ms": ms, "recall": rec}
                break
        if not kp:
            raise RuntimeError(f"no k' in {kprimes or KPRIMES} reaches recall {recall_target}")
    else:
        ms, _ = run(cur, 0)
        best = {"tuning": dict(cur), "kprime": 0, "ms": ms, "recall": 1.0}
    for _round in range(2):
        for field, values in space.items():
            for v in values:
                if v == best["tuning"][field]:
                    continue
                t = dict(best["tuning"])
                t[field] = v
                ms, rec = run(t, kp)
                if rec >= recall_target and ms < best["ms"]:
                    best = {"tuning": t, "kprime": kp, "ms": ms, "recall": rec}
    t = best["tuning"]
    index.set_tuning(mode, t["list_slack"], t["items_per_sm"], t["min_chunk_blocks"], t["bound_refresh"],
                     t["pilot_stride"])
    best["ms"] *= 1e3
    best["exact_ms"] = exact_ms * 1e3
    best["plan"] = "device, captured graph" if graph else "host"
    return best


def load_table(path: Optional[str] = None) -> Dict:
    path = path or DEFAULT_TABLE
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def save_entry(key: str, entry: Dict, path: Optional[str] = None) -> None:
    path = path or DEFAULT_TABLE
    table = load_table(path)
    table[key] = entry
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def lookup(n: int, mode: int, device: int = 0, path: Optional[str] = None) -> Optional[Dict]:
    return load_table(path).get(table_key(device_name(device), n, mode))


def main(argv=None) -> None:
    """python -m fknn.autotune --config 2 [--n N] [--sample Q] [--modes 1,0]:
    tunes an index of that synthetic workload on a query sample drawn with
    another seed than the workload's own queries and records the result."""
    import argparse

    import torch

    from . import api, datagen
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--sample", type=int, default=100000)
    ap.add_argument("--modes", default="1,0")
    ap.add_argument("--recall", type=float, default=0.99)
    ap.add_argument("--table", default=None)
    a = ap.parse_args(argv)
    w = datagen.WORKLOADS[a.config]
    n = a.n or w.n
    vecs, labels, ts = datagen.make_base(n, w.zipf_s, w.n_labels, 1234 + a.config)
    q, m = datagen.make_queries(a.sample, w.zipf_s, w.n_labels, w.window, w.balanced_types, 1234 + a.config,
                                 7777 + a.config)
    modes = [int(x) for x in a.modes.split(",")]
    idx = api.Index(vecs, labels, ts, build_bf16=_lib.MODE_BF16_RERANK in modes,
                    build_fp8=_lib.MODE_FP8_RERANK in modes)
    dq, dm = torch.from_numpy(q).cuda(), torch.from_numpy(m).cuda()
    for mode in modes:
        best = autotune(idx, dq, dm, mode, recall_target=a.recall, log=print)
        best.update({"workload": w.name, "n": n, "sample": a.sample})
        key = table_key(device_name(), n, mode)
        save_entry(key, best, a.table)
        print(json.dumps({"key": key, **best}), flush=True)
    idx.close()


if __name__ == "__main__":
    main()
