"""Small autotuner for the stage-kernel tile shape and radial chunk.

The fused stage kernel runs one CTA per (tile of TX x TY columns, chunk of kchunk radial
planes, face, run).  The best shape depends on the grid, the precision, the number of
fields and the batch size, so this module times every valid candidate for a given
workload on the current device (CUDA events on the solver's stream, a few full RK4 steps
each) and keeps the fastest.  Results are cached in a JSON file keyed by
(nx, nr, precision, nfields, nruns, device name); ``tuned_b200.json`` beside this module
holds the table measured on a B200 and is consulted first.

Usage: ``python -m solar_b200.autotune c2 --precision fp32 --nfields 4``.
"""
from __future__ import annotations

import argparse
import json
import os
from typing import Dict, List, Optional, Sequence, Tuple

from . import configs

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuned_b200.json")
CACHE = os.environ.get("SOLAR_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "solar_b200", "tuned.json"))

TILES = [(32, 16), (32, 8), (64, 8), (16, 16)]
CHUNK_DIVISORS = [0, 2, 3, 4, 5, 6, 8, 12]   # 0 = library default; else nr / d planes per CTA


def key(nx: int, nr: int, precision: str, nfields: int, nruns: int, device_name: str) -> str:
    return f"{device_name}|{nx}x{nr}|{precision}|f{nfields}|r{nruns}"


def device_name(device: int = 0) -> str:
    from . import _lib
    return _lib.device_name(device)


def candidates(nx: int, nr: int) -> List[Tuple[int, int, int]]:
    out = []
    for tx, ty in TILES:
        if nx % tx or nx % ty:
            continue
        for d in CHUNK_DIVISORS:
            kc = 0 if d == 0 else max(8, -(-nr // d))
            if (tx, ty, kc) not in out:
                out.append((tx, ty, kc))
    return out


def _load(path: str) -> Dict[str, dict]:
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def lookup(nx: int, nr: int, precision: str, nfields: int, nruns: int = 1, device: int = 0) -> Optional[Tuple[int, int, int]]:
    k = key(nx, nr, precision, nfields, nruns, device_name(device))
    for path in (CACHE, TABLE):
        hit = _load(path).get(k)
        if hit:
            return tuple(hit["tile"])
    return None


def tune(cfg: configs.Config, precision: str = "fp32", nfields: int = 4, nruns: int = 1,
         steps: int = 6, device: int = 0, save: bool = True,
         cands: Optional[Sequence[Tuple[int, int, int]]] = None) -> dict:
    """Time every candidate and return {"tile": best, "ms_per_step": ..., "all": {...}}."""
    from .solver import Solver
    results = {}
    for cand in (cands or candidates(cfg.nx, cfg.nr)):
        with Solver(cfg, precision=precision, nfields=nfields, nruns=nruns, device=device, tile=cand) as s:
            for r in range(nruns):
                s.init_sources(run=r)
            s.rk4(2)
            ms = min(s.time_rk4(steps)["total_ms"] for _ in range(2)) / steps
        results["%dx%d/k%d" % cand] = ms
    best_name = min(results, key=results.get)
    tx, ty = map(int, best_name.split("/")[0].split("x"))
    kc = int(best_name.split("/k")[1])
    out = {"tile": [tx, ty, kc], "ms_per_step": results[best_name], "all": results}
    if save:
        db = _load(CACHE)
        db[key(cfg.nx, cfg.nr, precision, nfields, nruns, device_name(device))] = out
        os.makedirs(os.path.dirname(CACHE), exist_ok=True)
        with open(CACHE, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", default="c2", nargs="?")
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--nfields", type=int, default=4)
    ap.add_argument("--nruns", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--out", default=None, help="also write the result table here")
    args = ap.parse_args()
    cfg = configs.get(args.config)
    res = tune(cfg, args.precision, args.nfields, args.nruns, args.steps)
    line = {key(cfg.nx, cfg.nr, args.precision, args.nfields, args.nruns, device_name()): res}
    print(json.dumps(line))
    if args.out:
        db = _load(args.out)
        db.update(line)
        with open(args.out, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
