"""Tile autotuner: per disk shape and precision, the azimuthal sweep's cells
per thread and the column sweeps' segment length that run fastest.

The reference's GPU build picks one block shape per kernel by timing a sweep
of shapes (scripts/blocks_function.py); here the choice is per disk shape,
because a batch mixes shapes: a disk's tiles depend only on its own shape,
never on the other members, so its arithmetic is the same alone and in any
mix.  Each knob is timed in a batch of copies of the shape large enough to
fill the GPU (one eager step per candidate, CUDA events per launch group,
best of `reps`), the two knobs one after the other (the azimuthal sweep and
the column sweeps are separate launches).

Table: JSON {"<Nx>x<Ny>x<Nz>:<precision>": {"sweep_x_cells": C,
"col_segment": NS, "ms": {...}}}.  `TileTable.default()` reads the table
shipped with the package (tiles_b200.json, tuned on a B200) and then a
machine-local one ($FB_TILES, or _lib/tiles.json) whose entries win.

    python -m fargo3d_b200.autotune [--workload batched|serving|all] [--out PATH]
"""
from __future__ import annotations

import argparse
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SHIPPED = os.path.join(HERE, "tiles_b200.json")
LOCAL = os.environ.get("FB_TILES", os.path.join(HERE, "_lib", "tiles.json"))

CX_CANDIDATES = (1, 2, 4, 8, 16)
NS_CANDIDATES = (4, 8, 16)


def shape_key(cfg, precision: str) -> str:
    return "%dx%dx%d:%s" % (cfg.nx, cfg.ny, cfg.nz if cfg.is3d else 1, precision)


SMEM_MAX = 227 * 1024


def cx_candidates(nx: int, precision: str = "fp32", is3d: bool = False):
    """Widths that tile a ring in 256 threads and whose whole rings per CTA
    (two buffers of 1 + nq fields and the velocity ring, each row padded by
    16 bytes) fit in shared memory."""
    esz, nq = (8 if precision == "fp64" else 4), (6 if is3d else 4)
    out = []
    for c in CX_CANDIDATES:
        if nx % c or nx // c > 256:
            continue
        nxp = nx + 16 // esz                                 # padded ring row in shared memory
        if (256 // (nx // c)) * nxp * (2 * (1 + nq) + 1) * esz <= SMEM_MAX:
            out.append(c)
    return out


_DEFAULT = [None, None]   # (file modification times, table) of TileTable.default()


class TileTable:
    def __init__(self, entries=None):
        self.entries = dict(entries or {})

    @classmethod
    def load(cls, *paths):
        t = cls()
        for p in paths:
            if p and os.path.exists(p):
                with open(p) as fh:
                    t.entries.update(json.load(fh))
        return t

    @classmethod
    def default(cls):
        """The shipped table under the machine-local one, read again only
        when either file changes."""
        key = tuple(os.stat(p).st_mtime_ns if os.path.exists(p) else None for p in (SHIPPED, LOCAL))
        if _DEFAULT[0] != key:
            _DEFAULT[:] = [key, cls.load(SHIPPED, LOCAL)]
        return cls(_DEFAULT[1].entries)

    def get(self, cfg, precision: str):
        e = self.entries.get(shape_key(cfg, precision))
        return (e["sweep_x_cells"], e["col_segment"]) if e else None

    def apply(self, batch):
        """Set every member's tiles whose shape the table lists."""
        for i, c in enumerate(batch.cfgs):
            t = self.get(c, batch.precision)
            if t and t[0] in cx_candidates(c.nx, batch.precision, c.is3d):
                batch.set_tiles(i, t[0], t[1])

    def save(self, path: str):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        with open(path, "w") as fh:
            json.dump(self.entries, fh, indent=1, sort_keys=True)


def tune_shape(cfg, precision: str, device: int = 0, min_cells: float = 4e6, reps: int = 3, max_copies: int = 64):
    """Time every candidate of both knobs for one shape; returns the table
    entry.  The copies differ only in their noise seed."""
    from .batch import Batch
    copies = int(min(max_copies, max(1, math.ceil(min_cells / cfg.active_cells))))
    cfgs = [cfg.replace(seed=cfg.seed + k) for k in range(copies)]
    b = Batch(cfgs, precision, device=device, tiles=None)
    b.load_initial_states()
    b.run(3)

    def best(group):
        t = min(b.profile_step()[group] for _ in range(reps))
        return t

    ms_x = {}
    for c in cx_candidates(cfg.nx, precision, cfg.is3d):
        for i in range(copies):
            b.set_tiles(i, c, 8)
        b.profile_step()   # rebuild + warm
        ms_x[c] = best("sweep_x")
    cx = min(ms_x, key=ms_x.get)
    ms_c = {}
    for ns in NS_CANDIDATES:
        for i in range(copies):
            b.set_tiles(i, cx, ns)
        b.profile_step()
        ms_c[ns] = best("sweep_cols")
    ns = min(ms_c, key=ms_c.get)
    b.close()
    return {"sweep_x_cells": cx, "col_segment": ns, "copies": copies,
            "ms": {"sweep_x": {str(k): v for k, v in ms_x.items()}, "sweep_cols": {str(k): v for k, v in ms_c.items()}}}


def shapes_of(name: str):
    from .setups import config_batched, config_fargo2d, config_p3disof
    from .serving import SERVING_SIZES
    out = []
    if name in ("batched", "all"):
        seen = set()
        for c in config_batched(64, 0):
            k = (c.nx, c.ny)
            if k not in seen:
                seen.add(k)
                out.append((c, "fp32"))
    if name in ("serving", "all"):
        from .setups import DiskConfig
        for nx, ny in SERVING_SIZES:
            out.append((DiskConfig(nx=nx, ny=ny, alpha_visc=True, alpha=1e-3, nu=0.0), "fp32"))
    if name == "all":
        out.append((config_fargo2d(384, 128), "fp64"))
        out.append((config_p3disof(512, 256, 48), "fp64"))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="all", choices=["batched", "serving", "all"])
    ap.add_argument("--out", default=LOCAL)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    table = TileTable.load(args.out)
    for cfg, prec in shapes_of(args.workload):
        key = shape_key(cfg, prec)
        if key in table.entries:
            continue
        table.entries[key] = tune_shape(cfg, prec, device=args.device)
        e = table.entries[key]
        print(key, "->", e["sweep_x_cells"], e["col_segment"], json.dumps(e["ms"]), flush=True)
        table.save(args.out)
    table.save(args.out)


if __name__ == "__main__":
    main()
