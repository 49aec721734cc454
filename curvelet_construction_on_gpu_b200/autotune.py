"""Per-bucket tuning tables: search them on sample batches, keep them as JSON.

An engine keeps one tuning per size bucket of a batch (its total edges,
cvl_tuning_bucket). Every tuning gives the same curvelets bit for bit; they
differ in time only. ``tune`` runs the engine's autotuner once per bucket on a
sample batch and returns the table; ``save``/``load`` keep it for later
processes on the same kind of GPU.
"""
from __future__ import annotations

import json

from . import _abi
from .api import CurveletParams, Engine

BUCKET_NAMES = ["<=64Ki", "<=512Ki", "<=4Mi", ">4Mi"]


def bucket_of(num_edges: int) -> int:
    return int(_abi.load().cvl_tuning_bucket(int(num_edges)))


def tune(engine: Engine, samples: dict, params: CurveletParams | None = None, passes: int = 1) -> dict:
    """samples: {bucket: list of maps}. Returns {bucket: {"tuning": …, "device_ms": …}}."""
    table = {}
    for bucket, maps in samples.items():
        n = sum(m.shape[0] for m in maps)
        if bucket_of(n) != int(bucket):
            raise ValueError(f"sample of {n} edges falls in bucket {bucket_of(n)}, not {bucket}")
        batch = engine.upload_batch(maps)
        try:
            t, ms = engine.autotune(batch, params, passes)
        finally:
            batch.close()
        table[int(bucket)] = {"tuning": t, "device_ms": ms, "edges": n}
    return table


def save(path: str, table: dict, device_name: str = "") -> None:
    with open(path, "w") as fh:
        json.dump({"device": device_name, "buckets": {str(k): v for k, v in table.items()}}, fh, indent=1)


def load(path: str, engine: Engine) -> dict:
    """Installs a saved table on the engine; returns it."""
    with open(path) as fh:
        data = json.load(fh)
    table = {int(k): v for k, v in data["buckets"].items()}
    for bucket, entry in table.items():
        engine.set_tuning(bucket, **entry["tuning"])
    return table
