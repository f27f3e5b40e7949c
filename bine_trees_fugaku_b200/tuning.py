"""Persistent autotuner table for batched launches.

Entries map a batch signature (item count, rank-count and size buckets,
device name) to the bine_batch_tuning_t the autotuner found fastest.  The
file is JSON with a SHA-256 checksum of its payload; a missing, corrupt or
mismatching file is ignored (the autotuner runs again), so a crash while
writing never poisons later runs (writes go to a temporary file that is
renamed into place).
"""
import hashlib
import json
import os

VERSION = 1


def _digest(payload):
    return hashlib.sha256(json.dumps(payload, sort_keys=True).encode()).hexdigest()


def load(path):
    try:
        with open(path) as f:
            doc = json.load(f)
    except (OSError, ValueError):
        return {}
    if doc.get("version") != VERSION or doc.get("sha256") != _digest(doc.get("entries", {})):
        return {}
    return doc["entries"]


def save(path, entries):
    doc = {"version": VERSION, "entries": entries, "sha256": _digest(entries)}
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(doc, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def signature(items, device_name):
    """Bucketed description of a batch: tunings transfer between batches
    with the same mix of rank counts and sizes."""
    import math

    n = len(items)
    ps = sorted(it[5] for it in items)
    sizes = sorted(it[3] for it in items)
    med = lambda v: v[len(v) // 2] if v else 0
    return (f"{device_name}|n{2 ** max(0, int(math.log2(max(1, n))))}|P{2 ** int(math.log2(max(1, med(ps))))}"
            f"|c{2 ** int(math.log2(max(1, med(sizes))))}")
