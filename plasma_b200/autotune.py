"""Measured autotuning of the library's tile-shape tables.

The reference picks its tile size nb from a Lua script (control/tuning.c,
tuning/default.lua); here the choice is measured on the GPU in use by the
library itself (plasma_autotune_potrf / plasma_autotune_batched,
include/plasma_b200.h).  This module runs them over a set of sizes and keeps
the resulting tables as JSON, so that a service can tune once and load the
tables at start-up.
"""
import ctypes
import json

from . import PlasmaRealDouble, PlasmaRealFloat, lib

PRECISIONS = {"f64": PlasmaRealDouble, "f32": PlasmaRealFloat}
POTRF_SIZES = (512, 1024, 2048, 4096, 8192, 16384, 32768)
BATCHED_ORDERS = (32, 64, 128, 256, 512)


def tune(potrf_sizes=POTRF_SIZES, batched_count=1024, precisions=("f64", "f32")):
    """Tunes the tables of the initialised library; returns them."""
    L = lib()
    out = {"potrf_nb": {}, "potrf_ms": {}, "batched_nb": {}}
    for p in precisions:
        d = PRECISIONS[p]
        out["potrf_nb"][p], out["potrf_ms"][p], out["batched_nb"][p] = {}, {}, {}
        for n in potrf_sizes:
            ms = ctypes.c_double()
            nb = L.plasma_autotune_potrf(d, n, ctypes.byref(ms))
            if nb <= 0:
                raise RuntimeError(f"plasma_autotune_potrf({p}, {n}) failed: {nb}")
            out["potrf_nb"][p][str(n)] = nb
            out["potrf_ms"][p][str(n)] = ms.value
        if batched_count:
            rc = L.plasma_autotune_batched(d, batched_count)
            if rc != 0:
                raise RuntimeError(f"plasma_autotune_batched({p}) failed: {rc}")
        for n in BATCHED_ORDERS:
            out["batched_nb"][p][str(n)] = L.plasma_tuning_get_batched_nb(d, n)
    return out


def save(tables, path):
    with open(path, "w") as f:
        json.dump(tables, f, indent=1)


def load(path):
    """Installs tables written by save() into the library."""
    L = lib()
    with open(path) as f:
        t = json.load(f)
    for p, table in t.get("potrf_nb", {}).items():
        for n, nb in table.items():
            L.plasma_tuning_set_potrf_nb(PRECISIONS[p], int(n), int(nb))
    for p, table in t.get("batched_nb", {}).items():
        for n, nb in table.items():
            L.plasma_tuning_set_batched_nb(PRECISIONS[p], int(n), int(nb))
    return t
