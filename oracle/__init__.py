"""CPU oracle of the MCML walk -- TEST INFRASTRUCTURE ONLY.

Binds ``oracle/_build/liboracle.so`` (built from ``mcml_oracle.cpp`` by
``make -C oracle``).  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module, as the checker; the
library never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from .config import ConfigError, Derived, Sim, read_config  # noqa: F401

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_BIN = HERE / "_ref" / "MCML_GPU"
REF_SHIM = HERE / "_ref" / "libtimeshim.so"

MAX_SDS = 30


class Stats(C.Structure):
    _fields_ = [
        ("photons", C.c_uint64),
        ("steps", C.c_uint64),
        ("detected", C.c_uint64 * MAX_SDS),
        ("wsum", C.c_double * MAX_SDS),
        ("wsq", C.c_double * MAX_SDS),
    ]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    vp = C.c_void_p
    lib.oracle_derive.argtypes = [vp, vp]
    lib.oracle_walk_stream.argtypes = [vp, C.c_int, vp, C.c_uint64, vp, vp, vp, vp]
    lib.oracle_walk_stream.restype = C.c_int
    lib.oracle_replay_stream.argtypes = [vp, C.c_int, C.c_int, vp, C.c_uint64, vp, vp, vp, vp,
                                         vp, vp]
    lib.oracle_replay_stream.restype = C.c_int
    lib.oracle_run.argtypes = [vp, C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int,
                               C.POINTER(Stats), vp, vp, vp, C.c_uint64, vp]
    lib.oracle_run.restype = C.c_int
    lib.oracle_replay.argtypes = [vp, C.c_int, C.c_uint64, C.c_uint64, vp, vp, C.c_int, vp, vp,
                                  vp, vp, C.c_uint32, C.c_uint32, C.c_float, C.c_float]
    lib.oracle_replay.restype = C.c_int
    lib.oracle_energy.argtypes = [vp, C.c_int, C.c_uint64, C.c_uint64, C.c_int, vp]
    lib.oracle_energy.restype = C.c_int
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def derive(sim) -> Derived:
    d = Derived()
    load().oracle_derive(C.byref(sim), C.byref(d))
    return d


def walk_stream(sim, u: np.ndarray, fp64: bool = False):
    """First pass of one photon on recorded uniforms.
    Returns (steps, [(sds, weight)], draws_used); steps = -1 if u ran out."""
    u = np.ascontiguousarray(u, dtype=np.float32)
    n_det = C.c_int(0)
    sds = np.zeros(MAX_SDS, dtype=np.int32)
    w = np.zeros(MAX_SDS, dtype=np.float64)
    used = C.c_uint64(0)
    steps = load().oracle_walk_stream(C.byref(sim), int(fp64), _p(u), u.size, C.byref(n_det),
                                      _p(sds), _p(w), C.byref(used))
    return steps, [(int(sds[i]), float(w[i])) for i in range(n_det.value)], int(used.value)


def replay_stream(sim, sds: int, u: np.ndarray, fp64: bool = False, grid=None):
    """Replay of one photon for 1-based sds on recorded uniforms.
    Returns (row[L+2] float64, interactions[L], A_rz or None, A0_z or None,
    used, w_exit) or None if the draws ran out; w_exit is the photon's weight
    as it leaves through the detector (before a ring detector weighs it)."""
    u = np.ascontiguousarray(u, dtype=np.float32)
    L = sim.num_layers
    row = np.zeros(L + 2, dtype=np.float64)
    inter = np.zeros(L, dtype=np.uint32)
    arz = a0z = None
    if grid is not None:
        nr, nz = grid
        arz = np.zeros((nz, nr), dtype=np.uint64)
        a0z = np.zeros(nz, dtype=np.uint64)
    used = C.c_uint64(0)
    w_exit = C.c_double(0.0)
    rc = load().oracle_replay_stream(C.byref(sim), int(fp64), sds, _p(u), u.size, _p(row),
                                     _p(inter), _p(arz), _p(a0z), C.byref(used), C.byref(w_exit))
    if rc != 0:
        return None
    return row, inter, arz, a0z, int(used.value), float(w_exit.value)


def run(sim, n: int, seed: int, *, first: int = 0, fp64: bool = False, threads: int = 0,
        det_cap: int = 1 << 20):
    """Statistical first pass with PCG32 per photon.  Returns (Stats,
    photon_ids, sds, weights) of the detections."""
    st = Stats()
    ids = np.zeros(det_cap, dtype=np.uint64)
    sds = np.zeros(det_cap, dtype=np.int32)
    w = np.zeros(det_cap, dtype=np.float64)
    nout = C.c_uint64(0)
    rc = load().oracle_run(C.byref(sim), int(fp64), seed, first, n, threads, C.byref(st),
                           _p(ids), _p(sds), _p(w), det_cap, C.byref(nout))
    if rc != 0:
        raise RuntimeError("oracle_run failed")
    k = min(int(nout.value), det_cap)
    return st, ids[:k], sds[:k], w[:k]


def replay(sim, seed: int, ids: np.ndarray, sds: np.ndarray, *, fp64: bool = False,
           threads: int = 0, grid=(1000, 500, 0.01, 0.01), tallies: bool = True):
    """Statistical replay of oracle detections.  Returns (rows, inter,
    A_rz (S,nz,nr) or None, A0_z (S,nz) or None)."""
    L = sim.num_layers
    S = sim.num_sds
    n = ids.size
    ids = np.ascontiguousarray(ids, dtype=np.uint64)
    sds = np.ascontiguousarray(sds, dtype=np.int32)
    rows = np.zeros((n, L + 2), dtype=np.float64)
    inter = np.zeros((n, L), dtype=np.uint32)
    nr, nz, dr, dz = grid
    arz = np.zeros((S, nz, nr), dtype=np.uint64) if tallies else None
    a0z = np.zeros((S, nz), dtype=np.uint64) if tallies else None
    rc = load().oracle_replay(C.byref(sim), int(fp64), seed, n, _p(ids), _p(sds), threads,
                              _p(rows), _p(inter), _p(arz), _p(a0z), nr, nz, dr, dz)
    if rc != 0:
        raise RuntimeError("oracle_replay failed")
    return rows, inter, arz, a0z


ENERGY_FIELDS = ("start", "absorbed", "top", "bottom", "capped", "roulette_lost",
                 "roulette_gained", "rounding")


def energy(sim, n: int, seed: int, *, fp64: bool = False, roulette: bool = True) -> dict:
    """Where the start weight of n photons went (weight quanta): see
    oracle_energy in mcml_oracle.cpp."""
    lib = load()
    out = np.zeros(8, np.float64)
    if lib.oracle_energy(C.byref(sim), int(fp64), seed, n, int(roulette), _p(out)) != 0:
        raise RuntimeError("oracle_energy failed")
    return dict(zip(ENERGY_FIELDS, out.tolist()))
