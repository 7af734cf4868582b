"""mcml_gpu_b200 -- B200-native MCML photon transport (Python host mirror).

The compute path is the CUDA library ``lib/libmcml_b200.so`` built from
``csrc/`` for sm_100a (``python -m mcml_gpu_b200.build``).  This module binds
its C ABI (``include/mcml_b200.h``) with ctypes and mirrors the reference's
host flow (MCML_GPU K3.02, transport.cu:57-272): parse the configuration,
run the first pass, replay the detected photons, write the output files.

There is no CPU fallback: every call that computes goes through the CUDA
library, and loading fails loudly when it has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

__all__ = [
    "MAX_LAYERS", "MAX_SDS", "MCMLError", "Sim", "Opts", "Result", "Derived",
    "DeviceInfo", "load_library", "lib_path", "parse_config", "derive", "make_sim",
    "Simulation", "Batch", "sample_sets", "shard", "uniform_stream", "device_count",
    "device_info", "checkpoint_info", "CheckpointInfo", "INCOMPLETE",
    "OUT_REPLAY", "OUT_ABSORBANCE", "OUT_PATHLENGTH", "OUT_AVERAGE_PL", "OUT_BINARY",
]

MAX_LAYERS = 10
MAX_SDS = 30
OUT_REPLAY, OUT_ABSORBANCE, OUT_PATHLENGTH, OUT_AVERAGE_PL, OUT_BINARY = 1, 2, 4, 8, 16

_PKG = Path(__file__).resolve().parent


def lib_path() -> Path:
    return _PKG / "lib" / "libmcml_b200.so"


class MCMLError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: status {status}: {message}")
        self.status = status
        self.message = message


class Sim(C.Structure):
    """mcml_sim: one simulation (sim_set.json fields + one input.txt line)."""
    _fields_ = [
        ("number_photons", C.c_uint64),
        ("num_layers", C.c_uint32),
        ("num_sds", C.c_uint32),
        ("upper_n", C.c_float),
        ("lower_n", C.c_float),
        ("detector_reflectance", C.c_float),
        ("source_probe_oblique", C.c_int32),
        ("detector_probe_oblique", C.c_int32),
        ("source_NA", C.c_float),
        ("source_radius", C.c_float),
        ("source_angle_deg", C.c_float),
        ("det_pos", C.c_float * MAX_SDS),
        ("det_NA", C.c_float * MAX_SDS),
        ("det_radius", C.c_float * MAX_SDS),
        ("det_angle_deg", C.c_float * MAX_SDS),
        ("height", C.c_float * MAX_LAYERS),
        ("mua", C.c_float * MAX_LAYERS),
        ("mus", C.c_float * MAX_LAYERS),
        ("n", C.c_float * MAX_LAYERS),
        ("g", C.c_float * MAX_LAYERS),
    ]


class Opts(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("slots", C.c_uint64),
        ("device", C.c_int32),
        ("grid_nr", C.c_uint32),
        ("grid_nz", C.c_uint32),
        ("grid_dr", C.c_float),
        ("grid_dz", C.c_float),
        ("record_capacity", C.c_uint64),
        ("stream", C.c_void_p),
        ("block_size", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("replay_step_budget", C.c_uint64),
        ("slot_begin", C.c_uint64),
    ]


class Result(C.Structure):
    _fields_ = [
        ("num_sds", C.c_uint32),
        ("photons", C.c_uint64),
        ("steps", C.c_uint64),
        ("detected", C.c_uint64 * MAX_SDS),
        ("weight_sum", C.c_double * MAX_SDS),
        ("weight_sumsq", C.c_double * MAX_SDS),
        ("reflectance", C.c_double * MAX_SDS),
        ("std_error", C.c_double * MAX_SDS),
        ("walk_ms", C.c_float),
        ("replay_ms", C.c_float),
        ("seed_ms", C.c_float),
        ("slots", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        s = self.num_sds
        return {
            "photons": int(self.photons),
            "steps": int(self.steps),
            "detected": [int(v) for v in self.detected[:s]],
            "weight_sum": list(self.weight_sum[:s]),
            "weight_sumsq": list(self.weight_sumsq[:s]),
            "reflectance": list(self.reflectance[:s]),
            "std_error": list(self.std_error[:s]),
            "walk_ms": float(self.walk_ms),
            "replay_ms": float(self.replay_ms),
            "seed_ms": float(self.seed_ms),
            "slots": int(self.slots),
        }


class Derived(C.Structure):
    _fields_ = [
        ("z_min", C.c_float * (MAX_LAYERS + 2)),
        ("z_max", C.c_float * (MAX_LAYERS + 2)),
        ("mutr", C.c_float * (MAX_LAYERS + 2)),
        ("start_weight", C.c_float),
        ("critical_angle", C.c_float * (MAX_SDS + 1)),
        ("det_angle_rad", C.c_float * (MAX_SDS + 1)),
    ]


class DeviceInfo(C.Structure):
    _fields_ = [
        ("name", C.c_char * 100),
        ("major", C.c_int32),
        ("minor", C.c_int32),
        ("sm_count", C.c_int32),
        ("max_threads_per_sm", C.c_int32),
        ("global_mem", C.c_uint64),
        ("reference_threads", C.c_uint64),
    ]


class DeviceOutputs(C.Structure):
    """mcml_device_outputs: a run's outputs in device memory."""
    _fields_ = [
        ("records", C.c_void_p),
        ("rows", C.c_void_p),
        ("A_rz", C.c_void_p),
        ("A0_z", C.c_void_p),
        ("n_records", C.c_uint64),
        ("detected", C.c_uint64 * MAX_SDS),
        ("arz_count", C.c_uint64),
        ("a0z_count", C.c_uint64),
        ("photons", C.c_uint64),
        ("row_len", C.c_uint32),
        ("stream", C.c_void_p),
    ]


class NoallocResult(C.Structure):
    """mcml_noalloc_result, written to device memory by mcml_run_noalloc."""
    _fields_ = [
        ("detected", C.c_uint64 * MAX_SDS),
        ("weight_sum", C.c_double * MAX_SDS),
        ("weight_sumsq", C.c_double * MAX_SDS),
        ("steps", C.c_uint64),
    ]


class BatchOpts(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("device", C.c_int32),
        ("photons_per_slot", C.c_uint32),
        ("block_size", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("stream", C.c_void_p),
        ("no_graph", C.c_int32),
    ]


class BatchTuning(C.Structure):
    _fields_ = [
        ("block_size", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("photons_per_slot", C.c_uint32),
        ("pilot_ms", C.c_float),
    ]


class CheckpointOpts(C.Structure):
    _fields_ = [
        ("path", C.c_char_p),
        ("chunk_slots", C.c_uint64),
        ("max_chunks", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class CheckpointInfo(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("seed", "slot_begin", "photons", "slots", "slots_done",
                                          "records", "steps", "launches")]


class HostData(C.Structure):
    _fields_ = [
        ("photons", C.c_uint64),
        ("detected", C.c_void_p),
        ("weight_sum", C.c_void_p),
        ("rows", C.c_void_p),
        ("A_rz", C.c_void_p),
        ("A0_z", C.c_void_p),
        ("grid_nr", C.c_uint32),
        ("grid_nz", C.c_uint32),
        ("grid_dr", C.c_float),
        ("grid_dz", C.c_float),
        ("gpu_name", C.c_char_p),
    ]


INCOMPLETE = 1  # MCML_INCOMPLETE: a checkpointed run stopped early

_lib: Optional[C.CDLL] = None

# (name, restype, argtypes) of every entry point of include/mcml_b200.h
_SIGNATURES = [
    ("mcml_version", C.c_char_p, []),
    ("mcml_strerror", C.c_char_p, [C.c_int]),
    ("mcml_last_error", C.c_char_p, []),
    ("mcml_device_count", C.c_int, [C.POINTER(C.c_int)]),
    ("mcml_get_device_info", C.c_int, [C.c_int, C.POINTER(DeviceInfo)]),
    ("mcml_parse_config", C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(Sim), C.c_int,
                                    C.POINTER(C.c_int)]),
    ("mcml_derive", C.c_int, [C.POINTER(Sim), C.POINTER(Derived)]),
    ("mcml_create", C.c_int, [C.POINTER(Sim), C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    ("mcml_set_sim", C.c_int, [C.c_void_p, C.POINTER(Sim)]),
    ("mcml_destroy", None, [C.c_void_p]),
    ("mcml_run", C.c_int, [C.c_void_p, C.POINTER(Result)]),
    ("mcml_launch_run", C.c_int, [C.c_void_p]),
    ("mcml_replay", C.c_int, [C.c_void_p, C.POINTER(Result)]),
    ("mcml_launch_replay", C.c_int, [C.c_void_p]),
    ("mcml_get_result", C.c_int, [C.c_void_p, C.POINTER(Result)]),
    ("mcml_get_detections", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_uint64, C.POINTER(C.c_uint64)]),
    ("mcml_get_rows", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64,
                                C.POINTER(C.c_uint64)]),
    ("mcml_get_tallies", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mcml_get_device_outputs", C.c_int, [C.c_void_p, C.POINTER(DeviceOutputs)]),
    ("mcml_average_pathlength", C.c_int, [C.c_void_p, C.c_void_p]),
    ("mcml_write_outputs", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_uint32,
                                     C.c_double, C.c_double]),
    ("mcml_uniform_stream", C.c_int, [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                      C.c_void_p]),
    ("mcml_run_noalloc", C.c_int, [C.POINTER(Sim), C.c_uint64, C.c_uint64, C.c_int,
                                   C.c_void_p, C.c_void_p]),
    ("mcml_batch_create", C.c_int, [C.c_void_p, C.c_int, C.POINTER(BatchOpts),
                                    C.POINTER(C.c_void_p)]),
    ("mcml_batch_autotune", C.c_int, [C.c_void_p, C.c_double, C.POINTER(BatchTuning)]),
    ("mcml_batch_run", C.c_int, [C.c_void_p, C.c_void_p]),
    ("mcml_batch_launch", C.c_int, [C.c_void_p]),
    ("mcml_batch_get_results", C.c_int, [C.c_void_p, C.c_void_p]),
    ("mcml_batch_destroy", None, [C.c_void_p]),
    ("mcml_run_checkpointed", C.c_int, [C.c_void_p, C.POINTER(CheckpointOpts),
                                        C.POINTER(Result)]),
    ("mcml_checkpoint_read_info", C.c_int, [C.c_char_p, C.POINTER(CheckpointInfo)]),
    ("mcml_write_host_outputs", C.c_int, [C.POINTER(Sim), C.POINTER(HostData), C.c_char_p,
                                          C.c_char_p, C.c_uint32, C.c_double, C.c_double]),
    ("mcml_probe_spin", C.c_int, [C.c_int, C.c_float, C.c_uint64, C.c_uint64, C.c_void_p]),
    ("mcml_probe_reflect", C.c_int, [C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint64,
                                     C.c_uint64, C.c_void_p]),
    ("mcml_format_rows_text", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p,
                                        C.c_uint64, C.POINTER(C.c_uint64)]),
]


def exported_symbols() -> list[str]:
    """Entry points this module binds (all of include/mcml_b200.h)."""
    return [s[0] for s in _SIGNATURES]


def load_library() -> C.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = lib_path()
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m mcml_gpu_b200.build`")
    lib = C.CDLL(str(p))
    for name, res, args in _SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _device_ptr(t, name: str, *, device: int, shape: Optional[tuple] = None) -> C.c_void_p:
    """Address of a torch tensor handed to a kernel: it must be a C-contiguous
    float32 tensor on CUDA device `device`, of `shape` where given (None
    entries match any size).  A host tensor's address would be read by the
    GPU as a device address; a strided or differently typed one would be
    read as garbage -- both are rejected here instead."""
    import torch
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name}: expected a torch tensor, got {type(t).__name__}")
    if t.device.type != "cuda" or t.device.index != device:
        raise ValueError(f"{name}: must be on cuda:{device}, is on {t.device}")
    if t.dtype != torch.float32:
        raise ValueError(f"{name}: must be float32, is {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: must be contiguous")
    if shape is not None and (t.dim() != len(shape) or
                              any(w is not None and w != g for w, g in zip(shape, t.shape))):
        raise ValueError(f"{name}: shape {tuple(t.shape)}, expected {shape}")
    return C.c_void_p(t.data_ptr())


def _check(rc: int, where: str) -> None:
    if rc != 0:
        lib = load_library()
        raise MCMLError(rc, where, lib.mcml_last_error().decode(errors="replace"))


def device_count() -> int:
    lib = load_library()
    n = C.c_int(0)
    rc = lib.mcml_device_count(C.byref(n))
    return n.value if rc == 0 else 0


def device_info(device: int = 0) -> DeviceInfo:
    lib = load_library()
    info = DeviceInfo()
    _check(lib.mcml_get_device_info(device, C.byref(info)), "mcml_get_device_info")
    return info


def parse_config(sim_json: os.PathLike | str, input_txt: os.PathLike | str) -> list[Sim]:
    """read_mua_mus (io.cpp:35-256): returns one Sim per simulation."""
    lib = load_library()
    n = C.c_int(0)
    _check(lib.mcml_parse_config(str(sim_json).encode(), str(input_txt).encode(), None, 0,
                                 C.byref(n)), "mcml_parse_config")
    arr = (Sim * n.value)()
    _check(lib.mcml_parse_config(str(sim_json).encode(), str(input_txt).encode(), arr, n.value,
                                 C.byref(n)), "mcml_parse_config")
    return list(arr)


def derive(sim: Sim) -> Derived:
    lib = load_library()
    d = Derived()
    _check(lib.mcml_derive(C.byref(sim), C.byref(d)), "mcml_derive")
    return d


def make_sim(layers: Sequence[Sequence[float]], detectors: Sequence[Sequence[float]], *,
             photons: int, upper_n: float = 1.457, lower_n: float = 1.457,
             detector_reflectance: float = 0.0, source_oblique: bool = True,
             detector_oblique: bool = True, source: Sequence[float] = (0.37, 0.075, 0.0)) -> Sim:
    """Builds a Sim.  layers: (height, mua, mus, n, g) per layer, the last
    layer's height ignored.  detectors: (pos, NA, radius, angle_deg).
    source: (NA, radius, angle_deg)."""
    s = Sim()
    s.number_photons = int(photons)
    s.num_layers = len(layers)
    s.num_sds = len(detectors)
    s.upper_n, s.lower_n = upper_n, lower_n
    s.detector_reflectance = detector_reflectance
    s.source_probe_oblique = int(bool(source_oblique))
    s.detector_probe_oblique = int(bool(detector_oblique))
    s.source_NA, s.source_radius, s.source_angle_deg = source
    for i, (h, mua, mus, n, g) in enumerate(layers):
        s.height[i], s.mua[i], s.mus[i], s.n[i], s.g[i] = h, mua, mus, n, g
    for i, (pos, na, r, ang) in enumerate(detectors):
        s.det_pos[i], s.det_NA[i], s.det_radius[i], s.det_angle_deg[i] = pos, na, r, ang
    return s


def shard(rank: int, world: int, photons: int, weak: bool = True) -> tuple[int, int]:
    """(first subsequence, photon count) of one rank of a multi-GPU run.

    Photons are independent, so ranks walk disjoint ranges of XORWOW
    subsequences and only their per-SDS sums and u64 tallies are added at
    the end.  weak: every rank walks `photons` photons (ranges rank*photons
    ...); strong: the ranks split `photons`.  A rank never uses more
    subsequences than it has photons, so starting each range at the rank's
    first photon index keeps the ranges disjoint."""
    if weak:
        return rank * photons, photons
    base, extra = divmod(photons, world)
    n = base + (1 if rank < extra else 0)
    return rank * base + min(rank, extra), n


def format_rows_text(rows: np.ndarray) -> bytes:
    """The bytes of pathlength_SDS_#.txt for these rows (n x row_len float32)."""
    lib = load_library()
    rows = np.ascontiguousarray(rows, dtype=np.float32)
    n, rl = (rows.shape[0], rows.shape[1]) if rows.ndim == 2 else (0, 1)
    size = C.c_uint64()
    _check(lib.mcml_format_rows_text(rows.ctypes.data, n, rl, None, 0, C.byref(size)),
           "mcml_format_rows_text")
    buf = C.create_string_buffer(max(int(size.value), 1))
    _check(lib.mcml_format_rows_text(rows.ctypes.data, n, rl, buf, size.value, C.byref(size)),
           "mcml_format_rows_text")
    return buf.raw[:size.value]


def probe_spin(g: float, n: int, seed: int = 1, device: int = 0) -> tuple[float, float]:
    """Mean cos and cos^2 of the walk's spin() with anisotropy g (GPU)."""
    lib = load_library()
    out = (C.c_double * 2)()
    _check(lib.mcml_probe_spin(device, g, n, seed, out), "mcml_probe_spin")
    return out[0], out[1]


def probe_reflect(n1: float, n2: float, cos_i: float, n: int, seed: int = 1,
                  device: int = 0) -> tuple[float, float]:
    """Reflected fraction and mean transmitted |dz| of the walk's reflect() (GPU)."""
    lib = load_library()
    out = (C.c_double * 2)()
    _check(lib.mcml_probe_reflect(device, n1, n2, cos_i, n, seed, out), "mcml_probe_reflect")
    return out[0], out[1]


def checkpoint_info(path: os.PathLike | str) -> CheckpointInfo:
    """Header of a checkpoint file, checked (no device needed)."""
    lib = load_library()
    info = CheckpointInfo()
    _check(lib.mcml_checkpoint_read_info(os.fsencode(str(path)), C.byref(info)),
           "mcml_checkpoint_read_info")
    return info


def uniform_stream(seed: int, subsequence: int, count: int, device: int = 0) -> np.ndarray:
    """The first `count` curand_uniform draws of XORWOW subsequence
    `subsequence` under `seed` (the stream of the reference's thread)."""
    lib = load_library()
    out = np.empty(count, dtype=np.float32)
    _check(lib.mcml_uniform_stream(device, seed, subsequence, count,
                                   out.ctypes.data_as(C.c_void_p)), "mcml_uniform_stream")
    return out


class Simulation:
    """One simulation context (mcml_ctx): first pass, replay, outputs."""

    def __init__(self, sim: Sim, *, seed: int = 0, slots: int = 0, device: int = 0,
                 grid: Optional[tuple] = None, record_capacity: int = 0,
                 stream: Optional[int] = None, block_size: int = 0, blocks_per_sm: int = 0,
                 replay_step_budget: int = 0, slot_begin: int = 0):
        self._lib = load_library()
        self.sim = sim
        o = Opts()
        o.seed = seed
        o.slots = slots
        o.device = device
        if grid is not None:
            o.grid_nr, o.grid_nz, o.grid_dr, o.grid_dz = grid
        o.record_capacity = record_capacity
        o.stream = stream
        o.block_size = block_size
        o.blocks_per_sm = blocks_per_sm
        o.replay_step_budget = replay_step_budget
        o.slot_begin = slot_begin
        self.opts = o
        self._ctx = C.c_void_p()
        _check(self._lib.mcml_create(C.byref(sim), C.byref(o), C.byref(self._ctx)),
               "mcml_create")

    @property
    def num_layers(self) -> int:
        return int(self.sim.num_layers)

    @property
    def num_sds(self) -> int:
        return int(self.sim.num_sds)

    @property
    def grid(self) -> tuple:
        o = self.opts
        return (o.grid_nr or 1000, o.grid_nz or 500, o.grid_dr or 0.01, o.grid_dz or 0.01)

    def set_sim(self, sim: Sim) -> None:
        _check(self._lib.mcml_set_sim(self._ctx, C.byref(sim)), "mcml_set_sim")
        self.sim = sim

    def run(self) -> Result:
        r = Result()
        _check(self._lib.mcml_run(self._ctx, C.byref(r)), "mcml_run")
        return r

    def run_checkpointed(self, path: os.PathLike | str, *, chunk_slots: int = 0,
                         max_chunks: int = 0) -> Optional[Result]:
        """First pass in launches of chunk_slots slots, checkpointed to
        `path` after each (resuming from it if present).  Returns the
        result, or None when max_chunks launches ran and slots remain."""
        o = CheckpointOpts(os.fsencode(str(path)), int(chunk_slots), int(max_chunks), 0)
        r = Result()
        rc = self._lib.mcml_run_checkpointed(self._ctx, C.byref(o), C.byref(r))
        if rc == INCOMPLETE:
            return None
        _check(rc, "mcml_run_checkpointed")
        return r

    def launch_run(self) -> None:
        _check(self._lib.mcml_launch_run(self._ctx), "mcml_launch_run")

    def launch_replay(self) -> None:
        _check(self._lib.mcml_launch_replay(self._ctx), "mcml_launch_replay")

    def result(self) -> Result:
        r = Result()
        _check(self._lib.mcml_get_result(self._ctx, C.byref(r)), "mcml_get_result")
        return r

    def replay(self) -> Result:
        r = Result()
        _check(self._lib.mcml_replay(self._ctx, C.byref(r)), "mcml_replay")
        return r

    def detections(self, sds: int) -> tuple[np.ndarray, np.ndarray]:
        n = C.c_uint64(0)
        _check(self._lib.mcml_get_detections(self._ctx, sds, None, None, 0, C.byref(n)),
               "mcml_get_detections")
        ids = np.empty(n.value, dtype=np.uint64)
        w = np.empty(n.value, dtype=np.float32)
        _check(self._lib.mcml_get_detections(self._ctx, sds, ids.ctypes.data_as(C.c_void_p),
                                             w.ctypes.data_as(C.c_void_p), n.value,
                                             C.byref(n)), "mcml_get_detections")
        return ids, w

    def rows(self, sds: int) -> tuple[np.ndarray, np.ndarray]:
        L = self.num_layers
        n = C.c_uint64(0)
        _check(self._lib.mcml_get_rows(self._ctx, sds, None, None, 0, C.byref(n)),
               "mcml_get_rows")
        rows = np.empty((n.value, L + 2), dtype=np.float32)
        inter = np.empty((n.value, L), dtype=np.uint32)
        _check(self._lib.mcml_get_rows(self._ctx, sds, rows.ctypes.data_as(C.c_void_p),
                                       inter.ctypes.data_as(C.c_void_p), n.value, C.byref(n)),
               "mcml_get_rows")
        return rows, inter

    def tallies(self) -> tuple[np.ndarray, np.ndarray]:
        nr, nz, _, _ = self.grid
        S = self.num_sds
        arz = np.empty((S, nz, nr), dtype=np.uint64)
        a0z = np.empty((S, nz), dtype=np.uint64)
        _check(self._lib.mcml_get_tallies(self._ctx, arz.ctypes.data_as(C.c_void_p),
                                          a0z.ctypes.data_as(C.c_void_p)), "mcml_get_tallies")
        return arz, a0z

    def device_outputs(self) -> dict:
        """The last run's outputs as torch tensors on this context's GPU,
        aliasing the library's memory (mcml_get_device_outputs): `records`
        (D, 10) float32 words of the 40-byte records (word 3 is the detected
        weight), `rows` (D, L+2) float32 or None, `A_rz` (S, nz, nr) and
        `A0_z` (S, nz) int64 views of the u64 quanta or None, `detected`
        (host list, per SDS), `photons`.  File order: SDS-major, photon
        order within an SDS.  Valid until the context's next run, replay or
        close; copy what must outlive that."""
        import torch
        o = DeviceOutputs()
        _check(self._lib.mcml_get_device_outputs(self._ctx, C.byref(o)),
               "mcml_get_device_outputs")
        dev = torch.device("cuda", self.opts.device)
        D, rl, S = int(o.n_records), int(o.row_len), self.num_sds
        nr, nz, _, _ = self.grid

        def view(ptr, shape, typestr):
            if not ptr or any(d == 0 for d in shape):
                return torch.zeros(shape, dtype=torch.float32 if typestr == "<f4" else torch.int64,
                                   device=dev)
            return torch.as_tensor(_CudaArray(ptr, shape, typestr), device=dev)
        return {
            "records": view(o.records, (D, 10), "<f4"),
            "rows": view(o.rows, (D, rl), "<f4") if o.rows else None,
            "A_rz": view(o.A_rz, (S, nz, nr), "<i8") if o.A_rz else None,
            "A0_z": view(o.A0_z, (S, nz), "<i8") if o.A0_z else None,
            "detected": [int(v) for v in o.detected[:S]],
            "photons": int(o.photons),
        }

    def average_pathlength(self) -> np.ndarray:
        out = np.empty(self.num_sds * self.num_layers, dtype=np.float64)
        _check(self._lib.mcml_average_pathlength(self._ctx, out.ctypes.data_as(C.c_void_p)),
               "mcml_average_pathlength")
        return out.reshape(self.num_sds, self.num_layers)

    def write_outputs(self, directory: str, output_txt: str, flags: int, sim_s: float = 0.0,
                      replay_s: float = 0.0) -> None:
        _check(self._lib.mcml_write_outputs(self._ctx, directory.encode(), output_txt.encode(),
                                            flags, sim_s, replay_s), "mcml_write_outputs")

    def close(self) -> None:
        if getattr(self, "_ctx", None) and self._ctx.value:
            self._lib.mcml_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _CudaArray:
    """A device buffer of the library seen through __cuda_array_interface__,
    so that torch.as_tensor wraps it without a copy."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"data": (int(ptr), False), "shape": tuple(shape),
                                         "typestr": typestr, "strides": None, "version": 2}


class Batch:
    """Many parameter sets in one persistent launch (mcml_batch_*).  Set b
    walks ceil(N_b / photons_per_slot) slots of seed + b, the same photons
    as Simulation(sims[b], seed=seed + b, slots=...) alone."""

    def __init__(self, sims: Sequence[Sim], *, seed: int = 0, device: int = 0,
                 photons_per_slot: int = 0, block_size: int = 0, blocks_per_sm: int = 0,
                 stream: Optional[int] = None, graph: bool = True):
        self._lib = load_library()
        self.sims = (Sim * len(sims))(*sims)
        o = BatchOpts()
        o.seed = seed
        o.device = device
        o.photons_per_slot = photons_per_slot
        o.block_size = block_size
        o.blocks_per_sm = blocks_per_sm
        o.stream = stream
        o.no_graph = 0 if graph else 1
        self._b = C.c_void_p()
        _check(self._lib.mcml_batch_create(self.sims, len(sims), C.byref(o), C.byref(self._b)),
               "mcml_batch_create")

    def autotune(self, photon_fraction: float = 1 / 16) -> BatchTuning:
        t = BatchTuning()
        _check(self._lib.mcml_batch_autotune(self._b, photon_fraction, C.byref(t)),
               "mcml_batch_autotune")
        return t

    def run(self) -> list:
        res = (Result * len(self.sims))()
        _check(self._lib.mcml_batch_run(self._b, res), "mcml_batch_run")
        return list(res)

    def launch(self) -> None:
        _check(self._lib.mcml_batch_launch(self._b), "mcml_batch_launch")

    def results(self) -> list:
        res = (Result * len(self.sims))()
        _check(self._lib.mcml_batch_get_results(self._b, res), "mcml_batch_get_results")
        return list(res)

    def close(self) -> None:
        if getattr(self, "_b", None) and self._b.value:
            self._lib.mcml_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sample_sets(base: Sim, count: int, seed: int, *, mua=(0.05, 0.5), mus=(50.0, 250.0),
                photons=(1e5, 1e7)) -> list:
    """Parameter sets for a batch: `base`'s geometry with per-layer mua and
    mus drawn uniformly and per-set photon counts drawn log-uniformly, from a
    seeded generator (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    out = []
    L = int(base.num_layers)
    for _ in range(count):
        s = Sim.from_buffer_copy(base)
        for l in range(L):
            s.mua[l] = float(rng.uniform(*mua))
            s.mus[l] = float(rng.uniform(*mus))
        s.number_photons = int(round(10 ** rng.uniform(np.log10(photons[0]), np.log10(photons[1]))))
        out.append(s)
    return out
