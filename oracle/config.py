"""Configuration reader of the oracle -- TEST INFRASTRUCTURE ONLY.

Reads ``sim_set.json`` and ``input.txt`` the way the reference's
``read_mua_mus`` does (io.cpp:35-256) into the ``mcml_sim`` structure of
include/mcml_b200.h, without the CUDA library: the CPU restatement, the
reference arm of bench.py and its CPU-baseline leg load only the oracle's
own ``liboracle.so`` (and libc for ``strtof``).

Numbers of input.txt are read as the reference's ``ifstream >> float``
reads them: one correctly rounded decimal-to-float conversion (libc
``strtof``), not through a double.  JSON numbers are doubles in the
reference's parser and narrowed to float where its structures hold floats.
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

MAX_LAYERS = 10  # PRESET_NUM_LAYER, header.h
MAX_SDS = 30     # PRESET_NUM_DETECTOR, header.h


class Sim(C.Structure):
    """mcml_sim of include/mcml_b200.h (same field order and types)."""
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


class Derived(C.Structure):
    """mcml_derived of include/mcml_b200.h."""
    _fields_ = [
        ("z_min", C.c_float * (MAX_LAYERS + 2)),
        ("z_max", C.c_float * (MAX_LAYERS + 2)),
        ("mutr", C.c_float * (MAX_LAYERS + 2)),
        ("start_weight", C.c_float),
        ("critical_angle", C.c_float * (MAX_SDS + 1)),
        ("det_angle_rad", C.c_float * (MAX_SDS + 1)),
    ]


_libc = C.CDLL(None)
_libc.strtof.restype = C.c_float
_libc.strtof.argtypes = [C.c_char_p, C.POINTER(C.c_char_p)]


def _to_float(token: str) -> float:
    return float(_libc.strtof(token.encode(), None))


class ConfigError(ValueError):
    """A configuration the reference rejects (its message, io.cpp:48-160)."""


def _flag(conf: dict, key: str) -> int:
    v = conf[key]
    if v == 1:
        return 1
    if v == 0:
        return 0
    raise ConfigError(f"{key}: {v}is not 1 or 0!")


def read_config(sim_json: str | Path, input_txt: str | Path) -> list[Sim]:
    """read_mua_mus (io.cpp:35-256): one Sim per simulation of the files."""
    conf = json.loads(Path(sim_json).read_text())
    n_sims = int(conf["number_simulation"])
    photons = int(conf["number_photons"])
    src_obl = _flag(conf, "source_probe_oblique")
    det_obl = _flag(conf, "detector_probe_oblique")
    refl = float(conf["detector_reflectance"])
    if refl < 0 or refl > 1:
        raise ConfigError(f"Detector reflectance: {refl} is out of range !")
    L = int(conf["number_layers"])
    if L > MAX_LAYERS:
        raise ConfigError("Number of layer is too large!")
    probes = conf["probes"]
    S = int(probes["num_SDS"])
    if S > MAX_SDS:
        raise ConfigError("Number of SDS is too large!")
    dets = probes["detectors"]
    if S != len(dets):
        raise ConfigError(f"Number of SDS : {S} not match the probe setting : {len(dets)} !")
    tokens = Path(input_txt).read_text().split()
    per_sim = 5 * (L - 1) + 4
    if len(tokens) < per_sim * n_sims:
        raise ConfigError("input.txt holds fewer values than the simulations need")
    out = []
    for i in range(n_sims):
        vals = [_to_float(t) for t in tokens[i * per_sim:(i + 1) * per_sim]]
        s = Sim()
        s.number_photons = photons
        s.num_layers = L
        s.num_sds = S
        s.upper_n = float(conf["upper_n"])
        s.lower_n = float(conf["lower_n"])
        s.detector_reflectance = refl
        s.source_probe_oblique = src_obl
        s.detector_probe_oblique = det_obl
        src = probes["source"]
        s.source_NA = float(src["NA"])
        s.source_radius = float(src["radius"])
        s.source_angle_deg = float(src["angle"])
        for d, det in enumerate(dets):
            s.det_pos[d] = float(det["pos"])
            s.det_NA[d] = float(det["NA"])
            s.det_radius[d] = float(det["radius"])
            s.det_angle_deg[d] = float(det["angle"])
        k = 0
        for l in range(L):
            if l < L - 1:
                s.height[l] = vals[k]
                k += 1
            s.mua[l], s.mus[l], s.n[l], s.g[l] = vals[k:k + 4]
            k += 4
        # the reference checks the last layer only (io.cpp:148-160)
        j = L - 1
        if not s.mus[j] > 0:
            raise ConfigError(f"Mus for simulation {i} layer {j} Error with value {s.mus[j]:g} !")
        if not s.n[j] > 1:
            raise ConfigError(f"n for simulation {i} layer {j} Error with value {s.n[j]:g} !")
        if s.g[j] > 1:
            raise ConfigError(f"g for simulation {i} layer {j} Error with value {s.g[j]:g} !")
        out.append(s)
    return out
