"""White Monte Carlo relabelling (mcml_wmc_rescale) from Python.

One replay of a baseline tissue gives, for every detected photon of an
SDS, its weight, per-layer pathlengths and per-layer interaction counts
(Simulation.rows).  rescale() turns them into that SDS's reflectance for
any number of (mua', mus') combinations in one GPU pass.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import MAX_LAYERS, _check, _device_ptr, load_library

__all__ = ["WmcSet", "Prepared", "rescale", "rescale_reference"]


class WmcSet(C.Structure):
    _fields_ = [
        ("pathlength", C.c_void_p),
        ("interactions", C.c_void_p),
        ("weight", C.c_void_p),
        ("count", C.c_uint64),
        ("num_layers", C.c_uint32),
    ]


def _bind(lib):
    if getattr(lib, "_wmc_bound", False):
        return
    lib.mcml_wmc_workspace_bytes.restype = C.c_uint64
    lib.mcml_wmc_workspace_bytes.argtypes = [C.c_uint64, C.c_uint64]
    lib.mcml_wmc_rescale.restype = C.c_int
    lib.mcml_wmc_rescale.argtypes = [C.POINTER(WmcSet), C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_uint64, C.c_double, C.c_void_p, C.c_void_p,
                                     C.c_uint64, C.c_void_p]
    lib._wmc_bound = True


class Prepared:
    """Replay rows and interaction counts of one SDS on the device, in the
    layer-major layout mcml_wmc_rescale reads."""

    def __init__(self, rows: np.ndarray, interactions: np.ndarray, device: int = 0):
        import torch
        dev = torch.device("cuda", device)
        rows = np.asarray(rows, dtype=np.float32)
        self.L = rows.shape[1] - 2
        self.D = rows.shape[0]
        self.device = device
        self.pl = torch.from_numpy(np.ascontiguousarray(rows[:, 1:self.L + 1].T)).to(dev)
        self.ni = torch.from_numpy(
            np.ascontiguousarray(np.asarray(interactions, np.float32).T)).to(dev)
        self.w = torch.from_numpy(np.ascontiguousarray(rows[:, 0])).to(dev)
        self._ws = None

    def rescale(self, base_mua, base_mus, combos, photons: int):
        """combos: (C, 2L) CUDA float32 tensor.  Returns C float64 reflectances
        (CUDA tensor), enqueued on the current torch stream."""
        import torch
        lib = load_library()
        _bind(lib)
        dev = torch.device("cuda", self.device)
        pc = _device_ptr(combos, "combos", device=self.device, shape=(None, 2 * self.L))
        Cn = combos.shape[0]
        out = torch.empty(Cn, dtype=torch.float64, device=dev)
        nbytes = int(lib.mcml_wmc_workspace_bytes(self.D, Cn))
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        s = WmcSet(self.pl.data_ptr(), self.ni.data_ptr(), self.w.data_ptr(), self.D, self.L)
        bm = (C.c_float * MAX_LAYERS)(*[float(v) for v in base_mua][:self.L])
        bs = (C.c_float * MAX_LAYERS)(*[float(v) for v in base_mus][:self.L])
        stream = torch.cuda.current_stream(dev).cuda_stream
        _check(lib.mcml_wmc_rescale(C.byref(s), bm, bs, pc, Cn,
                                    float(0xFFFFFFFF) * float(photons), C.c_void_p(out.data_ptr()),
                                    C.c_void_p(self._ws.data_ptr()), self._ws.numel(),
                                    C.c_void_p(stream)),
               "mcml_wmc_rescale")
        return out


def rescale(rows: np.ndarray, interactions: np.ndarray, base_mua, base_mus, combos, photons: int,
            device: int = 0):
    """rows: (D, L+2) float32 replay rows (weight, PL_1..L, steps);
    interactions: (D, L) counts; base_mua/base_mus: the run's L coefficients;
    combos: (C, 2L) array or CUDA tensor of (mua'_1..L, mus'_1..L);
    photons: N of the run.  Returns a float64 CUDA tensor of C reflectances."""
    import torch
    prep = Prepared(rows, interactions, device)
    if not torch.is_tensor(combos):
        combos = torch.from_numpy(np.asarray(combos, dtype=np.float32))
    combos = combos.to(torch.device("cuda", device), torch.float32).contiguous()
    return prep.rescale(base_mua, base_mus, combos, photons)


def rescale_reference(rows, interactions, base_mua, base_mus, combos, photons):
    """The same formula in float64 numpy (test oracle for the kernel's numerics)."""
    rows = np.asarray(rows, np.float64)
    L = rows.shape[1] - 2
    w, pl = rows[:, 0], rows[:, 1:L + 1]
    n = np.asarray(interactions, np.float64)
    combos = np.asarray(combos, np.float64)
    bm, bs = np.asarray(base_mua, np.float64)[:L], np.asarray(base_mus, np.float64)[:L]
    dmut = (combos[:, :L] - bm) + (combos[:, L:] - bs)
    logr = np.log(combos[:, L:] / bs)
    expo = -dmut @ pl.T + logr @ n.T
    return (np.exp(expo) * w[None, :]).sum(axis=1) / (4294967295.0 * photons)


# Entry points of include/mcml_b200.h bound by this module.
BOUND = ["mcml_wmc_rescale", "mcml_wmc_workspace_bytes"]
