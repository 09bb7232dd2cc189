"""Batched assembly of many independent meshes in one persistent, CUDA-graph
captured launch (db2_batch_* in the C ABI), and its autotuner.

Every member assembles kappa*inner(grad(u), grad(v))*dx on its own space
(P1 or P2, triangles or tetrahedra) with its own P1 kappa.  ``assemble()``
replays one captured graph (counter reset, kappa packing, one persistent
kernel over all tiles); ``assemble_loop()`` is the reference: one launch per
member.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import time

import numpy as np

from . import _capi
from ._capi import call
from .assembling import _PREC, _stream
from .la import Matrix


class BatchAssembler:
    def __init__(self, members, tile_threads=0, seg_cap_bytes=0, ctas_per_sm=0):
        """members: list of (FunctionSpace V, Function kappa on the P1 space of V's mesh)."""
        import torch
        self.members = list(members)
        n = len(self.members)
        if n == 0:
            raise ValueError("empty batch")
        self.matrices = []
        pats, kps, vps = (C.c_void_p * n)(), (C.c_void_p * n)(), (C.c_void_p * n)()
        forms = (_capi.DB2Form * n)()
        for i, (V, kappa) in enumerate(self.members):
            if kappa.function_space().mesh() is not V.mesh():
                raise ValueError(f"member {i}: kappa lives on another mesh")
            A = Matrix(V.pattern())
            self.matrices.append(A)
            pats[i] = V.pattern().handle
            kps[i] = kappa.tensor().data_ptr()
            vps[i] = A.values_tensor().data_ptr()
            forms[i] = _capi.make_form(_capi.FORM_DIFFUSION, _capi.COEFF_P1)
        self._keep = (pats, kps, vps, forms)
        h = C.c_void_p()
        torch.cuda.synchronize()
        call("db2_batch_create", n, pats, forms, kps, vps, int(tile_threads), int(seg_cap_bytes),
             int(ctas_per_sm), C.byref(h))
        self._h = h
        t, c, k = C.c_int64(), C.c_int64(), C.c_int()
        call("db2_batch_info", h, C.byref(t), C.byref(c), C.byref(k))
        self.ntiles, self.ncells, self.ctas = t.value, c.value, k.value
        self.params = (tile_threads, seg_cap_bytes, ctas_per_sm)

    def assemble(self, precision="fp64"):
        """One graph replay: all members' matrices."""
        call("db2_batch_assemble", self._h, _PREC[precision], _stream())
        return self.matrices

    def assemble_loop(self, precision="fp64"):
        """Reference: one kernel launch per member."""
        call("db2_batch_assemble_loop", self._h, _PREC[precision], _stream())
        return self.matrices

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _capi._lib is not None:
            _capi.lib().db2_batch_destroy(h)
            self._h = None


def _time(fn, reps=5):
    import torch
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


DEFAULT_CANDIDATES = [(t, c, k) for t in (64, 128, 256) for c in (12288, 24576, 49152)
                      for k in (0,)]


def batch_signature(members):
    """Key of a batch for the tuning cache: element mix and size histogram."""
    h = hashlib.sha1()
    for V, _ in members:
        h.update(f"{V.mesh().topology_dim()}:{V.degree()}:{int(np.log2(max(V.mesh().num_cells(), 1)))};".encode())
    return h.hexdigest()[:16]


def autotune(members, candidates=None, cache_path=None, precision="fp64", reps=5):
    """Pick (tile_threads, seg_cap_bytes, ctas_per_sm) for a batch by timing
    each candidate's graph replay; results are cached in a JSON file keyed by
    the batch signature.  Returns (best_params, {params: ms})."""
    cache_path = cache_path or os.path.join(os.path.expanduser("~"), ".cache", "dolfin_b200_tune.json")
    key = batch_signature(members) + ":" + precision
    cache = {}
    if os.path.exists(cache_path):
        try:
            with open(cache_path) as fh:
                cache = json.load(fh)
        except Exception:
            cache = {}
    if key in cache:
        return tuple(cache[key]["best"]), cache[key]["timings"]
    timings = {}
    best, best_ms = None, float("inf")
    for cand in candidates or DEFAULT_CANDIDATES:
        try:
            B = BatchAssembler(members, *cand)
        except _capi.DB2Error:
            continue
        ms = _time(lambda: B.assemble(precision), reps)
        timings[str(cand)] = ms
        if ms < best_ms:
            best, best_ms = cand, ms
        del B
    try:
        os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        cache[key] = {"best": list(best), "timings": timings, "when": time.time()}
        with open(cache_path, "w") as fh:
            json.dump(cache, fh)
    except OSError:
        pass
    return best, timings
