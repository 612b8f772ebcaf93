"""``SolveServer``: a solve service on one GPU (sdot_server_* in include/sdot.h).

Requests (one ``SotSolver.solve`` each, src/solvers/SotSolver.cc:105-215,
optionally over an epsilon-scaling sequence as in SemiDiscreteOT.cc:878-922)
are queued, admitted by device-memory budget into a fixed number of slots and
solved concurrently; ``submit`` returns a ticket, ``wait`` the potential and
the request's timings.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .parameters import SolverParameters
from .solver import SotSolver


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class SolveServer:
    def __init__(self, n_slots: int = 4, device: int = 0, memory_budget: int = 0):
        self._L = _lib.load()
        h = C.c_void_p()
        st = self._L.sdot_server_create(C.byref(h), int(device), int(n_slots), int(memory_budget))
        if st != _lib.SDOT_OK:
            raise _lib.SdotError(st, "sdot_server_create failed (no CUDA device?)")
        self._h = h
        self._sizes = {}

    def close(self):
        if getattr(self, "_h", None):
            self._L.sdot_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != _lib.SDOT_OK:
            raise _lib.SdotError(st, self._L.sdot_server_last_error(self._h).decode())

    def submit(self, source: dict, y, nu, params: SolverParameters, method: str = "auto",
               precision: str = "hybrid", hessian: str = "auto", psi0=None, epsilon_scaling_factor: float = 10.0,
               epsilon_scaling_steps: int = 1, intermediate_tolerance: float = 0.0, with_cells: bool = True) -> int:
        dim = int(np.asarray(y).shape[1])
        x = _f64(source["x"]).reshape(-1, dim)
        jxw, dens = _f64(source["jxw"]), _f64(source["density"])
        y, nu = _f64(y).reshape(-1, dim), _f64(nu)
        keep = [x, jxw, dens, y, nu]
        ncells, offs, ctr = 0, None, None
        if with_cells and "cell_offsets" in source:
            offs = np.ascontiguousarray(source["cell_offsets"], dtype=np.int64)
            ctr = _f64(source["cell_centers"]).reshape(-1, dim)
            ncells = ctr.shape[0]
            keep += [offs, ctr]
        p0 = None
        if psi0 is not None:
            p0 = _f64(psi0)
            keep.append(p0)
        req = _lib.Request(dim, x.shape[0], x.ctypes.data, jxw.ctypes.data, dens.ctypes.data, ncells,
                           offs.ctypes.data if offs is not None else None,
                           ctr.ctypes.data if ctr is not None else None, y.shape[0], y.ctypes.data, nu.ctypes.data,
                           p0.ctypes.data if p0 is not None else None, SotSolver._cparams(params),
                           _lib.METHOD[method], _lib.PRECISION[precision], _lib.HESSIAN_METHOD[hessian],
                           float(epsilon_scaling_factor), int(epsilon_scaling_steps), float(intermediate_tolerance))
        t = C.c_int64(0)
        self._check(self._L.sdot_server_submit(self._h, C.byref(req), C.byref(t)))
        self._sizes[t.value] = y.shape[0]
        return t.value

    def done(self, ticket: int) -> bool:
        return self._L.sdot_server_poll(self._h, int(ticket)) == 1

    def wait(self, ticket: int, timeout: float = 0.0, raise_on_error: bool = True):
        n = self._sizes.pop(int(ticket))
        psi = np.empty(n)
        r = _lib.Result()
        st = self._L.sdot_server_wait(self._h, int(ticket), float(timeout), psi.ctypes.data, C.byref(r))
        names = {v: k for k, v in _lib.METHOD.items()}
        res = {"status": _lib.STATUS_NAMES.get(r.status, r.status), "converged": bool(r.converged),
               "method": names.get(r.method, r.method), "iterations": r.iterations,
               "n_evaluations": r.n_evaluations, "last_value": r.last_value,
               "last_check_value": r.last_check_value, "queue_ms": r.queue_ms, "run_ms": r.run_ms,
               "latency_ms": r.latency_ms, "slot": r.slot, "message": r.message.decode(errors="replace")}
        if st == _lib.SDOT_ETIMEOUT:
            self._sizes[int(ticket)] = n
            raise TimeoutError(f"ticket {ticket} not done")
        if st != _lib.SDOT_OK and raise_on_error:
            raise _lib.SdotError(st, res["message"])
        return psi, res

    def stats(self) -> dict:
        s = _lib.ServerStats()
        self._check(self._L.sdot_server_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _lib.ServerStats._fields_}

    def reset_stats(self):
        self._check(self._L.sdot_server_reset_stats(self._h))
