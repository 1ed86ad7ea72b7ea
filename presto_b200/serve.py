"""Batched and served accelsearch: Python mirror of the ab_pool C ABI.

A SearchPool holds nworkers engine contexts on one GPU; submit() queues a
spectrum with its accelsearch options and returns a ticket, wait() returns
(candidates, latency_ms).  search_batch() runs many spectra (uneven lengths,
mixed zmax/wmax/numharm) through the pool and returns their candidate lists
in input order.
"""
import ctypes as C

import numpy as np

from .accel import ERRORS, AccelError, Cand, lib, make_params


class SearchPool:
    def __init__(self, device=0, nworkers=4, hbm_budget=0):
        self.L = lib()
        self.ptr = C.c_void_p()
        rc = self.L.ab_pool_create(int(device), int(nworkers), int(hbm_budget), C.byref(self.ptr))
        if rc:
            raise AccelError(f"ab_pool_create: {ERRORS.get(rc, rc)}")
        self.nworkers = nworkers

    def set_corr_path(self, path):
        """accel.CORR_FFT or accel.CORR_TC_SPLIT_BF16 for every worker (before
        any submit)."""
        self._check(self.L.ab_pool_set_corr_path(self.ptr, int(path)), "ab_pool_set_corr_path")

    def _check(self, rc, what):
        if rc:
            msg = self.L.ab_pool_last_error(self.ptr)
            raise AccelError(f"{what}: {ERRORS.get(rc, rc)}: {msg.decode() if msg else ''}")

    def submit(self, fft, N, dt, **opts):
        fft = np.ascontiguousarray(fft, dtype=np.complex64)
        p = make_params(N, dt, fft.size, **opts)
        t = C.c_longlong()
        self._check(self.L.ab_pool_submit(self.ptr, C.byref(p), fft.ctypes.data, C.byref(t)),
                    "ab_pool_submit")
        return t.value

    def wait(self, ticket):
        n = C.c_longlong()
        lat = C.c_double()
        self._check(self.L.ab_pool_wait(self.ptr, ticket, None, 0, C.byref(n), C.byref(lat)),
                    "ab_pool_wait")
        arr = (Cand * max(n.value, 1))()
        self._check(self.L.ab_pool_wait(self.ptr, ticket, arr, n.value, C.byref(n), C.byref(lat)),
                    "ab_pool_wait")
        return [(c.power, c.sigma, c.numharm, c.r, c.z, c.w) for c in arr[:n.value]], lat.value

    def search_batch(self, ffts, N_list, dt, opts_list=None):
        opts_list = opts_list or [{}] * len(ffts)
        tickets = [self.submit(f, n, dt, **o) for f, n, o in zip(ffts, N_list, opts_list)]
        return [self.wait(t)[0] for t in tickets]

    def stats(self):
        n = C.c_longlong()
        p50, p99, busy = C.c_double(), C.c_double(), C.c_double()
        self.L.ab_pool_stats(self.ptr, C.byref(n), C.byref(p50), C.byref(p99), C.byref(busy))
        return dict(completed=n.value, p50_ms=p50.value, p99_ms=p99.value, busy_ms=busy.value)

    def reset_stats(self):
        self.L.ab_pool_reset_stats(self.ptr)

    def close(self):
        if self.ptr:
            self.L.ab_pool_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
