"""ctypes binding of the CPU restatement oracle (oracle/_port/liboracle.so). Test infrastructure."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_port", "liboracle.so")
DATA = os.path.join(ROOT, "exaca_b200", "data")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(ROOT, "oracle", "exaca_oracle.cpp")):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True, capture_output=True)
        L = ctypes.CDLL(LIB)
        L.oracle_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_error.restype = ctypes.c_char_p
        L.oracle_free.argtypes = [ctypes.c_void_p]
        L.oracle_geometry.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]
        L.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        L.oracle_run_to.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_census.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
        L.oracle_cycle.argtypes = [ctypes.c_void_p]
        L.oracle_fields.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
        _lib = L
    return _lib


class Oracle:
    def __init__(self, input_file):
        self.h = lib().oracle_create(os.fsencode(input_file), os.fsencode(DATA))
        if not self.h:
            raise RuntimeError(lib().oracle_error().decode())
        g = (ctypes.c_longlong * 6)()
        lib().oracle_geometry(self.h, g)
        self.mx, self.my, self.nz, self.nz_active, self.n, self.na = list(g)

    def step(self, n):
        lib().oracle_step(self.h, n)

    def run(self):
        c = ctypes.c_int()
        lib().oracle_run(self.h, ctypes.byref(c))
        return c.value

    def run_to(self, stop_cycle):
        """The layer loop of run(), paused after cycle stop_cycle; True if it paused there."""
        c = ctypes.c_int()
        return lib().oracle_run_to(self.h, stop_cycle, ctypes.byref(c)) == 1

    @staticmethod
    def set_threads(n):
        """Host threads of CellCapture's dense first pass (the results do not depend on it)."""
        lib().oracle_set_threads(n)

    def census_lines(self):
        """The stdout lines the reference prints at the censuses run so far (src/CAupdate.cpp:776-780, 815)."""
        n = lib().oracle_census(self.h, None, 0)
        buf = (ctypes.c_longlong * (6 * max(n, 1)))()
        lib().oracle_census(self.h, buf, n)
        out = []
        for q in range(n):
            cyc, sh, uc, nn, rem, jump = buf[6 * q: 6 * q + 6]
            out.append(f"cycle = {cyc} Superheated liquid cells = {sh} Undercooled liquid cells = {uc} "
                       f"Number of nucleation events this layer {nn} Remaining liquid cells in future layers of "
                       f"this simulation = {rem}")
            if jump:
                out.append(f"Jumping to cycle {jump}")
        return out

    @property
    def cycle(self):
        return lib().oracle_cycle(self.h)

    def fields(self):
        """Cell fields, and the octahedron arrays of the current layer's active window."""
        g = (ctypes.c_longlong * 6)()
        lib().oracle_geometry(self.h, g)
        self.nz_active, self.na = int(g[3]), int(g[5])
        ct = np.empty(self.n, np.int32)
        gid = np.empty(self.n, np.int32)
        dl = np.empty(self.na, np.float32)
        doc = np.empty(3 * self.na, np.float32)
        cdl = np.empty(26 * self.na, np.float32)
        lib().oracle_fields(self.h, *(a.ctypes.data_as(ctypes.c_void_p) for a in (ct, gid, dl, doc, cdl)))
        return dict(cell_type=ct, grain_id=gid, dl=dl, doc=doc, cdl=cdl)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_free(self.h)
            self.h = None
