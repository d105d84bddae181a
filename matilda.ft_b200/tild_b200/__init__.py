"""Python binding of the B200-native TILD particle-mesh library (libtild_b200.so).

A thin ctypes layer over the C ABI in include/tild_b200.h.  The compute path is the
CUDA library; there is no Python or CPU fallback: importing this module loads the
in-tree ``lib/libtild_b200.so`` and raises if it is missing.

``Box`` mirrors MATILDA.FT's PS_Box surface: feed it the same ``box ps ... endBox``
script lines (PS_Box::readInput), then ``run_nvt`` (PS_Box::NVT), ``forces``
(PS_Box::forces), ``thermo`` (PS_Box::computeThermoProps).
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libtild_b200.so")

TILD_OK = 0
NOALLOC_SCRATCH_BYTES = 16 << 20   # TILD_NOALLOC_SCRATCH_BYTES of the C header
STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_PARSE", 3: "ERR_IO", 4: "ERR_CUDA", 5: "ERR_STATE",
          6: "ERR_UNSUPPORTED", 7: "ERR_DEVICE"}

# Every entry point of include/tild_b200.h with its ctypes signature.
_SIGS = {
    "tild_version": ([], ctypes.c_char_p),
    "tild_last_error": ([], ctypes.c_char_p),
    "tild_box_create": ([ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "tild_box_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "tild_box_set_stream": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_set_base_dir": ([ctypes.c_void_p, ctypes.c_char_p], ctypes.c_int),
    "tild_box_command": ([ctypes.c_void_p, ctypes.c_char_p], ctypes.c_int),
    "tild_box_read_input": ([ctypes.c_void_p, ctypes.c_char_p], ctypes.c_int),
    "tild_box_set_particles": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_set_bonds": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_set_angles": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_set_option": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64], ctypes.c_int),
    "tild_box_describe": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)],
                          ctypes.c_int),
    "tild_box_get_info": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_run_nvt": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "tild_box_step": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "tild_box_forces": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_thermo": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)],
                        ctypes.c_int),
    "tild_box_get_positions": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_set_positions": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_get_density": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
    "tild_box_modify": ([ctypes.c_void_p, ctypes.c_char_p], ctypes.c_int),
    "tild_box_get_grid_force": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_get_density_noalloc": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p],
                                     ctypes.c_int),
    "tild_box_grid_weights": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_structure_factor": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int32, ctypes.c_double,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_box_get_log": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64),
                          ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "tild_run_script_file": ([ctypes.c_char_p, ctypes.c_int], ctypes.c_int),
    "tild_box_stage_times": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)],
                             ctypes.c_int),
    "tild_pool_create": ([ctypes.c_int, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)],
                         ctypes.c_int),
    "tild_pool_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "tild_pool_submit": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)],
                         ctypes.c_int),
    "tild_pool_status": ([ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32),
                          ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p], ctypes.c_int),
    "tild_pool_wait": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "tild_pool_result": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                          ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "tild_pool_release": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "tild_pool_cancel": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "tild_pool_set_budget": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "tild_pool_stats": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
    "tild_batch_create": ([ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "tild_batch_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "tild_batch_add": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "tild_batch_size": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "tild_batch_step": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "tild_batch_set_streams": ([ctypes.c_void_p, ctypes.c_int32], ctypes.c_int),
}


class TildError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "?"), code, msg))
        self.code = code


class BoxInfo(ctypes.Structure):
    _fields_ = [("nstot", ctypes.c_int64), ("dim", ctypes.c_int32), ("nx", ctypes.c_int32 * 3),
                ("L", ctypes.c_float * 3), ("pmeorder", ctypes.c_int32), ("n_groups", ctypes.c_int32),
                ("n_potentials", ctypes.c_int32), ("n_density_fields", ctypes.c_int32),
                ("n_force_groups", ctypes.c_int32), ("n_bond_types", ctypes.c_int32),
                ("n_bonds", ctypes.c_int64), ("step", ctypes.c_int64), ("device_bytes", ctypes.c_int64)]


_lib = None


def lib():
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libtild_b200.so is not built (run `make -C matilda.ft_b200`): " + LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(rc):
    if rc != TILD_OK:
        raise TildError(rc, lib().tild_last_error().decode())


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Box:
    """One PS box on one GPU (PS_Box, PS_Box.h:19-212)."""

    def __init__(self, device=0, base_dir=None, options=None):
        h = ctypes.c_void_p()
        _check(lib().tild_box_create(int(device), ctypes.byref(h)))
        self._h = h
        if base_dir:
            _check(lib().tild_box_set_base_dir(self._h, base_dir.encode()))
        for k, v in (options or {}).items():
            self.set_option(k, v)

    def close(self):
        if getattr(self, "_h", None):
            _check(lib().tild_box_destroy(self._h))   # refused while the box belongs to a batch
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- input -------------------------------------------------------------------
    def command(self, line: str):
        _check(lib().tild_box_command(self._h, line.encode()))

    def read_input(self, text: str):
        _check(lib().tild_box_read_input(self._h, text.encode()))

    def set_option(self, key: str, value: int):
        _check(lib().tild_box_set_option(self._h, key.encode(), int(value)))

    def set_stream(self, stream_handle: int):
        _check(lib().tild_box_set_stream(self._h, ctypes.c_void_p(stream_handle)))

    def set_particles(self, x, types, mol=None, q=None):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(types, np.int32)
        m = None if mol is None else np.ascontiguousarray(mol, np.int32)
        qq = None if q is None else np.ascontiguousarray(q, np.float32)
        _check(lib().tild_box_set_particles(self._h, len(t), _ptr(x), _ptr(t), _ptr(m), _ptr(qq)))

    def set_bonds(self, pairs, btype=None):
        p = np.ascontiguousarray(pairs, np.int64).reshape(-1, 2)
        b = None if btype is None else np.ascontiguousarray(btype, np.int32)
        _check(lib().tild_box_set_bonds(self._h, len(p), _ptr(p), _ptr(b)))

    def set_angles(self, triples, atype=None):
        t = np.ascontiguousarray(triples, np.int64).reshape(-1, 3)
        a = None if atype is None else np.ascontiguousarray(atype, np.int32)
        _check(lib().tild_box_set_angles(self._h, len(t), _ptr(t), _ptr(a)))

    # -- queries -------------------------------------------------------------------
    def describe(self) -> dict:
        need = ctypes.c_int64()
        _check(lib().tild_box_describe(self._h, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(need.value)
        _check(lib().tild_box_describe(self._h, buf, need.value, None))
        return json.loads(buf.value.decode())

    def info(self) -> BoxInfo:
        out = BoxInfo()
        _check(lib().tild_box_get_info(self._h, ctypes.byref(out)))
        return out

    @property
    def N(self):
        return int(self.info().nstot)

    # -- run -----------------------------------------------------------------------
    def run_nvt(self, nsteps: int):
        _check(lib().tild_box_run_nvt(self._h, int(nsteps)))

    def step(self, nsteps: int = 1):
        _check(lib().tild_box_step(self._h, int(nsteps)))

    def forces(self):
        f = np.zeros((self.N, int(self.info().dim)), np.float32)
        _check(lib().tild_box_forces(self._h, _ptr(f)))
        return f

    def thermo_raw(self):
        """tild_box_thermo's values as one array: Upe, Ubond, per potential, virial[6]."""
        out = np.zeros(64, np.float64)
        n = ctypes.c_int()
        _check(lib().tild_box_thermo(self._h, _ptr(out), 64, ctypes.byref(n)))
        return out[: n.value].copy()

    def thermo(self):
        nmax = 64
        out = np.zeros(nmax, np.float64)
        n = ctypes.c_int()
        _check(lib().tild_box_thermo(self._h, _ptr(out), nmax, ctypes.byref(n)))
        npot = self.info().n_potentials
        v = out[: n.value]
        return dict(Upe=float(v[0]), Ubond=float(v[1]), potentials=[float(e) for e in v[2:2 + npot]],
                    virial=v[2 + npot:2 + npot + 6].copy(), pair_virial=v[8 + npot:14 + npot].copy(),
                    pressure=v[14 + npot:20 + npot].copy(), Uangle=float(v[20 + npot]))

    def positions(self):
        x = np.zeros((self.N, int(self.info().dim)), np.float32)
        _check(lib().tild_box_get_positions(self._h, _ptr(x)))
        return x

    def set_positions(self, x):
        x = np.ascontiguousarray(x, np.float32)
        _check(lib().tild_box_set_positions(self._h, _ptr(x)))

    def density(self, group: str, charge=False):
        i = self.info()
        rho = np.zeros(int(i.nx[0]) * int(i.nx[1]) * int(i.nx[2]), np.float32)
        _check(lib().tild_box_get_density(self._h, group.encode(), int(bool(charge)), _ptr(rho)))
        return rho

    def modify(self, rest: str):
        """A top-level `modify` line (without the word), e.g. "potential remove 1"."""
        _check(lib().tild_box_modify(self._h, rest.encode()))

    def grid_force(self, group: str):
        """PS_Group::d_gridForce of the last force evaluation, shape (M, Dim), x fastest."""
        i = self.info()
        D = int(i.dim)
        gf = np.zeros((int(i.nx[0]) * int(i.nx[1]) * int(i.nx[2]), D), np.float32)
        _check(lib().tild_box_get_grid_force(self._h, group.encode(), _ptr(gf)))
        return gf

    def density_noalloc(self, group: str, charge=False):
        """density() through the allocation-free entry point (static device scratch)."""
        i = self.info()
        rho = np.zeros(int(i.nx[0]) * int(i.nx[1]) * int(i.nx[2]), np.float32)
        _check(lib().tild_box_get_density_noalloc(self._h, group.encode(), int(bool(charge)), _ptr(rho)))
        return rho

    def structure_factor(self, group: str, nbins: int, kmax: float, charge=False):
        """(k, S(k), count) in nbins shells of |k| up to kmax (FP64)."""
        k, sk, n = (np.zeros(int(nbins), np.float64) for _ in range(3))
        _check(lib().tild_box_structure_factor(self._h, group.encode(), int(bool(charge)), int(nbins), float(kmax),
                                               _ptr(k), _ptr(sk), _ptr(n)))
        return k, sk, n

    def grid_weights(self):
        i = self.info()
        G = (i.pmeorder + 1) ** int(i.dim)
        inds = np.zeros((self.N, G), np.int32)
        w = np.zeros((self.N, G), np.float32)
        _check(lib().tild_box_grid_weights(self._h, _ptr(inds), _ptr(w)))
        return inds, w

    def log(self):
        rows, cols = ctypes.c_int64(), ctypes.c_int32()
        _check(lib().tild_box_get_log(self._h, None, ctypes.byref(rows), ctypes.byref(cols)))
        out = np.zeros((rows.value, cols.value), np.float64)
        _check(lib().tild_box_get_log(self._h, _ptr(out), None, None))
        return out


def run_script_file(path: str, device: int = 0):
    """Execute a MATILDA.FT input script (main.cu:21-156) with the B200 library."""
    _check(lib().tild_run_script_file(path.encode(), int(device)))


JOB_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


class Batch:
    """Replicas stepped together (tild_batch_*): every stage of a step is one kernel launch
    over all replicas, and a step's launches are one CUDA graph.  The boxes stay the
    caller's (read them as usual); close the batch before closing its boxes."""

    def __init__(self, device=0, streams=1):
        h = ctypes.c_void_p()
        _check(lib().tild_batch_create(int(device), ctypes.byref(h)))
        self._h = h
        self._boxes = []
        if streams != 1:
            _check(lib().tild_batch_set_streams(self._h, int(streams)))

    def add(self, box: "Box"):
        """Add a box whose endBox has been processed."""
        _check(lib().tild_batch_add(self._h, box._h))
        self._boxes.append(box)

    def step(self, n: int):
        """n steps of every replica."""
        _check(lib().tild_batch_step(self._h, int(n)))

    def __len__(self):
        n = ctypes.c_int32()
        _check(lib().tild_batch_size(self._h, ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            lib().tild_batch_destroy(self._h)
            self._h = None
            self._boxes = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Pool:
    """Jobs sharing one GPU (tild_pool_*): admission against a device-memory budget and
    continuous batching of their steps on per-job streams."""

    def __init__(self, device=0, mem_budget_bytes=16 << 30, max_active=0):
        h = ctypes.c_void_p()
        _check(lib().tild_pool_create(int(device), int(mem_budget_bytes), int(max_active), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().tild_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, box: Box, nsteps: int) -> int:
        """Hand a box (endBox not yet processed) to the pool; returns the job id.  On
        success the box handle is emptied (the pool owns the box)."""
        jid = ctypes.c_int64()
        _check(lib().tild_pool_submit(self._h, box._h, int(nsteps), ctypes.byref(jid)))
        return jid.value

    def status(self, job: int):
        st, done = ctypes.c_int32(), ctypes.c_int64()
        t = np.zeros(3, np.float64)
        _check(lib().tild_pool_status(self._h, int(job), ctypes.byref(st), ctypes.byref(done), _ptr(t)))
        return {"state": JOB_STATES[st.value], "steps_done": done.value,
                "submit_s": t[0], "admit_s": t[1], "done_s": t[2]}

    def wait(self, job: int):
        _check(lib().tild_pool_wait(self._h, int(job)))

    def result(self, job: int, n: int, dim: int = 3):
        x = np.zeros((n, dim), np.float32)
        th = np.zeros(64, np.float64)
        nw = ctypes.c_int32()
        _check(lib().tild_pool_result(self._h, int(job), _ptr(x), _ptr(th), 64, ctypes.byref(nw)))
        return x, th[: nw.value]

    def release(self, job: int):
        _check(lib().tild_pool_release(self._h, int(job)))

    def cancel(self, job: int):
        """Cancel a queued or running job (running: its in-flight chunks finish first)."""
        _check(lib().tild_pool_cancel(self._h, int(job)))

    def set_budget(self, mem_budget_bytes: int):
        """New memory budget for admissions from now on."""
        _check(lib().tild_pool_set_budget(self._h, int(mem_budget_bytes)))

    def stats(self) -> dict:
        v = np.zeros(7, np.int64)
        _check(lib().tild_pool_stats(self._h, _ptr(v), 7))
        return dict(zip(("queued", "running", "done", "failed", "bytes_in_use", "budget", "cancelled"),
                        (int(a) for a in v)))


def box_from_spec(spec, device=0, options=None, steps_script=False, base_dir=None):
    """Build a Box directly from a synth.SystemSpec (arrays instead of readData); output
    files (when the write_files option is on) go to base_dir."""
    b = Box(device, base_dir=base_dir, options=options)
    D = spec.dim
    b.command("Dim %d" % D)
    b.command("boxLengths " + " ".join("%.9g" % v for v in spec.L[:D]))
    b.command("grid " + " ".join(str(int(v)) for v in spec.grid[:D]))
    b.command("pmeorder %d" % spec.order)
    b.command("randSeed %d" % spec.seed)
    if spec.charges is not None:
        b.command("doCharges")
    if getattr(spec, "max_bonds", None):
        b.command("MAXBONDS %d" % spec.max_bonds)
    for t, lb in enumerate(spec.species):
        b.command("species %s mass %.9g mobility %.9g" % (lb, spec.masses[t], spec.mobility[t]))
    b.set_particles(spec.x, spec.types, spec.mol, spec.charges)
    if len(spec.bonds):
        b.command(spec.bond_command())
        b.set_bonds(spec.bonds)
    for line in spec.angle_commands():
        b.command(line)
    if len(spec.angles):
        b.set_angles(spec.angles, spec.angle_types)
    from . import synth
    for p in spec.potentials:
        b.command(synth.potential_command(p))
    b.command("integrator all %s delt %.9g" % (spec.integrator, spec.delt))
    b.command("logFreq %d" % spec.log_freq)
    return b
