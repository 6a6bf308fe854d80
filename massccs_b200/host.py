"""ctypes binding of libmassccs_host.so (include/massccs_host.h).

The reference's set-up (input.json, force field, target file, orientation,
ellipsoid, pre-draw) and reduction, as the product's host library implements
them, plus `run()`: the whole reference run with the trajectory loop on the
GPU engine.
"""
import ctypes
import os

import numpy as np

from . import engine as E

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libmassccs_host.so")

EXPORTS = ["mh_open", "mh_close", "mh_get_info", "mh_get_target", "mh_fill_params", "mh_predraw",
           "mh_reduce", "mh_run", "mh_run_devices", "mh_get_devices"]


class MhInfo(ctypes.Structure):
    _fields_ = [
        ("gas_flag", ctypes.c_int32), ("force_type", ctypes.c_int32), ("natoms", ctypes.c_int32),
        ("gas_natoms", ctypes.c_int32),
        ("nprobe", ctypes.c_uint32), ("niter", ctypes.c_uint32), ("seed", ctypes.c_uint32),
        ("nthreads", ctypes.c_uint32),
        ("short_range_cutoff", ctypes.c_int32), ("long_range_flag", ctypes.c_int32),
        ("long_range_cutoff", ctypes.c_int32), ("polarizability_flag", ctypes.c_int32),
        ("equipotential_flag", ctypes.c_int32), ("user_ff_flag", ctypes.c_int32),
        ("dt", ctypes.c_double), ("temperature", ctypes.c_double), ("skin", ctypes.c_double),
        ("lj_cutoff", ctypes.c_double), ("coul_cutoff", ctypes.c_double), ("alpha", ctypes.c_double),
        ("mu", ctypes.c_double), ("target_mass", ctypes.c_double), ("target_charge", ctypes.c_double),
        ("gas_mass", ctypes.c_double), ("gas_inertia", ctypes.c_double), ("d_bond", ctypes.c_double),
        ("a", ctypes.c_double), ("b", ctypes.c_double), ("c", ctypes.c_double), ("bmax", ctypes.c_double),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("Nz", ctypes.c_int32), ("Ncells", ctypes.c_int32),
        ("cell_size", ctypes.c_double),
        ("max_x", ctypes.c_double), ("max_y", ctypes.c_double), ("max_z", ctypes.c_double),
        ("radius", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_LIB = None


def load_library():
    global _LIB
    if _LIB is None:
        E.load_library()  # the host library links the engine
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"massccs_b200: host library missing at {LIB_PATH}; "
                               "build it with `python -m massccs_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        L.mh_open.argtypes = [ctypes.POINTER(vp), ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, sz]
        L.mh_close.argtypes = [vp]
        L.mh_close.restype = None
        L.mh_get_info.argtypes = [vp, ctypes.POINTER(MhInfo)]
        L.mh_get_target.argtypes = [vp] + [vp] * 9
        L.mh_fill_params.argtypes = [vp, ctypes.POINTER(E.CcsParams)]
        L.mh_predraw.argtypes = [vp, ctypes.c_uint32, sz, vp]
        L.mh_reduce.argtypes = [sz, sz, vp, vp, ctypes.c_double, vp, vp, vp, vp, vp, vp]
        L.mh_run.argtypes = [vp, ctypes.c_int, ctypes.POINTER(E.CcsParams), ctypes.c_int, vp, vp, vp]
        L.mh_run_devices.argtypes = [vp, ctypes.c_size_t, vp, ctypes.POINTER(E.CcsParams), ctypes.c_int, vp, vp, vp]
        L.mh_get_devices.argtypes = [vp, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class System:
    """The reference's System set-up for one input.json (System.cpp:19-144)."""

    def __init__(self, input_json, print_report=False):
        self._L = load_library()
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self._L.mh_open(ctypes.byref(h), os.fspath(input_json).encode(), int(print_report), err, 512)
        if rc != 0:
            raise E.CcsError("mh_open: " + err.value.decode())
        self._h = h
        info = MhInfo()
        self._L.mh_get_info(h, ctypes.byref(info))
        self.info = info.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            self._L.mh_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def target(self):
        n = self.info["natoms"]
        keys = ("x", "y", "z", "q", "m", "eps", "sig", "eps_c", "sig_c")
        arrs = {k: np.empty(n) for k in keys}
        self._L.mh_get_target(self._h, *[_p(arrs[k]) for k in keys])
        return arrs

    def params(self, **overrides):
        p = E.CcsParams()
        self._L.mh_fill_params(self._h, ctypes.byref(p))
        for k, v in overrides.items():
            setattr(p, k, v)
        return p

    def predraw(self, ntraj=None, seed=None):
        n = ntraj if ntraj is not None else self.info["nprobe"] * self.info["niter"]
        rnd = np.empty((9, n))
        self._L.mh_predraw(self._h, self.info["seed"] if seed is None else seed, n, _p(rnd))
        return rnd

    def engine(self, device=0, **overrides):
        """An Engine set up with this system's parameters and target."""
        eng = E.Engine(device)
        eng.set_params(self.params(**overrides))
        t = self.target()
        co2 = self.info["gas_flag"] == 3
        eng.set_target(t["x"], t["y"], t["z"], t["q"], t["eps"], t["sig"],
                       t["eps_c"] if co2 else None, t["sig_c"] if co2 else None)
        return eng

    def run(self, device=0, print_report=False, **overrides):
        """The whole run (pre-draw, GPU trajectories, reduction) -> (ccs, err, seconds)."""
        p = self.params(**overrides)
        ccs, err, secs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        rc = self._L.mh_run(self._h, device, ctypes.byref(p), int(print_report), ctypes.byref(ccs),
                            ctypes.byref(err), ctypes.byref(secs))
        if rc != 0:
            raise E.CcsError(f"mh_run failed: {rc}")
        return ccs.value, err.value, secs.value

    def run_devices(self, devices, print_report=False, **overrides):
        """The whole run as one job split over the given GPUs -> (ccs, err, seconds)."""
        p = self.params(**overrides)
        devs = (ctypes.c_int * len(devices))(*devices)
        ccs, err, secs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        rc = self._L.mh_run_devices(self._h, len(devices), devs, ctypes.byref(p), int(print_report),
                                    ctypes.byref(ccs), ctypes.byref(err), ctypes.byref(secs))
        if rc != 0:
            raise E.CcsError(f"mh_run_devices failed: {rc}")
        return ccs.value, err.value, secs.value

    def devices(self):
        """The GPUs named by input.json's "devices" key ([] when absent)."""
        buf = (ctypes.c_int * 64)()
        n = ctypes.c_size_t()
        self._L.mh_get_devices(self._h, buf, 64, ctypes.byref(n))
        return list(buf[:min(n.value, 64)])


def reduce(niter, nprobe, status, omc, bmax):
    """Per-iteration reduction of the reference (System.cpp:287-321)."""
    L = load_library()
    omega = np.empty(niter)
    nf, ns, nl = (np.empty(niter, dtype=np.int32) for _ in range(3))
    ccs, err = ctypes.c_double(), ctypes.c_double()
    st = np.ascontiguousarray(status, dtype=np.int8)
    om = np.ascontiguousarray(omc, dtype=np.float64)
    rc = L.mh_reduce(niter, nprobe, _p(st), _p(om), float(bmax), _p(omega), _p(nf), _p(ns), _p(nl),
                     ctypes.byref(ccs), ctypes.byref(err))
    if rc != 0:
        raise E.CcsError("mh_reduce failed")
    return {"omega": omega, "nfree": nf, "nscatter": ns, "nlost": nl, "ccs": ccs.value, "err": err.value}
