"""ctypes binding of the FP64 oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may import
this module; the product path never does.  See ccs_oracle.h for the C API and
the reference file:line each function restates.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("gas_flag", ctypes.c_int), ("force_type", ctypes.c_int), ("natoms", ctypes.c_int),
        ("gas_natoms", ctypes.c_int),
        ("nprobe", ctypes.c_uint), ("niter", ctypes.c_uint), ("seed", ctypes.c_uint),
        ("nthreads", ctypes.c_uint),
        ("short_range_cutoff", ctypes.c_int), ("long_range_flag", ctypes.c_int),
        ("long_range_cutoff", ctypes.c_int), ("polarizability_flag", ctypes.c_int),
        ("equipotential_flag", ctypes.c_int), ("user_ff_flag", ctypes.c_int),
        ("dt", ctypes.c_double), ("temperature", ctypes.c_double), ("skin", ctypes.c_double),
        ("lj_cutoff", ctypes.c_double), ("coul_cutoff", ctypes.c_double),
        ("alpha", ctypes.c_double),
        ("mu", ctypes.c_double), ("target_mass", ctypes.c_double),
        ("target_charge", ctypes.c_double), ("gas_mass", ctypes.c_double),
        ("gas_inertia", ctypes.c_double), ("d_bond", ctypes.c_double),
        ("a", ctypes.c_double), ("b", ctypes.c_double), ("c", ctypes.c_double),
        ("bmax", ctypes.c_double),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int), ("Ncells", ctypes.c_int),
        ("cell_size", ctypes.c_double),
        ("max_x", ctypes.c_double), ("max_y", ctypes.c_double), ("max_z", ctypes.c_double),
        ("radius", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


QUIRK_CO2_VCM = 1


def build():
    """Compile liboracle.so with its Makefile (gcc is in the image)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        d, i, vp = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        L.orc_open.restype = vp
        L.orc_open.argtypes = [ctypes.c_char_p, i, ctypes.c_char_p, i]
        L.orc_close.argtypes = [vp]
        L.orc_get_params.argtypes = [vp, P(OrcParams)]
        L.orc_get_target.argtypes = [vp] + [vp] * 9
        L.orc_predraw.argtypes = [vp, ctypes.c_uint, ctypes.c_size_t, vp]
        L.orc_mt19937.argtypes = [ctypes.c_uint, ctypes.c_size_t, vp]
        L.orc_run.argtypes = [vp, ctypes.c_size_t, vp, ctypes.c_size_t, i, i, vp, vp, vp, vp]
        L.orc_setup_one.restype = i
        L.orc_setup_one.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orc_vel_generator.restype = d
        L.orc_vel_generator.argtypes = [vp, d]
        L.orc_site_force.restype = i
        L.orc_site_force.argtypes = [vp, i, vp, vp, vp, vp]
        L.orc_reduce.argtypes = [ctypes.c_size_t, ctypes.c_size_t, vp, vp, d, vp, vp, vp, vp, vp, vp]
        L.orc_run_system.restype = i
        L.orc_run_system.argtypes = [vp, i, i, i, vp, vp]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def mt19937(seed, n):
    out = np.empty(n, dtype=np.uint32)
    lib().orc_mt19937(seed, n, _p(out))
    return out


class OracleSystem:
    """The reference's System set-up (System.cpp:19-144) built by the oracle."""

    def __init__(self, json_path, print_report=False):
        err = ctypes.create_string_buffer(512)
        h = lib().orc_open(json_path.encode(), int(print_report), err, 512)
        if not h:
            raise RuntimeError("oracle: " + err.value.decode())
        self._h = h
        p = OrcParams()
        lib().orc_get_params(h, ctypes.byref(p))
        self.params = p.as_dict()

    def close(self):
        if self._h:
            lib().orc_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def target(self):
        n = self.params["natoms"]
        arrs = {k: np.empty(n) for k in ("x", "y", "z", "q", "m", "eps", "sig", "eps_c", "sig_c")}
        lib().orc_get_target(self._h, *[_p(arrs[k]) for k in
                                         ("x", "y", "z", "q", "m", "eps", "sig", "eps_c", "sig_c")])
        return arrs

    def predraw(self, ntraj, seed=None):
        rnd = np.empty((9, ntraj))
        lib().orc_predraw(self._h, self.params["seed"] if seed is None else seed, ntraj, _p(rnd))
        return rnd

    def run(self, rnd, quirks=0, nthreads=0):
        rnd = np.ascontiguousarray(rnd, dtype=np.float64)
        n = rnd.shape[1]
        status = np.empty(n, dtype=np.int8)
        omc = np.empty(n)
        steps = np.empty(n, dtype=np.uint32)
        visits = np.empty(n, dtype=np.uint64)
        lib().orc_run(self._h, n, _p(rnd), n, quirks, nthreads, _p(status), _p(omc), _p(steps),
                      _p(visits))
        return {"status": status, "one_minus_cos": omc, "steps": steps, "visits": visits}

    def setup_one(self, u9):
        u = np.ascontiguousarray(u9, dtype=np.float64)
        pos, vel, rcm, vcm = np.zeros(9), np.zeros(9), np.zeros(3), np.zeros(3)
        hit = lib().orc_setup_one(self._h, _p(u), _p(pos), _p(vel), _p(rcm), _p(vcm))
        return hit, pos.reshape(3, 3), vel.reshape(3, 3), rcm, vcm

    def vel_generator(self, u):
        return lib().orc_vel_generator(self._h, float(u))

    def site_force(self, iatom, pos):
        p = np.ascontiguousarray(pos, dtype=np.float64)
        f = np.zeros(3)
        U = ctypes.c_double(0.0)
        vis = ctypes.c_uint64(0)
        rc = lib().orc_site_force(self._h, iatom, _p(p), _p(f), ctypes.byref(U), ctypes.byref(vis))
        if rc:
            raise ValueError("bad site")
        return f, U.value, vis.value

    def run_system(self, nthreads=0, quirks=0, print_report=False):
        ccs, err = ctypes.c_double(), ctypes.c_double()
        lib().orc_run_system(self._h, nthreads, quirks, int(print_report), ctypes.byref(ccs),
                             ctypes.byref(err))
        return ccs.value, err.value


def reduce(niter, nprobe, status, omc, bmax):
    omega = np.empty(niter)
    nf = np.empty(niter, dtype=np.int32)
    ns = np.empty(niter, dtype=np.int32)
    nl = np.empty(niter, dtype=np.int32)
    ccs, err = ctypes.c_double(), ctypes.c_double()
    st = np.ascontiguousarray(status, dtype=np.int8)
    om = np.ascontiguousarray(omc, dtype=np.float64)
    lib().orc_reduce(niter, nprobe, _p(st), _p(om), float(bmax), _p(omega), _p(nf), _p(ns), _p(nl),
                     ctypes.byref(ccs), ctypes.byref(err))
    return {"omega": omega, "nfree": nf, "nscatter": ns, "nlost": nl, "ccs": ccs.value,
            "err": err.value}
