"""ctypes binding of libmassccs_gpu.so (include/massccs_gpu.h).

The Python face of the drop-in boundary: the same entry points a C/C++ host
binds, with numpy arrays for the host buffers.  Loading fails loudly when the
CUDA library is missing -- there is no CPU fallback in the product path.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libmassccs_gpu.so")

GAS = {"He": 1, "N2": 2, "CO2": 3, "Ar": 4, "co2": 5}
PREC_FP32, PREC_FP64 = 0, 1
QUIRK_CO2_VCM = 1
STATUS_FREE, STATUS_SCATTER, STATUS_LOST, STATUS_CAPPED = 0, 1, 2, 3


class CcsParams(ctypes.Structure):
    _fields_ = [
        ("gas", ctypes.c_int32), ("force_type", ctypes.c_int32),
        ("dt", ctypes.c_double), ("temperature", ctypes.c_double), ("mu", ctypes.c_double),
        ("gas_inertia", ctypes.c_double), ("d_bond", ctypes.c_double), ("alpha", ctypes.c_double),
        ("lj_cutoff", ctypes.c_double), ("coul_cutoff", ctypes.c_double), ("skin", ctypes.c_double),
        ("a", ctypes.c_double), ("b", ctypes.c_double), ("c", ctypes.c_double),
        ("bmax", ctypes.c_double),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("precision", ctypes.c_int32), ("quirks", ctypes.c_int32),
        ("cell_size", ctypes.c_double),
        ("lanes_per_traj", ctypes.c_int32), ("block_size", ctypes.c_int32),
        ("max_steps_per_try", ctypes.c_uint32),
        ("watchdog_s", ctypes.c_double),
        ("schedule", ctypes.c_int32), ("park_steps", ctypes.c_uint32),
        ("resume_block", ctypes.c_int32), ("spec_tries", ctypes.c_int32),
    ]


class CcsStats(ctypes.Structure):
    _fields_ = [
        ("ntraj", ctypes.c_uint64), ("nfree", ctypes.c_uint64), ("nscatter", ctypes.c_uint64),
        ("nlost", ctypes.c_uint64), ("ncapped", ctypes.c_uint64),
        ("steps", ctypes.c_uint64), ("visits", ctypes.c_uint64), ("parked", ctypes.c_uint64),
        ("kernel_ms", ctypes.c_double), ("h2d_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double),
        ("lanes_per_traj", ctypes.c_int32), ("block_size", ctypes.c_int32),
        ("grid_size", ctypes.c_int32), ("speculated", ctypes.c_int32),
        ("lane_ms", ctypes.c_double), ("warp_ms", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CcsInfo(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("natoms", ctypes.c_int32),
        ("cell_size", ctypes.c_double), ("reach", ctypes.c_double),
        ("origin", ctypes.c_double * 3),
        ("charged", ctypes.c_int32), ("allpairs", ctypes.c_int32),
        ("max_cell_atoms", ctypes.c_int32), ("vel_table_len", ctypes.c_int32),
        ("sm_count", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["origin"] = list(self.origin)
        d["lanes_per_traj"] = self.reserved
        return d


class CcsFieldParams(ctypes.Structure):
    _fields_ = [
        ("samples", ctypes.c_int64), ("iterations", ctypes.c_int32), ("batch", ctypes.c_int32),
        ("log2_table", ctypes.c_int32), ("base_res", ctypes.c_int32), ("finest_res", ctypes.c_int32),
        ("validation", ctypes.c_int32),
        ("fallback_radius", ctypes.c_double), ("voxel", ctypes.c_double), ("err_voxel", ctypes.c_double),
        ("err_threshold", ctypes.c_double), ("near_fraction", ctypes.c_double), ("near_shell", ctypes.c_double),
        ("lr", ctypes.c_double), ("lam_u", ctypes.c_double), ("u0", ctypes.c_double), ("f0", ctypes.c_double),
        ("seed", ctypes.c_uint64), ("r_in", ctypes.c_double), ("r_out", ctypes.c_double),
    ]


class CcsFieldReport(ctypes.Structure):
    _fields_ = [
        ("domain_lo", ctypes.c_double * 3), ("domain_side", ctypes.c_double),
        ("levels", ctypes.c_int32), ("dense_levels", ctypes.c_int32), ("nfields", ctypes.c_int32),
        ("log2_table", ctypes.c_int32), ("res", ctypes.c_int32 * 16),
        ("samples", ctypes.c_int64), ("output_scale", ctypes.c_double * 5),
        ("gradient_scale", ctypes.c_double * 5),
        ("sample_ms", ctypes.c_double), ("label_ms", ctypes.c_double), ("train_ms", ctypes.c_double),
        ("validate_ms", ctypes.c_double), ("first_loss", ctypes.c_double), ("final_loss", ctypes.c_double),
        ("val_force_rel_rms", ctypes.c_double), ("val_force_rel_p99", ctypes.c_double),
        ("val_u_rel_rms", ctypes.c_double), ("exact_fraction", ctypes.c_double), ("err_voxels", ctypes.c_int64),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["domain_lo"] = list(self.domain_lo)
        d["res"] = list(self.res)
        d["output_scale"] = list(self.output_scale)[:self.nfields]
        d["gradient_scale"] = list(self.gradient_scale)[:self.nfields]
        return d


# Every symbol include/massccs_gpu.h declares.
EXPORTS = ["ccs_version", "ccs_create", "ccs_destroy", "ccs_params_default", "ccs_set_target",
           "ccs_set_params", "ccs_run", "ccs_run_device", "ccs_sync_stats", "ccs_eval_site_forces",
           "ccs_eval_setup", "ccs_get_info", "ccs_status_string", "ccs_last_error",
           "ccs_measure_fp32_peak", "ccs_run_device_noalloc", "ccs_run_batch",
           "ccs_field_params_default", "ccs_field_train", "ccs_field_enable", "ccs_field_eval",
           "ccs_field_setup", "ccs_field_get_weights", "ccs_field_set_weights", "ccs_field_loss_grad",
           "ccs_equipotential_points", "ccs_field_labels"]

_LIB = None


def load_library(path=LIB_PATH):
    """Load the engine library (no GPU needed to load it)."""
    global _LIB
    if _LIB is not None and path == LIB_PATH:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"massccs_b200: CUDA engine library missing at {path}; "
                           "build it with `python -m massccs_b200.build`")
    L = ctypes.CDLL(path)
    vp, sz, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    L.ccs_version.argtypes = [ctypes.POINTER(ctypes.c_int32)]
    L.ccs_create.argtypes = [ctypes.POINTER(vp), i32]
    L.ccs_destroy.argtypes = [vp]
    L.ccs_destroy.restype = None
    L.ccs_params_default.argtypes = [ctypes.POINTER(CcsParams)]
    L.ccs_params_default.restype = None
    L.ccs_set_target.argtypes = [vp, sz] + [vp] * 8
    L.ccs_set_params.argtypes = [vp, ctypes.POINTER(CcsParams)]
    L.ccs_run.argtypes = [vp, sz, ctypes.POINTER(vp), vp, vp, vp, vp, ctypes.POINTER(CcsStats)]
    L.ccs_run_device.argtypes = [vp, sz, vp, sz, vp, vp, vp, vp, vp]
    L.ccs_sync_stats.argtypes = [vp, ctypes.POINTER(CcsStats)]
    L.ccs_eval_site_forces.argtypes = [vp, sz, i32, vp, vp, vp, vp]
    L.ccs_eval_setup.argtypes = [vp, sz, ctypes.POINTER(vp), vp, vp, vp]
    L.ccs_get_info.argtypes = [vp, ctypes.POINTER(CcsInfo)]
    L.ccs_status_string.argtypes = [i32]
    L.ccs_status_string.restype = ctypes.c_char_p
    L.ccs_last_error.argtypes = [vp]
    L.ccs_last_error.restype = ctypes.c_char_p
    L.ccs_measure_fp32_peak.argtypes = [i32, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    L.ccs_run_device_noalloc.argtypes = [vp, sz, vp, sz, vp, vp, vp, vp, vp, ctypes.POINTER(CcsStats)]
    L.ccs_run_batch.argtypes = [ctypes.POINTER(vp), sz, ctypes.POINTER(sz), ctypes.POINTER(vp), vp, vp, vp, vp,
                                ctypes.POINTER(CcsStats)]
    L.ccs_field_params_default.argtypes = [ctypes.POINTER(CcsFieldParams)]
    L.ccs_field_params_default.restype = None
    L.ccs_field_train.argtypes = [vp, ctypes.POINTER(CcsFieldParams), ctypes.POINTER(CcsFieldReport)]
    L.ccs_field_setup.argtypes = [vp, ctypes.POINTER(CcsFieldParams), ctypes.POINTER(CcsFieldReport)]
    L.ccs_field_enable.argtypes = [vp, i32]
    L.ccs_field_eval.argtypes = [vp, sz, i32, vp, i32, vp, vp, vp, ctypes.POINTER(ctypes.c_int32)]
    L.ccs_field_get_weights.argtypes = [vp, vp, vp, vp]
    L.ccs_field_set_weights.argtypes = [vp, vp, vp, vp]
    L.ccs_field_loss_grad.argtypes = [vp, sz, vp, vp, ctypes.POINTER(ctypes.c_double), vp, vp]
    L.ccs_field_labels.argtypes = [vp, sz, vp, vp]
    if path == LIB_PATH:
        _LIB = L
    return L


def field_params(**kw):
    """ccs_field_params with the library's defaults, then the given fields."""
    p = CcsFieldParams()
    load_library().ccs_field_params_default(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def default_params(**kw):
    p = CcsParams()
    load_library().ccs_params_default(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class CcsError(RuntimeError):
    pass


class Engine:
    """One device context of the trajectory engine."""

    def __init__(self, device=0):
        self._L = load_library()
        h = ctypes.c_void_p()
        rc = self._L.ccs_create(ctypes.byref(h), device)
        if rc != 0:
            raise CcsError(f"ccs_create: {self._L.ccs_status_string(rc).decode()}")
        self._h = h
        self.gas = None

    def _check(self, rc, what):
        if rc != 0:
            msg = self._L.ccs_last_error(self._h).decode()
            raise CcsError(f"{what}: {self._L.ccs_status_string(rc).decode()}: {msg}")

    def close(self):
        if getattr(self, "_h", None):
            self._L.ccs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params=None, **kw):
        p = params if params is not None else default_params()
        for k, v in kw.items():
            setattr(p, k, v)
        self._check(self._L.ccs_set_params(self._h, ctypes.byref(p)), "ccs_set_params")
        self.gas = p.gas
        self.params = p
        return p

    def set_target(self, x, y, z, q, eps, sig, eps_c=None, sig_c=None):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in (x, y, z, q, eps, sig, eps_c, sig_c)]
        self._keep = arrs
        n = arrs[0].shape[0]
        self._check(self._L.ccs_set_target(self._h, n, *[_p(a) for a in arrs]), "ccs_set_target")

    def info(self):
        i = CcsInfo()
        self._check(self._L.ccs_get_info(self._h, ctypes.byref(i)), "ccs_get_info")
        return i.as_dict()

    @staticmethod
    def _rows(rnd):
        rnd = np.ascontiguousarray(rnd, dtype=np.float64)
        assert rnd.ndim == 2 and rnd.shape[0] == 9
        ptrs = (ctypes.c_void_p * 9)(*[rnd[k].ctypes.data for k in range(9)])
        return rnd, ptrs

    def run(self, rnd, want_steps=True, want_visits=True):
        """rnd: (9, n) array of the reference's pre-drawn values."""
        rnd, ptrs = self._rows(rnd)
        n = rnd.shape[1]
        status = np.empty(n, dtype=np.int8)
        omc = np.empty(n, dtype=np.float64)
        steps = np.empty(n, dtype=np.uint32) if want_steps else None
        visits = np.empty(n, dtype=np.uint32) if want_visits else None
        st = CcsStats()
        self._check(self._L.ccs_run(self._h, n, ptrs, _p(status), _p(omc), _p(steps), _p(visits),
                                    ctypes.byref(st)), "ccs_run")
        return {"status": status, "one_minus_cos": omc, "steps": steps, "visits": visits,
                "stats": st.as_dict()}

    def run_device(self, n, d_rnd, stride, d_status, d_omc, d_steps=0, d_visits=0, stream=0):
        """Asynchronous run on device pointers (ints), e.g. torch tensors' data_ptr()."""
        self._check(self._L.ccs_run_device(self._h, n, d_rnd, stride, d_status, d_omc,
                                           d_steps or None, d_visits or None, stream or None),
                    "ccs_run_device")

    def run_device_noalloc(self, n, d_rnd, stride, d_status, d_omc, d_steps=0, d_visits=0, stream=0,
                           want_stats=True):
        """ccs_run_device_noalloc: the same run with all scratch in the library's static
        device array (no device allocation); returns the statistics when asked."""
        st = CcsStats() if want_stats else None
        self._check(self._L.ccs_run_device_noalloc(self._h, n, d_rnd, stride, d_status, d_omc,
                                                   d_steps or None, d_visits or None, stream or None,
                                                   ctypes.byref(st) if st is not None else None),
                    "ccs_run_device_noalloc")
        return st.as_dict() if st is not None else None

    def sync_stats(self):
        st = CcsStats()
        self._check(self._L.ccs_sync_stats(self._h, ctypes.byref(st)), "ccs_sync_stats")
        return st.as_dict()

    # ---- learned field
    def field_train(self, **kw):
        """ccs_field_train with the default parameters overridden by kw; returns the report."""
        p = field_params(**kw)
        r = CcsFieldReport()
        self._check(self._L.ccs_field_train(self._h, ctypes.byref(p), ctypes.byref(r)), "ccs_field_train")
        self.field_nf = r.nfields
        self.field_log2 = r.log2_table
        return r.as_dict()

    def field_setup(self, **kw):
        p = field_params(**kw)
        r = CcsFieldReport()
        self._check(self._L.ccs_field_setup(self._h, ctypes.byref(p), ctypes.byref(r)), "ccs_field_setup")
        self.field_nf = r.nfields
        self.field_log2 = r.log2_table
        return r.as_dict()

    def field_enable(self, on=True):
        self._check(self._L.ccs_field_enable(self._h, 1 if on else 0), "ccs_field_enable")

    def field_eval(self, site, pos, path=0):
        """(u (n, k), g (n, k, 3), exact) of the k fields site `site` uses at pos (n x 3):
        values and minus their gradients; path 0 tensor cores, 1 warp."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = pos.shape[0]
        u = np.zeros((n, 4))
        g = np.zeros((n, 4, 3))
        ex = np.empty(n, dtype=np.int8)
        k = ctypes.c_int32()
        self._check(self._L.ccs_field_eval(self._h, n, site, _p(pos), path, _p(u), _p(g), _p(ex), ctypes.byref(k)),
                    "ccs_field_eval")
        return u[:, :k.value], g[:, :k.value], ex

    def _field_sizes(self):
        nt = 16 * (1 << self.field_log2) * 2
        nm = 64 * 32 + 64 + 64 * 64 + 64 + self.field_nf * 64 + self.field_nf
        return nt, nm

    def field_get_weights(self):
        """(table [16][T][2], mlp vector, scales: nf output then nf gradient scales)."""
        nt, nm = self._field_sizes()
        t = np.empty(nt, dtype=np.float32)
        m = np.empty(nm, dtype=np.float32)
        s = np.empty(2 * self.field_nf)
        self._check(self._L.ccs_field_get_weights(self._h, _p(t), _p(m), _p(s)), "ccs_field_get_weights")
        return t.reshape(16, -1, 2), m, s

    def field_set_weights(self, table, mlp, scales):
        t = np.ascontiguousarray(table, dtype=np.float32)
        m = np.ascontiguousarray(mlp, dtype=np.float32)
        sc = np.ascontiguousarray(scales, dtype=np.float64)
        assert sc.shape == (2 * self.field_nf,)
        self._check(self._L.ccs_field_set_weights(self._h, _p(t), _p(m), _p(sc)), "ccs_field_set_weights")

    def field_loss_grad(self, pos, labels):
        """Mean loss and its gradients (table [16][T][2], mlp vector) on the given samples."""
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        lab = np.ascontiguousarray(labels, dtype=np.float32)
        nt, nm = self._field_sizes()
        dt = np.empty(nt, dtype=np.float32)
        dm = np.empty(nm, dtype=np.float32)
        loss = ctypes.c_double()
        self._check(self._L.ccs_field_loss_grad(self._h, pos.shape[0], _p(pos), _p(lab), ctypes.byref(loss),
                                                _p(dt), _p(dm)), "ccs_field_loss_grad")
        return loss.value, dt.reshape(16, -1, 2), dm

    def field_labels(self, pos):
        """The far-part labels (n, nf, 4): value and minus the gradient of every field."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        out = np.empty((pos.shape[0], self.field_nf, 4))
        self._check(self._L.ccs_field_labels(self._h, pos.shape[0], _p(pos), _p(out)), "ccs_field_labels")
        return out

    def eval_site_forces(self, site, pos, want_visits=True):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = pos.shape[0]
        f = np.empty((n, 3))
        U = np.empty(n)
        vis = np.empty(n, dtype=np.uint32) if want_visits else None
        self._check(self._L.ccs_eval_site_forces(self._h, n, site, _p(pos), _p(f), _p(U), _p(vis)),
                    "ccs_eval_site_forces")
        return f, U, vis

    def eval_setup(self, rnd):
        rnd, ptrs = self._rows(rnd)
        n = rnd.shape[1]
        hit = np.empty(n, dtype=np.int8)
        pos = np.empty((n, 3, 3))
        vel = np.empty((n, 3, 3))
        self._check(self._L.ccs_eval_setup(self._h, n, ptrs, _p(hit), _p(pos), _p(vel)),
                    "ccs_eval_setup")
        return hit, pos, vel


def run_batch(engines, rnds, want_steps=True, want_visits=True):
    """ccs_run_batch: every engine's ion in one launch of each pass.

    engines: Engine objects (the first leads the run); rnds: one (9, n_i)
    pre-draw per ion.  Returns one result dict per ion (as Engine.run) and the
    run's statistics."""
    if len(engines) != len(rnds) or not engines:
        raise ValueError("one pre-draw per engine")
    L = engines[0]._L
    n = [int(r.shape[1]) for r in rnds]
    rnd = np.ascontiguousarray(np.concatenate([np.asarray(r, dtype=np.float64) for r in rnds], axis=1))
    total = rnd.shape[1]
    ptrs = (ctypes.c_void_p * 9)(*[rnd[k].ctypes.data for k in range(9)])
    hs = (ctypes.c_void_p * len(engines))(*[e._h.value for e in engines])
    ns = (ctypes.c_size_t * len(engines))(*n)
    status = np.empty(total, dtype=np.int8)
    omc = np.empty(total, dtype=np.float64)
    steps = np.empty(total, dtype=np.uint32) if want_steps else None
    visits = np.empty(total, dtype=np.uint32) if want_visits else None
    st = CcsStats()
    engines[0]._check(L.ccs_run_batch(hs, len(engines), ns, ptrs, _p(status), _p(omc), _p(steps), _p(visits),
                                      ctypes.byref(st)), "ccs_run_batch")
    out, o = [], 0
    for k in n:
        out.append({"status": status[o:o + k], "one_minus_cos": omc[o:o + k],
                    "steps": steps[o:o + k] if steps is not None else None,
                    "visits": visits[o:o + k] if visits is not None else None})
        o += k
    return out, st.as_dict()


def measure_fp32_peak(device=0, ms=200.0):
    """Sustained FP32 FMA TFLOP/s of the device (the plain path's roofline)."""
    v = ctypes.c_double(0)
    rc = load_library().ccs_measure_fp32_peak(device, ms, ctypes.byref(v))
    if rc != 0:
        raise CcsError(f"ccs_measure_fp32_peak failed: {rc}")
    return v.value


def params_from_system(sp, precision=PREC_FP32, quirks=0, **kw):
    """ccs_params from a dict of the reference's System scalars (keys as the
    orc_params / massccs_host set-up report them)."""
    p = default_params()
    p.gas = int(sp["gas_flag"])
    p.force_type = int(sp["force_type"])
    p.dt = sp["dt"]
    p.temperature = sp["temperature"]
    p.mu = sp["mu"]
    p.gas_inertia = sp.get("gas_inertia", 0.0)
    p.d_bond = sp.get("d_bond", 0.0)
    p.alpha = sp["alpha"]
    p.lj_cutoff = sp["lj_cutoff"]
    p.coul_cutoff = sp["coul_cutoff"]
    p.skin = sp["skin"]
    p.a, p.b, p.c, p.bmax = sp["a"], sp["b"], sp["c"], sp["bmax"]
    p.lx, p.ly, p.lz = sp["lx"], sp["ly"], sp["lz"]
    p.precision = precision
    p.quirks = quirks
    for k, v in kw.items():
        setattr(p, k, v)
    return p
