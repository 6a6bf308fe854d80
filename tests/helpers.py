"""Shared test helpers: input.json writing and oracle-built systems."""
import json
import os
import shutil
import tempfile

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

FLAGS = {  # force type -> (Short-range cutoff, Long-range forces, Long-range cutoff, polarizability)
    "atom": {1: ("no", "no", "no", "no"), 2: ("yes", "no", "yes", "no"),
             3: ("no", "yes", "no", "yes"), 4: ("yes", "yes", "yes", "yes")},
    "mol": {1: ("no", "no", "no", "no"), 2: ("yes", "no", "yes", "no"), 3: ("no", "yes", "no", "no"),
            4: ("yes", "yes", "yes", "no"), 5: ("no", "yes", "no", "yes"),
            6: ("yes", "yes", "yes", "yes")},
}


def input_dict(target, gas="He", ft=4, nprobe=1000, niter=10, seed=2104, ff=None, nthreads=0):
    kind = "mol" if gas in ("N2", "CO2") else "atom"
    fl = FLAGS[kind][ft]
    d = {"targetFileName": target, "numberProbe": nprobe, "nIter": niter, "seed": seed,
         "dt": 10.0, "Temp": 298.0, "skin": 0.01, "GasBuffer": gas, "Equipotential": "no",
         "Short-range cutoff": fl[0], "LJ-cutoff": 12.0, "Long-range forces": fl[1],
         "Long-range cutoff": fl[2], "Coul-cutoff": 25.0, "polarizability": fl[3]}
    if nthreads:
        d["nthreads"] = nthreads
    if ff:
        d["force-field"] = ff
    return d


def workdir(files=("c60.xyz", "04_1ubq_charge_4e_min.pqr", "uff.ff")):
    d = tempfile.mkdtemp(prefix="massccs_test_")
    for f in files:
        shutil.copy(os.path.join(GOLDEN, f), d)
    return d


def write_input(d, cfg, name="input.json"):
    p = os.path.join(d, name)
    with open(p, "w") as f:
        json.dump(cfg, f, indent=1)
    return p


def oracle_system(pyoracle, target="c60.xyz", gas="He", ft=4, nprobe=1000, niter=1, ff=None, d=None):
    d = d or workdir()
    p = write_input(d, input_dict(target, gas, ft, nprobe, niter, ff=ff))
    return pyoracle.OracleSystem(p)


def engine_for(sys_, precision=0, quirks=0, **kw):
    """An Engine configured from an oracle-built system (same target, same scalars)."""
    from massccs_b200 import engine as E
    eng = E.Engine(0)
    p = E.params_from_system(sys_.params, precision=precision, quirks=quirks, **kw)
    eng.set_params(p)
    t = sys_.target()
    co2 = sys_.params["gas_flag"] == 3
    eng.set_target(t["x"], t["y"], t["z"], t["q"], t["eps"], t["sig"],
                   t["eps_c"] if co2 else None, t["sig_c"] if co2 else None)
    return eng


def ccs_of(status, omc, bmax, niter, nprobe):
    from oracle import pyoracle
    return pyoracle.reduce(niter, nprobe, status, omc, bmax)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)
