"""Generate the golden fixtures of tests/golden/ from the reference project.

Run in a container where the reference is mounted (it reads /root/reference and
runs the reference binary built by `make -C oracle ref`):

    python tests/golden/make_golden.py

Writes
  c60.xyz, 04_1ubq_charge_4e_min.pqr, *.ff   the reference's example inputs
  shipped_logs.json   printed values of the reference's shipped outputs
                      (ccs_He.log, ccs_Ar.log, ccs_N2.log, ccs_CO2.log, ccs.out)
  reference_runs.json printed values of the reference binary on small runs of
                      every force type whose arithmetic is well defined
"""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

REF = os.environ.get("REFERENCE_DIR", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFBIN = os.path.join(ROOT, "oracle", "_ref", "massccs")

FLAGS = {  # (short-range cutoff, long-range forces, long-range cutoff, polarizability)
    "atom": {1: ("no", "no", "no", "no"), 2: ("yes", "no", "yes", "no"), 4: ("yes", "yes", "yes", "yes")},
    "mol": {1: ("no", "no", "no", "no"), 2: ("yes", "no", "yes", "no"), 3: ("no", "yes", "no", "no"),
            4: ("yes", "yes", "yes", "no"), 6: ("yes", "yes", "yes", "yes")},
}
# force types 3 (atomic) and 5 (molecular) read uninitialised accumulators in the
# reference (Force.cpp:517-522, 836-889), so their outputs are not reproducible.


def parse_report(text):
    it = []
    cur = {}
    for line in text.splitlines():
        m = re.match(r"^(Nfree|Nscatter|Nlost): (-?\d+)", line)
        if m:
            cur[m.group(1)] = int(m.group(2))
        m = re.match(r"^omega: (\S+)", line)
        if m:
            cur["omega"] = m.group(1)
            it.append(cur)
            cur = {}
    avg = re.search(r"average value of CCS = (\S+)", text)
    err = re.search(r"error value of CCS = (\S+)", text)
    return {"iterations": it, "ccs": avg.group(1) if avg else None, "err": err.group(1) if err else None}


def input_json(target, gas, flags, nprobe, niter, seed=2104, ff=None, nthreads=8):
    d = {"targetFileName": target, "numberProbe": nprobe, "nIter": niter, "seed": seed,
         "nthreads": nthreads, "dt": 10.0, "Temp": 298.0, "skin": 0.01, "GasBuffer": gas,
         "Equipotential": "no", "Short-range cutoff": flags[0], "LJ-cutoff": 12.0,
         "Long-range forces": flags[1], "Long-range cutoff": flags[2], "Coul-cutoff": 25.0,
         "polarizability": flags[3]}
    if ff:
        d["force-field"] = ff
    return d


def main():
    for f in ("c60.xyz", "04_1ubq_charge_4e_min.pqr", "uff.ff", "charmm.ff", "gromos.ff", "imos.ff", "oplsaa.ff"):
        shutil.copy(os.path.join(REF, f), os.path.join(HERE, f))
    logs = {}
    for name, tgt, gas in (("ccs_He.log", "c60.xyz", "He"), ("ccs_Ar.log", "c60.xyz", "Ar"),
                           ("ccs_N2.log", "c60.xyz", "N2"), ("ccs_CO2.log", "c60.xyz", "CO2"),
                           ("ccs.out", "04_1ubq_charge_4e_min.pqr", "He")):
        rep = parse_report(open(os.path.join(REF, name)).read())
        rep["input"] = input_json(tgt, gas, ("yes", "yes", "yes", "yes"), 10000, 10)
        logs[name] = rep
    json.dump(logs, open(os.path.join(HERE, "shipped_logs.json"), "w"), indent=1)

    if not os.path.exists(REFBIN):
        sys.exit("reference binary missing: run `make -C oracle ref` first")
    runs = []
    work = tempfile.mkdtemp()
    for f in ("c60.xyz", "04_1ubq_charge_4e_min.pqr", "uff.ff"):
        shutil.copy(os.path.join(HERE, f), work)
    cases = []
    for gas in ("He", "Ar", "co2", "N2", "CO2"):
        kind = "mol" if gas in ("N2", "CO2") else "atom"
        for ft, fl in FLAGS[kind].items():
            cases.append(("c60.xyz", gas, ft, fl, None))
    cases += [("04_1ubq_charge_4e_min.pqr", "He", 4, FLAGS["atom"][4], None),
              ("04_1ubq_charge_4e_min.pqr", "N2", 6, FLAGS["mol"][6], None),
              ("04_1ubq_charge_4e_min.pqr", "CO2", 4, FLAGS["mol"][4], None),
              ("c60.xyz", "He", 2, FLAGS["atom"][2], "uff.ff"),
              ("c60.xyz", "Ar", 4, FLAGS["atom"][4], "uff.ff")]
    for tgt, gas, ft, fl, ff in cases:
        nprobe, niter = 200, 5
        cfg = input_json(tgt, gas, fl, nprobe, niter, ff=ff)
        p = os.path.join(work, "input.json")
        json.dump(cfg, open(p, "w"))
        out = subprocess.run([REFBIN, "input.json"], cwd=work, capture_output=True, text=True,
                             timeout=600).stdout
        rep = parse_report(out)
        rep["input"] = cfg
        rep["force_type"] = ft
        runs.append(rep)
        print(tgt, gas, ft, rep["ccs"], rep["err"], flush=True)
    json.dump(runs, open(os.path.join(HERE, "reference_runs.json"), "w"), indent=1)
    shutil.rmtree(work)


if __name__ == "__main__":
    main()
