"""The drop-in CLI on the reference's own inputs (GPU).

`massccs input.json` prints the reference's report; in FP64 mode the engine
replays the shipped ccs_He.log / ccs.out iteration by iteration (the printed
6-digit omegas), in FP32 mode the CCS agrees within 0.5 %.
"""
import json
import os
import re
import subprocess

import pytest

from helpers import GOLDEN, workdir, write_input

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "massccs_b200", "bin", "massccs")


def _run(cfg):
    d = workdir()
    p = write_input(d, cfg)
    out = subprocess.run([CLI, p], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    om = re.findall(r"^omega: (\S+)", out.stdout, re.M)
    ccs = float(re.search(r"average value of CCS = (\S+)", out.stdout).group(1))
    return out.stdout, om, ccs


@pytest.mark.parametrize("log", ["ccs_He.log", "ccs.out"])
def test_cli_fp64_replays_shipped_log(log):
    rep = json.load(open(os.path.join(GOLDEN, "shipped_logs.json")))[log]
    cfg = dict(rep["input"], precision="fp64")
    text, om, ccs = _run(cfg)
    ref = [it["omega"] for it in rep["iterations"]]
    assert sum(a == b for a, b in zip(om, ref)) >= 8, (om, ref)
    assert abs(ccs - float(rep["ccs"])) / float(rep["ccs"]) < 1e-3
    for key in ("INPUT:: Simulation Parameters", "Geometric Ellipsoid", "Linked-cell", "Trajectory calculations",
                "CCS time", "error value of CCS"):
        assert key in text


@pytest.mark.parametrize("log", ["ccs_He.log", "ccs_Ar.log", "ccs_N2.log", "ccs.out"])
def test_cli_fp32_within_half_percent(log):
    rep = json.load(open(os.path.join(GOLDEN, "shipped_logs.json")))[log]
    text, om, ccs = _run(dict(rep["input"], precision="fp32"))
    assert len(om) == 10
    assert abs(ccs - float(rep["ccs"])) / float(rep["ccs"]) < 0.005, (ccs, rep["ccs"])
