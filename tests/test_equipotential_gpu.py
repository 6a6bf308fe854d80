"""The equipotential ellipsoid with its rays on the GPU ("setup_device": "gpu",
ccs_equipotential_points) against the host's own restatement of
Equipotential.cpp:19-715 (GPU, through the host C-ABI).

Both paths march the same rays in 0.1 A steps against the same energy
threshold; the GPU sums each point's all-atom potential in a fixed order in
FP64, the host in atom order, so a step can flip only where a potential
lands within rounding of the threshold.  Bar: every axis within 1e-3 of the
host's (a flipped step moves one of the ~500 fitted points by 0.1 A), and
the host's axes themselves are pinned to the reference binary's report in
test_host.py.
"""
import pytest

from helpers import input_dict, workdir, write_input

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("target,gas,ft", [("c60.xyz", "He", 4), ("c60.xyz", "N2", 6), ("c60.xyz", "CO2", 4),
                                            ("04_1ubq_charge_4e_min.pqr", "He", 4),
                                            ("04_1ubq_charge_4e_min.pqr", "N2", 6)])
def test_gpu_rays_match_host_rays(target, gas, ft):
    from massccs_b200 import host
    d = workdir()
    axes = {}
    for dev in ("cpu", "gpu"):
        cfg = dict(input_dict(target, gas, ft, nprobe=2, niter=1), Equipotential="yes", setup_device=dev)
        S = host.System(write_input(d, cfg, name=f"{dev}.json"))
        axes[dev] = [S.info[k] for k in "abc"]
        S.close()
    for a_cpu, a_gpu in zip(axes["cpu"], axes["gpu"]):
        assert abs(a_gpu - a_cpu) <= 1e-3 * a_cpu, axes
