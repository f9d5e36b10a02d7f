import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running check")
    config.addinivalue_line("markers", "fullsize: parity at a workload's stated size (1M, 4.2M molecules, 512 boxes)")


_FULLSIZE = []


def pytest_runtest_logreport(report):
    if report.when == "call" and "fullsize" in report.keywords:
        _FULLSIZE.append((report.nodeid.split("::")[-1], report.outcome, report.duration))


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    """Names the full-size parity tests and their outcome at the end of a quiet run."""
    if _FULLSIZE:
        terminalreporter.write_line("full-size parity against the oracle:")
        for name, outcome, dur in _FULLSIZE:
            terminalreporter.write_line(f"  {outcome:7s} {name} ({dur:.0f} s)")


def _build_oracle():
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)


_build_oracle()


def load_golden(name):
    import numpy as np

    return dict(np.load(os.path.join(GOLDEN, f"ref_{name}.npz")))


def system_from_golden(name):
    """Rebuild the seeded input system of a golden fixture."""
    import json

    import numpy as np

    from madpac_b200 import workloads as W

    g = load_golden(name)
    meta = json.load(open(os.path.join(GOLDEN, "ref_systems.json")))[name]
    comps = [W.Component(float(e), float(s), float(m), bool(d))
             for e, s, m, d in zip(g["eps"], g["sigma"], g["mass"], g["do_shift"])]
    return W.System(length=g["length"], components=comps, mix=g["mix"], ids=g["in_id"], cid=g["in_cid"],
                    r=g["in_r"], v=g["in_v"], temperature=meta["temperature"], cutoff=meta["cutoff"],
                    lj_cutoff=meta["lj_cutoff"], dt=meta["dt"], nve=meta["nve"], name=name), g, meta


GOLDEN_NAMES = ["fcc864_unshifted", "two_species_2048", "thermostat_500", "slab_8000", "wrap_864"]


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
