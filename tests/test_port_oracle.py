"""The multithreaded C restatement of the oracle (oracle/port.c), which
bench.py times as the CPU baseline, against the numpy oracle: same J, C^H,
kappa^H, cycle counts and next design on seeded cells, for both the cold and
the warm-started solves of consecutive OC iterations."""
import numpy as np
import pytest

from oracle import ihd_oracle as O
from oracle import port as P


@pytest.fixture(scope="module", autouse=True)
def _threads():
    P.build()
    P.set_threads(2)


@pytest.mark.parametrize("r,levels,spec,method", [
    (8, 3, "stiffness:0.5,thermal:0.5", "vcycle"),
    (16, 4, "stiffness:0.3333333333333333,shear:0.3333333333333333,thermal:0.3333333333333333", "vcycle"),
    (8, 2, "shear", "vcycle"),
    (16, 4, "stiffness:0.5,thermal:0.5", "pcg"),
])
def test_port_follows_the_oracle(r, levels, spec, method):
    w = O.parse_objective_spec(spec)
    x = O.seed_density(1, r, 2.0, 0.3).reshape(-1)
    cell = P.Cell(r, levels)
    prev = None
    for it in range(2):
        xp, ip = P.oc_iteration(x, cell, w, volfrac=0.3, rtol=1e-12, max_cycles=400, warm=True, method=method)
        xo, io = O.oc_iteration(x, r, w, volfrac=0.3, levels=levels, rtol=1e-12, max_cycles=400, u0=prev,
                                method=method)
        prev = io["res"]
        assert abs(ip["J"] - io["J"]) <= 1e-12 * abs(io["J"]), it
        if io["CH"] is not None:
            assert np.abs(ip["CH"] - io["CH"]).max() <= 1e-12 * np.abs(io["CH"]).max()
            assert ip["cycles_elastic"] == io["res"]["cycles_elastic"]
        if io["kappa"] is not None:
            assert np.abs(ip["kappa"] - io["kappa"]).max() <= 1e-12 * np.abs(io["kappa"]).max()
            assert ip["cycles_thermal"] == io["res"]["cycles_thermal"]
        assert np.abs(xp - xo).max() <= 1e-12
        assert abs(ip["dx_max"] - io["dx_max"]) <= 1e-12
        x = xo


def test_port_rejects_bad_arguments():
    cell = P.Cell(8, 3)
    with pytest.raises(ValueError):
        P.oc_iteration(np.full(512, 0.3), cell, {"thermal": 1.0}, volfrac=0.3, filter_k=2)
