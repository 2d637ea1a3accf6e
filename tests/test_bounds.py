"""Parameter-bound transforms of the fit (``tf_pwa/variable.py:1029-1130``)
against golden values computed by the reference's own ``Bound`` class
(``tests/golden/make_bound_golden.py``): y(x), dy/dx and the inverse, for
two-sided and one-sided bounds; and the bounds read from a config."""
import json
import os

import numpy as np

from common import CONFIGS, GOLDEN


def test_bound_transforms_match_reference():
    from tf_pwa_b200.variables import Bound

    for case in json.load(open(os.path.join(GOLDEN, "bounds.json"))):
        b = Bound(case["lower"], case["upper"])
        for x, y, d, xi in zip(case["x"], case["y"], case["dydx"], case["y2x_of_y"]):
            assert abs(b.x2y(x) - y) <= 1e-12 * max(1.0, abs(y))
            assert abs(b.dydx(x) - d) <= 1e-12
            # at a bound's turning point (dy/dx = 0) x is a square root of
            # the rounding of y: there the two agree to ~1e-8
            assert abs(b.y2x(y) - xi) <= 1e-7, (case["lower"], case["upper"], y, b.y2x(y), xi)
            # the inverse reproduces y
            assert abs(b.x2y(b.y2x(y)) - y) <= 1e-12 * max(1.0, abs(y))


def test_config_bounds(tmp_path):
    import yaml

    from tf_pwa_b200.api import ConfigLoader

    dic = yaml.safe_load(open(os.path.join(CONFIGS, "d2kpipi_float.yml")))
    dic["particle"]["R1"].update({"mass_min": 0.85, "mass_max": 0.95, "width_min": 0.01})
    f = tmp_path / "c.yml"
    f.write_text(yaml.safe_dump(dic))
    cl = ConfigLoader(str(f))
    assert cl.bound_dic == {"R1_mass": (0.85, 0.95), "R1_width": (0.01, None)}
    assert np.isfinite(list(cl.vm.get_all_val())).all()
