"""Golden values of the reference's parameter-bound transform.

Run in a container with the reference checkout (outputs are committed):

    python tests/golden/make_bound_golden.py /path/to/reference

Imports ``tf_pwa.variable.Bound`` through the TF-API stand-in in
``tests/golden/tfshim`` and records, for two-sided, lower-only and
upper-only bounds, x -> y, dy/dx and y -> x on a grid of points, in
``tests/golden/bounds.json``."""
import json
import os
import sys
import warnings

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    sys.path[:0] = [os.path.join(HERE, "tfshim"), ref_root]
    warnings.filterwarnings("ignore")
    from tf_pwa.variable import Bound

    cases = []
    for a, b in ((0.8, 1.0), (0.02, None), (None, 2.5)):
        bd = Bound(a, b)
        xs = [-2.0, -0.7, -0.1, 0.0, 0.3, 1.1, 2.4]
        ys = [bd.get_x2y(x) for x in xs]
        cases.append({
            "lower": a, "upper": b, "x": xs, "y": ys,
            "dydx": [bd.get_dydx(x) for x in xs],
            "y2x_of_y": [bd.get_y2x(y) for y in ys],
        })
    with open(os.path.join(HERE, "bounds.json"), "w") as f:
        json.dump(cases, f, indent=1)
    print("bounds.json:", len(cases), "cases")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
