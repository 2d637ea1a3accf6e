"""Record the reference package's Wigner small-d weight tables.

Run in a container that has the reference checkout (the output is
committed):

    python tests/golden/make_dfun_golden.py /path/to/reference

``tf_pwa.dfun.small_d_weight(2j)`` (the coefficients w[l, m'+j, m+j] of
sin^l(b/2) cos^(2j-l)(b/2) in d^j_{m'm}(b)) is called for 2j = 0 .. 10 with
the reference imported over the torch-backed TF-API stand-in in
``tests/golden/tfshim`` and written to ``tests/golden/small_d.json``.
"""
import json
import os
import sys
import warnings

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    sys.path[:0] = [os.path.join(HERE, "tfshim"), ref_root]
    warnings.filterwarnings("ignore")
    from tf_pwa.dfun import small_d_weight

    out = {str(j2): small_d_weight(j2).tolist() for j2 in range(11)}
    with open(os.path.join(HERE, "small_d.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
