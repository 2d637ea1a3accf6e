"""The per-event operation count of the oracle's forward pass (the work
unit of the compute roofline): independent of the number of events (only
per-event work is counted) and equal to the figures quoted with the
measurements."""
import numpy as np
import pytest

from common import load_golden, load_model

# (flops, specials) per event of sum |A|^2, oracle/flop_count.py convention
QUOTED = {"d2kpipi": (318, 77), "lc2pkpi": (1614, 228), "b2dstkpi": (6760, 1081)}


@pytest.mark.parametrize("name", sorted(QUOTED))
def test_forward_count_per_event(name):
    from oracle.flop_count import count_forward
    from oracle.pwa_oracle import OracleModel

    g, meta = load_golden(name)
    dc, vm, plan = load_model(meta["config"])
    m = OracleModel(dc.decay_group, plan)
    a = count_forward(m, g["fields_mc"][:, :400], meta["variables"])
    b = count_forward(m, g["fields_mc"][:, :1000], meta["variables"])
    np.testing.assert_allclose(a, b, rtol=1e-12)
    assert tuple(round(v) for v in b) == QUOTED[name]
