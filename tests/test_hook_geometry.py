"""The hook-sweep cables equal the reference's own drape builder (CPU).

HangingCable::build (src/apps/cable_hanging.cpp:18-47) at the sweep's
geometry (1.2 m, 120 segments, bar r 2 cm at 0.8 m, cable r 4 mm) and this
library's workloads.hanging_cable_points + Rod.centerline give the same
doubles, so the GPU sweep and the FP64 reference verdicts start from
identical cables.
"""
import numpy as np
import pytest

import ropephysics_b200 as rp
from ropephysics_b200 import workloads as W


@pytest.mark.parametrize("ratio", [1.0, 1.37, 2.5, 4.0])
@pytest.mark.parametrize("youngs", [1e8, 3e8])
def test_drape_matches_reference_builder(reference, ratio, youngs):
    h = reference.hanging(ratio, youngs, length=1.2, segments=120, bar_radius=0.02, bar_height=0.8)
    rr = reference.export(h)
    rod = rp.Rod.centerline(W.hanging_cable_points(ratio), rp.Material(youngs, **W.HOOK_MATERIAL),
                            frame_seed=(0, 1, 0))
    rod.b_rest_darboux[:] = 0.0
    for mine, ref in ((rod.x, rr.x[: rr.nP]), (rod.q, rr.q[: rr.nS]), (rod.inv_mass, rr.invMass[: rr.nP]),
                      (rod.s_compliance, rr.sComp[: rr.nSt]), (rod.b_compliance, rr.bComp[: rr.nB]),
                      (rod.b_rest_darboux, rr.bRestD[: rr.nB])):
        assert np.array_equal(mine, ref)
    reference.free(h)
