"""The reference's own penalties() through the harness (ref_penalties), on
the CPU: the checker the GPU penalty tests compare against, pinned here to
closed-form properties of the config-1 triaxial ellipsoid (semi-axes 1.0,
0.8 and 0.6 km; r = 0): its volume, a centred and axis-aligned inertia
tensor, the flattening its principal moments imply, and the reciprocal
rule of negative weights."""
import math

import numpy as np
import pytest

import cases
from oracle.bindings import Reference
from shape_b200 import engine as eng


@pytest.fixture(scope="module")
def session():
    m, p, ds = cases.c1()
    return Reference().session(m, p, deldops=[ds])


def test_ellipsoid_moment_penalties(session):
    pens = [(eng.PEN_VOLUME, 1.0), (eng.PEN_COMDEV, 1.0), (eng.PEN_INERTIADEV_UNI, 1.0), (eng.PEN_PA3TILT, 1.0),
            (eng.PEN_NONPA_UNI, 1.0), (eng.PEN_FLATTENING, 1.0), (eng.PEN_RDEV, 1.0), (eng.PEN_MAXRDEV, 1.0)]
    tot, base = session.penalties(pens)
    vol, comdev, idev, tilt, nonpa, flat, rdev, maxrdev = base
    assert abs(vol / (4 / 3 * math.pi * 1.0 * 0.8 * 0.6) - 1) < 0.02, vol
    assert comdev < 1e-20 and idev < 1e-12 and tilt < 1e-12, (comdev, idev, tilt)
    # principal moments ~ (b^2+c^2, a^2+c^2, a^2+b^2): I_x, I_y < I_z, and
    # b/c = sqrt(min(2c'^2... )) = sqrt(1.28 / 0.72) for the continuous body
    assert nonpa == 0.0
    assert abs(flat / (math.sqrt(1.28 / 0.72) - 1) ** 4 - 1) < 0.05, flat
    assert rdev == 0.0 and maxrdev == 0.0
    assert abs(tot - sum(base)) <= 1e-12 * tot


def test_edge_penalties_and_negative_weight(session):
    tot, base = session.penalties([(eng.PEN_NONSMOOTH, 2.0), (eng.PEN_CONCAVITY, 3.0), (eng.PEN_RDEV, -0.5)])
    assert base[0] > 0.0 and base[1] >= 0.0
    assert base[2] == 1.0e10                    # 1 / max(0, 1e-10)
    assert abs(tot - (2.0 * base[0] + 3.0 * base[1] + 0.5e10)) <= 1e-12 * tot
