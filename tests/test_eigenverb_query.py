"""eigenverb_collection.find_eigenverbs on the reference's own case
(eigenverbs/test/eigenverbs_test.cc:70-121): 80 simplified bottom
eigenverbs for D/E -80..-10 deg x AZ 0..90 deg in 10 deg steps, 1000 m
deep around 36N 16E, queried with the footprint at D/E -40, AZ 30."""
import math

import numpy as np

from underseamodelinglibrary_b200 import eigenverbs as E
from underseamodelinglibrary_b200 import types as T

DE_SPACING = AZ_SPACING = 10.0


def create_eigenverb(source, depth, de, az):
    """eigenverbs_test.cc:24-54"""
    de_rad, az_rad = math.radians(de), math.radians(az)
    grazing = abs(de_rad)
    slant = depth / math.sin(grazing)
    horz = depth / math.tan(grazing)
    v = E.eigenverb_model()
    v.sound_speed = 1500.0
    v.travel_time = slant / v.sound_speed
    v.power = np.full(1, 1e20)
    v.length = 0.5 * slant * math.radians(DE_SPACING) / math.sin(grazing)
    v.width = 0.5 * slant * math.radians(AZ_SPACING) * math.cos(grazing)
    p = T.wposition1(source, horz, az_rad)
    p.altitude(-depth)
    v.position = (p.rho, p.theta, p.phi)
    v.direction = az_rad
    v.grazing = grazing
    v.de_index = int((90.0 + de) / DE_SPACING - 1.0)
    v.az_index = int(az / AZ_SPACING)
    return v


def test_find_eigenverbs_reference_case():
    T.compute_earth_radius(36.0)
    source = T.wposition1(36.0, 16.0, 0.0)
    coll = E.eigenverb_collection(0)
    az = 0.0
    while az <= 90.0:
        de = -90.0 + DE_SPACING
        while de < 0.0:
            coll.add_eigenverb(create_eigenverb(source, 1000.0, de, az), E.BOTTOM)
            de += DE_SPACING
        az += AZ_SPACING
    assert coll.size(E.BOTTOM) == 80 and len(coll.eigenverbs(E.BOTTOM)) == 80
    bounding = create_eigenverb(source, 1000.0, -40.0, 30.0)
    found = coll.find_eigenverbs(bounding, E.BOTTOM)
    assert 0 < len(found) < 80
    keys = {(v.de_index, v.az_index) for v in found}
    assert (bounding.de_index, bounding.az_index) in keys   # its own footprint
    assert (0, 9) not in keys                               # D/E -80, AZ 90: far away
    # every hit is near the bounding footprint in D/E and AZ
    assert all(abs(d - bounding.de_index) <= 3 and abs(a - bounding.az_index) <= 3 for d, a in keys)
    # the search area grows with search_scale
    E.eigenverb_collection.search_scale = 3.0
    try:
        assert len(coll.find_eigenverbs(bounding, E.BOTTOM)) >= len(found)
    finally:
        E.eigenverb_collection.search_scale = 1.5
    assert coll.find_eigenverbs(bounding, E.SURFACE) == []
