"""Converts the STD14 environment of the reference's speed study
(studies/cmp_speed/std14profile.cdl and std14bathy.cdl, text dumps of the
netCDF files that studies/cmp_speed/cmp_speed.cc loads) into std14.npz
beside this script: the variables as float32, exactly as the CDL lists
them.  Run with the reference source tree's path as the argument."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from underseamodelinglibrary_b200.netcdf_cdl import read_cdl  # noqa: E402


def main(ref):
    prof = read_cdl(os.path.join(ref, "studies", "cmp_speed", "std14profile.cdl"))["data"]
    bathy = read_cdl(os.path.join(ref, "studies", "cmp_speed", "std14bathy.cdl"))["data"]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "std14.npz")
    np.savez_compressed(out, p_time=prof["time"].astype(np.float32), p_depth=prof["depth"].astype(np.float32),
                        p_lat=prof["lat"].astype(np.float32), p_lon=prof["lon"].astype(np.float32),
                        p_speed=prof["speed"].astype(np.float32), b_lat=bathy["lat"].astype(np.float32),
                        b_lon=bathy["lon"].astype(np.float32), b_depth=bathy["depth"].astype(np.float32))
    print(out, os.path.getsize(out))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
