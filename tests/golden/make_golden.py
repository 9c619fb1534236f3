"""Regenerates tests/golden/smoke_frame4.npz from the upstream golden data.

The upstream functional smoke test (test/functional/test.py:204-222,
template test/functional/parameters.xml.tmpl.in) compares frame 4 (the dump
at step 20) of ten field probes and two temperature probes against gzipped
text files under test/functional/true_data/<component>/<frame>/4.dat.gz.
Those files hold values printed with 6 significant digits, which float32
stores without loss, so they are kept here as float32 arrays, one per probe,
shaped (r_end - r_start, z_end - z_start).

Usage: python tests/golden/make_golden.py <upstream source root>
       (or set PDP3_REFERENCE to the upstream source root)
"""
import gzip
import os
import sys

import numpy as np

# component -> probe frame directory (test/functional/test.py:204-222)
FRAMES = {
    "E_r": "frame_0:0_32:256",
    "E_phi": "frame_32:256_64:512",
    "E_z": "frame_64:512_96:768",
    "H_r": "frame_96:768_128:1024",
    "H_phi": "frame_128:1024_160:1280",
    "H_z": "frame_160:1280_192:2046",
    "J_r": "frame_192:1536_244:1792",
    "J_phi": "frame_244:1792_255:2047",
    "J_z": "frame_0:0_32:256",
    "rho_beam": "frame_0:0_254:2046",
    "T/Electrons": "frame_100:100_150:150",
    "T/Ions": "frame_100:100_150:150",
}


def frame_box(name):
    a, b = name[len("frame_"):].split("_")
    r0, z0 = (int(x) for x in a.split(":"))
    r1, z1 = (int(x) for x in b.split(":"))
    return r0, z0, r1, z1


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PDP3_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <upstream source root> (or set PDP3_REFERENCE)")
    out = {}
    for comp, frame in FRAMES.items():
        path = os.path.join(root, "test", "functional", "true_data", comp, frame, "4.dat.gz")
        with gzip.open(path, "rt") as f:
            vals = np.array(f.read().split(), dtype=np.float64)
        r0, z0, r1, z1 = frame_box(frame)
        assert vals.size == (r1 - r0) * (z1 - z0), (comp, vals.size)
        key = comp.replace("/", "_")
        out[key] = vals.astype(np.float32).reshape(r1 - r0, z1 - z0)
        out[key + "__box"] = np.array([r0, z0, r1, z1], dtype=np.int32)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "smoke_frame4.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main()
