"""Writes the committed golden fixtures of the dense-stereo tests.

intel_tables.json: SHA-256 digests of the three approximation tables of Lux.Engine/Imaging/IntelApprox.Tables.cs, read as
text from a checkout of the reference whose root is the required first argument:

    python tests/golden/make_golden.py <path of the mprovenz/lux checkout>

The product's tables
(lux_b200/csrc/intel_approx_tables.h) are regenerated from the rcpss/rsqrtss instructions of an Intel host, not copied;
the test compares their digests with these.

oracle_small.npz: the oracle's outputs for a small seeded rectified pair (a regression fixture of the oracle itself).
"""
import hashlib
import json
import os
import re
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def reference_table_digests(ref_root):
    src = open(os.path.join(ref_root, "Lux.Engine", "Imaging", "IntelApprox.Tables.cs")).read()
    out = {}
    for name, body in re.findall(r"static ReadOnlySpan<uint> (\w+) => new uint\[\]\s*\{([^}]*)\}", src):
        vals = [int(v, 16) for v in re.findall(r"0x([0-9a-fA-F]+)u", body)]
        out[name] = {"count": len(vals), "sha256": hashlib.sha256(struct.pack("<%dI" % len(vals), *vals)).hexdigest()}
    return out


def main():
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: python tests/golden/make_golden.py <path of the mprovenz/lux checkout>")
    ref_root = sys.argv[1]
    d = reference_table_digests(ref_root)
    with open(os.path.join(HERE, "intel_tables.json"), "w") as f:
        json.dump({"source": "Lux.Engine/Imaging/IntelApprox.Tables.cs", "tables": d}, f, indent=1)
    sys.path.insert(0, ROOT)
    from lux_b200 import synth
    from oracle import oracle as O
    wl = synth.rectified_pair(48, 40, 16, seed=3, tile=8)
    filt = [O.box_filter3(im) for im in wl.images]
    L = O.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), img0=wl.images[0], img1=wl.images[1], raw=L["Raw"],
                        agg_pass1=L["AggPass1"], agg=L["Agg"], depth=L["Depth"], planes=L["Planes"])
    print(json.dumps(d, indent=1))


if __name__ == "__main__":
    main()
