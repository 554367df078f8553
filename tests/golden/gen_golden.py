"""Regenerate tests/golden/toolbox_golden.npz from the reference itself.

The reference toolbox is Fortran 77 and no Fortran compiler is available, so
its own source files are translated mechanically (oracle/f77toc.py) and built
with the reference's optimisation flags (make -C oracle ref).  This script runs
that build on the seeded cases of cases.py and stores inputs and outputs.

    make -C oracle ref && python tests/golden/gen_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import oracle  # noqa: E402
from cases import VARIANTS, make_inputs, run  # noqa: E402
from lsmlib_b200 import abi  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "toolbox_golden.npz")


def main():
    ref = oracle.reference_toolbox()
    blobs, meta = {}, {}
    for ci, case in enumerate(("smooth", "degenerate")):
        for si, sym in enumerate(sorted(abi.SIGNATURES)):
            for vi, var in enumerate(VARIANTS.get(sym, [{}])):
                key = "%s|%s|%d" % (case, sym, vi)
                fields, scalars, fb = make_inputs(sym, case, seed=1000 * ci + 10 * si + vi)
                scalars.update(var)
                out = run(ref, sym, fields, scalars, fb)
                meta[key] = {"scalars": scalars, "fb": list(fb),
                             "lo": {k: list(v.lo) for k, v in fields.items()},
                             "scalar_out": {k: v for k, v in out.items()
                                            if not isinstance(v, np.ndarray)}}
                for k, v in fields.items():
                    blobs[key + "|in|" + k] = v.data
                for k, v in out.items():
                    if isinstance(v, np.ndarray):
                        blobs[key + "|out|" + k] = v
    blobs["__meta__"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **blobs)
    print("wrote %s (%d cases, %.1f KB)" % (OUT, len(meta), os.path.getsize(OUT) / 1024))


if __name__ == "__main__":
    main()
