"""Loader for tests/golden/toolbox_golden.npz."""
import json
import os

import numpy as np

from lsmlib_b200.toolbox import Field

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                    "toolbox_golden.npz")


def load_cases():
    z = np.load(PATH)
    meta = json.loads(bytes(z["__meta__"]).decode())
    cases = []
    for key, m in sorted(meta.items()):
        fields = {}
        outs = dict(m["scalar_out"])
        for name in z.files:
            if name.startswith(key + "|in|"):
                arg = name.split("|")[-1]
                fields[arg] = Field(np.asfortranarray(z[name]), m["lo"][arg])
            elif name.startswith(key + "|out|"):
                outs[name.split("|")[-1]] = z[name]
        case, sym, _ = key.split("|")
        cases.append((key, sym, fields, m["scalars"], tuple(m["fb"]), outs))
    return cases


def assert_bitwise(got, want, what):
    for k, w in want.items():
        g = got[k]
        if isinstance(w, np.ndarray):
            assert g.shape == w.shape, (what, k)
            same = (g.view(np.uint64) == w.view(np.uint64))
            if not same.all():
                bad = np.argwhere(~same)[:5]
                raise AssertionError("%s %s: %d cells differ, e.g. %s got %r want %r"
                                     % (what, k, (~same).sum(), bad[0].tolist(),
                                        g[tuple(bad[0])], w[tuple(bad[0])]))
        else:
            assert np.float64(g).view(np.uint64) == np.float64(w).view(np.uint64), \
                (what, k, g, w)
