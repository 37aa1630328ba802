"""Access to the 20x10x10 bar fixtures (tests/golden/long/, written by
tests/golden/make_golden.py --long from the reference harness)."""
import hashlib
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LONG = os.path.join(HERE, "golden", "long")
LONG_CASES = ["bar20_bE0", "bar20_bE1"]


def load_long(name):
    with np.load(os.path.join(LONG, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def long_deck(name):
    return os.path.join(LONG, "decks", name)


def digest(a):
    """SHA-256 of the array's little-endian bytes, as the generator stores it."""
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.astype(a.dtype.newbyteorder("<")).tobytes()).hexdigest()


def same(a, sha):
    return digest(a) == str(sha)


def bdry_classes(x, fam_ptr, dims, spacing, horizon, center=(0.0, 0.0, 0.0)):
    """Which branch of InitBdryEffectFactor (pdDataManager.cpp:1397-1461)
    each node takes: 0 full family, 1 horizon meets one face (closed form),
    2 any other node (family sum)."""
    x = np.asarray(x).reshape(-1, 3)
    fam = np.diff(fam_ptr)
    ns = int(horizon / spacing) * spacing
    lo = [-dims[a] * 0.5 * spacing + center[a] for a in range(3)]
    hi = [dims[a] * 0.5 * spacing + center[a] for a in range(3)]
    out = np.full(len(x), 2, dtype=np.int32)
    for i, p in enumerate(x):
        if fam[i] == fam.max():
            out[i] = 0
            continue
        inner = [lo[a] + ns <= p[a] <= hi[a] - ns for a in range(3)]
        for a in range(3):
            o = [b for b in range(3) if b != a]
            near = (hi[a] - ns <= p[a] <= hi[a]) or (lo[a] <= p[a] <= lo[a] + ns)
            if near and inner[o[0]] and inner[o[1]]:
                out[i] = 1
                break
    return out
