"""Small numpy helpers shared by the tests (lattice tables, error norms)."""
import numpy as np

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1])

# reference nodeTypeMap octant masks (src/nodeTypeMap.h:10-44)
FACES = dict(WEST=0x55, EAST=0xAA, SOUTH=0x33, NORTH=0xCC, BACK=0x0F, FRONT=0xF0)


def wall_types():
    """All 26 face / edge / corner octant masks of a box."""
    import itertools
    out = {}
    axes = [("WEST", "EAST"), ("SOUTH", "NORTH"), ("BACK", "FRONT")]
    for sel in itertools.product(*[(None,) + a for a in axes]):
        names = [s for s in sel if s]
        if not names:
            continue
        m = 0
        for s in names:
            m |= FACES[s]
        out["_".join(names)] = m
    return out


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rel_linf(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
