"""Partially constrained velocity nodes for the bc3LHS / bc3Res / itrBC tests.

The reference prescribes one or two velocity components of a node through
ibits(iBC,3,3) = 1..6 and the coefficients BC(:,3:6) (itrbc.f90:33-101):
e.g. ibits = 1 fixes u1 = BC3 - BC4 u2 - BC5 u3 (a slip-type constraint),
ibits = 3 fixes u1 = BC3 - BC4 u3 and u2 = BC5 - BC6 u3.
"""
import numpy as np


def with_partial_constraints(m, masks=(1, 2, 3, 4, 5, 6), frac=0.5, seed=5):
    """Give a random fraction of the tube's no-slip wall nodes (iBC with all
    three velocity bits, zero BC) one of ``masks`` with random coefficients
    in [-0.4, 0.4] and zero targets.  Returns the node indices changed."""
    rng = np.random.default_rng(seed)
    inlet = set(int(i) for i in (m.inlet_nodes if m.inlet_nodes is not None else []))
    wall = [i for i in np.nonzero(((m.iBC >> 3) & 7) == 7)[0] if int(i) not in inlet]
    pick = np.array(sorted(rng.choice(wall, size=int(frac * len(wall)), replace=False)), dtype=np.int64)
    mk = np.array([masks[k % len(masks)] for k in range(len(pick))])
    m.iBC[pick] = (m.iBC[pick] & ~(7 << 3)) | (mk << 3)
    m.BC[pick, 2] = 0.0
    m.BC[pick, 3] = rng.uniform(-0.4, 0.4, len(pick))
    m.BC[pick, 4] = np.where(np.isin(mk, (1, 2, 4)), rng.uniform(-0.4, 0.4, len(pick)), 0.0)
    m.BC[pick, 5] = np.where(np.isin(mk, (3, 5, 6)), rng.uniform(-0.4, 0.4, len(pick)), 0.0)
    return pick
