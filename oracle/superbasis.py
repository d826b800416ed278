"""ORACLE -- test infrastructure only.

The superblock basis permutation that DMRG++ builds when it forms the product
of the left and right blocks (Basis::setToProduct, dmrg/Engine/Basis.h:162-330,
with the sector offsets of Basis::offsetsFromSizes, Basis.h:753-775), restated
in numpy so that the sector gather index (InitKronHamiltonian::copyIn,
InitKronHamiltonian.h:158-221) can be checked on realistic inputs:

* the product's quantum-number sectors are laid out in the order in which
  their quantum numbers are first met, left group outer, right group inner;
* inside a sector, the (left group ps, right group pe) blocks follow one
  another with pe outer and ps inner;
* inside a block, state (ileft, iright) sits at ileft + iright * leftSize;
* permInverse[(left state) + (right state) * nl] is that position.
"""
from __future__ import annotations

import numpy as np


def product_permutation(left_qns, left_sizes, right_qns, right_sizes):
    """Returns (perm_inverse, sectors): perm_inverse has nl*nr entries (uint64)
    and sectors maps each product quantum number to (offset, size)."""
    left_sizes = [int(s) for s in left_sizes]
    right_sizes = [int(s) for s in right_sizes]
    loff = np.concatenate([[0], np.cumsum(left_sizes)]).astype(np.int64)
    roff = np.concatenate([[0], np.cumsum(right_sizes)]).astype(np.int64)
    nl, nr = int(loff[-1]), int(roff[-1])

    def add(a, b):
        return tuple(x + y for x, y in zip(a, b))

    order, sizes = [], {}
    for ps, ql in enumerate(left_qns):
        for pe, qr in enumerate(right_qns):
            q = add(ql, qr)
            if q not in sizes:
                order.append(q)
                sizes[q] = 0
            sizes[q] += left_sizes[ps] * right_sizes[pe]
    sectors, off = {}, 0
    for q in order:
        sectors[q] = (off, sizes[q])
        off += sizes[q]
    extra = {q: 0 for q in order}
    perm_inverse = np.zeros(nl * nr, dtype=np.uint64)
    for pe, qr in enumerate(right_qns):
        for ps, ql in enumerate(left_qns):
            q = add(ql, qr)
            start = sectors[q][0] + extra[q]
            ls, rs = left_sizes[ps], right_sizes[pe]
            extra[q] += ls * rs
            il = np.arange(ls)[:, None]
            ir = np.arange(rs)[None, :]
            glob = (loff[ps] + il) + (roff[pe] + ir) * nl
            perm_inverse[glob.ravel()] = (start + il + ir * ls).ravel()
    return perm_inverse, sectors
