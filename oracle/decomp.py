"""Test infrastructure (the oracle): a numpy restatement of the sleeve
exchange of a decomposed grid, used only by the tests as the checker of the
library's swpc_halo_pack / swpc_halo_unpack and of the exchange over
torch.distributed.

global__comm_vel / global__comm_stress (src/swpc_3d/m_global.f90:393-609)
send, after each half step, the planes of the block's own cells that the
neighbour's stencils read, and write what arrives into the sleeve:
  velocity, to +x: Vx(iend-1), Vx(iend), Vy(iend), Vz(iend)        (:419-422)
            to -x: Vx(ibeg), Vy(ibeg), Vy(ibeg+1), Vz(ibeg), Vz(ibeg+1) (:424-428)
  stress,   to +x: Sxx(iend), Sxy(iend-1), Sxy(iend), Sxz(iend-1), Sxz(iend) (:529-533)
            to -x: Sxx(ibeg), Sxx(ibeg+1), Sxy(ibeg), Sxz(ibeg)     (:535-538)
and the same across y with the roles of x and y swapped (:435-444, :546-555);
P-SV and SH exchange across x only (src/swpc_psv/m_global.f90:312-420,
src/swpc_sh/m_global.f90:304-394).  Each plane spans the block's own cells of the
other horizontal axis and k = 1..nz, no corners.

Fields are memory boxes of shape (ny+6, nx+6, nz+6) (3D) or (nx+6, nz+6)
(2D) indexed [j+2, i+2, k+2]; the message is the concatenation, field by
field and plane by plane, of (perpendicular index, k) blocks with k fastest
-- the library's layout.
"""
from __future__ import annotations

import numpy as np

# field ids of the library (include/swpc_gpu.h)
VX, VY, VZ, SXX, SYY, SZZ, SYZ, SXZ, SXY = range(9)

# (field, planes sent to +, planes sent to -) per kind, half (0 stress,
# 1 velocity) and axis; "+" planes count back from the block's last cell
# (0 = iend), "-" planes forward from its first (1 = ibeg)
_X3 = {0: [(SXX, [0], [1, 2]), (SXY, [-1, 0], [1]), (SXZ, [-1, 0], [1])],
       1: [(VX, [-1, 0], [1]), (VY, [0], [1, 2]), (VZ, [0], [1, 2])]}
_Y3 = {0: [(SYY, [0], [1, 2]), (SXY, [-1, 0], [1]), (SYZ, [-1, 0], [1])],
       1: [(VX, [0], [1, 2]), (VY, [-1, 0], [1]), (VZ, [0], [1, 2])]}
_XPSV = {0: [(SXX, [0], [1, 2]), (SXZ, [-1, 0], [1])], 1: [(VX, [-1, 0], [1]), (VZ, [0], [1, 2])]}
_XSH = {0: [(SXY, [-1, 0], [1])], 1: [(VY, [0], [1, 2])]}


def halo_fields(kind: str, half: int, ax: int):
    if kind == "3d":
        return (_X3 if ax == 0 else _Y3)[half]
    if ax != 0:
        return []
    return (_XPSV if kind == "psv" else _XSH)[half]


def _plane(a: np.ndarray, ax: int, q: int, n_perp: int, threed: bool) -> np.ndarray:
    """Cells 1..n_perp x 1..nz of plane q (i = q for ax 0, j = q for ax 1)."""
    if not threed:
        return a[q + 2, 3:-3]
    if ax == 0:
        return a[3:3 + n_perp, q + 2, 3:-3]
    return a[q + 2, 3:3 + n_perp, 3:-3]


def pack(fields: dict, kind: str, half: int, side: int, nx: int, ny: int) -> np.ndarray:
    """The message a block with fields ``fields`` (id -> memory box) sends
    to its neighbour on ``side`` (0 -x, 1 +x, 2 -y, 3 +y)."""
    ax, up = side // 2, side % 2 == 1
    n = nx if ax == 0 else ny
    n_perp = ny if ax == 0 else nx
    out = []
    for f, to_plus, to_minus in halo_fields(kind, half, ax):
        for o in (to_plus if up else to_minus):
            q = n + o if up else o
            out.append(_plane(fields[f], ax, q, n_perp, kind == "3d").ravel())
    return np.concatenate(out) if out else np.zeros(0, np.float32)


def unpack(fields: dict, msg: np.ndarray, kind: str, half: int, side: int, nx: int, ny: int) -> None:
    """Write the message from the neighbour on ``side`` into the sleeve: from
    -x into planes -1, 0 (the sender's iend-1, iend), from +x into n+1, n+2."""
    ax, up = side // 2, side % 2 == 1
    n = nx if ax == 0 else ny
    n_perp = ny if ax == 0 else nx
    pos = 0
    for f, to_plus, to_minus in halo_fields(kind, half, ax):
        # what the lower neighbour sent "to +" lands in planes o (o <= 0);
        # what the upper one sent "to -" lands in n + o (o >= 1)
        for o in (to_minus if up else to_plus):
            q = n + o if up else o
            view = _plane(fields[f], ax, q, n_perp, kind == "3d")
            view[...] = msg[pos:pos + view.size].reshape(view.shape)
            pos += view.size
    assert pos == msg.size


def count(kind: str, half: int, side: int, nx: int, ny: int, nz: int) -> int:
    ax, up = side // 2, side % 2 == 1
    n_perp = (ny if kind == "3d" else 1) if ax == 0 else nx
    planes = sum(len(tp if up else tm) for _, tp, tm in halo_fields(kind, half, ax))
    return planes * n_perp * nz
