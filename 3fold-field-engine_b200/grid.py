"""Grid metadata and the block-sparse field layout (the reference's data contract).

``GridMeta`` and ``SparseField`` keep the reference's field names and meaning
(src/field_engine/faltkarna_v1.py:50-74): blocks of ``block``^3 voxels, block-linear id
``lin = (bi*n_by + bj)*n_bz + bk``, vertex-centred samples at ``x0 + index*pitch``, Lipschitz
margin ``sqrt(3)*block*pitch``, ``kind`` in {-1, 0, +1}, ascending ``active_ids``, tiles
(n_active, B, B, B) in C order, background -BIG / +BIG.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

BIG = 1.0e6          # background constant: interior -BIG, exterior +BIG (faltkarna_v1.py:46)
FIXPT_SCALE = 1.0e6  # int64 fixed-point scale of the determinism checksum (faltkarna_v1.py:47)


@dataclass
class GridMeta:
    x0: float
    y0: float
    z0: float
    pitch: float
    nx: int
    ny: int
    nz: int
    block: int = 8

    def __post_init__(self):
        self.n_bx = -(-self.nx // self.block)
        self.n_by = -(-self.ny // self.block)
        self.n_bz = -(-self.nz // self.block)
        self.n_blocks = self.n_bx * self.n_by * self.n_bz
        self.margin_mm = math.sqrt(3.0) * self.block * self.pitch

    @property
    def extent(self) -> float:
        """Largest absolute world coordinate a corner of the grid can take."""
        hi = [self.x0 + self.n_bx * self.block * self.pitch, self.y0 + self.n_by * self.block * self.pitch,
              self.z0 + self.n_bz * self.block * self.pitch]
        return float(max(abs(self.x0), abs(self.y0), abs(self.z0), *map(abs, hi), self.pitch))

    def guard(self) -> float:
        """Guard band of the float64 recheck: 4 float32 ulps of the grid's coordinate magnitude."""
        return float(4.0 * np.spacing(np.float32(self.extent)))


@dataclass
class SparseField:
    meta: GridMeta
    kind: np.ndarray            # (n_blocks,) int32: -1/0/+1
    active_ids: np.ndarray      # (n_active,) int32 block-linear id, kind == 0, ascending
    tiles: np.ndarray           # (n_active, block, block, block) float32
    corner_min_abs: np.ndarray  # (n_blocks,) float32, classification diagnostic
    stats: dict = field(default_factory=dict)


def block_ijk(lin, meta: GridMeta):
    """(bi, bj, bk) of block-linear ids (faltkarna_v1.py:77-82)."""
    n_by, n_bz = meta.n_by, meta.n_bz
    return lin // (n_by * n_bz), (lin // n_bz) % n_by, lin % n_bz


def konservering_check(volym_matt_mm3: float, volym_facit_mm3: float, tol_frac: float) -> dict:
    """Volume against an analytic reference within a declared band (faltkarna_v1.py:353-356)."""
    diff_frac = abs(volym_matt_mm3 - volym_facit_mm3) / max(abs(volym_facit_mm3), 1e-9)
    return dict(volym_matt_mm3=volym_matt_mm3, volym_facit_mm3=volym_facit_mm3, diff_frac=diff_frac,
                tol_frac=tol_frac, GRON=bool(diff_frac <= tol_frac))


def determinism_cert(varden: list) -> dict:
    """N runs must be bit-identical (faltkarna_v1.py:359-365)."""
    identiska = all(v == varden[0] for v in varden)
    return dict(n_korningar=len(varden), varden=varden, bit_identiska=bool(identiska))


def stats_of(meta: GridMeta, kind: np.ndarray, n_active: int) -> dict:
    b3 = meta.block ** 3
    return dict(n_blocks=int(meta.n_blocks), n_active=int(n_active), n_interior=int(np.sum(kind == -1)),
                n_exterior=int(np.sum(kind == 1)), active_voxels=int(n_active * b3),
                dense_voxels=int(meta.nx * meta.ny * meta.nz), margin_mm=meta.margin_mm)
