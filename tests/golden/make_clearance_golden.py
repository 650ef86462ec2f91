"""Generate tests/golden/clearance_golden.npz: the reference's EDT consumers on seeded occupancy grids.

Run where the reference is mounted (it is read, never written):

    FIELD_REFERENCE=<reference checkout> python tests/golden/make_clearance_golden.py   (or the checkout as argv[1])

The reference module itself computes every output: `bygg_gitterlaplacian` of
src/field_engine/opt/laplaceflode_v1.py:69-97 on the clearance `distance_transform_edt(~occ) * pitch`
(:313-314), and the route-validity mask of src/field_engine/opt/f33_1_topologi_v1.py:205-208
(`free & (edt_mm >= min_r_mm + margin_mm)`, margin two pitches), evaluated here as that expression.
Case k's arrays are stored under `k/<name>`; the occupancy grids are stored whole (they are small).
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FIELD_REFERENCE")
if not _ref_root:
    sys.exit("set FIELD_REFERENCE (or pass the reference checkout as the first argument)")
REF = Path(_ref_root)
sys.path.insert(0, str(REF / "src" / "field_engine" / "opt"))

import laplaceflode_v1 as LF  # noqa: E402
from scipy.ndimage import distance_transform_edt  # noqa: E402

# (shape, occupied fraction, pitch, p_kond, min_r in pitches)
CASES = [
    ((12, 10, 9), 0.10, 0.5, 1.5, 1.0),
    ((9, 13, 11), 0.40, 2.0, 1.5, 0.5),
    ((16, 16, 16), 0.03, 0.25, 1.5, 2.0),
    ((7, 5, 21), 0.70, 1.0, 0.0, 0.0),
    ((1, 17, 9), 0.25, 0.8, 1.5, 1.0),
    ((20, 3, 1), 0.15, 1.3, 2.0, 0.5),
    ((24, 24, 24), 0.08, 0.4, 1.5, 1.5),
    ((5, 5, 5), 0.96, 1.0, 1.5, 0.0),
]


def main():
    rng = np.random.default_rng(20261204)
    out = {}
    for k, (shape, frac, pitch, p_kond, min_r) in enumerate(CASES):
        occ = rng.random(shape) < frac
        occ.flat[int(rng.integers(occ.size))] = True  # at least one occupied cell
        edt_mm = distance_transform_edt(~occ) * pitch
        n, nodkarta, u, v, kond, L = LF.bygg_gitterlaplacian(occ, edt_mm, pitch, p_kond=p_kond)
        min_r_mm = min_r * pitch
        margin_mm = 2.0 * pitch
        valid = (~occ) & (edt_mm >= min_r_mm + margin_mm)
        for name, arr in dict(occ=occ, edt_mm=edt_mm, nodkarta=nodkarta, u=u, v=v, kond=kond, indptr=L.indptr,
                              indices=L.indices, data=L.data, valid=valid,
                              params=np.array([pitch, p_kond, min_r_mm, margin_mm, n], np.float64)).items():
            out[f"{k}/{name}"] = arr
    np.savez_compressed(HERE / "clearance_golden.npz", **out)
    print(f"{len(CASES)} cases -> {HERE / 'clearance_golden.npz'}")


if __name__ == "__main__":
    main()
