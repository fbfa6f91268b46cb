"""Colorspace matrices for the resolve (rb_resolve / rb_k_resolve).

colorspace_matrix restates Color::generateColorspaceConversionMatrix
(src/core/color.h:60-99): the XYZ -> RGB matrix of a set of primaries and a
white point, returned column-major (glm::mat3 order) as 9 float32. The
reference takes the D65 white point from its tabulated illuminant spectrum;
the default here is the CIE D65 chromaticity (0.3127, 0.3290) with Y = 1,
and a caller that has the spectrum passes its XYZ as `white_xyz`.
"""
from __future__ import annotations

import numpy as np

# Primaries' xy chromaticities (src/core/color.h:68-87).
PRIMARIES = {
    "sRGB": ((0.64, 0.33), (0.3, 0.6), (0.15, 0.06)),
    "DCI_P3": ((0.68, 0.32), (0.265, 0.690), (0.15, 0.06)),
    "Rec2020": ((0.708, 0.292), (0.170, 0.797), (0.131, 0.046)),
}
D65_XY = (0.3127, 0.3290)


def _xyY_to_XYZ(x: float, y: float, Y: float = 1.0) -> np.ndarray:
    """XYZ::fromxyY (src/core/color.h:38-43)."""
    if y == 0.0:
        return np.zeros(3)
    return np.array([x * Y / y, Y, (1.0 - x - y) * Y / y])


def colorspace_matrix(colorspace: str = "sRGB", white_xyz=None) -> np.ndarray:
    """XYZ -> RGB matrix, column-major, float32 (9 values)."""
    prim = PRIMARIES[colorspace]
    if white_xyz is None:
        white_xyz = _xyY_to_XYZ(*D65_XY)
    w = np.asarray(white_xyz, np.float64)
    rgb = np.stack([_xyY_to_XYZ(*p) for p in prim], axis=1)     # columns: r, g, b in XYZ
    c = np.linalg.solve(rgb, w)                                   # scale of each primary
    m = np.linalg.inv(rgb * c[None, :])
    return np.ascontiguousarray(m.T.reshape(9), np.float32)      # column-major


def white_of(matrix9) -> np.ndarray:
    """The white point XYZ a column-major XYZ -> RGB matrix maps to RGB (1, 1, 1)."""
    m = np.asarray(matrix9, np.float64).reshape(3, 3).T
    return np.linalg.solve(m, np.ones(3))
