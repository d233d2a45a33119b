"""Host-side tables of projector type 3 (volume of intersection).

The type-3 weight of a voxel is the volume its inscribed sphere shares with
the tube of response at the voxel centre's distance from the ray.  The
reference tabulates that volume once per geometry (computeVoxelVolumes,
omegatomo/projector/coordinates.py:133-207) and the kernel reads the table
at (distance - bmin) * 1000.  The same table is built here, in FP64 and
rounded to float32 at the end.
"""
from __future__ import annotations

import math

import numpy as np


def sphere_cylinder_volume(R, r, b):
    """Volume shared by a sphere of radius r and an infinite cylinder of
    radius R whose axis passes at distance b from the sphere's centre
    (b an array).  The closed form of Lamarche and Leroy, Comput. Phys.
    Commun. 59 (1990) 359-369, in complete elliptic integrals of the first,
    second and third kind; the third kind by quadrature as
    Pi(alpha, k) = int_0^1 dx / ((1 + alpha x^2) sqrt(1 - x^2) sqrt(1 - k x^2)).
    b = r + R (tangency) gives 0, as in the reference."""
    from scipy.integrate import quad
    from scipy.special import ellipe, ellipk
    b = np.asarray(b, dtype=np.float64)
    R, r = float(R), float(r)
    A = np.maximum(r * r, (b + R) ** 2)
    B = np.minimum(r * r, (b + R) ** 2)
    C = (b - R) ** 2
    # b = R gives C = 0: an infinite alpha and a NaN volume there, which the
    # table drops as the reference's does
    with np.errstate(divide='ignore', invalid='ignore'):
        k = np.abs((B - C) / (A - C))
        alpha = (B - C) / C
    s = (b + R) * (b - R)
    with np.errstate(divide='ignore', invalid='ignore'):
        third = np.array([quad(lambda x, a=a, m=m: 1.0 / ((1.0 + a * x * x) * math.sqrt(1.0 - x * x) *
                                                          math.sqrt(1.0 - m * x * x)), 0.0, 1.0)[0]
                          for a, m in zip(alpha, k)], dtype=np.float64)
    K = ellipk(k)
    E = ellipe(k)
    # Heaviside step of R - b with H(0) = 1/2
    H = np.where(R - b > 0, 1.0, np.where(R - b == 0, 0.5, 0.0))
    ball = 4.0 * np.pi / 3.0 * r ** 3 * H
    V = np.zeros_like(b)
    inner = r > b + R           # the cylinder lies inside the sphere's shadow
    outer = r < b + R
    with np.errstate(divide='ignore', invalid='ignore'):
        q = 4.0 / (3.0 * np.sqrt(A - C))
        v_in = ball + q * (third * A * A * s / C - K * (A * s - (A - B) * (A - C) / 3.0)
                           - E * (A - C) * (s + (4.0 * A - 2.0 * B - 2.0 * C) / 3.0))
        v_out = ball + q * (third * B * B * s / C + K * (s * (A - 2.0 * B) + (A - B) * (3.0 * B - C - 2.0 * A) / 3.0)
                            + E * (A - C) * (-s + (2.0 * A - 4.0 * B + 2.0 * C) / 3.0))
    V[inner] = v_in[inner]
    V[outer] = v_out[outer]
    return V


def voxel_volumes(options):
    """The type-3 table of a projector object (coordinates.py:192-206):
    scales options.voxel_radius to sqrt(2) * voxel_radius * max(dx, dy, dz) / 2,
    sets options.bmax = tube_radius + voxel_radius, tabulates the volume on
    distances 0..bmax at 1/1000 mm where the sphere reaches the tube, keeps
    the non-increasing part and sets options.V (float32), options.bmin and
    options.Vmax (the whole sphere)."""
    dp = max(float(np.ravel(options.dx)[0]), float(np.ravel(options.dy)[0]), float(np.ravel(options.dz)[0]))
    options.voxel_radius = math.sqrt(2.0) * float(options.voxel_radius) * (dp / 2.0)
    R, r = float(options.tube_radius), float(options.voxel_radius)
    options.bmax = R + r
    # the reference's distance grid: 10000 float32 samples, rounded to 1/1000 mm, unique
    b = np.linspace(0, options.bmax, 10000, dtype=np.float32)
    b = b[R <= (b + r)]
    b = np.unique(np.round(b * 10 ** 3) / 10 ** 3)
    V = sphere_cylinder_volume(R, r, b)
    keep = np.append(np.diff(V), 0.0) <= 0
    options.V = np.abs(V[keep]).astype(np.float32)
    options.Vmax = 4.0 * np.pi / 3.0 * r ** 3
    options.bmin = float(np.min(b[keep]))
