"""Projector option sets shared by the golden-fixture generator and the tests.

Each entry is a dict of ``projectorClass`` attributes.  ``pet_cfg0`` is the
CPU-runnable PET OSEM workload (288 crystals/ring x 16 rings, 600 mm ring,
144 x 144 x 31 span-3 sinograms, 64 x 64 x 16 image over 300 x 300 x 64 mm,
8 subsets); the others are small geometries that exercise the remaining
branches of the geometry code (TOF, ring blocks not divisible by
four, span 1, measurement-level subsets, cone-beam CT).
"""
import math

import numpy as np


def _pet(blocks, cpb, rings, diameter, ndist, nang, nx, nz, fov, axial, subsets=8, subset_type=8, span=3,
         ring_difference=None, **extra):
    d = dict(blocks_per_ring=blocks, cryst_per_block=cpb, cryst_per_block_axial=rings, linear_multip=1,
             cr_p=math.pi * diameter / (blocks * cpb), cr_pz=4.0, diameter=float(diameter),
             FOVa_x=float(fov), FOVa_y=float(fov), axial_fov=float(axial), rings=rings,
             det_per_ring=blocks * cpb, det_w_pseudo=blocks * cpb, Nx=nx, Ny=nx, Nz=nz, span=span,
             ring_difference=rings - 1 if ring_difference is None else ring_difference,
             Ndist=ndist, Nang=nang, projector_type=1, subsets=subsets, subsetType=subset_type, Niter=2,
             verbose=0)
    if span > 1 and "NSinos" not in extra:
        st = _segments(rings, span, d["ring_difference"], nz)
        d["NSinos"] = d["TotSinos"] = int(np.sum(st))
    d.update(extra)
    return d


def _segments(rings, span, ring_difference, nz):
    st = np.concatenate((np.array(rings * 2 - 1, ndmin=1),
                         np.arange(rings * 2 - 1 - (span + 1), max(nz - ring_difference * 2, rings - ring_difference),
                                   -span * 2)))
    return np.insert(np.repeat(st[1:], 2), 0, st[0])


CONFIGS = {
    # the CPU-runnable PET OSEM workload (plain method)
    "pet_cfg0": _pet(16, 18, 16, 600, 144, 144, 64, 16, 300, 64, NSinos=31, TotSinos=181),
    # small PET, all oblique segments, 4 subsets
    "pet_mini": _pet(8, 12, 8, 300, 40, 48, 32, 15, 180, 34, subsets=4),
    # small PET with 7 TOF bins
    "pet_mini_tof": _pet(8, 12, 8, 300, 40, 48, 32, 15, 180, 34, subsets=4, TOF_bins=7, TOF_bins_used=7,
                         TOF_FWHM=200e-12, TOF_width=7 * 0.0, ),
    # 14 blocks per ring (not divisible by four), span 1
    "pet_odd_span1": _pet(14, 10, 5, 400, 41, 70, 24, 9, 240, 22, subsets=5, span=1),
    # measurement-level subsets (every 4th column measurement)
    "pet_stype1": _pet(8, 6, 4, 300, 20, 24, 16, 7, 180, 18, subsets=4, subset_type=1),
    "pet_stype2": _pet(8, 6, 4, 300, 20, 24, 16, 7, 180, 18, subsets=3, subset_type=2),
    "pet_stype4": _pet(8, 6, 4, 300, 20, 24, 16, 7, 180, 18, subsets=4, subset_type=4),
    "pet_stype5": _pet(8, 6, 4, 300, 20, 24, 16, 7, 180, 18, subsets=4, subset_type=5),
    # cone-beam CT, flat panel (scaled-down 512x512-panel, 360-view geometry)
    "ct_mini": dict(CT=True, nRowsD=48, nColsD=40, nProjections=36, dPitchX=1.6, dPitchY=1.6,
                    sourceToCRot=500., sourceToDetector=1000., Nx=32, Ny=32, Nz=24, FOVa_x=64., FOVa_y=64.,
                    axial_fov=48., projector_type=1, subsets=6, subsetType=8, Niter=1, verbose=0,
                    angles=np.linspace(0, 2 * np.pi, 36, endpoint=False).astype(np.float32),
                    SinM=np.zeros((48, 40, 36), dtype=np.float32)),
}
# the same CT geometry with the branchless distance-driven projector (type 5)
CONFIGS["ct_mini5"] = dict(CONFIGS["ct_mini"], projector_type=5, subsets=1)
# type 5 with 0.5 mm voxels under 4 mm pixels: a pixel's footprint spans about
# four voxels laterally and axially (the opposite regime of ct_mini5, where a
# voxel's footprint spans several pixels)
CONFIGS["ct_fine5"] = dict(CT=True, nRowsD=24, nColsD=20, nProjections=30, dPitchX=4.0, dPitchY=4.0,
                           sourceToCRot=500., sourceToDetector=1000., Nx=64, Ny=64, Nz=48, FOVa_x=32.,
                           FOVa_y=32., axial_fov=24., projector_type=5, subsets=1, subsetType=8, Niter=1,
                           verbose=0, angles=np.linspace(0, 2 * np.pi, 30, endpoint=False).astype(np.float32),
                           SinM=np.zeros((24, 20, 30), dtype=np.float32))
# four of the 360 views (0, 91, 182 and 273 degrees) of the cone-beam CT
# benchmark geometry: 512 x 512 panel of 0.4 mm pixels, SOD 500 / SDD 1000 mm,
# 256^3 volume of 0.25 mm voxels (every voxel footprint lies on the panel)
_CFG1_ANGLES = np.linspace(0, 2 * np.pi, 360, endpoint=False).astype(np.float32)[[0, 91, 182, 273]]
CONFIGS["ct_cfg1_4v"] = dict(CT=True, nRowsD=512, nColsD=512, nProjections=4, dPitchX=0.4, dPitchY=0.4,
                             sourceToCRot=500., sourceToDetector=1000., Nx=256, Ny=256, Nz=256, FOVa_x=64.,
                             FOVa_y=64., axial_fov=64., projector_type=5, subsets=1, subsetType=8, Niter=1,
                             verbose=0, angles=_CFG1_ANGLES, SinM=np.zeros((512, 512, 4), dtype=np.float32))
# TOF width so that the bins cover the FOV diagonal: 7 bins of 85 mm / (c/2) seconds
CONFIGS["pet_mini_tof"]["TOF_width"] = 85.0 / (2.99792458e11 / 2.)
# projector type 4 (interpolation): PET, PET with TOF, PET with a sampling
# length of half a voxel and 3 subsets of type 1, CT
CONFIGS["pet_mini4"] = dict(CONFIGS["pet_mini"], projector_type=4)
CONFIGS["pet_mini4_tof"] = dict(CONFIGS["pet_mini_tof"], projector_type=4)
CONFIGS["pet_half4"] = dict(CONFIGS["pet_mini"], projector_type=4, dL=0.5, subsets=3, subsetType=1)
CONFIGS["ct_mini4"] = dict(CONFIGS["ct_mini"], projector_type=4, subsets=3)


def apply(options, cfg):
    for k, v in cfg.items():
        setattr(options, k, v.copy() if isinstance(v, np.ndarray) else v)
    return options


# Arrays compared bit for bit against the reference after addProjector()
GEOMETRY_KEYS = ["x", "z", "index", "nMeas", "nMeasSubset", "nProjSubset", "nTotMeas", "dx", "dy", "dz", "bx", "by",
                 "bz", "segment_table", "x0"]
# projector scales of types 4 and 5 (coordinates.py:209-269), compared when present
SCALE_KEYS = ["dScaleX4", "dScaleY4", "dScaleZ4", "dSizeX", "dSizeY", "dScaleX", "dScaleY", "dScaleZ", "dSizeZBP",
              "dSizeXBP", "kerroin", "dL"]
SCALAR_KEYS = ["nRowsD", "nColsD", "nProjections", "NSinos", "TotSinos", "dPitchX", "dPitchY", "sigma_x", "PET",
               "TOF", "Nang", "Ndist"]
