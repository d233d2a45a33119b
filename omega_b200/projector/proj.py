"""Drop-in ``projectorClass`` for OMEGA's matrix-free projector path.

Mirrors ``omegatomo.projector.proj.projectorClass`` (omegatomo/projector/proj.py:36)
for the projector path: users set the same attributes, call ``addProjector()``
(proj.py:520) and ``initProj()`` (proj.py:1913), then project with
``forwardProject(f, subset)`` / ``backwardProject(y, subset)``
(proj.py:1923-1933) or the operator sugar ``A * f`` and ``A.T() * y``
(proj.py:1936-1951).  Inputs and outputs are flat float32 CUDA torch tensors
(image Fortran order, length Nx*Ny*Nz; measurements of one subset in
sinogram order, length nRowsD*nColsD*nProjSubset[k] times the TOF bins).

Differences from the reference surface:
 * every call is stream-ordered on ``torch.cuda.current_stream()``; nothing
   synchronises (the reference synchronises after each call,
   projfunctions.py:435-436) -- ``.cpu()`` or ``torch.cuda.synchronize()`` is
   the caller's sync point (projector type 5 synchronises after each call to
   read the staged kernels' error word unless ``checkDeviceErrors = False``);
 * ``use_64bit_atomics = True`` selects the bit-deterministic int64
   fixed-point backprojection on CUDA (the reference only offers it on
   OpenCL and forces it off on CUDA, init.py:251-254);
 * ``bddRayBackprojection = True`` (projector type 5) backprojects with the
   ray-driven scatter, the exact adjoint of the forward projection, instead
   of the reference's voxel-driven gather; ``bddRayBackprojection = 'int64'``
   takes the same scatter in int64 fixed point, bit-identical run to run
   (the reference clears ``use_64bit_atomics`` for CT types 4 and 5, whose
   gathers have no fixed-point form);
 * with TOF the forward projection returns all bins of the subset
   ([bin0 rays, bin1 rays, ...]); the reference's Python path sizes the output
   for one bin only.
The kernels run in the native library (``omega_b200/lib/libomega_b200.so``);
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from .. import _native
from . import geometry as geo


class projectorClass:
    # Image and FOV
    x = np.empty(0, dtype=np.float32)
    y = np.empty(0, dtype=np.float32)
    z = np.empty(0, dtype=np.float32)
    # index-based events: (source, detector) crystal indices into x (2 per
    # crystal) and ring indices into z, 2 x events each
    trIndex = np.empty(0, dtype=np.uint16)
    axIndex = np.empty(0, dtype=np.uint16)
    x0 = np.empty(0, dtype=np.float32)
    Nx = 1
    Ny = 1
    Nz = 1
    FOVa_x = 0.
    FOVa_y = 0.
    axial_fov = 0.
    oOffsetX = 0.
    oOffsetY = 0.
    oOffsetZ = 0.
    flip_image = False
    offangle = 0.
    # PET scanner
    cryst_per_block = np.empty(0, dtype=np.uint32)
    cryst_per_block_axial = cryst_per_block
    transaxial_multip = 1
    blocks_per_ring = 1
    linear_multip = 0
    diameter = 0.
    cr_p = 0.
    cr_pz = 0.
    DOI = 0.
    rings = 0
    det_per_ring = 0
    det_w_pseudo = 0
    detectors = 0
    pseudot = np.empty(0, dtype=np.uint32)
    ringGaps = np.empty(0, dtype=np.int32)
    nLayers = 1
    # Sinogram
    span = 3
    ring_difference = 0
    Ndist = 400
    Nang = 1
    NSinos = 1      # proj.py declares NSinos twice; the later default (1) wins
    TotSinos = 0
    segment_table = np.empty(0, dtype=np.float32)
    ndist_side = 1
    sampling = 1
    use_raw_data = 0
    arc_correction = False
    # CT / panel
    CT = False
    PET = False
    SPECT = False
    nProjections = 1
    nRowsD = 0
    nColsD = 0
    dPitchX = 0.
    dPitchY = 0.
    angles = np.empty(0, dtype=np.float32)
    sourceToCRot = 1.
    sourceToDetector = 1.
    sourceOffsetCol = np.zeros(1, dtype=np.float32)
    sourceOffsetRow = np.zeros(1, dtype=np.float32)
    detOffsetRow = np.zeros(1, dtype=np.float32)
    detOffsetCol = np.zeros(1, dtype=np.float32)
    bedOffset = np.empty(0, dtype=np.float32)
    pitchRoll = np.empty(0, dtype=np.float32)
    uV = np.empty(0, dtype=np.float32)
    nBed = 1
    flat = 0.
    pitch = False
    useHelical = False
    # TOF
    TOF = False
    TOF_bins = 1
    TOF_bins_used = 1
    TOF_FWHM = 0.
    TOF_width = 0.
    TOF_offset = 0.
    TOFCenter = np.empty(0, dtype=np.float32)
    sigma_x = 0.
    # Built-in reconstruction (reconstructions_main): the algorithms of this
    # path and their parameters (proj.py:116-120, 236, 271, 275, 317, 370-420)
    OSEM = False
    OSL_OSEM = False
    ROSEM = False
    RAMLA = False
    BSREM = False
    ROSEM_MAP = False
    PKMA = False
    MRAMLA = False
    MBSREM = False
    lambdaN = np.empty(0, dtype=np.float32)
    alpha_PKMA = np.empty(0, dtype=np.float32)
    rho_PKMA = .45
    delta_PKMA = 100.
    U = 0.
    precondTypeImage = np.full((7, 1), False)
    precondTypeMeas = np.full((2, 1), False)
    # image preconditioner options (proj.py:107, 276-279, 362-363, 439 of the
    # reference): type 2's reference image, type 3's per-sub-iteration values,
    # type 4's bounds and window; PKMA's automatic relaxation
    referenceImage = np.empty(0, dtype=np.float32)
    alphaPrecond = np.empty(0, dtype=np.float32)
    gradV1 = 0.5
    gradV2 = 2.5
    gradInitIter = 1
    gradLastIter = 1
    computeRelaxationParameters = False
    relaxationScaling = False
    # the filtering-based measurement (PDHG) and image preconditioners
    # (proj.py:104, 116, 123, 170-171, 269 of the reference): window, cut-off,
    # filtering sub-iterations, PDHG's step while filtering, the relaxation
    # while filtering
    filterWindow = "hamming"
    cutoffFrequency = 1.
    normalFilterSigma = 0.25
    filteringIterations = 0
    tauCPFilt = 0.
    lambdaFiltered = np.empty(0, dtype=np.float32)
    PDHG = False
    TV = False
    RDP = False
    RDP_gamma = 1.
    Quad = False
    Huber = False
    huber_delta = 1.
    # GGMRF prior (GGMRF_p / q / c below); hyperbolic prior (proj.py:361)
    GGMRF = False
    hyperbolic = False
    hyperbolicDelta = 1.
    # weighted-mean prior (proj.py:97, 160, 316)
    weighted_mean = False
    weighted_weights = np.empty(0, dtype=np.float32)
    weighted_center_weight = 2.
    mean_type = 4
    # median root prior (proj.py MRP, med_no_norm)
    MRP = False
    med_no_norm = False
    # non-local priors (proj.py:329-349, 434-436, 454)
    NLM = False
    NLTV = False
    NLRD = False
    NLLange = False
    NLGGMRF = False
    NLM_MRP = False
    NLM_use_anatomical = False
    NLAdaptive = False
    NLAdaptiveConstant = 1.
    NLM_referenceImage = np.empty(0, dtype=np.float32)
    NLMsigma = 1.
    NLM_gauss = 2.
    Nlx = 1
    Nly = 1
    Nlz = 1
    GGMRF_p = 0.
    GGMRF_q = 0.
    GGMRF_c = 0.
    Ndx = 1
    Ndy = 1
    Ndz = 1
    weights = np.empty(0, dtype=np.float32)
    MAP = False
    beta = 0.
    TVsmoothing = 1e-4
    # TV variants (proj.py:316-328, 410, 440-441 of the reference): TVtype 4
    # SATV and 6 weighted TV with SATVPhi; TV_use_anatomical with the
    # reference image TV_referenceImage, TVtype 1 (tensor, T), 2 (C) or 5
    # (eta); the APLS prior with APLS_ref_image, eta and APLSsmoothing
    TV_use_anatomical = False
    TVtype = 1
    C = 1.
    SATVPhi = 1.
    eta = 1e-5
    APLSsmoothing = 1e-5
    APLS = False
    APLS_ref_image = np.empty(0, dtype=np.float32)
    TV_referenceImage = np.empty(0, dtype=np.float32)
    # proximal TV with PDHG (proj.py:119, 274, 353, 415 of the reference):
    # the TV dual step, L2 or max-norm ball, forward / backward differences
    ProxTV = False
    sigma2CP = 1.
    useL2Ball = True
    derivativeType = 0
    # the anisotropic-diffusion prior (proj.py:325-326, 334, 340-341 of the
    # reference): flux 1 exponential / 2 quadratic, diffusion 1 gradient /
    # 2 modified curvature, iterations, time step, conductance
    AD = False
    # the L-filter and FMH priors (proj.py:95-96, 150-151 of the reference):
    # their weights, or empty for the prepass's (lfilter_weights.m,
    # fmhWeights.m); oneD_weights picks the L-filter's one-dimensional set
    L = False
    FMH = False
    a_L = np.empty(0, dtype=np.float32)
    fmh_weights = np.empty(0, dtype=np.float32)
    oneD_weights = False
    fmh_center_weight = 4.
    FluxType = 1
    DiffusionType = 2
    NiterAD = 1
    TimeStepAD = 1.
    KAD = 1.
    # TGV with PDHG (proj.py:351-352, 360, 411 of the reference): the
    # first- and second-order ball radii, 2-D TGV (no z component of v)
    TGV = False
    alpha0TGV = 0.
    alpha1TGV = 0.
    use2DTGV = False
    tauCP = 0.
    sigmaCP = 1.
    thetaCP = 1.
    powerIterations = 20
    enforcePositivity = True
    usingLinearizedData = False
    storeFP = False
    # PSF blur around the projections (proj.py:1885-1911, projfunctions.py:
    # 194-200, 1403-1407): FWHM (mm) in x, y (and z)
    use_psf = False
    FWHM = np.array([0., 0., 0.], dtype=np.float32)
    # Projector
    projector_type = 11
    n_rays_transaxial = 1
    n_rays_axial = 1
    # Projector types 2 / 3 (proj.py:195, 256-257, 369): the orthogonal
    # tracer's width (tube_width_z; tube_width_xy > 0 spreads it in the slice)
    # and the volume tracer's tube / voxel radii
    tube_width_xy = 0.
    tube_width_z = 0.
    tube_radius = 1.
    voxel_radius = 1.
    dL = 0
    # forward-projection image reads: 'fp32' (default) or 'bf16' (types 1 and
    # 4; FP32 accumulation), with BF16 copies reserved for maxFramesBF16 images
    imageReadPrecision = 'fp32'
    maxFramesBF16 = 1
    # projector scales (coordinates.py:209-269 fills those of the chosen type)
    dScaleX4 = np.empty(0, dtype=np.float32)
    dScaleY4 = np.empty(0, dtype=np.float32)
    dScaleZ4 = np.empty(0, dtype=np.float32)
    dSizeX = np.empty(0, dtype=np.float32)
    dSizeY = np.empty(0, dtype=np.float32)
    dScaleX = np.empty(0, dtype=np.float32)
    dScaleY = np.empty(0, dtype=np.float32)
    dScaleZ = np.empty(0, dtype=np.float32)
    dSizeZBP = 0.
    dSizeXBP = 0.
    kerroin = np.empty(0, dtype=np.float32)
    useTotLength = True
    useImages = True
    useMAD = True
    meanFP = False
    meanBP = False
    use_psf = False
    use_64bit_atomics = False
    use_32bit_atomics = False
    bddRayBackprojection = False
    # type 5: read the staged kernels' device error word after every
    # projection (a device synchronisation) and raise when a bounded wait ran
    # out; False leaves the calls asynchronous and the check to the caller
    # (omega_b200._native.check_device)
    checkDeviceErrors = True
    global_factor = 1.
    epps = 1e-5
    # Subsets / reconstruction
    subsets = 1
    subsetType = 8
    subset = 0
    seed = -1
    Niter = 4
    partitions = 1
    Nt = 1
    listmode = 0
    useIndexBasedReconstruction = False
    SinM = np.empty(0, dtype=np.float32)
    verbose = 1
    # PET corrections applied inside the projector type-1 kernels
    # (projectorType123.cl NORM / ATN / ATNM / SCATTER options):
    # normalization and corrVector are per-measurement multipliers, vaimennus
    # an attenuation image (1/mm, CTAttenuation) or per-measurement factors
    attenuation_correction = 0
    normalization_correction = 0
    randoms_correction = 0
    scatter_correction = 0
    additionalCorrection = 0
    CTAttenuation = True
    normalization = np.empty(0, dtype=np.float32)
    vaimennus = np.empty(0, dtype=np.float32)
    corrVector = np.empty(0, dtype=np.float32)
    # randoms (or additive scatter) added to the forward projection of the
    # OSEM sub-iterations (randoms_correction), one value per measurement
    SinDelayed = np.empty(0, dtype=np.float32)
    maskFP = np.empty(0, dtype=np.uint8)
    maskBP = np.empty(0, dtype=np.uint8)
    # Execution flags of the reference surface (accepted for compatibility)
    useTorch = True
    useCUDA = True
    useCuPy = False
    useAF = False
    useCPU = False
    deviceNum = 0
    largeDim = False
    nMultiVolumes = 0
    trans = False
    projectorAdded = False
    projectorInitialized = False

    def __init__(self):
        self._handle = None
        self._device = None

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None:
            try:
                _native.lib().omb_destroy(h)
            except Exception:
                pass
            self._handle = None

    # ------------------------------------------------------------------
    # Geometry (proj.py:520-1066)
    # ------------------------------------------------------------------
    def addProjector(self):
        """Validates the options and computes the detector coordinates,
        subset indices, voxel grid and projector scales (proj.py:520-1066)."""
        self.projectorAdded = True
        if hasattr(self, 'dPitch') and self.dPitch > 0 and self.dPitchX == 0.:
            self.dPitchX = self.dPitch
        if hasattr(self, 'dPitch') and self.dPitch > 0 and self.dPitchY == 0.:
            self.dPitchY = self.dPitch
        if self.CT:
            self._ct_setup()
        cpb_empty = isinstance(self.cryst_per_block_axial, np.ndarray) and self.cryst_per_block_axial.size == 0
        cpb_set = (isinstance(self.cryst_per_block, np.ndarray) and self.cryst_per_block.size > 0) or (
            not isinstance(self.cryst_per_block, np.ndarray) and self.cryst_per_block > 0)
        if cpb_empty and cpb_set:
            self.cryst_per_block_axial = self.cryst_per_block
        if self.rings == 0 and not isinstance(self.cryst_per_block_axial, np.ndarray) and \
                self.cryst_per_block_axial >= 1 and self.linear_multip >= 1:
            self.rings = self.cryst_per_block_axial * self.linear_multip
        if self.dPitchX > 0. and self.dPitchY == 0.:
            self.dPitchY = self.dPitchX
        if self.cr_p > 0. and self.cr_pz == 0.:
            self.cr_pz = self.cr_p
        if self.cr_p == 0. and self.dPitchX > 0.:
            self.cr_p = self.dPitchX
        if self.cr_pz == 0. and self.dPitchY > 0.:
            self.cr_pz = self.dPitchY
        if self.axial_fov == 0. and (self.cr_pz > 0. or self.dPitchY > 0.):
            self.axial_fov = self.dPitchY if self.dPitchY > 0. else self.cr_pz
        if self.det_per_ring == 0 and self.blocks_per_ring >= 1 and not isinstance(self.cryst_per_block, np.ndarray) \
                and self.cryst_per_block >= 1:
            self.det_per_ring = self.blocks_per_ring * self.cryst_per_block
        if self.det_w_pseudo == 0:
            self.det_w_pseudo = self.det_per_ring
        if self.detectors == 0:
            self.detectors = self.det_w_pseudo * self.rings
        if self.ring_difference == 0 and self.rings > 0:
            self.ring_difference = self.rings - 1
        if self.segment_table.size == 0 and self.span > 0 and self.rings > 0:
            self.segment_table = geo.default_segment_table(self.rings, self.span, self.ring_difference, self._n(self.Nz))
        if self.Nang == 1 and self.det_per_ring > 1:
            self.Nang = self.det_per_ring // 2
        if self.span == 1:
            self.TotSinos = self.rings ** 2
            self.NSinos = self.TotSinos
        elif self.NSinos == 0:
            self.NSinos = int(np.sum(self.segment_table))
        if self.TotSinos == 0:
            self.TotSinos = self.NSinos
        self.OMEGAErrorCheck()
        self.TOF = self.TOF_bins > 1 and self.projector_type in (1, 11, 3, 33, 13, 31, 4, 14, 41, 44, 34, 43)
        if self.TOF:
            if self.TOF_bins_used == 0 and self.TOF_bins > 0:
                self.TOF_bins_used = self.TOF_bins
            if self.TOF_bins_used != self.TOF_bins:
                self.sigma_x = 0.
            elif self.TOFCenter.size == 0:
                self.sigma_x = geo.tof_sigma(self.TOF_FWHM)
                self.TOFCenter = geo.tof_centers(self.TOF_width, self.TOF_bins, self.TOF_offset)
            else:
                self.TOFCenter = np.float32(self.TOFCenter)
        else:
            self.sigma_x = 0.
        if self.maskFP.size > 1 or self.maskBP.size > 1:
            raise ValueError('Forward/backward projection masks are not supported by this projector build')
        if isinstance(self.partitions, np.ndarray):
            if self.partitions.size >= 1:
                self.Nt = self.partitions.size
        else:
            self.Nt = self.partitions
        if self.Nt > 1 and self.subsetType == 3:
            raise ValueError('Subset type 3 is not supported with dynamic data!')
        self._listmode_setup()
        if (not self.CT and not self.SPECT) and (((self.subsetType > 7 or (self.subsetType == 0 and self.listmode == 0))
                                                   and self.subsets > 1) or self.subsets == 1):
            self.nProjections = self.NSinos
            self.PET = True
        else:
            self.PET = False
            self.nProjections = self.NSinos
        if self.listmode:
            self.index, self.nMeas = self._listmode_subsets()
        else:
            self.index, self.nMeas = geo.subset_indices(self)
        self.x0 = np.asarray(self.x0).ravel('F')
        if self.CT and self.projector_type == 11 and not self.useCPU:
            self.projector_type = 4
        if self.CT:
            x_det, z_det = self.x, self.z
        elif self.listmode:
            x_det, z_det = self._listmode_coordinates()
            self.nRowsD = self.nColsD = 1
            # events in the subsets (the random split of subset type 3 leaves one out, as the reference's)
            self.nProjections = int(np.sum(self.nMeas))
        else:
            x_det, z_det = geo.pet_sinogram_coordinates(self)
            self.dPitch = self.cr_p
            self.dPitchY = self.cr_p
            self.dPitchX = self.cr_pz
            self.nProjections = self.NSinos
            self.nRowsD = self.Ndist
            self.nColsD = self.Nang
        self.nMeas = np.insert(np.cumsum(self.nMeas), 0, 0)
        for nm in ('Nx', 'Ny', 'Nz'):
            if not isinstance(getattr(self, nm), np.ndarray):
                setattr(self, nm, np.array(getattr(self, nm), dtype=np.uint32, ndmin=1))
        self.dx, self.dy, self.dz, self.bx, self.by, self.bz = geo.voxel_grid(self)
        if self.subsetType >= 8 and self.subsets > 1:
            if self.CT:
                x_det = np.reshape(x_det, (self.nProjections, 6))[self.index, :].ravel('C')
                z_det = np.reshape(z_det, (self.nProjections, 2))[self.index, :].ravel('C')
                self.uV = self.uV[self.index, :]
            else:
                z_det = np.reshape(z_det, (self.nProjections, -1))[self.index, :].ravel('C')
        self.x = np.asarray(x_det).astype(dtype=np.float32)
        self.z = np.asarray(z_det).astype(dtype=np.float32)
        self._x_sinogram = self.x if not (self.CT or self.listmode) else None
        self.x_center = np.array(self.bx[0].item(), ndmin=1).astype(np.float32)
        self.y_center = np.array(self.by[0].item(), ndmin=1).astype(np.float32)
        self.z_center = np.array(self.bz[0].item(), ndmin=1).astype(np.float32)
        if self.projector_type in (4, 5, 14, 41, 15, 45, 54, 51, 42, 43, 24, 34):
            geo.projector_scaling(self)
        # tube spread of types 2 / 3 (proj.py:1041-1055) and the type-3 table (proj.py:990)
        if self.projector_type in (3, 33, 13, 31, 32, 23, 43, 34):
            self.orthTransaxial = self.orthAxial = True
        elif self.projector_type in (2, 22, 12, 21, 24, 42):
            self.orthTransaxial = self.tube_width_xy > 0 or self.SPECT
            self.orthAxial = self.tube_width_z > 0 or self.SPECT
        if self.projector_type in (3, 33, 13, 31, 34, 43):
            from .orth import voxel_volumes
            voxel_volumes(self)
        else:
            self.V = np.zeros(1, dtype=np.float32)
        self.PSFKernel()
        if self.nMeas.size == 1:
            self.nMeas = np.insert(self.nMeas, 0, 0)
        if self.subsets > 1:
            self.subset = 0
        kerroin = self.nColsD * self.nRowsD if (self.subsetType >= 8 or self.subsets == 1) else 1
        self.nMeasSubset = np.zeros((self.subsets, 1), dtype=np.int64)
        self.nProjSubset = np.zeros((self.subsets, 1), dtype=np.int64)
        self.nTotMeas = self.nMeas * kerroin
        for kk in range(self.subsets):
            self.nMeasSubset[kk] = self.nMeas[kk + 1] * kerroin - self.nMeas[kk] * kerroin
            self.nProjSubset[kk] = self.nMeas[kk + 1] - self.nMeas[kk]
        self.N = self.Nx.astype(np.uint64) * self.Ny.astype(np.uint64) * self.Nz.astype(np.uint64)
        for nm in ('FOVa_x', 'FOVa_y', 'axial_fov'):
            if not isinstance(getattr(self, nm), np.ndarray):
                setattr(self, nm, np.array(getattr(self, nm), dtype=np.float32, ndmin=1))
        if self.use_32bit_atomics and self.use_64bit_atomics:
            self.use_64bit_atomics = False
        self.x0 = self.x0.astype(dtype=np.float32)

    # ------------------------------------------------------------------
    # List-mode and index-based event data (proj.py:777-850, 862-905;
    # indices.py:79-160, 346-412)
    # ------------------------------------------------------------------
    def PSFKernel(self):
        """The Gaussian PSF window (proj.py:1885-1911): half-widths
        ceil(2 sigma / d) voxels per axis (no z blur with two FWHM values),
        exp(-sum x^2 / (2 sigma^2)) normalised to sum 1, float32, x fastest."""
        if not self.use_psf:
            return
        # Python floats (weak scalars): the window is computed in float32, as the reference's
        fw = [float(v) for v in np.ravel(self.FWHM)]
        k = 2. * math.sqrt(2. * math.log(2.))
        d = [float(np.ravel(v)[0]) for v in (self.dx, self.dy, self.dz)]
        g = [math.ceil(2. * (fw[i] / k) / d[i]) for i in range(2)]
        g.append(math.ceil(2. * (fw[2] / k) / d[2]) if len(fw) >= 3 else 0)
        ax = [np.linspace(-g[i] * d[i], g[i] * d[i], 2 * g[i] + 1, dtype=np.float32) for i in range(2)]
        X = ax[0].reshape(-1, 1, 1)
        Y = ax[1].reshape(1, -1, 1)
        sx, sy = fw[0] / k, fw[1] / k
        if len(fw) >= 3:
            Z = np.linspace(-g[2] * d[2], g[2] * d[2], 2 * g[2] + 1, dtype=np.float32).reshape(1, 1, -1)
            gk = np.exp(-(X ** 2 / (2. * sx ** 2) + Y ** 2 / (2. * sy ** 2) + Z ** 2 / (2. * (fw[2] / k) ** 2)))
        else:
            gk = np.exp(-(X ** 2 / (2. * sx ** 2) + Y ** 2 / (2. * sy ** 2)))
        self.gaussK = np.asfortranarray((gk / np.sum(gk)).astype(np.float32))
        self.g_dim_x, self.g_dim_y, self.g_dim_z = g

    def _psf(self, f):
        """f blurred by the PSF window (a new device tensor)."""
        import torch
        if getattr(self, '_d_psf', None) is None or self._d_psf.device != f.device:
            self._d_psf = torch.from_numpy(np.ascontiguousarray(np.ravel(self.gaussK, order='F'),
                                                                dtype=np.float32)).to(f.device)
        out = torch.empty_like(f)
        nx, ny, nz = self._n(self.Nx), self._n(self.Ny), self._n(self.Nz)
        _native.call("omb_psf_convolve", ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(out.data_ptr()), nx, ny,
                     nz, ctypes.c_void_p(self._d_psf.data_ptr()), int(self.g_dim_x), int(self.g_dim_y),
                     int(self.g_dim_z), ctypes.c_void_p(torch.cuda.current_stream(f.device).cuda_stream))
        return out

    def _listmode_setup(self):
        """Detects event data: 6 coordinates per event in ``x`` (or ``x``,
        ``y``, ``z`` of 2 rows each), or detector index pairs ``trIndex`` /
        ``axIndex`` with ``useIndexBasedReconstruction``; each event is then
        one 1 x 1 "sinogram"."""
        self.listmode = 0
        if self.CT or self.SPECT or self.x is getattr(self, '_x_sinogram', None):
            return  # (the sinogram coordinates of an earlier addProjector are not events)
        if self.useIndexBasedReconstruction:
            n_events = np.size(self.trIndex) // 2
        else:
            x = np.asarray(self.x)
            nx = x.size
            sin_n = np.size(self.SinM)
            if nx == 0 or not (nx // 6 == sin_n and nx % 6 == 0 or nx // 2 == sin_n and x.ndim == 2 or
                               (sin_n == 0 and nx >= 6)):
                return
            if x.ndim == 2 and 2 in x.shape and np.size(self.y) == nx:
                # separate x, y, z of (source, detector): stack into 6 rows
                two = (lambda a: np.asarray(a).reshape(2, -1) if np.asarray(a).shape[0] == 2 else np.asarray(a).T)
                xx, yy, zz = two(self.x), two(self.y), two(self.z)
                self.x = np.vstack([xx[0], yy[0], zz[0], xx[1], yy[1], zz[1]])
            n_events = np.size(self.x) // 6
        if self.TOF_bins > 1:
            raise ValueError('TOF list-mode data is not supported by this projector build')
        self.Nang = 1
        self.Ndist = 1
        self.NSinos = int(n_events)
        self.TotSinos = self.NSinos
        self.listmode = 1

    def _listmode_subsets(self):
        """Subset indices of event data: type 0 contiguous blocks, 1 every
        subsets-th event, 3 a seeded random split (indices.py:79-160)."""
        n, S = int(self.NSinos), int(self.subsets)
        if S == 1:
            return np.zeros(1, dtype=np.uint32), np.array([n], dtype=np.int64)
        if self.subsetType not in (0, 1, 3):
            self.subsetType = 0
        if self.subsetType == 0:
            val = n // S
            last = n - val * (S - 1) if n % S > 0 else val
            return np.zeros(1, dtype=np.uint32), np.append(np.full(S - 1, val, dtype=np.int64), last)
        if self.subsetType == 1:
            parts = [np.arange(i, n, S, dtype=np.uint32) for i in range(S)]
        else:
            port = n // S
            gen = np.random.default_rng() if self.seed < 0 else np.random.default_rng(self.seed)
            perm = gen.permutation(n).astype(np.uint32)
            parts = [perm[port * i:-1] if i == S - 1 else perm[port * i:port * (i + 1)] for i in range(S)]
        return np.concatenate(parts), np.array([p.size for p in parts], dtype=np.int64)

    def _listmode_coordinates(self):
        """Event coordinates in subset order (indices.py:346-412): the 6 x
        events matrix, or (index-based) the crystal table and z with the
        index pairs reordered."""
        sub = self.subsets > 1 and self.subsetType > 0
        if self.useIndexBasedReconstruction:
            tr = np.asarray(self.trIndex, dtype=np.uint16).reshape(2, -1, order='F')
            ax = np.asarray(self.axIndex, dtype=np.uint16).reshape(2, -1, order='F')
            if sub:
                tr, ax = tr[:, self.index], ax[:, self.index]
            self.trIndex = np.asfortranarray(tr).ravel(order='F')
            self.axIndex = np.asfortranarray(ax).ravel(order='F')
            return np.asarray(self.x, dtype=np.float32).ravel(order='F'), \
                np.asarray(self.z, dtype=np.float32).ravel(order='F')
        x = np.asarray(self.x, dtype=np.float32)
        x = x.reshape(6, -1, order='F') if x.shape[0] != 6 else x
        if sub:
            x = x[:, self.index]
        return np.asfortranarray(x).ravel(order='F'), np.zeros(0, dtype=np.float32)

    @staticmethod
    def _n(v):
        return int(np.asarray(v).ravel()[0])

    def _ct_setup(self):
        """CT branch of addProjector (proj.py:528-568) and setCTCoordinates."""
        if not hasattr(self, 'nProjections') or self.nProjections == 0:
            self.nProjections = self.NSinos
        else:
            self.NSinos = self.nProjections
        self.NSinos = self.nProjections
        self.TotSinos = self.nProjections
        self.span = 3
        if self.nRowsD == 0:
            self.nRowsD = self.Ndist
        else:
            self.Ndist = self.nRowsD
        if self.nColsD == 0:
            self.nColsD = self.Nang
        else:
            self.Nang = self.nColsD
        self.use_raw_data = 0
        self.attenuation_correction = 0
        self.normalization_correction = 0
        self.rings = self.nColsD * self.nBed
        self.det_per_ring = self.nRowsD * self.nProjections
        self.arc_correction = False
        self.det_w_pseudo = self.det_per_ring
        self.cryst_per_block = self.nColsD * self.nRowsD
        if hasattr(self, 'dPitch') and self.dPitch > 0:
            self.cr_pz = self.dPitch
            self.cr_p = self.dPitch
        else:
            self.cr_pz = self.dPitchY
            self.cr_p = self.dPitchX
        self.angles = np.asarray(self.angles)
        if np.max(np.abs(self.angles.flatten())) > 6. * np.pi:
            self.angles = self.angles * (np.pi / 180.)
        if self.offangle > 0:
            self.angles = self.angles + self.offangle
        if self.subsets > 1 and 0 < self.subsetType < 8:
            raise ValueError('Subset types < 8 with CT data are not yet supported in Python! Use custom detector '
                             'coordinates instead or subset types >= 8.')
        if self.pitchRoll.size > 0 or self.useHelical or self.bedOffset.size > 0:
            raise ValueError('pitch/roll, helical and multi-bed CT geometries are not supported by this build')
        self.x, self.z, self.uV = geo.ct_source_detector(self)

    def OMEGAErrorCheck(self):
        """Option checks of the projector path (proj.py:1068-1283); the same
        conditions raise ValueError with the reference's messages."""
        if self.FOVa_x > 0 and self.FOVa_y == 0:
            self.FOVa_y = self.FOVa_x
        if not self.CT and not self.SPECT and self.span > self.ring_difference and self.NSinos > 1 and not self.use_raw_data:
            raise ValueError(f"Span value cannot be larger than ring difference ({self.ring_difference})!")
        if not self.CT and not self.SPECT and (self.span % 2 == 0 or self.span <= 0) and not self.use_raw_data:
            raise ValueError("Span value has to be odd and positive!")
        if not self.CT and not self.SPECT and self.ring_difference >= self.rings and not self.use_raw_data and self.rings > 0:
            self.ring_difference = self.rings - 1
        if not self.CT and not self.SPECT and self.ring_difference < 0 and not self.use_raw_data:
            raise ValueError("Ring difference has to be at least 0!")
        if not self.CT and not self.SPECT and self.Nang > self.det_w_pseudo / 2 and not self.use_raw_data and self.Nang > 1:
            raise ValueError(f"Number of sinogram angles can be at most the number of detectors per ring divided by two ({self.det_w_pseudo / 2})!")
        if not self.CT and not self.SPECT and self.TotSinos < self.NSinos and not self.use_raw_data and self.TotSinos > 0:
            self.TotSinos = self.NSinos
        if not self.CT and not self.SPECT and (self.ndist_side > 1 and self.Ndist % 2 == 0 or self.ndist_side < -1 and self.Ndist % 2 == 0) and not self.use_raw_data:
            raise ValueError("ndist_side can be either 1 or -1!")
        if not self.CT and not self.SPECT and self.ndist_side == 0 and self.Ndist % 2 == 0 and not self.use_raw_data:
            raise ValueError("ndist_side cannot be 0 when Ndist is even!")
        if self.Niter < 1:
            self.Niter = 1
        if self.subsets < 1:
            self.subsets = 1
        if self.projector_type not in [1, 2, 3, 4, 5, 6, 11, 14, 12, 13, 21, 22, 23, 24, 31, 32, 33, 34, 41, 42, 43,
                                       44, 45, 51, 15, 54, 55]:
            raise ValueError('The selected projector type is not supported!')
        if self.epps <= 0:
            self.epps = 1e-6
        if self.projector_type in [5, 15, 51, 45, 54] and not self.CT:
            raise ValueError('Projector type 5 is only supported with CT data!')
        if self.useCUDA and self.useCPU:
            raise ValueError('Both CUDA and CPU selected! Select only one!')
        if self.TOF_bins_used > 1 and (self.projector_type not in [1, 11, 3, 33, 31, 13, 4, 41, 14, 43, 34]) and not self.CT and not self.SPECT:
            raise ValueError('TOF is currently only supported with improved Siddon (projector_type = 1), interpolation-based projector (projector_type = 4) and volume of intersection (projector_type = 3)')
        if self.TOF_bins_used > 1 and self.TOF_width <= 0 and not self.CT and not self.SPECT:
            raise ValueError('TOF width (self.TOF_width) must be greater than zero.')
        if self.TOF_bins_used > 1 and self.TOF_FWHM == 0 and not self.CT and not self.SPECT:
            raise ValueError('TOF enabled, but the TOF FWHM (self.TOF_FWHM) is zero. FWHM must be nonzero.')
        if not self.largeDim and not np.asarray(self.x0).any():
            fill = 1e-4 if self.CT else 1.
            self.x0 = np.ones((self._n(self.Nx), self._n(self.Ny), self._n(self.Nz)), dtype=np.float32, order='F') * fill
        if not self.largeDim and np.asarray(self.x0).size < self._n(self.Nx) * self._n(self.Ny) * self._n(self.Nz):
            raise ValueError(f"Initial value has a matrix size smaller ({np.prod(np.shape(self.x0))}) than the actual image size ({self._n(self.Nx)*self._n(self.Ny)*self._n(self.Nz)})!")

    # ------------------------------------------------------------------
    # Device set-up (init.py:39-703)
    # ------------------------------------------------------------------
    def _fp_bp_types(self):
        pt = self.projector_type
        fp = {1: 1, 11: 1, 14: 1, 15: 1, 12: 1, 13: 1, 4: 4, 41: 4, 42: 4, 43: 4, 44: 4, 45: 4,
              5: 5, 51: 5, 52: 5, 53: 5, 54: 5, 55: 5,
              2: 2, 22: 2, 21: 2, 24: 2, 3: 3, 33: 3, 31: 3, 34: 3}.get(pt)
        bp = {1: 1, 11: 1, 21: 1, 31: 1, 41: 1, 51: 1, 4: 4, 14: 4, 24: 4, 34: 4, 44: 4, 54: 4,
              5: 5, 15: 5, 25: 5, 35: 5, 45: 5, 55: 5,
              2: 2, 22: 2, 12: 2, 42: 2, 3: 3, 33: 3, 13: 3, 43: 3}.get(pt)
        if fp is None or bp is None:
            raise ValueError(f'Projector type {pt} is not supported by this build')
        return fp, bp

    def _descriptor(self):
        fpt, bpt = self._fp_bp_types()
        self.FPType, self.BPType = fpt, bpt
        d = _native.GeometryDesc()
        d.struct_size = ctypes.sizeof(_native.GeometryDesc)
        d.abi_version = _native.OMB_ABI_VERSION
        if self.CT:
            d.modality = _native.OMB_CT_PANEL
        elif self.listmode:
            d.modality = _native.OMB_PET_INDEXED if self.useIndexBasedReconstruction else _native.OMB_PET_LISTMODE
        else:
            d.modality = _native.OMB_PET_SINOGRAM
        d.fp_type, d.bp_type = fpt, bpt
        d.nx, d.ny, d.nz = self._n(self.Nx), self._n(self.Ny), self._n(self.Nz)
        d.dx, d.dy, d.dz = float(self.dx[0]), float(self.dy[0]), float(self.dz[0])
        d.bx, d.by, d.bz = float(self.bx[0]), float(self.by[0]), float(self.bz[0])
        d.n_rows_d, d.n_cols_d = int(self.nRowsD), int(self.nColsD)
        d.n_proj = int(self.nProjections)
        d.n_subsets = int(self.subsets)
        d.subset_type = int(self.subsetType)
        keep = {}
        keep['n_meas'] = np.ascontiguousarray(np.asarray(self.nMeas, dtype=np.int64).ravel())
        keep['xy'] = np.ascontiguousarray(np.asarray(self.x, dtype=np.float32).ravel())
        keep['z'] = np.ascontiguousarray(np.asarray(self.z, dtype=np.float32).ravel())
        d.n_meas = _native.i64_ptr(keep['n_meas'])
        d.xy = _native.f32_ptr(keep['xy'])
        d.n_xy = keep['xy'].size
        d.z = _native.f32_ptr(keep['z'])
        d.n_z = keep['z'].size
        d.dpitch_x, d.dpitch_y = float(self.dPitchX), float(self.dPitchY)
        d.global_factor = float(self.global_factor)
        d.epps = float(self.epps)
        nb = int(self.TOF_bins_used) if self.TOF else 1
        d.tof_bins = nb
        d.sigma_x = float(self.sigma_x)
        if self.TOF:
            keep['tof'] = np.ascontiguousarray(np.asarray(self.TOFCenter, dtype=np.float32).ravel())
            d.tof_centers = _native.f32_ptr(keep['tof'])
        d.dL = float(self.dL)
        if fpt == 4 or bpt == 4:
            d.d_scale4[0], d.d_scale4[1], d.d_scale4[2] = (float(np.ravel(self.dScaleX4)[0]),
                                                           float(np.ravel(self.dScaleY4)[0]),
                                                           float(np.ravel(self.dScaleZ4)[0]))
            d.kerroin = float(np.ravel(self.kerroin)[0])
        if fpt == 5 or bpt == 5:
            d.d_size5[0], d.d_size5[1] = float(self.dSizeX[0]), float(self.dSizeY[0])
            d.d_scale5[0], d.d_scale5[1], d.d_scale5[2] = (float(self.dScaleX[0]), float(self.dScaleY[0]),
                                                           float(self.dScaleZ[0]))
        d.fixed64_workspace = 1 if (self.use_64bit_atomics or self.bddRayBackprojection == 'int64') else 0
        if not self.CT:
            d.n_rays_xy = int(self.n_rays_transaxial)
            d.n_rays_z = int(self.n_rays_axial)
        if 2 in (fpt, bpt) or 3 in (fpt, bpt):
            d.tube_width = float(self.tube_width_z)
            d.tube_radius = float(self.tube_radius)
            d.orth_xy = 1 if self.orthTransaxial else 0
            d.orth_z = 1 if self.orthAxial else 0
            if 3 in (fpt, bpt):
                keep['vol'] = np.ascontiguousarray(np.asarray(self.V, dtype=np.float32).ravel())
                d.vol_v = _native.f32_ptr(keep['vol'])
                d.n_vol_v = keep['vol'].size
                d.vol_bmin, d.vol_bmax, d.vol_vmax = float(self.bmin), float(self.bmax), float(self.Vmax)
        if self.listmode and self.useIndexBasedReconstruction:
            keep['tr'] = np.ascontiguousarray(np.asarray(self.trIndex, dtype=np.uint16).ravel())
            keep['ax'] = np.ascontiguousarray(np.asarray(self.axIndex, dtype=np.uint16).ravel())
            d.tr_index = keep['tr'].ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))
            d.ax_index = keep['ax'].ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))
        return d, keep

    def initProj(self):
        """Uploads the geometry to the current CUDA device and reorders the
        measurement data into subset order (init.py:39-703; parseInputs
        prepass.py:256-355)."""
        if not self.projectorAdded:
            self.addProjector()
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError('omega_b200 projectors need a CUDA device')
        self.projectorInitialized = True
        if self.TOF_bins_used == 0:
            self.TOF_bins_used = 1
        self._parse_inputs()
        desc, keep = self._descriptor()
        h = ctypes.c_void_p()
        _native.call("omb_create", ctypes.byref(desc), ctypes.byref(h))
        if self._handle is not None:
            _native.lib().omb_destroy(self._handle)
        self._handle = h
        self._device = torch.cuda.current_device()
        if self.imageReadPrecision not in ('fp32', 'bf16'):
            raise ValueError("imageReadPrecision must be 'fp32' or 'bf16'")
        if self.imageReadPrecision == 'bf16':
            _native.call("omb_set_read_precision", h, _native.OMB_READ_BF16, int(self.maxFramesBF16))
        self._set_corrections()
        del keep

    def _measurement_vectors(self):
        """The per-measurement correction vectors in use (name -> array)."""
        out = {}
        if self.normalization_correction:
            out['normalization'] = self.normalization
        if self.attenuation_correction and not self.CTAttenuation:
            out['vaimennus'] = self.vaimennus
        if self.additionalCorrection:
            out['corrVector'] = self.corrVector
        return out

    def _set_corrections(self):
        """Uploads the PET corrections: the product of the per-measurement
        multipliers (in subset order), the attenuation image and the randoms."""
        total = int(np.ravel(self.nTotMeas)[-1])
        if self.randoms_correction and not self.CT:
            r = np.ascontiguousarray(np.asarray(self.SinDelayed, dtype=np.float32).ravel(order='F'))
            if r.size != total:
                raise ValueError(f'SinDelayed must hold one value per measurement ({total}), got {r.size}')
            _native.call("omb_set_randoms", self._handle, r.ctypes.data_as(ctypes.c_void_p), r.size, None)
        if self.CT or not (self.normalization_correction or self.attenuation_correction or self.additionalCorrection):
            return
        w = None
        for name, v in self._measurement_vectors().items():
            v = np.asarray(v, dtype=np.float64).ravel(order='F')
            if v.size != total:
                raise ValueError(f'{name} must hold one value per measurement ({total}), got {v.size}')
            w = v if w is None else w * v
        mu = None
        if self.attenuation_correction and self.CTAttenuation:
            mu = np.asarray(self.vaimennus, dtype=np.float32).ravel(order='F')
            n_img = int(np.ravel(self.N)[0])
            if mu.size != n_img:
                raise ValueError(f'vaimennus must be an image of {n_img} voxels, got {mu.size}')
        keep = []

        def ptr(a):
            if a is None:
                return None, 0
            a = np.ascontiguousarray(a, dtype=np.float32)
            keep.append(a)
            return a.ctypes.data_as(ctypes.c_void_p), a.size

        wp, nw = ptr(w)
        mp, nm = ptr(mu)
        _native.call("omb_set_corrections", self._handle, wp, nw, mp, nm, None)
        del keep

    def _parse_inputs(self):
        """Reorders SinM and the per-measurement correction vectors into subset
        order (prepass.py:282-472, static data)."""
        if not (self.subsets > 1 and self.subsetType > 0):
            return
        if not getattr(self, '_corrections_ordered', False):
            vecs = dict(self._measurement_vectors())
            if self.randoms_correction:
                vecs['SinDelayed'] = self.SinDelayed
            for name, v in vecs.items():
                v = np.asarray(v, dtype=np.float32).ravel(order='F')
                if self.subsetType >= 8:
                    v = np.reshape(v, (self.nRowsD, self.nColsD, self.nProjections), order='F')[:, :, self.index]
                    v = v.ravel(order='F')
                elif v.size == np.size(self.index):
                    v = v[self.index]
                setattr(self, name, v)
            self._corrections_ordered = True
        if self.SinM.size == 0:
            return
        if self.Nt > 1:
            raise ValueError('dynamic data: reorder each frame with subsetMeasurements()')
        nb = int(self.TOF_bins_used) if self.TOF else 1
        if self.subsetType >= 8:
            s = np.reshape(self.SinM, (self.nRowsD, self.nColsD, self.nProjections, nb), order='F')
            s = s[:, :, self.index, :]
            self.SinM = s if self.TOF else s[:, :, :, 0]
        else:
            if self.TOF:
                s = np.reshape(self.SinM, (self.SinM.size // nb, nb), order='F')
                self.SinM = s[self.index, :]
            else:
                self.SinM = self.SinM.ravel(order='F')[self.index]

    def subsetMeasurements(self, m, subset):
        """Measurements of one subset from the subset-ordered flat vector
        ``m = SinM.ravel('F')`` in the layout the projector expects
        (all TOF bins of the subset: [bin0 rays, bin1 rays, ...])."""
        lo, hi = int(self.nTotMeas[subset]), int(self.nTotMeas[subset + 1])
        if not self.TOF:
            return m[lo:hi]
        per_bin = int(self.nTotMeas[-1])
        parts = [m[b * per_bin + lo:b * per_bin + hi] for b in range(int(self.TOF_bins_used))]
        import torch
        return torch.cat(parts) if isinstance(m, torch.Tensor) else np.concatenate(parts)

    # ------------------------------------------------------------------
    # Projections (projfunctions.py:86-1407)
    # ------------------------------------------------------------------
    def _check_ready(self):
        if not self.projectorInitialized or self._handle is None:
            self.initProj()

    def _as_device(self, a, n, what):
        import torch
        if isinstance(a, np.ndarray):
            a = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32).ravel()).cuda(self._device)
        if not isinstance(a, torch.Tensor):
            raise TypeError(f'{what} must be a torch tensor or a NumPy array')
        if not a.is_cuda:
            a = a.cuda(self._device)
        if a.dtype != torch.float32:
            a = a.float()
        a = a.reshape(-1)
        if not a.is_contiguous():
            a = a.contiguous()
        if a.numel() != n:
            raise ValueError(f'{what} has {a.numel()} elements, expected {n}')
        return a

    def measurementCount(self, subset):
        """Measurements (all TOF bins) of one subset, or of all with -1."""
        self._check_ready()
        m = int(_native.lib().omb_measurement_count(self._handle, int(subset)))
        if m < 0:
            _native.check("omb_measurement_count", -1)
        return m

    def forwardProject(self, f, subset=-1):
        """y = A_subset f (projfunctions.py:86)."""
        self._check_ready()
        import torch
        if subset == -1:
            subset = self.subset
        f = self._as_device(f, int(self.N[0]), 'image')
        if self.use_psf:
            f = self._psf(f)
        m = self.measurementCount(subset)
        y = torch.empty(m, dtype=torch.float32, device=f.device)
        stream = torch.cuda.current_stream(f.device).cuda_stream
        _native.call("omb_forward", self._handle, int(subset), ctypes.c_void_p(f.data_ptr()),
                     ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(stream))
        self._check_staged("omb_forward")
        return y

    def _check_staged(self, what):
        if int(np.ravel(self.projector_type)[0]) == 5 and self.checkDeviceErrors:
            _native.check_device(what)

    def backwardProject(self, y, subset=-1, sens=False):
        """f = A_subset^T y (projfunctions.py:735).  With ``sens=True`` also
        returns A_subset^T 1 (the reference's no_norm == 0 pass)."""
        self._check_ready()
        import torch
        if subset == -1:
            subset = self.subset
        m = self.measurementCount(subset)
        y = self._as_device(y, m, 'measurement')
        n = int(self.N[0])
        f = torch.empty(n, dtype=torch.float32, device=y.device)
        s = torch.empty(n, dtype=torch.float32, device=y.device) if sens else None
        stream = torch.cuda.current_stream(y.device).cuda_stream
        ray = self.bddRayBackprojection
        mode = _native.OMB_BP_FIXED64 if (self.use_64bit_atomics or ray == 'int64') else (
            _native.OMB_BP_RAY if ray else _native.OMB_BP_FLOAT_ATOMIC)
        _native.call("omb_backward", self._handle, int(subset), ctypes.c_void_p(y.data_ptr()),
                     ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(s.data_ptr() if s is not None else 0),
                     int(mode), ctypes.c_void_p(stream))
        self._check_staged("omb_backward")
        if self.use_psf:
            f = self._psf(f)
            s = self._psf(s) if sens else None
        return (f, s) if sens else f

    @property
    def tuning(self):
        """Launch shapes of this object's projector kernels (a dict)."""
        self._check_ready()
        t = _native.Tuning(struct_size=ctypes.sizeof(_native.Tuning))
        _native.call("omb_get_tuning", self._handle, ctypes.byref(t))
        return t.as_dict()

    @tuning.setter
    def tuning(self, values):
        self._check_ready()
        t = _native.Tuning(struct_size=ctypes.sizeof(_native.Tuning))
        _native.call("omb_get_tuning", self._handle, ctypes.byref(t))
        for k, v in dict(values).items():
            if k not in t.as_dict():
                raise KeyError(f"unknown tuning key {k!r}")
            setattr(t, k, int(v))
        _native.call("omb_set_tuning", self._handle, ctypes.byref(t))

    def autotune(self, n_frames=1, repeats=3):
        """Times the candidate launch shapes of the forward and backward
        projectors on this geometry (all subsets, n_frames images at once),
        keeps the fastest and returns them.  Synchronises the device."""
        self._check_ready()
        import torch
        dev = torch.device("cuda", self._device)
        t = _native.Tuning(struct_size=ctypes.sizeof(_native.Tuning))
        _native.call("omb_autotune", self._handle, int(n_frames), int(repeats), ctypes.byref(t),
                     ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
        return t.as_dict()

    def T(self):
        self.trans = True
        return self

    def __mul__(self, B):
        if self.trans:
            self.trans = False
            return self.backwardProject(B, self.subset)
        return self.forwardProject(B, self.subset)

    def __imul__(self, B):
        return self.__mul__(B)

    def __rmul__(self, B):
        return self

    def __truediv__(self, B):
        return self
