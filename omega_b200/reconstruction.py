"""Subset-update loops driven by the projectors: OSEM (PET) and PDHG with a
TV-gradient term (CT), plus the power method for the PDHG step size; the
built-in entry adds OSL-OSEM and the relaxed ROSEM / RAMLA / BSREM /
ROSEM-MAP (PET).

These are the loops of OMEGA's compiled reconstruction (reconstructionAF.h:
1053-1500) for the two algorithms on this path, run on the device through
the C-ABI with one host call per sub-iteration (or one CUDA-graph replay per
iteration).  All buffers are float32 CUDA torch tensors; nothing here
synchronises except the power method (which returns a host scalar).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(dev):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def power_method(options, n_iter=None, seed=0):
    """Largest eigenvalue of A^T A (options.powerIterations iterations by
    default, 20 in the reference; functions.hpp:2417-2540)."""
    import torch
    options._check_ready()
    n_iter = int(n_iter if n_iter is not None else getattr(options, "powerIterations", 20))
    dev = torch.device("cuda", options._device)
    n = int(options.N[0])
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.randn(n, generator=g).abs()
    x = (x / x.norm()).to(dev)
    wm = torch.empty(options.measurementCount(-1), device=dev)
    wi = torch.empty(n, device=dev)
    work = torch.empty(int(_native.lib().omb_power_workspace_bytes()) // 8 + 1, dtype=torch.float64, device=dev)
    L = ctypes.c_double()
    _native.call("omb_power_method", options._handle, n_iter, _ptr(x), _ptr(wm), _ptr(wi), _ptr(work),
                 ctypes.byref(L), _stream(dev))
    return L.value


class PDHG:
    """PDHG with the smoothed TV gradient (options.PDHG with options.TV in the
    reference), one subset.  Step sizes follow the reference: tau = 1/L from
    the power method, sigma = 1, theta = 1 (functions.hpp:2886-2905)."""

    def __init__(self, options, y, beta, tv_smooth=None, tau=None, sigma=1.0, theta=1.0, x0=None,
                 positivity=True):
        import torch
        options._check_ready()
        self.o = options
        self.dev = torch.device("cuda", options._device)
        n = int(options.N[0])
        m = options.measurementCount(-1)
        self.y = options._as_device(y, m, "measurement")
        if x0 is None:
            x0 = np.asarray(options.x0, dtype=np.float32)
        self.x = options._as_device(x0, n, "initial image").clone()
        self.x_next = torch.empty_like(self.x)
        self.u = self.x.clone()
        self.p = torch.zeros(m, device=self.dev)
        self.wm = torch.empty(m, device=self.dev)
        self.wi = torch.empty(n, device=self.dev)
        self.beta = float(beta)
        self.smooth = float(tv_smooth if tv_smooth is not None else getattr(options, "TVsmoothing", 1e-4))
        self.tau = float(tau) if tau is not None else 1.0 / power_method(options)
        self.sigma, self.theta = float(sigma), float(theta)
        self.positivity = 1 if positivity else 0
        self.graph = None

    def _step(self, x, x_next):
        _native.call("omb_pdhg_iteration", self.o._handle, _ptr(x), _ptr(x_next), _ptr(self.u), _ptr(self.p),
                     _ptr(self.y), self.tau, self.sigma, self.theta, self.beta, self.smooth, self.positivity,
                     _ptr(self.wm), _ptr(self.wi), _stream(self.dev))

    def iterate(self, n_iter, use_graph=False):
        """Runs n_iter iterations; returns the current image (a view)."""
        import torch
        if not use_graph or (self.graph is None and n_iter < 2):
            for _ in range(n_iter):
                self._step(self.x, self.x_next)
                self.x, self.x_next = self.x_next, self.x
            self.o._check_staged("PDHG.iterate")
            return self.x
        if self.graph is None:
            # one graph holds two iterations (x -> x_next -> x), so the
            # buffers are back in place after every replay
            s = torch.cuda.Stream(self.dev)
            s.wait_stream(torch.cuda.current_stream(self.dev))
            with torch.cuda.stream(s):
                self._step(self.x, self.x_next)  # warm-up outside the capture
                self._step(self.x_next, self.x)
            torch.cuda.current_stream(self.dev).wait_stream(s)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._step(self.x, self.x_next)
                self._step(self.x_next, self.x)
            n_iter -= 2
        for _ in range(n_iter // 2):
            self.graph.replay()
        if n_iter % 2:
            self._step(self.x, self.x_next)
            self.x, self.x_next = self.x_next, self.x
        self.o._check_staged("PDHG.iterate")
        return self.x


class OSEM:
    """OSEM for PET sinograms (options.OSEM in the reference): per-subset
    sensitivity images in the first pass, then the EM update per subset
    (computeForwardProject.h:76-101, algorithms.h:12-15)."""

    def __init__(self, options, m, x0=None):
        import torch
        options._check_ready()
        self.o = options
        self.dev = torch.device("cuda", options._device)
        n = int(options.N[0])
        S = int(options.subsets)
        if x0 is None:
            x0 = np.asarray(options.x0, dtype=np.float32)
        self.x = options._as_device(x0, n, "initial image").clone()
        self.y = [options._as_device(options.subsetMeasurements(m, s), options.measurementCount(s), "measurement")
                  for s in range(S)]
        self.sens = [torch.empty(n, device=self.dev) for _ in range(S)]
        for s in range(S):
            _native.call("omb_sensitivity", options._handle, s, _ptr(self.sens[s]), _stream(self.dev))
        self.wm = torch.empty(max(options.measurementCount(s) for s in range(S)), device=self.dev)
        self.wi = torch.empty(n, device=self.dev)
        self.graph = None

    def _iteration(self):
        st = _stream(self.dev)
        for s in range(int(self.o.subsets)):
            _native.call("omb_osem_subset", self.o._handle, s, _ptr(self.x), _ptr(self.y[s]), _ptr(self.sens[s]),
                         _ptr(self.wm), _ptr(self.wi), st)

    def iterate(self, n_iter, use_graph=False):
        import torch
        if not use_graph or (self.graph is None and n_iter < 1):
            for _ in range(n_iter):
                self._iteration()
            return self.x
        if self.graph is None:
            s = torch.cuda.Stream(self.dev)
            s.wait_stream(torch.cuda.current_stream(self.dev))
            with torch.cuda.stream(s):
                self._iteration()
            torch.cuda.current_stream(self.dev).wait_stream(s)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._iteration()
            n_iter -= 1
        for _ in range(n_iter):
            self.graph.replay()
        return self.x


class OSEMBatch:
    """OSEM for a batch of studies (or frames) that share one PET geometry:
    every sub-iteration is one omb_osem_subset_frames call, i.e. one forward
    and one backward launch for the whole batch.  `m`: (F, nTotMeas)
    measurements in subset order (host array or CUDA tensor); `x0`: (F, N)
    or one image broadcast to all F."""

    def __init__(self, options, m, x0=None):
        import torch
        options._check_ready()
        self.o = options
        self.dev = torch.device("cuda", options._device)
        n = int(options.N[0])
        S = int(options.subsets)
        M = options.measurementCount(-1)
        m = torch.as_tensor(m, dtype=torch.float32)
        if m.dim() != 2 or m.shape[1] != M:
            raise ValueError(f"measurements must be (frames, {M})")
        self.F = int(m.shape[0])
        self.y = m.to(self.dev).contiguous()
        if x0 is None:
            x0 = np.asarray(options.x0, dtype=np.float32).ravel()
        x0 = torch.as_tensor(np.asarray(x0, dtype=np.float32) if not torch.is_tensor(x0) else x0,
                             dtype=torch.float32).to(self.dev)
        self.x = (x0.reshape(1, n).expand(self.F, n) if x0.numel() == n else x0.reshape(self.F, n)).contiguous()
        self.offsets = [int(v) for v in np.asarray(options.nTotMeas).ravel()]
        self.sens = [torch.empty(n, device=self.dev) for _ in range(S)]
        for s in range(S):
            _native.call("omb_sensitivity", options._handle, s, _ptr(self.sens[s]), _stream(self.dev))
        mmax = max(options.measurementCount(s) for s in range(S))
        self.wm = torch.empty(self.F * mmax, device=self.dev)
        self.wi = torch.empty(self.F * n, device=self.dev)
        self.graph = None

    def _iteration(self):
        st = _stream(self.dev)
        n = int(self.o.N[0])
        M = self.y.shape[1]
        base = self.y.data_ptr()
        for s in range(int(self.o.subsets)):
            _native.call("omb_osem_subset_frames", self.o._handle, s, self.F, _ptr(self.x), n,
                         ctypes.c_void_p(base + 4 * self.offsets[s]), M, _ptr(self.sens[s]), _ptr(self.wm),
                         _ptr(self.wi), st)

    def iterate(self, n_iter, use_graph=False):
        import torch
        if not use_graph or (self.graph is None and n_iter < 1):
            for _ in range(n_iter):
                self._iteration()
            return self.x
        if self.graph is None:
            s = torch.cuda.Stream(self.dev)
            s.wait_stream(torch.cuda.current_stream(self.dev))
            with torch.cuda.stream(s):
                self._iteration()
            torch.cuda.current_stream(self.dev).wait_stream(s)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._iteration()
            n_iter -= 1
        for _ in range(n_iter):
            self.graph.replay()
        return self.x


_PET_METHODS = {'OSEM': _native.OMB_RECON_OSEM, 'OSL_OSEM': _native.OMB_RECON_OSL_OSEM,
                'ROSEM': _native.OMB_RECON_ROSEM, 'RAMLA': _native.OMB_RECON_RAMLA,
                'BSREM': _native.OMB_RECON_BSREM, 'ROSEM_MAP': _native.OMB_RECON_ROSEM_MAP,
                'PKMA': _native.OMB_RECON_PKMA, 'MRAMLA': _native.OMB_RECON_MRAMLA,
                'MBSREM': _native.OMB_RECON_MBSREM}
_PRIOR_METHODS = ('OSL_OSEM', 'BSREM', 'ROSEM_MAP', 'MBSREM')
_RELAXED = ('ROSEM', 'RAMLA', 'BSREM', 'ROSEM_MAP', 'PKMA', 'MRAMLA', 'MBSREM')


def relaxation(options):
    """Relaxation values lam[iter] of ROSEM / RAMLA / BSREM / ROSEM-MAP as the
    reference's prepass sets them (prepass.py:962-987): options.lambdaN when
    it holds at least Niter values (extra values ignored), else
    1 / (iter / 20 + 1); float32."""
    n = int(options.Niter)
    lam = np.asarray(getattr(options, 'lambdaN', np.empty(0)), dtype=np.float32).ravel()
    if lam.size == 0 or float(np.sum(lam)) == 0.:
        lam = np.zeros(0, dtype=np.float32)
    elif lam.size < n:
        print('Warning: The number of relaxation values must be at least the number of iterations times the '
              'number of subsets! Computing custom relaxation values.')
        lam = np.zeros(0, dtype=np.float32)
    elif lam.size > n:
        print('Warning: The number of relaxation values is more than the number of iterations. '
              'Later values are ignored!')
    if lam.size == 0:
        lam = np.array([1. / (i / 20. + 1.) for i in range(n)], dtype=np.float32)
    options.lambdaN = lam
    return np.ascontiguousarray(lam[:n], dtype=np.float32)


def momentum(options):
    """PKMA momentum alpha[iter * subsets + subset] as the reference's prepass
    sets it (prepass.py:998-1009): options.alpha_PKMA when it holds at least
    Niter * subsets values and is not all zero, else
    1 + rho_PKMA k / (k + delta_PKMA) over the sub-iteration count k; float32."""
    n = int(options.Niter) * int(options.subsets)
    a = np.asarray(getattr(options, 'alpha_PKMA', np.empty(0)), dtype=np.float32).ravel()
    if a.size < n or float(np.sum(a)) == 0.:
        if a.size < n:
            print('Warning: The number of PKMA alpha (momentum) values must be at least the number of iterations '
                  'times the number of subsets! Computing custom alpha values.')
        k = np.arange(n, dtype=np.float64)
        rho, delta = float(getattr(options, 'rho_PKMA', .45)), float(getattr(options, 'delta_PKMA', 100.))
        a = (1. + (rho * k) / (k + delta)).astype(np.float32)
    elif a.size > n:
        print('Warning: The number of PKMA alpha (momentum) values is higher than the total number of iterations '
              'times subsets. The final values will be ignored.')
    options.alpha_PKMA = a
    return np.ascontiguousarray(a[:n], dtype=np.float32)


def _check_preconditioners(options):
    """The preconditioner selections the built-in loop takes (before any
    device work): at most one of the image types 0-2; the filtering-based
    measurement preconditioner (1) is built for PDHG only."""
    pt_im = np.ravel(np.asarray(getattr(options, 'precondTypeImage', np.zeros(7, dtype=bool)), dtype=bool))
    pt_meas = np.ravel(np.asarray(getattr(options, 'precondTypeMeas', np.zeros(2, dtype=bool)), dtype=bool))
    if int(np.count_nonzero(pt_im[:3])) > 1:
        raise ValueError('Only one of the image preconditioners 0-2 can be selected')
    if pt_im.size > 5 and pt_im[5]:
        _check_image_filter(options)
        _filtered_relaxation(options, relaxation(options), int(getattr(options, 'filteringIterations', 0)),
                             int(options.subsets))
    if pt_meas.size > 1 and pt_meas[1]:
        raise ValueError('The filtering-based measurement preconditioner (type 1) is not built')


def _filtered_relaxation(options, lam, K, S):
    """The per-iteration relaxation with the filtering-based image
    preconditioner: options.lambdaFiltered (options.lambdaN when it is empty,
    or of another size with K < Niter * subsets) in the iterations whose
    sub-iterations all filter, lambdaN from sub-iteration K on; K = 0 or
    K >= Niter * subsets never switches.  A switch inside an iteration needs
    equal values there."""
    n = int(options.Niter)
    lf = np.asarray(getattr(options, 'lambdaFiltered', np.empty(0)), dtype=np.float32).ravel()
    lam_n = np.asarray(options.lambdaN, dtype=np.float32).ravel()
    if (lf.size != lam_n.size and K < S * n) or lf.size == 0:
        lf = lam_n
    if lf.size < n:
        raise ValueError('options.lambdaFiltered needs at least Niter values')
    out = lf[:n].astype(np.float32).copy()
    if 0 < K < S * n:
        for i in range(n):
            if i * S >= K:
                out[i] = lam[i]
            elif (i + 1) * S > K and lf[i] != lam[i]:
                raise ValueError('options.lambdaFiltered differing from lambdaN needs filteringIterations to be a '
                                 'multiple of subsets')
    options.lambdaFiltered = lf
    return np.ascontiguousarray(out, dtype=np.float32)


def _check_image_filter(options):
    """The filtering-based image preconditioner filters whole slices: Nf (the
    power of two at or above Nx) must cover Ny too."""
    nx, ny = int(np.ravel(options.Nx)[0]), int(np.ravel(options.Ny)[0])
    nf = int(2 ** np.ceil(np.log2(nx)))
    if ny > nf:
        raise ValueError('The filtering-based image preconditioner needs Ny <= 2^ceil(log2(Nx))')
    if nf > 2048:
        raise ValueError('The filtering-based image preconditioner is built for Nx <= 2048')


def _check_pdhg_preconditioners(options):
    """PDHG takes the filtering-based measurement (type 1) or image (type 5)
    preconditioner, one at a time; its other image and diagonal measurement
    preconditioners are not built."""
    pt_im = np.ravel(np.asarray(getattr(options, 'precondTypeImage', np.zeros(7, dtype=bool)), dtype=bool))
    pt_meas = np.ravel(np.asarray(getattr(options, 'precondTypeMeas', np.zeros(2, dtype=bool)), dtype=bool))
    if pt_im[:5].any() or (pt_im.size > 6 and pt_im[6]):
        raise ValueError('Image preconditioners 0-4 and 6 are built for PKMA / MRAMLA / MBSREM, not PDHG')
    if pt_im.size > 5 and pt_im[5]:
        _check_image_filter(options)
        if pt_meas.size > 1 and pt_meas[1]:
            raise ValueError('Select one of the filtering-based preconditioners (image type 5, measurement type 1)')
    if pt_meas.size and pt_meas[0]:
        raise ValueError('The diagonal measurement preconditioner (type 0) is built for PKMA / MRAMLA / MBSREM')
    if pt_meas.size > 1 and pt_meas[1] and int(options.subsets) > 1 and int(options.subsetType) < 8:
        raise ValueError('The filtering-based preconditioner needs whole projections per subset (subsetType >= 8)')


def reconstructions_main(options):
    """The built-in reconstruction (omegatomo/reconstruction/recomain.py:427-725,
    the compiled omegaMain entry) for the algorithms of this path:
    options.OSEM, options.ROSEM, options.RAMLA, options.MRAMLA and options.PKMA
    (PET; PKMA takes a prior when one is set), options.OSL_OSEM,
    options.BSREM, options.ROSEM_MAP and options.MBSREM with one prior
    (options.RDP, Quad, Huber, NLM, MRP, TV, APLS, GGMRF, hyperbolic or
    weighted_mean; PET, MAP; Ndx/Ndy/Ndz neighbourhood weights as the
    reference forms them; relaxation options.lambdaN, PKMA momentum
    options.alpha_PKMA, MRAMLA / MBSREM bound options.U) or options.PDHG with
    options.TV (TV, SATV, weighted and anatomical TV by options.TVtype and
    options.TV_use_anatomical, priors.tv_setup), options.Niter iterations
    from options.x0, run natively by
    omb_reconstruct.  CT data are linearised as log(flat / SinM) first
    (prepass.py:22-36; flat = max(SinM) when options.flat <= 0), negative PET
    counts set to 0.  Returns (image of shape (Nx, Ny, Nz, 1) in Fortran
    order, empty forward projections), as the reference does with storeFP
    off.  Reads options.use_graph (default True) to replay iterations as CUDA
    graphs."""
    import torch
    chosen = [k for k in _PET_METHODS if bool(getattr(options, k, False))]
    if options.PDHG:
        chosen.append('PDHG')
    if not chosen:
        raise ValueError('No reconstruction method selected, aborting.')
    if len(chosen) > 1:
        raise ValueError('Select one reconstruction method (' + ', '.join(list(_PET_METHODS) + ['PDHG']) + ')')
    method = chosen[0]
    quad, huber = bool(getattr(options, 'Quad', False)), bool(getattr(options, 'Huber', False))
    nlm = bool(getattr(options, 'NLM', False))
    mrp = bool(getattr(options, 'MRP', False))
    tvp = bool(getattr(options, 'TV', False)) and not options.PDHG   # TV as a prior of the MAP algorithms
    ggmrf = bool(getattr(options, 'GGMRF', False))
    hyper = bool(getattr(options, 'hyperbolic', False))
    wmean = bool(getattr(options, 'weighted_mean', False))
    apls = bool(getattr(options, 'APLS', False)) and not options.PDHG   # the APLS prior: TVKernel's APLS form
    ad = bool(getattr(options, 'AD', False))
    lf, fmh = bool(getattr(options, 'L', False)), bool(getattr(options, 'FMH', False))
    n_priors = (int(bool(options.RDP)) + int(quad) + int(huber) + int(nlm) + int(mrp) + int(tvp) + int(ggmrf) +
                int(hyper) + int(wmean) + int(apls) + int(ad) + int(lf) + int(fmh))
    prior = method in _PRIOR_METHODS or (method == 'PKMA' and n_priors > 0)
    if prior and n_priors != 1:
        raise ValueError(method + ' needs one prior: options.RDP, options.Quad, options.Huber, options.NLM, '
                                  'options.MRP, options.TV, options.APLS, options.GGMRF, options.hyperbolic, '
                                  'options.weighted_mean, options.AD, options.L or options.FMH')
    if prior and ad:
        if int(getattr(options, 'NiterAD', 1)) < 1 or not float(getattr(options, 'KAD', 1.)) > 0:
            raise ValueError('options.AD needs NiterAD >= 1 and KAD > 0')
        if int(getattr(options, 'FluxType', 1)) not in (1, 2) or int(getattr(options, 'DiffusionType', 2)) not in (1, 2):
            raise ValueError('options.FluxType and options.DiffusionType must be 1 or 2')
    if method in ('PKMA', 'MRAMLA', 'MBSREM'):
        _check_preconditioners(options)
    if method == 'PDHG':
        _check_pdhg_preconditioners(options)
    if method in ('MRAMLA', 'MBSREM') and getattr(options, 'randoms_correction', False) and \
            np.size(getattr(options, 'SinDelayed', [])) and not np.all(np.asarray(options.SinDelayed) > 0):
        raise ValueError(method + ' with randoms is built for positive randoms (the zero-randoms bound '
                         'epsilon_mramla is not built)')
    if method != 'PDHG' and options.CT:
        raise ValueError(method + ' is built for PET data')
    prox = bool(getattr(options, 'ProxTV', False))
    tgv = bool(getattr(options, 'TGV', False))
    if options.PDHG and not (options.TV or prox or tgv):
        raise ValueError('PDHG is built with the TV prior (options.TV = True), the proximal TV (options.ProxTV = '
                         'True) or TGV (options.TGV = True)')
    if options.PDHG and int(bool(options.TV)) + int(prox) + int(tgv) > 1:
        raise ValueError('Select one of options.TV, options.ProxTV and options.TGV')
    if prox and not options.PDHG:
        raise ValueError('options.ProxTV is built for PDHG')
    if tgv and not options.PDHG:
        raise ValueError('options.TGV is built for PDHG')
    if tgv:
        if not (float(getattr(options, 'alpha0TGV', 0.)) > 0 and float(getattr(options, 'alpha1TGV', 0.)) > 0):
            raise ValueError('options.TGV needs options.alpha0TGV > 0 and options.alpha1TGV > 0')
        if int(getattr(options, 'derivativeType', 0)) != 0:
            # the reference's ProxTGVSymmDeriv does not compile with DIFFTYPE 1 (auxKernels.cl:1422)
            raise ValueError('options.TGV is built with forward differences (derivativeType 0)')
    tv_set = None
    if (prior and (tvp or apls)) or (options.PDHG and options.TV):
        # the TV gradient variant of the TV / APLS options (ProjectorClass.h:900-918)
        from . import priors
        tv_set = priors.tv_setup(options, apls=apls)
    sin = np.asarray(options.SinM, dtype=np.float32)
    if options.CT and not options.usingLinearizedData:
        if options.flat <= 0:
            options.flat = float(np.max(sin))
        sin = np.log(np.float32(options.flat) / sin).astype(np.float32)
        options.usingLinearizedData = True
    elif not options.CT:
        sin = np.where(sin < 0, 0, sin).astype(np.float32)
    options.SinM = sin
    if not options.projectorAdded:
        options.addProjector()
    options.initProj()  # reorders SinM (and the correction vectors) into subset order
    dev = torch.device("cuda", options._device)
    n = int(np.ravel(options.N)[0])
    m = np.asarray(options.SinM, dtype=np.float32).ravel(order='F')
    S = int(options.subsets)
    if method != 'PDHG':
        parts = [np.asarray(options.subsetMeasurements(m, s)) for s in range(S)]
        y = torch.from_numpy(np.ascontiguousarray(np.concatenate(parts), dtype=np.float32)).to(dev)
    else:
        y = torch.from_numpy(np.ascontiguousarray(m, dtype=np.float32)).to(dev)
    x0 = np.asarray(options.x0, dtype=np.float32).ravel(order='F')
    if x0.size != n:
        x0 = np.ones(n, dtype=np.float32) * (float(x0[0]) if x0.size else 1e-4)
    x0 = torch.from_numpy(np.ascontiguousarray(x0)).to(dev)
    x = torch.empty(n, device=dev)
    p = _native.ReconParams(struct_size=ctypes.sizeof(_native.ReconParams))
    p.algorithm = _PET_METHODS.get(method, _native.OMB_RECON_PDHG_TV)
    p.rdp_gamma = float(getattr(options, 'RDP_gamma', 1.0))
    # RDP neighbours outside the image: clamped to the edge with options.useImages (the reference's default
    # texture reads), 0 without
    p.rdp_edge = 1 if getattr(options, 'useImages', True) else 0
    window = None
    lam = None
    mom = None
    if method in _RELAXED:
        lam = relaxation(options)
        p.relaxation = ctypes.c_void_p(lam.ctypes.data)
    if method == 'PKMA':
        mom = momentum(options)
        p.momentum = ctypes.c_void_p(mom.ctypes.data)
    if method in ('MRAMLA', 'MBSREM'):
        u = float(getattr(options, 'U', 0.))
        p.upper_bound = u if u > 0 else 10000.
    # image preconditioners of PKMA / MRAMLA / MBSREM (options.precondTypeImage, functions.hpp:2057-2106:
    # 0 rhs / D, 1 rhs x / D, 2 rhs max(x, ref) / D, 3 alphaPrecond, 4 gradient-based, 6 curvature) and
    # the measurement preconditioner type 0 (options.precondTypeMeas[0], the ratio over A 1); other
    # algorithms ignore them, as the reference does (proj.py:1079-1082)
    pt_im = np.ravel(np.asarray(getattr(options, 'precondTypeImage', np.zeros(7, dtype=bool)), dtype=bool))
    pt_meas = np.ravel(np.asarray(getattr(options, 'precondTypeMeas', np.zeros(2, dtype=bool)), dtype=bool))
    keep = []
    if method in ('PKMA', 'MRAMLA', 'MBSREM'):
        def on(k):
            return pt_im.size > k and bool(pt_im[k])
        p.precond = 1 if on(0) else (2 if on(1) else (3 if on(2) else 0))
        if on(2):
            ref = np.asarray(getattr(options, 'referenceImage', np.empty(0)), dtype=np.float32)
            if ref.size != n:
                raise ValueError('Image preconditioner type 2 needs options.referenceImage of the image size')
            rt = torch.from_numpy(np.ascontiguousarray(ref.ravel(order='F'))).to(dev)
            keep.append(rt)
            p.precond_ref = ctypes.c_void_p(rt.data_ptr())
        alpha_pre = None
        if on(3):
            alpha_pre = np.ascontiguousarray(np.ravel(getattr(options, 'alphaPrecond', np.empty(0))), dtype=np.float32)
            if alpha_pre.size < int(options.Niter) * S:
                raise ValueError('Image preconditioner type 3 needs options.alphaPrecond with Niter * subsets values')
            p.precond_alpha = ctypes.c_void_p(alpha_pre.ctypes.data)
        if on(4):
            p.precond_grad = 1
            p.grad_v[0] = float(getattr(options, 'gradV1', 0.5))
            p.grad_v[1] = float(getattr(options, 'gradV2', 2.5))
            p.grad_iters[0] = int(getattr(options, 'gradInitIter', 1))
            p.grad_iters[1] = int(getattr(options, 'gradLastIter', 1))
            p.diff_type = int(getattr(options, 'derivativeType', 0))
        if on(6):
            p.precond_curv = 1
        if on(5):
            # the filtering-based image preconditioner and its relaxation schedule (functions.hpp:2093-2099,
            # subiterStep.h:28-45, libHeader.h:1335-1338, prepass.py:1154-1156): lambdaFiltered in the
            # filtering sub-iterations, lambdaN from sub-iteration K on (never when K = 0)
            from . import filters
            nf, _, fh = filters.image_filter_2d(int(np.ravel(options.Nx)[0]), getattr(options, 'filterWindow', 'hamming'),
                                                 float(getattr(options, 'cutoffFrequency', 1.0)),
                                                 float(getattr(options, 'normalFilterSigma', 0.25)))
            th = torch.from_numpy(fh).to(dev)
            keep.append(th)
            p.img_filter_h = ctypes.c_void_p(th.data_ptr())
            p.img_filter_nf = nf
            K = int(getattr(options, 'filteringIterations', 0))
            p.filter_iters = K
            lam = _filtered_relaxation(options, lam, K, S)
            p.relaxation = ctypes.c_void_p(lam.ctypes.data)
        if pt_meas.size and pt_meas[0]:
            p.precond_meas = 1
    if method == 'PKMA':
        p.pkma_relax = (1 if getattr(options, 'computeRelaxationParameters', False) else 0) | \
            (2 if getattr(options, 'relaxationScaling', False) else 0)
    if prior:
        p.prior = (_native.OMB_PRIOR_LFILTER if lf else
                   _native.OMB_PRIOR_FMH if fmh else
                   _native.OMB_PRIOR_AD if ad else
                   _native.OMB_PRIOR_RDP if options.RDP else
                   (_native.OMB_PRIOR_NLM if nlm else
                    (_native.OMB_PRIOR_MRP if mrp else
                     (_native.OMB_PRIOR_TV if (tvp or apls) else
                      (_native.OMB_PRIOR_GGMRF if ggmrf else
                       (_native.OMB_PRIOR_HYPERBOLIC if hyper else
                        (_native.OMB_PRIOR_WMEAN if wmean else
                         (_native.OMB_PRIOR_QUAD if quad else _native.OMB_PRIOR_HUBER))))))))
        if ad:
            # the AD prior (priors.h:226-237, libHeader.h:1212-1232): time step, conductance, iterations,
            # flux 1 exponential / 2 quadratic, diffusion 1 gradient / 2 modified curvature
            p.ad_dt = float(getattr(options, 'TimeStepAD', 1.))
            p.ad_k = float(getattr(options, 'KAD', 1.))
            p.ad_niter = int(getattr(options, 'NiterAD', 1))
            p.ad_flux = int(getattr(options, 'FluxType', 1))
            p.ad_diffusion = int(getattr(options, 'DiffusionType', 2))
            p.mrp_no_norm = 1 if getattr(options, 'med_no_norm', False) else 0
        if lf or fmh:
            # the L-filter (priors.h:84-97) and FMH (priors.h:54-82) over Ndx / Ndy / Ndz, with the
            # MATLAB prepass's weights (lfilter_weights.m, fmhWeights.m) unless given
            from . import priors
            wl = torch.from_numpy(priors.lfilter_weights(options) if lf else priors.fmh_weights(options)).to(dev)
            keep.append(wl)
            if lf:
                p.lfilter_weights = ctypes.c_void_p(wl.data_ptr())
            else:
                p.fmh_weights = ctypes.c_void_p(wl.data_ptr())
            p.mrp_no_norm = 1 if getattr(options, 'med_no_norm', False) else 0
            p.prior_g[0], p.prior_g[1], p.prior_g[2] = priors.median_filter_window(options)
        if wmean:
            from . import priors
            mt = int(getattr(options, 'mean_type', 4))
            if mt not in (1, 2, 3, 4, 5, 6):
                raise ValueError('mean_type must be 1-6')
            w = priors.weighted_mean_weights(options)
            ww = torch.from_numpy(w).to(dev)
            keep.append(ww)
            p.wmean_weights = ctypes.c_void_p(ww.data_ptr())
            p.wmean_wsum = float(np.sum(w, dtype=np.float32))
            p.wmean_type = mt
            p.mrp_no_norm = 1 if getattr(options, 'med_no_norm', False) else 0
            p.prior_g[0], p.prior_g[1], p.prior_g[2] = int(options.Ndx), int(options.Ndy), int(options.Ndz)
        if hyper:
            # the quadratic prior's normalised weights and hyperbolicDelta (libHeader.h:1159-1162)
            from . import priors
            w = np.asarray(options.weights, dtype=np.float32) if np.size(options.weights) else \
                priors.neighbourhood_weights(options)
            wq = priors.normalised_weights(w) if not np.size(options.weights) else w[~np.isinf(w)]
            hw = torch.from_numpy(np.ascontiguousarray(wq, dtype=np.float32)).to(dev)
            keep.append(hw)
            p.hyper_weights = ctypes.c_void_p(hw.data_ptr())
            p.hyper_delta = float(getattr(options, 'hyperbolicDelta', 1.0))
            p.prior_g[0], p.prior_g[1], p.prior_g[2] = int(options.Ndx), int(options.Ndy), int(options.Ndz)
        if ggmrf:
            from . import priors
            gw = torch.from_numpy(priors.ggmrf_weights(options)).to(dev)
            keep.append(gw)
            p.ggmrf_weights = ctypes.c_void_p(gw.data_ptr())
            p.prior_g[0], p.prior_g[1], p.prior_g[2] = int(options.Ndx), int(options.Ndy), int(options.Ndz)
            p.ggmrf[0], p.ggmrf[1], p.ggmrf[2] = (float(options.GGMRF_p), float(options.GGMRF_q),
                                                 float(options.GGMRF_c))
        if mrp:
            # the median window is Ndx / Ndy / Ndz (priors.h:371-375)
            p.prior_g[0], p.prior_g[1], p.prior_g[2] = int(options.Ndx), int(options.Ndy), int(options.Ndz)
            p.mrp_no_norm = 1 if getattr(options, 'med_no_norm', False) else 0
        if nlm:
            # search window Ndx / Ndy / Ndz, patch Nlx / Nly / Nlz, h = NLMsigma^2 (libHeader.h:1285-1286;
            # ProjectorClass.h:841-870), gamma = RDP_gamma, GGMRF p / q / c
            from . import priors
            g = torch.from_numpy(priors.nlm_gaussian(options)).to(dev)
            keep.append(g)
            p.nlm_gaussian = ctypes.c_void_p(g.data_ptr())
            p.nlm_type = priors.nlm_type(options)
            p.prior_g[0], p.prior_g[1], p.prior_g[2] = int(options.Ndx), int(options.Ndy), int(options.Ndz)
            p.nlm_patch[0], p.nlm_patch[1], p.nlm_patch[2] = int(options.Nlx), int(options.Nly), int(options.Nlz)
            p.nlm_h = float(options.NLMsigma) ** 2
            p.nlm_adaptive = 1 if getattr(options, 'NLAdaptive', False) else 0
            p.nlm_adaptive_s = float(getattr(options, 'NLAdaptiveConstant', 1.0))
            p.ggmrf[0], p.ggmrf[1], p.ggmrf[2] = (float(getattr(options, k, 0.0)) for k in ('GGMRF_p', 'GGMRF_q',
                                                                                            'GGMRF_c'))
            if getattr(options, 'NLM_use_anatomical', False):
                r = np.asarray(options.NLM_referenceImage, dtype=np.float32).ravel(order='F')
                if r.size != n:
                    raise ValueError('NLM_referenceImage must have the size of the image')
                rt = torch.from_numpy(np.ascontiguousarray(r)).to(dev)
                keep.append(rt)
                p.nlm_ref = ctypes.c_void_p(rt.data_ptr())
        if quad or huber:
            from . import priors
            nd = (int(options.Ndx), int(options.Ndy), int(options.Ndz))
            w = np.asarray(options.weights, dtype=np.float32) if np.size(options.weights) else \
                priors.neighbourhood_weights(options)
            wq = priors.normalised_weights(w) if not np.size(options.weights) else w[~np.isinf(w)]
            options.weights_quad = wq
            window = torch.from_numpy(priors.prior_window(wq, *nd)).to(dev)
            p.prior_window = ctypes.c_void_p(window.data_ptr())
            p.prior_g[0], p.prior_g[1], p.prior_g[2] = nd
            p.huber_delta = float(getattr(options, 'huber_delta', 1.0))
    p.n_iter = int(options.Niter)
    p.beta = float(options.beta)
    p.tv_smoothing = float(options.TVsmoothing)
    if options.PDHG:
        # the filtering-based measurement preconditioner (precondTypeMeas[1], prepass.py:1121-1136,
        # functions.hpp:2109-2166); PDHG's other preconditioners are not built
        pt_meas_p = np.ravel(np.asarray(getattr(options, 'precondTypeMeas', np.zeros(2, dtype=bool)), dtype=bool))
        if pt_meas_p.size > 1 and pt_meas_p[1]:
            from . import filters
            nr = int(np.ravel(options.nRowsD)[0]) if options.CT else int(np.ravel(options.Ndist)[0])
            sig = float(np.ravel(options.sigmaCP)[0])
            if tgv:
                # the inverse filter's sigma times beta with TGV (prepass.py:1133-1134)
                sig *= float(options.beta)
            nf, _, _, fh, fhinv = filters.pdhg_row_filters(nr, sig, getattr(options, 'filterWindow', 'hamming'),
                                                           float(getattr(options, 'cutoffFrequency', 1.0)),
                                                           float(getattr(options, 'normalFilterSigma', 0.25)))
            th = torch.from_numpy(fh).to(dev)
            thi = torch.from_numpy(fhinv).to(dev)
            keep.extend([th, thi])
            p.filter_h = ctypes.c_void_p(th.data_ptr())
            p.filter_hinv = ctypes.c_void_p(thi.data_ptr())
            p.filter_nf = nf
            p.filter_rows = nr
            p.filter_iters = int(getattr(options, 'filteringIterations', 0))
            p.tau_filt = float(np.ravel(getattr(options, 'tauCPFilt', 0.0))[0])
        pt_im_p = np.ravel(np.asarray(getattr(options, 'precondTypeImage', np.zeros(7, dtype=bool)), dtype=bool))
        if pt_im_p.size > 5 and pt_im_p[5]:
            # the filtering-based image preconditioner: A^T p plus the TV term filtered in iterations
            # k < filteringIterations, tauCP the step while filtering
            from . import filters
            nf, _, fh = filters.image_filter_2d(int(np.ravel(options.Nx)[0]), getattr(options, 'filterWindow', 'hamming'),
                                                 float(getattr(options, 'cutoffFrequency', 1.0)),
                                                 float(getattr(options, 'normalFilterSigma', 0.25)))
            th = torch.from_numpy(fh).to(dev)
            keep.append(th)
            p.img_filter_h = ctypes.c_void_p(th.data_ptr())
            p.img_filter_nf = nf
            p.filter_iters = int(getattr(options, 'filteringIterations', 0))
    if options.PDHG and prox:
        # the proximal TV of the PDHG loop: dual step options.sigma2CP, the
        # beta ball (L2 or max norm), forward or backward differences
        p.tv_prox = 1
        p.sigma2 = float(np.ravel(getattr(options, 'sigma2CP', 1.0))[0])
        p.l2_ball = 1 if getattr(options, 'useL2Ball', True) else 0
        p.diff_type = int(getattr(options, 'derivativeType', 0))
        if p.diff_type not in (0, 1):
            raise ValueError('derivativeType must be 0 or 1')
        if not float(options.beta) > 0:
            raise ValueError('options.ProxTV needs options.beta > 0')
    if options.PDHG and tgv:
        # TGV of the PDHG loop (priors.h:284-313): the balls alpha0TGV,
        # alpha1TGV, the dual step sigma2CP; the data dual divides by
        # 1 + sigma beta
        p.tgv = 2 if bool(getattr(options, 'use2DTGV', False)) else 1
        p.alpha0_tgv = float(options.alpha0TGV)
        p.alpha1_tgv = float(options.alpha1TGV)
        p.sigma2 = float(np.ravel(getattr(options, 'sigma2CP', 1.0))[0])
        p.l2_ball = 1 if getattr(options, 'useL2Ball', True) else 0
        p.diff_type = 0
    if tv_set is not None:
        p.tv_variant, p.tv_sigma, p.tv_c, p.tv_smoothing, tv_ref = tv_set
        if tv_ref is not None:
            rt = torch.from_numpy(tv_ref).to(dev)
            keep.append(rt)
            p.tv_ref = ctypes.c_void_p(rt.data_ptr())
    p.tau = float(np.ravel(options.tauCP)[0]) if np.size(options.tauCP) else 0.0
    p.sigma = float(np.ravel(options.sigmaCP)[0])
    p.theta = float(np.ravel(options.thetaCP)[0])
    p.power_iterations = int(options.powerIterations)
    p.positivity = 1 if options.enforcePositivity else 0
    p.use_graph = 1 if getattr(options, 'use_graph', True) else 0
    _native.call("omb_reconstruct", options._handle, ctypes.byref(p), _ptr(y), _ptr(x0), _ptr(x), _stream(dev))
    options._check_staged("omb_reconstruct")
    options.tau_used = p.tau_used
    options.tau_used2 = p.tau_used2
    out = x.cpu().numpy().reshape((int(np.ravel(options.Nx)[0]), int(np.ravel(options.Ny)[0]),
                                   int(np.ravel(options.Nz)[0]), 1), order='F')
    return out, np.empty(0, dtype=np.float32)


def reconstructions_mainCT(options):
    """CT entry of the built-in reconstruction (recomain.py:377-401)."""
    options.CT = True
    return reconstructions_main(options)
