"""TEST INFRASTRUCTURE ONLY -- FP64 numpy restatements of the image-domain
steps around the projectors, for the parity tests:

* psf_convolve: Convolution3D_f (OMEGA source/opencl/auxKernels.cl:192-245),
  the window applied at every voxel with the image mirrored at its faces
  (edge voxel repeated: index -1 reads 0, N reads N-1);
* rdp_gradient: RDPKernel (auxKernels.cl:664-872), 6-neighbour form,
  neighbours outside the image 0 (the border-addressed texture of the
  reference's PyTorch/CuPy path, util/priors.py:143-146, and its buffer
  path) or clamped to the edge (the texture of its built-in path with
  useImages), both pinned to the kernel compiled on the host;
* nlm_gradient: the non-local kernels NLM (auxKernels.cl:297-620) with the
  image read clamped to its edges (the texture sampler of the reference's
  kernel path), and, with cpu_mode, the reference CPU function NLMFunc
  (source/cpp/NLM.h:15-142: interior voxels only, weight sum 1 / (sum +
  epps), NLTV's squared sum from 0), which oracle/_ref exports and pins;
* mrp_gradient: the median root prior (priors.h:4-25) on the symmetric
  padding; its median equals the reference CPU medianFilter3D (MRP.h),
  which oracle/_ref exports;
* lfilter_gradient / fmh_gradient: the L-filter and FMH priors (priors.h:
  54-97) over the reference's offsets grid (computeOffsets.m) on the same
  symmetric padding, with ArrayFire's sort / matmul / median written out.
"""
import numpy as np


def psf_convolve(img, shape, window, g):
    """img: flat, x fastest; window: flat (2gx+1)(2gy+1)(2gz+1), x fastest."""
    nx, ny, nz = shape
    gx, gy, gz = (int(v) for v in g)
    u = np.asarray(img, dtype=np.float64).reshape((nx, ny, nz), order='F')
    w = np.asarray(window, dtype=np.float64).reshape((2 * gx + 1, 2 * gy + 1, 2 * gz + 1), order='F')
    p = np.pad(u, ((gx, gx), (gy, gy), (gz, gz)), mode='symmetric')
    out = np.zeros_like(u)
    for k in range(2 * gz + 1):
        for j in range(2 * gy + 1):
            for i in range(2 * gx + 1):
                out += w[i, j, k] * p[i:i + nx, j:j + ny, k:k + nz]
    return out.ravel(order='F')


def rdp_gradient(u, shape, gamma, beta, epps=1e-8, clamp=False):
    """beta * dRDP(u)/du, 6 neighbours; outside the image 0, or (clamp) the
    edge voxel, the clamp-to-edge texture of the reference's built-in path
    (useImages)."""
    nx, ny, nz = shape
    a = np.asarray(u, dtype=np.float64).reshape((nx, ny, nz), order='F')
    p = np.pad(a, 1, mode='edge' if clamp else 'constant')

    def term(k):
        d = a - k
        div = a + k + gamma * np.abs(d)
        return d * (gamma * np.abs(d) + a + 3.0 * k + epps * epps) / (div * div + epps)

    c = p[1:-1, 1:-1, 1:-1]
    plus = term(p[2:, 1:-1, 1:-1]) + term(p[1:-1, 2:, 1:-1]) + term(p[1:-1, 1:-1, 2:])
    minus = term(p[:-2, 1:-1, 1:-1]) + term(p[1:-1, :-2, 1:-1]) + term(p[1:-1, 1:-1, :-2])
    plus[np.isnan(plus)] = 0.0
    minus[np.isnan(minus)] = 0.0
    assert c.shape == a.shape
    return (beta * (plus + minus)).ravel(order='F')


def _sgn(v):
    return np.sign(v)


def nlm_gradient(u, shape, gaussian, sw, pw, h, epps, nl_type, gamma=10.0, ggmrf=(2.0, 1.5, 0.001), u_ref=None,
                 cpu_mode=False, adaptive_s=None):
    """Non-local gradient of image u (flat, x fastest), without the weight:
    for every voxel j, over the search offsets k != 0 with patch distance
    d_k = sum_p g_p (P(j + p) - P(j + k + p))^2 (P = u_ref when given) and
    weight w_k = exp(-d_k / h):
      0 NLM:     sum w (u_j - u_k) / W        1 NLTV: the same / sqrt(sum w (u_j - u_k)^2 / W + epps)
      2 NLM-MRP: u_j - sum w u_k / W          3 NLRD, 4 NL Lange, 5 MRP + Lange, 6 NLGGMRF,
    W = epps + sum w (cpu_mode: 1 / (sum w + epps) and the NLTV sum from 0;
    a border of sw + pw voxels left 0).  adaptive_s (NLMADAPTIVE,
    auxKernels.cl:562-563): w_k = exp(-d_k / (d_k / |patch| h + adaptive_s))."""
    nx, ny, nz = shape
    sx, sy, sz = (int(v) for v in sw)
    px, py, pz = (int(v) for v in pw)
    ax, ay, az = sx + px, sy + py, sz + pz
    U = np.asarray(u, dtype=np.float64).reshape((nz, ny, nx))
    R = U if u_ref is None else np.asarray(u_ref, dtype=np.float64).reshape((nz, ny, nx))
    Up = np.pad(U, ((az, az), (ay, ay), (ax, ax)), mode='edge')
    Rp = np.pad(R, ((az, az), (ay, ay), (ax, ax)), mode='edge')
    g = np.asarray(gaussian, dtype=np.float64).reshape((2 * pz + 1, 2 * py + 1, 2 * px + 1))

    def sh(A, dz, dy, dx):
        return A[az + dz:az + dz + nz, ay + dy:ay + dy + ny, ax + dx:ax + dx + nx]
    uj = U
    wsum = np.zeros_like(U) if cpu_mode else np.full_like(U, epps)
    out = np.zeros_like(U)
    ala = np.zeros_like(U) if cpu_mode else np.full_like(U, epps)
    p_, q_, c_ = (float(v) for v in ggmrf)
    for i in range(-sx, sx + 1):
        for j in range(-sy, sy + 1):
            for k in range(-sz, sz + 1):
                if i == 0 and j == 0 and k == 0:
                    continue
                dist = np.zeros_like(U)
                for qz in range(-pz, pz + 1):
                    for qy in range(-py, py + 1):
                        for qx in range(-px, px + 1):
                            d = sh(Rp, qz, qy, qx) - sh(Rp, k + qz, j + qy, i + qx)
                            dist += g[qz + pz, qy + py, qx + px] * d * d
                if adaptive_s is not None:
                    psize = float((2 * px + 1) * (2 * py + 1) * (2 * pz + 1))
                    w = np.exp(-dist / ((dist / psize) * h + adaptive_s))
                else:
                    w = np.exp(-dist / h)
                wsum = wsum + w
                uk = sh(Up, k, j, i)
                if nl_type in (2, 5):
                    out += w * uk
                elif nl_type == 0:
                    out += w * (uj - uk)
                elif nl_type == 3:
                    dd = uj - uk
                    dp = uj + uk + gamma * np.abs(dd) + epps
                    out += w * dd * (gamma * np.abs(dd) + uj + 3.0 * uk + epps * epps) / (dp * dp)
                elif nl_type == 4:
                    dd = uj - uk
                    s_ = _sgn(dd)
                    out += w * (s_ - s_ / (np.abs(dd) / gamma + 1.0))
                elif nl_type == 6:
                    dd = uj - uk
                    dpq = 1.0 + np.abs(dd / c_) ** (p_ - q_)
                    out += w * (np.abs(dd) ** (p_ - 1.0) / dpq) * (p_ - gamma * (np.abs(dd) ** (p_ - q_) / dpq)) * _sgn(dd)
                else:
                    dd = uj - uk
                    out += w * dd
                    ala += w * dd * dd
    if cpu_mode:
        ws = np.where(wsum != 0.0, 1.0 / (wsum + epps), wsum)
    else:
        ws = 1.0 / wsum
    out = out * ws
    if nl_type == 2:
        out = uj - out
    elif nl_type == 5:
        o_ = uj - out
        s_ = _sgn(o_)
        out = s_ - s_ / (np.abs(o_) / gamma + 1.0)
    elif nl_type == 1:
        out = out / np.sqrt(ala * ws + epps)
    if cpu_mode:
        mask = np.zeros_like(U, dtype=bool)
        mask[az:nz - az, ay:ny - ay, ax:nx - ax] = True
        out = np.where(mask, out, 0.0)
    return out.ravel()


def mrp_gradient(u, shape, m, beta, epps, no_norm=False):
    """Median root prior gradient (priors.h:4-25): beta (u - med) / (med + epps)
    (no_norm: beta (u - med)), med the median of the (2m+1)^3-type window of u
    padded symmetrically (functions.hpp:216-260)."""
    nx, ny, nz = shape
    mx, my, mz = (int(v) for v in m)
    U = np.asarray(u, dtype=np.float64).reshape((nz, ny, nx))
    P = np.pad(U, ((mz, mz), (my, my), (mx, mx)), mode='symmetric')
    stack = [P[mz + k:mz + k + nz, my + j:my + j + ny, mx + i:mx + i + nx]
             for i in range(-mx, mx + 1) for j in range(-my, my + 1) for k in range(-mz, mz + 1)]
    med = np.median(np.stack(stack), axis=0)
    d = U - med
    return (beta * d if no_norm else d / (med + epps) * beta).ravel()


def _offset_columns(u, shape, m):
    """The window values of every voxel, one row per column of the offsets
    grid (computeOffsets.m: ndgrid over -Ndx..Ndx on every axis, x fastest;
    3 axes for Ndx = Ndy = Ndz, 2 for Ndx = Ndy = 1, Ndz = 0), on the image
    padded symmetrically by (Ndx, Ndy, Ndz) (functions.hpp:216-260)."""
    nx, ny, nz = shape
    mx, my, mz = (int(v) for v in m)
    assert (mx >= 1 and mx == my == mz) or (mx, my, mz) == (1, 1, 0)
    d = 3 if mz else 2
    w = 2 * mx + 1
    U = np.asarray(u, dtype=np.float64).reshape((nz, ny, nx))
    P = np.pad(U, ((mz, mz), (my, my), (mx, mx)), mode='symmetric')
    rows = []
    for c in range(w ** d):
        i, j, k = c % w - mx, (c // w) % w - my, (c // (w * w) - mz if d == 3 else 0)
        rows.append(P[mz + k:mz + k + nz, my + j:my + j + ny, mx + i:mx + i + nx].ravel())
    return np.stack(rows)


def lfilter_gradient(u, shape, m, a_l, beta, epps, no_norm=False):
    """L-filter prior (priors.h:84-97): the window values sorted ascending per
    voxel, their sum weighted by a_L, beta (u - s) / (s + epps) (no_norm:
    beta (u - s))."""
    V = np.sort(_offset_columns(u, shape, m), axis=0)
    s = np.asarray(a_l, dtype=np.float64) @ V
    d = np.asarray(u, dtype=np.float64).ravel() - s
    return beta * d if no_norm else d / (s + epps) * beta


def fmh_gradient(u, shape, m, fmh_w, beta, epps, no_norm=False):
    """FMH prior (priors.h:54-82): for ii < luup (4 when Nz = 1 or Ndz = 0,
    else 13) the offsets columns seq(Ndx ii, N - Ndx ii - 1, alku / Ndx - ii)
    (alku the centre column, N the column count) weighted by column ii of
    fmh_weights ((2 Ndx + 1) x luup, column-major); the centre value last;
    the median of the luup + 1 values (numpy's median: the mean of the
    middle two for an even count, as af::median); beta (u - med) / (med +
    epps) (no_norm: beta (u - med))."""
    nx, ny, nz = shape
    mx, my, mz = (int(v) for v in m)
    V = _offset_columns(u, shape, m)
    N = V.shape[0]
    alku = N // 2
    luup = 4 if (nz == 1 or mz == 0) else 13
    rows = 2 * mx + 1
    W = np.asarray(fmh_w, dtype=np.float64).reshape((rows, luup), order='F')
    vals = []
    for ii in range(luup):
        cols = list(range(mx * ii, N - mx * ii, alku // mx - ii))
        assert len(cols) == rows
        vals.append(W[:, ii] @ V[cols])
    vals.append(V[alku])
    med = np.median(np.stack(vals), axis=0)
    d = np.asarray(u, dtype=np.float64).ravel() - med
    return beta * d if no_norm else d / (med + epps) * beta


def padded_symmetric(u, shape, m):
    """u padded by the window on every side, x fastest (the median filter's input)."""
    nx, ny, nz = shape
    mx, my, mz = (int(v) for v in m)
    U = np.asarray(u, dtype=np.float64).reshape((nz, ny, nx))
    return np.ascontiguousarray(np.pad(U, ((mz, mz), (my, my), (mx, mx)), mode='symmetric').ravel())


def ggmrf_gradient(u, shape, s, weights, p, q, c, beta):
    """GGMRF gradient (GGMRFKernel, auxKernels.cl:878-980) in FP64, edge-clamped
    neighbours, weights in the kernel's order (x outermost, z fastest)."""
    nx, ny, nz = shape
    sx, sy, sz = (int(v) for v in s)
    U = np.asarray(u, dtype=np.float64).reshape((nz, ny, nx))
    P = np.pad(U, ((sz, sz), (sy, sy), (sx, sx)), mode='edge')
    cpq = c ** (p - q)
    pqc = (p - q) / c ** (p - q)
    out = np.zeros_like(U)
    uu = 0
    for i in range(-sx, sx + 1):
        for j in range(-sy, sy + 1):
            for k in range(-sz, sz + 1):
                if i == 0 and j == 0 and k == 0:
                    continue
                d = U - P[sz + k:sz + k + nz, sy + j:sy + j + ny, sx + i:sx + i + nx]
                a = np.abs(d)
                dcpq = np.abs(d / c) ** (p - q)
                dpq = 1.0 + dcpq
                with np.errstate(divide='ignore', invalid='ignore'):
                    t = weights[uu] * (a ** (p - 1.0) / dpq) * (p - pqc * ((dcpq * cpq) / dpq)) * np.sign(d)
                out += np.where(d != 0.0, t, 0.0)
                uu += 1
    return (beta * out).ravel()


def hyperbolic_gradient(u, shape, s, weights, delta, beta):
    """Hyperbolic prior gradient (hyperbolicKernel, auxKernels.cl:1591-1688) in
    FP64, edge-clamped neighbours, weights z outermost, x fastest."""
    nx, ny, nz = shape
    sx, sy, sz = (int(v) for v in s)
    U = np.asarray(u, dtype=np.float64).reshape((nz, ny, nx))
    P = np.pad(U, ((sz, sz), (sy, sy), (sx, sx)), mode='edge')
    out = np.zeros_like(U)
    uu = 0
    for k in range(-sz, sz + 1):
        for j in range(-sy, sy + 1):
            for i in range(-sx, sx + 1):
                if i == 0 and j == 0 and k == 0:
                    continue
                t = (U - P[sz + k:sz + k + nz, sy + j:sy + j + ny, sx + i:sx + i + nx]) / delta
                out += t / delta / np.sqrt(t * t + 1.0) * weights[uu]
                uu += 1
    return (beta * out).ravel()


def wmean_gradient(u, shape, m, weights, mean_type, beta, epps, no_norm=False):
    """Weighted-mean prior gradient, types 1-3 (priors.h:99-160) in FP64: the
    weighted arithmetic / harmonic / geometric mean of the symmetric-padded
    window, weights applied as a convolution (flipped)."""
    nx, ny, nz = shape
    mx, my, mz = (int(v) for v in m)
    U = np.asarray(u, dtype=np.float64).reshape((nz, ny, nx))
    P = np.pad(U, ((mz, mz), (my, my), (mx, mx)), mode='symmetric')
    W = np.asarray(weights, dtype=np.float64).reshape((2 * mz + 1, 2 * my + 1, 2 * mx + 1))
    f = {1: lambda a: a, 2: lambda a: 1.0 / a, 3: np.log}[mean_type]
    acc = np.zeros_like(U)
    for k in range(-mz, mz + 1):
        for j in range(-my, my + 1):
            for i in range(-mx, mx + 1):
                acc += W[mz - k, my - j, mx - i] * f(P[mz + k:mz + k + nz, my + j:my + j + ny, mx + i:mx + i + nx])
    mean = {1: lambda a: a, 2: lambda a: 1.0 / a, 3: np.exp}[mean_type](acc)
    d = U - mean
    return (beta * (d if no_norm else d / (mean + epps))).ravel()


def wmean_gradient46(u, shape, m, weights, mean_type, beta):
    """Weighted-mean prior gradient, types 4-6 (priors.h:125-210) in FP64.
    The image is mirrored by twice the window (functions.hpp:216-260 with
    2 Ndx ...), the weighted arithmetic / harmonic / geometric mean M (the
    weights divided by their sum, applied as a convolution) is taken over
    the image grown by the window on every side, and each voxel sums
    w_d g(u, M(x + d)) over the window's offsets d with the raw weights in
    x-fastest order: g = log(max(u / M, 1e-6)) (type 4); with u' = max(u,
    1e-6), (u' - M) / u' - ((u' - M) / (sqrt(2) u'))^2 (type 5), 1 - M / u'
    (type 6)."""
    nx, ny, nz = shape
    mx, my, mz = (int(v) for v in m)
    U = np.asarray(u, dtype=np.float64).reshape((nz, ny, nx))
    P = np.pad(U, ((2 * mz, 2 * mz), (2 * my, 2 * my), (2 * mx, 2 * mx)), mode='symmetric')
    W = np.asarray(weights, dtype=np.float64).reshape((2 * mz + 1, 2 * my + 1, 2 * mx + 1))
    Wn = W / W.sum()
    f = {4: lambda a: a, 5: lambda a: 1.0 / a, 6: np.log}[mean_type]
    ez, ey, ex = nz + 2 * mz, ny + 2 * my, nx + 2 * mx
    acc = np.zeros((ez, ey, ex))
    with np.errstate(divide='ignore'):
        FP = f(P)
    for k in range(-mz, mz + 1):
        for j in range(-my, my + 1):
            for i in range(-mx, mx + 1):
                acc += Wn[mz - k, my - j, mx - i] * FP[mz + k:mz + k + ez, my + j:my + j + ey, mx + i:mx + i + ex]
    with np.errstate(divide='ignore'):
        M = {4: lambda a: a, 5: lambda a: 1.0 / a, 6: np.exp}[mean_type](acc)
    ut = np.maximum(U, 1e-6)
    g = np.zeros_like(U)
    for l in range(2 * mz + 1):
        for k in range(2 * my + 1):
            for h in range(2 * mx + 1):
                Md = M[l:l + nz, k:k + ny, h:h + nx]
                if mean_type == 4:
                    with np.errstate(divide='ignore'):
                        t = np.log(np.maximum(U / Md, 1e-6))
                elif mean_type == 5:
                    t = (ut - Md) / ut - ((ut - Md) / (np.sqrt(2.0) * ut)) ** 2
                else:
                    t = 1.0 - Md / ut
                g += W[l, k, h] * t
    return (beta * g).ravel()


# ---------------------------------------------------------------------------
# Proximal TV of the PDHG loop (priors.h:261-281; auxKernels.cl:1141-1343
# ProxTVq, ProxTVDivergence, ProxTVGradient): the image differences with
# zero beyond the grid, the dual variable q = (qx, qy, qz) projected onto the
# alpha ball, its negative divergence added to the primal right-hand side.
# ---------------------------------------------------------------------------

def _diff(U, axis, forward):
    """Forward (next - this; the last voxel gives -this) or backward (this -
    previous; the first voxel gives this) difference along one axis of an
    (x, y, z) array."""
    out = np.empty_like(U)
    if forward:
        sl_a = [slice(None)] * 3
        sl_b = [slice(None)] * 3
        sl_a[axis] = slice(0, -1)
        sl_b[axis] = slice(1, None)
        out[tuple(sl_a)] = U[tuple(sl_b)] - U[tuple(sl_a)]
        last = [slice(None)] * 3
        last[axis] = slice(-1, None)
        out[tuple(last)] = -U[tuple(last)]
    else:
        sl_a = [slice(None)] * 3
        sl_b = [slice(None)] * 3
        sl_a[axis] = slice(1, None)
        sl_b[axis] = slice(0, -1)
        out[tuple(sl_a)] = U[tuple(sl_a)] - U[tuple(sl_b)]
        first = [slice(None)] * 3
        first[axis] = slice(0, 1)
        out[tuple(first)] = U[tuple(first)]
    return out


def proxtv_dual(x, q, shape, sigma2, alpha, l2=True, diff_type=0):
    """q <- P_alpha(q + sigma2 D x): D the forward differences (diff_type 0)
    or the backward ones (1); P the projection onto the per-voxel L2 ball of
    radius alpha (l2) or onto the max-norm ball.  q is (3, N), x fastest."""
    X = np.asarray(x, dtype=np.float64).reshape(shape, order='F')
    Qa = np.asarray(q, dtype=np.float64).reshape(3, -1)
    Q = np.stack([Qa[a].reshape(shape, order='F') for a in range(3)])
    g = np.stack([_diff(X, a, diff_type == 0) for a in range(3)])
    Qn = Q + sigma2 * g
    if l2:
        scale = np.maximum(1.0, np.sqrt((Qn ** 2).sum(axis=0)) / alpha)
    else:
        scale = np.maximum(np.abs(Qn).max(axis=0) / alpha, 1.0)
    Qn = Qn / scale
    return np.stack([Qn[a].ravel(order='F') for a in range(3)])


def proxtv_divergence(q, shape, diff_type=0):
    """The term ProxTVDivergence subtracts from the right-hand side: the sum
    over the axes of the backward differences of q (diff_type 0, the
    adjoint of the forward differences up to sign) or the forward ones (1)."""
    out = np.zeros(shape)
    for a in range(3):
        Q = np.asarray(q[a], dtype=np.float64).reshape(shape, order='F')
        out += _diff(Q, a, diff_type != 0)
    return out.ravel(order='F')


def proxtgv_step(x, q, r, v, rhs, shape, sigma2, alpha0, alpha1, theta, tau, l2=True, three_d=True):
    """One proximal TGV step of the PDHG loop (priors.h:284-313; ProxTVGradient
    with PROXTGV, ProxTVq, ProxTVDivergence, ProxTGVSymmDeriv, ProxTGVq,
    ProxTGVDivergence auxKernels.cl:1141-1560, forward differences):
      q <- P_alpha0(q + sigma2 (D x - v)),  rhs <- rhs - div q,
      r <- P_alpha1(r + sigma2 E v),
      v1 = v + tau (q + div_sym r),  v <- v1 + theta (v1 - v).
    3-D (three_d): v = (vx, vy, vz), r = (rxx, ryy, rzz, rxy, rxz, ryz);
    2-D (use2DTGV): v = (vx, vy), r = (rxx, ryy, rxy), and the z difference
    of x enters q without a v term.  P: the per-voxel L2 ball (off-diagonal
    terms counted twice) or the max-norm ball.  Arrays (k, N), x fastest;
    returns (q, r, v, rhs)."""
    def img(a):
        return np.asarray(a, dtype=np.float64).reshape(shape, order='F')

    def flat(a):
        return a.ravel(order='F')
    X = img(x)
    Q = [img(a) for a in np.asarray(q, dtype=np.float64).reshape(3, -1)]
    nr = 6 if three_d else 3
    nv = 3 if three_d else 2
    R = [img(a) for a in np.asarray(r, dtype=np.float64).reshape(nr, -1)]
    V = [img(a) for a in np.asarray(v, dtype=np.float64).reshape(nv, -1)]
    # TV part with v
    g = [_diff(X, a, True) for a in range(3)]
    for a in range(nv):
        g[a] = g[a] - V[a]
    Qn = [Q[a] + sigma2 * g[a] for a in range(3)]
    nq = np.sqrt(Qn[0] ** 2 + Qn[1] ** 2 + Qn[2] ** 2) if l2 else np.maximum(np.abs(Qn[2]), np.maximum(np.abs(Qn[0]), np.abs(Qn[1])))
    sq = np.maximum(1.0, nq / alpha0)
    Qn = [a / sq for a in Qn]
    div = sum(_diff(Qn[a], a, False) for a in range(3))
    rhs_n = np.asarray(rhs, dtype=np.float64) - flat(div)
    # symmetric derivative of v
    if three_d:
        E = [_diff(V[0], 0, True), _diff(V[1], 1, True), _diff(V[2], 2, True),
             0.5 * (_diff(V[0], 1, True) + _diff(V[1], 0, True)),
             0.5 * (_diff(V[0], 2, True) + _diff(V[2], 0, True)),
             0.5 * (_diff(V[1], 2, True) + _diff(V[2], 1, True))]
    else:
        E = [_diff(V[0], 0, True), _diff(V[1], 1, True), 0.5 * (_diff(V[0], 1, True) + _diff(V[1], 0, True))]
    Rn = [R[k] + sigma2 * E[k] for k in range(nr)]
    if three_d:
        dg, od = Rn[:3], Rn[3:]
    else:
        dg, od = Rn[:2] + [np.zeros_like(Rn[0])], Rn[2:] + [np.zeros_like(Rn[0])] * 2
    if l2:
        nrm = np.sqrt(dg[0] ** 2 + dg[1] ** 2 + dg[2] ** 2 + 2 * (od[0] ** 2 + od[1] ** 2 + od[2] ** 2))
        sr = np.maximum(1.0, nrm / alpha1)
    else:
        m = np.maximum(np.abs(od[2]), np.maximum(np.abs(od[1]), np.maximum(np.abs(od[0]), np.maximum(
            np.abs(dg[2]), np.maximum(np.abs(dg[0]), np.abs(dg[1]))))))
        sr = np.maximum(m / alpha1, 1.0)
    Rn = [a / sr for a in Rn]
    # v update with the divergence of the symmetric tensor
    if three_d:
        dv = [_diff(Rn[0], 0, False) + _diff(Rn[3], 1, False) + _diff(Rn[4], 2, False),
              _diff(Rn[1], 1, False) + _diff(Rn[3], 0, False) + _diff(Rn[5], 2, False),
              _diff(Rn[2], 2, False) + _diff(Rn[4], 0, False) + _diff(Rn[5], 1, False)]
    else:
        dv = [_diff(Rn[0], 0, False) + _diff(Rn[2], 1, False), _diff(Rn[1], 1, False) + _diff(Rn[2], 0, False)]
    Vn = []
    for a in range(nv):
        v1 = V[a] + tau * (Qn[a] + dv[a])
        Vn.append(v1 + theta * (v1 - V[a]))
    return (np.stack([flat(a) for a in Qn]), np.stack([flat(a) for a in Rn]), np.stack([flat(a) for a in Vn]),
            rhs_n)


# ---------------------------------------------------------------------------
# TV gradient variants of TVKernel (auxKernels.cl:1733-1990): the image read
# edge-clamped (the texture path), the anatomical reference S read as zero
# beyond the image (its buffer path).  variant: 'satv' (TVtype 4), 'tvw1'
# (TVtype 6), 'anat1' (anatomical TVtype 1, S = the 9 tensor channels),
# 'anat2' (anatomical TVtype 2, S = the reference image, weight C), 'apls'
# (anatomical TVtype 5 and APLS, S = the reference image, C = eta).
# ---------------------------------------------------------------------------

def _clamped(U, dx, dy, dz):
    nx, ny, nz = U.shape
    ix = np.clip(np.arange(nx) + dx, 0, nx - 1)
    iy = np.clip(np.arange(ny) + dy, 0, ny - 1)
    iz = np.clip(np.arange(nz) + dz, 0, nz - 1)
    return U[ix][:, iy][:, :, iz]


def _zero_beyond(S, dx, dy, dz):
    """S shifted by +1 along one axis with zero past the last voxel."""
    out = np.zeros_like(S)
    if dx:
        out[:-1] = S[1:]
    elif dy:
        out[:, :-1] = S[:, 1:]
    else:
        out[:, :, :-1] = S[:, :, 1:]
    return out


def tv_gradient_variant(u, shape, variant, smooth, beta, sigma=1.0, C=0.0, S=None):
    nx, ny, nz = shape
    U = np.asarray(u, dtype=np.float64).reshape(shape, order='F')
    c = U
    P = [_clamped(U, 1, 0, 0), _clamped(U, 0, 1, 0), _clamped(U, 0, 0, 1)]
    M = [_clamped(U, -1, 0, 0), _clamped(U, 0, -1, 0), _clamped(U, 0, 0, -1)]
    ui = (_clamped(U, -1, 1, 0), _clamped(U, -1, 0, 1))
    uj = (_clamped(U, 1, -1, 0), _clamped(U, 0, -1, 1))
    uk = (_clamped(U, 1, 0, -1), _clamped(U, 0, 1, -1))
    u1 = (c - M[0], ui[0] - M[0], ui[1] - M[0])
    u2 = (uj[0] - M[1], c - M[1], uj[1] - M[1])
    u3 = (uk[0] - M[2], uk[1] - M[2], c - M[2])

    def sq(v, w=(1.0, 1.0, 1.0)):
        return np.sqrt(w[0] * v[0] ** 2 + w[1] * v[1] ** 2 + w[2] * v[2] ** 2 + smooth)

    if variant == 'satv':
        g = 0.0
        for a in range(3):
            for nb in (P[a], M[a]):
                d = c - nb
                ua = d / (np.abs(d) + smooth)
                g = g + ua - ua / (np.abs(d) / sigma + 1.0)
        return (beta * g).ravel(order='F')
    if variant == 'tvw1':
        u4 = (P[0] - c, P[1] - c, P[2] - c)

        def wts(v):
            return tuple(np.exp(-(x / sigma) ** 2) for x in v)
        w4, w1, w2, w3 = wts(u4), wts(u1), wts(u2), wts(u3)
        g = (-(w4[0] * u4[0] + w4[1] * u4[1] + w4[2] * u4[2]) / sq(u4, w4) + w1[0] * (c - M[0]) / sq(u1, w1)
             + w2[1] * (c - M[1]) / sq(u2, w2) + w3[1] * (c - M[2]) / sq(u3, w3))
        return (beta * g).ravel(order='F')
    if variant == 'anat1':
        s = [np.asarray(S, dtype=np.float64)[k * nx * ny * nz:(k + 1) * nx * ny * nz].reshape(shape, order='F')
             for k in range(9)]

        def pv(v):
            return np.sqrt(v[0] ** 2 * s[0] + v[1] ** 2 * s[4] + v[2] ** 2 * s[8] + (s[1] + s[3]) * v[0] * v[1]
                           + (s[2] + s[6]) * v[0] * v[2] + (s[5] + s[7]) * v[1] * v[2] + smooth)
        val = (P[0] - c, P[1] - c, P[2] - c)
        dx = s[0] * 2 * (c - M[0]) + (s[3] + s[1]) * u1[1] + (s[2] + s[6]) * u1[2]
        dy = s[4] * 2 * (c - M[1]) + (s[5] + s[7]) * u2[2] + (s[3] + s[1]) * u2[0]
        dz = s[8] * 2 * (c - M[2]) + (s[6] + s[2]) * u3[0] + (s[5] + s[7]) * u3[1]
        d = ((s[1] + s[2] + s[3] + s[6]) * val[0] + (s[1] + s[3] + s[5] + s[7]) * val[1]
             + (s[2] + s[5] + s[6] + s[7]) * val[2] + 2 * (s[0] * val[0] + s[4] * val[1] + s[8] * val[2]))
        g = 0.5 * (d / pv(val) + dx / pv(u1) + dy / pv(u2) + dz / pv(u3))
        return (beta * g).ravel(order='F')
    R = np.asarray(S, dtype=np.float64).reshape(shape, order='F')
    Rp = (_zero_beyond(R, 1, 0, 0), _zero_beyond(R, 0, 1, 0), _zero_beyond(R, 0, 0, 1))
    apu = (P[0] - c, P[1] - c, P[2] - c)
    if variant == 'anat2':
        aS = (Rp[0] - R, Rp[1] - R, Rp[2] - R)
        p0 = np.sqrt(apu[0] ** 2 + apu[1] ** 2 + apu[2] ** 2 + C * (aS[0] ** 2 + aS[1] ** 2 + aS[2] ** 2) + smooth)
        g = ((3 * c - P[0] - P[1] - P[2]) / p0 + (c - M[0]) / sq(u1) + (c - M[1]) / sq(u2) + (c - M[2]) / sq(u3)
             + 1e-7)
        return (beta * g).ravel(order='F')
    if variant == 'apls':
        e = (Rp[0] - R, Rp[1] - R, Rp[2] - R)
        en = np.sqrt(e[0] ** 2 + e[1] ** 2 + e[2] ** 2 + C * C)
        e = (e[0] / en, e[1] / en, e[2] / en)
        apuR = Rp[0] * apu[0] + Rp[1] * apu[1] + Rp[2] * apu[2]
        p0 = np.sqrt(apu[0] ** 2 + apu[1] ** 2 + apu[2] ** 2 - apuR ** 2 + smooth)

        def pr(v):
            r = Rp[0] * v[0] + Rp[1] * v[1] + Rp[2] * v[2]
            return np.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2 + r * r + smooth)

        def edot(v):
            return e[0] * v[0] + e[1] * v[1] + e[2] * v[2]
        g = 0.5 * ((6 * c - 2 * (P[0] + P[1] + P[2]) + 2 * edot((c - P[0], c - P[1], c - P[2])) * (e[0] + e[1] + e[2]))
                   / p0 + 2 * (u1[0] - e[0] * edot(u1)) / pr(u1) + 2 * (u2[1] - e[1] * edot(u2)) / pr(u2)
                   + 2 * (u3[2] - e[2] * edot(u3)) / pr(u3) + 1e-7)
        return (beta * g).ravel(order='F')
    raise ValueError(variant)


def tv_anatomical_tensor(ref, shape, T):
    """The 9 channels of the anatomical TV type-1 weighting (prepass.py:496-
    533, assembleS): per voxel B = I - (1 - gamma) nu nu^T with nu the unit
    forward-difference gradient of the reference image and gamma =
    exp(-|grad|^2 / T^2); channels k = 3 row + col, each an image (x fastest)."""
    nx, ny, nz = shape
    a = np.asarray(ref, dtype=np.float32).reshape(shape, order='F')
    f = np.concatenate((-np.diff(a, axis=1), np.zeros((nx, 1, nz), np.float32)), axis=1).ravel('F')
    g = np.concatenate((-np.diff(a, axis=0), np.zeros((1, ny, nz), np.float32)), axis=0).ravel('F')
    h = np.concatenate((-np.diff(a, axis=2), np.zeros((nx, ny, 1), np.float32)), axis=2).ravel('F')
    gv = np.vstack((f, g, h))
    gn = np.linalg.norm(gv, axis=0)
    gamma = np.exp(-gn ** 2 / (T ** 2))
    out = np.empty((9, gn.size), dtype=np.float32)
    eye = np.eye(3)
    nu = np.where(gn > 0, gv / np.where(gn > 0, gn, 1.0), 0.0)
    for r in range(3):
        for col in range(3):
            # float32 (1 - gamma) times the float32 outer product, then the
            # FP64 subtraction from the identity, stored as float32
            out[3 * r + col] = (eye[r, col] - np.where(gn > 0, (np.float32(1.0) - gamma) * (nu[r] * nu[col]), 0.0))
    return out.ravel()


# ---------------------------------------------------------------------------
# Anisotropic-diffusion prior (priors.h:226-237): grad = (u - AD(u)) / (AD(u)
# + epps), or u - AD(u) with med_no_norm, AD = ArrayFire's anisotropicDiffusion
# (af::anisotropicDiffusion, ArrayFire 3.x; ArrayFire is not part of the
# reference tree).  Restated from the published schemes ArrayFire implements:
# each slice (the third dimension is a batch) diffused in 2-D with its edges
# replicated; per iteration u <- u + dt delta with the conductance c(g2) =
# exp(-g2 / K^2) (exponential flux) or 1 / (1 + g2 / K^2) (quadratic), g2
# the squared gradient at the half-way points (the difference across, plus a
# quarter of the squared mean of the two central differences along);
# gradient diffusion (Perona-Malik): delta = sum over the two axes of
# c_f d_f - c_b d_b; modified curvature diffusion (Whitaker-Xue): the fluxes
# c d / sqrt(1e-10 + g2), their divergence `speed` times the upwind gradient
# magnitude.  Parity unpinned: no reference output of this path exists here.
# ---------------------------------------------------------------------------

def ad_smooth(u, shape, dt, K, niter, exp_flux=True, mcde=True):
    U = np.asarray(u, dtype=np.float64).reshape(shape, order='F')
    inv = 1.0 / (float(K) * float(K))

    def cond(g2):
        return np.exp(-g2 * inv) if exp_flux else 1.0 / (1.0 + g2 * inv)
    for _ in range(int(niter)):
        P = np.pad(U, ((1, 1), (1, 1), (0, 0)), mode='edge')
        C = P[1:-1, 1:-1]
        E, W = P[2:, 1:-1], P[:-2, 1:-1]
        S, N = P[1:-1, 2:], P[1:-1, :-2]
        SE, NE, SW, NW = P[2:, 2:], P[2:, :-2], P[:-2, 2:], P[:-2, :-2]
        cx, cy = 0.5 * (E - W), 0.5 * (S - N)
        dfx, dbx, dfy, dby = E - C, C - W, S - C, C - N
        gfx = dfx ** 2 + 0.25 * (cy + 0.5 * (SE - NE)) ** 2
        gbx = dbx ** 2 + 0.25 * (cy + 0.5 * (SW - NW)) ** 2
        gfy = dfy ** 2 + 0.25 * (cx + 0.5 * (SE - SW)) ** 2
        gby = dby ** 2 + 0.25 * (cx + 0.5 * (NE - NW)) ** 2
        if not mcde:
            delta = cond(gfx) * dfx - cond(gbx) * dbx + cond(gfy) * dfy - cond(gby) * dby
        else:
            speed = (cond(gfx) * dfx / np.sqrt(1e-10 + gfx) - cond(gbx) * dbx / np.sqrt(1e-10 + gbx) +
                     cond(gfy) * dfy / np.sqrt(1e-10 + gfy) - cond(gby) * dby / np.sqrt(1e-10 + gby))
            up = (np.minimum(dbx, 0) ** 2 + np.maximum(dfx, 0) ** 2 + np.minimum(dby, 0) ** 2 +
                  np.maximum(dfy, 0) ** 2)
            dn = (np.maximum(dbx, 0) ** 2 + np.minimum(dfx, 0) ** 2 + np.maximum(dby, 0) ** 2 +
                  np.minimum(dfy, 0) ** 2)
            delta = np.sqrt(np.where(speed > 0, up, dn)) * speed
        U = C + dt * delta
    return U.ravel(order='F')


def ad_gradient(u, shape, dt, K, niter, exp_flux=True, mcde=True, epps=1e-8, no_norm=False):
    """The AD prior's gradient (priors.h:226-237), weight not included."""
    uu = np.asarray(u, dtype=np.float64)
    a = ad_smooth(uu, shape, dt, K, niter, exp_flux, mcde)
    return uu - a if no_norm else (uu - a) / (a + epps)
