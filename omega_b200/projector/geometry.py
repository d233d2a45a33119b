"""Scanner, sinogram and voxel-grid geometry for the projector surface.

Host-side restatement of the geometry that OMEGA computes once, before any
projection runs.  Every function here produces arrays that must equal the
reference's bit for bit (they define the ray end points the kernels trace and
the order of the measurements), so each one keeps the reference's arithmetic
order and its float32/float64 promotions:

* ``ring_detector_xy``      <- omegatomo/projector/detcoord.py:398-558 (computeCoordinates)
* ``detector_coordinates``  <- detcoord.py:326-396 (detectorCoordinates)
* ``sinogram_xy``           <- detcoord.py:589-700 (formDetectorIndices, sinogramCoordinates2D)
* ``sinogram_z``            <- detcoord.py:703-898 (sinogramCoordinates3D)
* ``ct_source_detector``    <- detcoord.py:22-121 (CTDetSource), 123-188 (setCTCoordinates),
                               190-218 (CTDetectorCoordinates)
* ``subset_indices``        <- omegatomo/projector/indices.py:20-275 (indexMaker)
* ``voxel_grid``            <- omegatomo/projector/coordinates.py:22-91 (computePixelSize)
* ``projector_scaling``     <- coordinates.py:209-269 (computeProjectorScalingValues)
* ``tof_centers``           <- omegatomo/projector/proj.py:685-705
* ``geom5_table``           <- omegatomo/projector/init.py:6-37 (computeGeom5)
"""
from __future__ import annotations

import math

import numpy as np


# ---------------------------------------------------------------------------
# PET: transaxial crystal positions on the ring
# ---------------------------------------------------------------------------

def _jump(sx, sy, cr_p, ang_prev, ang_cur, gap_x, gap_y):
    """Position of the first crystal of a new block (crosses the block gap).

    Same expression order as detcoord.py:455-460.
    """
    cx = sx - (cr_p * 0.5) * np.cos(np.radians(ang_cur)) - gap_x * np.cos(
        np.radians(ang_prev)) - gap_x * np.cos(np.radians(ang_cur)) - (
        cr_p * 0.5) * np.cos(np.radians(ang_prev))
    cy = sy + (cr_p * 0.5) * np.sin(np.radians(ang_cur)) + gap_y * np.sin(
        np.radians(ang_prev)) + gap_y * np.sin(np.radians(ang_cur)) + (
        cr_p * 0.5) * np.sin(np.radians(ang_prev))
    return cx, cy


def _step(sx, sy, cr_p, ang_cur):
    """Position of the next crystal inside a block (detcoord.py:462-463)."""
    return sx - cr_p * np.cos(np.radians(ang_cur)), sy + cr_p * np.sin(np.radians(ang_cur))


def ring_detector_xy(blocks_per_ring, transaxial_multip, cryst_per_block, diameter, cr_p,
                     use_pseudo):
    """Transaxial (x, y) of every crystal on one ring, float32.

    Walks a quarter of the ring block by block and mirrors it, exactly as
    detcoord.py:398-558 does.  Each crystal position is rounded to float32
    before it seeds the next one, as in the reference.
    """
    cpb_orig = cryst_per_block
    extra = 1 if use_pseudo else 0
    cpb = cryst_per_block + extra
    nb = blocks_per_ring * transaxial_multip
    angle = np.arange(90, -271, -360 / nb)
    widths = cpb_orig * cr_p * np.cos(np.radians(angle[:(nb // 2 + 1)]))
    widthsy = cpb_orig * cr_p * np.sin(np.radians(angle[:(nb // 2)]))
    gap_x = (diameter - np.sum(np.abs(widths))) / np.sum(np.cos(np.radians(angle[:(nb // 2 + 1)]))) / 2
    gap_y = (diameter - np.sum(np.abs(widthsy))) / np.sum(np.abs(np.sin(np.radians(angle[:(nb // 2)])))) / 2
    sx = diameter / 2.
    sy = -(cpb_orig / 2. + 0.5) * cr_p
    x = np.zeros(nb * cpb, dtype=np.float32)
    y = np.zeros(nb * cpb, dtype=np.float32)
    ii = 0

    def walk_block(blk, sx, sy, ii):
        for c in range(1, cpb + 1):
            if blk > 0 and c == 1:
                x[ii], y[ii] = _jump(sx, sy, cr_p, angle[blk - 1], angle[blk], gap_x, gap_y)
            else:
                x[ii], y[ii] = _step(sx, sy, cr_p, angle[blk])
            if c == cpb:
                sx = x[ii] + cr_p * np.cos(np.radians(angle[blk])) * extra
                sy = y[ii] - cr_p * np.sin(np.radians(angle[blk])) * extra
            else:
                sx = x[ii]
                sy = y[ii]
            ii += 1
        return sx, sy, ii

    blk = 0
    for blk in range(0, math.ceil(nb / 4)):
        sx, sy, ii = walk_block(blk, sx, sy, ii)

    quarter = (nb * cpb) // 4
    half = (nb * cpb) // 2
    if nb % 4 == 0:
        blk += 1
        x[ii], y[ii] = _jump(sx, sy, cr_p, angle[blk - 1], angle[blk], gap_x, gap_y)
        sx, sy = x[ii], y[ii]
        ii += 1
        for _ in range(2, cpb + 1):
            x[ii], y[ii] = _step(sx, sy, cr_p, angle[blk])
            sx, sy = x[ii], y[ii]
            ii += 1
        if use_pseudo:
            ii -= 1
            sx = x[ii] + cr_p * np.cos(np.radians(angle[blk])) * extra
            sy = y[ii] - cr_p * np.sin(np.radians(angle[blk])) * extra
            first = blk + 1
            ii += 1
            for blk in range(first, nb + 1):
                sx, sy, ii = walk_block(blk, sx, sy, ii)
        else:
            x[ii:ii + quarter] = -(np.flip(x[:quarter]))
            y[ii:ii + quarter] = np.flip(y[:quarter])
            x[ii + quarter:] = np.flip(x[cpb:half])
            y[ii + quarter:] = -(y[cpb:half])
    else:
        if use_pseudo:
            first = blk + 1
            for blk in range(first, nb + 1):
                sx, sy, ii = walk_block(blk, sx, sy, ii)
        else:
            q2 = quarter + cpb // 2
            x[ii:ii + q2] = -(np.flip(x[:q2]))
            y[ii:ii + q2] = np.flip(y[:q2])
            x[ii + q2:] = np.flip(x[cpb:half])
            y[ii + q2:] = -(y[cpb:half])
    return x, y


def detector_coordinates(o):
    """Ring crystal (x, y) with DOI, flip and detector-space rotation applied
    (detcoord.py:326-396; single-layer scanners)."""
    cpb = o.cryst_per_block
    if isinstance(cpb, np.ndarray):
        cpb = cpb.ravel()[0].item()
    diameter = o.diameter + o.DOI * 2
    if o.det_w_pseudo > o.det_per_ring:
        x, y = ring_detector_xy(o.blocks_per_ring, o.transaxial_multip, cpb, diameter, o.cr_p, True)
    else:
        x, y = ring_detector_xy(o.blocks_per_ring, o.transaxial_multip, cpb, diameter, o.cr_p, False)
    if o.flip_image:
        x = np.flip(x)
        y = np.flip(y)
    if o.offangle != 0:
        x = np.roll(x, int(np.round(o.offangle)))
        y = np.roll(y, int(np.round(o.offangle)))
    return x, y


def _detector_pairs(det_w_pseudo):
    """All unordered crystal pairs (a <= b), 0-based, in the order of
    detcoord.py:561-587 (formDetectorIndices)."""
    n = det_w_pseudo
    a = np.repeat(np.arange(n), np.arange(n, 0, -1))
    starts = np.repeat(np.arange(n), np.arange(n, 0, -1))
    offs = np.arange(a.size) - np.repeat(np.cumsum(np.r_[0, np.arange(n, 1, -1)]), np.arange(n, 0, -1))
    b = starts + offs
    return np.column_stack((a, b)).astype(np.int64)


def sinogram_xy(o, x, y):
    """Sinogram-bin LOR end points in the transaxial plane.

    Returns two (Ndist*Nang, 2) float32 arrays: column 0 is the first crystal,
    column 1 the second, bins in Fortran (radial fastest) order.
    Restates detcoord.py:589-700 (sinogramCoordinates2D) for one layer.
    """
    dwp = o.det_w_pseudo
    nang = o.Nang
    ndist = o.Ndist
    mashing = 1
    if nang < dwp // 2:
        mashing = dwp // nang // 2
        nang = nang * mashing
    L = _detector_pairs(dwp)
    xa = np.max(L, 1)
    ya = np.min(L, 1)
    j = ((xa + ya + dwp // 2 + 1) % dwp) // 2
    b = j + dwp // 2
    i = np.abs(xa - ya - dwp // 2)
    neg = (ya < j) | (b < xa)
    i[neg] = -i[neg]
    swap = np.logical_or((j * 2) < -i, i <= ((j - dwp // 2) * 2))
    L3 = L[swap, 0].copy()
    L[swap, 0] = L[swap, 1]
    L[swap, 1] = L3
    if ndist % 2 == 0:
        acc = np.logical_and(i <= (ndist // 2 + min(0, o.ndist_side)), i >= (-ndist // 2 + max(0, o.ndist_side)))
    else:
        acc = np.logical_and(i <= ndist // 2, i >= -(ndist // 2))
    j = j // (dwp // 2 // nang)
    i = i[acc]
    j = j[acc]
    if np.min(i) < 0:
        i = i + np.abs(np.min(i))
    L = L[acc, :]
    grids = []
    for src, col in ((x, 0), (y, 0), (x, 1), (y, 1)):
        g = np.zeros((ndist, nang), dtype=np.float32, order='F')
        np.add.at(g, (i, j), src[L[:, col]])
        if mashing > 1:
            g = g.reshape(ndist, nang // mashing, mashing).mean(axis=2)
        grids.append(g)
    xs, ys, xd, yd = grids
    xo = np.column_stack((xs.ravel('F'), xd.ravel('F')))
    yo = np.column_stack((ys.ravel('F'), yd.ravel('F')))
    return xo, yo


def sinogram_z(o):
    """Axial (z_source, z_detector) of every sinogram, float64 (TotSinos, 2).

    Restates detcoord.py:703-898 (sinogramCoordinates3D) for single-layer
    scanners without ring gaps: for span > 1 each oblique sinogram averages
    the ring pairs the span combines; span 1 lists every ring pair.
    """
    cr_pz = o.cr_pz
    rings = o.rings
    nz = rings * 2 - 1
    z_length = float(rings + 1) * cr_pz
    maxz = z_length
    if o.span > 1:
        zr = np.linspace(cr_pz, z_length + cr_pz, rings + 2)[:rings]
        zr -= maxz / 2
        zr = zr.reshape(-1, 1)
        pairs = np.zeros((rings, rings, 2))
        pairs[:, :, 0] = np.tile(zr, (1, rings))
        pairs[:, :, 1] = np.tile(zr.T, (rings, 1))
        pairs = pairs.reshape(rings * rings, 2)
        nseg = ((o.ring_difference - math.ceil(o.span / 2)) // o.span) + 1
        kkj = np.zeros(nseg, dtype=int)
        for kk in range(1, nseg + 1):
            kkj[kk - 1] = np.ceil(o.span / 2) + o.span * (kk - 1)
        off = np.cumsum(o.segment_table)
        z = np.zeros((o.TotSinos, 2))
        z[:nz + 1:2, 0] = pairs[::rings + 1, 0]
        z[:nz + 1:2, 1] = pairs[::rings + 1, 1]
        count = np.zeros(o.TotSinos)
        count[:nz + 1:2] = 1
        for jh in range(0, int(np.floor(o.span / 2))):
            for c in (0, 1):
                a1 = pairs[((jh + 1) * rings)::rings + 1, c]
                end2 = ((rings - jh + 1) * rings) if c == 0 else ((rings - jh) * rings)
                a2 = pairs[(jh + 1):end2:rings + 1, c]
                z[jh + 1:off[0] - jh:2, c] = z[jh + 1:off[0] - jh:2, c] + a1 + a2
            sel = np.isin(np.arange(0, nz), np.arange(jh + 1, off[0] - jh, 2))
            m = np.full(len(count), False)
            m[:len(sel)] = sel
            count[m] += 2
        ar1 = np.arange(1, o.TotSinos + 1)
        for ih in range(1, int(len(o.segment_table) / 2) + 1):
            for jh in range(1, o.span + 1):
                k0 = kkj[ih - 1] + jh - 1
                lo_a, hi_a = off[2 * (ih - 1)] + jh - 1, off[(2 * ih) - 1] - jh + 1
                lo_b, hi_b = off[(2 * ih - 1)] + jh - 1, off[(2 * ih)] - jh + 1
                z[lo_a:hi_a:2, 0] += pairs[(k0 * rings)::rings + 1, 0]
                z[lo_b:hi_b:2, 0] += pairs[k0:((rings - kkj[ih - 1] - jh + 2) * rings):rings + 1, 0]
                z[lo_a:hi_a:2, 1] += pairs[(k0 * rings)::(rings + 1), 1]
                z[lo_b:hi_b:2, 1] += pairs[k0:((rings - kkj[ih - 1] - jh + 1) * rings):rings + 1, 1]
                count[np.isin(ar1, np.arange(off[(2 * (ih - 1))] + jh, off[(2 * ih - 1)] - jh + 2, 2))] += 1
                count[np.isin(ar1, np.arange(off[(2 * ih - 1)] + jh, off[(2 * ih)] - jh + 2, 2))] += 1
        count[count == 0] = 1
        z[:, 0] /= count
        z[:, 1] /= count
    else:
        z = np.zeros((rings ** 2, 2))
        ones = np.ones((rings, 1))
        col = np.arange(0, cr_pz * rings, cr_pz).reshape(-1, 1)
        for t in range(1, rings + 1):
            z[(t - 1) * rings:t * rings, :] = np.hstack([cr_pz * (t - 1) * ones, col])
        z[np.isnan(z)] = np.inf
        z = z - (maxz / 2 - cr_pz)
    return z


def pet_sinogram_coordinates(o):
    """(x (Ndist*Nang, 4) float32 = [xs, ys, xd, yd], z (NSinos, 2) float64)
    for sinogram data (detcoord.py:220-283, use_raw_data == 0 branch)."""
    if isinstance(o.x, np.ndarray) and o.x.size > 1 and o.y.size > 1:
        z = o.z
        if not (z.size == o.x.size) and z.size < o.nProjections:
            z = np.zeros(o.x.shape, dtype=np.float32)
        return o.x, z
    xr, yr = detector_coordinates(o)
    xs, ys = sinogram_xy(o, xr, yr)
    z = sinogram_z(o)
    if not o.NSinos == o.TotSinos:
        z = z[0:o.NSinos, :]
    x = np.column_stack((xs[:, 0], ys[:, 0], xs[:, 1], ys[:, 1]))
    return x, z


def default_segment_table(rings, span, ring_difference, nz):
    """Sinograms per segment (proj.py:662-664)."""
    st = np.concatenate((np.array(rings * 2 - 1, ndmin=1),
                         np.arange(rings * 2 - 1 - (span + 1), max(nz - ring_difference * 2, rings - ring_difference), -span * 2)))
    return np.insert(np.repeat(st[1:], 2), 0, st[0])


# ---------------------------------------------------------------------------
# CT: source and flat-panel geometry
# ---------------------------------------------------------------------------

def ct_source_detector(o):
    """Source and panel-centre positions and panel direction vectors for
    circular cone-beam CT (detcoord.py:22-188, no pitch/roll, no helical).

    Returns x (nProjections, 6) = [sx, sy, sz, dx, dy, dz] and the panel row
    direction (nProjections, 2) scaled by dPitchX, which is both ``z`` and ``uV``.
    """
    n = o.nProjections
    ang = np.asarray(o.angles).reshape(1, 1, -1)
    R = np.concatenate((np.concatenate((np.cos(ang), -np.sin(ang)), axis=1),
                        np.concatenate((np.sin(ang), np.cos(ang)), axis=1)))

    def as_arr(v):
        return v if isinstance(v, np.ndarray) else np.array(v, dtype=np.float32)

    def tile_to(v):
        v = np.asarray(v).ravel()
        if v.size == 1:
            return np.tile(v, n)
        if v.size != n:
            return np.tile(v, n // v.size)
        return v

    src_x = -o.sourceToCRot if isinstance(o.sourceToCRot, np.ndarray) else np.array(-o.sourceToCRot, dtype=np.float32)
    src_x = tile_to(src_x)
    src_y = tile_to(as_arr(o.sourceOffsetRow))
    src_z = tile_to(as_arr(o.sourceOffsetCol))
    pair = np.concatenate((src_x, src_y)).T.reshape(2, 1, -1)
    sXY = np.squeeze(np.sum(R * np.transpose(pair, (1, 0, 2)), axis=1)).T
    if isinstance(o.sourceToCRot, np.ndarray):
        det_x = o.sourceToDetector - o.sourceToCRot
    else:
        det_x = np.array(o.sourceToDetector - o.sourceToCRot, dtype=np.float32, ndmin=1)
    det_y = np.array(o.detOffsetRow, dtype=np.float32) if not isinstance(o.detOffsetRow, np.ndarray) else (
        o.detOffsetRow if o.detOffsetRow.size > 0 else 0.)
    det_z = np.array(o.detOffsetCol, dtype=np.float32) if not isinstance(o.detOffsetCol, np.ndarray) else (
        o.detOffsetCol if o.detOffsetCol.size > 0 else 0.)
    det_x = np.reshape(det_x, (-1, 1, 1))
    det_y = np.reshape(det_y, (-1, 1, 1))
    if det_x.size != src_x.size:
        det_x = np.tile(det_x, (src_x.size // det_x.size, 1, 1))
    if det_y.size != src_y.size:
        det_y = np.tile(det_y, (src_y.size // det_y.size, 1, 1))
    det_z = np.asarray(det_z)
    if det_z.size != src_z.size:
        det_z = np.tile(det_z, src_z.size // det_z.size)
    XY = np.squeeze(np.sum(R * np.concatenate((det_x.reshape(1, 1, -1) if det_x.size > 1 else det_x,
                                               det_y.reshape(1, 1, -1) if det_y.size > 1 else det_y), axis=1), axis=1)).T
    xx = np.column_stack((sXY[:, 0], XY[:, 0]))
    yy = np.column_stack((sXY[:, 1], XY[:, 1]))
    if src_z.size == 1:
        zz = np.column_stack((np.tile(src_z, det_z.size), np.reshape(det_z, (-1, 1))))
    elif det_z.size == 1:
        zz = np.column_stack((np.reshape(src_z, (-1, 1)), np.tile(det_z, src_z.size)))
    else:
        zz = np.column_stack((src_z, np.reshape(det_z, (-1, 1))))
    angles = np.asarray(o.angles).reshape(-1, 1)
    uV = np.column_stack((-np.sin(angles), np.cos(angles)))
    if o.flip_image:
        yy = -yy
        uV[:, 1] = -uV[:, 1]
    x6 = np.column_stack((xx[:, 0], yy[:, 0], zz[:, 0], xx[:, 1], yy[:, 1], zz[:, 1]))
    # the reference assigns options.z = options.uV (one array), so the pitch
    # scaling below shows in both (detcoord.py:172-182)
    uV[:, 0] = uV[:, 0] * o.dPitchX
    uV[:, 1] = uV[:, 1] * o.dPitchX
    return x6, uV, uV


# ---------------------------------------------------------------------------
# Subsets
# ---------------------------------------------------------------------------

def _prime_factors(n):
    out = []
    d = 2
    while n > 1:
        while n % d == 0:
            out.append(d)
            n //= d
        d += 1
    return out


def subset_indices(o):
    """Subset membership and order (indices.py:20-275, sinogram/projection data).

    Returns (index, nMeas) where ``nMeas`` is the (subsets, 1) int64 count per
    subset (before the cumulative sum that addProjector applies).
    """
    S = o.subsets
    ndist, nang, nsinos = o.Ndist, o.Nang, o.NSinos
    tt = np.uint64 if o.CT else np.uint32
    total = ndist * nang * nsinos
    if S > 1 and o.subsetType < 8:
        index = np.empty(0, dtype=tt)
        nmeas = np.zeros((S, 1), dtype=np.int64)
        if o.subsetType == 4:
            top = np.size(np.arange(1, nang, S))
            for i in range(S):
                osa = np.size(np.arange(i, nang, S))
                idx1 = np.tile(np.arange(i * ndist, (i + 1) * ndist, 1), (osa * nsinos)).astype(tt)
                idx1 = idx1 + np.repeat(np.arange(0, osa * nsinos, 1) * ndist * S, ndist).astype(tt)
                if nang % S > 0:
                    er = osa - 1 if osa < top else nang % S - S
                    idx1 = (np.int64(idx1) + np.int64(np.repeat((np.arange(0, nsinos - 1, 1)) * ndist * er, ndist * osa))).astype(tt)
                index = np.append(index, idx1)
                nmeas[i] = np.size(idx1)
        elif o.subsetType == 5:
            apu = np.tile((np.tile(np.arange(0, nang * ndist, ndist, dtype=tt).T[None, :], (ndist, 1))
                           + np.arange(0, ndist, dtype=tt)[:, None])[:, :, None], (1, 1, nsinos)) \
                + np.transpose(np.arange(0, nang * ndist * nsinos, nang * ndist, dtype=tt)[:, None, None], (2, 1, 0))
            apu = np.transpose(apu, (0, 2, 1)).reshape(ndist * nsinos, -1, order='F')
            for i in range(S):
                idx1 = apu[i::S, :].T.ravel('F')
                index = np.append(index, idx1)
                nmeas[i] = np.size(idx1)
        elif o.subsetType == 1:
            # column-major re-indexing (indices.py:103-107 with ind2sub/sub2ind 277-325);
            # the int64 dimension arrays make the index int64, as in the reference
            dims = np.array((nang, ndist, nsinos))
            dims2 = np.array((ndist, nang, nsinos))
            for i in range(S):
                lin = np.arange(i, total, S).astype(tt)
                K = lin // (dims[0] * dims[1])
                J = (lin - K * (dims[0] * dims[1])) // dims[0]
                I = np.mod(lin - K * (dims[0] * dims[1]), dims[0])
                idx1 = K * dims2[0] * dims2[1] + J + I * dims2[0]
                index = np.append(index, idx1)
                nmeas[i] = np.size(idx1)
        elif o.subsetType == 2:
            for i in range(S):
                idx1 = np.arange(i, total, S).astype(tt)
                index = np.append(index, idx1)
                nmeas[i] = np.size(idx1)
        elif o.subsetType == 3:
            port = total // S
            gen = np.random.default_rng() if o.seed < 0 else np.random.default_rng(o.seed)
            apu = gen.permutation(total).astype(tt)
            for i in range(S):
                idx1 = apu[port * i:-1] if i == S - 1 else apu[port * i:port * (i + 1)]
                index = np.append(index, idx1)
                nmeas[i] = np.size(idx1)
        elif o.subsetType == 0:
            val = o.nProjections // S
            val_end = o.nProjections - val * (S - 1) if total % S > 0 else val
            nmeas = np.append(np.full(S - 1, val, dtype=np.int64), val_end)
            index = np.zeros(1, dtype=tt)
        else:
            raise ValueError('Subset types 6 and 7 are not supported')
    elif (S > 1 and o.subsetType in (8, 9, 10, 11)) or S == 1:
        nproj = o.nProjections
        step = nproj // S
        modi = np.mod(nproj, S)
        uu = int(modi > 0)
        i1, i2 = 0, step + uu
        index = np.empty(0, dtype=tt)
        nmeas = np.zeros((S, 1), dtype=np.int64)
        if o.subsetType == 8 and S > 1:
            for kk in range(S):
                idx1 = np.arange(kk, nproj, S).astype(tt)
                index = np.append(index, idx1)
                nmeas[kk] = np.size(idx1)
        elif o.subsetType == 9 and S > 1:
            gen = np.random.default_rng() if o.seed < 0 else np.random.default_rng(o.seed)
            apu = gen.permutation(nproj).astype(tt)
            for kk in range(S):
                idx1 = apu[i1:i2]
                index = np.append(index, idx1)
                nmeas[kk] = np.size(idx1)
                modi = modi - 1
                if modi <= 0:
                    uu = 0
                i1 = i2
                i2 = i2 + step + uu
        elif o.subsetType == 10 and S > 1:
            raise ValueError('Subset type 10 is not supported')
        elif o.subsetType == 11 and S > 1:
            n = _prime_factors(nproj)
            n2 = np.array(n)
            nn = np.flipud(np.cumprod(np.flipud(n2[1:])))
            p = np.zeros((len(n), nproj), dtype=tt)
            for ll in range(1, len(n) + 1):
                p1 = np.arange(n[ll - 1])
                if ll == 1:
                    p1 = np.tile(p1, nproj // np.size(p1))
                else:
                    p1 = np.repeat(p1, np.prod(n[:ll - 1]))
                    p1 = np.tile(p1, nproj // np.size(p1))
                p[ll - 1, :] = p1
            order = np.zeros(nproj, dtype=tt)
            for r in range(1, nproj + 1):
                order[r - 1] = np.sum(p[:len(nn), r - 1] * nn) + p[-1, r - 1]
            for kk in range(S):
                index = np.append(index, order[i1:i2])
                nmeas[kk] = np.size(order[i1:i2])
                modi -= 1
                if modi <= 0:
                    uu = 0
                i1 = i2
                i2 = i2 + step + uu
        else:
            index = np.arange(0, nproj).astype(tt)
            nmeas[0] = index.size
        if S == 1:
            nmeas[0] = o.NSinos
    else:
        raise ValueError('Invalid subset type!')
    if o.Nt > 1:
        nmeas = np.tile(nmeas, (o.Nt, 1)) if nmeas.ndim == 2 else np.tile(nmeas, o.Nt)
    return index, nmeas


# ---------------------------------------------------------------------------
# Voxel grid and projector scales
# ---------------------------------------------------------------------------

def voxel_grid(o):
    """Voxel size d and FOV corner b per axis (coordinates.py:22-91, one volume).

    Returns (dx, dy, dz, bx, by, bz) as float32 (1,) arrays.
    """
    fov = np.column_stack((o.FOVa_x, o.FOVa_y, o.axial_fov)).astype(dtype=np.float32)
    half = -(fov) / 2
    nx = int(np.asarray(o.Nx).ravel()[0])
    ny = int(np.asarray(o.Ny).ravel()[0])
    nz = int(np.asarray(o.Nz).ravel()[0])
    xx = np.linspace(half[0, 0] + o.oOffsetX, -half[0, 0] + o.oOffsetX, nx + 1, dtype=np.float32)
    yy = np.linspace(half[0, 1] + o.oOffsetY, -half[0, 1] + o.oOffsetY, ny + 1, dtype=np.float32)
    zz = np.linspace(half[0, 2] + o.oOffsetZ, -half[0, 2] + o.oOffsetZ, nz + 1, dtype=np.float32)
    f32 = lambda v: np.array([v], dtype=np.float32)
    return f32(xx[1] - xx[0]), f32(yy[1] - yy[0]), f32(zz[1] - zz[0]), f32(xx[0]), f32(yy[0]), f32(zz[0])


def projector_scaling(o):
    """Scales for the interpolation (type 4) and distance-driven (type 5)
    projectors (coordinates.py:209-269).  Sets the attributes on ``o``."""
    o.dScaleX4 = (1. / (o.dx * o.Nx)).astype(np.float32)
    o.dScaleY4 = (1. / (o.dy * o.Ny)).astype(np.float32)
    o.dScaleZ4 = (1. / (o.dz * o.Nz)).astype(np.float32)
    if o.projector_type in (5, 15, 45, 54, 51):
        o.dSizeY = (1. / (o.dy * o.Ny)).astype(np.float32)
        o.dSizeX = (1. / (o.dx * o.Nx)).astype(np.float32)
        o.dScaleX = (1. / (o.dx * (o.Nx + 1))).astype(np.float32)
        o.dScaleY = (1. / (o.dy * (o.Ny + 1))).astype(np.float32)
        o.dScaleZ = (1. / (o.dz * (o.Nz + 1))).astype(np.float32)
        o.dSizeZBP = (o.nColsD + 1) * o.dPitchX
        o.dSizeXBP = (o.nRowsD + 1) * o.dPitchY
    if o.projector_type in (4, 14, 41, 42, 43, 44, 45, 54):
        # the CT backprojection weight; PET data (no sourceToDetector) gives inf, as in the reference, unused
        with np.errstate(divide='ignore'):
            o.kerroin = (o.dx * o.dy * o.dz) / (o.dPitchX * o.dPitchY * o.sourceToDetector)
        fov0 = float(np.asarray(o.FOVa_x).ravel()[0])
        nx0 = float(np.asarray(o.Nx).ravel()[0])
        if o.dL == 0:
            o.dL = fov0 / nx0
        else:
            o.dL = o.dL * (fov0 / nx0)
    else:
        o.kerroin = np.zeros(1, dtype=np.float32)
    if o.projector_type in (4, 5, 14, 15, 45, 54) and o.CT:
        o.use_64bit_atomics = False
        o.use_32bit_atomics = False


def tof_centers(tof_width, tof_bins, tof_offset=0.):
    """Bin centres along the LOR in mm, centre bin first then alternating
    +1, -1, +2, ... (proj.py:695-703)."""
    c = 2.99792458e11
    edges = np.linspace(-tof_width * tof_bins / 2, tof_width * tof_bins / 2, tof_bins + 1, dtype=np.float32)
    edges = edges[0:-1] + tof_width / 2.
    centers = np.zeros(np.shape(edges), dtype=np.float32, order='F')
    mid = math.floor(np.size(edges) / 2)
    centers[0] = edges[mid]
    centers[1::2] = edges[mid + 1:]
    centers[2::2] = edges[mid - 1::-1]
    if tof_offset > 0:
        centers = centers + tof_offset
    return -centers * c / 2.


def tof_sigma(tof_fwhm):
    """Gaussian sigma in mm for a timing FWHM in seconds (proj.py:694)."""
    c = 2.99792458e11
    return (c * tof_fwhm / 2.) / (2. * math.sqrt(2. * math.log(2.)))


def geom5_table(x, uv, n_rows_d, n_cols_d, dpitch_y):
    """Per-projection constants of the voxel-driven distance-driven
    backprojection, 16 float32 each: s(3), d3(3), normX(3), normY(3),
    crossP(3), upperPart(1).  Same arithmetic as init.py:6-37 (no pitch)."""
    nproj = x.size // 6
    xs = np.reshape(x, (nproj, 6)).astype(np.float32, copy=False)
    s = xs[:, 0:3]
    d = xs[:, 3:6]
    ind_x = np.float32(n_rows_d) / np.float32(2.)
    ind_y = np.float32(n_cols_d) / np.float32(2.)
    uvs = np.reshape(uv, (nproj, 2)).astype(np.float32, copy=False)
    ax = np.zeros((nproj, 3), dtype=np.float32)
    ax[:, 0] = uvs[:, 0] * ind_x
    ax[:, 1] = uvs[:, 1] * ind_x
    ay = np.zeros((nproj, 3), dtype=np.float32)
    ay[:, 2] = ind_y * np.float32(dpitch_y)
    d3 = d - ax - ay
    d2 = ax - ay
    nx = ax / np.linalg.norm(ax, axis=1, keepdims=True)
    ny = ay / np.linalg.norm(ay, axis=1, keepdims=True)
    cp = np.cross(d2, d3 - d)
    up = np.sum(cp * (s - d), axis=1, keepdims=True)
    return np.ascontiguousarray(np.hstack((s, d3, nx, ny, cp, up)).astype(np.float32)).ravel()
