"""The detector-row filters of the filtering-based measurement preconditioner
(options.precondTypeMeas[1] with PDHG).

``ramp_filter`` follows omegatomo/reconstruction/rampfilt.py:10-57 (rampFilt:
the ramp |f| times the chosen window, zero above the cut-off, mirrored to N
taps), with its arithmetic types, so that the filter equals the reference's
bit for bit; ``pdhg_row_filters`` the prepass (prepass.py:1121-1136): Nf the
power of two at or above the detector rows, filter0 = rampFilt with its zero
frequency set to 1e-6, and the dual step's 1 + sigma filter0.  The kernels
filter by circular convolution, so both are returned as their real
time-domain taps (ifft).

``image_filter_2d`` builds the filter of the filtering-based image
preconditioner (options.precondTypeImage[5]): Nf = 2^ceil(log2 Nx)
(prepass.py:1106-1109) and F = f f^T / max(f f^T), f = rampFilt(Nf, ...),
the 2-D filter rampFilt.m:65-69 forms.  The reference's Python rampFilt with
use2D (rampfilt.py:55-58) tiles the 1-D array into one row of Nf^2 values and
builds an (Nf^2, Nf^2) product whose first Nf^2 values -- all the library
reads as its Nf x Nf filter (libHeader.h:1059) -- are f[0] f = 0, so through
that path the preconditioner zeroes the gradient; the filter here is the
MATLAB path's.  F is separable, so the kernels apply it as two 1-D
convolutions with the taps real(ifft(f)) / sqrt(max(f f^T)).
"""
from __future__ import annotations

import numpy as np


def ramp_filter(N, window="hamming", c=1.0, sigma=0.25):
    """rampFilt(N, window, c, sigma) (1-D): float32, N taps."""
    filt = np.linspace(0, N, int(N) // 2 + 1, dtype=np.float32) / N
    w = 2 * np.pi * np.arange(filt.shape[0]) / N
    if window == 'hamming':
        w = (.54 + .46 * np.cos(w / c))
        filt[1:] *= w[1:]
    elif window == 'hann':
        w = (.5 + .5 * np.cos(w / c))
        filt[1:] *= w[1:]
    elif window == 'blackman':
        w = (.42659 - .49656 * np.cos(w / c) + .076849 * np.cos(2 * w / c))
        filt[1:] *= w[1:]
    elif window == 'nuttal':
        w = (.355768 - .487396 * np.cos(w / c) + .144232 * np.cos(2 * w / c) - .012604 * np.cos(3 * w / c))
        filt[1:] *= w[1:]
    elif window == 'gaussian':
        # the reference fixes this window's width at 0.1 (its sigma argument is not used)
        s = 0.1
        w = np.exp((-1 / 2) * (((np.arange(filt.shape[0] - 1, -1, -1) - N / 2) / (s * (N / 2))) ** 2))
        filt[1:] *= w[1:]
    elif window == 'shepp-logan':
        with np.errstate(invalid='ignore', divide='ignore'):  # 0 / 0 at the zero frequency, not used
            w = np.sin(w / (2 * c)) / (w / (2 * c))
        filt[1:] *= w[1:]
    elif window == 'cosine':
        filt[1:] *= np.cos(w[1:] / (2 * c))
    elif window == 'parzen':
        # an integer array, as in the reference: the window values are truncated
        L = N + 1
        w = np.arange(filt.shape[0])
        a = np.abs(w) <= L / 4
        w[a] = 1 - 6 * (w[a] / (L / 2)) ** 2 * (1 - np.abs(w[a]) / (L / 2))
        b = np.logical_and(np.abs(w) > L / 4, np.abs(w) <= L / 2)
        w[b] = 2 * (1 - np.abs(w[b]) / (L / 2)) ** 3
        filt[1:] *= w[1:]
    filt[w > np.pi * c] = 0
    if N % 2:
        filt = np.concatenate((filt, filt[-2::-1]))
    else:
        filt = np.concatenate((filt, filt[-2:0:-1]))
    return filt


def pdhg_row_filters(n_rows, sigma, window="hamming", c=1.0, fsigma=0.25):
    """(Nf, filter0, Ffilter, h, hinv): the prepass's filters for n_rows
    detector rows and the dual step sigma, with h = real(ifft(filter0)) and
    hinv = real(ifft(1 / Ffilter)) as float32 taps."""
    nf = int(2 ** np.ceil(np.log2(n_rows)))
    filter0 = ramp_filter(nf, window, c, fsigma)
    filter0[0] = 1e-6
    filter0 = filter0.astype(np.float32)
    ff = np.fft.ifft(filter0) * float(sigma)
    ff[0] = ff[0] + 1
    ffilter = np.real(np.fft.fft(ff)).astype(np.float32)
    h = np.real(np.fft.ifft(filter0.astype(np.float64))).astype(np.float32)
    hinv = np.real(np.fft.ifft(1.0 / ffilter.astype(np.float64))).astype(np.float32)
    return nf, filter0, ffilter, h, hinv


def image_filter_2d(nx, window="hamming", c=1.0, fsigma=0.25):
    """(Nf, F, h): Nf the power of two at or above nx, F the Nf x Nf float32
    filter f f^T / max(f f^T) with f = rampFilt(Nf, window, c, fsigma), and h
    the float32 1-D taps real(ifft(f)) / sqrt(max(f f^T)) whose separable
    circular convolution applies F."""
    nf = int(2 ** np.ceil(np.log2(int(nx))))
    f = ramp_filter(nf, window, c, fsigma).astype(np.float32)
    ff = np.outer(f, f).astype(np.float32)
    m = float(ff.max())
    if not m > 0:
        raise ValueError('the image filter is zero everywhere')
    F = (ff / np.float32(m)).astype(np.float32)
    h = (np.real(np.fft.ifft(f.astype(np.float64))) / np.sqrt(m)).astype(np.float32)
    return nf, F, h
