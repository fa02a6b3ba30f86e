"""Seeded synthetic diffraction series in the shapes the spot finder is
benchmarked on. The reference publishes no dataset; these stand in for Eiger
data: module gaps at the masked sentinel, a Poisson background with a diffuse
ring, and 3D Gaussian reflections Poisson-sampled on top.

Every frame regenerates on its own from (seed, frame), so any window of a long
series can be produced without the rest.

Shapes are (height, width) = (slow, fast):
  small   256 x 384    12 frames, i.i.d. background, 48 planted reflections
  4M     2162 x 2068   module gaps, ring at r0 = 600, 2000 spots per frame
  16M    4362 x 4148   module gaps, ring at r0 = 1200, 6000 spots per frame
  stills 1062 x 1028, 2162 x 2068, 3269 x 3110, 4362 x 4148 (one-frame spots)
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.special import erf

SMALL = (256, 384)
EIGER_4M = (2162, 2068)
EIGER_16M = (4362, 4148)
STILL_SHAPES = ((1062, 1028), (2162, 2068), (3269, 3110), (4362, 4148))

BOX = 6  # half-width in pixels of the box a reflection is rendered into


@dataclass
class Series:
    height: int
    width: int
    frames: int
    seed: int
    dtype: type = np.uint16
    gaps: bool = True
    background: str = "ring"        # "ring" or "flat"
    flat_lambda: float = 1.0
    ring_r0: float = 600.0
    ring_width: float = 40.0
    centre: tuple | None = None      # (x, y) beam centre; default panel middle
    spots_per_frame: float = 2000.0
    sigma_xy: tuple = (0.8, 1.5)
    sigma_z: tuple = (0.5, 1.5)
    intensity: tuple = (50.0, 5.0e4)  # log-uniform bounds, or (I, I) fixed
    stills: bool = False             # every reflection on one frame only
    planted: int | None = None       # fixed count of reflections (small config)
    min_separation: float = 0.0
    _catalogue: dict = field(default=None, repr=False)
    _lam: np.ndarray = field(default=None, repr=False)

    @property
    def masked(self) -> int:
        return int(np.iinfo(self.dtype).max)

    @property
    def clip(self) -> int:
        # One below the top of the type, which is the masked sentinel itself
        # (max - 1 and above are masked), so saturated pixels read as masked
        # exactly as a real detector's saturation value does.
        return int(np.iinfo(self.dtype).max) - 1

    # -- the reflection catalogue for the whole series ----------------------
    def catalogue(self) -> dict:
        if self._catalogue is not None:
            return self._catalogue
        rng = np.random.default_rng([self.seed, 0xC47A])
        if self.planted is not None:
            n = self.planted
            xs, ys = [], []
            margin = 8
            while len(xs) < n:
                x = rng.uniform(margin, self.width - margin)
                y = rng.uniform(margin, self.height - margin)
                if all((x - a) ** 2 + (y - b) ** 2 >= self.min_separation ** 2
                       for a, b in zip(xs, ys)):
                    xs.append(x)
                    ys.append(y)
            x = np.array(xs)
            y = np.array(ys)
        else:
            n = int(round(self.spots_per_frame * self.frames))
            x = rng.uniform(0, self.width, n)
            y = rng.uniform(0, self.height, n)
        z = rng.integers(0, self.frames, n)
        sxy = rng.uniform(*self.sigma_xy, n) if self.sigma_xy[0] != self.sigma_xy[1] \
            else np.full(n, self.sigma_xy[0])
        sz = rng.uniform(*self.sigma_z, n) if self.sigma_z[0] != self.sigma_z[1] \
            else np.full(n, self.sigma_z[0])
        lo, hi = self.intensity
        inten = np.exp(rng.uniform(np.log(lo), np.log(hi), n)) if lo != hi else np.full(n, lo)
        order = np.argsort(z, kind="stable")
        self._catalogue = dict(x=x[order], y=y[order], z=z[order], sxy=sxy[order],
                               sz=sz[order], I=inten[order])
        return self._catalogue

    def lam(self) -> np.ndarray:
        if self._lam is not None:
            return self._lam
        if self.background == "flat":
            self._lam = np.full((self.height, self.width), self.flat_lambda)
        else:
            cx, cy = self.centre if self.centre is not None else (self.width / 2, self.height / 2)
            yy, xx = np.mgrid[0:self.height, 0:self.width]
            r = np.hypot(xx + 0.5 - cx, yy + 0.5 - cy)
            self._lam = 0.3 + 2.0 * np.exp(-(((r - self.ring_r0) / self.ring_width) ** 2))
        return self._lam

    def gap_mask(self) -> np.ndarray:
        rows = (np.arange(self.height) % 551) >= 514
        cols = (np.arange(self.width) % 1040) >= 1030
        return rows[:, None] | cols[None, :]

    # -- one frame ----------------------------------------------------------
    def frame(self, f: int) -> np.ndarray:
        rng = np.random.default_rng([self.seed, 1 + f])
        counts = rng.poisson(self.lam()).astype(np.float64)
        cat = self.catalogue()
        if self.stills:
            lo = np.searchsorted(cat["z"], f, "left")
            hi = np.searchsorted(cat["z"], f, "right")
        else:
            lo = np.searchsorted(cat["z"], f - 6, "left")
            hi = np.searchsorted(cat["z"], f + 6, "right")
        if hi > lo:
            self._render(counts, rng, f, slice(lo, hi))
        np.minimum(counts, self.clip, out=counts)
        img = counts.astype(self.dtype)
        if self.gaps:
            img[self.gap_mask()] = self.masked
        return img

    def _render(self, counts, rng, f, sel):
        cat = self.catalogue()
        x, y, z = cat["x"][sel], cat["y"][sel], cat["z"][sel]
        sxy, sz, inten = cat["sxy"][sel], cat["sz"][sel], cat["I"][sel]
        if self.stills:
            wz = np.ones(len(x))
        else:
            zc = z + 0.5
            a = (f - zc) / (np.sqrt(2.0) * sz)
            b = (f + 1 - zc) / (np.sqrt(2.0) * sz)
            wz = 0.5 * (erf(b) - erf(a))
        keep = wz > 1e-6
        x, y, sxy, inten, wz = x[keep], y[keep], sxy[keep], inten[keep], wz[keep]
        if len(x) == 0:
            return
        x0 = np.floor(x).astype(np.int64) - BOX
        y0 = np.floor(y).astype(np.int64) - BOX
        off = np.arange(2 * BOX + 1)
        px = x0[:, None] + off[None, :]
        py = y0[:, None] + off[None, :]
        s2 = np.sqrt(2.0) * sxy[:, None]
        wx = 0.5 * (erf((px + 1 - x[:, None]) / s2) - erf((px - x[:, None]) / s2))
        wy = 0.5 * (erf((py + 1 - y[:, None]) / s2) - erf((py - y[:, None]) / s2))
        expected = (inten * wz)[:, None, None] * wy[:, :, None] * wx[:, None, :]
        sample = rng.poisson(expected)
        yy = np.broadcast_to(py[:, :, None], sample.shape)
        xx = np.broadcast_to(px[:, None, :], sample.shape)
        ok = (yy >= 0) & (yy < self.height) & (xx >= 0) & (xx < self.width) & (sample > 0)
        np.add.at(counts, (yy[ok], xx[ok]), sample[ok])

    def frames_array(self, start: int, count: int) -> np.ndarray:
        return np.stack([self.frame(f) for f in range(start, start + count)])


def small(seed: int = 0x5EED0000) -> Series:
    """256 x 384 x 12, i.i.d. lambda = 1, 48 reflections of 2000 counts,
    sigma_xy 1.0, sigma_z 0.7, at least 8 px from the border and each other."""
    return Series(256, 384, 12, seed, gaps=False, background="flat", flat_lambda=1.0,
                  sigma_xy=(1.0, 1.0), sigma_z=(0.7, 0.7), intensity=(2000.0, 2000.0),
                  planted=48, min_separation=8.0)


def eiger_4m(frames: int = 100, seed: int = 0x5EED0001) -> Series:
    return Series(*EIGER_4M, frames, seed, ring_r0=600.0, centre=(1034.0, 1081.0),
                  spots_per_frame=2000.0)


def eiger_16m(frames: int = 3600, seed: int = 0x5EED0002, dtype=np.uint16) -> Series:
    hi = 2.0e6 if dtype == np.uint32 else 5.0e4
    return Series(*EIGER_16M, frames, seed, dtype=dtype, ring_r0=1200.0,
                  spots_per_frame=6000.0, intensity=(50.0, hi))


def still(shape, frames: int = 500, seed: int = 0x5EED0003) -> Series:
    h, w = shape
    return Series(h, w, frames, seed + h, ring_r0=600.0, stills=True,
                  spots_per_frame=0.5 * h * w / 1000.0)
