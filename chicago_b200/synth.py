"""Seeded synthetic RGB24 video content for parity tests and the benchmark.

The reference ships no dataset; its encoder API takes packed R8G8B8 frames
(src/video/evx3.h:87-90), so every workload here is generated from a seed:

* background: sum of 8 random-phase 2-D sinusoids with periods uniform in
  [4, 64] px, evaluated analytically at the panned position so quarter-pel pan
  is exact; two low-frequency chroma fields tint the R/G/B channels;
* global pan with a per-frame random velocity (uniform in [-vmax, vmax],
  quantised to 1/4 px);
* ``n_rects`` rectangles (16-64 px) with their own random texture and
  independent integer velocities, wrapping around the frame;
* Gaussian noise (sigma 3) per frame and channel;
* an optional scene cut: from ``cut_at`` on, the generator restarts from a
  fresh seed.

Only numpy is used; a 1080p frame takes a few tens of milliseconds.
"""
from __future__ import annotations

import numpy as np


class Scene:
    def __init__(self, width: int, height: int, seed: int, vmax: float = 6.0,
                 n_rects: int = 4, noise_sigma: float = 3.0):
        self.w, self.h = int(width), int(height)
        self.rng = np.random.default_rng(seed)
        r = self.rng
        self.vmax = float(vmax)
        self.noise_sigma = float(noise_sigma)
        # 8 luminance sinusoids: wave vector from a period in [4, 64] px and a
        # random orientation; amplitudes sum to about 90 grey levels.
        periods = r.uniform(4.0, 64.0, size=8)
        theta = r.uniform(0.0, np.pi, size=8)
        self.kx = 2 * np.pi * np.cos(theta) / periods
        self.ky = 2 * np.pi * np.sin(theta) / periods
        self.phase = r.uniform(0.0, 2 * np.pi, size=8)
        self.amp = r.uniform(6.0, 16.0, size=8)
        # Chroma tint fields (one long-period sinusoid per channel).
        cper = r.uniform(48.0, 160.0, size=3)
        cth = r.uniform(0.0, np.pi, size=3)
        self.ckx = 2 * np.pi * np.cos(cth) / cper
        self.cky = 2 * np.pi * np.sin(cth) / cper
        self.cph = r.uniform(0.0, 2 * np.pi, size=3)
        self.camp = r.uniform(10.0, 30.0, size=3)
        self.base = r.uniform(100.0, 150.0, size=3)
        # Rectangles: size, start position, velocity, texture.
        self.rects = []
        for _ in range(n_rects):
            rw, rh = int(r.integers(16, 65)), int(r.integers(16, 65))
            x0, y0 = float(r.uniform(0, self.w)), float(r.uniform(0, self.h))
            vx, vy = (int(v) for v in r.integers(-4, 5, size=2))
            tex = r.integers(0, 256, size=(rh // 4 + 1, rw // 4 + 1, 3)).astype(np.float32)
            tex = np.repeat(np.repeat(tex, 4, axis=0), 4, axis=1)[:rh, :rw]
            self.rects.append([x0, y0, vx, vy, tex])
        self.ox = 0.0
        self.oy = 0.0

    def _background(self) -> np.ndarray:
        xs = np.arange(self.w, dtype=np.float64) + self.ox
        ys = np.arange(self.h, dtype=np.float64) + self.oy
        lum = np.zeros((self.h, self.w), dtype=np.float64)
        for k in range(8):
            # sin(a x + b y + p) = sin(a x) cos(b y + p) + cos(a x) sin(b y + p)
            ax = self.kx[k] * xs
            by = self.ky[k] * ys + self.phase[k]
            lum += self.amp[k] * (np.outer(np.cos(by), np.sin(ax)) + np.outer(np.sin(by), np.cos(ax)))
        img = np.empty((self.h, self.w, 3), dtype=np.float64)
        for c in range(3):
            ax = self.ckx[c] * xs
            by = self.cky[c] * ys + self.cph[c]
            tint = self.camp[c] * (np.outer(np.cos(by), np.sin(ax)) + np.outer(np.sin(by), np.cos(ax)))
            img[:, :, c] = self.base[c] + lum + tint
        return img

    def next_frame(self) -> np.ndarray:
        img = self._background()
        for rc in self.rects:
            x0, y0, vx, vy, tex = rc
            rh, rw = tex.shape[:2]
            xi, yi = int(x0) % self.w, int(y0) % self.h
            ys = (np.arange(rh) + yi) % self.h
            xs = (np.arange(rw) + xi) % self.w
            img[np.ix_(ys, xs)] = tex
            rc[0] = x0 + vx
            rc[1] = y0 + vy
        img += self.rng.normal(0.0, self.noise_sigma, size=img.shape)
        # Advance the pan by a random quarter-pel velocity.
        self.ox += np.round(self.rng.uniform(-self.vmax, self.vmax) * 4.0) / 4.0
        self.oy += np.round(self.rng.uniform(-self.vmax, self.vmax) * 4.0) / 4.0
        return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def generate(width: int, height: int, frames: int, seed: int, vmax: float = 6.0,
             n_rects: int = 4, cut_at: int | None = None) -> np.ndarray:
    """Return ``frames`` RGB24 frames as a (frames, height, width, 3) uint8 array."""
    out = np.empty((frames, height, width, 3), dtype=np.uint8)
    scene = Scene(width, height, seed, vmax, n_rects)
    for t in range(frames):
        if cut_at is not None and t == cut_at:
            scene = Scene(width, height, seed + 7919, vmax, n_rects)
        out[t] = scene.next_frame()
    return out
