"""Seeded synthetic 4:2:0 sources standing in for the benchmark clips.

The reference's published numbers use real clips that are not available
here; these generators reproduce the shapes, motion and value
distributions the benchmark configurations describe:

* ``sinusoid_clip`` — 128 + a sum of 8 random 2-D sinusoids (periods
  8..64 px, amplitudes 10..40, random orientation and phase), translated
  every frame by a fixed global motion with separable bicubic (Keys,
  a = -0.5) resampling, plus Gaussian noise, clamped to [0, 255].  Chroma
  is generated the same way at half resolution from a second seed with
  half the motion.
* ``moving_rects_clip`` — the sinusoid background plus 16 axis-aligned
  rectangles (32..160 px sides) of uniform 0..255 noise texture, each with
  its own velocity drawn from [-6, 6]^2 px/frame.
* ``with_lines`` — static 1-px high-contrast lines over 5% of the area
  (screen-content-like detail that exercises the intra modes).

Everything is deterministic in the seeds.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

Frame = Tuple[np.ndarray, np.ndarray, np.ndarray]


def _texture(h: int, w: int, seed: int, origin: int = 0, n_waves: int = 8) -> np.ndarray:
    """Sinusoid field on an h x w canvas whose sample (origin, origin) is
    texture coordinate (0, 0), so the visible window does not depend on the
    canvas margin (and therefore not on the clip length)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64) - origin
    out = np.full((h, w), 128.0)
    for _ in range(n_waves):
        period = rng.uniform(8.0, 64.0)
        amp = rng.uniform(10.0, 40.0)
        theta = rng.uniform(0.0, np.pi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        out += amp * np.sin(2.0 * np.pi * (xx * np.cos(theta) + yy * np.sin(theta)) / period + phase)
    return out


def _keys(t: np.ndarray) -> np.ndarray:
    a = -0.5
    t = np.abs(t)
    return np.where(t <= 1, (a + 2) * t ** 3 - (a + 3) * t ** 2 + 1,
                    np.where(t < 2, a * t ** 3 - 5 * a * t ** 2 + 8 * a * t - 4 * a, 0.0))


def _shift_axis(img: np.ndarray, d: float, axis: int) -> np.ndarray:
    """Sample img at (index - d) along axis with bicubic weights, edges
    replicated."""
    n = img.shape[axis]
    base = np.floor(-d)
    frac = -d - base
    idx = np.arange(n)
    out = np.zeros_like(img)
    for k in range(-1, 3):
        w = float(_keys(np.array(frac - k)))
        src = np.clip(idx + int(base) + k, 0, n - 1)
        out += w * np.take(img, src, axis=axis)
    return out


def _shifted(base: np.ndarray, dx: float, dy: float, h: int, w: int, margin: int) -> np.ndarray:
    """Window of `base` (rendered with `margin` on each side) moved by
    (dx, dy) px, cropped to h x w."""
    img = _shift_axis(_shift_axis(base, dx, 1), dy, 0)
    return img[margin:margin + h, margin:margin + w]


def sinusoid_clip(width: int, height: int, frames: int, motion=(1.25, -0.5), noise_sigma: float = 2.0,
                  seed_luma: int = 1, seed_chroma: int = 2, seed_noise: int = 3) -> List[Frame]:
    return _render(width, height, frames, motion, noise_sigma, seed_luma, seed_chroma, seed_noise, None)


def moving_rects_clip(width: int, height: int, frames: int, motion=(2.5, 0.75), noise_sigma: float = 3.0,
                      seed_luma: int = 1, seed_chroma: int = 2, seed_noise: int = 3, seed_rects: int = 11,
                      n_rects: int = 16) -> List[Frame]:
    rng = np.random.default_rng(seed_rects)
    rects = []
    for _ in range(n_rects):
        rw, rh = int(rng.integers(32, 161)), int(rng.integers(32, 161))
        rw, rh = min(rw, width), min(rh, height)
        x0, y0 = rng.uniform(0, width - rw), rng.uniform(0, height - rh)
        vx, vy = rng.uniform(-6.0, 6.0), rng.uniform(-6.0, 6.0)
        tex_y = rng.integers(0, 256, size=(rh, rw)).astype(np.float64)
        tex_c = rng.integers(0, 256, size=(2, (rh + 1) // 2, (rw + 1) // 2)).astype(np.float64)
        rects.append((rw, rh, x0, y0, vx, vy, tex_y, tex_c))
    return _render(width, height, frames, motion, noise_sigma, seed_luma, seed_chroma, seed_noise, rects)


def _render(width, height, frames, motion, sigma, seed_l, seed_c, seed_n, rects) -> List[Frame]:
    vx, vy = motion
    span = int(np.ceil(max(abs(vx), abs(vy)) * frames)) + 4
    m = span
    base_y = _texture(height + 2 * m, width + 2 * m, seed_l, origin=m)
    mc = span // 2 + 4
    base_c = [_texture(height // 2 + 2 * mc, width // 2 + 2 * mc, seed_c * 1000 + k, origin=mc) for k in range(2)]
    noise = np.random.default_rng(seed_n)
    out: List[Frame] = []
    for t in range(frames):
        y = _shifted(base_y, vx * t, vy * t, height, width, m)
        cb = _shifted(base_c[0], vx * t / 2, vy * t / 2, height // 2, width // 2, mc)
        cr = _shifted(base_c[1], vx * t / 2, vy * t / 2, height // 2, width // 2, mc)
        if rects:
            for rw, rh, x0, y0, rvx, rvy, tex_y, tex_c in rects:
                px = int(round(x0 + rvx * t)) % max(1, width - rw + 1)
                py = int(round(y0 + rvy * t)) % max(1, height - rh + 1)
                y[py:py + rh, px:px + rw] = tex_y
                cx, cy = px // 2, py // 2
                ch, cw = tex_c.shape[1], tex_c.shape[2]
                ch, cw = min(ch, height // 2 - cy), min(cw, width // 2 - cx)
                cb[cy:cy + ch, cx:cx + cw] = tex_c[0, :ch, :cw]
                cr[cy:cy + ch, cx:cx + cw] = tex_c[1, :ch, :cw]
        y = y + noise.normal(0.0, sigma, size=y.shape)
        cb = cb + noise.normal(0.0, sigma, size=cb.shape)
        cr = cr + noise.normal(0.0, sigma, size=cr.shape)
        out.append(tuple(np.clip(np.rint(p), 0, 255).astype(np.uint8) for p in (y, cb, cr)))
    return out


def with_lines(frames: List[Frame], area_frac: float = 0.05, seed: int = 21) -> List[Frame]:
    """Overlay static 1-px high-contrast horizontal / vertical lines covering
    `area_frac` of the luma area (screen-content-like detail)."""
    h, w = frames[0][0].shape
    rng = np.random.default_rng(seed)
    mask = np.zeros((h, w), bool)
    val = np.zeros((h, w), np.uint8)
    target = int(area_frac * h * w)
    while mask.sum() < target:
        length = int(rng.integers(16, max(17, min(w, h) // 2)))
        v = 255 if rng.integers(0, 2) else 0
        if rng.integers(0, 2):
            y, x = int(rng.integers(0, h)), int(rng.integers(0, w - length))
            mask[y, x:x + length] = True
            val[y, x:x + length] = v
        else:
            y, x = int(rng.integers(0, h - length)), int(rng.integers(0, w))
            mask[y:y + length, x] = True
            val[y:y + length, x] = v
    out = []
    for (y, cb, cr) in frames:
        y2 = y.copy()
        y2[mask] = val[mask]
        out.append((y2, cb, cr))
    return out


def workload(name: str, frames: int = None, width: int = None, height: int = None) -> List[Frame]:
    """Named workloads: 'sinusoid' (320x240 sinusoid, motion (+1.25, -0.5),
    sigma 2), 'rects' (1280x720 sinusoid + rectangles, motion (+2.5, +0.75),
    sigma 3) and 'rects_lines' (1920x1080 rectangles + 1-px lines)."""
    if name == "sinusoid":
        return sinusoid_clip(width or 320, height or 240, frames or 30)
    if name == "rects":
        return moving_rects_clip(width or 1280, height or 720, frames or 60)
    if name == "rects_lines":
        return with_lines(moving_rects_clip(width or 1920, height or 1080, frames or 120, motion=(2.5, 0.75),
                                            noise_sigma=3.0))
    raise ValueError(name)


# ---------------------------------------------------------------------------
# Mixed-resolution stream sets (the batched and served workloads)
# ---------------------------------------------------------------------------
MIX_RESOLUTIONS = ((320, 240), (640, 360), (1280, 720), (1920, 1080))
MIX_QPS = (22, 27, 32, 37)


def mixed_streams(n: int = 64, frames: int = 32, seed: int = 7, stream_seed0: int = 1000):
    """Specs of `n` independent streams: resolution and QP drawn uniformly
    from MIX_RESOLUTIONS / MIX_QPS with `seed`; stream i renders the
    moving-rectangles generator from its own seed stream_seed0 + i.
    Returns a list of dicts {w, h, qp, seed, frames}."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        w, h = MIX_RESOLUTIONS[int(rng.integers(0, len(MIX_RESOLUTIONS)))]
        qp = MIX_QPS[int(rng.integers(0, len(MIX_QPS)))]
        out.append(dict(w=w, h=h, qp=qp, seed=stream_seed0 + i, frames=frames))
    return out


def stream_clip(spec, frames: int = None) -> List[Frame]:
    """Frames of one mixed-workload stream (moving rectangles over the
    sinusoid background, motion (+2.5, +0.75), sigma 3), all four seeds
    derived from the stream's own seed."""
    s = int(spec["seed"])
    return moving_rects_clip(spec["w"], spec["h"], frames or spec["frames"], seed_luma=4 * s,
                             seed_chroma=4 * s + 1, seed_noise=4 * s + 2, seed_rects=4 * s + 3)


def served_sessions(n: int = 2000, rate_per_s: float = 200.0, seed: int = 9, session_seed0: int = 5000):
    """Encode sessions arriving as a Poisson process of `rate_per_s`:
    exponential inter-arrival gaps, 8..64 frames (uniform), resolution and
    QP uniform over MIX_RESOLUTIONS / MIX_QPS, all from `seed`; session j
    renders from its own seed session_seed0 + j.  Returns a list of dicts
    {arrival_s, w, h, qp, seed, frames}."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for j in range(n):
        t += float(rng.exponential(1.0 / rate_per_s))
        w, h = MIX_RESOLUTIONS[int(rng.integers(0, len(MIX_RESOLUTIONS)))]
        qp = MIX_QPS[int(rng.integers(0, len(MIX_QPS)))]
        nf = int(rng.integers(8, 65))
        out.append(dict(arrival_s=t, w=w, h=h, qp=qp, seed=session_seed0 + j, frames=nf))
    return out
