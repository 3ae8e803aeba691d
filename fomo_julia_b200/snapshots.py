"""Headless wavefield snapshots for on_step (the reference's video recorder
without the video).

``src/visualization/video_recorder.jl`` records p, vel, vx or vz frames every
``skip`` steps with ``downsample``-fold subsampling and renders them to mp4
through CairoMakie.  Here the frames are extracted on the device
(``fomo_b200_wavefield_snapshot``) and kept in host memory; rendering is left
to the caller.

    rec = SnapshotRecorder(VideoConfig(fields=["p", "vel"], skip=5, downsample=2))
    run_shot(b, W, M, H, a, src, rec_, params, on_step=rec, step_chunk=rec.config.skip)
    frames = rec.frames["p"]            # list of (k, t, frame)
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


@dataclass
class VideoConfig:
    """VideoConfig (video_recorder.jl:68-82) without the rendering options'
    effect: fields, skip and downsample select the frames."""
    fields: Sequence[str] = ("p",)
    output_dir: str = "."
    prefix: str = "wavefield"
    time_scale: float = 0.01
    skip: int = 1
    downsample: int = 1
    clim: Optional[Tuple[float, float]] = None
    colormap: str = "balance"


class SnapshotRecorder:
    """MultiFieldRecorder (video_recorder.jl:113-141) as an on_step callback
    that keeps the frames: frames[field] is a list of (k, t, frame)."""

    def __init__(self, config: VideoConfig = VideoConfig(), max_frames: Optional[int] = None):
        for f in config.fields:
            if f not in ("p", "vel", "vx", "vz"):
                raise ValueError(f"Unknown field: {f}. Use p, vel, vx, or vz")
        if config.skip < 1 or config.downsample < 1:
            raise ValueError("skip and downsample must be >= 1")
        self.config = config
        self.max_frames = max_frames
        self.frames: Dict[str, List[tuple]] = {f: [] for f in config.fields}

    def __call__(self, W, info) -> bool:
        if info.k % self.config.skip != 0:
            return True
        for f in self.config.fields:
            if self.max_frames is None or len(self.frames[f]) < self.max_frames:
                self.frames[f].append((int(info.k), info.t, W.snapshot(f, self.config.downsample)))
        return True

    def stack(self, field_name: str) -> np.ndarray:
        """Frames of one field as an array (n_frames, nx_d, nz_d)."""
        return np.stack([fr for _, _, fr in self.frames[field_name]])
