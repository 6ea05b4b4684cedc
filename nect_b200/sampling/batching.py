"""Cutting one projection's shuffled detector pixels into ray batches.

The reference's projector defines which pixels a batch holds
(nect/sampling/projector.py:87-112); the fused trainer and the Projector
both take their batches from here, so the two cannot drift apart:

* a batch holds ``points_per_batch // points_per_ray`` rays;
* a projection has ``ceil(pixels / batch)`` batches;
* batch k starts at pixel k * batch of the permutation; a projection smaller
  than one batch yields all of its pixels as batch 0, and a partial batch at
  the end of a larger projection yields nothing (the reference skips it).
"""
from __future__ import annotations


def rays_per_batch(points_per_batch: int, points_per_ray: int) -> int:
    return points_per_batch // points_per_ray


def batches_per_projection(pixels: int, batch_rays: int) -> int:
    return -(-pixels // batch_rays)


def batch_window(pixels: int, batch_rays: int, batch_num: int) -> tuple[int, int] | None:
    """(first permutation index, ray count) of batch ``batch_num``, or None."""
    start = batch_num * batch_rays
    if start + batch_rays <= pixels:
        return start, batch_rays
    if batch_num == 0:
        return 0, pixels
    return None
