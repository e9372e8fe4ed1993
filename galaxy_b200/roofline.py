"""Algorithmic bytes and FLOPs of one step, per stage: the compulsory reads and writes of
each stage's inputs and outputs, once, with this implementation's record sizes. A
stage's roofline fraction is (these bytes / its measured time) / the measured HBM rate;
the walk's is its algorithmic FP32 flops over the FP32 rate (it is issue-bound, see
``issue_fraction``).

N particles, N - 1 internal nodes per system; P radix passes (4 with 30-bit keys and
8-bit digits, 3 with 10-bit digits, 8 with 63-bit keys); K key bytes (4 or 8).
"""

from __future__ import annotations

# Bytes per particle of each stage.
KICK_DRIFT_BBOX = 120  # pos, vel, acc read (72) + pos, vel written (48)
MORTON = 24            # pos read; + K for the code written (see stage_bytes)
BUILD = 256            # codes + order (8) and the gathered pos/mass (32) read; leaf64 (32),
#                        kids (8), parent links (8), agg64 (80), pair record (80) and the
#                        exchange word (8) written (siblings' aggregates are read from
#                        shared memory below each 256-leaf block, from L2 above it)
BUILD_INSIDE = 32      # theta >= 1/sqrt(3): box centre and half extents (FP32) per internal node
BUILD_QUAD = 80        # quadrupole: q64 (48) + FP32 copy (32) per internal node
WALK = 140             # pair record per internal node (80), target leaf (32) and order (4)
#                        read, acceleration (24) written; each record read once


def sort_passes(key64: bool = False, radix_bits: int = 8) -> int:
    """Radix passes of the sort: ceil(key bits / digit bits)."""
    return -(-(63 if key64 else 30) // (8 if key64 else radix_bits))


def stage_bytes(n: int, key64: bool = False, quad: bool = False, radix_bits: int = 8, inside: bool = False) -> dict:
    """Algorithmic bytes of each stage of one step for n particles (inside: theta >= 1/sqrt 3)."""
    kb = 8 if key64 else 4
    passes = sort_passes(key64, radix_bits)
    return {
        "kick_drift_bbox": KICK_DRIFT_BBOX * n,
        "morton": (MORTON + kb) * n,
        "sort_pass": 2 * (kb + 4) * n,  # (key, index) read and written once
        "sort": passes * 2 * (kb + 4) * n,
        "build": (BUILD + (BUILD_QUAD if quad else 0) + (BUILD_INSIDE if inside else 0)) * n,
        "walk": WALK * n,
    }


def walk_flops(leaf_terms: int, far_terms: int, opened: int, quad: bool = False) -> int:
    """FP32 flops of the walk from its interaction counts: 20 per leaf term (distance 3,
    r^2 + eps^2 6, inverse cube 2, mass 1, accumulate 6, compensation 2), 24 per far term
    (plus 30 for a quadrupole), 18 per opened node (the opening test)."""
    return 20 * leaf_terms + (24 + (30 if quad else 0)) * far_terms + 18 * opened


def hbm_fraction(nbytes: float, ms: float, peak_gbs: float) -> tuple[float, float]:
    """(achieved GB/s, fraction of peak) of nbytes moved in ms milliseconds."""
    gbs = nbytes / (ms * 1e-3) / 1e9
    return gbs, gbs / peak_gbs


def issue_fraction(warp_instructions: int, ms: float, sm_count: int = 148, sm_mhz: float = 1965.0) -> tuple[float, float]:
    """(achieved G warp instructions/s, fraction of the peak of one warp instruction per
    scheduler per clock, four schedulers per SM)."""
    rate = warp_instructions / (ms * 1e-3) / 1e9
    peak = sm_count * 4 * sm_mhz / 1e3
    return rate, rate / peak
