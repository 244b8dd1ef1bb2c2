"""Algorithmic work model of the photoelectric kernel (for the benchmark's roofline).

Counts are operations of the restated reference formulas (csrc/geom.cuh chords,
csrc/pe.cu sub-element body), counted by hand from the source: +, -, *, / and sqrt count
as one FP32 operation each, a fused multiply-add as two; divisions, square roots,
exponentials and reciprocals also count one MUFU (special-function unit) operation each.
Culling work (cone tests, slope rectangles, sub-lists) is not counted: the model is the
reference's arithmetic on the chords that are non-zero, a lower bound for any
implementation.

  box chord (general case): 3 differences, |d| (5 + sqrt), 3 reciprocal steps (div),
                            3 slabs x 4, 1 difference                = 25 flops, 4 MUFU
  cylinder chord:           47 flops + 9 div + 2 sqrt               = 58 flops, 11 MUFU
  per sub-element (fixed):  position 12, rotation 9, distance 8 + sqrt, cos 2, solid angle
                            24 (with one reciprocal), layer term 4, sub-element box 18,
                            self term 3, exp 3, extended ray 12, absorption 5, product 3,
                            sum 1                                     = 104 flops, 9 MUFU
  per sub-element boxes:    (L plate boxes + 2 inside-crystal chords + 1 absorption chord)
  per non-zero hole chord:  cylinder + 3                              = 61 flops, 11 MUFU
  per non-zero crystal chord: 2 frame changes 18 + box 25 + 2         = 45 flops, 4 MUFU

W(element) = sum over its 1024 sub-elements of the fixed terms and the boxes, plus the
per-hit terms for the non-zero chords counted by the kernel (sysmat_pe_work).
"""
from __future__ import annotations

BOX_FLOPS, BOX_MUFU = 25, 4
CYL_HIT_FLOPS, CYL_HIT_MUFU = 61, 11
CRY_HIT_FLOPS, CRY_HIT_MUFU = 45, 4
SUB_FLOPS, SUB_MUFU = 104, 9

# DRAM traffic of one pe_kernel launch, from one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum, --clock-control none) of the reference-mode kernel on crystals
# 0..255 x z-plane 16 of configuration 2 (2359296 elements, 548.6 ms): 3779840 B read +
# 226816 B written.  The block's output (9.4 MB) stays in L2 during the launch, so the figure
# is the tables' and output lines' first touches, not the output's write-back.
PE_DRAM_CAPTURE = {
    "bytes": 3779840 + 226816,
    "elements": 2359296,
    "command": "ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum "
               "--clock-control none -k regex:pe_kernel -s 3 -c 1 python bench.py --steps 1 --warmup 3 "
               "--det-count 256 --no-e2e --no-scatter --no-scatter2 --no-grid --no-batch --no-sampled --no-fp64 "
               "--no-local --no-cpu-baseline",
}


def pe_work(counts: dict, n_layers: int) -> tuple[float, float]:
    """(FP32 operations, MUFU operations) for a launch with the given work counters."""
    n_sub = counts["subelements"]
    boxes = n_layers + 3
    flops = n_sub * (SUB_FLOPS + BOX_FLOPS * boxes)
    flops += CYL_HIT_FLOPS * counts["hole_hits"] + CRY_HIT_FLOPS * counts["crystal_hits"]
    mufu = n_sub * (SUB_MUFU + BOX_MUFU * boxes)
    mufu += CYL_HIT_MUFU * counts["hole_hits"] + CRY_HIT_MUFU * counts["crystal_hits"]
    return float(flops), float(mufu)


def pe_traffic_per_launch(elements: int):
    """DRAM bytes of a pe_kernel launch over `elements` output elements: the captured launch's
    bytes scaled by its element count (the kernel's DRAM traffic is its output plus the
    L2-resident tables, so it grows with the elements), with the capture it came from; None
    without a capture."""
    cap = PE_DRAM_CAPTURE
    if not cap:
        return None
    return {"bytes": cap["bytes"] * elements / cap["elements"],
            "source": f"ncu capture ({cap['command']}): {cap['bytes']:.4g} DRAM bytes over "
                      f"{cap['elements']} elements, scaled to {elements} elements"}
