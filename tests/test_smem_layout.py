"""Bank layout of the stage kernel's shared-memory buffers (csrc/wenofv_stage.cuh), on CPU.

An 8-byte shared-memory access of a warp is served per half-warp: 16 lanes, 16 banks of 8
bytes.  The strides of the y-sweep rows (sy), the face states (sxf, syb, syt) and the warps'
exchange areas are chosen so that every writer and reader pattern of the 4-variable kernels
maps a half-warp to 16 distinct banks.  The strides are read from the header, the patterns
are the lane mappings of the phases: lane = 4 * (position or cell) + variable in the sweeps,
lane = 4 * face + Gauss point in the Riemann phase.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STAGE = os.path.join(ROOT, "two-phase-3equation-2d-pal-column_b200", "csrc", "wenofv_stage.cuh")


def _header():
    return open(STAGE).read()


def _stride(name):
    m = re.search(r"static constexpr int %s = NV == 4 \? (\d+) :" % name, _header())
    assert m, name
    return int(m.group(1))


def _sy_stride():
    m = re.search(r"if constexpr \(NV == 4 && RECON < 2\) return p \* (\d+) \+ g \* 4 \+ v;", _header())
    assert m
    return int(m.group(1))


def face_slot(v, f):
    return (v + f) & 3


def _distinct_banks(addresses):
    """addresses (in doubles) of one half-warp hit 16 distinct 8-byte banks"""
    return len({a % 16 for a in addresses}) == len(addresses) == 16


def test_layout_is_the_header_s():
    assert "if constexpr (NV == 4) return (v + f) & 3;" in _header()
    assert (_stride("FS"), _stride("BS"), _stride("YS"), _sy_stride()) == (36, 20, 20, 20)


@pytest.mark.parametrize("base", [0, 4, 8])  # half-warps start at cells 0, 4, 8, ... (any multiple of 4)
def test_face_states_writers_and_riemann_readers(base):
    FS, BS = _stride("FS"), _stride("BS")
    for stride, nk in ((FS, 8), (BS, 4)):
        for k in range(nk):  # x-face records: side * 4 + Gauss point; y-face records: Gauss point
            # x-sweep writers: lanes (cell c, variable v), one point k
            writers = [(base + c) * stride + k * 4 + face_slot(v, base + c) for c in range(4) for v in range(4)]
            assert _distinct_banks(writers)
        for v in range(4):
            # Riemann readers: lanes (face f, Gauss point gp), one variable v, both sides
            for side in (0, 4):
                readers = [(base + f) * stride + (side + gp) * 4 + face_slot(v, base + f) for f in range(4) for gp in range(4)]
                if stride == BS and side:
                    continue
                assert _distinct_banks(readers)


@pytest.mark.parametrize("base", [0, 4, 60])
def test_y_sweep_rows(base):
    YS = _sy_stride()
    for g in range(4):
        # y-sweep writers: lanes (position p, variable v); conservative x-sweep readers: lanes
        # (cell c, variable v) at one stencil offset: the same pattern
        assert _distinct_banks([(base + p) * YS + g * 4 + v for p in range(4) for v in range(4)])


def test_exchange_areas():
    # x-sweep exchange in sxf: 20 doubles per cell; writers (cell, variable) at one point, readers
    # load the point's 4 values (16 bytes at a time, the 4 lanes of a cell reading the same bytes)
    for gpi in range(4):
        assert _distinct_banks([cl * 20 + gpi * 4 + v for cl in range(4) for v in range(4)])
    # primitive x-sweep: lane gj writes variable k at slot k*4 + ((gj + k) & 3); lane v reads
    # point gpj at slot v*4 + ((gpj + v) & 3)
    for k in range(4):
        assert _distinct_banks([cl * 20 + k * 4 + ((gj + k) & 3) for cl in range(4) for gj in range(4)])
    for gpj in range(4):
        assert _distinct_banks([cl * 20 + v * 4 + ((gpj + v) & 3) for cl in range(4) for v in range(4)])
    # the primitive exchange hands lane v the value lane gj = gpj wrote for variable k = v
    for gpj in range(4):
        for v in range(4):
            assert v * 4 + ((gpj + v) & 3) == (lambda gj, k: k * 4 + ((gj + k) & 3))(gpj, v)
