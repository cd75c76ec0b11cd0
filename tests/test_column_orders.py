"""The evaluation orders of the coalesced column kernels, restated in Python
float64 and compared bit for bit with the orders they replace (CPU only).

* z-mean (ymkh_column.cu, zmean_p2_kernel): the reference's halving tree over
  a column (ymgpu2d/YM_Physics.cu:301-308: a[z] += a[z + NZ/2], ... 1) equals
  a pairwise binary counter over each residue class z mod 32, leaves in
  bit-reversed order, followed by a shuffle tree (strides 16 .. 1) over the
  32 class sums.
* hyperdiffusion (hyperdiff_seg_kernel): 32 z-segments updated in place from
  five-row windows, each segment's neighbour rows read before any write,
  equals the update from a copy of the column, whatever order the segments
  run in.
"""
from __future__ import annotations

import random
import struct

import pytest


def _bits(v: float) -> bytes:
    return struct.pack("<d", v)


def halving_tree(a: list) -> float:
    a = list(a)
    st = len(a) >> 1
    while st > 0:
        for i in range(st):
            a[i] = a[i] + a[i + st]
        st >>= 1
    return a[0]


def residue_counter_tree(a: list) -> float:
    nz = len(a)
    m = nz // 32
    logm = m.bit_length() - 1
    parts = []
    for lane in range(32):
        st = [0.0] * (logm + 1)
        for jj in range(m):
            j = 0
            for b in range(logm):
                j |= ((jj >> b) & 1) << (logm - 1 - b)
            carry, k = a[lane + 32 * j], 0
            for b in range(logm):
                if (jj >> b) & 1 == 0:
                    break
                carry = st[b] + carry
                k = b + 1
            st[k] = carry
        parts.append(st[logm])
    v = parts
    for d in (16, 8, 4, 2, 1):
        v = [v[i] + (v[i + d] if i + d < 32 else v[i]) for i in range(32)]
    return v[0]


@pytest.mark.parametrize("nz", [128, 256, 512, 1024, 4096])
def test_zmean_order_equals_halving_tree(nz):
    rng = random.Random(nz)
    for _ in range(8):
        a = [rng.gauss(0.0, 1.0) * 10.0 ** rng.randint(-8, 3) for _ in range(nz)]
        assert _bits(residue_counter_tree(a)) == _bits(halving_tree(a))


def hyperdiff_copy(col: list, mu: float) -> list:
    nz = len(col)
    out = []
    for z in range(nz):
        zm1 = nz - 1 if z == 0 else z - 1
        zm2 = z - 2 + nz if z <= 1 else z - 2
        zp1 = 0 if z == nz - 1 else z + 1
        zp2 = z + 2 - nz if z >= nz - 2 else z + 2
        d4 = col[zm2] - 4.0 * col[zm1] + 6.0 * col[z] - 4.0 * col[zp1] + col[zp2]
        out.append(col[z] - mu * d4)
    return out


def hyperdiff_segments(col: list, mu: float, order: list) -> list:
    nz = len(col)
    g = list(col)
    seg = nz // 32

    def at(z):
        return g[z + nz if z < 0 else (z - nz if z >= nz else z)]

    halo = [(at(w * seg - 2), at(w * seg - 1), at(w * seg + seg), at(w * seg + seg + 1)) for w in range(32)]
    for w in order:  # the barrier: every halo was read before any segment writes
        z0 = w * seg
        h0, h1, t0, t1 = halo[w]
        w0, w1, w2, w3 = h0, h1, at(z0), at(z0 + 1)
        for k in range(seg):
            w4 = at(z0 + k + 2) if k + 2 < seg else (t0 if k + 2 == seg else t1)
            d4 = w0 - 4.0 * w1 + 6.0 * w2 - 4.0 * w3 + w4
            g[z0 + k] = w2 - mu * d4
            w0, w1, w2, w3 = w1, w2, w3, w4
    return g


@pytest.mark.parametrize("nz", [64, 96, 128, 352, 1024])
def test_hyperdiff_segments_equal_copy_update(nz):
    rng = random.Random(7 * nz)
    for _ in range(4):
        col = [rng.gauss(0.0, 1.0) * 10.0 ** rng.randint(-6, 2) for _ in range(nz)]
        mu = 5e-5 * rng.random()
        order = list(range(32))
        rng.shuffle(order)
        want = hyperdiff_copy(col, mu)
        got = hyperdiff_segments(col, mu, order)
        assert [_bits(v) for v in got] == [_bits(v) for v in want]
