"""Writers of small TRR, XTC, DCD, GRO and PDB files for the reader tests.

They follow the published layouts (GROMACS TRR: XDR big-endian frames with a
"GMX_trn_file" header and block sizes; GROMACS XTC: XDR frames with the
compressed coordinates of xdr3dfcoord; CHARMM/NAMD DCD: Fortran unformatted
records; GRO and PDB fixed columns) and are test infrastructure only.  The XTC
compressor is this project's own: any stream that follows the format decodes
the same way, and this one makes its choices (which atoms form runs, when the
small-delta range grows or shrinks) so that every branch of the format occurs.
"""
from __future__ import annotations

import struct

import numpy as np


def write_trr(path, frames_nm, boxes_nm, times, double=False, with_v=False, with_f=False):
    real = "d" if double else "f"
    rs = 8 if double else 4
    with open(path, "wb") as fh:
        for k, (x, box, t) in enumerate(zip(frames_nm, boxes_nm, times)):
            n = x.shape[0]
            sizes = [0, 0, 9 * rs, 0, 0, 0, 0, 3 * n * rs, 3 * n * rs if with_v else 0,
                     3 * n * rs if with_f else 0]
            fh.write(struct.pack(">ii", 1993, 13))
            fh.write(struct.pack(">i", 12) + b"GMX_trn_file")
            fh.write(struct.pack(">10i", *sizes))
            fh.write(struct.pack(">iii", n, 100 * k, 0))
            fh.write(struct.pack(">" + real * 2, t, 0.0))
            fh.write(struct.pack(">" + real * 9, *np.asarray(box, np.float64).ravel()))
            fh.write(struct.pack(">" + real * (3 * n), *np.asarray(x, np.float64).ravel()))
            if with_v:
                fh.write(struct.pack(">" + real * (3 * n), *np.full(3 * n, 0.25)))
            if with_f:
                fh.write(struct.pack(">" + real * (3 * n), *np.full(3 * n, -7.0)))


def write_dcd(path, frames_a, cells=None, cosines=False, big_endian=False, dt=0.5, nset=None):
    e = ">" if big_endian else "<"
    n = frames_a.shape[1]
    F = frames_a.shape[0]

    def rec(payload: bytes) -> bytes:
        return struct.pack(e + "i", len(payload)) + payload + struct.pack(e + "i", len(payload))

    icntrl = [0] * 20
    icntrl[0] = F if nset is None else nset
    icntrl[2] = 1
    icntrl[19] = 24  # CHARMM version
    icntrl[10] = 1 if cells is not None else 0
    ints = [struct.pack(e + "i", v) for v in icntrl]
    ints[9] = struct.pack(e + "f", dt)
    head = b"CORD" + b"".join(ints)
    title = struct.pack(e + "i", 1) + b"test dcd".ljust(80)
    with open(path, "wb") as fh:
        fh.write(rec(head))
        fh.write(rec(title))
        fh.write(rec(struct.pack(e + "i", n)))
        for k in range(F):
            if cells is not None:
                a, b, c, al, be, ga = cells[k]
                if cosines:
                    al, be, ga = (float(np.cos(np.radians(v))) for v in (al, be, ga))
                fh.write(rec(struct.pack(e + "6d", a, ga, b, be, al, c)))
            for d in range(3):
                fh.write(rec(struct.pack(e + "%df" % n, *frames_a[k, :, d])))


def write_gro(path, names, resnames, frames_nm, boxes_nm, times=None):
    with open(path, "w") as fh:
        for k, x in enumerate(frames_nm):
            t = 0.0 if times is None else times[k]
            fh.write(f"test system t= {t:.5f}\n{len(names)}\n")
            for i, (a, r) in enumerate(zip(names, resnames)):
                fh.write("%5d%-5s%5s%5d%8.3f%8.3f%8.3f\n" % (i // 3 + 1, r, a, (i + 1) % 100000,
                                                             x[i, 0], x[i, 1], x[i, 2]))
            b = np.asarray(boxes_nm[k], np.float64)
            vals = [b[0, 0], b[1, 1], b[2, 2], b[0, 1], b[0, 2], b[1, 0], b[1, 2], b[2, 0], b[2, 1]]
            fh.write(" ".join("%10.5f" % v for v in vals) + "\n")


def write_pdb(path, names, resnames, elements, pos_a, cell=None):
    with open(path, "w") as fh:
        if cell is not None:
            fh.write("CRYST1%9.3f%9.3f%9.3f%7.2f%7.2f%7.2f P 1           1\n" % tuple(cell))
        for i, (a, r, el) in enumerate(zip(names, resnames, elements)):
            fh.write("ATOM  %5d %-4s %3s A%4d    %8.3f%8.3f%8.3f  1.00  0.00          %2s\n"
                     % (i + 1, a, r, i // 3 + 1, pos_a[i, 0], pos_a[i, 1], pos_a[i, 2], el))
        fh.write("END\n")


# small-delta ranges of the XTC format, ~2^(i/3) (the table every writer and
# reader of the format shares)
XTC_MAGIC = [0, 0, 0, 0, 0, 0, 0, 0, 0, 8, 10, 12, 16, 20, 25, 32, 40, 50, 64, 80, 101, 128, 161, 203,
             256, 322, 406, 512, 645, 812, 1024, 1290, 1625, 2048, 2580, 3250, 4096, 5060, 6501, 8192,
             10321, 13003, 16384, 20642, 26007, 32768, 41285, 52015, 65536, 82570, 104031, 131072,
             165140, 208063, 262144, 330280, 416127, 524287, 660561, 832255, 1048576, 1321122, 1664510,
             2097152, 2642245, 3329021, 4194304, 5284491, 6658042, 8388607, 10568983, 13316085, 16777216]
XTC_FIRST, XTC_LAST = 9, len(XTC_MAGIC) - 1


class _Bits:
    """Most-significant-bit-first bit writer."""

    def __init__(self):
        self.bits = []

    def put(self, value: int, n: int):
        for k in range(n - 1, -1, -1):
            self.bits.append((value >> k) & 1)

    def triple(self, digits, radices, nbits: int):
        """A mixed-radix number of nbits: bytes from the least significant up,
        the last one holding the remaining 1..8 bits."""
        n = (digits[0] * radices[1] + digits[1]) * radices[2] + digits[2]
        assert n < (1 << nbits)
        while nbits > 8:
            self.put(n & 0xFF, 8)
            n >>= 8
            nbits -= 8
        self.put(n, nbits)

    def payload(self) -> bytes:
        b = self.bits + [0] * (-len(self.bits) % 8)
        return bytes(int("".join(map(str, b[i:i + 8])), 2) for i in range(0, len(b), 8))


def xtc_ints(frame_nm, precision):
    """Integer coordinates round(x * precision), halves away from zero (float32 steps)."""
    v = np.asarray(frame_nm, np.float32) * np.float32(precision)
    return np.trunc(v + np.copysign(np.float32(0.5), v)).astype(np.int64)


def _compress(ints, smallidx, large, rng):
    n = ints.shape[0]
    lo = ints.min(axis=0)
    hi = ints.max(axis=0)
    if large:
        hi = np.maximum(hi, lo + (1 << 24) + 17)   # a range beyond 2^24 - 1: one number per axis
    size = (hi - lo + 1).astype(int)
    bits = _Bits()
    if large:
        b1 = [int(s).bit_length() for s in size]
    else:
        b3 = int(size[0] * size[1] * size[2]).bit_length()
    idx0 = smallidx
    prevrun, i = -1, 0
    while i < n:
        m = XTC_MAGIC[smallidx]
        half = m // 2
        smalls = []
        if i + 1 < n and np.all(np.abs(ints[i] - ints[i + 1]) < half):
            big = ints[i + 1]
            smalls.append(ints[i] - ints[i + 1] + half)    # written first in the frame
            prev, j = ints[i], i + 2
            while j < n and len(smalls) < 8 and np.all(np.abs(ints[j] - prev) < half):
                smalls.append(ints[j] - prev + half)
                prev, j = ints[j], j + 1
            used = j - i
        else:
            big, used = ints[i], 1
        run = 3 * len(smalls)
        # the next group's range: wider after a lone atom, narrower after a run
        # whose deltas fit the next smaller range, sometimes at random
        change = 0
        if run == 0 and smallidx < XTC_LAST and rng.random() < 0.7:
            change = 1
        elif run > 0 and smallidx > XTC_FIRST and rng.random() < 0.5:
            change = -1
        d = big - lo
        if large:
            for k in range(3):
                bits.put(int(d[k]), b1[k])
        else:
            bits.triple([int(v) for v in d], [int(v) for v in size], b3)
        if run != prevrun or change != 0:
            bits.put(1, 1)
            bits.put(run + change + 1, 5)
            prevrun = run
        else:
            bits.put(0, 1)
        for sm in smalls:
            bits.triple([int(v) for v in sm], [m, m, m], smallidx)
        smallidx += change
        i += used
    data = bits.payload()
    head = struct.pack(">3i", *[int(v) for v in lo]) + struct.pack(">3i", *[int(v) for v in hi])
    return head + struct.pack(">ii", idx0, len(data)) + data + b"\0" * (-len(data) % 4)


def write_xtc(path, frames_nm, boxes_nm, times, precision=1000.0, large=False, smallidx=20, seed=0):
    """Frames (natoms, 3) nm as XTC; returns the integer coordinates written per frame."""
    rng = np.random.default_rng(seed)
    written = []
    with open(path, "wb") as fh:
        for k, (x, box, t) in enumerate(zip(frames_nm, boxes_nm, times)):
            n = x.shape[0]
            fh.write(struct.pack(">iiif", 1995, n, 10 * k, t))
            fh.write(struct.pack(">9f", *np.asarray(box, np.float32).ravel()))
            fh.write(struct.pack(">i", n))
            if n <= 9:
                fh.write(struct.pack(">%df" % (3 * n), *np.asarray(x, np.float32).ravel()))
                written.append(None)
                continue
            ints = xtc_ints(x, precision)
            fh.write(struct.pack(">f", precision))
            fh.write(_compress(ints, smallidx, large, rng))
            written.append(ints)
    return written
