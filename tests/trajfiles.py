"""Writers of small TRR, DCD, GRO and PDB files for the reader tests.

They follow the published layouts (GROMACS TRR: XDR big-endian frames with a
"GMX_trn_file" header and block sizes; CHARMM/NAMD DCD: Fortran unformatted
records; GRO and PDB fixed columns) and are test infrastructure only.
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
