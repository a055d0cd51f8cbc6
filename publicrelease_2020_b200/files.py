"""The reference's SIC files, written from the library's results, for hosts
whose post-processing reads them (siclag_der.F reads ZPOT####, fod_opt reads
fforce.dat, users read SICD.DAT and SIC_ENERGY).  The library itself keeps
the potentials and Hamiltonian ingredients in GPU memory.

  ZPOT####     apotnl_sic.F:497-522: Fortran unformatted sequential, one
               record per mesh point holding POT(IMSH); #### = IRBSIC =
               IORBX + (LSPN-1)*NWFS(1)
  MGGA####     getvlxc.F:203-227: one record per point of MIXIN(1:4, IPTS),
               IPTS = 1 .. NMSH*NSPN (NSPN = 2 in the SIC call)
  SICD.DAT     main.F:718-727: per spin and FO the row SIC(1:NFRM, IWF),
               FORMAT(' ',15F12.5)
  SIC_ENERGY   main.F:746-759: a header line, then per FO
               RESULTS((1,2,4,6,9,10,11,12,13)), FORMAT(F4.0,20F11.6)
  fforce.dat   main.F:700-713, 731-737: per spin and FO DEBDAX(1:3),
               FORMAT(' ',3F20.12)

Unformatted records use gfortran's layout: a 4-byte little-endian record
length before and after each record."""
from __future__ import annotations

import os
import struct

import numpy as np

IRES = (1, 2, 4, 6, 9, 10, 11, 12, 13)
SIC_ENERGY_HEADER = (" FLO    Charge     Asymp      E_COUL     E_SIC      EXlocal    EClocal    "
                     "EXnonl     ECnonl")


def fortran_f(x, w, d):
    """Fortran Fw.d edit of one value as gfortran writes it: right-justified,
    a decimal point even for d = 0, the leading zero of |x| < 1 dropped when
    the field is too narrow for it, asterisks when the value does not fit."""
    s = f"{x:.{d}f}" + ("." if d == 0 else "")
    if len(s) > w and (s.startswith("0.") or s.startswith("-0.")):
        s = s.replace("0.", ".", 1)
    return s.rjust(w) if len(s) <= w else "*" * w


def format_line(values, w, d, per_line, lead=" "):
    """Lines of FORMAT(lead, per_line Fw.d) with format reversion."""
    vals = list(values)
    out = []
    for i in range(0, max(len(vals), 1), per_line):
        out.append(lead + "".join(fortran_f(v, w, d) for v in vals[i:i + per_line]))
    return out


def write_unformatted(path, records):
    """Fortran unformatted sequential file of float64 records."""
    with open(path, "wb") as f:
        for rec in records:
            b = np.ascontiguousarray(rec, dtype="<f8").tobytes()
            f.write(struct.pack("<i", len(b)))
            f.write(b)
            f.write(struct.pack("<i", len(b)))


def read_unformatted(path):
    """The float64 records of a Fortran unformatted sequential file."""
    out = []
    with open(path, "rb") as f:
        while True:
            h = f.read(4)
            if not h:
                break
            n = struct.unpack("<i", h)[0]
            out.append(np.frombuffer(f.read(n), dtype="<f8").copy())
            assert struct.unpack("<i", f.read(4))[0] == n
    return out


def write_zpot(dirpath, irbsic, pot):
    path = os.path.join(dirpath, f"ZPOT{irbsic:04d}")
    with open(path, "wb") as f:   # one 8-byte record per point, written in one pass
        rec = np.empty(len(pot), dtype=[("a", "<i4"), ("v", "<f8"), ("b", "<i4")])
        rec["a"] = 8
        rec["v"] = pot
        rec["b"] = 8
        f.write(rec.tobytes())
    return path


def write_mgga(dirpath, kxxo, mixin):
    path = os.path.join(dirpath, f"MGGA{kxxo:04d}")
    m = np.asarray(mixin, dtype=np.float64).reshape(-1, 4)
    with open(path, "wb") as f:
        rec = np.empty(len(m), dtype=[("a", "<i4"), ("v", "<f8", (4,)), ("b", "<i4")])
        rec["a"] = 32
        rec["v"] = m
        rec["b"] = 32
        f.write(rec.tobytes())
    return path


def write_sicd(path, sic, nfrm):
    """sic[s][l][j] = SIC(j, l, s) (the library's layout)."""
    lines = []
    for s, n in enumerate(nfrm):
        for iwf in range(n):
            lines += format_line([sic[s][iwf][jwf] for jwf in range(n)], 12, 5, 15)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_sic_energy(path, results, nfrm):
    lines = [SIC_ENERGY_HEADER]
    for s, n in enumerate(nfrm):
        for k in range(n):
            r = results[s][k]
            lines.append(fortran_f(r[0], 4, 0) + "".join(fortran_f(r[i - 1], 11, 6) for i in IRES[1:]))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_fforce(path, debdax, nfrm):
    lines = []
    for s, n in enumerate(nfrm):
        for k in range(n):
            lines += format_line(debdax[s][k][:3], 20, 12, 3)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_cycle_files(dirpath, ctx, out, potentials=True):
    """All files of one SIC block from a context and its cycle output."""
    sysm = ctx.sysm
    nfrm = [ctx.nfrm[s] for s in range(sysm.nspn)]
    write_sicd(os.path.join(dirpath, "SICD.DAT"), out["sic"], nfrm)
    write_sic_energy(os.path.join(dirpath, "SIC_ENERGY"), out["results"], nfrm)
    write_fforce(os.path.join(dirpath, "fforce.dat"), out["debdax"], nfrm)
    if potentials:
        mgga = sysm.xc[0] >= 3
        for s, n in enumerate(nfrm):
            for k in range(1, n + 1):
                irbsic = k + s * sysm.nwfs[0]
                write_zpot(dirpath, irbsic, ctx.apotnl_sic(s + 1, k)["pot"])
                if mgga:
                    write_mgga(dirpath, irbsic, ctx.mgga_mixin(s + 1, k))
