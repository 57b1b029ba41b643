"""Statistics files in the reference's formats (single rank, the files rank 0 writes).

Files and the reference lines they follow (units opened in turb.f90:351-395):

* ``collision.dat`` (unit 50, partlib.f90:1722-1735): ``time, icc1, icc2, icc3,
  colltype(1,1), colltype(1,2), colltype(2,2)``, format ``(1pe15.5, 7i10)``, on steps
  with icc1 + icc2 + icc3 > 0.
* ``detectpairs.dat`` (unit 51, partlib.f90:1740-1748): ``time, nir(1,1), nir(1,2),
  nir(2,2)``, format ``(1pe15.5, 3i10)``, on steps with sum(nir) > 0.
* histogram files (partlib.f90:1659-1718), one line per 5-step boundary
  (mod(istep+1, 5) == 0) with the nbin = 180 bins of the accumulated sums of the last
  five steps: ``nirbin{11,12,22}.dat`` format ``(<nbin>(I6))``; ``wrbin``, ``wxbin``,
  ``wybin``, ``wzbin``, ``urbin``, ``thetabin`` (divided by nirbin where that is
  non-zero) and ``wrtanbin`` ``{11,12,22}.dat`` format ``(<nbin>(1pe12.4))``.
* ``Vp11.dat``, ``Vp12.dat``, ``Vp22.dat`` (units 110, 120, 220, opened with
  position='append', partlib.f90:1768-1782): one line per contact-shell record in
  detection order, ``time, va(3), vb(3), xd(3), Wr`` in format
  ``(f10.6, 10(1x,f11.5))``, to unit index1*100 + index2*10.  A set pair whose unit the
  reference never opens (a set index above 2) goes to ``fort.<unit>``, the default file
  of an unopened unit.
* growth diagnostics, every 100th step of a growth run: ``size_dist.dat`` (unit 1001)
  ``istep, npart, npart_t, sizebin(1:360)`` in ``(2x, I10, I10, I10, 360(I10))``,
  ``mdens_dist.dat`` (1002) the same with ``mdensbin`` in ``360(1pe14.6)``
  (SIZE_DIST_LOGARITHMIC, partlib.f90:3921-3925), ``size_avg.dat`` (1003) ``istep, npart,
  npart_t, r_avg, r_max_avg`` and ``st_avg.dat`` (1004) ``istep, npart, npart_t, st_avg,
  st_max_avg`` in ``(2x, I10, I10, I10, 2(1pe14.6))`` (SIZE_AVG 3967-3969, LOCAL_St_AVG
  4325-4326).
* ``meanv_part_vel.dat`` (unit 106) and ``vel_mag_part.dat`` (unit 107), MEAN_VEL
  (partlib.f90:1889-1980): ``time, vpmean(:,1), vpvar(:,1), vpmean(:,2), vpvar(:,2)`` in
  ``13(1pe12.4)`` and ``time, vpabs(:,1), vphoriz(1), vpxyz(1), vpabs(:,2), vphoriz(2),
  vpxyz(2)`` in ``11(1pe12.4)``.

The reference writes set pairs (1,1), (1,2), (2,2) whatever nset is; with nset = 1 it
reads past its arrays for the set-2 entries.  Here an entry of a set above nset is 0.

``time`` is the simulation time at the start of the step (turb.f90:693 advances it after
the particle block).

Edit descriptors follow the Fortran rules: ``Iw`` right-justified, ``1PEw.d`` one digit
before the point and d after, exponent ``E+dd`` (``+ddd`` without the ``E`` for
|exponent| > 99), ``Fw.d`` with the leading zero; a field that does not fit is w
asterisks.  Decimal conversion is correctly rounded, as in the reference's runtime.
"""
from __future__ import annotations

import math
import os

import numpy as np

NBIN = 180
_PAIRS = ((1, 1), (1, 2), (2, 2))
_HIST_ORDER = ("nirbin", "wrbin", "wxbin", "wybin", "wzbin", "urbin", "thetabin", "wrtanbin")  # partlib.f90:1663-1705


# ------------------------------------------------------------------------------------
# Fortran edit descriptors
# ------------------------------------------------------------------------------------
def fmt_i(v, w):
    s = str(int(v))
    return "*" * w if len(s) > w else s.rjust(w)


def fmt_e1p(v, w, d):
    """1PEw.d."""
    v = float(v)
    if math.isnan(v):
        s = "NaN"
    elif math.isinf(v):
        s = ("-" if v < 0 else "+") + "Infinity"
        if len(s) > w:
            s = "-Inf" if v < 0 else "Inf"
    else:
        neg = math.copysign(1.0, v) < 0
        if v == 0.0:
            mant, ex = "0." + "0" * d, 0
        else:
            m, e = f"{abs(v):.{d}e}".split("e")
            mant, ex = m, int(e)
        if abs(ex) <= 99:
            es = "E" + ("-" if ex < 0 else "+") + f"{abs(ex):02d}"
        elif abs(ex) <= 999:
            es = ("-" if ex < 0 else "+") + f"{abs(ex):03d}"
        else:
            return "*" * w
        s = ("-" if neg else "") + mant + es
    return "*" * w if len(s) > w else s.rjust(w)


def fmt_f(v, w, d):
    """Fw.d."""
    v = float(v)
    if math.isnan(v):
        s = "NaN"
    elif math.isinf(v):
        s = "-Infinity" if v < 0 else "Infinity"
        if len(s) > w:
            s = "-Inf" if v < 0 else "Inf"
    else:
        s = f"{v:.{d}f}"
        if len(s) > w:   # the leading zero is optional
            if s.startswith("0."):
                s = s[1:]
            elif s.startswith("-0."):
                s = "-" + s[2:]
    return "*" * w if len(s) > w else s.rjust(w)


def line_e(values, w=12, d=4):
    return "".join(fmt_e1p(x, w, d) for x in values)


def line_i(values, w=6):
    return "".join(fmt_i(x, w) for x in values)


def collision_line(time, icc, colltype):
    """format (1pe15.5, 7i10), partlib.f90:1735."""
    return fmt_e1p(time, 15, 5) + "".join(fmt_i(x, 10) for x in (*icc, *_pair_values(colltype)))


def detectpairs_line(time, nir):
    """format (1pe15.5, 3i10), partlib.f90:1748."""
    return fmt_e1p(time, 15, 5) + "".join(fmt_i(x, 10) for x in _pair_values(nir))


def contact_line(time, rec12):
    """format (f10.6, 10(1x,f11.5)) of buffer(3:12), partlib.f90:1807."""
    return fmt_f(time, 10, 6) + "".join(" " + fmt_f(x, 11, 5) for x in rec12[2:12])


def _pair_values(m):
    """m(index1, index2) (nset, nset) array, 1-based pairs (1,1), (1,2), (2,2)."""
    m = np.asarray(m)
    return [int(m[a - 1, b - 1]) if max(a, b) <= m.shape[0] else 0 for a, b in _PAIRS]


def mean_vel_lines(time, mv, nset):
    """The two MEAN_VEL lines (formats 13(1pe12.4) and 11(1pe12.4), partlib.f90:1964-1970)
    from the 11*nset vector vpmean(3,nset), vpvar(3,nset), vpabs(3,nset), vphoriz(nset),
    vpxyz(nset)."""
    mv = np.asarray(mv, np.float64)
    vpmean = mv[0:3 * nset].reshape(nset, 3)
    vpvar = mv[3 * nset:6 * nset].reshape(nset, 3)
    vpabs = mv[6 * nset:9 * nset].reshape(nset, 3)
    vph = mv[9 * nset:10 * nset]
    vpxyz = mv[10 * nset:11 * nset]
    z3 = np.zeros(3)

    def s3(a, k):
        return a[k] if k < nset else z3

    def s1(a, k):
        return a[k] if k < nset else 0.0

    a = [time, *s3(vpmean, 0), *s3(vpvar, 0), *s3(vpmean, 1), *s3(vpvar, 1)]
    b = [time, *s3(vpabs, 0), s1(vph, 0), s1(vpxyz, 0), *s3(vpabs, 1), s1(vph, 1), s1(vpxyz, 1)]
    return line_e(a), line_e(b)


def histogram_lines(hist):
    """{file name: line} for one 5-step boundary.  hist: the dict of
    Partlib.histograms(written=True), arrays (nbin, nset, nset) indexed [bin, index2-1,
    index1-1]; thetabin already divided by nirbin."""
    out = {}
    nset = hist["nirbin"].shape[1]
    for name in _HIST_ORDER:
        h = np.asarray(hist[name])
        for (a, b) in _PAIRS:
            col = h[:, b - 1, a - 1] if max(a, b) <= nset else np.zeros(h.shape[0], h.dtype)
            fname = f"{name}{a}{b}.dat"
            out[fname] = line_i(col) if name == "nirbin" else line_e(col)
    return out


def _growth_head(istep, npart, npart_t):
    return "  " + fmt_i(istep, 10) + fmt_i(npart, 10) + fmt_i(npart_t, 10)


def size_dist_line(istep, npart, npart_t, sizebin):
    """format (2x, I10, I10, I10, 360(I10)), partlib.f90:3924."""
    return _growth_head(istep, npart, npart_t) + line_i(sizebin, 10)


def mdens_dist_line(istep, npart, npart_t, mdensbin):
    """format (2x, I10, I10, I10, 360(1pe14.6)), partlib.f90:3925."""
    return _growth_head(istep, npart, npart_t) + line_e(mdensbin, 14, 6)


def avg_line(istep, npart, npart_t, a, b):
    """format (2x, I10, I10, I10, 2(1pe14.6)), partlib.f90:3969 and 4326."""
    return _growth_head(istep, npart, npart_t) + line_e((a, b), 14, 6)


def vp_file(index1, index2):
    unit = index1 * 100 + index2 * 10
    return {110: "Vp11.dat", 120: "Vp12.dat", 220: "Vp22.dat"}.get(unit, f"fort.{unit}")


# ------------------------------------------------------------------------------------
# the directory of one run
# ------------------------------------------------------------------------------------
class StatFiles:
    """The statistics directory (``directstat``) of one run.

    All files are opened at construction, as turb.f90:351-395 opens its units: rank 0's
    files start empty (``fresh``; ``fresh=False`` appends, for a restarted run), the Vp
    files are always appended to (position='append').
    """

    def __init__(self, directstat, fresh=True):
        self.dir = directstat
        os.makedirs(directstat, exist_ok=True)
        self._fh = {}
        self._fresh = fresh
        for name in ("collision.dat", "detectpairs.dat", "meanv_part_vel.dat", "vel_mag_part.dat",
                     "size_dist.dat", "mdens_dist.dat", "size_avg.dat", "st_avg.dat",
                     *(f"{h}{a}{b}.dat" for h in _HIST_ORDER for a, b in _PAIRS)):
            self._f(name)
        for a, b in _PAIRS:
            self._f(vp_file(a, b), append=True)

    def _f(self, name, append=False):
        f = self._fh.get(name)
        if f is None:
            mode = "a" if (append or not self._fresh) else "w"
            f = open(os.path.join(self.dir, name), mode)
            self._fh[name] = f
        return f

    def _w(self, name, line, append=False):
        self._f(name, append).write(line + "\n")

    def close(self):
        for f in self._fh.values():
            f.close()
        self._fh.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def flush(self):
        for f in self._fh.values():
            f.flush()

    # -- COLLISION_DET outputs ---------------------------------------------------------
    def write_histograms(self, hist):
        for name, line in histogram_lines(hist).items():
            self._w(name, line)

    def write_counts(self, time, icc, colltype, nir):
        if sum(int(x) for x in icc) > 0:
            self._w("collision.dat", collision_line(time, icc, colltype))
        if int(np.sum(nir)) > 0:
            self._w("detectpairs.dat", detectpairs_line(time, nir))

    def write_contacts(self, time, rec):
        """rec: (n, 12) contact-shell records in detection order."""
        for r in np.asarray(rec, np.float64).reshape(-1, 12):
            self._w(vp_file(int(r[0]), int(r[1])), contact_line(time, r), append=True)

    def collision_det(self, time, partlib, report):
        """All files COLLISION_DET writes for the step just run by
        ``Partlib.collision_det`` or ``Partlib.particle_step`` (report: its CollReport),
        in the reference's order."""
        if report.written:
            self.write_histograms(partlib.histograms(written=True))
        colltype, nir = partlib.collision_counts()
        self.write_counts(time, tuple(report.icc), colltype, nir)
        if report.ncontact:
            _, rec = partlib.contacts()
            self.write_contacts(time, rec)

    # -- MEAN_VEL -----------------------------------------------------------------------
    def write_mean_vel(self, time, mv, nset):
        a, b = mean_vel_lines(time, mv, nset)
        self._w("meanv_part_vel.dat", a)
        self._w("vel_mag_part.dat", b)

    # -- growth diagnostics -------------------------------------------------------------
    def write_size_dist(self, istep, npart, npart_t, sizebin, mdensbin):
        self._w("size_dist.dat", size_dist_line(istep, npart, npart_t, sizebin))
        self._w("mdens_dist.dat", mdens_dist_line(istep, npart, npart_t, mdensbin))

    def write_size_avg(self, istep, npart, npart_t, r_avg, r_max_avg):
        self._w("size_avg.dat", avg_line(istep, npart, npart_t, r_avg, r_max_avg))

    def write_st_avg(self, istep, npart, npart_t, st_avg, st_max_avg):
        self._w("st_avg.dat", avg_line(istep, npart, npart_t, st_avg, st_max_avg))
