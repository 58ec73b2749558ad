"""Restart files of the reference (restart.c), text form.

``read_rdump`` parses a ``dumps/rdump-N`` file written by the reference's
restart_write() (restart.c:182-222; header write_restart_header,
restart.c:553-690, with the WRITERESTARTHEADER layout of global.h:929-935;
then the active zones' primitives, x1 fastest, "%21.15g " each), so a run
can continue on the device from a reference restart: upload ``prims`` with
HarmGPU.set_prims() (ghost zones then from bound_prims()) and t, dt,
realnstep with set_time().

``write_rdump`` writes the same layout.  The evolution state (t, dt, step
counts, knobs, primitives) comes from the caller or a context
(``rdump_header_from_context``); the accounting totals in the header
(pcumreg_tot, fladdreg_tot, sourceaddreg_tot, Ureg_init_tot, the failure
and floor counters, prMAX, lumvsr_tot) are diagnostics that the device step
does not accumulate: they are carried over from a header that was read, or
written as zeros.
"""
import numpy as np

# (name, printf conversion) in the order of WRITERESTARTHEADER
HEADER_FIELDS = (
    [("totalsize1", "d"), ("totalsize2", "d")]
    + [("t", "g"), ("tf", "g"), ("nstep", "d"), ("a", "g"), ("gam", "g"), ("cour", "g")]
    + [("DTd", "g"), ("DTavg", "g"), ("DTener", "g"), ("DTi", "g"), ("DTr", "d"), ("DTdebug", "g"),
       ("dump_cnt", "d"), ("image_cnt", "d"), ("rdump_cnt", "d"), ("avg_cnt", "d"), ("debug_cnt", "d")]
    + [("dt", "g"), ("lim", "d"), ("TIMEORDER", "d"), ("fluxmethod", "d"), ("FLUXB", "d"),
       ("UTOPRIMVERSION", "d"), ("failed", "d")]
    + [("R0", "g"), ("Rin", "g"), ("Rout", "g"), ("hslope", "g"), ("defcoord", "d")]
    + [("BC_X1UP", "d"), ("BC_X1DN", "d"), ("BC_X2UP", "d"), ("BC_X2DN", "d")]
    + [("realnstep", "d"), ("debugfail", "d"), ("whichrestart", "d"), ("cooling", "d"), ("restartsteps0", "d"),
       ("restartsteps1", "d")]
    + [(k, "d") for k in ("GAMMIEDUMP", "GAMMIEIMAGE", "GAMMIEENER", "DODIAGS", "DOENERDIAG", "DOGDUMPDIAG",
                          "DORDUMPDIAG", "DODUMPDIAG", "DOAVGDIAG", "DOIMAGEDIAG", "DOAREAMAPDIAG", "POSDEFMETRIC",
                          "periodicx1", "periodicx2", "binaryoutput", "sortedoutput")]
    + [(k, "g") for k in ("defcon", "SAFE", "RHOMIN", "UUMIN", "RHOMINLIMIT", "UUMINLIMIT", "BSQORHOLIMIT",
                          "BSQOULIMIT", "GAMMAMAX", "GAMMADAMP", "GAMMAFAIL")]
)
# accounting blocks after the fixed fields (NUMENERREGIONS 3, COMPDIM*2 = 4
# directions, NPRDUMP 8, NUMTSCALES 4 x NUMFAILFLOORFLAGS 9 as doubles)
ACCOUNTING_DOUBLES = 3 * 4 * 8 + 3 * 8 + 3 * 8 + 3 * 8 + 4 * 9 + 8
NPR = 8


def _fmt(conv, v):
    return "%21.15g" % float(v) if conv == "g" else "%d" % int(v)


def _header_line(h, accounting, rescaletype, lumvsr):
    parts = []
    for name, conv in HEADER_FIELDS:
        # WRITERESTARTHEADER joins debug_cnt and dt without a separator
        parts.append(_fmt(conv, h[name]) + ("" if name == "debug_cnt" else " "))
    out = "".join(parts)
    out += "".join("%21.15g " % float(x) for x in accounting)
    out += "%d " % int(rescaletype)
    out += "".join("%21.15g " % float(x) for x in lumvsr)
    return out + "\n"


def read_rdump(path):
    """Returns dict(header=dict, accounting=list, rescaletype=int,
    lumvsr=list, prims=[n1, n2, 8] active zones).  A file cut short or
    holding a token that is not a number raises ValueError naming the file
    and the part that is missing or bad; no partial state is returned."""
    with open(path, "r") as f:
        first = f.readline()
        rest = f.read()
    tok = first.split()
    nfixed = len(HEADER_FIELDS)
    if len(tok) < nfixed:
        raise ValueError(f"rdump {path}: header holds {len(tok)} of its {nfixed} fixed fields (file cut short?)")
    h = {}
    for (name, conv), s in zip(HEADER_FIELDS, tok[:nfixed]):
        try:
            h[name] = float(s) if conv == "g" else int(s)
        except ValueError:
            raise ValueError(f"rdump {path}: header field {name} = {s!r} is not a number") from None
    n1, n2 = h["totalsize1"], h["totalsize2"]
    if n1 <= 0 or n2 <= 0:
        raise ValueError(f"rdump {path}: grid {n1} x {n2} in the header")
    ntail = ACCOUNTING_DOUBLES + 1 + n1
    if len(tok) != nfixed + ntail:
        raise ValueError(f"rdump {path}: header holds {len(tok) - nfixed} accounting values where the "
                         f"{n1}-zone grid needs {ntail} (file cut short?)")
    try:
        acc = [float(x) for x in tok[nfixed:nfixed + ACCOUNTING_DOUBLES]]
        resc = int(tok[nfixed + ACCOUNTING_DOUBLES])
        lum = [float(x) for x in tok[nfixed + ACCOUNTING_DOUBLES + 1:]]
    except ValueError as e:
        raise ValueError(f"rdump {path}: bad accounting value in the header ({e})") from None
    try:
        vals = np.array(rest.split(), dtype=np.float64)
    except ValueError as e:
        raise ValueError(f"rdump {path}: a primitive is not a number ({e})") from None
    if vals.size != n1 * n2 * NPR:
        raise ValueError(f"rdump {path}: {vals.size} values for a {n1} x {n2} grid of {NPR} primitives "
                         f"(file cut short?)")
    if not np.isfinite(vals).all():
        raise ValueError(f"rdump {path}: {int((~np.isfinite(vals)).sum())} primitives are not finite")
    # DUMPLOOP order: j outer, i inner (global.h:1047)
    prims = vals.reshape(n2, n1, NPR).transpose(1, 0, 2).copy()
    return dict(header=h, accounting=acc, rescaletype=resc, lumvsr=lum, prims=prims)


def write_rdump(path, header, prims, accounting=None, rescaletype=0, lumvsr=None):
    """Writes a reference text restart file.  prims: [n1, n2, 8] active
    zones (or the full [n1+6, n2+6, 8] array, whose ghosts are dropped)."""
    n1, n2 = int(header["totalsize1"]), int(header["totalsize2"])
    p = np.asarray(prims, dtype=np.float64)
    if p.shape == (n1 + 6, n2 + 6, NPR):
        p = p[3:-3, 3:-3]
    if p.shape != (n1, n2, NPR):
        raise ValueError(f"prims shape {p.shape} does not match {n1} x {n2}")
    acc = list(accounting) if accounting is not None else [0.0] * ACCOUNTING_DOUBLES
    lum = list(lumvsr) if lumvsr is not None else [0.0] * n1
    lines = [_header_line(header, acc, rescaletype, lum)]
    pj = p.transpose(1, 0, 2).reshape(n1 * n2, NPR)
    lines.extend("".join("%21.15g " % x for x in row) + "\n" for row in pj.tolist())
    with open(path, "w") as f:
        f.write("".join(lines))


def rdump_header_from_context(h, template):
    """A header for write_rdump(): the template's fields (cadences, counters,
    coordinates, flags) with the context's time, step counts and grid."""
    st = h.sync(raise_on_fail=False)
    out = dict(template)
    out.update(t=st["t"], dt=st["dt"], nstep=st["realnstep"], realnstep=st["realnstep"], totalsize1=h.n1,
               totalsize2=h.n2)
    return out
