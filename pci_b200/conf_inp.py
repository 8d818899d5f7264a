"""The reference's configuration input CONF.INP, read and written, and
conf_pt's reordered list CONF_new.INP.

Layout, as conf_init reads it (src/conf_init.f90:37-135, 215-312): a name
line; `key = value` lines (a `#` starts a comment; keys are case-blind and
the reader keeps their first 4 characters, values their first 10); the first
line without `=` ends them (a blank one is skipped).  Then the Nso core
shells and the Nc configurations as shell codes, six to a line in the
fixed fields of `(6(4X,F7.4))` (field k spans columns 11k+4 .. 11k+10); a
configuration runs over as many lines as it takes to hold Ne electrons, and
on each line its shells end at the first empty or zero field, so lines
whose fields are blank (conf_pt's weight lines, its `<CI<` marker) add
nothing.

A shell code is +-(n/10 + l/100 + qq/10000) (pconf's decoding,
src/pconf.F90:506-529): 0.nlqq for n < 10 and 1.0lqq for n = 10, l one digit,
qq the occupation, the sign + for j = l + 1/2 and - for j = l - 1/2; the
orbital is the basis orbital with that n and kappa = -sign * (j + 1/2).
"""
from __future__ import annotations

import math

# ReadConfInp's defaults of the optional keys (conf_init.f90:219-231)
DEFAULTS = {"K_IS": 0, "C_IS": 0.0, "KLOW": 0, "KBRT": 0, "KOUT": 1, "GJ": 0.0, "N_IT": 20, "CUT0": 0.001,
            "NCPT": 0, "GNUC": 1.0, "QNUC": 1.0}
INT_KEYS = {"NSO", "NC", "KV", "NLV", "NE", "KL4", "NC4", "KOUT", "NCPT", "N_IT", "KBRT", "K_IS", "KLOW"}
REAL_KEYS = {"Z", "AM", "J", "JM", "GJ", "CRT4", "CUT0", "C_IS", "GNUC", "QNUC"}


def decode_qnl(x: float):
    """(n, l, 2j, kappa, q) of a shell code (src/pconf.F90:507-518)."""
    i = 1 if x >= 0 else -1
    d = abs(x) + 1e-14
    d = 10.0 * d
    n = int(d)
    d = 10.0 * (d - n)
    l = int(d)
    j2 = 2 * l + i
    kappa = -i * ((j2 + 1) // 2)
    d = 100.0 * (d - l)
    q = int(d + 0.1)
    return n, l, j2, kappa, q


def encode_qnl(n: int, l: int, j2: int, q: int) -> float:
    """The shell code of q electrons in (n, l, j = j2/2)."""
    if not (0 <= n <= 99 and 0 <= l <= 9 and 0 <= q <= 99):
        raise ValueError("a shell code holds n < 100, one digit of l and two of q")
    if j2 not in (2 * l + 1, 2 * l - 1):
        raise ValueError("j must be l +- 1/2")
    sign = 1.0 if j2 == 2 * l + 1 else -1.0
    return sign * (n / 10.0 + l / 100.0 + q / 10000.0)


def _electrons(x: float) -> int:
    """ReadConfigurations' electron count of a field (conf_init.f90:294-298)."""
    a = abs(x) + 1e-9
    return int(10000 * a) - 100 * int(100 * a)


def _fields(line: str):
    """The six F7.4 fields of a line; a blank field reads as 0."""
    out = []
    for k in range(6):
        f = line[11 * k + 4:11 * k + 11]
        s = f.strip()
        if not s:
            out.append(0.0)
            continue
        try:
            v = float(s)
        except ValueError:
            v = 0.0                      # a marker or label: no shell
        if "." not in s and "e" not in s.lower():
            v /= 1e4                     # F7.4 without a decimal point: four implied decimals
        out.append(v)
    return out


def read_conf_inp(text: str):
    """Parse CONF.INP text.  Returns dict name, params (upper-case keys, the
    optional ones defaulted), core ([Nso] shell codes) and configs ([Nc]
    lists of shell codes)."""
    lines = text.splitlines()
    if not lines:
        raise ValueError("empty CONF.INP")
    name = lines[0][1:17] if len(lines[0]) > 1 else ""
    params = dict(DEFAULTS)
    p = 1
    while p < len(lines) and "=" in lines[p]:
        key, val = lines[p].split("=", 1)
        key = key.strip()[:4].upper()
        val = val.strip()[:10]
        if "#" in val:
            val = val[:val.index("#")].strip()
        num = val.replace("d", "e").replace("D", "e")   # Fortran's double-precision exponent
        if key in INT_KEYS:
            params[key] = int(float(num))
        elif key in REAL_KEYS:
            params[key] = float(num)
        p += 1
    if p < len(lines) and lines[p].strip() == "":
        p += 1
    for k in ("NSO", "NC", "NE"):
        if k not in params:
            raise ValueError(f"CONF.INP has no {k}")
    nso, nc, ne = params["NSO"], params["NC"], params["NE"]
    core = []
    while len(core) < nso:
        if p >= len(lines):
            raise ValueError("CONF.INP ends inside the core shells")
        core.extend(_fields(lines[p])[:nso - len(core)])
        p += 1
    configs = []
    for ic in range(nc):
        shells, ne0 = [], 0
        while ne0 < ne:
            if p >= len(lines):
                raise ValueError(f"CONF.INP ends inside configuration {ic + 1}")
            for x in _fields(lines[p]):
                if abs(x) + 1e-9 < 1e-8:
                    break
                shells.append(x)
                ne0 += _electrons(x)
            p += 1
        if ne0 > ne:
            raise ValueError(f"too many electrons for configuration {ic + 1}")
        configs.append(shells)
    return {"name": name, "params": params, "core": core, "configs": configs}


def orbital_of(basis, x: float) -> int:
    """The 1-based basis orbital of a shell code (n and kappa match), as
    pconf's Init finds it; ValueError when there is none."""
    n, l, j2, kappa, q = decode_qnl(x)
    kk = getattr(basis, "kk", None)
    for ni in range(basis.ns):
        if int(basis.nn[ni]) != n:
            continue
        if kk is not None and int(kk[ni]) == kappa:
            return ni + 1
        if kk is None and int(basis.ll[ni]) == l and int(basis.jj[ni]) == j2:
            return ni + 1
    raise ValueError(f"no orbital for shell n={n} l={l} kappa={kappa}")


def configs_from_qnl(basis, configs_qnl):
    """The configurations as [(orbital, occupation)] shell lists."""
    return [[(orbital_of(basis, x), decode_qnl(x)[4]) for x in conf] for conf in configs_qnl]


def configs_to_qnl(basis, configs):
    """Shell codes of [(orbital, occupation)] configurations."""
    return [[encode_qnl(int(basis.nn[ni - 1]), int(basis.ll[ni - 1]), int(basis.jj[ni - 1]), int(q))
             for ni, q in conf] for conf in configs]


def _shell_lines(codes, number=None):
    """Six codes to a line in `(6(4X,F7.4))` fields; the first line may carry
    a configuration number in the first four columns (NewConfList's I4)."""
    out = []
    for k in range(0, max(len(codes), 1), 6):
        head = f"{number % 10000:4d}" if (number is not None and k == 0) else "    "
        row = codes[k:k + 6]
        out.append(head + "    ".join(f"{x:7.4f}" for x in row))
    return out


def write_conf_inp(name, params, core, configs, order=None, ci_marker_at=None, nr_lines=None):
    """CONF.INP text: the name line, `key = value` lines for params (in the
    given order), the core shells, then the configurations (each starting
    on its own line with its 1-based number).  order: the configuration
    indices to write (all, as given, by default); ci_marker_at: position in
    that order before which conf_pt's `<CI<` line goes; nr_lines: {position:
    text} lines written before the configuration at that position
    (NewConfList's NR-configuration lines)."""
    out = [" " + str(name)]                      # the reader keeps columns 2-17
    for k, v in params.items():
        if isinstance(v, float):
            out.append(f"{k} = {v:.6g}" if abs(v) >= 1e-3 or v == 0 else f"{k} = {v:.3e}")
        else:
            out.append(f"{k} = {v}")
    if core:
        for k in range(0, len(core), 6):
            out.append("".join(f"    {x:7.4f}" for x in core[k:k + 6]))
    order = list(range(len(configs))) if order is None else list(order)
    for pos, ic in enumerate(order):
        if ci_marker_at is not None and pos == ci_marker_at:
            out.append("<CI<")
        if nr_lines and pos in nr_lines:
            out.append(nr_lines[pos])
        out.extend(_shell_lines(configs[ic], pos + 1))
    out.append(" >>>>>>>>>> END <<<<<<<<<<")
    return "\n".join(out) + "\n"


def new_conf_inp(parsed, selection, layout):
    """NewConfList's CONF_new.INP (src/conf_pt.f90:1130-1264) from a parsed
    CONF.INP, pci_b200.conf_pt.select_configurations' result and the
    nr_layout of its configurations: the name marked `(reordered)`, Nc the
    new CI space, Kl4 and Nc4 updated where the input has them, and every
    configuration in the new order, each NR configuration headed by a line
    with its number, weight and shell count in columns that the reader
    skips, the `<CI<` line before the first configuration left out of the
    CI space."""
    params = dict(parsed["params"])
    params["NC"] = int(selection["nci"])
    if "KL4" in params:
        params["KL4"] = int(selection["kl4"])
    if "NC4" in params:
        params["NC4"] = int(selection["nc4"])
    nrn, nvcnr = layout["nrn"], layout["nvcnr"]
    nr_lines, pos, marker = {}, 0, None
    kept = selection["cutoff"]["w"][:, 1]
    for rank, (k, w) in enumerate(zip(selection["nr_order"], selection["weights"])):
        if marker is None and kept[k] == 0.0:
            marker = pos
        nr_lines[pos] = f"{(rank + 1) % 10000:4d}" + " " * 62 + f"{w:9.2E}" + f"{int(nvcnr[k]):6d}"
        pos += int(nrn[k])
    return write_conf_inp(parsed["name"].ljust(16)[:16] + " (reordered)", params, parsed["core"], parsed["configs"],
                          order=selection["conf_order"], ci_marker_at=marker, nr_lines=nr_lines)


def system_from_files(conf_inp, conf_int, conf_gnt=None, name=None):
    """A CISystem from the reference's input files, as pconf assembles it:
    CONF.INP (text, or a path) for the configurations and the job keys;
    CONF.INT for the orbital table (Nn, Kk, Ll, Jj of orbitals 1..Nsu, which
    the reference's Rint reads over CONF.DAT's, src/integrals.f90:35-52), Nso,
    the core energy and the radial integrals (Nx = sqrt(nrd)); CONF.GNT for
    the Gaunt factors (the exact 3j table of pci_b200.wigner when absent).
    Determinants are Dinit's over all orbitals' m-states (core included, as
    the reference numbers them); configurations without a determinant of
    2M = 2|Jm| are kept, as in the reference."""
    import os

    import numpy as np

    from . import files, wigner
    from .system import Basis, CISystem, enumerate_determinants, m_states

    text = conf_inp
    if "\n" not in str(conf_inp) and os.path.exists(str(conf_inp)):
        with open(conf_inp) as f:
            text = f.read()
    parsed = read_conf_inp(text)
    p = parsed["params"]
    # pconf drops the isotope-shift operator when |C_is| < 1e-6 (pconf.F90:335-336);
    # its terms in Hint / Gint (integrals.f90:141-143) are not part of this engine's H
    if p.get("K_IS", 0) != 0 and abs(p.get("C_IS", 0.0)) >= 1e-6:
        raise ValueError("CONF.INP asks for the isotope-shift operator (K_is, C_is), which this engine does not add to H")
    ci = files.read_int(conf_int)
    h = ci.header
    if int(h.nso) != p["NSO"]:
        raise ValueError(f"CONF.INT has Nso = {h.nso}, CONF.INP {p['NSO']}")
    if int(h.kbrt) != p.get("KBRT", 0):   # Rint stops here too (integrals.f90:53-60)
        raise ValueError(f"CONF.INT's integrals are for Kbrt = {h.kbrt}, CONF.INP asks for {p.get('KBRT', 0)}")
    orb = ci.orbitals
    basis = Basis(nn=orb[:, 0].astype(np.int32), ll=orb[:, 2].astype(np.int32), kk=orb[:, 1].astype(np.int32),
                  jj=orb[:, 3].astype(np.int32), nso=int(h.nso))
    configs = configs_from_qnl(basis, parsed["configs"])
    ne = p["NE"]
    mj = int(2 * abs(p["JM"]) + 0.01)
    iarr, ndc = enumerate_determinants(basis, configs, ne, mj)
    nsu = max(ni for c in configs for ni, _ in c)
    if nsu > basis.ns:
        raise ValueError(f"the configurations reach orbital {nsu}; CONF.INT holds {basis.ns}")
    jz, nh, _ = m_states(basis, nsu)
    nx = int(round(math.sqrt(h.nrd)))
    lut = files.hint_lut(ci.rint1, ci.iint1, nx)
    if conf_gnt is not None:
        nlx, per, gin, ggnt = files.read_gnt(conf_gnt)
        glut = files.gaunt_lut(gin, ggnt)
    else:
        nlx, gin, ggnt, per = wigner.gaunt_table(int(basis.ll[:nsu].max()))
        glut = wigner.gaunt_lut(gin, ggnt)
    params = dict(Nlv=p.get("NLV", 6), N_it=p.get("N_IT", 20), Crt4=p.get("CRT4", 1e-4), Kl4=p.get("KL4", 1),
                  Kv=p.get("KV", 4), MaxNd0=3000, Nc4=p.get("NC4", len(configs)), KXIJ=0, admix_crit=1e-6)
    return CISystem(name=name or parsed["name"].strip(), basis=basis, ne=ne, mj=mj, configs=configs, iarr=iarr,
                    ndc=ndc, jz=jz, nh=nh, nsu=nsu, nx=nx, hint_lut=lut, rint2=ci.rint2, iint2=ci.iint2,
                    iint3=ci.iint3, kbrt=int(h.kbrt), nlx=nlx, gaunt_in=gin, gaunt_gnt=ggnt, gaunt_per_wave=per,
                    gaunt_lut=glut, gj=float(p.get("GJ", 0.0)), xj_av=float(p.get("J", 0.0)),
                    ecore=float(h.ecore), params=params)
