"""Expected outputs of the reference driver (src/main.rs run_uniform /
run_octree) computed on the FP64 oracle, with Rust's float formats restated
in Python: the checker of the ``cavity_les`` tests (test infrastructure).

Rust formats (core::fmt), independent of the driver's C++ restatement:
  {:.p}   fixed, round-half-even on the exact value   -> rust_fixed
  {:.pe}  scientific, exponent without '+' / padding  -> rust_exp
  {:e}    shortest round-trip digits, scientific      -> rust_exp_short
  {}      shortest round-trip digits, positional      -> rust_display
"""
from __future__ import annotations

import math
from decimal import Decimal

import numpy as np

import oracle

DELTA_T = 1.0


def _special(x):
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return None


def rust_fixed(x, p):
    return _special(x) or f"{x:.{p}f}"


def _fix_exp(s):
    m, e = s.split("e")
    return f"{m}e{int(e)}"


def rust_exp(x, p):
    return _special(x) or _fix_exp(f"{x:.{p}e}")


def _shortest(x):
    """(sign, digits, e10): x = d0.d1d2... * 10**e10, shortest round trip."""
    t = Decimal(repr(float(x))).as_tuple()
    digits = "".join(map(str, t.digits)).lstrip("0") or "0"
    # value = int(digits_all) * 10**exponent; strip trailing zeros
    n_all = len(t.digits)
    lead = n_all - len("".join(map(str, t.digits)).lstrip("0") or "0")
    e10 = t.exponent + n_all - 1 - lead
    digits = digits.rstrip("0") or "0"
    return ("-" if t.sign else ""), digits, (0 if digits == "0" else e10)


def rust_exp_short(x):
    s = _special(x)
    if s:
        return s
    sign, d, e = _shortest(x)
    return f"{sign}{d[0]}{'.' + d[1:] if len(d) > 1 else ''}e{e}"


def rust_display(x):
    s = _special(x)
    if s:
        return s
    sign, d, e = _shortest(x)
    if d == "0":
        return sign + "0"
    if e >= 0:
        ip = e + 1
        if len(d) <= ip:
            return sign + d + "0" * (ip - len(d))
        return sign + d[:ip] + "." + d[ip:]
    return sign + "0." + "0" * (-e - 1) + d


# ---- run_uniform (src/main.rs:42-443) on the oracle --------------------------
def uniform_run(nx, ny, ra, steps, sample_start, sample_every, progress_every, pr=0.71, cs=0.10,
                pr_t=0.9, utarget=0.02, seed=42):
    s = oracle.OracleSolver(nx, ny, ra, pr, cs, pr_t, utarget, seed)
    n = nx * ny
    avg = oracle.OracleAverager(n)
    log = []
    for step in range(steps):
        s.step(1)
        if step % progress_every == 0 or step + 1 == steps:
            d = s.diag()
            log.append(f"step {step:>7} | w_max = {rust_fixed(d['max_uy'], 5)} | max_u = "
                       f"{rust_fixed(d['max_u'], 5)} | Nuc = {rust_fixed(d['nusselt_hot'], 4)} | Nuf = "
                       f"{rust_fixed(d['nusselt_cold'], 4)} | masse = {rust_fixed(d['total_mass'] / n, 6)} | "
                       f"nu_t_max = {rust_exp(d['nu_t_max'], 3)}")
        if step >= sample_start and (step - sample_start) % sample_every == 0:
            avg.accumulate(s)
    cnt, (ux, uy, t, nut, uu) = avg.means()
    info = s.info()
    out = {"progress.log": "".join(line + "\n" for line in log), "n_samples": cnt}
    psi = np.zeros(n)
    for ix in range(nx):
        acc = 0.0
        for iy in range(1, ny):
            acc += 0.5 * (ux[(iy - 1) * nx + ix] + ux[iy * nx + ix])
            psi[iy * nx + ix] = acc

    def nu_mean(hot):
        sm = 0.0
        for iy in range(ny):
            g = t[iy * nx + 1] - t[iy * nx + 2] if hot else t[iy * nx + nx - 3] - t[iy * nx + nx - 2]
            sm += abs(g)
        return (sm / ny) * info["lz"] / DELTA_T

    nuc, nuf = nu_mean(True), nu_mean(False)
    iy_mid, iy_075 = ny // 2, 3 * ny // 4
    uy_mid = [uy[iy_mid * nx + ix] for ix in range(nx)]
    uy_075 = [uy[iy_075 * nx + ix] for ix in range(nx)]

    def max_of(p):
        best, bi = 0.0, 1
        for i in range(1, nx - 1):
            if abs(p[i]) > best:
                best, bi = abs(p[i]), i
        return best, bi / (nx - 1)

    wmax_mid, x_mid = max_of(uy_mid)
    wmax_075, x_075 = max_of(uy_075)
    lines = ["x,y,ux,uy,T,psi,nu_t\n"]
    for iy in range(ny):
        for ix in range(nx):
            k = iy * nx + ix
            lines.append(f"{rust_fixed(float(ix), 6)},{rust_fixed(float(iy), 6)},{rust_exp(ux[k], 8)},"
                         f"{rust_exp(uy[k], 8)},{rust_exp(t[k], 8)},{rust_exp(psi[k], 8)},{rust_exp(nut[k], 8)}\n")
    out["fields_mean.csv"] = "".join(lines)
    out["profiles_w.csv"] = "x_norm,w_z05,w_z075\n" + "".join(
        f"{rust_fixed(ix / (nx - 1), 6)},{rust_exp(uy_mid[ix], 8)},{rust_exp(uy_075[ix], 8)}\n"
        for ix in range(nx))
    f = s.fields()
    rows = {}
    for key, name in (("temperature", "T"), ("ux", "U"), ("uy", "V")):
        rows[name] = "".join("".join(rust_exp(f[key][iy * nx + ix], 6) + " " for ix in range(nx)) + "\n"
                             for iy in range(ny))
    ext = f"0 {nx - 1} 0 {ny - 1} 0 0"
    out["snapshot.vti"] = (
        '<?xml version="1.0"?>\n'
        '<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian">\n'
        f'  <ImageData WholeExtent="{ext}" Origin="0 0 0" Spacing="1 1 1">\n'
        f'    <Piece Extent="{ext}">\n'
        '      <PointData Scalars="Temperature">\n'
        '        <DataArray type="Float64" Name="Temperature" format="ascii">\n'
        f'{rows["T"]}        </DataArray>\n'
        '        <DataArray type="Float64" Name="Ux" format="ascii">\n'
        f'{rows["U"]}        </DataArray>\n'
        '        <DataArray type="Float64" Name="Uy" format="ascii">\n'
        f'{rows["V"]}        </DataArray>\n'
        '      </PointData>\n      <CellData>\n      </CellData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n')
    snap = bytearray(b"CAVSNAP1") + np.array([nx, ny], dtype="<u8").tobytes()
    for key in ("rho", "ux", "uy", "temperature"):
        snap += np.ascontiguousarray(f[key], dtype="<f8").tobytes()
    out["snapshot.bin"] = bytes(snap)
    d = s.diag()
    out["summary"] = {"nuc": nuc, "nuf": nuf, "nu_vol": d["nusselt_volume"], "wmax_mid": wmax_mid,
                      "x_mid": x_mid, "wmax_075": wmax_075, "x_075": x_075, "yplus": d["y_plus_hot"]}
    out["summary.json"] = (
        "{\n"
        '  "case": "differentially_heated_cavity_2d",\n'
        f'  "ra": {rust_exp_short(ra)},\n'
        f'  "cs": {rust_display(cs)},\n'
        f'  "grid": [{{"nx": {nx}, "ny": {ny}}}],\n'
        f'  "aspect_ratio": {rust_fixed((ny - 1) / (nx - 1), 4)},\n'
        f'  "steps": {steps},\n'
        f'  "time_samples": {cnt},\n'
        f'  "nusselt_hot": {rust_fixed(nuc, 4)},\n'
        f'  "nusselt_cold": {rust_fixed(nuf, 4)},\n'
        f'  "nusselt_volume": {rust_fixed(d["nusselt_volume"], 4)},\n'
        f'  "wmax_z05": {rust_fixed(wmax_mid, 5)},\n'
        f'  "x_wmax_z05": {rust_fixed(x_mid, 5)},\n'
        f'  "wmax_z075": {rust_fixed(wmax_075, 5)},\n'
        f'  "x_wmax_z075": {rust_fixed(x_075, 5)},\n'
        f'  "y_plus_hot": {rust_fixed(d["y_plus_hot"], 3)},\n'
        '  "references_thesis_tab27": {\n'
        '    "nuc_snd": 102.0,\n'
        '    "nuc_les_these": [100.2, 100.5],\n'
        '    "wmax_z05": [0.22, 0.24],\n'
        '    "x_wmax_z05": 0.004,\n'
        '    "wmax_z075": [0.11, 0.17],\n'
        '    "x_wmax_z075": 0.005,\n'
        '    "s_half": [1.10, 1.20]\n'
        "  }\n"
        "}\n")
    return out


# ---- run_octree (src/main.rs:447-720) on the oracle --------------------------
def octree_progress(nx0, ny0, bl_width, ra, steps, sample_start, sample_every, progress_every, levels=2,
                    pr=0.71, utarget=0.02, seed=42):
    o = oracle.OracleOctree(nx0, ny0, bl_width, ra, pr, utarget, seed, levels=levels)
    log = []
    sums = [0.0, 0.0, 0.0, 0.0]
    cnt = 0
    nmax = imax = 0.0
    for step in range(steps):
        o.step_cavity(1)
        if step >= sample_start and (step - sample_start) % sample_every == 0:
            d = o.diag()
            for j, k in enumerate(("nu_hot", "nu_cold", "nu_hot_link0", "nu_hot_fine")):
                sums[j] += d[k]
            cnt += 1
        if step % progress_every == 0 or step + 1 == steps:
            d = o.diag()
            nmax = max(nmax, d["max_rho_dev"])
            imax = max(imax, d["max_rho_dev_ifaces"])
            log.append(f"step {step:>7} | max_rho_dev = {rust_exp(d['max_rho_dev'], 3)} | max_rho_dev_ifaces = "
                       f"{rust_exp(d['max_rho_dev_ifaces'], 3)} | masse = {rust_fixed(d['mass'], 6)} | Nuc = "
                       f"{rust_fixed(d['nu_hot'], 4)} | Nuc_link0 = {rust_fixed(d['nu_hot_link0'], 4)} | Nuf = "
                       f"{rust_fixed(d['nu_cold'], 4)} | Nu_fin = {rust_fixed(d['nu_hot_fine'], 4)} | max_u = "
                       f"{rust_fixed(d['max_u'], 5)}")
    return log, [v / cnt for v in sums] if cnt else None, cnt, nmax, imax
