"""Natural-parameter continuation over wall separation and pH.

Restates the sweep routines of the reference:

* `adjust_distancesZ` (`routines/adjust_distanceZ.jl:15-155`): the wall
  separation grows by `stepZ` per step; each step rebuilds the system, starts
  from the previous solution, solves, records the grand potential, the energy
  Omega + P_bulk H and the contact-value pressure, and the sweep stops after 20
  consecutive steps with |dE| < errP or past `stopZ`;
* `adjust_pH` (`routines/adjust_pH.jl:16-125`): pH (the pSpecies of the `Y`
  species) runs over start:step:stop; each step writes the analysis files and
  reads back the brush height and the average degree of ionisation, and the
  sweep stops once alpha reaches 0.99 (rising pH) or 0.01 (falling pH);
* `batched_distance_sweep`: the wall-separation sweep of many independent
  branches at once, every step of all branches solved in one batched device
  launch.

Warm start.  The routines copy the near-wall halves of the previous segment and
bond densities and PsiC into the new system, but the solver's unknowns are
(mu_ex_K, lng_K, Psi, PsiC) (`solver_dft.jl:13`) and `eval_spatial_density!`
recomputes the densities from them, so in the reference only PsiC carries over.
Here the unknowns themselves carry over: the point at distance d from the
nearer wall of the new slit takes the previous solution's value at distance d
from the same wall (linear interpolation; the previous slit's midpoint value
beyond its half width).  With an unchanged grid spacing and a change of H by
whole grid spacings this is the routines' index copy of the near-wall halves.

Grid.  A step with wall separation H and requested spacing dz uses the
reference's grid NP = cld(H, dz) + 1 whenever the device transform runs it
(native.grid_supported: NP >= 16 whose FFT length fits one CTA's shared memory,
by mixed radix or, for a prime factor above 61, by Bluestein's transform);
otherwise the spacing is an upper bound and
NP is the next supported size, at spacing H / (NP - 1) (nudged so that the
reference's rule gives exactly NP).  `grid="pow2"` keeps the earlier policy of
power-of-two grids, `grid="exact"` the requested spacing as is.
"""
from __future__ import annotations

import copy
import math
import os
from typing import List, Optional, Sequence

import numpy as np

from . import native
from .api import (IsingDFT, densities, eval_inhomogeneous, geometry_system, grand_potential, iLST, setup_iDFT,
                  state_fractions)
from .host.descriptor import numerics_from_dict
from .host.geometry import cld
from .output import brush_height_values, call_analysis, contact_value_theorem_arrays, jl


# ---- grid and warm start ------------------------------------------------------

def pow2_bin_width(H: float, dz: float) -> float:
    """Spacing <= dz for which NP = cld(H, spacing) + 1 is a power of two."""
    need = cld(H, dz) + 1
    NP = 1 << max(4, math.ceil(math.log2(need)))
    w = H / (NP - 1)
    while cld(H, w) + 1 > NP:
        w = math.nextafter(w, math.inf)
    while cld(H, w) + 1 < NP:
        w = math.nextafter(w, 0.0)
    return w


def _width_for(H: float, dz: float, NP: int) -> float:
    """Spacing near H / (NP - 1) for which NP = cld(H, spacing) + 1 exactly."""
    w = H / (NP - 1)
    while cld(H, w) + 1 > NP:
        w = math.nextafter(w, math.inf)
    while cld(H, w) + 1 < NP:
        w = math.nextafter(w, 0.0)
    return w


def supported_bin_width(H: float, dz: float) -> float:
    """dz when the device runs the reference's grid cld(H, dz) + 1, else the
    spacing < dz of the next grid size the device runs."""
    NP = cld(H, dz) + 1
    if native.grid_supported(NP):
        return dz
    NP = max(NP, 16)
    while not native.grid_supported(NP):
        NP += 1
        if NP > 1 << 16:
            raise ValueError(f"no device grid for H = {H} at spacing <= {dz}")
    return _width_for(H, dz, NP)


def set_distance(data: dict, H: float, dz: Optional[float] = None, grid: str = "device") -> None:
    """Wall separation H in place (data["geometry"]["dimensions"] = [H]); the
    spacing follows `grid` ("device", "pow2" or "exact", see the module text)."""
    g = data["geometry"]
    g["dimensions"] = [H]
    base = float(dz if dz is not None else g["bin_width"][0])
    if grid == "device":
        g["bin_width"] = [supported_bin_width(H, base)]
    elif grid == "pow2":
        g["bin_width"] = [pow2_bin_width(H, base)]
    elif grid == "exact":
        g["bin_width"] = [base]
    else:
        raise ValueError(f"grid must be 'device', 'pow2' or 'exact' (got {grid!r})")


def _resample(f: np.ndarray, np_old: int, dz_old: float, np_new: int, dz_new: float) -> np.ndarray:
    """Columns of f (grid index first) onto the new grid by distance to the
    nearer wall, in units of the old grid (exact index copies when the
    spacings are equal)."""
    r = dz_new / dz_old
    K = np.arange(np_new, dtype=np.float64)
    mid_old = (np_old - 1) / 2.0
    left = K <= (np_new - 1) / 2.0
    pos = np.where(left, np.minimum(K * r, mid_old), np.maximum((np_old - 1) - (np_new - 1 - K) * r, mid_old))
    i0 = np.clip(np.floor(pos).astype(np.int64), 0, np_old - 1)
    i1 = np.minimum(i0 + 1, np_old - 1)
    w = pos - i0
    flat = f.reshape(f.shape[0], -1)
    out = np.where(w[:, None] == 0.0, flat[i0], flat[i0] * (1.0 - w[:, None]) + flat[i1] * w[:, None])
    return out.reshape((np_new,) + f.shape[1:])


def resample_state(state, old_geometry, new_geometry):
    """(mu_ex_K, lng_K, Psi, PsiC) of a solved slit onto another slit's grid."""
    mu, lng, psi, psic = state
    a = (old_geometry.NP, old_geometry.bin_width, new_geometry.NP, new_geometry.bin_width)
    return (np.asfortranarray(_resample(np.asarray(mu), *a)), np.asfortranarray(_resample(np.asarray(lng), *a)),
            _resample(np.asarray(psi), *a), np.array(psic, dtype=np.float64))


# ---- measurements -------------------------------------------------------------

def slit_measurements(dft: IsingDFT) -> dict:
    """Omega, energy Omega + P_bulk H and the contact-value pressure of a solved slit."""
    H = dft.geometry.dimensions
    omega = grand_potential(dft)
    p_bulk = dft.bulk_system.bulk.pressure
    _, beads, _ = densities(dft)
    cvt = contact_value_theorem_arrays(beads, dft.bulk_system.molsys, dft.geometry)
    return {"distance": H, "NP": dft.NP, "omega": omega, "energy": omega + p_bulk * H, "Pressure": float(cvt[0]),
            "deltaP": float(cvt[0]) - p_bulk}


# ---- adjust_distancesZ --------------------------------------------------------

def _fmt_dir(prefix: str, v: float, digits: int = 2) -> str:
    return prefix + f"{v:0.{digits}f}"


def adjust_distancesZ(data: dict, startZ: float = 1.6, stopZ: float = 20.0, stepZ: float = 0.02, errP: float = 1e-6,
                      out_root: Optional[str] = "dist_sweep", dz: Optional[float] = None, grid: str = "device",
                      max_count: int = 20) -> List[dict]:
    """routines/adjust_distanceZ.jl:15-155 (files under out_root when given)."""
    data = copy.deepcopy(data)
    bulk = iLST(data)  # the bulk state does not depend on the wall separation
    results: List[dict] = []
    distance, count, i = startZ, 0, 0
    prev = None
    if out_root is not None:
        os.makedirs(out_root, exist_ok=True)
    while count < max_count:
        distance += stepZ
        i += 1
        set_distance(data, distance, dz, grid)
        geom = geometry_system(data)
        dft = setup_iDFT(data, bulk, geom)
        step_dir = None
        if out_root is not None:
            step_dir = os.path.join(out_root, _fmt_dir("dist_", distance))
            os.makedirs(step_dir, exist_ok=True)
        if prev is not None:
            dft.state = resample_state(prev[0], prev[1], geom)
        eval_inhomogeneous(dft, step_dir)
        m = slit_measurements(dft)
        delta_E = m["energy"] - results[-1]["energy"] if results else 10.0
        r = {"step": i, **m, "iterations": dft.iterations, "status": dft.status, "residual": dft.residual}
        results.append(r)
        if step_dir is not None:
            with open(os.path.join(step_dir, "run_info.csv"), "w") as fh:
                fh.write("step,distance,Pressure,deltaP,energy\n")
                fh.write(f"{i},{jl(r['distance'])},{jl(r['Pressure'])},{jl(r['deltaP'])},{jl(r['energy'])}\n")
        count = count + 1 if abs(delta_E) < errP else 0
        if distance > stopZ:
            count = max_count + 1
        prev = (dft.state, geom)
        dft.handle().close()
    if out_root is not None:
        final_E, final_dP = results[-1]["energy"], results[-1]["deltaP"]
        with open(os.path.join(out_root, "adjust_distancesZ_results.csv"), "w") as fh:
            fh.write("step,distance,Pressure,deltaP,energy,deltaE\n")
            for r in results:
                fh.write(f"{r['step']},{jl(r['distance'])},{jl(r['Pressure'])},{jl(r['deltaP'] - final_dP)},"
                         f"{jl(r['energy'])},{jl(r['energy'] - final_E)}\n")
    return results


# ---- adjust_pH ----------------------------------------------------------------

def julia_range(start: float, step: float, stop: float) -> List[float]:
    """start:step:stop for floats: the values that do not pass stop."""
    n = math.floor((stop - start) / step * (1 + 1e-12) + 1e-9) + 1
    return [start + k * step for k in range(max(n, 0))]


def read_brush_height(path: str) -> dict:
    """routines/adjust_pH.jl:246-276."""
    vals = {}
    if not os.path.isfile(path):
        return vals
    for ln in open(path):
        s = ln.strip()
        if not s or s.startswith("#"):
            continue
        parts = s.split()
        if len(parts) < 2:
            continue
        try:
            vals[parts[0]] = float(parts[1])
        except ValueError:
            continue
    return vals


def read_avg_state_fraction(path: str, state_index: int = 2) -> Optional[float]:
    """routines/adjust_pH.jl:278-295: the `avg` line's state_index-th entry."""
    alpha = None
    for ln in open(path):
        s = ln.strip()
        if not s.startswith("avg "):
            continue
        parts = s.split()
        if len(parts) >= 1 + state_index and parts[state_index]:
            alpha = float(parts[state_index])
    return alpha


def _set_pH(data: dict, pH: float) -> None:
    for sp in data["species"]:
        if sp.get("sequence") == "Y":
            sp["pSpecies"] = pH
            return


def adjust_pH(data: dict, startZ: float = 3.0, stopZ: float = 10.0, stepZ: float = 0.05,
              out_root: str = "pH_sweep") -> List[dict]:
    """routines/adjust_pH.jl:16-125.  The analysis files of every step are written
    under out_root/pH_<pH> and the brush height and alpha are read back from
    them, as the routine does; alpha is taken from the total_state_fractions
    file of the first species with dissociating segments."""
    data = copy.deepcopy(data)
    root = os.path.abspath(out_root)
    os.makedirs(root, exist_ok=True)
    results: List[dict] = []
    prev = None
    for i, pH in enumerate(julia_range(startZ, stepZ, stopZ), start=1):
        step_dir = os.path.join(out_root, _fmt_dir("pH_", pH))
        os.makedirs(step_dir, exist_ok=True)
        _set_pH(data, pH)
        bulk = iLST(data)
        geom = geometry_system(data)
        dft = setup_iDFT(data, bulk, geom)
        if prev is not None:
            dft.state = prev
        eval_inhomogeneous(dft, step_dir)
        ms = dft.bulk_system.molsys
        hb = read_brush_height(os.path.join(step_dir, "brush_height.txt"))
        if len(hb) > 1:
            raise ValueError("more than one grafted species in brush_height.txt")
        h = next(iter(hb.values())) if hb else float("nan")
        alpha = float("nan")
        for u, cfg in enumerate(ms.configurations):
            if any(len(f) > 1 for f in cfg.state_family):
                a = read_avg_state_fraction(os.path.join(step_dir, f"total_state_fractions_{ms.species[u]}.txt"), 2)
                alpha = float("nan") if a is None else a
                break
        r = {"step": i, "pH": pH, "brush_height": h, "alpha": alpha, "iterations": dft.iterations,
             "status": dft.status, "residual": dft.residual}
        results.append(r)
        summary = os.path.join(root, "summary_brush_alpha.csv")
        header = not os.path.isfile(summary) or os.path.getsize(summary) == 0
        with open(summary, "w" if header else "a") as fh:
            if header:
                fh.write("step,pH,brush_height,alpha\n")
            fh.write("%d,%.12g,%.12g,%.12g\n" % (i, pH, h, alpha))
        with open(os.path.join(step_dir, "run_info.csv"), "w" if i == 1 else "a") as fh:
            if i == 1:
                fh.write("step,pH,brush_height,alpha\n")
            fh.write(f"{i},{jl(pH)},{jl(h)},{jl(alpha)}\n")
        prev = dft.state
        dft.handle().close()
        if alpha >= 0.99 and stepZ > 0:
            break
        if alpha <= 0.01 and stepZ < 0:
            break
    return results


# ---- batched branches -----------------------------------------------------------

def batched_distance_sweep(branches: Sequence[dict], distances: Sequence[float], dz: Optional[float] = None,
                           grid: str = "device", num=None) -> List[List[dict]]:
    """Wall-separation sweep of independent branches (input datasets, one per
    branch, sharing the numerics): at every distance all branches are solved in
    one batched launch, each starting from its own previous solution.  Returns
    per branch the list of per-step measurements."""
    datas = [copy.deepcopy(b) for b in branches]
    bulks = [iLST(d) for d in datas]
    if num is None:
        num = numerics_from_dict(datas[0].get("numerical") or {})
    prev = [None] * len(datas)
    out: List[List[dict]] = [[] for _ in datas]
    for step, H in enumerate(distances, start=1):
        dfts = []
        for b, d in enumerate(datas):
            set_distance(d, H, dz, grid)
            geom = geometry_system(d)
            dft = setup_iDFT(d, bulks[b], geom)
            if prev[b] is not None:
                dft.state = resample_state(prev[b][0], prev[b][1], geom)
            dfts.append(dft)
        iters, errs, status = native.solve_batch([t.handle() for t in dfts], num)
        device_ms, launches, _ = native.last_batch_stats(len(dfts))
        for b, dft in enumerate(dfts):
            dft.iterations, dft.residual, dft.status = int(iters[b]), float(errs[b]), int(status[b])
            m = slit_measurements(dft)
            out[b].append({"step": step, **m, "iterations": int(iters[b]), "status": int(status[b]),
                           "residual": float(errs[b]), "batch_device_ms": device_ms})
            prev[b] = (dft.state, dft.geometry)
            dft.handle().close()
    return out


# ---- pseudo-arclength continuation in pH or graft density -------------------------
#
# Restates src/NonlinearSolvers/continuation/objective_pac.jl:41-289 (and its
# graft-density twin objective_pac_graft.jl, continuation variable ln(density)) on the
# unknowns the solver uses today, X = (mu_ex_K, lng_K, Psi, PsiC, pH) (the
# reference file flattens the segment densities, bond densities and PsiC, which
# the current solver_dft no longer iterates on).  As there:
#   * two natural steps start the branch (pH0, then pH0 + ds_init);
#   * the tangent is the normalised secant of the last two points, or the
#     three-point backward difference in arclength once three exist (:128-146);
#   * the predictor is X_k + dS t (:150-152);
#   * the corrected point satisfies G(x) = x and the hyperplane constraint
#     t . (X - X_k) = dS (objective_pac, :253-289);
#   * the arclength grows by |X - X_prev| and dS <- (dS + |X - X_prev|) / 2 (:164-172);
#   * the sweep stops outside pH (1.99, 12.01) or when alpha passes 0.99 going up
#     or 0.01 going down (:233-241).
# Differences: the reference folds the constraint into every Anderson step
# (pH <- pH_k + (dS - t_x . (G(x) - x_k)) / t_pH) and rebuilds the whole system
# per evaluation; here pH enters through the bulk state and the descriptor, so
# the corrector is a secant iteration on pH whose every evaluation is a
# warm-started device solve of x(pH) (the first update is the reference's
# formula).  The constraint uses the current dS (the reference freezes ds_init
# into it), and the alpha stop looks at the direction of pH along the tangent
# (the reference tests sign(dS), which is always positive).

def _pac_tangent(X_hist: Sequence[np.ndarray], S_hist: Sequence[float]) -> np.ndarray:
    """Unit tangent of the branch at its last point (objective_pac.jl:128-148)."""
    if len(X_hist) < 3:
        t = X_hist[-1] - X_hist[-2]
    else:
        ds1 = S_hist[-1] - S_hist[-2]
        ds2 = S_hist[-2] - S_hist[-3]
        a = ds1 / (ds2 * (ds1 + ds2))
        b = -(ds1 + ds2) / (ds1 * ds2)
        c = (2.0 * ds1 + ds2) / (ds1 * (ds1 + ds2))
        t = a * X_hist[-3] + b * X_hist[-2] + c * X_hist[-1]
    return t / np.linalg.norm(t)


def _branch_pH(data: dict) -> float:
    for sp in data["species"]:
        if sp.get("sequence") == "Y":
            return float(sp["pSpecies"])
    raise ValueError("pH continuation needs the proton species Y with a pSpecies")


def _alpha(dft: IsingDFT) -> float:
    """Average fraction of state 2 over the dissociating segments of the first
    species that has them (the routine's read_avg_state_fraction)."""
    for v in state_fractions(dft).values():
        a = v["avg"]
        return float(a[1]) if len(a) > 1 else float("nan")
    return float("nan")


def _set_log_graft(data: dict, v: float) -> None:
    """update_cont_var_graft (objective_pac_graft.jl:286-287): the first species'
    graft density is e^v."""
    data["species"][0]["fixed"]["density"] = math.exp(v)


def _log_graft(data: dict) -> float:
    return math.log(data["species"][0]["fixed"]["density"])


def _solve_points(datas, pHs, x0s, num, setter=_set_pH):
    """One batched device solve: branch b at parameter pHs[b] (set by `setter`),
    warm-started from x0s[b] (None: the reference's initial guess).  Returns the
    solved systems."""
    dfts = []
    for d, pH, x0 in zip(datas, pHs, x0s):
        setter(d, pH)
        dft = setup_iDFT(d, iLST(d), geometry_system(d))
        if x0 is not None:
            dft.handle().set_x(x0)
        dfts.append(dft)
    iters, errs, status = native.solve_batch([t.handle() for t in dfts], num)
    for b, dft in enumerate(dfts):
        dft.iterations, dft.residual, dft.status = int(iters[b]), float(errs[b]), int(status[b])
    return dfts


def pac_pH_branches(branches: Sequence[dict], ds_init: float = 0.05, max_steps: int = 200, num=None,
                    pH_range=(1.99, 12.01), corrector_tol: float = 1e-6, max_corrector: int = 10,
                    out_root: Optional[str] = None) -> List[List[dict]]:
    """Pseudo-arclength continuation in pH of independent branches (one input
    dataset each); every solve of a step is one batched launch over the branches
    still running.  Returns per branch the list of per-point records (pH, alpha,
    brush height, Omega, arclength, step length, corrector iterations).  With
    out_root, each point's analysis files go to out_root/b<branch>/pH_<pH>."""
    return _pac_branches(branches, "pH", ds_init, max_steps, num, pH_range, corrector_tol, max_corrector, out_root)


def pac_graft_branches(branches: Sequence[dict], ds_init: float = 0.05, max_steps: int = 200, num=None,
                       log_range=(-math.inf, 1.0), corrector_tol: float = 1e-6, max_corrector: int = 10,
                       out_root: Optional[str] = None) -> List[List[dict]]:
    """Pseudo-arclength continuation in the log of the first species' graft
    density (pac_continuation_graft, objective_pac_graft.jl:36-284): the same
    scheme with v = ln(density) as the continuation variable, run while v < 1,
    without the alpha stop; records carry graft_density = e^v, and the analysis
    files go to out_root/b<branch>/graft_<density>."""
    return _pac_branches(branches, "graft", ds_init, max_steps, num, log_range, corrector_tol, max_corrector,
                         out_root)


def _pac_branches(branches, kind, ds_init, max_steps, num, pH_range, corrector_tol, max_corrector, out_root):
    getter, setter = (_branch_pH, _set_pH) if kind == "pH" else (_log_graft, _set_log_graft)
    datas = [copy.deepcopy(b) for b in branches]
    if num is None:
        num = numerics_from_dict(datas[0].get("numerical") or {})
    nb = len(datas)
    out: List[List[dict]] = [[] for _ in datas]
    X_hist: List[List[np.ndarray]] = [[] for _ in datas]
    S_hist: List[List[float]] = [[] for _ in datas]
    dS = [float(ds_init)] * nb
    s = [0.0] * nb
    active = [True] * nb

    def record(b, dft, pH, step, corr, used_ds):
        x = dft.handle().get_x()
        X = np.concatenate([x, [pH]])
        rec = {"step": step, "alpha": _alpha(dft), "omega": grand_potential(dft),
               "iterations": dft.iterations, "status": dft.status, "residual": dft.residual,
               "corrector_iterations": corr, "dS": used_ds}
        hb = brush_height_values(densities(dft)[0], dft.bulk_system.molsys, dft.geometry, dft.descriptor.fixed_coord)
        rec["brush_height"] = next(iter(hb.values())) if hb else float("nan")
        if X_hist[b]:
            ds_actual = float(np.linalg.norm(X - X_hist[b][-1]))
            s[b] += ds_actual
            rec["ds_actual"] = ds_actual
        rec["arclength"] = s[b]
        if kind == "pH":
            rec["pH"] = pH
        else:
            rec["log_graft_density"] = pH
            rec["graft_density"] = math.exp(pH)
        X_hist[b] = (X_hist[b] + [X])[-3:]
        S_hist[b] = (S_hist[b] + [s[b]])[-3:]
        if out_root is not None:
            d = os.path.join(out_root, f"b{b}", _fmt_dir("pH_", pH, 3) if kind == "pH"
                             else _fmt_dir("graft_", math.exp(pH), 7))
            os.makedirs(d, exist_ok=True)
            call_analysis(dft, d)
        out[b].append(rec)
        return rec

    def ok(dft):
        return dft.status in (native.SDFT_OK, native.SDFT_MAX_ITERS)

    # two natural steps start every branch (objective_pac.jl:59-113)
    pH0 = [getter(d) for d in datas]
    dfts = _solve_points(datas, pH0, [None] * nb, num, setter)
    for b, dft in enumerate(dfts):
        record(b, dft, pH0[b], 1, 0, 0.0)
        active[b] = ok(dft)
    x1 = [dft.handle().get_x() for dft in dfts]
    for dft in dfts:
        dft.handle().close()
    idx = [b for b in range(nb) if active[b]]
    dfts = _solve_points([datas[b] for b in idx], [pH0[b] + dS[b] for b in idx], [x1[b] for b in idx], num, setter)
    for b, dft in zip(idx, dfts):
        record(b, dft, pH0[b] + dS[b], 2, 0, dS[b])
        active[b] = ok(dft)
        dft.handle().close()

    for step in range(3, max_steps + 1):
        idx = [b for b in range(nb) if active[b] and pH_range[0] < X_hist[b][-1][-1] < pH_range[1]]
        if not idx:
            break
        tang = {b: _pac_tangent(X_hist[b], S_hist[b]) for b in idx}
        Xk = {b: X_hist[b][-1] for b in idx}
        used = {b: dS[b] for b in idx}
        # corrector: secant on f(pH) = t . (X(pH) - X_k) - dS with X(pH) = (x(pH), pH)
        lam = {b: Xk[b][-1] + used[b] * tang[b][-1] for b in idx}
        xstart = {b: (Xk[b] + used[b] * tang[b])[:-1] for b in idx}
        hist = {b: [] for b in idx}  # (pH, f)
        done: dict = {}
        todo = list(idx)
        for it in range(max_corrector):
            if not todo:
                break
            dfts = _solve_points([datas[b] for b in todo], [lam[b] for b in todo], [xstart[b] for b in todo], num,
                                 setter)
            nxt = []
            for b, dft in zip(todo, dfts):
                t = tang[b]
                x = dft.handle().get_x()
                f = float(np.dot(t[:-1], x - Xk[b][:-1]) + t[-1] * (lam[b] - Xk[b][-1]) - used[b])
                hist[b].append((lam[b], f))
                last = it == max_corrector - 1
                if not ok(dft) or abs(f) <= corrector_tol * used[b] or last:
                    done[b] = (dft, it + 1, ok(dft) and abs(f) <= corrector_tol * used[b], f)
                    continue
                # a pH turning point has t_pH = 0: the constraint cannot move pH
                # there, so the branch's corrector stops as failed
                flat = abs(t[-1]) <= 1e-12 * max(float(np.max(np.abs(t))), 1e-300)
                if len(hist[b]) == 1:
                    # the reference's constraint update: pH = pH_k + (dS - t_x . (x - x_k)) / t_pH
                    new_lam = lam[b] - f / t[-1] if not flat else float("nan")
                else:
                    (l0, f0), (l1, f1) = hist[b][-2], hist[b][-1]
                    if f1 != f0:
                        new_lam = l1 - f1 * (l1 - l0) / (f1 - f0)
                    else:
                        new_lam = l1 - f1 / t[-1] if not flat else float("nan")
                if not np.isfinite(new_lam):
                    done[b] = (dft, it + 1, False, f)
                    continue
                lam[b] = new_lam
                xstart[b] = x
                dft.handle().close()
                nxt.append(b)
            todo = nxt
        for b in idx:
            dft, corr, converged, f = done[b]
            rec = record(b, dft, lam[b], step, corr, used[b])
            rec["corrector_converged"] = converged
            rec["constraint_residual"] = f  # t . (X - X_k) - dS at the accepted point
            dft.handle().close()
            if not ok(dft):
                active[b] = False
                continue
            dS[b] = (dS[b] + rec["ds_actual"]) / 2.0
            going_up = tang[b][-1] > 0
            if kind == "pH" and ((rec["alpha"] >= 0.99 and going_up) or (rec["alpha"] <= 0.01 and not going_up)):
                active[b] = False
    return out
