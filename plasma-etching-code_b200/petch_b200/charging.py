"""Floor-charging hooks on the device's per-face ion results (drop-ins for the reference's
_apply_hg_charging, petch/threed.py:1046-1110, and _apply_floor_charge_throttle, :1112-1147, with
the aspect-ratio tables of petch/charging2d.py and petch/charging_general.py).

An insulating (or passivated) floor charges up: part of the ion flux never lands on it.  The
tables give, against the feature's aspect ratio, the surviving floor fraction Q, the floor
potential V_f and the mean energy E_defl of the ions deflected onto the sidewall foot.  The device
reduces the mesh to four numbers (floor count, deepest floor face, the floor's m_i A, the foot's
area); the host interpolates the tables and evaluates the yields as the reference's host code does;
one kernel applies the result to every face.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .chemistry import _yields

# Hwang-Giapis published floor-charging values (JAP 82, 566), as tabulated by the reference
# (charging2d.py:1511-1518): aspect ratio -> floor flux fraction, floor potential (V), foot energy.
HG_AR = np.array([0.0, 1.0, 1.2, 1.6, 2.0, 2.6, 3.0, 3.6, 4.0])
HG_Q = np.array([1.0, 0.59, 0.55, 0.47, 0.40, 0.34, 0.30, 0.26, 0.22])
HG_VFLOOR = np.array([0.0, 8.0, 10.0, 15.0, 19.0, 25.0, 28.0, 31.0, 33.0])
HG_FOOT_E = np.array([0.0, 15.0, 16.5, 17.5, 20.0, 23.0, 25.0, 26.5, 27.5])
# petch's own first-principles charging table (charging_general.py:1038-1041)
PETCH_AR = np.array([1.0, 2.0, 3.0, 4.0])
PETCH_Q = np.array([0.704, 0.491, 0.406, 0.349])
PETCH_VFLOOR = np.array([9.5, 19.2, 27.7, 34.0])
PETCH_FOOT_E = np.array([16.6, 14.2, 18.8, 21.6])
# the de Boer deep-AR floor throttle (charging_general.py:1070-1071)
THROTTLE_AR = np.array([0.0, 1.0, 2.0, 3.0, 4.0, 8.0, 15.0, 25.0])
THROTTLE_Q = np.array([1.0, 0.704, 0.491, 0.406, 0.349, 0.25, 0.60, 0.50])


def charging_floor_profile(AR):
    """charging2d.charging_floor_profile: (Q, V_f, E_defl) of the Hwang-Giapis table."""
    AR = np.asarray(AR, float)
    return (np.interp(AR, HG_AR, HG_Q), np.interp(AR, HG_AR, HG_VFLOOR),
            np.interp(AR, HG_AR, HG_FOOT_E))


def petch_floor_profile(AR):
    """charging_general.petch_floor_profile: (Q, V_f, E_defl) of petch's own table."""
    AR = np.asarray(AR, float)
    return (np.interp(AR, PETCH_AR, PETCH_Q), np.interp(AR, PETCH_AR, PETCH_VFLOOR),
            np.interp(AR, PETCH_AR, PETCH_FOOT_E))


def floor_charge_throttle_profile(AR):
    """charging_general.floor_charge_throttle_profile: Q(AR) in [0, 1], 1 below the table,
    its last value above it."""
    AR = np.asarray(AR, float)
    return np.clip(np.interp(AR, THROTTLE_AR, THROTTLE_Q, left=1.0,
                             right=float(THROTTLE_Q[-1])), 0.0, 1.0)


def _classes(geo):
    hole = bool(geo.get('hole', False))
    band = 0.5 * float(geo['trench_width']) + 2.0 * float(geo['dx'])
    return (0.5 * float(geo['Lx']), 0.5 * float(geo['Ly']), band, int(hole),
            float(geo['sub_top']))


def _stats(fe, normals, foot_h):
    m = fe.mesh
    cx, cy, band, hole, sub_top = _classes(fe.geo)
    st = torch.empty(5, dtype=torch.float64, device="cuda")
    _lib.call("petch_charging_floor_stats", m.id, m.MT, m.centroid.data_ptr(),
              normals.data_ptr(), m.area.data_ptr(), fe.m_i.data_ptr(), cx, cy, band, hole,
              sub_top, float(foot_h), st.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return st.cpu().numpy()


def _apply(fe, normals, q4, add3, z_foot, yields_present):
    m = fe.mesh
    cx, cy, band, hole, sub_top = _classes(fe.geo)
    q = (ctypes.c_double * 4)(*[float(v) for v in q4])
    a = (ctypes.c_double * 3)(*[float(v) for v in add3])
    y = [fe.y[k].data_ptr() for k in range(3)] if yields_present else [None, None, None]
    _lib.call("petch_charging_apply", m.id, m.MT, m.centroid.data_ptr(), normals.data_ptr(), cx,
              cy, band, hole, sub_top, q, a, float(z_foot), fe.m_i.data_ptr(), y[0], y[1], y[2],
              torch.cuda.current_stream().cuda_stream)


def apply_hg_charging(fe, normals, mode):
    """_apply_hg_charging on a FluxEngine's device results (m_i and the yields y[0..2] =
    sputter, ion-enhanced, passivation), for flags.surface_charging in ("hg", "petch") on the
    faithful-ion path; normals are the into-gas normals of the mesh.  Returns the floor
    statistics used (or None when nothing applied)."""
    if mode not in ("hg", "petch") or fe.yields[0] is None:
        return None
    par, geo = fe.par, fe.geo
    W = float(geo['trench_width'])
    foot_h = max(0.3 * W, 2.0 * float(geo['dx']))
    n_floor, zmin, mA, n_foot, foot_area = _stats(fe, normals, foot_h)
    if n_floor == 0:
        return None
    AR = float(geo['sub_top'] - zmin) / max(W, 1e-9)
    prof = charging_floor_profile if mode == "hg" else petch_floor_profile
    Q, Vf, E_defl = (float(v) for v in prof(AR))
    y0 = _yields(par)
    yv = _yields(dict(par, Emean=max(par['Emean'] - Vf, 0.0)))
    r_ie = yv[0] / y0[0] if y0[0] > 0 else 0.0
    r_sp = yv[1] / y0[1] if y0[1] > 0 else 0.0
    r_p = yv[2] / y0[2] if y0[2] > 0 else 0.0
    defl_total = mA * (1.0 - Q)
    add = (0.0, 0.0, 0.0)
    if n_foot > 0 and defl_total > 0.0:
        fdefl = defl_total / max(foot_area, 1e-12)
        sE = np.sqrt(E_defl)
        add = (fdefl * par['A_sp'] * max(sE - np.sqrt(par['Eth_sp']), 0.0),
               fdefl * par['A_ie'] * max(sE - np.sqrt(par['Eth_ie']), 0.0),
               fdefl * par['A_p'] * max(sE - np.sqrt(par['Eth_p']), 0.0))
    _apply(fe, normals, (Q, Q * r_sp, Q * r_ie, Q * r_p), add, zmin + foot_h, True)
    return dict(AR=AR, Q=Q, Vf=Vf, E_defl=E_defl, n_floor=int(n_floor), z_floor=zmin)


def apply_floor_throttle(fe, normals):
    """_apply_floor_charge_throttle on a FluxEngine's device results: the floor faces' m_i (and
    yields, when present) times Q(AR).  The reference takes the float32 centroid means, so its
    depth sub_top - z_min is float32 arithmetic; so is this one."""
    geo = fe.geo
    n_floor, zmin, _, _, _ = _stats(fe, normals, 0.0)
    if n_floor == 0:
        return None
    depth = float(np.float32(geo['sub_top']) - np.float32(zmin))
    AR = depth / max(float(geo['trench_width']), 1e-9)
    Q = float(floor_charge_throttle_profile(AR))
    present = fe.yields[0] is not None
    _apply(fe, normals, (Q, Q, Q, Q), (0.0, 0.0, 0.0), -np.inf, present)
    return dict(AR=AR, Q=Q, n_floor=int(n_floor), z_floor=zmin)


def open_field_level(x):
    """np.percentile(x[x > 1e-6], 90) in float64, 1.0 when no face is above 1e-6: the open-field
    reference level of a flux (threed.py:862-863)."""
    x = np.asarray(x, np.float64)
    live = x[x > 1e-6]
    return float(np.percentile(live, 90)) if live.size else 1.0


def apply_electron_shadow(fe, n_neu, seed):
    """The surface-charging block of mc_flux_3d_coupled (threed.py:847-868) on a FluxEngine's
    device results, for flags.surface_charging truthy and charge_alpha > 0: n_neu electrons from
    the Gaussian-angle source (e_ang_sigma) land with unit sticking; m_e = their normalised
    arrival (times eFlux, clipped at 8, smoothed like the other fluxes); the host takes the two
    open-field levels from one read of m_i and m_e; one kernel multiplies m_i by the charging
    factor.  The yields are left as they are, as in the reference.  Returns the levels used."""
    par, geo, m = fe.par, fe.geo, fe.mesh
    s = torch.cuda.current_stream().cuda_stream
    if getattr(fe, "m_e", None) is None or fe.m_e.numel() != fe.MT:
        fe.m_e = torch.empty(fe.MT, device="cuda", dtype=torch.float32)
    A_src = float(geo['Lx'] * geo['Ly'])
    n_smooth = int(par.get('flux_smooth', 1))
    sm_alpha = float(par.get('flux_smooth_alpha', 1.0))
    work = fe.small[0:6]
    _lib.call("petch_trace_electrons", m.id, m.MT, m.MV, ctypes.byref(fe.dom),
              float(par.get('e_ang_sigma', 0.5)), int(seed * 9 + 7) & 0xffffffff, int(n_neu),
              fe.flux.data_ptr(), work.data_ptr(), s)
    _lib.call("petch_norm_smooth", m.id, m.MT, m.MV, fe.flux.data_ptr(),
              float(A_src / n_neu * float(par.get('eFlux', 1.0))), 0.0, 8.0, 1, n_smooth,
              sm_alpha, fe.m_e.data_ptr(), fe.tmp5.data_ptr(), fe.tmp5[m.MT:].data_ptr(), s)
    F = m.n_faces()
    ref_i = open_field_level(fe.m_i[:F].cpu().numpy())
    ref_e = open_field_level(fe.m_e[:F].cpu().numpy())
    alpha = float(par.get('charge_alpha', 0.0))
    _lib.call("petch_electron_shadow", m.id, m.MT, fe.m_e.data_ptr(), ref_i, ref_e, alpha,
              fe.m_i.data_ptr(), s)
    return dict(ref_i=ref_i, ref_e=ref_e, alpha=alpha)
