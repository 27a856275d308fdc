"""Scalar (per-run) chemistry constants computed on the host: the ion-energy-distribution
integrated yields (petch/chemistry.py:10-42).  The per-face chemistry itself runs on the device
(petch_belen_bare / petch_surface_rate)."""
import numpy as np


def _ied_yield(A, Eth, par):
    """Y = A * max(sqrt(E) - sqrt(Eth), 0) averaged over the ion energy distribution
    (par['ied_mode']: 'mean' | 'gauss' (25-point N(Emean, Esig) quadrature) | 'bimodal'
    (49-point arcsine of full width ied_dE)), as chemistry._ied_yield."""
    mode = par.get('ied_mode', 'mean')
    Em = float(par['Emean'])
    sEth = np.sqrt(max(Eth, 0.0))
    if mode == 'mean':
        return float(A * max(np.sqrt(max(Em, 0.0)) - sEth, 0.0))
    if mode == 'gauss':
        Es = float(par.get('Esig', 10.0))
        z = np.linspace(-3.5, 3.5, 25)
        w = np.exp(-0.5 * z * z)
        w /= w.sum()
        E = np.clip(Em + Es * z, 0.0, None)
        return float((w * A * np.maximum(np.sqrt(E) - sEth, 0.0)).sum())
    dE = float(par.get('ied_dE', 40.0))
    ph = np.linspace(0.0, np.pi, 49)
    E = np.clip(Em + 0.5 * dE * np.cos(ph), 0.0, None)
    return float(np.mean(A * np.maximum(np.sqrt(E) - sEth, 0.0)))


def _yields(par):
    """(Yie, Ysp, Yp) as chemistry._yields."""
    return (_ied_yield(par['A_ie'], par['Eth_ie'], par),
            _ied_yield(par['A_sp'], par['Eth_sp'], par),
            _ied_yield(par['A_p'], par['Eth_p'], par))
